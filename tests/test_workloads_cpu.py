"""Host-side logic of the full-size workload table: the seeded disk image the
Rician and TV workloads start from, and the learned pick (best measured of
the model's top 10 %) taken from a measured space."""
import numpy as np
import pytest

import ots
from ots import workloads as W


def test_disk_image_is_seeded_and_shaped():
    c1, f1 = W.disk_image(256, seed=5)
    c2, f2 = W.disk_image(256, seed=5)
    c3, _ = W.disk_image(256, seed=6)
    assert c1.shape == f1.shape == (256, 256)
    assert c1.dtype == f1.dtype == np.float32
    assert np.array_equal(c1, c2) and np.array_equal(f1, f2)
    assert not np.array_equal(c1, c3)
    # constant-intensity disks on a 0.1 background
    assert c1.min() == pytest.approx(0.1)
    assert c1.max() <= 1.0
    vals = np.unique(c1)
    assert 2 <= len(vals) <= 65
    assert 0.05 < float(np.mean(c1 > 0.1)) < 0.95
    # Rician noise: f = |s + n1 + i n2| is positive and biased upwards
    assert np.all(np.isfinite(f1)) and np.all(f1 >= 0)
    assert 0.0 < float(np.mean(f1 - c1)) < 0.02
    assert float(np.std(f1 - c1)) == pytest.approx(0.05, rel=0.2)


class _Ranker:
    """Stands in for the cost model: ranks by a fixed score per record."""

    def __init__(self, scores):
        self.scores = np.asarray(scores)

    def topk(self, X, k):
        assert X.shape[0] == len(self.scores)
        return list(np.argsort(-self.scores)[:k])


def _rec(T, g, kernel="tile"):
    geom = ots.derive_geometry(stencil="jacobi-2d", n=256, steps=8, T=T, bx=32, by=8, E=1,
                               kernel=kernel)
    return dict(stencil="jacobi-2d", kernel=kernel, T=T, bx=32, by=8, bz=1, E=1,
                status="ok", gupdates=g, geom=geom.as_dict())


def test_picks_keep_best_measured_of_top_k():
    recs = [_rec(T, g) for T, g in zip(range(1, 9), (10, 20, 30, 80, 50, 60, 70, 40))]
    recs += [_rec(T, 1.0) for T in range(1, 9)] + [_rec(1, 2.0) for _ in range(4)]
    recs.append(dict(stencil="jacobi-2d", kernel="tile", T=9, bx=32, by=8, bz=1, E=1,
                     status="OTS_ERR_GEOMETRY"))
    ok = [r for r in recs if r["status"] == "ok"]
    # the model likes records 5 and 6 best (60, 70), then 3 (80)
    scores = np.zeros(len(ok))
    scores[5], scores[6], scores[3] = 3.0, 2.0, 1.0
    p = W.picks("jacobi-2d", recs, _Ranker(scores))
    assert p["space"] == 20 and p["k"] == 2 and p["measured"] == 2
    assert p["top1"]["gupdates"] == 60
    assert p["picked"]["gupdates"] == 70  # best measured of the top 2, not the top-1
    assert W.config_of(p["picked"]) == dict(kernel="tile", T=7, bx=32, by=8, bz=1, E=1)
    # the plain one-step kernel is not ranked but always measured beside the picks
    slow = dict(recs[0], kernel="plain", gupdates=65.0)
    fast = dict(recs[0], kernel="plain", gupdates=95.0)
    for pl, want in ((slow, 65), (fast, 95)):
        # 10 % of 21 is 2 runs: the plain run and the model's top 1
        p = W.picks("jacobi-2d", recs + [pl], _Ranker(scores))
        assert p["space"] == 21 and p["k"] == 1 and p["measured"] == 2
        assert p["picked"]["gupdates"] == want


def test_workload_table_names_every_configured_stencil():
    base = [w for w in W.WORKLOADS if "variant" not in w]
    names = [w["stencil"] for w in base if not w.get("extra")]
    assert names == ["jacobi-2d", "jacobi-3d", "poisson-3d", "fdtd-2d", "rician-denoise-2d",
                     "cdsc-tv-update-2d"]
    assert sorted(w["stencil"] for w in base) == sorted(ots.STENCILS)
    # the fast-division rows: the three stencils that divide, each key unique
    fast = [w for w in W.WORKLOADS if w.get("variant") == "fast"]
    assert sorted(w["stencil"] for w in fast) == ["cdsc-tv-update-2d", "cs-3d",
                                                  "rician-denoise-2d"]
    keys = [W.workload_key(w) for w in W.WORKLOADS]
    assert len(set(keys)) == len(keys) and "rician-denoise-2d-fast" in keys
    assert W.variant_kw(fast[0]) == {"variant": ots.VARIANT_FAST} and W.variant_kw(base[0]) == {}
    assert all(w["stencil"] in W.BYTES_PER_UPDATE for w in W.WORKLOADS)
    assert set(W.HELD_OUT) == {w["stencil"] for w in W.WORKLOADS if w.get("held_out")}
