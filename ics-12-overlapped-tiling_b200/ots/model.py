"""Learned tile-configuration picker.

The reference ranks overlapped-tiling configurations with a Weka k-NN model
(scripts/run-weka.py:49-150) over features from scripts/extract-features.py
(:40-57 names, :108-127 derived ratios) and reports, per held-out benchmark,
``actual(pick) / best actual`` (scripts/parse-weka-results.py:19-37).  Here:

  * ``features()`` builds one vector per configuration from the geometry the
    library derives (no run needed): the reference's block sizes, time tile,
    elements per thread, per-block global/shared traffic, arithmetic
    intensity, block counts and array count, plus stencil radius,
    flops/point, arrays read/written, shared bytes per block, redundant
    compute, registers and occupancy;
  * ``MLP`` is the cost model, trained and evaluated on the GPU by the
    library's own CUDA kernels (ots_mlp_*), regressing log GUpdates/s;
  * ``leave_one_out()`` repeats the reference's protocol: train on every
    other stencil, rank the held-out stencil's space, measure only the top
    k (k = 10 % of the space) and keep the best measured -- the picker's
    cost is k runs instead of the exhaustive sweep's N.
"""
import ctypes
import json
import math

import numpy as np

from . import Geometry, OtsError, STENCILS, check, derive_geometry, lib

# stencil -> (flops/point, arrays read, arrays written) of the arithmetic the
# measured sweeps run (the baseline variant); flops are the reference's
# "Actual GFlop/s" constants (e.g. opencl/jacobi-2d/jacobi-2d.cpp:1001) except
# for the two Poisson stencils, whose constants (9, 27) count the reference's
# 9- and 27-point operators: their baseline 5- and 7-point updates with the
# right-hand side, (sum - h^2 f) / 2d, take 6 and 8 operations.
STENCIL_COST = {
    "jacobi-1d": (3, 1, 1), "jacobi-1d-5pt": (5, 1, 1), "jacobi-1d-7pt": (7, 1, 1),
    "jacobi-2d": (5, 1, 1), "jacobi-3d": (7, 1, 1), "poisson-2d": (6, 2, 1),
    "poisson-3d": (8, 2, 1), "gradient-2d": (15, 1, 1), "gradient-3d": (20, 1, 1),
    "fdtd-2d": (11, 3, 3), "rician-denoise-2d": (42, 2, 1), "cdsc-tv-update-2d": (59, 3, 1),
    "cs-3d": (65, 1, 1),
}

FEATURES = [
    "dims", "radius", "log_flops_pt", "arrays_read", "arrays_written", "T", "log2_bx",
    "log2_by", "log2_bz", "E", "is_stream", "log2_threads", "smem_kb", "useful_ratio",
    "redundancy", "ctas_per_sm", "occupancy", "registers", "log2_points", "bytes_per_update",
    "flops_per_byte", "log2_ctas", "waves", "T_times_flops", "global_ld_block_log2",
    "shared_over_global",
]


def features(stencil, cfg, geom):
    """Feature vector of one configuration.  `cfg` has T, bx, by, bz, E,
    kernel; `geom` is an ots Geometry or a dict with the same fields."""
    g = geom.as_dict() if hasattr(geom, "as_dict") else geom
    flops, ar, aw = STENCIL_COST[stencil]
    T = float(cfg["T"])
    thr = max(1, g["threads"][0] * g["threads"][1] * g["threads"][2])
    ctas = max(1, g["num_blocks"][0] * g["num_blocks"][1] * g["num_blocks"][2])
    cps = max(1, g.get("ctas_per_sm", 1) or 1)
    sms = max(1, g.get("sm_count", 148) or 148)
    ur = max(1e-3, g["useful_ratio"])
    bpu = 4.0 * (ar + aw) / T
    cells = max(1, g["comps"][0] * g["comps"][1] * g["comps"][2])
    gld = cells * ar
    sld = cells * ar * max(0.0, T - 1)
    v = [
        g["dims"], g["radius"], math.log(flops), ar, aw, T, math.log2(cfg["bx"]),
        math.log2(max(1, cfg.get("by", 1))), math.log2(max(1, cfg.get("bz", 1))), cfg["E"],
        1.0 if cfg.get("kernel") == "stream" else 0.0, math.log2(thr),
        g["shared_bytes"] / 1024.0, ur, 1.0 / ur, cps, min(1.0, cps * thr / 2048.0),
        g["registers"], math.log2(max(1, g["interior_points"])), bpu, flops / bpu,
        math.log2(ctas), ctas / float(sms * cps), T * flops, math.log2(max(1, gld)),
        sld / float(max(1, gld)),
    ]
    return np.asarray(v, np.float32)


class MLP:
    """The cost model (ots_mlp_* in libots)."""

    def __init__(self, n_in, hidden=64, layers=3, seed=0, device=0):
        L = _mlp_lib()
        h = ctypes.c_void_p()
        check(L.ots_mlp_create(n_in, hidden, layers, seed, device, ctypes.byref(h)))
        self.h, self.n_in, self.hidden, self.layers = h, n_in, hidden, layers
        self.norm = None

    def close(self):
        if getattr(self, "h", None):
            _mlp_lib().ots_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def num_params(self):
        n = ctypes.c_int64()
        check(_mlp_lib().ots_mlp_num_params(self.h, ctypes.byref(n)))
        return n.value

    def params(self):
        p = np.zeros(self.num_params(), np.float32)
        check(_mlp_lib().ots_mlp_get_params(self.h, _f(p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.num_params()
        check(_mlp_lib().ots_mlp_set_params(self.h, _f(p)))

    def set_normalization(self, mean, inv_std, y_mean, y_std):
        mean = np.ascontiguousarray(mean, np.float32)
        inv_std = np.ascontiguousarray(inv_std, np.float32)
        check(_mlp_lib().ots_mlp_set_normalization(self.h, _f(mean), _f(inv_std),
                                                   float(y_mean), float(y_std)))
        self.norm = (mean, inv_std, float(y_mean), float(y_std))

    def fit_normalization(self, X, y):
        mean = X.mean(axis=0)
        std = X.std(axis=0)
        inv = np.where(std > 1e-8, 1.0 / np.maximum(std, 1e-8), 0.0)
        self.set_normalization(mean, inv, float(y.mean()), float(max(y.std(), 1e-6)))

    def loss_grad(self, X, y):
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        loss = ctypes.c_float()
        g = np.zeros(self.num_params(), np.float32)
        check(_mlp_lib().ots_mlp_loss_grad(self.h, _f(X), _f(y), len(y), ctypes.byref(loss), _f(g)))
        return loss.value, g

    def fit(self, X, y, epochs=300, batch=128, lr=3e-3, weight_decay=1e-4, seed=0):
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        if self.norm is None:
            self.fit_normalization(X, y)
        loss = ctypes.c_float()
        check(_mlp_lib().ots_mlp_train(self.h, _f(X), _f(y), len(y), epochs, batch, lr,
                                       weight_decay, seed, ctypes.byref(loss)))
        return loss.value

    def predict(self, X):
        X = np.ascontiguousarray(X, np.float32)
        out = np.zeros(len(X), np.float32)
        check(_mlp_lib().ots_mlp_predict(self.h, _f(X), len(X), _f(out)))
        return out

    def topk(self, X, k):
        X = np.ascontiguousarray(X, np.float32)
        idx = np.zeros(k, np.int32)
        check(_mlp_lib().ots_mlp_topk(self.h, _f(X), len(X), k,
                                      idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        return idx

    def to_json(self):
        mean, inv, ym, ys = self.norm
        return {"n_in": self.n_in, "hidden": self.hidden, "layers": self.layers,
                "mean": mean.tolist(), "inv_std": inv.tolist(), "y_mean": ym, "y_std": ys,
                "params": self.params().tolist(), "features": FEATURES}

    @classmethod
    def from_json(cls, d, device=0):
        m = cls(d["n_in"], d["hidden"], d["layers"], device=device)
        m.set_normalization(np.array(d["mean"]), np.array(d["inv_std"]), d["y_mean"], d["y_std"])
        m.set_params(np.array(d["params"], np.float32))
        return m


_F = ctypes.POINTER(ctypes.c_float)


def _f(a):
    return a.ctypes.data_as(_F)


def _mlp_lib():
    L = lib()
    if not getattr(L, "_mlp_ready", False):
        st = ctypes.c_int
        vp = ctypes.c_void_p
        L.ots_mlp_create.argtypes = [ctypes.c_int32] * 3 + [ctypes.c_uint64, ctypes.c_int32,
                                                            ctypes.POINTER(vp)]
        L.ots_mlp_create.restype = st
        L.ots_mlp_destroy.argtypes = [vp]
        L.ots_mlp_destroy.restype = None
        L.ots_mlp_num_params.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.ots_mlp_num_params.restype = st
        L.ots_mlp_get_params.argtypes = [vp, _F]
        L.ots_mlp_get_params.restype = st
        L.ots_mlp_set_params.argtypes = [vp, _F]
        L.ots_mlp_set_params.restype = st
        L.ots_mlp_set_normalization.argtypes = [vp, _F, _F, ctypes.c_float, ctypes.c_float]
        L.ots_mlp_set_normalization.restype = st
        L.ots_mlp_loss_grad.argtypes = [vp, _F, _F, ctypes.c_int32, _F, _F]
        L.ots_mlp_loss_grad.restype = st
        L.ots_mlp_train.argtypes = [vp, _F, _F, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                    ctypes.c_float, ctypes.c_float, ctypes.c_uint64, _F]
        L.ots_mlp_train.restype = st
        L.ots_mlp_predict.argtypes = [vp, _F, ctypes.c_int32, _F]
        L.ots_mlp_predict.restype = st
        L.ots_mlp_topk.argtypes = [vp, _F, ctypes.c_int32, ctypes.c_int32,
                                   ctypes.POINTER(ctypes.c_int32)]
        L.ots_mlp_topk.restype = st
        L._mlp_ready = True
    return L


# ------------------------------------------------------------ evaluation --

def dataset(records):
    """(X, y, stencil per row, records) from sweep records with status ok.
    Target: log GUpdates/s.  The plain one-step kernel is not ranked (the
    picker always measures it beside the model's picks), so its records are
    left out."""
    rows = [r for r in records if r.get("status") == "ok" and r.get("gupdates", 0) > 0
            and r.get("kernel") != "plain"]
    X = np.stack([features(r["stencil"], r, r["geom"]) for r in rows]) if rows else np.zeros(
        (0, len(FEATURES)), np.float32)
    y = np.log(np.array([r["gupdates"] for r in rows], np.float64)).astype(np.float32)
    groups = [r["stencil"] for r in rows]
    return X, y, groups, rows


def expected_best_of_random(values, k):
    """E[max of k draws without replacement] from `values` (exact)."""
    v = np.sort(np.asarray(values, np.float64))  # ascending
    n = len(v)
    k = min(k, n)
    # P(max = v[i]) = C(i, k-1) / C(n, k)
    tot = 0.0
    logc = lambda a, b: math.lgamma(a + 1) - math.lgamma(b + 1) - math.lgamma(a - b + 1)
    den = logc(n, k)
    for i in range(k - 1, n):
        tot += v[i] * math.exp(logc(i, k - 1) - den)
    return tot


def plain_values(records):
    """stencil -> measured GUpdates/s of the plain one-step kernel."""
    return {r["stencil"]: r["gupdates"] for r in records
            if r.get("kernel") == "plain" and r.get("status") == "ok" and r.get("gupdates", 0) > 0}


def workload_records(configs):
    """The full-size workload sweeps of a bench --configs table (its per-
    workload 'records'), as dataset records with their stencil and size.  Rows
    in another arithmetic variant (the fast-division ones) are left out: the
    features do not carry the variant, so their times would contradict the
    baseline rows'."""
    out = []
    for w in configs.get("workloads", []):
        if w.get("variant", "baseline") != "baseline":
            continue
        for r in w.get("records", []):
            out.append(dict(r, stencil=w["stencil"], n=w["n"], steps=w["steps"]))
    return out


def leave_one_out_sizes(records, k_frac=0.10, hidden=64, layers=3, epochs=300, seed=0,
                        device=0):
    """Leave one stencil out over records of several problem sizes: train on
    every other stencil's records (all sizes), then for each size of the
    held-out stencil rank that size's space, measure the top k and the plain
    kernel (k + 1 = 10 % of the space) and report picked/best per size
    (keys 'stencil@n')."""
    by_size = {}
    for r in records:
        by_size.setdefault((r["stencil"], int(r.get("n", 0))), []).append(r)
    report = {}
    for s in sorted({k[0] for k in by_size}):
        train = [r for r in records if r["stencil"] != s]
        X, y, _, _ = dataset(train)
        if len(X) < 10:
            continue
        m = MLP(X.shape[1], hidden, layers, seed=seed, device=device)
        m.fit(X, y, epochs=epochs, seed=seed)
        for (st, n), recs in sorted(by_size.items()):
            if st != s:
                continue
            Xs, ys, _, rows = dataset(recs)
            if len(Xs) < 2:
                continue
            actual = np.exp(ys.astype(np.float64))
            p = plain_values(recs).get(s, 0.0)
            space = len(Xs) + (1 if p else 0)
            k = max(1, int(math.floor(k_frac * space)) - (1 if p else 0))
            top = m.topk(Xs, k)
            picked = max(float(np.max(actual[top])), p)
            best = max(float(np.max(actual)), p)
            report["%s@%d" % (s, n)] = {
                "space": space, "k": k, "measure_cost": (k + (1 if p else 0)) / float(space),
                "picked_over_best": picked / best, "picked_gupdates": picked,
                "best_gupdates": best,
                "top1_over_best": max(float(actual[top[0]]), p) / best,
                "random_k_over_best": expected_best_of_random(np.maximum(actual, p), k) / best,
                "picked_config": {q: rows[int(top[int(np.argmax(actual[top]))])][q]
                                  for q in ("kernel", "T", "bx", "by", "bz", "E")}}
        m.close()
    if report:
        report["_mean"] = {q: float(np.mean([v[q] for v in report.values()]))
                           for q in ("picked_over_best", "top1_over_best", "random_k_over_best",
                                     "measure_cost")}
    return report


def leave_one_out(records, k_frac=0.10, hidden=64, layers=3, epochs=300, batch=128, lr=3e-3,
                  weight_decay=1e-4, seed=0, device=0, held_out=None):
    """Train without stencil s, rank s's space, measure the top k -- and the
    plain one-step kernel, which the picker always measures (one more run):
    it is the fastest choice for some compute-bound stencils, and a handful
    of plain records is too few for the model to learn when.  Returns a
    report dict per held-out stencil and the means."""
    X, y, groups, rows = dataset(records)
    plain = plain_values(records)
    report = {}
    stencils = held_out or sorted(set(groups))
    for s in stencils:
        te = [i for i, g in enumerate(groups) if g == s]
        tr = [i for i, g in enumerate(groups) if g != s]
        if len(te) < 2 or len(tr) < 10:
            continue
        m = MLP(X.shape[1], hidden, layers, seed=seed, device=device)
        loss = m.fit(X[tr], y[tr], epochs=epochs, batch=batch, lr=lr, weight_decay=weight_decay,
                     seed=seed)
        actual = np.exp(y[te].astype(np.float64))
        p = plain.get(s, 0.0)
        space = len(te) + (1 if s in plain else 0)
        # the plain run counts against the same budget: k_frac of the space in all
        k = max(1, int(math.floor(k_frac * space)) - (1 if s in plain else 0))
        top = m.topk(X[te], k)
        picked = max(float(np.max(actual[top])), p)
        top1 = max(float(actual[top[0]]), p)
        best = max(float(np.max(actual)), p)
        rand_k = expected_best_of_random(np.maximum(actual, p), k)
        pred = m.predict(X[te])
        # rank correlation between predicted and measured
        rp = np.argsort(np.argsort(pred))
        ra = np.argsort(np.argsort(actual))
        spearman = float(np.corrcoef(rp, ra)[0, 1]) if len(te) > 2 else 0.0
        plain_rec = {"kernel": "plain", "T": 1, "bx": 0, "by": 0, "bz": 0, "E": 1}
        best_rec = rows[te[int(np.argmax(actual))]] if np.max(actual) >= p else plain_rec
        pick_rec = rows[te[int(top[int(np.argmax(actual[top]))])]] if np.max(actual[top]) >= p \
            else plain_rec
        # the same model ranking the tile-kernel configurations alone (the space
        # the reference's analytical model can rank)
        tile_only = None
        tsel = np.array([i for i, j in enumerate(te) if rows[j].get("kernel", "tile") == "tile"])
        if len(tsel) >= 2:
            at, pt = actual[tsel], np.asarray(pred)[tsel]
            kt = max(1, int(math.floor(k_frac * len(tsel))))
            order = np.argsort(-pt)
            tile_only = {"space": int(len(tsel)), "k": kt,
                         "picked_over_best": float(np.max(at[order[:kt]]) / np.max(at)),
                         "top1_over_best": float(at[order[0]] / np.max(at))}
        report[s] = {
            "space": space, "k": k, "measure_cost": (k + (1 if s in plain else 0)) / float(space),
            "plain_gupdates": p or None,
            "best_gupdates": best, "picked_gupdates": picked, "picked_over_best": picked / best,
            # the model alone: best of its k picks over the best time-tiled configuration
            "picked_over_best_tiled": float(np.max(actual[top]) / np.max(actual)),
            "top1_over_best": top1 / best, "random_k_over_best": rand_k / best,
            "median_over_best": float(np.median(actual)) / best, "spearman": spearman,
            "train_loss": loss,
            "best_config": {q: best_rec[q] for q in ("kernel", "T", "bx", "by", "bz", "E")},
            "picked_config": {q: pick_rec[q] for q in ("kernel", "T", "bx", "by", "bz", "E")},
            "tile_only": tile_only,
        }
        m.close()
    if report:
        report["_mean"] = {q: float(np.mean([v[q] for v in report.values()]))
                           for q in ("picked_over_best", "picked_over_best_tiled", "top1_over_best",
                                     "random_k_over_best", "median_over_best", "measure_cost",
                                     "spearman")}
    return report
