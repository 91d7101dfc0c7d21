"""Pins the CPU oracle to the reference's own code (CPU only).

The golden fixtures were produced by tests/golden/make_golden.py from the
reference's compiled CPU loops, fill loops and GeneratorParams derivations;
the oracle must reproduce them bit for bit.
"""
import ctypes
import json
import os

import numpy as np
import pytest

import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _loops():
    z = np.load(os.path.join(GOLD, "ref_loops.npz"))
    keys = sorted({k.split("_")[0] for k in z.files})
    return [(k, z[k + "_in"], z[k + "_out"], z[k + "_meta"]) for k in keys]


@pytest.mark.parametrize("case", _loops(), ids=lambda c: c[0])
def test_oracle_matches_reference_cpu_loop(case):
    key, x, y, meta = case
    sid, P, pad, steps, seed, real = [int(v) for v in meta]
    st = O.STENCILS[sid]
    got = O.sweep_f32(st, [x], steps=steps, lo=pad, hi=P - pad, variant=O.VARIANT_REF)[0]
    assert np.array_equal(got.view(np.uint32), y.view(np.uint32)), st


def test_oracle_fill_matches_reference_fills():
    z = np.load(os.path.join(GOLD, "ref_fills.npz"))
    for which in ("poisson_2d", "fdtd_2d", "cs_3d"):
        P, pad, seed, nf = [int(v) for v in z[which + "_meta"]]
        d = {"poisson_2d": 2, "fdtd_2d": 2, "cs_3d": 3}[which]
        mine = O.fill_ref(d, P, pad, P - pad, seed, nf)
        for i in range(nf):
            assert np.array_equal(mine[i], z["%s_%d" % (which, i)]), which
    P, pad, seed, _ = [int(v) for v in z["jacobi_1d_5pt_meta"]]
    out = np.zeros(P, np.float32)
    L = O.lib()
    L.orc_fill_ref_1d_runner.argtypes = [ctypes.c_int] * 3 + [ctypes.c_uint, O._F]
    L.orc_fill_ref_1d_runner(P, pad, P - pad, seed, O._fp(out))
    assert np.array_equal(out, z["jacobi_1d_5pt_0"])


def test_oracle_geometry_matches_reference_compute_derived():
    rows = json.load(open(os.path.join(GOLD, "ref_geometry.json")))
    assert len(rows) > 500
    for st, n, T, bx, by, bz, E, r in rows:
        g = O.geometry_ref(st, n, T, bx, by, bz, E)
        assert (r is None) == (g is None), (st, n, T, bx, by, bz, E)
        if r is None:
            continue
        assert (g.padding, g.padded_size, g.real_size, g.size_lcm) == (
            r["padding"], r["padded_size"], r["real_size"], r["size_lcm"])
        for a, ax in enumerate("xyz"[: O.dims(st)]):
            assert g.rpb[a] == r["rpb_" + ax]
            assert g.num_blocks[a] == r["num_blocks_" + ax]
            assert g.shared[a] == r["shared_" + ax]
            assert g.comps[a] == r["comps_" + ax]


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built here")
@pytest.mark.parametrize("st", sorted(O.REF_LOOPS))
def test_oracle_matches_live_reference_loops(st):
    """Same pin on fresh seeded inputs, against the live reference library."""
    d = O.dims(st)
    r = O.radius(st) if d == 1 else 1
    pad = 2 * r
    P = {1: 300, 2: 30}[d]
    x = O.fill_ref(d, P, pad, P - pad, 4242, 1)[0]
    want = O.ref_loop(st, x, pad, 6)
    got = O.sweep_f32(st, [x], steps=6, lo=pad, hi=P - pad, variant=O.VARIANT_REF)[0]
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
