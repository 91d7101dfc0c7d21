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


def _kernel_cases():
    p = os.path.join(GOLD, "ref_kernels.npz")
    z = np.load(p)
    keys = sorted({k.split("_")[0] for k in z.files})
    out = []
    for k in keys:
        meta = [int(v) for v in z[k + "_meta"]]
        nf, na = meta[8], meta[9]
        out.append((k, [z["%s_in%d" % (k, i)] for i in range(nf)],
                    [z["%s_aux%d" % (k, i)] for i in range(na)],
                    [z["%s_out%d" % (k, i)] for i in range(nf)], meta))
    return out


@pytest.mark.parametrize("case", _kernel_cases(),
                         ids=lambda c: "%s-%s-T%d" % (c[0], O.STENCILS[c[4][0]], c[4][6]))
def test_oracle_matches_reference_generated_kernel(case):
    """The seven stencils whose runners have no usable CPU check, pinned to
    the kernels the reference's own generators emit (fixtures made by
    tests/golden/make_golden.py: the generated OpenCL text run on the CPU by
    oracle/ref_clkernel.cpp, one thread per work-item, with the runner's
    launch loop).  Bit for bit: jacobi-3d (weight 0.143f), poisson-3d (26c -
    the 26 neighbours), gradient-3d, fdtd-2d (the reference's +Ey, no
    source), rician-denoise-2d, cdsc-tv-update-2d and cs-3d (its first
    step's y orientation, oracle variant 9), at T = 1 and -- for the 3D star
    stencils -- through the reference's in-tile time step at T = 2."""
    key, fields, aux, want, meta = case
    sid, P, pad, steps, seed, real, T, variant = meta[:8]
    st = O.STENCILS[sid]
    coef = float(np.float32(0.143)) if st == "jacobi-3d" else 0.0
    got = O.sweep_f32(st, fields, aux, steps=steps, lo=pad, hi=pad + real, variant=variant,
                      coef=coef)
    for f, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (
            st, f, float(np.max(np.abs(a.astype(np.float64) - b))))


def test_cs3d_orientation_variants_are_distinct_code_paths():
    """cs-3d's oracle variant 9 (the reference's first-step y orientation,
    pinned above) and variant 0 (y+1 as "p1" throughout, the in-tile steps' and the
    engine's) share every operation but the two y-axis neighbours: they agree
    where those neighbours are equal and differ on a generic field."""
    P, pad = 14, 1
    x = O.fill_ref(3, P, pad, P - pad, 3, 1)[0]
    c = O.sweep_f32("cs-3d", [x], steps=1, lo=pad, hi=P - pad, variant=0)[0]
    d = O.sweep_f32("cs-3d", [x], steps=1, lo=pad, hi=P - pad, variant=9)[0]
    assert not np.array_equal(c, d)
    # a field constant along y: the y-axis neighbours equal the centre
    flat = np.ascontiguousarray(np.repeat(x[:, 5:6, :], P, axis=1))
    flat[:, :pad, :] = 0
    flat[:, P - pad:, :] = 0
    e = O.sweep_f32("cs-3d", [flat], steps=1, lo=pad, hi=P - pad, variant=0)[0]
    f = O.sweep_f32("cs-3d", [flat], steps=1, lo=pad, hi=P - pad, variant=9)[0]
    inner = (slice(pad, P - pad), slice(pad + 1, P - pad - 1), slice(pad, P - pad))
    assert np.array_equal(e[inner], f[inner])


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built here")
def test_generated_kernel_pin_live_on_fresh_inputs():
    """The same pin run live (where the reference tree is present) on a
    fresh seed and a case not among the fixtures: jacobi-3d at T = 1 with
    E = 4 along y."""
    import build_ref
    if not os.path.exists(build_ref.GEN_LIB):
        pytest.skip("reference generators not built here")
    st, n, T, bx, by, bz, E, steps = "jacobi-3d", 16, 1, 4, 1, 4, 4, 3
    g = O.ref_geometry(st, n, T, bx, by, bz, E)
    P, pad, real = g["padded_size"], g["padding"], g["real_size"]
    x = O.fill_ref(3, P, pad, pad + real, 2024, 1)
    lib = build_ref.build_kernel_case(st, n, T, bx, by, bz, E, steps)
    want = O.ref_kernel_run(lib, x, [], T=T, steps=steps,
                            nb=[g["num_blocks_x"], g["num_blocks_y"], g["num_blocks_z"]],
                            bs=[bx, by, bz])[0]
    got = O.sweep_f32(st, x, steps=steps, lo=pad, hi=pad + real, variant=O.VARIANT_REF,
                      coef=float(np.float32(0.143)))[0]
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
