"""GPU parity: every stencil and kernel family through the C ABI against the
CPU oracle on identical seeded inputs.

Linear stencils (the Jacobi family, both Poisson variants, both FDTD
variants) and cs-3d (whose 1/sqrt terms are double expressions in the
reference's text, IEEE on both sides) must match bit for bit: the library is
built with -fmad=false and keeps the oracle's operand order.  The other
stencils with a 1/sqrt term use the GPU's float rsqrt (as the reference
kernels use OpenCL rsqrt) against a correctly rounded 1/sqrt on the CPU; their
tolerance is stated per stencil below.
"""
import numpy as np
import pytest

import oracle as O
import ots

EXACT = {"jacobi-1d", "jacobi-1d-5pt", "jacobi-1d-7pt", "jacobi-2d", "jacobi-3d", "poisson-2d",
         "poisson-3d", "fdtd-2d", "cs-3d"}
# Bound on max |gpu - cpu| / max(|cpu|, 1) after the step counts used here:
# a relative error where |cpu| >= 1 and an ABSOLUTE error where |cpu| < 1
# (the floor of 1 keeps cells near zero from dividing by ~0).  Rician and TV
# values lie in [0, 1) on these inputs, so theirs is an absolute bound.
# rsqrtf is within 2 ulp per call; gradient's 1/sqrt(1e-4 + sum d^2)
# amplifies that by its sensitivity to the differences d (measured 2.2e-5 on
# B200).
RTOL = {"gradient-2d": 1e-4, "gradient-3d": 1e-4, "rician-denoise-2d": 2e-5,
        "cdsc-tv-update-2d": 2e-5}


def inputs(plan, seed):
    state, aux = plan.fill_reference(seed=seed)
    if plan.stencil in ("poisson-2d", "poisson-3d"):
        aux = [np.where(a != 0, 2.0 * a - 1.0, 0.0).astype(np.float32) for a in aux]
    return state, aux


def run_and_check(stencil, n, steps, seed=123456, **kw):
    with ots.Plan(stencil, n, steps, device=0, **kw) as plan:
        g = plan.geometry
        state, aux = inputs(plan, seed)
        plan.upload(state, aux)
        plan.run()
        got = plan.download()
        want = O.sweep_f32(stencil, state, aux=aux, steps=steps, lo=g.padding,
                           hi=g.padding + g.real_size, variant=plan.params.variant,
                           coef=g.coef, h2=g.h2)
        for f, (a, b) in enumerate(zip(got, want)):
            if stencil in EXACT:
                bad = np.count_nonzero(a.view(np.uint32) != b.view(np.uint32))
                assert bad == 0, "%s field %d: %d cells differ (max |d| %g)" % (
                    stencil, f, bad, float(np.max(np.abs(a - b))))
            else:
                err = float(np.max(np.abs(a.astype(np.float64) - b) / np.maximum(np.abs(b), 1.0)))
                assert err <= RTOL[stencil], "%s field %d: rel err %g" % (stencil, f, err)
        return plan.geometry


# (stencil, n, steps, T, bx, by, bz, E)
TILE_CASES = [
    ("jacobi-1d", 1000, 9, 3, 64, 1, 1, 4),
    ("jacobi-1d", 777, 5, 1, 32, 1, 1, 1),
    ("jacobi-1d-5pt", 1003, 10, 4, 128, 1, 1, 2),
    ("jacobi-1d-7pt", 999, 7, 3, 64, 1, 1, 3),
    ("jacobi-2d", 67, 9, 4, 16, 16, 1, 1),
    ("jacobi-2d", 100, 64, 8, 32, 8, 1, 4),
    ("jacobi-2d", 33, 5, 2, 16, 4, 1, 12),
    ("poisson-2d", 71, 8, 3, 32, 8, 1, 2),
    ("gradient-2d", 61, 6, 3, 16, 8, 1, 3),
    ("fdtd-2d", 58, 11, 4, 32, 8, 1, 2),
    ("fdtd-2d", 40, 3, 1, 16, 16, 1, 1),
    ("rician-denoise-2d", 53, 5, 2, 32, 8, 1, 4),
    ("cdsc-tv-update-2d", 49, 6, 3, 16, 16, 1, 2),
    ("jacobi-3d", 37, 7, 3, 16, 8, 4, 4),
    ("jacobi-3d", 20, 4, 1, 8, 8, 8, 1),
    ("poisson-3d", 29, 5, 2, 16, 8, 2, 4),
    ("gradient-3d", 27, 4, 2, 16, 4, 2, 4),
    ("cs-3d", 25, 5, 2, 16, 8, 2, 3),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", TILE_CASES, ids=lambda c: "%s-n%d-T%d-E%d" % (c[0], c[1], c[3], c[7]))
def test_tile_kernel_matches_oracle(case):
    st, n, steps, T, bx, by, bz, E = case
    run_and_check(st, n, steps, T=T, bx=bx, by=by, bz=bz, E=E, kernel="tile")


@pytest.mark.gpu
@pytest.mark.parametrize("st", ots.STENCILS)
def test_plain_kernel_matches_oracle(st):
    d = O.dims(st)
    n = {1: 900, 2: 45, 3: 22}[d]
    run_and_check(st, n, 5, kernel="plain")


@pytest.mark.gpu
@pytest.mark.parametrize("st", ["jacobi-2d", "poisson-2d", "gradient-2d", "fdtd-2d", "jacobi-3d",
                                "poisson-3d", "cs-3d", "jacobi-1d-5pt"])
def test_reference_variant_and_compat_engine(st):
    d = O.dims(st)
    if d == 1:
        kw = dict(n=500, T=2, bx=64, by=1, bz=1, E=2)
    elif d == 2:
        kw = dict(n=70, T=3, bx=16, by=8, bz=1, E=2)
    else:
        kw = dict(n=30, T=1, bx=8, by=4, bz=4, E=2)
    steps = 6 if st not in ("poisson-2d", "poisson-3d") else 4
    g = run_and_check(st, kw.pop("n"), steps, engine=ots.ENGINE_COMPAT,
                      variant=ots.VARIANT_REF, kernel="tile", **kw)
    assert g.real_size % g.size_lcm == 0


@pytest.mark.gpu
@pytest.mark.parametrize("st", ["jacobi-3d", "poisson-3d", "gradient-3d"])
@pytest.mark.parametrize("T", [1, 2, 3, 4, 5, 8])
@pytest.mark.parametrize("E", [1, 2, 4])
def test_stream_kernel_matches_oracle(st, T, E):
    if T < 5:
        bx, by = {1: (16, 16), 2: (16, 8), 4: (16, 6)}[E]
    else:
        bx, by = {1: (8, 24), 2: (16, 12), 4: (16, 6)}[E]
    run_and_check(st, 41, 2 * T + 1, T=T, bx=bx, by=by, bz=1, E=E, kernel="stream")


@pytest.mark.gpu
@pytest.mark.parametrize("cy", [2, 3, 4, 8])
@pytest.mark.parametrize("st,T,E,bx,by", [
    ("jacobi-3d", 1, 2, 16, 8),
    ("jacobi-3d", 3, 2, 8, 16),
    ("jacobi-3d", 2, 4, 16, 4),
    ("jacobi-3d", 4, 1, 32, 8),
    ("poisson-3d", 3, 2, 16, 4),
    ("gradient-3d", 2, 1, 8, 8),
])
def test_stream_cluster_matches_oracle(cy, st, T, E, bx, by):
    # y-clustered tiles: rows cross CTA boundaries through distributed shared
    # memory; n not a multiple of the cluster tile, several z segments
    run_and_check(st, 70, 2 * T + 1, T=T, bx=bx, by=by, bz=1, E=E, kernel="stream", cy=cy)


@pytest.mark.gpu
def test_stream_cluster_block_one_row_and_partial():
    # by = 1: each thread is both the top and the bottom row of its CTA
    run_and_check("jacobi-3d", 45, 7, T=2, bx=32, by=1, bz=1, E=4, kernel="stream", cy=4)
    run_and_check("jacobi-3d", 133, 10, T=3, bx=16, by=8, bz=1, E=2, kernel="stream", cy=3)


@pytest.mark.gpu
def test_stream_kernel_partial_tiles_and_segments():
    # n not a multiple of the tile interior, more steps than one launch
    run_and_check("jacobi-3d", 133, 10, T=4, bx=32, by=6, bz=1, E=2, kernel="stream")
    run_and_check("jacobi-3d", 64, 13, T=3, bx=8, by=16, bz=1, E=2, kernel="stream")
    run_and_check("jacobi-3d", 150, 9, T=2, bx=32, by=4, bz=1, E=4, kernel="stream")


@pytest.mark.gpu
def test_steps_zero_and_shallow_last_launch():
    for steps in (0, 1, 5):
        run_and_check("jacobi-2d", 50, steps, T=4, bx=16, by=16, E=1, kernel="tile")
        run_and_check("jacobi-3d", 30, steps, T=4, bx=16, by=8, E=2, kernel="stream")


@pytest.mark.gpu
def test_repeated_runs_are_deterministic_and_continue():
    with ots.Plan("jacobi-3d", 48, 6, T=3, bx=16, by=8, bz=1, E=2, kernel="stream") as plan:
        state, _ = plan.fill_reference(seed=3)
        plan.upload(state)
        plan.run()
        plan.run()  # second call continues from the first call's result
        a = plan.download()[0]
        plan.upload(state)
        plan.run()
        plan.run()
        b = plan.download()[0]
        g = plan.geometry
        want = O.sweep_f32("jacobi-3d", state, steps=12, lo=g.padding, hi=g.padding + g.real_size,
                           coef=g.coef)[0]
    assert np.array_equal(a, b) and np.array_equal(a, want)


@pytest.mark.gpu
def test_kernel_families_agree_bitwise_on_one_plan():
    with ots.Plan("poisson-3d", 52, 9, T=3, bx=16, by=8, bz=1, E=2, kernel="stream") as plan:
        state, aux = inputs(plan, 11)
        outs = []
        for k in ("stream", "plain"):
            plan.upload(state, aux)
            plan.run(k)
            outs.append(plan.download()[0])
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("st", ["rician-denoise-2d", "cdsc-tv-update-2d"])
@pytest.mark.parametrize("T,bx,by,E", [(1, 32, 8, 1), (2, 32, 8, 8), (3, 16, 16, 2),
                                       (4, 64, 8, 4), (2, 16, 4, 3)])
def test_two_phase_tile_equals_fused_kernels_bitwise(st, T, bx, by, E):
    """The tile kernel runs Rician in two phases (g stored once per cell in
    shared memory); the plain kernel and the y-streamed kernel recompute g at
    every neighbour.  Same operations on the same values: the three agree bit
    for bit, as they do for TV (fused in every kernel), on the reference fill
    and on the disk image with Rician noise, with partial edge tiles."""
    from ots import workloads as W
    n, steps = 203, 7
    with ots.Plan(st, n, steps, T=T, bx=bx, by=by, bz=1, E=E, kernel="tile") as plan:
        g = plan.geometry
        sl = tuple(slice(g.padding, g.padding + g.real_size) for _ in range(2))
        fills = [inputs(plan, 3)]
        f = W.disk_image(g.padded_size, seed=9)[1]
        img = np.zeros_like(fills[0][0][0])
        img[sl] = f[sl]
        fills.append(([img.copy()], [img] if st == "rician-denoise-2d" else
                      [img, np.where(img != 0, 1.0, 0.0).astype(np.float32)]))
        for state, aux in fills:
            outs = []
            for k in ("tile", "plain", "stream"):
                plan.upload(state, aux)
                plan.run(k)
                outs.append(plan.download()[0])
            assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32)), "tile vs plain"
            assert np.array_equal(outs[0].view(np.uint32), outs[2].view(np.uint32)), "tile vs stream"


@pytest.mark.gpu
@pytest.mark.parametrize("st,n,steps,T,bx,by,E", [
    ("jacobi-2d", 67, 9, 4, 16, 16, 1),
    ("jacobi-2d", 100, 13, 3, 32, 8, 4),
    ("jacobi-2d", 33, 5, 2, 16, 4, 8),
    ("gradient-2d", 70, 7, 3, 16, 8, 2),
    ("poisson-2d", 71, 8, 3, 32, 8, 2),
    ("rician-denoise-2d", 66, 6, 2, 16, 8, 1),
])
def test_texture_kernel_matches_oracle(st, n, steps, T, bx, by, E):
    # first-step loads through the texture unit (border addressing = zero ring)
    g = run_and_check(st, n, steps, T=T, bx=bx, by=by, bz=1, E=E, kernel="tex")
    assert g.kernel == ots.KERNEL_TEX


@pytest.mark.gpu
def test_texture_kernel_equals_tile_kernel_bitwise_and_rejects_unsupported():
    with ots.Plan("jacobi-2d", 300, 20, T=4, bx=32, by=8, E=2, kernel="tex") as plan:
        state, _ = plan.fill_reference(seed=4)
        outs = []
        for k in ("tex", "tile", "plain"):
            plan.upload(state)
            plan.run(k)
            outs.append(plan.download()[0])
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))
    assert np.array_equal(outs[0].view(np.uint32), outs[2].view(np.uint32))
    for kw in (dict(stencil="fdtd-2d", n=64), dict(stencil="jacobi-3d", n=32)):
        with pytest.raises(ots.OtsError) as ei:
            ots.Plan(kw["stencil"], kw["n"], 4, T=2, bx=16, by=8, E=1, kernel="tex")
        assert ei.value.status_name == "UNSUPPORTED"


@pytest.mark.gpu
@pytest.mark.parametrize("st", ["jacobi-2d", "poisson-2d", "gradient-2d"])
@pytest.mark.parametrize("T", [1, 2, 3, 4, 5, 8])
def test_stream2d_kernel_matches_oracle(st, T):
    # y-streamed 2D kernel: n not a multiple of the strip interior, several
    # y segments, the last launch shallower than T
    g = run_and_check(st, 301, 2 * T + 1, T=T, bx=32, by=1, E=1, kernel="stream")
    assert g.kernel == ots.KERNEL_STREAM and g.num_blocks[0] >= 3


@pytest.mark.gpu
@pytest.mark.parametrize("st", ["jacobi-2d", "poisson-2d"])
@pytest.mark.parametrize("T", [1, 2, 3, 4, 5, 8])
def test_stream2d_packed_kernel_matches_oracle(st, T):
    # the packed-FP32 form, n a multiple of 4 (one mask per lane) and not (the
    # edge lane's cells masked one by one): bit for bit against the oracle and
    # against the scalar kernel (stream_impl 1), n not a multiple of the strip
    # interior, several y segments, the last launch shallower than T
    for n in (300, 301, 302, 303):
        outs = []
        for impl in (0, 1):
            with ots.Plan(st, n, 2 * T + 1, T=T, bx=32, by=1, E=1, kernel="stream",
                          impl=impl) as plan:
                assert plan.describe()["Stream Arithmetic"] == ("packed-fp32" if impl == 0
                                                                else "scalar")
                g = plan.geometry
                state, aux = inputs(plan, seed=31 + T)
                plan.upload(state, aux)
                plan.run()
                outs.append(plan.download()[0])
        want = O.sweep_f32(st, state, aux=aux, steps=2 * T + 1, lo=g.padding,
                           hi=g.padding + g.real_size, coef=g.coef, h2=g.h2)[0]
        for o in outs:
            assert np.array_equal(o.view(np.uint32), want.view(np.uint32)), n
    # edge sizes: a single strip, one row per segment, the reference weight
    for n, steps, by in ((4, 3, 1), (5, 3, 1), (128, 9, 1), (129, 7, 1), (240, 7, 16)):
        run_and_check(st, n, steps, T=T, bx=32, by=by, bz=1, E=1, kernel="stream")
    if st == "jacobi-2d":
        run_and_check(st, 64, 5, T=T, bx=32, by=1, bz=1, E=1, kernel="stream",
                      variant=ots.VARIANT_REF)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("T", [1, 2, 3, 5, 6])
def test_fdtd_stream_kernel_ragged_widths_and_segments_match_oracle(variant, T):
    # FDTD-2D's two-phase streamed kernel, bit for bit against the oracle with
    # the source row (variant 0) and the reference's +Ey (variant 1), rows not
    # a multiple of 4, in the model's segments and in 8-row ones (iterations
    # whose level rows all lie inside the grid skip the row test)
    for n in (140, 141, 143):
        outs = []
        for by in (1, 8):
            with ots.Plan("fdtd-2d", n, 2 * T + 1, T=T, bx=32, by=by, E=1, kernel="stream",
                          variant=variant) as plan:
                assert plan.describe()["Stream Arithmetic"] == "scalar"
                g = plan.geometry
                state, aux = inputs(plan, seed=41 + T)
                plan.upload(state, aux)
                plan.run()
                outs.append(plan.download())
        want = O.sweep_f32("fdtd-2d", state, aux=aux, steps=2 * T + 1, lo=g.padding,
                           hi=g.padding + g.real_size, variant=variant)
        for got in outs:
            for f, (a, b) in enumerate(zip(got, want)):
                assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (n, f)


@pytest.mark.gpu
@pytest.mark.parametrize("st,variant", [("fdtd-2d", 0), ("fdtd-2d", 1), ("rician-denoise-2d", 0),
                                        ("cdsc-tv-update-2d", 0), ("poisson-2d", 1)])
@pytest.mark.parametrize("T", [1, 2, 3, 4, 6])
def test_stream2d_generic_matches_oracle(st, variant, T):
    # the op's own apply() on register rows: several fields (FDTD and its
    # row-0 source), radius 2 (Rician), diagonal neighbours and two aux fields
    # (TV), the 9-point reference Poisson
    g = run_and_check(st, 150, 2 * T + 1, T=T, bx=32, by=1, E=1, kernel="stream",
                      variant=variant)
    assert g.kernel == ots.KERNEL_STREAM


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [0, 2])
@pytest.mark.parametrize("n,steps,T", [(150, 13, 1), (301, 9, 3), (257, 11, 4), (130, 7, 6)])
def test_stream2d_rician_two_phase_equals_tile_bitwise(variant, n, steps, T):
    # the streamed Rician kernel computes g once per cell a row ahead of its
    # update; the tile kernel (two-phase as well) and the plain kernel (g
    # recomputed at each neighbour) give the same bits
    with ots.Plan("rician-denoise-2d", n, steps, T=T, bx=32, by=1, E=1, kernel="stream",
                  variant=variant) as plan:
        state, aux = plan.fill_reference(seed=11 + T)
        g = plan.geometry
        cut = (slice(g.padding, g.padding + n),) * 2
        u, f = np.ascontiguousarray(state[0][cut]), np.ascontiguousarray(aux[0][cut])
        outs = []
        for k in ("stream", "plain"):
            plan.upload_interior([u], [f])
            plan.run(k)
            outs.append(plan.download_interior()[0])
    with ots.Plan("rician-denoise-2d", n, steps, T=2, bx=32, by=8, E=2, kernel="tile",
                  variant=variant) as plan:
        plan.upload_interior([u], [f])
        plan.run("tile")
        outs.append(plan.download_interior()[0])
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))
    assert np.array_equal(outs[0].view(np.uint32), outs[2].view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("st", ["jacobi-1d", "jacobi-1d-5pt", "jacobi-1d-7pt"])
@pytest.mark.parametrize("T,E", [(1, 4), (5, 4), (3, 8), (8, 16), (16, 16)])
def test_stream1d_register_kernel_matches_oracle(st, T, E):
    # T steps held in registers per warp strip; n not a multiple of the strip
    # interior, the last launch shallower than T
    g = run_and_check(st, 100003, 2 * T + 3, T=T, bx=32, by=1, E=E, kernel="stream")
    assert g.kernel == ots.KERNEL_STREAM and g.threads[0] == 32


@pytest.mark.gpu
def test_stream1d_edges_and_limits():
    for n, steps, T, E in ((3, 4, 2, 4), (128, 9, 4, 4), (129, 7, 30, 16), (5000, 0, 4, 8),
                           (5000, 1, 4, 8)):
        run_and_check("jacobi-1d", n, steps, T=T, bx=32, by=1, E=E, kernel="stream")
    with pytest.raises(ots.OtsError) as ei:  # 128 cells cannot hold 2 x 90 halo cells
        ots.Plan("jacobi-1d-7pt", 1000, 60, T=30, bx=32, by=1, E=4, kernel="stream")
    assert ei.value.status_name == "INVALID_GEOMETRY"
    with pytest.raises(ots.OtsError) as ei:
        ots.Plan("jacobi-1d", 1000, 8, T=4, bx=32, by=1, E=2, kernel="stream")
    assert ei.value.status_name == "UNSUPPORTED"


@pytest.mark.gpu
def test_stream2d_small_and_edge_grids():
    for n, steps, T in ((5, 3, 2), (128, 9, 4), (129, 7, 8), (1000, 13, 6)):
        run_and_check("jacobi-2d", n, steps, T=T, bx=32, by=1, E=1, kernel="stream")
    for steps in (0, 1):
        run_and_check("jacobi-2d", 64, steps, T=4, bx=32, by=1, E=1, kernel="stream")
    for st, n, steps, T in (("rician-denoise-2d", 7, 5, 3), ("fdtd-2d", 129, 11, 4),
                            ("cdsc-tv-update-2d", 300, 7, 6)):
        run_and_check(st, n, steps, T=T, bx=32, by=1, E=1, kernel="stream")
    with pytest.raises(ots.OtsError) as ei:
        ots.Plan("fdtd-2d", 64, 8, T=7, bx=32, by=1, E=1, kernel="stream")
    assert ei.value.status_name == "UNSUPPORTED"


@pytest.mark.gpu
def test_stream2d_full_size_equals_tile_and_plain_bitwise():
    """jacobi-2d 2048^2 x 64 steps (the 2D workload): stream, tile and plain
    kernels give identical bits."""
    with ots.Plan("jacobi-2d", 2048, 64, T=8, bx=32, by=1, E=1, kernel="stream") as plan:
        state, _ = plan.fill_reference(seed=123456)
        g = plan.geometry
        inner = np.ascontiguousarray(state[0][g.padding:g.padding + 2048,
                                              g.padding:g.padding + 2048])
        outs = []
        for k in ("stream", "plain"):
            plan.upload_interior([inner])
            plan.run(k)
            outs.append(plan.download_interior()[0])
    with ots.Plan("jacobi-2d", 2048, 64, T=4, bx=16, by=16, E=1, kernel="tile") as plan:
        plan.upload_interior([inner])
        plan.run()
        outs.append(plan.download_interior()[0])
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))
    assert np.array_equal(outs[0].view(np.uint32), outs[2].view(np.uint32))


@pytest.mark.gpu
def test_async_copies_pipeline_two_plans_like_the_blocking_calls():
    kw = dict(T=3, bx=16, by=8, bz=1, E=2, kernel="stream")
    with ots.Plan("poisson-3d", 70, 7, **kw) as a, ots.Plan("poisson-3d", 70, 7, **kw) as b:
        inner = [np.random.default_rng(s).random((70, 70, 70), dtype=np.float32) for s in (1, 2)]
        f = np.random.default_rng(3).random((70, 70, 70), dtype=np.float32)
        a.upload_interior([inner[0]], [f])
        a.run()
        want0 = a.download_interior()[0]
        a.upload_interior([inner[1]], [f])
        a.run()
        want1 = a.download_interior()[0]
        outs = [[np.zeros_like(inner[0])] for _ in range(4)]
        for s in range(4):  # a, b, a, b: each plan reused while the other runs
            pl = (a, b)[s % 2]
            pl.upload_interior_async([inner[s % 2]], [f])
            pl.run_async()
            pl.download_interior_async(outs[s])
        a.sync()
        b.sync()
    for s in range(4):
        want = want0 if s % 2 == 0 else want1
        assert np.array_equal(outs[s][0].view(np.uint32), want.view(np.uint32)), s
    with pytest.raises(ValueError):
        with ots.Plan("jacobi-3d", 16, 2, **kw) as c:
            c.upload_interior_async([np.zeros((16, 16, 16), np.float64)])


@pytest.mark.gpu
def test_interior_upload_download_roundtrip():
    with ots.Plan("fdtd-2d", 37, 3, T=2, bx=16, by=8, E=1, kernel="tile") as plan:
        state, _ = plan.fill_reference(seed=8)
        g = plan.geometry
        inner = [np.ascontiguousarray(s[g.padding:g.padding + g.real_size,
                                        g.padding:g.padding + g.real_size]) for s in state]
        plan.upload_interior(inner)
        plan.run()
        a = plan.download_interior()
        plan.upload(state)
        plan.run()
        b = plan.download()
        for x, y in zip(a, b):
            assert np.array_equal(x, y[g.padding:g.padding + g.real_size,
                                       g.padding:g.padding + g.real_size])


@pytest.mark.gpu
@pytest.mark.parametrize("limit", [1, 2, 3])
def test_phase_limited_kernels_run(limit):
    with ots.Plan("jacobi-2d", 64, 8, T=4, bx=16, by=16, E=1, kernel="tile",
                  phase_limit=limit) as plan:
        state, _ = plan.fill_reference()
        plan.upload(state)
        t = plan.run()
        assert t.launches == 2


@pytest.mark.gpu
def test_errors_are_statuses_not_crashes():
    with pytest.raises(ots.OtsError) as ei:
        ots.Plan("jacobi-3d", 64, 4, T=4, bx=32, by=64, bz=1, E=4, kernel="stream")
    assert ei.value.status_name in ("BLOCK_TOO_LARGE", "UNSUPPORTED", "SMEM_TOO_LARGE")
    with pytest.raises(ots.OtsError) as ei:
        ots.Plan("cs-3d", 32, 4, T=2, bx=16, by=8, bz=1, E=2, kernel="stream")
    assert ei.value.status_name == "UNSUPPORTED"
    with pytest.raises(ots.OtsError) as ei:
        ots.Plan("jacobi-2d", 64, 4, T=2, bx=64, by=32, E=1, kernel="tile")
    assert ei.value.status_name == "BLOCK_TOO_LARGE"
    with pytest.raises(ots.OtsError) as ei:
        ots.Plan("jacobi-2d", 64, 4, device=999)
    assert ei.value.status_name == "INVALID_ARGUMENT"


@pytest.mark.gpu
def test_full_size_jacobi_3d_cluster_tiled_equals_plain():
    """512^3 x 100 steps with y-clustered stream tiles (4 CTAs per cluster):
    identical bits to the plain one-step kernel."""
    n, steps = 512, 100
    with ots.Plan("jacobi-3d", n, steps, T=3, bx=16, by=8, bz=1, E=2, kernel="stream",
                  cy=4) as plan:
        state, _ = plan.fill_reference(seed=99)
        plan.upload(state)
        plan.run("stream")
        a = plan.download_interior()[0]
        plan.upload(state)
        plan.run("plain")
        b = plan.download_interior()[0]
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.gpu
def test_full_size_jacobi_3d_tiled_equals_plain_and_fp64_error():
    """512^3 x 100 steps (the headline workload): the z-streamed time tile and
    the plain one-step kernel give identical bits (size-independent property),
    and the result's max relative error against an FP64 sweep of a 96^3 cut
    with the same boundary stays within 1e-5."""
    n, steps = 512, 100
    with ots.Plan("jacobi-3d", n, steps, T=4, bx=32, by=8, bz=1, E=2, kernel="stream") as plan:
        state, _ = plan.fill_reference(seed=123456)
        plan.upload(state)
        plan.run("stream")
        a = plan.download_interior()[0]
        plan.upload(state)
        plan.run("plain")
        b = plan.download_interior()[0]
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.isfinite(a).all() and 0.0 < float(a.mean()) < 1.0
    # FP64 error on a smaller cube of the same workload shape
    m = 96
    with ots.Plan("jacobi-3d", m, steps, T=4, bx=32, by=8, bz=1, E=2, kernel="stream") as plan:
        state, _ = plan.fill_reference(seed=123456)
        plan.upload(state)
        plan.run()
        got = plan.download()[0]
        g = plan.geometry
    O.set_threads(8)
    ref64 = O.sweep_f64("jacobi-3d", state, steps=steps, lo=g.padding, hi=g.padding + m,
                        coef=g.coef)[0]
    mr, rms = O.error_vs_f64(got, ref64, g.padding, g.padding + m, floor=1e-6)
    assert mr <= 1e-5, mr


@pytest.mark.gpu
@pytest.mark.parametrize("st", ["jacobi-3d", "poisson-3d"])
@pytest.mark.parametrize("T", [1, 2, 3, 4])
@pytest.mark.parametrize("E,bx,by", [(4, 16, 16), (4, 16, 8), (4, 8, 16), (2, 16, 32),
                                     (2, 32, 16), (2, 16, 16)])
def test_packed_stream_kernel_matches_oracle(st, T, E, bx, by):
    """The packed-FP32 z-streamed kernel (pairs (v0, v2), (v1, v3) in 64-bit
    registers) in every instantiated block shape: bit for bit against the
    oracle, with n not a multiple of the tile interior, several z segments
    and a shallower last launch (Poisson-3D: its f ring as well)."""
    if st == "poisson-3d":
        # the f ring (T + 2 planes) beside the state ring and the exchange rows
        # can exceed a CTA's 227 KB at the tallest tiles: a clean refusal
        try:
            ots.derive_geometry(stencil=st, n=132, steps=2 * T + 1, T=T, bx=bx, by=by, bz=1,
                                E=E, kernel="stream")
        except ots.OtsError as e:
            assert e.status_name == "SMEM_TOO_LARGE" and (T, E, bx * by) == (4, 2, 512), (T, E)
            return
    for n in (60, 132):  # several tiles with partial edge tiles, and z segments
        g = run_and_check(st, n, 2 * T + 1, T=T, bx=bx, by=by, bz=1, E=E, kernel="stream")
        assert g.kernel == ots.KERNEL_STREAM
        with ots.Plan(st, n, 2 * T + 1, T=T, bx=bx, by=by, bz=1, E=E,
                      kernel="stream") as plan:
            assert plan.describe()["Stream Arithmetic"] == "packed-fp32"
    # shapes without a packed instantiation, and n % 4 != 0, run the scalar kernel
    with ots.Plan(st, 60, 5, T=2, bx=32, by=8, bz=1, E=2, kernel="stream") as plan:
        assert plan.describe()["Stream Arithmetic"] == "scalar"
    try:
        with ots.Plan(st, 61, 5, T=T, bx=bx, by=by, bz=1, E=E, kernel="stream") as plan:
            assert plan.describe()["Stream Arithmetic"] == "scalar"
    except ots.OtsError as e:
        # beyond the scalar kernel's thread limit, or (Poisson: its f ring)
        # beyond a CTA's shared memory
        assert (e.status_name == "BLOCK_TOO_LARGE" and bx * by > 256) or \
            (e.status_name == "SMEM_TOO_LARGE" and st == "poisson-3d")


@pytest.mark.gpu
@pytest.mark.parametrize("n,steps,T,E,bx,by", [(132, 9, 4, 4, 16, 16), (96, 7, 3, 4, 16, 16),
                                               (64, 8, 4, 2, 16, 16), (36, 5, 2, 4, 8, 16),
                                               (200, 4, 3, 2, 16, 32), (4, 6, 4, 4, 16, 16),
                                               (97, 7, 3, 4, 16, 16)])
@pytest.mark.parametrize("st", ["jacobi-3d", "poisson-3d"])
def test_packed_and_scalar_stream_kernels_agree_bitwise(st, n, steps, T, E, bx, by):
    """stream_impl 0 (packed) and 1 (scalar) on the same plan shape: identical
    bits, and both equal to the oracle (the reference weight 0.143 too)."""
    outs = []
    for impl in (0, 1):
        try:
            plan = ots.Plan(st, n, steps, T=T, bx=bx, by=by, bz=1, E=E, kernel="stream",
                            impl=impl)
        except ots.OtsError as e:
            # the scalar kernel's Poisson f ring needs more shared memory than
            # the packed kernel's at the tallest tiles
            assert impl == 1 and st == "poisson-3d" and e.status_name == "SMEM_TOO_LARGE"
            continue
        with plan:
            state, aux = inputs(plan, seed=21)
            plan.upload(state, aux)
            plan.run()
            outs.append(plan.download()[0])
            g = plan.geometry
    want = O.sweep_f32(st, state, aux=aux, steps=steps, lo=g.padding,
                       hi=g.padding + g.real_size, coef=g.coef, h2=g.h2)[0]
    for o in outs:
        assert np.array_equal(o.view(np.uint32), want.view(np.uint32))
    if st == "jacobi-3d":
        run_and_check("jacobi-3d", 45, 6, T=3, bx=16, by=16, bz=1, E=4, kernel="stream",
                      variant=ots.VARIANT_REF)


# Fast-division variant (OTS_VARIANT_FAST): div.approx.ftz.f32 (2 ulp) and
# the approximate rsqrt in place of IEEE division / correctly rounded 1/sqrt.  Bound on
# max |gpu - cpu| / max(|cpu|, 1) against the IEEE FP32 oracle after the step
# counts used here (relative above 1, absolute below; these stencils' values
# lie in [0, 1) on the reference fill, so the bound is absolute).
FAST_TOL = {"rician-denoise-2d": 2e-4, "cdsc-tv-update-2d": 2e-4, "cs-3d": 2e-4}


@pytest.mark.gpu
@pytest.mark.parametrize("st,n,kw", [
    ("rician-denoise-2d", 130, dict(kernel="tile", T=2, bx=32, by=8, E=4)),
    ("rician-denoise-2d", 130, dict(kernel="plain")),
    ("rician-denoise-2d", 130, dict(kernel="stream", T=3, bx=32, by=1, E=1)),
    ("cdsc-tv-update-2d", 130, dict(kernel="tile", T=3, bx=16, by=16, E=2)),
    ("cdsc-tv-update-2d", 130, dict(kernel="plain")),
    ("cs-3d", 44, dict(kernel="tile", T=2, bx=16, by=8, bz=2, E=3)),
    ("cs-3d", 44, dict(kernel="plain")),
])
def test_fast_division_variant_within_tolerance(st, n, kw):
    steps = 8
    with ots.Plan(st, n, steps, device=0, variant=ots.VARIANT_FAST, **kw) as plan:
        assert plan.describe()["Variant"] == "fast"
        g = plan.geometry
        state, aux = inputs(plan, 31)
        plan.upload(state, aux)
        plan.run()
        got = plan.download()[0]
    lo, hi = g.padding, g.padding + g.real_size
    want = O.sweep_f32(st, state, aux=aux, steps=steps, lo=lo, hi=hi)[0]
    err = float(np.max(np.abs(got.astype(np.float64) - want) / np.maximum(np.abs(want), 1.0)))
    assert err <= FAST_TOL[st], (st, kw, err)
    # against FP64: within a small factor of the IEEE FP32 oracle's own error
    ref64 = O.sweep_f64(st, state, aux=aux, steps=steps, lo=lo, hi=hi)[0]
    sl = tuple(slice(lo, hi) for _ in range(g.dims))
    e_fast = float(np.max(np.abs(got[sl] - ref64[sl])))
    e_ieee = float(np.max(np.abs(want[sl] - ref64[sl])))
    assert e_fast <= max(10.0 * e_ieee, FAST_TOL[st]), (e_fast, e_ieee)


def test_fast_variant_refused_for_other_stencils():
    with pytest.raises(ots.OtsError) as ei:
        ots.derive_geometry(stencil="jacobi-2d", n=64, steps=4, variant=ots.VARIANT_FAST)
    assert ei.value.status_name == "INVALID_ARGUMENT"
