"""Known-answer tests for the oracle (CPU).  They cover the seven stencils
whose reference CPU check cannot pin the oracle (jacobi-3d, poisson-3d,
gradient-3d, fdtd-2d, rician-denoise-2d, cdsc-tv-update-2d, cs-3d) and
cross-check the FP32 and FP64 sweeps of all thirteen."""
import numpy as np
import pytest

import oracle as O


def _const(d, P, pad, value=1.0):
    a = np.zeros((P,) * d, np.float32)
    sl = tuple(slice(pad, P - pad) for _ in range(d))
    a[sl] = value
    return a


def _deep(d, P, pad, depth):
    return tuple(slice(pad + depth, P - pad - depth) for _ in range(d))


@pytest.mark.parametrize("st,coef", [("jacobi-2d", 0.0), ("jacobi-3d", 0.0)])
def test_constant_field_is_a_fixed_point_of_unit_weight_jacobi(st, coef):
    d = O.dims(st)
    P, pad, steps = (24, 2, 5) if d == 3 else (40, 2, 7)
    a = _const(d, P, pad)
    out = O.sweep_f32(st, [a], steps=steps, lo=pad, hi=P - pad, coef=coef)[0]
    # 1/5 * 5 and (float)(1/7) * 7 round to exactly 1.0f; the boundary's
    # influence travels one cell per step
    assert np.all(out[_deep(d, P, pad, steps)] == 1.0)
    assert out[(pad,) * d] < 1.0


def test_jacobi_3d_reference_weight_shrinks_constant():
    a = _const(3, 20, 2)
    out = O.sweep_f32("jacobi-3d", [a], steps=2, lo=2, hi=18, variant=O.VARIANT_REF)[0]
    inner = out[_deep(3, 20, 2, 2)]
    assert np.allclose(inner, np.float32(0.143) * 7 * np.float32(0.143) * 7, rtol=1e-6)


@pytest.mark.parametrize("st", ["poisson-2d", "poisson-3d"])
def test_reference_poisson_annihilates_affine_fields(st):
    d = O.dims(st)
    P, pad = (30, 2) if d == 2 else (14, 2)
    idx = np.indices((P,) * d).astype(np.float32)
    a = np.zeros((P,) * d, np.float32)
    sl = tuple(slice(pad, P - pad) for _ in range(d))
    a[sl] = (0.25 * idx[-1] + 0.5 * idx[0] + 1.0)[sl]
    out = O.sweep_f32(st, [a], steps=1, lo=pad, hi=P - pad, variant=O.VARIANT_REF)[0]
    assert np.max(np.abs(out[_deep(d, P, pad, 1)])) < 1e-4


@pytest.mark.parametrize("st", ["poisson-2d", "poisson-3d"])
def test_baseline_poisson_keeps_affine_field_with_zero_rhs(st):
    d = O.dims(st)
    P, pad = (30, 2) if d == 2 else (14, 2)
    idx = np.indices((P,) * d).astype(np.float32)
    a = np.zeros((P,) * d, np.float32)
    sl = tuple(slice(pad, P - pad) for _ in range(d))
    a[sl] = (0.125 * idx[-1] + 2.0)[sl]
    f = np.zeros_like(a)
    out = O.sweep_f32(st, [a], aux=[f], steps=1, lo=pad, hi=P - pad, h2=0.01)[0]
    deep = _deep(d, P, pad, 1)
    assert np.allclose(out[deep], a[deep], rtol=1e-6)


def test_baseline_poisson_rhs_enters_with_minus_h2():
    P, pad = 12, 2
    a = np.zeros((P, P), np.float32)
    f = np.zeros_like(a)
    f[6, 6] = 1.0
    out = O.sweep_f32("poisson-2d", [a], aux=[f], steps=1, lo=pad, hi=P - pad, h2=0.5)[0]
    assert out[6, 6] == np.float32(-0.125) and np.count_nonzero(out) == 1


@pytest.mark.parametrize("st", ["gradient-2d", "gradient-3d"])
def test_gradient_constant_field_gains_one_over_sqrt_eps(st):
    d = O.dims(st)
    P, pad = (20, 2) if d == 2 else (12, 2)
    a = _const(d, P, pad, 0.5)
    out = O.sweep_f32(st, [a], steps=1, lo=pad, hi=P - pad)[0]
    assert np.allclose(out[_deep(d, P, pad, 1)], 0.5 + 100.0, rtol=1e-6)


def test_fdtd_source_and_first_hz_response():
    P, pad = 16, 1
    z = [np.zeros((P, P), np.float32) for _ in range(3)]
    ex, ey, hz = O.sweep_f32("fdtd-2d", z, steps=2, lo=pad, hi=P - pad)
    # step 0 drives Ey row 0 to 0 (nothing moves); step 1 drives it to 1 and
    # Hz on row 0 answers -0.7 * (Ey(1) - Ey(0)) = 0.7
    assert np.all(ey[pad, pad:P - pad] == 1.0)
    assert np.allclose(hz[pad, pad:P - pad - 1], 0.7)
    assert np.all(ex == 0.0)
    assert np.all(hz[pad + 2:P - pad, :] == 0.0)


def test_fdtd_reference_variant_has_no_source():
    P, pad = 12, 1
    z = [np.zeros((P, P), np.float32) for _ in range(3)]
    out = O.sweep_f32("fdtd-2d", z, steps=3, lo=pad, hi=P - pad, variant=O.VARIANT_REF)
    assert all(np.all(o == 0) for o in out)


@pytest.mark.parametrize("st", ["rician-denoise-2d", "cdsc-tv-update-2d", "cs-3d"])
def test_smoothing_stencils_keep_constant_field(st):
    d = O.dims(st)
    P, pad = (20, 2) if d == 2 else (12, 2)
    a = _const(d, P, pad, 0.75)
    aux = [_const(d, P, pad, 0.75) for _ in range(O.num_aux(st))]
    if st == "cdsc-tv-update-2d":
        aux = [_const(d, P, pad, 0.75), _const(d, P, pad, 1.0)]  # F = u, V = 1
    out = O.sweep_f32(st, [a], aux=aux, steps=1, lo=pad, hi=P - pad)[0]
    assert np.allclose(out[_deep(d, P, pad, 2)], 0.75, rtol=1e-5)


@pytest.mark.parametrize("st", O.STENCILS)
def test_fp32_sweep_tracks_fp64_sweep(st):
    d = O.dims(st)
    P = {1: 120, 2: 30, 3: 14}[d]
    pad = 3
    arrs = O.fill_ref(d, P, pad, P - pad, 5, O.num_state(st) + O.num_aux(st))
    state, aux = arrs[:O.num_state(st)], arrs[O.num_state(st):]
    if st == "cdsc-tv-update-2d":
        aux[1] = np.where(aux[1] > 0, aux[1] + 0.5, 0).astype(np.float32)
    steps = 4
    h2 = 1e-3
    a32 = O.sweep_f32(st, state, aux=aux, steps=steps, lo=pad, hi=P - pad, h2=h2)
    a64 = O.sweep_f64(st, state, aux=aux, steps=steps, lo=pad, hi=P - pad, h2=h2)
    for x, y in zip(a32, a64):
        mr, rms = O.error_vs_f64(x, y, pad, P - pad, floor=1.0)
        assert mr < 1e-5, (st, mr)


@pytest.mark.parametrize("st", sorted(O.SID))
def test_thread_count_does_not_change_a_bit(st):
    """The oracle splits every phase by rows (1D: by chunks of the line) over
    its threads; each cell is computed the same way whatever the split, so one
    thread and several threads agree bit for bit, in FP32 and FP64.  Sizes
    cover several 1D chunks and uneven row splits."""
    d = O.dims(st)
    n = {1: 40000, 2: 97, 3: 23}[d]
    pad = 3
    P = n + 2 * pad
    ns = O.num_state(st)
    arrs = O.fill_ref(d, P, pad, P - pad, 17, ns + O.num_aux(st))
    state, aux = arrs[:ns], arrs[ns:]
    try:
        for sweep in (O.sweep_f32, O.sweep_f64):
            O.set_threads(1)
            one = sweep(st, state, aux, steps=4, lo=pad, hi=P - pad, h2=1e-4)
            O.set_threads(7)
            many = sweep(st, state, aux, steps=4, lo=pad, hi=P - pad, h2=1e-4)
            for a, b in zip(one, many):
                assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), (st, sweep.__name__)
    finally:
        O.set_threads(1)
