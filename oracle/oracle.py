"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs may
import this module; the engine never does.  It loads

  * ``oracle/_build/libots_oracle.so`` -- the C restatement (ots_oracle.c),
  * ``oracle/_ref/libots_ref.so``      -- the reference's own CPU loops,
    GeneratorParams derivations and input fills compiled by build_ref.py
    (optional: absent where the reference tree never was).

Arrays are numpy, in the reference's padded layout (P^d, x fastest).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libots_oracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libots_ref.so")

STENCILS = [
    "jacobi-1d", "jacobi-1d-5pt", "jacobi-1d-7pt", "jacobi-2d", "jacobi-3d",
    "poisson-2d", "poisson-3d", "gradient-2d", "gradient-3d", "fdtd-2d",
    "rician-denoise-2d", "cdsc-tv-update-2d", "cs-3d",
]
SID = {n: i for i, n in enumerate(STENCILS)}
VARIANT_BASELINE, VARIANT_REF = 0, 1

_F = ctypes.POINTER(ctypes.c_float)
_D = ctypes.POINTER(ctypes.c_double)


class Geometry(ctypes.Structure):
    _fields_ = [("dims", ctypes.c_int), ("padding", ctypes.c_int),
                ("padded_size", ctypes.c_int), ("real_size", ctypes.c_int),
                ("size_lcm", ctypes.c_int), ("comps", ctypes.c_int * 3),
                ("rpb", ctypes.c_int * 3), ("num_blocks", ctypes.c_int * 3),
                ("shared", ctypes.c_int * 3)]


_lib = None
_ref = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        for name in ("orc_dims", "orc_num_state", "orc_num_aux", "orc_radius", "orc_set_threads"):
            getattr(L, name).argtypes = [ctypes.c_int]
            getattr(L, name).restype = ctypes.c_int
        L.orc_default_coef.argtypes = [ctypes.c_int, ctypes.c_int]
        L.orc_default_coef.restype = ctypes.c_float
        L.orc_geometry_ref.argtypes = [ctypes.c_int] * 7 + [ctypes.POINTER(Geometry)]
        L.orc_fill_ref.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_uint, ctypes.POINTER(_F), ctypes.c_int]
        sweep_args = [ctypes.c_int] * 6 + [ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                           ctypes.c_int]
        L.orc_sweep_f32.argtypes = sweep_args + [ctypes.POINTER(_F), ctypes.POINTER(_F)]
        L.orc_sweep_f64.argtypes = sweep_args + [ctypes.POINTER(_D), ctypes.POINTER(_D)]
        L.orc_compare.argtypes = [ctypes.c_int] * 4 + [_F, _F, _D, _D]
        L.orc_compare.restype = ctypes.c_int
        L.orc_error_vs_f64.argtypes = [ctypes.c_int] * 4 + [_F, _D, ctypes.c_double, _D, _D]
        _lib = L
    return _lib


def ref_available():
    return os.path.exists(REF_PATH)


def ref():
    """The reference's own compiled CPU code (oracle/_ref/libots_ref.so)."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError("oracle/_ref/libots_ref.so not built (run oracle/build_ref.py "
                               "where the reference tree is present)")
        _ref = ctypes.CDLL(REF_PATH)
    return _ref


def dims(stencil):
    return lib().orc_dims(SID[stencil])


def num_state(stencil):
    return lib().orc_num_state(SID[stencil])


def num_aux(stencil):
    return lib().orc_num_aux(SID[stencil])


def radius(stencil):
    return lib().orc_radius(SID[stencil])


def set_threads(n):
    return lib().orc_set_threads(int(n))


def default_coef(stencil, variant=VARIANT_BASELINE):
    return lib().orc_default_coef(SID[stencil], variant)


def geometry_ref(stencil, n, T, bx, by=1, bz=1, E=1):
    g = Geometry()
    rc = lib().orc_geometry_ref(SID[stencil], n, T, bx, by, bz, E, ctypes.byref(g))
    return None if rc != 0 else g


def _fp(a):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_F)


def _dp(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def shape(d, P):
    return (P,) * d


def fill_ref(d, P, lo, hi, seed, nfields):
    arrs = [np.zeros(shape(d, P), np.float32) for _ in range(nfields)]
    ptrs = (_F * nfields)(*[_fp(a) for a in arrs])
    lib().orc_fill_ref(d, P, lo, hi, seed, ptrs, nfields)
    return arrs


def sweep_f32(stencil, state, aux=(), steps=1, lo=None, hi=None, variant=VARIANT_BASELINE,
              coef=0.0, h2=0.0, t0=0, padding=None):
    """Run `steps` reference sweeps in place on copies of `state`; returns the
    new state list.  Interior = [lo, hi) on every axis."""
    d = state[0].ndim
    P = state[0].shape[0]
    st = [np.ascontiguousarray(s, np.float32).copy() for s in state]
    ax = [np.ascontiguousarray(a, np.float32) for a in aux]
    sp = (_F * max(1, len(st)))(*[_fp(a) for a in st])
    apn = (_F * max(1, len(ax)))(*[_fp(a) for a in ax])
    lib().orc_sweep_f32(SID[stencil], variant, d, P, lo, hi, coef, h2, steps, t0, sp, apn)
    return st


def sweep_f64(stencil, state, aux=(), steps=1, lo=None, hi=None, variant=VARIANT_BASELINE,
              coef=0.0, h2=0.0, t0=0):
    d = state[0].ndim
    P = state[0].shape[0]
    st = [np.ascontiguousarray(s, np.float64).copy() for s in state]
    ax = [np.ascontiguousarray(a, np.float64) for a in aux]
    sp = (_D * max(1, len(st)))(*[_dp(a) for a in st])
    apn = (_D * max(1, len(ax)))(*[_dp(a) for a in ax])
    lib().orc_sweep_f64(SID[stencil], variant, d, P, lo, hi, coef, h2, steps, t0, sp, apn)
    return st


def compare(host, device, lo, hi):
    """compareResults: returns (passed, error_norm, ref_norm)."""
    e = ctypes.c_double()
    r = ctypes.c_double()
    h = np.ascontiguousarray(host, np.float32)
    dv = np.ascontiguousarray(device, np.float32)
    ok = lib().orc_compare(h.ndim, h.shape[0], lo, hi, _fp(h), _fp(dv), ctypes.byref(e),
                           ctypes.byref(r))
    return bool(ok), e.value, r.value


def error_vs_f64(got, ref64, lo, hi, floor=1e-30):
    mr = ctypes.c_double()
    rms = ctypes.c_double()
    g = np.ascontiguousarray(got, np.float32)
    r = np.ascontiguousarray(ref64, np.float64)
    lib().orc_error_vs_f64(g.ndim, g.shape[0], lo, hi, _fp(g), _dp(r), floor, ctypes.byref(mr),
                           ctypes.byref(rms))
    return mr.value, rms.value


# ---- the reference's own compiled code ---------------------------------

REF_LOOPS = {"jacobi-1d": "ref_jacobi_1d", "jacobi-1d-5pt": "ref_jacobi_1d_5pt",
             "jacobi-1d-7pt": "ref_jacobi_1d_7pt", "jacobi-2d": "ref_jacobi_2d",
             "poisson-2d": "ref_poisson_2d",
             "gradient-2d": "ref_gradient_2d"}


def ref_loop(stencil, data, padding, steps):
    """Run the reference runner's own CPU verification loop on `data`."""
    fn = getattr(ref(), REF_LOOPS[stencil])
    fn.argtypes = [_F, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    out = np.ascontiguousarray(data, np.float32).copy()
    fn(_fp(out), out.shape[0], padding, steps)
    return out


def ref_geometry(stencil, n, T, bx, by=1, bz=1, E=1):
    """The reference runner's own GeneratorParams::computeDerived; returns
    None where it throws/asserts, else a dict."""
    fn = getattr(ref(), "ref_geometry_" + stencil.replace("-", "_"))
    o = (ctypes.c_int * 16)()
    fn.argtypes = [ctypes.c_int] * 6 + [ctypes.POINTER(ctypes.c_int)]
    rc = fn(n, T, bx, by, bz, E, o)
    if rc != 0:
        return None
    keys = ["padding", "padded_size", "real_size", "size_lcm", "comps_x", "comps_y", "comps_z",
            "rpb_x", "rpb_y", "rpb_z", "num_blocks_x", "num_blocks_y", "num_blocks_z",
            "shared_x", "shared_y", "shared_z"]
    return dict(zip(keys, list(o)))


def ref_fill(which, P, padding, seed):
    """The reference's own enabled fill loops: which in {poisson_2d, fdtd_2d,
    cs_3d, jacobi_1d_5pt}."""
    d = {"poisson_2d": 2, "fdtd_2d": 2, "cs_3d": 3, "jacobi_1d_5pt": 1}[which]
    nf = 3 if which == "fdtd_2d" else 1
    arrs = [np.zeros(shape(d, P), np.float32) for _ in range(nf)]
    fn = getattr(ref(), "ref_fill_" + which)
    fn.argtypes = [_F] * nf + [ctypes.c_int, ctypes.c_int, ctypes.c_uint]
    fn(*[_fp(a) for a in arrs], P, padding, seed)
    return arrs


def ref_kernel_run(lib_path, fields, aux=(), T=1, steps=1, nb=(1, 1, 1), bs=(1, 1, 1)):
    """Run a reference-generated kernel compiled for the CPU by
    build_ref.build_kernel_case (the runner's launch loop over copies of
    `fields`, aux read-only in the runner's argument order); returns the
    final fields."""
    lib = ctypes.CDLL(lib_path)
    fn = lib.clk_run
    fn.argtypes = [ctypes.POINTER(_F), ctypes.POINTER(_F), ctypes.c_int, ctypes.c_int,
                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                   ctypes.POINTER(ctypes.c_int)]
    st = [np.ascontiguousarray(f, np.float32).copy() for f in fields]
    ax = [np.ascontiguousarray(a, np.float32) for a in aux]
    sp = (_F * len(st))(*[_fp(a) for a in st])
    apn = (_F * max(1, len(ax)))(*[_fp(a) for a in ax])
    nbc = (ctypes.c_int * 3)(*nb)
    bsc = (ctypes.c_int * 3)(*bs)
    fn(sp, apn, len(st), st[0].shape[0], st[0].ndim, T, steps, nbc, bsc)
    return st
