"""Python host side of the overlapped time-tiling stencil engine.

A thin ctypes mirror of the C ABI in include/ots.h (libots.so, built in-tree
next to this package).  The call sequence mirrors one reference runner
(opencl/jacobi-2d/jacobi-2d.cpp:553-1048):

    plan = Plan(stencil="jacobi-2d", n=2048, steps=64, T=4, bx=16, by=16, E=1)
    state, aux = plan.fill_reference(seed=123456)   # srand/rand fill
    plan.upload(state, aux)                         # enqueueWriteBuffer
    timing = plan.run()                             # launch loop + events
    out = plan.download()                           # enqueueReadBuffer
    plan.describe()                                 # printProgramParameters keys

Arrays are numpy float32 in the reference layout (P^d, x fastest, interior at
[padding, padding + real_size) on every axis, zero ring).  Errors raise
OtsError carrying the library's status and message.  There is no CPU path:
if libots.so is missing the import fails.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "libots.so")

STENCILS = [
    "jacobi-1d", "jacobi-1d-5pt", "jacobi-1d-7pt", "jacobi-2d", "jacobi-3d",
    "poisson-2d", "poisson-3d", "gradient-2d", "gradient-3d", "fdtd-2d",
    "rician-denoise-2d", "cdsc-tv-update-2d", "cs-3d",
]
SID = {n: i for i, n in enumerate(STENCILS)}

ENGINE_NATIVE, ENGINE_COMPAT = 0, 1
KERNEL_AUTO, KERNEL_TILE, KERNEL_STREAM, KERNEL_PLAIN, KERNEL_TEX = 0, 1, 2, 3, 4
KERNELS = {"auto": 0, "tile": 1, "stream": 2, "plain": 3, "tex": 4}
VARIANT_BASELINE, VARIANT_REF, VARIANT_FAST = 0, 1, 2

STATUS = {0: "OK", 1: "INVALID_ARGUMENT", 2: "INVALID_GEOMETRY", 3: "SMEM_TOO_LARGE",
          4: "BLOCK_TOO_LARGE", 5: "CUDA", 6: "TIMEOUT", 7: "UNSUPPORTED", 8: "NO_DEVICE",
          9: "OUT_OF_MEMORY"}


class OtsError(RuntimeError):
    def __init__(self, status, message):
        self.status = status
        self.status_name = STATUS.get(status, str(status))
        super().__init__("%s: %s" % (self.status_name, message))


class Params(ctypes.Structure):
    _fields_ = [("stencil", ctypes.c_int32), ("problem_size", ctypes.c_int32),
                ("time_steps", ctypes.c_int32), ("time_tile", ctypes.c_int32),
                ("block_x", ctypes.c_int32), ("block_y", ctypes.c_int32),
                ("block_z", ctypes.c_int32), ("elements_per_thread", ctypes.c_int32),
                ("engine", ctypes.c_int32), ("kernel", ctypes.c_int32),
                ("variant", ctypes.c_int32), ("phase_limit", ctypes.c_int32),
                ("coef", ctypes.c_float), ("h2", ctypes.c_float), ("device", ctypes.c_int32),
                ("cluster_y", ctypes.c_int32), ("stream_impl", ctypes.c_int32),
                ("reserved", ctypes.c_int32 * 5)]


class Geometry(ctypes.Structure):
    _fields_ = [("dims", ctypes.c_int32), ("radius", ctypes.c_int32),
                ("num_fields", ctypes.c_int32), ("num_aux", ctypes.c_int32),
                ("padding", ctypes.c_int32), ("padded_size", ctypes.c_int32),
                ("real_size", ctypes.c_int32), ("size_lcm", ctypes.c_int32),
                ("comps", ctypes.c_int32 * 3), ("real_per_block", ctypes.c_int32 * 3),
                ("num_blocks", ctypes.c_int32 * 3), ("shared_size", ctypes.c_int32 * 3),
                ("threads", ctypes.c_int32 * 3), ("kernel", ctypes.c_int32),
                ("e_axis", ctypes.c_int32), ("launches", ctypes.c_int32),
                ("registers", ctypes.c_int32), ("shared_bytes", ctypes.c_int64),
                ("interior_points", ctypes.c_int64), ("flops_per_point", ctypes.c_double),
                ("useful_ratio", ctypes.c_double), ("coef", ctypes.c_float),
                ("h2", ctypes.c_float), ("ctas_per_sm", ctypes.c_int32),
                ("sm_count", ctypes.c_int32)]

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


class Timing(ctypes.Structure):
    _fields_ = [("event_ms", ctypes.c_double), ("wall_s", ctypes.c_double),
                ("launches", ctypes.c_int32), ("steps", ctypes.c_int32)]


_FP = ctypes.POINTER(ctypes.c_float)
_lib = None


def lib():
    """Load libots.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libots.so not found at %s: build it with "
                          "`python -c 'import __graft_entry__ as g; g.build()'`" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    st = ctypes.c_int
    L.ots_last_error.restype = ctypes.c_char_p
    L.ots_status_string.restype = ctypes.c_char_p
    L.ots_status_string.argtypes = [ctypes.c_int]
    L.ots_device_info.argtypes = [ctypes.c_int32, ctypes.c_char_p, ctypes.c_size_t,
                                  ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int64),
                                  ctypes.POINTER(ctypes.c_int64)]
    L.ots_device_info.restype = st
    L.ots_stencil_name.restype = ctypes.c_char_p
    L.ots_stencil_name.argtypes = [ctypes.c_int32]
    L.ots_stencil_from_name.argtypes = [ctypes.c_char_p]
    for fn in ("ots_stencil_dims", "ots_stencil_num_fields", "ots_stencil_num_aux"):
        getattr(L, fn).argtypes = [ctypes.c_int32]
        getattr(L, fn).restype = ctypes.c_int32
    L.ots_stencil_model_constants.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]
    L.ots_stencil_model_constants.restype = st
    L.ots_fill_reference.argtypes = [ctypes.c_int32] * 4 + [ctypes.c_uint32,
                                                            ctypes.POINTER(_FP), ctypes.c_int32]
    L.ots_fill_reference.restype = st
    L.ots_plan_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(ctypes.c_void_p)]
    L.ots_plan_create.restype = st
    L.ots_plan_destroy.argtypes = [ctypes.c_void_p]
    L.ots_plan_destroy.restype = None
    L.ots_plan_geometry.argtypes = [ctypes.c_void_p, ctypes.POINTER(Geometry)]
    L.ots_plan_geometry.restype = st
    L.ots_derive_geometry.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(Geometry)]
    L.ots_derive_geometry.restype = st
    for fn in ("ots_upload", "ots_upload_interior", "ots_upload_async",
               "ots_upload_interior_async"):
        getattr(L, fn).argtypes = [ctypes.c_void_p, ctypes.POINTER(_FP), ctypes.POINTER(_FP)]
        getattr(L, fn).restype = st
    for fn in ("ots_download", "ots_download_interior", "ots_download_async",
               "ots_download_interior_async"):
        getattr(L, fn).argtypes = [ctypes.c_void_p, ctypes.POINTER(_FP)]
        getattr(L, fn).restype = st
    L.ots_run.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(Timing)]
    L.ots_run.restype = st
    L.ots_run_async.argtypes = [ctypes.c_void_p, ctypes.c_int32]
    L.ots_run_async.restype = st
    L.ots_sync.argtypes = [ctypes.c_void_p]
    L.ots_sync.restype = st
    L.KV = ctypes.CFUNCTYPE(None, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_void_p)
    L.ots_describe.argtypes = [ctypes.c_void_p, L.KV, ctypes.c_void_p]
    L.ots_describe.restype = st
    for fn in ("ots_plan_device_state", "ots_plan_device_aux"):
        getattr(L, fn).argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]
        getattr(L, fn).restype = st
    L.ots_plan_stream.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    L.ots_plan_stream.restype = st
    L.ots_plan_enable_clocks.argtypes = [ctypes.c_void_p, ctypes.c_int32]
    L.ots_plan_enable_clocks.restype = st
    L.ots_plan_clock_records.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                         ctypes.POINTER(ctypes.c_int64)]
    L.ots_plan_clock_records.restype = st
    L.ots_plan_set_wait_limit.argtypes = [ctypes.c_void_p, ctypes.c_double]
    L.ots_plan_set_wait_limit.restype = st
    L.ots_plan_debug_hold_plane.argtypes = [ctypes.c_void_p, ctypes.c_int32]
    L.ots_plan_debug_hold_plane.restype = st
    L.ots_host_register.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
    L.ots_host_register.restype = st
    L.ots_host_unregister.argtypes = [ctypes.c_void_p]
    L.ots_host_unregister.restype = st
    _lib = L
    return L


def check(status):
    if status != 0:
        raise OtsError(status, lib().ots_last_error().decode())


def _fptrs(arrays):
    for a in arrays:
        if a.dtype != np.float32 or not a.flags.c_contiguous:
            raise ValueError("arrays must be C-contiguous float32")
    return (_FP * max(1, len(arrays)))(*[a.ctypes.data_as(_FP) for a in arrays])


def make_params(stencil, n, steps, T=1, bx=16, by=16, bz=1, E=1, engine=ENGINE_NATIVE,
                kernel=KERNEL_AUTO, variant=VARIANT_BASELINE, phase_limit=0, coef=0.0, h2=0.0,
                device=0, cy=1, impl=0):
    p = Params()
    p.stencil = SID[stencil] if isinstance(stencil, str) else int(stencil)
    p.problem_size, p.time_steps, p.time_tile = n, steps, T
    p.block_x, p.block_y, p.block_z, p.elements_per_thread = bx, by, bz, E
    p.engine = engine
    p.kernel = KERNELS[kernel] if isinstance(kernel, str) else kernel
    p.variant, p.phase_limit, p.coef, p.h2, p.device = variant, phase_limit, coef, h2, device
    p.cluster_y = cy
    p.stream_impl = impl
    return p


MODEL_CONSTANT_KEYS = ("phase2_global_loads", "phase2_shared_loads", "compute_per_point",
                       "phase3_shared_loads", "phase4_global_stores", "shared_stores",
                       "num_fields", "data_size")


def model_constants(stencil):
    """The runner's printed performance-model constants (dict), or None for
    the runners that print none."""
    sid = SID[stencil] if isinstance(stencil, str) else int(stencil)
    out = (ctypes.c_double * 8)()
    st = lib().ots_stencil_model_constants(sid, out)
    if st != 0:
        return None
    return dict(zip(MODEL_CONSTANT_KEYS, list(out)))


def derive_geometry(**kw):
    g = Geometry()
    check(lib().ots_derive_geometry(ctypes.byref(make_params(**kw)), ctypes.byref(g)))
    return g


def fill_disks(n, seed=2012, count=64, background=0.1, sigma=0.05):
    """(clean, noisy) n x n float32 images: ots_fill_disks (the Rician / TV
    workloads' input)."""
    noisy = np.zeros((n, n), np.float32)
    clean = np.zeros((n, n), np.float32)
    L = lib()
    fn = L.ots_fill_disks
    fn.argtypes = [ctypes.c_int32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_float,
                   ctypes.c_float, _FP, _FP]
    fn.restype = ctypes.c_int
    check(fn(n, seed, count, background, sigma, noisy.ctypes.data_as(_FP),
             clean.ctypes.data_as(_FP)))
    return clean, noisy


def fill_reference(dims, P, padding, real_size, seed, nfields):
    arrs = [np.zeros((P,) * dims, np.float32) for _ in range(nfields)]
    check(lib().ots_fill_reference(dims, P, padding, real_size, seed, _fptrs(arrs), nfields))
    return arrs


def device_info(device=0):
    name = ctypes.create_string_buffer(256)
    sms = ctypes.c_int32()
    smem = ctypes.c_int64()
    mem = ctypes.c_int64()
    check(lib().ots_device_info(device, name, 256, ctypes.byref(sms), ctypes.byref(smem),
                                ctypes.byref(mem)))
    return {"name": name.value.decode(), "sm_count": sms.value, "smem_per_block": smem.value,
            "global_mem": mem.value}


class Plan:
    """One stencil problem on one GPU (ots_plan_create ... ots_plan_destroy)."""

    def __init__(self, stencil, n, steps, **kw):
        self.params = make_params(stencil, n, steps, **kw)
        self.stencil = STENCILS[self.params.stencil]
        h = ctypes.c_void_p()
        check(lib().ots_plan_create(ctypes.byref(self.params), ctypes.byref(h)))
        self.handle = h
        g = Geometry()
        check(lib().ots_plan_geometry(self.handle, ctypes.byref(g)))
        self.geometry = g

    def close(self):
        if getattr(self, "handle", None):
            lib().ots_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def dims(self):
        return self.geometry.dims

    @property
    def padded_shape(self):
        return (self.geometry.padded_size,) * self.geometry.dims

    def fill_reference(self, seed=123456):
        g = self.geometry
        arrs = fill_reference(g.dims, g.padded_size, g.padding, g.real_size, seed,
                              g.num_fields + g.num_aux)
        return arrs[:g.num_fields], arrs[g.num_fields:]

    @property
    def interior_shape(self):
        return (self.geometry.real_size,) * self.geometry.dims

    def _checked(self, arrays, count, shape, what):
        arrs = [np.ascontiguousarray(a, np.float32) for a in arrays]
        if len(arrs) != count:
            raise ValueError("%s: expected %d arrays, got %d" % (what, count, len(arrs)))
        for a in arrs:
            if a.shape != shape:
                raise ValueError("%s: array shape %s, plan needs %s" % (what, a.shape, shape))
        return arrs

    def upload(self, state, aux=()):
        g = self.geometry
        st = self._checked(state, g.num_fields, self.padded_shape, "state")
        ax = self._checked(aux, g.num_aux, self.padded_shape, "aux")
        check(lib().ots_upload(self.handle, _fptrs(st), _fptrs(ax) if ax else None))

    def upload_interior(self, state, aux=()):
        g = self.geometry
        st = self._checked(state, g.num_fields, self.interior_shape, "state")
        ax = self._checked(aux, g.num_aux, self.interior_shape, "aux")
        check(lib().ots_upload_interior(self.handle, _fptrs(st), _fptrs(ax) if ax else None))

    def upload_interior_async(self, state, aux=()):
        """Enqueue the upload and return; the arrays (C-contiguous float32,
        ideally page-locked) must stay alive and unchanged until sync()."""
        g = self.geometry
        st = self._checked(state, g.num_fields, self.interior_shape, "state")
        ax = self._checked(aux, g.num_aux, self.interior_shape, "aux")
        if any(a is not b for a, b in zip(st, state)) or any(a is not b for a, b in zip(ax, aux)):
            raise ValueError("upload_interior_async: arrays must already be C-contiguous float32")
        check(lib().ots_upload_interior_async(self.handle, _fptrs(st), _fptrs(ax) if ax else None))

    def download_interior_async(self, out):
        """Enqueue the copy of the current state into `out` and return; valid
        after sync()."""
        g = self.geometry
        for a in out:
            if a.shape != self.interior_shape or a.dtype != np.float32 or not a.flags.c_contiguous:
                raise ValueError("download: need C-contiguous float32 %s" % (self.interior_shape,))
        if len(out) != g.num_fields:
            raise ValueError("download: expected %d arrays" % g.num_fields)
        check(lib().ots_download_interior_async(self.handle, _fptrs(out)))

    def run(self, kernel=KERNEL_AUTO):
        t = Timing()
        k = KERNELS[kernel] if isinstance(kernel, str) else kernel
        check(lib().ots_run(self.handle, k, ctypes.byref(t)))
        return t

    def run_async(self, kernel=KERNEL_AUTO):
        k = KERNELS[kernel] if isinstance(kernel, str) else kernel
        check(lib().ots_run_async(self.handle, k))

    def sync(self):
        check(lib().ots_sync(self.handle))

    def download(self, out=None):
        g = self.geometry
        if out is None:
            out = [np.zeros(self.padded_shape, np.float32) for _ in range(g.num_fields)]
        for a in out:
            if a.shape != self.padded_shape or a.dtype != np.float32 or not a.flags.c_contiguous:
                raise ValueError("download: need C-contiguous float32 %s" % (self.padded_shape,))
        if len(out) != g.num_fields:
            raise ValueError("download: expected %d arrays" % g.num_fields)
        check(lib().ots_download(self.handle, _fptrs(out)))
        return out

    def download_interior(self, out=None):
        g = self.geometry
        if out is None:
            out = [np.zeros(self.interior_shape, np.float32) for _ in range(g.num_fields)]
        for a in out:
            if a.shape != self.interior_shape or a.dtype != np.float32 or not a.flags.c_contiguous:
                raise ValueError("download: need C-contiguous float32 %s" % (self.interior_shape,))
        if len(out) != g.num_fields:
            raise ValueError("download: expected %d arrays" % g.num_fields)
        check(lib().ots_download_interior(self.handle, _fptrs(out)))
        return out

    def describe(self):
        kv = {}

        def cb(k, v, _):
            kv[k.decode()] = v.decode()

        f = lib().KV(cb)
        check(lib().ots_describe(self.handle, f, None))
        return kv

    def device_state_ptr(self, field=0):
        p = ctypes.c_void_p()
        check(lib().ots_plan_device_state(self.handle, field, ctypes.byref(p)))
        return p.value

    def enable_clocks(self, enable=True):
        """Record per-warp phase clocks of tile-kernel launches (-c)."""
        check(lib().ots_plan_enable_clocks(self.handle, 1 if enable else 0))

    def clock_records(self):
        """The last tile-kernel launch's records: a structured array with
        block_x, block_y, block_z, warp, sm and clock[5]."""
        import numpy as _np
        dt = _np.dtype([("block_x", "<u4"), ("block_y", "<u4"), ("block_z", "<u4"),
                        ("warp", "<u4"), ("sm", "<u4"), ("clock", "<u4", (5,))])
        n = ctypes.c_int64()
        check(lib().ots_plan_clock_records(self.handle, None, 0, ctypes.byref(n)))
        out = _np.zeros(n.value, dt)
        if n.value:
            check(lib().ots_plan_clock_records(self.handle, out.ctypes.data, n.value,
                                               ctypes.byref(n)))
        return out

    def set_wait_limit(self, seconds):
        """Limit of the 3D stream kernel's bounded device waits (2 s default)."""
        check(lib().ots_plan_set_wait_limit(self.handle, float(seconds)))

    def debug_hold_plane(self, plane):
        """Test hook: the first CTA never loads this running plane, so its
        wait runs out (the run reports TIMEOUT); -1 turns it off."""
        check(lib().ots_plan_debug_hold_plane(self.handle, int(plane)))

    def stream_ptr(self):
        p = ctypes.c_void_p()
        check(lib().ots_plan_stream(self.handle, ctypes.byref(p)))
        return p.value
