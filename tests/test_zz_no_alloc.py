"""Allocation-free cost-model inference: ots_mlp_predict_noalloc.

Some callers of the configuration picker cannot call cudaMalloc at the
moment they ask for a prediction -- an application that hands out all device
memory from its own pool and lets no library allocate behind its back.
ots_mlp_predict_noalloc serves them from a
fixed 2 MiB array compiled into libots: the caller passes device input and
output buffers and a stream, and the call allocates nothing.

This file is named to run after every other test file; it checks the new
entry point against the regular ots_mlp_predict on two calls in a row (the
second with different, larger input, so nothing may carry over from the
first) and that requests beyond the fixed array are refused.
"""
import ctypes

import numpy as np
import pytest

import ots
from ots import model


def _noalloc():
    L = model._mlp_lib()
    fn = L.ots_mlp_predict_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                   ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


@pytest.mark.gpu
def test_noalloc_inference_matches_regular_inference_on_two_calls():
    import torch
    fn = _noalloc()
    rng = np.random.default_rng(17)
    n_in = len(model.FEATURES)
    m = model.MLP(n_in, 64, 3, seed=23)
    Xfit = rng.normal(0, 3, (512, n_in)).astype(np.float32)
    yfit = rng.normal(5, 2, 512).astype(np.float32)
    m.fit_normalization(Xfit, yfit)
    m.fit(Xfit, yfit, epochs=20, batch=64, seed=1)
    stream = torch.cuda.current_stream()
    for n in (1000, 4096):
        X = rng.normal(0, 3, (n, n_in)).astype(np.float32)
        want = m.predict(X)
        dX = torch.from_numpy(X).cuda()
        dy = torch.full((n,), float("nan"), device="cuda")
        ots.check(fn(m.h, dX.data_ptr(), n, dy.data_ptr(), stream.cuda_stream))
        torch.cuda.synchronize()
        got = dy.cpu().numpy()
        # the same kernels in the same order: agreement to rounding noise
        assert np.allclose(got, want, rtol=1e-6, atol=1e-6), float(np.max(np.abs(got - want)))
    m.close()


@pytest.mark.gpu
def test_noalloc_inference_refuses_requests_beyond_its_fixed_array():
    import torch
    fn = _noalloc()
    n_in = len(model.FEATURES)
    m = model.MLP(n_in, 64, 3, seed=3)
    dX = torch.zeros((4097, n_in), device="cuda")
    dy = torch.zeros((4097,), device="cuda")
    st = fn(m.h, dX.data_ptr(), 4097, dy.data_ptr(), None)
    assert ots.STATUS[st] == "INVALID_ARGUMENT"
    assert "4096" in ots.lib().ots_last_error().decode()
    wide = model.MLP(n_in, 128, 3, seed=3)
    st = fn(wide.h, dX.data_ptr(), 10, dy.data_ptr(), None)
    assert ots.STATUS[st] == "UNSUPPORTED"
    m.close()
    wide.close()
