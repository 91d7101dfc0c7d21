"""Full-size oracle parity: the measured workloads at their stated sizes,
GPU result against the CPU oracle after the full step count.

  jacobi-3d   512^3 x 100  packed stream kernel (the tuned headline config)  bit for bit
  poisson-3d  512^3 x 100  packed stream kernel, RHS f = 2u - 1, h = 1/511   bit for bit
  fdtd-2d    4096^2 x 500  two-phase y-streamed kernel, source row          bit for bit
  rician     4096^2 x 200  two-phase tile and y-streamed kernels, disk image within bound
  tv         4096^2 x 200  plain kernel, disk image, V = 1                  within bound
  rician, tv (fast-division variant), the workloads' best configurations     within bound

The linear stencils must match bit for bit (-fmad=false, the oracle's operand
order).  Rician and TV take 1/sqrt with the GPU's rsqrtf (as the reference
kernels took OpenCL rsqrt) against a correctly rounded 1/sqrt on the CPU;
over 200 steps their results drift apart where g = 1/sqrt(eps + |grad u|^2)
is huge (flat regions of the image).  Their bound is the reference's own
check (compareResults, opencl/jacobi-2d/jacobi-2d.cpp:517-551: relative L2
error <= 1e-2) plus a maximum ABSOLUTE difference of 2e-2 (the images lie in
[0, 1.3]).  The fast-division variant (approximate division and rsqrt, the
latitude the reference's OpenCL build gave its kernels) is held to the same
relative-L2 check and a maximum absolute difference of 3e-2 against the IEEE
oracle.  The oracle runs on all host threads (a few tens of seconds).
"""
import json
import os

import numpy as np
import pytest

import oracle as O
import ots
from ots import workloads as W

TUNED = json.load(open(os.path.join(os.path.dirname(ots.__file__), "tuned.json")))


def _run(stencil, n, steps, cfg, variant=ots.VARIANT_BASELINE, fast=False):
    w = dict(stencil=stencil, n=n, steps=steps)
    if fast:  # the GPU in the fast-division variant, the oracle in IEEE
        w["variant"] = "fast"
    g, pst, pax, got = W.run_config(w, cfg)
    O.set_threads(os.cpu_count() or 1)
    lo, hi = g.padding, g.padding + g.real_size
    want = O.sweep_f32(stencil, pst, pax, steps=steps, lo=lo, hi=hi, coef=g.coef, h2=g.h2,
                       variant=variant)
    sl = tuple(slice(lo, hi) for _ in range(g.dims))
    return [a[sl] for a in got], [b[sl] for b in want]


def _bitwise(got, want):
    for f, (a, b) in enumerate(zip(got, want)):
        bad = int(np.count_nonzero(a.view(np.uint32) != b.view(np.uint32)))
        assert bad == 0, "field %d: %d cells differ (max |d| %g)" % (
            f, bad, float(np.max(np.abs(a.astype(np.float64) - b))))


@pytest.mark.gpu
def test_jacobi3d_512_100_headline_config_bitwise():
    c = TUNED["jacobi-3d/512/100"]
    cfg = {k: c[k] for k in ("kernel", "T", "bx", "by", "bz", "E")}
    got, want = _run("jacobi-3d", 512, 100, cfg)
    _bitwise(got, want)
    assert 0.0 < float(got[0].mean()) < 1.0


@pytest.mark.gpu
def test_poisson3d_512_100_bitwise():
    got, want = _run("poisson-3d", 512, 100, dict(kernel="stream", T=3, bx=16, by=16, bz=1, E=4))
    _bitwise(got, want)


@pytest.mark.gpu
def test_fdtd2d_4096_500_bitwise():
    got, want = _run("fdtd-2d", 4096, 500, dict(kernel="stream", T=5, bx=32, by=1, bz=1, E=1))
    _bitwise(got, want)


def _within_reference_check(got, want, max_abs):
    a, b = got[0].astype(np.float64), want[0].astype(np.float64)
    rel_l2 = float(np.sqrt(np.sum((a - b) ** 2)) / np.sqrt(np.sum(b ** 2)))
    mx = float(np.max(np.abs(a - b)))
    assert rel_l2 <= 1e-2 and mx <= max_abs, (rel_l2, mx)
    return rel_l2, mx


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", [dict(kernel="tile", T=2, bx=64, by=4, bz=1, E=8),
                                 dict(kernel="stream", T=1, bx=32, by=16, bz=1, E=1)],
                         ids=["tile", "stream"])
def test_rician_4096_200_within_reference_check(cfg):
    got, want = _run("rician-denoise-2d", 4096, 200, cfg)
    _within_reference_check(got, want, 2e-2)


@pytest.mark.gpu
@pytest.mark.parametrize("st,cfg", [
    ("rician-denoise-2d", dict(kernel="stream", T=2, bx=32, by=64, bz=1, E=1)),
    ("cdsc-tv-update-2d", dict(kernel="plain", T=1, bx=32, by=8, bz=1, E=1))])
def test_fast_division_4096_200_within_reference_check(st, cfg):
    got, want = _run(st, 4096, 200, cfg, fast=True)
    _within_reference_check(got, want, 3e-2)


@pytest.mark.gpu
def test_tv_4096_200_within_reference_check():
    got, want = _run("cdsc-tv-update-2d", 4096, 200, dict(kernel="plain", T=1, bx=32, by=8, bz=1, E=1))
    _within_reference_check(got, want, 2e-2)
