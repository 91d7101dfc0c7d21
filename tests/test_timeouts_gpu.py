"""Device-side failure detection without a GPU fault.

Every device wait of the library is bounded.  These tests make a wait run
out on purpose -- a flag that nothing ever sets -- with a short limit, and
check that the run reports OTS_ERR_TIMEOUT within about that limit and that
the same plan or batch then runs cleanly and matches the oracle:

* the batched engine: one grid's later chunks wait for a completion count
  that is never reached (ots_batch_debug_hold), in both item kinds;
* the 3D stream kernel: its first CTA arms the ring barrier of one plane but
  never loads that plane (ots_plan_debug_hold_plane), so the CTA gives up,
  drains the copies it still has in flight and leaves.
"""
import time

import numpy as np
import pytest

import oracle as O
import ots
from ots import OtsError
from ots import batch as B

from test_batch_gpu import GRIDS, check_same, oracle_run


def _batch_roundtrip(grids):
    b = B.Batch(grids)
    ins = B.inputs(grids, seed=11)
    try:
        b.set_wait_limit(0.05)
        b.debug_hold(0)
        for i, (s, a) in enumerate(ins):
            b.upload(i, s, a)
        t0 = time.time()
        with pytest.raises(OtsError) as ei:
            b.run()
        assert ei.value.status_name == "TIMEOUT"
        assert time.time() - t0 < 10.0
        # released: the same batch runs to completion and matches the oracle
        b.debug_hold(-1)
        for i, (s, a) in enumerate(ins):
            b.upload(i, s, a)
        b.run()
        for i, (g, (s, a)) in enumerate(zip(grids, ins)):
            check_same(g, b.download(i), oracle_run(g, s, a))
    finally:
        b.close()


@pytest.mark.gpu
def test_batch_dependency_wait_runs_out_then_batch_recovers():
    _batch_roundtrip([dict(g) for g in GRIDS])


@pytest.mark.gpu
def test_stream_batch_dependency_wait_runs_out_then_batch_recovers():
    grids = [dict(g) for g in GRIDS]
    B.pick_stream(grids, T=3)
    _batch_roundtrip(grids)


@pytest.mark.gpu
@pytest.mark.parametrize("stencil", ["jacobi-3d", "poisson-3d"])
def test_stream_kernel_ring_wait_runs_out_then_plan_recovers(stencil):
    n, steps = 40, 7
    with ots.Plan(stencil, n, steps, kernel="stream", T=3, bx=16, by=8, bz=1, E=2,
                  device=0) as plan:
        g = plan.geometry
        state, aux = plan.fill_reference(seed=5)
        plan.set_wait_limit(0.05)
        plan.debug_hold_plane(2)
        plan.upload(state, aux)
        t0 = time.time()
        with pytest.raises(OtsError) as ei:
            plan.run()
        assert ei.value.status_name == "TIMEOUT"
        assert time.time() - t0 < 10.0
        plan.debug_hold_plane(-1)
        plan.upload(state, aux)
        plan.run()
        got = plan.download()[0]
        want = O.sweep_f32(stencil, state, aux=aux, steps=steps, lo=g.padding,
                           hi=g.padding + g.real_size, coef=g.coef, h2=g.h2)[0]
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_wait_limit_argument_checks():
    # host-side checks only (no device work): limits outside (0, 60] s refused
    L = ots.lib()
    assert L.ots_plan_set_wait_limit(None, 1.0) == 1
    assert L.ots_plan_debug_hold_plane(None, 1) == 1
