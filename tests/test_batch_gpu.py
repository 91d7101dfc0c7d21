"""Batched engine (GPU): every grid of one persistent launch equals its own
CPU oracle run and the sequential comparators bit for bit."""
import numpy as np
import pytest

import oracle as O
from ots import OtsError
from ots import batch as B

GRIDS = [
    dict(stencil="jacobi-2d", n=130, steps=25, T=4, bx=32, E=2),
    dict(stencil="poisson-2d", n=67, steps=9, T=3, bx=16, E=4),
    dict(stencil="gradient-2d", n=45, steps=7, T=2, bx=64, E=1),
    dict(stencil="jacobi-2d", n=17, steps=30, T=8, bx=64, E=4),
    dict(stencil="poisson-2d", n=100, steps=1, T=5, bx=32, E=2),
    dict(stencil="jacobi-2d", n=64, steps=0, T=2, bx=16, E=2),
    dict(stencil="gradient-2d", n=90, steps=12, T=4, bx=32, E=4),
    dict(stencil="jacobi-2d", n=200, steps=16, T=1, bx=16, E=1),
]


def oracle_run(g, state, aux):
    n = g["n"]
    P = n + 2
    s = np.zeros((P, P), np.float32)
    s[1:-1, 1:-1] = state
    ax = []
    h2 = 0.0
    if g["stencil"] == "poisson-2d":
        a = np.zeros((P, P), np.float32)
        a[1:-1, 1:-1] = aux
        ax = [a]
        h2 = float(np.float32((1.0 / (n - 1)) ** 2))
    out = O.sweep_f32(g["stencil"], [s], aux=ax, steps=g["steps"], lo=1, hi=P - 1, h2=h2)[0]
    return out[1:-1, 1:-1]


def check_same(g, got, want):
    if g["stencil"] == "gradient-2d":
        # rsqrtf on the GPU against the oracle's correctly rounded 1/sqrt: the
        # difference accumulates with the step count
        err = np.max(np.abs(got.astype(np.float64) - want) / np.maximum(np.abs(want), 1.0))
        assert err <= 1e-4 * max(1.0, g["steps"] / 8.0), (g, err)
    else:
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), g


@pytest.mark.gpu
def test_batched_grids_match_oracle_and_sequential_runs():
    grids = [dict(g) for g in GRIDS]
    b = B.Batch(grids)
    ins = B.inputs(grids, seed=3)
    for i, (s, a) in enumerate(ins):
        b.upload(i, s, a)
    b.run()
    got = [b.download(i) for i in range(len(grids))]
    for g, (s, a), x in zip(grids, ins, got):
        check_same(g, x, oracle_run(g, s, a))
    for kind in ("tile", "plain"):
        for i, (s, a) in enumerate(ins):
            b.upload(i, s, a)
        b.run_sequential(kind)
        for i, g in enumerate(grids):
            y = b.download(i)
            assert np.array_equal(y.view(np.uint32), got[i].view(np.uint32)), (kind, g)
    # a second graph launch from the same inputs gives the same bits
    for i, (s, a) in enumerate(ins):
        b.upload(i, s, a)
    b.run()
    for i in range(len(grids)):
        assert np.array_equal(b.download(i), got[i])
    b.close()


@pytest.mark.gpu
def test_batch_rejects_unsupported_grids():
    with pytest.raises(OtsError) as ei:
        B.Batch([dict(stencil="fdtd-2d", n=32, steps=4, T=2, bx=32, E=2)])
    assert ei.value.status_name == "UNSUPPORTED"
    with pytest.raises(OtsError) as ei:
        B.Batch([dict(stencil="jacobi-2d", n=32, steps=4, T=2, bx=8, E=2)])
    assert ei.value.status_name == "UNSUPPORTED"
    with pytest.raises(OtsError) as ei:
        B.Batch([dict(stencil="jacobi-2d", n=32, steps=4, T=4, bx=64, E=1)])
    assert ei.value.status_name == "INVALID_GEOMETRY"


@pytest.mark.gpu
def test_workload_generator_matches_the_batched_definition():
    w = B.workload(256, 2012)
    assert len(w) == 256
    assert {g["stencil"] for g in w} == set(B.BATCH_STENCILS)
    assert all(64 <= g["n"] <= 2048 and 8 <= g["steps"] <= 256 for g in w)


STREAM_GRIDS = [
    dict(stencil="jacobi-2d", n=300, steps=25, T=4, by=1),
    dict(stencil="poisson-2d", n=67, steps=9, T=3, by=16),
    dict(stencil="gradient-2d", n=245, steps=7, T=2, by=40),
    dict(stencil="jacobi-2d", n=17, steps=30, T=4, by=1),
    dict(stencil="poisson-2d", n=130, steps=1, T=4, by=1),
    dict(stencil="jacobi-2d", n=64, steps=0, T=2, by=1),
    dict(stencil="gradient-2d", n=90, steps=13, T=4, by=8),
    dict(stencil="jacobi-2d", n=200, steps=16, T=1, by=1),
]


@pytest.mark.gpu
def test_batched_stream_items_match_oracle_and_sequential_runs():
    # warp items of the y-streamed kernel, last chunks shallower than T,
    # segment lengths from the library default and from block_y
    grids = [dict(g, kernel="stream") for g in STREAM_GRIDS]
    b = B.Batch(grids)
    ins = B.inputs(grids, seed=5)
    for i, (s, a) in enumerate(ins):
        b.upload(i, s, a)
    b.run()
    got = [b.download(i) for i in range(len(grids))]
    for g, (s, a), x in zip(grids, ins, got):
        check_same(g, x, oracle_run(g, s, a))
    for kind in ("stream", "plain"):
        for i, (s, a) in enumerate(ins):
            b.upload(i, s, a)
        b.run_sequential(kind)
        for i, g in enumerate(grids):
            y = b.download(i)
            assert np.array_equal(y.view(np.uint32), got[i].view(np.uint32)), (kind, g)
    for i, (s, a) in enumerate(ins):
        b.upload(i, s, a)
    b.run()
    for i in range(len(grids)):
        assert np.array_equal(b.download(i), got[i])
    with pytest.raises(OtsError):
        b.run_sequential("tile")
    b.close()


@pytest.mark.gpu
def test_batched_stream_rejects_mixed_and_deep_grids():
    with pytest.raises(OtsError) as ei:
        B.Batch([dict(stencil="jacobi-2d", n=64, steps=4, T=2, kernel="stream"),
                 dict(stencil="jacobi-2d", n=64, steps=4, T=2, bx=32, E=2)])
    assert ei.value.status_name == "UNSUPPORTED"
    with pytest.raises(OtsError) as ei:
        B.Batch([dict(stencil="jacobi-2d", n=64, steps=8, T=6, kernel="stream")])
    assert ei.value.status_name == "UNSUPPORTED"


@pytest.mark.gpu
def test_cost_model_picks_stream_shapes_per_grid_and_batch_matches_oracle():
    """The streamed batch with per-grid (T, rows per segment) from the
    shipped cost model: every pick is a valid menu entry within the grid's
    step count, and the one-launch result equals each grid's oracle run."""
    import json
    import os
    from ots import model as M
    path = os.path.join(os.path.dirname(B.__file__), "data", "cost_model.json")
    cm = M.MLP.from_json(json.load(open(path)))
    grids = [dict(g) for g in STREAM_GRIDS]
    B.pick_stream(grids, cm)
    for g in grids:
        assert g["kernel"] == "stream" and 1 <= g["T"] <= 4 and g["T"] <= max(1, g["steps"])
        assert g["by"] in (1, 16, 32, 64, 128)
    b = B.Batch(grids)
    ins = B.inputs(grids, seed=9)
    for i, (s, a) in enumerate(ins):
        b.upload(i, s, a)
    b.run()
    for i, (g, (s, a)) in enumerate(zip(grids, ins)):
        check_same(g, b.download(i), oracle_run(g, s, a))
    b.close()
    cm.close()
