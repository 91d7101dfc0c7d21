"""Batched grids: many uneven 2D grids in one persistent, graph-captured launch.

    python -m ots.batch [--grids 256] [--seed 2012] [--reps 5]

runs the batched workload -- 256 independent FP32 grids mixing jacobi-2d,
poisson-2d (Jacobi sweep with RHS) and gradient-2d, sides log-uniform in
[64, 2048], step counts uniform in 8..256, inputs uniform [0, 1) -- in two
single graph launches: tile items with each grid's (T, block, E) picked by the
learned cost model, and warp items of the y-streamed 2D kernel with each
grid's (T, rows per segment) picked by the cost model (beside it the same
grids with a fixed T = 4); it prints one JSON line with their aggregate
GUpdates/s against the same grids run one after another (one launch per step,
one tile launch per T steps, one streamed launch per T steps) and the picks.
"""
import argparse
import ctypes
import json
import math
import os

import numpy as np

from . import (KERNEL_PLAIN, KERNEL_STREAM, KERNEL_TILE, OtsError, Params, SID, Timing, check,
               derive_geometry, lib, make_params)

BATCH_STENCILS = ("jacobi-2d", "poisson-2d", "gradient-2d")
MENU = [dict(T=T, bx=bx, E=E) for T in range(1, 9) for bx in (16, 32, 64) for E in (1, 2, 4)]


def _blib():
    L = lib()
    if not getattr(L, "_batch_ready", False):
        vp = ctypes.c_void_p
        L.ots_batch_create.argtypes = [ctypes.POINTER(Params), ctypes.c_int32, ctypes.c_int32,
                                       ctypes.POINTER(vp)]
        L.ots_batch_create.restype = ctypes.c_int
        L.ots_batch_destroy.argtypes = [vp]
        L.ots_batch_destroy.restype = None
        L.ots_batch_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int64),
                                     ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
        L.ots_batch_info.restype = ctypes.c_int
        F = ctypes.POINTER(ctypes.c_float)
        L.ots_batch_upload.argtypes = [vp, ctypes.c_int32, F, F]
        L.ots_batch_upload.restype = ctypes.c_int
        L.ots_batch_download.argtypes = [vp, ctypes.c_int32, F]
        L.ots_batch_download.restype = ctypes.c_int
        L.ots_batch_run.argtypes = [vp, ctypes.POINTER(Timing)]
        L.ots_batch_run.restype = ctypes.c_int
        L.ots_batch_run_async.argtypes = [vp]
        L.ots_batch_run_async.restype = ctypes.c_int
        L.ots_batch_stream.argtypes = [vp, ctypes.POINTER(vp)]
        L.ots_batch_stream.restype = ctypes.c_int
        L.ots_batch_run_sequential.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(Timing)]
        L.ots_batch_run_sequential.restype = ctypes.c_int
        L.ots_batch_set_wait_limit.argtypes = [vp, ctypes.c_double]
        L.ots_batch_set_wait_limit.restype = ctypes.c_int
        L.ots_batch_debug_hold.argtypes = [vp, ctypes.c_int32]
        L.ots_batch_debug_hold.restype = ctypes.c_int
        L._batch_ready = True
    return L


def workload(count=256, seed=2012):
    """The batched benchmark's grids (seeded): stencil uniform over the three,
    side round(exp(U[ln 64, ln 2048])), steps uniform 8..256."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        st = BATCH_STENCILS[int(rng.integers(0, 3))]
        n = int(round(math.exp(rng.uniform(math.log(64), math.log(2048)))))
        steps = int(rng.integers(8, 257))
        out.append(dict(stencil=st, n=n, steps=steps))
    return out


def pick(grids, cost_model=None, device=0):
    """Choose (T, bx, E) per grid from MENU: the cost model's best predicted
    configuration, or T=4, 32 x 8, E=2 without a model."""
    from . import model as M
    for g in grids:
        if cost_model is None:
            g.update(T=4, bx=32, E=2)
            continue
        feats, cands = [], []
        for c in MENU:
            cfg = dict(kernel="tile", T=c["T"], bx=c["bx"], by=256 // c["bx"], bz=1, E=c["E"])
            try:
                geo = derive_geometry(stencil=g["stencil"], n=g["n"], steps=g["steps"], T=c["T"],
                                      bx=c["bx"], by=256 // c["bx"], bz=1, E=c["E"],
                                      kernel="tile", device=device)
            except OtsError:
                continue
            feats.append(M.features(g["stencil"], cfg, geo))
            cands.append(c)
        best = int(cost_model.topk(np.stack(feats), 1)[0])
        g.update(cands[best])
    return grids


# Rows per segment are the batch's own choice, not a grid's: a lone grid
# wants short segments for parallelism (16 rows is the single-launch optimum
# at 2048^2), but in a batch hundreds of grids share the GPU, and short
# segments only add halo rows (2 R T per segment: +50 % at 16 rows, T = 4;
# measured on the 256-grid batch at T = 4: 16 rows 673, 32 rows 805, 64 rows
# 918, 128 rows 908, 256 rows 807 GUpd/s).  The batch engine's 64 stays.
STREAM_ROWS = 64
STREAM_MENU = [dict(T=T, by=STREAM_ROWS) for T in range(1, 5)]
SATURATED_N = 2048  # grid side at which the model ranks (inside a batch the GPU is full)


def pick_stream(grids, cost_model=None, T=4, rows=1, device=0):
    """Stream-mode choice per grid.  With a cost model: the T (1..4 -- the
    batch kernel's strip halo covers T <= 4) the model predicts fastest for
    the grid's stencil at STREAM_ROWS rows per segment.  The model is trained
    on single launches, where a small grid cannot fill the GPU; inside a
    batch every grid shares a full GPU, so each grid is ranked at its
    saturated rate: the features of the same geometry on a grid of side
    max(n, SATURATED_N).  Without a model: T (at most the step count) and
    `rows` (1 = the batch engine's default of 64)."""
    from . import model as M
    for g in grids:
        if cost_model is None:
            g.update(kernel="stream", T=max(1, min(T, g["steps"])), bx=32, by=rows, E=1)
            continue
        feats, cands = [], []
        for c in STREAM_MENU:
            if c["T"] > max(1, g["steps"]):
                continue
            cfg = dict(kernel="stream", T=c["T"], bx=32, by=c["by"], bz=1, E=1)
            try:
                geo = derive_geometry(stencil=g["stencil"], n=max(g["n"], SATURATED_N),
                                      steps=g["steps"], T=c["T"], bx=32, by=c["by"], bz=1, E=1,
                                      kernel="stream", device=device)
            except OtsError:
                continue
            feats.append(M.features(g["stencil"], cfg, geo))
            cands.append(c)
        best = cands[int(cost_model.topk(np.stack(feats), 1)[0])]
        g.update(kernel="stream", T=best["T"], bx=32, by=best["by"], E=1)
    return grids


class Batch:
    """Grids with kernel="stream" (all of them) run as warp items of the
    y-streamed 2D kernel; otherwise as tile items with their own (T, bx, E)."""

    def __init__(self, grids, device=0):
        arr = (Params * len(grids))()
        for i, g in enumerate(grids):
            if g.get("kernel") == "stream":
                arr[i] = make_params(g["stencil"], g["n"], g["steps"], T=g["T"], bx=32,
                                     by=g.get("by", 1), E=1, kernel="stream", device=device)
            else:
                arr[i] = make_params(g["stencil"], g["n"], g["steps"], T=g["T"], bx=g["bx"],
                                     by=256 // g["bx"], E=g["E"], device=device)
        h = ctypes.c_void_p()
        check(_blib().ots_batch_create(arr, len(grids), device, ctypes.byref(h)))
        self.h = h
        self.grids = grids

    def close(self):
        if getattr(self, "h", None):
            _blib().ots_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        u, it, c = ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32()
        check(_blib().ots_batch_info(self.h, ctypes.byref(u), ctypes.byref(it), ctypes.byref(c)))
        return {"updates": u.value, "items": it.value, "ctas": c.value}

    def upload(self, i, state, aux=None):
        F = ctypes.POINTER(ctypes.c_float)
        s = np.ascontiguousarray(state, np.float32)
        n = self.grids[i]["n"]
        assert s.shape == (n, n)
        a = None if aux is None else np.ascontiguousarray(aux, np.float32)
        check(_blib().ots_batch_upload(self.h, i, s.ctypes.data_as(F),
                                       None if a is None else a.ctypes.data_as(F)))

    def download(self, i):
        n = self.grids[i]["n"]
        out = np.zeros((n, n), np.float32)
        check(_blib().ots_batch_download(self.h, i, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def run(self):
        t = Timing()
        check(_blib().ots_batch_run(self.h, ctypes.byref(t)))
        return t.event_ms * 1e-3

    def set_wait_limit(self, seconds):
        """Limit of each item's bounded wait for its grid's previous chunk."""
        check(_blib().ots_batch_set_wait_limit(self.h, float(seconds)))

    def debug_hold(self, grid):
        """Test hook: grid's later chunks wait for a count never reached (-1: off)."""
        check(_blib().ots_batch_debug_hold(self.h, int(grid)))

    def run_sequential(self, kernel="plain"):
        t = Timing()
        k = {"plain": KERNEL_PLAIN, "tile": KERNEL_TILE, "stream": KERNEL_STREAM}[kernel]
        check(_blib().ots_batch_run_sequential(self.h, k, ctypes.byref(t)))
        return t.event_ms * 1e-3, t.launches


def inputs(grids, seed=7):
    """Uniform [0, 1) interiors (and f in [-1, 1) for Poisson), seeded."""
    rng = np.random.default_rng(seed)
    out = []
    for g in grids:
        s = rng.random((g["n"], g["n"]), dtype=np.float32)
        a = (2.0 * rng.random((g["n"], g["n"]), dtype=np.float32) - 1.0) \
            if g["stencil"] == "poisson-2d" else None
        out.append((s, a))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--grids", type=int, default=256)
    ap.add_argument("--seed", type=int, default=2012)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--no-model", action="store_true")
    ap.add_argument("--mode", default="all", choices=["all", "stream-graph", "tile-graph"],
                    help="all: every comparison; stream-graph / tile-graph: only that one "
                    "graph-captured launch (e.g. under a profiler)")
    a = ap.parse_args(argv)
    from . import model as M
    cm = None
    if not a.no_model:
        path = os.path.join(os.path.dirname(__file__), "data", "cost_model.json")
        cm = M.MLP.from_json(json.load(open(path)))
    grids = pick(workload(a.grids, a.seed), cm)
    ins = inputs(grids)
    if a.mode != "all":
        one = Batch(pick_stream([dict(g) for g in grids], cm) if a.mode == "stream-graph"
                    else grids)
        for i, (s, x) in enumerate(ins):
            one.upload(i, s, x)
        one.run()  # warm-up
        ts = []
        for _ in range(a.reps):
            for i, (s, x) in enumerate(ins):
                one.upload(i, s, x)
            ts.append(one.run())
        info = one.info()
        one.close()
        t = sorted(ts)[len(ts) // 2]
        print(json.dumps({"metric": "GUpdates/s", "mode": a.mode, "updates": info["updates"],
                          "items": info["items"], "ctas": info["ctas"],
                          "value": info["updates"] / t / 1e9, "seconds": t}))
        return 0
    b = Batch(grids)

    def load():
        for i, (s, x) in enumerate(ins):
            b.upload(i, s, x)

    load()
    b.run()  # warm-up
    t_graph = []
    for _ in range(a.reps):
        load()
        t_graph.append(b.run())
    load()
    b.run_sequential("tile")
    t_tile = []
    for _ in range(max(1, a.reps // 2)):
        load()
        t_tile.append(b.run_sequential("tile")[0])
    load()
    t_plain, launches = b.run_sequential("plain")
    info = b.info()
    upd = info["updates"]
    tg = sorted(t_graph)[len(t_graph) // 2]
    tt = sorted(t_tile)[len(t_tile) // 2]
    b.close()
    # the same grids as warp items of the y-streamed kernel
    # the streamed batch: per-grid (T, rows) from the cost model, and the same
    # grids with the fixed choice (T = 4, the library's rows) beside it
    sgrids = pick_stream([dict(g) for g in grids], cm)
    fgrids = pick_stream([dict(g) for g in grids])
    bf = Batch(fgrids)
    for i, (s, x) in enumerate(ins):
        bf.upload(i, s, x)
    bf.run()
    t_sf = []
    for _ in range(a.reps):
        for i, (s, x) in enumerate(ins):
            bf.upload(i, s, x)
        t_sf.append(bf.run())
    bf.close()
    tsf = sorted(t_sf)[len(t_sf) // 2]
    bs = Batch(sgrids)

    def load_s():
        for i, (s, x) in enumerate(ins):
            bs.upload(i, s, x)

    load_s()
    bs.run()
    t_sg = []
    for _ in range(a.reps):
        load_s()
        t_sg.append(bs.run())
    load_s()
    bs.run_sequential("stream")
    t_ss = []
    for _ in range(max(1, a.reps // 2)):
        load_s()
        t_ss.append(bs.run_sequential("stream")[0])
    sinfo = bs.info()
    bs.close()
    tsg = sorted(t_sg)[len(t_sg) // 2]
    tss = sorted(t_ss)[len(t_ss) // 2]
    print(json.dumps({
        "metric": "GUpdates/s", "workload": "batched: %d grids jacobi-2d/poisson-2d/gradient-2d, "
        "sides 64..2048 log-uniform, steps 8..256 (seed %d)" % (a.grids, a.seed),
        "updates": upd, "items": info["items"], "ctas": info["ctas"],
        "graph_one_launch": {"value": upd / tg / 1e9, "seconds": tg},
        "sequential_tile": {"value": upd / tt / 1e9, "seconds": tt},
        "sequential_plain": {"value": upd / t_plain / 1e9, "seconds": t_plain,
                             "launches": launches},
        "speedup_vs_sequential_plain": t_plain / tg, "speedup_vs_sequential_tile": tt / tg,
        "configs_from": "cost model" if cm is not None else "default T=4 32x8 E=2",
        "stream_graph_one_launch": {"value": upd / tsg / 1e9, "seconds": tsg,
                                    "items": sinfo["items"], "ctas": sinfo["ctas"]},
        "sequential_stream": {"value": upd / tss / 1e9, "seconds": tss},
        "stream_speedup_vs_sequential_plain": t_plain / tsg,
        "stream_configs_from": "cost model" if cm is not None else "fixed T=4",
        "stream_graph_fixed_T4": {"value": upd / tsf / 1e9, "seconds": tsf},
        "stream_picks": [{"stencil": g["stencil"], "n": g["n"], "steps": g["steps"],
                          "T": g["T"], "rows": g["by"]} for g in sgrids],
    }))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
