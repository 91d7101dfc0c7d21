"""Exhaustive (T, block, E) sweep through the C ABI, in process.

This is the B200 counterpart of the reference's sweep harness
(scripts/utils.py:36-244, run_experiment): it expands parameter ranges
(``[lo, hi, step]`` as in scripts/utils.py:16-27), runs every configuration
of one workload on the GPU, records the runner's keys plus the measured
GUpdates/s, and skips invalid configurations the way the reference's
runner exits with "ERROR:"/"Consistency error!".  Results are the training
data of the learned cost model and the measure its picks are scored by.

Usage:
    python -m ots.sweep --stencil jacobi-3d -n 512 -t 100 --kernel stream \
        --T 1,8,1 --bx 16,32,64 --by 4,16,2 --E 1,2,4 --out sweep.json
"""
import argparse
import itertools
import json
import time

import numpy as np

from . import (ENGINE_COMPAT, ENGINE_NATIVE, KERNEL_PLAIN, OtsError, Plan, STENCILS)


def expand(spec):
    """'a,b,c' -> [a, b, c]; 'lo:hi:step' -> range inclusive (scripts/utils.py:16-27)."""
    if isinstance(spec, (list, tuple)):
        return list(spec)
    spec = str(spec)
    if ":" in spec:
        lo, hi, st = [int(v) for v in spec.split(":")]
        return list(range(lo, hi + 1, st))
    return [int(v) for v in spec.split(",")]


def make_inputs(plan, seed=123456):
    """Seeded inputs as dense interior arrays (independent of T, so one set
    serves every configuration of a sweep)."""
    state, aux = plan.fill_reference(seed=seed)
    if plan.stencil in ("poisson-2d", "poisson-3d"):
        aux = [np.where(a != 0, 2.0 * a - 1.0, 0.0).astype(np.float32) for a in aux]
    if plan.stencil == "cdsc-tv-update-2d":
        aux[1] = np.where(aux[1] != 0, 1.0, 0.0).astype(np.float32)  # V = 1
    g = plan.geometry
    sl = tuple(slice(g.padding, g.padding + g.real_size) for _ in range(g.dims))
    return ([np.ascontiguousarray(a[sl]) for a in state],
            [np.ascontiguousarray(a[sl]) for a in aux])


def measure(plan, kernel, reps=3, warmup=1):
    """Median event time (s) of full runs of the plan's step count."""
    for _ in range(warmup):
        plan.run(kernel)
    times = []
    for _ in range(reps):
        t = plan.run(kernel)
        times.append(t.event_ms * 1e-3)
    times.sort()
    return times[len(times) // 2]


def run_config(stencil, n, steps, cfg, engine=ENGINE_NATIVE, inputs=None, reps=3, device=0):
    """Measure one configuration; returns a record dict (status 'ok' or the
    library's error status, like a failed runner line)."""
    rec = dict(stencil=stencil, n=n, steps=steps, engine=engine, **cfg)
    try:
        plan = Plan(stencil, n, steps, engine=engine, device=device, **cfg)
    except OtsError as e:
        rec.update(status=e.status_name, error=str(e))
        return rec, None
    with plan:
        g = plan.geometry
        if inputs is None or inputs[0][0].shape != plan.interior_shape:
            inputs = make_inputs(plan)
        plan.upload_interior(*inputs)
        t0 = time.perf_counter()
        sec = measure(plan, cfg.get("kernel", "auto"), reps=reps)
        wall = time.perf_counter() - t0
        upd = float(g.interior_points) * steps
        rec.update(status="ok", seconds=sec, gupdates=upd / sec / 1e9,
                   gflops=upd * g.flops_per_point / sec / 1e9, registers=g.registers,
                   shared_bytes=g.shared_bytes, useful_ratio=g.useful_ratio,
                   launches=g.launches, num_blocks=list(g.num_blocks),
                   real_per_block=list(g.real_per_block), comps=list(g.comps),
                   measure_wall=wall)
        return rec, inputs


def sweep(stencil, n, steps, space, engine=ENGINE_NATIVE, reps=3, log=None, device=0):
    """Run every configuration of `space` (list of cfg dicts)."""
    out = []
    inputs = None
    for cfg in space:
        rec, inp = run_config(stencil, n, steps, cfg, engine=engine, inputs=inputs, reps=reps,
                              device=device)
        if inp is not None:
            inputs = inp
        out.append(rec)
        if log:
            log(rec)
    return out


def stream_space(Ts, bxs, bys, Es, cys=(1,)):
    """Stream-kernel configurations; cy > 1 stacks cy CTAs along y in one
    thread-block cluster sharing a tile (cy = 1 is recorded without the key)."""
    out = []
    for T, bx, by, E, cy in itertools.product(Ts, bxs, bys, Es, cys):
        c = dict(kernel="stream", T=T, bx=bx, by=by, bz=1, E=E)
        if cy > 1:
            c["cy"] = cy
        out.append(c)
    return out


def tile_space(Ts, bxs, bys, bzs, Es, kernel="tile"):
    return [dict(kernel=kernel, T=T, bx=bx, by=by, bz=bz, E=E)
            for T, bx, by, bz, E in itertools.product(Ts, bxs, bys, bzs, Es)]


def best(records):
    ok = [r for r in records if r.get("status") == "ok"]
    return max(ok, key=lambda r: r["gupdates"]) if ok else None


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawTextHelpFormatter)
    ap.add_argument("--stencil", required=True, choices=STENCILS)
    ap.add_argument("-n", type=int, required=True)
    ap.add_argument("-t", type=int, default=64)
    ap.add_argument("--kernel", default="tile", choices=["tile", "stream", "plain", "tex"])
    ap.add_argument("--engine", default="native", choices=["native", "compat"])
    ap.add_argument("--T", default="1:8:1")
    ap.add_argument("--bx", default="16,32,64")
    ap.add_argument("--by", default="4,8,16")
    ap.add_argument("--bz", default="1")
    ap.add_argument("--E", default="1,2,4")
    ap.add_argument("--cy", default="1", help="stream kernel: CTAs per cluster along y")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--out")
    a = ap.parse_args(argv)
    eng = ENGINE_NATIVE if a.engine == "native" else ENGINE_COMPAT
    if a.kernel == "stream":
        space = stream_space(expand(a.T), expand(a.bx), expand(a.by), expand(a.E), expand(a.cy))
    elif a.kernel == "plain":
        space = [dict(kernel="plain", T=1, bx=32, by=8, bz=1, E=1)]
    else:
        space = tile_space(expand(a.T), expand(a.bx), expand(a.by), expand(a.bz), expand(a.E),
                           kernel=a.kernel)

    def log(r):
        if r["status"] == "ok":
            print("%-7s T=%d b=%dx%dx%d E=%d cy=%d  %8.1f GUpd/s  regs=%d smem=%d" % (
                r["kernel"], r["T"], r["bx"], r["by"], r["bz"], r["E"], r.get("cy", 1),
                r["gupdates"], r["registers"], r["shared_bytes"]), flush=True)

    recs = sweep(a.stencil, a.n, a.t, space, engine=eng, reps=a.reps, log=log)
    b = best(recs)
    if b:
        print("BEST", json.dumps(b))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(recs, fh, indent=0)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
