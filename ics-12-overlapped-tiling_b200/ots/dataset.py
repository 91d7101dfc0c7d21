"""Collect the cost model's training data: exhaustive sweeps on this GPU.

For every stencil, a configuration space of the kind the reference swept
(scripts/c2050/*.yml: block sizes, time tile 1..8, elements per thread) is
measured through the C ABI; each record carries the configuration, the
geometry the library derived for it (block counts, shared bytes, registers,
occupancy, redundant-compute ratio) and the measured GUpdates/s.

    python -m ots.dataset --out ots/data/sweeps_b200.json [--quick]
"""
import argparse
import itertools
import json
import time

from . import OtsError, Plan, STENCILS, derive_geometry
from .sweep import make_inputs, measure

# workload per dimensionality (sized so one configuration measures in ms)
WORKLOAD = {1: (1 << 22, 64), 2: (2048, 64), 3: (256, 32)}


def space(stencil, dims, quick=False):
    cfgs = []
    if dims == 1:
        for T, bx, E in itertools.product(range(1, 9), (64, 128, 256, 512), (1, 2, 4, 8)):
            cfgs.append(dict(kernel="tile", T=T, bx=bx, by=1, bz=1, E=E))
        # the register kernel: T steps per launch, E cells per lane
        for T, E in itertools.product((1, 2, 4, 8, 16, 32, 64), (4, 8, 16)):
            cfgs.append(dict(kernel="stream", T=T, bx=32, by=1, bz=1, E=E))
    elif dims == 2:
        for T, bx, by, E in itertools.product(range(1, 9), (16, 32, 64), (4, 8, 16), (1, 2, 4, 8)):
            cfgs.append(dict(kernel="tile", T=T, bx=bx, by=by, bz=1, E=E))
        if stencil in ("jacobi-2d", "poisson-2d", "gradient-2d"):
            # y-streamed kernel: T and rows per segment (by; 1 = the library's choice)
            for T, by in itertools.product(range(1, 9), (1, 16, 32, 64, 128)):
                cfgs.append(dict(kernel="stream", T=T, bx=32, by=by, bz=1, E=1))
        else:
            # the generic y-streamed kernel (the op's apply on register rows)
            for T, by in itertools.product(range(1, 7), (1, 16, 64)):
                cfgs.append(dict(kernel="stream", T=T, bx=32, by=by, bz=1, E=1))
    else:
        for T, (bx, by, bz), E in itertools.product(
                range(1, 5), ((32, 4, 4), (32, 8, 2), (64, 4, 2), (16, 8, 4), (16, 16, 2)),
                (1, 2, 4)):
            cfgs.append(dict(kernel="tile", T=T, bx=bx, by=by, bz=bz, E=E))
        if stencil in ("jacobi-3d", "poisson-3d", "gradient-3d"):
            for T, bx, by, E in itertools.product(range(1, 7), (8, 16, 32), (8, 16, 32), (1, 2, 4)):
                cfgs.append(dict(kernel="stream", T=T, bx=bx, by=by, bz=1, E=E))
    # the plain one-step kernel is a candidate too: for compute-bound updates
    # time tiling buys nothing and one cell per thread can be fastest
    cfgs.append(dict(kernel="plain", T=1, bx=256 if dims == 1 else 32, by=1 if dims == 1 else 8,
                     bz=1, E=1))
    if quick:
        cfgs = cfgs[::7]
    return cfgs


def geom_dict(g):
    return {k: (list(v) if hasattr(v, "__len__") else v) for k, v in g.as_dict().items()}


def collect(stencils=None, quick=False, reps=3, device=0, log=print, kernel=None):
    records = []
    for st in stencils or STENCILS:
        dims = {"jacobi-1d": 1, "jacobi-1d-5pt": 1, "jacobi-1d-7pt": 1}.get(
            st, 3 if st.endswith("3d") else 2)
        n, steps = WORKLOAD[dims]
        inputs = None
        t0 = time.time()
        ok = 0
        for cfg in space(st, dims, quick):
            if kernel and cfg["kernel"] != kernel:
                continue
            rec = dict(stencil=st, n=n, steps=steps, **cfg)
            try:
                plan = Plan(st, n, steps, device=device, **cfg)
            except OtsError as e:
                rec.update(status=e.status_name)
                records.append(rec)
                continue
            with plan:
                if inputs is None or inputs[0][0].shape != plan.interior_shape:
                    inputs = make_inputs(plan)
                plan.upload_interior(*inputs)
                sec = measure(plan, cfg["kernel"], reps=reps)
                g = plan.geometry
                rec.update(status="ok", seconds=sec,
                           gupdates=float(g.interior_points) * steps / sec / 1e9,
                           geom=geom_dict(g))
                ok += 1
            records.append(rec)
        if log:
            best = max((r for r in records if r["stencil"] == st and r.get("status") == "ok"),
                       key=lambda r: r["gupdates"], default=None)
            log("%-18s %4d configs ok in %5.1f s; best %s" % (
                st, ok, time.time() - t0,
                None if best is None else "%.1f GUpd/s %s T=%d %dx%dx%d E=%d" % (
                    best["gupdates"], best["kernel"], best["T"], best["bx"], best["by"],
                    best["bz"], best["E"])))
    return records


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--out", required=True)
    ap.add_argument("--stencils", default=",".join(STENCILS))
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--kernel", help="collect only this kernel family's configurations")
    ap.add_argument("--merge", help="existing dataset: keep its records of other "
                    "(stencil, kernel) pairs and replace the collected ones")
    a = ap.parse_args(argv)
    recs = collect(a.stencils.split(","), a.quick, a.reps, kernel=a.kernel)
    if a.merge:
        old = json.load(open(a.merge))["records"]
        got = {(r["stencil"], r["kernel"]) for r in recs}
        recs = [r for r in old if (r["stencil"], r["kernel"]) not in got] + recs
    with open(a.out, "w") as fh:
        json.dump({"device": "B200", "workload": {str(k): v for k, v in WORKLOAD.items()},
                   "records": recs}, fh, separators=(",", ":"))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
