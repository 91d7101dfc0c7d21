"""The measured workloads at their full sizes, their seeded inputs, and the
three ways of choosing a configuration for each: the learned picker (the cost
model ranks the space, the top 10 % are measured, the best is kept), the
exhaustive sweep (every configuration measured) and the plain one-step
kernel.

Workloads (grid side, time steps):

  jacobi-2d       2048^2,  64 steps   reference fill (srand/rand, uniform [0,1))
  jacobi-3d        512^3, 100 steps   reference fill, weight 1/7
  poisson-3d       512^3, 100 steps   reference fill; RHS f = 2 u - 1 (uniform
                                      [-1,1)), h = 1/(n-1)
  fdtd-2d         4096^2, 500 steps   reference fill of Ex/Ey/Hz; source row
  rician-denoise  4096^2, 200 steps   disk image with Rician noise, u0 = f
  cdsc-tv-update  4096^2, 200 steps   the same image: u0 = F = f, V = 1

The last two are held out: each one's picks come from a cost model trained
without it (the reference's leave-one-out protocol,
scripts/run-weka.py:74-150).  Both, and cs-3d, are measured a second time in
the fast-division variant (approximate division and rsqrt, within the
tolerance the parity tests state; key '<stencil>-fast' for --configs).
The other seven stencils follow at the sizes the training data was measured
at (1D 4194304 cells x 64, 2D 2048^2 x 64, 3D 256^3 x 32 steps).

The disk image: 64 disks of constant intensity (uniform [0.2, 1.0], radius
uniform [n/64, n/12], centres uniform over the grid, later disks drawn over
earlier ones) on a 0.1 background; the noisy image is
f = sqrt((s + n1)^2 + n2^2) with n1, n2 ~ N(0, 0.05^2), the Rician noise model
whose sigma^2 = 0.0025 the Rician stencil assumes
(opencl/rician-denoise-2d/rician-denoise-2d.cpp:153-161); seeded SplitMix64
uniforms and Box-Muller normals (ots_fill_disks), so the CLI's
--init baseline and this table start from the same image.
"""
import json
import math
import os

import numpy as np

from . import VARIANT_FAST, OtsError, Plan
from . import model as M
from .dataset import space
from .sweep import make_inputs

WORKLOADS = [
    dict(name="jacobi-2d 2048^2 x 64", stencil="jacobi-2d", n=2048, steps=64),
    dict(name="jacobi-3d 512^3 x 100", stencil="jacobi-3d", n=512, steps=100),
    dict(name="poisson-3d 512^3 x 100", stencil="poisson-3d", n=512, steps=100),
    dict(name="fdtd-2d 4096^2 x 500", stencil="fdtd-2d", n=4096, steps=500),
    dict(name="rician-denoise-2d 4096^2 x 200", stencil="rician-denoise-2d", n=4096,
         steps=200, held_out=True),
    dict(name="cdsc-tv-update-2d 4096^2 x 200", stencil="cdsc-tv-update-2d", n=4096,
         steps=200, held_out=True),
    # the other seven stencils at the training-data sizes, so every stencil
    # has its FP64 error after the full step count
    dict(name="jacobi-1d 4194304 x 64", stencil="jacobi-1d", n=1 << 22, steps=64, extra=True),
    dict(name="jacobi-1d-5pt 4194304 x 64", stencil="jacobi-1d-5pt", n=1 << 22, steps=64,
         extra=True),
    dict(name="jacobi-1d-7pt 4194304 x 64", stencil="jacobi-1d-7pt", n=1 << 22, steps=64,
         extra=True),
    dict(name="poisson-2d 2048^2 x 64", stencil="poisson-2d", n=2048, steps=64, extra=True),
    dict(name="gradient-2d 2048^2 x 64", stencil="gradient-2d", n=2048, steps=64, extra=True),
    dict(name="gradient-3d 256^3 x 32", stencil="gradient-3d", n=256, steps=32, extra=True),
    dict(name="cs-3d 256^3 x 32", stencil="cs-3d", n=256, steps=32, extra=True),
    # the fast-division variant of the three stencils that divide
    dict(name="rician-denoise-2d 4096^2 x 200 (fast division)", stencil="rician-denoise-2d",
         n=4096, steps=200, held_out=True, variant="fast"),
    dict(name="cdsc-tv-update-2d 4096^2 x 200 (fast division)", stencil="cdsc-tv-update-2d",
         n=4096, steps=200, held_out=True, variant="fast"),
    dict(name="cs-3d 256^3 x 32 (fast division)", stencil="cs-3d", n=256, steps=32,
         extra=True, variant="fast"),
]


def workload_key(w):
    """The --configs selector of a workload: its stencil, '-fast' appended
    for the fast-division rows."""
    return w["stencil"] + ("-fast" if w.get("variant") == "fast" else "")


def variant_kw(w):
    """Plan keywords of the workload's arithmetic variant (none: baseline)."""
    return {"variant": VARIANT_FAST} if w.get("variant") == "fast" else {}
HELD_OUT = ("rician-denoise-2d", "cdsc-tv-update-2d")

# compulsory bytes per update of a one-step launch: read every field once,
# write every updated field once (FP32)
BYTES_PER_UPDATE = {"jacobi-2d": 8, "jacobi-3d": 8, "poisson-3d": 12, "fdtd-2d": 24,
                    "rician-denoise-2d": 12, "cdsc-tv-update-2d": 16, "jacobi-1d": 8,
                    "jacobi-1d-5pt": 8, "jacobi-1d-7pt": 8, "poisson-2d": 12,
                    "gradient-2d": 8, "gradient-3d": 8, "cs-3d": 8}

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


def disk_image(n, seed=2012, count=64, background=0.1, sigma=0.05):
    """(clean, noisy) n x n float32 images as described in the module doc
    (ots_fill_disks in libots, the generator the CLI's --init baseline uses)."""
    from . import fill_disks
    return fill_disks(n, seed, count, background, sigma)


_IMAGES = {}


def inputs(plan, seed=123456):
    """Interior (state, aux) arrays of the workload's inputs for `plan` (its
    real size may be below the grid side where the reference's size rule
    truncates; the disk image is then cropped)."""
    st = plan.stencil
    if st in HELD_OUT:
        n = plan.params.problem_size
        if n not in _IMAGES:
            _IMAGES[n] = disk_image(n)[1]
        rs = plan.geometry.real_size
        f = np.ascontiguousarray(_IMAGES[n][:rs, :rs])
        if st == "rician-denoise-2d":
            return [f.copy()], [f]
        return [f.copy()], [f, np.ones_like(f)]
    return make_inputs(plan, seed=seed)


def measure(plan, kernel, budget_s=0.6):
    """Median event time (s) of full runs: one warm-up run, then up to three
    timed runs while they fit `budget_s`.  A configuration whose warm-up run
    alone takes over a second (far from the best of any space here) keeps
    that time."""
    t = plan.run(kernel).event_ms * 1e-3
    if t > 1.0:
        return t
    times = []
    for _ in range(3):
        times.append(plan.run(kernel).event_ms * 1e-3)
        if sum(times) + t > budget_s:
            break
    times.sort()
    return times[len(times) // 2]


def sweep_workload(w, cfgs=None, device=0, log=None):
    """Measure every configuration of the workload's space; returns records
    with the geometry the model needs."""
    st, n, steps = w["stencil"], w["n"], w["steps"]
    dims = 1 if st.startswith("jacobi-1d") else 3 if st.endswith("3d") else 2
    recs = []
    cache = {}
    for cfg in cfgs or space(st, dims):
        rec = dict(stencil=st, n=n, steps=steps, **cfg)
        try:
            plan = Plan(st, n, steps, device=device, **variant_kw(w), **cfg)
        except OtsError as e:
            rec.update(status=e.status_name)
            recs.append(rec)
            continue
        with plan:
            g = plan.geometry
            key = g.real_size
            if key not in cache:
                cache.clear()
                cache[key] = inputs(plan)
            plan.upload_interior(*cache[key])
            sec = measure(plan, cfg["kernel"])
            rec.update(status="ok", seconds=sec,
                       gupdates=float(g.interior_points) * steps / sec / 1e9,
                       real_size=g.real_size,
                       geom={k: (list(v) if hasattr(v, "__len__") else v)
                             for k, v in g.as_dict().items()})
        recs.append(rec)
        if log:
            log(rec)
    return recs


def model_for(stencil, device=0, epochs=300, seed=0):
    """The cost model that picks for `stencil`: the shipped model, or for a
    held-out stencil one trained on the sweep data of every other stencil
    (leave one out, the reference's protocol: scripts/run-weka.py:74-150).
    Returns (model, description)."""
    if stencil not in HELD_OUT:
        with open(os.path.join(DATA, "cost_model.json")) as fh:
            return M.MLP.from_json(json.load(fh), device=device), "shipped cost model"
    with open(os.path.join(DATA, "sweeps_b200.json")) as fh:
        recs = [r for r in json.load(fh)["records"] if r.get("stencil") != stencil]
    # the full-size workload sweeps of the other stencils, as the shipped
    # model is trained on both sizes
    cpath = os.path.join(DATA, "configs_b200.json")
    if os.path.exists(cpath):
        with open(cpath) as fh:
            recs += [r for r in M.workload_records(json.load(fh)) if r["stencil"] != stencil]
    X, y, _, _ = M.dataset(recs)
    m = M.MLP(X.shape[1], 64, 3, seed=seed, device=device)
    m.fit(X, y, epochs=epochs, seed=seed)
    return m, "trained without %s" % stencil


def picks(stencil, recs, cost_model, k_frac=0.10):
    """The learned pick from measured records: rank every valid time-tiled
    configuration, keep the best measured of the top k and of the plain
    one-step kernel (always measured), and the model's top-1 (with plain)."""
    ok = [r for r in recs if r.get("status") == "ok" and r.get("kernel") != "plain"]
    plain = [r for r in recs if r.get("status") == "ok" and r.get("kernel") == "plain"]
    if not ok:
        return None
    X = np.stack([M.features(stencil, r, r["geom"]) for r in ok])
    # the plain runs count against the same budget: k_frac of the space in all
    k = max(1, int(math.floor(k_frac * (len(ok) + len(plain)))) - len(plain))
    top = [int(i) for i in cost_model.topk(X, k)]
    picked = max([ok[i] for i in top] + plain, key=lambda r: r["gupdates"])
    top1 = max([ok[top[0]]] + plain, key=lambda r: r["gupdates"])
    return {"space": len(ok) + len(plain), "k": k, "measured": k + len(plain), "picked": picked,
            "top1": top1}


def learned_pick(w, cost_model, k_frac=0.10, device=0):
    """The learned picker live, measuring only what it picks: rank the
    workload's whole space with the cost model from the geometry alone (no
    run), measure the top k and the plain one-step kernel (k + 1 = 10 % of
    the space, the picker's budget), keep the best measured.  Returns
    (best record, k, space size)."""
    st, n, steps = w["stencil"], w["n"], w["steps"]
    dims = 1 if st.startswith("jacobi-1d") else 3 if st.endswith("3d") else 2
    cands, feats = [], []
    plain = None
    for cfg in space(st, dims):
        if cfg["kernel"] == "plain":
            plain = cfg
            continue
        try:
            g = derive_geometry_for(st, n, steps, cfg, device, **variant_kw(w))
        except OtsError:
            continue
        cands.append(cfg)
        feats.append(M.features(st, cfg, {k: (list(v) if hasattr(v, "__len__") else v)
                                          for k, v in g.as_dict().items()}))
    size = len(cands) + 1
    k = max(1, int(math.floor(k_frac * size)) - 1)
    top = [int(i) for i in cost_model.topk(np.stack(feats), k)]
    recs = sweep_workload(w, [cands[i] for i in top] + [plain], device=device)
    ok = [r for r in recs if r.get("status") == "ok"]
    return max(ok, key=lambda r: r["gupdates"]), k, size


def derive_geometry_for(stencil, n, steps, cfg, device=0, **kw):
    from . import derive_geometry
    return derive_geometry(stencil=stencil, n=n, steps=steps, T=cfg["T"], bx=cfg["bx"],
                           by=cfg["by"], bz=cfg["bz"], E=cfg["E"], kernel=cfg["kernel"],
                           device=device, **kw)


def config_of(rec):
    return {q: rec[q] for q in ("kernel", "T", "bx", "by", "bz", "E")}


def plain_record(w, device=0):
    """The plain one-step-per-launch kernel on the workload."""
    one_d = w["stencil"].startswith("jacobi-1d")
    cfg = dict(kernel="plain", T=1, bx=256 if one_d else 32, by=1 if one_d else 8, bz=1, E=1)
    return sweep_workload(w, [cfg], device=device)[0]


def run_config(w, cfg, device=0):
    """(plan geometry, padded inputs, padded outputs) of one full run of the
    workload with `cfg`; the inputs come back padded so a CPU sweep can
    start from the same state."""
    with Plan(w["stencil"], w["n"], w["steps"], device=device, **variant_kw(w), **cfg) as plan:
        g = plan.geometry
        st, ax = inputs(plan)
        plan.upload_interior(st, ax)
        pad = tuple(slice(g.padding, g.padding + g.real_size) for _ in range(g.dims))
        def padded(a):
            out = np.zeros((g.padded_size,) * g.dims, np.float32)
            out[pad] = a
            return out
        pst, pax = [padded(a) for a in st], [padded(a) for a in ax]
        plan.run(cfg["kernel"])
        got = plan.download()
        return g, pst, pax, got


def repick(table, device=0):
    """Recompute every workload's learned pick in a --configs table from its
    recorded measurements with the current cost models (no new runs)."""
    for w in table["workloads"]:
        cm, desc = model_for(w["stencil"], device=device)
        pk = picks(w["stencil"], w["records"], cm)
        cm.close()
        best = w["exhaustive"]["gupdates"]
        w["learned"] = {"gupdates": pk["picked"]["gupdates"], "config": config_of(pk["picked"]),
                        "k": pk["k"], "measured": pk["measured"],
                        "over_best": pk["picked"]["gupdates"] / best,
                        "top1_gupdates": pk["top1"]["gupdates"],
                        "top1_config": config_of(pk["top1"]),
                        "top1_over_best": pk["top1"]["gupdates"] / best, "model": desc}
    return table


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description="re-evaluate the learned picks of a --configs table")
    ap.add_argument("--repick", required=True, help="bench --configs table (JSON)")
    ap.add_argument("--out", required=True)
    a = ap.parse_args(argv)
    t = repick(json.load(open(a.repick)))
    with open(a.out, "w") as fh:
        json.dump(t, fh, indent=1)
    for w in t["workloads"]:
        print("%-32s learned %.1f (%.3f of best, %d measured) %s" % (
            w["workload"], w["learned"]["gupdates"], w["learned"]["over_best"],
            w["learned"]["measured"], w["learned"]["config"]))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
