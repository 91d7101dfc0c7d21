"""Analytical performance model of the overlapped tile kernel, re-parameterised
for B200: the comparator the learned picker is measured against.

This restates the reference's own model (scripts/run-model.py): per
configuration an occupancy estimate (``occupancy_of``, run-model.py:9-62),
then a per-stage cost (run-model.py:300-560) -- phase 1 set-up, phase 2 the
global-memory step with an L1 cache model keyed on the runner's
phase2_global_loads, phase 3 the (T-1) shared-memory steps, phase 4 the
write-back -- each stage the max of an issue-bound and a latency+bandwidth
term, times the number of waves of resident blocks, times the launches.  The
configuration with the least simulated time is the model's pick; the report
is the reference's "Best Overall" (percent slowdown of the pick against the
measured best, run-model.py:588-600) and "Best One Percent".

Constants (``ARCH``):

* ``c2050`` -- scripts/c2050/c2050.arch as published;
* ``b200``  -- the same quantities for one B200: 148 SMs at 1.965 GHz, 64
  warps / 2048 threads / 32 blocks / 64 K registers / 228 KB shared per SM;
  B_gmem from the measured copy bandwidth (128 B per warp access over
  bytes/clock/SM); issue costs scaled by the 4 schedulers per SM (Fermi
  issued one warp instruction per SM clock); SFU costs by the 16 SFUs per SM;
  latencies for HBM3e and shared memory; half of a 128 KB L1 for the cache
  model; a launch penalty for a stream-ordered launch.

Two deliberate differences from the script, both because this engine reports
its geometry: block counts, registers and the block's real (useful) extent
come from the library's derived geometry (the script recomputes the latter
assuming E along y, while the native 3D tile puts E along z); and a
configuration whose phase-2 load count has no cache formula falls back to the
no-cache branch instead of exiting.

    python -m ots.analytic --data ots/data/sweeps_b200.json [--arch b200]
    python -m ots.analytic --dat j2d.dat --arch b200     # reference-style CSV
"""
import argparse
import csv
import json
import math
import os

ARCH = {
    # scripts/c2050/c2050.arch
    "c2050": dict(total_shared=49152.0, max_warps_per_sm=48.0, max_threads_per_sm=1536.0,
                  max_blocks_per_sm=8.0, max_regs_per_sm=32768.0, num_sm=14.0, clock=1.15e9,
                  c_load=2.0, c_op=1.0, sfu_glb=16.0, sfu_shd=4.0, B_gmem=18.0, B_smem=2.0,
                  L_gmem=750.0, L_smem=32.0, launch_penalty=0.0, warp_size=32.0,
                  l1_model_bytes=16384.0 * 0.5, phase1=(10.0, 20.0), max_regs_per_thread=63.0),
    "b200": dict(total_shared=233472.0, max_warps_per_sm=64.0, max_threads_per_sm=2048.0,
                 max_blocks_per_sm=32.0, max_regs_per_sm=65536.0, num_sm=148.0, clock=1.965e9,
                 c_load=0.5, c_op=0.25, sfu_glb=4.0, sfu_shd=1.0, B_gmem=None, B_smem=2.0,
                 L_gmem=900.0, L_smem=30.0, launch_penalty=6000.0, warp_size=32.0,
                 l1_model_bytes=131072.0 * 0.5, phase1=(2.5, 5.0), max_regs_per_thread=255.0),
}
HBM_FALLBACK_GBS = 6650.0


def b200_arch(hbm_gbs=None):
    """B200 constants; B_gmem from the measured HBM copy bandwidth."""
    a = dict(ARCH["b200"])
    if hbm_gbs is None:
        hbm_gbs = HBM_FALLBACK_GBS
        path = os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(
            os.path.abspath(__file__)))), "MEASURED_PEAKS.json")
        try:
            with open(path) as fh:
                hbm_gbs = float(json.load(fh)["hbm_gbs"])
        except Exception:
            pass
    bytes_per_clk_sm = hbm_gbs * 1e9 / (a["num_sm"] * a["clock"])
    a["B_gmem"] = 128.0 / bytes_per_clk_sm
    a["hbm_gbs"] = hbm_gbs
    return a


def get_arch(name):
    return b200_arch() if name == "b200" else dict(ARCH[name])


def _i(run, k, default=None):
    v = run.get(k, default)
    return int(float(v))


def shared_estimate(run):
    """Shared bytes per block as the model estimates them (run-model.py:24-33),
    with E on the tile's E axis."""
    x, y, z = _i(run, "Block Size X"), _i(run, "Block Size Y"), _i(run, "Block Size Z")
    e, dim = _i(run, "Elements/Thread"), _i(run, "Dimensions")
    eax = _i(run, "e_axis", 1 if dim > 1 else 0)
    ext = [x, y, z]
    ext[eax] *= e
    if dim == 1:
        s = (ext[0] + 2.0) * 4.0
    elif dim == 2:
        s = (ext[0] + 2.0) * (ext[1] + 2.0) * 4.0
    else:
        s = (ext[0] + 2.0) * (ext[1] + 2.0) * (ext[2] + 2.0) * 4.0
    return s * float(run["num_fields"])


def occupancy(run, arch):
    """(active warps per SM, blocks per SM) -- run-model.py:9-62."""
    x, y, z = _i(run, "Block Size X"), _i(run, "Block Size Y"), _i(run, "Block Size Z")
    regs = _i(run, "Register Usage")
    warps_per_block = x * y * z / arch["warp_size"]
    regs_per_block = regs * x * y * z
    total_blocks = _i(run, "Num Blocks X") * _i(run, "Num Blocks Y") * _i(run, "Num Blocks Z")
    by_warps = math.floor(arch["max_warps_per_sm"] / warps_per_block)
    by_shared = math.floor(arch["total_shared"] / shared_estimate(run))
    by_regs = math.floor(arch["max_regs_per_sm"] / regs_per_block) if regs_per_block else by_warps
    bps = min(by_warps, by_shared, by_regs, math.ceil(total_blocks / arch["num_sm"]))
    bps = max(min(bps, arch["max_blocks_per_sm"]), 1.0)
    return warps_per_block * bps, bps


def _phase2_global(run, e, x, y, z, dim, arch):
    """Global loads per thread in phase 2 after L1 hits (the 'fermi' cache
    model of run-model.py:329-420, keyed on phase2_global_loads)."""
    g2 = float(run["phase2_global_loads"])
    cap_bytes = arch["l1_model_bytes"]

    def cached(miss_num, tile_bytes):
        miss = miss_num / (g2 * e)
        hit = 1.0 - miss
        cap = cap_bytes / tile_bytes
        if cap < 1.0:
            hit *= cap
        return (1.0 - hit) * g2 * e

    if dim == 3 and g2 == 7.0:
        return cached(3.0 * e + 4.0, (y * e + 2) * (x + 2) * (z + 2) * 4.0)
    if dim == 3 and g2 == 27.0:
        return 9.0 * e + 18.0
    if dim == 2 and g2 == 5.0:
        return cached(e + 4.0, (y * e + 2) * (x + 2) * 4.0)
    if dim == 2 and g2 == 9.0:
        return min(3 * e + 6.0, g2 * e)
    if dim == 2 and g2 == 7.0:
        return cached(2.0 * e + 5.0, (y * e + 2) * (x + 2) * (z + 2) * 4.0)
    if dim == 2 and g2 == 13.0:
        return min(e + 4.0, g2 * e)
    return g2 * e  # no formula for this load count: no cache


def simulate(run, arch):
    """Simulated seconds for one run (run-model.py:205-560) and the terms."""
    x, y, z = _i(run, "Block Size X"), _i(run, "Block Size Y"), _i(run, "Block Size Z")
    e, t, dim = _i(run, "Elements/Thread"), _i(run, "Time Tile Size"), _i(run, "Dimensions")
    steps = _i(run, "Time Steps")
    phase_limit = _i(run, "phase_limit", 0)
    aw, bps = occupancy(run, arch)
    total_blocks = _i(run, "Num Blocks X") * _i(run, "Num Blocks Y") * _i(run, "Num Blocks Z")
    num_stages = math.ceil(total_blocks / (bps * arch["num_sm"]))
    full = steps // t
    extra = steps % t
    extra_global = 1 if extra > 0 else 0
    extra_shared = max(0, extra - 1)

    p2_glb = _phase2_global(run, e, x, y, z, dim, arch)
    g2 = float(run["phase2_global_loads"])
    p2_shd = float(run["phase2_shared_loads"]) * e + (g2 * e - p2_glb)
    p3_shd = float(run["phase3_shared_loads"]) * e
    k_op = (float(run["compute_per_point"]) - 1.0) * e
    k_sfu = 1.0 * e
    c_load, c_op = arch["c_load"], arch["c_op"]
    Bp = arch["B_gmem"] + (1.0 + 1.0 / (x / 32.0))
    t_glb = max(c_load * (p2_glb + p2_shd) * aw + c_op * k_op * aw + arch["sfu_glb"] * k_sfu * aw,
                arch["L_gmem"] + c_load + max(Bp * p2_glb * aw, arch["B_smem"] * p2_shd * aw))
    t_shd = max(c_load * p3_shd * aw + c_op * k_op * aw + arch["sfu_shd"] * k_sfu * aw,
                arch["L_smem"] + c_load + arch["B_smem"] * p3_shd * aw)
    write_back = arch["L_gmem"] + c_load + arch["B_gmem"] * float(run["phase4_global_stores"]) * aw
    a1, b1 = arch["phase1"]
    t_phase1 = (a1 * e + b1) * aw
    if phase_limit == 1:
        t_stage, t_extra = 0.0, 0.0
    elif phase_limit == 2:
        t_stage, t_extra = t_glb + write_back, extra_global * t_glb
    elif phase_limit == 3:
        t_stage, t_extra = (t - 1) * t_shd, extra_shared * t_shd
    else:
        t_stage = t_glb + (t - 1) * t_shd + write_back
        t_extra = extra_global * t_glb + extra_shared * t_shd + extra_global * write_back
    t_stage += t_phase1
    if extra_global:
        t_extra += t_phase1
    clk = (t_stage * num_stages + arch["launch_penalty"]) * full
    if extra_global:
        clk += t_extra * num_stages + arch["launch_penalty"]
    return clk / arch["clock"], dict(active_warps=aw, blocks_per_sm=bps, num_stages=num_stages,
                                     t_glb=t_glb, t_shd=t_shd, t_phase1=t_phase1,
                                     write_back=write_back, p2_glb=p2_glb)


def runs_from_records(records, constants):
    """Sweep records (ots.sweep / ots.dataset) -> run dicts with the runner's
    key names; tile-kernel runs of stencils with model constants only."""
    out = []
    for r in records:
        if r.get("status") != "ok" or r.get("kernel", "tile") != "tile":
            continue
        c = constants.get(r["stencil"])
        if c is None:
            continue
        g = r["geom"]
        run = {"stencil": r["stencil"], "Block Size X": r["bx"], "Block Size Y": r["by"],
               "Block Size Z": r["bz"], "Elements/Thread": r["E"], "Time Tile Size": r["T"],
               "Dimensions": g["dims"], "Register Usage": g["registers"],
               "Num Blocks X": g["num_blocks"][0], "Num Blocks Y": g["num_blocks"][1],
               "Num Blocks Z": g["num_blocks"][2], "Time Steps": r["steps"], "phase_limit": 0,
               "e_axis": g.get("e_axis", 1), "EventElapsed": r["seconds"],
               "gupdates": r["gupdates"]}
        run.update(c)
        out.append(run)
    return out


def rank(runs, arch):
    """Runs the model can rank (registers below the cap), sorted by simulated
    time; each run gets 'sim_elapsed'."""
    keep = []
    for run in runs:
        if _i(run, "Register Usage") >= arch["max_regs_per_thread"] - 1:
            continue  # at the register cap: spills (run-model.py:235-236)
        run = dict(run)
        run["sim_elapsed"] = simulate(run, arch)[0]
        keep.append(run)
    keep.sort(key=lambda q: q["sim_elapsed"])
    return keep


def evaluate(runs, arch, k_frac=0.10):
    """Per stencil: the model's pick against the measured best (as time
    ratios, and as the reference's percent slowdowns)."""
    by = {}
    for run in runs:
        by.setdefault(run.get("stencil", "?"), []).append(run)
    report = {}
    for s, rs in sorted(by.items()):
        ranked = rank(rs, arch)
        if not ranked:
            continue
        best_t = min(float(q["EventElapsed"]) for q in rs)
        n1 = max(1, int(math.ceil(len(rs) * 0.01)))
        k = max(1, int(math.floor(k_frac * len(rs))))
        top1_t = float(ranked[0]["EventElapsed"])
        one_pct = min(float(q["EventElapsed"]) for q in ranked[:n1])
        topk = min(float(q["EventElapsed"]) for q in ranked[:k])
        pred = [q["sim_elapsed"] for q in ranked]
        act = [float(q["EventElapsed"]) for q in ranked]
        report[s] = {
            "space": len(rs), "ranked": len(ranked), "k": k,
            "top1_over_best": best_t / top1_t, "topk_over_best": best_t / topk,
            "best_overall_pct": (top1_t / best_t - 1.0) * 100.0,
            "best_one_percent_pct": (one_pct / best_t - 1.0) * 100.0,
            "spearman": _spearman(pred, act),
            "picked_config": {q: ranked[0][q] for q in ("Block Size X", "Block Size Y",
                                                       "Block Size Z", "Time Tile Size",
                                                       "Elements/Thread")},
        }
    if report:
        report["_mean"] = {q: sum(v[q] for v in report.values()) / len(report)
                           for q in ("top1_over_best", "topk_over_best", "best_overall_pct",
                                     "spearman")}
    return report


def _spearman(a, b):
    n = len(a)
    if n < 3:
        return 0.0

    def ranks(v):
        order = sorted(range(n), key=lambda i: v[i])
        r = [0.0] * n
        for pos, i in enumerate(order):
            r[i] = float(pos)
        return r

    ra, rb = ranks(a), ranks(b)
    ma, mb = sum(ra) / n, sum(rb) / n
    cov = sum((p - ma) * (q - mb) for p, q in zip(ra, rb))
    va = math.sqrt(sum((p - ma) ** 2 for p in ra))
    vb = math.sqrt(sum((q - mb) ** 2 for q in rb))
    return cov / (va * vb) if va > 0 and vb > 0 else 0.0


def read_dat(path):
    """A results CSV as scripts/results-to-csv.py writes it (header row and
    data rows each ending in a comma)."""
    with open(path) as fh:
        rows = list(csv.reader(fh))
    hdr = [h for h in rows[0] if h != ""]
    return [dict(zip(hdr, r[:len(hdr)])) for r in rows[1:] if len(r) >= len(hdr)]


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawTextHelpFormatter)
    ap.add_argument("--data", help="sweep records JSON (ots.dataset / ots.sweep)")
    ap.add_argument("--dat", help="results CSV in the reference's .dat layout")
    ap.add_argument("--arch", default="b200", choices=sorted(ARCH))
    ap.add_argument("--report")
    a = ap.parse_args(argv)
    arch = get_arch(a.arch)
    if a.data:
        from . import STENCILS, model_constants
        recs = json.load(open(a.data))
        recs = recs["records"] if isinstance(recs, dict) else recs
        consts = {s: model_constants(s) for s in STENCILS}
        runs = runs_from_records(recs, consts)
    elif a.dat:
        runs = read_dat(a.dat)
        for r in runs:
            r.setdefault("stencil", os.path.basename(a.dat))
    else:
        ap.error("give --data or --dat")
    rep = evaluate(runs, arch)
    for s, v in rep.items():
        if s == "_mean":
            continue
        print("%-18s ranked=%4d top1/best=%.3f top-k/best=%.3f  Best Overall: %.1f %%  "
              "Best One Percent: %.1f %%  rho=%.2f" % (s, v["ranked"], v["top1_over_best"],
                                                       v["topk_over_best"], v["best_overall_pct"],
                                                       v["best_one_percent_pct"], v["spearman"]))
    if "_mean" in rep:
        print("MEAN", json.dumps(rep["_mean"]))
    if a.report:
        with open(a.report, "w") as fh:
            json.dump(rep, fh, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
