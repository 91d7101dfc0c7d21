#!/usr/bin/env python3
"""Benchmark: FP32 Jacobi-3D 7-point, 512^3 interior, 100 time steps.

One "step" of this bench is one full run of the workload (100 time steps over
the 512^3 grid, ceil(100/T) kernel launches).  Reported metric: grid-point
updates per second (GUpdates/s = 512^3 * 100 / time), whole job over all
ranks.

  value    device time (CUDA events on the plan's stream) with the input
           resident in HBM; the z-streamed time-tiled kernel with the
           exhaustive-sweep-tuned (T, block, E) from tuned.json.
  e2e      the same metric through the public C ABI with host buffers, wall
           clock: each step uploads its dense 512^3 input from page-locked
           memory (ots_upload_interior_async), runs the 100 steps and
           downloads the result (ots_download_interior_async); three plans
           (--e2e-depth) rotate, so a step's host-to-device copy, the
           previous step's kernels and the one before's device-to-host copy
           run at the same time.
  plain    the plain one-step-per-launch kernel, same device timing, and the
           strongest one-step kernel we have (the z-streamed kernel at T=1
           in its best block shape): the >= 2x target's comparator is
           plain.best_one_step (speedup_vs_best_one_step).
  learned  the learned picker live: the shipped cost model ranks the whole
           configuration space from geometry alone, the top 10 % (with the
           plain kernel) are measured, the best is kept; reported with its
           configuration, how many were measured, and its ratio to the
           exhaustive-sweep best (value).
  roofline HBM: algorithmic bytes per launch (read + write each cell once,
           8 B x 512^3) / average launch time, against the measured copy
           bandwidth in MEASURED_PEAKS.json.
  cpu_baseline  the CPU oracle (a C restatement of the reference's per-point
           arithmetic) on a bounded sample of the same grid, one core.

Inputs (2 x 537 MB) are larger than the 126 MB L2, so no flush is needed.

--impl reference times the reference's CPU path (the oracle restatement;
the reference's own jacobi-3d CPU check indexes out of bounds and cannot
run) on all host cores, on a bounded sample of the same workload.

Multi-GPU: replicas only (the reference is single-device): each rank runs
its own 512^3 problem on its own GPU; the timed region is bracketed by
barriers and the time is the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ics-12-overlapped-tiling_b200"))

N, STEPS = 512, 100
STENCIL = "jacobi-3d"
BYTES_PER_UPDATE = 8.0       # read + write each cell once per launch (T=1 equivalent)
FLOPS_PER_UPDATE = 7.0       # reference constant, opencl/jacobi-3d/jacobi-3d.cpp:915-917
DEFAULT_CFG = dict(kernel="stream", T=4, bx=32, by=8, bz=1, E=4)


def tuned_config(key="jacobi-3d/512/100"):
    path = os.path.join(ROOT, "ics-12-overlapped-tiling_b200", "ots", "tuned.json")
    try:
        with open(path) as fh:
            cfg = json.load(fh)[key]
        return dict(kernel=cfg["kernel"], T=cfg["T"], bx=cfg["bx"], by=cfg["by"], bz=cfg.get("bz", 1),
                    E=cfg["E"]), "exhaustive-sweep best (tuned.json)"
    except Exception:
        if key.endswith("one-step"):
            return dict(kernel="stream", T=1, bx=16, by=8, bz=1, E=4), "default"
        return dict(DEFAULT_CFG), "default"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            m = json.load(fh)
        return float(m["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def bound_at_T(stencil, T, bytes_per_update, hbm_gbs, sm_count=148):
    """The roofline that bounds a configuration at time-tile depth T:
    min(HBM x T / B_u, FP32 / F_u) in GUpdates/s -- a launch reads and writes
    B_u bytes per cell once and advances T steps; FP32 = SMs x 128 lanes x
    the maximum SM clock (MEASURED_PEAKS.json sm_max_mhz), one scalar
    operation per lane and clock; F_u the operations per update of the
    measured (baseline) arithmetic."""
    sys.path.insert(0, os.path.join(ROOT, "ics-12-overlapped-tiling_b200"))
    from ots.model import STENCIL_COST
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            mhz = float(json.load(fh).get("sm_max_mhz", 1965.0))
    except Exception:
        mhz = 1965.0
    mem = hbm_gbs * T / bytes_per_update
    fp = sm_count * 128 * mhz * 1e6 / STENCIL_COST[stencil][0] / 1e9
    return {"gupdates": min(mem, fp), "bound": "hbm" if mem <= fp else "fp32",
            "hbm_x_T_over_bytes": mem, "fp32_over_ops": fp, "T": T}


def profile_traffic(kernel):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as fh:
            t = json.load(fh)
        e = t.get("%s/%s" % (STENCIL, kernel))
        return None if e is None else float(e["bytes_per_launch_full"])
    except Exception:
        return None


class Clocks:
    """Samples nvidia-smi (with its timestamps) around the timed region.
    nvidia-smi takes a moment to start, so the sampler is started first and
    the timed region begins only once the first sample is in; mark() brackets
    the region, and the summary keeps the samples taken inside it (at least
    the one before and the one after)."""

    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", "ots_clocks_%d.csv" % os.getpid())
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
            deadline = time.time() + 10.0
            while time.time() < deadline and self.proc.poll() is None:
                self.fh.flush()
                if os.path.getsize(self.path) > 0:
                    break
                time.sleep(0.05)
        except Exception:
            self.proc = None
        return self

    def mark(self, which):
        if which == "start":
            self.t0 = time.time()
        else:
            self.t1 = time.time()

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.1)  # one more sample after the region
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        try:
            self.fh.close()
        except Exception:
            pass

    @staticmethod
    def _stamp(text):
        import datetime
        try:
            return datetime.datetime.strptime(text, "%Y/%m/%d %H:%M:%S.%f").timestamp()
        except ValueError:
            return None

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 8:
                    rows.append((self._stamp(parts[0]), parts[1:]))
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        inside = rows
        if self.t0 is not None and self.t1 is not None and all(t is not None for t, _ in rows):
            inside = [r for r in rows if self.t0 <= r[0] <= self.t1]
            before = [r for r in rows if r[0] < self.t0][-1:]
            after = [r for r in rows if r[0] > self.t1][:1]
            if not inside:
                inside = before + after
        vals = [v for _, v in inside]
        sm = sorted(float(r[0]) for r in vals if r[0].replace(".", "").isdigit())
        mx = max((float(r[1]) for r in vals if r[1].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in vals for i in range(4) if r[3 + i] == "Active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx,
                "reasons": reasons, "samples": len(vals)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reduce_max(t, world):
    """Max over ranks (the slowest replica sets the job's time)."""
    if world == 1:
        return t
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    x = torch.tensor([t], dtype=torch.float64, device=dev)
    dist.all_reduce(x, op=dist.ReduceOp.MAX)
    return float(x.item())


def job_value(updates_per_rank, world, seconds_max):
    """Whole-job GUpdates/s: every rank's updates over the slowest rank's time."""
    return float(updates_per_rank) * world / seconds_max / 1e9


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_sample(threads, target_s):
    """Time the CPU oracle on 512^3 with as many steps as fit ~target_s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle as O  # the checker, used here only as the CPU baseline
    O.set_threads(threads)
    pad = 1
    P = N + 2 * pad
    x = O.fill_ref(3, P, pad, P - pad, 123456, 1)[0]
    t0 = time.perf_counter()
    O.sweep_f32(STENCIL, [x], steps=1, lo=pad, hi=P - pad, coef=float(np.float32(1.0 / 7.0)))
    one = time.perf_counter() - t0
    k = max(1, min(100, int(target_s / max(one, 1e-3))))
    t0 = time.perf_counter()
    O.sweep_f32(STENCIL, [x], steps=k, lo=pad, hi=P - pad, coef=float(np.float32(1.0 / 7.0)))
    el = time.perf_counter() - t0
    return float(N) ** 3 * k / el / 1e9, k, el


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.set_threads(threads)
    pad = 1
    P = N + 2 * pad
    x = O.fill_ref(3, P, pad, P - pad, 123456, 1)[0]
    sample_steps = 4  # several steps per call amortise the per-call array copies
    coef = 1.0 / 7.0
    for _ in range(args.warmup):
        O.sweep_f32(STENCIL, [x], steps=1, lo=pad, hi=P - pad, coef=coef)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.sweep_f32(STENCIL, [x], steps=sample_steps, lo=pad, hi=P - pad, coef=coef)
    el = time.perf_counter() - t0
    v = float(N) ** 3 * sample_steps * args.steps / el / 1e9
    sample = "512^3 x %d time steps per bench step (of the workload's 100), %d threads" % (
        sample_steps, threads)
    print(json.dumps({
        "impl": "reference", "metric": "GUpdates/s", "value": v, "unit": "GUpdates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (srand(123456) uniform [0,1))",
        "config": {"workload": "jacobi-3d 7-point FP32, 512^3 interior, 100 steps, zero Dirichlet",
                   "sample": sample},
        "cpu_baseline": {"value": v, "unit": "GUpdates/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": "GUpdates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))
    return 0


def cpu_rate(fn, updates_per_step, max_steps, target_s):
    """GUpdates/s of `fn(k)` (k steps) on a bounded sample: one step first,
    then as many steps as fit about `target_s`."""
    t0 = time.perf_counter()
    fn(1)
    one = time.perf_counter() - t0
    k = max(1, min(max_steps, int(target_s / max(one, 1e-3))))
    if k == 1:
        return updates_per_step / one / 1e9, 1, one
    t0 = time.perf_counter()
    fn(k)
    el = time.perf_counter() - t0
    return updates_per_step * k / el / 1e9, k, el


def run_configs(args):
    """--configs: every workload of ots.workloads at its full size.  Per
    workload: the exhaustive sweep's best, the learned pick (best measured of
    the cost model's top 10 %), the plain one-step kernel, the CPU path on one
    thread (the reference's own loop where it compiles, else the oracle
    restatement) and on all host threads (bounded samples), and the result of
    the best configuration checked against the CPU oracle: bit for bit
    against the FP32 restatement, max / RMS error against the FP64 one.
    One JSON line per workload on stdout; all of them in --configs-out."""
    import numpy as np
    import ots
    from ots import workloads as W
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # the checker and the CPU baselines
    threads = os.cpu_count() or 1
    peak, peak_src = peaks()
    want = None if args.configs == "all" else set(args.configs.split(","))
    lines = []
    for w in W.WORKLOADS:
        st = w["stencil"]
        if want and W.workload_key(w) not in want:
            continue
        t_start = time.time()
        done = [0]

        def progress(rec):
            done[0] += 1
            if done[0] % 50 == 0:
                sys.stderr.write("%s: %d configurations, %.0f s\n" % (
                    w["name"], done[0], time.time() - t_start))

        recs = W.sweep_workload(w, log=progress)
        ok = [r for r in recs if r.get("status") == "ok"]
        best = max(ok, key=lambda r: r["gupdates"])
        cm, cm_desc = W.model_for(st)
        pk = W.picks(st, recs, cm)
        cm.close()
        plain = W.plain_record(w)
        t_sweep = time.time() - t_start
        line = {"workload": w["name"], "stencil": st, "variant": w.get("variant", "baseline"),
                "n": w["n"], "steps": w["steps"],
                "space": len(ok), "invalid": len(recs) - len(ok),
                "exhaustive": {"gupdates": best["gupdates"], "config": W.config_of(best)},
                "learned": {"gupdates": pk["picked"]["gupdates"],
                            "config": W.config_of(pk["picked"]), "k": pk["k"],
                            "measured": pk["measured"],
                            "over_best": pk["picked"]["gupdates"] / best["gupdates"],
                            "top1_gupdates": pk["top1"]["gupdates"],
                            "top1_config": W.config_of(pk["top1"]),
                            "top1_over_best": pk["top1"]["gupdates"] / best["gupdates"],
                            "model": cm_desc},
                "plain": {"gupdates": plain.get("gupdates"), "config": W.config_of(plain)},
                "speedup_vs_plain": best["gupdates"] / plain["gupdates"]
                if plain.get("gupdates") else None,
                "gpu_sweep_seconds": t_sweep}
        bpu = W.BYTES_PER_UPDATE[st]
        line["one_step_hbm_roofline"] = {
            "gupdates": peak / bpu, "bytes_per_update": bpu, "peak_gbs": peak,
            "peak_source": peak_src, "best_over_roofline": best["gupdates"] / (peak / bpu)}
        bt = bound_at_T(st, best["T"], bpu, peak)
        bt["best_over_bound"] = best["gupdates"] / bt["gupdates"]
        line["bound_T"] = bt
        if st == "jacobi-2d":  # the T sweep at 16 x 16 blocks the workload names
            ts = W.sweep_workload(w, [dict(kernel="tile", T=T, bx=16, by=16, bz=1, E=1)
                                      for T in range(1, 9)])
            line["tile_16x16_by_T"] = {str(r["T"]): r.get("gupdates") for r in ts}

        # the best configuration's result against the CPU oracle
        g, pst, pax, got = W.run_config(w, W.config_of(best))
        lo, hi = g.padding, g.padding + g.real_size
        sl = tuple(slice(lo, hi) for _ in range(g.dims))
        O.set_threads(threads)
        t0 = time.perf_counter()
        want32 = O.sweep_f32(st, pst, pax, steps=w["steps"], lo=lo, hi=hi, coef=g.coef, h2=g.h2)
        t32 = time.perf_counter() - t0
        bitwise = all(np.array_equal(a[sl].view(np.uint32), b[sl].view(np.uint32))
                      for a, b in zip(got, want32))
        # the parity tests' metric: max |gpu - cpu| / max(|cpu|, 1)
        vs32 = max(float(np.max(np.abs(a[sl].astype(np.float64) - b[sl]) /
                                np.maximum(np.abs(b[sl]), 1.0))) for a, b in zip(got, want32))
        t0 = time.perf_counter()
        want64 = O.sweep_f64(st, pst, pax, steps=w["steps"], lo=lo, hi=hi, coef=g.coef, h2=g.h2)
        t64 = time.perf_counter() - t0

        def errors(res):
            out = []
            for a, b in zip(res, want64):
                mr, rms = O.error_vs_f64(a, b, lo, hi, floor=1e-6)
                ref_max = float(np.max(np.abs(b[sl])))
                max_abs = float(np.max(np.abs(a[sl].astype(np.float64) - b[sl])))
                out.append({"max_rel": mr, "rms": rms, "max_abs": max_abs,
                            "max_abs_over_max_ref": max_abs / ref_max if ref_max else None})
            return out

        fields, fields32 = errors(got), errors(want32)
        del want32, want64
        line["check"] = {"config": W.config_of(best), "bitwise_equal_fp32_oracle": bool(bitwise),
                         "max_rel_diff_vs_fp32_oracle": vs32,
                         "fp64": fields, "fp32_oracle_vs_fp64": fields32, "max_rel_floor": 1e-6,
                         "cpu_seconds": {"fp32": t32, "fp64": t64, "threads": threads}}

        # CPU baselines on bounded samples of the same grid
        x0 = [a.copy() for a in pst]
        upd = float(g.interior_points)
        if st in O.REF_LOOPS and O.ref_available():
            fn1 = lambda k: O.ref_loop(st, x0[0], g.padding, k)
            kind = "reference"
        else:
            def fn1(k):
                O.set_threads(1)
                O.sweep_f32(st, x0, pax, steps=k, lo=lo, hi=hi, coef=g.coef, h2=g.h2)
            kind = "port"
        v1, k1, e1 = cpu_rate(fn1, upd, w["steps"], 5.0)
        O.set_threads(threads)
        vn, kn, en = cpu_rate(lambda k: O.sweep_f32(st, x0, pax, steps=k, lo=lo, hi=hi,
                                                    coef=g.coef, h2=g.h2),
                              upd, w["steps"], 5.0)
        line["cpu_one_thread"] = {"value": v1, "unit": "GUpdates/s", "cores": 1, "kind": kind,
                                  "sample": "%d of %d steps (%.1f s)" % (k1, w["steps"], e1)}
        line["cpu_all_threads"] = {"value": vn, "unit": "GUpdates/s", "cores": threads,
                                   "kind": "port",
                                   "sample": "%d of %d steps (%.1f s)" % (kn, w["steps"], en)}
        line["seconds"] = time.time() - t_start
        print(json.dumps(line), flush=True)
        # every measured configuration (with the geometry the cost model
        # reads), so pickers can be re-evaluated offline on the full sizes
        line["records"] = [{k: r[k] for k in ("kernel", "T", "bx", "by", "bz", "E", "status",
                                              "gupdates", "geom") if k in r} for r in recs]
        lines.append(line)
        if args.configs_out:  # rewritten after every workload
            with open(args.configs_out, "w") as fh:
                json.dump({"device": ots.device_info(0)["name"], "host_threads": threads,
                           "workloads": lines}, fh, indent=1)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the live learned pick")
    ap.add_argument("--e2e-depth", type=int, default=3,
                    help="plans in flight in the end-to-end leg (each holds 2 x 537 MB)")
    ap.add_argument("--configs", help="measure the listed workloads (stencil names, comma "
                    "separated, '<stencil>-fast' for a fast-division row, or 'all') at full "
                    "size instead of the bench line")
    ap.add_argument("--configs-out", help="write the --configs results to this JSON file")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        return run_reference(args)
    if args.configs:
        return run_configs(args)

    world, rank, local = dist_setup()
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import ots

    cfg, cfg_src = tuned_config()
    plan = ots.Plan(STENCIL, N, STEPS, device=local, **cfg)
    g = plan.geometry
    state, aux = plan.fill_reference(seed=123456 + rank)
    plan.upload(state, aux)
    sl = tuple(slice(g.padding, g.padding + g.real_size) for _ in range(g.dims))
    inner = ([np.ascontiguousarray(a[sl]) for a in state], [np.ascontiguousarray(a[sl]) for a in aux])
    stream = torch.cuda.ExternalStream(plan.stream_ptr(), device=local)
    launches_per_step = g.launches

    def timed(kernel, k):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier(world)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(k):
            plan.run_async(kernel)
        e1.record(stream)
        plan.sync()
        torch.cuda.synchronize()
        barrier(world)
        return e0.elapsed_time(e1) / 1e3

    # warm-up
    for _ in range(args.warmup):
        plan.run_async(cfg["kernel"])
    plan.sync()
    with Clocks(local) as clk:
        clk.mark("start")
        el = timed(cfg["kernel"], args.steps)
        clk.mark("end")
    el_max = reduce_max(el, world)
    value = job_value(float(N) ** 3 * STEPS * args.steps, world, el_max)
    avg_launch = el / (args.steps * launches_per_step)

    # plain one-step comparator (same plan, same data)
    for _ in range(max(1, args.warmup // 3)):
        plan.run_async("plain")
    plan.sync()
    el_plain = reduce_max(timed("plain", max(1, args.steps // 2)), world)
    plain_value = float(N) ** 3 * STEPS * max(1, args.steps // 2) * world / el_plain / 1e9
    # the z-streamed kernel at T=1 (its best block shape from the same sweep)
    # is the strongest one-step-per-launch kernel we have
    plain_best = plain_value
    c1, _ = tuned_config("jacobi-3d/512/100/one-step")
    try:
        p1 = ots.Plan(STENCIL, N, STEPS, device=local, kernel="stream", T=1, bx=c1["bx"],
                      by=c1["by"], bz=1, E=c1["E"])
        p1.upload_interior(*inner)
        s1 = torch.cuda.ExternalStream(p1.stream_ptr(), device=local)
        for _ in range(2):
            p1.run_async()
        p1.sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s1)
        for _ in range(max(1, args.steps // 2)):
            p1.run_async()
        e1.record(s1)
        p1.sync()
        t1 = reduce_max(e0.elapsed_time(e1) / 1e3, world)
        stream_t1 = float(N) ** 3 * STEPS * max(1, args.steps // 2) * world / t1 / 1e9
        plain_best = max(plain_best, stream_t1)
        p1.close()
    except Exception:
        stream_t1 = None

    # end to end through the C ABI with page-locked host buffers: every step
    # uploads its own input, runs the 100 steps and downloads its result; the
    # plans rotate on their own streams, so the copy engines (one per
    # direction) and the kernels work on three different problems at once
    # (ots_upload_interior_async / ots_run_async / ots_download_interior_async)
    e2e = None
    latency_ms = None
    if not args.no_e2e:
        depth = max(1, args.e2e_depth)
        plans = [plan] + [ots.Plan(STENCIL, N, STEPS, device=local, **cfg) for _ in range(depth - 1)]
        host_in = [np.ascontiguousarray(a, np.float32) for a in inner[0]]
        aux_in = [np.ascontiguousarray(a, np.float32) for a in inner[1]]
        host_out = [[np.zeros_like(a) for a in host_in] for _ in range(depth)]
        L = ots.lib()
        pinned = host_in + aux_in + [a for o in host_out for a in o]
        for a in pinned:
            ots.check(L.ots_host_register(a.ctypes.data, a.nbytes))
        h2d = sum(a.nbytes for a in host_in + aux_in)
        d2h = sum(a.nbytes for a in host_out[0])

        def e2e_step(s):
            pl = plans[s % depth]
            pl.upload_interior_async(host_in, aux_in)
            pl.run_async(cfg["kernel"])
            pl.download_interior_async(host_out[s % depth])

        for s in range(depth):  # warm-up: every plan once
            e2e_step(s)
        for pl in plans:
            pl.sync()
        # latency of one problem alone: upload, 100 steps, download (wall)
        lat = []
        for _ in range(3):
            t0 = time.perf_counter()
            plan.upload_interior_async(host_in, aux_in)
            plan.run_async(cfg["kernel"])
            plan.download_interior_async(host_out[0])
            plan.sync()
            lat.append(time.perf_counter() - t0)
        latency_ms = sorted(lat)[1] * 1e3
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for s in range(args.steps):
            e2e_step(s)
        for pl in plans:
            pl.sync()
        torch.cuda.synchronize()
        t_e2e = reduce_max(time.perf_counter() - t0, world)
        barrier(world)
        same = all(np.array_equal(a.view(np.uint32), b.view(np.uint32))
                   for o in host_out[1:] for a, b in zip(host_out[0], o))
        for a in pinned:
            L.ots_host_unregister(a.ctypes.data)
        for pl in plans[1:]:
            pl.close()
        e2e = {"value": job_value(float(N) ** 3 * STEPS * args.steps, world, t_e2e),
               "unit": "GUpdates/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "pipeline": "%d plans rotate on their own streams; each step: upload its "
                           "input, 100 steps, download its result (wall clock, all copies in)" % depth,
               "results_identical_across_plans": bool(same),
               "latency_ms_one_problem": latency_ms,
               "latency_note": "one problem alone through the same calls: its upload, "
                               "100 steps and download in sequence (wall clock, median of 3)"}

    # the learned picker live on the same workload (rank 0 measures; the
    # picker is a host-side tool, not part of the timed job)
    learned = None
    if not args.no_learned and rank == 0:
        try:
            from ots import model as M
            from ots import workloads as W
            with open(os.path.join(ROOT, "ics-12-overlapped-tiling_b200", "ots", "data",
                                   "cost_model.json")) as fh:
                cm = M.MLP.from_json(json.load(fh), device=local)
            best_l, k, size = W.learned_pick(dict(stencil=STENCIL, n=N, steps=STEPS), cm,
                                             device=local)
            cm.close()
            learned = {"gupdates": best_l["gupdates"], "config": W.config_of(best_l),
                       "measured": k + 1, "space": size,
                       "over_exhaustive_best": best_l["gupdates"] / (value / world),
                       "model": "shipped cost model (ots/data/cost_model.json)"}
        except Exception as e:  # report, never fake
            learned = {"error": str(e)}

    peak, peak_src = peaks()
    bytes_per_launch = BYTES_PER_UPDATE * float(N) ** 3
    achieved = bytes_per_launch / avg_launch / 1e9
    traffic = profile_traffic(cfg["kernel"])
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "peak_source": peak_src + " (MEASURED_PEAKS.json hbm_gbs)",
                "note": "achieved = compulsory 8 B/cell per launch; each launch advances T steps"}

    cpu = None
    if rank == 0 and not args.no_cpu:
        try:
            v, k, el_cpu = cpu_sample(1, 10.0)
            cpu = {"value": v, "unit": "GUpdates/s", "cores": 1, "kind": "port",
                   "sample": "512^3 x %d time steps (%.1f s), single thread" % (k, el_cpu)}
        except Exception as e:  # report, never fake
            cpu = {"value": None, "unit": "GUpdates/s", "cores": 1, "kind": "port",
                   "sample": "failed: %s" % e}

    line = {
        "metric": "GUpdates/s", "value": value, "unit": "GUpdates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el_max / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: srand(123456) rand()/(RAND_MAX+1) interior, zero Dirichlet ring",
        "config": {"workload": "jacobi-3d 7-point FP32, 512^3 interior, 100 steps, weight 1/7",
                   "kernel": cfg["kernel"], "T": cfg["T"], "block": [cfg["bx"], cfg["by"], cfg["bz"]],
                   "E": cfg["E"], "config_source": cfg_src, "parallelism": "replicas x%d" % world,
                   "l2": "inputs larger than L2 (2 x 537 MB vs 126 MB); no flush"},
        "plain": {"value": plain_value, "unit": "GUpdates/s", "kernel": "plain one-step",
                  "stream_T1": stream_t1,
                  "stream_T1_config": [c1["bx"], c1["by"], c1["E"]],
                  "best_one_step": plain_best,
                  "speedup_vs_plain": value / plain_value if plain_value else None,
                  "speedup_vs_best_one_step": value / plain_best if plain_best else None},
        "learned": learned,
        "gpu_launches": launches_per_step * args.steps,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clk.summary(),
        "flops": {"per_update": FLOPS_PER_UPDATE,
                  "tflops": value * FLOPS_PER_UPDATE / 1e3},
    }
    if rank == 0:
        print(json.dumps(line))
    plan.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
