"""The drop-in runner CLI on the GPU: the reference's Key: value protocol and
its -v check, the -c phase-clock dump, the -p phase-limited kernels, and the
YAML experiment harness driving the CLI end to end into a .dat CSV that the
analytical model reads."""
import os
import subprocess

import numpy as np
import pytest

import ots
from ots import analytic as A
from ots import harness as H

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "ics-12-overlapped-tiling_b200", "bin")


def cli(stencil, *args, timeout=120):
    r = subprocess.run([os.path.join(BIN, "ots-" + stencil)] + [str(a) for a in args],
                       capture_output=True, text=True, timeout=timeout)
    kv = {}
    for line in r.stdout.splitlines():
        if ":" in line:
            k, v = line.split(":", 1)
            kv[k.strip()] = v.strip()
    return r, kv


REF_KEYS = ["Time Tile Size", "Block Size X", "Block Size Y", "Num Blocks X", "Num Blocks Y",
            "Elements/Thread", "Shared Size", "Total FP/Block", "Useful FP/Block", "Useful Ratio",
            "Global Loads/Block", "Global Stores/Block", "Shared Loads/Block",
            "Shared Stores/Block", "Real Per Block X", "Real Per Block Y", "Padded Size",
            "Time Steps", "Register Usage", "EventElapsed", "ProfileTimerResolution",
            "Elapsed Time", "Actual GFlop/s", "Real Size", "Device GFlop/s", "phase2_global_loads",
            "phase2_shared_loads", "compute_per_point", "phase3_shared_loads",
            "phase4_global_stores", "shared_stores", "num_fields", "data_size", "Dimensions"]


@pytest.mark.gpu
@pytest.mark.parametrize("stencil,args", [
    ("jacobi-2d", ["-n", 500, "-t", 12, "-s", 4, "-x", 32, "-y", 8, "-e", 2]),
    ("jacobi-1d", ["-n", 100000, "-t", 9, "-s", 3, "-x", 128, "-e", 4]),
    ("gradient-2d", ["-n", 300, "-t", 6, "-s", 2, "-x", 16, "-y", 16]),
    ("rician-denoise-2d", ["-n", 300, "-t", 6, "-s", 2, "-x", 16, "-y", 16]),
])
def test_cli_protocol_and_verify(stencil, args):
    r, kv = cli(stencil, "-v", *args)
    assert r.returncode == 0, r.stdout + r.stderr
    for k in REF_KEYS:
        if stencil == "jacobi-1d" and k in ("Block Size Y", "Num Blocks Y", "Real Per Block Y"):
            continue
        assert k in kv, k
    assert kv["Correctness"] == "PASSED"
    assert float(kv["Error Norm"]) <= 1e-2 * float(kv["Ref Norm"])
    assert 0.0 < float(kv["Useful Ratio"]) <= 1.0


@pytest.mark.gpu
def test_cli_reports_reference_errors():
    r, _ = cli("jacobi-2d", "-n", 256, "-t", 4, "-s", 9, "-x", 16, "-y", 4)
    assert r.returncode == 1 and "ERROR" in r.stdout
    r, _ = cli("jacobi-2d", "-n", 256, "-t", 4, "-s", 1, "-x", 64, "-y", 32)
    assert r.returncode == 1 and "too large" in r.stdout


@pytest.mark.gpu
def test_clock_dump_records_every_warp_in_phase_order():
    with ots.Plan("jacobi-2d", 300, 8, T=4, bx=32, by=8, E=2, kernel="tile") as plan:
        state, _ = plan.fill_reference(seed=5)
        plan.upload(state)
        plan.run()
        plain = plan.download()[0]
        plan.enable_clocks(True)
        plan.upload(state)
        plan.run()
        with_clocks = plan.download()[0]
        rec = plan.clock_records()
        g = plan.geometry
    assert np.array_equal(plain.view(np.uint32), with_clocks.view(np.uint32))
    warps = g.threads[0] * g.threads[1] * g.threads[2] // 32
    assert len(rec) == g.num_blocks[0] * g.num_blocks[1] * g.num_blocks[2] * warps
    assert set(rec["warp"]) == set(range(warps))
    assert rec["sm"].max() < g.sm_count
    d = np.diff(rec["clock"].astype(np.int64), axis=1) % (1 << 32)  # 32-bit %clock wraps
    assert (d < (1 << 31)).all()                                       # monotone per warp
    assert (d[:, 1] > 0).all()                                         # the load + step take time


@pytest.mark.gpu
def test_cli_dump_clocks_and_phase_limits():
    r, kv = cli("jacobi-2d", "-n", 512, "-t", 8, "-s", 4, "-x", 32, "-y", 8, "-c", 1)
    assert r.returncode == 0
    assert "bx,by,warp,sm,clock0,clock1,clock2,clock3,clock4," in r.stderr
    rows = [l for l in r.stderr.splitlines() if l and l[0].isdigit()]
    assert rows and all(l.split(",")[3] == "1" for l in rows)   # SM 1, as the reference
    t = {}
    for pl in (0, 1, 2, 3):
        r, kv = cli("jacobi-2d", "-n", 2048, "-t", 16, "-s", 4, "-x", 32, "-y", 16, "-p", pl)
        assert r.returncode == 0 and kv["phase_limit"] == str(pl)
        t[pl] = float(kv["EventElapsed"])
    assert t[1] < t[0] and t[2] < t[0] and t[3] < t[0]


@pytest.mark.gpu
def test_yaml_experiment_through_cli_to_analytic_model(tmp_path):
    y = tmp_path / "j2d.yml"
    y.write_text("name: Jacobi 2D\noutfile: j2d.raw.dat\nbinary: ../../build.out/ocl-jacobi-2d\n"
                 "dimensions: 2\nphase_limit: 0\ncounters: l1_global_load_hit\nparameters:\n"
                 "    block_size_x: [32, 64, 32]\n    block_size_y: [4, 8, 4]\n"
                 "    time_tile_size: [1, 3, 2]\n    problem_size: 1024\n    time_steps: 16\n"
                 "    elements_per_thread: [1, 2]\n")
    logs = []
    ok, failed = H.run_experiment(str(y), log=logs.append)
    # by = 4, E = 1 at T = 3 leaves no interior: those two runs fail as the
    # reference runner does ("Consistency error!") and are left out of the file
    assert ok == 14 and failed == 2, "\n".join(logs)
    assert sum("Consistency error" in l for l in logs) == 2
    raw = open(tmp_path / "j2d.raw.dat").read().splitlines()
    assert raw[0].startswith("1#")
    dat = tmp_path / "j2d.dat"
    dat.write_text(H.results_to_csv(raw))
    rows = A.read_dat(str(dat))
    assert len(rows) == 14
    for row in rows:
        row["stencil"] = "jacobi-2d"
    rep = A.evaluate(rows, A.get_arch("b200"))
    assert rep["jacobi-2d"]["ranked"] == 14
    assert 0.0 < rep["jacobi-2d"]["top1_over_best"] <= 1.0


@pytest.mark.gpu
@pytest.mark.parametrize("stencil,args", [
    ("rician-denoise-2d", ["-n", 256, "-t", 4, "-s", 2, "-x", 32, "-y", 8, "-e", 4]),
    ("cdsc-tv-update-2d", ["-n", 256, "-t", 4, "-s", 2, "-x", 32, "-y", 8, "-e", 2]),
    ("poisson-3d", ["-n", 40, "-t", 4, "-s", 2, "-x", 16, "-y", 8, "-z", 1, "-e", 2,
                    "--kernel", "stream"]),
])
def test_cli_init_baseline_runs_the_benchmark_inputs(stencil, args):
    """--init baseline starts from the benchmark workloads' inputs (the disk
    image with Rician noise for Rician / TV, f in [-1, 1) for Poisson); the
    runner's -v check passes on them, and they are not the reference fill."""
    common = args + ["--engine", "native", "--variant", "baseline", "-v"]
    r_ref, kv_ref = cli(stencil, *common)
    r_base, kv_base = cli(stencil, *(common + ["--init", "baseline"]))
    assert r_ref.returncode == 0 and r_base.returncode == 0, r_base.stderr
    assert kv_base["Correctness"] == "PASSED" and kv_ref["Correctness"] == "PASSED"
    assert kv_base["Ref Norm"] != kv_ref["Ref Norm"]
