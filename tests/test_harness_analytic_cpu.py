"""The reference-compatible experiment harness and the analytical-model
comparator, on the CPU: range syntax and loop order of scripts/utils.py, the
raw -> CSV conversion of scripts/results-to-csv.py, the model's arithmetic on
a hand-worked case, and its ranking of the committed B200 sweep."""
import json
import os

import pytest

import ots
from ots import analytic as A
from ots import harness as H

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DATA = os.path.join(ROOT, "ics-12-overlapped-tiling_b200", "ots", "data")


def test_parse_range_matches_reference_syntax():
    assert H.parse_range(6000) == [6000]
    assert H.parse_range([32, 128, 32]) == [32, 64, 96, 128]
    assert H.parse_range([1, 4]) == [1, 2, 3, 4]
    assert H.parse_range([7]) == [7]
    with pytest.raises(ValueError):
        H.parse_range([1, 2, 3, 4])


def test_experiment_loop_order_and_flags(tmp_path):
    y = tmp_path / "exp.yml"
    y.write_text("name: t\noutfile: t.raw.dat\nbinary: ../../build.out/ocl-jacobi-3d\n"
                 "dimensions: 3\nphase_limit: 2\ncounters: l1_global_load_hit\n"
                 "parameters:\n  block_size_x: [32, 64, 32]\n  time_tile_size: [1, 2]\n"
                 "  problem_size: 96\n")
    exp = H.load_experiment(str(y))
    assert exp["block_size_y"] == [16] and exp["block_size_z"] == [8]  # reference defaults
    assert exp["time_steps"] == [64] and exp["elements_per_thread"] == [1]
    cfgs = H.configurations(exp, "/tmp/k")
    assert len(cfgs) == 4
    # T varies slower than x (utils.py loop nest: ps, ts, e, tt, x, y, z)
    assert [c[c.index("-s") + 1] for c in cfgs] == ["1", "1", "2", "2"]
    assert [c[c.index("-x") + 1] for c in cfgs] == ["32", "64", "32", "64"]
    assert cfgs[0][:12] == ["-n", "96", "-t", "64", "-e", "1", "-s", "1", "-x", "32", "-p", "2"]
    assert cfgs[0][-4:] == ["-y", "16", "-z", "8"]


def test_reference_runner_name_resolves_to_drop_in():
    exe = H.resolve_binary("../../build.out/ocl-jacobi-2d", ROOT)
    assert exe.endswith(os.path.join("bin", "ots-jacobi-2d"))
    with pytest.raises(FileNotFoundError):
        H.resolve_binary("no-such-runner", ROOT)


def test_results_to_csv_layout_and_skips():
    raw = ["1#Block Size X: 32\n", "1#EventElapsed: 0.5\n", "2#Block Size X: 64\n",
           "2#EventElapsed: 0.25\n", "3#Block Size X: 16\n", "noise line\n"]
    warns = []
    txt = H.results_to_csv(raw, warn=warns.append)
    assert txt.splitlines() == ["Block Size X,EventElapsed,", "32,0.5,", "64,0.25,"]
    assert any("Skipping run 3" in w for w in warns)


def test_model_constants_through_the_abi():
    c = ots.model_constants("jacobi-2d")
    assert [c[k] for k in ots.MODEL_CONSTANT_KEYS] == [5, 0, 5, 5, 1, 1, 1, 4]
    assert ots.model_constants("fdtd-2d")["num_fields"] == 3
    assert ots.model_constants("cs-3d") is None
    assert ots.model_constants("jacobi-1d-5pt") is None


C2050_J2D_ROW = {  # first row of the reference's scripts/c2050/j2d.dat
    "Block Size X": 32, "Block Size Y": 4, "Block Size Z": 1, "Elements/Thread": 1,
    "Time Tile Size": 1, "Dimensions": 2, "Register Usage": 11, "Num Blocks X": 187,
    "Num Blocks Y": 1500, "Num Blocks Z": 1, "Time Steps": 64, "phase_limit": 0,
    "phase2_global_loads": 5, "phase2_shared_loads": 0, "compute_per_point": 5,
    "phase3_shared_loads": 5, "phase4_global_stores": 1, "shared_stores": 1, "num_fields": 1,
    "data_size": 4, "EventElapsed": 0.39824}


def test_model_arithmetic_on_a_hand_worked_case():
    # C2050 constants.  Occupancy: 4 warps/block; blocks by warps 12, by shared
    # floor(49152/816)=60, by registers floor(32768/1408)=23 -> 12 -> cap 8:
    # 32 active warps; 280500 blocks -> 2505 waves.  Phase 2: 5 loads, L1 miss
    # rate (e+4)/(5e) = 1 -> 5 global loads; t_glb = max(2*5*32 + 4*32 + 16*32,
    # 750 + 2 + 20*5*32) = 3952.  t_shd = max(2*5*32 + 4*32 + 4*32, 34 + 320)
    # = 576 (unused at T=1).  write-back 750 + 2 + 18*32 = 1328; phase 1
    # (10+20)*32 = 960.  Stage 6240 cycles x 2505 waves x 64 launches.
    sim, d = A.simulate(C2050_J2D_ROW, A.get_arch("c2050"))
    assert d["active_warps"] == 32 and d["num_stages"] == 2505
    assert d["t_glb"] == 3952 and d["t_shd"] == 576 and d["write_back"] == 1328
    assert sim == pytest.approx(6240.0 * 2505 * 64 / 1.15e9, rel=1e-12)


def test_model_phase_limits_and_register_cap():
    arch = A.get_arch("c2050")
    r1 = dict(C2050_J2D_ROW, phase_limit=1)
    s1, d = A.simulate(r1, arch)
    assert s1 == pytest.approx(d["t_phase1"] * 2505 * 64 / 1.15e9)
    r3 = dict(C2050_J2D_ROW, **{"Time Tile Size": 4, "phase_limit": 3})
    s3, d3 = A.simulate(r3, arch)
    assert s3 == pytest.approx(((3 * d3["t_shd"] + d3["t_phase1"]) * 2505 * 16) / 1.15e9)
    capped = dict(C2050_J2D_ROW, **{"Register Usage": 63})
    assert len(A.rank([C2050_J2D_ROW, capped], arch)) == 1


def test_b200_constants_from_measured_bandwidth():
    a = A.b200_arch(hbm_gbs=6539.2)
    assert a["B_gmem"] == pytest.approx(128.0 / (6539.2e9 / (148 * 1.965e9)))
    assert a["num_sm"] == 148 and a["max_warps_per_sm"] == 64


def test_analytic_ranking_of_the_b200_sweep_and_the_learned_gain():
    recs = json.load(open(os.path.join(DATA, "sweeps_b200.json")))["records"]
    consts = {s: ots.model_constants(s) for s in ots.STENCILS}
    runs = A.runs_from_records(recs, consts)
    rep = A.evaluate(runs, A.get_arch("b200"))
    assert set(k for k in rep if k != "_mean") >= {"jacobi-2d", "rician-denoise-2d",
                                                    "cdsc-tv-update-2d", "fdtd-2d"}
    assert rep["_mean"]["spearman"] > 0.8          # the model ranks, not guesses
    # the C2050 constants rank the B200 measurements worse than the B200 ones
    rep_old = A.evaluate(runs, A.get_arch("c2050"))
    assert rep["_mean"]["top1_over_best"] > rep_old["_mean"]["top1_over_best"]
    # both methods meet the picker target (within 5 % of the exhaustive best
    # at a 10 % measuring budget) on the held-out stencils; the learned one
    # is reported beside the analytical one, not asserted to win
    mlp = json.load(open(os.path.join(DATA, "picker_report_b200.json")))
    for s in ("rician-denoise-2d", "cdsc-tv-update-2d"):
        assert mlp[s]["picked_over_best"] >= 0.95
        assert rep[s]["topk_over_best"] >= 0.95
    assert mlp["_mean"]["picked_over_best"] >= 0.95


def test_read_dat_reference_layout(tmp_path):
    p = tmp_path / "x.dat"
    p.write_text("Block Size X,EventElapsed,\n32,0.5,\n64,0.25,\n")
    rows = A.read_dat(str(p))
    assert rows == [{"Block Size X": "32", "EventElapsed": "0.5"},
                    {"Block Size X": "64", "EventElapsed": "0.25"}]


def test_watchdog_skips_a_hung_run_and_the_sweep_continues(tmp_path):
    """scripts/utils.py:134-145: a run that outlives the watchdog is killed,
    reported as a failure and left out of the raw file; the next runs go on.
    The runner is a fake script that hangs (sleeps) for block size 64 only."""
    runner = tmp_path / "fake-runner"
    runner.write_text(
        "#!/bin/sh\n"
        "bx=0\n"
        "while [ $# -gt 0 ]; do [ \"$1\" = -x ] && bx=$2; shift; done\n"
        "if [ \"$bx\" = 64 ]; then exec sleep 30; fi\n"
        "echo \"Block Size X: $bx\"\n"
        "echo \"EventElapsed: 0.5\"\n")
    runner.chmod(0o755)
    y = tmp_path / "exp.yml"
    y.write_text("name: wd\noutfile: wd.raw.dat\nbinary: fake-runner\ndimensions: 2\n"
                 "parameters:\n  block_size_x: [32, 96, 32]\n  problem_size: 64\n")
    logs = []
    t0 = __import__("time").time()
    ok, failed = H.run_experiment(str(y), watchdog=1.0, log=logs.append)
    assert __import__("time").time() - t0 < 20
    assert (ok, failed) == (2, 1)
    assert "Watchdog timer expired!" in logs
    assert logs.index("Watchdog timer expired!") > logs.index("Running 2 of 3")
    assert "Running 3 of 3" in logs  # the sweep went on past the hung run
    raw = (tmp_path / "wd.raw.dat").read_text().splitlines()
    assert raw == ["1#Block Size X: 32", "1#EventElapsed: 0.5",
                   "3#Block Size X: 96", "3#EventElapsed: 0.5"]
