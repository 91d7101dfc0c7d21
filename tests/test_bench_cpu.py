"""bench.py's host-side helpers on the CPU: the clock sampler's summary keeps
only the samples taken inside the timed region (nvidia-smi rows carry their
timestamps), and the bound(T) roofline of the workload table."""
import datetime
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _row(t, sm, reasons=("Not Active",) * 4):
    stamp = datetime.datetime.fromtimestamp(t).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
    return ", ".join([stamp, str(sm), "1965", "700.00"] + list(reasons)) + "\n"


def test_clock_summary_keeps_the_timed_region(tmp_path):
    c = bench.Clocks(0)
    c.path = str(tmp_path / "clocks.csv")
    t0 = 1_800_000_000.0
    with open(c.path, "w") as fh:
        fh.write(_row(t0 - 1.0, 900))   # idle, before the region
        for i in range(5):
            fh.write(_row(t0 + 0.1 + 0.1 * i, 1965 if i != 2 else 1950,
                          ("Not Active",) * 3 + ("Active",) if i == 4 else ("Not Active",) * 4))
        fh.write(_row(t0 + 2.0, 700))   # after it
    c.t0, c.t1 = t0, t0 + 0.6
    s = c.summary()
    assert s["samples"] == 5 and s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]


def test_clock_summary_falls_back_to_the_neighbouring_samples(tmp_path):
    # a region shorter than the sampling period: the samples just before and
    # after it stand in
    c = bench.Clocks(0)
    c.path = str(tmp_path / "clocks.csv")
    t0 = 1_800_000_000.0
    with open(c.path, "w") as fh:
        fh.write(_row(t0 - 5.0, 500))
        fh.write(_row(t0 - 0.02, 1960))
        fh.write(_row(t0 + 0.05, 1965))
        fh.write(_row(t0 + 3.0, 600))
    c.t0, c.t1 = t0, t0 + 0.01
    s = c.summary()
    assert s["samples"] == 2 and s["sm_mhz"] == 1965.0


def test_clock_summary_without_samples(tmp_path):
    c = bench.Clocks(0)
    c.path = str(tmp_path / "missing.csv")
    assert c.summary()["reasons"] == ["nvidia-smi unavailable"]


def test_bound_at_T():
    # jacobi-3d at T = 4: HBM-bound, 6551.7 GB/s x 4 / 8 B
    b = bench.bound_at_T("jacobi-3d", 4, 8, 6551.7)
    assert b["bound"] == "hbm" and b["gupdates"] == pytest.approx(3275.85)
    # jacobi-1d at T = 32: the FP32 term (3 operations per update) binds
    b = bench.bound_at_T("jacobi-1d", 32, 8, 6551.7)
    assert b["bound"] == "fp32" and b["gupdates"] == pytest.approx(148 * 128 * 1.965 / 3, rel=1e-3)
