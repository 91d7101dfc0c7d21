"""Experiment harness that runs the reference's YAML experiment files against
the drop-in CLI, and the raw-to-CSV converter.

    python -m ots.harness scripts/c2050/j2d.yml [more.yml ...]   # raw N#Key: value file
    python -m ots.harness --to-csv j2d.raw.dat > j2d.dat          # .dat CSV

An experiment file is the reference's format (scripts/c2050/j2d.yml;
loader scripts/utils.py:36-88): ``name``, ``outfile``, ``binary``,
``dimensions``, ``phase_limit``, ``counters`` and ``parameters`` whose values
are a scalar or a ``[lo, hi, step]`` / ``[lo, hi]`` / ``[v]`` range
(utils.py:16-27), with the same defaults (problem_size 128, time_steps 64,
time_tile_size 1, elements_per_thread 1, block 16 x 16 x 8).  Every
permutation runs in the reference's loop order (problem size, steps, E, T,
x, y, z; utils.py:96-113) with its flags (``-n -t -e -s -x -p -w [-y] [-z]``,
utils.py:115-136) under a 15 s watchdog (utils.py:134-145); the stdout lines
of each successful run are written as ``<run>#<line>`` (utils.py:154-156), and
failures are reported as ``- FAILURE:`` with the run's output.

``binary`` may name the reference runner (``../../build.out/ocl-jacobi-2d``):
a path that does not exist and whose name is ``ocl-<stencil>`` or
``ots-<stencil>`` resolves to this package's ``bin/ots-<stencil>``.

Not reproduced: hardware counters through the legacy CUDA profiler
(``counters:``; COMPUTE_PROFILE, utils.py:176-230) -- take ncu metrics
instead -- and the FP/SFU instruction counts the reference grepped out of
disassembled kernels (utils.py:159-174).

The converter follows scripts/results-to-csv.py: one row per run, columns in
the order of the first run's keys, every field followed by a comma, runs that
miss a column skipped with a warning on stderr.
"""
import argparse
import os
import subprocess
import sys
import tempfile
import time

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def parse_range(value):
    """scripts/utils.py:16-27: int -> [v]; [lo, hi, step] / [lo, hi] -> the
    inclusive range; [v] -> [v]."""
    if isinstance(value, int):
        return [value]
    value = list(value)
    if len(value) == 3:
        return list(range(value[0], value[1] + 1, value[2]))
    if len(value) == 2:
        return list(range(value[0], value[1] + 1))
    if len(value) == 1:
        return [value[0]]
    raise ValueError("unable to handle range %r" % (value,))


def load_experiment(path):
    import yaml
    with open(path) as fh:
        data = yaml.safe_load(fh)
    params = data.get("parameters", {}) or {}
    dims = int(data["dimensions"])

    def q(name, default):
        return parse_range(params[name]) if name in params else default

    exp = {
        "name": data.get("name", os.path.basename(path)),
        "outfile": data["outfile"],
        "binary": data["binary"],
        "dimensions": dims,
        "phase_limit": int(data.get("phase_limit", 0) or 0),
        "counters": [c.strip() for c in str(data.get("counters", "")).split(",") if c.strip()],
        "elements_per_thread": q("elements_per_thread", [1]),
        "problem_size": q("problem_size", [128]),
        "time_steps": q("time_steps", [64]),
        "time_tile_size": q("time_tile_size", [1]),
        "block_size_x": q("block_size_x", [16]),
        "block_size_y": q("block_size_y", [16]) if dims > 1 else [1],
        "block_size_z": (q("block_size_z", [8]) if dims > 2 else [1]) if dims > 1 else [1],
        "dir": os.path.dirname(os.path.abspath(path)),
    }
    return exp


def configurations(exp, kernel_file):
    """Argument lists in the reference's loop order (utils.py:96-136)."""
    out = []
    for ps in exp["problem_size"]:
        for ts in exp["time_steps"]:
            for e in exp["elements_per_thread"]:
                for tt in exp["time_tile_size"]:
                    for bx in exp["block_size_x"]:
                        for by in exp["block_size_y"]:
                            for bz in exp["block_size_z"]:
                                args = ["-n", str(ps), "-t", str(ts), "-e", str(e), "-s", str(tt),
                                        "-x", str(bx), "-p", str(exp["phase_limit"]),
                                        "-w", kernel_file]
                                if exp["dimensions"] > 1:
                                    args += ["-y", str(by)]
                                    if exp["dimensions"] > 2:
                                        args += ["-z", str(bz)]
                                out.append(args)
    return out


def resolve_binary(binary, base_dir):
    """The experiment's runner, or this package's drop-in CLI for it."""
    for cand in (binary, os.path.join(base_dir, binary)):
        if os.path.isfile(cand) and os.access(cand, os.X_OK):
            return cand
    name = os.path.basename(binary)
    for prefix in ("ocl-", "ots-"):
        if name.startswith(prefix):
            mine = os.path.join(PKG, "bin", "ots-" + name[len(prefix):])
            if os.path.exists(mine):
                return mine
    raise FileNotFoundError("runner %r not found (and no bin/ots-<stencil> for it)" % binary)


def run_experiment(path, binary=None, outfile=None, watchdog=15.0, extra_args=(), log=print):
    """Run one experiment file; returns (ok runs, failed runs)."""
    exp = load_experiment(path)
    exe = resolve_binary(binary or exp["binary"], exp["dir"])
    out_path = outfile or exp["outfile"]
    if not os.path.isabs(out_path) and outfile is None:
        out_path = os.path.join(exp["dir"], out_path)
    if exp["counters"]:
        log("note: counters %s are not collected (legacy profiler); use ncu" % exp["counters"])
    tmpdir = tempfile.mkdtemp(prefix="ots-harness-")
    kernel_file = os.path.join(tmpdir, "temp-kernel.txt")
    cfgs = configurations(exp, kernel_file)
    log("Number of Runs: %d" % len(cfgs))
    ok = failed = 0
    t_all = time.time()
    with open(out_path, "w") as out:
        for curr, args in enumerate(cfgs, start=1):
            log("Running %d of %d" % (curr, len(cfgs)))
            t0 = time.time()
            try:
                proc = subprocess.run([exe] + args + list(extra_args), capture_output=True,
                                      text=True, timeout=watchdog)
                rc, so, se = proc.returncode, proc.stdout, proc.stderr
            except subprocess.TimeoutExpired as e:
                log("Watchdog timer expired!")
                rc, so, se = -1, e.stdout or "", e.stderr or ""
                so = so.decode() if isinstance(so, bytes) else so
                se = se.decode() if isinstance(se, bytes) else se
            if rc != 0:
                failed += 1
                log("- FAILURE:")
                log(so)
                log(se)
            else:
                ok += 1
                for line in so.splitlines():
                    out.write("%d#%s\n" % (curr, line))
                out.flush()
            el = time.time() - t0
            total = time.time() - t_all
            rem = int(total / curr * (len(cfgs) - curr))
            log("Elapsed: %f  Total: %f  Remaining: %d:%d:%d" % (el, total, rem // 3600,
                                                                 (rem // 60) % 60, rem % 60))
    return ok, failed


def results_to_csv(lines, warn=None):
    """Raw 'N#Key: value' lines -> CSV text (scripts/results-to-csv.py)."""
    warn = warn or (lambda m: sys.stderr.write(m + "\n"))
    runs = {}
    order = []
    for line in lines:
        line = line.strip()
        if not line or "#" not in line:
            continue
        run, data = line.split("#", 1)
        if ":" not in data:
            continue
        key, value = data.split(":", 1)
        run = int(run)
        if run not in runs:
            runs[run] = {}
            order.append(run)
        runs[run][key.strip()] = value.strip()
    if not order:
        return ""
    columns = list(runs[order[0]].keys())
    out = ["".join("%s," % c for c in columns)]
    for run in order:
        vals = runs[run]
        missing = [c for c in columns if c not in vals]
        if missing:
            for c in missing:
                warn("Warning: missing %s for run %d" % (c, run))
            warn("Skipping run %d" % run)
            continue
        out.append("".join("%s," % vals[c] for c in columns))
    return "\n".join(out) + "\n"


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawTextHelpFormatter)
    ap.add_argument("files", nargs="+", help="experiment .yml files, or a raw file with --to-csv")
    ap.add_argument("--to-csv", action="store_true", help="convert raw N#Key: value files to CSV")
    ap.add_argument("--binary", help="override the experiment's runner")
    ap.add_argument("--outfile", help="override the experiment's outfile")
    ap.add_argument("--watchdog", type=float, default=15.0)
    a = ap.parse_args(argv)
    if a.to_csv:
        lines = []
        for f in a.files:
            with open(f) as fh:
                lines += fh.readlines()
        sys.stdout.write(results_to_csv(lines))
        return 0
    for f in a.files:
        print("=== Running %s" % f)
        run_experiment(f, binary=a.binary, outfile=a.outfile, watchdog=a.watchdog)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
