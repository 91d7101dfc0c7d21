#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/ from the reference's OWN code.

Run where the reference checkout exists (it builds oracle/_ref first via
oracle/build_ref.py).  Everything computed here comes out of the reference's
compiled source: its CPU verification loops, its enabled input-fill loops and
its GeneratorParams::computeDerived for all thirteen runners.  The fixtures
are small and committed; tests/test_oracle_pin.py checks the oracle against
them bit for bit on any machine, including ones without the reference.

Outputs:
  ref_loops.npz     inputs and outputs of the reference CPU loops
  ref_fills.npz     outputs of the reference fill loops
  ref_geometry.json computeDerived results for a seeded sample of parameters
  ref_kernels.npz   inputs and outputs of the kernels the reference's own
                    generators emit (XGenerator::generate), run on the CPU by
                    oracle/ref_clkernel.cpp, for the seven stencils whose
                    runners have no usable CPU check

    python tests/golden/make_golden.py [loops] [fills] [geometry] [kernels]

writes the named fixtures (all four without arguments).
"""
import json
import os
import random
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import build_ref  # noqa: E402
import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

# (stencil, n, T, bx, by, E, steps, seed)
LOOP_CASES = [
    ("jacobi-1d", 150, 3, 16, 1, 2, 9, 123456),
    ("jacobi-1d-5pt", 170, 2, 32, 1, 1, 11, 99),
    ("jacobi-1d-7pt", 190, 2, 16, 1, 3, 8, 7),
    ("jacobi-2d", 40, 2, 16, 8, 1, 12, 123456),
    ("jacobi-2d", 37, 1, 16, 16, 1, 5, 31337),
    ("poisson-2d", 36, 2, 8, 8, 1, 10, 123456),
    ("gradient-2d", 44, 3, 16, 4, 3, 9, 123456),
]


def loops():
    out = {}
    for k, (st, n, T, bx, by, E, steps, seed) in enumerate(LOOP_CASES):
        g = O.ref_geometry(st, n, T, bx, by, 1, E)
        P, pad, real = g["padded_size"], g["padding"], g["real_size"]
        d = O.dims(st)
        # reference fill scheme over the runner's interior [pad, pad+real)
        x = O.fill_ref(d, P, pad, pad + real, seed, 1)[0]
        y = O.ref_loop(st, x, pad, steps)
        key = "c%d" % k
        out[key + "_in"] = x
        out[key + "_out"] = y
        out[key + "_meta"] = np.array([O.SID[st], P, pad, steps, seed, real], np.int64)
    np.savez_compressed(os.path.join(HERE, "ref_loops.npz"), **out)


def fills():
    out = {}
    for which, P, pad, seed in [("poisson_2d", 33, 3, 123456), ("fdtd_2d", 21, 2, 42),
                                ("cs_3d", 13, 2, 123456), ("jacobi_1d_5pt", 40, 4, 5)]:
        arrs = O.ref_fill(which, P, pad, seed)
        for i, a in enumerate(arrs):
            out["%s_%d" % (which, i)] = a
        out[which + "_meta"] = np.array([P, pad, seed, len(arrs)], np.int64)
    np.savez_compressed(os.path.join(HERE, "ref_fills.npz"), **out)


def geometry():
    rnd = random.Random(20121212)
    rows = []
    for st in O.STENCILS:
        d = O.dims(st)
        for _ in range(60):
            n = rnd.choice([100, 200, 512, 1000, 2048, 6000])
            T = rnd.randint(1, 8)
            bx = rnd.choice([8, 16, 32, 64, 128])
            by = rnd.choice([2, 4, 8, 16]) if d >= 2 else 1
            bz = rnd.choice([2, 4, 8]) if d == 3 else 1
            E = rnd.randint(1, 6)
            # The reference divides by realPerBlock* before checking it, so
            # a zero there raises SIGFPE inside the reference itself: such
            # combinations are sampled by the oracle tests, not here.
            r_ = O.radius(st) if d == 1 else 1
            rpb = [bx * (E if d == 1 else 1) - 2 * r_ * (T - 1)]
            if d >= 2:
                rpb.append(by * E - 2 * (T - 1))
            if d == 3:
                rpb.append(bz - 2 * (T - 1))
            if 0 in rpb:
                continue
            r = O.ref_geometry(st, n, T, bx, by, bz, E)
            rows.append([st, n, T, bx, by, bz, E, r])
    with open(os.path.join(HERE, "ref_geometry.json"), "w") as fh:
        json.dump(rows, fh, separators=(",", ":"))


# Generated-kernel cases: (stencil, n, T, bx, by, bz, E, steps, seed, oracle variant).
# Constraints that keep each case clear of the reference kernels' known
# defects (each stated with the kernel lines it concerns):
#   * 3D: bx == bz, so the local array declared [sZ][sY][sZ] has the shape
#     the kernel indexes ([sZ][sY][sX], opencl/jacobi-3d/jacobi-3d.cpp:189-190);
#   * 3D at T = 2: one tile along z (n == bz - 2), so the write-back that
#     ignores writeValidZ (:400-405) writes only the zero ring's planes;
#   * fdtd-2d and rician at T = 1: one tile covering the interior -- their
#     second phase reads E' / g of the cells right of and below the tile,
#     which no work-item of the tile computes; with one tile those cells are
#     the zero ring and read as zero;
#   * cs-3d: oracle variant 9, the first step's y-axis orientation
#     (cs-3d.cpp:259-283).
KERNEL_CASES = [
    ("jacobi-3d", 16, 1, 4, 4, 4, 1, 5, 123456, 1),
    ("jacobi-3d", 16, 1, 4, 2, 4, 2, 4, 77, 1),
    ("jacobi-3d", 6, 2, 8, 4, 8, 1, 6, 123456, 1),
    ("jacobi-3d", 6, 2, 8, 2, 8, 2, 7, 5, 1),
    ("poisson-3d", 12, 1, 4, 4, 4, 1, 3, 123456, 1),
    ("poisson-3d", 6, 2, 8, 4, 8, 1, 4, 9, 1),
    ("gradient-3d", 12, 1, 4, 4, 4, 1, 4, 123456, 0),
    ("gradient-3d", 6, 2, 8, 4, 8, 1, 4, 11, 0),
    ("cs-3d", 12, 1, 4, 4, 4, 1, 4, 123456, 9),
    ("fdtd-2d", 16, 1, 16, 16, 1, 1, 6, 123456, 1),
    ("rician-denoise-2d", 16, 1, 16, 16, 1, 1, 4, 123456, 0),
    ("cdsc-tv-update-2d", 24, 1, 8, 8, 1, 1, 4, 123456, 0),
]


def kernels():
    """Each case: the reference fill scheme over the runner's interior (every
    state and aux field, interleaved per cell), the generated kernel run by
    the runner's launch loop; jacobi-3d's kernel carries its 0.143f weight."""
    out = {}
    for k, (st, n, T, bx, by, bz, E, steps, seed, variant) in enumerate(KERNEL_CASES):
        g = O.ref_geometry(st, n, T, bx, by, bz, E)
        P, pad, real = g["padded_size"], g["padding"], g["real_size"]
        d = O.dims(st)
        nf, na = O.num_state(st), O.num_aux(st)
        arrs = O.fill_ref(d, P, pad, pad + real, seed, nf + na)
        fields, aux = arrs[:nf], arrs[nf:]
        # the runner's argument order: TV takes (input, V, F, ...); the
        # oracle's aux order is (F, V)
        ref_aux = aux[::-1] if st == "cdsc-tv-update-2d" else aux
        nb = [g["num_blocks_x"], g["num_blocks_y"] if d >= 2 else 1,
              g["num_blocks_z"] if d == 3 else 1]
        bs = [bx, by if d >= 2 else 1, bz if d == 3 else 1]
        lib = build_ref.build_kernel_case(st, n, T, bx, by, bz, E, steps)
        res = O.ref_kernel_run(lib, fields, ref_aux, T=T, steps=steps, nb=nb, bs=bs)
        key = "k%02d" % k
        for i, a in enumerate(fields):
            out["%s_in%d" % (key, i)] = a
        for i, a in enumerate(aux):
            out["%s_aux%d" % (key, i)] = a
        for i, a in enumerate(res):
            out["%s_out%d" % (key, i)] = a
        out[key + "_meta"] = np.array([O.SID[st], P, pad, steps, seed, real, T, variant,
                                       nf, na, bx, by, bz, E], np.int64)
    np.savez_compressed(os.path.join(HERE, "ref_kernels.npz"), **out)


if __name__ == "__main__":
    if not build_ref.build(verbose=True):
        sys.exit("reference tree not found: set OTS_REFERENCE_DIR to the reference checkout "
                 "(the golden fixtures are generated where it exists)")
    which = sys.argv[1:] or ["loops", "fills", "geometry", "kernels"]
    for name in which:
        {"loops": loops, "fills": fills, "geometry": geometry, "kernels": kernels}[name]()
    print("golden fixtures written to", HERE, ":", " ".join(which))
