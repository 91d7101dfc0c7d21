#!/usr/bin/env python3
"""Build recipe for oracle/_ref: the reference's own CPU verification loops.

TEST INFRASTRUCTURE ONLY.  Run where a reference checkout is present; its
location comes from the caller (build(ref_root)) or $OTS_REFERENCE_DIR, and
without either nothing is built.  For each pinned
stencil it copies the CPU loop of the reference runner -- the lines between
``memcpy(refB, hostData, arraySize);`` and ``memcpy(reference, refA,
arraySize);`` of its main() -- verbatim into ``oracle/_ref/<name>_loop.inc``
(git-ignored; nothing from the reference is committed), then compiles
``oracle/ref_harness.cpp`` around those loops with the reference's own flags
(``g++ -O2``, config.ninja:4) into ``oracle/_ref/libots_ref.so``.

The built library is the "reference" CPU baseline and the generator of the
golden vectors in tests/golden/.  When the reference tree is absent (e.g. on
a machine that only received the prebuilt library) this script does nothing.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")

# name -> reference runner source, relative to the reference root
LOOPS = {
    "jacobi_1d": "opencl/jacobi-1d/jacobi-1d.cpp",
    "jacobi_1d_5pt": "opencl/jacobi-1d-5pt/jacobi-1d-5pt.cpp",
    "jacobi_1d_7pt": "opencl/jacobi-1d-7pt/jacobi-1d-7pt.cpp",
    "jacobi_2d": "opencl/jacobi-2d/jacobi-2d.cpp",
    "poisson_2d": "opencl/poisson-2d/poisson-2d.cpp",
    "gradient_2d": "opencl/gradient-2d/gradient-2d.cpp",
}
# jacobi-3d's loop (opencl/jacobi-3d/jacobi-3d.cpp:726-747) is deliberately
# not built: its unparenthesised ARRAY_REF macro reads out of bounds.

# name -> runner whose input fill loop is enabled (not under #if 0)
FILLS = {
    "fill_poisson_2d": ("opencl/poisson-2d/poisson-2d.cpp", 2, ["hostData"]),
    "fill_fdtd_2d": ("opencl/fdtd-2d/fdtd-2d.cpp", 2, ["hostDataEX", "hostDataEY", "hostDataHZ"]),
    "fill_cs_3d": ("opencl/cs-3d/cs-3d.cpp", 3, ["hostData"]),
    "fill_jacobi_1d_5pt": ("opencl/jacobi-1d-5pt/jacobi-1d-5pt.cpp", 1, ["hostData"]),
}

# name -> (runner source, dims, has blockSizeY/Z members)
GEOMETRY = {
    "jacobi_1d": ("opencl/jacobi-1d/jacobi-1d.cpp", 1),
    "jacobi_1d_5pt": ("opencl/jacobi-1d-5pt/jacobi-1d-5pt.cpp", 1),
    "jacobi_1d_7pt": ("opencl/jacobi-1d-7pt/jacobi-1d-7pt.cpp", 1),
    "jacobi_2d": ("opencl/jacobi-2d/jacobi-2d.cpp", 2),
    "jacobi_3d": ("opencl/jacobi-3d/jacobi-3d.cpp", 3),
    "poisson_2d": ("opencl/poisson-2d/poisson-2d.cpp", 2),
    "poisson_3d": ("opencl/poisson-3d/poisson-3d.cpp", 3),
    "gradient_2d": ("opencl/gradient-2d/gradient-2d.cpp", 2),
    "gradient_3d": ("opencl/gradient-3d/gradient-3d.cpp", 3),
    "fdtd_2d": ("opencl/fdtd-2d/fdtd-2d.cpp", 2),
    "rician_denoise_2d": ("opencl/rician-denoise-2d/rician-denoise-2d.cpp", 2),
    "cdsc_tv_update_2d": ("opencl/cdsc-tv-update-2d/cdsc-tv-update-2d.cpp", 2),
    "cs_3d": ("opencl/cs-3d/cs-3d.cpp", 3),
}

START = "memcpy(refB, hostData, arraySize);"
END = "memcpy(reference, refA, arraySize);"


def extract(ref_root, rel):
    path = os.path.join(ref_root, rel)
    with open(path) as fh:
        lines = fh.readlines()
    s = next(i for i, l in enumerate(lines) if l.strip() == START)
    e = next(i for i, l in enumerate(lines) if i > s and l.strip() == END)
    body = lines[s + 1:e]
    if not any("for(int t = 0; t < params.timeSteps; ++t)" in l for l in body):
        raise RuntimeError("%s: CPU loop not found between the markers" % rel)
    # 1-based line number of the first copied line, for diagnostics
    return s + 2, "".join(body), path


def extract_between(path, start_pred, end_pred):
    with open(path) as fh:
        lines = fh.readlines()
    s = next(i for i, l in enumerate(lines) if start_pred(l))
    e = next(i for i, l in enumerate(lines) if i > s and end_pred(l))
    return s + 1, "".join(lines[s:e + 1])


def gen_geometry_and_fill(ref_root):
    """Generate oracle/_ref/ref_gen.cpp: each runner's GeneratorParams struct
    (copied verbatim into its own namespace) behind a C entry point, and the
    enabled input-fill loops behind C entry points.  boost::math::gcd/lcm are
    supplied by oracle/ref_shim.hpp."""
    out = ['#include "ref_shim.hpp"\n']
    for name, (rel, dims) in GEOMETRY.items():
        path = os.path.join(ref_root, rel)
        line, body = extract_between(path, lambda l: l.startswith("struct GeneratorParams"),
                                     lambda l: l.startswith("};"))
        out.append("namespace geo_%s {\n#line %d \"%s\"\n%s\n}\n" % (name, line, path, body))
        sets = ["p.problemSize = n;", "p.timeTileSize = T;", "p.blockSizeX = bx;",
                "p.elementsPerThread = E;"]
        gets = ["o[0] = p.padding;", "o[1] = p.paddedSize;", "o[2] = p.realSize;",
                "o[3] = p.sizeLCM;", "o[4] = p.compsPerBlockX;", "o[7] = p.realPerBlockX;",
                "o[10] = p.numBlocksX;", "o[13] = p.sharedSizeX;"]
        if dims >= 2:
            sets += ["p.blockSizeY = by;"]
            gets += ["o[5] = p.compsPerBlockY;", "o[8] = p.realPerBlockY;",
                     "o[11] = p.numBlocksY;", "o[14] = p.sharedSizeY;"]
        if dims >= 3:
            sets += ["p.blockSizeZ = bz;"]
            gets += ["o[6] = p.compsPerBlockZ;", "o[9] = p.realPerBlockZ;",
                     "o[12] = p.numBlocksZ;", "o[15] = p.sharedSizeZ;"]
        out.append(
            'extern "C" int ref_geometry_%s(int n, int T, int bx, int by, int bz, int E, int* o) {\n'
            "  (void)by; (void)bz;\n"
            "  for (int i = 0; i < 16; ++i) o[i] = 0;\n"
            "  try {\n    geo_%s::GeneratorParams p;\n    %s\n    p.computeDerived();\n    %s\n"
            "  } catch (...) { return -1; }\n  return 0;\n}\n"
            % (name, name, " ".join(sets), " ".join(gets)))
    for name, (rel, dims, arrays) in FILLS.items():
        path = os.path.join(ref_root, rel)
        line, body = extract_between(path, lambda l: l.strip() == "// Fill host arrays",
                                     lambda l: l.strip() == "// Compute reference")
        args = ", ".join("float* %s" % a for a in arrays)
        out.append(
            'extern "C" void ref_%s(%s, int paddedSize, int padding, unsigned seed) {\n'
            "  RefParams params; params.paddedSize = paddedSize; params.padding = padding;\n"
            "  params.timeSteps = 0;\n  srand(seed);\n#line %d \"%s\"\n%s\n}\n"
            % (name, args, line, path, body))
    with open(os.path.join(OUT, "ref_gen.cpp"), "w") as fh:
        fh.write("".join(out))


# Generated-kernel pins: name -> (runner source, generator class, stencil id
# in the oracle's numbering).  These seven runners have no usable CPU check
# (Jacobi copies, a commented-out one, or jacobi-3d's out-of-bounds loop), so
# the oracle is pinned to the kernels their own generators emit.
GENERATORS = {
    "jacobi_3d": ("opencl/jacobi-3d/jacobi-3d.cpp", "Jacobi3DGenerator", 4),
    "poisson_3d": ("opencl/poisson-3d/poisson-3d.cpp", "Poisson3DGenerator", 6),
    "gradient_3d": ("opencl/gradient-3d/gradient-3d.cpp", "Gradient3DGenerator", 8),
    "fdtd_2d": ("opencl/fdtd-2d/fdtd-2d.cpp", "FDTD2DGenerator", 9),
    "rician_denoise_2d": ("opencl/rician-denoise-2d/rician-denoise-2d.cpp",
                          "Rician2DGenerator", 10),
    "cdsc_tv_update_2d": ("opencl/cdsc-tv-update-2d/cdsc-tv-update-2d.cpp",
                          "TVUpdate2DGenerator", 11),
    "cs_3d": ("opencl/cs-3d/cs-3d.cpp", "CS3DGenerator", 12),
}
GEN_LIB = os.path.join(OUT, "libots_refgen.so")


def gen_generators(ref_root, cxx="g++"):
    """oracle/_ref/ref_generators.cpp -> libots_refgen.so: each runner's
    GeneratorParams and XGenerator (its source from ``struct GeneratorParams``
    up to ``compareResults``, copied verbatim into its own namespace) behind
    ``extern "C" int gen_<name>(n, T, bx, by, bz, E, steps, buf, cap)``,
    which fills ``buf`` with the kernel text generate() returns (-1 if
    computeDerived throws, -2 if the text does not fit)."""
    out = ['#include <cstring>\n#include <iostream>\n#include <sstream>\n#include <string>\n',
           '#include "ref_shim.hpp"\n',
           # printProgramParameters (never called here) names printValue
           "template <class V> void printValue(const std::string&, const V&) {}\n",
           '#include "ProgramGenerator.hpp"\n',
           "namespace ot {\nProgramGenerator::ProgramGenerator() {}\n"
           "ProgramGenerator::~ProgramGenerator() {}\n"
           "std::string ProgramGenerator::getProgram() { return std::string(); }\n}\n"]
    for name, (rel, cls, _) in GENERATORS.items():
        path = os.path.join(ref_root, rel)
        line, body = extract_between(path, lambda l: l.startswith("struct GeneratorParams"),
                                     lambda l: l.startswith("void compareResults("))
        body = body[:body.rindex("void compareResults(")]
        out.append("namespace refgen_%s {\nusing namespace ot;\n#line %d \"%s\"\n%s\n}\n"
                   % (name, line, path, body))
        out.append(
            'extern "C" int gen_%s(int n, int T, int bx, int by, int bz, int E, int steps,\n'
            "                      char* buf, int cap) {\n"
            "  std::string text;\n"
            "  try {\n"
            "    refgen_%s::GeneratorParams p;\n"
            "    p.problemSize = n; p.timeTileSize = T; p.timeSteps = steps;\n"
            "    p.blockSizeX = bx; p.blockSizeY = by; p.blockSizeZ = bz;\n"
            "    p.elementsPerThread = E;\n"
            "    refgen_%s::%s g;\n"
            "    text = g.generate(p);\n"
            "  } catch (...) { return -1; }\n"
            "  if ((int)text.size() + 1 > cap) return -2;\n"
            "  std::memcpy(buf, text.c_str(), text.size() + 1);\n"
            "  return (int)text.size();\n}\n" % (name, name, name, cls))
    src = os.path.join(OUT, "ref_generators.cpp")
    with open(src, "w") as fh:
        fh.write("".join(out))
    inc = os.path.join(ref_root, "opencl", "common", "inc")
    subprocess.check_call([cxx, "-O1", "-fPIC", "-shared", "-w", "-I", HERE, "-I", inc, src,
                           "-o", GEN_LIB])


def kernel_text(stencil, n, T, bx, by, bz, E, steps):
    """The kernel source the reference's generator emits for one case (needs
    libots_refgen.so, built by build())."""
    import ctypes
    lib = ctypes.CDLL(GEN_LIB)
    fn = getattr(lib, "gen_" + stencil.replace("-", "_"))
    fn.argtypes = [ctypes.c_int] * 7 + [ctypes.c_char_p, ctypes.c_int]
    buf = ctypes.create_string_buffer(1 << 22)
    rc = fn(n, T, bx, by, bz, E, steps, buf, len(buf))
    if rc < 0:
        raise ValueError("reference generator refused %s n=%d T=%d %dx%dx%d E=%d (rc %d)"
                         % (stencil, n, T, bx, by, bz, E, rc))
    return buf.value.decode()


# Rician's phase 2 stores the new value into bufferU while neighbouring
# work-items still read bufferU in the same phase (a race,
# opencl/rician-denoise-2d/rician-denoise-2d.cpp:322-329).  At T = 1 nothing
# reads that store (the write-back takes local0), so the case drops it.
RICIAN_T1_DEAD_STORE = "    bufferU[get_local_id(1)*1+0+1][get_local_id(0)+1] = local0;\n"


def build_kernel_case(stencil, n, T, bx, by, bz, E, steps, cxx="g++"):
    """Emit one case's kernel text with the reference's generator and compile
    oracle/ref_clkernel.cpp around it; returns the shared library's path."""
    text = kernel_text(stencil, n, T, bx, by, bz, E, steps)
    if stencil == "rician-denoise-2d":
        if T != 1 or E != 1 or text.count(RICIAN_T1_DEAD_STORE) != 1:
            raise ValueError("rician pin cases are T = 1, E = 1 only")
        text = text.replace(RICIAN_T1_DEAD_STORE, "")
    tag = "%s_n%d_T%d_%dx%dx%d_E%d_s%d" % (stencil.replace("-", "_"), n, T, bx, by, bz, E, steps)
    cl = os.path.join(OUT, "clk_%s.cl" % tag)
    with open(cl, "w") as fh:
        fh.write(text)
    lib = os.path.join(OUT, "libclk_%s.so" % tag)
    sid = GENERATORS[stencil.replace("-", "_")][2]
    subprocess.check_call([cxx, "-std=c++20", "-O1", "-ffp-contract=off", "-fPIC", "-shared",
                           "-pthread", "-w", '-DOTS_CL_KERNEL_FILE="%s"' % cl,
                           "-DOTS_CL_STENCIL=%d" % sid, os.path.join(HERE, "ref_clkernel.cpp"),
                           "-o", lib])
    return lib


# The reference's own CUDA Jacobi-2D runner (cuda/jacobi-2d/jacobi-2d.cu),
# built at T = 1 (its jacobi_2d_kernel_notimetiling, :88-105) for sm_100a: a
# GPU data point of the reference beside the engine's kernels.
CUDA_JACOBI2D = os.path.join(OUT, "ref_cuda_jacobi2d")


def build_cuda_jacobi2d(ref_root, nvcc="nvcc"):
    src = os.path.join(ref_root, "cuda", "jacobi-2d", "jacobi-2d.cu")
    if not os.path.exists(src):
        return False
    subprocess.check_call([nvcc, "-O3", "-gencode", "arch=compute_100a,code=sm_100a",
                           "-DTIME_TILE_SIZE=1", "-w", src, "-o", CUDA_JACOBI2D])
    return True


def build(ref_root=None, cxx="g++", verbose=False):
    ref_root = ref_root or os.environ.get("OTS_REFERENCE_DIR")
    if not ref_root or not os.path.isdir(os.path.join(ref_root, "opencl")):
        if verbose:
            print("build_ref: reference tree not present; keeping prebuilt oracle/_ref")
        return False
    os.makedirs(OUT, exist_ok=True)
    for name, rel in LOOPS.items():
        line, body, path = extract(ref_root, rel)
        with open(os.path.join(OUT, name + "_loop.inc"), "w") as fh:
            fh.write('#line %d "%s"\n' % (line, path))
            fh.write(body)
    gen_geometry_and_fill(ref_root)
    gen_generators(ref_root, cxx)
    try:
        build_cuda_jacobi2d(ref_root)
    except (OSError, subprocess.CalledProcessError) as e:  # optional data point
        if verbose:
            print("build_ref: reference CUDA jacobi-2d not built:", e)
    lib = os.path.join(OUT, "libots_ref.so")
    cmd = [cxx, "-O2", "-g", "-fPIC", "-shared", "-I", OUT, "-I", HERE,
           os.path.join(HERE, "ref_harness.cpp"), os.path.join(OUT, "ref_gen.cpp"), "-o", lib]
    subprocess.check_call(cmd)
    if verbose:
        print("build_ref: built", lib)
    return True


if __name__ == "__main__":
    ok = build(sys.argv[1] if len(sys.argv) > 1 else None, verbose=True)
    sys.exit(0)
