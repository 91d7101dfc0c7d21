// ref_harness.cpp -- runs the reference's OWN CPU verification loops.
//
// TEST INFRASTRUCTURE ONLY (the checker, never the product).  The reference
// runners cannot be built here (boost, OpenCL and GL headers are absent), but
// their CPU verification loops are self-contained.  oracle/build_ref.py
// extracts each loop verbatim from the reference source file into
// oracle/_ref/<name>_loop.inc (never committed) and compiles this harness
// around it with the reference's flags (g++ -O2, config.ninja:4).  The
// harness recreates the variables the loop reads -- `params.timeSteps`,
// `params.padding`, `params.paddedSize`, `refA`, `refB`, `arraySize` -- the
// way each runner's main() declares them, then hands back refA.
//
// Loops used (reference file:line):
//   jacobi-1d      opencl/jacobi-1d/jacobi-1d.cpp:631-640
//   jacobi-1d-5pt  opencl/jacobi-1d-5pt/jacobi-1d-5pt.cpp:505-516
//   jacobi-1d-7pt  opencl/jacobi-1d-7pt/jacobi-1d-7pt.cpp:513-526
//   jacobi-2d      opencl/jacobi-2d/jacobi-2d.cpp:821-834
//   poisson-2d     opencl/poisson-2d/poisson-2d.cpp:641-654
//   gradient-2d    opencl/gradient-2d/gradient-2d.cpp:686-705
// jacobi-3d's loop (opencl/jacobi-3d/jacobi-3d.cpp:726-747) is left out: its
// ARRAY_REF macro does not parenthesise its index arguments, so the loop
// reads y/z neighbours at wrong and partly out-of-bounds offsets.
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>

namespace {
struct RefParams {
  int32_t timeSteps;
  int32_t padding;
  int32_t paddedSize;
};
}  // namespace


#define OTS_REF_PROLOGUE(DIMS)                                       \
  RefParams params;                                                  \
  params.timeSteps = timeSteps;                                      \
  params.padding = padding;                                          \
  params.paddedSize = paddedSize;                                    \
  int arraySize = 1;                                                 \
  for (int d_ = 0; d_ < DIMS; ++d_) arraySize *= params.paddedSize;  \
  arraySize *= (int)sizeof(float);                                   \
  float* refA = new float[arraySize / sizeof(float)];                \
  float* refB = new float[arraySize / sizeof(float)];                \
  memcpy(refA, data, arraySize);                                     \
  memcpy(refB, data, arraySize);

#define OTS_REF_EPILOGUE        \
  memcpy(data, refA, arraySize); \
  delete[] refA;                 \
  delete[] refB;                 \
  return 0;

extern "C" int ref_jacobi_1d(float* data, int paddedSize, int padding, int timeSteps) {
  OTS_REF_PROLOGUE(1)
#include "jacobi_1d_loop.inc"
  OTS_REF_EPILOGUE
}

extern "C" int ref_jacobi_1d_5pt(float* data, int paddedSize, int padding, int timeSteps) {
  OTS_REF_PROLOGUE(1)
#include "jacobi_1d_5pt_loop.inc"
  OTS_REF_EPILOGUE
}

extern "C" int ref_jacobi_1d_7pt(float* data, int paddedSize, int padding, int timeSteps) {
  OTS_REF_PROLOGUE(1)
#include "jacobi_1d_7pt_loop.inc"
  OTS_REF_EPILOGUE
}

extern "C" int ref_jacobi_2d(float* data, int paddedSize, int padding, int timeSteps) {
  OTS_REF_PROLOGUE(2)
#include "jacobi_2d_loop.inc"
  OTS_REF_EPILOGUE
}

extern "C" int ref_poisson_2d(float* data, int paddedSize, int padding, int timeSteps) {
  OTS_REF_PROLOGUE(2)
#include "poisson_2d_loop.inc"
  OTS_REF_EPILOGUE
}

extern "C" int ref_gradient_2d(float* data, int paddedSize, int padding, int timeSteps) {
  OTS_REF_PROLOGUE(2)
#include "gradient_2d_loop.inc"
  OTS_REF_EPILOGUE
}
