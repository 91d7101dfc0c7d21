// ref_shim.hpp -- context the reference's GeneratorParams structs and fill
// loops need when compiled outside their runners (test infrastructure only;
// see build_ref.py).  Supplies boost::math::gcd/lcm (Euclid's algorithm,
// non-negative results, lcm(0, x) = 0 as boost defines them), turns the
// reference's assert() into an exception so an invalid geometry is reported
// instead of aborting, and declares the RefParams holder used by the fills.
#ifndef OTS_REF_SHIM_HPP
#define OTS_REF_SHIM_HPP
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>

namespace boost {
namespace math {
template <typename T>
T gcd(T a, T b) {
  if (a < 0) a = -a;
  if (b < 0) b = -b;
  while (b != 0) {
    T t = a % b;
    a = b;
    b = t;
  }
  return a;
}
template <typename T>
T lcm(T a, T b) {
  if (a == 0 || b == 0) return 0;
  T g = gcd(a, b);
  T l = a / g * b;
  return l < 0 ? -l : l;
}
}  // namespace math
}  // namespace boost

#undef assert
#define assert(cond)                                              \
  do {                                                            \
    if (!(cond)) throw std::runtime_error("reference assertion"); \
  } while (0)

namespace {
struct RefParams {
  int32_t timeSteps;
  int32_t padding;
  int32_t paddedSize;
};
}  // namespace
#endif
