// host_shim.h -- lets libsvo_b200/csrc/traverse.cuh compile as host C++.
//
// TEST INFRASTRUCTURE ONLY (tests/test_traverse_host.py).  The device
// intrinsics the traversal uses map to their IEEE single-precision host
// equivalents (round to nearest, no contraction: the file is built with
// -ffp-contract=off), so the host build runs the kernel's own traversal code
// and its results can be compared with the oracle without a GPU.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#define __device__
#define __forceinline__ inline
#define __restrict__

struct uint2 {
  uint32_t x, y;
};
inline uint2 make_uint2(uint32_t a, uint32_t b) { return uint2{a, b}; }
inline float __fadd_rn(float a, float b) { return a + b; }
inline float __fsub_rn(float a, float b) { return a - b; }
inline float __fmul_rn(float a, float b) { return a * b; }
inline float __fdiv_rn(float a, float b) { return a / b; }
inline float __frcp_rn(float a) { return 1.0f / a; }
inline int __popc(uint32_t v) { return __builtin_popcount(v); }
inline uint2 __ldg(const uint2* p) { return *p; }
inline uint32_t __float_as_uint(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}
inline float __uint_as_float(uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
inline float __int_as_float(int u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
using std::isfinite;
inline float fabsf(float x) { return std::fabs(x); }
