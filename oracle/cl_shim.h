// cl_shim.h -- lets the reference's OpenCL C kernel source compile as host C++.
//
// TEST INFRASTRUCTURE ONLY (see oracle/build_ref.py).  The reference's
// opencl/treeletRenderer_rgba.cl is read at build time, its OpenCL vector
// literals `(floatN)(...)` are rewritten to `make_floatN(...)` in memory, and
// the result is compiled after this header so that the reference's own
// sample(), intersectAABB(), ray generation and shading code run on the CPU.
//
// OpenCL built-ins whose results the OpenCL specification leaves to the
// implementation are pinned here to the same definitions the oracle uses:
//   normalize(v) = v / sqrt(dot(v, v)),  dot = (x*x + y*y) + z*z (+ w*w),
//   max(a, b) = (a < b) ? b : a,  min(a, b) = (b < a) ? b : a,
//   sign(x) per OpenCL C (x itself for +-0, 0 for NaN).
#pragma once
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

using std::fabs;
using std::pow;
using std::round;
using std::sqrt;

struct float3 {
  float x, y, z;
};
struct float4 {
  union {
    struct {
      float x, y, z, w;
    };
    float3 xyz;
  };
};
struct int2 {
  int x, y;
};
struct float16 {
  float s[16];
};

inline float3 make_float3(float a, float b, float c) { return float3{a, b, c}; }
inline float4 make_float4(float a, float b, float c, float d) {
  float4 v;
  v.x = a;
  v.y = b;
  v.z = c;
  v.w = d;
  return v;
}
inline float4 make_float4(float3 a, float d) { return make_float4(a.x, a.y, a.z, d); }
inline int2 make_int2(int a, int b) { return int2{a, b}; }

inline float3 operator+(float3 a, float3 b) { return float3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline float3 operator-(float3 a, float3 b) { return float3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline float3 operator-(float3 a) { return float3{-a.x, -a.y, -a.z}; }
template <class T>
inline float3 operator*(float3 a, T s) {
  const float f = (float)s;
  return float3{a.x * f, a.y * f, a.z * f};
}
template <class T>
inline float3 operator*(T s, float3 a) {
  const float f = (float)s;
  return float3{f * a.x, f * a.y, f * a.z};
}
inline float4 operator+(float4 a, float4 b) {
  return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
inline float4 operator-(float4 a, float4 b) {
  return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}
inline float4 operator+(float4 a, float s) { return make_float4(a.x + s, a.y + s, a.z + s, a.w + s); }
template <class T>
inline float4 operator*(float4 a, T s) {
  const float f = (float)s;
  return make_float4(a.x * f, a.y * f, a.z * f, a.w * f);
}

inline float dot(float3 a, float3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline float dot(float4 a, float4 b) { return ((a.x * b.x + a.y * b.y) + a.z * b.z) + a.w * b.w; }
inline float3 normalize(float3 v) {
  const float l = std::sqrt(dot(v, v));
  return float3{v.x / l, v.y / l, v.z / l};
}
inline float4 normalize(float4 v) {
  const float l = std::sqrt(dot(v, v));
  return make_float4(v.x / l, v.y / l, v.z / l, v.w / l);
}

inline float max(float a, float b) { return (a < b) ? b : a; }
inline float min(float a, float b) { return (b < a) ? b : a; }
inline int max(int a, int b) { return (a < b) ? b : a; }
inline int min(int a, int b) { return (b < a) ? b : a; }
inline float sign(float v) {
  if (v > 0.0f) return 1.0f;
  if (v < 0.0f) return -1.0f;
  if (v == 0.0f) return v;
  return 0.0f;
}
inline float smoothstep(float e0, float e1, float x) {
  float t = (x - e0) / (e1 - e0);
  t = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);
  return t * t * (3.0f - 2.0f * t);
}

// image2d_t: a host float RGBA image the harness reads back.
struct cl_shim_image {
  float* rgba;
  uint32_t width;
};
typedef cl_shim_image* image2d_t;
inline void write_imagef(image2d_t img, int2 p, float4 c) {
  float* px = img->rgba + 4 * ((size_t)p.y * img->width + (size_t)p.x);
  px[0] = c.x;
  px[1] = c.y;
  px[2] = c.z;
  px[3] = c.w;
}

// NDRange work-item id of the calling host thread.
extern thread_local size_t cl_shim_global_id[2];
inline size_t get_global_id(int dim) { return cl_shim_global_id[dim]; }

#define __kernel
#define __global
#define __write_only
#define private
