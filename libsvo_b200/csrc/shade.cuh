// shade.cuh -- ray generation, the fused RGBA8 epilogue and result stores,
// shared by the per-frame and the batched kernels.
#pragma once
#include <cstdint>

#include "../../include/libsvo_b200.h"
#include "traverse.cuh"

namespace svo {

// float -> unsigned 8-bit normalised: round(clamp(c, 0, 1) * 255), NaN -> 0.
__device__ __forceinline__ uint32_t to_unorm8(float c) {
  c = c > 0.0f ? (c < 1.0f ? c : 1.0f) : 0.0f;
  return __float2uint_rz(__fadd_rn(__fmul_rn(c, 255.0f), 0.5f));
}

__device__ __forceinline__ uint32_t pack_rgba8(float r, float g, float b, float a) {
  return to_unorm8(r) | (to_unorm8(g) << 8) | (to_unorm8(b) << 16) | (to_unorm8(a) << 24);
}

// renderToBuffer's view-mode switch (opencl/treeletRenderer_rgba.cl:644-694)
// followed by the float -> RGBA8 conversion.
__device__ __forceinline__ uint32_t shade(int mode, const RayHit& h,
                                          const uint2* __restrict__ attribs, uint64_t num_nodes,
                                          int S) {
  const float k = 0.003921569f;
  switch (mode) {
    case 0:
    case 1: {
      if (h.hit && (uint64_t)h.node < num_nodes) {
        const uint2 a = __ldg(attribs + h.node);
        const uint32_t v = mode == 0 ? a.y : a.x;
        const float r = (float)(v >> 24), g = (float)((v >> 16) & 255u),
                    b = (float)((v >> 8) & 255u);
        if (mode == 0)
          return pack_rgba8(__fmul_rn(r, k), __fmul_rn(g, k), __fmul_rn(b, k), 1.0f);
        return pack_rgba8(__fmul_rn(__fsub_rn(__fmul_rn(r, k), 0.5f), 2.0f),
                          __fmul_rn(__fsub_rn(__fmul_rn(g, k), 0.5f), 2.0f),
                          __fmul_rn(__fsub_rn(__fmul_rn(b, k), 0.5f), 2.0f), 1.0f);
      }
      return pack_rgba8(0.2f, 0.3f, 0.2f, 1.0f);
    }
    case 3: {
      const float v = __fmul_rn(__fdiv_rn((float)h.depth, (float)S), (float)h.hit);
      return pack_rgba8(v, v, v, 1.0f);
    }
    case 4: {
      const float v = __fsub_rn(1.0f, __fmul_rn(h.t, 0.1f));
      return pack_rgba8(v, v, v, 1.0f);
    }
    case 5: {
      const float v = __fsub_rn(1.0f, __fdiv_rn((float)h.loops, 200.0f));
      return pack_rgba8(v, v, v, 1.0f);
    }
    default:
      return pack_rgba8(0.0f, 0.0f, 0.0f, 1.0f);
  }
}

// OpenCL dot() and normalize() pinned to (x*x + y*y) + z*z and v / sqrt(dot).
__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
  return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}
__device__ __forceinline__ void normalize3(float& x, float& y, float& z) {
  const float l = __fsqrt_rn(dot3(x, y, z, x, y, z));
  x = __fdiv_rn(x, l);
  y = __fdiv_rn(y, l);
  z = __fdiv_rn(z, l);
}

// getNormal / getColor (opencl/treeletRenderer_rgba.cl:388-404).
__device__ __forceinline__ void unpack_normal(uint32_t v, float& x, float& y, float& z) {
  const float k = 0.003921569f;
  x = __fmul_rn(__fsub_rn(__fmul_rn((float)(v >> 24), k), 0.5f), 2.0f);
  y = __fmul_rn(__fsub_rn(__fmul_rn((float)((v >> 16) & 255u), k), 0.5f), 2.0f);
  z = __fmul_rn(__fsub_rn(__fmul_rn((float)((v >> 8) & 255u), k), 0.5f), 2.0f);
}
__device__ __forceinline__ void unpack_color(uint32_t v, float c[4]) {
  const float k = 0.003921569f;
  c[0] = __fmul_rn((float)(v >> 24), k);
  c[1] = __fmul_rn((float)((v >> 16) & 255u), k);
  c[2] = __fmul_rn((float)((v >> 8) & 255u), k);
  c[3] = __fmul_rn((float)(v & 255u), k);
}

// smoothstep(0, 1, x) with t = clamp(x, 0, 1) and t * t * (3 - 2t) in that order.
__device__ __forceinline__ float smoothstep01(float x) {
  const float t = x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x);
  return __fmul_rn(__fmul_rn(t, t), __fsub_rn(3.0f, __fmul_rn(2.0f, t)));
}

// Adjust (opencl/treeletRenderer_rgba.cl:518-528).  Gamma is the double
// literal 0.80, so the power and the scaling by 255 run in double.
__device__ __forceinline__ float wl_adjust(float color, float factor) {
  if (color == 0.0f) return 0.0f;
  const int res = (int)round(255.0 * pow((double)__fmul_rn(color, factor), 0.80));
  return (float)(res < 0 ? 0 : (res > 255 ? 255 : res));
}

// DataPointToColor(value, 0, vmax) (opencl/treeletRenderer_rgba.cl:532-603):
// the value mapped to a visible wavelength, then to RGB.
__device__ __forceinline__ void wavelength_color(float value, float vmax, float rgb[3]) {
  const float w = __fadd_rn(__fmul_rn(__fdiv_rn(__fsub_rn(value, 0.0f), __fsub_rn(vmax, 0.0f)), 400.0f),
                            380.0f);
  float r, g, b, f;
  if (380.0f <= w && w <= 440.0f) {
    r = __fdiv_rn(-__fsub_rn(w, 440.0f), 60.0f);
    g = 0.0f;
    b = 1.0f;
  } else if (440.0f < w && w <= 490.0f) {
    r = 0.0f;
    g = __fdiv_rn(__fsub_rn(w, 440.0f), 50.0f);
    b = 1.0f;
  } else if (490.0f < w && w <= 510.0f) {
    r = 0.0f;
    g = 1.0f;
    b = __fdiv_rn(-__fsub_rn(w, 510.0f), 20.0f);
  } else if (510.0f < w && w <= 580.0f) {
    r = __fdiv_rn(__fsub_rn(w, 510.0f), 70.0f);
    g = 1.0f;
    b = 0.0f;
  } else if (580.0f < w && w <= 645.0f) {
    r = 1.0f;
    g = __fdiv_rn(-__fsub_rn(w, 645.0f), 65.0f);
    b = 0.0f;
  } else if (645.0f < w && w <= 780.0f) {
    r = 1.0f;
    g = 0.0f;
    b = 0.0f;
  } else {
    r = g = b = 0.0f;
  }
  if (380.0f <= w && w <= 420.0f)
    f = __fadd_rn(0.3f, __fdiv_rn(__fmul_rn(0.7f, __fsub_rn(w, 380.0f)), 40.0f));
  else if (420.0f < w && w <= 701.0f)
    f = 1.0f;
  else if (701.0f < w && w <= 780.0f)
    f = __fadd_rn(0.3f, __fdiv_rn(__fmul_rn(0.7f, __fsub_rn(780.0f, w)), 79.0f));
  else
    f = 0.0f;
  const float fac = __fdiv_rn(1.0f, 255.0f);
  rgb[0] = __fmul_rn(wl_adjust(r, f), fac);
  rgb[1] = __fmul_rn(wl_adjust(g, f), fac);
  rgb[2] = __fmul_rn(wl_adjust(b, f), fac);
}

// The view modes that need more than the hit record: 2 (iteration count as a
// wavelength colour), 6 (shade_phong, :451-504, whose shadow ray is compiled
// out in the reference) and 7 (LOD quality, :715-733).  d is the unclamped
// primary direction.  Modes 6 and 7 use the node centre and the quality that
// only the treelet traversal reports.
__device__ __forceinline__ uint32_t shade_ext(int mode, const RayHit& h,
                                              const uint2* __restrict__ attribs,
                                              uint64_t num_nodes, int S, float tsr, float dx,
                                              float dy, float dz) {
  if (mode == 2) {
    float rgb[3];
    wavelength_color((float)h.loops, (float)(S * 30), rgb);
    return pack_rgba8(rgb[0], rgb[1], rgb[2], 1.0f);
  }
  if (mode == 7) {
    if (!h.hit) return pack_rgba8(0.6f, 0.3f, 0.3f, 1.0f);
    const float q = h.leaf ? __fsub_rn(h.sx2, __fmul_rn(tsr, h.tc_min)) : 0.0f;
    const float v = __fsqrt_rn(__fsqrt_rn(q));
    return pack_rgba8(v, v, v, 1.0f);
  }
  // mode 6
  if (!h.hit) return pack_rgba8(0.4f, 0.6f, 0.4f, 1.0f);
  if ((uint64_t)h.node >= num_nodes) return pack_rgba8(0.0f, 0.0f, 0.0f, 1.0f);
  const uint2 a = __ldg(attribs + h.node);
  float nx, ny, nz, c[4];
  unpack_normal(a.x, nx, ny, nz);
  normalize3(nx, ny, nz);
  unpack_color(a.y, c);
  float lx = __fsub_rn(-120.0f, h.cx), ly = __fsub_rn(0.0f, h.cy), lz = __fsub_rn(0.0f, h.cz);
  normalize3(lx, ly, lz);
  const float ndl = cl_max(0.0f, dot3(nx, ny, nz, lx, ly, lz));
  float rfx = __fsub_rn(__fmul_rn(__fmul_rn(2.0f, nx), ndl), lx);
  float rfy = __fsub_rn(__fmul_rn(__fmul_rn(2.0f, ny), ndl), ly);
  float rfz = __fsub_rn(__fmul_rn(__fmul_rn(2.0f, nz), ndl), lz);
  normalize3(rfx, rfy, rfz);
  const float rdv = cl_max(0.0f, dot3(rfx, rfy, rfz, -dx, -dy, -dz));
  const float spec = __fmul_rn(cl_max(0.0f, powf(rdv, 10.0f)), ndl > 0.0f ? 1.0f : 0.0f);
  // shadow = 1 - 0: color * 0.5 + (color * nDotL * 1 + specular * 1 * 0.2) * 0.5
  const float s = __fmul_rn(spec, 0.2f);
  float o[3];
  for (int i = 0; i < 3; ++i)
    o[i] = smoothstep01(__fadd_rn(__fmul_rn(c[i], 0.5f), __fmul_rn(__fadd_rn(__fmul_rn(c[i], ndl), s), 0.5f)));
  return pack_rgba8(o[0], o[1], o[2], 1.0f);
}

__device__ __forceinline__ void store_hit(svo_hit* hits, uint64_t i, const RayHit& h) {
  uint4 w;
  w.x = h.node;
  w.y = __float_as_uint(h.t);
  w.z = (h.depth & 0xFFFFu) | ((h.hit & 0xFFu) << 16) | ((h.flags & 0xFFu) << 24);
  w.w = (h.loops & 0xFFFFu) | (h.fetches << 16);
  reinterpret_cast<uint4*>(hits)[i] = w;
}

__device__ __forceinline__ void count_stats(svo_stats* stats, const RayHit& h) {
  if (stats == nullptr) return;
  if (h.flags == SVO_HITFLAG_CAPPED) atomicAdd(&stats->capped_rays, 1u);
  if (h.flags == SVO_HITFLAG_BOUNDS) atomicAdd(&stats->bounds_errors, 1u);
}

// renderToBuffer ray generation (opencl/treeletRenderer_rgba.cl:627-633).
__device__ __forceinline__ void pixel_ray(const svo_frame_params& p, uint32_t x, uint32_t y,
                                          float o[3], float& dx, float& dy, float& dz) {
  const float fx = (float)x;
  const float fy = (float)(p.height - y);
  const float qx = __fadd_rn(__fadd_rn(p.far_lower_left[0], __fmul_rn(p.pixel_far_h[0], fx)),
                             __fmul_rn(p.pixel_far_v[0], fy));
  const float qy = __fadd_rn(__fadd_rn(p.far_lower_left[1], __fmul_rn(p.pixel_far_h[1], fx)),
                             __fmul_rn(p.pixel_far_v[1], fy));
  const float qz = __fadd_rn(__fadd_rn(p.far_lower_left[2], __fmul_rn(p.pixel_far_h[2], fx)),
                             __fmul_rn(p.pixel_far_v[2], fy));
  const float vx = __fsub_rn(qx, p.camera_position[0]);
  const float vy = __fsub_rn(qy, p.camera_position[1]);
  const float vz = __fsub_rn(qz, p.camera_position[2]);
  const float len =
      __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz)));
  dx = __fdiv_rn(vx, len);
  dy = __fdiv_rn(vy, len);
  dz = __fdiv_rn(vz, len);
  o[0] = p.camera_position[0];
  o[1] = p.camera_position[1];
  o[2] = p.camera_position[2];
}

}  // namespace svo
