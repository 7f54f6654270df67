// shade.cuh -- ray generation, the fused RGBA8 epilogue and result stores,
// shared by the per-frame and the batched kernels.
#pragma once
#include <cstdint>

#include "../../include/libsvo_b200.h"
#include "traverse.cuh"

namespace svo {

__device__ __forceinline__ uint32_t to_unorm8(float c) {
  c = c < 0.0f ? 0.0f : (c > 1.0f ? 1.0f : c);
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
