// render.cu -- the per-frame ray cast (renderToBuffer) and explicit-ray cast.
//
// Replaces the OpenCL kernel renderToBuffer (opencl/treeletRenderer_rgba.cl:
// 610-734) and its enqueue (projects/raycast_serialized_opencl/src/
// raycast_serialized_opencl.cpp:729-747).  One thread per pixel; a warp
// covers an 8x4 pixel tile so neighbouring rays walk the same nodes; a block
// of 256 threads covers 16x16 pixels.  The RGBA8 epilogue is fused.
#include <cuda_runtime.h>

#include "render.h"
#include "traverse.cuh"

namespace svo {

namespace {

constexpr int kBlockW = 16;
constexpr int kBlockH = 16;
constexpr int kThreads = kBlockW * kBlockH;

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

template <bool kFlat>
__global__ void __launch_bounds__(kThreads) render_frame_kernel(
    const uint2* __restrict__ nodes, const uint2* __restrict__ attribs, uint64_t num_nodes,
    const svo_frame_params p, int S, uint32_t* __restrict__ rgba, svo_hit* __restrict__ hits,
    svo_stats* __restrict__ stats) {
  extern __shared__ uint2 stack_smem[];
  const int t = threadIdx.x;
  const int warp = t >> 5, lane = t & 31;
  // warp w covers pixels [8*(w&1), +8) x [4*(w>>1), +4) of the 16x16 block
  const uint32_t x = blockIdx.x * kBlockW + (warp & 1) * 8 + (lane & 7);
  const uint32_t y = blockIdx.y * kBlockH + (warp >> 1) * 4 + (lane >> 3);
  if (x >= p.width || y >= p.height) return;
  float o[3], dx, dy, dz;
  pixel_ray(p, x, y, o, dx, dy, dz);
  const RayHit h = cast_ray<kFlat>(nodes, num_nodes, o, dx, dy, dz, p.t_scale_ratio, S,
                                   stack_smem + t, kThreads);
  const uint64_t pix = (uint64_t)y * p.width + x;
  rgba[pix] = shade(p.mode, h, attribs, num_nodes, S);
  if (hits != nullptr) store_hit(hits, pix, h);
  count_stats(stats, h);
}

template <bool kFlat>
__global__ void __launch_bounds__(kThreads) trace_rays_kernel(
    const uint2* __restrict__ nodes, uint64_t num_nodes, const float* __restrict__ origins,
    const float* __restrict__ dirs, uint64_t n, float tsr, int S, svo_hit* __restrict__ hits,
    svo_stats* __restrict__ stats) {
  extern __shared__ uint2 stack_smem[];
  const uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
  if (i >= n) return;
  const float o[3] = {origins[3 * i], origins[3 * i + 1], origins[3 * i + 2]};
  const RayHit h = cast_ray<kFlat>(nodes, num_nodes, o, dirs[3 * i], dirs[3 * i + 1],
                                   dirs[3 * i + 2], tsr, S, stack_smem + threadIdx.x, kThreads);
  store_hit(hits, i, h);
  count_stats(stats, h);
}

}  // namespace

size_t render_smem_bytes(int S) { return (size_t)S * kThreads * sizeof(uint2); }

int launch_render(const svo_node* nodes, const svo_attrib* attribs, uint64_t num_nodes,
                  const svo_frame_params& p, const svo_trace_cfg& cfg, uint32_t* rgba,
                  svo_hit* hits, svo_stats* stats, cudaStream_t stream) {
  if (p.width == 0 || p.height == 0) return SVO_OK;
  const dim3 grid((p.width + kBlockW - 1) / kBlockW, (p.height + kBlockH - 1) / kBlockH);
  const int S = cfg.stack_size;
  const size_t smem = render_smem_bytes(S);
  const uint2* n2 = reinterpret_cast<const uint2*>(nodes);
  const uint2* a2 = reinterpret_cast<const uint2*>(attribs);
  if (cfg.traversal == SVO_TRAVERSAL_FLAT)
    render_frame_kernel<true><<<grid, kThreads, smem, stream>>>(n2, a2, num_nodes, p, S, rgba,
                                                                hits, stats);
  else
    render_frame_kernel<false><<<grid, kThreads, smem, stream>>>(n2, a2, num_nodes, p, S, rgba,
                                                                 hits, stats);
  return cudaGetLastError() == cudaSuccess ? SVO_OK : SVO_ERR_CUDA;
}

int launch_trace_rays(const svo_node* nodes, uint64_t num_nodes, const float* origins,
                      const float* dirs, uint64_t n, float tsr, const svo_trace_cfg& cfg,
                      svo_hit* hits, svo_stats* stats, cudaStream_t stream) {
  if (n == 0) return SVO_OK;
  const uint64_t blocks = (n + kThreads - 1) / kThreads;
  if (blocks > 0x7FFFFFFFull) return SVO_ERR_RANGE;
  const int S = cfg.stack_size;
  const size_t smem = render_smem_bytes(S);
  const uint2* n2 = reinterpret_cast<const uint2*>(nodes);
  if (cfg.traversal == SVO_TRAVERSAL_FLAT)
    trace_rays_kernel<true><<<(unsigned)blocks, kThreads, smem, stream>>>(
        n2, num_nodes, origins, dirs, n, tsr, S, hits, stats);
  else
    trace_rays_kernel<false><<<(unsigned)blocks, kThreads, smem, stream>>>(
        n2, num_nodes, origins, dirs, n, tsr, S, hits, stats);
  return cudaGetLastError() == cudaSuccess ? SVO_OK : SVO_ERR_CUDA;
}

}  // namespace svo
