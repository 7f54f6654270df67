// render.cu -- the per-frame ray cast (renderToBuffer) and explicit-ray cast.
//
// Replaces the OpenCL kernel renderToBuffer (opencl/treeletRenderer_rgba.cl:
// 610-734) and its enqueue (projects/raycast_serialized_opencl/src/
// raycast_serialized_opencl.cpp:729-747).  One thread per pixel; a warp
// covers an 8x4 pixel tile so neighbouring rays walk the same nodes; a block
// of 256 threads covers 16x16 pixels.  The RGBA8 epilogue is fused.
#include <cuda_runtime.h>

#include "render.h"
#include "shade.cuh"
#include "traverse.cuh"

namespace svo {

namespace {

constexpr int kBlockW = 16;
constexpr int kBlockH = 16;
constexpr int kThreads = kBlockW * kBlockH;

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
  const RayHit h = cast_ray<kFlat>(GlobalFetch{nodes}, num_nodes, o, dx, dy, dz, p.t_scale_ratio,
                                   S, stack_smem + t, kThreads);
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
  const RayHit h = cast_ray<kFlat>(GlobalFetch{nodes}, num_nodes, o, dirs[3 * i], dirs[3 * i + 1],
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
