// render.cu -- the per-frame ray cast (renderToBuffer) and explicit-ray cast.
//
// Replaces the OpenCL kernel renderToBuffer (opencl/treeletRenderer_rgba.cl:
// 610-734) and its enqueue (projects/raycast_serialized_opencl/src/
// raycast_serialized_opencl.cpp:729-747).  One thread per pixel; a warp
// covers an 8x4 pixel tile so neighbouring rays walk the same nodes; a block
// of 128 threads covers 16x8 pixels (smaller blocks than 16x16 measured 3 %
// faster on a 1080p frame and 10 % on 512x512: the last wave is shorter).
// The RGBA8 epilogue is fused.
#include <cuda_runtime.h>

#include "render.h"
#include "shade.cuh"
#include "traverse.cuh"

namespace svo {

namespace {

constexpr int kBlockW = 16;  // 128 threads: finer blocks balance the tail of a frame
constexpr int kBlockH = 8;
constexpr int kThreads = kBlockW * kBlockH;

// kExt: view modes 2, 6 and 7 (shade_ext); the other modes compile without
// the extra exit state.
template <bool kFlat, bool kExt>
__global__ void __launch_bounds__(kThreads) render_frame_kernel(
    const uint2* __restrict__ nodes, const uint2* __restrict__ attribs, uint64_t num_nodes,
    const svo_frame_params p, int S, uint32_t* __restrict__ rgba, svo_hit* __restrict__ hits,
    svo_stats* __restrict__ stats, uint32_t y0) {
  extern __shared__ uint2 stack_smem[];
  const int t = threadIdx.x;
  const int warp = t >> 5, lane = t & 31;
  // warp w covers pixels [8*(w&1), +8) x [4*(w>>1), +4) of the 16x8 block;
  // rows start at y0 (frames taller than one grid's rows take several launches)
  const uint32_t x = blockIdx.x * kBlockW + (warp % (kBlockW / 8)) * 8 + (lane & 7);
  const uint32_t y = y0 + blockIdx.y * kBlockH + (warp / (kBlockW / 8)) * 4 + (lane >> 3);
  if (x >= p.width || y >= p.height) return;
  float o[3], dx, dy, dz;
  pixel_ray(p, x, y, o, dx, dy, dz);
  const RayHit h = cast_ray<kFlat>(GlobalFetch{nodes}, num_nodes, o, dx, dy, dz, p.t_scale_ratio,
                                   S, stack_smem + t, kThreads);
  const uint64_t pix = (uint64_t)y * p.width + x;
  rgba[pix] = kExt ? shade_ext(p.mode, h, attribs, num_nodes, S, p.t_scale_ratio, dx, dy, dz)
                   : shade(p.mode, h, attribs, num_nodes, S);
  if (hits != nullptr) store_hit(hits, pix, h);
  count_stats(stats, h);
}

// Primary ray plus one shadow ray per hit, shaded as shade_diffuse_color_shadow
// (opencl/fillFrameBuffer_rgba.cl:494-529) with the live renderer's attribute
// addressing (attribute index = node index, :388-404):
//   n = getNormal, c = getColor, nDotL = max(0, dot(n, L)),
//   shadow = sample(nodeCenter + n * offset, L, tsr_shadow) ? 1 : 0,
//   colour = c * nDotL * (1 - shadow) + c * 0.2, alpha 1; misses, and hits
//   outside the pool, (0.2, 0.3, 0.2).
// The shadow ray reuses the primary ray's stack columns.
__global__ void __launch_bounds__(kThreads) render_shadow_kernel(
    const uint2* __restrict__ nodes, const uint2* __restrict__ attribs, uint64_t num_nodes,
    const svo_frame_params p, const svo_shadow_cfg sc, int S, uint32_t* __restrict__ rgba,
    svo_hit* __restrict__ hits, svo_hit* __restrict__ shadow_hits,
    svo_stats* __restrict__ stats, uint32_t y0) {
  extern __shared__ uint2 stack_smem[];
  const int t = threadIdx.x;
  const int warp = t >> 5, lane = t & 31;
  const uint32_t x = blockIdx.x * kBlockW + (warp % (kBlockW / 8)) * 8 + (lane & 7);
  const uint32_t y = y0 + blockIdx.y * kBlockH + (warp / (kBlockW / 8)) * 4 + (lane >> 3);
  if (x >= p.width || y >= p.height) return;
  float o[3], dx, dy, dz;
  pixel_ray(p, x, y, o, dx, dy, dz);
  const RayHit h = cast_ray<false>(GlobalFetch{nodes}, num_nodes, o, dx, dy, dz, p.t_scale_ratio,
                                   S, stack_smem + t, kThreads);
  const uint64_t pix = (uint64_t)y * p.width + x;
  uint32_t out = pack_rgba8(0.2f, 0.3f, 0.2f, 1.0f);
  RayHit sh;
  sh.node = 0u;
  sh.t = 0.0f;
  sh.depth = sh.hit = sh.flags = sh.loops = sh.fetches = 0u;
  if (h.hit && (uint64_t)h.node < num_nodes) {
    {
      const uint2 a = __ldg(attribs + h.node);
      float nx, ny, nz, c[4];
      unpack_normal(a.x, nx, ny, nz);
      unpack_color(a.y, c);
      const float lx = sc.light_direction[0], ly = sc.light_direction[1],
                  lz = sc.light_direction[2];
      const float ndl = cl_max(0.0f, dot3(nx, ny, nz, lx, ly, lz));
      const float so[3] = {__fadd_rn(h.cx, __fmul_rn(nx, sc.normal_offset)),
                           __fadd_rn(h.cy, __fmul_rn(ny, sc.normal_offset)),
                           __fadd_rn(h.cz, __fmul_rn(nz, sc.normal_offset))};
      sh = cast_ray<false>(GlobalFetch{nodes}, num_nodes, so, lx, ly, lz, sc.t_scale_ratio, S,
                           stack_smem + t, kThreads);
      const float lit = __fsub_rn(1.0f, sh.hit ? 1.0f : 0.0f);
      float r[3];
      for (int i = 0; i < 3; ++i)
        r[i] = __fadd_rn(__fmul_rn(__fmul_rn(c[i], ndl), lit), __fmul_rn(c[i], 0.2f));
      out = pack_rgba8(r[0], r[1], r[2], 1.0f);
      count_stats(stats, sh);
    }
  }
  rgba[pix] = out;
  if (hits != nullptr) store_hit(hits, pix, h);
  if (shadow_hits != nullptr) store_hit(shadow_hits, pix, sh);
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

// Rows of one launch: a grid has at most 65535 blocks along y.
constexpr uint32_t kRowsPerLaunch = 65535u * kBlockH;

int launch_render(const svo_node* nodes, const svo_attrib* attribs, uint64_t num_nodes,
                  const svo_frame_params& p, const svo_trace_cfg& cfg, uint32_t* rgba,
                  svo_hit* hits, svo_stats* stats, cudaStream_t stream) {
  if (p.width == 0 || p.height == 0) return SVO_OK;
  if (p.height > 0xFFFFFFF0u) return SVO_ERR_RANGE;  // row indices stay below 2^32
  const int S = cfg.stack_size;
  const size_t smem = render_smem_bytes(S);
  const uint2* n2 = reinterpret_cast<const uint2*>(nodes);
  const uint2* a2 = reinterpret_cast<const uint2*>(attribs);
  const bool ext = p.mode == 2 || p.mode == 6 || p.mode == 7;
  const bool flat = cfg.traversal == SVO_TRAVERSAL_FLAT;
  auto* fn = flat ? (ext ? render_frame_kernel<true, true> : render_frame_kernel<true, false>)
                  : (ext ? render_frame_kernel<false, true> : render_frame_kernel<false, false>);
  for (uint32_t y0 = 0; y0 < p.height; y0 += kRowsPerLaunch) {
    const uint32_t rows = p.height - y0 < kRowsPerLaunch ? p.height - y0 : kRowsPerLaunch;
    const dim3 grid((p.width + kBlockW - 1) / kBlockW, (rows + kBlockH - 1) / kBlockH);
    fn<<<grid, kThreads, smem, stream>>>(n2, a2, num_nodes, p, S, rgba, hits, stats, y0);
    if (cudaGetLastError() != cudaSuccess) return SVO_ERR_CUDA;
  }
  return SVO_OK;
}

int launch_render_shadow(const svo_node* nodes, const svo_attrib* attribs, uint64_t num_nodes,
                         const svo_frame_params& p, const svo_shadow_cfg& sc, int S,
                         uint32_t* rgba, svo_hit* hits, svo_hit* shadow_hits, svo_stats* stats,
                         cudaStream_t stream) {
  if (p.width == 0 || p.height == 0) return SVO_OK;
  if (p.height > 0xFFFFFFF0u) return SVO_ERR_RANGE;  // row indices stay below 2^32
  for (uint32_t y0 = 0; y0 < p.height; y0 += kRowsPerLaunch) {
    const uint32_t rows = p.height - y0 < kRowsPerLaunch ? p.height - y0 : kRowsPerLaunch;
    const dim3 grid((p.width + kBlockW - 1) / kBlockW, (rows + kBlockH - 1) / kBlockH);
    render_shadow_kernel<<<grid, kThreads, render_smem_bytes(S), stream>>>(
        reinterpret_cast<const uint2*>(nodes), reinterpret_cast<const uint2*>(attribs), num_nodes,
        p, sc, S, rgba, hits, shadow_hits, stats, y0);
    if (cudaGetLastError() != cudaSuccess) return SVO_ERR_CUDA;
  }
  return SVO_OK;
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
