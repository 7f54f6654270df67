// batch.cu -- many views of uneven size over one or several resident octrees
// in one persistent launch.
//
// The reference renders one frame per kernel enqueue
// (raycast_serialized_opencl.cpp:729-747).  Here the launch unit is a ragged
// table of views: every view is cut into tiles of 32 x R pixels (tile_w x
// tile_h*R, R rays per lane), the tiles of all views are numbered one after
// another, and a persistent grid of warps pulls tile numbers from a global
// counter until the table is exhausted.  A warp finds its view by binary
// search over the views' first tile numbers, casts the tile's rays with the
// same traversal as the per-frame kernel (a lane takes R of them, one below
// the other tile_h rows apart), and writes RGBA8 (and optional hit records)
// into that view's output.  Blocks may stage the top records of octree 0 in shared
// memory.  Everything the launch reads lives in device descriptor tables, so
// the counter reset plus the launch are captured once as a CUDA graph and
// replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "batch.h"
#include "errors.h"
#include "shade.cuh"
#include "traverse.cuh"

namespace svo {

namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;

template <bool kExt, bool kTreelet>
__device__ __forceinline__ void trace_tile_pixel(const BatchView& v, const BatchOctree& oct,
                                                 uint32_t x, uint32_t y, const uint2* top,
                                                 uint32_t top_count, uint2* stack, int stride,
                                                 svo_stats* stats) {
  float o[3], dx, dy, dz;
  pixel_ray(v.params, x, y, o, dx, dy, dz);
  RayHit h;
  if (kTreelet)
    h = cast_ray<false>(GlobalFetch{oct.nodes}, oct.num_nodes, o, dx, dy, dz,
                        v.params.t_scale_ratio, oct.stack_size, stack, stride);
  else if (oct.traversal == SVO_TRAVERSAL_FLAT)
    h = cast_ray<true>(GlobalFetch{oct.nodes}, oct.num_nodes, o, dx, dy, dz,
                       v.params.t_scale_ratio, oct.stack_size, stack, stride);
  else if (top_count)
    h = cast_ray<false>(StagedFetch{oct.nodes, top, top_count}, oct.num_nodes, o, dx, dy, dz,
                        v.params.t_scale_ratio, oct.stack_size, stack, stride);
  else
    h = cast_ray<false>(GlobalFetch{oct.nodes}, oct.num_nodes, o, dx, dy, dz,
                        v.params.t_scale_ratio, oct.stack_size, stack, stride);
  const uint64_t pix = (uint64_t)y * v.params.width + x;
  const int m = v.params.mode;
  v.rgba[pix] = (kExt && (m == 2 || m == 6 || m == 7))
                    ? shade_ext(m, h, oct.attribs, oct.num_nodes, oct.stack_size,
                                v.params.t_scale_ratio, dx, dy, dz)
                    : shade(m, h, oct.attribs, oct.num_nodes, oct.stack_size);
  if (v.hits != nullptr) store_hit(v.hits, pix, h);
  count_stats(stats, h);
}

// kExt: some view uses view mode 2, 6 or 7 (shade_ext); batches without
// them run the instantiation that carries no extra exit state.
// kTreelet: every octree takes the treelet traversal and no records are
// staged, so only that traversal is compiled in (the register count and the
// loop are then the per-frame kernel's).
template <int TW, int TH, bool kExt, bool kTreelet>
__device__ __forceinline__ void batch_body(const BatchView* __restrict__ views, uint32_t num_views,
                                           const BatchOctree* __restrict__ octrees, uint64_t total_tiles,
                                           unsigned long long* __restrict__ counter, svo_stats* stats,
                                           int max_s, uint32_t top_nodes, uint32_t rays_per_lane) {
  static_assert(TW * TH == 32, "a tile row is one warp of rays");
  extern __shared__ uint2 smem[];
  uint2* stack = smem + threadIdx.x;
  const int stride = blockDim.x;
  uint2* top = smem + (size_t)max_s * blockDim.x;
  uint32_t top_count = 0;
  if (!kTreelet && top_nodes) {
    const BatchOctree o0 = octrees[0];
    top_count = (uint32_t)min((uint64_t)top_nodes, o0.num_nodes);
    for (uint32_t i = threadIdx.x; i < top_count; i += blockDim.x) top[i] = __ldg(o0.nodes + i);
    __syncthreads();
  }
  const uint32_t lane = threadIdx.x & 31u;
  for (;;) {
    unsigned long long tile = 0;
    if (lane == 0) tile = atomicAdd(counter, 1ull);
    tile = __shfl_sync(kFull, tile, 0);
    if (tile >= total_tiles) return;
    // the view holding this tile: last view whose first tile is <= tile
    uint32_t lo = 0, hi = num_views - 1;
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (views[mid].tile_begin <= tile)
        lo = mid;
      else
        hi = mid - 1;
    }
    const BatchView& v = views[lo];
    const uint64_t local = tile - v.tile_begin;
    const uint32_t ty = (uint32_t)(local / v.tiles_x), tx = (uint32_t)(local % v.tiles_x);
    const uint32_t x = tx * TW + lane % TW;
    const BatchOctree& oct = octrees[v.octree];
    for (uint32_t r = 0; r < rays_per_lane; ++r) {
      const uint32_t y = (ty * rays_per_lane + r) * TH + lane / TW;
      if (x < v.params.width && y < v.params.height)
        trace_tile_pixel<kExt, kTreelet>(v, oct, x, y, top, v.octree == 0 ? top_count : 0u, stack, stride,
                                         stats);
    }
    __syncwarp();
  }
}

template <int TW, int TH, bool kExt, bool kTreelet>
__global__ void batch_kernel(const BatchView* __restrict__ views, uint32_t num_views,
                             const BatchOctree* __restrict__ octrees, uint64_t total_tiles,
                             unsigned long long* __restrict__ counter, svo_stats* stats, int max_s,
                             uint32_t top_nodes, uint32_t rays_per_lane) {
  batch_body<TW, TH, kExt, kTreelet>(views, num_views, octrees, total_tiles, counter, stats, max_s,
                                     top_nodes, rays_per_lane);
}

// The same kernel for 128-thread blocks, held to 8 resident blocks per SM:
// 62 registers without spills instead of 65 and 7 blocks (the terrain batch
// of 64 views: 7.92 against 8.34 ms; at 9 blocks the registers spill and it
// is slower again).
template <int TW, int TH, bool kExt, bool kTreelet>
__global__ void __launch_bounds__(128, 8) batch_kernel_128(
    const BatchView* __restrict__ views, uint32_t num_views, const BatchOctree* __restrict__ octrees,
    uint64_t total_tiles, unsigned long long* __restrict__ counter, svo_stats* stats, int max_s,
    uint32_t top_nodes, uint32_t rays_per_lane) {
  batch_body<TW, TH, kExt, kTreelet>(views, num_views, octrees, total_tiles, counter, stats, max_s,
                                     top_nodes, rays_per_lane);
}

typedef void (*BatchKernelFn)(const BatchView*, uint32_t, const BatchOctree*, uint64_t,
                              unsigned long long*, svo_stats*, int, uint32_t, uint32_t);

template <bool kExt, bool kTreelet>
BatchKernelFn kernel_for_t(uint32_t tw, uint32_t th, bool block128) {
  if (tw == 8 && th == 4)
    return block128 ? batch_kernel_128<8, 4, kExt, kTreelet> : batch_kernel<8, 4, kExt, kTreelet>;
  if (tw == 16 && th == 2)
    return block128 ? batch_kernel_128<16, 2, kExt, kTreelet> : batch_kernel<16, 2, kExt, kTreelet>;
  if (tw == 4 && th == 8)
    return block128 ? batch_kernel_128<4, 8, kExt, kTreelet> : batch_kernel<4, 8, kExt, kTreelet>;
  if (tw == 32 && th == 1)
    return block128 ? batch_kernel_128<32, 1, kExt, kTreelet> : batch_kernel<32, 1, kExt, kTreelet>;
  return nullptr;
}

// threads: the block size the kernel is launched with (128 takes the
// register-bounded instantiation)
BatchKernelFn kernel_for(uint32_t tw, uint32_t th, bool ext, bool treelet_only, uint32_t threads) {
  const bool b128 = threads == 128;
  if (treelet_only)
    return ext ? kernel_for_t<true, true>(tw, th, b128) : kernel_for_t<false, true>(tw, th, b128);
  return ext ? kernel_for_t<true, false>(tw, th, b128) : kernel_for_t<false, false>(tw, th, b128);
}

}  // namespace

bool batch_tile_supported(uint32_t tw, uint32_t th) {
  return kernel_for(tw, th, false, false, 0) != nullptr;
}

bool batch_treelet_only(const BatchOctree* octrees, uint32_t num_octrees, uint32_t top_nodes) {
  if (top_nodes) return false;
  for (uint32_t i = 0; i < num_octrees; ++i)
    if (octrees[i].traversal != SVO_TRAVERSAL_TREELET) return false;
  return true;
}

bool batch_needs_ext(const BatchView* views, uint32_t num_views) {
  for (uint32_t i = 0; i < num_views; ++i) {
    const int32_t m = views[i].params.mode;
    if (m == 2 || m == 6 || m == 7) return true;
  }
  return false;
}

size_t batch_smem_bytes(int max_s, uint32_t threads, uint32_t top_nodes) {
  return ((size_t)max_s * threads + top_nodes) * sizeof(uint2);
}

int launch_batch(const BatchLaunch& L, cudaStream_t stream) {
  BatchKernelFn fn = kernel_for(L.tile_w, L.tile_h, L.ext, L.treelet_only, L.threads);
  if (!fn) return SVO_ERR_NOTSUP;
  const size_t smem = batch_smem_bytes(L.max_s, L.threads, L.top_nodes);
  if (smem > 48u * 1024u) {
    SVO_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  if (L.rays_per_lane < 1 || L.rays_per_lane > 4) return SVO_ERR_RANGE;
  fn<<<L.blocks, L.threads, smem, stream>>>(L.views, L.num_views, L.octrees, L.total_tiles,
                                             L.counter, L.stats, L.max_s, L.top_nodes, L.rays_per_lane);
  return cuda_status(cudaGetLastError());
}

int batch_grid(uint32_t tile_w, uint32_t tile_h, int max_s, uint32_t threads, uint32_t top_nodes,
               uint32_t blocks_per_sm, uint32_t* blocks, bool ext, bool treelet_only) {
  BatchKernelFn fn = kernel_for(tile_w, tile_h, ext, treelet_only, threads);
  if (!fn) return SVO_ERR_NOTSUP;
  const size_t smem = batch_smem_bytes(max_s, threads, top_nodes);
  if (smem > 48u * 1024u) {
    SVO_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  int dev = 0, sms = 0, fit = 0;
  SVO_CUDA_TRY(cudaGetDevice(&dev));
  SVO_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  SVO_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, fn, (int)threads, smem));
  if (fit <= 0) return SVO_ERR_RANGE;
  const uint32_t per_sm = blocks_per_sm ? std::min<uint32_t>(blocks_per_sm, (uint32_t)fit) : (uint32_t)fit;
  *blocks = per_sm * (uint32_t)sms;
  return SVO_OK;
}

}  // namespace svo
