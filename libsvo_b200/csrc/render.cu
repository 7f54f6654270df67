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

#include <mutex>

#include "render.h"
#include "shade.cuh"
#include "traverse.cuh"

namespace svo {

namespace {

constexpr int kBlockW = 16;  // 128 threads: finer blocks balance the tail of a frame
constexpr int kBlockH = 8;
constexpr int kThreads = kBlockW * kBlockH;

// kExt: view modes 2, 6 and 7 (shade_ext); the other modes compile without
// the extra exit state.  `order` (optional, 1-D grid): block b casts the
// 16x8 block order[b] of a frame gx blocks wide, so blocks go to the SMs in
// that order; without it the grid is the frame's blocks in raster order.
template <bool kFlat, bool kExt>
__global__ void __launch_bounds__(kThreads) render_frame_kernel(
    const uint2* __restrict__ nodes, const uint2* __restrict__ attribs, uint64_t num_nodes,
    const svo_frame_params p, int S, uint32_t* __restrict__ rgba, svo_hit* __restrict__ hits,
    svo_stats* __restrict__ stats, uint32_t y0, const uint32_t* __restrict__ order, uint32_t gx) {
  extern __shared__ uint2 stack_smem[];
  const int t = threadIdx.x;
  const int warp = t >> 5, lane = t & 31;
  uint32_t bx = blockIdx.x, by = blockIdx.y;
  if (order != nullptr) {
    const uint32_t b = order[blockIdx.x];
    bx = b % gx;
    by = b / gx;
  }
  // warp w covers pixels [8*(w&1), +8) x [4*(w>>1), +4) of the 16x8 block;
  // rows start at y0 (frames taller than one grid's rows take several launches)
  const uint32_t x = bx * kBlockW + (warp % (kBlockW / 8)) * 8 + (lane & 7);
  const uint32_t y = y0 + by * kBlockH + (warp / (kBlockW / 8)) * 4 + (lane >> 3);
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

// ---- longest-first dispatch ------------------------------------------------
// A frame's blocks differ in cost by two orders of magnitude (rays that graze
// a surface run hundreds of iterations, most rays a dozen), and raster order
// starts some of the longest blocks last, where they run on after the other
// SMs are done.  Large frames therefore estimate each 16x8 block's cost first
// (its two 8x8 cells' top-left rays, cut off at kCostCap iterations), sort the
// blocks by it, costliest first, and hand the frame kernel that order.  Every
// pixel is still cast by the same code: only the order the blocks start in
// changes.  On the 1920x1080 icosphere frame the ordered frame kernel takes
// 254 us against 311 us in raster order, about the 246 us of its longest
// block alone.  The estimate is a chain of dependent node reads per ray, so
// its time grows with the cap: 48 iterations measured best (32 and 96 order
// the frame worse or cost more than they save).
constexpr uint32_t kCostCap = 48;
constexpr uint32_t kCostSamples = kBlockW / 8;  // one ray per 8x8 cell of a block
constexpr uint64_t kOrderMinPixels = 1ull << 20;
constexpr uint32_t kSortThreads = 1024;
// the sort keeps one byte per block in shared memory
constexpr uint32_t kOrderMaxBlocks = 160u * 1024u;

// sample_cost[b * 2 + c]: iterations of block b's sample ray c, capped (0
// for a sample outside the frame).  One byte per sample, every byte written,
// so the array needs no clearing.
template <bool kFlat>
__global__ void __launch_bounds__(kThreads) block_cost_kernel(
    const uint2* __restrict__ nodes, uint64_t num_nodes, const svo_frame_params p, int S,
    uint32_t gx, uint32_t nblocks, uint8_t* __restrict__ sample_cost) {
  extern __shared__ uint2 stack_smem[];
  const uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
  if (i >= (uint64_t)nblocks * kCostSamples) return;
  const uint32_t b = (uint32_t)(i / kCostSamples), c = (uint32_t)(i % kCostSamples);
  const uint32_t x = (b % gx) * kBlockW + c * 8, y = (b / gx) * kBlockH;
  uint32_t loops = 0u;
  if (x < p.width && y < p.height) {
    float o[3], dx, dy, dz;
    pixel_ray(p, x, y, o, dx, dy, dz);
    loops = cast_ray<kFlat>(GlobalFetch{nodes}, num_nodes, o, dx, dy, dz, p.t_scale_ratio, S,
                            stack_smem + threadIdx.x, kThreads, kCostCap)
                .loops;
  }
  sample_cost[i] = (uint8_t)min(loops, kCostCap);
}

// The lanes of the warp whose key equals this lane's, for keys below 128:
// seven ballots, one per key bit (cheaper than __match_any_sync, whose
// latency made the sort several times slower).
__device__ __forceinline__ uint32_t same_key_lanes(uint32_t k) {
  uint32_t peers = 0xFFFFFFFFu;
#pragma unroll
  for (int bit = 0; bit < 7; ++bit) {
    const bool set = (k >> bit) & 1u;
    const uint32_t b = __ballot_sync(0xFFFFFFFFu, set);
    peers &= set ? b : ~b;
  }
  return peers;
}

// One block of kSortThreads: order[] = block indices sorted by cost,
// costliest first, blocks of equal cost in raster order (a stable counting
// sort, so neighbouring blocks of a bucket still start together).  The
// sample costs come in as 16-byte loads, all of a thread's issued before any
// is used, and each block's cost (the larger of its two samples) is kept in
// shared memory.  Warp w sorts the w-th contiguous run of blocks: per-warp
// bucket counts, one scan over (bucket, warp), then each warp places its run
// 32 blocks at a time, ranking equal buckets inside a step by lane order.
// sample_cost is padded to a multiple of 16 bytes.
__global__ void __launch_bounds__(kSortThreads) block_order_kernel(
    const uint8_t* __restrict__ sample_cost, uint32_t n, uint32_t* __restrict__ order) {
  static_assert(kCostSamples == 2, "a block's cost is the larger of two samples");
  static_assert(kCostCap + 1 < 128, "bucket keys (and the dead-lane key) fit 7 bits");
  constexpr uint32_t kWarps = kSortThreads / 32, kBuckets = kCostCap + 1;
  extern __shared__ __align__(16) uint8_t block_cost[];  // n rounded up to 8 bytes
  __shared__ uint32_t count[kBuckets][kWarps];
  __shared__ uint32_t warp_total[kWarps];
  const uint32_t warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  {  // 16 sample bytes -> 8 block costs per load
    const uint4* src = reinterpret_cast<const uint4*>(sample_cost);
    const uint32_t vecs = (n + 7) / 8;
    constexpr uint32_t kUnroll = 8;
    for (uint32_t base = 0; base < vecs; base += kUnroll * kSortThreads) {
      uint4 v[kUnroll];
#pragma unroll
      for (uint32_t u = 0; u < kUnroll; ++u) {
        const uint32_t q = base + u * kSortThreads + threadIdx.x;
        v[u] = q < vecs ? src[q] : make_uint4(0u, 0u, 0u, 0u);
      }
#pragma unroll
      for (uint32_t u = 0; u < kUnroll; ++u) {
        const uint32_t q = base + u * kSortThreads + threadIdx.x;
        if (q < vecs) {
          // byte 2j of __vmaxu4(w, w >> 8) is max(byte 2j, byte 2j+1) of w
          const uint32_t mx = __vmaxu4(v[u].x, v[u].x >> 8), my = __vmaxu4(v[u].y, v[u].y >> 8);
          const uint32_t mz = __vmaxu4(v[u].z, v[u].z >> 8), mw = __vmaxu4(v[u].w, v[u].w >> 8);
          *reinterpret_cast<uint2*>(block_cost + 8 * q) =
              make_uint2(__byte_perm(mx, my, 0x6420), __byte_perm(mz, mw, 0x6420));
        }
      }
    }
  }
  for (uint32_t k = threadIdx.x; k < kBuckets * kWarps; k += kSortThreads) (&count[0][0])[k] = 0;
  __syncthreads();
  const uint32_t run = (n + kWarps - 1) / kWarps;
  const uint32_t lo = min(warp * run, n), hi = min(lo + run, n);
  for (uint32_t base = lo; base < hi; base += 32) {  // per-warp bucket counts
    const uint32_t i = base + lane;
    const uint32_t k = i < hi ? block_cost[i] : kBuckets;  // kBuckets matches no live lane
    const uint32_t peers = same_key_lanes(k);
    if (i < hi && __popc(peers & ((1u << lane) - 1u)) == 0) count[k][warp] += __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  {  // run starts: exclusive scan over j = (kCostCap - bucket) * kWarps + warp
    constexpr uint32_t kEntries = kBuckets * kWarps;
    constexpr uint32_t kPer = (kEntries + kSortThreads - 1) / kSortThreads;
    auto at = [&](uint32_t j) -> uint32_t& { return count[kCostCap - j / kWarps][j % kWarps]; };
    uint32_t v[kPer], s = 0;
    for (uint32_t q = 0; q < kPer; ++q) {
      const uint32_t j = threadIdx.x * kPer + q;
      v[q] = j < kEntries ? at(j) : 0u;
      s += v[q];
    }
    uint32_t x = s;  // inclusive scan of s over the warp
    for (uint32_t d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
      if (lane >= d) x += y;
    }
    if (lane == 31) warp_total[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = warp_total[lane];
      for (uint32_t d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, d);
        if (lane >= d) w += y;
      }
      warp_total[lane] = w;
    }
    __syncthreads();
    uint32_t pos = x - s + (warp ? warp_total[warp - 1] : 0u);
    for (uint32_t q = 0; q < kPer; ++q) {
      const uint32_t j = threadIdx.x * kPer + q;
      if (j < kEntries) {
        at(j) = pos;
        pos += v[q];
      }
    }
  }
  __syncthreads();
  for (uint32_t base = lo; base < hi; base += 32) {
    const uint32_t i = base + lane;
    const bool live = i < hi;
    const uint32_t k = live ? block_cost[i] : kBuckets;
    const uint32_t peers = same_key_lanes(k);
    const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    if (live) order[count[k][warp] + rank] = i;
    __syncwarp();
    if (live && rank == 0) count[k][warp] += __popc(peers);
    __syncwarp();
  }
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

namespace {

// The scratch of longest-first dispatch (8 bytes per block) comes from a
// memory pool of the library's own, one per device, in stream order: calls
// on different streams get different scratch, and the pool keeps up to 64 MB
// between calls instead of returning it at every synchronisation.
constexpr int kMaxDevices = 64;
cudaMemPool_t g_order_pool[kMaxDevices] = {};
std::mutex g_order_pool_mu;

cudaMemPool_t order_pool() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lock(g_order_pool_mu);
  if (!g_order_pool[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
    uint64_t keep = 64ull << 20;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    g_order_pool[dev] = pool;
  }
  return g_order_pool[dev];
}

// Longest-first order of the frame's blocks into *order (stream-ordered
// scratch the caller frees); false when the frame is small or scratch is not
// available, and the raster launch is used instead.
bool order_blocks(const uint2* nodes, uint64_t num_nodes, const svo_frame_params& p, int S,
                  bool flat, uint32_t gx, uint32_t nblocks, cudaStream_t stream, uint32_t** order) {
  if ((uint64_t)p.width * p.height < kOrderMinPixels || nblocks > kOrderMaxBlocks) return false;
  cudaMemPool_t pool = order_pool();
  if (!pool) {
    cudaGetLastError();
    return false;
  }
  // scratch: order[nblocks] (padded to 16 bytes), then the sample costs
  // (2 bytes a block, padded to whole 16-byte loads of the sort)
  const size_t padded = (nblocks + 7u) & ~7u;
  const size_t order_bytes = padded * sizeof(uint32_t);
  uint32_t* scratch = nullptr;
  if (cudaMallocFromPoolAsync((void**)&scratch, order_bytes + 2 * padded, pool, stream) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  uint8_t* sample_cost = reinterpret_cast<uint8_t*>(scratch) + order_bytes;
  const uint64_t samples = (uint64_t)nblocks * kCostSamples;
  const unsigned grid = (unsigned)((samples + kThreads - 1) / kThreads);
  const size_t smem = render_smem_bytes(S);
  if (flat)
    block_cost_kernel<true><<<grid, kThreads, smem, stream>>>(nodes, num_nodes, p, S, gx, nblocks, sample_cost);
  else
    block_cost_kernel<false><<<grid, kThreads, smem, stream>>>(nodes, num_nodes, p, S, gx, nblocks, sample_cost);
  bool ok = cudaGetLastError() == cudaSuccess;
  if (ok && padded > 48u * 1024u)
    ok = cudaFuncSetAttribute(block_order_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)padded) == cudaSuccess;
  if (ok) {
    block_order_kernel<<<1, kSortThreads, padded, stream>>>(sample_cost, nblocks, scratch);
    ok = cudaGetLastError() == cudaSuccess;
  }
  if (!ok) {
    cudaFreeAsync(scratch, stream);
    cudaGetLastError();
    return false;
  }
  *order = scratch;
  return true;
}

}  // namespace

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
  const uint32_t gx = (p.width + kBlockW - 1) / kBlockW;
  const uint64_t nblocks64 = (uint64_t)gx * ((p.height + kBlockH - 1) / kBlockH);
  uint32_t* order = nullptr;
  if (nblocks64 <= 0x7FFFFFFFull &&
      order_blocks(n2, num_nodes, p, S, flat, gx, (uint32_t)nblocks64, stream, &order)) {
    fn<<<(unsigned)nblocks64, kThreads, smem, stream>>>(n2, a2, num_nodes, p, S, rgba, hits, stats, 0u,
                                                       order, gx);
    const cudaError_t e = cudaGetLastError();
    cudaFreeAsync(order, stream);
    return e == cudaSuccess ? SVO_OK : SVO_ERR_CUDA;
  }
  for (uint32_t y0 = 0; y0 < p.height; y0 += kRowsPerLaunch) {
    const uint32_t rows = p.height - y0 < kRowsPerLaunch ? p.height - y0 : kRowsPerLaunch;
    const dim3 grid(gx, (rows + kBlockH - 1) / kBlockH);
    fn<<<grid, kThreads, smem, stream>>>(n2, a2, num_nodes, p, S, rgba, hits, stats, y0, nullptr, gx);
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
  const uint2* n2 = reinterpret_cast<const uint2*>(nodes);
  const uint2* a2 = reinterpret_cast<const uint2*>(attribs);
  // Raster order: ordering by primary-ray cost made the 3840x2160 shadow
  // frame slower (2.02 against 1.79 ms), the shadow rays' cost being unknown
  // to the estimate and neighbouring blocks no longer sharing the caches.
  const uint32_t gx = (p.width + kBlockW - 1) / kBlockW;
  for (uint32_t y0 = 0; y0 < p.height; y0 += kRowsPerLaunch) {
    const uint32_t rows = p.height - y0 < kRowsPerLaunch ? p.height - y0 : kRowsPerLaunch;
    const dim3 grid(gx, (rows + kBlockH - 1) / kBlockH);
    render_shadow_kernel<<<grid, kThreads, render_smem_bytes(S), stream>>>(
        n2, a2, num_nodes, p, sc, S, rgba, hits, shadow_hits, stats, y0);
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
