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

// ---- longest-first dispatch ------------------------------------------------
// A frame's blocks differ in cost by two orders of magnitude (rays that graze
// a surface run hundreds of iterations, most rays a dozen), and raster order
// starts some of the longest blocks last, where they run on after the other
// SMs are done.  Large frames therefore estimate each 16x8 block's cost first
// (its two 8x8 cells' centre rays, cut off at kCostCap iterations) and
// append the block to the list of its cost bucket; block r of the frame
// kernel then casts the r-th block of the buckets taken costliest first.
// Every pixel is still cast by the same code: only the order the blocks
// start in changes.  On the 1920x1080 icosphere frame the ordered frame
// kernel takes 254 us against 311 us in raster order, about the 246 us of
// its longest block alone.  The estimate is a chain of dependent node reads
// per ray, so its time grows with the cap, and a low cap ranks the blocks
// worse: frames took 0.2910, 0.2900 and 0.2965 ms with caps 40, 48 and 63.
// The cells' centre rays rank them better than their top-left rays (0.2827
// against 0.2873 ms); four samples a block (one per warp tile) cost more in
// the estimate than they gained (0.297 ms).
constexpr uint32_t kCostCap = 48;
constexpr uint32_t kCostBuckets = kCostCap + 1;
constexpr uint32_t kCostSamples = kBlockW / 8;  // one ray per 8x8 cell of a block
constexpr uint64_t kOrderMinPixels = 1ull << 20;
constexpr uint32_t kOrderMaxBlocks = 1u << 20;
static_assert(kCostSamples == 2, "a block's cost is the larger of two adjacent lanes' samples");
static_assert(kCostBuckets > 32 && kCostBuckets <= 64, "one warp scans the buckets, two per lane");

// count[k]: blocks of estimated cost k; list[k * nblocks + j]: the j-th of
// them.  count == nullptr: raster order.
struct BlockOrder {
  const uint32_t* count;
  const uint32_t* list;
  uint32_t nblocks;
};

// The lanes of the warp whose key equals this lane's, for keys below 128:
// seven ballots, one per key bit.  All 32 lanes take part.
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

// The r-th block in cost order (buckets kCostCap down to 0, each in the
// order its blocks were appended).  Called by one whole warp; every lane
// returns the block.
__device__ __forceinline__ uint32_t ordered_block(const BlockOrder& o, uint32_t r, uint32_t lane) {
  const uint32_t k1 = lane + 32 < kCostBuckets ? kCostCap - 32 - lane : 0u;
  const uint32_t c0 = __ldg(o.count + (kCostCap - lane));
  const uint32_t c1 = lane + 32 < kCostBuckets ? __ldg(o.count + k1) : 0u;
  uint32_t p0 = c0, p1 = c1;  // inclusive prefix sums, bucket kCostCap first
  for (uint32_t d = 1; d < 32; d <<= 1) {
    const uint32_t y0 = __shfl_up_sync(0xFFFFFFFFu, p0, d);
    const uint32_t y1 = __shfl_up_sync(0xFFFFFFFFu, p1, d);
    if (lane >= d) {
      p0 += y0;
      p1 += y1;
    }
  }
  p1 += __shfl_sync(0xFFFFFFFFu, p0, 31);
  uint32_t m = __ballot_sync(0xFFFFFFFFu, p0 > r);
  uint32_t bucket, before;
  if (m != 0u) {
    const int l = __ffs(m) - 1;
    bucket = kCostCap - (uint32_t)l;
    before = __shfl_sync(0xFFFFFFFFu, p0 - c0, l);
  } else {
    m = __ballot_sync(0xFFFFFFFFu, p1 > r);
    if (m == 0u) return r;  // not reached: the buckets hold every block once
    const int l = __ffs(m) - 1;
    bucket = kCostCap - 32 - (uint32_t)l;
    before = __shfl_sync(0xFFFFFFFFu, p1 - c1, l);
  }
  return __ldg(o.list + (uint64_t)bucket * o.nblocks + (r - before));
}

// kExt: view modes 2, 6 and 7 (shade_ext); the other modes compile without
// the extra exit state.  With `order` (1-D grid) block r casts the r-th block
// in estimated-cost order of a frame gx blocks wide; without it the grid is
// the frame's blocks in raster order.
template <bool kFlat, bool kExt>
__global__ void __launch_bounds__(kThreads) render_frame_kernel(
    const uint2* __restrict__ nodes, const uint2* __restrict__ attribs, uint64_t num_nodes,
    const svo_frame_params p, int S, uint32_t* __restrict__ rgba, svo_hit* __restrict__ hits,
    svo_stats* __restrict__ stats, uint32_t y0, const BlockOrder order, uint32_t gx) {
  extern __shared__ uint2 stack_smem[];
  const int t = threadIdx.x;
  const int warp = t >> 5, lane = t & 31;
  uint32_t bx = blockIdx.x, by = blockIdx.y;
  if (order.count != nullptr) {
    __shared__ uint32_t block;
    // launched as a programmatic dependent of the estimate: wait until its
    // bucket lists are complete and visible
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (warp == 0) {
      const uint32_t b = ordered_block(order, blockIdx.x, (uint32_t)lane);
      if (lane == 0) block = b;
    }
    __syncthreads();
    bx = block % gx;
    by = block / gx;
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

// The cost estimate: one thread per sample ray, the two samples of block b
// in lanes 2b and 2b+1 of a warp.  The block's cost (the larger sample,
// capped) picks its bucket, and the block is appended to that bucket's list
// (one atomic per bucket and warp, so neighbouring blocks of a bucket stay
// together).
template <bool kFlat>
__global__ void __launch_bounds__(kThreads) block_cost_kernel(
    const uint2* __restrict__ nodes, uint64_t num_nodes, const svo_frame_params p, int S,
    uint32_t gx, uint32_t nblocks, uint32_t* __restrict__ count, uint32_t* __restrict__ list) {
  extern __shared__ uint2 stack_smem[];
  const uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
  const uint32_t lane = threadIdx.x % 32;
  // the frame kernel may be scheduled once every block of this grid has
  // started (it waits for this grid's completion before reading the lists)
  asm volatile("griddepcontrol.launch_dependents;");
  const bool live = i < (uint64_t)nblocks * kCostSamples;
  const uint32_t b = (uint32_t)(i / kCostSamples), c = (uint32_t)(i % kCostSamples);
  // the cell's centre pixel (pixel 4, 4 of the 8x8 cell; clamped to the
  // frame in cells cut by its edge)
  const uint32_t x0 = (b % gx) * kBlockW + c * 8, y0 = (b / gx) * kBlockH;
  const uint32_t x = min(x0 + 4u, p.width - 1u), y = min(y0 + 4u, p.height - 1u);
  uint32_t loops = 0u;
  if (live && x0 < p.width && y0 < p.height) {
    float o[3], dx, dy, dz;
    pixel_ray(p, x, y, o, dx, dy, dz);
    loops = cast_ray<kFlat>(GlobalFetch{nodes}, num_nodes, o, dx, dy, dz, p.t_scale_ratio, S,
                            stack_smem + threadIdx.x, kThreads, kCostCap)
                .loops;
  }
  const uint32_t cost = min(max(loops, __shfl_xor_sync(0xFFFFFFFFu, loops, 1)), kCostCap);
  const bool appends = live && c == 0;
  const uint32_t peers = same_key_lanes(appends ? cost : kCostBuckets) & 0x55555555u;
  if (appends) {
    const int first = __ffs(peers) - 1;
    uint32_t base = 0u;
    if ((int)lane == first) base = atomicAdd(count + cost, (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, first);
    list[(uint64_t)cost * nblocks + base + __popc(peers & ((1u << lane) - 1u))] = b;
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

// The scratch of longest-first dispatch (196 bytes per block) comes from a
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
// scratch the caller frees with cudaFreeAsync(order->count)); false when the
// frame is small or scratch is not available, and the raster launch is used
// instead.
bool order_blocks(const uint2* nodes, uint64_t num_nodes, const svo_frame_params& p, int S,
                  bool flat, uint32_t gx, uint32_t nblocks, cudaStream_t stream, BlockOrder* order) {
  if ((uint64_t)p.width * p.height < kOrderMinPixels || nblocks > kOrderMaxBlocks) return false;
  cudaMemPool_t pool = order_pool();
  if (!pool) {
    cudaGetLastError();
    return false;
  }
  // scratch: the bucket counts (256 bytes), then the bucket lists
  constexpr size_t kCountBytes = 256;
  static_assert(kCostBuckets * sizeof(uint32_t) <= kCountBytes, "counts fit their header");
  uint32_t* scratch = nullptr;
  const size_t bytes = kCountBytes + (size_t)kCostBuckets * nblocks * sizeof(uint32_t);
  if (cudaMallocFromPoolAsync((void**)&scratch, bytes, pool, stream) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  uint32_t* list = scratch + kCountBytes / sizeof(uint32_t);
  const uint64_t samples = (uint64_t)nblocks * kCostSamples;
  const unsigned grid = (unsigned)((samples + kThreads - 1) / kThreads);
  const size_t smem = render_smem_bytes(S);
  bool ok = cudaMemsetAsync(scratch, 0, kCountBytes, stream) == cudaSuccess;
  if (ok) {
    if (flat)
      block_cost_kernel<true><<<grid, kThreads, smem, stream>>>(nodes, num_nodes, p, S, gx, nblocks, scratch, list);
    else
      block_cost_kernel<false><<<grid, kThreads, smem, stream>>>(nodes, num_nodes, p, S, gx, nblocks, scratch, list);
    ok = cudaGetLastError() == cudaSuccess;
  }
  if (!ok) {
    cudaFreeAsync(scratch, stream);
    cudaGetLastError();
    return false;
  }
  *order = BlockOrder{scratch, list, nblocks};
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
  BlockOrder order{nullptr, nullptr, 0u};
  if (nblocks64 <= 0x7FFFFFFFull &&
      order_blocks(n2, num_nodes, p, S, flat, gx, (uint32_t)nblocks64, stream, &order)) {
    // programmatic dependent launch: the frame kernel's launch and first
    // blocks overlap the estimate's last microseconds (0.5 % on the 1080p frame)
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3((unsigned)nblocks64);
    lc.blockDim = dim3(kThreads);
    lc.dynamicSmemBytes = smem;
    lc.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&lc, fn, n2, a2, num_nodes, p, S, rgba, hits, stats, 0u, order, gx);
    const cudaError_t last = cudaGetLastError();  // clears a launch error
    if (e == cudaSuccess) e = last;
    cudaFreeAsync(const_cast<uint32_t*>(order.count), stream);
    return e == cudaSuccess ? SVO_OK : SVO_ERR_CUDA;
  }
  for (uint32_t y0 = 0; y0 < p.height; y0 += kRowsPerLaunch) {
    const uint32_t rows = p.height - y0 < kRowsPerLaunch ? p.height - y0 : kRowsPerLaunch;
    const dim3 grid(gx, (rows + kBlockH - 1) / kBlockH);
    fn<<<grid, kThreads, smem, stream>>>(n2, a2, num_nodes, p, S, rgba, hits, stats, y0,
                                         BlockOrder{nullptr, nullptr, 0u}, gx);
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
  // One pass in raster order: ordering by primary-ray cost made the
  // 3840x2160 shadow frame slower (2.02 against 1.79 ms), the shadow rays'
  // cost being unknown to the estimate and neighbouring blocks no longer
  // sharing the caches.  Two passes (the primary rays longest first, each
  // hit appended to a job list, then one shadow ray per job in full warps)
  // were slower still: 2.22 against 1.79 ms, and 0.626 against 0.529 ms at
  // 1920x1080, where the shadow pass alone took 330 us for 504 k rays.  A
  // shadow ray cast right after its primary ray finds the nodes of its
  // descent in L1; cast in a later pass it reads them from L2 again.
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
