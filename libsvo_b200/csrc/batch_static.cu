// batch_static.cu -- the batched ray cast without any allocation.
//
// Some callers cannot let a library allocate device memory: a host
// application (an engine, a serving process) that owns and budgets every
// byte of HBM through its own allocator and hands its plugins only fixed
// buffers, or a latency-critical frame loop where cudaMalloc/cudaFree could
// synchronise the device and stall.  svo_render_batch_static serves them: it
// runs the same batch kernel as svo_batcher_launch, but its scratch -- the
// view and octree descriptor tables and the tile counter -- lives in the
// fixed array below, which every GPU that loads this library holds from load
// to process exit.  The caller still passes the octree pools and the output
// buffers.
//
// Limits: at most kStaticMaxViews views and kStaticMaxOctrees octrees per
// call (SVO_ERR_RANGE beyond that).  Every call uses the same array, and it
// keeps the last call's contents: each call rewrites the tables and zeroes
// the counter before its launch, and calls whose work overlaps on the GPU
// (other streams or host threads) race on the array.
//
// The tables reach the array as the parameter of a small loader kernel
// (passed by value, so no host memory is read after the call returns), and
// the batch kernel launched right after it on the same stream reads them.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "../../include/libsvo_b200.h"
#include "batch.h"
#include "errors.h"

namespace svo {
namespace {

constexpr uint32_t kStaticMaxViews = 256;
constexpr uint32_t kStaticMaxOctrees = 16;
constexpr size_t kCounterBytes = 256;  // tile counter, padded to keep the tables aligned
constexpr size_t kOctreeOffset = kCounterBytes;
constexpr size_t kViewOffset = kOctreeOffset + kStaticMaxOctrees * sizeof(BatchOctree);
constexpr size_t kScratchBytes = kViewOffset + kStaticMaxViews * sizeof(BatchView);
static_assert(kViewOffset % 16 == 0, "descriptor alignment");

// The scratch array (29,440 bytes).  In host code this name is only a
// stand-in for the symbol; its device address comes from
// cudaGetSymbolAddress, looked up once per device.
static __device__ __align__(256) unsigned char g_batch_scratch[kScratchBytes];

// The call's descriptor tables, passed to the loader kernel by value
// (29,192 bytes, within the 32,764-byte kernel-parameter limit).
struct StaticTables {
  BatchOctree octrees[kStaticMaxOctrees];
  BatchView views[kStaticMaxViews];
  uint32_t num_octrees;
  uint32_t num_views;
};
static_assert(sizeof(StaticTables) <= 32764, "kernel parameter limit");

// Copies the used part of the tables into the scratch array and zeroes the
// tile counter; one block.
__global__ void load_static_tables(const __grid_constant__ StaticTables t, unsigned char* scratch) {
  const uint32_t* oct = reinterpret_cast<const uint32_t*>(t.octrees);
  const uint32_t* view = reinterpret_cast<const uint32_t*>(t.views);
  uint32_t* d_oct = reinterpret_cast<uint32_t*>(scratch + kOctreeOffset);
  uint32_t* d_view = reinterpret_cast<uint32_t*>(scratch + kViewOffset);
  const uint32_t oct_words = t.num_octrees * (uint32_t)(sizeof(BatchOctree) / 4);
  const uint32_t view_words = t.num_views * (uint32_t)(sizeof(BatchView) / 4);
  for (uint32_t i = threadIdx.x; i < oct_words; i += blockDim.x) d_oct[i] = oct[i];
  for (uint32_t i = threadIdx.x; i < view_words; i += blockDim.x) d_view[i] = view[i];
  if (threadIdx.x == 0) *reinterpret_cast<unsigned long long*>(scratch) = 0ull;
}

constexpr int kMaxDevices = 64;
void* g_scratch_address[kMaxDevices] = {};
std::mutex g_scratch_mutex;

// Device address of g_batch_scratch on the current device.  The first call
// on a device does the lookup with that device current and keeps it for the
// life of the process (a cudaDeviceReset would move the array; the library
// is not used across one).
int scratch_address(unsigned char** out) {
  int dev = 0;
  SVO_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return SVO_ERR_RANGE;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_address[dev]) {
    void* p = nullptr;
    SVO_CUDA_TRY(cudaGetSymbolAddress(&p, g_batch_scratch));
    if (!p) return SVO_ERR_CUDA;
    g_scratch_address[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_scratch_address[dev]);
  return SVO_OK;
}

}  // namespace
}  // namespace svo

extern "C" int svo_render_batch_static(const svo_octree_desc* octrees, uint32_t num_octrees,
                                       const svo_view_desc* views, uint32_t num_views,
                                       uint32_t tile_w, uint32_t tile_h, svo_stats* d_stats,
                                       void* stream) {
  using namespace svo;
  if (!octrees || !views || num_views == 0 || num_octrees == 0) return SVO_ERR_INVALID;
  if (num_views > kStaticMaxViews || num_octrees > kStaticMaxOctrees) return SVO_ERR_RANGE;
  if (!batch_tile_supported(tile_w, tile_h)) return SVO_ERR_NOTSUP;
  // the tables are built in a host-stack struct and handed to the loader
  // kernel by value: nothing is allocated
  StaticTables tables;
  tables.num_octrees = num_octrees;
  tables.num_views = num_views;
  BatchView* host_views = tables.views;
  BatchOctree* host_octrees = tables.octrees;
  const uint64_t tiles = layout_views(views, num_views, num_octrees, tile_w, tile_h, host_views);
  if (tiles == 0) return SVO_ERR_INVALID;
  int max_s = 2;
  for (uint32_t i = 0; i < num_octrees; ++i) {
    const svo_octree_desc& o = octrees[i];
    if (!o.d_nodes || o.num_nodes == 0 || o.num_nodes > 0x100000000ull) return SVO_ERR_INVALID;
    if (o.traversal != SVO_TRAVERSAL_TREELET && o.traversal != SVO_TRAVERSAL_FLAT) return SVO_ERR_NOTSUP;
    if (o.stack_size < 2 || o.stack_size > 24) return SVO_ERR_RANGE;
    host_octrees[i] = BatchOctree{reinterpret_cast<const uint2*>(o.d_nodes),
                                  reinterpret_cast<const uint2*>(o.d_attribs), o.num_nodes,
                                  o.traversal, o.stack_size};
    max_s = std::max(max_s, (int)o.stack_size);
  }
  const int mrc = check_batch_modes(views, num_views, octrees);
  if (mrc != SVO_OK) return mrc;
  unsigned char* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc != SVO_OK) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  load_static_tables<<<1, 256, 0, s>>>(tables, scratch);
  SVO_CUDA_TRY(cudaGetLastError());
  BatchLaunch L;
  L.views = reinterpret_cast<const BatchView*>(scratch + kViewOffset);
  L.num_views = num_views;
  L.octrees = reinterpret_cast<const BatchOctree*>(scratch + kOctreeOffset);
  L.total_tiles = tiles;
  L.counter = reinterpret_cast<unsigned long long*>(scratch);
  L.stats = d_stats;
  L.max_s = max_s;
  L.top_nodes = 0;
  L.tile_w = tile_w;
  L.tile_h = tile_h;
  L.threads = 256;
  L.ext = batch_needs_ext(host_views, num_views);
  L.treelet_only = batch_treelet_only(host_octrees, num_octrees, 0);
  rc = batch_grid(tile_w, tile_h, max_s, L.threads, 0, 0, &L.blocks, L.ext, L.treelet_only);
  if (rc != SVO_OK) return rc;
  return launch_batch(L, s);
}
