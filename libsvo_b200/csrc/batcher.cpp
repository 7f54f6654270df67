// batcher.cpp -- host side of the batched ray cast (svo_batcher_* in the C ABI).
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/libsvo_b200.h"
#include "batch.h"
#include "errors.h"

namespace svo {

uint64_t layout_views(const svo_view_desc* views, uint32_t num_views, uint32_t num_octrees,
                      uint32_t tile_w, uint32_t tile_h, BatchView* out) {
  uint64_t tiles = 0;
  for (uint32_t i = 0; i < num_views; ++i) {
    const svo_view_desc& v = views[i];
    const int32_t m = v.params.mode;
    if (v.octree >= num_octrees || !v.d_rgba || v.params.width == 0 || v.params.height == 0)
      return 0;
    if (m < 0 || m > 7) return 0;
    BatchView& b = out[i];
    b.params = v.params;
    b.octree = v.octree;
    b.tiles_x = (v.params.width + tile_w - 1) / tile_w;
    const uint64_t ty = (v.params.height + tile_h - 1) / tile_h;
    b.tile_begin = tiles;
    b.rgba = v.d_rgba;
    b.hits = v.d_hits;
    tiles += (uint64_t)b.tiles_x * ty;
  }
  return tiles;
}

int check_batch_modes(const svo_view_desc* views, uint32_t num_views,
                      const svo_octree_desc* octrees) {
  for (uint32_t i = 0; i < num_views; ++i) {
    const int32_t m = views[i].params.mode;
    const svo_octree_desc& o = octrees[views[i].octree];
    if ((m == 0 || m == 1 || m == 6) && !o.d_attribs) return SVO_ERR_INVALID;
    if ((m == 6 || m == 7) && o.traversal != SVO_TRAVERSAL_TREELET) return SVO_ERR_NOTSUP;
  }
  return SVO_OK;
}

}  // namespace svo

struct svo_batcher {
  uint32_t max_views = 0, max_octrees = 0;
  svo::BatchView* d_views = nullptr;
  svo::BatchOctree* d_octrees = nullptr;
  unsigned long long* d_counter = nullptr;
  svo::BatchView* h_views = nullptr;      // pinned staging
  svo::BatchOctree* h_octrees = nullptr;  // pinned staging
  std::vector<svo_view_desc> views;
  std::vector<svo_octree_desc> octrees;
  svo_batch_cfg cfg{};
  svo::BatchLaunch launch;
  uint64_t rays = 0;
  bool ready = false;
  cudaStream_t capture_stream = nullptr;
  cudaGraphExec_t exec = nullptr;
  svo_stats* exec_stats = nullptr;

  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
  }
  ~svo_batcher() {
    drop_graph();
    if (capture_stream) cudaStreamDestroy(capture_stream);
    cudaFree(d_views);
    cudaFree(d_octrees);
    cudaFree(d_counter);
    cudaFreeHost(h_views);
    cudaFreeHost(h_octrees);
  }
};

namespace {

int check_cfg(const svo_batch_cfg& c) {
  if (!svo::batch_tile_supported(c.tile_w, c.tile_h)) return SVO_ERR_NOTSUP;
  if (c.block_threads < 64 || c.block_threads > 1024 || c.block_threads % 32) return SVO_ERR_RANGE;
  if (c.top_nodes > 16384) return SVO_ERR_RANGE;
  if (c.rays_per_lane != 0 && c.rays_per_lane != 1 && c.rays_per_lane != 2 && c.rays_per_lane != 4)
    return SVO_ERR_RANGE;
  return SVO_OK;
}

// Lays out and uploads the batch for configuration `c`.
int apply(svo_batcher* b, const svo_batch_cfg& c, cudaStream_t stream) {
  int rc = check_cfg(c);
  if (rc != SVO_OK) return rc;
  const uint32_t nv = (uint32_t)b->views.size(), no = (uint32_t)b->octrees.size();
  SVO_CUDA_TRY(cudaStreamSynchronize(stream));  // staging may still feed earlier copies
  const uint32_t rays_per_lane = c.rays_per_lane ? c.rays_per_lane : 1u;
  const uint64_t tiles =
      svo::layout_views(b->views.data(), nv, no, c.tile_w, c.tile_h * rays_per_lane, b->h_views);
  if (tiles == 0) return SVO_ERR_INVALID;
  int max_s = 2;
  for (uint32_t i = 0; i < no; ++i) {
    const svo_octree_desc& o = b->octrees[i];
    if (!o.d_nodes || o.num_nodes == 0 || o.num_nodes > 0x100000000ull) return SVO_ERR_INVALID;
    if (o.traversal != SVO_TRAVERSAL_TREELET && o.traversal != SVO_TRAVERSAL_FLAT) return SVO_ERR_NOTSUP;
    if (o.stack_size < 2 || o.stack_size > 24) return SVO_ERR_RANGE;
    b->h_octrees[i] = svo::BatchOctree{reinterpret_cast<const uint2*>(o.d_nodes),
                                       reinterpret_cast<const uint2*>(o.d_attribs), o.num_nodes,
                                       o.traversal, o.stack_size};
    max_s = std::max(max_s, (int)o.stack_size);
  }
  int mrc = svo::check_batch_modes(b->views.data(), nv, b->octrees.data());
  if (mrc != SVO_OK) return mrc;
  SVO_CUDA_TRY(cudaMemcpyAsync(b->d_views, b->h_views, nv * sizeof(svo::BatchView),
                               cudaMemcpyHostToDevice, stream));
  SVO_CUDA_TRY(cudaMemcpyAsync(b->d_octrees, b->h_octrees, no * sizeof(svo::BatchOctree),
                               cudaMemcpyHostToDevice, stream));
  svo::BatchLaunch L;
  L.views = b->d_views;
  L.num_views = nv;
  L.octrees = b->d_octrees;
  L.total_tiles = tiles;
  L.counter = b->d_counter;
  L.max_s = max_s;
  L.top_nodes = c.top_nodes;
  L.tile_w = c.tile_w;
  L.tile_h = c.tile_h;
  L.rays_per_lane = rays_per_lane;
  L.threads = c.block_threads;
  L.ext = svo::batch_needs_ext(b->h_views, nv);
  L.treelet_only = svo::batch_treelet_only(b->h_octrees, no, c.top_nodes);
  rc = svo::batch_grid(c.tile_w, c.tile_h, max_s, c.block_threads, c.top_nodes, c.blocks_per_sm,
                       &L.blocks, L.ext, L.treelet_only);
  if (rc != SVO_OK) return rc;
  b->launch = L;
  b->cfg = c;
  b->drop_graph();
  b->ready = true;
  return SVO_OK;
}

int launch_plain(svo_batcher* b, svo_stats* stats, cudaStream_t stream) {
  SVO_CUDA_TRY(cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned long long), stream));
  svo::BatchLaunch L = b->launch;
  L.stats = stats;
  return svo::launch_batch(L, stream);
}

}  // namespace

extern "C" {

int svo_batcher_create(uint32_t max_views, uint32_t max_octrees, svo_batcher** out) {
  if (!out || max_views == 0 || max_octrees == 0) return SVO_ERR_INVALID;
  if (max_views > (1u << 20) || max_octrees > 4096) return SVO_ERR_RANGE;
  *out = nullptr;
  svo_batcher* b = new (std::nothrow) svo_batcher;
  if (!b) return SVO_ERR_NOMEM;
  b->max_views = max_views;
  b->max_octrees = max_octrees;
  int rc = SVO_OK;
  if (rc == SVO_OK) rc = svo::cuda_status(cudaMalloc(&b->d_views, max_views * sizeof(svo::BatchView)));
  if (rc == SVO_OK)
    rc = svo::cuda_status(cudaMalloc(&b->d_octrees, max_octrees * sizeof(svo::BatchOctree)));
  if (rc == SVO_OK) rc = svo::cuda_status(cudaMalloc(&b->d_counter, sizeof(unsigned long long)));
  if (rc == SVO_OK)
    rc = svo::cuda_status(cudaMallocHost(&b->h_views, max_views * sizeof(svo::BatchView)));
  if (rc == SVO_OK)
    rc = svo::cuda_status(cudaMallocHost(&b->h_octrees, max_octrees * sizeof(svo::BatchOctree)));
  if (rc == SVO_OK)
    rc = svo::cuda_status(cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking));
  if (rc != SVO_OK) {
    delete b;
    return rc;
  }
  *out = b;
  return SVO_OK;
}

void svo_batcher_destroy(svo_batcher* b) { delete b; }

int svo_batcher_set(svo_batcher* b, const svo_octree_desc* octrees, uint32_t num_octrees,
                    const svo_view_desc* views, uint32_t num_views, const svo_batch_cfg* cfg,
                    void* stream) {
  if (!b || !octrees || !views || !cfg || num_views == 0 || num_octrees == 0) return SVO_ERR_INVALID;
  if (num_views > b->max_views || num_octrees > b->max_octrees) return SVO_ERR_RANGE;
  try {
    b->views.assign(views, views + num_views);
    b->octrees.assign(octrees, octrees + num_octrees);
  } catch (const std::bad_alloc&) {
    return SVO_ERR_NOMEM;
  }
  b->rays = 0;
  for (uint32_t i = 0; i < num_views; ++i)
    b->rays += (uint64_t)views[i].params.width * views[i].params.height;
  b->ready = false;
  return apply(b, *cfg, (cudaStream_t)stream);
}

int svo_batcher_launch(svo_batcher* b, svo_stats* d_stats, void* stream) {
  if (!b || !b->ready) return SVO_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  if (!b->cfg.use_graph) return launch_plain(b, d_stats, s);
  if (!b->exec || b->exec_stats != d_stats) {
    b->drop_graph();
    SVO_CUDA_TRY(cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal));
    const int rc = launch_plain(b, d_stats, b->capture_stream);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->capture_stream, &graph);
    if (rc != SVO_OK) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    SVO_CUDA_TRY(e);
    const cudaError_t ie = cudaGraphInstantiate(&b->exec, graph, 0);
    cudaGraphDestroy(graph);
    SVO_CUDA_TRY(ie);
    b->exec_stats = d_stats;
  }
  SVO_CUDA_TRY(cudaGraphLaunch(b->exec, s));
  return SVO_OK;
}

int svo_batcher_autotune(svo_batcher* b, uint32_t reps, void* stream, svo_batch_cfg* best,
                         float* best_ms) {
  if (!b || !b->ready) return SVO_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  reps = std::max<uint32_t>(1, reps);
  static const uint32_t shapes[][2] = {{8, 4}, {16, 2}, {4, 8}, {32, 1}};
  static const uint32_t threads[] = {128, 256, 512};
  static const uint32_t tops[] = {0, 1024};
  static const uint32_t rays[] = {1, 2, 4};
  const svo_batch_cfg base = b->cfg;
  svo_batch_cfg win = base;
  float win_ms = 1e30f;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  SVO_CUDA_TRY(cudaEventCreate(&e0));
  SVO_CUDA_TRY(cudaEventCreate(&e1));
  int rc = SVO_OK;
  std::vector<svo_batch_cfg> cands;
  for (const auto& sh : shapes)
    for (uint32_t t : threads)
      for (uint32_t top : tops)
        for (uint32_t rpl : rays) {
          svo_batch_cfg c = base;
          c.tile_w = sh[0];
          c.tile_h = sh[1];
          c.block_threads = t;
          c.top_nodes = top;
          c.rays_per_lane = rpl;
          c.use_graph = 0;
          cands.push_back(c);
        }
  for (const svo_batch_cfg& c : cands) {
    if (apply(b, c, s) != SVO_OK) continue;  // e.g. does not fit in shared memory
    rc = launch_plain(b, nullptr, s);  // warm-up
    if (rc != SVO_OK) break;
    rc = svo::cuda_status(cudaEventRecord(e0, s));
    for (uint32_t r = 0; r < reps && rc == SVO_OK; ++r) rc = launch_plain(b, nullptr, s);
    if (rc == SVO_OK) rc = svo::cuda_status(cudaEventRecord(e1, s));
    if (rc == SVO_OK) rc = svo::cuda_status(cudaEventSynchronize(e1));
    float ms = 0.0f;
    if (rc == SVO_OK) rc = svo::cuda_status(cudaEventElapsedTime(&ms, e0, e1));
    if (rc != SVO_OK) break;
    ms /= (float)reps;
    if (ms < win_ms) {
      win_ms = ms;
      win = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != SVO_OK) return rc;
  if (win_ms >= 1e30f) return SVO_ERR_NOTSUP;
  win.use_graph = base.use_graph;
  rc = apply(b, win, s);
  if (rc != SVO_OK) return rc;
  if (best) *best = win;
  if (best_ms) *best_ms = win_ms;
  return SVO_OK;
}

int svo_batcher_size(svo_batcher* b, uint64_t* tiles, uint64_t* rays) {
  if (!b || !b->ready) return SVO_ERR_INVALID;
  if (tiles) *tiles = b->launch.total_tiles;
  if (rays) *rays = b->rays;
  return SVO_OK;
}

}  // extern "C"
