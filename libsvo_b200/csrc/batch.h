// batch.h -- device descriptor tables and the launcher of the batch kernel.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "../../include/libsvo_b200.h"

namespace svo {

// One view as the kernel reads it: the frame parameters, its octree, and
// where its tiles start in the batch-wide tile numbering.
struct BatchView {
  svo_frame_params params;
  uint32_t octree;
  uint32_t tiles_x;
  uint64_t tile_begin;
  uint32_t* rgba;
  svo_hit* hits;
};
static_assert(sizeof(BatchView) == 112, "descriptor layout");

struct BatchOctree {
  const uint2* nodes;
  const uint2* attribs;
  uint64_t num_nodes;
  int32_t traversal;
  int32_t stack_size;
};
static_assert(sizeof(BatchOctree) == 32, "descriptor layout");

struct BatchLaunch {
  const BatchView* views = nullptr;
  uint32_t num_views = 0;
  const BatchOctree* octrees = nullptr;
  uint64_t total_tiles = 0;
  unsigned long long* counter = nullptr;
  svo_stats* stats = nullptr;
  int max_s = 13;
  uint32_t top_nodes = 0;
  uint32_t tile_w = 8, tile_h = 4;
  uint32_t rays_per_lane = 1;  // a tile is tile_w x (tile_h * rays_per_lane) pixels
  uint32_t threads = 256, blocks = 0;
  bool ext = false;           // some view uses view mode 2, 6 or 7
  bool treelet_only = false;  // treelet traversal everywhere, nothing staged
};

bool batch_tile_supported(uint32_t tile_w, uint32_t tile_h);
size_t batch_smem_bytes(int max_s, uint32_t threads, uint32_t top_nodes);
// Persistent grid size: blocks_per_sm (0 = as many as fit) times the SM count.
int batch_grid(uint32_t tile_w, uint32_t tile_h, int max_s, uint32_t threads, uint32_t top_nodes,
               uint32_t blocks_per_sm, uint32_t* blocks, bool ext = false,
               bool treelet_only = false);
// Whether a view of the table uses view mode 2, 6 or 7.
bool batch_needs_ext(const BatchView* views, uint32_t num_views);
// Whether every octree takes the treelet traversal and no records are staged
// (the launch then runs the instantiation without the other traversals).
bool batch_treelet_only(const BatchOctree* octrees, uint32_t num_octrees, uint32_t top_nodes);
// Launches the kernel; the caller has zeroed *counter on the same stream.
int launch_batch(const BatchLaunch& launch, cudaStream_t stream);

// Fills `out` (num_views entries) from the caller's view descriptors for
// tiles of tile_w x tile_h pixels; returns the total tile count, or 0 if a
// descriptor is invalid (view modes 0-7 are valid; whether the octree suits
// the mode is check_batch_modes's).
uint64_t layout_views(const svo_view_desc* views, uint32_t num_views, uint32_t num_octrees,
                      uint32_t tile_w, uint32_t tile_h, BatchView* out);
// Per view: attributes present for modes 0, 1 and 6, the treelet traversal
// for modes 6 and 7 (their node centre and quality).
int check_batch_modes(const svo_view_desc* views, uint32_t num_views,
                      const svo_octree_desc* octrees);

}  // namespace svo
