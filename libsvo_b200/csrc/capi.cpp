// capi.cpp -- the extern "C" boundary declared in include/libsvo_b200.h.
//
// Every entry point validates its arguments, turns C++ exceptions (allocation
// failures) into status codes, and never terminates the process.
#include <algorithm>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>
#include <thread>
#include <atomic>

#include "../../include/libsvo_b200.h"
#include "errors.h"
#include "feedback.h"
#include "gpu_builder.h"
#include "memory_manager.h"
#include "render.h"
#include "scene.h"

struct svo_mm {
  explicit svo_mm(cudaStream_t s) : impl(s) {}
  svo::TreeletMemoryManagerCuda impl;
};

namespace svo {
namespace {
thread_local std::string g_last_error;
}
void set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }
const char* last_error() { return g_last_error.c_str(); }
}  // namespace svo

namespace {

template <class Fn>
int guarded(Fn&& fn) {
  try {
    return fn();
  } catch (const std::bad_alloc&) {
    return SVO_ERR_NOMEM;
  } catch (...) {
    return SVO_ERR_INVALID;
  }
}

int check_cfg(const svo_trace_cfg* cfg) {
  if (!cfg) return SVO_ERR_INVALID;
  if (cfg->traversal != SVO_TRAVERSAL_TREELET && cfg->traversal != SVO_TRAVERSAL_FLAT)
    return SVO_ERR_NOTSUP;
  if (cfg->stack_size < 2 || cfg->stack_size > 24) return SVO_ERR_RANGE;
  return SVO_OK;
}

int check_mode(int32_t mode) {
  return (mode == 0 || mode == 1 || mode == 3 || mode == 4 || mode == 5) ? SVO_OK : SVO_ERR_NOTSUP;
}

// The per-frame kernel also shades modes 2, 6 and 7; 6 and 7 need the node
// centre and quality that only the treelet traversal reports.
int check_frame_mode(int32_t mode, int32_t traversal) {
  if (mode == 2) return SVO_OK;
  if (mode == 6 || mode == 7) return traversal == SVO_TRAVERSAL_TREELET ? SVO_OK : SVO_ERR_NOTSUP;
  return check_mode(mode);
}

int build_scene(uint32_t depth, std::vector<uint64_t>& codes, std::vector<svo_attrib>& attribs,
                uint32_t treelet_levels, uint32_t treelet_bytes, svo_scene** out) {
  svo::Octree tree;
  int rc = svo::octree_from_leaves(depth, std::move(codes), std::move(attribs), tree);
  if (rc != SVO_OK) return rc;
  std::unique_ptr<svo_scene> s(new svo_scene);
  rc = svo::cut_treelets(tree, treelet_levels, treelet_bytes, *s);
  if (rc != SVO_OK) return rc;
  *out = s.release();
  return SVO_OK;
}

// Copies analysis lists to caller arrays (svo_mm_analyse_feedback*).
int export_lists(int rc, const std::vector<std::pair<int32_t, float>>& nw,
                 const std::vector<std::pair<int32_t, float>>& old, int32_t* new_gids,
                 float* new_errors, uint32_t new_capacity, uint32_t* num_new, int32_t* old_gids,
                 float* old_errors, uint32_t old_capacity, uint32_t* num_old) {
  if (num_new) *num_new = (uint32_t)nw.size();
  if (num_old) *num_old = (uint32_t)old.size();
  if (rc != SVO_OK) return rc;
  if ((new_gids || new_errors) && nw.size() > new_capacity) return SVO_ERR_RANGE;
  if ((old_gids || old_errors) && old.size() > old_capacity) return SVO_ERR_RANGE;
  for (size_t i = 0; i < nw.size(); ++i) {
    if (new_gids) new_gids[i] = nw[i].first;
    if (new_errors) new_errors[i] = nw[i].second;
  }
  for (size_t i = 0; i < old.size(); ++i) {
    if (old_gids) old_gids[i] = old[i].first;
    if (old_errors) old_errors[i] = old[i].second;
  }
  return SVO_OK;
}

}  // namespace

extern "C" {

const char* svo_version(void) { return "libsvo_b200 0.1"; }
const char* svo_last_error(void) { return svo::last_error(); }

// ---- scenes ---------------------------------------------------------------

int svo_scene_build_menger(uint32_t level, uint32_t depth, uint64_t seed, uint32_t treelet_levels,
                           uint32_t treelet_bytes, svo_scene** out) {
  if (!out) return SVO_ERR_INVALID;
  *out = nullptr;
  return guarded([&] {
    std::vector<uint64_t> codes;
    std::vector<svo_attrib> attribs;
    int rc = svo::build_menger(level, depth, seed, codes, attribs);
    if (rc != SVO_OK) return rc;
    return build_scene(depth, codes, attribs, treelet_levels, treelet_bytes, out);
  });
}

int svo_scene_build_mesh_attributed(const float* h_vertices, const float* h_normals,
                                    const float* h_colors, uint64_t num_vertices,
                                    const uint32_t* h_triangles, uint64_t num_triangles,
                                    uint32_t depth, uint32_t treelet_levels,
                                    uint32_t treelet_bytes, int32_t threads, svo_scene** out) {
  if (!out || !h_vertices || !h_triangles) return SVO_ERR_INVALID;
  *out = nullptr;
  return guarded([&] {
    std::vector<uint64_t> codes;
    std::vector<svo_attrib> attribs;
    int rc = svo::build_mesh_leaves(h_vertices, h_normals, h_colors, num_vertices, h_triangles,
                                    num_triangles, depth, threads, codes, attribs);
    if (rc != SVO_OK) return rc;
    return build_scene(depth, codes, attribs, treelet_levels, treelet_bytes, out);
  });
}

int svo_scene_build_mesh(const float* h_vertices, uint64_t num_vertices,
                         const uint32_t* h_triangles, uint64_t num_triangles, uint32_t depth,
                         uint32_t treelet_levels, uint32_t treelet_bytes, int32_t threads,
                         svo_scene** out) {
  return svo_scene_build_mesh_attributed(h_vertices, nullptr, nullptr, num_vertices, h_triangles,
                                         num_triangles, depth, treelet_levels, treelet_bytes,
                                         threads, out);
}

struct svo_device_scene {
  svo::DeviceScene impl;
};

int svo_device_scene_build_mesh_attributed(const float* h_vertices, const float* h_normals,
                                           const float* h_colors, uint64_t num_vertices,
                                           const uint32_t* h_triangles, uint64_t num_triangles,
                                           uint32_t depth, uint32_t treelet_levels, void* stream,
                                           svo_device_scene** out) {
  if (!out || !h_vertices || !h_triangles) return SVO_ERR_INVALID;
  if ((h_normals == nullptr) != (h_colors == nullptr)) return SVO_ERR_INVALID;
  *out = nullptr;
  return guarded([&] {
    std::unique_ptr<svo_device_scene> s(new svo_device_scene);
    const int rc = s->impl.build_mesh(h_vertices, h_normals, h_colors, num_vertices, h_triangles,
                                      num_triangles, depth, treelet_levels, (cudaStream_t)stream);
    if (rc != SVO_OK) return rc;
    *out = s.release();
    return SVO_OK;
  });
}

int svo_device_scene_build_mesh(const float* h_vertices, uint64_t num_vertices,
                                const uint32_t* h_triangles, uint64_t num_triangles,
                                uint32_t depth, uint32_t treelet_levels, void* stream,
                                svo_device_scene** out) {
  return svo_device_scene_build_mesh_attributed(h_vertices, nullptr, nullptr, num_vertices,
                                                h_triangles, num_triangles, depth, treelet_levels,
                                                stream, out);
}

int svo_device_scene_info_get(const svo_device_scene* scene, svo_scene_info* out) {
  if (!scene || !out) return SVO_ERR_INVALID;
  const svo::DeviceScene& d = scene->impl;
  out->num_treelets = d.num_treelets;
  out->treelet_bytes = (uint32_t)(d.nodes_per_slot * 8);
  out->nodes_per_treelet = (uint32_t)d.nodes_per_slot;
  out->max_depth = d.depth;
  out->total_nodes = d.treelet_nodes;
  out->leaf_voxels = d.leaf_voxels;
  return SVO_OK;
}

int svo_device_scene_buffers(const svo_device_scene* scene, const svo_node** d_nodes,
                             const svo_attrib** d_attribs, uint64_t* num_nodes) {
  if (!scene) return SVO_ERR_INVALID;
  if (d_nodes) *d_nodes = scene->impl.d_nodes;
  if (d_attribs) *d_attribs = scene->impl.d_attribs;
  if (num_nodes) *num_nodes = scene->impl.pool_nodes;
  return SVO_OK;
}

int svo_device_scene_copy(const svo_device_scene* scene, uint64_t first, uint64_t count,
                          svo_node* h_nodes, svo_attrib* h_attribs) {
  if (!scene) return SVO_ERR_INVALID;
  const svo::DeviceScene& d = scene->impl;
  if (first > d.pool_nodes || count > d.pool_nodes - first) return SVO_ERR_RANGE;
  if (count == 0) return SVO_OK;
  if (h_nodes)
    SVO_CUDA_TRY(cudaMemcpy(h_nodes, d.d_nodes + first, count * sizeof(svo_node),
                            cudaMemcpyDeviceToHost));
  if (h_attribs)
    SVO_CUDA_TRY(cudaMemcpy(h_attribs, d.d_attribs + first, count * sizeof(svo_attrib),
                            cudaMemcpyDeviceToHost));
  return SVO_OK;
}

int svo_device_scene_counts(const svo_device_scene* scene, uint64_t* octree_nodes,
                            uint64_t* overlaps) {
  if (!scene) return SVO_ERR_INVALID;
  if (octree_nodes) *octree_nodes = scene->impl.octree_nodes;
  if (overlaps) *overlaps = scene->impl.pairs;
  return SVO_OK;
}

void svo_device_scene_destroy(svo_device_scene* scene) { delete scene; }

int svo_scene_from_pool(const svo_node* h_nodes, const svo_attrib* h_attribs, uint32_t num_slots,
                        uint32_t treelet_bytes, uint32_t max_depth, uint64_t leaf_voxels,
                        svo_scene** out) {
  if (!out || !h_nodes || !h_attribs) return SVO_ERR_INVALID;
  *out = nullptr;
  return guarded([&] {
    std::unique_ptr<svo_scene> s(new svo_scene);
    const int rc = svo::scene_from_pool(h_nodes, h_attribs, num_slots, treelet_bytes, max_depth,
                                        leaf_voxels, *s);
    if (rc != SVO_OK) return rc;
    *out = s.release();
    return SVO_OK;
  });
}

int svo_mm_create_from_device_scene(const svo_device_scene* scene, uint64_t incore_bytes, void* stream,
                                    svo_mm** out) {
  if (!out || !scene) return SVO_ERR_INVALID;
  *out = nullptr;
  return guarded([&] {
    const svo::DeviceScene& d = scene->impl;
    const uint64_t N = d.nodes_per_slot;
    svo_scene s;
    s.treelet_bytes = (uint32_t)(N * 8);
    s.max_depth = d.depth;
    s.leaf_voxels = d.leaf_voxels;
    s.treelets.resize(d.num_treelets);
    // the pool comes to the host in pieces of about 256 MB and is turned into
    // treelets piece by piece: the host never holds a second copy of it
    const uint64_t per = std::max<uint64_t>(1, (256ull << 20) / (N * sizeof(svo_node)));
    std::vector<svo_node> hn(per * N);
    std::vector<svo_attrib> ha(per * N);
    cudaStream_t st = (cudaStream_t)stream;
    for (uint64_t g0 = 0; g0 < d.num_treelets; g0 += per) {
      const uint64_t k = std::min<uint64_t>(per, d.num_treelets - g0);
      SVO_CUDA_TRY(cudaMemcpyAsync(hn.data(), d.d_nodes + g0 * N, k * N * sizeof(svo_node),
                                   cudaMemcpyDeviceToHost, st));
      SVO_CUDA_TRY(cudaMemcpyAsync(ha.data(), d.d_attribs + g0 * N, k * N * sizeof(svo_attrib),
                                   cudaMemcpyDeviceToHost, st));
      SVO_CUDA_TRY(cudaStreamSynchronize(st));
      // slots are independent (a slot writes its own treelet and the headers
      // of its sub-treelets, each of which has one parent): host threads
      // take them in turn
      std::atomic<uint64_t> next{0};
      std::atomic<int> status{SVO_OK};
      auto work = [&] {
        for (uint64_t i = next.fetch_add(1); i < k; i = next.fetch_add(1)) {
          const int rc = svo::unpatch_slot((uint32_t)(g0 + i), N, d.num_treelets, hn.data() + i * N,
                                           ha.data() + i * N, s);
          if (rc != SVO_OK) status.store(rc);
        }
      };
      const unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
      std::vector<std::thread> pool;
      for (unsigned t = 1; t < nt; ++t) pool.emplace_back(work);
      work();
      for (auto& th : pool) th.join();
      if (status.load() != SVO_OK) return status.load();
    }
    std::unique_ptr<svo_mm> mm(new svo_mm(st));
    const int rc = mm->impl.init(std::move(s), incore_bytes);
    if (rc != SVO_OK) return rc;
    *out = mm.release();
    return SVO_OK;
  });
}

int svo_scene_write(const svo_scene* scene, const char* path_base) {
  if (!scene || !path_base) return SVO_ERR_INVALID;
  return guarded([&] { return svo::write_scene(*scene, path_base); });
}

int svo_scene_read(const char* path_base, svo_scene** out) {
  if (!out || !path_base) return SVO_ERR_INVALID;
  *out = nullptr;
  return guarded([&] {
    std::unique_ptr<svo_scene> s(new svo_scene);
    const int rc = svo::read_scene(path_base, *s);
    if (rc != SVO_OK) return rc;
    *out = s.release();
    return SVO_OK;
  });
}

int svo_scene_info_get(const svo_scene* scene, svo_scene_info* out) {
  if (!scene || !out) return SVO_ERR_INVALID;
  out->num_treelets = (uint32_t)scene->treelets.size();
  out->treelet_bytes = scene->treelet_bytes;
  out->nodes_per_treelet = scene->treelet_bytes / 8;
  out->max_depth = scene->max_depth;
  uint64_t total = 0;
  for (const auto& t : scene->treelets) total += t.num_nodes;
  out->total_nodes = total;
  out->leaf_voxels = scene->leaf_voxels;
  return SVO_OK;
}

int svo_scene_treelet(const svo_scene* scene, uint32_t gid, uint32_t* num_nodes,
                      uint32_t* num_leaves, int32_t* parent_gid, int32_t* parent_leaf_position,
                      int32_t* parent_leaf_idx, int32_t* parent_leaf_parent_position) {
  if (!scene || gid >= scene->treelets.size()) return SVO_ERR_INVALID;
  const auto& t = scene->treelets[gid];
  if (num_nodes) *num_nodes = t.num_nodes;
  if (num_leaves) *num_leaves = t.num_leaves;
  if (parent_gid) *parent_gid = t.parent_gid;
  if (parent_leaf_position) *parent_leaf_position = t.parent_leaf_position;
  if (parent_leaf_idx) *parent_leaf_idx = t.parent_leaf_idx;
  if (parent_leaf_parent_position) *parent_leaf_parent_position = t.parent_leaf_parent_position;
  return SVO_OK;
}

int svo_scene_flatten(const svo_scene* scene, svo_node* h_nodes, svo_attrib* h_attribs,
                      uint64_t capacity, uint64_t* num_nodes) {
  if (!scene) return SVO_ERR_INVALID;
  return guarded([&] {
    const bool want = h_nodes || h_attribs;
    std::vector<svo_node> nodes;
    std::vector<svo_attrib> attribs;
    uint64_t n = 0;
    const int rc = svo::flatten_scene(*scene, want ? &nodes : nullptr, want ? &attribs : nullptr, &n);
    if (rc != SVO_OK) return rc;
    if (num_nodes) *num_nodes = n;
    if (!want) return SVO_OK;
    if (capacity < n) return SVO_ERR_RANGE;
    if (h_nodes) std::memcpy(h_nodes, nodes.data(), n * sizeof(svo_node));
    if (h_attribs) std::memcpy(h_attribs, attribs.data(), n * sizeof(svo_attrib));
    return SVO_OK;
  });
}

void svo_scene_destroy(svo_scene* scene) { delete scene; }

// ---- memory manager -------------------------------------------------------

int svo_mm_create_from_scene(const svo_scene* scene, uint64_t incore_bytes, void* stream,
                             svo_mm** out) {
  if (!out || !scene) return SVO_ERR_INVALID;
  *out = nullptr;
  return guarded([&] {
    svo_scene copy = *scene;
    std::unique_ptr<svo_mm> mm(new svo_mm((cudaStream_t)stream));
    const int rc = mm->impl.init(std::move(copy), incore_bytes);
    if (rc != SVO_OK) return rc;
    *out = mm.release();
    return SVO_OK;
  });
}

int svo_mm_create(const char* svo_path_base, uint64_t incore_bytes, void* stream, svo_mm** out) {
  if (!out || !svo_path_base) return SVO_ERR_INVALID;
  *out = nullptr;
  return guarded([&] {
    svo_scene s;
    int rc = svo::read_scene(svo_path_base, s);
    if (rc != SVO_OK) return rc;
    std::unique_ptr<svo_mm> mm(new svo_mm((cudaStream_t)stream));
    rc = mm->impl.init(std::move(s), incore_bytes);
    if (rc != SVO_OK) return rc;
    *out = mm.release();
    return SVO_OK;
  });
}

void svo_mm_destroy(svo_mm* mm) { delete mm; }

int svo_mm_init_device_buffer(svo_mm* mm) {
  if (!mm) return SVO_ERR_INVALID;
  return guarded([&] { return mm->impl.init_device_buffer(); });
}

int svo_mm_get_device_buffers(svo_mm* mm, const svo_node** d_nodes, const svo_attrib** d_attribs,
                              uint64_t* num_nodes) {
  if (!mm || !mm->impl.device_ready()) return SVO_ERR_INVALID;
  if (d_nodes) *d_nodes = mm->impl.device_nodes();
  if (d_attribs) *d_attribs = mm->impl.device_attribs();
  if (num_nodes) *num_nodes = mm->impl.incore_nodes();
  return SVO_OK;
}

int svo_mm_insert_treelet(svo_mm* mm, int32_t treelet_gid, int32_t visibility, float error) {
  if (!mm) return SVO_ERR_INVALID;
  if (mm->impl.analysis_pending()) return SVO_ERR_BUSY;  // between _begin and _end
  return guarded([&] {
    svo::TreeletMemoryManager::SlotInfo s;
    s.treelet_gid = treelet_gid;
    s.visibility = visibility;
    s.error = error;
    return mm->impl.insert_treelet(s);
  });
}

int svo_mm_remove_treelet(svo_mm* mm, int32_t treelet_gid) {
  if (!mm) return SVO_ERR_INVALID;
  if (mm->impl.analysis_pending()) return SVO_ERR_BUSY;  // between _begin and _end
  return guarded([&] { return mm->impl.remove_treelet(treelet_gid); });
}

int svo_mm_free_incore_position(svo_mm* mm) {
  if (!mm) return SVO_ERR_INVALID;
  if (mm->impl.analysis_pending()) return SVO_ERR_BUSY;  // between _begin and _end
  return guarded([&] { return mm->impl.free_incore_position(); });
}

int svo_mm_update_client_side(svo_mm* mm, const int32_t* new_gids, const float* new_errors,
                              uint32_t num_new, const int32_t* old_gids, uint32_t num_old) {
  if (!mm || (num_new && !new_gids) || (num_old && !old_gids)) return SVO_ERR_INVALID;
  if (mm->impl.analysis_pending()) return SVO_ERR_BUSY;  // between _begin and _end
  return guarded([&] {
    return mm->impl.update_client_side(new_gids, new_errors, num_new, old_gids, num_old);
  });
}

int svo_mm_set_upload_policy(svo_mm* mm, int32_t policy) {
  if (!mm) return SVO_ERR_INVALID;
  return mm->impl.set_upload_policy(policy);
}

int svo_mm_set_upload_ratio(svo_mm* mm, float ratio) {
  if (!mm) return SVO_ERR_INVALID;
  return mm->impl.set_upload_ratio(ratio);
}

int svo_mm_update_device_memory(svo_mm* mm, uint32_t* num_copy_calls) {
  if (!mm) return SVO_ERR_INVALID;
  if (mm->impl.analysis_pending()) return SVO_ERR_BUSY;  // between _begin and _end
  return guarded([&] { return mm->impl.update_device_memory(num_copy_calls); });
}

int svo_mm_plan_uploads(svo_mm* mm, uint32_t* h_first_slots, uint32_t* h_slot_counts,
                        uint32_t capacity, uint32_t* num_ranges) {
  if (!mm) return SVO_ERR_INVALID;
  return guarded([&] {
    const auto r = mm->impl.upload_ranges();
    if (num_ranges) *num_ranges = (uint32_t)r.size();
    if (!h_first_slots && !h_slot_counts) return SVO_OK;
    if (capacity < r.size()) return SVO_ERR_RANGE;
    for (size_t i = 0; i < r.size(); ++i) {
      if (h_first_slots) h_first_slots[i] = r[i].first;
      if (h_slot_counts) h_slot_counts[i] = r[i].second;
    }
    return SVO_OK;
  });
}

int svo_mm_reset(svo_mm* mm) {
  if (!mm) return SVO_ERR_INVALID;
  if (mm->impl.analysis_pending()) return SVO_ERR_BUSY;  // between _begin and _end
  return guarded([&] { return mm->impl.reset_incore_buffer(); });
}

int svo_mm_insert_all(svo_mm* mm, uint32_t* num_inserted) {
  if (!mm) return SVO_ERR_INVALID;
  if (mm->impl.analysis_pending()) return SVO_ERR_BUSY;  // between _begin and _end
  return guarded([&] { return mm->impl.insert_all(num_inserted); });
}

int svo_mm_info_get(svo_mm* mm, svo_mm_info* out) {
  if (!mm || !out) return SVO_ERR_INVALID;
  const auto& m = mm->impl;
  out->num_treelets = m.num_treelets();
  out->treelet_bytes = m.treelet_bytes();
  out->nodes_per_treelet = m.nodes_per_treelet();
  out->num_slots = m.num_slots();
  out->free_slots = m.free_slots();
  out->slots_to_upload = (uint32_t)m.slots_to_upload().size();
  out->incore_nodes = m.incore_nodes();
  out->device_bytes = m.device_bytes();
  return SVO_OK;
}

int svo_mm_get_slot(svo_mm* mm, uint32_t slot, svo_slot_info* out) {
  if (!mm || !out || slot >= mm->impl.num_slots()) return SVO_ERR_INVALID;
  const auto& s = mm->impl.slot(slot);
  out->treelet_gid = s.treelet_gid;
  out->visibility = s.visibility;
  out->error = s.error;
  return SVO_OK;
}

int svo_mm_treelet_slot(svo_mm* mm, int32_t treelet_gid, int32_t* slot) {
  if (!mm || !slot || treelet_gid < 0 || (uint32_t)treelet_gid >= mm->impl.num_treelets())
    return SVO_ERR_INVALID;
  *slot = mm->impl.treelet_slot(treelet_gid);
  return SVO_OK;
}

int svo_mm_copy_incore(svo_mm* mm, uint64_t first, uint64_t count, svo_node* h_nodes,
                       svo_attrib* h_attribs) {
  if (!mm) return SVO_ERR_INVALID;
  const uint64_t n = mm->impl.incore_nodes();
  if (first > n || count > n - first) return SVO_ERR_RANGE;
  if (h_nodes) std::memcpy(h_nodes, mm->impl.host_nodes() + first, count * sizeof(svo_node));
  if (h_attribs)
    std::memcpy(h_attribs, mm->impl.host_attribs() + first, count * sizeof(svo_attrib));
  return SVO_OK;
}

int svo_mm_slots_to_upload(svo_mm* mm, uint32_t* h_slots, uint32_t capacity, uint32_t* count) {
  if (!mm) return SVO_ERR_INVALID;
  const auto& up = mm->impl.slots_to_upload();
  if (count) *count = (uint32_t)up.size();
  if (!h_slots) return SVO_OK;
  uint32_t i = 0;
  for (uint32_t s : up) {
    if (i == capacity) break;
    h_slots[i++] = s;
  }
  return SVO_OK;
}

// ---- ray cast -------------------------------------------------------------

int svo_render(const svo_node* d_nodes, const svo_attrib* d_attribs, uint64_t num_nodes,
               const svo_frame_params* params, const svo_trace_cfg* cfg, uint32_t* d_rgba,
               svo_hit* d_hits, svo_stats* d_stats, void* stream) {
  if (!params || !d_nodes || !d_rgba || num_nodes == 0 || num_nodes > 0x100000000ull)
    return SVO_ERR_INVALID;
  int rc = check_cfg(cfg);
  if (rc != SVO_OK) return rc;
  rc = check_frame_mode(params->mode, cfg->traversal);
  if (rc != SVO_OK) return rc;
  if ((params->mode == 0 || params->mode == 1 || params->mode == 6) && !d_attribs)
    return SVO_ERR_INVALID;
  return svo::launch_render(d_nodes, d_attribs, num_nodes, *params, *cfg, d_rgba, d_hits, d_stats,
                            (cudaStream_t)stream);
}

int svo_render_shadow(const svo_node* d_nodes, const svo_attrib* d_attribs, uint64_t num_nodes,
                      const svo_frame_params* params, const svo_trace_cfg* cfg,
                      const svo_shadow_cfg* shadow, uint32_t* d_rgba, svo_hit* d_hits,
                      svo_hit* d_shadow_hits, svo_stats* d_stats, void* stream) {
  if (!params || !shadow || !d_nodes || !d_attribs || !d_rgba || num_nodes == 0 ||
      num_nodes > 0x100000000ull)
    return SVO_ERR_INVALID;
  const int rc = check_cfg(cfg);
  if (rc != SVO_OK) return rc;
  if (cfg->traversal != SVO_TRAVERSAL_TREELET) return SVO_ERR_NOTSUP;
  if (shadow->reserved != 0u) return SVO_ERR_INVALID;
  return svo::launch_render_shadow(d_nodes, d_attribs, num_nodes, *params, *shadow,
                                   cfg->stack_size, d_rgba, d_hits, d_shadow_hits, d_stats,
                                   (cudaStream_t)stream);
}

int svo_trace_rays(const svo_node* d_nodes, uint64_t num_nodes, const float* d_origins,
                   const float* d_dirs, uint64_t n, float t_scale_ratio, const svo_trace_cfg* cfg,
                   svo_hit* d_hits, svo_stats* d_stats, void* stream) {
  if (!d_nodes || !d_origins || !d_dirs || !d_hits || num_nodes == 0 ||
      num_nodes > 0x100000000ull)
    return SVO_ERR_INVALID;
  const int rc = check_cfg(cfg);
  if (rc != SVO_OK) return rc;
  return svo::launch_trace_rays(d_nodes, num_nodes, d_origins, d_dirs, n, t_scale_ratio, *cfg,
                                d_hits, d_stats, (cudaStream_t)stream);
}

int svo_mm_render(svo_mm* mm, const svo_frame_params* params, const svo_trace_cfg* cfg,
                  uint32_t* d_rgba, svo_hit* d_hits, void* stream) {
  if (!mm || !mm->impl.device_ready()) return SVO_ERR_INVALID;
  cudaStream_t s = stream ? (cudaStream_t)stream : mm->impl.render_stream();
  int rc = mm->impl.wait_uploads(s);
  if (rc != SVO_OK) return rc;
  return svo_render(mm->impl.device_nodes(), mm->impl.device_attribs(), mm->impl.incore_nodes(),
                    params, cfg, d_rgba, d_hits, mm->impl.device_stats(), s);
}

int svo_mm_render_shadow(svo_mm* mm, const svo_frame_params* params, const svo_trace_cfg* cfg,
                         const svo_shadow_cfg* shadow, uint32_t* d_rgba, svo_hit* d_hits,
                         svo_hit* d_shadow_hits, void* stream) {
  if (!mm || !mm->impl.device_ready()) return SVO_ERR_INVALID;
  cudaStream_t s = stream ? (cudaStream_t)stream : mm->impl.render_stream();
  int rc = mm->impl.wait_uploads(s);
  if (rc != SVO_OK) return rc;
  return svo_render_shadow(mm->impl.device_nodes(), mm->impl.device_attribs(),
                           mm->impl.incore_nodes(), params, cfg, shadow, d_rgba, d_hits,
                           d_shadow_hits, mm->impl.device_stats(), s);
}

int svo_mm_render_host(svo_mm* mm, const svo_frame_params* params, const svo_trace_cfg* cfg,
                       uint32_t* h_rgba, void* stream) {
  if (!mm || !params || !h_rgba || !mm->impl.device_ready()) return SVO_ERR_INVALID;
  cudaStream_t s = stream ? (cudaStream_t)stream : mm->impl.render_stream();
  const uint64_t pixels = (uint64_t)params->width * params->height;
  if (pixels == 0) return SVO_OK;
  uint32_t* d_rgba = nullptr;
  int rc = mm->impl.rgba_scratch(pixels, &d_rgba);
  if (rc != SVO_OK) return rc;
  rc = svo_mm_render(mm, params, cfg, d_rgba, nullptr, s);
  if (rc != SVO_OK) return rc;
  SVO_CUDA_TRY(cudaMemcpyAsync(h_rgba, d_rgba, pixels * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  SVO_CUDA_TRY(cudaStreamSynchronize(s));
  return SVO_OK;
}

int svo_mm_render_host_async(svo_mm* mm, const svo_frame_params* params, const svo_trace_cfg* cfg,
                             uint32_t* h_rgba, void* stream) {
  if (!mm || !params || !h_rgba || !mm->impl.device_ready()) return SVO_ERR_INVALID;
  int rc = check_cfg(cfg);
  if (rc != SVO_OK) return rc;
  rc = check_frame_mode(params->mode, cfg->traversal);
  if (rc != SVO_OK) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : mm->impl.render_stream();
  return guarded([&] { return mm->impl.render_to_host_async(*params, *cfg, h_rgba, s); });
}

int svo_mm_render_shadow_host_async(svo_mm* mm, const svo_frame_params* params,
                                    const svo_trace_cfg* cfg, const svo_shadow_cfg* shadow,
                                    uint32_t* h_rgba, void* stream) {
  if (!mm || !params || !shadow || !h_rgba || !mm->impl.device_ready()) return SVO_ERR_INVALID;
  const int rc = check_cfg(cfg);
  if (rc != SVO_OK) return rc;
  if (cfg->traversal != SVO_TRAVERSAL_TREELET) return SVO_ERR_NOTSUP;
  if (shadow->reserved != 0u) return SVO_ERR_INVALID;
  cudaStream_t s = stream ? (cudaStream_t)stream : mm->impl.render_stream();
  return guarded([&] { return mm->impl.render_to_host_async(*params, *cfg, h_rgba, s, shadow); });
}

int svo_mm_sync(svo_mm* mm, void* stream, svo_stats* out) {
  if (!mm || !mm->impl.device_ready()) return SVO_ERR_INVALID;
  cudaStream_t s = stream ? (cudaStream_t)stream : mm->impl.render_stream();
  svo_stats st;
  SVO_CUDA_TRY(cudaStreamSynchronize(s));
  const int rc = mm->impl.wait_host_frames();
  if (rc != SVO_OK) return rc;
  SVO_CUDA_TRY(cudaMemcpy(&st, mm->impl.device_stats(), sizeof(st), cudaMemcpyDeviceToHost));
  SVO_CUDA_TRY(cudaMemset(mm->impl.device_stats(), 0, sizeof(svo_stats)));
  if (out) *out = st;
  return SVO_OK;
}

// ---- analysis pass ----------------------------------------------------------

int svo_feedback_render(const svo_node* d_nodes, uint64_t num_nodes, const svo_frame_params* params,
                        int32_t stack_size, svo_feedback* d_feedback, uint32_t* d_rgba,
                        void* stream) {
  if (!d_nodes || !params || !d_feedback || num_nodes == 0 || num_nodes > 0x100000000ull)
    return SVO_ERR_INVALID;
  if (stack_size < 2 || stack_size > 24) return SVO_ERR_RANGE;
  return svo::launch_feedback(d_nodes, num_nodes, *params, stack_size, d_feedback, d_rgba,
                              (cudaStream_t)stream);
}

int svo_mm_analyse_feedback(svo_mm* mm, const svo_feedback* h_feedback, uint64_t n, uint32_t max_new,
                            int32_t* new_gids, float* new_errors, uint32_t new_capacity,
                            uint32_t* num_new, int32_t* old_gids, float* old_errors,
                            uint32_t old_capacity, uint32_t* num_old) {
  if (!mm || (n && !h_feedback)) return SVO_ERR_INVALID;
  return guarded([&] {
    std::vector<std::pair<int32_t, float>> nw, old;
    const uint32_t cap = max_new ? max_new : mm->impl.default_max_new_treelets();
    const int rc = mm->impl.analyse_feedback(h_feedback, n, cap, nw, old);
    return export_lists(rc, nw, old, new_gids, new_errors, new_capacity, num_new, old_gids,
                        old_errors, old_capacity, num_old);
  });
}

int svo_mm_analyse_feedback_device(svo_mm* mm, const svo_feedback* d_feedback, uint64_t n,
                                   uint32_t max_new, void* stream, int32_t* new_gids,
                                   float* new_errors, uint32_t new_capacity, uint32_t* num_new,
                                   int32_t* old_gids, float* old_errors, uint32_t old_capacity,
                                   uint32_t* num_old) {
  if (!mm || (n && !d_feedback) || !mm->impl.device_ready()) return SVO_ERR_INVALID;
  return guarded([&] {
    std::vector<std::pair<int32_t, float>> nw, old;
    const uint32_t cap = max_new ? max_new : mm->impl.default_max_new_treelets();
    cudaStream_t s = stream ? (cudaStream_t)stream : mm->impl.render_stream();
    const int rc = mm->impl.analyse_feedback_device(d_feedback, n, cap, nw, old, s);
    return export_lists(rc, nw, old, new_gids, new_errors, new_capacity, num_new, old_gids,
                        old_errors, old_capacity, num_old);
  });
}

int svo_mm_set_analysis_budget(svo_mm* mm, uint64_t bytes) {
  if (!mm) return SVO_ERR_INVALID;
  const uint64_t tb = mm->impl.treelet_bytes();
  const uint64_t n = bytes / tb;
  if (bytes && n == 0) return SVO_ERR_RANGE;
  mm->impl.set_max_new_treelets((uint32_t)std::min<uint64_t>(n, 0xFFFFFFFFull));
  return SVO_OK;
}

int svo_mm_set_eviction(svo_mm* mm, int32_t rule) {
  if (!mm) return SVO_ERR_INVALID;
  if (rule != SVO_EVICT_REFERENCE && rule != SVO_EVICT_ANY_UNSEEN) return SVO_ERR_NOTSUP;
  mm->impl.set_evict_any_invisible(rule == SVO_EVICT_ANY_UNSEEN);
  return SVO_OK;
}

int svo_mm_analysis_requested(svo_mm* mm, uint32_t* requested) {
  if (!mm || !requested) return SVO_ERR_INVALID;
  *requested = mm->impl.last_requested();
  return SVO_OK;
}

int svo_mm_analysis_step(svo_mm* mm, const svo_frame_params* frame, uint32_t divisor,
                         float jitter_x, float jitter_y, int32_t stack_size, void* stream,
                         uint32_t* num_new, uint32_t* num_old) {
  if (!mm || !frame || divisor == 0 || !mm->impl.device_ready()) return SVO_ERR_INVALID;
  if (stack_size < 2 || stack_size > 24) return SVO_ERR_RANGE;
  return guarded([&] {
    return mm->impl.analysis_step(*frame, divisor, jitter_x, jitter_y, stack_size, (cudaStream_t)stream,
                                  num_new, num_old);
  });
}

int svo_mm_analysis_begin(svo_mm* mm, const svo_frame_params* frame, uint32_t divisor,
                          float jitter_x, float jitter_y, int32_t stack_size, void* stream) {
  if (!mm || !frame || divisor == 0 || !mm->impl.device_ready()) return SVO_ERR_INVALID;
  if (stack_size < 2 || stack_size > 24) return SVO_ERR_RANGE;
  return guarded([&] {
    return mm->impl.analysis_begin(*frame, divisor, jitter_x, jitter_y, stack_size,
                                   (cudaStream_t)stream);
  });
}

int svo_mm_analysis_end(svo_mm* mm, void* after_stream, uint32_t* num_new, uint32_t* num_old) {
  if (!mm || !mm->impl.device_ready()) return SVO_ERR_INVALID;
  return guarded([&] { return mm->impl.analysis_end((cudaStream_t)after_stream, num_new, num_old); });
}

}  // extern "C"
