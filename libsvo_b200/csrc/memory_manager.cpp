// memory_manager.cpp -- see memory_manager.h.
#include "memory_manager.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <thread>

#include "analysis.h"
#include "errors.h"
#include "feedback.h"
#include "render.h"
#include "upload.h"

namespace svo {

TreeletMemoryManager::~TreeletMemoryManager() {
  std::free(incore_);
  std::free(incore_attr_);
}

int TreeletMemoryManager::init(svo_scene&& scene, uint64_t incore_bytes) {
  if (scene.treelets.empty() || scene.treelet_bytes < 128 || scene.treelet_bytes % 8 != 0)
    return SVO_ERR_INVALID;
  if (incore_bytes < scene.treelet_bytes) return SVO_ERR_RANGE;  // not even the root treelet
  scene_ = std::move(scene);
  N_ = scene_.treelet_bytes / 8;
  const uint64_t slots = incore_bytes / scene_.treelet_bytes;
  if (slots * (uint64_t)N_ > 0xFFFFFFFFull) return SVO_ERR_RANGE;  // uint32 node indices
  slots_.assign(slots, SlotInfo());
  // lazily zeroed host mirror of the incore buffer
  incore_ = (svo_node*)std::calloc(slots * N_, sizeof(svo_node));
  incore_attr_ = (svo_attrib*)std::calloc(slots * N_, sizeof(svo_attrib));
  if (!incore_ || !incore_attr_) return SVO_ERR_NOMEM;
  return reset_incore_buffer();
}

int TreeletMemoryManager::reset_incore_buffer() {
  before_host_write();
  free_.clear();
  upload_.clear();
  children_.assign(scene_.treelets.size(), std::set<int32_t>());
  slot_of_.assign(scene_.treelets.size(), -1);
  for (auto& s : slots_) s = SlotInfo();
  // push order as in the reference: slot 0 ends on top of the stack
  const uint32_t n = (uint32_t)slots_.size();
  for (uint32_t i = 1; i != n + 1; ++i) free_.push_back(n - i);
  search_pos_ = 1;
  SlotInfo root;
  root.treelet_gid = 0;
  root.visibility = kMaxVisibility;
  root.error = 999.0f;
  return insert_treelet(root);
}

int TreeletMemoryManager::insert_treelet(const SlotInfo& tve) {
  const int32_t gid = tve.treelet_gid;
  if (gid < 0 || (uint32_t)gid >= scene_.treelets.size()) return SVO_ERR_INVALID;
  if (slot_of_[gid] >= 0) return SVO_ERR_INVALID;  // already resident
  const TreeletData& t = scene_.treelets[gid];
  if (gid != 0 && slot_of_[t.parent_gid] < 0) return SVO_ERR_INVALID;  // parent not resident
  if (free_.empty()) {
    const int rc = free_incore_position();
    if (rc != SVO_OK) return rc;
    if (gid != 0 && slot_of_[t.parent_gid] < 0) return SVO_ERR_BUSY;  // parent was evicted
  }
  before_host_write();
  const uint32_t slot = free_.back();
  free_.pop_back();
  slots_[slot] = tve;
  slot_of_[gid] = (int32_t)slot;
  const uint64_t pos = (uint64_t)slot * N_;
  if (defer_) {
    pending_gid_[slot] = gid;
    pending_ops_[slot].clear();
    pending_slots_.push_back(slot);
  } else {
    copy_body(slot, gid);
  }
  mark_upload(slot);
  if (gid == 0) return SVO_OK;
  // patch the parent's leaf (TreeletMemoryManager.cpp:518-545): the leaf
  // becomes a copy of the treelet's root pointing into its slot, and its
  // flag in the leaf's parent is cleared
  const uint32_t pslot = (uint32_t)slot_of_[t.parent_gid];
  LeafWrite w;
  w.leaf = (uint64_t)pslot * N_ + (uint64_t)t.parent_leaf_position;
  w.leaf_parent = (uint64_t)pslot * N_ + (uint64_t)t.parent_leaf_parent_position;
  w.value = t.nodes[0];
  w.value.first_child = (uint32_t)((int64_t)(pos + 1) - (int64_t)w.leaf);
  w.bit = 1u << (uint32_t)t.parent_leaf_idx;
  w.set = false;
  write_leaf(pslot, w);
  mark_upload(pslot);
  children_[t.parent_gid].insert(gid);
  return SVO_OK;
}

int TreeletMemoryManager::remove_treelet(int32_t gid) {
  if (gid <= 0 || (uint32_t)gid >= scene_.treelets.size()) return SVO_ERR_INVALID;
  if (slot_of_[gid] < 0) return SVO_ERR_INVALID;
  const TreeletData& t = scene_.treelets[gid];
  const int32_t pslot = slot_of_[t.parent_gid];
  if (pslot < 0) return SVO_ERR_INVALID;
  before_host_write();
  const uint32_t slot = (uint32_t)slot_of_[gid];
  complete_pending(slot);
  // restore the original leaf and its leaf flag (TreeletMemoryManager.cpp:679-683)
  const TreeletData& pt = scene_.treelets[t.parent_gid];
  LeafWrite w;
  w.leaf = (uint64_t)pslot * N_ + (uint64_t)t.parent_leaf_position;
  w.leaf_parent = (uint64_t)pslot * N_ + (uint64_t)t.parent_leaf_parent_position;
  w.value = (uint32_t)t.parent_leaf_position < pt.num_nodes ? pt.nodes[t.parent_leaf_position]
                                                            : svo_node{0u, 0u};
  w.bit = 1u << (uint32_t)t.parent_leaf_idx;
  w.set = true;
  write_leaf((uint32_t)pslot, w);
  mark_upload((uint32_t)pslot);
  slots_[slot] = SlotInfo();
  free_.push_back(slot);
  slot_of_[gid] = -1;
  children_[t.parent_gid].erase(gid);
  return SVO_OK;
}

void TreeletMemoryManager::copy_body(uint32_t slot, int32_t gid) {
  const TreeletData& t = scene_.treelets[gid];
  const uint64_t pos = (uint64_t)slot * N_;
  std::memcpy(incore_ + pos, t.nodes.data(), (size_t)t.num_nodes * sizeof(svo_node));
  std::memset(incore_ + pos + t.num_nodes, 0, (size_t)(N_ - t.num_nodes) * sizeof(svo_node));
  std::memcpy(incore_attr_ + pos, t.attribs.data(), (size_t)t.num_nodes * sizeof(svo_attrib));
  std::memset(incore_attr_ + pos + t.num_nodes, 0, (size_t)(N_ - t.num_nodes) * sizeof(svo_attrib));
}

void TreeletMemoryManager::write_leaf(uint32_t pslot, const LeafWrite& w) {
  if (defer_ && pending_gid_[pslot] >= 0) {
    pending_ops_[pslot].push_back(w);
    return;
  }
  incore_[w.leaf] = w.value;
  if (w.set)
    incore_[w.leaf_parent].masks |= w.bit;
  else
    incore_[w.leaf_parent].masks &= ~w.bit;
}

void TreeletMemoryManager::complete_pending(uint32_t slot) {
  if (!defer_ || pending_gid_[slot] < 0) return;
  const int32_t gid = pending_gid_[slot];
  pending_gid_[slot] = -1;
  copy_body(slot, gid);
  for (const LeafWrite& w : pending_ops_[slot]) write_leaf(slot, w);
  pending_ops_[slot].clear();
}

void TreeletMemoryManager::begin_deferred() {
  pending_gid_.assign(slots_.size(), -1);
  pending_ops_.resize(slots_.size());
  pending_slots_.clear();
  defer_ = true;
}

void TreeletMemoryManager::end_deferred() {
  std::vector<uint32_t> todo;
  for (uint32_t s : pending_slots_)
    if (pending_gid_[s] >= 0) todo.push_back(s);  // a slot placed twice is listed twice
  std::sort(todo.begin(), todo.end());
  todo.erase(std::unique(todo.begin(), todo.end()), todo.end());
  // bodies first, on up to 8 threads for more than 16 slots ...
  auto bodies = [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; ++i) copy_body(todo[i], pending_gid_[todo[i]]);
  };
  static const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t parts = todo.size() > 16 ? std::min<size_t>(std::min<size_t>(8, hw), todo.size() / 8) : 1;
  std::vector<std::thread> workers;
  size_t started = 1;  // part 0 runs on this thread
  try {
    for (; started < parts; ++started)
      workers.emplace_back(bodies, todo.size() * started / parts, todo.size() * (started + 1) / parts);
  } catch (...) {  // no more threads: the rest runs here
  }
  bodies(0, parts ? todo.size() / parts : todo.size());
  if (started < parts) bodies(todo.size() * started / parts, todo.size());
  for (std::thread& w : workers) w.join();
  // ... then, per slot in order, the writes aimed at it
  defer_ = false;
  for (uint32_t s : todo) {
    for (const LeafWrite& w : pending_ops_[s]) write_leaf(s, w);
    pending_ops_[s].clear();
    pending_gid_[s] = -1;
  }
  pending_slots_.clear();
}

int TreeletMemoryManager::free_incore_position() {
  const uint32_t n = (uint32_t)slots_.size();
  if (n <= 1) return SVO_ERR_BUSY;
  if (search_pos_ >= n) search_pos_ = 1;
  int32_t freeable = 0;
  uint32_t tests = 0;
  for (uint32_t i = 0; i != n; ++i) {
    const SlotInfo& s = slots_[search_pos_];
    if (s.visibility < 0 && s.treelet_gid != -1) {
      const int32_t parent = scene_.treelets[s.treelet_gid].parent_gid;
      const int32_t ps = slot_of_[parent];
      if (ps >= 0 && (evict_any_invisible_ || slots_[ps].visibility < 0)) {
        freeable = s.treelet_gid;
        break;
      }
    }
    ++search_pos_;
    ++tests;
    if (search_pos_ == n) search_pos_ = 1;
    if (tests == kNumProbes) break;
  }
  if (freeable == 0) return SVO_ERR_BUSY;
  // every treelet attached below the freeable one goes too (.cpp:603-648)
  std::deque<int32_t> q;
  q.push_back(freeable);
  std::vector<int32_t> to_clear;
  while (!q.empty()) {
    const int32_t p = q.front();
    q.pop_front();
    for (int32_t c : children_[p]) {
      q.push_back(c);
      to_clear.push_back(c);
    }
    children_[p].clear();
  }
  before_host_write();
  for (int32_t c : to_clear) {
    const int32_t s = slot_of_[c];
    if (s > 0) {
      complete_pending((uint32_t)s);
      free_.push_back((uint32_t)s);
      slot_of_[c] = -1;
      slots_[s] = SlotInfo();
    }
  }
  return remove_treelet(freeable);
}

int TreeletMemoryManager::update_client_side(const int32_t* new_gids, const float* new_errors,
                                             uint32_t num_new, const int32_t* old_gids,
                                             uint32_t num_old, bool skip_unplaceable,
                                             uint32_t* inserted) {
  if (inserted) *inserted = 0;
  for (uint32_t i = 1; i < slots_.size(); ++i) --slots_[i].visibility;
  for (uint32_t i = 0; i < num_old; ++i) {
    const int32_t g = old_gids[i];
    if (g < 0 || (uint32_t)g >= scene_.treelets.size() || slot_of_[g] < 0) return SVO_ERR_INVALID;
    slots_[slot_of_[g]].visibility = kMaxVisibility;
  }
  int rc = SVO_OK;
  begin_deferred();
  try {
    for (uint32_t i = 0; i < num_new; ++i) {
      SlotInfo s;
      s.treelet_gid = new_gids[i];
      s.visibility = kMaxVisibility;
      s.error = new_errors ? new_errors[i] : 0.0f;
      // A treelet is unplaceable when no slot can be freed, or when its parent
      // is not resident (an earlier insertion of the same update evicted it);
      // the reference ignores these failures (TreeletMemoryManager.cpp:428-431)
      // and the next analysis pass asks for the treelet again.
      const bool parent_gone = s.treelet_gid > 0 && (uint32_t)s.treelet_gid < scene_.treelets.size() &&
                               slot_of_[s.treelet_gid] < 0 &&
                               slot_of_[scene_.treelets[s.treelet_gid].parent_gid] < 0;
      const int r = insert_treelet(s);
      if (r == SVO_OK) {
        if (inserted) ++*inserted;
        continue;
      }
      if (skip_unplaceable && (r == SVO_ERR_BUSY || (r == SVO_ERR_INVALID && parent_gone))) continue;
      if (rc == SVO_OK) rc = r;  // keep going, report the first failure
    }
  } catch (...) {  // (an allocation failed) the slots placed so far get their bodies
    end_deferred();
    throw;
  }
  end_deferred();
  return rc;
}

int TreeletMemoryManager::insert_all(uint32_t* inserted) {
  uint32_t n = 0;
  int rc = SVO_OK;
  for (uint32_t g = 1; g < scene_.treelets.size(); ++g) {
    if (slot_of_[g] >= 0) continue;
    if (free_.empty()) {
      rc = SVO_ERR_BUSY;
      break;
    }
    SlotInfo s;
    s.treelet_gid = (int32_t)g;
    s.visibility = kMaxVisibility;
    s.error = 0.0f;
    const int r = insert_treelet(s);
    if (r != SVO_OK) {
      rc = r;
      break;
    }
    ++n;
  }
  if (inserted) *inserted = n;
  return rc;
}

int TreeletMemoryManager::set_upload_ratio(float ratio) {
  if (!(ratio >= 0.0f && ratio <= 1.0f)) return SVO_ERR_RANGE;
  upload_ratio_ = ratio;
  return SVO_OK;
}

std::vector<std::pair<uint32_t, uint32_t>> TreeletMemoryManager::upload_ranges() const {
  std::vector<std::pair<uint32_t, uint32_t>> out;
  const float ratio_limit = upload_ratio_ * 2.0f;
  auto it = upload_.begin();
  while (it != upload_.end()) {
    const uint32_t start = *it;
    uint32_t num_slots = 1, num_treelets = 1;
    while (it != upload_.end()) {
      const int dist = (int)*it - (int)start;
      const float ratio = (float)(num_treelets + 1) / (float)(dist + 1);
      if (ratio >= ratio_limit) {
        num_slots = (uint32_t)dist + 1;
        ++num_treelets;
        ++it;
      } else {
        break;
      }
    }
    out.emplace_back(start, num_slots);
  }
  return out;
}

// ---------------------------------------------------------------------------

TreeletMemoryManagerCuda::~TreeletMemoryManagerCuda() {
  if (copy_stream_) cudaStreamSynchronize(copy_stream_);
  if (mirror_pinned_) {
    cudaHostUnregister(incore_);
    cudaHostUnregister(incore_attr_);
  }
  if (h_slot_ids_) cudaFreeHost(h_slot_ids_);
  if (d2h_stream_) cudaStreamSynchronize(d2h_stream_);
  for (int i = 0; i < 2; ++i) {
    cudaFree(d_img_[i]);
    if (cast_done_[i]) cudaEventDestroy(cast_done_[i]);
    if (copy_done_[i]) cudaEventDestroy(copy_done_[i]);
  }
  if (d2h_stream_) cudaStreamDestroy(d2h_stream_);
  if (owns_device_) {
    cudaFree(d_nodes_);
    cudaFree(d_attribs_);
  }
  cudaFree(d_stats_);
  cudaFree(d_rgba_);
  cudaFree(d_feedback_);
  cudaFree(d_slot_gid_);
  cudaFree(d_parent_);
  cudaFree(d_keys_);
  if (h_slot_gid_) cudaFreeHost(h_slot_gid_);
  if (h_keys_) cudaFreeHost(h_keys_);
  for (int i = 0; i < 2; ++i) {
    if (stage_evt_[i]) cudaEventDestroy(stage_evt_[i]);
    if (stage_[i]) cudaFreeHost(stage_[i]);
    if (h_ids_[i]) cudaFreeHost(h_ids_[i]);
    cudaFree(d_stage_[i]);
    cudaFree(d_ids_[i]);
  }
  if (upload_done_) cudaEventDestroy(upload_done_);
  if (analysis_done_) cudaEventDestroy(analysis_done_);
  if (after_done_) cudaEventDestroy(after_done_);
  if (copy_stream_) cudaStreamDestroy(copy_stream_);
}

int TreeletMemoryManagerCuda::init_transfer() {
  if (copy_stream_) return SVO_OK;
  SVO_CUDA_TRY(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
  SVO_CUDA_TRY(cudaEventCreateWithFlags(&upload_done_, cudaEventDisableTiming));
  for (int i = 0; i < 2; ++i) {
    SVO_CUDA_TRY(cudaEventCreateWithFlags(&stage_evt_[i], cudaEventDisableTiming));
    SVO_CUDA_TRY(cudaMallocHost(&stage_[i], kStageBytes));
  }
  SVO_CUDA_TRY(cudaMalloc(&d_stats_, sizeof(svo_stats)));
  SVO_CUDA_TRY(cudaMemsetAsync(d_stats_, 0, sizeof(svo_stats), copy_stream_));
  return SVO_OK;
}

// whole-buffer upload, as clCreateBuffer(COPY_HOST_PTR) does
// (TreeletMemoryManagerCl.cpp:106-112)
int TreeletMemoryManagerCuda::upload_all() {
  const uint64_t n = incore_nodes();
  if (mirror_pinned_) {
    // page-locked mirror: two DMA copies straight from it, no staging
    SVO_CUDA_TRY(cudaMemcpyAsync(d_nodes_, incore_, n * sizeof(svo_node), cudaMemcpyHostToDevice,
                                 copy_stream_));
    SVO_CUDA_TRY(cudaMemcpyAsync(d_attribs_, incore_attr_, n * sizeof(svo_attrib),
                                 cudaMemcpyHostToDevice, copy_stream_));
  } else {
    const int rc = stage_copies({{d_nodes_, incore_, n * sizeof(svo_node)},
                                 {d_attribs_, incore_attr_, n * sizeof(svo_attrib)}});
    if (rc != SVO_OK) return rc;
  }
  SVO_CUDA_TRY(cudaEventRecord(upload_done_, copy_stream_));
  upload_pending_ = true;
  upload_.clear();
  return SVO_OK;
}

int TreeletMemoryManagerCuda::init_device_buffer() {
  if (d_nodes_) return SVO_OK;
  int rc = init_transfer();
  if (rc != SVO_OK) return rc;
  const uint64_t n = incore_nodes();
  if (cudaMalloc(&d_nodes_, n * sizeof(svo_node)) != cudaSuccess ||
      cudaMalloc(&d_attribs_, n * sizeof(svo_attrib)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(d_nodes_);
    cudaFree(d_attribs_);
    d_nodes_ = nullptr;
    d_attribs_ = nullptr;
    return SVO_ERR_NOMEM;
  }
  owns_device_ = true;
  device_bytes_ = n * (sizeof(svo_node) + sizeof(svo_attrib));
  return upload_all();
}

int TreeletMemoryManagerCuda::attach_device_buffers(svo_node* d_nodes, svo_attrib* d_attribs) {
  if (d_nodes_ || !d_nodes || !d_attribs) return SVO_ERR_INVALID;
  int rc = init_transfer();
  if (rc != SVO_OK) return rc;
  d_nodes_ = d_nodes;
  d_attribs_ = d_attribs;
  owns_device_ = false;
  device_bytes_ = incore_nodes() * (sizeof(svo_node) + sizeof(svo_attrib));
  return upload_all();
}

int TreeletMemoryManagerCuda::detach_device_buffers() {
  if (!d_nodes_ || owns_device_) return SVO_ERR_INVALID;
  SVO_CUDA_TRY(cudaStreamSynchronize(copy_stream_));
  d_nodes_ = nullptr;
  d_attribs_ = nullptr;
  device_bytes_ = 0;
  upload_pending_ = false;
  return SVO_OK;
}

namespace {

struct HostPiece {
  char* dst;
  const char* src;
  uint64_t bytes;
};

// Host-to-host copies of `pieces` (`total` bytes) on up to 8 threads, each
// taking an equal span of the concatenated bytes; serial below 4 MB or when
// no thread can be started.
void copy_pieces(const std::vector<HostPiece>& pieces, uint64_t total) {
  auto span = [&](uint64_t lo, uint64_t hi) {
    uint64_t off = 0;
    for (const HostPiece& p : pieces) {
      const uint64_t a = std::max(lo, off), b = std::min(hi, off + p.bytes);
      if (a < b) std::memcpy(p.dst + (a - off), p.src + (a - off), (size_t)(b - a));
      off += p.bytes;
      if (off >= hi) break;
    }
  };
  static const uint64_t hw = std::max(1u, std::thread::hardware_concurrency());
  const uint64_t parts = std::min<uint64_t>(std::min<uint64_t>(8, hw), total / (1ull << 20));
  if (parts <= 1 || total < (4ull << 20)) {
    span(0, total);
    return;
  }
  std::vector<std::thread> workers;
  uint64_t started = 1;  // span 0 runs on this thread
  try {
    for (; started < parts; ++started)
      workers.emplace_back(span, total * started / parts, total * (started + 1) / parts);
  } catch (...) {  // no more threads: the rest runs here
  }
  span(0, total / parts);
  if (started < parts) span(total * started / parts, total);
  for (std::thread& w : workers) w.join();
}

}  // namespace

int TreeletMemoryManagerCuda::stage_copies(const std::vector<StagedCopy>& copies) {
  for (const StagedCopy& c : copies) {
    char* d = (char*)c.dst;
    const char* s = (const char*)c.src;
    uint64_t bytes = c.bytes;
    while (bytes) {
      const uint64_t n = std::min(bytes, kStageBytes);
      const int h = stage_next_;
      stage_next_ ^= 1;
      SVO_CUDA_TRY(cudaEventSynchronize(stage_evt_[h]));
      // small pieces land at the start of a half, which stays in the host's
      // caches; large ones are copied into it on several threads
      if (n >= (4ull << 20))
        copy_pieces({HostPiece{(char*)stage_[h], s, n}}, n);
      else
        std::memcpy(stage_[h], s, (size_t)n);
      SVO_CUDA_TRY(cudaMemcpyAsync(d, stage_[h], n, cudaMemcpyHostToDevice, copy_stream_));
      SVO_CUDA_TRY(cudaEventRecord(stage_evt_[h], copy_stream_));
      s += n;
      d += n;
      bytes -= n;
    }
  }
  return SVO_OK;
}

int TreeletMemoryManagerCuda::set_upload_policy(int policy) {
  if (policy != SVO_UPLOAD_COALESCED && policy != SVO_UPLOAD_PACKED && policy != SVO_UPLOAD_PINNED)
    return SVO_ERR_NOTSUP;
  if (policy == SVO_UPLOAD_PINNED && !mirror_pinned_) {
    const uint64_t bytes = incore_nodes() * sizeof(svo_node);
    cudaError_t e = cudaHostRegister(incore_, bytes, cudaHostRegisterMapped);
    if (e == cudaSuccess) {
      e = cudaHostRegister(incore_attr_, bytes, cudaHostRegisterMapped);
      if (e != cudaSuccess) cudaHostUnregister(incore_);
    }
    void* dn = nullptr;
    void* da = nullptr;
    void* di = nullptr;
    if (e == cudaSuccess && !h_slot_ids_)
      e = cudaHostAlloc(&h_slot_ids_, (size_t)num_slots() * sizeof(uint32_t), cudaHostAllocMapped);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer(&dn, incore_, 0);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer(&da, incore_attr_, 0);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer(&di, h_slot_ids_, 0);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return cuda_status(e);
    }
    mapped_nodes_ = (const svo_node*)dn;
    mapped_attribs_ = (const svo_attrib*)da;
    mapped_slot_ids_ = (const uint32_t*)di;
    mirror_pinned_ = true;
  }
  upload_policy_ = policy;
  return SVO_OK;
}

// With the mirror page-locked, the gather kernel and whole-pool uploads read
// it directly: a host-side change waits for the copies still in flight.
void TreeletMemoryManagerCuda::before_host_write() {
  if (mirror_pinned_ && upload_pending_ && copy_stream_) cudaStreamSynchronize(copy_stream_);
}

// Dirty slots packed back to back into a ring half ({nodes, attributes} per
// slot), one copy of the packed bytes and one of the slot ids, then the
// scatter kernel, all on the copy stream; the next use of a half waits for
// the event recorded after its scatter.
int TreeletMemoryManagerCuda::upload_packed(uint32_t* copy_calls) {
  const uint64_t slot_bytes = (uint64_t)N_ * (sizeof(svo_node) + sizeof(svo_attrib));
  // chunks of about 4 MB, so that packing the next chunk overlaps the copy
  // of the previous one
  const uint64_t chunk = std::min<uint64_t>(kStageBytes, std::max<uint64_t>(slot_bytes, 4ull << 20));
  const uint64_t per_half = chunk / slot_bytes;
  for (int i = 0; i < 2; ++i) {
    if (!d_stage_[i]) SVO_CUDA_TRY(cudaMalloc(&d_stage_[i], kStageBytes));
    if (!h_ids_[i]) SVO_CUDA_TRY(cudaMallocHost(&h_ids_[i], per_half * sizeof(uint32_t)));
    if (!d_ids_[i]) SVO_CUDA_TRY(cudaMalloc(&d_ids_[i], per_half * sizeof(uint32_t)));
  }
  uint32_t calls = 0;
  auto it = upload_.begin();
  while (it != upload_.end()) {
    const int h = stage_next_;
    stage_next_ ^= 1;
    SVO_CUDA_TRY(cudaEventSynchronize(stage_evt_[h]));
    char* dst = (char*)stage_[h];
    uint32_t k = 0;
    for (; it != upload_.end() && k < per_half; ++it, ++k) {
      const uint64_t first = (uint64_t)*it * N_;
      std::memcpy(dst, incore_ + first, (size_t)N_ * sizeof(svo_node));
      std::memcpy(dst + (size_t)N_ * sizeof(svo_node), incore_attr_ + first,
                  (size_t)N_ * sizeof(svo_attrib));
      dst += slot_bytes;
      h_ids_[h][k] = *it;
    }
    SVO_CUDA_TRY(cudaMemcpyAsync(d_stage_[h], stage_[h], k * slot_bytes, cudaMemcpyHostToDevice,
                                 copy_stream_));
    SVO_CUDA_TRY(cudaMemcpyAsync(d_ids_[h], h_ids_[h], k * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice, copy_stream_));
    const int rc = launch_slot_scatter(d_stage_[h], d_ids_[h], k, N_, d_nodes_, d_attribs_,
                                       copy_stream_);
    if (rc != SVO_OK) return rc;
    SVO_CUDA_TRY(cudaEventRecord(stage_evt_[h], copy_stream_));
    ++calls;
  }
  if (copy_calls) *copy_calls = calls;
  return SVO_OK;
}

int TreeletMemoryManagerCuda::update_device_memory(uint32_t* copy_calls) {
  if (copy_calls) *copy_calls = 0;
  if (upload_.empty()) return SVO_OK;
  if (!d_nodes_) return SVO_ERR_INVALID;  // init_device_buffer first
  const uint64_t slot_bytes = (uint64_t)N_ * (sizeof(svo_node) + sizeof(svo_attrib));
  if (upload_policy_ == SVO_UPLOAD_PACKED && slot_bytes <= kStageBytes) {
    const int rc = upload_packed(copy_calls);
    if (rc != SVO_OK) return rc;
    SVO_CUDA_TRY(cudaEventRecord(upload_done_, copy_stream_));
    upload_pending_ = true;
    upload_.clear();
    return SVO_OK;
  }
  if (upload_policy_ == SVO_UPLOAD_PINNED) {
    // the slot-id list is read by the previous gather until it finishes
    if (upload_pending_) SVO_CUDA_TRY(cudaStreamSynchronize(copy_stream_));
    uint32_t k = 0;
    for (uint32_t s : upload_) h_slot_ids_[k++] = s;
    const int rc = launch_slot_gather(mapped_nodes_, mapped_attribs_, mapped_slot_ids_, k, N_,
                                      d_nodes_, d_attribs_, copy_stream_);
    if (rc != SVO_OK) return rc;
    SVO_CUDA_TRY(cudaEventRecord(upload_done_, copy_stream_));
    upload_pending_ = true;
    if (copy_calls) *copy_calls = 1;
    upload_.clear();
    return SVO_OK;
  }
  const auto ranges = upload_ranges();
  std::vector<StagedCopy> copies;
  copies.reserve(2 * ranges.size());
  for (const auto& r : ranges) {
    const uint64_t first = (uint64_t)r.first * N_;
    const uint64_t count = (uint64_t)r.second * N_;
    copies.push_back({d_nodes_ + first, incore_ + first, count * sizeof(svo_node)});
    copies.push_back({d_attribs_ + first, incore_attr_ + first, count * sizeof(svo_attrib)});
  }
  const int rc = stage_copies(copies);
  if (rc != SVO_OK) return rc;
  SVO_CUDA_TRY(cudaEventRecord(upload_done_, copy_stream_));
  upload_pending_ = true;
  if (copy_calls) *copy_calls = (uint32_t)ranges.size();
  upload_.clear();
  return SVO_OK;
}

int TreeletMemoryManagerCuda::reset_incore_buffer() {
  const int rc = TreeletMemoryManager::reset_incore_buffer();
  if (rc != SVO_OK || !d_nodes_) return rc;
  // the device copy must match the fresh mirror: upload everything again
  for (uint32_t s = 0; s < num_slots(); ++s) mark_upload(s);
  return update_device_memory(nullptr);
}

int TreeletMemoryManagerCuda::wait_uploads(cudaStream_t stream) {
  if (!upload_pending_) return SVO_OK;
  SVO_CUDA_TRY(cudaStreamWaitEvent(stream, upload_done_, 0));
  return SVO_OK;
}

int TreeletMemoryManagerCuda::rgba_scratch(uint64_t pixels, uint32_t** out) {
  if (pixels > d_rgba_pixels_) {
    cudaFree(d_rgba_);
    d_rgba_ = nullptr;
    d_rgba_pixels_ = 0;
    SVO_CUDA_TRY(cudaMalloc(&d_rgba_, pixels * sizeof(uint32_t)));
    d_rgba_pixels_ = pixels;
  }
  *out = d_rgba_;
  return SVO_OK;
}

int TreeletMemoryManagerCuda::render_to_host_async(const svo_frame_params& p,
                                                   const svo_trace_cfg& cfg, uint32_t* h_rgba,
                                                   cudaStream_t stream,
                                                   const svo_shadow_cfg* shadow) {
  const uint64_t pixels = (uint64_t)p.width * p.height;
  if (pixels == 0) return SVO_OK;
  if (!d2h_stream_) {
    SVO_CUDA_TRY(cudaStreamCreateWithFlags(&d2h_stream_, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i) {
      SVO_CUDA_TRY(cudaEventCreateWithFlags(&cast_done_[i], cudaEventDisableTiming));
      SVO_CUDA_TRY(cudaEventCreateWithFlags(&copy_done_[i], cudaEventDisableTiming));
    }
  }
  const int k = img_next_;
  img_next_ ^= 1;
  if (pixels > d_img_pixels_[k]) {
    SVO_CUDA_TRY(cudaStreamSynchronize(d2h_stream_));  // the image may still be copied out
    SVO_CUDA_TRY(cudaStreamSynchronize(stream));
    cudaFree(d_img_[k]);
    d_img_[k] = nullptr;
    d_img_pixels_[k] = 0;
    SVO_CUDA_TRY(cudaMalloc(&d_img_[k], pixels * sizeof(uint32_t)));
    d_img_pixels_[k] = pixels;
  }
  // the cast may overwrite image k once its previous copy has left
  SVO_CUDA_TRY(cudaStreamWaitEvent(stream, copy_done_[k], 0));
  int rc = wait_uploads(stream);
  if (rc != SVO_OK) return rc;
  rc = shadow ? launch_render_shadow(d_nodes_, d_attribs_, incore_nodes(), p, *shadow,
                                     cfg.stack_size, d_img_[k], nullptr, nullptr, d_stats_, stream)
              : launch_render(d_nodes_, d_attribs_, incore_nodes(), p, cfg, d_img_[k], nullptr,
                              d_stats_, stream);
  if (rc != SVO_OK) return rc;
  SVO_CUDA_TRY(cudaEventRecord(cast_done_[k], stream));
  SVO_CUDA_TRY(cudaStreamWaitEvent(d2h_stream_, cast_done_[k], 0));
  SVO_CUDA_TRY(cudaMemcpyAsync(h_rgba, d_img_[k], pixels * sizeof(uint32_t),
                               cudaMemcpyDeviceToHost, d2h_stream_));
  SVO_CUDA_TRY(cudaEventRecord(copy_done_[k], d2h_stream_));
  return SVO_OK;
}

int TreeletMemoryManagerCuda::wait_host_frames() {
  if (d2h_stream_) SVO_CUDA_TRY(cudaStreamSynchronize(d2h_stream_));
  return SVO_OK;
}

int TreeletMemoryManagerCuda::init_analysis() {
  if (d_keys_) return SVO_OK;
  const uint32_t T = num_treelets(), S = num_slots();
  const size_t key_words = 2 * ((size_t)T + 1) + 1;
  std::vector<int32_t> parent(T > 0 ? T : 1, 0);
  for (uint32_t g = 0; g < T; ++g) parent[g] = scene_.treelets[g].parent_gid;
  int32_t* d_slot = nullptr;
  int32_t* h_slot = nullptr;
  int32_t* d_par = nullptr;
  uint32_t* d_keys = nullptr;
  uint32_t* h_keys = nullptr;
  auto fail = [&](cudaError_t e) {
    cudaFree(d_slot);
    cudaFree(d_par);
    cudaFree(d_keys);
    if (h_slot) cudaFreeHost(h_slot);
    if (h_keys) cudaFreeHost(h_keys);
    return cuda_status(e);
  };
  cudaError_t e = cudaMalloc(&d_slot, (size_t)S * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMallocHost(&h_slot, (size_t)S * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc(&d_par, parent.size() * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc(&d_keys, key_words * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMallocHost(&h_keys, key_words * sizeof(uint32_t));
  if (e == cudaSuccess)
    e = cudaMemcpy(d_par, parent.data(), parent.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail(e);
  d_slot_gid_ = d_slot;
  h_slot_gid_ = h_slot;
  d_parent_ = d_par;
  d_keys_ = d_keys;
  h_keys_ = h_keys;
  return SVO_OK;
}

int TreeletMemoryManagerCuda::launch_fold(const svo_feedback* d_fb, uint64_t n, cudaStream_t stream) {
  if (n > 0 && !d_fb) return SVO_ERR_INVALID;
  int rc = init_analysis();
  if (rc != SVO_OK) return rc;
  const uint32_t T = num_treelets(), S = num_slots();
  const size_t words = 2 * ((size_t)T + 1) + 1;
  uint32_t* d_new = d_keys_;
  uint32_t* d_old = d_keys_ + (T + 1);
  uint32_t* d_status = d_keys_ + 2 * ((size_t)T + 1);
  // The page-locked slot table is free: every fold's copies are waited for
  // (read_fold, or a failed launch's synchronisation) before the next one.
  for (uint32_t i = 0; i < S; ++i) h_slot_gid_[i] = slots_[i].treelet_gid;
  cudaError_t e = cudaMemcpyAsync(d_slot_gid_, h_slot_gid_, (size_t)S * sizeof(int32_t),
                                  cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_keys_, 0, words * sizeof(uint32_t), stream);
  if (e == cudaSuccess) {
    rc = launch_analyse(d_fb, n, d_slot_gid_, S, N_, d_parent_, T, d_new, d_old, d_status, stream);
    if (rc == SVO_OK)
      e = cudaMemcpyAsync(h_keys_, d_keys_, words * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                          stream);
  }
  if (e != cudaSuccess || rc != SVO_OK) {
    cudaStreamSynchronize(stream);  // the copies may still read the slot table
    return e != cudaSuccess ? cuda_status(e) : rc;
  }
  return SVO_OK;
}

int TreeletMemoryManagerCuda::read_fold(uint32_t max_new,
                                        std::vector<std::pair<int32_t, float>>& out_new,
                                        std::vector<std::pair<int32_t, float>>& out_old) {
  const uint32_t T = num_treelets();
  if (h_keys_[2 * ((size_t)T + 1)] & kAnalyseRejected) return SVO_ERR_RANGE;
  const uint32_t* h_new = h_keys_;
  const uint32_t* h_old = h_keys_ + (T + 1);
  for (uint32_t g = 0; g <= T; ++g) {
    if (h_new[g]) out_new.emplace_back((int32_t)g, key_error(h_new[g]));
    if (h_old[g]) out_old.emplace_back((int32_t)g, key_error(h_old[g]));
  }
  auto by_error = [](const std::pair<int32_t, float>& a, const std::pair<int32_t, float>& b) {
    return a.second > b.second;
  };
  std::stable_sort(out_new.begin(), out_new.end(), by_error);
  std::stable_sort(out_old.begin(), out_old.end(), by_error);
  if (out_new.size() > max_new) out_new.resize(max_new);
  return SVO_OK;
}

int TreeletMemoryManagerCuda::analyse_feedback_device(
    const svo_feedback* d_fb, uint64_t n, uint32_t max_new,
    std::vector<std::pair<int32_t, float>>& out_new, std::vector<std::pair<int32_t, float>>& out_old,
    cudaStream_t stream) {
  out_new.clear();
  out_old.clear();
  const int rc = launch_fold(d_fb, n, stream);
  if (rc != SVO_OK) return rc;
  SVO_CUDA_TRY(cudaStreamSynchronize(stream));
  return read_fold(max_new, out_new, out_old);
}

int TreeletMemoryManagerCuda::feedback_scratch(uint64_t records, svo_feedback** out) {
  if (records > d_feedback_records_) {
    // grown at least twofold (cudaFree waits for the whole device, so views
    // of random sizes should reallocate only a few times)
    const uint64_t grow = std::max<uint64_t>(records, 2 * d_feedback_records_);
    cudaFree(d_feedback_);
    d_feedback_ = nullptr;
    d_feedback_records_ = 0;
    SVO_CUDA_TRY(cudaMalloc(&d_feedback_, grow * sizeof(svo_feedback)));
    d_feedback_records_ = grow;
  }
  *out = d_feedback_;
  return SVO_OK;
}

int TreeletMemoryManagerCuda::analysis_begin(const svo_frame_params& frame, uint32_t divisor,
                                             float jitter_x, float jitter_y, int32_t stack_size,
                                             cudaStream_t stream) {
  last_requested_ = 0;
  if (analysis_pending_) return SVO_ERR_BUSY;  // the previous half-step was not ended
  if (divisor == 0 || !device_ready()) return SVO_ERR_INVALID;
  if (stack_size < 2 || stack_size > 24) return SVO_ERR_RANGE;
  cudaStream_t s = stream ? stream : render_stream_;
  // analysis buffer and its one-pixel far-plane vectors
  // (RenderPassAnalyse.cpp:168-193): same frustum, coarser pixels
  svo_frame_params a = frame;
  a.width = std::max(1u, frame.width / divisor);
  a.height = std::max(1u, frame.height / divisor);
  const double sx = (double)frame.width / a.width, sy = (double)frame.height / a.height;
  for (int k = 0; k < 3; ++k) {
    a.pixel_far_h[k] = (float)(frame.pixel_far_h[k] * sx);
    a.pixel_far_v[k] = (float)(frame.pixel_far_v[k] * sy);
    a.far_lower_left[k] = (float)(frame.far_lower_left[k] +
                                  jitter_x * (double)divisor * frame.pixel_far_h[k] * 0.5 +
                                  jitter_y * (double)divisor * frame.pixel_far_v[k] * 0.5);
  }
  const uint64_t n = (uint64_t)a.width * a.height;
  svo_feedback* d_fb = nullptr;
  int rc = feedback_scratch(n, &d_fb);
  if (rc != SVO_OK) return rc;
  rc = wait_uploads(s);
  if (rc != SVO_OK) return rc;
  if (!analysis_done_) SVO_CUDA_TRY(cudaEventCreateWithFlags(&analysis_done_, cudaEventDisableTiming));
  rc = launch_feedback(device_nodes(), incore_nodes(), a, stack_size, d_fb, nullptr, s);
  if (rc != SVO_OK) return rc;
  // the records stay on the GPU; only per-treelet results come back
  rc = launch_fold(d_fb, n, s);
  if (rc != SVO_OK) return rc;
  SVO_CUDA_TRY(cudaEventRecord(analysis_done_, s));
  analysis_pending_ = true;
  return SVO_OK;
}

int TreeletMemoryManagerCuda::analysis_end(cudaStream_t after, uint32_t* num_new, uint32_t* num_old,
                                           uint32_t* num_requested) {
  if (num_new) *num_new = 0;
  if (num_old) *num_old = 0;
  if (num_requested) *num_requested = 0;
  if (!analysis_pending_) return SVO_ERR_INVALID;
  analysis_pending_ = false;
  SVO_CUDA_TRY(cudaEventSynchronize(analysis_done_));
  std::vector<std::pair<int32_t, float>> nw, old;
  int rc = read_fold(max_new_treelets(), nw, old);
  if (num_new) *num_new = (uint32_t)nw.size();
  if (num_old) *num_old = (uint32_t)old.size();
  if (num_requested) *num_requested = (uint32_t)nw.size();
  last_requested_ = (uint32_t)nw.size();
  if (rc != SVO_OK) return rc;
  std::vector<int32_t> ng(nw.size()), og(old.size());
  std::vector<float> ne(nw.size());
  for (size_t i = 0; i < nw.size(); ++i) ng[i] = nw[i].first, ne[i] = nw[i].second;
  for (size_t i = 0; i < old.size(); ++i) og[i] = old[i].first;
  uint32_t placed = 0;
  rc = update_client_side(ng.data(), ne.data(), (uint32_t)ng.size(), og.data(), (uint32_t)og.size(),
                          true, &placed);
  if (num_new) *num_new = placed;
  // the upload overwrites slots that the work already queued on `after` (a
  // frame cast from the pool) may still read
  if (!upload_.empty()) {
    cudaStream_t w = after ? after : render_stream_;
    if (!after_done_) SVO_CUDA_TRY(cudaEventCreateWithFlags(&after_done_, cudaEventDisableTiming));
    if (!copy_stream_) {  // created with the staging by init_transfer
      const int t = init_transfer();
      if (t != SVO_OK) return t;
    }
    SVO_CUDA_TRY(cudaEventRecord(after_done_, w));
    SVO_CUDA_TRY(cudaStreamWaitEvent(copy_stream_, after_done_, 0));
  }
  const int up = update_device_memory(nullptr);
  return rc != SVO_OK ? rc : up;
}

int TreeletMemoryManagerCuda::analysis_step(const svo_frame_params& frame, uint32_t divisor,
                                            float jitter_x, float jitter_y, int32_t stack_size,
                                            cudaStream_t stream, uint32_t* num_new,
                                            uint32_t* num_old, uint32_t* num_requested) {
  if (num_new) *num_new = 0;
  if (num_old) *num_old = 0;
  if (num_requested) *num_requested = 0;
  const int rc = analysis_begin(frame, divisor, jitter_x, jitter_y, stack_size, stream);
  if (rc != SVO_OK) return rc;
  return analysis_end(stream ? stream : render_stream_, num_new, num_old, num_requested);
}

}  // namespace svo
