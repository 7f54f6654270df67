// memory_manager.h -- the treelet incore buffer and its device copy.
//
// TreeletMemoryManager keeps the host-side bookkeeping of
// src/TreeletMemoryManager.{h,cpp}: a fixed number of treelet slots, a stack
// of free slots, per-slot visibility, the child treelets resident below each
// treelet, and the set of slots to upload.  TreeletMemoryManagerCuda replaces
// TreeletMemoryManagerCl (src/TreeletMemoryManagerCl.{h,cpp}): the incore
// buffer lives in HBM, dirty slots go up through a pinned staging ring with
// cudaMemcpyAsync on a side stream, and renders wait on an event for them.
//
// The host mirror is plain (pageable, lazily zeroed) memory, so that large
// budgets do not pin host RAM; only the staging ring is pinned.  No CUDA call
// is made before init_device_buffer(), so the bookkeeping runs without a GPU.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <set>
#include <vector>

#include "../../include/libsvo_b200.h"
#include "scene.h"

namespace svo {

class TreeletMemoryManager {
 public:
  struct SlotInfo {  // src/TreeletMemoryManager.h:72-89
    int32_t treelet_gid = -1;
    int32_t visibility = 0;
    float error = 100000.0f;
  };
  static constexpr int32_t kMaxVisibility = 8;  // MAX_VISIBILITY, TreeletMemoryManager.cpp:47
  static constexpr uint32_t kNumProbes = 100;   // freeIncorePosition probe budget

  virtual ~TreeletMemoryManager();

  // ctor + loadFromFile + resetIncoreBuffer (TreeletMemoryManager.cpp:72-102)
  int init(svo_scene&& scene, uint64_t incore_bytes);

  int insert_treelet(const SlotInfo& tve);           // .cpp:456-548
  int remove_treelet(int32_t gid);                   // .cpp:666-700
  int free_incore_position();                        // .cpp:561-653
  // updateClientSideIncoreBuffer.  skip_unplaceable: treelets that find no
  // slot, or whose parent is not resident, are skipped instead of reported
  // (as the reference does); *inserted counts the treelets placed.
  int update_client_side(const int32_t* new_gids, const float* new_errors, uint32_t num_new,
                         const int32_t* old_gids, uint32_t num_old, bool skip_unplaceable = false,
                         uint32_t* inserted = nullptr);  // .cpp:393-443
  virtual int reset_incore_buffer();                 // .cpp:304-380
  int insert_all(uint32_t* inserted);

  uint32_t num_treelets() const { return (uint32_t)scene_.treelets.size(); }
  uint32_t treelet_bytes() const { return scene_.treelet_bytes; }
  uint32_t nodes_per_treelet() const { return N_; }
  uint32_t num_slots() const { return (uint32_t)slots_.size(); }
  uint32_t free_slots() const { return (uint32_t)free_.size(); }
  uint64_t incore_nodes() const { return (uint64_t)slots_.size() * N_; }
  const std::set<uint32_t>& slots_to_upload() const { return upload_; }
  const SlotInfo& slot(uint32_t i) const { return slots_[i]; }
  int32_t treelet_slot(int32_t gid) const { return slot_of_[gid]; }
  const svo_node* host_nodes() const { return incore_; }
  const svo_attrib* host_attribs() const { return incore_attr_; }
  const svo_scene& scene() const { return scene_; }

  // performAnalysePass's processing of the feedback records
  // (src/RenderPassAnalyse.cpp:218-356): newly visible treelets (cut to
  // max_new) and visible resident treelets, each as (gid, error), largest
  // error first.  SVO_ERR_RANGE (and empty lists) on records the reference
  // rejects.
  int analyse_feedback(const svo_feedback* fb, uint64_t n, uint32_t max_new,
                       std::vector<std::pair<int32_t, float>>& out_new,
                       std::vector<std::pair<int32_t, float>>& out_old) const;
  // 12 MB worth of treelets (RenderPassAnalyse.cpp:340).
  uint32_t default_max_new_treelets() const;
  // Newly visible treelets one analysis step may place: the reference's
  // 12 MB worth (src/RenderPassAnalyse.cpp:340) unless set; 0 restores it.
  void set_max_new_treelets(uint32_t n) { max_new_ = n; }
  uint32_t max_new_treelets() const { return max_new_ ? max_new_ : default_max_new_treelets(); }
  // Newly visible treelets the last analysis step asked for, placed or not.
  uint32_t last_requested() const { return last_requested_; }
  // Marks every resident treelet but the root unseen (visibility -1), as if
  // it had not been seen for as many passes as the reference's visibility
  // counter lasts: the next analysis pass marks what its view sees again, and
  // everything else can be evicted at once instead of after 9 passes.
  void mark_all_unseen() {
    for (uint32_t i = 1; i < slots_.size(); ++i)
      if (slots_[i].treelet_gid >= 0) slots_[i].visibility = -1;
  }
  // After an analysis step that placed nothing, the steps that follow for
  // the same view see the same pool and repeat it, except that treelets the
  // view does not see count down towards eviction.  This jumps to the end of
  // that countdown (every treelet the last step did not see becomes
  // invisible at once) and returns whether that changed any slot; false
  // means the treelets the view sees fill the pool and no further step can
  // place anything.
  bool expire_unseen() {
    bool changed = false;
    for (uint32_t i = 1; i < slots_.size(); ++i)
      if (slots_[i].treelet_gid >= 0 && slots_[i].visibility >= 0 &&
          slots_[i].visibility < kMaxVisibility) {
        slots_[i].visibility = -1;
        changed = true;
      }
    return changed;
  }
  // freeIncorePosition evicts a treelet only when it and its parent are both
  // invisible (src/TreeletMemoryManager.cpp:571-579); since the root's slot
  // never ages, the root's own sub-treelets then stay for good.  With `any`
  // set, an invisible treelet goes whatever its parent's visibility (its
  // subtree with it), so that a small region serving views that jump across
  // the octree can always make room.  Off by default (the reference's rule).
  void set_evict_any_invisible(bool any) { evict_any_invisible_ = any; }

  // Slot ranges the reference's updateDeviceMemory would copy
  // (TreeletMemoryManagerCl.cpp:177-236), as (first slot, slot count).  A
  // range keeps growing over the next dirty slot while (treelets + 1) /
  // (slot distance + 1) >= 2 * ratio; the reference hard-codes ratio 0.6,
  // ratio 1 copies every slot alone, ratio 0 one range over all dirty slots.
  std::vector<std::pair<uint32_t, uint32_t>> upload_ranges() const;
  // 0 <= ratio <= 1 (a larger ratio would stop the reference's loop from
  // advancing).
  int set_upload_ratio(float ratio);
  float upload_ratio() const { return upload_ratio_; }

 protected:
  // Called before the host mirror changes, so uploads still reading it
  // (none with the staging ring) can finish first.
  virtual void before_host_write() {}
  void mark_upload(uint32_t slot) { upload_.insert(slot); }

  svo_scene scene_;
  uint32_t N_ = 0;
  svo_node* incore_ = nullptr;
  svo_attrib* incore_attr_ = nullptr;
  std::vector<SlotInfo> slots_;
  std::vector<int32_t> slot_of_;
  std::vector<std::set<int32_t>> children_;
  std::vector<uint32_t> free_;  // top = back()
  std::set<uint32_t> upload_;
  uint32_t search_pos_ = 1;
  float upload_ratio_ = 0.6f;
  bool evict_any_invisible_ = false;
  uint32_t max_new_ = 0;
  uint32_t last_requested_ = 0;

  // Deferred slot bodies.  update_client_side places many treelets at once;
  // copying each one's records into the host mirror as it is placed made the
  // copies (about 200 KB a treelet) run one after another on one thread.
  // While deferring, a placed treelet's body is copied at the end of the
  // update, all bodies in parallel; the leaf patches and restores aimed at a
  // slot whose body is still pending are kept in order and applied after
  // it, and a pending slot that is evicted or freed during the update is
  // completed on the spot first.  The mirror then ends up exactly as with
  // immediate copies.
  struct LeafWrite {
    uint64_t leaf, leaf_parent;
    svo_node value;
    uint32_t bit;
    bool set;  // set the leaf flag (a restore) or clear it (a patch)
  };
  void begin_deferred();
  void end_deferred();
  void copy_body(uint32_t slot, int32_t gid);
  void complete_pending(uint32_t slot);
  void write_leaf(uint32_t pslot, const LeafWrite& w);
  bool defer_ = false;
  std::vector<int32_t> pending_gid_;                // per slot: gid whose body is pending, or -1
  std::vector<std::vector<LeafWrite>> pending_ops_;  // per slot: writes after that body
  std::vector<uint32_t> pending_slots_;
};

class TreeletMemoryManagerCuda : public TreeletMemoryManager {
 public:
  explicit TreeletMemoryManagerCuda(cudaStream_t render_stream) : render_stream_(render_stream) {}
  ~TreeletMemoryManagerCuda() override;

  int init_device_buffer();                         // initClBuffer
  // Uses caller-owned device buffers of incore_nodes() records each instead
  // of allocating, and uploads the whole incore buffer into them.
  int attach_device_buffers(svo_node* d_nodes, svo_attrib* d_attribs);
  // Forgets attached buffers (after waiting for uploads into them).
  int detach_device_buffers();
  int update_device_memory(uint32_t* copy_calls);   // updateDeviceMemory
  // SVO_UPLOAD_COALESCED: the reference's slot ranges (upload_ranges), each
  // staged through the pinned ring.  SVO_UPLOAD_PACKED: only the dirty slots,
  // packed back to back into the pinned ring, one host-to-device copy per
  // 4 MB chunk, and a scatter kernel that moves each slot to its place.
  // SVO_UPLOAD_PINNED: the mirror itself is page-locked and mapped; one
  // kernel reads the dirty slots from it over PCIe and writes them in place,
  // and whole-pool uploads (init_device_buffer, attach_device_buffers) are
  // two DMA copies straight from it.
  int set_upload_policy(int policy);
  int upload_policy() const { return upload_policy_; }
  int reset_incore_buffer() override;

  const svo_node* device_nodes() const { return d_nodes_; }
  const svo_attrib* device_attribs() const { return d_attribs_; }
  bool device_ready() const { return d_nodes_ != nullptr; }
  cudaStream_t render_stream() const { return render_stream_; }
  svo_stats* device_stats() const { return d_stats_; }
  uint64_t device_bytes() const { return device_bytes_; }

  // Orders work on `stream` after the pending uploads.
  int wait_uploads(cudaStream_t stream);
  // Device RGBA scratch for host-output renders (grown on demand).
  int rgba_scratch(uint64_t pixels, uint32_t** out);
  // Asynchronous host-output frames: cast on `stream` into one of two device
  // images, copied to `h_rgba` on a second stream, so the copy of a frame
  // overlaps the cast of the next.  wait_host_frames() blocks until every
  // copy issued so far has landed.  With `shadow` the frame is the primary +
  // shadow ray frame (launch_render_shadow) instead of renderToBuffer's.
  int render_to_host_async(const svo_frame_params& p, const svo_trace_cfg& cfg, uint32_t* h_rgba,
                           cudaStream_t stream, const svo_shadow_cfg* shadow = nullptr);
  int wait_host_frames();
  // Device feedback-record scratch for analysis passes (grown on demand).
  int feedback_scratch(uint64_t records, svo_feedback** out);
  // analyse_feedback over n records in device memory: the records are folded
  // on the GPU into per-treelet largest-error arrays (launch_analyse) and
  // only those come back, 4 bytes per treelet each.  Same lists and statuses
  // as analyse_feedback on the same records.  Blocks until the lists are on
  // the host.
  int analyse_feedback_device(const svo_feedback* d_fb, uint64_t n, uint32_t max_new,
                              std::vector<std::pair<int32_t, float>>& out_new,
                              std::vector<std::pair<int32_t, float>>& out_old,
                              cudaStream_t stream);
  // One dynamic-loading step of the reference's frame loop
  // (raycast_serialized_opencl.cpp:684-716; RenderPassAnalyse::
  // performAnalysePass, src/RenderPassAnalyse.cpp:150-369): the analysis
  // rays over `frame` at 1/divisor resolution with the far plane jittered by
  // (jitter_x, jitter_y) * divisor / 2 frame pixels, the records analysed on
  // the GPU, treelets inserted (new ones that find no slot are skipped, as
  // the reference ignores its insertion results) and the dirty slots
  // uploaded.  *num_new: treelets placed; *num_old: visible resident ones;
  // *num_requested (optional): newly visible treelets the pass asked for,
  // placed or not (0 once the view needs nothing that is not resident).
  int analysis_step(const svo_frame_params& frame, uint32_t divisor, float jitter_x,
                    float jitter_y, int32_t stack_size, cudaStream_t stream, uint32_t* num_new,
                    uint32_t* num_old, uint32_t* num_requested = nullptr);
  // The same step in two halves, so that the analysis of the next view can
  // run beside the frame still being cast: begin launches the analysis rays
  // and the fold on `stream` (after this manager's pending uploads) and
  // returns; end waits for them, inserts and evicts on the host and uploads
  // the dirty slots once the work already queued on `after` (the frame
  // reading the pool) is done.  Nothing may change the slots in between.
  // analysis_step(..., s, ...) is analysis_begin(..., s) + analysis_end(s, ...).
  int analysis_begin(const svo_frame_params& frame, uint32_t divisor, float jitter_x,
                     float jitter_y, int32_t stack_size, cudaStream_t stream);
  int analysis_end(cudaStream_t after, uint32_t* num_new, uint32_t* num_old,
                   uint32_t* num_requested = nullptr);
  // A begun analysis step not yet ended (the slots must not change).
  bool analysis_pending() const { return analysis_pending_; }

 private:
  int init_analysis();
  // the device fold of analyse_feedback_device, launched on `stream` (keys
  // copied back asynchronously), and the reading of its keys once done
  int launch_fold(const svo_feedback* d_fb, uint64_t n, cudaStream_t stream);
  int read_fold(uint32_t max_new, std::vector<std::pair<int32_t, float>>& out_new,
                std::vector<std::pair<int32_t, float>>& out_old);
  bool analysis_pending_ = false;
  cudaEvent_t analysis_done_ = nullptr;
  cudaEvent_t after_done_ = nullptr;
  // One host-to-device copy through the pinned ring.
  struct StagedCopy {
    void* dst;
    const void* src;
    uint64_t bytes;
  };
  // The copies, in order, through the pinned ring, in pieces of at most one
  // half: each piece waits for its half's previous copy, is copied into it
  // (on several host threads from 4 MB up) and goes out with one
  // cudaMemcpyAsync, so its transfer overlaps the host copy of the next.
  int stage_copies(const std::vector<StagedCopy>& copies);
  int upload_packed(uint32_t* copy_calls);
  void before_host_write() override;
  int init_transfer();
  int upload_all();

  cudaStream_t render_stream_ = nullptr;
  cudaStream_t copy_stream_ = nullptr;
  cudaEvent_t upload_done_ = nullptr;
  bool upload_pending_ = false;
  svo_node* d_nodes_ = nullptr;
  svo_attrib* d_attribs_ = nullptr;
  bool owns_device_ = false;
  svo_stats* d_stats_ = nullptr;
  uint64_t device_bytes_ = 0;
  static constexpr uint64_t kStageBytes = 32ull << 20;  // per half of the ring
  void* stage_[2] = {nullptr, nullptr};
  cudaEvent_t stage_evt_[2] = {nullptr, nullptr};
  // packed uploads: device halves of the ring and the slot ids of each half
  void* d_stage_[2] = {nullptr, nullptr};
  uint32_t* h_ids_[2] = {nullptr, nullptr};
  uint32_t* d_ids_[2] = {nullptr, nullptr};
  int upload_policy_ = SVO_UPLOAD_COALESCED;
  bool mirror_pinned_ = false;  // incore_ / incore_attr_ registered with CUDA
  const svo_node* mapped_nodes_ = nullptr;     // their device-side addresses
  const svo_attrib* mapped_attribs_ = nullptr;
  uint32_t* h_slot_ids_ = nullptr;             // page-locked, mapped
  const uint32_t* mapped_slot_ids_ = nullptr;
  int stage_next_ = 0;
  uint32_t* d_rgba_ = nullptr;
  uint64_t d_rgba_pixels_ = 0;
  // asynchronous host-output frames
  uint32_t* d_img_[2] = {nullptr, nullptr};
  uint64_t d_img_pixels_[2] = {0, 0};
  cudaStream_t d2h_stream_ = nullptr;
  cudaEvent_t cast_done_[2] = {nullptr, nullptr};
  cudaEvent_t copy_done_[2] = {nullptr, nullptr};
  int img_next_ = 0;
  svo_feedback* d_feedback_ = nullptr;
  uint64_t d_feedback_records_ = 0;
  // device analysis: the slot -> gid table (refreshed per pass through a
  // page-locked copy), treelet parents, and the key arrays
  // [new: T + 1 | old: T + 1 | status] with their page-locked host copy
  int32_t* d_slot_gid_ = nullptr;
  int32_t* h_slot_gid_ = nullptr;
  int32_t* d_parent_ = nullptr;
  uint32_t* d_keys_ = nullptr;
  uint32_t* h_keys_ = nullptr;
};

}  // namespace svo
