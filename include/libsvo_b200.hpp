/*
 * libsvo_b200.hpp -- C++ drop-in for the reference's TreeletMemoryManagerCl.
 *
 * A header-only class over the C ABI (libsvo_b200.h) with the method names
 * of svo::TreeletMemoryManager / svo::TreeletMemoryManagerCl
 * (src/TreeletMemoryManager.h:97-157, src/TreeletMemoryManagerCl.h:64-109),
 * so that an application written against the OpenCL manager switches by
 * changing the class name and the two buffer getters:
 *
 *   reference                               here
 *   TreeletMemoryManagerCl(path, bytes, ctx) TreeletMemoryManagerCuda(path, bytes, stream)
 *   initClBuffer()                          initDeviceBuffer()
 *   getClIncoreBufferGid()                  getDeviceIncoreBuffer()      (device pointer)
 *   getClAttributeIncoreBufferGid()         getDeviceAttributeBuffer()   (device pointer)
 *   setKernelArg*(renderToBuffer) + enqueue renderToBuffer(params, d_rgba, ...)
 *
 * Every other method keeps its reference name and argument meaning.  The
 * differences are stated at each method: the host incore buffers come back
 * as copies (the reference hands out references to its vectors), the
 * reference's RenderPassAnalyse* argument is replaced by the analysis lists
 * it carries, and errors are reported (the reference prints to std::cerr or
 * calls exit(0)): the constructor throws svo::Error, and methods that
 * returned void in the reference return bool here.  Include after the CUDA
 * runtime header if cudaStream_t is to be passed (any pointer converts).
 */
#ifndef LIBSVO_B200_HPP
#define LIBSVO_B200_HPP

#include <cstdint>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "libsvo_b200.h"

namespace svo {

// A failed call: the library's status code and its last CUDA error string.
class Error : public std::runtime_error {
 public:
  Error(const std::string& what, int status)
      : std::runtime_error(what + ": status " + std::to_string(status) + " " + svo_last_error()),
        status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

class TreeletMemoryManagerCuda {
 public:
  // TreeletMemoryManager::SlotInfo (src/TreeletMemoryManager.h:72-89), with
  // the reference's field names and defaults.
  struct SlotInfo {
    SlotInfo() : _treeletGid(-1), _visibility(0), _error(100000.0f) {}
    SlotInfo(int treeletGid, int visibility, float error)
        : _treeletGid(treeletGid), _visibility(visibility), _error(error) {}
    int _treeletGid;
    int _visibility;
    float _error;
  };

  // The lists RenderPassAnalyse hands to updateClientSideIncoreBuffer
  // (src/RenderPassAnalyse.cpp:218-356): newly visible treelets with their
  // errors, largest first, and the visible resident treelets.
  struct AnalysisLists {
    std::vector<int32_t> newGids;
    std::vector<float> newErrors;
    std::vector<int32_t> oldGids;
  };

  // TreeletMemoryManagerCl(svoFilePath, incoreBufferSizeInByte, clContext):
  // loads <svoFilePath>.svo / .ia and resets the incore buffer.  `stream`
  // (a cudaStream_t, or nullptr for the legacy default stream) takes the
  // place of the ClContext: renders run on it, uploads on a side stream
  // ordered by events.  Throws svo::Error where the reference exit(0)s.
  TreeletMemoryManagerCuda(const std::string& svoFilePath, uint64_t incoreBufferSizeInByte,
                           void* stream = nullptr) {
    check(svo_mm_create(svoFilePath.c_str(), incoreBufferSizeInByte, stream, &mm_), "svo_mm_create");
  }
  // The same over an in-memory scene (copied).
  TreeletMemoryManagerCuda(const svo_scene* scene, uint64_t incoreBufferSizeInByte,
                           void* stream = nullptr) {
    check(svo_mm_create_from_scene(scene, incoreBufferSizeInByte, stream, &mm_),
          "svo_mm_create_from_scene");
  }
  ~TreeletMemoryManagerCuda() {
    if (mm_) svo_mm_destroy(mm_);
  }
  TreeletMemoryManagerCuda(const TreeletMemoryManagerCuda&) = delete;
  TreeletMemoryManagerCuda& operator=(const TreeletMemoryManagerCuda&) = delete;
  TreeletMemoryManagerCuda(TreeletMemoryManagerCuda&& o) noexcept : mm_(std::exchange(o.mm_, nullptr)) {}
  TreeletMemoryManagerCuda& operator=(TreeletMemoryManagerCuda&& o) noexcept {
    if (this != &o) {
      if (mm_) svo_mm_destroy(mm_);
      mm_ = std::exchange(o.mm_, nullptr);
    }
    return *this;
  }

  // initClBuffer (src/TreeletMemoryManagerCl.cpp:101-113): allocates the
  // device node and attribute buffers and uploads the incore buffer.
  void initDeviceBuffer() { check(svo_mm_init_device_buffer(mm_), "svo_mm_init_device_buffer"); }
  // getClIncoreBufferGid / getClAttributeIncoreBufferGid: device pointers.
  const svo_node* getDeviceIncoreBuffer() const { return buffers().nodes; }
  const svo_attrib* getDeviceAttributeBuffer() const { return buffers().attribs; }
  uint64_t getDeviceIncoreBufferSize() const { return buffers().count; }

  unsigned getTreeletSizeInByte() const { return info().treelet_bytes; }
  unsigned getNumNodesPerTreelet() const { return info().nodes_per_treelet; }
  unsigned getNumTreelets() const { return info().num_treelets; }

  // getIncoreBuffer / getAttributeIncoreBuffer: copies of the host mirror.
  std::vector<svo_node> getIncoreBuffer() const {
    std::vector<svo_node> v(info().incore_nodes);
    check(svo_mm_copy_incore(mm_, 0, v.size(), v.data(), nullptr), "svo_mm_copy_incore");
    return v;
  }
  std::vector<svo_attrib> getAttributeIncoreBuffer() const {
    std::vector<svo_attrib> v(info().incore_nodes);
    check(svo_mm_copy_incore(mm_, 0, v.size(), nullptr, v.data()), "svo_mm_copy_incore");
    return v;
  }

  // updateClientSideIncoreBuffer(RenderPassAnalyse*)
  // (src/TreeletMemoryManager.cpp:393-443) with the analysis lists passed
  // directly.  Returns false when a treelet could not be placed (the
  // reference ignores that; the next analysis asks again).
  bool updateClientSideIncoreBuffer(const AnalysisLists& a) {
    if (a.newGids.size() != a.newErrors.size()) return false;
    return svo_mm_update_client_side(mm_, a.newGids.data(), a.newErrors.data(),
                                     (uint32_t)a.newGids.size(), a.oldGids.data(),
                                     (uint32_t)a.oldGids.size()) == SVO_OK;
  }
  // RenderPassAnalyse::performAnalysePass plus updateClientSideIncoreBuffer
  // and updateDeviceMemory: one dynamic-loading step of the reference's frame
  // loop (raycast_serialized_opencl.cpp:684-716) for `frame` at
  // 1/`divisor` resolution.  Returns the number of treelets placed.
  uint32_t performAnalysePass(const svo_frame_params& frame, uint32_t divisor = 8,
                              float jitterX = 0.0f, float jitterY = 0.0f, int32_t stackSize = 13,
                              void* stream = nullptr, uint32_t* numVisibleResident = nullptr) {
    uint32_t placed = 0, old = 0;
    check(svo_mm_analysis_step(mm_, &frame, divisor, jitterX, jitterY, stackSize, stream, &placed, &old),
          "svo_mm_analysis_step");
    if (numVisibleResident) *numVisibleResident = old;
    return placed;
  }

  // performAnalysePass in two halves (no reference counterpart): begin
  // launches the analysis on `stream`; end places and evicts, then uploads
  // after the work queued on `afterStream`.  Begun for view k+1 before frame
  // k is cast on another stream and ended after, the step runs beside that
  // frame and the frames are those of the sequential loop.
  void beginAnalysePass(const svo_frame_params& frame, uint32_t divisor = 8, float jitterX = 0.0f,
                        float jitterY = 0.0f, int32_t stackSize = 13, void* stream = nullptr) {
    check(svo_mm_analysis_begin(mm_, &frame, divisor, jitterX, jitterY, stackSize, stream),
          "svo_mm_analysis_begin");
  }
  uint32_t endAnalysePass(void* afterStream = nullptr, uint32_t* numVisibleResident = nullptr) {
    uint32_t placed = 0, old = 0;
    check(svo_mm_analysis_end(mm_, afterStream, &placed, &old), "svo_mm_analysis_end");
    if (numVisibleResident) *numVisibleResident = old;
    return placed;
  }

  // insertTreeletIntoIncoreBuffer (src/TreeletMemoryManager.cpp:456-548).
  bool insertTreeletIntoIncoreBuffer(const SlotInfo& tve) {
    return svo_mm_insert_treelet(mm_, tve._treeletGid, tve._visibility, tve._error) == SVO_OK;
  }
  // removeTreeletFromIncoreBuffer (src/TreeletMemoryManager.cpp:666-700).
  bool removeTreeletFromIncoreBuffer(int treeletGid) {
    return svo_mm_remove_treelet(mm_, treeletGid) == SVO_OK;
  }
  // freeIncorePosition (src/TreeletMemoryManager.cpp:561-653); the
  // reference does not read its argument either.
  bool freeIncorePosition(const SlotInfo& = SlotInfo()) {
    return svo_mm_free_incore_position(mm_) == SVO_OK;
  }

  // updateDeviceMemory (src/TreeletMemoryManagerCl.cpp:155-251): the dirty
  // slots as asynchronous copies; renders issued afterwards wait for them.
  // *numCopyCalls (optional) receives the number of copies.
  bool updateDeviceMemory(uint32_t* numCopyCalls = nullptr) {
    return svo_mm_update_device_memory(mm_, numCopyCalls) == SVO_OK;
  }
  // resetIncoreBuffer (src/TreeletMemoryManager.cpp:304-380).
  bool resetIncoreBuffer() { return svo_mm_reset(mm_) == SVO_OK; }

  // getFreeIncoreSlotStack().size(): the number of free slots.
  unsigned getNumFreeIncoreSlots() const { return info().free_slots; }
  // getIncoreSlotsToUpload (src/TreeletMemoryManager.h:153).
  std::set<int> getIncoreSlotsToUpload() const {
    std::vector<uint32_t> v(info().slots_to_upload);
    uint32_t n = 0;
    check(svo_mm_slots_to_upload(mm_, v.data(), (uint32_t)v.size(), &n), "svo_mm_slots_to_upload");
    return std::set<int>(v.begin(), v.begin() + n);
  }
  // getSlots (src/TreeletMemoryManager.h:157): a copy, one SlotInfo per slot.
  std::vector<SlotInfo> getSlots() const {
    const uint32_t n = info().num_slots;
    std::vector<SlotInfo> v(n);
    for (uint32_t i = 0; i < n; ++i) {
      svo_slot_info s;
      check(svo_mm_get_slot(mm_, i, &s), "svo_mm_get_slot");
      v[i] = SlotInfo(s.treelet_gid, s.visibility, s.error);
    }
    return v;
  }
  // Treelet::getSlotGid for a gid: its slot, or -1 when not resident.
  int getTreeletSlotGid(int treeletGid) const {
    int32_t slot = -1;
    check(svo_mm_treelet_slot(mm_, treeletGid, &slot), "svo_mm_treelet_slot");
    return slot;
  }

  // The renderToBuffer launch (setKernelArg* + enqueueKernel,
  // raycast_serialized_opencl.cpp:729-747) over the incore buffer, after
  // pending uploads; asynchronous on `stream`.
  bool renderToBuffer(const svo_frame_params& params, uint32_t* d_rgba, svo_hit* d_hits = nullptr,
                      void* stream = nullptr, int32_t stackSize = 13) {
    svo_trace_cfg cfg;
    cfg.traversal = SVO_TRAVERSAL_TREELET;
    cfg.stack_size = stackSize;
    return svo_mm_render(mm_, &params, &cfg, d_rgba, d_hits, stream) == SVO_OK;
  }
  // The blocking form with the image read back to host memory.
  bool renderToHostBuffer(const svo_frame_params& params, uint32_t* h_rgba, void* stream = nullptr,
                          int32_t stackSize = 13) {
    svo_trace_cfg cfg;
    cfg.traversal = SVO_TRAVERSAL_TREELET;
    cfg.stack_size = stackSize;
    return svo_mm_render_host(mm_, &params, &cfg, h_rgba, stream) == SVO_OK;
  }
  // Frame loops: the image of each call lands in h_rgba (page-locked) by the
  // next sync(); its copy overlaps the next call's cast.  With `shadow`, the
  // primary + shadow ray frame.
  bool renderToHostBufferAsync(const svo_frame_params& params, uint32_t* h_rgba,
                               const svo_shadow_cfg* shadow = nullptr, void* stream = nullptr,
                               int32_t stackSize = 13) {
    svo_trace_cfg cfg;
    cfg.traversal = SVO_TRAVERSAL_TREELET;
    cfg.stack_size = stackSize;
    return (shadow ? svo_mm_render_shadow_host_async(mm_, &params, &cfg, shadow, h_rgba, stream)
                   : svo_mm_render_host_async(mm_, &params, &cfg, h_rgba, stream)) == SVO_OK;
  }
  // Waits for `stream` and returns the watchdog and bounds counters of the
  // renders since the last call.
  svo_stats sync(void* stream = nullptr) {
    svo_stats s;
    check(svo_mm_sync(mm_, stream, &s), "svo_mm_sync");
    return s;
  }

  svo_mm* handle() const { return mm_; }

 private:
  struct Buffers {
    const svo_node* nodes;
    const svo_attrib* attribs;
    uint64_t count;
  };
  static void check(int rc, const char* what) {
    if (rc != SVO_OK) throw Error(what, rc);
  }
  svo_mm_info info() const {
    svo_mm_info i;
    check(svo_mm_info_get(mm_, &i), "svo_mm_info_get");
    return i;
  }
  Buffers buffers() const {
    Buffers b{nullptr, nullptr, 0};
    check(svo_mm_get_device_buffers(mm_, &b.nodes, &b.attribs, &b.count), "svo_mm_get_device_buffers");
    return b;
  }
  svo_mm* mm_ = nullptr;
};

}  // namespace svo

#endif  // LIBSVO_B200_HPP
