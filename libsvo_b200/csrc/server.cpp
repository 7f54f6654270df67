// server.cpp -- request loop over resident octrees (svo_server_* in the C ABI).
//
// The reference pages treelets of one octree per frame, driven by its
// analysis pass, and renders one frame per kernel (src/TreeletMemoryManager.cpp:
// 393-548, raycast_serialized_opencl.cpp:680-747).  The server turns that
// into a request loop: clients submit cast requests (an octree and a camera)
// at any time; a dispatcher thread admits them against an HBM budget and an
// in-flight ray budget, pages the treelets of their octrees into one
// pre-allocated device pool (the octree's TreeletMemoryManagerCuda uploads
// its slots through its pinned staging ring on its side stream -- or, once
// svo_server_set_upload_policy page-locked its host copy, as two DMA copies
// straight from it -- and the launch waits on the upload event), and
// launches every admitted request
// together as one batch on the next free stream.  Requests that arrive while
// batches run are launched in further batches on other streams, so their
// work overlaps on the device (continuous batching).  Octrees no batch uses
// are evicted least recently used first when the pool is full.  A host
// callback on each batch's stream timestamps completion.
//
// An octree whose pools exceed the budget (or one registered with
// svo_server_add_octree_paged) is not made resident whole: it keeps a fixed
// region of treelet slots in the pool and a worker thread of its own, which
// serves its requests one by one, each after analysis passes over the
// request's view at full resolution until no new treelet is placed
// (treelets paged in and out of the region by visibility, the reference's
// out-of-core loop), so a request whose visible treelets fit the region gets
// the image of the fully resident octree.
//
// In SVO_SERVE_PLAIN mode the same loop launches the per-frame kernel once
// per request on a single stream instead: the plain baseline.  In
// SVO_SERVE_PLAIN_STREAMED mode the dispatcher launches each admitted
// request's per-frame kernel at once, round robin over `streams` streams,
// with no launch slots and no host callback: a CUDA event recorded after
// each launch is polled for its completion (the ungated plain baseline).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <system_error>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/libsvo_b200.h"
#include "errors.h"
#include "memory_manager.h"
#include "render.h"
#include "scene.h"

namespace {

using Clock = std::chrono::steady_clock;

// First-fit allocator over one device allocation; offsets aligned to 256 B.
class DevicePool {
 public:
  int init(uint64_t bytes) {
    size_ = bytes & ~255ull;
    if (size_ == 0) return SVO_ERR_RANGE;
    SVO_CUDA_TRY(cudaMalloc(&base_, size_));
    free_.clear();
    free_[0] = size_;
    return SVO_OK;
  }
  ~DevicePool() { cudaFree(base_); }
  bool alloc(uint64_t bytes, uint64_t* off) {
    bytes = (bytes + 255) & ~255ull;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      *off = it->first;
      const uint64_t rest = it->second - bytes, start = it->first + bytes;
      free_.erase(it);
      if (rest) free_[start] = rest;
      return true;
    }
    return false;
  }
  void release(uint64_t off, uint64_t bytes) {
    bytes = (bytes + 255) & ~255ull;
    auto it = free_.emplace(off, bytes).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
      it->second += next->second;
      free_.erase(next);
    }
    if (it != free_.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == it->first) {
        prev->second += it->second;
        free_.erase(it);
      }
    }
  }
  char* base() const { return static_cast<char*>(base_); }
  uint64_t size() const { return size_; }

 private:
  void* base_ = nullptr;
  uint64_t size_ = 0;
  std::map<uint64_t, uint64_t> free_;
};

// Serves the requests of one treelet-paged octree, in arrival order.
struct PagedWorker {
  std::thread thread;
  cudaStream_t stream = nullptr;
  std::deque<uint64_t> queue;  // tickets, guarded by the server's mutex
  std::condition_variable cv;
  bool stop = false;
};

struct ServedOctree {
  std::unique_ptr<svo::TreeletMemoryManagerCuda> mm;
  int32_t stack_size = 13;
  uint64_t node_bytes = 0;  // per pool (nodes, then attributes)
  bool resident = false;
  uint64_t pool_off = 0;
  uint32_t refs = 0;  // batches in flight that read it
  uint64_t last_use = 0;
  bool paged = false;  // a fixed region of slots, paged by its worker
  std::unique_ptr<PagedWorker> worker;
};

// Analysis passes before a paged request gives up converging and renders
// with what is resident.
constexpr uint32_t kMaxPagingSteps = 64;
// A request also stops paging once it has placed this many times its
// region's slots: a view whose treelets fit is placed once (treelets of
// earlier views go first, its own stay marked visible while it converges),
// so beyond that the view is swapping its own treelets in and out.
constexpr uint32_t kMaxRegionRefills = 2;

struct Request {
  svo_request r{};
  svo_request_result res{};
  bool done = false;
};

struct Launch;

}  // namespace

struct svo_server {
  svo_server_cfg cfg{};
  Clock::time_point t0;
  DevicePool pool;
  std::vector<ServedOctree> octrees;

  std::mutex mu;  // pending, requests, results, octree table
  std::condition_variable cv_user;
  std::condition_variable cv_dispatch;
  std::deque<uint64_t> pending;
  std::unordered_map<uint64_t, Request> requests;
  uint64_t next_ticket = 1;
  bool stop = false;
  int fatal = SVO_OK;

  struct Slot {
    cudaStream_t stream = nullptr;
    svo_batcher* batcher = nullptr;
    bool busy = false;
    std::vector<uint64_t> tickets;
    std::vector<uint32_t> octrees;  // octree ids pinned by this launch
    uint64_t rays = 0;
    double done_s = 0.0;            // written by the stream callback
    svo_server* owner = nullptr;
    uint32_t index = 0;
  };
  std::vector<Slot> slots;
  std::mutex cmu;  // completion queue (the only lock stream callbacks take)
  std::deque<uint32_t> completed;
  std::atomic<uint32_t> completions{0};
  // Host callbacks launched and callbacks past their last access to this
  // object; the server is freed only once both agree.
  std::atomic<uint64_t> callbacks_launched{0};
  std::atomic<uint64_t> callbacks_exited{0};

  // SVO_SERVE_PLAIN_STREAMED: launches in flight, each with the event
  // recorded after it, and recycled events
  struct Streamed {
    uint64_t ticket;
    cudaEvent_t done;
    uint32_t octree;
    uint64_t rays;
  };
  std::vector<Streamed> streamed;
  std::vector<cudaEvent_t> spare_events;
  uint32_t next_stream = 0;

  uint64_t inflight_rays = 0;
  bool blocked = false;  // admission stopped on a limit; cleared by completions
  uint64_t use_clock = 0;
  uint32_t batch_seq = 0;
  svo_server_stats stats{};
  std::thread dispatcher;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

void CUDART_CB on_slot_done(void* p) {
  auto* slot = static_cast<svo_server::Slot*>(p);
  svo_server* s = slot->owner;
  slot->done_s = s->now();
  {
    std::lock_guard<std::mutex> lk(s->cmu);
    s->completed.push_back(slot->index);
    s->completions.fetch_add(1);
  }
  s->cv_dispatch.notify_one();
  s->callbacks_exited.fetch_add(1, std::memory_order_release);  // last access to *s
}

// Makes octree `id` resident, evicting idle octrees if the pool is full.
// Called by the dispatcher with `mu` held.
// Allocates `need` bytes of the pool, evicting idle whole-resident octrees
// (least recently used first, never `keep` or a paged octree's region).
// Called with `mu` held.
int alloc_evicting(svo_server* s, uint64_t need, int keep, uint64_t* off) {
  while (!s->pool.alloc(need, off)) {
    int victim = -1;
    bool in_flight = false;  // an octree pinned by running work will free up later
    for (uint32_t i = 0; i < s->octrees.size(); ++i) {
      const ServedOctree& c = s->octrees[i];
      if ((int)i == keep || c.paged || !c.resident) continue;
      if (c.refs) {
        in_flight = true;
        continue;
      }
      if (victim < 0 || c.last_use < s->octrees[victim].last_use) victim = (int)i;
    }
    // nothing to evict and nothing that will be released: the space is held
    // by paged regions for good, so waiting would not help
    if (victim < 0) return (need > s->pool.size() || !in_flight) ? SVO_ERR_RANGE : SVO_ERR_BUSY;
    ServedOctree& v = s->octrees[victim];
    int rc = v.mm->detach_device_buffers();
    if (rc != SVO_OK) return rc;
    s->pool.release(v.pool_off, 2 * ((v.node_bytes + 255) & ~255ull));
    v.resident = false;
    s->stats.octree_evictions++;
    s->stats.resident_octrees--;
    s->stats.resident_bytes -= 2 * v.node_bytes;
  }
  return SVO_OK;
}

int ensure_resident(svo_server* s, uint32_t id) {
  ServedOctree& o = s->octrees[id];
  o.last_use = ++s->use_clock;
  if (o.resident) return SVO_OK;
  const uint64_t need = 2 * ((o.node_bytes + 255) & ~255ull);
  uint64_t off = 0;
  const int arc = alloc_evicting(s, need, (int)id, &off);
  if (arc != SVO_OK) return arc;
  char* base = s->pool.base() + off;
  const uint64_t attr_off = (o.node_bytes + 255) & ~255ull;
  const int rc = o.mm->attach_device_buffers(reinterpret_cast<svo_node*>(base),
                                            reinterpret_cast<svo_attrib*>(base + attr_off));
  if (rc != SVO_OK) {
    s->pool.release(off, need);
    return rc;
  }
  o.pool_off = off;
  o.resident = true;
  s->stats.octree_loads++;
  s->stats.treelets_paged_in += o.mm->num_treelets();
  s->stats.bytes_uploaded += 2 * o.node_bytes;
  s->stats.resident_octrees++;
  s->stats.resident_bytes += 2 * o.node_bytes;
  return SVO_OK;
}

// A paged octree's worker: per request, analysis passes over the request's
// view at full resolution until a pass places no new treelet (at most
// kMaxPagingSteps), then the per-frame kernel, waited for on the worker's
// stream.
void paged_worker_loop(svo_server* s, uint32_t id) {
  PagedWorker* w = nullptr;
  svo::TreeletMemoryManagerCuda* mm = nullptr;
  int32_t S = 13;
  uint64_t slot_bytes = 0;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    w = s->octrees[id].worker.get();
    mm = s->octrees[id].mm.get();
    S = s->octrees[id].stack_size;
    slot_bytes = 2ull * mm->treelet_bytes();
  }
  for (;;) {
    uint64_t t = 0;
    svo_request r{};
    {
      std::unique_lock<std::mutex> lk(s->mu);
      w->cv.wait(lk, [&] { return w->stop || !w->queue.empty(); });
      if (w->stop) return;  // queued requests are cancelled by the destroyer
      t = w->queue.front();
      w->queue.pop_front();
      Request& q = s->requests[t];
      q.res.launch_s = s->now();
      q.res.batch = s->batch_seq++;
      s->stats.batches++;
      r = q.r;
    }
    uint32_t placed = 0;
    int rc = SVO_OK;
    bool converged = false;
    // a new view: what it does not see may make room at once
    mm->mark_all_unseen();
    const auto paging_start = std::chrono::steady_clock::now();
    uint32_t passes = 0;
    for (uint32_t step = 0; step < kMaxPagingSteps; ++step) {
      // converged when the pass asks for nothing new.  A pass that places
      // nothing leaves the pool as it was, so the next passes would repeat
      // it while the treelets this view does not see count down to
      // eviction: skip to the end of the countdown, or, when the view sees
      // every treelet of the region, stop (the view does not fit and is
      // cast from what is resident, coarser where treelets are missing)
      uint32_t nw = 0, old = 0, asked = 0;
      rc = mm->analysis_step(r.params, 1, 0.0f, 0.0f, S, w->stream, &nw, &old, &asked);
      if (rc != SVO_OK) break;
      ++passes;
      placed += nw;
      if (asked == 0) {
        converged = true;
        break;
      }
      if (nw == 0 && !mm->expire_unseen()) break;
      if (placed >= kMaxRegionRefills * mm->num_slots()) break;
    }
    if (rc == SVO_OK) rc = mm->wait_uploads(w->stream);
    if (rc == SVO_OK) rc = svo::cuda_status(cudaStreamSynchronize(w->stream));
    const uint64_t paging_us = (uint64_t)std::chrono::duration_cast<std::chrono::microseconds>(
                                   std::chrono::steady_clock::now() - paging_start)
                                   .count();
    if (rc == SVO_OK) {
      const svo_trace_cfg tc{SVO_TRAVERSAL_TREELET, S};
      rc = svo::launch_render(mm->device_nodes(), mm->device_attribs(), mm->incore_nodes(), r.params, tc,
                              r.d_rgba, nullptr, nullptr, w->stream);
    }
    if (rc == SVO_OK) rc = svo::cuda_status(cudaStreamSynchronize(w->stream));
    std::lock_guard<std::mutex> lk(s->mu);
    Request& q = s->requests[t];
    q.res.done_s = s->now();
    q.res.status = rc;
    q.done = true;
    s->stats.requests_done++;
    s->stats.rays_done += (uint64_t)r.params.width * r.params.height;
    s->stats.treelets_paged_in += placed;
    s->stats.bytes_uploaded += placed * slot_bytes;
    s->stats.analysis_passes += passes;
    s->stats.paging_us += paging_us;
    if (rc == SVO_OK && !converged) s->stats.paged_unconverged++;
    s->cv_user.notify_all();
  }
}

// Hands pending requests on paged octrees to their workers.  Called with
// `mu` held.
void route_paged(svo_server* s) {
  for (auto it = s->pending.begin(); it != s->pending.end();) {
    ServedOctree& o = s->octrees[s->requests[*it].r.octree];
    if (!o.paged) {
      ++it;
      continue;
    }
    o.worker->queue.push_back(*it);
    o.worker->cv.notify_one();
    it = s->pending.erase(it);
  }
}

void finish_slot(svo_server* s, svo_server::Slot& slot) {
  // called with mu held
  for (uint64_t t : slot.tickets) {
    auto it = s->requests.find(t);
    if (it == s->requests.end()) continue;
    it->second.res.done_s = slot.done_s;
    it->second.res.status = SVO_OK;
    it->second.done = true;
    s->stats.requests_done++;
  }
  for (uint32_t id : slot.octrees) s->octrees[id].refs--;
  s->inflight_rays -= slot.rays;
  s->stats.rays_done += slot.rays;
  slot.tickets.clear();
  slot.octrees.clear();
  slot.rays = 0;
  slot.busy = false;
}

// Launches the requests in `slot.tickets` (octrees already resident and pinned).
int launch_slot(svo_server* s, svo_server::Slot& slot) {
  const bool plain = s->cfg.mode == SVO_SERVE_PLAIN;
  std::vector<svo_octree_desc> descs;
  std::vector<uint32_t> remap(s->octrees.size(), UINT32_MAX);
  std::vector<svo_view_desc> views;
  for (uint32_t id : slot.octrees) {
    ServedOctree& o = s->octrees[id];
    int rc = o.mm->wait_uploads(slot.stream);
    if (rc != SVO_OK) return rc;
    remap[id] = (uint32_t)descs.size();
    descs.push_back(svo_octree_desc{o.mm->device_nodes(), o.mm->device_attribs(),
                                    o.mm->incore_nodes(), SVO_TRAVERSAL_TREELET, o.stack_size});
  }
  const double t_launch = s->now();
  for (uint64_t t : slot.tickets) {
    Request& q = s->requests[t];
    q.res.launch_s = t_launch;
    q.res.batch = s->batch_seq;
    svo_view_desc v{};
    v.params = q.r.params;
    v.octree = remap[q.r.octree];
    v.d_rgba = q.r.d_rgba;
    v.d_hits = nullptr;
    views.push_back(v);
  }
  s->batch_seq++;
  s->stats.batches++;
  if (plain) {
    for (const svo_view_desc& v : views) {
      const svo_octree_desc& d = descs[v.octree];
      const svo_trace_cfg tc{SVO_TRAVERSAL_TREELET, d.stack_size};
      const int rc = svo::launch_render(d.d_nodes, d.d_attribs, d.num_nodes, v.params, tc, v.d_rgba,
                                        nullptr, nullptr, slot.stream);
      if (rc != SVO_OK) return rc;
    }
  } else {
    const svo_batch_cfg bc{s->cfg.tile_w, s->cfg.tile_h, s->cfg.block_threads, 0, 0, 0};
    int rc = svo_batcher_set(slot.batcher, descs.data(), (uint32_t)descs.size(), views.data(),
                             (uint32_t)views.size(), &bc, slot.stream);
    if (rc != SVO_OK) return rc;
    rc = svo_batcher_launch(slot.batcher, nullptr, slot.stream);
    if (rc != SVO_OK) return rc;
  }
  SVO_CUDA_TRY(cudaLaunchHostFunc(slot.stream, on_slot_done, &slot));
  s->callbacks_launched.fetch_add(1);
  return SVO_OK;
}

void dispatch_loop(svo_server* s) {
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    s->cv_dispatch.wait_for(lk, std::chrono::microseconds(200), [&] {
      if (s->completions.load() > 0) return true;
      bool busy = false, idle = false;
      for (auto& sl : s->slots) (sl.busy ? busy : idle) = true;
      if (s->stop) return !busy;  // stopping: wake for completions or to exit
      return !s->pending.empty() && !s->blocked && idle;
    });
    // completions
    std::deque<uint32_t> done;
    {
      std::lock_guard<std::mutex> ck(s->cmu);
      done.swap(s->completed);
      s->completions.fetch_sub((uint32_t)done.size());
    }
    if (!done.empty()) {
      for (uint32_t i : done) finish_slot(s, s->slots[i]);
      s->blocked = false;
      s->cv_user.notify_all();
    }
    route_paged(s);
    bool busy_any = false;
    for (auto& sl : s->slots) busy_any |= sl.busy;
    if (s->stop && s->pending.empty() && !busy_any) return;
    if (s->fatal != SVO_OK) continue;
    // admit and launch while a stream is free
    for (;;) {
      if (s->pending.empty()) break;
      svo_server::Slot* slot = nullptr;
      for (auto& sl : s->slots)
        if (!sl.busy) {
          slot = &sl;
          break;
        }
      if (!slot) break;
      const uint32_t max_views = s->cfg.mode == SVO_SERVE_PLAIN ? 1u : s->cfg.max_batch_views;
      // Residency-aware admission, in arrival order within each pass:
      //  1. requests whose octree is resident (no paging needed);
      //  2. otherwise the oldest request: its octree is paged in (evicting
      //     idle octrees least recently used first), and pass 1 runs again
      //     so every pending request for that octree rides on the same load.
      // A request waiting longer than kMaxWait goes straight to step 2, so
      // no request starves behind a stream of requests on resident octrees.
      constexpr double kMaxWait = 0.05;
      auto admit = [&](std::deque<uint64_t>::iterator it) {
        const uint64_t t = *it;
        Request& q = s->requests[t];
        ServedOctree& o = s->octrees[q.r.octree];
        if (std::find(slot->octrees.begin(), slot->octrees.end(), q.r.octree) == slot->octrees.end()) {
          slot->octrees.push_back(q.r.octree);
          o.refs++;
        }
        slot->tickets.push_back(t);
        slot->rays += (uint64_t)q.r.params.width * q.r.params.height;
        return s->pending.erase(it);
      };
      auto fits = [&](const Request& q) {
        const uint64_t rays = (uint64_t)q.r.params.width * q.r.params.height;
        if (slot->tickets.size() >= max_views) return false;
        if (s->inflight_rays + slot->rays == 0) return true;  // always admit one
        return s->inflight_rays + slot->rays + rays <= s->cfg.max_inflight_rays;
      };
      auto admit_resident = [&] {
        for (auto it = s->pending.begin(); it != s->pending.end();) {
          const Request& q = s->requests[*it];
          if (!fits(q)) break;
          if (s->octrees[q.r.octree].resident) {
            s->octrees[q.r.octree].last_use = ++s->use_clock;
            it = admit(it);
          } else {
            ++it;
          }
        }
      };
      const bool starving =
          !s->pending.empty() && s->now() - s->requests[s->pending.front()].res.submit_s > kMaxWait;
      if (!starving) admit_resident();
      while (slot->tickets.empty() && !s->pending.empty()) {
        Request& q = s->requests[s->pending.front()];
        if (!fits(q)) break;
        const int rc = ensure_resident(s, q.r.octree);
        if (rc == SVO_ERR_BUSY) break;  // the pool is held by running batches: retry later
        if (rc != SVO_OK) {  // cannot ever fit, or a CUDA error
          s->pending.pop_front();
          q.res.status = rc;
          q.done = true;
          s->cv_user.notify_all();
          continue;
        }
        admit(s->pending.begin());
        admit_resident();
      }
      if (slot->tickets.empty()) {
        s->blocked = !s->pending.empty();  // wait for a completion before retrying
        break;
      }
      slot->busy = true;
      s->inflight_rays += slot->rays;
      const int rc = launch_slot(s, *slot);
      if (rc != SVO_OK) {
        s->fatal = rc;
        for (uint64_t t : slot->tickets) {
          s->requests[t].res.status = rc;
          s->requests[t].done = true;
        }
        for (uint32_t id : slot->octrees) s->octrees[id].refs--;
        s->inflight_rays -= slot->rays;
        slot->tickets.clear();
        slot->octrees.clear();
        slot->rays = 0;
        slot->busy = false;
        s->cv_user.notify_all();
        break;
      }
    }
  }
}

// SVO_SERVE_PLAIN_STREAMED: one per-frame kernel per request, launched as
// soon as the request is admitted (residency and the in-flight ray budget as
// in the other modes), round robin over the slots' streams; completions are
// found by polling the event recorded after each launch, every 20 us while
// launches are in flight.  Called with `mu` held by the dispatcher.
int streamed_launch(svo_server* s, uint64_t t) {
  Request& q = s->requests[t];
  ServedOctree& o = s->octrees[q.r.octree];
  svo_server::Slot& slot = s->slots[s->next_stream];
  s->next_stream = (s->next_stream + 1) % (uint32_t)s->slots.size();
  int rc = o.mm->wait_uploads(slot.stream);
  if (rc != SVO_OK) return rc;
  q.res.launch_s = s->now();
  q.res.batch = s->batch_seq++;
  s->stats.batches++;
  const svo_trace_cfg tc{SVO_TRAVERSAL_TREELET, o.stack_size};
  rc = svo::launch_render(o.mm->device_nodes(), o.mm->device_attribs(), o.mm->incore_nodes(),
                          q.r.params, tc, q.r.d_rgba, nullptr, nullptr, slot.stream);
  if (rc != SVO_OK) return rc;
  cudaEvent_t ev = nullptr;
  if (!s->spare_events.empty()) {
    ev = s->spare_events.back();
    s->spare_events.pop_back();
  } else {
    SVO_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  }
  const cudaError_t e = cudaEventRecord(ev, slot.stream);
  if (e != cudaSuccess) {
    s->spare_events.push_back(ev);
    return svo::cuda_status(e);
  }
  const uint64_t rays = (uint64_t)q.r.params.width * q.r.params.height;
  o.refs++;
  s->inflight_rays += rays;
  s->streamed.push_back(svo_server::Streamed{t, ev, q.r.octree, rays});
  return SVO_OK;
}

void dispatch_loop_streamed(svo_server* s) {
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    if (s->streamed.empty()) {
      s->cv_dispatch.wait_for(lk, std::chrono::microseconds(200), [&] {
        return s->stop || (!s->pending.empty() && !s->blocked);
      });
    } else {
      lk.unlock();
      std::this_thread::sleep_for(std::chrono::microseconds(20));
      lk.lock();
    }
    // completions, in any order
    bool any_done = false;
    for (size_t i = 0; i < s->streamed.size();) {
      svo_server::Streamed& f = s->streamed[i];
      const cudaError_t e = cudaEventQuery(f.done);
      if (e == cudaErrorNotReady) {
        ++i;
        continue;
      }
      Request& q = s->requests[f.ticket];
      q.res.done_s = s->now();
      q.res.status = e == cudaSuccess ? SVO_OK : svo::cuda_status(e);
      q.done = true;
      s->stats.requests_done++;
      s->stats.rays_done += f.rays;
      s->octrees[f.octree].refs--;
      s->inflight_rays -= f.rays;
      s->spare_events.push_back(f.done);
      f = s->streamed.back();
      s->streamed.pop_back();
      any_done = true;
    }
    if (any_done) {
      s->blocked = false;
      s->cv_user.notify_all();
    }
    route_paged(s);
    if (s->stop && s->pending.empty() && s->streamed.empty()) return;
    if (s->fatal != SVO_OK) continue;
    // admission in arrival order, requests on resident octrees first (as in
    // the batched mode); the oldest request pages its octree in when nothing
    // else can go, or when it has waited longer than 50 ms
    constexpr double kMaxWait = 0.05;
    auto fits = [&](const Request& q) {
      const uint64_t rays = (uint64_t)q.r.params.width * q.r.params.height;
      return s->inflight_rays == 0 || s->inflight_rays + rays <= s->cfg.max_inflight_rays;
    };
    bool launched = true;
    while (launched && !s->pending.empty()) {
      launched = false;
      const bool starving = s->now() - s->requests[s->pending.front()].res.submit_s > kMaxWait;
      if (!starving) {
        for (auto it = s->pending.begin(); it != s->pending.end();) {
          const Request& q = s->requests[*it];
          if (!fits(q)) break;
          if (!s->octrees[q.r.octree].resident) {
            ++it;
            continue;
          }
          s->octrees[q.r.octree].last_use = ++s->use_clock;
          const uint64_t t = *it;
          const int rc = streamed_launch(s, t);
          if (rc != SVO_OK) {
            s->fatal = rc;
            break;
          }
          it = s->pending.erase(it);
          launched = true;
        }
      }
      if (s->fatal != SVO_OK || s->pending.empty()) break;
      Request& q = s->requests[s->pending.front()];
      if (!fits(q)) break;
      const int rc = ensure_resident(s, q.r.octree);
      if (rc == SVO_ERR_BUSY) break;  // the pool is held by launches in flight
      if (rc != SVO_OK) {
        s->pending.pop_front();
        q.res.status = rc;
        q.done = true;
        s->cv_user.notify_all();
        launched = true;
        continue;
      }
      const int lrc = streamed_launch(s, s->pending.front());
      if (lrc != SVO_OK) {
        s->fatal = lrc;
        break;
      }
      s->pending.pop_front();
      launched = true;
    }
    if (s->fatal != SVO_OK) {
      for (uint64_t t : s->pending) {
        s->requests[t].res.status = s->fatal;
        s->requests[t].done = true;
      }
      s->pending.clear();
      s->cv_user.notify_all();
    }
    s->blocked = !s->pending.empty() && !s->streamed.empty();
  }
}

// The pool, the slots' streams and batchers, and the dispatcher thread.
int start_server(svo_server* s, const svo_server_cfg* cfg) {
  int rc = s->pool.init(cfg->hbm_budget_bytes);
  // Plain mode queues one per-frame kernel per request back to back on a
  // single stream (its slots share that stream); batched mode gives every
  // slot its own stream and batcher so batches overlap.
  s->slots.resize(cfg->streams);
  for (uint32_t i = 0; i < cfg->streams && rc == SVO_OK; ++i) {
    auto& sl = s->slots[i];
    sl.owner = s;
    sl.index = i;
    if (cfg->mode == SVO_SERVE_PLAIN && i > 0) {
      sl.stream = s->slots[0].stream;
      continue;
    }
    rc = svo::cuda_status(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking));
    if (rc == SVO_OK && cfg->mode == SVO_SERVE_BATCHED)
      rc = svo_batcher_create(cfg->max_batch_views, 64, &sl.batcher);
  }
  if (rc != SVO_OK) return rc;
  s->dispatcher = std::thread(cfg->mode == SVO_SERVE_PLAIN_STREAMED ? dispatch_loop_streamed : dispatch_loop, s);
  return SVO_OK;
}

}  // namespace

extern "C" {

int svo_server_create(const svo_server_cfg* cfg, svo_server** out) {
  if (!cfg || !out) return SVO_ERR_INVALID;
  *out = nullptr;
  if (cfg->streams == 0 || cfg->streams > 16 || cfg->max_batch_views == 0 ||
      cfg->max_batch_views > 4096 || cfg->max_inflight_rays == 0)
    return SVO_ERR_RANGE;
  if (cfg->mode != SVO_SERVE_BATCHED && cfg->mode != SVO_SERVE_PLAIN &&
      cfg->mode != SVO_SERVE_PLAIN_STREAMED)
    return SVO_ERR_NOTSUP;
  auto* s = new (std::nothrow) svo_server;
  if (!s) return SVO_ERR_NOMEM;
  s->cfg = *cfg;
  if (s->cfg.tile_w == 0) s->cfg.tile_w = 8, s->cfg.tile_h = 4;
  if (s->cfg.block_threads == 0) s->cfg.block_threads = 128;
  s->t0 = Clock::now();
  int rc = SVO_OK;
  try {
    rc = start_server(s, cfg);
  } catch (const std::bad_alloc&) {
    rc = SVO_ERR_NOMEM;
  } catch (...) {  // std::thread could not start
    rc = SVO_ERR_INVALID;
  }
  if (rc != SVO_OK) {
    svo_server_destroy(s);
    return rc;
  }
  *out = s;
  return SVO_OK;
}

void svo_server_destroy(svo_server* s) {
  if (!s) return;
  if (s->dispatcher.joinable()) {
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->stop = true;
      // requests never launched end as cancelled
      for (uint64_t t : s->pending) {
        s->requests[t].res.status = SVO_ERR_CANCELED;
        s->requests[t].done = true;
      }
      s->pending.clear();
    }
    s->cv_dispatch.notify_one();
    s->dispatcher.join();
  }
  // paged octrees' workers: requests still queued end as cancelled
  for (auto& o : s->octrees) {
    if (!o.worker) continue;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      o.worker->stop = true;
      for (uint64_t t : o.worker->queue) {
        s->requests[t].res.status = SVO_ERR_CANCELED;
        s->requests[t].done = true;
      }
      o.worker->queue.clear();
    }
    o.worker->cv.notify_one();
    if (o.worker->thread.joinable()) o.worker->thread.join();
    if (o.worker->stream) {
      cudaStreamSynchronize(o.worker->stream);
      cudaStreamDestroy(o.worker->stream);
    }
  }
  s->cv_user.notify_all();
  // plain mode: all slots share slot 0's stream, destroyed once at the end
  for (auto& sl : s->slots)
    if (sl.stream) cudaStreamSynchronize(sl.stream);
  for (auto& f : s->streamed) cudaEventDestroy(f.done);  // (none left after a clean stop)
  for (cudaEvent_t e : s->spare_events) cudaEventDestroy(e);
  for (uint32_t i = 0; i < s->slots.size(); ++i) {
    auto& sl = s->slots[i];
    if (sl.batcher) svo_batcher_destroy(sl.batcher);
    const bool shared = s->cfg.mode == SVO_SERVE_PLAIN && i > 0;
    if (sl.stream && !shared) cudaStreamDestroy(sl.stream);
  }
  // A callback may still be inside its notify when its completion has been
  // processed: wait (bounded) until every callback is past its last access.
  // If one never gets there, the object is leaked rather than freed under it.
  const auto deadline = Clock::now() + std::chrono::seconds(10);
  while (s->callbacks_exited.load(std::memory_order_acquire) != s->callbacks_launched.load()) {
    if (Clock::now() > deadline) return;
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  delete s;
}

}  // extern "C"

namespace {

// Registers an octree: whole-resident on demand, or treelet-paged in a
// region of `region_bytes` (node and attribute halves) when `paged`.
int add_octree(svo_server* s, const svo_scene* scene, int32_t stack_size, bool paged,
               uint64_t region_bytes, uint32_t* id) {
  if (!s || !scene || !id || scene->treelets.empty()) return SVO_ERR_INVALID;
  if (stack_size < 2 || stack_size > 24) return SVO_ERR_RANGE;
  try {
    ServedOctree o;
    o.mm.reset(new svo::TreeletMemoryManagerCuda(nullptr));
    svo_scene copy = *scene;
    const uint64_t tb = scene->treelet_bytes;
    const uint64_t whole = 2 * ((tb * scene->treelets.size() + 255) & ~255ull);
    if (!paged && whole > s->pool.size()) {  // cannot be resident whole: a quarter of the budget
      paged = true;
      region_bytes = s->pool.size() / 4;
    }
    uint64_t slots = scene->treelets.size();
    if (paged) {
      slots = std::min<uint64_t>(slots, (region_bytes / 2) / tb);
      if (slots < 2) return SVO_ERR_RANGE;  // the root and one more treelet at least
    }
    int rc = o.mm->init(std::move(copy), slots * tb);
    if (rc != SVO_OK) return rc;
    if (!paged) {
      uint32_t n = 0;
      rc = o.mm->insert_all(&n);
      if (rc != SVO_OK) return rc;
    } else {
      // requests look anywhere: any treelet their views no longer see may go,
      // and one pass may fill the whole region
      o.mm->set_evict_any_invisible(true);
      o.mm->set_max_new_treelets((uint32_t)slots);
    }
    o.stack_size = stack_size;
    o.node_bytes = o.mm->incore_nodes() * sizeof(svo_node);
    o.paged = paged;
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->octrees.size() >= 64) return SVO_ERR_RANGE;
    if (paged) {
      // the region is held for the server's life; only the root treelet is
      // resident at first
      const uint64_t need = 2 * ((o.node_bytes + 255) & ~255ull);
      uint64_t off = 0;
      rc = alloc_evicting(s, need, -1, &off);
      if (rc != SVO_OK) return rc;
      char* base = s->pool.base() + off;
      rc = o.mm->attach_device_buffers(reinterpret_cast<svo_node*>(base),
                                       reinterpret_cast<svo_attrib*>(base + need / 2));
      if (rc == SVO_OK) rc = o.mm->wait_uploads(nullptr);
      if (rc == SVO_OK) rc = svo::cuda_status(cudaStreamSynchronize(nullptr));
      if (rc != SVO_OK) {
        s->pool.release(off, need);
        return rc;
      }
      o.pool_off = off;
      o.resident = true;
      o.worker.reset(new PagedWorker);
      rc = svo::cuda_status(cudaStreamCreateWithFlags(&o.worker->stream, cudaStreamNonBlocking));
      if (rc != SVO_OK) {
        s->pool.release(off, need);
        return rc;
      }
      s->stats.resident_bytes += need;
    }
    s->octrees.push_back(std::move(o));
    *id = (uint32_t)s->octrees.size() - 1;
    if (paged) s->octrees.back().worker->thread = std::thread(paged_worker_loop, s, *id);
  } catch (const std::bad_alloc&) {
    return SVO_ERR_NOMEM;
  } catch (const std::system_error&) {  // the worker thread could not start
    return SVO_ERR_NOMEM;
  }
  return SVO_OK;
}

}  // namespace

extern "C" {

int svo_server_add_octree(svo_server* s, const svo_scene* scene, int32_t stack_size, uint32_t* id) {
  return add_octree(s, scene, stack_size, false, 0, id);
}

int svo_server_add_octree_paged(svo_server* s, const svo_scene* scene, int32_t stack_size,
                                uint64_t region_bytes, uint32_t* id) {
  return add_octree(s, scene, stack_size, true, region_bytes, id);
}

int svo_server_set_upload_policy(svo_server* s, uint32_t octree, int32_t policy) {
  if (!s) return SVO_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  if (octree >= s->octrees.size()) return SVO_ERR_INVALID;
  try {
    return s->octrees[octree].mm->set_upload_policy(policy);
  } catch (const std::bad_alloc&) {
    return SVO_ERR_NOMEM;
  }
}

int svo_server_submit(svo_server* s, const svo_request* req, uint64_t* ticket) {
  const double submitted = s ? s->now() : 0.0;  // before waiting for the lock
  if (!s || !req || !ticket || !req->d_rgba) return SVO_ERR_INVALID;
  const int32_t m = req->params.mode;
  if (m < 0 || m > 7) return SVO_ERR_NOTSUP;
  if (req->params.width == 0 || req->params.height == 0) return SVO_ERR_INVALID;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (req->octree >= s->octrees.size() || s->stop) return SVO_ERR_INVALID;
    const uint64_t t = s->next_ticket++;
    Request& q = s->requests[t];
    q.r = *req;
    q.res.status = SVO_ERR_BUSY;
    q.res.submit_s = submitted;
    s->pending.push_back(t);
    s->blocked = false;
    *ticket = t;
  }
  s->cv_dispatch.notify_one();
  return SVO_OK;
}

int svo_server_wait(svo_server* s, uint64_t ticket, uint32_t timeout_ms, svo_request_result* out) {
  if (!s) return SVO_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->requests.find(ticket);
  if (it == s->requests.end()) return SVO_ERR_INVALID;
  const bool ok = s->cv_user.wait_for(lk, std::chrono::milliseconds(timeout_ms),
                                      [&] { return s->requests[ticket].done; });
  if (!ok) return SVO_ERR_TIMEOUT;
  if (out) *out = s->requests[ticket].res;
  return SVO_OK;
}

int svo_server_poll(svo_server* s, uint64_t ticket, svo_request_result* out) {
  const int rc = svo_server_wait(s, ticket, 0, out);
  return rc == SVO_ERR_TIMEOUT ? SVO_ERR_BUSY : rc;
}

int svo_server_cancel(svo_server* s, uint64_t ticket) {
  if (!s) return SVO_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->requests.find(ticket);
  if (it == s->requests.end()) return SVO_ERR_INVALID;
  auto p = std::find(s->pending.begin(), s->pending.end(), ticket);
  if (p == s->pending.end()) return it->second.done ? SVO_OK : SVO_ERR_BUSY;  // running
  s->pending.erase(p);
  it->second.res.status = SVO_ERR_CANCELED;
  it->second.done = true;
  s->cv_user.notify_all();
  return SVO_OK;
}

int svo_server_release(svo_server* s, uint64_t ticket) {
  if (!s) return SVO_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->requests.find(ticket);
  if (it == s->requests.end()) return SVO_ERR_INVALID;
  if (!it->second.done) return SVO_ERR_BUSY;
  s->requests.erase(it);
  return SVO_OK;
}

int svo_server_stats_get(svo_server* s, svo_server_stats* out) {
  if (!s || !out) return SVO_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  return SVO_OK;
}

int svo_server_replay(svo_server* s, const svo_request* reqs, const double* arrival_s, uint32_t n,
                      uint32_t timeout_ms, svo_request_result* results) {
  if (!s || (n && (!reqs || !arrival_s || !results))) return SVO_ERR_INVALID;
  std::vector<uint64_t> tickets(n, 0);
  const auto start = Clock::now();
  for (uint32_t i = 0; i < n; ++i) {
    const auto due = start + std::chrono::duration_cast<Clock::duration>(
                                 std::chrono::duration<double>(arrival_s[i]));
    const auto early = due - std::chrono::microseconds(100);
    if (Clock::now() < early) std::this_thread::sleep_until(early);
    while (Clock::now() < due) {
    }
    const int rc = svo_server_submit(s, &reqs[i], &tickets[i]);
    if (rc != SVO_OK) return rc;
  }
  int first = SVO_OK;
  for (uint32_t i = 0; i < n; ++i) {
    const int rc = svo_server_wait(s, tickets[i], timeout_ms, &results[i]);
    if (rc != SVO_OK) {
      results[i].status = rc;
      if (first == SVO_OK) first = rc;
    } else {
      svo_server_release(s, tickets[i]);
    }
  }
  return first;
}

}  // extern "C"
