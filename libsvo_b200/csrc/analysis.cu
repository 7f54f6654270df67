// analysis.cu -- the analysis pass's record processing on the GPU: the
// device form of TreeletMemoryManager::analyse_feedback, which restates
// RenderPassAnalyse::performAnalysePass (src/RenderPassAnalyse.cpp:218-356).
//
// One thread per feedback record folds the record into two per-treelet
// arrays with atomicMax over an order-preserving integer image of the error:
// the largest error seen for each newly visible sub-treelet, and the largest
// error of each treelet on the path from the hit node's treelet up to the
// root (the root itself gets 99 once any record hits).  Only these arrays,
// 4 bytes per treelet each, go back to the host instead of the records; the
// host lists the set entries in ascending gid order -- the order in which
// the reference's std::map is iterated -- and sorts them by error as before.
#include <cuda_runtime.h>

#include "analysis.h"

namespace svo {

namespace {

__device__ __forceinline__ uint32_t error_key_d(float e) {
  const uint32_t b = __float_as_uint(e);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__global__ void analyse_kernel(const int4* __restrict__ records, uint64_t n,
                               const int32_t* __restrict__ slot_gid, uint32_t num_slots,
                               uint32_t nodes_per_slot, const int32_t* __restrict__ parent,
                               uint32_t num_treelets, uint32_t* __restrict__ new_key,
                               uint32_t* __restrict__ old_key, uint32_t* __restrict__ status) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int4 e = __ldg(records + i);
    const int32_t node_id = e.x, sub = e.z;
    if (node_id == 0) continue;
    const uint32_t key = error_key_d(__int_as_float(e.y));
    // the reference rejects the whole pass on these records (:257-263, :286-304)
    if (sub != 0) {
      if (node_id < 0 || (uint32_t)sub > num_treelets) {
        atomicOr(status, kAnalyseRejected);
        continue;
      }
      atomicMax(new_key + sub, key);
    }
    const uint32_t slot = (uint32_t)node_id / nodes_per_slot;
    if (slot > num_treelets || slot >= num_slots) {
      atomicOr(status, kAnalyseRejected);
      continue;
    }
    const int32_t gid = slot_gid[slot];
    if (gid < 0 || (uint32_t)gid > num_treelets) {
      atomicOr(status, kAnalyseRejected);
      continue;
    }
    // addNodeAndItsParentTreeletsToVisibleTreelets (:381-420); the walk is
    // bounded so that a parent table with a cycle ends it with an error
    bool ok = true;
    uint32_t steps = 0;
    for (int32_t g = gid; g != 0;) {
      if ((uint32_t)g > num_treelets) {  // a parent entry outside the table
        atomicOr(status, kAnalyseRejected);
        ok = false;
        break;
      }
      atomicMax(old_key + g, key);
      if ((uint32_t)g >= num_treelets || ++steps > num_treelets) {
        atomicOr(status, kAnalyseRejected);
        ok = false;
        break;
      }
      g = parent[g];
    }
    if (ok) atomicMax(old_key, error_key_d(99.0f));
  }
}

}  // namespace

int launch_analyse(const svo_feedback* records, uint64_t n, const int32_t* slot_gid,
                   uint32_t num_slots, uint32_t nodes_per_slot, const int32_t* parent,
                   uint32_t num_treelets, uint32_t* new_key, uint32_t* old_key, uint32_t* status,
                   cudaStream_t stream) {
  if (n == 0) return SVO_OK;
  if (nodes_per_slot == 0) return SVO_ERR_INVALID;
  constexpr uint32_t kThreads = 256;
  const uint64_t want = (n + kThreads - 1) / kThreads;
  const uint32_t blocks = (uint32_t)(want < 4096 ? want : 4096);
  analyse_kernel<<<blocks, kThreads, 0, stream>>>(reinterpret_cast<const int4*>(records), n,
                                                  slot_gid, num_slots, nodes_per_slot, parent,
                                                  num_treelets, new_key, old_key, status);
  return cudaGetLastError() == cudaSuccess ? SVO_OK : SVO_ERR_CUDA;
}

}  // namespace svo
