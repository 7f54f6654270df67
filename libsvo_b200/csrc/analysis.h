// analysis.h -- the analysis pass's record processing on the GPU.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "../../include/libsvo_b200.h"

namespace svo {

constexpr uint32_t kAnalyseRejected = 1u;  // a record the reference rejects

// Order-preserving image of a float error as an unsigned key (larger error,
// larger key; every non-NaN error has a key above 0, so 0 marks "not seen").
inline uint32_t error_key(float e) {
  uint32_t b;
  std::memcpy(&b, &e, 4);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
inline float key_error(uint32_t k) {
  const uint32_t b = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
  float e;
  std::memcpy(&e, &b, 4);
  return e;
}

// Folds n feedback records (device) into new_key[0..num_treelets] (largest
// error key per newly visible sub-treelet gid) and old_key[0..num_treelets]
// (largest error key per visible resident treelet and its ancestors, the
// root at 99); both arrays and *status must be zeroed first.  slot_gid[s] is
// the gid resident in slot s (-1 when free), parent[g] the parent gid of
// treelet g.  Sets kAnalyseRejected in *status on a record the reference
// rejects.
int launch_analyse(const svo_feedback* records, uint64_t n, const int32_t* slot_gid,
                   uint32_t num_slots, uint32_t nodes_per_slot, const int32_t* parent,
                   uint32_t num_treelets, uint32_t* new_key, uint32_t* old_key, uint32_t* status,
                   cudaStream_t stream);

}  // namespace svo
