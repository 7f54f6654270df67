// errors.h -- CUDA status -> library status, with the last CUDA error kept
// per host thread for svo_last_error().
#pragma once
#include <cuda_runtime.h>

#include "../../include/libsvo_b200.h"

namespace svo {

void set_last_error(const char* msg);
const char* last_error();

inline int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return SVO_OK;
  set_last_error(cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? SVO_ERR_NOMEM : SVO_ERR_CUDA;
}

}  // namespace svo

#define SVO_CUDA_TRY(call)                               \
  do {                                                   \
    const int svo_rc_ = ::svo::cuda_status((call));      \
    if (svo_rc_ != SVO_OK) return svo_rc_;               \
  } while (0)
