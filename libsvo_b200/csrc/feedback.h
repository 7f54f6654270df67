// feedback.h -- launcher of the analysis-pass kernel.
#pragma once
#include <cuda_runtime.h>

#include "../../include/libsvo_b200.h"

namespace svo {

int launch_feedback(const svo_node* nodes, uint64_t num_nodes, const svo_frame_params& p, int S,
                    svo_feedback* out, uint32_t* rgba, cudaStream_t stream);

}  // namespace svo
