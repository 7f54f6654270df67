// upload.h -- device side of the packed slot upload (upload.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/libsvo_b200.h"

namespace svo {

// Moves `count` packed slots ({N nodes, N attributes} each, back to back in
// `stage`) to slot ids[i] of the node and attribute pools.
int launch_slot_scatter(const void* stage, const uint32_t* ids, uint32_t count, uint64_t N,
                        svo_node* nodes, svo_attrib* attribs, cudaStream_t stream);

// Reads `count` slots ids[i] straight from the page-locked, mapped host
// mirror (host_nodes / host_attribs are its device-side addresses) and
// writes them to the same slots of the device pools.
int launch_slot_gather(const svo_node* host_nodes, const svo_attrib* host_attribs,
                       const uint32_t* ids, uint32_t count, uint64_t N, svo_node* nodes,
                       svo_attrib* attribs, cudaStream_t stream);

}  // namespace svo
