// render.h -- host-side launchers of the ray-cast kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "../../include/libsvo_b200.h"

namespace svo {

size_t render_smem_bytes(int stack_size);

int launch_render(const svo_node* nodes, const svo_attrib* attribs, uint64_t num_nodes,
                  const svo_frame_params& p, const svo_trace_cfg& cfg, uint32_t* rgba,
                  svo_hit* hits, svo_stats* stats, cudaStream_t stream);

int launch_render_shadow(const svo_node* nodes, const svo_attrib* attribs, uint64_t num_nodes,
                         const svo_frame_params& p, const svo_shadow_cfg& sc, int stack_size,
                         uint32_t* rgba, svo_hit* hits, svo_hit* shadow_hits, svo_stats* stats,
                         cudaStream_t stream);

int launch_trace_rays(const svo_node* nodes, uint64_t num_nodes, const float* origins,
                      const float* dirs, uint64_t n, float tsr, const svo_trace_cfg& cfg,
                      svo_hit* hits, svo_stats* stats, cudaStream_t stream);

}  // namespace svo
