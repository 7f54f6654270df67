// traverse_host.cpp -- the kernels' traversal (libsvo_b200/csrc/traverse.cuh)
// built for the host.  TEST INFRASTRUCTURE ONLY: see host_shim.h.
#include "host_shim.h"

#include "../../libsvo_b200/csrc/traverse.cuh"

extern "C" void host_cast_rays(const uint32_t* nodes, uint64_t num_nodes, const float* origins,
                               const float* dirs, uint64_t n, float tsr, int S, int flat,
                               void* hits) {
  uint2 stack[svo::kMaxStack];
  const svo::GlobalFetch fetch{reinterpret_cast<const uint2*>(nodes)};
  uint32_t* out = static_cast<uint32_t*>(hits);
  for (uint64_t i = 0; i < n; ++i) {
    const float o[3] = {origins[3 * i], origins[3 * i + 1], origins[3 * i + 2]};
    const float dx = dirs[3 * i], dy = dirs[3 * i + 1], dz = dirs[3 * i + 2];
    const svo::RayHit h =
        flat ? svo::cast_ray<true>(fetch, num_nodes, o, dx, dy, dz, tsr, S, stack, 1)
             : svo::cast_ray<false>(fetch, num_nodes, o, dx, dy, dz, tsr, S, stack, 1);
    // the 16-byte svo_hit record, as the kernels' store_hit writes it
    uint32_t* w = out + 4 * i;
    w[0] = h.node;
    w[1] = __float_as_uint(h.t);
    w[2] = (h.depth & 0xFFFFu) | ((h.hit & 0xFFu) << 16) | ((h.flags & 0xFFu) << 24);
    w[3] = (h.loops & 0xFFFFu) | (h.fetches << 16);
  }
}
