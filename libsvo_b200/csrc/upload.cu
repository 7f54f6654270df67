// upload.cu -- scatter of packed incore slots into the device pools.
//
// The packed upload (TreeletMemoryManagerCuda::upload_packed) replaces the
// reference's per-range buffer writes (src/TreeletMemoryManagerCl.cpp:
// 177-236): only dirty slots cross PCIe, in one copy per 32 MB, and this
// kernel places them at HBM bandwidth.  One block per slot; 8-byte records,
// coalesced on both sides.
#include <cuda_runtime.h>

#include "upload.h"

namespace svo {

namespace {

__global__ void __launch_bounds__(256) slot_scatter_kernel(const uint2* __restrict__ stage,
                                                           const uint32_t* __restrict__ ids,
                                                           uint64_t N, uint2* __restrict__ nodes,
                                                           uint2* __restrict__ attribs) {
  const uint2* src = stage + (uint64_t)blockIdx.x * 2 * N;
  const uint64_t dst = (uint64_t)ids[blockIdx.x] * N;
  for (uint64_t i = threadIdx.x; i < N; i += blockDim.x) {
    nodes[dst + i] = src[i];
    attribs[dst + i] = src[N + i];
  }
}

// One block per dirty slot; each thread keeps several 16-byte reads of
// mapped host memory in flight, so the PCIe link stays busy without one DMA
// call per slot.
__global__ void __launch_bounds__(256) slot_gather_kernel(const uint2* __restrict__ hn,
                                                          const uint2* __restrict__ ha,
                                                          const uint32_t* __restrict__ ids,
                                                          uint64_t N, uint2* __restrict__ nodes,
                                                          uint2* __restrict__ attribs) {
  const uint64_t base = (uint64_t)ids[blockIdx.x] * N;
  constexpr int kUnroll = 4;
  for (uint64_t i0 = threadIdx.x; i0 < N; i0 += (uint64_t)blockDim.x * kUnroll) {
    uint2 a[kUnroll], b[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const uint64_t i = i0 + (uint64_t)u * blockDim.x;
      if (i < N) {
        a[u] = hn[base + i];
        b[u] = ha[base + i];
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const uint64_t i = i0 + (uint64_t)u * blockDim.x;
      if (i < N) {
        nodes[base + i] = a[u];
        attribs[base + i] = b[u];
      }
    }
  }
}

}  // namespace

int launch_slot_gather(const svo_node* host_nodes, const svo_attrib* host_attribs,
                       const uint32_t* ids, uint32_t count, uint64_t N, svo_node* nodes,
                       svo_attrib* attribs, cudaStream_t stream) {
  if (count == 0) return SVO_OK;
  slot_gather_kernel<<<count, 256, 0, stream>>>(
      reinterpret_cast<const uint2*>(host_nodes), reinterpret_cast<const uint2*>(host_attribs), ids,
      N, reinterpret_cast<uint2*>(nodes), reinterpret_cast<uint2*>(attribs));
  return cudaGetLastError() == cudaSuccess ? SVO_OK : SVO_ERR_CUDA;
}

int launch_slot_scatter(const void* stage, const uint32_t* ids, uint32_t count, uint64_t N,
                        svo_node* nodes, svo_attrib* attribs, cudaStream_t stream) {
  if (count == 0) return SVO_OK;
  slot_scatter_kernel<<<count, 256, 0, stream>>>(reinterpret_cast<const uint2*>(stage), ids, N,
                                                 reinterpret_cast<uint2*>(nodes),
                                                 reinterpret_cast<uint2*>(attribs));
  return cudaGetLastError() == cudaSuccess ? SVO_OK : SVO_ERR_CUDA;
}

}  // namespace svo
