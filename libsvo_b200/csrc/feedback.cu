// feedback.cu -- the analysis pass: renderToFeedbackBuffer / sampleAnalyse
// (opencl/treeletRenderer_rgba.cl:761-1011).
//
// One analysis ray per pixel of a (usually reduced-resolution) buffer, cast
// with the same traversal as sample().  Where sample() stops at a leaf, the
// record carries the leaf's first-child field -- the gid of its sub-treelet
// when that treelet is not resident, 0 for a leaf of the whole octree -- and
// the LOD error scale_exp2 - tScaleRatio * tcMin; an LOD stop records the LOD
// flag as its error; a miss, or a ray the watchdog ends, leaves the record at
// its initial {0, 0, 0, 9999999}.  The host turns the records into the
// treelets to page in (TreeletMemoryManager::analyse_feedback).
#include <cuda_runtime.h>

#include "feedback.h"
#include "shade.cuh"
#include "traverse.cuh"

namespace svo {

namespace {

// One warp (8x4 pixels) per block: analysis buffers are small (128x128 for
// a 1024x1024 frame at the reference's divisor 8), and one-warp blocks
// spread their few rays over all SMs.
constexpr int kBlockW = 8;
constexpr int kBlockH = 4;
constexpr int kThreads = kBlockW * kBlockH;

__global__ void __launch_bounds__(kThreads) feedback_kernel(
    const uint2* __restrict__ nodes, uint64_t num_nodes, const svo_frame_params p, int S,
    svo_feedback* __restrict__ out, uint32_t* __restrict__ rgba, uint32_t y0) {
  extern __shared__ uint2 stack_smem[];
  const int t = threadIdx.x;
  const int warp = t >> 5, lane = t & 31;
  const uint32_t x = blockIdx.x * kBlockW + (warp % (kBlockW / 8)) * 8 + (lane & 7);
  const uint32_t y = y0 + blockIdx.y * kBlockH + (warp / (kBlockW / 8)) * 4 + (lane >> 3);
  if (x >= p.width || y >= p.height) return;
  float o[3], dx, dy, dz;
  pixel_ray(p, x, y, o, dx, dy, dz);
  const RayHit h = cast_ray<false>(GlobalFetch{nodes}, num_nodes, o, dx, dy, dz, p.t_scale_ratio,
                                   S, stack_smem + t, kThreads);
  int32_t node_id = 0, sub = 0;
  float error = 0.0f, t_min = 9999999.0f;
  if (h.hit && h.flags != SVO_HITFLAG_CAPPED) {
    node_id = (int32_t)h.node;
    t_min = h.tc_min;
    const float lod = __fmul_rn(p.t_scale_ratio, h.tc_min);
    if (h.leaf) {
      error = __fsub_rn(h.sx2, lod);
      sub = (uint64_t)h.node < num_nodes ? (int32_t)__ldg(nodes + h.node).x : 0;
    } else {
      error = lod > h.sx2 ? 1.0f : 0.0f;
    }
  }
  const uint64_t pix = (uint64_t)y * p.width + x;
  reinterpret_cast<int4*>(out)[pix] =
      make_int4(node_id, __float_as_int(error), sub, __float_as_int(t_min));
  if (rgba != nullptr)
    rgba[pix] = node_id != 0 ? pack_rgba8(__int2float_rn(sub), 0.0f, error, 1.0f)
                             : pack_rgba8(0.2f, 0.3f, 0.2f, 1.0f);
}

}  // namespace

int launch_feedback(const svo_node* nodes, uint64_t num_nodes, const svo_frame_params& p, int S,
                    svo_feedback* out, uint32_t* rgba, cudaStream_t stream) {
  if (p.width == 0 || p.height == 0) return SVO_OK;
  if (p.height > 0xFFFFFFF0u) return SVO_ERR_RANGE;  // row indices stay below 2^32
  const size_t smem = (size_t)S * kThreads * sizeof(uint2);
  constexpr uint32_t kRowsPerLaunch = 65535u * kBlockH;  // grid rows are at most 65535
  for (uint32_t y0 = 0; y0 < p.height; y0 += kRowsPerLaunch) {
    const uint32_t rows = p.height - y0 < kRowsPerLaunch ? p.height - y0 : kRowsPerLaunch;
    const dim3 grid((p.width + kBlockW - 1) / kBlockW, (rows + kBlockH - 1) / kBlockH);
    feedback_kernel<<<grid, kThreads, smem, stream>>>(reinterpret_cast<const uint2*>(nodes),
                                                       num_nodes, p, S, out, rgba, y0);
    if (cudaGetLastError() != cudaSuccess) return SVO_ERR_CUDA;
  }
  return SVO_OK;
}

}  // namespace svo
