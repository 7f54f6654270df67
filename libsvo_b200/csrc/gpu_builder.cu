// gpu_builder.cu -- mesh -> octree -> treelets -> fully resident incore pool,
// on the GPU.
//
// The same scene the host builder produces (csrc/scene.cpp:
// build_mesh_leaves, octree_from_leaves, cut_treelets) followed by
// TreeletMemoryManager::insert_all (csrc/memory_manager.cpp), bit for bit,
// for the scale of the largest configuration (about 10^9 leaves), where the
// host path would need tens of GB of host memory and hours of CPU time.  It
// stands in for the reference's TreeletBuilderFromFaces::buildFromQueue
// (src/TreeletBuilderFromFaces.cpp:189-365), TreeletBuildManager
// (src/TreeletBuildManager.cpp:150-258) and the insertion loop of
// TreeletMemoryManager (src/TreeletMemoryManager.cpp:518-545).
//
// Pipeline, all in device memory:
//  1. face normals, one thread per triangle;
//  2. voxelisation per spatial chunk (the top octree level(s)): a count pass
//     and an emit pass, one thread per triangle, walking columns along the
//     dominant normal axis exactly like the host builder, with the
//     separating-axis triangle/box test; each overlap is a 64-bit key
//     (code within the chunk << tri_bits | triangle);
//  3. radix sort of the keys (CUB), so equal codes are grouped with their
//     triangles ascending, then one thread per run sums the face normals in
//     that order -> leaf codes and attributes;
//  4. octree levels bottom-up: one thread per parent over its <= 8 children
//     (valid mask, first child, averaged attributes as the host does);
//  5. the treelet cut in closed form: treelet boundaries sit on fixed levels
//     (stop_level), each treelet is the breadth-first fill of its root's
//     subtree down to the next boundary, so its nodes at a level are one
//     contiguous range of that level, its local positions are range offsets,
//     and the treelet ids are range offsets of the boundary levels; one block
//     per treelet writes its slot, with every sub-treelet root patched into
//     its parent's leaf as insert_all does.
//
// FP32 arithmetic uses explicit round-to-nearest intrinsics in the host
// builder's operation order (the library is built with -fmad=false), so the
// attributes and the voxel sets match the host builder's bit for bit.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "../../include/libsvo_b200.h"
#include "errors.h"
#include "gpu_builder.h"

namespace svo {

namespace {

// ---- shared arithmetic (host builder: csrc/scene.cpp) ----------------------

__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }  // std::max

__device__ __forceinline__ uint64_t split3(uint32_t a) {
  uint64_t x = a & 0x1fffffu;
  x = (x | x << 32) & 0x1f00000000ffffull;
  x = (x | x << 16) & 0x1f0000ff0000ffull;
  x = (x | x << 8) & 0x100f00f00f00f00full;
  x = (x | x << 4) & 0x10c30c30c30c30c3ull;
  x = (x | x << 2) & 0x1249249249249249ull;
  return x;
}
__device__ __forceinline__ uint64_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  return (split3(x) << 2) | (split3(y) << 1) | split3(z);
}

__device__ __forceinline__ uint32_t unorm8(float c) {
  if (!(c > 0.0f)) return 0u;
  if (c >= 1.0f) return 255u;
  return __float2uint_rz(__fadd_rn(__fmul_rn(c, 255.0f), 0.5f));
}
__device__ __forceinline__ uint32_t pack_color(float r, float g, float b) {
  return (unorm8(r) << 24) | (unorm8(g) << 16) | (unorm8(b) << 8) | 255u;
}
__device__ __forceinline__ uint32_t pack_normal(float x, float y, float z) {
  return pack_color(__fadd_rn(__fmul_rn(x, 0.5f), 0.5f), __fadd_rn(__fmul_rn(y, 0.5f), 0.5f),
                    __fadd_rn(__fmul_rn(z, 0.5f), 0.5f));
}
__device__ __forceinline__ void unpack_color(uint32_t v, float rgb[3]) {
  rgb[0] = __fdiv_rn((float)(v >> 24), 255.0f);
  rgb[1] = __fdiv_rn((float)((v >> 16) & 255u), 255.0f);
  rgb[2] = __fdiv_rn((float)((v >> 8) & 255u), 255.0f);
}
__device__ __forceinline__ float len3(float x, float y, float z) {
  return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
}

// cell_floor of the host builder: floor(x) clamped to [-2, R + 1], NaN -> -2.
__device__ __forceinline__ int cell_floor(float x, uint32_t R) {
  const float hi = __fadd_rn((float)R, 1.0f);
  if (!(x >= -2.0f)) return -2;
  if (x > hi) return (int)R + 1;
  return __float2int_rz(floorf(x));
}

__device__ __forceinline__ float dot3(float ax, float ay, float az, const float v[3]) {
  return __fadd_rn(__fadd_rn(__fmul_rn(ax, v[0]), __fmul_rn(ay, v[1])), __fmul_rn(az, v[2]));
}

__device__ __forceinline__ bool separated(float ax, float ay, float az, const float v0[3],
                                          const float v1[3], const float v2[3], float h) {
  const float p0 = dot3(ax, ay, az, v0), p1 = dot3(ax, ay, az, v1), p2 = dot3(ax, ay, az, v2);
  const float mn = smin(p0, smin(p1, p2)), mx = smax(p0, smax(p1, p2));
  const float r = __fmul_rn(h, __fadd_rn(__fadd_rn(fabsf(ax), fabsf(ay)), fabsf(az)));
  return mn > r || mx < -r;
}

// tri_box_overlap of the host builder (Akenine-Moeller 2001, restated there).
__device__ bool tri_box_overlap(const float bc[3], float h, const float a[3], const float b[3],
                                const float c[3]) {
  float v0[3], v1[3], v2[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    v0[i] = __fsub_rn(a[i], bc[i]);
    v1[i] = __fsub_rn(b[i], bc[i]);
    v2[i] = __fsub_rn(c[i], bc[i]);
  }
  const float e[3][3] = {{__fsub_rn(v1[0], v0[0]), __fsub_rn(v1[1], v0[1]), __fsub_rn(v1[2], v0[2])},
                         {__fsub_rn(v2[0], v1[0]), __fsub_rn(v2[1], v1[1]), __fsub_rn(v2[2], v1[2])},
                         {__fsub_rn(v0[0], v2[0]), __fsub_rn(v0[1], v2[1]), __fsub_rn(v0[2], v2[2])}};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float* ek = e[k];
    if (separated(0.0f, ek[2], -ek[1], v0, v1, v2, h)) return false;
    if (separated(-ek[2], 0.0f, ek[0], v0, v1, v2, h)) return false;
    if (separated(ek[1], -ek[0], 0.0f, v0, v1, v2, h)) return false;
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float mn = smin(v0[i], smin(v1[i], v2[i]));
    const float mx = smax(v0[i], smax(v1[i], v2[i]));
    if (mn > h || mx < -h) return false;
  }
  const float n[3] = {
      __fsub_rn(__fmul_rn(e[0][1], e[1][2]), __fmul_rn(e[0][2], e[1][1])),
      __fsub_rn(__fmul_rn(e[0][2], e[1][0]), __fmul_rn(e[0][0], e[1][2])),
      __fsub_rn(__fmul_rn(e[0][0], e[1][1]), __fmul_rn(e[0][1], e[1][0]))};
  const float d = -dot3(n[0], n[1], n[2], v0);
  float vmin[3], vmax[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    vmin[i] = n[i] > 0.0f ? -h : h;
    vmax[i] = n[i] > 0.0f ? h : -h;
  }
  if (__fadd_rn(dot3(n[0], n[1], n[2], vmin), d) > 0.0f) return false;
  return __fadd_rn(dot3(n[0], n[1], n[2], vmax), d) >= 0.0f;
}

// ---- 1. face normals ---------------------------------------------------------

__global__ void face_normals_kernel(const float* __restrict__ V, const uint32_t* __restrict__ T,
                                    uint64_t nt, float* __restrict__ fn) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const float* a = V + 3 * (uint64_t)T[3 * t];
  const float* b = V + 3 * (uint64_t)T[3 * t + 1];
  const float* c = V + 3 * (uint64_t)T[3 * t + 2];
  const float n0 = __fsub_rn(__fmul_rn(__fsub_rn(b[1], a[1]), __fsub_rn(c[2], a[2])),
                             __fmul_rn(__fsub_rn(b[2], a[2]), __fsub_rn(c[1], a[1])));
  const float n1 = __fsub_rn(__fmul_rn(__fsub_rn(b[2], a[2]), __fsub_rn(c[0], a[0])),
                             __fmul_rn(__fsub_rn(b[0], a[0]), __fsub_rn(c[2], a[2])));
  const float n2 = __fsub_rn(__fmul_rn(__fsub_rn(b[0], a[0]), __fsub_rn(c[1], a[1])),
                             __fmul_rn(__fsub_rn(b[1], a[1]), __fsub_rn(c[0], a[0])));
  const float len = len3(n0, n1, n2);
  if (len > 0.0f) {
    fn[3 * t] = __fdiv_rn(n0, len);
    fn[3 * t + 1] = __fdiv_rn(n1, len);
    fn[3 * t + 2] = __fdiv_rn(n2, len);
  } else {
    fn[3 * t] = 0.0f;
    fn[3 * t + 1] = 0.0f;
    fn[3 * t + 2] = 1.0f;
  }
}

// ---- 2. voxelisation ---------------------------------------------------------

struct Chunk {
  int lo[3], hi[3];    // voxel range of the chunk, inclusive
  uint32_t shift;      // 3 * (depth - chunk_levels): bits of a code inside the chunk
  uint32_t tri_bits;   // bits of the triangle index in a key
};

// Walks the host builder's candidate voxels of triangle t inside the chunk;
// calls emit(code) for each overlapping voxel, in the host's order.
template <class Emit>
__device__ __forceinline__ void voxel_walk(const float* __restrict__ V,
                                           const uint32_t* __restrict__ T, uint64_t t,
                                           uint32_t depth, const Chunk& ch, Emit&& emit) {
  const uint32_t R = 1u << depth;
  const float Rf = (float)R;
  const float inv = __fdiv_rn(1.0f, Rf);
  const float h = __fmul_rn(0.5f, inv);
  float a[3], b[3], c[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    a[k] = V[3 * (uint64_t)T[3 * t] + k];
    b[k] = V[3 * (uint64_t)T[3 * t + 1] + k];
    c[k] = V[3 * (uint64_t)T[3 * t + 2] + k];
  }
  const float n[3] = {__fsub_rn(__fmul_rn(__fsub_rn(b[1], a[1]), __fsub_rn(c[2], a[2])),
                                __fmul_rn(__fsub_rn(b[2], a[2]), __fsub_rn(c[1], a[1]))),
                      __fsub_rn(__fmul_rn(__fsub_rn(b[2], a[2]), __fsub_rn(c[0], a[0])),
                                __fmul_rn(__fsub_rn(b[0], a[0]), __fsub_rn(c[2], a[2]))),
                      __fsub_rn(__fmul_rn(__fsub_rn(b[0], a[0]), __fsub_rn(c[1], a[1])),
                                __fmul_rn(__fsub_rn(b[1], a[1]), __fsub_rn(c[0], a[0])))};
  int lo[3], hi[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float mn = smin(a[k], smin(b[k], c[k]));
    const float mx = smax(a[k], smax(b[k], c[k]));
    lo[k] = max(0, cell_floor(__fmul_rn(__fadd_rn(mn, 0.5f), Rf), R));
    hi[k] = min((int)R - 1, cell_floor(__fmul_rn(__fadd_rn(mx, 0.5f), Rf), R));
    if (lo[k] > hi[k]) lo[k] = hi[k] + 1;
  }
  if (lo[0] > hi[0] || lo[1] > hi[1] || lo[2] > hi[2]) return;
  int w = 0;
  if (fabsf(n[1]) > fabsf(n[w])) w = 1;
  if (fabsf(n[2]) > fabsf(n[w])) w = 2;
  const int u = (w + 1) % 3, v = (w + 2) % 3;
  const float pd = dot3(n[0], n[1], n[2], a);
  // the chunk restricts the (u, v) range and each column's w range
  const int ulo = max(lo[u], ch.lo[u]), uhi = min(hi[u], ch.hi[u]);
  const int vlo = max(lo[v], ch.lo[v]), vhi = min(hi[v], ch.hi[v]);
  for (int iu = ulo; iu <= uhi; ++iu)
    for (int iv = vlo; iv <= vhi; ++iv) {
      int wlo = lo[w], whi = hi[w];
      if (n[w] != 0.0f) {
        const float u0 = __fadd_rn(-0.5f, __fmul_rn((float)iu, inv)), u1 = __fadd_rn(u0, inv);
        const float v0 = __fadd_rn(-0.5f, __fmul_rn((float)iv, inv)), v1 = __fadd_rn(v0, inv);
        float wmin = 1e30f, wmax = -1e30f;
        const float us[2] = {u0, u1}, vs[2] = {v0, v1};
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const float ww = __fdiv_rn(
                __fsub_rn(__fsub_rn(pd, __fmul_rn(n[u], us[i])), __fmul_rn(n[v], vs[j])), n[w]);
            wmin = smin(wmin, ww);
            wmax = smax(wmax, ww);
          }
        wlo = max(wlo, cell_floor(__fmul_rn(__fadd_rn(wmin, 0.5f), Rf), R) - 1);
        whi = min(whi, cell_floor(__fmul_rn(__fadd_rn(wmax, 0.5f), Rf), R) + 1);
      }
      wlo = max(wlo, ch.lo[w]);
      whi = min(whi, ch.hi[w]);
      for (int iw = wlo; iw <= whi; ++iw) {
        int ijk[3];
        ijk[u] = iu;
        ijk[v] = iv;
        ijk[w] = iw;
        const float bc[3] = {__fadd_rn(-0.5f, __fmul_rn(__fadd_rn((float)ijk[0], 0.5f), inv)),
                             __fadd_rn(-0.5f, __fmul_rn(__fadd_rn((float)ijk[1], 0.5f), inv)),
                             __fadd_rn(-0.5f, __fmul_rn(__fadd_rn((float)ijk[2], 0.5f), inv))};
        if (tri_box_overlap(bc, h, a, b, c))
          emit(morton3((uint32_t)ijk[0], (uint32_t)ijk[1], (uint32_t)ijk[2]));
      }
    }
}

__global__ void voxel_count_kernel(const float* __restrict__ V, const uint32_t* __restrict__ T,
                                   uint64_t nt, uint32_t depth, Chunk ch,
                                   uint64_t* __restrict__ counts) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  uint64_t n = 0;
  voxel_walk(V, T, t, depth, ch, [&](uint64_t) { ++n; });
  counts[t] = n;
}

__global__ void voxel_emit_kernel(const float* __restrict__ V, const uint32_t* __restrict__ T,
                                  uint64_t nt, uint32_t depth, Chunk ch,
                                  const uint64_t* __restrict__ offsets,
                                  uint64_t* __restrict__ keys) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  uint64_t pos = offsets[t];
  const uint64_t low = ch.shift >= 64 ? ~0ull : ((1ull << ch.shift) - 1ull);
  voxel_walk(V, T, t, depth, ch,
             [&](uint64_t code) { keys[pos++] = ((code & low) << ch.tri_bits) | t; });
}

// ---- 3. leaves -----------------------------------------------------------------

__global__ void run_heads_kernel(const uint64_t* __restrict__ keys, uint64_t n, uint32_t tri_bits,
                                 uint32_t* __restrict__ heads) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  heads[i] = (i == 0 || (keys[i] >> tri_bits) != (keys[i - 1] >> tri_bits)) ? 1u : 0u;
}

// One thread per run of equal codes: the normalised sum of the face normals
// in triangle order (host: build_mesh_leaves' final loop).
__global__ void leaf_reduce_kernel(const uint64_t* __restrict__ keys, uint64_t n,
                                   uint32_t tri_bits, uint64_t chunk_base,
                                   const uint32_t* __restrict__ heads,
                                   const uint32_t* __restrict__ run_of,
                                   const float* __restrict__ fn, uint64_t* __restrict__ codes,
                                   svo_attrib* __restrict__ attribs) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !heads[i]) return;
  const uint64_t code = keys[i] >> tri_bits;
  const uint64_t tmask = (1ull << tri_bits) - 1ull;
  float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f;
  uint64_t j = i;
  do {
    const uint64_t t = keys[j] & tmask;
    s0 = __fadd_rn(s0, fn[3 * t]);
    s1 = __fadd_rn(s1, fn[3 * t + 1]);
    s2 = __fadd_rn(s2, fn[3 * t + 2]);
    ++j;
  } while (j < n && (keys[j] >> tri_bits) == code);
  const float len = len3(s0, s1, s2);
  if (len > 0.0f) {
    s0 = __fdiv_rn(s0, len);
    s1 = __fdiv_rn(s1, len);
    s2 = __fdiv_rn(s2, len);
  } else {
    s0 = 0.0f;
    s1 = 0.0f;
    s2 = 1.0f;
  }
  const uint32_t r = run_of[i];
  codes[r] = chunk_base | code;
  const uint32_t packed = pack_normal(s0, s1, s2);
  attribs[r] = svo_attrib{packed, packed};  // colour = normal * 0.5 + 0.5 = the packed normal
}

__device__ __forceinline__ uint32_t compact3(uint64_t x) {
  x &= 0x1249249249249249ull;
  x = (x ^ (x >> 2)) & 0x10c30c30c30c30c3ull;
  x = (x ^ (x >> 4)) & 0x100f00f00f00f00full;
  x = (x ^ (x >> 8)) & 0x1f0000ff0000ffull;
  x = (x ^ (x >> 16)) & 0x1f00000000ffffull;
  x = (x ^ (x >> 32)) & 0x1fffffull;
  return (uint32_t)x;
}

// leaf_contribution of the host builder (csrc/scene.cpp), operation for
// operation: the reference's interpolated vertex normal and colour of one
// triangle at the voxel centre c.
__device__ void leaf_contribution(const float* __restrict__ V, const float* __restrict__ N,
                                  const float* __restrict__ C, const uint32_t* tri,
                                  const float c[3], float n_out[3], float c_out[3]) {
  const float* p0 = V + 3 * (uint64_t)tri[0];
  const float* p1 = V + 3 * (uint64_t)tri[1];
  const float* p2 = V + 3 * (uint64_t)tri[2];
  const float* n0 = N + 3 * (uint64_t)tri[0];
  const float* n1 = N + 3 * (uint64_t)tri[1];
  const float* n2 = N + 3 * (uint64_t)tri[2];
  const float* c0 = C + 3 * (uint64_t)tri[0];
  const float* c1 = C + 3 * (uint64_t)tri[1];
  const float* c2 = C + 3 * (uint64_t)tri[2];
  float d[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) d[k] = __fdiv_rn(__fadd_rn(__fadd_rn(n0[k], n1[k]), n2[k]), 3.0f);
  float len = len3(d[0], d[1], d[2]);
  if (len > 0.0f) {
#pragma unroll
    for (int k = 0; k < 3; ++k) d[k] = __fdiv_rn(d[k], len);
  }
  const float e1[3] = {__fsub_rn(p1[0], p0[0]), __fsub_rn(p1[1], p0[1]), __fsub_rn(p1[2], p0[2])};
  const float e2[3] = {__fsub_rn(p2[0], p0[0]), __fsub_rn(p2[1], p0[1]), __fsub_rn(p2[2], p0[2])};
  const float pv[3] = {__fsub_rn(__fmul_rn(d[1], e2[2]), __fmul_rn(d[2], e2[1])),
                       __fsub_rn(__fmul_rn(d[2], e2[0]), __fmul_rn(d[0], e2[2])),
                       __fsub_rn(__fmul_rn(d[0], e2[1]), __fmul_rn(d[1], e2[0]))};
  const float det = dot3(e1[0], e1[1], e1[2], pv);
  float u = 0.0f, v = 0.0f;
  if (!(det > -1e-8f && det < 1e-8f)) {
    const float inv = __fdiv_rn(1.0f, det);
    const float tv[3] = {__fsub_rn(c[0], p0[0]), __fsub_rn(c[1], p0[1]), __fsub_rn(c[2], p0[2])};
    u = __fmul_rn(dot3(tv[0], tv[1], tv[2], pv), inv);
    const float qv[3] = {__fsub_rn(__fmul_rn(tv[1], e1[2]), __fmul_rn(tv[2], e1[1])),
                         __fsub_rn(__fmul_rn(tv[2], e1[0]), __fmul_rn(tv[0], e1[2])),
                         __fsub_rn(__fmul_rn(tv[0], e1[1]), __fmul_rn(tv[1], e1[0]))};
    v = __fmul_rn(dot3(d[0], d[1], d[2], qv), inv);
  }
  u = u < 0.0f ? 0.0f : (u > 1.0f ? 1.0f : u);
  v = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
  const float w = __fsub_rn(__fsub_rn(1.0f, u), v);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    n_out[k] = __fadd_rn(__fadd_rn(__fmul_rn(n0[k], w), __fmul_rn(n1[k], u)), __fmul_rn(n2[k], v));
    c_out[k] = __fadd_rn(__fadd_rn(__fmul_rn(c0[k], w), __fmul_rn(c1[k], u)), __fmul_rn(c2[k], v));
  }
  len = len3(n_out[0], n_out[1], n_out[2]);
  if (len > 0.0f) {
#pragma unroll
    for (int k = 0; k < 3; ++k) n_out[k] = __fdiv_rn(n_out[k], len);
  }
}

// One thread per run of equal codes, with per-vertex attributes: the mean of
// the triangles' interpolated normals (normalised) and colours.
__global__ void leaf_reduce_attr_kernel(const uint64_t* __restrict__ keys, uint64_t n,
                                        uint32_t tri_bits, uint64_t chunk_base, uint32_t depth,
                                        const uint32_t* __restrict__ heads,
                                        const uint32_t* __restrict__ run_of,
                                        const float* __restrict__ V, const float* __restrict__ N,
                                        const float* __restrict__ C,
                                        const uint32_t* __restrict__ T,
                                        uint64_t* __restrict__ codes,
                                        svo_attrib* __restrict__ attribs) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !heads[i]) return;
  const uint64_t code = keys[i] >> tri_bits;
  const uint64_t full = chunk_base | code;
  const uint64_t tmask = (1ull << tri_bits) - 1ull;
  const float inv_r = __fdiv_rn(1.0f, (float)(1u << depth));
  const uint32_t x = compact3(full >> 2), y = compact3(full >> 1), z = compact3(full);
  const float c[3] = {__fadd_rn(-0.5f, __fmul_rn(__fadd_rn((float)x, 0.5f), inv_r)),
                      __fadd_rn(-0.5f, __fmul_rn(__fadd_rn((float)y, 0.5f), inv_r)),
                      __fadd_rn(-0.5f, __fmul_rn(__fadd_rn((float)z, 0.5f), inv_r))};
  float sn[3] = {0.0f, 0.0f, 0.0f}, sc[3] = {0.0f, 0.0f, 0.0f};
  uint64_t j = i;
  do {
    const uint64_t t = keys[j] & tmask;
    float nn[3], cc[3];
    leaf_contribution(V, N, C, T + 3 * t, c, nn, cc);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      sn[k] = __fadd_rn(sn[k], nn[k]);
      sc[k] = __fadd_rn(sc[k], cc[k]);
    }
    ++j;
  } while (j < n && (keys[j] >> tri_bits) == code);
  const float cnt = (float)(j - i);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    sn[k] = __fdiv_rn(sn[k], cnt);
    sc[k] = __fdiv_rn(sc[k], cnt);
  }
  const float len = len3(sn[0], sn[1], sn[2]);
  if (len > 0.0f) {
#pragma unroll
    for (int k = 0; k < 3; ++k) sn[k] = __fdiv_rn(sn[k], len);
  } else {
    sn[0] = 0.0f;
    sn[1] = 0.0f;
    sn[2] = 1.0f;
  }
  const uint32_t r = run_of[i];
  codes[r] = full;
  attribs[r] = svo_attrib{pack_normal(sn[0], sn[1], sn[2]), pack_color(sc[0], sc[1], sc[2])};
}

// ---- 4. levels -------------------------------------------------------------------

__global__ void parent_heads_kernel(const uint64_t* __restrict__ codes, uint64_t n,
                                    uint32_t* __restrict__ heads) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  heads[i] = (i == 0 || (codes[i] >> 3) != (codes[i - 1] >> 3)) ? 1u : 0u;
}

// One thread per parent (host: octree_from_leaves' inner loop).
__global__ void parent_reduce_kernel(const uint64_t* __restrict__ cc,
                                     const svo_attrib* __restrict__ ca, uint64_t n,
                                     const uint32_t* __restrict__ heads,
                                     const uint32_t* __restrict__ run_of,
                                     uint64_t* __restrict__ pc, uint8_t* __restrict__ pm,
                                     uint32_t* __restrict__ pf, svo_attrib* __restrict__ pa) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !heads[i]) return;
  const uint64_t parent = cc[i] >> 3;
  uint32_t mask = 0;
  float n0 = 0.0f, n1 = 0.0f, n2 = 0.0f, c0 = 0.0f, c1 = 0.0f, c2 = 0.0f;
  uint64_t j = i;
  do {
    mask |= 1u << (uint32_t)(cc[j] & 7u);
    float v[3];
    unpack_color(ca[j].packed_normal, v);
    n0 = __fadd_rn(n0, __fmul_rn(__fsub_rn(v[0], 0.5f), 2.0f));
    n1 = __fadd_rn(n1, __fmul_rn(__fsub_rn(v[1], 0.5f), 2.0f));
    n2 = __fadd_rn(n2, __fmul_rn(__fsub_rn(v[2], 0.5f), 2.0f));
    unpack_color(ca[j].packed_color, v);
    c0 = __fadd_rn(c0, v[0]);
    c1 = __fadd_rn(c1, v[1]);
    c2 = __fadd_rn(c2, v[2]);
    ++j;
  } while (j < n && (cc[j] >> 3) == parent);
  const float cnt = (float)(j - i);
  n0 = __fdiv_rn(n0, cnt);
  n1 = __fdiv_rn(n1, cnt);
  n2 = __fdiv_rn(n2, cnt);
  c0 = __fdiv_rn(c0, cnt);
  c1 = __fdiv_rn(c1, cnt);
  c2 = __fdiv_rn(c2, cnt);
  const float len = len3(n0, n1, n2);
  if (len > 0.0f) {
    n0 = __fdiv_rn(n0, len);
    n1 = __fdiv_rn(n1, len);
    n2 = __fdiv_rn(n2, len);
  } else {
    n0 = 0.0f;
    n1 = 0.0f;
    n2 = 1.0f;
  }
  const uint32_t r = run_of[i];
  pc[r] = parent;
  pm[r] = (uint8_t)mask;
  pf[r] = (uint32_t)i;
  pa[r] = svo_attrib{pack_normal(n0, n1, n2), pack_color(c0, c1, c2)};
}

// ---- 5. treelet cut ------------------------------------------------------------

constexpr int kMaxLevels = 22;

struct LevelPtrs {
  const uint8_t* masks[kMaxLevels];
  const uint32_t* first[kMaxLevels];
  const svo_attrib* attribs[kMaxLevels];
};

struct Partition {           // treelets rooted at one boundary level
  uint32_t root_level;
  uint32_t stop_level;
  uint32_t gid_base;         // gid of the partition's first treelet
  uint32_t count;            // treelets in the partition (nodes at root_level)
};

struct CutParams {
  Partition parts[kMaxLevels];
  uint32_t num_parts;
  uint32_t depth;
  uint64_t N;                // nodes per slot
};

// Subtree ranges of treelet (part, root index): lo/hi per level and the
// treelet's local offset of each level.  Returns the node count.
__device__ uint64_t treelet_ranges(const LevelPtrs& L, uint32_t r, uint32_t s, uint64_t root,
                                   uint64_t* lo, uint64_t* hi, uint64_t* off) {
  lo[0] = root;
  hi[0] = root + 1;
  off[0] = 0;
  uint64_t total = 1;
  for (uint32_t l = r; l < s; ++l) {
    const uint32_t k = l - r;
    const uint64_t last = hi[k] - 1;
    lo[k + 1] = L.first[l][lo[k]];
    hi[k + 1] = (uint64_t)L.first[l][last] + (uint64_t)__popc(L.masks[l][last]);
    off[k + 1] = total;
    total += hi[k + 1] - lo[k + 1];
  }
  return total;
}

__global__ void treelet_sizes_kernel(LevelPtrs L, CutParams cp, uint32_t num_treelets,
                                     unsigned long long* __restrict__ stats) {
  const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= num_treelets) return;
  uint32_t p = 0;
  while (p + 1 < cp.num_parts && gid >= cp.parts[p + 1].gid_base) ++p;
  const Partition& P = cp.parts[p];
  uint64_t lo[kMaxLevels], hi[kMaxLevels], off[kMaxLevels];
  const uint64_t n = treelet_ranges(L, P.root_level, P.stop_level, gid - P.gid_base, lo, hi, off);
  atomicMax(stats, (unsigned long long)n);
  atomicAdd(stats + 1, (unsigned long long)n);
}

// One block per treelet: its slot (slot = gid, as insert_all fills an empty
// pool) with every sub-treelet root copied into this treelet's leaf and
// re-pointed (insert_treelet's patch), leaf flags of resident sub-treelets
// cleared, tail left zero.
__global__ void __launch_bounds__(256) cut_kernel(LevelPtrs L, CutParams cp,
                                                  uint32_t num_treelets,
                                                  uint2* __restrict__ nodes,
                                                  svo_attrib* __restrict__ attribs) {
  const uint32_t gid = blockIdx.x;
  if (gid >= num_treelets) return;
  __shared__ uint64_t lo[kMaxLevels], hi[kMaxLevels], off[kMaxLevels];
  __shared__ uint32_t part;
  if (threadIdx.x == 0) {
    uint32_t p = 0;
    while (p + 1 < cp.num_parts && gid >= cp.parts[p + 1].gid_base) ++p;
    part = p;
    treelet_ranges(L, cp.parts[p].root_level, cp.parts[p].stop_level, gid - cp.parts[p].gid_base,
                   lo, hi, off);
  }
  __syncthreads();
  const Partition& P = cp.parts[part];
  const uint32_t r = P.root_level, s = P.stop_level, D = cp.depth;
  const uint64_t base = (uint64_t)gid * cp.N;
  // the sub-treelets' partition and its stop level (their roots' leaf flags)
  const bool has_sub = s < D;
  const uint32_t sub_base = has_sub ? cp.parts[part + 1].gid_base : 0u;
  const uint32_t sub_stop = has_sub ? cp.parts[part + 1].stop_level : 0u;
  for (uint32_t l = r; l <= s; ++l) {
    const uint32_t k = l - r;
    const uint64_t lo_l = lo[k], cnt = hi[k] - lo[k];
    for (uint64_t e = threadIdx.x; e < cnt; e += blockDim.x) {
      const uint64_t g = lo_l + e;
      const uint64_t p = off[k] + e;
      attribs[base + p] = L.attribs[l][g];
      uint2 rec;
      if (l < s) {
        const uint32_t m = L.masks[l][g];
        const uint64_t child = off[k + 1] + ((uint64_t)L.first[l][g] - lo[k + 1]);
        const uint32_t leaf = (l + 1 == s && s == D) ? m : 0u;
        rec = make_uint2((uint32_t)(child - p), (m << 8) | leaf);
      } else if (!has_sub) {
        rec = make_uint2(0u, 0u);
      } else {
        // leaf holding a copy of sub-treelet c's root, first child at c's slot + 1;
        // the copy is taken when c is inserted, before c's own sub-treelets
        // clear the leaf flags in c's slot, so it keeps them
        const uint64_t c = (uint64_t)sub_base + g;
        const uint32_t m = L.masks[l][g];
        const uint32_t leaf = (l + 1 == sub_stop) ? m : 0u;
        rec = make_uint2((uint32_t)((c * cp.N + 1u) - (base + p)), (m << 8) | leaf);
      }
      nodes[base + p] = rec;
    }
  }
}

// ---- host side -----------------------------------------------------------------------

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) {
    o.p = nullptr;
    o.n = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      reset();
      p = o.p;
      n = o.n;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DevBuf() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t count) {
    reset();
    if (count == 0) count = 1;
    const cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    n = count;
    return cudaSuccess;
  }
};

struct Level {
  uint64_t size = 0;
  DevBuf<uint8_t> masks;
  DevBuf<uint32_t> first;
  DevBuf<svo_attrib> attribs;
};

uint32_t bits_for(uint64_t v) {
  uint32_t b = 1;
  while (b < 64 && (1ull << b) < v) ++b;
  return b;
}

// The host builder's stop_level (csrc/scene.cpp).
uint32_t stop_level_of(uint32_t D, uint32_t L, uint32_t r) {
  if (L == 0) return D;
  const uint32_t m = (D - r) % L;
  uint32_t stop = r + (m == 0 ? L : m);
  if (stop == r + 1 && stop < D && r > 0) stop = std::min(D, stop + L);
  return stop;
}

#define GB_TRY(x)                                              \
  do {                                                         \
    const cudaError_t e_ = (x);                                \
    if (e_ != cudaSuccess) return cuda_status(e_);             \
  } while (0)

unsigned grid_of(uint64_t n, unsigned threads) {
  return (unsigned)((n + threads - 1) / threads);
}

// exclusive sum of u32 flags into u32 positions; returns the total
int scan_flags(const uint32_t* flags, uint32_t* pos, uint64_t n, uint64_t* total,
               cudaStream_t st) {
  size_t bytes = 0;
  GB_TRY(cub::DeviceScan::ExclusiveSum(nullptr, bytes, flags, pos, n, st));
  DevBuf<uint8_t> tmp;
  GB_TRY(tmp.alloc(bytes));
  GB_TRY(cub::DeviceScan::ExclusiveSum(tmp.p, bytes, flags, pos, n, st));
  uint32_t last_pos = 0, last_flag = 0;
  GB_TRY(cudaMemcpyAsync(&last_pos, pos + n - 1, 4, cudaMemcpyDeviceToHost, st));
  GB_TRY(cudaMemcpyAsync(&last_flag, flags + n - 1, 4, cudaMemcpyDeviceToHost, st));
  GB_TRY(cudaStreamSynchronize(st));
  *total = (uint64_t)last_pos + last_flag;
  return SVO_OK;
}

}  // namespace

int DeviceScene::build_mesh(const float* h_vertices, const float* h_normals,
                            const float* h_colors, uint64_t nv, const uint32_t* h_triangles,
                            uint64_t nt, uint32_t depth_, uint32_t treelet_levels,
                            cudaStream_t st) {
  if (depth_ < 1 || depth_ > 21) return SVO_ERR_RANGE;
  if (nt == 0 || nv == 0) return SVO_ERR_INVALID;
  if ((h_normals == nullptr) != (h_colors == nullptr)) return SVO_ERR_INVALID;
  for (uint64_t i = 0; i < 3 * nt; ++i)
    if (h_triangles[i] >= nv) return SVO_ERR_INVALID;
  depth = depth_;
  const uint32_t tri_bits = bits_for(nt);
  // chunk levels: enough that a key (code inside the chunk, triangle) fits 64 bits
  uint32_t chunk_levels = 1;
  while (chunk_levels < depth && 3 * (depth - chunk_levels) + tri_bits > 64) ++chunk_levels;
  if (chunk_levels > 3 || 3 * (depth - chunk_levels) + tri_bits > 64) return SVO_ERR_RANGE;
  chunk_levels = std::min(chunk_levels, depth);

  DevBuf<float> dV, dFn, dN, dC;
  DevBuf<uint32_t> dT;
  GB_TRY(dV.alloc(3 * nv));
  GB_TRY(dT.alloc(3 * nt));
  GB_TRY(dFn.alloc(3 * nt));
  GB_TRY(cudaMemcpyAsync(dV.p, h_vertices, 3 * nv * sizeof(float), cudaMemcpyHostToDevice, st));
  const bool attributed = h_normals != nullptr;
  if (attributed) {
    GB_TRY(dN.alloc(3 * nv));
    GB_TRY(dC.alloc(3 * nv));
    GB_TRY(cudaMemcpyAsync(dN.p, h_normals, 3 * nv * sizeof(float), cudaMemcpyHostToDevice, st));
    GB_TRY(cudaMemcpyAsync(dC.p, h_colors, 3 * nv * sizeof(float), cudaMemcpyHostToDevice, st));
  }
  GB_TRY(cudaMemcpyAsync(dT.p, h_triangles, 3 * nt * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  face_normals_kernel<<<grid_of(nt, 256), 256, 0, st>>>(dV.p, dT.p, nt, dFn.p);
  GB_TRY(cudaGetLastError());

  // -- voxelise chunk by chunk; each chunk's leaves are sorted and unique
  const uint32_t R = 1u << depth;
  const uint32_t C = 1u << chunk_levels;  // chunks per axis
  const uint32_t cs = R / C;              // voxels per chunk per axis
  DevBuf<uint64_t> counts, offsets;
  GB_TRY(counts.alloc(nt));
  GB_TRY(offsets.alloc(nt));
  std::vector<DevBuf<uint64_t>> chunk_codes;
  std::vector<DevBuf<svo_attrib>> chunk_attr;
  std::vector<uint64_t> chunk_leaves;
  const uint32_t num_chunks = C * C * C;
  for (uint32_t ci = 0; ci < num_chunks; ++ci) {
    // chunk ci in Morton order: its code prefix is ci
    uint32_t cxyz[3] = {0, 0, 0};
    for (uint32_t b = 0; b < chunk_levels; ++b) {
      cxyz[0] |= ((ci >> (3 * b + 2)) & 1u) << b;
      cxyz[1] |= ((ci >> (3 * b + 1)) & 1u) << b;
      cxyz[2] |= ((ci >> (3 * b)) & 1u) << b;
    }
    Chunk ch;
    for (int k = 0; k < 3; ++k) {
      ch.lo[k] = (int)(cxyz[k] * cs);
      ch.hi[k] = (int)((cxyz[k] + 1) * cs) - 1;
    }
    ch.shift = 3 * (depth - chunk_levels);
    ch.tri_bits = tri_bits;
    voxel_count_kernel<<<grid_of(nt, 128), 128, 0, st>>>(dV.p, dT.p, nt, depth, ch, counts.p);
    GB_TRY(cudaGetLastError());
    size_t bytes = 0;
    GB_TRY(cub::DeviceScan::ExclusiveSum(nullptr, bytes, counts.p, offsets.p, nt, st));
    {
      DevBuf<uint8_t> tmp;
      GB_TRY(tmp.alloc(bytes));
      GB_TRY(cub::DeviceScan::ExclusiveSum(tmp.p, bytes, counts.p, offsets.p, nt, st));
    }
    uint64_t last_off = 0, last_cnt = 0;
    GB_TRY(cudaMemcpyAsync(&last_off, offsets.p + nt - 1, 8, cudaMemcpyDeviceToHost, st));
    GB_TRY(cudaMemcpyAsync(&last_cnt, counts.p + nt - 1, 8, cudaMemcpyDeviceToHost, st));
    GB_TRY(cudaStreamSynchronize(st));
    const uint64_t P = last_off + last_cnt;
    pairs += P;
    chunk_codes.emplace_back();
    chunk_attr.emplace_back();
    chunk_leaves.push_back(0);
    if (P == 0) continue;
    DevBuf<uint64_t> keys, sorted;
    GB_TRY(keys.alloc(P));
    GB_TRY(sorted.alloc(P));
    voxel_emit_kernel<<<grid_of(nt, 128), 128, 0, st>>>(dV.p, dT.p, nt, depth, ch, offsets.p,
                                                       keys.p);
    GB_TRY(cudaGetLastError());
    bytes = 0;
    const int end_bit = (int)(ch.shift + tri_bits);
    GB_TRY(cub::DeviceRadixSort::SortKeys(nullptr, bytes, keys.p, sorted.p, P, 0, end_bit, st));
    {
      DevBuf<uint8_t> tmp;
      GB_TRY(tmp.alloc(bytes));
      GB_TRY(cub::DeviceRadixSort::SortKeys(tmp.p, bytes, keys.p, sorted.p, P, 0, end_bit, st));
    }
    keys.reset();
    DevBuf<uint32_t> heads, run_of;
    GB_TRY(heads.alloc(P));
    GB_TRY(run_of.alloc(P));
    run_heads_kernel<<<grid_of(P, 256), 256, 0, st>>>(sorted.p, P, tri_bits, heads.p);
    GB_TRY(cudaGetLastError());
    uint64_t M = 0;
    int rc = scan_flags(heads.p, run_of.p, P, &M, st);
    if (rc != SVO_OK) return rc;
    GB_TRY(chunk_codes.back().alloc(M));
    GB_TRY(chunk_attr.back().alloc(M));
    if (attributed)
      leaf_reduce_attr_kernel<<<grid_of(P, 256), 256, 0, st>>>(
          sorted.p, P, tri_bits, (uint64_t)ci << ch.shift, depth, heads.p, run_of.p, dV.p, dN.p,
          dC.p, dT.p, chunk_codes.back().p, chunk_attr.back().p);
    else
      leaf_reduce_kernel<<<grid_of(P, 256), 256, 0, st>>>(
          sorted.p, P, tri_bits, (uint64_t)ci << ch.shift, heads.p, run_of.p, dFn.p,
          chunk_codes.back().p, chunk_attr.back().p);
    GB_TRY(cudaGetLastError());
    chunk_leaves.back() = M;
  }
  counts.reset();
  offsets.reset();
  dV.reset();
  dT.reset();
  dFn.reset();
  dN.reset();
  dC.reset();

  // -- concatenate the chunks' leaves
  leaf_voxels = 0;
  for (uint64_t m : chunk_leaves) leaf_voxels += m;
  if (leaf_voxels == 0) return SVO_ERR_INVALID;
  if (leaf_voxels > 0xFFFFFFFFull) return SVO_ERR_RANGE;
  std::vector<Level> levels(depth + 1);
  DevBuf<uint64_t> codes;
  GB_TRY(codes.alloc(leaf_voxels));
  GB_TRY(levels[depth].attribs.alloc(leaf_voxels));
  {
    uint64_t at = 0;
    for (uint32_t ci = 0; ci < num_chunks; ++ci) {
      const uint64_t m = chunk_leaves[ci];
      if (m == 0) continue;
      GB_TRY(cudaMemcpyAsync(codes.p + at, chunk_codes[ci].p, m * 8, cudaMemcpyDeviceToDevice, st));
      GB_TRY(cudaMemcpyAsync(levels[depth].attribs.p + at, chunk_attr[ci].p, m * 8,
                             cudaMemcpyDeviceToDevice, st));
      at += m;
    }
    GB_TRY(cudaStreamSynchronize(st));
    chunk_codes.clear();
    chunk_attr.clear();
  }
  levels[depth].size = leaf_voxels;

  // -- levels bottom-up
  for (int d = (int)depth - 1; d >= 0; --d) {
    const uint64_t n = levels[d + 1].size;
    DevBuf<uint32_t> heads, run_of;
    GB_TRY(heads.alloc(n));
    GB_TRY(run_of.alloc(n));
    parent_heads_kernel<<<grid_of(n, 256), 256, 0, st>>>(codes.p, n, heads.p);
    GB_TRY(cudaGetLastError());
    uint64_t np = 0;
    int rc = scan_flags(heads.p, run_of.p, n, &np, st);
    if (rc != SVO_OK) return rc;
    DevBuf<uint64_t> pcodes;
    Level& lv = levels[d];
    GB_TRY(pcodes.alloc(np));
    GB_TRY(lv.masks.alloc(np));
    GB_TRY(lv.first.alloc(np));
    GB_TRY(lv.attribs.alloc(np));
    parent_reduce_kernel<<<grid_of(n, 256), 256, 0, st>>>(codes.p, levels[d + 1].attribs.p, n,
                                                          heads.p, run_of.p, pcodes.p, lv.masks.p,
                                                          lv.first.p, lv.attribs.p);
    GB_TRY(cudaGetLastError());
    lv.size = np;
    codes = std::move(pcodes);
  }
  if (levels[0].size != 1) return SVO_ERR_INVALID;
  codes.reset();
  octree_nodes = 0;
  for (const Level& lv : levels) octree_nodes += lv.size;

  // -- partitions (treelet boundary levels) and gids
  CutParams cp{};
  cp.depth = depth;
  uint64_t gid_next = 0;
  uint32_t np = 0;
  for (uint32_t r = 0; r < depth; r = stop_level_of(depth, treelet_levels, r)) {
    if (np >= (uint32_t)kMaxLevels) return SVO_ERR_RANGE;
    Partition& P = cp.parts[np++];
    P.root_level = r;
    P.stop_level = stop_level_of(depth, treelet_levels, r);
    P.gid_base = (uint32_t)gid_next;
    P.count = (uint32_t)levels[r].size;
    gid_next += levels[r].size;
    if (gid_next > 0x7FFFFFFFull) return SVO_ERR_RANGE;
  }
  cp.num_parts = np;
  num_treelets = (uint32_t)gid_next;
  LevelPtrs L{};
  for (uint32_t d = 0; d <= depth; ++d) {
    L.masks[d] = levels[d].masks.p;
    L.first[d] = levels[d].first.p;
    L.attribs[d] = levels[d].attribs.p;
  }

  // -- slot size: the largest treelet + 8 (cut_treelets' automatic size)
  {
    DevBuf<unsigned long long> stats;  // {largest treelet, sum of treelet sizes}
    GB_TRY(stats.alloc(2));
    GB_TRY(cudaMemsetAsync(stats.p, 0, 16, st));
    treelet_sizes_kernel<<<grid_of(num_treelets, 128), 128, 0, st>>>(L, cp, num_treelets, stats.p);
    GB_TRY(cudaGetLastError());
    unsigned long long h[2] = {0, 0};
    GB_TRY(cudaMemcpyAsync(h, stats.p, 16, cudaMemcpyDeviceToHost, st));
    GB_TRY(cudaStreamSynchronize(st));
    nodes_per_slot = h[0] + 8;
    treelet_nodes = h[1];
  }
  if (nodes_per_slot < 16 || nodes_per_slot * 8 > 0xFFFFFFFFull) return SVO_ERR_RANGE;
  if ((uint64_t)num_treelets * nodes_per_slot > 0x100000000ull) return SVO_ERR_RANGE;
  cp.N = nodes_per_slot;
  pool_nodes = (uint64_t)num_treelets * nodes_per_slot;

  // -- the pool
  GB_TRY(cudaMalloc(&d_nodes, pool_nodes * sizeof(svo_node)));
  GB_TRY(cudaMalloc(&d_attribs, pool_nodes * sizeof(svo_attrib)));
  GB_TRY(cudaMemsetAsync(d_nodes, 0, pool_nodes * sizeof(svo_node), st));
  GB_TRY(cudaMemsetAsync(d_attribs, 0, pool_nodes * sizeof(svo_attrib), st));
  cut_kernel<<<num_treelets, 256, 0, st>>>(L, cp, num_treelets, reinterpret_cast<uint2*>(d_nodes),
                                           d_attribs);
  GB_TRY(cudaGetLastError());
  GB_TRY(cudaStreamSynchronize(st));
  return SVO_OK;
}

DeviceScene::~DeviceScene() {
  if (d_nodes) cudaFree(d_nodes);
  if (d_attribs) cudaFree(d_attribs);
}

}  // namespace svo
