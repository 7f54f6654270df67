// traverse.cuh -- per-ray sparse-voxel-octree descent for sm_100a.
//
// Restates the reference's two traversals bit for bit:
//   * treelet: sample() in opencl/treeletRenderer_rgba.cl:201-382 over the
//     TreeletMemoryManager incore pool (first-child indices relative to the
//     node, added mod 2^32; src/TreeletMemoryManager.cpp:531-539);
//   * flat:    CpuRaycasterSingleRay3::traversSvo
//     (src/incore/CpuRaycasterSingleRay3.cpp:159-387) over a breadth-first
//     pool with absolute first-child indices.
//
// Every FP32 operation is an explicit round-to-nearest intrinsic, so no
// multiply-add is ever contracted and the operation order is the
// reference's.  Divisions, reciprocals and the square root are the IEEE
// correctly rounded ones.  OpenCL's max(a, b) is (a < b) ? b : a.
//
// Storage.  The reference keeps {node, tMin, tMax, centre} per stack level.
// Two facts shrink that to {node, tMax}:
//   - a level's tMin is only read again after popping back to it, and at the
//     push it was set to the pushed child's tcMax, which is the child frame's
//     tMax and never changes afterwards; so on a pop tMin := popped tMax;
//   - node centres are exact dyadic numbers (-0.5 + (2i+1) 2^-(k+1) for a
//     depth-k node with lattice coordinate i): a child's centre is its
//     parent's +- half the child size, so a pop recovers the parent's centre
//     exactly from the child's and the low bit of the lattice coordinate.
// The stack lives in shared memory, one 8-byte word per level per thread,
// laid out [level][thread] so a warp's accesses are contiguous.
#pragma once
#include <cstdint>

#include "../../include/libsvo_b200.h"

namespace svo {

constexpr int kMaxStack = 24;  // largest supported stack_size / flat depth

struct RayHit {
  uint32_t node;
  float t;
  uint32_t depth;
  uint32_t hit;
  uint32_t flags;
  uint32_t loops;
  uint32_t fetches;  // loop iterations that read the parent node
  // set on a leaf or LOD stop, for the analysis pass and the quality view:
  // the hit child's entry distance, the child size, and whether the child was
  // a leaf (the watchdog stop sets tMin, the current size and leaf = 1, so
  // that quality = sx2 - tScaleRatio * tc_min holds for both)
  float tc_min;
  float sx2;
  uint32_t leaf;
  // SampleResult.nodeCenter: the hit child's centre, or the current node's
  // when the watchdog ends the ray (shadow rays start there)
  float cx, cy, cz;
};

__device__ __forceinline__ float cl_max(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float cl_min(float a, float b) { return (b < a) ? b : a; }

// OpenCL sign(): +-1, the argument itself for +-0, 0 for NaN.
__device__ __forceinline__ float cl_sign(float v) {
  return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : (v == 0.0f ? v : 0.0f));
}

// 2^e for -126 <= e <= 0, exact.
__device__ __forceinline__ float pow2i(int e) { return __int_as_float((127 + e) << 23); }

// Centre coordinate of lattice cell i at depth k: -0.5 + (2i+1) * 2^-(k+1).
__device__ __forceinline__ float cell_center(uint32_t i, int k) {
  return __fadd_rn(-0.5f, __fmul_rn((float)(2u * i + 1u), pow2i(-(k + 1))));
}

// intersectAABB (opencl/treeletRenderer_rgba.cl:100-178) against [-0.5,0.5]^3.
__device__ __forceinline__ bool root_slab(const float o[3], const float d[3], float& t_min,
                                          float& t_max) {
  float t_near = -10000000.0f;
  float t_far = 10000000.0f;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    if (d[i] == 0.0f && (-0.5f > o[i] || 0.5f < o[i])) return false;
    float t1 = __fdiv_rn(__fsub_rn(-0.5f, o[i]), d[i]);
    float t2 = __fdiv_rn(__fsub_rn(0.5f, o[i]), d[i]);
    if (t1 > t2) {
      const float s = t1;
      t1 = t2;
      t2 = s;
    }
    if (t1 > t_near) t_near = t1;
    if (t2 < t_far) t_far = t2;
    if (t_near > t_far) return false;
    if (t_far < 0.0f) return false;
  }
  t_min = t_near;
  t_max = t_far;
  return true;
}

// Node-record fetch policies.  GlobalFetch reads through the read-only
// cache; StagedFetch serves the first `count` records (the top levels of a
// breadth-first treelet pool) from a shared-memory copy.
struct GlobalFetch {
  const uint2* __restrict__ nodes;
  __device__ __forceinline__ uint2 operator()(uint32_t i) const { return __ldg(nodes + i); }
};
struct StagedFetch {
  const uint2* __restrict__ nodes;
  const uint2* top;
  uint32_t count;
  __device__ __forceinline__ uint2 operator()(uint32_t i) const {
    return i < count ? top[i] : __ldg(nodes + i);
  }
};

// A saved traversal state for the cycle search of very long rays (descend):
// frame node, scale and tMin bits, the stacked frames, and the loop and fetch
// counts when it was saved.  Lives in local memory (volatile, so the hot
// loop's registers are not spent on it); only rays that run kCycleFrom
// iterations or more touch it -- on the 1080p icosphere frame the 8 rays the
// watchdog stops, which otherwise run alone for 980 iterations after the rest
// of the frame is done (a search from iteration 64 or 256 made the many long
// rays below 512 pay for the checks and the frame slower).
constexpr uint32_t kCycleFrom = 512;
struct CycleMark {
  uint32_t node, scale, tmin, loops, fetches, next_save;
  uint32_t stack[2 * kMaxStack];
};

// The descent loop.  kFlat selects the CpuRaycasterSingleRay3 rules; S is
// the stack size (treelet) or the octree depth (flat).  `stack` points at
// this thread's column of the shared-memory stack, `stride` words apart.
//
// Per frame (set on push and pop) the registers hold the node, its tMin and
// tMax, its centre, the child size sx2 and half of it, and the node record,
// which is loaded as soon as the node is known so the load overlaps the
// entry-point arithmetic of the next iteration.
//
// kSigned: the reference orders each child's slab distances with a compare
// and swap (tx0 > tx1).  When the reciprocal r is finite, rounding is
// monotone, so the swap happens exactly when r < 0 (equal values swap to
// themselves): the near face is lo when r > 0 and hi when r < 0.  A child's
// two faces along an axis are the parent's mid plane c and its outer face
// c +- sx2 (exact dyadic numbers, the values the reference's childCenter +-
// childSizeHalf produce), so each axis costs the distance to the mid plane,
// the distance to the outer face and the max of the two (the far face); the
// min (the near face) is taken only for a valid child, the one case that
// reads tcMin.  Rays with an infinite or NaN reciprocal (a direction
// component of exactly zero) or a -0 origin coordinate (see cast_ray) take
// kSigned = false, the literal compare and swap.
template <bool kFlat, bool kSigned, class Fetch>
__device__ __forceinline__ void descend(const Fetch& fetch, uint64_t num_nodes,
                                        const float o[3], float dx, float dy, float dz, float rx,
                                        float px, float ry, float py, float rz, float pz,
                                        float t_min, float t_max, float tsr, int S, uint2* stack,
                                        int stride, RayHit& h, uint32_t loop_cap) {
  const float eps = 0.00001f;
  // the reference's watchdog, or the caller's smaller cap (cost estimates)
  const uint32_t watchdog = (uint32_t)((S + 1) * (S + 1) * 5);
  const uint32_t max_loops = loop_cap && loop_cap < watchdog ? loop_cap : watchdog;
  int scale = S - 1;
  uint32_t node = 0u;
  float tmin = t_min, tmax = t_max;
  uint32_t ix = 0u, iy = 0u, iz = 0u;  // lattice coordinate at depth S-1-scale
  float cx = 0.0f, cy = 0.0f, cz = 0.0f;
  float sx2 = 0.5f, half = 0.25f;
  bool in_pool = num_nodes > 0u;
  uint2 nd = in_pool ? fetch(0u) : make_uint2(0u, 0u);
  uint32_t loops = 0u, fetches = 0u;
  // pools hold at most 2^32 nodes, so the in-pool test of a 32-bit index is
  // one 32-bit compare against the last index
  const uint32_t last_node = num_nodes ? (uint32_t)(num_nodes - 1u) : 0u;
  uint2* sp = stack;  // the next free stack word: level S-1-scale
  uint32_t check_at = max_loops < kCycleFrom ? max_loops : kCycleFrom;
  volatile CycleMark mark;
  auto capped = [&]() {
    h.flags = SVO_HITFLAG_CAPPED;
    h.loops = loops;
    h.fetches = fetches;
    if (!kFlat) {  // sample() reports the current node as a hit (:268-277)
      h.hit = 1u;
      h.node = node;
      h.depth = (uint32_t)(S - scale);
      h.t = tmin;
      h.cx = cx;
      h.cy = cy;
      h.cz = cz;
      // quality = scale_exp2 - tScaleRatio * tMin, as for a leaf
      h.tc_min = tmin;
      h.sx2 = sx2;
      h.leaf = 1u;
    }
  };

  for (;;) {  // ends by a return, or by a pop above the root
    ++loops;
    if (loops >= check_at) {
      if (loops == max_loops) {
        capped();
        return;
      }
      // Cold path (rays past kCycleFrom iterations only).  The state at the
      // start of an iteration is the frame's node, scale and tMin and the
      // stacked frames: a frame's tMax depends only on its box and the ray,
      // and the box on the nodes stacked above it.  Once that state recurs,
      // the ray repeats the same iterations with period p until the
      // watchdog, so whole periods are skipped (loop and fetch counts
      // advanced by them) and the iterations left run as usual: the watchdog
      // then stops the ray in the state, and with the counts, the reference
      // reaches.  States are saved at iterations kCycleFrom, 2 kCycleFrom, ...
      // (Brent's cycle search) and compared with every later iteration.
      check_at = loops + 1u;
      const uint32_t depth = (uint32_t)(S - 1 - scale);
      bool same = loops > kCycleFrom && mark.node == node && mark.scale == (uint32_t)scale &&
                  mark.tmin == __float_as_uint(tmin);
      for (uint32_t j = 0; same && j < depth; ++j) {
        const uint2 a = stack[j * stride];
        same = a.x == mark.stack[2 * j] && a.y == mark.stack[2 * j + 1];
      }
      if (same) {
        const uint32_t period = loops - mark.loops;
        const uint32_t skip = (max_loops - loops) / period;
        fetches += skip * (fetches - mark.fetches);
        loops += skip * period;
        check_at = max_loops;
        if (loops == max_loops) {
          capped();
          return;
        }
      } else if (loops == kCycleFrom || loops == mark.next_save) {
        mark.node = node;
        mark.scale = (uint32_t)scale;
        mark.tmin = __float_as_uint(tmin);
        mark.loops = loops;
        mark.fetches = fetches;
        mark.next_save = 2u * loops;
        for (uint32_t j = 0; j < depth; ++j) {
          const uint2 a = stack[j * stride];
          mark.stack[2 * j] = a.x;
          mark.stack[2 * j + 1] = a.y;
        }
      }
    }
    bool pop;
    if (kFlat)
      pop = (tmax < 0.0f) || (fabsf(__fsub_rn(tmin, tmax)) < eps) || !(tmin < tmax);
    else
      pop = (tmax < 0.0f) || !(fabsf(__fsub_rn(tmin, tmax)) > eps);
    if (pop) {
      ++scale;
      if (scale >= S) break;
      sp -= stride;
      const uint2 e = *sp;
      tmin = tmax;
      node = e.x;
      tmax = __uint_as_float(e.y);
      // a stacked node passed the in-pool test before its children were
      // tested, so the popped one is in the pool
      in_pool = true;
      nd = fetch(node);
      // parent centre = child centre -+ the child's sx2 (exact)
      cx = __fadd_rn(cx, (ix & 1u) ? -sx2 : sx2);
      cy = __fadd_rn(cy, (iy & 1u) ? -sx2 : sx2);
      cz = __fadd_rn(cz, (iz & 1u) ? -sx2 : sx2);
      ix >>= 1;
      iy >>= 1;
      iz >>= 1;
      half = sx2;  // the parent's half child size is the child's size (exact)
      sx2 = __fmul_rn(sx2, 2.0f);
      continue;
    }
    // childEntryPoint = (o + (tMin + eps) d) - centre and its sign test: in
    // IEEE arithmetic with subnormals, a - b > 0 exactly when a > b (a - b
    // rounds to 0 only when a == b), so the subtraction is left out
    const float te = __fadd_rn(tmin, eps);
    const bool bxp = __fadd_rn(o[0], __fmul_rn(te, dx)) > cx;
    const bool byp = __fadd_rn(o[1], __fmul_rn(te, dy)) > cy;
    const bool bzp = __fadd_rn(o[2], __fmul_rn(te, dz)) > cz;
    float tx0, tx1, ty0, ty1, tz0, tz1;
    float mx = 0.0f, my = 0.0f, mz = 0.0f, ox = 0.0f, oy = 0.0f, oz = 0.0f;
    if (kSigned) {
      // The child's faces are the mid plane c and its outer face c +- sx2;
      // the far one is the farther (the near ones, needed only for a valid
      // child, are taken there).  No NaN and no -0 here, so the hardware
      // min/max give the reference's order bit for bit.
      mx = __fadd_rn(__fmul_rn(rx, cx), px);
      my = __fadd_rn(__fmul_rn(ry, cy), py);
      mz = __fadd_rn(__fmul_rn(rz, cz), pz);
      ox = __fadd_rn(__fmul_rn(rx, __fadd_rn(cx, bxp ? sx2 : -sx2)), px);
      oy = __fadd_rn(__fmul_rn(ry, __fadd_rn(cy, byp ? sx2 : -sx2)), py);
      oz = __fadd_rn(__fmul_rn(rz, __fadd_rn(cz, bzp ? sx2 : -sx2)), pz);
      tx0 = ty0 = tz0 = 0.0f;
      tx1 = fmaxf(mx, ox);
      ty1 = fmaxf(my, oy);
      tz1 = fmaxf(mz, oz);
    } else {
      // child centre (-0.5 + b) * sx2 + c = c +- half; faces ccx -+ half
      const float ccx = __fadd_rn(bxp ? half : -half, cx);
      const float ccy = __fadd_rn(byp ? half : -half, cy);
      const float ccz = __fadd_rn(bzp ? half : -half, cz);
      tx0 = __fadd_rn(__fmul_rn(rx, __fsub_rn(ccx, half)), px);
      tx1 = __fadd_rn(__fmul_rn(rx, __fadd_rn(ccx, half)), px);
      if (tx0 > tx1) {
        const float s = tx0;
        tx0 = tx1;
        tx1 = s;
      }
      ty0 = __fadd_rn(__fmul_rn(ry, __fsub_rn(ccy, half)), py);
      ty1 = __fadd_rn(__fmul_rn(ry, __fadd_rn(ccy, half)), py);
      if (ty0 > ty1) {
        const float s = ty0;
        ty0 = ty1;
        ty1 = s;
      }
      tz0 = __fadd_rn(__fmul_rn(rz, __fsub_rn(ccz, half)), pz);
      tz1 = __fadd_rn(__fmul_rn(rz, __fadd_rn(ccz, half)), pz);
      if (tz0 > tz1) {
        const float s = tz0;
        tz0 = tz1;
        tz1 = s;
      }
    }
    // kSigned: no NaN and no -0 among the distances (see cast_ray), so the
    // hardware min/max equal the reference's max/min bit for bit
    const float tc_max = kSigned ? fminf(tx1, fminf(ty1, tz1)) : cl_min(tx1, cl_min(ty1, tz1));
    auto near_max = [&]() {
      return kSigned ? fmaxf(fminf(mx, ox), fmaxf(fminf(my, oy), fminf(mz, oz)))
                     : cl_max(tx0, cl_max(ty0, tz0));
    };

    if (!in_pool) {
      h.flags = SVO_HITFLAG_BOUNDS;
      h.loops = loops;
      h.fetches = fetches;
      return;
    }
    ++fetches;
    const uint32_t bx = bxp, by = byp, bz = bzp;
    const uint32_t ci = (bx << 2) | (by << 1) | bz;
    const uint32_t masks = nd.y;
    const uint32_t sh = masks >> ci;  // bit 8: valid, bit 0: leaf
    if (sh & 0x100u) {
      const float tc_min = near_max();
      const uint32_t below = __popc(masks & ((0x100u << ci) - 0x100u));
      const uint32_t child = (kFlat ? 0u : node) + nd.x + below;
      const bool leaf = sh & 1u;
      const bool lod = kFlat ? (__fmul_rn(tsr, tc_max) > sx2)
                             : (__fmul_rn(tsr, tc_min) > sx2 || scale == 1);
      if (leaf || lod) {
        h.hit = 1u;
        h.node = child;
        h.depth = (uint32_t)((leaf || kFlat) ? (S - scale) : (S - scale + 1));
        h.t = tmin;
        h.loops = loops;
        h.fetches = fetches;
        h.tc_min = tc_min;
        h.sx2 = sx2;
        h.leaf = leaf ? 1u : 0u;
        h.cx = __fadd_rn(bxp ? half : -half, cx);
        h.cy = __fadd_rn(byp ? half : -half, cy);
        h.cz = __fadd_rn(bzp ? half : -half, cz);
        return;
      }
      if (kFlat && scale == 0) {  // non-leaf below the octree's depth: corrupt pool
        h.flags = SVO_HITFLAG_BOUNDS;
        h.loops = loops;
        h.fetches = fetches;
        return;
      }
      // push: the current frame's tMin becomes tc_max (recovered on pop)
      *sp = make_uint2(node, __float_as_uint(tmax));
      sp += stride;
      --scale;
      node = child;
      in_pool = node <= last_node;
      if (in_pool) nd = fetch(node);
      tmin = tc_min;
      tmax = tc_max;
      ix = (ix << 1) | bx;
      iy = (iy << 1) | by;
      iz = (iz << 1) | bz;
      cx = __fadd_rn(bx ? half : -half, cx);
      cy = __fadd_rn(by ? half : -half, cy);
      cz = __fadd_rn(bz ? half : -half, cz);
      sx2 = half;
      half = __fmul_rn(half, 0.5f);
      continue;
    }
    tmin = tc_max;  // advance to the next sibling
  }
  h.hit = 0u;
  h.node = 0u;
  h.depth = 0u;
  h.t = kFlat ? 0.0f : t_max;
  h.loops = loops;
  h.fetches = fetches;
}

// One ray: root box test, direction clamp, then the descent.  loop_cap > 0
// stops the ray after that many iterations instead of the watchdog's (S+1)^2*5
// (used only to estimate costs; results under a cap are not the reference's).
template <bool kFlat, class Fetch>
__device__ __forceinline__ RayHit cast_ray(const Fetch& fetch, uint64_t num_nodes,
                                           const float o[3], float dx, float dy, float dz,
                                           float tsr, int S, uint2* stack, int stride,
                                           uint32_t loop_cap = 0u) {
  RayHit h;
  h.node = 0u;
  h.t = 0.0f;
  h.depth = 0u;
  h.hit = 0u;
  h.flags = 0u;
  h.loops = 0u;
  h.fetches = 0u;
  h.tc_min = 0.0f;
  h.sx2 = 0.0f;
  h.leaf = 0u;
  h.cx = 0.0f;
  h.cy = 0.0f;
  h.cz = 0.0f;

  float t_min, t_max;
  {
    const float d0[3] = {dx, dy, dz};
    if (!root_slab(o, d0, t_min, t_max)) {
      h.flags = SVO_HITFLAG_BOXMISS;
      return h;
    }
  }
  // Direction clamp: sample() replaces |d| < 1e-4 by 1e-4 * sign(d)
  // (:231-239); traversSvo replaces |d| < 1e-5 by 1e-5 * sign(d) * 10 (:184-186).
  if (kFlat) {
    const float eps = 0.00001f;
    if (fabsf(dx) < eps) dx = __fmul_rn(__fmul_rn(eps, cl_sign(dx)), 10.0f);
    if (fabsf(dy) < eps) dy = __fmul_rn(__fmul_rn(eps, cl_sign(dy)), 10.0f);
    if (fabsf(dz) < eps) dz = __fmul_rn(__fmul_rn(eps, cl_sign(dz)), 10.0f);
  } else {
    const float mn = 0.0001f;
    if (fabsf(dx) < mn) dx = __fmul_rn(mn, cl_sign(dx));
    if (fabsf(dy) < mn) dy = __fmul_rn(mn, cl_sign(dy));
    if (fabsf(dz) < mn) dz = __fmul_rn(mn, cl_sign(dz));
  }
  const float rx = __frcp_rn(dx), px = __fmul_rn(-o[0], rx);
  const float ry = __frcp_rn(dy), py = __fmul_rn(-o[1], ry);
  const float rz = __frcp_rn(dz), pz = __fmul_rn(-o[2], rz);
  // kSigned needs finite reciprocals.  It also takes the hardware min/max:
  // with finite r, a slab distance r * plane + p is -0 only for the plane at
  // 0 when the origin coordinate is -0 and r < 0 (x + (-x) rounds to +0), so
  // rays with a -0 origin coordinate keep the reference's compare/select.
  const bool neg_zero = __float_as_uint(o[0]) == 0x80000000u ||
                        __float_as_uint(o[1]) == 0x80000000u ||
                        __float_as_uint(o[2]) == 0x80000000u;
  if (isfinite(rx) && isfinite(ry) && isfinite(rz) && !neg_zero)
    descend<kFlat, true>(fetch, num_nodes, o, dx, dy, dz, rx, px, ry, py, rz, pz, t_min, t_max,
                         tsr, S, stack, stride, h, loop_cap);
  else
    descend<kFlat, false>(fetch, num_nodes, o, dx, dy, dz, rx, px, ry, py, rz, pz, t_min, t_max,
                          tsr, S, stack, stride, h, loop_cap);
  return h;
}

}  // namespace svo
