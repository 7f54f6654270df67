// oracle.cpp -- CPU restatement of libsvo's per-ray sparse-voxel-octree cast.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
// path in libsvo_b200/csrc; it is never linked into the product library and
// the product never calls it.  Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg load it.
//
// Parity pinning: the traversal below is checked against the reference's own
// OpenCL C source (opencl/treeletRenderer_rgba.cl), compiled for the host as
// C++ through oracle/cl_shim.h by oracle/build_ref.py into oracle/_ref/.  The
// tests compare this restatement with that build ray by ray and pixel by pixel.
//
// Two traversal variants, both restated in the reference's operation order:
//   * treelet  -- sample() in opencl/treeletRenderer_rgba.cl:201-382, over the
//                 TreeletMemoryManager incore pool (relative first-child
//                 indices, uint32 wrap-around, src/TreeletMemoryManager.cpp:531-539).
//   * flat     -- CpuRaycasterSingleRay3::traversSvo
//                 (src/incore/CpuRaycasterSingleRay3.cpp:159-387) over a flat
//                 breadth-first pool with absolute first-child indices
//                 (src/incore/SvoBranch.cpp:233-308).
//
// Floating point: FP32 only, compiled with -ffp-contract=off so that every
// multiply and add rounds separately, exactly as written.  Where OpenCL leaves
// a built-in implementation-defined, this file pins it:
//   normalize(v) = v / sqrt(dot(v, v)) with dot = (x*x + y*y) + z*z,
//   max(a, b)    = (a < b) ? b : a   (OpenCL C 1.x definition of max),
//   min(a, b)    = (b < a) ? b : a,
//   sign(v)      = 1, -1, or v itself for +-0 and 0 for NaN (OpenCL sign()),
//   pow(2, k)    = exact power of two.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

struct V3 {
  float x, y, z;
};

// OpenCL C sign(): +1 for x > 0, -1 for x < 0, x for +-0, 0 for NaN.
inline float cl_sign(float v) {
  if (v > 0.0f) return 1.0f;
  if (v < 0.0f) return -1.0f;
  if (v == 0.0f) return v;
  return 0.0f;
}
inline float cl_max(float a, float b) { return (a < b) ? b : a; }
inline float cl_min(float a, float b) { return (b < a) ? b : a; }
inline float pow2i(int e) { return std::ldexp(1.0f, e); }

inline bool valid_bit(uint32_t masks, uint32_t i) { return (masks >> (i + 8u)) & 1u; }
inline bool leaf_bit(uint32_t masks, uint32_t i) { return (masks >> i) & 1u; }

// getNthchildIdx (opencl/treeletRenderer_rgba.cl:84-95): first child plus the
// number of valid siblings in front of childIdx, wrapping mod 2^32.
inline uint32_t nth_child(uint32_t masks, uint32_t first_child, uint32_t child_idx) {
  uint32_t index = first_child;
  for (uint32_t i = 0; i != child_idx; ++i) index += valid_bit(masks, i) ? 1u : 0u;
  return index;
}

struct Hit {
  uint32_t node;
  float t;
  uint16_t depth;
  uint8_t hit;
  uint8_t flags;
  uint16_t loops;
  uint16_t fetches;
};
static_assert(sizeof(Hit) == 16, "hit record is 16 bytes");

enum : uint8_t { kFlagCapped = 1, kFlagBounds = 2, kFlagBoxMiss = 4 };

// intersectAABB (opencl/treeletRenderer_rgba.cl:100-178): slab test against
// the root cube [-0.5, 0.5]^3 with the unclamped ray direction.
bool root_slab(const V3& o, const V3& d, float& t_min, float& t_max) {
  float t_near = -10000000.0f;
  float t_far = 10000000.0f;
  const float r = 0.5f;
  const float oa[3] = {o.x, o.y, o.z};
  const float da[3] = {d.x, d.y, d.z};
  for (int i = 0; i != 3; ++i) {
    if (da[i] == 0.0f && (-r > oa[i] || r < oa[i])) return false;
    float t1 = (-r - oa[i]) / da[i];
    float t2 = (r - oa[i]) / da[i];
    if (t1 > t2) std::swap(t1, t2);
    if (t1 > t_near) t_near = t1;
    if (t2 < t_far) t_far = t2;
    if (t_near > t_far) return false;
    if (t_far < 0.0f) return false;
  }
  t_min = t_near;
  t_max = t_far;
  return true;
}

struct Frame {
  float tmin, tmax;
  uint32_t node;
  V3 center;
};

// Per-ray statistics: the number of loop iterations that fetched the parent
// node to test a child's valid bit (the algorithmic node reads of the ray).
struct RayCount {
  uint64_t fetches = 0;
};

// The rest of SampleResult on a hit: nodeCenter and quality.
struct Exit {
  V3 center{0.0f, 0.0f, 0.0f};
  float quality = 0.0f;
};

// sample() (opencl/treeletRenderer_rgba.cl:201-382), stack size `S`
// (MAX_STACK_SIZE, 13 in the reference) and maximum descent depth S-1
// (MAX_SVO_RAYCAST_DEPTH).  `out` (optional) receives nodeCenter and quality.
Hit cast_treelet(const uint32_t* nodes, uint64_t num_nodes, V3 o, V3 d, float tsr, int S,
                 RayCount& rc, Exit* out = nullptr) {
  Hit h{};
  float t_min, t_max;
  if (!root_slab(o, d, t_min, t_max)) {
    h.flags = kFlagBoxMiss;
    return h;
  }
  const int scale_max = S;
  int scale = scale_max - 1;
  const float min_normal = 0.0001f;
  const float eps = 0.00001f;
  Frame stack[32];
  stack[scale] = Frame{t_min, t_max, 0u, V3{0.0f, 0.0f, 0.0f}};

  if (std::fabs(d.x) < min_normal) d.x = min_normal * cl_sign(d.x);
  if (std::fabs(d.y) < min_normal) d.y = min_normal * cl_sign(d.y);
  if (std::fabs(d.z) < min_normal) d.z = min_normal * cl_sign(d.z);

  const float rx = 1.0f / d.x, px = -o.x * rx;
  const float ry = 1.0f / d.y, py = -o.y * ry;
  const float rz = 1.0f / d.z, pz = -o.z * rz;

  uint32_t loops = 0, fetches = 0;
  const uint32_t max_loops = (uint32_t)((scale_max + 1) * (scale_max + 1) * 5);

  while (scale < scale_max) {
    Frame& p = stack[scale];
    const float sx2 = pow2i(scale - scale_max);
    const float half = sx2 * 0.5f;
    ++loops;
    if (loops == max_loops) {  // watchdog: reports the current parent as a hit
      h.hit = 1;
      h.node = p.node;
      h.depth = (uint16_t)(scale_max - scale);
      h.t = p.tmin;
      h.loops = (uint16_t)loops;
      h.fetches = (uint16_t)fetches;
      h.flags = kFlagCapped;
      if (out) *out = Exit{p.center, sx2 - tsr * p.tmin};
      return h;
    }
    if (p.tmax < 0.0f) {
      ++scale;
      continue;
    }
    if (!(std::fabs(p.tmin - p.tmax) > eps)) {
      ++scale;
      continue;
    }
    const float te = p.tmin + eps;
    const float ex = (o.x + te * d.x) - p.center.x;
    const float ey = (o.y + te * d.y) - p.center.y;
    const float ez = (o.z + te * d.z) - p.center.z;
    const uint32_t ci = 4u * (ex > 0.0f) + 2u * (ey > 0.0f) + (ez > 0.0f);
    const V3 cc{(-0.5f + (float)((ci & 4u) != 0)) * sx2 + p.center.x,
                (-0.5f + (float)((ci & 2u) != 0)) * sx2 + p.center.y,
                (-0.5f + (float)((ci & 1u) != 0)) * sx2 + p.center.z};
    float tx0 = rx * (cc.x - half) + px, tx1 = rx * (cc.x + half) + px;
    if (tx0 > tx1) std::swap(tx0, tx1);
    float ty0 = ry * (cc.y - half) + py, ty1 = ry * (cc.y + half) + py;
    if (ty0 > ty1) std::swap(ty0, ty1);
    float tz0 = rz * (cc.z - half) + pz, tz1 = rz * (cc.z + half) + pz;
    if (tz0 > tz1) std::swap(tz0, tz1);
    const float tc_min = cl_max(tx0, cl_max(ty0, tz0));
    const float tc_max = cl_min(tx1, cl_min(ty1, tz1));

    if (p.node >= num_nodes) {
      h.flags = kFlagBounds;
      h.loops = (uint16_t)loops;
      h.fetches = (uint16_t)fetches;
      return h;
    }
    ++fetches;
    const uint32_t fc = nodes[2 * (uint64_t)p.node];
    const uint32_t masks = nodes[2 * (uint64_t)p.node + 1];
    if (valid_bit(masks, ci)) {
      const uint32_t child = p.node + nth_child(masks, fc, ci);
      if (leaf_bit(masks, ci)) {
        h.hit = 1;
        h.node = child;
        h.depth = (uint16_t)(scale_max - scale);
        h.t = p.tmin;
        h.loops = (uint16_t)loops;
        h.fetches = (uint16_t)fetches;
        if (out) *out = Exit{cc, sx2 - tsr * tc_min};
        return h;
      }
      if (tsr * tc_min > sx2 || scale_max - scale == scale_max - 1) {
        h.hit = 1;
        h.node = child;
        h.depth = (uint16_t)(scale_max - scale + 1);
        h.t = p.tmin;
        h.loops = (uint16_t)loops;
        h.fetches = (uint16_t)fetches;
        if (out) *out = Exit{cc, 0.0f};
        return h;
      }
      p.tmin = tc_max;
      --scale;
      stack[scale] = Frame{tc_min, tc_max, child, cc};
      continue;
    }
    p.tmin = tc_max;  // advance to the next sibling
  }
  h.hit = 0;
  h.node = 0;
  h.depth = 0;
  h.t = t_max;
  h.loops = (uint16_t)loops;
  h.fetches = (uint16_t)fetches;
  return h;
}

// CpuRaycasterSingleRay3::traversSvo (src/incore/CpuRaycasterSingleRay3.cpp:159-387)
// over a flat pool whose first-child fields are absolute.  `scale_max` is the
// octree's maximum depth (SvoBranch::getMaxDepth()).  The root box test is the
// same slab test as the treelet variant (gloost::BoundingBox is not part of the
// reference).
Hit cast_flat(const uint32_t* nodes, uint64_t num_nodes, V3 o, V3 d, float tsr, int scale_max,
              RayCount& rc) {
  Hit h{};
  float t_min, t_max;
  if (!root_slab(o, d, t_min, t_max)) {
    h.flags = kFlagBoxMiss;
    return h;
  }
  int scale = scale_max - 1;
  const float eps = 0.00001f;
  Frame stack[33];
  stack[scale] = Frame{t_min, t_max, 0u, V3{0.0f, 0.0f, 0.0f}};

  if (std::fabs(d.x) < eps) d.x = eps * cl_sign(d.x) * 10.0f;
  if (std::fabs(d.y) < eps) d.y = eps * cl_sign(d.y) * 10.0f;
  if (std::fabs(d.z) < eps) d.z = eps * cl_sign(d.z) * 10.0f;

  const float rx = 1.0f / d.x, px = -o.x * rx;
  const float ry = 1.0f / d.y, py = -o.y * ry;
  const float rz = 1.0f / d.z, pz = -o.z * rz;

  uint32_t loops = 0, fetches = 0;
  const uint32_t max_loops = (uint32_t)((scale_max + 1) * (scale_max + 1) * 5);
  bool refetch = true;
  Frame p{};
  float sx2 = 0.5f, half = 0.25f;

  while (scale < scale_max) {
    ++loops;
    if (loops == max_loops) {  // watchdog: the flat variant reports a miss
      h.hit = 0;
      h.node = 0;
      h.loops = (uint16_t)loops;
      h.fetches = (uint16_t)fetches;
      h.flags = kFlagCapped;
      return h;
    }
    if (refetch) {
      p = stack[scale];
      sx2 = pow2i(scale - scale_max);
      half = sx2 * 0.5f;
      refetch = false;
    }
    if (p.tmax < 0.0f) {
      ++scale;
      refetch = true;
      continue;
    }
    if (std::fabs(p.tmin - p.tmax) < eps) {
      ++scale;
      refetch = true;
      continue;
    }
    if (!(p.tmin < p.tmax)) {
      ++scale;
      refetch = true;
      continue;
    }
    const float te = p.tmin + eps;
    const float ex = (o.x + te * d.x) - p.center.x;
    const float ey = (o.y + te * d.y) - p.center.y;
    const float ez = (o.z + te * d.z) - p.center.z;
    const uint32_t ci = 4u * (ex > 0.0f) + 2u * (ey > 0.0f) + (ez > 0.0f);
    const V3 cc{(-0.5f + (float)((ci & 4u) != 0)) * sx2 + p.center.x,
                (-0.5f + (float)((ci & 2u) != 0)) * sx2 + p.center.y,
                (-0.5f + (float)((ci & 1u) != 0)) * sx2 + p.center.z};
    float tx0 = rx * (cc.x - half) + px, tx1 = rx * (cc.x + half) + px;
    if (tx0 > tx1) std::swap(tx0, tx1);
    float ty0 = ry * (cc.y - half) + py, ty1 = ry * (cc.y + half) + py;
    if (ty0 > ty1) std::swap(ty0, ty1);
    float tz0 = rz * (cc.z - half) + pz, tz1 = rz * (cc.z + half) + pz;
    if (tz0 > tz1) std::swap(tz0, tz1);
    const float tc_min = cl_max(tx0, cl_max(ty0, tz0));
    const float tc_max = cl_min(tx1, cl_min(ty1, tz1));

    if (p.node >= num_nodes) {
      h.flags = kFlagBounds;
      h.loops = (uint16_t)loops;
      h.fetches = (uint16_t)fetches;
      return h;
    }
    ++fetches;
    const uint32_t fc = nodes[2 * (uint64_t)p.node];
    const uint32_t masks = nodes[2 * (uint64_t)p.node + 1];
    if (valid_bit(masks, ci)) {
      const uint32_t child = nth_child(masks, fc, ci);
      if (leaf_bit(masks, ci)) {
        h.hit = 1;
        h.node = child;
        h.depth = (uint16_t)(scale_max - scale);
        h.t = p.tmin;
        h.loops = (uint16_t)loops;
        h.fetches = (uint16_t)fetches;
        return h;
      }
      if (tsr * tc_max > sx2) {
        h.hit = 1;
        h.node = child;
        h.depth = (uint16_t)(scale_max - scale);
        h.t = p.tmin;
        h.loops = (uint16_t)loops;
        h.fetches = (uint16_t)fetches;
        return h;
      }
      if (scale == 0) {
        // a non-leaf child below the octree's depth: only a corrupt pool gets
        // here, and the reference would index its stack at -1
        h.flags = kFlagBounds;
        h.loops = (uint16_t)loops;
        h.fetches = (uint16_t)fetches;
        return h;
      }
      stack[scale].tmin = tc_max;
      --scale;
      stack[scale] = Frame{tc_min, tc_max, child, cc};
      refetch = true;
      continue;
    }
    p.tmin = tc_max;  // advance (local copy only, as in the reference)
  }
  h.hit = 0;
  h.node = 0;
  h.depth = 0;
  h.t = 0.0f;
  h.loops = (uint16_t)loops;
  h.fetches = (uint16_t)fetches;
  return h;
}

// sampleAnalyse (opencl/treeletRenderer_rgba.cl:773-953): the analysis ray.
// Same descent as sample(); it reports {node, error, sub-treelet gid, tcMin}
// at a leaf or LOD stop and nothing on a miss or when the watchdog fires.
struct Feedback {
  int32_t node_id;
  float error;
  int32_t sub_treelet_gid;
  float t_min;
};
static_assert(sizeof(Feedback) == 16, "FeedBackDataElement is 16 bytes");

Feedback analyse_ray(const uint32_t* nodes, uint64_t num_nodes, V3 o, V3 d, float tsr, int S) {
  Feedback e{0, 0.0f, 0, 9999999.0f};
  float t_min, t_max;
  if (!root_slab(o, d, t_min, t_max)) return e;
  const int scale_max = S;
  int scale = scale_max - 1;
  const float min_normal = 0.0001f;
  const float eps = 0.00001f;
  Frame stack[32];
  stack[scale] = Frame{t_min, t_max, 0u, V3{0.0f, 0.0f, 0.0f}};
  if (std::fabs(d.x) < min_normal) d.x = min_normal * cl_sign(d.x);
  if (std::fabs(d.y) < min_normal) d.y = min_normal * cl_sign(d.y);
  if (std::fabs(d.z) < min_normal) d.z = min_normal * cl_sign(d.z);
  const float rx = 1.0f / d.x, px = -o.x * rx;
  const float ry = 1.0f / d.y, py = -o.y * ry;
  const float rz = 1.0f / d.z, pz = -o.z * rz;
  uint32_t loops = 0;
  const uint32_t max_loops = (uint32_t)((scale_max + 1) * (scale_max + 1) * 5);
  while (scale < scale_max) {
    ++loops;
    if (loops == max_loops) break;
    Frame& p = stack[scale];
    const float sx2 = pow2i(scale - scale_max);
    const float half = sx2 * 0.5f;
    if (p.tmax < 0.0f) {
      ++scale;
      continue;
    }
    if (!(std::fabs(p.tmin - p.tmax) > eps)) {
      ++scale;
      continue;
    }
    const float te = p.tmin + eps;
    const float ex = (o.x + te * d.x) - p.center.x;
    const float ey = (o.y + te * d.y) - p.center.y;
    const float ez = (o.z + te * d.z) - p.center.z;
    const uint32_t ci = 4u * (ex > 0.0f) + 2u * (ey > 0.0f) + (ez > 0.0f);
    const V3 cc{(-0.5f + (float)((ci & 4u) != 0)) * sx2 + p.center.x,
                (-0.5f + (float)((ci & 2u) != 0)) * sx2 + p.center.y,
                (-0.5f + (float)((ci & 1u) != 0)) * sx2 + p.center.z};
    float tx0 = rx * (cc.x - half) + px, tx1 = rx * (cc.x + half) + px;
    if (tx0 > tx1) std::swap(tx0, tx1);
    float ty0 = ry * (cc.y - half) + py, ty1 = ry * (cc.y + half) + py;
    if (ty0 > ty1) std::swap(ty0, ty1);
    float tz0 = rz * (cc.z - half) + pz, tz1 = rz * (cc.z + half) + pz;
    if (tz0 > tz1) std::swap(tz0, tz1);
    const float tc_min = cl_max(tx0, cl_max(ty0, tz0));
    const float tc_max = cl_min(tx1, cl_min(ty1, tz1));
    if (p.node >= num_nodes) return e;
    const uint32_t fc = nodes[2 * (uint64_t)p.node];
    const uint32_t masks = nodes[2 * (uint64_t)p.node + 1];
    if (valid_bit(masks, ci)) {
      const uint32_t child = p.node + nth_child(masks, fc, ci);
      if (leaf_bit(masks, ci)) {
        e.node_id = (int32_t)child;
        e.error = sx2 - tsr * tc_min;
        e.sub_treelet_gid = child < num_nodes ? (int32_t)nodes[2 * (uint64_t)child] : 0;
        e.t_min = tc_min;
        return e;
      }
      if (tsr * tc_min > sx2 || scale_max - scale == scale_max - 1) {
        e.node_id = (int32_t)child;
        e.error = (tsr * tc_min > sx2) ? 1.0f : 0.0f;
        e.sub_treelet_gid = 0;
        e.t_min = tc_min;
        return e;
      }
      p.tmin = tc_max;
      --scale;
      stack[scale] = Frame{tc_min, tc_max, child, cc};
      continue;
    }
    p.tmin = tc_max;
  }
  return e;
}

struct FrameParams {
  uint32_t width, height;
  float t_scale_ratio;
  int32_t mode;
  float pfh[4], pfv[4], fll[4], cam[4];
};
static_assert(sizeof(FrameParams) == 80, "frame params layout");

// renderToBuffer ray generation (opencl/treeletRenderer_rgba.cl:627-633;
// the CPU twin is raycast_serialized_cpu.cpp:467-471).
inline void pixel_ray(const FrameParams& fp, uint32_t x, uint32_t y, V3& o, V3& d) {
  const float fx = (float)x;
  const float fy = (float)((uint32_t)(int32_t)fp.height - y);
  const float qx = (fp.fll[0] + fp.pfh[0] * fx) + fp.pfv[0] * fy;
  const float qy = (fp.fll[1] + fp.pfh[1] * fx) + fp.pfv[1] * fy;
  const float qz = (fp.fll[2] + fp.pfh[2] * fx) + fp.pfv[2] * fy;
  const float dx = qx - fp.cam[0], dy = qy - fp.cam[1], dz = qz - fp.cam[2];
  const float len = std::sqrt((dx * dx + dy * dy) + dz * dz);
  d = V3{dx / len, dy / len, dz / len};
  o = V3{fp.cam[0], fp.cam[1], fp.cam[2]};
}

// float -> unsigned 8-bit normalised: round(clamp(c, 0, 1) * 255), NaN -> 0.
inline uint32_t to_unorm8(float c) {
  c = c > 0.0f ? (c < 1.0f ? c : 1.0f) : 0.0f;
  return (uint32_t)(c * 255.0f + 0.5f);
}
inline uint32_t pack_rgba8(float r, float g, float b, float a) {
  return to_unorm8(r) | (to_unorm8(g) << 8) | (to_unorm8(b) << 16) | (to_unorm8(a) << 24);
}

// unpackRgbaFromUnsigned (opencl/treeletRenderer_rgba.cl:183-195): r is the
// most significant byte.
inline void unpack_rgba(uint32_t v, float out[4]) {
  out[3] = (float)(v & 255u);
  out[2] = (float)((v >> 8) & 255u);
  out[1] = (float)((v >> 16) & 255u);
  out[0] = (float)((v >> 24) & 255u);
}

inline float dot3(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline V3 normalize3(V3 v) {
  const float l = std::sqrt(dot3(v, v));
  return V3{v.x / l, v.y / l, v.z / l};
}

// getNormal (opencl/treeletRenderer_rgba.cl:388-393).
inline V3 get_normal(uint32_t packed) {
  const float k = 0.003921569f;
  float c[4];
  unpack_rgba(packed, c);
  return V3{(c[0] * k - 0.5f) * 2.0f, (c[1] * k - 0.5f) * 2.0f, (c[2] * k - 0.5f) * 2.0f};
}

// smoothstep(0, 1, x): t = clamp((x - 0) / (1 - 0), 0, 1), t * t * (3 - 2t).
inline float smoothstep01(float x) {
  const float t = x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x);
  return t * t * (3.0f - 2.0f * t);
}

// Adjust (opencl/treeletRenderer_rgba.cl:518-528): Gamma is the double
// literal 0.80, so the power and the scaling by 255 run in double.
inline float wl_adjust(float color, float factor) {
  if (color == 0.0f) return 0.0f;
  const int res = (int)std::round(255.0 * std::pow((double)(color * factor), 0.80));
  return (float)std::min(255, std::max(0, res));
}

// DataPointToColor(value, 0, vmax) (opencl/treeletRenderer_rgba.cl:532-603).
void wavelength_color(float value, float vmax, float rgb[3]) {
  const float w = (value - 0.0f) / (vmax - 0.0f) * (780.0f - 380.0f) + 380.0f;
  float r, g, b, f;
  if (380.0f <= w && w <= 440.0f) {
    r = -(w - 440.0f) / (440.0f - 380.0f);
    g = 0.0f;
    b = 1.0f;
  } else if (440.0f < w && w <= 490.0f) {
    r = 0.0f;
    g = (w - 440.0f) / (490.0f - 440.0f);
    b = 1.0f;
  } else if (490.0f < w && w <= 510.0f) {
    r = 0.0f;
    g = 1.0f;
    b = -(w - 510.0f) / (510.0f - 490.0f);
  } else if (510.0f < w && w <= 580.0f) {
    r = (w - 510.0f) / (580.0f - 510.0f);
    g = 1.0f;
    b = 0.0f;
  } else if (580.0f < w && w <= 645.0f) {
    r = 1.0f;
    g = -(w - 645.0f) / (645.0f - 580.0f);
    b = 0.0f;
  } else if (645.0f < w && w <= 780.0f) {
    r = 1.0f;
    g = 0.0f;
    b = 0.0f;
  } else {
    r = g = b = 0.0f;
  }
  if (380.0f <= w && w <= 420.0f)
    f = 0.3f + 0.7f * (w - 380.0f) / (420.0f - 380.0f);
  else if (420.0f < w && w <= 701.0f)
    f = 1.0f;
  else if (701.0f < w && w <= 780.0f)
    f = 0.3f + 0.7f * (780.0f - w) / (780.0f - 701.0f);
  else
    f = 0.0f;
  const float fac = 1.0f / 255.0f;
  rgb[0] = wl_adjust(r, f) * fac;
  rgb[1] = wl_adjust(g, f) * fac;
  rgb[2] = wl_adjust(b, f) * fac;
}

// shade_phong (opencl/treeletRenderer_rgba.cl:451-504; its shadow ray is
// compiled out, so shadow = 1 - 0).  d is the unclamped primary direction.
void shade_phong(const Hit& h, const Exit& ex, V3 d, const uint32_t* attribs, uint64_t num_nodes,
                 float rgba[4]) {
  if (!h.hit) {
    rgba[0] = 0.4f;
    rgba[1] = 0.6f;
    rgba[2] = 0.4f;
    rgba[3] = 1.0f;
    return;
  }
  if (h.node >= num_nodes) {  // outside the pool: the reference reads out of bounds
    rgba[0] = rgba[1] = rgba[2] = 0.0f;
    rgba[3] = 1.0f;
    return;
  }
  const float k = 0.003921569f;
  const V3 n = normalize3(get_normal(attribs[2 * (uint64_t)h.node]));
  float c[4];
  unpack_rgba(attribs[2 * (uint64_t)h.node + 1], c);
  for (float& v : c) v = v * k;
  const V3 l = normalize3(V3{-120.0f - ex.center.x, 0.0f - ex.center.y, 0.0f - ex.center.z});
  const float ndl = cl_max(0.0f, dot3(n, l));
  const V3 rf = normalize3(V3{((2.0f * n.x) * ndl) - l.x, ((2.0f * n.y) * ndl) - l.y,
                              ((2.0f * n.z) * ndl) - l.z});
  const float rdv = cl_max(0.0f, dot3(rf, V3{-d.x, -d.y, -d.z}));
  const float spec = cl_max(0.0f, std::pow(rdv, 10.0f)) * (float)(ndl > 0.0f);
  const float shadow = 1.0f - 0.0f;
  for (int i = 0; i < 3; ++i)
    rgba[i] = smoothstep01(c[i] * 0.5f + ((c[i] * ndl) * shadow + (spec * shadow) * 0.2f) * 0.5f);
  rgba[3] = 1.0f;
}

// Fragment colour for view mode `mode` (renderToBuffer's switch,
// opencl/treeletRenderer_rgba.cl:644-734): 0 colour, 1 normal, 2 iteration
// count as a wavelength colour, 3 octree depth, 4 pixel depth, 5 iteration
// count, 6 Phong, 7 LOD quality.  `ex` and `d` are used by modes 6 and 7.
void shade(int mode, const Hit& h, const uint32_t* attribs, uint64_t num_nodes, int S,
           float rgba[4], const Exit& ex = Exit{}, V3 d = V3{0.0f, 0.0f, 0.0f}) {
  const float k = 0.003921569f;
  switch (mode) {
    case 2:
      wavelength_color((float)h.loops, (float)(S * 30), rgba);
      rgba[3] = 1.0f;
      return;
    case 6:
      shade_phong(h, ex, d, attribs, num_nodes, rgba);
      return;
    case 7:
      if (h.hit) {
        const float q = std::sqrt(std::sqrt(ex.quality));
        rgba[0] = rgba[1] = rgba[2] = q;
      } else {
        rgba[0] = 0.6f;
        rgba[1] = 0.3f;
        rgba[2] = 0.3f;
      }
      rgba[3] = 1.0f;
      return;
    case 0:
    case 1:
      if (h.hit && h.node < num_nodes) {
        float c[4];
        unpack_rgba(attribs[2 * (uint64_t)h.node + (mode == 0 ? 1 : 0)], c);
        if (mode == 0) {
          rgba[0] = c[0] * k;
          rgba[1] = c[1] * k;
          rgba[2] = c[2] * k;
        } else {
          rgba[0] = (c[0] * k - 0.5f) * 2.0f;
          rgba[1] = (c[1] * k - 0.5f) * 2.0f;
          rgba[2] = (c[2] * k - 0.5f) * 2.0f;
        }
        rgba[3] = 1.0f;
      } else {
        rgba[0] = 0.2f;
        rgba[1] = 0.3f;
        rgba[2] = 0.2f;
        rgba[3] = 1.0f;
      }
      return;
    case 3: {
      const float v = (float)h.depth / (float)S;
      rgba[0] = rgba[1] = rgba[2] = v * (float)h.hit;
      rgba[3] = 1.0f;
      return;
    }
    case 4: {
      const float v = 1.0f - h.t * 0.1f;
      rgba[0] = rgba[1] = rgba[2] = v;
      rgba[3] = 1.0f;
      return;
    }
    case 5: {
      const float v = 1.0f - (float)h.loops / 200.0f;
      rgba[0] = rgba[1] = rgba[2] = v;
      rgba[3] = 1.0f;
      return;
    }
    default:
      rgba[0] = rgba[1] = rgba[2] = 0.0f;
      rgba[3] = 1.0f;
      return;
  }
}

inline Hit cast_any(int flat, const uint32_t* nodes, uint64_t n, V3 o, V3 d, float tsr, int S,
                    RayCount& rc, Exit* ex = nullptr) {
  return flat ? cast_flat(nodes, n, o, d, tsr, S, rc)
              : cast_treelet(nodes, n, o, d, tsr, S, rc, ex);
}

template <class Fn>
void parallel_lines(uint32_t height, uint32_t lines_per_job, int threads, Fn&& fn) {
  if (threads <= 1) {
    for (uint32_t y = 0; y < height; ++y) fn(y);
    return;
  }
  std::atomic<uint32_t> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&] {
      for (;;) {
        const uint32_t y0 = next.fetch_add(lines_per_job);
        if (y0 >= height) return;
        const uint32_t y1 = std::min(height, y0 + lines_per_job);
        for (uint32_t y = y0; y < y1; ++y) fn(y);
      }
    });
  for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {

// Casts one frame.  nodes/attribs: `num_nodes` 8-byte records (uint32 pairs).
// flat = 0: sample() over a treelet incore pool, `S` = MAX_STACK_SIZE.
// flat = 1: CpuRaycasterSingleRay3 over a flat pool, `S` = octree max depth.
// Outputs (each optional): rgba8 (W*H uint32, byte 0 = red), rgbaf (W*H*4
// floats, the renderToBuffer fragment colour), hits (W*H 16-byte records).
// Returns the total number of node fetches (see RayCount).
uint64_t oracle_render(const uint32_t* nodes, const uint32_t* attribs, uint64_t num_nodes,
                       const void* params, int flat, int S, uint32_t* rgba8, float* rgbaf,
                       void* hits, int threads) {
  const FrameParams& fp = *(const FrameParams*)params;
  std::atomic<uint64_t> total{0};
  Hit* hrec = (Hit*)hits;
  parallel_lines(fp.height, 4, threads, [&](uint32_t y) {
    RayCount rc;
    for (uint32_t x = 0; x < fp.width; ++x) {
      V3 o, d;
      pixel_ray(fp, x, y, o, d);
      Exit ex;
      const Hit h = cast_any(flat, nodes, num_nodes, o, d, fp.t_scale_ratio, S, rc, &ex);
      rc.fetches += h.fetches;
      const uint64_t pix = (uint64_t)y * fp.width + x;
      if (hrec) hrec[pix] = h;
      if (rgba8 || rgbaf) {
        float c[4];
        shade(fp.mode, h, attribs, num_nodes, S, c, ex, d);
        if (rgba8) rgba8[pix] = pack_rgba8(c[0], c[1], c[2], c[3]);
        if (rgbaf) std::memcpy(rgbaf + 4 * pix, c, sizeof(c));
      }
    }
    total.fetch_add(rc.fetches, std::memory_order_relaxed);
  });
  return total.load();
}

// Primary ray plus one shadow ray per hit (treelet traversal), shaded as
// shade_diffuse_color_shadow (opencl/fillFrameBuffer_rgba.cl:494-529) with the
// live renderer's attribute index (= node index):
//   n = getNormal, c = getColor, nDotL = max(0, dot(n, L)),
//   shadow = sample(nodeCenter + n * offset, L, shadow_tsr) ? 1 : 0,
//   colour = c * nDotL * (1 - shadow) + c * 0.2, alpha 1; misses and hits
//   outside the pool (0.2, 0.3, 0.2).
// light: the unit direction toward the light, used as given.  Outputs as in
// oracle_render, plus shadow_hits (zeros where no shadow ray was cast).
// Returns the node fetches of both ray kinds.
// Rows [y0, y1) of the frame only: the outputs hold (y1 - y0) * W entries,
// row y at (y - y0) * W.
uint64_t oracle_render_shadow_rows(const uint32_t* nodes, const uint32_t* attribs,
                                   uint64_t num_nodes, const void* params, int S,
                                   const float* light, float shadow_tsr, float offset, uint32_t y0,
                                   uint32_t y1, uint32_t* rgba8, float* rgbaf, void* hits,
                                   void* shadow_hits, int threads) {
  const FrameParams& fp = *(const FrameParams*)params;
  std::atomic<uint64_t> total{0};
  Hit* hrec = (Hit*)hits;
  Hit* srec = (Hit*)shadow_hits;
  const V3 l{light[0], light[1], light[2]};
  if (y1 > fp.height) y1 = fp.height;
  if (y0 >= y1) return 0;
  parallel_lines(y1 - y0, 4, threads, [&](uint32_t yr) {
    const uint32_t y = y0 + yr;
    RayCount rc;
    for (uint32_t x = 0; x < fp.width; ++x) {
      V3 o, d;
      pixel_ray(fp, x, y, o, d);
      Exit ex;
      const Hit h = cast_treelet(nodes, num_nodes, o, d, fp.t_scale_ratio, S, rc, &ex);
      rc.fetches += h.fetches;
      Hit sh{};
      float c[4] = {0.2f, 0.3f, 0.2f, 1.0f};
      if (h.hit && h.node < num_nodes) {
        const V3 n = get_normal(attribs[2 * (uint64_t)h.node]);
        float col[4];
        unpack_rgba(attribs[2 * (uint64_t)h.node + 1], col);
        const float k = 0.003921569f;
        for (float& v : col) v = v * k;
        const float ndl = cl_max(0.0f, dot3(n, l));
        const V3 so{ex.center.x + n.x * offset, ex.center.y + n.y * offset,
                    ex.center.z + n.z * offset};
        sh = cast_treelet(nodes, num_nodes, so, l, shadow_tsr, S, rc);
        rc.fetches += sh.fetches;
        const float shadow = sh.hit ? 1.0f : 0.0f;
        for (int i = 0; i < 3; ++i) c[i] = col[i] * ndl * (1.0f - shadow) + col[i] * 0.2f;
        c[3] = 1.0f;
      }
      const uint64_t pix = (uint64_t)yr * fp.width + x;
      if (hrec) hrec[pix] = h;
      if (srec) srec[pix] = sh;
      if (rgba8) rgba8[pix] = pack_rgba8(c[0], c[1], c[2], c[3]);
      if (rgbaf) std::memcpy(rgbaf + 4 * pix, c, sizeof(c));
    }
    total.fetch_add(rc.fetches, std::memory_order_relaxed);
  });
  return total.load();
}

uint64_t oracle_render_shadow(const uint32_t* nodes, const uint32_t* attribs, uint64_t num_nodes,
                              const void* params, int S, const float* light, float shadow_tsr,
                              float offset, uint32_t* rgba8, float* rgbaf,
                              void* hits, void* shadow_hits, int threads) {
  const FrameParams& fp = *(const FrameParams*)params;
  return oracle_render_shadow_rows(nodes, attribs, num_nodes, params, S, light, shadow_tsr, offset,
                                   0, fp.height, rgba8, rgbaf, hits, shadow_hits, threads);
}

// Casts an explicit list of rays (origins and directions, 3 floats each).
uint64_t oracle_cast_rays(const uint32_t* nodes, uint64_t num_nodes, const float* origins,
                          const float* dirs, uint64_t n, float tsr, int flat, int S, void* hits,
                          int threads) {
  Hit* hrec = (Hit*)hits;
  std::atomic<uint64_t> total{0};
  const uint32_t lines = (uint32_t)((n + 1023) / 1024);
  parallel_lines(lines, 1, threads, [&](uint32_t line) {
    RayCount rc;
    const uint64_t i0 = (uint64_t)line * 1024, i1 = std::min<uint64_t>(n, i0 + 1024);
    for (uint64_t i = i0; i < i1; ++i) {
      const V3 o{origins[3 * i], origins[3 * i + 1], origins[3 * i + 2]};
      const V3 d{dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]};
      hrec[i] = cast_any(flat, nodes, num_nodes, o, d, tsr, S, rc);
      rc.fetches += hrec[i].fetches;
    }
    total.fetch_add(rc.fetches, std::memory_order_relaxed);
  });
  return total.load();
}

// Generates the primary rays of a frame (renderToBuffer ray generation) so that
// tests can feed identical rays to other implementations.
void oracle_pixel_rays(const void* params, float* origins, float* dirs) {
  const FrameParams& fp = *(const FrameParams*)params;
  for (uint32_t y = 0; y < fp.height; ++y)
    for (uint32_t x = 0; x < fp.width; ++x) {
      V3 o, d;
      pixel_ray(fp, x, y, o, d);
      const uint64_t i = (uint64_t)y * fp.width + x;
      origins[3 * i] = o.x;
      origins[3 * i + 1] = o.y;
      origins[3 * i + 2] = o.z;
      dirs[3 * i] = d.x;
      dirs[3 * i + 1] = d.y;
      dirs[3 * i + 2] = d.z;
    }
}

// renderToFeedbackBuffer (opencl/treeletRenderer_rgba.cl:960-1011) over a
// whole analysis buffer: one 16-byte record per pixel and (optional) the
// debug colour per pixel as floats.
void oracle_feedback(const uint32_t* nodes, uint64_t num_nodes, const void* params, int S,
                     void* records, float* rgbaf, int threads) {
  const FrameParams& fp = *(const FrameParams*)params;
  Feedback* out = (Feedback*)records;
  parallel_lines(fp.height, 4, threads, [&](uint32_t y) {
    for (uint32_t x = 0; x < fp.width; ++x) {
      V3 o, d;
      pixel_ray(fp, x, y, o, d);
      const Feedback e = analyse_ray(nodes, num_nodes, o, d, fp.t_scale_ratio, S);
      const uint64_t pix = (uint64_t)y * fp.width + x;
      out[pix] = e;
      if (rgbaf) {
        float* c = rgbaf + 4 * pix;
        if (e.node_id != 0) {
          c[0] = (float)e.sub_treelet_gid;
          c[1] = 0.0f;
          c[2] = e.error;
        } else {
          c[0] = 0.2f;
          c[1] = 0.3f;
          c[2] = 0.2f;
        }
        c[3] = 1.0f;
      }
    }
  });
}

int oracle_hit_record_size(void) { return (int)sizeof(Hit); }

}  // extern "C"
