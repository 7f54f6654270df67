// scene.cpp -- octree construction, treelet cut, files and flattening.
//
// The octree is built level by level from its leaves: a node exists when one
// of its eight children does, children are serialised in child-index order
// (4x + 2y + z, the order sample() decodes), and inner attributes are the
// averages of the children's (src/attribute_generators/
// Ag_colorAndNormalsTriangles.cpp:250-300).  The treelet cut then follows
// the reference's builder: breadth-first fill of a fixed-size treelet
// (src/TreeletBuilderFromFaces.cpp:189-365), leaves left in the queue become
// the roots of sub-treelets whose gid is written into the leaf
// (src/TreeletBuildManager.cpp:211-233), treelets processed first in, first
// out.  One addition: treelet boundaries at fixed levels (every
// `treelet_levels` levels, counted up from the leaves), so a scene can be cut
// into treelets of a given number of levels; the slot size then defaults to
// the largest such treelet.
#include "scene.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <thread>

namespace svo {

uint64_t Octree::total_nodes() const {
  uint64_t n = 0;
  for (const auto& c : codes) n += c.size();
  return n;
}

namespace {

uint64_t split3(uint32_t a) {
  uint64_t x = a & 0x1fffffu;
  x = (x | x << 32) & 0x1f00000000ffffull;
  x = (x | x << 16) & 0x1f0000ff0000ffull;
  x = (x | x << 8) & 0x100f00f00f00f00full;
  x = (x | x << 4) & 0x10c30c30c30c30c3ull;
  x = (x | x << 2) & 0x1249249249249249ull;
  return x;
}

uint32_t unorm8(float c) {
  if (!(c > 0.0f)) return 0u;  // also maps NaN to 0
  if (c >= 1.0f) return 255u;
  return (uint32_t)(c * 255.0f + 0.5f);
}

uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

int resolve_threads(int threads) {
  if (threads > 0) return threads;
  const unsigned hc = std::thread::hardware_concurrency();
  return hc ? (int)hc : 1;
}

template <class Fn>
void parallel_for(uint64_t n, int threads, Fn&& fn) {
  threads = resolve_threads(threads);
  if (threads <= 1 || n < 2) {
    for (uint64_t i = 0; i < n; ++i) fn(i, 0);
    return;
  }
  std::atomic<uint64_t> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&, t] {
      for (;;) {
        const uint64_t i = next.fetch_add(1);
        if (i >= n) return;
        fn(i, t);
      }
    });
  for (auto& th : pool) th.join();
}

}  // namespace

namespace {
uint32_t compact3(uint64_t x) {
  x &= 0x1249249249249249ull;
  x = (x ^ (x >> 2)) & 0x10c30c30c30c30c3ull;
  x = (x ^ (x >> 4)) & 0x100f00f00f00f00full;
  x = (x ^ (x >> 8)) & 0x1f0000ff0000ffull;
  x = (x ^ (x >> 16)) & 0x1f00000000ffffull;
  x = (x ^ (x >> 32)) & 0x1fffffull;
  return (uint32_t)x;
}
}  // namespace

void morton3_decode(uint64_t code, uint32_t& x, uint32_t& y, uint32_t& z) {
  x = compact3(code >> 2);
  y = compact3(code >> 1);
  z = compact3(code);
}

uint64_t morton3(uint32_t x, uint32_t y, uint32_t z, uint32_t depth) {
  (void)depth;
  return (split3(x) << 2) | (split3(y) << 1) | split3(z);
}

uint32_t pack_color(float r, float g, float b) {
  return (unorm8(r) << 24) | (unorm8(g) << 16) | (unorm8(b) << 8) | 255u;
}
uint32_t pack_normal(float x, float y, float z) {
  return pack_color(x * 0.5f + 0.5f, y * 0.5f + 0.5f, z * 0.5f + 0.5f);
}
void unpack_color(uint32_t v, float rgb[3]) {
  rgb[0] = (float)(v >> 24) / 255.0f;
  rgb[1] = (float)((v >> 16) & 255u) / 255.0f;
  rgb[2] = (float)((v >> 8) & 255u) / 255.0f;
}
void unpack_normal(uint32_t v, float n[3]) {
  unpack_color(v, n);
  for (int i = 0; i < 3; ++i) n[i] = (n[i] - 0.5f) * 2.0f;
}

// ---------------------------------------------------------------------------
// leaves -> level arrays

int octree_from_leaves(uint32_t depth, std::vector<uint64_t>&& codes,
                       std::vector<svo_attrib>&& leaf_attribs, Octree& out) {
  if (depth < 1 || depth > 21) return SVO_ERR_RANGE;
  if (codes.empty() || codes.size() != leaf_attribs.size()) return SVO_ERR_INVALID;
  out = Octree();
  out.depth = depth;
  out.codes.resize(depth + 1);
  out.masks.resize(depth + 1);
  out.first.resize(depth + 1);
  out.attribs.resize(depth + 1);
  out.codes[depth] = std::move(codes);
  out.attribs[depth] = std::move(leaf_attribs);
  for (int d = (int)depth - 1; d >= 0; --d) {
    const auto& cc = out.codes[d + 1];
    const auto& ca = out.attribs[d + 1];
    auto& pc = out.codes[d];
    auto& pm = out.masks[d];
    auto& pf = out.first[d];
    auto& pa = out.attribs[d];
    uint64_t i = 0;
    const uint64_t n = cc.size();
    while (i < n) {
      const uint64_t parent = cc[i] >> 3;
      uint64_t j = i;
      uint8_t mask = 0;
      float nsum[3] = {0.0f, 0.0f, 0.0f}, csum[3] = {0.0f, 0.0f, 0.0f};
      while (j < n && (cc[j] >> 3) == parent) {
        mask |= (uint8_t)(1u << (cc[j] & 7u));
        float v[3];
        unpack_normal(ca[j].packed_normal, v);
        for (int k = 0; k < 3; ++k) nsum[k] += v[k];
        unpack_color(ca[j].packed_color, v);
        for (int k = 0; k < 3; ++k) csum[k] += v[k];
        ++j;
      }
      const float cnt = (float)(j - i);
      for (int k = 0; k < 3; ++k) {
        nsum[k] /= cnt;
        csum[k] /= cnt;
      }
      const float len = std::sqrt(nsum[0] * nsum[0] + nsum[1] * nsum[1] + nsum[2] * nsum[2]);
      if (len > 0.0f)
        for (int k = 0; k < 3; ++k) nsum[k] /= len;
      else
        nsum[0] = 0.0f, nsum[1] = 0.0f, nsum[2] = 1.0f;
      pc.push_back(parent);
      pm.push_back(mask);
      pf.push_back(i);
      pa.push_back(svo_attrib{pack_normal(nsum[0], nsum[1], nsum[2]),
                              pack_color(csum[0], csum[1], csum[2])});
      i = j;
    }
  }
  if (out.codes[0].size() != 1) return SVO_ERR_INVALID;
  return SVO_OK;
}

// ---------------------------------------------------------------------------
// treelet cut

namespace {

// Nodes within `levels` levels below node (level, index), root included.
uint64_t bounded_count(const Octree& t, uint32_t level, uint64_t index, uint32_t levels) {
  uint64_t lo = index, hi = index + 1, total = 1;
  const uint32_t last = std::min(t.depth, level + levels);
  for (uint32_t l = level; l < last; ++l) {
    const uint64_t nlo = t.first[l][lo];
    const uint64_t nhi = t.first[l][hi - 1] + (uint64_t)__builtin_popcount(t.masks[l][hi - 1]);
    lo = nlo;
    hi = nhi;
    total += hi - lo;
  }
  return total;
}

// Treelet boundaries sit at the levels D, D-L, D-2L, ...: a treelet rooted
// at level r expands down to the next boundary below it, so every treelet
// but the top one spans exactly L levels and ends on the octree's leaves.
//
// A treelet other than the top one never spans a single level above the
// leaves.  Its sub-treelet leaves would then hang off its root node, and the
// manager clears their leaf flag in the treelet's own slot
// (TreeletMemoryManager.cpp:535) while the traversal reads the copy of that
// root made earlier in the parent's leaf (:532): the sub-treelets would be
// resident but never reached.
uint32_t stop_level(uint32_t D, uint32_t L, uint32_t r) {
  if (L == 0) return D;
  const uint32_t m = (D - r) % L;
  uint32_t stop = r + (m == 0 ? L : m);
  if (stop == r + 1 && stop < D && r > 0) stop = std::min(D, stop + L);
  return stop;
}

struct TreeletRoot {
  uint32_t level;
  uint64_t index;
  uint32_t gid;
  int32_t parent_gid, leaf_pos, leaf_idx, leaf_parent_pos;
};

struct FillItem {
  uint32_t level;
  uint64_t index;
  uint32_t local;
  uint32_t parent_local;
  uint32_t idx;
};

}  // namespace

int cut_treelets(const Octree& tree, uint32_t treelet_levels, uint32_t treelet_bytes,
                 svo_scene& out) {
  const uint32_t D = tree.depth;
  uint64_t N;
  if (treelet_bytes == 0) {
    uint64_t need = 0;
    if (treelet_levels == 0) {
      need = tree.total_nodes();
    } else {
      for (uint32_t r = 0; r < D; r = stop_level(D, treelet_levels, r))
        for (uint64_t i = 0; i < tree.codes[r].size(); ++i)
          need = std::max(need, bounded_count(tree, r, i, stop_level(D, treelet_levels, r) - r));
    }
    N = need + 8;
  } else {
    if (treelet_bytes % 8 != 0) return SVO_ERR_INVALID;
    N = treelet_bytes / 8;
  }
  if (N < 16) return SVO_ERR_RANGE;
  if (N * 8 > 0xFFFFFFFFull) return SVO_ERR_RANGE;

  out = svo_scene();
  out.treelet_bytes = (uint32_t)(N * 8);
  out.max_depth = D;
  out.leaf_voxels = tree.codes[D].size();

  std::deque<TreeletRoot> roots;
  roots.push_back(TreeletRoot{0, 0, 0, 0, 0, 0, 0});
  uint64_t next_gid = 1;
  std::deque<FillItem> q;
  while (!roots.empty()) {
    const TreeletRoot r = roots.front();
    roots.pop_front();
    TreeletData t;
    t.gid = r.gid;
    t.mem_size = (uint32_t)(N * 8);
    t.parent_gid = r.parent_gid;
    t.parent_leaf_position = r.leaf_pos;
    t.parent_leaf_idx = r.leaf_idx;
    t.parent_leaf_parent_position = r.leaf_parent_pos;
    t.nodes.push_back(svo_node{0u, 0u});
    t.attribs.push_back(tree.attribs[r.level][r.index]);
    const uint32_t stop = stop_level(D, treelet_levels, r.level);
    q.clear();
    q.push_back(FillItem{r.level, r.index, 0u, 0u, 0u});
    uint64_t current = 1;
    while (!q.empty() && current < N - 8 && q.front().level < stop) {
      const FillItem f = q.front();
      const uint8_t m = tree.masks[f.level][f.index];
      const uint64_t fc = tree.first[f.level][f.index];
      uint32_t rank = 0;
      for (uint32_t c = 0; c < 8; ++c) {
        if (!((m >> c) & 1u)) continue;
        svo_node& parent = t.nodes[f.local];
        if (rank == 0) parent.first_child = (uint32_t)((int64_t)current - (int64_t)f.local);
        parent.masks |= 1u << (c + 8u);
        const uint64_t child_index = fc + rank;
        ++rank;
        t.nodes.push_back(svo_node{0u, 0u});
        t.attribs.push_back(tree.attribs[f.level + 1][child_index]);
        q.push_back(FillItem{f.level + 1, child_index, (uint32_t)current, f.local, c});
        ++current;
      }
      q.pop_front();
    }
    t.num_nodes = (uint32_t)current;
    t.num_leaves = (uint32_t)q.size();
    for (const FillItem& f : q) {
      if (f.local == 0) return SVO_ERR_RANGE;  // treelet too small to expand its root
      // see stop_level(): sub-treelets must not hang off a non-top root
      if (t.gid != 0 && f.parent_local == 0 && f.level < D) return SVO_ERR_RANGE;
      t.nodes[f.parent_local].masks |= 1u << f.idx;
      if (f.level < D) {
        if (next_gid > 0x7FFFFFFFull) return SVO_ERR_RANGE;
        const uint32_t gid = (uint32_t)next_gid++;
        t.nodes[f.local].first_child = gid;
        roots.push_back(TreeletRoot{f.level, f.index, gid, (int32_t)t.gid, (int32_t)f.local,
                                    (int32_t)f.idx, (int32_t)f.parent_local});
      }
    }
    out.treelets.push_back(std::move(t));
  }
  return SVO_OK;
}

// ---------------------------------------------------------------------------
// Menger sponge

int build_menger(uint32_t level, uint32_t depth, uint64_t seed, std::vector<uint64_t>& codes,
                 std::vector<svo_attrib>& attribs) {
  if (depth < 1 || depth > 21 || level > 13) return SVO_ERR_RANGE;
  uint64_t side = 1;
  for (uint32_t i = 0; i < level; ++i) side *= 3;
  const uint64_t lattice = 1ull << depth;
  if (side > lattice) return SVO_ERR_RANGE;
  const uint32_t off = (uint32_t)((lattice - side) / 2);
  // digit tables: solid iff no base-3 position has two or more 1 digits
  std::vector<uint8_t> ones_mask(side);  // bit k set when digit k of v is 1
  for (uint64_t v = 0; v < side; ++v) {
    uint64_t x = v;
    uint8_t m = 0;
    for (uint32_t k = 0; k < level; ++k, x /= 3)
      if (x % 3 == 1) m |= (uint8_t)(1u << k);
    ones_mask[v] = m;
  }
  codes.clear();
  attribs.clear();
  const uint32_t up = pack_normal(0.0f, 0.0f, 1.0f);
  for (uint64_t x = 0; x < side; ++x)
    for (uint64_t y = 0; y < side; ++y) {
      const uint8_t mxy = ones_mask[x] & ones_mask[y];
      for (uint64_t z = 0; z < side; ++z) {
        const uint8_t mx = ones_mask[x], my = ones_mask[y], mz = ones_mask[z];
        if ((mxy | (mx & mz) | (my & mz)) != 0) continue;
        const uint32_t X = off + (uint32_t)x, Y = off + (uint32_t)y, Z = off + (uint32_t)z;
        codes.push_back(morton3(X, Y, Z, depth));
        const uint64_t h = splitmix64((uint64_t)X | ((uint64_t)Y << 21) | ((uint64_t)Z << 42) ^
                                      (seed * 0x9E3779B97F4A7C15ull));
        attribs.push_back(svo_attrib{up, (uint32_t)(h & 0xFFFFFF00ull) | 255u});
      }
    }
  // sort by code, attributes alongside
  std::vector<uint64_t> order(codes.size());
  for (uint64_t i = 0; i < order.size(); ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) { return codes[a] < codes[b]; });
  std::vector<uint64_t> c2(codes.size());
  std::vector<svo_attrib> a2(codes.size());
  for (uint64_t i = 0; i < order.size(); ++i) {
    c2[i] = codes[order[i]];
    a2[i] = attribs[order[i]];
  }
  codes.swap(c2);
  attribs.swap(a2);
  return SVO_OK;
}

// ---------------------------------------------------------------------------
// triangle mesh voxeliser

namespace {

// Triangle / axis-aligned box overlap by the separating axis theorem
// (Akenine-Moeller, "Fast 3D Triangle-Box Overlap Testing", 2001): the three
// box normals, the triangle normal and the nine edge/axis cross products.
bool tri_box_overlap(const float bc[3], float h, const float* a, const float* b, const float* c) {
  float v0[3], v1[3], v2[3];
  for (int i = 0; i < 3; ++i) {
    v0[i] = a[i] - bc[i];
    v1[i] = b[i] - bc[i];
    v2[i] = c[i] - bc[i];
  }
  const float e[3][3] = {{v1[0] - v0[0], v1[1] - v0[1], v1[2] - v0[2]},
                         {v2[0] - v1[0], v2[1] - v1[1], v2[2] - v1[2]},
                         {v0[0] - v2[0], v0[1] - v2[1], v0[2] - v2[2]}};
  auto separated = [&](float ax, float ay, float az) {
    const float p0 = ax * v0[0] + ay * v0[1] + az * v0[2];
    const float p1 = ax * v1[0] + ay * v1[1] + az * v1[2];
    const float p2 = ax * v2[0] + ay * v2[1] + az * v2[2];
    const float mn = std::min(p0, std::min(p1, p2)), mx = std::max(p0, std::max(p1, p2));
    const float r = h * (std::fabs(ax) + std::fabs(ay) + std::fabs(az));
    return mn > r || mx < -r;
  };
  for (int k = 0; k < 3; ++k) {
    const float* ek = e[k];
    if (separated(0.0f, ek[2], -ek[1])) return false;
    if (separated(-ek[2], 0.0f, ek[0])) return false;
    if (separated(ek[1], -ek[0], 0.0f)) return false;
  }
  for (int i = 0; i < 3; ++i) {
    const float mn = std::min(v0[i], std::min(v1[i], v2[i]));
    const float mx = std::max(v0[i], std::max(v1[i], v2[i]));
    if (mn > h || mx < -h) return false;
  }
  const float n[3] = {e[0][1] * e[1][2] - e[0][2] * e[1][1], e[0][2] * e[1][0] - e[0][0] * e[1][2],
                      e[0][0] * e[1][1] - e[0][1] * e[1][0]};
  const float d = -(n[0] * v0[0] + n[1] * v0[1] + n[2] * v0[2]);
  float vmin[3], vmax[3];
  for (int i = 0; i < 3; ++i) {
    if (n[i] > 0.0f) {
      vmin[i] = -h;
      vmax[i] = h;
    } else {
      vmin[i] = h;
      vmax[i] = -h;
    }
  }
  if (n[0] * vmin[0] + n[1] * vmin[1] + n[2] * vmin[2] + d > 0.0f) return false;
  return n[0] * vmax[0] + n[1] * vmax[1] + n[2] * vmax[2] + d >= 0.0f;
}

// floor(x) as a lattice coordinate, clamped to [-2, R + 1] (NaN -> -2) so
// that degenerate triangles cannot overflow the int conversion; every caller
// clamps the result into [0, R - 1] afterwards, so the clamp changes nothing
// for coordinates inside the cube.  The GPU builder uses the same rule.
int cell_floor(float x, uint32_t R) {
  const float hi = (float)R + 1.0f;
  if (!(x >= -2.0f)) return -2;
  if (x > hi) return (int)R + 1;
  return (int)std::floor(x);
}

// One triangle's contribution to a leaf (src/attribute_generators/
// Ag_colorAndNormalsTriangles.cpp:110-135 with BuilderTriangleFace.cpp:211-329):
// the barycentric (u, v) where the ray from the voxel centre along the
// triangle's mean vertex normal meets the triangle's plane (Moeller-Trumbore,
// det within +-1e-8 = parallel: the reference leaves u, v unset there, this
// takes u = v = 0), clamped to [0, 1]; the normalised interpolated vertex
// normal and the interpolated vertex colour, w = (1 - u) - v.  FP32, in this
// order; the GPU builder repeats it operation for operation.
void leaf_contribution(const float* V, const float* N, const float* C, const uint32_t* tri,
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
  for (int k = 0; k < 3; ++k) d[k] = ((n0[k] + n1[k]) + n2[k]) / 3.0f;
  float len = std::sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]);
  if (len > 0.0f)
    for (int k = 0; k < 3; ++k) d[k] = d[k] / len;
  const float e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
  const float e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
  const float pv[3] = {d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2],
                       d[0] * e2[1] - d[1] * e2[0]};
  const float det = (e1[0] * pv[0] + e1[1] * pv[1]) + e1[2] * pv[2];
  float u = 0.0f, v = 0.0f;
  if (!(det > -1e-8f && det < 1e-8f)) {
    const float inv = 1.0f / det;
    const float tv[3] = {c[0] - p0[0], c[1] - p0[1], c[2] - p0[2]};
    u = ((tv[0] * pv[0] + tv[1] * pv[1]) + tv[2] * pv[2]) * inv;
    const float qv[3] = {tv[1] * e1[2] - tv[2] * e1[1], tv[2] * e1[0] - tv[0] * e1[2],
                         tv[0] * e1[1] - tv[1] * e1[0]};
    v = ((d[0] * qv[0] + d[1] * qv[1]) + d[2] * qv[2]) * inv;
  }
  u = u < 0.0f ? 0.0f : (u > 1.0f ? 1.0f : u);
  v = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
  const float w = (1.0f - u) - v;
  for (int k = 0; k < 3; ++k) {
    n_out[k] = (n0[k] * w + n1[k] * u) + n2[k] * v;
    c_out[k] = (c0[k] * w + c1[k] * u) + c2[k] * v;
  }
  len = std::sqrt((n_out[0] * n_out[0] + n_out[1] * n_out[1]) + n_out[2] * n_out[2]);
  if (len > 0.0f)
    for (int k = 0; k < 3; ++k) n_out[k] = n_out[k] / len;
}

struct VoxelTri {
  uint64_t code;
  uint32_t tri;
  uint32_t pad;
};

}  // namespace

int build_mesh_leaves(const float* V, const float* NV, const float* CV, uint64_t nv,
                      const uint32_t* T, uint64_t nt, uint32_t depth, int threads,
                      std::vector<uint64_t>& codes, std::vector<svo_attrib>& attribs) {
  if (depth < 1 || depth > 21) return SVO_ERR_RANGE;
  if (nt == 0 || nv == 0) return SVO_ERR_INVALID;
  if ((NV == nullptr) != (CV == nullptr)) return SVO_ERR_INVALID;
  for (uint64_t i = 0; i < 3 * nt; ++i)
    if (T[i] >= nv) return SVO_ERR_INVALID;
  threads = resolve_threads(threads);
  const uint32_t R = 1u << depth;
  const float inv = 1.0f / (float)R;
  const float h = 0.5f * inv;
  std::vector<std::vector<VoxelTri>> per_thread(threads);
  std::vector<float> fnormal(3 * nt);
  const uint64_t chunk = 4096;
  const uint64_t chunks = (nt + chunk - 1) / chunk;
  parallel_for(chunks, threads, [&](uint64_t ci, int tid) {
    auto& outv = per_thread[tid];
    const uint64_t t0 = ci * chunk, t1 = std::min(nt, t0 + chunk);
    for (uint64_t t = t0; t < t1; ++t) {
      const float* a = V + 3 * (uint64_t)T[3 * t];
      const float* b = V + 3 * (uint64_t)T[3 * t + 1];
      const float* c = V + 3 * (uint64_t)T[3 * t + 2];
      float n[3] = {(b[1] - a[1]) * (c[2] - a[2]) - (b[2] - a[2]) * (c[1] - a[1]),
                    (b[2] - a[2]) * (c[0] - a[0]) - (b[0] - a[0]) * (c[2] - a[2]),
                    (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0])};
      const float len = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
      if (len > 0.0f)
        for (int k = 0; k < 3; ++k) fnormal[3 * t + k] = n[k] / len;
      else
        fnormal[3 * t] = 0.0f, fnormal[3 * t + 1] = 0.0f, fnormal[3 * t + 2] = 1.0f;
      int lo[3], hi[3];
      for (int k = 0; k < 3; ++k) {
        const float mn = std::min(a[k], std::min(b[k], c[k]));
        const float mx = std::max(a[k], std::max(b[k], c[k]));
        lo[k] = std::max(0, cell_floor((mn + 0.5f) * (float)R, R));
        hi[k] = std::min((int)R - 1, cell_floor((mx + 0.5f) * (float)R, R));
        if (lo[k] > hi[k]) lo[k] = hi[k] + 1;
      }
      if (lo[0] > hi[0] || lo[1] > hi[1] || lo[2] > hi[2]) continue;
      // walk columns along the dominant normal axis w; the plane crosses a
      // column within a few voxels, found from the plane at the cell corners
      int w = 0;
      if (std::fabs(n[1]) > std::fabs(n[w])) w = 1;
      if (std::fabs(n[2]) > std::fabs(n[w])) w = 2;
      const int u = (w + 1) % 3, v = (w + 2) % 3;
      const float pd = n[0] * a[0] + n[1] * a[1] + n[2] * a[2];
      for (int iu = lo[u]; iu <= hi[u]; ++iu)
        for (int iv = lo[v]; iv <= hi[v]; ++iv) {
          int wlo = lo[w], whi = hi[w];
          if (n[w] != 0.0f) {
            const float u0 = -0.5f + (float)iu * inv, u1 = u0 + inv;
            const float v0 = -0.5f + (float)iv * inv, v1 = v0 + inv;
            float wmin = 1e30f, wmax = -1e30f;
            const float us[2] = {u0, u1}, vs[2] = {v0, v1};
            for (float uu : us)
              for (float vv : vs) {
                const float ww = (pd - n[u] * uu - n[v] * vv) / n[w];
                wmin = std::min(wmin, ww);
                wmax = std::max(wmax, ww);
              }
            wlo = std::max(wlo, cell_floor((wmin + 0.5f) * (float)R, R) - 1);
            whi = std::min(whi, cell_floor((wmax + 0.5f) * (float)R, R) + 1);
          }
          for (int iw = wlo; iw <= whi; ++iw) {
            int ijk[3];
            ijk[u] = iu;
            ijk[v] = iv;
            ijk[w] = iw;
            const float bc[3] = {-0.5f + ((float)ijk[0] + 0.5f) * inv,
                                 -0.5f + ((float)ijk[1] + 0.5f) * inv,
                                 -0.5f + ((float)ijk[2] + 0.5f) * inv};
            if (tri_box_overlap(bc, h, a, b, c))
              outv.push_back(VoxelTri{morton3((uint32_t)ijk[0], (uint32_t)ijk[1], (uint32_t)ijk[2], depth),
                                      (uint32_t)t, 0u});
          }
        }
    }
  });
  // bucket by the top 3 levels of the code, sort each bucket by (code, tri)
  const uint32_t top_levels = std::min<uint32_t>(3, depth);
  const uint32_t shift = 3 * (depth - top_levels);
  const uint32_t nb = 1u << (3 * top_levels);
  std::vector<uint64_t> bucket_start(nb + 1, 0);
  for (auto& pv : per_thread)
    for (const VoxelTri& e : pv) ++bucket_start[(e.code >> shift) + 1];
  for (uint32_t i = 0; i < nb; ++i) bucket_start[i + 1] += bucket_start[i];
  std::vector<VoxelTri> all(bucket_start[nb]);
  {
    std::vector<uint64_t> pos(bucket_start.begin(), bucket_start.end() - 1);
    for (auto& pv : per_thread) {
      for (const VoxelTri& e : pv) all[pos[e.code >> shift]++] = e;
      std::vector<VoxelTri>().swap(pv);
    }
  }
  parallel_for(nb, threads, [&](uint64_t bi, int) {
    std::sort(all.begin() + bucket_start[bi], all.begin() + bucket_start[bi + 1],
              [](const VoxelTri& x, const VoxelTri& y) {
                return x.code != y.code ? x.code < y.code : x.tri < y.tri;
              });
  });
  codes.clear();
  attribs.clear();
  uint64_t i = 0;
  if (NV) {  // the reference's interpolated attributes, averaged over the triangles
    const float inv_r = 1.0f / (float)R;
    while (i < all.size()) {
      uint64_t j = i;
      uint32_t x, y, z;
      morton3_decode(all[i].code, x, y, z);
      const float c[3] = {-0.5f + ((float)x + 0.5f) * inv_r, -0.5f + ((float)y + 0.5f) * inv_r,
                          -0.5f + ((float)z + 0.5f) * inv_r};
      float sn[3] = {0.0f, 0.0f, 0.0f}, sc[3] = {0.0f, 0.0f, 0.0f};
      while (j < all.size() && all[j].code == all[i].code) {
        float n[3], col[3];
        leaf_contribution(V, NV, CV, T + 3 * (uint64_t)all[j].tri, c, n, col);
        for (int k = 0; k < 3; ++k) {
          sn[k] += n[k];
          sc[k] += col[k];
        }
        ++j;
      }
      const float cnt = (float)(j - i);
      for (int k = 0; k < 3; ++k) {
        sn[k] = sn[k] / cnt;
        sc[k] = sc[k] / cnt;
      }
      const float len = std::sqrt((sn[0] * sn[0] + sn[1] * sn[1]) + sn[2] * sn[2]);
      if (len > 0.0f)
        for (int k = 0; k < 3; ++k) sn[k] = sn[k] / len;
      else
        sn[0] = 0.0f, sn[1] = 0.0f, sn[2] = 1.0f;
      codes.push_back(all[i].code);
      attribs.push_back(svo_attrib{pack_normal(sn[0], sn[1], sn[2]), pack_color(sc[0], sc[1], sc[2])});
      i = j;
    }
    return codes.empty() ? SVO_ERR_INVALID : SVO_OK;
  }
  while (i < all.size()) {
    uint64_t j = i;
    float s[3] = {0.0f, 0.0f, 0.0f};
    while (j < all.size() && all[j].code == all[i].code) {
      for (int k = 0; k < 3; ++k) s[k] += fnormal[3 * (uint64_t)all[j].tri + k];
      ++j;
    }
    const float len = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    if (len > 0.0f)
      for (int k = 0; k < 3; ++k) s[k] /= len;
    else
      s[0] = 0.0f, s[1] = 0.0f, s[2] = 1.0f;
    codes.push_back(all[i].code);
    attribs.push_back(svo_attrib{pack_normal(s[0], s[1], s[2]),
                                 pack_color(s[0] * 0.5f + 0.5f, s[1] * 0.5f + 0.5f, s[2] * 0.5f + 0.5f)});
    i = j;
  }
  if (codes.empty()) return SVO_ERR_INVALID;
  return SVO_OK;
}

// ---------------------------------------------------------------------------
// files

namespace {

bool put_u32(FILE* f, uint32_t v) { return std::fwrite(&v, 4, 1, f) == 1; }
bool get_u32(FILE* f, uint32_t& v) { return std::fread(&v, 4, 1, f) == 1; }

}  // namespace

int write_scene(const svo_scene& s, const std::string& base) {
  FILE* f = std::fopen((base + ".svo").c_str(), "wb");
  if (!f) return SVO_ERR_IO;
  bool ok = put_u32(f, (uint32_t)s.treelets.size()) && put_u32(f, s.treelet_bytes);
  for (const TreeletData& t : s.treelets) {
    if (!ok) break;
    ok = put_u32(f, t.num_nodes) && put_u32(f, t.num_leaves) && put_u32(f, t.mem_size) &&
         put_u32(f, t.gid) && put_u32(f, (uint32_t)t.parent_gid) &&
         put_u32(f, (uint32_t)t.parent_leaf_position) && put_u32(f, (uint32_t)t.parent_leaf_idx) &&
         put_u32(f, (uint32_t)t.parent_leaf_parent_position) &&
         std::fwrite(t.nodes.data(), sizeof(svo_node), t.num_nodes, f) == t.num_nodes;
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return SVO_ERR_IO;
  f = std::fopen((base + ".ia").c_str(), "wb");
  if (!f) return SVO_ERR_IO;
  ok = put_u32(f, (uint32_t)s.treelets.size());
  for (const TreeletData& t : s.treelets) {
    if (!ok) break;
    ok = put_u32(f, t.num_nodes) && put_u32(f, (uint32_t)sizeof(svo_attrib)) &&
         std::fwrite(t.attribs.data(), sizeof(svo_attrib), t.num_nodes, f) == t.num_nodes;
  }
  ok = (std::fclose(f) == 0) && ok;
  return ok ? SVO_OK : SVO_ERR_IO;
}

namespace {
uint32_t walk_max_depth(const svo_scene& s);
}

int read_scene(const std::string& base, svo_scene& s) {
  s = svo_scene();
  FILE* f = std::fopen((base + ".svo").c_str(), "rb");
  if (!f) return SVO_ERR_NOENT;
  uint32_t n = 0, bytes = 0;
  int rc = SVO_OK;
  if (!get_u32(f, n) || !get_u32(f, bytes) || n == 0 || bytes < 128 || bytes % 8 != 0) rc = SVO_ERR_IO;
  if (rc == SVO_OK) {
    s.treelet_bytes = bytes;
    s.treelets.resize(n);
    for (uint32_t i = 0; i < n && rc == SVO_OK; ++i) {
      TreeletData& t = s.treelets[i];
      uint32_t h[8];
      for (int k = 0; k < 8 && rc == SVO_OK; ++k)
        if (!get_u32(f, h[k])) rc = SVO_ERR_IO;
      if (rc != SVO_OK) break;
      t.num_nodes = h[0];
      t.num_leaves = h[1];
      t.mem_size = h[2];
      t.gid = h[3];
      t.parent_gid = (int32_t)h[4];
      t.parent_leaf_position = (int32_t)h[5];
      t.parent_leaf_idx = (int32_t)h[6];
      t.parent_leaf_parent_position = (int32_t)h[7];
      if (t.mem_size != bytes || t.num_nodes == 0 || t.num_nodes > bytes / 8 || t.gid != i ||
          t.parent_gid < 0 || (uint32_t)t.parent_gid >= n || t.parent_leaf_idx < 0 ||
          t.parent_leaf_idx > 7 || t.parent_leaf_position < 0 ||
          (uint32_t)t.parent_leaf_position >= bytes / 8 || t.parent_leaf_parent_position < 0 ||
          (uint32_t)t.parent_leaf_parent_position >= bytes / 8) {
        rc = SVO_ERR_IO;
        break;
      }
      t.nodes.resize(t.num_nodes);
      if (std::fread(t.nodes.data(), sizeof(svo_node), t.num_nodes, f) != t.num_nodes) rc = SVO_ERR_IO;
    }
  }
  std::fclose(f);
  if (rc != SVO_OK) {
    s = svo_scene();
    return rc;
  }
  f = std::fopen((base + ".ia").c_str(), "rb");
  if (!f) {
    s = svo_scene();
    return SVO_ERR_NOENT;
  }
  uint32_t na = 0;
  if (!get_u32(f, na) || na != n) rc = SVO_ERR_IO;
  for (uint32_t i = 0; i < n && rc == SVO_OK; ++i) {
    TreeletData& t = s.treelets[i];
    uint32_t cnt = 0, stride = 0;
    if (!get_u32(f, cnt) || !get_u32(f, stride) || cnt != t.num_nodes || stride != sizeof(svo_attrib)) {
      rc = SVO_ERR_IO;
      break;
    }
    t.attribs.resize(cnt);
    if (std::fread(t.attribs.data(), sizeof(svo_attrib), cnt, f) != cnt) rc = SVO_ERR_IO;
  }
  std::fclose(f);
  if (rc != SVO_OK) {
    s = svo_scene();
    return rc;
  }
  s.max_depth = walk_max_depth(s);
  return SVO_OK;
}

// ---------------------------------------------------------------------------
// flattening (SvoBranch::serializeSvo layout)

namespace {

struct Ref {
  uint32_t gid;
  uint32_t local;
  uint32_t depth;
};

// A treelet node is a real leaf when its parent flags it as a leaf and it
// carries no sub-treelet gid (src/TreeletBuildManager.cpp:229-233).
template <class Visit>
bool walk(const svo_scene& s, Visit&& visit) {
  std::deque<Ref> q;
  q.push_back(Ref{0, 0, 0});
  const uint32_t nt = (uint32_t)s.treelets.size();
  while (!q.empty()) {
    const Ref r = q.front();
    q.pop_front();
    const TreeletData& t = s.treelets[r.gid];
    if (r.local >= t.num_nodes) return false;
    const svo_node& nd = t.nodes[r.local];
    uint32_t child_ids[8];
    Ref children[8];
    uint32_t nc = 0;
    uint32_t rank = 0;
    for (uint32_t c = 0; c < 8; ++c) {
      if (!((nd.masks >> (c + 8)) & 1u)) continue;
      const uint32_t local = r.local + nd.first_child + rank;
      ++rank;
      if (local >= t.num_nodes) return false;
      Ref ch{r.gid, local, r.depth + 1};
      if ((nd.masks >> c) & 1u) {
        const uint32_t sub = t.nodes[local].first_child;
        if (sub != 0) {
          if (sub >= nt) return false;
          ch = Ref{sub, 0, r.depth + 1};
        }
      }
      child_ids[nc] = c;
      children[nc++] = ch;
    }
    if (!visit(r, nd, children, child_ids, nc)) return false;
    for (uint32_t i = 0; i < nc; ++i) q.push_back(children[i]);
  }
  return true;
}

uint32_t walk_max_depth(const svo_scene& s) {
  uint32_t md = 0;
  walk(s, [&](const Ref& r, const svo_node&, const Ref*, const uint32_t*, uint32_t) {
    md = std::max(md, r.depth);
    return true;
  });
  return md;
}

}  // namespace

int flatten_scene(const svo_scene& s, std::vector<svo_node>* nodes,
                  std::vector<svo_attrib>* attribs, uint64_t* count) {
  if (s.treelets.empty()) return SVO_ERR_INVALID;
  uint64_t emitted = 1;  // root is node 0
  if (nodes) nodes->clear();
  if (attribs) attribs->clear();
  if (nodes) nodes->push_back(svo_node{0u, 0u});
  if (attribs) attribs->push_back(s.treelets[0].attribs[0]);
  uint64_t index = 0;  // BFS index of the node being visited
  const bool ok = walk(s, [&](const Ref&, const svo_node& nd, const Ref* ch, const uint32_t* cid,
                              uint32_t nc) {
    if (nodes) {
      uint32_t masks = 0;
      for (uint32_t i = 0; i < nc; ++i) {
        masks |= 1u << (cid[i] + 8);
        const TreeletData& ct = s.treelets[ch[i].gid];
        const svo_node& cn = ct.nodes[ch[i].local];
        const bool treelet_leaf = ch[i].local != 0 && ((nd.masks >> cid[i]) & 1u);
        if (treelet_leaf && cn.first_child == 0) masks |= 1u << cid[i];
      }
      (*nodes)[index].masks = masks;
      (*nodes)[index].first_child = nc ? (uint32_t)emitted : 0u;
    }
    for (uint32_t i = 0; i < nc; ++i) {
      if (nodes) nodes->push_back(svo_node{0u, 0u});
      if (attribs) attribs->push_back(s.treelets[ch[i].gid].attribs[ch[i].local]);
    }
    emitted += nc;
    ++index;
    if (emitted > 0xFFFFFFFFull) return false;
    return true;
  });
  if (!ok) return SVO_ERR_INVALID;
  if (count) *count = emitted;
  return SVO_OK;
}

}  // namespace svo
