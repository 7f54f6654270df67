// pool_scene.cpp -- a fully resident incore pool back to treelets.
//
// A pool in which every treelet g sits in slot g with its sub-treelets
// attached (what svo_mm_insert_all leaves in an incore buffer big enough for
// the whole octree, and what the GPU builder writes straight into HBM) holds
// every treelet's records, only patched where a sub-treelet hangs off a
// leaf: insertTreeletIntoIncoreBuffer (src/TreeletMemoryManager.cpp:518-545)
// copies the sub-treelet's root over the leaf, points its first child at the
// sub-treelet's slot + 1 and clears the leaf's flag in its parent node.  A
// treelet's own pointers stay inside its slot, so a valid node whose first
// child lands in another slot is such a patched leaf, and the slot it lands
// in names the sub-treelet.  Undoing the patch gives back the treelet file
// records (src/Treelet.cpp:403-419: the leaf stores the sub-treelet's gid,
// its flag is set in its parent) and the sub-treelet's header (parent gid,
// leaf position, child index, leaf parent position; src/Treelet.h:194-203),
// so an octree built on the GPU can be handed to a manager with a small
// incore buffer and paged like one read from a file.
#include <algorithm>
#include <cstring>

#include "errors.h"
#include "scene.h"

namespace svo {

// Slot g of a resident pool (its N node and attribute records, starting at
// pool index base = g * N) into scene.treelets[g]; the headers of the
// sub-treelets it links to are written into their entries.
int unpatch_slot(uint32_t g, uint64_t N, uint32_t num_slots, const svo_node* nodes,
                 const svo_attrib* attribs, svo_scene& scene) {
  if (g >= scene.treelets.size() || N < 2) return SVO_ERR_INVALID;
  const uint64_t base = (uint64_t)g * N;
  TreeletData& t = scene.treelets[g];
  t.gid = g;
  t.mem_size = (uint32_t)(N * 8);
  t.nodes.assign(nodes, nodes + N);
  // the treelet's extent: breadth-first from its root; the records of a
  // treelet are its reachable nodes, children after their parents
  uint64_t count = 1;
  std::vector<int32_t> sub(N, -1);  // local node -> sub-treelet gid when patched
  for (uint64_t i = 0; i < count; ++i) {
    const svo_node nd = t.nodes[i];
    const uint32_t valid = (nd.masks >> 8) & 0xFFu;
    if (!valid) continue;
    const uint64_t target = (uint32_t)((uint32_t)(base + i) + nd.first_child);
    if (target >= base && target < base + N) {
      const uint64_t last = target - base + (uint64_t)__builtin_popcount(valid) - 1;
      if (last >= N || target - base <= i) return SVO_ERR_INVALID;  // corrupt pool
      count = std::max(count, last + 1);
      continue;
    }
    // a patched leaf: the copy of sub-treelet c's root points at c's slot + 1
    const uint64_t c = target / N;
    if (i == 0 || target % N != 1 || c >= num_slots || c == g) return SVO_ERR_INVALID;
    sub[i] = (int32_t)c;
  }
  // undo the patches: the leaf holds the sub-treelet's gid, its flag is set
  // in its parent; the sub-treelet learns where it hangs
  uint32_t leaves = 0;
  for (uint64_t i = 0; i < count; ++i) {
    svo_node& nd = t.nodes[i];
    const uint32_t valid = (nd.masks >> 8) & 0xFFu;
    if (!valid || sub[i] >= 0) continue;
    const uint64_t first = (uint32_t)((uint32_t)(base + i) + nd.first_child) - base;
    uint32_t rank = 0;
    for (uint32_t b = 0; b < 8; ++b) {
      if (!((valid >> b) & 1u)) continue;
      const uint64_t j = first + rank++;
      const int32_t c = sub[j];
      if (c < 0) continue;
      nd.masks |= 1u << b;
      TreeletData& ct = scene.treelets[(uint32_t)c];
      ct.parent_gid = (int32_t)g;
      ct.parent_leaf_position = (int32_t)j;
      ct.parent_leaf_idx = (int32_t)b;
      ct.parent_leaf_parent_position = (int32_t)i;
    }
  }
  for (uint64_t i = 0; i < count; ++i) {
    if (sub[i] >= 0) t.nodes[i] = svo_node{(uint32_t)sub[i], 0u};
    if (!((t.nodes[i].masks >> 8) & 0xFFu)) ++leaves;  // not expanded in this treelet
  }
  t.nodes.resize(count);
  t.attribs.assign(attribs, attribs + count);
  t.num_nodes = (uint32_t)count;
  t.num_leaves = leaves;
  if (g == 0) {
    t.parent_gid = 0;
    t.parent_leaf_position = 0;
    t.parent_leaf_idx = 0;
    t.parent_leaf_parent_position = 0;
  }
  return SVO_OK;
}

int scene_from_pool(const svo_node* nodes, const svo_attrib* attribs, uint32_t num_slots,
                    uint32_t treelet_bytes, uint32_t max_depth, uint64_t leaf_voxels,
                    svo_scene& out) {
  if (!nodes || !attribs || num_slots == 0 || treelet_bytes < 16 || treelet_bytes % 8)
    return SVO_ERR_INVALID;
  const uint64_t N = treelet_bytes / 8;
  out = svo_scene();
  out.treelet_bytes = treelet_bytes;
  out.max_depth = max_depth;
  out.leaf_voxels = leaf_voxels;
  out.treelets.resize(num_slots);
  for (uint32_t g = 0; g < num_slots; ++g) {
    const int rc = unpatch_slot(g, N, num_slots, nodes + (uint64_t)g * N, attribs + (uint64_t)g * N, out);
    if (rc != SVO_OK) return rc;
  }
  return SVO_OK;
}

}  // namespace svo
