// scene.h -- octrees cut into treelets (host side).
//
// A scene is what the reference's TreeletBuildManager writes and
// TreeletMemoryManager::loadFromFile reads back: a list of fixed-size
// treelets (src/Treelet.h:62-216) plus one attribute record per node.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/libsvo_b200.h"

namespace svo {

// One treelet: the header fields of src/Treelet.h:194-203 and its nodes and
// attributes.  Only the first num_nodes records are stored; a slot holds
// mem_size / 8 records and the tail is zero.
struct TreeletData {
  uint32_t num_nodes = 0;
  uint32_t num_leaves = 0;
  uint32_t mem_size = 0;
  uint32_t gid = 0;
  int32_t parent_gid = 0;
  int32_t parent_leaf_position = 0;
  int32_t parent_leaf_idx = 0;
  int32_t parent_leaf_parent_position = 0;
  std::vector<svo_node> nodes;
  std::vector<svo_attrib> attribs;
};

// Full octree as per-level arrays.  Level d holds the nodes at depth d in
// Morton order (child index 4x+2y+z, as in sample()); children of a node are
// contiguous in the next level, starting at first[d][i].
struct Octree {
  uint32_t depth = 0;
  std::vector<std::vector<uint64_t>> codes;
  std::vector<std::vector<uint8_t>> masks;
  std::vector<std::vector<uint64_t>> first;
  std::vector<std::vector<svo_attrib>> attribs;
  uint64_t total_nodes() const;
};

}  // namespace svo

struct svo_scene {
  uint32_t treelet_bytes = 0;
  uint32_t max_depth = 0;
  uint64_t leaf_voxels = 0;
  std::vector<svo::TreeletData> treelets;
};

namespace svo {

// Leaves at `depth` (sorted, unique Morton codes) -> octree with attributes
// averaged bottom-up.
int octree_from_leaves(uint32_t depth, std::vector<uint64_t>&& codes,
                       std::vector<svo_attrib>&& leaf_attribs, Octree& out);

// Breadth-first treelet cut (the fill rule of
// src/TreeletBuilderFromFaces.cpp:189-365 and the treelet queue of
// src/TreeletBuildManager.cpp:150-258).
int cut_treelets(const Octree& tree, uint32_t treelet_levels, uint32_t treelet_bytes,
                 svo_scene& out);

int build_menger(uint32_t level, uint32_t depth, uint64_t seed, std::vector<uint64_t>& codes,
                 std::vector<svo_attrib>& attribs);

// Leaves of a triangle mesh.  With per-vertex normals and colours (both
// non-NULL, num_vertices x 3 floats each) a leaf gets the reference's rule
// (interpolated_leaf_attribute); without them, the normalised sum of the
// overlapping face normals and colour = normal * 0.5 + 0.5.
int build_mesh_leaves(const float* vertices, const float* normals, const float* colors,
                      uint64_t num_vertices, const uint32_t* triangles, uint64_t num_triangles,
                      uint32_t depth, int threads, std::vector<uint64_t>& codes,
                      std::vector<svo_attrib>& attribs);

// Morton code -> lattice coordinates (inverse of morton3).
void morton3_decode(uint64_t code, uint32_t& x, uint32_t& y, uint32_t& z);

int write_scene(const svo_scene& s, const std::string& base);
int read_scene(const std::string& base, svo_scene& s);

int flatten_scene(const svo_scene& s, std::vector<svo_node>* nodes, std::vector<svo_attrib>* attribs,
                  uint64_t* count);

// A fully resident incore pool (treelet g in slot g, sub-treelets attached)
// back to the treelets and headers it was filled from (pool_scene.cpp).
// unpatch_slot fills scene.treelets[g] from slot g's N records and the
// headers of the sub-treelets that slot links to.
int unpatch_slot(uint32_t g, uint64_t N, uint32_t num_slots, const svo_node* nodes,
                 const svo_attrib* attribs, svo_scene& scene);
int scene_from_pool(const svo_node* nodes, const svo_attrib* attribs, uint32_t num_slots,
                    uint32_t treelet_bytes, uint32_t max_depth, uint64_t leaf_voxels,
                    svo_scene& out);

// Colour/normal packing (gloost's compressAsColor / compressAsNormal are not
// part of the reference; these are the inverses of the kernel's unpacking,
// opencl/treeletRenderer_rgba.cl:183-195, 388-404).
uint32_t pack_color(float r, float g, float b);
uint32_t pack_normal(float x, float y, float z);
void unpack_color(uint32_t v, float rgb[3]);
void unpack_normal(uint32_t v, float n[3]);

uint64_t morton3(uint32_t x, uint32_t y, uint32_t z, uint32_t depth);

}  // namespace svo
