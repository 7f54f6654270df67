// gpu_builder.h -- the mesh -> fully resident incore pool builder on the GPU
// (gpu_builder.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/libsvo_b200.h"

namespace svo {

// A scene built on the device: the incore pool of a TreeletMemoryManager
// whose every treelet is resident (treelet gid g in slot g), in HBM.
struct DeviceScene {
  uint32_t depth = 0;
  uint32_t num_treelets = 0;
  uint64_t nodes_per_slot = 0;  // N = largest treelet + 8
  uint64_t pool_nodes = 0;      // num_treelets * N
  uint64_t octree_nodes = 0;    // octree nodes (all levels)
  uint64_t treelet_nodes = 0;   // sum of the treelets' node counts (boundary nodes twice)
  uint64_t leaf_voxels = 0;
  uint64_t pairs = 0;           // voxel/triangle overlaps found by the voxeliser
  svo_node* d_nodes = nullptr;
  svo_attrib* d_attribs = nullptr;

  DeviceScene() = default;
  DeviceScene(const DeviceScene&) = delete;
  DeviceScene& operator=(const DeviceScene&) = delete;
  ~DeviceScene();

  // h_normals / h_colors: per-vertex attributes (both or neither), as the
  // host builder's build_mesh_leaves takes them.
  int build_mesh(const float* h_vertices, const float* h_normals, const float* h_colors,
                 uint64_t num_vertices, const uint32_t* h_triangles, uint64_t num_triangles,
                 uint32_t depth, uint32_t treelet_levels, cudaStream_t stream);
};

}  // namespace svo
