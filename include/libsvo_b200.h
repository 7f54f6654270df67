/*
 * libsvo_b200.h -- C ABI of the B200-native libsvo treelet ray cast.
 *
 * The entry points replace, one for one, the reference's OpenCL path:
 * TreeletMemoryManager / TreeletMemoryManagerCl (src/TreeletMemoryManager.h,
 * src/TreeletMemoryManagerCl.h) and the renderToBuffer kernel launch
 * (projects/raycast_serialized_opencl/src/raycast_serialized_opencl.cpp:
 * 315-324, 716, 729-747; kernel opencl/treeletRenderer_rgba.cl:610-734).
 *
 * Conventions
 *   - Every function returns an int status: SVO_OK (0) or a negative code.
 *     Nothing calls exit(); errors are never printed in place of a status.
 *   - Pointers named d_* are CUDA device pointers owned by the caller; h_*
 *     are host pointers.  `stream` is a cudaStream_t passed as void* (NULL =
 *     the legacy default stream).
 *   - Launches are asynchronous on `stream` unless stated otherwise.
 *   - Handles are not thread-safe: one manager per host thread, or locking
 *     by the caller (the reference is single-threaded too).
 */
#ifndef LIBSVO_B200_H
#define LIBSVO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define SVO_OK 0
#define SVO_ERR_NOENT (-2)     /* file not found (the reference exit(0)s)   */
#define SVO_ERR_IO (-5)        /* short read, bad header, write failure     */
#define SVO_ERR_NOMEM (-12)    /* host or device allocation failed          */
#define SVO_ERR_BUSY (-16)     /* no incore slot could be freed             */
#define SVO_ERR_INVALID (-22)  /* bad argument, id or size                  */
#define SVO_ERR_RANGE (-34)    /* value beyond a stated maximum             */
#define SVO_ERR_NOTSUP (-95)   /* mode or variant not supported             */
#define SVO_ERR_TIMEOUT (-110) /* a bounded wait gave up                    */
#define SVO_ERR_CANCELED (-125)/* request cancelled                         */
#define SVO_ERR_CUDA (-1000)   /* a CUDA runtime call failed                */

/* ---- data layouts ------------------------------------------------------ */

/* CpuSvoNode (src/CpuSvoNode.h:100-102; OpenCL SvoNode
 * opencl/treeletRenderer_rgba.cl:15-19).  masks: leaf bits 0-7, valid bits
 * 8-15.  first_child is relative to the node itself inside a treelet pool
 * (stored signed, read unsigned, adds wrap mod 2^32) and absolute in a flat
 * pool; a treelet leaf with a sub-treelet stores that treelet's gid. */
typedef struct svo_node {
  uint32_t first_child;
  uint32_t masks;
} svo_node;

/* Attribs (opencl/treeletRenderer_rgba.cl:23-26): packed normal and colour,
 * colour = r<<24 | g<<16 | b<<8 | a.  Same index as the node. */
typedef struct svo_attrib {
  uint32_t packed_normal;
  uint32_t packed_color;
} svo_attrib;

/* renderToBuffer kernel arguments 3..9 (opencl/treeletRenderer_rgba.cl:
 * 614-620) as plain floats.  The w components are ignored. */
typedef struct svo_frame_params {
  uint32_t width;           /* frameBufferSize.x                         */
  uint32_t height;          /* frameBufferSize.y                         */
  float t_scale_ratio;      /* frameBufferSize.z (LOD footprint per t)   */
  int32_t mode;             /* otherParams.x: 0 colour, 1 normal,
                               2 loops as wavelength colour, 3 octree
                               depth, 4 pixel depth, 5 loops, 6 Phong,
                               7 LOD quality (6, 7: treelet traversal
                               only)                                     */
  float pixel_far_h[4];     /* pixelFarVectorH                           */
  float pixel_far_v[4];     /* pixelFarVectorV                           */
  float far_lower_left[4];  /* far_lower_left                            */
  float camera_position[4]; /* cameraPosition                            */
} svo_frame_params;

/* Traversal variant. */
#define SVO_TRAVERSAL_TREELET 0 /* sample(), treeletRenderer_rgba.cl:201-382 */
#define SVO_TRAVERSAL_FLAT 1    /* CpuRaycasterSingleRay3::traversSvo        */

typedef struct svo_trace_cfg {
  int32_t traversal;  /* SVO_TRAVERSAL_*                                   */
  int32_t stack_size; /* treelet: MAX_STACK_SIZE (13 in the reference; the
                         descent stops at depth stack_size-1).  flat: the
                         octree's max depth.  Range 2..24.                 */
} svo_trace_cfg;

/* Per-pixel hit record (SampleResult fields used for parity). */
typedef struct svo_hit {
  uint32_t node_index; /* incore node index of the hit (0 on a miss)       */
  float t;             /* parent tMin at the hit; root tMax on a miss      */
  uint16_t depth;      /* SampleResult.depth                               */
  uint8_t hit;         /* 1 = hit                                          */
  uint8_t flags;       /* SVO_HITFLAG_*                                    */
  uint16_t loops;      /* SampleResult.numWhileLoops                       */
  uint16_t fetches;    /* loop iterations that read the parent node (each
                          one 8-byte node read of the algorithm)            */
} svo_hit;

#define SVO_HITFLAG_CAPPED 1  /* the maxLoops watchdog ended the ray           */
#define SVO_HITFLAG_BOUNDS 2  /* a node index fell outside the pool: ray ended */
#define SVO_HITFLAG_BOXMISS 4 /* the ray missed the root cube                  */

/* Device-side counters a launch adds to (optional). */
typedef struct svo_stats {
  uint32_t capped_rays;   /* rays ended by the loop watchdog             */
  uint32_t bounds_errors; /* rays that met an out-of-pool node index     */
  uint32_t reserved[2];
} svo_stats;

/* ---- scenes (octree construction, host side) --------------------------- */

typedef struct svo_scene svo_scene;

typedef struct svo_scene_info {
  uint32_t num_treelets;
  uint32_t treelet_bytes;     /* Treelet::getMemSize(), uniform slot size */
  uint32_t nodes_per_treelet; /* treelet_bytes / 8                        */
  uint32_t max_depth;         /* deepest node level                       */
  uint64_t total_nodes;       /* sum of Treelet::getNumNodes()            */
  uint64_t leaf_voxels;       /* voxels at max_depth                      */
} svo_scene_info;

/* Menger sponge of `level` (3^level cells per axis) voxelised at `depth`
 * (2^depth lattice, sponge centred), colour = hash(x, y, z, seed).  Treelets
 * are cut breadth first with the reference's fill rule
 * (src/TreeletBuilderFromFaces.cpp:200).  treelet_levels = L > 0 puts
 * treelet boundaries at depths D, D-L, D-2L, ... (D = octree depth): every
 * treelet below the top one spans L levels and ends on the leaves; 0 = no
 * level boundaries.  treelet_bytes = 0 picks the smallest slot size that
 * holds the largest treelet whole (the whole octree when L = 0). */
int svo_scene_build_menger(uint32_t level, uint32_t depth, uint64_t seed, uint32_t treelet_levels,
                           uint32_t treelet_bytes, svo_scene** out);

/* Triangle mesh (inside the unit cube centred at the origin) voxelised at
 * `depth` with a triangle/box overlap test; leaf colour from the averaged
 * face normal, inner nodes averaged from their children
 * (src/attribute_generators/Ag_colorAndNormalsTriangles.cpp:175-300). */
int svo_scene_build_mesh(const float* h_vertices, uint64_t num_vertices,
                         const uint32_t* h_triangles, uint64_t num_triangles, uint32_t depth,
                         uint32_t treelet_levels, uint32_t treelet_bytes, int32_t threads,
                         svo_scene** out);

/* ---- scenes built on the GPU ------------------------------------------- */

/* svo_scene_build_mesh + svo_mm_create_from_scene + svo_mm_insert_all +
 * svo_mm_init_device_buffer in one step on the GPU, for octrees too large to
 * build on the host: the mesh is voxelised, the octree built and cut into
 * treelets in device memory, and every treelet written to its slot of a
 * fully resident incore pool (treelet gid g in slot g, sub-treelet roots
 * patched into their parents' leaves), bit for bit the pool the host path
 * produces.  Stands in for TreeletBuilderFromFaces / TreeletBuildManager
 * (src/TreeletBuilderFromFaces.cpp:189-365, src/TreeletBuildManager.cpp:
 * 150-258) and the insertion loop (src/TreeletMemoryManager.cpp:518-545).
 * The slot size is always the automatic one (largest treelet + 8 nodes).
 * Blocks until the pool is built; scratch memory is freed before returning. */
typedef struct svo_device_scene svo_device_scene;
int svo_device_scene_build_mesh(const float* h_vertices, uint64_t num_vertices,
                                const uint32_t* h_triangles, uint64_t num_triangles,
                                uint32_t depth, uint32_t treelet_levels, void* stream,
                                svo_device_scene** out);
/* As svo_scene_info_get of the equivalent host scene. */
int svo_device_scene_info_get(const svo_device_scene* scene, svo_scene_info* out);
/* The pool: num_nodes = num_treelets * nodes_per_treelet records each. */
int svo_device_scene_buffers(const svo_device_scene* scene, const svo_node** d_nodes,
                             const svo_attrib** d_attribs, uint64_t* num_nodes);
/* Copies pool records [first, first + count) to host memory (either output
 * may be NULL); blocking. */
int svo_device_scene_copy(const svo_device_scene* scene, uint64_t first, uint64_t count,
                          svo_node* h_nodes, svo_attrib* h_attribs);
/* Octree nodes over all levels and voxel/triangle overlaps found. */
int svo_device_scene_counts(const svo_device_scene* scene, uint64_t* octree_nodes,
                            uint64_t* overlaps);
void svo_device_scene_destroy(svo_device_scene* scene);
/* Undoes svo_mm_insert_all: a fully resident incore pool (treelet g in slot
 * g, num_slots slots of treelet_bytes, every sub-treelet attached by the
 * patch of insertTreeletIntoIncoreBuffer, src/TreeletMemoryManager.cpp:
 * 518-545) back into the treelets and headers of the treelet file
 * (src/Treelet.cpp:403-419, src/Treelet.h:194-203).  SVO_ERR_INVALID on a
 * pool that is not such a pool. */
int svo_scene_from_pool(const svo_node* h_nodes, const svo_attrib* h_attribs, uint32_t num_slots,
                        uint32_t treelet_bytes, uint32_t max_depth, uint64_t leaf_voxels,
                        svo_scene** out);

/* svo_scene_build_mesh / svo_device_scene_build_mesh with per-vertex normals
 * and colours (num_vertices x 3 floats each, colours in [0, 1]; both or
 * neither).  A leaf then gets the reference's attributes
 * (src/attribute_generators/Ag_colorAndNormalsTriangles.cpp:110-155 with
 * src/BuilderTriangleFace.cpp:211-329): for each overlapping triangle the
 * barycentric (u, v) of the voxel centre along the triangle's mean vertex
 * normal, clamped to [0, 1], the normalised interpolated vertex normal and the
 * interpolated colour; their mean over the triangles, the normal normalised.
 * Without them: normalised sum of the face normals, colour = normal*0.5+0.5. */
int svo_scene_build_mesh_attributed(const float* h_vertices, const float* h_normals,
                                    const float* h_colors, uint64_t num_vertices,
                                    const uint32_t* h_triangles, uint64_t num_triangles,
                                    uint32_t depth, uint32_t treelet_levels,
                                    uint32_t treelet_bytes, int32_t threads, svo_scene** out);
int svo_device_scene_build_mesh_attributed(const float* h_vertices, const float* h_normals,
                                           const float* h_colors, uint64_t num_vertices,
                                           const uint32_t* h_triangles, uint64_t num_triangles,
                                           uint32_t depth, uint32_t treelet_levels, void* stream,
                                           svo_device_scene** out);
/* Per-vertex attributes for a mesh: normals = normalised sum of the adjacent
 * (area-weighted) face normals; colours = a seeded smooth field of the
 * position.  Writes num_vertices x 3 floats to each output. */
int svo_mesh_vertex_attributes(const float* h_vertices, uint64_t num_vertices,
                               const uint32_t* h_triangles, uint64_t num_triangles, uint64_t seed,
                               float* h_normals, float* h_colors);

/* PLY meshes, the input of the reference's octree builder
 * (projects/octree_builder/src/octree_builder.cpp:85-157: "*.ply files with
 * per vertex color and normals").  ascii and binary_little_endian; vertex
 * x, y, z and, when present, nx, ny, nz and red, green, blue (integer
 * colours / 255); faces as vertex index lists, polygons split into fans.
 * SVO_ERR_NOTSUP for big-endian files. */
#define SVO_MESH_HAS_NORMALS 1u
#define SVO_MESH_HAS_COLORS 2u
typedef struct svo_mesh svo_mesh;
int svo_mesh_load_ply(const char* path, svo_mesh** out);
int svo_mesh_info(const svo_mesh* mesh, uint64_t* num_vertices, uint64_t* num_triangles,
                  uint32_t* flags);
/* Copies num_vertices x 3 floats (positions, normals, colours) and
 * num_triangles x 3 indices; any output may be NULL, a missing attribute
 * requested is SVO_ERR_INVALID. */
int svo_mesh_copy(const svo_mesh* mesh, float* h_vertices, float* h_normals, float* h_colors,
                  uint32_t* h_triangles);
void svo_mesh_destroy(svo_mesh* mesh);
/* The octree builder's placement (octree_builder.cpp:130-157): rotation by
 * rotate_x_deg about x, the bounding box centred at the origin and its
 * largest side scaled to 1, normals (optional) rotated and normalised; in
 * place. */
int svo_mesh_fit_unit_cube(float* h_vertices, float* h_normals, uint64_t num_vertices,
                           float rotate_x_deg);

/* Seeded synthetic meshes (inputs for svo_scene_build_mesh).  The reference
 * voxelises scanned PLY meshes that are not part of it; these stand in with
 * the triangle counts of the benchmark configurations.  Call *_size first.
 * Icosphere: 20 * 4^subdivisions faces, vertex radius
 * radius + amplitude * fbm(direction) (3D value noise, `octaves` octaves
 * from base `frequency`).  Terrain: grid x grid vertices over [-0.5,0.5]^2 in
 * x/z, y = base + height * fbm01(x, z). */
int svo_mesh_icosphere_size(uint32_t subdivisions, uint64_t* num_vertices, uint64_t* num_triangles);
int svo_mesh_icosphere(uint32_t subdivisions, float radius, uint32_t octaves, float amplitude,
                       float frequency, uint64_t seed, float* h_vertices, uint32_t* h_triangles);
int svo_mesh_terrain_size(uint32_t grid, uint64_t* num_vertices, uint64_t* num_triangles);
int svo_mesh_terrain(uint32_t grid, uint32_t octaves, float base, float height, float frequency,
                     uint64_t seed, float* h_vertices, uint32_t* h_triangles);

/* Writes / reads `<path_base>.svo` (the reference's treelet file layout,
 * src/TreeletBuildManager.cpp:305-312, src/Treelet.cpp:403-419) and
 * `<path_base>.ia` (per-treelet attribute records). */
int svo_scene_write(const svo_scene* scene, const char* path_base);
int svo_scene_read(const char* path_base, svo_scene** out);
int svo_scene_info_get(const svo_scene* scene, svo_scene_info* out);
/* Treelet header fields (src/Treelet.h:194-203). */
int svo_scene_treelet(const svo_scene* scene, uint32_t gid, uint32_t* num_nodes,
                      uint32_t* num_leaves, int32_t* parent_gid, int32_t* parent_leaf_position,
                      int32_t* parent_leaf_idx, int32_t* parent_leaf_parent_position);
/* Flat breadth-first pool with absolute first-child indices (the
 * SvoBranch::serializeSvo layout, src/incore/SvoBranch.cpp:233-308).
 * Pass NULL outputs to query the node count. */
int svo_scene_flatten(const svo_scene* scene, svo_node* h_nodes, svo_attrib* h_attribs,
                      uint64_t capacity, uint64_t* num_nodes);
void svo_scene_destroy(svo_scene* scene);

/* ---- treelet memory manager (TreeletMemoryManager + ...Cl) ------------- */

typedef struct svo_mm svo_mm;

typedef struct svo_mm_info {
  uint32_t num_treelets;
  uint32_t treelet_bytes;
  uint32_t nodes_per_treelet;
  uint32_t num_slots;
  uint32_t free_slots;
  uint32_t slots_to_upload;
  uint64_t incore_nodes;      /* slots * nodes_per_treelet                 */
  uint64_t device_bytes;      /* node + attribute device buffers           */
} svo_mm_info;

typedef struct svo_slot_info { /* TreeletMemoryManager::SlotInfo (.h:72-89) */
  int32_t treelet_gid;         /* -1 = empty                                 */
  int32_t visibility;
  float error;
} svo_slot_info;

/* TreeletMemoryManagerCl(svoFilePath, incoreBufferSizeInByte, ClContext*)
 * (src/TreeletMemoryManagerCl.h:69-71; loads <path>.svo/.ia and resets the
 * incore buffer, src/TreeletMemoryManager.cpp:72-102).  `stream` is the
 * stream renders run on; uploads use a side stream ordered by events. */
int svo_mm_create(const char* svo_path_base, uint64_t incore_bytes, void* stream, svo_mm** out);
/* Same, from an in-memory scene (copied; the scene stays owned by the caller). */
int svo_mm_create_from_scene(const svo_scene* scene, uint64_t incore_bytes, void* stream,
                             svo_mm** out);
/* A manager over a GPU-built octree whose incore buffer may be far smaller
 * than the octree: the device pool is copied to host memory in pieces of
 * about 256 MB and turned back into treelets and their headers (as
 * svo_scene_from_pool), which become the manager's host copy, paged into an
 * incore buffer of incore_bytes by insertion or the analysis pass like an
 * octree read with svo_mm_create.  The device scene is left as it is.
 * Blocking. */
int svo_mm_create_from_device_scene(const svo_device_scene* scene, uint64_t incore_bytes,
                                    void* stream, svo_mm** out);
void svo_mm_destroy(svo_mm* mm);

/* initClBuffer (src/TreeletMemoryManagerCl.cpp:101-113): allocates the
 * device node and attribute buffers and uploads the whole incore buffer. */
int svo_mm_init_device_buffer(svo_mm* mm);
/* getClIncoreBufferGid / getClAttributeIncoreBufferGid (.h:82-85). */
int svo_mm_get_device_buffers(svo_mm* mm, const svo_node** d_nodes, const svo_attrib** d_attribs,
                              uint64_t* num_nodes);
/* insertTreeletIntoIncoreBuffer (src/TreeletMemoryManager.cpp:456-548).
 * SVO_ERR_BUSY when no slot is free and none can be freed; SVO_ERR_INVALID
 * when the treelet's parent is not resident (the reference would patch an
 * unrelated node). */
int svo_mm_insert_treelet(svo_mm* mm, int32_t treelet_gid, int32_t visibility, float error);
/* removeTreeletFromIncoreBuffer (src/TreeletMemoryManager.cpp:666-700). */
int svo_mm_remove_treelet(svo_mm* mm, int32_t treelet_gid);
/* freeIncorePosition (src/TreeletMemoryManager.cpp:561-653). */
int svo_mm_free_incore_position(svo_mm* mm);
/* updateClientSideIncoreBuffer (src/TreeletMemoryManager.cpp:393-443) with
 * the analysis results passed as arrays (new visible treelets and their
 * errors; treelets already resident and still visible). */
int svo_mm_update_client_side(svo_mm* mm, const int32_t* new_gids, const float* new_errors,
                              uint32_t num_new, const int32_t* old_gids, uint32_t num_old);
/* updateDeviceMemory (src/TreeletMemoryManagerCl.cpp:155-251): uploads the
 * dirty slots, merging neighbours with the reference's 0.6 coalescing rule,
 * as async copies on the side stream; renders issued afterwards wait for
 * them.  *num_copy_calls (optional) receives the number of ranges (packed
 * policy: the number of packed copies). */
int svo_mm_update_device_memory(svo_mm* mm, uint32_t* num_copy_calls);
/* Upload policies.  COALESCED (default): the reference's slot ranges, each
 * staged through a pinned ring.  PACKED: only dirty slots, packed back to
 * back into the ring in 4 MB chunks (one copy per chunk), placed by a scatter
 * kernel.  PINNED: the host mirror is page-locked and mapped
 * (cudaHostRegister, so it costs its size in locked host memory) and one
 * kernel reads the dirty slots from it over PCIe and writes them in place;
 * host-side treelet changes then wait for a gather still reading the mirror.
 * All leave the same device pool.  No reference
 * counterpart: the reference hard-codes the coalesced form. */
#define SVO_UPLOAD_COALESCED 0
#define SVO_UPLOAD_PACKED 1
#define SVO_UPLOAD_PINNED 2
int svo_mm_set_upload_policy(svo_mm* mm, int32_t policy);
/* The coalescing ratio of the COALESCED policy: a range grows over the next
 * dirty slot while (treelets + 1) / (slot distance + 1) >= 2 * ratio.  The
 * reference's value is 0.6 (TreeletMemoryManagerCl.cpp:188); 1 copies each
 * slot alone, 0 copies one range from the first to the last dirty slot.
 * SVO_ERR_RANGE outside [0, 1]. */
int svo_mm_set_upload_ratio(svo_mm* mm, float ratio);
/* The copy ranges the next svo_mm_update_device_memory will issue: slot
 * ranges (first slot, slot count) merged with the 0.6 rule of
 * TreeletMemoryManagerCl.cpp:177-211.  Pass NULL arrays to query the count. */
int svo_mm_plan_uploads(svo_mm* mm, uint32_t* h_first_slots, uint32_t* h_slot_counts,
                        uint32_t capacity, uint32_t* num_ranges);
/* resetIncoreBuffer (src/TreeletMemoryManager.cpp:304-380). */
int svo_mm_reset(svo_mm* mm);
/* Inserts treelets in gid order (parents first) until every treelet is
 * resident or the slots run out.  No reference counterpart: it replaces the
 * analysis-driven fill for fully resident scenes. */
int svo_mm_insert_all(svo_mm* mm, uint32_t* num_inserted);
int svo_mm_info_get(svo_mm* mm, svo_mm_info* out);
/* getSlots (src/TreeletMemoryManager.h:157). */
int svo_mm_get_slot(svo_mm* mm, uint32_t slot, svo_slot_info* out);
/* Treelet::getSlotGid for a gid: the slot, or -1 when not resident. */
int svo_mm_treelet_slot(svo_mm* mm, int32_t treelet_gid, int32_t* slot);
/* getIncoreBuffer / getAttributeIncoreBuffer (host mirror), nodes
 * [first, first+count). Either output may be NULL. */
int svo_mm_copy_incore(svo_mm* mm, uint64_t first, uint64_t count, svo_node* h_nodes,
                       svo_attrib* h_attribs);
/* getIncoreSlotsToUpload (.h:153): up to `capacity` slot ids, ascending. */
int svo_mm_slots_to_upload(svo_mm* mm, uint32_t* h_slots, uint32_t capacity, uint32_t* count);

/* ---- ray cast ---------------------------------------------------------- */

/* renderToBuffer over a whole frame (opencl/treeletRenderer_rgba.cl:
 * 610-734; enqueue raycast_serialized_opencl.cpp:729-747).  Writes W*H
 * RGBA8 pixels (byte 0 red) to d_rgba and, when d_hits is not NULL, one
 * svo_hit per pixel.  d_stats (optional) accumulates counters. */
int svo_render(const svo_node* d_nodes, const svo_attrib* d_attribs, uint64_t num_nodes,
               const svo_frame_params* params, const svo_trace_cfg* cfg, uint32_t* d_rgba,
               svo_hit* d_hits, svo_stats* d_stats, void* stream);

/* sample() on explicit rays (d_origins, d_dirs: n x 3 floats). */
int svo_trace_rays(const svo_node* d_nodes, uint64_t num_nodes, const float* d_origins,
                   const float* d_dirs, uint64_t n, float t_scale_ratio,
                   const svo_trace_cfg* cfg, svo_hit* d_hits, svo_stats* d_stats, void* stream);

/* svo_render over the manager's incore buffer, after its pending uploads.
 * Counters accumulate in the manager (read with svo_mm_sync). */
int svo_mm_render(svo_mm* mm, const svo_frame_params* params, const svo_trace_cfg* cfg,
                  uint32_t* d_rgba, svo_hit* d_hits, void* stream);
/* Blocking frame into host memory: launch, copy the W*H RGBA8 image to
 * h_rgba, wait.  This is the reference's blocking enqueueKernel plus the
 * image read back. */
int svo_mm_render_host(svo_mm* mm, const svo_frame_params* params, const svo_trace_cfg* cfg,
                       uint32_t* h_rgba, void* stream);
/* Shadow rays: one per primary hit, toward a directional light. */
typedef struct svo_shadow_cfg {
  float light_direction[3]; /* unit vector toward the light, used as given  */
  float t_scale_ratio;      /* tScaleRatio of the shadow rays (0.001)      */
  float normal_offset;      /* origin = hit node centre + normal * offset
                               (0.01)                                      */
  uint32_t reserved;        /* 0                                           */
} svo_shadow_cfg;

/* Primary ray plus one shadow ray per hit, shaded as
 * shade_diffuse_color_shadow (opencl/fillFrameBuffer_rgba.cl:494-529; the
 * live renderer's shade_phong has its shadow ray compiled out, :475-484) with
 * the live renderer's attribute index (= node index): the shadow ray is
 * sample() (opencl/treeletRenderer_rgba.cl:201-382) from nodeCenter +
 * normal * offset.  params->mode is ignored; treelet traversal only.  Writes
 * RGBA8 to d_rgba and, when not NULL, the primary and the shadow hit record
 * per pixel (zeros where no shadow ray was cast). */
int svo_render_shadow(const svo_node* d_nodes, const svo_attrib* d_attribs, uint64_t num_nodes,
                      const svo_frame_params* params, const svo_trace_cfg* cfg,
                      const svo_shadow_cfg* shadow, uint32_t* d_rgba, svo_hit* d_hits,
                      svo_hit* d_shadow_hits, svo_stats* d_stats, void* stream);
/* svo_render_shadow over the manager's incore buffer, after its pending
 * uploads; counters accumulate in the manager. */
int svo_mm_render_shadow(svo_mm* mm, const svo_frame_params* params, const svo_trace_cfg* cfg,
                         const svo_shadow_cfg* shadow, uint32_t* d_rgba, svo_hit* d_hits,
                         svo_hit* d_shadow_hits, void* stream);

/* Non-blocking svo_mm_render_host for frame loops: the frame is cast on
 * `stream` into one of two device images and copied to h_rgba on a second
 * stream, so the copy of one frame overlaps the cast of the next.  h_rgba
 * (page-locked host memory, W*H RGBA8) holds the frame once svo_mm_sync
 * returns; it must stay valid until then. */
int svo_mm_render_host_async(svo_mm* mm, const svo_frame_params* params, const svo_trace_cfg* cfg,
                             uint32_t* h_rgba, void* stream);
/* svo_mm_render_host_async for the primary + shadow ray frame
 * (svo_mm_render_shadow's image, pipelined the same way; the two calls
 * share the manager's two device images). */
int svo_mm_render_shadow_host_async(svo_mm* mm, const svo_frame_params* params,
                                    const svo_trace_cfg* cfg, const svo_shadow_cfg* shadow,
                                    uint32_t* h_rgba, void* stream);
/* Waits for `stream` and for every svo_mm_render_host_async and
 * svo_mm_render_shadow_host_async copy, and
 * returns the manager's accumulated counters
 * (capped rays = the watchdog status word), then clears them. */
int svo_mm_sync(svo_mm* mm, void* stream, svo_stats* out);

/* ---- analysis pass: visibility-driven paging --------------------------- */

/* FeedBackDataElement (opencl/treeletRenderer_rgba.cl:761-766). */
typedef struct svo_feedback {
  int32_t node_id;         /* incore index of the node the ray stopped at, 0 = none */
  float error;             /* leaf: scale_exp2 - tScaleRatio*tcMin; LOD stop: 1/0  */
  int32_t sub_treelet_gid; /* leaf's sub-treelet gid when not resident, else 0     */
  float t_min;             /* tcMin of that node; 9999999 when nothing was hit     */
} svo_feedback;

/* renderToFeedbackBuffer (opencl/treeletRenderer_rgba.cl:960-1011): one
 * analysis ray per pixel of `params` (sampleAnalyse, :773-953), one record
 * per pixel into d_feedback; d_rgba (optional) receives the kernel's debug
 * colour as RGBA8. */
int svo_feedback_render(const svo_node* d_nodes, uint64_t num_nodes, const svo_frame_params* params,
                        int32_t stack_size, svo_feedback* d_feedback, uint32_t* d_rgba,
                        void* stream);
/* RenderPassAnalyse::performAnalysePass's processing of the records
 * (src/RenderPassAnalyse.cpp:218-356): newly visible treelets (at most
 * max_new; 0 = the reference's 12 MB worth) and visible resident treelets
 * with their ancestors, as gid/error arrays, largest error first; pass them
 * to svo_mm_update_client_side.  SVO_ERR_RANGE with empty lists on records
 * the reference rejects.  Capacities smaller than the lists give
 * SVO_ERR_RANGE with the needed counts in *num_new / *num_old. */
int svo_mm_analyse_feedback(svo_mm* mm, const svo_feedback* h_feedback, uint64_t n, uint32_t max_new,
                            int32_t* new_gids, float* new_errors, uint32_t new_capacity,
                            uint32_t* num_new, int32_t* old_gids, float* old_errors,
                            uint32_t old_capacity, uint32_t* num_old);
/* The same processing over records in device memory (d_feedback, as
 * svo_feedback_render writes them): the records are folded on the GPU into
 * per-treelet largest errors and only those come back (4 bytes per treelet
 * per list instead of 16 bytes per record); lists and statuses as
 * svo_mm_analyse_feedback on the same records.  Blocks until the lists are
 * on the host.  Needs svo_mm_init_device_buffer. */
int svo_mm_analyse_feedback_device(svo_mm* mm, const svo_feedback* d_feedback, uint64_t n,
                                   uint32_t max_new, void* stream, int32_t* new_gids,
                                   float* new_errors, uint32_t new_capacity, uint32_t* num_new,
                                   int32_t* old_gids, float* old_errors, uint32_t old_capacity,
                                   uint32_t* num_old);
/* One dynamic-loading step of the reference's frame loop
 * (raycast_serialized_opencl.cpp:684-716): the analysis pass over the
 * frame's view at (width/divisor, height/divisor) with the far plane's
 * origin offset by (jitter_x, jitter_y) * divisor / 2 frame pixels (the
 * reference's "rumble", RenderPassAnalyse.cpp:176-184; jitter in [-1, 1]),
 * records analysed on the GPU (svo_mm_analyse_feedback_device), treelets
 * inserted (evicting by visibility) and uploaded.  Blocks until the analysis
 * lists are on the host.  *num_new: the treelets placed; like the
 * reference's updateClientSideIncoreBuffer, the step skips new treelets that
 * find no slot under memory pressure (the next step asks for them again).
 * *num_old: visible resident treelets. */
/* The bytes of newly visible treelets one analysis step may place: the
 * reference's pass is capped at 12 MB (maxTreeletsToPropergate,
 * src/RenderPassAnalyse.cpp:340), paced for PCIe 2; 0 restores that cap.
 * SVO_ERR_RANGE below one treelet. */
int svo_mm_set_analysis_budget(svo_mm* mm, uint64_t bytes);
/* Which treelet freeIncorePosition may evict.  SVO_EVICT_REFERENCE (default,
 * src/TreeletMemoryManager.cpp:571-579): one unseen for the visibility
 * counter's 9 passes whose parent is unseen too; the root's slot never ages,
 * so its own sub-treelets are never evicted.  SVO_EVICT_ANY_UNSEEN: any
 * unseen treelet, whatever its parent (its attached subtree goes with it),
 * so that a buffer full of treelets one view no longer sees makes room for
 * the next.  No reference counterpart. */
#define SVO_EVICT_REFERENCE 0
#define SVO_EVICT_ANY_UNSEEN 1
int svo_mm_set_eviction(svo_mm* mm, int32_t rule);
/* Newly visible treelets the last svo_mm_analysis_step asked for, placed or
 * not: 0 once the view needs no treelet that is not resident (the step's
 * *num_new counts only those placed, which a full buffer keeps at 0). */
int svo_mm_analysis_requested(svo_mm* mm, uint32_t* requested);
int svo_mm_analysis_step(svo_mm* mm, const svo_frame_params* frame, uint32_t divisor,
                         float jitter_x, float jitter_y, int32_t stack_size, void* stream,
                         uint32_t* num_new, uint32_t* num_old);
/* svo_mm_analysis_step in two halves (no reference counterpart: the
 * reference runs the analysis pass, the update and the frame one after the
 * other).  _begin launches the analysis rays and the GPU fold on `stream`
 * (after the manager's pending uploads) and returns; _end waits for them,
 * inserts and evicts on the host and uploads the dirty slots once the work
 * already queued on `after_stream` is done.  A loop that begins the analysis
 * of view k+1 before casting frame k on another stream, and ends it after,
 * overlaps the two and produces the frames of the sequential loop: both read
 * the same pool.  No insertion, removal, update or other analysis may come
 * between _begin and _end: those calls return SVO_ERR_BUSY meanwhile, as
 * does a second _begin; _end without _begin is SVO_ERR_INVALID. */
int svo_mm_analysis_begin(svo_mm* mm, const svo_frame_params* frame, uint32_t divisor,
                          float jitter_x, float jitter_y, int32_t stack_size, void* stream);
int svo_mm_analysis_end(svo_mm* mm, void* after_stream, uint32_t* num_new, uint32_t* num_old);

/* ---- batched views: one persistent launch ------------------------------ */

/* A resident octree: device node and attribute pools (e.g. from
 * svo_mm_get_device_buffers) and how to traverse them. */
typedef struct svo_octree_desc {
  const svo_node* d_nodes;
  const svo_attrib* d_attribs;
  uint64_t num_nodes;
  int32_t traversal;  /* SVO_TRAVERSAL_*                                   */
  int32_t stack_size; /* as in svo_trace_cfg                               */
} svo_octree_desc;

/* One view of a batch: renderToBuffer's arguments, the octree it looks at
 * (index into the batch's octree table) and its outputs. */
typedef struct svo_view_desc {
  svo_frame_params params;
  uint32_t octree;
  uint32_t reserved;
  uint32_t* d_rgba; /* width*height RGBA8 pixels, byte 0 red           */
  svo_hit* d_hits;  /* optional, width*height records                   */
} svo_view_desc;

typedef struct svo_batch_cfg {
  uint32_t tile_w, tile_h;  /* pixels per warp tile: 8x4, 16x2, 4x8 or 32x1  */
  uint32_t block_threads;   /* multiple of 32, 64..1024                      */
  uint32_t blocks_per_sm;   /* persistent blocks per SM, 0 = as many as fit  */
  uint32_t top_nodes;       /* records of octree 0 staged in shared memory   */
  uint32_t use_graph;       /* replay a captured CUDA graph                  */
  uint32_t rays_per_lane;   /* rays a lane casts per tile: 1, 2 or 4 (0 = 1);
                               a tile is tile_w x (tile_h * rays_per_lane)
                               pixels, one counter pull per tile              */
} svo_batch_cfg;

/* The launch unit of the reference is one frame (renderToBuffer enqueue,
 * raycast_serialized_opencl.cpp:742-747); a batcher casts a ragged table of
 * views over one or several octrees in one persistent, work-stealing launch
 * (32-pixel tiles pulled from a device counter).  A batcher owns the device
 * descriptor tables (allocated at creation) and is not thread-safe. */
typedef struct svo_batcher svo_batcher;
int svo_batcher_create(uint32_t max_views, uint32_t max_octrees, svo_batcher** out);
void svo_batcher_destroy(svo_batcher* b);
/* Sets the batch: validates and uploads the descriptors (waits for earlier
 * work on `stream` first).  The octree pools and outputs must stay valid
 * while launches of this batch run. */
int svo_batcher_set(svo_batcher* b, const svo_octree_desc* octrees, uint32_t num_octrees,
                    const svo_view_desc* views, uint32_t num_views, const svo_batch_cfg* cfg,
                    void* stream);
/* Casts every view of the current batch (asynchronous).  d_stats
 * (optional) accumulates counters.  With cfg.use_graph the counter reset
 * and the kernel are captured as a CUDA graph on the first launch and
 * replayed afterwards. */
int svo_batcher_launch(svo_batcher* b, svo_stats* d_stats, void* stream);
/* Times each tile shape, block size, top-node staging and rays per lane
 * on the current batch (`reps` launches each), keeps the fastest as the
 * batch's configuration and returns it with its time per launch. */
int svo_batcher_autotune(svo_batcher* b, uint32_t reps, void* stream, svo_batch_cfg* best,
                         float* best_ms);
/* Total tiles and rays of the current batch. */
int svo_batcher_size(svo_batcher* b, uint64_t* tiles, uint64_t* rays);

/* The batched cast for callers that may not allocate device memory (no
 * counterpart in the reference).  A host that owns and budgets all of HBM
 * through its own allocator, or a latency-critical loop where cudaMalloc /
 * cudaFree could synchronise the device, passes its octree pools and output
 * buffers and nothing is allocated: the descriptor tables and the tile
 * counter live in a fixed 29,440-byte device array inside the library, held
 * by every GPU that loads it until the process exits.  At most 256 views and
 * 16 octrees per call (SVO_ERR_RANGE otherwise); tile 8x4, 16x2, 4x8 or 32x1;
 * 256-thread persistent blocks.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) with that device current
 * and keeps it for the life of the process (do not use the library across a
 * cudaDeviceReset); make that first call before any stream capture.  The
 * descriptor tables reach the array as the by-value parameter of a small
 * loader kernel launched on `stream` before the cast, so no host memory of
 * the call is read after it returns.  All calls share the one array, which
 * keeps the last call's contents; each call rewrites it and zeroes its
 * counter, and calls whose work overlaps on the GPU race. */
int svo_render_batch_static(const svo_octree_desc* octrees, uint32_t num_octrees,
                            const svo_view_desc* views, uint32_t num_views, uint32_t tile_w,
                            uint32_t tile_h, svo_stats* d_stats, void* stream);

/* ---- serving: a request loop over resident octrees --------------------- */

/* The reference pages treelets for one octree per frame and renders one
 * frame per kernel (TreeletMemoryManager::updateClientSideIncoreBuffer,
 * src/TreeletMemoryManager.cpp:393-548; raycast_serialized_opencl.cpp:
 * 680-747).  A server accepts cast requests at any time from any thread:
 * a dispatcher thread admits them against an HBM budget (octree pools) and
 * an in-flight ray budget, pages the treelets of their octrees into one
 * pre-allocated device pool through pinned asynchronous copies on a side
 * stream (evicting the least recently used idle octree when full), and
 * launches everything admitted as one batch on the next free stream, so work
 * that arrives while other batches run overlaps with them on the device. */
#define SVO_SERVE_BATCHED 0 /* batched launches on `streams` streams       */
#define SVO_SERVE_PLAIN 1   /* one per-frame kernel per request, one stream */
/* One per-frame kernel per request, launched as soon as it is admitted,
 * round robin over `streams` streams, completion by polled CUDA events: no
 * launch slots and no host callback gate the plain kernel. */
#define SVO_SERVE_PLAIN_STREAMED 2

typedef struct svo_server_cfg {
  uint64_t hbm_budget_bytes;  /* device pool for octree node+attribute pools */
  uint64_t max_inflight_rays; /* admission: rays launched, not yet finished  */
  uint32_t streams;           /* concurrent launches, 1..16                  */
  uint32_t max_batch_views;   /* requests per batched launch                 */
  uint32_t mode;              /* SVO_SERVE_*                                 */
  uint32_t tile_w, tile_h;    /* batch tile shape (0 = 8x4)                   */
  uint32_t block_threads;     /* batch block size (0 = 128)                  */
} svo_server_cfg;

typedef struct svo_request {
  uint32_t octree; /* id from svo_server_add_octree                       */
  uint32_t reserved;
  svo_frame_params params;
  uint32_t* d_rgba; /* width*height RGBA8 output, device, owned by caller */
} svo_request;

typedef struct svo_request_result {
  int32_t status;  /* SVO_OK, SVO_ERR_CANCELED, or the error that ended it */
  uint32_t batch;  /* launch sequence number                               */
  double submit_s; /* server clock, seconds since svo_server_create        */
  double launch_s;
  double done_s;   /* stamped by a callback when the launch finished       */
} svo_request_result;

typedef struct svo_server_stats {
  uint64_t requests_done, rays_done, batches;
  uint64_t octree_loads, octree_evictions, treelets_paged_in, bytes_uploaded;
  uint64_t resident_bytes;
  uint32_t resident_octrees;
  uint32_t paged_unconverged; /* paged requests cast after the last analysis
                                 pass still placed treelets (region too small
                                 for the view)                                */
  uint64_t analysis_passes;   /* analysis passes run for paged requests       */
  uint64_t paging_us;         /* time paged workers spent in those passes and
                                 their uploads, summed over workers           */
} svo_server_stats;

typedef struct svo_server svo_server;
/* Allocates the device pool (hbm_budget_bytes) and starts the dispatcher. */
int svo_server_create(const svo_server_cfg* cfg, svo_server** out);
/* Cancels requests not yet launched, waits for running ones, frees all. */
void svo_server_destroy(svo_server* s);
/* Registers an octree (copied) with the given stack size; not resident
 * until a request needs it.  An octree whose node and attribute pools
 * together exceed the budget is registered as by
 * svo_server_add_octree_paged with a quarter of the budget as its region.
 * A request whose octree cannot be made resident even with every idle
 * octree evicted (paged regions hold the space) ends with SVO_ERR_RANGE. */
int svo_server_add_octree(svo_server* s, const svo_scene* scene, int32_t stack_size, uint32_t* id);
/* Registers an octree served by treelet paging: it holds `region_bytes` of
 * the pool (node and attribute halves: region_bytes / (2 * treelet_bytes)
 * slots, at least 2, at most one per treelet) for the server's life, starting
 * with its root treelet alone, and a worker thread of its own serves its
 * requests in arrival order.  Per request the worker runs analysis passes
 * over the request's view at full resolution (svo_mm_analysis_step: the
 * treelets it sees paged in, invisible ones evicted) until a pass places no
 * new treelet, at most 48 passes, then casts the frame; when the treelets
 * the view needs fit the region, the image is the fully resident octree's.
 * The reference's out-of-core loop (src/TreeletMemoryManager.cpp:393-548,
 * src/RenderPassAnalyse.cpp:218-356) applied per request.  SVO_ERR_BUSY if
 * the pool cannot give the region now. */
int svo_server_add_octree_paged(svo_server* s, const svo_scene* scene, int32_t stack_size,
                                uint64_t region_bytes, uint32_t* id);
/* How octree `octree` reaches the device pool (SVO_UPLOAD_*).
 * SVO_UPLOAD_PINNED page-locks its host copy once, here, so that every
 * later load is two DMA copies at PCIe speed issued without host copying
 * (default: staged through a pinned ring, bound by the host memcpy). */
int svo_server_set_upload_policy(svo_server* s, uint32_t octree, int32_t policy);
int svo_server_submit(svo_server* s, const svo_request* req, uint64_t* ticket);
/* Bounded wait: SVO_ERR_TIMEOUT after timeout_ms. */
int svo_server_wait(svo_server* s, uint64_t ticket, uint32_t timeout_ms, svo_request_result* out);
/* SVO_ERR_BUSY while the request is pending or running. */
int svo_server_poll(svo_server* s, uint64_t ticket, svo_request_result* out);
/* Cancels a request not yet launched (SVO_ERR_BUSY if it is running). */
int svo_server_cancel(svo_server* s, uint64_t ticket);
/* Forgets a finished request's record. */
int svo_server_release(svo_server* s, uint64_t ticket);
int svo_server_stats_get(svo_server* s, svo_server_stats* out);
/* Load generator: submits reqs[i] at arrival_s[i] seconds after the call,
 * then waits (each wait bounded by timeout_ms) and fills results[i]. */
int svo_server_replay(svo_server* s, const svo_request* reqs, const double* arrival_s, uint32_t n,
                      uint32_t timeout_ms, svo_request_result* results);

/* ---- misc -------------------------------------------------------------- */
const char* svo_version(void);
/* Last CUDA error string seen by the library on this thread ("" if none). */
const char* svo_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* LIBSVO_B200_H */
