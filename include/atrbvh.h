/*
 * atrbvh.h -- C ABI of the B200 ATRBVH build-and-traverse library.
 *
 * Every entry point returns an int status (ATR_OK = 0); atr_last_error()
 * gives a message for the calling thread.  Nothing calls exit().  All device
 * work is enqueued on the context's CUDA stream; functions that return host
 * data synchronise that stream.  Plain pointers and sizes only: vertices are
 * three float4 per triangle (x, y, z, w; w ignored), node boxes are float4.
 *
 * Each declaration names the reference interface it replaces
 * (leonardo-domingues/atrbvh, paths relative to the project root).
 */
#ifndef ATRBVH_H
#define ATRBVH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum atr_status {
    ATR_OK = 0,
    ATR_ERR_INVALID_ARG = 1,  /* bad size, pointer or parameter */
    ATR_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    ATR_ERR_OOM = 3,          /* device allocation failed */
    ATR_ERR_UNSUPPORTED = 4,  /* parameter outside the supported range */
    ATR_ERR_DEVICE_WAIT = 5,  /* a bounded device-side wait gave up */
    ATR_ERR_NO_DEVICE = 6,    /* no CUDA device / wrong architecture */
    ATR_ERR_NOT_RESIDENT = 7  /* server refit of a mesh id it does not hold */
};

enum atr_scene_kind { ATR_SCENE_UNIFORM = 0, ATR_SCENE_CLUSTERED = 1 };

typedef struct atr_ctx atr_ctx;
typedef struct atr_scene atr_scene;
typedef struct atr_tree atr_tree;
typedef struct atr_collapsed atr_collapsed;
typedef struct atr_compact atr_compact;
typedef struct atr_batch atr_batch;
typedef struct atr_plan atr_plan;

/* Device-resident tree in the reference's structure-of-arrays layout
 * (BVHRT-Core/src/SoABVHTree.h:21-34): 2N-1 nodes, internal nodes [0, N-2],
 * leaves [N-1, 2N-2], root 0.  Leaves have left = right = -1 and data = the
 * triangle index; internal nodes have data = -1; the root's parent is -1. */
typedef struct atr_tree_view {
    uint32_t num_triangles;
    int32_t root;
    int32_t* parent;
    int32_t* left;
    int32_t* right;
    int32_t* data;
    float* bbox_min; /* float4 per node */
    float* bbox_max; /* float4 per node */
    float* area;
} atr_tree_view;

/* Collapsed tree (BVHRT-Core/src/BVHCollapsedTree.h:9-58).  A node with
 * data >= 0 is a leaf: with triangle_count > 1, data is the offset of its
 * triangle list in triangle_indices; otherwise data is the triangle index. */
typedef struct atr_collapsed_view {
    uint32_t num_triangles;
    int32_t root;
    int32_t* parent;
    int32_t* left;
    int32_t* right;
    int32_t* data;
    int32_t* triangle_count;
    float* bbox_min;
    float* bbox_max;
    int32_t* triangle_indices; /* num_triangles entries */
} atr_collapsed_view;

/* Compact2 traversal layout (gpu-ray-traversal/src/rt/cuda/CudaBVH.hpp:41-55):
 * 64-byte nodes of child boxes (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y),
 * (c1 ...), (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z), (child0, child1, 0, 0) where
 * an inner child is its float4 offset and a leaf child is ~(float4 offset of
 * its first Woop triangle); three float4 per Woop triangle and a float4 of
 * 0x80000000 after each leaf; tri_index holds the triangle id at each
 * triangle's first float4. */
typedef struct atr_compact_view {
    int64_t num_nodes;
    int64_t num_woop;
    int32_t* nodes;     /* 16 int32 per node */
    float* woop;        /* 4 floats per entry */
    int32_t* tri_index; /* one per Woop float4 entry */
    int32_t max_depth;  /* deepest inner-node level (root = 1) */
} atr_compact_view;

/* ---- errors, version ------------------------------------------------- */
const char* atr_last_error(void);
const char* atr_version(void);

/* ---- context: one per host thread; owns a stream and scratch ---------
 * Replaces the reference's implicit legacy default stream
 * (BVHRT-Core/src/TimeKernelExecution.h:14-32) and checkCudaError/exit
 * (BVHRT-Core/src/CudaErrorCheck.h:12-23).  stream may be NULL (a new stream
 * is created) or a cudaStream_t the caller keeps ownership of. */
int atr_ctx_create(int device, void* stream, atr_ctx** out);
int atr_ctx_destroy(atr_ctx* ctx);
int atr_ctx_synchronize(atr_ctx* ctx); /* also reports device-side errors */
int atr_ctx_get_stream(atr_ctx* ctx, void** stream);
/* Launch tuning of this context's kernels (no counterpart in the reference,
 * whose launch shapes are fixed: AgglomerativeTreelet.cu:556-595).  Results
 * do not depend on the tuning; only speed does.
 *   ATR_TUNE_ATR_WARPS      ATRBVH warps per block: 2, 4 or 8 (default).
 *   ATR_TUNE_ATR_GROUP_MIN  fewest treelet roots reached by one warp at once
 *                           that are restructured side by side in lane groups
 *                           (2..32; 33 = never; default 2).
 *   ATR_TUNE_SORT_BITS      radix-sort digit width of LBVH builds: 8 (default;
 *                           4 passes over 30-bit codes, 8 over 63-bit) or 10
 *                           (3 and 7 passes).
 *   ATR_TUNE_ATR_LEVELS     ATRBVH levels of treelet roots restructured level
 *                           by level in lane groups (0..64; default 12; 0 =
 *                           all by the bottom-up warp pass).
 *   ATR_TUNE_QUAD_MIN       fewest treelet roots of one level that the level
 *                           pass restructures in four-lane groups, eight per
 *                           warp, instead of 32/G per warp (-1 = never;
 *                           default 20000).
 *   ATR_TUNE_WARP_MAX       most treelet roots of one level that the level
 *                           pass restructures one per warp, with the
 *                           treelet's slots and distances in registers
 *                           (treelets of at most 11 leaves; 0 = never;
 *                           default 4096). */
enum atr_tune_knob {
    ATR_TUNE_ATR_WARPS = 0,
    ATR_TUNE_ATR_GROUP_MIN = 1,
    ATR_TUNE_SORT_BITS = 2,
    ATR_TUNE_ATR_LEVELS = 3,
    ATR_TUNE_QUAD_MIN = 4,
    ATR_TUNE_WARP_MAX = 5
};
int atr_ctx_set_tuning(atr_ctx* ctx, int knob, int value);
int atr_ctx_get_tuning(atr_ctx* ctx, int knob, int* value);
/* Number of kernels this context has enqueued since it was created. */
int atr_ctx_launch_count(atr_ctx* ctx, uint64_t* count);
/* Per-phase CUDA-event timing of the next builds (milliseconds). */
int atr_ctx_set_timing(atr_ctx* ctx, int enable);
int atr_ctx_phase_times(atr_ctx* ctx, float* ms, int capacity, int* count);
/* Comma-separated phase names matching the last atr_ctx_phase_times call. */
const char* atr_ctx_phase_names(atr_ctx* ctx);

/* ---- scene -------------------------------------------------------------
 * Replaces BVHRT::SceneWrapper(numberOfTriangles, float4* vertices, float3
 * bbMin, float3 bbMax) (BVHRT-Core/src/SceneWrapper.h:25-26; H2D upload at
 * SceneWrapper.cpp:24-29).  bbox_min/bbox_max (3 floats each) may be NULL: the
 * scene box is then reduced on the device, seeding the maximum with the
 * smallest positive normal float as gpu-ray-traversal/src/rt/SceneConverter.cpp:31-34
 * does.  vertices_on_device != 0: vertices is a device pointer that is copied. */
int atr_scene_create(atr_ctx* ctx, const float* vertices, uint32_t num_triangles,
                     const float* bbox_min, const float* bbox_max, int vertices_on_device,
                     atr_scene** out);
int atr_scene_destroy(atr_scene* scene);
int atr_scene_bounds(atr_ctx* ctx, const atr_scene* scene, float* bbox_min, float* bbox_max);
int atr_scene_device_vertices(const atr_scene* scene, float** vertices, uint32_t* num_triangles);
/* Replace the vertex positions (same triangle count) for a refit. */
int atr_scene_set_vertices(atr_ctx* ctx, atr_scene* scene, const float* vertices,
                           int vertices_on_device);

/* ---- LBVH ----------------------------------------------------------------
 * Replaces BVHRT::LBVHBuilder::BuildTree(const SceneWrapper*)
 * (BVHRT-Core/src/LBVHBuilder.h:31, LBVHBuilder.cpp:21-130).  morton_bits is
 * 30 (LBVHBuilder(false)) or 63 (LBVHBuilder(true)). */
int atr_build_lbvh(atr_ctx* ctx, const atr_scene* scene, int morton_bits, atr_tree** out);
/* The triangle-splitting LBVH: the reference's primitive-box path
 * (BVHRT-Core/src/LBVH.h:36-68 generateMortonCodes(64)TSKernel, :96-124
 * buildTreeTSKernel, :140-155 calculateNodeBoundingBoxesTSKernel; LBVH.cu:
 * 99-161, 320-428, 572-669), which no builder of the reference calls.  One
 * leaf per primitive: Morton codes from the primitive boxes' centroids
 * normalised to the scene box, leaf boxes from the primitive boxes, leaf data
 * indices from data_indices (the triangle each primitive belongs to; several
 * leaves may name one triangle).  prim_bmin / prim_bmax: num_primitives
 * float4 each and data_indices: device pointers; scene_bmin / scene_bmax:
 * 3 host floats.  The tree then optimises, collapses and flattens (with the
 * scene of the triangles) as any other; atr_refit rejects it
 * (ATR_ERR_UNSUPPORTED), since its leaves are not whole triangles. */
int atr_build_lbvh_split(atr_ctx* ctx, uint32_t num_primitives, const float* prim_bmin,
                         const float* prim_bmax, const uint32_t* data_indices,
                         const float* scene_bmin, const float* scene_bmax, int morton_bits,
                         atr_tree** out);
/* Triangle splitting for atr_build_lbvh_split (no counterpart in the
 * reference, which has the primitive-box build but no step that makes the
 * boxes).  Up to split_ratio * n extra primitives (at most max_primitives in
 * all, at most 8 per triangle) are shared out by how much box surface each
 * triangle wastes; each split triangle is bisected at the middle of the
 * longest axis of its largest fragment, and every fragment gets the tight
 * box of the triangle clipped to its region.  Writes the fragments' boxes
 * (float4, w = 0) and triangle indices to the device buffers (room for
 * max_primitives), fragments of one triangle together in triangle order,
 * and their count to *num_primitives (host; synchronises the context). */
int atr_split_triangles(atr_ctx* ctx, const atr_scene* scene, float split_ratio,
                        uint32_t max_primitives, float* prim_bmin, float* prim_bmax,
                        uint32_t* data_indices, uint32_t* num_primitives);
int atr_tree_destroy(atr_tree* tree);
/* BVHTreeInstanceManager::FreeDeviceTree (BVHTreeInstanceManager.h:67). */
int atr_tree_view_get(const atr_tree* tree, atr_tree_view* view);
/* BVHTreeInstanceManager::DeviceToHostTree (BVHTreeInstanceManager.h:57):
 * copies the arrays to host buffers (2N-1 entries; float4 per node box);
 * any pointer may be NULL. */
int atr_tree_download(atr_ctx* ctx, const atr_tree* tree, int32_t* parent, int32_t* left,
                      int32_t* right, int32_t* data, float* bbox_min, float* bbox_max,
                      float* area);
/* SoABVHTree::SAH (BVHRT-Core/src/SoABVHTree.cpp:50-74): the reference's
 * sequential float sum over the areas, evaluated on the host after a copy. */
int atr_tree_sah(atr_ctx* ctx, const atr_tree* tree, float ci, float ct, float* sah);
/* Sorted Morton keys (as uint64) and triangle order kept from the last build
 * of this tree (the reference's sort output, CubWrapper.cu:37). */
int atr_tree_sorted_keys(atr_ctx* ctx, const atr_tree* tree, uint64_t* keys, uint32_t* indices);

/* ---- low-level device entry points (LBVH.h:20-155, CubWrapper.h:18-34) ----
 * Device pointers; keys are uint32 (bits 30) or uint64 (bits 63). */
int atr_device_morton(atr_ctx* ctx, const float* vertices, uint32_t num_triangles,
                      const float* bbox_min, const float* bbox_max, int morton_bits,
                      void* keys);
int atr_device_sort_pairs(atr_ctx* ctx, void* keys, uint32_t* values, uint32_t count,
                          int key_bits);

/* ---- optimisers ------------------------------------------------------------
 * AgglomerativeTreeletOptimizer(treeletSize, iterations)::Optimize
 * (BVHRT-Core/src/AgglomerativeTreeletOptimizer.h:24, .cpp:24-110); treelet
 * sizes 3..20 (the reference's shared-memory kernel range). */
int atr_optimize_atrbvh(atr_ctx* ctx, atr_tree* tree, int treelet_size, int iterations,
                        float ci, float ct);
/* TRBVHOptimizer(treeletSize, iterations)::Optimize
 * (BVHRT-Core/src/TRBVHOptimizer.h:27, .cpp:21-128); treelet size 7. */
int atr_optimize_trbvh(atr_ctx* ctx, atr_tree* tree, int treelet_size, int iterations,
                       float ci, float ct);
/* Bottom-up box refit of an existing topology from the scene's current
 * vertices (the refit pass of BVHRT-Core/src/LBVH.cu:465-570 on a resident tree). */
int atr_refit(atr_ctx* ctx, atr_tree* tree, const atr_scene* scene);

/* Refit that allocates no device memory.  No counterpart in the reference.
 * For callers that cannot allocate when they refit -- a frame or serving
 * loop running under a fixed, pre-reserved memory budget, or code that may
 * only enqueue work on a stream it was given.  The caller passes the tree's
 * device arrays (atr_tree_view_get, or its own copies) and the mesh's device
 * vertices; the per-node counters live in a fixed __device__ array inside the
 * library: at most 1,048,576 triangles (larger meshes are rejected; use
 * atr_refit), one array per device for the life of the process, shared by all
 * calls -- calls that overlap on the GPU race, so order them on one stream.
 * Each call made outside stream capture looks up the array's address afresh
 * (so a device reset cannot leave a stale one); a call inside a capture uses
 * the address of the last uncaptured call on that device, so make one
 * uncaptured call on a device, and again after a reset, before capturing.
 * stream may be NULL (legacy default stream). */
int atr_refit_noalloc(void* stream, uint32_t num_triangles, const float* vertices,
                      const int32_t* parent, const int32_t* left, const int32_t* right,
                      const int32_t* data, float* bbox_min, float* bbox_max, float* area);

/* ---- collapse ----------------------------------------------------------------
 * BVHTreeCollapser::Collapse(BVHTree*, float* sah, ci, ct)
 * (BVHRT-Core/src/BVHTreeCollapser.h:39, .cpp:21-93).  max_leaf = 0 reproduces
 * the reference (no leaf-size limit); max_leaf > 0 also forbids collapsing
 * subtrees with more triangles.  sah receives cost[root] / area[root]. */
int atr_collapse(atr_ctx* ctx, const atr_tree* tree, float ci, float ct, int max_leaf,
                 atr_collapsed** out, float* sah);
int atr_collapsed_destroy(atr_collapsed* collapsed);
int atr_collapsed_view_get(const atr_collapsed* collapsed, atr_collapsed_view* view);
/* BVHTreeInstanceManager::DeviceToHostCollapsedTree (BVHTreeInstanceManager.h:113). */
int atr_collapsed_download(atr_ctx* ctx, const atr_collapsed* collapsed, int32_t* parent,
                           int32_t* left, int32_t* right, int32_t* data,
                           int32_t* triangle_count, float* bbox_min, float* bbox_max,
                           int32_t* triangle_indices);

/* ---- traversal layout + closest-hit traversal ------------------------------
 * CudaBVH(const BVHCollapsedTree*, Scene*, BVHLayout_Compact2)
 * (gpu-ray-traversal/src/rt/cuda/CudaBVH.cpp:60-79, createCompact :469-574,
 * woopifyTri :579-600), built on the device. */
int atr_flatten_compact2(atr_ctx* ctx, const atr_collapsed* collapsed, const atr_scene* scene,
                         atr_compact** out);
int atr_compact_destroy(atr_compact* compact);
int atr_compact_view_get(const atr_compact* compact, atr_compact_view* view);
/* Host copies of CudaBVH's m_nodes / m_triWoop / m_triIndex buffers
 * (gpu-ray-traversal/src/rt/cuda/CudaBVH.cpp:566-573); sizes from the view. */
int atr_compact_download(atr_ctx* ctx, const atr_compact* compact, int32_t* nodes, float* woop,
                         int32_t* tri_index);
/* The trace() kernel ABI (gpu-ray-traversal/src/rt/kernels/CudaTracerKernels.hpp:73-86,
 * kepler_dynamic_fetch.cu:61-320): rays are float4 (origin, tmin), float4
 * (direction, tmax) on the device; results are int4 (triangle id or -1,
 * float bits of t, 0, 0) on the device. */
int atr_trace(atr_ctx* ctx, const atr_compact* compact, const float* rays, int64_t num_rays,
              int any_hit, int32_t* results);

/* ---- build plans: the steady-state single-mesh build as one CUDA graph -----
 * The sequence Renderer::getCudaBVH runs per rebuild -- LBVHBuilder::BuildTree,
 * an optimiser, BVHTreeCollapser::Collapse (BVHRT-Core/src/LBVHBuilder.cpp:60-97,
 * AgglomerativeTreeletOptimizer.cpp:75-92, BVHTreeCollapser.cpp:21-93) and,
 * with flatten, CudaBVH's Compact2 conversion -- into outputs the plan owns
 * for one scene.  atr_plan_run enqueues the whole build; with use_graph the
 * first run captures it into a CUDA graph and later runs replay it with one
 * launch (captured again when the context's launch tuning changes).  A run
 * reads the scene's current vertices and bounds, so a plan also rebuilds a
 * deforming mesh.  The results are read through atr_plan_tree /
 * atr_plan_collapsed / atr_plan_compact (the last reads the layout sizes and
 * synchronises) and atr_plan_sah; atr_plan_times gives the device time of the
 * last run's build (Morton through collapse) and flatten; atr_plan_phase_times
 * the per-phase device times of the last replay when the graph was captured
 * with the context's phase timing on (atr_ctx_set_timing; the graph is captured
 * again when that setting changes), else none.  The plan's
 * collapsed tree shares the plan's tree's links and boxes (parent, left,
 * right, bmin, bmax; a collapse leaves them unchanged) and owns its data,
 * counts and leaf lists: both are read-only views, rewritten by each run. */
typedef struct atr_plan_params {
    int32_t morton_bits;   /* 30 or 63 */
    int32_t optimizer;     /* 0 none, 1 ATRBVH, 2 TRBVH */
    int32_t treelet_size;
    int32_t iterations;
    float ci, ct;
    int32_t max_leaf;      /* collapse leaf cap, 0 = uncapped (the reference) */
    int32_t flatten;       /* also build the Compact2 layout */
} atr_plan_params;
int atr_plan_create(atr_ctx* ctx, const atr_scene* scene, const atr_plan_params* params, atr_plan** out);
int atr_plan_run(atr_ctx* ctx, atr_plan* plan, int use_graph);
int atr_plan_tree(const atr_plan* plan, const atr_tree** tree);
int atr_plan_collapsed(const atr_plan* plan, const atr_collapsed** collapsed);
int atr_plan_compact(atr_ctx* ctx, atr_plan* plan, const atr_compact** compact);
int atr_plan_sah(atr_ctx* ctx, atr_plan* plan, float* sah);
int atr_plan_times(atr_ctx* ctx, atr_plan* plan, float* build_ms, float* flatten_ms);
/* Device ms of each phase of the last graph replay (marks recorded inside the
 * graph), and their comma-separated names, as atr_ctx_phase_times does for
 * eager calls. */
int atr_plan_phase_times(atr_ctx* ctx, atr_plan* plan, float* ms, int capacity, int* count);
const char* atr_plan_phase_names(const atr_plan* plan);
int atr_plan_destroy(atr_plan* plan);

/* ---- on-disk cache of the traversal layout ----------------------------------
 * CudaBVH::serialize / CudaBVH(InputStream&)
 * (gpu-ray-traversal/src/rt/cuda/CudaBVH.cpp:108-123; Buffer stream format
 * framework/gpu/Buffer.cpp:331-362): the image is the layout as a
 * little-endian S32 (BVHLayout_Compact2 = 5), then the node, Woop and
 * triangle-index buffers, each a little-endian S64 byte count and the bytes,
 * so files load in either implementation.  atr_compact_serialize with out =
 * NULL only reports the size.  atr_compact_deserialize checks the sizes and
 * every child reference before copying to the device, and recomputes the
 * layout depth from the references.  atr_cache_key stands in for the file name
 * hash of Renderer::getCudaBVH (gpu-ray-traversal/src/rt/cuda/Renderer.cpp:137-141:
 * scene, platform and build-parameter hashes with the layout): a 64-bit hash of
 * the vertex bytes, the layout and every build parameter below. */
typedef struct atr_cache_params {
    int32_t morton_bits;   /* 30 or 63 */
    int32_t optimizer;     /* 0 none, 1 ATRBVH, 2 TRBVH */
    int32_t treelet_size;
    int32_t iterations;
    float ci, ct;          /* collapse costs */
    int32_t max_leaf;      /* collapse leaf cap, 0 = uncapped */
} atr_cache_params;
int atr_compact_serialize(atr_ctx* ctx, const atr_compact* compact, void* out, uint64_t capacity,
                          uint64_t* size);
int atr_compact_deserialize(atr_ctx* ctx, const void* image, uint64_t size, atr_compact** out);
int atr_cache_key(const float* vertices, uint32_t num_triangles, const atr_cache_params* params,
                  uint64_t* key);

/* ---- segmented batch builds (no counterpart in the reference, which builds
 * one mesh per call: LBVHBuilder.cpp:21-130 and the optimisers per mesh) ------
 * Meshes laid end to end: mesh m owns triangles [tri_offsets[m],
 * tri_offsets[m+1]) of `vertices` (host or device), each with >= 2 triangles.
 * bounds (6 floats per mesh: min xyz, max xyz) may be NULL: each mesh's box is
 * then reduced on the device as atr_scene_create does.  One build runs every
 * stage once over all meshes; each mesh's arrays (local indices, from
 * atr_batch_mesh_view) equal those of atr_build_lbvh + optimiser on that mesh
 * alone.  optimizer: 0 none, 1 ATRBVH(treelet_size, iterations), 2 TRBVH(7,
 * iterations).  atr_batch_set_params gives each mesh its own ATRBVH treelet
 * size and iteration count (both arrays, or both NULL to clear).  use_graph
 * captures the build into a CUDA graph on first use and replays it while the
 * parameters stay the same. */
int atr_batch_create(atr_ctx* ctx, const float* vertices, const uint32_t* tri_offsets,
                     uint32_t num_meshes, const float* bounds, int vertices_on_device,
                     atr_batch** out);
int atr_batch_destroy(atr_batch* batch);
int atr_batch_set_params(atr_ctx* ctx, atr_batch* batch, const uint8_t* treelet_sizes,
                         const uint8_t* iterations);
int atr_batch_build(atr_ctx* ctx, atr_batch* batch, int optimizer, int treelet_size, int iterations,
                    float ci, float ct, int use_graph);
int atr_batch_info(const atr_batch* batch, uint32_t* num_meshes, uint32_t* num_triangles,
                   uint64_t* total_nodes);
int atr_batch_mesh_view(const atr_batch* batch, uint32_t mesh, atr_tree_view* view);
int atr_batch_download_mesh(atr_ctx* ctx, const atr_batch* batch, uint32_t mesh, int32_t* parent,
                            int32_t* left, int32_t* right, int32_t* data, float* bbox_min,
                            float* bbox_max, float* area);
/* Per-mesh SoABVHTree::SAH (sequential float sums), num_meshes values. */
int atr_batch_sah(atr_ctx* ctx, const atr_batch* batch, float ci, float ct, float* sah);
/* Collapse every mesh (as atr_collapse per mesh; sah may be NULL, else one
 * value per mesh), then lay every mesh out in Compact2 (as
 * atr_flatten_compact2 per mesh). */
int atr_batch_collapse(atr_ctx* ctx, atr_batch* batch, float ci, float ct, int max_leaf, float* sah);
int atr_batch_flatten(atr_ctx* ctx, atr_batch* batch);
int atr_batch_compact_view(const atr_batch* batch, uint32_t mesh, atr_compact_view* view);
int atr_batch_compact_download(atr_ctx* ctx, const atr_batch* batch, uint32_t mesh, int32_t* nodes,
                               float* woop, int32_t* tri_index);
/* Merged ray queue: rays [ray_offsets[g], ray_offsets[g+1]) trace mesh
 * group_mesh[g] (host arrays, groups entries / groups+1 offsets); rays and
 * results are device arrays as in atr_trace; triangle ids are mesh-local. */
int atr_batch_trace(atr_ctx* ctx, const atr_batch* batch, const float* rays, int64_t num_rays,
                    const uint32_t* ray_offsets, const uint32_t* group_mesh, uint32_t groups,
                    int any_hit, int32_t* results);
/* Replace one mesh's vertices (same count), refit its tree, and (when the
 * batch was flattened) re-collapse and re-flatten that mesh in place. */
int atr_batch_refit_mesh(atr_ctx* ctx, atr_batch* batch, uint32_t mesh, const float* vertices,
                         int vertices_on_device);

/* ---- autotuner (no counterpart in the reference, whose treelet size and
 * iteration count are fixed per run by gpu-ray-traversal/src/rt/BVHRTSettings.cpp:7-84
 * and whose launch shapes are constants, AgglomerativeTreelet.cu:556-595) ------
 * Size class c holds meshes of [2^c, 2^(c+1)) triangles.  For each class in
 * [min_class, max_class] a sample batch of about sample_triangles triangles
 * (the uniform-centroid distribution, each mesh in its own box) is built with
 * ATRBVH(9,2); every ATRBVH(treelet 5..9, iterations 1..3) is then timed and
 * the fastest whose summed per-mesh SAH is at most (1 + sah_tolerance) times
 * that of ATRBVH(9,2) is kept; then the ATRBVH warps per block (2, 4, 8) and
 * sort digit width (8, 10) that build it fastest.  Takes seconds; results are
 * timings of this GPU. */
typedef struct atr_tune_entry {
    uint8_t treelet;
    uint8_t iterations;
    uint8_t atr_warps;
    uint8_t sort_bits;
    float build_ms;          /* median LBVH+ATRBVH time of the class sample, tuned */
    float reference_ms;      /* same with ATRBVH(9,2) at the context's launch shape */
    float sah_ratio;         /* summed SAH of the tuned build / that of ATRBVH(9,2) */
    uint32_t sample_triangles;
    uint32_t sample_meshes;
} atr_tune_entry;

typedef struct atr_tune_table {
    atr_tune_entry cls[32];
    uint32_t tuned_mask;     /* bit c set: class c was tuned */
} atr_tune_table;

typedef struct atr_autotune_config {
    uint32_t min_class, max_class;  /* within [1, 29] */
    uint64_t sample_triangles;      /* per class (at least two meshes are used) */
    float sah_tolerance;            /* 0: SAH no worse than ATRBVH(9,2) */
    uint32_t reps;                  /* timed builds per candidate (median) */
    uint64_t seed;
} atr_autotune_config;

int atr_autotune(atr_ctx* ctx, const atr_autotune_config* config, atr_tune_table* table);
/* Outcome of atr_batch_autotune: the batch's own build time (CUDA-graph
 * replays, median) and summed per-mesh SAH with ATRBVH(9,2) at the context's
 * launch shape and with the tuned table, and whether the table was kept. */
typedef struct atr_tune_outcome {
    float default_ms, tuned_ms;
    double default_sah, tuned_sah;
    int32_t kept;
} atr_tune_outcome;
/* Tunes the size classes present in the batch (atr_autotune on class
 * samples), then times the batch itself both ways and keeps the table only
 * when it builds the batch faster at a summed SAH within the tolerance;
 * otherwise every entry is reset to ATRBVH(9,2) at the context's launch
 * shape.  The batch and the context are left with the kept parameters. */
int atr_batch_autotune(atr_ctx* ctx, atr_batch* batch, const atr_autotune_config* config,
                       atr_tune_table* table, atr_tune_outcome* outcome);
/* The entry for a mesh of num_triangles: its class, or the nearest tuned one. */
int atr_tune_lookup(const atr_tune_table* table, uint32_t num_triangles, atr_tune_entry* entry);
/* Per-mesh treelet size and iterations of a batch from the table
 * (atr_batch_set_params), and the context's ATRBVH warps and sort digit width
 * from the class holding most of the batch's triangles. */
int atr_batch_apply_tuning(atr_ctx* ctx, atr_batch* batch, const atr_tune_table* table);

/* ---- serving loop (no counterpart in the reference, whose Renderer builds
 * and traces one scene at a time: gpu-ray-traversal/src/rt/cuda/Renderer.cpp:85-105,
 * 115-265) ---------------------------------------------------------------------
 * A request builds a mesh (or refits a mesh kept resident by an earlier
 * build) and traces rays against it.  Requests are admitted while their
 * estimated device memory fits the budget beside the resident meshes (idle
 * resident meshes are evicted oldest-use first to make room); each free lane
 * (own stream and thread) takes every admissible waiting request at once,
 * builds the new meshes in one segmented batch, refits the resident ones,
 * traces all their rays in one merged queue and copies the results back, so
 * requests that arrive while other lanes are busy run beside them on the
 * device.  Each result equals that of the same request run alone.  Host
 * buffers of a request must stay valid until atr_server_wait returns it. */
typedef struct atr_server atr_server;

enum { ATR_REQ_BUILD = 0, ATR_REQ_REFIT = 1 };

typedef struct atr_request {
    int kind;               /* ATR_REQ_BUILD or ATR_REQ_REFIT */
    uint64_t mesh_id;       /* build: id to keep the mesh under; refit: resident mesh */
    const float* vertices;  /* host, 3 float4 per triangle; refit: same count as built */
    uint32_t num_triangles; /* build: >= 2; refit: ignored (the resident count is used) */
    const float* rays;      /* host, 2 float4 per ray (origin+tmin, direction+tmax) */
    uint32_t num_rays;
    int32_t* results;       /* host, 4 int32 per ray as atr_trace (mesh-local ids) */
    int keep_resident;      /* build: keep the BVH on the device for refits */
} atr_request;

typedef struct atr_request_result {
    int status;             /* ATR_OK or an error code (message in `error`) */
    float sah;              /* SAH of the collapsed tree (Ci 1.2, Ct 1) */
    double queue_ms;        /* submit -> taken by a lane */
    double latency_ms;      /* submit -> results in host memory */
    uint32_t batch_requests;/* requests in the lane batch that carried it */
    uint32_t lane;
    char error[160];
} atr_request_result;

typedef struct atr_server_config {
    uint64_t hbm_budget_bytes;     /* device memory the server may hold */
    uint32_t lanes;                /* concurrent lane threads/streams (1..8) */
    uint32_t max_batch_requests;   /* requests per lane batch */
    uint64_t max_batch_triangles;  /* triangles per segmented build */
    int treelet_size;              /* ATRBVH treelet size when no size-class table */
    int iterations;                /* ATRBVH iterations when no size-class table */
    int max_leaf;                  /* collapse leaf cap (0: none) */
    const uint8_t* class_treelet;  /* 32 entries by floor(log2(triangles)), or NULL */
    const uint8_t* class_iters;    /* 32 entries, or NULL */
} atr_server_config;

typedef struct atr_server_stats {
    uint64_t completed, failed, builds, refits, evictions;
    uint64_t triangles_built, triangles_refit, rays_traced;
    uint64_t lane_batches;
    uint32_t max_batch_requests_seen;
    uint32_t max_lanes_busy;       /* most lanes that held a batch at once */
    uint32_t resident_meshes;
    uint64_t resident_bytes, peak_bytes;
    double p50_ms, p99_ms, mean_ms, max_ms;
    double overlap_fraction;       /* share of busy time with >= 2 lanes busy */
    double busy_ms;                /* time with >= 1 lane busy */
    double host_copy_ms;           /* lane time in host staging copies (pageable buffers) */
    double lane_batch_ms;          /* lane time from a batch's first copy to its results */
} atr_server_stats;

/* Request buffers (vertices, rays, results) in page-locked host memory
 * (cudaHostAlloc or cudaHostRegister) are copied to and from the device
 * directly; pageable ones go through a lane's pinned staging buffer. */
int atr_server_create(int device, const atr_server_config* config, atr_server** out);
int atr_server_submit(atr_server* server, const atr_request* request, uint64_t* ticket);
/* Blocks until the request is done; each ticket can be waited on once, by one
 * thread (a second concurrent waiter gets ATR_ERR_INVALID_ARG). */
int atr_server_wait(atr_server* server, uint64_t ticket, atr_request_result* result);
/* Drop a resident mesh (its memory is freed once no lane uses it). */
int atr_server_release(atr_server* server, uint64_t mesh_id);
int atr_server_stats_get(atr_server* server, atr_server_stats* stats);
/* Finishes queued work, then frees everything. */
int atr_server_destroy(atr_server* server);

/* One cosine-weighted diffuse bounce ray per primary result (the diffuse
 * workload of gpu-ray-traversal/src/rt/ray/RayGenKernels.cu:114-223 with one
 * sample): device arrays; misses produce rays with tmax = -1. */
int atr_gen_bounce_rays(atr_ctx* ctx, const atr_scene* scene, const float* rays,
                        const int32_t* results, int64_t num_rays, uint64_t seed, float* out_rays);

/* Ambient-occlusion rays, RayGen::ao / rayGenAOKernel
 * (gpu-ray-traversal/src/rt/ray/RayGen.cpp:120-150, RayGenKernels.cu:114-223):
 * num_samples rays per input ray of rays[first, first + count) (device
 * arrays; results as atr_trace writes them), written to out_rays[0,
 * count * num_samples) in input order, sample-minor.  The range is the
 * reference's batching of secondary rays (firstInputSlot / numInputRays):
 * a large primary batch is processed in slices that bound the output.  Misses
 * give rays with tmax = -1.  seed is RayGenAOInput::randomSeed. */
int atr_gen_ao_rays(atr_ctx* ctx, const atr_scene* scene, const float* rays, const int32_t* results,
                    int64_t first, int64_t count, int num_samples, float max_dist, uint32_t seed,
                    float* out_rays);
/* RayBuffer::mortonSort (gpu-ray-traversal/src/rt/ray/RayBuffer.cpp:103-160), on
 * the device: rays sorted by the 192-bit Morton key of origin (in the box of
 * the origins and end points) and direction, into out_rays (must not alias
 * rays); slot_to_id (may be NULL = identity) is carried to out_slot_to_id,
 * and out_id_to_slot is its inverse (either output may be NULL).  Equal keys
 * keep their input order. */
int atr_sort_rays(atr_ctx* ctx, const float* rays, const int32_t* slot_to_id, int64_t num_rays,
                  float* out_rays, int32_t* out_slot_to_id, int32_t* out_id_to_slot);

/* ---- synthetic workloads (host memory; deterministic in seed) ---------- */
int atr_gen_scene(int kind, uint32_t num_triangles, uint64_t seed, float* vertices);
int atr_gen_batch_sizes(uint32_t count, uint32_t min_tris, uint32_t max_tris, uint64_t seed,
                        uint32_t* sizes);
int atr_gen_batch_scene(uint32_t count, const uint32_t* sizes, uint64_t seed, float* vertices);
int atr_gen_rays_pinhole(uint32_t width, uint32_t height, const float* eye, float fov_deg,
                         float* rays);
int atr_gen_rays_random(uint64_t count, uint64_t seed, const float* bbox_min,
                        const float* bbox_max, float* rays);

#ifdef __cplusplus
}
#endif

#endif /* ATRBVH_H */
