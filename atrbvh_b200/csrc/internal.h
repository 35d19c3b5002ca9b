// Internal definitions shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/atrbvh.h"

namespace atr {

void set_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define ATR_CUDA(call)                                                             \
    do {                                                                           \
        cudaError_t _e = (call);                                                   \
        if (_e != cudaSuccess) return ::atr::cuda_fail(_e, #call, __FILE__, __LINE__); \
    } while (0)

#define ATR_REQUIRE(cond, code, ...)           \
    do {                                       \
        if (!(cond)) {                         \
            ::atr::set_error(__VA_ARGS__);     \
            return (code);                     \
        }                                      \
    } while (0)

#define ATR_TRY(expr)                 \
    do {                              \
        int _s = (expr);              \
        if (_s != ATR_OK) return _s;  \
    } while (0)

// Device-side error bits (ORed into atr_ctx::d_error by kernels whose bounded
// waits give up).
enum : uint32_t {
    kErrSortLookback = 1u,
    kErrBuildClimb = 2u,
    kErrTreeletClimb = 4u,
    kErrTraceStack = 8u,
    kErrCollapse = 16u,
    kErrLevelList = 32u,  // a level list would overflow its capacity (entries dropped)
};

constexpr int kNumSms = 148;  // B200

// Round up to a multiple of 256 bytes (alignment of every sub-array).
inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// What the LBVH build's climb leaves for the first ATRBVH iteration: the
// optimiser's per-node record (node-indexed in the batch layout) -- subtree
// triangle count, nodesSah under the reference's default constants, the
// next iteration's nodesSah (the same value below `gamma` triangles, where the
// node is not a treelet root; 0 otherwise, until the optimiser writes it) and
// the node's level among the nodes of at least `gamma` triangles (0 below
// gamma, else 1 + the larger level of its children; gamma per mesh when
// seg_gamma is set).
struct BuildPrepass {
    int4* rec = nullptr;
    int gamma = 0;
    const uint8_t* seg_gamma = nullptr;  // per-mesh gamma (device), in place of gamma when set
};
// Primitive boxes of a triangle-splitting build (BVHRT-Core/src/LBVH.cu:99-161,
// 320-428, 572-669): one box per primitive (a triangle or a fragment of one)
// and the triangle it belongs to.  When bmin is set the LBVH build takes
// Morton codes from the boxes' centroids, leaf boxes from the boxes and leaf
// data indices from `data`, in place of the triangles' vertices.
struct PrimBoxes {
    const float4* bmin = nullptr;
    const float4* bmax = nullptr;
    const uint32_t* data = nullptr;
};

constexpr float kPrepassCi = 1.2f;  // AgglomerativeTreelet.h:75 defaults
constexpr float kPrepassCt = 1.0f;
constexpr int kPrepassGamma = 9;    // AgglomerativeTreeletOptimizer.h:24 default treelet size

}  // namespace atr

struct atr_ctx {
    int device = 0;
    int num_sms = atr::kNumSms;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    uint32_t* d_error = nullptr;  // device error bits
    uint64_t launches = 0;        // kernels enqueued by this context
    bool timing = false;
    // Launch tuning (atr_ctx_set_tuning): ATRBVH warps per block (2, 4, 8);
    // fewest simultaneous treelet roots in a warp that are restructured in
    // lane groups (33: never; a single root always takes the whole warp).
    int atr_warps = 8;
    int atr_group_min = 2;
    // Radix sort digit width of LBVH builds: 8 (4 passes for 30-bit codes)
    // or 10 (3 passes).
    int sort_bits = 8;
    // ATRBVH levels restructured by the level passes (one thread per
    // treelet) before the dataflow pass takes the rest; 0 = dataflow only.
    int atr_levels = 12;
    // A level pass over at least this many treelet roots restructures them in
    // four-lane groups (eight per warp); -1 = never.
    int atr_quad_min = 20000;
    int atr_warp_max = 4096;
    struct Phase {
        std::string name;
        cudaEvent_t a, b;
    };
    std::vector<Phase> phases;
    // While a build plan captures its graph: phase marks become external
    // record nodes, so each replay records them again.
    bool capture_marks = false;
    std::vector<float> phase_ms;
    std::string phase_names;  // comma-separated names of the last atr_ctx_phase_times

    // Stream-ordered allocation from this context's own pool.  A pool per
    // context keeps contexts that run side by side on one device from
    // waiting on each other: a pool shared by several streams may make an
    // allocation on one stream wait for a free enqueued on another.
    cudaMemPool_t pool = nullptr;
    int alloc(void** p, size_t bytes);
    void release(void* p);
    // Phase timing helpers (no-ops unless timing is enabled).
    void phase_begin(const char* name);
    void phase_end();
};

struct atr_scene {
    atr_ctx* ctx = nullptr;
    uint32_t n = 0;
    float4* verts = nullptr;  // 3 per triangle
    float* d_bounds = nullptr;  // min.xyz, max.xyz on the device
};

namespace atr {
// Plan of the refit of one topology (refit.cu): per level, CTA slot offsets,
// the inputs (source and node, parent slot) and the internal nodes (node,
// parent slot, child slots) in CTA-local slot order.
struct RefitPlan {
    static constexpr int kMaxLevels = 8;
    struct Level {
        uint32_t ctas = 0, inputs = 0, internal = 0;
        uint32_t *cta_in = nullptr, *cta_int = nullptr;
        int32_t *in_src = nullptr, *in_node = nullptr, *it_node = nullptr;
        uint16_t *in_par = nullptr, *it_par = nullptr;
        uint32_t* it_kids = nullptr;
    };
    int levels = 0;
    Level lv[kMaxLevels];
    std::vector<void*> blocks;  // device allocations of the levels
};
}  // namespace atr

struct atr_tree {
    atr_ctx* ctx = nullptr;
    uint32_t n = 0;
    void* block = nullptr;
    int32_t *parent = nullptr, *left = nullptr, *right = nullptr, *data = nullptr;
    float4 *bmin = nullptr, *bmax = nullptr;
    float* area = nullptr;
    // Leaf ranges of the internal nodes, valid while `karras` (the topology is
    // the LBVH build's own; optimisers clear it).
    int2* range = nullptr;
    bool karras = false;
    // Prepass arrays of the last LBVH build for the first ATRBVH iteration
    // (released by the first optimiser or refit that makes them stale).
    void* prepass_block = nullptr;
    atr::BuildPrepass prepass{};
    // Sort output kept from the build (keys as stored: uint32 or uint64).
    void* sorted_keys = nullptr;
    uint32_t* sorted_idx = nullptr;
    int morton_bits = 30;
    // Refit plan of the current topology (built by the second refit of the
    // topology -- a topology refit once never pays for a plan; released
    // whenever the topology changes).  no_refit_plan: the topology has no
    // plan (too deep a top); refits climb instead.
    atr::RefitPlan* refit_plan = nullptr;
    bool no_refit_plan = false;
    int refits = 0;  // refits of the current topology
    // Leaves are primitive boxes of a triangle-splitting build (a refit from
    // whole triangles would not reproduce them).
    bool split = false;
};

struct atr_collapsed {
    atr_ctx* ctx = nullptr;
    uint32_t n = 0;
    // Collapsed from a triangle-splitting build: n counts primitives, and the
    // data indices name triangles of the scene the primitives were split from.
    bool split = false;
    void* block = nullptr;
    int32_t *parent = nullptr, *left = nullptr, *right = nullptr, *data = nullptr, *count = nullptr;
    float4 *bmin = nullptr, *bmax = nullptr;
    int32_t* tri_indices = nullptr;
};

struct atr_compact {
    atr_ctx* ctx = nullptr;
    int64_t num_nodes = 0;
    int64_t num_woop = 0;
    int32_t max_depth = 0;
    int4* nodes = nullptr;
    float4* woop = nullptr;
    int32_t* tri_index = nullptr;
};

namespace atr {

struct Segs;       // common.cuh: meshes of a batch laid end to end
struct TreeRefs;   // treelet.cuh

// Output arrays of a (possibly batched) tree in the reference SoA layout.
struct TreeOut {
    int32_t *parent, *left, *right, *data;
    float4 *bmin, *bmax;
    float* area;
    // Leaf range (first, last sorted leaf, local) of every internal node of a
    // freshly built radix tree; written by the LBVH build when not NULL.
    int2* range = nullptr;
};

// Collapsed-tree arrays (possibly batched: per-mesh node slices, per-mesh
// triangle-list slices).
struct CollapsedOut {
    int32_t *parent, *left, *right, *data, *count;
    float4 *bmin, *bmax;
    int32_t* tri_indices;
};

// Allocate the SoA arrays of a tree with n triangles in one block.
int tree_alloc(atr_ctx* ctx, uint32_t n, atr_tree** out);
int collapse_segs(atr_ctx* ctx, const Segs& segs, size_t total_nodes, const TreeOut& src,
                  const CollapsedOut& dst, float ci, float ct, int max_leaf, float* d_sah_parts);
int flatten_segs(atr_ctx* ctx, const Segs& segs, const CollapsedOut& c, const float4* verts, int4* nodes,
                 float4* woop, int32_t* tri_index, int64_t* d_sizes);
struct RayMeshMap;  // trace.cu
int trace_run(atr_ctx* ctx, const int4* nodes, const float4* woop, const int32_t* tri, const RayMeshMap& map,
              int max_depth, const float4* rays, int64_t n, int any_hit, int4* res);
int trace_batch(atr_ctx* ctx, const int4* nodes, const float4* woop, const int32_t* tri, const uint32_t* ray_off,
                const uint32_t* group_mesh, const uint32_t* tri_off, uint32_t groups, int max_depth,
                const float4* rays, int64_t n, int any_hit, int4* res);
// Bottom-up box refit of one tree (local indices) from vertices of its mesh.
int refit_arrays(atr_ctx* ctx, uint32_t n, const TreeOut& t, const float4* verts);
// Refit plans (refit.cu): build for a topology (ATR_ERR_UNSUPPORTED: the
// topology has no plan), run, free.  tree_topology_changed drops a tree's plan.
int refit_plan_build(atr_ctx* ctx, uint32_t n, const TreeOut& t, RefitPlan** out);
int refit_plan_run(atr_ctx* ctx, const RefitPlan& p, const TreeOut& t, const float4* verts);
void refit_plan_free(atr_ctx* ctx, RefitPlan* p);
void tree_topology_changed(atr_tree* t);
// atr_batch_refit_mesh that also returns the mesh's collapsed-tree SAH
// (h_sah may be NULL).
int batch_refit_mesh(atr_ctx* ctx, atr_batch* b, uint32_t mesh, const float* vertices, int on_device,
                     float* h_sah);

// Collapsed-tree arrays for n triangles in one block, and the single-mesh
// collapse into them (d_sah_parts, may be NULL: cost and area of the root).
int collapsed_alloc(atr_ctx* ctx, uint32_t n, atr_collapsed** out);
int collapsed_alloc_sharing(atr_ctx* ctx, const atr_tree* tree, atr_collapsed** out);
int zero_words_async(atr_ctx* ctx, uint32_t* p, size_t words);
int collapse_into(atr_ctx* ctx, const atr_tree* tree, float ci, float ct, int max_leaf, atr_collapsed* c,
                  float* d_sah_parts);

// Single-mesh LBVH into an allocated tree (keeps the sort output).
int lbvh_build_into(atr_ctx* ctx, const float4* verts, uint32_t n, const float* d_bounds,
                    int morton_bits, atr_tree* t, const PrimBoxes* prims = nullptr);
// LBVH of every mesh of segs (tiles = sort tiles over all meshes); bounds
// holds 6 floats per mesh.  keep_keys/keep_idx (may be NULL) receive the
// sorted keys and global triangle order.
int lbvh_build_segs(atr_ctx* ctx, const Segs& segs, uint32_t tiles, const float4* verts,
                    const float* d_bounds, int morton_bits, const TreeOut& out, void** keep_keys,
                    uint32_t** keep_idx, const BuildPrepass* prepass = nullptr,
                    const PrimBoxes* prims = nullptr);
// Allocate the prepass record for total_nodes nodes (*block receives the
// allocation).
int prepass_alloc(atr_ctx* ctx, size_t total_nodes, void** block, BuildPrepass* pp);

int atrbvh_run(atr_ctx* ctx, const TreeRefs& g, const Segs& segs, size_t total_nodes, int tsize,
               int max_tsize, int iterations, const uint8_t* seg_tsize, const uint8_t* seg_iters, float ci,
               float ct, const int2* karras_ranges = nullptr, const BuildPrepass* prepass = nullptr);
int atrbvh_group_width(int max_tsize);
int atrbvh_prepare();  // kernel attributes; once per context
int trbvh_run(atr_ctx* ctx, const TreeRefs& g, const Segs& segs, size_t total_nodes, int iterations,
              const uint8_t* seg_iters, float ci, float ct);

constexpr uint32_t kSortTileSize = 3072;  // triangles per sort tile (lbvh.cu)
int lbvh_prepare();                       // kernel attributes; once per context

}  // namespace atr
