// Segmented batch builds: many meshes of uneven sizes built together.
//
// The meshes' triangles are laid end to end; every kernel of the LBVH,
// ATRBVH and TRBVH stages runs once over the whole batch (one launch per
// stage and iteration), with each thread, tile or treelet working inside its
// own mesh: per-mesh scene boxes and Morton normalisation, per-mesh digit
// histograms and tile-prefix scans that restart at each mesh in the sort, per-mesh radix trees
// with local node indices, and treelets formed and rewritten within one
// mesh.  Every mesh's arrays therefore equal those of a build of that mesh
// alone.  Steady-state builds can be captured once into a CUDA graph and
// replayed.

#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "treelet.cuh"

struct atr_batch {
    atr_ctx* ctx = nullptr;
    uint32_t count = 0;
    uint32_t n = 0;
    uint32_t tiles = 0;
    size_t total_nodes = 0;
    std::vector<uint32_t> h_tri_off, h_tile_off;
    void* meta = nullptr;  // d_tri_off, d_tile_off, d_tsize, d_iters, bounds
    uint32_t* d_tri_off = nullptr;
    uint32_t* d_tile_off = nullptr;
    uint8_t* d_tsize = nullptr;
    uint8_t* d_iters = nullptr;
    bool per_mesh_params = false;
    int max_iters = 0;
    int max_tsize = 0;
    float* d_bounds = nullptr;
    float4* verts = nullptr;
    void* block = nullptr;
    atr::TreeOut tree{};
    cudaGraphExec_t graph = nullptr;
    int graph_key[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // build parameters and launch tuning of the graph
    float graph_cf[2] = {0, 0};
    uint64_t graph_launches = 0;
    // Collapsed trees and Compact2 layouts (allocated on first use).
    void* col_block = nullptr;
    atr::CollapsedOut col{};
    void* cp_block = nullptr;
    int4* cp_nodes = nullptr;
    float4* cp_woop = nullptr;
    int32_t* cp_tri = nullptr;
    int64_t* d_sizes = nullptr;  // per mesh: nodes then woop entries
    std::vector<int64_t> h_sizes;
    std::atomic<int32_t> max_depth{0};  // refits of different meshes may raise it from several lanes
    bool flattened = false;
    // Parameters of the last atr_batch_collapse (reused when one mesh is refit).
    float col_ci = 1.2f, col_ct = 1.0f;
    int col_max_leaf = 0;
};

namespace atr {
namespace {

__device__ __forceinline__ uint32_t f2o(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}

// Per-mesh scene box, one block per sort tile; ordered-integer atomics.
__global__ void __launch_bounds__(256) k_seg_bounds(Segs segs, const float4* __restrict__ v,
                                                     uint32_t* __restrict__ enc) {
    const uint32_t m = segs.seg_of_tile(blockIdx.x);
    const uint32_t t0 = segs.tri_begin(m) + (blockIdx.x - segs.tile_begin(m)) * kSortTileSize;
    const uint32_t t1 = min(t0 + kSortTileSize, segs.tri_end(m));
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint64_t k = 3ull * t0 + threadIdx.x; k < 3ull * t1; k += blockDim.x) {
        const float4 p = __ldg(v + k);
        mn[0] = fminf(mn[0], p.x); mn[1] = fminf(mn[1], p.y); mn[2] = fminf(mn[2], p.z);
        mx[0] = fmaxf(mx[0], p.x); mx[1] = fmaxf(mx[1], p.y); mx[2] = fmaxf(mx[2], p.z);
    }
    for (int o = 16; o > 0; o >>= 1)
        for (int k = 0; k < 3; ++k) {
            mn[k] = fminf(mn[k], __shfl_xor_sync(kFull, mn[k], o));
            mx[k] = fmaxf(mx[k], __shfl_xor_sync(kFull, mx[k], o));
        }
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 3; ++k) {
            atomicMin(enc + 6 * m + k, f2o(mn[k]));
            atomicMax(enc + 6 * m + 3 + k, f2o(mx[k]));
        }
}

// Seeds the maximum with the smallest positive normal float, as
// gpu-ray-traversal/src/rt/SceneConverter.cpp:31-34 does.
__global__ void k_seg_bounds_final(uint32_t count, const uint32_t* __restrict__ enc, float* __restrict__ out) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= count) return;
    for (int k = 0; k < 3; ++k) {
        out[6 * m + k] = fminf(FLT_MAX, o2f(enc[6 * m + k]));
        out[6 * m + 3 + k] = fmaxf(FLT_MIN, o2f(enc[6 * m + 3 + k]));
    }
}

__global__ void k_seg_bounds_init(uint32_t count, uint32_t* __restrict__ enc) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= 6 * count) return;
    enc[j] = (j % 6) < 3 ? 0xffffffffu : 0u;
}

int batch_run(atr_ctx* ctx, atr_batch* b, int optimizer, int tsize, int iterations, float ci, float ct) {
    const Segs segs{b->d_tri_off, b->d_tile_off, b->count, b->n};
    // The LBVH climb leaves its prepass for ATRBVH's first iteration.
    void* ppb = nullptr;
    BuildPrepass pp{};
    const bool want_pp = optimizer == 1 && (b->per_mesh_params ? b->max_iters : iterations) > 0 &&
                         ctx->atr_levels > 0 && ci == kPrepassCi && ct == kPrepassCt;
    if (want_pp) {
        ATR_TRY(prepass_alloc(ctx, b->total_nodes, &ppb, &pp));
        if (b->per_mesh_params) pp.seg_gamma = b->d_tsize;  // first iteration: gamma = each mesh's treelet size
        else pp.gamma = tsize;
    }
    int st = lbvh_build_segs(ctx, segs, b->tiles, b->verts, b->d_bounds, 30, b->tree, nullptr, nullptr,
                             want_pp ? &pp : nullptr);
    if (st != ATR_OK) { ctx->release(ppb); return st; }
    TreeRefs g{b->n, b->tree.parent, b->tree.left, b->tree.right, b->tree.bmin, b->tree.bmax, b->tree.area, nullptr};
    const uint8_t* ts = b->per_mesh_params ? b->d_tsize : nullptr;
    const uint8_t* it = b->per_mesh_params ? b->d_iters : nullptr;
    const int iters = b->per_mesh_params ? b->max_iters : iterations;
    if (optimizer == 1) {
        st = atrbvh_run(ctx, g, segs, b->total_nodes, tsize, b->per_mesh_params ? b->max_tsize : tsize, iters, ts, it,
                        ci, ct, b->tree.range, want_pp ? &pp : nullptr);
        ctx->release(ppb);
        return st;
    }
    ctx->release(ppb);
    if (optimizer == 2) return trbvh_run(ctx, g, segs, b->total_nodes, iters, it, ci, ct);
    return ATR_OK;
}

}  // namespace
}  // namespace atr

using namespace atr;

extern "C" {

int atr_batch_create(atr_ctx* ctx, const float* vertices, const uint32_t* tri_offsets, uint32_t count,
                     const float* bounds, int on_device, atr_batch** out) {
    ATR_REQUIRE(ctx && vertices && tri_offsets && out, ATR_ERR_INVALID_ARG, "atr_batch_create: NULL argument");
    ATR_REQUIRE(count >= 1, ATR_ERR_INVALID_ARG, "atr_batch_create: no meshes");
    ATR_REQUIRE(tri_offsets[0] == 0, ATR_ERR_INVALID_ARG, "atr_batch_create: tri_offsets[0] must be 0");
    for (uint32_t m = 0; m < count; ++m)
        ATR_REQUIRE(tri_offsets[m + 1] >= tri_offsets[m] + 2, ATR_ERR_INVALID_ARG,
                    "atr_batch_create: mesh %u has fewer than 2 triangles", m);
    const uint64_t n = tri_offsets[count];
    ATR_REQUIRE(n < (1u << 30), ATR_ERR_INVALID_ARG, "atr_batch_create: %llu triangles >= 2^30",
                (unsigned long long)n);
    *out = nullptr;
    atr_batch* b = new atr_batch();
    b->ctx = ctx;
    b->count = count;
    b->n = (uint32_t)n;
    b->h_tri_off.assign(tri_offsets, tri_offsets + count + 1);
    b->h_tile_off.resize(count + 1);
    b->h_tile_off[0] = 0;
    for (uint32_t m = 0; m < count; ++m)
        b->h_tile_off[m + 1] = b->h_tile_off[m] + (tri_offsets[m + 1] - tri_offsets[m] + kSortTileSize - 1) / kSortTileSize;
    b->tiles = b->h_tile_off[count];
    b->total_nodes = 2 * n - count;
    const size_t off_b = align256((count + 1) * 4ull), par_b = align256(count), bnd_b = align256(24ull * count);
    int st = ctx->alloc(&b->meta, 2 * off_b + 2 * par_b + 2 * bnd_b);
    if (st == ATR_OK) st = ctx->alloc(reinterpret_cast<void**>(&b->verts), n * 48);
    const size_t nn = b->total_nodes, b4 = align256(nn * 4), b16 = align256(nn * 16);
    const size_t b8 = align256((size_t)(n - count) * 8);
    if (st == ATR_OK) st = ctx->alloc(&b->block, 5 * b4 + 2 * b16 + b8);
    if (st != ATR_OK) { atr_batch_destroy(b); return st; }
    char* p = static_cast<char*>(b->meta);
    b->d_tri_off = reinterpret_cast<uint32_t*>(p); p += off_b;
    b->d_tile_off = reinterpret_cast<uint32_t*>(p); p += off_b;
    b->d_tsize = reinterpret_cast<uint8_t*>(p); p += par_b;
    b->d_iters = reinterpret_cast<uint8_t*>(p); p += par_b;
    b->d_bounds = reinterpret_cast<float*>(p); p += bnd_b;
    uint32_t* enc = reinterpret_cast<uint32_t*>(p);
    char* q = static_cast<char*>(b->block);
    b->tree.parent = reinterpret_cast<int32_t*>(q); q += b4;
    b->tree.left = reinterpret_cast<int32_t*>(q); q += b4;
    b->tree.right = reinterpret_cast<int32_t*>(q); q += b4;
    b->tree.data = reinterpret_cast<int32_t*>(q); q += b4;
    b->tree.area = reinterpret_cast<float*>(q); q += b4;
    b->tree.bmin = reinterpret_cast<float4*>(q); q += b16;
    b->tree.bmax = reinterpret_cast<float4*>(q); q += b16;
    b->tree.range = reinterpret_cast<int2*>(q);
    cudaStream_t s = ctx->stream;
    cudaMemcpyAsync(b->d_tri_off, b->h_tri_off.data(), (count + 1) * 4ull, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b->d_tile_off, b->h_tile_off.data(), (count + 1) * 4ull, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b->verts, vertices, n * 48, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s);
    if (bounds) {
        cudaMemcpyAsync(b->d_bounds, bounds, 24ull * count, cudaMemcpyHostToDevice, s);
    } else {
        const Segs segs{b->d_tri_off, b->d_tile_off, count, b->n};
        k_seg_bounds_init<<<(6 * count + 255) / 256, 256, 0, s>>>(count, enc);
        k_seg_bounds<<<b->tiles, 256, 0, s>>>(segs, b->verts, enc);
        k_seg_bounds_final<<<(count + 255) / 256, 256, 0, s>>>(count, enc, b->d_bounds);
        ctx->launches += 3;
    }
    cudaError_t e = cudaStreamSynchronize(s);  // host arrays above are the batch's own; sync for errors
    if (e != cudaSuccess) { atr_batch_destroy(b); return cuda_fail(e, "atr_batch_create", __FILE__, __LINE__); }
    *out = b;
    return ATR_OK;
}

int atr_batch_destroy(atr_batch* b) {
    if (!b) return ATR_OK;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->ctx->release(b->col_block);
    b->ctx->release(b->cp_block);
    b->ctx->release(b->block);
    b->ctx->release(b->verts);
    b->ctx->release(b->meta);
    delete b;
    return ATR_OK;
}

int atr_batch_set_params(atr_ctx* ctx, atr_batch* b, const uint8_t* treelet_sizes, const uint8_t* iterations) {
    ATR_REQUIRE(ctx && b, ATR_ERR_INVALID_ARG, "atr_batch_set_params: NULL argument");
    if (!treelet_sizes && !iterations) {
        b->per_mesh_params = false;
        return ATR_OK;
    }
    ATR_REQUIRE(treelet_sizes && iterations, ATR_ERR_INVALID_ARG, "atr_batch_set_params: give both arrays");
    int mx = 0, mts = 0;
    for (uint32_t m = 0; m < b->count; ++m) {
        ATR_REQUIRE(treelet_sizes[m] >= 3 && treelet_sizes[m] <= 20, ATR_ERR_UNSUPPORTED,
                    "atr_batch_set_params: treelet size %d of mesh %u", treelet_sizes[m], m);
        ATR_REQUIRE(iterations[m] <= 24, ATR_ERR_INVALID_ARG, "atr_batch_set_params: iterations %d", iterations[m]);
        mx = std::max(mx, (int)iterations[m]);
        mts = std::max(mts, (int)treelet_sizes[m]);
    }
    ATR_CUDA(cudaMemcpyAsync(b->d_tsize, treelet_sizes, b->count, cudaMemcpyHostToDevice, ctx->stream));
    ATR_CUDA(cudaMemcpyAsync(b->d_iters, iterations, b->count, cudaMemcpyHostToDevice, ctx->stream));
    ATR_CUDA(cudaStreamSynchronize(ctx->stream));
    b->per_mesh_params = true;
    b->max_iters = mx;
    b->max_tsize = mts;
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
    return ATR_OK;
}

int atr_batch_build(atr_ctx* ctx, atr_batch* b, int optimizer, int treelet_size, int iterations, float ci, float ct,
                    int use_graph) {
    ATR_REQUIRE(ctx && b, ATR_ERR_INVALID_ARG, "atr_batch_build: NULL argument");
    ATR_REQUIRE(optimizer >= 0 && optimizer <= 2, ATR_ERR_INVALID_ARG, "atr_batch_build: optimizer %d", optimizer);
    ATR_REQUIRE(optimizer != 1 || (treelet_size >= 3 && treelet_size <= 20), ATR_ERR_UNSUPPORTED,
                "atr_batch_build: treelet size %d", treelet_size);
    ATR_REQUIRE(optimizer != 2 || treelet_size == 7, ATR_ERR_UNSUPPORTED, "atr_batch_build: TRBVH treelet %d",
                treelet_size);
    ATR_REQUIRE(iterations >= 0 && iterations <= 24, ATR_ERR_INVALID_ARG, "atr_batch_build: iterations %d",
                iterations);
    if (!use_graph) return batch_run(ctx, b, optimizer, treelet_size, iterations, ci, ct);
    const int key[10] = {optimizer,        treelet_size,       iterations,      b->per_mesh_params ? 1 : 0,
                         ctx->atr_warps,   ctx->atr_group_min, ctx->sort_bits,  ctx->atr_levels,
                         ctx->atr_quad_min, ctx->atr_warp_max};
    const bool same = b->graph && std::memcmp(key, b->graph_key, sizeof(key)) == 0 && b->graph_cf[0] == ci &&
                      b->graph_cf[1] == ct;
    if (!same) {
        if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
        const bool timing = ctx->timing;
        ctx->timing = false;
        const uint64_t l0 = ctx->launches;
        cudaGraph_t graph = nullptr;
        ATR_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        const int st = batch_run(ctx, b, optimizer, treelet_size, iterations, ci, ct);
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
        ctx->timing = timing;
        if (st != ATR_OK) { if (graph) cudaGraphDestroy(graph); return st; }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture", __FILE__, __LINE__);
        e = cudaGraphInstantiate(&b->graph, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) { b->graph = nullptr; return cuda_fail(e, "cudaGraphInstantiate", __FILE__, __LINE__); }
        b->graph_launches = ctx->launches - l0;
        ctx->launches = l0;
        std::memcpy(b->graph_key, key, sizeof(key));
        b->graph_cf[0] = ci;
        b->graph_cf[1] = ct;
    }
    ctx->phase_begin("batch");
    ATR_CUDA(cudaGraphLaunch(b->graph, ctx->stream));
    ctx->phase_end();
    ctx->launches += b->graph_launches;
    return ATR_OK;
}

int atr_batch_info(const atr_batch* b, uint32_t* count, uint32_t* num_triangles, uint64_t* total_nodes) {
    ATR_REQUIRE(b, ATR_ERR_INVALID_ARG, "atr_batch_info: NULL argument");
    if (count) *count = b->count;
    if (num_triangles) *num_triangles = b->n;
    if (total_nodes) *total_nodes = b->total_nodes;
    return ATR_OK;
}

int atr_batch_mesh_view(const atr_batch* b, uint32_t mesh, atr_tree_view* v) {
    ATR_REQUIRE(b && v, ATR_ERR_INVALID_ARG, "atr_batch_mesh_view: NULL argument");
    ATR_REQUIRE(mesh < b->count, ATR_ERR_INVALID_ARG, "atr_batch_mesh_view: mesh %u of %u", mesh, b->count);
    const size_t base = 2 * (size_t)b->h_tri_off[mesh] - mesh;
    v->num_triangles = b->h_tri_off[mesh + 1] - b->h_tri_off[mesh];
    v->root = 0;
    v->parent = b->tree.parent + base;
    v->left = b->tree.left + base;
    v->right = b->tree.right + base;
    v->data = b->tree.data + base;
    v->bbox_min = reinterpret_cast<float*>(b->tree.bmin + base);
    v->bbox_max = reinterpret_cast<float*>(b->tree.bmax + base);
    v->area = b->tree.area + base;
    return ATR_OK;
}

int atr_batch_download_mesh(atr_ctx* ctx, const atr_batch* b, uint32_t mesh, int32_t* parent, int32_t* left,
                            int32_t* right, int32_t* data, float* bmin, float* bmax, float* area) {
    ATR_REQUIRE(ctx && b, ATR_ERR_INVALID_ARG, "atr_batch_download_mesh: NULL argument");
    atr_tree_view v;
    ATR_TRY(atr_batch_mesh_view(b, mesh, &v));
    const size_t nn = 2 * (size_t)v.num_triangles - 1;
    cudaStream_t s = ctx->stream;
    if (parent) ATR_CUDA(cudaMemcpyAsync(parent, v.parent, nn * 4, cudaMemcpyDeviceToHost, s));
    if (left) ATR_CUDA(cudaMemcpyAsync(left, v.left, nn * 4, cudaMemcpyDeviceToHost, s));
    if (right) ATR_CUDA(cudaMemcpyAsync(right, v.right, nn * 4, cudaMemcpyDeviceToHost, s));
    if (data) ATR_CUDA(cudaMemcpyAsync(data, v.data, nn * 4, cudaMemcpyDeviceToHost, s));
    if (bmin) ATR_CUDA(cudaMemcpyAsync(bmin, v.bbox_min, nn * 16, cudaMemcpyDeviceToHost, s));
    if (bmax) ATR_CUDA(cudaMemcpyAsync(bmax, v.bbox_max, nn * 16, cudaMemcpyDeviceToHost, s));
    if (area) ATR_CUDA(cudaMemcpyAsync(area, v.area, nn * 4, cudaMemcpyDeviceToHost, s));
    return atr_ctx_synchronize(ctx);
}

static int batch_alloc_outputs(atr_ctx* ctx, atr_batch* b) {
    const size_t nn = b->total_nodes, n = b->n;
    if (!b->col_block) {
        const size_t b4 = align256(nn * 4), b16 = align256(nn * 16);
        ATR_TRY(ctx->alloc(&b->col_block, 5 * b4 + 2 * b16 + align256(n * 4)));
        char* p = static_cast<char*>(b->col_block);
        b->col.parent = reinterpret_cast<int32_t*>(p); p += b4;
        b->col.left = reinterpret_cast<int32_t*>(p); p += b4;
        b->col.right = reinterpret_cast<int32_t*>(p); p += b4;
        b->col.data = reinterpret_cast<int32_t*>(p); p += b4;
        b->col.count = reinterpret_cast<int32_t*>(p); p += b4;
        b->col.bmin = reinterpret_cast<float4*>(p); p += b16;
        b->col.bmax = reinterpret_cast<float4*>(p); p += b16;
        b->col.tri_indices = reinterpret_cast<int32_t*>(p);
    }
    if (!b->cp_block) {
        const size_t bn = align256((n - b->count) * 64), bw = align256(n * 64), bt = align256(n * 16);
        const size_t bs = align256(b->count * 16ull + 8);
        ATR_TRY(ctx->alloc(&b->cp_block, bn + bw + bt + bs));
        char* p = static_cast<char*>(b->cp_block);
        b->cp_nodes = reinterpret_cast<int4*>(p); p += bn;
        b->cp_woop = reinterpret_cast<float4*>(p); p += bw;
        b->cp_tri = reinterpret_cast<int32_t*>(p); p += bt;
        b->d_sizes = reinterpret_cast<int64_t*>(p);
    }
    return ATR_OK;
}

int atr_batch_collapse(atr_ctx* ctx, atr_batch* b, float ci, float ct, int max_leaf, float* sah) {
    ATR_REQUIRE(ctx && b, ATR_ERR_INVALID_ARG, "atr_batch_collapse: NULL argument");
    ATR_REQUIRE(max_leaf >= 0, ATR_ERR_INVALID_ARG, "atr_batch_collapse: max_leaf %d", max_leaf);
    ATR_TRY(batch_alloc_outputs(ctx, b));
    const Segs segs{b->d_tri_off, b->d_tile_off, b->count, b->n};
    float* parts = nullptr;
    if (sah) ATR_TRY(ctx->alloc(reinterpret_cast<void**>(&parts), 8ull * b->count));
    ctx->phase_begin("collapse");
    int st = collapse_segs(ctx, segs, b->total_nodes, b->tree, b->col, ci, ct, max_leaf, parts);
    ctx->phase_end();
    if (st == ATR_OK && sah) {
        std::vector<float> h(2ull * b->count);
        cudaError_t e = cudaMemcpyAsync(h.data(), parts, h.size() * 4, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) st = atr_ctx_synchronize(ctx);
        else st = cuda_fail(e, "cudaMemcpyAsync(sah)", __FILE__, __LINE__);
        if (st == ATR_OK)
            for (uint32_t m = 0; m < b->count; ++m) sah[m] = h[2 * m] / h[2 * m + 1];
    }
    ctx->release(parts);
    b->col_ci = ci;
    b->col_ct = ct;
    b->col_max_leaf = max_leaf;
    b->flattened = false;
    return st;
}

int atr_batch_flatten(atr_ctx* ctx, atr_batch* b) {
    ATR_REQUIRE(ctx && b, ATR_ERR_INVALID_ARG, "atr_batch_flatten: NULL argument");
    ATR_REQUIRE(b->col_block, ATR_ERR_INVALID_ARG, "atr_batch_flatten: collapse the batch first");
    const Segs segs{b->d_tri_off, b->d_tile_off, b->count, b->n};
    ctx->phase_begin("flatten");
    int st = flatten_segs(ctx, segs, b->col, b->verts, b->cp_nodes, b->cp_woop, b->cp_tri, b->d_sizes);
    ctx->phase_end();
    ATR_TRY(st);
    b->h_sizes.resize(2ull * b->count + 1);
    ATR_CUDA(cudaMemcpyAsync(b->h_sizes.data(), b->d_sizes, b->h_sizes.size() * 8, cudaMemcpyDeviceToHost,
                             ctx->stream));
    ATR_CUDA(cudaStreamSynchronize(ctx->stream));
    b->max_depth = (int32_t)b->h_sizes[2ull * b->count];
    b->flattened = true;
    return ATR_OK;
}

int atr_batch_compact_view(const atr_batch* b, uint32_t mesh, atr_compact_view* v) {
    ATR_REQUIRE(b && v, ATR_ERR_INVALID_ARG, "atr_batch_compact_view: NULL argument");
    ATR_REQUIRE(b->flattened, ATR_ERR_INVALID_ARG, "atr_batch_compact_view: flatten the batch first");
    ATR_REQUIRE(mesh < b->count, ATR_ERR_INVALID_ARG, "atr_batch_compact_view: mesh %u of %u", mesh, b->count);
    const size_t s0 = b->h_tri_off[mesh];
    v->num_nodes = b->h_sizes[mesh];
    v->num_woop = b->h_sizes[b->count + mesh];
    v->nodes = reinterpret_cast<int32_t*>(b->cp_nodes + 4 * (s0 - mesh));
    v->woop = reinterpret_cast<float*>(b->cp_woop + 4 * s0);
    v->tri_index = b->cp_tri + 4 * s0;
    v->max_depth = b->max_depth;
    return ATR_OK;
}

int atr_batch_compact_download(atr_ctx* ctx, const atr_batch* b, uint32_t mesh, int32_t* nodes, float* woop,
                               int32_t* tri) {
    ATR_REQUIRE(ctx, ATR_ERR_INVALID_ARG, "atr_batch_compact_download: NULL argument");
    atr_compact_view v;
    ATR_TRY(atr_batch_compact_view(b, mesh, &v));
    cudaStream_t s = ctx->stream;
    if (nodes) ATR_CUDA(cudaMemcpyAsync(nodes, v.nodes, (size_t)v.num_nodes * 64, cudaMemcpyDeviceToHost, s));
    if (woop) ATR_CUDA(cudaMemcpyAsync(woop, v.woop, (size_t)v.num_woop * 16, cudaMemcpyDeviceToHost, s));
    if (tri) ATR_CUDA(cudaMemcpyAsync(tri, v.tri_index, (size_t)v.num_woop * 4, cudaMemcpyDeviceToHost, s));
    return atr_ctx_synchronize(ctx);
}

int atr_batch_trace(atr_ctx* ctx, const atr_batch* b, const float* rays, int64_t num_rays,
                    const uint32_t* ray_offsets, const uint32_t* group_mesh, uint32_t groups, int any_hit,
                    int32_t* results) {
    ATR_REQUIRE(ctx && b && rays && results && ray_offsets && group_mesh, ATR_ERR_INVALID_ARG,
                "atr_batch_trace: NULL argument");
    ATR_REQUIRE(b->flattened, ATR_ERR_INVALID_ARG, "atr_batch_trace: flatten the batch first");
    ATR_REQUIRE(groups >= 1 && ray_offsets[0] == 0 && (int64_t)ray_offsets[groups] == num_rays,
                ATR_ERR_INVALID_ARG, "atr_batch_trace: ray_offsets must run from 0 to num_rays");
    for (uint32_t g = 0; g < groups; ++g) {
        ATR_REQUIRE(group_mesh[g] < b->count, ATR_ERR_INVALID_ARG, "atr_batch_trace: group %u mesh %u", g,
                    group_mesh[g]);
        ATR_REQUIRE(ray_offsets[g + 1] >= ray_offsets[g], ATR_ERR_INVALID_ARG, "atr_batch_trace: offsets decrease");
    }
    uint32_t* map = nullptr;
    ATR_TRY(ctx->alloc(reinterpret_cast<void**>(&map), (2ull * groups + 1) * 4));
    cudaError_t e = cudaMemcpyAsync(map, ray_offsets, (groups + 1) * 4ull, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(map + groups + 1, group_mesh, groups * 4ull, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) {
        ctx->release(map);
        return cuda_fail(e, "cudaMemcpyAsync(ray groups)", __FILE__, __LINE__);
    }
    const int st = trace_batch(ctx, b->cp_nodes, b->cp_woop, b->cp_tri, map, map + groups + 1, b->d_tri_off, groups,
                               b->max_depth, reinterpret_cast<const float4*>(rays), num_rays, any_hit,
                               reinterpret_cast<int4*>(results));
    ctx->release(map);
    return st;
}

int atr_batch_refit_mesh(atr_ctx* ctx, atr_batch* b, uint32_t mesh, const float* vertices, int on_device) {
    return atr::batch_refit_mesh(ctx, b, mesh, vertices, on_device, nullptr);
}

}  // extern "C"

namespace atr {

int batch_refit_mesh(atr_ctx* ctx, atr_batch* b, uint32_t mesh, const float* vertices, int on_device,
                     float* h_sah) {
    ATR_REQUIRE(ctx && b && vertices, ATR_ERR_INVALID_ARG, "atr_batch_refit_mesh: NULL argument");
    ATR_REQUIRE(mesh < b->count, ATR_ERR_INVALID_ARG, "atr_batch_refit_mesh: mesh %u of %u", mesh, b->count);
    const size_t s0 = b->h_tri_off[mesh];
    const uint32_t n = b->h_tri_off[mesh + 1] - b->h_tri_off[mesh];
    ATR_CUDA(cudaMemcpyAsync(b->verts + 3 * s0, vertices, n * 48ull,
                             on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
    const size_t nb = 2 * s0 - mesh;
    const TreeOut t{b->tree.parent + nb, b->tree.left + nb, b->tree.right + nb, b->tree.data + nb,
                    b->tree.bmin + nb, b->tree.bmax + nb, b->tree.area + nb};
    ATR_TRY(refit_arrays(ctx, n, t, b->verts + 3 * s0));
    if (!b->flattened) return ATR_OK;
    // Re-collapse and re-flatten this mesh only, in place in its slices.
    const Segs one{nullptr, nullptr, 1u, n};
    const CollapsedOut c{b->col.parent + nb, b->col.left + nb, b->col.right + nb, b->col.data + nb,
                         b->col.count + nb, b->col.bmin + nb, b->col.bmax + nb, b->col.tri_indices + s0};
    // sizes: Compact2 node and Woop counts, depth, then (when asked) the SAH parts.
    int64_t* sizes = nullptr;
    ATR_TRY(ctx->alloc(reinterpret_cast<void**>(&sizes), 32));
    float* parts = h_sah ? reinterpret_cast<float*>(sizes + 3) : nullptr;
    int st = collapse_segs(ctx, one, 2 * (size_t)n - 1, t, c, b->col_ci, b->col_ct, b->col_max_leaf, parts);
    if (st == ATR_OK)
        st = flatten_segs(ctx, one, c, b->verts + 3 * s0, b->cp_nodes + 4 * (s0 - mesh), b->cp_woop + 4 * s0,
                          b->cp_tri + 4 * s0, sizes);
    int64_t h[4] = {0, 0, 0, 0};
    if (st == ATR_OK) {
        cudaError_t e = cudaMemcpyAsync(h, sizes, 32, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) st = cuda_fail(e, "cudaMemcpy(sizes)", __FILE__, __LINE__);
    }
    ctx->release(sizes);
    ATR_TRY(st);
    if (h_sah) {
        float p[2];
        std::memcpy(p, h + 3, 8);
        *h_sah = p[0] / p[1];
    }
    b->h_sizes[mesh] = h[0];
    b->h_sizes[b->count + mesh] = h[1];
    for (int32_t d = b->max_depth.load(); (int32_t)h[2] > d && !b->max_depth.compare_exchange_weak(d, (int32_t)h[2]);) {
    }
    return ATR_OK;
}

}  // namespace atr

extern "C" {

int atr_batch_sah(atr_ctx* ctx, const atr_batch* b, float ci, float ct, float* sah) {
    ATR_REQUIRE(ctx && b && sah, ATR_ERR_INVALID_ARG, "atr_batch_sah: NULL argument");
    std::vector<float> area(b->total_nodes);
    ATR_CUDA(cudaMemcpyAsync(area.data(), b->tree.area, area.size() * 4, cudaMemcpyDeviceToHost, ctx->stream));
    ATR_TRY(atr_ctx_synchronize(ctx));
    for (uint32_t m = 0; m < b->count; ++m) {
        const uint32_t n = b->h_tri_off[m + 1] - b->h_tri_off[m];
        const float* a = area.data() + (2 * (size_t)b->h_tri_off[m] - m);
        const float total = a[0];
        float si = total, sl = 0.0f;
        for (uint32_t i = 1; i < n - 1; ++i) si += a[i];
        for (uint32_t i = n - 1; i < 2 * n - 1; ++i) sl += a[i];
        sah[m] = (ci * si + ct * sl) / total;
    }
    return ATR_OK;
}

}  // extern "C"
