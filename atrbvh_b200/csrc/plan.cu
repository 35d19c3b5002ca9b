// Build plans: the steady-state single-mesh build replayed from a CUDA graph.
//
// The reference rebuilds a mesh by calling LBVHBuilder::BuildTree, an
// optimiser and BVHTreeCollapser::Collapse in sequence
// (BVHRT-Core/src/LBVHBuilder.cpp:60-97, AgglomerativeTreeletOptimizer.cpp:75-92,
// BVHTreeCollapser.cpp:21-93), each allocating its outputs and launching its
// kernels one by one.  A plan owns the outputs (tree, collapsed tree and,
// optionally, the Compact2 layout at its worst-case size) for one scene and
// one set of build parameters, and enqueues the whole sequence into them.
// With use_graph the first run captures that sequence into a CUDA graph and
// later runs replay it with one launch; a change of the context's launch
// tuning captures it again.  Every allocation made during a run (sort
// buffers, prepass, scan and climb scratch) is also freed within the run, so
// the graph owns no memory between replays.  The run enqueues only: results
// and sizes are read on request.

#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "internal.h"

struct atr_plan {
    atr_ctx* ctx = nullptr;
    const atr_scene* scene = nullptr;
    atr_plan_params p{};
    atr_tree* tree = nullptr;
    atr_collapsed* col = nullptr;
    atr_compact* cp = nullptr;
    void* block = nullptr;            // sizes (3 int64) and SAH parts (2 floats)
    int64_t* d_sizes = nullptr;
    float* d_sah = nullptr;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};  // start, collapsed, end
    cudaGraphExec_t graph = nullptr;
    int graph_key[6] = {0, 0, 0, 0, 0, 0};
    bool graph_phases = false;  // the graph records per-phase marks
    uint64_t graph_launches = 0;
    bool ran = false;
    bool sizes_read = false;
    // Phase marks recorded inside the graph (morton, sort, build, atrbvh or
    // trbvh, collapse, flatten), re-recorded by every replay.
    std::vector<atr_ctx::Phase> phases;
    std::string phase_names;
    bool graph_ran = false;
};

namespace atr {
namespace {

void plan_tuning_key(const atr_ctx* ctx, int key[6]) {
    key[0] = ctx->atr_warps;
    key[1] = ctx->atr_group_min;
    key[2] = ctx->sort_bits;
    key[3] = ctx->atr_levels;
    key[4] = ctx->atr_quad_min;
    key[5] = ctx->atr_warp_max;
}

// Marks a point of the run; while capturing, as an external record node so
// that the graph records the event each time it runs.
int plan_mark(atr_ctx* ctx, cudaEvent_t ev, bool capturing) {
    ATR_CUDA(capturing ? cudaEventRecordWithFlags(ev, ctx->stream, cudaEventRecordExternal)
                       : cudaEventRecord(ev, ctx->stream));
    return ATR_OK;
}

// The whole build, enqueued on the context's stream into the plan's arrays.
int plan_enqueue(atr_ctx* ctx, atr_plan* P, bool capturing) {
    const atr_plan_params& p = P->p;
    atr_tree* t = P->tree;
    const uint32_t n = t->n;
    ATR_TRY(plan_mark(ctx, P->ev[0], capturing));
    ATR_TRY(lbvh_build_into(ctx, P->scene->verts, n, P->scene->d_bounds, p.morton_bits, t));
    if (p.optimizer == 1) {
        ATR_TRY(atr_optimize_atrbvh(ctx, t, p.treelet_size, p.iterations, p.ci, p.ct));
    } else if (p.optimizer == 2) {
        ATR_TRY(atr_optimize_trbvh(ctx, t, p.treelet_size, p.iterations, p.ci, p.ct));
    }
    // Nothing allocated by this run outlives it.
    ctx->release(t->prepass_block);
    t->prepass_block = nullptr;
    t->prepass = BuildPrepass{};
    ctx->release(t->sorted_keys);
    ctx->release(t->sorted_idx);
    t->sorted_keys = nullptr;
    t->sorted_idx = nullptr;
    ctx->phase_begin("collapse");
    const int cst = collapse_into(ctx, t, p.ci, p.ct, p.max_leaf, P->col, P->d_sah);
    ctx->phase_end();
    ATR_TRY(cst);
    ATR_TRY(plan_mark(ctx, P->ev[1], capturing));
    if (p.flatten) {
        const Segs segs{nullptr, nullptr, 1u, n};
        const atr_collapsed* c = P->col;
        const CollapsedOut co{c->parent, c->left, c->right, c->data, c->count, c->bmin, c->bmax, c->tri_indices};
        ctx->phase_begin("flatten");
        const int fst = flatten_segs(ctx, segs, co, P->scene->verts, P->cp->nodes, P->cp->woop, P->cp->tri_index,
                                     P->d_sizes);
        ctx->phase_end();
        ATR_TRY(fst);
    }
    ATR_TRY(plan_mark(ctx, P->ev[2], capturing));
    return ATR_OK;
}

}  // namespace
}  // namespace atr

using namespace atr;

extern "C" {

int atr_plan_create(atr_ctx* ctx, const atr_scene* scene, const atr_plan_params* params, atr_plan** out) {
    ATR_REQUIRE(ctx && scene && params && out, ATR_ERR_INVALID_ARG, "atr_plan_create: NULL argument");
    const atr_plan_params& p = *params;
    ATR_REQUIRE(p.morton_bits == 30 || p.morton_bits == 63, ATR_ERR_UNSUPPORTED,
                "atr_plan_create: morton_bits must be 30 or 63 (got %d)", p.morton_bits);
    ATR_REQUIRE(p.optimizer >= 0 && p.optimizer <= 2, ATR_ERR_INVALID_ARG, "atr_plan_create: optimizer %d",
                p.optimizer);
    ATR_REQUIRE(p.optimizer != 1 || (p.treelet_size >= 3 && p.treelet_size <= 20), ATR_ERR_UNSUPPORTED,
                "atr_plan_create: ATRBVH treelet size %d outside [3, 20]", p.treelet_size);
    ATR_REQUIRE(p.optimizer != 2 || p.treelet_size == 7, ATR_ERR_UNSUPPORTED,
                "atr_plan_create: TRBVH treelet size %d (the reference's subset kernel covers 7)", p.treelet_size);
    ATR_REQUIRE(p.iterations >= 0 && p.iterations <= 24, ATR_ERR_INVALID_ARG, "atr_plan_create: iterations %d",
                p.iterations);
    ATR_REQUIRE(p.max_leaf >= 0, ATR_ERR_INVALID_ARG, "atr_plan_create: max_leaf %d < 0", p.max_leaf);
    *out = nullptr;
    atr_plan* P = new atr_plan();
    P->ctx = ctx;
    P->scene = scene;
    P->p = p;
    const uint32_t n = scene->n;
    int st = tree_alloc(ctx, n, &P->tree);
    // The plan's collapsed tree shares its tree's links and boxes: the plan
    // rewrites both on every run and hands out neither for writing.
    if (st == ATR_OK) st = collapsed_alloc_sharing(ctx, P->tree, &P->col);
    if (st == ATR_OK) st = ctx->alloc(&P->block, 256);
    if (st == ATR_OK && p.flatten) {
        // Upper bounds: every inner node; three entries and a terminator per triangle.
        P->cp = new atr_compact();
        P->cp->ctx = ctx;
        st = ctx->alloc(reinterpret_cast<void**>(&P->cp->nodes), (size_t)(n - 1) * 64);
        if (st == ATR_OK) st = ctx->alloc(reinterpret_cast<void**>(&P->cp->woop), (size_t)n * 4 * 16);
        if (st == ATR_OK) st = ctx->alloc(reinterpret_cast<void**>(&P->cp->tri_index), (size_t)n * 4 * 4);
    }
    for (int k = 0; k < 3 && st == ATR_OK; ++k) {
        const cudaError_t e = cudaEventCreate(&P->ev[k]);
        if (e != cudaSuccess) st = cuda_fail(e, "cudaEventCreate", __FILE__, __LINE__);
    }
    if (st == ATR_OK) {
        P->d_sizes = static_cast<int64_t*>(P->block);
        P->d_sah = reinterpret_cast<float*>(static_cast<char*>(P->block) + 32);
        const cudaError_t e = cudaMemsetAsync(P->block, 0, 256, ctx->stream);
        if (e != cudaSuccess) st = cuda_fail(e, "cudaMemsetAsync(plan)", __FILE__, __LINE__);
    }
    if (st != ATR_OK) {
        atr_plan_destroy(P);
        return st;
    }
    *out = P;
    return ATR_OK;
}

int atr_plan_run(atr_ctx* ctx, atr_plan* P, int use_graph) {
    ATR_REQUIRE(ctx && P, ATR_ERR_INVALID_ARG, "atr_plan_run: NULL argument");
    ATR_REQUIRE(ctx == P->ctx, ATR_ERR_INVALID_ARG, "atr_plan_run: the plan belongs to another context");
    atr_tree* t = P->tree;
    // Allocations an earlier eager run left on the tree go before any capture.
    tree_topology_changed(t);
    ctx->release(t->prepass_block);
    t->prepass_block = nullptr;
    t->prepass = BuildPrepass{};
    ctx->release(t->sorted_keys);
    ctx->release(t->sorted_idx);
    t->sorted_keys = nullptr;
    t->sorted_idx = nullptr;
    P->sizes_read = false;
    if (!use_graph) {
        ctx->phase_begin("plan");
        const int st = plan_enqueue(ctx, P, false);
        ctx->phase_end();
        P->ran = st == ATR_OK;
        return st;
    }
    int key[6];
    plan_tuning_key(ctx, key);
    // Per-phase marks are captured when the context times phases: each is an
    // event node at a stage boundary, which leaves the device idle for several
    // microseconds, so a graph captured without them is a little faster.
    if (!P->graph || std::memcmp(key, P->graph_key, sizeof(key)) != 0 || P->graph_phases != ctx->timing) {
        if (P->graph) {
            cudaGraphExecDestroy(P->graph);
            P->graph = nullptr;
        }
        for (auto& ph : P->phases) {
            cudaEventDestroy(ph.a);
            cudaEventDestroy(ph.b);
        }
        P->phases.clear();
        // The capture records its own phase marks (kept by the plan) when the
        // context times phases.
        const bool timing = ctx->timing;
        std::vector<atr_ctx::Phase> outer;
        outer.swap(ctx->phases);
        ctx->capture_marks = true;
        const uint64_t l0 = ctx->launches;
        cudaGraph_t graph = nullptr;
        cudaError_t be = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
        const int st = be == cudaSuccess ? plan_enqueue(ctx, P, true) : ATR_OK;
        const cudaError_t e = be == cudaSuccess ? cudaStreamEndCapture(ctx->stream, &graph) : be;
        ctx->timing = timing;
        ctx->capture_marks = false;
        P->phases.swap(ctx->phases);
        ctx->phases.swap(outer);
        if (st != ATR_OK) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture(plan)", __FILE__, __LINE__);
        const cudaError_t ie = cudaGraphInstantiate(&P->graph, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) {
            P->graph = nullptr;
            return cuda_fail(ie, "cudaGraphInstantiate(plan)", __FILE__, __LINE__);
        }
        P->graph_launches = ctx->launches - l0;
        ctx->launches = l0;
        std::memcpy(P->graph_key, key, sizeof(key));
        P->graph_phases = timing;
    }
    ctx->phase_begin("plan");
    ATR_CUDA(cudaGraphLaunch(P->graph, ctx->stream));
    ctx->phase_end();
    ctx->launches += P->graph_launches;
    P->ran = true;
    P->graph_ran = true;
    return ATR_OK;
}

int atr_plan_phase_times(atr_ctx* ctx, atr_plan* P, float* ms, int capacity, int* count) {
    ATR_REQUIRE(ctx && P && count, ATR_ERR_INVALID_ARG, "atr_plan_phase_times: NULL argument");
    ATR_REQUIRE(P->graph_ran, ATR_ERR_INVALID_ARG, "atr_plan_phase_times: no graph replay yet");
    ATR_CUDA(cudaEventSynchronize(P->ev[2]));
    int k = 0;
    P->phase_names.clear();
    for (auto& ph : P->phases) {
        float t = 0.0f;
        ATR_CUDA(cudaEventElapsedTime(&t, ph.a, ph.b));
        if (ms && k < capacity) ms[k] = t;
        if (!P->phase_names.empty()) P->phase_names += ",";
        P->phase_names += ph.name;
        ++k;
    }
    *count = k;
    return ATR_OK;
}

const char* atr_plan_phase_names(const atr_plan* P) { return P ? P->phase_names.c_str() : ""; }

int atr_plan_tree(const atr_plan* P, const atr_tree** tree) {
    ATR_REQUIRE(P && tree, ATR_ERR_INVALID_ARG, "atr_plan_tree: NULL argument");
    *tree = P->tree;
    return ATR_OK;
}

int atr_plan_collapsed(const atr_plan* P, const atr_collapsed** collapsed) {
    ATR_REQUIRE(P && collapsed, ATR_ERR_INVALID_ARG, "atr_plan_collapsed: NULL argument");
    *collapsed = P->col;
    return ATR_OK;
}

int atr_plan_compact(atr_ctx* ctx, atr_plan* P, const atr_compact** compact) {
    ATR_REQUIRE(ctx && P && compact, ATR_ERR_INVALID_ARG, "atr_plan_compact: NULL argument");
    ATR_REQUIRE(P->cp, ATR_ERR_INVALID_ARG, "atr_plan_compact: the plan was created without flatten");
    ATR_REQUIRE(P->ran, ATR_ERR_INVALID_ARG, "atr_plan_compact: the plan has not run");
    if (!P->sizes_read) {
        int64_t h[3];
        ATR_CUDA(cudaMemcpyAsync(h, P->d_sizes, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        ATR_TRY(atr_ctx_synchronize(ctx));
        P->cp->num_nodes = h[0];
        P->cp->num_woop = h[1];
        P->cp->max_depth = (int32_t)h[2];
        P->sizes_read = true;
    }
    *compact = P->cp;
    return ATR_OK;
}

int atr_plan_sah(atr_ctx* ctx, atr_plan* P, float* sah) {
    ATR_REQUIRE(ctx && P && sah, ATR_ERR_INVALID_ARG, "atr_plan_sah: NULL argument");
    ATR_REQUIRE(P->ran, ATR_ERR_INVALID_ARG, "atr_plan_sah: the plan has not run");
    float h[2];
    ATR_CUDA(cudaMemcpyAsync(h, P->d_sah, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    ATR_TRY(atr_ctx_synchronize(ctx));
    *sah = h[0] / h[1];
    return ATR_OK;
}

int atr_plan_times(atr_ctx* ctx, atr_plan* P, float* build_ms, float* flatten_ms) {
    ATR_REQUIRE(ctx && P, ATR_ERR_INVALID_ARG, "atr_plan_times: NULL argument");
    ATR_REQUIRE(P->ran, ATR_ERR_INVALID_ARG, "atr_plan_times: the plan has not run");
    ATR_CUDA(cudaEventSynchronize(P->ev[2]));
    if (build_ms) ATR_CUDA(cudaEventElapsedTime(build_ms, P->ev[0], P->ev[1]));
    if (flatten_ms) ATR_CUDA(cudaEventElapsedTime(flatten_ms, P->ev[1], P->ev[2]));
    return ATR_OK;
}

int atr_plan_destroy(atr_plan* P) {
    if (!P) return ATR_OK;
    if (P->graph) cudaGraphExecDestroy(P->graph);
    for (auto& ph : P->phases) {
        cudaEventDestroy(ph.a);
        cudaEventDestroy(ph.b);
    }
    for (cudaEvent_t e : P->ev)
        if (e) cudaEventDestroy(e);
    atr_tree_destroy(P->tree);
    atr_collapsed_destroy(P->col);
    atr_compact_destroy(P->cp);
    if (P->ctx) P->ctx->release(P->block);
    delete P;
    return ATR_OK;
}

}  // extern "C"
