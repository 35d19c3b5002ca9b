// ATRBVH: agglomerative treelet restructuring on sm_100a.
//
// Semantics follow BVHRT-Core/src/AgglomerativeTreelet.cu:392-554 (bottom-up
// pass, one thread per leaf; the second child to arrive processes a node; a
// warp restructures the treelets of its lanes' nodes whose subtree holds at
// least gamma triangles) and AgglomerativeTreeletOptimizer.cpp:73-92 (gamma
// starts at the treelet size and doubles per iteration).  The treelet state
// lives in registers, one treelet leaf per lane; only the distance matrix is
// in shared memory.  Every reduction keeps the reference's shuffle-down tree
// and strict comparisons, so ties resolve as in the reference.
//
// Memory ordering: a node's data is published by the thread that finished it
// (plain stores, fence, atomic); the second arrival fences after its atomic
// and reads descendants through L2 (ld.cg), and __syncwarp orders the other
// lanes of the warp behind it.

#include "common.cuh"
#include "internal.h"
#include "treelet.cuh"

namespace atr {
namespace {

constexpr int kAtrWarps = 4;

// One treelet rooted at `root`, processed by the whole warp.
__device__ bool process_treelet(const TreeRefs& t, int root, float root_sah, int tsize, float ci,
                                float* dist) {
    const int lane = threadIdx.x & 31;

    // ---- formTreelet ----
    int internal_node;
    LeafSlot slot;
    if (!form_treelet(t, root, tsize, slot, internal_node)) return false;

    // ---- agglomerative merge (AgglomerativeTreelet.cu:476-532) ----
    Box box;
    box.mnx = slot.mn.x; box.mny = slot.mn.y; box.mnz = slot.mn.z;
    box.mxx = slot.mx.x; box.mxy = slot.mx.y; box.mxz = slot.mx.z;
    int node = slot.node;
    float sah = slot.sah;
    int right_node = -1;  // treeletLeaves[lane] after the merge that fills this lane
    float la = 0.0f;      // treeletLeavesAreas[lane]

    const int npairs = tsize * (tsize - 1) / 2;
    for (int base = 0; base < npairs; base += 32) {
        const int j = base + lane;
        int r = 0, c = 0;
        if (j < npairs) trm_rc(j, r, c);
        const Box a = shfl_box(box, r);
        const Box b = shfl_box(box, c);
        if (j < npairs) dist[j] = union_area(a, b);
    }
    __syncwarp();

    for (int last = tsize - 1; last > 0; --last) {
        // findMinimumDistance (:83-99): strided scan, strict <, shuffle-down reduce.
        const int msize = last * (last + 1) / 2;
        float best = FLT_MAX;
        int bi = 0;
        for (int j = lane; j < msize; j += 32) {
            const float d = dist[j];
            if (d < best) { best = d; bi = j; }
        }
#pragma unroll
        for (int sh = 16; sh > 0; sh >>= 1) {
            const float ob = __shfl_down_sync(kFull, best, sh);
            const int oi = __shfl_down_sync(kFull, bi, sh);
            if (ob < best) { best = ob; bi = oi; }
        }
        const int mi = __shfl_sync(kFull, bi, 0);
        int jr, jc;
        trm_rc(mi, jr, jc);

        // updateState (:101-150).
        const float sah_new = __fadd_rn(__shfl_sync(kFull, sah, jr), __shfl_sync(kFull, sah, jc));
        const int left_index = __shfl_sync(kFull, node, jr);
        const int right_index = __shfl_sync(kFull, node, jc);
        const Box bjr = shfl_box(box, jr);
        const Box bjc = shfl_box(box, jc);
        Box A;
        A.mnx = fminf(bjc.mnx, bjr.mnx); A.mny = fminf(bjc.mny, bjr.mny); A.mnz = fminf(bjc.mnz, bjr.mnz);
        A.mxx = fmaxf(bjc.mxx, bjr.mxx); A.mxy = fmaxf(bjc.mxy, bjr.mxy); A.mxz = fmaxf(bjc.mxz, bjr.mxz);
        const int new_internal = __shfl_sync(kFull, internal_node, last - 1);
        const float la_new = __fadd_rn(sah_new, __fmul_rn(ci, box_area(A.mnx, A.mny, A.mnz, A.mxx, A.mxy, A.mxz)));
        if (lane == jc) {
            node = new_internal;
            box = A;
            sah = la_new;
        }
        if (lane == last) la = la_new;
        const int last_index = __shfl_sync(kFull, node, last);
        const float sah_last = __shfl_sync(kFull, sah, last);
        const Box blast = shfl_box(box, last);
        if (lane == jr) {
            node = last_index;
            sah = sah_last;
            box = blast;
        }
        if (lane == last) {
            node = left_index;
            right_node = right_index;
            box = A;
        }

        // updateDistancesMatrix (:152-188).
        if (last > 1) {
            float moved = 0.0f;
            const bool mv = lane < last && lane != jr;
            if (mv) moved = dist[trm_idx(last, lane)];
            __syncwarp();
            if (mv) dist[trm_idx(max(jr, lane), min(jr, lane))] = moved;
            __syncwarp();
            int r = lane, c = lane;
            const bool up = lane < last && lane != jc;
            if (up) { r = max(jc, lane); c = min(jc, lane); }
            const Box br = shfl_box(box, r);
            const Box bc = shfl_box(box, c);
            const float d = union_area(br, bc);
            if (up) dist[trm_idx(r, c)] = d;
            __syncwarp();
        }
    }

    // ---- updateTreelet (:190-212) ----
    const float la1 = __shfl_sync(kFull, la, 1);
    const int ni = __shfl_sync(kFull, internal_node, lane > 0 ? lane - 1 : 0);
    if (la1 < root_sah && lane >= 1 && lane < tsize) {
        t.left[ni] = node;
        t.right[ni] = right_node;
        t.parent[node] = ni;
        t.parent[right_node] = ni;
        t.nsah[ni] = la;
        const float4 mn = make_float4(box.mnx, box.mny, box.mnz, 0.0f);
        const float4 mx = make_float4(box.mxx, box.mxy, box.mxz, 0.0f);
        t.bmin[ni] = mn;
        t.bmax[ni] = mx;
        t.area[ni] = box_area(mn, mx);
    }
    __syncwarp();
    return true;
}

// One iteration over every mesh of `segs`: thread i starts at the i-th sorted
// leaf of the batch.  Each mesh has its own treelet size and iteration count
// when `seg_tsize`/`seg_iters` are given; a mesh whose iterations are done
// sits this launch out.  Treelets are processed with the refs of the mesh of
// the lane that owns the root.
__global__ void __launch_bounds__(kAtrWarps * 32) k_atrbvh(TreeRefs g, Segs segs, int32_t* __restrict__ subtree,
                                                           uint32_t* __restrict__ counters, int tsize_all,
                                                           const uint8_t* __restrict__ seg_tsize,
                                                           const uint8_t* __restrict__ seg_iters, int iteration,
                                                           float ci, float ct, uint32_t* err) {
    __shared__ float s_dist[kAtrWarps][kMaxDist];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    int cur = -1, base = 0, cbase = 0, tsize = tsize_all;
    uint32_t nm = 2;
    if (i < segs.n) {
        const uint32_t m = segs.seg_of_tri(i);
        const uint32_t s0 = segs.tri_begin(m);
        nm = segs.tri_end(m) - s0;
        base = segs.node_base(m);
        cbase = segs.inner_base(m);
        if (seg_tsize) tsize = seg_tsize[m];
        if (!seg_iters || iteration < (int)seg_iters[m]) {
            const int leaf = base + (int)(i - s0) + (int)nm - 1;
            subtree[leaf] = 1;
            g.nsah[leaf] = __fmul_rn(ct, g.area[leaf]);
            cur = g.parent[leaf];
        }
    }
    const int gamma = tsize << iteration;
    while (__any_sync(kFull, cur >= 0)) {
        bool second = false;
        if (cur >= 0) {
            __threadfence();
            if (atomicAdd(&counters[cbase + cur], 1u) == 0u) cur = -1;
            else { second = true; __threadfence(); }
        }
        int cnt = 0;
        float my_sah = 0.0f;
        if (second) {
            const int x = base + cur;
            const int l = base + ld_cg(g.left + x), r = base + ld_cg(g.right + x);
            const float a = ld_cg(g.area + x);
            cnt = ld_cg(subtree + l) + ld_cg(subtree + r);
            my_sah = __fadd_rn(__fadd_rn(__fmul_rn(ci, a), ld_cg(g.nsah + l)), ld_cg(g.nsah + r));
            subtree[x] = cnt;
            g.nsah[x] = my_sah;
        }
        unsigned vote = __ballot_sync(kFull, cnt >= gamma);
        if (vote) __syncwarp();
        while (vote) {
            const int rl = __ffs(vote) - 1;
            const int root = __shfl_sync(kFull, cur, rl);
            const float rsah = __shfl_sync(kFull, my_sah, rl);
            const int rbase = __shfl_sync(kFull, base, rl);
            const uint32_t rn = __shfl_sync(kFull, nm, rl);
            const int rts = __shfl_sync(kFull, tsize, rl);
            if (!process_treelet(rebase(g, rbase, rn), root, rsah, rts, ci, s_dist[w]) && lane == 0)
                set_error_bits(err, kErrTreeletClimb);
            vote &= vote - 1;
        }
        if (cur >= 0) cur = ld_cg(g.parent + base + cur);
    }
}

}  // namespace

// ATRBVH over every mesh of `segs` (total_nodes = sum of 2n_m - 1).  tsize and
// iterations apply to all meshes unless per-mesh arrays are given, in which
// case `iterations` is their maximum.
int atrbvh_run(atr_ctx* ctx, const TreeRefs& g_in, const Segs& segs, size_t total_nodes, int tsize,
               int iterations, const uint8_t* seg_tsize, const uint8_t* seg_iters, float ci, float ct) {
    if (iterations <= 0) return ATR_OK;
    const size_t inner = segs.n - segs.count;
    void* scratch = nullptr;
    const size_t b_sub = align256(total_nodes * 4), b_sah = align256(total_nodes * 4), b_ctr = align256(inner * 4);
    ATR_TRY(ctx->alloc(&scratch, b_sub + b_sah + b_ctr));
    char* p = static_cast<char*>(scratch);
    int32_t* subtree = reinterpret_cast<int32_t*>(p);
    TreeRefs g = g_in;
    g.nsah = reinterpret_cast<float*>(p + b_sub);
    uint32_t* counters = reinterpret_cast<uint32_t*>(p + b_sub + b_sah);
    const int threads = kAtrWarps * 32;
    const uint32_t blocks = (segs.n + threads - 1) / threads;
    ctx->phase_begin("atrbvh");
    for (int it = 0; it < iterations; ++it) {
        cudaMemsetAsync(counters, 0, inner * 4, ctx->stream);
        k_atrbvh<<<blocks, threads, 0, ctx->stream>>>(g, segs, subtree, counters, tsize, seg_tsize, seg_iters, it,
                                                      ci, ct, ctx->d_error);
    }
    ctx->phase_end();
    ctx->launches += iterations;
    cudaError_t e = cudaGetLastError();
    ctx->release(scratch);
    if (e != cudaSuccess) return cuda_fail(e, "k_atrbvh launch", __FILE__, __LINE__);
    return ATR_OK;
}

}  // namespace atr

using namespace atr;

extern "C" int atr_optimize_atrbvh(atr_ctx* ctx, atr_tree* tree, int tsize, int iterations, float ci, float ct) {
    ATR_REQUIRE(ctx && tree, ATR_ERR_INVALID_ARG, "atr_optimize_atrbvh: NULL argument");
    ATR_REQUIRE(tsize >= 3 && tsize <= kMaxTreelet, ATR_ERR_UNSUPPORTED,
                "atr_optimize_atrbvh: treelet size %d outside [3, %d]", tsize, kMaxTreelet);
    ATR_REQUIRE(iterations >= 0 && iterations <= 24, ATR_ERR_INVALID_ARG, "atr_optimize_atrbvh: iterations %d",
                iterations);
    const uint32_t n = tree->n;
    TreeRefs g{n, tree->parent, tree->left, tree->right, tree->bmin, tree->bmax, tree->area, nullptr};
    Segs segs{nullptr, nullptr, 1u, n};
    return atrbvh_run(ctx, g, segs, 2 * (size_t)n - 1, tsize, iterations, nullptr, nullptr, ci, ct);
}
