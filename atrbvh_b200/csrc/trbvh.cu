// TRBVH: treelet restructuring by dynamic programming over leaf subsets
// (Karras & Aila 2013), treelet size 7, on sm_100a.
//
// Semantics follow BVHRT-Core/src/TRBVH.cu:329-479 and TRBVHOptimizer.cpp:91-106:
// the same bottom-up pass as ATRBVH; per treelet the 128 subset boxes and
// areas, leaf costs = nodesSah, and for every subset S of 2..7 leaves
//   C(S) = min(ci*A(S) + min_P [C(P) + C(S\P)], ct*A(S)*T)
// with T the treelet's triangle count (:126-128).  Partitions are enumerated
// and reduced exactly as the reference does (sizes 2..5 one lane per subset,
// (p - delta) & S order; size 6 four lanes per subset; size 7 all 32 lanes; the
// lower lane keeps ties), so the chosen partitions match.  The rebuild
// (:222-327) proceeds round by round; in each round left children take
// internal nodes before right children, each in lane order, and a right
// child's nodesSah is written from the left partition's cost as in :309.
// Subset boxes, costs and masks live in shared memory (the reference keeps
// the boxes in a per-warp global scratch buffer).

#include "common.cuh"
#include "internal.h"
#include "treelet.cuh"

namespace atr {
namespace {

constexpr int kTrWarps = 4;
constexpr int kTr = 7;
constexpr int kSubsets = 1 << kTr;

struct TrShared {
    float mnx[kSubsets], mny[kSubsets], mnz[kSubsets];
    float mxx[kSubsets], mxy[kSubsets], mxz[kSubsets];
    float cost[kSubsets];
    int8_t mask[kSubsets];
    int stack_node[8];
    int stack_set[8];
};

// Subsets of 7 leaves grouped by size (2..5), each group in ascending order.
__constant__ uint8_t c_by_size[112];
__constant__ uint8_t c_size_start[5];  // start of sizes 2,3,4,5 and end

__device__ bool process_trbvh(const TreeRefs& t, int root, float root_sah, int tri_count, float ci, float ct,
                              TrShared& sm) {
    const int lane = threadIdx.x & 31;
    int internal_node;
    LeafSlot slot;
    if (!form_treelet(t, root, kTr, slot, internal_node)) return false;

    // Subset boxes and areas (calculateSubsetSurfaceAreas :37-98).
    float lmn[3][kTr], lmx[3][kTr];
#pragma unroll
    for (int i = 0; i < kTr; ++i) {
        lmn[0][i] = __shfl_sync(kFull, slot.mn.x, i);
        lmn[1][i] = __shfl_sync(kFull, slot.mn.y, i);
        lmn[2][i] = __shfl_sync(kFull, slot.mn.z, i);
        lmx[0][i] = __shfl_sync(kFull, slot.mx.x, i);
        lmx[1][i] = __shfl_sync(kFull, slot.mx.y, i);
        lmx[2][i] = __shfl_sync(kFull, slot.mx.z, i);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int s = lane * 4 + j;
        float a0 = FLT_MAX, a1 = FLT_MAX, a2 = FLT_MAX, b0 = -FLT_MAX, b1 = -FLT_MAX, b2 = -FLT_MAX;
#pragma unroll
        for (int i = 0; i < kTr; ++i) {
            if (s & (1 << i)) {
                a0 = fminf(lmn[0][i], a0); a1 = fminf(lmn[1][i], a1); a2 = fminf(lmn[2][i], a2);
                b0 = fmaxf(lmx[0][i], b0); b1 = fmaxf(lmx[1][i], b1); b2 = fmaxf(lmx[2][i], b2);
            }
        }
        sm.mnx[s] = a0; sm.mny[s] = a1; sm.mnz[s] = a2;
        sm.mxx[s] = b0; sm.mxy[s] = b1; sm.mxz[s] = b2;
        sm.cost[s] = box_area(a0, a1, a2, b0, b1, b2);
        sm.mask[s] = 0;
    }
    __syncwarp();
    if (lane < kTr) sm.cost[1 << lane] = slot.sah;
    __syncwarp();
    const float T = (float)tri_count;

    // Sizes 2..5 (processSchedule :100-134), one lane per subset.
    for (int g = 0; g < 4; ++g) {
        const int b = c_size_start[g], e = c_size_start[g + 1];
        for (int k0 = b; k0 < e; k0 += 32) {
            const int k = k0 + lane;
            float opt = FLT_MAX;
            int optp = 0;
            int s = 0;
            if (k < e) {
                s = c_by_size[k];
                const int delta = (s - 1) & s;
                int p = (-delta) & s;
                while (p != 0) {
                    const float c = __fadd_rn(sm.cost[p], sm.cost[p ^ s]);
                    if (c < opt) { opt = c; optp = p; }
                    p = (p - delta) & s;
                }
            }
            __syncwarp();
            if (k < e) {
                const float area = sm.cost[s];
                sm.cost[s] = fminf(__fadd_rn(__fmul_rn(ci, area), opt), __fmul_rn(__fmul_rn(ct, area), T));
                sm.mask[s] = (int8_t)optp;
            }
            __syncwarp();
        }
    }

    // Size 6: four lanes per subset, reduced within the group (processSubsets :136-189).
    {
        float opt = FLT_MAX;
        int optp = 0;
        const int k = lane >> 2;
        const int s = (kSubsets - 1) & ~(1 << k);
        if (lane < 4 * kTr) {
            const int left_mask = -(1 << max(k - 1, 0));
            int base = (lane & 3) + 1;
            const int np = (1 << (kTr - 2)) - 1;
            int p = (((base & left_mask) << 1) | (base & ~left_mask)) << 1;
            for (int j = lane & 3; j < np; j += 4) {
                const float c = __fadd_rn(sm.cost[p], sm.cost[p ^ s]);
                if (c < opt) { opt = c; optp = p; }
                base += 4;
                p = (((base & left_mask) << 1) | (base & ~left_mask)) << 1;
            }
        }
#pragma unroll
        for (int sh = 2; sh > 0; sh >>= 1) {
            const float ov = __shfl_down_sync(kFull, opt, sh);
            const int op = __shfl_down_sync(kFull, optp, sh);
            if (ov < opt) { opt = ov; optp = op; }
        }
        __syncwarp();
        if (lane < 4 * kTr && (lane & 3) == 0) {
            const float area = sm.cost[s];
            sm.cost[s] = fminf(__fadd_rn(__fmul_rn(ci, area), opt), __fmul_rn(__fmul_rn(ct, area), T));
            sm.mask[s] = (int8_t)optp;
        }
        __syncwarp();
    }
    // Size 7: all lanes, 32-lane reduction (:193-219).
    {
        const int s = kSubsets - 1;
        float opt = FLT_MAX;
        int optp = 0;
        int p = (lane + 1) * 2;
        for (int j = lane; j < (1 << (kTr - 1)) - 1; j += 32) {
            const float c = __fadd_rn(sm.cost[p], sm.cost[p ^ s]);
            if (c < opt) { opt = c; optp = p; }
            p += 64;
        }
#pragma unroll
        for (int sh = 16; sh > 0; sh >>= 1) {
            const float ov = __shfl_down_sync(kFull, opt, sh);
            const int op = __shfl_down_sync(kFull, optp, sh);
            if (ov < opt) { opt = ov; optp = op; }
        }
        __syncwarp();
        if (lane == 0) {
            const float area = sm.cost[s];
            sm.cost[s] = fminf(__fadd_rn(__fmul_rn(ci, area), opt), __fmul_rn(__fmul_rn(ct, area), T));
            sm.mask[s] = (int8_t)optp;
        }
        __syncwarp();
    }

    // Rebuild (updateTreelet :222-327).
    if (!(sm.cost[kSubsets - 1] < root_sah)) return true;
    int e_node = lane == 0 ? root : 0;
    int e_set = lane == 0 ? kSubsets - 1 : 0;
    int size = 1;
    int cur = 1;
    const uint32_t lt = lanemask_lt();
    while (size > 0) {
        const bool act = lane < size;
        const int P = act ? (int)sm.mask[e_set] : 0;
        const int Q = act ? (int)(int8_t)(P ^ e_set) : 0;
        // Left children.
        const bool li = act && __popc((unsigned)P) > 1;
        const unsigned lb = __ballot_sync(kFull, li);
        const int lslot = cur + __popc(lb & lt);
        const int lint = __shfl_sync(kFull, internal_node, li ? lslot : 0);
        const int lleaf = __shfl_sync(kFull, slot.node, act && !li ? __ffs(P) - 1 : 0);
        cur += __popc(lb);
        // Right children.
        const bool ri = act && __popc((unsigned)Q) > 1;
        const unsigned rb = __ballot_sync(kFull, ri);
        const int rslot = cur + __popc(rb & lt);
        const int rint = __shfl_sync(kFull, internal_node, ri ? rslot : 0);
        const int rleaf = __shfl_sync(kFull, slot.node, act && !ri ? __ffs(Q) - 1 : 0);
        cur += __popc(rb);
        __syncwarp();
        if (act) {
            const int lc = li ? lint : lleaf;
            const int rc = ri ? rint : rleaf;
            t.left[e_node] = lc;
            t.parent[lc] = e_node;
            t.right[e_node] = rc;
            t.parent[rc] = e_node;
            if (li) {
                const float4 mn = make_float4(sm.mnx[P], sm.mny[P], sm.mnz[P], 0.0f);
                const float4 mx = make_float4(sm.mxx[P], sm.mxy[P], sm.mxz[P], 0.0f);
                t.bmin[lc] = mn;
                t.bmax[lc] = mx;
                t.area[lc] = box_area(mn, mx);
                t.nsah[lc] = sm.cost[P];
                const int pos = __popc(lb & lt);
                sm.stack_node[pos] = lc;
                sm.stack_set[pos] = P;
            }
            if (ri) {
                const float4 mn = make_float4(sm.mnx[Q], sm.mny[Q], sm.mnz[Q], 0.0f);
                const float4 mx = make_float4(sm.mxx[Q], sm.mxy[Q], sm.mxz[Q], 0.0f);
                t.bmin[rc] = mn;
                t.bmax[rc] = mx;
                t.area[rc] = box_area(mn, mx);
                t.nsah[rc] = sm.cost[P];
                const int pos = __popc(lb) + __popc(rb & lt);
                sm.stack_node[pos] = rc;
                sm.stack_set[pos] = Q;
            }
        }
        __syncwarp();
        size = __popc(lb) + __popc(rb);
        if (lane < size) {
            e_node = sm.stack_node[lane];
            e_set = sm.stack_set[lane];
        }
        __syncwarp();
    }
    return true;
}

__global__ void __launch_bounds__(kTrWarps * 32) k_trbvh(TreeRefs g, Segs segs, int32_t* __restrict__ subtree,
                                                         uint32_t* __restrict__ counters,
                                                         const uint8_t* __restrict__ seg_iters, int iteration,
                                                         float ci, float ct, uint32_t* err) {
    __shared__ TrShared s_tr[kTrWarps];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    int cur = -1, base = 0, cbase = 0;
    uint32_t nm = 2;
    if (i < segs.n) {
        const uint32_t m = segs.seg_of_tri(i);
        const uint32_t s0 = segs.tri_begin(m);
        nm = segs.tri_end(m) - s0;
        base = segs.node_base(m);
        cbase = segs.inner_base(m);
        if (!seg_iters || iteration < (int)seg_iters[m]) {
            const int leaf = base + (int)(i - s0) + (int)nm - 1;
            subtree[leaf] = 1;
            g.nsah[leaf] = __fmul_rn(ct, g.area[leaf]);
            cur = g.parent[leaf];
        }
    }
    const int gamma = kTr << iteration;
    while (__any_sync(kFull, cur >= 0)) {
        bool second = false;
        if (cur >= 0) {
            fence_acq_rel_gpu();
            if (atomicAdd(&counters[cbase + cur], 1u) == 0u) cur = -1;
            else { second = true; fence_acq_rel_gpu(); }
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
            const int rcnt = __shfl_sync(kFull, cnt, rl);
            const int rbase = __shfl_sync(kFull, base, rl);
            const uint32_t rn = __shfl_sync(kFull, nm, rl);
            if (!process_trbvh(rebase(g, rbase, rn), root, rsah, rcnt, ci, ct, s_tr[w]) && lane == 0)
                set_error_bits(err, kErrTreeletClimb);
            vote &= vote - 1;
        }
        if (cur >= 0) cur = ld_cg(g.parent + base + cur);
    }
}

bool g_tables_ready = false;

int upload_tables() {
    if (g_tables_ready) return ATR_OK;
    uint8_t by[112];
    uint8_t start[5];
    int k = 0;
    for (int size = 2; size <= 5; ++size) {
        start[size - 2] = (uint8_t)k;
        for (int s = 1; s < kSubsets; ++s)
            if (__builtin_popcount(s) == size) by[k++] = (uint8_t)s;
    }
    start[4] = (uint8_t)k;
    ATR_CUDA(cudaMemcpyToSymbol(c_by_size, by, sizeof(by)));
    ATR_CUDA(cudaMemcpyToSymbol(c_size_start, start, sizeof(start)));
    g_tables_ready = true;
    return ATR_OK;
}

}  // namespace

// TRBVH (treelet 7) over every mesh of `segs`; seg_iters optionally gives
// each mesh its own iteration count (`iterations` is then their maximum).
int trbvh_run(atr_ctx* ctx, const TreeRefs& g_in, const Segs& segs, size_t total_nodes, int iterations,
              const uint8_t* seg_iters, float ci, float ct) {
    if (iterations <= 0) return ATR_OK;
    ATR_TRY(upload_tables());
    const size_t inner = segs.n - segs.count;
    void* scratch = nullptr;
    const size_t b = align256(total_nodes * 4);
    ATR_TRY(ctx->alloc(&scratch, 2 * b + align256(inner * 4)));
    char* p = static_cast<char*>(scratch);
    int32_t* subtree = reinterpret_cast<int32_t*>(p);
    TreeRefs g = g_in;
    g.nsah = reinterpret_cast<float*>(p + b);
    uint32_t* counters = reinterpret_cast<uint32_t*>(p + 2 * b);
    const int threads = kTrWarps * 32;
    const uint32_t blocks = (segs.n + threads - 1) / threads;
    ctx->phase_begin("trbvh");
    for (int it = 0; it < iterations; ++it) {
        cudaMemsetAsync(counters, 0, inner * 4, ctx->stream);
        k_trbvh<<<blocks, threads, 0, ctx->stream>>>(g, segs, subtree, counters, seg_iters, it, ci, ct,
                                                     ctx->d_error);
    }
    ctx->phase_end();
    ctx->launches += iterations;
    cudaError_t e = cudaGetLastError();
    ctx->release(scratch);
    if (e != cudaSuccess) return cuda_fail(e, "k_trbvh launch", __FILE__, __LINE__);
    return ATR_OK;
}

}  // namespace atr

using namespace atr;

extern "C" int atr_optimize_trbvh(atr_ctx* ctx, atr_tree* tree, int tsize, int iterations, float ci, float ct) {
    ATR_REQUIRE(ctx && tree, ATR_ERR_INVALID_ARG, "atr_optimize_trbvh: NULL argument");
    ATR_REQUIRE(tsize == kTr, ATR_ERR_UNSUPPORTED,
                "atr_optimize_trbvh: treelet size %d unsupported (the reference's subset kernel covers 7)", tsize);
    ATR_REQUIRE(iterations >= 0 && iterations <= 24, ATR_ERR_INVALID_ARG, "atr_optimize_trbvh: iterations %d",
                iterations);
    const uint32_t n = tree->n;
    TreeRefs g{n, tree->parent, tree->left, tree->right, tree->bmin, tree->bmax, tree->area, nullptr};
    Segs segs{nullptr, nullptr, 1u, n};
    tree->karras = false;
    tree_topology_changed(tree);
    ctx->release(tree->prepass_block);
    tree->prepass_block = nullptr;
    tree->prepass = BuildPrepass{};
    return trbvh_run(ctx, g, segs, 2 * (size_t)n - 1, iterations, nullptr, ci, ct);
}
