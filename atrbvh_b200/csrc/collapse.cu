// Leaf collapse (BVHRT-Core/src/TreeCollapser.cu:13-285, BVHTreeCollapser.cpp:21-93).
//
// The collapsed tree starts as a copy of the tree (TreeCollapser.cu:13-30),
// made inside pass 1: each leaf's thread copies its leaf, and the first of
// the two threads reaching an internal node -- which stops there -- copies
// that node.  Pass 1 (bottom-up, one thread per leaf, second arrival
// continues) computes, per
// node: triangle count, SAH cost (ci*A + cL + cR, or ct*A*count when that is
// cheaper -- :47-84), the collapse flag, and whether a climbing thread of the
// reference's emission kernel (:173-237) would pass the node upward.  The reference emits, at every
// node reached by two such threads that is not collapsed, each child holding
// more than one triangle as a multi-triangle leaf; pass 1 records those
// children.  A scan gives their list offsets in node order (the reference
// takes them from an atomicAdd, so its offsets vary between runs while the
// lists themselves do not).  Pass 2 writes each triangle at its rank in the
// right-first stack order of writeSubtreeLeavesNonrecursive (:95-137): the
// number of leaves in right subtrees hanging off its path below the emitted
// node.

#include "common.cuh"
#include "internal.h"

namespace atr {

int exclusive_scan_u32(atr_ctx* ctx, const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* d_total);

namespace {

struct CollapseRefs {
    uint32_t n;
    const float* area;
    const int32_t* parent;
    const int32_t* left;
    const int32_t* right;
    const int32_t* data;
    const float4* bmin;
    const float4* bmax;
    int32_t* c_parent;
    int32_t* c_left;
    int32_t* c_right;
    int32_t* c_data;
    int32_t* c_count;
    float4* c_bmin;
    float4* c_bmax;
    // Per node: (SAH cost bits, triangle count << 1 | pass flag), one 8-byte
    // record so a climbing thread reads each child with one load.
    int2* rec;
    uint32_t* emit_cnt;
    // False when the collapsed tree shares the source tree's links and boxes
    // (a collapse leaves them as they are): only data and counts are written.
    bool copy;
};

// Segmented: thread i starts at the i-th leaf of the batch; node arrays are
// addressed from the mesh's first node (local indices); each mesh's lists
// live in its own slice [tri_begin, tri_end) of tri_indices.  A node's area
// is its box's surface area (the tree's area array).
//
// A child's record travels to its parent through the parent's 64-bit slot:
// the first arrival exchanges its record in and stops, the second takes the
// sibling's record out of the exchange.  Nothing else is read that another
// thread of this pass writes, so the exchanges need no ordering, and the next
// node's links are loaded while the exchange is in flight.  A record is never
// zero (its count is at least one); zero marks an empty slot.
__device__ __forceinline__ unsigned long long pack_rec(int2 v) {
    return (unsigned long long)(uint32_t)v.x | ((unsigned long long)(uint32_t)v.y << 32);
}

__global__ void __launch_bounds__(256) k_collapse_cost(CollapseRefs g, Segs segs,
                                                        unsigned long long* __restrict__ slots, float ci, float ct,
                                                        int max_leaf) {
    const uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= segs.n) return;
    const uint32_t m = segs.seg_of_tri(gi);
    const uint32_t s0 = segs.tri_begin(m);
    const uint32_t n = segs.tri_end(m) - s0;
    const int nb = segs.node_base(m);
    unsigned long long* const slot = slots + segs.inner_base(m);
    int ch = (int)(gi - s0) + (int)n - 1;
    int cur = g.parent[nb + ch];
    int2 mine = make_int2(__float_as_int(__fmul_rn(ct, g.area[nb + ch])), (1 << 1) | 1);
    g.c_count[nb + ch] = 1;
    g.rec[nb + ch] = mine;
    // The leaf's copy (data >= 0, no children).
    g.c_data[nb + ch] = g.data[nb + ch];
    if (g.copy) {
        g.c_parent[nb + ch] = cur;
        g.c_left[nb + ch] = g.left[nb + ch];
        g.c_right[nb + ch] = g.right[nb + ch];
        g.c_bmin[nb + ch] = g.bmin[nb + ch];
        g.c_bmax[nb + ch] = g.bmax[nb + ch];
    }
    if (cur < 0) return;
    int l = g.left[nb + cur], r = g.right[nb + cur], up = g.parent[nb + cur];
    float a = g.area[nb + cur];
    while (true) {
        int nl = 0, nr = 0, nup = -1;
        float na = 0.0f;
        if (up >= 0) {
            nl = g.left[nb + up];
            nr = g.right[nb + up];
            nup = g.parent[nb + up];
            na = g.area[nb + up];
        }
        const unsigned long long other = atomicExch(slot + cur, pack_rec(mine));
        if (other == 0ull) {
            // First of the two children: the node's copy, then stop.
            const int x = nb + cur;
            g.c_data[x] = g.data[x];
            if (g.copy) {
                g.c_parent[x] = up;
                g.c_left[x] = l;
                g.c_right[x] = r;
                g.c_bmin[x] = g.bmin[x];
                g.c_bmax[x] = g.bmax[x];
            }
            return;
        }
        const int2 sib = make_int2((int)(uint32_t)other, (int)(uint32_t)(other >> 32));
        const bool from_left = ch == l;
        const int2 el = from_left ? mine : sib, er = from_left ? sib : mine;
        const int cl = el.y >> 1, cr = er.y >> 1;
        const float kl = __int_as_float(el.x), kr = __int_as_float(er.x);
        const int pl = el.y & 1, pr = er.y & 1;
        const int cnt = cl + cr;
        float c = __fadd_rn(__fadd_rn(__fmul_rn(ci, a), kl), kr);
        const float leaf_cost = __fmul_rn(__fmul_rn(ct, a), (float)cnt);
        const bool col = leaf_cost < c && (max_leaf <= 0 || cnt <= max_leaf);
        if (col) c = leaf_cost;
        const bool reached = pl && pr;
        const int x = nb + cur;
        if (reached && !col) {
            if (cl > 1) g.emit_cnt[nb + l] = (uint32_t)cl;
            if (cr > 1) g.emit_cnt[nb + r] = (uint32_t)cr;
        }
        mine = make_int2(__float_as_int(c), (cnt << 1) | (reached && col ? 1 : 0));
        g.c_count[x] = cnt;
        g.rec[x] = mine;
        if (up < 0) return;
        ch = cur;
        cur = up;
        l = nl;
        r = nr;
        up = nup;
        a = na;
    }
}

__global__ void __launch_bounds__(256) k_collapse_emit(CollapseRefs g, Segs segs, const uint32_t* __restrict__ offsets,
                                                        int32_t* __restrict__ tri_indices) {
    const uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= segs.n) return;
    const uint32_t m = segs.seg_of_tri(gi);
    const uint32_t s0 = segs.tri_begin(m);
    const uint32_t n = segs.tri_end(m) - s0;
    const int nb = segs.node_base(m);
    const int leaf = (int)(gi - s0) + (int)n - 1;
    int ch = leaf, a = g.parent[nb + leaf], top = -1;
    uint32_t rank = 0;
    while (a >= 0 && (g.rec[nb + a].y & 1)) {
        if (g.left[nb + a] == ch) rank += (uint32_t)g.c_count[nb + g.right[nb + a]];
        top = a;
        ch = a;
        a = g.parent[nb + a];
    }
    if (top < 0 || g.emit_cnt[nb + top] == 0) return;
    const uint32_t off = offsets[nb + top] - offsets[nb];  // local to the mesh's list slice
    tri_indices[s0 + off + rank] = g.data[nb + leaf];
    if (rank == 0) g.c_data[nb + top] = (int32_t)off;
}

__global__ void k_sah_parts(Segs segs, const int2* __restrict__ rec, const float* __restrict__ area,
                            float* __restrict__ out) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= segs.count) return;
    const int nb = segs.node_base(m);
    out[2 * m] = __int_as_float(rec[nb].x);
    out[2 * m + 1] = area[nb];
}

}  // namespace

int collapsed_alloc(atr_ctx* ctx, uint32_t n, atr_collapsed** out) {
    const size_t nn = 2 * (size_t)n - 1;
    const size_t b4 = align256(nn * 4), b16 = align256(nn * 16);
    atr_collapsed* c = new atr_collapsed();
    c->ctx = ctx;
    c->n = n;
    int s = ctx->alloc(&c->block, 5 * b4 + 2 * b16 + align256((size_t)n * 4));
    if (s != ATR_OK) { delete c; return s; }
    char* p = static_cast<char*>(c->block);
    c->parent = reinterpret_cast<int32_t*>(p); p += b4;
    c->left = reinterpret_cast<int32_t*>(p); p += b4;
    c->right = reinterpret_cast<int32_t*>(p); p += b4;
    c->data = reinterpret_cast<int32_t*>(p); p += b4;
    c->count = reinterpret_cast<int32_t*>(p); p += b4;
    c->bmin = reinterpret_cast<float4*>(p); p += b16;
    c->bmax = reinterpret_cast<float4*>(p); p += b16;
    c->tri_indices = reinterpret_cast<int32_t*>(p);
    *out = c;
    return ATR_OK;
}

// A collapsed tree that shares `tree`'s links and boxes (parent, left, right,
// bmin, bmax: a collapse leaves them as they are) and owns only its data,
// counts and leaf lists -- for a holder of both that never changes the tree
// without collapsing again (a build plan).
int collapsed_alloc_sharing(atr_ctx* ctx, const atr_tree* tree, atr_collapsed** out) {
    const uint32_t n = tree->n;
    const size_t nn = 2 * (size_t)n - 1;
    const size_t b4 = align256(nn * 4);
    atr_collapsed* c = new atr_collapsed();
    c->ctx = ctx;
    c->n = n;
    int s = ctx->alloc(&c->block, 2 * b4 + align256((size_t)n * 4));
    if (s != ATR_OK) { delete c; return s; }
    char* p = static_cast<char*>(c->block);
    c->data = reinterpret_cast<int32_t*>(p); p += b4;
    c->count = reinterpret_cast<int32_t*>(p); p += b4;
    c->tri_indices = reinterpret_cast<int32_t*>(p);
    c->parent = tree->parent;
    c->left = tree->left;
    c->right = tree->right;
    c->bmin = tree->bmin;
    c->bmax = tree->bmax;
    *out = c;
    return ATR_OK;
}

// Collapse every mesh of segs (total_nodes = sum of 2n_m - 1).  src holds the
// optimised trees, dst the collapsed arrays; d_sah_parts (optional) receives
// cost[root] and area[root] of every mesh (2 floats per mesh).
int collapse_segs(atr_ctx* ctx, const Segs& segs, size_t total_nodes, const TreeOut& src, const CollapsedOut& dst,
                  float ci, float ct, int max_leaf, float* d_sah_parts) {
    const uint32_t n = segs.n;
    const size_t nn = total_nodes;
    void* scratch = nullptr;
    const size_t b4 = align256(nn * 4);
    const size_t inner = n - segs.count;
    ATR_TRY(ctx->alloc(&scratch, align256(nn * 8) + 2 * b4 + align256(inner * 4)));
    char* p = static_cast<char*>(scratch);
    int2* rec = reinterpret_cast<int2*>(p); p += align256(nn * 8);
    uint32_t* emit = reinterpret_cast<uint32_t*>(p); p += b4;
    uint32_t* offs = reinterpret_cast<uint32_t*>(p); p += b4;
    // The exchange slots (8 B per inner node, at most 4 B per node) are dead
    // once the cost pass ends, before the scan writes the list offsets.
    unsigned long long* slots = reinterpret_cast<unsigned long long*>(offs);
    cudaStream_t s = ctx->stream;
    // The climb reads a zero slot as "no sibling yet": a failed clear must stop here.
    cudaError_t me = cudaMemsetAsync(slots, 0, inner * 8, s);
    if (me == cudaSuccess) me = cudaMemsetAsync(emit, 0, nn * 4, s);
    if (me == cudaSuccess) me = cudaMemsetAsync(dst.tri_indices, 0xff, (size_t)n * 4, s);
    if (me != cudaSuccess) {
        ctx->release(scratch);
        return cuda_fail(me, "collapse scratch clear", __FILE__, __LINE__);
    }
    const bool shared = dst.parent == src.parent && dst.left == src.left && dst.right == src.right &&
                        dst.bmin == src.bmin && dst.bmax == src.bmax;
    CollapseRefs r{n,        src.area,  src.parent, src.left,  src.right, src.data, src.bmin, src.bmax,
                   dst.parent, dst.left, dst.right, dst.data, dst.count, dst.bmin, dst.bmax, rec,
                   emit,     !shared};
    const unsigned blocks = (n + 255) / 256;
    k_collapse_cost<<<blocks, 256, 0, s>>>(r, segs, slots, ci, ct, max_leaf);
    ctx->launches += 1;
    int st = exclusive_scan_u32(ctx, emit, offs, nn, nullptr);
    if (st == ATR_OK) {
        k_collapse_emit<<<blocks, 256, 0, s>>>(r, segs, offs, dst.tri_indices);
        ctx->launches += 1;
        if (d_sah_parts) {
            k_sah_parts<<<(segs.count + 255) / 256, 256, 0, s>>>(segs, rec, src.area, d_sah_parts);
            ctx->launches += 1;
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = cuda_fail(e, "collapse kernels", __FILE__, __LINE__);
    }
    ctx->release(scratch);
    return st;
}

int collapse_into(atr_ctx* ctx, const atr_tree* tree, float ci, float ct, int max_leaf, atr_collapsed* c,
                  float* d_sah_parts) {
    const Segs segs{nullptr, nullptr, 1u, tree->n};
    const TreeOut src{tree->parent, tree->left, tree->right, tree->data, tree->bmin, tree->bmax, tree->area};
    const CollapsedOut dst{c->parent, c->left, c->right, c->data, c->count, c->bmin, c->bmax, c->tri_indices};
    return collapse_segs(ctx, segs, 2 * (size_t)tree->n - 1, src, dst, ci, ct, max_leaf, d_sah_parts);
}

}  // namespace atr

using namespace atr;

extern "C" {

int atr_collapse(atr_ctx* ctx, const atr_tree* tree, float ci, float ct, int max_leaf, atr_collapsed** out,
                 float* sah) {
    ATR_REQUIRE(ctx && tree && out, ATR_ERR_INVALID_ARG, "atr_collapse: NULL argument");
    ATR_REQUIRE(max_leaf >= 0, ATR_ERR_INVALID_ARG, "atr_collapse: max_leaf %d < 0", max_leaf);
    *out = nullptr;
    atr_collapsed* c = nullptr;
    ATR_TRY(collapsed_alloc(ctx, tree->n, &c));
    float* parts = nullptr;
    int st = ATR_OK;
    if (sah) st = ctx->alloc(reinterpret_cast<void**>(&parts), 8);
    ctx->phase_begin("collapse");
    if (st == ATR_OK) st = collapse_into(ctx, tree, ci, ct, max_leaf, c, parts);
    ctx->phase_end();
    c->split = tree->split;
    if (st == ATR_OK && sah) {
        float h[2];
        cudaError_t e = cudaMemcpyAsync(h, parts, 8, cudaMemcpyDeviceToHost, ctx->stream);
        if (e != cudaSuccess) st = cuda_fail(e, "cudaMemcpyAsync(sah)", __FILE__, __LINE__);
        if (st == ATR_OK) st = atr_ctx_synchronize(ctx);
        if (st == ATR_OK) *sah = h[0] / h[1];
    }
    ctx->release(parts);
    if (st != ATR_OK) { atr_collapsed_destroy(c); return st; }
    *out = c;
    return ATR_OK;
}

int atr_collapsed_destroy(atr_collapsed* c) {
    if (!c) return ATR_OK;
    c->ctx->release(c->block);
    delete c;
    return ATR_OK;
}

int atr_collapsed_view_get(const atr_collapsed* c, atr_collapsed_view* v) {
    ATR_REQUIRE(c && v, ATR_ERR_INVALID_ARG, "atr_collapsed_view_get: NULL argument");
    v->num_triangles = c->n;
    v->root = 0;
    v->parent = c->parent;
    v->left = c->left;
    v->right = c->right;
    v->data = c->data;
    v->triangle_count = c->count;
    v->bbox_min = reinterpret_cast<float*>(c->bmin);
    v->bbox_max = reinterpret_cast<float*>(c->bmax);
    v->triangle_indices = c->tri_indices;
    return ATR_OK;
}

int atr_collapsed_download(atr_ctx* ctx, const atr_collapsed* c, int32_t* parent, int32_t* left, int32_t* right,
                           int32_t* data, int32_t* count, float* bmin, float* bmax, int32_t* tri) {
    ATR_REQUIRE(ctx && c, ATR_ERR_INVALID_ARG, "atr_collapsed_download: NULL argument");
    const size_t nn = 2 * (size_t)c->n - 1;
    cudaStream_t s = ctx->stream;
    if (parent) ATR_CUDA(cudaMemcpyAsync(parent, c->parent, nn * 4, cudaMemcpyDeviceToHost, s));
    if (left) ATR_CUDA(cudaMemcpyAsync(left, c->left, nn * 4, cudaMemcpyDeviceToHost, s));
    if (right) ATR_CUDA(cudaMemcpyAsync(right, c->right, nn * 4, cudaMemcpyDeviceToHost, s));
    if (data) ATR_CUDA(cudaMemcpyAsync(data, c->data, nn * 4, cudaMemcpyDeviceToHost, s));
    if (count) ATR_CUDA(cudaMemcpyAsync(count, c->count, nn * 4, cudaMemcpyDeviceToHost, s));
    if (bmin) ATR_CUDA(cudaMemcpyAsync(bmin, c->bmin, nn * 16, cudaMemcpyDeviceToHost, s));
    if (bmax) ATR_CUDA(cudaMemcpyAsync(bmax, c->bmax, nn * 16, cudaMemcpyDeviceToHost, s));
    if (tri) ATR_CUDA(cudaMemcpyAsync(tri, c->tri_indices, (size_t)c->n * 4, cudaMemcpyDeviceToHost, s));
    return atr_ctx_synchronize(ctx);
}

}  // extern "C"
