// Compact2 traversal layout with Woop triangles, built on the device.
//
// Byte-identical to the reference's host conversion
// gpu-ray-traversal/src/rt/cuda/CudaBVH.cpp:469-574 (createCompact for a
// collapsed tree) and :579-600 (woopifyTri), which walks the tree with a LIFO
// stack: popping node X allots node records to X's inner children (left, then
// right) and appends the Woop triangles of X's leaf children (left, then
// right, each followed by a 0x80000000 terminator).  Nodes are therefore
// popped in right-first preorder.  Here:
//   1. bottom-up: per node, inner-node count of its subtree I, its number of
//      inner children, and the Woop entries of its leaf children;
//   2. pointer jumping over inner nodes: pop rank
//        rank(X) = sum over the path of 1 + [X' is a left child] * I(sibling),
//      depth, and whether a leaf of the collapsed tree lies above (unreached);
//   3. scatter by rank, two exclusive scans -> node slot and Woop offset;
//   4. one thread per reachable inner node writes its 64-byte record and its
//      leaf children's Woop triangles.
// The Woop transform restates FW::MatrixBase::inverted
// (gpu-ray-traversal/src/framework/base/Math.hpp:961-983, 3x3 determinant
// :934-939) with round-to-nearest operations in the reference's order.

#include "common.cuh"
#include "internal.h"

namespace atr {

int exclusive_scan_u32(atr_ctx* ctx, const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* d_total);

namespace {

constexpr int kJumpRounds = 8;  // enough for depth < 256; more rounds run if needed

struct FlatRefs {
    uint32_t n;
    const int32_t* parent;
    const int32_t* left;
    const int32_t* right;
    const int32_t* data;
    const int32_t* count;
    const float4* bmin;
    const float4* bmax;
    const int32_t* tri;
};

__device__ __forceinline__ bool c_leaf(const FlatRefs& t, int x) { return t.data[x] >= 0; }
__device__ __forceinline__ uint32_t woop_entries(const FlatRefs& t, int x) {
    const int c = t.count[x];
    return 3u * (uint32_t)(c > 1 ? c : 1) + 1u;
}

// Pass 1: inner-node counts, inner-children counts, Woop entries of leaf children.
__global__ void __launch_bounds__(256) k_flat_counts(FlatRefs t, uint32_t* __restrict__ icnt,
                                                      uint32_t* __restrict__ ic, uint32_t* __restrict__ tw,
                                                      uint32_t* __restrict__ counters) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.n) return;
    int cur = t.parent[(int)i + (int)t.n - 1];
    while (cur >= 0) {
        __threadfence();
        if (atomicAdd(&counters[cur], 1u) == 0u) return;
        __threadfence();
        const int l = t.left[cur], r = t.right[cur];
        const bool ll = c_leaf(t, l), rl = c_leaf(t, r);
        const uint32_t il = ll ? 0u : (uint32_t)ld_cg(reinterpret_cast<const int*>(icnt) + l);
        const uint32_t ir = rl ? 0u : (uint32_t)ld_cg(reinterpret_cast<const int*>(icnt) + r);
        icnt[cur] = c_leaf(t, cur) ? 0u : 1u + il + ir;
        ic[cur] = (ll ? 0u : 1u) + (rl ? 0u : 1u);
        tw[cur] = (ll ? woop_entries(t, l) : 0u) + (rl ? woop_entries(t, r) : 0u);
        cur = t.parent[cur];
    }
}

// Pointer-jumping initialisation over inner nodes.
__global__ void __launch_bounds__(256) k_flat_jump_init(FlatRefs t, const uint32_t* __restrict__ icnt,
                                                         int2* __restrict__ acc, int* __restrict__ jmp) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= t.n - 1) return;
    const int p = t.parent[x];
    if (p < 0) {
        acc[x] = make_int2(0, 0);
        jmp[x] = -1;
        return;
    }
    const bool is_left = t.left[p] == (int)x;
    const int sib = is_left ? t.right[p] : t.left[p];
    const int sib_inner = c_leaf(t, sib) ? 0 : (int)icnt[sib];
    const int val = 1 + (is_left ? sib_inner : 0);
    // .x: rank contribution, .y: depth in the low 16 bits and an
    // above-is-a-leaf flag in bit 30.
    const int blocked = c_leaf(t, (int)x) ? (1 << 30) : 0;
    acc[x] = make_int2(val, 1 | blocked);
    jmp[x] = p;
}

__global__ void __launch_bounds__(256) k_flat_jump(uint32_t m, const int2* __restrict__ acc_in,
                                                    const int* __restrict__ jmp_in, int2* __restrict__ acc_out,
                                                    int* __restrict__ jmp_out, uint32_t* __restrict__ pending) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= m) return;
    const int j = jmp_in[x];
    int2 a = acc_in[x];
    int nj = -1;
    if (j >= 0) {
        const int2 b = acc_in[j];
        a.x += b.x;
        a.y = ((a.y & 0xffff) + (b.y & 0xffff)) | ((a.y | b.y) & (1 << 30));
        nj = jmp_in[j];
        if (nj >= 0) *pending = 1u;
    }
    acc_out[x] = a;
    jmp_out[x] = nj;
}

// A node is reachable from the root through inner nodes when no node on its
// path (itself included) is a leaf of the collapsed tree.  The flag folded in
// above includes the node itself; inner nodes of the layout are exactly the
// reachable ones that are not leaves.
__global__ void __launch_bounds__(256) k_flat_scatter(FlatRefs t, const int2* __restrict__ acc,
                                                       const uint32_t* __restrict__ ic,
                                                       const uint32_t* __restrict__ tw,
                                                       uint32_t* __restrict__ ic_by_rank,
                                                       uint32_t* __restrict__ tw_by_rank,
                                                       int* __restrict__ max_depth) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= t.n - 1) return;
    const int2 a = acc[x];
    if (a.y & (1 << 30)) return;
    ic_by_rank[a.x] = ic[x];
    tw_by_rank[a.x] = tw[x];
    atomicMax(max_depth, (a.y & 0xffff) + 1);
}

__device__ __forceinline__ float det3(const float s[3][3]) {
    // v00*v11*v22 - v00*v12*v21 + v10*v21*v02 - v10*v22*v01 + v20*v01*v12 - v20*v02*v11
    float r = __fmul_rn(__fmul_rn(s[0][0], s[1][1]), s[2][2]);
    r = __fsub_rn(r, __fmul_rn(__fmul_rn(s[0][0], s[1][2]), s[2][1]));
    r = __fadd_rn(r, __fmul_rn(__fmul_rn(s[1][0], s[2][1]), s[0][2]));
    r = __fsub_rn(r, __fmul_rn(__fmul_rn(s[1][0], s[2][2]), s[0][1]));
    r = __fadd_rn(r, __fmul_rn(__fmul_rn(s[2][0], s[0][1]), s[1][2]));
    r = __fsub_rn(r, __fmul_rn(__fmul_rn(s[2][0], s[0][2]), s[1][1]));
    return r;
}

__device__ void woopify(const float4* __restrict__ v, int tri, float4* __restrict__ out) {
    const float4 a = v[3 * (size_t)tri], b = v[3 * (size_t)tri + 1], c = v[3 * (size_t)tri + 2];
    const float c0[3] = {__fsub_rn(a.x, c.x), __fsub_rn(a.y, c.y), __fsub_rn(a.z, c.z)};
    const float c1[3] = {__fsub_rn(b.x, c.x), __fsub_rn(b.y, c.y), __fsub_rn(b.z, c.z)};
    const float c2[3] = {__fsub_rn(__fmul_rn(c0[1], c1[2]), __fmul_rn(c0[2], c1[1])),
                         __fsub_rn(__fmul_rn(c0[2], c1[0]), __fmul_rn(c0[0], c1[2])),
                         __fsub_rn(__fmul_rn(c0[0], c1[1]), __fmul_rn(c0[1], c1[0]))};
    float M[4][4];
    for (int r = 0; r < 3; ++r) { M[r][0] = c0[r]; M[r][1] = c1[r]; M[r][2] = c2[r]; }
    M[0][3] = c.x; M[1][3] = c.y; M[2][3] = c.z;
    M[3][0] = 0.0f; M[3][1] = 0.0f; M[3][2] = 0.0f; M[3][3] = 1.0f;
    float R[3][4];  // rows 0..2 of the inverse are all the layout needs
    float d = 0.0f, si = 1.0f;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float sj = si;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float s[3][3];
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int l = 0; l < 3; ++l) s[k][l] = M[k < j ? k : k + 1][l < i ? l : l + 1];
            const float dd = __fmul_rn(det3(s), sj);
            if (i < 3) R[i][j] = dd;
            d = __fadd_rn(d, __fmul_rn(dd, M[j][i]));
            sj = -sj;
        }
        si = -si;
    }
    const float rd = d != 0.0f ? __fdiv_rn(1.0f, d) : 0.0f;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) R[i][j] = __fmul_rn(__fmul_rn(R[i][j], rd), 4.0f);
    out[0] = make_float4(R[2][0], R[2][1], R[2][2], -R[2][3]);
    out[1] = make_float4(R[0][0], R[0][1], R[0][2], R[0][3]);
    out[2] = make_float4(R[1][0], R[1][1], R[1][2], R[1][3]);
}

__global__ void __launch_bounds__(256) k_flat_slots(FlatRefs t, const int2* __restrict__ acc,
                                                     const uint32_t* __restrict__ ic,
                                                     const uint32_t* __restrict__ s_by_rank,
                                                     int* __restrict__ slot_of) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= t.n - 1) return;
    const int2 a = acc[x];
    if (a.y & (1 << 30)) return;
    if (t.parent[x] < 0) slot_of[x] = 0;
    const int l = t.left[x], r = t.right[x];
    const uint32_t base = 1u + s_by_rank[a.x];
    const bool li = !c_leaf(t, l), ri = !c_leaf(t, r);
    if (li) slot_of[l] = (int)base;
    if (ri) slot_of[r] = (int)(base + (li ? 1u : 0u));
}

__global__ void __launch_bounds__(128) k_flat_write(FlatRefs t, const float4* __restrict__ verts,
                                                     const int2* __restrict__ acc,
                                                     const uint32_t* __restrict__ w_by_rank,
                                                     const int* __restrict__ slot_of, int4* __restrict__ nodes,
                                                     float4* __restrict__ woop, int32_t* __restrict__ tri_index) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= t.n - 1) return;
    const int2 a = acc[x];
    if (a.y & (1 << 30)) return;
    const int ch[2] = {t.left[x], t.right[x]};
    int cref[2];
    uint32_t w = w_by_rank[a.x];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int c = ch[k];
        if (!c_leaf(t, c)) {
            cref[k] = 4 * slot_of[c];
            continue;
        }
        cref[k] = ~(int)w;
        const int cnt = t.count[c];
        const int d = t.data[c];
        const int m = cnt > 1 ? cnt : 1;
        for (int j = 0; j < m; ++j) {
            const int tri = cnt > 1 ? t.tri[d + j] : d;
            woopify(verts, tri, woop + w);
            tri_index[w] = tri;
            tri_index[w + 1] = 0;
            tri_index[w + 2] = 0;
            w += 3;
        }
        const float term = __int_as_float((int)0x80000000u);
        woop[w] = make_float4(term, term, term, term);
        tri_index[w] = 0;
        w += 1;
    }
    const float4 lm = t.bmin[ch[0]], lx = t.bmax[ch[0]], rm = t.bmin[ch[1]], rx = t.bmax[ch[1]];
    int4* dst = nodes + 4 * (size_t)slot_of[x];
    dst[0] = make_int4(__float_as_int(lm.x), __float_as_int(lx.x), __float_as_int(lm.y), __float_as_int(lx.y));
    dst[1] = make_int4(__float_as_int(rm.x), __float_as_int(rx.x), __float_as_int(rm.y), __float_as_int(rx.y));
    dst[2] = make_int4(__float_as_int(lm.z), __float_as_int(lx.z), __float_as_int(rm.z), __float_as_int(rx.z));
    dst[3] = make_int4(cref[0], cref[1], 0, 0);
}

}  // namespace
}  // namespace atr

using namespace atr;

extern "C" {

int atr_flatten_compact2(atr_ctx* ctx, const atr_collapsed* c, const atr_scene* scene, atr_compact** out) {
    ATR_REQUIRE(ctx && c && scene && out, ATR_ERR_INVALID_ARG, "atr_flatten_compact2: NULL argument");
    ATR_REQUIRE(c->n == scene->n, ATR_ERR_INVALID_ARG, "atr_flatten_compact2: tree/scene size mismatch");
    *out = nullptr;
    const uint32_t n = c->n;
    const uint32_t m = n - 1;  // inner nodes of the binary tree
    cudaStream_t s = ctx->stream;
    atr_compact* cp = new atr_compact();
    cp->ctx = ctx;
    // Upper bounds: every inner node, and 3 entries per triangle + 1 terminator per triangle.
    int st = ctx->alloc(reinterpret_cast<void**>(&cp->nodes), (size_t)m * 64);
    if (st == ATR_OK) st = ctx->alloc(reinterpret_cast<void**>(&cp->woop), (size_t)n * 4 * 16);
    if (st == ATR_OK) st = ctx->alloc(reinterpret_cast<void**>(&cp->tri_index), (size_t)n * 4 * 4);
    void* scratch = nullptr;
    const size_t bm = align256((size_t)m * 4), b2 = align256((size_t)m * 8);
    if (st == ATR_OK) st = ctx->alloc(&scratch, 7 * bm + 2 * b2 + 2 * bm + 256);
    if (st != ATR_OK) {
        ctx->release(scratch);
        atr_compact_destroy(cp);
        return st;
    }
    char* p = static_cast<char*>(scratch);
    uint32_t* icnt = reinterpret_cast<uint32_t*>(p); p += bm;
    uint32_t* ic = reinterpret_cast<uint32_t*>(p); p += bm;
    uint32_t* tw = reinterpret_cast<uint32_t*>(p); p += bm;
    uint32_t* counters = reinterpret_cast<uint32_t*>(p); p += bm;
    int* jmp0 = reinterpret_cast<int*>(p); p += bm;
    int* jmp1 = reinterpret_cast<int*>(p); p += bm;
    int* slot_of = reinterpret_cast<int*>(p); p += bm;
    int2* acc0 = reinterpret_cast<int2*>(p); p += b2;
    int2* acc1 = reinterpret_cast<int2*>(p); p += b2;
    uint32_t* ic_r = reinterpret_cast<uint32_t*>(p); p += bm;
    uint32_t* tw_r = reinterpret_cast<uint32_t*>(p); p += bm;
    uint32_t* flags = reinterpret_cast<uint32_t*>(p);  // [0] pending, [1] max depth, [2] totals
    FlatRefs t{n, c->parent, c->left, c->right, c->data, c->count, c->bmin, c->bmax, c->tri_indices};
    const unsigned gb = (n + 255) / 256, gm = (m + 255) / 256;
    cudaMemsetAsync(counters, 0, (size_t)m * 4, s);
    cudaMemsetAsync(ic_r, 0, 2 * bm, s);
    cudaMemsetAsync(flags, 0, 256, s);
    ctx->phase_begin("flatten");
    k_flat_counts<<<gb, 256, 0, s>>>(t, icnt, ic, tw, counters);
    k_flat_jump_init<<<gm, 256, 0, s>>>(t, icnt, acc0, jmp0);
    ctx->launches += 2;
    int2* ai = acc0; int2* ao = acc1;
    int* ji = jmp0; int* jo = jmp1;
    // 2^8 ancestors per 8 rounds; the flag of the last round of a block tells
    // whether any jump pointer is still live (depth >= 256 needs more rounds).
    for (int round = 0; round < 8 * kJumpRounds; ++round) {
        const bool check = round % kJumpRounds == kJumpRounds - 1;
        if (check) cudaMemsetAsync(flags, 0, 4, s);
        k_flat_jump<<<gm, 256, 0, s>>>(m, ai, ji, ao, jo, flags);
        ctx->launches += 1;
        std::swap(ai, ao);
        std::swap(ji, jo);
        if (check) {
            uint32_t pending = 0;
            cudaMemcpyAsync(&pending, flags, 4, cudaMemcpyDeviceToHost, s);
            cudaStreamSynchronize(s);
            if (!pending) break;
        }
    }
    k_flat_scatter<<<gm, 256, 0, s>>>(t, ai, ic, tw, ic_r, tw_r, reinterpret_cast<int*>(flags + 1));
    ctx->launches += 1;
    st = exclusive_scan_u32(ctx, ic_r, ic_r, m, flags + 2);
    if (st == ATR_OK) st = exclusive_scan_u32(ctx, tw_r, tw_r, m, flags + 3);
    if (st == ATR_OK) {
        k_flat_slots<<<gm, 256, 0, s>>>(t, ai, ic, ic_r, slot_of);
        k_flat_write<<<(m + 127) / 128, 128, 0, s>>>(t, scene->verts, ai, tw_r, slot_of, cp->nodes, cp->woop,
                                                      cp->tri_index);
        ctx->launches += 2;
        uint32_t h[4];
        cudaMemcpyAsync(h, flags, 16, cudaMemcpyDeviceToHost, s);
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(e, "flatten kernels", __FILE__, __LINE__);
        cp->num_nodes = (int64_t)h[2] + 1;
        cp->num_woop = (int64_t)h[3];
        cp->max_depth = (int32_t)h[1];
    }
    ctx->phase_end();
    ctx->release(scratch);
    if (st != ATR_OK) { atr_compact_destroy(cp); return st; }
    *out = cp;
    return ATR_OK;
}

int atr_compact_destroy(atr_compact* cp) {
    if (!cp) return ATR_OK;
    cp->ctx->release(cp->nodes);
    cp->ctx->release(cp->woop);
    cp->ctx->release(cp->tri_index);
    delete cp;
    return ATR_OK;
}

int atr_compact_download(atr_ctx* ctx, const atr_compact* cp, int32_t* nodes, float* woop, int32_t* tri) {
    ATR_REQUIRE(ctx && cp, ATR_ERR_INVALID_ARG, "atr_compact_download: NULL argument");
    cudaStream_t s = ctx->stream;
    if (nodes) ATR_CUDA(cudaMemcpyAsync(nodes, cp->nodes, (size_t)cp->num_nodes * 64, cudaMemcpyDeviceToHost, s));
    if (woop) ATR_CUDA(cudaMemcpyAsync(woop, cp->woop, (size_t)cp->num_woop * 16, cudaMemcpyDeviceToHost, s));
    if (tri) ATR_CUDA(cudaMemcpyAsync(tri, cp->tri_index, (size_t)cp->num_woop * 4, cudaMemcpyDeviceToHost, s));
    return atr_ctx_synchronize(ctx);
}

int atr_compact_view_get(const atr_compact* cp, atr_compact_view* v) {
    ATR_REQUIRE(cp && v, ATR_ERR_INVALID_ARG, "atr_compact_view_get: NULL argument");
    v->num_nodes = cp->num_nodes;
    v->num_woop = cp->num_woop;
    v->nodes = reinterpret_cast<int32_t*>(cp->nodes);
    v->woop = reinterpret_cast<float*>(cp->woop);
    v->tri_index = cp->tri_index;
    v->max_depth = cp->max_depth;
    return ATR_OK;
}

}  // extern "C"
