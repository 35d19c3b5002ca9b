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

constexpr int kPendingWord = 8;    // flags[8 + r * kPendingStride]: jumps left after round r (r < 34)
constexpr int kPendingStride = 8;  // one 32-byte sector per round
constexpr size_t kFlagBytes = 4 * (kPendingWord + 34 * kPendingStride);

struct FlatRefs {
    const int32_t* parent;
    const int32_t* left;
    const int32_t* right;
    const int32_t* data;
    const int32_t* count;
    const float4* bmin;
    const float4* bmax;
    const int32_t* tri;
};

// Segment view of thread gi: the mesh, its first node (nb), its first inner
// node (cb), its first triangle (s0), its triangle count (n) and the local
// index li of the leaf (and of the inner node) this thread owns.
struct SegPos {
    uint32_t m, s0, n, li;
    int nb, cb;
};
__device__ __forceinline__ SegPos seg_pos(const Segs& segs, uint32_t gi) {
    SegPos p;
    p.m = segs.seg_of_tri(gi);
    p.s0 = segs.tri_begin(p.m);
    p.n = segs.tri_end(p.m) - p.s0;
    p.li = gi - p.s0;
    p.nb = segs.node_base(p.m);
    p.cb = segs.inner_base(p.m);
    return p;
}

__device__ __forceinline__ bool c_leaf(const FlatRefs& t, int nb, int x) { return t.data[nb + x] >= 0; }
__device__ __forceinline__ uint32_t woop_entries(const FlatRefs& t, int nb, int x) {
    const int c = t.count[nb + x];
    return 3u * (uint32_t)(c > 1 ? c : 1) + 1u;
}

// Pass 1: per inner node, inner nodes in its subtree, inner children, Woop
// entries of its leaf children (inner arrays are indexed cb + local index).
// A child's inner-node count reaches its parent through the parent's 64-bit
// slot (bit 32 marks it present): the first arrival exchanges its count in
// and stops, the second takes the sibling's out of the exchange.  Nothing
// else read here is written by this pass, so the exchanges need no ordering,
// and the next node's links load while the exchange is in flight.
__global__ void __launch_bounds__(256) k_flat_counts(FlatRefs t, Segs segs, uint32_t* __restrict__ icnt,
                                                      uint32_t* __restrict__ ic, uint32_t* __restrict__ tw,
                                                      unsigned long long* __restrict__ slots) {
    const uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= segs.n) return;
    const SegPos q = seg_pos(segs, gi);
    int ch = (int)q.li + (int)q.n - 1;
    int cur = t.parent[q.nb + ch];
    if (cur < 0) return;
    uint32_t mine = 0u;  // inner nodes below ch counted by the parent (none under a leaf)
    int l = t.left[q.nb + cur], r = t.right[q.nb + cur], up = t.parent[q.nb + cur];
    bool cleaf = c_leaf(t, q.nb, cur);
    while (true) {
        int nl = 0, nr = 0, nup = -1;
        bool ncleaf = false;
        if (up >= 0) {
            nl = t.left[q.nb + up];
            nr = t.right[q.nb + up];
            nup = t.parent[q.nb + up];
            ncleaf = c_leaf(t, q.nb, up);
        }
        const bool ll = c_leaf(t, q.nb, l), rl = c_leaf(t, q.nb, r);
        const unsigned long long other = atomicExch(slots + q.cb + cur, (1ull << 32) | mine);
        if (other == 0ull) return;
        const uint32_t sib = (uint32_t)other;
        const bool from_left = ch == l;
        const uint32_t il = from_left ? mine : sib, ir = from_left ? sib : mine;
        const uint32_t v = cleaf ? 0u : 1u + il + ir;
        icnt[q.cb + cur] = v;
        ic[q.cb + cur] = (ll ? 0u : 1u) + (rl ? 0u : 1u);
        tw[q.cb + cur] = (ll ? woop_entries(t, q.nb, l) : 0u) + (rl ? woop_entries(t, q.nb, r) : 0u);
        if (up < 0) return;
        mine = v;
        ch = cur;
        cur = up;
        l = nl;
        r = nr;
        up = nup;
        cleaf = ncleaf;
    }
}

// Pointer-jumping initialisation; thread gi owns inner node li of its mesh.
// .x: pop-rank contribution; .y: depth in the low 16 bits, bit 30 set when a
// leaf of the collapsed tree lies on the path (the node itself included).
__global__ void __launch_bounds__(256) k_flat_jump_init(FlatRefs t, Segs segs, const uint32_t* __restrict__ icnt,
                                                         int2* __restrict__ acc, int* __restrict__ jmp) {
    const uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= segs.n) return;
    const SegPos q = seg_pos(segs, gi);
    if (q.li >= q.n - 1) return;
    const int x = (int)q.li;
    const int gx = q.cb + x;
    const int p = t.parent[q.nb + x];
    if (p < 0) {
        acc[gx] = make_int2(0, 0);
        jmp[gx] = -1;
        return;
    }
    const bool is_left = t.left[q.nb + p] == x;
    const int sib = is_left ? t.right[q.nb + p] : t.left[q.nb + p];
    const int sib_inner = c_leaf(t, q.nb, sib) ? 0 : (int)icnt[q.cb + sib];
    const int val = 1 + (is_left ? sib_inner : 0);
    const int blocked = c_leaf(t, q.nb, x) ? (1 << 30) : 0;
    acc[gx] = make_int2(val, 1 | blocked);
    jmp[gx] = q.cb + p;
}

// Round r of pointer jumping reads buffer r & 1 and writes buffer (r + 1) & 1;
// pending[r * kPendingStride] records whether any jump is left after it (one
// 32-byte sector per round, one store per block).  A round whose predecessor
// left none does nothing, except the first such round of odd index, which
// moves the finished sums into buffer 0: the host launches a fixed number of
// rounds and never waits, and the result is always in buffer 0.  A node whose
// jump ran out (-1) copies its sums into the other buffer once and marks both
// jump words -2; later rounds skip it.  Readers of its jump word see -1 or -2,
// both "no further ancestor".
__global__ void __launch_bounds__(256) k_flat_jump(uint32_t m, int round, const int2* __restrict__ acc_in,
                                                    int* jmp_in, int2* __restrict__ acc_out,
                                                    int* __restrict__ jmp_out, uint32_t* __restrict__ pending) {
    __shared__ int s_state;  // 0 jump, 1 idle, 2 idle and move buffer 1 to buffer 0
    __shared__ int s_any;
    if (threadIdx.x == 0) {
        int st = 0;
        if (round > 0 && pending[(round - 1) * kPendingStride] == 0u)
            st = (round & 1) && (round == 1 || pending[(round - 2) * kPendingStride] != 0u) ? 2 : 1;
        s_state = st;
        s_any = 0;
    }
    __syncthreads();
    const int st = s_state;
    if (st == 1) return;
    const uint32_t stride = gridDim.x * blockDim.x;
    bool any = false;
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < m; x += stride) {
        if (st == 2) {
            acc_out[x] = acc_in[x];
            continue;
        }
        const int j = jmp_in[x];
        if (j < 0) {
            if (j == -1) {
                acc_out[x] = acc_in[x];
                jmp_out[x] = -2;
                jmp_in[x] = -2;
            }
            continue;
        }
        int2 a = acc_in[x];
        const int2 b = acc_in[j];
        a.x += b.x;
        a.y = ((a.y & 0xffff) + (b.y & 0xffff)) | ((a.y | b.y) & (1 << 30));
        const int nj = jmp_in[j];
        acc_out[x] = a;
        jmp_out[x] = nj < 0 ? -1 : nj;
        any |= nj >= 0;
    }
    if (st != 0) return;
    if (any) s_any = 1;
    __syncthreads();
    if (threadIdx.x == 0 && s_any) pending[round * kPendingStride] = 1u;
}

// Inner nodes of the layout are the reachable ones (no collapsed-tree leaf on
// their path); scatter their inner-child counts and Woop sizes by pop rank.
__global__ void __launch_bounds__(256) k_flat_scatter(Segs segs, const int2* __restrict__ acc,
                                                       const uint32_t* __restrict__ ic,
                                                       const uint32_t* __restrict__ tw,
                                                       uint32_t* __restrict__ ic_by_rank,
                                                       uint32_t* __restrict__ tw_by_rank,
                                                       int* __restrict__ max_depth) {
    const uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x;
    int depth = 0;
    if (gi < segs.n) {
        const SegPos q = seg_pos(segs, gi);
        if (q.li < q.n - 1) {
            const int gx = q.cb + (int)q.li;
            const int2 a = acc[gx];
            if (!(a.y & (1 << 30))) {
                ic_by_rank[q.cb + a.x] = ic[gx];
                tw_by_rank[q.cb + a.x] = tw[gx];
                depth = (a.y & 0xffff) + 1;
            }
        }
    }
    // One atomic per warp on the shared maximum.
    depth = __reduce_max_sync(0xffffffffu, depth);
    if ((threadIdx.x & 31) == 0 && depth > 0) atomicMax(max_depth, depth);
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

__global__ void __launch_bounds__(256) k_flat_slots(FlatRefs t, Segs segs, const int2* __restrict__ acc,
                                                     const uint32_t* __restrict__ s_by_rank,
                                                     int* __restrict__ slot_of) {
    const uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= segs.n) return;
    const SegPos q = seg_pos(segs, gi);
    if (q.li >= q.n - 1) return;
    const int x = (int)q.li;
    const int2 a = acc[q.cb + x];
    if (a.y & (1 << 30)) return;
    if (t.parent[q.nb + x] < 0) slot_of[q.cb + x] = 0;
    const int l = t.left[q.nb + x], r = t.right[q.nb + x];
    const uint32_t base = 1u + s_by_rank[q.cb + a.x] - s_by_rank[q.cb];
    const bool li = !c_leaf(t, q.nb, l), ri = !c_leaf(t, q.nb, r);
    if (li) slot_of[q.cb + l] = (int)base;
    if (ri) slot_of[q.cb + r] = (int)(base + (li ? 1u : 0u));
}

// One thread per reachable inner node: its 64-byte record in the mesh's node
// slice (first node 4 * cb in float4 units), the terminators of its leaf
// children's Woop lists in the mesh's Woop slice (first entry 4 * s0).  The
// Woop triangles of a warp's leaf children are then spread over the warp's
// lanes (an exclusive scan of the nodes' triangle counts in shared memory,
// item u to the node whose range holds it), so a node with long leaf lists
// does not hold the warp while the others idle.
constexpr int kWriteThreads = 128;

__global__ void __launch_bounds__(kWriteThreads) k_flat_write(FlatRefs t, Segs segs, const float4* __restrict__ verts,
                                                     const int2* __restrict__ acc,
                                                     const uint32_t* __restrict__ w_by_rank,
                                                     const int* __restrict__ slot_of, int4* __restrict__ nodes,
                                                     float4* __restrict__ woop, int32_t* __restrict__ tri_index) {
    constexpr int W = kWriteThreads / 32;
    __shared__ uint32_t s_pre[W][32], s_n0[W][32], s_w[W][2][32], s_s0[W][32];
    __shared__ int32_t s_d[W][2][32];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t items[2] = {0u, 0u}, wk[2] = {0u, 0u};
    int32_t dk[2] = {0, 0};
    uint32_t s0 = 0;
    bool multi[2] = {false, false};
    if (gi < segs.n) {
        const SegPos q = seg_pos(segs, gi);
        s0 = q.s0;
        const int x = (int)q.li;
        const int2 a = q.li < q.n - 1 ? acc[q.cb + x] : make_int2(0, 1 << 30);
        if (!(a.y & (1 << 30))) {
            float4* mw = woop + 4 * (size_t)q.s0;
            int32_t* mt = tri_index + 4 * (size_t)q.s0;
            const int ch[2] = {t.left[q.nb + x], t.right[q.nb + x]};
            int cref[2];
            uint32_t w = w_by_rank[q.cb + a.x] - w_by_rank[q.cb];
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int c = ch[k];
                if (!c_leaf(t, q.nb, c)) {
                    cref[k] = 4 * slot_of[q.cb + c];
                    continue;
                }
                cref[k] = ~(int)w;
                const int cnt = t.count[q.nb + c];
                multi[k] = cnt > 1;
                items[k] = (uint32_t)(cnt > 1 ? cnt : 1);
                wk[k] = w;
                dk[k] = t.data[q.nb + c];
                w += 3u * items[k];
                const float term = __int_as_float((int)0x80000000u);
                mw[w] = make_float4(term, term, term, term);
                mt[w] = 0;
                w += 1;
            }
            const float4 lm = t.bmin[q.nb + ch[0]], lx = t.bmax[q.nb + ch[0]];
            const float4 rm = t.bmin[q.nb + ch[1]], rx = t.bmax[q.nb + ch[1]];
            int4* dst = nodes + 4 * ((size_t)q.cb + (size_t)slot_of[q.cb + x]);
            dst[0] = make_int4(__float_as_int(lm.x), __float_as_int(lx.x), __float_as_int(lm.y), __float_as_int(lx.y));
            dst[1] = make_int4(__float_as_int(rm.x), __float_as_int(rx.x), __float_as_int(rm.y), __float_as_int(rx.y));
            dst[2] = make_int4(__float_as_int(lm.z), __float_as_int(lx.z), __float_as_int(rm.z), __float_as_int(rx.z));
            dst[3] = make_int4(cref[0], cref[1], 0, 0);
        }
    }
    // Items of this lane: items[0] triangles of the left leaf child, then
    // items[1] of the right.
    const uint32_t mine = items[0] + items[1];
    uint32_t incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
    }
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    s_pre[wp][lane] = incl - mine;
    s_n0[wp][lane] = items[0];
    s_w[wp][0][lane] = wk[0];
    s_w[wp][1][lane] = wk[1];
    // A single-triangle leaf's data is the triangle (sign bit set here);
    // a list leaf's data is its list offset.
    s_d[wp][0][lane] = dk[0] | (multi[0] ? 0 : (int32_t)0x80000000);
    s_d[wp][1][lane] = dk[1] | (multi[1] ? 0 : (int32_t)0x80000000);
    s_s0[wp][lane] = s0;
    __syncwarp();
    for (uint32_t u = lane; u < total; u += 32) {
        // The node holding item u: the last lane whose range starts at or
        // before u (lanes without items share the next lane's start).
        int o = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1)
            if (s_pre[wp][o + step] <= u) o += step;
        const uint32_t loc = u - s_pre[wp][o];
        const int k = loc < s_n0[wp][o] ? 0 : 1;
        const uint32_t j = loc - (k ? s_n0[wp][o] : 0u);
        const int32_t dd = s_d[wp][k][o];
        const uint32_t ms0 = s_s0[wp][o];
        const int d = dd & 0x7fffffff;
        const int tri = dd >= 0 ? t.tri[ms0 + (uint32_t)d + j] : d;
        const uint32_t w = s_w[wp][k][o] + 3u * j;
        woopify(verts + 3 * (size_t)ms0, tri, woop + 4 * (size_t)ms0 + w);
        int32_t* mt = tri_index + 4 * (size_t)ms0;
        mt[w] = tri;
        mt[w + 1] = 0;
        mt[w + 2] = 0;
    }
}

// Per-mesh sizes: inner nodes = 1 + inner children, Woop entries.
__global__ void k_flat_sizes(Segs segs, const uint32_t* __restrict__ ic_scan, const uint32_t* __restrict__ tw_scan,
                             const uint32_t* __restrict__ totals, const int* __restrict__ max_depth,
                             int64_t* __restrict__ nodes_out, int64_t* __restrict__ woop_out,
                             int64_t* __restrict__ depth_out) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m == 0) *depth_out = *max_depth;
    if (m >= segs.count) return;
    const int cb = segs.inner_base(m);
    const bool last = m + 1 == segs.count;
    const uint32_t ic_end = last ? totals[0] : ic_scan[segs.inner_base(m + 1)];
    const uint32_t tw_end = last ? totals[1] : tw_scan[segs.inner_base(m + 1)];
    nodes_out[m] = 1 + (int64_t)(ic_end - ic_scan[cb]);
    woop_out[m] = (int64_t)(tw_end - tw_scan[cb]);
}

}  // namespace

// Compact2 layout of every mesh of segs into per-mesh slices of nodes (mesh m
// from node inner_base(m)), woop and tri_index (mesh m from entry 4 *
// tri_begin(m)).  d_sizes receives 2 * count + 1 int64: nodes per mesh, Woop
// entries per mesh, then the deepest inner level over all meshes.  Stream
// ordered: nothing here waits for the device.
int flatten_segs(atr_ctx* ctx, const Segs& segs, const CollapsedOut& c, const float4* verts, int4* nodes,
                 float4* woop, int32_t* tri_index, int64_t* d_sizes) {
    const uint32_t n = segs.n;
    const uint32_t m = n - segs.count;  // inner nodes over all meshes
    cudaStream_t s = ctx->stream;
    void* scratch = nullptr;
    const size_t bm = align256((size_t)m * 4), b2 = align256((size_t)m * 8);
    ATR_TRY(ctx->alloc(&scratch, 9 * bm + 2 * b2 + kFlagBytes));
    char* p = static_cast<char*>(scratch);
    uint32_t* icnt = reinterpret_cast<uint32_t*>(p); p += bm;
    uint32_t* ic = reinterpret_cast<uint32_t*>(p); p += bm;
    uint32_t* tw = reinterpret_cast<uint32_t*>(p); p += bm;
    p += bm;  // spare word per inner node: the scratch keeps its size (and its place in the pool)
    int* jmp0 = reinterpret_cast<int*>(p); p += bm;
    int* jmp1 = reinterpret_cast<int*>(p); p += bm;
    int* slot_of = reinterpret_cast<int*>(p); p += bm;
    int2* acc0 = reinterpret_cast<int2*>(p); p += b2;
    int2* acc1 = reinterpret_cast<int2*>(p); p += b2;
    uint32_t* ic_r = reinterpret_cast<uint32_t*>(p); p += bm;
    uint32_t* tw_r = reinterpret_cast<uint32_t*>(p); p += bm;
    uint32_t* flags = reinterpret_cast<uint32_t*>(p);  // [1] max depth, [2..3] totals, then pending
    FlatRefs t{c.parent, c.left, c.right, c.data, c.count, c.bmin, c.bmax, c.tri_indices};
    const unsigned gb = (n + 255) / 256, gm = (m + 255) / 256;
    // The exchange slots of pass 1 (8 B per inner node) live in acc0, which
    // k_flat_jump_init overwrites for every inner node afterwards.
    unsigned long long* const slots = reinterpret_cast<unsigned long long*>(acc0);
    // The count climb reads a zero slot as "no sibling yet": a failed clear must stop here.
    cudaError_t me = cudaMemsetAsync(slots, 0, (size_t)m * 8, s);
    if (me == cudaSuccess) me = cudaMemsetAsync(ic_r, 0, 2 * bm, s);
    if (me == cudaSuccess) me = cudaMemsetAsync(flags, 0, kFlagBytes, s);
    if (me != cudaSuccess) {
        ctx->release(scratch);
        return cuda_fail(me, "flatten scratch clear", __FILE__, __LINE__);
    }
    k_flat_counts<<<gb, 256, 0, s>>>(t, segs, icnt, ic, tw, slots);
    k_flat_jump_init<<<gb, 256, 0, s>>>(t, segs, icnt, acc0, jmp0);
    ctx->launches += 2;
    // Depth <= m, and after round r every jump spans 2^(r+1) ancestors, so the
    // last working round is below bits(m) and round bits(m) + 1 is idle.
    if (m > 0) {
        const int rounds = 34 - __builtin_clz(m);
        int2* acc[2] = {acc0, acc1};
        int* jmp[2] = {jmp0, jmp1};
        const unsigned gj = std::min(gm, (unsigned)ctx->num_sms * 8u);
        for (int r = 0; r < rounds; ++r)
            k_flat_jump<<<gj, 256, 0, s>>>(m, r, acc[r & 1], jmp[r & 1], acc[(r + 1) & 1], jmp[(r + 1) & 1],
                                           flags + kPendingWord);
        ctx->launches += rounds;
    }
    const int2* ai = acc0;
    k_flat_scatter<<<gb, 256, 0, s>>>(segs, ai, ic, tw, ic_r, tw_r, reinterpret_cast<int*>(flags + 1));
    ctx->launches += 1;
    int st = exclusive_scan_u32(ctx, ic_r, ic_r, m, flags + 2);
    if (st == ATR_OK) st = exclusive_scan_u32(ctx, tw_r, tw_r, m, flags + 3);
    if (st == ATR_OK) {
        k_flat_slots<<<gb, 256, 0, s>>>(t, segs, ai, ic_r, slot_of);
        k_flat_write<<<(n + kWriteThreads - 1) / kWriteThreads, kWriteThreads, 0, s>>>(t, segs, verts, ai, tw_r,
                                                                                       slot_of, nodes, woop, tri_index);
        k_flat_sizes<<<(segs.count + 255) / 256, 256, 0, s>>>(segs, ic_r, tw_r, flags + 2,
                                                             reinterpret_cast<const int*>(flags + 1), d_sizes,
                                                             d_sizes + segs.count, d_sizes + 2 * segs.count);
        ctx->launches += 3;
    }
    ctx->release(scratch);
    return st;
}

}  // namespace atr

using namespace atr;

extern "C" {

int atr_flatten_compact2(atr_ctx* ctx, const atr_collapsed* c, const atr_scene* scene, atr_compact** out) {
    ATR_REQUIRE(ctx && c && scene && out, ATR_ERR_INVALID_ARG, "atr_flatten_compact2: NULL argument");
    ATR_REQUIRE(c->n == scene->n || c->split, ATR_ERR_INVALID_ARG,
                "atr_flatten_compact2: tree/scene size mismatch");
    *out = nullptr;
    const uint32_t n = c->n;
    atr_compact* cp = new atr_compact();
    cp->ctx = ctx;
    // Upper bounds: every inner node, and 3 entries per triangle + 1 terminator per triangle.
    int st = ctx->alloc(reinterpret_cast<void**>(&cp->nodes), (size_t)(n - 1) * 64);
    if (st == ATR_OK) st = ctx->alloc(reinterpret_cast<void**>(&cp->woop), (size_t)n * 4 * 16);
    if (st == ATR_OK) st = ctx->alloc(reinterpret_cast<void**>(&cp->tri_index), (size_t)n * 4 * 4);
    int64_t* sizes = nullptr;
    if (st == ATR_OK) st = ctx->alloc(reinterpret_cast<void**>(&sizes), 24);
    if (st != ATR_OK) {
        ctx->release(sizes);
        atr_compact_destroy(cp);
        return st;
    }
    const Segs segs{nullptr, nullptr, 1u, n};
    const CollapsedOut co{c->parent, c->left, c->right, c->data, c->count, c->bmin, c->bmax, c->tri_indices};
    ctx->phase_begin("flatten");
    st = flatten_segs(ctx, segs, co, scene->verts, cp->nodes, cp->woop, cp->tri_index, sizes);
    ctx->phase_end();
    if (st == ATR_OK) {
        int64_t h[3];
        cudaError_t e = cudaMemcpyAsync(h, sizes, 24, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) st = cuda_fail(e, "flatten kernels", __FILE__, __LINE__);
        cp->num_nodes = h[0];
        cp->num_woop = h[1];
        cp->max_depth = (int32_t)h[2];
    }
    ctx->release(sizes);
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
