// ORACLE -- test infrastructure only.
//
// CPU restatement of the reference's ATRBVH build-and-traverse path, used as the
// parity checker by tests/, __graft_entry__.smoke() and the CPU-baseline leg of
// bench.py.  Nothing in the product links or calls this file.
//
// Each function cites the reference file:line it restates (paths relative to the
// reference project root).  Floating point follows the reference's arithmetic
// order with no contraction (build with -ffp-contract=off, no -ffast-math):
//   * surface area 2*(x*y + x*z + y*z)      BVHRT-Core/src/Commons.cuh:99-125
//   * union surface area                    BVHRT-Core/src/Commons.cuh:156-164
//   * Woop 4x4 cofactor inverse             gpu-ray-traversal/src/framework/base/Math.hpp:902-983
// The traversal arithmetic is pinned to the explicit FMA policy that the product
// kernel also uses (slab = fma(bound, idir, -orig*idir); Woop dot products as
// FMA chains; IEEE division for 1/d).  The reference compiles its traversal
// with -use_fast_math (gpu-ray-traversal/src/rt/cuda/CudaTracer.cpp:40), whose
// approximate reciprocal is not restated here.
//
// Parallel (OpenMP) entry points give the timed host-core baseline; they produce
// results identical to the single-thread entry points (post-order task
// parallelism over disjoint subtrees; see the per-function notes).

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct F4 { float x, y, z, w; };

inline bool is_internal(int idx, uint32_t n) { return (uint32_t)idx < n - 1u; }

// BVHRT-Core/src/Commons.cuh:99-107 (float3/float4 overloads are identical)
inline float box_area(float mnx, float mny, float mnz, float mxx, float mxy, float mxz) {
    float sx = mxx - mnx, sy = mxy - mny, sz = mxz - mnz;
    return 2.0f * (sx * sy + sx * sz + sy * sz);
}
inline float box_area(const F4& mn, const F4& mx) {
    return box_area(mn.x, mn.y, mn.z, mx.x, mx.y, mx.z);
}

// BVHRT-Core/src/Commons.cuh:156-164: max(maxA,maxB) - min(minA,minB) per axis.
inline float union_area(const float* mnA, const float* mxA, const float* mnB, const float* mxB) {
    float sx = fmaxf(mxA[0], mxB[0]) - fminf(mnA[0], mnB[0]);
    float sy = fmaxf(mxA[1], mxB[1]) - fminf(mnA[1], mnB[1]);
    float sz = fmaxf(mxA[2], mxB[2]) - fminf(mnA[2], mnB[2]);
    return 2.0f * (sx * sy + sx * sz + sy * sz);
}

// BVHRT-Core/src/Commons.cuh:481-488
inline uint32_t expand_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

// BVHRT-Core/src/Commons.cuh:606-618 (restated with shifts and masks)
inline uint64_t expand_bits64(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}

// BVHRT-Core/src/LBVH.cu:14-40: centroid of the triangle's AABB.
inline void tri_centroid(const F4* v, uint32_t tri, float c[3]) {
    const F4& a = v[3 * (size_t)tri], &b = v[3 * (size_t)tri + 1], &d = v[3 * (size_t)tri + 2];
    float mnx = fminf(fminf(a.x, b.x), d.x), mxx = fmaxf(fmaxf(a.x, b.x), d.x);
    float mny = fminf(fminf(a.y, b.y), d.y), mxy = fmaxf(fmaxf(a.y, b.y), d.y);
    float mnz = fminf(fminf(a.z, b.z), d.z), mxz = fmaxf(fmaxf(a.z, b.z), d.z);
    c[0] = (mxx + mnx) * 0.5f;
    c[1] = (mxy + mny) * 0.5f;
    c[2] = (mxz + mnz) * 0.5f;
}

// BVHRT-Core/src/Commons.cuh:426-434 (normalize) + :497-510 (30-bit code)
inline uint32_t morton30(const float c[3], const float* bmin, const float* bmax) {
    uint32_t q[3];
    for (int k = 0; k < 3; ++k) {
        float nrm = (c[k] - bmin[k]) / (bmax[k] - bmin[k]);
        q[k] = expand_bits((uint32_t)fminf(fmaxf(nrm * 1024.0f, 0.0f), 1023.0f));
    }
    return q[0] * 4u + q[1] * 2u + q[2];
}

// BVHRT-Core/src/Commons.cuh:627-640 (63-bit code)
inline uint64_t morton63(const float c[3], const float* bmin, const float* bmax) {
    uint64_t q[3];
    for (int k = 0; k < 3; ++k) {
        float nrm = (c[k] - bmin[k]) / (bmax[k] - bmin[k]);
        q[k] = expand_bits64((uint64_t)fminf(fmaxf(nrm * 2097152.0f, 0.0f), 2097151.0f));
    }
    return q[0] * 4u + q[1] * 2u + q[2];
}

inline int clz32(uint32_t x) { return x ? __builtin_clz(x) : 32; }
inline int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }

// BVHRT-Core/src/LBVH.cu:163-201: common prefix with index tie-break; 0 out of range.
template <typename K> inline int lcp(const K* keys, uint32_t n, int i, int j, K ki);
template <> inline int lcp<uint32_t>(const uint32_t* keys, uint32_t n, int i, int j, uint32_t ki) {
    if (j < 0 || j >= (int)n) return 0;
    uint32_t kj = keys[j];
    if (ki == kj) return 32 + clz32((uint32_t)(i ^ j));
    return clz32(ki ^ kj);
}
template <> inline int lcp<uint64_t>(const uint64_t* keys, uint32_t n, int i, int j, uint64_t ki) {
    if (j < 0 || j >= (int)n) return 0;
    uint64_t kj = keys[j];
    if (ki == kj) return 64 + clz64((uint64_t)(uint32_t)(i ^ j));
    return clz64(ki ^ kj);
}

// BVHRT-Core/src/LBVH.cu:208-316: one internal node of the Karras radix tree.
template <typename K>
void karras_node(const K* keys, const uint32_t* sidx, uint32_t n, int i,
                 int32_t* parent, int32_t* left, int32_t* right, int32_t* data) {
    const K ki = keys[i];
    const int d1 = lcp(keys, n, i, i + 1, ki);
    const int d2 = lcp(keys, n, i, i - 1, ki);
    const int dir = (d1 - d2 > 0) - (d1 - d2 < 0);
    const int dmin = lcp(keys, n, i, i - dir, ki);
    int lmax = 128;
    while (lcp(keys, n, i, i + lmax * dir, ki) > dmin) lmax *= 4;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (lcp(keys, n, i, i + (l + t) * dir, ki) > dmin) l += t;
    const int j = i + l * dir;
    const int dnode = lcp(keys, n, i, j, ki);
    int s = 0;
    const int maxdiv = 1 << (32 - clz32((uint32_t)l));
    for (int div = 2; div <= maxdiv; div *= 2) {
        int t = (l + div - 1) / div;
        if (lcp(keys, n, i, i + (s + t) * dir, ki) > dnode) s += t;
    }
    const int split = i + s * dir + std::min(dir, 0);
    int li, ri;
    if (std::min(i, j) == split) { li = split + (int)n - 1; data[li] = (int32_t)sidx[split]; }
    else li = split;
    if (std::max(i, j) == split + 1) { ri = split + (int)n; data[ri] = (int32_t)sidx[split + 1]; }
    else ri = split + 1;
    right[i] = ri;
    left[i] = li;
    parent[li] = i;
    parent[ri] = i;
    data[i] = -1;
    if (i == 0) parent[0] = -1;
}

struct Tree {
    uint32_t n;
    int32_t *parent, *left, *right, *data;
    F4 *bmin, *bmax;
    float* area;
};

// Post-order over internal nodes with an explicit stack (left subtree first).
// visit(x) is called after both children of x were visited.  Children indices of
// x are read when x is first reached; visiting descendants never changes them.
template <typename Fn>
void post_order(const Tree& t, int root, Fn&& visit) {
    if (!is_internal(root, t.n)) return;
    std::vector<std::pair<int, int>> st;
    st.reserve(128);
    st.push_back({root, 0});
    while (!st.empty()) {
        auto& top = st.back();
        int x = top.first;
        if (top.second == 0) {
            top.second = 1;
            int r = t.right[x], l = t.left[x];
            if (is_internal(r, t.n)) st.push_back({r, 0});
            if (is_internal(l, t.n)) st.push_back({l, 0});
        } else {
            st.pop_back();
            visit(x);
        }
    }
}

// Task-parallel post-order: subtrees below depth `par_depth` run sequentially.
template <typename Fn>
void post_order_par(const Tree& t, int x, int depth, int par_depth, Fn& visit) {
    if (!is_internal(x, t.n)) return;
    if (depth >= par_depth) { post_order(t, x, visit); return; }
    int l = t.left[x], r = t.right[x];
#ifdef _OPENMP
#pragma omp task shared(t, visit) firstprivate(l, depth, par_depth)
    post_order_par(t, l, depth + 1, par_depth, visit);
    post_order_par(t, r, depth + 1, par_depth, visit);
#pragma omp taskwait
#else
    post_order_par(t, l, depth + 1, par_depth, visit);
    post_order_par(t, r, depth + 1, par_depth, visit);
#endif
    visit(x);
}

template <typename Fn>
void run_post_order(const Tree& t, int threads, Fn& visit) {
#ifdef _OPENMP
    if (threads > 1) {
#pragma omp parallel num_threads(threads)
#pragma omp single
        post_order_par(t, 0, 0, 14, visit);
        return;
    }
#endif
    (void)threads;
    post_order(t, 0, visit);
}

// Shuffle-down tree reduction over lanes [0, count) as written in
// BVHRT-Core/src/Treelet.cuh:23-39 and AgglomerativeTreelet.cu:65-81: at each
// step lane i (i < c - c/2) takes lane i + c/2 when the other value is strictly
// better; the lower lane keeps ties.  Result is in lane 0.
template <typename Better>
void reduce_down(int count, float* val, int* idx, Better better) {
    int c = count;
    int sh = c / 2;
    while (c > 1) {
        for (int i = 0; i < c - sh; ++i)
            if (better(val[i + sh], val[i])) { val[i] = val[i + sh]; idx[i] = idx[i + sh]; }
        c = (c + 1) / 2;
        sh = c / 2;
    }
}

// BVHRT-Core/src/Treelet.cuh:57-114
void form_treelet(const Tree& t, int root, int tsize, int* internal, int* leaves, float* la) {
    const int l0 = t.left[root], r0 = t.right[root];
    internal[0] = root;
    leaves[0] = l0;
    leaves[1] = r0;
    la[0] = t.area[l0];
    la[1] = t.area[r0];
    for (int it = 0; it < tsize - 2; ++it) {
        const int m = 2 + it;
        float v[32];
        int ix[32];
        for (int k = 0; k < m; ++k) {
            ix[k] = k;
            v[k] = is_internal(leaves[k], t.n) ? la[k] : -FLT_MAX;
        }
        reduce_down(m, v, ix, [](float o, float s) { return o > s; });
        const int largest = ix[0];
        const int rep = leaves[largest];
        const int l = t.left[rep], r = t.right[rep];
        internal[it + 1] = rep;
        leaves[largest] = l;
        leaves[it + 2] = r;
        la[largest] = t.area[l];
        la[it + 2] = t.area[r];
    }
}

// BVHRT-Core/src/TriangularMatrix.cuh:148-168 restated with integer arithmetic
// (row r, column c < r stored at r(r-1)/2 + c).
inline int trm_index(int r, int c) { return r * (r - 1) / 2 + c; }
inline void trm_row_col(int k, int& r, int& c) {
    r = 1;
    while ((r + 1) * r / 2 <= k) ++r;
    c = k - r * (r - 1) / 2;
}

// One agglomerative treelet: BVHRT-Core/src/AgglomerativeTreelet.cu:476-546
// (formTreelet, distance matrix :18-63, merge loop :511-532 with
// findMinimumDistance :83-99, updateState :101-150, updateDistancesMatrix
// :152-188, updateTreelet :190-212).
void atrbvh_treelet(Tree& t, int root, int n, float* nodes_sah, float ci) {
    int internal[32], leaves[32];
    float la[32];
    form_treelet(t, root, n, internal, leaves, la);

    // Per-"lane" state (lanes 0..n-1).
    int node[32];
    float sah[32];
    float mn[32][3], mx[32][3];
    for (int k = 0; k < n; ++k) {
        const F4& a = t.bmin[leaves[k]];
        const F4& b = t.bmax[leaves[k]];
        mn[k][0] = a.x; mn[k][1] = a.y; mn[k][2] = a.z;
        mx[k][0] = b.x; mx[k][1] = b.y; mx[k][2] = b.z;
        node[k] = leaves[k];
        sah[k] = nodes_sah[leaves[k]];
    }
    float D[32 * 31 / 2];
    for (int a = 1; a < n; ++a)
        for (int b = 0; b < a; ++b) D[trm_index(a, b)] = union_area(mn[a], mx[a], mn[b], mx[b]);

    for (int last = n - 1; last > 0; --last) {
        // findMinimumDistance: per-lane strided scan with strict <, then the
        // 32-lane shuffle-down reduction (strict <, lower lane keeps ties).
        const int msize = last * (last + 1) / 2;
        float bv[32];
        int bi[32];
        for (int ln = 0; ln < 32; ++ln) {
            bv[ln] = FLT_MAX;
            bi[ln] = 0;
            for (int j = ln; j < msize; j += 32)
                if (D[j] < bv[ln]) { bv[ln] = D[j]; bi[ln] = j; }
        }
        reduce_down(32, bv, bi, [](float o, float s) { return o < s; });
        int jr, jc;
        trm_row_col(bi[0], jr, jc);

        // updateState
        const float sah_new = sah[jr] + sah[jc];
        const int left_index = node[jr];
        const int right_index = node[jc];
        float amn[3], amx[3];
        for (int k = 0; k < 3; ++k) {
            amn[k] = fminf(mn[jc][k], mn[jr][k]);
            amx[k] = fmaxf(mx[jc][k], mx[jr][k]);
        }
        node[jc] = internal[last - 1];
        for (int k = 0; k < 3; ++k) { mn[jc][k] = amn[k]; mx[jc][k] = amx[k]; }
        const float area = box_area(amn[0], amn[1], amn[2], amx[0], amx[1], amx[2]);
        la[last] = sah_new + ci * area;
        sah[jc] = la[last];
        const int last_index = node[last];
        const float sah_last = sah[last];
        float bmn[3], bmx[3];
        for (int k = 0; k < 3; ++k) { bmn[k] = mn[last][k]; bmx[k] = mx[last][k]; }
        node[jr] = last_index;
        sah[jr] = sah_last;
        for (int k = 0; k < 3; ++k) { mn[jr][k] = bmn[k]; mx[jr][k] = bmx[k]; }
        node[last] = left_index;
        leaves[last] = right_index;
        for (int k = 0; k < 3; ++k) { mn[last][k] = amn[k]; mx[last][k] = amx[k]; }

        // updateDistancesMatrix
        if (last > 1) {
            float src[32];
            for (int ln = 0; ln < last; ++ln)
                if (ln != jr) src[ln] = D[trm_index(last, ln)];
            for (int ln = 0; ln < last; ++ln)
                if (ln != jr) D[trm_index(std::max(jr, ln), std::min(jr, ln))] = src[ln];
            for (int ln = 0; ln < last; ++ln) {
                if (ln == jc) continue;
                const int r = std::max(jc, ln), c = std::min(jc, ln);
                D[trm_index(r, c)] = union_area(mn[r], mx[r], mn[c], mx[c]);
            }
        }
    }

    // updateTreelet
    if (la[1] < nodes_sah[internal[0]]) {
        for (int ln = 1; ln < n; ++ln) {
            const int ni = internal[ln - 1];
            t.left[ni] = node[ln];
            t.right[ni] = leaves[ln];
            t.parent[node[ln]] = ni;
            t.parent[leaves[ln]] = ni;
            nodes_sah[ni] = la[ln];
            F4 a{mn[ln][0], mn[ln][1], mn[ln][2], 0.0f};
            F4 b{mx[ln][0], mx[ln][1], mx[ln][2], 0.0f};
            t.bmin[ni] = a;
            t.bmax[ni] = b;
            t.area[ni] = box_area(a, b);
        }
    }
}

// One TRBVH treelet (treelet size 7): BVHRT-Core/src/TRBVH.cu:405-471 with
// calculateSubsetSurfaceAreas :37-98, processSchedule :100-134 (subset sizes
// 2..n-2, partitions enumerated by (p - delta) & S, strict <), processSubsets
// :136-220 (sizes n-1 and n split over lanes and reduced with reduceOptimal
// :23-35) and updateTreelet :222-327 (round-by-round rebuild; left children
// take internal nodes before right children, each in lane order; the right
// child's nodesSah is written from costs[partition] as in :309).
void trbvh_treelet(Tree& t, int root, float* nodes_sah, const int* subtree, float ci, float ct,
                   std::vector<float>& scratch_box) {
    const int n = 7;
    const int nsub = 1 << n;
    int internal[32], leaves[32];
    float la[32];
    form_treelet(t, root, n, internal, leaves, la);

    float* smn = scratch_box.data();          // nsub * 3
    float* smx = smn + nsub * 3;              // nsub * 3
    float costs[1 << 7];
    signed char masks[1 << 7];
    std::memset(masks, 0, sizeof(masks));
    for (int s = 0; s < nsub; ++s) {
        float a[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, b[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int i = 0; i < n; ++i) {
            if (!(s & (1 << i))) continue;
            const F4& lm = t.bmin[leaves[i]];
            const F4& lx = t.bmax[leaves[i]];
            a[0] = fminf(lm.x, a[0]); a[1] = fminf(lm.y, a[1]); a[2] = fminf(lm.z, a[2]);
            b[0] = fmaxf(lx.x, b[0]); b[1] = fmaxf(lx.y, b[1]); b[2] = fmaxf(lx.z, b[2]);
        }
        for (int k = 0; k < 3; ++k) { smn[s * 3 + k] = a[k]; smx[s * 3 + k] = b[k]; }
        costs[s] = box_area(a[0], a[1], a[2], b[0], b[1], b[2]);
    }
    for (int i = 0; i < n; ++i) costs[1 << i] = nodes_sah[leaves[i]];
    const int T = subtree[internal[0]];
    const float Tf = (float)T;

    // Sizes 2 .. n-2, in increasing size (each depends only on smaller subsets).
    for (int size = 2; size <= n - 2; ++size) {
        for (int s = 1; s < nsub; ++s) {
            if (__builtin_popcount((unsigned)s) != size) continue;
            float opt = FLT_MAX;
            int optp = 0;
            const int delta = (s - 1) & s;
            int p = (-delta) & s;
            while (p != 0) {
                float c = costs[p] + costs[p ^ s];
                if (c < opt) { opt = c; optp = p; }
                p = (p - delta) & s;
            }
            costs[s] = fminf(ci * costs[s] + opt, ct * costs[s] * Tf);
            masks[s] = (signed char)optp;
        }
    }
    // Size n-1: four lanes per subset, then a 2-step reduction within the group.
    {
        float lv[32];
        int lp[32];
        for (int ln = 0; ln < 4 * n; ++ln) {
            const int k = ln / 4;
            const int s = (nsub - 1) & ~(1 << k);
            const int left_mask = -(1 << std::max(k - 1, 0));
            int base = (ln & 3) + 1;
            float opt = FLT_MAX;
            int optp = 0;
            const int np = (1 << (n - 2)) - 1;
            int p = (((base & left_mask) << 1) | (base & ~left_mask)) << 1;
            for (int j = (ln & 3); j < np; j += 4) {
                float c = costs[p] + costs[p ^ s];
                if (c < opt) { opt = c; optp = p; }
                base += 4;
                p = (((base & left_mask) << 1) | (base & ~left_mask)) << 1;
            }
            lv[ln] = opt;
            lp[ln] = optp;
        }
        for (int g = 0; g < n; ++g) {
            float v[4] = {lv[4 * g], lv[4 * g + 1], lv[4 * g + 2], lv[4 * g + 3]};
            int ix[4] = {lp[4 * g], lp[4 * g + 1], lp[4 * g + 2], lp[4 * g + 3]};
            reduce_down(4, v, ix, [](float o, float s2) { return o < s2; });
            const int s = (nsub - 1) & ~(1 << g);
            costs[s] = fminf(ci * costs[s] + v[0], ct * costs[s] * Tf);
            masks[s] = (signed char)ix[0];
        }
    }
    // Size n: 32 lanes, then the 32-lane reduction.
    {
        const int s = nsub - 1;
        const int np = (1 << (n - 1)) - 1;
        float v[32];
        int ix[32];
        for (int ln = 0; ln < 32; ++ln) {
            float opt = FLT_MAX;
            int optp = 0;
            int p = (ln + 1) * 2;
            for (int j = ln; j < np; j += 32) {
                float c = costs[p] + costs[p ^ s];
                if (c < opt) { opt = c; optp = p; }
                p += 64;
            }
            v[ln] = opt;
            ix[ln] = optp;
        }
        reduce_down(32, v, ix, [](float o, float s2) { return o < s2; });
        costs[s] = fminf(ci * costs[s] + v[0], ct * costs[s] * Tf);
        masks[s] = (signed char)ix[0];
    }

    if (!(costs[nsub - 1] < nodes_sah[internal[0]])) return;
    std::vector<std::pair<int, int>> stack{{internal[0], nsub - 1}}, next;
    int cur = 1;
    while (!stack.empty()) {
        next.clear();
        for (auto& e : stack) {
            const int part = masks[e.second];
            if (__builtin_popcount((unsigned)part) > 1) {
                const int child = internal[cur++];
                t.left[e.first] = child;
                t.parent[child] = e.first;
                F4 a{smn[part * 3], smn[part * 3 + 1], smn[part * 3 + 2], 0.0f};
                F4 b{smx[part * 3], smx[part * 3 + 1], smx[part * 3 + 2], 0.0f};
                t.bmin[child] = a;
                t.bmax[child] = b;
                t.area[child] = box_area(a, b);
                nodes_sah[child] = costs[part];
                next.push_back({child, part});
            } else {
                const int child = leaves[__builtin_ffs(part) - 1];
                t.left[e.first] = child;
                t.parent[child] = e.first;
            }
        }
        for (auto& e : stack) {
            const int part = masks[e.second];
            const int comp = (signed char)(part ^ e.second);
            if (__builtin_popcount((unsigned)comp) > 1) {
                const int child = internal[cur++];
                t.right[e.first] = child;
                t.parent[child] = e.first;
                F4 a{smn[comp * 3], smn[comp * 3 + 1], smn[comp * 3 + 2], 0.0f};
                F4 b{smx[comp * 3], smx[comp * 3 + 1], smx[comp * 3 + 2], 0.0f};
                t.bmin[child] = a;
                t.bmax[child] = b;
                t.area[child] = box_area(a, b);
                nodes_sah[child] = costs[part];
                next.push_back({child, comp});
            } else {
                const int child = leaves[__builtin_ffs(comp) - 1];
                t.right[e.first] = child;
                t.parent[child] = e.first;
            }
        }
        stack.swap(next);
    }
}

Tree make_tree(uint32_t n, int32_t* parent, int32_t* left, int32_t* right, int32_t* data,
               float* bmin4, float* bmax4, float* area) {
    Tree t;
    t.n = n;
    t.parent = parent;
    t.left = left;
    t.right = right;
    t.data = data;
    t.bmin = reinterpret_cast<F4*>(bmin4);
    t.bmax = reinterpret_cast<F4*>(bmax4);
    t.area = area;
    return t;
}

int nthreads_or_max(int threads) {
#ifdef _OPENMP
    return threads > 0 ? threads : omp_get_max_threads();
#else
    (void)threads;
    return 1;
#endif
}

}  // namespace

extern "C" {

// Number of host threads the parallel entry points use when asked for 0.
int orc_max_threads(void) { return nthreads_or_max(0); }

// Point-level forms of the arithmetic above, for the pins against the
// reference's own helpers (BVHRT-Core/src/Commons.cuh:99-194, 481-510, 606-662):
// a point already normalised to the unit cube, boxes as three floats.
uint32_t orc_expand_bits(uint32_t v) { return expand_bits(v); }
uint32_t orc_morton30_point(float x, float y, float z) {
    const float c[3] = {x, y, z}, lo[3] = {0.0f, 0.0f, 0.0f}, hi[3] = {1.0f, 1.0f, 1.0f};
    return morton30(c, lo, hi);
}
uint64_t orc_morton63_point(float x, float y, float z) {
    const float c[3] = {x, y, z}, lo[3] = {0.0f, 0.0f, 0.0f}, hi[3] = {1.0f, 1.0f, 1.0f};
    return morton63(c, lo, hi);
}
float orc_box_area(const float* mn, const float* mx) { return box_area(mn[0], mn[1], mn[2], mx[0], mx[1], mx[2]); }
float orc_union_area(const float* mn1, const float* mx1, const float* mn2, const float* mx2) {
    return union_area(mn1, mx1, mn2, mx2);
}

// Scene AABB over all vertices: gpu-ray-traversal/src/rt/SceneConverter.cpp:28-60.
// The max is seeded with numeric_limits<float>::min() (the smallest positive
// normal float), as in the reference.
void orc_scene_aabb(const float* verts, uint32_t n, float* bbmin, float* bbmax) {
    const F4* v = reinterpret_cast<const F4*>(verts);
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float mx[3] = {FLT_MIN, FLT_MIN, FLT_MIN};
    for (size_t i = 0; i < 3 * (size_t)n; ++i) {
        mn[0] = std::min(mn[0], v[i].x); mn[1] = std::min(mn[1], v[i].y); mn[2] = std::min(mn[2], v[i].z);
        mx[0] = std::max(mx[0], v[i].x); mx[1] = std::max(mx[1], v[i].y); mx[2] = std::max(mx[2], v[i].z);
    }
    for (int k = 0; k < 3; ++k) { bbmin[k] = mn[k]; bbmax[k] = mx[k]; }
}

// BVHRT-Core/src/LBVH.cu:53-74 (30-bit) and :76-97 (63-bit when keys64 != NULL).
void orc_morton(const float* verts, uint32_t n, const float* bbmin, const float* bbmax,
                uint32_t* keys32, uint64_t* keys64, int threads) {
    const F4* v = reinterpret_cast<const F4*>(verts);
    const int nt = nthreads_or_max(threads);
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        float c[3];
        tri_centroid(v, (uint32_t)i, c);
        if (keys64) keys64[i] = morton63(c, bbmin, bbmax);
        else keys32[i] = morton30(c, bbmin, bbmax);
    }
}

// Stable ascending sort of (key, index) with iota indices: the contract of
// cub::DeviceRadixSort::SortPairs used at BVHRT-Core/src/CubWrapper.cu:37.
// LSD radix sort with 8-bit digits (stable by construction).
void orc_sort_pairs32(uint32_t* keys, uint32_t* idx, uint32_t n, int threads) {
    std::vector<uint32_t> k2(n), i2(n);
    for (uint32_t i = 0; i < n; ++i) idx[i] = i;
    uint32_t *ka = keys, *ia = idx, *kb = k2.data(), *ib = i2.data();
    const int nt = nthreads_or_max(threads);
    std::vector<uint32_t> hist((size_t)nt * 256);
    for (int pass = 0; pass < 4; ++pass) {
        const int sh = pass * 8;
        std::fill(hist.begin(), hist.end(), 0u);
#pragma omp parallel num_threads(nt)
        {
#ifdef _OPENMP
            const int tid = omp_get_thread_num();
            const int tn = omp_get_num_threads();
#else
            const int tid = 0, tn = 1;
#endif
            const uint64_t lo = (uint64_t)n * tid / tn, hi = (uint64_t)n * (tid + 1) / tn;
            uint32_t* h = &hist[(size_t)tid * 256];
            for (uint64_t i = lo; i < hi; ++i) h[(ka[i] >> sh) & 255u]++;
#pragma omp barrier
#pragma omp single
            {
                uint32_t run = 0;
                for (int d = 0; d < 256; ++d)
                    for (int t2 = 0; t2 < tn; ++t2) {
                        uint32_t c = hist[(size_t)t2 * 256 + d];
                        hist[(size_t)t2 * 256 + d] = run;
                        run += c;
                    }
            }
            for (uint64_t i = lo; i < hi; ++i) {
                uint32_t p = h[(ka[i] >> sh) & 255u]++;
                kb[p] = ka[i];
                ib[p] = ia[i];
            }
        }
        std::swap(ka, kb);
        std::swap(ia, ib);
    }
    // Four passes: result is back in the caller's arrays.
}

void orc_sort_pairs64(uint64_t* keys, uint32_t* idx, uint32_t n) {
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
    std::vector<uint64_t> k2(n);
    for (uint32_t i = 0; i < n; ++i) { k2[i] = keys[order[i]]; idx[i] = order[i]; }
    std::memcpy(keys, k2.data(), sizeof(uint64_t) * n);
}

// BVHRT-Core/src/LBVH.cu:208-316 over all internal nodes.
void orc_karras(const uint32_t* keys32, const uint64_t* keys64, const uint32_t* sidx, uint32_t n,
                int32_t* parent, int32_t* left, int32_t* right, int32_t* data, int threads) {
    const int nt = nthreads_or_max(threads);
#pragma omp parallel for num_threads(nt) schedule(static, 4096)
    for (int64_t i = 0; i < (int64_t)n - 1; ++i) {
        if (keys64) karras_node<uint64_t>(keys64, sidx, n, (int)i, parent, left, right, data);
        else karras_node<uint32_t>(keys32, sidx, n, (int)i, parent, left, right, data);
    }
}

// BVHRT-Core/src/LBVH.cu:430-570: leaf boxes from the triangle's vertices,
// internal boxes as unions, area per node; leaves get left = right = -1.
// The .w lanes (left uninitialised by the reference) are written as 0.
void orc_refit(const float* verts, uint32_t n, int32_t* parent, int32_t* left, int32_t* right,
               int32_t* data, float* bmin4, float* bmax4, float* area, int threads) {
    Tree t = make_tree(n, parent, left, right, data, bmin4, bmax4, area);
    const F4* v = reinterpret_cast<const F4*>(verts);
    const int nt = nthreads_or_max(threads);
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const int leaf = (int)i + (int)n - 1;
        const uint32_t tri = (uint32_t)t.data[leaf];
        const F4& a = v[3 * (size_t)tri], &b = v[3 * (size_t)tri + 1], &c = v[3 * (size_t)tri + 2];
        F4 mn{fminf(fminf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y), fminf(fminf(a.z, b.z), c.z), 0.0f};
        F4 mx{fmaxf(fmaxf(a.x, b.x), c.x), fmaxf(fmaxf(a.y, b.y), c.y), fmaxf(fmaxf(a.z, b.z), c.z), 0.0f};
        t.left[leaf] = -1;
        t.right[leaf] = -1;
        t.bmin[leaf] = mn;
        t.bmax[leaf] = mx;
        t.area[leaf] = box_area(mn, mx);
    }
    auto visit = [&](int x) {
        const int l = t.left[x], r = t.right[x];
        F4 mn{fminf(t.bmin[l].x, t.bmin[r].x), fminf(t.bmin[l].y, t.bmin[r].y), fminf(t.bmin[l].z, t.bmin[r].z), 0.0f};
        F4 mx{fmaxf(t.bmax[l].x, t.bmax[r].x), fmaxf(t.bmax[l].y, t.bmax[r].y), fmaxf(t.bmax[l].z, t.bmax[r].z), 0.0f};
        t.bmin[x] = mn;
        t.bmax[x] = mx;
        t.area[x] = box_area(mn, mx);
    };
    if (n > 1) run_post_order(t, nt, visit);
}

// Full LBVH: BVHRT-Core/src/LBVHBuilder.cpp:36-130 (Morton, sort, tree, refit).
// sorted_keys/sorted_idx may be NULL.  morton_bits is 30 or 63.
int orc_build_lbvh(const float* verts, uint32_t n, const float* bbmin, const float* bbmax, int morton_bits,
                   int32_t* parent, int32_t* left, int32_t* right, int32_t* data, float* bmin4,
                   float* bmax4, float* area, uint64_t* sorted_keys, uint32_t* sorted_idx, int threads) {
    if (n < 2 || (morton_bits != 30 && morton_bits != 63)) return 1;
    std::vector<uint32_t> idx(n);
    if (morton_bits == 30) {
        std::vector<uint32_t> k(n);
        orc_morton(verts, n, bbmin, bbmax, k.data(), nullptr, threads);
        orc_sort_pairs32(k.data(), idx.data(), n, threads);
        orc_karras(k.data(), nullptr, idx.data(), n, parent, left, right, data, threads);
        if (sorted_keys) for (uint32_t i = 0; i < n; ++i) sorted_keys[i] = k[i];
    } else {
        std::vector<uint64_t> k(n);
        orc_morton(verts, n, bbmin, bbmax, nullptr, k.data(), threads);
        orc_sort_pairs64(k.data(), idx.data(), n);
        orc_karras(nullptr, k.data(), idx.data(), n, parent, left, right, data, threads);
        if (sorted_keys) std::memcpy(sorted_keys, k.data(), sizeof(uint64_t) * n);
    }
    if (sorted_idx) std::memcpy(sorted_idx, idx.data(), sizeof(uint32_t) * n);
    orc_refit(verts, n, parent, left, right, data, bmin4, bmax4, area, threads);
    return 0;
}

// ATRBVH optimiser: BVHRT-Core/src/AgglomerativeTreeletOptimizer.cpp:73-92
// (gamma = treeletSize, doubled per iteration) over the bottom-up pass of
// AgglomerativeTreelet.cu:392-554 (leaves: subtree = 1, nodesSah = ct*area;
// internal: subtree = sum, nodesSah = ci*area + sahL + sahR; treelets at nodes
// whose subtree holds >= gamma triangles).  The reference's bottom-up order
// processes every node after both children, and treelets in disjoint subtrees
// are independent, so a post-order pass gives the same tree.
int orc_atrbvh(uint32_t n, int32_t* parent, int32_t* left, int32_t* right, int32_t* data,
               float* bmin4, float* bmax4, float* area, int treelet, int iterations, float ci,
               float ct, int threads) {
    if (treelet < 3 || treelet > 20 || iterations < 0 || n < 2) return 1;
    Tree t = make_tree(n, parent, left, right, data, bmin4, bmax4, area);
    const size_t nn = 2 * (size_t)n - 1;
    std::vector<int> subtree(nn);
    std::vector<float> nsah(nn);
    int gamma = treelet;
    const int nt = nthreads_or_max(threads);
    for (int it = 0; it < iterations; ++it) {
        for (size_t i = n - 1; i < nn; ++i) {
            subtree[i] = 1;
            nsah[i] = ct * t.area[i];
        }
        auto visit = [&](int x) {
            const int l = t.left[x], r = t.right[x];
            const int cnt = subtree[l] + subtree[r];
            subtree[x] = cnt;
            nsah[x] = ci * t.area[x] + nsah[l] + nsah[r];
            if (cnt >= gamma) atrbvh_treelet(t, x, treelet, nsah.data(), ci);
        };
        run_post_order(t, nt, visit);
        gamma *= 2;
    }
    return 0;
}

// TRBVH optimiser (treelet size 7 only: the reference's subset-box kernel,
// BVHRT-Core/src/TRBVH.cu:48-97, covers the 2^n subsets only for n = 7):
// BVHRT-Core/src/TRBVHOptimizer.cpp:91-106 over TRBVH.cu:329-479.
int orc_trbvh(uint32_t n, int32_t* parent, int32_t* left, int32_t* right, int32_t* data,
              float* bmin4, float* bmax4, float* area, int treelet, int iterations, float ci,
              float ct, int threads) {
    if (treelet != 7 || iterations < 0 || n < 2) return 1;
    Tree t = make_tree(n, parent, left, right, data, bmin4, bmax4, area);
    const size_t nn = 2 * (size_t)n - 1;
    std::vector<int> subtree(nn);
    std::vector<float> nsah(nn);
    int gamma = treelet;
    const int nt = nthreads_or_max(threads);
    for (int it = 0; it < iterations; ++it) {
        for (size_t i = n - 1; i < nn; ++i) {
            subtree[i] = 1;
            nsah[i] = ct * t.area[i];
        }
        auto visit = [&](int x) {
            thread_local std::vector<float> scratch((1 << 7) * 6);
            const int l = t.left[x], r = t.right[x];
            const int cnt = subtree[l] + subtree[r];
            subtree[x] = cnt;
            nsah[x] = ci * t.area[x] + nsah[l] + nsah[r];
            if (cnt >= gamma) trbvh_treelet(t, x, nsah.data(), subtree.data(), ci, ct, scratch);
        };
        run_post_order(t, nt, visit);
        gamma *= 2;
    }
    return 0;
}

// Triangle-splitting LBVH: the reference's primitive-box kernels.
// BVHRT-Core/src/LBVH.cu:99-161: Morton codes of each primitive box's
// centroid (min + max) / 2 normalised to the scene box, routing indices iota;
// the sort; :320-428: the tree, a leaf's data index dataIndices[routing];
// :572-669: leaf boxes from the primitive boxes through the routing index,
// unions above.  pbmin4 / pbmax4: n float4; pdata: n triangle indices.
int orc_build_lbvh_split(uint32_t n, const float* pbmin4, const float* pbmax4, const uint32_t* pdata,
                         const float* sbmin, const float* sbmax, int morton_bits, int32_t* parent, int32_t* left,
                         int32_t* right, int32_t* data, float* bmin4, float* bmax4, float* area, int threads) {
    if (n < 2 || (morton_bits != 30 && morton_bits != 63)) return 1;
    const F4* bmn = reinterpret_cast<const F4*>(pbmin4);
    const F4* bmx = reinterpret_cast<const F4*>(pbmax4);
    std::vector<uint32_t> route(n), leaf_data(n);
    auto centroid = [&](uint32_t i, float c[3]) {
        c[0] = (bmn[i].x + bmx[i].x) / 2.0f;
        c[1] = (bmn[i].y + bmx[i].y) / 2.0f;
        c[2] = (bmn[i].z + bmx[i].z) / 2.0f;
    };
    if (morton_bits == 30) {
        std::vector<uint32_t> k(n);
        for (uint32_t i = 0; i < n; ++i) { float c[3]; centroid(i, c); k[i] = morton30(c, sbmin, sbmax); }
        orc_sort_pairs32(k.data(), route.data(), n, threads);
        for (uint32_t i = 0; i < n; ++i) leaf_data[i] = pdata[route[i]];
        orc_karras(k.data(), nullptr, leaf_data.data(), n, parent, left, right, data, threads);
    } else {
        std::vector<uint64_t> k(n);
        for (uint32_t i = 0; i < n; ++i) { float c[3]; centroid(i, c); k[i] = morton63(c, sbmin, sbmax); }
        orc_sort_pairs64(k.data(), route.data(), n);
        for (uint32_t i = 0; i < n; ++i) leaf_data[i] = pdata[route[i]];
        orc_karras(nullptr, k.data(), leaf_data.data(), n, parent, left, right, data, threads);
    }
    Tree t = make_tree(n, parent, left, right, data, bmin4, bmax4, area);
    for (uint32_t i = 0; i < n; ++i) {
        const int leaf = (int)i + (int)n - 1;
        const F4 mn{bmn[route[i]].x, bmn[route[i]].y, bmn[route[i]].z, 0.0f};
        const F4 mx{bmx[route[i]].x, bmx[route[i]].y, bmx[route[i]].z, 0.0f};
        t.left[leaf] = -1;
        t.right[leaf] = -1;
        t.bmin[leaf] = mn;
        t.bmax[leaf] = mx;
        t.area[leaf] = box_area(mn, mx);
    }
    auto visit = [&](int x) {
        const int l = t.left[x], r = t.right[x];
        F4 mn{fminf(t.bmin[l].x, t.bmin[r].x), fminf(t.bmin[l].y, t.bmin[r].y), fminf(t.bmin[l].z, t.bmin[r].z), 0.0f};
        F4 mx{fmaxf(t.bmax[l].x, t.bmax[r].x), fmaxf(t.bmax[l].y, t.bmax[r].y), fmaxf(t.bmax[l].z, t.bmax[r].z), 0.0f};
        t.bmin[x] = mn;
        t.bmax[x] = mx;
        t.area[x] = box_area(mn, mx);
    };
    run_post_order(t, nthreads_or_max(threads), visit);
    return 0;
}

// Triangle splitting (no counterpart in the reference: its primitive-box
// build above has no step that makes the boxes).  The product's scheme,
// restated with the same operations in the same order: priority
// sqrt(max(0, SA(box) - 2 * area)), integer shares floor(p / p_max * 2^16),
// s_t = min(7, floor(q_t * K / 2^16)) splits with K the largest scale whose
// splits fit the budget (binary search over the shares' histogram), each bisecting the
// largest fragment's region at the middle of its tight box's longest axis
// and clipping the triangle to both halves.  Returns the primitive count, or
// -1 when max_prims is too small.
namespace split_detail {
struct TriV { float v[3][3]; };
inline float sa_box(const float* mn, const float* mx) {
    return box_area(mn[0], mn[1], mn[2], mx[0], mx[1], mx[2]);
}
float priority(const TriV& T) {
    float mn[3], mx[3];
    for (int a = 0; a < 3; ++a) {
        mn[a] = fminf(fminf(T.v[0][a], T.v[1][a]), T.v[2][a]);
        mx[a] = fmaxf(fmaxf(T.v[0][a], T.v[1][a]), T.v[2][a]);
    }
    const float ux = T.v[1][0] - T.v[0][0], uy = T.v[1][1] - T.v[0][1], uz = T.v[1][2] - T.v[0][2];
    const float wx = T.v[2][0] - T.v[0][0], wy = T.v[2][1] - T.v[0][1], wz = T.v[2][2] - T.v[0][2];
    const float cx = uy * wz - uz * wy;
    const float cy = uz * wx - ux * wz;
    const float cz = ux * wy - uy * wx;
    const float len2 = (cx * cx + cy * cy) + cz * cz;
    const float ar = 0.5f * std::sqrt(len2);
    const float waste = sa_box(mn, mx) - 2.0f * ar;
    return waste > 0.0f ? std::sqrt(waste) : 0.0f;
}
bool clip_box(const TriV& T, const float* rmn, const float* rmx, float* omn, float* omx) {
    float P[9][3], Q[9][3];
    int np = 3;
    for (int k = 0; k < 3; ++k)
        for (int a = 0; a < 3; ++a) P[k][a] = T.v[k][a];
    for (int plane = 0; plane < 6; ++plane) {
        const int ax = plane >> 1;
        const bool upper = plane & 1;
        const float c = upper ? rmx[ax] : rmn[ax];
        int nq = 0;
        for (int i = 0; i < np; ++i) {
            const float* p = P[i];
            const float* q = P[i + 1 < np ? i + 1 : 0];
            const bool pin = upper ? p[ax] <= c : p[ax] >= c;
            const bool qin = upper ? q[ax] <= c : q[ax] >= c;
            if (pin && nq < 9) { Q[nq][0] = p[0]; Q[nq][1] = p[1]; Q[nq][2] = p[2]; ++nq; }
            if (pin != qin && nq < 9) {
                const float t = (c - p[ax]) / (q[ax] - p[ax]);
                for (int a = 0; a < 3; ++a) Q[nq][a] = a == ax ? c : p[a] + t * (q[a] - p[a]);
                ++nq;
            }
        }
        np = nq;
        if (np == 0) return false;
        for (int i = 0; i < np; ++i) { P[i][0] = Q[i][0]; P[i][1] = Q[i][1]; P[i][2] = Q[i][2]; }
    }
    for (int a = 0; a < 3; ++a) {
        float lo = P[0][a], hi = P[0][a];
        for (int i = 1; i < np; ++i) { lo = fminf(lo, P[i][a]); hi = fmaxf(hi, P[i][a]); }
        omn[a] = fmaxf(lo, rmn[a]);
        omx[a] = fminf(hi, rmx[a]);
        if (omn[a] > omx[a]) return false;
    }
    return true;
}
}  // namespace split_detail

int64_t orc_split_triangles(const float* verts, uint32_t n, float split_ratio, uint32_t max_prims,
                            float* out_bmin4, float* out_bmax4, uint32_t* out_data) {
    using namespace split_detail;
    const F4* v = reinterpret_cast<const F4*>(verts);
    auto tri = [&](uint32_t t) {
        TriV T;
        for (int k = 0; k < 3; ++k) {
            const F4& p = v[3 * (size_t)t + k];
            T.v[k][0] = p.x; T.v[k][1] = p.y; T.v[k][2] = p.z;
        }
        return T;
    };
    uint64_t budget = (uint64_t)((double)split_ratio * (double)n);
    if (budget > (uint64_t)max_prims - n) budget = (uint64_t)max_prims - n;
    std::vector<float> prio(n);
    float pmax = 0.0f;
    for (uint32_t t = 0; t < n; ++t) { prio[t] = priority(tri(t)); pmax = fmaxf(pmax, prio[t]); }
    std::vector<uint32_t> share(n), count(n), hist(65537, 0u);
    for (uint32_t t = 0; t < n; ++t) {
        share[t] = pmax > 0.0f ? (uint32_t)fminf((prio[t] / pmax) * 65536.0f, 65536.0f) : 0u;
        if (share[t]) hist[share[t]]++;
    }
    auto splits_of = [](uint32_t q, uint64_t K) {
        const uint64_t s = (uint64_t)q * K / 65536u;
        return (uint32_t)(s < 7 ? s : 7);
    };
    auto sum_splits = [&](uint64_t K) {
        uint64_t s = 0;
        for (uint32_t q = 1; q <= 65536u; ++q)
            if (hist[q]) s += (uint64_t)hist[q] * splits_of(q, K);
        return s;
    };
    // The largest scale K whose splits fit the budget.
    uint64_t lo = 0, hi = 7ull * 65536u + 1;
    uint64_t K;
    if (sum_splits(hi) <= budget) {
        K = hi;
    } else {
        while (hi - lo > 1) {
            const uint64_t mid = lo + (hi - lo) / 2;
            if (sum_splits(mid) <= budget) lo = mid; else hi = mid;
        }
        K = lo;
    }
    uint64_t total = 0;
    for (uint32_t t = 0; t < n; ++t) {
        count[t] = 1u + splits_of(share[t], K);
        total += count[t];
    }
    if (total > max_prims) return -1;
    F4* omn = reinterpret_cast<F4*>(out_bmin4);
    F4* omx = reinterpret_cast<F4*>(out_bmax4);
    uint64_t o = 0;
    for (uint32_t t = 0; t < n; ++t) {
        const TriV T = tri(t);
        const int c = (int)count[t];
        float rmn[8][3], rmx[8][3], fmn[8][3], fmx[8][3];
        for (int a = 0; a < 3; ++a) {
            fmn[0][a] = rmn[0][a] = fminf(fminf(T.v[0][a], T.v[1][a]), T.v[2][a]);
            fmx[0][a] = rmx[0][a] = fmaxf(fmaxf(T.v[0][a], T.v[1][a]), T.v[2][a]);
        }
        int have = 1;
        while (have < c) {
            int b = 0;
            float bs = sa_box(fmn[0], fmx[0]);
            for (int k = 1; k < have; ++k) {
                const float sk = sa_box(fmn[k], fmx[k]);
                if (sk > bs) { bs = sk; b = k; }
            }
            int ax = 0;
            float ext = fmx[b][0] - fmn[b][0];
            for (int a = 1; a < 3; ++a) {
                const float e = fmx[b][a] - fmn[b][a];
                if (e > ext) { ext = e; ax = a; }
            }
            const float mid = (fmn[b][ax] + fmx[b][ax]) * 0.5f;
            float lmn[3], lmx[3], hmn[3], hmx[3], alo[3], ahi[3], blo[3], bhi[3];
            for (int a = 0; a < 3; ++a) { lmn[a] = hmn[a] = rmn[b][a]; lmx[a] = hmx[a] = rmx[b][a]; }
            lmx[ax] = mid;
            hmn[ax] = mid;
            if (!(ext > 0.0f) || !clip_box(T, lmn, lmx, alo, ahi) || !clip_box(T, hmn, hmx, blo, bhi)) break;
            for (int a = 0; a < 3; ++a) {
                rmn[b][a] = lmn[a]; rmx[b][a] = lmx[a]; fmn[b][a] = alo[a]; fmx[b][a] = ahi[a];
                rmn[have][a] = hmn[a]; rmx[have][a] = hmx[a]; fmn[have][a] = blo[a]; fmx[have][a] = bhi[a];
            }
            ++have;
        }
        for (int k = 0; k < c; ++k) {
            const int f = k < have ? k : have - 1;
            omn[o + k] = F4{fmn[f][0], fmn[f][1], fmn[f][2], 0.0f};
            omx[o + k] = F4{fmx[f][0], fmx[f][1], fmx[f][2], 0.0f};
            out_data[o + k] = t;
        }
        o += (uint64_t)c;
    }
    return (int64_t)total;
}

// BVHRT-Core/src/SoABVHTree.cpp:50-74 (sequential float sums in index order).
float orc_sah(uint32_t n, const float* area, int root, float ci, float ct) {
    const float total = area[root];
    float si = total;
    float sl = 0.0f;
    for (uint32_t i = 0; i < n - 1; ++i)
        if ((int)i != root) si += area[i];
    for (uint32_t i = n - 1; i < 2 * n - 1; ++i) sl += area[i];
    return (ci * si + ct * sl) / total;
}

// Leaf collapse: BVHRT-Core/src/TreeCollapser.cu:13-237 and
// BVHTreeCollapser.cpp:21-93.
//   copyTree :13-30, cost/collapse flags/triangle counts :32-93 (leaf cost from
//   the box, collapse when ct*A*count < ci*A + cL + cR), emission :173-237: a
//   climbing thread continues through collapsed nodes, and the second arrival at
//   a node that is not collapsed turns each child with more than one triangle
//   into a leaf listing its subtree's triangles (right-first stack order of
//   writeSubtreeLeavesNonrecursive :95-137).  A node is reached by a second
//   arrival only when both children pass a thread upward (a leaf, or a reached
//   collapsed node).
// max_leaf > 0 additionally forbids collapsing subtrees with more triangles
// (not in the reference; 0 reproduces it).  Offsets into tri_indices are
// assigned in ascending node order (the reference's atomicAdd order is not
// deterministic; per-leaf lists are).  Returns the SAH cost[root]/area[root].
float orc_collapse(uint32_t n, const int32_t* parent, const int32_t* left, const int32_t* right,
                   const int32_t* data, const float* bmin4, const float* bmax4, const float* area,
                   float ci, float ct, int max_leaf, int32_t* c_parent, int32_t* c_left,
                   int32_t* c_right, int32_t* c_data, int32_t* c_count, float* c_bmin4,
                   float* c_bmax4, int32_t* tri_indices, float* cost_out) {
    const size_t nn = 2 * (size_t)n - 1;
    Tree t = make_tree(n, const_cast<int32_t*>(parent), const_cast<int32_t*>(left),
                       const_cast<int32_t*>(right), const_cast<int32_t*>(data),
                       const_cast<float*>(bmin4), const_cast<float*>(bmax4), const_cast<float*>(area));
    std::memcpy(c_parent, parent, nn * 4);
    std::memcpy(c_left, left, nn * 4);
    std::memcpy(c_right, right, nn * 4);
    std::memcpy(c_data, data, nn * 4);
    std::memcpy(c_bmin4, bmin4, nn * 16);
    std::memcpy(c_bmax4, bmax4, nn * 16);
    std::vector<float> cost(nn);
    std::vector<char> collapse(nn, 0);
    for (size_t i = n - 1; i < nn; ++i) {
        c_count[i] = 1;
        cost[i] = ct * box_area(t.bmin[i], t.bmax[i]);
        collapse[i] = 1;
    }
    auto vcost = [&](int x) {
        const int l = t.left[x], r = t.right[x];
        const int cnt = c_count[l] + c_count[r];
        c_count[x] = cnt;
        const float a = box_area(t.bmin[x], t.bmax[x]);
        cost[x] = ci * a + cost[l] + cost[r];
        const float leaf_cost = ct * a * (float)cnt;
        if (leaf_cost < cost[x] && (max_leaf <= 0 || cnt <= max_leaf)) {
            cost[x] = leaf_cost;
            collapse[x] = 1;
        }
        c_data[x] = -1;
    };
    post_order(t, 0, vcost);

    // pass[x]: a thread leaves x upward.  reached[x]: x got its second arrival.
    std::vector<char> pass(nn, 0);
    for (size_t i = n - 1; i < nn; ++i) pass[i] = 1;
    std::vector<int> emit;  // nodes that become multi-triangle leaves
    auto vemit = [&](int x) {
        const int l = t.left[x], r = t.right[x];
        const bool reached = pass[l] && pass[r];
        pass[x] = reached && collapse[x];
        if (reached && !collapse[x]) {
            if (c_count[l] > 1) emit.push_back(l);
            if (c_count[r] > 1) emit.push_back(r);
        }
    };
    post_order(t, 0, vemit);
    std::sort(emit.begin(), emit.end());
    int offset = 0;
    std::vector<int> st;
    for (int c : emit) {
        const int cnt = c_count[c];
        int pos = 0;
        // writeSubtreeLeavesNonrecursive: stack of {left, right}, right popped first.
        st.clear();
        st.push_back(t.left[c]);
        st.push_back(t.right[c]);
        while (!st.empty()) {
            const int x = st.back();
            st.pop_back();
            if (!is_internal(x, n)) {
                const int d = t.data[x];
                bool unique = true;
                for (int k = 0; k < pos; ++k)
                    if (tri_indices[offset + k] == d) { unique = false; break; }
                if (unique) tri_indices[offset + pos++] = d;
            } else {
                st.push_back(t.left[x]);
                st.push_back(t.right[x]);
            }
        }
        c_data[c] = offset;
        c_count[c] = pos;
        offset += cnt;
    }
    if (cost_out) std::memcpy(cost_out, cost.data(), nn * 4);
    return cost[0] / area[0];
}

// Compact2 layout of a collapsed tree with Woop triangles:
// gpu-ray-traversal/src/rt/cuda/CudaBVH.cpp:469-574 (LIFO DFS from the root;
// 64-byte nodes; inner child = float4 offset (nodeOffsetSizeDiv 16), leaf child =
// ~(float4 offset into the Woop array); per triangle 3 float4 + triIndex;
// terminator float4 of 0x80000000 with triIndex 0) and :579-600 (woopifyTri).
// Returns 0 and writes the element counts; arrays must hold 4*(n-1) int4 nodes
// and 4*n float4/int Woop entries.
int orc_flatten_compact2(uint32_t n, const int32_t* c_left, const int32_t* c_right,
                         const int32_t* c_data, const int32_t* c_count, const float* c_bmin4,
                         const float* c_bmax4, const int32_t* tri_indices, const float* verts,
                         int32_t* nodes, float* woop, int32_t* tri_index, int64_t* num_nodes,
                         int64_t* num_woop) {
    const F4* bmn = reinterpret_cast<const F4*>(c_bmin4);
    const F4* bmx = reinterpret_cast<const F4*>(c_bmax4);
    const F4* v = reinterpret_cast<const F4*>(verts);
    auto bits = [](float f) { int32_t i; std::memcpy(&i, &f, 4); return i; };
    int64_t nvec = 4;  // node data in int4 units (root pre-allocated)
    int64_t wvec = 0;  // Woop data in float4 units
    std::vector<std::pair<int, int64_t>> stack{{0, 0}};
    auto woopify = [&](int tri, int64_t at) {
        const F4& a = v[3 * (size_t)tri], &b = v[3 * (size_t)tri + 1], &c = v[3 * (size_t)tri + 2];
        float c0[3] = {a.x - c.x, a.y - c.y, a.z - c.z};
        float c1[3] = {b.x - c.x, b.y - c.y, b.z - c.z};
        float c2[3] = {c0[1] * c1[2] - c0[2] * c1[1], c0[2] * c1[0] - c0[0] * c1[2],
                       c0[0] * c1[1] - c0[1] * c1[0]};
        float M[4][4];  // M[row][col]
        for (int r = 0; r < 3; ++r) { M[r][0] = c0[r]; M[r][1] = c1[r]; M[r][2] = c2[r]; }
        M[0][3] = c.x; M[1][3] = c.y; M[2][3] = c.z;
        M[3][0] = 0.0f; M[3][1] = 0.0f; M[3][2] = 0.0f; M[3][3] = 1.0f;
        // MatrixBase::inverted (Math.hpp:961-983) with detImpl for 3x3 (:934-939).
        float R[4][4];
        float d = 0.0f, si = 1.0f;
        for (int i = 0; i < 4; ++i) {
            float sj = si;
            for (int j = 0; j < 4; ++j) {
                float s[3][3];
                for (int k = 0; k < 3; ++k)
                    for (int l = 0; l < 3; ++l) s[k][l] = M[k < j ? k : k + 1][l < i ? l : l + 1];
                float det = s[0][0] * s[1][1] * s[2][2] - s[0][0] * s[1][2] * s[2][1] +
                            s[1][0] * s[2][1] * s[0][2] - s[1][0] * s[2][2] * s[0][1] +
                            s[2][0] * s[0][1] * s[1][2] - s[2][0] * s[0][2] * s[1][1];
                float dd = det * sj;
                R[i][j] = dd;
                d += dd * M[j][i];
                sj = -sj;
            }
            si = -si;
        }
        const float rd = d != 0.0f ? 1.0f / d : 0.0f;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) R[i][j] = R[i][j] * rd * 4.0f;
        float* w = woop + 4 * at;
        w[0] = R[2][0]; w[1] = R[2][1]; w[2] = R[2][2]; w[3] = -R[2][3];
        w[4] = R[0][0]; w[5] = R[0][1]; w[6] = R[0][2]; w[7] = R[0][3];
        w[8] = R[1][0]; w[9] = R[1][1]; w[10] = R[1][2]; w[11] = R[1][3];
        tri_index[at] = tri; tri_index[at + 1] = 0; tri_index[at + 2] = 0;
    };
    while (!stack.empty()) {
        auto e = stack.back();
        stack.pop_back();
        const int ch[2] = {c_left[e.first], c_right[e.first]};
        int32_t cidx[2];
        for (int k = 0; k < 2; ++k) {
            const int c = ch[k];
            if (c_data[c] < 0) {
                cidx[k] = (int32_t)nvec;  // byte offset / 16
                stack.push_back({c, nvec / 4});
                nvec += 4;
            } else {
                cidx[k] = ~(int32_t)wvec;
                const int cnt = c_count[c];
                if (cnt > 1) {
                    for (int j = 0; j < cnt; ++j) { woopify(tri_indices[c_data[c] + j], wvec); wvec += 3; }
                } else {
                    woopify(c_data[c], wvec);
                    wvec += 3;
                }
                int32_t term = (int32_t)0x80000000u;
                std::memcpy(woop + 4 * wvec + 0, &term, 4);
                std::memcpy(woop + 4 * wvec + 1, &term, 4);
                std::memcpy(woop + 4 * wvec + 2, &term, 4);
                std::memcpy(woop + 4 * wvec + 3, &term, 4);
                tri_index[wvec] = 0;
                wvec += 1;
            }
        }
        int32_t* dst = nodes + 16 * e.second;
        const F4 &lm = bmn[ch[0]], &lx = bmx[ch[0]], &rm = bmn[ch[1]], &rx = bmx[ch[1]];
        dst[0] = bits(lm.x); dst[1] = bits(lx.x); dst[2] = bits(lm.y); dst[3] = bits(lx.y);
        dst[4] = bits(rm.x); dst[5] = bits(rx.x); dst[6] = bits(rm.y); dst[7] = bits(rx.y);
        dst[8] = bits(lm.z); dst[9] = bits(lx.z); dst[10] = bits(rm.z); dst[11] = bits(rx.z);
        dst[12] = cidx[0]; dst[13] = cidx[1]; dst[14] = 0; dst[15] = 0;
    }
    *num_nodes = nvec / 4;
    *num_woop = wvec;
    return 0;
}

// Closest/any-hit traversal of one ray over the Compact2 layout:
// gpu-ray-traversal/src/rt/kernels/kepler_dynamic_fetch.cu:95-317 executed by a
// single lane (a found leaf is processed before traversal continues), with the
// span helpers of CudaTracerKernels.hpp:182-189 (integer min/max on float bits,
// as the video-instruction forms compute them).
namespace {
const int kSentinel = 0x76543210;
inline int imin(int a, int b) { return a < b ? a : b; }
inline int imax(int a, int b) { return a > b ? a : b; }
inline float fb(int i) { float f; std::memcpy(&f, &i, 4); return f; }
inline int bf(float f) { int i; std::memcpy(&i, &f, 4); return i; }
inline float span_begin(float a0, float a1, float b0, float b1, float c0, float c1, float d) {
    int t = imax(imin(bf(c0), bf(c1)), bf(d));
    return fb(imax(imax(bf(fminf(a0, a1)), bf(fminf(b0, b1))), t));
}
inline float span_end(float a0, float a1, float b0, float b1, float c0, float c1, float d) {
    int t = imin(imax(bf(c0), bf(c1)), bf(d));
    return fb(imin(imin(bf(fmaxf(a0, a1)), bf(fmaxf(b0, b1))), t));
}
void trace_one(const F4* nodes, const F4* woop, const int32_t* tri_index, const F4& o, const F4& dd,
               int any_hit, int32_t* out4) {
    const float ooeps = 8.271806125530277e-25f;  // 2^-80
    const float ox = o.x, oy = o.y, oz = o.z, tmin = o.w;
    const float dx = dd.x, dy = dd.y, dz = dd.z;
    float hitT = dd.w;
    const float idx = 1.0f / (fabsf(dx) > ooeps ? dx : copysignf(ooeps, dx));
    const float idy = 1.0f / (fabsf(dy) > ooeps ? dy : copysignf(ooeps, dy));
    const float idz = 1.0f / (fabsf(dz) > ooeps ? dz : copysignf(ooeps, dz));
    const float oodx = ox * idx, oody = oy * idy, oodz = oz * idz;
    int stack[64];
    int sp = 0;
    stack[0] = kSentinel;
    int leafAddr = 0, nodeAddr = 0, hitIndex = -1;
    while (nodeAddr != kSentinel) {
        while ((unsigned)nodeAddr < (unsigned)kSentinel) {
            const F4 n0 = nodes[nodeAddr + 0], n1 = nodes[nodeAddr + 1], nz = nodes[nodeAddr + 2];
            const F4 tmp = nodes[nodeAddr + 3];
            int c0 = bf(tmp.x), c1 = bf(tmp.y);
            const float c0lox = fmaf(n0.x, idx, -oodx), c0hix = fmaf(n0.y, idx, -oodx);
            const float c0loy = fmaf(n0.z, idy, -oody), c0hiy = fmaf(n0.w, idy, -oody);
            const float c0loz = fmaf(nz.x, idz, -oodz), c0hiz = fmaf(nz.y, idz, -oodz);
            const float c1loz = fmaf(nz.z, idz, -oodz), c1hiz = fmaf(nz.w, idz, -oodz);
            const float c0min = span_begin(c0lox, c0hix, c0loy, c0hiy, c0loz, c0hiz, tmin);
            const float c0max = span_end(c0lox, c0hix, c0loy, c0hiy, c0loz, c0hiz, hitT);
            const float c1lox = fmaf(n1.x, idx, -oodx), c1hix = fmaf(n1.y, idx, -oodx);
            const float c1loy = fmaf(n1.z, idy, -oody), c1hiy = fmaf(n1.w, idy, -oody);
            const float c1min = span_begin(c1lox, c1hix, c1loy, c1hiy, c1loz, c1hiz, tmin);
            const float c1max = span_end(c1lox, c1hix, c1loy, c1hiy, c1loz, c1hiz, hitT);
            const bool swp = (c1min < c0min);
            const bool t0 = (c0max >= c0min), t1 = (c1max >= c1min);
            if (!t0 && !t1) {
                nodeAddr = stack[sp--];
            } else {
                nodeAddr = t0 ? c0 : c1;
                if (t0 && t1) {
                    if (swp) std::swap(nodeAddr, c1);
                    stack[++sp] = c1;
                }
            }
            if (nodeAddr < 0 && leafAddr >= 0) {
                leafAddr = nodeAddr;
                nodeAddr = stack[sp--];
            }
            if (leafAddr < 0) break;  // a single lane: every lane holds a leaf
        }
        while (leafAddr < 0) {
            for (int triAddr = ~leafAddr;; triAddr += 3) {
                const F4 v00 = woop[triAddr + 0], v11 = woop[triAddr + 1], v22 = woop[triAddr + 2];
                if (bf(v00.x) == (int)0x80000000u) break;
                const float Oz = fmaf(-oz, v00.z, fmaf(-oy, v00.y, fmaf(-ox, v00.x, v00.w)));
                const float invDz = 1.0f / fmaf(dz, v00.z, fmaf(dy, v00.y, dx * v00.x));
                const float t = Oz * invDz;
                if (t > tmin && t < hitT) {
                    const float Ox = fmaf(oz, v11.z, fmaf(oy, v11.y, fmaf(ox, v11.x, v11.w)));
                    const float Dx = fmaf(dz, v11.z, fmaf(dy, v11.y, dx * v11.x));
                    const float u = fmaf(t, Dx, Ox);
                    if (u >= 0.0f) {
                        const float Oy = fmaf(oz, v22.z, fmaf(oy, v22.y, fmaf(ox, v22.x, v22.w)));
                        const float Dy = fmaf(dz, v22.z, fmaf(dy, v22.y, dx * v22.x));
                        const float vv = fmaf(t, Dy, Oy);
                        if (vv >= 0.0f && u + vv <= 1.0f) {
                            hitT = t;
                            hitIndex = triAddr;
                            if (any_hit) { nodeAddr = kSentinel; break; }
                        }
                    }
                }
            }
            leafAddr = nodeAddr;
            if (nodeAddr < 0) nodeAddr = stack[sp--];
        }
    }
    out4[0] = hitIndex == -1 ? -1 : tri_index[hitIndex];
    out4[1] = bf(hitT);
}
}  // namespace

void orc_trace(const float* nodes, const float* woop, const int32_t* tri_index, const float* rays,
               int64_t nrays, int any_hit, int32_t* results, int threads) {
    const F4* nd = reinterpret_cast<const F4*>(nodes);
    const F4* w = reinterpret_cast<const F4*>(woop);
    const F4* r = reinterpret_cast<const F4*>(rays);
    const int nt = nthreads_or_max(threads);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
    for (int64_t i = 0; i < nrays; ++i) {
        int32_t* out = results + 4 * i;
        trace_one(nd, w, tri_index, r[2 * i], r[2 * i + 1], any_hit, out);
        out[2] = 0;
        out[3] = 0;
    }
}

// AgglomerativeScheduler::GenerateScheduleLower
// (BVHRT-Core/src/AgglomerativeScheduler.cpp:46-85): the 32-lane pair schedule,
// two (i<<8)|j pairs per int.  Returns the schedule size.
int orc_atrbvh_schedule(int treelet, int warp, int32_t* out, int cap) {
    const int elems = treelet * (treelet - 1) / 2;
    const int per = 2 * warp;
    const int iters = (elems + per - 1) / per;
    const int size = iters * warp;
    if (size > cap) return -size;
    std::fill(out, out + size, 0);
    int count = 0;
    float mult = 0.0f;
    for (int i = 0; i < treelet; ++i)
        for (int j = 0; j < i; ++j) {
            const int at = count + (int)mult * warp;
            out[at] = (out[at] << 16) | (i << 8) | j;
            if (++count == warp) { mult += 0.5f; count = 0; }
        }
    if ((int)(mult + 0.5f) > (int)mult)
        for (int i = count; i < 32; ++i) {
            const int at = i + (int)mult * warp;
            out[at] = out[at] << 16;
        }
    return size;
}

}  // extern "C"
