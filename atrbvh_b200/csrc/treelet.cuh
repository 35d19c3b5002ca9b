// Treelet formation and lane-held treelet state shared by the ATRBVH and
// TRBVH kernels (BVHRT-Core/src/Treelet.cuh:23-114).
#pragma once

#include "common.cuh"

namespace atr {

constexpr int kMaxTreelet = 20;
constexpr int kMaxDist = kMaxTreelet * (kMaxTreelet - 1) / 2;  // 190

__device__ __forceinline__ bool is_internal(int idx, uint32_t n) { return (uint32_t)idx < n - 1u; }

// Row/column of flat index k of the strictly lower triangular matrix stored
// row by row (r(r-1)/2 + c): BVHRT-Core/src/TriangularMatrix.cuh:150-168.
__device__ __forceinline__ void trm_rc(int k, int& r, int& c) {
    r = (int)__fmul_rn(__fadd_rn(1.0f, __fsqrt_rn((float)(8 * k + 1))), 0.5f);
    if (r * (r - 1) / 2 > k) --r;
    if ((r + 1) * r / 2 <= k) ++r;
    c = k - r * (r - 1) / 2;
}
__device__ __forceinline__ int trm_idx(int r, int c) { return r * (r - 1) / 2 + c; }

struct Box {
    float mnx, mny, mnz, mxx, mxy, mxz;
};

__device__ __forceinline__ Box shfl_box(const Box& b, int src) {
    Box o;
    o.mnx = __shfl_sync(kFull, b.mnx, src);
    o.mny = __shfl_sync(kFull, b.mny, src);
    o.mnz = __shfl_sync(kFull, b.mnz, src);
    o.mxx = __shfl_sync(kFull, b.mxx, src);
    o.mxy = __shfl_sync(kFull, b.mxy, src);
    o.mxz = __shfl_sync(kFull, b.mxz, src);
    return o;
}

// Surface area of the union of two boxes (Commons.cuh:156-164).
__device__ __forceinline__ float union_area(const Box& a, const Box& b) {
    return sa3(__fsub_rn(fmaxf(a.mxx, b.mxx), fminf(a.mnx, b.mnx)),
               __fsub_rn(fmaxf(a.mxy, b.mxy), fminf(a.mny, b.mny)),
               __fsub_rn(fmaxf(a.mxz, b.mxz), fminf(a.mnz, b.mnz)));
}

struct TreeRefs {
    uint32_t n;
    int32_t* parent;
    int32_t* left;
    int32_t* right;
    float4* bmin;
    float4* bmax;
    float* area;
    float* nsah;
};

// The refs of one mesh of a batch: arrays start at the mesh's first node.
__device__ __forceinline__ TreeRefs rebase(const TreeRefs& g, int base, uint32_t n) {
    TreeRefs t = g;
    t.n = n;
    t.parent += base;
    t.left += base;
    t.right += base;
    t.bmin += base;
    t.bmax += base;
    t.area += base;
    t.nsah += base;
    return t;
}

// Lane-held treelet leaf with everything later steps need, loaded as soon as
// the lane receives the node.
struct LeafSlot {
    int node;
    float area;
    int cl = -1, cr = -1;  // children (internal nodes only)
    float cal, car;  // children's areas
    float4 mn, mx;   // box
    float sah;       // nodesSah
};

__device__ __forceinline__ void load_slot(const TreeRefs& t, LeafSlot& s, int node, float area) {
    s.node = node;
    s.area = area;
    s.mn = ld_cg(t.bmin + node);
    s.mx = ld_cg(t.bmax + node);
    s.sah = ld_cg(t.nsah + node);
    if (is_internal(node, t.n)) {
        s.cl = ld_cg(t.left + node);
        s.cr = ld_cg(t.right + node);
        s.cal = ld_cg(t.area + s.cl);
        s.car = ld_cg(t.area + s.cr);
    }
}


// formTreelet (Treelet.cuh:57-114): starting from the root's two children,
// repeatedly expand the treelet leaf with the largest area that is an
// internal node (shuffle-down argmax over the current leaves, strict >, the
// lower lane keeps ties); its children take its slot and slot it+2.  Lane k
// ends holding treelet leaf k in `slot` and treeletInternalNodes[k] in
// `internal_node`.  Returns false only for a malformed tree.
__device__ __forceinline__ bool form_treelet(const TreeRefs& t, int root, int tsize, LeafSlot& slot,
                                             int& internal_node) {
    const int lane = threadIdx.x & 31;
    internal_node = lane == 0 ? root : -1;
    slot.node = -1;
    slot.cl = slot.cr = -1;
    {
        const int l0 = ld_cg(t.left + root), r0 = ld_cg(t.right + root);
        if (lane < 2) {
            const int nd = lane == 0 ? l0 : r0;
            load_slot(t, slot, nd, ld_cg(t.area + nd));
        }
    }
    for (int it = 0; it < tsize - 2; ++it) {
        const int m = 2 + it;
        float v = -FLT_MAX;
        int ix = lane;
        if (lane < m) v = is_internal(slot.node, t.n) ? slot.area : -FLT_MAX;
        int c = m, sh = m / 2;
        while (c > 1) {
            const float ov = __shfl_down_sync(kFull, v, sh);
            const int oi = __shfl_down_sync(kFull, ix, sh);
            if (lane < c - sh && ov > v) { v = ov; ix = oi; }
            c = (c + 1) / 2;
            sh = c / 2;
        }
        const int largest = __shfl_sync(kFull, ix, 0);
        const int rep = __shfl_sync(kFull, slot.node, largest);
        if (!is_internal(rep, t.n)) return false;
        const int L = __shfl_sync(kFull, slot.cl, largest);
        const int R = __shfl_sync(kFull, slot.cr, largest);
        const float aL = __shfl_sync(kFull, slot.cal, largest);
        const float aR = __shfl_sync(kFull, slot.car, largest);
        if (lane == it + 1) internal_node = rep;
        if (lane == largest) load_slot(t, slot, L, aL);
        if (lane == it + 2) load_slot(t, slot, R, aR);
    }
    return true;
}

}  // namespace atr
