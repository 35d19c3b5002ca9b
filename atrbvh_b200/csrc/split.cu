// Triangle splitting for the LBVH's primitive-box path (the reference's
// triangle-splitting kernels, BVHRT-Core/src/LBVH.cu:99-161,320-428,572-669,
// build from per-primitive boxes and data indices but the reference has no
// step that makes the boxes; this is that step).
//
// Skinny or diagonal triangles have boxes much larger than themselves, and
// a Morton-ordered tree over those boxes overlaps badly.  Splitting such a
// triangle into fragments -- tight boxes of the triangle clipped to halves of
// its box -- lets the build separate them.  The scheme follows the idea of
// Karras and Aila, "Fast Parallel Construction of High-Quality Bounding
// Volume Hierarchies" (HPG 2013): a global budget of extra primitives is
// shared out by a per-triangle priority, and each triangle is bisected
// repeatedly at the middle of the longest axis of its largest fragment.
//
//   priority   p_t = sqrt(max(0, SA(box_t) - 2 * area_t)): the box surface a
//              triangle wastes (a triangle in an axis plane wastes none);
//   share      q_t = floor(p_t / p_max * 2^16), an integer;
//   splits     s_t = min(kMaxSplits, floor(q_t * K / 2^16)) with K the largest
//              integer whose splits fit the budget -- found on the host from
//              the histogram of the shares, so it is exact and order-free;
//   fragments  1 + s_t per triangle, written at the exclusive scan of the
//              counts in triangle order: start from the triangle's box; s_t
//              times take the fragment with the largest box surface area
//              (first on ties), split its region at the middle of its tight
//              box's longest axis (x, then y, then z on ties) and give each
//              half the tight box of the triangle clipped to that half
//              (Sutherland-Hodgman against the region's six planes).  A half
//              the clipping leaves empty ends the triangle's splitting; its
//              remaining fragments repeat the last one (a valid, redundant
//              leaf).
//
// Every float operation is a named round-to-nearest operation in a fixed
// order, so the CPU restatement reproduces the fragments bit for bit.

#include <vector>

#include "common.cuh"
#include "internal.h"

namespace atr {

int exclusive_scan_u32(atr_ctx* ctx, const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* d_total);

namespace {

constexpr int kMaxSplits = 7;          // fragments per triangle: at most 8
constexpr int kClipVerts = 9;          // a triangle clipped by six planes
constexpr float kShareScale = 65536.0f;

__device__ __forceinline__ uint32_t f2o(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}

struct Tri {
    float v[3][3];
};

__device__ __forceinline__ Tri load_tri(const float4* verts, uint32_t t) {
    Tri r;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float4 p = __ldg(verts + 3 * (size_t)t + k);
        r.v[k][0] = p.x;
        r.v[k][1] = p.y;
        r.v[k][2] = p.z;
    }
    return r;
}

__device__ __forceinline__ float sa_box(const float* mn, const float* mx) {
    return sa3(__fsub_rn(mx[0], mn[0]), __fsub_rn(mx[1], mn[1]), __fsub_rn(mx[2], mn[2]));
}

// Priority of a triangle: sqrt(max(0, SA(box) - 2 * area)), area from the
// cross product's length: 0.5 * sqrt(cx^2 + cy^2 + cz^2).
__device__ float tri_priority(const Tri& T) {
    float mn[3], mx[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        mn[a] = fminf(fminf(T.v[0][a], T.v[1][a]), T.v[2][a]);
        mx[a] = fmaxf(fmaxf(T.v[0][a], T.v[1][a]), T.v[2][a]);
    }
    const float ux = __fsub_rn(T.v[1][0], T.v[0][0]), uy = __fsub_rn(T.v[1][1], T.v[0][1]),
                uz = __fsub_rn(T.v[1][2], T.v[0][2]);
    const float wx = __fsub_rn(T.v[2][0], T.v[0][0]), wy = __fsub_rn(T.v[2][1], T.v[0][1]),
                wz = __fsub_rn(T.v[2][2], T.v[0][2]);
    const float cx = __fsub_rn(__fmul_rn(uy, wz), __fmul_rn(uz, wy));
    const float cy = __fsub_rn(__fmul_rn(uz, wx), __fmul_rn(ux, wz));
    const float cz = __fsub_rn(__fmul_rn(ux, wy), __fmul_rn(uy, wx));
    const float len2 = __fadd_rn(__fadd_rn(__fmul_rn(cx, cx), __fmul_rn(cy, cy)), __fmul_rn(cz, cz));
    const float area = __fmul_rn(0.5f, __fsqrt_rn(len2));
    const float waste = __fsub_rn(sa_box(mn, mx), __fmul_rn(2.0f, area));
    return waste > 0.0f ? __fsqrt_rn(waste) : 0.0f;
}

// Tight box of the triangle clipped to the region [rmn, rmx]; false when the
// clipped polygon is empty.
__device__ bool clip_box(const Tri& T, const float* rmn, const float* rmx, float* omn, float* omx) {
    float P[kClipVerts][3], Q[kClipVerts][3];
    int np = 3;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int a = 0; a < 3; ++a) P[k][a] = T.v[k][a];
    for (int plane = 0; plane < 6; ++plane) {
        const int ax = plane >> 1;
        const bool upper = plane & 1;  // keep x <= c (upper) or x >= c (lower)
        const float c = upper ? rmx[ax] : rmn[ax];
        int nq = 0;
        for (int i = 0; i < np; ++i) {
            const float* p = P[i];
            const float* q = P[i + 1 < np ? i + 1 : 0];
            const bool pin = upper ? p[ax] <= c : p[ax] >= c;
            const bool qin = upper ? q[ax] <= c : q[ax] >= c;
            if (pin && nq < kClipVerts) {
                Q[nq][0] = p[0]; Q[nq][1] = p[1]; Q[nq][2] = p[2];
                ++nq;
            }
            if (pin != qin && nq < kClipVerts) {
                // Crossing point: t = (c - p) / (q - p) on the plane's axis, the
                // other axes p + t * (q - p); the plane's axis takes c.
                const float t = __fdiv_rn(__fsub_rn(c, p[ax]), __fsub_rn(q[ax], p[ax]));
#pragma unroll
                for (int a = 0; a < 3; ++a)
                    Q[nq][a] = a == ax ? c : __fadd_rn(p[a], __fmul_rn(t, __fsub_rn(q[a], p[a])));
                ++nq;
            }
        }
        np = nq;
        if (np == 0) return false;
        for (int i = 0; i < np; ++i) { P[i][0] = Q[i][0]; P[i][1] = Q[i][1]; P[i][2] = Q[i][2]; }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float lo = P[0][a], hi = P[0][a];
        for (int i = 1; i < np; ++i) {
            lo = fminf(lo, P[i][a]);
            hi = fmaxf(hi, P[i][a]);
        }
        // Inside the region whatever the crossing points' rounding.
        omn[a] = fmaxf(lo, rmn[a]);
        omx[a] = fminf(hi, rmx[a]);
        if (omn[a] > omx[a]) return false;
    }
    return true;
}

// Priorities and their maximum (as an ordered integer).
__global__ void __launch_bounds__(256) k_split_priority(const float4* __restrict__ verts, uint32_t n,
                                                        float* __restrict__ prio, uint32_t* __restrict__ pmax) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    float p = 0.0f;
    if (t < n) {
        p = tri_priority(load_tri(verts, t));
        prio[t] = p;
    }
    for (int o = 16; o > 0; o >>= 1) p = fmaxf(p, __shfl_xor_sync(kFull, p, o));
    if ((threadIdx.x & 31) == 0) atomicMax(pmax, f2o(p));
}

// Integer shares q_t and their histogram (kShares + 1 bins).
constexpr uint32_t kShares = 65536;

__global__ void __launch_bounds__(256) k_split_share(uint32_t n, const float* __restrict__ prio,
                                                     const uint32_t* __restrict__ pmax, uint32_t* __restrict__ share,
                                                     uint32_t* __restrict__ hist) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float m = o2f(*pmax);
    const uint32_t q = m > 0.0f ? (uint32_t)fminf(__fmul_rn(__fdiv_rn(prio[t], m), kShareScale), kShareScale) : 0u;
    share[t] = q;
    if (q) atomicAdd(&hist[q], 1u);
}

// Splits of a triangle with share q under the scale K.
__host__ __device__ __forceinline__ uint32_t splits_of(uint32_t q, uint64_t K) {
    const uint64_t s = (uint64_t)q * K / kShares;
    return (uint32_t)(s < (uint64_t)kMaxSplits ? s : (uint64_t)kMaxSplits);
}

// Fragment counts 1 + s_t.
__global__ void __launch_bounds__(256) k_split_counts(uint32_t n, uint64_t K, const uint32_t* __restrict__ share,
                                                      uint32_t* __restrict__ count) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) count[t] = 1u + splits_of(share[t], K);
}

// The largest K whose splits fit the budget, from the share histogram.
uint64_t split_scale(const std::vector<uint32_t>& hist, uint64_t budget) {
    auto total = [&](uint64_t K) {
        uint64_t s = 0;
        for (uint32_t q = 1; q <= kShares; ++q)
            if (hist[q]) s += (uint64_t)hist[q] * splits_of(q, K);
        return s;
    };
    uint64_t lo = 0, hi = (uint64_t)kMaxSplits * kShares + 1;  // total(hi) is the most splits there can be
    if (total(hi) <= budget) return hi;
    while (hi - lo > 1) {  // total(lo) <= budget < total(hi)
        const uint64_t mid = lo + (hi - lo) / 2;
        if (total(mid) <= budget) lo = mid; else hi = mid;
    }
    return lo;
}

// The fragments of every triangle at its offset.
__global__ void __launch_bounds__(128) k_split_emit(const float4* __restrict__ verts, uint32_t n,
                                                    const uint32_t* __restrict__ count,
                                                    const uint32_t* __restrict__ offset, float4* __restrict__ out_min,
                                                    float4* __restrict__ out_max, uint32_t* __restrict__ out_data) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const Tri T = load_tri(verts, t);
    const int c = (int)count[t];
    float rmn[kMaxSplits + 1][3], rmx[kMaxSplits + 1][3];  // regions
    float fmn[kMaxSplits + 1][3], fmx[kMaxSplits + 1][3];  // tight boxes
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        fmn[0][a] = rmn[0][a] = fminf(fminf(T.v[0][a], T.v[1][a]), T.v[2][a]);
        fmx[0][a] = rmx[0][a] = fmaxf(fmaxf(T.v[0][a], T.v[1][a]), T.v[2][a]);
    }
    int have = 1;
    while (have < c) {
        // Largest tight box by surface area, first on ties.
        int b = 0;
        float bs = sa_box(fmn[0], fmx[0]);
        for (int k = 1; k < have; ++k) {
            const float sk = sa_box(fmn[k], fmx[k]);
            if (sk > bs) { bs = sk; b = k; }
        }
        // Longest axis of its tight box (x, y, z on ties), split at the middle.
        int ax = 0;
        float ext = __fsub_rn(fmx[b][0], fmn[b][0]);
#pragma unroll
        for (int a = 1; a < 3; ++a) {
            const float e = __fsub_rn(fmx[b][a], fmn[b][a]);
            if (e > ext) { ext = e; ax = a; }
        }
        const float mid = __fmul_rn(__fadd_rn(fmn[b][ax], fmx[b][ax]), 0.5f);
        float lmn[3], lmx[3], hmn[3], hmx[3], alo[3], ahi[3], blo[3], bhi[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            lmn[a] = rmn[b][a]; lmx[a] = rmx[b][a];
            hmn[a] = rmn[b][a]; hmx[a] = rmx[b][a];
        }
        lmx[ax] = mid;
        hmn[ax] = mid;
        if (!(ext > 0.0f) || !clip_box(T, lmn, lmx, alo, ahi) || !clip_box(T, hmn, hmx, blo, bhi)) break;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            rmn[b][a] = lmn[a]; rmx[b][a] = lmx[a]; fmn[b][a] = alo[a]; fmx[b][a] = ahi[a];
            rmn[have][a] = hmn[a]; rmx[have][a] = hmx[a]; fmn[have][a] = blo[a]; fmx[have][a] = bhi[a];
        }
        ++have;
    }
    const uint32_t o = offset[t];
    for (int k = 0; k < c; ++k) {
        const int f = k < have ? k : have - 1;
        out_min[o + k] = make_float4(fmn[f][0], fmn[f][1], fmn[f][2], 0.0f);
        out_max[o + k] = make_float4(fmx[f][0], fmx[f][1], fmx[f][2], 0.0f);
        out_data[o + k] = t;
    }
}

}  // namespace
}  // namespace atr

using namespace atr;

extern "C" {

int atr_split_triangles(atr_ctx* ctx, const atr_scene* scene, float split_ratio, uint32_t max_primitives,
                        float* prim_bmin, float* prim_bmax, uint32_t* data_indices, uint32_t* num_primitives) {
    ATR_REQUIRE(ctx && scene && prim_bmin && prim_bmax && data_indices && num_primitives, ATR_ERR_INVALID_ARG,
                "atr_split_triangles: NULL argument");
    ATR_REQUIRE(split_ratio >= 0.0f && split_ratio <= (float)kMaxSplits, ATR_ERR_INVALID_ARG,
                "atr_split_triangles: split ratio %g outside [0, %d]", split_ratio, kMaxSplits);
    const uint32_t n = scene->n;
    ATR_REQUIRE(max_primitives >= n, ATR_ERR_INVALID_ARG,
                "atr_split_triangles: room for %u primitives, the scene has %u triangles", max_primitives, n);
    // Extra primitives: the ratio's share of n, within the caller's room.
    uint64_t budget = (uint64_t)((double)split_ratio * (double)n);
    if (budget > (uint64_t)max_primitives - n) budget = (uint64_t)max_primitives - n;
    cudaStream_t s = ctx->stream;
    void* scratch = nullptr;
    const size_t n4 = align256((size_t)n * 4);
    const size_t h4 = align256((size_t)(kShares + 1) * 4);
    ATR_TRY(ctx->alloc(&scratch, 4 * n4 + h4 + 256));
    char* p = static_cast<char*>(scratch);
    float* prio = reinterpret_cast<float*>(p); p += n4;
    uint32_t* share = reinterpret_cast<uint32_t*>(p); p += n4;
    uint32_t* count = reinterpret_cast<uint32_t*>(p); p += n4;
    uint32_t* offset = reinterpret_cast<uint32_t*>(p); p += n4;
    uint32_t* hist = reinterpret_cast<uint32_t*>(p); p += h4;
    uint32_t* pmax = reinterpret_cast<uint32_t*>(p);
    uint32_t* total = reinterpret_cast<uint32_t*>(p + 16);
    cudaError_t e = cudaMemsetAsync(hist, 0, h4 + 256, s);
    const unsigned g = (n + 255) / 256;
    std::vector<uint32_t> h_hist(kShares + 1);
    if (e == cudaSuccess) {
        k_split_priority<<<g, 256, 0, s>>>(scene->verts, n, prio, pmax);
        k_split_share<<<g, 256, 0, s>>>(n, prio, pmax, share, hist);
        ctx->launches += 2;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_hist.data(), hist, (kShares + 1) * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) {
        k_split_counts<<<g, 256, 0, s>>>(n, split_scale(h_hist, budget), share, count);
        ctx->launches += 1;
        e = cudaGetLastError();
    }
    int st = e == cudaSuccess ? exclusive_scan_u32(ctx, count, offset, n, total)
                              : cuda_fail(e, "atr_split_triangles", __FILE__, __LINE__);
    uint32_t h_total = 0;
    if (st == ATR_OK) {
        e = cudaMemcpyAsync(&h_total, total, 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(e, "atr_split_triangles count", __FILE__, __LINE__);
    }
    if (st == ATR_OK && h_total > max_primitives) {
        set_error("atr_split_triangles: %u primitives exceed the room for %u", h_total, max_primitives);
        st = ATR_ERR_INVALID_ARG;
    }
    if (st == ATR_OK) {
        k_split_emit<<<(n + 127) / 128, 128, 0, s>>>(scene->verts, n, count, offset,
                                                     reinterpret_cast<float4*>(prim_bmin),
                                                     reinterpret_cast<float4*>(prim_bmax), data_indices);
        ctx->launches += 1;
        e = cudaGetLastError();
        if (e != cudaSuccess) st = cuda_fail(e, "k_split_emit launch", __FILE__, __LINE__);
    }
    ctx->release(scratch);
    if (st == ATR_OK) *num_primitives = h_total;
    return st;
}

}  // extern "C"
