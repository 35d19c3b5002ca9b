// Device helpers shared by the kernels.
#pragma once

#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

namespace atr {

constexpr unsigned kFull = 0xffffffffu;

// Surface area 2*(x*y + x*z + y*z) evaluated in the reference's order with
// no contraction (BVHRT-Core/src/Commons.cuh:99-125).
__device__ __forceinline__ float sa3(float sx, float sy, float sz) {
    return __fmul_rn(2.0f, __fadd_rn(__fadd_rn(__fmul_rn(sx, sy), __fmul_rn(sx, sz)), __fmul_rn(sy, sz)));
}
__device__ __forceinline__ float box_area(const float4& mn, const float4& mx) {
    return sa3(__fsub_rn(mx.x, mn.x), __fsub_rn(mx.y, mn.y), __fsub_rn(mx.z, mn.z));
}
__device__ __forceinline__ float box_area(float mnx, float mny, float mnz, float mxx, float mxy, float mxz) {
    return sa3(__fsub_rn(mxx, mnx), __fsub_rn(mxy, mny), __fsub_rn(mxz, mnz));
}

// L2-coherent loads for data written by other SMs during the same kernel.
__device__ __forceinline__ float4 ld_cg(const float4* p) { return __ldcg(p); }
__device__ __forceinline__ int ld_cg(const int* p) { return __ldcg(p); }
__device__ __forceinline__ float ld_cg(const float* p) { return __ldcg(p); }

// Release/acquire fence at GPU scope (fence.acq_rel.gpu).  Placed before a
// relaxed atomic it makes the thread's earlier writes (and writes it has
// observed, e.g. its warp's behind a __syncwarp) visible to a thread whose
// atomic reads the result and which then runs the same fence before its
// loads; lighter than the sequentially consistent __threadfence().
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Atomic add with acquire-release semantics at GPU scope: one instruction in
// place of fence, relaxed atomic, fence on the bottom-up arrival counters.
__device__ __forceinline__ uint32_t atomic_add_acq_rel_gpu(uint32_t* p, uint32_t v) {
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Atomic exchange with acquire-release semantics at GPU scope (the arrival
// slots of the LBVH climb): one instruction in place of fence, exchange, fence.
__device__ __forceinline__ int atomic_exch_acq_rel_gpu(int* p, int v) {
    int old;
    asm volatile("atom.acq_rel.gpu.global.exch.b32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// 16-byte global-to-shared copy through L2 (cp.async.cg) that leaves no
// register pending: a later reader waits only for its own copies.
__device__ __forceinline__ void cp_async16_cg(void* smem, const void* gmem) {
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
// 4-byte form (cp.async.ca: through L1; for data no other thread of the
// running launch writes).
__device__ __forceinline__ void cp_async4_ca(void* smem, const void* gmem) {
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ void set_error_bits(uint32_t* err, uint32_t bits) {
    if (err) atomicOr(err, bits);
}

// Meshes of a batch laid end to end.  Mesh m owns triangles
// [tri_off[m], tri_off[m+1]), sort tiles [tile_off[m], tile_off[m+1]) and,
// in every per-node array, the 2n_m - 1 nodes starting at
// 2 * tri_off[m] - m (its own reference layout with local indices).  A
// single mesh passes count = 1 and no arrays.
struct Segs {
    const uint32_t* tri_off;
    const uint32_t* tile_off;
    uint32_t count;
    uint32_t n;  // total triangles

    __device__ __forceinline__ uint32_t find(const uint32_t* off, uint32_t x) const {
        uint32_t lo = 0, hi = count;  // off[lo] <= x < off[hi]
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(off + mid) <= x) lo = mid; else hi = mid;
        }
        return lo;
    }
    __device__ __forceinline__ uint32_t seg_of_tri(uint32_t i) const { return count == 1 ? 0u : find(tri_off, i); }
    __device__ __forceinline__ uint32_t seg_of_tile(uint32_t t) const { return count == 1 ? 0u : find(tile_off, t); }
    __device__ __forceinline__ uint32_t tri_begin(uint32_t m) const { return count == 1 ? 0u : __ldg(tri_off + m); }
    __device__ __forceinline__ uint32_t tri_end(uint32_t m) const { return count == 1 ? n : __ldg(tri_off + m + 1); }
    __device__ __forceinline__ uint32_t tile_begin(uint32_t m) const { return count == 1 ? 0u : __ldg(tile_off + m); }
    // First node of mesh m in per-node arrays, first internal node in per-internal arrays.
    __device__ __forceinline__ int node_base(uint32_t m) const { return (int)(2 * tri_begin(m) - m); }
    __device__ __forceinline__ int inner_base(uint32_t m) const { return (int)(tri_begin(m) - m); }
};

}  // namespace atr
