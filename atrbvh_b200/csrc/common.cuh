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

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ void set_error_bits(uint32_t* err, uint32_t bits) {
    if (err) atomicOr(err, bits);
}

}  // namespace atr
