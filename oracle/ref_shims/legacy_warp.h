// ORACLE -- test infrastructure only.
//
// Force-included when the reference's BVHRT-Core sources are compiled for
// sm_100a (oracle/build.py).  CUDA 12 no longer declares the pre-Volta warp
// intrinsics __shfl / __shfl_down for sm_70+, and the reference calls them and
// __ballot without a member mask.  Each is mapped to its *_sync form over the
// lanes active at the call (after a __syncwarp over the same lanes), which is
// the lock-step behaviour the reference was written for.  The reference's own
// host files also rely on headers that MSVC pulled in implicitly.
#pragma once

#include <cstddef>
#include <cstdio>
#include <iostream>
#include <set>
#include <vector>

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>

#ifdef __CUDACC__
__device__ __forceinline__ int atr_legacy_shfl(int v, int lane) {
    const unsigned m = __activemask();
    __syncwarp(m);
    return __shfl_sync(m, v, lane);
}
__device__ __forceinline__ float atr_legacy_shfl(float v, int lane) {
    const unsigned m = __activemask();
    __syncwarp(m);
    return __shfl_sync(m, v, lane);
}
__device__ __forceinline__ int atr_legacy_shfl_down(int v, unsigned d) {
    const unsigned m = __activemask();
    __syncwarp(m);
    return __shfl_down_sync(m, v, d);
}
__device__ __forceinline__ float atr_legacy_shfl_down(float v, unsigned d) {
    const unsigned m = __activemask();
    __syncwarp(m);
    return __shfl_down_sync(m, v, d);
}
__device__ __forceinline__ unsigned atr_legacy_ballot(int p) {
    const unsigned m = __activemask();
    return __ballot_sync(m, p);
}
#define __shfl(v, l) atr_legacy_shfl((v), (l))
#define __shfl_down(v, d) atr_legacy_shfl_down((v), (d))
#define __ballot(p) atr_legacy_ballot((p))
#endif
