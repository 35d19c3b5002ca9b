// ORACLE -- test infrastructure only.
//
// Stands in for the CUDA runtime header when the reference's sources are
// compiled for the host execution model (simt.h): the types and the calls the
// reference makes, over host memory (simt.cpp).
#pragma once

#include "simt.h"

typedef int cudaError_t;
enum : int { cudaSuccess = 0, cudaErrorMemoryAllocation = 2 };
typedef void* cudaStream_t;
struct simt_event;
typedef simt_event* cudaEvent_t;
enum cudaMemcpyKind {
    cudaMemcpyHostToHost = 0,
    cudaMemcpyHostToDevice = 1,
    cudaMemcpyDeviceToHost = 2,
    cudaMemcpyDeviceToDevice = 3,
    cudaMemcpyDefault = 4
};
enum cudaFuncCache {
    cudaFuncCachePreferNone = 0,
    cudaFuncCachePreferShared = 1,
    cudaFuncCachePreferL1 = 2,
    cudaFuncCachePreferEqual = 3
};

cudaError_t cudaMalloc(void** p, size_t bytes);
template <class T>
inline cudaError_t cudaMalloc(T** p, size_t bytes) {
    return cudaMalloc(reinterpret_cast<void**>(p), bytes);
}
cudaError_t cudaFree(void* p);
cudaError_t cudaMemcpy(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind);
cudaError_t cudaMemset(void* p, int value, size_t bytes);
cudaError_t cudaDeviceSynchronize();
cudaError_t cudaGetLastError();
const char* cudaGetErrorString(cudaError_t e);
cudaError_t cudaEventCreate(cudaEvent_t* e);
cudaError_t cudaEventRecord(cudaEvent_t e, cudaStream_t stream = nullptr);
cudaError_t cudaEventSynchronize(cudaEvent_t e);
cudaError_t cudaEventElapsedTime(float* ms, cudaEvent_t start, cudaEvent_t stop);
cudaError_t cudaEventDestroy(cudaEvent_t e);
template <class F>
inline cudaError_t cudaFuncSetCacheConfig(F, cudaFuncCache) {
    return cudaSuccess;
}
