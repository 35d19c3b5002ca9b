// ORACLE -- test infrastructure only.
//
// Stands in for BVHRT-Core/src/CubWrapper.cu when the reference is compiled
// here.  That file does not compile against its bundled CUB 1.3.2 under CUDA
// 12.9 (CUB/Thrust version check, then removed texture references in
// cub/iterator/tex_ref_input_iterator.cuh).  The reference's call is
// cub::DeviceRadixSort::SortPairs, a stable ascending (key, value) sort whose
// result the caller reads from the *Out buffers (LBVHBuilder.cpp:74-102); the
// toolkit's CUB performs the same sort into those buffers.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

namespace BVHRT {

template <typename T>
static float sort_into_out(unsigned int n, T** keysIn, T** keysOut, unsigned int** valuesIn,
                           unsigned int** valuesOut) {
    void* temp = nullptr;
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(temp, bytes, *keysIn, *keysOut, *valuesIn, *valuesOut, (int)n);
    cudaMalloc(&temp, bytes);
    cub::DeviceRadixSort::SortPairs(temp, bytes, *keysIn, *keysOut, *valuesIn, *valuesOut, (int)n);
    cudaDeviceSynchronize();
    cudaFree(temp);
    return 0.0f;
}

float DeviceSort(unsigned int numberOfElements, unsigned int** keysIn, unsigned int** keysOut,
                 unsigned int** valuesIn, unsigned int** valuesOut) {
    return sort_into_out<unsigned int>(numberOfElements, keysIn, keysOut, valuesIn, valuesOut);
}

float DeviceSort(unsigned int numberOfElements, unsigned long long int** keysIn,
                 unsigned long long int** keysOut, unsigned int** valuesIn, unsigned int** valuesOut) {
    return sort_into_out<unsigned long long int>(numberOfElements, keysIn, keysOut, valuesIn,
                                                 valuesOut);
}

}  // namespace BVHRT
