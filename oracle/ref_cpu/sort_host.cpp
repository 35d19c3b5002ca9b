// ORACLE -- test infrastructure only.
//
// Stands in for BVHRT-Core/src/CubWrapper.cu under the host execution model.
// The reference's DeviceSort sorts (key, index) pairs with CUB's stable LSD
// radix sort over all key bits, in a DoubleBuffer; its final lines assign the
// result pointers to its own parameters, not through them
// (CubWrapper.cu:62-72), so the caller (LBVHBuilder.cpp:74-81) reads the
// sorted pairs from the *Out buffers it passed, where an odd number of CUB
// passes leaves them.  This stand-in performs that sort, stable and ascending
// by key, into the *Out buffers.
#include <algorithm>
#include <numeric>
#include <vector>

#include "CubWrapper.h"

namespace BVHRT {
namespace {

template <class T>
float stable_pairs(unsigned int n, T** keys_in, T** keys_out, unsigned int** values_in, unsigned int** values_out) {
    std::vector<unsigned int> order(n);
    std::iota(order.begin(), order.end(), 0u);
    const T* k = *keys_in;
    std::stable_sort(order.begin(), order.end(), [k](unsigned int a, unsigned int b) { return k[a] < k[b]; });
    std::vector<T> ks(n);
    std::vector<unsigned int> vs(n);
    for (unsigned int i = 0; i < n; ++i) {
        ks[i] = k[order[i]];
        vs[i] = (*values_in)[order[i]];
    }
    std::copy(ks.begin(), ks.end(), *keys_out);
    std::copy(vs.begin(), vs.end(), *values_out);
    return 0.0f;
}

}  // namespace

float DeviceSort(unsigned int numberOfElements, unsigned int** keysIn, unsigned int** keysOut,
                 unsigned int** valuesIn, unsigned int** valuesOut) {
    return stable_pairs(numberOfElements, keysIn, keysOut, valuesIn, valuesOut);
}

float DeviceSort(unsigned int numberOfElements, unsigned long long int** keysIn, unsigned long long int** keysOut,
                 unsigned int** valuesIn, unsigned int** valuesOut) {
    return stable_pairs(numberOfElements, keysIn, keysOut, valuesIn, valuesOut);
}

}  // namespace BVHRT
