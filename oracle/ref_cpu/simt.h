// ORACLE -- test infrastructure only.
//
// A host-side execution model for CUDA kernel source, used to compile the
// reference's own BVHRT-Core kernels with g++ and run them on the CPU (the
// reference is the parity anchor; nothing in the product uses this).
//
// Model:
//   * every CUDA thread of a block is a fiber with its own stack; one block
//     runs at a time, blocks in blockIdx order, so global memory is
//     sequentially consistent and `static` storage serves as __shared__;
//   * a thread runs until it reaches a warp collective (__shfl, __shfl_down,
//     __ballot), __syncthreads() or its end; lanes of a warp run in lane
//     order between collectives;
//   * a warp collective completes when every live lane of the warp waits in
//     one; when they wait at different call sites (a collective inside a
//     branch that some lanes skipped), the lanes furthest back in program
//     order complete theirs first, as a divergent path of a pre-Volta warp
//     runs to its reconvergence point first.  __syncthreads() completes when
//     every live thread of the block waits in one.  Threads that have
//     returned take no part, as on the hardware;
//   * atomics are plain read-modify-writes (one fiber runs at a time).
// Code written for the pre-Volta lock-step warp (a lane reading what another
// lane wrote with no collective in between) needs an explicit warp sync at
// that point; the build recipe inserts SIMT_WARP_SYNC(id) where the reference
// relies on it, and documents each place.
#pragma once

// Standard headers first: the reference's Commons.cuh defines function-like
// min/max macros for host code, which must not reach these headers.
#include <algorithm>
#include <cassert>
#include <cfloat>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <limits>
#include <memory>
#include <set>
#include <sstream>
#include <string>
#include <vector>

struct float3 {
    float x, y, z;
};
struct alignas(16) float4 {
    float x, y, z, w;
};
struct uint3 {
    unsigned int x, y, z;
};
struct dim3 {
    unsigned int x, y, z;
    constexpr dim3(unsigned int a = 1, unsigned int b = 1, unsigned int c = 1) : x(a), y(b), z(c) {}
};

namespace simt {

enum Collective { kShfl = 0, kShflDown = 1, kBallot = 2, kWarpSync = 3 };

const uint3& thread_index();
const uint3& block_index();
const dim3& block_dim();
const dim3& grid_dim();
// Deposits this lane's operand and waits for the warp; returns the lane's result.
uint64_t warp_collective(int kind, uint64_t value, int arg);
void block_barrier();
void* dynamic_shared();

struct Launch {
    dim3 grid, block;
    size_t shared;
    Launch(dim3 g, dim3 b, size_t s = 0, void* stream = nullptr) : grid(g), block(b), shared(s) { (void)stream; }
};
// Runs body() once per thread of every block of cfg.
void run(const Launch& cfg, const std::function<void()>& body);

// Counters of the last run(), for tests of the model itself.
struct Stats {
    uint64_t blocks, threads, collectives, barriers, inactive_sources, divergent;
};
Stats last_stats();

template <class T>
inline uint64_t bits_of(T v) {
    static_assert(sizeof(T) <= 8, "collective operand wider than 64 bits");
    uint64_t b = 0;
    std::memcpy(&b, &v, sizeof(T));
    return b;
}
template <class T>
inline T from_bits(uint64_t b) {
    T v;
    std::memcpy(&v, &b, sizeof(T));
    return v;
}

}  // namespace simt

#define threadIdx (::simt::thread_index())
#define blockIdx (::simt::block_index())
#define blockDim (::simt::block_dim())
#define gridDim (::simt::grid_dim())

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __noinline__
#define __launch_bounds__(...)
#define __shared__ static
#define __restrict__

// A warp sync inserted into the reference's source; each place has its own id.
#define SIMT_WARP_SYNC(id) ((void)::simt::warp_collective(::simt::kWarpSync, 0, (id)))

// Legacy (mask-less) warp intrinsics over the lanes that reach them.
template <class T>
inline T __shfl(T v, int src_lane, int width = 32) {
    assert(width == 32);
    (void)width;
    return simt::from_bits<T>(simt::warp_collective(simt::kShfl, simt::bits_of(v), src_lane));
}
template <class T>
inline T __shfl_down(T v, unsigned int delta, int width = 32) {
    assert(width == 32);
    (void)width;
    return simt::from_bits<T>(simt::warp_collective(simt::kShflDown, simt::bits_of(v), (int)delta));
}
inline unsigned int __ballot(int predicate) {
    return (unsigned int)simt::warp_collective(simt::kBallot, predicate != 0, 0);
}
inline void __syncthreads() { simt::block_barrier(); }
inline void __threadfence() {}
inline void __threadfence_block() {}

inline int __ffs(int x) { return x ? __builtin_ctz((unsigned int)x) + 1 : 0; }
inline int __popc(unsigned int x) { return __builtin_popcount(x); }
inline int __clz(int x) { return x ? __builtin_clz((unsigned int)x) : 32; }
inline int __clzll(long long int x) { return x ? __builtin_clzll((unsigned long long int)x) : 64; }

inline unsigned int atomicAdd(unsigned int* a, unsigned int v) {
    const unsigned int old = *a;
    *a = old + v;
    return old;
}
inline int atomicAdd(int* a, int v) {
    const int old = *a;
    *a = old + v;
    return old;
}
inline unsigned int atomicExch(unsigned int* a, unsigned int v) {
    const unsigned int old = *a;
    *a = v;
    return old;
}
inline int atomicExch(int* a, int v) {
    const int old = *a;
    *a = v;
    return old;
}

// Device-side min/max (CUDA's overloads; floats follow fminf/fmaxf).  Host
// translation units of the reference get its own macros instead.
#ifdef __CUDA_ARCH__
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline unsigned int min(unsigned int a, unsigned int b) { return a < b ? a : b; }
inline unsigned int max(unsigned int a, unsigned int b) { return a > b ? a : b; }
// Mixed signedness compares as unsigned, as CUDA's overloads do.
inline unsigned int min(int a, unsigned int b) { return min((unsigned int)a, b); }
inline unsigned int min(unsigned int a, int b) { return min(a, (unsigned int)b); }
inline unsigned int max(int a, unsigned int b) { return max((unsigned int)a, b); }
inline unsigned int max(unsigned int a, int b) { return max(a, (unsigned int)b); }
inline long long int min(long long int a, long long int b) { return a < b ? a : b; }
inline long long int max(long long int a, long long int b) { return a > b ? a : b; }
inline unsigned long long int min(unsigned long long int a, unsigned long long int b) { return a < b ? a : b; }
inline unsigned long long int max(unsigned long long int a, unsigned long long int b) { return a > b ? a : b; }
inline float min(float a, float b) { return fminf(a, b); }
inline float max(float a, float b) { return fmaxf(a, b); }
#endif
