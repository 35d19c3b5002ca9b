// Exclusive prefix sum of uint32 values (reduce, scan the tile sums, scan the
// tiles), used for deterministic output offsets.  Three short launches with no
// inter-block waiting: every tile's sum is read once, scanned by one block,
// and added back while the tiles are scanned.  Sums wrap modulo 2^32.

#include "common.cuh"
#include "internal.h"

namespace atr {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr int kSumThreads = 1024;

// Loads the kScanItems consecutive values of this thread (four 16-byte loads
// when the pointer allows; the L1 merges the warp's neighbouring halves).
__device__ __forceinline__ void load_items(const uint32_t* __restrict__ in, uint64_t n, uint64_t base, bool vec,
                                           uint32_t (&v)[kScanItems]) {
    if (vec) {
#pragma unroll
        for (int q = 0; q < kScanItems / 4; ++q) {
            const uint4 u = __ldg(reinterpret_cast<const uint4*>(in + base) + q);
            v[4 * q] = u.x;
            v[4 * q + 1] = u.y;
            v[4 * q + 2] = u.z;
            v[4 * q + 3] = u.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) v[k] = base + k < n ? in[base + k] : 0u;
    }
}

// Exclusive block scan of one value per thread; *block_total gets the sum.
template <int T>
__device__ __forceinline__ uint32_t block_exclusive(uint32_t x, uint32_t* s_warp, uint32_t* block_total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[w] = inc;
    __syncthreads();
    uint32_t wb = 0, tot = 0;
#pragma unroll
    for (int j = 0; j < T / 32; ++j) {
        const uint32_t s = s_warp[j];
        if (j < w) wb += s;
        tot += s;
    }
    *block_total = tot;
    return wb + inc - x;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_sums(const uint32_t* __restrict__ in, uint64_t n,
                                                            uint32_t* __restrict__ sums) {
    __shared__ uint32_t s_warp[kScanThreads / 32];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    const bool vec = (reinterpret_cast<uintptr_t>(in) & 15u) == 0 && base + kScanItems <= n;
    uint32_t v[kScanItems];
    load_items(in, n, base, vec, v);
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) s += v[k];
    s = __reduce_add_sync(kFull, s);
    if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
#pragma unroll
        for (int j = 0; j < kScanThreads / 32; ++j) t += s_warp[j];
        sums[blockIdx.x] = t;
    }
}

// One block: exclusive scan of the tile sums in place; *total gets their sum.
__global__ void __launch_bounds__(kSumThreads) k_scan_tiles(uint32_t* __restrict__ sums, uint32_t tiles,
                                                            uint32_t* __restrict__ total) {
    __shared__ uint32_t s_warp[kSumThreads / 32];
    const uint32_t per = (tiles + kSumThreads - 1) / kSumThreads;
    const uint32_t b = threadIdx.x * per;
    uint32_t own = 0;
    for (uint32_t k = 0; k < per; ++k)
        if (b + k < tiles) own += sums[b + k];
    uint32_t tot;
    uint32_t run = block_exclusive<kSumThreads>(own, s_warp, &tot);
    for (uint32_t k = 0; k < per; ++k)
        if (b + k < tiles) {
            const uint32_t x = sums[b + k];
            sums[b + k] = run;
            run += x;
        }
    if (total && threadIdx.x == 0) *total = tot;
}

__global__ void __launch_bounds__(kScanThreads) k_scan(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                       uint64_t n, const uint32_t* __restrict__ prefix) {
    __shared__ uint32_t s_warp[kScanThreads / 32];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    const bool vec = ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15u) == 0 &&
                     base + kScanItems <= n;
    uint32_t v[kScanItems];
    load_items(in, n, base, vec, v);
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) sum += v[k];
    uint32_t tot;
    uint32_t run = prefix[blockIdx.x] + block_exclusive<kScanThreads>(sum, s_warp, &tot);
    if (vec) {
#pragma unroll
        for (int q = 0; q < kScanItems / 4; ++q) {
            uint4 u;
            u.x = run; run += v[4 * q];
            u.y = run; run += v[4 * q + 1];
            u.z = run; run += v[4 * q + 2];
            u.w = run; run += v[4 * q + 3];
            reinterpret_cast<uint4*>(out + base)[q] = u;
        }
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            if (base + k < n) out[base + k] = run;
            run += v[k];
        }
    }
}

__global__ void __launch_bounds__(256) k_zero_words(uint32_t* __restrict__ p, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        p[i] = 0u;
}

}  // namespace

// Zeroes `words` 32-bit words on the context's stream with a kernel.  Inside a
// captured graph a small memset node between two kernels cost 5-17 us of idle
// device time (measured at the LBVH and level-list histograms); a kernel node
// follows its neighbours without that hand-off.
int zero_words_async(atr_ctx* ctx, uint32_t* p, size_t words) {
    if (words == 0) return ATR_OK;
    const size_t want = (words + 255) / 256, cap = (size_t)ctx->num_sms * 8;
    k_zero_words<<<(unsigned)(want < cap ? want : cap), 256, 0, ctx->stream>>>(p, words);
    ctx->launches += 1;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "k_zero_words", __FILE__, __LINE__);
    return ATR_OK;
}

// out may equal in: every thread reads its own values before it writes them.
int exclusive_scan_u32(atr_ctx* ctx, const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* d_total) {
    if (n == 0) return ATR_OK;
    const uint64_t tiles = (n + kScanTile - 1) / kScanTile;
    ATR_REQUIRE(tiles <= (1ull << 31), ATR_ERR_INVALID_ARG, "exclusive_scan_u32: %llu values",
                (unsigned long long)n);
    void* tmp = nullptr;
    ATR_TRY(ctx->alloc(&tmp, tiles * 4));
    uint32_t* sums = static_cast<uint32_t*>(tmp);
    cudaStream_t s = ctx->stream;
    k_scan_sums<<<(unsigned)tiles, kScanThreads, 0, s>>>(in, n, sums);
    k_scan_tiles<<<1, kSumThreads, 0, s>>>(sums, (uint32_t)tiles, d_total);
    k_scan<<<(unsigned)tiles, kScanThreads, 0, s>>>(in, out, n, sums);
    ctx->launches += 3;
    cudaError_t e = cudaGetLastError();
    ctx->release(tmp);
    if (e != cudaSuccess) return cuda_fail(e, "k_scan launch", __FILE__, __LINE__);
    return ATR_OK;
}

}  // namespace atr
