// Exclusive prefix sum of uint32 values in one pass (decoupled look-back over
// 4096-element tiles), used for deterministic output offsets.  Totals must
// stay below 2^30.

#include "common.cuh"
#include "internal.h"

namespace atr {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr uint32_t kAgg = 0x40000000u, kInc = 0x80000000u, kVal = 0x3fffffffu;
constexpr uint32_t kPollLimit = 1u << 26;

__global__ void __launch_bounds__(kScanThreads) k_scan(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                       uint64_t n, uint32_t* __restrict__ status,
                                                       uint32_t* __restrict__ ticket, uint32_t* __restrict__ total,
                                                       uint32_t* __restrict__ err) {
    __shared__ uint32_t s_tile, s_prefix;
    __shared__ uint32_t s_warp[kScanThreads / 32];
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    // Each thread owns kScanItems consecutive values: four 16-byte loads when
    // the pointers allow it (the L1 merges the warp's neighbouring halves).
    const bool vec = ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15u) == 0 &&
                     base + kScanItems <= n;
    uint32_t v[kScanItems];
    if (vec) {
#pragma unroll
        for (int q = 0; q < kScanItems / 4; ++q) {
            const uint4 u = __ldg(reinterpret_cast<const uint4*>(in + base) + q);
            v[4 * q] = u.x; v[4 * q + 1] = u.y; v[4 * q + 2] = u.z; v[4 * q + 3] = u.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) v[k] = base + k < n ? in[base + k] : 0u;
    }
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) sum += v[k];
    // Block exclusive scan of the per-thread sums.
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[w] = inc;
    __syncthreads();
    uint32_t wb = 0, tile_sum = 0;
#pragma unroll
    for (int j = 0; j < kScanThreads / 32; ++j) {
        if (j < w) wb += s_warp[j];
        tile_sum += s_warp[j];
    }
    const uint32_t excl = wb + inc - sum;
    // Decoupled look-back by warp 0, 32 predecessors per step: the nearest
    // inclusive prefix plus the aggregates between it and this tile.
    if (w == 0) {
        uint32_t prefix = 0;
        if (tile == 0) {
            if (lane == 0) __stcg(status, kInc | tile_sum);
        } else {
            if (lane == 0) __stcg(status + tile, kAgg | tile_sum);
            int64_t top = (int64_t)tile - 1;
            uint32_t polls = 0;
            while (true) {
                const int64_t k = top - lane;
                const uint32_t st = k >= 0 ? *reinterpret_cast<volatile uint32_t*>(status + k) : kInc;
                if (__any_sync(kFull, (st & (kAgg | kInc)) == 0u)) {
                    if (++polls > kPollLimit) {
                        if (lane == 0) set_error_bits(err, kErrCollapse);
                        break;
                    }
                    continue;
                }
                const uint32_t incs = __ballot_sync(kFull, (st & kInc) != 0u);
                if (incs) {
                    const int first = __ffs(incs) - 1;
                    prefix += __reduce_add_sync(kFull, lane <= first ? (st & kVal) : 0u);
                    break;
                }
                prefix += __reduce_add_sync(kFull, st & kVal);
                top -= 32;
            }
            if (lane == 0) __stcg(status + tile, kInc | (prefix + tile_sum));
        }
        if (lane == 0) {
            s_prefix = prefix;
            if (total && (uint64_t)(tile + 1) * kScanTile >= n) *total = prefix + tile_sum;
        }
    }
    __syncthreads();
    uint32_t run = s_prefix + excl;
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

}  // namespace

int exclusive_scan_u32(atr_ctx* ctx, const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* d_total) {
    if (n == 0) return ATR_OK;
    const uint64_t tiles = (n + kScanTile - 1) / kScanTile;
    void* tmp = nullptr;
    ATR_TRY(ctx->alloc(&tmp, align256(tiles * 4) + 256));
    uint32_t* status = static_cast<uint32_t*>(tmp);
    uint32_t* ticket = reinterpret_cast<uint32_t*>(static_cast<char*>(tmp) + align256(tiles * 4));
    cudaMemsetAsync(tmp, 0, align256(tiles * 4) + 256, ctx->stream);
    k_scan<<<(unsigned)tiles, kScanThreads, 0, ctx->stream>>>(in, out, n, status, ticket, d_total, ctx->d_error);
    ctx->launches += 1;
    cudaError_t e = cudaGetLastError();
    ctx->release(tmp);
    if (e != cudaSuccess) return cuda_fail(e, "k_scan launch", __FILE__, __LINE__);
    return ATR_OK;
}

}  // namespace atr
