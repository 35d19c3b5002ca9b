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
    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? in[base + k] : 0u;
        sum += v[k];
    }
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
    for (int j = 0; j < kScanThreads / 32; ++j) {
        if (j < w) wb += s_warp[j];
        tile_sum += s_warp[j];
    }
    const uint32_t excl = wb + inc - sum;
    if (threadIdx.x == 0) {
        uint32_t prefix = 0;
        if (tile == 0) {
            __stcg(status, kInc | tile_sum);
        } else {
            __stcg(status + tile, kAgg | tile_sum);
            int64_t k = (int64_t)tile - 1;
            uint32_t polls = 0;
            while (k >= 0) {
                const uint32_t s = *reinterpret_cast<volatile uint32_t*>(status + k);
                if (s & kInc) { prefix += s & kVal; break; }
                if (s & kAgg) { prefix += s & kVal; --k; continue; }
                if (++polls > kPollLimit) { set_error_bits(err, kErrCollapse); break; }
            }
            __stcg(status + tile, kInc | (prefix + tile_sum));
        }
        s_prefix = prefix;
        if (total && (uint64_t)(tile + 1) * kScanTile >= n) *total = prefix + tile_sum;
    }
    __syncthreads();
    uint32_t run = s_prefix + excl;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
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
