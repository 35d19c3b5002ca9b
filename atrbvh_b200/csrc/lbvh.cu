// LBVH construction on sm_100a:
//   scene bounds  -> Morton codes (+ all radix-digit histograms in the same pass)
//   -> LSD radix sort of (key, triangle index): tile counts, tile prefixes, scatter
//   -> one bottom-up pass that builds the Karras radix tree and refits its
//      boxes at the same time.
//
// The tree is bit-identical to the reference's two-kernel build
// (BVHRT-Core/src/LBVH.cu:208-316 topology, :465-570 refit): the binary radix
// tree over the (key, index) pairs is unique, and internal node numbering
// follows Karras (a node covering [l, r] is stored at r when it is its
// parent's left child and at l when it is the right child; the root at 0).

#include <climits>
#include <cstdio>
#include <utility>

#include "common.cuh"
#include "internal.h"

namespace atr {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 12;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kSortWarps = kSortThreads / 32;

// Digit plan of an LSD sort of K keys with BITS-bit digits.  8-bit digits
// cover every key bit (4 passes for uint32, 8 for uint64).  10-bit digits are
// used for Morton codes only, whose top bits are always zero: 30-bit codes in
// uint32 take 3 passes and 63-bit codes in uint64 take 7.
template <typename K, int BITS>
struct SortPlan {
    static_assert(BITS == 8 || BITS == 10, "digit width");
    static constexpr int kDigits = 1 << BITS;
    static constexpr int kPasses = BITS == 8 ? (int)sizeof(K) : (sizeof(K) == 4 ? 3 : 7);
    static constexpr int kPerThread = kDigits / kSortThreads;  // digits per thread in tile-wide steps
    // Dynamic shared memory of one scatter block: the tile's keys and
    // values, per-warp digit counters, digit starts and global bases.
    static constexpr size_t kSmem = (size_t)kSortTile * (sizeof(K) + 4) + (size_t)(kSortWarps + 2) * kDigits * 4;
};

// ---- scene bounds (SceneConverter.cpp:28-60 on the device) -----------------
__global__ void __launch_bounds__(256) k_bounds_partial(const float4* __restrict__ v, uint64_t nv,
                                                         float* __restrict__ partial) {
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float mx[3] = {FLT_MIN, FLT_MIN, FLT_MIN};
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nv;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float4 p = __ldg(v + i);
        mn[0] = fminf(mn[0], p.x); mn[1] = fminf(mn[1], p.y); mn[2] = fminf(mn[2], p.z);
        mx[0] = fmaxf(mx[0], p.x); mx[1] = fmaxf(mx[1], p.y); mx[2] = fmaxf(mx[2], p.z);
    }
    for (int o = 16; o > 0; o >>= 1)
        for (int k = 0; k < 3; ++k) {
            mn[k] = fminf(mn[k], __shfl_xor_sync(kFull, mn[k], o));
            mx[k] = fmaxf(mx[k], __shfl_xor_sync(kFull, mx[k], o));
        }
    __shared__ float s[8][6];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 3; ++k) { s[w][k] = mn[k]; s[w][3 + k] = mx[k]; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int j = 1; j < (int)(blockDim.x >> 5); ++j)
            for (int k = 0; k < 3; ++k) {
                s[0][k] = fminf(s[0][k], s[j][k]);
                s[0][3 + k] = fmaxf(s[0][3 + k], s[j][3 + k]);
            }
        for (int k = 0; k < 6; ++k) partial[blockIdx.x * 6 + k] = s[0][k];
    }
}

__global__ void k_bounds_final(const float* __restrict__ partial, int np, float* __restrict__ out) {
    if (threadIdx.x != 0) return;
    float r[6] = {FLT_MAX, FLT_MAX, FLT_MAX, FLT_MIN, FLT_MIN, FLT_MIN};
    for (int j = 0; j < np; ++j)
        for (int k = 0; k < 3; ++k) {
            r[k] = fminf(r[k], partial[j * 6 + k]);
            r[3 + k] = fmaxf(r[3 + k], partial[j * 6 + 3 + k]);
        }
    for (int k = 0; k < 6; ++k) out[k] = r[k];
}

// ---- Morton codes (LBVH.cu:14-97, Commons.cuh:426-510,606-662) ---------------
__device__ __forceinline__ uint32_t expand10(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
__device__ __forceinline__ uint64_t expand21(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}

template <typename K>
__device__ __forceinline__ K morton_code(float cx, float cy, float cz, const float* b);

template <>
__device__ __forceinline__ uint32_t morton_code<uint32_t>(float cx, float cy, float cz, const float* b) {
    const float c[3] = {cx, cy, cz};
    uint32_t q[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float nrm = __fdiv_rn(__fsub_rn(c[k], b[k]), __fsub_rn(b[3 + k], b[k]));
        q[k] = expand10(__float2uint_rz(fminf(fmaxf(__fmul_rn(nrm, 1024.0f), 0.0f), 1023.0f)));
    }
    return q[0] * 4u + q[1] * 2u + q[2];
}
template <>
__device__ __forceinline__ uint64_t morton_code<uint64_t>(float cx, float cy, float cz, const float* b) {
    const float c[3] = {cx, cy, cz};
    uint64_t q[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float nrm = __fdiv_rn(__fsub_rn(c[k], b[k]), __fsub_rn(b[3 + k], b[k]));
        q[k] = expand21(__float2ull_rz(fminf(fmaxf(__fmul_rn(nrm, 2097152.0f), 0.0f), 2097151.0f)));
    }
    return q[0] * 4u + q[1] * 2u + q[2];
}

// One block per sort tile (kSortTile triangles of one mesh); histograms of
// every digit of every pass are accumulated in shared memory and added to the
// mesh's histograms (P x D per mesh) once per block; the block's own counts
// of the first pass's digits are the sort's first tile counts (D per tile in
// tile_counts).  Each mesh is normalised to its own box (6 floats per mesh
// in `bounds`).
template <typename K, int BITS>
__global__ void __launch_bounds__(256) k_morton(Segs segs, const float4* __restrict__ v,
                                                 const float* __restrict__ bounds, K* __restrict__ keys,
                                                 uint32_t* __restrict__ hist, uint32_t* __restrict__ tile_counts,
                                                 PrimBoxes pr) {
    constexpr int P = SortPlan<K, BITS>::kPasses, D = SortPlan<K, BITS>::kDigits;
    __shared__ uint32_t sh[P * D];
    __shared__ float sb[6];
    const uint32_t m = segs.seg_of_tile(blockIdx.x);
    const uint32_t t0 = segs.tri_begin(m) + (blockIdx.x - segs.tile_begin(m)) * kSortTile;
    const uint32_t t1 = min(t0 + kSortTile, segs.tri_end(m));
    for (int j = threadIdx.x; j < P * D; j += blockDim.x) sh[j] = 0;
    if (threadIdx.x < 6) sb[threadIdx.x] = bounds[6 * m + threadIdx.x];
    __syncthreads();
    for (uint32_t t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
        float cx, cy, cz;
        if (pr.bmin) {
            // A primitive box's centroid, (min + max) / 2 (LBVH.cu:41-49; the
            // halving is exact, so it equals the product by 0.5).
            const float4 lo = __ldg(pr.bmin + t), hi = __ldg(pr.bmax + t);
            cx = __fmul_rn(__fadd_rn(lo.x, hi.x), 0.5f);
            cy = __fmul_rn(__fadd_rn(lo.y, hi.y), 0.5f);
            cz = __fmul_rn(__fadd_rn(lo.z, hi.z), 0.5f);
        } else {
            const float4 a = __ldg(v + 3 * (size_t)t), b = __ldg(v + 3 * (size_t)t + 1), c = __ldg(v + 3 * (size_t)t + 2);
            cx = __fmul_rn(__fadd_rn(fmaxf(fmaxf(a.x, b.x), c.x), fminf(fminf(a.x, b.x), c.x)), 0.5f);
            cy = __fmul_rn(__fadd_rn(fmaxf(fmaxf(a.y, b.y), c.y), fminf(fminf(a.y, b.y), c.y)), 0.5f);
            cz = __fmul_rn(__fadd_rn(fmaxf(fmaxf(a.z, b.z), c.z), fminf(fminf(a.z, b.z), c.z)), 0.5f);
        }
        const K code = morton_code<K>(cx, cy, cz, sb);
        keys[t] = code;
        if (hist) {
#pragma unroll
            for (int p = 0; p < P; ++p) atomicAdd(&sh[p * D + (uint32_t)((code >> (BITS * p)) & (D - 1))], 1u);
        }
    }
    if (!hist) return;
    __syncthreads();
    for (int j = threadIdx.x; j < P * D; j += blockDim.x)
        if (sh[j]) atomicAdd(&hist[(size_t)m * P * D + j], sh[j]);
    if (tile_counts)
        for (int j = threadIdx.x; j < D; j += blockDim.x) tile_counts[(size_t)blockIdx.x * D + j] = sh[j];
}

// 8-bit digit histograms of arbitrary keys (the generic sort entry point).
template <typename K>
__global__ void __launch_bounds__(256) k_histogram(const K* __restrict__ keys, uint32_t n,
                                                    uint32_t* __restrict__ hist) {
    constexpr int P = SortPlan<K, 8>::kPasses;
    __shared__ uint32_t sh[P * 256];
    for (int j = threadIdx.x; j < P * 256; j += blockDim.x) sh[j] = 0;
    __syncthreads();
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const K code = keys[t];
#pragma unroll
        for (int p = 0; p < P; ++p) atomicAdd(&sh[p * 256 + (uint32_t)((code >> (8 * p)) & 255u)], 1u);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < P * 256; j += blockDim.x)
        if (sh[j]) atomicAdd(&hist[j], sh[j]);
}

// Exclusive scan of 256 values held one per thread of a 256-thread block.
__device__ __forceinline__ uint32_t block_exclusive_scan256(uint32_t x, uint32_t* s_warp) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[w] = inc;
    __syncthreads();
    uint32_t wbase = 0;
    for (int j = 0; j < w; ++j) wbase += s_warp[j];
    __syncthreads();
    return wbase + inc - x;
}

// Exclusive scan over the block of R consecutive values per thread (thread t
// holds values t*R .. t*R+R-1).
template <int R>
__device__ __forceinline__ void block_exclusive_scan(const uint32_t (&x)[R], uint32_t (&out)[R], uint32_t* s_warp) {
    uint32_t tot = 0;
#pragma unroll
    for (int r = 0; r < R; ++r) tot += x[r];
    uint32_t run = block_exclusive_scan256(tot, s_warp);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        out[r] = run;
        run += x[r];
    }
}

// ---- radix sort pass: tile counts -> tile prefixes -> scatter -----------------
// A pass over keys already split into tiles of kSortTile (a tile holds keys of
// one mesh only):
//   k_tile_counts  every tile's digit counts (pass 0 of an LBVH build takes
//                  them from k_morton instead);
//   k_tile_prefix  in place, the exclusive sum of each digit's counts over the
//                  mesh's earlier tiles (a segmented scan down every digit's
//                  column);
//   k_scatter      ranks the tile's keys, adds the tile prefix to the mesh's
//                  digit start and writes every key to its place.
// Each scatter block finds its offsets ready, so no tile waits on another
// (the decoupled look-back this replaces spent a third of every pass walking
// over the aggregates of the tiles running beside it).

// Tile counts of digit `pass` (D per tile, tile-major).  A thread loads its
// kSortItems keys at once and counts them with shared atomics into its warp's
// own histogram (no ranks are needed here); the warps' histograms are summed
// at the end.
template <typename K, int BITS>
__global__ void __launch_bounds__(kSortThreads) k_tile_counts(Segs segs, const K* __restrict__ keys, int pass,
                                                               uint32_t* __restrict__ counts) {
    constexpr int D = SortPlan<K, BITS>::kDigits;
    __shared__ uint32_t sh[kSortWarps][D];
    const int shift = BITS * pass;
    const uint32_t tile = blockIdx.x;
    const uint32_t m = segs.seg_of_tile(tile);
    const uint32_t base = segs.tri_begin(m) + (tile - segs.tile_begin(m)) * kSortTile;
    const uint32_t end = min(base + (uint32_t)kSortTile, segs.tri_end(m));
    for (int j = threadIdx.x; j < kSortWarps * D; j += kSortThreads) (&sh[0][0])[j] = 0;
    uint32_t dg[kSortItems];
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t i = base + r * kSortThreads + threadIdx.x;
        dg[r] = i < end ? (uint32_t)((keys[i] >> shift) & (D - 1)) : (uint32_t)D;
    }
    __syncthreads();
    uint32_t* const wh = sh[threadIdx.x >> 5];
#pragma unroll
    for (int r = 0; r < kSortItems; ++r)
        if (dg[r] < (uint32_t)D) atomicAdd(&wh[dg[r]], 1u);
    __syncthreads();
    for (int j = threadIdx.x; j < D; j += kSortThreads) {
        uint32_t c = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) c += sh[w][j];
        counts[(size_t)tile * D + j] = c;
    }
}

// In place: counts[t][d] -> the sum of counts[t'][d] over the earlier tiles
// t' of t's mesh within t's chunk of kPrefixChunk tiles.  Block (x, y) takes
// 32 digits (one per lane) and chunk y, split into 32 runs of 8 tiles (one
// per warp): run sums, a segmented scan of the run sums in shared memory (a
// run holding a mesh's first tile restarts the sum), then each run again from
// its carry.  The chunk's segmented total (sum since its last mesh start, top
// bit set when it holds one) goes to chunk_tot; k_chunk_carry turns those
// into each chunk's carry from earlier chunks, which the scatter adds for a
// tile whose mesh began before its chunk.
constexpr int kPrefixRuns = 32;
constexpr int kPrefixRunTiles = 8;
constexpr uint32_t kPrefixChunk = kPrefixRuns * kPrefixRunTiles;
constexpr uint32_t kCutBit = 0x80000000u;

// Tile of the next mesh start after mesh m (none: ~0).
__device__ __forceinline__ uint32_t next_mesh_tile(const Segs& segs, uint32_t m) {
    return m + 1 < segs.count ? segs.tile_begin(m + 1) : 0xffffffffu;
}

template <int D>
__global__ void __launch_bounds__(32 * kPrefixRuns) k_tile_prefix(Segs segs, uint32_t tiles,
                                                                   uint32_t* __restrict__ counts,
                                                                   uint32_t* __restrict__ chunk_tot) {
    __shared__ uint32_t s_sum[kPrefixRuns][32];
    __shared__ uint8_t s_cut[kPrefixRuns][32];
    const int lane = threadIdx.x & 31, run = threadIdx.x >> 5;
    const uint32_t d = blockIdx.x * 32 + lane;
    const uint32_t c0 = blockIdx.y * kPrefixChunk;
    const uint32_t t0 = min(tiles, c0 + run * kPrefixRunTiles), t1 = min(tiles, t0 + kPrefixRunTiles);
    const uint32_t m0 = t0 < t1 ? segs.seg_of_tile(t0) : 0;
    const bool starts = t0 < t1 && t0 == segs.tile_begin(m0);  // the run begins a mesh
    const uint32_t next0 = t0 < t1 ? next_mesh_tile(segs, m0) : 0xffffffffu;
    uint32_t v[kPrefixRunTiles];
#pragma unroll
    for (int u = 0; u < kPrefixRunTiles; ++u) v[u] = t0 + u < t1 ? counts[(size_t)(t0 + u) * D + d] : 0u;
    uint32_t sum = 0;
    bool cut = starts;
    {
        uint32_t m = m0, next = next0;
#pragma unroll
        for (int u = 0; u < kPrefixRunTiles; ++u) {
            if (t0 + u < t1 && t0 + u == next) {  // a mesh starts here: the run's sum restarts
                sum = 0;
                cut = true;
                next = next_mesh_tile(segs, ++m);
            }
            sum += v[u];
        }
    }
    s_sum[run][lane] = sum;
    s_cut[run][lane] = cut;
    __syncthreads();
    // Carry into this run from the chunk's earlier runs, back to the last cut.
    uint32_t carry = 0;
    if (!starts)
        for (int r = run - 1; r >= 0; --r) {
            carry += s_sum[r][lane];
            if (s_cut[r][lane]) break;
        }
    if (run == kPrefixRuns - 1) {
        bool any = false;
        for (int r = 0; r < kPrefixRuns; ++r) any |= s_cut[r][lane] != 0;
        chunk_tot[(size_t)blockIdx.y * D + d] = (cut ? sum : carry + sum) | (any ? kCutBit : 0u);
    }
    uint32_t acc = carry;
    uint32_t m = m0, next = next0;
#pragma unroll
    for (int u = 0; u < kPrefixRunTiles; ++u) {
        if (t0 + u >= t1) break;
        if (t0 + u == next) {
            acc = 0;
            next = next_mesh_tile(segs, ++m);
        }
        counts[(size_t)(t0 + u) * D + d] = acc;
        acc += v[u];
    }
}

// In place over the chunk totals: chunk_tot[y][d] -> the segmented sum of the
// earlier chunks' totals (what a tile of chunk y whose mesh began before the
// chunk adds to its prefix).  One thread per digit walks the chunks.
template <int D>
__global__ void __launch_bounds__(256) k_chunk_carry(uint32_t chunks, uint32_t* __restrict__ chunk_tot) {
    const uint32_t d = blockIdx.x * 256 + threadIdx.x;
    if (d >= (uint32_t)D) return;
    uint32_t acc = 0;
    for (uint32_t y0 = 0; y0 < chunks; y0 += 8) {
        uint32_t v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = y0 + u < chunks ? chunk_tot[(size_t)(y0 + u) * D + d] : 0u;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if (y0 + u >= chunks) break;
            chunk_tot[(size_t)(y0 + u) * D + d] = acc;
            acc = (v[u] & kCutBit) ? (v[u] & ~kCutBit) : acc + v[u];
        }
    }
}

// Stable scatter of one tile: keys of one digit keep their input order
// (each warp ranks a contiguous run of the tile in order, warps in order).
// Segmented: keys move only within their mesh (hist holds P x D counts per
// mesh, prefix the tile's offsets within its chunk from k_tile_prefix,
// chunk_carry the chunk's carry for tiles whose mesh began before the chunk).  Each
// thread owns R = D / 256 consecutive digits in the tile-wide steps.
template <typename K, bool kIota, int BITS>
__global__ void __launch_bounds__(kSortThreads, sizeof(K) == 4 ? 4 : 3) k_scatter(
        Segs segs, const K* __restrict__ kin, const uint32_t* __restrict__ vin, K* __restrict__ kout,
        uint32_t* __restrict__ vout, int pass, const uint32_t* __restrict__ hist,
        const uint32_t* __restrict__ prefix, const uint32_t* __restrict__ chunk_carry) {
    using Plan = SortPlan<K, BITS>;
    constexpr int P = Plan::kPasses, D = Plan::kDigits, R = Plan::kPerThread;
    const int shift = BITS * pass;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K* s_keys = reinterpret_cast<K*>(smem_raw);
    uint32_t* s_vals = reinterpret_cast<uint32_t*>(s_keys + kSortTile);
    uint32_t* s_wh = s_vals + kSortTile;         // [kSortWarps][D] per-warp digit counters
    uint32_t* s_dstart = s_wh + kSortWarps * D;  // [D] digit start within the tile
    uint32_t* s_gbase = s_dstart + D;            // [D] output base minus digit start
    __shared__ uint32_t s_scan[kSortWarps];

    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int j = threadIdx.x; j < kSortWarps * D; j += kSortThreads) s_wh[j] = 0;
    __syncthreads();
    const uint32_t tile = blockIdx.x;
    const uint32_t m = segs.seg_of_tile(tile);
    const uint32_t seg_start = segs.tri_begin(m), seg_end = segs.tri_end(m);
    const uint32_t base = seg_start + (tile - segs.tile_begin(m)) * kSortTile;
    const uint32_t valid_n = min((uint32_t)kSortTile, seg_end - base);
    const uint32_t end = base + valid_n;

    K key[kSortItems];
    uint32_t val[kSortItems];
    uint32_t rank[kSortItems];
    const uint32_t lt = lanemask_lt();
    uint32_t* const wh = s_wh + w * D;
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t idx = base + (uint32_t)w * (kSortItems * 32) + r * 32 + lane;
        const bool valid = idx < end;
        key[r] = valid ? kin[idx] : (K)0;
        val[r] = kIota ? (uint32_t)idx : (valid ? vin[idx] : 0u);
    }
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const bool valid = base + (uint32_t)w * (kSortItems * 32) + r * 32 + lane < end;
        const uint32_t d = valid ? (uint32_t)((key[r] >> shift) & (D - 1)) : (uint32_t)D;
        const uint32_t peers = __match_any_sync(kFull, d);
        const uint32_t before = __popc(peers & lt);
        uint32_t cnt = 0;
        if (valid) cnt = wh[d];
        __syncwarp();
        if (valid && before == 0) wh[d] = cnt + __popc(peers);
        __syncwarp();
        rank[r] = valid ? cnt + before : 0xffffffffu;
    }
    __syncthreads();

    // Per-digit exclusive offsets across warps, tile totals, digit starts.
    uint32_t count[R], hv[R], dstart[R], gdig[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int d = threadIdx.x * R + r;
        uint32_t run = 0;
#pragma unroll
        for (int j = 0; j < kSortWarps; ++j) {
            const uint32_t c = s_wh[j * D + d];
            s_wh[j * D + d] = run;
            run += c;
        }
        count[r] = run;
        hv[r] = hist[((size_t)m * P + pass) * D + d];
    }
    block_exclusive_scan<R>(count, dstart, s_scan);
    block_exclusive_scan<R>(hv, gdig, s_scan);
    const uint32_t chunk = tile / kPrefixChunk, chunk0 = chunk * kPrefixChunk;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int d = threadIdx.x * R + r;
        s_dstart[d] = dstart[r];
        const uint32_t carry = segs.tile_begin(m) < chunk0 ? chunk_carry[(size_t)chunk * D + d] : 0u;
        s_gbase[d] = seg_start + gdig[r] + prefix[(size_t)tile * D + d] + carry - dstart[r];
    }
    __syncthreads();

    // Scatter into shared memory in digit order, then write out coalesced.
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        if (rank[r] == 0xffffffffu) continue;
        const uint32_t dd = (uint32_t)((key[r] >> shift) & (D - 1));
        const uint32_t p = s_dstart[dd] + wh[dd] + rank[r];
        s_keys[p] = key[r];
        s_vals[p] = val[r];
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < valid_n; i += kSortThreads) {
        const K kk = s_keys[i];
        const uint32_t dd = (uint32_t)((kk >> shift) & (D - 1));
        const uint32_t dst = s_gbase[dd] + i;
        if (dst >= seg_start && dst < seg_end) {  // holds whenever hist matches the keys
            kout[dst] = kk;
            vout[dst] = s_vals[i];
        }
    }
}

// ---- fused Karras build + refit ------------------------------------------------
// Common prefix of the adjacent sorted pairs (k, k+1) with the reference's
// index tie-break (LBVH.cu:163-201).
__device__ __forceinline__ int delta_adj(const uint32_t* keys, int k) {
    const uint32_t a = keys[k], b = keys[k + 1];
    return a == b ? 32 + __clz(k ^ (k + 1)) : __clz(a ^ b);
}
__device__ __forceinline__ int delta_adj(const uint64_t* keys, int k) {
    const uint64_t a = keys[k], b = keys[k + 1];
    return a == b ? 64 + __clzll((long long)(k ^ (k + 1))) : __clzll((long long)(a ^ b));
}

// One thread per sorted leaf climbs while it is the second of two siblings to
// arrive (an atomic exchange on the parent's split position carries the
// first arrival's far range end).  Each node's record is written once.
// Segmented: thread i finds its mesh; keys, slots and node arrays are
// addressed from the mesh's first entry, so every mesh gets exactly the tree
// a build of that mesh alone produces (local node and triangle indices).
//
// Two passes.  k_build_block: a block owns 256 consecutive sorted leaves and
// finishes every node whose split position and the one after it lie in its
// range, with the arrival slots, the adjacent-key deltas and the finished
// boxes in shared memory.  Such a node's children lie in the block, so the
// climb meets no other block.  A climb that reaches a split on the block's
// first or last leaf stops and is recorded (at most one per block edge); at
// the end the block writes its slots, a single arrival or -1, to the global
// slot array.  k_build_top continues the recorded climbs with global atomic
// exchanges; a slot written by the block pass carries its first arrival.
struct BuildEdge {
    int32_t mesh, node, l, r;  // mesh < 0: no climb stopped at this edge
};

template <typename K>
struct BuildOut {
    int32_t *parent, *left, *right, *data;
    float4 *bmin, *bmax;
    float* area;
    int32_t* slot;
    int2* range;
    BuildPrepass pp;
};

// Record of the internal node p over leaves [pl, pr] with children lc, rc
// (the children's parent links are the caller's).
template <typename K>
__device__ __forceinline__ void write_inner(const BuildOut<K>& o, const Segs& segs, uint32_t m, int nb, int p, int pl,
                                            int pr, int lc, int rc, float4 mn, float4 mx, float pa, float ns,
                                            int lvl) {
    o.left[nb + p] = lc;
    o.right[nb + p] = rc;
    o.data[nb + p] = -1;
    if (o.range) o.range[segs.inner_base(m) + p] = make_int2(pl, pr);
    o.bmin[nb + p] = mn;
    o.bmax[nb + p] = mx;
    o.area[nb + p] = pa;
    if (o.pp.rec) {
        const int cnt = pr - pl + 1;
        const int gam = o.pp.seg_gamma ? (int)o.pp.seg_gamma[m] : o.pp.gamma;
        o.pp.rec[nb + p] = make_int4(cnt, __float_as_int(ns), cnt < gam ? __float_as_int(ns) : 0, lvl);
    }
}

constexpr int kBuildBlock = 256;

template <typename K>
__global__ void __launch_bounds__(kBuildBlock) k_build_block(Segs segs, const K* __restrict__ keys_all,
                                                             const uint32_t* __restrict__ sidx,
                                                             const float4* __restrict__ verts, BuildOut<K> o,
                                                             BuildEdge* __restrict__ edges, PrimBoxes pr) {
    __shared__ float4 s_lmn[kBuildBlock], s_lmx[kBuildBlock], s_imn[kBuildBlock], s_imx[kBuildBlock];
    __shared__ float s_lns[kBuildBlock], s_ins[kBuildBlock];
    __shared__ int s_ilv[kBuildBlock];  // prepass levels of the block's finished internal nodes
    __shared__ int s_slot[kBuildBlock];
    __shared__ int s_delta[kBuildBlock + 1];  // delta at sorted position B0 - 1 + k
    // Records of the internal nodes the block finishes, by block position
    // (internal node p of a mesh sits at its sorted position p), and the
    // parents it assigns: written out coalesced once the block's climbs end.
    __shared__ int s_left[kBuildBlock], s_right[kBuildBlock];  // kUnset: not finished here
    __shared__ int2 s_rng[kBuildBlock];
    __shared__ int s_ipar[kBuildBlock], s_lpar[kBuildBlock];   // parents of internal node / leaf
    constexpr int kUnset = INT_MIN;
    const int tid = threadIdx.x;
    const uint32_t B0 = blockIdx.x * kBuildBlock;
    const uint32_t gi = B0 + tid;
    const bool live = gi < segs.n;
    s_slot[tid] = -1;
    s_left[tid] = kUnset;
    s_ipar[tid] = kUnset;
    s_lpar[tid] = kUnset;
    if (tid < 2) edges[2 * blockIdx.x + tid] = BuildEdge{-1, -1, -1, -1};
    uint32_t m = 0, s0 = 0, n = 1, i = 0;
    int nb = 0, last = 0;
    const K* keys = keys_all;
    float4 mn = make_float4(0.f, 0.f, 0.f, 0.f), mx = mn;
    float my_ns = 0.0f;
    s_delta[tid] = -1;
    if (tid == kBuildBlock - 1) s_delta[kBuildBlock] = -1;
    if (live) {
        m = segs.seg_of_tri(gi);
        s0 = segs.tri_begin(m);
        n = segs.tri_end(m) - s0;
        i = gi - s0;
        nb = segs.node_base(m);
        last = (int)n - 1;
        keys = keys_all + s0;
        const uint32_t gtri = sidx[gi];
        int32_t dat;
        if (pr.bmin) {
            // A primitive's leaf: its box and its triangle (LBVH.cu:372-397,
            // :600-611 through the routing index).
            const float4 lo = __ldg(pr.bmin + gtri), hi = __ldg(pr.bmax + gtri);
            mn = make_float4(lo.x, lo.y, lo.z, 0.0f);
            mx = make_float4(hi.x, hi.y, hi.z, 0.0f);
            dat = (int32_t)__ldg(pr.data + gtri);
        } else {
            const float4 a = __ldg(verts + 3 * (size_t)gtri), b = __ldg(verts + 3 * (size_t)gtri + 1),
                         c = __ldg(verts + 3 * (size_t)gtri + 2);
            mn = make_float4(fminf(fminf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y), fminf(fminf(a.z, b.z), c.z),
                             0.0f);
            mx = make_float4(fmaxf(fmaxf(a.x, b.x), c.x), fmaxf(fmaxf(a.y, b.y), c.y), fmaxf(fmaxf(a.z, b.z), c.z),
                             0.0f);
            dat = (int32_t)(gtri - s0);
        }
        const int leaf = (int)i + last;
        o.left[nb + leaf] = -1;
        o.right[nb + leaf] = -1;
        o.data[nb + leaf] = dat;
        o.bmin[nb + leaf] = mn;
        o.bmax[nb + leaf] = mx;
        const float my_area = box_area(mn, mx);
        o.area[nb + leaf] = my_area;
        // Prepass for the first ATRBVH iteration: this subtree's nodesSah under
        // the default constants, (ci*A + left) + right bottom-up from ct*A at leaves.
        my_ns = __fmul_rn(kPrepassCt, my_area);
        if (o.pp.rec) o.pp.rec[nb + leaf] = make_int4(1, __float_as_int(my_ns), __float_as_int(my_ns), 0);
        s_lmn[tid] = mn;
        s_lmx[tid] = mx;
        s_lns[tid] = my_ns;
        // Deltas within the mesh only: the climb never reads one across meshes.
        if (i > 0) s_delta[tid] = delta_adj(keys, (int)i - 1);
        if (tid == kBuildBlock - 1 && (int)i < last) s_delta[kBuildBlock] = delta_adj(keys, (int)i);
    }
    __syncthreads();
    if (live) {
        const int off = (int)s0 - (int)B0;  // block position of mesh-local sorted index 0
        auto sd = [&](int x) { return s_delta[off + x + 1]; };
        int l = (int)i, r = (int)i, node = (int)i + last;
        int my_lv = 0;
        int dl = l > 0 ? sd(l - 1) : -1;
        int dr = r < last ? sd(r) : -1;
        while (true) {
            const bool is_left = dr > dl;
            const int split = is_left ? r : l - 1;
            const int bs = off + split;  // block position of the split
            if (bs < 0 || bs >= kBuildBlock - 1) {
                edges[2 * blockIdx.x + (bs < 0 ? 0 : 1)] = BuildEdge{(int32_t)m, node, l, r};
                break;
            }
            __threadfence_block();
            const int other = atomicExch(&s_slot[bs], is_left ? l : r);
            if (other < 0) break;  // first of the two children
            __threadfence_block();
            const int pl = is_left ? l : other;
            const int pr = is_left ? other : r;
            const int lc = split == pl ? split + last : split;
            const int rc = split + 1 == pr ? split + 1 + last : split + 1;
            const bool sib_leaf = is_left ? split + 1 == pr : split == pl;
            const int sib = is_left ? rc : lc;
            const int sp = off + (sib_leaf ? sib - last : sib);
            const float4 smn = sib_leaf ? s_lmn[sp] : s_imn[sp];
            const float4 smx = sib_leaf ? s_lmx[sp] : s_imx[sp];
            mn = make_float4(fminf(mn.x, smn.x), fminf(mn.y, smn.y), fminf(mn.z, smn.z), 0.0f);
            mx = make_float4(fmaxf(mx.x, smx.x), fmaxf(mx.y, smx.y), fmaxf(mx.z, smx.z), 0.0f);
            const bool root = pl == 0 && pr == last;
            int p = 0;
            if (!root) {
                dl = pl > 0 ? sd(pl - 1) : -1;
                dr = pr < last ? sd(pr) : -1;
                p = dr > dl ? pr : pl;
            }
            const float pa = box_area(mn, mx);
            if (o.pp.rec) {
                const float sns = sib_leaf ? s_lns[sp] : s_ins[sp];
                my_ns = __fadd_rn(__fadd_rn(__fmul_rn(kPrepassCi, pa), is_left ? my_ns : sns), is_left ? sns : my_ns);
                const int gam = o.pp.seg_gamma ? (int)o.pp.seg_gamma[m] : o.pp.gamma;
                my_lv = pr - pl + 1 >= gam ? 1 + max(my_lv, sib_leaf ? 0 : s_ilv[sp]) : 0;
            }
            s_left[off + p] = lc;
            s_right[off + p] = rc;
            s_rng[off + p] = make_int2(pl, pr);
            // The left child sits at position split, the right at split + 1.
            (split == pl ? s_lpar : s_ipar)[off + split] = p;
            (split + 1 == pr ? s_lpar : s_ipar)[off + split + 1] = p;
            s_imn[off + p] = mn;
            s_imx[off + p] = mx;
            s_ins[off + p] = my_ns;
            s_ilv[off + p] = my_lv;
            if (root) {
                s_ipar[off] = -1;
                break;
            }
            node = p;
            l = pl;
            r = pr;
        }
    }
    __syncthreads();
    if (live) {
        if (s_left[tid] != kUnset) {  // internal node i, finished by this block
            const int2 rg = s_rng[tid];
            write_inner(o, segs, m, nb, (int)i, rg.x, rg.y, s_left[tid], s_right[tid], s_imn[tid], s_imx[tid],
                        box_area(s_imn[tid], s_imx[tid]), s_ins[tid], s_ilv[tid]);
        }
        if (s_ipar[tid] != kUnset) o.parent[nb + (int)i] = s_ipar[tid];
        if (s_lpar[tid] != kUnset) o.parent[nb + (int)i + last] = s_lpar[tid];
        if ((int)i < last) o.slot[segs.inner_base(m) + i] = s_slot[tid];
    }
}

template <typename K>
__global__ void __launch_bounds__(256) k_build_top(Segs segs, const K* __restrict__ keys_all, BuildOut<K> o,
                                                   const BuildEdge* __restrict__ edges, uint32_t count) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const BuildEdge e = edges[t];
    if (e.mesh < 0) return;
    const uint32_t m = (uint32_t)e.mesh;
    const uint32_t s0 = segs.tri_begin(m);
    const int last = (int)(segs.tri_end(m) - s0) - 1;
    const int nb = segs.node_base(m);
    const K* keys = keys_all + s0;
    int32_t* slot = o.slot + segs.inner_base(m);
    float4 mn = ld_cg(o.bmin + nb + e.node), mx = ld_cg(o.bmax + nb + e.node);
    float my_ns = 0.0f;
    int my_lv = 0;
    if (o.pp.rec) {
        const int4 r0 = __ldcg(o.pp.rec + nb + e.node);
        my_ns = __int_as_float(r0.y);
        my_lv = r0.w;  // 0 at a leaf
    }
    int l = e.l, r = e.r;
    int dl = l > 0 ? delta_adj(keys, l - 1) : -1;
    int dr = r < last ? delta_adj(keys, r) : -1;
    while (true) {
        const bool is_left = dr > dl;
        const int split = is_left ? r : l - 1;
        const int other = atomic_exch_acq_rel_gpu(&slot[split], is_left ? l : r);
        if (other < 0) return;  // first of the two children: the sibling finishes the parent
        const int pl = is_left ? l : other;
        const int pr = is_left ? other : r;
        const int lc = split == pl ? split + last : split;
        const int rc = split + 1 == pr ? split + 1 + last : split + 1;
        const int sib = is_left ? rc : lc;
        const float4 smn = ld_cg(o.bmin + nb + sib), smx = ld_cg(o.bmax + nb + sib);
        mn = make_float4(fminf(mn.x, smn.x), fminf(mn.y, smn.y), fminf(mn.z, smn.z), 0.0f);
        mx = make_float4(fmaxf(mx.x, smx.x), fmaxf(mx.y, smx.y), fmaxf(mx.z, smx.z), 0.0f);
        const bool root = pl == 0 && pr == last;
        int p = 0;
        if (!root) {
            dl = pl > 0 ? delta_adj(keys, pl - 1) : -1;
            dr = pr < last ? delta_adj(keys, pr) : -1;
            p = dr > dl ? pr : pl;
        }
        const float pa = box_area(mn, mx);
        if (o.pp.rec) {
            const int4 sr = __ldcg(o.pp.rec + nb + sib);
            const float sns = __int_as_float(sr.y);
            my_ns = __fadd_rn(__fadd_rn(__fmul_rn(kPrepassCi, pa), is_left ? my_ns : sns), is_left ? sns : my_ns);
            my_lv = pr - pl + 1 >= (o.pp.seg_gamma ? (int)o.pp.seg_gamma[m] : o.pp.gamma) ? 1 + max(my_lv, sr.w)
                                                                                          : 0;
        }
        write_inner(o, segs, m, nb, p, pl, pr, lc, rc, mn, mx, pa, my_ns, my_lv);
        o.parent[nb + lc] = p;
        o.parent[nb + rc] = p;
        if (root) {
            o.parent[nb] = -1;
            return;
        }
        l = pl;
        r = pr;
    }
}

// ---- refit of an existing topology ---------------------------------------------
__global__ void __launch_bounds__(256) k_refit(const float4* __restrict__ verts, uint32_t n,
                                                const int32_t* __restrict__ parent,
                                                const int32_t* __restrict__ left,
                                                const int32_t* __restrict__ right,
                                                const int32_t* __restrict__ data,
                                                float4* __restrict__ bmin, float4* __restrict__ bmax,
                                                float* __restrict__ area, uint32_t* __restrict__ counters) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int leaf = (int)i + (int)n - 1;
    const uint32_t tri = (uint32_t)data[leaf];
    const float4 a = __ldg(verts + 3 * (size_t)tri), b = __ldg(verts + 3 * (size_t)tri + 1),
                 c = __ldg(verts + 3 * (size_t)tri + 2);
    float4 mn = make_float4(fminf(fminf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y), fminf(fminf(a.z, b.z), c.z), 0.0f);
    float4 mx = make_float4(fmaxf(fmaxf(a.x, b.x), c.x), fmaxf(fmaxf(a.y, b.y), c.y), fmaxf(fmaxf(a.z, b.z), c.z), 0.0f);
    bmin[leaf] = mn;
    bmax[leaf] = mx;
    area[leaf] = box_area(mn, mx);
    int cur = parent[leaf];
    while (cur >= 0) {
        fence_acq_rel_gpu();
        if (atomicAdd(&counters[cur], 1u) == 0u) return;
        fence_acq_rel_gpu();
        const int l = left[cur], r = right[cur];
        const float4 lm = ld_cg(bmin + l), lx = ld_cg(bmax + l), rm = ld_cg(bmin + r), rx = ld_cg(bmax + r);
        mn = make_float4(fminf(lm.x, rm.x), fminf(lm.y, rm.y), fminf(lm.z, rm.z), 0.0f);
        mx = make_float4(fmaxf(lx.x, rx.x), fmaxf(lx.y, rx.y), fmaxf(lx.z, rx.z), 0.0f);
        bmin[cur] = mn;
        bmax[cur] = mx;
        area[cur] = box_area(mn, mx);
        cur = parent[cur];
    }
}

int grid_for(atr_ctx* ctx, uint64_t work, int per_sm_blocks, int threads) {
    const uint64_t need = (work + threads - 1) / threads;
    const uint64_t cap = (uint64_t)ctx->num_sms * per_sm_blocks;
    return (int)(need < cap ? (need ? need : 1) : cap);
}

// Sort (key, value) pairs of every mesh of `segs` (each mesh on its own) with
// BITS-bit digits.  *keys / *vals hold the input; with an odd number of
// passes the output lands in a second pair of buffers, which then replaces
// them (*keys and *vals are then separate ctx->alloc allocations that are
// released: owned = true); with an even number it lands back in place
// (required when !owned).  hist holds P x D digit counts per mesh when
// hist_ready; otherwise (single mesh, 8-bit digits only) it is computed here.
// tile_counts0, when given, holds the first pass's tile counts (from
// k_morton; tiles x D) and is consumed.  With iota the first pass generates
// the values (global element indices).
template <typename K, int BITS>
int sort_pairs(atr_ctx* ctx, const Segs& segs, uint32_t tiles, K** keys, uint32_t** vals, uint32_t* hist,
               bool hist_ready, bool iota, bool owned, uint32_t* tile_counts0 = nullptr) {
    using Plan = SortPlan<K, BITS>;
    constexpr int P = Plan::kPasses, D = Plan::kDigits;
    static_assert(BITS == 8 || P % 2 == 1, "10-bit plans have an odd pass count");
    ATR_REQUIRE(owned || P % 2 == 0, ATR_ERR_INVALID_ARG, "sort: odd pass count needs owned buffers");
    ATR_REQUIRE(hist_ready || BITS == 8, ATR_ERR_INVALID_ARG, "sort: 10-bit digits need Morton histograms");
    const uint32_t n = segs.n;
    const size_t cbytes = align256((size_t)tiles * D * 4);
    const uint32_t chunks = (tiles + kPrefixChunk - 1) / kPrefixChunk;
    const size_t tbytes = align256((size_t)chunks * D * 4);
    void* tmp = nullptr;
    void* k2v = nullptr;
    void* v2v = nullptr;
    const size_t hb = hist ? 0 : align256(P * D * 4);
    ATR_TRY(ctx->alloc(&k2v, (size_t)n * sizeof(K)));
    int st = ctx->alloc(&v2v, (size_t)n * 4);
    if (st == ATR_OK) st = ctx->alloc(&tmp, (tile_counts0 ? 0 : cbytes) + tbytes + hb);
    if (st != ATR_OK) { ctx->release(k2v); ctx->release(v2v); return st; }
    K* k2 = static_cast<K*>(k2v);
    uint32_t* v2 = static_cast<uint32_t*>(v2v);
    char* p = static_cast<char*>(tmp);
    uint32_t* counts = tile_counts0;
    if (!counts) { counts = reinterpret_cast<uint32_t*>(p); p += cbytes; }
    uint32_t* chunk_tot = reinterpret_cast<uint32_t*>(p);
    p += tbytes;
    if (!hist) hist = reinterpret_cast<uint32_t*>(p);
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaSuccess;
    if (!hist_ready) {
        e = cudaMemsetAsync(hist, 0, P * D * 4, s);
        if (e == cudaSuccess) k_histogram<K><<<grid_for(ctx, n, 4, 256), 256, 0, s>>>(*keys, n, hist);
        ctx->launches += 1;
    }
    K* ka = *keys; K* kb2 = k2;
    uint32_t* va = *vals; uint32_t* vb2 = v2;
    const dim3 prefix_grid((unsigned)(D / 32), chunks);
    for (int pass = 0; pass < P && e == cudaSuccess; ++pass) {
        if (pass > 0 || !tile_counts0) {
            k_tile_counts<K, BITS><<<tiles, kSortThreads, 0, s>>>(segs, ka, pass, counts);
            ctx->launches += 1;
        }
        k_tile_prefix<D><<<prefix_grid, 32 * kPrefixRuns, 0, s>>>(segs, tiles, counts, chunk_tot);
        if (chunks > 1) {
            k_chunk_carry<D><<<(D + 255) / 256, 256, 0, s>>>(chunks, chunk_tot);
            ctx->launches += 1;
        }
        if (pass == 0 && iota)
            k_scatter<K, true, BITS><<<tiles, kSortThreads, Plan::kSmem, s>>>(segs, ka, va, kb2, vb2, pass, hist,
                                                                              counts, chunk_tot);
        else
            k_scatter<K, false, BITS><<<tiles, kSortThreads, Plan::kSmem, s>>>(segs, ka, va, kb2, vb2, pass, hist,
                                                                               counts, chunk_tot);
        ctx->launches += 2;
        std::swap(ka, kb2);
        std::swap(va, vb2);
        e = cudaGetLastError();
    }
    ctx->release(tmp);
    if (P % 2 == 1) {
        // Output in the second pair: hand it to the caller, release the first.
        ctx->release(*keys);
        ctx->release(*vals);
        *keys = k2;
        *vals = v2;
    } else {
        ctx->release(k2v);
        ctx->release(v2v);
    }
    if (e != cudaSuccess) return cuda_fail(e, "sort launch", __FILE__, __LINE__);
    return ATR_OK;
}

template <typename K, int BITS>
int build_typed(atr_ctx* ctx, const Segs& segs, uint32_t tiles, const float4* verts, const float* d_bounds,
                const TreeOut& t, void** keep_keys, uint32_t** keep_idx, const BuildPrepass* prepass,
                const PrimBoxes& pr) {
    constexpr int P = SortPlan<K, BITS>::kPasses, D = SortPlan<K, BITS>::kDigits;
    const uint32_t n = segs.n;
    cudaStream_t s = ctx->stream;
    void* kv = nullptr;
    void* iv = nullptr;
    void* aux = nullptr;
    const size_t hbytes = (size_t)segs.count * P * D * 4;
    const size_t cbytes = (size_t)tiles * D * 4;
    const size_t inner = n - segs.count;
    ATR_TRY(ctx->alloc(&kv, (size_t)n * sizeof(K)));
    int st = ctx->alloc(&iv, (size_t)n * 4);
    const uint32_t bblocks = (n + kBuildBlock - 1) / kBuildBlock;
    const size_t ebytes = (size_t)bblocks * 2 * sizeof(BuildEdge);
    if (st == ATR_OK)
        st = ctx->alloc(&aux, align256(hbytes) + align256(cbytes) + align256(inner * 4) + align256(ebytes));
    if (st != ATR_OK) { ctx->release(kv); ctx->release(iv); return st; }
    K* keys = static_cast<K*>(kv);
    uint32_t* idx = static_cast<uint32_t*>(iv);
    char* ap = static_cast<char*>(aux);
    uint32_t* hist = reinterpret_cast<uint32_t*>(ap); ap += align256(hbytes);
    uint32_t* tile_counts = reinterpret_cast<uint32_t*>(ap); ap += align256(cbytes);
    int32_t* slot = reinterpret_cast<int32_t*>(ap); ap += align256(inner * 4);
    BuildEdge* edges = reinterpret_cast<BuildEdge*>(ap);
    const int zs = zero_words_async(ctx, hist, hbytes / 4);
    if (zs != ATR_OK) {
        ctx->release(aux); ctx->release(kv); ctx->release(iv);
        return zs;
    }

    ctx->phase_begin("morton");
    k_morton<K, BITS><<<tiles, 256, 0, s>>>(segs, verts, d_bounds, keys, hist, tile_counts, pr);
    ctx->phase_end();
    ctx->launches += 1;
    ctx->phase_begin("sort");
    st = sort_pairs<K, BITS>(ctx, segs, tiles, &keys, &idx, hist, true, true, true, tile_counts);
    ctx->phase_end();
    if (st == ATR_OK) {
        ctx->phase_begin("build");
        const BuildOut<K> o{t.parent, t.left,  t.right, t.data,
                            t.bmin,   t.bmax,  t.area,  slot,
                            t.range,  prepass ? *prepass : BuildPrepass{}};
        k_build_block<K><<<bblocks, kBuildBlock, 0, s>>>(segs, keys, idx, verts, o, edges, pr);
        k_build_top<K><<<(2 * bblocks + 255) / 256, 256, 0, s>>>(segs, keys, o, edges, 2 * bblocks);
        ctx->phase_end();
        ctx->launches += 2;
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = cuda_fail(e, "k_build launch", __FILE__, __LINE__);
    }
    ctx->release(aux);
    if (st != ATR_OK || !keep_keys) { ctx->release(keys); ctx->release(idx); return st; }
    *keep_keys = keys;
    *keep_idx = idx;
    return ATR_OK;
}

}  // namespace

static_assert(kSortTile == (int)kSortTileSize, "sort tile size");

template <typename K, int BITS>
cudaError_t scatter_attrs() {
    const int smem = (int)SortPlan<K, BITS>::kSmem;
    cudaError_t e = cudaFuncSetAttribute(k_scatter<K, true, BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_scatter<K, false, BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    return e;
}

// Kernel attributes, set once per context before any capture.
int lbvh_prepare() {
    ATR_CUDA((scatter_attrs<uint32_t, 8>()));
    ATR_CUDA((scatter_attrs<uint32_t, 10>()));
    ATR_CUDA((scatter_attrs<uint64_t, 8>()));
    ATR_CUDA((scatter_attrs<uint64_t, 10>()));
    return ATR_OK;
}

int lbvh_build_segs(atr_ctx* ctx, const Segs& segs, uint32_t tiles, const float4* verts, const float* d_bounds,
                    int morton_bits, const TreeOut& out, void** keep_keys, uint32_t** keep_idx,
                    const BuildPrepass* pp, const PrimBoxes* prims) {
    const bool ten = ctx->sort_bits == 10;
    const PrimBoxes pr = prims ? *prims : PrimBoxes{};
    if (morton_bits == 30)
        return ten ? build_typed<uint32_t, 10>(ctx, segs, tiles, verts, d_bounds, out, keep_keys, keep_idx, pp, pr)
                   : build_typed<uint32_t, 8>(ctx, segs, tiles, verts, d_bounds, out, keep_keys, keep_idx, pp, pr);
    return ten ? build_typed<uint64_t, 10>(ctx, segs, tiles, verts, d_bounds, out, keep_keys, keep_idx, pp, pr)
               : build_typed<uint64_t, 8>(ctx, segs, tiles, verts, d_bounds, out, keep_keys, keep_idx, pp, pr);
}

int prepass_alloc(atr_ctx* ctx, size_t total_nodes, void** block, BuildPrepass* pp) {
    ATR_TRY(ctx->alloc(block, total_nodes * 16));
    pp->rec = static_cast<int4*>(*block);
    pp->gamma = kPrepassGamma;
    return ATR_OK;
}

int lbvh_build_into(atr_ctx* ctx, const float4* verts, uint32_t n, const float* d_bounds, int morton_bits,
                    atr_tree* t, const PrimBoxes* prims) {
    t->morton_bits = morton_bits;
    t->split = prims != nullptr;
    tree_topology_changed(t);
    Segs segs{nullptr, nullptr, 1u, n};
    const uint32_t tiles = (n + kSortTile - 1) / kSortTile;
    TreeOut out{t->parent, t->left, t->right, t->data, t->bmin, t->bmax, t->area, t->range};
    void* keys = nullptr;
    uint32_t* idx = nullptr;
    // The prepass is kept with the tree for a following ATRBVH (level passes on).
    ctx->release(t->prepass_block);
    t->prepass_block = nullptr;
    t->prepass = BuildPrepass{};
    if (ctx->atr_levels > 0)
        ATR_TRY(prepass_alloc(ctx, 2 * (size_t)n - 1, &t->prepass_block, &t->prepass));
    ATR_TRY(lbvh_build_segs(ctx, segs, tiles, verts, d_bounds, morton_bits, out, &keys, &idx,
                            t->prepass_block ? &t->prepass : nullptr, prims));
    ctx->release(t->sorted_keys);
    ctx->release(t->sorted_idx);
    t->sorted_keys = keys;
    t->sorted_idx = idx;
    t->karras = true;
    return ATR_OK;
}

int refit_arrays(atr_ctx* ctx, uint32_t n, const TreeOut& t, const float4* verts) {
    void* ctr = nullptr;
    ATR_TRY(ctx->alloc(&ctr, (size_t)(n - 1) * 4));
    cudaMemsetAsync(ctr, 0, (size_t)(n - 1) * 4, ctx->stream);
    k_refit<<<(n + 255) / 256, 256, 0, ctx->stream>>>(verts, n, t.parent, t.left, t.right, t.data, t.bmin, t.bmax,
                                                      t.area, static_cast<uint32_t*>(ctr));
    ctx->launches += 1;
    cudaError_t e = cudaGetLastError();
    ctx->release(ctr);
    if (e != cudaSuccess) return cuda_fail(e, "k_refit launch", __FILE__, __LINE__);
    return ATR_OK;
}

// Caller-given scene bounds written by the device from kernel arguments, so
// that creating a scene from host bounds enqueues without waiting for the
// vertex upload (no host buffer has to outlive the call).
__global__ void k_set_bounds(float* __restrict__ out, float x0, float y0, float z0, float x1, float y1, float z1) {
    out[0] = x0;
    out[1] = y0;
    out[2] = z0;
    out[3] = x1;
    out[4] = y1;
    out[5] = z1;
}

int scene_bounds_device(atr_ctx* ctx, const float4* verts, uint32_t n, float* d_out) {
    const uint64_t nv = 3ull * n;
    const int blocks = grid_for(ctx, nv, 2, 256);
    void* part = nullptr;
    ATR_TRY(ctx->alloc(&part, (size_t)blocks * 6 * 4));
    k_bounds_partial<<<blocks, 256, 0, ctx->stream>>>(verts, nv, static_cast<float*>(part));
    k_bounds_final<<<1, 32, 0, ctx->stream>>>(static_cast<float*>(part), blocks, d_out);
    ctx->launches += 2;
    cudaError_t e = cudaGetLastError();
    ctx->release(part);
    if (e != cudaSuccess) return cuda_fail(e, "k_bounds launch", __FILE__, __LINE__);
    return ATR_OK;
}

}  // namespace atr

using namespace atr;

extern "C" {

int atr_scene_create(atr_ctx* ctx, const float* vertices, uint32_t n, const float* bbmin, const float* bbmax,
                     int on_device, atr_scene** out) {
    ATR_REQUIRE(ctx && vertices && out, ATR_ERR_INVALID_ARG, "atr_scene_create: NULL argument");
    ATR_REQUIRE(n >= 2 && n < (1u << 30), ATR_ERR_INVALID_ARG,
                "atr_scene_create: triangle count %u outside [2, 2^30)", n);
    ATR_REQUIRE((bbmin == nullptr) == (bbmax == nullptr), ATR_ERR_INVALID_ARG,
                "atr_scene_create: give both bounds or neither");
    *out = nullptr;
    atr_scene* s = new atr_scene();
    s->ctx = ctx;
    s->n = n;
    int st = ctx->alloc(reinterpret_cast<void**>(&s->verts), (size_t)n * 48);
    if (st == ATR_OK) st = ctx->alloc(reinterpret_cast<void**>(&s->d_bounds), 256);
    if (st != ATR_OK) { atr_scene_destroy(s); return st; }
    cudaError_t e = cudaMemcpyAsync(s->verts, vertices, (size_t)n * 48,
                                    on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) { atr_scene_destroy(s); return cuda_fail(e, "cudaMemcpyAsync(vertices)", __FILE__, __LINE__); }
    if (bbmin) {
        k_set_bounds<<<1, 1, 0, ctx->stream>>>(s->d_bounds, bbmin[0], bbmin[1], bbmin[2], bbmax[0], bbmax[1],
                                               bbmax[2]);
        ctx->launches += 1;
        e = cudaGetLastError();
        if (e != cudaSuccess) { atr_scene_destroy(s); return cuda_fail(e, "k_set_bounds", __FILE__, __LINE__); }
    } else {
        st = scene_bounds_device(ctx, s->verts, n, s->d_bounds);
        if (st != ATR_OK) { atr_scene_destroy(s); return st; }
    }
    *out = s;
    return ATR_OK;
}

int atr_scene_set_vertices(atr_ctx* ctx, atr_scene* s, const float* vertices, int on_device) {
    ATR_REQUIRE(ctx && s && vertices, ATR_ERR_INVALID_ARG, "atr_scene_set_vertices: NULL argument");
    ATR_CUDA(cudaMemcpyAsync(s->verts, vertices, (size_t)s->n * 48,
                             on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
    return ATR_OK;
}

int atr_build_lbvh(atr_ctx* ctx, const atr_scene* scene, int morton_bits, atr_tree** out) {
    ATR_REQUIRE(ctx && scene && out, ATR_ERR_INVALID_ARG, "atr_build_lbvh: NULL argument");
    ATR_REQUIRE(morton_bits == 30 || morton_bits == 63, ATR_ERR_UNSUPPORTED,
                "atr_build_lbvh: morton_bits must be 30 or 63 (got %d)", morton_bits);
    *out = nullptr;
    atr_tree* t = nullptr;
    ATR_TRY(tree_alloc(ctx, scene->n, &t));
    int st = lbvh_build_into(ctx, scene->verts, scene->n, scene->d_bounds, morton_bits, t);
    if (st != ATR_OK) { atr_tree_destroy(t); return st; }
    *out = t;
    return ATR_OK;
}

int atr_build_lbvh_split(atr_ctx* ctx, uint32_t num_primitives, const float* prim_bmin, const float* prim_bmax,
                         const uint32_t* data_indices, const float* scene_bmin, const float* scene_bmax,
                         int morton_bits, atr_tree** out) {
    ATR_REQUIRE(ctx && prim_bmin && prim_bmax && data_indices && scene_bmin && scene_bmax && out,
                ATR_ERR_INVALID_ARG, "atr_build_lbvh_split: NULL argument");
    ATR_REQUIRE(num_primitives >= 2 && num_primitives < (1u << 30), ATR_ERR_INVALID_ARG,
                "atr_build_lbvh_split: primitive count %u outside [2, 2^30)", num_primitives);
    ATR_REQUIRE(morton_bits == 30 || morton_bits == 63, ATR_ERR_UNSUPPORTED,
                "atr_build_lbvh_split: morton_bits must be 30 or 63 (got %d)", morton_bits);
    *out = nullptr;
    atr_tree* t = nullptr;
    ATR_TRY(tree_alloc(ctx, num_primitives, &t));
    float* d_bounds = nullptr;
    int st = ctx->alloc(reinterpret_cast<void**>(&d_bounds), 256);
    if (st != ATR_OK) { atr_tree_destroy(t); return st; }
    k_set_bounds<<<1, 1, 0, ctx->stream>>>(d_bounds, scene_bmin[0], scene_bmin[1], scene_bmin[2], scene_bmax[0],
                                           scene_bmax[1], scene_bmax[2]);
    ctx->launches += 1;
    const PrimBoxes pr{reinterpret_cast<const float4*>(prim_bmin), reinterpret_cast<const float4*>(prim_bmax),
                       data_indices};
    st = lbvh_build_into(ctx, nullptr, num_primitives, d_bounds, morton_bits, t, &pr);
    ctx->release(d_bounds);
    if (st != ATR_OK) { atr_tree_destroy(t); return st; }
    *out = t;
    return ATR_OK;
}

int atr_refit(atr_ctx* ctx, atr_tree* tree, const atr_scene* scene) {
    ATR_REQUIRE(ctx && tree && scene, ATR_ERR_INVALID_ARG, "atr_refit: NULL argument");
    ATR_REQUIRE(!tree->split, ATR_ERR_UNSUPPORTED,
                "atr_refit: the tree's leaves are primitive boxes of a triangle-splitting build (rebuild it)");
    ATR_REQUIRE(tree->n == scene->n, ATR_ERR_INVALID_ARG, "atr_refit: tree has %u triangles, scene %u",
                tree->n, scene->n);
    // New boxes make the build's prepass (areas, costs) stale.
    ctx->release(tree->prepass_block);
    tree->prepass_block = nullptr;
    tree->prepass = BuildPrepass{};
    const TreeOut t{tree->parent, tree->left, tree->right, tree->data, tree->bmin, tree->bmax, tree->area};
    if (!tree->refit_plan && !tree->no_refit_plan && ++tree->refits >= 2) {
        const int st = refit_plan_build(ctx, tree->n, t, &tree->refit_plan);
        if (st == ATR_ERR_UNSUPPORTED) tree->no_refit_plan = true;
        else if (st != ATR_OK) return st;
    }
    if (tree->refit_plan) return refit_plan_run(ctx, *tree->refit_plan, t, scene->verts);
    return refit_arrays(ctx, tree->n, t, scene->verts);
}

int atr_device_morton(atr_ctx* ctx, const float* vertices, uint32_t n, const float* bbmin, const float* bbmax,
                      int morton_bits, void* keys) {
    ATR_REQUIRE(ctx && vertices && bbmin && bbmax && keys, ATR_ERR_INVALID_ARG, "atr_device_morton: NULL argument");
    ATR_REQUIRE(morton_bits == 30 || morton_bits == 63, ATR_ERR_UNSUPPORTED, "atr_device_morton: bits %d", morton_bits);
    ATR_REQUIRE(n > 0, ATR_ERR_INVALID_ARG, "atr_device_morton: no triangles");
    void* b = nullptr;
    ATR_TRY(ctx->alloc(&b, 32));
    float h[6] = {bbmin[0], bbmin[1], bbmin[2], bbmax[0], bbmax[1], bbmax[2]};
    cudaMemcpyAsync(b, h, sizeof(h), cudaMemcpyHostToDevice, ctx->stream);
    const float4* v = reinterpret_cast<const float4*>(vertices);
    Segs segs{nullptr, nullptr, 1u, n};
    const uint32_t tiles = (n + kSortTile - 1) / kSortTile;
    if (morton_bits == 30)
        k_morton<uint32_t, 8><<<tiles, 256, 0, ctx->stream>>>(segs, v, static_cast<float*>(b),
                                                              static_cast<uint32_t*>(keys), nullptr, nullptr,
                                                              PrimBoxes{});
    else
        k_morton<uint64_t, 8><<<tiles, 256, 0, ctx->stream>>>(segs, v, static_cast<float*>(b),
                                                              static_cast<uint64_t*>(keys), nullptr, nullptr,
                                                              PrimBoxes{});
    ctx->launches += 1;
    cudaError_t e = cudaStreamSynchronize(ctx->stream);  // h is a stack array
    ctx->release(b);
    if (e != cudaSuccess) return cuda_fail(e, "k_morton", __FILE__, __LINE__);
    return ATR_OK;
}

int atr_device_sort_pairs(atr_ctx* ctx, void* keys, uint32_t* values, uint32_t count, int key_bits) {
    ATR_REQUIRE(ctx && keys && values, ATR_ERR_INVALID_ARG, "atr_device_sort_pairs: NULL argument");
    ATR_REQUIRE(count < (1u << 30), ATR_ERR_INVALID_ARG, "atr_device_sort_pairs: count %u >= 2^30", count);
    if (count == 0) return ATR_OK;
    Segs segs{nullptr, nullptr, 1u, count};
    const uint32_t tiles = (count + kSortTile - 1) / kSortTile;
    if (key_bits <= 32) {
        uint32_t* k = static_cast<uint32_t*>(keys);
        return sort_pairs<uint32_t, 8>(ctx, segs, tiles, &k, &values, nullptr, false, false, false);
    }
    uint64_t* k = static_cast<uint64_t*>(keys);
    return sort_pairs<uint64_t, 8>(ctx, segs, tiles, &k, &values, nullptr, false, false, false);
}

}  // extern "C"
