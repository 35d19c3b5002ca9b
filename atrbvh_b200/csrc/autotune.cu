// Autotuner: per size class (floor(log2(triangles))), the ATRBVH treelet size
// and iteration count, the ATRBVH block size and the sort digit width that
// build a class sample fastest at equal SAH.
//
// The reference has no tuner: its parameters are fixed per run
// (gpu-ray-traversal/src/rt/BVHRTSettings.cpp:7-84, treeletSize/iterations) and
// its launch shapes are constants (AgglomerativeTreelet.cu:556-595).  Here,
// for each class a sample batch of meshes of the config-0 distribution with
// sizes in [2^c, 2^(c+1)) is built first with ATRBVH(9,2), the reference
// quality point; every (treelet 5..9, iterations 1..3) pair is then built and
// timed, and the fastest pair whose summed per-mesh SAH is at most (1 + tol)
// times that of ATRBVH(9,2) is kept (ATRBVH(9,2) itself always qualifies).
// Block size (2, 4, 8 warps) and digit width (8, 10 bits) change only the
// speed, so they are tuned afterwards on the kept pair, checking that the SAH
// does not move.  Times are CUDA-event medians of `reps` builds after one
// warm-up build.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace atr {
namespace {

// Per-mesh SAH parts in double: sum of internal areas, sum of leaf areas,
// root area (thread i owns leaf i and internal node i of its mesh).
__global__ void __launch_bounds__(256) k_seg_sah_parts(Segs segs, const float* __restrict__ area,
                                                        double* __restrict__ parts) {
    const uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= segs.n) return;
    const uint32_t m = segs.seg_of_tri(gi);
    const uint32_t s0 = segs.tri_begin(m);
    const uint32_t n = segs.tri_end(m) - s0;
    const uint32_t li = gi - s0;
    const int nb = segs.node_base(m);
    atomicAdd(&parts[3 * m + 1], (double)area[nb + (int)(li + n - 1)]);
    if (li < n - 1) atomicAdd(&parts[3 * m], (double)area[nb + (int)li]);
    if (li == 0) parts[3 * m + 2] = (double)area[nb];
}

struct Sample {
    atr_batch* b = nullptr;
    std::vector<uint32_t> off;
    uint32_t n = 0;
};

// Sum over the sample's meshes of (1.2 * internal + 1.0 * leaf) / root area.
int sample_sah(atr_ctx* ctx, const Sample& s, double* out) {
    atr_tree_view v0;
    ATR_TRY(atr_batch_mesh_view(s.b, 0, &v0));
    const uint32_t count = (uint32_t)s.off.size() - 1;
    uint32_t* d_off = nullptr;
    double* parts = nullptr;
    ATR_TRY(ctx->alloc(reinterpret_cast<void**>(&d_off), (count + 1) * 4ull));
    int st = ctx->alloc(reinterpret_cast<void**>(&parts), count * 24ull);
    if (st != ATR_OK) { ctx->release(d_off); return st; }
    // Tile offsets are not used by this kernel: pass the triangle offsets twice.
    cudaMemcpyAsync(d_off, s.off.data(), (count + 1) * 4ull, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemsetAsync(parts, 0, count * 24ull, ctx->stream);
    const Segs segs{d_off, d_off, count, s.n};
    k_seg_sah_parts<<<(s.n + 255) / 256, 256, 0, ctx->stream>>>(segs, v0.area, parts);
    ctx->launches += 1;
    std::vector<double> h(3ull * count);
    cudaMemcpyAsync(h.data(), parts, count * 24ull, cudaMemcpyDeviceToHost, ctx->stream);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    ctx->release(d_off);
    ctx->release(parts);
    if (e != cudaSuccess) return cuda_fail(e, "autotune SAH", __FILE__, __LINE__);
    double sum = 0.0;
    for (uint32_t m = 0; m < count; ++m) sum += (1.2 * h[3 * m] + 1.0 * h[3 * m + 1]) / h[3 * m + 2];
    *out = sum;
    return ATR_OK;
}

// Median device time of `reps` builds after one warm-up build.
int time_builds(atr_ctx* ctx, atr_batch* b, int treelet, int iters, uint32_t reps, float* ms) {
    ATR_TRY(atr_batch_build(ctx, b, 1, treelet, iters, 1.2f, 1.0f, 0));
    cudaEvent_t e0, e1;
    ATR_CUDA(cudaEventCreate(&e0));
    ATR_CUDA(cudaEventCreate(&e1));
    std::vector<float> t;
    int st = ATR_OK;
    for (uint32_t r = 0; r < reps && st == ATR_OK; ++r) {
        cudaEventRecord(e0, ctx->stream);
        st = atr_batch_build(ctx, b, 1, treelet, iters, 1.2f, 1.0f, 0);
        cudaEventRecord(e1, ctx->stream);
        if (st != ATR_OK) break;
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) { st = cuda_fail(e, "autotune timing", __FILE__, __LINE__); break; }
        float x = 0.0f;
        cudaEventElapsedTime(&x, e0, e1);
        t.push_back(x);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ATR_TRY(st);
    std::sort(t.begin(), t.end());
    *ms = t[t.size() / 2];
    return atr_ctx_synchronize(ctx);
}

}  // namespace
}  // namespace atr

using namespace atr;

extern "C" {

int atr_autotune(atr_ctx* ctx, const atr_autotune_config* cfg, atr_tune_table* out) {
    ATR_REQUIRE(ctx && cfg && out, ATR_ERR_INVALID_ARG, "atr_autotune: NULL argument");
    ATR_REQUIRE(cfg->min_class >= 1 && cfg->min_class <= cfg->max_class && cfg->max_class <= 29,
                ATR_ERR_INVALID_ARG, "atr_autotune: class range [%u, %u] outside [1, 29]", cfg->min_class,
                cfg->max_class);
    ATR_REQUIRE(cfg->reps >= 1 && cfg->reps <= 64, ATR_ERR_INVALID_ARG, "atr_autotune: reps %u", cfg->reps);
    ATR_REQUIRE(cfg->sah_tolerance >= 0.0f && cfg->sah_tolerance < 1.0f, ATR_ERR_INVALID_ARG,
                "atr_autotune: tolerance %g outside [0, 1)", (double)cfg->sah_tolerance);
    std::memset(out, 0, sizeof(*out));
    const int warps0 = ctx->atr_warps, bits0 = ctx->sort_bits;
    int st = ATR_OK;
    for (uint32_t c = cfg->min_class; c <= cfg->max_class && st == ATR_OK; ++c) {
        // Sample: meshes of sizes uniform in [2^c, 2^(c+1)), about
        // sample_triangles in all (at least two meshes, at most 4096).
        const uint64_t lo = 1ull << c, hi = 2ull << c;
        uint64_t want = std::max<uint64_t>(cfg->sample_triangles, 2 * lo);
        uint32_t count = (uint32_t)std::min<uint64_t>(4096, std::max<uint64_t>(2, want / (lo + lo / 2)));
        while ((uint64_t)count * hi >= (1ull << 30)) --count;
        Sample s;
        s.off.assign(count + 1, 0);
        std::vector<uint32_t> sizes(count);
        uint64_t x = cfg->seed * 0x9E3779B97F4A7C15ull + c;
        for (uint32_t m = 0; m < count; ++m) {
            x = x * 6364136223846793005ull + 1442695040888963407ull;
            sizes[m] = (uint32_t)(lo + ((x >> 33) % (hi - lo)));
            s.off[m + 1] = s.off[m] + sizes[m];
        }
        s.n = s.off[count];
        std::vector<float> verts((size_t)s.n * 12);
        st = atr_gen_batch_scene(count, sizes.data(), cfg->seed + c, verts.data());
        if (st == ATR_OK) st = atr_batch_create(ctx, verts.data(), s.off.data(), count, nullptr, 0, &s.b);
        if (st != ATR_OK) break;
        // The reference point: ATRBVH(9,2) at the context's own launch shape.
        ctx->atr_warps = warps0;
        ctx->sort_bits = bits0;
        double sah_ref = 0.0, sah = 0.0;
        float ms_ref = 0.0f;
        st = time_builds(ctx, s.b, 9, 2, cfg->reps, &ms_ref);
        if (st == ATR_OK) st = sample_sah(ctx, s, &sah_ref);
        int best_t = 9, best_i = 2;
        float best_ms = ms_ref;
        double best_sah = sah_ref;
        for (int t = 5; t <= 9 && st == ATR_OK; ++t)
            for (int it = 1; it <= 3 && st == ATR_OK; ++it) {
                if (t == 9 && it == 2) continue;
                float ms = 0.0f;
                st = time_builds(ctx, s.b, t, it, cfg->reps, &ms);
                if (st == ATR_OK) st = sample_sah(ctx, s, &sah);
                if (st == ATR_OK && sah <= sah_ref * (1.0 + cfg->sah_tolerance) && ms < best_ms) {
                    best_t = t;
                    best_i = it;
                    best_ms = ms;
                    best_sah = sah;
                }
            }
        int best_w = warps0, best_b = bits0;
        for (int w : {2, 4, 8})
            for (int bits : {8, 10}) {
                if (st != ATR_OK || (w == warps0 && bits == bits0)) continue;
                ctx->atr_warps = w;
                ctx->sort_bits = bits;
                float ms = 0.0f;
                st = time_builds(ctx, s.b, best_t, best_i, cfg->reps, &ms);
                if (st == ATR_OK) st = sample_sah(ctx, s, &sah);
                if (st == ATR_OK && sah != best_sah) {
                    set_error("atr_autotune: SAH changed with launch tuning (class %u)", c);
                    st = ATR_ERR_CUDA;
                }
                if (st == ATR_OK && ms < best_ms) {
                    best_w = w;
                    best_b = bits;
                    best_ms = ms;
                }
            }
        atr_batch_destroy(s.b);
        if (st != ATR_OK) break;
        atr_tune_entry& e = out->cls[c];
        e.treelet = (uint8_t)best_t;
        e.iterations = (uint8_t)best_i;
        e.atr_warps = (uint8_t)best_w;
        e.sort_bits = (uint8_t)best_b;
        e.build_ms = best_ms;
        e.reference_ms = ms_ref;
        e.sah_ratio = (float)(best_sah / sah_ref);
        e.sample_triangles = s.n;
        e.sample_meshes = count;
        out->tuned_mask |= 1u << c;
    }
    ctx->atr_warps = warps0;
    ctx->sort_bits = bits0;
    return st;
}

// Median device time of `reps` builds of a whole batch (graph replays) after
// one warm-up, and its summed per-mesh SAH.
int time_batch(atr_ctx* ctx, atr_batch* b, uint32_t reps, float* ms, double* sah) {
    ATR_TRY(atr_batch_build(ctx, b, 1, 9, 2, 1.2f, 1.0f, 1));
    cudaEvent_t e0, e1;
    ATR_CUDA(cudaEventCreate(&e0));
    ATR_CUDA(cudaEventCreate(&e1));
    std::vector<float> t;
    int st = ATR_OK;
    for (uint32_t r = 0; r < reps && st == ATR_OK; ++r) {
        cudaEventRecord(e0, ctx->stream);
        st = atr_batch_build(ctx, b, 1, 9, 2, 1.2f, 1.0f, 1);
        cudaEventRecord(e1, ctx->stream);
        if (st != ATR_OK) break;
        const cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) { st = cuda_fail(e, "batch autotune timing", __FILE__, __LINE__); break; }
        float x = 0.0f;
        cudaEventElapsedTime(&x, e0, e1);
        t.push_back(x);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ATR_TRY(st);
    std::sort(t.begin(), t.end());
    *ms = t[t.size() / 2];
    uint32_t count = 0, n = 0;
    uint64_t nodes = 0;
    ATR_TRY(atr_batch_info(b, &count, &n, &nodes));
    std::vector<float> per(count);
    ATR_TRY(atr_batch_sah(ctx, b, 1.2f, 1.0f, per.data()));
    double sum = 0.0;
    for (float x : per) sum += x;
    *sah = sum;
    return ATR_OK;
}

// Class entry used for a mesh of n triangles: its own class when tuned, else
// the nearest tuned class.
static const atr_tune_entry* entry_for(const atr_tune_table* t, uint32_t n) {
    int c = 31 - __builtin_clz(n);
    for (int d = 0; d < 32; ++d) {
        if (c - d >= 0 && (t->tuned_mask >> (c - d) & 1u)) return &t->cls[c - d];
        if (c + d < 32 && (t->tuned_mask >> (c + d) & 1u)) return &t->cls[c + d];
    }
    return nullptr;
}

int atr_tune_lookup(const atr_tune_table* t, uint32_t num_triangles, atr_tune_entry* entry) {
    ATR_REQUIRE(t && entry, ATR_ERR_INVALID_ARG, "atr_tune_lookup: NULL argument");
    ATR_REQUIRE(t->tuned_mask != 0, ATR_ERR_INVALID_ARG, "atr_tune_lookup: empty table");
    ATR_REQUIRE(num_triangles >= 2, ATR_ERR_INVALID_ARG, "atr_tune_lookup: %u triangles", num_triangles);
    *entry = *entry_for(t, num_triangles);
    return ATR_OK;
}

int atr_batch_apply_tuning(atr_ctx* ctx, atr_batch* b, const atr_tune_table* t) {
    ATR_REQUIRE(ctx && b && t, ATR_ERR_INVALID_ARG, "atr_batch_apply_tuning: NULL argument");
    ATR_REQUIRE(t->tuned_mask != 0, ATR_ERR_INVALID_ARG, "atr_batch_apply_tuning: empty table");
    uint32_t count = 0, n = 0;
    uint64_t nodes = 0;
    ATR_TRY(atr_batch_info(b, &count, &n, &nodes));
    std::vector<uint8_t> ts(count), it(count);
    uint64_t tris_in[32] = {};
    for (uint32_t m = 0; m < count; ++m) {
        atr_tree_view v;
        ATR_TRY(atr_batch_mesh_view(b, m, &v));
        const atr_tune_entry* e = entry_for(t, v.num_triangles);
        ts[m] = e->treelet;
        it[m] = e->iterations;
        tris_in[e - t->cls] += v.num_triangles;
    }
    // Launch shape of the class that holds the most triangles.
    int dom = 0;
    for (int c = 1; c < 32; ++c)
        if (tris_in[c] > tris_in[dom]) dom = c;
    ctx->atr_warps = t->cls[dom].atr_warps;
    ctx->sort_bits = t->cls[dom].sort_bits;
    return atr_batch_set_params(ctx, b, ts.data(), it.data());
}

// Tunes the size classes present in a batch on class samples, then builds the
// batch itself with ATRBVH(9,2) at the context's launch shape and with the
// tuned table, and keeps the table only when the batch builds faster with it
// at a summed SAH within the tolerance; otherwise every entry is reset to
// the reference point, so the table applied to this batch is never slower
// than the defaults.  The batch is left with the kept parameters applied.
int atr_batch_autotune(atr_ctx* ctx, atr_batch* b, const atr_autotune_config* cfg, atr_tune_table* out,
                       atr_tune_outcome* outcome) {
    ATR_REQUIRE(ctx && b && cfg && out && outcome, ATR_ERR_INVALID_ARG, "atr_batch_autotune: NULL argument");
    std::memset(out, 0, sizeof(*out));
    std::memset(outcome, 0, sizeof(*outcome));
    uint32_t count = 0, n = 0;
    uint64_t nodes = 0;
    ATR_TRY(atr_batch_info(b, &count, &n, &nodes));
    uint32_t present = 0;
    for (uint32_t m = 0; m < count; ++m) {
        atr_tree_view v;
        ATR_TRY(atr_batch_mesh_view(b, m, &v));
        present |= 1u << (31 - __builtin_clz(v.num_triangles));
    }
    const int warps0 = ctx->atr_warps, bits0 = ctx->sort_bits;
    // Reference: the batch with ATRBVH(9,2) everywhere at the context's launch shape.
    ATR_TRY(atr_batch_set_params(ctx, b, nullptr, nullptr));
    ATR_TRY(time_batch(ctx, b, cfg->reps, &outcome->default_ms, &outcome->default_sah));
    for (uint32_t c = 1; c < 30; ++c) {
        if (!(present >> c & 1u)) continue;
        atr_autotune_config one = *cfg;
        one.min_class = one.max_class = c;
        atr_tune_table t;
        ATR_TRY(atr_autotune(ctx, &one, &t));
        out->cls[c] = t.cls[c];
        out->tuned_mask |= 1u << c;
    }
    int st = atr_batch_apply_tuning(ctx, b, out);
    if (st == ATR_OK) st = time_batch(ctx, b, cfg->reps, &outcome->tuned_ms, &outcome->tuned_sah);
    if (st != ATR_OK) {
        ctx->atr_warps = warps0;
        ctx->sort_bits = bits0;
        return st;
    }
    outcome->kept = outcome->tuned_ms < outcome->default_ms &&
                    outcome->tuned_sah <= outcome->default_sah * (1.0 + (double)cfg->sah_tolerance);
    if (!outcome->kept) {
        for (uint32_t c = 0; c < 32; ++c) {
            if (!(out->tuned_mask >> c & 1u)) continue;
            atr_tune_entry& e = out->cls[c];
            e.treelet = 9;
            e.iterations = 2;
            e.atr_warps = (uint8_t)warps0;
            e.sort_bits = (uint8_t)bits0;
            e.build_ms = e.reference_ms;
            e.sah_ratio = 1.0f;
        }
        ctx->atr_warps = warps0;
        ctx->sort_bits = bits0;
        ATR_TRY(atr_batch_set_params(ctx, b, nullptr, nullptr));
    }
    return ATR_OK;
}

}  // extern "C"
