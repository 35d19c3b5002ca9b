// On-disk cache image of the Compact2 traversal layout.
//
// The image is the reference's CudaBVH stream format
// (gpu-ray-traversal/src/rt/cuda/CudaBVH.cpp:108-123 with the framework's
// Buffer::writeToStream, framework/gpu/Buffer.cpp:331-362): the layout as a
// little-endian S32 (BVHLayout_Compact2 = 5,
// rt/kernels/CudaTracerKernels.hpp:45-55), then m_nodes, m_triWoop and
// m_triIndex, each as a little-endian S64 byte count followed by the bytes.
// A file written here loads in the reference's CudaBVH(InputStream&) and the
// other way round.  Loading validates the sizes and every child reference
// before anything reaches the device, and recomputes the layout's depth
// (which the format does not store) from the child references.
//
// The cache key plays the role of the reference's file name hash
// (gpu-ray-traversal/src/rt/cuda/Renderer.cpp:137-141: scene, platform and
// build-parameter hashes with the layout): a 64-bit hash over the format,
// the vertex bytes and every build parameter that changes the layout.

#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace {

constexpr int32_t kLayoutCompact2 = 5;
constexpr uint64_t kHeaderBytes = 4 + 3 * 8;

void put_u32(unsigned char* p, uint32_t v) {
    for (int i = 0; i < 4; ++i) p[i] = (unsigned char)(v >> (8 * i));
}
void put_u64(unsigned char* p, uint64_t v) {
    for (int i = 0; i < 8; ++i) p[i] = (unsigned char)(v >> (8 * i));
}
uint32_t get_u32(const unsigned char* p) {
    uint32_t v = 0;
    for (int i = 0; i < 4; ++i) v |= (uint32_t)p[i] << (8 * i);
    return v;
}
uint64_t get_u64(const unsigned char* p) {
    uint64_t v = 0;
    for (int i = 0; i < 8; ++i) v |= (uint64_t)p[i] << (8 * i);
    return v;
}

// 64-bit mixing (the finaliser of splitmix64, Steele/Lea/Flood, OOPSLA'14).
inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Order-dependent hash of a byte range: 8-byte words folded into a running
// state, the tail zero-padded, the length mixed in last.
uint64_t hash_bytes(const unsigned char* p, uint64_t n, uint64_t seed) {
    uint64_t h = mix64(seed ^ 0x6A09E667F3BCC909ull);
    uint64_t i = 0;
    for (; i + 8 <= n; i += 8) {
        uint64_t w;
        std::memcpy(&w, p + i, 8);
        h = mix64(h ^ (w + 0x9E3779B97F4A7C15ull)) + (h << 7 | h >> 57);
    }
    if (i < n) {
        uint64_t w = 0;
        std::memcpy(&w, p + i, n - i);
        h = mix64(h ^ (w + 0x9E3779B97F4A7C15ull)) + (h << 7 | h >> 57);
    }
    return mix64(h ^ n);
}

}  // namespace

using namespace atr;

extern "C" {

int atr_compact_serialize(atr_ctx* ctx, const atr_compact* c, void* out, uint64_t capacity, uint64_t* size) {
    ATR_REQUIRE(ctx && c && size, ATR_ERR_INVALID_ARG, "atr_compact_serialize: NULL argument");
    const uint64_t nb = (uint64_t)c->num_nodes * 64, wb = (uint64_t)c->num_woop * 16, tb = (uint64_t)c->num_woop * 4;
    *size = kHeaderBytes + nb + wb + tb;
    if (!out) return ATR_OK;
    ATR_REQUIRE(capacity >= *size, ATR_ERR_INVALID_ARG,
                "atr_compact_serialize: image needs %llu bytes, buffer holds %llu", (unsigned long long)*size,
                (unsigned long long)capacity);
    unsigned char* p = static_cast<unsigned char*>(out);
    put_u32(p, (uint32_t)kLayoutCompact2);
    p += 4;
    put_u64(p, nb);
    ATR_CUDA(cudaMemcpyAsync(p + 8, c->nodes, nb, cudaMemcpyDeviceToHost, ctx->stream));
    p += 8 + nb;
    put_u64(p, wb);
    ATR_CUDA(cudaMemcpyAsync(p + 8, c->woop, wb, cudaMemcpyDeviceToHost, ctx->stream));
    p += 8 + wb;
    put_u64(p, tb);
    ATR_CUDA(cudaMemcpyAsync(p + 8, c->tri_index, tb, cudaMemcpyDeviceToHost, ctx->stream));
    return atr_ctx_synchronize(ctx);
}

int atr_compact_deserialize(atr_ctx* ctx, const void* image, uint64_t size, atr_compact** out) {
    ATR_REQUIRE(ctx && image && out, ATR_ERR_INVALID_ARG, "atr_compact_deserialize: NULL argument");
    *out = nullptr;
    const unsigned char* p = static_cast<const unsigned char*>(image);
    ATR_REQUIRE(size >= kHeaderBytes, ATR_ERR_INVALID_ARG, "atr_compact_deserialize: %llu bytes is too short",
                (unsigned long long)size);
    const int32_t layout = (int32_t)get_u32(p);
    ATR_REQUIRE(layout == kLayoutCompact2, ATR_ERR_UNSUPPORTED,
                "atr_compact_deserialize: layout %d is not BVHLayout_Compact2 (5)", layout);
    uint64_t at = 4;
    uint64_t len[3];
    const unsigned char* data[3];
    for (int k = 0; k < 3; ++k) {
        ATR_REQUIRE(size - at >= 8, ATR_ERR_INVALID_ARG, "atr_compact_deserialize: truncated image");
        len[k] = get_u64(p + at);
        at += 8;
        ATR_REQUIRE(len[k] <= size - at, ATR_ERR_INVALID_ARG, "atr_compact_deserialize: truncated image");
        data[k] = p + at;
        at += len[k];
    }
    ATR_REQUIRE(at == size, ATR_ERR_INVALID_ARG, "atr_compact_deserialize: %llu trailing bytes",
                (unsigned long long)(size - at));
    ATR_REQUIRE(len[0] > 0 && len[0] % 64 == 0 && len[1] % 16 == 0 && len[2] * 4 == len[1],
                ATR_ERR_INVALID_ARG, "atr_compact_deserialize: inconsistent buffer sizes %llu/%llu/%llu",
                (unsigned long long)len[0], (unsigned long long)len[1], (unsigned long long)len[2]);
    const int64_t num_nodes = (int64_t)(len[0] / 64), num_woop = (int64_t)(len[1] / 16);
    ATR_REQUIRE(num_nodes < (1ll << 29) && num_woop < (1ll << 31), ATR_ERR_INVALID_ARG,
                "atr_compact_deserialize: layout too large");
    // Child references: inner children are float4 offsets of later node
    // records (the layout is a preorder), leaves are ~(Woop float4 offset)
    // with a terminated triangle list.  Depth: inner-node levels, root 1.
    std::vector<int32_t> level((size_t)num_nodes, 0);
    level[0] = 1;
    int32_t depth = 1;
    const int32_t* terms = reinterpret_cast<const int32_t*>(data[1]);
    for (int64_t k = 0; k < num_nodes; ++k) {
        int32_t ref[2];
        std::memcpy(ref, data[0] + 64 * k + 48, 8);
        ATR_REQUIRE(level[(size_t)k] > 0, ATR_ERR_INVALID_ARG, "atr_compact_deserialize: node %lld is unreachable",
                    (long long)k);
        for (int s = 0; s < 2; ++s) {
            if (ref[s] >= 0) {
                const int64_t child = ref[s] / 4;
                ATR_REQUIRE(ref[s] % 4 == 0 && child > k && child < num_nodes && level[(size_t)child] == 0,
                            ATR_ERR_INVALID_ARG, "atr_compact_deserialize: bad inner reference %d in node %lld",
                            ref[s], (long long)k);
                level[(size_t)child] = level[(size_t)k] + 1;
                depth = std::max(depth, level[(size_t)child]);
            } else {
                const int64_t w = ~(int64_t)ref[s];
                ATR_REQUIRE(w + 4 <= num_woop, ATR_ERR_INVALID_ARG,
                            "atr_compact_deserialize: bad leaf reference %d in node %lld", ref[s], (long long)k);
                int64_t e = w;
                while (e < num_woop && terms[4 * e] != (int32_t)0x80000000) e += 3;
                ATR_REQUIRE(e < num_woop && e > w, ATR_ERR_INVALID_ARG,
                            "atr_compact_deserialize: unterminated leaf at node %lld", (long long)k);
            }
        }
    }
    atr_compact* c = new atr_compact();
    c->ctx = ctx;
    c->num_nodes = num_nodes;
    c->num_woop = num_woop;
    c->max_depth = depth;
    int st = ctx->alloc(reinterpret_cast<void**>(&c->nodes), len[0]);
    if (st == ATR_OK) st = ctx->alloc(reinterpret_cast<void**>(&c->woop), std::max<uint64_t>(len[1], 16));
    if (st == ATR_OK) st = ctx->alloc(reinterpret_cast<void**>(&c->tri_index), std::max<uint64_t>(len[2], 4));
    cudaError_t e = cudaSuccess;
    if (st == ATR_OK) e = cudaMemcpyAsync(c->nodes, data[0], len[0], cudaMemcpyHostToDevice, ctx->stream);
    if (st == ATR_OK && e == cudaSuccess && len[1])
        e = cudaMemcpyAsync(c->woop, data[1], len[1], cudaMemcpyHostToDevice, ctx->stream);
    if (st == ATR_OK && e == cudaSuccess && len[2])
        e = cudaMemcpyAsync(c->tri_index, data[2], len[2], cudaMemcpyHostToDevice, ctx->stream);
    if (st == ATR_OK && e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);  // the image may be freed next
    if (st == ATR_OK && e != cudaSuccess) st = cuda_fail(e, "atr_compact_deserialize copies", __FILE__, __LINE__);
    if (st != ATR_OK) {
        atr_compact_destroy(c);
        return st;
    }
    *out = c;
    return ATR_OK;
}

int atr_cache_key(const float* vertices, uint32_t num_triangles, const atr_cache_params* params, uint64_t* key) {
    ATR_REQUIRE(vertices && params && key, ATR_ERR_INVALID_ARG, "atr_cache_key: NULL argument");
    const unsigned char* v = reinterpret_cast<const unsigned char*>(vertices);
    const uint64_t bytes = (uint64_t)num_triangles * 48;
    // Chunks hashed in parallel, then folded in order.
    const uint64_t chunk = 1ull << 22;
    const int64_t chunks = (int64_t)((bytes + chunk - 1) / chunk);
    std::vector<uint64_t> part((size_t)std::max<int64_t>(chunks, 1), 0);
#pragma omp parallel for schedule(static) if (chunks > 4)
    for (int64_t k = 0; k < chunks; ++k) {
        const uint64_t b = (uint64_t)k * chunk;
        part[(size_t)k] = hash_bytes(v + b, std::min(chunk, bytes - b), (uint64_t)k);
    }
    uint64_t h = hash_bytes(reinterpret_cast<const unsigned char*>(part.data()), part.size() * 8, bytes);
    const int32_t fields[6] = {kLayoutCompact2, params->morton_bits, params->optimizer, params->treelet_size,
                               params->iterations, params->max_leaf};
    float costs[2] = {params->ci, params->ct};
    h = hash_bytes(reinterpret_cast<const unsigned char*>(fields), sizeof(fields), h);
    h = hash_bytes(reinterpret_cast<const unsigned char*>(costs), sizeof(costs), h);
    *key = h;
    return ATR_OK;
}

}  // extern "C"
