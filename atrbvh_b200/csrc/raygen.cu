// Secondary-ray workloads on the device: ambient-occlusion rays from the hits
// of a ray batch, and the Morton sort of a ray batch for coherence.
//
// AO rays restate rayGenAOKernel (gpu-ray-traversal/src/rt/ray/RayGenKernels.cu:114-223):
// for each input ray of [first, first + count), origin = o + d * max(t - 1e-4, 0),
// the hit triangle's geometric normal (normalize(cross(v1 - v0, v2 - v0)),
// gpu-ray-traversal/src/rt/Scene.cpp:74; (1, 0, 0) on a miss) turned against
// the ray, a tangent frame rotated by an angle from two rounds of Bob
// Jenkins' 96-bit mix of (seed + index, golden ratio, golden ratio), and
// samples at the base-2 / base-3 Halton points (i + 1) warped to a
// cosine-weighted hemisphere; tmax = max_dist, or -1 for a miss.  Vector
// arithmetic is done with explicit round-to-nearest operations in the
// reference's order, sines and cosines in double precision rounded to float,
// so the result does not depend on the compiler (the reference compiles this
// kernel with -use_fast_math, whose approximate sine, cosine and reciprocal
// are not restated).
//
// The ray sort restates RayBuffer::mortonSort (gpu-ray-traversal/src/rt/ray/RayBuffer.cpp:103-160,
// RayBufferKernels.cu): the box of the ray origins and end points, a 192-bit
// key interleaving bit i of six 32-bit coordinates -- the origin normalised to
// the box scaled by 2^24, the normalised direction mapped to [0, 1] scaled by
// 2^21 -- at position 6i + axis, rays reordered by ascending key with the
// slot-to-id map carried along.  The reference sorts the keys on the host
// with an unstable sort; here equal keys keep their slot order (three stable
// 64-bit LSD radix sorts), which is a deterministic choice among its orders.

#include "common.cuh"
#include "internal.h"

namespace atr {
namespace {

struct V3 {
    float x, y, z;
};

__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 sub(V3 a, V3 b) { return v3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)); }
__device__ __forceinline__ V3 scale(V3 a, float s) { return v3(__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)); }
__device__ __forceinline__ V3 add(V3 a, V3 b) { return v3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)); }
__device__ __forceinline__ float dot(V3 a, V3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return v3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
              __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
// v * (1 / |v|), and (0, 0, 0) for a zero vector.
__device__ __forceinline__ V3 normalized(V3 a) {
    const float len = __fsqrt_rn(dot(a, a));
    const float r = len != 0.0f ? __fdiv_rn(1.0f, len) : 0.0f;
    return scale(a, r);
}

__device__ __forceinline__ void jenkins_mix(uint32_t& a, uint32_t& b, uint32_t& c) {
    a -= b; a -= c; a ^= (c >> 13);
    b -= c; b -= a; b ^= (a << 8);
    c -= a; c -= b; c ^= (b >> 13);
    a -= b; a -= c; a ^= (c >> 12);
    b -= c; b -= a; b ^= (a << 16);
    c -= a; c -= b; c ^= (b >> 5);
    a -= b; a -= c; a ^= (c >> 3);
    b -= c; b -= a; b ^= (a << 10);
    c -= a; c -= b; c ^= (b >> 15);
}

constexpr float kPi = 3.14159265358979323846f;

__global__ void __launch_bounds__(256) k_ao_rays(const float4* __restrict__ verts, const float4* __restrict__ rays,
                                                 const int4* __restrict__ res, int64_t first, int64_t count,
                                                 int samples, float max_dist, uint32_t seed,
                                                 float4* __restrict__ out) {
    const int64_t task = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (task >= count) return;
    const int64_t slot = first + task;
    const float4 o4 = rays[2 * slot], d4 = rays[2 * slot + 1];
    const int4 r = res[slot];
    const V3 o = v3(o4.x, o4.y, o4.z), d = v3(d4.x, d4.y, d4.z);
    const float s = fmaxf(__fsub_rn(__int_as_float(r.y), 1.0e-4f), 0.0f);
    const V3 origin = add(o, scale(d, s));
    const int tri = r.x;
    V3 n = v3(1.0f, 0.0f, 0.0f);
    if (tri != -1) {
        const float4 a = verts[3 * (size_t)tri], b = verts[3 * (size_t)tri + 1], c = verts[3 * (size_t)tri + 2];
        const V3 va = v3(a.x, a.y, a.z);
        n = normalized(cross(sub(v3(b.x, b.y, b.z), va), sub(v3(c.x, c.y, c.z), va)));
    }
    if (dot(n, d) > 0.0f) n = v3(-n.x, -n.y, -n.z);
    const float ax = fabsf(n.x), ay = fabsf(n.y), az = fabsf(n.z);
    const float nm = fmaxf(fmaxf(ax, ay), az);
    V3 perp = v3(n.y, -n.x, 0.0f);
    if (nm == az) perp = v3(0.0f, n.z, -n.y);
    else if (nm == ax) perp = v3(-n.z, 0.0f, n.x);
    perp = normalized(perp);
    const V3 biperp = cross(n, perp);
    uint32_t ha = seed + (uint32_t)task, hb = 0x9e3779b9u, hc = 0x9e3779b9u;
    jenkins_mix(ha, hb, hc);
    jenkins_mix(ha, hb, hc);
    const float angle = __fmul_rn(__fmul_rn(__fmul_rn(2.0f, kPi), (float)hc), 2.3283064365386963e-10f);
    const float ca = (float)cos((double)angle), sa = (float)sin((double)angle);
    const V3 t0 = add(scale(perp, ca), scale(biperp, sa));
    const V3 t1 = add(scale(perp, -sa), scale(biperp, ca));
    float4* dst = out + 2 * task * samples;
    for (int i = 0; i < samples; ++i) {
        float x = 0.0f, xadd = 1.0f;
        for (uint32_t h = (uint32_t)i + 1; h != 0; h >>= 1) {
            xadd = __fmul_rn(xadd, 0.5f);
            if (h & 1) x = __fadd_rn(x, xadd);
        }
        float y = 0.0f, yadd = 1.0f;
        for (int h = i + 1; h != 0; h /= 3) {
            yadd = __fmul_rn(yadd, 1.0f / 3.0f);
            y = __fadd_rn(y, __fmul_rn((float)(h % 3), yadd));
        }
        const float phi = __fmul_rn(__fmul_rn(2.0f, kPi), y);
        const float rr = __fsqrt_rn(x);
        const float px = __fmul_rn(rr, (float)cos((double)phi)), py = __fmul_rn(rr, (float)sin((double)phi));
        const float pz = __fsqrt_rn(__fsub_rn(__fsub_rn(1.0f, __fmul_rn(px, px)), __fmul_rn(py, py)));
        const V3 w = normalized(add(add(scale(t0, px), scale(t1, py)), scale(n, pz)));
        dst[2 * i] = make_float4(origin.x, origin.y, origin.z, 0.0f);
        dst[2 * i + 1] = make_float4(w.x, w.y, w.z, tri == -1 ? -1.0f : max_dist);
    }
}

// Box of the ray origins and end points (origin + direction * tmax): one
// partial box per block, then one block folds them (min/max are exact, so the
// result does not depend on the order).
__global__ void __launch_bounds__(256) k_ray_box_partial(const float4* __restrict__ rays, int64_t n,
                                                         float* __restrict__ partial) {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float4 o = rays[2 * i], d = rays[2 * i + 1];
        const float e[3] = {__fadd_rn(o.x, __fmul_rn(d.x, d.w)), __fadd_rn(o.y, __fmul_rn(d.y, d.w)),
                            __fadd_rn(o.z, __fmul_rn(d.z, d.w))};
        const float p[3] = {o.x, o.y, o.z};
        for (int k = 0; k < 3; ++k) {
            lo[k] = fminf(fminf(lo[k], p[k]), e[k]);
            hi[k] = fmaxf(fmaxf(hi[k], p[k]), e[k]);
        }
    }
    __shared__ float s[6][256];
    for (int k = 0; k < 3; ++k) {
        s[k][threadIdx.x] = lo[k];
        s[3 + k][threadIdx.x] = hi[k];
    }
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int k = 0; k < 3; ++k) {
                s[k][threadIdx.x] = fminf(s[k][threadIdx.x], s[k][threadIdx.x + w]);
                s[3 + k][threadIdx.x] = fmaxf(s[3 + k][threadIdx.x], s[3 + k][threadIdx.x + w]);
            }
        __syncthreads();
    }
    if (threadIdx.x < 6) partial[6 * blockIdx.x + threadIdx.x] = s[threadIdx.x][0];
}

__global__ void __launch_bounds__(256) k_ray_box_final(const float* __restrict__ partial, int np,
                                                       float* __restrict__ box) {
    if (threadIdx.x >= 6) return;
    const int k = threadIdx.x;
    float v = partial[k];
    for (int b = 1; b < np; ++b) v = k < 3 ? fminf(v, partial[6 * b + k]) : fmaxf(v, partial[6 * b + k]);
    box[k] = v;
}

// Float to uint32 as the device converts (truncation, saturating, NaN to 0).
__device__ __forceinline__ uint32_t to_u32(float v) { return __float2uint_rz(v); }

// Word w (0 = least significant) of the 192-bit key of coordinates c[6]:
// bit b of word w is bit (32w + b) / 6 of coordinate (32w + b) % 6.
__device__ __forceinline__ uint64_t key_half(const uint32_t c[6], int half) {
    uint64_t k = 0;
    for (int b = 0; b < 64; ++b) {
        const int p = 64 * half + b;
        k |= (uint64_t)((c[p % 6] >> (p / 6)) & 1u) << b;
    }
    return k;
}

__global__ void __launch_bounds__(256) k_ray_coords(const float4* __restrict__ rays, int64_t n,
                                                    const float* __restrict__ box, uint32_t* __restrict__ coords) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 o = rays[2 * i], d = rays[2 * i + 1];
    const float p[3] = {o.x, o.y, o.z};
    const V3 nd = normalized(v3(d.x, d.y, d.z));
    const float q[3] = {nd.x, nd.y, nd.z};
    for (int k = 0; k < 3; ++k) {
        const float a = __fdiv_rn(__fsub_rn(p[k], box[k]), __fsub_rn(box[3 + k], box[k]));
        const float b = __fmul_rn(__fadd_rn(q[k], 1.0f), 0.5f);
        coords[6 * i + k] = to_u32(__fmul_rn(__fmul_rn(a, 256.0f), 65536.0f));
        coords[6 * i + 3 + k] = to_u32(__fmul_rn(__fmul_rn(b, 32.0f), 65536.0f));
    }
}

// Key half `half` of the ray now at position j of the permutation.
__global__ void __launch_bounds__(256) k_ray_key_gather(const uint32_t* __restrict__ coords,
                                                        const uint32_t* __restrict__ perm, int64_t n, int half,
                                                        unsigned long long* __restrict__ keys) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t* c = coords + 6 * (size_t)perm[j];
    const uint32_t cc[6] = {c[0], c[1], c[2], c[3], c[4], c[5]};
    keys[j] = key_half(cc, half);
}

__global__ void __launch_bounds__(256) k_ray_reorder(const float4* __restrict__ in, const int32_t* __restrict__ in_s2i,
                                                     const uint32_t* __restrict__ perm, int64_t n,
                                                     float4* __restrict__ out, int32_t* __restrict__ out_s2i,
                                                     int32_t* __restrict__ out_i2s) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t old = perm[j];
    out[2 * j] = in[2 * (size_t)old];
    out[2 * j + 1] = in[2 * (size_t)old + 1];
    const int32_t id = in_s2i ? in_s2i[old] : (int32_t)old;
    if (out_s2i) out_s2i[j] = id;
    if (out_i2s) out_i2s[id] = (int32_t)j;
}

__global__ void __launch_bounds__(256) k_iota(uint32_t* __restrict__ v, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) v[i] = (uint32_t)i;
}

}  // namespace
}  // namespace atr

using namespace atr;

extern "C" {

int atr_gen_ao_rays(atr_ctx* ctx, const atr_scene* scene, const float* rays, const int32_t* results,
                    int64_t first, int64_t count, int num_samples, float max_dist, uint32_t seed, float* out) {
    ATR_REQUIRE(ctx && scene && rays && results && out, ATR_ERR_INVALID_ARG, "atr_gen_ao_rays: NULL argument");
    ATR_REQUIRE(first >= 0 && count >= 0, ATR_ERR_INVALID_ARG, "atr_gen_ao_rays: negative range");
    ATR_REQUIRE(num_samples >= 1 && num_samples <= 4096, ATR_ERR_INVALID_ARG, "atr_gen_ao_rays: %d samples",
                num_samples);
    if (count == 0) return ATR_OK;
    k_ao_rays<<<(unsigned)((count + 255) / 256), 256, 0, ctx->stream>>>(
        scene->verts, reinterpret_cast<const float4*>(rays), reinterpret_cast<const int4*>(results), first, count,
        num_samples, max_dist, seed, reinterpret_cast<float4*>(out));
    ctx->launches += 1;
    ATR_CUDA(cudaGetLastError());
    return ATR_OK;
}

int atr_sort_rays(atr_ctx* ctx, const float* rays, const int32_t* slot_to_id, int64_t n, float* out_rays,
                  int32_t* out_slot_to_id, int32_t* out_id_to_slot) {
    ATR_REQUIRE(ctx && rays && out_rays, ATR_ERR_INVALID_ARG, "atr_sort_rays: NULL argument");
    ATR_REQUIRE(out_rays != rays, ATR_ERR_INVALID_ARG, "atr_sort_rays: out_rays must not alias rays");
    ATR_REQUIRE(n >= 0 && n < (1ll << 30), ATR_ERR_INVALID_ARG, "atr_sort_rays: %lld rays", (long long)n);
    if (n == 0) return ATR_OK;
    cudaStream_t s = ctx->stream;
    const unsigned blocks = (unsigned)((n + 255) / 256);
    const int np = (int)std::min<int64_t>((n + 255) / 256, 1024);
    void* scratch = nullptr;
    const size_t bp = align256((size_t)np * 24 + 24), bc = align256((size_t)n * 24), bk = align256((size_t)n * 8),
                 bperm = align256((size_t)n * 4);
    ATR_TRY(ctx->alloc(&scratch, bp + bc + bk + bperm));
    char* p = static_cast<char*>(scratch);
    float* partial = reinterpret_cast<float*>(p);
    float* box = partial + 6 * np;
    p += bp;
    uint32_t* coords = reinterpret_cast<uint32_t*>(p); p += bc;
    unsigned long long* keys = reinterpret_cast<unsigned long long*>(p); p += bk;
    uint32_t* perm = reinterpret_cast<uint32_t*>(p);
    const float4* r4 = reinterpret_cast<const float4*>(rays);
    ctx->phase_begin("ray_sort");
    k_ray_box_partial<<<np, 256, 0, s>>>(r4, n, partial);
    k_ray_box_final<<<1, 32, 0, s>>>(partial, np, box);
    k_ray_coords<<<blocks, 256, 0, s>>>(r4, n, box, coords);
    k_iota<<<blocks, 256, 0, s>>>(perm, n);
    ctx->launches += 4;
    int st = ATR_OK;
    for (int half = 0; half < 3 && st == ATR_OK; ++half) {
        k_ray_key_gather<<<blocks, 256, 0, s>>>(coords, perm, n, half, keys);
        ctx->launches += 1;
        st = atr_device_sort_pairs(ctx, keys, perm, (uint32_t)n, 64);
    }
    if (st == ATR_OK) {
        k_ray_reorder<<<blocks, 256, 0, s>>>(r4, slot_to_id, perm, n, reinterpret_cast<float4*>(out_rays),
                                             out_slot_to_id, out_id_to_slot);
        ctx->launches += 1;
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = cuda_fail(e, "atr_sort_rays kernels", __FILE__, __LINE__);
    }
    ctx->phase_end();
    ctx->release(scratch);
    return st;
}

}  // extern "C"
