// Closest-hit / any-hit traversal of the Compact2 layout on sm_100a.
//
// Per ray this is gpu-ray-traversal/src/rt/kernels/kepler_dynamic_fetch.cu:95-317
// as one lane executes it: slab tests of both children, nearer child first,
// the farther one pushed; a leaf reached during the descent is processed
// before the descent continues (the reference may postpone it while other
// lanes still descend, which only changes the culling bound used for nodes
// whose leaves cannot hold a closer hit); Woop ray/triangle tests with
// t > tmin, t < hitT, u >= 0, v >= 0, u + v <= 1 keep the first hit on ties.
// The span helpers keep the reference's integer min/max on float bits
// (CudaTracerKernels.hpp:182-189).  Arithmetic: slab = fma(bound, 1/d, -o/d),
// Woop dot products as fma chains, IEEE reciprocal; the CPU oracle uses the
// same operations.
//
// Warps are persistent and refill terminated lanes from a global ray counter
// (warp-aggregated atomic), breaking out to refill whenever fewer than 20
// lanes of a warp are still traversing (the reference's dynamic fetch).

#include "common.cuh"
#include "internal.h"

namespace atr {

// Which layout each ray traverses: with groups == 0 every ray uses the arrays
// as given; otherwise rays [ray_off[g], ray_off[g+1]) trace mesh
// group_mesh[g] of a batch whose mesh m starts at node 4 * (tri_off[m] - m)
// (float4 units) and Woop entry 4 * tri_off[m].
struct RayMeshMap {
    const uint32_t* ray_off;
    const uint32_t* group_mesh;
    const uint32_t* tri_off;
    uint32_t groups;
};

namespace {

constexpr int kSentinel = 0x76543210;
constexpr int kDynamicFetch = 20;

__device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }
__device__ __forceinline__ int imax(int a, int b) { return a > b ? a : b; }

__device__ __forceinline__ float span_begin(float a0, float a1, float b0, float b1, float c0, float c1, float d) {
    const int t = imax(imin(__float_as_int(c0), __float_as_int(c1)), __float_as_int(d));
    return __int_as_float(imax(imax(__float_as_int(fminf(a0, a1)), __float_as_int(fminf(b0, b1))), t));
}
__device__ __forceinline__ float span_end(float a0, float a1, float b0, float b1, float c0, float c1, float d) {
    const int t = imin(imax(__float_as_int(c0), __float_as_int(c1)), __float_as_int(d));
    return __int_as_float(imin(imin(__float_as_int(fmaxf(a0, a1)), __float_as_int(fmaxf(b0, b1))), t));
}

template <int kStack>
__global__ void __launch_bounds__(128) k_trace(const float4* __restrict__ nodes_all,
                                               const float4* __restrict__ woop_all,
                                               const int* __restrict__ tri_all, RayMeshMap map,
                                               const float4* __restrict__ rays, int64_t nrays, int any_hit,
                                               int4* __restrict__ results, unsigned long long* __restrict__ counter,
                                               uint32_t* __restrict__ err) {
    int stack[kStack];
    const int lane = threadIdx.x & 31;
    float ox = 0, oy = 0, oz = 0, tmin = 0, dx = 0, dy = 0, dz = 0, hitT = 0;
    float idx = 0, idy = 0, idz = 0, oodx = 0, oody = 0, oodz = 0;
    int nodeAddr = kSentinel, leafAddr = 0, hitIndex = -1, sp = 0;
    long long rayidx = 0;
    bool overflow = false;
    const float4* nodes = nodes_all;
    const float4* woop = woop_all;
    const int* tri_index = tri_all;

    while (true) {
        const bool terminated = nodeAddr == kSentinel;
        const unsigned active = __activemask();
        const unsigned mt = __ballot_sync(active, terminated);
        if (terminated) {
            const int leader = __ffs(mt) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(mt));
            base = __shfl_sync(mt, base, leader);
            rayidx = (long long)base + __popc(mt & lanemask_lt());
            if (rayidx >= nrays) break;
            if (map.groups) {
                uint32_t lo = 0, hi = map.groups;
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if ((long long)__ldg(map.ray_off + mid) <= rayidx) lo = mid; else hi = mid;
                }
                const uint32_t mesh = __ldg(map.group_mesh + lo);
                const uint32_t s0 = __ldg(map.tri_off + mesh);
                nodes = nodes_all + 4 * ((size_t)s0 - mesh);
                woop = woop_all + 4 * (size_t)s0;
                tri_index = tri_all + 4 * (size_t)s0;
            }
            const float4 o = __ldg(rays + 2 * rayidx), d = __ldg(rays + 2 * rayidx + 1);
            ox = o.x; oy = o.y; oz = o.z; tmin = o.w;
            dx = d.x; dy = d.y; dz = d.z; hitT = d.w;
            const float ooeps = 8.271806125530277e-25f;  // 2^-80
            idx = __fdiv_rn(1.0f, fabsf(dx) > ooeps ? dx : copysignf(ooeps, dx));
            idy = __fdiv_rn(1.0f, fabsf(dy) > ooeps ? dy : copysignf(ooeps, dy));
            idz = __fdiv_rn(1.0f, fabsf(dz) > ooeps ? dz : copysignf(ooeps, dz));
            oodx = __fmul_rn(ox, idx);
            oody = __fmul_rn(oy, idy);
            oodz = __fmul_rn(oz, idz);
            stack[0] = kSentinel;
            sp = 0;
            leafAddr = 0;
            nodeAddr = 0;
            hitIndex = -1;
            overflow = false;
        }

        while (nodeAddr != kSentinel) {
            while ((unsigned)nodeAddr < (unsigned)kSentinel) {
                const float4 n0 = __ldg(nodes + nodeAddr), n1 = __ldg(nodes + nodeAddr + 1);
                const float4 nz = __ldg(nodes + nodeAddr + 2), cn = __ldg(nodes + nodeAddr + 3);
                int c0 = __float_as_int(cn.x), c1 = __float_as_int(cn.y);
                const float c0lox = __fmaf_rn(n0.x, idx, -oodx), c0hix = __fmaf_rn(n0.y, idx, -oodx);
                const float c0loy = __fmaf_rn(n0.z, idy, -oody), c0hiy = __fmaf_rn(n0.w, idy, -oody);
                const float c0loz = __fmaf_rn(nz.x, idz, -oodz), c0hiz = __fmaf_rn(nz.y, idz, -oodz);
                const float c1loz = __fmaf_rn(nz.z, idz, -oodz), c1hiz = __fmaf_rn(nz.w, idz, -oodz);
                const float c0min = span_begin(c0lox, c0hix, c0loy, c0hiy, c0loz, c0hiz, tmin);
                const float c0max = span_end(c0lox, c0hix, c0loy, c0hiy, c0loz, c0hiz, hitT);
                const float c1lox = __fmaf_rn(n1.x, idx, -oodx), c1hix = __fmaf_rn(n1.y, idx, -oodx);
                const float c1loy = __fmaf_rn(n1.z, idy, -oody), c1hiy = __fmaf_rn(n1.w, idy, -oody);
                const float c1min = span_begin(c1lox, c1hix, c1loy, c1hiy, c1loz, c1hiz, tmin);
                const float c1max = span_end(c1lox, c1hix, c1loy, c1hiy, c1loz, c1hiz, hitT);
                const bool swp = c1min < c0min;
                const bool t0 = c0max >= c0min, t1 = c1max >= c1min;
                if (!t0 && !t1) {
                    nodeAddr = stack[sp--];
                } else {
                    nodeAddr = t0 ? c0 : c1;
                    if (t0 && t1) {
                        if (swp) { const int tmp = nodeAddr; nodeAddr = c1; c1 = tmp; }
                        if (sp + 1 >= kStack) {  // deeper than the stack: give the ray up
                            overflow = true;
                            nodeAddr = kSentinel;
                            leafAddr = 0;
                            break;
                        }
                        stack[++sp] = c1;
                    }
                }
                if (nodeAddr < 0 && leafAddr >= 0) {
                    leafAddr = nodeAddr;
                    nodeAddr = stack[sp--];
                }
                if (leafAddr < 0) break;
            }
            while (leafAddr < 0) {
                for (int triAddr = ~leafAddr;; triAddr += 3) {
                    const float4 v00 = __ldg(woop + triAddr);
                    if (__float_as_int(v00.x) == (int)0x80000000u) break;
                    const float4 v11 = __ldg(woop + triAddr + 1), v22 = __ldg(woop + triAddr + 2);
                    const float Oz = __fmaf_rn(-oz, v00.z, __fmaf_rn(-oy, v00.y, __fmaf_rn(-ox, v00.x, v00.w)));
                    const float invDz = __fdiv_rn(1.0f, __fmaf_rn(dz, v00.z, __fmaf_rn(dy, v00.y, __fmul_rn(dx, v00.x))));
                    const float t = __fmul_rn(Oz, invDz);
                    if (t > tmin && t < hitT) {
                        const float Ox = __fmaf_rn(oz, v11.z, __fmaf_rn(oy, v11.y, __fmaf_rn(ox, v11.x, v11.w)));
                        const float Dx = __fmaf_rn(dz, v11.z, __fmaf_rn(dy, v11.y, __fmul_rn(dx, v11.x)));
                        const float u = __fmaf_rn(t, Dx, Ox);
                        if (u >= 0.0f) {
                            const float Oy = __fmaf_rn(oz, v22.z, __fmaf_rn(oy, v22.y, __fmaf_rn(ox, v22.x, v22.w)));
                            const float Dy = __fmaf_rn(dz, v22.z, __fmaf_rn(dy, v22.y, __fmul_rn(dx, v22.x)));
                            const float v = __fmaf_rn(t, Dy, Oy);
                            if (v >= 0.0f && __fadd_rn(u, v) <= 1.0f) {
                                hitT = t;
                                hitIndex = triAddr;
                                if (any_hit) { nodeAddr = kSentinel; break; }
                            }
                        }
                    }
                }
                leafAddr = nodeAddr;
                if (nodeAddr < 0) nodeAddr = stack[sp--];
            }
            if (__popc(__activemask()) < kDynamicFetch) break;
        }
        if (nodeAddr == kSentinel) {
            if (overflow) set_error_bits(err, kErrTraceStack);
            const int id = hitIndex == -1 ? -1 : __ldg(tri_index + hitIndex);
            results[rayidx] = make_int4(id, __float_as_int(hitT), 0, 0);
        }
    }
}

template <int kStack>
void launch_trace(atr_ctx* ctx, const int4* nodes, const float4* woop, const int32_t* tri, const RayMeshMap& map,
                  const float4* rays, int64_t n, int any_hit, int4* res, unsigned long long* counter) {
    static int blocks_per_sm = 0;
    if (!blocks_per_sm) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_trace<kStack>, 128, 0);
        if (blocks_per_sm < 1) blocks_per_sm = 1;
    }
    const int64_t need = (n + 127) / 128;
    int64_t grid = (int64_t)ctx->num_sms * blocks_per_sm;
    if (need < grid) grid = need;
    k_trace<kStack><<<(unsigned)grid, 128, 0, ctx->stream>>>(reinterpret_cast<const float4*>(nodes), woop, tri, map,
                                                             rays, n, any_hit, res, counter, ctx->d_error);
    ctx->launches += 1;
}

// Cosine-weighted diffuse bounce per primary hit (the workload of
// gpu-ray-traversal/src/rt/ray/RayGenKernels.cu:114-223 with one sample):
// origin backed off the hit by 1e-4 along the ray, geometric normal facing
// the ray, direction from a counter-based hash of (seed, ray); misses get
// tmax = -1 and never hit.
__global__ void __launch_bounds__(256) k_bounce(const float4* __restrict__ verts, const float4* __restrict__ rays,
                                                const int4* __restrict__ res, int64_t n, uint64_t seed,
                                                float4* __restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 o = rays[2 * i], d = rays[2 * i + 1];
    const int4 r = res[i];
    if (r.x < 0) {
        out[2 * i] = o;
        out[2 * i + 1] = make_float4(d.x, d.y, d.z, -1.0f);
        return;
    }
    const float t = fmaxf(__int_as_float(r.y) - 1e-4f, 0.0f);
    const float4 p = make_float4(o.x + d.x * t, o.y + d.y * t, o.z + d.z * t, 0.0f);
    const float4 a = verts[3 * (size_t)r.x], b = verts[3 * (size_t)r.x + 1], c = verts[3 * (size_t)r.x + 2];
    const float e1x = b.x - a.x, e1y = b.y - a.y, e1z = b.z - a.z;
    const float e2x = c.x - a.x, e2y = c.y - a.y, e2z = c.z - a.z;
    float nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
    float len = sqrtf(nx * nx + ny * ny + nz * nz);
    if (len == 0.0f) { nx = 1.0f; ny = 0.0f; nz = 0.0f; len = 1.0f; }
    nx /= len; ny /= len; nz /= len;
    if (nx * d.x + ny * d.y + nz * d.z > 0.0f) { nx = -nx; ny = -ny; nz = -nz; }
    // Orthonormal basis around n.
    float tx, ty, tz;
    if (fabsf(nx) > fabsf(nz)) { tx = -ny; ty = nx; tz = 0.0f; } else { tx = 0.0f; ty = -nz; tz = ny; }
    const float tl = rsqrtf(tx * tx + ty * ty + tz * tz);
    tx *= tl; ty *= tl; tz *= tl;
    const float bx = ny * tz - nz * ty, by = nz * tx - nx * tz, bz = nx * ty - ny * tx;
    // Two uniforms from a 64-bit mix of (seed, i).
    unsigned long long h = seed ^ (0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1));
    h ^= h >> 30; h *= 0xBF58476D1CE4E5B9ull; h ^= h >> 27; h *= 0x94D049BB133111EBull; h ^= h >> 31;
    const float u1 = (float)(h >> 40) * (1.0f / 16777216.0f);
    const float u2 = (float)((h >> 16) & 0xFFFFFF) * (1.0f / 16777216.0f);
    const float rr = sqrtf(u1), phi = 6.2831853f * u2;
    const float x = rr * cosf(phi), y = rr * sinf(phi), z = sqrtf(fmaxf(0.0f, 1.0f - u1));
    float wx = x * tx + y * bx + z * nx, wy = x * ty + y * by + z * ny, wz = x * tz + y * bz + z * nz;
    const float wl = rsqrtf(wx * wx + wy * wy + wz * wz);
    out[2 * i] = p;
    out[2 * i + 1] = make_float4(wx * wl, wy * wl, wz * wl, 1e30f);
}

}  // namespace

int trace_run(atr_ctx* ctx, const int4* nodes, const float4* woop, const int32_t* tri, const RayMeshMap& map,
              int max_depth, const float4* rays, int64_t n, int any_hit, int4* res) {
    if (n == 0) return ATR_OK;
    unsigned long long* counter = nullptr;
    ATR_TRY(ctx->alloc(reinterpret_cast<void**>(&counter), 8));
    cudaMemsetAsync(counter, 0, 8, ctx->stream);
    int st = ATR_OK;
    ctx->phase_begin("trace");
    if (max_depth + 1 < 64) launch_trace<64>(ctx, nodes, woop, tri, map, rays, n, any_hit, res, counter);
    else if (max_depth + 1 < 256) launch_trace<256>(ctx, nodes, woop, tri, map, rays, n, any_hit, res, counter);
    else st = ATR_ERR_UNSUPPORTED;
    ctx->phase_end();
    ctx->release(counter);
    if (st == ATR_ERR_UNSUPPORTED) {
        set_error("trace: layout depth %d exceeds the traversal stack", max_depth);
        return st;
    }
    ATR_CUDA(cudaGetLastError());
    return ATR_OK;
}

int trace_batch(atr_ctx* ctx, const int4* nodes, const float4* woop, const int32_t* tri, const uint32_t* ray_off,
                const uint32_t* group_mesh, const uint32_t* tri_off, uint32_t groups, int max_depth,
                const float4* rays, int64_t n, int any_hit, int4* res) {
    const RayMeshMap map{ray_off, group_mesh, tri_off, groups};
    return trace_run(ctx, nodes, woop, tri, map, max_depth, rays, n, any_hit, res);
}

}  // namespace atr

using namespace atr;

extern "C" {

int atr_trace(atr_ctx* ctx, const atr_compact* cp, const float* rays, int64_t n, int any_hit, int32_t* results) {
    ATR_REQUIRE(ctx && cp && rays && results, ATR_ERR_INVALID_ARG, "atr_trace: NULL argument");
    ATR_REQUIRE(n >= 0, ATR_ERR_INVALID_ARG, "atr_trace: negative ray count");
    const RayMeshMap map{nullptr, nullptr, nullptr, 0u};
    return trace_run(ctx, cp->nodes, cp->woop, cp->tri_index, map, cp->max_depth, reinterpret_cast<const float4*>(rays),
                     n, any_hit, reinterpret_cast<int4*>(results));
}

int atr_gen_bounce_rays(atr_ctx* ctx, const atr_scene* scene, const float* rays, const int32_t* results, int64_t n,
                        uint64_t seed, float* out) {
    ATR_REQUIRE(ctx && scene && rays && results && out, ATR_ERR_INVALID_ARG, "atr_gen_bounce_rays: NULL argument");
    if (n <= 0) return ATR_OK;
    k_bounce<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(
        scene->verts, reinterpret_cast<const float4*>(rays), reinterpret_cast<const int4*>(results), n, seed,
        reinterpret_cast<float4*>(out));
    ctx->launches += 1;
    ATR_CUDA(cudaGetLastError());
    return ATR_OK;
}

}  // extern "C"
