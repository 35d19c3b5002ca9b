// ORACLE -- test infrastructure only.
//
// Host restatement of the secondary-ray workloads, the checker for
// atrbvh_b200/csrc/raygen.cu:
//   * ambient-occlusion rays: gpu-ray-traversal/src/rt/ray/RayGenKernels.cu:114-223
//     (rayGenAOKernel), with the triangle normal of gpu-ray-traversal/src/rt/Scene.cpp:74
//     and Bob Jenkins' 96-bit mix (RayGenKernels.cu:34-45);
//   * the Morton ray sort: gpu-ray-traversal/src/rt/ray/RayBuffer.cpp:103-160 and
//     RayBufferKernels.cu (box of origins and end points, 192-bit key with
//     bit i of coordinate k at position 6i + k, ascending key order).
// Float arithmetic follows the reference's operation order with no
// contraction (build with -ffp-contract=off); sines and cosines are taken in
// double precision and rounded to float, as the device code does; float to
// uint32 conversions truncate and saturate (NaN to 0) as the device's do.
// Equal ray keys keep their slot order.

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

namespace {

struct V3 {
    float x, y, z;
};
V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 add(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 scale(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
V3 cross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
V3 normalized(V3 a) {
    const float len = std::sqrt(dot(a, a));
    const float r = len != 0.0f ? 1.0f / len : 0.0f;
    return scale(a, r);
}

void mix96(uint32_t& a, uint32_t& b, uint32_t& c) {
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

uint32_t to_u32(float v) {
    if (!(v > 0.0f)) return 0u;
    if (v >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)v;
}

const float kPi = 3.14159265358979323846f;

}  // namespace

extern "C" {

// rays: 8 floats per ray (origin, tmin, direction, tmax); results: 4 int32
// per ray (triangle id or -1, bits of t, ...); out: count * samples rays.
void orc_gen_ao_rays(const float* verts, const float* rays, const int32_t* results, int64_t first, int64_t count,
                     int samples, float max_dist, uint32_t seed, float* out) {
    for (int64_t task = 0; task < count; ++task) {
        const int64_t slot = first + task;
        const float* r = rays + 8 * slot;
        const V3 o{r[0], r[1], r[2]}, d{r[4], r[5], r[6]};
        float t;
        std::memcpy(&t, results + 4 * slot + 1, 4);
        const float s = std::fmax(t - 1.0e-4f, 0.0f);
        const V3 origin = add(o, scale(d, s));
        const int tri = results[4 * slot];
        V3 n{1.0f, 0.0f, 0.0f};
        if (tri != -1) {
            const float* a = verts + 12 * (size_t)tri;
            const V3 va{a[0], a[1], a[2]}, vb{a[4], a[5], a[6]}, vc{a[8], a[9], a[10]};
            n = normalized(cross(sub(vb, va), sub(vc, va)));
        }
        if (dot(n, d) > 0.0f) n = V3{-n.x, -n.y, -n.z};
        const float ax = std::fabs(n.x), ay = std::fabs(n.y), az = std::fabs(n.z);
        const float nm = std::fmax(std::fmax(ax, ay), az);
        V3 perp{n.y, -n.x, 0.0f};
        if (nm == az) perp = V3{0.0f, n.z, -n.y};
        else if (nm == ax) perp = V3{-n.z, 0.0f, n.x};
        perp = normalized(perp);
        const V3 biperp = cross(n, perp);
        uint32_t ha = seed + (uint32_t)task, hb = 0x9e3779b9u, hc = 0x9e3779b9u;
        mix96(ha, hb, hc);
        mix96(ha, hb, hc);
        const float angle = ((2.0f * kPi) * (float)hc) * 2.3283064365386963e-10f;
        const float ca = (float)std::cos((double)angle), sa = (float)std::sin((double)angle);
        const V3 t0 = add(scale(perp, ca), scale(biperp, sa));
        const V3 t1 = add(scale(perp, -sa), scale(biperp, ca));
        float* dst = out + 8 * task * samples;
        for (int i = 0; i < samples; ++i) {
            float x = 0.0f, xadd = 1.0f;
            for (uint32_t h = (uint32_t)i + 1; h != 0; h >>= 1) {
                xadd = xadd * 0.5f;
                if (h & 1) x = x + xadd;
            }
            float y = 0.0f, yadd = 1.0f;
            for (int h = i + 1; h != 0; h /= 3) {
                yadd = yadd * (1.0f / 3.0f);
                y = y + (float)(h % 3) * yadd;
            }
            const float phi = (2.0f * kPi) * y;
            const float rr = std::sqrt(x);
            const float px = rr * (float)std::cos((double)phi), py = rr * (float)std::sin((double)phi);
            const float pz = std::sqrt((1.0f - px * px) - py * py);
            const V3 w = normalized(add(add(scale(t0, px), scale(t1, py)), scale(n, pz)));
            float* q = dst + 8 * i;
            q[0] = origin.x; q[1] = origin.y; q[2] = origin.z; q[3] = 0.0f;
            q[4] = w.x; q[5] = w.y; q[6] = w.z; q[7] = tri == -1 ? -1.0f : max_dist;
        }
    }
}

// Sorted order of rays (perm[j] = old slot of the ray at new position j) and
// the box used (6 floats).
void orc_sort_rays(const float* rays, int64_t n, uint32_t* perm, float* box_out) {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int64_t i = 0; i < n; ++i) {
        const float* r = rays + 8 * i;
        for (int k = 0; k < 3; ++k) {
            const float e = r[k] + r[4 + k] * r[7];
            lo[k] = std::fmin(std::fmin(lo[k], r[k]), e);
            hi[k] = std::fmax(std::fmax(hi[k], r[k]), e);
        }
    }
    std::vector<uint32_t> key((size_t)n * 6);  // six 32-bit words, least significant first
    for (int64_t i = 0; i < n; ++i) {
        const float* r = rays + 8 * i;
        const V3 nd = normalized(V3{r[4], r[5], r[6]});
        const float q[3] = {nd.x, nd.y, nd.z};
        uint32_t c[6];
        for (int k = 0; k < 3; ++k) {
            const float a = (r[k] - lo[k]) / (hi[k] - lo[k]);
            const float b = (q[k] + 1.0f) * 0.5f;
            c[k] = to_u32((a * 256.0f) * 65536.0f);
            c[3 + k] = to_u32((b * 32.0f) * 65536.0f);
        }
        uint32_t* w = key.data() + 6 * i;
        std::memset(w, 0, 24);
        for (int k = 0; k < 6; ++k)
            for (int b = 0; b < 32; ++b) {
                const int p = k + 6 * b;
                w[p >> 5] |= ((c[k] >> b) & 1u) << (p & 31);
            }
    }
    std::vector<uint32_t> order((size_t)n);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        const uint32_t* ka = key.data() + 6 * (size_t)a;
        const uint32_t* kb = key.data() + 6 * (size_t)b;
        for (int w = 5; w >= 0; --w)
            if (ka[w] != kb[w]) return ka[w] < kb[w];
        return false;
    });
    std::copy(order.begin(), order.end(), perm);
    for (int k = 0; k < 3; ++k) {
        box_out[k] = lo[k];
        box_out[3 + k] = hi[k];
    }
}

}  // extern "C"
