// Seeded synthetic scenes and rays.
//
// Every value is a function of (seed, stream, element index) through a
// counter-based Philox4x32-10 generator (Salmon et al., "Parallel random
// numbers: as easy as 1, 2, 3", SC'11), so scenes are identical however many
// host threads produce them.  Gaussians use Box-Muller in double precision.
//
// Scene layout matches the reference's triangle soup
// (BVHRT-Core/src/Scene.h:12-18): three float4 vertices per triangle, w = 0.

#include <cmath>
#include <cstdint>
#include <cstring>

#include "../../include/atrbvh.h"

namespace {

struct Philox {
    uint32_t v[4];
};

inline Philox philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c0 = n0;
        c1 = (uint32_t)p1;
        c2 = n2;
        c3 = (uint32_t)p0;
    }
    return Philox{{c0, c1, c2, c3}};
}

// Uniform in [0, 1) with 24 random bits (exact in float).
inline float u01f(uint32_t u) { return (float)(u >> 8) * (1.0f / 16777216.0f); }
// Uniform in (0, 1) in double.
inline double u01d(uint32_t u) { return ((double)u + 0.5) * (1.0 / 4294967296.0); }

inline void gauss2(uint32_t a, uint32_t b, double& g0, double& g1) {
    const double r = std::sqrt(-2.0 * std::log(u01d(a)));
    const double th = 6.283185307179586 * u01d(b);
    g0 = r * std::cos(th);
    g1 = r * std::sin(th);
}

// Nine N(0,1) samples for triangle `i` of stream `s`.
inline void nine_gauss(uint32_t i, uint32_t s, uint64_t seed, uint32_t tag, double g[10]) {
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32) ^ 0x41545242u;
    Philox b = philox(i, 1, s, tag, k0, k1);
    Philox c = philox(i, 2, s, tag, k0, k1);
    Philox d = philox(i, 3, s, tag, k0, k1);
    gauss2(b.v[0], b.v[1], g[0], g[1]);
    gauss2(b.v[2], b.v[3], g[2], g[3]);
    gauss2(c.v[0], c.v[1], g[4], g[5]);
    gauss2(c.v[2], c.v[3], g[6], g[7]);
    gauss2(d.v[0], d.v[1], g[8], g[9]);
}

inline void put_tri(float* out, uint64_t i, const float v[9]) {
    float* o = out + 12 * i;
    for (int k = 0; k < 3; ++k) {
        o[4 * k + 0] = v[3 * k + 0];
        o[4 * k + 1] = v[3 * k + 1];
        o[4 * k + 2] = v[3 * k + 2];
        o[4 * k + 3] = 0.0f;
    }
}

// One triangle of the unit-cube distribution: centroid ~ U[0,1)^3 scaled by
// `scale` and shifted by `off`; each vertex = centroid + N(0, sigma^2).
inline void cube_tri(uint32_t i, uint32_t s, uint64_t seed, double sigma, const double off[3],
                     double scale, float v[9]) {
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32) ^ 0x41545242u;
    Philox a = philox(i, 0, s, 0xC1u, k0, k1);
    double c[3] = {off[0] + scale * u01f(a.v[0]), off[1] + scale * u01f(a.v[1]),
                   off[2] + scale * u01f(a.v[2])};
    double g[10];
    nine_gauss(i, s, seed, 0xC1u, g);
    for (int k = 0; k < 9; ++k) v[k] = (float)(c[k % 3] + scale * sigma * g[k]);
}

}  // namespace

extern "C" {

int atr_gen_scene(int kind, uint32_t n, uint64_t seed, float* out) {
    if (!out || n == 0) return ATR_ERR_INVALID_ARG;
    if (kind == ATR_SCENE_UNIFORM) {
        const double off[3] = {0.0, 0.0, 0.0};
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; ++i) {
            float v[9];
            cube_tri((uint32_t)i, 0, seed, 0.005, off, 1.0, v);
            put_tri(out, (uint64_t)i, v);
        }
        return ATR_OK;
    }
    if (kind == ATR_SCENE_CLUSTERED) {
        // 64 anisotropic Gaussian components (means U[0,1]^3, per-axis sigma
        // log-uniform in [0.005, 0.1]) for 75% of the triangles, vertex offsets
        // N(0, 0.002^2); the rest is a ground-plane quad grid at y = 0 over
        // [0,1]^2 (1024 x 512 quads for 4,194,304 triangles).
        const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32) ^ 0x41545242u;
        double mean[64][3], sig[64][3];
        for (int c = 0; c < 64; ++c) {
            Philox a = philox((uint32_t)c, 0, 0, 0xC2u, k0, k1);
            Philox b = philox((uint32_t)c, 1, 0, 0xC2u, k0, k1);
            const double lo = std::log(0.005), hi = std::log(0.1);
            for (int k = 0; k < 3; ++k) {
                mean[c][k] = u01f(a.v[k]);
                sig[c][k] = std::exp(lo + (hi - lo) * u01f(b.v[k]));
            }
        }
        const uint64_t plane_quads = (uint64_t)n / 8;
        const uint64_t gx = plane_quads < 1024 ? plane_quads : 1024;
        const uint64_t gz = gx ? plane_quads / gx : 0;
        const uint64_t plane_tris = 2 * gx * gz;
        const uint64_t nmix = (uint64_t)n - plane_tris;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)nmix; ++i) {
            Philox a = philox((uint32_t)i, 0, 1, 0xC3u, k0, k1);
            const int c = (int)(a.v[0] & 63u);
            double g[10];
            nine_gauss((uint32_t)i, 1, seed, 0xC3u, g);
            double gc[4];
            Philox e = philox((uint32_t)i, 4, 1, 0xC3u, k0, k1);
            gauss2(e.v[0], e.v[1], gc[0], gc[1]);
            gauss2(e.v[2], e.v[3], gc[2], gc[3]);
            const double cen[3] = {mean[c][0] + sig[c][0] * gc[0], mean[c][1] + sig[c][1] * gc[1],
                                   mean[c][2] + sig[c][2] * gc[2]};
            float v[9];
            for (int k = 0; k < 9; ++k) v[k] = (float)(cen[k % 3] + 0.002 * g[k]);
            put_tri(out, (uint64_t)i, v);
        }
#pragma omp parallel for schedule(static)
        for (int64_t q = 0; q < (int64_t)(gx * gz); ++q) {
            const uint64_t ax = (uint64_t)q % gx, az = (uint64_t)q / gx;
            const float x0 = (float)ax / (float)gx, x1 = (float)(ax + 1) / (float)gx;
            const float z0 = (float)az / (float)gz, z1 = (float)(az + 1) / (float)gz;
            const float t0[9] = {x0, 0.0f, z0, x1, 0.0f, z0, x1, 0.0f, z1};
            const float t1[9] = {x0, 0.0f, z0, x1, 0.0f, z1, x0, 0.0f, z1};
            put_tri(out, nmix + 2 * (uint64_t)q, t0);
            put_tri(out, nmix + 2 * (uint64_t)q + 1, t1);
        }
        return ATR_OK;
    }
    return ATR_ERR_INVALID_ARG;
}

int atr_gen_batch_sizes(uint32_t count, uint32_t min_tris, uint32_t max_tris, uint64_t seed,
                        uint32_t* sizes) {
    if (!sizes || min_tris < 2 || max_tris < min_tris) return ATR_ERR_INVALID_ARG;
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32) ^ 0x41545242u;
    const double lo = std::log((double)min_tris), hi = std::log((double)max_tris);
    for (uint32_t i = 0; i < count; ++i) {
        Philox a = philox(i, 0, 0, 0xB4u, k0, k1);
        double s = std::floor(std::exp(lo + (hi - lo) * u01d(a.v[0])));
        if (s < min_tris) s = min_tris;
        if (s > max_tris) s = max_tris;
        sizes[i] = (uint32_t)s;
    }
    return ATR_OK;
}

int atr_gen_batch_scene(uint32_t count, const uint32_t* sizes, uint64_t seed, float* out) {
    if (!sizes || !out) return ATR_ERR_INVALID_ARG;
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32) ^ 0x41545242u;
    uint64_t base = 0;
    for (uint32_t m = 0; m < count; ++m) {
        Philox a = philox(m, 1, 0, 0xB4u, k0, k1);
        const double off[3] = {16.0 * u01f(a.v[0]), 16.0 * u01f(a.v[1]), 16.0 * u01f(a.v[2])};
        const uint32_t nm = sizes[m];
#pragma omp parallel for schedule(static) if (nm > 65536)
        for (int64_t i = 0; i < (int64_t)nm; ++i) {
            float v[9];
            cube_tri((uint32_t)i, 2 + m, seed, 0.005, off, 1.0, v);
            put_tri(out, base + (uint64_t)i, v);
        }
        base += nm;
    }
    return ATR_OK;
}

int atr_gen_rays_pinhole(uint32_t width, uint32_t height, const float* eye, float fov_deg,
                         float* rays) {
    if (!rays || !eye || width == 0 || height == 0) return ATR_ERR_INVALID_ARG;
    const double th = std::tan(0.5 * fov_deg * 3.14159265358979323846 / 180.0);
    const double aspect = (double)width / (double)height;
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < (int64_t)width * height; ++p) {
        const uint64_t px = (uint64_t)p % width, py = (uint64_t)p / width;
        double dx = (2.0 * ((double)px + 0.5) / width - 1.0) * th * aspect;
        double dy = (1.0 - 2.0 * ((double)py + 0.5) / height) * th;
        double dz = 1.0;
        const double inv = 1.0 / std::sqrt(dx * dx + dy * dy + dz * dz);
        float* r = rays + 8 * p;
        r[0] = eye[0]; r[1] = eye[1]; r[2] = eye[2]; r[3] = 0.0f;
        r[4] = (float)(dx * inv); r[5] = (float)(dy * inv); r[6] = (float)(dz * inv); r[7] = 1e30f;
    }
    return ATR_OK;
}

int atr_gen_rays_random(uint64_t n, uint64_t seed, const float* bbmin, const float* bbmax,
                        float* rays) {
    if (!rays || !bbmin || !bbmax) return ATR_ERR_INVALID_ARG;
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32) ^ 0x41545242u;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        Philox a = philox((uint32_t)i, (uint32_t)((uint64_t)i >> 32), 7, 0xA1u, k0, k1);
        Philox b = philox((uint32_t)i, (uint32_t)((uint64_t)i >> 32), 8, 0xA1u, k0, k1);
        double g[4];
        gauss2(b.v[0], b.v[1], g[0], g[1]);
        gauss2(b.v[2], b.v[3], g[2], g[3]);
        double len = std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
        if (len == 0.0) { g[0] = 1.0; len = 1.0; }
        float* r = rays + 8 * i;
        for (int k = 0; k < 3; ++k)
            r[k] = (float)(bbmin[k] + (double)(bbmax[k] - bbmin[k]) * u01f(a.v[k]));
        r[3] = 0.0f;
        for (int k = 0; k < 3; ++k) r[4 + k] = (float)(g[k] / len);
        r[7] = 1e30f;
    }
    return ATR_OK;
}

}  // extern "C"
