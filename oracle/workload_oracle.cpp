// ORACLE -- test infrastructure only.
//
// The seeded synthetic scenes and rays of the benchmark configurations,
// generated on the host by the checker itself, so that the timed host-core
// baseline and the reference arm of bench.py need nothing from the product
// library.  tests/test_cpu_oracle.py pins these generators to the committed
// workload digests and to the product's own generator, element for element.
//
// Definition of the streams (identical bits wherever they are generated):
//   * counter-based Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel
//     random numbers: as easy as 1, 2, 3", SC'11) with counter
//     (element, sub-stream, stream, tag) and key (seed low word,
//     seed high word ^ 0x41545242);
//   * uniform floats from the top 24 bits (exact in float), uniform doubles
//     in (0, 1) from (u + 0.5) / 2^32;
//   * Gaussians by the Box-Muller transform in double precision.

#include <cmath>
#include <cstdint>

namespace {

struct Ctr {
    uint32_t w[4];
};

Ctr philox10(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3, uint32_t key0, uint32_t key1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int round = 0; round < 10; ++round) {
        if (round > 0) {
            key0 += W0;
            key1 += W1;
        }
        const uint64_t a = (uint64_t)M0 * x0;
        const uint64_t b = (uint64_t)M1 * x2;
        const uint32_t y0 = (uint32_t)(b >> 32) ^ x1 ^ key0;
        const uint32_t y2 = (uint32_t)(a >> 32) ^ x3 ^ key1;
        x1 = (uint32_t)b;
        x3 = (uint32_t)a;
        x0 = y0;
        x2 = y2;
    }
    return Ctr{{x0, x1, x2, x3}};
}

struct Key {
    uint32_t k0, k1;
    explicit Key(uint64_t seed) : k0((uint32_t)seed), k1((uint32_t)(seed >> 32) ^ 0x41545242u) {}
    Ctr at(uint32_t e, uint32_t sub, uint32_t stream, uint32_t tag) const {
        return philox10(e, sub, stream, tag, k0, k1);
    }
};

float unit_f(uint32_t u) { return (float)(u >> 8) * (1.0f / 16777216.0f); }
double unit_d(uint32_t u) { return ((double)u + 0.5) * (1.0 / 4294967296.0); }

void box_muller(uint32_t a, uint32_t b, double* z0, double* z1) {
    const double radius = std::sqrt(-2.0 * std::log(unit_d(a)));
    const double angle = 6.283185307179586 * unit_d(b);
    *z0 = radius * std::cos(angle);
    *z1 = radius * std::sin(angle);
}

// Nine standard normals per triangle, from sub-streams 1..3 of (e, stream, tag).
void normals9(const Key& key, uint32_t e, uint32_t stream, uint32_t tag, double z[10]) {
    for (int j = 0; j < 3; ++j) {
        const Ctr c = key.at(e, 1 + j, stream, tag);
        box_muller(c.w[0], c.w[1], &z[4 * j], &z[4 * j + 1]);
        if (j < 2) box_muller(c.w[2], c.w[3], &z[4 * j + 2], &z[4 * j + 3]);
    }
}

void store_triangle(float* out, uint64_t t, const float xyz[9]) {
    float* o = out + 12 * t;
    for (int vtx = 0; vtx < 3; ++vtx) {
        for (int a = 0; a < 3; ++a) o[4 * vtx + a] = xyz[3 * vtx + a];
        o[4 * vtx + 3] = 0.0f;
    }
}

// Centroid uniform in [off, off + scale)^3, each vertex offset by
// N(0, (scale * sigma)^2) per component.
void unit_cube_triangle(const Key& key, uint32_t e, uint32_t stream, double sigma, const double off[3],
                        double scale, float xyz[9]) {
    const Ctr c = key.at(e, 0, stream, 0xC1u);
    const double centre[3] = {off[0] + scale * unit_f(c.w[0]), off[1] + scale * unit_f(c.w[1]),
                              off[2] + scale * unit_f(c.w[2])};
    double z[10];
    normals9(key, e, stream, 0xC1u, z);
    for (int k = 0; k < 9; ++k) xyz[k] = (float)(centre[k % 3] + scale * sigma * z[k]);
}

}  // namespace

extern "C" {

// kind 0: unit-cube scene (centroids U[0,1)^3, vertex offsets N(0, 0.005^2)).
// kind 1: clustered scene (64 anisotropic Gaussians for the triangles before
// the ground plane, vertex offsets N(0, 0.002^2); a y = 0 quad grid over
// [0,1]^2 of min(n/8, 1024) x (n/8 / that) quads, two triangles each, last).
int orc_gen_scene(int kind, uint32_t n, uint64_t seed, float* out) {
    if (!out || n == 0) return 1;
    const Key key(seed);
    if (kind == 0) {
        const double zero[3] = {0.0, 0.0, 0.0};
#pragma omp parallel for schedule(static)
        for (int64_t t = 0; t < (int64_t)n; ++t) {
            float xyz[9];
            unit_cube_triangle(key, (uint32_t)t, 0, 0.005, zero, 1.0, xyz);
            store_triangle(out, (uint64_t)t, xyz);
        }
        return 0;
    }
    if (kind != 1) return 1;
    double mu[64][3], sd[64][3];
    const double log_lo = std::log(0.005), log_hi = std::log(0.1);
    for (uint32_t g = 0; g < 64; ++g) {
        const Ctr m = key.at(g, 0, 0, 0xC2u), s = key.at(g, 1, 0, 0xC2u);
        for (int a = 0; a < 3; ++a) {
            mu[g][a] = unit_f(m.w[a]);
            sd[g][a] = std::exp(log_lo + (log_hi - log_lo) * unit_f(s.w[a]));
        }
    }
    const uint64_t quads = (uint64_t)n / 8;
    const uint64_t nx = quads < 1024 ? quads : 1024;
    const uint64_t nz = nx ? quads / nx : 0;
    const uint64_t gaussian_tris = (uint64_t)n - 2 * nx * nz;
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < (int64_t)gaussian_tris; ++t) {
        const uint32_t e = (uint32_t)t;
        const int g = (int)(key.at(e, 0, 1, 0xC3u).w[0] & 63u);
        double z[10], zc[4];
        normals9(key, e, 1, 0xC3u, z);
        const Ctr c = key.at(e, 4, 1, 0xC3u);
        box_muller(c.w[0], c.w[1], &zc[0], &zc[1]);
        box_muller(c.w[2], c.w[3], &zc[2], &zc[3]);
        double centre[3];
        for (int a = 0; a < 3; ++a) centre[a] = mu[g][a] + sd[g][a] * zc[a];
        float xyz[9];
        for (int k = 0; k < 9; ++k) xyz[k] = (float)(centre[k % 3] + 0.002 * z[k]);
        store_triangle(out, (uint64_t)t, xyz);
    }
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < (int64_t)(nx * nz); ++q) {
        const uint64_t ix = (uint64_t)q % nx, iz = (uint64_t)q / nx;
        const float xa = (float)ix / (float)nx, xb = (float)(ix + 1) / (float)nx;
        const float za = (float)iz / (float)nz, zb = (float)(iz + 1) / (float)nz;
        const float lower[9] = {xa, 0.0f, za, xb, 0.0f, za, xb, 0.0f, zb};
        const float upper[9] = {xa, 0.0f, za, xb, 0.0f, zb, xa, 0.0f, zb};
        store_triangle(out, gaussian_tris + 2 * (uint64_t)q, lower);
        store_triangle(out, gaussian_tris + 2 * (uint64_t)q + 1, upper);
    }
    return 0;
}

// Pinhole primary rays, one per pixel in row-major order: origin `eye`,
// tmin 0, tmax 1e30, direction through the pixel centre of a view looking
// down +z with vertical field of view fov_deg.
int orc_gen_rays_pinhole(uint32_t width, uint32_t height, const float* eye, float fov_deg, float* rays) {
    if (!rays || !eye || width == 0 || height == 0) return 1;
    const double half = std::tan(0.5 * fov_deg * 3.14159265358979323846 / 180.0);
    const double aspect = (double)width / (double)height;
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < (int64_t)width * height; ++p) {
        const uint64_t col = (uint64_t)p % width, row = (uint64_t)p / width;
        const double dx = (2.0 * ((double)col + 0.5) / width - 1.0) * half * aspect;
        const double dy = (1.0 - 2.0 * ((double)row + 0.5) / height) * half;
        const double dz = 1.0;
        const double inv_len = 1.0 / std::sqrt(dx * dx + dy * dy + dz * dz);
        float* r = rays + 8 * p;
        r[0] = eye[0];
        r[1] = eye[1];
        r[2] = eye[2];
        r[3] = 0.0f;
        r[4] = (float)(dx * inv_len);
        r[5] = (float)(dy * inv_len);
        r[6] = (float)(dz * inv_len);
        r[7] = 1e30f;
    }
    return 0;
}

// Random rays: origins uniform in [bbmin, bbmax), directions uniform on the
// sphere (normalised Gaussian triplets), tmin 0, tmax 1e30.
int orc_gen_rays_random(uint64_t n, uint64_t seed, const float* bbmin, const float* bbmax, float* rays) {
    if (!rays || !bbmin || !bbmax) return 1;
    const Key key(seed);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const uint32_t lo = (uint32_t)i, hi = (uint32_t)((uint64_t)i >> 32);
        const Ctr o = key.at(lo, hi, 7, 0xA1u), d = key.at(lo, hi, 8, 0xA1u);
        double z[4];
        box_muller(d.w[0], d.w[1], &z[0], &z[1]);
        box_muller(d.w[2], d.w[3], &z[2], &z[3]);
        double len = std::sqrt(z[0] * z[0] + z[1] * z[1] + z[2] * z[2]);
        if (len == 0.0) {
            z[0] = 1.0;
            len = 1.0;
        }
        float* r = rays + 8 * i;
        for (int a = 0; a < 3; ++a) r[a] = (float)(bbmin[a] + (double)(bbmax[a] - bbmin[a]) * unit_f(o.w[a]));
        r[3] = 0.0f;
        for (int a = 0; a < 3; ++a) r[4 + a] = (float)(z[a] / len);
        r[7] = 1e30f;
    }
    return 0;
}

// Mesh sizes of the batched workload: floor(exp(U(ln lo, ln hi))) clamped to [lo, hi].
int orc_gen_batch_sizes(uint32_t count, uint32_t lo, uint32_t hi, uint64_t seed, uint32_t* sizes) {
    if (!sizes || lo < 2 || hi < lo) return 1;
    const Key key(seed);
    const double a = std::log((double)lo), b = std::log((double)hi);
    for (uint32_t m = 0; m < count; ++m) {
        double s = std::floor(std::exp(a + (b - a) * unit_d(key.at(m, 0, 0, 0xB4u).w[0])));
        s = s < lo ? lo : (s > hi ? hi : s);
        sizes[m] = (uint32_t)s;
    }
    return 0;
}

// Meshes end to end; mesh m is a unit-cube scene (stream 2 + m) shifted by a
// random offset in [0, 16)^3.
int orc_gen_batch_scene(uint32_t count, const uint32_t* sizes, uint64_t seed, float* out) {
    if (!sizes || !out) return 1;
    const Key key(seed);
    uint64_t first = 0;
    for (uint32_t m = 0; m < count; ++m) {
        const Ctr c = key.at(m, 1, 0, 0xB4u);
        const double off[3] = {16.0 * unit_f(c.w[0]), 16.0 * unit_f(c.w[1]), 16.0 * unit_f(c.w[2])};
#pragma omp parallel for schedule(static) if (sizes[m] > 65536)
        for (int64_t t = 0; t < (int64_t)sizes[m]; ++t) {
            float xyz[9];
            unit_cube_triangle(key, (uint32_t)t, 2 + m, 0.005, off, 1.0, xyz);
            store_triangle(out, first + (uint64_t)t, xyz);
        }
        first += sizes[m];
    }
    return 0;
}

}  // extern "C"
