// The oracle's own copy of the seeded benchmark inputs (test infrastructure).
//
// The CPU reference leg of the benchmark builds its scene and rays with these
// functions, so it never maps the product library.  They restate the workload
// definitions (displaced icosphere, ball rays, triangle soup, pinhole camera
// rays) with the reference's PCG32 (src/core/rng.rs:21-63, oracle_common.h)
// in double precision; tests/test_golden.py checks that they produce the same
// bytes as the product's generators.
#include <cmath>
#include <cstdint>
#include <limits>
#include <unordered_map>
#include <vector>

#include "oracle.h"
#include "oracle_common.h"

namespace {

constexpr double kPi = 3.14159265358979323846;

struct V3 {
    double x, y, z;
};

V3 unit(V3 v) {
    const double len = std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
    return {v.x / len, v.y / len, v.z / len};
}

// Direction on S^2 from two uniforms: z = 1 - 2u, phi = 2 pi v.
V3 sphere_point(double u, double v) {
    const double z = 1.0 - 2.0 * u;
    const double r = std::sqrt(std::fmax(0.0, 1.0 - z * z));
    const double phi = 2.0 * kPi * v;
    return {r * std::cos(phi), r * std::sin(phi), z};
}

void put_ray(float* rec, const float o[3], V3 d, float tmax) {
    rec[0] = o[0]; rec[1] = o[1]; rec[2] = o[2]; rec[3] = 0.0f;
    rec[4] = (float)d.x; rec[5] = (float)d.y; rec[6] = (float)d.z; rec[7] = tmax;
}

}  // namespace

extern "C" {

void orc_wl_icosphere_counts(uint32_t level, uint32_t* nv, uint32_t* nt) {
    uint64_t faces = 20;
    for (uint32_t l = 0; l < level; ++l) faces *= 4;
    *nt = (uint32_t)faces;
    *nv = (uint32_t)(faces / 2 + 2);
}

// Icosahedron (12 golden-ratio vertices, 20 faces) split `level` times, each
// edge midpoint created once (in face order, edges ab, bc, ca) and pushed to
// the unit sphere; each face becomes (a,ab,ca) (b,bc,ab) (c,ca,bc) (ab,bc,ca).
// Vertex radius: radius * (1 + amplitude * sum_k sin(4k x + phi_k) cos(4k y)
// sin(4k z)), phases phi_k = 2 pi * uniform_float of Rng::new(seed).
void orc_wl_icosphere(uint32_t level, uint64_t seed, float amplitude, float radius, const float centre[3],
                      float* xyz, uint32_t* idx) {
    const double g = 0.5 * (1.0 + std::sqrt(5.0));
    std::vector<V3> vtx;
    const double base[12][3] = {{-1, g, 0}, {1, g, 0}, {-1, -g, 0}, {1, -g, 0}, {0, -1, g}, {0, 1, g},
                                {0, -1, -g}, {0, 1, -g}, {g, 0, -1}, {g, 0, 1}, {-g, 0, -1}, {-g, 0, 1}};
    for (const auto& b : base) vtx.push_back(unit({b[0], b[1], b[2]}));
    std::vector<uint32_t> tri = {0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4,
                                 11, 10, 2, 10, 7, 6, 7, 1, 8, 3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8,
                                 3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1};
    for (uint32_t l = 0; l < level; ++l) {
        std::unordered_map<uint64_t, uint32_t> edge_mid;
        auto mid = [&](uint32_t a, uint32_t b) {
            const uint64_t key = a < b ? ((uint64_t)a << 32 | b) : ((uint64_t)b << 32 | a);
            auto it = edge_mid.find(key);
            if (it != edge_mid.end()) return it->second;
            const V3 m = unit({(vtx[a].x + vtx[b].x) * 0.5, (vtx[a].y + vtx[b].y) * 0.5,
                               (vtx[a].z + vtx[b].z) * 0.5});
            vtx.push_back(m);
            const uint32_t id = (uint32_t)(vtx.size() - 1);
            edge_mid[key] = id;
            return id;
        };
        std::vector<uint32_t> next;
        next.reserve(tri.size() * 4);
        for (size_t f = 0; f < tri.size(); f += 3) {
            const uint32_t a = tri[f], b = tri[f + 1], c = tri[f + 2];
            const uint32_t ab = mid(a, b), bc = mid(b, c), ca = mid(c, a);
            for (uint32_t v : {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca}) next.push_back(v);
        }
        tri.swap(next);
    }
    orc::Rng rng(seed);
    double phase[4];
    for (double& p : phase) p = 2.0 * kPi * (double)rng.uniform_float();
    for (size_t i = 0; i < vtx.size(); ++i) {
        const V3 p = vtx[i];
        double sum = 0.0;
        for (int k = 1; k <= 4; ++k) {
            const double w = 4.0 * k;
            sum += std::sin(w * p.x + phase[k - 1]) * std::cos(w * p.y) * std::sin(w * p.z);
        }
        const double r = (double)radius * (1.0 + (double)amplitude * sum);
        xyz[3 * i] = (float)((double)centre[0] + r * p.x);
        xyz[3 * i + 1] = (float)((double)centre[1] + r * p.y);
        xyz[3 * i + 2] = (float)((double)centre[2] + r * p.z);
    }
    for (size_t i = 0; i < tri.size(); ++i) idx[i] = tri[i];
}

// n rays of Rng::new(seed) after `skip` discarded draws: five uniforms per ray
// (origin radius * cbrt(u0) along sphere_point(u1, u2), direction
// sphere_point(u3, u4)); the first n_closest have tmax = inf, the others one
// more uniform for tmax in [tmax_lo, tmax_hi].  Records are 8 floats.
void orc_wl_ball_rays(uint64_t seed, uint64_t skip, uint64_t n, uint64_t n_closest, float radius, float tmax_lo,
                      float tmax_hi, float* out) {
    orc::Rng rng(seed);
    for (uint64_t i = 0; i < skip; ++i) rng.uniform_u32();
    for (uint64_t i = 0; i < n; ++i) {
        double u[5];
        for (double& x : u) x = rng.uniform_float();
        const double rad = (double)radius * std::cbrt(u[0]);
        const V3 p = sphere_point(u[1], u[2]);
        const float o[3] = {(float)(rad * p.x), (float)(rad * p.y), (float)(rad * p.z)};
        float tmax = std::numeric_limits<float>::infinity();
        if (i >= n_closest) {
            const double w = rng.uniform_float();
            tmax = (float)((double)tmax_lo + ((double)tmax_hi - (double)tmax_lo) * w);
        }
        put_ray(out + 8 * i, o, sphere_point(u[3], u[4]), tmax);
    }
}

// n triangles of Rng::new(seed): a centre of three uniforms, then per vertex
// per axis centre + (2 s u - s); indices 3t, 3t+1, 3t+2.
void orc_wl_soup(uint64_t seed, uint32_t n, float spread, float* xyz, uint32_t* idx) {
    orc::Rng rng(seed);
    const double s = spread;
    for (uint32_t t = 0; t < n; ++t) {
        double c[3];
        for (double& x : c) x = rng.uniform_float();
        for (int v = 0; v < 3; ++v) {
            for (int k = 0; k < 3; ++k)
                xyz[9 * (size_t)t + 3 * v + k] = (float)(c[k] + (2.0 * s * (double)rng.uniform_float() - s));
            idx[3 * (size_t)t + v] = 3 * t + v;
        }
    }
}

// width x height pinhole rays through pixel centres from `eye` along +z,
// vertical field of view fov_deg, up +y, tmax = inf.
void orc_wl_camera_rays(uint32_t width, uint32_t height, const float eye[3], float fov_deg, float* out) {
    const double half = std::tan(0.5 * (double)fov_deg * kPi / 180.0);
    const double aspect = (double)width / (double)height;
    for (uint32_t y = 0; y < height; ++y)
        for (uint32_t x = 0; x < width; ++x) {
            const double sx = ((x + 0.5) / width * 2.0 - 1.0) * half * aspect;
            const double sy = (1.0 - (y + 0.5) / height * 2.0) * half;
            put_ray(out + 8 * ((size_t)y * width + x), eye, unit({sx, sy, 1.0}),
                    std::numeric_limits<float>::infinity());
        }
}

}  // extern "C"
