// Seeded synthetic scenes and rays (see include/illume_workloads.h).
#include "illume_workloads.h"

#include <cmath>
#include <limits>
#include <unordered_map>
#include <vector>

#include "pcg32.h"

namespace {

const double kPiD = 3.14159265358979323846;

struct D3 { double x, y, z; };
inline D3 normalized(D3 v) {
    double l = std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
    return {v.x / l, v.y / l, v.z / l};
}

}  // namespace

extern "C" {

void ilm_wl_rng_floats(uint64_t seq, uint64_t n, float* out) {
    ilm::Pcg32 r(seq);
    for (uint64_t i = 0; i < n; ++i) out[i] = r.uniform_float();
}

void ilm_wl_rng_u32(uint64_t seq, uint64_t n, uint32_t* out) {
    ilm::Pcg32 r(seq);
    for (uint64_t i = 0; i < n; ++i) out[i] = r.uniform_u32();
}

void ilm_wl_soup(uint64_t seed, uint32_t n, float spread, float* xyz, uint32_t* idx) {
    ilm::Pcg32 r(seed);
    const double s = spread;
    for (uint32_t t = 0; t < n; ++t) {
        double c[3];
        for (int k = 0; k < 3; ++k) c[k] = r.uniform_float();
        for (int v = 0; v < 3; ++v)
            for (int k = 0; k < 3; ++k) {
                double u = r.uniform_float();
                xyz[9 * (size_t)t + 3 * v + k] = (float)(c[k] + (2.0 * s * u - s));
            }
        idx[3 * (size_t)t] = 3 * t;
        idx[3 * (size_t)t + 1] = 3 * t + 1;
        idx[3 * (size_t)t + 2] = 3 * t + 2;
    }
}

void ilm_wl_icosphere_counts(uint32_t level, uint32_t* nv, uint32_t* nt) {
    uint64_t f = 1;
    for (uint32_t i = 0; i < level; ++i) f *= 4;
    *nv = (uint32_t)(10 * f + 2);
    *nt = (uint32_t)(20 * f);
}

void ilm_wl_icosphere(uint32_t level, uint64_t seed, float amplitude, float radius,
                      const float centre[3], float* xyz, uint32_t* idx) {
    const double t = (1.0 + std::sqrt(5.0)) / 2.0;
    std::vector<D3> v = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0},
                         {0, -1, t}, {0, 1, t}, {0, -1, -t}, {0, 1, -t},
                         {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    for (auto& p : v) p = normalized(p);
    std::vector<uint32_t> f = {0, 11, 5, 0, 5, 1,  0, 1, 7,   0, 7, 10, 0, 10, 11,
                               1, 5, 9,  5, 11, 4, 11, 10, 2, 10, 7, 6, 7, 1, 8,
                               3, 9, 4,  3, 4, 2,  3, 2, 6,   3, 6, 8,  3, 8, 9,
                               4, 9, 5,  2, 4, 11, 6, 2, 10,  8, 6, 7,  9, 8, 1};
    for (uint32_t l = 0; l < level; ++l) {
        std::unordered_map<uint64_t, uint32_t> mid;
        mid.reserve(f.size());
        auto midpoint = [&](uint32_t a, uint32_t b) -> uint32_t {
            uint64_t key = a < b ? ((uint64_t)a << 32) | b : ((uint64_t)b << 32) | a;
            auto it = mid.find(key);
            if (it != mid.end()) return it->second;
            D3 m = normalized({(v[a].x + v[b].x) * 0.5, (v[a].y + v[b].y) * 0.5,
                               (v[a].z + v[b].z) * 0.5});
            v.push_back(m);
            uint32_t id = (uint32_t)v.size() - 1;
            mid.emplace(key, id);
            return id;
        };
        std::vector<uint32_t> nf;
        nf.reserve(f.size() * 4);
        for (size_t i = 0; i < f.size(); i += 3) {
            uint32_t a = f[i], b = f[i + 1], c = f[i + 2];
            uint32_t ab = midpoint(a, b), bc = midpoint(b, c), ca = midpoint(c, a);
            uint32_t tris[12] = {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca};
            nf.insert(nf.end(), tris, tris + 12);
        }
        f.swap(nf);
    }
    ilm::Pcg32 r(seed);
    double phase[4];
    for (int k = 0; k < 4; ++k) phase[k] = 2.0 * kPiD * (double)r.uniform_float();
    for (size_t i = 0; i < v.size(); ++i) {
        const D3& p = v[i];
        double s = 0.0;
        for (int k = 1; k <= 4; ++k) {
            double w = 4.0 * k;
            s += std::sin(w * p.x + phase[k - 1]) * std::cos(w * p.y) * std::sin(w * p.z);
        }
        double rr = (double)radius * (1.0 + (double)amplitude * s);
        xyz[3 * i] = (float)((double)centre[0] + rr * p.x);
        xyz[3 * i + 1] = (float)((double)centre[1] + rr * p.y);
        xyz[3 * i + 2] = (float)((double)centre[2] + rr * p.z);
    }
    for (size_t i = 0; i < f.size(); ++i) idx[i] = f[i];
}

void ilm_wl_camera_rays(uint32_t width, uint32_t height, const float eye[3], float fov_deg,
                        ilm_ray* out) {
    const double th = std::tan(0.5 * (double)fov_deg * kPiD / 180.0);
    const double aspect = (double)width / (double)height;
    for (uint32_t y = 0; y < height; ++y)
        for (uint32_t x = 0; x < width; ++x) {
            double sx = ((x + 0.5) / width * 2.0 - 1.0) * th * aspect;
            double sy = (1.0 - (y + 0.5) / height * 2.0) * th;
            D3 d = normalized({sx, sy, 1.0});
            ilm_ray& r = out[(size_t)y * width + x];
            r.o[0] = eye[0]; r.o[1] = eye[1]; r.o[2] = eye[2];
            r.tmin = 0.0f;
            r.d[0] = (float)d.x; r.d[1] = (float)d.y; r.d[2] = (float)d.z;
            r.tmax = std::numeric_limits<float>::infinity();
        }
}

void ilm_wl_cornell_counts(uint32_t ico_level, uint32_t* nv, uint32_t* nt) {
    uint32_t iv, it;
    ilm_wl_icosphere_counts(ico_level, &iv, &it);
    *nv = 5 * 4 + 4 + 2 * 8 + iv;
    *nt = 5 * 2 + 2 + 2 * 12 + it;
}

void ilm_wl_cornell(uint32_t ico_level, uint64_t seed, float* xyz, uint32_t* idx, uint32_t* mat, float* albedo,
                    float* emission) {
    const float alb[4][3] = {{0.73f, 0.73f, 0.73f}, {0.63f, 0.065f, 0.05f}, {0.14f, 0.45f, 0.09f}, {0, 0, 0}};
    const float emi[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {15.0f, 15.0f, 15.0f}};
    for (int m = 0; m < 4; ++m)
        for (int k = 0; k < 3; ++k) { albedo[3 * m + k] = alb[m][k]; emission[3 * m + k] = emi[m][k]; }
    uint32_t nv = 0, nt = 0;
    auto vert = [&](double x, double y, double z) {
        xyz[3 * nv] = (float)x; xyz[3 * nv + 1] = (float)y; xyz[3 * nv + 2] = (float)z;
        return nv++;
    };
    auto tri = [&](uint32_t a, uint32_t b, uint32_t c, uint32_t m) {
        idx[3 * nt] = a; idx[3 * nt + 1] = b; idx[3 * nt + 2] = c;
        mat[nt++] = m;
    };
    // quad a-b-c-d as triangles (a,b,c) and (a,c,d)
    auto quad = [&](const double* a, const double* b, const double* c, const double* d, uint32_t m) {
        uint32_t ia = vert(a[0], a[1], a[2]), ib = vert(b[0], b[1], b[2]);
        uint32_t ic = vert(c[0], c[1], c[2]), id = vert(d[0], d[1], d[2]);
        tri(ia, ib, ic, m);
        tri(ia, ic, id, m);
    };
    const double f0[3] = {0, 0, 0}, f1[3] = {1, 0, 0}, f2[3] = {1, 0, 1}, f3[3] = {0, 0, 1};
    const double c0[3] = {0, 1, 0}, c1[3] = {1, 1, 0}, c2[3] = {1, 1, 1}, c3[3] = {0, 1, 1};
    quad(f0, f3, f2, f1, 0);   // floor
    quad(c0, c1, c2, c3, 0);   // ceiling
    quad(f3, c3, c2, f2, 0);   // back wall z = 1
    quad(f0, c0, c3, f3, 1);   // left wall x = 0 (red)
    quad(f1, f2, c2, c1, 2);   // right wall x = 1 (green)
    // light: (x0,h,z0) (x1,h,z0) (x1,h,z1) (x0,h,z1) -> both normals -y
    const double h = 0.999, lx0 = 0.375, lx1 = 0.625, lz0 = 0.375, lz1 = 0.625;
    const double l0[3] = {lx0, h, lz0}, l1[3] = {lx1, h, lz0}, l2[3] = {lx1, h, lz1}, l3[3] = {lx0, h, lz1};
    quad(l0, l1, l2, l3, 3);
    auto box = [&](double cx, double cy, double cz, double sx, double sy, double sz, double deg) {
        double a = deg * kPiD / 180.0, ca = std::cos(a), sa = std::sin(a);
        uint32_t base = nv;
        for (int k = 0; k < 8; ++k) {
            double x = (k & 1 ? 0.5 : -0.5) * sx, y = (k & 2 ? 0.5 : -0.5) * sy, z = (k & 4 ? 0.5 : -0.5) * sz;
            vert(cx + ca * x + sa * z, cy + y, cz - sa * x + ca * z);
        }
        const int faces[6][4] = {{0, 2, 3, 1}, {4, 5, 7, 6}, {0, 1, 5, 4}, {2, 6, 7, 3}, {0, 4, 6, 2}, {1, 3, 7, 5}};
        for (auto& fc : faces) {
            tri(base + fc[0], base + fc[1], base + fc[2], 0);
            tri(base + fc[0], base + fc[2], base + fc[3], 0);
        }
    };
    box(0.33, 0.3, 0.65, 0.3, 0.6, 0.3, 18.0);
    box(0.66, 0.15, 0.33, 0.3, 0.3, 0.3, -18.0);
    uint32_t iv, it;
    ilm_wl_icosphere_counts(ico_level, &iv, &it);
    const float centre[3] = {0.66f, 0.52f, 0.33f};
    ilm_wl_icosphere(ico_level, seed, 0.05f, 0.2f, centre, xyz + 3 * (size_t)nv, idx + 3 * (size_t)nt);
    for (uint32_t i = 0; i < 3 * it; ++i) idx[3 * (size_t)nt + i] += nv;
    for (uint32_t i = 0; i < it; ++i) mat[nt + i] = 0;
}

void ilm_wl_ball_rays(uint64_t seed, uint64_t skip, uint64_t n, uint64_t n_closest,
                      float radius, float tmax_lo, float tmax_hi, ilm_ray* out) {
    ilm::Pcg32 r(seed);
    for (uint64_t i = 0; i < skip; ++i) r.uniform_u32();
    auto sphere_dir = [&](double u, double v) -> D3 {
        double z = 1.0 - 2.0 * u;
        double rr = std::sqrt(std::fmax(0.0, 1.0 - z * z));
        double phi = 2.0 * kPiD * v;
        return {rr * std::cos(phi), rr * std::sin(phi), z};
    };
    for (uint64_t i = 0; i < n; ++i) {
        double u0 = r.uniform_float(), u1 = r.uniform_float(), u2 = r.uniform_float();
        double u3 = r.uniform_float(), u4 = r.uniform_float();
        double rad = (double)radius * std::cbrt(u0);
        D3 po = sphere_dir(u1, u2);
        D3 d = sphere_dir(u3, u4);
        ilm_ray& ray = out[i];
        ray.o[0] = (float)(rad * po.x); ray.o[1] = (float)(rad * po.y); ray.o[2] = (float)(rad * po.z);
        ray.tmin = 0.0f;
        ray.d[0] = (float)d.x; ray.d[1] = (float)d.y; ray.d[2] = (float)d.z;
        if (i < n_closest) {
            ray.tmax = std::numeric_limits<float>::infinity();
        } else {
            double u5 = r.uniform_float();
            ray.tmax = (float)((double)tmax_lo + ((double)tmax_hi - (double)tmax_lo) * u5);
        }
    }
}

}  // extern "C"
