// CPU restatement of the path-tracing loop (test infrastructure only).
//
// rs_illume has no PathIntegrator (src/integrators/mod.rs declares only `ao`),
// no area light, no matte material and no stratified sampler; the pieces that
// exist are SamplerIntegratorBase::render (core/integrator.rs:48-145),
// uniform_sample_one_light / estimate_direct (integrator.rs:321-494), BSDF +
// LambertianReflection (core/reflection/mod.rs:50-276,
// reflection/lambertian_reflection.rs:7-45), the sampling warps
// (core/sampling.rs) and the spawn-ray offsets (core/interaction.rs:33-72,
// geometry/ray.rs:79-102).  This file wires those into the PBR-book path
// integrator loop (throughput beta, emission on the camera bounce, one-light
// NEE with MIS, cosine BSDF sampling, Russian roulette), with a one-sided
// diffuse area light per emissive triangle (Triangle::sample,
// shapes/triangle.rs:616-642; Shape::sample_with_point / pdf_with_point,
// core/shape.rs:40-83) and Lambertian materials.
//
// Repairs applied: D16 (BSDF::sample_f samples in the local frame), D20 (box
// film: a pixel is the mean of its samples), D21 (the BSDF-sampled light term
// is accumulated), D25 (pdf_with_point divides by |cos|*area; shape.rs:77-78
// multiplies by area).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>
#include <vector>

#include "oracle.h"
#include "oracle_common.h"

namespace orc {
namespace {

struct V { float x, y, z; };
inline V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V operator*(V a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V operator*(float s, V a) { return {a.x * s, a.y * s, a.z * s}; }
inline V operator-(V a) { return {-a.x, -a.y, -a.z}; }
inline float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V vabs(V a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
// Vector3::cross in f64 (geometry/vector3.rs:67-82)
inline V cross(V a, V b) {
    double ax = a.x, ay = a.y, az = a.z, bx = b.x, by = b.y, bz = b.z;
    return {(float)(ay * bz - az * by), (float)(az * bx - ax * bz), (float)(ax * by - ay * bx)};
}
inline float length(V a) { return std::sqrt(dot(a, a)); }
inline V normalize(V a) { return a * (1.0f / length(a)); }
inline float comp(V a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

struct RGB { float r, g, b; };
inline RGB operator+(RGB a, RGB b) { return {a.r + b.r, a.g + b.g, a.b + b.b}; }
inline RGB operator*(RGB a, RGB b) { return {a.r * b.r, a.g * b.g, a.b * b.b}; }
inline RGB operator*(RGB a, float s) { return {a.r * s, a.g * s, a.b * s}; }
inline bool is_black(RGB a) { return a.r == 0.0f && a.g == 0.0f && a.b == 0.0f; }
inline float max_comp(RGB a) { return std::fmax(a.r, std::fmax(a.g, a.b)); }
// RGBSpectrum::y (core/spectrum.rs:498-501)
inline float luminance(RGB a) { return 0.212671f * a.r + 0.715160f * a.g + 0.072169f * a.b; }

// offset_ray_origin (geometry/ray.rs:79-102)
V offset_ray_origin(V p, V perr, V n, V w) {
    float d = dot(vabs(n), perr);
    V off = n * d;
    if (dot(w, n) < 0.0f) off = -off;
    V po = p + off;
    float* c = &po.x;
    const float* o = &off.x;
    for (int i = 0; i < 3; ++i) {
        if (o[i] > 0.0f) c[i] = next_float_up(c[i]);
        else if (o[i] < 0.0f) c[i] = next_float_down(c[i]);
    }
    return po;
}

// coordinate_system (geometry/vector3.rs:520-540)
void coordinate_system(V v1, V* v2, V* v3) {
    if (std::fabs(v1.x) > std::fabs(v1.y)) {
        float l = std::sqrt(v1.x * v1.x + v1.z * v1.z);
        *v2 = {-v1.z / l, 0.0f, v1.x / l};
    } else {
        float l = std::sqrt(v1.y * v1.y + v1.z * v1.z);
        *v2 = {0.0f, v1.z / l, -v1.y / l};
    }
    *v3 = cross(v1, *v2);
}

// concentric_sample_disk / cosine_sample_hemisphere (core/sampling.rs:210-230, 316-320)
V cosine_sample_hemisphere(float u0, float u1) {
    float ox = u0 * 2.0f - 1.0f, oy = u1 * 2.0f - 1.0f;
    float dx = 0.0f, dy = 0.0f;
    if (!(ox == 0.0f && oy == 0.0f)) {
        float r, th;
        const float kPi4 = kPi / 4.0f, kPi2 = kPi / 2.0f;
        if (std::fabs(ox) > std::fabs(oy)) { r = ox; th = kPi4 * (oy / ox); }
        else { r = oy; th = kPi2 - kPi4 * (ox / oy); }
        dx = r * std::cos(th);
        dy = r * std::sin(th);
    }
    float z = std::sqrt(std::fmax(0.0f, 1.0f - dx * dx - dy * dy));
    return {dx, dy, z};
}

// power_heuristic (core/sampling.rs:333-337)
inline float power_heuristic(float f, float g) { return (f * f) / (f * f + g * g); }

struct Tri { V p0, p1, p2; };

struct PtScene {
    void* scene;
    std::vector<Tri> tris;
    const uint32_t* mat;
    const float* albedo;
    const float* emission;
    std::vector<uint32_t> lights;   // emissive triangle ids
};

RGB albedo_of(const PtScene& s, uint32_t prim) {
    const float* a = s.albedo + 3 * s.mat[prim];
    return {a[0], a[1], a[2]};
}
RGB emission_of(const PtScene& s, uint32_t prim) {
    const float* a = s.emission + 3 * s.mat[prim];
    return {a[0], a[1], a[2]};
}

struct Isect {
    V p, perr, n, wo;
    uint32_t prim;
};

// Surface data of a triangle hit (triangle.rs:295-331): p = sum b_i p_i,
// p_error = gamma(7) * sum |b_i p_i|, n = normalize((p0-p2) x (p1-p2)).
Isect make_isect(const PtScene& s, const orc_hit& h, V d) {
    const Tri& t = s.tris[h.prim];
    float b1 = h.u, b2 = h.v, b0 = 1.0f - b1 - b2;
    Isect it;
    it.prim = h.prim;
    it.p = b0 * t.p0 + b1 * t.p1 + b2 * t.p2;
    V e = vabs(b0 * t.p0) + vabs(b1 * t.p1) + vabs(b2 * t.p2);
    it.perr = e * gamma(7);
    it.n = normalize(cross(t.p0 - t.p2, t.p1 - t.p2));
    it.wo = -d;
    return it;
}

// Lambertian BSDF in the frame of n (reflection/mod.rs:61-107, 108-129;
// lambertian_reflection.rs:22-28; BxDF::pdf mod.rs:357-359).
struct Bsdf {
    V ss, ts, ns, ng;
    RGB r;
    V to_local(V v) const { return {dot(v, ss), dot(v, ts), dot(v, ns)}; }
    V to_world(V v) const {
        return {ss.x * v.x + ts.x * v.y + ns.x * v.z, ss.y * v.x + ts.y * v.y + ns.y * v.z,
                ss.z * v.x + ts.z * v.y + ns.z * v.z};
    }
    RGB f(V wo_w, V wi_w) const {
        V wo = to_local(wo_w);
        if (wo.z == 0.0f) return {0, 0, 0};
        bool reflect = dot(wi_w, ng) * dot(wo_w, ng) > 0.0f;
        return reflect ? r * (1.0f / kPi) : RGB{0, 0, 0};
    }
    float pdf(V wo_w, V wi_w) const {
        V wo = to_local(wo_w), wi = to_local(wi_w);
        if (wo.z == 0.0f) return 0.0f;
        return (wo.z * wi.z > 0.0f) ? std::fabs(wi.z) * (1.0f / kPi) : 0.0f;
    }
    // BSDF::sample_f with one lobe (mod.rs:164-244), sampling in the local
    // frame (D16).
    RGB sample_f(V wo_w, float u0, float u1, V* wi_w, float* pdf_out) const {
        V wo = to_local(wo_w);
        *pdf_out = 0.0f;
        if (wo.z == 0.0f) return {0, 0, 0};
        V wi = cosine_sample_hemisphere(u0, u1);
        if (wo.z < 0.0f) wi.z = -wi.z;
        *pdf_out = (wo.z * wi.z > 0.0f) ? std::fabs(wi.z) * (1.0f / kPi) : 0.0f;
        if (*pdf_out == 0.0f) return {0, 0, 0};
        *wi_w = to_world(wi);
        return f(wo_w, *wi_w);
    }
};

Bsdf make_bsdf(const PtScene& s, const Isect& it) {
    Bsdf b;
    b.ns = it.n;
    b.ng = it.n;
    coordinate_system(it.n, &b.ss, &b.ts);
    b.r = albedo_of(s, it.prim);
    return b;
}

// Rays traced, and their binary-BVH node visits and primitive tests.
struct Counters {
    uint64_t ext = 0, shadow = 0;
    uint64_t ext_nodes = 0, ext_tris = 0, shadow_nodes = 0, shadow_tris = 0;
};

bool occluded(const PtScene& s, V o, V d, float tmax, Counters& c) {
    orc_ray r{{o.x, o.y, o.z}, 0.0f, {d.x, d.y, d.z}, tmax};
    uint8_t occ = 0;
    uint32_t nv = 0, nt = 0;
    orc_trace_any1_counted(s.scene, &r, &occ, &nv, &nt);
    ++c.shadow;
    c.shadow_nodes += nv;
    c.shadow_tris += nt;
    return occ != 0;
}

bool closest(const PtScene& s, V o, V d, orc_hit* h, Counters& c) {
    orc_ray r{{o.x, o.y, o.z}, 0.0f, {d.x, d.y, d.z}, INFINITY};
    uint32_t nv = 0, nt = 0;
    orc_trace_closest1_counted(s.scene, &r, h, &nv, &nt);
    ++c.ext;
    c.ext_nodes += nv;
    c.ext_tris += nt;
    return h->prim != 0xFFFFFFFFu;
}

// Triangle::area (triangle.rs:609-614)
float tri_area(const Tri& t) { return 0.5f * length(cross(t.p1 - t.p0, t.p2 - t.p0)); }

// estimate_direct for a diffuse area light on triangle `light`
// (integrator.rs:353-494 with D21, D25).
RGB estimate_direct(const PtScene& s, const Isect& it, const Bsdf& bsdf, uint32_t light, float ul0, float ul1,
                    float us0, float us1, Counters& cnt) {
    RGB ld{0, 0, 0};
    const Tri& lt = s.tris[light];
    RGB lemit = emission_of(s, light);
    float area = tri_area(lt);
    V nl = normalize(cross(lt.p1 - lt.p0, lt.p2 - lt.p0));   // triangle.rs:625
    // -- light sampling: uniform_sample_triangle (sampling.rs:264-267)
    float su0 = std::sqrt(ul0);
    float b0 = 1.0f - su0, b1 = ul1 * su0, b2 = 1.0f - b0 - b1;
    V pl = b0 * lt.p0 + b1 * lt.p1 + b2 * lt.p2;
    V pl_err = (vabs(b0 * lt.p0) + vabs(b1 * lt.p1) + vabs(b2 * lt.p2)) * gamma(6);
    V wi = pl - it.p;
    float light_pdf = 0.0f;
    RGB li{0, 0, 0};
    if (dot(wi, wi) != 0.0f) {
        float d2 = dot(wi, wi);
        wi = normalize(wi);
        light_pdf = (1.0f / area) * d2 / std::fabs(dot(nl, -wi));
        if (std::isinf(light_pdf)) light_pdf = 0.0f;
        li = dot(nl, -wi) > 0.0f ? lemit : RGB{0, 0, 0};
    }
    if (light_pdf > 0.0f && !is_black(li)) {
        RGB f = bsdf.f(it.wo, wi) * std::fabs(dot(wi, bsdf.ns));
        float scat_pdf = bsdf.pdf(it.wo, wi);
        if (!is_black(f)) {
            // VisibilityTester::unoccluded via spawn_ray_to (interaction.rs:60-72)
            V o = offset_ray_origin(it.p, it.perr, it.n, pl - it.p);
            V tgt = offset_ray_origin(pl, pl_err, nl, o - pl);
            if (!occluded(s, o, tgt - o, 1.0f - 0.0001f, cnt)) {
                float w = power_heuristic(light_pdf, scat_pdf);
                ld = ld + f * li * (w / light_pdf);
            }
        }
    }
    // -- BSDF sampling with MIS
    V wb;
    float scat_pdf = 0.0f;
    RGB f = bsdf.sample_f(it.wo, us0, us1, &wb, &scat_pdf);
    if (!is_black(f) && scat_pdf > 0.0f) {
        f = f * std::fabs(dot(wb, bsdf.ns));
        V o = offset_ray_origin(it.p, it.perr, it.n, wb);   // spawn_ray (interaction.rs:33-43)
        // pdf_li = Shape::pdf_with_point: hit the light's own shape
        orc_ray r{{o.x, o.y, o.z}, 0.0f, {wb.x, wb.y, wb.z}, INFINITY};
        float tl[4];
        if (!orc_triangle_intersect(&lt.p0.x, &lt.p1.x, &lt.p2.x, &r, 1, tl)) return ld;
        V pli = tl[1] * lt.p0 + tl[2] * lt.p1 + tl[3] * lt.p2;
        V dd = pli - it.p;
        float lp = dot(dd, dd) / (std::fabs(dot(nl, wb)) * area);
        if (std::isinf(lp)) lp = 0.0f;
        if (lp == 0.0f) return ld;
        float w = power_heuristic(scat_pdf, lp);
        orc_hit h;
        if (closest(s, o, wb, &h, cnt) && h.prim == light) {
            RGB le = dot(nl, -wb) > 0.0f ? lemit : RGB{0, 0, 0};
            ld = ld + f * le * (w / scat_pdf);
        }
    }
    return ld;
}

// PBR-book PathIntegrator::Li with this file's estimate_direct.
RGB li(const PtScene& s, V o, V d, Rng& rng, uint32_t max_depth, uint32_t rr_depth, Counters& cnt) {
    RGB L{0, 0, 0}, beta{1, 1, 1};
    for (uint32_t bounces = 0;; ++bounces) {
        orc_hit h;
        bool found = closest(s, o, d, &h, cnt);
        if (bounces == 0 && found) {
            Isect it = make_isect(s, h, d);
            if (dot(it.n, it.wo) > 0.0f) L = L + beta * emission_of(s, h.prim);   // one-sided Le
        }
        if (!found || bounces >= max_depth) break;
        Isect it = make_isect(s, h, d);
        Bsdf bsdf = make_bsdf(s, it);
        // uniform_sample_one_light (integrator.rs:321-350)
        float ul = rng.uniform_float();
        float u_l0 = rng.uniform_float(), u_l1 = rng.uniform_float();
        float u_s0 = rng.uniform_float(), u_s1 = rng.uniform_float();
        if (!s.lights.empty()) {
            size_t nl = s.lights.size();
            size_t k = (size_t)(ul * (float)nl);
            if (k > nl - 1) k = nl - 1;
            RGB ld = estimate_direct(s, it, bsdf, s.lights[k], u_l0, u_l1, u_s0, u_s1, cnt);
            L = L + beta * ld * (float)nl;
        }
        // continuation
        float u0 = rng.uniform_float(), u1 = rng.uniform_float();
        V wi;
        float pdf;
        RGB f = bsdf.sample_f(it.wo, u0, u1, &wi, &pdf);
        float urr = rng.uniform_float();
        if (is_black(f) || pdf == 0.0f) break;
        beta = beta * f * (std::fabs(dot(wi, bsdf.ns)) / pdf);
        o = offset_ray_origin(it.p, it.perr, it.n, wi);
        d = wi;
        if (bounces >= rr_depth) {   // Russian roulette from bounce rr_depth on
            float q = std::fmax(0.05f, 1.0f - max_comp(beta));
            if (urr < q) break;
            beta = beta * (1.0f / (1.0f - q));
        }
        // The loop would trace the next segment only to stop at max_depth, and
        // with Lambertian surfaces that intersection adds no radiance (emission
        // is added on the camera segment only), so it is not traced.
        if (bounces + 1 >= max_depth) break;
    }
    return L;
}

}  // namespace
}  // namespace orc

using namespace orc;

// FilmTile::add_sample (film.rs:288-333) with D20 repaired (footprint upper
// corner floor(p + radius) + 1, both loops run): the sample's L times the
// table weight of each pixel within the filter radius, and the weight.
static void film_splat(float* sums, float* wsum, uint32_t width, uint32_t height, const float* table, float rx,
                       float ry, float fx, float fy, const RGB& L) {
    const float dx = fx - 0.5f, dy = fy - 0.5f;
    const float irx = 1.0f / rx, iry = 1.0f / ry;
    int x0 = (int)std::ceil(dx - rx), y0 = (int)std::ceil(dy - ry);
    int x1 = (int)std::floor(dx + rx) + 1, y1 = (int)std::floor(dy + ry) + 1;
    x0 = std::max(x0, 0); y0 = std::max(y0, 0);
    x1 = std::min(x1, (int)width); y1 = std::min(y1, (int)height);
    for (int y = y0; y < y1; ++y) {
        int ify = std::min((int)std::floor(std::fabs(((float)y - dy) * iry * 16.0f)), 15);
        for (int x = x0; x < x1; ++x) {
            int ifx = std::min((int)std::floor(std::fabs(((float)x - dx) * irx * 16.0f)), 15);
            float w = table[ify * 16 + ifx];
            size_t p = (size_t)y * width + x;
            sums[3 * p] += L.r * w;
            sums[3 * p + 1] += L.g * w;
            sums[3 * p + 2] += L.b * w;
            wsum[p] += w;
        }
    }
}

extern "C" int orc_render_pt_filtered(void* scene, const float* verts, const uint32_t* idx, uint32_t nt,
                                      const uint32_t* prim_material, const float* albedo, const float* emission,
                                      const float eye[3], float fov_deg, uint32_t width, uint32_t height,
                                      uint32_t spp, uint32_t max_depth, uint32_t rr_depth, uint64_t seed,
                                      const float* table, float rx, float ry, int nthreads, float* rgb_out,
                                      uint64_t* ray_counts, const float* camera_to_world) {
    uint32_t ns = (uint32_t)std::lround(std::sqrt((double)spp));
    if (ns * ns != spp || width == 0 || height == 0 || !(rx > 0.0f) || !(ry > 0.0f)) return -1;
    PtScene s;
    s.scene = scene;
    s.mat = prim_material;
    s.albedo = albedo;
    s.emission = emission;
    s.tris.resize(nt);
    for (uint32_t i = 0; i < nt; ++i) {
        const float* a = verts + 3 * idx[3 * i];
        const float* b = verts + 3 * idx[3 * i + 1];
        const float* c = verts + 3 * idx[3 * i + 2];
        s.tris[i] = {{a[0], a[1], a[2]}, {b[0], b[1], b[2]}, {c[0], c[1], c[2]}};
        const float* e = emission + 3 * prim_material[i];
        if (e[0] > 0.0f || e[1] > 0.0f || e[2] > 0.0f) s.lights.push_back(i);
    }
    const float th = std::tan(0.5f * fov_deg * kPi / 180.0f);
    const float aspect = (float)width / (float)height;
    if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
    const size_t npix = (size_t)width * height;
    std::vector<std::vector<float>> sums(nthreads, std::vector<float>(3 * npix, 0.0f)),
        wsums(nthreads, std::vector<float>(npix, 0.0f));
    std::atomic<uint32_t> next_row{0};
    std::atomic<uint64_t> ext{0}, sh{0};
    auto worker = [&](int tid) {
        Counters cnt;
        for (;;) {
            uint32_t py = next_row.fetch_add(1);
            if (py >= height) break;
            for (uint32_t px = 0; px < width; ++px) {
                Rng rng((seed << 32) ^ ((uint64_t)py * width + px));
                for (uint32_t k = 0; k < spp; ++k) {
                    float jx = rng.uniform_float(), jy = rng.uniform_float();
                    float fx = (float)px + ((float)(k % ns) + jx) / (float)ns;
                    float fy = (float)py + ((float)(k / ns) + jy) / (float)ns;
                    float sx = (fx / (float)width * 2.0f - 1.0f) * th * aspect;
                    float sy = (1.0f - fy / (float)height * 2.0f) * th;
                    V d = normalize(V{sx, sy, 1.0f});
                    if (camera_to_world) {   // camera-space direction to world space
                        const float* m = camera_to_world;
                        d = V{m[0] * d.x + m[1] * d.y + m[2] * d.z, m[3] * d.x + m[4] * d.y + m[5] * d.z,
                              m[6] * d.x + m[7] * d.y + m[8] * d.z};
                    }
                    RGB L = li(s, V{eye[0], eye[1], eye[2]}, d, rng, max_depth, rr_depth, cnt);
                    if (std::isnan(L.r) || std::isnan(L.g) || std::isnan(L.b) || luminance(L) < -1e-5f ||
                        std::isinf(luminance(L)))
                        L = {0, 0, 0};
                    film_splat(sums[tid].data(), wsums[tid].data(), width, height, table, rx, ry, fx, fy, L);
                }
            }
        }
        ext += cnt.ext;
        sh += cnt.shadow;
    };
    std::vector<std::thread> th_;
    for (int i = 0; i < nthreads; ++i) th_.emplace_back(worker, i);
    for (auto& t : th_) t.join();
    // merge the threads' films, then Film::write_image's division (film.rs:187-226)
    for (size_t p = 0; p < npix; ++p) {
        float w = 0.0f, c[3] = {0.0f, 0.0f, 0.0f};
        for (int t = 0; t < nthreads; ++t) {
            w += wsums[t][p];
            for (int k = 0; k < 3; ++k) c[k] += sums[t][3 * p + k];
        }
        for (int k = 0; k < 3; ++k) rgb_out[3 * p + k] = w != 0.0f ? c[k] * (1.0f / w) : 0.0f;
    }
    if (ray_counts) { ray_counts[0] = ext.load(); ray_counts[1] = sh.load(); }
    return 0;
}

extern "C" int orc_render_pt(void* scene, const float* verts, const uint32_t* idx, uint32_t nt,
                             const uint32_t* prim_material, const float* albedo, const float* emission,
                             const float eye[3], float fov_deg, uint32_t width, uint32_t height, uint32_t spp,
                             uint32_t max_depth, uint32_t rr_depth, uint64_t seed, uint32_t x0, uint32_t y0,
                             uint32_t x1, uint32_t y1, int nthreads, float* rgb_out, uint64_t* ray_counts) {
    uint32_t ns = (uint32_t)std::lround(std::sqrt((double)spp));
    if (ns * ns != spp || x1 <= x0 || y1 <= y0 || x1 > width || y1 > height) return -1;
    PtScene s;
    s.scene = scene;
    s.mat = prim_material;
    s.albedo = albedo;
    s.emission = emission;
    s.tris.resize(nt);
    for (uint32_t i = 0; i < nt; ++i) {
        const float* a = verts + 3 * idx[3 * i];
        const float* b = verts + 3 * idx[3 * i + 1];
        const float* c = verts + 3 * idx[3 * i + 2];
        s.tris[i] = {{a[0], a[1], a[2]}, {b[0], b[1], b[2]}, {c[0], c[1], c[2]}};
        const float* e = emission + 3 * prim_material[i];
        if (e[0] > 0.0f || e[1] > 0.0f || e[2] > 0.0f) s.lights.push_back(i);
    }
    const float th = std::tan(0.5f * fov_deg * kPi / 180.0f);
    const float aspect = (float)width / (float)height;
    const uint32_t w = x1 - x0, hgt = y1 - y0;
    if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
    std::atomic<uint32_t> next_row{0};
    std::atomic<uint64_t> ext{0}, sh{0}, ext_nodes{0}, ext_tris{0}, sh_nodes{0}, sh_tris{0};
    auto worker = [&]() {
        Counters cnt;
        for (;;) {
            uint32_t row = next_row.fetch_add(1);
            if (row >= hgt) break;
            uint32_t py = y0 + row;
            for (uint32_t px = x0; px < x1; ++px) {
                Rng rng((seed << 32) ^ ((uint64_t)py * width + px));
                RGB sum{0, 0, 0};
                for (uint32_t k = 0; k < spp; ++k) {
                    // stratified pixel sample (ns x ns jittered strata)
                    float jx = rng.uniform_float(), jy = rng.uniform_float();
                    float fx = (float)px + ((float)(k % ns) + jx) / (float)ns;
                    float fy = (float)py + ((float)(k / ns) + jy) / (float)ns;
                    float sx = (fx / (float)width * 2.0f - 1.0f) * th * aspect;
                    float sy = (1.0f - fy / (float)height * 2.0f) * th;
                    V d = normalize(V{sx, sy, 1.0f});
                    RGB L = li(s, V{eye[0], eye[1], eye[2]}, d, rng, max_depth, rr_depth, cnt);
                    // radiance guard (integrator.rs:113-122)
                    if (std::isnan(L.r) || std::isnan(L.g) || std::isnan(L.b) || luminance(L) < -1e-5f ||
                        std::isinf(luminance(L)))
                        L = {0, 0, 0};
                    sum = sum + L;
                }
                float* out = rgb_out + 3 * ((size_t)row * w + (px - x0));
                out[0] = sum.r / (float)spp;
                out[1] = sum.g / (float)spp;
                out[2] = sum.b / (float)spp;
            }
        }
        ext += cnt.ext;
        sh += cnt.shadow;
        ext_nodes += cnt.ext_nodes;
        ext_tris += cnt.ext_tris;
        sh_nodes += cnt.shadow_nodes;
        sh_tris += cnt.shadow_tris;
    };
    std::vector<std::thread> th_;
    for (int i = 0; i < nthreads; ++i) th_.emplace_back(worker);
    for (auto& t : th_) t.join();
    if (ray_counts) {
        ray_counts[0] = ext.load(); ray_counts[1] = sh.load();
        ray_counts[2] = ext_nodes.load(); ray_counts[3] = ext_tris.load();
        ray_counts[4] = sh_nodes.load(); ray_counts[5] = sh_tris.load();
    }
    return 0;
}
