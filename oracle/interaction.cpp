// Oracle (test infrastructure): the SurfaceInteraction that
// Triangle::intersect builds after its hit test, restated from
// shapes/triangle.rs:264-415, core/interaction.rs:262-339 and
// core/geometry/vector3.rs (cross in f64 67-83, normalize 85-95,
// coordinate_system 520-537), normal3.rs face_forward (45-50).
// Repairs: D14 (uv determinant duv02.x*duv12.y - duv02.y*duv12.x) and D27
// (SurfaceInteraction::new stores Shading::default(); here the shading frame
// starts as the geometric one, as in pbrt).  Built with -ffp-contract=off.
#include <cmath>
#include <cstring>

#include "oracle.h"

namespace {

struct V {
    float x, y, z;
};
V add(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V sub(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V mul(float s, V a) { return {s * a.x, s * a.y, s * a.z}; }
V neg(V a) { return {-a.x, -a.y, -a.z}; }
float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
float len2(V a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
V cross(V a, V b) {   // vector3.rs:67-83
    double ax = a.x, ay = a.y, az = a.z, bx = b.x, by = b.y, bz = b.z;
    return {(float)((ay * bz) - (az * by)), (float)((az * bx) - (ax * bz)), (float)((ax * by) - (ay * bx))};
}
V normalize(V a) {   // vector3.rs:85-95
    float inv = 1.0f / std::sqrt(len2(a));
    return {a.x * inv, a.y * inv, a.z * inv};
}
void coordinate_system(V v1, V& v2, V& v3) {   // vector3.rs:520-537
    if (std::fabs(v1.x) > std::fabs(v1.y)) {
        float l = std::sqrt(v1.x * v1.x + v1.z * v1.z);
        v2 = {-v1.z / l, 0.0f, v1.x / l};
    } else {
        float l = std::sqrt(v1.y * v1.y + v1.z * v1.z);
        v2 = {0.0f, v1.z / l, -v1.y / l};
    }
    v3 = cross(v1, v2);
}
V at(const float* a, int i) { return {a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }
V interp(float b0, float b1, float b2, V a, V b, V c) { return add(add(mul(b0, a), mul(b1, b)), mul(b2, c)); }
void put(float* d, V v) { d[0] = v.x; d[1] = v.y; d[2] = v.z; }

constexpr float kEps = 0x1p-24f;   // MACHINE_EPSILON (pbrt.rs:23)
float gamma(int n) { return ((float)n * kEps) / (1.0f - (float)n * kEps); }   // pbrt.rs:129-131

}  // namespace

extern "C" int orc_surface_interaction(const float* p, const float* nrm, const float* tan, const float* uvs,
                                       int reverse, const orc_ray* r, orc_si* out) {
    std::memset(out, 0, sizeof *out);
    float hit[4];
    if (!orc_triangle_intersect(p, p + 3, p + 6, r, 1, hit)) return 0;
    const float t = hit[0], b0 = hit[1], b1 = hit[2], b2 = hit[3];
    const V p0 = at(p, 0), p1 = at(p, 1), p2 = at(p, 2);
    // get_uvs (triangle.rs:96-112)
    float uv[3][2] = {{0.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 1.0f}};
    if (uvs)
        for (int k = 0; k < 3; ++k) { uv[k][0] = uvs[2 * k]; uv[k][1] = uvs[2 * k + 1]; }
    // triangle.rs:264-292
    const float duv02x = uv[0][0] - uv[2][0], duv02y = uv[0][1] - uv[2][1];
    const float duv12x = uv[1][0] - uv[2][0], duv12y = uv[1][1] - uv[2][1];
    const V dp02 = sub(p0, p2), dp12 = sub(p1, p2);
    const float det = duv02x * duv12y - duv02y * duv12x;
    const bool degenerate_uv = std::fabs(det) < 1e-8f;
    V dpdu{0, 0, 0}, dpdv{0, 0, 0};
    if (!degenerate_uv) {
        const float invdet = 1.0f / det;
        dpdu = mul(invdet, sub(mul(duv12y, dp02), mul(duv02y, dp12)));
        dpdv = mul(invdet, add(mul(-duv12x, dp02), mul(duv02x, dp12)));
    }
    if (degenerate_uv || len2(cross(dpdu, dpdv)) == 0.0f) {
        const V ng = cross(sub(p2, p0), sub(p1, p0));
        if (len2(ng) == 0.0f) return 0;
        coordinate_system(normalize(ng), dpdu, dpdv);
    }
    // triangle.rs:295-305
    const float g7 = gamma(7);
    const V perr{g7 * (std::fabs(b0 * p0.x) + std::fabs(b1 * p1.x) + std::fabs(b2 * p2.x)),
                 g7 * (std::fabs(b0 * p0.y) + std::fabs(b1 * p1.y) + std::fabs(b2 * p2.y)),
                 g7 * (std::fabs(b0 * p0.z) + std::fabs(b1 * p1.z) + std::fabs(b2 * p2.z))};
    const V phit = interp(b0, b1, b2, p0, p1, p2);
    out->uv[0] = b0 * uv[0][0] + b1 * uv[1][0] + b2 * uv[2][0];
    out->uv[1] = b0 * uv[0][1] + b1 * uv[1][1] + b2 * uv[2][1];
    // normal override (triangle.rs:322-331)
    V n = normalize(cross(dp02, dp12));
    if (reverse) n = neg(n);
    V sn = n, sdpdu = dpdu, sdpdv = dpdv, sdndu{0, 0, 0}, sdndv{0, 0, 0};
    if (nrm || tan) {
        // triangle.rs:333-414
        V ns = n;
        if (nrm) {
            V nn = interp(b0, b1, b2, at(nrm, 0), at(nrm, 1), at(nrm, 2));
            if (len2(nn) > 0.0f) ns = normalize(nn);
        }
        V ss = normalize(dpdu);
        if (tan) {
            V s = interp(b0, b1, b2, at(tan, 0), at(tan, 1), at(tan, 2));
            if (len2(s) > 0.0f) ss = normalize(s);
        }
        V ts = cross(ss, ns);
        if (len2(ts) > 0.0f) {
            ts = normalize(ts);
            ss = cross(ts, ns);
        } else {
            coordinate_system(ns, ss, ts);
        }
        V dndu{0, 0, 0}, dndv{0, 0, 0};
        if (nrm) {
            const V n0 = at(nrm, 0), n1 = at(nrm, 1), n2 = at(nrm, 2);
            const V dn1 = sub(n0, n2), dn2 = sub(n1, n2);
            const float det2 = duv02x * duv12y - duv02y * duv12x;
            if (std::fabs(det2) < 1e-8f) {
                const V dn = cross(sub(n2, n0), sub(n1, n0));
                if (len2(dn) != 0.0f) coordinate_system(dn, dndu, dndv);
            } else {
                const float inv = 1.0f / det2;
                dndu = mul(inv, sub(mul(duv12y, dn1), mul(duv02y, dn2)));
                dndv = mul(inv, add(mul(-duv12x, dn1), mul(duv02x, dn2)));
            }
        }
        if (reverse) ts = neg(ts);
        // set_shading_geometry(ss, ts, dndu, dndv, true) (interaction.rs:318-339)
        sn = normalize(cross(ss, ts));
        if (dot(n, sn) < 0.0f) n = neg(n);
        sdpdu = ss; sdpdv = ts; sdndu = dndu; sdndv = dndv;
    }
    out->kind = 1;
    out->t = t;
    put(out->p, phit); put(out->p_error, perr); put(out->n, n);
    put(out->dpdu, dpdu); put(out->dpdv, dpdv);
    put(out->shading_n, sn); put(out->shading_dpdu, sdpdu); put(out->shading_dpdv, sdpdv);
    put(out->shading_dndu, sdndu); put(out->shading_dndv, sdndv);
    put(out->wo, {-r->d[0], -r->d[1], -r->d[2]});
    return 1;
}
