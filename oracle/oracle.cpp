// CPU oracle: scalar restatement of rs_illume's ray-query hot path.
// TEST INFRASTRUCTURE ONLY (see oracle.h).  Built with -ffp-contract=off
// -fno-fast-math so every float expression rounds exactly as the Rust source
// (Rust never fuses multiply-add).  All citations are paths inside the
// rs_illume repository.
#include "oracle.h"
#include "oracle_common.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace orc {

// ---------------------------------------------------------------- geometry
struct V3 { float x, y, z; };
static inline float comp(const V3& v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
static inline V3 sub(const V3& a, const V3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
// Vector3::cross evaluates in f64 and rounds to f32 (geometry/vector3.rs:67-82)
static inline V3 cross64(const V3& a, const V3& b) {
    double ax = a.x, ay = a.y, az = a.z, bx = b.x, by = b.y, bz = b.z;
    return {(float)((ay * bz) - (az * by)), (float)((az * bx) - (ax * bz)),
            (float)((ax * by) - (ay * bx))};
}
// Vector3::length_squared (vector3.rs:43-48)
static inline float length_sq(const V3& v) { return v.x * v.x + v.y * v.y + v.z * v.z; }

// Bounds3<f32> with Default min=MAX, max=MIN (geometry/bounds3.rs:357-368)
struct B3 {
    V3 mn{std::numeric_limits<float>::max(), std::numeric_limits<float>::max(),
          std::numeric_limits<float>::max()};
    V3 mx{-std::numeric_limits<float>::max(), -std::numeric_limits<float>::max(),
          -std::numeric_limits<float>::max()};
};
// Point3::min / max (geometry/point3.rs:70-92)
static inline V3 pmin(const V3& a, const V3& b) {
    return {a.x < b.x ? a.x : b.x, a.y < b.y ? a.y : b.y, a.z < b.z ? a.z : b.z};
}
static inline V3 pmax(const V3& a, const V3& b) {
    return {a.x > b.x ? a.x : b.x, a.y > b.y ? a.y : b.y, a.z > b.z ? a.z : b.z};
}
// Bounding3::union (bounds3.rs:37-47)
static inline B3 bunion(const B3& a, const B3& b) { B3 r; r.mn = pmin(a.mn, b.mn); r.mx = pmax(a.mx, b.mx); return r; }
static inline B3 bunion_pt(const B3& a, const V3& p) { B3 r; r.mn = pmin(a.mn, p); r.mx = pmax(a.mx, p); return r; }
// Bounding3::maximum_extent (bounds3.rs:53-56)
static inline int maximum_extent(const B3& b) {
    V3 d = sub(b.mx, b.mn);
    if (d.x > d.y && d.x > d.z) return 0;
    if (d.y > d.z) return 1;
    return 2;
}
// Bounding3::surface_area (bounds3.rs:59-62)
static inline float surface_area(const B3& b) {
    V3 d = sub(b.mx, b.mn);
    return 2.0f * (d.x * d.y + d.x * d.z + d.y * d.z);
}
// Bounds3::centroid (bounds3.rs:238-242)
static inline V3 centroid(const B3& b) {
    return {b.mn.x * 0.5f + b.mx.x * 0.5f, b.mn.y * 0.5f + b.mx.y * 0.5f, b.mn.z * 0.5f + b.mx.z * 0.5f};
}
// Bounds3::offset (bounds3.rs:178-193)
static inline V3 offset(const B3& b, const V3& p) {
    V3 o = sub(p, b.mn);
    if (b.mx.x > b.mn.x) o.x /= b.mx.x - b.mn.x;
    if (b.mx.y > b.mn.y) o.y /= b.mx.y - b.mn.y;
    if (b.mx.z > b.mn.z) o.z /= b.mx.z - b.mn.z;
    return o;
}

struct Ray { V3 o, d; float t_max; };

// D26: a slab distance (bound - o) * inv_dir is NaN exactly when the ray lies
// in that bounding plane with a zero direction component (0 * inf).  The
// reference's comparisons then reject the box, although the ray touches it,
// and its watertight triangle test accepts hits on an edge lying in that
// plane, so such hits are lost.  The repair treats the slab as unconstrained.
static inline void unconstrain_nan(float* lo, float* hi) {
    if (std::isnan(*lo)) *lo = -std::numeric_limits<float>::infinity();
    if (std::isnan(*hi)) *hi = std::numeric_limits<float>::infinity();
}

// Bounding3::intersect_p with precomputed inv_dir (bounds3.rs:284-318), D26
static inline bool box_intersect_p(const orc_bvh_node& n, const Ray& ray, const V3& inv_dir,
                                   const int dir_is_neg[3]) {
    const float* mm[2] = {n.bmin, n.bmax};
    const float robust = 1.0f + 2.0f * gamma(3);
    float t_min = (mm[dir_is_neg[0]][0] - ray.o.x) * inv_dir.x;
    float t_max = (mm[1 - dir_is_neg[0]][0] - ray.o.x) * inv_dir.x;
    float ty_min = (mm[dir_is_neg[1]][1] - ray.o.y) * inv_dir.y;
    float ty_max = (mm[1 - dir_is_neg[1]][1] - ray.o.y) * inv_dir.y;
    unconstrain_nan(&t_min, &t_max);
    unconstrain_nan(&ty_min, &ty_max);
    t_max *= robust;
    ty_max *= robust;
    if (t_min > ty_max || ty_min > t_max) return false;
    if (ty_min > t_min) t_min = ty_min;
    if (ty_max < t_max) t_max = ty_max;
    float tz_min = (mm[dir_is_neg[2]][2] - ray.o.z) * inv_dir.z;
    float tz_max = (mm[1 - dir_is_neg[2]][2] - ray.o.z) * inv_dir.z;
    unconstrain_nan(&tz_min, &tz_max);
    tz_max *= robust;
    if (t_min > tz_max || tz_min > t_max) return false;
    if (tz_min > t_min) t_min = tz_min;
    if (tz_max < t_max) t_max = tz_max;
    return (t_min < ray.t_max) && (t_max > 0.0f);
}

// ---------------------------------------------------------------- triangle.rs
// Watertight ray-triangle test, Triangle::intersect (triangle.rs:142-262,
// 281-289) and Triangle::intersect_p (triangle.rs:421-541).  `closest`
// selects intersect(), which additionally rejects triangles whose geometric
// normal (p2-p0)x(p1-p0) has zero squared length (triangle.rs:281-289; D14
// makes the uv-determinant branch unreachable, so this is the check that
// runs).  D11 (3-element permute) and D12 (true max_component) repaired.
static bool triangle_test(const V3& p0, const V3& p1, const V3& p2, const Ray& ray,
                          bool closest, float* t_out, float* b_out) {
    // translate (157-159)
    V3 p0t = sub(p0, ray.o), p1t = sub(p1, ray.o), p2t = sub(p2, ray.o);
    // permute (162-174); max_dimension (vector3.rs:140-150)
    V3 ad{std::fabs(ray.d.x), std::fabs(ray.d.y), std::fabs(ray.d.z)};
    int kz = (ad.x > ad.y) ? (ad.x > ad.z ? 0 : 2) : (ad.y > ad.z ? 1 : 2);
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    V3 d{comp(ray.d, kx), comp(ray.d, ky), comp(ray.d, kz)};
    p0t = {comp(p0t, kx), comp(p0t, ky), comp(p0t, kz)};
    p1t = {comp(p1t, kx), comp(p1t, ky), comp(p1t, kz)};
    p2t = {comp(p2t, kx), comp(p2t, ky), comp(p2t, kz)};
    // shear (177-185)
    float sx = -d.x / d.z, sy = -d.y / d.z, sz = 1.0f / d.z;
    p0t.x += sx * p0t.z; p0t.y += sy * p0t.z;
    p1t.x += sx * p1t.z; p1t.y += sy * p1t.z;
    p2t.x += sx * p2t.z; p2t.y += sy * p2t.z;
    // edge functions (188-190)
    float e0 = p1t.x * p2t.y - p1t.y * p2t.x;
    float e1 = p2t.x * p0t.y - p2t.y * p0t.x;
    float e2 = p0t.x * p1t.y - p0t.y * p1t.x;
    // f64 fallback at edges (193-204)
    if (e0 == 0.0f || e1 == 0.0f || e2 == 0.0f) {
        double p2txp1ty = (double)p2t.x * (double)p1t.y;
        double p2typ1tx = (double)p2t.y * (double)p1t.x;
        e0 = (float)(p2typ1tx - p2txp1ty);
        double p0txp2ty = (double)p0t.x * (double)p2t.y;
        double p0typ2tx = (double)p0t.y * (double)p2t.x;
        e1 = (float)(p0typ2tx - p0txp2ty);
        double p1txp0ty = (double)p1t.x * (double)p0t.y;
        double p1typ0tx = (double)p1t.y * (double)p0t.x;
        e2 = (float)(p1typ0tx - p1txp0ty);
    }
    // edge and determinant tests (207-215)
    if ((e0 < 0.0f || e1 < 0.0f || e2 < 0.0f) && (e0 > 0.0f || e1 > 0.0f || e2 > 0.0f)) return false;
    float det = e0 + e1 + e2;
    if (det == 0.0f) return false;
    // scaled hit distance and range test (218-229)
    p0t.z *= sz; p1t.z *= sz; p2t.z *= sz;
    float t_scaled = e0 * p0t.z + e1 * p1t.z + e2 * p2t.z;
    if (det < 0.0f && (t_scaled >= 0.0f || t_scaled < ray.t_max * det)) return false;
    else if (det > 0.0f && (t_scaled <= 0.0f || t_scaled > ray.t_max * det)) return false;
    // barycentrics and t (232-236)
    float inv_det = 1.0f / det;
    float b0 = e0 * inv_det, b1 = e1 * inv_det, b2 = e2 * inv_det;
    float t = t_scaled * inv_det;
    // conservative t > 0 (241-262), max_component repaired (D12)
    auto max3 = [](float a, float b, float c) { float m = a > b ? a : b; return m > c ? m : c; };
    float max_zt = max3(std::fabs(p0t.z), std::fabs(p1t.z), std::fabs(p2t.z));
    float delta_z = gamma(3) * max_zt;
    float max_xt = max3(std::fabs(p0t.x), std::fabs(p1t.x), std::fabs(p2t.x));
    float max_yt = max3(std::fabs(p0t.y), std::fabs(p1t.y), std::fabs(p2t.y));
    float delta_x = gamma(5) * (max_xt + max_zt);
    float delta_y = gamma(5) * (max_yt + max_zt);
    float delta_e = 2.0f * (gamma(2) * max_xt * max_yt + delta_y * max_xt + delta_x * max_yt);
    float max_e = max3(std::fabs(e0), std::fabs(e1), std::fabs(e2));
    float delta_t = 3.0f * (gamma(3) * max_e * max_zt + delta_e * max_zt + delta_z * max_e) *
                    std::fabs(inv_det);
    if (t <= delta_t) return false;
    if (closest) {
        // degenerate-triangle rejection (281-289)
        V3 ng = cross64(sub(p2, p0), sub(p1, p0));
        if (length_sq(ng) == 0.0f) return false;
    }
    *t_out = t;
    b_out[0] = b0; b_out[1] = b1; b_out[2] = b2;
    return true;
}

// ---------------------------------------------------------------- efloat.rs
// EFloat interval arithmetic (core/efloat.rs:5-257).  D23: the scalar
// operators (Add/Sub/Mul/Div<f32>, Mul<EFloat> for f32, efloat.rs:123-195)
// build EFloat::new(rhs, rhs), i.e. an error equal to the value itself, which
// turns `* -0.5` into an interval with low > high and trips check(); repaired
// to an exact constant EFloat::new(rhs, 0.0) as pbrt-v3 does.
struct EF {
    float v, low, high;
};
static inline EF ef_new(float v, float err) {        // efloat.rs:12-29
    if (err == 0.0f) return {v, v, v};
    return {v, next_float_down(v - err), next_float_up(v + err)};
}
static inline EF ef_add(EF a, EF b) {                 // efloat.rs:108-118
    return {a.v + b.v, next_float_down(a.low + b.low), next_float_up(a.high + b.high)};
}
static inline EF ef_sub(EF a, EF b) {                 // efloat.rs:127-137
    return {a.v - b.v, next_float_down(a.low - b.low), next_float_up(a.high - b.high)};
}
static inline EF ef_mul(EF a, EF b) {                 // efloat.rs:146-162
    float p0 = a.low * b.low, p1 = a.high * b.low, p2 = a.low * b.high, p3 = a.high * b.high;
    float lo = std::fmin(std::fmin(std::fmin(p0, p1), p2), p3);
    float hi = std::fmax(std::fmax(std::fmax(p0, p1), p2), p3);
    return {a.v * b.v, next_float_down(lo), next_float_up(hi)};
}
static inline EF ef_div(EF a, EF b) {                 // efloat.rs:180-205
    if (b.low < 0.0f && b.high > 0.0f)
        return {a.v / b.v, -std::numeric_limits<float>::infinity(), std::numeric_limits<float>::infinity()};
    float d0 = a.low / b.low, d1 = a.high / b.low, d2 = a.low / b.high, d3 = a.high / b.high;
    float lo = std::fmin(std::fmin(std::fmin(d0, d1), d2), d3);
    float hi = std::fmax(std::fmax(std::fmax(d0, d1), d2), d3);
    return {a.v / b.v, next_float_down(lo), next_float_up(hi)};
}
// quadratic (efloat.rs:232-257)
static bool ef_quadratic(EF a, EF b, EF c, EF* t0, EF* t1) {
    double discrim = (double)b.v * (double)b.v - 4.0 * (double)a.v * (double)c.v;
    if (discrim < 0.0) return false;
    double root = std::sqrt(discrim);
    EF froot = ef_new((float)root, kMachineEps * (float)root);
    EF q = (b.v < 0.0f) ? ef_mul(ef_sub(b, froot), ef_new(-0.5f, 0.0f))
                        : ef_mul(ef_add(b, froot), ef_new(-0.5f, 0.0f));
    *t0 = ef_div(q, a);
    *t1 = ef_div(c, q);
    if (t0->v > t1->v) { EF s = *t0; *t0 = *t1; *t1 = s; }
    return true;
}

// ---------------------------------------------------------------- sphere.rs
// A sphere or another quadric.  z_min / z_max bound the object box in z for
// every kind (disk: both = height; cone: 0 and height).
struct Sphere {
    float m[16], mi[16];   // object_to_world, world_to_object (row-major)
    float radius, z_min, z_max, theta_min, theta_max, phi_max;
    float inner_radius, height;
    V3 p1, p2;             // hyperboloid: the swept segment (after the p2.z == 0 swap)
    float ah, ch;          // hyperboloid: ah (x^2 + y^2) - ch z^2 = 1
    int kind;              // 0 sphere, 1 disk, 2 cylinder, 3 cone, 4 paraboloid, 5 hyperboloid, 6 curve
    bool reverse;
    // curve segment: the curve's control points and end widths, the segment's
    // u range, the type and the ribbon normals (CurveCommon, curve.rs:20-61)
    V3 ccp[4];
    float width[2], u_min, u_max;
    int ctype;
    V3 n[2];
    float normal_angle, inv_sin_normal_angle;
};

static inline float lerpf(float t, float a, float b) { return a * (1.0f - t) + b * t; }   // pbrt.rs:41-47
static inline V3 lerp3(float t, const V3& a, const V3& b) {
    return {lerpf(t, a.x, b.x), lerpf(t, a.y, b.y), lerpf(t, a.z, b.z)};
}
// blossom_bezier (curve.rs:406-412)
static V3 blossom_bezier(const V3* p, float u0, float u1, float u2) {
    V3 a[3] = {lerp3(u0, p[0], p[1]), lerp3(u0, p[1], p[2]), lerp3(u0, p[2], p[3])};
    V3 b[2] = {lerp3(u1, a[0], a[1]), lerp3(u1, a[1], a[2])};
    return lerp3(u2, b[0], b[1]);
}
// The segment's control points (curve.rs:256-261 and 290-295).
static void segment_cp(const Sphere& s, V3* cp) {
    cp[0] = blossom_bezier(s.ccp, s.u_min, s.u_min, s.u_min);
    cp[1] = blossom_bezier(s.ccp, s.u_min, s.u_min, s.u_max);
    cp[2] = blossom_bezier(s.ccp, s.u_min, s.u_max, s.u_max);
    cp[3] = blossom_bezier(s.ccp, s.u_max, s.u_max, s.u_max);
}
// Curve::new with CurveCommon::new (curve.rs:30-91).
static Sphere curve_new(const orc_curve_desc& d) {
    Sphere s;
    std::memset(&s, 0, sizeof s);
    std::memcpy(s.m, d.object_to_world, sizeof s.m);
    std::memcpy(s.mi, d.world_to_object, sizeof s.mi);
    s.kind = 6;
    s.reverse = d.reverse_orientation != 0;
    for (int i = 0; i < 4; ++i) s.ccp[i] = {d.cp[3 * i], d.cp[3 * i + 1], d.cp[3 * i + 2]};
    s.width[0] = d.width[0];
    s.width[1] = d.width[1];
    s.u_min = d.u_min;
    s.u_max = d.u_max;
    s.ctype = d.type;
    if (d.type == 2) {
        for (int e = 0; e < 2; ++e) {
            V3 v{d.n[3 * e], d.n[3 * e + 1], d.n[3 * e + 2]};
            float inv = 1.0f / std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
            s.n[e] = {v.x * inv, v.y * inv, v.z * inv};
        }
        float dot = s.n[0].x * s.n[1].x + s.n[0].y * s.n[1].y + s.n[0].z * s.n[1].z;
        s.normal_angle = std::acos(dot < 0.0f ? 0.0f : (dot > 1.0f ? 1.0f : dot));
        s.inv_sin_normal_angle = 1.0f / std::sin(s.normal_angle);
    }
    return s;
}
// Sphere::new (sphere.rs:50-75; D22: made public), Disk::new (disk.rs:27-47),
// Cylinder::new (cylinder.rs:26-46; D29: phi_max in radians of the clamped
// degrees and z_min <= z_max, as pbrt), Cone::new (cone.rs:26-41).
static Sphere sphere_new(const orc_sphere_desc& d) {
    Sphere s;
    std::memset(&s, 0, sizeof s);
    std::memcpy(s.m, d.object_to_world, sizeof s.m);
    std::memcpy(s.mi, d.world_to_object, sizeof s.mi);
    auto clamp = [](float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); };
    float mn = std::fmin(d.z_min, d.z_max), mx = std::fmax(d.z_min, d.z_max);
    s.kind = d.kind;
    s.radius = d.radius;
    // radians(): FRAC_PI_180 * deg (pbrt.rs:51-53)
    s.phi_max = (kPi / 180.0f) * clamp(d.phi_max_deg, 0.0f, 360.0f);
    s.reverse = d.reverse_orientation != 0;
    switch (d.kind) {
        case 1:   // disk
            s.height = d.height;
            s.inner_radius = d.inner_radius;
            s.z_min = s.z_max = d.height;
            break;
        case 2:   // cylinder
            s.z_min = mn;
            s.z_max = mx;
            break;
        case 3:   // cone
            s.height = d.height;
            s.z_min = 0.0f;
            s.z_max = d.height;
            break;
        case 4:   // paraboloid (paraboloid.rs:26-47; z range ordered as pbrt)
            s.z_min = mn;
            s.z_max = mx;
            break;
        case 5: {   // hyperboloid (hyperboloid.rs:31-77)
            V3 p1{d.p1[0], d.p1[1], d.p1[2]}, p2{d.p2[0], d.p2[1], d.p2[2]};
            float radius1 = std::sqrt(p1.x * p1.x + p1.y * p1.y);
            float radius2 = std::sqrt(p2.x * p2.x + p2.y * p2.y);
            s.radius = std::fmax(radius1, radius2);
            s.z_min = std::fmin(p1.z, p2.z);
            s.z_max = std::fmax(p1.z, p2.z);
            // D33: swap when p2.z == 0 (the reference swaps when it is not),
            // and iterate until both coefficients are finite (not only
            // until neither is infinite), as pbrt
            if (p2.z == 0.0f) std::swap(p1, p2);
            V3 pp = p1;
            float ah = std::numeric_limits<float>::infinity(), ch = ah;
            for (int it = 0; it < 64 && !(std::isfinite(ah) && std::isfinite(ch)); ++it) {
                pp = {pp.x + 2.0f * (p2.x - p1.x), pp.y + 2.0f * (p2.y - p1.y), pp.z + 2.0f * (p2.z - p1.z)};
                float xy1 = pp.x * pp.x + pp.y * pp.y;
                float xy2 = p2.x * p2.x + p2.y * p2.y;
                ah = (1.0f / xy1 - (pp.z * pp.z) / (xy1 * p2.z * p2.z)) /
                     (1.0f - (xy2 * pp.z * pp.z) / (xy1 * p2.z * p2.z));
                ch = (ah * xy2 - 1.0f) / (p2.z * p2.z);
            }
            s.p1 = p1;
            s.p2 = p2;
            s.ah = ah;
            s.ch = ch;
            break;
        }
        default:   // sphere
            s.z_min = clamp(mn, -d.radius, d.radius);
            s.z_max = clamp(mx, -d.radius, d.radius);
            s.theta_min = std::acos(clamp(mn / d.radius, -1.0f, 1.0f));
            s.theta_max = std::acos(clamp(mx / d.radius, -1.0f, 1.0f));
    }
    return s;
}
// Transform::transform_bounds -> Bounds3::transform (bounds3.rs:320-356)
static B3 sphere_world_bound(const Sphere& s) {
    B3 ob;
    ob.mn = {-s.radius, -s.radius, s.z_min};
    ob.mx = {s.radius, s.radius, s.z_max};
    if (s.kind == 6) {   // Curve::object_bound (curve.rs:255-268)
        V3 cp[4];
        segment_cp(s, cp);
        B3 b;
        b = bunion_pt(b, cp[0]);
        b = bunion_pt(b, cp[1]);
        b = bunion_pt(b, cp[2]);
        b = bunion_pt(b, cp[3]);
        float w = std::fmax(lerpf(s.u_min, s.width[0], s.width[1]), lerpf(s.u_max, s.width[0], s.width[1])) * 0.5f;
        ob.mn = {b.mn.x - w, b.mn.y - w, b.mn.z - w};
        ob.mx = {b.mx.x + w, b.mx.y + w, b.mx.z + w};
    }
    float bmin[3] = {s.m[3], s.m[7], s.m[11]}, bmax[3] = {s.m[3], s.m[7], s.m[11]};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            float a = s.m[4 * i + j] * comp(ob.mn, j);
            float b = s.m[4 * i + j] * comp(ob.mx, j);
            if (a < b) { bmin[i] += a; bmax[i] += b; } else { bmin[i] += b; bmax[i] += a; }
        }
    B3 r;
    r.mn = {bmin[0], bmin[1], bmin[2]};
    r.mx = {bmax[0], bmax[1], bmax[2]};
    return r;
}
// Transform::transform_ray_with_error (transform.rs:392-435), using
// transform_point_with_error (224-247) and transform_vector_with_error (296-309).
static void transform_ray_with_error(const float* m, const Ray& r, V3* o, V3* d, V3* oe, V3* de) {
    float x = r.o.x, y = r.o.y, z = r.o.z;
    float xp = (m[0] * x + m[1] * y) + (m[2] * z + m[3]);
    float yp = (m[4] * x + m[5] * y) + (m[6] * z + m[7]);
    float zp = (m[8] * x + m[9] * y) + (m[10] * z + m[11]);
    float wp = (m[12] * x + m[13] * y) + (m[14] * z + m[15]);
    float xs = std::fabs(m[0] * x) + std::fabs(m[1] * y) + std::fabs(m[2] * z) + std::fabs(m[3]);
    float ys = std::fabs(m[4] * x) + std::fabs(m[5] * y) + std::fabs(m[6] * z) + std::fabs(m[7]);
    float zs = std::fabs(m[8] * x) + std::fabs(m[9] * y) + std::fabs(m[10] * z) + std::fabs(m[11]);
    float g3 = gamma(3);
    *oe = {xs * g3, ys * g3, zs * g3};
    if (wp == 1.0f) *o = {xp, yp, zp}; else *o = {xp / wp, yp / wp, zp / wp};
    x = r.d.x; y = r.d.y; z = r.d.z;
    de->x = g3 * (std::fabs(m[0] * x) + std::fabs(m[1] * y) + std::fabs(m[2] * z));
    de->y = g3 * (std::fabs(m[4] * x) + std::fabs(m[5] * y) + std::fabs(m[6] * z));
    de->z = g3 * (std::fabs(m[8] * x) + std::fabs(m[9] * y) + std::fabs(m[10] * z));
    *d = {m[0] * x + m[1] * y + m[2] * z, m[4] * x + m[5] * y + m[6] * z, m[8] * x + m[9] * y + m[10] * z};
    float ls = length_sq(*d);
    if (ls > 0.0f) {
        float dt = (std::fabs(d->x) * oe->x + std::fabs(d->y) * oe->y + std::fabs(d->z) * oe->z) / ls;
        o->x += d->x * dt; o->y += d->y * dt; o->z += d->z * dt;
    }
}
// Sphere::intersect / intersect_p (sphere.rs:105-188 and 238-323).  D24:
// Point3::distance (point3.rs:62-66) returns sqrt(p.o) instead of |p-o|, so
// the refine step would divide by zero; repaired to the Euclidean distance.
static bool sphere_test(const Sphere& s, const Ray& world_ray, float* t_out, float* uv_out) {
    V3 o, d, oe, de;
    transform_ray_with_error(s.mi, world_ray, &o, &d, &oe, &de);
    float t_max = world_ray.t_max;
    EF ox = ef_new(o.x, oe.x), oy = ef_new(o.y, oe.y), oz = ef_new(o.z, oe.z);
    EF dx = ef_new(d.x, de.x), dy = ef_new(d.y, de.y), dz = ef_new(d.z, de.z);
    EF a = ef_add(ef_add(ef_mul(dx, dx), ef_mul(dy, dy)), ef_mul(dz, dz));
    EF b = ef_mul(ef_add(ef_add(ef_mul(dx, ox), ef_mul(dy, oy)), ef_mul(dz, oz)), ef_new(2.0f, 0.0f));
    EF rr = ef_new(s.radius, 0.0f);
    EF c = ef_sub(ef_add(ef_add(ef_mul(ox, ox), ef_mul(oy, oy)), ef_mul(oz, oz)), ef_mul(rr, rr));
    EF t0, t1;
    if (!ef_quadratic(a, b, c, &t0, &t1)) return false;
    if (t0.high > t_max || t1.low <= 0.0f) return false;
    EF th = t0;
    if (th.low <= 0.0f) {
        th = t1;
        if (th.high > t_max) return false;
    }
    auto hit_point = [&](float t, V3* p, float* phi) {
        *p = {o.x + d.x * t, o.y + d.y * t, o.z + d.z * t};
        float dist = std::sqrt(p->x * p->x + p->y * p->y + p->z * p->z);  // D24
        float k = s.radius / dist;
        p->x *= k; p->y *= k; p->z *= k;
        if (p->x == 0.0f && p->y == 0.0f) p->x = 1e-5f * s.radius;
        *phi = std::atan2(p->y, p->x);
        if (*phi < 0.0f) *phi += 2.0f * kPi;
    };
    V3 p; float phi;
    hit_point(th.v, &p, &phi);
    auto clipped = [&](const V3& q, float ph) {
        return (s.z_min > -s.radius && q.z < s.z_min) || (s.z_max < s.radius && q.z > s.z_max) ||
               ph > s.phi_max;
    };
    if (clipped(p, phi)) {
        if (th.v == t1.v) return false;
        if (t1.high > t_max) return false;
        th = t1;
        hit_point(th.v, &p, &phi);
        if (clipped(p, phi)) return false;
    }
    // parametric (u, v) (sphere.rs:191-193)
    float u = phi / s.phi_max;
    float zr = p.z / s.radius;
    zr = zr < -1.0f ? -1.0f : (zr > 1.0f ? 1.0f : zr);
    float theta = std::acos(zr);
    float v = (theta - s.theta_min) / (s.theta_max - s.theta_min);
    *t_out = th.v;
    uv_out[0] = u; uv_out[1] = v;
    return true;
}

// Disk::intersect / intersect_p (disk.rs:110-166, 168-203): the plane z =
// height in object space, then the radii and phi_max.
static bool disk_test(const Sphere& s, const Ray& world_ray, float* t_out, float* uv_out) {
    V3 o, d, oe, de;
    transform_ray_with_error(s.mi, world_ray, &o, &d, &oe, &de);
    if (d.z == 0.0f) return false;
    float t = (s.height - o.z) / d.z;
    if (t <= 0.0f || t >= world_ray.t_max) return false;
    V3 p{o.x + d.x * t, o.y + d.y * t, o.z + d.z * t};
    float dist2 = p.x * p.x + p.y * p.y;
    if (dist2 > s.radius * s.radius || dist2 < s.inner_radius * s.inner_radius) return false;
    float phi = std::atan2(p.y, p.x);
    if (phi < 0.0f) phi += 2.0f * kPi;
    if (phi > s.phi_max) return false;
    float r_hit = std::sqrt(dist2);
    *t_out = t;
    uv_out[0] = phi / s.phi_max;
    uv_out[1] = (s.radius - r_hit) / (s.radius - s.inner_radius);
    return true;
}

// The nearest root of [t0, t1] within (0, t_max] (sphere.rs:135-144 and the
// same lines of cylinder.rs / cone.rs); false when neither qualifies.
static bool nearest_root(const EF& t0, const EF& t1, float t_max, EF* th) {
    if (t0.high > t_max || t1.low <= 0.0f) return false;
    *th = t0;
    if (th->low <= 0.0f) {
        *th = t1;
        if (th->high > t_max) return false;
    }
    return true;
}

// Cylinder::intersect / intersect_p (cylinder.rs:77-...): x^2 + y^2 = r^2,
// the hit refined onto the radius, clipped by z and phi (retry with t1).
static bool cylinder_test(const Sphere& s, const Ray& world_ray, float* t_out, float* uv_out) {
    V3 o, d, oe, de;
    transform_ray_with_error(s.mi, world_ray, &o, &d, &oe, &de);
    EF ox = ef_new(o.x, oe.x), oy = ef_new(o.y, oe.y);
    EF dx = ef_new(d.x, de.x), dy = ef_new(d.y, de.y);
    EF a = ef_add(ef_mul(dx, dx), ef_mul(dy, dy));
    EF b = ef_mul(ef_add(ef_mul(dx, ox), ef_mul(dy, oy)), ef_new(2.0f, 0.0f));
    EF rr = ef_new(s.radius, 0.0f);
    EF c = ef_sub(ef_add(ef_mul(ox, ox), ef_mul(oy, oy)), ef_mul(rr, rr));
    EF t0, t1, th;
    if (!ef_quadratic(a, b, c, &t0, &t1)) return false;
    if (!nearest_root(t0, t1, world_ray.t_max, &th)) return false;
    V3 p;
    float phi;
    auto hit_point = [&](float t) {
        p = {o.x + d.x * t, o.y + d.y * t, o.z + d.z * t};
        float hit_rad = std::sqrt(p.x * p.x + p.y * p.y);
        p.x *= s.radius / hit_rad;
        p.y *= s.radius / hit_rad;
        phi = std::atan2(p.y, p.x);
        if (phi < 0.0f) phi += 2.0f * kPi;
    };
    auto clipped = [&]() { return p.z < s.z_min || p.z > s.z_max || phi > s.phi_max; };
    hit_point(th.v);
    if (clipped()) {
        if (th.v == t1.v) return false;
        if (t1.high > world_ray.t_max) return false;
        th = t1;
        hit_point(th.v);
        if (clipped()) return false;
    }
    *t_out = th.v;
    uv_out[0] = phi / s.phi_max;
    uv_out[1] = (p.z - s.z_min) / (s.z_max - s.z_min);
    return true;
}

// Cone::intersect / intersect_p (cone.rs:91-...): x^2 + y^2 = k (z - h)^2
// with k = (r / h)^2, clipped by 0 <= z <= h and phi (retry with t1).  D28:
// the reference's b = dx*ox + dy*oy - k*dz*(oz - h)*2 doubles only the last
// term; repaired to 2 (dx*ox + dy*oy - k*dz*(oz - h)) as pbrt.
static bool cone_test(const Sphere& s, const Ray& world_ray, float* t_out, float* uv_out) {
    V3 o, d, oe, de;
    transform_ray_with_error(s.mi, world_ray, &o, &d, &oe, &de);
    EF ox = ef_new(o.x, oe.x), oy = ef_new(o.y, oe.y), oz = ef_new(o.z, oe.z);
    EF dx = ef_new(d.x, de.x), dy = ef_new(d.y, de.y), dz = ef_new(d.z, de.z);
    EF k = ef_div(ef_new(s.radius, 0.0f), ef_new(s.height, 0.0f));
    k = ef_mul(k, k);
    EF ozh = ef_sub(oz, ef_new(s.height, 0.0f));
    EF a = ef_sub(ef_add(ef_mul(dx, dx), ef_mul(dy, dy)), ef_mul(ef_mul(k, dz), dz));
    EF b = ef_mul(ef_sub(ef_add(ef_mul(dx, ox), ef_mul(dy, oy)), ef_mul(ef_mul(k, dz), ozh)), ef_new(2.0f, 0.0f));
    EF c = ef_sub(ef_add(ef_mul(ox, ox), ef_mul(oy, oy)), ef_mul(ef_mul(k, ozh), ozh));
    EF t0, t1, th;
    if (!ef_quadratic(a, b, c, &t0, &t1)) return false;
    if (!nearest_root(t0, t1, world_ray.t_max, &th)) return false;
    V3 p;
    float phi;
    auto hit_point = [&](float t) {
        p = {o.x + d.x * t, o.y + d.y * t, o.z + d.z * t};
        phi = std::atan2(p.y, p.x);
        if (phi < 0.0f) phi += 2.0f * kPi;
    };
    auto clipped = [&]() { return p.z < 0.0f || p.z > s.height || phi > s.phi_max; };
    hit_point(th.v);
    if (clipped()) {
        if (th.v == t1.v) return false;
        if (t1.high > world_ray.t_max) return false;
        th = t1;
        hit_point(th.v);
        if (clipped()) return false;
    }
    *t_out = th.v;
    uv_out[0] = phi / s.phi_max;
    uv_out[1] = p.z / s.height;
    return true;
}

// Paraboloid::intersect / intersect_p (paraboloid.rs:95-...): k (x^2 + y^2)
// = z with k = z_max / r^2 in EFloat, clipped by z and phi (retry with t1).
static bool paraboloid_test(const Sphere& s, const Ray& world_ray, float* t_out, float* uv_out) {
    V3 o, d, oe, de;
    transform_ray_with_error(s.mi, world_ray, &o, &d, &oe, &de);
    EF ox = ef_new(o.x, oe.x), oy = ef_new(o.y, oe.y), oz = ef_new(o.z, oe.z);
    EF dx = ef_new(d.x, de.x), dy = ef_new(d.y, de.y), dz = ef_new(d.z, de.z);
    EF k = ef_div(ef_new(s.z_max, 0.0f), ef_mul(ef_new(s.radius, 0.0f), ef_new(s.radius, 0.0f)));
    EF a = ef_mul(k, ef_add(ef_mul(dx, dx), ef_mul(dy, dy)));
    // D23: the reference's `* 2.0` builds an interval as wide as the value; exact 2
    EF b = ef_sub(ef_mul(ef_mul(k, ef_add(ef_mul(dx, ox), ef_mul(dy, oy))), ef_new(2.0f, 0.0f)), dz);
    EF c = ef_sub(ef_mul(k, ef_add(ef_mul(ox, ox), ef_mul(oy, oy))), oz);
    EF t0, t1, th;
    if (!ef_quadratic(a, b, c, &t0, &t1)) return false;
    if (!nearest_root(t0, t1, world_ray.t_max, &th)) return false;
    V3 p;
    float phi;
    auto hit_point = [&](float t) {
        p = {o.x + d.x * t, o.y + d.y * t, o.z + d.z * t};
        phi = std::atan2(p.y, p.x);
        if (phi < 0.0f) phi += 2.0f * kPi;
    };
    auto clipped = [&]() { return p.z < s.z_min || p.z > s.z_max || phi > s.phi_max; };
    hit_point(th.v);
    if (clipped()) {
        if (th.v == t1.v) return false;
        if (t1.high > world_ray.t_max) return false;
        th = t1;
        hit_point(th.v);
        if (clipped()) return false;
    }
    *t_out = th.v;
    uv_out[0] = phi / s.phi_max;
    uv_out[1] = (p.z - s.z_min) / (s.z_max - s.z_min);
    return true;
}

// Hyperboloid::intersect / intersect_p (hyperboloid.rs:128-...): ah (x^2 +
// y^2) - ch z^2 = 1, clipped by z and phi (retry with t1); phi is measured
// from the swept point pr = (1 - v) p1 + v p2 at the hit's height.
// D34: c = ah ox^2 + ah oy^2 - ch oz^2 - 1 (line 149 has - oz^2 - ch).
// D35: the first phi is atan2(pr.x py - px pr.y, px pr.x + py pr.y) (line 169
// applies atan2 to pr.y alone; line 180 has it right).
static bool hyperboloid_test(const Sphere& s, const Ray& world_ray, float* t_out, float* uv_out) {
    V3 o, d, oe, de;
    transform_ray_with_error(s.mi, world_ray, &o, &d, &oe, &de);
    EF ox = ef_new(o.x, oe.x), oy = ef_new(o.y, oe.y), oz = ef_new(o.z, oe.z);
    EF dx = ef_new(d.x, de.x), dy = ef_new(d.y, de.y), dz = ef_new(d.z, de.z);
    EF ah = ef_new(s.ah, 0.0f), ch = ef_new(s.ch, 0.0f);
    EF a = ef_sub(ef_add(ef_mul(ef_mul(dx, dx), ah), ef_mul(ef_mul(dy, dy), ah)), ef_mul(ef_mul(dz, dz), ch));
    EF b = ef_mul(ef_new(2.0f, 0.0f),
                  ef_sub(ef_add(ef_mul(ef_mul(dx, ox), ah), ef_mul(ef_mul(dy, oy), ah)), ef_mul(ef_mul(dz, oz), ch)));
    EF c = ef_sub(ef_sub(ef_add(ef_mul(ef_mul(ox, ox), ah), ef_mul(ef_mul(oy, oy), ah)), ef_mul(ef_mul(oz, oz), ch)),
                  ef_new(1.0f, 0.0f));
    EF t0, t1, th;
    if (!ef_quadratic(a, b, c, &t0, &t1)) return false;
    if (!nearest_root(t0, t1, world_ray.t_max, &th)) return false;
    V3 p;
    float phi, v;
    auto hit_point = [&](float t) {
        p = {o.x + d.x * t, o.y + d.y * t, o.z + d.z * t};
        v = (p.z - s.p1.z) / (s.p2.z - s.p1.z);
        V3 pr{s.p1.x * (1.0f - v) + s.p2.x * v, s.p1.y * (1.0f - v) + s.p2.y * v, 0.0f};
        phi = std::atan2(pr.x * p.y - p.x * pr.y, p.x * pr.x + p.y * pr.y);
        if (phi < 0.0f) phi += 2.0f * kPi;
    };
    auto clipped = [&]() { return p.z < s.z_min || p.z > s.z_max || phi > s.phi_max; };
    hit_point(th.v);
    if (clipped()) {
        if (th.v == t1.v) return false;
        if (t1.high > world_ray.t_max) return false;
        th = t1;
        hit_point(th.v);
        if (clipped()) return false;
    }
    *t_out = th.v;
    uv_out[0] = phi / s.phi_max;
    uv_out[1] = v;
    return true;
}

// ---------------------------------------------------------------- curve.rs
static inline V3 add3(const V3& a, const V3& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 scl3(const V3& a, float s) { return {a.x * s, a.y * s, a.z * s}; }
static inline float dot3(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 norm3(const V3& a) { return scl3(a, 1.0f / std::sqrt(dot3(a, a))); }   // vector3.rs:85-95

// subdivide_bezier (curve.rs:414-423)
static void subdivide_bezier(const V3* cp, V3* out) {
    out[0] = cp[0];
    out[1] = scl3(add3(cp[0], cp[1]), 0.5f);
    out[2] = scl3(add3(add3(cp[0], scl3(cp[1], 2.0f)), cp[2]), 0.25f);
    out[3] = scl3(add3(add3(add3(cp[0], scl3(cp[1], 3.0f)), scl3(cp[2], 3.0f)), cp[3]), 0.125f);
    out[4] = scl3(add3(add3(cp[1], scl3(cp[2], 2.0f)), cp[3]), 0.25f);
    out[5] = scl3(add3(cp[2], cp[3]), 0.5f);
    out[6] = cp[3];
}
// eval_bezier (curve.rs:425-446)
static V3 eval_bezier(const V3* cp, float u, V3* deriv) {
    V3 c1[3] = {lerp3(u, cp[0], cp[1]), lerp3(u, cp[1], cp[2]), lerp3(u, cp[2], cp[3])};
    V3 c2[2] = {lerp3(u, c1[0], c1[1]), lerp3(u, c1[1], c1[2])};
    V3 dd = sub(c2[1], c2[0]);
    *deriv = dot3(dd, dd) > 0.0f ? scl3(dd, 3.0f) : sub(cp[3], cp[0]);
    return lerp3(u, c2[0], c2[1]);
}
// The segment against the ray's beam, padded by half its width (curve.rs:116-140).
static bool beam_overlaps(const V3* c, float max_width, float z_max) {
    float hw = 0.5f * max_width;
    if (std::fmax(std::fmax(c[0].y, c[1].y), std::fmax(c[2].y, c[3].y)) + hw < 0.0f ||
        std::fmin(std::fmin(c[0].y, c[1].y), std::fmin(c[2].y, c[3].y)) - hw > 0.0f)
        return false;
    if (std::fmax(std::fmax(c[0].x, c[1].x), std::fmax(c[2].x, c[3].x)) + hw < 0.0f ||
        std::fmin(std::fmin(c[0].x, c[1].x), std::fmin(c[2].x, c[3].x)) - hw > 0.0f)
        return false;
    return !(std::fmax(std::fmax(c[0].z, c[1].z), std::fmax(c[2].z, c[3].z)) + hw < 0.0f ||
             std::fmin(std::fmin(c[0].z, c[1].z), std::fmin(c[2].z, c[3].z)) - hw > z_max);
}

struct CurveHit { float t, u, v; bool hit; };

// Curve::recursive_intersect (curve.rs:94-252), t / u / v only.  Repairs:
// the halves come from the subdivided points (the reference slices the
// parent's four points), and the nearer of the halves' hits is kept (the
// reference keeps the last one found); later halves are tested against the
// nearest hit so far.
static void recursive_intersect(const Sphere& s, const V3* cp, const V3& d, float ray_len, float u0, float u1,
                                int depth, float* z_max, CurveHit* best) {
    if (depth > 0) {
        V3 split[7];
        subdivide_bezier(cp, split);
        float u[3] = {u0, (u0 + u1) * 0.5f, u1};
        for (int seg = 0; seg < 2; ++seg) {
            const V3* cps = split + 3 * seg;
            float mw = std::fmax(lerpf(u[seg], s.width[0], s.width[1]), lerpf(u[seg + 1], s.width[0], s.width[1]));
            if (!beam_overlaps(cps, mw, *z_max)) continue;
            recursive_intersect(s, cps, d, ray_len, u[seg], u[seg + 1], depth - 1, z_max, best);
        }
        return;
    }
    float edge = (cp[1].y - cp[0].y) * -cp[0].y + cp[0].x * (cp[0].x - cp[1].x);
    if (edge < 0.0f) return;
    edge = (cp[2].y - cp[3].y) * -cp[3].y + cp[3].x * (cp[3].x - cp[2].x);
    if (edge < 0.0f) return;
    float sx = cp[3].x - cp[0].x, sy = cp[3].y - cp[0].y;
    float denom = sx * sx + sy * sy;
    if (denom == 0.0f) return;
    float w = (-cp[0].x * sx + -cp[0].y * sy) / denom;
    float u = std::fmin(std::fmax(lerpf(w, u0, u1), u0), u1);
    float hit_width = lerpf(u, s.width[0], s.width[1]);
    if (s.ctype == 2) {
        // D38: parallel normals (angle 0) give 0 * inf = NaN weights in the
        // reference (curve.rs:185-191); the ribbon then keeps n0
        V3 nh = s.n[0];
        if (s.normal_angle != 0.0f) {
            float sin0 = std::sin((1.0f - u) * s.normal_angle) * s.inv_sin_normal_angle;
            float sin1 = std::sin(u * s.normal_angle) * s.inv_sin_normal_angle;
            nh = add3(scl3(s.n[0], sin0), scl3(s.n[1], sin1));
        }
        hit_width *= std::fabs(dot3(nh, d)) / ray_len;
    }
    V3 dpcdw;
    V3 pc = eval_bezier(cp, std::fmin(std::fmax(w, 0.0f), 1.0f), &dpcdw);
    float dist2 = pc.x * pc.x + pc.y * pc.y;
    if (dist2 > hit_width * hit_width * 0.25f) return;
    if (pc.z < 0.0f || pc.z > *z_max) return;
    float dist = std::sqrt(dist2);
    float edge_func = dpcdw.x * -pc.y + pc.x * dpcdw.y;
    float v = edge_func > 0.0f ? 0.5f + dist / hit_width : 0.5f - dist / hit_width;
    float t = pc.z / ray_len;
    if (!best->hit || t < best->t) {
        *best = CurveHit{t, u, v, true};
        *z_max = pc.z;
    }
}

// Curve::intersect (curve.rs:278-375).  The ray frame is the reference's
// look_at(o, o + d, up) with its inverse applied as the transpose of the
// orthonormal frame; Vector3::cross is evaluated in f64 (vector3.rs:67-83).
static bool curve_test(const Sphere& s, const Ray& world_ray, float* t_out, float* uv_out) {
    V3 o, d, oe, de;
    transform_ray_with_error(s.mi, world_ray, &o, &d, &oe, &de);
    V3 cp_obj[4];
    segment_cp(s, cp_obj);
    V3 dx = cross64(d, sub(cp_obj[3], cp_obj[0]));
    if (length_sq(dx) == 0.0f) {   // coordinate_system (vector3.rs:520-545)
        if (std::fabs(d.x) > std::fabs(d.y)) {
            float len = std::sqrt(d.x * d.x + d.z * d.z);
            dx = {-d.z / len, 0.0f, d.x / len};
        } else {
            float len = std::sqrt(d.y * d.y + d.z * d.z);
            dx = {0.0f, d.z / len, -d.y / len};
        }
    }
    V3 dir = norm3(sub(add3(o, d), o));
    V3 right = norm3(cross64(norm3(dx), dir));
    V3 new_up = cross64(dir, right);
    V3 cp[4];
    for (int i = 0; i < 4; ++i) {
        V3 q = sub(cp_obj[i], o);
        cp[i] = {dot3(right, q), dot3(new_up, q), dot3(dir, q)};
    }
    float ray_len = std::sqrt(dot3(d, d));
    float z_max = ray_len * world_ray.t_max;
    float max_width = std::fmax(lerpf(s.u_min, s.width[0], s.width[1]), lerpf(s.u_max, s.width[0], s.width[1]));
    if (!beam_overlaps(cp, max_width, z_max)) return false;
    float l0 = 0.0f;
    for (int i = 0; i < 2; ++i)
        l0 = std::fmax(l0, std::fmax(std::fmax(std::fabs(cp[i].x - 2.0f * cp[i + 1].x + cp[i + 2].x),
                                               std::fabs(cp[i].y - 2.0f * cp[i + 1].y + cp[i + 2].y)),
                                     std::fabs(cp[i].z - 2.0f * cp[i + 1].z + cp[i + 2].z)));
    float eps = std::fmax(s.width[0], s.width[1]) * 0.05f;
    auto log2i = [](float v) -> int {   // curve.rs:340-350
        if (v < 1.0f) return 0;
        uint32_t bits = f2u(v);
        return (int)(bits >> 23) - 127 + ((bits & (1u << 22)) ? 1 : 0);
    };
    int r0 = log2i(1.41421356237f * 6.0f * l0 / (8.0f * eps)) / 2;
    int max_depth = r0 < 0 ? 0 : (r0 > 10 ? 10 : r0);
    CurveHit best{0, 0, 0, false};
    recursive_intersect(s, cp, d, ray_len, s.u_min, s.u_max, max_depth, &z_max, &best);
    if (!best.hit) return false;
    *t_out = best.t;
    uv_out[0] = best.u;
    uv_out[1] = best.v;
    return true;
}

static bool quadric_test(const Sphere& s, const Ray& ray, float* t_out, float* uv_out) {
    switch (s.kind) {
        case 6: return curve_test(s, ray, t_out, uv_out);
        case 1: return disk_test(s, ray, t_out, uv_out);
        case 2: return cylinder_test(s, ray, t_out, uv_out);
        case 3: return cone_test(s, ray, t_out, uv_out);
        case 4: return paraboloid_test(s, ray, t_out, uv_out);
        case 5: return hyperboloid_test(s, ray, t_out, uv_out);
        default: return sphere_test(s, ray, t_out, uv_out);
    }
}

// ---------------------------------------------------------------- bvh.rs
struct PrimInfo { uint32_t prim; B3 bounds; V3 centroid; };
struct BuildNode {
    B3 bounds;
    int child[2] = {-1, -1};
    int split_axis = 0;
    uint32_t first_prim_offset = 0, n_primitives = 0;
};
struct BucketInfo { uint32_t count = 0; B3 bounds; };

struct Builder {
    int max_prims;
    std::vector<PrimInfo>& info;
    std::vector<BuildNode> nodes;
    std::vector<uint32_t> ordered;
    Builder(int mp, std::vector<PrimInfo>& pi) : max_prims(mp), info(pi) {}

    int make_leaf(uint32_t start, uint32_t end, const B3& bounds) {
        BuildNode n;
        n.first_prim_offset = (uint32_t)ordered.size();
        for (uint32_t i = start; i < end; ++i) ordered.push_back(info[i].prim);
        n.n_primitives = end - start;
        n.bounds = bounds;
        nodes.push_back(n);
        return (int)nodes.size() - 1;
    }
    // SAH bucket of a centroid; D2 (bvh.rs:176,219): cast after multiplying.
    static int bucket_of(const B3& cb, const V3& c, int dim) {
        int b = (int)(12.0f * comp(offset(cb, c), dim));
        if (b == 12) b = 11;
        return b;
    }
    // recursive_build (bvh.rs:95-247), SAH path; D1 (centroid bounds are a
    // union of centroids), D2, D3 (argmin, first minimum wins) repaired; D7
    // (leaf on zero centroid extent) and D8 (split criterion) kept.
    int build(uint32_t start, uint32_t end) {
        B3 bounds;
        for (uint32_t i = start; i < end; ++i) bounds = bunion(bounds, info[i].bounds);
        uint32_t n = end - start;
        if (n == 1) return make_leaf(start, end, bounds);
        B3 cb;
        for (uint32_t i = start; i < end; ++i) cb = bunion_pt(cb, info[i].centroid);
        int dim = maximum_extent(cb);
        uint32_t mid = (start + end) / 2;
        if (comp(cb.mx, dim) == comp(cb.mn, dim)) return make_leaf(start, end, bounds);
        if (n <= 2) {
            // partial_sort(mid) of two elements (slice_extension.rs:45-72): one
            // pivot pass that swaps iff c[1] < c[0].
            if (comp(info[start + 1].centroid, dim) < comp(info[start].centroid, dim))
                std::swap(info[start], info[start + 1]);
        } else {
            BucketInfo buckets[12];
            for (uint32_t i = start; i < end; ++i) {
                int b = bucket_of(cb, info[i].centroid, dim);
                buckets[b].count += 1;
                buckets[b].bounds = bunion(buckets[b].bounds, info[i].bounds);
            }
            float cost[11];
            for (int i = 0; i < 11; ++i) {
                B3 b0, b1;
                uint32_t c0 = 0, c1 = 0;
                for (int j = 0; j <= i; ++j) { b0 = bunion(b0, buckets[j].bounds); c0 += buckets[j].count; }
                for (int j = i + 1; j < 12; ++j) { b1 = bunion(b1, buckets[j].bounds); c1 += buckets[j].count; }
                cost[i] = 1.0f + ((float)c0 * surface_area(b0) + (float)c1 * surface_area(b1)) /
                                     surface_area(bounds);
            }
            float min_cost = cost[0];
            int split = 0;
            for (int i = 1; i < 11; ++i)
                if (cost[i] < min_cost) { min_cost = cost[i]; split = i; }
            float leaf_cost = (float)n;
            if (n > (uint32_t)max_prims || min_cost < leaf_cost) {
                // SliceExtension::partition (slice_extension.rs:20-43)
                uint32_t first = end;
                for (uint32_t i = start; i < end; ++i)
                    if (!(bucket_of(cb, info[i].centroid, dim) <= split)) { first = i; break; }
                if (first != end) {
                    for (uint32_t i = first; i < end; ++i)
                        if (bucket_of(cb, info[i].centroid, dim) <= split) { std::swap(info[i], info[first]); ++first; }
                }
                mid = first;
            } else {
                return make_leaf(start, end, bounds);
            }
        }
        int self = (int)nodes.size();
        nodes.push_back(BuildNode());
        int c0 = build(start, mid);
        int c1 = build(mid, end);
        // init_interior (bvh.rs:707-719)
        nodes[self].bounds = bunion(nodes[c0].bounds, nodes[c1].bounds);
        nodes[self].split_axis = dim;
        nodes[self].child[0] = c0;
        nodes[self].child[1] = c1;
        nodes[self].n_primitives = 0;
        return self;
    }
};

// flatten_bvh_tree (bvh.rs:504-537): depth-first, first child adjacent.
static uint32_t flatten(const std::vector<BuildNode>& bn, int node, std::vector<orc_bvh_node>& out, uint32_t* offset) {
    uint32_t my = (*offset)++;
    const BuildNode& b = bn[node];
    orc_bvh_node ln;
    std::memset(&ln, 0, sizeof ln);
    ln.bmin[0] = b.bounds.mn.x; ln.bmin[1] = b.bounds.mn.y; ln.bmin[2] = b.bounds.mn.z;
    ln.bmax[0] = b.bounds.mx.x; ln.bmax[1] = b.bounds.mx.y; ln.bmax[2] = b.bounds.mx.z;
    if (b.n_primitives > 0) {
        ln.offset = (int32_t)b.first_prim_offset;
        ln.n_prims = (uint16_t)b.n_primitives;
        out[my] = ln;
    } else {
        flatten(bn, b.child[0], out, offset);
        ln.offset = (int32_t)flatten(bn, b.child[1], out, offset);
        ln.axis = (uint8_t)b.split_axis;
        out[my] = ln;
    }
    return my;
}

struct Scene {
    std::vector<V3> verts;
    std::vector<uint32_t> idx;
    uint32_t nt = 0;
    std::vector<Sphere> spheres;
    std::vector<orc_bvh_node> nodes;
    std::vector<uint32_t> prims;      // ordered primitive ids
    double build_seconds = 0;
};

static B3 tri_bound(const Scene& s, uint32_t t) {
    // Triangle::world_bound (triangle.rs:126-132)
    const V3& p0 = s.verts[s.idx[3 * t]];
    const V3& p1 = s.verts[s.idx[3 * t + 1]];
    const V3& p2 = s.verts[s.idx[3 * t + 2]];
    B3 b;
    b.mn = pmin(p0, p1);
    b.mx = pmax(p0, p1);
    return bunion_pt(b, p2);
}

// Test one primitive; returns hit and fills t / uv (u=b1, v=b2 for triangles).
static bool prim_test(const Scene& s, uint32_t prim, const Ray& ray, bool closest, float* t, float* uv) {
    if (prim < s.nt) {
        float b[3];
        bool h = triangle_test(s.verts[s.idx[3 * prim]], s.verts[s.idx[3 * prim + 1]],
                               s.verts[s.idx[3 * prim + 2]], ray, closest, t, b);
        if (h) { uv[0] = b[1]; uv[1] = b[2]; }
        return h;
    }
    return quadric_test(s.spheres[prim - s.nt], ray, t, uv);
}

// BVHAccel::intersect (bvh.rs:563-612).  D4: the far child is pushed in both
// branches.  D5: the traversal owns a mutable t_max that every primitive test
// sees and that shrinks on each accepted hit.  Ties: a hit is accepted when
// t < best or (t == best and its primitive id is smaller), so the result does
// not depend on visit order except for near-ties.
static int trace_closest(const Scene& s, const orc_ray& r, orc_hit* hit, uint32_t* nv, uint32_t* nt) {
    hit->prim = 0xFFFFFFFFu; hit->t = r.tmax; hit->u = 0; hit->v = 0;
    uint32_t visits = 0, tests = 0;
    int overflow = 0;
    if (!s.nodes.empty()) {
        Ray ray{{r.o[0], r.o[1], r.o[2]}, {r.d[0], r.d[1], r.d[2]}, r.tmax};
        V3 inv{1.0f / ray.d.x, 1.0f / ray.d.y, 1.0f / ray.d.z};
        int neg[3] = {inv.x < 0.0f, inv.y < 0.0f, inv.z < 0.0f};
        uint32_t stack[64];
        int sp = 0;
        uint32_t cur = 0;
        for (;;) {
            const orc_bvh_node& n = s.nodes[cur];
            ++visits;
            if (box_intersect_p(n, ray, inv, neg)) {
                if (n.n_prims > 0) {
                    for (uint32_t i = 0; i < n.n_prims; ++i) {
                        uint32_t prim = s.prims[n.offset + i];
                        float t, uv[2];
                        ++tests;
                        if (prim_test(s, prim, ray, true, &t, uv) &&
                            (t < ray.t_max || (t == ray.t_max && prim < hit->prim))) {
                            ray.t_max = t;
                            hit->prim = prim; hit->t = t; hit->u = uv[0]; hit->v = uv[1];
                        }
                    }
                    if (sp == 0) break;
                    cur = stack[--sp];
                } else {
                    if (sp == 64) { overflow = 1; break; }
                    if (neg[n.axis]) { stack[sp++] = cur + 1; cur = (uint32_t)n.offset; }
                    else { stack[sp++] = (uint32_t)n.offset; cur = cur + 1; }
                }
            } else {
                if (sp == 0) break;
                cur = stack[--sp];
            }
        }
    }
    if (hit->prim == 0xFFFFFFFFu) hit->t = r.tmax;
    if (nv) *nv = visits;
    if (nt) *nt = tests;
    return overflow;
}

// BVHAccel::intersect_p (bvh.rs:614-662), D4 repaired.
static int trace_any(const Scene& s, const orc_ray& r, uint8_t* occ, uint32_t* nv, uint32_t* nt) {
    uint32_t visits = 0, tests = 0;
    int overflow = 0;
    *occ = 0;
    if (!s.nodes.empty()) {
        Ray ray{{r.o[0], r.o[1], r.o[2]}, {r.d[0], r.d[1], r.d[2]}, r.tmax};
        V3 inv{1.0f / ray.d.x, 1.0f / ray.d.y, 1.0f / ray.d.z};
        int neg[3] = {inv.x < 0.0f, inv.y < 0.0f, inv.z < 0.0f};
        uint32_t stack[64];
        int sp = 0;
        uint32_t cur = 0;
        for (;;) {
            const orc_bvh_node& n = s.nodes[cur];
            ++visits;
            if (box_intersect_p(n, ray, inv, neg)) {
                if (n.n_prims > 0) {
                    bool found = false;
                    for (uint32_t i = 0; i < n.n_prims; ++i) {
                        float t, uv[2];
                        ++tests;
                        if (prim_test(s, s.prims[n.offset + i], ray, false, &t, uv)) { found = true; break; }
                    }
                    if (found) { *occ = 1; break; }
                    if (sp == 0) break;
                    cur = stack[--sp];
                } else {
                    if (sp == 64) { overflow = 1; break; }
                    if (neg[n.axis]) { stack[sp++] = cur + 1; cur = (uint32_t)n.offset; }
                    else { stack[sp++] = (uint32_t)n.offset; cur = cur + 1; }
                }
            } else {
                if (sp == 0) break;
                cur = stack[--sp];
            }
        }
    }
    if (nv) *nv = visits;
    if (nt) *nt = tests;
    return overflow;
}

static double g_last_trace_seconds = 0.0;

template <class F>
static int64_t parallel_rays(uint64_t n, int nthreads, F&& fn) {
    if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
    if (nthreads <= 0) nthreads = 1;
    std::atomic<uint64_t> next{0};
    std::atomic<int64_t> overflow{0};
    const uint64_t chunk = 256;
    auto worker = [&]() {
        int64_t local = 0;
        for (;;) {
            uint64_t b = next.fetch_add(chunk);
            if (b >= n) break;
            uint64_t e = b + chunk < n ? b + chunk : n;
            for (uint64_t i = b; i < e; ++i) local += fn(i);
        }
        overflow += local;
    };
    auto t0 = std::chrono::steady_clock::now();
    if (nthreads == 1) worker();
    else {
        std::vector<std::thread> th;
        for (int i = 0; i < nthreads; ++i) th.emplace_back(worker);
        for (auto& t : th) t.join();
    }
    g_last_trace_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return overflow.load();
}

// ---------------------------------------------------------------- kd-tree
// KdTreeAccel (accelerators/kdtreeaccel.rs:11-596) over a Scene's primitives.
// Repairs, shared with the product: the split axis is rebound on each retry
// (kdtreeaccel.rs:130 binds it immutably, 189 assigns it); equal edges are
// ordered by primitive id after (position, start before end) so that the
// tree is fixed; a leaf's run is read entry by entry (kdtreeaccel.rs:351 and
// 440 read `offset + 1` on every iteration).

enum KdEdgeType { kStart = 0, kEnd = 1 };
struct KdEdge { float t; uint32_t prim; int type; };

struct KdTree {
    const Scene* scene = nullptr;
    int isect_cost = 80, traversal_cost = 1;
    float empty_bonus = 0.5f;
    uint32_t max_prims = 1;
    int max_depth = 0;
    std::vector<orc_kd_node> nodes;
    uint32_t n_alloced = 0, next_free = 0;
    std::vector<uint32_t> prim_indices;
    std::vector<B3> prim_bounds;
    B3 bounds;
};

static bool kd_is_leaf(const orc_kd_node& n) { return (n.flags & 3u) == 3u; }

// KdAccelNode::init_leaf (kdtreeaccel.rs:476-490)
static void kd_init_leaf(KdTree& k, uint32_t node, const uint32_t* prim_nums, uint32_t np) {
    orc_kd_node& n = k.nodes[node];
    n.flags = 3u | (np << 2);
    if (np == 0) n.word = 0;
    else if (np == 1) n.word = prim_nums[0];
    else {
        n.word = (uint32_t)k.prim_indices.size();
        for (uint32_t i = 0; i < np; ++i) k.prim_indices.push_back(prim_nums[i]);
    }
}

// build_tree (kdtreeaccel.rs:90-244), with the reference's scratch buffers:
// prims0 is reused by the below child, prims1 + n by both children.
static void kd_build_tree(KdTree& k, uint32_t node_num, const B3& node_bounds, const uint32_t* prim_nums,
                          uint32_t n_primitives, int depth, std::vector<KdEdge>* edges, uint32_t* prims0,
                          uint32_t* prims1, int bad_refines) {
    if (k.next_free == k.n_alloced) {
        uint32_t n_new = std::max(2 * k.n_alloced, 512u);
        k.nodes.resize(n_new, orc_kd_node{0, 0});
        k.n_alloced = n_new;
    }
    ++k.next_free;
    if (n_primitives <= k.max_prims || depth == 0) {
        kd_init_leaf(k, node_num, prim_nums, n_primitives);
        return;
    }
    int best_axis = -1, best_offset = -1;
    float best_cost = std::numeric_limits<float>::infinity();
    float old_cost = (float)((uint64_t)k.isect_cost * n_primitives);
    float total_sa = surface_area(node_bounds);
    float inv_total_sa = 1.0f / total_sa;
    V3 d = sub(node_bounds.mx, node_bounds.mn);
    int axis = maximum_extent(node_bounds);
    int retries = 0;
    for (;;) {
        std::vector<KdEdge>& e = edges[axis];
        for (uint32_t i = 0; i < n_primitives; ++i) {
            uint32_t pn = prim_nums[i];
            const B3& b = k.prim_bounds[pn];
            e[2 * i] = KdEdge{comp(b.mn, axis), pn, kStart};
            e[2 * i + 1] = KdEdge{comp(b.mx, axis), pn, kEnd};
        }
        std::sort(e.begin(), e.begin() + 2 * n_primitives, [](const KdEdge& a, const KdEdge& b) {
            if (a.t == b.t) {
                if (a.type != b.type) return a.type < b.type;
                return a.prim < b.prim;
            }
            return a.t < b.t;
        });
        uint32_t n_below = 0, n_above = n_primitives;
        for (uint32_t i = 0; i < 2 * n_primitives; ++i) {
            if (e[i].type == kEnd) --n_above;
            float edge_t = e[i].t;
            float lo = comp(node_bounds.mn, axis), hi = comp(node_bounds.mx, axis);
            if (edge_t > lo && edge_t < hi) {
                int a0 = (axis + 1) % 3, a1 = (axis + 2) % 3;
                float below_sa = 2.0f * (comp(d, a0) * comp(d, a1) + (edge_t - lo) * (comp(d, a0) + comp(d, a1)));
                float above_sa = 2.0f * (comp(d, a0) * comp(d, a1) + (hi - edge_t) * (comp(d, a0) + comp(d, a1)));
                float p_below = below_sa * inv_total_sa;
                float p_above = above_sa * inv_total_sa;
                float eb = (n_above == 0 || n_below == 0) ? k.empty_bonus : 0.0f;
                float cost = (float)k.traversal_cost +
                             (float)k.isect_cost * (1.0f - eb) * (p_below * (float)n_below + p_above * (float)n_above);
                if (cost < best_cost) {
                    best_cost = cost;
                    best_axis = axis;
                    best_offset = (int)i;
                }
            }
            if (e[i].type == kStart) ++n_below;
        }
        if (best_axis == -1 && retries < 2) {
            ++retries;
            axis = (axis + 1) % 3;
            continue;
        }
        break;
    }
    if (best_cost > old_cost) ++bad_refines;
    if ((best_cost > 4.0f * old_cost && n_primitives < 16) || best_axis == -1 || bad_refines == 3) {
        kd_init_leaf(k, node_num, prim_nums, n_primitives);
        return;
    }
    const std::vector<KdEdge>& e = edges[best_axis];
    uint32_t n0 = 0, n1 = 0;
    for (int i = 0; i < best_offset; ++i)
        if (e[i].type == kStart) prims0[n0++] = e[i].prim;
    for (uint32_t i = (uint32_t)best_offset + 1; i < 2 * n_primitives; ++i)
        if (e[i].type == kEnd) prims1[n1++] = e[i].prim;
    float t_split = e[best_offset].t;
    B3 bounds0 = node_bounds, bounds1 = node_bounds;
    if (best_axis == 0) { bounds0.mx.x = t_split; bounds1.mn.x = t_split; }
    else if (best_axis == 1) { bounds0.mx.y = t_split; bounds1.mn.y = t_split; }
    else { bounds0.mx.z = t_split; bounds1.mn.z = t_split; }
    kd_build_tree(k, node_num + 1, bounds0, prims0, n0, depth - 1, edges, prims0, prims1 + n_primitives,
                  bad_refines);
    uint32_t above_child = k.next_free;
    // KdAccelNode::init_interior (kdtreeaccel.rs:492-496)
    std::memcpy(&k.nodes[node_num].word, &t_split, 4);
    k.nodes[node_num].flags = (uint32_t)best_axis | (above_child << 2);
    kd_build_tree(k, above_child, bounds1, prims1, n1, depth - 1, edges, prims0, prims1 + n_primitives,
                  bad_refines);
}

// Bounds3::intersect_ray (geometry/bounds3.rs:253-282)
static bool bounds_intersect_ray(const B3& b, const Ray& ray, float* hit0, float* hit1) {
    float t0 = 0.0f, t1 = ray.t_max;
    for (int i = 0; i < 3; ++i) {
        float inv = 1.0f / comp(ray.d, i);
        float t_near = (comp(b.mn, i) - comp(ray.o, i)) * inv;
        float t_far = (comp(b.mx, i) - comp(ray.o, i)) * inv;
        if (t_near > t_far) std::swap(t_near, t_far);
        t_far *= 1.0f + 2.0f * gamma(3);
        if (t_near > t0) t0 = t_near;
        if (t_far < t1) t1 = t_far;
        if (t0 > t1) return false;
    }
    *hit0 = t0;
    *hit1 = t1;
    return true;
}

struct KdToDo { uint32_t node; float t_min, t_max; };

// KdTreeAccel::intersect / intersect_p (kdtreeaccel.rs:256-465).  The closest
// form owns t_max as the BVH traversal does, with the same tie rule.
static int kd_trace(const KdTree& k, const orc_ray& r, bool closest, orc_hit* hit, uint8_t* occ, uint32_t* nv,
                    uint32_t* nt) {
    if (hit) { hit->prim = 0xFFFFFFFFu; hit->t = r.tmax; hit->u = 0; hit->v = 0; }
    if (occ) *occ = 0;
    uint32_t visits = 0, tests = 0;
    struct Count {
        uint32_t *nv, *nt, *visits, *tests;
        ~Count() { if (nv) *nv = *visits; if (nt) *nt = *tests; }
    } count{nv, nt, &visits, &tests};
    if (k.nodes.empty()) return 0;
    Ray ray{{r.o[0], r.o[1], r.o[2]}, {r.d[0], r.d[1], r.d[2]}, r.tmax};
    float t_min, t_max;
    if (!bounds_intersect_ray(k.bounds, ray, &t_min, &t_max)) return 0;
    V3 inv_dir{1.0f / ray.d.x, 1.0f / ray.d.y, 1.0f / ray.d.z};
    KdToDo todo[64];
    int todo_pos = 0;
    uint32_t node = 0;
    for (;;) {
        if (ray.t_max < t_min) break;
        const orc_kd_node& n = k.nodes[node];
        ++visits;
        if (!kd_is_leaf(n)) {
            int axis = (int)(n.flags & 3u);
            float split;
            std::memcpy(&split, &n.word, 4);
            float t_plane = (split - comp(ray.o, axis)) * comp(inv_dir, axis);
            bool below_first = comp(ray.o, axis) < split || (comp(ray.o, axis) == split && comp(ray.d, axis) <= 0.0f);
            uint32_t first = below_first ? node + 1 : (n.flags >> 2);
            uint32_t second = below_first ? (n.flags >> 2) : node + 1;
            if (t_plane > t_max || t_plane <= 0.0f) {
                node = first;
            } else if (t_plane < t_min) {
                node = second;
            } else {
                if (todo_pos == 64) return 1;
                todo[todo_pos++] = KdToDo{second, t_plane, t_max};
                node = first;
                t_max = t_plane;
            }
            continue;
        }
        uint32_t np = n.flags >> 2;
        for (uint32_t i = 0; i < np; ++i) {
            uint32_t prim = np == 1 ? n.word : k.prim_indices[n.word + i];
            float t, uv[2];
            ++tests;
            if (prim_test(*k.scene, prim, ray, closest, &t, uv)) {
                if (!closest) { *occ = 1; return 0; }
                if (t < ray.t_max || (t == ray.t_max && prim < hit->prim)) {
                    ray.t_max = t;
                    hit->prim = prim; hit->t = t; hit->u = uv[0]; hit->v = uv[1];
                }
            }
        }
        if (todo_pos == 0) break;
        --todo_pos;
        node = todo[todo_pos].node;
        t_min = todo[todo_pos].t_min;
        t_max = todo[todo_pos].t_max;
    }
    return 0;
}

}  // namespace orc

using namespace orc;

extern "C" {

float orc_gamma(int n) { return gamma(n); }
float orc_next_float_up(float v) { return next_float_up(v); }
float orc_next_float_down(float v) { return next_float_down(v); }

void orc_rng_u32(uint64_t seq, uint64_t n, uint32_t* out) {
    Rng r(seq);
    for (uint64_t i = 0; i < n; ++i) out[i] = r.uniform_u32();
}
void orc_rng_floats(uint64_t seq, uint64_t n, float* out) {
    Rng r(seq);
    for (uint64_t i = 0; i < n; ++i) out[i] = r.uniform_float();
}
void orc_rng_floats_advanced(uint64_t seq, int64_t delta, uint64_t n, float* out) {
    Rng r(seq);
    r.advance(delta);
    for (uint64_t i = 0; i < n; ++i) out[i] = r.uniform_float();
}

void* orc_scene_create(const float* verts, uint32_t nv, const uint32_t* idx, uint32_t nt,
                       const orc_sphere_desc* spheres, uint32_t ns, int max_prims_in_node) {
    return orc_scene_create_curves(verts, nv, idx, nt, spheres, ns, nullptr, 0, max_prims_in_node);
}

void* orc_scene_create_curves(const float* verts, uint32_t nv, const uint32_t* idx, uint32_t nt,
                              const orc_sphere_desc* spheres, uint32_t ns, const orc_curve_desc* curves,
                              uint32_t nc, int max_prims_in_node) {
    auto t0 = std::chrono::steady_clock::now();
    Scene* s = new Scene();
    s->verts.resize(nv);
    for (uint32_t i = 0; i < nv; ++i) s->verts[i] = {verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]};
    s->idx.assign(idx, idx + 3 * (size_t)nt);
    s->nt = nt;
    for (uint32_t i = 0; i < ns; ++i) s->spheres.push_back(sphere_new(spheres[i]));
    for (uint32_t i = 0; i < nc; ++i) s->spheres.push_back(curve_new(curves[i]));
    uint32_t np = nt + ns + nc;
    if (np > 0) {
        // BVHPrimitiveInfo per primitive (bvh.rs:50-53, 730-737)
        std::vector<PrimInfo> info(np);
        for (uint32_t i = 0; i < np; ++i) {
            info[i].prim = i;
            info[i].bounds = (i < nt) ? tri_bound(*s, i) : sphere_world_bound(s->spheres[i - nt]);
            info[i].centroid = centroid(info[i].bounds);
        }
        Builder b(max_prims_in_node, info);
        b.nodes.reserve(2 * (size_t)np);
        b.ordered.reserve(np);
        int root = b.build(0, np);
        s->nodes.resize(b.nodes.size());
        uint32_t off = 0;
        flatten(b.nodes, root, s->nodes, &off);
        s->prims = std::move(b.ordered);
    }
    s->build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return s;
}
void orc_scene_destroy(void* scene) { delete (Scene*)scene; }
uint32_t orc_scene_node_count(void* scene) { return (uint32_t)((Scene*)scene)->nodes.size(); }
void orc_scene_nodes(void* scene, orc_bvh_node* out) {
    Scene* s = (Scene*)scene;
    if (!s->nodes.empty()) std::memcpy(out, s->nodes.data(), s->nodes.size() * sizeof(orc_bvh_node));
}
void orc_scene_prim_order(void* scene, uint32_t* out) {
    Scene* s = (Scene*)scene;
    if (!s->prims.empty()) std::memcpy(out, s->prims.data(), s->prims.size() * 4);
}
void orc_scene_world_bound(void* scene, float out[6]) {
    // BVHAccel::world_bound (bvh.rs:555-561)
    Scene* s = (Scene*)scene;
    B3 b;
    if (!s->nodes.empty()) {
        b.mn = {s->nodes[0].bmin[0], s->nodes[0].bmin[1], s->nodes[0].bmin[2]};
        b.mx = {s->nodes[0].bmax[0], s->nodes[0].bmax[1], s->nodes[0].bmax[2]};
    }
    out[0] = b.mn.x; out[1] = b.mn.y; out[2] = b.mn.z;
    out[3] = b.mx.x; out[4] = b.mx.y; out[5] = b.mx.z;
}
double orc_scene_build_seconds(void* scene) { return ((Scene*)scene)->build_seconds; }

int64_t orc_intersect(void* scene, const orc_ray* rays, uint64_t n, orc_hit* hits,
                      uint32_t* node_visits, uint32_t* prim_tests, int nthreads) {
    const Scene& s = *(Scene*)scene;
    return parallel_rays(n, nthreads, [&](uint64_t i) {
        return trace_closest(s, rays[i], &hits[i], node_visits ? &node_visits[i] : nullptr,
                             prim_tests ? &prim_tests[i] : nullptr);
    });
}
int64_t orc_intersect_p(void* scene, const orc_ray* rays, uint64_t n, uint8_t* occluded,
                        uint32_t* node_visits, uint32_t* prim_tests, int nthreads) {
    const Scene& s = *(Scene*)scene;
    return parallel_rays(n, nthreads, [&](uint64_t i) {
        return trace_any(s, rays[i], &occluded[i], node_visits ? &node_visits[i] : nullptr,
                         prim_tests ? &prim_tests[i] : nullptr);
    });
}

int orc_triangle_intersect(const float* p0, const float* p1, const float* p2, const orc_ray* r,
                           int closest, float* out) {
    Ray ray{{r->o[0], r->o[1], r->o[2]}, {r->d[0], r->d[1], r->d[2]}, r->tmax};
    float t, b[3];
    if (!triangle_test({p0[0], p0[1], p0[2]}, {p1[0], p1[1], p1[2]}, {p2[0], p2[1], p2[2]}, ray,
                       closest != 0, &t, b))
        return 0;
    out[0] = t; out[1] = b[0]; out[2] = b[1]; out[3] = b[2];
    return 1;
}

int orc_sphere_intersect(const orc_sphere_desc* sd, const orc_ray* r, int closest, float* out) {
    (void)closest;
    Sphere s = sphere_new(*sd);
    Ray ray{{r->o[0], r->o[1], r->o[2]}, {r->d[0], r->d[1], r->d[2]}, r->tmax};
    float t, uv[2];
    if (!quadric_test(s, ray, &t, uv)) return 0;
    out[0] = t; out[1] = uv[0]; out[2] = uv[1];
    return 1;
}

int orc_curve_intersect(const orc_curve_desc* cd, const orc_ray* r, float* out) {
    Sphere s = curve_new(*cd);
    Ray ray{{r->o[0], r->o[1], r->o[2]}, {r->d[0], r->d[1], r->d[2]}, r->tmax};
    float t, uv[2];
    if (!curve_test(s, ray, &t, uv)) return 0;
    out[0] = t; out[1] = uv[0]; out[2] = uv[1];
    return 1;
}

void orc_sphere_world_bound(const orc_sphere_desc* sd, float out[6]) {
    B3 b = sphere_world_bound(sphere_new(*sd));
    out[0] = b.mn.x; out[1] = b.mn.y; out[2] = b.mn.z;
    out[3] = b.mx.x; out[4] = b.mx.y; out[5] = b.mx.z;
}

double orc_last_trace_seconds(void) { return g_last_trace_seconds; }

int orc_trace_closest1(void* scene, const orc_ray* ray, orc_hit* hit) {
    return trace_closest(*(Scene*)scene, *ray, hit, nullptr, nullptr);
}

int orc_trace_any1(void* scene, const orc_ray* ray, uint8_t* occluded) {
    return trace_any(*(Scene*)scene, *ray, occluded, nullptr, nullptr);
}

int orc_trace_closest1_counted(void* scene, const orc_ray* ray, orc_hit* hit, uint32_t* nv, uint32_t* nt) {
    return trace_closest(*(Scene*)scene, *ray, hit, nv, nt);
}

int orc_trace_any1_counted(void* scene, const orc_ray* ray, uint8_t* occluded, uint32_t* nv, uint32_t* nt) {
    return trace_any(*(Scene*)scene, *ray, occluded, nv, nt);
}

void* orc_kdtree_create(void* scene, int isect_cost, int traversal_cost, float empty_bonus, uint32_t max_prims,
                        int max_depth) {
    const Scene* s = (const Scene*)scene;
    KdTree* k = new KdTree();
    k->scene = s;
    k->isect_cost = isect_cost;
    k->traversal_cost = traversal_cost;
    k->empty_bonus = empty_bonus;
    k->max_prims = max_prims;
    uint32_t np = s->nt + (uint32_t)s->spheres.size();
    // kdtreeaccel.rs:34-46
    if (max_depth <= 0) max_depth = np ? (int)std::lround(8.0 + 1.3 * std::log2((double)np)) : 0;
    k->max_depth = max_depth;
    k->prim_bounds.resize(np);
    for (uint32_t i = 0; i < np; ++i) {
        k->prim_bounds[i] = i < s->nt ? tri_bound(*s, i) : sphere_world_bound(s->spheres[i - s->nt]);
        k->bounds = bunion(k->bounds, k->prim_bounds[i]);
    }
    if (np == 0) return k;
    std::vector<KdEdge> edges[3];
    for (auto& e : edges) e.resize(2 * (size_t)np);
    std::vector<uint32_t> prims0(np), prims1(((size_t)max_depth + 1) * np), prim_nums(np);
    for (uint32_t i = 0; i < np; ++i) prim_nums[i] = i;
    kd_build_tree(*k, 0, k->bounds, prim_nums.data(), np, max_depth, edges, prims0.data(), prims1.data(), 0);
    k->nodes.resize(k->next_free);
    return k;
}
void orc_kdtree_destroy(void* kd) { delete (KdTree*)kd; }
uint32_t orc_kdtree_node_count(void* kd) { return (uint32_t)((KdTree*)kd)->nodes.size(); }
uint32_t orc_kdtree_index_count(void* kd) { return (uint32_t)((KdTree*)kd)->prim_indices.size(); }
int orc_kdtree_max_depth(void* kd) { return ((KdTree*)kd)->max_depth; }
void orc_kdtree_nodes(void* kd, orc_kd_node* out) {
    KdTree* k = (KdTree*)kd;
    if (!k->nodes.empty()) std::memcpy(out, k->nodes.data(), k->nodes.size() * sizeof(orc_kd_node));
}
void orc_kdtree_indices(void* kd, uint32_t* out) {
    KdTree* k = (KdTree*)kd;
    if (!k->prim_indices.empty()) std::memcpy(out, k->prim_indices.data(), k->prim_indices.size() * 4);
}
int64_t orc_kdtree_intersect(void* kd, const orc_ray* rays, uint64_t n, orc_hit* hits, uint32_t* node_visits,
                             uint32_t* prim_tests, int nthreads) {
    const KdTree& k = *(KdTree*)kd;
    return parallel_rays(n, nthreads, [&](uint64_t i) {
        return kd_trace(k, rays[i], true, &hits[i], nullptr, node_visits ? &node_visits[i] : nullptr,
                        prim_tests ? &prim_tests[i] : nullptr);
    });
}
int64_t orc_kdtree_intersect_p(void* kd, const orc_ray* rays, uint64_t n, uint8_t* occluded, uint32_t* node_visits,
                               uint32_t* prim_tests, int nthreads) {
    const KdTree& k = *(KdTree*)kd;
    return parallel_rays(n, nthreads, [&](uint64_t i) {
        return kd_trace(k, rays[i], false, nullptr, &occluded[i], node_visits ? &node_visits[i] : nullptr,
                        prim_tests ? &prim_tests[i] : nullptr);
    });
}

}  // extern "C"
