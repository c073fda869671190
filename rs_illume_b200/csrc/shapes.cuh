// Device-side shape tests.  Every floating-point step is written with an
// explicit round-to-nearest intrinsic (__fadd_rn, __fmul_rn, __fdiv_rn, ...),
// which the compiler never fuses into FMA, so each expression rounds exactly
// as the reference's Rust source (Rust does not contract a*b+c).  The
// results are therefore bit-identical to the reference's arithmetic.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "layout.h"

namespace ilm {

// gamma(n) = n*eps / (1 - n*eps), eps = 2^-24 (core/pbrt.rs:172-174),
// evaluated in f32 exactly as the reference does.
constexpr float kGamma2 = 0x1.000002p-23f;
constexpr float kGamma3 = 0x1.800004p-23f;
constexpr float kGamma5 = 0x1.400006p-22f;
constexpr float kGamma7 = 0x1.c0000cp-22f;
// 1 + 2*gamma(3): far-plane scale of Bounds3::intersect_p (bounds3.rs:292-307)
constexpr float kBoxRobust = 0x1.000006p+0f;
constexpr float kMachineEps = 0x1p-24f;
constexpr float kPiF = 3.14159265358979323846f;

// Per-ray constants of the watertight test (triangle.rs:162-185), computed
// once per ray; the reference recomputes the same values per triangle.
struct TriRay {
    float ox, oy, oz;   // origin, permuted (kx, ky, kz)
    float sx, sy, sz;   // shear constants
    int kz;
};

__device__ __forceinline__ float3 permute3(float x, float y, float z, int kz) {
    // kz = 2: (x,y,z); kz = 0: (y,z,x); kz = 1: (z,x,y)  (kx = kz+1, ky = kx+1 mod 3)
    float a = kz == 0 ? y : (kz == 1 ? z : x);
    float b = kz == 0 ? z : (kz == 1 ? x : y);
    float c = kz == 0 ? x : (kz == 1 ? y : z);
    return make_float3(a, b, c);
}

__device__ __forceinline__ TriRay make_tri_ray(float ox, float oy, float oz, float dx, float dy, float dz) {
    TriRay r;
    float ax = fabsf(dx), ay = fabsf(dy), az = fabsf(dz);
    // Vector3::max_dimension (geometry/vector3.rs:140-150)
    r.kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    float3 d = permute3(dx, dy, dz, r.kz);
    float3 o = permute3(ox, oy, oz, r.kz);
    r.ox = o.x; r.oy = o.y; r.oz = o.z;
    r.sx = __fdiv_rn(-d.x, d.z);
    r.sy = __fdiv_rn(-d.y, d.z);
    r.sz = __fdiv_rn(1.0f, d.z);
    return r;
}

__device__ __forceinline__ float max3f(float a, float b, float c) { return fmaxf(fmaxf(a, b), c); }

// Watertight ray-triangle test: Triangle::intersect / intersect_p
// (shapes/triangle.rs:156-262 and 435-541).  Returns true with t and
// barycentrics b1, b2 (and b0 when asked) on a hit with 0 < t and t_scaled
// within tmax.
__device__ __forceinline__ bool triangle_test(const TriRay& r, float3 p0, float3 p1, float3 p2,
                                              float tmax, float& t_out, float& b1_out,
                                              float& b2_out, float* b0_out = nullptr) {
    // translate + permute (157-174)
    float3 a = permute3(p0.x, p0.y, p0.z, r.kz);
    float3 b = permute3(p1.x, p1.y, p1.z, r.kz);
    float3 c = permute3(p2.x, p2.y, p2.z, r.kz);
    a.x = __fsub_rn(a.x, r.ox); a.y = __fsub_rn(a.y, r.oy); a.z = __fsub_rn(a.z, r.oz);
    b.x = __fsub_rn(b.x, r.ox); b.y = __fsub_rn(b.y, r.oy); b.z = __fsub_rn(b.z, r.oz);
    c.x = __fsub_rn(c.x, r.ox); c.y = __fsub_rn(c.y, r.oy); c.z = __fsub_rn(c.z, r.oz);
    // shear (180-185)
    a.x = __fadd_rn(a.x, __fmul_rn(r.sx, a.z)); a.y = __fadd_rn(a.y, __fmul_rn(r.sy, a.z));
    b.x = __fadd_rn(b.x, __fmul_rn(r.sx, b.z)); b.y = __fadd_rn(b.y, __fmul_rn(r.sy, b.z));
    c.x = __fadd_rn(c.x, __fmul_rn(r.sx, c.z)); c.y = __fadd_rn(c.y, __fmul_rn(r.sy, c.z));
    // edge functions (188-190)
    float e0 = __fsub_rn(__fmul_rn(b.x, c.y), __fmul_rn(b.y, c.x));
    float e1 = __fsub_rn(__fmul_rn(c.x, a.y), __fmul_rn(c.y, a.x));
    float e2 = __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x));
    // double-precision recomputation at edges (193-204); products of two
    // floats are exact in double, so only the difference rounds.
    if (e0 == 0.0f || e1 == 0.0f || e2 == 0.0f) {
        e0 = __double2float_rn(__dsub_rn(__dmul_rn((double)c.y, (double)b.x), __dmul_rn((double)c.x, (double)b.y)));
        e1 = __double2float_rn(__dsub_rn(__dmul_rn((double)a.y, (double)c.x), __dmul_rn((double)a.x, (double)c.y)));
        e2 = __double2float_rn(__dsub_rn(__dmul_rn((double)b.y, (double)a.x), __dmul_rn((double)b.x, (double)a.y)));
    }
    // edge-sign and determinant tests (207-215)
    if ((e0 < 0.0f || e1 < 0.0f || e2 < 0.0f) && (e0 > 0.0f || e1 > 0.0f || e2 > 0.0f)) return false;
    float det = __fadd_rn(__fadd_rn(e0, e1), e2);
    if (det == 0.0f) return false;
    // scaled distance and range test (218-229)
    float az = __fmul_rn(a.z, r.sz), bz = __fmul_rn(b.z, r.sz), cz = __fmul_rn(c.z, r.sz);
    float ts = __fadd_rn(__fadd_rn(__fmul_rn(e0, az), __fmul_rn(e1, bz)), __fmul_rn(e2, cz));
    float tmd = __fmul_rn(tmax, det);
    if (det < 0.0f && (ts >= 0.0f || ts < tmd)) return false;
    if (det > 0.0f && (ts <= 0.0f || ts > tmd)) return false;
    // barycentrics and t (232-236)
    float inv_det = __fdiv_rn(1.0f, det);
    float t = __fmul_rn(ts, inv_det);
    // conservative t > 0 check (241-262), with max_component taken as the true
    // maximum (geometry/vector3.rs:106-111 returns the wrong component when
    // x > y but z > x)
    float max_zt = max3f(fabsf(az), fabsf(bz), fabsf(cz));
    float delta_z = __fmul_rn(kGamma3, max_zt);
    float max_xt = max3f(fabsf(a.x), fabsf(b.x), fabsf(c.x));
    float max_yt = max3f(fabsf(a.y), fabsf(b.y), fabsf(c.y));
    float delta_x = __fmul_rn(kGamma5, __fadd_rn(max_xt, max_zt));
    float delta_y = __fmul_rn(kGamma5, __fadd_rn(max_yt, max_zt));
    float delta_e = __fmul_rn(2.0f, __fadd_rn(__fadd_rn(__fmul_rn(__fmul_rn(kGamma2, max_xt), max_yt),
                                                        __fmul_rn(delta_y, max_xt)),
                                              __fmul_rn(delta_x, max_yt)));
    float max_e = max3f(fabsf(e0), fabsf(e1), fabsf(e2));
    float delta_t = __fmul_rn(
        __fmul_rn(3.0f, __fadd_rn(__fadd_rn(__fmul_rn(__fmul_rn(kGamma3, max_e), max_zt),
                                            __fmul_rn(delta_e, max_zt)),
                                  __fmul_rn(delta_z, max_e))),
        fabsf(inv_det));
    if (t <= delta_t) return false;
    t_out = t;
    b1_out = __fmul_rn(e1, inv_det);
    b2_out = __fmul_rn(e2, inv_det);
    if (b0_out) *b0_out = __fmul_rn(e0, inv_det);
    return true;
}

// ------------------------------------------------------------------ EFloat
// Interval float of core/efloat.rs:5-257.  Scalar constants enter as exact
// intervals (efloat.rs:123-195 uses the value itself as the error bound, which
// makes `* -0.5` produce low > high; pbrt-v3 uses an exact constant).
struct EF { float v, lo, hi; };

__device__ __forceinline__ float next_up(float v) {       // core/pbrt.rs:129-147
    if (isinf(v) && v > 0.0f) return v;
    if (v == -0.0f) v = 0.0f;
    uint32_t u = __float_as_uint(v);
    u = v >= 0.0f ? u + 1u : u - 1u;
    return __uint_as_float(u);
}
__device__ __forceinline__ float next_down(float v) {     // core/pbrt.rs:151-169
    if (isinf(v) && v < 0.0f) return v;
    if (v == 0.0f) v = -0.0f;
    uint32_t u = __float_as_uint(v);
    u = v > 0.0f ? u - 1u : u + 1u;
    return __uint_as_float(u);
}
__device__ __forceinline__ EF ef_new(float v, float err) {
    if (err == 0.0f) return {v, v, v};
    return {v, next_down(__fsub_rn(v, err)), next_up(__fadd_rn(v, err))};
}
__device__ __forceinline__ EF ef_add(EF a, EF b) {
    return {__fadd_rn(a.v, b.v), next_down(__fadd_rn(a.lo, b.lo)), next_up(__fadd_rn(a.hi, b.hi))};
}
__device__ __forceinline__ EF ef_sub(EF a, EF b) {
    return {__fsub_rn(a.v, b.v), next_down(__fsub_rn(a.lo, b.lo)), next_up(__fsub_rn(a.hi, b.hi))};
}
__device__ __forceinline__ EF ef_mul(EF a, EF b) {
    float p0 = __fmul_rn(a.lo, b.lo), p1 = __fmul_rn(a.hi, b.lo), p2 = __fmul_rn(a.lo, b.hi),
          p3 = __fmul_rn(a.hi, b.hi);
    return {__fmul_rn(a.v, b.v), next_down(fminf(fminf(fminf(p0, p1), p2), p3)),
            next_up(fmaxf(fmaxf(fmaxf(p0, p1), p2), p3))};
}
__device__ __forceinline__ EF ef_div(EF a, EF b) {
    if (b.lo < 0.0f && b.hi > 0.0f) return {__fdiv_rn(a.v, b.v), -INFINITY, INFINITY};
    float d0 = __fdiv_rn(a.lo, b.lo), d1 = __fdiv_rn(a.hi, b.lo), d2 = __fdiv_rn(a.lo, b.hi),
          d3 = __fdiv_rn(a.hi, b.hi);
    return {__fdiv_rn(a.v, b.v), next_down(fminf(fminf(fminf(d0, d1), d2), d3)),
            next_up(fmaxf(fmaxf(fmaxf(d0, d1), d2), d3))};
}

// A ray in a quadric's object space with its error bounds:
// Transform::transform_ray_with_error (core/transform.rs:392-435).
struct ObjRay {
    float ox, oy, oz, oex, oey, oez;   // origin and its error
    float dx, dy, dz, dex, dey, dez;   // direction and its error
};

__device__ __forceinline__ ObjRay xform_ray(const float* m, float rox, float roy, float roz, float rdx, float rdy,
                                           float rdz) {
    // transform_point_with_error (transform.rs:224-247)
    float xp = __fadd_rn(__fadd_rn(__fmul_rn(m[0], rox), __fmul_rn(m[1], roy)), __fadd_rn(__fmul_rn(m[2], roz), m[3]));
    float yp = __fadd_rn(__fadd_rn(__fmul_rn(m[4], rox), __fmul_rn(m[5], roy)), __fadd_rn(__fmul_rn(m[6], roz), m[7]));
    float zp = __fadd_rn(__fadd_rn(__fmul_rn(m[8], rox), __fmul_rn(m[9], roy)), __fadd_rn(__fmul_rn(m[10], roz), m[11]));
    float wp = __fadd_rn(__fadd_rn(__fmul_rn(m[12], rox), __fmul_rn(m[13], roy)), __fadd_rn(__fmul_rn(m[14], roz), m[15]));
    float xs = __fadd_rn(__fadd_rn(__fadd_rn(fabsf(__fmul_rn(m[0], rox)), fabsf(__fmul_rn(m[1], roy))), fabsf(__fmul_rn(m[2], roz))), fabsf(m[3]));
    float ys = __fadd_rn(__fadd_rn(__fadd_rn(fabsf(__fmul_rn(m[4], rox)), fabsf(__fmul_rn(m[5], roy))), fabsf(__fmul_rn(m[6], roz))), fabsf(m[7]));
    float zs = __fadd_rn(__fadd_rn(__fadd_rn(fabsf(__fmul_rn(m[8], rox)), fabsf(__fmul_rn(m[9], roy))), fabsf(__fmul_rn(m[10], roz))), fabsf(m[11]));
    float oex = __fmul_rn(xs, kGamma3), oey = __fmul_rn(ys, kGamma3), oez = __fmul_rn(zs, kGamma3);
    float ox, oy, oz;
    if (wp == 1.0f) { ox = xp; oy = yp; oz = zp; }
    else { ox = __fdiv_rn(xp, wp); oy = __fdiv_rn(yp, wp); oz = __fdiv_rn(zp, wp); }
    // transform_vector_with_error (transform.rs:296-309)
    float dex = __fmul_rn(kGamma3, __fadd_rn(__fadd_rn(fabsf(__fmul_rn(m[0], rdx)), fabsf(__fmul_rn(m[1], rdy))), fabsf(__fmul_rn(m[2], rdz))));
    float dey = __fmul_rn(kGamma3, __fadd_rn(__fadd_rn(fabsf(__fmul_rn(m[4], rdx)), fabsf(__fmul_rn(m[5], rdy))), fabsf(__fmul_rn(m[6], rdz))));
    float dez = __fmul_rn(kGamma3, __fadd_rn(__fadd_rn(fabsf(__fmul_rn(m[8], rdx)), fabsf(__fmul_rn(m[9], rdy))), fabsf(__fmul_rn(m[10], rdz))));
    float dx = __fadd_rn(__fadd_rn(__fmul_rn(m[0], rdx), __fmul_rn(m[1], rdy)), __fmul_rn(m[2], rdz));
    float dy = __fadd_rn(__fadd_rn(__fmul_rn(m[4], rdx), __fmul_rn(m[5], rdy)), __fmul_rn(m[6], rdz));
    float dz = __fadd_rn(__fadd_rn(__fmul_rn(m[8], rdx), __fmul_rn(m[9], rdy)), __fmul_rn(m[10], rdz));
    float ls = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    if (ls > 0.0f) {
        float dt = __fdiv_rn(__fadd_rn(__fadd_rn(__fmul_rn(fabsf(dx), oex), __fmul_rn(fabsf(dy), oey)), __fmul_rn(fabsf(dz), oez)), ls);
        ox = __fadd_rn(ox, __fmul_rn(dx, dt));
        oy = __fadd_rn(oy, __fmul_rn(dy, dt));
        oz = __fadd_rn(oz, __fmul_rn(dz, dt));
    }
    return ObjRay{ox, oy, oz, oex, oey, oez, dx, dy, dz, dex, dey, dez};
}

// EFloat quadratic (efloat.rs:232-257): false without real roots; t0 <= t1.
__device__ __forceinline__ bool ef_quadratic(EF a, EF b, EF c, EF& t0, EF& t1) {
    double disc = __dsub_rn(__dmul_rn((double)b.v, (double)b.v), __dmul_rn(__dmul_rn(4.0, (double)a.v), (double)c.v));
    if (disc < 0.0) return false;
    double root = __dsqrt_rn(disc);
    float fr = __double2float_rn(root);
    EF froot = ef_new(fr, __fmul_rn(kMachineEps, fr));
    EF half = EF{-0.5f, -0.5f, -0.5f};
    EF q = (b.v < 0.0f) ? ef_mul(ef_sub(b, froot), half) : ef_mul(ef_add(b, froot), half);
    t0 = ef_div(q, a);
    t1 = ef_div(c, q);
    if (t0.v > t1.v) { EF sw = t0; t0 = t1; t1 = sw; }
    return true;
}

// Nearest root within (0, tmax] (sphere.rs:135-144; the same lines in
// cylinder.rs and cone.rs).
__device__ __forceinline__ bool nearest_root(const EF& t0, const EF& t1, float tmax, EF& th) {
    if (t0.hi > tmax || t1.lo <= 0.0f) return false;
    th = t0;
    if (th.lo <= 0.0f) {
        th = t1;
        if (th.hi > tmax) return false;
    }
    return true;
}

__device__ __forceinline__ float phi_of(float y, float x) {
    float phi = atan2f(y, x);
    if (phi < 0.0f) phi = __fadd_rn(phi, 2.0f * kPiF);
    return phi;
}

// Sphere::intersect / intersect_p (shapes/sphere.rs:105-188, 238-323).  The
// refine step uses the Euclidean distance (point3.rs:62-66 computes sqrt of a
// dot product instead).  Returns t and the parametric (u, v).
__device__ __forceinline__ bool sphere_test(const SphereRec& s, const ObjRay& r, float tmax, float& t_out,
                                            float& u_out, float& v_out) {
    const float ox = r.ox, oy = r.oy, oz = r.oz, dx = r.dx, dy = r.dy, dz = r.dz;
    // quadratic coefficients (sphere.rs:116-126)
    EF eox = ef_new(ox, r.oex), eoy = ef_new(oy, r.oey), eoz = ef_new(oz, r.oez);
    EF edx = ef_new(dx, r.dex), edy = ef_new(dy, r.dey), edz = ef_new(dz, r.dez);
    EF a = ef_add(ef_add(ef_mul(edx, edx), ef_mul(edy, edy)), ef_mul(edz, edz));
    EF b = ef_mul(ef_add(ef_add(ef_mul(edx, eox), ef_mul(edy, eoy)), ef_mul(edz, eoz)), EF{2.0f, 2.0f, 2.0f});
    EF rr = EF{s.radius, s.radius, s.radius};
    EF c = ef_sub(ef_add(ef_add(ef_mul(eox, eox), ef_mul(eoy, eoy)), ef_mul(eoz, eoz)), ef_mul(rr, rr));
    EF t0, t1, th;
    if (!ef_quadratic(a, b, c, t0, t1)) return false;
    if (!nearest_root(t0, t1, tmax, th)) return false;
    float px, py, pz, phi;
    auto hit_point = [&](float t) {
        px = __fadd_rn(ox, __fmul_rn(dx, t));
        py = __fadd_rn(oy, __fmul_rn(dy, t));
        pz = __fadd_rn(oz, __fmul_rn(dz, t));
        float dist = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(px, px), __fmul_rn(py, py)), __fmul_rn(pz, pz)));
        float k = __fdiv_rn(s.radius, dist);
        px = __fmul_rn(px, k); py = __fmul_rn(py, k); pz = __fmul_rn(pz, k);
        if (px == 0.0f && py == 0.0f) px = __fmul_rn(1e-5f, s.radius);
        phi = phi_of(py, px);
    };
    auto clipped = [&]() {
        return (s.z_min > -s.radius && pz < s.z_min) || (s.z_max < s.radius && pz > s.z_max) || phi > s.phi_max;
    };
    hit_point(th.v);
    if (clipped()) {
        if (th.v == t1.v) return false;
        if (t1.hi > tmax) return false;
        th = t1;
        hit_point(th.v);
        if (clipped()) return false;
    }
    float zr = fminf(fmaxf(__fdiv_rn(pz, s.radius), -1.0f), 1.0f);
    float theta = acosf(zr);
    t_out = th.v;
    u_out = __fdiv_rn(phi, s.phi_max);
    v_out = __fdiv_rn(__fsub_rn(theta, s.theta_min), __fsub_rn(s.theta_max, s.theta_min));
    return true;
}

// Disk::intersect / intersect_p (disk.rs:110-166, 168-203): the plane
// z = height, then the radii and phi_max.  Disk records keep the height in
// z_min (= z_max) and the inner radius in theta_min.
__device__ __forceinline__ bool disk_test(const SphereRec& s, const ObjRay& r, float tmax, float& t_out,
                                          float& u_out, float& v_out) {
    const float height = s.z_min, inner = s.theta_min;
    if (r.dz == 0.0f) return false;
    float t = __fdiv_rn(__fsub_rn(height, r.oz), r.dz);
    if (t <= 0.0f || t >= tmax) return false;
    float px = __fadd_rn(r.ox, __fmul_rn(r.dx, t)), py = __fadd_rn(r.oy, __fmul_rn(r.dy, t));
    float dist2 = __fadd_rn(__fmul_rn(px, px), __fmul_rn(py, py));
    if (dist2 > __fmul_rn(s.radius, s.radius) || dist2 < __fmul_rn(inner, inner)) return false;
    float phi = phi_of(py, px);
    if (phi > s.phi_max) return false;
    float r_hit = __fsqrt_rn(dist2);
    t_out = t;
    u_out = __fdiv_rn(phi, s.phi_max);
    v_out = __fdiv_rn(__fsub_rn(s.radius, r_hit), __fsub_rn(s.radius, inner));
    return true;
}

// Cylinder::intersect / intersect_p (cylinder.rs:77-...): x^2 + y^2 = r^2,
// the hit refined onto the radius, clipped by z and phi (retry with t1).
__device__ __forceinline__ bool cylinder_test(const SphereRec& s, const ObjRay& r, float tmax, float& t_out,
                                              float& u_out, float& v_out) {
    EF eox = ef_new(r.ox, r.oex), eoy = ef_new(r.oy, r.oey);
    EF edx = ef_new(r.dx, r.dex), edy = ef_new(r.dy, r.dey);
    EF a = ef_add(ef_mul(edx, edx), ef_mul(edy, edy));
    EF b = ef_mul(ef_add(ef_mul(edx, eox), ef_mul(edy, eoy)), EF{2.0f, 2.0f, 2.0f});
    EF rr = EF{s.radius, s.radius, s.radius};
    EF c = ef_sub(ef_add(ef_mul(eox, eox), ef_mul(eoy, eoy)), ef_mul(rr, rr));
    EF t0, t1, th;
    if (!ef_quadratic(a, b, c, t0, t1)) return false;
    if (!nearest_root(t0, t1, tmax, th)) return false;
    float px, py, pz, phi;
    auto hit_point = [&](float t) {
        px = __fadd_rn(r.ox, __fmul_rn(r.dx, t));
        py = __fadd_rn(r.oy, __fmul_rn(r.dy, t));
        pz = __fadd_rn(r.oz, __fmul_rn(r.dz, t));
        float hit_rad = __fsqrt_rn(__fadd_rn(__fmul_rn(px, px), __fmul_rn(py, py)));
        px = __fmul_rn(px, __fdiv_rn(s.radius, hit_rad));
        py = __fmul_rn(py, __fdiv_rn(s.radius, hit_rad));
        phi = phi_of(py, px);
    };
    auto clipped = [&]() { return pz < s.z_min || pz > s.z_max || phi > s.phi_max; };
    hit_point(th.v);
    if (clipped()) {
        if (th.v == t1.v) return false;
        if (t1.hi > tmax) return false;
        th = t1;
        hit_point(th.v);
        if (clipped()) return false;
    }
    t_out = th.v;
    u_out = __fdiv_rn(phi, s.phi_max);
    v_out = __fdiv_rn(__fsub_rn(pz, s.z_min), __fsub_rn(s.z_max, s.z_min));
    return true;
}

// Cone::intersect / intersect_p (cone.rs:91-...): x^2 + y^2 = k (z - h)^2,
// k = (r / h)^2, clipped by 0 <= z <= h and phi (retry with t1).  Cone
// records keep the height in z_max.  b = 2 (dx ox + dy oy - k dz (oz - h))
// (the reference doubles only the last term; repaired as pbrt).
__device__ __forceinline__ bool cone_test(const SphereRec& s, const ObjRay& r, float tmax, float& t_out,
                                          float& u_out, float& v_out) {
    const float height = s.z_max;
    EF eox = ef_new(r.ox, r.oex), eoy = ef_new(r.oy, r.oey), eoz = ef_new(r.oz, r.oez);
    EF edx = ef_new(r.dx, r.dex), edy = ef_new(r.dy, r.dey), edz = ef_new(r.dz, r.dez);
    EF k = ef_div(EF{s.radius, s.radius, s.radius}, EF{height, height, height});
    k = ef_mul(k, k);
    EF ozh = ef_sub(eoz, EF{height, height, height});
    EF a = ef_sub(ef_add(ef_mul(edx, edx), ef_mul(edy, edy)), ef_mul(ef_mul(k, edz), edz));
    EF b = ef_mul(ef_sub(ef_add(ef_mul(edx, eox), ef_mul(edy, eoy)), ef_mul(ef_mul(k, edz), ozh)),
                  EF{2.0f, 2.0f, 2.0f});
    EF c = ef_sub(ef_add(ef_mul(eox, eox), ef_mul(eoy, eoy)), ef_mul(ef_mul(k, ozh), ozh));
    EF t0, t1, th;
    if (!ef_quadratic(a, b, c, t0, t1)) return false;
    if (!nearest_root(t0, t1, tmax, th)) return false;
    float px, py, pz, phi;
    auto hit_point = [&](float t) {
        px = __fadd_rn(r.ox, __fmul_rn(r.dx, t));
        py = __fadd_rn(r.oy, __fmul_rn(r.dy, t));
        pz = __fadd_rn(r.oz, __fmul_rn(r.dz, t));
        phi = phi_of(py, px);
    };
    auto clipped = [&]() { return pz < 0.0f || pz > height || phi > s.phi_max; };
    hit_point(th.v);
    if (clipped()) {
        if (th.v == t1.v) return false;
        if (t1.hi > tmax) return false;
        th = t1;
        hit_point(th.v);
        if (clipped()) return false;
    }
    t_out = th.v;
    u_out = __fdiv_rn(phi, s.phi_max);
    v_out = __fdiv_rn(pz, height);
    return true;
}

// Paraboloid::intersect / intersect_p (paraboloid.rs:95-...):
// k (x^2 + y^2) = z with k = z_max / r^2, clipped by z and phi (retry with t1).
// b = k (dx ox + dy oy) * 2 - dz with the 2 exact.
__device__ __forceinline__ bool paraboloid_test(const SphereRec& s, const ObjRay& r, float tmax, float& t_out,
                                                float& u_out, float& v_out) {
    EF eox = ef_new(r.ox, r.oex), eoy = ef_new(r.oy, r.oey), eoz = ef_new(r.oz, r.oez);
    EF edx = ef_new(r.dx, r.dex), edy = ef_new(r.dy, r.dey), edz = ef_new(r.dz, r.dez);
    EF rr = EF{s.radius, s.radius, s.radius};
    EF k = ef_div(EF{s.z_max, s.z_max, s.z_max}, ef_mul(rr, rr));
    EF a = ef_mul(k, ef_add(ef_mul(edx, edx), ef_mul(edy, edy)));
    EF b = ef_sub(ef_mul(ef_mul(k, ef_add(ef_mul(edx, eox), ef_mul(edy, eoy))), EF{2.0f, 2.0f, 2.0f}), edz);
    EF c = ef_sub(ef_mul(k, ef_add(ef_mul(eox, eox), ef_mul(eoy, eoy))), eoz);
    EF t0, t1, th;
    if (!ef_quadratic(a, b, c, t0, t1)) return false;
    if (!nearest_root(t0, t1, tmax, th)) return false;
    float px, py, pz, phi;
    auto hit_point = [&](float t) {
        px = __fadd_rn(r.ox, __fmul_rn(r.dx, t));
        py = __fadd_rn(r.oy, __fmul_rn(r.dy, t));
        pz = __fadd_rn(r.oz, __fmul_rn(r.dz, t));
        phi = phi_of(py, px);
    };
    auto clipped = [&]() { return pz < s.z_min || pz > s.z_max || phi > s.phi_max; };
    hit_point(th.v);
    if (clipped()) {
        if (th.v == t1.v) return false;
        if (t1.hi > tmax) return false;
        th = t1;
        hit_point(th.v);
        if (clipped()) return false;
    }
    t_out = th.v;
    u_out = __fdiv_rn(phi, s.phi_max);
    v_out = __fdiv_rn(__fsub_rn(pz, s.z_min), __fsub_rn(s.z_max, s.z_min));
    return true;
}

// Hyperboloid::intersect / intersect_p (hyperboloid.rs:128-...):
// ah (x^2 + y^2) - ch z^2 = 1 through p1, p2 (aux[0..5]; ah, ch in aux[6..7]),
// clipped by z and phi, where phi is the angle between the hit and the swept
// point at its height.  Repaired as pbrt: c = ah ox^2 + ah oy^2 - ch oz^2 - 1
// (hyperboloid.rs:149 subtracts oz^2 and ch), and the first phi is
// atan2(pr.x py - px pr.y, px pr.x + py pr.y) (line 169 applies atan2 to pr.y
// alone).
__device__ __forceinline__ bool hyperboloid_test(const SphereRec& s, const ObjRay& r, float tmax, float& t_out,
                                                 float& u_out, float& v_out) {
    const float p1x = s.aux[0], p1y = s.aux[1], p1z = s.aux[2], p2x = s.aux[3], p2y = s.aux[4], p2z = s.aux[5];
    const EF ah = EF{s.aux[6], s.aux[6], s.aux[6]}, ch = EF{s.aux[7], s.aux[7], s.aux[7]};
    EF eox = ef_new(r.ox, r.oex), eoy = ef_new(r.oy, r.oey), eoz = ef_new(r.oz, r.oez);
    EF edx = ef_new(r.dx, r.dex), edy = ef_new(r.dy, r.dey), edz = ef_new(r.dz, r.dez);
    EF a = ef_sub(ef_add(ef_mul(ef_mul(edx, edx), ah), ef_mul(ef_mul(edy, edy), ah)), ef_mul(ef_mul(edz, edz), ch));
    EF b = ef_mul(EF{2.0f, 2.0f, 2.0f}, ef_sub(ef_add(ef_mul(ef_mul(edx, eox), ah), ef_mul(ef_mul(edy, eoy), ah)),
                                                 ef_mul(ef_mul(edz, eoz), ch)));
    EF c = ef_sub(ef_sub(ef_add(ef_mul(ef_mul(eox, eox), ah), ef_mul(ef_mul(eoy, eoy), ah)),
                         ef_mul(ef_mul(eoz, eoz), ch)),
                  EF{1.0f, 1.0f, 1.0f});
    EF t0, t1, th;
    if (!ef_quadratic(a, b, c, t0, t1)) return false;
    if (!nearest_root(t0, t1, tmax, th)) return false;
    float px, py, pz, phi, v;
    auto hit_point = [&](float t) {
        px = __fadd_rn(r.ox, __fmul_rn(r.dx, t));
        py = __fadd_rn(r.oy, __fmul_rn(r.dy, t));
        pz = __fadd_rn(r.oz, __fmul_rn(r.dz, t));
        v = __fdiv_rn(__fsub_rn(pz, p1z), __fsub_rn(p2z, p1z));
        float w = __fsub_rn(1.0f, v);
        float prx = __fadd_rn(__fmul_rn(p1x, w), __fmul_rn(p2x, v));
        float pry = __fadd_rn(__fmul_rn(p1y, w), __fmul_rn(p2y, v));
        phi = phi_of(__fsub_rn(__fmul_rn(prx, py), __fmul_rn(px, pry)),
                     __fadd_rn(__fmul_rn(px, prx), __fmul_rn(py, pry)));
    };
    auto clipped = [&]() { return pz < s.z_min || pz > s.z_max || phi > s.phi_max; };
    hit_point(th.v);
    if (clipped()) {
        if (th.v == t1.v) return false;
        if (t1.hi > tmax) return false;
        th = t1;
        hit_point(th.v);
        if (clipped()) return false;
    }
    t_out = th.v;
    u_out = __fdiv_rn(phi, s.phi_max);
    v_out = v;
    return true;
}

// ------------------------------------------------------------------ curves
// Curve::intersect (shapes/curve.rs:278-375 and recursive_intersect 94-252).
// Curve records (kind kQuadricCurve): aux[0..11] the segment's cubic Bezier
// control points (blossomed on the host for [u_min, u_max]), aux[12..13] the
// curve's widths at u = 0 and 1, aux[14..15] u_min and u_max, aux[16..21] the
// ribbon normals n0, n1 (unit), aux[22] their angle, aux[23] 1 / sin(angle);
// theta_min holds the curve type (0 flat, 1 cylinder, 2 ribbon).  Every
// operation is a round-to-nearest intrinsic, so nothing contracts to an FMA.
struct CP3 {
    float x, y, z;
};
__device__ __forceinline__ CP3 cp_add(CP3 a, CP3 b) { return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)}; }
__device__ __forceinline__ CP3 cp_sub(CP3 a, CP3 b) { return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)}; }
__device__ __forceinline__ CP3 cp_scale(CP3 a, float s) { return {__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)}; }
__device__ __forceinline__ float cp_dot(CP3 a, CP3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
// Vector3::cross in f64 (geometry/vector3.rs:67-83), rounded once to float.
__device__ __forceinline__ CP3 cp_cross(CP3 a, CP3 b) {
    return {__double2float_rn(__dsub_rn(__dmul_rn((double)a.y, (double)b.z), __dmul_rn((double)a.z, (double)b.y))),
            __double2float_rn(__dsub_rn(__dmul_rn((double)a.z, (double)b.x), __dmul_rn((double)a.x, (double)b.z))),
            __double2float_rn(__dsub_rn(__dmul_rn((double)a.x, (double)b.y), __dmul_rn((double)a.y, (double)b.x)))};
}
// Vector3::normalize (vector3.rs:85-95): times 1 / length.
__device__ __forceinline__ CP3 cp_normalize(CP3 a) { return cp_scale(a, __fdiv_rn(1.0f, __fsqrt_rn(cp_dot(a, a)))); }
// lerp(t, a, b) = a (1 - t) + b t (core/pbrt.rs:41-47)
__device__ __forceinline__ float cp_lerpf(float t, float a, float b) {
    return __fadd_rn(__fmul_rn(a, __fsub_rn(1.0f, t)), __fmul_rn(b, t));
}
__device__ __forceinline__ CP3 cp_lerp(float t, CP3 a, CP3 b) {
    return {cp_lerpf(t, a.x, b.x), cp_lerpf(t, a.y, b.y), cp_lerpf(t, a.z, b.z)};
}

// eval_bezier (curve.rs:425-446): the point at u and the derivative.
__device__ __forceinline__ CP3 cp_eval(const CP3* cp, float u, CP3& deriv) {
    CP3 a0 = cp_lerp(u, cp[0], cp[1]), a1 = cp_lerp(u, cp[1], cp[2]), a2 = cp_lerp(u, cp[2], cp[3]);
    CP3 b0 = cp_lerp(u, a0, a1), b1 = cp_lerp(u, a1, a2);
    CP3 db = cp_sub(b1, b0);
    deriv = cp_dot(db, db) > 0.0f ? cp_scale(db, 3.0f) : cp_sub(cp[3], cp[0]);
    return cp_lerp(u, b0, b1);
}

// subdivide_bezier (curve.rs:414-423): the two halves share out[3].
__device__ __forceinline__ void cp_split(const CP3* cp, CP3* out) {
    out[0] = cp[0];
    out[1] = cp_scale(cp_add(cp[0], cp[1]), 0.5f);
    out[2] = cp_scale(cp_add(cp_add(cp[0], cp_scale(cp[1], 2.0f)), cp[2]), 0.25f);
    out[3] = cp_scale(cp_add(cp_add(cp_add(cp[0], cp_scale(cp[1], 3.0f)), cp_scale(cp[2], 3.0f)), cp[3]), 0.125f);
    out[4] = cp_scale(cp_add(cp_add(cp[1], cp_scale(cp[2], 2.0f)), cp[3]), 0.25f);
    out[5] = cp_scale(cp_add(cp[2], cp[3]), 0.5f);
    out[6] = cp[3];
}

// The bound test of a segment against the ray's zero-width beam, padded by
// half the width (curve.rs:116-140).
__device__ __forceinline__ bool cp_overlaps(const CP3* c, float half_w, float z_max) {
    float ymax = fmaxf(fmaxf(c[0].y, c[1].y), fmaxf(c[2].y, c[3].y));
    float ymin = fminf(fminf(c[0].y, c[1].y), fminf(c[2].y, c[3].y));
    if (__fadd_rn(ymax, half_w) < 0.0f || __fsub_rn(ymin, half_w) > 0.0f) return false;
    float xmax = fmaxf(fmaxf(c[0].x, c[1].x), fmaxf(c[2].x, c[3].x));
    float xmin = fminf(fminf(c[0].x, c[1].x), fminf(c[2].x, c[3].x));
    if (__fadd_rn(xmax, half_w) < 0.0f || __fsub_rn(xmin, half_w) > 0.0f) return false;
    float zmax = fmaxf(fmaxf(c[0].z, c[1].z), fmaxf(c[2].z, c[3].z));
    float zmin = fminf(fminf(c[0].z, c[1].z), fminf(c[2].z, c[3].z));
    return !(__fadd_rn(zmax, half_w) < 0.0f || __fsub_rn(zmin, half_w) > z_max);
}

// Integer log2 rounded to nearest for v >= 1, else 0 (curve.rs:340-350).
__device__ __forceinline__ int curve_log2(float v) {
    if (v < 1.0f) return 0;
    uint32_t bits = __float_as_uint(v);
    return (int)(bits >> 23) - 127 + ((bits & (1u << 22)) ? 1 : 0);
}

static __device__ __noinline__ bool curve_test(const SphereRec& s, const ObjRay& r, float tmax, float& t_out,
                                        float& u_out, float& v_out) {
    const CP3 d{r.dx, r.dy, r.dz}, o{r.ox, r.oy, r.oz};
    CP3 obj[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) obj[i] = CP3{s.aux[3 * i], s.aux[3 * i + 1], s.aux[3 * i + 2]};
    const float w0 = s.aux[12], w1 = s.aux[13], u_min = s.aux[14], u_max = s.aux[15];
    const int type = (int)s.theta_min;
    // the ray's frame: z along the ray, y towards the chord (curve.rs:305-320)
    CP3 up = cp_cross(d, cp_sub(obj[3], obj[0]));
    if (cp_dot(up, up) == 0.0f) {   // coordinate_system(d) (vector3.rs:520-545)
        if (fabsf(d.x) > fabsf(d.y)) {
            float len = __fsqrt_rn(__fadd_rn(__fmul_rn(d.x, d.x), __fmul_rn(d.z, d.z)));
            up = CP3{__fdiv_rn(-d.z, len), 0.0f, __fdiv_rn(d.x, len)};
        } else {
            float len = __fsqrt_rn(__fadd_rn(__fmul_rn(d.y, d.y), __fmul_rn(d.z, d.z)));
            up = CP3{0.0f, __fdiv_rn(d.z, len), __fdiv_rn(-d.y, len)};
        }
    }
    // Transform::look_at(o, o + d, up) (transform.rs:181-209); its inverse is
    // applied as the transpose of the orthonormal frame
    CP3 dir = cp_normalize(cp_sub(cp_add(o, d), o));
    CP3 right = cp_normalize(cp_cross(cp_normalize(up), dir));
    CP3 new_up = cp_cross(dir, right);
    CP3 c[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        CP3 q = cp_sub(obj[i], o);
        c[i] = CP3{cp_dot(right, q), cp_dot(new_up, q), cp_dot(dir, q)};
    }
    const float ray_len = __fsqrt_rn(cp_dot(d, d));
    float z_max = __fmul_rn(ray_len, tmax);
    const float max_w = fmaxf(cp_lerpf(u_min, w0, w1), cp_lerpf(u_max, w0, w1));
    if (!cp_overlaps(c, __fmul_rn(0.5f, max_w), z_max)) return false;
    // refinement depth (curve.rs:332-357)
    float l0 = 0.0f;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        float lx = fabsf(__fadd_rn(__fsub_rn(c[i].x, __fmul_rn(2.0f, c[i + 1].x)), c[i + 2].x));
        float ly = fabsf(__fadd_rn(__fsub_rn(c[i].y, __fmul_rn(2.0f, c[i + 1].y)), c[i + 2].y));
        float lz = fabsf(__fadd_rn(__fsub_rn(c[i].z, __fmul_rn(2.0f, c[i + 1].z)), c[i + 2].z));
        l0 = fmaxf(l0, fmaxf(fmaxf(lx, ly), lz));
    }
    const float eps = __fmul_rn(fmaxf(w0, w1), 0.05f);
    int r0 = curve_log2(__fdiv_rn(__fmul_rn(__fmul_rn(1.41421356237f, 6.0f), l0), __fmul_rn(8.0f, eps))) / 2;
    const int max_depth = r0 < 0 ? 0 : (r0 > 10 ? 10 : r0);
    // depth-first over the halves, first half first; the nearest hit of the
    // whole curve is kept (curve.rs:146-153 keeps the last one found)
    struct Seg {
        CP3 cp[4];
        float u0, u1;
        int depth;
    };
    Seg stack[11];
    int sp = 0;
    stack[sp++] = Seg{{c[0], c[1], c[2], c[3]}, u_min, u_max, max_depth};
    bool hit = false;
    while (sp > 0) {
        Seg g = stack[--sp];
        if (g.depth > 0) {
            CP3 sp7[7];
            cp_split(g.cp, sp7);
            const float um = __fmul_rn(__fadd_rn(g.u0, g.u1), 0.5f);
            const float us[3] = {g.u0, um, g.u1};
            for (int seg = 1; seg >= 0; --seg) {   // pushed second half first
                const CP3* cps = sp7 + 3 * seg;
                float mw = fmaxf(cp_lerpf(us[seg], w0, w1), cp_lerpf(us[seg + 1], w0, w1));
                if (!cp_overlaps(cps, __fmul_rn(0.5f, mw), z_max)) continue;
                stack[sp++] = Seg{{cps[0], cps[1], cps[2], cps[3]}, us[seg], us[seg + 1], g.depth - 1};
            }
            continue;
        }
        const CP3* cp = g.cp;
        // the sample point must lie between the end tangents' perpendiculars
        float edge = __fadd_rn(__fmul_rn(__fsub_rn(cp[1].y, cp[0].y), -cp[0].y),
                               __fmul_rn(cp[0].x, __fsub_rn(cp[0].x, cp[1].x)));
        if (edge < 0.0f) continue;
        edge = __fadd_rn(__fmul_rn(__fsub_rn(cp[2].y, cp[3].y), -cp[3].y), __fmul_rn(cp[3].x, __fsub_rn(cp[3].x, cp[2].x)));
        if (edge < 0.0f) continue;
        const float sdx = __fsub_rn(cp[3].x, cp[0].x), sdy = __fsub_rn(cp[3].y, cp[0].y);
        const float denom = __fadd_rn(__fmul_rn(sdx, sdx), __fmul_rn(sdy, sdy));
        if (denom == 0.0f) continue;
        const float w = __fdiv_rn(__fadd_rn(__fmul_rn(-cp[0].x, sdx), __fmul_rn(-cp[0].y, sdy)), denom);
        const float u = fminf(fmaxf(cp_lerpf(w, g.u0, g.u1), g.u0), g.u1);
        float hit_w = cp_lerpf(u, w0, w1);
        if (type == 2) {   // ribbon: the width seen along the ray
            // parallel normals (angle 0) keep n0 instead of 0 * inf weights
            CP3 nh = CP3{s.aux[16], s.aux[17], s.aux[18]};
            if (s.aux[22] != 0.0f) {
                float sin0 = __fmul_rn(sinf(__fmul_rn(__fsub_rn(1.0f, u), s.aux[22])), s.aux[23]);
                float sin1 = __fmul_rn(sinf(__fmul_rn(u, s.aux[22])), s.aux[23]);
                nh = cp_add(cp_scale(nh, sin0), cp_scale(CP3{s.aux[19], s.aux[20], s.aux[21]}, sin1));
            }
            hit_w = __fmul_rn(hit_w, __fdiv_rn(fabsf(cp_dot(nh, d)), ray_len));
        }
        CP3 dpcdw;
        const CP3 pc = cp_eval(cp, fminf(fmaxf(w, 0.0f), 1.0f), dpcdw);
        const float dist2 = __fadd_rn(__fmul_rn(pc.x, pc.x), __fmul_rn(pc.y, pc.y));
        if (dist2 > __fmul_rn(__fmul_rn(hit_w, hit_w), 0.25f)) continue;
        if (pc.z < 0.0f || pc.z > z_max) continue;
        const float dist = __fsqrt_rn(dist2);
        const float edge_fn = __fadd_rn(__fmul_rn(dpcdw.x, -pc.y), __fmul_rn(pc.x, dpcdw.y));
        const float v = edge_fn > 0.0f ? __fadd_rn(0.5f, __fdiv_rn(dist, hit_w)) : __fsub_rn(0.5f, __fdiv_rn(dist, hit_w));
        const float t = __fdiv_rn(pc.z, ray_len);
        if (!hit || t < t_out) {
            t_out = t;
            u_out = u;
            v_out = v;
            hit = true;
            z_max = pc.z;   // later segments must come nearer
        }
    }
    return hit;
}

// The quadric record's test (SphereRec::kind), in its object space.
static __device__ __noinline__ bool quadric_test(const SphereRec& s, float rox, float roy, float roz, float rdx,
                                                 float rdy, float rdz, float tmax, float& t_out, float& u_out,
                                                 float& v_out) {
    const ObjRay r = xform_ray(s.w2o, rox, roy, roz, rdx, rdy, rdz);
    switch (s.kind) {
        case kQuadricDisk: return disk_test(s, r, tmax, t_out, u_out, v_out);
        case kQuadricCylinder: return cylinder_test(s, r, tmax, t_out, u_out, v_out);
        case kQuadricCone: return cone_test(s, r, tmax, t_out, u_out, v_out);
        case kQuadricParaboloid: return paraboloid_test(s, r, tmax, t_out, u_out, v_out);
        case kQuadricHyperboloid: return hyperboloid_test(s, r, tmax, t_out, u_out, v_out);
        case kQuadricCurve: return curve_test(s, r, tmax, t_out, u_out, v_out);
        default: return sphere_test(s, r, tmax, t_out, u_out, v_out);
    }
}

}  // namespace ilm
