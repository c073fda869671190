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
        default: return sphere_test(s, r, tmax, t_out, u_out, v_out);
    }
}

}  // namespace ilm
