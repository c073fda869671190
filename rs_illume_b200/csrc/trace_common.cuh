// Device helpers shared by the ray-query kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "illume_gpu.h"
#include "kernels.h"
#include "layout.h"
#include "shapes.cuh"

namespace ilm {

struct RayIn {
    float ox, oy, oz, dx, dy, dz, tmax;
};

__device__ __forceinline__ RayIn load_ray(const ilm_ray* rays, uint64_t i) {
    const float4* p = reinterpret_cast<const float4*>(rays + i);
    float4 a = __ldg(p), b = __ldg(p + 1);
    return {a.x, a.y, a.z, b.x, b.y, b.z, b.w};
}

__device__ __forceinline__ void store_hit(ilm_hit* hits, uint64_t i, uint32_t prim, float t, float u, float v) {
    reinterpret_cast<float4*>(hits)[i] = make_float4(__uint_as_float(prim), t, u, v);
}

__device__ __forceinline__ void write_miss(uint64_t i, const RayIn& r, ilm_hit* hits, uint32_t* occ) {
    if (occ) occ[i] = 0u;
    else store_hit(hits, i, ILM_MISS, r.tmax, 0.0f, 0.0f);
}

__device__ __forceinline__ uint64_t ray_count(const TraceArgs& a) {
    if (a.n_dev) {
        uint64_t m = *a.n_dev;
        return m < a.n ? m : a.n;
    }
    return a.n;
}

// Tests primitive record `r` (index in traversal order).  The shear constants
// of the triangle test are set up on the first primitive a ray reaches.
// kAnalytic = false compiles the triangle test alone, for accels without
// quadric or curve records: the call into the analytic shapes' tests costs a
// kernel registers (spills at the 64-register occupancy target) even when it
// never runs.
template <bool kClosest, bool kAnalytic = true>
__device__ __forceinline__ bool prim_test(const PrimRec* __restrict__ prims, const SphereRec* __restrict__ spheres,
                                          uint32_t r, TriRay& tr, bool& tr_ready, const RayIn& ray, float tmax,
                                          float& t, float& u, float& v, uint32_t& prim_id) {
    const float4* p = reinterpret_cast<const float4*>(prims + r);
    float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    uint32_t flags = __float_as_uint(b.w);
    prim_id = __float_as_uint(a.w);
    if (kAnalytic && (flags & kPrimSphere)) {
        return quadric_test(spheres[__float_as_uint(c.w)], ray.ox, ray.oy, ray.oz, ray.dx, ray.dy, ray.dz,
                            tmax, t, u, v);
    }
    if (kClosest && (flags & kPrimDegenerate)) return false;
    if (!tr_ready) {
        tr = make_tri_ray(ray.ox, ray.oy, ray.oz, ray.dx, ray.dy, ray.dz);
        tr_ready = true;
    }
    return triangle_test(tr, make_float3(a.x, a.y, a.z), make_float3(b.x, b.y, b.z),
                         make_float3(c.x, c.y, c.z), tmax, t, u, v);
}

// A slab distance is NaN exactly when the ray lies in that bounding plane with
// a zero direction component (0 * inf); the slab then does not constrain the
// ray (the reference's comparisons would reject the box and lose hits on
// edges lying in the plane).
__device__ __forceinline__ void unconstrain_nan(float& lo, float& hi) {
    if (isnan(lo)) lo = -INFINITY;
    if (isnan(hi)) hi = INFINITY;
}

// Bounds3::intersect_p with precomputed inv_dir / dir_is_neg
// (geometry/bounds3.rs:284-318), on an explicit box, with NaN slabs
// unconstrained.
__device__ __forceinline__ bool box_intersect_p(float minx, float miny, float minz, float maxx, float maxy,
                                                float maxz, const RayIn& r, float ix, float iy, float iz, bool nx,
                                                bool ny, bool nz, float tmax) {
    float t_min = __fmul_rn(__fsub_rn(nx ? maxx : minx, r.ox), ix);
    float t_max = __fmul_rn(__fsub_rn(nx ? minx : maxx, r.ox), ix);
    float ty_min = __fmul_rn(__fsub_rn(ny ? maxy : miny, r.oy), iy);
    float ty_max = __fmul_rn(__fsub_rn(ny ? miny : maxy, r.oy), iy);
    unconstrain_nan(t_min, t_max);
    unconstrain_nan(ty_min, ty_max);
    t_max = __fmul_rn(t_max, kBoxRobust);
    ty_max = __fmul_rn(ty_max, kBoxRobust);
    if (t_min > ty_max || ty_min > t_max) return false;
    if (ty_min > t_min) t_min = ty_min;
    if (ty_max < t_max) t_max = ty_max;
    float tz_min = __fmul_rn(__fsub_rn(nz ? maxz : minz, r.oz), iz);
    float tz_max = __fmul_rn(__fsub_rn(nz ? minz : maxz, r.oz), iz);
    unconstrain_nan(tz_min, tz_max);
    tz_max = __fmul_rn(tz_max, kBoxRobust);
    if (t_min > tz_max || tz_min > t_max) return false;
    if (tz_min > t_min) t_min = tz_min;
    if (tz_max < t_max) t_max = tz_max;
    return (t_min < tmax) && (t_max > 0.0f);
}

// The root box test a tracer's enters() performs (Bounds3::intersect_p on the
// world bound with the ray's own tmax), for rays not yet in a tracer.
__device__ __forceinline__ bool root_enters(const RayIn& r, const float* b) {
    const float ix = __frcp_rn(r.dx), iy = __frcp_rn(r.dy), iz = __frcp_rn(r.dz);   // == 1/d exactly
    return box_intersect_p(b[0], b[1], b[2], b[3], b[4], b[5], r, ix, iy, iz, ix < 0.0f, iy < 0.0f, iz < 0.0f,
                           r.tmax);
}


}  // namespace ilm
