// SurfaceInteraction reconstruction for closest hits: what Triangle::intersect
// builds after its hit test (shapes/triangle.rs:264-415) through
// SurfaceInteraction::new and set_shading_geometry (core/interaction.rs:262-339).
//
// One thread per (ray, hit).  The barycentrics are recomputed with the
// traversal's own watertight test (so b0 = e0/det is the reference's, not
// 1 - b1 - b2), and every expression rounds as the Rust source does:
// round-to-nearest intrinsics (no contraction), cross products in double
// (Vector3::cross, geometry/vector3.rs:67-83), normalize as v * (1/length)
// (vector3.rs:85-95), coordinate_system dividing by the length
// (vector3.rs:520-537).
// Repairs: D14 (uv determinant duv02.x*duv12.y - duv02.y*duv12.x) and D27
// (SurfaceInteraction::new keeps Shading::default(); the shading frame starts
// as the geometric one, n, dpdu, dpdv, dndu, dndv, as in pbrt).
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "context.h"
#include "illume_gpu.h"
#include "shapes.cuh"

namespace ilm {
namespace {

constexpr uint32_t kShadeSphere = 0xFFFFFFFFu;
enum : uint32_t { kHasN = 1, kHasS = 2, kHasUV = 4, kReverse = 8 };

struct V3 { float x, y, z; };

__device__ __forceinline__ V3 vadd(V3 a, V3 b) { return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)}; }
__device__ __forceinline__ V3 vsub(V3 a, V3 b) { return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)}; }
__device__ __forceinline__ V3 vmul(float s, V3 a) { return {__fmul_rn(s, a.x), __fmul_rn(s, a.y), __fmul_rn(s, a.z)}; }
__device__ __forceinline__ V3 vneg(V3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ float vdot(V3 a, V3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ float vlen2(V3 a) { return vdot(a, a); }
// Vector3::cross: products and differences in double, rounded to float
__device__ __forceinline__ V3 vcross(V3 a, V3 b) {
    double ax = a.x, ay = a.y, az = a.z, bx = b.x, by = b.y, bz = b.z;
    return {__double2float_rn(__dsub_rn(__dmul_rn(ay, bz), __dmul_rn(az, by))),
            __double2float_rn(__dsub_rn(__dmul_rn(az, bx), __dmul_rn(ax, bz))),
            __double2float_rn(__dsub_rn(__dmul_rn(ax, by), __dmul_rn(ay, bx)))};
}
__device__ __forceinline__ V3 vnormalize(V3 a) { return vmul(__fdiv_rn(1.0f, __fsqrt_rn(vlen2(a))), a); }
__device__ __forceinline__ void coordinate_system(V3 v1, V3& v2, V3& v3) {
    if (fabsf(v1.x) > fabsf(v1.y)) {
        float len = __fsqrt_rn(__fadd_rn(__fmul_rn(v1.x, v1.x), __fmul_rn(v1.z, v1.z)));
        v2 = {__fdiv_rn(-v1.z, len), 0.0f, __fdiv_rn(v1.x, len)};
    } else {
        float len = __fsqrt_rn(__fadd_rn(__fmul_rn(v1.y, v1.y), __fmul_rn(v1.z, v1.z)));
        v2 = {0.0f, __fdiv_rn(v1.z, len), __fdiv_rn(-v1.y, len)};
    }
    v3 = vcross(v1, v2);
}
// b0*a + b1*b + b2*c, summed left to right
__device__ __forceinline__ V3 interp(float b0, float b1, float b2, V3 a, V3 b, V3 c) {
    return vadd(vadd(vmul(b0, a), vmul(b1, b)), vmul(b2, c));
}

struct ShadeArgs {
    const float* vtx;
    const float* nrm;
    const float* tan;
    const float* uv;
    const uint4* tri;
    const uint32_t* mesh;
    uint32_t n_prims;
};

__device__ __forceinline__ V3 load3(const float* a, uint32_t i) { return {a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }
__device__ __forceinline__ void put3(float* d, V3 v) { d[0] = v.x; d[1] = v.y; d[2] = v.z; }

__global__ void k_surface_interactions(ShadeArgs sa, const ilm_ray* __restrict__ rays, const ilm_hit* __restrict__ hits,
                                       uint64_t n, ilm_surface_interaction* __restrict__ out) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ilm_surface_interaction si;
    memset(&si, 0, sizeof si);
    const ilm_ray r = rays[i];
    const ilm_hit h = hits[i];
    si.prim = h.prim;
    si.t = h.t;
    si.kind = ILM_SI_MISS;
    const V3 o{r.o[0], r.o[1], r.o[2]}, d{r.d[0], r.d[1], r.d[2]};
    if (h.prim >= sa.n_prims) {   // miss (or a flagged traversal error)
        out[i] = si;
        return;
    }
    put3(si.wo, vneg(d));
    const uint4 tv = sa.tri[h.prim];
    if (tv.w == kShadeSphere) {
        si.kind = ILM_SI_SPHERE;
        put3(si.p, vadd(o, vmul(h.t, d)));
        out[i] = si;
        return;
    }
    const uint32_t flags = sa.mesh[tv.w];
    const V3 p0 = load3(sa.vtx, tv.x), p1 = load3(sa.vtx, tv.y), p2 = load3(sa.vtx, tv.z);
    // barycentrics of the hit, as the traversal computed them
    TriRay tr = make_tri_ray(o.x, o.y, o.z, d.x, d.y, d.z);
    float t, b0, b1, b2;
    if (!triangle_test(tr, make_float3(p0.x, p0.y, p0.z), make_float3(p1.x, p1.y, p1.z),
                       make_float3(p2.x, p2.y, p2.z), INFINITY, t, b1, b2, &b0)) {
        out[i] = si;   // not a hit of this triangle: left as a miss
        return;
    }
    // uv parameterisation (triangle.rs:96-112; default (0,0), (1,0), (1,1))
    float uv0[2] = {0.0f, 0.0f}, uv1[2] = {1.0f, 0.0f}, uv2[2] = {1.0f, 1.0f};
    if (flags & kHasUV) {
        uv0[0] = sa.uv[2 * tv.x]; uv0[1] = sa.uv[2 * tv.x + 1];
        uv1[0] = sa.uv[2 * tv.y]; uv1[1] = sa.uv[2 * tv.y + 1];
        uv2[0] = sa.uv[2 * tv.z]; uv2[1] = sa.uv[2 * tv.z + 1];
    }
    // partial derivatives (triangle.rs:264-292)
    const float duv02x = __fsub_rn(uv0[0], uv2[0]), duv02y = __fsub_rn(uv0[1], uv2[1]);
    const float duv12x = __fsub_rn(uv1[0], uv2[0]), duv12y = __fsub_rn(uv1[1], uv2[1]);
    const V3 dp02 = vsub(p0, p2), dp12 = vsub(p1, p2);
    const float det = __fsub_rn(__fmul_rn(duv02x, duv12y), __fmul_rn(duv02y, duv12x));
    const bool degenerate_uv = fabsf(det) < 1e-8f;
    V3 dpdu{0, 0, 0}, dpdv{0, 0, 0};
    if (!degenerate_uv) {
        const float invdet = __fdiv_rn(1.0f, det);
        dpdu = vmul(invdet, vsub(vmul(duv12y, dp02), vmul(duv02y, dp12)));
        dpdv = vmul(invdet, vadd(vmul(-duv12x, dp02), vmul(duv02x, dp12)));
    }
    if (degenerate_uv || vlen2(vcross(dpdu, dpdv)) == 0.0f) {
        const V3 ng = vcross(vsub(p2, p0), vsub(p1, p0));
        if (vlen2(ng) == 0.0f) {   // degenerate triangle: the reference reports no hit
            out[i] = si;
            return;
        }
        coordinate_system(vnormalize(ng), dpdu, dpdv);
    }
    // error bound and hit point (triangle.rs:295-305)
    const V3 perr{__fmul_rn(kGamma7, __fadd_rn(__fadd_rn(fabsf(__fmul_rn(b0, p0.x)), fabsf(__fmul_rn(b1, p1.x))),
                                             fabsf(__fmul_rn(b2, p2.x)))),
                  __fmul_rn(kGamma7, __fadd_rn(__fadd_rn(fabsf(__fmul_rn(b0, p0.y)), fabsf(__fmul_rn(b1, p1.y))),
                                             fabsf(__fmul_rn(b2, p2.y)))),
                  __fmul_rn(kGamma7, __fadd_rn(__fadd_rn(fabsf(__fmul_rn(b0, p0.z)), fabsf(__fmul_rn(b1, p1.z))),
                                             fabsf(__fmul_rn(b2, p2.z))))};
    const V3 phit = interp(b0, b1, b2, p0, p1, p2);
    si.uv[0] = __fadd_rn(__fadd_rn(__fmul_rn(b0, uv0[0]), __fmul_rn(b1, uv1[0])), __fmul_rn(b2, uv2[0]));
    si.uv[1] = __fadd_rn(__fadd_rn(__fmul_rn(b0, uv0[1]), __fmul_rn(b1, uv1[1])), __fmul_rn(b2, uv2[1]));
    const bool reverse = (flags & kReverse) != 0;   // world-space meshes: no handedness swap
    // SurfaceInteraction::new (interaction.rs:262-316) then the triangle's
    // normal override (triangle.rs:322-331)
    V3 nrm = vnormalize(vcross(dp02, dp12));
    if (reverse) nrm = vneg(nrm);
    V3 sn = nrm, sdpdu = dpdu, sdpdv = dpdv, sdndu{0, 0, 0}, sdndv{0, 0, 0};
    if (flags & (kHasN | kHasS)) {
        // shading geometry (triangle.rs:333-414)
        V3 ns = nrm;
        if (flags & kHasN) {
            V3 nn = interp(b0, b1, b2, load3(sa.nrm, tv.x), load3(sa.nrm, tv.y), load3(sa.nrm, tv.z));
            if (vlen2(nn) > 0.0f) ns = vnormalize(nn);
        }
        V3 ss = vnormalize(dpdu);
        if (flags & kHasS) {
            V3 s = interp(b0, b1, b2, load3(sa.tan, tv.x), load3(sa.tan, tv.y), load3(sa.tan, tv.z));
            if (vlen2(s) > 0.0f) ss = vnormalize(s);
        }
        V3 ts = vcross(ss, ns);
        if (vlen2(ts) > 0.0f) {
            ts = vnormalize(ts);
            ss = vcross(ts, ns);
        } else {
            coordinate_system(ns, ss, ts);
        }
        V3 dndu{0, 0, 0}, dndv{0, 0, 0};
        if (flags & kHasN) {
            const V3 n0 = load3(sa.nrm, tv.x), n1 = load3(sa.nrm, tv.y), n2 = load3(sa.nrm, tv.z);
            const V3 dn1 = vsub(n0, n2), dn2 = vsub(n1, n2);
            const float det2 = __fsub_rn(__fmul_rn(duv02x, duv12y), __fmul_rn(duv02y, duv12x));
            if (fabsf(det2) < 1e-8f) {
                const V3 dn = vcross(vsub(n2, n0), vsub(n1, n0));
                if (vlen2(dn) != 0.0f) coordinate_system(dn, dndu, dndv);
            } else {
                const float inv = __fdiv_rn(1.0f, det2);
                dndu = vmul(inv, vsub(vmul(duv12y, dn1), vmul(duv02y, dn2)));
                dndv = vmul(inv, vadd(vmul(-duv12x, dn1), vmul(duv02x, dn2)));
            }
        }
        if (reverse) ts = vneg(ts);
        // set_shading_geometry(ss, ts, dndu, dndv, true) (interaction.rs:318-339)
        sn = vnormalize(vcross(ss, ts));
        if (vdot(nrm, sn) < 0.0f) nrm = vneg(nrm);
        sdpdu = ss; sdpdv = ts; sdndu = dndu; sdndv = dndv;
    }
    si.kind = ILM_SI_TRIANGLE;
    si.t = t;
    put3(si.p, phit); put3(si.p_error, perr); put3(si.n, nrm);
    put3(si.dpdu, dpdu); put3(si.dpdv, dpdv);
    put3(si.shading_n, sn); put3(si.shading_dpdu, sdpdu); put3(si.shading_dpdv, sdpdv);
    put3(si.shading_dndu, sdndu); put3(si.shading_dndv, sdndv);
    out[i] = si;
}

// Builds the accel's shading data from its meshes (once).
int32_t ensure_shading(ilm_context* ctx, Accel& acc) {
    ShadingData& sd = acc.shading;
    if (sd.ready) return ILM_OK;
    std::vector<float> vtx, nrm, tan, uv;
    std::vector<uint4> tri;
    std::vector<uint32_t> mesh;
    for (size_t k = 0; k < acc.mesh_ids.size(); ++k) {
        auto it = ctx->meshes.find(acc.mesh_ids[k]);
        if (it == ctx->meshes.end()) { set_error(ctx, "surface interactions: a mesh of the accel is gone"); return ILM_ERR_NOT_FOUND; }
        const Mesh& m = *it->second;
        if (m.is_spheres) {
            for (uint32_t p = 0; p < m.n_prims; ++p) tri.push_back(make_uint4(0, 0, 0, kShadeSphere));
            continue;
        }
        const uint32_t base = (uint32_t)(vtx.size() / 3), nv = (uint32_t)(m.xyz.size() / 3);
        vtx.insert(vtx.end(), m.xyz.begin(), m.xyz.end());
        auto append = [&](std::vector<float>& dst, const std::vector<float>& src, size_t per) {
            if (src.empty()) dst.resize(dst.size() + per * nv, 0.0f);
            else dst.insert(dst.end(), src.begin(), src.end());
        };
        append(nrm, m.n, 3);
        append(tan, m.s, 3);
        append(uv, m.uv, 2);
        uint32_t flags = (m.n.empty() ? 0u : (uint32_t)kHasN) | (m.s.empty() ? 0u : (uint32_t)kHasS) |
                         (m.uv.empty() ? 0u : (uint32_t)kHasUV) | (m.reverse ? (uint32_t)kReverse : 0u);
        const uint32_t slot = (uint32_t)mesh.size();
        mesh.push_back(flags);
        for (uint32_t p = 0; p < m.n_prims; ++p)
            tri.push_back(make_uint4(base + m.idx[3 * p], base + m.idx[3 * p + 1], base + m.idx[3 * p + 2], slot));
    }
    if (mesh.empty()) mesh.push_back(0);
    if (vtx.empty()) { vtx.resize(3, 0.0f); nrm.resize(3, 0.0f); tan.resize(3, 0.0f); uv.resize(2, 0.0f); }
    if (tri.empty()) tri.push_back(make_uint4(0, 0, 0, kShadeSphere));
    cudaError_t e;
    struct Up { DeviceBuffer& b; const void* src; size_t bytes; } ups[] = {
        {sd.vtx, vtx.data(), vtx.size() * 4}, {sd.nrm, nrm.data(), nrm.size() * 4}, {sd.tan, tan.data(), tan.size() * 4},
        {sd.uv, uv.data(), uv.size() * 4},    {sd.tri, tri.data(), tri.size() * 16}, {sd.mesh, mesh.data(), mesh.size() * 4}};
    for (auto& u : ups) {
        if ((e = u.b.reserve(u.bytes)) != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc(shading)");
        if ((e = cudaMemcpy(u.b.ptr, u.src, u.bytes, cudaMemcpyHostToDevice)) != cudaSuccess)
            return cuda_fail(ctx, e, "cudaMemcpy(shading)");
    }
    sd.ready = true;
    return ILM_OK;
}

}  // namespace
}  // namespace ilm

using namespace ilm;

extern "C" int32_t ilm_surface_interactions(ilm_context* ctx, ilm_accel_id accel, const ilm_ray* rays,
                                            const ilm_hit* hits, uint64_t n, ilm_surface_interaction* out,
                                            void* stream) {
    if (!ctx || (n && (!rays || !hits || !out))) return ILM_ERR_INVALID_ARGUMENT;
    if (n == 0) return ILM_OK;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ILM_ERR_CUDA;
    Accel* acc = find_accel(ctx, accel);
    if (!acc) { set_error(ctx, "ilm_surface_interactions: unknown accel id"); return ILM_ERR_NOT_FOUND; }
    int32_t st = ensure_shading(ctx, *acc);
    if (st != ILM_OK) return st;
    PtrKind kr = classify(rays), kh = classify(hits), ko = classify(out);
    if (kr != kh || kr != ko) {
        set_error(ctx, "ilm_surface_interactions: rays, hits and output must all be host or all device memory");
        return ILM_ERR_INVALID_ARGUMENT;
    }
    const ShadingData& sd = acc->shading;
    ShadeArgs sa{static_cast<const float*>(sd.vtx.ptr), static_cast<const float*>(sd.nrm.ptr),
                 static_cast<const float*>(sd.tan.ptr),  static_cast<const float*>(sd.uv.ptr),
                 static_cast<const uint4*>(sd.tri.ptr),  static_cast<const uint32_t*>(sd.mesh.ptr),
                 acc->host.n_prims};
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    cudaError_t e;
    const unsigned block = 128;
    if (kr == PtrKind::kDevice) {
        k_surface_interactions<<<(unsigned)((n + block - 1) / block), block, 0, s>>>(sa, rays, hits, n, out);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "k_surface_interactions");
        return ILM_OK;
    }
    DeviceBuffer dr, dh, dout;
    if ((e = dr.reserve(n * sizeof(ilm_ray))) != cudaSuccess || (e = dh.reserve(n * sizeof(ilm_hit))) != cudaSuccess ||
        (e = dout.reserve(n * sizeof(ilm_surface_interaction))) != cudaSuccess)
        return cuda_fail(ctx, e, "cudaMalloc(surface interactions)");
    cudaMemcpyAsync(dr.ptr, rays, n * sizeof(ilm_ray), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dh.ptr, hits, n * sizeof(ilm_hit), cudaMemcpyHostToDevice, s);
    k_surface_interactions<<<(unsigned)((n + block - 1) / block), block, 0, s>>>(
        sa, static_cast<const ilm_ray*>(dr.ptr), static_cast<const ilm_hit*>(dh.ptr), n,
        static_cast<ilm_surface_interaction*>(dout.ptr));
    cudaMemcpyAsync(out, dout.ptr, n * sizeof(ilm_surface_interaction), cudaMemcpyDeviceToHost, s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(ctx, e, "ilm_surface_interactions");
    return ILM_OK;
}
