// Wavefront path tracer on the ray-query kernels.
//
// The estimator is the PBR-book path loop with the reference's one-light
// direct lighting (core/integrator.rs:321-494, with the BSDF-sampled MIS term
// accumulated), Lambertian reflection (reflection/lambertian_reflection.rs:
// f = R/pi, cosine sampling, reflection/mod.rs:300-315), one-sided diffuse
// area lights on emissive triangles (shapes/triangle.rs:616-642, pdf converted
// to solid angle as core/shape.rs:40-83 with |cos|*area in the denominator),
// spawn offsets (geometry/ray.rs:79-102, core/interaction.rs:33-72) and
// Russian roulette q = max(0.05, 1 - max(beta)) from bounce rr_depth.
//
// Paths are processed in waves of P.  Per bounce:
//   extend  closest-hit of the path queue      (persistent trace kernel)
//   shade   emission on the camera segment; light sample -> shadow queue;
//           BSDF sample: if it hits the chosen light's triangle, a visibility
//           ray up to that point -> shadow queue (equivalent to the
//           reference's closest-hit-is-this-light test); continuation with
//           Russian roulette -> next path queue
//   shadow  any-hit of the shadow queue        (persistent trace kernel)
//   accum   unoccluded contributions -> film (float atomics)
// Queues are compacted with a warp ballot, a prefix popcount and one atomicAdd
// per warp.  Queue sizes live in device memory, so a bounce is a fixed launch
// sequence, captured once per queue parity as a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "context.h"
#include "illume_gpu.h"
#include "kernels.h"
#include "pcg32.h"
#include "pt.h"
#include "shapes.cuh"

namespace ilm {
namespace {

// counts[] layout
enum : int { kQ0 = 0, kQ1 = 1, kShadow = 2, kDepth = 3, kTotClosest = 4, kTotShadow = 5, kDropped = 6,
             kNumCounts = 8 };

struct PtArgs {
    const float4* tri;        // 3 per primitive: p0 (w = material), p1, p2
    const float4* mat;        // 2 per material: albedo, emission
    const uint32_t* lights;   // emissive primitive ids
    const float4* light_geo;  // per light: normal (xyz), area (w)
    uint32_t n_lights;
    float* film;              // RGB sums, 3 per pixel
    uint32_t width, height, npix, spp, ns;
    float eye_x, eye_y, eye_z, tan_half, aspect;
    uint32_t max_depth, rr_depth;
    unsigned long long seed;
    ilm_ray* rays[2];
    float4* beta[2];          // throughput rgb, pixel (bits)
    uint2* rng[2];            // PCG state (lo, hi)
    uint32_t* pid[2];         // path id (selects the PCG stream)
    const ilm_hit* hits;
    ilm_ray* srays;
    float4* scontrib;         // contribution rgb, pixel (bits)
    const uint32_t* socc;
    unsigned long long* counts;
};

__device__ __forceinline__ float3 f3(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 normalize3(float3 a) { return a * rsqrtf(dot3(a, a)); }
__device__ __forceinline__ float3 abs3(float3 a) { return make_float3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
__device__ __forceinline__ float max3c(float3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }

__device__ __forceinline__ uint64_t path_seq(unsigned long long seed, uint32_t id) {
    return (seed << 32) ^ (unsigned long long)id;
}

// offset_ray_origin (geometry/ray.rs:79-102)
__device__ __forceinline__ float3 offset_origin(float3 p, float3 perr, float3 n, float3 w) {
    float d = dot3(abs3(n), perr);
    float3 off = n * d;
    if (dot3(w, n) < 0.0f) off = off * -1.0f;
    float3 po = p + off;
    po.x = off.x > 0.0f ? next_up(po.x) : (off.x < 0.0f ? next_down(po.x) : po.x);
    po.y = off.y > 0.0f ? next_up(po.y) : (off.y < 0.0f ? next_down(po.y) : po.y);
    po.z = off.z > 0.0f ? next_up(po.z) : (off.z < 0.0f ? next_down(po.z) : po.z);
    return po;
}

// coordinate_system (geometry/vector3.rs:520-540)
__device__ __forceinline__ void frame(float3 n, float3& s, float3& t) {
    if (fabsf(n.x) > fabsf(n.y)) {
        float l = sqrtf(n.x * n.x + n.z * n.z);
        s = make_float3(-n.z / l, 0.0f, n.x / l);
    } else {
        float l = sqrtf(n.y * n.y + n.z * n.z);
        s = make_float3(0.0f, n.z / l, -n.y / l);
    }
    t = cross3(n, s);
}

// concentric_sample_disk + cosine_sample_hemisphere (core/sampling.rs:210-230, 316-320)
__device__ __forceinline__ float3 cosine_hemisphere(float u0, float u1) {
    float ox = u0 * 2.0f - 1.0f, oy = u1 * 2.0f - 1.0f;
    float dx = 0.0f, dy = 0.0f;
    if (!(ox == 0.0f && oy == 0.0f)) {
        float r, th;
        if (fabsf(ox) > fabsf(oy)) { r = ox; th = (kPiF / 4.0f) * (oy / ox); }
        else { r = oy; th = kPiF / 2.0f - (kPiF / 4.0f) * (ox / oy); }
        float sn, cs;
        sincosf(th, &sn, &cs);
        dx = r * cs;
        dy = r * sn;
    }
    return make_float3(dx, dy, sqrtf(fmaxf(0.0f, 1.0f - dx * dx - dy * dy)));
}

__device__ __forceinline__ float power_heuristic(float f, float g) { return (f * f) / (f * f + g * g); }

__device__ __forceinline__ bool good(float3 c) {
    float y = 0.212671f * c.x + 0.715160f * c.y + 0.072169f * c.z;   // RGBSpectrum::y (spectrum.rs:498-501)
    return isfinite(c.x) && isfinite(c.y) && isfinite(c.z) && y >= 0.0f && (c.x > 0.0f || c.y > 0.0f || c.z > 0.0f);
}

__device__ __forceinline__ void film_add(const PtArgs& a, uint32_t pixel, float3 c) {
    if (!good(c)) return;
    atomicAdd(&a.film[3 * pixel], c.x);
    atomicAdd(&a.film[3 * pixel + 1], c.y);
    atomicAdd(&a.film[3 * pixel + 2], c.z);
}

// Warp-aggregated append: one atomicAdd per warp, slots in lane order.
__device__ __forceinline__ uint32_t warp_append(unsigned long long* counter, bool want) {
    unsigned m = __ballot_sync(0xFFFFFFFFu, want);
    if (m == 0u) return 0u;
    unsigned lane = threadIdx.x & 31u;
    int leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if ((int)lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(m));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    return (uint32_t)base + __popc(m & ((1u << lane) - 1u));
}

__global__ void k_pt_camera(PtArgs a, unsigned long long p0, uint32_t count) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k == 0) {
        a.counts[kQ0] = count;
        a.counts[kQ1] = 0;
        a.counts[kShadow] = 0;
        a.counts[kDepth] = 0;
    }
    if (k >= count) return;
    uint32_t id = (uint32_t)(p0 + k);
    uint32_t pixel = id % a.npix, sample = id / a.npix;
    uint32_t px = pixel % a.width, py = pixel / a.width;
    Pcg32 rng(path_seq(a.seed, id));
    float jx = rng.uniform_float(), jy = rng.uniform_float();
    float fx = (float)px + ((float)(sample % a.ns) + jx) / (float)a.ns;
    float fy = (float)py + ((float)(sample / a.ns) + jy) / (float)a.ns;
    float sx = (fx / (float)a.width * 2.0f - 1.0f) * a.tan_half * a.aspect;
    float sy = (1.0f - fy / (float)a.height * 2.0f) * a.tan_half;
    float3 d = normalize3(make_float3(sx, sy, 1.0f));
    reinterpret_cast<float4*>(a.rays[0])[2 * k] = make_float4(a.eye_x, a.eye_y, a.eye_z, 0.0f);
    reinterpret_cast<float4*>(a.rays[0])[2 * k + 1] = make_float4(d.x, d.y, d.z, INFINITY);
    a.beta[0][k] = make_float4(1.0f, 1.0f, 1.0f, __uint_as_float(pixel));
    a.rng[0][k] = make_uint2((uint32_t)rng.state, (uint32_t)(rng.state >> 32));
    a.pid[0][k] = id;
}

__global__ void __launch_bounds__(256) k_pt_shade(PtArgs a, int cur) {
    const uint32_t n = (uint32_t)a.counts[cur];
    const uint32_t depth = (uint32_t)a.counts[kDepth];
    const int nxt = cur ^ 1;
    const uint32_t stride = gridDim.x * blockDim.x;
    // every lane of a warp runs the same number of iterations (warp_append needs the whole warp)
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
        uint32_t i = base + threadIdx.x;
        bool valid = i < n;
        bool cont = false, push_l = false, push_b = false;
        ilm_ray ray_l, ray_b, ray_c;
        float3 c_l = make_float3(0, 0, 0), c_b = make_float3(0, 0, 0);
        float4 beta_out = make_float4(0, 0, 0, 0);
        uint2 rng_out = make_uint2(0, 0);
        uint32_t id = 0, pixel = 0;
        if (valid) {
            float4 b4 = a.beta[cur][i];
            float3 beta = f3(b4);
            pixel = __float_as_uint(b4.w);
            id = a.pid[cur][i];
            uint2 rs = a.rng[cur][i];
            Pcg32 rng;
            rng.inc = (path_seq(a.seed, id) << 1u) | 1u;
            rng.state = (uint64_t)rs.x | ((uint64_t)rs.y << 32);
            ilm_hit h = a.hits[i];
            const float4* rp = reinterpret_cast<const float4*>(a.rays[cur] + i);
            float4 r1 = rp[1];
            if (h.prim == kHitTraversalError) {
                atomicAdd(&a.counts[kDropped], 1ull);
            } else if (h.prim != ILM_MISS) {
                float4 t0 = a.tri[3 * h.prim], t1 = a.tri[3 * h.prim + 1], t2 = a.tri[3 * h.prim + 2];
                uint32_t m = __float_as_uint(t0.w);
                float3 p0 = f3(t0), p1 = f3(t1), p2 = f3(t2);
                float b1 = h.u, b2 = h.v, b0 = 1.0f - b1 - b2;
                float3 p = p0 * b0 + p1 * b1 + p2 * b2;
                float3 perr = (abs3(p0 * b0) + abs3(p1 * b1) + abs3(p2 * b2)) * 0x1.c0000cp-22f;   // gamma(7)
                float3 nrm = normalize3(cross3(p0 - p2, p1 - p2));
                float3 wo = make_float3(-r1.x, -r1.y, -r1.z);
                float3 albedo = f3(a.mat[2 * m]);
                if (depth == 0) {
                    float3 le = f3(a.mat[2 * m + 1]);
                    if (dot3(nrm, wo) > 0.0f) film_add(a, pixel, beta * le);
                }
                float3 ss, ts;
                frame(nrm, ss, ts);
                float wo_z = dot3(wo, nrm);
                float u_sel = rng.uniform_float();
                float ul0 = rng.uniform_float(), ul1 = rng.uniform_float();
                float us0 = rng.uniform_float(), us1 = rng.uniform_float();
                // a black BSDF (f = 0) casts no visibility rays and ends the path
                const bool black = albedo.x == 0.0f && albedo.y == 0.0f && albedo.z == 0.0f;
                if (a.n_lights > 0 && wo_z != 0.0f && !black) {
                    uint32_t k = min((uint32_t)(u_sel * (float)a.n_lights), a.n_lights - 1u);
                    uint32_t lp_id = a.lights[k];
                    float4 lg = a.light_geo[k];
                    float3 nl = f3(lg);
                    float area = lg.w;
                    float3 q0 = f3(a.tri[3 * lp_id]), q1 = f3(a.tri[3 * lp_id + 1]), q2 = f3(a.tri[3 * lp_id + 2]);
                    float3 le = f3(a.mat[2 * __float_as_uint(a.tri[3 * lp_id].w) + 1]);
                    float nlf = (float)a.n_lights;
                    // light sample (uniform_sample_triangle, sampling.rs:264-267)
                    float su = sqrtf(ul0);
                    float c0 = 1.0f - su, c1 = ul1 * su, c2 = 1.0f - c0 - c1;
                    float3 pl = q0 * c0 + q1 * c1 + q2 * c2;
                    float3 pl_err = (abs3(q0 * c0) + abs3(q1 * c1) + abs3(q2 * c2)) * 0x1.80000ap-22f;   // gamma(6)
                    float3 wi = pl - p;
                    float d2 = dot3(wi, wi);
                    if (d2 > 0.0f) {
                        wi = wi * rsqrtf(d2);
                        float cl = dot3(nl, wi * -1.0f);
                        float light_pdf = d2 / (fabsf(cl) * area);
                        float wi_z = dot3(wi, nrm);
                        bool reflect = wi_z * wo_z > 0.0f;
                        if (cl > 0.0f && isfinite(light_pdf) && light_pdf > 0.0f && reflect) {
                            float scat_pdf = fabsf(wi_z) * (1.0f / kPiF);
                            float w = power_heuristic(light_pdf, scat_pdf);
                            c_l = beta * albedo * le * ((1.0f / kPiF) * fabsf(wi_z) * w / light_pdf * nlf);
                            float3 o = offset_origin(p, perr, nrm, pl - p);
                            float3 tgt = offset_origin(pl, pl_err, nl, o - pl);
                            float3 dd = tgt - o;
                            ray_l = {{o.x, o.y, o.z}, 0.0f, {dd.x, dd.y, dd.z}, 1.0f - 0.0001f};
                            push_l = true;
                        }
                    }
                    // BSDF sample with MIS
                    float3 wl = cosine_hemisphere(us0, us1);
                    if (wo_z < 0.0f) wl.z = -wl.z;
                    float3 wb = ss * wl.x + ts * wl.y + nrm * wl.z;
                    float scat_pdf = fabsf(wl.z) * (1.0f / kPiF);
                    float wb_z = dot3(wb, nrm);
                    if (scat_pdf > 0.0f && wb_z * wo_z > 0.0f) {
                        float3 o = offset_origin(p, perr, nrm, wb);
                        TriRay tr = make_tri_ray(o.x, o.y, o.z, wb.x, wb.y, wb.z);
                        float tl, lb1, lb2;
                        if (triangle_test(tr, q0, q1, q2, INFINITY, tl, lb1, lb2)) {
                            float3 pli = q0 * (1.0f - lb1 - lb2) + q1 * lb1 + q2 * lb2;
                            float3 dv = pli - p;
                            float lpdf = dot3(dv, dv) / (fabsf(dot3(nl, wb)) * area);
                            if (isfinite(lpdf) && lpdf > 0.0f && dot3(nl, wb) < 0.0f) {
                                float w = power_heuristic(scat_pdf, lpdf);
                                c_b = beta * albedo * le * ((1.0f / kPiF) * fabsf(wb_z) * w / scat_pdf * nlf);
                                ray_b = {{o.x, o.y, o.z}, 0.0f, {wb.x, wb.y, wb.z}, tl * (1.0f - 0.0001f)};
                                push_b = true;
                            }
                        }
                    }
                }
                // continuation
                float u0 = rng.uniform_float(), u1 = rng.uniform_float();
                float urr = rng.uniform_float();
                float3 wl = cosine_hemisphere(u0, u1);
                if (wo_z < 0.0f) wl.z = -wl.z;
                float3 wi = ss * wl.x + ts * wl.y + nrm * wl.z;
                float pdf = fabsf(wl.z) * (1.0f / kPiF);
                float wi_z = dot3(wi, nrm);
                if (!black && wo_z != 0.0f && pdf > 0.0f && wi_z * wo_z > 0.0f) {
                    float3 nb = beta * albedo * ((1.0f / kPiF) * fabsf(wi_z) / pdf);
                    bool alive = true;
                    if (depth >= a.rr_depth) {
                        float q = fmaxf(0.05f, 1.0f - max3c(nb));
                        if (urr < q) alive = false;
                        else nb = nb * (1.0f / (1.0f - q));
                    }
                    if (alive && depth + 1 < a.max_depth) {
                        float3 o = offset_origin(p, perr, nrm, wi);
                        ray_c = {{o.x, o.y, o.z}, 0.0f, {wi.x, wi.y, wi.z}, INFINITY};
                        beta_out = make_float4(nb.x, nb.y, nb.z, __uint_as_float(pixel));
                        rng_out = make_uint2((uint32_t)rng.state, (uint32_t)(rng.state >> 32));
                        cont = true;
                    }
                }
            }
        }
        uint32_t slot = warp_append(&a.counts[nxt], cont);
        if (cont) {
            float4* rr = reinterpret_cast<float4*>(a.rays[nxt] + slot);
            rr[0] = make_float4(ray_c.o[0], ray_c.o[1], ray_c.o[2], 0.0f);
            rr[1] = make_float4(ray_c.d[0], ray_c.d[1], ray_c.d[2], ray_c.tmax);
            a.beta[nxt][slot] = beta_out;
            a.rng[nxt][slot] = rng_out;
            a.pid[nxt][slot] = id;
        }
        uint32_t sl = warp_append(&a.counts[kShadow], push_l);
        if (push_l) {
            float4* rr = reinterpret_cast<float4*>(a.srays + sl);
            rr[0] = make_float4(ray_l.o[0], ray_l.o[1], ray_l.o[2], 0.0f);
            rr[1] = make_float4(ray_l.d[0], ray_l.d[1], ray_l.d[2], ray_l.tmax);
            a.scontrib[sl] = make_float4(c_l.x, c_l.y, c_l.z, __uint_as_float(pixel));
        }
        uint32_t sb = warp_append(&a.counts[kShadow], push_b);
        if (push_b) {
            float4* rr = reinterpret_cast<float4*>(a.srays + sb);
            rr[0] = make_float4(ray_b.o[0], ray_b.o[1], ray_b.o[2], 0.0f);
            rr[1] = make_float4(ray_b.d[0], ray_b.d[1], ray_b.d[2], ray_b.tmax);
            a.scontrib[sb] = make_float4(c_b.x, c_b.y, c_b.z, __uint_as_float(pixel));
        }
    }
}

__global__ void k_pt_accum(PtArgs a) {
    const uint32_t n = (uint32_t)a.counts[kShadow];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (a.socc[i] == 0u) {
            float4 c = a.scontrib[i];
            film_add(a, __float_as_uint(c.w), make_float3(c.x, c.y, c.z));
        }
    }
}

__global__ void k_pt_advance(PtArgs a, int cur) {
    a.counts[kTotClosest] += a.counts[cur];
    a.counts[kTotShadow] += a.counts[kShadow];
    a.counts[cur] = 0;
    a.counts[kShadow] = 0;
    a.counts[kDepth] += 1;
}

__global__ void k_pt_resolve(const float* film, float* out, uint32_t n3, float inv_spp) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n3) out[i] = film[i] * inv_spp;
}

}  // namespace
}  // namespace ilm

using namespace ilm;

namespace {

// One bounce: extend, shade, shadow, accumulate, advance (queue parity cur).
cudaError_t bounce(const PtArgs& a, const DeviceAccel& da, const LaunchParams& lp, uint32_t cap, uint32_t* err,
                   int cur, int blocks, cudaStream_t s) {
    cudaError_t e = launch_trace(da, a.rays[cur], cap, const_cast<ilm_hit*>(a.hits), nullptr, err, lp, s,
                                 a.counts + cur);
    if (e != cudaSuccess) return e;
    k_pt_shade<<<blocks, 256, 0, s>>>(a, cur);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    e = launch_trace(da, a.srays, 2ull * cap, nullptr, const_cast<uint32_t*>(a.socc), err, lp, s,
                     a.counts + kShadow);
    if (e != cudaSuccess) return e;
    k_pt_accum<<<blocks, 256, 0, s>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_pt_advance<<<1, 1, 0, s>>>(a, cur);
    return cudaGetLastError();
}

}  // namespace

extern "C" {

int32_t ilm_pt_scene_create(ilm_context* ctx, ilm_accel_id accel, const ilm_pt_scene_desc* desc,
                            ilm_pt_scene_id* out) {
    if (!ctx || !desc || !out) return ILM_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ILM_ERR_CUDA;
    Accel* acc = find_accel(ctx, accel);
    if (!acc) { set_error(ctx, "ilm_pt_scene_create: unknown accel id"); return ILM_ERR_NOT_FOUND; }
    const HostLayout& h = acc->host;
    if (!desc->prim_material || !desc->albedo || !desc->emission || desc->n_materials == 0 || desc->width == 0 ||
        desc->height == 0 || !(desc->fov_deg > 0.0f && desc->fov_deg < 180.0f)) {
        set_error(ctx, "ilm_pt_scene_create: invalid scene description");
        return ILM_ERR_INVALID_ARGUMENT;
    }
    auto sc = std::make_unique<PtScene>();
    sc->accel = accel;
    sc->desc = *desc;
    uint32_t np = h.n_prims;
    std::vector<float> tri(12ull * np, 0.0f);
    for (const PrimRec& r : h.records) {
        if (r.flags & kPrimSphere) {
            set_error(ctx, "ilm_pt_scene_create: path tracing supports triangle meshes only");
            return ILM_ERR_INVALID_ARGUMENT;
        }
        uint32_t m = desc->prim_material[r.prim];
        if (m >= desc->n_materials) {
            set_error(ctx, "ilm_pt_scene_create: material index out of range");
            return ILM_ERR_INVALID_ARGUMENT;
        }
        float* t = &tri[12ull * r.prim];
        std::memcpy(t, r.p0, 12);
        std::memcpy(t + 4, r.p1, 12);
        std::memcpy(t + 8, r.p2, 12);
        std::memcpy(t + 3, &m, 4);
    }
    std::vector<float> mat(8ull * desc->n_materials, 0.0f);
    for (uint32_t m = 0; m < desc->n_materials; ++m)
        for (int k = 0; k < 3; ++k) {
            mat[8 * m + k] = desc->albedo[3 * m + k];
            mat[8 * m + 4 + k] = desc->emission[3 * m + k];
        }
    std::vector<uint32_t> lights;
    std::vector<float> lgeo;
    for (uint32_t p = 0; p < np; ++p) {
        uint32_t m = desc->prim_material[p];
        const float* e = desc->emission + 3 * m;
        if (!(e[0] > 0.0f || e[1] > 0.0f || e[2] > 0.0f)) continue;
        const float* t = &tri[12ull * p];
        double a[3] = {t[4] - t[0], t[5] - t[1], t[6] - t[2]}, b[3] = {t[8] - t[0], t[9] - t[1], t[10] - t[2]};
        double c[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
        double l = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
        if (l == 0.0) continue;
        lights.push_back(p);
        // n = normalize((p1-p0) x (p2-p0)) (triangle.rs:625), area = |.|/2 (triangle.rs:609-614)
        lgeo.insert(lgeo.end(), {(float)(c[0] / l), (float)(c[1] / l), (float)(c[2] / l), (float)(0.5 * l)});
    }
    sc->n_lights = (uint32_t)lights.size();
    if (cudaError_t e = sc->d_tri.reserve(tri.size() * 4); e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    if (cudaError_t e = sc->d_mat.reserve(mat.size() * 4); e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    if (np) cudaMemcpy(sc->d_tri.ptr, tri.data(), tri.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(sc->d_mat.ptr, mat.data(), mat.size() * 4, cudaMemcpyHostToDevice);
    if (!lights.empty()) {
        if (cudaError_t e = sc->d_lights.reserve(lights.size() * 4); e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
        if (cudaError_t e = sc->d_light_geo.reserve(lgeo.size() * 4); e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
        cudaMemcpy(sc->d_lights.ptr, lights.data(), lights.size() * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(sc->d_light_geo.ptr, lgeo.data(), lgeo.size() * 4, cudaMemcpyHostToDevice);
    }
    if (cudaError_t e = cudaGetLastError(); e != cudaSuccess) return cuda_fail(ctx, e, "ilm_pt_scene_create");
    ilm_pt_scene_id id = ctx->next_pt++;
    ctx->pt_scenes[id] = std::move(sc);
    *out = id;
    return ILM_OK;
}

int32_t ilm_render_pt(ilm_context* ctx, ilm_pt_scene_id scene, const ilm_pt_opts* opts, float* rgb_out,
                      ilm_pt_stats* stats) {
    if (!ctx || !opts || !rgb_out) return ILM_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ILM_ERR_CUDA;
    auto it = ctx->pt_scenes.find(scene);
    if (it == ctx->pt_scenes.end()) { set_error(ctx, "ilm_render_pt: unknown scene id"); return ILM_ERR_NOT_FOUND; }
    PtScene& sc = *it->second;
    Accel* acc = find_accel(ctx, sc.accel);
    if (!acc) { set_error(ctx, "ilm_render_pt: the scene's accel was destroyed"); return ILM_ERR_NOT_FOUND; }
    const ilm_pt_scene_desc& d = sc.desc;
    uint32_t ns = (uint32_t)std::lround(std::sqrt((double)opts->spp));
    if (opts->spp == 0 || ns * ns != opts->spp || opts->max_depth == 0) {
        set_error(ctx, "ilm_render_pt: spp must be a non-zero perfect square and max_depth >= 1");
        return ILM_ERR_INVALID_ARGUMENT;
    }
    const uint64_t npix = (uint64_t)d.width * d.height;
    const uint64_t total = npix * opts->spp;
    if (total >= (1ull << 32)) { set_error(ctx, "ilm_render_pt: more than 2^32 paths"); return ILM_ERR_INVALID_ARGUMENT; }
    uint32_t P = opts->wave_paths ? opts->wave_paths : (1u << 21);
    if ((uint64_t)P > total) P = (uint32_t)total;
    // buffers
    PtBuffers& b = sc.buf;
    auto rsv = [&](DeviceBuffer& db, size_t bytes) { return db.reserve(bytes); };
    cudaError_t e = cudaSuccess;
    for (int q = 0; q < 2 && e == cudaSuccess; ++q) {
        if ((e = rsv(b.rays[q], (size_t)P * sizeof(ilm_ray))) != cudaSuccess) break;
        if ((e = rsv(b.beta[q], (size_t)P * 16)) != cudaSuccess) break;
        if ((e = rsv(b.rng[q], (size_t)P * 8)) != cudaSuccess) break;
        e = rsv(b.pid[q], (size_t)P * 4);
    }
    if (e == cudaSuccess) e = rsv(b.hits, (size_t)P * sizeof(ilm_hit));
    if (e == cudaSuccess) e = rsv(b.srays, (size_t)2 * P * sizeof(ilm_ray));
    if (e == cudaSuccess) e = rsv(b.scontrib, (size_t)2 * P * 16);
    if (e == cudaSuccess) e = rsv(b.socc, (size_t)2 * P * 4);
    if (e == cudaSuccess) e = rsv(b.counts, kNumCounts * 8);
    if (e == cudaSuccess) e = rsv(b.film, npix * 12);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "ilm_render_pt buffers");
    if (!b.stream) {
        if ((e = cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking)) != cudaSuccess)
            return cuda_fail(ctx, e, "cudaStreamCreate");
        cudaEventCreate(&b.ev0);
        cudaEventCreate(&b.ev1);
    }
    cudaStream_t s = b.stream;
    PtArgs a;
    a.tri = static_cast<const float4*>(sc.d_tri.ptr);
    a.mat = static_cast<const float4*>(sc.d_mat.ptr);
    a.lights = static_cast<const uint32_t*>(sc.d_lights.ptr);
    a.light_geo = static_cast<const float4*>(sc.d_light_geo.ptr);
    a.n_lights = sc.n_lights;
    a.film = static_cast<float*>(b.film.ptr);
    a.width = d.width; a.height = d.height; a.npix = (uint32_t)npix; a.spp = opts->spp; a.ns = ns;
    a.eye_x = d.eye[0]; a.eye_y = d.eye[1]; a.eye_z = d.eye[2];
    a.tan_half = std::tan(0.5f * d.fov_deg * 3.14159265358979323846f / 180.0f);
    a.aspect = (float)d.width / (float)d.height;
    a.max_depth = opts->max_depth; a.rr_depth = opts->rr_depth; a.seed = opts->seed;
    for (int q = 0; q < 2; ++q) {
        a.rays[q] = static_cast<ilm_ray*>(b.rays[q].ptr);
        a.beta[q] = static_cast<float4*>(b.beta[q].ptr);
        a.rng[q] = static_cast<uint2*>(b.rng[q].ptr);
        a.pid[q] = static_cast<uint32_t*>(b.pid[q].ptr);
    }
    a.hits = static_cast<const ilm_hit*>(b.hits.ptr);
    a.srays = static_cast<ilm_ray*>(b.srays.ptr);
    a.scontrib = static_cast<float4*>(b.scontrib.ptr);
    a.socc = static_cast<const uint32_t*>(b.socc.ptr);
    a.counts = static_cast<unsigned long long*>(b.counts.ptr);
    DeviceAccel da = acc->view();
    unsigned long long* counter = ctx->counter_for(s);
    if (!counter) return ILM_ERR_OUT_OF_MEMORY;
    LaunchParams lp{ctx->stack_depth, ctx->block_size, ctx->max_iter, 1, counter,
                    (ctx->flags & ILM_FLAG_HIGH_OCCUPANCY) ? 8 : 0};
    uint32_t* err = static_cast<uint32_t*>(ctx->err_word.ptr);
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, ctx->device);
    const int blocks = dev_sms * 8;

    cudaMemsetAsync(a.counts, 0, kNumCounts * 8, s);
    cudaMemsetAsync(a.film, 0, npix * 12, s);
    // graphs: one per queue parity, captured on first use for this buffer set
    cudaGraphExec_t graphs[2] = {nullptr, nullptr};
    if (opts->use_graphs) {
        // One eager bounce over empty queues (every kernel returns at once)
        // does the launchers' one-time setup outside the capture.
        if ((e = bounce(a, da, lp, P, err, 0, blocks, s)) != cudaSuccess) return cuda_fail(ctx, e, "bounce");
        for (int q = 0; q < 2; ++q) {
            cudaGraph_t g;
            if ((e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
                return cuda_fail(ctx, e, "cudaStreamBeginCapture");
            cudaError_t eb = bounce(a, da, lp, P, err, q, blocks, s);
            e = cudaStreamEndCapture(s, &g);
            if (eb != cudaSuccess) return cuda_fail(ctx, eb, "bounce capture");
            if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&graphs[q], g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGraphInstantiate");
        }
    }
    cudaEventRecord(b.ev0, s);
    uint32_t waves = 0;
    for (uint64_t p0 = 0; p0 < total; p0 += P, ++waves) {
        uint32_t cnt = (uint32_t)(total - p0 < P ? total - p0 : P);
        k_pt_camera<<<(cnt + 255) / 256, 256, 0, s>>>(a, p0, cnt);
        for (uint32_t depth = 0; depth < opts->max_depth; ++depth) {
            int cur = depth & 1;
            if (opts->use_graphs) e = cudaGraphLaunch(graphs[cur], s);
            else e = bounce(a, da, lp, P, err, cur, blocks, s);
            if (e != cudaSuccess) break;
        }
        if (e != cudaSuccess) break;
    }
    cudaEventRecord(b.ev1, s);
    for (auto& g : graphs) if (g) cudaGraphExecDestroy(g);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "ilm_render_pt launch");
    // resolve into the output (device) or a device temp then copy (host)
    PtrKind k = classify(rgb_out);
    float* dst = rgb_out;
    if (k == PtrKind::kHost) {
        if ((e = b.out.reserve(npix * 12)) != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc(out)");
        dst = static_cast<float*>(b.out.ptr);
    }
    uint32_t n3 = (uint32_t)(npix * 3);
    k_pt_resolve<<<(n3 + 255) / 256, 256, 0, s>>>(a.film, dst, n3, 1.0f / (float)opts->spp);
    if (k == PtrKind::kHost) cudaMemcpyAsync(rgb_out, dst, npix * 12, cudaMemcpyDeviceToHost, s);
    unsigned long long cnts[kNumCounts];
    cudaMemcpyAsync(cnts, a.counts, sizeof cnts, cudaMemcpyDeviceToHost, s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(ctx, e, "ilm_render_pt");
    if (stats) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, b.ev0, b.ev1);
        stats->closest_rays = cnts[kTotClosest];
        stats->shadow_rays = cnts[kTotShadow];
        stats->seconds = ms * 1e-3;
        stats->waves = waves;
    }
    // cnts[kTotClosest/kTotShadow] accumulate over the waves of this call only:
    // the counters are cleared at the start of every render.
    if (cnts[kDropped]) {
        set_error(ctx, "ilm_render_pt: some paths reached the traversal limits and were dropped");
        return ILM_ERR_TRAVERSAL_LIMIT;
    }
    return ILM_OK;
}

}  // extern "C"
