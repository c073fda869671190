// Wavefront path tracer on the ray-query kernels, with an optional neural
// radiance cache.
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
//
// Radiance-cache mode (kNrc): each path tracks its spread
//   a0 = d1^2 / (4 pi |cos1|),  s_n = sum_{i=2..n} sqrt(d_i^2 / (pdf_{i-1} |cos_i|)),
// and a rendering path ends at vertex n >= 1 once s_n^2 > c * a0: the cache's
// prediction at that vertex, times the path throughput, replaces the rest of
// the path.  Training paths (one in `train_stride`) never end early; every
// vertex they reach records its cache inputs and 1/throughput, and each
// unoccluded contribution c of the path adds c / beta_k to the target of
// every earlier vertex k: the target is the reflected radiance the rest of the
// path estimated there.  After the wave the queries are answered in one
// batch and the network takes one training step on the recorded vertices.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "context.h"
#include "illume_gpu.h"
#include "kernels.h"
#include "nrc.h"
#include "pcg32.h"
#include "pt.h"
#include "shapes.cuh"

namespace ilm {
namespace {

// counts[] layout
enum : int { kQ0 = 0, kQ1 = 1, kShadow = 2, kDepth = 3, kTotClosest = 4, kTotShadow = 5, kDropped = 6,
             kQueries = 7, kTrainSlots = 8, kSamples = 9, kTotQueries = 10, kTotSamples = 11, kFrame = 12,
             kTrainRows = 13,   // samples gathered by the last frame (kept across renders; trained next frame)
             kNumCounts = 16 };
constexpr uint32_t kNone = 0xFFFFFFFFu;
// A training path's word: slot (bits 0-23) and the vertices it still goes on
// for past the point where a rendering path would end (bits 24-30;
// kNotReached before that point).  Rendering paths hold kNone.
constexpr uint32_t kSlotMask = 0xFFFFFFu, kNotReached = 0x7Fu;
constexpr int kRec = 18;   // training vertex: inputs (12), 1/beta (3), target (3)
constexpr uint32_t kMinTrainStride = 16;   // at most one path in 16 trains (the rest use the cache)

struct PtArgs {
    const float4* tri;        // 3 per primitive: p0 (w = material), p1, p2
    const float4* mat;        // 2 per material: albedo, emission
    const uint32_t* lights;   // emissive primitive ids
    const float4* light_geo;  // per light: normal (xyz), area (w)
    uint32_t n_lights;
    float* film;              // RGB sums, 3 per pixel
    float* wsum;              // filter weight sums per pixel (general filters only)
    const float* ftable;      // the film's 16 x 16 filter weight table (film.rs:70-82)
    float frx, fry, firx, firy;   // filter radius and its inverse
    int fbox;                 // 1: box of radius 0.5, each sample to its own pixel with weight 1
    uint32_t width, height, npix, spp, ns;
    float eye_x, eye_y, eye_z, tan_half, aspect;
    float cam[9];                  // camera-to-world 3x3, row-major
    uint32_t max_depth, rr_depth;
    unsigned long long seed;
    ilm_ray* rays[2];
    float4* beta[2];          // throughput rgb, path id (bits)
    uint2* rng[2];            // PCG state (lo, hi)
    uint32_t* pid[2];         // path id (selects the PCG stream)
    const ilm_hit* hits;
    ilm_ray* srays;
    float4* scontrib;         // contribution rgb, path id (bits)
    const uint32_t* socc;
    unsigned long long* counts;
    // radiance-cache mode
    float4* spread[2];        // s, a0, pdf of the last direction, training word (bits)
    float* q_in;              // queries: 12 floats each
    float4* q_beta;           // throughput rgb, path id (bits)
    uint2* q_train;           // training slot (or kNone) and depth of the query vertex
    const float* q_out;       // predictions: 3 floats each
    uint32_t q_cap;
    float* t_rec;             // [slot][depth][kRec]
    uint32_t* t_count;        // vertices recorded per slot
    uint32_t t_cap, train_stride;   // one path in train_stride trains (0: none)
    uint32_t train_suffix;          // vertices a training path goes on for past the rendering end
    float spread_c;
    uint2* s_train;           // per shadow entry: training slot, depth
    float* t_in;              // gathered training inputs (12 each)
    float* t_tg;              // gathered training targets (3 each)
    uint32_t sample_cap;
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

// Raster position of path `id`'s camera sample: pixel, ns x ns stratum and
// the first two draws of the path's PCG stream (the camera kernel draws the
// same two numbers first).
__device__ __forceinline__ void sample_position(const PtArgs& a, uint32_t id, float& fx, float& fy) {
    uint32_t pixel = id % a.npix, sample = (id / a.npix) % a.spp;
    uint32_t px = pixel % a.width, py = pixel / a.width;
    Pcg32 rng(path_seq(a.seed, id));
    float jx = rng.uniform_float(), jy = rng.uniform_float();
    fx = (float)px + ((float)(sample % a.ns) + jx) / (float)a.ns;
    fy = (float)py + ((float)(sample / a.ns) + jy) / (float)a.ns;
}

// FilmTile::add_sample (film.rs:288-333, D20 repaired: the footprint's upper
// corner is floor(p + radius) + 1 and both loops run): every pixel within the
// filter radius of the sample gets weight table[ify][ifx] (the table at the
// pixel's offset), times c, or only the weight with weight_only.
__device__ __forceinline__ void splat(const PtArgs& a, float fx, float fy, float3 c, bool weight_only) {
    const float dx = __fsub_rn(fx, 0.5f), dy = __fsub_rn(fy, 0.5f);
    int x0 = (int)ceilf(__fsub_rn(dx, a.frx)), y0 = (int)ceilf(__fsub_rn(dy, a.fry));
    int x1 = (int)floorf(__fadd_rn(dx, a.frx)) + 1, y1 = (int)floorf(__fadd_rn(dy, a.fry)) + 1;
    x0 = max(x0, 0); y0 = max(y0, 0);
    x1 = min(x1, (int)a.width); y1 = min(y1, (int)a.height);
    for (int y = y0; y < y1; ++y) {
        int ify = min((int)floorf(fabsf(__fmul_rn(__fmul_rn(__fsub_rn((float)y, dy), a.firy), 16.0f))), 15);
        for (int x = x0; x < x1; ++x) {
            int ifx = min((int)floorf(fabsf(__fmul_rn(__fmul_rn(__fsub_rn((float)x, dx), a.firx), 16.0f))), 15);
            float w = a.ftable[ify * 16 + ifx];
            size_t p = (size_t)y * a.width + x;
            if (weight_only) {
                atomicAdd(&a.wsum[p], w);
            } else {
                atomicAdd(&a.film[3 * p], __fmul_rn(c.x, w));
                atomicAdd(&a.film[3 * p + 1], __fmul_rn(c.y, w));
                atomicAdd(&a.film[3 * p + 2], __fmul_rn(c.z, w));
            }
        }
    }
}

// A contribution c of path `id` to the film.
__device__ __forceinline__ void film_add(const PtArgs& a, uint32_t id, float3 c) {
    if (!good(c)) return;
    if (a.fbox) {
        uint32_t pixel = id % a.npix;
        atomicAdd(&a.film[3 * pixel], c.x);
        atomicAdd(&a.film[3 * pixel + 1], c.y);
        atomicAdd(&a.film[3 * pixel + 2], c.z);
        return;
    }
    float fx, fy;
    sample_position(a, id, fx, fy);
    splat(a, fx, fy, c, false);
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

__device__ __forceinline__ void put_ray(ilm_ray* q, uint32_t slot, float3 o, float3 d, float tmax) {
    float4* rr = reinterpret_cast<float4*>(q + slot);
    rr[0] = make_float4(o.x, o.y, o.z, 0.0f);
    rr[1] = make_float4(d.x, d.y, d.z, tmax);
}

template <bool kNrc>
__global__ void k_pt_camera(PtArgs a, unsigned long long p0, uint32_t count) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k == 0) {
        a.counts[kQ0] = count;
        a.counts[kQ1] = 0;
        a.counts[kShadow] = 0;
        a.counts[kDepth] = 0;
    }
    const bool valid = k < count;
    uint32_t frame = 0;
    if (kNrc) {   // frame f renders path ids f * count ... (the frame counter lives in counts[])
        frame = (uint32_t)a.counts[kFrame];
        p0 = (unsigned long long)frame * count;
    }
    const uint32_t id = (uint32_t)(p0 + k);
    uint32_t tw = kNone;
    if (kNrc) {
        // kQueries, kTrainSlots and kSamples were zeroed before this launch
        bool train = valid && a.train_stride && (id % a.train_stride) == frame % a.train_stride;
        uint32_t s = warp_append(&a.counts[kTrainSlots], train);
        if (train && s < a.t_cap) { tw = s | (kNotReached << 24); a.t_count[s] = 0; }
    }
    if (!valid) return;
    uint32_t pixel = id % a.npix, sample = (id / a.npix) % a.spp;
    uint32_t px = pixel % a.width, py = pixel / a.width;
    Pcg32 rng(path_seq(a.seed, id));
    float jx = rng.uniform_float(), jy = rng.uniform_float();
    float fx = (float)px + ((float)(sample % a.ns) + jx) / (float)a.ns;
    float fy = (float)py + ((float)(sample / a.ns) + jy) / (float)a.ns;
    float sx = (fx / (float)a.width * 2.0f - 1.0f) * a.tan_half * a.aspect;
    float sy = (1.0f - fy / (float)a.height * 2.0f) * a.tan_half;
    float3 c = normalize3(make_float3(sx, sy, 1.0f));
    // camera-to-world (exact for the identity: 1*x + 0*y + 0*z == x)
    float3 d = make_float3(__fadd_rn(__fadd_rn(__fmul_rn(a.cam[0], c.x), __fmul_rn(a.cam[1], c.y)), __fmul_rn(a.cam[2], c.z)),
                           __fadd_rn(__fadd_rn(__fmul_rn(a.cam[3], c.x), __fmul_rn(a.cam[4], c.y)), __fmul_rn(a.cam[5], c.z)),
                           __fadd_rn(__fadd_rn(__fmul_rn(a.cam[6], c.x), __fmul_rn(a.cam[7], c.y)), __fmul_rn(a.cam[8], c.z)));
    put_ray(a.rays[0], k, make_float3(a.eye_x, a.eye_y, a.eye_z), d, INFINITY);
    a.beta[0][k] = make_float4(1.0f, 1.0f, 1.0f, __uint_as_float(id));
    if (!a.fbox) splat(a, fx, fy, make_float3(0.0f, 0.0f, 0.0f), true);   // the sample's filter weights
    a.rng[0][k] = make_uint2((uint32_t)rng.state, (uint32_t)(rng.state >> 32));
    a.pid[0][k] = id;
    if (kNrc) a.spread[0][k] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(tw));
}

template <bool kNrc>
__global__ void __launch_bounds__(256) k_pt_shade(PtArgs a, int cur) {
    const uint32_t n = (uint32_t)a.counts[cur];
    const uint32_t depth = (uint32_t)a.counts[kDepth];
    const int nxt = cur ^ 1;
    const uint32_t stride = gridDim.x * blockDim.x;
    // every lane of a warp runs the same number of iterations (warp_append needs the whole warp)
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
        uint32_t i = base + threadIdx.x;
        bool valid = i < n;
        bool cont = false, push_l = false, push_b = false, query = false;
        float3 o_l, d_l, o_b, d_b, o_c, d_c;
        float tm_l = 0.0f, tm_b = 0.0f;
        float3 c_l = make_float3(0, 0, 0), c_b = make_float3(0, 0, 0);
        float4 beta_out = make_float4(0, 0, 0, 0), spread_next = make_float4(0, 0, 0, 0);
        uint2 rng_out = make_uint2(0, 0);
        uint32_t id = 0, fid = 0, tw = kNone;
        float3 q_p, q_wo, q_n, q_alb, q_beta;
        if (valid) {
            float4 b4 = a.beta[cur][i];
            float3 beta = f3(b4);
            fid = __float_as_uint(b4.w);
            id = a.pid[cur][i];
            uint2 rs = a.rng[cur][i];
            Pcg32 rng;
            rng.inc = (path_seq(a.seed, id) << 1u) | 1u;
            rng.state = (uint64_t)rs.x | ((uint64_t)rs.y << 32);
            float4 sp = kNrc ? a.spread[cur][i] : make_float4(0, 0, 0, 0);
            if (kNrc) tw = __float_as_uint(sp.w);
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
                    if (dot3(nrm, wo) > 0.0f) film_add(a, fid, beta * le);
                }
                float wo_z = dot3(wo, nrm);
                bool cache_here = false;
                if (kNrc) {
                    float cosv = fmaxf(fabsf(wo_z), 1e-6f);
                    float t2 = h.t * h.t;
                    if (depth == 0) { sp.x = 0.0f; sp.y = t2 / (4.0f * kPiF * cosv); }
                    else sp.x += sqrtf(t2 / (fmaxf(sp.z, 1e-12f) * cosv));
                    const bool spread_out = depth >= 1 && sp.x * sp.x > a.spread_c * sp.y;
                    if (tw == kNone) {
                        cache_here = spread_out;
                    } else {
                        // a training path goes on for train_suffix vertices past
                        // the rendering end, then it too ends in the cache
                        uint32_t left = tw >> 24;
                        if (left == kNotReached) {
                            if (spread_out) {
                                left = min(a.train_suffix, kNotReached - 1u);
                                cache_here = left == 0;
                            }
                        } else {
                            left -= 1;
                            cache_here = left == 0;
                        }
                        tw = (tw & kSlotMask) | (left << 24);
                    }
                    const uint32_t slot = tw == kNone ? kNone : tw & kSlotMask;
                    const bool record = slot != kNone && !cache_here;
                    if (cache_here || record) {
                        q_p = p; q_wo = wo; q_n = nrm; q_alb = albedo; q_beta = beta;
                    }
                    if (record) {
                        float* rec = a.t_rec + ((size_t)slot * a.max_depth + depth) * kRec;
                        float in[12] = {p.x, p.y, p.z, wo.x, wo.y, wo.z, nrm.x, nrm.y, nrm.z,
                                        albedo.x, albedo.y, albedo.z};
#pragma unroll
                        for (int q = 0; q < 12; ++q) rec[q] = in[q];
                        rec[12] = beta.x > 0.0f ? 1.0f / beta.x : 0.0f;
                        rec[13] = beta.y > 0.0f ? 1.0f / beta.y : 0.0f;
                        rec[14] = beta.z > 0.0f ? 1.0f / beta.z : 0.0f;
                        rec[15] = rec[16] = rec[17] = 0.0f;
                        a.t_count[slot] = depth + 1;
                    }
                    query = cache_here;
                }
                if (!cache_here) {
                    float3 ss, ts;
                    frame(nrm, ss, ts);
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
                                o_l = offset_origin(p, perr, nrm, pl - p);
                                float3 tgt = offset_origin(pl, pl_err, nl, o_l - pl);
                                d_l = tgt - o_l;
                                tm_l = 1.0f - 0.0001f;
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
                                    o_b = o;
                                    d_b = wb;
                                    tm_b = tl * (1.0f - 0.0001f);
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
                            o_c = offset_origin(p, perr, nrm, wi);
                            d_c = wi;
                            beta_out = make_float4(nb.x, nb.y, nb.z, __uint_as_float(fid));
                            rng_out = make_uint2((uint32_t)rng.state, (uint32_t)(rng.state >> 32));
                            spread_next = make_float4(sp.x, sp.y, pdf, __uint_as_float(tw));
                            cont = true;
                        }
                    }
                }
            }
        }
        uint32_t s = warp_append(&a.counts[nxt], cont);
        if (cont) {
            put_ray(a.rays[nxt], s, o_c, d_c, INFINITY);
            a.beta[nxt][s] = beta_out;
            a.rng[nxt][s] = rng_out;
            a.pid[nxt][s] = id;
            if (kNrc) a.spread[nxt][s] = spread_next;
        }
        uint32_t sl = warp_append(&a.counts[kShadow], push_l);
        if (push_l) {
            put_ray(a.srays, sl, o_l, d_l, tm_l);
            a.scontrib[sl] = make_float4(c_l.x, c_l.y, c_l.z, __uint_as_float(fid));
            if (kNrc) a.s_train[sl] = make_uint2(tw == kNone ? kNone : tw & kSlotMask, depth);
        }
        uint32_t sb = warp_append(&a.counts[kShadow], push_b);
        if (push_b) {
            put_ray(a.srays, sb, o_b, d_b, tm_b);
            a.scontrib[sb] = make_float4(c_b.x, c_b.y, c_b.z, __uint_as_float(fid));
            if (kNrc) a.s_train[sb] = make_uint2(tw == kNone ? kNone : tw & kSlotMask, depth);
        }
        if (kNrc) {
            uint32_t sq = warp_append(&a.counts[kQueries], query);
            if (query && sq < a.q_cap) {
                float* qi = a.q_in + 12 * (size_t)sq;
                float in[12] = {q_p.x, q_p.y, q_p.z, q_wo.x, q_wo.y, q_wo.z, q_n.x, q_n.y, q_n.z,
                                q_alb.x, q_alb.y, q_alb.z};
#pragma unroll
                for (int q = 0; q < 12; ++q) qi[q] = in[q];
                a.q_beta[sq] = make_float4(q_beta.x, q_beta.y, q_beta.z, __uint_as_float(fid));
                a.q_train[sq] = make_uint2(tw == kNone ? kNone : tw & kSlotMask, depth);
            }
        }
    }
}

template <bool kNrc>
__global__ void k_pt_accum(PtArgs a) {
    const uint32_t n = (uint32_t)a.counts[kShadow];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (a.socc[i] != 0u) continue;
        float4 c4 = a.scontrib[i];
        float3 c = make_float3(c4.x, c4.y, c4.z);
        film_add(a, __float_as_uint(c4.w), c);
        if (kNrc) {
            uint2 st = a.s_train[i];
            if (st.x != kNone && good(c)) {
                // every vertex up to the one that cast this ray gets c / beta_k
                for (uint32_t k = 0; k <= st.y && k < a.max_depth; ++k) {
                    float* rec = a.t_rec + ((size_t)st.x * a.max_depth + k) * kRec;
                    atomicAdd(&rec[15], c.x * rec[12]);
                    atomicAdd(&rec[16], c.y * rec[13]);
                    atomicAdd(&rec[17], c.z * rec[14]);
                }
            }
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

// Flattens the recorded training vertices (at most sample_cap = n_batches *
// batch_rows).  Sample r goes to row (r % n_batches) * batch_rows + r / n_batches,
// so batch j (rows j * batch_rows ...) takes every n_batches-th sample and
// spans the whole image rather than one band of it.
__global__ void k_nrc_gather(PtArgs a, uint32_t n_batches, uint32_t batch_rows) {
    uint32_t slots = (uint32_t)min(a.counts[kTrainSlots], (unsigned long long)a.t_cap);
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < slots; s += gridDim.x * blockDim.x) {
        uint32_t c = a.t_count[s];
        if (c == 0) continue;
        unsigned long long pos = atomicAdd(&a.counts[kSamples], (unsigned long long)c);
        for (uint32_t k = 0; k < c && pos + k < a.sample_cap; ++k) {
            const float* rec = a.t_rec + ((size_t)s * a.max_depth + k) * kRec;
            uint32_t r = (uint32_t)(pos + k);
            size_t row = (size_t)(r % n_batches) * batch_rows + r / n_batches;
            float* in = a.t_in + 12 * row;
            for (int q = 0; q < 12; ++q) in[q] = rec[q];
            float* tg = a.t_tg + 3 * row;
            tg[0] = rec[15]; tg[1] = rec[16]; tg[2] = rec[17];
        }
    }
}

// film += throughput * max(prediction, 0) for every query of the frame; a
// training path's final query also adds that radiance / beta_k to the target
// of each vertex k it recorded (self-training).
__global__ void k_nrc_apply(PtArgs a) {
    uint32_t n = (uint32_t)min(a.counts[kQueries], (unsigned long long)a.q_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 b = a.q_beta[i];
        const float* p = a.q_out + 3 * (size_t)i;
        float3 c = make_float3(b.x * fmaxf(p[0], 0.0f), b.y * fmaxf(p[1], 0.0f), b.z * fmaxf(p[2], 0.0f));
        film_add(a, __float_as_uint(b.w), c);
        uint2 qt = a.q_train[i];
        if (qt.x != kNone && good(c)) {
            for (uint32_t k = 0; k < qt.y && k < a.max_depth; ++k) {
                float* rec = a.t_rec + ((size_t)qt.x * a.max_depth + k) * kRec;
                atomicAdd(&rec[15], c.x * rec[12]);
                atomicAdd(&rec[16], c.y * rec[13]);
                atomicAdd(&rec[17], c.z * rec[14]);
            }
        }
    }
}

// End of a frame: running totals and the frame counter.
__global__ void k_nrc_tally(PtArgs a, uint32_t sample_cap) {
    a.counts[kTotQueries] += min(a.counts[kQueries], (unsigned long long)a.q_cap);
    a.counts[kTotSamples] += min(a.counts[kSamples], (unsigned long long)sample_cap);
    a.counts[kFrame] += 1;
    a.counts[kTrainRows] = a.counts[kSamples];
}

// Film::write_image's division (film.rs:187-226): contribution sums times
// 1 / (filter weight sum), zero where no weight landed; for the pixel box
// film the weight sum of every pixel is its sample count.
__global__ void k_pt_resolve(const float* film, const float* wsum, float* out, uint32_t n3, float inv_spp) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n3) return;
    if (!wsum) {
        out[i] = film[i] * inv_spp;
    } else {
        float w = wsum[i / 3];
        out[i] = w != 0.0f ? film[i] * (1.0f / w) : 0.0f;
    }
}

// One bounce: extend, shade, shadow, accumulate, advance (queue parity cur).
template <bool kNrc>
cudaError_t bounce(const PtArgs& a, const DeviceAccel& da, const LaunchParams& lp, uint32_t cap, uint32_t* err,
                   int cur, int blocks, cudaStream_t s) {
    cudaError_t e = launch_trace(da, a.rays[cur], cap, const_cast<ilm_hit*>(a.hits), nullptr, err, lp, s,
                                 a.counts + cur);
    if (e != cudaSuccess) return e;
    k_pt_shade<kNrc><<<blocks, 256, 0, s>>>(a, cur);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    e = launch_trace(da, a.srays, 2ull * cap, nullptr, const_cast<uint32_t*>(a.socc), err, lp, s,
                     a.counts + kShadow);
    if (e != cudaSuccess) return e;
    k_pt_accum<kNrc><<<blocks, 256, 0, s>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_pt_advance<<<1, 1, 0, s>>>(a, cur);
    return cudaGetLastError();
}

// Everything a render needs; shared by ilm_render_pt and ilm_render_nrc.
struct RenderSetup {
    PtArgs a;
    DeviceAccel da;
    LaunchParams lp;
    uint32_t* err;
    int blocks;
    uint32_t P;
    uint64_t npix, total;
    cudaStream_t s;
};

int32_t setup_render(ilm_context* ctx, PtScene& sc, uint32_t spp, uint32_t max_depth, uint32_t rr_depth,
                     uint64_t seed, uint32_t wave_paths, uint64_t total_paths, bool nrc, RenderSetup& r,
                     const ilm_filter_desc* filter = nullptr) {
    Accel* acc = find_accel(ctx, sc.accel);
    if (!acc) { set_error(ctx, "render: the scene's accel was destroyed"); return ILM_ERR_NOT_FOUND; }
    const ilm_pt_scene_desc& d = sc.desc;
    uint32_t ns = (uint32_t)std::lround(std::sqrt((double)spp));
    if (spp == 0 || ns * ns != spp || max_depth == 0) {
        set_error(ctx, "render: spp must be a non-zero perfect square and max_depth >= 1");
        return ILM_ERR_INVALID_ARGUMENT;
    }
    r.npix = (uint64_t)d.width * d.height;
    r.total = total_paths;
    if (r.total >= (1ull << 32)) { set_error(ctx, "render: more than 2^32 paths"); return ILM_ERR_INVALID_ARGUMENT; }
    uint32_t P = wave_paths ? wave_paths : (1u << 21);
    if ((uint64_t)P > r.total) P = (uint32_t)r.total;
    r.P = P;
    PtBuffers& b = sc.buf;
    cudaError_t e = cudaSuccess;
    for (int q = 0; q < 2 && e == cudaSuccess; ++q) {
        if ((e = b.rays[q].reserve((size_t)P * sizeof(ilm_ray))) != cudaSuccess) break;
        if ((e = b.beta[q].reserve((size_t)P * 16)) != cudaSuccess) break;
        if ((e = b.rng[q].reserve((size_t)P * 8)) != cudaSuccess) break;
        if ((e = b.pid[q].reserve((size_t)P * 4)) != cudaSuccess) break;
        if (nrc) e = b.spread[q].reserve((size_t)P * 16);
    }
    if (e == cudaSuccess) e = b.hits.reserve((size_t)P * sizeof(ilm_hit));
    if (e == cudaSuccess) e = b.srays.reserve((size_t)2 * P * sizeof(ilm_ray));
    if (e == cudaSuccess) e = b.scontrib.reserve((size_t)2 * P * 16);
    if (e == cudaSuccess) e = b.socc.reserve((size_t)2 * P * 4);
    const bool fresh_counts = b.counts.bytes < kNumCounts * 8;
    if (e == cudaSuccess) e = b.counts.reserve(kNumCounts * 8);
    if (e == cudaSuccess) e = b.film.reserve(r.npix * 12);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "render buffers");
    if (!b.stream) {
        if ((e = cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking)) != cudaSuccess)
            return cuda_fail(ctx, e, "cudaStreamCreate");
        cudaEventCreate(&b.ev0);
        cudaEventCreate(&b.ev1);
    }
    r.s = b.stream;
    PtArgs& a = r.a;
    std::memset(&a, 0, sizeof a);
    a.tri = static_cast<const float4*>(sc.d_tri.ptr);
    a.mat = static_cast<const float4*>(sc.d_mat.ptr);
    a.lights = static_cast<const uint32_t*>(sc.d_lights.ptr);
    a.light_geo = static_cast<const float4*>(sc.d_light_geo.ptr);
    a.n_lights = sc.n_lights;
    a.film = static_cast<float*>(b.film.ptr);
    a.width = d.width; a.height = d.height; a.npix = (uint32_t)r.npix; a.spp = spp; a.ns = ns;
    a.eye_x = d.eye[0]; a.eye_y = d.eye[1]; a.eye_z = d.eye[2];
    a.tan_half = std::tan(0.5f * d.fov_deg * 3.14159265358979323846f / 180.0f);
    a.aspect = (float)d.width / (float)d.height;
    bool zero = true;
    for (int q = 0; q < 9; ++q) zero = zero && d.camera_to_world[q] == 0.0f;
    for (int q = 0; q < 9; ++q) a.cam[q] = zero ? (q % 4 == 0 ? 1.0f : 0.0f) : d.camera_to_world[q];
    a.max_depth = max_depth; a.rr_depth = rr_depth; a.seed = seed;
    for (int q = 0; q < 2; ++q) {
        a.rays[q] = static_cast<ilm_ray*>(b.rays[q].ptr);
        a.beta[q] = static_cast<float4*>(b.beta[q].ptr);
        a.rng[q] = static_cast<uint2*>(b.rng[q].ptr);
        a.pid[q] = static_cast<uint32_t*>(b.pid[q].ptr);
        a.spread[q] = static_cast<float4*>(b.spread[q].ptr);
    }
    a.hits = static_cast<const ilm_hit*>(b.hits.ptr);
    a.srays = static_cast<ilm_ray*>(b.srays.ptr);
    a.scontrib = static_cast<float4*>(b.scontrib.ptr);
    a.socc = static_cast<const uint32_t*>(b.socc.ptr);
    a.counts = static_cast<unsigned long long*>(b.counts.ptr);
    r.da = acc->view();
    unsigned long long* counter = ctx->counter_for(r.s);
    if (!counter) return ILM_ERR_OUT_OF_MEMORY;
    r.lp = LaunchParams{ctx->stack_depth, ctx->block_size, ctx->max_iter, 1, counter,
                        (ctx->flags & ILM_FLAG_HIGH_OCCUPANCY) ? 8 : 0,
                        1};   // pooled refill with the split tail (2,484-2,491 against 2,451
                              // Mrays/s for lanes that refill one by one, at 7 blocks per SM)
    // Queues of at most one wave (late bounces, training suffixes) run one
    // thread per ray with the split tail instead.
    r.lp.split_tail = split_tail_of(ctx);
    r.lp.queue_split = r.lp.split_tail;
    r.err = static_cast<uint32_t*>(ctx->err_word.ptr);
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, ctx->device);
    r.blocks = dev_sms * 8;
    // film filter: the default (no filter, or the box of radius 0.5) puts each
    // sample in its own pixel; any other filter splats through its table
    a.fbox = 1;
    a.wsum = nullptr;
    if (filter && filter->radius[0] > 0.0f &&
        !(filter->kind == ILM_FILTER_BOX && filter->radius[0] == 0.5f && filter->radius[1] == 0.5f)) {
        float table[ILM_FILTER_TABLE_WIDTH * ILM_FILTER_TABLE_WIDTH];
        if (ilm_filter_table(filter, table) != ILM_OK) {
            set_error(ctx, "render: invalid film filter");
            return ILM_ERR_INVALID_ARGUMENT;
        }
        if ((e = b.ftable.reserve(sizeof table)) != cudaSuccess || (e = b.wsum.reserve(r.npix * 4)) != cudaSuccess)
            return cuda_fail(ctx, e, "film filter buffers");
        cudaMemcpyAsync(b.ftable.ptr, table, sizeof table, cudaMemcpyHostToDevice, r.s);
        cudaMemsetAsync(b.wsum.ptr, 0, r.npix * 4, r.s);
        a.fbox = 0;
        a.ftable = static_cast<const float*>(b.ftable.ptr);
        a.wsum = static_cast<float*>(b.wsum.ptr);
        a.frx = filter->radius[0];
        a.fry = filter->radius[1];
        a.firx = 1.0f / filter->radius[0];
        a.firy = 1.0f / filter->radius[1];
    }
    // everything but kTrainRows restarts; that one is kept for the next render's first frame
    cudaMemsetAsync(a.counts, 0, (fresh_counts ? kNumCounts : kTrainRows) * 8, r.s);
    cudaMemsetAsync(a.film, 0, r.npix * 12, r.s);
    return ILM_OK;
}

// Resolves the film into rgb_out (host or device) and reads the counters.
int32_t finish_render(ilm_context* ctx, PtScene& sc, RenderSetup& r, float* rgb_out, float inv_spp,
                      unsigned long long* cnts) {
    PtBuffers& b = sc.buf;
    cudaError_t e;
    PtrKind k = classify(rgb_out);
    float* dst = rgb_out;
    if (k == PtrKind::kHost) {
        if ((e = b.out.reserve(r.npix * 12)) != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc(out)");
        dst = static_cast<float*>(b.out.ptr);
    }
    uint32_t n3 = (uint32_t)(r.npix * 3);
    k_pt_resolve<<<(n3 + 255) / 256, 256, 0, r.s>>>(r.a.film, r.a.wsum, dst, n3, inv_spp);
    if (k == PtrKind::kHost) cudaMemcpyAsync(rgb_out, dst, r.npix * 12, cudaMemcpyDeviceToHost, r.s);
    cudaMemcpyAsync(cnts, r.a.counts, kNumCounts * 8, cudaMemcpyDeviceToHost, r.s);
    if ((e = cudaStreamSynchronize(r.s)) != cudaSuccess) return cuda_fail(ctx, e, "render");
    return ILM_OK;
}

}  // namespace
}  // namespace ilm

using namespace ilm;

extern "C" {

int32_t ilm_pt_scene_create(ilm_context* ctx, ilm_accel_id accel, const ilm_pt_scene_desc* desc,
                            ilm_pt_scene_id* out) {
    if (!ctx || !desc || !out) return ILM_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ILM_ERR_CUDA;
    Accel* acc = find_accel(ctx, accel);
    if (!acc) { set_error(ctx, "ilm_pt_scene_create: unknown accel id"); return ILM_ERR_NOT_FOUND; }
    const HostLayout& h = acc->host;
    if (!desc->prim_material || !desc->albedo || !desc->emission || desc->n_materials == 0 || desc->width == 0 ||
        desc->height == 0 || !(desc->fov_deg > 0.0f && desc->fov_deg < 180.0f) ||
        !std::all_of(desc->camera_to_world, desc->camera_to_world + 9, [](float v) { return std::isfinite(v); })) {
        set_error(ctx, "ilm_pt_scene_create: invalid scene description");
        return ILM_ERR_INVALID_ARGUMENT;
    }
    auto sc = std::make_unique<PtScene>();
    sc->accel = accel;
    sc->desc = *desc;
    for (int k = 0; k < 6; ++k) sc->bound[k] = h.bound[k];
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
    cudaError_t e;
    if ((e = sc->d_tri.reserve(tri.size() * 4 + 16)) != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    if ((e = sc->d_mat.reserve(mat.size() * 4)) != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    if (np) cudaMemcpy(sc->d_tri.ptr, tri.data(), tri.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(sc->d_mat.ptr, mat.data(), mat.size() * 4, cudaMemcpyHostToDevice);
    if (!lights.empty()) {
        if ((e = sc->d_lights.reserve(lights.size() * 4)) != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
        if ((e = sc->d_light_geo.reserve(lgeo.size() * 4)) != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
        cudaMemcpy(sc->d_lights.ptr, lights.data(), lights.size() * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(sc->d_light_geo.ptr, lgeo.data(), lgeo.size() * 4, cudaMemcpyHostToDevice);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "ilm_pt_scene_create");
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
    RenderSetup r;
    uint64_t total = (uint64_t)sc.desc.width * sc.desc.height * opts->spp;
    int32_t st = setup_render(ctx, sc, opts->spp, opts->max_depth, opts->rr_depth, opts->seed, opts->wave_paths,
                              total, false, r, &opts->filter);
    if (st != ILM_OK) return st;
    PtArgs& a = r.a;
    cudaStream_t s = r.s;
    cudaError_t e = cudaSuccess;
    cudaGraphExec_t graphs[2] = {nullptr, nullptr};
    if (opts->use_graphs) {
        // One eager bounce over empty queues (every kernel returns at once)
        // does the launchers' one-time setup outside the capture.
        if ((e = bounce<false>(a, r.da, r.lp, r.P, r.err, 0, r.blocks, s)) != cudaSuccess)
            return cuda_fail(ctx, e, "bounce");
        for (int q = 0; q < 2; ++q) {
            cudaGraph_t g;
            if ((e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
                return cuda_fail(ctx, e, "cudaStreamBeginCapture");
            cudaError_t eb = bounce<false>(a, r.da, r.lp, r.P, r.err, q, r.blocks, s);
            e = cudaStreamEndCapture(s, &g);
            if (eb != cudaSuccess) return cuda_fail(ctx, eb, "bounce capture");
            if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&graphs[q], g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGraphInstantiate");
        }
    }
    cudaEventRecord(sc.buf.ev0, s);
    uint32_t waves = 0;
    for (uint64_t p0 = 0; p0 < r.total; p0 += r.P, ++waves) {
        uint32_t cnt = (uint32_t)(r.total - p0 < r.P ? r.total - p0 : r.P);
        k_pt_camera<false><<<(cnt + 255) / 256, 256, 0, s>>>(a, p0, cnt);
        for (uint32_t depth = 0; depth < opts->max_depth; ++depth) {
            int cur = depth & 1;
            if (opts->use_graphs) e = cudaGraphLaunch(graphs[cur], s);
            else e = bounce<false>(a, r.da, r.lp, r.P, r.err, cur, r.blocks, s);
            if (e != cudaSuccess) break;
        }
        if (e != cudaSuccess) break;
    }
    cudaEventRecord(sc.buf.ev1, s);
    for (auto& g : graphs) if (g) cudaGraphExecDestroy(g);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "ilm_render_pt launch");
    unsigned long long cnts[kNumCounts];
    if ((st = finish_render(ctx, sc, r, rgb_out, 1.0f / (float)opts->spp, cnts)) != ILM_OK) return st;
    if (stats) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, sc.buf.ev0, sc.buf.ev1);
        stats->closest_rays = cnts[kTotClosest];
        stats->shadow_rays = cnts[kTotShadow];
        stats->seconds = ms * 1e-3;
        stats->waves = waves;
    }
    if (cnts[kDropped]) {
        set_error(ctx, "ilm_render_pt: some paths reached the traversal limits and were dropped");
        return ILM_ERR_TRAVERSAL_LIMIT;
    }
    return ILM_OK;
}

int32_t ilm_render_nrc(ilm_context* ctx, ilm_pt_scene_id scene, ilm_nrc* nrc, const ilm_nrc_render_opts* o,
                       float* rgb_out, ilm_nrc_render_stats* stats) {
    if (!ctx || !nrc || !o || !rgb_out) return ILM_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ILM_ERR_CUDA;
    auto it = ctx->pt_scenes.find(scene);
    if (it == ctx->pt_scenes.end()) { set_error(ctx, "ilm_render_nrc: unknown scene id"); return ILM_ERR_NOT_FOUND; }
    if (o->frames == 0 && !(o->time_budget_s > 0.0)) {
        set_error(ctx, "ilm_render_nrc: give frames or a time budget");
        return ILM_ERR_INVALID_ARGUMENT;
    }
    PtScene& sc = *it->second;
    const uint64_t npix = (uint64_t)sc.desc.width * sc.desc.height;
    const uint32_t spf = o->spp_per_frame ? o->spp_per_frame : 1;
    if (npix * spf > (1ull << 27)) {
        set_error(ctx, "ilm_render_nrc: width * height * spp_per_frame above 2^27");
        return ILM_ERR_INVALID_ARGUMENT;
    }
    // path ids are 32-bit: frame * paths-per-frame stays below 2^32
    const uint32_t id_frames = (uint32_t)(((1ull << 32) - 1) / (npix * spf));
    const uint32_t max_frames = std::min(o->frames ? o->frames : 1000000u, id_frames);
    RenderSetup r;
    int32_t st = setup_render(ctx, sc, spf, o->max_depth, o->rr_depth, o->seed, (uint32_t)(npix * spf),
                              npix * spf * (uint64_t)max_frames, true, r);
    if (st != ILM_OK) return st;
    const uint32_t P = (uint32_t)(npix * spf);
    r.P = P;
    PtBuffers& b = sc.buf;
    const uint32_t train_paths = o->train_paths ? o->train_paths : 16384u;
    const uint32_t n_batches = o->train_steps ? o->train_steps : 4u;
    const uint32_t batch_rows = ((o->train_samples ? o->train_samples : 65536u) + n_batches - 1) / n_batches;
    const uint32_t sample_cap = batch_rows * n_batches;
    // with training off there are no training paths
    const uint32_t stride = o->train ? (uint32_t)std::max<uint64_t>(kMinTrainStride, P / train_paths) : 0u;
    const uint32_t t_cap = stride ? P / stride + 1 : 1;
    const uint32_t q_cap = P + t_cap;
    cudaError_t e = cudaSuccess;
    if ((e = b.q_in.reserve((size_t)q_cap * 48)) == cudaSuccess &&
        (e = b.q_beta.reserve((size_t)q_cap * 16)) == cudaSuccess &&
        (e = b.q_train.reserve((size_t)q_cap * 8)) == cudaSuccess &&
        (e = b.q_out.reserve((size_t)q_cap * 12)) == cudaSuccess &&
        (e = b.t_rec.reserve((size_t)t_cap * o->max_depth * kRec * 4)) == cudaSuccess &&
        (e = b.t_count.reserve((size_t)t_cap * 4)) == cudaSuccess &&
        (e = b.s_train.reserve((size_t)2 * P * 8)) == cudaSuccess &&
        (e = b.t_in.reserve((size_t)sample_cap * 48)) == cudaSuccess &&
        (e = b.t_tg.reserve((size_t)sample_cap * 12)) == cudaSuccess)
        e = nrc_reserve(nrc, batch_rows);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "nrc render buffers");
    PtArgs& a = r.a;
    a.q_in = static_cast<float*>(b.q_in.ptr);
    a.q_beta = static_cast<float4*>(b.q_beta.ptr);
    a.q_train = static_cast<uint2*>(b.q_train.ptr);
    a.q_out = static_cast<const float*>(b.q_out.ptr);
    a.q_cap = q_cap;
    a.t_rec = static_cast<float*>(b.t_rec.ptr);
    a.t_count = static_cast<uint32_t*>(b.t_count.ptr);
    a.t_cap = t_cap;
    a.train_stride = stride;
    a.train_suffix = o->train_suffix ? o->train_suffix : 1u;
    a.spread_c = o->spread_c > 0.0f ? o->spread_c : 0.01f;
    a.s_train = static_cast<uint2*>(b.s_train.ptr);
    a.t_in = static_cast<float*>(b.t_in.ptr);
    a.t_tg = static_cast<float*>(b.t_tg.ptr);
    a.sample_cap = sample_cap;
    cudaStream_t s = r.s;
    if (!b.train_stream) {
        if ((e = cudaStreamCreateWithFlags(&b.train_stream, cudaStreamNonBlocking)) != cudaSuccess)
            return cuda_fail(ctx, e, "cudaStreamCreate");
        cudaEventCreateWithFlags(&b.fork, cudaEventDisableTiming);
        cudaEventCreateWithFlags(&b.join, cudaEventDisableTiming);
    }
    // samples kept from an earlier render are trained on only if they were
    // gathered with this batch layout
    if (!o->train || b.train_layout[0] != n_batches || b.train_layout[1] != batch_rows)
        cudaMemsetAsync(a.counts + kTrainRows, 0, sizeof(unsigned long long), s);
    b.train_layout[0] = n_batches;
    b.train_layout[1] = batch_rows;
    // One frame, all on the device.  The training branch (train_steps Adam
    // steps on the samples the previous frame gathered) runs beside the camera
    // and the bounces, whose later, shorter queues leave most SMs idle; the
    // cache queries are answered after both, then applied, this frame's
    // samples gathered and the counters tallied.  Queue sizes and the frame
    // index stay in device memory, so the frame is one CUDA graph replayed
    // every frame.
    cudaStream_t ts = b.train_stream;
    auto enqueue_frame = [&]() -> cudaError_t {
        cudaError_t e2;
        if (o->train) {
            cudaEventRecord(b.fork, s);
            cudaStreamWaitEvent(ts, b.fork, 0);
            for (uint32_t j = 0; j < n_batches; ++j) {
                size_t row = (size_t)j * batch_rows;
                if ((e2 = nrc_train_async(nrc, a.t_in + 12 * row, a.t_tg + 3 * row,
                                          NrcCount{a.counts + kTrainRows, sample_cap, n_batches, j}, ts)) !=
                    cudaSuccess)
                    return e2;
            }
            cudaEventRecord(b.join, ts);
        }
        if ((e2 = cudaMemsetAsync(a.counts + kQueries, 0, 3 * sizeof(unsigned long long), s)) != cudaSuccess)
            return e2;
        k_pt_camera<true><<<(P + 255) / 256, 256, 0, s>>>(a, 0, P);
        for (uint32_t depth = 0; depth < o->max_depth; ++depth)
            if ((e2 = bounce<true>(a, r.da, r.lp, P, r.err, depth & 1, r.blocks, s)) != cudaSuccess) return e2;
        if (o->train) cudaStreamWaitEvent(s, b.join, 0);
        if ((e2 = nrc_infer_async(nrc, a.q_in, NrcCount{a.counts + kQueries, q_cap, 1, 0},
                                  static_cast<float*>(b.q_out.ptr), s)) != cudaSuccess)
            return e2;
        k_nrc_apply<<<r.blocks, 256, 0, s>>>(a);
        k_nrc_gather<<<r.blocks, 256, 0, s>>>(a, n_batches, batch_rows);
        k_nrc_tally<<<1, 1, 0, s>>>(a, sample_cap);
        return cudaGetLastError();
    };
    // one eager bounce over the empty queues does the launchers' one-time
    // setup outside the capture
    if ((e = bounce<true>(a, r.da, r.lp, P, r.err, 0, r.blocks, s)) != cudaSuccess) return cuda_fail(ctx, e, "bounce");
    cudaGraphExec_t frame_graph = nullptr;
    {
        cudaGraph_t g = nullptr;
        if ((e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
            return cuda_fail(ctx, e, "cudaStreamBeginCapture");
        cudaError_t ef = enqueue_frame();
        e = cudaStreamEndCapture(s, &g);
        if (e == cudaSuccess) e = ef;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&frame_graph, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "nrc frame graph");
    }
    // frames; with a time budget the host keeps one frame queued ahead and
    // stops launching once the finished frames reach the budget
    cudaEvent_t done[2];
    cudaEventCreate(&done[0]);
    cudaEventCreate(&done[1]);
    cudaEventRecord(b.ev0, s);
    uint32_t frame = 0;
    for (; frame < max_frames; ++frame) {
        if ((e = cudaGraphLaunch(frame_graph, s)) != cudaSuccess) break;
        cudaEventRecord(done[frame & 1], s);
        if (o->time_budget_s > 0.0 && frame >= 1) {
            if ((e = cudaEventSynchronize(done[(frame - 1) & 1])) != cudaSuccess) break;
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, b.ev0, done[(frame - 1) & 1]);
            if (ms * 1e-3 >= o->time_budget_s) { ++frame; break; }
        }
    }
    cudaEventRecord(b.ev1, s);
    cudaGraphExecDestroy(frame_graph);
    if (e != cudaSuccess) {
        cudaEventDestroy(done[0]);
        cudaEventDestroy(done[1]);
        return cuda_fail(ctx, e, "ilm_render_nrc");
    }
    unsigned long long cnts[kNumCounts];
    st = finish_render(ctx, sc, r, rgb_out, 1.0f / (float)(spf * std::max(frame, 1u)), cnts);
    cudaEventDestroy(done[0]);
    cudaEventDestroy(done[1]);
    if (st != ILM_OK) return st;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, b.ev0, b.ev1);
    uint32_t net_err = 0;
    cudaMemcpy(&net_err, nrc_error_word(nrc), 4, cudaMemcpyDeviceToHost);
    if (net_err) {
        set_error(ctx, "ilm_render_nrc: a tensor-core wait of the cache network ran out of time");
        return ILM_ERR_TIMEOUT;
    }
    float loss = 0.0f;
    uint32_t last_nt = (uint32_t)std::min<unsigned long long>(cnts[kSamples], sample_cap);
    if (o->train && last_nt) {
        // loss of the network on the first batch of the last frame, for reporting
        uint32_t n0 = (last_nt + n_batches - 1) / n_batches;
        if ((st = ilm_nrc_gradients(ctx, nrc, a.t_in, a.t_tg, n0, nullptr, &loss)) != ILM_OK) return st;
    }
    if (stats) {
        stats->frames = frame;
        stats->seconds = ms * 1e-3;
        stats->closest_rays = cnts[kTotClosest];
        stats->shadow_rays = cnts[kTotShadow];
        stats->queries = cnts[kTotQueries];
        stats->train_samples = cnts[kTotSamples];
        stats->last_loss = loss;
    }
    if (cnts[kDropped]) {
        set_error(ctx, "ilm_render_nrc: some paths reached the traversal limits and were dropped");
        return ILM_ERR_TRAVERSAL_LIMIT;
    }
    return ILM_OK;
}

}  // extern "C"
