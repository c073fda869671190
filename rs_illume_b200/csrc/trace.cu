// Ray-query kernels for sm_100a: BVHAccel::intersect / intersect_p
// (accelerators/bvh.rs:563-662) over batches of 32-byte rays.
//
//  * width 2: the reference's own 32-byte binary nodes and ordered stack
//    traversal (near child by dir_is_neg[axis]).
//  * width 4 / 8: compressed wide nodes (8-bit quantised child boxes on a
//    per-node grid, 64 / 80 bytes per node) collapsed from the same SAH tree;
//    hit children are sorted by entry distance with a sorting network and
//    pushed far-to-near on a per-thread stack.
//
// Primitive records (48 bytes) are stored in traversal order so a leaf is one
// contiguous run of 16-byte loads.  Closest hit keeps the smallest t, ties to
// the smaller primitive id; any-hit stops at the first accepted primitive.
// Every loop is bounded: stack overflow and an iteration cap set a bit in the
// context's error word and mark the ray's record, and the thread exits.
#include <cuda_runtime.h>
#include <stdint.h>

#include "illume_gpu.h"
#include "kernels.h"
#include "layout.h"
#include "shapes.cuh"

namespace ilm {

namespace {

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

// Tests primitive record `r` (index in traversal order).
template <bool kClosest>
__device__ __forceinline__ bool prim_test(const PrimRec* __restrict__ prims, const SphereRec* __restrict__ spheres,
                                          uint32_t r, const TriRay& tr, const RayIn& ray, float tmax,
                                          float& t, float& u, float& v, uint32_t& prim_id) {
    const float4* p = reinterpret_cast<const float4*>(prims + r);
    float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    uint32_t flags = __float_as_uint(b.w);
    prim_id = __float_as_uint(a.w);
    if (flags & kPrimSphere) {
        return sphere_test(spheres[__float_as_uint(c.w)], ray.ox, ray.oy, ray.oz, ray.dx, ray.dy, ray.dz,
                           tmax, t, u, v);
    }
    if (kClosest && (flags & kPrimDegenerate)) return false;
    return triangle_test(tr, make_float3(a.x, a.y, a.z), make_float3(b.x, b.y, b.z),
                         make_float3(c.x, c.y, c.z), tmax, t, u, v);
}

// ------------------------------------------------------------------ binary
// Bounds3::intersect_p with precomputed inv_dir / dir_is_neg (bounds3.rs:284-318).
__device__ __forceinline__ bool bin_box(const float4& n0, const float4& n1, const RayIn& r, float ix, float iy,
                                        float iz, bool nx, bool ny, bool nz, float tmax) {
    // n0 = (minx, miny, minz, maxx), n1 = (maxy, maxz, offset, n/axis)
    float t_min = __fmul_rn(__fsub_rn(nx ? n0.w : n0.x, r.ox), ix);
    float t_max = __fmul_rn(__fsub_rn(nx ? n0.x : n0.w, r.ox), ix);
    float ty_min = __fmul_rn(__fsub_rn(ny ? n1.x : n0.y, r.oy), iy);
    float ty_max = __fmul_rn(__fsub_rn(ny ? n0.y : n1.x, r.oy), iy);
    t_max = __fmul_rn(t_max, kBoxRobust);
    ty_max = __fmul_rn(ty_max, kBoxRobust);
    if (t_min > ty_max || ty_min > t_max) return false;
    if (ty_min > t_min) t_min = ty_min;
    if (ty_max < t_max) t_max = ty_max;
    float tz_min = __fmul_rn(__fsub_rn(nz ? n1.y : n0.z, r.oz), iz);
    float tz_max = __fmul_rn(__fsub_rn(nz ? n0.z : n1.y, r.oz), iz);
    tz_max = __fmul_rn(tz_max, kBoxRobust);
    if (t_min > tz_max || tz_min > t_max) return false;
    if (tz_min > t_min) t_min = tz_min;
    if (tz_max < t_max) t_max = tz_max;
    return (t_min < tmax) && (t_max > 0.0f);
}

template <bool kAny>
__global__ void __launch_bounds__(128) k_trace_bin(const BinNode* __restrict__ nodes, uint32_t n_nodes,
                                                   const PrimRec* __restrict__ prims,
                                                   const SphereRec* __restrict__ spheres,
                                                   const ilm_ray* __restrict__ rays, uint64_t n,
                                                   ilm_hit* __restrict__ hits, uint32_t* __restrict__ occ,
                                                   uint32_t* __restrict__ err, uint32_t max_iter) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    RayIn ray = load_ray(rays, i);
    float best_t = ray.tmax, bu = 0.0f, bv = 0.0f;
    uint32_t best = ILM_MISS;
    bool occluded = false;
    uint32_t status = 0;
    if (n_nodes > 0) {
        TriRay tr = make_tri_ray(ray.ox, ray.oy, ray.oz, ray.dx, ray.dy, ray.dz);
        float ix = __fdiv_rn(1.0f, ray.dx), iy = __fdiv_rn(1.0f, ray.dy), iz = __fdiv_rn(1.0f, ray.dz);
        bool negx = ix < 0.0f, negy = iy < 0.0f, negz = iz < 0.0f;
        uint32_t stack[64];
        int sp = 0;
        uint32_t cur = 0, iter = 0;
        for (;;) {
            if (++iter > max_iter) { status = kErrIterationCap; break; }
            const float4* np = reinterpret_cast<const float4*>(nodes + cur);
            float4 n0 = __ldg(np), n1 = __ldg(np + 1);
            if (bin_box(n0, n1, ray, ix, iy, iz, negx, negy, negz, kAny ? ray.tmax : best_t)) {
                uint32_t meta = __float_as_uint(n1.w);
                uint32_t nprims = meta & 0xFFFFu;
                uint32_t off = __float_as_uint(n1.z);
                if (nprims > 0) {
                    for (uint32_t k = 0; k < nprims; ++k) {
                        float t, u, v;
                        uint32_t pid;
                        if (kAny) {
                            if (prim_test<false>(prims, spheres, off + k, tr, ray, ray.tmax, t, u, v, pid)) {
                                occluded = true;
                                break;
                            }
                        } else if (prim_test<true>(prims, spheres, off + k, tr, ray, best_t, t, u, v, pid) &&
                                   (t < best_t || (t == best_t && pid < best))) {
                            best_t = t; best = pid; bu = u; bv = v;
                        }
                    }
                    if (kAny && occluded) break;
                    if (sp == 0) break;
                    cur = stack[--sp];
                } else {
                    if (sp == 64) { status = kErrStackOverflow; break; }
                    uint32_t axis = (meta >> 16) & 0xFFu;
                    bool neg = axis == 0 ? negx : (axis == 1 ? negy : negz);
                    if (neg) { stack[sp++] = cur + 1; cur = off; }
                    else { stack[sp++] = off; cur = cur + 1; }
                }
            } else {
                if (sp == 0) break;
                cur = stack[--sp];
            }
        }
    }
    if (status) atomicOr(err, status);
    if (kAny) {
        occ[i] = status ? kHitTraversalError : (occluded ? 1u : 0u);
    } else {
        if (status) store_hit(hits, i, kHitTraversalError, ray.tmax, 0.0f, 0.0f);
        else store_hit(hits, i, best, best == ILM_MISS ? ray.tmax : best_t, bu, bv);
    }
}

// ------------------------------------------------------------------ wide
template <int W> struct WideWords;
template <> struct WideWords<8> {
    static constexpr int kWords = 5;
};
template <> struct WideWords<4> {
    static constexpr int kWords = 4;
};

// Byte i of a W-byte array split over 32-bit words lo (bytes 0-3) and hi (4-7).
template <int W>
__device__ __forceinline__ uint32_t byte_of(uint32_t lo, uint32_t hi, int i) {
    return ((i < 4 ? lo : hi) >> (8 * (i & 3))) & 0xFFu;
}

// Decoded node, with near/far planes already swapped for the ray octant.
template <int W>
struct WideView {
    float ox, oy, oz, sx, sy, sz;
    uint32_t imask, child_base, prim_base;
    uint32_t meta[2];
    uint32_t nq[3][2], fq[3][2];   // near / far quantised planes per axis
};

template <int W>
__device__ __forceinline__ WideView<W> load_wide(const uint4* __restrict__ nodes, uint32_t idx, bool negx,
                                                 bool negy, bool negz) {
    WideView<W> v;
    const uint4* p = nodes + (size_t)idx * WideWords<W>::kWords;
    uint4 w0 = __ldg(p), w1 = __ldg(p + 1), w2 = __ldg(p + 2), w3 = __ldg(p + 3);
    v.ox = __uint_as_float(w0.x); v.oy = __uint_as_float(w0.y); v.oz = __uint_as_float(w0.z);
    v.sx = __uint_as_float((w0.w & 0xFFu) << 23);
    v.sy = __uint_as_float(((w0.w >> 8) & 0xFFu) << 23);
    v.sz = __uint_as_float(((w0.w >> 16) & 0xFFu) << 23);
    v.imask = w0.w >> 24;
    v.child_base = w1.x;
    v.prim_base = w1.y;
    uint32_t lo[3][2], hi[3][2];
    if (W == 8) {
        uint4 w4 = __ldg(p + 4);
        v.meta[0] = w1.z; v.meta[1] = w1.w;
        lo[0][0] = w2.x; lo[0][1] = w2.y; lo[1][0] = w2.z; lo[1][1] = w2.w;
        lo[2][0] = w3.x; lo[2][1] = w3.y; hi[0][0] = w3.z; hi[0][1] = w3.w;
        hi[1][0] = w4.x; hi[1][1] = w4.y; hi[2][0] = w4.z; hi[2][1] = w4.w;
    } else {
        v.meta[0] = w1.z; v.meta[1] = 0;
        lo[0][0] = w1.w; lo[1][0] = w2.x; lo[2][0] = w2.y; hi[0][0] = w2.z; hi[1][0] = w2.w;
        hi[2][0] = w3.x;
        lo[0][1] = lo[1][1] = lo[2][1] = hi[0][1] = hi[1][1] = hi[2][1] = 0;
    }
    bool neg[3] = {negx, negy, negz};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            v.nq[a][h] = neg[a] ? hi[a][h] : lo[a][h];
            v.fq[a][h] = neg[a] ? lo[a][h] : hi[a][h];
        }
    return v;
}

// Slab test of child i (Bounds3::intersect_p semantics on the dequantised
// box; fmaxf/fminf skip a NaN slab, which can only widen the accepted set).
template <int W>
__device__ __forceinline__ bool child_hit(const WideView<W>& v, int i, const RayIn& r, float ix, float iy,
                                          float iz, float tmax, float& tn_out) {
    uint32_t m = byte_of<W>(v.meta[0], v.meta[1], i);
    float nx = fmaf((float)byte_of<W>(v.nq[0][0], v.nq[0][1], i), v.sx, v.ox);
    float fx = fmaf((float)byte_of<W>(v.fq[0][0], v.fq[0][1], i), v.sx, v.ox);
    float ny = fmaf((float)byte_of<W>(v.nq[1][0], v.nq[1][1], i), v.sy, v.oy);
    float fy = fmaf((float)byte_of<W>(v.fq[1][0], v.fq[1][1], i), v.sy, v.oy);
    float nz = fmaf((float)byte_of<W>(v.nq[2][0], v.nq[2][1], i), v.sz, v.oz);
    float fz = fmaf((float)byte_of<W>(v.fq[2][0], v.fq[2][1], i), v.sz, v.oz);
    float tnx = __fmul_rn(__fsub_rn(nx, r.ox), ix), tfx = __fmul_rn(__fsub_rn(fx, r.ox), ix);
    float tny = __fmul_rn(__fsub_rn(ny, r.oy), iy), tfy = __fmul_rn(__fsub_rn(fy, r.oy), iy);
    float tnz = __fmul_rn(__fsub_rn(nz, r.oz), iz), tfz = __fmul_rn(__fsub_rn(fz, r.oz), iz);
    float tn = fmaxf(fmaxf(tnx, tny), tnz);
    float tf = __fmul_rn(fminf(fminf(tfx, tfy), tfz), kBoxRobust);
    tn_out = tn;
    return m != 0u && tn <= tf && tn < tmax && tf > 0.0f;
}

template <int W>
__device__ __forceinline__ uint32_t child_entry(const WideView<W>& v, uint32_t slot) {
    uint32_t m = byte_of<W>(v.meta[0], v.meta[1], (int)slot);
    if ((v.imask >> slot) & 1u) return v.child_base + (m & 31u);
    return kLeafFlag | ((v.prim_base + (m & 31u)) << 3) | ((m >> 5) - 1u);
}

__device__ __forceinline__ void cswap(uint32_t& a, uint32_t& b) {
    uint32_t lo = min(a, b), hi = max(a, b);
    a = lo; b = hi;
}

template <int W>
__device__ __forceinline__ void sort_keys(uint32_t* k) {
    if (W == 8) {
        // Batcher odd-even merge sort, 19 comparators
        cswap(k[0], k[1]); cswap(k[2], k[3]); cswap(k[4], k[5]); cswap(k[6], k[7]);
        cswap(k[0], k[2]); cswap(k[1], k[3]); cswap(k[4], k[6]); cswap(k[5], k[7]);
        cswap(k[1], k[2]); cswap(k[5], k[6]);
        cswap(k[0], k[4]); cswap(k[1], k[5]); cswap(k[2], k[6]); cswap(k[3], k[7]);
        cswap(k[2], k[4]); cswap(k[3], k[5]);
        cswap(k[1], k[2]); cswap(k[3], k[4]); cswap(k[5], k[6]);
    } else {
        cswap(k[0], k[1]); cswap(k[2], k[3]);
        cswap(k[0], k[2]); cswap(k[1], k[3]);
        cswap(k[1], k[2]);
    }
}

template <int W, int kStack, bool kAny>
__global__ void __launch_bounds__(128) k_trace_wide(const uint4* __restrict__ nodes, uint32_t n_nodes,
                                                    const PrimRec* __restrict__ prims,
                                                    const SphereRec* __restrict__ spheres,
                                                    const ilm_ray* __restrict__ rays, uint64_t n,
                                                    ilm_hit* __restrict__ hits, uint32_t* __restrict__ occ,
                                                    uint32_t* __restrict__ err, uint32_t max_iter) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    RayIn ray = load_ray(rays, i);
    float best_t = ray.tmax, bu = 0.0f, bv = 0.0f;
    uint32_t best = ILM_MISS;
    bool occluded = false;
    uint32_t status = 0;
    if (n_nodes > 0) {
        TriRay tr = make_tri_ray(ray.ox, ray.oy, ray.oz, ray.dx, ray.dy, ray.dz);
        float ix = __fdiv_rn(1.0f, ray.dx), iy = __fdiv_rn(1.0f, ray.dy), iz = __fdiv_rn(1.0f, ray.dz);
        bool negx = ix < 0.0f, negy = iy < 0.0f, negz = iz < 0.0f;
        uint2 stack[kStack];
        int sp = 0;
        uint32_t cur = 0, iter = 0;
        for (;;) {
            if (++iter > max_iter) { status = kErrIterationCap; break; }
            bool descend = false;
            if (cur & kLeafFlag) {
                uint32_t start = (cur & ~kLeafFlag) >> 3, cnt = (cur & 7u) + 1u;
                for (uint32_t k = 0; k < cnt; ++k) {
                    float t, u, v;
                    uint32_t pid;
                    if (kAny) {
                        if (prim_test<false>(prims, spheres, start + k, tr, ray, ray.tmax, t, u, v, pid)) {
                            occluded = true;
                            break;
                        }
                    } else if (prim_test<true>(prims, spheres, start + k, tr, ray, best_t, t, u, v, pid) &&
                               (t < best_t || (t == best_t && pid < best))) {
                        best_t = t; best = pid; bu = u; bv = v;
                    }
                }
                if (kAny && occluded) break;
            } else {
                WideView<W> nv = load_wide<W>(nodes, cur, negx, negy, negz);
                float lim = kAny ? ray.tmax : best_t;
                if (kAny) {
                    // any order will do: push every hit child, continue with the first
                    uint32_t first = 0xFFFFFFFFu;
                    bool ovf = false;
#pragma unroll
                    for (int c = 0; c < W; ++c) {
                        float tn;
                        if (child_hit<W>(nv, c, ray, ix, iy, iz, lim, tn)) {
                            uint32_t e = child_entry<W>(nv, (uint32_t)c);
                            if (first == 0xFFFFFFFFu) first = e;
                            else if (sp < kStack) stack[sp++] = make_uint2(e, 0u);
                            else ovf = true;
                        }
                    }
                    if (ovf) { status = kErrStackOverflow; break; }
                    if (first != 0xFFFFFFFFu) { cur = first; descend = true; }
                } else {
                    uint32_t keys[W];
                    int nhit = 0;
#pragma unroll
                    for (int c = 0; c < W; ++c) {
                        float tn;
                        bool h = child_hit<W>(nv, c, ray, ix, iy, iz, lim, tn);
                        keys[c] = h ? ((__float_as_uint(fmaxf(tn, 0.0f)) & ~7u) | (uint32_t)c) : 0xFFFFFFFFu;
                        nhit += h ? 1 : 0;
                    }
                    if (nhit > 0) {
                        sort_keys<W>(keys);
                        if (sp + nhit - 1 > kStack) { status = kErrStackOverflow; break; }
#pragma unroll
                        for (int j = W - 1; j >= 1; --j)
                            if (j < nhit) stack[sp++] = make_uint2(child_entry<W>(nv, keys[j] & 7u), keys[j] & ~7u);
                        cur = child_entry<W>(nv, keys[0] & 7u);
                        descend = true;
                    }
                }
            }
            if (descend) continue;
            bool found = false;
            while (sp > 0) {
                uint2 e = stack[--sp];
                if (kAny || __uint_as_float(e.y) < best_t) { cur = e.x; found = true; break; }
            }
            if (!found) break;
        }
    }
    if (status) atomicOr(err, status);
    if (kAny) {
        occ[i] = status ? kHitTraversalError : (occluded ? 1u : 0u);
    } else {
        if (status) store_hit(hits, i, kHitTraversalError, ray.tmax, 0.0f, 0.0f);
        else store_hit(hits, i, best, best == ILM_MISS ? ray.tmax : best_t, bu, bv);
    }
}

template <int W, int kStack>
cudaError_t launch_wide(const DeviceAccel& a, const ilm_ray* rays, uint64_t n, ilm_hit* hits, uint32_t* occ,
                        uint32_t* err, const LaunchParams& lp, cudaStream_t s) {
    unsigned block = 128;
    unsigned grid = (unsigned)((n + block - 1) / block);
    const uint4* nodes = reinterpret_cast<const uint4*>(a.nodes);
    if (occ)
        k_trace_wide<W, kStack, true><<<grid, block, 0, s>>>(nodes, a.n_nodes, a.prims, a.spheres, rays, n, hits,
                                                             occ, err, lp.max_iter);
    else
        k_trace_wide<W, kStack, false><<<grid, block, 0, s>>>(nodes, a.n_nodes, a.prims, a.spheres, rays, n, hits,
                                                              occ, err, lp.max_iter);
    return cudaGetLastError();
}

}  // namespace

bool kernels_loadable(cudaFuncAttributes* attr) {
    return cudaFuncGetAttributes(attr, k_trace_bin<false>) == cudaSuccess;
}

cudaError_t launch_trace(const DeviceAccel& a, const ilm_ray* rays, uint64_t n, ilm_hit* hits, uint32_t* occ,
                         uint32_t* err, const LaunchParams& lp, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    if (a.width == 2) {
        unsigned block = 128;
        unsigned grid = (unsigned)((n + block - 1) / block);
        const BinNode* nodes = reinterpret_cast<const BinNode*>(a.nodes);
        if (occ)
            k_trace_bin<true><<<grid, block, 0, s>>>(nodes, a.n_nodes, a.prims, a.spheres, rays, n, hits, occ, err,
                                                     lp.max_iter);
        else
            k_trace_bin<false><<<grid, block, 0, s>>>(nodes, a.n_nodes, a.prims, a.spheres, rays, n, hits, occ, err,
                                                      lp.max_iter);
        return cudaGetLastError();
    }
    bool deep = lp.stack_depth > 32;
    if (a.width == 8) return deep ? launch_wide<8, 64>(a, rays, n, hits, occ, err, lp, s)
                                  : launch_wide<8, 32>(a, rays, n, hits, occ, err, lp, s);
    return deep ? launch_wide<4, 64>(a, rays, n, hits, occ, err, lp, s)
                : launch_wide<4, 32>(a, rays, n, hits, occ, err, lp, s);
}

}  // namespace ilm
