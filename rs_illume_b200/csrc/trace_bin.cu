// Binary-BVH ray queries: the reference's 32-byte LinearBVHNode layout and
// its ordered stack traversal (accelerators/bvh.rs:563-662), one thread per
// ray.  The near child is the one selected by dir_is_neg[axis]; the far one is
// pushed on a 64-entry stack (bvh.rs:573).
#include "trace_common.cuh"

namespace ilm {

namespace {

template <bool kAny>
__global__ void __launch_bounds__(128) k_trace_bin(TraceArgs a) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ray_count(a)) return;
    const BinNode* __restrict__ nodes = static_cast<const BinNode*>(a.nodes);
    RayIn ray = load_ray(a.rays, i);
    float best_t = ray.tmax, bu = 0.0f, bv = 0.0f;
    uint32_t best = ILM_MISS;
    bool occluded = false;
    uint32_t status = 0;
    if (a.n_nodes > 0) {
        TriRay tr;
        bool tr_ready = false;
        float ix = __frcp_rn(ray.dx), iy = __frcp_rn(ray.dy), iz = __frcp_rn(ray.dz);   // == 1/d exactly
        bool negx = ix < 0.0f, negy = iy < 0.0f, negz = iz < 0.0f;
        uint32_t stack[64];
        int sp = 0;
        uint32_t cur = 0, iter = 0;
        for (;;) {
            if (++iter > a.max_iter) { status = kErrIterationCap; break; }
            const float4* np = reinterpret_cast<const float4*>(nodes + cur);
            float4 n0 = __ldg(np), n1 = __ldg(np + 1);
            // n0 = (minx, miny, minz, maxx), n1 = (maxy, maxz, offset, n_prims | axis << 16)
            if (box_intersect_p(n0.x, n0.y, n0.z, n0.w, n1.x, n1.y, ray, ix, iy, iz, negx, negy, negz,
                                kAny ? ray.tmax : best_t)) {
                uint32_t meta = __float_as_uint(n1.w);
                uint32_t nprims = meta & 0xFFFFu;
                uint32_t off = __float_as_uint(n1.z);
                if (nprims > 0) {
                    for (uint32_t k = 0; k < nprims; ++k) {
                        float t, u, v;
                        uint32_t pid;
                        if (kAny) {
                            if (prim_test<false>(a.prims, a.spheres, off + k, tr, tr_ready, ray, ray.tmax, t, u, v,
                                                 pid)) {
                                occluded = true;
                                break;
                            }
                        } else if (prim_test<true>(a.prims, a.spheres, off + k, tr, tr_ready, ray, best_t, t, u, v,
                                                   pid) &&
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
    if (status) atomicOr(a.err, status);
    if (kAny) {
        a.occ[i] = status ? kHitTraversalError : (occluded ? 1u : 0u);
    } else {
        if (status) store_hit(a.hits, i, kHitTraversalError, ray.tmax, 0.0f, 0.0f);
        else store_hit(a.hits, i, best, best == ILM_MISS ? ray.tmax : best_t, bu, bv);
    }
}

}  // namespace

bool kernels_loadable(cudaFuncAttributes* attr) {
    return cudaFuncGetAttributes(attr, k_trace_bin<false>) == cudaSuccess;
}

cudaError_t launch_trace_binary(const TraceArgs& t, cudaStream_t s) {
    const unsigned block = 128;
    unsigned grid = (unsigned)((t.n + block - 1) / block);
    if (t.occ) k_trace_bin<true><<<grid, block, 0, s>>>(t);
    else k_trace_bin<false><<<grid, block, 0, s>>>(t);
    return cudaGetLastError();
}

}  // namespace ilm
