// kd-tree ray queries: KdTreeAccel::intersect / intersect_p
// (accelerators/kdtreeaccel.rs:256-465).
//
// The ray's parametric range is clipped to the tree's bound
// (Bounds3::intersect_ray, geometry/bounds3.rs:253-282); each interior node
// sends the ray to the child on its origin's side of the split first and, when
// the split plane falls inside the current range, defers the other child with
// the range beyond the plane.  Traversal ends when the closest hit so far lies
// before the next range.  Every comparison keeps the reference's form, so a
// ray lying in a split plane (0 * inf = NaN plane distance) visits both
// children as the reference does.
//
// Deferred entries hold (node, t_min) only: an entry's t_max is always the
// t_min of the entry beneath it (the root range's end for the bottom one),
// because the range being traversed ends where the last deferred range
// starts.  The values restored are the reference's, bit for bit.
//
// Leaf runs test primitives by id (records are stored in id order).  The
// reference's multi-primitive leaf loop reads the run's second entry n times
// (`primitive_indices_offset + 1`, kdtreeaccel.rs:351 and 440); this loop
// reads entry k on iteration k.
//
// Schedules: one thread per ray (grid), or persistent warps that claim rays in
// chunks and refill finished lanes (the wide BVH kernels' scheme); every loop
// iteration advances a lane by one node or one leaf.  The pooled persistent
// kernel also splits its tail as the wide one does: once every ray is claimed,
// idle lanes take the top deferred entry of their warp's unfinished rays with
// its range (KdTracer::give / take).
#include "wide_tracer.cuh"

namespace ilm {

namespace {

// One slab of Bounds3::intersect_ray.
__device__ __forceinline__ bool clip_slab(float lo, float hi, float o, float inv, float& t0, float& t1) {
    float t_near = __fmul_rn(__fsub_rn(lo, o), inv);
    float t_far = __fmul_rn(__fsub_rn(hi, o), inv);
    if (t_near > t_far) {
        float s = t_near;
        t_near = t_far;
        t_far = s;
    }
    t_far = __fmul_rn(t_far, kBoxRobust);
    if (t_near > t0) t0 = t_near;
    if (t_far < t1) t1 = t_far;
    return !(t0 > t1);
}

__device__ __forceinline__ float pick(uint32_t axis, float x, float y, float z) {
    return axis == 0 ? x : (axis == 1 ? y : z);
}

constexpr int kKdBlock = 128;

template <bool kAny, bool kAnalytic>
struct KdTracer {
    RayIn ray;
    float ix, iy, iz;
    float t_min, t_max, t_root;      // current range; end of the root range
    float best_t, bu, bv;
    uint32_t best, status, cur, iter;
    int sp;
    bool tr_ready, occluded;
    TriRay tr;
    uint2* stack;                    // (node, t_min bits): the launching kernel's array of kKdMaxDepth

    // The stack stays outside the struct, for the reason WideTracerSorted's does.
    __device__ __forceinline__ explicit KdTracer(uint2* s) : stack(s) {}

    __device__ __forceinline__ void init(const RayIn& r) {
        ray = r;
        best_t = r.tmax; bu = 0.0f; bv = 0.0f;
        best = ILM_MISS;
        status = 0; cur = 0; iter = 0; sp = 0;
        tr_ready = false; occluded = false;
        ix = __frcp_rn(r.dx); iy = __frcp_rn(r.dy); iz = __frcp_rn(r.dz);   // == 1/d exactly
    }

    // The tree-bound clip of KdTreeAccel::intersect (kdtreeaccel.rs:258-264).
    __device__ __forceinline__ bool enters(const float* b) {
        t_min = 0.0f;
        t_max = ray.tmax;
        bool in = clip_slab(b[0], b[3], ray.ox, ix, t_min, t_max) && clip_slab(b[1], b[4], ray.oy, iy, t_min, t_max) &&
                  clip_slab(b[2], b[5], ray.oz, iz, t_min, t_max);
        t_root = t_max;
        return in;
    }

    // One node or one leaf; true when the ray is finished.
    __device__ __forceinline__ bool step(const TraceArgs& a) {
        if ((kAny ? ray.tmax : best_t) < t_min) return true;
        if (++iter > a.max_iter) { status = kErrIterationCap; return true; }
        const uint2 nd = __ldg(static_cast<const uint2*>(a.nodes) + cur);
        const uint32_t axis = nd.y & 3u;
        if (axis != kKdLeaf) {
            const float split = __uint_as_float(nd.x);
            const float o = pick(axis, ray.ox, ray.oy, ray.oz);
            const float d = pick(axis, ray.dx, ray.dy, ray.dz);
            const float t_plane = __fmul_rn(__fsub_rn(split, o), pick(axis, ix, iy, iz));
            const bool below_first = o < split || (o == split && d <= 0.0f);
            const uint32_t above = nd.y >> 2;
            const uint32_t first = below_first ? cur + 1 : above;
            const uint32_t second = below_first ? above : cur + 1;
            if (t_plane > t_max || t_plane <= 0.0f) {
                cur = first;
            } else if (t_plane < t_min) {
                cur = second;
            } else {
                if (sp == kKdMaxDepth) { status = kErrStackOverflow; return true; }
                stack[sp++] = make_uint2(second, __float_as_uint(t_plane));
                cur = first;
                t_max = t_plane;
            }
            return false;
        }
        const uint32_t n = nd.y >> 2;
        for (uint32_t k = 0; k < n; ++k) {
            const uint32_t r = n == 1 ? nd.x : __ldg(a.kd_index + nd.x + k);
            float t, u, v;
            uint32_t pid;
            if (kAny) {
                if (prim_test<false, kAnalytic>(a.prims, a.spheres, r, tr, tr_ready, ray, ray.tmax, t, u, v, pid)) {
                    occluded = true;
                    return true;
                }
            } else if (prim_test<true, kAnalytic>(a.prims, a.spheres, r, tr, tr_ready, ray, best_t, t, u, v, pid) &&
                       (t < best_t || (t == best_t && pid < best))) {
                best_t = t; best = pid; bu = u; bv = v;
            }
        }
        if (sp == 0) return true;
        --sp;
        cur = stack[sp].x;
        t_min = __uint_as_float(stack[sp].y);
        t_max = sp > 0 ? __uint_as_float(stack[sp - 1].y) : t_root;
        return false;
    }

    __device__ __forceinline__ void write(uint64_t i, const TraceArgs& a) const {
        if (status) atomicOr(a.err, status);
        if (kAny) {
            a.occ[i] = status ? kHitTraversalError : (occluded ? 1u : 0u);
        } else {
            if (status) store_hit(a.hits, i, kHitTraversalError, ray.tmax, 0.0f, 0.0f);
            else store_hit(a.hits, i, best, best == ILM_MISS ? ray.tmax : best_t, bu, bv);
        }
    }

    // Split tail (share_subtrees): stages the top deferred entry for another
    // lane with its range [its t_min, the t_min of the entry beneath or the
    // root range's end], the ray, its reciprocals, the best distance and the
    // owner lane; the donor's own ranges are unchanged, since the range it
    // traverses already ends where the given one starts.  take() adopts a
    // staging (false for an entry the donor's early exit would have skipped).
    __device__ __forceinline__ void give(uint4* s, uint32_t owner) {
        --sp;
        const uint2 e = stack[sp];
        const float lo = __uint_as_float(e.y);
        const float hi = sp > 0 ? __uint_as_float(stack[sp - 1].y) : t_root;
        const bool live = !((kAny ? ray.tmax : best_t) < lo);
        s[0] = make_uint4(live ? e.x : kNoEntry, __float_as_uint(ray.tmax), __float_as_uint(best_t), owner);
        s[1] = make_uint4(__float_as_uint(ray.ox), __float_as_uint(ray.oy), __float_as_uint(ray.oz),
                          __float_as_uint(ix));
        s[2] = make_uint4(__float_as_uint(ray.dx), __float_as_uint(ray.dy), __float_as_uint(ray.dz),
                          __float_as_uint(iy));
        s[3] = make_uint4(__float_as_uint(iz), __float_as_uint(lo), __float_as_uint(hi), 0u);
    }
    __device__ __forceinline__ bool take(const uint4* s, uint32_t& owner) {
        const uint4 h = s[0];
        if (h.x == kNoEntry) return false;
        const uint4 r0 = s[1], r1 = s[2], r2 = s[3];
        ray = RayIn{__uint_as_float(r0.x), __uint_as_float(r0.y), __uint_as_float(r0.z), __uint_as_float(r1.x),
                    __uint_as_float(r1.y), __uint_as_float(r1.z), __uint_as_float(h.y)};
        ix = __uint_as_float(r0.w); iy = __uint_as_float(r1.w); iz = __uint_as_float(r2.x);
        best_t = __uint_as_float(h.z); bu = 0.0f; bv = 0.0f;
        best = ILM_MISS;
        status = 0; iter = 0; sp = 0;
        tr_ready = false; occluded = false;
        cur = h.x;
        t_min = __uint_as_float(r2.y);
        t_max = t_root = __uint_as_float(r2.z);
        owner = h.w;
        return true;
    }
};

template <bool kAny, bool kAnalytic>
__global__ void __launch_bounds__(kKdBlock) k_trace_kd(TraceArgs a) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ray_count(a)) return;
    RayIn r = load_ray(a.rays, i);
    uint2 stk[kKdMaxDepth];
    KdTracer<kAny, kAnalytic> T(stk);
    T.init(r);
    if (a.n_nodes == 0 || !T.enters(a.bound)) { write_miss(i, r, a.hits, a.occ); return; }
    while (!T.step(a)) {}
    T.write(i, a);
}

// kPool: as in the wide kernel, the whole warp tests each claimed chunk
// against the tree's bound and pools the rays that enter (true), or each
// idle lane tests its own claims (false).
template <bool kAny, int kMinBlocks, bool kAnalytic, bool kPool>
__global__ void __launch_bounds__(kKdBlock, kMinBlocks) k_trace_kd_persistent(TraceArgs a) {
    const uint64_t n = ray_count(a);
    const unsigned chunk = n < 2ull * gridDim.x * blockDim.x ? 32u : kChunk;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned below = (1u << lane) - 1u;
    uint2 stk[kKdMaxDepth];
    KdTracer<kAny, kAnalytic> T(stk);
    bool exhausted = false;                             // warp-uniform
    if constexpr (kPool) {
        // The wide kernel's pooled schedule and split tail (share_subtrees,
        // merge_helpers; the lane roles of wide_tracer.cuh).
        __shared__ __align__(16) uint32_t s_warp[kKdBlock / 32][kWarpWords];
        uint32_t* warp_words = s_warp[threadIdx.x >> 5];
        uint32_t* pool = warp_words;                    // offsets of the pooled rays in their chunk
        uint32_t* ids = warp_words + kPoolWords;        // each lane's ray id (owners)
        unsigned pool_n = 0;                            // warp-uniform
        unsigned long long pool_base = 0;               // warp-uniform
        uint32_t st = kFree | (lane << 2);
        for (;;) {
            if (!exhausted) {
                unsigned need = __ballot_sync(0xFFFFFFFFu, role_of(st) == kFree);
                while (need != 0u) {
                    if (pool_n == 0) {
                        unsigned long long b = 0;
                        if (lane == 0) b = atomicAdd(a.counter, (unsigned long long)chunk);
                        b = __shfl_sync(0xFFFFFFFFu, b, 0);
                        if (b >= n) { exhausted = true; break; }
                        for (unsigned k = 0; k < chunk; k += 32u) {
                            const uint64_t rid = b + k + lane;
                            bool enter = false;
                            if (rid < n) {
                                const RayIn r = load_ray(a.rays, rid);
                                KdTracer<kAny, kAnalytic> probe(nullptr);   // root clip only: no stack
                                probe.init(r);
                                enter = a.n_nodes != 0 && probe.enters(a.bound);
                                if (!enter) write_miss(rid, r, a.hits, a.occ);
                            }
                            const unsigned m = __ballot_sync(0xFFFFFFFFu, enter);
                            if (enter) pool[pool_n + __popc(m & below)] = k + lane;
                            pool_n += __popc(m);
                        }
                        __syncwarp();
                        pool_base = b;
                        continue;
                    }
                    const unsigned rank = __popc(need & below);
                    const unsigned take = min((unsigned)__popc(need), pool_n);
                    if (((need >> lane) & 1u) && rank < take) {
                        const uint64_t id = pool_base + pool[pool_n - 1u - rank];
                        ids[2 * lane] = (uint32_t)id;
                        ids[2 * lane + 1] = (uint32_t)(id >> 32);
                        T.init(load_ray(a.rays, id));
                        T.enters(a.bound);              // true: the probe passed; sets the clip range
                        st = kOwner | (lane << 2);
                    }
                    pool_n -= take;
                    __syncwarp();
                    need = __ballot_sync(0xFFFFFFFFu, role_of(st) == kFree);
                }
            }
            const bool tail = exhausted && a.split_tail;   // warp-uniform
            bool owner_occluded = false;
            if (tail) {
                if (kAny) owner_occluded = __shfl_sync(0xFFFFFFFFu, (int)T.occluded, owner_of(st));
                share_subtrees<KdTracer<kAny, kAnalytic>, kAny>(T, st, owner_occluded, warp_words);
                if (kAny) owner_occluded = __shfl_sync(0xFFFFFFFFu, (int)T.occluded, owner_of(st));
            }
            if (!__any_sync(0xFFFFFFFFu, role_of(st) != kFree)) break;
            const uint32_t role = role_of(st);
            bool done = false;
            if ((role == kOwner || role == kHelper) && owner_occluded) done = true;
            else if (role == kOwner || role == kHelper) done = T.step(a);
            if (tail) {
                const unsigned fin = __ballot_sync(0xFFFFFFFFu, role == kHelper && done);
                if (fin) merge_helpers<KdTracer<kAny, kAnalytic>, kAny>(T, st, fin);
                if (role == kHelper && done) st = kFree | (lane << 2);
                if (role == kOwner && done) st = (st & ~3u) | kWaiting;
                if (role_of(st) == kWaiting && (st >> 8) == 0u) {
                    T.write((uint64_t)ids[2 * lane] | ((uint64_t)ids[2 * lane + 1] << 32), a);
                    st = kFree | (lane << 2);
                }
            } else if (done) {
                T.write((uint64_t)ids[2 * lane] | ((uint64_t)ids[2 * lane + 1] << 32), a);
                st = kFree | (lane << 2);
            }
        }
        return;
    }
    bool active = false;
    uint64_t id = 0;
    unsigned long long chunk_next = 0, chunk_end = 0;   // warp-uniform
    for (;;) {
        unsigned need = __ballot_sync(0xFFFFFFFFu, !active);
        // Hand rays to idle lanes; rays missing the tree's bound are answered
        // here.  Every pass hands out >= 1 ray or claims a chunk.
        while (need != 0u && !exhausted) {
            if (chunk_next == chunk_end) {
                unsigned long long b = 0;
                if (lane == 0) b = atomicAdd(a.counter, (unsigned long long)chunk);
                b = __shfl_sync(0xFFFFFFFFu, b, 0);
                if (b >= n) { exhausted = true; break; }
                chunk_next = b;
                chunk_end = b + chunk < n ? b + chunk : n;
            }
            unsigned avail = (unsigned)(chunk_end - chunk_next);
            unsigned rank = __popc(need & below);
            if (((need >> lane) & 1u) && rank < avail) {
                id = chunk_next + rank;
                RayIn r = load_ray(a.rays, id);
                T.init(r);
                if (a.n_nodes != 0 && T.enters(a.bound)) active = true;
                else write_miss(id, r, a.hits, a.occ);
            }
            chunk_next += min((unsigned)__popc(need), avail);
            need = __ballot_sync(0xFFFFFFFFu, !active);
        }
        if (!__any_sync(0xFFFFFFFFu, active)) break;   // only reached once exhausted
        if (active && T.step(a)) {
            T.write(id, a);
            active = false;
        }
    }
}

template <int kMinBlocks, bool kAnalytic, bool kPool>
cudaError_t launch_persistent(const TraceArgs& t, cudaStream_t s) {
    const unsigned block = kKdBlock;
    auto kc = k_trace_kd_persistent<false, kMinBlocks, kAnalytic, kPool>;
    auto ka = k_trace_kd_persistent<true, kMinBlocks, kAnalytic, kPool>;
    uint64_t grid = resident_blocks(t.occ ? (const void*)ka : (const void*)kc, (int)block);
    if (grid == 0) return cudaErrorInvalidConfiguration;
    const uint64_t need_blocks = (t.n + block - 1) / block;
    if (grid > need_blocks) grid = need_blocks;
    cudaError_t e = cudaMemsetAsync(t.counter, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    if (t.occ) ka<<<(unsigned)grid, block, 0, s>>>(t);
    else kc<<<(unsigned)grid, block, 0, s>>>(t);
    return cudaGetLastError();
}

template <bool kAnalytic>
cudaError_t launch_kd(const TraceArgs& t, const LaunchParams& lp, cudaStream_t s) {
    if (lp.persistent && t.counter) {
        if (lp.root_pool)
            return lp.min_blocks >= 8 ? launch_persistent<8, kAnalytic, true>(t, s)
                                      : launch_persistent<1, kAnalytic, true>(t, s);
        return lp.min_blocks >= 8 ? launch_persistent<8, kAnalytic, false>(t, s)
                                  : launch_persistent<1, kAnalytic, false>(t, s);
    }
    const unsigned block = kKdBlock;
    unsigned grid = (unsigned)((t.n + block - 1) / block);
    if (t.occ) k_trace_kd<true, kAnalytic><<<grid, block, 0, s>>>(t);
    else k_trace_kd<false, kAnalytic><<<grid, block, 0, s>>>(t);
    return cudaGetLastError();
}

}  // namespace

// Trees without quadric or curve records run the triangle-only variants.
cudaError_t launch_trace_kd(const TraceArgs& t, const LaunchParams& lp, cudaStream_t s) {
    return t.spheres ? launch_kd<true>(t, lp, s) : launch_kd<false>(t, lp, s);
}

}  // namespace ilm
