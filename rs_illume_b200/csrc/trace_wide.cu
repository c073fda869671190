// Wide-BVH ray queries (W = 4 or 8 children per node); the traversal state
// is WideTracer (wide_tracer.cuh).
//
// Schedules:
//  * grid: one thread per ray.
//  * persistent (default): a grid sized to fill the GPU once; each warp claims
//    rays 64 at a time (32 for short queues) from a device counter and hands
//    them to lanes that are free.  A claimed ray is first tested against the
//    scene's root box; rays that miss it (most incoherent rays) are answered
//    at once and never occupy a lane (see k_trace_wide_persistent's kPool for
//    the two ways of doing so).  Each loop iteration advances every busy lane
//    by exactly one node or one leaf, then refills finished lanes, so a warp
//    stays full while its rays differ in length.
//  * split tail (pooled persistent kernel once every ray is claimed, and the
//    one-thread-per-ray kernel k_trace_wide_split throughout): idle lanes
//    take stacked subtrees of their warp's unfinished rays (share_subtrees in
//    wide_tracer.cuh), so a launch does not wait on its longest rays alone.
#include <algorithm>

#include "wide_tracer.cuh"

namespace ilm {

namespace {

template <int W, int kStack, bool kAny, bool kAnalytic>
__global__ void __launch_bounds__(128) k_trace_wide(TraceArgs a) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ray_count(a)) return;
    RayIn r = load_ray(a.rays, i);
    using Tracer = WideTracer<W, kStack, kAny, kAnalytic>;
    typename Tracer::Entry stk[Tracer::kDepth];
    Tracer T(stk);
    T.init(r);
    if (a.n_nodes == 0 || !T.enters(a.bound)) { write_miss(i, r, a.hits, a.occ); return; }
    while (!T.step(a)) {}
    T.write(i, a);
}

// One thread per ray with the split tail from the start: a lane whose ray
// missed the scene's root box or has finished takes subtrees of its warp's
// unfinished rays (share_subtrees).  A one-wave query is all tail: its
// launch lasts as long as its longest rays.
template <int W, int kStack, bool kAny, bool kAnalytic>
__global__ void __launch_bounds__(128) k_trace_wide_split(TraceArgs a) {
    const unsigned lane = threadIdx.x & 31u;
    // Lane `lane` < warp_rays of warp w starts on ray w * warp_rays + lane;
    // the other lanes start idle and help from the first pass.
    __shared__ __align__(16) uint32_t s_warp[4][kWarpWords];
    uint32_t* warp_words = s_warp[threadIdx.x >> 5];
    uint32_t* ids = warp_words + kPoolWords;
    using Tracer = WideTracer<W, kStack, kAny, kAnalytic>;
    typename Tracer::Entry stk[Tracer::kDepth];
    Tracer T(stk);
    uint32_t st = kFree | (lane << 2);
    const uint64_t n = ray_count(a);
    if (a.small_max && n > a.small_max) return;   // the persistent launch beside this one has it
    const uint32_t warp_rays = a.warp_rays ? a.warp_rays
                                           : (2 * n <= (uint64_t)gridDim.x * blockDim.x ? 16u : 32u);
    const uint64_t warp_id = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t i = warp_id * warp_rays + lane;
    if (lane < warp_rays && i < n) {
        const RayIn r = load_ray(a.rays, i);
        T.init(r);
        if (a.n_nodes != 0 && T.enters(a.bound)) {
            ids[2 * lane] = (uint32_t)i;
            ids[2 * lane + 1] = (uint32_t)(i >> 32);
            st = kOwner | (lane << 2);
        } else {
            write_miss(i, r, a.hits, a.occ);
        }
    }
    for (;;) {
        bool owner_occluded = kAny && __shfl_sync(0xFFFFFFFFu, (int)T.occluded, owner_of(st));
        share_subtrees<Tracer, kAny>(T, st, owner_occluded, warp_words);
        if (kAny) owner_occluded = __shfl_sync(0xFFFFFFFFu, (int)T.occluded, owner_of(st));
        if (!__any_sync(0xFFFFFFFFu, role_of(st) != kFree)) break;
        const uint32_t role = role_of(st);
        bool done = false;
        if ((role == kOwner || role == kHelper) && owner_occluded) done = true;
        else if (role == kOwner || role == kHelper) done = T.step(a);
        const unsigned fin = __ballot_sync(0xFFFFFFFFu, role == kHelper && done);
        if (fin) merge_helpers<Tracer, kAny>(T, st, fin);
        if (role == kHelper && done) st = kFree | (lane << 2);
        if (role == kOwner && done) st = (st & ~3u) | kWaiting;
        if (role_of(st) == kWaiting && (st >> 8) == 0u) {
            T.write((uint64_t)ids[2 * lane] | ((uint64_t)ids[2 * lane + 1] << 32), a);
            st = kFree | (lane << 2);
        }
    }
}

// kMinBlocks > 0 asks the compiler for that many resident 128-thread blocks
// per SM (the high-occupancy build: 7 for the pooled kernel, up to 72
// registers; 8 for the lane-refill kernel, 64 registers).
// kPool selects how claimed rays reach idle lanes:
//  * true: the whole warp tests each claimed chunk against the root box, two
//    rays per lane, answers the misses at full width, and keeps the rays that
//    enter in a per-warp pool in shared memory; idle lanes take rays from the
//    pool.  For incoherent batches most rays miss the scene, and this keeps
//    the lanes that are still traversing from waiting while a few idle lanes
//    test misses one at a time (5,330 against 4,420 Mrays/s on the 2M-ray
//    ball workload).  This kernel carries the split tail.
//  * false: each idle lane tests its own claims, repeating until one enters
//    (ILM_FLAG_LANE_REFILL); no split tail.
template <int W, int kStack, bool kAny, int kMinBlocks, bool kAnalytic, bool kPool>
__global__ void __launch_bounds__(128, kMinBlocks) k_trace_wide_persistent(TraceArgs a) {
    const uint64_t n = ray_count(a);
    if (n <= a.small_max) return;                  // the one-thread-per-ray launch beside this one has it
    // A short queue (fewer than two rays per resident lane) is claimed one ray
    // per lane, so that its rays run side by side rather than two per lane.
    const unsigned chunk = n < 2ull * gridDim.x * blockDim.x ? 32u : kChunk;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned below = (1u << lane) - 1u;
    using Tracer = WideTracer<W, kStack, kAny, kAnalytic>;
    typename Tracer::Entry stk[Tracer::kDepth];
    Tracer T(stk);
    bool exhausted = false;                             // warp-uniform
    if constexpr (kPool) {
        __shared__ __align__(16) uint32_t s_warp[4][kWarpWords];
        uint32_t* warp_words = s_warp[threadIdx.x >> 5];
        uint32_t* pool = warp_words;                    // offsets of the pooled rays in their chunk
        uint32_t* ids = warp_words + kPoolWords;        // each lane's ray id (owners)
        unsigned pool_n = 0;                            // warp-uniform
        unsigned long long pool_base = 0;               // warp-uniform: the pooled rays' chunk
        uint32_t st = kFree | (lane << 2);
        for (;;) {
            if (!exhausted) {
                unsigned need = __ballot_sync(0xFFFFFFFFu, role_of(st) == kFree);
                // Every pass either hands out pooled rays or claims and filters
                // a chunk (claims are only made with an empty pool), so the
                // loop ends.
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
                                enter = a.n_nodes != 0 && root_enters(r, a.bound);
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
                        st = kOwner | (lane << 2);
                    }
                    pool_n -= take;
                    __syncwarp();
                    need = __ballot_sync(0xFFFFFFFFu, role_of(st) == kFree);
                }
            }
            // Subtrees are shared once the counter has run out (warp-uniform).
            // Before that every busy lane is an owner, and the closest-hit
            // kernel skips the helpers' bookkeeping (measured 1 % faster); the
            // any-hit kernel keeps it throughout (2 % faster that way).
            const bool split_now = exhausted && a.split_tail;
            const bool tail = kAny || split_now;
            // A helper of an occluded any-hit ray has nothing left to find.
            bool owner_occluded = kAny && __shfl_sync(0xFFFFFFFFu, (int)T.occluded, owner_of(st));
            if (split_now) {
                share_subtrees<Tracer, kAny>(T, st, owner_occluded, warp_words);
                // Lanes that just took a subtree have a new owner.
                if (kAny) owner_occluded = __shfl_sync(0xFFFFFFFFu, (int)T.occluded, owner_of(st));
            }
            if (!__any_sync(0xFFFFFFFFu, role_of(st) != kFree)) break;   // only once exhausted
            const uint32_t role = role_of(st);
            bool done = false;
            // An any-hit ray one of its helpers found occluded is finished.
            if ((role == kOwner || role == kHelper) && owner_occluded) done = true;
            else if (role == kOwner || role == kHelper) done = T.step(a);
            if (tail) {
                const unsigned fin = __ballot_sync(0xFFFFFFFFu, role == kHelper && done);
                if (fin) merge_helpers<Tracer, kAny>(T, st, fin);
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
    } else {
        bool active = false;
        uint64_t id = 0;
        unsigned long long chunk_next = 0, chunk_end = 0;   // warp-uniform
        for (;;) {
            unsigned need = __ballot_sync(0xFFFFFFFFu, !active);
            // Hand rays to idle lanes; rays missing the root box are answered here.
            // Every pass hands out >= 1 ray or claims a chunk, so the loop ends.
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
}

template <int W, int kStack, int kMinBlocks, bool kAnalytic, bool kPool>
cudaError_t launch_persistent(const TraceArgs& t, cudaStream_t s) {
    const unsigned block = 128;
    auto kc = k_trace_wide_persistent<W, kStack, false, kMinBlocks, kAnalytic, kPool>;
    auto ka = k_trace_wide_persistent<W, kStack, true, kMinBlocks, kAnalytic, kPool>;
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

template <int W, int kStack, int kMinBlocks, bool kAnalytic>
cudaError_t launch_pooled(const TraceArgs& t, const LaunchParams& lp, cudaStream_t s) {
    // High occupancy: the pooled kernel at 7 resident blocks per SM (up to 72
    // registers: its split tail's state fits without spills; 8,063-8,070
    // against 7,699-7,704 Mrays/s closest hit at 8 blocks), the lane-refill
    // kernel at 8 (64 registers, no spills).
    constexpr int kPooledBlocks = kMinBlocks >= 8 ? 7 : kMinBlocks;
    return lp.root_pool ? launch_persistent<W, kStack, kPooledBlocks, kAnalytic, true>(t, s)
                        : launch_persistent<W, kStack, kMinBlocks, kAnalytic, false>(t, s);
}

template <int W, int kStack, bool kAnalytic>
cudaError_t launch_variant(const TraceArgs& t, const LaunchParams& lp, cudaStream_t s) {
    const unsigned block = 128;
    if (lp.persistent && t.counter) {
        if (lp.queue_split && t.n_dev && t.split_tail) {
            // A queue whose count is known on the device only: a count of at
            // most one wave of the split kernel runs there (all of its rays
            // resident at once, idle lanes helping from the start), a larger
            // one on the persistent kernel.
            auto kc = k_trace_wide_split<W, kStack, false, kAnalytic>;
            auto ka = k_trace_wide_split<W, kStack, true, kAnalytic>;
            const uint64_t wave_blocks = resident_blocks(t.occ ? (const void*)ka : (const void*)kc, (int)block);
            const uint64_t blocks = std::min<uint64_t>(wave_blocks, (t.n + block - 1) / block);
            if (blocks > 0) {
                TraceArgs q = t;
                q.small_max = blocks * block;
                q.warp_rays = 0;                    // 16 rays a warp when the count allows
                if (t.occ) ka<<<(unsigned)blocks, block, 0, s>>>(q);
                else kc<<<(unsigned)blocks, block, 0, s>>>(q);
                cudaError_t e = cudaGetLastError();
                if (e != cudaSuccess) return e;
                return lp.min_blocks >= 8 ? launch_pooled<W, kStack, 8, kAnalytic>(q, lp, s)
                                          : launch_pooled<W, kStack, 1, kAnalytic>(q, lp, s);
            }
        }
        return lp.min_blocks >= 8 ? launch_pooled<W, kStack, 8, kAnalytic>(t, lp, s)
                                  : launch_pooled<W, kStack, 1, kAnalytic>(t, lp, s);
    }
    unsigned grid = (unsigned)((t.n + block - 1) / block);
    if (t.split_tail) {
        // A query that fits half a wave starts each warp with 16 rays, so
        // that half its lanes help from the first pass.
        auto kc = k_trace_wide_split<W, kStack, false, kAnalytic>;
        auto ka = k_trace_wide_split<W, kStack, true, kAnalytic>;
        const uint64_t wave = resident_blocks(t.occ ? (const void*)ka : (const void*)kc, (int)block) * block;
        TraceArgs q = t;
        q.warp_rays = 2 * t.n <= wave ? 16u : 32u;
        const uint64_t rays_per_block = (uint64_t)q.warp_rays * (block / 32);
        const unsigned g = (unsigned)((t.n + rays_per_block - 1) / rays_per_block);
        if (t.occ) ka<<<g, block, 0, s>>>(q);
        else kc<<<g, block, 0, s>>>(q);
        return cudaGetLastError();
    }
    if (t.occ) k_trace_wide<W, kStack, true, kAnalytic><<<grid, block, 0, s>>>(t);
    else k_trace_wide<W, kStack, false, kAnalytic><<<grid, block, 0, s>>>(t);
    return cudaGetLastError();
}

// Accels without quadric or curve records run the triangle-only variants.
template <int W, int kStack>
cudaError_t launch(const TraceArgs& t, const LaunchParams& lp, cudaStream_t s) {
    return t.spheres ? launch_variant<W, kStack, true>(t, lp, s) : launch_variant<W, kStack, false>(t, lp, s);
}

}  // namespace

uint64_t wide_grid_wave(int width, int stack_depth) {
    const bool w8 = width == 8, deep = stack_depth > 32;
    const void* k = w8 ? (deep ? (const void*)k_trace_wide<8, 64, false, true> : (const void*)k_trace_wide<8, 32, false, true>)
                       : (deep ? (const void*)k_trace_wide<4, 64, false, true> : (const void*)k_trace_wide<4, 32, false, true>);
    return resident_blocks(k, 128) * 128u;
}

cudaError_t launch_trace_wide(int width, const TraceArgs& t, const LaunchParams& lp, cudaStream_t s) {
    bool deep = lp.stack_depth > 32;
    if (width == 8) return deep ? launch<8, 64>(t, lp, s) : launch<8, 32>(t, lp, s);
    return deep ? launch<4, 64>(t, lp, s) : launch<4, 32>(t, lp, s);
}

}  // namespace ilm
