// Batched ray queries: many scenes, each with its own ray batch of any size,
// in one persistent launch per BVH width (2, 4 or 8).
//
// The batches are concatenated into one index space.  Warps claim rays 64 at a
// time from a device counter as in the single-scene persistent kernel; each
// lane finds its ray's batch by binary search over the batch start offsets and
// traverses that batch's BVH, so lanes of one warp may serve different scenes
// and a small batch never leaves the GPU partly idle.  A plan (scene table +
// launch sequence) is captured once as a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <vector>

#include "context.h"
#include "illume_gpu.h"
#include "wide_tracer.cuh"

namespace ilm {

// One batch in the device table.
struct BatchEntry {
    const void* nodes;
    const PrimRec* prims;
    const SphereRec* spheres;
    const ilm_ray* rays;
    ilm_hit* hits;
    uint32_t* occ;
    unsigned long long first;   // index of the batch's first ray in the concatenation
    unsigned long long n;
    uint32_t n_nodes;
    uint32_t pad;
    float bound[6];
};

struct BatchTable {
    const BatchEntry* entries;
    uint32_t n_batches;
    unsigned long long total;
    uint32_t* err;
    uint32_t max_iter;
    unsigned long long* counter;
};

namespace {

__device__ __forceinline__ uint32_t find_batch(const BatchTable& t, unsigned long long g) {
    uint32_t lo = 0, hi = t.n_batches;   // largest b with entries[b].first <= g
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&t.entries[mid].first) <= g) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ TraceArgs args_of(const BatchTable& t, uint32_t b) {
    const BatchEntry& e = t.entries[b];
    TraceArgs a;
    a.nodes = e.nodes;
    a.n_nodes = e.n_nodes;
    a.prims = e.prims;
    a.spheres = e.spheres;
    a.rays = e.rays;
    a.n = e.n;
    a.n_dev = nullptr;
    a.hits = e.hits;
    a.occ = e.occ;
    a.err = t.err;
    a.max_iter = t.max_iter;
    a.counter = t.counter;
#pragma unroll
    for (int k = 0; k < 6; ++k) a.bound[k] = e.bound[k];
    return a;
}

// Rays are claimed from the concatenation 64 at a time.  The whole warp
// tests each claimed chunk against the root boxes of the rays' scenes (two
// rays per lane), answers the misses at full width and keeps the rays that
// enter in a per-warp pool in shared memory, from which idle lanes take rays
// (the single-scene kernel's kPool schedule).  7 resident blocks per SM (up
// to 72 registers, no spills of the per-lane scene arguments): 4,880-4,896
// against 4,806-4,810 Mrays/s at 8 blocks (64 registers) on the 32-scene set.
template <int W, int kStack, bool kAny, bool kAnalytic>
__global__ void __launch_bounds__(128, 7) k_trace_batched(BatchTable tab) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned below = (1u << lane) - 1u;
    __shared__ uint32_t s_pool[4][kChunk];              // per warp: offsets of the pooled rays in their chunk
    uint32_t* pool = s_pool[threadIdx.x >> 5];
    unsigned pool_n = 0;                                // warp-uniform
    unsigned long long pool_base = 0;                   // warp-uniform
    using Tracer = WideTracer<W, kStack, kAny, kAnalytic>;
    typename Tracer::Entry stk[Tracer::kDepth];
    Tracer T(stk);
    TraceArgs a;
    bool active = false;
    uint64_t id = 0;
    bool exhausted = false;                             // warp-uniform
    const unsigned long long n = tab.total;
    for (;;) {
        unsigned need = __ballot_sync(0xFFFFFFFFu, !active);
        while (need != 0u) {
            if (pool_n == 0) {
                if (exhausted) break;
                unsigned long long b = 0;
                if (lane == 0) b = atomicAdd(tab.counter, (unsigned long long)kChunk);
                b = __shfl_sync(0xFFFFFFFFu, b, 0);
                if (b >= n) { exhausted = true; break; }
                for (unsigned k = 0; k < kChunk; k += 32u) {
                    const unsigned long long g = b + k + lane;
                    bool enter = false;
                    if (g < n) {
                        const BatchEntry& e = tab.entries[find_batch(tab, g)];
                        const uint64_t rid = g - e.first;
                        const RayIn r = load_ray(e.rays, rid);
                        enter = e.n_nodes != 0 && root_enters(r, e.bound);
                        if (!enter) write_miss(rid, r, e.hits, e.occ);
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
                const unsigned long long g = pool_base + pool[pool_n - 1u - rank];
                const uint32_t bi = find_batch(tab, g);
                a = args_of(tab, bi);
                id = g - tab.entries[bi].first;
                T.init(load_ray(a.rays, id));
                active = true;
            }
            pool_n -= take;
            __syncwarp();
            need = __ballot_sync(0xFFFFFFFFu, !active);
        }
        if (!__any_sync(0xFFFFFFFFu, active)) break;   // only once exhausted with an empty pool
        if (active && T.step(a)) {
            T.write(id, a);
            active = false;
        }
    }
}

template <int W, int kStack, bool kAnalytic>
cudaError_t launch_batched_variant(const BatchTable& t, bool any, cudaStream_t s) {
    const unsigned block = 128;
    auto kc = k_trace_batched<W, kStack, false, kAnalytic>;
    auto ka = k_trace_batched<W, kStack, true, kAnalytic>;
    const uint64_t resident = resident_blocks(any ? (const void*)ka : (const void*)kc, (int)block);
    if (resident == 0) return cudaErrorInvalidConfiguration;
    uint64_t grid = std::min<uint64_t>(resident, (t.total + block - 1) / block);
    if (grid == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(t.counter, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    if (any) ka<<<(unsigned)grid, block, 0, s>>>(t);
    else kc<<<(unsigned)grid, block, 0, s>>>(t);
    return cudaGetLastError();
}

// Tables without quadric or curve records run the triangle-only variant.
template <int W, int kStack>
cudaError_t launch_batched(const BatchTable& t, bool any, bool analytic, cudaStream_t s) {
    return analytic ? launch_batched_variant<W, kStack, true>(t, any, s)
                    : launch_batched_variant<W, kStack, false>(t, any, s);
}

}  // namespace
}  // namespace ilm

using namespace ilm;

// A captured batch: one sub-table per (BVH width, stack depth) present.
struct ilm_batch_plan {
    struct Group {
        int width;
        bool deep = true;        // 64-entry stack (else 32); binary nodes always 64
        bool analytic = false;   // some accel holds quadric or curve records
        DeviceBuffer table, counter;
        BatchTable t;
    };
    std::vector<std::unique_ptr<Group>> groups;
    bool any = false;
    cudaStream_t capture = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t total_rays = 0;
    ~ilm_batch_plan() {
        if (exec) cudaGraphExecDestroy(exec);
        if (capture) cudaStreamDestroy(capture);
    }
};

namespace {

cudaError_t launch_plan(const ilm_batch_plan& p, cudaStream_t s) {
    for (const auto& g : p.groups) {
        cudaError_t e;
        const bool deep = g->deep;
        const bool an = g->analytic;
        if (g->width == 8)
            e = deep ? launch_batched<8, 64>(g->t, p.any, an, s) : launch_batched<8, 32>(g->t, p.any, an, s);
        else if (g->width == 4)
            e = deep ? launch_batched<4, 64>(g->t, p.any, an, s) : launch_batched<4, 32>(g->t, p.any, an, s);
        else   // binary nodes: the reference's 64-entry stack
            e = launch_batched<2, 64>(g->t, p.any, an, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int32_t build_plan(ilm_context* ctx, const ilm_batch_desc* batches, uint32_t n, int32_t any_hit,
                   std::unique_ptr<ilm_batch_plan>& out) {
    auto plan = std::make_unique<ilm_batch_plan>();
    plan->any = any_hit != 0;
    // sub-tables by width (2, 4, 8) and stack depth (32, 64): an accel's own
    // stack depth (ilm_accel_set_launch, ilm_autotune), else the context's
    const int widths[3] = {2, 4, 8};
    std::vector<BatchEntry> per_width[3][2];
    for (uint32_t i = 0; i < n; ++i) {
        const ilm_batch_desc& b = batches[i];
        Accel* a = find_accel(ctx, b.accel);
        if (!a) { set_error(ctx, "batched: unknown accel id"); return ILM_ERR_NOT_FOUND; }
        int w = a->host.width;
        if (w != 2 && w != 4 && w != 8) {
            set_error(ctx, "batched: accels must be BVHs of width 2, 4 or 8 (not kd-trees)");
            return ILM_ERR_INVALID_ARGUMENT;
        }
        void* out_ptr = plan->any ? (void*)b.occluded : (void*)b.hits;
        if (b.n > 0 && (!b.rays || !out_ptr || classify(b.rays) != PtrKind::kDevice ||
                        classify(out_ptr) != PtrKind::kDevice || ((uintptr_t)b.rays & 15u) ||
                        (!plan->any && ((uintptr_t)b.hits & 15u)) || (plan->any && ((uintptr_t)b.occluded & 3u)))) {
            set_error(ctx, "batched: rays and results must be 16-byte aligned device buffers");
            return ILM_ERR_INVALID_ARGUMENT;
        }
        if (b.n == 0) continue;
        DeviceAccel da = a->view();
        BatchEntry e;
        e.nodes = da.nodes;
        e.prims = da.prims;
        e.spheres = da.spheres;
        e.rays = b.rays;
        e.hits = plan->any ? nullptr : b.hits;
        e.occ = plan->any ? b.occluded : nullptr;
        e.n = b.n;
        e.n_nodes = da.n_nodes;
        e.pad = 0;
        for (int k = 0; k < 6; ++k) e.bound[k] = da.bound[k];
        const int depth = a->stack_depth > 0 ? a->stack_depth : ctx->stack_depth;
        per_width[w == 2 ? 0 : (w == 4 ? 1 : 2)][w == 2 || depth > 32].push_back(e);
    }
    for (int k = 0; k < 6; ++k) {
        auto& v = per_width[k / 2][k % 2];
        if (v.empty()) continue;
        unsigned long long first = 0;
        for (auto& e : v) { e.first = first; first += e.n; }
        auto g = std::make_unique<ilm_batch_plan::Group>();
        g->width = widths[k / 2];
        g->deep = (k % 2) != 0;
        for (const auto& e : v) g->analytic = g->analytic || e.spheres != nullptr;
        cudaError_t ce = g->table.reserve(v.size() * sizeof(BatchEntry));
        if (ce == cudaSuccess) ce = g->counter.reserve(sizeof(unsigned long long));
        if (ce == cudaSuccess) ce = cudaMemcpy(g->table.ptr, v.data(), v.size() * sizeof(BatchEntry), cudaMemcpyHostToDevice);
        if (ce != cudaSuccess) return cuda_fail(ctx, ce, "batched: table upload");
        g->t.entries = static_cast<const BatchEntry*>(g->table.ptr);
        g->t.n_batches = (uint32_t)v.size();
        g->t.total = first;
        g->t.err = static_cast<uint32_t*>(ctx->err_word.ptr);
        g->t.max_iter = ctx->max_iter;
        g->t.counter = static_cast<unsigned long long*>(g->counter.ptr);
        plan->total_rays += first;
        plan->groups.push_back(std::move(g));
    }
    out = std::move(plan);
    return ILM_OK;
}

}  // namespace

extern "C" {

int32_t ilm_batch_plan_create(ilm_context* ctx, const ilm_batch_desc* batches, uint32_t n, int32_t any_hit,
                              ilm_batch_plan** out) {
    if (!ctx || !out || (n > 0 && !batches)) return ILM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ILM_ERR_CUDA;
    std::unique_ptr<ilm_batch_plan> plan;
    int32_t st = build_plan(ctx, batches, n, any_hit, plan);
    if (st != ILM_OK) return st;
    cudaError_t e = cudaStreamCreateWithFlags(&plan->capture, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamCreate");
    // one eager run does the launchers' one-time setup outside the capture
    if ((e = launch_plan(*plan, plan->capture)) != cudaSuccess) return cuda_fail(ctx, e, "batched launch");
    if ((e = cudaStreamSynchronize(plan->capture)) != cudaSuccess) return cuda_fail(ctx, e, "batched launch");
    cudaGraph_t g;
    if ((e = cudaStreamBeginCapture(plan->capture, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
        return cuda_fail(ctx, e, "cudaStreamBeginCapture");
    cudaError_t le = launch_plan(*plan, plan->capture);
    e = cudaStreamEndCapture(plan->capture, &g);
    if (le != cudaSuccess) return cuda_fail(ctx, le, "batched capture");
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&plan->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGraphInstantiate");
    *out = plan.release();
    return ILM_OK;
}

int32_t ilm_batch_plan_launch(ilm_context* ctx, ilm_batch_plan* plan, void* stream) {
    if (!ctx || !plan) return ILM_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ILM_ERR_CUDA;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    cudaError_t e = cudaGraphLaunch(plan->exec, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGraphLaunch");
    return ILM_OK;
}

int32_t ilm_batch_plan_destroy(ilm_context* ctx, ilm_batch_plan* plan) {
    if (!ctx || !plan) return ILM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    delete plan;
    return ILM_OK;
}

int32_t ilm_intersect_batched(ilm_context* ctx, const ilm_batch_desc* batches, uint32_t n, int32_t any_hit,
                              void* stream) {
    if (!ctx || (n > 0 && !batches)) return ILM_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ILM_ERR_CUDA;
    std::unique_ptr<ilm_batch_plan> plan;
    int32_t st = build_plan(ctx, batches, n, any_hit, plan);
    if (st != ILM_OK) return st;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    cudaError_t e = launch_plan(*plan, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batched launch");
    // the plan's table and counters must outlive the launch
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(ctx, e, "batched launch");
    return ILM_OK;
}

}  // extern "C"
