// Host-visible declarations of the kernel launchers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "illume_gpu.h"
#include "layout.h"

namespace ilm {

// Device view of one acceleration structure.
struct DeviceAccel {
    int width;                 // 2, 4, 8, or kLayoutKdTree
    const void* nodes;         // BinNode[], WideNode<W>[] or KdNode[]
    uint32_t n_nodes;
    const PrimRec* prims;      // traversal-ordered primitive records
    uint32_t n_records;
    const SphereRec* spheres;
    const uint32_t* kd_index;  // kd-tree leaf runs (null for the BVH layouts)
    float bound[6];            // world bound (root box), min xyz / max xyz
};

struct LaunchParams {
    int stack_depth;           // > 32 selects the 64-entry stack variant
    int block_size;
    uint32_t max_iter;         // per-ray loop cap
    int persistent;            // wide layouts: persistent schedule (needs `counter`)
    unsigned long long* counter;   // device work counter, private to the launch's stream
    int min_blocks;            // persistent kernel occupancy hint (8 = 64-register variant)
    int root_pool;             // persistent schedule: claimed chunks tested against the root box by the
                               // whole warp, entering rays pooled per warp (1), or each idle lane
                               // testing its own claims (0)
    int split_tail = 0;        // pooled persistent schedule: once the work counter has run out, idle
                               // lanes take stacked subtrees of their warp's unfinished rays
    int queue_split = 0;       // persistent queries with a device-side count (path queues): the
                               // one-thread-per-ray split kernel is launched beside the persistent
                               // one and answers counts of at most one wave; each kernel returns at
                               // once when the count is the other's
};

// Everything a trace kernel reads, passed by value.
struct TraceArgs {
    const void* nodes;
    uint32_t n_nodes;
    const PrimRec* prims;
    const SphereRec* spheres;
    const ilm_ray* rays;
    uint64_t n;                        // ray count (upper bound when n_dev is set)
    const unsigned long long* n_dev;   // optional device-side ray count
    ilm_hit* hits;                     // closest hit output (any-hit: null)
    uint32_t* occ;                     // any-hit output (closest: null)
    uint32_t* err;
    uint32_t max_iter;
    unsigned long long* counter;       // persistent-schedule work counter
    float bound[6];
    const uint32_t* kd_index;          // kd-tree leaf runs
    uint32_t split_tail = 0;           // LaunchParams::split_tail
    uint64_t small_max = 0;            // LaunchParams::queue_split: counts up to this go to the
                                       // one-thread-per-ray kernel (0: no such split)
    uint32_t warp_rays = 32;           // k_trace_wide_split: rays a warp starts with (16 or 32; 0: 16
                                       // when the count fits half the launch, else 32)
};

// occ == nullptr: closest hit into `hits`; otherwise any-hit into `occ`.
// When n_dev is non-null the kernels trace min(*n_dev, n) rays.
cudaError_t launch_trace(const DeviceAccel& a, const ilm_ray* rays, uint64_t n, ilm_hit* hits, uint32_t* occ,
                         uint32_t* err, const LaunchParams& lp, cudaStream_t s,
                         const unsigned long long* n_dev = nullptr);

cudaError_t launch_trace_binary(const TraceArgs& t, cudaStream_t s);
cudaError_t launch_trace_kd(const TraceArgs& t, const LaunchParams& lp, cudaStream_t s);
cudaError_t launch_trace_wide(int width, const TraceArgs& t, const LaunchParams& lp, cudaStream_t s);
// Rays that one wave of the one-thread-per-ray wide kernel holds resident on
// the current device (0 when unknown).
uint64_t wide_grid_wave(int width, int stack_depth);

// SMs x resident blocks per SM of `kernel` at `block` threads on the current
// device (at least one block per SM), cached per (device, kernel) and safe to
// call from several host threads; 0 when the query fails.
uint64_t resident_blocks(const void* kernel, int block);

}  // namespace ilm
