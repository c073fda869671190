// Host-visible declarations of the kernel launchers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "illume_gpu.h"
#include "layout.h"

namespace ilm {

// Device view of one acceleration structure.
struct DeviceAccel {
    int width;                 // 2, 4, 8
    const void* nodes;         // BinNode[] or WideNode<W>[]
    uint32_t n_nodes;
    const PrimRec* prims;      // traversal-ordered primitive records
    uint32_t n_records;
    const SphereRec* spheres;
};

struct LaunchParams {
    int stack_depth;           // > 32 selects the 64-entry stack variant
    int block_size;
    uint32_t max_iter;         // per-ray loop cap
};

// occ == nullptr: closest hit into `hits`; otherwise any-hit into `occ`.
cudaError_t launch_trace(const DeviceAccel& a, const ilm_ray* rays, uint64_t n, ilm_hit* hits, uint32_t* occ,
                         uint32_t* err, const LaunchParams& lp, cudaStream_t s);

}  // namespace ilm
