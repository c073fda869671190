// Dispatch of the ray-query kernels (trace_bin.cu, trace_wide.cu, trace_kd.cu).
#include <map>
#include <mutex>
#include <utility>

#include "kernels.h"

namespace ilm {

uint64_t resident_blocks(const void* kernel, int block) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, uint64_t> cache;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find({dev, kernel});
        if (it != cache.end()) return it->second;
    }
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    const uint64_t r = (uint64_t)sms * (uint64_t)(per_sm > 0 ? per_sm : 1);
    std::lock_guard<std::mutex> lock(mu);
    cache[{dev, kernel}] = r;
    return r;
}

cudaError_t launch_trace(const DeviceAccel& a, const ilm_ray* rays, uint64_t n, ilm_hit* hits, uint32_t* occ,
                         uint32_t* err, const LaunchParams& lp, cudaStream_t s, const unsigned long long* n_dev) {
    if (n == 0) return cudaSuccess;
    TraceArgs t;
    t.nodes = a.nodes;
    t.n_nodes = a.n_nodes;
    t.prims = a.prims;
    t.spheres = a.spheres;
    t.rays = rays;
    t.n = n;
    t.n_dev = n_dev;
    t.hits = hits;
    t.occ = occ;
    t.err = err;
    t.max_iter = lp.max_iter;
    t.counter = lp.counter;
    for (int k = 0; k < 6; ++k) t.bound[k] = a.bound[k];
    t.kd_index = a.kd_index;
    t.split_tail = lp.split_tail ? 1u : 0u;
    if (a.width == kLayoutKdTree) return launch_trace_kd(t, lp, s);
    if (a.width == 2) return launch_trace_binary(t, s);
    return launch_trace_wide(a.width, t, lp, s);
}

}  // namespace ilm
