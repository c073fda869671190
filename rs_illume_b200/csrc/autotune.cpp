// Autotuner: picks the BVH width, stack depth, schedule and occupancy variant
// for a scene and a sample of its rays by timing every combination on the
// device (CUDA events on the context's stream, median of 3 after a warm-up).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "context.h"
#include "illume_gpu.h"

using namespace ilm;

namespace {

using Key = std::tuple<int, int, int>;   // any-hit, log2 primitives, log2 sample size

int ilog2(uint64_t v) {
    int r = 0;
    while (v > 1) { v >>= 1; ++r; }
    return r;
}

}  // namespace

extern "C" {

int32_t ilm_accel_set_launch(ilm_context* ctx, ilm_accel_id accel, const ilm_launch_opts* opts) {
    if (!ctx || !opts) return ILM_ERR_INVALID_ARGUMENT;
    Accel* a = find_accel(ctx, accel);
    if (!a) return ILM_ERR_NOT_FOUND;
    if ((opts->stack_depth != 32 && opts->stack_depth != 64) || opts->schedule < 0 || opts->schedule > 1 ||
        opts->high_occupancy < 0 || opts->high_occupancy > 1)
        return ILM_ERR_INVALID_ARGUMENT;
    a->stack_depth = opts->stack_depth;
    a->schedule = opts->schedule;
    a->high_occupancy = opts->high_occupancy;
    return ILM_OK;
}

int32_t ilm_autotune(ilm_context* ctx, const ilm_mesh_id* meshes, uint32_t n_meshes, const ilm_ray* sample,
                     uint64_t n, int32_t any_hit, int32_t force, ilm_tune_result* out) {
    if (!ctx || !out || !sample || n == 0 || !meshes || n_meshes == 0) return ILM_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ILM_ERR_CUDA;
    uint64_t prims = 0;
    for (uint32_t k = 0; k < n_meshes; ++k) {
        auto it = ctx->meshes.find(meshes[k]);
        if (it == ctx->meshes.end()) return ILM_ERR_NOT_FOUND;
        prims += it->second->n_prims;
    }
    Key key{any_hit != 0, ilog2(prims), ilog2(n)};
    if (!force) {
        auto& m = ctx->tune_cache;
        auto it = m.find(key);
        if (it != m.end()) {
            *out = it->second;
            out->from_cache = 1;
            return ILM_OK;
        }
    }
    // device copies of the sample and a result buffer
    DeviceBuffer d_rays, d_out;
    const ilm_ray* rays = sample;
    cudaError_t e;
    if (classify(sample) == PtrKind::kHost) {
        if ((e = d_rays.reserve(n * sizeof(ilm_ray))) != cudaSuccess) return cuda_fail(ctx, e, "autotune");
        if ((e = cudaMemcpy(d_rays.ptr, sample, n * sizeof(ilm_ray), cudaMemcpyHostToDevice)) != cudaSuccess)
            return cuda_fail(ctx, e, "autotune");
        rays = static_cast<const ilm_ray*>(d_rays.ptr);
    }
    if ((e = d_out.reserve(n * sizeof(ilm_hit))) != cudaSuccess) return cuda_fail(ctx, e, "autotune");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto run = [&](ilm_accel_id acc) -> int32_t {
        return any_hit ? ilm_intersect_any(ctx, acc, rays, n, static_cast<uint32_t*>(d_out.ptr), ctx->stream)
                       : ilm_intersect_closest(ctx, acc, rays, n, static_cast<ilm_hit*>(d_out.ptr), ctx->stream);
    };
    auto time_it = [&](ilm_accel_id acc, double* ms_out) -> int32_t {
        int32_t st = run(acc);   // warm-up
        if (st != ILM_OK) return st;
        std::vector<double> t;
        for (int k = 0; k < 3; ++k) {
            cudaEventRecord(e0, ctx->stream);
            if ((st = run(acc)) != ILM_OK) return st;
            cudaEventRecord(e1, ctx->stream);
            cudaEventSynchronize(e1);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            t.push_back(ms);
        }
        std::sort(t.begin(), t.end());
        *ms_out = t[1];
        return ILM_OK;
    };
    ilm_tune_result best{};
    best.ms = 1e30;
    best.baseline_ms = 0.0;
    uint32_t tried = 0;
    int32_t status = ILM_OK;
    for (int width : {2, 4, 8}) {
        ilm_build_opts bo{width, 4};
        ilm_accel_id acc = 0;
        if ((status = ilm_accel_build(ctx, meshes, n_meshes, &bo, &acc)) != ILM_OK) break;
        std::vector<ilm_launch_opts> choices;
        if (width == 2) choices.push_back({64, 1, 0});
        else
            for (int sd : {32, 64}) {
                choices.push_back({sd, 0, 0});
                choices.push_back({sd, 0, 1});
                choices.push_back({sd, 1, 0});
            }
        for (const ilm_launch_opts& c : choices) {
            if (width != 2) ilm_accel_set_launch(ctx, acc, &c);
            double ms = 0.0;
            if ((status = time_it(acc, &ms)) != ILM_OK) break;
            ++tried;
            if (width == 8 && c.stack_depth == 64 && c.schedule == 0 && c.high_occupancy == 0) best.baseline_ms = ms;
            if (ms < best.ms) {
                best.ms = ms;
                best.width = width;
                best.launch = c;
            }
        }
        ilm_accel_destroy(ctx, acc);
        if (status != ILM_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (status != ILM_OK) return status;
    best.n_tried = tried;
    best.from_cache = 0;
    ctx->tune_cache[key] = best;
    *out = best;
    return ILM_OK;
}

}  // extern "C"
