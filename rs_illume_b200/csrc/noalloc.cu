// ilm_intersect_closest_noalloc: closest-hit queries that allocate nothing.
//
// Who needs this: callers that must not call cudaMalloc/cudaFree once set up.
// For example, a renderer's per-frame loop that keeps a fixed memory budget,
// a host that lets a caching allocator (such as PyTorch's) own the device
// memory, or a thread that must not stall the device: cudaMalloc and cudaFree
// can synchronise the device.  ilm_intersect_closest may allocate on its first
// use of a stream (the persistent schedule's work counter) and whenever host
// buffers need staging space; this entry point instead uses one fixed
// scratch array that the library holds on every GPU that loads it.
//
// The kernel is the persistent closest-hit traversal of trace_wide.cu (or the
// binary traversal for width-2 accels).  Its scratch -- the work counter, the
// error word and, for host buffers, the staging copies of rays and hits -- lives
// in g_noalloc_scratch below.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "context.h"
#include "illume_gpu.h"
#include "kernels.h"

namespace ilm {
namespace {

constexpr uint64_t kMaxRays = ILM_NOALLOC_MAX_RAYS;
constexpr size_t kHeader = 256;   // work counter (8 B) + error word (4 B), padded
constexpr size_t kScratchBytes = kHeader + kMaxRays * (sizeof(ilm_ray) + sizeof(ilm_hit));

// The scratch: 3 MiB + 256 B on every GPU that loads the library, until exit.
// In host code this name is only a handle for cudaGetSymbolAddress, never a
// device address.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_setup_mutex;

// Device address of the scratch on `device`, resolved once per device with
// that device current.
cudaError_t scratch_address(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_addr[device]);
    return cudaSuccess;
}

}  // namespace
}  // namespace ilm

using namespace ilm;

extern "C" int32_t ilm_intersect_closest_noalloc(ilm_context* ctx, ilm_accel_id accel, const ilm_ray* rays,
                                                 uint64_t n, ilm_hit* hits, void* stream) {
    if (!ctx) return ILM_ERR_INVALID_ARGUMENT;
    if (n == 0) return ILM_OK;
    if (n > kMaxRays) {
        char buf[160];
        std::snprintf(buf, sizeof buf,
                      "ilm_intersect_closest_noalloc: %llu rays exceed the fixed scratch limit of %llu rays per call",
                      (unsigned long long)n, (unsigned long long)kMaxRays);
        set_error(ctx, buf);
        return ILM_ERR_INVALID_ARGUMENT;
    }
    if (!rays || !hits || ((uintptr_t)rays & 15u) || ((uintptr_t)hits & 15u)) {
        set_error(ctx, "ilm_intersect_closest_noalloc: null or non-16-byte-aligned ray/hit buffer");
        return ILM_ERR_INVALID_ARGUMENT;
    }
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
    Accel* a = find_accel(ctx, accel);
    if (!a) {
        set_error(ctx, "ilm_intersect_closest_noalloc: unknown accel id");
        return ILM_ERR_NOT_FOUND;
    }
    unsigned char* scratch = nullptr;
    e = scratch_address(ctx->device, &scratch);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGetSymbolAddress(noalloc scratch)");
    unsigned long long* counter = reinterpret_cast<unsigned long long*>(scratch);
    uint32_t* err = reinterpret_cast<uint32_t*>(scratch + 8);
    ilm_ray* d_rays = reinterpret_cast<ilm_ray*>(scratch + kHeader);
    ilm_hit* d_hits = reinterpret_cast<ilm_hit*>(scratch + kHeader + kMaxRays * sizeof(ilm_ray));

    PtrKind kr = classify(rays), kh = classify(hits);
    if (kr != kh) {
        set_error(ctx, "ilm_intersect_closest_noalloc: rays and hits must both be device or both host memory");
        return ILM_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    const int persistent = (ctx->flags & ILM_FLAG_GRID_SCHEDULE) ? 0 : 1;
    LaunchParams lp{ctx->stack_depth, ctx->block_size, ctx->max_iter, persistent, counter,
                    (ctx->flags & ILM_FLAG_HIGH_OCCUPANCY) ? 8 : 0};
    DeviceAccel da = a->view();
    // The array keeps the previous call's contents: the counter and the error
    // word must start at zero.
    e = cudaMemsetAsync(scratch, 0, 16, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemsetAsync(noalloc scratch)");
    if (kr == PtrKind::kDevice) {
        e = launch_trace(da, rays, n, hits, nullptr, err, lp, s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "trace launch");
        return ILM_OK;
    }
    e = cudaMemcpyAsync(d_rays, rays, n * sizeof(ilm_ray), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync(rays)");
    e = launch_trace(da, d_rays, n, d_hits, nullptr, err, lp, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "trace launch");
    e = cudaMemcpyAsync(hits, d_hits, n * sizeof(ilm_hit), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync(hits)");
    uint32_t flags = 0;
    e = cudaMemcpyAsync(&flags, err, sizeof flags, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync(error word)");
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamSynchronize");
    if (flags) {
        set_error(ctx, "ilm_intersect_closest_noalloc: traversal limit reached; affected records are marked");
        return ILM_ERR_TRAVERSAL_LIMIT;
    }
    return ILM_OK;
}
