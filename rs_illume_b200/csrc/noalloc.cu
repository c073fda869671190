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
// The kernel is the closest-hit traversal of the accel's layout, with the
// launch choices ilm_intersect_closest makes for the accel (its own stack
// depth, schedule and occupancy, else the context's).  Its scratch -- the
// persistent schedule's work counter and, for host buffers, the staging
// copies of rays and hits -- lives in g_noalloc_scratch below.  Rays that hit
// a traversal limit set the context's error word, which the context
// allocated when it was created, so ilm_device_errors reports them for both
// entry points.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "context.h"
#include "illume_gpu.h"
#include "kernels.h"

namespace ilm {
namespace {

constexpr uint64_t kMaxRays = ILM_NOALLOC_MAX_RAYS;
constexpr size_t kHeader = 256;   // work counter (8 B), padded
constexpr size_t kScratchBytes = kHeader + kMaxRays * (sizeof(ilm_ray) + sizeof(ilm_hit));

// The scratch: 3 MiB + 256 B on every GPU that loads the library, until exit.
// In host code this name is only a handle for cudaGetSymbolAddress, never a
// device address.  The address is resolved once per device and cached for
// the life of the process, so the device must not be reset (cudaDeviceReset)
// while the library is loaded.
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
    ilm_ray* d_rays = reinterpret_cast<ilm_ray*>(scratch + kHeader);
    ilm_hit* d_hits = reinterpret_cast<ilm_hit*>(scratch + kHeader + kMaxRays * sizeof(ilm_ray));
    uint32_t* err = static_cast<uint32_t*>(ctx->err_word.ptr);

    PtrKind kr = classify(rays), kh = classify(hits);
    if (kr != kh) {
        set_error(ctx, "ilm_intersect_closest_noalloc: rays and hits must both be device or both host memory");
        return ILM_ERR_INVALID_ARGUMENT;
    }
    if (kr == PtrKind::kHost) {
        if (int32_t rc = validate_host_rays(ctx, rays, n)) return rc;
    }
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    LaunchParams lp = accel_launch(ctx, a);
    lp.counter = counter;
    DeviceAccel da = a->view();
    // The array keeps the previous call's contents: the work counter must
    // start at zero (the persistent launch zeroes it too; this keeps the
    // array's state independent of the schedule).
    e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s);
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
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamSynchronize");
    // This call's own limit hits are the records it marked (the error word
    // also holds earlier calls' flags until ilm_device_errors resets it).
    for (uint64_t i = 0; i < n; ++i)
        if (hits[i].prim == kHitTraversalError) {
            set_error(ctx, "ilm_intersect_closest_noalloc: traversal limit reached; affected records are marked");
            return ILM_ERR_TRAVERSAL_LIMIT;
        }
    return ILM_OK;
}
