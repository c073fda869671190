// Library-internal state behind the opaque ilm_context handle.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "builder.h"
#include "illume_gpu.h"
#include "kernels.h"
#include "layout.h"

namespace ilm {

struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer();
    cudaError_t reserve(size_t n);   // grows (discarding contents) when too small
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

struct Mesh {
    bool is_spheres = false;
    std::vector<float> xyz;          // world-space vertices
    std::vector<uint32_t> idx;
    std::vector<SphereRec> spheres;
    uint32_t n_prims = 0;
    // optional per-vertex shading data (ilm_mesh_set_attrs)
    std::vector<float> n, s, uv;
    bool reverse = false;
    bool built = false;              // used by an accel build: attributes are fixed
};

// Per-accel data for rebuilding SurfaceInteractions (built on first use):
// vertices and attributes of all its triangle meshes, concatenated, and per
// primitive id its three global vertex indices and its mesh slot.
struct ShadingData {
    DeviceBuffer vtx, nrm, tan, uv;  // 3, 3, 3, 2 floats per vertex
    DeviceBuffer tri;                // uint4 per primitive: i0, i1, i2, mesh slot (kShadeSphere for spheres)
    DeviceBuffer mesh;               // uint32 flags per mesh slot
    bool ready = false;
};

struct Accel {
    HostLayout host;                 // SAH tree, prim order, bound (device copies below)
    DeviceBuffer d_nodes, d_prims, d_spheres, d_kd_index;
    uint64_t device_bytes = 0;
    double build_seconds = 0.0;
    // per-accel launch choices (ilm_accel_set_launch); -1 = context default
    int stack_depth = -1, schedule = -1, high_occupancy = -1;
    std::vector<ilm_mesh_id> mesh_ids;   // the shapes, in primitive-id order
    ShadingData shading;

    DeviceAccel view() const {
        DeviceAccel a;
        a.width = host.width;
        a.nodes = d_nodes.ptr;
        a.n_nodes = host.n_nodes;
        a.prims = static_cast<const PrimRec*>(d_prims.ptr);
        a.n_records = (uint32_t)host.records.size();
        a.spheres = static_cast<const SphereRec*>(d_spheres.ptr);
        a.kd_index = static_cast<const uint32_t*>(d_kd_index.ptr);
        for (int k = 0; k < 6; ++k) a.bound[k] = host.bound[k];
        return a;
    }
};

// Host-buffer queries: a copy-in and a copy-out stream and a ring of staging
// slots, each with its own trace stream (traces of consecutive chunks overlap,
// since a small trace lasts as long as its slowest ray) and the events that
// hand the slot from one stream to the next.
constexpr int kPipeStreams = 2;
constexpr int kStageSlots = 4;

struct Stage {
    DeviceBuffer rays, out;
    cudaStream_t run = nullptr;
    cudaEvent_t in = nullptr, ran = nullptr, out_done = nullptr;
};

// Chunk sizes for n rays with a steady chunk of c: the first and last chunks
// ramp (c/8, c/4, c/2) so the copy-in of the first chunk and the trace and
// copy-out of the last one are short; small batches use equal chunks.
std::vector<uint64_t> stage_plan(uint64_t n, uint64_t c);

enum class PtrKind { kHost, kDevice };

}  // namespace ilm

#include "pt.h"

struct ilm_context {
    int device = 0;
    int stack_depth = 64;
    int block_size = 128;
    int flags = 0;
    uint32_t max_iter = 1u << 20;   // kDefaultMaxIter
    cudaStream_t stream = nullptr;
    cudaStream_t pipe[ilm::kPipeStreams] = {nullptr, nullptr};
    cudaEvent_t fence = nullptr;
    ilm::Stage stage[ilm::kStageSlots];
    uint64_t stage_chunk = 1ull << 19;
    ilm::DeviceBuffer err_word;
    std::string last_error;
    std::map<ilm_mesh_id, std::unique_ptr<ilm::Mesh>> meshes;
    std::map<ilm_accel_id, std::unique_ptr<ilm::Accel>> accels;
    ilm_mesh_id next_mesh = 1;
    ilm_accel_id next_accel = 1;
    std::map<ilm_pt_scene_id, std::unique_ptr<ilm::PtScene>> pt_scenes;
    ilm_pt_scene_id next_pt = 1;
    // autotune results per (any-hit, log2 primitives, log2 sample size)
    std::map<std::tuple<int, int, int>, ilm_tune_result> tune_cache;
    // Work counters of the persistent schedule, one per stream: launches on one
    // stream run in order, so a counter is never shared by two live launches.
    std::map<cudaStream_t, std::unique_ptr<ilm::DeviceBuffer>> counters;
    unsigned long long* counter_for(cudaStream_t s) {
        auto& b = counters[s];
        if (!b) {
            b.reset(new ilm::DeviceBuffer());
            if (b->reserve(sizeof(unsigned long long)) != cudaSuccess) {
                counters.erase(s);
                return nullptr;
            }
        }
        return static_cast<unsigned long long*>(b->ptr);
    }
    void scratch_release() { counters.clear(); }
};

namespace ilm {
void set_error(ilm_context* ctx, const std::string& msg);
int32_t cuda_fail(ilm_context* ctx, cudaError_t e, const char* what);
PtrKind classify(const void* p);
Accel* find_accel(ilm_context* ctx, ilm_accel_id id);

// Default per-ray traversal loop cap (ilm_config.max_iterations = 0).
constexpr uint32_t kDefaultMaxIter = 1u << 20;

// Whether the pooled persistent schedule splits its tail (ILM_FLAG_NO_TAIL_SPLIT).
inline int split_tail_of(const ilm_context* ctx) {
    return !(ctx->flags & ILM_FLAG_NO_TAIL_SPLIT) && ctx->max_iter >= kDefaultMaxIter;
}

// Launch choices of a query on accel `a`: the accel's own (ilm_accel_set_launch,
// ilm_autotune) where it has them, else the context's.  The work counter is
// left null for the caller to supply.
inline LaunchParams accel_launch(const ilm_context* ctx, const Accel* a) {
    const int persistent = a->schedule >= 0 ? (a->schedule == 0) : !(ctx->flags & ILM_FLAG_GRID_SCHEDULE);
    const int high_occ = a->high_occupancy >= 0 ? a->high_occupancy : (ctx->flags & ILM_FLAG_HIGH_OCCUPANCY) != 0;
    LaunchParams lp{a->stack_depth > 0 ? a->stack_depth : ctx->stack_depth, ctx->block_size, ctx->max_iter,
                    persistent, nullptr, high_occ ? 8 : 0, (ctx->flags & ILM_FLAG_LANE_REFILL) ? 0 : 1};
    lp.split_tail = split_tail_of(ctx);
    return lp;
}

// ILM_FLAG_VALIDATE_RAYS on host rays: ILM_OK, or ILM_ERR_INVALID_ARGUMENT with
// the first bad ray named in the context's error string.
int32_t validate_host_rays(ilm_context* ctx, const ilm_ray* rays, uint64_t n);
// True when this library's kernels have an image for the current device.
bool kernels_loadable(cudaFuncAttributes* attr);
}  // namespace ilm
