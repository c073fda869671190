// C ABI of the ray-query library (include/illume_gpu.h).
#include "illume_gpu.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "builder.h"
#include "context.h"
#include "kernels.h"

using namespace ilm;

namespace ilm {

void set_error(ilm_context* ctx, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
}

int32_t cuda_fail(ilm_context* ctx, cudaError_t e, const char* what) {
    char buf[256];
    std::snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    set_error(ctx, buf);
    return e == cudaErrorMemoryAllocation ? ILM_ERR_OUT_OF_MEMORY : ILM_ERR_CUDA;
}

DeviceBuffer::~DeviceBuffer() {
    if (ptr) cudaFree(ptr);
}

cudaError_t DeviceBuffer::reserve(size_t n) {
    if (n <= bytes) return cudaSuccess;
    if (ptr) { cudaFree(ptr); ptr = nullptr; bytes = 0; }
    cudaError_t e = cudaMalloc(&ptr, n);
    if (e == cudaSuccess) bytes = n;
    return e;
}

std::vector<uint64_t> stage_plan(uint64_t n, uint64_t c) {
    std::vector<uint64_t> plan;
    const uint64_t ramp = c / 8 + c / 4 + c / 2;
    if (n < 2 * ramp + c) {
        // equal chunks, at least four when the batch allows
        uint64_t k = std::max<uint64_t>(1, std::min<uint64_t>(4, (n + 4095) / 4096));
        k = std::max(k, (n + c - 1) / c);
        for (uint64_t off = 0, i = 0; i < k; ++i) {
            uint64_t cnt = (n - off) / (k - i);
            plan.push_back(cnt);
            off += cnt;
        }
        return plan;
    }
    for (uint64_t d : {c / 8, c / 4, c / 2}) plan.push_back(d);
    uint64_t middle = n - 2 * ramp, k = (middle + c - 1) / c;
    for (uint64_t off = 0, i = 0; i < k; ++i) {
        uint64_t cnt = (middle - off) / (k - i);
        plan.push_back(cnt);
        off += cnt;
    }
    for (uint64_t d : {c / 2, c / 4, c / 8}) plan.push_back(d);
    return plan;
}

PtrKind classify(const void* p) {
    cudaPointerAttributes attr;
    cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess) { cudaGetLastError(); return PtrKind::kHost; }
    if (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) return PtrKind::kDevice;
    return PtrKind::kHost;
}

Accel* find_accel(ilm_context* ctx, ilm_accel_id id) {
    auto it = ctx->accels.find(id);
    return it == ctx->accels.end() ? nullptr : it->second.get();
}

int32_t validate_host_rays(ilm_context* ctx, const ilm_ray* rays, uint64_t n) {
    if (!(ctx->flags & ILM_FLAG_VALIDATE_RAYS)) return ILM_OK;
    for (uint64_t i = 0; i < n; ++i) {
        const ilm_ray& r = rays[i];
        bool ok = std::isfinite(r.o[0]) && std::isfinite(r.o[1]) && std::isfinite(r.o[2]) &&
                  std::isfinite(r.d[0]) && std::isfinite(r.d[1]) && std::isfinite(r.d[2]) &&
                  !(r.d[0] == 0.0f && r.d[1] == 0.0f && r.d[2] == 0.0f) && !(r.tmax < 0.0f) &&
                  !std::isnan(r.tmax);
        if (!ok) {
            char buf[128];
            std::snprintf(buf, sizeof buf, "ray %llu is invalid (non-finite, zero direction or tmax < 0)",
                          (unsigned long long)i);
            set_error(ctx, buf);
            return ILM_ERR_INVALID_ARGUMENT;
        }
    }
    return ILM_OK;
}

}  // namespace ilm

#define ILM_CHECK_CTX(ctx)                                   \
    do {                                                     \
        if (!(ctx)) return ILM_ERR_INVALID_ARGUMENT;         \
        cudaError_t _e = cudaSetDevice((ctx)->device);       \
        if (_e != cudaSuccess) return cuda_fail((ctx), _e, "cudaSetDevice"); \
    } while (0)

#define ILM_CUDA(ctx, call, what)                            \
    do {                                                     \
        cudaError_t _e = (call);                             \
        if (_e != cudaSuccess) return cuda_fail((ctx), _e, what); \
    } while (0)

extern "C" {

const char* ilm_last_error_string(const ilm_context* ctx) {
    if (!ctx) return "no context";
    return ctx->last_error.c_str();
}

int32_t ilm_context_create(ilm_context** out, const ilm_config* cfg) {
    if (!out) return ILM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return ILM_ERR_NO_DEVICE;
    }
    int dev = cfg ? cfg->device : 0;
    if (dev < 0 || dev >= ndev) return ILM_ERR_INVALID_ARGUMENT;
    if (cfg && (cfg->stack_depth < 0 || cfg->stack_depth > 64 || cfg->block_size < 0 || cfg->block_size > 1024))
        return ILM_ERR_INVALID_ARGUMENT;
    std::unique_ptr<ilm_context> ctx(new ilm_context());
    ctx->device = dev;
    ctx->stack_depth = (cfg && cfg->stack_depth) ? cfg->stack_depth : 64;
    ctx->block_size = (cfg && cfg->block_size) ? cfg->block_size : 128;
    ctx->flags = cfg ? cfg->flags : 0;
    if (cfg && cfg->max_iterations) ctx->max_iter = cfg->max_iterations;
    if (cudaSetDevice(dev) != cudaSuccess) return ILM_ERR_NO_DEVICE;
    // Fail early when the library's kernels cannot run on the device.
    cudaFuncAttributes fa;
    if (!kernels_loadable(&fa)) {
        cudaGetLastError();
        return ILM_ERR_NO_DEVICE;
    }
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return ILM_ERR_CUDA;
    for (auto& s : ctx->pipe)
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return ILM_ERR_CUDA;
    if (cudaEventCreateWithFlags(&ctx->fence, cudaEventDisableTiming) != cudaSuccess) return ILM_ERR_CUDA;
    for (auto& st : ctx->stage) {
        if (cudaStreamCreateWithFlags(&st.run, cudaStreamNonBlocking) != cudaSuccess) return ILM_ERR_CUDA;
        for (cudaEvent_t* e : {&st.in, &st.ran, &st.out_done})
            if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess) return ILM_ERR_CUDA;
    }
    if (ctx->err_word.reserve(sizeof(uint32_t)) != cudaSuccess) return ILM_ERR_OUT_OF_MEMORY;
    if (cudaMemset(ctx->err_word.ptr, 0, sizeof(uint32_t)) != cudaSuccess) return ILM_ERR_CUDA;
    *out = ctx.release();
    return ILM_OK;
}

int32_t ilm_context_set_stage_chunk(ilm_context* ctx, uint64_t rays) {
    ILM_CHECK_CTX(ctx);
    if (rays < 4096 || rays > (1ull << 24)) {
        set_error(ctx, "ilm_context_set_stage_chunk: chunk must be 4096 .. 2^24 rays");
        return ILM_ERR_INVALID_ARGUMENT;
    }
    cudaError_t e = cudaDeviceSynchronize();   // no staging buffer may be in use
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaDeviceSynchronize");
    ctx->stage_chunk = rays;
    return ILM_OK;
}

int32_t ilm_context_destroy(ilm_context* ctx) {
    if (!ctx) return ILM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    ctx->pt_scenes.clear();
    ctx->accels.clear();
    for (auto& st : ctx->stage) {
        st.rays.release();
        st.out.release();
        for (cudaEvent_t e : {st.in, st.ran, st.out_done}) if (e) cudaEventDestroy(e);
        if (st.run) cudaStreamDestroy(st.run);
    }
    ctx->err_word.release();
    ctx->scratch_release();
    if (ctx->fence) cudaEventDestroy(ctx->fence);
    for (auto& s : ctx->pipe) if (s) cudaStreamDestroy(s);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return ILM_OK;
}

int32_t ilm_mesh_upload(ilm_context* ctx, const float* xyz, uint32_t nv, const uint32_t* idx, uint32_t nt,
                        ilm_mesh_id* out) {
    if (!ctx || !out) return ILM_ERR_INVALID_ARGUMENT;
    if ((nv > 0 && !xyz) || (nt > 0 && !idx)) {
        set_error(ctx, "ilm_mesh_upload: null vertex or index pointer");
        return ILM_ERR_INVALID_ARGUMENT;
    }
    for (uint64_t i = 0; i < 3ull * nv; ++i)
        if (!std::isfinite(xyz[i])) {
            set_error(ctx, "ilm_mesh_upload: non-finite vertex coordinate");
            return ILM_ERR_INVALID_ARGUMENT;
        }
    for (uint64_t i = 0; i < 3ull * nt; ++i)
        if (idx[i] >= nv) {
            set_error(ctx, "ilm_mesh_upload: vertex index out of range");
            return ILM_ERR_INVALID_ARGUMENT;
        }
    auto m = std::make_unique<Mesh>();
    m->is_spheres = false;
    m->xyz.assign(xyz, xyz + 3ull * nv);
    m->idx.assign(idx, idx + 3ull * nt);
    m->n_prims = nt;
    ilm_mesh_id id = ctx->next_mesh++;
    ctx->meshes[id] = std::move(m);
    *out = id;
    return ILM_OK;
}

int32_t ilm_mesh_set_attrs(ilm_context* ctx, ilm_mesh_id mesh, const ilm_mesh_attrs* attrs) {
    if (!ctx || !attrs) return ILM_ERR_INVALID_ARGUMENT;
    auto it = ctx->meshes.find(mesh);
    if (it == ctx->meshes.end()) {
        set_error(ctx, "ilm_mesh_set_attrs: unknown mesh id");
        return ILM_ERR_NOT_FOUND;
    }
    Mesh& m = *it->second;
    if (m.is_spheres || m.built) {
        set_error(ctx, "ilm_mesh_set_attrs: not a triangle mesh, or already used by an accel build");
        return ILM_ERR_INVALID_ARGUMENT;
    }
    const size_t nv = m.xyz.size() / 3;
    auto take = [&](const float* src, size_t per, std::vector<float>& dst) -> bool {
        dst.clear();
        if (!src) return true;
        dst.assign(src, src + per * nv);
        for (float v : dst)
            if (!std::isfinite(v)) return false;
        return true;
    };
    if (!take(attrs->n, 3, m.n) || !take(attrs->s, 3, m.s) || !take(attrs->uv, 2, m.uv)) {
        set_error(ctx, "ilm_mesh_set_attrs: non-finite attribute value");
        m.n.clear(); m.s.clear(); m.uv.clear();
        return ILM_ERR_INVALID_ARGUMENT;
    }
    m.reverse = attrs->reverse_orientation != 0;
    return ILM_OK;
}

// The record of one quadric description; null on success, else why it is
// rejected.
static const char* quadric_record(const ilm_sphere_desc& d, SphereRec* out) {
    const bool hyper = d.kind == ILM_QUADRIC_HYPERBOLOID;
    if (!hyper && (!(d.radius > 0.0f) || !std::isfinite(d.radius))) return "radius must be positive and finite";
    for (int k = 0; k < 3; ++k)
        if (!std::isfinite(d.p1[k]) || !std::isfinite(d.p2[k])) return "invalid quadric parameters";
    if (d.kind < ILM_QUADRIC_SPHERE || d.kind > ILM_QUADRIC_HYPERBOLOID ||
        (d.kind == ILM_QUADRIC_CONE && !(d.height > 0.0f)) ||
        (d.kind == ILM_QUADRIC_DISK && !(d.inner_radius >= 0.0f && d.inner_radius < d.radius)) ||
        (d.kind == ILM_QUADRIC_CYLINDER && !(d.z_min != d.z_max)) ||
        (d.kind == ILM_QUADRIC_PARABOLOID && !(d.z_min != d.z_max && std::fmax(d.z_min, d.z_max) > 0.0f)) ||
        !std::isfinite(d.height) || !std::isfinite(d.z_min) || !std::isfinite(d.z_max))
        return "invalid quadric parameters";
    SphereInput in;
    std::memcpy(in.o2w, d.object_to_world, sizeof in.o2w);
    std::memcpy(in.w2o, d.world_to_object, sizeof in.w2o);
    in.radius = d.radius; in.z_min = d.z_min; in.z_max = d.z_max; in.phi_max_deg = d.phi_max_deg;
    in.reverse = d.reverse_orientation;
    in.kind = d.kind; in.height = d.height; in.inner_radius = d.inner_radius;
    for (int k = 0; k < 3; ++k) { in.p1[k] = d.p1[k]; in.p2[k] = d.p2[k]; }
    if (!make_sphere(in, out)) return "hyperboloid points give no finite implicit form";
    return nullptr;
}

int32_t ilm_spheres_upload(ilm_context* ctx, const ilm_sphere_desc* spheres, uint32_t n, ilm_mesh_id* out) {
    if (!ctx || !out || (n > 0 && !spheres)) return ILM_ERR_INVALID_ARGUMENT;
    auto m = std::make_unique<Mesh>();
    m->is_spheres = true;
    for (uint32_t i = 0; i < n; ++i) {
        SphereRec rec;
        if (const char* why = quadric_record(spheres[i], &rec)) {
            set_error(ctx, std::string("ilm_spheres_upload: ") + why);
            return ILM_ERR_INVALID_ARGUMENT;
        }
        m->spheres.push_back(rec);
    }
    m->n_prims = n;
    ilm_mesh_id id = ctx->next_mesh++;
    ctx->meshes[id] = std::move(m);
    *out = id;
    return ILM_OK;
}

// The shape views of `meshes`, which become fixed (their attributes can no
// longer change).
static int32_t mesh_views(ilm_context* ctx, const char* who, const ilm_mesh_id* meshes, uint32_t n_meshes,
                          std::vector<MeshView>& views) {
    for (uint32_t k = 0; k < n_meshes; ++k) {
        auto it = ctx->meshes.find(meshes[k]);
        if (it == ctx->meshes.end()) {
            set_error(ctx, std::string(who) + ": unknown mesh id");
            return ILM_ERR_NOT_FOUND;
        }
        const Mesh& m = *it->second;
        views.push_back({m.is_spheres, m.xyz.data(), m.idx.data(), m.spheres.data(), m.n_prims});
    }
    for (uint32_t k = 0; k < n_meshes; ++k) ctx->meshes[meshes[k]]->built = true;
    return ILM_OK;
}

// Copies a host layout to the device and registers the accel.
static int32_t upload_accel(ilm_context* ctx, std::unique_ptr<Accel> acc, std::chrono::steady_clock::time_point t0,
                            ilm_accel_id* out) {
    const HostLayout& h = acc->host;
    auto put = [&](DeviceBuffer& d, const void* src, size_t bytes, const char* what) -> int32_t {
        if (!bytes) return ILM_OK;
        ILM_CUDA(ctx, d.reserve(bytes), what);
        ILM_CUDA(ctx, cudaMemcpy(d.ptr, src, bytes, cudaMemcpyHostToDevice), what);
        return ILM_OK;
    };
    const size_t rb = h.records.size() * sizeof(PrimRec), sb = h.spheres.size() * sizeof(SphereRec),
                 kb = h.kd_index.size() * sizeof(uint32_t);
    int32_t rc;
    if ((rc = put(acc->d_nodes, h.node_bytes.data(), h.node_bytes.size(), "upload(nodes)")) != ILM_OK) return rc;
    if ((rc = put(acc->d_prims, h.records.data(), rb, "upload(prims)")) != ILM_OK) return rc;
    if ((rc = put(acc->d_spheres, h.spheres.data(), sb, "upload(spheres)")) != ILM_OK) return rc;
    if ((rc = put(acc->d_kd_index, h.kd_index.data(), kb, "upload(kd index)")) != ILM_OK) return rc;
    acc->device_bytes = h.node_bytes.size() + rb + sb + kb;
    acc->build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    ilm_accel_id id = ctx->next_accel++;
    ctx->accels[id] = std::move(acc);
    *out = id;
    return ILM_OK;
}

int32_t ilm_curves_upload(ilm_context* ctx, const ilm_curve_desc* curves, uint32_t n, ilm_mesh_id* out) {
    if (!ctx || !out || (n > 0 && !curves)) return ILM_ERR_INVALID_ARGUMENT;
    auto m = std::make_unique<Mesh>();
    m->is_spheres = true;
    for (uint32_t i = 0; i < n; ++i) {
        const ilm_curve_desc& d = curves[i];
        bool ok = d.type >= ILM_CURVE_FLAT && d.type <= ILM_CURVE_RIBBON && d.width[0] > 0.0f && d.width[1] > 0.0f &&
                  std::isfinite(d.width[0]) && std::isfinite(d.width[1]) && d.u_min >= 0.0f && d.u_min < d.u_max &&
                  d.u_max <= 1.0f;
        for (float v : d.cp) ok = ok && std::isfinite(v);
        if (d.type == ILM_CURVE_RIBBON)
            for (int e = 0; e < 2; ++e) {
                const float* nv = d.n + 3 * e;
                ok = ok && std::isfinite(nv[0]) && std::isfinite(nv[1]) && std::isfinite(nv[2]) &&
                     (nv[0] != 0.0f || nv[1] != 0.0f || nv[2] != 0.0f);
            }
        if (!ok) {
            set_error(ctx, "ilm_curves_upload: invalid curve (type, widths, u range, control points or normals)");
            return ILM_ERR_INVALID_ARGUMENT;
        }
        CurveInput in;
        std::memcpy(in.o2w, d.object_to_world, sizeof in.o2w);
        std::memcpy(in.w2o, d.world_to_object, sizeof in.w2o);
        std::memcpy(in.cp, d.cp, sizeof in.cp);
        std::memcpy(in.width, d.width, sizeof in.width);
        std::memcpy(in.n, d.n, sizeof in.n);
        in.u_min = d.u_min;
        in.u_max = d.u_max;
        in.type = d.type;
        in.reverse = d.reverse_orientation;
        m->spheres.push_back(make_curve(in));
    }
    m->n_prims = n;
    ilm_mesh_id id = ctx->next_mesh++;
    ctx->meshes[id] = std::move(m);
    *out = id;
    return ILM_OK;
}

int32_t ilm_accel_build(ilm_context* ctx, const ilm_mesh_id* meshes, uint32_t n_meshes, const ilm_build_opts* opts,
                        ilm_accel_id* out) {
    ILM_CHECK_CTX(ctx);
    if (!out || (n_meshes > 0 && !meshes)) return ILM_ERR_INVALID_ARGUMENT;
    int width = opts ? opts->width : 8;
    int max_prims = opts ? opts->max_prims_in_node : 4;
    auto t0 = std::chrono::steady_clock::now();
    std::vector<MeshView> views;
    if (int32_t rc = mesh_views(ctx, "ilm_accel_build", meshes, n_meshes, views)) return rc;
    auto acc = std::make_unique<Accel>();
    acc->mesh_ids.assign(meshes, meshes + n_meshes);
    std::string msg = build_layout(views, width, max_prims, (int)std::thread::hardware_concurrency(), acc->host);
    if (!msg.empty()) {
        set_error(ctx, "ilm_accel_build: " + msg);
        return ILM_ERR_INVALID_ARGUMENT;
    }
    return upload_accel(ctx, std::move(acc), t0, out);
}

static KdParams kd_params(const ilm_kdtree_opts* o) {
    KdParams p;
    if (o) {
        p.isect_cost = o->isect_cost;
        p.traversal_cost = o->traversal_cost;
        p.empty_bonus = o->empty_bonus;
        p.max_prims = o->max_prims;
        p.max_depth = o->max_depth;
    }
    return p;
}

int32_t ilm_kdtree_build(ilm_context* ctx, const ilm_mesh_id* meshes, uint32_t n_meshes, const ilm_kdtree_opts* opts,
                         ilm_accel_id* out) {
    ILM_CHECK_CTX(ctx);
    if (!out || (n_meshes > 0 && !meshes)) return ILM_ERR_INVALID_ARGUMENT;
    auto t0 = std::chrono::steady_clock::now();
    std::vector<MeshView> views;
    if (int32_t rc = mesh_views(ctx, "ilm_kdtree_build", meshes, n_meshes, views)) return rc;
    auto acc = std::make_unique<Accel>();
    acc->mesh_ids.assign(meshes, meshes + n_meshes);
    std::string msg =
        build_kd_layout(views, kd_params(opts), (int)std::thread::hardware_concurrency(), acc->host);
    if (!msg.empty()) {
        set_error(ctx, "ilm_kdtree_build: " + msg);
        return ILM_ERR_INVALID_ARGUMENT;
    }
    return upload_accel(ctx, std::move(acc), t0, out);
}

int32_t ilm_accel_destroy(ilm_context* ctx, ilm_accel_id accel) {
    ILM_CHECK_CTX(ctx);
    auto it = ctx->accels.find(accel);
    if (it == ctx->accels.end()) return ILM_ERR_NOT_FOUND;
    cudaDeviceSynchronize();
    ctx->accels.erase(it);
    return ILM_OK;
}

int32_t ilm_accel_world_bound(ilm_context* ctx, ilm_accel_id accel, float out[6]) {
    if (!ctx || !out) return ILM_ERR_INVALID_ARGUMENT;
    Accel* a = find_accel(ctx, accel);
    if (!a) return ILM_ERR_NOT_FOUND;
    std::memcpy(out, a->host.bound, sizeof a->host.bound);
    return ILM_OK;
}

int32_t ilm_accel_get_info(ilm_context* ctx, ilm_accel_id accel, ilm_accel_info* out) {
    if (!ctx || !out) return ILM_ERR_INVALID_ARGUMENT;
    Accel* a = find_accel(ctx, accel);
    if (!a) return ILM_ERR_NOT_FOUND;
    out->n_prims = a->host.n_prims;
    out->n_binary_nodes = (uint32_t)a->host.bin_nodes.size();
    out->n_nodes = a->host.n_nodes;
    out->width = (uint32_t)a->host.width;
    out->device_bytes = a->device_bytes;
    out->build_seconds = a->build_seconds;
    out->n_leaf_refs = (uint32_t)a->host.kd_index.size();
    out->max_depth = (uint32_t)a->host.kd_max_depth;
    return ILM_OK;
}

int32_t ilm_accel_kd_nodes(ilm_context* ctx, ilm_accel_id accel, void* out_nodes, uint32_t* out_index) {
    if (!ctx) return ILM_ERR_INVALID_ARGUMENT;
    Accel* a = find_accel(ctx, accel);
    if (!a) return ILM_ERR_NOT_FOUND;
    if (a->host.width != kLayoutKdTree) {
        set_error(ctx, "ilm_accel_kd_nodes: not a kd-tree accel");
        return ILM_ERR_INVALID_ARGUMENT;
    }
    if (out_nodes && !a->host.node_bytes.empty())
        std::memcpy(out_nodes, a->host.node_bytes.data(), a->host.node_bytes.size());
    if (out_index && !a->host.kd_index.empty())
        std::memcpy(out_index, a->host.kd_index.data(), a->host.kd_index.size() * 4);
    return ILM_OK;
}

int32_t ilm_accel_binary_nodes(ilm_context* ctx, ilm_accel_id accel, void* out_nodes, uint32_t* out_prim_order) {
    if (!ctx) return ILM_ERR_INVALID_ARGUMENT;
    Accel* a = find_accel(ctx, accel);
    if (!a) return ILM_ERR_NOT_FOUND;
    if (out_nodes && !a->host.bin_nodes.empty())
        std::memcpy(out_nodes, a->host.bin_nodes.data(), a->host.bin_nodes.size() * sizeof(BinNode));
    if (out_prim_order && !a->host.prim_order.empty())
        std::memcpy(out_prim_order, a->host.prim_order.data(), a->host.prim_order.size() * 4);
    return ILM_OK;
}

static int32_t intersect_impl(ilm_context* ctx, ilm_accel_id accel, const ilm_ray* rays, uint64_t n, ilm_hit* hits,
                              uint32_t* occ, void* stream) {
    ILM_CHECK_CTX(ctx);
    void* out = occ ? (void*)occ : (void*)hits;
    if (n == 0) return ILM_OK;
    if (!rays || !out) {
        set_error(ctx, "null ray or result pointer");
        return ILM_ERR_INVALID_ARGUMENT;
    }
    if (((uintptr_t)rays & 15u) || (!occ && ((uintptr_t)hits & 15u)) || (occ && ((uintptr_t)occ & 3u))) {
        set_error(ctx, "ray/hit buffers must be 16-byte aligned (occlusion flags 4-byte aligned)");
        return ILM_ERR_INVALID_ARGUMENT;
    }
    Accel* a = find_accel(ctx, accel);
    if (!a) {
        set_error(ctx, "unknown accel id");
        return ILM_ERR_NOT_FOUND;
    }
    DeviceAccel da = a->view();
    LaunchParams lp = accel_launch(ctx, a);
    int persistent = lp.persistent;
    // By default a batch that one wave of the one-thread-per-ray kernel holds
    // runs that kernel: every ray is resident at once, so the persistent
    // schedule's claiming buys nothing (measured: 440 against 361 Mrays/s for
    // 65,536 camera rays).
    if (a->schedule < 0 && persistent && da.width != 2 && da.width != kLayoutKdTree &&
        n <= wide_grid_wave(da.width, lp.stack_depth))
        persistent = lp.persistent = 0;
    uint32_t* err = static_cast<uint32_t*>(ctx->err_word.ptr);
    cudaStream_t user = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    PtrKind kr = classify(rays), ko = classify(out);
    if (kr != ko) {
        set_error(ctx, "rays and results must both be device memory or both host memory");
        return ILM_ERR_INVALID_ARGUMENT;
    }
    auto counter = [&](cudaStream_t s) -> unsigned long long* {
        return persistent ? ctx->counter_for(s) : nullptr;
    };
    if (kr == PtrKind::kDevice) {
        lp.counter = counter(user);
        if (persistent && !lp.counter) return ILM_ERR_OUT_OF_MEMORY;
        ILM_CUDA(ctx, launch_trace(da, rays, n, hits, occ, err, lp, user), "trace launch");
        return ILM_OK;
    }
    if (int32_t rc = validate_host_rays(ctx, rays, n)) return rc;
    // Host buffers: chunks staged through a ring of device slots.  Copy-in and
    // copy-out have a stream each, so the host link carries rays in and
    // results out at once; each slot traces on its own stream, so traces of
    // consecutive chunks overlap.  A slot is refilled once its trace (rays)
    // and copy-out (results) are done.
    // Staged chunks of the wide layouts run one thread per ray unless the
    // accel names a schedule: a persistent launch holds every SM until its
    // slowest ray ends, so the next chunk's trace queues behind it, while
    // one-thread-per-ray blocks retire as their rays end and the next chunk's
    // blocks take their place (measured: 1,314 against 1,277 Mrays/s for 2M
    // incoherent rays in 512K-ray chunks).
    if (a->schedule < 0 && da.width != 2 && da.width != kLayoutKdTree) persistent = lp.persistent = 0;
    const size_t out_rec = occ ? sizeof(uint32_t) : sizeof(ilm_hit);
    const std::vector<uint64_t> plan = stage_plan(n, ctx->stage_chunk);
    const uint64_t biggest = *std::max_element(plan.begin(), plan.end());
    for (auto& st : ctx->stage) {
        ILM_CUDA(ctx, st.rays.reserve(biggest * sizeof(ilm_ray)), "cudaMalloc(stage rays)");
        ILM_CUDA(ctx, st.out.reserve(biggest * sizeof(ilm_hit)), "cudaMalloc(stage out)");
    }
    cudaStream_t in_s = ctx->pipe[0], out_s = ctx->pipe[1];
    ILM_CUDA(ctx, cudaEventRecord(ctx->fence, user), "cudaEventRecord");
    for (auto& s : ctx->pipe) ILM_CUDA(ctx, cudaStreamWaitEvent(s, ctx->fence, 0), "cudaStreamWaitEvent");
    for (auto& st : ctx->stage) ILM_CUDA(ctx, cudaStreamWaitEvent(st.run, ctx->fence, 0), "cudaStreamWaitEvent");
    uint64_t off = 0;
    for (size_t c = 0; c < plan.size(); ++c) {
        const uint64_t cnt = plan[c];
        Stage& st = ctx->stage[c % kStageSlots];
        const bool reused = c >= (size_t)kStageSlots;
        if (reused) ILM_CUDA(ctx, cudaStreamWaitEvent(in_s, st.ran, 0), "cudaStreamWaitEvent");
        ILM_CUDA(ctx, cudaMemcpyAsync(st.rays.ptr, rays + off, cnt * sizeof(ilm_ray), cudaMemcpyHostToDevice, in_s),
                 "cudaMemcpyAsync(rays)");
        ILM_CUDA(ctx, cudaEventRecord(st.in, in_s), "cudaEventRecord");
        ILM_CUDA(ctx, cudaStreamWaitEvent(st.run, st.in, 0), "cudaStreamWaitEvent");
        if (reused) ILM_CUDA(ctx, cudaStreamWaitEvent(st.run, st.out_done, 0), "cudaStreamWaitEvent");
        lp.counter = counter(st.run);
        if (persistent && !lp.counter) return ILM_ERR_OUT_OF_MEMORY;
        ILM_CUDA(ctx,
                 launch_trace(da, static_cast<const ilm_ray*>(st.rays.ptr), cnt,
                              occ ? nullptr : static_cast<ilm_hit*>(st.out.ptr),
                              occ ? static_cast<uint32_t*>(st.out.ptr) : nullptr, err, lp, st.run),
                 "trace launch");
        ILM_CUDA(ctx, cudaEventRecord(st.ran, st.run), "cudaEventRecord");
        ILM_CUDA(ctx, cudaStreamWaitEvent(out_s, st.ran, 0), "cudaStreamWaitEvent");
        void* dst = occ ? (void*)(occ + off) : (void*)(hits + off);
        ILM_CUDA(ctx, cudaMemcpyAsync(dst, st.out.ptr, cnt * out_rec, cudaMemcpyDeviceToHost, out_s),
                 "cudaMemcpyAsync(results)");
        ILM_CUDA(ctx, cudaEventRecord(st.out_done, out_s), "cudaEventRecord");
        off += cnt;
    }
    for (auto& s : ctx->pipe) ILM_CUDA(ctx, cudaStreamSynchronize(s), "cudaStreamSynchronize");
    for (auto& st : ctx->stage) ILM_CUDA(ctx, cudaStreamSynchronize(st.run), "cudaStreamSynchronize");
    return ILM_OK;
}

int32_t ilm_intersect_closest(ilm_context* ctx, ilm_accel_id accel, const ilm_ray* rays, uint64_t n, ilm_hit* hits,
                              void* stream) {
    if (!ctx) return ILM_ERR_INVALID_ARGUMENT;
    if (n > 0 && !hits) { set_error(ctx, "null hit pointer"); return ILM_ERR_INVALID_ARGUMENT; }
    return intersect_impl(ctx, accel, rays, n, hits, nullptr, stream);
}

int32_t ilm_intersect_any(ilm_context* ctx, ilm_accel_id accel, const ilm_ray* rays, uint64_t n, uint32_t* occluded,
                          void* stream) {
    if (!ctx) return ILM_ERR_INVALID_ARGUMENT;
    if (n > 0 && !occluded) { set_error(ctx, "null occlusion pointer"); return ILM_ERR_INVALID_ARGUMENT; }
    return intersect_impl(ctx, accel, rays, n, nullptr, occluded, stream);
}

struct ilm_host_layout {
    ilm::HostLayout h;
    double seconds = 0.0;
};

// Shape views of one triangle mesh followed by one quadric set, for the
// host-only builds.
static int32_t host_views(const float* xyz, uint32_t nv, const uint32_t* idx, uint32_t nt,
                          const ilm_sphere_desc* spheres, uint32_t ns, std::vector<SphereRec>& sph,
                          std::vector<MeshView>& views) {
    if ((nv > 0 && !xyz) || (nt > 0 && !idx) || (ns > 0 && !spheres)) return ILM_ERR_INVALID_ARGUMENT;
    for (uint64_t i = 0; i < 3ull * nt; ++i)
        if (idx[i] >= nv) return ILM_ERR_INVALID_ARGUMENT;
    for (uint64_t i = 0; i < 3ull * nv; ++i)
        if (!std::isfinite(xyz[i])) return ILM_ERR_INVALID_ARGUMENT;
    sph.resize(ns);
    for (uint32_t i = 0; i < ns; ++i)
        if (quadric_record(spheres[i], &sph[i])) return ILM_ERR_INVALID_ARGUMENT;
    if (nt > 0) views.push_back({false, xyz, idx, nullptr, nt});
    if (ns > 0) views.push_back({true, nullptr, nullptr, sph.data(), ns});
    return ILM_OK;
}

int32_t ilm_host_layout_build(const float* xyz, uint32_t nv, const uint32_t* idx, uint32_t nt,
                              const ilm_sphere_desc* spheres, uint32_t ns, const ilm_build_opts* opts,
                              ilm_host_layout** out) {
    if (!out) return ILM_ERR_INVALID_ARGUMENT;
    std::vector<SphereRec> sph;
    std::vector<MeshView> views;
    if (int32_t rc = host_views(xyz, nv, idx, nt, spheres, ns, sph, views)) return rc;
    auto t0 = std::chrono::steady_clock::now();
    std::unique_ptr<ilm_host_layout> hl(new ilm_host_layout());
    std::string msg = build_layout(views, opts ? opts->width : 8, opts ? opts->max_prims_in_node : 4,
                                   (int)std::thread::hardware_concurrency(), hl->h);
    if (!msg.empty()) return ILM_ERR_INVALID_ARGUMENT;
    hl->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = hl.release();
    return ILM_OK;
}

int32_t ilm_host_kdtree_build(const float* xyz, uint32_t nv, const uint32_t* idx, uint32_t nt,
                              const ilm_sphere_desc* spheres, uint32_t ns, const ilm_kdtree_opts* opts,
                              int32_t threads, ilm_host_layout** out) {
    if (!out) return ILM_ERR_INVALID_ARGUMENT;
    std::vector<SphereRec> sph;
    std::vector<MeshView> views;
    if (int32_t rc = host_views(xyz, nv, idx, nt, spheres, ns, sph, views)) return rc;
    auto t0 = std::chrono::steady_clock::now();
    std::unique_ptr<ilm_host_layout> hl(new ilm_host_layout());
    int nth = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
    std::string msg = build_kd_layout(views, kd_params(opts), nth, hl->h);
    if (!msg.empty()) return ILM_ERR_INVALID_ARGUMENT;
    hl->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = hl.release();
    return ILM_OK;
}

int32_t ilm_host_layout_kd_index(const ilm_host_layout* hl, uint32_t* out) {
    if (!hl || !out) return ILM_ERR_INVALID_ARGUMENT;
    if (!hl->h.kd_index.empty()) std::memcpy(out, hl->h.kd_index.data(), hl->h.kd_index.size() * 4);
    return ILM_OK;
}

int32_t ilm_host_layout_info(const ilm_host_layout* hl, ilm_accel_info* out) {
    if (!hl || !out) return ILM_ERR_INVALID_ARGUMENT;
    const HostLayout& h = hl->h;
    out->n_prims = h.n_prims;
    out->n_binary_nodes = (uint32_t)h.bin_nodes.size();
    out->n_nodes = h.n_nodes;
    out->width = (uint32_t)h.width;
    out->device_bytes = h.node_bytes.size() + h.records.size() * sizeof(PrimRec) +
                        h.spheres.size() * sizeof(SphereRec) + h.kd_index.size() * sizeof(uint32_t);
    out->build_seconds = hl->seconds;
    out->n_leaf_refs = (uint32_t)h.kd_index.size();
    out->max_depth = (uint32_t)h.kd_max_depth;
    return ILM_OK;
}

int32_t ilm_host_layout_copy(const ilm_host_layout* hl, void* bin_nodes, uint32_t* prim_order, void* nodes,
                             void* records, float* bound) {
    if (!hl) return ILM_ERR_INVALID_ARGUMENT;
    const HostLayout& h = hl->h;
    if (bin_nodes && !h.bin_nodes.empty()) std::memcpy(bin_nodes, h.bin_nodes.data(), h.bin_nodes.size() * sizeof(BinNode));
    if (prim_order && !h.prim_order.empty()) std::memcpy(prim_order, h.prim_order.data(), h.prim_order.size() * 4);
    if (nodes && !h.node_bytes.empty()) std::memcpy(nodes, h.node_bytes.data(), h.node_bytes.size());
    if (records && !h.records.empty()) std::memcpy(records, h.records.data(), h.records.size() * sizeof(PrimRec));
    if (bound) std::memcpy(bound, h.bound, sizeof h.bound);
    return ILM_OK;
}

int32_t ilm_host_layout_destroy(ilm_host_layout* hl) {
    if (!hl) return ILM_ERR_INVALID_ARGUMENT;
    delete hl;
    return ILM_OK;
}

int32_t ilm_device_errors(ilm_context* ctx, uint32_t* out_flags, int32_t reset) {
    ILM_CHECK_CTX(ctx);
    if (!out_flags) return ILM_ERR_INVALID_ARGUMENT;
    ILM_CUDA(ctx, cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    ILM_CUDA(ctx, cudaMemcpy(out_flags, ctx->err_word.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost), "cudaMemcpy(err)");
    if (reset) ILM_CUDA(ctx, cudaMemset(ctx->err_word.ptr, 0, sizeof(uint32_t)), "cudaMemset(err)");
    return ILM_OK;
}

int32_t ilm_synchronize(ilm_context* ctx, void* stream, double timeout_s) {
    ILM_CHECK_CTX(ctx);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaStreamQuery(s);
        if (e == cudaSuccess) return ILM_OK;
        if (e != cudaErrorNotReady) return cuda_fail(ctx, e, "cudaStreamQuery");
        double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > timeout_s) {
            set_error(ctx, "ilm_synchronize: timed out");
            return ILM_ERR_TIMEOUT;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

}  // extern "C"
