/*
 * illume_gpu.h — C ABI of the B200 ray-query / path-tracing library.
 *
 * This is the drop-in boundary for rs_illume's aggregate.  In the reference
 * every aggregate implements `trait Primitive` (src/core/primitive/mod.rs:9-20):
 *   world_bound()  -> Box<dyn Bounding3<Float>>
 *   intersect(&Ray) -> Option<SurfaceInteraction>
 *   intersect_p(&Ray) -> bool
 * and `BVHAccel` (src/accelerators/bvh.rs:24-93, 540-663) is the CPU
 * implementation this library replaces.  A GPU aggregate is one context plus
 * one accel id; the batch entry points below are the intended path, and a
 * single-ray `Primitive::intersect` is a batch of one.
 *
 * Conventions
 *  - Every function returns int32_t status: ILM_OK (0) or a negative ILM_ERR_*.
 *    No exception or abort crosses this boundary; ilm_last_error_string()
 *    describes the last failure on a context.
 *  - Ray/hit pointers may be device memory (stream-ordered, asynchronous) or
 *    host memory (pageable or pinned; the call stages through device buffers
 *    and returns when the results are back in host memory).
 *  - `stream` is a cudaStream_t passed as void*; NULL selects the context's
 *    own (non-blocking) stream, which is not ordered with other streams.  A
 *    caller whose buffers come from work on the legacy default stream passes
 *    cudaStreamLegacy, or cudaStreamPerThread for the per-thread one.
 *  - Primitive ids: meshes and sphere sets passed to ilm_accel_build are
 *    numbered in list order; triangles of a mesh (or spheres of a set) take
 *    consecutive ids.  This matches BVHAccel's `primitives` vector order.
 *  - One context per host thread, or external serialisation.
 */
#ifndef ILLUME_GPU_H
#define ILLUME_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------------------------------------------- status */
enum {
    ILM_OK = 0,
    ILM_ERR_INVALID_ARGUMENT = -1,   /* null/misaligned pointer, bad size/id */
    ILM_ERR_OUT_OF_MEMORY = -2,
    ILM_ERR_CUDA = -3,               /* a CUDA runtime call failed */
    ILM_ERR_TRAVERSAL_LIMIT = -4,    /* a ray overflowed the traversal stack or
                                        iteration cap; its record is flagged */
    ILM_ERR_TIMEOUT = -5,            /* host watchdog gave up waiting */
    ILM_ERR_NOT_FOUND = -6,          /* unknown mesh / accel id */
    ILM_ERR_NO_DEVICE = -7           /* no CUDA device or the kernels are missing */
};

/* ----------------------------------------------------------------- records */
/* Ray record, 32 bytes: replaces geometry/ray.rs:11-19 (o, d, t_max; the
 * time/medium/differential fields are not used on this path). */
typedef struct { float o[3]; float tmin; float d[3]; float tmax; } ilm_ray;
/* Closest-hit record, 16 bytes: primitive id (ILM_MISS on a miss), t, and
 * (u, v).  Triangles: u = b1, v = b2, so the hit point is
 * b0*p0 + b1*p1 + b2*p2 with b0 = 1-u-v (shapes/triangle.rs:232-236).
 * Spheres: the parametric (u, v) of shapes/sphere.rs:191-193. */
typedef struct { uint32_t prim; float t; float u; float v; } ilm_hit;
#define ILM_MISS 0xFFFFFFFFu

/* Sphere or another quadric.  Transforms are row-major 4x4, m[i][j] at
 * [4*i + j]; world_to_object must be the inverse.  kind selects
 *   ILM_QUADRIC_SPHERE   Sphere::new (shapes/sphere.rs:50-75): radius, z_min, z_max, phi_max_deg;
 *   ILM_QUADRIC_DISK     Disk::new (disk.rs:27-47): height, radius, inner_radius, phi_max_deg;
 *   ILM_QUADRIC_CYLINDER Cylinder::new (cylinder.rs:26-46): radius, z_min, z_max, phi_max_deg
 *                        (in degrees and ordered, as pbrt; the reference keeps the raw values);
 *   ILM_QUADRIC_CONE     Cone::new (cone.rs:26-41): height, radius, phi_max_deg;
 *   ILM_QUADRIC_PARABOLOID  Paraboloid::new (paraboloid.rs:26-47): radius, z_min, z_max
 *                        (ordered, as pbrt), phi_max_deg;
 *   ILM_QUADRIC_HYPERBOLOID Hyperboloid::new (hyperboloid.rs:31-77): the points p1, p2
 *                        swept around z, phi_max_deg (pbrt's p2.z == 0 swap).
 * Zero-initialised extra fields keep the sphere layout of earlier callers. */
enum {
    ILM_QUADRIC_SPHERE = 0, ILM_QUADRIC_DISK = 1, ILM_QUADRIC_CYLINDER = 2, ILM_QUADRIC_CONE = 3,
    ILM_QUADRIC_PARABOLOID = 4, ILM_QUADRIC_HYPERBOLOID = 5
};
typedef struct {
    float object_to_world[16];
    float world_to_object[16];
    float radius, z_min, z_max, phi_max_deg;
    int32_t reverse_orientation;
    int32_t kind;
    float height, inner_radius;
    float p1[3], p2[3];
} ilm_sphere_desc;

typedef struct {
    int32_t device;        /* CUDA device ordinal */
    int32_t stack_depth;   /* traversal stack entries per ray, <= 64 (0 = 64) */
    int32_t block_size;    /* threads per block for traversal (0 = default) */
    int32_t flags;         /* ILM_FLAG_* */
    uint32_t max_iterations; /* per-ray traversal loop cap (0 = 2^20) */
} ilm_config;
/* Validate host-resident rays (finite origin/direction, non-zero direction,
 * tmax >= 0) before any launch; an invalid ray fails the call with
 * ILM_ERR_INVALID_ARGUMENT. */
#define ILM_FLAG_VALIDATE_RAYS 1
/* Wide layouts: one thread per ray instead of the default persistent schedule
 * (warps claim rays in chunks from a per-stream device counter and refill
 * finished lanes). */
#define ILM_FLAG_GRID_SCHEDULE 2
/* Persistent schedule compiled for many resident blocks per SM instead of
 * the compiler's register choice: 7 (up to 72 registers per thread) for the
 * pooled kernel, 8 (64) for the lane-refill kernel. */
#define ILM_FLAG_HIGH_OCCUPANCY 4
/* Persistent schedule: each idle lane tests its own claimed rays against the
 * scene's root box instead of the whole warp testing each claimed chunk and
 * pooling the rays that enter.  This kernel has no split tail.  The answers
 * are the same either way, up to exact ties in t (see ILM_FLAG_NO_TAIL_SPLIT). */
#define ILM_FLAG_LANE_REFILL 8
/* Turns off the split tail, on by default: in the pooled persistent
 * schedule once every ray of the query has been claimed, and in the
 * one-thread-per-ray kernel throughout, idle lanes help their warp's
 * unfinished rays by taking subtrees from their traversal stacks.  The
 * answers are the same either way, except that of two hits at exactly the
 * same t the split keeps the smaller primitive id where the lone traversal
 * may keep the first it found.  The split tail is also off whenever
 * max_iterations is below its default of 2^20, so that which rays reach a
 * lowered cap does not depend on which lanes traversed them. */
#define ILM_FLAG_NO_TAIL_SPLIT 16

typedef struct {
    int32_t width;             /* 2 (the reference's binary layout), 4 or 8 */
    int32_t max_prims_in_node; /* BVHAccel::new max_prims_in_node (4 in all configs) */
} ilm_build_opts;

typedef struct {
    uint32_t n_prims;
    uint32_t n_binary_nodes;   /* nodes of the SAH binary tree (bvh.rs layout) */
    uint32_t n_nodes;          /* nodes of the device layout for `width` */
    uint32_t width;            /* BVH width (2, 4, 8), or ILM_LAYOUT_KDTREE */
    uint64_t device_bytes;     /* nodes + primitive records (+ kd leaf runs) in HBM */
    double build_seconds;      /* host build (+ collapse) + upload */
    uint32_t n_leaf_refs;      /* kd-tree: entries of the leaf index list */
    uint32_t max_depth;        /* kd-tree: the depth limit used */
} ilm_accel_info;
/* ilm_accel_info.width of a kd-tree accel. */
#define ILM_LAYOUT_KDTREE 1

/* KdTreeAccel::new parameters (accelerators/kdtreeaccel.rs:25-32).  A NULL
 * opts pointer selects 80, 1, 0.5, 1, -1 (pbrt-v3's kd-tree defaults; the
 * reference has no factory of its own). */
typedef struct {
    int32_t isect_cost;
    int32_t traversal_cost;
    float empty_bonus;         /* in [0, 1] */
    uint32_t max_prims;
    int32_t max_depth;         /* <= 0: round(8 + 1.3 log2(N)); at most 64 */
} ilm_kdtree_opts;

typedef uint32_t ilm_mesh_id;
typedef uint32_t ilm_accel_id;
typedef struct ilm_context ilm_context;

/* ----------------------------------------------------------------- context */
int32_t ilm_context_create(ilm_context** out, const ilm_config* cfg);
int32_t ilm_context_destroy(ilm_context* ctx);
/* Last error message on ctx (static string for ctx == NULL). Never NULL. */
const char* ilm_last_error_string(const ilm_context* ctx);
/* Rays per chunk when host ray / result buffers are copied through device
 * staging: copy-in and copy-out run on their own streams (the host link
 * carries both directions at once) and a ring of four slots traces on four
 * streams; the first and last chunks ramp from chunk/8.  4096 .. 2^24,
 * default 524288. */
int32_t ilm_context_set_stage_chunk(ilm_context* ctx, uint64_t rays);

/* One segment of a cubic Bezier curve (shapes/curve.rs:14-91): the curve's
 * object-space control points and widths at u = 0 and 1, the part
 * [u_min, u_max] this primitive covers (pbrt splits a curve into 2^splitdepth
 * segments), and for ribbons the normals at u = 0 and 1.  Flat and cylinder
 * curves intersect alike (they differ only in shading). */
enum { ILM_CURVE_FLAT = 0, ILM_CURVE_CYLINDER = 1, ILM_CURVE_RIBBON = 2 };
typedef struct {
    float object_to_world[16];
    float world_to_object[16];
    float cp[12];
    float width[2];
    float n[6];
    float u_min, u_max;
    int32_t type;
    int32_t reverse_orientation;
} ilm_curve_desc;

/* ----------------------------------------------------------------- shapes */
/* TriangleMesh::new (shapes/triangle.rs:36-73) with world-space vertices:
 * xyz holds 3*nv floats, idx holds 3*nt vertex indices.  Host memory is
 * copied; the caller keeps ownership. */
int32_t ilm_mesh_upload(ilm_context* ctx, const float* xyz, uint32_t nv,
                        const uint32_t* idx, uint32_t nt, ilm_mesh_id* out);
/* A set of spheres and other quadrics (shapes/{sphere,disk,cylinder,cone}.rs). */
int32_t ilm_spheres_upload(ilm_context* ctx, const ilm_sphere_desc* spheres, uint32_t n,
                           ilm_mesh_id* out);
/* A set of curve segments (Curve::intersect, shapes/curve.rs:278-375: the
 * segment projected into the ray's frame and refined by recursive Bezier
 * subdivision to a depth set by its flatness; hits report t, u along the
 * curve and v across it).  Widths must be positive, u_min < u_max in [0, 1]. */
int32_t ilm_curves_upload(ilm_context* ctx, const ilm_curve_desc* curves, uint32_t n, ilm_mesh_id* out);

/* ----------------------------------------------------------------- accel */
/* BVHAccel::new (accelerators/bvh.rs:32-93): SAH recursive build with 12
 * buckets (bvh.rs:95-247), flattened depth-first (bvh.rs:504-537), then laid
 * out for `width` (2 = the reference's 32-byte nodes; 4/8 = compressed wide
 * nodes collapsed from the same binary tree). */
int32_t ilm_accel_build(ilm_context* ctx, const ilm_mesh_id* meshes, uint32_t n_meshes,
                        const ilm_build_opts* opts, ilm_accel_id* out);
/* KdTreeAccel::new (accelerators/kdtreeaccel.rs:25-244): SAH over sorted
 * bound edges, one axis at a time, 8-byte nodes (kdtreeaccel.rs:470-545) laid
 * out depth first.  The accel answers every query below (closest and any
 * hit, the no-alloc form, surface interactions, path tracing) through
 * KdTreeAccel::intersect / intersect_p (kdtreeaccel.rs:256-465): front-to-
 * back traversal with a 64-entry stack of deferred far children.  Not
 * accepted by the batched queries, which run the wide BVH layouts. */
int32_t ilm_kdtree_build(ilm_context* ctx, const ilm_mesh_id* meshes, uint32_t n_meshes,
                         const ilm_kdtree_opts* opts, ilm_accel_id* out);
/* Copies of a kd-tree accel's nodes (info.n_nodes x 8 bytes: word = split
 * bits, the primitive of a one-primitive leaf or the first slot of a leaf's
 * run; flags = axis or 3 for a leaf, and above-child or count << 2) and of its
 * leaf index list (info.n_leaf_refs primitive ids). */
int32_t ilm_accel_kd_nodes(ilm_context* ctx, ilm_accel_id accel, void* out_nodes, uint32_t* out_index);
int32_t ilm_accel_destroy(ilm_context* ctx, ilm_accel_id accel);
/* Primitive::world_bound for BVHAccel (bvh.rs:555-561): {min xyz, max xyz}. */
int32_t ilm_accel_world_bound(ilm_context* ctx, ilm_accel_id accel, float out[6]);
int32_t ilm_accel_get_info(ilm_context* ctx, ilm_accel_id accel, ilm_accel_info* out);
/* Copies of the SAH binary tree (32-byte nodes as bvh.rs:665-673) and the
 * ordered primitive ids, for inspection. */
int32_t ilm_accel_binary_nodes(ilm_context* ctx, ilm_accel_id accel, void* out_nodes,
                               uint32_t* out_prim_order);

/* ------------------------------------------------- surface interactions */
/* Optional per-vertex data of a triangle mesh (TriangleMesh::new,
 * shapes/triangle.rs:36-73): shading normals n and tangents s (3 floats per
 * vertex), parametric uv (2 floats per vertex), each NULL when absent, and
 * reverse_orientation.  Set before the mesh is used by ilm_accel_build. */
typedef struct {
    const float* n;
    const float* s;
    const float* uv;
    int32_t reverse_orientation;
} ilm_mesh_attrs;
int32_t ilm_mesh_set_attrs(ilm_context* ctx, ilm_mesh_id mesh, const ilm_mesh_attrs* attrs);

/* The SurfaceInteraction that Triangle::intersect builds for a hit
 * (shapes/triangle.rs:264-415 with SurfaceInteraction::new and
 * set_shading_geometry, core/interaction.rs:262-339): the barycentrics are
 * recomputed with the same watertight arithmetic as the traversal, then
 * uv, dpdu/dpdv (uv determinant as in pbrt, D14 repaired; coordinate frame of
 * the geometric normal when degenerate), p and its error bound gamma(7),
 * the geometric normal of (p0-p2)x(p1-p2) (flipped for reverse_orientation),
 * and, when the mesh has normals or tangents, the shading frame and dndu/dndv.
 * Without them the shading frame is the geometric one (n, dpdu, dpdv, 0, 0). */
typedef struct {
    float p[3], p_error[3];
    float n[3];
    float uv[2];
    float dpdu[3], dpdv[3], dndu[3], dndv[3];
    float shading_n[3], shading_dpdu[3], shading_dpdv[3], shading_dndu[3], shading_dndv[3];
    float wo[3];
    float t;
    uint32_t prim;
    uint32_t kind;   /* ILM_SI_MISS, ILM_SI_TRIANGLE, or ILM_SI_SPHERE (p, wo, t, prim only) */
} ilm_surface_interaction;
enum { ILM_SI_MISS = 0, ILM_SI_TRIANGLE = 1, ILM_SI_SPHERE = 2 };
/* For each (ray, hit) pair from ilm_intersect_closest on the same accel, its
 * SurfaceInteraction (176 bytes).  Buffers all on the host (the call returns
 * with the results) or all on the device (stream-ordered). */
int32_t ilm_surface_interactions(ilm_context* ctx, ilm_accel_id accel, const ilm_ray* rays, const ilm_hit* hits,
                                 uint64_t n, ilm_surface_interaction* out, void* stream);

/* Host-only build of the same structure, for inspection and tests (no GPU
 * needed): one triangle mesh followed by one sphere set.  ilm_host_layout_copy
 * fills any non-NULL output: binary nodes (32 B each), ordered primitive ids,
 * the device node array (n_nodes * 32/64/80 B for width 2/4/8), the 48-byte
 * primitive records, and the world bound (6 floats). */
typedef struct ilm_host_layout ilm_host_layout;
int32_t ilm_host_layout_build(const float* xyz, uint32_t nv, const uint32_t* idx, uint32_t nt,
                              const ilm_sphere_desc* spheres, uint32_t ns, const ilm_build_opts* opts,
                              ilm_host_layout** out);
int32_t ilm_host_layout_info(const ilm_host_layout* layout, ilm_accel_info* out);
int32_t ilm_host_layout_copy(const ilm_host_layout* layout, void* bin_nodes, uint32_t* prim_order, void* nodes,
                             void* records, float* bound);
int32_t ilm_host_layout_destroy(ilm_host_layout* layout);
/* Host-only kd-tree build on up to `threads` host threads (<= 0: all); the
 * nodes do not depend on the thread count.  ilm_host_layout_copy's `nodes`
 * receives the kd nodes, `records` one record per primitive id. */
int32_t ilm_host_kdtree_build(const float* xyz, uint32_t nv, const uint32_t* idx, uint32_t nt,
                              const ilm_sphere_desc* spheres, uint32_t ns, const ilm_kdtree_opts* opts,
                              int32_t threads, ilm_host_layout** out);
/* The kd-tree's leaf index list (info.n_leaf_refs entries). */
int32_t ilm_host_layout_kd_index(const ilm_host_layout* layout, uint32_t* out);

/* ----------------------------------------------------------------- queries */
/* Primitive::intersect for BVHAccel (bvh.rs:563-612), batched: one closest
 * hit per ray.  Ties at equal t resolve to the smaller primitive id. */
int32_t ilm_intersect_closest(ilm_context* ctx, ilm_accel_id accel, const ilm_ray* rays,
                              uint64_t n, ilm_hit* hits, void* stream);
/* Primitive::intersect_p for BVHAccel (bvh.rs:614-662), batched:
 * occluded[i] = 1 when any primitive is hit with 0 < t <= rays[i].tmax. */
int32_t ilm_intersect_any(ilm_context* ctx, ilm_accel_id accel, const ilm_ray* rays,
                          uint64_t n, uint32_t* occluded, void* stream);

/* Closest hit without allocating (no counterpart in the reference).  For
 * callers that must not call cudaMalloc/cudaFree once set up: a render loop
 * with a fixed memory budget, a process whose device memory is owned by a
 * caching allocator, or a thread that must not stall the device (cudaMalloc
 * and cudaFree can synchronise it).  Same results as ilm_intersect_closest:
 * the same kernel with the same launch choices (the accel's own stack depth,
 * schedule and occupancy from ilm_accel_set_launch / ilm_autotune, else the
 * context's), and the same ILM_FLAG_VALIDATE_RAYS check of host rays.
 * Its scratch is one fixed array that the library holds on every GPU that
 * loads it, until exit: 3 MiB + 256 B (a work counter and staging for up to
 * ILM_NOALLOC_MAX_RAYS rays and hits).
 *  - n > ILM_NOALLOC_MAX_RAYS fails with ILM_ERR_INVALID_ARGUMENT.
 *  - The first call on a device resolves the array's address on that device;
 *    make that first call before any stream capture.  The address is kept
 *    for the life of the process: do not reset the device (cudaDeviceReset)
 *    while the library is loaded.
 *  - All calls share the array: calls that overlap on the GPU race.
 *    Serialise them (one stream, or wait between calls).
 *  - Rays that reach a traversal limit are marked in their records and set
 *    the context's error word (read it with ilm_device_errors), as with
 *    ilm_intersect_closest.  Host buffers: returns with the hits in host
 *    memory, and ILM_ERR_TRAVERSAL_LIMIT if this call marked a record.
 *    Device buffers: stream-ordered. */
#define ILM_NOALLOC_MAX_RAYS 65536
int32_t ilm_intersect_closest_noalloc(ilm_context* ctx, ilm_accel_id accel, const ilm_ray* rays,
                                      uint64_t n, ilm_hit* hits, void* stream);

/* ------------------------------------------------------- batched queries */
/* Many scenes with ray batches of any size, traced by one persistent launch
 * per BVH width (2, 4 or 8): BVHAccel::intersect / intersect_p of each batch's
 * accel over its rays.  All buffers are device memory. */
typedef struct {
    ilm_accel_id accel;
    const ilm_ray* rays;
    uint64_t n;
    ilm_hit* hits;         /* closest hit output (NULL for any-hit) */
    uint32_t* occluded;    /* any-hit output (NULL for closest hit) */
} ilm_batch_desc;
typedef struct ilm_batch_plan ilm_batch_plan;
/* Uploads the scene table and captures the launch sequence as a CUDA graph
 * (runs it once while doing so).  The plan keeps the buffer pointers: launch
 * it again after refilling the rays. */
int32_t ilm_batch_plan_create(ilm_context* ctx, const ilm_batch_desc* batches, uint32_t n,
                              int32_t any_hit, ilm_batch_plan** out);
/* Replays the plan on `stream`.  Launches of one plan must not overlap. */
int32_t ilm_batch_plan_launch(ilm_context* ctx, ilm_batch_plan* plan, void* stream);
int32_t ilm_batch_plan_destroy(ilm_context* ctx, ilm_batch_plan* plan);
/* One-shot form (builds, launches and waits). */
int32_t ilm_intersect_batched(ilm_context* ctx, const ilm_batch_desc* batches, uint32_t n,
                              int32_t any_hit, void* stream);

/* -------------------------------------------------------------- autotune */
/* Launch choices of one accel. */
typedef struct {
    int32_t stack_depth;     /* 32 or 64 */
    int32_t schedule;        /* 0 persistent, 1 one thread per ray */
    int32_t high_occupancy;  /* 1: 8 resident blocks per SM (64 registers) */
} ilm_launch_opts;
/* Overrides the context's launch choices for queries on `accel`. */
int32_t ilm_accel_set_launch(ilm_context* ctx, ilm_accel_id accel, const ilm_launch_opts* opts);

typedef struct {
    int32_t width;           /* best BVH width (2, 4 or 8) */
    ilm_launch_opts launch;  /* best launch choices at that width */
    double ms;               /* its median time on the sample */
    double baseline_ms;      /* width 8, context defaults, same sample */
    uint32_t n_tried;
    int32_t from_cache;      /* 1 when answered from the context's cache */
} ilm_tune_result;
/* Builds the shapes' accel at widths 2, 4 and 8, times every launch choice on
 * `sample` (device or host rays; any_hit selects the query) with CUDA events
 * (median of 3 after a warm-up) and returns the fastest.  Results are cached
 * in the context per (query kind, log2 of the primitive count, log2 of the
 * sample size); force = 1 re-measures. */
int32_t ilm_autotune(ilm_context* ctx, const ilm_mesh_id* meshes, uint32_t n_meshes, const ilm_ray* sample,
                     uint64_t n, int32_t any_hit, int32_t force, ilm_tune_result* out);

/* Film filters (the filters/ directory) and the film's weight table (core/film.rs:70-82):
 * table[y*16 + x] = evaluate((x + 0.5) * radius.x / 16, (y + 0.5) * radius.y / 16). */
enum {
    ILM_FILTER_BOX = 0,        /* filters/box_filter.rs */
    ILM_FILTER_TRIANGLE = 1,   /* filters/triangle.rs */
    ILM_FILTER_GAUSSIAN = 2,   /* filters/gaussian.rs: a = alpha */
    ILM_FILTER_MITCHELL = 3,   /* filters/mitchell.rs: a = B, b = C */
    ILM_FILTER_LANCZOS = 4     /* filters/sinc.rs: a = tau */
};
typedef struct {
    int32_t kind;
    float radius[2];
    float a, b;
} ilm_filter_desc;
#define ILM_FILTER_TABLE_WIDTH 16

/* ----------------------------------------------------------- path tracing */
/* Wavefront path tracer over a triangle accel: the PBR-book path loop with
 * the reference's one-light direct lighting with MIS
 * (core/integrator.rs:321-494), Lambertian BSDF
 * (reflection/lambertian_reflection.rs), one-sided diffuse area lights (one
 * per emissive triangle; Triangle::sample, shapes/triangle.rs:616-642),
 * cosine BSDF sampling and Russian roulette.  The reference has no
 * PathIntegrator; its render loop is core/integrator.rs:48-145. */
typedef struct {
    const uint32_t* prim_material;  /* material index per primitive (host memory) */
    const float* albedo;            /* Lambertian reflectance, 3 floats per material */
    const float* emission;          /* emitted radiance along the triangle normal
                                       normalize((p0-p2) x (p1-p2)), 3 per material */
    uint32_t n_materials;
    float eye[3];                   /* pinhole camera at eye, looking +z, up +y (in camera space) */
    float fov_deg;                  /* vertical field of view */
    uint32_t width, height;
    float camera_to_world[9];       /* row-major 3x3 taking camera-space directions to world space
                                       (a LookAt frame, possibly mirrored); all zero = identity */
} ilm_pt_scene_desc;

typedef struct {
    uint32_t spp;          /* samples per pixel: a perfect square, sqrt(spp)^2 jittered strata */
    uint32_t max_depth;    /* bounces (8 in the benchmark) */
    uint32_t rr_depth;     /* Russian roulette from this bounce on (3) */
    uint64_t seed;
    uint32_t wave_paths;   /* paths in flight per wave (0 = 2^21) */
    int32_t use_graphs;    /* replay each bounce as a CUDA graph */
    ilm_filter_desc filter; /* film filter (FilmTile::add_sample, film.rs:288-333); radius 0 or the box
                               of radius 0.5: each sample counts in its own pixel */
} ilm_pt_opts;

typedef struct {
    uint64_t closest_rays; /* camera + continuation rays */
    uint64_t shadow_rays;  /* light-sample and BSDF-sample visibility rays */
    double seconds;        /* device time of the render (CUDA events) */
    uint32_t waves;
} ilm_pt_stats;

typedef uint32_t ilm_pt_scene_id;
/* Materials and lights for `accel` (triangle meshes only). */
int32_t ilm_pt_scene_create(ilm_context* ctx, ilm_accel_id accel, const ilm_pt_scene_desc* desc,
                            ilm_pt_scene_id* out);
/* Renders width x height RGB (3 floats per pixel, row 0 at the top): the mean
 * of spp samples per pixel.  rgb_out may be host or device memory. */
int32_t ilm_render_pt(ilm_context* ctx, ilm_pt_scene_id scene, const ilm_pt_opts* opts, float* rgb_out,
                      ilm_pt_stats* stats);

/* ------------------------------------------------- neural radiance cache */
/* A small MLP that predicts the radiance leaving a surface point (no
 * counterpart in the reference; a learned stand-in for the tail of a path).
 * Inputs per sample: 12 floats = position xyz, outgoing direction xyz (unit),
 * normal xyz (unit), albedo rgb.  Encoding: 12-frequency sin/cos of the
 * position normalised to `bound`, one-blob (32 bins) of the direction's and
 * normal's (theta/pi, phi/2pi), albedo: 203 inputs.  Network: 5 hidden layers
 * of 64 with ReLU, 3 outputs, no biases, BF16 weights with FP32 accumulation
 * on tensor cores; FP32 master weights; Adam; loss = mean of
 * (p - y)^2 / (p^2 + 0.01) with p held constant in the denominator. */
typedef struct {
    float lr, beta1, beta2, eps;   /* Adam (1e-2, 0.9, 0.99, 1e-10 in the benchmark) */
    uint64_t seed;                 /* weight initialisation (He-uniform from PCG32) */
    float bound[6];                /* scene bound for the position encoding */
    float ema;                     /* inference uses a moving average of the weights over
                                      Adam steps with this decay (0.99); 0 = latest weights */
    float weight_decay;            /* decoupled weight decay (AdamW): each step also subtracts
                                      lr * weight_decay * w; 0 = none (1.0 in the benchmark,
                                      where it keeps the online-trained cache smooth: steady
                                      per-frame relMSE 0.30 against 0.345, mean image within 1%) */
} ilm_nrc_config;
typedef struct ilm_nrc ilm_nrc;
#define ILM_NRC_PARAMS 30720       /* FP32 master weights: 64x208, 4 x 64x64, 16x64 (rows 3..15 zero) */
int32_t ilm_nrc_create(ilm_context* ctx, const ilm_nrc_config* cfg, ilm_nrc** out);
int32_t ilm_nrc_destroy(ilm_context* ctx, ilm_nrc* nrc);
/* Reads (get) and/or replaces (set) the FP32 master weights, row-major
 * [out][in] per layer, layers in order. */
int32_t ilm_nrc_params(ilm_context* ctx, ilm_nrc* nrc, float* get, const float* set);
/* out[n][3] = network(inputs[n][12]); host or device buffers. */
int32_t ilm_nrc_infer(ilm_context* ctx, ilm_nrc* nrc, const float* inputs, uint64_t n, float* out, void* stream);
/* One Adam step on the batch; *loss (optional) receives the batch loss. */
int32_t ilm_nrc_train_step(ilm_context* ctx, ilm_nrc* nrc, const float* inputs, const float* targets,
                           uint64_t n, float* loss, void* stream);
/* Loss gradient with respect to the master weights (ILM_NRC_PARAMS floats),
 * without a step (for checking). */
int32_t ilm_nrc_gradients(ilm_context* ctx, ilm_nrc* nrc, const float* inputs, const float* targets,
                          uint64_t n, float* grad_out, float* loss);
/* The 208 bf16 inputs the network sees for each sample (n x 416 bytes). */
int32_t ilm_nrc_encode(ilm_context* ctx, ilm_nrc* nrc, const float* inputs, uint64_t n, void* enc_out);

/* Path tracing with the radiance cache (no counterpart in the reference; the
 * estimator around it is ilm_render_pt's).  Frames of spp_per_frame samples
 * per pixel are averaged.  A rendering path ends at its first vertex n >= 1
 * whose path spread satisfies s_n^2 > spread_c * a0 (a0 = d1^2 / (4 pi |cos1|),
 * s_n = sum_{i=2..n} sqrt(d_i^2 / (pdf_{i-1} |cos_i|))), adding throughput x
 * the cache's prediction there.  One path in max(16, P / train_paths) (P =
 * paths per frame) runs to the end and its vertices become training samples
 * (at most train_samples per frame); after each frame (if `train`) the network
 * takes train_steps Adam steps on interleaved subsets of them.  A frame runs on
 * the device as one CUDA graph; with a time budget, frames are launched until
 * the finished ones reach it (the frame queued by then is completed and
 * counted). */
typedef struct {
    uint32_t frames;          /* frames to render (0 = until time_budget_s) */
    uint32_t spp_per_frame;   /* a perfect square (0 = 1) */
    uint32_t max_depth, rr_depth;
    uint64_t seed;
    float spread_c;           /* 0 = 0.01 */
    uint32_t train_paths;     /* training paths per frame (0 = 16384) */
    uint32_t train_samples;   /* training samples per frame at most (0 = 65536) */
    double time_budget_s;     /* stop after the frame that reaches this device time (0 = no budget) */
    int32_t train;            /* 1: train after every frame; 0: inference only (no training paths) */
    uint32_t train_steps;     /* Adam steps per frame, each on every train_steps-th sample (0 = 4) */
    uint32_t train_suffix;    /* a training path goes on for this many vertices past the point where a
                                 rendering path ends, then ends in the cache too, whose prediction
                                 joins its targets (0 = 1; >= max_depth: full-length paths) */
} ilm_nrc_render_opts;

typedef struct {
    uint32_t frames;
    double seconds;           /* device time of all frames (CUDA events) */
    uint64_t closest_rays, shadow_rays;
    uint64_t queries;         /* cache queries answered */
    uint64_t train_samples;   /* training samples used */
    float last_loss;          /* network loss on the last frame's training batch */
} ilm_nrc_render_stats;

int32_t ilm_render_nrc(ilm_context* ctx, ilm_pt_scene_id scene, ilm_nrc* nrc, const ilm_nrc_render_opts* opts,
                       float* rgb_out, ilm_nrc_render_stats* stats);

/* ------------------------------------------------------- film output (host) */
/* write_image_pfm (core/imageio.rs:264-310): "PF\n<w> <h>\n-1\n", then the
 * rows bottom to top, 3 little-endian floats per pixel.  rgb holds
 * width*height*3 floats, row 0 at the top (as ilm_render_pt writes them).
 * No context or GPU is needed. */
int32_t ilm_write_pfm(const char* path, const float* rgb, uint32_t width, uint32_t height);
/* Reads a 3-channel PFM of either byte order back into top-to-bottom rows.
 * With rgb == NULL only *width and *height are filled; otherwise rgb must
 * hold (*width)*(*height)*3 floats for the size given on input. */
int32_t ilm_read_pfm(const char* path, float* rgb, uint32_t* width, uint32_t* height);

/* One filter value at film offset (x, y) from the sample. */
int32_t ilm_filter_evaluate(const ilm_filter_desc* filter, float x, float y, float* out);
int32_t ilm_filter_table(const ilm_filter_desc* filter, float* table /* 16 x 16 */);

/* ------------------------------------------------------ scene files (host) */
/* pbrt-v3 scene files, the format whose syntax tree core/parser/ast.rs
 * defines (the reference parses to that tree and constructs no scene,
 * core/parser/mod.rs:36-46; its parser module is missing).  Loading runs the
 * directives against pbrt's graphics state -- the current transform and its
 * named copies, AttributeBegin/End and TransformBegin/End stacks, materials,
 * area lights, ReverseOrientation, object instancing, Include -- and keeps:
 *  - Shape "trianglemesh" (P, indices, N, S, uv/st) with world-space vertices;
 *    a shape whose orientation is reversed (ReverseOrientation, or a
 *    transform that swaps handedness) has its triangles' last two indices
 *    swapped, so (p0-p2)x(p1-p2) is the normal pbrt's Triangle reports;
 *  - Shape "sphere", "disk", "cylinder", "cone", "paraboloid", "hyperboloid"
 *    with their pbrt parameters and defaults, under the current transform;
 *  - Shape "loopsubdiv" (levels, indices, P) as the subdivided triangle mesh
 *    with its limit normals;
 *  - Shape "curve" (P: 4 control points, width / width0 / width1, type flat /
 *    cylinder / ribbon with N at both ends, splitdepth 3) as 2^splitdepth
 *    curve segments under the current transform;
 *  - Material "matte" Kd (other types: their Kd, else 0.5, with a warning),
 *    MakeNamedMaterial / NamedMaterial, AreaLightSource "diffuse" L x scale;
 *  - Camera "perspective" fov (of the shorter image axis) under LookAt or any
 *    transform, Film xresolution / yresolution, Sampler pixelsamples (or
 *    xsamples x ysamples; rounded up to a square), Integrator maxdepth,
 *    PixelFilter box / triangle / gaussian / mitchell / sinc, Accelerator
 *    "bvh" maxnodeprims or "kdtree" with its costs.
 * Directives this library cannot represent (point / spot / distant /
 * infinite lights, textures, media, plymesh, curves, other cameras) are
 * skipped with a warning.  Syntax errors fail with a "file:line: message". */
/* Loop subdivision surface (shapes/loop_subdiv.rs, pbrt-v3's LoopSubdivide):
 * `levels` (0 .. 10) refinements of a triangle mesh by Loop's vertex and edge
 * rules, vertices then moved to the limit surface, with limit normals.  Call
 * with out_xyz == NULL to get *out_nv and *out_nt; call again with those
 * counts in *out_nv / *out_nt and buffers of 3 * nv floats (out_xyz, out_n,
 * out_n may be NULL) and 3 * nt indices.  Non-manifold input or buffers
 * smaller than the result fail with ILM_ERR_INVALID_ARGUMENT. */
int32_t ilm_loop_subdivide(const float* xyz, uint32_t nv, const uint32_t* idx, uint32_t nt, uint32_t levels,
                           uint32_t* out_nv, uint32_t* out_nt, float* out_xyz, uint32_t* out_idx, float* out_n);

typedef struct ilm_scene_file ilm_scene_file;
typedef struct {
    uint32_t n_meshes, n_triangles, n_vertices, n_quadrics;
    uint32_t n_materials;      /* distinct (albedo, emission) pairs */
    uint32_t n_emissive;       /* triangles under an area light */
    uint32_t width, height;    /* Film */
    uint32_t spp;              /* Sampler, a perfect square */
    uint32_t max_depth;        /* Integrator "path" maxdepth (pbrt default 5) */
    float eye[3];              /* camera position */
    float camera_to_world[9];  /* row-major 3x3 */
    float fov_deg;             /* vertical field of view for ilm_pt_scene_desc */
    ilm_filter_desc filter;
    int32_t accelerator;       /* 0 = "bvh", 1 = "kdtree" */
    ilm_build_opts bvh;
    ilm_kdtree_opts kdtree;
    uint32_t n_warnings;
    uint32_t n_curves;         /* curve segments */
} ilm_scene_file_info;
/* Loads `path`; on failure *out is NULL and `error` (error_len bytes, may be
 * NULL) holds the message. */
int32_t ilm_scene_file_load(const char* path, char* error, size_t error_len, ilm_scene_file** out);
/* The same from text in memory; Include paths are relative to base_dir. */
int32_t ilm_scene_file_parse(const char* text, const char* base_dir, char* error, size_t error_len,
                             ilm_scene_file** out);
int32_t ilm_scene_file_info_get(const ilm_scene_file* sf, ilm_scene_file_info* out);
/* Warnings, one per line (valid until the scene file is destroyed). */
const char* ilm_scene_file_warnings(const ilm_scene_file* sf);
/* Triangle mesh k: vertex count and triangle count (nv, nt may be NULL), and
 * copies of its arrays into any non-NULL output: xyz (3 nv), idx (3 nt),
 * n / s (3 nv; *has_n / *has_s say whether the file gave them), uv (2 nv;
 * *has_uv), material (the mesh's material index). */
int32_t ilm_scene_file_mesh(const ilm_scene_file* sf, uint32_t k, uint32_t* nv, uint32_t* nt, float* xyz,
                            uint32_t* idx, float* n, float* s, float* uv, int32_t* has_n, int32_t* has_s,
                            int32_t* has_uv, uint32_t* material);
/* The quadrics (n_quadrics descriptions) and their material indices. */
int32_t ilm_scene_file_quadrics(const ilm_scene_file* sf, ilm_sphere_desc* out, uint32_t* material);
/* The curve segments (n_curves descriptions) and their material indices. */
int32_t ilm_scene_file_curves(const ilm_scene_file* sf, ilm_curve_desc* out, uint32_t* material);
/* The material table: albedo and emission, 3 floats each per material. */
int32_t ilm_scene_file_materials(const ilm_scene_file* sf, float* albedo, float* emission);
/* Uploads the shapes to ctx (one mesh per trianglemesh, with its N / S / uv,
 * then one quadric set) and builds the accelerator the file names.
 * Primitive ids run over the meshes in file order, then the quadrics, then
 * the curve segments.  With pt_out non-NULL and triangles only, also creates
 * the path-tracing scene (camera, film size, materials); with quadrics or
 * curves present *pt_out is 0. */
int32_t ilm_scene_file_build(ilm_context* ctx, const ilm_scene_file* sf, ilm_accel_id* accel_out,
                             ilm_pt_scene_id* pt_out);
int32_t ilm_scene_file_destroy(ilm_scene_file* sf);
/* The directive tree of a scene description, read by the loader's tokenizer
 * and argument grammar but not run: what the reference's parse_to_ast
 * returns (core/parser/mod.rs:19-34; grammar of core/parser/parsers/).  JSON:
 * {"directives": [node...], "comments": [text after '#'...]}, a node being
 * {"directive", "file", "line", "num": [numeric arguments], "str": [quoted
 * arguments or ActiveTransform's word], "params": [{"type", "name", "num",
 * "str"}...]} plus "children" for AttributeBegin, TransformBegin,
 * ObjectBegin and WorldBegin blocks (the matching end closes the block and
 * is not listed).  Include is replaced by the named file's directives, its
 * path relative to the including file or, from text, to base_dir.
 * *json_len = the JSON's length; up to json_cap - 1 bytes of it and a NUL
 * are written to json (json_cap = 0 only measures).  On a syntax error
 * returns ILM_ERR_INVALID_ARGUMENT with the message in `error`. */
int32_t ilm_scene_syntax(const char* text, const char* base_dir, char* json, size_t json_cap, size_t* json_len,
                         char* error, size_t error_len);

/* Device error word accumulated by the kernels since the last reset
 * (bit 0: traversal stack overflow, bit 1: iteration cap).  Synchronises. */
int32_t ilm_device_errors(ilm_context* ctx, uint32_t* out_flags, int32_t reset);
/* Waits for `stream` (NULL = context stream) for at most timeout_s seconds;
 * ILM_ERR_TIMEOUT if it is still busy. */
int32_t ilm_synchronize(ilm_context* ctx, void* stream, double timeout_s);

#ifdef __cplusplus
}
#endif
#endif
