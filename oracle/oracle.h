/*
 * CPU oracle for the ray-query / path-tracing hot path of rs_illume.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a scalar C++ restatement of the
 * reference's Rust code (rs_illume, a pbrt-v3 port).  It exists so that the
 * GPU product can be checked against it and so that the CPU baseline can be
 * timed.  The product library (rs_illume_b200) never links or calls it; only
 * tests/, __graft_entry__.smoke() and bench.py's CPU legs do.
 *
 * Parity status: the reference crate ships no test, golden vector or fixture
 * for this path and cannot be compiled (no Rust toolchain; the crate itself
 * has compile errors), so parity with the reference is UNPINNED by the
 * reference's own tests.  The restatement is pinned instead to analytic
 * known-answer cases (tests/test_oracle_kat.py) and follows the cited lines.
 * Where the reference is wrong or does not compile, the repair is applied and
 * numbered (D1..D24); the product applies the same repairs.
 */
#ifndef ILLUME_ORACLE_H
#define ILLUME_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 32-byte ray record: origin, t_min (unused, 0), direction, t_max. */
typedef struct { float o[3]; float tmin; float d[3]; float tmax; } orc_ray;
/* 16-byte hit record: primitive id (0xFFFFFFFF = miss), t, u (=b1), v (=b2). */
typedef struct { uint32_t prim; float t; float u; float v; } orc_hit;

/* Quadric shape: object_to_world / world_to_object are row-major 4x4
 * (m[i][j] at [4*i+j]).  kind 0: Sphere (shapes/sphere.rs:15-75; radius,
 * z_min, z_max, phi_max); 1: Disk (disk.rs:27-47; height, radius,
 * inner_radius, phi_max); 2: Cylinder (cylinder.rs:26-46; radius, z_min,
 * z_max, phi_max); 3: Cone (cone.rs:26-41; height, radius, phi_max);
 * 4: Paraboloid (paraboloid.rs:26-47; radius, z_min, z_max, phi_max);
 * 5: Hyperboloid (hyperboloid.rs:31-77; p1, p2, phi_max). */
typedef struct {
    float object_to_world[16];
    float world_to_object[16];
    float radius, z_min, z_max, phi_max_deg;
    int32_t reverse_orientation;
    int32_t kind;
    float height, inner_radius;
    float p1[3], p2[3];
} orc_sphere_desc;

/* One segment of a cubic Bezier curve (shapes/curve.rs:14-91): control
 * points, widths at u = 0 and 1, normals at u = 0 and 1 (ribbons), the
 * segment's u range, type 0 flat, 1 cylinder, 2 ribbon. */
typedef struct {
    float object_to_world[16];
    float world_to_object[16];
    float cp[12];
    float width[2];
    float n[6];
    float u_min, u_max;
    int32_t type;
    int32_t reverse_orientation;
} orc_curve_desc;

/* 32-byte flattened BVH node (accelerators/bvh.rs:665-673, 32 B per D6). */
typedef struct {
    float bmin[3], bmax[3];
    int32_t offset;      /* leaf: first primitive; interior: second child */
    uint16_t n_prims;    /* 0 = interior */
    uint8_t axis;
    uint8_t pad;
} orc_bvh_node;

/* Constants of core/pbrt.rs (gamma(n), SHADOW_EPSILON). */
float orc_gamma(int n);
float orc_next_float_up(float v);
float orc_next_float_down(float v);

/* PCG32 (core/rng.rs:15-63). Writes n draws of Rng::new(seq). */
void orc_rng_u32(uint64_t seq, uint64_t n, uint32_t* out);
void orc_rng_floats(uint64_t seq, uint64_t n, float* out);
/* Rng::new(seq) advanced by delta draws (D18 repaired), then n draws. */
void orc_rng_floats_advanced(uint64_t seq, int64_t delta, uint64_t n, float* out);

/* Scene = triangles (world-space vertices + 3 indices each) followed by
 * spheres.  Primitive ids: triangles 0..nt-1, spheres nt..nt+ns-1.
 * Builds the SAH BVHAccel (bvh.rs:32-93) with max_prims_in_node. */
void* orc_scene_create(const float* verts, uint32_t nv, const uint32_t* idx,
                       uint32_t nt, const orc_sphere_desc* spheres, uint32_t ns,
                       int max_prims_in_node);
/* The same with curve segments after the quadrics (their primitive ids
 * follow the quadrics'). */
void* orc_scene_create_curves(const float* verts, uint32_t nv, const uint32_t* idx, uint32_t nt,
                              const orc_sphere_desc* spheres, uint32_t ns, const orc_curve_desc* curves,
                              uint32_t nc, int max_prims_in_node);
void orc_scene_destroy(void* scene);
uint32_t orc_scene_node_count(void* scene);
void orc_scene_nodes(void* scene, orc_bvh_node* out);
void orc_scene_prim_order(void* scene, uint32_t* out);
void orc_scene_world_bound(void* scene, float out[6]);
double orc_scene_build_seconds(void* scene);

/* BVHAccel::intersect over a ray batch (bvh.rs:563-612 with D4/D5).
 * node_visits / prim_tests may be NULL; otherwise per-ray counters.
 * Returns number of rays whose 64-entry stack overflowed (0 expected). */
int64_t orc_intersect(void* scene, const orc_ray* rays, uint64_t n, orc_hit* hits,
                      uint32_t* node_visits, uint32_t* prim_tests, int nthreads);
/* BVHAccel::intersect_p (bvh.rs:614-662 with D4). */
int64_t orc_intersect_p(void* scene, const orc_ray* rays, uint64_t n, uint8_t* occluded,
                        uint32_t* node_visits, uint32_t* prim_tests, int nthreads);

/* Single-shape tests for known-answer checks.  out = {t, b0, b1, b2}. */
int orc_triangle_intersect(const float* p0, const float* p1, const float* p2,
                           const orc_ray* r, int closest, float* out);
/* The SurfaceInteraction of a hit on triangle p (9 floats), with optional
 * per-vertex normals / tangents (9 floats) and uvs (6 floats); 1 on a hit.
 * Same layout as ilm_surface_interaction (kind 1 = triangle). */
typedef struct {
    float p[3], p_error[3];
    float n[3];
    float uv[2];
    float dpdu[3], dpdv[3], dndu[3], dndv[3];
    float shading_n[3], shading_dpdu[3], shading_dpdv[3], shading_dndu[3], shading_dndv[3];
    float wo[3];
    float t;
    uint32_t prim;
    uint32_t kind;
} orc_si;
int orc_surface_interaction(const float* p, const float* n, const float* s, const float* uv, int reverse,
                            const orc_ray* r, orc_si* out);
/* Full-frame render through a filtered film: each sample's L is splatted
 * with the 16 x 16 filter table (table[y*16 + x], radius rx, ry) as
 * FilmTile::add_sample does (film.rs:288-333, D20 repaired).  camera_to_world
 * (row-major 3x3, may be NULL) turns the camera-space direction into world
 * space. */
int orc_render_pt_filtered(void* scene, const float* verts, const uint32_t* idx, uint32_t nt,
                           const uint32_t* prim_material, const float* albedo, const float* emission,
                           const float eye[3], float fov_deg, uint32_t width, uint32_t height, uint32_t spp,
                           uint32_t max_depth, uint32_t rr_depth, uint64_t seed, const float* table, float rx,
                           float ry, int nthreads, float* rgb_out, uint64_t* ray_counts,
                           const float* camera_to_world);
/* out = {t, u, v}. */
int orc_sphere_intersect(const orc_sphere_desc* s, const orc_ray* r, int closest, float* out);
void orc_sphere_world_bound(const orc_sphere_desc* s, float out[6]);
/* Curve::intersect (curve.rs:278-375): out = {t, u, v}; 1 on a hit. */
int orc_curve_intersect(const orc_curve_desc* c, const orc_ray* r, float* out);

/* Single-ray forms (used by the path-tracer restatement). Return 1 on stack overflow. */
int orc_trace_closest1(void* scene, const orc_ray* ray, orc_hit* hit);
int orc_trace_any1(void* scene, const orc_ray* ray, uint8_t* occluded);
// The same, also returning the ray's node visits and primitive tests.
int orc_trace_closest1_counted(void* scene, const orc_ray* ray, orc_hit* hit, uint32_t* nv, uint32_t* nt);
int orc_trace_any1_counted(void* scene, const orc_ray* ray, uint8_t* occluded, uint32_t* nv, uint32_t* nt);

/* Path tracer (oracle/pt.cpp): renders pixels [x0,x1) x [y0,y1) of a
 * width x height pinhole image (eye, looking +z, up +y, vertical fov) with
 * spp stratified samples (spp must be a square), Lambertian triangles
 * (albedo[3*material]) and one-sided diffuse emitters (emission[3*material]),
 * max_depth bounces, Russian roulette from bounce rr_depth.  `scene` must have
 * been created from the same triangles.  rgb_out: 3 floats per pixel, row-major
 * over the window; ray_counts (6 entries): closest-hit rays, shadow rays, and
 * their binary-BVH node visits and primitive tests (closest: [2], [3];
 * shadow: [4], [5]). */
int orc_render_pt(void* scene, const float* verts, const uint32_t* idx, uint32_t nt,
                  const uint32_t* prim_material, const float* albedo, const float* emission,
                  const float eye[3], float fov_deg, uint32_t width, uint32_t height, uint32_t spp,
                  uint32_t max_depth, uint32_t rr_depth, uint64_t seed, uint32_t x0, uint32_t y0,
                  uint32_t x1, uint32_t y1, int nthreads, float* rgb_out, uint64_t* ray_counts);

/* KdTreeAccel (accelerators/kdtreeaccel.rs:11-596) over the scene's
 * primitives (the scene must outlive it).  max_depth <= 0: the reference's
 * default.  Nodes are the 8-byte KdAccelNode: word = split bits, the one
 * primitive or the run's first slot; flags = axis or 3 (leaf), and above
 * child or count << 2. */
typedef struct { uint32_t word, flags; } orc_kd_node;
void* orc_kdtree_create(void* scene, int isect_cost, int traversal_cost, float empty_bonus, uint32_t max_prims,
                        int max_depth);
void orc_kdtree_destroy(void* kd);
uint32_t orc_kdtree_node_count(void* kd);
uint32_t orc_kdtree_index_count(void* kd);
int orc_kdtree_max_depth(void* kd);
void orc_kdtree_nodes(void* kd, orc_kd_node* out);
void orc_kdtree_indices(void* kd, uint32_t* out);
/* KdTreeAccel::intersect / intersect_p over a ray batch; returns the number
 * of rays whose 64-entry stack overflowed.  node_visits / prim_tests may be
 * NULL; otherwise per-ray counters. */
int64_t orc_kdtree_intersect(void* kd, const orc_ray* rays, uint64_t n, orc_hit* hits, uint32_t* node_visits,
                             uint32_t* prim_tests, int nthreads);
int64_t orc_kdtree_intersect_p(void* kd, const orc_ray* rays, uint64_t n, uint8_t* occluded, uint32_t* node_visits,
                               uint32_t* prim_tests, int nthreads);

/* Wall-clock seconds spent by the last orc_intersect/_p call (traversal only). */
double orc_last_trace_seconds(void);

#ifdef __cplusplus
}
#endif
#endif
