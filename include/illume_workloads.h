/*
 * illume_workloads.h — seeded synthetic scenes and ray batches.
 *
 * Not a reference interface: the reference has no benchmark inputs, so the
 * benchmark and test inputs are generated procedurally.  All draws come from
 * PCG32 with the reference's constants and output function
 * (src/core/rng.rs:9-63, Rng::new(seq) = set_sequence(seq)).  Geometry is
 * computed in double precision and rounded to float once, so the outputs are
 * bit-reproducible on any IEEE host.
 */
#ifndef ILLUME_WORKLOADS_H
#define ILLUME_WORKLOADS_H

#include <stdint.h>
#include "illume_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* n draws of Rng::new(seq).uniform_float() / uniform_uint32(). */
void ilm_wl_rng_floats(uint64_t seq, uint64_t n, float* out);
void ilm_wl_rng_u32(uint64_t seq, uint64_t n, uint32_t* out);

/* Random triangle soup: triangle i has centre c ~ U[0,1]^3 and vertices
 * c + U[-spread, spread]^3 (draw order cx,cy,cz, then x,y,z of each vertex).
 * xyz: 9*n floats; idx: 3*n (0,1,2,3,...). */
void ilm_wl_soup(uint64_t seed, uint32_t n, float spread, float* xyz, uint32_t* idx);

/* Icosphere by midpoint subdivision of an icosahedron, `level` times,
 * vertices pushed to the unit sphere; then displaced radially:
 *   r = 1 + amplitude * sum_{k=1..4} sin(4k x + phi_k) cos(4k y) sin(4k z)
 * with phi_k = 2*pi*u_k, u_k the first 4 draws of Rng::new(seed); finally
 * p = centre + radius * r * (x, y, z).
 * nv = 10*4^level + 2, nt = 20*4^level. */
void ilm_wl_icosphere_counts(uint32_t level, uint32_t* nv, uint32_t* nt);
void ilm_wl_icosphere(uint32_t level, uint64_t seed, float amplitude, float radius,
                      const float centre[3], float* xyz, uint32_t* idx);

/* Pinhole primary rays, one per pixel centre, row 0 at the top: eye, looking
 * +z, up +y, vertical field of view fov_deg; ray index = y*width + x. */
void ilm_wl_camera_rays(uint32_t width, uint32_t height, const float eye[3], float fov_deg,
                        ilm_ray* out);

/* Incoherent rays: origins uniform in a ball (radius * cbrt(u)), directions
 * uniform on S^2 (z = 1-2u, phi = 2*pi*v).  Rays [0, n_closest) have
 * tmax = +inf; the rest are shadow rays with tmax ~ U[tmax_lo, tmax_hi].
 * Draws from Rng::new(seed) after discarding `skip` draws. */
void ilm_wl_ball_rays(uint64_t seed, uint64_t skip, uint64_t n, uint64_t n_closest,
                      float radius, float tmax_lo, float tmax_hi, ilm_ray* out);

/* Procedural Cornell box in [0,1]^3 (y up, open towards -z):
 *   floor y=0, ceiling y=1, back wall z=1 (white 0.73), left wall x=0 (red
 *   0.63/0.065/0.05), right wall x=1 (green 0.14/0.45/0.09), 2 triangles each;
 *   ceiling light quad x,z in [0.375,0.625] at y=0.999, emitting 15 downwards
 *   (both triangles' normals (p0-p2)x(p1-p2) point -y), 2 triangles;
 *   tall box 0.3x0.6x0.3 centred (0.33, 0.3, 0.65) rotated +18 deg about y and
 *   short box 0.3x0.3x0.3 centred (0.66, 0.15, 0.33) rotated -18 deg, white,
 *   12 triangles each; displaced icosphere (see ilm_wl_icosphere) of
 *   `ico_level`, radius 0.2, amplitude 0.05, phases from Rng::new(seed),
 *   centred (0.66, 0.52, 0.33), white.
 * Materials: 0 white, 1 red, 2 green, 3 light (albedo 0, emission 15).
 * Camera for this scene: eye (0.5, 0.5, -1.37), looking +z, fov 40 deg.
 * mat: one material index per triangle; albedo / emission: 4 x RGB. */
#define ILM_CORNELL_N_MATERIALS 4
void ilm_wl_cornell_counts(uint32_t ico_level, uint32_t* nv, uint32_t* nt);
void ilm_wl_cornell(uint32_t ico_level, uint64_t seed, float* xyz, uint32_t* idx, uint32_t* mat,
                    float* albedo, float* emission);

#ifdef __cplusplus
}
#endif
#endif
