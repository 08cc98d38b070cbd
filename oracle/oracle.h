/*
 * oracle.h — CPU oracle for the spectral path-tracing path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code; only the tests, the smoke check and the benchmark's CPU
 * baseline leg do, to check the CUDA path against it.
 *
 * The oracle restates the reference's WGSL hot path in C++ FP32 (same
 * operation order, same RNG consumption order), with closest-hit / any-hit
 * queries answered by an FP64 ray-triangle test in place of the Vulkan
 * driver's ray queries.  Each function cites the reference line it follows.
 *
 * Parity status: the reference has no tests, golden vectors or fixtures, and
 * its code path (wgpu -> Vulkan ray query) cannot run on this machine.  Its
 * shader source can: oracle/wgsl_translate.py translates shader.wgsl,
 * photon_emit.wgsl and build_grid.wgsl mechanically into C++ and
 * oracle/ref_harness.cpp runs them with their ray queries answered by
 * orc_ray_query below.  Against that run this restatement is bit-exact —
 * shading functions, camera rays, stored photons, grid lists, accumulated
 * frames and images (tests/test_oracle_ref_pin.py, fixtures from
 * tests/golden/make_ref_golden.py) — besides the closed-form known answers
 * of tests/golden/golden.json.  What the Vulkan driver decides (traversal
 * order, intersection rounding, the precision of exp / pow / sin / cos) is
 * not pinned by either: both runs use this oracle's FP64 queries and libm.
 */
#ifndef SRT_ORACLE_H
#define SRT_ORACLE_H

#include <stdint.h>
#include "../include/srt.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_scene orc_scene;

orc_scene* orc_scene_create(const srt_scene_arrays* arrays);
void orc_scene_destroy(orc_scene* s);
uint64_t orc_scene_num_tris(const orc_scene* s);

/* FP64 queries.  brute = 1 tests every triangle, otherwise an FP64 BVH.
 * Closest: (t, prim, u, v) lexicographic min over (t, prim); t_second (may be
 * NULL) is the smallest t of any OTHER triangle hit (inf if none), used to
 * detect ties, in both modes.
 * Any-hit (any_hit = 1): prim = 0 hit / 0xFFFFFFFF miss. */
void orc_trace(const orc_scene* s, const srt_ray* rays, uint32_t n, int any_hit, int brute,
               double* t_out, uint32_t* prim_out, double* u_out, double* v_out, double* t_second);

/* FP64: for ray i and flattened triangle prims[i], the ray parameter where
 * the ray's line meets the triangle's plane, the distance from that point
 * to the triangle's boundary (positive inside, negative outside) and
 * (cos_out, may be NULL) |cos| of the angle between ray and plane normal. */
void orc_tri_probe(const orc_scene* s, const srt_ray* rays, const uint32_t* prims, uint32_t n, double* t_out,
                   double* edge_out, double* cos_out);

/* Same op codes and record layouts as srt_test_device_math, plus
 * 102 blackbody_radiance of photon_emit.wgsl (in f32[2] -> out f32[1]),
 * 109 fresnel_thin_film_1d (cos, n1, n2, n3, d, lambda: in f32[6] -> out f32[1]),
 * 110 reflectance (cos, ior: in f32[2] -> out f32[1]). */
int orc_device_math(int op, uint32_t n, const void* in, void* out, const void* aux);

/* Photon emission for emitter ids [0, n_photons) (photon_emit.wgsl:154-331).
 * Writes the stored photons in emitter order (the order a sequential run of
 * the reference's atomicAdd would produce) and returns how many. */
uint32_t orc_photon_emit(const orc_scene* s, uint32_t n_photons, uint32_t frame, uint32_t max_bounces,
                         srt_photon* out, uint32_t* emitter_out, int n_threads);

/* Grid over a photon set (build_grid.wgsl:25-73, sort form): same outputs
 * as srt_photon_grid_build. */
void orc_photon_grid_build(const srt_photon* photons, uint32_t n, uint32_t frame, float cell,
                           uint32_t hash_bits, uint64_t* keys_out, uint32_t* ranges_out);

/* gather_photons (shader.wgsl:297-342) for n_q queries of 10 floats. */
void orc_photon_gather(const srt_photon* photons, uint32_t n, const float* queries, uint32_t n_q,
                       uint32_t frame, const srt_params* params, float* out);

/* One full frame (renderer/mod.rs:168-207): photon pass, grid, camera paths
 * for rows y with y % row_stride == row_phase (all rows: 1, 0), accumulate
 * and tonemap.  accum (w*h*4 floats) is read when cam->frame_count > 0 and
 * written for the rendered rows; ldr (w*h*4 bytes, may be NULL) likewise.
 * radiance_out (may be NULL): w*h*4 spectral radiance of the hero tuple
 * before XYZ conversion, for per-path comparisons.  stats_out (may be NULL):
 * [paths, closest rays, shadow rays, photons emitted, photons stored]. */
void orc_render_frame(const orc_scene* s, const srt_camera_uniform* cam, uint32_t w, uint32_t h,
                      const srt_params* params, uint32_t row_stride, uint32_t row_phase,
                      float* accum, uint8_t* ldr, float* radiance_out, uint64_t* stats_out, int n_threads);

/* The same frame with the photon pass replaced by a given photon set
 * (photons_in, n_photons_in, e.g. read back from the GPU's photon pass), so
 * that camera paths can be compared on identical photon maps. */
void orc_render_frame_photons(const orc_scene* s, const srt_camera_uniform* cam, uint32_t w, uint32_t h,
                              const srt_params* params, const srt_photon* photons_in, uint32_t n_photons_in,
                              uint32_t row_stride, uint32_t row_phase, float* accum, uint8_t* ldr,
                              float* radiance_out, uint64_t* stats_out, int n_threads);

/* One ray query as the oracle's shading code sees it: the part of a frame that
 * the Vulkan driver answers in the reference (rayQueryProceed on opaque
 * triangles).  any_hit = 1 (RAY_FLAG_TERMINATE_ON_FIRST_HIT) fills only hit.
 * Closest hits: t rounded to FP32, the instance, the primitive within its
 * mesh, the barycentrics u, v of vertices 1 and 2 and the front-face flag
 * (counter-clockwise as seen from the ray, in object space).  Used by
 * oracle/ref_harness.cpp to run the reference's translated shaders. */
typedef struct orc_query_hit {
    uint32_t hit, inst, prim, front;
    float t, u, v, pad;
} orc_query_hit;
void orc_ray_query(const orc_scene* s, const float o[3], const float d[3], float tmin, float tmax, int any_hit,
                   orc_query_hit* out);
/* The FP32 world-to-object 3x3 (row-major) of instance inst, as the oracle's
 * shading uses it. */
void orc_instance_w2o(const orc_scene* s, uint32_t inst, float out[9]);

int orc_max_threads(void);

/* The oracle's own scene generator (scenes.cpp): the arrays and camera
 * {x, y, z, yaw, pitch} of a preset (srt_preset), built without the product
 * library.  orc_preset_arrays points into the preset, which owns them. */
typedef struct orc_preset orc_preset;
orc_preset* orc_preset_create(int preset, uint32_t seed);
void orc_preset_destroy(orc_preset* s);
void orc_preset_arrays(const orc_preset* s, srt_scene_arrays* out, float camera[5]);
/* camera.rs:178-194 with closed-form inverses */
void orc_camera_uniform(const float pos[3], float yaw, float pitch, float aspect, uint32_t frame,
                        srt_camera_uniform* out);

#ifdef __cplusplus
}
#endif

#endif
