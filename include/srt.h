/*
 * srt.h — C ABI of the B200-native spectral path tracer.
 *
 * This is the drop-in boundary for the per-frame spectral path-tracing path of
 * wgpu-spectral-rt.  Each entry point names the reference interface it
 * replaces (path:line inside the reference project).  All signatures use
 * plain C types, pointers and sizes; no CUDA or torch type appears here.
 *
 * Ownership: the library owns every device allocation.  Host arrays passed in
 * are copied before the call returns.  Handles may be destroyed in any order:
 * a context destroyed while scenes, renderers or batches created on it are
 * alive is released with the last of them.  A handle is not thread-safe; use
 * one context per host thread.
 *
 * Errors: every call returns an srt_status.  No exception or abort crosses
 * the ABI.  srt_get_error_string(ctx) returns the last error text of a
 * context (NULL ctx: the last error of a failed srt_ctx_create).
 */
#ifndef SRT_H
#define SRT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SRT_ABI_VERSION 4u

/* Status codes.  Replaces unwrap()/panic! and wgpu::SurfaceError
 * (src/app.rs:70-77, src/wgpu_ctx.rs:36-42). */
typedef enum srt_status {
    SRT_OK = 0,
    SRT_ERR_INVALID_ARG = 1,
    SRT_ERR_OOM = 2,
    SRT_ERR_CUDA = 3,
    SRT_ERR_TIMEOUT = 4,       /* a bounded device wait gave up */
    SRT_ERR_DEVICE_ASSERT = 5, /* a device-side check recorded an error */
    SRT_ERR_NO_DEVICE = 6,
    SRT_ERR_UNSUPPORTED = 7,
    SRT_ERR_CAPACITY = 8       /* the request exceeds a fixed capacity of the library */
} srt_status;

/* ------------------------------------------------------------------------ */
/* Record layouts.  Byte-compatible with the reference's #[repr(C)] types.  */
/* ------------------------------------------------------------------------ */

/* src/scene/geometry.rs:4-9 (32 B). pos.w = 1, normal.w = 0. */
typedef struct srt_vertex {
    float pos[4];
    float normal[4];
} srt_vertex;

/* src/scene/builder.rs:5-10 (32 B).
 * extra.x = material type:
 *   0 Lambert (color.rgb reflectance)
 *   1 GGX metal (extra.y roughness alpha, clamped >= 0.001)
 *   2 Cauchy dielectric (extra.z = A, extra.w = B in um^2)
 *   3 blackbody emitter (color.r = temperature K, color.g = intensity,
 *     extra.y > 0: emit from both faces)
 *   4 Airy thin film (extra.y = thickness nm (>= 50), extra.z = n2, extra.w = n3)
 *   5 thin-film-coated GGX (no reference counterpart): color.w = roughness
 *     alpha, extra.y = film thickness nm, extra.z = n2 film, extra.w = n3
 *     substrate; reflection only. */
typedef struct srt_material {
    float color[4];
    float extra[4];
} srt_material;

/* src/scene/builder.rs:13-20 (64 B). World-space light triangle.
 * params = (type, temperature K, intensity, pad). */
typedef struct srt_light {
    float v0[4];
    float v1[4];
    float v2[4];
    float params[4];
} srt_light;

/* src/scene/builder.rs:22-28 (16 B). */
typedef struct srt_mesh_info {
    uint32_t vertex_offset;
    uint32_t index_offset;
    uint32_t pad[2];
} srt_mesh_info;

/* One instance: src/scene/builder.rs:41-45 (InstanceData).  transform is a
 * column-major 4x4 object-to-world matrix (glam Mat4 memory order). */
typedef struct srt_instance {
    uint32_t mesh_id;
    uint32_t mat_id;
    uint32_t pad[2];
    float transform[16];
} srt_instance;

/* src/scene/camera.rs:4-13 (272 B).  Matrices are column-major. */
typedef struct srt_camera_uniform {
    float view_inverse[16];
    float proj_inverse[16];
    float view[16];
    float proj[16];
    uint32_t frame_count;
    uint32_t pad[3];
} srt_camera_uniform;

/* src/renderer/shaders/photon_emit.wgsl:19-24 (32 B). */
typedef struct srt_photon {
    float position[3];
    float wavelength;
    float direction[3];
    float energy;
} srt_photon;

/* A ray for the batch trace entry points (32 B):
 * origin.xyz, tmin, direction.xyz, tmax. */
typedef struct srt_ray {
    float origin[3];
    float tmin;
    float dir[3];
    float tmax;
} srt_ray;

/* Closest-hit record (16 B).  prim = flattened triangle id (instance-major:
 * instance i's triangles follow instance i-1's), 0xFFFFFFFF on a miss.
 * u, v = barycentric weights of vertices 1 and 2 (the ray-query
 * "barycentrics", src/renderer/shaders/shader.wgsl:541-544). */
typedef struct srt_hit {
    float t;
    uint32_t prim;
    float u;
    float v;
} srt_hit;

/* Per-renderer parameters.  Defaults (srt_params_default) reproduce the
 * reference's hard-coded constants. */
typedef struct srt_params {
    uint32_t max_depth;          /* MAX_DEPTH override 12: renderer/compute_pass.rs:26 */
    uint32_t photons_per_frame;  /* MAX_PHOTONS 2^20: renderer/mod.rs:18; 0 disables the photon pass */
    uint32_t hash_bits;          /* log2 HASH_SIZE = 22: renderer/mod.rs:19 */
    uint32_t photon_max_bounces; /* 5: photon_emit.wgsl:219 */
    uint32_t gather_cap;         /* 64: shader.wgsl:312 */
    uint32_t flags;              /* SRT_FLAG_* */
    float cell_size;             /* CELL_SIZE 0.02: shader.wgsl:275, build_grid.wgsl:23 */
    float gather_radius0;        /* initial radius 0.02: shader.wgsl:302 */
    float radius_exponent;       /* -0.15: shader.wgsl:303 */
    float spectral_radius;       /* 20 nm: shader.wgsl:279 */
    float photon_norm_count;     /* count in the density estimate; 0 = photons_per_frame
                                    (the reference divides by MAX_PHOTON: shader.wgsl:339) */
    uint32_t block_size;         /* trace/shade block size; 0 = autotuned default */
    uint32_t seed;               /* added to the per-frame random seeds of camera paths and
                                    photons; 0 = the reference's sample streams */
} srt_params;

#define SRT_FLAG_FP64_ACCUM   0x1u  /* keep an FP64 accumulation buffer beside the FP32 one */
#define SRT_FLAG_NO_GRAPH     0x2u  /* launch kernels directly instead of a CUDA graph */
#define SRT_FLAG_STAGE_TIMING 0x4u  /* record per-stage CUDA events (srt_renderer_get_stats) */
#define SRT_FLAG_COUNT_VISITS 0x8u  /* traversal counts visited nodes and tested triangles */
#define SRT_FLAG_RAY_SORT     0x10u /* sort secondary camera rays by direction and origin before
                                       tracing (pays off only when the BVH does not fit in L2) */
#define SRT_FLAG_GUIDING      0x20u /* neural path guiding of Lambert continuations (no reference
                                       counterpart): a learned vMF mixture, one-sample MIS with the
                                       cosine lobe, trained after every frame; not with RAY_SORT */
#define SRT_FLAG_GUIDE_FROZEN 0x40u /* with SRT_FLAG_GUIDING: sample the guide, do not train it */

/* Per-renderer statistics of the frames rendered since the last reset. */
typedef struct srt_stats {
    uint64_t frames;
    uint64_t paths;             /* camera paths started */
    uint64_t rays_closest;      /* camera-path closest-hit rays */
    uint64_t rays_shadow;       /* any-hit (shadow) rays */
    uint64_t rays_photon;       /* photon-pass closest-hit rays */
    uint64_t photons_emitted;
    uint64_t photons_stored;
    uint64_t nodes_visited[3];  /* SRT_FLAG_COUNT_VISITS only: camera closest, shadow, photon */
    uint64_t tris_tested[3];    /* SRT_FLAG_COUNT_VISITS only: camera closest, shadow, photon */
    double ms_photon_pass;      /* SRT_FLAG_STAGE_TIMING only: summed stage times */
    double ms_trace_closest;
    double ms_shade;
    double ms_trace_shadow;
    double ms_finalize;
    double ms_raygen;
    uint64_t launches_trace_closest;
    uint64_t kernel_launches;   /* kernels launched by the library in these frames */
    double ms_guide_train;      /* SRT_FLAG_STAGE_TIMING + SRT_FLAG_GUIDING: training step times */
    double ms_tail;             /* SRT_FLAG_STAGE_TIMING: the tail kernel (srt_renderer_set_tail) */
    uint32_t tail_first;        /* first bounce the tail kernel runs (max_depth: none) */
    uint32_t pad;
} srt_stats;

/* Per-bounce statistics of a renderer's frames since the last
 * srt_renderer_reset_stats (diagnostics of the wavefront; no reference
 * counterpart).  Index [kind][bounce], kind 0 camera closest-hit rays, 1 shadow
 * rays, 2 photon rays: rays traced; with SRT_FLAG_COUNT_VISITS the BVH8 nodes
 * visited and triangles tested; with SRT_FLAG_STAGE_TIMING the traversal time
 * (CUDA events) of the closest-hit (ms[0]) and shadow (ms[1]) launches. */
#define SRT_MAX_BOUNCE_STATS 32
typedef struct srt_bounce_stats {
    uint64_t rays[3][SRT_MAX_BOUNCE_STATS];
    uint64_t nodes[3][SRT_MAX_BOUNCE_STATS];
    uint64_t tris[3][SRT_MAX_BOUNCE_STATS];
    double ms[2][SRT_MAX_BOUNCE_STATS];
} srt_bounce_stats;

typedef struct srt_ctx srt_ctx;
typedef struct srt_scene srt_scene;
typedef struct srt_scene_builder srt_scene_builder;
typedef struct srt_renderer srt_renderer;

/* ------------------------------------------------------------------------ */
/* Context: replaces WgpuContext::new / resize (src/wgpu_ctx.rs:13-81).       */
/* ------------------------------------------------------------------------ */

/* Create a context on CUDA device `device`.  `stream` is a cudaStream_t to
 * launch on (NULL: the library creates a non-blocking stream). */
srt_status srt_ctx_create(int device, void* stream, srt_ctx** out);
srt_status srt_ctx_destroy(srt_ctx* ctx);
const char* srt_get_error_string(const srt_ctx* ctx);
/* The cudaStream_t the context launches on. */
void* srt_ctx_stream(srt_ctx* ctx);
/* Wait for the context's stream; returns a pending device error, if any. */
srt_status srt_ctx_synchronize(srt_ctx* ctx);
uint32_t srt_abi_version(void);
/* Number of SMs of the context's device. */
int srt_ctx_sm_count(const srt_ctx* ctx);
/* BVH builder for the scenes built next on this context: binned SAH
 * (default) or the Morton-ordered LBVH.  Both are collapsed into the same
 * 8-wide compressed nodes; the choice changes speed, never results. */
#define SRT_BVH_SAH  0
#define SRT_BVH_LBVH 1
srt_status srt_ctx_set_bvh_builder(srt_ctx* ctx, int builder);
/* Children per BVH node (2..8, default 8) for the scenes built next: the
 * collapse stops expanding a node at `width` children; nodes keep the 8-slot
 * compressed format, so the same traversal runs every width.  Like the
 * builder, the width changes speed, never results.  No reference
 * counterpart (the driver builds the reference's BLAS/TLAS). */
srt_status srt_ctx_set_bvh_width(srt_ctx* ctx, uint32_t width);
/* Triangles of the largest BVH leaf (1..3, default 2) for the scenes built
 * next: a collapsed subtree of at most that many triangles is listed in its
 * parent node, a larger one becomes a node.  Smaller leaves mean more node
 * visits and fewer triangle tests per ray (config 2: 2 is faster than 3 for
 * closest hits, slower for shadow rays, faster per frame).  Rebuilds
 * (srt_scene_rebuild_bvh) keep the scene's leaf size.  Changes speed, never
 * results.  No reference counterpart (the driver builds the reference's
 * BLAS/TLAS). */
srt_status srt_ctx_set_bvh_leaf_size(srt_ctx* ctx, uint32_t max_triangles);
/* Rebuilds a scene's tree with `width` children per node (same builder).
 * Waits for the device; renderers and batches using the scene pick up the
 * new tree at their next frame (they capture their frame again). */
srt_status srt_scene_rebuild_bvh(srt_scene* s, uint32_t width);
srt_status srt_scene_bvh_width(const srt_scene* s, uint32_t* width);

/* ------------------------------------------------------------------------ */
/* Scene API: SceneBuilder (src/scene/builder.rs:47-267).                     */
/* The builder is host-only; srt_scene_builder_build uploads it and builds    */
/* the acceleration structure on the GPU (builder.rs:131-266).                */
/* ------------------------------------------------------------------------ */

srt_status srt_scene_builder_create(srt_scene_builder** out);
srt_status srt_scene_builder_destroy(srt_scene_builder* b);
/* builder.rs:70-74 */
uint32_t srt_scene_builder_add_material(srt_scene_builder* b, const srt_material* m);
/* builder.rs:76-91 */
uint32_t srt_scene_builder_add_mesh(srt_scene_builder* b, const srt_vertex* v, uint32_t n_vertices,
                                    const uint32_t* indices, uint32_t n_indices);
/* builder.rs:93-99; transform column-major 4x4 */
srt_status srt_scene_builder_add_instance(srt_scene_builder* b, uint32_t mesh_id, uint32_t mat_id,
                                          const float transform[16]);
/* builder.rs:101-129: adds the instance and one world-space srt_light per triangle */
srt_status srt_scene_builder_add_light_instance(srt_scene_builder* b, uint32_t mesh_id, uint32_t mat_id,
                                                const float transform[16], const float params[4]);
/* Counts and read-only views of the builder's host arrays (for CPU comparisons and
 * for srt_scene_build).  Pointers stay valid until the builder changes. */
typedef struct srt_scene_arrays {
    const srt_vertex* vertices;     uint32_t n_vertices;
    const uint32_t* indices;        uint32_t n_indices;
    const srt_mesh_info* mesh_infos; uint32_t n_meshes;
    const srt_material* materials;  uint32_t n_materials;
    const srt_instance* instances;  uint32_t n_instances;
    const srt_light* lights;        uint32_t n_lights;
} srt_scene_arrays;
srt_status srt_scene_builder_arrays(const srt_scene_builder* b, srt_scene_arrays* out);
srt_status srt_scene_builder_build(srt_ctx* ctx, const srt_scene_builder* b, srt_scene** out);

/* Flat form of SceneBuilder::build: uploads already-assembled arrays.
 * n_lights may be 0 (no light sampling, no photons). */
srt_status srt_scene_build(srt_ctx* ctx, const srt_scene_arrays* arrays, srt_scene** out);
srt_status srt_scene_destroy(srt_scene* s);
/* Moves instances (scene-side GPU ingestion for dynamic scenes; no reference
 * counterpart): ids[k] gets the column-major object-to-world transform
 * transforms[16 k .. 16 k + 15].  On the device: the moved instances'
 * triangles are re-transformed, the light triangles of moved light
 * instances (srt_scene_builder_add_light_instance) re-expanded, and the BVH8
 * refitted (same topology; boxes recomputed bottom-up and re-quantised).
 * Buffers are updated in place, so renderers (and their captured graphs)
 * keep working; the scene bounds used to normalise guide inputs stay as
 * built.  Waits for the context's stream before and after. */
srt_status srt_scene_update_instances(srt_scene* scene, const uint32_t* ids, const float* transforms, uint32_t n);
/* The scene's world-space light triangles as the device holds them (for a
 * builder scene: expanded on the GPU); *count = number of lights. */
srt_status srt_scene_read_lights(srt_scene* scene, srt_light* out, uint32_t capacity, uint32_t* count);
/* Raw copies of the BVH8 nodes (80 B each) and leaf triangle slots (48 B). */
srt_status srt_scene_read_bvh(srt_scene* scene, void* nodes, uint64_t node_bytes, void* tris, uint64_t tri_bytes);
/* Flattened triangle count and BVH node count of a built scene. */
srt_status srt_scene_info(const srt_scene* s, uint64_t* n_triangles, uint64_t* n_nodes, uint32_t* bvh_depth);

/* Procedural geometry (src/scene/geometry.rs:12-232).  Call with NULL
 * outputs to query counts, then with arrays of at least that size. */
srt_status srt_geometry_plane(srt_vertex* v, uint32_t* n_v, uint32_t* idx, uint32_t* n_i);
srt_status srt_geometry_cube(srt_vertex* v, uint32_t* n_v, uint32_t* idx, uint32_t* n_i);
srt_status srt_geometry_icosphere(uint32_t subdivisions, srt_vertex* v, uint32_t* n_v, uint32_t* idx, uint32_t* n_i);
/* UV sphere, radius 0.5: `slices` around, `stacks` from pole to pole. */
srt_status srt_geometry_uv_sphere(uint32_t slices, uint32_t stacks, srt_vertex* v, uint32_t* n_v, uint32_t* idx, uint32_t* n_i);

/* Scene presets (src/scene/cornell_box.rs:6-110, src/scene/custom.rs:6-116)
 * and the benchmark scenes.  Each fills an empty builder and returns the
 * preset's default camera (position xyz, yaw, pitch in radians). */
typedef enum srt_preset {
    SRT_PRESET_CORNELL_BOX = 0,   /* cornell_box.rs:6-110 */
    SRT_PRESET_CUSTOM_PRISM = 1,  /* custom.rs:6-116 */
    SRT_PRESET_CONFIG1 = 2,       /* Cornell walls + 2-tri light + dispersive UV sphere */
    SRT_PRESET_CONFIG2 = 3,       /* displaced level-8 icosphere + 64 coated GGX spheres */
    SRT_PRESET_CAUSTIC_SLAB = 4,  /* dispersive slab under a slit light + floor + config-1 mesh */
    SRT_PRESET_INDIRECT_ROOM = 5, /* Cornell walls lit only by the ceiling spot above an
                                     upward-facing light hidden under a panel (guiding study) */
    SRT_PRESET_BATCH_RANDOM = 6   /* seeded batch scene: a triangle budget log-uniform in
                                     [1e4, 2e6] filled by a displaced icosphere and GGX,
                                     thin-film and dielectric UV spheres in a Cornell room */
} srt_preset;
srt_status srt_scene_builder_add_preset(srt_scene_builder* b, int preset, uint32_t seed, float camera_out[5]);

/* CameraController::build_uniform (src/scene/camera.rs:178-194):
 * look_at_rh + perspective_rh(45 deg, aspect, 0.1, 100). */
srt_status srt_camera_build_uniform(const float position[3], float yaw, float pitch, float aspect,
                                    uint32_t frame_count, srt_camera_uniform* out);

/* ------------------------------------------------------------------------ */
/* Renderer API: Renderer::new / render (src/renderer/mod.rs:45-207).         */
/* ------------------------------------------------------------------------ */

srt_params srt_params_default(void);
srt_status srt_renderer_create(srt_ctx* ctx, srt_scene* scene, uint32_t width, uint32_t height,
                               const srt_params* params, srt_renderer** out);
srt_status srt_renderer_destroy(srt_renderer* r);
/* One frame = one sample per pixel: photon emit -> grid build -> camera
 * paths -> accumulate + tonemap (renderer/mod.rs:168-207).  cam->frame_count
 * seeds the RNG and resets the accumulation when 0 (engine.rs:154-166,
 * shader.wgsl:803-805).  Asynchronous on the context's stream.  A frame also
 * builds, beside its camera paths, the photon map of frame count
 * cam->frame_count + 1 for the next call; a call with another count, or after
 * the scene changed, builds its own map first.  The images are those of
 * building each frame's map inside the frame. */
srt_status srt_render_frame(srt_renderer* r, const srt_camera_uniform* cam);
/* Renderer.frame_count (renderer/mod.rs:30, incremented at :204). */
uint32_t srt_renderer_frame_count(const srt_renderer* r);
srt_status srt_renderer_set_frame_count(srt_renderer* r, uint32_t frame_count);
/* Zero the accumulation buffers and set frame_count to 0 (engine.rs:154-156). */
srt_status srt_reset_accumulation(srt_renderer* r);
/* Linear accumulation (shader.wgsl:801-808): width*height float4
 * (sum r, sum g, sum b, sample count), row 0 = bottom row. */
srt_status srt_read_accum_f32(srt_renderer* r, float* rgba);
/* FP64 accumulation (SRT_FLAG_FP64_ACCUM): width*height double4. */
srt_status srt_read_accum_f64(srt_renderer* r, double* rgba);
/* Resume of an accumulation (no reference counterpart; the reference keeps
 * its sums only in GPU memory): loads w*h RGBA FP64 sums in the layout
 * srt_read_accum_f64 returns into the FP64 accumulation, and their FP32
 * roundings into the FP32 one.  A later frame whose camera uniform carries
 * frame_count N > 0 adds to them, so a long render read back after N frames
 * continues where it stopped.  Requires SRT_FLAG_FP64_ACCUM. */
srt_status srt_write_accum_f64(srt_renderer* r, const double* rgba);
/* Tonemapped RGBA8 storage texture (shader.wgsl:809-822), row 0 = bottom
 * row, `pitch` bytes per row (>= 4*width). */
srt_status srt_read_ldr_rgba8(srt_renderer* r, uint8_t* out, uint32_t pitch);
/* Read-back without a stall (no reference counterpart): enqueues, after the
 * frames rendered so far, a copy of the RGBA8 image (row 0 first, tightly
 * packed) into one of two pinned host slots the renderer owns, and returns
 * a ticket.  srt_ldr_wait(ticket) blocks until that copy has landed and
 * points *pixels at it; the slot is reused by the second read_ldr_async
 * after it, so a ticket is valid until then.  A frame loop that renders
 * frame k+1 before waiting for frame k's ticket keeps the GPU busy. */
srt_status srt_read_ldr_async(srt_renderer* r, uint32_t* ticket);
srt_status srt_ldr_wait(srt_renderer* r, uint32_t ticket, const uint8_t** pixels);
/* Engine::save_screenshot + ScreenshotSaver (engine.rs:191-244,
 * screenshot.rs:27-103): row flip, sRGB OETF of the 8-bit values, PNG file. */
srt_status srt_save_screenshot(srt_renderer* r, const char* path);
/* ScreenshotSaver::process_and_save (screenshot.rs:27-103) on host memory:
 * `rgba` holds h rows of `pitch` bytes, row 0 = bottom row; writes a PNG
 * with the rows flipped and the sRGB OETF applied to the 8-bit values. */
srt_status srt_screenshot_write(const char* path, const uint8_t* rgba, uint32_t width, uint32_t height,
                                uint32_t pitch);
/* The same two steps with the PNG encoding on a worker thread, as the
 * reference's engine does with its screenshot channel (engine.rs:39-45,
 * :242): srt_save_screenshot_async reads the image back (synchronously, like
 * Engine::save_screenshot) and queues the encoding and the file write;
 * srt_screenshot_write_async copies `rgba` and queues the same.  Jobs run in
 * order on one library-owned thread.  srt_screenshot_flush blocks until every
 * queued write is done and returns in *failed_writes (may be NULL) how many
 * failed since the previous flush.  Queued writes finish before the process
 * exits. */
srt_status srt_save_screenshot_async(srt_renderer* r, const char* path);
srt_status srt_screenshot_write_async(const char* path, const uint8_t* rgba, uint32_t width, uint32_t height,
                                      uint32_t pitch);
srt_status srt_screenshot_flush(uint32_t* failed_writes);
srt_status srt_renderer_get_stats(srt_renderer* r, srt_stats* out);
srt_status srt_renderer_get_bounce_stats(srt_renderer* r, srt_bounce_stats* out);
/* Bounces first_bounce .. max_depth - 1 of every frame run as one persistent
 * kernel that follows each remaining path to its end (closest hit, shading,
 * shadow ray) instead of one closest-hit, shading and shadow launch per
 * bounce: the same arithmetic per path, so the same image, with the latency
 * of the short last bounces paid once.  It runs one path per thread at a
 * time, so it pays once the live paths fit in about one wave of it.
 * SRT_TAIL_AUTO (the default): the renderer reads back the path counts of
 * its first frame without waiting for them and, once they are there, starts
 * the tail at the first bounce >= 1 whose live paths fit in one wave of the
 * tail kernel's resident threads (a batch: the scenes' paths summed), for a
 * guiding renderer not before the end of its guided bounces; frames before
 * that run bounce by bounce.  0 = bounce by bounce.  Not used with
 * SRT_FLAG_RAY_SORT, nor where a set number of guided bounces reaches it
 * (srt_renderer_guide_set_bounces).  srt_stats.tail_first reports the bounce
 * in use.  No reference counterpart. */
#define SRT_TAIL_AUTO 0xFFFFFFFFu
srt_status srt_renderer_set_tail(srt_renderer* r, uint32_t first_bounce);
srt_status srt_renderer_reset_stats(srt_renderer* r);
/* The photon set of the last frame in emission order (photon_emit.wgsl
 * storage): copies min(count, capacity) photons to `out` (may be NULL) and
 * the stored count to *count. */
srt_status srt_renderer_read_photons(srt_renderer* r, srt_photon* out, uint32_t capacity, uint32_t* count);

/* ------------------------------------------------------------------------ */
/* Path kernels exposed on their own (parity checks and batch users).        */
/* ------------------------------------------------------------------------ */

/* Closest-hit (any_hit = 0) or any-hit (any_hit = 1, terminate on first hit)
 * queries for a batch of rays in host memory: the ray queries of
 * shader.wgsl:561-566, :654-659 and photon_emit.wgsl:222-227.  Any-hit
 * writes prim = 0 for a hit and 0xFFFFFFFF for a miss. */
srt_status srt_trace_rays(srt_scene* s, const srt_ray* rays, uint32_t n, srt_hit* hits, int any_hit);

/* Photon hash grid over a given photon set (build_grid.wgsl:25-73), built
 * by a stable radix sort of cell keys instead of linked lists.
 * keys_out[i]  = (hash << 32) | photon index, ascending (n entries);
 *                photons with energy == 0 get hash = 2^hash_bits.
 * ranges_out   = 2^hash_bits pairs (start, end) into keys_out, (0,0) empty.
 * Any output may be NULL. */
srt_status srt_photon_grid_build(srt_ctx* ctx, const srt_photon* photons, uint32_t n, uint32_t frame_count,
                                 float cell_size, uint32_t hash_bits, uint64_t* keys_out, uint32_t* ranges_out);

/* Photon hash grid that allocates nothing.  This entry point has no
 * counterpart in the reference.
 *
 * Who it is for: callers that cannot call cudaMalloc, e.g. an engine or
 * framework whose own pool allocator already owns the GPU's memory (an
 * allocation behind its back can fail or fragment the pool), or a real-time
 * frame loop that forbids allocation once it is running.
 *
 * It computes the same keys_out and ranges_out as srt_photon_grid_build, but
 * every pointer is DEVICE memory owned by the caller (photons: n records;
 * keys_out: n entries; ranges_out: 2 * 2^hash_bits entries; either output
 * may be NULL) and the work is enqueued on `stream` (a cudaStream_t, NULL =
 * legacy default stream) of the current device.  No context is needed.
 * Temporary storage comes from one fixed __device__ array in the library
 * (16.5 MiB, held by every GPU that loads the library until exit); n above
 * SRT_GRID_NOALLOC_MAX_PHOTONS returns SRT_ERR_CAPACITY.  Alignment:
 * photons 16 bytes, keys_out and ranges_out 8 bytes; a misaligned pointer
 * returns SRT_ERR_INVALID_ARG before any device work.  n = 0 only clears
 * ranges_out.
 *
 * The first call on a device looks up that array's device address (once per
 * device, with the device current); make that first call before any stream
 * capture.  The address belongs to the CUDA context that was current at the
 * lookup: a call under another context of the same device (after
 * cudaDeviceReset, or one made current through the driver API) looks it up
 * again, so make such a call outside stream capture too.  All calls share
 * the array: calls that overlap on the GPU race and must be serialised by the
 * caller.  Launch failures are reported from each launch's own status; an
 * error that an unrelated earlier call left pending is neither reported nor
 * cleared.  Asynchronous: synchronise `stream` before reading the outputs. */
#define SRT_GRID_NOALLOC_MAX_PHOTONS (1u << 20)
srt_status srt_photon_grid_build_noalloc(void* stream, const srt_photon* photons, uint32_t n, uint32_t frame_count,
                                         float cell_size, uint32_t hash_bits, uint64_t* keys_out,
                                         uint32_t* ranges_out);

/* Density estimate at query points (gather_photons, shader.wgsl:297-342)
 * against a photon set: builds the grid then gathers.  query = n_q records
 * of (position.xyz, normal.xyz, wavelengths[4]) = 10 floats; out = 4 floats
 * per query. */
srt_status srt_photon_gather(srt_ctx* ctx, const srt_photon* photons, uint32_t n, const float* queries,
                             uint32_t n_q, uint32_t frame_count, const srt_params* params, float* out);

/* Device unit kernels over the shading math, for parity checks.  op:
 *  0 pcg_hash(u32 in[i]) -> u32 out[i]
 *  1 sample_cie_xyz(lambda)                       in f32[1] -> out f32[3]
 *  2 blackbody_radiance(lambda, T)                in f32[2] -> out f32[1]
 *  3 rgb_to_spectrum(rgb[3], lambda[4])           in f32[7] -> out f32[4]
 *  4 fresnel_thin_film(cos, n1, n2, n3, d, lambda[4]) in f32[9] -> out f32[4]
 *  5 hero wavelengths from rng seed               in u32[1] -> out f32[5] (4 lambdas, sum pdf)
 *  6 sample_bsdf: in f32[24] = r_dir[3], ffnormal[3], material[8], front(0/1),
 *    wavelengths[4], throughput[4], rng seed (bits) -> out f32[10] =
 *    scatter_dir[3], attenuation[4], absorbed(0/1), rng out (bits), pad
 *  7 grid hash(position[3], frame bits, cell)     in f32[5] -> out u32[1]
 *  8 camera ray(cam uniform from `aux`, pixel x, y, width, height as bits, rng seed) in u32[5]
 *    -> out f32[7] origin[3] dir[3] rng out (bits)
 * in/out strides are the per-op sizes above; n records. */
srt_status srt_test_device_math(srt_ctx* ctx, int op, uint32_t n, const void* in, void* out, const void* aux);

/* ------------------------------------------------------------------------ */
/* Neural path guiding (no reference counterpart; SRT_FLAG_GUIDING).          */
/* Network: 10 inputs (position in the scene bounds, shading normal,          */
/* outgoing direction, wavelength) -> sin/cos encoding of 6 octaves (128)     */
/* -> 4 x 64 ReLU -> 48 outputs: 8 vMF lobes (direction 3, log kappa,          */
/* logit) and the selection logit.  Weights: one float vector of              */
/* srt_guide_param_count() values, W_l [out][in] row-major then b_l, l=0..4.  */
/* ------------------------------------------------------------------------ */
uint32_t srt_guide_param_count(void);
/* Deterministic initial weights (He-uniform, output layer scaled by 0.1). */
srt_status srt_guide_default_weights(uint64_t seed, float* out, uint32_t n);
/* Checkpoint / restore of a guiding renderer's FP32 weights (restore resets Adam). */
srt_status srt_renderer_guide_get_weights(srt_renderer* r, float* out, uint32_t n);
srt_status srt_renderer_guide_set_weights(srt_renderer* r, const float* w, uint32_t n);
/* Checkpoint / resume of the whole training state: FP32 weights and the two
 * Adam moments (srt_guide_param_count() floats each) and the Adam step count.
 * set_state puts all of it back, so training continues where it stopped. */
/* Failure-path test: one block waits on a device barrier that never
 * completes, giving up after `polls` polls (1..2^20) like the tensor-core
 * kernels' bounded waits; returns SRT_ERR_TIMEOUT, and the context stays
 * usable. */
srt_status srt_test_wait_timeout(srt_ctx* ctx, uint32_t polls);
srt_status srt_renderer_guide_get_state(srt_renderer* r, float* params, float* adam_m, float* adam_v,
                                        uint32_t* adam_step);
srt_status srt_renderer_guide_set_state(srt_renderer* r, const float* params, const float* adam_m,
                                        const float* adam_v, uint32_t adam_step);
srt_status srt_renderer_guide_info(srt_renderer* r, uint32_t* adam_steps, uint32_t* record_threshold);
/* Adam learning rate (default 1e-3; < 0 keeps it) and training samples
 * recorded per frame (default 65536, at most 262144; 0 keeps it). */
srt_status srt_renderer_guide_configure(srt_renderer* r, float lr, uint32_t batch);
/* Adam steps per frame (1..16, default 1): the frame's training records are
 * split into `steps` consecutive sub-batches, one forward/backward, gradient
 * and Adam step each. */
srt_status srt_renderer_guide_set_steps(srt_renderer* r, uint32_t steps);
/* Guided bounces (>= 1, default 8): the guide samples the Lambert
 * continuations of bounces < `bounces` (and trains on them); later Lambert
 * vertices sample the cosine lobe as the reference does.  The automatic tail
 * (srt_renderer_set_tail) starts after the guided bounces; a set tail that
 * would start before their end is not used.  The estimator stays unbiased
 * either way; fewer guided bounces trade variance for time. */
srt_status srt_renderer_guide_set_bounces(srt_renderer* r, uint32_t bounces);
/* Test entry points (host buffers).  forward: x [n][10] -> raw outputs [n][48].
 * mixture: raw [n][48], omega [n][3], u [n][3] -> [n][4] = (pdf(omega),
 * sampled direction).  train: loss gradients summed over n samples
 * (weights as given) and, when params_out/m_out/v_out are non-NULL, one Adam
 * step (gradients divided by n; step adam_step + 1). */
srt_status srt_guide_test_forward(srt_ctx* ctx, const float* params, const float* x, uint32_t n, float* out);
/* The same forward pass on the tcgen05 / tensor-memory kernel. */
srt_status srt_guide_test_forward_tc(srt_ctx* ctx, const float* params, const float* x, uint32_t n, float* out);
/* Inference kernel of a guiding renderer: mma.sync fragments or tcgen05 MMAs
 * into tensor memory (same network, same results up to FP32 summation order). */
#define SRT_GUIDE_INFER_MMA_SYNC 0
#define SRT_GUIDE_INFER_TCGEN05  1
srt_status srt_renderer_guide_set_inference(srt_renderer* r, int kind);
/* Training step kernels of a guiding renderer: mma.sync forward/backward
 * with a split-K weight-gradient product, or one fused tcgen05 kernel per
 * step (forward, loss gradient, backward and weight gradients of 128-record
 * tiles, the weight gradients accumulated in tensor memory; the default).
 * The batched renderer's grouped training uses the mma.sync kernels. */
#define SRT_GUIDE_TRAIN_MMA_SYNC 0
#define SRT_GUIDE_TRAIN_TCGEN05  1
srt_status srt_renderer_guide_set_training(srt_renderer* r, int kind);
srt_status srt_guide_test_mixture(srt_ctx* ctx, const float* raw, const float* omega, const float* u, uint32_t n,
                                  float* out);
/* The same for the mixture functions of the tcgen05 inference kernel (fast
 * exponentials, logarithms, reciprocal square roots and division). */
srt_status srt_guide_test_mixture_tc(srt_ctx* ctx, const float* raw, const float* omega, const float* u, uint32_t n,
                                     float* out);
srt_status srt_guide_test_train(srt_ctx* ctx, const float* params, const float* adam_m, const float* adam_v,
                                uint32_t adam_step, float lr, const float* x, const float* omega,
                                const float* pdf_bsdf, const float* weight, uint32_t n, float* grad_out,
                                float* params_out, float* m_out, float* v_out);
/* The same on the fused tcgen05 training kernel. */
srt_status srt_guide_test_train_tc(srt_ctx* ctx, const float* params, const float* adam_m, const float* adam_v,
                                   uint32_t adam_step, float lr, const float* x, const float* omega,
                                   const float* pdf_bsdf, const float* weight, uint32_t n, float* grad_out,
                                   float* params_out, float* m_out, float* v_out);

/* ------------------------------------------------------------------------ */
/* Headless presentation: the reference's raster steps as CUDA kernels.       */
/* ------------------------------------------------------------------------ */
/* Letterbox blit (shaders/blit.wgsl:7-34, renderer/blit_pass.rs:114-154):
 * the RGBA8 image src (sw x sh) drawn as an aspect-fit quad into an RGBA8
 * window (ww x wh, row 0 at the top) cleared to blue, nearest-texel
 * sampling; srgb_target encodes with the sRGB OETF as an *Srgb swapchain
 * format would.  Host buffers, tightly packed. */
srt_status srt_blit_letterbox(srt_ctx* ctx, const uint8_t* src, uint32_t sw, uint32_t sh, uint32_t ww,
                              uint32_t wh, int srgb_target, uint8_t* out);
/* The same for the renderer's current RGBA8 image. */
srt_status srt_renderer_blit(srt_renderer* r, uint32_t ww, uint32_t wh, int srgb_target, uint8_t* out);
/* Photon point splat (shaders/debug_photons.wgsl:24-47, renderer/
 * debug_photons_pass.rs:74-139): photons with non-zero energy projected with
 * cam's view and proj matrices, one pixel each, colour (1, 0.6, 0.1) x 0.3
 * added (saturating) to rgba (w x h, in/out), alpha set to 0.3. */
srt_status srt_photon_splat(srt_ctx* ctx, const srt_photon* photons, uint32_t n, const srt_camera_uniform* cam,
                            uint32_t w, uint32_t h, uint8_t* rgba);
/* The same for the photons the renderer stored in its last frame. */
srt_status srt_renderer_splat_photons(srt_renderer* r, const srt_camera_uniform* cam, uint32_t w, uint32_t h,
                                      uint8_t* rgba);

/* ------------------------------------------------------------------------ */
/* Batched rendering (no reference counterpart): many scenes and viewports   */
/* of uneven size per iteration.  Per-scene photon passes, ray generation,   */
/* shading and finalisation run as parallel branches of one CUDA graph; the  */
/* closest-hit and shadow rays of all scenes are traced in one persistent    */
/* launch per bounce over per-scene queues (warps whose finished lanes take  */
/* the next ray of any scene).                                               */
/* ------------------------------------------------------------------------ */
typedef struct srt_batch srt_batch;
typedef struct srt_batch_tuning {
    uint32_t blocks_per_sm;  /* resident blocks per SM of the batched traversal (1..8) */
    uint32_t chunk;          /* rays a warp draws from the shared queue at once (32..1024, x32); the
                                default persistent traversal hands rays out lane by lane and ignores it */
    float ms_per_iteration;  /* autotune: time of one iteration with this choice */
    uint32_t candidates;     /* autotune: configurations timed */
    uint32_t bvh_width;      /* autotune: children per node of the scenes' trees it kept (it times the
                                other of 8 and 4 by rebuilding the trees; 0 = widths differ, not tuned) */
} srt_batch_tuning;
/* n <= 64 scenes; params: n entries (NULL: defaults); no STAGE_TIMING,
 * COUNT_VISITS or RAY_SORT flag in a batch. */
srt_status srt_batch_create(srt_ctx* ctx, uint32_t n, srt_scene* const* scenes, const uint32_t* widths,
                            const uint32_t* heights, const srt_params* params, srt_batch** out);
srt_status srt_batch_destroy(srt_batch* b);
uint32_t srt_batch_size(const srt_batch* b);
/* Borrowed handle of scene i's renderer: read its accumulation, image, stats
 * and photons with the srt_renderer_* calls; it is not destroyed or rendered
 * on its own. */
srt_renderer* srt_batch_renderer(srt_batch* b, uint32_t i);
/* One iteration (one sample per pixel) of every scene whose active[i] != 0
 * (active NULL: all); cams: n camera uniforms. */
srt_status srt_batch_render(srt_batch* b, const srt_camera_uniform* cams, const uint8_t* active);
srt_status srt_batch_get_tuning(const srt_batch* b, srt_batch_tuning* out);
srt_status srt_batch_set_tuning(srt_batch* b, const srt_batch_tuning* t);
/* Times `iterations` iterations of every candidate (blocks per SM; x chunk
 * for the chunked traversal), keeps the fastest, then clears every scene's
 * accumulation and statistics;
 * guided scenes get back the network and Adam state they had before. */
srt_status srt_batch_autotune(srt_batch* b, const srt_camera_uniform* cams, uint32_t iterations,
                              srt_batch_tuning* out);

#ifdef __cplusplus
}
#endif

#endif /* SRT_H */
