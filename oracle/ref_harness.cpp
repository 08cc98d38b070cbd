// ref_harness.cpp — runs the reference's own WGSL compute shaders on the CPU.
//
// TEST INFRASTRUCTURE ONLY.  oracle/wgsl_translate.py turns the reference's
// shader.wgsl, photon_emit.wgsl and build_grid.wgsl (read where they lie in
// the reference tree) into C++ under oracle/_ref/; this file binds their
// buffers the way the reference's passes do (renderer/mod.rs:168-207,
// photon_emit_pass.rs, build_grid_pass.rs, compute_pass.rs), dispatches
// their entry points (the photon and grid passes one invocation after
// another for a deterministic order, or concurrently for timing; the camera
// pass row-parallel, its invocations independent), and answers their ray
// queries with the oracle's FP64 query (orc_ray_query) — the part that the
// Vulkan driver answers in the reference.  The oracle's hand restatement
// (oracle.cpp) is then checked against this run of the reference's code
// (tests/test_oracle_ref_pin.py, tests/golden/make_ref_golden.py), and
// bench.py's reference arm times it.  The entry points bind module-scope
// state: one call at a time per process.
//
// Built by `make -C oracle ref` into oracle/_ref/libref_wgsl.so, only where
// the reference tree is present; nothing here is committed output.
#include <omp.h>

#include <cstring>
#include <vector>

#include "oracle.h"
#include "ref_runtime.h"

#include "_ref/shader.inc"
#include "_ref/photon_emit.inc"
#include "_ref/build_grid.inc"

using namespace wgsl_rt;

namespace {

static_assert(sizeof(wgsl_shader::Camera) == 260, "Camera uniform layout");
static_assert(sizeof(wgsl_shader::Photon) == 32 && sizeof(wgsl_photon_emit::Photon) == 32 &&
                  sizeof(wgsl_build_grid::Photon) == 32,
              "Photon layout");
static_assert(sizeof(wgsl_shader::Material) == 32 && sizeof(wgsl_shader::Vertex) == 32 &&
                  sizeof(wgsl_shader::MeshInfo) == 16 && sizeof(wgsl_shader::LightInfo) == 64,
              "record layouts");

constexpr uint32_t kMaxPhotons = 1u << 20;  // renderer/mod.rs MAX_PHOTONS (the dispatch size)
constexpr uint32_t kHashSize = 1u << 22;    // HASH_SIZE of both shaders

template <class Cam>
void load_camera(Cam& c, const srt_camera_uniform* u) {
    std::memcpy(static_cast<void*>(&c), u, sizeof(Cam));
}

}  // namespace

struct ref_scene {
    orc_scene* orc = nullptr;
    std::vector<srt_vertex> vertices;
    std::vector<uint32_t> indices;
    std::vector<srt_mesh_info> meshes;
    std::vector<srt_material> materials;
    std::vector<srt_light> lights;
    std::vector<uint32_t> custom;  // per instance: (mesh_id << 16) | mat_id (builder.rs:240)
    std::vector<mat4x3f> w2o;      // per instance world_to_object (columns)
    acceleration_structure tlas;
};

namespace {

// rayQueryProceed on the reference's opaque triangles (builder.rs:153):
// the oracle's FP64 query, reported in the fields the shaders read.
void trace_cb(void* ctx, const RayDesc& d, RayIntersection& out) {
    const ref_scene* S = static_cast<const ref_scene*>(ctx);
    const float o[3] = {d.origin.x, d.origin.y, d.origin.z}, dir[3] = {d.dir.x, d.dir.y, d.dir.z};
    const int any = (d.flags & RAY_FLAG_TERMINATE_ON_FIRST_HIT) != 0u;
    orc_query_hit h;
    orc_ray_query(S->orc, o, dir, d.tmin, d.tmax, any, &h);
    out = RayIntersection{};
    if (!h.hit) return;
    out.kind = 1u;
    if (any) return;  // the shadow ray reads only kind (shader.wgsl:654-659)
    out.t = h.t;
    out.instance_custom_data = S->custom[h.inst];
    out.instance_index = h.inst;
    out.primitive_index = h.prim;
    out.barycentrics = vec2f(h.u, h.v);
    out.front_face = h.front != 0u;
    out.world_to_object = S->w2o[h.inst];
}

template <class T, class U>
StorageArray<T> bind(const std::vector<U>& v) {
    static_assert(sizeof(T) == sizeof(U), "binding layout");
    StorageArray<T> a;
    a.p = reinterpret_cast<T*>(const_cast<U*>(v.data()));
    a.n = (uint32_t)v.size();
    return a;
}
template <class T, class U>
StorageArray<T> bind(U* p, uint32_t n) {
    static_assert(sizeof(T) == sizeof(U), "binding layout");
    StorageArray<T> a;
    a.p = reinterpret_cast<T*>(p);
    a.n = n;
    return a;
}

// Thread-local record of the first ray query of an invocation (the camera
// ray), for the camera-ray pin.
thread_local bool g_capture = false;
thread_local RayDesc g_first{};
void trace_capture_cb(void* ctx, const RayDesc& d, RayIntersection& out) {
    if (g_capture) {
        g_first = d;
        g_capture = false;
    }
    out = RayIntersection{};  // a miss: the invocation ends after its camera ray
}

}  // namespace

extern "C" {

ref_scene* ref_scene_create(const srt_scene_arrays* a) {
    ref_scene* s = new ref_scene();
    s->orc = orc_scene_create(a);
    s->vertices.assign(a->vertices, a->vertices + a->n_vertices);
    s->indices.assign(a->indices, a->indices + a->n_indices);
    s->meshes.assign(a->mesh_infos, a->mesh_infos + a->n_meshes);
    s->materials.assign(a->materials, a->materials + a->n_materials);
    s->lights.assign(a->lights, a->lights + a->n_lights);
    for (uint32_t i = 0; i < a->n_instances; ++i) {
        const srt_instance& in = a->instances[i];
        s->custom.push_back((in.mesh_id << 16) | in.mat_id);
        float w[9];
        orc_instance_w2o(s->orc, i, w);  // row-major 3x3
        mat4x3f m;
        for (uint32_t c = 0; c < 3; ++c) m.c[c] = vec3f(w[c], w[3 + c], w[6 + c]);
        // translation column: -W t (unused by the shaders, filled for completeness)
        const float* M = in.transform;
        const float tx = M[12], ty = M[13], tz = M[14];
        m.c[3] = vec3f(-(w[0] * tx + w[1] * ty + w[2] * tz), -(w[3] * tx + w[4] * ty + w[5] * tz),
                       -(w[6] * tx + w[7] * ty + w[8] * tz));
        s->w2o.push_back(m);
    }
    s->tlas.ctx = s;
    s->tlas.trace = trace_cb;
    return s;
}

void ref_scene_destroy(ref_scene* s) {
    if (!s) return;
    orc_scene_destroy(s->orc);
    delete s;
}

// Photon pass (photon_emit.wgsl main) for emitter ids [0, n_emit).  With
// n_threads = 1 the invocations run in id order (the order a sequential run
// of its atomicAdd gives, which the oracle reproduces); with more threads
// (0 = all) they run concurrently and the stored photons land in the order
// the atomic hands out, as on a GPU.  photons must hold 2^20 records (the
// reference's buffer); returns the atomic counter, which can exceed the
// number stored.
uint32_t ref_photon_emit(ref_scene* s, const srt_camera_uniform* cam, uint32_t n_emit, srt_photon* photons,
                         int n_threads) {
    namespace P = wgsl_photon_emit;
    P::tlas = s->tlas;
    P::lights = bind<P::LightInfo>(s->lights);
    P::photons = bind<P::Photon>(photons, kMaxPhotons);
    P::photon_count.v = 0u;
    load_camera(P::camera, cam);
    P::materials = bind<P::Material>(s->materials);
    P::vertices = bind<P::Vertex>(s->vertices);
    P::indices = bind<uint32_t>(s->indices);
    P::mesh_infos = bind<P::MeshInfo>(s->meshes);
    if (n_threads == 1) {
        for (uint32_t i = 0; i < n_emit; ++i) P::cs_main(vec3u(i, 0u, 0u));
    } else {
#pragma omp parallel for schedule(dynamic, 1024) num_threads(n_threads > 0 ? n_threads : omp_get_max_threads())
        for (uint32_t i = 0; i < n_emit; ++i) P::cs_main(vec3u(i, 0u, 0u));
    }
    return P::photon_count.v;
}

// Grid pass (build_grid.wgsl main) over the dispatch of 2^20 ids, in id
// order with n_threads = 1, concurrently otherwise (the lists' order then
// varies as on a GPU).  grid_head: 2^22 entries (cleared here to 0xFFFFFFFF
// as renderer/mod.rs:179 does), grid_next: 2^20.
void ref_build_grid(const srt_camera_uniform* cam, srt_photon* photons, uint32_t count, uint32_t* grid_head,
                    uint32_t* grid_next, int n_threads) {
    namespace G = wgsl_build_grid;
    for (uint32_t i = 0; i < kHashSize; ++i) grid_head[i] = 0xFFFFFFFFu;
    G::photons = bind<G::Photon>(photons, kMaxPhotons);
    G::photon_count.v = count;
    G::grid_head = bind<Atomic<uint32_t>>(grid_head, kHashSize);
    G::grid_next = bind<uint32_t>(grid_next, kMaxPhotons);
    load_camera(G::camera, cam);
    if (n_threads == 1) {
        for (uint32_t i = 0; i < kMaxPhotons; ++i) G::cs_main(vec3u(i, 0u, 0u));
    } else {
#pragma omp parallel for schedule(static) num_threads(n_threads > 0 ? n_threads : omp_get_max_threads())
        for (uint32_t i = 0; i < kMaxPhotons; ++i) G::cs_main(vec3u(i, 0u, 0u));
    }
}

// Camera pass (shader.wgsl main) over a w x h target with MAX_DEPTH
// max_depth: reads accum (w*h*4 floats) when the frame count is > 0 and
// writes it; ldr = the rgba8unorm storage texture (w*h*4 bytes).
void ref_camera_pass(ref_scene* s, const srt_camera_uniform* cam, uint32_t w, uint32_t h, uint32_t max_depth,
                     srt_photon* photons, uint32_t* grid_head, uint32_t* grid_next, float* accum, uint8_t* ldr,
                     int n_threads) {
    namespace S = wgsl_shader;
    S::MAX_DEPTH = max_depth;
    S::tlas = s->tlas;
    S::out_tex.w = w;
    S::out_tex.h = h;
    S::out_tex.rgba8 = ldr;
    load_camera(S::camera, cam);
    S::materials = bind<S::Material>(s->materials);
    S::accumulation = bind<vec4f>(reinterpret_cast<vec4f*>(accum), w * h);
    S::vertices = bind<S::Vertex>(s->vertices);
    S::indices = bind<uint32_t>(s->indices);
    S::mesh_infos = bind<S::MeshInfo>(s->meshes);
    S::lights = bind<S::LightInfo>(s->lights);
    S::photons = bind<S::Photon>(photons, kMaxPhotons);
    S::grid_head = bind<uint32_t>(grid_head, kHashSize);
    S::grid_next = bind<uint32_t>(grid_next, kMaxPhotons);
    // invocations write disjoint pixels; ray queries read the scene only
#pragma omp parallel for schedule(dynamic, 1) num_threads(n_threads > 0 ? n_threads : omp_get_max_threads())
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x) S::cs_main(vec3u(x, y, 0u));
}

// The camera ray of each listed pixel as the reference's main computes it:
// the first ray query of the invocation (which is then answered with a miss).
// pix: n (x, y) pairs; out: n x 6 floats (origin, direction).
void ref_camera_rays(const srt_camera_uniform* cam, uint32_t w, uint32_t h, const uint32_t* pix, uint32_t n,
                     float* out) {
    namespace S = wgsl_shader;
    static std::vector<vec4f> accum;
    static std::vector<uint8_t> ldr;
    accum.assign((size_t)w * h, vec4f(0.0f));
    ldr.assign((size_t)w * h * 4, 0);
    acceleration_structure cap;
    cap.trace = trace_capture_cb;
    S::MAX_DEPTH = 1u;
    S::tlas = cap;
    S::out_tex.w = w;
    S::out_tex.h = h;
    S::out_tex.rgba8 = ldr.data();
    load_camera(S::camera, cam);
    S::accumulation = bind<vec4f>(accum);
    for (uint32_t i = 0; i < n; ++i) {
        g_capture = true;
        S::cs_main(vec3u(pix[2 * i], pix[2 * i + 1], 0u));
        const RayDesc& d = g_first;
        float* o = out + 6 * (size_t)i;
        o[0] = d.origin.x;
        o[1] = d.origin.y;
        o[2] = d.origin.z;
        o[3] = d.dir.x;
        o[4] = d.dir.y;
        o[5] = d.dir.z;
    }
}

// The reference's shading functions one at a time, with the op codes and
// record layouts of orc_device_math / srt_test_device_math:
//  0 pcg_hash, 1 sample_cie_xyz, 2 blackbody_radiance (shader.wgsl),
//  3 rgb_to_spectrum_vec4, 4 fresnel_thin_film, 6 sample_bsdf (rng seed in,
//  rng state out), 7 the grid hash of build_grid.wgsl (cell must be 0.02, the
//  shader's CELL_SIZE); and, with no orc_device_math counterpart:
//  102 blackbody_radiance of photon_emit.wgsl, in f32[2] -> out f32[1];
//  109 fresnel_thin_film_1d of photon_emit.wgsl (cos, n1, n2, n3, d, lambda)
//      in f32[6] -> out f32[1];
//  110 reflectance (Schlick, shader.wgsl:264-269) (cos, ior) in f32[2] -> f32[1].
// Returns 1 for an op the reference has no function for.
int ref_device_math(int op, uint32_t n, const void* in, void* out) {
    namespace S = wgsl_shader;
    const float* fi = static_cast<const float*>(in);
    const uint32_t* ui = static_cast<const uint32_t*>(in);
    float* fo = static_cast<float*>(out);
    uint32_t* uo = static_cast<uint32_t*>(out);
    for (uint32_t i = 0; i < n; ++i) {
        switch (op) {
            case 0:
                uo[i] = S::pcg_hash(ui[i]);
                break;
            case 1: {
                const vec3f c = S::sample_cie_xyz(fi[i]);
                fo[3 * i] = c.x;
                fo[3 * i + 1] = c.y;
                fo[3 * i + 2] = c.z;
            } break;
            case 2:
                fo[i] = S::blackbody_radiance(fi[2 * i], fi[2 * i + 1]);
                break;
            case 102:
                fo[i] = wgsl_photon_emit::blackbody_radiance(fi[2 * i], fi[2 * i + 1]);
                break;
            case 3: {
                const float* a = fi + 7 * i;
                const vec4f r = S::rgb_to_spectrum_vec4(vec3f(a[0], a[1], a[2]), vec4f(a[3], a[4], a[5], a[6]));
                std::memcpy(fo + 4 * i, &r, 16);
            } break;
            case 4: {
                const float* a = fi + 9 * i;
                const vec4f r = S::fresnel_thin_film(a[0], a[1], a[2], a[3], a[4], vec4f(a[5], a[6], a[7], a[8]));
                std::memcpy(fo + 4 * i, &r, 16);
            } break;
            case 109: {
                const float* a = fi + 6 * i;
                fo[i] = wgsl_photon_emit::fresnel_thin_film_1d(a[0], a[1], a[2], a[3], a[4], a[5]);
            } break;
            case 110:
                fo[i] = S::reflectance(fi[2 * i], fi[2 * i + 1]);
                break;
            case 6: {
                const float* a = fi + 24 * i;
                S::Material m;
                std::memcpy(static_cast<void*>(&m), a + 6, 32);
                uint32_t seed;
                std::memcpy(&seed, a + 23, 4);
                S::rng_seed = seed;
                const S::ScatterRecord r =
                    S::sample_bsdf(vec3f(a[0], a[1], a[2]), vec3f(a[3], a[4], a[5]), m, a[14] != 0.0f,
                                   vec4f(a[15], a[16], a[17], a[18]), vec4f(a[19], a[20], a[21], a[22]));
                float* o = fo + 10 * i;
                o[0] = r.scatter_dir.x;
                o[1] = r.scatter_dir.y;
                o[2] = r.scatter_dir.z;
                std::memcpy(o + 3, &r.attenuation, 16);
                o[7] = r.absorbed ? 1.0f : 0.0f;
                std::memcpy(o + 8, &S::rng_seed, 4);
                o[9] = 0.0f;
            } break;
            case 7: {
                const float* a = fi + 5 * i;
                uint32_t frame;
                std::memcpy(&frame, a + 3, 4);
                if (a[4] != wgsl_build_grid::CELL_SIZE) return 1;
                wgsl_build_grid::camera.frame_count = frame;
                uo[i] = wgsl_build_grid::hash_position(vec3f(a[0], a[1], a[2]));
            } break;
            default:
                return 1;
        }
    }
    return 0;
}

}  // extern "C"
