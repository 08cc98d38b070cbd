// capi.cu — implementation of the C ABI declared in include/srt.h.
//
// Host side of the path: the CUDA context that replaces WgpuContext
// (src/wgpu_ctx.rs), scene upload + GPU BVH build that replace
// SceneBuilder::build (src/scene/builder.rs:131-266), and the renderer that
// replaces Renderer::new / render (src/renderer/mod.rs:45-207) and the
// engine's screenshot readback (src/engine.rs:191-244).
#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "bvh_build.h"
#include "host_scene.h"
#include "radix_sort.cuh"
#include "render_kernels.h"
#include "umma.cuh"

using namespace srt;

namespace {
std::string g_last_create_error;

bool env_fault(const char* what) {
    // Host-side fault injection for the error paths: SRT_FAULT=alloc|launch
    const char* f = std::getenv("SRT_FAULT");
    return f && std::strcmp(f, what) == 0;
}
}  // namespace

struct srt_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int sm_count = 0;
    std::string err;
    uint32_t* d_err = nullptr;  // device error word for batch entry points
    // Scenes, renderers and batches created on this context that are still
    // alive; srt_ctx_destroy defers the release until the last one is gone,
    // so handles may be destroyed in any order (e.g. by a garbage collector).
    int children = 0;
    bool closing = false;
    int bvh_builder = 0;  // SRT_BVH_* for the scenes built next
    int bvh_width = 8;    // children per BVH node for the scenes built next
    uint32_t bvh_leaf = 2;  // triangles of the largest BVH leaf for the scenes built next
};

namespace {
void ctx_free(srt_ctx* c) {
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    cudaFree(c->d_err);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
}
void ctx_retain(srt_ctx* c) { ++c->children; }
void ctx_release(srt_ctx* c) {
    if (--c->children == 0 && c->closing) ctx_free(c);
}
}  // namespace

namespace {

srt_status fail(srt_ctx* c, srt_status s, const std::string& msg) {
    if (c) c->err = msg;
    return s;
}
srt_status cuda_fail(srt_ctx* c, cudaError_t e, const char* where) {
    return fail(c, e == cudaErrorMemoryAllocation ? SRT_ERR_OOM : SRT_ERR_CUDA,
                std::string(where) + ": " + cudaGetErrorString(e));
}

#define CUDA_TRY(ctx, expr)                                \
    do {                                                   \
        cudaError_t _e = (expr);                           \
        if (_e != cudaSuccess) return cuda_fail(ctx, _e, #expr); \
    } while (0)

template <typename T>
cudaError_t dev_alloc(T** p, size_t count) {
    if (env_fault("alloc")) return cudaErrorMemoryAllocation;
    return cudaMalloc((void**)p, sizeof(T) * (count ? count : 1));
}

// Reads and clears a device error word.
srt_status check_device_error(srt_ctx* c, uint32_t* d_err) {
    uint32_t h = 0;
    CUDA_TRY(c, cudaMemcpyAsync(&h, d_err, 4, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    if (h != 0u) {
        CUDA_TRY(c, cudaMemsetAsync(d_err, 0, 4, c->stream));
        char buf[96];
        if (h & ERR_MMA_TIMEOUT) {  // a bounded wait gave up; the context stays usable
            std::snprintf(buf, sizeof buf, "a bounded device wait gave up (error word 0x%x)", h);
            return fail(c, SRT_ERR_TIMEOUT, buf);
        }
        std::snprintf(buf, sizeof buf, "device check failed (error word 0x%x)", h);
        return fail(c, SRT_ERR_DEVICE_ASSERT, buf);
    }
    return SRT_OK;
}

}  // namespace

// ====================================================================== context
extern "C" {

uint32_t srt_abi_version(void) { return SRT_ABI_VERSION; }

srt_status srt_ctx_create(int device, void* stream, srt_ctx** out) {
    if (!out) return SRT_ERR_INVALID_ARG;
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        g_last_create_error = "no CUDA device";
        return SRT_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) {
        g_last_create_error = "device index out of range";
        return SRT_ERR_INVALID_ARG;
    }
    std::unique_ptr<srt_ctx> c(new (std::nothrow) srt_ctx());
    if (!c) return SRT_ERR_OOM;
    c->device = device;
    if ((e = cudaSetDevice(device)) != cudaSuccess) {
        g_last_create_error = cudaGetErrorString(e);
        return SRT_ERR_CUDA;
    }
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (stream) {
        c->stream = (cudaStream_t)stream;
    } else {
        if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) {
            g_last_create_error = cudaGetErrorString(e);
            return SRT_ERR_CUDA;
        }
        c->own_stream = true;
    }
    if ((e = dev_alloc(&c->d_err, 1)) != cudaSuccess || (e = cudaMemset(c->d_err, 0, 4)) != cudaSuccess) {
        g_last_create_error = cudaGetErrorString(e);
        if (c->own_stream) cudaStreamDestroy(c->stream);
        return e == cudaErrorMemoryAllocation ? SRT_ERR_OOM : SRT_ERR_CUDA;
    }
    *out = c.release();
    return SRT_OK;
}

srt_status srt_ctx_destroy(srt_ctx* c) {
    if (!c || c->closing) return SRT_ERR_INVALID_ARG;
    if (c->children > 0) {
        c->closing = true;  // released with its last scene, renderer or batch
        cudaSetDevice(c->device);
        cudaStreamSynchronize(c->stream);
        return SRT_OK;
    }
    ctx_free(c);
    return SRT_OK;
}

srt_status srt_ctx_set_bvh_builder(srt_ctx* c, int builder) {
    if (!c || (builder != SRT_BVH_SAH && builder != SRT_BVH_LBVH)) return SRT_ERR_INVALID_ARG;
    c->bvh_builder = builder;
    return SRT_OK;
}

srt_status srt_ctx_set_bvh_width(srt_ctx* c, uint32_t width) {
    if (!c || width < 2 || width > 8) return SRT_ERR_INVALID_ARG;
    c->bvh_width = (int)width;
    return SRT_OK;
}

srt_status srt_ctx_set_bvh_leaf_size(srt_ctx* c, uint32_t max_triangles) {
    if (!c || max_triangles < 1 || max_triangles > 3) return SRT_ERR_INVALID_ARG;
    c->bvh_leaf = max_triangles;
    return SRT_OK;
}

const char* srt_get_error_string(const srt_ctx* c) { return c ? c->err.c_str() : g_last_create_error.c_str(); }
void* srt_ctx_stream(srt_ctx* c) { return c ? (void*)c->stream : nullptr; }
int srt_ctx_sm_count(const srt_ctx* c) { return c ? c->sm_count : 0; }

srt_status srt_ctx_synchronize(srt_ctx* c) {
    if (!c) return SRT_ERR_INVALID_ARG;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    CUDA_TRY(c, cudaGetLastError());
    return SRT_OK;
}

// ====================================================================== scene builder (host)
srt_status srt_scene_builder_create(srt_scene_builder** out) {
    if (!out) return SRT_ERR_INVALID_ARG;
    *out = new (std::nothrow) srt_scene_builder();
    return *out ? SRT_OK : SRT_ERR_OOM;
}
srt_status srt_scene_builder_destroy(srt_scene_builder* b) {
    delete b;
    return SRT_OK;
}
uint32_t srt_scene_builder_add_material(srt_scene_builder* b, const srt_material* m) {
    return (b && m) ? b->add_material(*m) : 0xFFFFFFFFu;
}
uint32_t srt_scene_builder_add_mesh(srt_scene_builder* b, const srt_vertex* v, uint32_t nv, const uint32_t* idx,
                                    uint32_t ni) {
    if (!b || (!v && nv) || (!idx && ni) || ni % 3u) return 0xFFFFFFFFu;
    for (uint32_t i = 0; i < ni; ++i)
        if (idx[i] >= nv) return 0xFFFFFFFFu;
    return b->add_mesh(v, nv, idx, ni);
}
srt_status srt_scene_builder_add_instance(srt_scene_builder* b, uint32_t mesh, uint32_t mat, const float t[16]) {
    if (!b || !t || mesh >= b->mesh_infos.size()) return SRT_ERR_INVALID_ARG;
    Mat4 m;
    std::memcpy(m.m, t, 64);
    b->add_instance(mesh, mat, m);
    return SRT_OK;
}
srt_status srt_scene_builder_add_light_instance(srt_scene_builder* b, uint32_t mesh, uint32_t mat, const float t[16],
                                                const float params[4]) {
    if (!b || !t || !params || mesh >= b->mesh_infos.size()) return SRT_ERR_INVALID_ARG;
    Mat4 m;
    std::memcpy(m.m, t, 64);
    b->add_light_instance(mesh, mat, m, params);
    return SRT_OK;
}
srt_status srt_scene_builder_arrays(const srt_scene_builder* b, srt_scene_arrays* o) {
    if (!b || !o) return SRT_ERR_INVALID_ARG;
    o->vertices = b->vertices.data();
    o->n_vertices = (uint32_t)b->vertices.size();
    o->indices = b->indices.data();
    o->n_indices = (uint32_t)b->indices.size();
    o->mesh_infos = b->mesh_infos.data();
    o->n_meshes = (uint32_t)b->mesh_infos.size();
    o->materials = b->materials.data();
    o->n_materials = (uint32_t)b->materials.size();
    o->instances = b->instances.data();
    o->n_instances = (uint32_t)b->instances.size();
    o->lights = b->lights.data();
    o->n_lights = (uint32_t)b->lights.size();
    return SRT_OK;
}
srt_status srt_scene_builder_add_preset(srt_scene_builder* b, int preset, uint32_t seed, float camera_out[5]) {
    if (!b) return SRT_ERR_INVALID_ARG;
    float cam[5];
    if (!preset_fill(b, preset, seed, cam)) return SRT_ERR_INVALID_ARG;
    if (camera_out) std::memcpy(camera_out, cam, sizeof cam);
    return SRT_OK;
}

static srt_status geom_out(const std::vector<srt_vertex>& v, const std::vector<uint32_t>& i, srt_vertex* vo,
                           uint32_t* nv, uint32_t* io, uint32_t* ni) {
    if (!nv || !ni) return SRT_ERR_INVALID_ARG;
    if (vo) {
        if (*nv < v.size()) return SRT_ERR_INVALID_ARG;
        std::memcpy(vo, v.data(), v.size() * sizeof(srt_vertex));
    }
    if (io) {
        if (*ni < i.size()) return SRT_ERR_INVALID_ARG;
        std::memcpy(io, i.data(), i.size() * 4);
    }
    *nv = (uint32_t)v.size();
    *ni = (uint32_t)i.size();
    return SRT_OK;
}
srt_status srt_geometry_plane(srt_vertex* v, uint32_t* nv, uint32_t* i, uint32_t* ni) {
    std::vector<srt_vertex> vv;
    std::vector<uint32_t> ii;
    geom_plane(vv, ii);
    return geom_out(vv, ii, v, nv, i, ni);
}
srt_status srt_geometry_cube(srt_vertex* v, uint32_t* nv, uint32_t* i, uint32_t* ni) {
    std::vector<srt_vertex> vv;
    std::vector<uint32_t> ii;
    geom_cube(vv, ii);
    return geom_out(vv, ii, v, nv, i, ni);
}
srt_status srt_geometry_icosphere(uint32_t sub, srt_vertex* v, uint32_t* nv, uint32_t* i, uint32_t* ni) {
    if (sub > 10) return SRT_ERR_INVALID_ARG;
    std::vector<srt_vertex> vv;
    std::vector<uint32_t> ii;
    geom_icosphere(sub, vv, ii);
    return geom_out(vv, ii, v, nv, i, ni);
}
srt_status srt_geometry_uv_sphere(uint32_t slices, uint32_t stacks, srt_vertex* v, uint32_t* nv, uint32_t* i,
                                  uint32_t* ni) {
    if (slices < 3 || stacks < 2 || slices > 4096 || stacks > 4096) return SRT_ERR_INVALID_ARG;
    std::vector<srt_vertex> vv;
    std::vector<uint32_t> ii;
    geom_uv_sphere(slices, stacks, vv, ii);
    return geom_out(vv, ii, v, nv, i, ni);
}

srt_status srt_camera_build_uniform(const float position[3], float yaw, float pitch, float aspect, uint32_t frame,
                                    srt_camera_uniform* out) {
    if (!position || !out || !(aspect > 0.0f)) return SRT_ERR_INVALID_ARG;
    camera_build_uniform(position, yaw, pitch, aspect, frame, out);
    return SRT_OK;
}

}  // extern "C"

// ====================================================================== scene (device)
struct srt_scene {
    srt_ctx* ctx = nullptr;
    float4* vtx = nullptr;
    uint32_t* idx = nullptr;
    uint4* mesh_infos = nullptr;
    float4* materials = nullptr;
    float4* lights = nullptr;
    InstDev* inst = nullptr;
    InstFwd* fwd = nullptr;
    BvhOutputs bvh{};
    DevScene dev{};
    uint64_t n_tris = 0;
    uint32_t n_lights = 0;
    // instance updates: host copies of the instances, light instances (device),
    // refit scratch
    std::vector<srt_instance> h_inst;
    std::vector<uint32_t> h_mesh_tris;
    std::vector<InstDev> h_instdev;
    LightInst* light_insts = nullptr;
    uint32_t n_light_insts = 0;
    uint8_t* moved = nullptr;
    float4* refit_aux = nullptr;
    uint32_t* refit_err = nullptr;
    // tree rebuilds: renderers compare gen with the one they captured
    uint32_t gen = 0;
    // any change of the geometry (instance updates, rebuilds): a photon map
    // built ahead of a frame is stale after it
    uint32_t version = 0;
    int builder = BVH_BUILDER_SAH;
    int width = 8;
    uint32_t leaf = 2;  // triangles of the largest leaf (rebuilds keep it)
    uint32_t n_inst = 0;
    ~srt_scene() {
        cudaFree(light_insts);
        cudaFree(moved);
        cudaFree(refit_aux);
        cudaFree(refit_err);
        cudaFree(vtx);
        cudaFree(idx);
        cudaFree(mesh_infos);
        cudaFree(materials);
        cudaFree(lights);
        cudaFree(inst);
        cudaFree(fwd);
        cudaFree(bvh.nodes);
        cudaFree(bvh.tris);
        cudaFree(bvh.tri_inst);
    }
};

namespace {
template <typename T>
cudaError_t upload(T** dst, const void* src, size_t bytes, size_t alloc_bytes, cudaStream_t st) {
    cudaError_t e = dev_alloc((char**)dst, alloc_bytes ? alloc_bytes : 16);
    if (e != cudaSuccess) return e;
    if (bytes) e = cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, st);
    return e;
}
}  // namespace

namespace {
// World-to-object rows (FP64 inverse of the 3x3 part) and object-to-world
// rows of one instance; false when the transform is singular.
bool instance_rows(const srt_instance& in, InstDev* d, InstFwd* f) {
    const float* M = in.transform;
    double r[9] = {M[0], M[4], M[8], M[1], M[5], M[9], M[2], M[6], M[10]};  // row-major 3x3
    double det = r[0] * (r[4] * r[8] - r[5] * r[7]) - r[1] * (r[3] * r[8] - r[5] * r[6]) +
                 r[2] * (r[3] * r[7] - r[4] * r[6]);
    if (!(std::fabs(det) > 0.0) || !std::isfinite(det)) return false;
    for (int k = 12; k < 15; ++k)
        if (!std::isfinite(M[k])) return false;
    double iv[9] = {(r[4] * r[8] - r[5] * r[7]) / det, (r[2] * r[7] - r[1] * r[8]) / det,
                    (r[1] * r[5] - r[2] * r[4]) / det, (r[5] * r[6] - r[3] * r[8]) / det,
                    (r[0] * r[8] - r[2] * r[6]) / det, (r[2] * r[3] - r[0] * r[5]) / det,
                    (r[3] * r[7] - r[4] * r[6]) / det, (r[1] * r[6] - r[0] * r[7]) / det,
                    (r[0] * r[4] - r[1] * r[3]) / det};
    d->w2o0 = make_float4((float)iv[0], (float)iv[1], (float)iv[2], 0.f);
    d->w2o1 = make_float4((float)iv[3], (float)iv[4], (float)iv[5], 0.f);
    d->w2o2 = make_float4((float)iv[6], (float)iv[7], (float)iv[8], 0.f);
    f->r0 = make_float4(M[0], M[4], M[8], M[12]);
    f->r1 = make_float4(M[1], M[5], M[9], M[13]);
    f->r2 = make_float4(M[2], M[6], M[10], M[14]);
    return true;
}

srt_status scene_build_impl(srt_ctx* c, const srt_scene_arrays* a,
                            const std::vector<srt_light_instance_rec>* light_instances, srt_scene** out);
}  // namespace

extern "C" srt_status srt_scene_build(srt_ctx* c, const srt_scene_arrays* a, srt_scene** out) {
    return scene_build_impl(c, a, nullptr, out);
}

namespace {
srt_status scene_build_impl(srt_ctx* c, const srt_scene_arrays* a,
                            const std::vector<srt_light_instance_rec>* light_instances, srt_scene** out) {
    if (!c || !a || !out) return SRT_ERR_INVALID_ARG;
    *out = nullptr;
    cudaSetDevice(c->device);
    // ---- validation on the host: every device index is checked here
    if ((a->n_vertices && !a->vertices) || (a->n_indices && !a->indices) || (a->n_meshes && !a->mesh_infos) ||
        (a->n_materials && !a->materials) || (a->n_instances && !a->instances) || (a->n_lights && !a->lights))
        return fail(c, SRT_ERR_INVALID_ARG, "null array with nonzero count");
    std::vector<uint32_t> mesh_tris(a->n_meshes);
    for (uint32_t m = 0; m < a->n_meshes; ++m) {
        uint32_t io = a->mesh_infos[m].index_offset;
        uint32_t end = m + 1 < a->n_meshes ? a->mesh_infos[m + 1].index_offset : a->n_indices;
        if (io > end || end > a->n_indices || (end - io) % 3u)
            return fail(c, SRT_ERR_INVALID_ARG, "mesh index ranges must be consecutive multiples of 3");
        mesh_tris[m] = (end - io) / 3u;
        uint32_t vend = m + 1 < a->n_meshes ? a->mesh_infos[m + 1].vertex_offset : a->n_vertices;
        uint32_t vo = a->mesh_infos[m].vertex_offset;
        for (uint32_t i = io; i < end; ++i)
            if ((uint64_t)a->indices[i] + vo >= a->n_vertices || a->indices[i] + vo >= vend)
                return fail(c, SRT_ERR_INVALID_ARG, "vertex index out of range");
    }
    std::vector<InstDev> inst(a->n_instances);
    std::vector<InstFwd> fwd(a->n_instances);
    uint64_t total = 0;
    for (uint32_t i = 0; i < a->n_instances; ++i) {
        const srt_instance& in = a->instances[i];
        if (in.mesh_id >= a->n_meshes || in.mat_id >= a->n_materials)
            return fail(c, SRT_ERR_INVALID_ARG, "instance mesh/material id out of range");
        InstDev d{};
        if (!instance_rows(in, &d, &fwd[i])) return fail(c, SRT_ERR_INVALID_ARG, "instance transform is singular");
        d.mesh_id = in.mesh_id;
        d.mat_id = in.mat_id;
        d.tri_offset = (uint32_t)total;
        d.tri_count = mesh_tris[in.mesh_id];
        inst[i] = d;
        total += mesh_tris[in.mesh_id];
    }
    if (total >= 0x7FFFFFFFull) return fail(c, SRT_ERR_INVALID_ARG, "too many triangles");
    std::unique_ptr<srt_scene> s(new (std::nothrow) srt_scene());
    if (!s) return SRT_ERR_OOM;
    s->ctx = c;
    cudaStream_t st = c->stream;
    CUDA_TRY(c, upload(&s->vtx, a->vertices, sizeof(srt_vertex) * a->n_vertices, sizeof(srt_vertex) * a->n_vertices, st));
    CUDA_TRY(c, upload(&s->idx, a->indices, 4ull * a->n_indices, 4ull * a->n_indices, st));
    CUDA_TRY(c, upload(&s->mesh_infos, a->mesh_infos, 16ull * a->n_meshes, 16ull * a->n_meshes, st));
    CUDA_TRY(c, upload(&s->materials, a->materials, 32ull * a->n_materials, 32ull * a->n_materials, st));
    CUDA_TRY(c, upload(&s->lights, a->lights, 64ull * a->n_lights, 64ull * a->n_lights, st));
    CUDA_TRY(c, upload(&s->inst, inst.data(), sizeof(InstDev) * inst.size(), sizeof(InstDev) * inst.size(), st));
    CUDA_TRY(c, upload(&s->fwd, fwd.data(), sizeof(InstFwd) * fwd.size(), sizeof(InstFwd) * fwd.size(), st));
    BvhInputs bi{s->vtx, s->idx, s->mesh_infos, s->inst, s->fwd, a->n_instances, (uint32_t)total,
                 c->bvh_builder == SRT_BVH_LBVH ? BVH_BUILDER_LBVH : BVH_BUILDER_SAH, c->bvh_width, c->bvh_leaf};
    s->builder = bi.builder;
    s->width = bi.width;
    s->leaf = bi.leaf_max;
    s->n_inst = a->n_instances;
    std::string msg;
    cudaError_t e = build_bvh8(bi, st, &s->bvh, &msg);
    if (e != cudaSuccess) return fail(c, e == cudaErrorMemoryAllocation ? SRT_ERR_OOM : SRT_ERR_CUDA, "BVH build: " + msg);
    if (s->bvh.depth > (uint32_t)TRAV_STACK)
        return fail(c, SRT_ERR_UNSUPPORTED, "BVH deeper than the traversal stack");
    CUDA_TRY(c, cudaStreamSynchronize(st));
    s->n_tris = total;
    s->n_lights = a->n_lights;
    DevScene& d = s->dev;
    d.vtx = s->vtx;
    d.indices = s->idx;
    d.mesh_infos = s->mesh_infos;
    d.materials = s->materials;
    d.lights = s->lights;
    d.n_lights = a->n_lights;
    d.inst = s->inst;
    d.tri_inst = s->bvh.tri_inst;
    d.nodes = s->bvh.nodes;
    d.tris = s->bvh.tris;
    d.n_nodes = s->bvh.n_nodes;
    d.n_tris = (uint32_t)total;
    d.depth = s->bvh.depth;
    {
        // world bounds: each instance's object-space vertex box, transformed
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (uint32_t i = 0; i < a->n_instances; ++i) {
            const srt_instance& in = a->instances[i];
            uint32_t m = in.mesh_id;
            uint32_t vb = a->mesh_infos[m].vertex_offset;
            uint32_t ve = m + 1 < a->n_meshes ? a->mesh_infos[m + 1].vertex_offset : a->n_vertices;
            double olo[3] = {1e300, 1e300, 1e300}, ohi[3] = {-1e300, -1e300, -1e300};
            for (uint32_t v = vb; v < ve; ++v)
                for (int k = 0; k < 3; ++k) {
                    olo[k] = std::min(olo[k], (double)a->vertices[v].pos[k]);
                    ohi[k] = std::max(ohi[k], (double)a->vertices[v].pos[k]);
                }
            if (olo[0] > ohi[0]) continue;
            const float* M = in.transform;
            for (int c8 = 0; c8 < 8; ++c8) {
                double p[3] = {(c8 & 1) ? ohi[0] : olo[0], (c8 & 2) ? ohi[1] : olo[1], (c8 & 4) ? ohi[2] : olo[2]};
                for (int r = 0; r < 3; ++r) {
                    double w = M[r] * p[0] + M[4 + r] * p[1] + M[8 + r] * p[2] + M[12 + r];
                    lo[r] = std::min(lo[r], w);
                    hi[r] = std::max(hi[r], w);
                }
            }
        }
        if (lo[0] > hi[0]) lo[0] = lo[1] = lo[2] = hi[0] = hi[1] = hi[2] = 0.0;
        float inv[3];
        for (int k = 0; k < 3; ++k) inv[k] = (float)(1.0 / std::max(hi[k] - lo[k], 1e-6));
        d.bmin = make_float4((float)lo[0], (float)lo[1], (float)lo[2], 0.f);
        d.binv = make_float4(inv[0], inv[1], inv[2], 0.f);
    }
    s->h_inst.assign(a->instances, a->instances + a->n_instances);
    s->h_mesh_tris = mesh_tris;
    s->h_instdev = inst;
    if (light_instances && !light_instances->empty()) {
        // scene-side GPU ingestion: the light instances' triangles are
        // expanded to world space on the device (builder.rs:101-129)
        std::vector<LightInst> li;
        for (const srt_light_instance_rec& r : *light_instances) {
            if (r.instance >= a->n_instances || (uint64_t)r.first_light + r.count > a->n_lights ||
                r.count != mesh_tris[a->instances[r.instance].mesh_id])
                return fail(c, SRT_ERR_INVALID_ARG, "light instance record out of range");
            LightInst L{r.instance, r.first_light, r.count, 0u,
                        make_float4(r.params[0], r.params[1], r.params[2], r.params[3])};
            li.push_back(L);
        }
        CUDA_TRY(c, upload(&s->light_insts, li.data(), sizeof(LightInst) * li.size(), sizeof(LightInst) * li.size(), st));
        s->n_light_insts = (uint32_t)li.size();
        launch_expand_lights(s->light_insts, s->n_light_insts, nullptr, s->vtx, s->idx, s->mesh_infos, s->inst, s->fwd,
                             s->lights, st);
        CUDA_TRY(c, cudaGetLastError());
        CUDA_TRY(c, cudaStreamSynchronize(st));
    }
    ctx_retain(c);
    *out = s.release();
    return SRT_OK;
}
}  // namespace

extern "C" srt_status srt_scene_builder_build(srt_ctx* c, const srt_scene_builder* b, srt_scene** out) {
    srt_scene_arrays a;
    srt_status st = srt_scene_builder_arrays(b, &a);
    if (st != SRT_OK) return st;
    return scene_build_impl(c, &a, &b->light_instances, out);
}

extern "C" srt_status srt_scene_update_instances(srt_scene* s, const uint32_t* ids, const float* transforms,
                                                 uint32_t n) {
    if (!s || (n && (!ids || !transforms))) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = s->ctx;
    cudaSetDevice(c->device);
    cudaStream_t st = c->stream;
    const uint32_t ni = (uint32_t)s->h_inst.size();
    if (n == 0 || ni == 0) return SRT_OK;
    s->version += 1;
    std::vector<InstDev> nd(n);
    std::vector<InstFwd> nf(n);
    for (uint32_t k = 0; k < n; ++k) {
        if (ids[k] >= ni) return fail(c, SRT_ERR_INVALID_ARG, "instance id out of range");
        srt_instance in = s->h_inst[ids[k]];
        std::memcpy(in.transform, transforms + 16ull * k, 64);
        nd[k] = s->h_instdev[ids[k]];
        if (!instance_rows(in, &nd[k], &nf[k])) return fail(c, SRT_ERR_INVALID_ARG, "instance transform is singular");
    }
    if (!s->moved) {
        CUDA_TRY(c, dev_alloc(&s->moved, ni));
        CUDA_TRY(c, dev_alloc(&s->refit_aux, 2ull * std::max(1u, s->bvh.n_nodes)));
        CUDA_TRY(c, dev_alloc(&s->refit_err, 1));
    }
    std::vector<uint8_t> moved(ni, 0);
    CUDA_TRY(c, cudaStreamSynchronize(st));  // frames in flight read the instances
    for (uint32_t k = 0; k < n; ++k) {
        uint32_t i = ids[k];
        moved[i] = 1;
        std::memcpy(s->h_inst[i].transform, transforms + 16ull * k, 64);
        s->h_instdev[i] = nd[k];
        CUDA_TRY(c, cudaMemcpyAsync(s->inst + i, &nd[k], sizeof(InstDev), cudaMemcpyHostToDevice, st));
        CUDA_TRY(c, cudaMemcpyAsync(s->fwd + i, &nf[k], sizeof(InstFwd), cudaMemcpyHostToDevice, st));
    }
    CUDA_TRY(c, cudaMemcpyAsync(s->moved, moved.data(), ni, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemsetAsync(s->refit_err, 0, 4, st));
    launch_update_slots(s->bvh.tris, (uint32_t)s->n_tris, s->bvh.tri_inst, s->moved, s->vtx, s->idx, s->mesh_infos,
                        s->inst, s->fwd, st);
    launch_expand_lights(s->light_insts, s->n_light_insts, s->moved, s->vtx, s->idx, s->mesh_infos, s->inst, s->fwd,
                         s->lights, st);
    refit_bvh8(s->bvh.nodes, s->bvh.tris, s->bvh, s->refit_aux, s->refit_err, st);
    CUDA_TRY(c, cudaGetLastError());
    uint32_t herr = 0;
    CUDA_TRY(c, cudaMemcpyAsync(&herr, s->refit_err, 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaStreamSynchronize(st));
    if (herr) return fail(c, SRT_ERR_DEVICE_ASSERT, "BVH refit could not quantise a node");
    return SRT_OK;
}

extern "C" srt_status srt_scene_read_lights(srt_scene* s, srt_light* out, uint32_t capacity, uint32_t* count) {
    if (!s || !count) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = s->ctx;
    cudaSetDevice(c->device);
    *count = s->n_lights;
    uint32_t m = std::min(capacity, s->n_lights);
    if (out && m) {
        CUDA_TRY(c, cudaMemcpyAsync(out, s->lights, 64ull * m, cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    }
    return SRT_OK;
}

extern "C" srt_status srt_scene_read_bvh(srt_scene* s, void* nodes, uint64_t node_bytes, void* tris,
                                         uint64_t tri_bytes) {
    if (!s) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = s->ctx;
    cudaSetDevice(c->device);
    if (nodes && node_bytes) {
        if (node_bytes > 80ull * s->bvh.n_nodes) return SRT_ERR_INVALID_ARG;
        CUDA_TRY(c, cudaMemcpyAsync(nodes, s->bvh.nodes, node_bytes, cudaMemcpyDeviceToHost, c->stream));
    }
    if (tris && tri_bytes) {
        if (tri_bytes > 48ull * s->n_tris) return SRT_ERR_INVALID_ARG;
        CUDA_TRY(c, cudaMemcpyAsync(tris, s->bvh.tris, tri_bytes, cudaMemcpyDeviceToHost, c->stream));
    }
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SRT_OK;
}

extern "C" srt_status srt_scene_destroy(srt_scene* s) {
    if (!s) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = s->ctx;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    delete s;
    ctx_release(c);
    return SRT_OK;
}

extern "C" srt_status srt_scene_info(const srt_scene* s, uint64_t* n_tris, uint64_t* n_nodes, uint32_t* depth) {
    if (!s) return SRT_ERR_INVALID_ARG;
    if (n_tris) *n_tris = s->n_tris;
    if (n_nodes) *n_nodes = s->bvh.n_nodes;
    if (depth) *depth = s->bvh.depth;
    return SRT_OK;
}

extern "C" srt_status srt_scene_rebuild_bvh(srt_scene* s, uint32_t width) {
    if (!s || width < 2 || width > 8) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = s->ctx;
    cudaSetDevice(c->device);
    cudaStream_t st = c->stream;
    CUDA_TRY(c, cudaDeviceSynchronize());  // no frame of any renderer still reads the old tree
    BvhInputs bi{s->vtx, s->idx, s->mesh_infos, s->inst, s->fwd, s->n_inst, (uint32_t)s->n_tris, s->builder,
                 (int)width, s->leaf};
    BvhOutputs nb{};
    std::string msg;
    cudaError_t e = build_bvh8(bi, st, &nb, &msg);
    if (e == cudaSuccess && nb.depth > (uint32_t)TRAV_STACK) {
        e = cudaErrorInvalidValue;
        msg = "BVH deeper than the traversal stack";
    }
    if (e != cudaSuccess) {
        cudaFree(nb.nodes);
        cudaFree(nb.tris);
        cudaFree(nb.tri_inst);
        return fail(c, e == cudaErrorMemoryAllocation ? SRT_ERR_OOM : SRT_ERR_CUDA, "BVH rebuild: " + msg);
    }
    cudaFree(s->bvh.nodes);
    cudaFree(s->bvh.tris);
    cudaFree(s->bvh.tri_inst);
    s->bvh = nb;
    // refit scratch is sized by the node count: allocated again on the next update
    cudaFree(s->moved);
    cudaFree(s->refit_aux);
    cudaFree(s->refit_err);
    s->moved = nullptr;
    s->refit_aux = nullptr;
    s->refit_err = nullptr;
    s->width = (int)width;
    DevScene& d = s->dev;
    d.tri_inst = s->bvh.tri_inst;
    d.nodes = s->bvh.nodes;
    d.tris = s->bvh.tris;
    d.n_nodes = s->bvh.n_nodes;
    d.depth = s->bvh.depth;
    s->gen += 1;
    s->version += 1;
    return SRT_OK;
}

extern "C" srt_status srt_scene_bvh_width(const srt_scene* s, uint32_t* width) {
    if (!s || !width) return SRT_ERR_INVALID_ARG;
    *width = (uint32_t)s->width;
    return SRT_OK;
}

// ====================================================================== renderer
// The tail kernel (launch_tail) follows each remaining path through its
// last bounces in one launch, one thread per path at a time: it pays once
// the live paths fit in about one wave of it, and costs where many long paths
// remain (1080p: config 2 from bounce 5, 118k paths, 10.76 vs 11.04 ms per
// frame; the caustic-slab scene from bounce 5, 202k paths, 7.05 vs 5.93 ms,
// from bounce 7, 69k paths, 5.92 ms).  SRT_TAIL_AUTO (the default) starts it
// at the first bounce whose live paths in the renderer's first frame number
// at most SRT_TAIL_WAVES waves of the tail kernel's resident threads.
#ifndef SRT_TAIL_WAVES
#define SRT_TAIL_WAVES 1.0
#endif
// Guided bounces by default: the first eight.  A guiding renderer's
// automatic tail starts after them (the tail kernel samples cosine lobes).
// The caustic-slab scene at 1080p: relMSE at equal time 0.0500 with bounces
// 0..4 guided, 0.0487 with 0..7, 0.0497 with all; frame 6.59 ms with 0..7
// and the tail from bounce 8, 6.80 ms with all bounces guided.  The number
// is fixed rather than taken from the automatic tail because it changes the
// estimator: a frame's image must not depend on when a read-back landed.
#ifndef SRT_GUIDE_BOUNCES_DEFAULT
#define SRT_GUIDE_BOUNCES_DEFAULT 8u
#endif
// Frames enqueue independent stages on two branches (srt_renderer::record_overlapped).
#ifndef SRT_FRAME_OVERLAP
#define SRT_FRAME_OVERLAP 1
#endif
// A frame builds the next frame's photon map beside its own camera paths
// (srt_renderer::record_overlapped with a photon set).
#ifndef SRT_PHOTON_PIPELINE
#define SRT_PHOTON_PIPELINE 1
#endif

struct srt_renderer {
    srt_ctx* ctx = nullptr;
    srt_scene* scene = nullptr;
    uint32_t scene_gen = 0;  // scene->gen when args.scene was taken

    // After a tree rebuild of the scene: new tree pointers, a new capture.
    void refresh_scene() {
        if (scene_gen == scene->gen) return;
        scene_gen = scene->gen;
        args.scene = scene->dev;
        args_gen += 1;
        drop_graph();
    }
    uint32_t w = 0, h = 0;
    srt_params p{};
    FrameArgs args{};
    srt_camera_uniform* cam_dev = nullptr;
    srt_camera_uniform* cam_ring = nullptr;  // pinned staging
    cudaEvent_t ring_ev[4] = {};
    int ring_i = 0;
    FrameCounters* counters = nullptr;
    DevStats* stats = nullptr;
    uint32_t* err = nullptr;
    PathBuffers pb{};
    PhotonBuffers ph{};
    float4* accum = nullptr;
    double4* accum64 = nullptr;
    uchar4* ldr = nullptr;
    cudaStream_t cap_stream = nullptr;
    cudaStream_t side_stream = nullptr;  // the second branch of an overlapped frame
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    // guiding: the previous frame's training steps run on a third branch of
    // the next overlapped frame (beside its photon pass and first closest
    // hits); train_pending = the last frame's steps have not run yet
    cudaStream_t train_stream = nullptr;
    cudaEvent_t tfork_ev = nullptr, tjoin_ev = nullptr;
    bool train_pending = false;
    cudaGraphExec_t graph = nullptr;
    int launches_per_frame = 0;
    uint32_t frame_count = 0;
    uint64_t frames = 0, launches = 0, photons_emitted = 0, trace_launches = 0;
    double ms[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // photon, -, closest, shade, shadow, finalize, raygen, guide
                                                 // training, tail
    double ms_bounce[2][MAX_BOUNCES + 1] = {};  // closest-hit and shadow traversal per bounce
    std::vector<cudaEvent_t> ev;
    GuideArgs guide{};  // SRT_FLAG_GUIDING only
    // asynchronous RGBA8 read-back: two pinned slots used in turn
    uint8_t* ldr_pinned[2] = {nullptr, nullptr};
    cudaEvent_t ldr_ev[2] = {nullptr, nullptr};
    uint32_t ldr_calls = 0;

    // Photon-pass pipelining (SRT_PHOTON_PIPELINE): frame F's graph builds the
    // photon map of frame F + 1 on a branch of its own, beside F's camera
    // paths, which gather from the map built during the frame before.  The
    // photon arrays the camera paths read (stored photons, sorted photons,
    // grid ranges) and the photon pass's counters exist twice (set 0 is
    // `ph`'s); the working arrays are shared, since one photon pass runs at a
    // time.  A frame whose frame count is not the one predicted (or after a
    // scene change) first builds its own map.
    struct PipeSet {
        float4 *photons = nullptr, *sorted = nullptr;
        uint2* ranges = nullptr;
        FrameCounters* counters = nullptr;       // the photon pass's
        srt_camera_uniform* cam = nullptr;       // device: the photon pass's frame count
    } pipe[2];
    bool pipe_alloc = false;
    bool pipe_valid = false;                     // set pipe_cur holds the map of frame pipe_next
    int pipe_cur = 0;
    uint32_t pipe_next = 0;
    uint32_t pipe_scene_version = 0;
    int last_set = -1;                           // set the last frame gathered from (-1: `ph`, `counters`)
    cudaGraphExec_t pipe_graph[2] = {nullptr, nullptr};
    int pipe_launches[2] = {0, 0};
    cudaStream_t ph_stream = nullptr;
    cudaEvent_t pfork_ev = nullptr, pjoin_ev = nullptr;
    srt_camera_uniform* ph_ring = nullptr;       // pinned staging, 4 slots (with cam_ring's events)

    // The photon pass's arguments writing set s, and the camera paths'
    // arguments gathering from set s.
    FrameArgs photon_args(int s, const srt_camera_uniform* cam = nullptr) const {
        FrameArgs a = args;
        a.counters = pipe[s].counters;
        a.ph_counters = pipe[s].counters;
        a.cam = cam ? cam : pipe[s].cam;
        a.ph.photons = pipe[s].photons;
        a.ph.sorted = pipe[s].sorted;
        a.ph.ranges = pipe[s].ranges;
        return a;
    }
    FrameArgs camera_args(int s) const {
        FrameArgs a = args;
        a.ph_counters = pipe[s].counters;
        a.ph.photons = pipe[s].photons;
        a.ph.sorted = pipe[s].sorted;
        a.ph.ranges = pipe[s].ranges;
        a.gather.photons = pipe[s].sorted;
        a.gather.ranges = pipe[s].ranges;
        return a;
    }
    // In a batched capture: the photon set this renderer's camera paths
    // gather from (-1: `args` as they are), and the arguments that follow.
    int batch_set = -1;
    FrameArgs frame_args() const { return batch_set >= 0 ? camera_args(batch_set) : args; }
    bool can_pipeline() const { return p.photons_per_frame > 0 && scene->n_lights > 0; }
    // The photon map of the last frame rendered (its counters and stored photons).
    const FrameCounters* last_photon_counters() const { return last_set >= 0 ? pipe[last_set].counters : counters; }
    const float4* last_photons() const { return last_set >= 0 ? pipe[last_set].photons : ph.photons; }
    // The second photon set, both sets' counters and uniforms, the photon
    // branch's stream and events, the pinned staging (once).
    cudaError_t ensure_pipe() {
        if (pipe_alloc) return cudaSuccess;
        cudaError_t e;
        const uint32_t cap = ph.capacity;
        pipe[0].photons = ph.photons;
        pipe[0].sorted = ph.sorted;
        pipe[0].ranges = ph.ranges;
        if ((e = dev_alloc(&pipe[1].photons, 2ull * cap)) != cudaSuccess) return e;
        if ((e = dev_alloc(&pipe[1].sorted, 2ull * cap)) != cudaSuccess) return e;
        if ((e = dev_alloc(&pipe[1].ranges, (size_t)1 << p.hash_bits)) != cudaSuccess) return e;
        if ((e = cudaMemset(pipe[1].ranges, 0, sizeof(uint2) << p.hash_bits)) != cudaSuccess) return e;
        for (auto& ps : pipe) {
            if ((e = dev_alloc(&ps.counters, 1)) != cudaSuccess) return e;
            if ((e = cudaMemset(ps.counters, 0, sizeof(FrameCounters))) != cudaSuccess) return e;
            if ((e = dev_alloc(&ps.cam, 1)) != cudaSuccess) return e;
        }
        if ((e = cudaMallocHost((void**)&ph_ring, 8 * sizeof(srt_camera_uniform))) != cudaSuccess) return e;
        if ((e = cudaStreamCreateWithFlags(&ph_stream, cudaStreamNonBlocking)) != cudaSuccess) return e;
        if ((e = cudaEventCreateWithFlags(&pfork_ev, cudaEventDisableTiming)) != cudaSuccess) return e;
        if ((e = cudaEventCreateWithFlags(&pjoin_ev, cudaEventDisableTiming)) != cudaSuccess) return e;
        pipe_alloc = true;
        return cudaSuccess;
    }
    void drop_pipe_graphs() {
        for (auto& g : pipe_graph)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
        pipe_valid = false;
    }

    ~srt_renderer() {
        if (graph) cudaGraphExecDestroy(graph);
        for (auto& g : pipe_graph)
            if (g) cudaGraphExecDestroy(g);
        if (ph_stream) cudaStreamDestroy(ph_stream);
        if (pfork_ev) cudaEventDestroy(pfork_ev);
        if (pjoin_ev) cudaEventDestroy(pjoin_ev);
        cudaFreeHost(ph_ring);
        for (int k = 0; k < 2; ++k) {
            if (k == 1) {  // set 0's arrays are `ph`'s, freed below
                cudaFree(pipe[k].photons);
                cudaFree(pipe[k].sorted);
                cudaFree(pipe[k].ranges);
            }
            cudaFree(pipe[k].counters);
            cudaFree(pipe[k].cam);
        }
        if (counts_ev) cudaEventDestroy(counts_ev);
        if (counts_host) cudaFreeHost(counts_host);
        if (cap_stream) cudaStreamDestroy(cap_stream);
        if (side_stream) cudaStreamDestroy(side_stream);
        if (fork_ev) cudaEventDestroy(fork_ev);
        if (join_ev) cudaEventDestroy(join_ev);
        if (train_stream) cudaStreamDestroy(train_stream);
        if (tfork_ev) cudaEventDestroy(tfork_ev);
        if (tjoin_ev) cudaEventDestroy(tjoin_ev);
        for (auto& e : ring_ev)
            if (e) cudaEventDestroy(e);
        for (auto& e : ev) cudaEventDestroy(e);
        cudaFree(cam_dev);
        cudaFreeHost(cam_ring);
        for (int k = 0; k < 2; ++k) {
            cudaFreeHost(ldr_pinned[k]);
            if (ldr_ev[k]) cudaEventDestroy(ldr_ev[k]);
        }
        cudaFree(counters);
        cudaFree(stats);
        cudaFree(err);
        void* bufs[] = {pb.ray_o, pb.ray_d, pb.hit, pb.thr, pb.wl, pb.rad, pb.misc, pb.queue[0], pb.queue[1],
                        pb.sh_o, pb.sh_d, pb.sh_c, pb.sh_id, pb.sort_keys, pb.sort_keys_alt, pb.sort_vals_alt,
                        pb.sort_scratch, ph.ray_o, ph.ray_d, ph.state, ph.hit, ph.flags,
                        ph.queue[0], ph.queue[1], ph.staging, ph.block_counts, ph.photons, ph.sorted,
                        ph.keys, ph.vals, ph.keys2, ph.vals2, ph.sort_scratch, ph.ranges, accum, accum64, ldr};
        for (void* b : bufs) cudaFree(b);
        guide_free(guide);
    }

    // Enqueues one frame (after the camera upload).  stage timing: events
    // between stages (only when `timed`, which keeps every stage in order).
    // First bounce handled by the tail kernel (launch_tail): SRT_TAIL_AUTO,
    // 0 (none) or a bounce; used where the whole remainder of a path can run
    // in one kernel (no ray reordering, no guided vertex left).  tail_auto is
    // the automatic choice, 0 until the first frame's path counts are back.
    uint32_t tail_first = SRT_TAIL_AUTO;
    uint32_t tail_auto = 0;
    uint32_t* counts_host = nullptr;  // pinned: paths entering each bounce of one frame
    cudaEvent_t counts_ev = nullptr;
    int counts_state = 0;             // 0: not requested, 1: copy in flight, 2: read
    // A guiding renderer's tail starts after its guided bounces: the
    // automatic one right after them, a set one not at all if it would start
    // before their end.
    uint32_t tail_start() const {
        uint32_t t = tail_first == SRT_TAIL_AUTO ? tail_auto : tail_first;
        if (t != 0u && args.guiding && args.guide_bounces > t) t = tail_first == SRT_TAIL_AUTO ? args.guide_bounces : 0u;
        if (t == 0u || t >= p.max_depth || args.ray_sort) return p.max_depth;
        return t;
    }
    // The automatic tail start from one frame's path counts (paths[b] = paths
    // entering bounce b): the first bounce >= 1 whose paths fit in
    // SRT_TAIL_WAVES waves of the tail kernel, 0 if none.
    static uint32_t choose_tail(const uint32_t* paths, uint32_t max_depth, double capacity) {
        for (uint32_t b = 1; b < max_depth; ++b)
            if ((double)paths[b] <= SRT_TAIL_WAVES * capacity) return b;
        return 0u;
    }
    // Drops the captured frame (its shape changed).
    void drop_graph() {
        if (graph) {
            cudaGraphExecDestroy(graph);
            graph = nullptr;
        }
        drop_pipe_graphs();
    }
    // SRT_TAIL_AUTO: after the first frame, read its path counts back without
    // waiting and, once they are there, choose the tail (the next frame is
    // captured with it; the image does not change).
    void auto_tail_before_frame() {
        if (tail_first != SRT_TAIL_AUTO || counts_state != 1) return;
        if (cudaEventQuery(counts_ev) != cudaSuccess) return;
        counts_state = 2;
        const uint32_t t = choose_tail(counts_host, p.max_depth, (double)tail_threads(args));
        if (t != tail_auto) {
            tail_auto = t;
            drop_graph();
        }
    }
    void auto_tail_after_frame(cudaStream_t st) {
        if (tail_first != SRT_TAIL_AUTO || counts_state != 0) return;
        if (cudaMemcpyAsync(counts_host, counters->paths, sizeof(uint32_t) * (MAX_BOUNCES + 1), cudaMemcpyDeviceToHost,
                            st) == cudaSuccess &&
            cudaEventRecord(counts_ev, st) == cudaSuccess)
            counts_state = 1;
    }

    // Enqueues one frame (after the camera upload).  With stage timing,
    // events between stages (stage_of[i]: the stage and bounce of the
    // interval that ends at event i), every stage in order.
    std::vector<std::pair<int, int>> stage_of;
    int record(cudaStream_t st, bool timed) {
        if (!timed && SRT_FRAME_OVERLAP) return record_overlapped(st);
        int n = 0;
        size_t e = 0;
        stage_of.clear();
        auto mark = [&](int stage, int bounce) {
            if (timed) {
                cudaEventRecord(ev[e++], st);
                stage_of.emplace_back(stage, bounce);
            }
        };
        cudaMemsetAsync(counters, 0, sizeof(FrameCounters), st);
        mark(-1, 0);
        if (p.photons_per_frame > 0 && scene->n_lights > 0) {
            // without lights the reference emits nothing (photon_emit.wgsl:161-162); the grid stays empty
            FrameArgs& a = args;
            n += launch_photon_pass(a, st);
        }
        mark(0, 0);  // photon pass
        n += launch_raygen(args, st);
        mark(6, 0);
        const uint32_t tail = tail_start();
        for (uint32_t b = 0; b < tail; ++b) {
            n += launch_bounce(args, b, st, 1);
            mark(2, (int)b);
            n += launch_bounce(args, b, st, 2);
            mark(3, (int)b);
            n += launch_bounce(args, b, st, 3);
            mark(4, (int)b);
        }
        if (tail < p.max_depth) {
            n += launch_tail(args, tail, st);
            mark(8, (int)tail);
        }
        n += launch_finalize(args, st);
        n += launch_frame_stats(args, st);
        mark(5, 0);
        if (args.guiding) n += launch_guide_train(args, st);
        mark(7, 0);
        return n;
    }

    // The same frame with independent stages side by side (two branches that
    // fork from and join `st`): the camera rays and their first closest hits
    // beside the photon pass (neither reads the other's buffers; shading
    // joins them), and after each shading step the shadow rays of bounce b
    // beside the closest hits of bounce b + 1 (the shadow rays add to the
    // path radiance, which the shading of b + 1 reads after the join; the
    // closest hits read and write only rays, queues and hits).  The results
    // are those of the serial order.
    // `set` >= 0: the pipelined frame (SRT_PHOTON_PIPELINE): the camera paths
    // gather from photon set `set`, built before this frame, while a branch of
    // its own builds the next frame's map into set `set` ^ 1 (frame count from
    // pipe[set ^ 1].cam), joined at the frame's end.
    int record_overlapped(cudaStream_t st, int set = -1) {
        int n = 0;
        cudaStream_t s2 = side_stream;
        auto fork = [&]() {
            cudaEventRecord(fork_ev, st);
            cudaStreamWaitEvent(s2, fork_ev, 0);
        };
        auto join = [&]() {
            cudaEventRecord(join_ev, s2);
            cudaStreamWaitEvent(st, join_ev, 0);
        };
        const bool pipelined = set >= 0;
        FrameArgs ca;
        if (pipelined) ca = camera_args(set);
        FrameArgs& A = pipelined ? ca : args;
        cudaMemsetAsync(counters, 0, sizeof(FrameCounters), st);
        const bool deferred = args.guiding != 0;
        if (deferred) {
            // the previous frame's Adam steps and frame-end bookkeeping: they
            // read that frame's training records and write the network, which
            // nothing before this frame's shading touches (none on the first
            // frame: no records)
            cudaEventRecord(tfork_ev, st);
            cudaStreamWaitEvent(train_stream, tfork_ev, 0);
            n += launch_guide_steps(A, train_stream);
            cudaEventRecord(tjoin_ev, train_stream);
        }
        if (pipelined) {
            const int nx = set ^ 1;
            cudaEventRecord(pfork_ev, st);
            cudaStreamWaitEvent(ph_stream, pfork_ev, 0);
            cudaMemsetAsync(pipe[nx].counters, 0, sizeof(FrameCounters), ph_stream);
            FrameArgs pa = photon_args(nx);
            n += launch_photon_pass(pa, ph_stream);
            cudaEventRecord(pjoin_ev, ph_stream);
            n += launch_raygen(A, st);
            n += launch_bounce(A, 0, st, 1);
        } else {
            fork();
            n += launch_raygen(A, s2);
            n += launch_bounce(A, 0, s2, 1);
            if (p.photons_per_frame > 0 && scene->n_lights > 0) n += launch_photon_pass(args, st);
            join();
        }
        if (deferred) cudaStreamWaitEvent(st, tjoin_ev, 0);
        const uint32_t tail = tail_start();
        for (uint32_t b = 0; b < p.max_depth; ++b) {
            n += launch_bounce(A, b, st, 2);
            if (b + 1 == tail) {
                // the tail kernel shades paths whose radiance these shadow rays add to: after them
                n += launch_bounce(A, b, st, 3);
                n += launch_tail(A, tail, st);
                break;
            }
            if (b + 1 < p.max_depth) {
                fork();
                n += launch_bounce(A, b, s2, 3);
                n += launch_bounce(A, b + 1, st, 1);
                join();
            } else {
                n += launch_bounce(A, b, st, 3);
            }
        }
        n += launch_finalize(A, st);
        n += launch_frame_stats(A, st);
        // the training weights read this frame's path radiance: before the
        // next frame's camera rays reset it; the steps run in the next frame
        if (deferred) n += launch_guide_targets(A, st);
        if (pipelined) cudaStreamWaitEvent(st, pjoin_ev, 0);
        return n;
    }

    // Runs training steps that a frame left to the next one (before the
    // guide's state is read or changed from the host).
    int flush_training(cudaStream_t st) {
        if (!train_pending) return 0;
        train_pending = false;
        return launch_guide_steps(args, st);
    }

    // The same frame in parts for the batched renderer, which traces the
    // rays of all its scenes in shared launches between them.
    void record_clear(cudaStream_t st) { cudaMemsetAsync(counters, 0, sizeof(FrameCounters), st); }
    int record_photons(cudaStream_t st) {
        return p.photons_per_frame > 0 && scene->n_lights > 0 ? launch_photon_pass(args, st) : 0;
    }
    int record_raygen(cudaStream_t st) { return launch_raygen(frame_args(), st); }
    // guide = false: the guided continuation and the training step are left
    // to the batch's grouped guide kernels
    int record_shade(uint32_t b, cudaStream_t st, bool guide) {
        return b < p.max_depth ? launch_bounce(frame_args(), b, st, guide ? 2 : 4) : 0;
    }
    int record_end(cudaStream_t st, bool guide) {
        const FrameArgs A = frame_args();
        int n = launch_finalize(A, st) + launch_frame_stats(A, st);
        if (args.guiding && guide) n += launch_guide_train(A, st);
        return n;
    }
    MultiTraceItem trace_item(uint32_t b, bool shadow) const {
        MultiTraceItem it{};
        it.s = args.scene;
        it.err = args.err;
        if (shadow) {
            it.count = &counters->shadow[b];
            it.ro = pb.sh_o;
            it.rd = pb.sh_d;
            it.sh_id = pb.sh_id;
            it.sh_c = pb.sh_c;
            it.rad = pb.rad;
        } else {
            it.queue = pb.queue[b & 1];
            it.count = &counters->paths[b];
            it.ro = pb.ray_o;
            it.rd = pb.ray_d;
            it.hit = pb.hit;
        }
        return it;
    }
    bool batch_owned = false;
    uint32_t args_gen = 0;  // bumped when kernel arguments change outside a capture (a batch re-captures)
};

extern "C" srt_params srt_params_default(void) {
    srt_params p{};
    p.max_depth = 12;
    p.photons_per_frame = 1u << 20;
    p.hash_bits = 22;
    p.photon_max_bounces = 5;
    p.gather_cap = 64;
    p.flags = 0;
    p.cell_size = 0.02f;
    p.gather_radius0 = 0.02f;
    p.radius_exponent = -0.15f;
    p.spectral_radius = 20.0f;
    p.photon_norm_count = 0.0f;
    p.block_size = 0;
    return p;
}

extern "C" srt_status srt_renderer_create(srt_ctx* c, srt_scene* s, uint32_t w, uint32_t h, const srt_params* prm,
                                          srt_renderer** out) {
    if (!c || !s || !out || w == 0 || h == 0) return SRT_ERR_INVALID_ARG;
    *out = nullptr;
    srt_params p = prm ? *prm : srt_params_default();
    if (p.max_depth == 0 || p.max_depth > (uint32_t)MAX_BOUNCES) return fail(c, SRT_ERR_INVALID_ARG, "max_depth must be 1..31");
    if (p.hash_bits < 4 || p.hash_bits > 26) return fail(c, SRT_ERR_INVALID_ARG, "hash_bits must be 4..26");
    if (p.photons_per_frame > (1u << 26)) return fail(c, SRT_ERR_INVALID_ARG, "photons_per_frame above 2^26");
    if (!(p.cell_size > 0.f) || !(p.gather_radius0 > 0.f) || !(p.spectral_radius > 0.f) ||
        p.photon_max_bounces > (uint32_t)MAX_PHOTON_BOUNCES)
        return fail(c, SRT_ERR_INVALID_ARG, "invalid photon parameters (photon_max_bounces must be <= 16)");
    if ((uint64_t)w * h > (1ull << 28)) return fail(c, SRT_ERR_INVALID_ARG, "viewport too large");
    if ((p.flags & SRT_FLAG_GUIDING) && (p.flags & SRT_FLAG_RAY_SORT))
        return fail(c, SRT_ERR_INVALID_ARG, "SRT_FLAG_GUIDING and SRT_FLAG_RAY_SORT cannot be combined");
    cudaSetDevice(c->device);
    std::unique_ptr<srt_renderer> r(new (std::nothrow) srt_renderer());
    if (!r) return SRT_ERR_OOM;
    r->ctx = c;
    r->scene = s;
    r->w = w;
    r->h = h;
    r->p = p;
    size_t np = (size_t)w * h;
    CUDA_TRY(c, dev_alloc(&r->cam_dev, 1));
    CUDA_TRY(c, cudaMallocHost((void**)&r->cam_ring, 4 * sizeof(srt_camera_uniform)));
    for (auto& e : r->ring_ev) CUDA_TRY(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CUDA_TRY(c, dev_alloc(&r->counters, 1));
    CUDA_TRY(c, dev_alloc(&r->stats, 1));
    CUDA_TRY(c, dev_alloc(&r->err, 1));
    CUDA_TRY(c, cudaMemset(r->stats, 0, sizeof(DevStats)));
    CUDA_TRY(c, cudaMemset(r->err, 0, 4));
    PathBuffers& pb = r->pb;
    CUDA_TRY(c, dev_alloc(&pb.ray_o, np));
    CUDA_TRY(c, dev_alloc(&pb.ray_d, np));
    CUDA_TRY(c, dev_alloc(&pb.hit, np));
    CUDA_TRY(c, dev_alloc(&pb.thr, np));
    CUDA_TRY(c, dev_alloc(&pb.wl, np));
    CUDA_TRY(c, dev_alloc(&pb.rad, np));
    CUDA_TRY(c, dev_alloc(&pb.misc, np));
    CUDA_TRY(c, dev_alloc(&pb.queue[0], np));
    CUDA_TRY(c, dev_alloc(&pb.queue[1], np));
    CUDA_TRY(c, dev_alloc(&pb.sh_o, np));
    CUDA_TRY(c, dev_alloc(&pb.sh_d, np));
    CUDA_TRY(c, dev_alloc(&pb.sh_c, np));
    CUDA_TRY(c, dev_alloc(&pb.sh_id, np));
    if (p.flags & SRT_FLAG_RAY_SORT) {
        CUDA_TRY(c, dev_alloc(&pb.sort_keys, np));
        CUDA_TRY(c, dev_alloc(&pb.sort_keys_alt, np));
        CUDA_TRY(c, dev_alloc(&pb.sort_vals_alt, np));
        CUDA_TRY(c, dev_alloc(&pb.sort_scratch, radix_scratch_words((uint32_t)np)));
    }
    CUDA_TRY(c, dev_alloc(&r->accum, np));
    CUDA_TRY(c, cudaMemset(r->accum, 0, np * sizeof(float4)));
    if (p.flags & SRT_FLAG_FP64_ACCUM) {
        CUDA_TRY(c, dev_alloc(&r->accum64, np));
        CUDA_TRY(c, cudaMemset(r->accum64, 0, np * sizeof(double4)));
    }
    CUDA_TRY(c, dev_alloc(&r->ldr, np));
    CUDA_TRY(c, cudaMemset(r->ldr, 0, np * 4));
    PhotonBuffers& ph = r->ph;
    uint32_t cap = p.photons_per_frame;
    ph.capacity = cap;
    ph.n_blocks = (cap + PHOTON_BLOCK - 1) / PHOTON_BLOCK;
    if (cap > 0) {
        size_t slots = (size_t)ph.n_blocks * PHOTON_BLOCK;
        CUDA_TRY(c, dev_alloc(&ph.ray_o, slots));
        CUDA_TRY(c, dev_alloc(&ph.ray_d, slots));
        CUDA_TRY(c, dev_alloc(&ph.state, slots));
        CUDA_TRY(c, dev_alloc(&ph.hit, slots));
        CUDA_TRY(c, dev_alloc(&ph.flags, slots));
        CUDA_TRY(c, cudaMemset(ph.flags, 0, slots));
        CUDA_TRY(c, dev_alloc(&ph.queue[0], slots));
        CUDA_TRY(c, dev_alloc(&ph.queue[1], slots));
        CUDA_TRY(c, dev_alloc(&ph.staging, 2ull * slots));
        CUDA_TRY(c, dev_alloc(&ph.block_counts, ph.n_blocks));
        CUDA_TRY(c, dev_alloc(&ph.photons, 2ull * cap));
        CUDA_TRY(c, dev_alloc(&ph.sorted, 2ull * cap));
        CUDA_TRY(c, dev_alloc(&ph.keys, cap));
        CUDA_TRY(c, dev_alloc(&ph.vals, cap));
        CUDA_TRY(c, dev_alloc(&ph.keys2, cap));
        CUDA_TRY(c, dev_alloc(&ph.vals2, cap));
        CUDA_TRY(c, dev_alloc(&ph.sort_scratch, radix_scratch_words(cap)));
        CUDA_TRY(c, dev_alloc(&ph.ranges, (size_t)1 << p.hash_bits));
        CUDA_TRY(c, cudaMemset(ph.ranges, 0, sizeof(uint2) << p.hash_bits));
    }
    FrameArgs& a = r->args;
    a.scene = s->dev;
    r->scene_gen = s->gen;
    a.cam = r->cam_dev;
    a.width = w;
    a.height = h;
    a.max_depth = p.max_depth;
    a.photons_per_frame = p.photons_per_frame;
    a.photon_max_bounces = p.photon_max_bounces;
    a.counters = r->counters;
    a.ph_counters = r->counters;
    a.stats = r->stats;
    a.err = r->err;
    a.pb = pb;
    a.ph = ph;
    a.gather.photons = ph.sorted;
    a.gather.ranges = ph.ranges;
    a.gather.hash_bits = p.hash_bits;
    a.gather.cap = p.gather_cap;
    a.gather.cell = p.cell_size;
    a.gather.r0 = p.gather_radius0;
    a.gather.rexp = p.radius_exponent;
    a.gather.spectral_radius = p.spectral_radius;
    a.gather.inv_norm_count = 1.0f / (p.photon_norm_count > 0.f ? p.photon_norm_count : (float)(cap ? cap : 1u));
    a.gather.enabled = cap > 0;
    a.accum = r->accum;
    a.accum64 = r->accum64;
    a.ldr = r->ldr;
    a.count_visits = (p.flags & SRT_FLAG_COUNT_VISITS) ? 1 : 0;
    a.block_size = (int)p.block_size;
    a.ray_sort = (p.flags & SRT_FLAG_RAY_SORT) ? 1 : 0;
    a.sm_count = c->sm_count;
    a.seed = p.seed;
    if (p.flags & SRT_FLAG_GUIDING) {
        CUDA_TRY(c, guide_configure());
        CUDA_TRY(c, guide_alloc(r->guide, np));
        std::vector<float> w(G_NPARAMS);
        guide_default_params(1, w.data());
        CUDA_TRY(c, guide_upload(r->guide, w.data(), nullptr, nullptr, 0));
        r->guide.train = (p.flags & SRT_FLAG_GUIDE_FROZEN) ? 0 : 1;
        // the fused tcgen05 step by default: 0.283 vs 0.354 ms per 2^18-record
        // step at 1080p, the same error curves (caustic-slab scene, 20-s arms)
        r->guide.tc_train = 1;
        r->guide.err = r->err;
        a.guiding = 1;
        a.guide_bounces = SRT_GUIDE_BOUNCES_DEFAULT;
        a.guide = r->guide;
    }
    size_t n_events = 5 + 3 * (size_t)p.max_depth;
    r->ev.resize(n_events);
    for (auto& e : r->ev) CUDA_TRY(c, cudaEventCreate(&e));
    CUDA_TRY(c, cudaStreamCreateWithFlags(&r->cap_stream, cudaStreamNonBlocking));
    CUDA_TRY(c, cudaStreamCreateWithFlags(&r->side_stream, cudaStreamNonBlocking));
    CUDA_TRY(c, cudaEventCreateWithFlags(&r->fork_ev, cudaEventDisableTiming));
    CUDA_TRY(c, cudaEventCreateWithFlags(&r->join_ev, cudaEventDisableTiming));
    CUDA_TRY(c, cudaStreamCreateWithFlags(&r->train_stream, cudaStreamNonBlocking));
    CUDA_TRY(c, cudaEventCreateWithFlags(&r->tfork_ev, cudaEventDisableTiming));
    CUDA_TRY(c, cudaEventCreateWithFlags(&r->tjoin_ev, cudaEventDisableTiming));
    CUDA_TRY(c, cudaMallocHost(&r->counts_host, sizeof(uint32_t) * (MAX_BOUNCES + 1)));
    CUDA_TRY(c, cudaEventCreateWithFlags(&r->counts_ev, cudaEventDisableTiming));
    if (env_fault("launch")) return fail(c, SRT_ERR_CUDA, "injected launch failure");
    ctx_retain(c);
    *out = r.release();
    return SRT_OK;
}

extern "C" srt_status srt_renderer_destroy(srt_renderer* r) {
    if (!r || r->batch_owned) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    delete r;
    ctx_release(c);
    return SRT_OK;
}

extern "C" srt_status srt_render_frame(srt_renderer* r, const srt_camera_uniform* cam) {
    if (!r || !cam || r->batch_owned) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    cudaSetDevice(c->device);
    r->refresh_scene();
    r->auto_tail_before_frame();
    cudaStream_t st = c->stream;
    int slot = r->ring_i++ & 3;
    CUDA_TRY(c, cudaEventSynchronize(r->ring_ev[slot]));
    r->cam_ring[slot] = *cam;
    CUDA_TRY(c, cudaMemcpyAsync(r->cam_dev, &r->cam_ring[slot], sizeof(srt_camera_uniform), cudaMemcpyHostToDevice, st));
    bool timed = (r->p.flags & SRT_FLAG_STAGE_TIMING) != 0;
    bool use_graph = !timed && !(r->p.flags & SRT_FLAG_NO_GRAPH);
    const bool pipelined = SRT_PHOTON_PIPELINE && SRT_FRAME_OVERLAP && !timed && r->p.photons_per_frame > 0 &&
                           r->scene->n_lights > 0;
    if (pipelined) {
        CUDA_TRY(c, r->ensure_pipe());
        // this frame's photon map: built during the last frame, or now
        const uint32_t F = cam->frame_count;
        const int cur = r->pipe_cur;
        srt_camera_uniform* pr = r->ph_ring + 2 * slot;
        pr[0] = *cam;
        pr[1] = *cam;
        pr[1].frame_count = F + 1u;  // the next frame's photon pass
        if (!(r->pipe_valid && r->pipe_next == F && r->pipe_scene_version == r->scene->version)) {
            CUDA_TRY(c, cudaMemcpyAsync(r->pipe[cur].cam, pr, sizeof *pr, cudaMemcpyHostToDevice, st));
            CUDA_TRY(c, cudaMemsetAsync(r->pipe[cur].counters, 0, sizeof(FrameCounters), st));
            FrameArgs pa = r->photon_args(cur);
            r->launches += (uint64_t)launch_photon_pass(pa, st);
            CUDA_TRY(c, cudaGetLastError());
        }
        CUDA_TRY(c, cudaMemcpyAsync(r->pipe[cur ^ 1].cam, pr + 1, sizeof *pr, cudaMemcpyHostToDevice, st));
        CUDA_TRY(c, cudaEventRecord(r->ring_ev[slot], st));
        if (use_graph) {
            if (!r->pipe_graph[cur]) {
                cudaGraph_t g;
                CUDA_TRY(c, cudaStreamBeginCapture(r->cap_stream, cudaStreamCaptureModeThreadLocal));
                r->pipe_launches[cur] = r->record_overlapped(r->cap_stream, cur);
                CUDA_TRY(c, cudaStreamEndCapture(r->cap_stream, &g));
                cudaError_t e = cudaGraphInstantiate(&r->pipe_graph[cur], g, 0);
                cudaGraphDestroy(g);
                CUDA_TRY(c, e);
            }
            CUDA_TRY(c, cudaGraphLaunch(r->pipe_graph[cur], st));
            r->launches += (uint64_t)r->pipe_launches[cur];
        } else {
            r->launches += (uint64_t)r->record_overlapped(st, cur);
            CUDA_TRY(c, cudaGetLastError());
        }
        r->last_set = cur;
        r->pipe_cur = cur ^ 1;
        r->pipe_next = F + 1u;
        r->pipe_valid = true;
        r->pipe_scene_version = r->scene->version;
    } else if (use_graph) {
        CUDA_TRY(c, cudaEventRecord(r->ring_ev[slot], st));
        if (!r->graph) {
            cudaGraph_t g;
            CUDA_TRY(c, cudaStreamBeginCapture(r->cap_stream, cudaStreamCaptureModeThreadLocal));
            r->launches_per_frame = r->record(r->cap_stream, false);
            CUDA_TRY(c, cudaStreamEndCapture(r->cap_stream, &g));
            cudaError_t e = cudaGraphInstantiate(&r->graph, g, 0);
            cudaGraphDestroy(g);
            CUDA_TRY(c, e);
        }
        CUDA_TRY(c, cudaGraphLaunch(r->graph, st));
        r->launches += (uint64_t)r->launches_per_frame;
        r->last_set = -1;
    } else {
        CUDA_TRY(c, cudaEventRecord(r->ring_ev[slot], st));
        r->last_set = -1;
        int n = r->record(st, timed);
        r->launches += (uint64_t)n;
        CUDA_TRY(c, cudaGetLastError());
        if (timed) {
            // the last event this frame recorded (a frame with the tail kernel records fewer)
            CUDA_TRY(c, cudaEventSynchronize(r->ev[r->stage_of.size() - 1]));
            float t;
            auto el = [&](size_t a, size_t b) {
                cudaEventElapsedTime(&t, r->ev[a], r->ev[b]);
                return (double)t;
            };
            for (size_t i = 1; i < r->stage_of.size(); ++i) {
                const int stage = r->stage_of[i].first, b = r->stage_of[i].second;
                const double t_ms = el(i - 1, i);
                r->ms[stage] += t_ms;
                if (stage == 2) r->ms_bounce[0][b] += t_ms;
                if (stage == 4) r->ms_bounce[1][b] += t_ms;
            }
        }
    }
    r->auto_tail_after_frame(st);
    // an overlapped guided frame leaves its training steps to the next frame
    r->train_pending = r->args.guiding && !timed && SRT_FRAME_OVERLAP;
    r->trace_launches += r->tail_start();
    r->frames += 1;
    r->photons_emitted += r->p.photons_per_frame;
    r->frame_count += 1;  // renderer/mod.rs:204
    return SRT_OK;
}

extern "C" uint32_t srt_renderer_frame_count(const srt_renderer* r) { return r ? r->frame_count : 0u; }
extern "C" srt_status srt_renderer_set_frame_count(srt_renderer* r, uint32_t f) {
    if (!r) return SRT_ERR_INVALID_ARG;
    r->frame_count = f;
    return SRT_OK;
}

extern "C" srt_status srt_reset_accumulation(srt_renderer* r) {
    if (!r) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    size_t np = (size_t)r->w * r->h;
    CUDA_TRY(c, cudaMemsetAsync(r->accum, 0, np * sizeof(float4), c->stream));
    if (r->accum64) CUDA_TRY(c, cudaMemsetAsync(r->accum64, 0, np * sizeof(double4), c->stream));
    r->frame_count = 0;
    return SRT_OK;
}

extern "C" srt_status srt_read_accum_f32(srt_renderer* r, float* rgba) {
    if (!r || !rgba) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    CUDA_TRY(c, cudaMemcpyAsync(rgba, r->accum, (size_t)r->w * r->h * sizeof(float4), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return check_device_error(c, r->err);
}

extern "C" srt_status srt_read_accum_f64(srt_renderer* r, double* rgba) {
    if (!r || !rgba) return SRT_ERR_INVALID_ARG;
    if (!r->accum64) return fail(r->ctx, SRT_ERR_INVALID_ARG, "renderer created without SRT_FLAG_FP64_ACCUM");
    srt_ctx* c = r->ctx;
    CUDA_TRY(c, cudaMemcpyAsync(rgba, r->accum64, (size_t)r->w * r->h * sizeof(double4), cudaMemcpyDeviceToHost,
                                c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return check_device_error(c, r->err);
}

extern "C" srt_status srt_write_accum_f64(srt_renderer* r, const double* rgba) {
    if (!r || !rgba) return SRT_ERR_INVALID_ARG;
    if (!r->accum64) return fail(r->ctx, SRT_ERR_INVALID_ARG, "renderer created without SRT_FLAG_FP64_ACCUM");
    srt_ctx* c = r->ctx;
    cudaSetDevice(c->device);
    const size_t np = (size_t)r->w * r->h;
    std::vector<float4> f(np);
    for (size_t i = 0; i < np; ++i)
        f[i] = make_float4((float)rgba[4 * i], (float)rgba[4 * i + 1], (float)rgba[4 * i + 2], (float)rgba[4 * i + 3]);
    CUDA_TRY(c, cudaMemcpyAsync(r->accum64, rgba, np * sizeof(double4), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(r->accum, f.data(), np * sizeof(float4), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SRT_OK;
}

extern "C" srt_status srt_read_ldr_rgba8(srt_renderer* r, uint8_t* out, uint32_t pitch) {
    if (!r || !out || pitch < 4 * r->w) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    CUDA_TRY(c, cudaMemcpy2DAsync(out, pitch, r->ldr, 4 * r->w, 4 * r->w, r->h, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return check_device_error(c, r->err);
}

extern "C" srt_status srt_read_ldr_async(srt_renderer* r, uint32_t* ticket) {
    if (!r || !ticket) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    cudaSetDevice(c->device);
    const size_t bytes = (size_t)4 * r->w * r->h;
    if (!r->ldr_pinned[0]) {
        for (int k = 0; k < 2; ++k) {
            CUDA_TRY(c, cudaMallocHost((void**)&r->ldr_pinned[k], bytes));
            CUDA_TRY(c, cudaEventCreateWithFlags(&r->ldr_ev[k], cudaEventDisableTiming));
        }
    }
    const uint32_t slot = r->ldr_calls & 1u;
    CUDA_TRY(c, cudaEventSynchronize(r->ldr_ev[slot]));  // the slot's previous copy has landed
    CUDA_TRY(c, cudaMemcpyAsync(r->ldr_pinned[slot], r->ldr, bytes, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaEventRecord(r->ldr_ev[slot], c->stream));
    *ticket = r->ldr_calls++;
    return SRT_OK;
}

extern "C" srt_status srt_ldr_wait(srt_renderer* r, uint32_t ticket, const uint8_t** pixels) {
    if (!r || !pixels || !r->ldr_pinned[0] || ticket >= r->ldr_calls || ticket + 2u < r->ldr_calls)
        return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    cudaSetDevice(c->device);
    CUDA_TRY(c, cudaEventSynchronize(r->ldr_ev[ticket & 1u]));
    *pixels = r->ldr_pinned[ticket & 1u];
    return SRT_OK;
}

extern "C" srt_status srt_save_screenshot(srt_renderer* r, const char* path) {
    if (!r || !path) return SRT_ERR_INVALID_ARG;
    uint32_t pitch = (4 * r->w + 255u) & ~255u;  // utils/wgpu.rs:53-58
    std::vector<uint8_t> buf((size_t)pitch * r->h);
    srt_status s = srt_read_ldr_rgba8(r, buf.data(), pitch);
    if (s != SRT_OK) return s;
    if (!write_screenshot_png(path, buf.data(), r->w, r->h, pitch))
        return fail(r->ctx, SRT_ERR_INVALID_ARG, std::string("cannot write ") + path);
    return SRT_OK;
}

extern "C" srt_status srt_save_screenshot_async(srt_renderer* r, const char* path) {
    if (!r || !path) return SRT_ERR_INVALID_ARG;
    uint32_t pitch = (4 * r->w + 255u) & ~255u;  // utils/wgpu.rs:53-58
    std::vector<uint8_t> buf((size_t)pitch * r->h);
    srt_status s = srt_read_ldr_rgba8(r, buf.data(), pitch);
    if (s != SRT_OK) return s;
    try {
        screenshot_enqueue(path, std::move(buf), r->w, r->h, pitch);
    } catch (const std::exception& e) {
        return fail(r->ctx, SRT_ERR_OOM, std::string("screenshot worker: ") + e.what());
    }
    return SRT_OK;
}

extern "C" srt_status srt_screenshot_write(const char* path, const uint8_t* rgba, uint32_t w, uint32_t h,
                                           uint32_t pitch) {
    if (!path || !rgba || w == 0 || h == 0 || pitch < 4 * w) return SRT_ERR_INVALID_ARG;
    return write_screenshot_png(path, rgba, w, h, pitch) ? SRT_OK : SRT_ERR_INVALID_ARG;
}

extern "C" srt_status srt_renderer_get_stats(srt_renderer* r, srt_stats* out) {
    if (!r || !out) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    DevStats d;
    CUDA_TRY(c, cudaMemcpyAsync(&d, r->stats, sizeof d, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    std::memset(out, 0, sizeof *out);
    out->frames = r->frames;
    out->paths = d.paths;
    out->rays_closest = d.closest_rays;
    out->rays_shadow = d.shadow_rays;
    out->rays_photon = d.photon_rays;
    out->photons_emitted = r->photons_emitted;
    out->photons_stored = d.photons_stored;
    for (int k = 0; k < 3; ++k)
        for (int b = 0; b <= MAX_BOUNCES; ++b) {
            out->nodes_visited[k] += d.nodes_bounce[k][b];
            out->tris_tested[k] += d.tris_bounce[k][b];
        }
    out->ms_photon_pass = r->ms[0];
    out->ms_trace_closest = r->ms[2];
    out->ms_shade = r->ms[3];
    out->ms_trace_shadow = r->ms[4];
    out->ms_finalize = r->ms[5];
    out->ms_raygen = r->ms[6];
    out->ms_guide_train = r->ms[7];
    out->ms_tail = r->ms[8];
    out->tail_first = r->tail_start();
    out->launches_trace_closest = r->trace_launches;
    out->kernel_launches = r->launches;
    return check_device_error(c, r->err);
}

extern "C" srt_status srt_renderer_get_bounce_stats(srt_renderer* r, srt_bounce_stats* out) {
    if (!r || !out) return SRT_ERR_INVALID_ARG;
    static_assert(SRT_MAX_BOUNCE_STATS == MAX_BOUNCES + 1, "per-bounce arrays");
    srt_ctx* c = r->ctx;
    DevStats d;
    CUDA_TRY(c, cudaMemcpyAsync(&d, r->stats, sizeof d, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    std::memset(out, 0, sizeof *out);
    for (int k = 0; k < 3; ++k)
        for (int b = 0; b <= MAX_BOUNCES; ++b) {
            out->rays[k][b] = d.rays_bounce[k][b];
            out->nodes[k][b] = d.nodes_bounce[k][b];
            out->tris[k][b] = d.tris_bounce[k][b];
        }
    for (int k = 0; k < 2; ++k)
        for (int b = 0; b <= MAX_BOUNCES; ++b) out->ms[k][b] = r->ms_bounce[k][b];
    return check_device_error(c, r->err);
}

extern "C" srt_status srt_renderer_set_tail(srt_renderer* r, uint32_t first_bounce) {
    if (!r || r->batch_owned) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    cudaSetDevice(c->device);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    r->tail_first = first_bounce;
    r->drop_graph();  // the tail shapes the captured frame
    r->args_gen += 1;
    return SRT_OK;
}

extern "C" srt_status srt_renderer_reset_stats(srt_renderer* r) {
    if (!r) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    CUDA_TRY(c, cudaMemsetAsync(r->stats, 0, sizeof(DevStats), c->stream));
    r->frames = r->launches = r->photons_emitted = r->trace_launches = 0;
    for (double& m : r->ms) m = 0.0;
    for (auto& row : r->ms_bounce)
        for (double& m : row) m = 0.0;
    return SRT_OK;
}

extern "C" srt_status srt_renderer_read_photons(srt_renderer* r, srt_photon* out, uint32_t capacity, uint32_t* count) {
    if (!r || !count) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    FrameCounters fc;
    CUDA_TRY(c, cudaMemcpyAsync(&fc, r->last_photon_counters(), sizeof fc, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    *count = r->p.photons_per_frame ? fc.photons_stored : 0u;
    uint32_t n = std::min(*count, capacity);
    if (out && n) {
        CUDA_TRY(c, cudaMemcpyAsync(out, r->last_photons(), (size_t)n * sizeof(srt_photon), cudaMemcpyDeviceToHost,
                                    c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    }
    return check_device_error(c, r->err);
}

// ====================================================================== standalone kernels
namespace {
struct TempPhotons {
    PhotonBuffers ph{};
    float4* src = nullptr;
    ~TempPhotons() {
        void* bufs[] = {ph.sorted, ph.keys, ph.vals, ph.keys2, ph.vals2, ph.sort_scratch, ph.ranges, src};
        for (void* b : bufs) cudaFree(b);
    }
};

srt_status temp_grid(srt_ctx* c, const srt_photon* photons, uint32_t n, uint32_t frame, float cell, uint32_t bits,
                     TempPhotons& t) {
    CUDA_TRY(c, dev_alloc(&t.src, 2ull * n));
    CUDA_TRY(c, dev_alloc(&t.ph.sorted, 2ull * n));
    CUDA_TRY(c, dev_alloc(&t.ph.keys, n));
    CUDA_TRY(c, dev_alloc(&t.ph.vals, n));
    CUDA_TRY(c, dev_alloc(&t.ph.keys2, n));
    CUDA_TRY(c, dev_alloc(&t.ph.vals2, n));
    CUDA_TRY(c, dev_alloc(&t.ph.sort_scratch, radix_scratch_words(n)));
    CUDA_TRY(c, dev_alloc(&t.ph.ranges, (size_t)1 << bits));
    if (n) CUDA_TRY(c, cudaMemcpyAsync(t.src, photons, (size_t)n * 32, cudaMemcpyHostToDevice, c->stream));
    t.ph.capacity = n;
    launch_grid_build(t.src, n, frame, cell, bits, t.ph, c->stream);
    CUDA_TRY(c, cudaGetLastError());
    return SRT_OK;
}
}  // namespace

extern "C" srt_status srt_photon_grid_build(srt_ctx* c, const srt_photon* photons, uint32_t n, uint32_t frame,
                                            float cell, uint32_t bits, uint64_t* keys_out, uint32_t* ranges_out) {
    if (!c || (!photons && n) || bits < 4 || bits > 26 || !(cell > 0.f) || n >= (1u << 30)) return SRT_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    TempPhotons t;
    srt_status s = temp_grid(c, photons, n, frame, cell, bits, t);
    if (s != SRT_OK) return s;
    if (keys_out && n) {
        std::vector<uint32_t> k(n), v(n);
        CUDA_TRY(c, cudaMemcpyAsync(k.data(), t.ph.sorted_keys, 4ull * n, cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(c, cudaMemcpyAsync(v.data(), t.ph.sorted_vals, 4ull * n, cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        for (uint32_t i = 0; i < n; ++i) keys_out[i] = ((uint64_t)k[i] << 32) | v[i];
    }
    if (ranges_out)
        CUDA_TRY(c, cudaMemcpyAsync(ranges_out, t.ph.ranges, sizeof(uint2) << bits, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SRT_OK;
}

extern "C" srt_status srt_photon_gather(srt_ctx* c, const srt_photon* photons, uint32_t n, const float* queries,
                                        uint32_t n_q, uint32_t frame, const srt_params* p, float* out) {
    if (!c || !p || (!photons && n) || (!queries && n_q) || (!out && n_q)) return SRT_ERR_INVALID_ARG;
    if (p->hash_bits < 4 || p->hash_bits > 26 || !(p->cell_size > 0.f) || n >= (1u << 30)) return SRT_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    TempPhotons t;
    srt_status s = temp_grid(c, photons, n, frame, p->cell_size, p->hash_bits, t);
    if (s != SRT_OK) return s;
    float* dq = nullptr;
    float4* dout = nullptr;
    CUDA_TRY(c, dev_alloc(&dq, 10ull * n_q));
    cudaError_t e = dev_alloc(&dout, n_q);
    if (e != cudaSuccess) {
        cudaFree(dq);
        return cuda_fail(c, e, "alloc");
    }
    GatherArgs g{};
    g.photons = t.ph.sorted;
    g.ranges = t.ph.ranges;
    g.hash_bits = p->hash_bits;
    g.cap = p->gather_cap;
    g.cell = p->cell_size;
    g.r0 = p->gather_radius0;
    g.rexp = p->radius_exponent;
    g.spectral_radius = p->spectral_radius;
    float nc = p->photon_norm_count > 0.f ? p->photon_norm_count : (float)(p->photons_per_frame ? p->photons_per_frame : 1u);
    g.inv_norm_count = 1.0f / nc;
    g.enabled = 1;
    if (n_q) cudaMemcpyAsync(dq, queries, 40ull * n_q, cudaMemcpyHostToDevice, c->stream);
    launch_gather_queries(g, frame, dq, n_q, dout, c->stream);
    if (n_q) cudaMemcpyAsync(out, dout, 16ull * n_q, cudaMemcpyDeviceToHost, c->stream);
    e = cudaStreamSynchronize(c->stream);
    cudaFree(dq);
    cudaFree(dout);
    if (e != cudaSuccess) return cuda_fail(c, e, "gather");
    return SRT_OK;
}

extern "C" srt_status srt_trace_rays(srt_scene* s, const srt_ray* rays, uint32_t n, srt_hit* hits, int any_hit) {
    if (!s || (n && (!rays || !hits))) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = s->ctx;
    cudaSetDevice(c->device);
    if (n == 0) return SRT_OK;
    float4 *dr = nullptr, *dh = nullptr;
    CUDA_TRY(c, dev_alloc(&dr, 2ull * n));
    cudaError_t e = dev_alloc(&dh, n);
    if (e != cudaSuccess) {
        cudaFree(dr);
        return cuda_fail(c, e, "alloc");
    }
    cudaMemcpyAsync(dr, rays, 32ull * n, cudaMemcpyHostToDevice, c->stream);
    launch_trace_batch(s->dev, dr, n, dh, any_hit, c->d_err, c->stream);
    cudaMemcpyAsync(hits, dh, 16ull * n, cudaMemcpyDeviceToHost, c->stream);
    e = cudaStreamSynchronize(c->stream);
    cudaFree(dr);
    cudaFree(dh);
    if (e != cudaSuccess) return cuda_fail(c, e, "trace");
    return check_device_error(c, c->d_err);
}

extern "C" srt_status srt_test_device_math(srt_ctx* c, int op, uint32_t n, const void* in, void* out, const void* aux) {
    static const size_t in_sz[9] = {4, 4, 8, 28, 36, 4, 96, 20, 20};
    static const size_t out_sz[9] = {4, 12, 4, 16, 16, 20, 40, 4, 28};
    if (!c || op < 0 || op > 8 || (n && (!in || !out)) || (op == 8 && !aux)) return SRT_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    if (n == 0) return SRT_OK;
    void *din = nullptr, *dout = nullptr, *daux = nullptr;
    CUDA_TRY(c, dev_alloc((char**)&din, in_sz[op] * n));
    cudaError_t e = dev_alloc((char**)&dout, out_sz[op] * n);
    if (e == cudaSuccess && op == 8) e = dev_alloc((char**)&daux, sizeof(srt_camera_uniform));
    if (e == cudaSuccess) e = cudaMemcpyAsync(din, in, in_sz[op] * n, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && op == 8)
        e = cudaMemcpyAsync(daux, aux, sizeof(srt_camera_uniform), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        launch_test_math(op, n, din, dout, daux, c->stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, out_sz[op] * n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(din);
    cudaFree(dout);
    cudaFree(daux);
    if (e != cudaSuccess) return cuda_fail(c, e, "test_device_math");
    return SRT_OK;
}

// ------------------------------------------------------------------ path guiding
extern "C" uint32_t srt_guide_param_count(void) { return (uint32_t)G_NPARAMS; }

extern "C" srt_status srt_guide_default_weights(uint64_t seed, float* out, uint32_t n) {
    if (!out || n != (uint32_t)G_NPARAMS) return SRT_ERR_INVALID_ARG;
    guide_default_params(seed, out);
    return SRT_OK;
}

namespace {
// Pending training steps of the last frame run before the host reads or
// changes the guide's state, so it sees every frame's step.
srt_status guide_flush(srt_renderer* r) {
    srt_ctx* c = r->ctx;
    cudaSetDevice(c->device);
    r->launches += (uint64_t)r->flush_training(c->stream);
    CUDA_TRY(c, cudaGetLastError());
    return SRT_OK;
}
}  // namespace

extern "C" srt_status srt_renderer_guide_get_weights(srt_renderer* r, float* out, uint32_t n) {
    if (!r || !out || n != (uint32_t)G_NPARAMS) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    if (!r->args.guiding) return fail(c, SRT_ERR_INVALID_ARG, "renderer was created without SRT_FLAG_GUIDING");
    if (srt_status fs = guide_flush(r)) return fs;
    cudaSetDevice(c->device);
    CUDA_TRY(c, cudaMemcpyAsync(out, r->guide.net.master, n * 4, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SRT_OK;
}

extern "C" srt_status srt_renderer_guide_set_weights(srt_renderer* r, const float* w, uint32_t n) {
    if (!r || !w || n != (uint32_t)G_NPARAMS) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    if (!r->args.guiding) return fail(c, SRT_ERR_INVALID_ARG, "renderer was created without SRT_FLAG_GUIDING");
    if (srt_status fs = guide_flush(r)) return fs;
    cudaSetDevice(c->device);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    CUDA_TRY(c, guide_upload(r->guide, w, nullptr, nullptr, 0));
    return SRT_OK;
}

extern "C" srt_status srt_test_wait_timeout(srt_ctx* c, uint32_t polls) {
    if (!c || polls == 0 || polls > (1u << 20)) return SRT_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    launch_test_wait_timeout(polls, c->d_err, c->stream);
    CUDA_TRY(c, cudaGetLastError());
    return check_device_error(c, c->d_err);
}

extern "C" srt_status srt_renderer_guide_get_state(srt_renderer* r, float* params, float* adam_m, float* adam_v,
                                                   uint32_t* adam_step) {
    if (!r || !params || !adam_m || !adam_v || !adam_step) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    if (!r->args.guiding) return fail(c, SRT_ERR_INVALID_ARG, "renderer was created without SRT_FLAG_GUIDING");
    if (srt_status fs = guide_flush(r)) return fs;
    cudaSetDevice(c->device);
    GuideCounters gc;
    const size_t bytes = (size_t)G_NPARAMS * 4;
    CUDA_TRY(c, cudaMemcpyAsync(params, r->guide.net.master, bytes, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(adam_m, r->guide.net.adam_m, bytes, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(adam_v, r->guide.net.adam_v, bytes, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(&gc, r->guide.gc, sizeof gc, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    *adam_step = gc.adam_step;
    return SRT_OK;
}

extern "C" srt_status srt_renderer_guide_set_state(srt_renderer* r, const float* params, const float* adam_m,
                                                   const float* adam_v, uint32_t adam_step) {
    if (!r || !params || !adam_m || !adam_v) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    if (!r->args.guiding) return fail(c, SRT_ERR_INVALID_ARG, "renderer was created without SRT_FLAG_GUIDING");
    if (srt_status fs = guide_flush(r)) return fs;
    cudaSetDevice(c->device);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    CUDA_TRY(c, guide_upload(r->guide, params, adam_m, adam_v, adam_step));
    return SRT_OK;
}

extern "C" srt_status srt_renderer_guide_info(srt_renderer* r, uint32_t* adam_steps, uint32_t* threshold) {
    if (!r) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    if (!r->args.guiding) return fail(c, SRT_ERR_INVALID_ARG, "renderer was created without SRT_FLAG_GUIDING");
    if (srt_status fs = guide_flush(r)) return fs;
    cudaSetDevice(c->device);
    GuideCounters gc;
    CUDA_TRY(c, cudaMemcpyAsync(&gc, r->guide.gc, sizeof gc, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    if (adam_steps) *adam_steps = gc.adam_step;
    if (threshold) *threshold = gc.threshold;
    return SRT_OK;
}

extern "C" srt_status srt_renderer_guide_configure(srt_renderer* r, float lr, uint32_t batch) {
    if (!r || !(lr < 1.0f) || batch > G_REC_CAP) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    if (!r->args.guiding) return fail(c, SRT_ERR_INVALID_ARG, "renderer was created without SRT_FLAG_GUIDING");
    if (srt_status fs = guide_flush(r)) return fs;
    cudaSetDevice(c->device);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    if (lr >= 0.0f) r->guide.lr = lr;
    if (batch > 0) r->guide.batch = batch;
    r->args.guide = r->guide;
    r->args_gen += 1;
    r->drop_graph();  // both are kernel arguments of the captured frame
    return SRT_OK;
}

extern "C" srt_status srt_renderer_guide_set_steps(srt_renderer* r, uint32_t steps) {
    if (!r || steps < 1 || steps > 16) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    if (!r->args.guiding) return fail(c, SRT_ERR_INVALID_ARG, "renderer was created without SRT_FLAG_GUIDING");
    if (srt_status fs = guide_flush(r)) return fs;
    cudaSetDevice(c->device);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    r->guide.steps = steps;
    r->args.guide = r->guide;
    r->args_gen += 1;
    r->drop_graph();  // the step count shapes the captured frame
    return SRT_OK;
}

extern "C" srt_status srt_renderer_guide_set_bounces(srt_renderer* r, uint32_t bounces) {
    if (!r || bounces < 1) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    if (!r->args.guiding) return fail(c, SRT_ERR_INVALID_ARG, "renderer was created without SRT_FLAG_GUIDING");
    if (srt_status fs = guide_flush(r)) return fs;
    cudaSetDevice(c->device);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    r->args.guide_bounces = std::min<uint32_t>(bounces, MAX_BOUNCES + 1);
    r->args_gen += 1;
    r->drop_graph();  // the guided bounces shape the captured frame
    return SRT_OK;
}

namespace {
struct GuideScratch {
    GuideArgs g{};
    float* x = nullptr;
    float* y = nullptr;
    float* z = nullptr;
    ~GuideScratch() {
        guide_free(g);
        cudaFree(x);
        cudaFree(y);
        cudaFree(z);
    }
};
}  // namespace

namespace {
srt_status guide_test_forward(srt_ctx* c, const float* params, const float* x, uint32_t n, float* out, int tc) {
    if (!c || !params || (n && (!x || !out))) return SRT_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    if (n == 0) return SRT_OK;
    GuideScratch s;
    CUDA_TRY(c, guide_configure());
    CUDA_TRY(c, guide_alloc(s.g, 0));
    CUDA_TRY(c, guide_upload(s.g, params, nullptr, nullptr, 0));
    CUDA_TRY(c, dev_alloc(&s.x, (size_t)n * G_IN));
    CUDA_TRY(c, dev_alloc(&s.y, (size_t)n * G_OUT));
    CUDA_TRY(c, cudaMemcpyAsync(s.x, x, (size_t)n * G_IN * 4, cudaMemcpyHostToDevice, c->stream));
    launch_guide_test_forward(s.g.net, s.x, n, s.y, tc, c->d_err, c->stream);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaMemcpyAsync(out, s.y, (size_t)n * G_OUT * 4, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return check_device_error(c, c->d_err);
}
}  // namespace

extern "C" srt_status srt_guide_test_forward(srt_ctx* c, const float* params, const float* x, uint32_t n, float* out) {
    return guide_test_forward(c, params, x, n, out, 0);
}

extern "C" srt_status srt_guide_test_forward_tc(srt_ctx* c, const float* params, const float* x, uint32_t n,
                                                float* out) {
    return guide_test_forward(c, params, x, n, out, 1);
}

extern "C" srt_status srt_renderer_guide_set_training(srt_renderer* r, int kind) {
    if (!r || (kind != SRT_GUIDE_TRAIN_MMA_SYNC && kind != SRT_GUIDE_TRAIN_TCGEN05)) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    if (!r->args.guiding) return fail(c, SRT_ERR_INVALID_ARG, "renderer was created without SRT_FLAG_GUIDING");
    if (srt_status fs = guide_flush(r)) return fs;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    r->guide.tc_train = kind == SRT_GUIDE_TRAIN_TCGEN05 ? 1 : 0;
    r->args.guide = r->guide;
    r->args_gen += 1;
    r->drop_graph();  // the choice is baked into the captured frame
    return SRT_OK;
}

extern "C" srt_status srt_renderer_guide_set_inference(srt_renderer* r, int kind) {
    if (!r || (kind != SRT_GUIDE_INFER_MMA_SYNC && kind != SRT_GUIDE_INFER_TCGEN05)) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    if (!r->args.guiding) return fail(c, SRT_ERR_INVALID_ARG, "renderer was created without SRT_FLAG_GUIDING");
    if (srt_status fs = guide_flush(r)) return fs;
    cudaSetDevice(c->device);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    r->guide.tc = kind == SRT_GUIDE_INFER_TCGEN05 ? 1 : 0;
    r->args.guide = r->guide;
    r->args_gen += 1;
    r->drop_graph();  // the choice is baked into the captured frame
    return SRT_OK;
}

namespace {
srt_status guide_test_mixture(srt_ctx* c, const float* raw, const float* omega, const float* u, uint32_t n,
                              float* out, int tc) {
    if (!c || (n && (!raw || !omega || !u || !out))) return SRT_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    if (n == 0) return SRT_OK;
    GuideScratch s;
    CUDA_TRY(c, dev_alloc(&s.x, (size_t)n * (G_OUT + 6)));
    CUDA_TRY(c, dev_alloc(&s.y, (size_t)n * 4));
    float* d_raw = s.x;
    float* d_om = s.x + (size_t)n * G_OUT;
    float* d_u = d_om + (size_t)n * 3;
    CUDA_TRY(c, cudaMemcpyAsync(d_raw, raw, (size_t)n * G_OUT * 4, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(d_om, omega, (size_t)n * 12, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(d_u, u, (size_t)n * 12, cudaMemcpyHostToDevice, c->stream));
    launch_guide_test_mixture(d_raw, d_om, d_u, n, s.y, tc, c->stream);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaMemcpyAsync(out, s.y, (size_t)n * 16, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SRT_OK;
}
}  // namespace

extern "C" srt_status srt_guide_test_mixture(srt_ctx* c, const float* raw, const float* omega, const float* u,
                                             uint32_t n, float* out) {
    return guide_test_mixture(c, raw, omega, u, n, out, 0);
}

extern "C" srt_status srt_guide_test_mixture_tc(srt_ctx* c, const float* raw, const float* omega, const float* u,
                                                uint32_t n, float* out) {
    return guide_test_mixture(c, raw, omega, u, n, out, 1);
}

namespace {
srt_status guide_test_train(srt_ctx* c, const float* params, const float* adam_m, const float* adam_v,
                            uint32_t adam_step, float lr, const float* x, const float* omega, const float* pdf_bsdf,
                            const float* weight, uint32_t n, float* grad_out, float* params_out, float* m_out,
                            float* v_out, int tc) {
    if (!c || !params || !x || !omega || !pdf_bsdf || !weight || !grad_out || n == 0 || n > G_REC_CAP)
        return SRT_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    GuideScratch s;
    CUDA_TRY(c, guide_configure());
    CUDA_TRY(c, guide_alloc(s.g, 0));
    CUDA_TRY(c, guide_upload(s.g, params, adam_m, adam_v, adam_step));
    s.g.lr = lr;
    s.g.batch = n;
    s.g.tc_train = tc;
    s.g.err = c->d_err;
    std::vector<float4> x0(n), x1(n), x2(n), w(n), b(n);
    for (uint32_t i = 0; i < n; ++i) {
        const float* xi = x + (size_t)i * G_IN;
        x0[i] = make_float4(xi[0], xi[1], xi[2], xi[3]);
        x1[i] = make_float4(xi[4], xi[5], xi[6], xi[7]);
        x2[i] = make_float4(xi[8], xi[9], 0.f, 0.f);
        w[i] = make_float4(omega[3 * i], omega[3 * i + 1], omega[3 * i + 2], 1.0f);
        b[i] = make_float4(pdf_bsdf[i], 0.f, 0.f, 0.f);
    }
    CUDA_TRY(c, cudaMemcpy(s.g.rec.x0, x0.data(), n * 16, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(s.g.rec.x1, x1.data(), n * 16, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(s.g.rec.x2, x2.data(), n * 16, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(s.g.rec.w, w.data(), n * 16, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(s.g.rec.b, b.data(), n * 16, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(s.g.rec.weight, weight, n * 4, cudaMemcpyHostToDevice));
    // weights are used as given: their mean is set to 1 by weight_sum = n
    GuideCounters gc{};
    gc.records = n;
    gc.weight_sum = (float)n;
    gc.adam_step = adam_step;
    CUDA_TRY(c, cudaMemcpy(s.g.gc, &gc, sizeof gc, cudaMemcpyHostToDevice));
    launch_guide_test_train(s.g, 0, c->stream);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaMemcpyAsync(grad_out, s.g.net.grad, G_NPARAMS * 4, cudaMemcpyDeviceToHost, c->stream));
    if (params_out || m_out || v_out) {
        launch_guide_test_train(s.g, 1, c->stream);
        CUDA_TRY(c, cudaGetLastError());
        if (params_out)
            CUDA_TRY(c, cudaMemcpyAsync(params_out, s.g.net.master, G_NPARAMS * 4, cudaMemcpyDeviceToHost, c->stream));
        if (m_out) CUDA_TRY(c, cudaMemcpyAsync(m_out, s.g.net.adam_m, G_NPARAMS * 4, cudaMemcpyDeviceToHost, c->stream));
        if (v_out) CUDA_TRY(c, cudaMemcpyAsync(v_out, s.g.net.adam_v, G_NPARAMS * 4, cudaMemcpyDeviceToHost, c->stream));
    }
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return check_device_error(c, c->d_err);
}
}  // namespace

extern "C" srt_status srt_guide_test_train(srt_ctx* c, const float* params, const float* adam_m, const float* adam_v,
                                           uint32_t adam_step, float lr, const float* x, const float* omega,
                                           const float* pdf_bsdf, const float* weight, uint32_t n, float* grad_out,
                                           float* params_out, float* m_out, float* v_out) {
    return guide_test_train(c, params, adam_m, adam_v, adam_step, lr, x, omega, pdf_bsdf, weight, n, grad_out,
                            params_out, m_out, v_out, 0);
}

extern "C" srt_status srt_guide_test_train_tc(srt_ctx* c, const float* params, const float* adam_m,
                                              const float* adam_v, uint32_t adam_step, float lr, const float* x,
                                              const float* omega, const float* pdf_bsdf, const float* weight,
                                              uint32_t n, float* grad_out, float* params_out, float* m_out,
                                              float* v_out) {
    return guide_test_train(c, params, adam_m, adam_v, adam_step, lr, x, omega, pdf_bsdf, weight, n, grad_out,
                            params_out, m_out, v_out, 1);
}

// ------------------------------------------------------------------ headless presentation
namespace {
struct DevBufs {
    std::vector<void*> p;
    ~DevBufs() {
        for (void* b : p) cudaFree(b);
    }
    template <class T>
    cudaError_t alloc(T** out, size_t n) {
        cudaError_t e = cudaMalloc((void**)out, n * sizeof(T));
        if (e == cudaSuccess) p.push_back(*out);
        return e;
    }
};
}  // namespace

extern "C" srt_status srt_blit_letterbox(srt_ctx* c, const uint8_t* src, uint32_t sw, uint32_t sh, uint32_t ww,
                                         uint32_t wh, int srgb_target, uint8_t* out) {
    if (!c || !src || !out || sw == 0 || sh == 0 || ww == 0 || wh == 0) return SRT_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    DevBufs b;
    uchar4 *ds = nullptr, *dd = nullptr;
    CUDA_TRY(c, b.alloc(&ds, (size_t)sw * sh));
    CUDA_TRY(c, b.alloc(&dd, (size_t)ww * wh));
    CUDA_TRY(c, cudaMemcpyAsync(ds, src, (size_t)sw * sh * 4, cudaMemcpyHostToDevice, c->stream));
    launch_blit_letterbox(ds, sw, sh, dd, ww, wh, srgb_target, c->stream);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaMemcpyAsync(out, dd, (size_t)ww * wh * 4, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SRT_OK;
}

extern "C" srt_status srt_renderer_blit(srt_renderer* r, uint32_t ww, uint32_t wh, int srgb_target, uint8_t* out) {
    if (!r || !out || ww == 0 || wh == 0) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    cudaSetDevice(c->device);
    DevBufs b;
    uchar4* dd = nullptr;
    CUDA_TRY(c, b.alloc(&dd, (size_t)ww * wh));
    launch_blit_letterbox(r->ldr, r->w, r->h, dd, ww, wh, srgb_target, c->stream);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaMemcpyAsync(out, dd, (size_t)ww * wh * 4, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SRT_OK;
}

extern "C" srt_status srt_photon_splat(srt_ctx* c, const srt_photon* photons, uint32_t n,
                                       const srt_camera_uniform* cam, uint32_t w, uint32_t h, uint8_t* rgba) {
    if (!c || !cam || !rgba || (n && !photons) || w == 0 || h == 0) return SRT_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    DevBufs b;
    float4* dp = nullptr;
    srt_camera_uniform* dc = nullptr;
    uint32_t* counts = nullptr;
    uchar4* img = nullptr;
    CUDA_TRY(c, b.alloc(&dp, 2 * (size_t)(n ? n : 1)));
    CUDA_TRY(c, b.alloc(&dc, 1));
    CUDA_TRY(c, b.alloc(&counts, (size_t)w * h));
    CUDA_TRY(c, b.alloc(&img, (size_t)w * h));
    if (n) CUDA_TRY(c, cudaMemcpyAsync(dp, photons, (size_t)n * sizeof(srt_photon), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(dc, cam, sizeof *cam, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(img, rgba, (size_t)w * h * 4, cudaMemcpyHostToDevice, c->stream));
    launch_photon_splat(dp, n, dc, w, h, counts, img, c->stream);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaMemcpyAsync(rgba, img, (size_t)w * h * 4, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SRT_OK;
}

extern "C" srt_status srt_renderer_splat_photons(srt_renderer* r, const srt_camera_uniform* cam, uint32_t w,
                                                 uint32_t h, uint8_t* rgba) {
    if (!r || !cam || !rgba || w == 0 || h == 0) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = r->ctx;
    cudaSetDevice(c->device);
    FrameCounters fc;
    CUDA_TRY(c, cudaMemcpyAsync(&fc, r->last_photon_counters(), sizeof fc, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    uint32_t n = r->p.photons_per_frame ? std::min(fc.photons_stored, r->p.photons_per_frame) : 0u;
    DevBufs b;
    srt_camera_uniform* dc = nullptr;
    uint32_t* counts = nullptr;
    uchar4* img = nullptr;
    CUDA_TRY(c, b.alloc(&dc, 1));
    CUDA_TRY(c, b.alloc(&counts, (size_t)w * h));
    CUDA_TRY(c, b.alloc(&img, (size_t)w * h));
    CUDA_TRY(c, cudaMemcpyAsync(dc, cam, sizeof *cam, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(img, rgba, (size_t)w * h * 4, cudaMemcpyHostToDevice, c->stream));
    launch_photon_splat(r->last_photons(), n, dc, w, h, counts, img, c->stream);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaMemcpyAsync(rgba, img, (size_t)w * h * 4, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return check_device_error(c, r->err);
}

// ------------------------------------------------------------------ batched renderer
// Many scenes (each with its own viewport, parameters and accumulation) per
// iteration: per-scene photon passes, ray generation, shading and
// finalisation run as parallel branches of one CUDA graph; the closest-hit
// and shadow rays of all scenes are traced in one launch per bounce
// (k_trace_multi).  The graph is re-captured when the set of active scenes
// or the tuning changes.
// 1: the batch builds each scene's next photon map during the current
// iteration, as single renderers do (SRT_PHOTON_PIPELINE); bit-identical.
// 0 (the default): each scene's photon pass inside its iteration, beside the
// camera rays.  Measured on the 32-scene batch (all scenes active): 131 vs
// 118 ms per iteration — the scenes' concurrent branches already fill the
// GPU, and photon passes that run through the whole iteration slow its
// shared persistent traversal launches.
#ifndef SRT_BATCH_PHOTON_PIPELINE
#define SRT_BATCH_PHOTON_PIPELINE 0
#endif
// 1: the batch shades all its scenes' vertices of a bounce in one launch
// (k_shade_multi); 0 (the default): one shading launch per scene on its
// graph branch, the branches running at once.  Measured on the 32-scene
// batch (256^2..1024^2 viewports, all scenes active): 120.2 ms per iteration
// with the branches, 123.5 ms with the single launch (it reads the frame
// arguments from shared memory and spills more registers).
#ifndef SRT_BATCH_SHADE_MULTI
#define SRT_BATCH_SHADE_MULTI 0
#endif

struct srt_batch {
    srt_ctx* ctx = nullptr;
    std::vector<srt_renderer*> r;
    srt_camera_uniform* cams_dev = nullptr;
    srt_camera_uniform* cams_host = nullptr;  // pinned, 2 slots of n
    cudaEvent_t up_ev[2] = {};
    int up_i = 0;
    MultiTraceItem* items_dev = nullptr;  // [2 kinds][MAX_BOUNCES][MAX_BATCH]
    uint32_t* fetch_dev = nullptr;        // [4][MAX_BOUNCES]: closest-hit, shadow, guide, shading chunk counters
    FrameArgs* guide_items_dev = nullptr; // [MAX_BATCH] frame arguments of the guided renderers
    FrameArgs* shade_items_dev = nullptr; // [MAX_BATCH] frame arguments of the active renderers
    std::vector<uint32_t> graph_gen;      // the renderers' args_gen at capture
    std::vector<cudaStream_t> side;
    cudaStream_t cap = nullptr;
    cudaEvent_t fork_ev = nullptr;
    std::vector<cudaEvent_t> join_ev;
    cudaStream_t ovl = nullptr;  // shadow rays of bounce b beside the closest hits of b + 1
    cudaEvent_t ovl_fork = nullptr, ovl_join = nullptr;
    cudaGraphExec_t graph = nullptr;
    std::vector<uint8_t> graph_active;
    int graph_launches = 0;
    srt_batch_tuning tune{8, 32, 0.0f, 0, 8};
    uint32_t max_depth = 0;
    bool small_stack = true;
    // SRT_TAIL_AUTO for the batch: the first iteration's path counts of every
    // active scene (each renderer's counts_host), summed, choose one tail
    // start for the scenes whose renderers leave it automatic
    int counts_state = 0;  // 0: not requested, 1: copies in flight, 2: read
    cudaEvent_t counts_ev = nullptr;
    std::vector<uint8_t> counts_active;
    bool recapture = false;
    // photon-pass pipelining of the scenes whose renderers can (a photon
    // pass): each iteration builds the next iteration's photon maps on a
    // branch per scene (ph_side), joined at the iteration's end; the photon
    // passes' camera uniforms (frame counts) at ph_cams_dev[set * n + scene]
    std::vector<cudaStream_t> ph_side;
    std::vector<cudaEvent_t> ph_join;
    srt_camera_uniform* ph_cams_dev = nullptr;
    srt_camera_uniform* ph_cams_host = nullptr;  // pinned, 2 slots of 2n
    std::vector<int> graph_sets;                  // each scene's photon set at capture (-1: none)
    bool pipelines(const srt_renderer* x) const { return SRT_BATCH_PHOTON_PIPELINE && x->can_pipeline(); }

    ~srt_batch() {
        if (graph) cudaGraphExecDestroy(graph);
        for (auto s : side)
            if (s) cudaStreamDestroy(s);
        if (cap) cudaStreamDestroy(cap);
        if (fork_ev) cudaEventDestroy(fork_ev);
        if (ovl) cudaStreamDestroy(ovl);
        if (ovl_fork) cudaEventDestroy(ovl_fork);
        if (ovl_join) cudaEventDestroy(ovl_join);
        if (counts_ev) cudaEventDestroy(counts_ev);
        for (auto st : ph_side)
            if (st) cudaStreamDestroy(st);
        for (auto e : ph_join)
            if (e) cudaEventDestroy(e);
        cudaFree(ph_cams_dev);
        cudaFreeHost(ph_cams_host);
        for (auto e : join_ev)
            if (e) cudaEventDestroy(e);
        for (auto& e : up_ev)
            if (e) cudaEventDestroy(e);
        cudaFree(cams_dev);
        cudaFreeHost(cams_host);
        cudaFree(items_dev);
        cudaFree(fetch_dev);
        cudaFree(guide_items_dev);
        cudaFree(shade_items_dev);
        for (srt_renderer* x : r) {
            if (x) {
                x->batch_owned = false;
                delete x;
                ctx_release(ctx);
            }
        }
    }

    srt_status capture(const std::vector<uint8_t>& active) {
        srt_ctx* c = ctx;
        // frames in flight read the item tables that are rewritten below
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        if (graph) {
            cudaGraphExecDestroy(graph);
            graph = nullptr;
        }
        // the deepest tree sets the traversal stack (trees may have been rebuilt)
        small_stack = true;
        for (srt_renderer* x : r)
            if (x->args.scene.depth > (uint32_t)TRAV_STACK_SMALL) small_stack = false;
        std::vector<int> act;
        for (size_t i = 0; i < r.size(); ++i)
            if (active[i]) act.push_back((int)i);
        const int na = (int)act.size();
        // the photon set each scene's camera paths gather from (restored on every exit)
        struct SetGuard {
            std::vector<srt_renderer*>& r;
            ~SetGuard() {
                for (srt_renderer* x : r) x->batch_set = -1;
            }
        } set_guard{r};
        std::vector<int> sets(r.size(), -1);
        for (int k = 0; k < na; ++k)
            if (pipelines(r[act[k]])) sets[act[k]] = r[act[k]]->batch_set = r[act[k]]->pipe_cur;
        std::vector<MultiTraceItem> items((size_t)2 * MAX_BOUNCES * MAX_BATCH);
        for (uint32_t b = 0; b < max_depth; ++b)
            for (int k = 0; k < na; ++k) {
                items[((size_t)0 * MAX_BOUNCES + b) * MAX_BATCH + k] = r[act[k]]->trace_item(b, false);
                items[((size_t)1 * MAX_BOUNCES + b) * MAX_BATCH + k] = r[act[k]]->trace_item(b, true);
            }
        CUDA_TRY(c, cudaMemcpy(items_dev, items.data(), items.size() * sizeof(MultiTraceItem), cudaMemcpyHostToDevice));
        // guided renderers: their continuations and training steps run as
        // grouped launches over all of them (their frame arguments are
        // uploaded once the capture has recorded every per-renderer launch)
        std::vector<srt_renderer*> guided;
        uint32_t guide_depth = 0, guide_steps = 1;
        for (int k = 0; k < na; ++k)
            if (r[act[k]]->args.guiding) {
                guided.push_back(r[act[k]]);
                guide_depth = std::max(guide_depth, r[act[k]]->p.max_depth);
                guide_steps = std::max(guide_steps, r[act[k]]->args.guide.steps);
            }
        const int ng = (int)guided.size();
        cudaGraph_t g;
        int n = 0;
        CUDA_TRY(c, cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        auto fork_join = [&](auto&& body) {
            cudaEventRecord(fork_ev, cap);
            for (int k = 0; k < na; ++k) {
                cudaStreamWaitEvent(side[k], fork_ev, 0);
                n += body(r[act[k]], side[k]);
                cudaEventRecord(join_ev[k], side[k]);
            }
            for (int k = 0; k < na; ++k) cudaStreamWaitEvent(cap, join_ev[k], 0);
        };
        cudaMemsetAsync(fetch_dev, 0, sizeof(uint32_t) * 4 * MAX_BOUNCES, cap);
        for (int k = 0; k < na; ++k) r[act[k]]->record_clear(cap);
        auto closest = [&](uint32_t b, cudaStream_t s) {
            return launch_trace_multi(items_dev + (size_t)b * MAX_BATCH, na, 0, small_stack, fetch_dev + b,
                                      (int)tune.blocks_per_sm, tune.chunk, c->sm_count, s);
        };
        auto shadow = [&](uint32_t b, cudaStream_t s) {
            return launch_trace_multi(items_dev + ((size_t)MAX_BOUNCES + b) * MAX_BATCH, na, 1, small_stack,
                                      fetch_dev + MAX_BOUNCES + b, (int)tune.blocks_per_sm, tune.chunk, c->sm_count,
                                      s);
        };
        // the scenes' photon passes on their branches: a pipelined scene's
        // builds the next iteration's map beside the whole iteration (joined
        // at its end); another's builds this iteration's map beside the
        // camera rays and their first closest hits (shading, after the join,
        // reads both)
        const size_t nr = r.size();
        cudaEventRecord(fork_ev, cap);
        for (int k = 0; k < na; ++k) {
            srt_renderer* x = r[act[k]];
            if (sets[act[k]] >= 0) {
                const int nx = sets[act[k]] ^ 1;
                cudaStreamWaitEvent(ph_side[k], fork_ev, 0);
                cudaMemsetAsync(x->pipe[nx].counters, 0, sizeof(FrameCounters), ph_side[k]);
                FrameArgs pa = x->photon_args(nx, ph_cams_dev + (size_t)nx * nr + act[k]);
                n += launch_photon_pass(pa, ph_side[k]);
                cudaEventRecord(ph_join[k], ph_side[k]);
            } else {
                cudaStreamWaitEvent(side[k], fork_ev, 0);
                n += x->record_photons(side[k]);
                cudaEventRecord(join_ev[k], side[k]);
            }
        }
        for (int k = 0; k < na; ++k) n += r[act[k]]->record_raygen(cap);
        n += closest(0, cap);
        for (int k = 0; k < na; ++k)
            if (sets[act[k]] < 0) cudaStreamWaitEvent(cap, join_ev[k], 0);
        // the tail: from the latest first tail bounce of the scenes, each
        // scene's remaining bounces run in its own tail launch on its branch
        uint32_t tail = 0;
        for (int k = 0; k < na; ++k) tail = std::max(tail, r[act[k]]->tail_start());
        for (uint32_t b = 0; b < max_depth; ++b) {
            if (SRT_BATCH_SHADE_MULTI)
                n += launch_shade_multi(shade_items_dev, na, b, fetch_dev + 3 * MAX_BOUNCES + b, c->sm_count, cap);
            else
                fork_join([b](srt_renderer* x, cudaStream_t s) { return x->record_shade(b, s, false); });
            if (ng && b + 1 < guide_depth)
                n += launch_guide_infer_multi(guide_items_dev, ng, b, fetch_dev + 2 * MAX_BOUNCES + b, c->sm_count,
                                              cap);
            if (b + 1 == tail) {
                n += shadow(b, cap);
                fork_join([tail](srt_renderer* x, cudaStream_t s) { return launch_tail(x->frame_args(), tail, s); });
                break;
            }
            if (b + 1 < max_depth) {
                // independent: the shadow rays add to the radiance, the closest hits read rays and queues
                cudaEventRecord(ovl_fork, cap);
                cudaStreamWaitEvent(ovl, ovl_fork, 0);
                n += shadow(b, ovl);
                n += closest(b + 1, cap);
                cudaEventRecord(ovl_join, ovl);
                cudaStreamWaitEvent(cap, ovl_join, 0);
            } else {
                n += shadow(b, cap);
            }
        }
        fork_join([](srt_renderer* x, cudaStream_t s) { return x->record_end(s, false); });
        if (ng) n += launch_guide_train_multi(guide_items_dev, ng, guide_steps, c->sm_count, cap);
        for (int k = 0; k < na; ++k)
            if (sets[act[k]] >= 0) cudaStreamWaitEvent(cap, ph_join[k], 0);
        cudaError_t e = cudaStreamEndCapture(cap, &g);
        CUDA_TRY(c, e);
        {
            std::vector<FrameArgs> sargs;
            for (int k = 0; k < na; ++k) sargs.push_back(r[act[k]]->frame_args());
            e = cudaMemcpy(shade_items_dev, sargs.data(), na * sizeof(FrameArgs), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) cudaGraphDestroy(g);
            CUDA_TRY(c, e);
        }
        if (ng) {
            std::vector<FrameArgs> gargs;
            for (srt_renderer* x : guided) gargs.push_back(x->frame_args());
            e = cudaMemcpy(guide_items_dev, gargs.data(), ng * sizeof(FrameArgs), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) cudaGraphDestroy(g);
            CUDA_TRY(c, e);
        }
        e = cudaGraphInstantiate(&graph, g, 0);
        cudaGraphDestroy(g);
        CUDA_TRY(c, e);
        graph_active = active;
        graph_gen.clear();
        for (srt_renderer* x : r) graph_gen.push_back(x->args_gen);
        graph_sets = sets;
        graph_launches = n;
        recapture = false;
        return SRT_OK;
    }

    srt_status render(const srt_camera_uniform* cams, const uint8_t* active_in) {
        srt_ctx* c = ctx;
        cudaSetDevice(c->device);
        const size_t n = r.size();
        std::vector<uint8_t> active(n, 1);
        if (active_in)
            for (size_t i = 0; i < n; ++i) active[i] = active_in[i] ? 1 : 0;
        bool any = false;
        for (uint8_t a : active) any = any || a;
        if (!any) return SRT_OK;
        for (srt_renderer* x : r) x->refresh_scene();  // trees rebuilt since the capture
        auto_tail_before();
        for (size_t i = 0; i < n; ++i)
            if (active[i] && pipelines(r[i])) CUDA_TRY(c, r[i]->ensure_pipe());
        bool stale = recapture || graph_gen.size() != n || graph_sets.size() != n;
        for (size_t i = 0; i < n && !stale; ++i)
            stale = graph_gen[i] != r[i]->args_gen ||
                    (active[i] && graph_sets[i] != (pipelines(r[i]) ? r[i]->pipe_cur : -1));
        if (!graph || active != graph_active || stale) {
            srt_status s = capture(active);
            if (s != SRT_OK) return s;
        }
        int slot = up_i++ & 1;
        CUDA_TRY(c, cudaEventSynchronize(up_ev[slot]));
        std::memcpy(cams_host + slot * n, cams, n * sizeof(srt_camera_uniform));
        CUDA_TRY(c, cudaMemcpyAsync(cams_dev, cams_host + slot * n, n * sizeof(srt_camera_uniform),
                                    cudaMemcpyHostToDevice, c->stream));
        // the pipelined scenes' photon-pass uniforms: this iteration's frame
        // count in the set it gathers from (for a map built now), the next
        // one in the other set (the map this iteration builds ahead)
        srt_camera_uniform* pc = ph_cams_host + slot * 2 * n;
        std::vector<uint8_t> build_now(n, 0);
        for (size_t i = 0; i < n; ++i) {
            srt_renderer* x = r[i];
            if (!active[i] || !pipelines(x)) continue;
            const int cur = x->pipe_cur;
            const uint32_t F = cams[i].frame_count;
            pc[(size_t)cur * n + i] = cams[i];
            pc[(size_t)(cur ^ 1) * n + i] = cams[i];
            pc[(size_t)(cur ^ 1) * n + i].frame_count = F + 1u;
            build_now[i] = !(x->pipe_valid && x->pipe_next == F && x->pipe_scene_version == x->scene->version);
        }
        CUDA_TRY(c, cudaMemcpyAsync(ph_cams_dev, pc, 2 * n * sizeof(srt_camera_uniform), cudaMemcpyHostToDevice,
                                    c->stream));
        CUDA_TRY(c, cudaEventRecord(up_ev[slot], c->stream));
        for (size_t i = 0; i < n; ++i) {
            if (!build_now[i]) continue;  // a frame count or scene the map built ahead is not for
            srt_renderer* x = r[i];
            const int cur = x->pipe_cur;
            CUDA_TRY(c, cudaMemsetAsync(x->pipe[cur].counters, 0, sizeof(FrameCounters), c->stream));
            FrameArgs pa = x->photon_args(cur, ph_cams_dev + (size_t)cur * n + i);
            r[0]->launches += (uint64_t)launch_photon_pass(pa, c->stream);
            CUDA_TRY(c, cudaGetLastError());
        }
        CUDA_TRY(c, cudaGraphLaunch(graph, c->stream));
        for (size_t i = 0; i < n; ++i) {
            if (!active[i]) continue;
            srt_renderer* x = r[i];
            x->frames += 1;
            x->photons_emitted += x->p.photons_per_frame;
            x->frame_count += 1;
            if (pipelines(x)) {
                x->last_set = x->pipe_cur;
                x->pipe_cur ^= 1;
                x->pipe_next = cams[i].frame_count + 1u;
                x->pipe_valid = true;
                x->pipe_scene_version = x->scene->version;
            } else {
                x->last_set = -1;
            }
        }
        if (!r.empty()) r[0]->launches += (uint64_t)graph_launches;
        auto_tail_after(active);
        return SRT_OK;
    }

    void auto_tail_after(const std::vector<uint8_t>& active) {
        if (counts_state != 0) return;
        bool any_auto = false;
        for (srt_renderer* x : r) any_auto = any_auto || x->tail_first == SRT_TAIL_AUTO;
        if (!any_auto) return;
        for (size_t i = 0; i < r.size(); ++i)
            if (active[i] && cudaMemcpyAsync(r[i]->counts_host, r[i]->counters->paths,
                                             sizeof(uint32_t) * (MAX_BOUNCES + 1), cudaMemcpyDeviceToHost,
                                             ctx->stream) != cudaSuccess)
                return;
        if (cudaEventRecord(counts_ev, ctx->stream) != cudaSuccess) return;
        counts_active = active;
        counts_state = 1;
    }
    void auto_tail_before() {
        if (counts_state != 1 || cudaEventQuery(counts_ev) != cudaSuccess) return;
        counts_state = 2;
        std::vector<uint32_t> sum(MAX_BOUNCES + 1, 0u);
        uint32_t depth = 0;
        int first = -1;
        for (size_t i = 0; i < r.size(); ++i) {
            if (!counts_active[i]) continue;
            if (first < 0) first = (int)i;
            depth = std::max(depth, r[i]->p.max_depth);
            for (int b = 0; b <= MAX_BOUNCES; ++b) sum[b] += r[i]->counts_host[b];
        }
        if (first < 0) return;
        const uint32_t t = srt_renderer::choose_tail(sum.data(), depth, (double)tail_threads(r[first]->args));
        for (srt_renderer* x : r) {
            if (x->tail_first != SRT_TAIL_AUTO || x->tail_auto == t) continue;
            x->tail_auto = t;
            recapture = true;
        }
    }
};

extern "C" srt_status srt_batch_create(srt_ctx* c, uint32_t n, srt_scene* const* scenes, const uint32_t* widths,
                                       const uint32_t* heights, const srt_params* params, srt_batch** out) {
    if (!c || !out || n == 0 || n > (uint32_t)MAX_BATCH || !scenes || !widths || !heights) return SRT_ERR_INVALID_ARG;
    *out = nullptr;
    cudaSetDevice(c->device);
    std::unique_ptr<srt_batch> B(new (std::nothrow) srt_batch());
    if (!B) return SRT_ERR_OOM;
    B->ctx = c;
    CUDA_TRY(c, dev_alloc(&B->cams_dev, n));
    CUDA_TRY(c, cudaMallocHost((void**)&B->cams_host, 2 * n * sizeof(srt_camera_uniform)));
    std::memset(B->cams_host, 0, 2 * n * sizeof(srt_camera_uniform));
    CUDA_TRY(c, cudaMemset(B->cams_dev, 0, n * sizeof(srt_camera_uniform)));
    for (auto& e : B->up_ev) CUDA_TRY(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CUDA_TRY(c, dev_alloc(&B->items_dev, (size_t)2 * MAX_BOUNCES * MAX_BATCH));
    CUDA_TRY(c, dev_alloc(&B->fetch_dev, (size_t)4 * MAX_BOUNCES));
    CUDA_TRY(c, dev_alloc(&B->guide_items_dev, (size_t)MAX_BATCH));
    CUDA_TRY(c, dev_alloc(&B->shade_items_dev, (size_t)MAX_BATCH));
    CUDA_TRY(c, cudaEventCreateWithFlags(&B->counts_ev, cudaEventDisableTiming));
    CUDA_TRY(c, cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking));
    CUDA_TRY(c, cudaEventCreateWithFlags(&B->fork_ev, cudaEventDisableTiming));
    CUDA_TRY(c, cudaStreamCreateWithFlags(&B->ovl, cudaStreamNonBlocking));
    CUDA_TRY(c, cudaEventCreateWithFlags(&B->ovl_fork, cudaEventDisableTiming));
    CUDA_TRY(c, cudaEventCreateWithFlags(&B->ovl_join, cudaEventDisableTiming));
    B->side.assign(n, nullptr);
    B->join_ev.assign(n, nullptr);
    B->ph_side.assign(n, nullptr);
    B->ph_join.assign(n, nullptr);
    for (uint32_t i = 0; i < n; ++i) {
        CUDA_TRY(c, cudaStreamCreateWithFlags(&B->side[i], cudaStreamNonBlocking));
        CUDA_TRY(c, cudaEventCreateWithFlags(&B->join_ev[i], cudaEventDisableTiming));
        CUDA_TRY(c, cudaStreamCreateWithFlags(&B->ph_side[i], cudaStreamNonBlocking));
        CUDA_TRY(c, cudaEventCreateWithFlags(&B->ph_join[i], cudaEventDisableTiming));
    }
    CUDA_TRY(c, dev_alloc(&B->ph_cams_dev, 2ull * n));
    CUDA_TRY(c, cudaMemset(B->ph_cams_dev, 0, 2ull * n * sizeof(srt_camera_uniform)));
    CUDA_TRY(c, cudaMallocHost((void**)&B->ph_cams_host, 4ull * n * sizeof(srt_camera_uniform)));
    for (uint32_t i = 0; i < n; ++i) {
        srt_params p = params ? params[i] : srt_params_default();
        if (p.flags & (SRT_FLAG_STAGE_TIMING | SRT_FLAG_COUNT_VISITS | SRT_FLAG_RAY_SORT))
            return fail(c, SRT_ERR_INVALID_ARG, "batched scenes take no STAGE_TIMING, COUNT_VISITS or RAY_SORT flag");
        srt_renderer* x = nullptr;
        srt_status s = srt_renderer_create(c, scenes[i], widths[i], heights[i], &p, &x);
        if (s != SRT_OK) return s;
        x->batch_owned = true;
        x->args.cam = B->cams_dev + i;
        B->r.push_back(x);
        B->max_depth = std::max(B->max_depth, p.max_depth);
        if (scenes[i]->dev.depth > (uint32_t)TRAV_STACK_SMALL) B->small_stack = false;
    }
    ctx_retain(c);
    *out = B.release();
    return SRT_OK;
}

extern "C" srt_status srt_batch_destroy(srt_batch* b) {
    if (!b) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = b->ctx;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    delete b;
    ctx_release(c);
    return SRT_OK;
}

extern "C" uint32_t srt_batch_size(const srt_batch* b) { return b ? (uint32_t)b->r.size() : 0u; }

extern "C" srt_renderer* srt_batch_renderer(srt_batch* b, uint32_t i) {
    return (b && i < b->r.size()) ? b->r[i] : nullptr;
}

extern "C" srt_status srt_batch_render(srt_batch* b, const srt_camera_uniform* cams, const uint8_t* active) {
    if (!b || !cams) return SRT_ERR_INVALID_ARG;
    return b->render(cams, active);
}

extern "C" srt_status srt_batch_get_tuning(const srt_batch* b, srt_batch_tuning* out) {
    if (!b || !out) return SRT_ERR_INVALID_ARG;
    *out = b->tune;
    return SRT_OK;
}

extern "C" srt_status srt_batch_set_tuning(srt_batch* b, const srt_batch_tuning* t) {
    if (!b || !t || t->blocks_per_sm < 1 || t->blocks_per_sm > 8 || t->chunk < 32 || t->chunk > 1024 ||
        t->chunk % 32 != 0)
        return SRT_ERR_INVALID_ARG;
    b->tune.blocks_per_sm = t->blocks_per_sm;
    b->tune.chunk = t->chunk;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return SRT_OK;
}

extern "C" srt_status srt_batch_autotune(srt_batch* b, const srt_camera_uniform* cams, uint32_t iterations,
                                         srt_batch_tuning* out) {
    if (!b || !cams || iterations == 0) return SRT_ERR_INVALID_ARG;
    srt_ctx* c = b->ctx;
    cudaSetDevice(c->device);
    static const uint32_t bps[] = {2, 4, 8};
    // the persistent traversal (SRT_BATCH_TRACE_PT) takes rays lane by lane:
    // the chunk is not a knob then
    static const uint32_t chunk_list[] = {32, 64, 128};
    const size_t n_chunks = SRT_BATCH_TRACE_PT ? 1 : 3;
    cudaEvent_t e0, e1;
    CUDA_TRY(c, cudaEventCreate(&e0));
    CUDA_TRY(c, cudaEventCreate(&e1));
    srt_batch_tuning best{8, 32, 3.4e38f, 0, 0};
    srt_status st = SRT_OK;
    // guided scenes train during the tuning frames: their networks and Adam
    // state are saved here and put back afterwards
    std::vector<void*> saved(b->r.size(), nullptr);
    for (size_t i = 0; i < b->r.size(); ++i)
        if (b->r[i]->args.guiding) {
            cudaError_t e = cudaMalloc(&saved[i], guide_state_bytes());
            if (e == cudaSuccess) e = guide_state_copy(b->r[i]->guide, saved[i], true, c->stream);
            if (e != cudaSuccess) {
                for (void* p : saved) cudaFree(p);
                return fail(c, e == cudaErrorMemoryAllocation ? SRT_ERR_OOM : SRT_ERR_CUDA, cudaGetErrorString(e));
            }
        }
    for (uint32_t bp : bps)
        for (size_t ci = 0; ci < n_chunks; ++ci) {
            const uint32_t ch = chunk_list[ci];
            srt_batch_tuning t{bp, ch, 0.0f, 0, 0};
            srt_batch_set_tuning(b, &t);
            st = b->render(cams, nullptr);  // capture + warm-up
            if (st != SRT_OK) break;
            cudaEventRecord(e0, c->stream);
            for (uint32_t i = 0; i < iterations && st == SRT_OK; ++i) st = b->render(cams, nullptr);
            cudaEventRecord(e1, c->stream);
            if (st != SRT_OK) break;
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            ms /= (float)iterations;
            best.candidates += 1;
            if (ms < best.ms_per_iteration) {
                best.blocks_per_sm = bp;
                best.chunk = ch;
                best.ms_per_iteration = ms;
            }
        }
    // BVH node width: the scenes' trees rebuilt with 4 children per node and
    // timed with the best traversal setting; kept if faster, else rebuilt at
    // their width.  The tree changes speed, never results.
    best.bvh_width = 0;
    {
        std::vector<srt_scene*> sc;
        for (srt_renderer* x : b->r)
            if (std::find(sc.begin(), sc.end(), x->scene) == sc.end()) sc.push_back(x->scene);
        uint32_t w0 = (uint32_t)sc[0]->width;
        bool uniform = true;
        for (srt_scene* x : sc) uniform = uniform && (uint32_t)x->width == w0;
        best.bvh_width = uniform ? w0 : 0;
        const uint32_t alt = w0 == 8u ? 4u : 8u;
        if (st == SRT_OK && uniform) {
            for (srt_scene* x : sc)
                if (st == SRT_OK) st = srt_scene_rebuild_bvh(x, alt);
            srt_batch_tuning t{best.blocks_per_sm, best.chunk, 0.0f, 0, 0};
            srt_batch_set_tuning(b, &t);
            if (st == SRT_OK) st = b->render(cams, nullptr);
            float ms = 3.4e38f;
            if (st == SRT_OK) {
                cudaEventRecord(e0, c->stream);
                for (uint32_t i = 0; i < iterations && st == SRT_OK; ++i) st = b->render(cams, nullptr);
                cudaEventRecord(e1, c->stream);
                if (st == SRT_OK) {
                    cudaEventSynchronize(e1);
                    cudaEventElapsedTime(&ms, e0, e1);
                    ms /= (float)iterations;
                }
            }
            best.candidates += 1;
            if (st == SRT_OK && ms < best.ms_per_iteration) {
                best.ms_per_iteration = ms;
                best.bvh_width = alt;
            } else {
                for (srt_scene* x : sc)
                    if ((uint32_t)x->width != w0) {
                        srt_status s2 = srt_scene_rebuild_bvh(x, w0);
                        if (st == SRT_OK) st = s2;
                    }
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaError_t restored = cudaSuccess;
    for (size_t i = 0; i < b->r.size(); ++i)
        if (saved[i]) {
            if (restored == cudaSuccess) restored = guide_state_copy(b->r[i]->guide, saved[i], false, c->stream);
        }
    cudaStreamSynchronize(c->stream);
    for (void* p : saved) cudaFree(p);
    if (st != SRT_OK) return st;
    CUDA_TRY(c, restored);
    uint32_t n_cand = best.candidates;
    srt_batch_set_tuning(b, &best);
    b->tune.ms_per_iteration = best.ms_per_iteration;
    b->tune.candidates = n_cand;
    b->tune.bvh_width = best.bvh_width;
    // the tuning frames are not part of any image
    for (srt_renderer* x : b->r) {
        srt_status s = srt_reset_accumulation(x);
        if (s != SRT_OK) return s;
        srt_renderer_reset_stats(x);
    }
    if (out) *out = b->tune;
    return SRT_OK;
}
