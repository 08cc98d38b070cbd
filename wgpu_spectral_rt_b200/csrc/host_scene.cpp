// host_scene.cpp — scene builder, procedural geometry, scene presets, camera
// uniform and screenshot writer (host C++).
//
// Reference counterparts: src/scene/builder.rs, geometry.rs, camera.rs,
// cornell_box.rs, custom.rs and src/screenshot.rs.
#include "host_scene.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <unordered_map>

// ------------------------------------------------------------------ Mat4
Mat4 mat4_identity() {
    Mat4 r{};
    r.m[0] = r.m[5] = r.m[10] = r.m[15] = 1.0f;
    return r;
}
Mat4 mat4_mul(const Mat4& a, const Mat4& b) {
    Mat4 r{};
    for (int c = 0; c < 4; ++c)
        for (int row = 0; row < 4; ++row)
            r.m[4 * c + row] = a.m[row] * b.m[4 * c] + a.m[4 + row] * b.m[4 * c + 1] + a.m[8 + row] * b.m[4 * c + 2] +
                               a.m[12 + row] * b.m[4 * c + 3];
    return r;
}
Mat4 mat4_translation(float x, float y, float z) {
    Mat4 r = mat4_identity();
    r.m[12] = x;
    r.m[13] = y;
    r.m[14] = z;
    return r;
}
Mat4 mat4_scale(float x, float y, float z) {
    Mat4 r{};
    r.m[0] = x;
    r.m[5] = y;
    r.m[10] = z;
    r.m[15] = 1.0f;
    return r;
}
Mat4 mat4_rotation_x(float a) {
    float s = std::sin(a), c = std::cos(a);
    Mat4 r = mat4_identity();
    r.m[5] = c;
    r.m[6] = s;
    r.m[9] = -s;
    r.m[10] = c;
    return r;
}
Mat4 mat4_rotation_y(float a) {
    float s = std::sin(a), c = std::cos(a);
    Mat4 r = mat4_identity();
    r.m[0] = c;
    r.m[2] = -s;
    r.m[8] = s;
    r.m[10] = c;
    return r;
}
Mat4 mat4_rotation_z(float a) {
    float s = std::sin(a), c = std::cos(a);
    Mat4 r = mat4_identity();
    r.m[0] = c;
    r.m[1] = s;
    r.m[4] = -s;
    r.m[5] = c;
    return r;
}
static void mat4_apply(const Mat4& t, const float p[3], float w, float out[4]) {
    for (int r = 0; r < 4; ++r) out[r] = t.m[r] * p[0] + t.m[4 + r] * p[1] + t.m[8 + r] * p[2] + t.m[12 + r] * w;
}

// ------------------------------------------------------------------ builder
uint32_t srt_scene_builder::add_material(const srt_material& m) {  // builder.rs:70-74
    materials.push_back(m);
    return (uint32_t)materials.size() - 1;
}
uint32_t srt_scene_builder::add_mesh(const srt_vertex* v, uint32_t nv, const uint32_t* idx, uint32_t ni) {
    // builder.rs:76-91: record offsets into the global buffers
    srt_mesh_info mi{};
    mi.vertex_offset = (uint32_t)vertices.size();
    mi.index_offset = (uint32_t)indices.size();
    mesh_infos.push_back(mi);
    vertices.insert(vertices.end(), v, v + nv);
    indices.insert(indices.end(), idx, idx + ni);
    mesh_tris.push_back(ni / 3u);
    return (uint32_t)mesh_infos.size() - 1;
}
void srt_scene_builder::add_instance(uint32_t mesh, uint32_t mat, const Mat4& t) {  // builder.rs:93-99
    srt_instance in{};
    in.mesh_id = mesh;
    in.mat_id = mat;
    std::memcpy(in.transform, t.m, sizeof(t.m));
    instances.push_back(in);
}
void srt_scene_builder::add_light_instance(uint32_t mesh, uint32_t mat, const Mat4& t, const float params[4]) {
    // builder.rs:101-129: one world-space LightInfo per triangle
    add_instance(mesh, mat, t);
    srt_light_instance_rec rec{(uint32_t)instances.size() - 1u, (uint32_t)lights.size(), mesh_tris[mesh], {}};
    std::memcpy(rec.params, params, 16);
    light_instances.push_back(rec);
    const srt_mesh_info& mi = mesh_infos[mesh];
    for (uint32_t k = 0; k < mesh_tris[mesh]; ++k) {
        srt_light L{};
        float* dst[3] = {L.v0, L.v1, L.v2};
        for (int c = 0; c < 3; ++c) {
            const float* p = vertices[mi.vertex_offset + indices[mi.index_offset + 3 * k + c]].pos;
            float o[4];
            mat4_apply(t, p, 1.0f, o);
            dst[c][0] = o[0];
            dst[c][1] = o[1];
            dst[c][2] = o[2];
            dst[c][3] = 1.0f;
        }
        std::memcpy(L.params, params, 16);
        lights.push_back(L);
    }
}

// ------------------------------------------------------------------ geometry (geometry.rs)
static srt_vertex mkv(float px, float py, float pz, float nx, float ny, float nz) {
    srt_vertex v;
    v.pos[0] = px;
    v.pos[1] = py;
    v.pos[2] = pz;
    v.pos[3] = 1.0f;
    v.normal[0] = nx;
    v.normal[1] = ny;
    v.normal[2] = nz;
    v.normal[3] = 0.0f;
    return v;
}

void geom_plane(std::vector<srt_vertex>& v, std::vector<uint32_t>& i) {  // geometry.rs:12-35
    v = {mkv(-0.5f, 0.f, 0.5f, 0.f, 1.f, 0.f), mkv(0.5f, 0.f, 0.5f, 0.f, 1.f, 0.f),
         mkv(-0.5f, 0.f, -0.5f, 0.f, 1.f, 0.f), mkv(0.5f, 0.f, -0.5f, 0.f, 1.f, 0.f)};
    i = {0, 1, 2, 2, 1, 3};
}

void geom_cube(std::vector<srt_vertex>& v, std::vector<uint32_t>& i) {  // geometry.rs:38-126
    struct Side {
        float n[3], a[3], b[3], c[3], d[3];
    };
    static const Side sides[6] = {
        {{0, 0, 1}, {-0.5f, -0.5f, 0.5f}, {0.5f, -0.5f, 0.5f}, {0.5f, 0.5f, 0.5f}, {-0.5f, 0.5f, 0.5f}},
        {{0, 0, -1}, {0.5f, -0.5f, -0.5f}, {-0.5f, -0.5f, -0.5f}, {-0.5f, 0.5f, -0.5f}, {0.5f, 0.5f, -0.5f}},
        {{0, 1, 0}, {-0.5f, 0.5f, 0.5f}, {0.5f, 0.5f, 0.5f}, {0.5f, 0.5f, -0.5f}, {-0.5f, 0.5f, -0.5f}},
        {{0, -1, 0}, {-0.5f, -0.5f, -0.5f}, {0.5f, -0.5f, -0.5f}, {0.5f, -0.5f, 0.5f}, {-0.5f, -0.5f, 0.5f}},
        {{1, 0, 0}, {0.5f, -0.5f, 0.5f}, {0.5f, -0.5f, -0.5f}, {0.5f, 0.5f, -0.5f}, {0.5f, 0.5f, 0.5f}},
        {{-1, 0, 0}, {-0.5f, -0.5f, -0.5f}, {-0.5f, -0.5f, 0.5f}, {-0.5f, 0.5f, 0.5f}, {-0.5f, 0.5f, -0.5f}},
    };
    v.clear();
    i.clear();
    uint32_t base = 0;
    for (const Side& s : sides) {
        for (const float* p : {s.a, s.b, s.c, s.d}) v.push_back(mkv(p[0], p[1], p[2], s.n[0], s.n[1], s.n[2]));
        for (uint32_t k : {0u, 1u, 2u, 0u, 2u, 3u}) i.push_back(base + k);
        base += 4;
    }
}

namespace {
struct PairHash {
    size_t operator()(uint64_t k) const { return (size_t)(k * 0x9E3779B97F4A7C15ull >> 17); }
};
}  // namespace

void geom_icosphere(uint32_t subdivisions, std::vector<srt_vertex>& v, std::vector<uint32_t>& idx) {
    // geometry.rs:129-232: 12 golden-ratio vertices projected to radius 0.5,
    // 20 faces, each subdivision splits a face into 4 via cached midpoints.
    v.clear();
    idx.clear();
    const float t = (1.0f + std::sqrt(5.0f)) / 2.0f;
    auto add_vertex = [&](float x, float y, float z) {
        float len = std::sqrt(x * x + y * y + z * z);
        float nx = x / len, ny = y / len, nz = z / len;
        v.push_back(mkv(nx * 0.5f, ny * 0.5f, nz * 0.5f, nx, ny, nz));
        return (uint32_t)v.size() - 1;
    };
    add_vertex(-1, t, 0);
    add_vertex(1, t, 0);
    add_vertex(-1, -t, 0);
    add_vertex(1, -t, 0);
    add_vertex(0, -1, t);
    add_vertex(0, 1, t);
    add_vertex(0, -1, -t);
    add_vertex(0, 1, -t);
    add_vertex(t, 0, -1);
    add_vertex(t, 0, 1);
    add_vertex(-t, 0, -1);
    add_vertex(-t, 0, 1);
    std::vector<uint32_t> faces = {0, 11, 5, 0, 5,  1,  0,  1,  7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11,
                                   4, 11, 10, 2, 10, 7, 6, 7, 1, 8, 3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6,
                                   8, 3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1};
    std::unordered_map<uint64_t, uint32_t, PairHash> cache;
    auto midpoint = [&](uint32_t p1, uint32_t p2) {
        uint64_t key = p1 < p2 ? ((uint64_t)p1 << 32 | p2) : ((uint64_t)p2 << 32 | p1);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
        const float* a = v[p1].pos;
        const float* b = v[p2].pos;
        float mx = (a[0] + b[0]) * 0.5f, my = (a[1] + b[1]) * 0.5f, mz = (a[2] + b[2]) * 0.5f;
        float len = std::sqrt(mx * mx + my * my + mz * mz);
        float nx = mx / len, ny = my / len, nz = mz / len;
        v.push_back(mkv(nx * 0.5f, ny * 0.5f, nz * 0.5f, nx, ny, nz));
        uint32_t id = (uint32_t)v.size() - 1;
        cache.emplace(key, id);
        return id;
    };
    for (uint32_t s = 0; s < subdivisions; ++s) {
        cache.reserve(faces.size());
        std::vector<uint32_t> nf;
        nf.reserve(faces.size() * 4);
        for (size_t f = 0; f < faces.size(); f += 3) {
            uint32_t v1 = faces[f], v2 = faces[f + 1], v3 = faces[f + 2];
            uint32_t a = midpoint(v1, v2);
            uint32_t b = midpoint(v2, v3);
            uint32_t c = midpoint(v3, v1);
            uint32_t q[12] = {v1, a, c, v2, b, a, v3, c, b, a, b, c};
            nf.insert(nf.end(), q, q + 12);
        }
        faces.swap(nf);
    }
    idx = faces;
}

void geom_uv_sphere(uint32_t slices, uint32_t stacks, std::vector<srt_vertex>& v, std::vector<uint32_t>& idx) {
    // Latitude-longitude sphere of radius 0.5 wound counter-clockwise seen
    // from outside.  Rings 0..stacks (ring 0 = +y pole, ring `stacks` = -y
    // pole), each with slices+1 vertices (seam duplicated).  The top band is
    // a triangle fan; every other band is split into two triangles per quad,
    // so the bottom band carries `slices` zero-area triangles:
    // slices * (2 * stacks - 1) triangles in total (64 x 32 -> 4032).
    v.clear();
    idx.clear();
    const double PI_D = 3.14159265358979323846;
    for (uint32_t r = 0; r <= stacks; ++r) {
        double th = PI_D * r / stacks;
        for (uint32_t s = 0; s <= slices; ++s) {
            double ph = 2.0 * PI_D * s / slices;
            float nx = (float)(std::sin(th) * std::cos(ph)), ny = (float)std::cos(th),
                  nz = (float)(-std::sin(th) * std::sin(ph));
            v.push_back(mkv(0.5f * nx, 0.5f * ny, 0.5f * nz, nx, ny, nz));
        }
    }
    uint32_t row = slices + 1;
    for (uint32_t r = 0; r < stacks; ++r)
        for (uint32_t s = 0; s < slices; ++s) {
            uint32_t a = r * row + s, b = a + 1, c = a + row, d = c + 1;
            if (r == 0) {
                for (uint32_t k : {a, c, d}) idx.push_back(k);
            } else {
                for (uint32_t k : {a, c, d, a, d, b}) idx.push_back(k);
            }
        }
}

namespace {
inline uint32_t pcg(uint32_t x) {
    uint32_t s = x * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
inline float lattice(int x, int y, int z, uint32_t seed) {
    uint32_t h = pcg((uint32_t)x * 73856093u ^ pcg((uint32_t)y * 19349663u ^ pcg((uint32_t)z * 83492791u ^ seed)));
    return (float)(h >> 8) * (2.0f / 16777215.0f) - 1.0f;  // [-1, 1]
}
inline float smooth(float t) { return t * t * (3.0f - 2.0f * t); }
float value_noise(float x, float y, float z, uint32_t seed) {
    int ix = (int)std::floor(x), iy = (int)std::floor(y), iz = (int)std::floor(z);
    float fx = smooth(x - ix), fy = smooth(y - iy), fz = smooth(z - iz);
    float c[2][2][2];
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            for (int d = 0; d < 2; ++d) c[a][b][d] = lattice(ix + a, iy + b, iz + d, seed);
    auto lerp = [](float p, float q, float t) { return p + (q - p) * t; };
    float x00 = lerp(c[0][0][0], c[1][0][0], fx), x10 = lerp(c[0][1][0], c[1][1][0], fx);
    float x01 = lerp(c[0][0][1], c[1][0][1], fx), x11 = lerp(c[0][1][1], c[1][1][1], fx);
    return lerp(lerp(x00, x10, fy), lerp(x01, x11, fy), fz);
}
}  // namespace

void geom_displace(std::vector<srt_vertex>& v, const std::vector<uint32_t>& idx, float amplitude, uint32_t seed) {
    // r = 0.5 + amplitude * fbm(n), fbm = 3 octaves of value noise
    // (base frequency 4, lacunarity 2, gain 0.5), normalised to [-1, 1].
    for (auto& vx : v) {
        float nx = vx.normal[0], ny = vx.normal[1], nz = vx.normal[2];
        float f = 4.0f, amp = 1.0f, sum = 0.0f, norm = 0.0f;
        for (int o = 0; o < 3; ++o) {
            sum += amp * value_noise(nx * f, ny * f, nz * f, seed + 0x9E3779B9u * (uint32_t)o);
            norm += amp;
            f *= 2.0f;
            amp *= 0.5f;
        }
        float r = 0.5f + amplitude * (sum / norm);
        vx.pos[0] = nx * r;
        vx.pos[1] = ny * r;
        vx.pos[2] = nz * r;
    }
    std::vector<double> acc(3 * v.size(), 0.0);
    for (size_t f = 0; f + 2 < idx.size(); f += 3) {
        const float* a = v[idx[f]].pos;
        const float* b = v[idx[f + 1]].pos;
        const float* c = v[idx[f + 2]].pos;
        double e1[3] = {(double)b[0] - a[0], (double)b[1] - a[1], (double)b[2] - a[2]};
        double e2[3] = {(double)c[0] - a[0], (double)c[1] - a[1], (double)c[2] - a[2]};
        double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        for (int k = 0; k < 3; ++k)
            for (int d = 0; d < 3; ++d) acc[3 * idx[f + k] + d] += n[d];
    }
    for (size_t i = 0; i < v.size(); ++i) {
        double l = std::sqrt(acc[3 * i] * acc[3 * i] + acc[3 * i + 1] * acc[3 * i + 1] + acc[3 * i + 2] * acc[3 * i + 2]);
        if (l > 0) {
            v[i].normal[0] = (float)(acc[3 * i] / l);
            v[i].normal[1] = (float)(acc[3 * i + 1] / l);
            v[i].normal[2] = (float)(acc[3 * i + 2] / l);
        }
    }
}

// ------------------------------------------------------------------ presets
static srt_material mat(float r, float g, float b, float a, float t, float e1, float e2, float e3) {
    srt_material m;
    m.color[0] = r;
    m.color[1] = g;
    m.color[2] = b;
    m.color[3] = a;
    m.extra[0] = t;
    m.extra[1] = e1;
    m.extra[2] = e2;
    m.extra[3] = e3;
    return m;
}

static uint32_t add_geom(srt_scene_builder* b, void (*gen)(std::vector<srt_vertex>&, std::vector<uint32_t>&)) {
    std::vector<srt_vertex> v;
    std::vector<uint32_t> i;
    gen(v, i);
    return b->add_mesh(v.data(), (uint32_t)v.size(), i.data(), (uint32_t)i.size());
}

static const float F_PI = 3.14159265358979f;
static const float F_PI_2 = 1.57079632679490f;

// Cornell walls shared by the Cornell presets (cornell_box.rs:46-85)
static void cornell_walls(srt_scene_builder* b, uint32_t plane, uint32_t white, uint32_t red, uint32_t green) {
    Mat4 s2 = mat4_scale(2, 2, 2);
    b->add_instance(plane, white, mat4_mul(mat4_translation(0, -1, 0), s2));
    b->add_instance(plane, white, mat4_mul(mat4_mul(mat4_translation(0, 1, 0), mat4_rotation_x(F_PI)), s2));
    b->add_instance(plane, white, mat4_mul(mat4_mul(mat4_translation(0, 0, -1), mat4_rotation_x(F_PI_2)), s2));
    b->add_instance(plane, red, mat4_mul(mat4_mul(mat4_translation(-1, 0, 0), mat4_rotation_z(-F_PI_2)), s2));
    b->add_instance(plane, green, mat4_mul(mat4_mul(mat4_translation(1, 0, 0), mat4_rotation_z(F_PI_2)), s2));
}

static void default_camera(float cam[5]) {  // camera.rs:38-40
    cam[0] = 0.0f;
    cam[1] = 0.0f;
    cam[2] = 3.0f;
    cam[3] = -F_PI_2;
    cam[4] = 0.0f;
}

bool preset_fill(srt_scene_builder* b, int preset, uint32_t seed, float cam[5]) {
    default_camera(cam);
    switch (preset) {
        case SRT_PRESET_CORNELL_BOX: {  // cornell_box.rs:6-110
            uint32_t light = b->add_material(mat(6500, 1, 0, 1, 3, 0, 0, 0));
            uint32_t red = b->add_material(mat(0.65f, 0.05f, 0.05f, 1, 0, 0, 0, 0));
            uint32_t green = b->add_material(mat(0.12f, 0.45f, 0.15f, 1, 0, 0, 0, 0));
            uint32_t white = b->add_material(mat(0.73f, 0.73f, 0.73f, 1, 0, 0, 0, 0));
            uint32_t glass = b->add_material(mat(1, 1, 1, 1, 2, 0, 1.5f, 0.01f));
            uint32_t bubble = b->add_material(mat(1, 1, 1, 1, 4, 500.0f, 1.33f, 1.0f));
            uint32_t plane = add_geom(b, geom_plane);
            uint32_t cube = add_geom(b, geom_cube);
            std::vector<srt_vertex> sv;
            std::vector<uint32_t> si;
            geom_icosphere(4, sv, si);
            uint32_t sphere = b->add_mesh(sv.data(), (uint32_t)sv.size(), si.data(), (uint32_t)si.size());
            cornell_walls(b, plane, white, red, green);
            float lp[4] = {0.0f, 6500.0f, 1.0f, 0.0f};
            b->add_light_instance(
                plane, light,
                mat4_mul(mat4_mul(mat4_translation(0, 0.99f, 0), mat4_rotation_x(F_PI)), mat4_scale(0.5f, 0.5f, 0.5f)),
                lp);
            b->add_instance(cube, glass,
                            mat4_mul(mat4_mul(mat4_translation(-0.35f, -0.4f + 0.002f, -0.3f), mat4_rotation_y(0.4f)),
                                     mat4_scale(0.6f, 1.2f, 0.6f)));
            b->add_instance(sphere, bubble,
                            mat4_mul(mat4_translation(0.4f, -0.64f, 0.3f), mat4_scale(0.75f, 0.75f, 0.75f)));
            return true;
        }
        case SRT_PRESET_CUSTOM_PRISM: {  // custom.rs:6-116
            uint32_t light = b->add_material(mat(6500, 5, 0, 1, 3, 0, 0, 0));
            uint32_t wall = b->add_material(mat(0.01f, 0.01f, 0.01f, 1, 0, 0, 0, 0));
            uint32_t canvas = b->add_material(mat(0.95f, 0.95f, 0.95f, 1, 0, 0, 0, 0));
            uint32_t prism = b->add_material(mat(1, 1, 1, 1, 2, 0, 1.6f, 0.12f));
            uint32_t bubble = b->add_material(mat(1, 1, 1, 1, 4, 500.0f, 1.33f, 1.0f));
            uint32_t plane = add_geom(b, geom_plane);
            uint32_t cube = add_geom(b, geom_cube);
            std::vector<srt_vertex> sv;
            std::vector<uint32_t> si;
            geom_icosphere(4, sv, si);
            uint32_t sphere = b->add_mesh(sv.data(), (uint32_t)sv.size(), si.data(), (uint32_t)si.size());
            const float room = 4.0f;
            Mat4 sr = mat4_scale(room * 2, room * 2, room * 2);
            b->add_instance(plane, wall, mat4_mul(mat4_translation(0, -1, 0), sr));
            b->add_instance(plane, wall, mat4_mul(mat4_mul(mat4_translation(0, room - 1.0f, 0), mat4_rotation_x(F_PI)), sr));
            b->add_instance(plane, wall,
                            mat4_mul(mat4_mul(mat4_translation(0, room * 0.5f - 1.0f, -room), mat4_rotation_x(F_PI_2)), sr));
            b->add_instance(cube, canvas, mat4_mul(mat4_translation(0.5f, -0.55f, 0), mat4_scale(5, 0.1f, 3)));
            float lp[4] = {0.0f, 6500.0f, 5.0f, 0.0f};
            b->add_light_instance(plane, light,
                                  mat4_mul(mat4_mul(mat4_translation(-2.0f, -0.2f, 0), mat4_rotation_z(-F_PI_2 + 0.02f)),
                                           mat4_scale(0.5f, 1.0f, 0.02f)),
                                  lp);
            b->add_instance(cube, prism,
                            mat4_mul(mat4_mul(mat4_translation(-1.1f, -0.2f, 0), mat4_rotation_y(0.7f)),
                                     mat4_scale(0.5f, 0.8f, 0.5f)));
            b->add_instance(sphere, bubble, mat4_mul(mat4_translation(1.0f, -0.1f, -0.5f), mat4_scale(0.6f, 0.6f, 0.6f)));
            return true;
        }
        case SRT_PRESET_CONFIG1: {
            // Cornell walls (10 tris) + 2-tri 6500 K light + dispersive UV
            // sphere (64 x 32, Cauchy A = 1.5, B = 0.0042 um^2).
            uint32_t light = b->add_material(mat(6500, 1, 0, 1, 3, 0, 0, 0));
            uint32_t red = b->add_material(mat(0.65f, 0.05f, 0.05f, 1, 0, 0, 0, 0));
            uint32_t green = b->add_material(mat(0.12f, 0.45f, 0.15f, 1, 0, 0, 0, 0));
            uint32_t white = b->add_material(mat(0.73f, 0.73f, 0.73f, 1, 0, 0, 0, 0));
            uint32_t glass = b->add_material(mat(1, 1, 1, 1, 2, 0, 1.5f, 0.0042f));
            uint32_t plane = add_geom(b, geom_plane);
            std::vector<srt_vertex> sv;
            std::vector<uint32_t> si;
            geom_uv_sphere(64, 32, sv, si);
            uint32_t sphere = b->add_mesh(sv.data(), (uint32_t)sv.size(), si.data(), (uint32_t)si.size());
            cornell_walls(b, plane, white, red, green);
            float lp[4] = {0.0f, 6500.0f, 1.0f, 0.0f};
            b->add_light_instance(
                plane, light,
                mat4_mul(mat4_mul(mat4_translation(0, 0.99f, 0), mat4_rotation_x(F_PI)), mat4_scale(0.5f, 0.5f, 0.5f)),
                lp);
            b->add_instance(sphere, glass, mat4_mul(mat4_translation(0.0f, -0.548f, 0.0f), mat4_scale(0.9f, 0.9f, 0.9f)));
            return true;
        }
        case SRT_PRESET_CONFIG2: {
            // Displaced icosphere level 8 (1,310,720 tris; value-noise
            // amplitude 0.05) + 64 thin-film-coated GGX UV spheres
            // (alpha ~ U[0.05, 0.5], film d ~ U[200, 800] nm, n2 = 1.33 over
            // n3 = 1.5) in an 8 x 4 x 8 room lit by a 1.5 x 1.5 area light.
            uint32_t light = b->add_material(mat(6500, 3, 0, 1, 3, 0, 0, 0));
            uint32_t red = b->add_material(mat(0.65f, 0.05f, 0.05f, 1, 0, 0, 0, 0));
            uint32_t green = b->add_material(mat(0.12f, 0.45f, 0.15f, 1, 0, 0, 0, 0));
            uint32_t white = b->add_material(mat(0.73f, 0.73f, 0.73f, 1, 0, 0, 0, 0));
            uint32_t stone = b->add_material(mat(0.8f, 0.75f, 0.7f, 1, 0, 0, 0, 0));
            uint32_t plane = add_geom(b, geom_plane);
            std::vector<srt_vertex> v;
            std::vector<uint32_t> i;
            geom_icosphere(8, v, i);
            geom_displace(v, i, 0.05f, seed);
            uint32_t ico = b->add_mesh(v.data(), (uint32_t)v.size(), i.data(), (uint32_t)i.size());
            geom_uv_sphere(64, 32, v, i);
            uint32_t ball = b->add_mesh(v.data(), (uint32_t)v.size(), i.data(), (uint32_t)i.size());
            Mat4 s8 = mat4_scale(8, 8, 8);
            b->add_instance(plane, white, mat4_mul(mat4_translation(0, -1, 0), s8));
            b->add_instance(plane, white, mat4_mul(mat4_mul(mat4_translation(0, 3, 0), mat4_rotation_x(F_PI)), s8));
            b->add_instance(plane, white, mat4_mul(mat4_mul(mat4_translation(0, 1, -4), mat4_rotation_x(F_PI_2)), s8));
            b->add_instance(plane, red, mat4_mul(mat4_mul(mat4_translation(-4, 1, 0), mat4_rotation_z(-F_PI_2)), s8));
            b->add_instance(plane, green, mat4_mul(mat4_mul(mat4_translation(4, 1, 0), mat4_rotation_z(F_PI_2)), s8));
            float lp[4] = {0.0f, 6500.0f, 3.0f, 0.0f};
            b->add_light_instance(
                plane, light,
                mat4_mul(mat4_mul(mat4_translation(0, 2.99f, -0.5f), mat4_rotation_x(F_PI)), mat4_scale(1.5f, 1.5f, 1.5f)),
                lp);
            b->add_instance(ico, stone, mat4_mul(mat4_translation(0, 0.2f, -1.0f), mat4_scale(2.4f, 2.4f, 2.4f)));
            uint32_t st = seed * 2654435761u + 12345u;
            auto rnd = [&]() {
                st = pcg(st);
                return (float)st / 4294967296.0f;
            };
            const int rings[2] = {22, 42};
            const float radii[2] = {1.75f, 2.75f};
            const float rs = 0.18f;
            for (int r = 0; r < 2; ++r)
                for (int k = 0; k < rings[r]; ++k) {
                    float ang = 2.0f * F_PI * ((float)k + 0.5f * (float)r) / (float)rings[r];
                    float alpha = 0.05f + 0.45f * rnd();
                    float d = 200.0f + 600.0f * rnd();
                    uint32_t m = b->add_material(mat(1, 1, 1, alpha, 5, d, 1.33f, 1.5f));
                    b->add_instance(ball, m,
                                    mat4_mul(mat4_translation(radii[r] * std::cos(ang), -1.0f + rs,
                                                              -1.0f + radii[r] * std::sin(ang)),
                                             mat4_scale(2 * rs, 2 * rs, 2 * rs)));
                }
            cam[0] = 0.0f;
            cam[1] = 1.0f;
            cam[2] = 6.0f;
            cam[3] = -F_PI_2;
            cam[4] = -0.12f;
            return true;
        }
        case SRT_PRESET_CAUSTIC_SLAB: {
            // Dispersive glass slab (Cauchy A = 1.5, B = 0.01 um^2) under a
            // 0.05-wide slit light, above a diffuse floor, beside the
            // config-1 UV sphere mesh (diffuse), in a dark room.
            uint32_t light = b->add_material(mat(6500, 40, 0, 1, 3, 0, 0, 0));
            uint32_t floor_m = b->add_material(mat(0.8f, 0.8f, 0.8f, 1, 0, 0, 0, 0));
            uint32_t wall = b->add_material(mat(0.3f, 0.3f, 0.3f, 1, 0, 0, 0, 0));
            uint32_t glass = b->add_material(mat(1, 1, 1, 1, 2, 0, 1.5f, 0.01f));
            uint32_t stone = b->add_material(mat(0.6f, 0.5f, 0.4f, 1, 0, 0, 0, 0));
            uint32_t plane = add_geom(b, geom_plane);
            uint32_t cube = add_geom(b, geom_cube);
            std::vector<srt_vertex> sv;
            std::vector<uint32_t> si;
            geom_uv_sphere(64, 32, sv, si);
            uint32_t sphere = b->add_mesh(sv.data(), (uint32_t)sv.size(), si.data(), (uint32_t)si.size());
            cornell_walls(b, plane, floor_m, wall, wall);
            float lp[4] = {0.0f, 6500.0f, 40.0f, 0.0f};
            b->add_light_instance(
                plane, light,
                mat4_mul(mat4_mul(mat4_translation(-0.3f, 0.99f, 0), mat4_rotation_x(F_PI)), mat4_scale(0.05f, 1.0f, 1.2f)),
                lp);
            b->add_instance(cube, glass,
                            mat4_mul(mat4_mul(mat4_translation(-0.2f, 0.3f, 0.0f), mat4_rotation_z(0.35f)),
                                     mat4_scale(0.9f, 0.12f, 1.0f)));
            b->add_instance(sphere, stone, mat4_mul(mat4_translation(0.5f, -0.65f, -0.3f), mat4_scale(0.7f, 0.7f, 0.7f)));
            return true;
        }
        case SRT_PRESET_INDIRECT_ROOM: {
            // Cornell walls; a 0.3 x 0.3 light 0.05 below the ceiling, facing
            // it, hidden from the room by a 0.5 x 0.5 panel just below it.
            // Every room point is lit through the small bright ceiling spot
            // alone (its light samples face away), the case where guided
            // sampling of the diffuse continuation pays off.
            uint32_t light = b->add_material(mat(6500, 8, 0, 1, 3, 0, 0, 0));
            uint32_t red = b->add_material(mat(0.65f, 0.05f, 0.05f, 1, 0, 0, 0, 0));
            uint32_t green = b->add_material(mat(0.12f, 0.45f, 0.15f, 1, 0, 0, 0, 0));
            uint32_t white = b->add_material(mat(0.73f, 0.73f, 0.73f, 1, 0, 0, 0, 0));
            uint32_t plane = add_geom(b, geom_plane);
            uint32_t cube = add_geom(b, geom_cube);
            cornell_walls(b, plane, white, red, green);
            float lp[4] = {0.0f, 6500.0f, 8.0f, 0.0f};
            b->add_light_instance(plane, light, mat4_mul(mat4_translation(0, 0.95f, 0), mat4_scale(0.3f, 0.3f, 0.3f)), lp);
            b->add_instance(cube, white, mat4_mul(mat4_translation(0, 0.93f, 0), mat4_scale(0.5f, 0.02f, 0.5f)));
            b->add_instance(cube, white,
                            mat4_mul(mat4_mul(mat4_translation(-0.35f, -0.6f, -0.3f), mat4_rotation_y(0.4f)),
                                     mat4_scale(0.5f, 0.8f, 0.5f)));
            return true;
        }
        case SRT_PRESET_BATCH_RANDOM: {
            uint32_t st = pcg(seed * 747796405u + 2891336453u);
            auto rnd = [&]() {
                st = pcg(st);
                return (float)st / 4294967296.0f;
            };
            const double budget = std::exp(std::log(1e4) + rnd() * (std::log(2e6) - std::log(1e4)));
            uint32_t light = b->add_material(mat(6500, 2, 0, 1, 3, 0, 0, 0));
            uint32_t red = b->add_material(mat(0.65f, 0.05f, 0.05f, 1, 0, 0, 0, 0));
            uint32_t green = b->add_material(mat(0.12f, 0.45f, 0.15f, 1, 0, 0, 0, 0));
            uint32_t white = b->add_material(mat(0.73f, 0.73f, 0.73f, 1, 0, 0, 0, 0));
            // draws are sequenced explicitly: the evaluation order of function
            // arguments is unspecified in C++
            const float sr = 0.3f + 0.5f * rnd();
            const float sg = 0.3f + 0.5f * rnd();
            const float sb = 0.3f + 0.5f * rnd();
            uint32_t stone = b->add_material(mat(sr, sg, sb, 1, 0, 0, 0, 0));
            uint32_t plane = add_geom(b, geom_plane);
            cornell_walls(b, plane, white, red, green);
            float lp[4] = {0.0f, 6500.0f, 2.0f, 0.0f};
            b->add_light_instance(
                plane, light,
                mat4_mul(mat4_mul(mat4_translation(0, 0.99f, 0), mat4_rotation_x(F_PI)), mat4_scale(0.6f, 0.6f, 0.6f)),
                lp);
            // the largest displaced icosphere within the budget (level 4..8)
            uint32_t level = 4;
            while (level < 8 && 20.0 * std::pow(4.0, (double)(level + 1)) <= budget) ++level;
            std::vector<srt_vertex> v;
            std::vector<uint32_t> i;
            geom_icosphere(level, v, i);
            geom_displace(v, i, 0.05f, seed);
            uint32_t ico = b->add_mesh(v.data(), (uint32_t)v.size(), i.data(), (uint32_t)i.size());
            b->add_instance(ico, stone, mat4_mul(mat4_translation(-0.3f, -0.45f, -0.2f), mat4_scale(0.9f, 0.9f, 0.9f)));
            double used = 20.0 * std::pow(4.0, (double)level);
            geom_uv_sphere(64, 32, v, i);
            uint32_t ball = b->add_mesh(v.data(), (uint32_t)v.size(), i.data(), (uint32_t)i.size());
            const double per_ball = (double)(i.size() / 3);
            for (int k = 0; used + per_ball <= budget && k < 512; ++k, used += per_ball) {
                float kind = rnd();
                uint32_t m;
                if (kind < 0.4f) {
                    const float rough = 0.05f + 0.45f * rnd();
                    m = b->add_material(mat(0.9f, 0.8f, 0.7f, 1, 1, rough, 0, 0));
                } else if (kind < 0.8f) {
                    const float alpha = 0.05f + 0.45f * rnd();
                    const float film = 200.0f + 600.0f * rnd();
                    m = b->add_material(mat(1, 1, 1, alpha, 5, film, 1.33f, 1.5f));
                } else {
                    m = b->add_material(mat(1, 1, 1, 1, 2, 0, 1.5f, 0.0042f));
                }
                const float r = 0.05f + 0.1f * rnd();
                const float px = -0.85f + 1.7f * rnd();
                const float py = -1.0f + r + 1.2f * rnd();
                const float pz = -0.85f + 1.7f * rnd();
                b->add_instance(ball, m, mat4_mul(mat4_translation(px, py, pz), mat4_scale(2 * r, 2 * r, 2 * r)));
            }
            return true;
        }
        default:
            return false;
    }
}

// ------------------------------------------------------------------ camera (camera.rs:178-194)
static void inverse4(const float* m, float* out) {
    double a[16], inv[16];
    for (int i = 0; i < 16; ++i) a[i] = m[i];
    inv[0] = a[5] * a[10] * a[15] - a[5] * a[11] * a[14] - a[9] * a[6] * a[15] + a[9] * a[7] * a[14] +
             a[13] * a[6] * a[11] - a[13] * a[7] * a[10];
    inv[4] = -a[4] * a[10] * a[15] + a[4] * a[11] * a[14] + a[8] * a[6] * a[15] - a[8] * a[7] * a[14] -
             a[12] * a[6] * a[11] + a[12] * a[7] * a[10];
    inv[8] = a[4] * a[9] * a[15] - a[4] * a[11] * a[13] - a[8] * a[5] * a[15] + a[8] * a[7] * a[13] +
             a[12] * a[5] * a[11] - a[12] * a[7] * a[9];
    inv[12] = -a[4] * a[9] * a[14] + a[4] * a[10] * a[13] + a[8] * a[5] * a[14] - a[8] * a[6] * a[13] -
              a[12] * a[5] * a[10] + a[12] * a[6] * a[9];
    inv[1] = -a[1] * a[10] * a[15] + a[1] * a[11] * a[14] + a[9] * a[2] * a[15] - a[9] * a[3] * a[14] -
             a[13] * a[2] * a[11] + a[13] * a[3] * a[10];
    inv[5] = a[0] * a[10] * a[15] - a[0] * a[11] * a[14] - a[8] * a[2] * a[15] + a[8] * a[3] * a[14] +
             a[12] * a[2] * a[11] - a[12] * a[3] * a[10];
    inv[9] = -a[0] * a[9] * a[15] + a[0] * a[11] * a[13] + a[8] * a[1] * a[15] - a[8] * a[3] * a[13] -
             a[12] * a[1] * a[11] + a[12] * a[3] * a[9];
    inv[13] = a[0] * a[9] * a[14] - a[0] * a[10] * a[13] - a[8] * a[1] * a[14] + a[8] * a[2] * a[13] +
              a[12] * a[1] * a[10] - a[12] * a[2] * a[9];
    inv[2] = a[1] * a[6] * a[15] - a[1] * a[7] * a[14] - a[5] * a[2] * a[15] + a[5] * a[3] * a[14] +
             a[13] * a[2] * a[7] - a[13] * a[3] * a[6];
    inv[6] = -a[0] * a[6] * a[15] + a[0] * a[7] * a[14] + a[4] * a[2] * a[15] - a[4] * a[3] * a[14] -
             a[12] * a[2] * a[7] + a[12] * a[3] * a[6];
    inv[10] = a[0] * a[5] * a[15] - a[0] * a[7] * a[13] - a[4] * a[1] * a[15] + a[4] * a[3] * a[13] +
              a[12] * a[1] * a[7] - a[12] * a[3] * a[5];
    inv[14] = -a[0] * a[5] * a[14] + a[0] * a[6] * a[13] + a[4] * a[1] * a[14] - a[4] * a[2] * a[13] -
              a[12] * a[1] * a[6] + a[12] * a[2] * a[5];
    inv[3] = -a[1] * a[6] * a[11] + a[1] * a[7] * a[10] + a[5] * a[2] * a[11] - a[5] * a[3] * a[10] -
             a[9] * a[2] * a[7] + a[9] * a[3] * a[6];
    inv[7] = a[0] * a[6] * a[11] - a[0] * a[7] * a[10] - a[4] * a[2] * a[11] + a[4] * a[3] * a[10] +
             a[8] * a[2] * a[7] - a[8] * a[3] * a[6];
    inv[11] = -a[0] * a[5] * a[11] + a[0] * a[7] * a[9] + a[4] * a[1] * a[11] - a[4] * a[3] * a[9] -
              a[8] * a[1] * a[7] + a[8] * a[3] * a[5];
    inv[15] = a[0] * a[5] * a[10] - a[0] * a[6] * a[9] - a[4] * a[1] * a[10] + a[4] * a[2] * a[9] +
              a[8] * a[1] * a[6] - a[8] * a[2] * a[5];
    double det = a[0] * inv[0] + a[1] * inv[4] + a[2] * inv[8] + a[3] * inv[12];
    for (int i = 0; i < 16; ++i) out[i] = (float)(inv[i] / det);
}

void camera_build_uniform(const float pos[3], float yaw, float pitch, float aspect, uint32_t frame,
                          srt_camera_uniform* out) {
    float sy = std::sin(yaw), cy = std::cos(yaw), sp = std::sin(pitch), cp = std::cos(pitch);
    float f[3] = {cp * cy, sp, cp * sy};
    float fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    for (float& x : f) x /= fl;
    // look_at_rh(eye, eye + forward, +Y) = look_to_rh(eye, forward, +Y)
    float up[3] = {0, 1, 0};
    float s[3] = {f[1] * up[2] - f[2] * up[1], f[2] * up[0] - f[0] * up[2], f[0] * up[1] - f[1] * up[0]};
    float sl = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    for (float& x : s) x /= sl;
    float u[3] = {s[1] * f[2] - s[2] * f[1], s[2] * f[0] - s[0] * f[2], s[0] * f[1] - s[1] * f[0]};
    float view[16] = {s[0], u[0], -f[0], 0, s[1], u[1], -f[1], 0, s[2], u[2], -f[2], 0,
                      -(pos[0] * s[0] + pos[1] * s[1] + pos[2] * s[2]),
                      -(pos[0] * u[0] + pos[1] * u[1] + pos[2] * u[2]),
                      pos[0] * f[0] + pos[1] * f[1] + pos[2] * f[2], 1};
    // perspective_rh(45 deg, aspect, 0.1, 100), depth range [0, 1]
    const float fov = 45.0f * 3.14159265358979f / 180.0f, zn = 0.1f, zf = 100.0f;
    float sf = std::sin(0.5f * fov), cf = std::cos(0.5f * fov);
    float h = cf / sf, w = h / aspect, r = zf / (zn - zf);
    float proj[16] = {w, 0, 0, 0, 0, h, 0, 0, 0, 0, r, -1, 0, 0, r * zn, 0};
    std::memset(out, 0, sizeof(*out));
    std::memcpy(out->view, view, 64);
    std::memcpy(out->proj, proj, 64);
    inverse4(view, out->view_inverse);
    inverse4(proj, out->proj_inverse);
    out->frame_count = frame;
}

// ------------------------------------------------------------------ screenshot (screenshot.rs:27-103)
uint8_t srgb_oetf_u8(uint8_t c) {
    // screenshot.rs:55-63: the stored value is linear; apply the sRGB OETF
    float cf = (float)c / 255.0f;
    float s = cf <= 0.0031308f ? cf * 12.92f : 1.055f * std::pow(cf, 1.0f / 2.4f) - 0.055f;
    s = std::min(std::max(s, 0.0f), 1.0f) * 255.0f;
    return (uint8_t)std::round(s);
}

namespace {
uint32_t crc_table[256];
bool crc_init = false;
uint32_t crc32(const uint8_t* p, size_t n, uint32_t c = 0xFFFFFFFFu) {
    if (!crc_init) {
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t x = i;
            for (int k = 0; k < 8; ++k) x = (x & 1) ? 0xEDB88320u ^ (x >> 1) : x >> 1;
            crc_table[i] = x;
        }
        crc_init = true;
    }
    for (size_t i = 0; i < n; ++i) c = crc_table[(c ^ p[i]) & 0xFF] ^ (c >> 8);
    return c;
}
void put32(std::vector<uint8_t>& o, uint32_t v) {
    o.push_back(v >> 24);
    o.push_back(v >> 16);
    o.push_back(v >> 8);
    o.push_back(v);
}
void chunk(std::vector<uint8_t>& out, const char* type, const std::vector<uint8_t>& data) {
    put32(out, (uint32_t)data.size());
    size_t start = out.size();
    out.insert(out.end(), type, type + 4);
    out.insert(out.end(), data.begin(), data.end());
    put32(out, crc32(out.data() + start, out.size() - start) ^ 0xFFFFFFFFu);
}
}  // namespace

bool write_screenshot_png(const std::string& path, const uint8_t* rgba, uint32_t w, uint32_t h, uint32_t pitch) {
    // filter-0 scanlines, top row first (the source rows are bottom-up)
    std::vector<uint8_t> raw;
    raw.reserve((size_t)h * (4 * w + 1));
    for (uint32_t r = 0; r < h; ++r) {
        const uint8_t* src = rgba + (size_t)(h - 1 - r) * pitch;
        raw.push_back(0);
        for (uint32_t x = 0; x < w; ++x) {
            raw.push_back(srgb_oetf_u8(src[4 * x]));
            raw.push_back(srgb_oetf_u8(src[4 * x + 1]));
            raw.push_back(srgb_oetf_u8(src[4 * x + 2]));
            raw.push_back(255);
        }
    }
    // zlib stream of stored deflate blocks
    std::vector<uint8_t> z = {0x78, 0x01};
    size_t pos = 0;
    do {
        size_t n = std::min<size_t>(65535, raw.size() - pos);
        bool last = pos + n == raw.size();
        z.push_back(last ? 1 : 0);
        z.push_back(n & 0xFF);
        z.push_back(n >> 8);
        z.push_back(~n & 0xFF);
        z.push_back((~n >> 8) & 0xFF);
        z.insert(z.end(), raw.begin() + pos, raw.begin() + pos + n);
        pos += n;
    } while (pos < raw.size());
    uint32_t a = 1, b = 0;
    for (uint8_t c : raw) {
        a = (a + c) % 65521u;
        b = (b + a) % 65521u;
    }
    put32(z, (b << 16) | a);
    std::vector<uint8_t> png = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n'};
    std::vector<uint8_t> ihdr;
    put32(ihdr, w);
    put32(ihdr, h);
    ihdr.insert(ihdr.end(), {8, 6, 0, 0, 0});
    chunk(png, "IHDR", ihdr);
    chunk(png, "IDAT", z);
    chunk(png, "IEND", {});
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    bool ok = std::fwrite(png.data(), 1, png.size(), f) == png.size();
    std::fclose(f);
    return ok;
}
