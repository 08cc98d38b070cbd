/*
 * scenes.cpp — the oracle's own scene generator.  TEST INFRASTRUCTURE ONLY.
 *
 * Builds the scene arrays (vertices, indices, mesh infos, materials,
 * instances, light triangles) and the camera uniform of every preset without
 * the product library, so that the CPU baseline and the tests get their
 * inputs from code that is independent of what they check.  A CPU test
 * compares these arrays with the product's, byte for byte.
 *
 * Restated from the reference:
 *   plane, cube, icosphere          src/scene/geometry.rs:12-232
 *   light triangles of a light      src/scene/builder.rs:101-129
 *   Cornell box                     src/scene/cornell_box.rs:6-110
 *   prism scene                     src/scene/custom.rs:6-116
 *   camera uniform                  src/scene/camera.rs:178-194 (look_at_rh,
 *                                   perspective_rh(45 deg, aspect, 0.1, 100))
 * Restated from this project's definitions of its synthetic workloads (no
 * reference counterpart): the latitude-longitude sphere, the value-noise
 * displacement of the icosphere, and the config-1, config-2, caustic-slab,
 * indirect-room and seeded batch scenes.
 *
 * Every float operation is written in the order the definitions give, so the
 * arrays match bit for bit; the camera inverses are computed in closed form
 * (rigid view, diagonal-plus-corner projection) and agree to rounding only.
 */
#include <cmath>
#include <cstring>
#include <map>
#include <utility>
#include <vector>

#include "oracle.h"

namespace {

// ---------------------------------------------------------------- 4x4 affine (column-major, glam order)
struct M4 {
    float c[16];
};

M4 ident() {
    M4 m{};
    m.c[0] = m.c[5] = m.c[10] = m.c[15] = 1.0f;
    return m;
}
// a * b; each entry summed left to right like glam's Mat4 * Mat4
M4 operator*(const M4& a, const M4& b) {
    M4 r{};
    for (int col = 0; col < 4; ++col)
        for (int row = 0; row < 4; ++row) {
            float acc = a.c[row] * b.c[4 * col];
            acc = acc + a.c[4 + row] * b.c[4 * col + 1];
            acc = acc + a.c[8 + row] * b.c[4 * col + 2];
            acc = acc + a.c[12 + row] * b.c[4 * col + 3];
            r.c[4 * col + row] = acc;
        }
    return r;
}
M4 translate(float x, float y, float z) {
    M4 m = ident();
    m.c[12] = x;
    m.c[13] = y;
    m.c[14] = z;
    return m;
}
M4 scale(float x, float y, float z) {
    M4 m{};
    m.c[0] = x;
    m.c[5] = y;
    m.c[10] = z;
    m.c[15] = 1.0f;
    return m;
}
M4 scale(float s) { return scale(s, s, s); }
// glam Mat4::from_rotation_{x,y,z}
M4 rot(int axis, float a) {
    float s = std::sin(a), c = std::cos(a);
    M4 m = ident();
    int i = (axis + 1) % 3, j = (axis + 2) % 3;  // the rotated plane (i -> j)
    m.c[4 * i + i] = c;
    m.c[4 * i + j] = s;
    m.c[4 * j + i] = -s;
    m.c[4 * j + j] = c;
    return m;
}

const float kPi = 3.14159265358979f;   // std::f32::consts::PI
const float kPi2 = 1.57079632679490f;  // std::f32::consts::FRAC_PI_2

uint32_t pcg(uint32_t v) {  // PCG-RXS-M-XS, the hash the project seeds its scenes with
    uint32_t state = v * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}

// ---------------------------------------------------------------- meshes
struct Mesh {
    std::vector<srt_vertex> v;
    std::vector<uint32_t> i;
};

srt_vertex vert(float px, float py, float pz, float nx, float ny, float nz) {
    srt_vertex x{};
    x.pos[0] = px;
    x.pos[1] = py;
    x.pos[2] = pz;
    x.pos[3] = 1.0f;
    x.normal[0] = nx;
    x.normal[1] = ny;
    x.normal[2] = nz;
    x.normal[3] = 0.0f;
    return x;
}

Mesh plane() {  // geometry.rs:12-35: unit quad in the xz plane, normal +y
    Mesh m;
    const float q[4][2] = {{-0.5f, 0.5f}, {0.5f, 0.5f}, {-0.5f, -0.5f}, {0.5f, -0.5f}};
    for (auto& p : q) m.v.push_back(vert(p[0], 0.0f, p[1], 0.0f, 1.0f, 0.0f));
    m.i = {0, 1, 2, 2, 1, 3};
    return m;
}

Mesh cube() {  // geometry.rs:38-126: 6 faces x 4 vertices, two triangles each
    // per face: normal axis and sign, then the four corners as +-1 patterns
    // of (x, y, z) * 0.5 in the reference's order
    static const int faces[6][3 + 12] = {
        {0, 0, 1, -1, -1, 1, 1, -1, 1, 1, 1, 1, -1, 1, 1},
        {0, 0, -1, 1, -1, -1, -1, -1, -1, -1, 1, -1, 1, 1, -1},
        {0, 1, 0, -1, 1, 1, 1, 1, 1, 1, 1, -1, -1, 1, -1},
        {0, -1, 0, -1, -1, -1, 1, -1, -1, 1, -1, 1, -1, -1, 1},
        {1, 0, 0, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, 1, 1},
        {-1, 0, 0, -1, -1, -1, -1, -1, 1, -1, 1, 1, -1, 1, -1},
    };
    Mesh m;
    for (int f = 0; f < 6; ++f) {
        const int* F = faces[f];
        uint32_t base = (uint32_t)m.v.size();
        for (int k = 0; k < 4; ++k)
            m.v.push_back(vert(0.5f * (float)F[3 + 3 * k], 0.5f * (float)F[4 + 3 * k], 0.5f * (float)F[5 + 3 * k],
                               (float)F[0], (float)F[1], (float)F[2]));
        const uint32_t tri[6] = {0, 1, 2, 0, 2, 3};
        for (uint32_t t : tri) m.i.push_back(base + t);
    }
    return m;
}

// geometry.rs:129-232: icosahedron on the sphere of radius 0.5, each
// subdivision splits every face into four through cached edge midpoints
Mesh icosphere(uint32_t subdivisions) {
    Mesh m;
    auto push_unit = [&](float x, float y, float z) {
        float len = std::sqrt(x * x + y * y + z * z);
        float nx = x / len, ny = y / len, nz = z / len;
        m.v.push_back(vert(nx * 0.5f, ny * 0.5f, nz * 0.5f, nx, ny, nz));
        return (uint32_t)(m.v.size() - 1);
    };
    const float g = (1.0f + std::sqrt(5.0f)) / 2.0f;
    // (a, b) with a = +-1, b = +-g on the three cyclic coordinate planes
    const float base[12][3] = {{-1, g, 0}, {1, g, 0}, {-1, -g, 0}, {1, -g, 0}, {0, -1, g},  {0, 1, g},
                               {0, -1, -g}, {0, 1, -g}, {g, 0, -1}, {g, 0, 1},  {-g, 0, -1}, {-g, 0, 1}};
    for (auto& p : base) push_unit(p[0], p[1], p[2]);
    std::vector<uint32_t> tris = {0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4,
                                  11, 10, 2, 10, 7, 6, 7, 1, 8, 3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8,
                                  3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1};
    std::map<std::pair<uint32_t, uint32_t>, uint32_t> mid;
    auto midpoint = [&](uint32_t a, uint32_t b) {
        std::pair<uint32_t, uint32_t> key = a < b ? std::make_pair(a, b) : std::make_pair(b, a);
        auto it = mid.find(key);
        if (it != mid.end()) return it->second;
        const float* p = m.v[a].pos;
        const float* q = m.v[b].pos;
        float x = (p[0] + q[0]) * 0.5f, y = (p[1] + q[1]) * 0.5f, z = (p[2] + q[2]) * 0.5f;
        uint32_t id = push_unit(x, y, z);
        mid[key] = id;
        return id;
    };
    for (uint32_t level = 0; level < subdivisions; ++level) {
        std::vector<uint32_t> out;
        out.reserve(tris.size() * 4);
        for (size_t f = 0; f < tris.size(); f += 3) {
            uint32_t p = tris[f], q = tris[f + 1], r = tris[f + 2];
            uint32_t pq = midpoint(p, q), qr = midpoint(q, r), rp = midpoint(r, p);
            for (uint32_t x : {p, pq, rp, q, qr, pq, r, rp, qr, pq, qr, rp}) out.push_back(x);
        }
        tris.swap(out);
    }
    m.i = tris;
    return m;
}

// Latitude-longitude sphere of radius 0.5: rings from the +y pole (ring 0)
// to the -y pole, slices + 1 vertices per ring (seam repeated); the top band
// is a fan, every other band two triangles per quad (the bottom band's are
// degenerate): slices * (2 * stacks - 1) triangles.
Mesh uv_sphere(uint32_t slices, uint32_t stacks) {
    Mesh m;
    const double pi = 3.14159265358979323846;
    for (uint32_t r = 0; r <= stacks; ++r) {
        double theta = pi * r / stacks;
        for (uint32_t s = 0; s <= slices; ++s) {
            double phi = 2.0 * pi * s / slices;
            float nx = (float)(std::sin(theta) * std::cos(phi));
            float ny = (float)std::cos(theta);
            float nz = (float)(-std::sin(theta) * std::sin(phi));
            m.v.push_back(vert(0.5f * nx, 0.5f * ny, 0.5f * nz, nx, ny, nz));
        }
    }
    const uint32_t w = slices + 1;
    for (uint32_t r = 0; r < stacks; ++r)
        for (uint32_t s = 0; s < slices; ++s) {
            uint32_t a = r * w + s, b = a + 1, c = a + w, d = c + 1;
            if (r == 0) {
                m.i.insert(m.i.end(), {a, c, d});
            } else {
                m.i.insert(m.i.end(), {a, c, d, a, d, b});
            }
        }
    return m;
}

// Value noise on the integer lattice: corner values from nested PCG hashes of
// the lattice coordinates (spatial-hash primes) and the seed, in [-1, 1];
// smoothstep-weighted trilinear blend.
float lattice_value(int x, int y, int z, uint32_t seed) {
    uint32_t h = pcg((uint32_t)z * 83492791u ^ seed);
    h = pcg((uint32_t)y * 19349663u ^ h);
    h = pcg((uint32_t)x * 73856093u ^ h);
    return (float)(h >> 8) * (2.0f / 16777215.0f) - 1.0f;
}
float noise3(float x, float y, float z, uint32_t seed) {
    float fx0 = std::floor(x), fy0 = std::floor(y), fz0 = std::floor(z);
    int x0 = (int)fx0, y0 = (int)fy0, z0 = (int)fz0;
    auto fade = [](float t) { return t * t * (3.0f - 2.0f * t); };
    float u = fade(x - x0), v = fade(y - y0), w = fade(z - z0);
    auto mix = [](float a, float b, float t) { return a + (b - a) * t; };
    float c000 = lattice_value(x0, y0, z0, seed), c100 = lattice_value(x0 + 1, y0, z0, seed);
    float c010 = lattice_value(x0, y0 + 1, z0, seed), c110 = lattice_value(x0 + 1, y0 + 1, z0, seed);
    float c001 = lattice_value(x0, y0, z0 + 1, seed), c101 = lattice_value(x0 + 1, y0, z0 + 1, seed);
    float c011 = lattice_value(x0, y0 + 1, z0 + 1, seed), c111 = lattice_value(x0 + 1, y0 + 1, z0 + 1, seed);
    float y0z0 = mix(c000, c100, u), y1z0 = mix(c010, c110, u);
    float y0z1 = mix(c001, c101, u), y1z1 = mix(c011, c111, u);
    return mix(mix(y0z0, y1z0, v), mix(y0z1, y1z1, v), w);
}

// Radial displacement r = 0.5 + amplitude * fbm(unit normal), fbm = three
// octaves (frequency 4, 8, 16; weights 1, 1/2, 1/4; divided by their sum),
// then area-weighted vertex normals accumulated in FP64.
void displace(Mesh& m, float amplitude, uint32_t seed) {
    for (srt_vertex& x : m.v) {
        const float n0 = x.normal[0], n1 = x.normal[1], n2 = x.normal[2];
        float freq = 4.0f, weight = 1.0f, total = 0.0f, wsum = 0.0f;
        for (uint32_t octave = 0; octave < 3; ++octave) {
            total += weight * noise3(n0 * freq, n1 * freq, n2 * freq, seed + 0x9E3779B9u * octave);
            wsum += weight;
            freq *= 2.0f;
            weight *= 0.5f;
        }
        const float r = 0.5f + amplitude * (total / wsum);
        x.pos[0] = n0 * r;
        x.pos[1] = n1 * r;
        x.pos[2] = n2 * r;
    }
    std::vector<double> nsum(3 * m.v.size(), 0.0);
    for (size_t f = 0; f + 2 < m.i.size(); f += 3) {
        const float* a = m.v[m.i[f]].pos;
        const float* b = m.v[m.i[f + 1]].pos;
        const float* c = m.v[m.i[f + 2]].pos;
        const double ux = (double)b[0] - a[0], uy = (double)b[1] - a[1], uz = (double)b[2] - a[2];
        const double vx = (double)c[0] - a[0], vy = (double)c[1] - a[1], vz = (double)c[2] - a[2];
        const double cx = uy * vz - uz * vy, cy = uz * vx - ux * vz, cz = ux * vy - uy * vx;
        for (int k = 0; k < 3; ++k) {
            double* s = &nsum[3 * (size_t)m.i[f + k]];
            s[0] += cx;
            s[1] += cy;
            s[2] += cz;
        }
    }
    for (size_t k = 0; k < m.v.size(); ++k) {
        const double* s = &nsum[3 * k];
        double len = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
        if (len > 0.0)
            for (int c = 0; c < 3; ++c) m.v[k].normal[c] = (float)(s[c] / len);
    }
}

}  // namespace

// ---------------------------------------------------------------- the builder (builder.rs:47-129)
struct orc_preset {
    std::vector<srt_vertex> vertices;
    std::vector<uint32_t> indices;
    std::vector<srt_mesh_info> meshes;
    std::vector<uint32_t> mesh_tri_count;
    std::vector<srt_material> materials;
    std::vector<srt_instance> instances;
    std::vector<srt_light> lights;
    float camera[5];

    uint32_t material(float r, float g, float b, float a, float e0, float e1, float e2, float e3) {
        srt_material x;
        const float v[8] = {r, g, b, a, e0, e1, e2, e3};
        std::memcpy(x.color, v, 16);
        std::memcpy(x.extra, v + 4, 16);
        materials.push_back(x);
        return (uint32_t)materials.size() - 1;
    }
    uint32_t mesh(const Mesh& m) {
        srt_mesh_info info{};
        info.vertex_offset = (uint32_t)vertices.size();
        info.index_offset = (uint32_t)indices.size();
        meshes.push_back(info);
        mesh_tri_count.push_back((uint32_t)(m.i.size() / 3));
        vertices.insert(vertices.end(), m.v.begin(), m.v.end());
        indices.insert(indices.end(), m.i.begin(), m.i.end());
        return (uint32_t)meshes.size() - 1;
    }
    void instance(uint32_t mesh_id, uint32_t mat_id, const M4& t) {
        srt_instance x{};
        x.mesh_id = mesh_id;
        x.mat_id = mat_id;
        std::memcpy(x.transform, t.c, 64);
        instances.push_back(x);
    }
    // builder.rs:101-129: the instance plus one world-space light triangle
    // per mesh triangle (transform * (v, 1), summed like glam's Mat4 * Vec4)
    void light(uint32_t mesh_id, uint32_t mat_id, const M4& t, const float params[4]) {
        instance(mesh_id, mat_id, t);
        const srt_mesh_info& info = meshes[mesh_id];
        for (uint32_t k = 0; k < mesh_tri_count[mesh_id]; ++k) {
            srt_light L{};
            float* corner[3] = {L.v0, L.v1, L.v2};
            for (int c = 0; c < 3; ++c) {
                const float* p = vertices[info.vertex_offset + indices[info.index_offset + 3 * k + c]].pos;
                for (int row = 0; row < 3; ++row) {
                    float acc = t.c[row] * p[0];
                    acc = acc + t.c[4 + row] * p[1];
                    acc = acc + t.c[8 + row] * p[2];
                    acc = acc + t.c[12 + row] * 1.0f;
                    corner[c][row] = acc;
                }
                corner[c][3] = 1.0f;
            }
            std::memcpy(L.params, params, 16);
            lights.push_back(L);
        }
    }
};

namespace {

void room_walls(orc_preset& s, uint32_t plane_m, uint32_t floor_ceil_back, uint32_t left, uint32_t right) {
    // cornell_box.rs:46-85: floor, ceiling, back wall, left, right (plane scaled 2)
    const M4 s2 = scale(2.0f);
    s.instance(plane_m, floor_ceil_back, translate(0, -1, 0) * s2);
    s.instance(plane_m, floor_ceil_back, translate(0, 1, 0) * rot(0, kPi) * s2);
    s.instance(plane_m, floor_ceil_back, translate(0, 0, -1) * rot(0, kPi2) * s2);
    s.instance(plane_m, left, translate(-1, 0, 0) * rot(2, -kPi2) * s2);
    s.instance(plane_m, right, translate(1, 0, 0) * rot(2, kPi2) * s2);
}

bool fill(orc_preset& s, int preset, uint32_t seed) {
    // camera.rs:38-40: position (0, 0, 3), yaw -90 degrees, pitch 0
    const float cam0[5] = {0.0f, 0.0f, 3.0f, -kPi2, 0.0f};
    std::memcpy(s.camera, cam0, sizeof(cam0));
    switch (preset) {
        case SRT_PRESET_CORNELL_BOX: {  // cornell_box.rs:6-110
            uint32_t m_light = s.material(6500, 1, 0, 1, 3, 0, 0, 0);
            uint32_t m_red = s.material(0.65f, 0.05f, 0.05f, 1, 0, 0, 0, 0);
            uint32_t m_green = s.material(0.12f, 0.45f, 0.15f, 1, 0, 0, 0, 0);
            uint32_t m_white = s.material(0.73f, 0.73f, 0.73f, 1, 0, 0, 0, 0);
            uint32_t m_glass = s.material(1, 1, 1, 1, 2, 0, 1.5f, 0.01f);
            uint32_t m_bubble = s.material(1, 1, 1, 1, 4, 500.0f, 1.33f, 1.0f);
            uint32_t g_plane = s.mesh(plane()), g_cube = s.mesh(cube()), g_sphere = s.mesh(icosphere(4));
            room_walls(s, g_plane, m_white, m_red, m_green);
            const float lp[4] = {0.0f, 6500.0f, 1.0f, 0.0f};
            s.light(g_plane, m_light, translate(0, 0.99f, 0) * rot(0, kPi) * scale(0.5f), lp);
            s.instance(g_cube, m_glass, translate(-0.35f, -0.4f + 0.002f, -0.3f) * rot(1, 0.4f) * scale(0.6f, 1.2f, 0.6f));
            s.instance(g_sphere, m_bubble, translate(0.4f, -0.64f, 0.3f) * scale(0.75f));
            return true;
        }
        case SRT_PRESET_CUSTOM_PRISM: {  // custom.rs:6-116
            uint32_t m_light = s.material(6500, 5, 0, 1, 3, 0, 0, 0);
            uint32_t m_wall = s.material(0.01f, 0.01f, 0.01f, 1, 0, 0, 0, 0);
            uint32_t m_canvas = s.material(0.95f, 0.95f, 0.95f, 1, 0, 0, 0, 0);
            uint32_t m_prism = s.material(1, 1, 1, 1, 2, 0, 1.6f, 0.12f);
            uint32_t m_bubble = s.material(1, 1, 1, 1, 4, 500.0f, 1.33f, 1.0f);
            uint32_t g_plane = s.mesh(plane()), g_cube = s.mesh(cube()), g_sphere = s.mesh(icosphere(4));
            const float room = 4.0f;
            const M4 sr = scale(room * 2.0f);
            s.instance(g_plane, m_wall, translate(0, -1, 0) * sr);
            s.instance(g_plane, m_wall, translate(0, room - 1.0f, 0) * rot(0, kPi) * sr);
            s.instance(g_plane, m_wall, translate(0, room * 0.5f - 1.0f, -room) * rot(0, kPi2) * sr);
            s.instance(g_cube, m_canvas, translate(0.5f, -0.55f, 0) * scale(5, 0.1f, 3));
            const float lp[4] = {0.0f, 6500.0f, 5.0f, 0.0f};
            s.light(g_plane, m_light, translate(-2.0f, -0.2f, 0) * rot(2, -kPi2 + 0.02f) * scale(0.5f, 1.0f, 0.02f), lp);
            s.instance(g_cube, m_prism, translate(-1.1f, -0.2f, 0) * rot(1, 0.7f) * scale(0.5f, 0.8f, 0.5f));
            s.instance(g_sphere, m_bubble, translate(1.0f, -0.1f, -0.5f) * scale(0.6f));
            return true;
        }
        case SRT_PRESET_CONFIG1: {
            // Cornell walls + 2-triangle 6500 K light + dispersive UV sphere
            // (64 x 32, Cauchy A = 1.5, B = 0.0042 um^2)
            uint32_t m_light = s.material(6500, 1, 0, 1, 3, 0, 0, 0);
            uint32_t m_red = s.material(0.65f, 0.05f, 0.05f, 1, 0, 0, 0, 0);
            uint32_t m_green = s.material(0.12f, 0.45f, 0.15f, 1, 0, 0, 0, 0);
            uint32_t m_white = s.material(0.73f, 0.73f, 0.73f, 1, 0, 0, 0, 0);
            uint32_t m_glass = s.material(1, 1, 1, 1, 2, 0, 1.5f, 0.0042f);
            uint32_t g_plane = s.mesh(plane()), g_sphere = s.mesh(uv_sphere(64, 32));
            room_walls(s, g_plane, m_white, m_red, m_green);
            const float lp[4] = {0.0f, 6500.0f, 1.0f, 0.0f};
            s.light(g_plane, m_light, translate(0, 0.99f, 0) * rot(0, kPi) * scale(0.5f), lp);
            s.instance(g_sphere, m_glass, translate(0.0f, -0.548f, 0.0f) * scale(0.9f));
            return true;
        }
        case SRT_PRESET_CONFIG2: {
            // level-8 icosphere displaced by value noise (amplitude 0.05) +
            // 64 thin-film-coated GGX spheres on two rings (22 + 42) in an
            // 8 x 4 x 8 room under a 1.5 x 1.5 light
            uint32_t m_light = s.material(6500, 3, 0, 1, 3, 0, 0, 0);
            uint32_t m_red = s.material(0.65f, 0.05f, 0.05f, 1, 0, 0, 0, 0);
            uint32_t m_green = s.material(0.12f, 0.45f, 0.15f, 1, 0, 0, 0, 0);
            uint32_t m_white = s.material(0.73f, 0.73f, 0.73f, 1, 0, 0, 0, 0);
            uint32_t m_stone = s.material(0.8f, 0.75f, 0.7f, 1, 0, 0, 0, 0);
            uint32_t g_plane = s.mesh(plane());
            Mesh ico = icosphere(8);
            displace(ico, 0.05f, seed);
            uint32_t g_ico = s.mesh(ico);
            uint32_t g_ball = s.mesh(uv_sphere(64, 32));
            const M4 s8 = scale(8.0f);
            s.instance(g_plane, m_white, translate(0, -1, 0) * s8);
            s.instance(g_plane, m_white, translate(0, 3, 0) * rot(0, kPi) * s8);
            s.instance(g_plane, m_white, translate(0, 1, -4) * rot(0, kPi2) * s8);
            s.instance(g_plane, m_red, translate(-4, 1, 0) * rot(2, -kPi2) * s8);
            s.instance(g_plane, m_green, translate(4, 1, 0) * rot(2, kPi2) * s8);
            const float lp[4] = {0.0f, 6500.0f, 3.0f, 0.0f};
            s.light(g_plane, m_light, translate(0, 2.99f, -0.5f) * rot(0, kPi) * scale(1.5f), lp);
            s.instance(g_ico, m_stone, translate(0, 0.2f, -1.0f) * scale(2.4f));
            uint32_t state = seed * 2654435761u + 12345u;
            auto uniform01 = [&]() {
                state = pcg(state);
                return (float)state / 4294967296.0f;
            };
            const int per_ring[2] = {22, 42};
            const float ring_r[2] = {1.75f, 2.75f};
            const float ball_r = 0.18f;
            for (int ring = 0; ring < 2; ++ring)
                for (int k = 0; k < per_ring[ring]; ++k) {
                    float ang = 2.0f * kPi * ((float)k + 0.5f * (float)ring) / (float)per_ring[ring];
                    float alpha = 0.05f + 0.45f * uniform01();
                    float film = 200.0f + 600.0f * uniform01();
                    uint32_t m = s.material(1, 1, 1, alpha, 5, film, 1.33f, 1.5f);
                    s.instance(g_ball, m,
                               translate(ring_r[ring] * std::cos(ang), -1.0f + ball_r, -1.0f + ring_r[ring] * std::sin(ang)) *
                                   scale(2 * ball_r));
                }
            const float cam[5] = {0.0f, 1.0f, 6.0f, -kPi2, -0.12f};
            std::memcpy(s.camera, cam, sizeof(cam));
            return true;
        }
        case SRT_PRESET_CAUSTIC_SLAB: {
            // dispersive slab (A = 1.5, B = 0.01 um^2) under a 0.05-wide slit
            // light above a diffuse floor, beside the config-1 sphere mesh
            uint32_t m_light = s.material(6500, 40, 0, 1, 3, 0, 0, 0);
            uint32_t m_floor = s.material(0.8f, 0.8f, 0.8f, 1, 0, 0, 0, 0);
            uint32_t m_wall = s.material(0.3f, 0.3f, 0.3f, 1, 0, 0, 0, 0);
            uint32_t m_glass = s.material(1, 1, 1, 1, 2, 0, 1.5f, 0.01f);
            uint32_t m_stone = s.material(0.6f, 0.5f, 0.4f, 1, 0, 0, 0, 0);
            uint32_t g_plane = s.mesh(plane()), g_cube = s.mesh(cube()), g_sphere = s.mesh(uv_sphere(64, 32));
            room_walls(s, g_plane, m_floor, m_wall, m_wall);
            const float lp[4] = {0.0f, 6500.0f, 40.0f, 0.0f};
            s.light(g_plane, m_light, translate(-0.3f, 0.99f, 0) * rot(0, kPi) * scale(0.05f, 1.0f, 1.2f), lp);
            s.instance(g_cube, m_glass, translate(-0.2f, 0.3f, 0.0f) * rot(2, 0.35f) * scale(0.9f, 0.12f, 1.0f));
            s.instance(g_sphere, m_stone, translate(0.5f, -0.65f, -0.3f) * scale(0.7f));
            return true;
        }
        case SRT_PRESET_INDIRECT_ROOM: {
            // Cornell walls, a 0.3 x 0.3 light facing the ceiling behind a
            // 0.5 x 0.5 panel, one box
            uint32_t m_light = s.material(6500, 8, 0, 1, 3, 0, 0, 0);
            uint32_t m_red = s.material(0.65f, 0.05f, 0.05f, 1, 0, 0, 0, 0);
            uint32_t m_green = s.material(0.12f, 0.45f, 0.15f, 1, 0, 0, 0, 0);
            uint32_t m_white = s.material(0.73f, 0.73f, 0.73f, 1, 0, 0, 0, 0);
            uint32_t g_plane = s.mesh(plane()), g_cube = s.mesh(cube());
            room_walls(s, g_plane, m_white, m_red, m_green);
            const float lp[4] = {0.0f, 6500.0f, 8.0f, 0.0f};
            s.light(g_plane, m_light, translate(0, 0.95f, 0) * scale(0.3f), lp);
            s.instance(g_cube, m_white, translate(0, 0.93f, 0) * scale(0.5f, 0.02f, 0.5f));
            s.instance(g_cube, m_white, translate(-0.35f, -0.6f, -0.3f) * rot(1, 0.4f) * scale(0.5f, 0.8f, 0.5f));
            return true;
        }
        case SRT_PRESET_BATCH_RANDOM: {
            // seeded scene of the batched workloads: a triangle budget
            // log-uniform in [1e4, 2e6]; Cornell walls, a 0.6 light, the
            // largest displaced icosphere (level 4..8) within the budget, then
            // 64 x 32 UV spheres (GGX, coated GGX or dispersive glass) until
            // the budget or 512 spheres
            uint32_t state = pcg(seed * 747796405u + 2891336453u);
            auto uniform01 = [&]() {
                state = pcg(state);
                return (float)state / 4294967296.0f;
            };
            const double budget = std::exp(std::log(1e4) + uniform01() * (std::log(2e6) - std::log(1e4)));
            uint32_t m_light = s.material(6500, 2, 0, 1, 3, 0, 0, 0);
            uint32_t m_red = s.material(0.65f, 0.05f, 0.05f, 1, 0, 0, 0, 0);
            uint32_t m_green = s.material(0.12f, 0.45f, 0.15f, 1, 0, 0, 0, 0);
            uint32_t m_white = s.material(0.73f, 0.73f, 0.73f, 1, 0, 0, 0, 0);
            float sr = 0.3f + 0.5f * uniform01();
            float sg = 0.3f + 0.5f * uniform01();
            float sb = 0.3f + 0.5f * uniform01();
            uint32_t m_stone = s.material(sr, sg, sb, 1, 0, 0, 0, 0);
            uint32_t g_plane = s.mesh(plane());
            room_walls(s, g_plane, m_white, m_red, m_green);
            const float lp[4] = {0.0f, 6500.0f, 2.0f, 0.0f};
            s.light(g_plane, m_light, translate(0, 0.99f, 0) * rot(0, kPi) * scale(0.6f), lp);
            uint32_t level = 4;
            while (level < 8 && 20.0 * std::pow(4.0, (double)(level + 1)) <= budget) ++level;
            Mesh ico = icosphere(level);
            displace(ico, 0.05f, seed);
            uint32_t g_ico = s.mesh(ico);
            s.instance(g_ico, m_stone, translate(-0.3f, -0.45f, -0.2f) * scale(0.9f));
            double used = 20.0 * std::pow(4.0, (double)level);
            Mesh ball = uv_sphere(64, 32);
            const double per_ball = (double)(ball.i.size() / 3);
            uint32_t g_ball = s.mesh(ball);
            for (int k = 0; used + per_ball <= budget && k < 512; ++k, used += per_ball) {
                float kind = uniform01();
                uint32_t m;
                if (kind < 0.4f) {
                    float rough = 0.05f + 0.45f * uniform01();
                    m = s.material(0.9f, 0.8f, 0.7f, 1, 1, rough, 0, 0);
                } else if (kind < 0.8f) {
                    float alpha = 0.05f + 0.45f * uniform01();
                    float film = 200.0f + 600.0f * uniform01();
                    m = s.material(1, 1, 1, alpha, 5, film, 1.33f, 1.5f);
                } else {
                    m = s.material(1, 1, 1, 1, 2, 0, 1.5f, 0.0042f);
                }
                float r = 0.05f + 0.1f * uniform01();
                float px = -0.85f + 1.7f * uniform01();
                float py = -1.0f + r + 1.2f * uniform01();
                float pz = -0.85f + 1.7f * uniform01();
                s.instance(g_ball, m, translate(px, py, pz) * scale(2 * r));
            }
            return true;
        }
        default:
            return false;
    }
}

}  // namespace

orc_preset* orc_preset_create(int preset, uint32_t seed) {
    orc_preset* s = new orc_preset();
    if (!fill(*s, preset, seed)) {
        delete s;
        return nullptr;
    }
    return s;
}

void orc_preset_destroy(orc_preset* s) { delete s; }

void orc_preset_arrays(const orc_preset* s, srt_scene_arrays* out, float camera[5]) {
    out->vertices = s->vertices.data();
    out->n_vertices = (uint32_t)s->vertices.size();
    out->indices = s->indices.data();
    out->n_indices = (uint32_t)s->indices.size();
    out->mesh_infos = s->meshes.data();
    out->n_meshes = (uint32_t)s->meshes.size();
    out->materials = s->materials.data();
    out->n_materials = (uint32_t)s->materials.size();
    out->instances = s->instances.data();
    out->n_instances = (uint32_t)s->instances.size();
    out->lights = s->lights.data();
    out->n_lights = (uint32_t)s->lights.size();
    if (camera) std::memcpy(camera, s->camera, sizeof(s->camera));
}

// camera.rs:178-194.  view = look_at_rh(eye, eye + forward, +y) with
// forward = normalize(cos p cos y, sin p, cos p sin y); proj =
// perspective_rh(45 degrees, aspect, 0.1, 100) with depth in [0, 1].  The
// inverses are closed forms: the view is rigid (columns right, up, -forward
// and the eye), the projection's inverse has 1/w, 1/h and the inverted
// depth block.
void orc_camera_uniform(const float pos[3], float yaw, float pitch, float aspect, uint32_t frame,
                        srt_camera_uniform* out) {
    std::memset(out, 0, sizeof(*out));
    float sy = std::sin(yaw), cy = std::cos(yaw), sp = std::sin(pitch), cp = std::cos(pitch);
    float f[3] = {cp * cy, sp, cp * sy};
    float fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    for (float& x : f) x /= fl;
    // right = normalize(forward x up), up' = right x forward
    float r[3] = {f[1] * 0.0f - f[2] * 1.0f, f[2] * 0.0f - f[0] * 0.0f, f[0] * 1.0f - f[1] * 0.0f};
    float rl = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    for (float& x : r) x /= rl;
    float u[3] = {r[1] * f[2] - r[2] * f[1], r[2] * f[0] - r[0] * f[2], r[0] * f[1] - r[1] * f[0]};
    float* V = out->view;
    for (int k = 0; k < 3; ++k) {
        V[4 * k + 0] = r[k];
        V[4 * k + 1] = u[k];
        V[4 * k + 2] = -f[k];
        V[4 * k + 3] = 0.0f;
    }
    V[12] = -(pos[0] * r[0] + pos[1] * r[1] + pos[2] * r[2]);
    V[13] = -(pos[0] * u[0] + pos[1] * u[1] + pos[2] * u[2]);
    V[14] = pos[0] * f[0] + pos[1] * f[1] + pos[2] * f[2];
    V[15] = 1.0f;
    float* VI = out->view_inverse;
    for (int k = 0; k < 3; ++k) {
        VI[0 + k] = r[k];
        VI[4 + k] = u[k];
        VI[8 + k] = -f[k];
        VI[12 + k] = pos[k];
    }
    VI[15] = 1.0f;
    const float fov = 45.0f * 3.14159265358979f / 180.0f, zn = 0.1f, zf = 100.0f;
    float h = std::cos(0.5f * fov) / std::sin(0.5f * fov), w = h / aspect, q = zf / (zn - zf);
    float* P = out->proj;
    P[0] = w;
    P[5] = h;
    P[10] = q;
    P[11] = -1.0f;
    P[14] = q * zn;
    float* PI = out->proj_inverse;
    PI[0] = 1.0f / w;
    PI[5] = 1.0f / h;
    PI[11] = 1.0f / (q * zn);  // w' = z_clip / (q zn) + w_clip / zn
    PI[14] = -1.0f;
    PI[15] = 1.0f / zn;
    out->frame_count = frame;
}
