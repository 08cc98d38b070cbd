// host_scene.h — host-side scene description shared by the C ABI and the
// device upload.  Mirrors SceneBuilder (src/scene/builder.rs:47-267).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/srt.h"

struct Mat4 {  // column-major, glam Mat4 memory order
    float m[16];
};

Mat4 mat4_identity();
Mat4 mat4_mul(const Mat4& a, const Mat4& b);
Mat4 mat4_translation(float x, float y, float z);
Mat4 mat4_scale(float x, float y, float z);
Mat4 mat4_rotation_x(float a);
Mat4 mat4_rotation_y(float a);
Mat4 mat4_rotation_z(float a);

// A light instance recorded by the builder: its triangles became
// lights[first_light .. first_light + count).
struct srt_light_instance_rec {
    uint32_t instance, first_light, count;
    float params[4];
};

struct srt_scene_builder {
    std::vector<srt_light_instance_rec> light_instances;
    std::vector<srt_vertex> vertices;
    std::vector<uint32_t> indices;
    std::vector<srt_mesh_info> mesh_infos;
    std::vector<srt_material> materials;
    std::vector<srt_instance> instances;
    std::vector<srt_light> lights;
    // per mesh: triangle count (for the light expansion and the flattening)
    std::vector<uint32_t> mesh_tris;

    uint32_t add_material(const srt_material& m);
    uint32_t add_mesh(const srt_vertex* v, uint32_t nv, const uint32_t* idx, uint32_t ni);
    void add_instance(uint32_t mesh, uint32_t mat, const Mat4& t);
    void add_light_instance(uint32_t mesh, uint32_t mat, const Mat4& t, const float params[4]);
};

// geometry.rs generators
void geom_plane(std::vector<srt_vertex>& v, std::vector<uint32_t>& i);
void geom_cube(std::vector<srt_vertex>& v, std::vector<uint32_t>& i);
void geom_icosphere(uint32_t subdivisions, std::vector<srt_vertex>& v, std::vector<uint32_t>& i);
void geom_uv_sphere(uint32_t slices, uint32_t stacks, std::vector<srt_vertex>& v, std::vector<uint32_t>& i);
// Displaces an icosphere radially by seeded 3-octave value noise and
// recomputes area-weighted vertex normals.
void geom_displace(std::vector<srt_vertex>& v, const std::vector<uint32_t>& i, float amplitude, uint32_t seed);

// Presets; camera = {x, y, z, yaw, pitch}
bool preset_fill(srt_scene_builder* b, int preset, uint32_t seed, float camera[5]);

// camera.rs:178-194
void camera_build_uniform(const float pos[3], float yaw, float pitch, float aspect, uint32_t frame,
                          srt_camera_uniform* out);

// screenshot.rs:27-103: padded RGBA8 rows (row 0 = bottom) -> PNG with the
// rows flipped and the sRGB OETF applied to the 8-bit values.
bool write_screenshot_png(const std::string& path, const uint8_t* rgba, uint32_t w, uint32_t h, uint32_t pitch);
// The same on the library's screenshot worker thread (screenshot_worker.cpp):
// the job owns `rgba`; srt_screenshot_flush waits for it.
void screenshot_enqueue(const std::string& path, std::vector<uint8_t>&& rgba, uint32_t w, uint32_t h,
                        uint32_t pitch);
uint8_t srgb_oetf_u8(uint8_t c);
