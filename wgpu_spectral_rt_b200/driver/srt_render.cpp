// srt_render — headless driver of the C ABI (include/srt.h).
//
// The native caller that stands where the reference's Rust engine loop
// stands (src/engine.rs:139-244: build the scene, create the renderer, per
// frame write the camera uniform with the frame count and render, then save a
// screenshot), without a window: it renders a preset scene for a number of
// frames and writes the tonemapped image as a PNG (src/screenshot.rs:27-103).
// It uses nothing but the C ABI, so it is also the template for binding the
// library from any language with a C FFI.
//
//   srt_render --preset 0 --width 640 --height 480 --frames 64 --out cornell.png
//
// Prints one line of timing (frames, ms per frame, Mpaths/s) measured with a
// host clock around the rendering after a context synchronisation.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "srt.h"

namespace {

struct Options {
    int device = 0;
    int preset = SRT_PRESET_CORNELL_BOX;
    uint32_t seed = 0;
    uint32_t width = 640, height = 480, frames = 16;
    int max_depth = -1;        // < 0: the library default
    long photons = -1;         // < 0: the library default
    bool guiding = false;
    int tail = -1;             // < 0: automatic
    std::string out = "srt_render.png";
};

void usage(FILE* f) {
    std::fprintf(f,
                 "usage: srt_render [--device N] [--preset N] [--seed N] [--width W] [--height H]\n"
                 "                  [--frames F] [--depth D] [--photons P] [--guiding] [--tail B]\n"
                 "                  [--out PATH] [--version] [--help]\n"
                 "presets: 0 Cornell box, 1 custom prism, 2 config 1, 3 config 2, 4 caustic slab,\n"
                 "         5 indirect room, 6 batch-random (seeded)\n");
}

bool parse_uint(const char* s, unsigned long max, unsigned long* out) {
    char* end = nullptr;
    unsigned long v = std::strtoul(s, &end, 10);
    if (!s[0] || *end || v > max) return false;
    *out = v;
    return true;
}

// 0: run, 1: exit 0 (help/version printed), 2: bad arguments
int parse(int argc, char** argv, Options& o) {
    for (int i = 1; i < argc; ++i) {
        const char* a = argv[i];
        auto value = [&](unsigned long max, unsigned long* v) {
            return i + 1 < argc && parse_uint(argv[++i], max, v);
        };
        unsigned long v = 0;
        if (!std::strcmp(a, "--help") || !std::strcmp(a, "-h")) {
            usage(stdout);
            return 1;
        } else if (!std::strcmp(a, "--version")) {
            std::printf("srt_render: library ABI %u, header ABI %u\n", srt_abi_version(), SRT_ABI_VERSION);
            return 1;
        } else if (!std::strcmp(a, "--guiding")) {
            o.guiding = true;
        } else if (!std::strcmp(a, "--out")) {
            if (i + 1 >= argc) return 2;
            o.out = argv[++i];
        } else if (!std::strcmp(a, "--device")) {
            if (!value(64, &v)) return 2;
            o.device = (int)v;
        } else if (!std::strcmp(a, "--preset")) {
            if (!value(SRT_PRESET_BATCH_RANDOM, &v)) return 2;
            o.preset = (int)v;
        } else if (!std::strcmp(a, "--seed")) {
            if (!value(0xFFFFFFFFul, &v)) return 2;
            o.seed = (uint32_t)v;
        } else if (!std::strcmp(a, "--width")) {
            if (!value(16384, &v) || v == 0) return 2;
            o.width = (uint32_t)v;
        } else if (!std::strcmp(a, "--height")) {
            if (!value(16384, &v) || v == 0) return 2;
            o.height = (uint32_t)v;
        } else if (!std::strcmp(a, "--frames")) {
            if (!value(1ul << 24, &v) || v == 0) return 2;
            o.frames = (uint32_t)v;
        } else if (!std::strcmp(a, "--depth")) {
            if (!value(31, &v) || v == 0) return 2;
            o.max_depth = (int)v;
        } else if (!std::strcmp(a, "--photons")) {
            if (!value(1ul << 26, &v)) return 2;
            o.photons = (long)v;
        } else if (!std::strcmp(a, "--tail")) {
            if (!value(31, &v)) return 2;
            o.tail = (int)v;
        } else {
            return 2;
        }
    }
    return 0;
}

// Reports a failed call with the context's last error text.
bool ok(srt_status s, const srt_ctx* ctx, const char* what) {
    if (s == SRT_OK) return true;
    const char* msg = srt_get_error_string(ctx);
    std::fprintf(stderr, "srt_render: %s failed (status %d): %s\n", what, (int)s, msg ? msg : "");
    return false;
}

}  // namespace

int main(int argc, char** argv) {
    Options o;
    const int pr = parse(argc, argv, o);
    if (pr == 1) return 0;
    if (pr == 2) {
        usage(stderr);
        return 2;
    }
    if (srt_abi_version() != SRT_ABI_VERSION) {
        std::fprintf(stderr, "srt_render: library ABI %u, header ABI %u\n", srt_abi_version(), SRT_ABI_VERSION);
        return 1;
    }
    int rc = 1;
    srt_ctx* ctx = nullptr;
    srt_scene_builder* builder = nullptr;
    srt_scene* scene = nullptr;
    srt_renderer* r = nullptr;
    float cam[5] = {0, 0, 0, 0, 0};  // position xyz, yaw, pitch
    srt_params p = srt_params_default();
    if (o.max_depth > 0) p.max_depth = (uint32_t)o.max_depth;
    if (o.photons >= 0) p.photons_per_frame = (uint32_t)o.photons;
    if (o.guiding) p.flags |= SRT_FLAG_GUIDING;
    const float aspect = (float)o.width / (float)o.height;
    srt_camera_uniform u;
    srt_stats st;
    double ms = 0.0;

    if (!ok(srt_ctx_create(o.device, nullptr, &ctx), nullptr, "srt_ctx_create")) goto done;
    // SceneBuilder::build (scene/builder.rs:131-266) from a preset scene
    if (!ok(srt_scene_builder_create(&builder), ctx, "srt_scene_builder_create")) goto done;
    if (!ok(srt_scene_builder_add_preset(builder, o.preset, o.seed, cam), ctx, "srt_scene_builder_add_preset"))
        goto done;
    if (!ok(srt_scene_builder_build(ctx, builder, &scene), ctx, "srt_scene_builder_build")) goto done;
    // Renderer::new (renderer/mod.rs:45)
    if (!ok(srt_renderer_create(ctx, scene, o.width, o.height, &p, &r), ctx, "srt_renderer_create")) goto done;
    if (o.tail >= 0 && !ok(srt_renderer_set_tail(r, (uint32_t)o.tail), ctx, "srt_renderer_set_tail")) goto done;
    {
        // the engine's frame loop (engine.rs:154-166): the uniform carries the
        // frame count, which seeds the samples and restarts the accumulation at 0
        if (!ok(srt_ctx_synchronize(ctx), ctx, "srt_ctx_synchronize")) goto done;
        const auto t0 = std::chrono::steady_clock::now();
        for (uint32_t f = 0; f < o.frames; ++f) {
            if (!ok(srt_camera_build_uniform(cam, cam[3], cam[4], aspect, f, &u), ctx, "srt_camera_build_uniform"))
                goto done;
            if (!ok(srt_render_frame(r, &u), ctx, "srt_render_frame")) goto done;
        }
        if (!ok(srt_ctx_synchronize(ctx), ctx, "srt_ctx_synchronize")) goto done;
        ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    // Engine::save_screenshot (engine.rs:191-244, screenshot.rs:27-103)
    if (!ok(srt_save_screenshot(r, o.out.c_str()), ctx, "srt_save_screenshot")) goto done;
    if (!ok(srt_renderer_get_stats(r, &st), ctx, "srt_renderer_get_stats")) goto done;
    std::printf("srt_render: preset %d, %ux%u, %u frames, %.3f ms per frame, %.2f Mpaths/s, %llu closest-hit rays, "
                "tail from bounce %u -> %s\n",
                o.preset, o.width, o.height, o.frames, ms / o.frames,
                (double)o.width * o.height * o.frames / (ms * 1e3), (unsigned long long)st.rays_closest,
                st.tail_first, o.out.c_str());
    rc = 0;
done:
    if (r) srt_renderer_destroy(r);
    if (scene) srt_scene_destroy(scene);
    if (builder) srt_scene_builder_destroy(builder);
    if (ctx) srt_ctx_destroy(ctx);
    return rc;
}
