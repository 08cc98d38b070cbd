// render_kernels.h — launch interface of the per-frame kernels
// (render_kernels.cu).  Host code fills these argument blocks; every
// launcher returns the number of kernels it launched.
#pragma once

#include "device_common.cuh"
#include "guide.cuh"

namespace srt {

constexpr int MAX_BOUNCES = 31;     // max_depth limit (queue counters per bounce)
constexpr int MAX_PHOTON_BOUNCES = 16;  // photon_max_bounces limit (the reference uses 5)
constexpr int PHOTON_BLOCK = 128;   // emitter ids per photon-trace block
constexpr int TRACE_BLOCK = 128;

// Device counters of one frame (zeroed at frame start).
struct FrameCounters {
    uint32_t paths[MAX_BOUNCES + 1];    // active paths entering bounce i
    uint32_t shadow[MAX_BOUNCES + 1];   // shadow rays emitted at bounce i
    uint32_t photon_paths[MAX_PHOTON_BOUNCES + 1];  // live photon paths entering bounce i
    uint32_t fetch[3][MAX_BOUNCES + 1];  // persistent traversal: next queue position, by TRAV_* kind and bounce
    uint32_t photons_stored;
    uint32_t pad[2];
};

// Device statistics accumulated over frames (64-bit).
struct DevStats {
    unsigned long long closest_rays;   // camera-path closest-hit rays
    unsigned long long shadow_rays;
    unsigned long long photon_rays;    // photon-pass closest-hit rays
    unsigned long long photons_stored;
    unsigned long long paths;
    // by ray kind (TRAV_CLOSEST, TRAV_SHADOW, TRAV_PHOTON) and bounce;
    // node visits and triangle tests with SRT_FLAG_COUNT_VISITS only
    unsigned long long rays_bounce[3][MAX_BOUNCES + 1];
    unsigned long long nodes_bounce[3][MAX_BOUNCES + 1];
    unsigned long long tris_bounce[3][MAX_BOUNCES + 1];
};

constexpr int TRAV_CLOSEST = 0, TRAV_SHADOW = 1, TRAV_PHOTON = 2;

struct PathBuffers {
    float4 *ray_o, *ray_d, *hit, *thr, *wl, *rad;
    uint4* misc;  // rng, flags, pixel, pad
    uint32_t* queue[2];
    float4 *sh_o, *sh_d, *sh_c;
    uint32_t* sh_id;
    // ray reordering of the live queue between bounces
    uint32_t *sort_keys, *sort_keys_alt, *sort_vals_alt, *sort_scratch;
};

struct PhotonBuffers {
    float4 *ray_o, *ray_d;  // per emitter: ray origin + tmin, direction + tmax
    float4* state;          // per emitter: wavelength, energy, rng (bits), flags (bits)
    float4* hit;            // per emitter: closest hit (t, triangle, u, v)
    uint8_t* flags;         // per emitter: 1 if a photon was stored
    uint32_t* queue[2];     // live emitter ids after bounce 0
    float4* staging;        // per emitter: the stored photon, 2 float4
    uint32_t* block_counts; // per block of PHOTON_BLOCK emitters; scanned in place into offsets
    float4* photons;        // emission order, 2 per photon
    float4* sorted;         // (hash, index) order, 2 per photon
    uint32_t *keys, *vals, *keys2, *vals2;
    uint32_t* sort_scratch;
    uint2* ranges;          // 2^hash_bits (start, end)
    uint32_t capacity;      // = photons per frame
    uint32_t n_blocks;
    // after a sort: which buffers hold the sorted keys / values
    uint32_t *sorted_keys, *sorted_vals;
};

struct GatherArgs {
    const float4* photons;  // sorted
    const uint2* ranges;
    uint32_t hash_bits;
    uint32_t cap;
    float cell, r0, rexp, spectral_radius, inv_norm_count;
    int enabled;
};

struct FrameArgs {
    DevScene scene;
    const srt_camera_uniform* cam;  // device
    uint32_t width, height;
    uint32_t max_depth;
    uint32_t photons_per_frame;
    uint32_t photon_max_bounces;
    FrameCounters* counters;
    // the counters of the photon pass whose map this frame gathers from (its
    // photon rays go into the frame's statistics): `counters` unless the
    // renderer builds the next frame's photon map during this frame
    const FrameCounters* ph_counters;
    DevStats* stats;
    uint32_t* err;
    PathBuffers pb;
    PhotonBuffers ph;
    GatherArgs gather;
    float4* accum;
    double4* accum64;  // optional
    uchar4* ldr;
    int count_visits;
    int block_size;
    int ray_sort;  // sort the live queue by (direction, origin) before each bounce >= 1
    int sm_count;  // persistent traversal grid = sm_count * blocks per SM
    uint32_t seed; // added to the per-frame seeds of camera paths and photons (0: reference streams)
    int guiding;   // Lambert continuations sampled by the guide (k_guide_infer)
    uint32_t guide_bounces;  // guided Lambert vertices: bounces < guide_bounces (later ones sample the cosine)
    GuideArgs guide;
};

// Photon pass: trace, compaction, grid keys, radix sort, ranges.
int launch_photon_pass(FrameArgs& a, cudaStream_t st);
// Camera paths: raygen, then per bounce trace / shade / shadow; finalize.
int launch_raygen(const FrameArgs& a, cudaStream_t st);
int launch_bounce(const FrameArgs& a, uint32_t bounce, cudaStream_t st,
                  int stage /* 0 all, 1 trace, 2 shade, 3 shadow, 4 shade without the guided continuation */);
int launch_trace_closest(const FrameArgs& a, uint32_t bounce, cudaStream_t st);  // trace_kernels.cu
int launch_trace_shadow(const FrameArgs& a, uint32_t bounce, cudaStream_t st);   // trace_kernels.cu
// Closest hit for the rays named by queue[0 .. *count) (queue NULL: 0 .. *count),
// max_n bounding *count; traversal statistics go to slot `kind` (TRAV_*).
// `fetch` is a zeroed counter the persistent warps draw queue positions from.
int launch_trace_queue(const DevScene& s, uint32_t bounce, const uint32_t* queue, const uint32_t* count,
                       uint32_t* fetch, uint32_t max_n, const float4* ro, const float4* rd, float4* hit, int kind, int count_visits,
                       uint32_t* err, DevStats* stats, int sm_count, cudaStream_t st);  // trace_kernels.cu
// Bounces first .. max_depth - 1 of the paths queued for bounce `first`, in
// one persistent launch (closest hit, shading and shadow ray per path).
int launch_tail(const FrameArgs& a, uint32_t first, cudaStream_t st);
// Threads of one launch_tail wave for these frame arguments (one path each at once).
uint32_t tail_threads(const FrameArgs& a);
// The shading of bounce `bounce` of n_items scenes (device table of their
// frame arguments) in one persistent launch; *fetch starts at 0.
int launch_shade_multi(const FrameArgs* items, int n_items, uint32_t bounce, uint32_t* fetch, int sm_count,
                       cudaStream_t st);
int launch_finalize(const FrameArgs& a, cudaStream_t st);
int launch_frame_stats(const FrameArgs& a, cudaStream_t st);

// Headless presentation (present.cu): letterbox blit of an RGBA8 image into a
// window-sized RGBA8 target, and the photon point splat over an RGBA8 target
// (counts: w*h scratch words).
void letterbox_scale(uint32_t tw, uint32_t th, uint32_t ww, uint32_t wh, float* sx, float* sy);
int launch_blit_letterbox(const uchar4* src, uint32_t sw, uint32_t sh, uchar4* dst, uint32_t ww, uint32_t wh,
                          int srgb, cudaStream_t st);
int launch_photon_splat(const float4* photons, uint32_t n, const srt_camera_uniform* cam, uint32_t w, uint32_t h,
                        uint32_t* counts, uchar4* img, cudaStream_t st);

// Batched rendering: the rays of one kind and bounce of many scenes, traced
// in one launch (trace_kernels.cu).  Visit counting is not available here.
constexpr int MAX_BATCH = 64;
// The batch's rays of all scenes in persistent warps with refill
// (k_trace_multi_pt) instead of chunks of one scene traced lane per ray:
// 32-scene batch 107.2 vs 116.4 ms per iteration, the same images.  The
// chunk of srt_batch_tuning then has no effect.
#ifndef SRT_BATCH_TRACE_PT
#define SRT_BATCH_TRACE_PT 1
#endif
struct MultiTraceItem {
    DevScene s;
    const uint32_t* queue;  // closest: path ids (NULL: identity)
    const uint32_t* count;  // device ray count
    const float4 *ro, *rd;
    float4* hit;            // closest
    const uint32_t* sh_id;  // shadow
    const float4* sh_c;
    float4* rad;
    uint32_t* err;
};
int launch_trace_multi(const MultiTraceItem* items, int n_items, int any_hit, bool small_stack, uint32_t* fetch,
                       int blocks_per_sm, uint32_t chunk, int sm_count, cudaStream_t st);

// Grid over a photon array already on the device (n on host).
int launch_grid_build(const float4* photons, uint32_t n, uint32_t frame, float cell, uint32_t hash_bits,
                      PhotonBuffers& ph, cudaStream_t st);
int launch_gather_queries(const GatherArgs& g, uint32_t frame, const float* queries, uint32_t n_q, float4* out,
                          cudaStream_t st);
int launch_trace_batch(const DevScene& s, const float4* rays, uint32_t n, float4* hits, int any_hit, uint32_t* err,
                       cudaStream_t st);
int launch_test_math(int op, uint32_t n, const void* in, void* out, const void* aux, cudaStream_t st);

}  // namespace srt
