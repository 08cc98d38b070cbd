// render_kernels.cu — per-frame kernels of the spectral path tracer.
//
// One frame = one sample per pixel (src/renderer/mod.rs:168-207):
//   photon pass   photon_emit.wgsl:154-331 as a wavefront (emit, direction
//                 sort, per bounce trace + shade, emitter-ordered compaction
//                 of the stored photons) and the grid (build_grid.wgsl:25-73)
//                 as cell keys + radix sort + ranges
//   camera paths  shader.wgsl:708-823 as a wavefront: raygen, then per
//                 bounce trace_closest -> shade -> trace_shadow over SoA
//                 queues compacted with warp ballots; finalize converts the
//                 hero tuple to sRGB, accumulates and tonemaps.
#include "radix_sort.cuh"
#include "render_kernels.h"

// Resident blocks of TRACE_BLOCK threads per SM the shading kernels are
// compiled for.  8 caps them at 64 registers (the unbounded build takes 87,
// 108 with guiding, and runs 20 warps per SM): the spills stay in L1 and the
// doubled warp count hides the photon-gather latency better (measured shading
// per frame: config 2 1.98 -> 1.79 ms, the guiding scene 2.94 -> 2.58 ms).
#ifndef SRT_SHADE_MIN_BLOCKS
#define SRT_SHADE_MIN_BLOCKS 8
#endif

namespace srt {

namespace {

constexpr uint32_t FLAG_DIFFUSE = 0x1u;  // has_hit_diffuse (shader.wgsl:554)
constexpr uint32_t FLAG_CAUSTIC = 0x2u;  // is_caustic_path (shader.wgsl:555)

SRT_DEV uint32_t warp_push(bool pred, uint32_t* counter) {
    uint32_t mask = __ballot_sync(0xFFFFFFFFu, pred);
    int lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (mask) {
        int leader = __ffs(mask) - 1;
        if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
        base = __shfl_sync(0xFFFFFFFFu, base, leader);
    }
    return base + __popc(mask & ((1u << lane) - 1u));
}

// gather_photons: shader.wgsl:297-342 over a sorted range; the walk goes
// from the highest photon index down (the LIFO order of the reference's
// linked list for in-order insertion), at most `cap` entries.
SRT_DEV float4 gather(const GatherArgs& g, uint32_t frame, float3 hit_pos, float3 normal, float4 wl) {
    float3 j = grid_jitter(frame, g.cell);
    float r = g.r0 * powf((float)(frame + 1u), g.rexp);
    float r2 = r * r;
    uint32_t h = grid_hash(hit_pos, j, g.cell, g.hash_bits);
    uint2 rg = __ldg(&g.ranges[h]);
    float4 total = splat4(0.f);
    uint32_t stop = rg.y - min(rg.y - rg.x, g.cap);
    for (uint32_t i = rg.y; i > stop; --i) {
        float4 pa = __ldg(&g.photons[2 * (i - 1)]);
        float4 pb = __ldg(&g.photons[2 * (i - 1) + 1]);
        float3 dd = hit_pos - xyz(pa);
        float d2 = dot(dd, dd);
        if (d2 < r2 && dot(normal, xyz(pb)) > 0.0f) {
            float sw = 1.0f - (sqrtf(d2) / r);
            float4 spw = f4(fmaxf(1.0f - fabsf(wl.x - pa.w) / g.spectral_radius, 0.f),
                            fmaxf(1.0f - fabsf(wl.y - pa.w) / g.spectral_radius, 0.f),
                            fmaxf(1.0f - fabsf(wl.z - pa.w) / g.spectral_radius, 0.f),
                            fmaxf(1.0f - fabsf(wl.w - pa.w) / g.spectral_radius, 0.f));
            total = total + spw * (pb.w * sw);
        }
    }
    float density = (3.0f / (PI * r2)) * (1.0f / g.spectral_radius) * g.inv_norm_count;
    return total * density;
}

// ------------------------------------------------------------------ photon pass
// The photon pass of photon_emit.wgsl:154-331 as a wavefront: emit every
// photon path (one thread per emitter id), then per bounce: the shared
// closest-hit kernel over the live queue and a shading kernel for the
// photon's material logic.  A stored photon lands in its emitter's slot and is
// flagged; an emitter-ordered compaction afterwards reproduces the order a
// sequential run of the reference's atomicAdd gives.
//
// SRT_PHOTON_DIR_SORT sorts the emitted rays by an octahedral direction key
// first, so that a warp traces rays of similar direction.  It paid while
// photon rays were traced one per thread; with the persistent warps (refill,
// warp-synchronous node visits) it no longer does: config-2 photon pass 2.25
// ms unsorted vs 2.45 ms sorted on 24 bits (2.36 on 16, 2.29 on 8), the same
// photons.
#ifndef SRT_PHOTON_DIR_SORT
#define SRT_PHOTON_DIR_SORT 0
#endif

// Octahedral 12+12-bit direction code, Morton-interleaved (24 bits).
SRT_DEV uint32_t dir_key(float3 d) {
    float s = fabsf(d.x) + fabsf(d.y) + fabsf(d.z);
    float px = d.x / s, py = d.y / s;
    if (d.z < 0.0f) {
        float qx = (1.0f - fabsf(py)) * (px >= 0.0f ? 1.0f : -1.0f);
        float qy = (1.0f - fabsf(px)) * (py >= 0.0f ? 1.0f : -1.0f);
        px = qx;
        py = qy;
    }
    uint32_t ux = (uint32_t)fminf(fmaxf((px * 0.5f + 0.5f) * 4096.0f, 0.0f), 4095.0f);
    uint32_t uy = (uint32_t)fminf(fmaxf((py * 0.5f + 0.5f) * 4096.0f, 0.0f), 4095.0f);
    uint32_t k = 0;
#pragma unroll
    for (int b = 0; b < 12; ++b) k |= (((ux >> b) & 1u) << (2 * b)) | (((uy >> b) & 1u) << (2 * b + 1));
    return k;
}

// Sort key of a secondary camera ray: direction first (octahedral 7+7 bits,
// Morton order), then origin (6 bits per axis of the scene bounds, Morton).
SRT_DEV uint32_t ray_sort_key(float3 o, float3 d, float4 bmin, float4 binv) {
    uint32_t dk = dir_key(d) >> 10;  // top 7 bits of each octahedral coordinate
    uint32_t q[3];
    q[0] = (uint32_t)fminf(fmaxf((o.x - bmin.x) * binv.x * 64.0f, 0.0f), 63.0f);
    q[1] = (uint32_t)fminf(fmaxf((o.y - bmin.y) * binv.y * 64.0f, 0.0f), 63.0f);
    q[2] = (uint32_t)fminf(fmaxf((o.z - bmin.z) * binv.z * 64.0f, 0.0f), 63.0f);
    uint32_t ok = 0;
#pragma unroll
    for (int b = 0; b < 6; ++b)
        ok |= (((q[0] >> b) & 1u) << (3 * b)) | (((q[1] >> b) & 1u) << (3 * b + 1)) | (((q[2] >> b) & 1u) << (3 * b + 2));
    return (dk << 18) | ok;
}

constexpr uint32_t PH_CAUSTIC = 0x1u;

// Emission: photon_emit.wgsl:159-214.
__global__ void k_photon_emit(FrameArgs a) {
    uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.photons_per_frame) return;
    const DevScene& S = a.scene;
    uint32_t frame = a.cam->frame_count;
    uint32_t s = pcg_hash(e + frame * 927163u + a.seed);
    uint32_t nl = S.n_lights;  // > 0: the pass is skipped without lights
    uint32_t li = min(__float2uint_rz(rng_next(s) * (float)nl), nl - 1u);
    float4 L0 = S.lights[4 * li], L1 = S.lights[4 * li + 1], L2 = S.lights[4 * li + 2], LP = S.lights[4 * li + 3];
    float3 v0 = xyz(L0), v1 = xyz(L1), v2 = xyz(L2);
    float3 c = cross(v1 - v0, v2 - v0);
    float3 normal = normalize(c);
    float area = length(c) * 0.5f;
    float r1 = rng_next(s);
    float r2 = rng_next(s);
    float sr1 = sqrtf(r1);
    float u = 1.0f - sr1, v = r2 * sr1, w = 1.0f - u - v;
    float3 emit_pos = v0 * u + v1 * v + v2 * w;
    float3 emit_dir = normalize(normal + random_unit_vector(s));
    float cmin = cauchy_cdf(LAMBDA_MIN), cmax = cauchy_cdf(LAMBDA_MAX), crange = cmax - cmin;
    float lambda =
        clampf(555.0f + 40.0f * tanf(PI * ((cmin + rng_next(s) * crange) - 0.5f)), LAMBDA_MIN, LAMBDA_MAX);
    float dw = (lambda - 555.0f) / 40.0f;
    float pdf = (1.0f / (crange * PI * 40.0f)) / (1.0f + dw * dw);
    float energy = (blackbody(lambda, LP.y) / pdf) * area * PI * LP.z;
    float3 pos = emit_pos + emit_dir * 0.001f;
    a.ph.ray_o[e] = f4(pos.x, pos.y, pos.z, 0.0001f);
    a.ph.ray_d[e] = f4(emit_dir.x, emit_dir.y, emit_dir.z, 100.0f);
    a.ph.state[e] = f4(lambda, energy, __uint_as_float(s), __uint_as_float(0u));
    a.ph.flags[e] = 0u;
    if (SRT_PHOTON_DIR_SORT) {
        a.ph.keys[e] = dir_key(emit_dir);
        a.ph.vals[e] = e;
    }
    if (e == 0) a.counters->photon_paths[0] = a.photons_per_frame;
}

// One bounce of the photon loop after its closest-hit query
// (photon_emit.wgsl:227-330).  Material type 5 (no reference counterpart)
// reflects with the probability of the film's Airy reflectance, else absorbs.
__global__ void __launch_bounds__(TRACE_BLOCK, SRT_SHADE_MIN_BLOCKS) k_photon_shade(FrameArgs a, uint32_t bounce) {
    uint32_t n = a.counters->photon_paths[bounce];
    if (blockIdx.x * blockDim.x >= n) return;
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    const DevScene& S = a.scene;
    const uint32_t* qin = bounce == 0 ? a.ph.sorted_vals : a.ph.queue[bounce & 1];
    bool alive = false;
    uint32_t e = q < n ? (qin ? qin[q] : q) : 0u;
    if (q < n) {
        float4 h = a.ph.hit[e];
        uint32_t prim = __float_as_uint(h.y);
        if (prim != MISS) {
            float4 o4 = a.ph.ray_o[e], d4 = a.ph.ray_d[e], st = a.ph.state[e];
            float3 pos = xyz(o4), dir = xyz(d4);
            float lambda = st.x, energy = st.y;
            uint32_t s = __float_as_uint(st.z), fl = __float_as_uint(st.w);
            Surface sf = surface_at(S, prim, h.z, h.w, dir);
            float4 extra = S.materials[2 * sf.mat + 1];
            float3 ffn = sf.front ? sf.wn : -sf.wn;
            uint32_t type = (uint32_t)extra.x;
            float3 hp = pos + dir * h.x;
            bool caustic = (fl & PH_CAUSTIC) != 0u;
            if (type == 0u) {
                if (caustic) {
                    a.ph.staging[2 * e] = f4(hp.x, hp.y, hp.z, lambda);
                    a.ph.staging[2 * e + 1] = f4(-dir.x, -dir.y, -dir.z, energy);
                    a.ph.flags[e] = 1u;
                }
            } else if (type == 1u) {
                dir = reflect(normalize(dir), ffn);
                pos = hp + ffn * 0.001f;
                alive = true;
            } else if (type == 2u) {
                float lum = lambda / 1000.0f;
                float ir = extra.z + (extra.w / (lum * lum));
                float ratio = sf.front ? 1.0f / ir : ir;
                float3 ud = normalize(dir);
                float ct = fminf(dot(-ud, ffn), 1.0f);
                float stn = sqrtf(1.0f - ct * ct);
                if (ratio * stn > 1.0f || schlick(ct, ratio) > rng_next(s)) {
                    dir = reflect(ud, ffn);
                } else {
                    caustic = true;
                    dir = refract(ud, ffn, ratio);
                }
                pos = hp + (dot(dir, ffn) > 0.0f ? ffn : -ffn) * 0.001f;
                alive = true;
            } else if (type == 4u) {
                float3 ud = normalize(dir);
                float ct = fminf(dot(-ud, ffn), 1.0f);
                // select(n1 / n3, n3 / n1, is_front_face) with n1 = 1
                float ratio = sf.front ? extra.w / 1.0f : 1.0f / extra.w;
                float stt = ratio * ratio * (1.0f - ct * ct);
                if (stt > 1.0f) {
                    dir = reflect(ud, ffn);
                } else {
                    bool tir;
                    float F = thin_film1(ct, 1.0f, extra.z, extra.w, fmaxf(extra.y, 50.0f), lambda, tir);
                    dir = rng_next(s) < F ? reflect(ud, ffn) : refract(ud, ffn, ratio);
                }
                caustic = true;  // the position is not advanced (photon_emit.wgsl:291-326)
                alive = true;
            } else if (type == 5u) {
                float3 ud = normalize(dir);
                float ct = fminf(dot(-ud, ffn), 1.0f);
                bool tir;
                float F = thin_film1(ct, 1.0f, extra.z, extra.w, fmaxf(extra.y, 50.0f), lambda, tir);
                if (rng_next(s) < F) {
                    dir = reflect(ud, ffn);
                    pos = hp + ffn * 0.001f;
                    caustic = true;
                    alive = true;
                }
            }
            if (bounce + 1u >= a.photon_max_bounces) alive = false;
            if (alive) {
                a.ph.ray_o[e] = f4(pos.x, pos.y, pos.z, 0.0001f);
                a.ph.ray_d[e] = f4(dir.x, dir.y, dir.z, 100.0f);
                a.ph.state[e] = f4(lambda, energy, __uint_as_float(s), __uint_as_float(caustic ? PH_CAUSTIC : 0u));
            }
        }
    }
    uint32_t slot = warp_push(alive, &a.counters->photon_paths[bounce + 1]);
    if (alive) a.ph.queue[(bounce + 1) & 1][slot] = e;
}

// Emitter-ordered compaction of the stored photons: per-block counts, an
// exclusive scan of the counts (k_rs_rowscan), then the scatter.
__global__ void __launch_bounds__(PHOTON_BLOCK) k_deposit_count(FrameArgs a) {
    __shared__ uint32_t warp_cnt[PHOTON_BLOCK / 32];
    uint32_t e = blockIdx.x * PHOTON_BLOCK + threadIdx.x;
    bool stored = e < a.photons_per_frame && a.ph.flags[e] != 0u;
    uint32_t m = __ballot_sync(0xFFFFFFFFu, stored);
    if ((threadIdx.x & 31) == 0) warp_cnt[threadIdx.x >> 5] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < PHOTON_BLOCK / 32; ++w) t += warp_cnt[w];
        a.ph.block_counts[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(PHOTON_BLOCK) k_deposit_scatter(FrameArgs a) {
    __shared__ uint32_t warp_cnt[PHOTON_BLOCK / 32];
    uint32_t e = blockIdx.x * PHOTON_BLOCK + threadIdx.x;
    bool stored = e < a.photons_per_frame && a.ph.flags[e] != 0u;
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t m = __ballot_sync(0xFFFFFFFFu, stored);
    if (lane == 0) warp_cnt[warp] = __popc(m);
    __syncthreads();
    uint32_t before = a.ph.block_counts[blockIdx.x];
    for (int w = 0; w < warp; ++w) before += warp_cnt[w];
    if (stored) {
        uint32_t dst = before + __popc(m & ((1u << lane) - 1u));
        a.ph.photons[2 * dst] = a.ph.staging[2 * e];
        a.ph.photons[2 * dst + 1] = a.ph.staging[2 * e + 1];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        atomicAdd(&a.stats->photons_stored, (unsigned long long)a.counters->photons_stored);
}

__global__ void k_grid_keys(const float4* __restrict__ photons, const uint32_t* n_dev, uint32_t n_host,
                            const uint32_t* frame_dev, uint32_t frame_host, float cell, uint32_t hash_bits,
                            uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    uint32_t n = n_dev ? *n_dev : n_host;
    uint32_t frame = frame_dev ? *frame_dev : frame_host;
    float3 j = grid_jitter(frame, cell);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 p0 = photons[2 * i], p1 = photons[2 * i + 1];
        keys[i] = p1.w == 0.0f ? (1u << hash_bits) : grid_hash(xyz(p0), j, cell, hash_bits);
        vals[i] = i;
    }
}

__global__ void k_grid_ranges(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                              const uint32_t* n_dev, uint32_t n_host, uint32_t hash_bits,
                              const float4* __restrict__ photons, float4* __restrict__ sorted, uint2* __restrict__ ranges) {
    uint32_t n = n_dev ? *n_dev : n_host;
    uint32_t sentinel = 1u << hash_bits;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t h = keys[i];
        uint32_t v = vals[i];
        sorted[2 * i] = photons[2 * v];
        sorted[2 * i + 1] = photons[2 * v + 1];
        if (h >= sentinel) continue;
        if (i == 0 || keys[i - 1] != h) ranges[h].x = i;
        if (i + 1 == n || keys[i + 1] != h) ranges[h].y = i + 1;
    }
}

// ------------------------------------------------------------------ camera paths
// Bounce-0 queue order (SRT_RAYGEN_TILE): queue position q -> pixel, with
// the pixels of a warp in an 8 x 4 tile (bands of 4 rows, 8-column blocks
// within a band; narrower blocks and bands at the right and bottom edges)
// instead of a 32 x 1 strip.  A bijection of [0, w h).  Config-2 camera rays
// of bounce 0: 0.383 vs 0.428 ms (a warp's rays closer in both directions);
// a path's result does not depend on its queue position.
#ifndef SRT_RAYGEN_TILE
#define SRT_RAYGEN_TILE 1
#endif
SRT_DEV void tile_pixel(uint32_t q, uint32_t w, uint32_t h, uint32_t& x, uint32_t& y) {
    const uint32_t band = q / (4u * w), y0 = 4u * band;
    const uint32_t hb = min(4u, h - y0);
    const uint32_t r = q - y0 * w;  // position inside the band
    const uint32_t blk = r / (8u * hb), x0 = 8u * blk;
    const uint32_t wb = min(8u, w - x0);
    const uint32_t t = r - x0 * hb;  // position inside the block
    x = x0 + t % wb;
    y = y0 + t / wb;
}

__global__ void k_raygen(FrameArgs a) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t n = a.width * a.height;
    if (q >= n) return;
    const srt_camera_uniform& cam = *a.cam;
    uint32_t x, y;
    if (SRT_RAYGEN_TILE) tile_pixel(q, a.width, a.height, x, y);
    else {
        x = q % a.width;
        y = q / a.width;
    }
    const uint32_t p = x + y * a.width;
    uint32_t s = pcg_hash(x + y * a.width + cam.frame_count * 927163u + a.seed);
    float3 o, d;
    camera_ray(cam, x, y, a.width, a.height, s, o, d);
    float4 wl = sample_hero(s);
    a.pb.ray_o[p] = f4(o.x, o.y, o.z, 0.0001f);
    a.pb.ray_d[p] = f4(d.x, d.y, d.z, 100.0f);
    a.pb.thr[p] = splat4(1.0f);
    a.pb.wl[p] = wl;
    a.pb.rad[p] = splat4(0.0f);
    a.pb.misc[p] = make_uint4(s, 0u, p, 0u);
    a.pb.queue[0][q] = p;
    if (q == 0) a.counters->paths[0] = n;
}

struct LightSample {
    float3 dir;
    float dist, pdf;
    float4 radiance;
};

// sample_random_light: shader.wgsl:477-528
SRT_DEV LightSample sample_light(const DevScene& S, float3 hp, float4 wl, uint32_t& s) {
    LightSample ls;
    ls.pdf = 0.f;
    uint32_t nl = S.n_lights;
    if (nl == 0u) return ls;
    uint32_t li = min(__float2uint_rz(rng_next(s) * (float)nl), nl - 1u);
    float4 L0 = S.lights[4 * li], L1 = S.lights[4 * li + 1], L2 = S.lights[4 * li + 2], LP = S.lights[4 * li + 3];
    float r1 = rng_next(s);
    float r2 = rng_next(s);
    float sr1 = sqrtf(r1);
    float u = 1.0f - sr1, v = r2 * sr1, w = 1.0f - u - v;
    float3 v0 = xyz(L0), v1 = xyz(L1), v2 = xyz(L2);
    float3 p = v0 * u + v1 * v + v2 * w;
    float3 c = cross(v1 - v0, v2 - v0);
    float3 normal = normalize(c);
    float area = length(c) * 0.5f;
    float3 to = p - hp;
    float d2 = dot(to, to);
    float dist = sqrtf(d2);
    float3 l = to / dist;
    float cl = fmaxf(dot(normal, -l), 0.0f);
    if (cl <= 0.0001f) return ls;
    ls.dir = l;
    ls.dist = dist;
    ls.pdf = d2 / (area * (float)nl * cl);
    ls.radiance = blackbody4(wl, LP.y) * LP.z;
    return ls;
}

// What one path's vertex produced: the continuation (written to the path
// state when alive), a shadow ray, or a vertex deferred to the guide.
struct VertexOut {
    bool alive = false, shadow = false, guided = false;
    float3 sh_o = f3(0.f, 0.f, 0.f), sh_d = f3(0.f, 0.f, 0.f);
    float sh_tmax = 0.f;
    float4 sh_c = splat4(0.f);
    uint32_t key = 0u;
    float4 g_p = splat4(0.f), g_n = splat4(0.f), g_wo = splat4(0.f), g_spec = splat4(0.f);
};

// One iteration of ray_color's bounce loop after the closest-hit query
// (shader.wgsl:568-700) for path `id`, whose hit is in a.pb.hit[id]: writes
// the path's radiance and, when it continues, its next ray and state.
// GUIDE: Lambert continuations of bounces < guide_bounces are left to
// k_guide_infer (guide.cu); every guided renderer records the radiance a
// training record's next vertex sees.
template <bool GUIDE>
SRT_DEV VertexOut shade_vertex(const FrameArgs& a, uint32_t id, uint32_t bounce) {
    VertexOut out;
    const DevScene& S = a.scene;
    float4 h = a.pb.hit[id];
    uint32_t prim = __float_as_uint(h.y);
    if (prim == MISS) return out;
    float4 o4 = a.pb.ray_o[id], d4 = a.pb.ray_d[id];
    float3 o = xyz(o4), d = xyz(d4);
    float4 thr = a.pb.thr[id], wl = a.pb.wl[id], rad = a.pb.rad[id];
    uint4 misc = a.pb.misc[id];
    uint32_t s = misc.x, flags = misc.y;
    // a training record of the previous vertex: radiance before this vertex
    if (GUIDE && misc.w != 0u) a.guide.rec.rad[misc.w - 1u] = rad;
    Surface sf = surface_at(S, prim, h.z, h.w, d);
    float4 color = S.materials[2 * sf.mat], extra = S.materials[2 * sf.mat + 1];
    float3 ffn = sf.front ? sf.wn : -sf.wn;
    uint32_t type = (uint32_t)extra.x;
    if (type == 3u) {
        if (!(flags & FLAG_CAUSTIC) && (sf.front || extra.y > 0.0f)) {
            float4 em = blackbody4(wl, color.x) * color.y;
            a.pb.rad[id] = rad + em * thr;
        }
        return out;
    }
    if (type == 0u) flags = (flags | FLAG_DIFFUSE) & ~FLAG_CAUSTIC;
    else if (type == 2u && (flags & FLAG_DIFFUSE)) flags |= FLAG_CAUSTIC;
    if (type == 0u) {
        float4 spec = rgb_to_spectrum4(xyz(color), wl);
        float3 hp = o + d * h.x;
        if (a.gather.enabled) {
            float4 gl = gather(a.gather, a.cam->frame_count, hp, ffn, wl);
            rad = rad + thr * (spec / PI) * gl;
        }
        LightSample ls = sample_light(S, hp, wl, s);
        if (ls.pdf > 0.0f) {
            float ct = fmaxf(dot(ffn, ls.dir), 0.0f);
            float bpdf = ct / PI;
            float mis = ls.pdf / (ls.pdf + bpdf);
            out.sh_c = thr * (spec / PI) * ls.radiance * ct * (mis / ls.pdf);
            out.sh_o = hp;
            out.sh_d = ls.dir;
            out.sh_tmax = ls.dist - 0.001f;
            out.shadow = true;
        }
        a.pb.rad[id] = rad;
        if (GUIDE && bounce + 1u < a.max_depth && bounce < a.guide_bounces) {
            out.guided = true;
            out.g_p = f4(hp.x, hp.y, hp.z, wl.x);
            out.g_n = f4(ffn.x, ffn.y, ffn.z, 0.f);
            out.g_wo = f4(-d.x, -d.y, -d.z, 0.f);
            out.g_spec = spec;
            a.pb.misc[id] = make_uint4(s, flags, misc.z, 0u);
            return out;
        }
    }
    Scatter sc = sample_bsdf(d, ffn, color, extra, sf.front, wl, thr, s);
    if (!sc.absorbed) {
        thr = thr * sc.att;
        o = o + d * h.x;
        bool alive = true;
        if (bounce > 3u) {
            float p = max4(thr);
            if (rng_next(s) > p) alive = false;
            else thr = thr / p;
        }
        if (bounce + 1u >= a.max_depth) alive = false;
        if (alive) {
            a.pb.thr[id] = thr;
            a.pb.ray_o[id] = f4(o.x, o.y, o.z, 0.0001f);
            a.pb.ray_d[id] = f4(sc.dir.x, sc.dir.y, sc.dir.z, 100.0f);
            a.pb.misc[id] = make_uint4(s, flags, misc.z, 0u);
            if (a.ray_sort) out.key = ray_sort_key(o, sc.dir, S.bmin, S.binv);
        }
        out.alive = alive;
    }
    return out;
}

// One bounce of every live path: shade_vertex, then the live paths, shadow
// rays and guided vertices go to their queues (warp-aggregated slots).
// shade_slot is one thread's vertex: queue position q of `bounce` (q >= n:
// no vertex; the thread still takes part in the warp's queue pushes).
template <bool GUIDE>
SRT_DEV void shade_slot(const FrameArgs& a, uint32_t bounce, uint32_t q, uint32_t n) {
    bool valid = q < n;
    uint32_t id = valid ? a.pb.queue[bounce & 1][q] : 0u;
    VertexOut v;
    if (valid) v = shade_vertex<GUIDE>(a, id, bounce);
    uint32_t slot = warp_push(v.alive, &a.counters->paths[bounce + 1]);
    if (v.alive) {
        a.pb.queue[(bounce + 1) & 1][slot] = id;
        if (a.ray_sort) a.pb.sort_keys[slot] = v.key;
    }
    uint32_t sslot = warp_push(v.shadow, &a.counters->shadow[bounce]);
    if (v.shadow) {
        a.pb.sh_o[sslot] = f4(v.sh_o.x, v.sh_o.y, v.sh_o.z, 0.001f);
        a.pb.sh_d[sslot] = f4(v.sh_d.x, v.sh_d.y, v.sh_d.z, v.sh_tmax);
        a.pb.sh_c[sslot] = v.sh_c;
        a.pb.sh_id[sslot] = id;
    }
    if (GUIDE) {
        uint32_t gslot = warp_push(v.guided, &a.guide.gc->verts[bounce]);
        if (v.guided) {
            a.guide.gv.p[gslot] = v.g_p;
            a.guide.gv.n[gslot] = v.g_n;
            a.guide.gv.wo[gslot] = v.g_wo;
            a.guide.gv.spec[gslot] = v.g_spec;
            a.guide.gv.id[gslot] = id;
        }
    }
}

template <bool GUIDE>
__global__ void __launch_bounds__(TRACE_BLOCK, SRT_SHADE_MIN_BLOCKS) k_shade(FrameArgs a, uint32_t bounce) {
    uint32_t n = a.counters->paths[bounce];
    if (blockIdx.x * blockDim.x >= n) return;
    shade_slot<GUIDE>(a, bounce, blockIdx.x * blockDim.x + threadIdx.x, n);
}

// The shading of many scenes in one launch (the batched renderer): a virtual
// queue concatenates the scenes' path queues of this bounce, each padded to
// whole blocks, so a block's chunk belongs to one scene; blocks draw chunks
// from *fetch and copy that scene's frame arguments into shared memory when
// the scene changes.  Per vertex the work is k_shade's (guided scenes write
// their Lambert vertices for the grouped guide inference).
__global__ void __launch_bounds__(TRACE_BLOCK, SRT_SHADE_MIN_BLOCKS)
    k_shade_multi(const FrameArgs* __restrict__ items, int n_items, uint32_t bounce, uint32_t* __restrict__ fetch) {
    __shared__ FrameArgs sa;
    __shared__ uint32_t pre[MAX_BATCH + 1];
    __shared__ uint32_t chunk;
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (int i = 0; i < n_items; ++i) {
            pre[i] = acc;
            acc += (items[i].counters->paths[bounce] + TRACE_BLOCK - 1u) / TRACE_BLOCK;
        }
        pre[n_items] = acc;
    }
    int cur = -1;
    constexpr int kWords = (int)(sizeof(FrameArgs) / sizeof(uint32_t));
    static_assert(sizeof(FrameArgs) % sizeof(uint32_t) == 0, "FrameArgs is copied as words");
    while (true) {
        __syncthreads();  // the previous chunk is done with `chunk` and `sa`
        if (threadIdx.x == 0) chunk = atomicAdd(fetch, 1u);
        __syncthreads();
        const uint32_t c = chunk;
        if (c >= pre[n_items]) break;
        int sc = 0;
        while (sc + 1 < n_items && pre[sc + 1] <= c) ++sc;
        if (sc != cur) {  // block-uniform
            const uint32_t* src = reinterpret_cast<const uint32_t*>(items + sc);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&sa);
            for (int k = (int)threadIdx.x; k < kWords; k += TRACE_BLOCK) dst[k] = src[k];
            cur = sc;
            __syncthreads();
        }
        const uint32_t n = sa.counters->paths[bounce];
        const uint32_t q = (c - pre[sc]) * TRACE_BLOCK + threadIdx.x;
        if (sa.guiding) shade_slot<true>(sa, bounce, q, n);
        else shade_slot<false>(sa, bounce, q, n);
    }
}

// Resident blocks per SM the tail kernel is compiled for (traversal and
// shading in one kernel: 4 blocks of 128 allow 128 registers).
#ifndef SRT_TAIL_MIN_BLOCKS
#define SRT_TAIL_MIN_BLOCKS 4
#endif

// The last bounces of the live paths in one persistent launch: each thread
// takes a path entering bounce `first` and follows it to its end (closest
// hit, shade_vertex, its shadow ray), then takes the next path.  Per path
// the operations and the order of its radiance updates are those of the
// bounce-by-bounce wavefront (the traversal rounds alike in every kernel), so
// the image is bit-identical; where few paths remain, one launch replaces a
// chain of launches that each last as long as their slowest ray.
template <bool GUIDE, bool COUNT, int STACK>
__global__ void __launch_bounds__(TRACE_BLOCK, SRT_TAIL_MIN_BLOCKS) k_tail(FrameArgs a, uint32_t first) {
    extern __shared__ uint2 stack_smem[];
    __shared__ uint32_t n_closest[MAX_BOUNCES + 1], n_shadow[MAX_BOUNCES + 1];
    for (uint32_t i = threadIdx.x; i <= (uint32_t)MAX_BOUNCES; i += blockDim.x) n_closest[i] = n_shadow[i] = 0u;
    __syncthreads();
    uint2* stack = stack_smem + threadIdx.x;
    const uint32_t n = a.counters->paths[first];
    uint32_t* fetch = &a.counters->fetch[TRAV_CLOSEST][first];
    const uint32_t* queue = a.pb.queue[first & 1];
    while (true) {
        const uint32_t q = atomicAdd(fetch, 1u);
        if (q >= n) break;
        const uint32_t id = queue[q];
        for (uint32_t b = first; b < a.max_depth; ++b) {
            if (b > first) atomicAdd(&n_closest[b], 1u);  // paths[first] was counted by the last shading step
            const float4 o = a.pb.ray_o[id], d = a.pb.ray_d[id];
            float t = 0.f, u = 0.f, v = 0.f;
            uint32_t prim;
            TravCounters tc{&a.stats->nodes_bounce[TRAV_CLOSEST][b], &a.stats->tris_bounce[TRAV_CLOSEST][b]};
            const bool h = traverse<false, COUNT, STACK>(a.scene, Ray{xyz(o), xyz(d), o.w, d.w}, stack, TRACE_BLOCK, t,
                                                         prim, u, v, a.err, tc);
            a.pb.hit[id] = h ? make_float4(t, __uint_as_float(prim), u, v) : make_float4(0.f, __uint_as_float(MISS), 0.f, 0.f);
            const VertexOut vo = shade_vertex<GUIDE>(a, id, b);
            if (vo.shadow) {
                atomicAdd(&n_shadow[b], 1u);
                TravCounters ts{&a.stats->nodes_bounce[TRAV_SHADOW][b], &a.stats->tris_bounce[TRAV_SHADOW][b]};
                const bool occluded = traverse<true, COUNT, STACK>(a.scene, Ray{vo.sh_o, vo.sh_d, 0.001f, vo.sh_tmax},
                                                                   stack, TRACE_BLOCK, t, prim, u, v, a.err, ts);
                if (!occluded) {  // as the shadow-ray kernel adds it (shader.wgsl:659-669)
                    const float4 r = a.pb.rad[id], c = vo.sh_c;
                    a.pb.rad[id] = make_float4(__fadd_rn(r.x, c.x), __fadd_rn(r.y, c.y), __fadd_rn(r.z, c.z),
                                               __fadd_rn(r.w, c.w));
                }
            }
            if (!vo.alive) break;
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i <= (uint32_t)MAX_BOUNCES; i += blockDim.x) {
        if (n_closest[i]) atomicAdd(&a.counters->paths[i], n_closest[i]);
        if (n_shadow[i]) atomicAdd(&a.counters->shadow[i], n_shadow[i]);
    }
}

// Resident blocks per SM of one k_tail instantiation (its grid is one wave).
template <bool GUIDE, bool COUNT, int STACK>
int tail_per_sm() {
    static int per_sm = 0;
    if (per_sm == 0) {
        int x = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&x, k_tail<GUIDE, COUNT, STACK>, TRACE_BLOCK,
                                                          sizeof(uint2) * STACK * TRACE_BLOCK) != cudaSuccess ||
            x < 1)
            x = 1;
        per_sm = x;
    }
    return per_sm;
}

template <bool GUIDE, bool COUNT, int STACK>
int launch_tail_t(const FrameArgs& a, uint32_t first, cudaStream_t st) {
    const size_t smem = sizeof(uint2) * STACK * TRACE_BLOCK;
    const uint32_t grid = (uint32_t)(a.sm_count > 0 ? a.sm_count : 148) * (uint32_t)tail_per_sm<GUIDE, COUNT, STACK>();
    k_tail<GUIDE, COUNT, STACK><<<grid, TRACE_BLOCK, smem, st>>>(a, first);
    return 1;
}

// shader.wgsl:774-822: hero tuple -> XYZ / sum pdf -> linear sRGB ->
// accumulate (reset at frame 0) -> mean -> Reinhard on luma -> RGBA8.
__global__ void k_finalize(FrameArgs a) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.width * a.height) return;
    float4 L = a.pb.rad[p], wl = a.pb.wl[p];
    float3 c = f3(0.f, 0.f, 0.f);
    c = c + sample_cie_xyz(wl.x) * L.x;
    c = c + sample_cie_xyz(wl.y) * L.y;
    c = c + sample_cie_xyz(wl.z) * L.z;
    c = c + sample_cie_xyz(wl.w) * L.w;
    c = c * (1.0f / hero_pdf_sum(wl));
    float3 rgb = xyz_to_srgb(c);
    uint32_t frame = a.cam->frame_count;
    float4 acc = frame > 0u ? a.accum[p] : splat4(0.f);
    acc = acc + f4(rgb.x, rgb.y, rgb.z, 1.0f);
    a.accum[p] = acc;
    if (a.accum64) {
        double4 d = frame > 0u ? a.accum64[p] : make_double4(0, 0, 0, 0);
        a.accum64[p] = make_double4(d.x + rgb.x, d.y + rgb.y, d.z + rgb.z, d.w + 1.0);
    }
    float3 fc = f3(fmaxf(acc.x / acc.w * 1.0f, 0.f), fmaxf(acc.y / acc.w * 1.0f, 0.f), fmaxf(acc.z / acc.w * 1.0f, 0.f));
    float luma = fc.x * 0.2126f + fc.y * 0.7152f + fc.z * 0.0722f;
    float mapped = luma / (luma + 1.0f);
    if (luma > 0.00001f) fc = fc * (mapped / luma);
    a.ldr[p] = make_uchar4((unsigned char)__float2uint_rn(clampf(fc.x, 0.f, 1.f) * 255.0f),
                           (unsigned char)__float2uint_rn(clampf(fc.y, 0.f, 1.f) * 255.0f),
                           (unsigned char)__float2uint_rn(clampf(fc.z, 0.f, 1.f) * 255.0f), 255);
}

__global__ void k_frame_stats(FrameArgs a) {
    if (threadIdx.x != 0) return;
    unsigned long long c = 0, s = 0;
    for (uint32_t i = 0; i < a.max_depth; ++i) {
        c += a.counters->paths[i];
        s += a.counters->shadow[i];
        a.stats->rays_bounce[TRAV_CLOSEST][i] += a.counters->paths[i];
        a.stats->rays_bounce[TRAV_SHADOW][i] += a.counters->shadow[i];
    }
    a.stats->closest_rays += c;
    a.stats->shadow_rays += s;
    a.stats->paths += a.counters->paths[0];
    unsigned long long pr = 0;
    if (a.photons_per_frame > 0u)
        for (uint32_t i = 0; i < a.photon_max_bounces; ++i) {
            pr += a.ph_counters->photon_paths[i];
            a.stats->rays_bounce[TRAV_PHOTON][i] += a.ph_counters->photon_paths[i];
        }
    a.stats->photon_rays += pr;
}

// ------------------------------------------------------------------ batch / test kernels
__global__ void k_gather_queries(GatherArgs g, uint32_t frame, const float* __restrict__ q, uint32_t n,
                                 float4* __restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = q + 10 * i;
    out[i] = gather(g, frame, f3(a[0], a[1], a[2]), f3(a[3], a[4], a[5]), f4(a[6], a[7], a[8], a[9]));
}

__global__ void k_test_math(int op, uint32_t n, const void* __restrict__ in, void* __restrict__ out,
                            const void* __restrict__ aux) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* fi = (const float*)in;
    const uint32_t* ui = (const uint32_t*)in;
    float* fo = (float*)out;
    uint32_t* uo = (uint32_t*)out;
    switch (op) {
        case 0:
            uo[i] = pcg_hash(ui[i]);
            break;
        case 1: {
            float3 c = sample_cie_xyz(fi[i]);
            fo[3 * i] = c.x;
            fo[3 * i + 1] = c.y;
            fo[3 * i + 2] = c.z;
        } break;
        case 2:
            fo[i] = blackbody(fi[2 * i], fi[2 * i + 1]);
            break;
        case 3: {
            const float* p = fi + 7 * i;
            float4 r = rgb_to_spectrum4(f3(p[0], p[1], p[2]), f4(p[3], p[4], p[5], p[6]));
            reinterpret_cast<float4*>(fo)[i] = r;
        } break;
        case 4: {
            const float* p = fi + 9 * i;
            reinterpret_cast<float4*>(fo)[i] = thin_film4(p[0], p[1], p[2], p[3], p[4], f4(p[5], p[6], p[7], p[8]));
        } break;
        case 5: {
            uint32_t s = ui[i];
            float4 w = sample_hero(s);
            float* o = fo + 5 * i;
            o[0] = w.x;
            o[1] = w.y;
            o[2] = w.z;
            o[3] = w.w;
            o[4] = hero_pdf_sum(w);
        } break;
        case 6: {
            const float* p = fi + 24 * i;
            uint32_t s = __float_as_uint(p[23]);
            Scatter sc = sample_bsdf(f3(p[0], p[1], p[2]), f3(p[3], p[4], p[5]), f4(p[6], p[7], p[8], p[9]),
                                     f4(p[10], p[11], p[12], p[13]), p[14] != 0.0f, f4(p[15], p[16], p[17], p[18]),
                                     f4(p[19], p[20], p[21], p[22]), s);
            float* o = fo + 10 * i;
            o[0] = sc.dir.x;
            o[1] = sc.dir.y;
            o[2] = sc.dir.z;
            o[3] = sc.att.x;
            o[4] = sc.att.y;
            o[5] = sc.att.z;
            o[6] = sc.att.w;
            o[7] = sc.absorbed ? 1.0f : 0.0f;
            o[8] = __uint_as_float(s);
            o[9] = 0.f;
        } break;
        case 7: {
            const float* p = fi + 5 * i;
            float3 j = grid_jitter(__float_as_uint(p[3]), p[4]);
            uo[i] = grid_hash(f3(p[0], p[1], p[2]), j, p[4], 22);
        } break;
        case 8: {
            const uint32_t* p = ui + 5 * i;
            uint32_t s = p[4];
            float3 o, d;
            camera_ray(*(const srt_camera_uniform*)aux, p[0], p[1], p[2], p[3], s, o, d);
            float* r = fo + 7 * i;
            r[0] = o.x;
            r[1] = o.y;
            r[2] = o.z;
            r[3] = d.x;
            r[4] = d.y;
            r[5] = d.z;
            r[6] = __uint_as_float(s);
        } break;
        default:
            break;
    }
}

inline uint32_t blocks_for(uint64_t n, uint32_t b) { return (uint32_t)((n + b - 1) / b); }

}  // namespace

// ------------------------------------------------------------------ launchers
int launch_photon_pass(FrameArgs& a, cudaStream_t st) {
    int launches = 0;
    const uint32_t n = a.photons_per_frame;
    // emit (with SRT_PHOTON_DIR_SORT, then order the emitted rays by direction)
    k_photon_emit<<<blocks_for(n, 256), 256, 0, st>>>(a);
    ++launches;
    uint32_t* order = nullptr;  // bounce-0 queue: emitter order
    if (SRT_PHOTON_DIR_SORT) {
        uint32_t* dir_keys;
        launches += sort_pairs(a.ph.keys, a.ph.vals, a.ph.keys2, a.ph.vals2, n, nullptr, 0, 24, a.ph.sort_scratch,
                               st, &dir_keys, &order);
    }
    a.ph.sorted_vals = order;  // bounce-0 queue (read by k_photon_shade at bounce 0)
    for (uint32_t b = 0; b < a.photon_max_bounces; ++b) {
        launches += launch_trace_queue(a.scene, b, b == 0 ? order : a.ph.queue[b & 1], &a.counters->photon_paths[b],
                                       &a.counters->fetch[TRAV_PHOTON][b], n, a.ph.ray_o, a.ph.ray_d, a.ph.hit,
                                       TRAV_PHOTON, a.count_visits, a.err, a.stats, a.sm_count, st);
        k_photon_shade<<<blocks_for(n, TRACE_BLOCK), TRACE_BLOCK, 0, st>>>(a, b);
        ++launches;
    }
    // stored photons in emitter order
    k_deposit_count<<<a.ph.n_blocks, PHOTON_BLOCK, 0, st>>>(a);
    k_rs_rowscan<<<1, 1024, 0, st>>>(a.ph.block_counts, a.ph.n_blocks, &a.counters->photons_stored);
    k_deposit_scatter<<<a.ph.n_blocks, PHOTON_BLOCK, 0, st>>>(a);
    launches += 3;
    uint32_t grid = 148 * 8;
    k_grid_keys<<<grid, 256, 0, st>>>(a.ph.photons, &a.counters->photons_stored, 0,
                                      &a.cam->frame_count, 0, a.gather.cell, a.gather.hash_bits, a.ph.keys, a.ph.vals);
    ++launches;
    launches += sort_pairs(a.ph.keys, a.ph.vals, a.ph.keys2, a.ph.vals2, a.ph.capacity, &a.counters->photons_stored, 0,
                           (int)a.gather.hash_bits + 1, a.ph.sort_scratch, st, &a.ph.sorted_keys, &a.ph.sorted_vals);
    cudaMemsetAsync(a.ph.ranges, 0, sizeof(uint2) << a.gather.hash_bits, st);
    k_grid_ranges<<<grid, 256, 0, st>>>(a.ph.sorted_keys, a.ph.sorted_vals, &a.counters->photons_stored, 0,
                                        a.gather.hash_bits, a.ph.photons, a.ph.sorted, a.ph.ranges);
    ++launches;
    return launches;
}

int launch_grid_build(const float4* photons, uint32_t n, uint32_t frame, float cell, uint32_t hash_bits,
                      PhotonBuffers& ph, cudaStream_t st) {
    int launches = 0;
    uint32_t grid = 148 * 8;
    k_grid_keys<<<grid, 256, 0, st>>>(photons, nullptr, n, nullptr, frame, cell, hash_bits, ph.keys, ph.vals);
    ++launches;
    launches += sort_pairs(ph.keys, ph.vals, ph.keys2, ph.vals2, n, nullptr, 0, (int)hash_bits + 1, ph.sort_scratch, st,
                           &ph.sorted_keys, &ph.sorted_vals);
    cudaMemsetAsync(ph.ranges, 0, sizeof(uint2) << hash_bits, st);
    k_grid_ranges<<<grid, 256, 0, st>>>(ph.sorted_keys, ph.sorted_vals, nullptr, n, hash_bits, photons, ph.sorted,
                                        ph.ranges);
    ++launches;
    return launches;
}

int launch_raygen(const FrameArgs& a, cudaStream_t st) {
    k_raygen<<<blocks_for((uint64_t)a.width * a.height, 256), 256, 0, st>>>(a);
    return 1;
}

int launch_bounce(const FrameArgs& a, uint32_t bounce, cudaStream_t st, int stage) {
    int launches = 0;
    uint32_t grid = blocks_for((uint64_t)a.width * a.height, TRACE_BLOCK);
    if (stage == 0 || stage == 1) launches += launch_trace_closest(a, bounce, st);
    if (stage == 0 || stage == 2 || stage == 4) {
        if (a.guiding) k_shade<true><<<grid, TRACE_BLOCK, 0, st>>>(a, bounce);
        else k_shade<false><<<grid, TRACE_BLOCK, 0, st>>>(a, bounce);
        ++launches;
        if (a.guiding && stage != 4 && bounce + 1 < a.max_depth && bounce < a.guide_bounces)
            launches += launch_guide_infer(a, bounce, st);
        if (a.ray_sort && bounce + 1 < a.max_depth) {
            // 4 passes: the sorted queue lands back in the queue buffer
            uint32_t *sk, *sv;
            launches += sort_pairs(a.pb.sort_keys, a.pb.queue[(bounce + 1) & 1], a.pb.sort_keys_alt,
                                   a.pb.sort_vals_alt, a.width * a.height, &a.counters->paths[bounce + 1], 0, 32,
                                   a.pb.sort_scratch, st, &sk, &sv);
        }
    }
    if (stage == 0 || stage == 3) launches += launch_trace_shadow(a, bounce, st);
    return launches;
}

int launch_shade_multi(const FrameArgs* items, int n_items, uint32_t bounce, uint32_t* fetch, int sm_count,
                       cudaStream_t st) {
    if (n_items <= 0) return 0;
    const uint32_t grid = (uint32_t)(sm_count > 0 ? sm_count : 148) * SRT_SHADE_MIN_BLOCKS;
    k_shade_multi<<<grid, TRACE_BLOCK, 0, st>>>(items, n_items, bounce, fetch);
    return 1;
}

int launch_finalize(const FrameArgs& a, cudaStream_t st) {
    k_finalize<<<blocks_for((uint64_t)a.width * a.height, 256), 256, 0, st>>>(a);
    return 1;
}

int launch_frame_stats(const FrameArgs& a, cudaStream_t st) {
    k_frame_stats<<<1, 32, 0, st>>>(a);
    return 1;
}

uint32_t tail_threads(const FrameArgs& a) {
    const bool small = a.scene.depth <= (uint32_t)TRAV_STACK_SMALL;
    const bool g = a.guiding != 0, c = a.count_visits != 0;
    int per_sm;
    if (c) per_sm = g ? (small ? tail_per_sm<true, true, TRAV_STACK_SMALL>() : tail_per_sm<true, true, TRAV_STACK>())
                      : (small ? tail_per_sm<false, true, TRAV_STACK_SMALL>() : tail_per_sm<false, true, TRAV_STACK>());
    else per_sm = g ? (small ? tail_per_sm<true, false, TRAV_STACK_SMALL>() : tail_per_sm<true, false, TRAV_STACK>())
                    : (small ? tail_per_sm<false, false, TRAV_STACK_SMALL>() : tail_per_sm<false, false, TRAV_STACK>());
    return (uint32_t)(a.sm_count > 0 ? a.sm_count : 148) * (uint32_t)per_sm * TRACE_BLOCK;
}

int launch_tail(const FrameArgs& a, uint32_t first, cudaStream_t st) {
    if (first >= a.max_depth) return 0;
    const bool small = a.scene.depth <= (uint32_t)TRAV_STACK_SMALL;
    const bool g = a.guiding != 0;
    if (a.count_visits) {
        if (g) return small ? launch_tail_t<true, true, TRAV_STACK_SMALL>(a, first, st) : launch_tail_t<true, true, TRAV_STACK>(a, first, st);
        return small ? launch_tail_t<false, true, TRAV_STACK_SMALL>(a, first, st) : launch_tail_t<false, true, TRAV_STACK>(a, first, st);
    }
    if (g) return small ? launch_tail_t<true, false, TRAV_STACK_SMALL>(a, first, st) : launch_tail_t<true, false, TRAV_STACK>(a, first, st);
    return small ? launch_tail_t<false, false, TRAV_STACK_SMALL>(a, first, st) : launch_tail_t<false, false, TRAV_STACK>(a, first, st);
}

int launch_gather_queries(const GatherArgs& g, uint32_t frame, const float* queries, uint32_t n_q, float4* out,
                          cudaStream_t st) {
    if (n_q == 0) return 0;
    k_gather_queries<<<blocks_for(n_q, 128), 128, 0, st>>>(g, frame, queries, n_q, out);
    return 1;
}

int launch_test_math(int op, uint32_t n, const void* in, void* out, const void* aux, cudaStream_t st) {
    if (n == 0) return 0;
    k_test_math<<<blocks_for(n, 128), 128, 0, st>>>(op, n, in, out, aux);
    return 1;
}

}  // namespace srt
