// device_common.cuh — device data layouts and shading math of the spectral
// path tracer (sm_100a).
//
// The shading functions follow the reference WGSL (path:line cited at each
// one) in FP32; they are written for the GPU (float4 SIMD-style helpers,
// register-resident state) and checked against the CPU oracle.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/srt.h"

#define SRT_DEV __device__ __forceinline__

namespace srt {

constexpr float PI = 3.14159265359f;  // shader.wgsl:6
constexpr float LAMBDA_MIN = 380.0f;  // shader.wgsl:81-83
constexpr float LAMBDA_MAX = 780.0f;
constexpr float LAMBDA_RANGE = LAMBDA_MAX - LAMBDA_MIN;
constexpr uint32_t MISS = 0xFFFFFFFFu;
constexpr int TRAV_STACK = 32;        // BVH8 traversal stack entries per thread (deepest supported tree)
constexpr int TRAV_STACK_SMALL = 16;  // stack for trees of at most 16 levels (less shared memory, more warps)

// Device error word bits (read back by the host after synchronising).
constexpr uint32_t ERR_STACK_OVERFLOW = 0x1u;
constexpr uint32_t ERR_QUEUE_OVERFLOW = 0x2u;
constexpr uint32_t ERR_BAD_INDEX = 0x4u;

// ------------------------------------------------------------------ layouts
// Per instance (64 B): mesh/material ids, first flattened triangle and the
// rows of world_to_object (inverse of the instance's linear part).
struct InstDev {
    uint32_t mesh_id, mat_id, tri_offset, tri_count;
    float4 w2o0, w2o1, w2o2;  // rows; .w unused
};

// Compressed 8-wide BVH node, 80 B = 5 x uint4 (layout of Ylitie, Karras and
// Laine, HPG 2017):
//  w0..2  origin p (float x3)     w3  exponent bytes ex, ey, ez, imask
//  w4     first child node index  w5  first triangle slot index
//  w6..7  meta[8]: 0 empty; (7 << 5) internal child; (count << 5) | offset
//         for a leaf of `count` (1..3) triangles starting at
//         first triangle slot + offset
//  w8..19 qlo.x[8] qlo.y[8] qlo.z[8] qhi.x[8] qhi.y[8] qhi.z[8]
// Child bounds = p + 2^(e-127) * q.
struct Node8 {
    uint4 a, b, c, d, e;
};
static_assert(sizeof(Node8) == 80, "Node8 must be 80 bytes");

// A leaf triangle slot (48 B): world-space v0.xyz + flattened triangle id
// (bits in .w), v1.xyz, v2.xyz.
struct TriSlot {
    float4 v0, v1, v2;
};

struct DevScene {
    const float4* vtx;          // srt_vertex: pos, normal
    const uint32_t* indices;
    const uint4* mesh_infos;    // srt_mesh_info
    const float4* materials;    // srt_material: color, extra
    const float4* lights;       // srt_light: v0, v1, v2, params
    uint32_t n_lights;
    const InstDev* inst;
    const uint32_t* tri_inst;   // flattened triangle -> instance
    const Node8* nodes;
    const TriSlot* tris;
    uint32_t n_nodes;
    uint32_t n_tris;
    uint32_t depth;  // 8-wide levels: a traversal stack needs at least this many entries
    float4 bmin;     // world bounds of the scene (xyz), for ray sort keys
    float4 binv;     // 1 / extent of the bounds (xyz)
};

// ------------------------------------------------------------------ vector helpers
SRT_DEV float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
SRT_DEV float3 xyz(float4 a) { return make_float3(a.x, a.y, a.z); }
SRT_DEV float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
SRT_DEV float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
SRT_DEV float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
SRT_DEV float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
SRT_DEV float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
SRT_DEV float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
SRT_DEV float3 cross(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
SRT_DEV float length(float3 a) { return sqrtf(dot(a, a)); }
SRT_DEV float3 normalize(float3 a) { return a / length(a); }
SRT_DEV float3 reflect(float3 i, float3 n) { return i - n * (2.0f * dot(n, i)); }
SRT_DEV float3 refract(float3 i, float3 n, float eta) {
    float ni = dot(n, i);
    float k = 1.0f - eta * eta * (1.0f - ni * ni);
    if (k < 0.0f) return f3(0.f, 0.f, 0.f);
    return i * eta - n * (eta * ni + sqrtf(k));
}
SRT_DEV float4 f4(float x, float y, float z, float w) { return make_float4(x, y, z, w); }
SRT_DEV float4 splat4(float s) { return make_float4(s, s, s, s); }
SRT_DEV float4 operator+(float4 a, float4 b) { return f4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
SRT_DEV float4 operator-(float4 a, float4 b) { return f4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
SRT_DEV float4 operator*(float4 a, float4 b) { return f4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }
SRT_DEV float4 operator/(float4 a, float4 b) { return f4(a.x / b.x, a.y / b.y, a.z / b.z, a.w / b.w); }
SRT_DEV float4 operator*(float4 a, float s) { return f4(a.x * s, a.y * s, a.z * s, a.w * s); }
SRT_DEV float4 operator/(float4 a, float s) { return f4(a.x / s, a.y / s, a.z / s, a.w / s); }
SRT_DEV float max4(float4 a) { return fmaxf(fmaxf(a.x, a.y), fmaxf(a.z, a.w)); }
SRT_DEV float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
SRT_DEV float sq(float x) { return x * x; }
SRT_DEV float signf(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }

// ------------------------------------------------------------------ RNG (shader.wgsl:144-169)
SRT_DEV uint32_t pcg_hash(uint32_t input) {
    uint32_t state = input * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
// rand(): f32(u32) / 4294967295.0 — the f32 constant is 2^32, so the
// quotient is an exact scaling of the rounded u32.
SRT_DEV float rng_next(uint32_t& s) {
    s = pcg_hash(s);
    return __fdiv_rn(__uint2float_rn(s), 4294967296.0f);
}
SRT_DEV float3 random_unit_vector(uint32_t& s) {
    float u1 = rng_next(s);
    float u2 = rng_next(s);
    float z = 1.0f - 2.0f * u1;
    float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    float phi = 2.0f * PI * u2;
    float sp, cp;
    sincosf(phi, &sp, &cp);
    return f3(r * cp, r * sp, z);
}

// ------------------------------------------------------------------ spectra
// sample_cie_xyz: shader.wgsl:85-97 (pow(x, 2.0) read as x*x)
SRT_DEV float3 sample_cie_xyz(float l) {
    float x = expf(-sq((l - 599.8f) / 37.9f)) * 1.056f + expf(-sq((l - 442.0f) / 16.0f)) * 0.362f -
              expf(-sq((l - 501.1f) / 26.7f)) * 0.065f;
    float y = expf(-sq((l - 568.8f) / 46.9f)) * 0.821f + expf(-sq((l - 530.9f) / 16.3f)) * 0.286f;
    float z = expf(-sq((l - 437.0f) / 11.8f)) * 1.217f + expf(-sq((l - 459.0f) / 26.0f)) * 0.681f;
    return f3(fmaxf(0.0f, x), fmaxf(0.0f, y), fmaxf(0.0f, z));
}
// XYZ_TO_SRGB: shader.wgsl:100-104
SRT_DEV float3 xyz_to_srgb(float3 c) {
    return f3(3.2404542f * c.x - 1.5371385f * c.y - 0.4985314f * c.z,
              -0.9692660f * c.x + 1.8760108f * c.y + 0.0415560f * c.z,
              0.0556434f * c.x - 0.2040259f * c.y + 1.0572252f * c.z);
}
// rgb_to_spectrum_eval: shader.wgsl:106-117
SRT_DEV float rgb_to_spectrum(float3 rgb, float l) {
    float white = fminf(rgb.x, fminf(rgb.y, rgb.z));
    float cr = fmaxf(rgb.x - white, 0.f), cg = fmaxf(rgb.y - white, 0.f), cb = fmaxf(rgb.z - white, 0.f);
    float r = cr * expf(-sq((l - 630.0f) / 20.0f));
    float g = cg * expf(-sq((l - 525.0f) / 20.0f));
    float b = cb * expf(-sq((l - 460.0f) / 20.0f));
    return clampf(white + r + g + b, 0.0f, 0.99f);
}
SRT_DEV float4 rgb_to_spectrum4(float3 rgb, float4 wl) {
    return f4(rgb_to_spectrum(rgb, wl.x), rgb_to_spectrum(rgb, wl.y), rgb_to_spectrum(rgb, wl.z),
              rgb_to_spectrum(rgb, wl.w));
}
// blackbody_radiance: shader.wgsl:128-139
SRT_DEV float blackbody(float lambda_nm, float temp_k) {
    float lm = lambda_nm * 1e-9f;
    const float h = 6.62607015e-34f, c = 299792458.0f, k = 1.380649e-23f;
    float c1 = 2.0f * h * c * c;
    float c2 = (h * c) / (k * temp_k);
    return c1 / (powf(lm, 5.0f) * (expf(c2 / lm) - 1.0f)) * 1e-13f;
}
SRT_DEV float4 blackbody4(float4 wl, float t) {
    return f4(blackbody(wl.x, t), blackbody(wl.y, t), blackbody(wl.z, t), blackbody(wl.w, t));
}

// ------------------------------------------------------------------ BSDF math
// Airy reflectance of a film, one wavelength (photon_emit.wgsl:107-132;
// the vec4 form shader.wgsl:233-262 runs the same per component).
// Returns 1 and sets tir on total internal reflection.
SRT_DEV float thin_film1(float cos1, float n1, float n2, float n3, float d, float lambda, bool& tir) {
    float s1 = fmaxf(0.0f, 1.0f - cos1 * cos1);
    float s2 = (n1 / n2) * (n1 / n2) * s1;
    tir = true;
    if (s2 >= 1.0f) return 1.0f;
    float c2 = sqrtf(1.0f - s2);
    float s3 = (n1 / n3) * (n1 / n3) * s1;
    if (s3 >= 1.0f) return 1.0f;
    tir = false;
    float c3 = sqrtf(1.0f - s3);
    float r12 = (n1 * cos1 - n2 * c2) / (n1 * cos1 + n2 * c2);
    float r23 = (n2 * c2 - n3 * c3) / (n2 * c2 + n3 * c3);
    float a = r12 * r12, b = r23 * r23;
    float cd = cosf((4.0f * PI * n2 * d * c2) / lambda);
    float num = a + b + 2.0f * r12 * r23 * cd;
    float den = 1.0f + a * b + 2.0f * r12 * r23 * cd;
    return clampf(num / den, 0.0f, 1.0f);
}
SRT_DEV float4 thin_film4(float cos1, float n1, float n2, float n3, float d, float4 wl) {
    bool tir;
    float x = thin_film1(cos1, n1, n2, n3, d, wl.x, tir);
    if (tir) return splat4(1.0f);
    return f4(x, thin_film1(cos1, n1, n2, n3, d, wl.y, tir), thin_film1(cos1, n1, n2, n3, d, wl.z, tir),
              thin_film1(cos1, n1, n2, n3, d, wl.w, tir));
}
// reflectance (Schlick): shader.wgsl:264-268
SRT_DEV float schlick(float cosine, float ri) {
    float r0 = (1.0f - ri) / (1.0f + ri);
    r0 = r0 * r0;
    return r0 + (1.0f - r0) * powf(1.0f - cosine, 5.0f);
}
SRT_DEV float g1_schlick_ggx(float nv, float r) {  // shader.wgsl:207-213
    float k = (r * r) / 2.0f;
    return nv / (nv * (1.0f - k) + k);
}
// GGX half vector in the frame of n (shader.wgsl:171-205; the basis keeps
// the reference's division by sign(n.z) + n.z).
SRT_DEV float3 ggx_half_vector(float3 n, float alpha, uint32_t& s) {
    float a2 = alpha * alpha;
    float r1 = rng_next(s);
    float r2 = rng_next(s);
    float phi = 2.0f * PI * r1;
    float ct = sqrtf((1.0f - r2) / (1.0f + (a2 - 1.0f) * r2));
    float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
    float sp, cp;
    sincosf(phi, &sp, &cp);
    float3 h = f3(cp * st, sp * st, ct);
    float sg = signf(n.z);
    float a = -1.0f / (sg + n.z);
    float b = n.x * n.y * a;
    float3 right = f3(1.0f + sg * n.x * n.x * a, sg * b, -sg * n.x);
    float3 up = f3(b, sg + n.y * n.y * a, -n.y);
    return normalize(right * h.x + up * h.y + n * h.z);
}

struct Scatter {
    float3 dir;
    float4 att;
    bool absorbed;
};

// sample_bsdf: shader.wgsl:347-471.  Type 5 (no reference counterpart):
// GGX sampling as type 1 with the film's Airy reflectance in place of
// Schlick's F; roughness in color.w, film d/n2/n3 in extra.yzw.
SRT_DEV Scatter sample_bsdf(float3 r_dir, float3 ffn, float4 color, float4 extra, bool front, float4 wl,
                            float4 thr, uint32_t& s) {
    Scatter rec;
    rec.absorbed = false;
    rec.dir = f3(0.f, 0.f, 0.f);
    rec.att = splat4(0.f);
    uint32_t type = (uint32_t)extra.x;
    float4 spec = rgb_to_spectrum4(xyz(color), wl);
    if (type == 1u || type == 5u) {
        float alpha = fmaxf(type == 1u ? extra.y : color.w, 0.001f);
        float3 v = normalize(-r_dir);
        float3 h = ggx_half_vector(ffn, alpha, s);
        float3 l = reflect(-v, h);
        float nl = dot(ffn, l), nv = dot(ffn, v);
        if (nl > 0.0f && nv > 0.0f) {
            float nh = fmaxf(dot(ffn, h), 0.0f);
            float vh = fmaxf(dot(v, h), 0.0f);
            float4 F;
            if (type == 1u) {
                float p = powf(clampf(1.0f - vh, 0.0f, 1.0f), 5.0f);
                F = spec + (splat4(1.0f) - spec) * p;
            } else {
                F = thin_film4(vh, 1.0f, extra.z, extra.w, fmaxf(extra.y, 50.0f), wl);
            }
            float G = g1_schlick_ggx(nl, alpha) * g1_schlick_ggx(nv, alpha);
            rec.att = (F * G * vh) / fmaxf(nv * nh, 0.0001f);
            rec.dir = l;
        } else {
            rec.absorbed = true;
        }
    } else if (type == 2u) {
        float lum = wl.x / 1000.0f;
        float ir = extra.z + (extra.w / (lum * lum));
        float ratio = front ? 1.0f / ir : ir;
        float3 u = normalize(r_dir);
        float ct = fminf(dot(-u, ffn), 1.0f);
        float si2 = fmaxf(0.0f, 1.0f - ct * ct);
        float st2 = ratio * ratio * si2;
        if (st2 >= 1.0f) {
            rec.dir = reflect(u, ffn);
            rec.att = splat4(1.0f);
        } else {
            float ctt = sqrtf(1.0f - st2);
            if (schlick(front ? ct : ctt, ratio) > rng_next(s)) {
                rec.dir = reflect(u, ffn);
                rec.att = splat4(1.0f);
            } else {
                rec.dir = refract(u, ffn, ratio);
                float4 base = spec * (ratio * ratio);
                if (extra.w > 0.0f) {
                    bool collapsed = thr.y < 0.0001f && thr.z < 0.0001f && thr.w < 0.0001f;
                    rec.att = f4(base.x * (collapsed ? 1.0f : 4.0f), 0.f, 0.f, 0.f);
                } else {
                    rec.att = base;
                }
            }
        }
    } else if (type == 4u) {
        float3 u = normalize(r_dir);
        float c1 = fminf(dot(-u, ffn), 1.0f);
        float4 F = thin_film4(c1, 1.0f, extra.z, extra.w, fmaxf(extra.y, 50.0f), wl);
        float p = F.x;
        if (rng_next(s) < p) {
            rec.dir = reflect(u, ffn);
            rec.att = F / p;
        } else {
            rec.dir = u;
            rec.att = (splat4(1.0f) - F) / (1.0f - p);
        }
    } else {
        float3 d = ffn + random_unit_vector(s);
        if (length(d) < 0.001f) d = ffn;
        rec.dir = normalize(d);
        rec.att = spec;
    }
    return rec;
}

// Hero wavelengths (shader.wgsl:734-767) and the sum of their pdfs (:782-797).
SRT_DEV float cauchy_cdf(float x) { return (1.0f / PI) * atanf((x - 555.0f) / 40.0f) + 0.5f; }
SRT_DEV float lambda_wrap(float x) {  // WGSL float %: e1 - e2 * trunc(e1 / e2)
    float a = x - LAMBDA_MIN;
    return LAMBDA_MIN + (a - LAMBDA_RANGE * truncf(a / LAMBDA_RANGE));
}
SRT_DEV float4 sample_hero(uint32_t& s) {
    float cmin = cauchy_cdf(LAMBDA_MIN), cmax = cauchy_cdf(LAMBDA_MAX);
    float u = cmin + rng_next(s) * (cmax - cmin);
    float hero = clampf(555.0f + 40.0f * tanf(PI * (u - 0.5f)), LAMBDA_MIN, LAMBDA_MAX);
    const float q = LAMBDA_RANGE / 4.0f;
    float4 w = f4(lambda_wrap(hero), lambda_wrap(hero + q), lambda_wrap(hero + q * 2.0f), lambda_wrap(hero + q * 3.0f));
    float rot = rng_next(s);
    if (rot < 0.25f) {
    } else if (rot < 0.5f) {
        w = f4(w.y, w.z, w.w, w.x);
    } else if (rot < 0.75f) {
        w = f4(w.z, w.w, w.x, w.y);
    } else {
        w = f4(w.w, w.x, w.y, w.z);
    }
    return w;
}
SRT_DEV float hero_pdf_sum(float4 w) {
    float cmin = cauchy_cdf(LAMBDA_MIN), cmax = cauchy_cdf(LAMBDA_MAX);
    float norm = 1.0f / ((cmax - cmin) * PI * 40.0f);
    float a = (w.x - 555.0f) / 40.0f, b = (w.y - 555.0f) / 40.0f, c = (w.z - 555.0f) / 40.0f,
          d = (w.w - 555.0f) / 40.0f;
    return norm / (1.0f + a * a) + norm / (1.0f + b * b) + norm / (1.0f + c * c) + norm / (1.0f + d * d);
}

// ------------------------------------------------------------------ photon grid hashing
// get_grid_jitter + hash_position: build_grid.wgsl:25-52.  Written with
// explicitly rounded intrinsics so that no multiply-add is contracted: the
// cell keys are compared bit for bit.
SRT_DEV float3 grid_jitter(uint32_t frame, float cell) {
    uint32_t seed = pcg_hash(frame * 114514u);
    float rx = __fdiv_rn(__uint2float_rn(seed & 0xFFu), 255.0f);
    float ry = __fdiv_rn(__uint2float_rn((seed >> 8u) & 0xFFu), 255.0f);
    float rz = __fdiv_rn(__uint2float_rn((seed >> 16u) & 0xFFu), 255.0f);
    return f3(__fmul_rn(__fsub_rn(rx, 0.5f), cell), __fmul_rn(__fsub_rn(ry, 0.5f), cell),
              __fmul_rn(__fsub_rn(rz, 0.5f), cell));
}
SRT_DEV uint32_t grid_hash(float3 p, float3 j, float cell, uint32_t hash_bits) {
    // f32 -> i32 conversion saturates as in WGSL (cvt.rzi.s32.f32 does)
    int gx = __float2int_rz(floorf(__fdiv_rn(__fadd_rn(p.x, j.x), cell)));
    int gy = __float2int_rz(floorf(__fdiv_rn(__fadd_rn(p.y, j.y), cell)));
    int gz = __float2int_rz(floorf(__fdiv_rn(__fadd_rn(p.z, j.z), cell)));
    uint32_t h = ((uint32_t)gx * 73856093u) ^ ((uint32_t)gy * 19349663u) ^ ((uint32_t)gz * 83492791u);
    return h & ((1u << hash_bits) - 1u);
}

// ------------------------------------------------------------------ camera ray (shader.wgsl:713-728)
SRT_DEV void camera_ray(const srt_camera_uniform& cam, uint32_t x, uint32_t y, uint32_t w, uint32_t h,
                        uint32_t& s, float3& o, float3& d) {
    const float* vi = cam.view_inverse;
    const float* pi = cam.proj_inverse;
    float jx = rng_next(s);
    float jy = rng_next(s);
    float nx = ((float)x + jx) / (float)w * 2.0f - 1.0f;
    float ny = ((float)y + jy) / (float)h * 2.0f - 1.0f;
    float t[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        // row r of (view_inv * proj_inv), then times (nx, ny, 1, 1)
        float m0 = vi[r] * pi[0] + vi[4 + r] * pi[1] + vi[8 + r] * pi[2] + vi[12 + r] * pi[3];
        float m1 = vi[r] * pi[4] + vi[4 + r] * pi[5] + vi[8 + r] * pi[6] + vi[12 + r] * pi[7];
        float m2 = vi[r] * pi[8] + vi[4 + r] * pi[9] + vi[8 + r] * pi[10] + vi[12 + r] * pi[11];
        float m3 = vi[r] * pi[12] + vi[4 + r] * pi[13] + vi[8 + r] * pi[14] + vi[12 + r] * pi[15];
        t[r] = m0 * nx + m1 * ny + m2 + m3;
    }
    o = f3(vi[12], vi[13], vi[14]);
    d = normalize(f3(t[0] / t[3], t[1] / t[3], t[2] / t[3]) - o);
}

// ------------------------------------------------------------------ traversal
struct Ray {
    float3 o, d;
    float tmin, tmax;
};

// Watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2013) with the
// FP64 fallback for edge functions that evaluate to exactly zero.
struct RayShear {
    int kx, ky, kz;
    float sx, sy, sz;
};
SRT_DEV float comp(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
SRT_DEV RayShear make_shear(float3 d) {
    RayShear r;
    float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    r.kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    r.kx = r.kz == 2 ? 0 : r.kz + 1;
    r.ky = r.kx == 2 ? 0 : r.kx + 1;
    float dz = comp(d, r.kz);
    if (dz < 0.0f) {
        int t = r.kx;
        r.kx = r.ky;
        r.ky = t;
    }
    r.sx = comp(d, r.kx) / dz;
    r.sy = comp(d, r.ky) / dz;
    r.sz = 1.0f / dz;
    return r;
}
SRT_DEV float comp_i(float3 v, uint32_t k) { return k == 0u ? v.x : (k == 1u ? v.y : v.z); }
// The watertight test on vertices v0, v1, v2 for a ray from o sheared by
// (kx, ky, kz, sx, sy, sz).  Every rounding is written out (explicit fused
// multiply-adds and products), so the test gives the same bits in every
// translation unit whatever its contraction setting.  Returns true on a hit
// with tmin <= t <= tmax; u, v = weights of v1, v2.
SRT_DEV bool tri_test(float3 v0, float3 v1, float3 v2, float3 o, uint32_t kx, uint32_t ky, uint32_t kz, float sx,
                      float sy, float sz, float tmin, float tmax, float& t, float& u, float& v) {
    const float3 A = v0 - o, B = v1 - o, C = v2 - o;
    const float Az = comp_i(A, kz), Bz = comp_i(B, kz), Cz = comp_i(C, kz);
    const float Ax = fmaf(-sx, Az, comp_i(A, kx)), Ay = fmaf(-sy, Az, comp_i(A, ky));
    const float Bx = fmaf(-sx, Bz, comp_i(B, kx)), By = fmaf(-sy, Bz, comp_i(B, ky));
    const float Cx = fmaf(-sx, Cz, comp_i(C, kx)), Cy = fmaf(-sy, Cz, comp_i(C, ky));
    float U = fmaf(Cx, By, -__fmul_rn(Cy, Bx));
    float V = fmaf(Ax, Cy, -__fmul_rn(Ay, Cx));
    float W = fmaf(Bx, Ay, -__fmul_rn(By, Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {  // FP64 fallback: exact products
        U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
        V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = __fadd_rn(__fadd_rn(U, V), W);
    if (det == 0.0f) return false;
    const float inv = __frcp_rn(det);
    const float T = fmaf(W, __fmul_rn(sz, Cz), fmaf(V, __fmul_rn(sz, Bz), __fmul_rn(U, __fmul_rn(sz, Az))));
    const float tt = __fmul_rn(T, inv);
    if (!(tt >= tmin && tt <= tmax)) return false;
    t = tt;
    u = __fmul_rn(V, inv);
    v = __fmul_rn(W, inv);
    return true;
}
SRT_DEV bool intersect_tri(const Ray& ray, const RayShear& sh, float3 v0, float3 v1, float3 v2, float& t, float& u,
                           float& v) {
    return tri_test(v0, v1, v2, ray.o, (uint32_t)sh.kx, (uint32_t)sh.ky, (uint32_t)sh.kz, sh.sx, sh.sy, sh.sz,
                    ray.tmin, ray.tmax, t, u, v);
}

SRT_DEV uint32_t byte_of(uint32_t w, int i) { return (w >> (8 * i)) & 0xFFu; }
// Byte k of w plus 2^23 as a float, without the integer-to-float conversion
// unit: one byte permute builds the bit pattern 0x4B0000bb (= 2^23 + b
// exactly).  The slab test folds the 2^23 bias into its addend,
// t = fma(2^23 + q, a, b - 2^23 a), whose rounding moves a plane by at most
// half a quantum; the builder pads every child box by one quantum.
SRT_DEV float qbyte(uint32_t w, uint32_t k) { return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7440u | k)); }
SRT_DEV float unbias(float a, float b) { return fmaf(-8388608.0f, a, b); }

// Two fused multiply-adds: one packed fma.rn.f32x2 with SRT_TRAV_FMA2 (the
// slab test of a child computes its near and far plane of an axis at once;
// measured 1.3 % off a config-2 frame), two scalar ones otherwise.  Both
// round each lane once, like fmaf.
#ifndef SRT_TRAV_FMA2
#define SRT_TRAV_FMA2 1
#endif
SRT_DEV float2 fma2(float2 a, float2 b, float2 c) {
#if SRT_TRAV_FMA2
    uint64_t x, y, z, r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(x) : "f"(a.x), "f"(a.y));
    asm("mov.b64 %0, {%1, %2};" : "=l"(y) : "f"(b.x), "f"(b.y));
    asm("mov.b64 %0, {%1, %2};" : "=l"(z) : "f"(c.x), "f"(c.y));
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(x), "l"(y), "l"(z));
    float2 o;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(o.x), "=f"(o.y) : "l"(r));
    return o;
#else
    return make_float2(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y));
#endif
}

// Child bookkeeping of a node visit in one pass after the slab tests
// (SRT_TRAV_LEAN, the default: a hit mask from the child loop, then the octant
// order of the internal children and the leaves' triangle bits once per node)
// instead of per child (config-2 closest-hit 3.35 vs 3.43 ms per frame).
#ifndef SRT_TRAV_LEAN
#define SRT_TRAV_LEAN 1
#endif

struct TravCounters {
    unsigned long long* nodes;
    unsigned long long* tris;
};

// Asynchronous 16-byte copies global -> shared (cp.async, L1-cached): a
// lane starts fetching the next node into its shared-memory slot, tests
// the pending triangles meanwhile, then waits for its own copies.
SRT_DEV void cp_async16(void* smem, const void* gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
SRT_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
SRT_DEV void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
// Node idx into this lane's slot: 5 chunks, chunk k at nbuf[k * stride].
SRT_DEV void fetch_node_async(const DevScene& S, uint32_t idx, uint4* nbuf, int stride) {
    const uint4* np = reinterpret_cast<const uint4*>(S.nodes + idx);
#pragma unroll
    for (int k = 0; k < 5; ++k) cp_async16(nbuf + k * stride, np + k);
    cp_async_commit();
}

// Child slab tests of one node (words w0..w4) for a ray with inverse
// direction idir and octant oct: the node's hit internal children (bits
// 24..31, ordered by octant) | imask, and its hit triangle bits.
SRT_DEV void node_children(uint4 w0, uint4 w1, uint4 w2, uint4 w3, uint4 w4, float3 o, float3 idir, uint32_t oct,
                           float tmin, float tbest, uint2& g, uint2& tg) {
    float sx = __uint_as_float((w0.w & 0xFFu) << 23), sy = __uint_as_float(((w0.w >> 8) & 0xFFu) << 23),
          sz = __uint_as_float(((w0.w >> 16) & 0xFFu) << 23);
    uint32_t imask = w0.w >> 24;
    float ax = sx * idir.x, ay = sy * idir.y, az = sz * idir.z;
    float bx = unbias(ax, (__uint_as_float(w0.x) - o.x) * idir.x), by = unbias(ay, (__uint_as_float(w0.y) - o.y) * idir.y),
          bz = unbias(az, (__uint_as_float(w0.z) - o.z) * idir.z);
    uint32_t nx0 = (oct & 1u) ? w3.z : w2.x, nx1 = (oct & 1u) ? w3.w : w2.y;
    uint32_t fx0 = (oct & 1u) ? w2.x : w3.z, fx1 = (oct & 1u) ? w2.y : w3.w;
    uint32_t ny0 = (oct & 2u) ? w4.x : w2.z, ny1 = (oct & 2u) ? w4.y : w2.w;
    uint32_t fy0 = (oct & 2u) ? w2.z : w4.x, fy1 = (oct & 2u) ? w2.w : w4.y;
    uint32_t nz0 = (oct & 4u) ? w4.z : w3.x, nz1 = (oct & 4u) ? w4.w : w3.y;
    uint32_t fz0 = (oct & 4u) ? w3.x : w4.z, fz1 = (oct & 4u) ? w3.y : w4.w;
    const float robust = 1.0000004f;
#if SRT_TRAV_LEAN
    // the child loop only collects which slots are hit; the octant order of
    // the internal children and the leaves' triangle bits follow once per node
    uint32_t hitmask = 0u;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t k = (uint32_t)(i & 3);
        const uint32_t m = byte_of(i < 4 ? w1.z : w1.w, k);
        const float2 tx = fma2(make_float2(qbyte(i < 4 ? nx0 : nx1, k), qbyte(i < 4 ? fx0 : fx1, k)),
                               make_float2(ax, ax), make_float2(bx, bx));
        const float2 ty = fma2(make_float2(qbyte(i < 4 ? ny0 : ny1, k), qbyte(i < 4 ? fy0 : fy1, k)),
                               make_float2(ay, ay), make_float2(by, by));
        const float2 tz = fma2(make_float2(qbyte(i < 4 ? nz0 : nz1, k), qbyte(i < 4 ? fz0 : fz1, k)),
                               make_float2(az, az), make_float2(bz, bz));
        const float tn = fmaxf(fmaxf(tx.x, ty.x), fmaxf(tz.x, tmin));
        const float tf = fminf(fminf(tx.y, ty.y), fminf(tz.y, tbest)) * robust;
        hitmask |= (m != 0u && tn <= tf) ? (1u << i) : 0u;
    }
    // internal children: slot i -> bit i ^ (oct ^ 7) (three conditional swaps)
    uint32_t ib = hitmask & imask;
    const uint32_t x = oct ^ 7u;
    ib = (x & 1u) ? (((ib & 0x55u) << 1) | ((ib >> 1) & 0x55u)) : ib;
    ib = (x & 2u) ? (((ib & 0x33u) << 2) | ((ib >> 2) & 0x33u)) : ib;
    ib = (x & 4u) ? (((ib & 0x0Fu) << 4) | ((ib >> 4) & 0x0Fu)) : ib;
    // leaves: their triangles' bits
    uint32_t lb = hitmask & ~imask, tris = 0u;
    while (lb != 0u) {
        const uint32_t i = (uint32_t)(__ffs(lb) - 1);
        lb &= lb - 1u;
        const uint32_t m = ((i < 4u ? w1.z : w1.w) >> (8u * (i & 3u))) & 0xFFu;
        tris |= ((1u << (m >> 5)) - 1u) << (m & 31u);
    }
    g = make_uint2(w1.x, (ib << 24) | imask);
    tg = make_uint2(w1.y, tris);
#else
    uint32_t hits = 0u;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t k = (uint32_t)(i & 3);
        uint32_t m = byte_of(i < 4 ? w1.z : w1.w, k);
        const float2 tx = fma2(make_float2(qbyte(i < 4 ? nx0 : nx1, k), qbyte(i < 4 ? fx0 : fx1, k)),
                               make_float2(ax, ax), make_float2(bx, bx));
        const float2 ty = fma2(make_float2(qbyte(i < 4 ? ny0 : ny1, k), qbyte(i < 4 ? fy0 : fy1, k)),
                               make_float2(ay, ay), make_float2(by, by));
        const float2 tz = fma2(make_float2(qbyte(i < 4 ? nz0 : nz1, k), qbyte(i < 4 ? fz0 : fz1, k)),
                               make_float2(az, az), make_float2(bz, bz));
        float tn = fmaxf(fmaxf(tx.x, ty.x), fmaxf(tz.x, tmin));
        float tf = fminf(fminf(tx.y, ty.y), fminf(tz.y, tbest)) * robust;
        if (m != 0u && tn <= tf) {
            uint32_t c = m >> 5;
            if (c == 7u) hits |= 1u << (24 + ((uint32_t)i ^ (oct ^ 7u)));
            else hits |= ((1u << c) - 1u) << (m & 31u);
        }
    }
    g = make_uint2(w1.x, (hits & 0xFF000000u) | imask);
    tg = make_uint2(w1.y, hits & 0x00FFFFFFu);
#endif
}

// Stack-based traversal of the compressed BVH8.  A node group holds the
// hit internal children of one node (bits 24..31 of .y, ordered so that the
// highest bit is the nearest child for this ray octant) plus the node's
// imask (bits 0..7); triangle hits go straight to the triangle loop.
// ANY: return at the first hit in [tmin, tmax].  Closest: lexicographic
// minimum of (t, flattened triangle id), independent of traversal order.
// `stack` is this thread's slice of shared memory, stride `stride` entries,
// STACK entries deep (at least the tree depth: one entry per level).
template <bool ANY, bool COUNT, int STACK = TRAV_STACK, bool PF = false>
SRT_DEV bool traverse(const DevScene& S, Ray ray, uint2* stack, int stride, float& t_out, uint32_t& prim_out,
                      float& u_out, float& v_out, uint32_t* err, TravCounters cnt, uint4* nbuf = nullptr) {
    prim_out = MISS;
    if (S.n_nodes == 0u) return false;
    if (!(ray.d.x != 0.0f || ray.d.y != 0.0f || ray.d.z != 0.0f)) return false;
    if (!(ray.tmin <= ray.tmax)) return false;
    RayShear sh = make_shear(ray.d);
    const float eps = 1e-12f;
    float3 idir = f3(1.0f / (fabsf(ray.d.x) > eps ? ray.d.x : copysignf(eps, ray.d.x)),
                     1.0f / (fabsf(ray.d.y) > eps ? ray.d.y : copysignf(eps, ray.d.y)),
                     1.0f / (fabsf(ray.d.z) > eps ? ray.d.z : copysignf(eps, ray.d.z)));
    uint32_t oct = (ray.d.x < 0.f ? 1u : 0u) | (ray.d.y < 0.f ? 2u : 0u) | (ray.d.z < 0.f ? 4u : 0u);
    float tbest = ray.tmax;
    uint32_t best = MISS;
    float bu = 0.f, bv = 0.f;
    int sp = 0;
    uint32_t n_nodes = 0, n_tris = 0;
    // virtual group holding the root as child slot 0
    uint2 g = make_uint2(0u, (1u << (24 + (0u ^ (oct ^ 7u)))) | 1u);
    uint2 tg = make_uint2(0u, 0u);
    while (true) {
        // ---- with PF: pick the next node and start fetching it before the
        // triangle tests of the last node (the same visiting order)
        bool have = true;
        if (PF) {
            if ((g.y & 0xFF000000u) == 0u) {
                if (sp == 0) have = false;
                else {
                    --sp;
                    g = stack[sp * stride];
                }
            }
            if (have) {
                int bit = 31 - __clz(g.y & 0xFF000000u);
                g.y &= ~(1u << bit);
                uint32_t slot = (uint32_t)(bit - 24) ^ (oct ^ 7u);
                uint32_t idx = g.x + __popc(g.y & ((1u << slot) - 1u) & 0xFFu);
                if (g.y & 0xFF000000u) {
                    if (sp >= STACK) {
                        atomicOr(err, ERR_STACK_OVERFLOW);
                        break;
                    }
                    stack[sp * stride] = g;
                    ++sp;
                }
                if (idx >= S.n_nodes) {
                    atomicOr(err, ERR_BAD_INDEX);
                    break;
                }
                fetch_node_async(S, idx, nbuf, stride);
            }
        }
        // ---- triangles of the last node
        while (tg.y != 0u) {
            int b = __ffs(tg.y) - 1;
            tg.y &= tg.y - 1u;
            const TriSlot* ts = S.tris + tg.x + (uint32_t)b;
            float4 a0 = __ldg(&ts->v0), a1 = __ldg(&ts->v1), a2 = __ldg(&ts->v2);
            if (COUNT) ++n_tris;
            float t, u, v;
            Ray r = ray;
            r.tmax = tbest;
            if (intersect_tri(r, sh, xyz(a0), xyz(a1), xyz(a2), t, u, v)) {
                uint32_t id = __float_as_uint(a0.w);
                if (ANY) {
                    if (PF) cp_async_wait_all();  // no copy into the slot outlives the ray
                    t_out = t;
                    prim_out = id;
                    if (COUNT) {
                        atomicAdd(cnt.nodes, (unsigned long long)n_nodes);
                        atomicAdd(cnt.tris, (unsigned long long)n_tris);
                    }
                    return true;
                }
                if (t < tbest || id < best) {  // (t, id) lexicographic; t <= tbest holds here
                    if (t < tbest || (t == tbest && id < best)) {
                        tbest = t;
                        best = id;
                        bu = u;
                        bv = v;
                    }
                }
            }
        }
        if (PF) {
            if (!have) break;
            cp_async_wait_all();
            if (COUNT) ++n_nodes;
            node_children(nbuf[0], nbuf[stride], nbuf[2 * stride], nbuf[3 * stride], nbuf[4 * stride], ray.o, idir, oct,
                          ray.tmin, tbest, g, tg);
            continue;
        }
        // ---- next node
        if ((g.y & 0xFF000000u) == 0u) {
            if (sp == 0) break;
            --sp;
            g = stack[sp * stride];
        }
        int bit = 31 - __clz(g.y & 0xFF000000u);
        g.y &= ~(1u << bit);
        uint32_t slot = (uint32_t)(bit - 24) ^ (oct ^ 7u);
        uint32_t idx = g.x + __popc(g.y & ((1u << slot) - 1u) & 0xFFu);
        if (g.y & 0xFF000000u) {
            if (sp >= STACK) {
                atomicOr(err, ERR_STACK_OVERFLOW);
                break;
            }
            stack[sp * stride] = g;
            ++sp;
        }
        if (idx >= S.n_nodes) {
            atomicOr(err, ERR_BAD_INDEX);
            break;
        }
        const uint4* np = reinterpret_cast<const uint4*>(S.nodes + idx);
        uint4 w0 = __ldg(np), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3), w4 = __ldg(np + 4);
        if (COUNT) ++n_nodes;
        node_children(w0, w1, w2, w3, w4, ray.o, idir, oct, ray.tmin, tbest, g, tg);
    }
    if (COUNT) {
        atomicAdd(cnt.nodes, (unsigned long long)n_nodes);
        atomicAdd(cnt.tris, (unsigned long long)n_tris);
    }
    if (ANY) return false;
    if (best == MISS) return false;
    t_out = tbest;
    prim_out = best;
    u_out = bu;
    v_out = bv;
    return true;
}

// ------------------------------------------------------------------ resumable traversal
// The same traversal as traverse<>, split into an init and a step so that a
// persistent warp can hand a finished lane a new ray between steps.  One
// step = the pending triangle tests of the last node + one node visit.
#ifndef SRT_TRAV_ONE_TRI_PER_STEP
#define SRT_TRAV_ONE_TRI_PER_STEP 0
#endif
// Closest-hit steps: the lanes of a warp that entered a step wait for each
// other before the node visit (__syncwarp), so that it runs with all of them
// at once instead of in the groups in which they left the triangle loop and
// the stack pop (measured on bounce 1 of config 2: 0.75M warp node visits
// with 21.8 lanes each instead of 1.09M with 15.0; closest-hit 3.29 vs
// 3.37 ms per frame).  Any-hit steps use pooled triangle tests instead
// (pool_tris); the two together measured slower than either alone.
#ifndef SRT_TRAV_WARPSYNC
#define SRT_TRAV_WARPSYNC 1
#endif

// The top entry of the traversal stack in registers (SRT_TRAV_REG_TOP): a
// push keeps the new group in `top` and moves the previous top to shared
// memory; a pop takes `top` if there is one.  A group pushed at a node visit
// and popped when that node's subtree is done never touches shared memory.
#ifndef SRT_TRAV_REG_TOP
#define SRT_TRAV_REG_TOP 0
#endif
constexpr uint32_t AXES_HAS_TOP = 1u << 16;  // TravState.axes: `top` holds an entry

struct TravState {
    float3 o, idir;
    float tmin, tbest;
    float sx, sy, sz;
    uint32_t axes;  // kx | ky << 2 | kz << 4 | oct << 8 (| AXES_HAS_TOP)
    uint2 g, tg;
    int sp;
    uint32_t best;
    float bu, bv;
#if SRT_TRAV_REG_TOP
    uint2 top;
#endif
};

// Pops the next node group into T.g; false when the stack is empty.
SRT_DEV bool trav_pop(TravState& T, const uint2* stack, int stride) {
#if SRT_TRAV_REG_TOP
    if (T.axes & AXES_HAS_TOP) {
        T.g = T.top;
        T.axes &= ~AXES_HAS_TOP;
        return true;
    }
#endif
    if (T.sp == 0) return false;
    --T.sp;
    T.g = stack[T.sp * stride];
    return true;
}
// Pushes T.g; false when STACK shared-memory entries are in use (overflow).
template <int STACK>
SRT_DEV bool trav_push(TravState& T, uint2* stack, int stride) {
#if SRT_TRAV_REG_TOP
    if (T.axes & AXES_HAS_TOP) {
        if (T.sp >= STACK) return false;
        stack[T.sp * stride] = T.top;
        ++T.sp;
    }
    T.top = T.g;
    T.axes |= AXES_HAS_TOP;
    return true;
#else
    if (T.sp >= STACK) return false;
    stack[T.sp * stride] = T.g;
    ++T.sp;
    return true;
#endif
}

// Returns false when the ray cannot hit anything (finished at once).
SRT_DEV bool trav_init(TravState& T, const DevScene& S, float3 o, float3 d, float tmin, float tmax) {
    T.best = MISS;
    T.tbest = tmax;
    T.tmin = tmin;
    T.sp = 0;
    T.tg = make_uint2(0u, 0u);
    T.g = make_uint2(0u, 0u);
    T.bu = T.bv = 0.f;
    T.o = o;
    if (S.n_nodes == 0u || !(d.x != 0.0f || d.y != 0.0f || d.z != 0.0f) || !(tmin <= tmax)) return false;
    RayShear sh = make_shear(d);
    T.sx = sh.sx;
    T.sy = sh.sy;
    T.sz = sh.sz;
    const float eps = 1e-12f;
    T.idir = f3(1.0f / (fabsf(d.x) > eps ? d.x : copysignf(eps, d.x)),
                1.0f / (fabsf(d.y) > eps ? d.y : copysignf(eps, d.y)),
                1.0f / (fabsf(d.z) > eps ? d.z : copysignf(eps, d.z)));
    uint32_t oct = (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
    T.axes = (uint32_t)sh.kx | ((uint32_t)sh.ky << 2) | ((uint32_t)sh.kz << 4) | (oct << 8);
    T.g = make_uint2(0u, (1u << (24 + (0u ^ (oct ^ 7u)))) | 1u);
    return true;
}

// Pooled triangle tests (SRT_TRAV_POOL), called by all 32 lanes of a warp
// at once: the triangles pending at the lanes' last node visits (T.tg of the
// lanes with `live` set) are numbered across the warp by a prefix sum and
// dealt out one per lane per round, so a round tests up to 32 triangles
// whatever lanes they belong to (idle lanes work too), instead of each lane
// looping over its own with the others waiting.  A lane fetches its task's
// ray from the owning lane (shuffles), tests it with the same tri_test, and
// a segmented minimum over the lanes of one owner (tasks of a lane are
// consecutive) gives the owner the lexicographic minimum of (t, id) and its
// (u, v); the owner keeps it if it beats its best.  The closest hit does not
// depend on the order of the tests, so results are unchanged; any-hit rays
// stop at their first hit (T.best != MISS afterwards).  Leaves T.tg empty.
// Used by the persistent any-hit kernel (SRT_TRAV_POOL): the triangle loop of
// bounce-1 closest-hit steps ran 2.15M warp iterations per config-2 frame
// with 4.45 of 32 lanes busy; pooled, the shadow rays of bounces 1-4 take
// 1.57 instead of 1.94 ms per frame.  Closest-hit steps measured no gain
// alone and 1.6x slower with the closest-hit warp sync (SRT_TRAV_POOL=2
// pools them too).
#ifndef SRT_TRAV_POOL
#define SRT_TRAV_POOL 1
#endif
// MULTI: the lanes trace rays of different scenes (the batched renderer's
// persistent launch), so a task reads the triangles of its owner's scene.
template <bool ANY, bool MULTI = false>
SRT_DEV void pool_tris(const DevScene& S, TravState& T, bool live, uint32_t& n_tris) {
    constexpr uint32_t FULL = 0xFFFFFFFFu;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t cnt = live ? (uint32_t)__popc(T.tg.y) : 0u;
    uint32_t incl = cnt;
#pragma unroll
    for (uint32_t d = 1; d < 32u; d <<= 1) {
        const uint32_t v = __shfl_up_sync(FULL, incl, d);
        if (lane >= d) incl += v;
    }
    const uint32_t total = __shfl_sync(FULL, incl, 31);
    if (total == 0u) return;
    const uint32_t excl = incl - cnt;
    for (uint32_t base = 0; base < total; base += 32u) {
        const uint32_t task = base + lane;
        const bool have = task < total;
        // owner = the number of lanes whose tasks end at or before this one
        uint32_t o = 0;
#pragma unroll
        for (uint32_t step = 16; step >= 1u; step >>= 1) {
            const uint32_t v = __shfl_sync(FULL, incl, (int)(o + step - 1u));
            if (v <= task) o += step;
        }
        o = have ? o : 31u;
        const uint32_t o_excl = __shfl_sync(FULL, excl, (int)o);
        const uint32_t gx = __shfl_sync(FULL, T.tg.x, (int)o), gy = __shfl_sync(FULL, T.tg.y, (int)o);
        const float ox = __shfl_sync(FULL, T.o.x, (int)o), oy = __shfl_sync(FULL, T.o.y, (int)o),
                    oz = __shfl_sync(FULL, T.o.z, (int)o);
        const float sx = __shfl_sync(FULL, T.sx, (int)o), sy = __shfl_sync(FULL, T.sy, (int)o),
                    sz = __shfl_sync(FULL, T.sz, (int)o);
        const float tmin = __shfl_sync(FULL, T.tmin, (int)o), tmax = __shfl_sync(FULL, T.tbest, (int)o);
        const uint32_t axes = __shfl_sync(FULL, T.axes, (int)o);
        uint32_t klo = 0xFFFFFFFFu, khi = 0xFFFFFFFFu;  // (t bits, id) of a hit, else all ones
        float hu = 0.f, hv = 0.f;
        const TriSlot* tris = S.tris;
        if (MULTI)
            tris = reinterpret_cast<const TriSlot*>(
                __shfl_sync(FULL, reinterpret_cast<unsigned long long>(S.tris), (int)o));
        if (have) {
            const uint32_t bit = __fns(gy, 0u, (int)(task - o_excl + 1u)) & 31u;  // always found: task < incl[o]
            const TriSlot* ts = tris + gx + bit;
            const float4 a0 = __ldg(&ts->v0), a1 = __ldg(&ts->v1), a2 = __ldg(&ts->v2);
            ++n_tris;
            float t, u, v;
            if (tri_test(xyz(a0), xyz(a1), xyz(a2), f3(ox, oy, oz), axes & 3u, (axes >> 2) & 3u, (axes >> 4) & 3u, sx,
                         sy, sz, tmin, tmax, t, u, v)) {
                khi = __float_as_uint(t);  // t >= tmin > 0: the bits order like the values
                klo = __float_as_uint(a0.w);
                hu = u;
                hv = v;
            }
        }
        // segmented minimum over the lanes of one owner (consecutive lanes)
        const uint32_t own = have ? o : 32u;
#pragma unroll
        for (uint32_t d = 1; d < 32u; d <<= 1) {
            const uint32_t olo = __shfl_down_sync(FULL, klo, d), ohi = __shfl_down_sync(FULL, khi, d);
            const float ou = __shfl_down_sync(FULL, hu, d), ov = __shfl_down_sync(FULL, hv, d);
            const uint32_t oo = __shfl_down_sync(FULL, own, d);
            if (lane + d < 32u && oo == own && (ohi < khi || (ohi == khi && olo < klo))) {
                khi = ohi;
                klo = olo;
                hu = ou;
                hv = ov;
            }
        }
        // each owner reads the minimum at the first lane of its segment
        const bool mine = cnt > 0u && incl > base && excl < base + 32u;
        const uint32_t first = mine ? (excl > base ? excl - base : 0u) : lane;
        const uint32_t rlo = __shfl_sync(FULL, klo, (int)first), rhi = __shfl_sync(FULL, khi, (int)first);
        const float ru = __shfl_sync(FULL, hu, (int)first), rv = __shfl_sync(FULL, hv, (int)first);
        if (mine && rhi != 0xFFFFFFFFu) {
            if (ANY) {
                if (T.best == MISS) {
                    T.best = rlo;
                    T.tbest = __uint_as_float(rhi);
                }
            } else {
                const uint32_t chi = __float_as_uint(T.tbest);
                if (rhi < chi || (rhi == chi && rlo < T.best)) {
                    T.tbest = __uint_as_float(rhi);
                    T.best = rlo;
                    T.bu = ru;
                    T.bv = rv;
                }
            }
        }
    }
    if (live) T.tg.y = 0u;
}

// Returns true when the ray is finished (for ANY: T.best != MISS on a hit).
template <bool ANY, int STACK, bool PF = false>
SRT_DEV bool trav_step(const DevScene& S, TravState& T, uint2* stack, int stride, uint32_t* err, uint32_t& n_nodes,
                       uint32_t& n_tris, uint4* nbuf = nullptr) {
    const uint32_t kx = T.axes & 3u, ky = (T.axes >> 2) & 3u, kz = (T.axes >> 4) & 3u, oct = (T.axes >> 8) & 7u;
    // `entered`: the lanes converged at the step's start.  Every one of them
    // reaches the __syncwarp below (nothing before it returns), so the sync is
    // well formed.  Syncing the ballot of all lanes that take the step instead
    // (a stronger wait) measured slower: closest-hit 3.40 vs 3.30 ms per frame.
    constexpr bool kSync = SRT_TRAV_WARPSYNC && !ANY && !PF && !SRT_TRAV_ONE_TRI_PER_STEP;
    const uint32_t entered = kSync ? __activemask() : 0u;
    bool any_hit = false;
    bool have = true;
    if (PF) {
        // pick the next node and start fetching it; the triangle tests below
        // run while the copy is in flight (same visiting order)
        if ((T.g.y & 0xFF000000u) == 0u) {
            if (T.sp == 0) have = false;
            else {
                --T.sp;
                T.g = stack[T.sp * stride];
            }
        }
        if (have) {
            int bit = 31 - __clz(T.g.y & 0xFF000000u);
            T.g.y &= ~(1u << bit);
            uint32_t slot = (uint32_t)(bit - 24) ^ (oct ^ 7u);
            uint32_t idx = T.g.x + __popc(T.g.y & ((1u << slot) - 1u) & 0xFFu);
            if (T.g.y & 0xFF000000u) {
                if (T.sp >= STACK) {
                    atomicOr(err, ERR_STACK_OVERFLOW);
                    return true;
                }
                stack[T.sp * stride] = T.g;
                ++T.sp;
            }
            if (idx >= S.n_nodes) {
                atomicOr(err, ERR_BAD_INDEX);
                return true;
            }
            fetch_node_async(S, idx, nbuf, stride);
        }
    }
#if SRT_TRAV_ONE_TRI_PER_STEP
    // one item per step: a triangle if one is pending, else a node, so a lane
    // with a long triangle list does not hold up the lanes visiting nodes
    const bool tri_step = T.tg.y != 0u;
    for (int once = 0; once < 1 && T.tg.y != 0u; ++once) {
#else
    while (T.tg.y != 0u) {
#endif
        int b = __ffs(T.tg.y) - 1;
        T.tg.y &= T.tg.y - 1u;
        const TriSlot* ts = S.tris + T.tg.x + (uint32_t)b;
        float4 a0 = __ldg(&ts->v0), a1 = __ldg(&ts->v1), a2 = __ldg(&ts->v2);
        ++n_tris;
        float t, tu, tv;
        if (!tri_test(xyz(a0), xyz(a1), xyz(a2), T.o, kx, ky, kz, T.sx, T.sy, T.sz, T.tmin, T.tbest, t, tu, tv))
            continue;
        uint32_t id = __float_as_uint(a0.w);
        if (ANY) {
            if (PF && have) cp_async_wait_all();  // no copy into the slot outlives the ray
            T.best = id;
            T.tbest = t;
            if (!kSync) return true;
            any_hit = true;
            break;
        }
        if (t < T.tbest || id < T.best) {  // (t, id) lexicographic; t <= tbest holds here
            T.tbest = t;
            T.best = id;
            T.bu = tu;
            T.bv = tv;
        }
    }

#if SRT_TRAV_ONE_TRI_PER_STEP
    if (tri_step) return false;
#endif
    if (PF) {
        if (!have) return true;
        cp_async_wait_all();
        ++n_nodes;
        node_children(nbuf[0], nbuf[stride], nbuf[2 * stride], nbuf[3 * stride], nbuf[4 * stride], T.o, T.idir, oct,
                      T.tmin, T.tbest, T.g, T.tg);
        return false;
    }
    if constexpr (kSync) {
        // the same steps with every exit (an any-hit, the end of the tree, an
        // error) deferred past one __syncwarp, which every lane that entered
        // the step reaches (nothing above returns), so that the node fetch and
        // slab tests run with all lanes still tracing at once
        bool fin = ANY && any_hit;
        uint32_t idx = 0u;
        if (!fin && (T.g.y & 0xFF000000u) == 0u) fin = !trav_pop(T, stack, stride);
        if (!fin) {
            const int bit = 31 - __clz(T.g.y & 0xFF000000u);
            T.g.y &= ~(1u << bit);
            const uint32_t slot = (uint32_t)(bit - 24) ^ (oct ^ 7u);
            idx = T.g.x + __popc(T.g.y & ((1u << slot) - 1u) & 0xFFu);
            if ((T.g.y & 0xFF000000u) && !trav_push<STACK>(T, stack, stride)) {
                atomicOr(err, ERR_STACK_OVERFLOW);
                fin = true;
            }
            if (!fin && idx >= S.n_nodes) {
                atomicOr(err, ERR_BAD_INDEX);
                fin = true;
            }
        }
        __syncwarp(entered);
        if (fin) return true;
        const uint4* np = reinterpret_cast<const uint4*>(S.nodes + idx);
        uint4 w0 = __ldg(np), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3), w4 = __ldg(np + 4);
        ++n_nodes;
        node_children(w0, w1, w2, w3, w4, T.o, T.idir, oct, T.tmin, T.tbest, T.g, T.tg);
        return false;
    }
    if ((T.g.y & 0xFF000000u) == 0u && !trav_pop(T, stack, stride)) return true;
    int bit = 31 - __clz(T.g.y & 0xFF000000u);
    T.g.y &= ~(1u << bit);
    uint32_t slot = (uint32_t)(bit - 24) ^ (oct ^ 7u);
    uint32_t idx = T.g.x + __popc(T.g.y & ((1u << slot) - 1u) & 0xFFu);
    if ((T.g.y & 0xFF000000u) && !trav_push<STACK>(T, stack, stride)) {
        atomicOr(err, ERR_STACK_OVERFLOW);
        return true;
    }
    if (idx >= S.n_nodes) {
        atomicOr(err, ERR_BAD_INDEX);
        return true;
    }
    const uint4* np = reinterpret_cast<const uint4*>(S.nodes + idx);
    uint4 w0 = __ldg(np), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3), w4 = __ldg(np + 4);
    ++n_nodes;
    node_children(w0, w1, w2, w3, w4, T.o, T.idir, oct, T.tmin, T.tbest, T.g, T.tg);
    return false;
}

// ------------------------------------------------------------------ surface data at a hit
struct Surface {
    uint32_t inst, mat;
    float3 wn;     // normalised world shading normal (not face-forwarded)
    bool front;
};

// get_interpolated_normal (shader.wgsl:530-545), the world transform
// (:573-576) and the ray query's front_face: counter-clockwise as seen from
// the ray in object space.
SRT_DEV Surface surface_at(const DevScene& S, uint32_t prim, float u, float v, float3 dir_world) {
    Surface sf;
    uint32_t ii = __ldg(&S.tri_inst[prim]);
    const InstDev& in = S.inst[ii];
    uint4 mi = __ldg(&S.mesh_infos[in.mesh_id]);
    uint32_t io = mi.y + (prim - in.tri_offset) * 3u;
    uint32_t i0 = __ldg(&S.indices[io]) + mi.x, i1 = __ldg(&S.indices[io + 1]) + mi.x,
             i2 = __ldg(&S.indices[io + 2]) + mi.x;
    float4 p0 = __ldg(&S.vtx[2 * i0]), n0 = __ldg(&S.vtx[2 * i0 + 1]);
    float4 p1 = __ldg(&S.vtx[2 * i1]), n1 = __ldg(&S.vtx[2 * i1 + 1]);
    float4 p2 = __ldg(&S.vtx[2 * i2]), n2 = __ldg(&S.vtx[2 * i2 + 1]);
    float w = 1.0f - u - v;
    float3 ln = normalize(xyz(n0) * w + xyz(n1) * u + xyz(n2) * v);
    float4 r0 = in.w2o0, r1 = in.w2o1, r2 = in.w2o2;
    // local_normal * mat3x3(w2o columns) = transpose(W2O) * n
    float3 wn = f3(ln.x * r0.x + ln.y * r1.x + ln.z * r2.x, ln.x * r0.y + ln.y * r1.y + ln.z * r2.y,
                   ln.x * r0.z + ln.y * r1.z + ln.z * r2.z);
    sf.wn = normalize(wn);
    float3 dobj = f3(dot(xyz(r0), dir_world), dot(xyz(r1), dir_world), dot(xyz(r2), dir_world));
    float3 gn = cross(xyz(p1) - xyz(p0), xyz(p2) - xyz(p0));
    sf.front = dot(dobj, gn) < 0.0f;
    sf.inst = ii;
    sf.mat = in.mat_id;
    return sf;
}

}  // namespace srt
