// oracle.cpp — CPU oracle of the spectral path-tracing path.
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py, to check the CUDA path.  The product library never
// links or calls it.
//
// Every shading function restates the reference WGSL in FP32 with the same
// operation order and the same RNG consumption order; citations are
// path:line inside the reference project.  Ray queries (a Vulkan driver call
// in the reference) are answered in FP64: an exact Moller-Trumbore test per
// triangle, brute force or through an FP64 BVH.
//
// Two reading choices are recorded here because the WGSL leaves them open:
//  * pow(x, 2.0) with x < 0 (sample_cie_xyz, rgb_to_spectrum_eval) is
//    undefined in SPIR-V; shader compilers lower pow(x, 2.0) to x*x, and so
//    does this oracle.
//  * Vulkan reports front_face for a triangle wound counter-clockwise as
//    seen from the ray, i.e. dot(dir_obj, (v1-v0) x (v2-v0)) < 0 in object
//    space; the reference scenes light correctly only under this reading.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const float PI = 3.14159265359f;  // shader.wgsl:6
const float LAMBDA_MIN = 380.0f;  // shader.wgsl:81-83
const float LAMBDA_MAX = 780.0f;
const float LAMBDA_RANGE = LAMBDA_MAX - LAMBDA_MIN;

struct f3 {
    float x, y, z;
};
struct f4 {
    float x, y, z, w;
};
inline f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
inline f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline f3 cross(f3 a, f3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float length(f3 a) { return std::sqrt(dot(a, a)); }
inline f3 normalize(f3 a) { return a / length(a); }
// WGSL reflect(e1, e2) = e1 - 2 * dot(e2, e1) * e2
inline f3 reflect(f3 i, f3 n) { return i - n * (2.0f * dot(n, i)); }
// WGSL refract(e1, e2, e3)
inline f3 refract(f3 i, f3 n, float eta) {
    float ni = dot(n, i);
    float k = 1.0f - eta * eta * (1.0f - ni * ni);
    if (k < 0.0f) return {0.f, 0.f, 0.f};
    return i * eta - n * (eta * ni + std::sqrt(k));
}
inline f4 operator+(f4 a, f4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
inline f4 operator-(f4 a, f4 b) { return {a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; }
inline f4 operator*(f4 a, f4 b) { return {a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w}; }
inline f4 operator/(f4 a, f4 b) { return {a.x / b.x, a.y / b.y, a.z / b.z, a.w / b.w}; }
inline f4 operator*(f4 a, float s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
inline f4 operator/(f4 a, float s) { return {a.x / s, a.y / s, a.z / s, a.w / s}; }
inline f4 splat(float s) { return {s, s, s, s}; }
inline float sgn(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }
inline float clampf(float x, float lo, float hi) { return std::min(std::max(x, lo), hi); }
inline float sq(float x) { return x * x; }

// ---------------------------------------------------------------- RNG
// pcg_hash: shader.wgsl:151-155 (= photon_emit.wgsl:72-76)
inline uint32_t pcg_hash(uint32_t input) {
    uint32_t state = input * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
struct Rng {
    uint32_t s;
    // rand: shader.wgsl:157-160
    float next() {
        s = pcg_hash(s);
        return (float)s / 4294967295.0f;
    }
};
// random_unit_vector: shader.wgsl:162-169
inline f3 random_unit_vector(Rng& r) {
    float u1 = r.next();
    float u2 = r.next();
    float z = 1.0f - 2.0f * u1;
    float rr = std::sqrt(std::max(0.0f, 1.0f - z * z));
    float phi = 2.0f * PI * u2;
    return {rr * std::cos(phi), rr * std::sin(phi), z};
}

// ---------------------------------------------------------------- spectra
// sample_cie_xyz: shader.wgsl:85-97
inline f3 sample_cie_xyz(float l) {
    float x = std::exp(-sq((l - 599.8f) / 37.9f)) * 1.056f + std::exp(-sq((l - 442.0f) / 16.0f)) * 0.362f -
              std::exp(-sq((l - 501.1f) / 26.7f)) * 0.065f;
    float y = std::exp(-sq((l - 568.8f) / 46.9f)) * 0.821f + std::exp(-sq((l - 530.9f) / 16.3f)) * 0.286f;
    float z = std::exp(-sq((l - 437.0f) / 11.8f)) * 1.217f + std::exp(-sq((l - 459.0f) / 26.0f)) * 0.681f;
    return {std::max(0.0f, x), std::max(0.0f, y), std::max(0.0f, z)};
}
// XYZ_TO_SRGB (column-major): shader.wgsl:100-104
inline f3 xyz_to_srgb(f3 c) {
    return {3.2404542f * c.x + -1.5371385f * c.y + -0.4985314f * c.z,
            -0.9692660f * c.x + 1.8760108f * c.y + 0.0415560f * c.z,
            0.0556434f * c.x + -0.2040259f * c.y + 1.0572252f * c.z};
}
// rgb_to_spectrum_eval: shader.wgsl:106-117
inline float rgb_to_spectrum_eval(f3 rgb, float l) {
    float white = std::min(rgb.x, std::min(rgb.y, rgb.z));
    float cr = std::max(rgb.x - white, 0.0f), cg = std::max(rgb.y - white, 0.0f), cb = std::max(rgb.z - white, 0.0f);
    const float gw = 20.0f;
    float r_val = cr * std::exp(-sq((l - 630.0f) / gw));
    float g_val = cg * std::exp(-sq((l - 525.0f) / gw));
    float b_val = cb * std::exp(-sq((l - 460.0f) / gw));
    return clampf(white + r_val + g_val + b_val, 0.0f, 0.99f);
}
inline f4 rgb_to_spectrum_vec4(f3 rgb, f4 wl) {  // shader.wgsl:119-126
    return {rgb_to_spectrum_eval(rgb, wl.x), rgb_to_spectrum_eval(rgb, wl.y), rgb_to_spectrum_eval(rgb, wl.z),
            rgb_to_spectrum_eval(rgb, wl.w)};
}
// blackbody_radiance: shader.wgsl:128-139
inline float blackbody_radiance(float lambda_nm, float temp_k) {
    float lambda_m = lambda_nm * 1e-9f;
    const float h = 6.62607015e-34f;
    const float c = 299792458.0f;
    const float k = 1.380649e-23f;
    float c1 = 2.0f * h * c * c;
    float c2 = (h * c) / (k * temp_k);
    float radiance = c1 / (std::pow(lambda_m, 5.0f) * (std::exp(c2 / lambda_m) - 1.0f));
    return radiance * 1e-13f;
}
inline f4 blackbody4(f4 wl, float t) {
    return {blackbody_radiance(wl.x, t), blackbody_radiance(wl.y, t), blackbody_radiance(wl.z, t),
            blackbody_radiance(wl.w, t)};
}

// ---------------------------------------------------------------- BSDF math
struct Mat3 {
    f3 c0, c1, c2;
};
// build_orthonormal_basis: shader.wgsl:171-188 (inf at n.z == 0 kept)
inline Mat3 build_orthonormal_basis(f3 n) {
    float s = sgn(n.z);
    float a = -1.0f / (s + n.z);
    float b = n.x * n.y * a;
    f3 right = {1.0f + s * n.x * n.x * a, s * b, -s * n.x};
    f3 up = {b, s + n.y * n.y * a, -n.y};
    return {right, up, n};
}
// sample_ggx_half_vector: shader.wgsl:193-205
inline f3 sample_ggx_half_vector(f3 n, float roughness, Rng& rng) {
    float a2 = roughness * roughness;
    float r1 = rng.next();
    float r2 = rng.next();
    float phi = 2.0f * PI * r1;
    float cos_theta = std::sqrt((1.0f - r2) / (1.0f + (a2 - 1.0f) * r2));
    float sin_theta = std::sqrt(std::max(0.0f, 1.0f - cos_theta * cos_theta));
    f3 ht = {std::cos(phi) * sin_theta, std::sin(phi) * sin_theta, cos_theta};
    Mat3 tbn = build_orthonormal_basis(n);
    return normalize(tbn.c0 * ht.x + tbn.c1 * ht.y + tbn.c2 * ht.z);
}
// geometry_schlick_ggx / geometry_smith: shader.wgsl:207-219
inline float geometry_schlick_ggx(float n_dot_v, float roughness) {
    float a = roughness;
    float k = (a * a) / 2.0f;
    return n_dot_v / (n_dot_v * (1.0f - k) + k);
}
inline float geometry_smith(float n_dot_v, float n_dot_l, float roughness) {
    float ggx2 = geometry_schlick_ggx(n_dot_v, roughness);
    float ggx1 = geometry_schlick_ggx(n_dot_l, roughness);
    return ggx1 * ggx2;
}
// fresnel_schlick_vec4: shader.wgsl:222-224
inline f4 fresnel_schlick_vec4(float cos_theta, f4 f0) {
    float p = std::pow(clampf(1.0f - cos_theta, 0.0f, 1.0f), 5.0f);
    return f0 + (splat(1.0f) - f0) * p;
}
// fresnel_thin_film (one wavelength): photon_emit.wgsl:107-132; the vec4
// form (shader.wgsl:233-262) applies the same arithmetic per component.
inline float thin_film_1(float cos1, float n1, float n2, float n3, float d, float lambda, bool* tir) {
    float sin1_sq = std::max(0.0f, 1.0f - cos1 * cos1);
    float sin2_sq = (n1 / n2) * (n1 / n2) * sin1_sq;
    if (sin2_sq >= 1.0f) {
        *tir = true;
        return 1.0f;
    }
    float cos2 = std::sqrt(1.0f - sin2_sq);
    float sin3_sq = (n1 / n3) * (n1 / n3) * sin1_sq;
    if (sin3_sq >= 1.0f) {
        *tir = true;
        return 1.0f;
    }
    float cos3 = std::sqrt(1.0f - sin3_sq);
    float r12 = (n1 * cos1 - n2 * cos2) / (n1 * cos1 + n2 * cos2);
    float r23 = (n2 * cos2 - n3 * cos3) / (n2 * cos2 + n3 * cos3);
    float r12_sq = r12 * r12;
    float r23_sq = r23 * r23;
    float delta = (4.0f * PI * n2 * d * cos2) / lambda;
    float cd = std::cos(delta);
    float num = r12_sq + r23_sq + 2.0f * r12 * r23 * cd;
    float den = 1.0f + r12_sq * r23_sq + 2.0f * r12 * r23 * cd;
    *tir = false;
    return clampf(num / den, 0.0f, 1.0f);
}
inline f4 fresnel_thin_film(float cos1, float n1, float n2, float n3, float d, f4 wl) {
    bool tir;
    float x = thin_film_1(cos1, n1, n2, n3, d, wl.x, &tir);
    if (tir) return splat(1.0f);
    return {x, thin_film_1(cos1, n1, n2, n3, d, wl.y, &tir), thin_film_1(cos1, n1, n2, n3, d, wl.z, &tir),
            thin_film_1(cos1, n1, n2, n3, d, wl.w, &tir)};
}
// reflectance (Schlick): shader.wgsl:264-268
inline float reflectance(float cosine, float ref_idx) {
    float r0 = (1.0f - ref_idx) / (1.0f + ref_idx);
    r0 = r0 * r0;
    return r0 + (1.0f - r0) * std::pow((1.0f - cosine), 5.0f);
}

struct Scatter {
    f3 dir;
    f4 att;
    bool absorbed;
};

// sample_bsdf: shader.wgsl:347-471.  Material type 5 (thin-film-coated
// GGX) has no reference counterpart: GGX half-vector sampling as type 1
// with the Airy reflectance of the film replacing Schlick's F.
Scatter sample_bsdf(f3 r_dir, f3 ffn, const srt_material& mat, bool front, f4 wl, f4 thr, Rng& rng) {
    Scatter rec;
    rec.absorbed = false;
    rec.dir = {0, 0, 0};
    rec.att = splat(0.f);
    uint32_t type = (uint32_t)mat.extra[0];
    f3 v = normalize(-r_dir);
    f3 rgb = {mat.color[0], mat.color[1], mat.color[2]};
    f4 spec = rgb_to_spectrum_vec4(rgb, wl);
    if (type == 1u || type == 5u) {
        float roughness = std::max(type == 1u ? mat.extra[1] : mat.color[3], 0.001f);
        f3 h = sample_ggx_half_vector(ffn, roughness, rng);
        f3 l = reflect(-v, h);
        float n_dot_l = dot(ffn, l);
        float n_dot_v = dot(ffn, v);
        if (n_dot_l > 0.0f && n_dot_v > 0.0f) {
            float n_dot_h = std::max(dot(ffn, h), 0.0f);
            float v_dot_h = std::max(dot(v, h), 0.0f);
            f4 F = type == 1u ? fresnel_schlick_vec4(v_dot_h, spec)
                              : fresnel_thin_film(v_dot_h, 1.0f, mat.extra[2], mat.extra[3],
                                                  std::max(mat.extra[1], 50.0f), wl);
            float G = geometry_smith(n_dot_v, n_dot_l, roughness);
            f4 weight = (F * G * v_dot_h) / std::max(n_dot_v * n_dot_h, 0.0001f);
            rec.dir = l;
            rec.att = weight;
        } else {
            rec.absorbed = true;
        }
    } else if (type == 2u) {
        float A = mat.extra[2];
        float B = mat.extra[3];
        float lambda_um = wl.x / 1000.0f;
        float ir = A + (B / (lambda_um * lambda_um));
        float ratio = front ? 1.0f / ir : ir;
        f3 unit_dir = normalize(r_dir);
        float cos_theta = std::min(dot(-unit_dir, ffn), 1.0f);
        float sin_i2 = std::max(0.0f, 1.0f - cos_theta * cos_theta);
        float sin_t2 = ratio * ratio * sin_i2;
        if (sin_t2 >= 1.0f) {
            rec.dir = reflect(unit_dir, ffn);
            rec.att = splat(1.0f);
        } else {
            float cos_t = std::sqrt(1.0f - sin_t2);
            float cos_f = front ? cos_theta : cos_t;
            if (reflectance(cos_f, ratio) > rng.next()) {
                rec.dir = reflect(unit_dir, ffn);
                rec.att = splat(1.0f);
            } else {
                rec.dir = refract(unit_dir, ffn, ratio);
                float scale = ratio * ratio;
                f4 base = spec * scale;
                if (B > 0.0f) {
                    bool collapsed = (thr.y < 0.0001f && thr.z < 0.0001f && thr.w < 0.0001f);
                    float mult = collapsed ? 1.0f : 4.0f;
                    rec.att = {base.x * mult, 0.f, 0.f, 0.f};
                } else {
                    rec.att = base;
                }
            }
        }
    } else if (type == 4u) {
        float n2 = mat.extra[2], n3 = mat.extra[3];
        float d = std::max(mat.extra[1], 50.0f);
        f3 unit_dir = normalize(r_dir);
        float cos1 = std::min(dot(-unit_dir, ffn), 1.0f);
        f4 F = fresnel_thin_film(cos1, 1.0f, n2, n3, d, wl);
        float p = F.x;
        if (rng.next() < p) {
            rec.dir = reflect(unit_dir, ffn);
            rec.att = F / p;
        } else {
            rec.dir = unit_dir;
            rec.att = (splat(1.0f) - F) / (1.0f - p);
        }
    } else {
        f3 s = ffn + random_unit_vector(rng);
        if (length(s) < 0.001f) s = ffn;
        rec.dir = normalize(s);
        rec.att = spec;
    }
    return rec;
}

// Hero wavelength tuple: shader.wgsl:734-767 and pdf sum :782-797.
struct Hero {
    f4 wl;
    float sum_pdf;
};
inline float cauchy_cdf(float x) { return (1.0f / PI) * std::atan((x - 555.0f) / 40.0f) + 0.5f; }
inline Hero sample_hero(Rng& rng) {
    const float peak = 555.0f, gamma = 40.0f;
    float cdf_min = cauchy_cdf(LAMBDA_MIN);
    float cdf_max = cauchy_cdf(LAMBDA_MAX);
    float cdf_range = cdf_max - cdf_min;
    float u = cdf_min + rng.next() * cdf_range;
    float hero = peak + gamma * std::tan(PI * (u - 0.5f));
    hero = clampf(hero, LAMBDA_MIN, LAMBDA_MAX);
    float q = LAMBDA_RANGE / 4.0f;
    f4 w = {hero, hero + q * 1.0f, hero + q * 2.0f, hero + q * 3.0f};
    auto wrap = [](float x) {  // WGSL float %: e1 - e2 * trunc(e1 / e2)
        float a = x - LAMBDA_MIN;
        return LAMBDA_MIN + (a - LAMBDA_RANGE * std::trunc(a / LAMBDA_RANGE));
    };
    w = {wrap(w.x), wrap(w.y), wrap(w.z), wrap(w.w)};
    float rot = rng.next();
    if (rot < 0.25f) {
    } else if (rot < 0.5f) {
        w = {w.y, w.z, w.w, w.x};
    } else if (rot < 0.75f) {
        w = {w.z, w.w, w.x, w.y};
    } else {
        w = {w.w, w.x, w.y, w.z};
    }
    float pdf_norm = 1.0f / (cdf_range * PI * gamma);
    auto pdf = [&](float x) {
        float d = (x - peak) / gamma;
        return pdf_norm / (1.0f + d * d);
    };
    Hero h;
    h.wl = w;
    h.sum_pdf = pdf(w.x) + pdf(w.y) + pdf(w.z) + pdf(w.w);
    return h;
}

// ---------------------------------------------------------------- photon grid
// get_grid_jitter: build_grid.wgsl:25-38 (= shader.wgsl:282-295)
inline f3 grid_jitter(uint32_t frame, float cell) {
    uint32_t seed = pcg_hash(frame * 114514u);
    float rx = (float)(seed & 0xFFu) / 255.0f;
    float ry = (float)((seed >> 8u) & 0xFFu) / 255.0f;
    float rz = (float)((seed >> 16u) & 0xFFu) / 255.0f;
    return {(rx - 0.5f) * cell, (ry - 0.5f) * cell, (rz - 0.5f) * cell};
}
// hash_position: build_grid.wgsl:41-52 (shader.wgsl:300-308)
inline uint32_t hash_position(f3 p, f3 jitter, float cell, uint32_t hash_bits) {
    float fx = std::floor((p.x + jitter.x) / cell);
    float fy = std::floor((p.y + jitter.y) / cell);
    float fz = std::floor((p.z + jitter.z) / cell);
    auto to_i32 = [](float f) -> int32_t {  // WGSL f32 -> i32 saturates
        if (!(f == f)) return 0;
        if (f >= 2147483520.0f) return 2147483647;
        if (f <= -2147483648.0f) return (-2147483647 - 1);
        return (int32_t)f;
    };
    uint32_t gx = (uint32_t)to_i32(fx), gy = (uint32_t)to_i32(fy), gz = (uint32_t)to_i32(fz);
    uint32_t h = (gx * 73856093u) ^ (gy * 19349663u) ^ (gz * 83492791u);
    return h & ((1u << hash_bits) - 1u);
}

struct Grid {
    std::vector<srt_photon> sorted;  // photons in ascending (hash, index) order
    std::vector<uint32_t> ranges;    // 2 * 2^hash_bits
    uint32_t hash_bits = 22;
};

void grid_build(const srt_photon* ph, uint32_t n, uint32_t frame, float cell, uint32_t hash_bits,
                std::vector<uint64_t>& keys, Grid* g) {
    f3 j = grid_jitter(frame, cell);
    keys.resize(n);
    uint32_t sentinel = 1u << hash_bits;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t h = ph[i].energy == 0.0f
                         ? sentinel
                         : hash_position({ph[i].position[0], ph[i].position[1], ph[i].position[2]}, j, cell,
                                         hash_bits);
        keys[i] = ((uint64_t)h << 32) | i;
    }
    std::sort(keys.begin(), keys.end());
    if (g) {
        g->hash_bits = hash_bits;
        g->ranges.assign(2ull << hash_bits, 0u);
        g->sorted.resize(n);
        for (uint32_t i = 0; i < n; ++i) g->sorted[i] = ph[(uint32_t)keys[i]];
        for (uint32_t i = 0; i < n; ++i) {
            uint32_t h = (uint32_t)(keys[i] >> 32);
            if (h >= sentinel) break;
            if (i == 0 || (uint32_t)(keys[i - 1] >> 32) != h) g->ranges[2 * h] = i;
            if (i + 1 == n || (uint32_t)(keys[i + 1] >> 32) != h) g->ranges[2 * h + 1] = i + 1;
        }
    }
}

struct GatherParams {
    float cell, r0, rexp, spectral_radius, norm_count;
    uint32_t cap;
};

// gather_photons: shader.wgsl:297-342.  The reference walks a per-bucket
// linked list (LIFO of insertion, capped at 64 entries); here the bucket
// is the sorted range and the walk goes from the highest photon index down.
f4 gather_photons(const Grid& g, f3 hit_pos, f3 normal, f4 wl, uint32_t frame, const GatherParams& gp) {
    f4 total = splat(0.f);
    f3 jitter = grid_jitter(frame, gp.cell);
    float current_radius = gp.r0 * std::pow((float)(frame + 1u), gp.rexp);
    float r_sq = current_radius * current_radius;
    uint32_t h = hash_position(hit_pos, jitter, gp.cell, g.hash_bits);
    uint32_t start = g.ranges[2 * h], end = g.ranges[2 * h + 1];
    uint32_t visited = 0;
    for (uint32_t i = end; i > start && visited < gp.cap; --i, ++visited) {
        const srt_photon& p = g.sorted[i - 1];
        f3 pp = {p.position[0], p.position[1], p.position[2]};
        f3 dd = hit_pos - pp;
        float dist_sq = dot(dd, dd);
        if (dist_sq < r_sq) {
            f3 pd = {p.direction[0], p.direction[1], p.direction[2]};
            if (dot(normal, pd) > 0.0f) {
                float dist = std::sqrt(dist_sq);
                float sw = 1.0f - (dist / current_radius);
                f4 ld = {std::fabs(wl.x - p.wavelength), std::fabs(wl.y - p.wavelength),
                         std::fabs(wl.z - p.wavelength), std::fabs(wl.w - p.wavelength)};
                f4 spw = {std::max(1.0f - ld.x / gp.spectral_radius, 0.0f),
                          std::max(1.0f - ld.y / gp.spectral_radius, 0.0f),
                          std::max(1.0f - ld.z / gp.spectral_radius, 0.0f),
                          std::max(1.0f - ld.w / gp.spectral_radius, 0.0f)};
                total = total + spw * (p.energy * sw);
            }
        }
    }
    float spatial_norm = 3.0f / (PI * r_sq);
    float spectral_norm = 1.0f / gp.spectral_radius;
    float count_norm = 1.0f / gp.norm_count;
    float density = spatial_norm * spectral_norm * count_norm;
    return total * density;
}

}  // namespace

// ---------------------------------------------------------------- scene
struct orc_scene {
    std::vector<srt_vertex> vertices;
    std::vector<uint32_t> indices;
    std::vector<srt_mesh_info> meshes;
    std::vector<srt_material> materials;
    std::vector<srt_instance> instances;
    std::vector<srt_light> lights;
    // per instance
    std::vector<double> w2o;     // 9 doubles per instance, row-major
    std::vector<float> w2o_f;    // the same as float (world_to_object 3x3)
    // flattened triangles, instance-major
    std::vector<double> tv;      // 9 doubles per triangle (world v0, v1, v2)
    std::vector<uint32_t> tinst; // instance of each triangle
    std::vector<uint32_t> tprim; // primitive index within the mesh
    std::vector<uint32_t> inst_first;  // first flattened triangle of each instance
    // FP64 BVH
    struct Node {
        double lo[3], hi[3];
        uint32_t left, right;  // children (internal) / first, count (leaf)
        uint32_t leaf;
    };
    std::vector<Node> nodes;
    std::vector<uint32_t> order;
};

namespace {

struct DRay {
    double o[3], d[3];
    double tmin, tmax;
};

// Exact-as-FP64 Moller-Trumbore: returns t (or -1), barycentrics of v1, v2.
inline bool tri_hit(const double* v, const DRay& r, double* t, double* u, double* w) {
    double e1[3] = {v[3] - v[0], v[4] - v[1], v[5] - v[2]};
    double e2[3] = {v[6] - v[0], v[7] - v[1], v[8] - v[2]};
    double p[3] = {r.d[1] * e2[2] - r.d[2] * e2[1], r.d[2] * e2[0] - r.d[0] * e2[2], r.d[0] * e2[1] - r.d[1] * e2[0]};
    double det = e1[0] * p[0] + e1[1] * p[1] + e1[2] * p[2];
    if (det == 0.0) return false;
    double inv = 1.0 / det;
    double s[3] = {r.o[0] - v[0], r.o[1] - v[1], r.o[2] - v[2]};
    double uu = (s[0] * p[0] + s[1] * p[1] + s[2] * p[2]) * inv;
    if (uu < 0.0 || uu > 1.0) return false;
    double q[3] = {s[1] * e1[2] - s[2] * e1[1], s[2] * e1[0] - s[0] * e1[2], s[0] * e1[1] - s[1] * e1[0]};
    double vv = (r.d[0] * q[0] + r.d[1] * q[1] + r.d[2] * q[2]) * inv;
    if (vv < 0.0 || uu + vv > 1.0) return false;
    double tt = (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]) * inv;
    if (!(tt >= r.tmin && tt <= r.tmax)) return false;
    *t = tt;
    *u = uu;
    *w = vv;
    return true;
}

inline bool box_hit(const orc_scene::Node& n, const DRay& r, const double* inv, double tmax) {
    double t0 = r.tmin, t1 = tmax;
    for (int a = 0; a < 3; ++a) {
        double ta = (n.lo[a] - r.o[a]) * inv[a];
        double tb = (n.hi[a] - r.o[a]) * inv[a];
        if (ta > tb) std::swap(ta, tb);
        if (std::isnan(ta) || std::isnan(tb)) {  // origin on a slab plane with zero direction
            if (r.o[a] < n.lo[a] || r.o[a] > n.hi[a]) return false;
            continue;
        }
        t0 = std::max(t0, ta);
        t1 = std::min(t1, tb);
        if (t0 > t1 * (1.0 + 1e-12) + 1e-300) return false;
    }
    return true;
}

void build_bvh(orc_scene* s) {
    size_t n = s->tinst.size();
    s->order.resize(n);
    for (size_t i = 0; i < n; ++i) s->order[i] = (uint32_t)i;
    std::vector<double> cen(3 * n);
    for (size_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a)
            cen[3 * i + a] = (s->tv[9 * i + a] + s->tv[9 * i + 3 + a] + s->tv[9 * i + 6 + a]) / 3.0;
    s->nodes.clear();
    s->nodes.reserve(2 * n / 3 + 4);
    struct Item {
        uint32_t node, b, e;
    };
    std::vector<Item> st;
    s->nodes.push_back({});
    st.push_back({0, 0, (uint32_t)n});
    while (!st.empty()) {
        Item it = st.back();
        st.pop_back();
        orc_scene::Node nd;
        double clo[3] = {1e300, 1e300, 1e300}, chi[3] = {-1e300, -1e300, -1e300};
        for (int a = 0; a < 3; ++a) {
            nd.lo[a] = 1e300;
            nd.hi[a] = -1e300;
        }
        for (uint32_t i = it.b; i < it.e; ++i) {
            uint32_t t = s->order[i];
            for (int k = 0; k < 3; ++k)
                for (int a = 0; a < 3; ++a) {
                    nd.lo[a] = std::min(nd.lo[a], s->tv[9 * t + 3 * k + a]);
                    nd.hi[a] = std::max(nd.hi[a], s->tv[9 * t + 3 * k + a]);
                }
            for (int a = 0; a < 3; ++a) {
                clo[a] = std::min(clo[a], cen[3 * t + a]);
                chi[a] = std::max(chi[a], cen[3 * t + a]);
            }
        }
        uint32_t cnt = it.e - it.b;
        if (cnt <= 4) {
            nd.leaf = 1;
            nd.left = it.b;
            nd.right = cnt;
            s->nodes[it.node] = nd;
            continue;
        }
        int axis = 0;
        for (int a = 1; a < 3; ++a)
            if (chi[a] - clo[a] > chi[axis] - clo[axis]) axis = a;
        uint32_t mid = it.b + cnt / 2;
        std::nth_element(s->order.begin() + it.b, s->order.begin() + mid, s->order.begin() + it.e,
                         [&](uint32_t x, uint32_t y) {
                             return cen[3 * x + axis] < cen[3 * y + axis] ||
                                    (cen[3 * x + axis] == cen[3 * y + axis] && x < y);
                         });
        nd.leaf = 0;
        nd.left = (uint32_t)s->nodes.size();
        nd.right = nd.left + 1;
        s->nodes.push_back({});
        s->nodes.push_back({});
        s->nodes[it.node] = nd;
        st.push_back({nd.left, it.b, mid});
        st.push_back({nd.right, mid, it.e});
    }
}

struct Hit {
    bool hit;
    double t;
    uint32_t prim;
    double u, v;
    double t2;  // best t among other triangles (brute force, or the BVH with want_t2)
};

Hit closest(const orc_scene* s, const DRay& r, bool brute, bool any, bool want_t2 = false) {
    Hit h{false, std::numeric_limits<double>::infinity(), 0xFFFFFFFFu, 0, 0, std::numeric_limits<double>::infinity()};
    if (brute) {
        size_t n = s->tinst.size();
        for (size_t i = 0; i < n; ++i) {
            double t, u, v;
            if (!tri_hit(&s->tv[9 * i], r, &t, &u, &v)) continue;
            if (any) {
                h.hit = true;
                h.prim = 0;
                return h;
            }
            if (!h.hit || t < h.t) {
                if (h.hit) h.t2 = std::min(h.t2, h.t);
                h = {true, t, (uint32_t)i, u, v, h.t2};
            } else {
                h.t2 = std::min(h.t2, t);
            }
        }
        return h;
    }
    double inv[3];
    for (int a = 0; a < 3; ++a) inv[a] = 1.0 / r.d[a];
    uint32_t stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const orc_scene::Node& nd = s->nodes[stack[--sp]];
        // with want_t2, boxes are culled at the second-best t so that the
        // nearest hit of any other triangle is found too
        double tcur = h.hit ? (want_t2 ? std::min(h.t2, r.tmax) : h.t) : r.tmax;
        if (!box_hit(nd, r, inv, tcur)) continue;
        if (nd.leaf) {
            for (uint32_t k = 0; k < nd.right; ++k) {
                uint32_t i = s->order[nd.left + k];
                double t, u, v;
                if (!tri_hit(&s->tv[9 * i], r, &t, &u, &v)) continue;
                if (any) {
                    h.hit = true;
                    h.prim = 0;
                    return h;
                }
                if (!h.hit || t < h.t || (t == h.t && i < h.prim)) {
                    if (h.hit) h.t2 = std::min(h.t2, h.t);
                    h = {true, t, i, u, v, h.t2};
                } else {
                    h.t2 = std::min(h.t2, t);
                }
            }
        } else {
            if (sp + 2 > 128) continue;
            stack[sp++] = nd.right;
            stack[sp++] = nd.left;
        }
    }
    return h;
}

// ---------------------------------------------------------------- shading context
struct HitInfo {
    bool hit;
    float t;
    uint32_t inst, prim;
    float u, v;
    bool front;
};

HitInfo query(const orc_scene* s, f3 o, f3 d, float tmin, float tmax, uint64_t* counter) {
    if (counter) ++*counter;
    DRay r{{o.x, o.y, o.z}, {d.x, d.y, d.z}, tmin, tmax};
    HitInfo hi{};
    if (!(d.x != 0.f || d.y != 0.f || d.z != 0.f)) return hi;  // zero direction: no hit
    Hit h = closest(s, r, false, false);
    if (!h.hit) return hi;
    hi.hit = true;
    hi.t = (float)h.t;
    hi.inst = s->tinst[h.prim];
    hi.prim = s->tprim[h.prim];
    hi.u = (float)h.u;
    hi.v = (float)h.v;
    // front face in object space: CCW as seen from the ray
    const double* w = &s->w2o[9 * hi.inst];
    double dobj[3] = {w[0] * d.x + w[1] * d.y + w[2] * d.z, w[3] * d.x + w[4] * d.y + w[5] * d.z,
                      w[6] * d.x + w[7] * d.y + w[8] * d.z};
    const srt_instance& in = s->instances[hi.inst];
    const srt_mesh_info& mi = s->meshes[in.mesh_id];
    uint32_t base = mi.index_offset + hi.prim * 3u;
    const float* p0 = s->vertices[s->indices[base] + mi.vertex_offset].pos;
    const float* p1 = s->vertices[s->indices[base + 1] + mi.vertex_offset].pos;
    const float* p2 = s->vertices[s->indices[base + 2] + mi.vertex_offset].pos;
    double e1[3] = {(double)p1[0] - p0[0], (double)p1[1] - p0[1], (double)p1[2] - p0[2]};
    double e2[3] = {(double)p2[0] - p0[0], (double)p2[1] - p0[1], (double)p2[2] - p0[2]};
    double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    hi.front = (dobj[0] * n[0] + dobj[1] * n[1] + dobj[2] * n[2]) < 0.0;
    return hi;
}

bool occluded(const orc_scene* s, f3 o, f3 d, float tmin, float tmax, uint64_t* counter) {
    if (counter) ++*counter;
    if (!(d.x != 0.f || d.y != 0.f || d.z != 0.f)) return false;
    DRay r{{o.x, o.y, o.z}, {d.x, d.y, d.z}, tmin, tmax};
    return closest(s, r, false, true).hit;
}

// get_interpolated_normal (shader.wgsl:530-545) + world transform (:573-579)
f3 world_normal(const orc_scene* s, const HitInfo& h) {
    const srt_instance& in = s->instances[h.inst];
    const srt_mesh_info& mi = s->meshes[in.mesh_id];
    uint32_t io = mi.index_offset + h.prim * 3u;
    const float* n0 = s->vertices[s->indices[io] + mi.vertex_offset].normal;
    const float* n1 = s->vertices[s->indices[io + 1] + mi.vertex_offset].normal;
    const float* n2 = s->vertices[s->indices[io + 2] + mi.vertex_offset].normal;
    float w = 1.0f - h.u - h.v;
    f3 a = {n0[0], n0[1], n0[2]}, b = {n1[0], n1[1], n1[2]}, c = {n2[0], n2[1], n2[2]};
    f3 ln = normalize(a * w + b * h.u + c * h.v);
    // local_normal * mat3x3(w2o columns) = transpose(W2O) * n
    const float* m = &s->w2o_f[9 * h.inst];  // row-major
    f3 wn = {ln.x * m[0] + ln.y * m[3] + ln.z * m[6], ln.x * m[1] + ln.y * m[4] + ln.z * m[7],
             ln.x * m[2] + ln.y * m[5] + ln.z * m[8]};
    return normalize(wn);
}

struct LightSample {
    f3 dir;
    float dist, pdf;
    f4 radiance;
};

// sample_random_light: shader.wgsl:477-528
LightSample sample_random_light(const orc_scene* s, f3 hit_pos, f4 wl, Rng& rng) {
    LightSample ls{};
    uint32_t nl = (uint32_t)s->lights.size();
    if (nl == 0u) {
        ls.pdf = 0.f;
        return ls;
    }
    uint32_t li = std::min((uint32_t)(rng.next() * (float)nl), nl - 1u);
    const srt_light& L = s->lights[li];
    float r1 = rng.next();
    float r2 = rng.next();
    float sqrt_r1 = std::sqrt(r1);
    float u = 1.0f - sqrt_r1;
    float v = r2 * sqrt_r1;
    float w = 1.0f - u - v;
    f3 v0 = {L.v0[0], L.v0[1], L.v0[2]}, v1 = {L.v1[0], L.v1[1], L.v1[2]}, v2 = {L.v2[0], L.v2[1], L.v2[2]};
    f3 p = v0 * u + v1 * v + v2 * w;
    f3 e1 = v1 - v0, e2 = v2 - v0;
    f3 normal = normalize(cross(e1, e2));
    float area = length(cross(e1, e2)) * 0.5f;
    f3 to = p - hit_pos;
    float dist_sq = dot(to, to);
    float dist = std::sqrt(dist_sq);
    f3 l = to / dist;
    float cos_light = std::max(dot(normal, -l), 0.0f);
    if (cos_light <= 0.0001f) {
        ls.pdf = 0.f;
        return ls;
    }
    ls.dir = l;
    ls.dist = dist;
    ls.pdf = dist_sq / (area * (float)nl * cos_light);
    ls.radiance = blackbody4(wl, L.params[1]) * L.params[2];
    return ls;
}

struct Counters {
    uint64_t closest = 0, shadow = 0;
};

// ray_color: shader.wgsl:547-703 (MAX_DEPTH = params->max_depth)
f4 ray_color(const orc_scene* s, f3 ro, f3 rd, f4 wl, Rng& rng, const Grid* grid, const GatherParams& gp,
             uint32_t frame, uint32_t max_depth, Counters* cnt) {
    const float T_MIN = 0.0001f, T_MAX = 100.0f;
    f4 acc = splat(0.f);
    f4 thr = splat(1.f);
    bool has_hit_diffuse = false, is_caustic_path = false;
    for (uint32_t i = 0; i < max_depth; ++i) {
        HitInfo h = query(s, ro, rd, T_MIN, T_MAX, cnt ? &cnt->closest : nullptr);
        if (!h.hit) break;
        const srt_material& mat = s->materials[s->instances[h.inst].mat_id];
        f3 wn = world_normal(s, h);
        bool front = h.front;
        f3 ffn = front ? wn : -wn;
        uint32_t type = (uint32_t)mat.extra[0];
        if (type == 3u) {
            if (is_caustic_path) break;
            f4 em = blackbody4(wl, mat.color[0]) * mat.color[1];
            bool no_cull = mat.extra[1] > 0.0f;
            if (front || no_cull) acc = acc + em * thr;  // the MIS weight at :603-627 is never applied
            break;
        }
        if (type == 0u) {
            has_hit_diffuse = true;
            is_caustic_path = false;
        } else if (type == 2u) {
            if (has_hit_diffuse) is_caustic_path = true;
        }
        if (type == 0u) {
            f4 spec = rgb_to_spectrum_vec4({mat.color[0], mat.color[1], mat.color[2]}, wl);
            f3 hit_pos = ro + rd * h.t;
            if (grid) {
                f4 gl = gather_photons(*grid, hit_pos, ffn, wl, frame, gp);
                acc = acc + thr * (spec / PI) * gl;
            } else {
                (void)0;  // no photon pass: the gather of an empty grid adds 0 * density
            }
            LightSample ls = sample_random_light(s, hit_pos, wl, rng);
            if (ls.pdf > 0.0f) {
                if (!occluded(s, hit_pos, ls.dir, 0.001f, ls.dist - 0.001f, cnt ? &cnt->shadow : nullptr)) {
                    float cos_theta = std::max(dot(ffn, ls.dir), 0.0f);
                    f4 bsdf_eval = spec / PI;
                    float bsdf_pdf = cos_theta / PI;
                    float mis = ls.pdf / (ls.pdf + bsdf_pdf);
                    acc = acc + thr * bsdf_eval * ls.radiance * cos_theta * (mis / ls.pdf);
                }
            }
        }
        Scatter sc = sample_bsdf(rd, ffn, mat, front, wl, thr, rng);
        if (sc.absorbed) break;
        thr = thr * sc.att;
        ro = ro + rd * h.t;
        rd = sc.dir;
        if (i > 3u) {
            float p = std::max(std::max(thr.x, thr.y), std::max(thr.z, thr.w));
            if (rng.next() > p) break;
            thr = thr / p;
        }
    }
    return acc;
}

struct Emitted {
    bool stored;
    srt_photon p;
};

// photon_emit main: photon_emit.wgsl:154-331.  Material type 5 (no
// reference counterpart) reflects specularly with the probability of the
// film's Airy reflectance at the photon wavelength, else absorbs.
Emitted emit_photon(const orc_scene* s, uint32_t id, uint32_t frame, uint32_t max_bounces, Counters* cnt,
                    uint32_t seed = 0) {
    Emitted out{};
    Rng rng{pcg_hash(id + frame * 927163u + seed)};
    uint32_t nl = (uint32_t)s->lights.size();
    if (nl == 0u) return out;
    uint32_t li = std::min((uint32_t)(rng.next() * (float)nl), nl - 1u);
    const srt_light& L = s->lights[li];
    f3 v0 = {L.v0[0], L.v0[1], L.v0[2]}, v1 = {L.v1[0], L.v1[1], L.v1[2]}, v2 = {L.v2[0], L.v2[1], L.v2[2]};
    f3 e1 = v1 - v0, e2 = v2 - v0;
    f3 normal = normalize(cross(e1, e2));
    float light_area = length(cross(e1, e2)) * 0.5f;
    float r1 = rng.next();
    float r2 = rng.next();
    float sqrt_r1 = std::sqrt(r1);
    float u = 1.0f - sqrt_r1;
    float v = r2 * sqrt_r1;
    float w = 1.0f - u - v;
    f3 emit_pos = v0 * u + v1 * v + v2 * w;
    f3 emit_dir = normalize(normal + random_unit_vector(rng));
    float temp_k = L.params[1];
    float intensity = L.params[2];
    const float peak = 555.0f, gamma = 40.0f;
    float cdf_min = cauchy_cdf(LAMBDA_MIN);
    float cdf_max = cauchy_cdf(LAMBDA_MAX);
    float cdf_range = cdf_max - cdf_min;
    float rnd = cdf_min + rng.next() * cdf_range;
    float lambda = peak + gamma * std::tan(PI * (rnd - 0.5f));
    lambda = clampf(lambda, LAMBDA_MIN, LAMBDA_MAX);
    float pdf_norm = 1.0f / (cdf_range * PI * gamma);
    float dw = (lambda - peak) / gamma;
    float pdf = pdf_norm / (1.0f + dw * dw);
    float radiance = blackbody_radiance(lambda, temp_k);
    float flux = (radiance / pdf) * light_area * PI;
    float energy = flux * intensity;
    f3 ray_pos = emit_pos + emit_dir * 0.001f;
    f3 ray_dir = emit_dir;
    bool is_caustic = false;
    for (uint32_t depth = 0; depth < max_bounces; ++depth) {
        HitInfo h = query(s, ray_pos, ray_dir, 0.0001f, 100.0f, cnt ? &cnt->closest : nullptr);
        if (!h.hit) break;
        const srt_material& mat = s->materials[s->instances[h.inst].mat_id];
        f3 wn = world_normal(s, h);
        f3 ffn = h.front ? wn : -wn;
        uint32_t type = (uint32_t)mat.extra[0];
        f3 hit_pos = ray_pos + ray_dir * h.t;
        if (type == 0u) {
            if (is_caustic) {
                out.stored = true;
                f3 nd = -ray_dir;
                out.p = {{hit_pos.x, hit_pos.y, hit_pos.z}, lambda, {nd.x, nd.y, nd.z}, energy};
            }
            break;
        } else if (type == 1u) {
            ray_dir = reflect(normalize(ray_dir), ffn);
            ray_pos = hit_pos + ffn * 0.001f;
        } else if (type == 2u) {
            float A = mat.extra[2], B = mat.extra[3];
            float lambda_um = lambda / 1000.0f;
            float ir = A + (B / (lambda_um * lambda_um));
            float ratio = h.front ? 1.0f / ir : ir;
            f3 unit_dir = normalize(ray_dir);
            float cos_theta = std::min(dot(-unit_dir, ffn), 1.0f);
            float sin_theta = std::sqrt(1.0f - cos_theta * cos_theta);
            float r0 = (1.0f - ratio) / (1.0f + ratio);
            r0 = r0 * r0;
            float refl = r0 + (1.0f - r0) * std::pow((1.0f - cos_theta), 5.0f);
            if (ratio * sin_theta > 1.0f || refl > rng.next()) {
                ray_dir = reflect(unit_dir, ffn);
                f3 off = dot(ray_dir, ffn) > 0.0f ? ffn : -ffn;
                ray_pos = hit_pos + off * 0.001f;
            } else {
                is_caustic = true;
                ray_dir = refract(unit_dir, ffn, ratio);
                f3 off = dot(ray_dir, ffn) > 0.0f ? ffn : -ffn;
                ray_pos = hit_pos + off * 0.001f;
            }
        } else if (type == 4u) {
            float n2 = mat.extra[2], n3 = mat.extra[3];
            float d = std::max(mat.extra[1], 50.0f);
            f3 unit_dir = normalize(ray_dir);
            float cos_theta = std::min(dot(-unit_dir, ffn), 1.0f);
            // select(n1 / n3, n3 / n1, is_front_face): n3 / n1 on the front face
            float ratio = h.front ? n3 / 1.0f : 1.0f / n3;
            float sin_t_sq = ratio * ratio * (1.0f - cos_theta * cos_theta);
            if (sin_t_sq > 1.0f) {
                ray_dir = reflect(unit_dir, ffn);
                is_caustic = true;
            } else {
                bool tir;
                float F = thin_film_1(cos_theta, 1.0f, n2, n3, d, lambda, &tir);
                if (rng.next() < F) {
                    ray_dir = reflect(unit_dir, ffn);
                    is_caustic = true;
                } else {
                    ray_dir = refract(unit_dir, ffn, ratio);
                    is_caustic = true;
                }
            }
            // ray_pos is not advanced here (photon_emit.wgsl:291-326)
        } else if (type == 5u) {
            f3 unit_dir = normalize(ray_dir);
            float cos_theta = std::min(dot(-unit_dir, ffn), 1.0f);
            bool tir;
            float F = thin_film_1(cos_theta, 1.0f, mat.extra[2], mat.extra[3], std::max(mat.extra[1], 50.0f),
                                  lambda, &tir);
            if (rng.next() < F) {
                ray_dir = reflect(unit_dir, ffn);
                ray_pos = hit_pos + ffn * 0.001f;
                is_caustic = true;
            } else {
                break;
            }
        } else {
            break;
        }
    }
    return out;
}

GatherParams gather_params(const srt_params* p) {
    GatherParams g;
    g.cell = p->cell_size;
    g.r0 = p->gather_radius0;
    g.rexp = p->radius_exponent;
    g.spectral_radius = p->spectral_radius;
    g.norm_count = p->photon_norm_count > 0.f ? p->photon_norm_count : (float)p->photons_per_frame;
    g.cap = p->gather_cap;
    return g;
}

inline float u2f(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline uint32_t f2u(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

// Camera ray: shader.wgsl:713-728.  Returns the rng after the two jitter draws.
void camera_ray(const srt_camera_uniform* cam, uint32_t x, uint32_t y, uint32_t w, uint32_t h, Rng& rng, f3* o,
                f3* d) {
    const float* vi = cam->view_inverse;
    const float* pi = cam->proj_inverse;
    f3 origin = {vi[12], vi[13], vi[14]};
    float jx = rng.next();
    float jy = rng.next();
    float ux = ((float)x + jx) / (float)w;
    float uy = ((float)y + jy) / (float)h;
    float nx = ux * 2.0f - 1.0f, ny = uy * 2.0f - 1.0f;
    // (view_inv * proj_inv) * vec4(ndc, 1, 1)
    float m[16];
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r)
            m[4 * c + r] = vi[r] * pi[4 * c] + vi[4 + r] * pi[4 * c + 1] + vi[8 + r] * pi[4 * c + 2] +
                           vi[12 + r] * pi[4 * c + 3];
    float t[4];
    for (int r = 0; r < 4; ++r) t[r] = m[r] * nx + m[4 + r] * ny + m[8 + r] * 1.0f + m[12 + r] * 1.0f;
    f3 tw = {t[0] / t[3], t[1] / t[3], t[2] / t[3]};
    *o = origin;
    *d = normalize(tw - origin);
}

}  // namespace

// ==================================================================== C API
extern "C" {

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

orc_scene* orc_scene_create(const srt_scene_arrays* a) {
    orc_scene* s = new orc_scene();
    s->vertices.assign(a->vertices, a->vertices + a->n_vertices);
    s->indices.assign(a->indices, a->indices + a->n_indices);
    s->meshes.assign(a->mesh_infos, a->mesh_infos + a->n_meshes);
    s->materials.assign(a->materials, a->materials + a->n_materials);
    s->instances.assign(a->instances, a->instances + a->n_instances);
    s->lights.assign(a->lights, a->lights + a->n_lights);
    size_t ni = s->instances.size();
    s->w2o.resize(9 * ni);
    s->w2o_f.resize(9 * ni);
    s->inst_first.resize(ni);
    // mesh triangle counts: meshes occupy consecutive index ranges
    std::vector<uint32_t> mesh_tris(s->meshes.size());
    for (size_t m = 0; m < s->meshes.size(); ++m) {
        uint32_t end = m + 1 < s->meshes.size() ? s->meshes[m + 1].index_offset : (uint32_t)s->indices.size();
        mesh_tris[m] = (end - s->meshes[m].index_offset) / 3u;
    }
    size_t total = 0;
    for (size_t i = 0; i < ni; ++i) {
        s->inst_first[i] = (uint32_t)total;
        total += mesh_tris[s->instances[i].mesh_id];
    }
    s->tv.resize(9 * total);
    s->tinst.resize(total);
    s->tprim.resize(total);
    for (size_t i = 0; i < ni; ++i) {
        const float* M = s->instances[i].transform;  // column-major
        double a3[9] = {M[0], M[4], M[8], M[1], M[5], M[9], M[2], M[6], M[10]};  // row-major 3x3
        double det = a3[0] * (a3[4] * a3[8] - a3[5] * a3[7]) - a3[1] * (a3[3] * a3[8] - a3[5] * a3[6]) +
                     a3[2] * (a3[3] * a3[7] - a3[4] * a3[6]);
        double inv[9] = {(a3[4] * a3[8] - a3[5] * a3[7]) / det, (a3[2] * a3[7] - a3[1] * a3[8]) / det,
                         (a3[1] * a3[5] - a3[2] * a3[4]) / det, (a3[5] * a3[6] - a3[3] * a3[8]) / det,
                         (a3[0] * a3[8] - a3[2] * a3[6]) / det, (a3[2] * a3[3] - a3[0] * a3[5]) / det,
                         (a3[3] * a3[7] - a3[4] * a3[6]) / det, (a3[1] * a3[6] - a3[0] * a3[7]) / det,
                         (a3[0] * a3[4] - a3[1] * a3[3]) / det};
        for (int k = 0; k < 9; ++k) {
            s->w2o[9 * i + k] = inv[k];
            s->w2o_f[9 * i + k] = (float)inv[k];
        }
        uint32_t mesh = s->instances[i].mesh_id;
        const srt_mesh_info& mi = s->meshes[mesh];
        for (uint32_t p = 0; p < mesh_tris[mesh]; ++p) {
            size_t t = s->inst_first[i] + p;
            s->tinst[t] = (uint32_t)i;
            s->tprim[t] = p;
            for (int k = 0; k < 3; ++k) {
                const float* v = s->vertices[s->indices[mi.index_offset + 3 * p + k] + mi.vertex_offset].pos;
                for (int r = 0; r < 3; ++r)
                    s->tv[9 * t + 3 * k + r] =
                        (double)M[r] * v[0] + (double)M[4 + r] * v[1] + (double)M[8 + r] * v[2] + (double)M[12 + r];
            }
        }
    }
    build_bvh(s);
    return s;
}

void orc_scene_destroy(orc_scene* s) { delete s; }

void orc_ray_query(const orc_scene* s, const float o[3], const float d[3], float tmin, float tmax, int any_hit,
                   orc_query_hit* out) {
    *out = orc_query_hit{};
    const f3 of = {o[0], o[1], o[2]}, df = {d[0], d[1], d[2]};
    if (any_hit) {
        out->hit = occluded(s, of, df, tmin, tmax, nullptr) ? 1u : 0u;
        return;
    }
    const HitInfo h = query(s, of, df, tmin, tmax, nullptr);
    if (!h.hit) return;
    out->hit = 1u;
    out->inst = h.inst;
    out->prim = h.prim;
    out->front = h.front ? 1u : 0u;
    out->t = h.t;
    out->u = h.u;
    out->v = h.v;
}

void orc_instance_w2o(const orc_scene* s, uint32_t inst, float out[9]) {
    for (int k = 0; k < 9; ++k) out[k] = s->w2o_f[9 * (size_t)inst + k];
}
uint64_t orc_scene_num_tris(const orc_scene* s) { return s->tinst.size(); }

void orc_trace(const orc_scene* s, const srt_ray* rays, uint32_t n, int any_hit, int brute, double* t_out,
               uint32_t* prim_out, double* u_out, double* v_out, double* t_second) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const srt_ray& r = rays[i];
        DRay d{{r.origin[0], r.origin[1], r.origin[2]}, {r.dir[0], r.dir[1], r.dir[2]}, r.tmin, r.tmax};
        Hit h{};
        h.hit = false;
        h.t2 = std::numeric_limits<double>::infinity();
        if (r.dir[0] != 0.f || r.dir[1] != 0.f || r.dir[2] != 0.f)
            h = closest(s, d, brute != 0, any_hit != 0, t_second != nullptr);
        if (t_out) t_out[i] = h.hit ? h.t : std::numeric_limits<double>::infinity();
        if (prim_out) prim_out[i] = h.hit ? h.prim : 0xFFFFFFFFu;
        if (u_out) u_out[i] = h.hit ? h.u : 0.0;
        if (v_out) v_out[i] = h.hit ? h.v : 0.0;
        if (t_second) t_second[i] = h.t2;
    }
}

// Where the line of each ray meets the plane of the given flattened triangle
// (FP64, world space): the ray parameter t there and the distance from that
// point to the triangle's boundary (the nearest of its three edge segments),
// positive inside the triangle and negative outside.  A ray that passes
// within a small distance of a triangle's boundary is one whose hit or miss
// of that triangle FP32 arithmetic can decide either way.  cos_out (may be
// NULL): |cos| of the angle between the ray and the plane's normal (the
// point's uncertainty along the ray grows as 1 / cos).  prim = 0xFFFFFFFF
// or a ray parallel to the plane gives t = inf, distance = inf and cos = 0.
void orc_tri_probe(const orc_scene* s, const srt_ray* rays, const uint32_t* prims, uint32_t n, double* t_out,
                   double* edge_out, double* cos_out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const double inf = std::numeric_limits<double>::infinity();
        t_out[i] = inf;
        edge_out[i] = inf;
        if (cos_out) cos_out[i] = 0.0;
        uint32_t p = prims[i];
        if (p >= s->tinst.size()) continue;
        const double* v = &s->tv[9 * (size_t)p];
        const srt_ray& r = rays[i];
        double o[3] = {r.origin[0], r.origin[1], r.origin[2]}, d[3] = {r.dir[0], r.dir[1], r.dir[2]};
        double e1[3] = {v[3] - v[0], v[4] - v[1], v[5] - v[2]};
        double e2[3] = {v[6] - v[0], v[7] - v[1], v[8] - v[2]};
        double nrm[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        double den = nrm[0] * d[0] + nrm[1] * d[1] + nrm[2] * d[2];
        if (den == 0.0) continue;
        double t = (nrm[0] * (v[0] - o[0]) + nrm[1] * (v[1] - o[1]) + nrm[2] * (v[2] - o[2])) / den;
        double x[3] = {o[0] + t * d[0], o[1] + t * d[1], o[2] + t * d[2]};
        // inside test by the signs of the edge normals' dot products
        bool inside = true;
        double dist = inf;
        for (int k = 0; k < 3; ++k) {
            const double* a = v + 3 * k;
            const double* b = v + 3 * ((k + 1) % 3);
            double ab[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
            double ax[3] = {x[0] - a[0], x[1] - a[1], x[2] - a[2]};
            double c[3] = {ab[1] * ax[2] - ab[2] * ax[1], ab[2] * ax[0] - ab[0] * ax[2], ab[0] * ax[1] - ab[1] * ax[0]};
            if (c[0] * nrm[0] + c[1] * nrm[1] + c[2] * nrm[2] < 0.0) inside = false;
            double l2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
            double f = l2 > 0.0 ? (ax[0] * ab[0] + ax[1] * ab[1] + ax[2] * ab[2]) / l2 : 0.0;
            f = std::min(1.0, std::max(0.0, f));
            double q[3] = {ax[0] - f * ab[0], ax[1] - f * ab[1], ax[2] - f * ab[2]};
            dist = std::min(dist, std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]));
        }
        t_out[i] = t;
        edge_out[i] = inside ? dist : -dist;
        if (cos_out) {
            double nl = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
            double dl = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            cos_out[i] = std::fabs(den) / (nl * dl);
        }
    }
}

int orc_device_math(int op, uint32_t n, const void* in, void* out, const void* aux) {
    const float* fi = (const float*)in;
    const uint32_t* ui = (const uint32_t*)in;
    float* fo = (float*)out;
    uint32_t* uo = (uint32_t*)out;
    for (uint32_t i = 0; i < n; ++i) {
        switch (op) {
            case 0:
                uo[i] = pcg_hash(ui[i]);
                break;
            case 1: {
                f3 c = sample_cie_xyz(fi[i]);
                fo[3 * i] = c.x;
                fo[3 * i + 1] = c.y;
                fo[3 * i + 2] = c.z;
            } break;
            case 2:
                fo[i] = blackbody_radiance(fi[2 * i], fi[2 * i + 1]);
                break;
            case 102:  // photon_emit.wgsl:93-105 (the same arithmetic as shader.wgsl's copy)
                fo[i] = blackbody_radiance(fi[2 * i], fi[2 * i + 1]);
                break;
            case 109: {  // fresnel_thin_film_1d, photon_emit.wgsl:107-132
                const float* a = fi + 6 * i;
                bool tir;
                fo[i] = thin_film_1(a[0], a[1], a[2], a[3], a[4], a[5], &tir);
            } break;
            case 110:  // reflectance, shader.wgsl:264-269
                fo[i] = reflectance(fi[2 * i], fi[2 * i + 1]);
                break;
            case 3: {
                const float* a = fi + 7 * i;
                f4 r = rgb_to_spectrum_vec4({a[0], a[1], a[2]}, {a[3], a[4], a[5], a[6]});
                std::memcpy(fo + 4 * i, &r, 16);
            } break;
            case 4: {
                const float* a = fi + 9 * i;
                f4 r = fresnel_thin_film(a[0], a[1], a[2], a[3], a[4], {a[5], a[6], a[7], a[8]});
                std::memcpy(fo + 4 * i, &r, 16);
            } break;
            case 5: {
                Rng rng{ui[i]};
                Hero h = sample_hero(rng);
                std::memcpy(fo + 5 * i, &h.wl, 16);
                fo[5 * i + 4] = h.sum_pdf;
            } break;
            case 6: {
                const float* a = fi + 24 * i;
                srt_material m;
                std::memcpy(&m, a + 6, 32);
                Rng rng{f2u(a[23])};
                Scatter sc = sample_bsdf({a[0], a[1], a[2]}, {a[3], a[4], a[5]}, m, a[14] != 0.0f,
                                         {a[15], a[16], a[17], a[18]}, {a[19], a[20], a[21], a[22]}, rng);
                float* o = fo + 10 * i;
                o[0] = sc.dir.x;
                o[1] = sc.dir.y;
                o[2] = sc.dir.z;
                std::memcpy(o + 3, &sc.att, 16);
                o[7] = sc.absorbed ? 1.0f : 0.0f;
                o[8] = u2f(rng.s);
                o[9] = 0.f;
            } break;
            case 7: {
                const float* a = fi + 5 * i;
                f3 j = grid_jitter(f2u(a[3]), a[4]);
                uo[i] = hash_position({a[0], a[1], a[2]}, j, a[4], 22);
            } break;
            case 8: {
                const uint32_t* a = ui + 5 * i;
                Rng rng{a[4]};
                f3 o, d;
                camera_ray((const srt_camera_uniform*)aux, a[0], a[1], a[2], a[3], rng, &o, &d);
                float* r = fo + 7 * i;
                r[0] = o.x;
                r[1] = o.y;
                r[2] = o.z;
                r[3] = d.x;
                r[4] = d.y;
                r[5] = d.z;
                r[6] = u2f(rng.s);
            } break;
            default:
                return 1;
        }
    }
    return 0;
}

uint32_t orc_photon_emit(const orc_scene* s, uint32_t n_photons, uint32_t frame, uint32_t max_bounces,
                         srt_photon* out, uint32_t* emitter_out, int n_threads) {
    std::vector<Emitted> em(n_photons);
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < (int64_t)n_photons; ++i) em[i] = emit_photon(s, (uint32_t)i, frame, max_bounces, nullptr);
    uint32_t c = 0;
    for (uint32_t i = 0; i < n_photons; ++i)
        if (em[i].stored) {
            if (out) out[c] = em[i].p;
            if (emitter_out) emitter_out[c] = i;
            ++c;
        }
    return c;
}

void orc_photon_grid_build(const srt_photon* photons, uint32_t n, uint32_t frame, float cell, uint32_t hash_bits,
                           uint64_t* keys_out, uint32_t* ranges_out) {
    std::vector<uint64_t> keys;
    Grid g;
    grid_build(photons, n, frame, cell, hash_bits, keys, ranges_out ? &g : nullptr);
    if (keys_out) std::memcpy(keys_out, keys.data(), 8ull * n);
    if (ranges_out) std::memcpy(ranges_out, g.ranges.data(), 4ull * g.ranges.size());
}

void orc_photon_gather(const srt_photon* photons, uint32_t n, const float* q, uint32_t n_q, uint32_t frame,
                       const srt_params* params, float* out) {
    std::vector<uint64_t> keys;
    Grid g;
    grid_build(photons, n, frame, params->cell_size, params->hash_bits, keys, &g);
    GatherParams gp = gather_params(params);
    for (uint32_t i = 0; i < n_q; ++i) {
        const float* a = q + 10 * i;
        f4 r = gather_photons(g, {a[0], a[1], a[2]}, {a[3], a[4], a[5]}, {a[6], a[7], a[8], a[9]}, frame, gp);
        std::memcpy(out + 4 * i, &r, 16);
    }
}

void orc_render_frame(const orc_scene* s, const srt_camera_uniform* cam, uint32_t w, uint32_t h,
                      const srt_params* params, uint32_t row_stride, uint32_t row_phase, float* accum, uint8_t* ldr,
                      float* radiance_out, uint64_t* stats_out, int n_threads) {
    orc_render_frame_photons(s, cam, w, h, params, nullptr, 0, row_stride, row_phase, accum, ldr, radiance_out,
                             stats_out, n_threads);
}

void orc_render_frame_photons(const orc_scene* s, const srt_camera_uniform* cam, uint32_t w, uint32_t h,
                              const srt_params* params, const srt_photon* photons_in, uint32_t n_photons_in,
                              uint32_t row_stride, uint32_t row_phase, float* accum, uint8_t* ldr,
                              float* radiance_out, uint64_t* stats_out, int n_threads) {
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
    uint32_t frame = cam->frame_count;
    Counters cnt;
    // 1. photon pass + grid (renderer/mod.rs:177-193)
    Grid grid;
    bool have_grid = params->photons_per_frame > 0;
    uint32_t stored = 0;
    if (have_grid && photons_in) {
        // the given photon set (e.g. another implementation's photon pass)
        stored = n_photons_in;
        std::vector<uint64_t> keys;
        grid_build(photons_in, stored, frame, params->cell_size, params->hash_bits, keys, &grid);
    } else if (have_grid) {
        uint32_t np = params->photons_per_frame;
        std::vector<Emitted> em(np);
        uint64_t ph_rays = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : ph_rays)
        for (int64_t i = 0; i < (int64_t)np; ++i) {
            Counters local;
            em[i] = emit_photon(s, (uint32_t)i, frame, params->photon_max_bounces, &local, params->seed);
            ph_rays += local.closest;
        }
        cnt.closest += ph_rays;
        std::vector<srt_photon> ph;
        ph.reserve(np / 8);
        for (uint32_t i = 0; i < np; ++i)
            if (em[i].stored) ph.push_back(em[i].p);
        stored = (uint32_t)ph.size();
        std::vector<uint64_t> keys;
        grid_build(ph.data(), stored, frame, params->cell_size, params->hash_bits, keys, &grid);
    }
    GatherParams gp = gather_params(params);
    if (row_stride == 0) row_stride = 1;
    // 2. camera paths (shader.wgsl:708-823)
    int64_t total = (int64_t)w * h;
    uint64_t n_closest = 0, n_shadow = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : n_closest, n_shadow)
    for (int64_t idx = 0; idx < total; ++idx) {
        uint32_t x = (uint32_t)(idx % w), y = (uint32_t)(idx / w);
        if (y % row_stride != row_phase) continue;
        Rng rng{pcg_hash(x + y * w + frame * 927163u + params->seed)};
        f3 o, d;
        camera_ray(cam, x, y, w, h, rng, &o, &d);
        Hero hero = sample_hero(rng);
        Counters local;
        f4 L = ray_color(s, o, d, hero.wl, rng, have_grid ? &grid : nullptr, gp, frame, params->max_depth, &local);
        n_closest += local.closest;
        n_shadow += local.shadow;
        if (radiance_out) std::memcpy(radiance_out + 4 * idx, &L, 16);
        f3 xyz = {0, 0, 0};
        f4 wl = hero.wl;
        xyz = xyz + sample_cie_xyz(wl.x) * L.x;
        xyz = xyz + sample_cie_xyz(wl.y) * L.y;
        xyz = xyz + sample_cie_xyz(wl.z) * L.z;
        xyz = xyz + sample_cie_xyz(wl.w) * L.w;
        xyz = xyz * (1.0f / hero.sum_pdf);
        f3 rgb = xyz_to_srgb(xyz);
        f4 cur = splat(0.f);
        if (frame > 0u) std::memcpy(&cur, accum + 4 * idx, 16);
        f4 na = cur + f4{rgb.x, rgb.y, rgb.z, 1.0f};
        std::memcpy(accum + 4 * idx, &na, 16);
        if (ldr) {
            // shader.wgsl:809-822
            f3 fc = {std::max(na.x / na.w * 1.0f, 0.0f), std::max(na.y / na.w * 1.0f, 0.0f),
                     std::max(na.z / na.w * 1.0f, 0.0f)};
            float luma = fc.x * 0.2126f + fc.y * 0.7152f + fc.z * 0.0722f;
            float mapped = luma / (luma + 1.0f);
            if (luma > 0.00001f) fc = fc * (mapped / luma);
            auto q = [](float c) { return (uint8_t)std::nearbyint(clampf(c, 0.0f, 1.0f) * 255.0f); };
            ldr[4 * idx] = q(fc.x);
            ldr[4 * idx + 1] = q(fc.y);
            ldr[4 * idx + 2] = q(fc.z);
            ldr[4 * idx + 3] = 255;
        }
    }
    if (stats_out) {
        uint64_t paths = 0;
        for (uint32_t y = 0; y < h; ++y)
            if (y % row_stride == row_phase) paths += w;
        stats_out[0] = paths;
        stats_out[1] = cnt.closest + n_closest;
        stats_out[2] = n_shadow;
        stats_out[3] = have_grid ? params->photons_per_frame : 0;
        stats_out[4] = stored;
    }
}

}  // extern "C"
