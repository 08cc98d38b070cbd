// guide.cu — neural path guiding kernels (BF16 tensor cores, FP32 accumulate).
//
// The guide replaces the cosine sampling of Lambert vertices
// (shader.wgsl:461-467) by a one-sample mixture of the learned vMF mixture q
// and the cosine lobe: with probability sel sample q, else the BSDF; the
// weight is f cos / (sel q + (1 - sel) cos / pi), so the estimator stays
// unbiased and converges to the same image as the plain method (the NEE
// weight of shader.wgsl:666 keeps its cos / pi term).
//
// Matrix products use mma.sync.m16n8k16 (bf16 x bf16 -> fp32).  A warp owns
// 16 samples; the accumulator fragments of two adjacent 8-column tiles form
// the A fragment of the next layer's 16-wide k step, so hidden activations
// stay in registers between layers.  Training: a forward/backward pass that
// writes every layer's activations and deltas (bf16), a split-K weight
// gradient product over the samples, and Adam on FP32 master weights.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "guide.cuh"
#include "render_kernels.h"
#include "umma.cuh"

namespace srt {

namespace {

constexpr int GWI = 8;  // warps per block of the inference kernels (2 blocks per SM)
constexpr int GWT = 8;  // warps per block of the training forward/backward kernel (1 block per SM)
// Per-warp staging of the inference kernels: the encoded rows (16 x 136
// bf16); the raw outputs (16 x 52 fp32) reuse the same bytes once the
// first layer has taken its A fragments.
constexpr int IN_BYTES = 16 * g_pad(G_ENC) * 2;
static_assert(16 * 52 * 4 <= IN_BYTES, "outputs alias the encoded rows");

SRT_DEV uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

SRT_DEV void mma16816(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
SRT_DEV void ldsm4(uint32_t (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
SRT_DEV void ldsm4t(uint32_t (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
SRT_DEV uint32_t pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}
// pack2 of max(lo, 0), max(hi, 0): the conversion applies the ReLU itself.
SRT_DEV uint32_t pack2_relu(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;\n" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}
SRT_DEV float2 unpack2(uint32_t u) {
    __nv_bfloat162 v = *reinterpret_cast<__nv_bfloat162*>(&u);
    return __bfloat1622float2(v);
}

// A fragment (16 x 16 at column k0) of a row-major bf16 matrix in shared memory.
SRT_DEV void load_a(uint32_t (&a)[4], const __nv_bfloat16* m, int stride, int k0) {
    int t = threadIdx.x & 31;
    const __nv_bfloat16* p = m + ((t & 7) + 8 * ((t >> 3) & 1)) * stride + k0 + 8 * (t >> 4);
    ldsm4(a, p);
}
// B fragments of two 8-column tiles (n0, n0 + 8) at k0 from W [n][k] row-major.
SRT_DEV void load_b2(uint32_t (&b)[4], const __nv_bfloat16* W, int stride, int n0, int k0) {
    int t = threadIdx.x & 31;
    const __nv_bfloat16* p = W + (n0 + (t & 7) + 8 * (t >> 4)) * stride + k0 + 8 * ((t >> 3) & 1);
    ldsm4(b, p);
}
// The same fragments from B stored [k][n] row-major (transposing loads).
SRT_DEV void load_b2t(uint32_t (&b)[4], const __nv_bfloat16* B, int stride, int n0, int k0) {
    int t = threadIdx.x & 31;
    const __nv_bfloat16* p = B + (k0 + (t & 7) + 8 * ((t >> 3) & 1)) * stride + n0 + 8 * (t >> 4);
    ldsm4t(b, p);
}

// One dense layer for the warp's 16 samples: c = a W^T + bias.
template <int K, int N>
SRT_DEV void layer(const uint32_t (&a)[K / 16][4], const __nv_bfloat16* W, const float* bias, float (&c)[N / 8][4]) {
    int t = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < N / 8; ++j) {
        float b0 = bias[8 * j + 2 * (t & 3)], b1 = bias[8 * j + 2 * (t & 3) + 1];
        c[j][0] = b0;
        c[j][1] = b1;
        c[j][2] = b0;
        c[j][3] = b1;
    }
#pragma unroll
    for (int s = 0; s < K / 16; ++s) {
#pragma unroll
        for (int j = 0; j < N / 8; j += 2) {
            uint32_t b[4];
            load_b2(b, W, g_pad(K), 8 * j, 16 * s);
            mma16816(c[j], a[s], b[0], b[1]);
            mma16816(c[j + 1], a[s], b[2], b[3]);
        }
    }
}

// Accumulators -> next A fragments (ReLU, bf16).
template <int N>
SRT_DEV void relu_to_a(const float (&c)[N / 8][4], uint32_t (&a)[N / 16][4]) {
#pragma unroll
    for (int s = 0; s < N / 16; ++s) {
        a[s][0] = pack2_relu(c[2 * s][0], c[2 * s][1]);
        a[s][1] = pack2_relu(c[2 * s][2], c[2 * s][3]);
        a[s][2] = pack2_relu(c[2 * s + 1][0], c[2 * s + 1][1]);
        a[s][3] = pack2_relu(c[2 * s + 1][2], c[2 * s + 1][3]);
    }
}

// Frequency encoding of 5 of the 10 inputs (half h) of one sample into its
// bf16 row: feature 12 d + 2 k = sin(2^k pi x_d), + 1 = cos; 120..127 = 0.
// Octaves k >= 1 come from the double-angle identities with every rounding
// pinned (sin' = (2 s) c, cos' = fma(c, c, -(s s))), so a CPU restatement
// reproduces them bit for bit from the same octave-0 values.
SRT_DEV void encode_half(const float* x, int h, __nv_bfloat16* row) {
#pragma unroll
    for (int dd = 0; dd < 5; ++dd) {
        int d = 5 * h + dd;
        float s, c;
        sincospif(x[d], &s, &c);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            row[12 * d + 2 * k] = __float2bfloat16_rn(s);
            row[12 * d + 2 * k + 1] = __float2bfloat16_rn(c);
            float s2 = __fmul_rn(__fmul_rn(2.0f, s), c);
            float c2 = __fmaf_rn(c, c, -__fmul_rn(s, s));
            s = s2;
            c = c2;
        }
    }
    if (h == 1)
        for (int f = 120; f < 128; ++f) row[f] = __float2bfloat16_rn(0.0f);
}

// Raw outputs of one sample -> mixture parameters.
struct Mix {
    float3 mu[G_LOBES];
    float kappa[G_LOBES];
    float pi[G_LOBES];
    float sel, sel_sig;
    float norm[G_LOBES];
    float lk[G_LOBES];
    float c[G_LOBES];   // vMF normalisation kappa / (2 pi (1 - e^-2kappa))
    float e2[G_LOBES];  // e^-2kappa
};
SRT_DEV void mixture(const float* r, Mix& m) {
    float mx = -3.4e38f;
#pragma unroll
    for (int j = 0; j < G_LOBES; ++j) mx = fmaxf(mx, r[5 * j + 4]);
    float sum = 0.f;
#pragma unroll
    for (int j = 0; j < G_LOBES; ++j) {
        float3 v = f3(r[5 * j], r[5 * j + 1], r[5 * j + 2]);
        float n = fmaxf(length(v), 1e-12f);
        m.norm[j] = n;
        m.mu[j] = v / n;
        m.lk[j] = r[5 * j + 3];
        m.kappa[j] = expf(clampf(r[5 * j + 3], G_KAPPA_LO, G_KAPPA_HI));
        m.c[j] = m.kappa[j] / (2.0f * PI * (-expm1f(-2.0f * m.kappa[j])));
        m.e2[j] = expf(-2.0f * m.kappa[j]);
        m.pi[j] = expf(r[5 * j + 4] - mx);
        sum += m.pi[j];
    }
#pragma unroll
    for (int j = 0; j < G_LOBES; ++j) m.pi[j] /= sum;
    m.sel_sig = 1.0f / (1.0f + expf(-r[40]));
    m.sel = G_SEL_LO + G_SEL_SPAN * m.sel_sig;
}
// The mixture with the hardware's fast approximations (the tcgen05 inference
// path and training): exponentials and logarithms through ex2 / lg2 (__expf,
// __logf), reciprocal square roots for normalisation, approximate division.
// Their relative errors (~1e-6) are far below the noise of one sample, and
// sampling and pdf evaluation use the same functions.
SRT_DEV void mixture_fast(const float* r, Mix& m) {
    float mx = -3.4e38f;
#pragma unroll
    for (int j = 0; j < G_LOBES; ++j) mx = fmaxf(mx, r[5 * j + 4]);
    float sum = 0.f;
#pragma unroll
    for (int j = 0; j < G_LOBES; ++j) {
        const float3 v = f3(r[5 * j], r[5 * j + 1], r[5 * j + 2]);
        const float d2 = dot(v, v);
        const float inv = rsqrtf(fmaxf(d2, 1e-24f));
        m.norm[j] = d2 * inv;
        m.mu[j] = v * inv;
        m.lk[j] = r[5 * j + 3];
        const float k = __expf(clampf(r[5 * j + 3], G_KAPPA_LO, G_KAPPA_HI));
        const float e2 = __expf(-2.0f * k);
        m.kappa[j] = k;
        m.e2[j] = e2;
        m.c[j] = __fdividef(k, 2.0f * PI * (1.0f - e2));
        m.pi[j] = __expf(r[5 * j + 4] - mx);
        sum += m.pi[j];
    }
    const float isum = __fdividef(1.0f, sum);
#pragma unroll
    for (int j = 0; j < G_LOBES; ++j) m.pi[j] *= isum;
    m.sel_sig = __fdividef(1.0f, 1.0f + __expf(-r[40]));
    m.sel = G_SEL_LO + G_SEL_SPAN * m.sel_sig;
}
SRT_DEV float3 normalize_fast(float3 a) { return a * rsqrtf(dot(a, a)); }
SRT_DEV float3 vmf_sample_fast(float3 mu, float k, float e2, float u1, float u2) {
    float w = 1.0f + __fdividef(__logf(u1 + (1.0f - u1) * e2), k);
    w = clampf(w, -1.0f, 1.0f);
    const float r = sqrtf(fmaxf(0.0f, 1.0f - w * w));
    float sp, cp;
    sincospif(2.0f * u2, &sp, &cp);
    const float3 t = fabsf(mu.x) > 0.9f ? f3(0.f, 1.f, 0.f) : f3(1.f, 0.f, 0.f);
    const float3 b1 = normalize_fast(cross(mu, t));
    const float3 b2 = cross(mu, b1);
    return normalize_fast(mu * w + b1 * (r * cp) + b2 * (r * sp));
}
SRT_DEV float vmf(float3 mu, float k, float3 w) {
    return k / (2.0f * PI * (-expm1f(-2.0f * k))) * expf(k * (dot(mu, w) - 1.0f));
}
// Sample a vMF lobe (Wenzel Jakob's stable form of Wood's method); e2 = e^-2k.
SRT_DEV float3 vmf_sample_e2(float3 mu, float k, float e2, float u1, float u2) {
    float w = 1.0f + logf(u1 + (1.0f - u1) * e2) / k;
    w = clampf(w, -1.0f, 1.0f);
    float r = sqrtf(fmaxf(0.0f, 1.0f - w * w));
    float sp, cp;
    sincospif(2.0f * u2, &sp, &cp);
    float3 t = fabsf(mu.x) > 0.9f ? f3(0.f, 1.f, 0.f) : f3(1.f, 0.f, 0.f);
    float3 b1 = normalize(cross(mu, t));
    float3 b2 = cross(mu, b1);
    return normalize(mu * w + b1 * (r * cp) + b2 * (r * sp));
}
SRT_DEV float3 vmf_sample(float3 mu, float k, float u1, float u2) {
    return vmf_sample_e2(mu, k, expf(-2.0f * k), u1, u2);
}

// Copies a rows x cols bf16 matrix (rows contiguous in global memory) into
// shared memory rows padded to g_pad(cols), 16 bytes per load.
// The copies are asynchronous (cp.async, all in flight at once); the caller
// waits with cp_async_wait_all() and then synchronises the block.
SRT_DEV void copy_rows(__nv_bfloat16* dst, const __nv_bfloat16* src, int rows, int cols) {
    const int cpr = cols / 8;  // 16-byte chunks per row
    for (int i = threadIdx.x; i < rows * cpr; i += blockDim.x) {
        int r = i / cpr, c = i - r * cpr;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst + r * g_pad(cols) + 8 * c)),
                     "l"(src + 8 * i));
    }
}
SRT_DEV void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// The mixture of one sample held by a lane pair (lanes l and l ^ 16): this
// lane owns lobes 4 half .. 4 half + 3.  Every function here is called by
// all 32 lanes of the warp (it shuffles).
struct HalfMix {
    float3 mu[4];
    float kappa[4];
    float pi[4];  // normalised over all 8 lobes
    float cdf0;   // total weight of lobes 0..3
    float sel;
};
SRT_DEV void half_mixture(const float* r, int half, HalfMix& m) {
    float mx = -3.4e38f;
#pragma unroll
    for (int i = 0; i < 4; ++i) mx = fmaxf(mx, r[5 * (4 * half + i) + 4]);
    mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, 16));
    float sum = 0.f;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int j = 4 * half + i;
        float3 v = f3(r[5 * j], r[5 * j + 1], r[5 * j + 2]);
        m.mu[i] = v / fmaxf(length(v), 1e-12f);
        m.kappa[i] = expf(clampf(r[5 * j + 3], G_KAPPA_LO, G_KAPPA_HI));
        m.pi[i] = expf(r[5 * j + 4] - mx);
        sum += m.pi[i];
    }
    const float other = __shfl_xor_sync(0xFFFFFFFFu, sum, 16);
    const float inv = 1.0f / (sum + other);
#pragma unroll
    for (int i = 0; i < 4; ++i) m.pi[i] *= inv;
    m.cdf0 = (half == 0 ? sum : other) * inv;
    m.sel = G_SEL_LO + G_SEL_SPAN / (1.0f + expf(-r[40]));
}
// Direction drawn from the mixture with (u0: lobe, u1, u2: vMF); the lobe's
// owner samples it and both lanes receive it.
SRT_DEV float3 half_sample(const HalfMix& m, int half, float u0, float u1, float u2) {
    const bool first = u0 < m.cdf0;  // the lobe lies in lanes-0 half
    const bool mine = (half == 0) == first;
    float acc = half == 0 ? 0.f : m.cdf0;
    float3 mu = m.mu[3];
    float k = m.kappa[3];  // rounding fallback: the half's last lobe
    bool found = false;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        acc += m.pi[i];
        if (!found && u0 < acc) {
            found = true;
            mu = m.mu[i];
            k = m.kappa[i];
        }
    }
    float3 d = mine ? vmf_sample(mu, k, u1, u2) : f3(0.f, 0.f, 0.f);
    const int owner = (threadIdx.x & 15) | (first ? 0 : 16);
    return f3(__shfl_sync(0xFFFFFFFFu, d.x, owner), __shfl_sync(0xFFFFFFFFu, d.y, owner),
              __shfl_sync(0xFFFFFFFFu, d.z, owner));
}
SRT_DEV float half_pdf(const HalfMix& m, float3 w) {
    float q = 0.f;
#pragma unroll
    for (int i = 0; i < 4; ++i) q += m.pi[i] * vmf(m.mu[i], m.kappa[i], w);
    return q + __shfl_xor_sync(0xFFFFFFFFu, q, 16);
}

// Loads all layer weights (bf16, padded rows) and biases into shared memory.
// Every weight block starts on a 16-byte boundary (g_woff(l) is a multiple of 8).
SRT_DEV void load_weights(const GuideNet& net, __nv_bfloat16* sw, float* sb) {
    int off = 0;
    for (int l = 0; l < G_LAYERS; ++l) {
        copy_rows(sw + off, net.wbf + g_woff(l), g_out(l), g_in(l));
        off += g_out(l) * g_pad(g_in(l));
    }
    int bo = 0;
    for (int l = 0; l < G_LAYERS; ++l) {
        for (int i = threadIdx.x; i < g_out(l); i += blockDim.x) sb[bo + i] = net.master[g_boff(l) + i];
        bo += g_out(l);
    }
    cp_async_wait_all();
}
constexpr int SW_ELEMS = G_HID * g_pad(G_ENC) + 3 * G_HID * g_pad(G_HID) + G_OUT * g_pad(G_HID);
constexpr int SB_ELEMS = 4 * G_HID + G_OUT;
SRT_DEV const __nv_bfloat16* wl(const __nv_bfloat16* sw, int l) {
    int off = 0;
    for (int i = 0; i < l; ++i) off += g_out(i) * g_pad(g_in(i));
    return sw + off;
}
SRT_DEV const float* bl(const float* sb, int l) { return sb + l * G_HID; }

// Forward pass of the warp's 16 encoded samples (smem rows `in`) -> raw
// outputs in smem `out` [16][52].  With `act`, post-ReLU activations are also
// stored to smem (act[l] [16][72]).
SRT_DEV void forward16(const __nv_bfloat16* sw, const float* sb, const __nv_bfloat16* in, float* out,
                       __nv_bfloat16* act) {
    int t = threadIdx.x & 31;
    int g = t >> 2, cq = t & 3;
    float c[8][4];
    {
        uint32_t a0[8][4];
#pragma unroll
        for (int s = 0; s < 8; ++s) load_a(a0[s], in, g_pad(G_ENC), 16 * s);
        layer<G_ENC, G_HID>(a0, wl(sw, 0), bl(sb, 0), c);
    }
    uint32_t a[4][4];
#pragma unroll
    for (int l = 1; l < 4; ++l) {
        relu_to_a<G_HID>(c, a);
        if (act) {
            __nv_bfloat16* m = act + (l - 1) * 16 * g_pad(G_HID);
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                *reinterpret_cast<uint32_t*>(m + g * g_pad(G_HID) + 16 * s + 2 * cq) = a[s][0];
                *reinterpret_cast<uint32_t*>(m + (g + 8) * g_pad(G_HID) + 16 * s + 2 * cq) = a[s][1];
                *reinterpret_cast<uint32_t*>(m + g * g_pad(G_HID) + 16 * s + 8 + 2 * cq) = a[s][2];
                *reinterpret_cast<uint32_t*>(m + (g + 8) * g_pad(G_HID) + 16 * s + 8 + 2 * cq) = a[s][3];
            }
        }
        layer<G_HID, G_HID>(a, wl(sw, l), bl(sb, l), c);
    }
    relu_to_a<G_HID>(c, a);
    if (act) {
        __nv_bfloat16* m = act + 3 * 16 * g_pad(G_HID);
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            *reinterpret_cast<uint32_t*>(m + g * g_pad(G_HID) + 16 * s + 2 * cq) = a[s][0];
            *reinterpret_cast<uint32_t*>(m + (g + 8) * g_pad(G_HID) + 16 * s + 2 * cq) = a[s][1];
            *reinterpret_cast<uint32_t*>(m + g * g_pad(G_HID) + 16 * s + 8 + 2 * cq) = a[s][2];
            *reinterpret_cast<uint32_t*>(m + (g + 8) * g_pad(G_HID) + 16 * s + 8 + 2 * cq) = a[s][3];
        }
    }
    float o[6][4];
    layer<G_HID, G_OUT>(a, wl(sw, 4), bl(sb, 4), o);
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        out[g * 52 + 8 * j + 2 * cq] = o[j][0];
        out[g * 52 + 8 * j + 2 * cq + 1] = o[j][1];
        out[(g + 8) * 52 + 8 * j + 2 * cq] = o[j][2];
        out[(g + 8) * 52 + 8 * j + 2 * cq + 1] = o[j][3];
    }
}

// Network inputs of a vertex, each mapped to [0, 1].
SRT_DEV void vertex_inputs(float3 p, float3 n, float3 wo, float lambda, float4 bmin, float4 binv, float* x) {
    x[0] = (p.x - bmin.x) * binv.x;
    x[1] = (p.y - bmin.y) * binv.y;
    x[2] = (p.z - bmin.z) * binv.z;
    x[3] = n.x * 0.5f + 0.5f;
    x[4] = n.y * 0.5f + 0.5f;
    x[5] = n.z * 0.5f + 0.5f;
    x[6] = wo.x * 0.5f + 0.5f;
    x[7] = wo.y * 0.5f + 0.5f;
    x[8] = wo.z * 0.5f + 0.5f;
    x[9] = (lambda - LAMBDA_MIN) / LAMBDA_RANGE;
}

// Warp-aggregated counter updates from the lanes that execute the call
// together (one atomic per warp instead of one per lane; every guided vertex
// counts itself, so per-lane atomics on one address would queue in L2):
// agg_add adds the lanes' count, agg_slot also hands each lane its own slot.
SRT_DEV void agg_add(uint32_t* ctr) {
    const uint32_t m = __activemask();
    if ((threadIdx.x & 31u) == (uint32_t)(__ffs(m) - 1)) atomicAdd(ctr, (uint32_t)__popc(m));
}
SRT_DEV uint32_t agg_slot(uint32_t* ctr) {
    const uint32_t m = __activemask();
    const uint32_t lane = threadIdx.x & 31u;
    const int leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == (uint32_t)leader) base = atomicAdd(ctr, (uint32_t)__popc(m));
    base = __shfl_sync(m, base, leader);
    return base + (uint32_t)__popc(m & ((1u << lane) - 1u));
}

// Throughput, training record, Russian roulette and the next ray of guided
// vertex v (path id) once its direction is drawn; the direction's sampling
// pdf is sel q + (1 - sel) cos / pi.  Returns whether the path continues.
SRT_DEV bool finish_vertex(const FrameArgs& a, uint32_t bounce, uint32_t frame, uint32_t v, uint32_t id, float4 p,
                           float3 ffn, uint4 misc, uint32_t s, float3 dir, float sel, float q) {
    const GuideArgs& G = a.guide;
    const DevScene& S = a.scene;
    const float4 wo4 = G.gv.wo[v], spec = G.gv.spec[v];
    float4 thr = a.pb.thr[id];
    const float3 hp = xyz(p);
    float cosv = dot(ffn, dir);
    uint32_t rec = 0u;  // record index + 1 (0: none)
    bool alive = false;
    if (cosv > 0.0f) {
        float pb = cosv / PI;
        float pdf = sel * q + (1.0f - sel) * pb;
        float4 att = spec * (pb / pdf);  // (spec / pi) cos / pdf
        thr = thr * att;
        // training sample (a hashed subset of the vertices)
        if (G.train) {
            agg_add(&G.gc->candidates);
            uint32_t h = pcg_hash(id ^ (bounce << 24) ^ (frame * 0x9E3779B9u)) & 0xFFFFu;
            if (h < G.gc->threshold) {
                uint32_t r = agg_slot(&G.gc->records);
                if (r < G.batch) {
                    float x[G_IN];
                    vertex_inputs(hp, ffn, xyz(wo4), p.w, S.bmin, S.binv, x);
                    G.rec.x0[r] = f4(x[0], x[1], x[2], x[3]);
                    G.rec.x1[r] = f4(x[4], x[5], x[6], x[7]);
                    G.rec.x2[r] = f4(x[8], x[9], 0.f, 0.f);
                    G.rec.w[r] = f4(dir.x, dir.y, dir.z, pdf);
                    float fcos = (spec.x + spec.y + spec.z + spec.w) * 0.25f * pb;
                    G.rec.b[r] = f4(pb, fcos, 0.f, 0.f);
                    G.rec.thr[r] = thr;
                    G.rec.rad[r] = splat4(__int_as_float(0x7FC00000));  // NaN: not reached yet
                    G.rec.pid[r] = id;
                    rec = r + 1u;
                }
            }
        }
        alive = true;
        if (bounce > 3u) {
            float pr = max4(thr);
            if (rng_next(s) > pr) alive = false;
            else thr = thr / pr;
        }
        if (bounce + 1u >= a.max_depth) alive = false;
    }
    if (alive) {
        a.pb.thr[id] = thr;
        a.pb.ray_o[id] = f4(hp.x, hp.y, hp.z, 0.0001f);
        a.pb.ray_d[id] = f4(dir.x, dir.y, dir.z, 100.0f);
    }
    a.pb.misc[id] = make_uint4(s, misc.y, misc.z, rec);
    return alive;
}

}  // namespace

// ---------------------------------------------------------------- inference
// The continuation of every Lambert vertex of this bounce (the tail of
// shader.wgsl:677-700 for material 0): mixture sampling, throughput,
// Russian roulette, next queue; plus the recording of training samples.
__global__ void __launch_bounds__(GWI * 32, 2) k_guide_infer(FrameArgs a, uint32_t bounce) {
    const GuideArgs& G = a.guide;
    extern __shared__ __align__(1024) unsigned char smem[];
    __nv_bfloat16* sw = reinterpret_cast<__nv_bfloat16*>(smem);
    float* sb = reinterpret_cast<float*>(sw + SW_ELEMS);
    unsigned char* wbase = reinterpret_cast<unsigned char*>(sb + SB_ELEMS);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __nv_bfloat16* in = reinterpret_cast<__nv_bfloat16*>(wbase + warp * IN_BYTES);
    float* out = reinterpret_cast<float*>(in);
    const uint32_t n = G.gc->verts[bounce];
    if (blockIdx.x * GWI * 16 >= n) return;
    load_weights(G.net, sw, sb);
    __syncthreads();
    const DevScene& S = a.scene;
    const uint32_t frame = a.cam->frame_count;
    for (uint32_t base = (blockIdx.x * GWI + warp) * 16; base < n; base += gridDim.x * GWI * 16) {
        // encode: two lanes per sample
        {
            uint32_t v = base + (lane & 15);
            float x[G_IN];
            if (v < n) {
                float4 p = G.gv.p[v], nn = G.gv.n[v], wo = G.gv.wo[v];
                vertex_inputs(xyz(p), xyz(nn), xyz(wo), p.w, S.bmin, S.binv, x);
            } else {
                for (int i = 0; i < G_IN; ++i) x[i] = 0.f;
            }
            encode_half(x, lane >> 4, in + (lane & 15) * g_pad(G_ENC));
        }
        __syncwarp();
        forward16(sw, sb, in, out, nullptr);
        __syncwarp();
        // mixture sampling: lanes l and l + 16 share sample l & 15, four lobes each
        const int sl = lane & 15, half = lane >> 4;
        const uint32_t v = base + sl;
        const bool valid = v < n;
        HalfMix m;
        half_mixture(out + sl * 52, half, m);
        uint32_t id = 0, s = 0;
        float4 p = splat4(0.f), nn = splat4(0.f);
        uint4 misc = make_uint4(0, 0, 0, 0);
        if (valid) {
            id = G.gv.id[v];
            p = G.gv.p[v];
            nn = G.gv.n[v];
            misc = a.pb.misc[id];
            s = misc.x;
        }
        const float3 ffn = xyz(nn);
        // both lanes of a pair replay the same random stream
        const bool use_guide = valid && rng_next(s) < m.sel;
        float u0 = 0.f, u1 = 0.f, u2 = 0.f;
        float3 dir = ffn;
        if (use_guide) {
            u0 = rng_next(s);
            u1 = rng_next(s);
            u2 = rng_next(s);
        } else if (valid) {
            float3 d = ffn + random_unit_vector(s);  // shader.wgsl:462-466
            if (length(d) < 0.001f) d = ffn;
            dir = normalize(d);
        }
        const float3 gdir = half_sample(m, half, u0, u1, u2);
        if (use_guide) dir = gdir;
        const float q = half_pdf(m, dir);
        bool alive = false;
        if (valid && half == 0) alive = finish_vertex(a, bounce, frame, v, id, p, ffn, misc, s, dir, m.sel, q);
        // push the survivors into the next bounce's queue
        uint32_t mask = __ballot_sync(0xFFFFFFFFu, alive);
        uint32_t slot_base = 0;
        if (mask) {
            int leader = __ffs(mask) - 1;
            if (lane == leader) slot_base = atomicAdd(&a.counters->paths[bounce + 1], (uint32_t)__popc(mask));
            slot_base = __shfl_sync(0xFFFFFFFFu, slot_base, leader);
        }
        if (alive) a.pb.queue[(bounce + 1) & 1][slot_base + __popc(mask & ((1u << lane) - 1u))] = id;
        __syncwarp();
    }
}

// ---------------------------------------------------------------- training
// Per record: the radiance that arrived along the sampled direction and the
// training weight F / p = L f cos / p.  Records whose path ended before its
// next vertex carry no later radiance (L = 0).
// The records of training step `step` (of G.steps this frame): records
// step, step + steps, step + 2 steps, ...  Records are stored in the order
// their vertices were shaded (by bounce, then roughly by pixel), so strided
// sub-batches each sample the whole frame.
struct StepRecs {
    uint32_t count, first, stride;
};
SRT_DEV StepRecs step_recs(const GuideArgs& G, int step) {
    const uint32_t n = min(G.gc->records, G.batch);
    const uint32_t k = max(G.steps, 1u), f = (uint32_t)step;
    return StepRecs{n > f ? (n - f + k - 1u) / k : 0u, f, k};
}
SRT_DEV uint32_t rec_at(const StepRecs& sr, uint32_t j) { return sr.first + j * sr.stride; }

SRT_DEV void guide_targets(const FrameArgs& a) {
    const GuideArgs& G = a.guide;
    if (!G.train) return;
    uint32_t n = min(G.gc->records, G.batch);
    float local = 0.f;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        float4 fin = a.pb.rad[G.rec.pid[r]];
        float4 nx = G.rec.rad[r];
        if (nx.x != nx.x) nx = fin;
        float4 t = G.rec.thr[r];
        float L = 0.f;
        L += t.x > 0.f ? (fin.x - nx.x) / t.x : 0.f;
        L += t.y > 0.f ? (fin.y - nx.y) / t.y : 0.f;
        L += t.z > 0.f ? (fin.z - nx.z) / t.z : 0.f;
        L += t.w > 0.f ? (fin.w - nx.w) / t.w : 0.f;
        L = fmaxf(L * 0.25f, 0.f);
        float4 w = G.rec.w[r], b = G.rec.b[r];
        float wt = L * b.y / fmaxf(w.w, 1e-20f);
        if (!(wt < 3.4e38f)) wt = 0.f;
        G.rec.weight[r] = wt;
        local += wt;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xFFFFFFFFu, local, o);
    if ((threadIdx.x & 31) == 0 && local != 0.f) atomicAdd(&G.gc->weight_sum, local);
}
__global__ void k_guide_targets(FrameArgs a) { guide_targets(a); }
// many renderers: blockIdx.y = item
__global__ void k_guide_targets_multi(const FrameArgs* __restrict__ items) { guide_targets(items[blockIdx.y]); }

// Gradient of the loss of one record with respect to the 48 raw outputs
// (gr[41..47] are untouched): -w log q(omega) for the lobes and
// -w log(sel q + (1 - sel) p_bsdf) for the selection output with q held
// fixed.  w4 = sampled direction, b4.x = BSDF pdf, wt = normalised weight.
SRT_DEV void loss_grad(const float* raw, float4 w4, float4 b4, float wt, float* gr) {
    Mix m;
    mixture_fast(raw, m);
    float3 om = xyz(w4);
    float vm[G_LOBES], q = 0.f;
    for (int j = 0; j < G_LOBES; ++j) {
        vm[j] = m.c[j] * __expf(m.kappa[j] * (dot(m.mu[j], om) - 1.0f));
        q += m.pi[j] * vm[j];
    }
    q = fmaxf(q, 1e-30f);
    const float iq = 1.0f / q;
    for (int j = 0; j < G_LOBES; ++j) {
        float gam = m.pi[j] * vm[j] * iq;
        gr[5 * j + 4] = wt * (m.pi[j] - gam);
        float k = m.kappa[j];
        float mw = dot(m.mu[j], om);
        float dl = 1.0f / k - 2.0f / expm1f(2.0f * k) + mw - 1.0f;
        bool inside = m.lk[j] > G_KAPPA_LO && m.lk[j] < G_KAPPA_HI;
        gr[5 * j + 3] = inside ? -wt * gam * dl * k : 0.f;
        float3 gd = (om - m.mu[j] * mw) * __fdividef(-wt * gam * k, m.norm[j]);
        gr[5 * j] = gd.x;
        gr[5 * j + 1] = gd.y;
        gr[5 * j + 2] = gd.z;
    }
    float pb = b4.x;
    float pmix = fmaxf(m.sel * q + (1.0f - m.sel) * pb, 1e-30f);
    gr[40] = __fdividef(-wt * (q - pb), pmix) * G_SEL_SPAN * m.sel_sig * (1.0f - m.sel_sig);
}

// Forward + backward of 16 records per warp: stores the encoded inputs,
// post-ReLU activations and per-layer deltas (bf16) for the weight-gradient
// product.  Loss per sample (weight w normalised by the batch mean):
//   -w log q(omega) for the lobes, -w log(sel q + (1 - sel) p_bsdf) for sel.
SRT_DEV void guide_fwdbwd(const GuideArgs& G, int step) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __nv_bfloat16* sw = reinterpret_cast<__nv_bfloat16*>(smem);
    float* sb = reinterpret_cast<float*>(sw + SW_ELEMS);
    unsigned char* wbase = reinterpret_cast<unsigned char*>(sb + SB_ELEMS);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int per_warp = 16 * g_pad(G_ENC) * 2 + 4 * 16 * g_pad(G_HID) * 2 + 16 * 52 * 4 + 16 * g_pad(G_OUT) * 2;
    __nv_bfloat16* in = reinterpret_cast<__nv_bfloat16*>(wbase + warp * per_warp);
    __nv_bfloat16* act = in + 16 * g_pad(G_ENC);
    float* out = reinterpret_cast<float*>(act + 4 * 16 * g_pad(G_HID));
    __nv_bfloat16* d4 = reinterpret_cast<__nv_bfloat16*>(out + 16 * 52);
    const uint32_t n_all = min(G.gc->records, G.batch);
    const StepRecs sr = step_recs(G, step);
    const uint32_t n = sr.count;  // this step's records, by index j (record rec_at(sr, j))
    if (blockIdx.x * GWT * 16 >= n) return;
    load_weights(G.net, sw, sb);
    __syncthreads();
    const float inv_mean = G.gc->weight_sum > 0.f ? (float)n_all / G.gc->weight_sum : 0.f;
    const int g = lane >> 2, cq = lane & 3;
    for (uint32_t base = (blockIdx.x * GWT + warp) * 16; base < n; base += gridDim.x * GWT * 16) {
        {
            const uint32_t j = base + (lane & 15), r = rec_at(sr, j);
            float x[G_IN];
            if (j < n) {
                float4 x0 = G.rec.x0[r], x1 = G.rec.x1[r], x2 = G.rec.x2[r];
                x[0] = x0.x; x[1] = x0.y; x[2] = x0.z; x[3] = x0.w;
                x[4] = x1.x; x[5] = x1.y; x[6] = x1.z; x[7] = x1.w;
                x[8] = x2.x; x[9] = x2.y;
            } else {
                for (int i = 0; i < G_IN; ++i) x[i] = 0.f;
            }
            encode_half(x, lane >> 4, in + (lane & 15) * g_pad(G_ENC));
        }
        __syncwarp();
        forward16(sw, sb, in, out, act);
        __syncwarp();
        // output gradient, one lane per sample
        if (lane < 16) {
            const uint32_t j = base + lane, r = rec_at(sr, j);
            float gr[G_OUT];
            for (int i = 0; i < G_OUT; ++i) gr[i] = 0.f;
            if (j < n) loss_grad(out + lane * 52, G.rec.w[r], G.rec.b[r], G.rec.weight[r] * inv_mean, gr);
            for (int i = 0; i < G_OUT; i += 2)
                *reinterpret_cast<uint32_t*>(d4 + lane * g_pad(G_OUT) + i) = pack2(gr[i], gr[i + 1]);
        }
        __syncwarp();
        // store inputs, activations and the output delta for the weight gradients
        for (int e = lane; e < 16 * (G_ACT_STRIDE / 8); e += 32) {
            int row = e / (G_ACT_STRIDE / 8), ch = e % (G_ACT_STRIDE / 8);
            if (base + row >= n) continue;
            const uint32_t r = rec_at(sr, base + row);
            const __nv_bfloat16* src = ch < 16 ? in + row * g_pad(G_ENC) + 8 * ch
                                               : act + ((ch - 16) / 8) * 16 * g_pad(G_HID) + row * g_pad(G_HID) +
                                                     8 * ((ch - 16) % 8);
            *reinterpret_cast<uint4*>(G.rec.act + (size_t)r * G_ACT_STRIDE + 8 * ch) =
                *reinterpret_cast<const uint4*>(src);
        }
        for (int e = lane; e < 16 * (G_OUT / 8); e += 32) {
            int row = e / (G_OUT / 8), ch = e % (G_OUT / 8);
            if (base + row >= n) continue;
            const uint32_t r = rec_at(sr, base + row);
            *reinterpret_cast<uint4*>(G.rec.delta + (size_t)r * G_DELTA_STRIDE + g_delta_off(4) + 8 * ch) =
                *reinterpret_cast<const uint4*>(d4 + row * g_pad(G_OUT) + 8 * ch);
        }
        // backward: delta_l = (delta_{l+1} W_{l+1}) * relu'(a_l), l = 3..0
        uint32_t da[4][4];  // A fragments of the current delta (K up to 64)
#pragma unroll
        for (int s = 0; s < 3; ++s) load_a(da[s], d4, g_pad(G_OUT), 16 * s);
#pragma unroll
        for (int l = 3; l >= 0; --l) {
            const int K = l == 3 ? G_OUT : G_HID;
            float c[8][4];
#pragma unroll
            for (int j = 0; j < 8; ++j) c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.f;
            const __nv_bfloat16* W = wl(sw, l + 1);  // [out = K][in = 64]: B[k][n] = W[k][n]
#pragma unroll
            for (int s = 0; s < K / 16; ++s) {
#pragma unroll
                for (int j = 0; j < 8; j += 2) {
                    uint32_t b[4];
                    load_b2t(b, W, g_pad(G_HID), 8 * j, 16 * s);
                    mma16816(c[j], da[s], b[0], b[1]);
                    mma16816(c[j + 1], da[s], b[2], b[3]);
                }
            }
            // relu' mask from the stored activation a_l
            const __nv_bfloat16* am = act + l * 16 * g_pad(G_HID);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                float2 lo = unpack2(*reinterpret_cast<const uint32_t*>(am + g * g_pad(G_HID) + 8 * j + 2 * cq));
                float2 hi = unpack2(*reinterpret_cast<const uint32_t*>(am + (g + 8) * g_pad(G_HID) + 8 * j + 2 * cq));
                c[j][0] = lo.x > 0.f ? c[j][0] : 0.f;
                c[j][1] = lo.y > 0.f ? c[j][1] : 0.f;
                c[j][2] = hi.x > 0.f ? c[j][2] : 0.f;
                c[j][3] = hi.y > 0.f ? c[j][3] : 0.f;
            }
            // to A fragments (no ReLU: already masked) and to global memory
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                da[s][0] = pack2(c[2 * s][0], c[2 * s][1]);
                da[s][1] = pack2(c[2 * s][2], c[2 * s][3]);
                da[s][2] = pack2(c[2 * s + 1][0], c[2 * s + 1][1]);
                da[s][3] = pack2(c[2 * s + 1][2], c[2 * s + 1][3]);
            }
            const bool ok0 = base + g < n, ok1 = base + g + 8 < n;
            const uint32_t r0 = rec_at(sr, base + g), r1 = rec_at(sr, base + g + 8);
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                __nv_bfloat16* d0 = G.rec.delta + g_delta_off(l) + 16 * s + 2 * cq;
                if (ok0) {
                    *reinterpret_cast<uint32_t*>(d0 + (size_t)r0 * G_DELTA_STRIDE) = da[s][0];
                    *reinterpret_cast<uint32_t*>(d0 + (size_t)r0 * G_DELTA_STRIDE + 8) = da[s][2];
                }
                if (ok1) {
                    *reinterpret_cast<uint32_t*>(d0 + (size_t)r1 * G_DELTA_STRIDE) = da[s][1];
                    *reinterpret_cast<uint32_t*>(d0 + (size_t)r1 * G_DELTA_STRIDE + 8) = da[s][3];
                }
            }
        }
        __syncwarp();
    }
}
__global__ void __launch_bounds__(GWT * 32) k_guide_fwdbwd(GuideArgs G, int step) { guide_fwdbwd(G, step); }
// many renderers (blockIdx.y = item), those that train and take this step
__global__ void __launch_bounds__(GWT * 32) k_guide_fwdbwd_multi(const FrameArgs* __restrict__ items, int step) {
    const GuideArgs& G = items[blockIdx.y].guide;
    if (G.train && (uint32_t)step < G.steps) guide_fwdbwd(G, step);
}

// Weight gradients dW_l = sum_s delta_l[s]^T a_{l-1}[s] (and bias sums),
// split over the samples; job (blockIdx.y): 0, 1 = layer 0 input halves,
// 2..5 = layers 1..4.  8 warps: warp w owns output rows 16 (w & 3) .. + 15
// and input columns 32 (w >> 2) .. + 31 of the 64 x 64 block.
constexpr int WGRAD_BLOCKS = 64;  // sample splits per job
SRT_DEV void guide_wgrad(const GuideArgs& G, int step) {
    __shared__ __align__(16) __nv_bfloat16 sd[32 * g_pad(G_HID)];
    __shared__ __align__(16) __nv_bfloat16 sa[32 * g_pad(G_HID)];
    const StepRecs sr = step_recs(G, step);
    const uint32_t n = sr.count;
    const int job = blockIdx.y;
    const int l = job <= 1 ? 0 : job - 1;
    const int in0 = job == 1 ? 64 : 0;
    const int nout = g_out(l), nin = g_in(l);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mt = warp & 3, nh = warp >> 2;
    const bool active_rows = 16 * mt < nout;
    float c[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.f;
    float bsum = 0.f;
    const uint32_t chunk = 32;
    uint32_t per = (((n + gridDim.x - 1) / gridDim.x) + chunk - 1) / chunk * chunk;
    uint32_t s0 = blockIdx.x * per, s1 = min(n, s0 + per);
    for (uint32_t s = s0; s < s1; s += chunk) {
        // stage 32 samples: deltas (out columns) and activations (input columns)
        {
            int row = threadIdx.x >> 3, ch = threadIdx.x & 7;
            const uint32_t r = rec_at(sr, s + row);
            uint4 dv = make_uint4(0, 0, 0, 0), av = make_uint4(0, 0, 0, 0);
            if (s + row < s1) {
                if (8 * ch < nout)
                    dv = *reinterpret_cast<const uint4*>(G.rec.delta + (size_t)r * G_DELTA_STRIDE + g_delta_off(l) + 8 * ch);
                av = *reinterpret_cast<const uint4*>(G.rec.act + (size_t)r * G_ACT_STRIDE + g_act_off(l - 1) + in0 + 8 * ch);
            }
            *reinterpret_cast<uint4*>(sd + row * g_pad(G_HID) + 8 * ch) = dv;
            *reinterpret_cast<uint4*>(sa + row * g_pad(G_HID) + 8 * ch) = av;
        }
        __syncthreads();
        if (job != 1 && threadIdx.x < nout) {
            for (int row = 0; row < 32; ++row) bsum += __bfloat162float(sd[row * g_pad(G_HID) + threadIdx.x]);
        }
        if (active_rows) {
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
                uint32_t af[4];
                {
                    // A = delta^T: rows = outputs 16 mt.., k = samples 16 ks..
                    const __nv_bfloat16* p =
                        sd + (16 * ks + (lane & 7) + 8 * (lane >> 4)) * g_pad(G_HID) + 16 * mt + 8 * ((lane >> 3) & 1);
                    ldsm4t(af, p);
                }
#pragma unroll
                for (int jp = 0; jp < 2; ++jp) {
                    uint32_t bf[4];
                    // B = activations: k = samples 16 ks.., n = inputs 32 nh + 16 jp ..
                    const __nv_bfloat16* p = sa + (16 * ks + (lane & 7) + 8 * ((lane >> 3) & 1)) * g_pad(G_HID) +
                                             32 * nh + 16 * jp + 8 * (lane >> 4);
                    ldsm4t(bf, p);
                    mma16816(c[2 * jp], af, bf[0], bf[1]);
                    mma16816(c[2 * jp + 1], af, bf[2], bf[3]);
                }
            }
        }
        __syncthreads();
    }
    if (s0 >= s1) return;
    if (active_rows) {
        const int g = lane >> 2, cq = lane & 3;
        float* gw = G.net.grad + g_woff(l);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            int col = in0 + 32 * nh + 8 * j + 2 * cq;
            int r0 = 16 * mt + g, r1 = r0 + 8;
            atomicAdd(gw + r0 * nin + col, c[j][0]);
            atomicAdd(gw + r0 * nin + col + 1, c[j][1]);
            atomicAdd(gw + r1 * nin + col, c[j][2]);
            atomicAdd(gw + r1 * nin + col + 1, c[j][3]);
        }
    }
    if (job != 1 && threadIdx.x < nout && bsum != 0.f) atomicAdd(G.net.grad + g_boff(l) + threadIdx.x, bsum);
}
__global__ void __launch_bounds__(256) k_guide_wgrad(GuideArgs G, int step) { guide_wgrad(G, step); }
// many renderers: blockIdx.z = item
__global__ void __launch_bounds__(256) k_guide_wgrad_multi(const FrameArgs* __restrict__ items, int step) {
    const GuideArgs& G = items[blockIdx.z].guide;
    if (G.train && (uint32_t)step < G.steps) guide_wgrad(G, step);
}

// Adam on the FP32 master weights (gradients are sums over the batch and
// are divided by its size), then the bf16 copies; clears the gradients.
SRT_DEV void guide_adam(const GuideArgs& G, int step) {
    const uint32_t n = step_recs(G, step).count;
    if (n == 0) return;
    const float inv = 1.0f / (float)n;
    const float t = (float)(G.gc->adam_step + 1u + (uint32_t)step);
    const float b1t = 1.0f - powf(0.9f, t), b2t = 1.0f - powf(0.999f, t);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < G_NPARAMS; i += gridDim.x * blockDim.x) {
        float gr = G.net.grad[i] * inv;
        G.net.grad[i] = 0.f;
        float m = 0.9f * G.net.adam_m[i] + 0.1f * gr;
        float v = 0.999f * G.net.adam_v[i] + 0.001f * gr * gr;
        G.net.adam_m[i] = m;
        G.net.adam_v[i] = v;
        float w = G.net.master[i] - G.lr * (m / b1t) / (sqrtf(v / b2t) + 1e-8f);
        G.net.master[i] = w;
        int l = 0;
        while (l < 4 && i >= g_woff(l + 1)) ++l;
        if (i - g_woff(l) < g_in(l) * g_out(l)) G.net.wbf[i] = __float2bfloat16_rn(w);
    }
}
__global__ void k_guide_adam(GuideArgs G, int step) { guide_adam(G, step); }
// many renderers: blockIdx.y = item
__global__ void k_guide_adam_multi(const FrameArgs* __restrict__ items, int step) {
    const GuideArgs& G = items[blockIdx.y].guide;
    if (G.train && (uint32_t)step < G.steps) guide_adam(G, step);
}

// Next frame's recording threshold (of 65536) so that about 90 % of the
// training batch fills; counts the Adam step; clears the per-frame counters.
SRT_DEV void guide_frame_end(const GuideArgs& G, int trained) {
    GuideCounters* gc = G.gc;
    if (threadIdx.x < 32) gc->verts[threadIdx.x] = 0u;
    if (threadIdx.x != 0) return;
    uint32_t c = gc->candidates;
    if (c > 0) {
        double t = 65536.0 * 0.9 * (double)G.batch / (double)c;
        gc->threshold = (uint32_t)fmin(65536.0, fmax(1.0, t));
    }
    if (trained && gc->records > 0u) gc->adam_step += max(G.steps, 1u);
    gc->records = 0u;
    gc->candidates = 0u;
    gc->weight_sum = 0.f;
}
__global__ void k_guide_frame_end(GuideArgs G, int trained) { guide_frame_end(G, trained); }
// many renderers: one block per item
__global__ void k_guide_frame_end_multi(const FrameArgs* __restrict__ items) {
    const GuideArgs& G = items[blockIdx.x].guide;
    guide_frame_end(G, G.train);
}

// ---------------------------------------------------------------- test kernels
// Forward pass of n samples (inputs [n][10]) -> raw outputs [n][48].
__global__ void __launch_bounds__(GWI * 32, 2) k_guide_test_forward(GuideNet net, const float* __restrict__ x,
                                                                    uint32_t n, float* __restrict__ y) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __nv_bfloat16* sw = reinterpret_cast<__nv_bfloat16*>(smem);
    float* sb = reinterpret_cast<float*>(sw + SW_ELEMS);
    unsigned char* wbase = reinterpret_cast<unsigned char*>(sb + SB_ELEMS);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __nv_bfloat16* in = reinterpret_cast<__nv_bfloat16*>(wbase + warp * IN_BYTES);
    float* out = reinterpret_cast<float*>(in);
    load_weights(net, sw, sb);
    __syncthreads();
    for (uint32_t base = (blockIdx.x * GWI + warp) * 16; base < n; base += gridDim.x * GWI * 16) {
        uint32_t r = base + (lane & 15);
        float xi[G_IN];
        for (int i = 0; i < G_IN; ++i) xi[i] = r < n ? x[(size_t)r * G_IN + i] : 0.f;
        encode_half(xi, lane >> 4, in + (lane & 15) * g_pad(G_ENC));
        __syncwarp();
        forward16(sw, sb, in, out, nullptr);
        __syncwarp();
        if (lane < 16 && base + lane < n)
            for (int i = 0; i < G_OUT; ++i) y[(size_t)(base + lane) * G_OUT + i] = out[lane * 52 + i];
        __syncwarp();
    }
}

// Mixture pdf and samples from raw outputs: out[i] = (pdf(omega_i), sample
// xyz), evaluated by lane pairs exactly as in k_guide_infer.
__global__ void k_guide_test_mixture(const float* __restrict__ raw, const float* __restrict__ omega,
                                     const float* __restrict__ u, uint32_t n, float* __restrict__ out) {
    const int lane = threadIdx.x & 31, half = lane >> 4;
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) / 32 * 16 + (lane & 15);
    const bool valid = i < n;
    float r[G_OUT];
    for (int k = 0; k < G_OUT; ++k) r[k] = valid ? raw[(size_t)i * G_OUT + k] : 0.f;
    HalfMix m;
    half_mixture(r, half, m);
    float3 w = valid ? f3(omega[3 * i], omega[3 * i + 1], omega[3 * i + 2]) : f3(0.f, 0.f, 1.f);
    const float pdf = half_pdf(m, w);
    const float3 d = valid ? half_sample(m, half, u[3 * i], u[3 * i + 1], u[3 * i + 2])
                           : half_sample(m, half, 0.f, 0.5f, 0.5f);
    if (valid && half == 0) {
        out[4 * i] = pdf;
        out[4 * i + 1] = d.x;
        out[4 * i + 2] = d.y;
        out[4 * i + 3] = d.z;
    }
}

// ---------------------------------------------------------------- tcgen05 inference
// The same network on the fifth-generation tensor cores.  A block runs two
// independent groups of 128 threads (warps 0-3 and 4-7); a group owns 128
// vertices (M = 128 rows).  The encoded rows and each hidden layer's
// activations live in the group's shared-memory A buffer in the K-major
// core-matrix layout (umma.cuh), the weights (shared by both groups) as the
// B operands (N = 64, or 48 for the output layer), and every layer is K / 16
// tcgen05.mma instructions issued by one thread of the group into the
// group's 128 x 64 FP32 accumulator in tensor memory.  Thread t reads row t
// back (tcgen05.ld), adds the bias, applies ReLU and writes the bf16 row of
// the next layer's A operand; after the output layer it holds its vertex's
// 48 raw outputs in registers and samples its mixture alone.  While one
// group waits for its MMAs the other runs its epilogue or mixture code.
namespace {

constexpr int TC_ROWS = 128;
constexpr int TC_GROUPS = 2;
constexpr uint32_t TC_TMEM_COLS = 64 * TC_GROUPS;
constexpr uint32_t TC_WAIT_POLLS = 1u << 22;
__host__ __device__ constexpr uint32_t tc_woff(int l) { return l == 0 ? 0u : 16384u + 8192u * (uint32_t)(l - 1); }
constexpr uint32_t TC_A_BYTES = TC_ROWS * G_ENC * 2;
__host__ __device__ constexpr uint32_t tc_aoff(int g) { return 47104u + TC_A_BYTES * (uint32_t)g; }
constexpr uint32_t TC_B_OFF = tc_aoff(TC_GROUPS);
constexpr uint32_t TC_BAR_OFF = TC_B_OFF + SB_ELEMS * 4;  // one mbarrier per group, then the TMEM base
constexpr uint32_t TC_SMEM = TC_BAR_OFF + 8 * TC_GROUPS + 16;
static_assert(tc_woff(4) + G_OUT * G_HID * 2 == tc_aoff(0), "tcgen05 weight layout");
static_assert(tc_aoff(0) % 128 == 0 && TC_B_OFF % 16 == 0 && TC_BAR_OFF % 8 == 0, "tcgen05 shared-memory alignment");
static_assert(2 * (TC_SMEM + 1024) <= 228 * 1024, "two blocks per SM");
// the grouped kernel: rows per chunk, and its chunk table after the single-renderer layout
constexpr uint32_t TC_CHUNK = TC_ROWS * TC_GROUPS;
constexpr uint32_t TC_SMEM_MULTI = TC_SMEM + 4 * (MAX_BATCH + 1) + 8;
static_assert(TC_SMEM % 4 == 0 && 2 * (TC_SMEM_MULTI + 1024) <= 228 * 1024, "grouped kernel: two blocks per SM");

// Barrier of one 128-thread group (ids 1 and 2; 0 is the block barrier).
SRT_DEV void group_sync(uint32_t id) { asm volatile("bar.sync %0, 128;\n" ::"r"(id) : "memory"); }
// AND of `pred` over the group, also a barrier.
SRT_DEV bool group_and(uint32_t id, bool pred) {
    uint32_t r;
    asm volatile(
        "{\n"
        ".reg .pred p, q;\n"
        "setp.ne.u32 q, %1, 0;\n"
        "bar.red.and.pred p, %2, 128, q;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(id)
        : "memory");
    return r != 0u;
}

// Weights of all layers into the core-matrix layout (cp.async) and biases.
SRT_DEV void load_weights_tc(const GuideNet& net, unsigned char* smem, float* sb) {
    for (int l = 0; l < G_LAYERS; ++l) {
        const int K = g_in(l), N = g_out(l), cpr = K / 8;
        for (int i = threadIdx.x; i < N * cpr; i += blockDim.x) {
            const int n = i / cpr, kc = i - n * cpr;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(
                             smem_u32(smem + tc_woff(l) + umma_offset((uint32_t)n, 8u * kc, (uint32_t)K))),
                         "l"(net.wbf + g_woff(l) + n * K + 8 * kc));
        }
    }
    int bo = 0;
    for (int l = 0; l < G_LAYERS; ++l) {
        for (int i = threadIdx.x; i < g_out(l); i += blockDim.x) sb[bo + i] = net.master[g_boff(l) + i];
        bo += g_out(l);
    }
    cp_async_wait_all();
    fence_async_smem();  // the tensor core reads them through the async proxy
}

// Row `row` of the A operand (K = 128): the frequency encoding of x, with the
// octave recurrence of encode_half.
SRT_DEV void encode_row_tc(const float* x, unsigned char* A, uint32_t row) {
    uint32_t pk[G_ENC / 2];
#pragma unroll
    for (int d = 0; d < G_IN; ++d) {
        float s, c;
        sincospif(x[d], &s, &c);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            pk[6 * d + k] = pack2(s, c);  // features 12 d + 2 k (sin), + 1 (cos)
            float s2 = __fmul_rn(__fmul_rn(2.0f, s), c);
            float c2 = __fmaf_rn(c, c, -__fmul_rn(s, s));
            s = s2;
            c = c2;
        }
    }
#pragma unroll
    for (int i = 60; i < 64; ++i) pk[i] = 0u;
#pragma unroll
    for (int ch = 0; ch < G_ENC / 8; ++ch)
        *reinterpret_cast<uint4*>(A + umma_offset(row, 8u * ch, G_ENC)) =
            make_uint4(pk[4 * ch], pk[4 * ch + 1], pk[4 * ch + 2], pk[4 * ch + 3]);
}

// Bias + ReLU of 16 accumulator columns into 8 packed bf16 pairs.
SRT_DEV void relu_pack16(const uint32_t (&r)[16], const float* bias, uint32_t* out) {
#pragma unroll
    for (int i = 0; i < 8; ++i)
        out[i] = pack2_relu(__uint_as_float(r[2 * i]) + bias[2 * i], __uint_as_float(r[2 * i + 1]) + bias[2 * i + 1]);
}

// A group of 128 threads: its A buffer, accumulator columns, mbarrier and
// barrier id; `row` = the thread's row (and TMEM lane).
struct TcGroup {
    unsigned char* A;
    uint32_t tmem;  // lane 0, the group's first column
    uint64_t* mbar;
    uint32_t bar;
    uint32_t row;
};

// The five layers for the group's 128 rows (A holds the encoded rows, made
// visible to the async proxy by the caller's fence + group barrier).  On
// return `out` holds this thread's raw outputs.  False (for every thread of
// the group) when a layer's MMAs did not complete within the wait limit;
// `phase` then still names the phase that did not complete.
SRT_DEV bool mlp_tc(const TcGroup& g, const unsigned char* smem, const float* sb, uint32_t& phase,
                    float (&out)[G_OUT]) {
    const uint32_t a_addr = smem_u32(g.A), w_addr = smem_u32(smem);
    const uint32_t taddr = g.tmem + (((g.row >> 5) * 32u) << 16);
#pragma unroll
    for (int l = 0; l < G_LAYERS; ++l) {
        const uint32_t K = (uint32_t)g_in(l), N = (uint32_t)g_out(l), SBO = K / 8u * 128u;
        if (g.row == 0) {
            tc_fence_after();
            for (uint32_t s = 0; s < K / 16u; ++s)
                umma_bf16(g.tmem, umma_desc(a_addr + 256u * s, 128u, SBO),
                          umma_desc(w_addr + tc_woff(l) + 256u * s, 128u, SBO), umma_idesc_bf16(TC_ROWS, N), s);
            umma_commit(g.mbar);
        }
        if (!group_and(g.bar, mbar_wait(g.mbar, phase, TC_WAIT_POLLS))) return false;
        phase ^= 1u;
        tc_fence_after();
        const float* bias = sb + G_HID * l;
        uint32_t r0[16], r1[16], r2[16];
        tmem_ld16(taddr, r0);
        tmem_ld16(taddr + 16u, r1);
        tmem_ld16(taddr + 32u, r2);
        if (l < G_LAYERS - 1) {
            uint32_t r3[16];
            tmem_ld16(taddr + 48u, r3);
            tmem_wait16(r0);
            tmem_wait16(r1);
            tmem_wait16(r2);
            tmem_wait16(r3);
            uint32_t pk[32];
            relu_pack16(r0, bias, pk);
            relu_pack16(r1, bias + 16, pk + 8);
            relu_pack16(r2, bias + 32, pk + 16);
            relu_pack16(r3, bias + 48, pk + 24);
#pragma unroll
            for (int ch = 0; ch < G_HID / 8; ++ch)
                *reinterpret_cast<uint4*>(g.A + umma_offset(g.row, 8u * ch, G_HID)) =
                    make_uint4(pk[4 * ch], pk[4 * ch + 1], pk[4 * ch + 2], pk[4 * ch + 3]);
            fence_async_smem();
        } else {
            tmem_wait16(r0);
            tmem_wait16(r1);
            tmem_wait16(r2);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                out[i] = __uint_as_float(r0[i]) + bias[i];
                out[16 + i] = __uint_as_float(r1[i]) + bias[16 + i];
                out[32 + i] = __uint_as_float(r2[i]) + bias[32 + i];
            }
        }
        tc_fence_before();
        group_sync(g.bar);
    }
    return true;
}

SRT_DEV float mix_pdf(const Mix& m, float3 w) {
    float q = 0.f;
#pragma unroll
    for (int j = 0; j < G_LOBES; ++j) q += m.pi[j] * (m.c[j] * __expf(m.kappa[j] * (dot(m.mu[j], w) - 1.0f)));
    return q;
}
// Lobe j = first with u0 below the cumulative weight (the last lobe on
// rounding), then a vMF direction from (u1, u2).
SRT_DEV float3 mix_sample(const Mix& m, float u0, float u1, float u2) {
    float acc = 0.f;
    float3 mu = m.mu[G_LOBES - 1];
    float k = m.kappa[G_LOBES - 1], e2 = m.e2[G_LOBES - 1];
    bool found = false;
#pragma unroll
    for (int j = 0; j < G_LOBES; ++j) {
        acc += m.pi[j];
        if (!found && u0 < acc) {
            found = true;
            mu = m.mu[j];
            k = m.kappa[j];
            e2 = m.e2[j];
        }
    }
    return vmf_sample_fast(mu, k, e2, u1, u2);
}

// Block set-up (tensor-memory allocation, mbarriers, the weights of `net`
// unless null) and this thread's group.
SRT_DEV TcGroup tc_setup(unsigned char* smem, const GuideNet* net, float*& sb) {
    sb = reinterpret_cast<float*>(smem + TC_B_OFF);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + TC_BAR_OFF);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + TC_BAR_OFF + 8 * TC_GROUPS);
    if ((threadIdx.x >> 5) == 0) {
        tmem_alloc(tslot, TC_TMEM_COLS);
        tmem_relinquish();
    }
    if (threadIdx.x < TC_GROUPS) mbar_init(bars + threadIdx.x, 1);
    if (net) load_weights_tc(*net, smem, sb);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t grp = threadIdx.x / TC_ROWS;
    TcGroup g;
    g.A = smem + tc_aoff((int)grp);
    g.tmem = *tslot + 64u * grp;
    g.mbar = bars + grp;
    g.bar = 1u + grp;
    g.row = threadIdx.x % TC_ROWS;
    return g;
}
// After a timed-out layer: record it and give the group's MMAs in flight one
// more bounded wait; then (every path, whole block) free the tensor memory.
SRT_DEV void tc_teardown(const TcGroup& g, bool ok, uint32_t phase, uint32_t* err) {
    if (!ok) {
        if (g.row == 0) atomicOr(err, ERR_MMA_TIMEOUT);
        mbar_wait(g.mbar, phase, TC_WAIT_POLLS);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if ((threadIdx.x >> 5) == 0) tmem_dealloc(g.tmem, TC_TMEM_COLS);  // warp 0: group 0, base column
}

}  // namespace

// One 128-row tile of guided vertices (rows base .. base + 127 of n) of the
// renderer `a`: encoding, the network on the tensor cores, mixture
// sampling, the vertex continuation and the push into the next queue.
// False when the network's MMAs did not complete (nothing was written).
SRT_DEV bool infer_tile_tc(const FrameArgs& a, uint32_t bounce, const TcGroup& grp, const unsigned char* smem,
                           const float* sb, uint32_t base, uint32_t n, uint32_t& phase) {
    const GuideArgs& G = a.guide;
    const DevScene& S = a.scene;
    const uint32_t frame = a.cam->frame_count;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t v = base + grp.row;
    const bool valid = v < n;
    float x[G_IN];
    float4 p = splat4(0.f), nn = splat4(0.f);
    if (valid) {
        p = G.gv.p[v];
        nn = G.gv.n[v];
        float4 wo = G.gv.wo[v];
        vertex_inputs(xyz(p), xyz(nn), xyz(wo), p.w, S.bmin, S.binv, x);
    } else {
        for (int i = 0; i < G_IN; ++i) x[i] = 0.f;
    }
    encode_row_tc(x, grp.A, grp.row);
    fence_async_smem();
    group_sync(grp.bar);
    float raw[G_OUT];
    if (!mlp_tc(grp, smem, sb, phase, raw)) return false;
    bool alive = false;
    uint32_t id = 0;
    if (valid) {
        Mix m;
        mixture_fast(raw, m);
        id = G.gv.id[v];
        const uint4 misc = a.pb.misc[id];
        uint32_t s = misc.x;
        const float3 ffn = xyz(nn);
        float3 dir;
        if (rng_next(s) < m.sel) {
            const float u0 = rng_next(s), u1 = rng_next(s), u2 = rng_next(s);
            dir = mix_sample(m, u0, u1, u2);
        } else {
            float3 d = ffn + random_unit_vector(s);  // shader.wgsl:462-466
            if (length(d) < 0.001f) d = ffn;
            dir = normalize(d);
        }
        alive = finish_vertex(a, bounce, frame, v, id, p, ffn, misc, s, dir, m.sel, mix_pdf(m, dir));
    }
    const uint32_t mask = __ballot_sync(0xFFFFFFFFu, alive);
    uint32_t slot_base = 0;
    if (mask) {
        const int leader = __ffs(mask) - 1;
        if ((int)lane == leader) slot_base = atomicAdd(&a.counters->paths[bounce + 1], (uint32_t)__popc(mask));
        slot_base = __shfl_sync(0xFFFFFFFFu, slot_base, leader);
    }
    if (alive) a.pb.queue[(bounce + 1) & 1][slot_base + __popc(mask & ((1u << lane) - 1u))] = id;
    return true;
}

__global__ void __launch_bounds__(TC_ROWS * TC_GROUPS, 2) k_guide_infer_tc(FrameArgs a, uint32_t bounce) {
    const GuideArgs& G = a.guide;
    extern __shared__ __align__(1024) unsigned char smem[];
    const uint32_t n = G.gc->verts[bounce];
    if (blockIdx.x * TC_ROWS * TC_GROUPS >= n) return;
    float* sb;
    const TcGroup grp = tc_setup(smem, &G.net, sb);
    uint32_t phase = 0;
    bool ok = true;
    for (uint32_t base = (blockIdx.x * TC_GROUPS + threadIdx.x / TC_ROWS) * TC_ROWS; base < n;
         base += gridDim.x * TC_GROUPS * TC_ROWS) {
        if (!infer_tile_tc(a, bounce, grp, smem, sb, base, n, phase)) {
            ok = false;
            break;
        }
    }
    tc_teardown(grp, ok, phase, a.err);
}

// Guided vertices of many renderers (the batched renderer) in one persistent
// launch: a virtual queue concatenates every item's vertices of this bounce,
// each item padded to whole chunks of TC_CHUNK rows; a block draws chunks
// from *fetch (zeroed per frame), loads the network of the chunk's item when
// it differs from the one it holds, and its two groups run the chunk's two
// 128-row tiles.  Items whose path depth ends at this bounce take no chunk.
__global__ void __launch_bounds__(TC_ROWS * TC_GROUPS, 2)
    k_guide_infer_tc_multi(const FrameArgs* __restrict__ items, int n_items, uint32_t bounce,
                           uint32_t* __restrict__ fetch) {
    extern __shared__ __align__(1024) unsigned char smem[];
    uint32_t* pre = reinterpret_cast<uint32_t*>(smem + TC_SMEM);  // chunk offset of each item, then the total
    volatile uint32_t* slot = pre + MAX_BATCH + 1;                 // the chunk drawn, by iteration parity
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (int i = 0; i < n_items; ++i) {
            pre[i] = acc;
            const FrameArgs& a = items[i];
            const uint32_t n = bounce + 1u < a.max_depth ? a.guide.gc->verts[bounce] : 0u;
            acc += (n + TC_CHUNK - 1u) / TC_CHUNK;
        }
        pre[n_items] = acc;
    }
    __syncthreads();
    const uint32_t total = pre[n_items];
    if (blockIdx.x >= total) return;
    float* sb;
    const TcGroup grp = tc_setup(smem, nullptr, sb);
    const uint32_t g = threadIdx.x / TC_ROWS;
    int cur = -1;
    uint32_t phase = 0;
    bool ok = true;
    for (uint32_t it = 0;; ++it) {
        if (threadIdx.x == 0) slot[it & 1u] = atomicAdd(fetch, 1u);
        // the barrier also ends every group's previous tile (weights free to reload)
        if (__syncthreads_or(!ok)) break;
        const uint32_t c = slot[it & 1u];
        if (c >= total) break;
        int k = 0;
        while (k + 1 < n_items && pre[k + 1] <= c) ++k;
        const FrameArgs& a = items[k];
        if (k != cur) {
            load_weights_tc(a.guide.net, smem, sb);
            __syncthreads();
            cur = k;
        }
        const uint32_t n = a.guide.gc->verts[bounce];
        const uint32_t base = (c - pre[k]) * TC_CHUNK + g * TC_ROWS;
        if (base < n && !infer_tile_tc(a, bounce, grp, smem, sb, base, n, phase)) ok = false;
    }
    tc_teardown(grp, ok, phase, items[cur < 0 ? 0 : cur].err);
}

// The tcgen05 path's mixture: pdf at omega and a direction sampled with u, one sample per thread.
__global__ void k_guide_test_mixture_tc(const float* __restrict__ raw, const float* __restrict__ omega,
                                        const float* __restrict__ u, uint32_t n, float* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float r[G_OUT];
    for (int k = 0; k < G_OUT; ++k) r[k] = raw[(size_t)i * G_OUT + k];
    Mix m;
    mixture_fast(r, m);
    const float3 d = mix_sample(m, u[3 * i], u[3 * i + 1], u[3 * i + 2]);
    out[4 * i] = mix_pdf(m, f3(omega[3 * i], omega[3 * i + 1], omega[3 * i + 2]));
    out[4 * i + 1] = d.x;
    out[4 * i + 2] = d.y;
    out[4 * i + 3] = d.z;
}

// A wait that cannot complete, for the failure-path test: an mbarrier that
// expects one arrival and never gets it.  The bounded wait gives up after
// `polls` polls and records ERR_MMA_TIMEOUT, as the inference kernels' MMA
// waits do; nothing stays in flight.
__global__ void k_test_wait_timeout(uint32_t polls, uint32_t* err) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    const bool done = mbar_wait(&bar, 0, polls);
    if (!done && threadIdx.x == 0) atomicOr(err, ERR_MMA_TIMEOUT);
}

// Forward pass of n samples on the tcgen05 path (inputs [n][10] -> raw outputs [n][48]).
__global__ void __launch_bounds__(TC_ROWS * TC_GROUPS, 2) k_guide_test_forward_tc(GuideNet net,
                                                                                  const float* __restrict__ x,
                                                                                  uint32_t n, float* __restrict__ y,
                                                                                  uint32_t* err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    float* sb;
    const TcGroup grp = tc_setup(smem, &net, sb);
    uint32_t phase = 0;
    bool ok = true;
    for (uint32_t base = (blockIdx.x * TC_GROUPS + threadIdx.x / TC_ROWS) * TC_ROWS; base < n;
         base += gridDim.x * TC_GROUPS * TC_ROWS) {
        const uint32_t r = base + grp.row;
        float xi[G_IN];
        for (int i = 0; i < G_IN; ++i) xi[i] = r < n ? x[(size_t)r * G_IN + i] : 0.f;
        encode_row_tc(xi, grp.A, grp.row);
        fence_async_smem();
        group_sync(grp.bar);
        float raw[G_OUT];
        if (!mlp_tc(grp, smem, sb, phase, raw)) {
            ok = false;
            break;
        }
        if (r < n)
            for (int i = 0; i < G_OUT; ++i) y[(size_t)r * G_OUT + i] = raw[i];
    }
    tc_teardown(grp, ok, phase, err);
}

// ---------------------------------------------------------------- training on tcgen05
// One training step of the network on the fifth-generation tensor cores,
// fused: a block (128 threads, thread r = record row r of a 128-record
// tile) runs, per tile, the five forward layers (D = A W^T into tensor
// memory, bias + ReLU by the epilogue into the next A operand), the loss
// gradient, and the backward pass: per layer one product
// delta_{l-1} = (delta_l W_l) * relu'(a_{l-1}) and the weight-gradient
// product dW_l += delta_l^T a_{l-1}, both issued together.  The weight
// gradients accumulate in tensor memory over all of the block's tiles and
// reach the global gradient once, at the end; activations and deltas never
// leave shared memory.
//
// Operands: the K-major core-matrix layout of umma.cuh (the forward A, the
// weights, and the deltas as A of the backward product).  The same bytes
// read with the MN-major descriptor form serve the transposed products: the
// weights as B of the backward product (n = input, k = output) and the
// deltas and activations as the A and B of the weight gradient (k = record).
// In the MN-major no-swizzle form a core matrix is 8 (k) rows of 16 bytes
// holding 8 consecutive (mn) elements, adjacent core matrices along MN are
// 128 bytes apart (the stride byte offset) and along K `lbo` bytes apart
// (the leading byte offset): for a K-major buffer of K columns this is the
// buffer's row-block stride K / 8 * 128.
constexpr uint32_t TT_X_OFF = 47104u;                     // encoded inputs, 128 x 128
constexpr uint32_t TT_H_OFF = TT_X_OFF + 32768u;          // a0..a3, 4 x (128 x 64)
constexpr uint32_t TT_D_OFF = TT_H_OFF + 4u * 16384u;     // deltas, 2 x (128 x 64), ping-pong
// The weight-gradient product reads its A (out x 128 records) with M = 128
// rows; rows beyond the layer's outputs are other bytes of the buffers (their
// products are never read).  The slack after the second delta buffer keeps
// every operand read of the MN-major products inside the block's shared
// memory even if the two stride fields were taken the other way round
// (MN stride = the K-block stride): 30 KB.
constexpr uint32_t TT_B_OFF = TT_D_OFF + 2u * 16384u + 30720u;
constexpr uint32_t TT_BAR_OFF = TT_B_OFF + SB_ELEMS * 4;  // mbarrier, then the TMEM base
constexpr uint32_t TT_SMEM = TT_BAR_OFF + 16u;
constexpr uint32_t TT_TMEM_COLS = 512;
// tensor-memory columns: [0, 64) the layer products, then dW_0 .. dW_4
__host__ __device__ constexpr uint32_t tt_dw_col(int l) { return l == 0 ? 64u : 192u + 64u * (uint32_t)(l - 1); }
static_assert(tt_dw_col(4) + 64u <= TT_TMEM_COLS && TT_SMEM + 1024 <= 227 * 1024, "training kernel resources");
static_assert(TT_B_OFF % 16 == 0 && TT_BAR_OFF % 8 == 0, "training kernel alignment");

SRT_DEV uint32_t tt_idesc(uint32_t N, uint32_t a_mn, uint32_t b_mn) {
    return umma_idesc_bf16(128u, N) | (a_mn << 15) | (b_mn << 16);
}

// Bounded wait of the block on the MMAs committed to `mbar`; false for the
// whole block if they did not complete.
SRT_DEV bool tt_wait(uint64_t* mbar, uint32_t& phase) {
    const bool ok = __syncthreads_and(mbar_wait(mbar, phase, TC_WAIT_POLLS)) != 0;
    if (ok) phase ^= 1u;
    tc_fence_after();
    return ok;
}

__global__ void __launch_bounds__(128, 1) k_guide_train_tc(GuideArgs G, int step) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const StepRecs sr = step_recs(G, step);
    const uint32_t n = sr.count;
    const uint32_t n_tiles = (n + 127u) / 128u;
    if (blockIdx.x >= n_tiles) return;
    float* sb = reinterpret_cast<float*>(smem + TT_B_OFF);
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + TT_BAR_OFF);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + TT_BAR_OFF + 8);
    if ((threadIdx.x >> 5) == 0) {
        tmem_alloc(tslot, TT_TMEM_COLS);
        tmem_relinquish();
    }
    if (threadIdx.x == 0) mbar_init(mbar, 1);
    load_weights_tc(G.net, smem, sb);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t r = threadIdx.x;
    const uint32_t trow = tmem + (((r >> 5) * 32u) << 16);  // this thread's lane
    unsigned char* X = smem + TT_X_OFF;
    const uint32_t w_addr = smem_u32(smem), x_addr = smem_u32(X);
    const uint32_t n_all = min(G.gc->records, G.batch);
    const float inv_mean = G.gc->weight_sum > 0.f ? (float)n_all / G.gc->weight_sum : 0.f;
    uint32_t phase = 0;
    bool ok = true, first = true;
    float db[G_LAYERS] = {0.f, 0.f, 0.f, 0.f, 0.f};  // bias gradient of output r of each layer
    for (uint32_t tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
        const uint32_t j = tile * 128u + r;
        const bool valid = j < n;
        const uint32_t rec = rec_at(sr, valid ? j : 0u);
        float x[G_IN];
        if (valid) {
            const float4 x0 = G.rec.x0[rec], x1 = G.rec.x1[rec], x2 = G.rec.x2[rec];
            x[0] = x0.x; x[1] = x0.y; x[2] = x0.z; x[3] = x0.w;
            x[4] = x1.x; x[5] = x1.y; x[6] = x1.z; x[7] = x1.w;
            x[8] = x2.x; x[9] = x2.y;
        } else {
            for (int i = 0; i < G_IN; ++i) x[i] = 0.f;
        }
        encode_row_tc(x, X, r);
        fence_async_smem();
        __syncthreads();
        // ---- forward: a_l = relu(a_{l-1} W_l^T + b_l), raw = a_3 W_4^T + b_4
        uint32_t mask[4][2];  // ReLU derivative bits of a_0 .. a_3
        float raw[G_OUT];
        for (int l = 0; l < G_LAYERS && ok; ++l) {
            const uint32_t K = (uint32_t)g_in(l), N = (uint32_t)g_out(l), SBO = K / 8u * 128u;
            const uint32_t a_addr = l == 0 ? x_addr : smem_u32(smem + TT_H_OFF + 16384u * (uint32_t)(l - 1));
            if (r == 0) {
                tc_fence_after();
                for (uint32_t k = 0; k < K / 16u; ++k)
                    umma_bf16(tmem, umma_desc(a_addr + 256u * k, 128u, SBO),
                              umma_desc(w_addr + tc_woff(l) + 256u * k, 128u, SBO), tt_idesc(N, 0, 0), k);
                umma_commit(mbar);
            }
            ok = tt_wait(mbar, phase);
            if (!ok) break;
            const float* bias = sb + G_HID * l;
            uint32_t v[4][16];
            for (uint32_t c = 0; c < N / 16u; ++c) tmem_ld16(trow + 16u * c, v[c]);
            for (uint32_t c = 0; c < N / 16u; ++c) tmem_wait16(v[c]);
            if (l < G_LAYERS - 1) {
                unsigned char* H = smem + TT_H_OFF + 16384u * (uint32_t)l;
                mask[l][0] = mask[l][1] = 0u;
                for (int ch = 0; ch < G_HID / 8; ++ch) {
                    uint32_t pk[4];
                    for (int i = 0; i < 4; ++i) {
                        const int col = 8 * ch + 2 * i;
                        const float z0 = __uint_as_float(v[col >> 4][col & 15]) + bias[col];
                        const float z1 = __uint_as_float(v[(col + 1) >> 4][(col + 1) & 15]) + bias[col + 1];
                        pk[i] = pack2_relu(z0, z1);
                        // a ReLU derivative of 1 where the stored activation is nonzero
                        if (pk[i] & 0xFFFFu) mask[l][col >> 5] |= 1u << (col & 31);
                        if (pk[i] >> 16) mask[l][(col + 1) >> 5] |= 1u << ((col + 1) & 31);
                    }
                    *reinterpret_cast<uint4*>(H + umma_offset(r, 8u * (uint32_t)ch, G_HID)) =
                        make_uint4(pk[0], pk[1], pk[2], pk[3]);
                }
                fence_async_smem();
            } else {
                for (int i = 0; i < G_OUT; ++i) raw[i] = __uint_as_float(v[i >> 4][i & 15]) + bias[i];
            }
            tc_fence_before();
            __syncthreads();
        }
        if (!ok) break;
        // ---- the output delta (0 for rows past the step's records)
        {
            float gr[G_OUT];
            for (int i = 0; i < G_OUT; ++i) gr[i] = 0.f;
            if (valid) loss_grad(raw, G.rec.w[rec], G.rec.b[rec], G.rec.weight[rec] * inv_mean, gr);
            unsigned char* D = smem + TT_D_OFF;
            for (int ch = 0; ch < G_OUT / 8; ++ch)
                *reinterpret_cast<uint4*>(D + umma_offset(r, 8u * (uint32_t)ch, G_OUT)) =
                    make_uint4(pack2(gr[8 * ch], gr[8 * ch + 1]), pack2(gr[8 * ch + 2], gr[8 * ch + 3]),
                               pack2(gr[8 * ch + 4], gr[8 * ch + 5]), pack2(gr[8 * ch + 6], gr[8 * ch + 7]));
            fence_async_smem();
        }
        __syncthreads();
        // ---- backward
        uint32_t cur = 0;
        for (int l = G_LAYERS - 1; l >= 0 && ok; --l) {
            const uint32_t out_l = (uint32_t)g_out(l), in_l = (uint32_t)g_in(l);
            unsigned char* Dc = smem + TT_D_OFF + 16384u * cur;
            // bias gradient: the sum of this layer's delta over the tile (bf16 as stored)
            if (r < out_l) {
                float acc = 0.f;
                for (uint32_t row = 0; row < 128u; ++row)
                    acc += __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(Dc + umma_offset(row, r, out_l)));
                db[l] += acc;
            }
            const uint32_t d_addr = smem_u32(Dc);
            const uint32_t in_addr = l == 0 ? x_addr : smem_u32(smem + TT_H_OFF + 16384u * (uint32_t)(l - 1));
            const uint32_t d_lbo = out_l / 8u * 128u, in_lbo = in_l / 8u * 128u;
            if (r == 0) {
                tc_fence_after();
                if (l > 0) {
                    // delta_l W_l: A = delta_l (K-major, k = output), B = W_l read MN-major (n = input)
                    for (uint32_t k = 0; k < out_l / 16u; ++k)
                        umma_bf16(tmem, umma_desc(d_addr + 256u * k, 128u, d_lbo),
                                  umma_desc(w_addr + tc_woff(l) + 2u * in_lbo * k, in_lbo, 128u), tt_idesc(in_l, 0, 1),
                                  k);
                }
                // dW_l += delta_l^T a_{l-1}: both read MN-major, k = record
                for (uint32_t k = 0; k < 8u; ++k)
                    umma_bf16(tmem + tt_dw_col(l), umma_desc(d_addr + 2u * d_lbo * k, d_lbo, 128u),
                              umma_desc(in_addr + 2u * in_lbo * k, in_lbo, 128u), tt_idesc(in_l, 1, 1),
                              (first && k == 0) ? 0u : 1u);
                umma_commit(mbar);
            }
            ok = tt_wait(mbar, phase);
            if (!ok || l == 0) break;
            // delta_{l-1} = (delta_l W_l) * relu'(a_{l-1}) into the other buffer
            uint32_t v[4][16];
            for (uint32_t c = 0; c < 4u; ++c) tmem_ld16(trow + 16u * c, v[c]);
            for (uint32_t c = 0; c < 4u; ++c) tmem_wait16(v[c]);
            unsigned char* Dn = smem + TT_D_OFF + 16384u * (cur ^ 1u);
            for (int ch = 0; ch < G_HID / 8; ++ch) {
                uint32_t pk[4];
                for (int i = 0; i < 4; ++i) {
                    const int col = 8 * ch + 2 * i;
                    const float g0 = (mask[l - 1][col >> 5] >> (col & 31)) & 1u ? __uint_as_float(v[col >> 4][col & 15]) : 0.f;
                    const float g1 = (mask[l - 1][(col + 1) >> 5] >> ((col + 1) & 31)) & 1u
                                         ? __uint_as_float(v[(col + 1) >> 4][(col + 1) & 15])
                                         : 0.f;
                    pk[i] = pack2(g0, g1);
                }
                *reinterpret_cast<uint4*>(Dn + umma_offset(r, 8u * (uint32_t)ch, G_HID)) =
                    make_uint4(pk[0], pk[1], pk[2], pk[3]);
            }
            fence_async_smem();
            tc_fence_before();
            __syncthreads();
            cur ^= 1u;
        }
        if (!ok) break;
        first = false;
        tc_fence_before();
        __syncthreads();  // the next tile overwrites the operands of this tile's last products
    }
    if (ok && !first) {
        // the block's weight gradients: TMEM lane r holds output row r of each dW_l
        for (int l = 0; l < G_LAYERS; ++l) {
            const uint32_t out_l = (uint32_t)g_out(l), in_l = (uint32_t)g_in(l);
            float* gw = G.net.grad + g_woff(l);
            for (uint32_t c0 = 0; c0 < in_l; c0 += 16u) {
                uint32_t v[16];
                tmem_ld16(trow + tt_dw_col(l) + c0, v);
                tmem_wait16(v);
                if (r < out_l)
                    for (int i = 0; i < 16; ++i) atomicAdd(gw + r * in_l + c0 + (uint32_t)i, __uint_as_float(v[i]));
            }
            if (r < out_l && db[l] != 0.f) atomicAdd(G.net.grad + g_boff(l) + r, db[l]);
        }
    }
    if (!ok) {
        if (r == 0 && G.err) atomicOr(G.err, ERR_MMA_TIMEOUT);
        mbar_wait(mbar, phase, TC_WAIT_POLLS);  // MMAs still in flight: one more bounded wait
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if ((threadIdx.x >> 5) == 0) tmem_dealloc(tmem, TT_TMEM_COLS);
}

// ---------------------------------------------------------------- launchers
size_t guide_infer_smem() {
    return SW_ELEMS * 2 + SB_ELEMS * 4 + GWI * IN_BYTES;
}
size_t guide_train_smem() {
    return SW_ELEMS * 2 + SB_ELEMS * 4 +
           GWT * (16 * g_pad(G_ENC) * 2 + 4 * 16 * g_pad(G_HID) * 2 + 16 * 52 * 4 + 16 * g_pad(G_OUT) * 2);
}

cudaError_t guide_configure() {
    cudaError_t e = cudaFuncSetAttribute(k_guide_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)guide_infer_smem());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_guide_test_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)guide_infer_smem());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_guide_fwdbwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)guide_train_smem());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_guide_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_guide_test_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_guide_infer_tc_multi, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)TC_SMEM_MULTI);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_guide_fwdbwd_multi, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)guide_train_smem());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_guide_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TT_SMEM);
    return e;
}

int launch_guide_infer(const FrameArgs& a, uint32_t bounce, cudaStream_t st) {
    uint32_t grid = (uint32_t)(a.sm_count > 0 ? a.sm_count : 148) * 2;
    if (a.guide.tc) k_guide_infer_tc<<<grid, TC_ROWS * TC_GROUPS, TC_SMEM, st>>>(a, bounce);
    else k_guide_infer<<<grid, GWI * 32, guide_infer_smem(), st>>>(a, bounce);
    return 1;
}

namespace {
int launch_train_steps(const GuideArgs& g, int sm, int adam, cudaStream_t st) {
    int n = 0;
    for (int k = 0; k < (int)std::max(g.steps, 1u); ++k) {
        if (g.tc_train) {
            k_guide_train_tc<<<sm, 128, TT_SMEM, st>>>(g, k);
            n += 1;
        } else {
            k_guide_fwdbwd<<<sm, GWT * 32, guide_train_smem(), st>>>(g, k);
            dim3 wg(WGRAD_BLOCKS, 6);
            k_guide_wgrad<<<wg, 256, 0, st>>>(g, k);
            n += 2;
        }
        if (!adam) continue;
        k_guide_adam<<<(G_NPARAMS + 255) / 256, 256, 0, st>>>(g, k);
        ++n;
    }
    return n;
}
}  // namespace

int launch_guide_train(const FrameArgs& a, cudaStream_t st) {
    return launch_guide_targets(a, st) + launch_guide_steps(a, st);
}

int launch_guide_targets(const FrameArgs& a, cudaStream_t st) {
    if (!a.guide.train) return 0;
    const int sm = a.sm_count > 0 ? a.sm_count : 148;
    k_guide_targets<<<sm * 4, 256, 0, st>>>(a);
    return 1;
}

int launch_guide_steps(const FrameArgs& a, cudaStream_t st) {
    const GuideArgs& g = a.guide;
    const int sm = a.sm_count > 0 ? a.sm_count : 148;
    int n = g.train ? launch_train_steps(g, sm, 1, st) : 0;
    k_guide_frame_end<<<1, 32, 0, st>>>(g, g.train);
    return n + 1;
}

int launch_guide_infer_multi(const FrameArgs* items, int n_items, uint32_t bounce, uint32_t* fetch, int sm_count,
                             cudaStream_t st) {
    if (n_items <= 0) return 0;
    const uint32_t grid = (uint32_t)(sm_count > 0 ? sm_count : 148) * 2;
    k_guide_infer_tc_multi<<<grid, TC_ROWS * TC_GROUPS, TC_SMEM_MULTI, st>>>(items, n_items, bounce, fetch);
    return 1;
}

int launch_guide_train_multi(const FrameArgs* items, int n_items, uint32_t max_steps, int sm_count,
                             cudaStream_t st) {
    if (n_items <= 0) return 0;
    const uint32_t sm = (uint32_t)(sm_count > 0 ? sm_count : 148);
    const uint32_t per = std::max(8u, 2u * sm / (uint32_t)n_items);  // forward/backward blocks per item
    const uint32_t n = (uint32_t)n_items;
    k_guide_targets_multi<<<dim3(std::max(8u, 4u * sm / n), n), 256, 0, st>>>(items);
    int launches = 2;
    for (int k = 0; k < (int)std::max(max_steps, 1u); ++k) {
        k_guide_fwdbwd_multi<<<dim3(per, n), GWT * 32, guide_train_smem(), st>>>(items, k);
        k_guide_wgrad_multi<<<dim3(WGRAD_BLOCKS, 6, n), 256, 0, st>>>(items, k);
        k_guide_adam_multi<<<dim3((G_NPARAMS + 255) / 256, n), 256, 0, st>>>(items, k);
        launches += 3;
    }
    k_guide_frame_end_multi<<<n, 32, 0, st>>>(items);
    return launches;
}

int launch_test_wait_timeout(uint32_t polls, uint32_t* err, cudaStream_t st) {
    k_test_wait_timeout<<<1, 32, 0, st>>>(polls, err);
    return 1;
}

int launch_guide_test_train(const GuideArgs& g, int phase, cudaStream_t st) {
    if (phase == 0) return launch_train_steps(g, 148, 0, st);
    k_guide_adam<<<(G_NPARAMS + 255) / 256, 256, 0, st>>>(g, 0);
    return 1;
}

// ---------------------------------------------------------------- host side
namespace {
template <class T>
cudaError_t galloc(T** p, size_t n) {
    return cudaMalloc((void**)p, n * sizeof(T));
}
// splitmix64: the deterministic stream of the default initialisation
uint64_t splitmix(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
}  // namespace

void guide_default_params(uint64_t seed, float* out) {
    uint64_t x = seed;
    for (int l = 0; l < G_LAYERS; ++l) {
        // He-uniform; the output layer starts 10x smaller so the first
        // mixtures are broad and nearly uniform
        float a = sqrtf(6.0f / (float)g_in(l)) * (l == 4 ? 0.1f : 1.0f);
        for (int i = 0; i < g_in(l) * g_out(l); ++i) {
            double u = (double)(splitmix(x) >> 11) * (1.0 / 9007199254740992.0);
            out[g_woff(l) + i] = (float)((2.0 * u - 1.0) * a);
        }
        for (int i = 0; i < g_out(l); ++i) out[g_boff(l) + i] = 0.0f;
    }
    for (int j = 0; j < G_LOBES; ++j) out[g_boff(4) + 5 * j + 3] = 1.0f;  // kappa ~ e
    out[g_boff(4) + 40] = -1.0f;  // selection ~ 0.05 + 0.85 sigmoid(-1) = 0.28
}

cudaError_t guide_alloc(GuideArgs& g, size_t n_verts) {
    g = GuideArgs{};
    g.steps = 1;
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
    };
    chk(galloc(&g.net.master, G_NPARAMS));
    chk(galloc(&g.net.wbf, G_NPARAMS));
    chk(galloc(&g.net.adam_m, G_NPARAMS));
    chk(galloc(&g.net.adam_v, G_NPARAMS));
    chk(galloc(&g.net.grad, G_NPARAMS));
    if (n_verts > 0) {
        chk(galloc(&g.gv.p, n_verts));
        chk(galloc(&g.gv.n, n_verts));
        chk(galloc(&g.gv.wo, n_verts));
        chk(galloc(&g.gv.spec, n_verts));
        chk(galloc(&g.gv.id, n_verts));
    }
    chk(galloc(&g.rec.x0, G_REC_CAP));
    chk(galloc(&g.rec.x1, G_REC_CAP));
    chk(galloc(&g.rec.x2, G_REC_CAP));
    chk(galloc(&g.rec.w, G_REC_CAP));
    chk(galloc(&g.rec.b, G_REC_CAP));
    chk(galloc(&g.rec.thr, G_REC_CAP));
    chk(galloc(&g.rec.rad, G_REC_CAP));
    chk(galloc(&g.rec.pid, G_REC_CAP));
    chk(galloc(&g.rec.weight, G_REC_CAP));
    chk(galloc(&g.rec.act, (size_t)G_REC_CAP * G_ACT_STRIDE));
    chk(galloc(&g.rec.delta, (size_t)G_REC_CAP * G_DELTA_STRIDE));
    chk(galloc(&g.gc, 1));
    if (e == cudaSuccess) {
        GuideCounters gc{};
        gc.threshold = 65536u;
        e = cudaMemcpy(g.gc, &gc, sizeof(gc), cudaMemcpyHostToDevice);
    }
    g.lr = 1e-3f;
    g.train = 1;
    g.batch = G_BATCH_DEFAULT;
    g.tc = 1;
    return e;
}

void guide_free(GuideArgs& g) {
    void* bufs[] = {g.net.master, g.net.wbf, g.net.adam_m, g.net.adam_v, g.net.grad,
                    g.gv.p, g.gv.n, g.gv.wo, g.gv.spec, g.gv.id, g.rec.x0, g.rec.x1, g.rec.x2, g.rec.w, g.rec.b,
                    g.rec.thr, g.rec.rad, g.rec.pid, g.rec.weight, g.rec.act, g.rec.delta, g.gc};
    for (void* b : bufs) cudaFree(b);
    g = GuideArgs{};
}

size_t guide_state_bytes() { return (size_t)G_NPARAMS * (4 * 3 + 2) + sizeof(GuideCounters); }

cudaError_t guide_state_copy(GuideArgs& g, void* buf, bool save, cudaStream_t st) {
    unsigned char* b = static_cast<unsigned char*>(buf);
    void* parts[] = {g.net.master, g.net.adam_m, g.net.adam_v, g.net.wbf, g.gc};
    const size_t sizes[] = {(size_t)G_NPARAMS * 4, (size_t)G_NPARAMS * 4, (size_t)G_NPARAMS * 4, (size_t)G_NPARAMS * 2,
                            sizeof(GuideCounters)};
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 5 && e == cudaSuccess; ++i) {
        e = save ? cudaMemcpyAsync(b, parts[i], sizes[i], cudaMemcpyDeviceToDevice, st)
                 : cudaMemcpyAsync(parts[i], b, sizes[i], cudaMemcpyDeviceToDevice, st);
        b += sizes[i];
    }
    return e;
}

cudaError_t guide_upload(GuideArgs& g, const float* params, const float* adam_m, const float* adam_v,
                         uint32_t adam_step) {
    std::vector<__nv_bfloat16> wbf(G_NPARAMS, __float2bfloat16_rn(0.0f));
    for (int l = 0; l < G_LAYERS; ++l)
        for (int k = 0; k < g_in(l) * g_out(l); ++k)
            wbf[g_woff(l) + k] = __float2bfloat16_rn(params[g_woff(l) + k]);
    std::vector<float> zero(G_NPARAMS, 0.0f);
    cudaError_t e = cudaMemcpy(g.net.master, params, G_NPARAMS * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(g.net.wbf, wbf.data(), G_NPARAMS * 2, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(g.net.adam_m, adam_m ? adam_m : zero.data(), G_NPARAMS * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(g.net.adam_v, adam_v ? adam_v : zero.data(), G_NPARAMS * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(g.net.grad, zero.data(), G_NPARAMS * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(&g.gc->adam_step, &adam_step, 4, cudaMemcpyHostToDevice);
    return e;
}

int launch_guide_test_forward(const GuideNet& net, const float* x, uint32_t n, float* y, int tc, uint32_t* err,
                              cudaStream_t st) {
    if (tc) k_guide_test_forward_tc<<<128, TC_ROWS * TC_GROUPS, TC_SMEM, st>>>(net, x, n, y, err);
    else k_guide_test_forward<<<64, GWI * 32, guide_infer_smem(), st>>>(net, x, n, y);
    return 1;
}
int launch_guide_test_mixture(const float* raw, const float* omega, const float* u, uint32_t n, float* out,
                              int tc, cudaStream_t st) {
    if (tc) {
        k_guide_test_mixture_tc<<<(n + 127) / 128, 128, 0, st>>>(raw, omega, u, n, out);
        return 1;
    }
    k_guide_test_mixture<<<(n + 63) / 64, 128, 0, st>>>(raw, omega, u, n, out);  // 16 samples per warp
    return 1;
}

}  // namespace srt
