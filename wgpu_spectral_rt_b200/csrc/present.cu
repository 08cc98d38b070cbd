// present.cu — the reference's two raster steps, redone headless as CUDA
// kernels writing a device RGBA8 buffer:
//
// * letterbox blit (shaders/blit.wgsl:7-34, renderer/blit_pass.rs:114-154):
//   the rendered image drawn as an aspect-fit quad over a window-sized
//   target cleared to blue, sampled nearest-texel (the default sampler,
//   renderer/mod.rs:112), optionally sRGB-encoded as an sRGB swapchain
//   format would;
// * photon point splat (shaders/debug_photons.wgsl:24-47,
//   renderer/debug_photons_pass.rs:74-139): every photon with non-zero
//   energy projected by the camera's view and projection matrices to one
//   pixel, colour (1, 0.6, 0.1) with alpha 0.3 blended additively
//   (src * alpha + dst, saturating) over the target, alpha replaced.
//
// The raster rules are restated for pixel centres: a window pixel belongs to
// the quad when its centre's NDC lies in [-sx, sx) x (-sy, sy]; the quad's
// uv is affine in NDC; a point covers the pixel containing its position.
// Splat blending adds k contributions at once and rounds once (a raster
// blend rounds after each photon; the overlay is a debug view).
#include <cstdint>
#include <cstring>
#include <vector>

#include "render_kernels.h"

namespace srt {

namespace {

__device__ __forceinline__ float srgb_oetf(float c) {
    return c <= 0.0031308f ? 12.92f * c : 1.055f * powf(c, 1.0f / 2.4f) - 0.055f;
}

__global__ void k_blit_letterbox(const uchar4* __restrict__ src, uint32_t sw, uint32_t sh, uchar4* __restrict__ dst,
                                 uint32_t ww, uint32_t wh, float sx, float sy, int srgb) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ww * wh) return;
    uint32_t x = i % ww, y = i / ww;
    float xn = ((float)x + 0.5f) / (float)ww * 2.0f - 1.0f;
    float yn = 1.0f - ((float)y + 0.5f) / (float)wh * 2.0f;
    uchar4 c = make_uchar4(0, 0, 255, 255);  // LoadOp::Clear(BLUE), blit_pass.rs:169
    if (xn >= -sx && xn < sx && yn > -sy && yn <= sy) {
        float u = (xn / sx + 1.0f) * 0.5f, v = (yn / sy + 1.0f) * 0.5f;
        uint32_t tx = min((uint32_t)fmaxf(floorf(u * (float)sw), 0.0f), sw - 1u);
        uint32_t ty = min((uint32_t)fmaxf(floorf(v * (float)sh), 0.0f), sh - 1u);
        c = src[(size_t)ty * sw + tx];
        if (srgb) {
            c.x = (unsigned char)__float2uint_rn(srgb_oetf((float)c.x / 255.0f) * 255.0f);
            c.y = (unsigned char)__float2uint_rn(srgb_oetf((float)c.y / 255.0f) * 255.0f);
            c.z = (unsigned char)__float2uint_rn(srgb_oetf((float)c.z / 255.0f) * 255.0f);
        }
    }
    dst[i] = c;
}

// clip = proj * view * (p, 1) with the uniform's column-major matrices.
__global__ void k_photon_splat_count(const float4* __restrict__ photons, uint32_t n,
                                     const srt_camera_uniform* __restrict__ cam, uint32_t w, uint32_t h,
                                     uint32_t* __restrict__ counts) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 p = photons[2 * i], d = photons[2 * i + 1];
    if (d.w == 0.0f) return;  // debug_photons.wgsl:28-31
    const float* V = cam->view;
    const float* P = cam->proj;
    float v[4], c[4];
    for (int r = 0; r < 4; ++r) v[r] = V[r] * p.x + V[4 + r] * p.y + V[8 + r] * p.z + V[12 + r];
    for (int r = 0; r < 4; ++r) c[r] = P[r] * v[0] + P[4 + r] * v[1] + P[8 + r] * v[2] + P[12 + r] * v[3];
    float cw = c[3];
    if (!(cw > 0.0f) || c[0] < -cw || c[0] > cw || c[1] < -cw || c[1] > cw || c[2] < 0.0f || c[2] > cw) return;
    float fx = (c[0] / cw + 1.0f) * 0.5f * (float)w, fy = (1.0f - c[1] / cw) * 0.5f * (float)h;
    uint32_t px = min((uint32_t)fx, w - 1u), py = min((uint32_t)fy, h - 1u);
    atomicAdd(&counts[(size_t)py * w + px], 1u);
}

__global__ void k_photon_splat_resolve(const uint32_t* __restrict__ counts, uchar4* __restrict__ img, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t k = counts[i];
    if (k == 0u) return;
    uchar4 d = img[i];
    const float a = 0.3f, fk = (float)k;
    float r = fminf((float)d.x / 255.0f + fk * (1.0f * a), 1.0f);
    float g = fminf((float)d.y / 255.0f + fk * (0.6f * a), 1.0f);
    float b = fminf((float)d.z / 255.0f + fk * (0.1f * a), 1.0f);
    img[i] = make_uchar4((unsigned char)__float2uint_rn(r * 255.0f), (unsigned char)__float2uint_rn(g * 255.0f),
                         (unsigned char)__float2uint_rn(b * 255.0f), (unsigned char)__float2uint_rn(a * 255.0f));
}

}  // namespace

void letterbox_scale(uint32_t tw, uint32_t th, uint32_t ww, uint32_t wh, float* sx, float* sy) {
    // blit_pass.rs:123-140
    float target_aspect = (float)tw / (float)th;
    float window_aspect = (float)ww / (float)wh;
    *sx = 1.0f;
    *sy = 1.0f;
    if (window_aspect > target_aspect) *sx = target_aspect / window_aspect;
    else *sy = window_aspect / target_aspect;
}

int launch_blit_letterbox(const uchar4* src, uint32_t sw, uint32_t sh, uchar4* dst, uint32_t ww, uint32_t wh,
                          int srgb, cudaStream_t st) {
    float sx, sy;
    letterbox_scale(sw, sh, ww, wh, &sx, &sy);
    uint32_t n = ww * wh;
    k_blit_letterbox<<<(n + 255) / 256, 256, 0, st>>>(src, sw, sh, dst, ww, wh, sx, sy, srgb);
    return 1;
}

int launch_photon_splat(const float4* photons, uint32_t n, const srt_camera_uniform* cam, uint32_t w, uint32_t h,
                        uint32_t* counts, uchar4* img, cudaStream_t st) {
    uint32_t np = w * h;
    cudaMemsetAsync(counts, 0, (size_t)np * 4, st);
    int launches = 0;
    if (n) {
        k_photon_splat_count<<<(n + 255) / 256, 256, 0, st>>>(photons, n, cam, w, h, counts);
        ++launches;
    }
    k_photon_splat_resolve<<<(np + 255) / 256, 256, 0, st>>>(counts, img, np);
    return launches + 1;
}

}  // namespace srt
