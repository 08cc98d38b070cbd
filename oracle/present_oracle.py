"""CPU restatement of the reference's two raster steps (numpy, float32).

TEST INFRASTRUCTURE ONLY: the oracle for the CUDA presentation kernels.

* Letterbox blit: renderer/blit_pass.rs:114-154 (scale of the quad from the
  target and window aspect ratios), shaders/blit.wgsl:7-34 (a quad over
  NDC [-1, 1]^2 scaled by (sx, sy), uv (0, 0) at NDC (-1, -1), sampled with
  the default sampler: nearest texel, clamp to edge), renderer/blit_pass.rs:
  169 (target cleared to blue).  Restated per pixel centre: the window pixel
  (x, y) (row 0 at the top) has NDC ((x + 0.5) / W * 2 - 1, 1 - (y + 0.5) /
  H * 2); it is inside the quad when -sx <= xn < sx and -sy < yn <= sy.
* Photon splat: shaders/debug_photons.wgsl:24-47 (clip = proj * view *
  (p, 1), photons with zero energy skipped, colour (1, 0.6, 0.1, 0.3)),
  renderer/debug_photons_pass.rs:86-99 (additive blend src * alpha + dst,
  alpha replaced, point list).  A point covers the pixel containing its
  position; the k photons of a pixel are added at once.

Every float operation is done in float32 in the kernel's order.
"""
from __future__ import annotations

import numpy as np

F = np.float32


def letterbox_scale(tw, th, ww, wh):
    ta = F(tw) / F(th)
    wa = F(ww) / F(wh)
    if wa > ta:
        return ta / wa, F(1.0)
    return F(1.0), wa / ta


def _srgb_oetf(c):
    c = c.astype(np.float64)
    return np.where(c <= 0.0031308, 12.92 * c, 1.055 * np.power(c, 1.0 / 2.4) - 0.055)


def blit_letterbox(src: np.ndarray, ww: int, wh: int, srgb: bool = False) -> np.ndarray:
    sh, sw = src.shape[:2]
    sx, sy = letterbox_scale(sw, sh, ww, wh)
    x = np.arange(ww, dtype=F)
    y = np.arange(wh, dtype=F)
    xn = (x + F(0.5)) / F(ww) * F(2.0) - F(1.0)
    yn = F(1.0) - (y + F(0.5)) / F(wh) * F(2.0)
    XN, YN = np.meshgrid(xn, yn)
    inside = (XN >= -sx) & (XN < sx) & (YN > -sy) & (YN <= sy)
    u = (XN / sx + F(1.0)) * F(0.5)
    v = (YN / sy + F(1.0)) * F(0.5)
    tx = np.minimum(np.maximum(np.floor(u * F(sw)), 0), sw - 1).astype(np.int64)
    ty = np.minimum(np.maximum(np.floor(v * F(sh)), 0), sh - 1).astype(np.int64)
    out = np.zeros((wh, ww, 4), np.uint8)
    out[...] = (0, 0, 255, 255)
    c = src[ty, tx]
    if srgb:
        c = c.copy()
        c[..., :3] = np.rint(_srgb_oetf(c[..., :3] / 255.0) * 255.0).astype(np.uint8)
    out[inside] = c[inside]
    return out


def photon_pixels(photons: np.ndarray, view: np.ndarray, proj: np.ndarray, w: int, h: int):
    """Pixel index (y * w + x) of every visible photon with non-zero energy."""
    p = photons.astype(F)
    keep = p[:, 7] != 0
    p = p[keep]
    V = view.astype(F).reshape(4, 4)  # column-major: V[col, row]
    P = proj.astype(F).reshape(4, 4)
    v = [((V[0, r] * p[:, 0] + V[1, r] * p[:, 1]) + V[2, r] * p[:, 2]) + V[3, r] for r in range(4)]
    c = [((P[0, r] * v[0] + P[1, r] * v[1]) + P[2, r] * v[2]) + P[3, r] * v[3] for r in range(4)]
    cw = c[3]
    ok = (cw > 0) & (c[0] >= -cw) & (c[0] <= cw) & (c[1] >= -cw) & (c[1] <= cw) & (c[2] >= 0) & (c[2] <= cw)
    fx = (c[0][ok] / cw[ok] + F(1.0)) * F(0.5) * F(w)
    fy = (F(1.0) - c[1][ok] / cw[ok]) * F(0.5) * F(h)
    px = np.minimum(fx.astype(np.int64), w - 1)
    py = np.minimum(fy.astype(np.int64), h - 1)
    return py * w + px


def photon_splat(photons: np.ndarray, view: np.ndarray, proj: np.ndarray, rgba: np.ndarray) -> np.ndarray:
    h, w = rgba.shape[:2]
    counts = np.bincount(photon_pixels(photons, view, proj, w, h), minlength=w * h).reshape(h, w)
    out = rgba.copy()
    k = counts.astype(F)
    hit = counts > 0
    a = F(0.3)
    for ch, col in enumerate((F(1.0), F(0.6), F(0.1))):
        val = np.minimum(rgba[..., ch].astype(F) / F(255.0) + k * (col * a), F(1.0))
        out[..., ch] = np.where(hit, np.rint(val * F(255.0)).astype(np.uint8), rgba[..., ch])
    out[..., 3] = np.where(hit, np.uint8(np.rint(a * F(255.0))), rgba[..., 3])
    return out
