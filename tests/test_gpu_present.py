"""Headless presentation kernels against their CPU restatement
(oracle/present_oracle.py): letterbox blit (both aspect cases, sRGB target)
and the photon point splat; the renderer entry points against the
standalone ones.  The first test runs on CPU (the restatement's geometry)."""
from __future__ import annotations

import math

import numpy as np
import pytest

import present_oracle as po


def test_letterbox_geometry_cpu():
    # a square image in a 2:1 window: the quad covers the middle half
    src = np.full((10, 10, 4), 200, np.uint8)
    out = po.blit_letterbox(src, 40, 20)
    assert np.all(out[:, :10] == (0, 0, 255, 255)) and np.all(out[:, 30:] == (0, 0, 255, 255))
    assert np.all(out[:, 10:30] == 200)
    # a wide image in a square window: bars above and below
    src = np.zeros((4, 20, 4), np.uint8)
    src[0] = 9  # top texel row
    out = po.blit_letterbox(src, 20, 20)
    rows = np.where(np.any(out[:, 0] != (0, 0, 255, 255), axis=1))[0]
    assert rows.min() == 8 and rows.max() == 11
    # uv (0, 0) (texel row 0) lands at the bottom of the quad (blit.wgsl:10-27)
    assert np.all(out[11, :, :3] == 9) and not np.any(out[8, :, :3] == 9)


@pytest.mark.gpu
@pytest.mark.parametrize("sw,sh,ww,wh", [(64, 48, 200, 100), (64, 48, 100, 200), (37, 91, 91, 37), (16, 16, 16, 16),
                                         (1920, 1080, 1280, 1024)])
def test_blit_matches_oracle(srt, ctx, sw, sh, ww, wh):
    rng = np.random.default_rng(sw * 7 + ww)
    src = rng.integers(0, 256, (sh, sw, 4), dtype=np.uint8)
    out = srt.blit_letterbox(ctx, src, ww, wh)
    np.testing.assert_array_equal(out, po.blit_letterbox(src, ww, wh))
    out_s = srt.blit_letterbox(ctx, src, ww, wh, srgb_target=True)
    ref_s = po.blit_letterbox(src, ww, wh, srgb=True)
    diff = np.abs(out_s.astype(int) - ref_s.astype(int))
    assert diff.max() <= 1 and np.mean(diff > 0) < 1e-3  # powf vs FP64 pow at rounding ties


def _camera(srt, aspect):
    return srt.camera_uniform([0.0, 0.0, 3.0], -math.pi / 2, 0.0, aspect, 0)


@pytest.mark.gpu
@pytest.mark.parametrize("n,w,h", [(0, 32, 24), (1, 32, 24), (50_000, 160, 120), (300_000, 640, 360)])
def test_photon_splat_matches_oracle(srt, ctx, n, w, h):
    rng = np.random.default_rng(n + w)
    ph = np.zeros((n, 8), np.float32)
    ph[:, 0:3] = rng.uniform(-1.5, 1.5, (n, 3))
    ph[:, 3] = rng.uniform(380, 780, n)
    ph[:, 7] = np.where(rng.uniform(size=n) < 0.1, 0.0, rng.uniform(0.1, 2.0, n))  # some never stored
    cam = _camera(srt, w / h)
    base = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    out = srt.photon_splat(ctx, ph, cam, base)
    view = np.array(cam.view, np.float32)
    proj = np.array(cam.proj, np.float32)
    np.testing.assert_array_equal(out, po.photon_splat(ph, view, proj, base))


@pytest.mark.gpu
def test_renderer_blit_and_splat(srt, ctx):
    b = srt.SceneBuilder()
    cam = b.add_preset(srt.PRESET_CONFIG1)
    scene = b.build(ctx)
    w, h = 96, 64
    r = srt.Renderer(ctx, scene, w, h, srt.default_params(photons_per_frame=1 << 16))
    u = srt.CameraController(*cam).build_uniform(w / h, 0)
    r.render(u)
    ldr = r.read_ldr()
    np.testing.assert_array_equal(r.blit(160, 90), srt.blit_letterbox(ctx, ldr, 160, 90))
    window = r.blit(w, h)
    photons = r.read_photons()
    assert len(photons) > 0
    np.testing.assert_array_equal(r.splat_photons(u, window), srt.photon_splat(ctx, photons, u, window))
    r.close()
    scene.close()


@pytest.mark.gpu
def test_async_ldr_readback(srt, ctx):
    """srt_read_ldr_async + srt_ldr_wait return each frame's image (pinned
    slots used in turn) while the next frame is already enqueued."""
    b = srt.SceneBuilder()
    cam = b.add_preset(srt.PRESET_CORNELL_BOX)
    scene = b.build(ctx)
    w, h = 64, 48
    p = srt.default_params(photons_per_frame=1 << 14)
    ra, rs = srt.Renderer(ctx, scene, w, h, p), srt.Renderer(ctx, scene, w, h, p)
    ctl = srt.CameraController(*cam)
    tickets, got, want = [], [], []
    for f in range(5):
        u = ctl.build_uniform(w / h, f)
        ra.render(u)
        tickets.append(ra.read_ldr_async())
        if f >= 1:
            got.append(ra.ldr_wait(tickets[f - 1]).copy())
        rs.render(u)
        want.append(rs.read_ldr())
    got.append(ra.ldr_wait(tickets[-1]).copy())
    for g, x in zip(got, want):
        np.testing.assert_array_equal(g, x)
    with pytest.raises(srt.SrtError):
        ra.ldr_wait(tickets[0])  # its slot has been reused
    ra.close()
    rs.close()
    scene.close()
