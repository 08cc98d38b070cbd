"""The tail kernel (srt_renderer_set_tail): the last bounces of every path in
one persistent launch give the same image, bit for bit, and the same ray
counts as the bounce-by-bounce wavefront, on scenes with every material kind,
at several first bounces, with and without the frame graph, and for a guided
renderer whose guided bounces end before the tail."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _frames(srt, ctx, preset, w, h, params, tail, frames=3, guide_bounces=None):
    b = srt.SceneBuilder()
    cam = b.add_preset(preset)
    scene = b.build(ctx)
    r = srt.Renderer(ctx, scene, w, h, params)
    r.set_tail(tail)
    if guide_bounces is not None:
        r.set_guide_bounces(guide_bounces)
    ctl = srt.CameraController(*cam)
    for f in range(frames):
        r.render(ctl.build_uniform(w / h, f))
    acc, st = r.read_accum(), r.stats()
    r.close()
    scene.close()
    return acc, st


@pytest.mark.parametrize("preset,depth", [(0, 12), (2, 8), (3, 12), (4, 16)])
@pytest.mark.parametrize("flags", [0, 2])  # graph, no graph
def test_tail_matches_bounce_by_bounce(srt, ctx, preset, depth, flags):
    p = srt.default_params(photons_per_frame=1 << 15, max_depth=depth, flags=flags)
    ref, st_ref = _frames(srt, ctx, preset, 48, 32, p, 0)
    assert st_ref["tail_first"] == depth
    for tail in (1, 4, 5):
        acc, st = _frames(srt, ctx, preset, 48, 32, p, tail)
        assert st["tail_first"] == tail
        np.testing.assert_array_equal(acc, ref)
        for k in ("rays_closest", "rays_shadow", "paths"):
            assert st[k] == st_ref[k], (tail, k)


def test_tail_stage_timing_and_counts(srt, ctx):
    p = srt.default_params(photons_per_frame=1 << 15, max_depth=12, flags=srt.FLAG_STAGE_TIMING | srt.FLAG_COUNT_VISITS)
    ref, st_ref = _frames(srt, ctx, 3, 48, 32, srt.default_params(photons_per_frame=1 << 15, max_depth=12), 0)
    acc, st = _frames(srt, ctx, 3, 48, 32, p, 5)
    np.testing.assert_array_equal(acc, ref)
    assert st["ms_tail"] > 0 and st["launches_trace_closest"] == 3 * 5
    assert st["rays_closest"] == st_ref["rays_closest"]


def test_guided_tail_after_the_guided_bounces(srt, ctx):
    """A guided renderer (frozen guide, so both runs see the same network)
    with guided bounces 0..2 and the tail from bounce 3 renders the frames of
    the same renderer bounce by bounce."""
    p = srt.default_params(photons_per_frame=1 << 14, max_depth=16, flags=srt.FLAG_GUIDING | srt.FLAG_GUIDE_FROZEN)
    ref, _ = _frames(srt, ctx, 4, 40, 24, p, 0, guide_bounces=3)
    acc, st = _frames(srt, ctx, 4, 40, 24, p, 3, guide_bounces=3)
    assert st["tail_first"] == 3
    np.testing.assert_array_equal(acc, ref)
    # guided bounces reaching the tail's first bounce: bounce by bounce
    _, st2 = _frames(srt, ctx, 4, 40, 24, p, 3, guide_bounces=4)
    assert st2["tail_first"] == 16


def test_automatic_tail_start(srt, ctx):
    """SRT_TAIL_AUTO (the default): after the first frame's path counts are
    back, the renderer starts the tail at the first bounce whose live paths
    fit in one wave of the tail kernel; a small image fits from bounce 1.  The
    image is that of the bounce-by-bounce frames, whenever the choice lands."""
    p = srt.default_params(photons_per_frame=1 << 15, max_depth=12)
    ref, _ = _frames(srt, ctx, 3, 48, 32, p, 0, frames=4)
    b = srt.SceneBuilder()
    cam = b.add_preset(3)
    scene = b.build(ctx)
    r = srt.Renderer(ctx, scene, 48, 32, p)
    ctl = srt.CameraController(*cam)
    r.render(ctl.build_uniform(1.5, 0))
    assert r.stats()["tail_first"] == 12  # bounce by bounce until the counts are read
    ctx.synchronize()
    for f in range(1, 4):
        r.render(ctl.build_uniform(1.5, f))
    assert r.stats()["tail_first"] == 1
    np.testing.assert_array_equal(r.read_accum(), ref)
    r.close()
    scene.close()


def test_automatic_tail_starts_after_the_guided_bounces(srt, ctx):
    """A guiding renderer's automatic tail starts after its guided bounces
    (default 8), and its frames equal the bounce-by-bounce ones (frozen guide)."""
    p = srt.default_params(photons_per_frame=1 << 14, max_depth=16, flags=srt.FLAG_GUIDING | srt.FLAG_GUIDE_FROZEN)
    ref, _ = _frames(srt, ctx, 4, 40, 24, p, 0, frames=4)
    b = srt.SceneBuilder()
    cam = b.add_preset(4)
    scene = b.build(ctx)
    r = srt.Renderer(ctx, scene, 40, 24, p)
    ctl = srt.CameraController(*cam)
    r.render(ctl.build_uniform(40 / 24, 0))
    ctx.synchronize()
    for f in range(1, 4):
        r.render(ctl.build_uniform(40 / 24, f))
    assert r.stats()["tail_first"] == 8
    np.testing.assert_array_equal(r.read_accum(), ref)
    r.close()
    scene.close()
