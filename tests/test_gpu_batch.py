"""Batched rendering (srt_batch_*): scenes of uneven size in one CUDA graph per
iteration, their rays traced in shared launches, give the same images as
rendering each scene alone; inactive scenes are left untouched; the
autotuner picks one of its candidates and clears the tuning frames."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scenes(srt, ctx):
    out = []
    for preset in (srt.PRESET_CORNELL_BOX, srt.PRESET_CONFIG1, srt.PRESET_CAUSTIC_SLAB):
        b = srt.SceneBuilder()
        cam = b.add_preset(preset)
        out.append((b.build(ctx), srt.CameraController(*cam)))
    return out


SIZES = [(64, 48), (96, 64), (80, 80)]


def _params(srt):
    return [srt.default_params(photons_per_frame=1 << 16, max_depth=8),
            srt.default_params(photons_per_frame=1 << 15),
            srt.default_params(photons_per_frame=1 << 16, max_depth=16, seed=7)]


def _cams(ctls, frame):
    return [c.build_uniform(w / h, frame) for c, (w, h) in zip(ctls, SIZES)]


def test_batch_matches_single_scene_renders(srt, ctx):
    sc = _scenes(srt, ctx)
    scenes, ctls = [s for s, _ in sc], [c for _, c in sc]
    params = _params(srt)
    batch = srt.Batch(ctx, scenes, SIZES, params)
    frames = 4
    for f in range(frames):
        batch.render(_cams(ctls, f))
    ctx.synchronize()
    for i, (scene, (w, h)) in enumerate(zip(scenes, SIZES)):
        r = srt.Renderer(ctx, scene, w, h, params[i])
        for f in range(frames):
            r.render(ctls[i].build_uniform(w / h, f))
        ref = r.read_accum()
        got = batch.renderers[i].read_accum()
        np.testing.assert_array_equal(got, ref)
        np.testing.assert_array_equal(batch.renderers[i].read_ldr(), r.read_ldr())
        st = batch.renderers[i].stats()
        assert st["frames"] == frames and st["paths"] == frames * w * h
        r.close()
    # an inactive scene keeps its image
    before = batch.renderers[1].read_accum()
    batch.render(_cams(ctls, frames), active=[1, 0, 1])
    ctx.synchronize()
    np.testing.assert_array_equal(batch.renderers[1].read_accum(), before)
    assert batch.renderers[0].stats()["frames"] == frames + 1
    assert batch.renderers[1].stats()["frames"] == frames
    batch.close()


def test_batch_scene_matches_oracle(srt, orc, ctx):
    """One scene of a batch (config 1, 96x64) against the CPU oracle frame by
    frame, on the photon set the batch's photon pass produced: the same
    per-pixel agreement as single-scene frames."""
    from conftest import rel_err, relmse

    sc = _scenes(srt, ctx)
    scenes, ctls = [s for s, _ in sc], [c for _, c in sc]
    params = _params(srt)
    batch = srt.Batch(ctx, scenes, SIZES, params)
    k = 1
    w, h = SIZES[k]
    b = srt.SceneBuilder()
    b.add_preset(srt.PRESET_CONFIG1)
    o = orc.OracleScene(b.arrays())
    acc_o = np.zeros((h, w, 4), np.float32)
    frames = 2
    for f in range(frames):
        cams = _cams(ctls, f)
        batch.render(cams)
        ph = batch.renderers[k].read_photons()
        acc_o, _, _, _ = o.render_frame(cams[k], w, h, params[k], acc_o, want_ldr=False, photons=ph)
    acc_g = batch.renderers[k].read_accum()
    e = rel_err(acc_g[..., :3], acc_o[..., :3], floor=1e-3)
    pix_ok = (e < 1e-3).all(-1)
    rm = relmse(acc_g[..., :3] / frames, acc_o[..., :3] / frames)
    print(f"[parity] batch scene {k}: pixels agreeing {pix_ok.mean():.5f}, relMSE {rm:.3e}", flush=True)
    assert pix_ok.mean() >= 0.99
    assert rm < 1e-4
    batch.close()
    o.close()


def test_batch_autotune(srt, ctx):
    sc = _scenes(srt, ctx)
    scenes, ctls = [s for s, _ in sc], [c for _, c in sc]
    batch = srt.Batch(ctx, scenes, SIZES, _params(srt))
    t = batch.autotune(_cams(ctls, 0), iterations=1)
    # 3 resident-block settings of the persistent traversal (which hands rays
    # out lane by lane: the chunk is no knob), then the trees rebuilt with 4
    # children per node
    assert t["candidates"] == 4
    assert t["blocks_per_sm"] in (2, 4, 8) and t["chunk"] == 32
    assert t["bvh_width"] in (4, 8)
    assert all(s.info()["width"] == t["bvh_width"] for s in scenes)
    assert t["ms_per_iteration"] > 0
    assert batch.tuning()["chunk"] == t["chunk"]
    for r in batch.renderers:
        assert not np.any(r.read_accum())  # tuning frames cleared
        assert r.stats()["frames"] == 0
    batch.render(_cams(ctls, 0))
    ctx.synchronize()
    assert all(r.stats()["frames"] == 1 for r in batch.renderers)
    with pytest.raises(srt.SrtError):
        batch.renderers[0].render(_cams(ctls, 1)[0])
    batch.close()


def test_handles_destroyed_in_any_order(srt):
    """The context outlives its scenes, renderers and batches whatever the
    order of the destroy calls (garbage collectors pick their own order)."""
    ctx = srt.Context(0)
    b = srt.SceneBuilder()
    cam = b.add_preset(srt.PRESET_CORNELL_BOX)
    scene = b.build(ctx)
    r = srt.Renderer(ctx, scene, 32, 24, srt.default_params(photons_per_frame=1 << 12))
    batch = srt.Batch(ctx, [scene], [(16, 16)], [srt.default_params(photons_per_frame=1 << 12)])
    r.render(srt.CameraController(*cam).build_uniform(32 / 24, 0))
    batch.render([srt.CameraController(*cam).build_uniform(1.0, 0)])
    ctx.close()  # deferred: children alive
    img = r.read_accum()
    assert img.shape == (24, 32, 4) and np.all(np.isfinite(img))
    scene.close()
    batch.close()
    r.close()


def _guided(srt, p, frozen):
    p.flags |= srt.FLAG_GUIDING | (srt.FLAG_GUIDE_FROZEN if frozen else 0)
    return p


def test_batch_guided_matches_single_scene_renders(srt, ctx):
    """Guided scenes of a batch have their Lambert continuations sampled by one
    grouped tcgen05 launch per bounce, whose tiles load the network of their
    own scene; with frozen networks (a different one per scene) the images
    equal those of the same renderers rendered alone.  The middle scene is
    plain (a mixed batch)."""
    sc = _scenes(srt, ctx)
    scenes, ctls = [s for s, _ in sc], [c for _, c in sc]
    params = _params(srt)
    params[0] = _guided(srt, params[0], True)
    params[2] = _guided(srt, params[2], True)
    weights = {0: srt.guide_default_weights(11), 2: srt.guide_default_weights(12)}
    batch = srt.Batch(ctx, scenes, SIZES, params)
    for i, w in weights.items():
        batch.renderers[i].set_guide_weights(w)
    frames = 3
    for f in range(frames):
        batch.render(_cams(ctls, f))
    ctx.synchronize()
    for i, (scene, (w, h)) in enumerate(zip(scenes, SIZES)):
        r = srt.Renderer(ctx, scene, w, h, params[i])
        if i in weights:
            r.set_guide_weights(weights[i])
        for f in range(frames):
            r.render(ctls[i].build_uniform(w / h, f))
        np.testing.assert_array_equal(batch.renderers[i].read_accum(), r.read_accum())
        r.close()
    batch.close()


def test_batch_guided_training_matches_single_scene_training(srt, ctx):
    """The grouped training step (targets, forward/backward, weight gradients,
    Adam: one launch each for all guided scenes) moves every scene's network
    as the single-renderer step does: after one frame the two updates agree
    up to the summation order of the gradients (Adam's first step is
    lr * g / (|g| + eps), so only parameters with |g| near eps may differ)."""
    sc = _scenes(srt, ctx)
    scenes, ctls = [s for s, _ in sc], [c for _, c in sc]
    params = [_guided(srt, p, False) for p in _params(srt)]
    lr = 1e-4
    w0 = [srt.guide_default_weights(21 + i) for i in range(3)]
    batch = srt.Batch(ctx, scenes, SIZES, params)
    for i, x in enumerate(batch.renderers):
        x.set_guide_weights(w0[i])
        x.configure_guide(lr=lr)
    batch.render(_cams(ctls, 0))
    ctx.synchronize()
    for i, (scene, (w, h)) in enumerate(zip(scenes, SIZES)):
        r = srt.Renderer(ctx, scene, w, h, params[i])
        r.set_guide_weights(w0[i])
        r.configure_guide(lr=lr)
        r.render(ctls[i].build_uniform(w / h, 0))
        ref, got = r.guide_weights(), batch.renderers[i].guide_weights()
        assert r.guide_info()["adam_steps"] == 1
        assert batch.renderers[i].guide_info()["adam_steps"] == 1
        moved = np.abs(ref - w0[i]) > 0.5 * lr
        assert moved.mean() > 0.1
        d = np.abs(got - ref)
        assert d.max() <= 2 * lr + 1e-6
        assert (d[moved] <= 1e-2 * lr).mean() > 0.99
        r.close()
    for f in range(1, 4):
        batch.render(_cams(ctls, f))
    ctx.synchronize()
    for x in batch.renderers:
        assert x.guide_info()["adam_steps"] == 4
        assert np.all(np.isfinite(x.read_accum()))
    batch.close()


def test_batch_autotune_leaves_guided_networks_untouched(srt, ctx):
    """The tuning frames train nothing: a guided scene's weights and Adam step
    count are the same before and after srt_batch_autotune."""
    sc = _scenes(srt, ctx)
    scenes, ctls = [s for s, _ in sc], [c for _, c in sc]
    params = [_guided(srt, p, False) for p in _params(srt)]
    batch = srt.Batch(ctx, scenes, SIZES, params)
    batch.render(_cams(ctls, 0))  # one trained iteration first
    ctx.synchronize()
    before = [(x.guide_weights(), x.guide_info()["adam_steps"]) for x in batch.renderers]
    assert all(steps == 1 for _, steps in before)
    batch.autotune(_cams(ctls, 1), iterations=1)
    for x, (w, steps) in zip(batch.renderers, before):
        np.testing.assert_array_equal(x.guide_weights(), w)
        assert x.guide_info()["adam_steps"] == steps
    batch.render(_cams(ctls, 2))
    ctx.synchronize()
    assert all(x.guide_info()["adam_steps"] == 2 for x in batch.renderers)
    batch.close()
