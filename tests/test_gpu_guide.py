"""Neural path guiding on the GPU against the FP64 guiding oracle: network
forward pass (bf16 tensor cores, fp32 accumulation), mixture density and
sampling, loss gradients of the fused forward/backward + weight-gradient
kernels, the Adam step, and the guided renderer (unbiased against plain
path tracing, frozen-weight determinism, checkpoint round trip)."""
from __future__ import annotations

import math

import numpy as np
import pytest

import guide_oracle as go

pytestmark = pytest.mark.gpu


def _weights(srt, seed, out_scale=1.0):
    w = srt.guide_default_weights(seed).astype(np.float64)
    rng = np.random.default_rng(seed)
    o4 = sum(fi * fo + fo for fi, fo in go.DIMS[:4])
    w[o4:o4 + 64 * 48] *= out_scale  # wider output range than the default init
    # non-zero biases exercise the bias paths
    o = 0
    for fi, fo in go.DIMS:
        o += fi * fo
        w[o:o + fo] += rng.uniform(-0.1, 0.1, fo)
        o += fo
    return w.astype(np.float32)


def _batch(rng, n):
    x = rng.uniform(0, 1, (n, 10)).astype(np.float32)
    om = rng.normal(size=(n, 3))
    om /= np.linalg.norm(om, axis=1, keepdims=True)
    pb = rng.uniform(0.05, 0.5, n).astype(np.float32)
    w = rng.exponential(1.0, n).astype(np.float32)
    return x, om.astype(np.float32), pb, w


@pytest.mark.parametrize("tcgen05", [False, True], ids=["mma_sync", "tcgen05"])
@pytest.mark.parametrize("n,out_scale", [(1, 1.0), (37, 1.0), (4096, 10.0), (100_003, 1.0)])
def test_forward_matches_oracle(srt, ctx, n, out_scale, tcgen05):
    rng = np.random.default_rng(n)
    w = _weights(srt, 7 + n, out_scale)
    x, _, _, _ = _batch(rng, n)
    y = srt.guide_forward(ctx, w, x, tcgen05=tcgen05)
    params = go.unpack(w)
    emu, _ = go.forward_bf16(params, x.astype(np.float64))
    ref, _ = go.forward(params, x.astype(np.float64))
    scale = max(1.0, np.abs(emu).max())
    # bf16 roundings repeated in the oracle: fp32 accumulation order remains,
    # and the rare activation that lands on the other side of a bf16 rounding
    # boundary (one bf16 ulp times its outgoing weights)
    err = np.abs(y - emu)
    assert np.median(err) <= 1e-6 * scale
    assert np.mean(err.max(1) > 1e-4 * scale) < 0.05  # samples touched by a flip
    assert err.max() <= 2e-2 * scale
    # plain FP64: the bf16 error budget of a 5-layer network
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 3e-2
    assert np.all(y[:, 41:] == y[:, 41:])  # finite padding outputs


@pytest.mark.parametrize("tc", [False, True], ids=["mma_sync", "tcgen05"])
def test_mixture_pdf_and_samples_match_oracle(srt, ctx, tc):
    rng = np.random.default_rng(11)
    n = 20_000
    raw = rng.normal(0, 1.5, (n, 48)).astype(np.float32)
    raw[:, 3:40:5] = rng.uniform(-5, 8, (n, 8))  # log kappa across and beyond the clamp
    om = rng.normal(size=(n, 3))
    om /= np.linalg.norm(om, axis=1, keepdims=True)
    u = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    out = srt.guide_mixture(ctx, raw, om.astype(np.float32), u, tcgen05=tc)
    mu, kappa, pi, _, _ = go.mixture(raw.astype(np.float64))
    q = (pi * go.vmf_pdf(mu, kappa, om[:, None, :].astype(np.float32).astype(np.float64))).sum(1)
    # exp(kappa (mu.w - 1)) with kappa up to e^7: fp32 dot products carry ~1e-4
    assert np.quantile(np.abs(out[:, 0] - q) / q, 0.999) < 2e-3
    j, d = go.mixture_sample(raw.astype(np.float64), u.astype(np.float64))
    np.testing.assert_allclose(np.linalg.norm(out[:, 1:], axis=1), 1.0, atol=1e-5)
    cos = np.sum(out[:, 1:] * d, axis=1)
    # a lobe choice on the cdf boundary may differ in fp32; everything else agrees
    assert np.mean(cos > 1 - 1e-4) > 0.999


@pytest.mark.parametrize("tc", [False, True], ids=["mma_sync", "tcgen05"])
def test_mixture_sampling_statistics(srt, ctx, tc):
    rng = np.random.default_rng(12)
    n = 200_000
    raw = np.zeros((n, 48), np.float32)
    raw[:, 4:40:5] = -30.0  # one dominant lobe (lobe 0)
    raw[:, 4] = 0.0
    raw[:, 0:3] = [0.3, -0.5, 0.8]
    kappa = 20.0
    raw[:, 3] = math.log(kappa)
    om = np.tile(np.array([0.0, 0.0, 1.0], np.float32), (n, 1))
    out = srt.guide_mixture(ctx, raw, om, rng.uniform(0, 1, (n, 3)).astype(np.float32), tcgen05=tc)
    mu = np.array([0.3, -0.5, 0.8]) / np.linalg.norm([0.3, -0.5, 0.8])
    mean_cos = (out[:, 1:] @ mu).mean()
    assert mean_cos == pytest.approx(1 / math.tanh(kappa) - 1 / kappa, abs=2e-3)


@pytest.mark.parametrize("tc", [False, True], ids=["mma_sync", "tcgen05"])
@pytest.mark.parametrize("n,out_scale", [(16, 1.0), (1000, 4.0), (65_536, 1.0)])
def test_gradients_match_oracle(srt, ctx, n, out_scale, tc):
    rng = np.random.default_rng(100 + n)
    w = _weights(srt, 3 + n, out_scale)
    x, om, pb, wt = _batch(rng, n)
    grad = srt.guide_train_step(ctx, w, x, om, pb, wt, adam=False, tcgen05=tc)
    params = go.unpack(w)
    raw16, ins = go.forward_bf16(params, x.astype(np.float64))
    _, gout16 = go.loss_and_output_grad(raw16, om.astype(np.float64), wt.astype(np.float64), pb.astype(np.float64))
    emu = go.flatten(go.backward_bf16(params, ins, gout16))
    raw, acts = go.forward(params, x.astype(np.float64))
    _, gout = go.loss_and_output_grad(raw, om.astype(np.float64), wt.astype(np.float64), pb.astype(np.float64))
    ref = go.flatten(go.backward(params, acts, gout))
    o = 0
    for li, (fi, fo) in enumerate(go.DIMS):
        for part, size in (("W", fi * fo), ("b", fo)):
            g, e = grad[o:o + size].astype(np.float64), emu[o:o + size]
            o += size
            err = np.linalg.norm(g - e) / max(np.linalg.norm(e), 1e-12)
            assert err < 2e-2, (li, part, err)
    cosine = grad @ ref / (np.linalg.norm(grad) * np.linalg.norm(ref))
    assert cosine > 0.99


def test_tcgen05_training_matches_mma_sync(srt, ctx):
    """The fused tcgen05 training step against the mma.sync kernels on the
    same records: the same bf16 products with FP32 accumulation in another
    summation order, so the gradients agree closely (relative Frobenius error
    per layer), and a renderer trained with it moves its weights like the
    mma.sync renderer does."""
    rng = np.random.default_rng(77)
    n = 40_000
    w = _weights(srt, 77)
    x, om, pb, wt = _batch(rng, n)
    g0 = srt.guide_train_step(ctx, w, x, om, pb, wt, adam=False)
    g1 = srt.guide_train_step(ctx, w, x, om, pb, wt, adam=False, tcgen05=True)
    o = 0
    for li, (fi, fo) in enumerate(go.DIMS):
        for part, size in (("W", fi * fo), ("b", fo)):
            a, b = g1[o:o + size].astype(np.float64), g0[o:o + size].astype(np.float64)
            o += size
            err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
            print(f"[parity] tcgen05 vs mma.sync gradient layer {li} {part}: {err:.2e}", flush=True)
            assert err < 1e-2, (li, part, err)
    # renderers: two frames of training each
    b_ = srt.SceneBuilder()
    cam = b_.add_preset(srt.PRESET_CORNELL_BOX)
    scene = b_.build(ctx)
    ctl = srt.CameraController(*cam)
    ws = []
    for kind in (srt.GUIDE_TRAIN_MMA_SYNC, srt.GUIDE_TRAIN_TCGEN05):
        r = srt.Renderer(ctx, scene, 64, 48, srt.default_params(photons_per_frame=1 << 14, flags=srt.FLAG_GUIDING))
        r.set_guide_training(kind)
        w0 = r.guide_weights()
        for f in range(2):
            r.render(ctl.build_uniform(64 / 48, f))
        ws.append(r.guide_weights() - w0)
        assert r.guide_info()["adam_steps"] == 2
        r.close()
    moved = np.abs(ws[0]) > 1e-6
    assert moved.mean() > 0.5
    close = np.abs(ws[1] - ws[0]) <= 0.02 * 1e-3 + 0.05 * np.abs(ws[0])
    assert close[moved].mean() > 0.95, close[moved].mean()
    scene.close()


def test_adam_step_matches_oracle(srt, ctx):
    rng = np.random.default_rng(21)
    n = 512
    w = _weights(srt, 21)
    x, om, pb, wt = _batch(rng, n)
    m = rng.normal(0, 1e-3, w.size).astype(np.float32)
    v = rng.uniform(0, 1e-5, w.size).astype(np.float32)
    step, lr = 6, 2e-3
    grad, pw, pm, pv = srt.guide_train_step(ctx, w, x, om, pb, wt, m, v, step, lr)
    params = go.unpack(w)
    g = go.unpack(grad.astype(np.float64) / n)
    mm, vv = go.unpack(m.astype(np.float64)), go.unpack(v.astype(np.float64))
    mlist = [[a, b] for a, b in mm]
    vlist = [[a, b] for a, b in vv]
    new = go.adam_step(params, g, mlist, vlist, step + 1, lr=lr)
    ref = np.concatenate([np.concatenate([W.reshape(-1), b]) for W, b in new])
    np.testing.assert_allclose(pw, ref, rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(pm, np.concatenate([np.concatenate([a.reshape(-1), b]) for a, b in mlist]),
                               rtol=1e-5, atol=1e-10)
    np.testing.assert_allclose(pv, np.concatenate([np.concatenate([a.reshape(-1), b]) for a, b in vlist]),
                               rtol=1e-5, atol=1e-12)


def _render(srt, ctx, scene, cam, w, h, flags, frames, weights=None, photons=0):
    p = srt.default_params(photons_per_frame=photons, flags=flags)
    r = srt.Renderer(ctx, scene, w, h, p)
    if weights is not None:
        r.set_guide_weights(weights)
    ctl = srt.CameraController(*cam)
    for f in range(frames):
        r.render(ctl.build_uniform(w / h, f))
    ctx.synchronize()
    return r


def test_guided_render_is_unbiased(srt, ctx):
    """Guided and plain path tracing converge to the same image (Cornell box)."""
    b = srt.SceneBuilder()
    cam = b.add_preset(srt.PRESET_CORNELL_BOX)
    scene = b.build(ctx)
    w, h, frames = 64, 48, 2048
    plain = _render(srt, ctx, scene, cam, w, h, srt.FLAG_FP64_ACCUM, frames)
    guided = _render(srt, ctx, scene, cam, w, h, srt.FLAG_FP64_ACCUM | srt.FLAG_GUIDING, frames)
    a = plain.read_accum64()
    g = guided.read_accum64()
    la = a[..., :3].sum(-1) / a[..., 3]
    lg = g[..., :3].sum(-1) / g[..., 3]
    assert lg.mean() == pytest.approx(la.mean(), rel=1e-2)
    # 8x8 blocks agree within their noise
    ba = la.reshape(h // 8, 8, w // 8, 8).mean((1, 3))
    bg = lg.reshape(h // 8, 8, w // 8, 8).mean((1, 3))
    assert np.median(np.abs(bg - ba) / np.maximum(ba, 1e-3)) < 0.02
    info = guided.guide_info()
    assert info["adam_steps"] == frames
    assert 0 < info["record_threshold"] <= 65536
    st = guided.stats()
    assert st["frames"] == frames
    wts = guided.guide_weights()
    assert np.all(np.isfinite(wts))
    assert not np.array_equal(wts, srt.guide_default_weights(1))  # it trained
    plain.close()
    guided.close()


def test_several_adam_steps_per_frame(srt, ctx):
    """srt_renderer_guide_set_steps: each frame's records split into strided
    sub-batches, one Adam step each; in a batch, scenes keep their own count."""
    b = srt.SceneBuilder()
    cam = b.add_preset(srt.PRESET_CORNELL_BOX)
    scene = b.build(ctx)
    w, h, frames = 48, 32, 6
    ctl = srt.CameraController(*cam)
    one = srt.Renderer(ctx, scene, w, h, srt.default_params(photons_per_frame=1 << 14, flags=srt.FLAG_GUIDING))
    four = srt.Renderer(ctx, scene, w, h, srt.default_params(photons_per_frame=1 << 14, flags=srt.FLAG_GUIDING))
    four.set_guide_steps(4)
    for f in range(frames):
        one.render(ctl.build_uniform(w / h, f))
        four.render(ctl.build_uniform(w / h, f))
    ctx.synchronize()
    assert one.guide_info()["adam_steps"] == frames
    assert four.guide_info()["adam_steps"] == 4 * frames
    w1, w4 = one.guide_weights(), four.guide_weights()
    w0 = srt.guide_default_weights(1)
    assert np.all(np.isfinite(w4))
    # Adam moves a parameter by at most ~lr per step: four steps per frame move further
    assert np.abs(w4 - w0).max() > 1.5 * np.abs(w1 - w0).max()
    with pytest.raises(srt.SrtError):
        one.set_guide_steps(0)
    one.close()
    four.close()
    params = [srt.default_params(photons_per_frame=1 << 14, flags=srt.FLAG_GUIDING) for _ in range(2)]
    batch = srt.Batch(ctx, [scene, scene], [(w, h), (32, 32)], params)
    batch.renderers[1].set_guide_steps(3)
    for f in range(2):
        batch.render([ctl.build_uniform(w / h, f), ctl.build_uniform(1.0, f)])
    ctx.synchronize()
    assert [x.guide_info()["adam_steps"] for x in batch.renderers] == [2, 6]
    batch.close()


def test_guide_training_state_checkpoint(srt, ctx):
    """srt_renderer_guide_get_state / set_state: weights, Adam moments and step
    count move to a new renderer unchanged, and its training counts on from
    there."""
    b = srt.SceneBuilder()
    cam = b.add_preset(srt.PRESET_CORNELL_BOX)
    scene = b.build(ctx)
    w, h = 48, 32
    trained = _render(srt, ctx, scene, cam, w, h, srt.FLAG_GUIDING, 8)
    st = trained.guide_state()
    assert st["adam_step"] == 8 and np.any(st["adam_m"] != 0) and np.all(st["adam_v"] >= 0)
    np.testing.assert_array_equal(st["params"], trained.guide_weights())
    r = _render(srt, ctx, scene, cam, w, h, srt.FLAG_GUIDING, 0)
    r.set_guide_state(st)
    back = r.guide_state()
    for k in ("params", "adam_m", "adam_v"):
        np.testing.assert_array_equal(back[k], st[k])
    assert back["adam_step"] == 8 and r.guide_info()["adam_steps"] == 8
    ctl = srt.CameraController(*cam)
    for f in range(8, 10):
        r.render(ctl.build_uniform(w / h, f))
    ctx.synchronize()
    assert r.guide_info()["adam_steps"] == 10
    assert np.all(np.isfinite(r.guide_weights()))
    trained.close()
    r.close()


def test_frozen_guide_is_deterministic_and_restores(srt, ctx):
    b = srt.SceneBuilder()
    cam = b.add_preset(srt.PRESET_CORNELL_BOX)
    scene = b.build(ctx)
    w, h = 48, 32
    trained = _render(srt, ctx, scene, cam, w, h, srt.FLAG_GUIDING, 64)
    ckpt = trained.guide_weights()
    flags = srt.FLAG_GUIDING | srt.FLAG_GUIDE_FROZEN
    r1 = _render(srt, ctx, scene, cam, w, h, flags, 8, weights=ckpt)
    r2 = _render(srt, ctx, scene, cam, w, h, flags | srt.FLAG_NO_GRAPH, 8, weights=ckpt)
    np.testing.assert_array_equal(r1.read_accum(), r2.read_accum())
    np.testing.assert_array_equal(r1.guide_weights(), ckpt)  # frozen: no update
    assert r1.guide_info()["adam_steps"] == 0
    for r in (trained, r1, r2):
        r.close()


def test_guiding_rejects_ray_sort(srt, ctx):
    b = srt.SceneBuilder()
    b.add_preset(srt.PRESET_CORNELL_BOX)
    scene = b.build(ctx)
    with pytest.raises(RuntimeError):
        srt.Renderer(ctx, scene, 16, 16, srt.default_params(flags=srt.FLAG_GUIDING | srt.FLAG_RAY_SORT))


def test_trained_guide_reduces_error(srt, ctx):
    """What the guide gains: on a room lit only through a small ceiling spot,
    guided path tracing (learning online from frame 0) reaches a lower error
    than plain path tracing at the same sample count, against a 16384-spp FP64
    reference on decorrelated sample streams.  The per-pixel relative squared
    error is heavy-tailed (a few firefly pixels carry up to half of the mean,
    so the mean moves between runs of the online training), so the test
    compares its median (measured gain 1.9x) and its mean without the worst
    1 % of pixels (measured gain 1.25-1.55x)."""
    b = srt.SceneBuilder()
    cam = b.add_preset(srt.PRESET_INDIRECT_ROOM)
    scene = b.build(ctx)
    w, h = 64, 48
    ctl = srt.CameraController(*cam)

    def run(flags, frames, seed=0):
        p = srt.default_params(photons_per_frame=0, flags=flags | srt.FLAG_FP64_ACCUM, seed=seed)
        r = srt.Renderer(ctx, scene, w, h, p)
        for f in range(frames):
            r.render(ctl.build_uniform(w / h, f))
        a = r.read_accum64()
        r.close()
        return a[..., :3] / a[..., 3:4]

    ref = run(0, 16384, seed=0x5EED0001)
    plain = run(0, 1024)
    guided = run(srt.FLAG_GUIDING, 1024)
    def errors(x):
        e = np.sort(np.mean((x - ref) ** 2 / (ref ** 2 + 0.01), axis=-1).ravel())
        return float(np.median(e)), float(e[:int(0.99 * e.size)].mean())

    med_p, trim_p = errors(plain)
    med_g, trim_g = errors(guided)
    assert med_g * 1.4 < med_p, (med_p, med_g)
    assert trim_g * 1.1 < trim_p, (trim_p, trim_g)


def test_tcgen05_and_mma_sync_inference_agree(srt, ctx):
    """The two inference kernels (tcgen05 MMAs into tensor memory, and
    mma.sync fragments) run the same frozen network: their raw outputs agree
    to FP32 summation order, so the guided images agree up to the rare
    sampling decision that flips."""
    b = srt.SceneBuilder()
    cam = b.add_preset(srt.PRESET_CORNELL_BOX)
    scene = b.build(ctx)
    trained = _render(srt, ctx, scene, cam, 48, 32, srt.FLAG_GUIDING, 64)
    ckpt = trained.guide_weights()
    flags = srt.FLAG_GUIDING | srt.FLAG_GUIDE_FROZEN | srt.FLAG_FP64_ACCUM
    out = []
    for kind in (srt.GUIDE_INFER_TCGEN05, srt.GUIDE_INFER_MMA_SYNC):
        p = srt.default_params(photons_per_frame=0, flags=flags)
        r = srt.Renderer(ctx, scene, 48, 32, p)
        r.set_guide_weights(ckpt)
        r.set_guide_inference(kind)
        ctl = srt.CameraController(*cam)
        for f in range(64):
            r.render(ctl.build_uniform(48 / 32, f))
        a = r.read_accum64()
        out.append(a[..., :3] / a[..., 3:4])
        r.close()
    tc, mma = out
    close = np.all(np.abs(tc - mma) <= 1e-4 * np.maximum(np.abs(mma), 1e-3), axis=-1)
    assert np.mean(close) > 0.9
    assert tc.mean() == pytest.approx(mma.mean(), rel=5e-3)
    trained.close()
