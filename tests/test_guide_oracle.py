"""The FP64 guiding oracle checks itself: analytic loss gradients against
central finite differences, the mixture density's normalisation, the vMF
sampler's mean cosine, and the bf16 emulation against plain FP64.  CPU only."""
from __future__ import annotations

import math

import numpy as np
import pytest

import guide_oracle as go


def _params(rng, out_scale=1.0):
    flat = np.zeros(go.N_PARAMS)
    o = 0
    for li, (fi, fo) in enumerate(go.DIMS):
        a = math.sqrt(6.0 / fi) * (out_scale if li == 4 else 1.0)
        flat[o:o + fi * fo] = rng.uniform(-a, a, fi * fo)
        o += fi * fo
        flat[o:o + fo] = rng.uniform(-0.1, 0.1, fo)
        o += fo
    return go.unpack(flat)


def _batch(rng, n):
    x = rng.uniform(0, 1, (n, 10))
    om = rng.normal(size=(n, 3))
    om /= np.linalg.norm(om, axis=1, keepdims=True)
    pb = rng.uniform(0.05, 0.5, n)
    w = rng.exponential(1.0, n)
    return x, om, pb, w


def _surrogate(raw, raw0, om, pb, w):
    """Per-sample loss whose gradient the oracle defines: -w log q(raw) -
    w log(sel(raw) q(raw0) + (1 - sel(raw)) pb), q held at raw0 in the second
    term (the selection output learns against the current mixture)."""
    mu, kappa, pi, sel, _ = go.mixture(raw)
    q = (pi * go.vmf_pdf(mu, kappa, om[:, None, :])).sum(1)
    mu0, k0, pi0, _, _ = go.mixture(raw0)
    q0 = (pi0 * go.vmf_pdf(mu0, k0, om[:, None, :])).sum(1)
    return -w * np.log(q) - w * np.log(sel * q0 + (1 - sel) * pb)


def _total_loss(params, params0, x, om, pb, w):
    raw, _ = go.forward(params, x)
    raw0, _ = go.forward(params0, x)
    return _surrogate(raw, raw0, om, pb, w).sum()


def test_output_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    n = 16
    raw = rng.normal(0, 1.0, (n, 48))
    _, om, pb, w = _batch(rng, n)
    _, g = go.loss_and_output_grad(raw, om, w, pb)
    h = 1e-6
    for i in range(48):
        if i in range(41, 48):  # unused outputs
            assert np.all(g[:, i] == 0.0)
            continue
        rp, rm = raw.copy(), raw.copy()
        rp[:, i] += h
        rm[:, i] -= h
        fd = (_surrogate(rp, raw, om, pb, w) - _surrogate(rm, raw, om, pb, w)) / (2 * h)
        np.testing.assert_allclose(g[:, i], fd, rtol=1e-5, atol=1e-7)


def test_parameter_gradient_matches_finite_differences():
    rng = np.random.default_rng(2)
    params = _params(rng, out_scale=1.0)
    x, om, pb, w = _batch(rng, 8)
    raw, acts = go.forward(params, x)
    _, gout = go.loss_and_output_grad(raw, om, w, pb)
    grads = go.backward(params, acts, gout)
    h = 1e-6
    for li in range(5):
        W, b = params[li]
        for _ in range(6):
            o, i = rng.integers(W.shape[0]), rng.integers(W.shape[1])
            Wp = [(a.copy(), c.copy()) for a, c in params]
            Wm = [(a.copy(), c.copy()) for a, c in params]
            Wp[li][0][o, i] += h
            Wm[li][0][o, i] -= h
            fd = (_total_loss(Wp, params, x, om, pb, w) - _total_loss(Wm, params, x, om, pb, w)) / (2 * h)
            assert grads[li][0][o, i] == pytest.approx(fd, rel=1e-4, abs=1e-7)
        o = rng.integers(b.shape[0])
        bp = [(a.copy(), c.copy()) for a, c in params]
        bm = [(a.copy(), c.copy()) for a, c in params]
        bp[li][1][o] += h
        bm[li][1][o] -= h
        fd = (_total_loss(bp, params, x, om, pb, w) - _total_loss(bm, params, x, om, pb, w)) / (2 * h)
        assert grads[li][1][o] == pytest.approx(fd, rel=1e-4, abs=1e-7)


def test_mixture_density_integrates_to_one():
    rng = np.random.default_rng(3)
    raw = rng.normal(0, 1.5, (4, 48))
    mu, kappa, pi, _, _ = go.mixture(raw)
    # Fibonacci sphere quadrature
    m = 400_000
    k = np.arange(m) + 0.5
    z = 1 - 2 * k / m
    phi = math.pi * (1 + 5 ** 0.5) * k
    r = np.sqrt(1 - z * z)
    dirs = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
    for s in range(4):
        pdf = (pi[s][None] * go.vmf_pdf(mu[s][None], kappa[s][None], dirs[:, None, :])).sum(1)
        assert pdf.mean() * 4 * math.pi == pytest.approx(1.0, rel=2e-3)


@pytest.mark.parametrize("kappa", [0.05, 1.0, 20.0, 1000.0])
def test_vmf_sampler_mean_cosine(kappa):
    rng = np.random.default_rng(4)
    n = 200_000
    mu = np.array([0.3, -0.5, 0.8])
    mu /= np.linalg.norm(mu)
    d = go.vmf_sample(np.broadcast_to(mu, (n, 3)), kappa, rng.uniform(size=n), rng.uniform(size=n))
    np.testing.assert_allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-12)
    expected = 1.0 / math.tanh(kappa) - 1.0 / kappa
    assert (d @ mu).mean() == pytest.approx(expected, abs=4e-3)


def test_bf16_emulation_close_to_fp64():
    rng = np.random.default_rng(5)
    params = _params(rng)
    x, om, pb, w = _batch(rng, 256)
    raw, acts = go.forward(params, x)
    raw16, ins = go.forward_bf16(params, x)
    assert np.linalg.norm(raw16 - raw) / np.linalg.norm(raw) < 2e-2
    _, g = go.loss_and_output_grad(raw, om, w, pb)
    _, g16 = go.loss_and_output_grad(raw16, om, w, pb)
    a = go.flatten(go.backward(params, acts, g))
    b = go.flatten(go.backward_bf16(params, ins, g16))
    assert a @ b / (np.linalg.norm(a) * np.linalg.norm(b)) > 0.99
