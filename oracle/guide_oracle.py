"""FP64 CPU oracle of the neural path-guiding network (numpy).

TEST INFRASTRUCTURE ONLY: the oracle for the CUDA guiding kernels.  The
reference has no path guiding; this restates the project's own definition of
the network, the vMF mixture and the training loss in float64, so that the
GPU's forward outputs, mixture pdfs, loss gradients and Adam steps can be
compared with an independent implementation.

Network: 10 inputs -> frequency encoding (6 octaves, sin and cos of
2^k * pi * x for each input, 120 features, zero-padded to 128) -> 64 -> 64
-> 64 -> 64 (ReLU) -> 48 linear outputs.  Output layout: lobe j (0..7) uses
r[5j..5j+2] (direction, normalised), r[5j+3] (log kappa, clamped to [-4, 7]),
r[5j+4] (mixture logit); r[40] is the selection logit:
sel = 0.05 + 0.85 * sigmoid(r[40]).  Weights W_l are [out, in] row-major.
"""
from __future__ import annotations

import math

import numpy as np

N_IN = 10
N_FREQ = 6
ENC = 128
HID = 64
OUT = 48
LOBES = 8
DIMS = [(ENC, HID), (HID, HID), (HID, HID), (HID, HID), (HID, OUT)]
KAPPA_LO, KAPPA_HI = -4.0, 7.0
SEL_LO, SEL_SPAN = 0.05, 0.85


def encode(x: np.ndarray) -> np.ndarray:
    """x: [n, 10] in roughly [0, 1] -> [n, 128]; feature 12*d + 2*k + {0: sin, 1: cos}."""
    n = x.shape[0]
    e = np.zeros((n, ENC), np.float64)
    for d in range(N_IN):
        for k in range(N_FREQ):
            a = (2.0 ** k) * math.pi * x[:, d]
            e[:, 12 * d + 2 * k] = np.sin(a)
            e[:, 12 * d + 2 * k + 1] = np.cos(a)
    return e


def forward(params, x: np.ndarray):
    """params: list of (W [out, in], b [out]).  Returns (raw outputs, activations)."""
    a = encode(x)
    acts = [a]
    for li, (W, b) in enumerate(params):
        z = a @ W.T + b
        a = np.maximum(z, 0.0) if li < 4 else z
        acts.append(a)
    return a, acts


def mixture(raw: np.ndarray):
    """raw [n, 48] -> (mu [n, 8, 3], kappa [n, 8], pi [n, 8], sel [n], internals)."""
    v = raw[:, :40].reshape(-1, LOBES, 5)
    dirv = v[:, :, 0:3]
    norm = np.maximum(np.linalg.norm(dirv, axis=2), 1e-12)
    mu = dirv / norm[..., None]
    lk = np.clip(v[:, :, 3], KAPPA_LO, KAPPA_HI)
    kappa = np.exp(lk)
    logit = v[:, :, 4]
    w = np.exp(logit - logit.max(1, keepdims=True))
    pi = w / w.sum(1, keepdims=True)
    s = 1.0 / (1.0 + np.exp(-raw[:, 40]))
    sel = SEL_LO + SEL_SPAN * s
    return mu, kappa, pi, sel, (norm, v[:, :, 3], s)


def vmf_pdf(mu, kappa, w):
    """mu [.., 3], kappa [..], w [.., 3] -> density on the unit sphere."""
    c = kappa / (2.0 * math.pi * (-np.expm1(-2.0 * kappa)))
    return c * np.exp(kappa * ((mu * w).sum(-1) - 1.0))


def loss_and_output_grad(raw, omega, weight, pdf_bsdf):
    """Per-sample loss L = -weight * log q(omega) - weight * log p_mix(omega)
    (the second term only moves the selection output) and dL/draw [n, 48]."""
    mu, kappa, pi, sel, (norm, lk_raw, s) = mixture(raw)
    vm = vmf_pdf(mu, kappa, omega[:, None, :])  # [n, 8]
    q = (pi * vm).sum(1)
    pmix = sel * q + (1.0 - sel) * pdf_bsdf
    loss = -weight * np.log(q) - weight * np.log(pmix)
    g = np.zeros_like(raw)
    gamma = pi * vm / q[:, None]
    wq = weight[:, None]
    # logits
    glogit = wq * (pi - gamma)
    # kappa (through exp, zero outside the clamp)
    mw = (mu * omega[:, None, :]).sum(-1)
    dlog_dk = 1.0 / kappa - 2.0 / np.expm1(2.0 * kappa) + mw - 1.0
    gk = -wq * gamma * dlog_dk * kappa
    inside = (lk_raw > KAPPA_LO) & (lk_raw < KAPPA_HI)
    gk = np.where(inside, gk, 0.0)
    # direction (through normalisation)
    gdir = -(wq * gamma * kappa)[..., None] * (omega[:, None, :] - mw[..., None] * mu) / norm[..., None]
    v = np.zeros((raw.shape[0], LOBES, 5))
    v[:, :, 0:3] = gdir
    v[:, :, 3] = gk
    v[:, :, 4] = glogit
    g[:, :40] = v.reshape(-1, 40)
    dsel = -weight * (q - pdf_bsdf) / pmix
    g[:, 40] = dsel * SEL_SPAN * s * (1.0 - s)
    return loss, g


def backward(params, acts, gout):
    """Weight and bias gradients summed over the batch."""
    grads = [None] * 5
    delta = gout
    for li in range(4, -1, -1):
        W, b = params[li]
        a_prev = acts[li]
        grads[li] = (delta.T @ a_prev, delta.sum(0))
        if li > 0:
            delta = (delta @ W) * (acts[li] > 0.0)
    return grads


def adam_step(params, grads, m, v, t, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    out = []
    for li in range(5):
        W, b = params[li]
        gW, gb = grads[li]
        nw = []
        for k, (p, g) in enumerate(((W, gW), (b, gb))):
            m[li][k] = b1 * m[li][k] + (1 - b1) * g
            v[li][k] = b2 * v[li][k] + (1 - b2) * g * g
            mh = m[li][k] / (1 - b1 ** t)
            vh = v[li][k] / (1 - b2 ** t)
            nw.append(p - lr * mh / (np.sqrt(vh) + eps))
        out.append(tuple(nw))
    return out


def unpack(flat: np.ndarray):
    """Flat float parameter vector (W0, b0, W1, b1, ...) -> list of (W, b)."""
    params, o = [], 0
    for fi, fo in DIMS:
        W = flat[o:o + fi * fo].reshape(fo, fi).astype(np.float64)
        o += fi * fo
        b = flat[o:o + fo].astype(np.float64)
        o += fo
        params.append((W, b))
    return params


N_PARAMS = sum(fi * fo + fo for fi, fo in DIMS)


# --------------------------------------------------------------------------- bf16 emulation
# The GPU rounds the encoding, the hidden activations, the output gradient
# and the hidden deltas to bf16 (round to nearest even) and accumulates
# products in fp32.  These helpers repeat those roundings in float64 so
# that the remaining difference is accumulation order alone.


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to the nearest bf16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def encode_f32(x: np.ndarray) -> np.ndarray:
    """The encoding as the GPU evaluates it in fp32: octave 0 = sin, cos of
    pi x rounded to fp32; octave k + 1 from octave k by the double-angle
    identities with the GPU's roundings: sin' = f32(f32(2 s) c), cos' =
    f32(c c - f32(s s)) (one fused multiply-add)."""
    n = x.shape[0]
    e = np.zeros((n, ENC), np.float64)
    for d in range(N_IN):
        xd = x[:, d].astype(np.float32).astype(np.float64)
        s = np.sin(math.pi * xd).astype(np.float32)
        c = np.cos(math.pi * xd).astype(np.float32)
        for k in range(N_FREQ):
            e[:, 12 * d + 2 * k] = s
            e[:, 12 * d + 2 * k + 1] = c
            s2 = ((np.float32(2.0) * s) * c).astype(np.float32)
            ss = (s * s).astype(np.float32)
            c2 = (c.astype(np.float64) * c.astype(np.float64) - ss.astype(np.float64)).astype(np.float32)
            s, c = s2, c2
    return e


def forward_bf16(params, x: np.ndarray):
    """Forward pass with the GPU's encoding and bf16 roundings.  Returns (raw, layer inputs)."""
    a = bf16(encode_f32(x))
    ins = [a]
    for li, (W, b) in enumerate(params):
        z = a @ bf16(W).T + b.astype(np.float32).astype(np.float64)
        if li < 4:
            a = bf16(np.maximum(z, 0.0))
            ins.append(a)
        else:
            a = z
    return a, ins


def backward_bf16(params, ins, gout):
    """Weight and bias gradients with the GPU's bf16 roundings of the deltas."""
    grads = [None] * 5
    delta = bf16(gout)
    for li in range(4, -1, -1):
        W, _ = params[li]
        grads[li] = (delta.T @ ins[li], delta.sum(0))
        if li > 0:
            delta = bf16((delta @ bf16(W)) * (ins[li] > 0.0))
    return grads


def flatten(grads) -> np.ndarray:
    return np.concatenate([np.concatenate([gW.reshape(-1), gb]) for gW, gb in grads])


def vmf_sample(mu, kappa, u1, u2):
    """Direction of one vMF lobe: w = 1 + log(u1 + (1 - u1) exp(-2 kappa)) / kappa
    (inverse CDF of the cosine, the stable form of Wood's method), azimuth
    2 pi u2 in the frame b1 = normalize(mu x t), b2 = mu x b1 with
    t = (0, 1, 0) when |mu.x| > 0.9, else (1, 0, 0)."""
    mu = np.asarray(mu, np.float64)
    w = np.clip(1.0 + np.log(u1 + (1.0 - u1) * np.exp(-2.0 * kappa)) / kappa, -1.0, 1.0)
    r = np.sqrt(np.maximum(0.0, 1.0 - w * w))
    t = np.where(np.abs(mu[..., :1]) > 0.9, np.array([0.0, 1.0, 0.0]), np.array([1.0, 0.0, 0.0]))
    b1 = np.cross(mu, t)
    b1 /= np.linalg.norm(b1, axis=-1, keepdims=True)
    b2 = np.cross(mu, b1)
    phi = 2.0 * math.pi * u2
    d = mu * w[..., None] + b1 * (r * np.cos(phi))[..., None] + b2 * (r * np.sin(phi))[..., None]
    return d / np.linalg.norm(d, axis=-1, keepdims=True)


def mixture_sample(raw, u):
    """raw [n, 48], u [n, 3] -> (lobe index, direction [n, 3]): lobe = first j
    with u0 < cumulative pi_j, then vmf_sample with (u1, u2)."""
    mu, kappa, pi, _, _ = mixture(raw)
    cdf = np.cumsum(pi, 1)
    j = np.minimum((u[:, :1] >= cdf).sum(1), LOBES - 1)
    idx = np.arange(len(raw))
    return j, vmf_sample(mu[idx, j], kappa[idx, j], u[:, 1], u[:, 2])
