"""Generates tests/golden/golden.json: known-answer vectors for the oracle.

The reference (Rust + WGSL on a Vulkan ray-query device) cannot run here and
ships no tests or fixtures, so these vectors come from an independent numpy
restatement of the reference formulas, written separately from the C++
oracle, plus closed forms:

  pcg_hash / rand           shader.wgsl:144-160 (u32 arithmetic mod 2^32)
  camera rng seeds          shader.wgsl:146-148, photon_emit.wgsl:66-70
  grid jitter + hash        build_grid.wgsl:25-52 in float32, bit-exact
  sorted cell keys          (hash << 32) | photon index, stable by index
  sample_cie_xyz            shader.wgsl:85-97 in float64
  blackbody_radiance        shader.wgsl:128-139 in float64; Wien peak
  Airy thin film            closed forms at normal incidence: invisible film
                            (n2 = n1), quarter-wave and half-wave layers
  Cauchy hero pdf           shader.wgsl:782-797 in float64

Run:  python tests/golden/make_golden.py   (rewrites golden.json)
"""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np

M32 = 0xFFFFFFFF


def pcg_hash(x: int) -> int:
    state = (x * 747796405 + 2891336453) & M32
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & M32
    return ((word >> 22) ^ word) & M32


def rand_f32(seed: int):
    s = pcg_hash(seed)
    return s, np.float32(s) / np.float32(4294967295.0)


def jitter(frame: int, cell: np.float32):
    seed = pcg_hash((frame * 114514) & M32)
    r = [np.float32(np.float32((seed >> (8 * k)) & 0xFF) / np.float32(255.0)) for k in range(3)]
    return [np.float32((x - np.float32(0.5)) * cell) for x in r]


def grid_hash(p, frame: int, cell: float, bits: int = 22) -> int:
    c = np.float32(cell)
    j = jitter(frame, c)
    g = []
    for a in range(3):
        f = np.floor(np.float32(np.float32(p[a]) + j[a]) / c)
        g.append(int(f) & M32)
    h = ((g[0] * 73856093) ^ (g[1] * 19349663) ^ (g[2] * 83492791)) & M32
    return h & ((1 << bits) - 1)


def cie64(l: float):
    def g(mu, s):
        return math.exp(-((l - mu) / s) ** 2)

    x = g(599.8, 37.9) * 1.056 + g(442.0, 16.0) * 0.362 - g(501.1, 26.7) * 0.065
    y = g(568.8, 46.9) * 0.821 + g(530.9, 16.3) * 0.286
    z = g(437.0, 11.8) * 1.217 + g(459.0, 26.0) * 0.681
    return [max(0.0, x), max(0.0, y), max(0.0, z)]


def blackbody64(lnm: float, t: float) -> float:
    h, c, k = 6.62607015e-34, 299792458.0, 1.380649e-23
    lm = lnm * 1e-9
    return 2 * h * c * c / (lm ** 5 * (math.exp(h * c / (k * t * lm)) - 1)) * 1e-13


def airy_normal(n1, n2, n3, d, lam):
    r12 = (n1 - n2) / (n1 + n2)
    r23 = (n2 - n3) / (n2 + n3)
    cd = math.cos(4 * math.pi * n2 * d / lam)
    return (r12 ** 2 + r23 ** 2 + 2 * r12 * r23 * cd) / (1 + r12 ** 2 * r23 ** 2 + 2 * r12 * r23 * cd)


def hero_pdf(l: float) -> float:
    cmin = math.atan((380 - 555) / 40) / math.pi + 0.5
    cmax = math.atan((780 - 555) / 40) / math.pi + 0.5
    return 1.0 / ((cmax - cmin) * math.pi * 40) / (1 + ((l - 555) / 40) ** 2)


def main():
    rng = np.random.default_rng(20240611)
    out = {}
    ins = [0, 1, 2, 3, 927163, 114514, 0xFFFFFFFF, 0x80000000, 12345678] + [int(x) for x in
                                                                             rng.integers(0, 2 ** 32, 23)]
    out["pcg_hash"] = {"in": ins, "out": [pcg_hash(x) for x in ins]}
    # rng streams of camera pixels (x + y*W + frame*927163) and photon ids
    streams = []
    for (x, y, w, f) in [(0, 0, 256, 0), (17, 3, 256, 0), (255, 255, 256, 5), (100, 40, 1920, 63)]:
        seed = pcg_hash((x + y * w + f * 927163) & M32)
        vals = []
        s = seed
        for _ in range(8):
            s, r = rand_f32(s)
            vals.append(float(r))
        streams.append({"x": x, "y": y, "w": w, "frame": f, "init": seed, "rand": vals})
    out["rng_streams"] = streams
    # grid hashes (bit-exact float32)
    cases = []
    for _ in range(300):
        p = rng.uniform(-3, 3, 3).astype(np.float32)
        f = int(rng.integers(0, 1000))
        cases.append({"p": [float(v) for v in p], "frame": f, "cell": 0.02, "h": grid_hash(p, f, 0.02)})
    for p in ([0.0, 0.0, 0.0], [-0.01, 0.01, -1e-8], [0.02, -0.02, 0.04], [1.0, -1.0, 0.99], [-50.0, 50.0, 99.99]):
        for f in (0, 1, 7):
            cases.append({"p": p, "frame": f, "cell": 0.02, "h": grid_hash(np.float32(p), f, 0.02)})
    out["grid_hash"] = cases
    out["jitter"] = [{"frame": f, "j": [float(v) for v in jitter(f, np.float32(0.02))]} for f in (0, 1, 2, 99, 4096)]
    # a small photon set and its sorted keys / ranges
    n = 200
    pos = rng.uniform(-0.05, 0.05, (n, 3)).astype(np.float32)
    pos[:40] = pos[0]  # a crowded cell
    ph = np.zeros((n, 8), np.float32)
    ph[:, 0:3] = pos
    ph[:, 3] = rng.uniform(380, 780, n)
    ph[:, 4:7] = rng.normal(size=(n, 3))
    ph[:, 7] = rng.uniform(0.1, 2.0, n)
    ph[5, 7] = 0.0  # zero energy -> sentinel bucket
    frame = 3
    hs = [(1 << 22) if ph[i, 7] == 0 else grid_hash(ph[i, 0:3], frame, 0.02) for i in range(n)]
    keys = sorted(((h << 32) | i) for i, h in enumerate(hs))
    out["photon_grid"] = {"photons": ph.tolist(), "frame": frame, "cell": 0.02, "hash_bits": 22,
                          "keys": [str(k) for k in keys]}
    out["cie"] = [{"l": l, "xyz": cie64(l)} for l in range(380, 781, 20)]
    out["blackbody"] = [{"l": l, "T": t, "B": blackbody64(l, t)} for l in (380.0, 450.0, 555.0, 700.0, 780.0)
                        for t in (3000.0, 6500.0)]
    out["wien_peak_nm_6500K"] = 2.897771955e-3 / 6500 * 1e9
    films = []
    for lam in (400.0, 550.0, 700.0):
        films.append({"n1": 1.0, "n2": 1.0, "n3": 1.5, "d": 300.0, "lam": lam, "R": airy_normal(1.0, 1.0, 1.5, 300.0, lam)})
        films.append({"n1": 1.0, "n2": 1.33, "n3": 1.5, "d": lam / (4 * 1.33), "lam": lam,
                      "R": airy_normal(1.0, 1.33, 1.5, lam / (4 * 1.33), lam)})
        films.append({"n1": 1.0, "n2": 1.33, "n3": 1.0, "d": lam / (2 * 1.33), "lam": lam,
                      "R": airy_normal(1.0, 1.33, 1.0, lam / (2 * 1.33), lam)})
    out["thin_film_normal"] = films
    out["hero_pdf"] = [{"l": l, "pdf": hero_pdf(l)} for l in (380.0, 480.0, 555.0, 600.0, 780.0)]
    Path(__file__).with_name("golden.json").write_text(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
