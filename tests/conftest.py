"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def srt():
    import wgpu_spectral_rt_b200 as m

    if not m.LIB_PATH.exists():
        from wgpu_spectral_rt_b200 import build

        build.build()
    m.lib()
    return m


@pytest.fixture(scope="session")
def orc():
    import binding

    binding.lib()
    return binding


@pytest.fixture(scope="session")
def ctx(srt):
    c = srt.Context(0)
    yield c
    c.close()


def make_scene_builder(srt, preset, seed=0):
    b = srt.SceneBuilder()
    cam = b.add_preset(preset, seed)
    return b, cam


def rel_err(a, b, floor=1e-7):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), floor)


def random_rays(n, rng, center=(0.0, 0.0, 0.0), spread=0.9, tmin=1e-4, tmax=100.0):
    """Rays from random points inside a box toward random directions: float32 [n, 8]."""
    o = np.asarray(center, np.float32) + rng.uniform(-spread, spread, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3] = tmin
    r[:, 4:7] = d
    r[:, 7] = tmax
    return r


def relmse(x, ref):
    """mean over pixels and RGB of (x - ref)^2 / (ref^2 + 0.01) on linear radiance."""
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 0.01)))


MISS = 0xFFFFFFFF
# Named exclusion set of the closest-hit comparison.  The GPU answers in FP32
# (world-space vertices rounded once, watertight edge functions) and the
# oracle in FP64, so a ray whose hit or miss of a triangle FP32 rounding can
# decide either way is not a disagreement:
#   tie    another triangle is hit within |dt| < 1e-6 of the nearest (the
#          north-star rule)
#   edge   the ray passes within EDGE_REL * scale * (1 + 1 / |cos|) of the
#          boundary of the oracle's hit triangle or of the GPU's (FP64 distance
#          in world units; scale = max(1, |origin|inf, |hit point|inf), the
#          magnitude of the FP32 coordinates involved; cos = cosine between
#          the ray and the triangle's normal: a plane position uncertain by d
#          moves the hit point d / |cos| along a grazing ray)
#   range  the oracle's or the GPU's triangle is met within
#          RANGE_REL * scale * (1 + 1 / |cos|) of tmin or tmax (a ray leaving
#          a surface nearly tangentially meets its own triangle at
#          t = offset / |cos|, which FP32 rounding puts on either side of tmin)
# Hit distances of agreeing ids: |dt| <= 1e-5 t + EDGE_REL * scale / |cos|.
EDGE_REL = 2.0 ** -19
RANGE_REL = 2.0 ** -19


def closest_hit_parity(scene, oracle, rays, brute=True, hits=None):
    """Compares GPU closest hits with the FP64 oracle on `rays` [n, 8].
    Returns a dict with the masks and counts; `bad` are disagreements outside
    the named exclusion set (must be empty)."""
    g = scene.trace(rays) if hits is None else hits
    t, prim, u, v, t2 = oracle.trace(rays, brute=brute)
    pg = g["prim"]
    hit_o, hit_g = prim != MISS, pg != MISS
    o = rays[:, 0:3].astype(np.float64)
    d = rays[:, 4:7].astype(np.float64)
    tt = np.where(hit_o, t, np.where(hit_g, g["t"].astype(np.float64), 0.0))
    x = o + tt[:, None] * d
    scale = np.maximum(1.0, np.maximum(np.abs(o).max(1), np.abs(x).max(1)))
    with np.errstate(invalid="ignore"):
        tie = hit_o & (np.abs(t2 - t) < 1e-6)
    tp_o, e_o, c_o = oracle.tri_probe(rays, prim, with_cos=True)
    tp_g, e_g, c_g = oracle.tri_probe(rays, pg, with_cos=True)
    with np.errstate(divide="ignore"):
        slack_o = EDGE_REL * scale * (1.0 + 1.0 / np.maximum(c_o, 1e-12))
        slack_g = EDGE_REL * scale * (1.0 + 1.0 / np.maximum(c_g, 1e-12))
    edge = (np.abs(e_o) < slack_o) | (np.abs(e_g) < slack_g)
    with np.errstate(divide="ignore", invalid="ignore"):
        r_o = RANGE_REL * scale * (1.0 + 1.0 / np.maximum(c_o, 1e-12))
        r_g = RANGE_REL * scale * (1.0 + 1.0 / np.maximum(c_g, 1e-12))
        rng_ = ((np.abs(tp_o - rays[:, 3]) < r_o) | (np.abs(tp_o - rays[:, 7]) < r_o) |
                (np.abs(tp_g - rays[:, 3]) < r_g) | (np.abs(tp_g - rays[:, 7]) < r_g))
    excluded = tie | edge | rng_
    mismatch = pg != prim
    both = hit_o & hit_g & (pg == prim)
    # |dt| relative to its bound 1e-5 t + EDGE_REL scale / |cos| (<= 1 passes)
    dt = np.abs(g["t"][both].astype(np.float64) - t[both]) / (
        1e-5 * np.maximum(1.0, t[both]) + EDGE_REL * scale[both] / np.maximum(c_o[both], 1e-12))
    return {"n": len(rays), "hits": int(hit_o.sum()), "mismatch": int(mismatch.sum()),
            "excluded": int(excluded.sum()), "tie": int(tie.sum()), "edge": int(edge.sum()),
            "range": int(rng_.sum()), "mismatch_excluded": int((mismatch & excluded).sum()),
            "bad": np.nonzero(mismatch & ~excluded)[0], "max_dt_over_bound": float(dt.max()) if dt.size else 0.0,
            # the largest boundary distances among the disagreements, in units of the slack
            "mismatch_edge_rel": np.sort(np.minimum(np.abs(e_o) / slack_o, np.abs(e_g) / slack_g)[mismatch])[-8:],
            "g": g, "t": t, "prim": prim}


def report(name, d):
    """One line of parity statistics (shown with pytest -s or -rP)."""
    keys = ("n", "hits", "mismatch", "mismatch_excluded", "excluded", "tie", "edge", "range", "max_dt_over_bound")
    print(f"[parity] {name}: " + ", ".join(f"{k}={d[k]}" for k in keys if k in d)
          + (f", bad={len(d['bad'])}" if "bad" in d else "")
          + (f", mismatch_edge_rel_max={list(np.round(d['mismatch_edge_rel'], 9))}" if "mismatch_edge_rel" in d else ""),
          flush=True)
