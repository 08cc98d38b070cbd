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
