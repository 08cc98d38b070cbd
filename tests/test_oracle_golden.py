"""Pins the CPU oracle against the golden vectors (tests/golden/golden.json)
and against closed forms.  CPU only."""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

GOLDEN = json.loads((Path(__file__).parent / "golden" / "golden.json").read_text())


def test_pcg_hash_bit_exact(orc):
    g = GOLDEN["pcg_hash"]
    out = orc.device_math(0, np.array(g["in"], np.uint32))
    assert out[:, 0].tolist() == g["out"]


def test_rng_streams(orc):
    # rand() sequence: f32(u32) / 4294967295.0 after each pcg step
    for s in GOLDEN["rng_streams"]:
        seed = s["init"]
        vals = []
        x = np.array([seed], np.uint32)
        for _ in range(8):
            x = orc.device_math(0, x)[:, 0].astype(np.uint32)
            vals.append(float(np.float32(x[0]) / np.float32(4294967295.0)))
        assert vals == pytest.approx(s["rand"], rel=0, abs=0)


def test_grid_hash_bit_exact(orc):
    rows = []
    for c in GOLDEN["grid_hash"]:
        rows.append([*c["p"], np.array([c["frame"]], np.uint32).view(np.float32)[0], c["cell"]])
    out = orc.device_math(7, np.array(rows, np.float32))
    assert out[:, 0].tolist() == [c["h"] for c in GOLDEN["grid_hash"]]


def test_photon_grid_keys_golden(orc):
    g = GOLDEN["photon_grid"]
    keys, ranges = orc.photon_grid_build(np.array(g["photons"], np.float32), g["frame"], g["cell"], g["hash_bits"])
    assert [int(k) for k in keys] == [int(k) for k in g["keys"]]
    # ranges cover exactly the non-sentinel photons, each bucket contiguous
    h = (keys >> np.uint64(32)).astype(np.int64)
    valid = h < (1 << g["hash_bits"])
    for b in np.unique(h[valid]):
        idx = np.nonzero(h == b)[0]
        assert ranges[b].tolist() == [idx[0], idx[-1] + 1]
    assert int((ranges[:, 1] - ranges[:, 0]).sum()) == int(valid.sum())


def test_cie_fit(orc):
    ls = np.array([c["l"] for c in GOLDEN["cie"]], np.float32)
    out = orc.device_math(1, ls)
    ref = np.array([c["xyz"] for c in GOLDEN["cie"]])
    np.testing.assert_allclose(out, ref, rtol=2e-5, atol=1e-7)


def test_blackbody_and_wien_peak(orc):
    rows = np.array([[c["l"], c["T"]] for c in GOLDEN["blackbody"]], np.float32)
    out = orc.device_math(2, rows)[:, 0]
    np.testing.assert_allclose(out, [c["B"] for c in GOLDEN["blackbody"]], rtol=2e-5)
    ls = np.arange(380.0, 780.0, 0.25, dtype=np.float32)
    b = orc.device_math(2, np.stack([ls, np.full_like(ls, 6500.0)], 1).astype(np.float32))[:, 0]
    assert abs(float(ls[np.argmax(b)]) - GOLDEN["wien_peak_nm_6500K"]) < 0.5


def test_thin_film_closed_forms(orc):
    rows = []
    for f in GOLDEN["thin_film_normal"]:
        rows.append([1.0, f["n1"], f["n2"], f["n3"], f["d"], f["lam"], f["lam"], f["lam"], f["lam"]])
    out = orc.device_math(4, np.array(rows, np.float32))
    ref = np.array([f["R"] for f in GOLDEN["thin_film_normal"]])
    np.testing.assert_allclose(out[:, 0], ref, rtol=1e-4, atol=1e-6)
    # total internal reflection returns 1 for every wavelength
    tir = orc.device_math(4, np.array([[0.1, 1.5, 1.0, 1.0, 300, 400, 500, 600, 700]], np.float32))
    assert tir.tolist() == [[1.0, 1.0, 1.0, 1.0]]


def test_rgb_to_spectrum(orc):
    rng = np.random.default_rng(1)
    rows = np.concatenate([rng.uniform(0, 1, (64, 3)), rng.uniform(380, 780, (64, 4))], 1).astype(np.float32)
    out = orc.device_math(3, rows)
    rgb = rows[:, :3].astype(np.float64)
    white = rgb.min(1, keepdims=True)
    c = np.maximum(rgb - white, 0)
    lam = rows[:, 3:].astype(np.float64)
    ref = white + c[:, :1] * np.exp(-((lam - 630) / 20) ** 2) + c[:, 1:2] * np.exp(-((lam - 525) / 20) ** 2) + \
        c[:, 2:3] * np.exp(-((lam - 460) / 20) ** 2)
    np.testing.assert_allclose(out, np.clip(ref, 0, 0.99), rtol=2e-5, atol=1e-7)


def test_hero_wavelengths(orc):
    seeds = np.arange(4096, dtype=np.uint32) * np.uint32(2654435761)
    out = orc.device_math(5, seeds)
    wl, s = out[:, :4].astype(np.float64), out[:, 4]
    assert wl.min() >= 380.0 and wl.max() <= 780.0
    d = np.mod(np.round(np.diff(np.sort(wl, 1), axis=1)), 100)
    assert np.all(d == 0)  # four wavelengths spaced by 100 nm (mod 400)
    cmin = math.atan((380 - 555) / 40) / math.pi + 0.5
    cmax = math.atan((780 - 555) / 40) / math.pi + 0.5
    exact = (1.0 / ((cmax - cmin) * math.pi * 40) / (1 + ((wl - 555) / 40) ** 2)).sum(1)
    np.testing.assert_allclose(s, exact, rtol=1e-5)
    # the truncated Cauchy pdf integrates to one over [380, 780]
    xs = np.linspace(380, 780, 400001)
    integral = np.trapezoid(1.0 / ((cmax - cmin) * math.pi * 40) / (1 + ((xs - 555) / 40) ** 2), xs)
    assert abs(integral - 1.0) < 1e-6
    for p in GOLDEN["hero_pdf"]:
        assert 1.0 / ((cmax - cmin) * math.pi * 40) / (1 + ((p["l"] - 555) / 40) ** 2) == pytest.approx(p["pdf"])


def _bsdf_row(r_dir, n, mat, front, wl, thr, seed):
    return [*r_dir, *n, *mat, 1.0 if front else 0.0, *wl, *thr, np.array([seed], np.uint32).view(np.float32)[0]]


def test_bsdf_lambert_and_limits(orc):
    # Lambert: direction in the hemisphere of n, attenuation = reflectance spectrum
    rng = np.random.default_rng(7)
    rows = []
    for k in range(256):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        rows.append(_bsdf_row(-n, n, [0.5, 0.4, 0.3, 1, 0, 0, 0, 0], True, [450, 550, 650, 750], [1, 1, 1, 1], k * 7919))
    out = orc.device_math(6, np.array(rows, np.float32))
    ns = np.array(rows)[:, 3:6]
    assert np.all((out[:, :3] * ns).sum(1) > -1e-6)
    assert np.all(out[:, 7] == 0)
    # dielectric at normal incidence: Schlick r0 decides, refraction keeps the direction
    row = _bsdf_row([0, 0, -1], [0, 0, 1], [1, 1, 1, 1, 2, 0, 1.5, 0.0], True, [550, 450, 650, 750], [1, 1, 1, 1], 3)
    o = orc.device_math(6, np.array([row], np.float32))[0]
    assert o[7] == 0 and (np.allclose(o[:3], [0, 0, -1], atol=1e-6) or np.allclose(o[:3], [0, 0, 1], atol=1e-6))
    # dispersive glass collapses the tuple onto the hero wavelength (x4) on refraction
    for seed in range(64):
        row = _bsdf_row([0, 0, -1], [0, 0, 1], [1, 1, 1, 1, 2, 0, 1.5, 0.01], True, [550, 450, 650, 750], [1, 1, 1, 1], seed)
        o = orc.device_math(6, np.array([row], np.float32))[0]
        if o[2] < 0:  # refracted
            ir = 1.5 + 0.01 / 0.55 ** 2
            assert o[4] == 0 and o[5] == 0 and o[6] == 0
            assert o[3] == pytest.approx(4 * 0.99 / ir ** 2, rel=1e-5)
            break
    else:
        pytest.fail("no refraction sampled")


def test_lambert_directions_are_cosine_distributed(orc):
    """The Lambert continuation normalize(n + unit vector) (shader.wgsl:462-466)
    is cosine-weighted about n: E[cos] = 2/3, E[cos^2] = 1/2, azimuth uniform;
    its attenuation is the reflectance spectrum, the same for every sample."""
    n_s = 40_000
    rows = [_bsdf_row([0, 0, -1], [0, 0, 1], [0.5, 0.4, 0.3, 1, 0, 0, 0, 0], True, [450, 550, 650, 750],
                      [1, 1, 1, 1], 7919 * k + 1) for k in range(n_s)]
    out = orc.device_math(6, np.array(rows, np.float32))[:, :8].astype(np.float64)  # 8, 9: RNG state bits
    c = out[:, 2]
    assert np.all(c > -1e-6) and np.all(out[:, 7] == 0)
    tol = 4 / math.sqrt(n_s)
    assert abs(c.mean() - 2 / 3) < tol * 0.25
    assert abs((c ** 2).mean() - 0.5) < tol * 0.3
    phi = np.arctan2(out[:, 1], out[:, 0])
    hist, _ = np.histogram(phi, bins=8, range=(-math.pi, math.pi))
    assert np.all(np.abs(hist / n_s - 1 / 8) < 0.01)
    att = out[:, 3:7]
    assert np.all(att == att[0]) and np.all((att[0] > 0) & (att[0] <= 0.99))
