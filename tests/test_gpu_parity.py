"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Tolerances:
  integer / hash / key / index work      bit-exact
  shading math (BSDF, film, spectra)     1e-5 relative; the relative error of a
                                         value v is |a - b| / max(|a|, |b|, f) with
                                         f = 1e-3 for quantities bounded by ~1 that
                                         reach zero by cancellation (CIE lobes, film
                                         reflectance); unit directions compare by
                                         absolute difference
  closest-hit triangle ids               exact, except the named exclusion set of
                                         tests/conftest.py: ties |dt| < 1e-6, rays
                                         passing within EDGE_REL * scale of a
                                         triangle boundary, hits at the range ends
  whole frames                           per-pixel agreement of >= 97 % of the
                                         pixels within 1e-3 relative, and an image
                                         relMSE below 1e-4 against the oracle
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import closest_hit_parity, random_rays, rel_err, relmse, report

pytestmark = pytest.mark.gpu


def _bits(x):
    return np.array([x], np.uint32).view(np.float32)[0]


# ------------------------------------------------------------------ device math
def test_pcg_bit_exact(ctx, srt, orc):
    x = np.random.default_rng(0).integers(0, 2 ** 32, 100000, dtype=np.uint64).astype(np.uint32)
    assert np.array_equal(srt.device_math(ctx, 0, x), orc.device_math(0, x))


def test_spectral_math(ctx, srt, orc):
    rng = np.random.default_rng(1)
    ls = rng.uniform(380, 780, 20000).astype(np.float32)
    assert rel_err(srt.device_math(ctx, 1, ls), orc.device_math(1, ls), floor=1e-3).max() < 1e-5
    bb = np.stack([ls, rng.uniform(1000, 12000, len(ls))], 1).astype(np.float32)
    assert rel_err(srt.device_math(ctx, 2, bb), orc.device_math(2, bb)).max() < 1e-5
    r2s = np.concatenate([rng.uniform(0, 1, (20000, 3)), rng.uniform(380, 780, (20000, 4))], 1).astype(np.float32)
    assert rel_err(srt.device_math(ctx, 3, r2s), orc.device_math(3, r2s)).max() < 1e-5


def test_thin_film(ctx, srt, orc):
    rng = np.random.default_rng(2)
    n = 50000
    rows = np.stack([rng.uniform(0, 1, n), np.ones(n), rng.uniform(1.0, 2.0, n), rng.uniform(1.0, 2.0, n),
                     rng.uniform(50, 1000, n), *rng.uniform(380, 780, (4, n))], 1).astype(np.float32)
    g = srt.device_math(ctx, 4, rows)
    o = orc.device_math(4, rows)
    assert rel_err(g, o, floor=1e-3).max() < 1e-5


def test_hero_wavelengths(ctx, srt, orc):
    seeds = np.random.default_rng(3).integers(0, 2 ** 32, 50000, dtype=np.uint64).astype(np.uint32)
    g, o = srt.device_math(ctx, 5, seeds), orc.device_math(5, seeds)
    assert rel_err(g, o).max() < 1e-5


def _bsdf_cases(n, rng):
    rows = []
    mats = [
        [0.7, 0.3, 0.2, 1, 0, 0, 0, 0],  # Lambert
        [0.9, 0.6, 0.3, 1, 1, 0.3, 0, 0],  # GGX metal
        [0.9, 0.6, 0.3, 1, 1, 0.0, 0, 0],  # GGX at the roughness clamp
        [1, 1, 1, 1, 2, 0, 1.5, 0.0],  # glass, no dispersion
        [1, 1, 1, 1, 2, 0, 1.5, 0.0042],  # dispersive glass
        [1, 1, 1, 1, 4, 500, 1.33, 1.0],  # soap film
        [1, 1, 1, 1, 4, 30, 1.33, 1.5],  # film thinner than the 50 nm clamp
        [1, 1, 1, 0.2, 5, 400, 1.33, 1.5],  # coated GGX
    ]
    for k in range(n):
        nrm = rng.normal(size=3)
        nrm /= np.linalg.norm(nrm)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        if np.dot(d, nrm) > 0:
            d = -d
        mat = mats[k % len(mats)]
        front = bool(rng.integers(0, 2))
        wl = rng.uniform(380, 780, 4)
        thr = rng.uniform(0, 1, 4) if k % 3 else np.array([0.7, 0, 0, 0])
        rows.append([*d, *nrm, *mat, 1.0 if front else 0.0, *wl, *thr, _bits(int(rng.integers(0, 2 ** 32)))])
    return np.array(rows, np.float32)


GRAZING = 1e-2


def test_sample_bsdf(ctx, srt, orc):
    rows = _bsdf_cases(40000, np.random.default_rng(4))
    g = srt.device_math(ctx, 6, rows)
    o = orc.device_math(6, rows)
    # the same random numbers were consumed (rng state bit-exact)...
    same_rng = g[:, 8].view(np.uint32) == o[:, 8].view(np.uint32)
    same_branch = (g[:, 7] == o[:, 7])
    assert same_rng.mean() > 0.999 and same_branch.mean() > 0.999
    ok = same_rng & same_branch & (o[:, 7] == 0)
    # ...sampled unit directions agree to 1e-5 absolute...
    assert np.abs(g[ok, :3] - o[ok, :3]).max() < 1e-5
    # ...and the weights within 1e-5 relative outside the grazing set: the
    # incident or the sampled direction within GRAZING of the tangent plane
    # (|cos| < GRAZING), where the 1/cos factors amplify the last-ulp
    # differences of the GPU's and the host's transcendental functions
    err = rel_err(g[:, 3:7], o[:, 3:7], floor=1e-6).max(1)
    nrm = rows[:, 3:6].astype(np.float64)
    cos_i = np.abs((rows[:, 0:3] * nrm).sum(1))
    cos_o = np.abs((o[:, 0:3] * nrm).sum(1))
    grazing = np.minimum(cos_i, cos_o) < GRAZING
    sel = ok & ~grazing
    worst = np.argsort(-np.where(sel, err, 0))[:6]
    print(f"[parity] bsdf: n={len(rows)}, compared={int(sel.sum())}, grazing={int((ok & grazing).sum())}, "
          f"max err={err[sel].max():.3e}; worst (type, cos_i, cos_o, err): "
          + "; ".join(f"({rows[k, 10]:.0f}, {cos_i[k]:.2e}, {cos_o[k]:.2e}, {err[k]:.2e})" for k in worst), flush=True)
    assert err[sel].max() < 1e-5
    assert err[ok & grazing].max() < 1e-2


def test_grid_hash_bit_exact(ctx, srt, orc):
    rng = np.random.default_rng(5)
    n = 100000
    rows = np.concatenate([rng.uniform(-10, 10, (n, 3)), np.zeros((n, 1)), np.full((n, 1), 0.02)], 1).astype(np.float32)
    rows[:, 3] = rng.integers(0, 100000, n).astype(np.uint32).view(np.float32)
    assert np.array_equal(srt.device_math(ctx, 7, rows), orc.device_math(7, rows))


def test_camera_rays(ctx, srt, orc):
    cam = srt.camera_uniform([0.1, 0.2, 3.0], -math.pi / 2 + 0.1, 0.05, 16 / 9, 7)
    rng = np.random.default_rng(6)
    n = 20000
    rows = np.stack([rng.integers(0, 1920, n), rng.integers(0, 1080, n), np.full(n, 1920), np.full(n, 1080),
                     rng.integers(0, 2 ** 32, n)], 1).astype(np.uint32)
    g = srt.device_math(ctx, 8, rows, cam)
    o = orc.device_math(8, rows, cam)
    assert np.array_equal(g[:, 6].view(np.uint32), o[:, 6].view(np.uint32))
    assert np.abs(g[:, :6] - o[:, :6]).max() < 1e-5


# ------------------------------------------------------------------ photon grid
def _photons(n, rng, spread=0.3, crowd=0):
    p = np.zeros((n, 8), np.float32)
    p[:, 0:3] = rng.uniform(-spread, spread, (n, 3))
    if crowd:
        p[:crowd, 0:3] = p[0, 0:3]
    p[:, 3] = rng.uniform(380, 780, n)
    d = rng.normal(size=(n, 3))
    p[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    p[:, 7] = rng.uniform(0.01, 5, n)
    p[rng.integers(0, n, n // 50), 7] = 0.0  # zero-energy photons go to the sentinel bucket
    return p


@pytest.mark.parametrize("n,frame,crowd", [(0, 0, 0), (1, 0, 0), (777, 3, 300), (100000, 11, 5000),
                                           ((1 << 20), 2, 0)])
def test_photon_grid_bit_exact(ctx, srt, orc, n, frame, crowd):
    ph = _photons(n, np.random.default_rng(n + frame), crowd=crowd)
    kg, rg = srt.photon_grid_build(ctx, ph, frame)
    ko, ro = orc.photon_grid_build(ph, frame)
    assert np.array_equal(kg, ko)
    assert np.array_equal(rg, ro)


def test_photon_grid_golden(ctx, srt):
    import json
    from pathlib import Path

    g = json.loads((Path(__file__).parent / "golden" / "golden.json").read_text())["photon_grid"]
    k, _ = srt.photon_grid_build(ctx, np.array(g["photons"], np.float32), g["frame"], g["cell"], g["hash_bits"])
    assert [int(x) for x in k] == [int(x) for x in g["keys"]]


def test_photon_grid_full_size_properties(ctx, srt):
    # 4M photons (the config-2 photon count): sortedness, permutation, ranges
    n = 1 << 22
    ph = _photons(n, np.random.default_rng(9), spread=2.0)
    k, r = srt.photon_grid_build(ctx, ph, 5)
    assert np.all(k[1:] > k[:-1])  # strictly ascending (keys are unique)
    idx = (k & np.uint64(0xFFFFFFFF)).astype(np.int64)
    assert np.array_equal(np.sort(idx), np.arange(n))
    h = (k >> np.uint64(32)).astype(np.int64)
    assert np.array_equal(h == (1 << 22), ph[idx, 7] == 0)
    nonempty = r[:, 1] > r[:, 0]
    assert int((r[nonempty, 1] - r[nonempty, 0]).sum()) == int((h < (1 << 22)).sum())
    b = np.nonzero(nonempty)[0]
    assert np.all(h[r[b, 0]] == b) and np.all(h[r[b, 1] - 1] == b)


def test_gather(ctx, srt, orc):
    rng = np.random.default_rng(10)
    ph = _photons(20000, rng, spread=0.1, crowd=200)
    nq = 5000
    q = np.zeros((nq, 10), np.float32)
    q[:, 0:3] = ph[rng.integers(0, len(ph), nq), 0:3] + rng.normal(0, 0.005, (nq, 3))
    nrm = rng.normal(size=(nq, 3))
    q[:, 3:6] = nrm / np.linalg.norm(nrm, axis=1, keepdims=True)
    q[:, 6:10] = rng.uniform(380, 780, (nq, 4))
    p = srt.default_params()
    for frame in (0, 9):
        g = srt.photon_gather(ctx, ph, q, frame, p)
        o = orc.photon_gather(ph, q, frame, p)
        assert rel_err(g, o, floor=1e-3 * max(1e-30, float(np.abs(o).max()))).max() < 1e-4


# ------------------------------------------------------------------ traversal
@pytest.fixture(scope="module")
def config1(srt, orc, ctx):
    b = srt.SceneBuilder()
    cam = b.add_preset(srt.PRESET_CONFIG1)
    scene = b.build(ctx)
    o = orc.OracleScene(b.arrays())
    yield b, scene, o, cam
    scene.close()
    o.close()


@pytest.fixture(scope="module")
def cornell(srt, orc, ctx):
    b = srt.SceneBuilder()
    cam = b.add_preset(srt.PRESET_CORNELL_BOX)
    scene = b.build(ctx)
    o = orc.OracleScene(b.arrays())
    yield b, scene, o, cam
    scene.close()
    o.close()


@pytest.mark.parametrize("which", ["config1", "cornell"])
def test_closest_hit_ids(request, which):
    """Exact triangle ids outside the named exclusion set (ties, rays within
    EDGE_REL * scale of a triangle boundary, hits at the ends of the range;
    tests/conftest.py)."""
    b, scene, o, _ = request.getfixturevalue(which)
    rays = random_rays(40000, np.random.default_rng(11), spread=0.9)
    d = closest_hit_parity(scene, o, rays, brute=True)
    report(which, d)
    assert len(d["bad"]) == 0, d["bad"][:10]
    assert d["max_dt_over_bound"] <= 1.0


def test_any_hit(config1):
    _, scene, o, _ = config1
    rays = random_rays(40000, np.random.default_rng(12), spread=0.9)
    rays[:, 7] = np.random.default_rng(13).uniform(0.01, 2.5, len(rays))
    g = scene.trace(rays, any_hit=True)
    _, prim, *_ = o.trace(rays, any_hit=True, brute=True)
    t, pc, *_ = o.trace(rays, brute=True)
    near_end = np.abs(t - rays[:, 7]) < 1e-5  # hit exactly at tmax: rounding decides
    agree = ((g["prim"] == 0) == (prim == 0)) | near_end
    assert agree.mean() > 0.9995


def test_degenerate_rays(config1):
    _, scene, _, _ = config1
    r = np.zeros((4, 8), np.float32)
    r[:, 3] = 1e-4
    r[:, 7] = 100
    r[1, 4:7] = [0, 1, 0]  # axis-aligned: hits the ceiling
    r[2, 4:7] = [0, 0, 0]  # zero direction: miss
    r[3, 4:7] = [1, 0, 0]
    r[3, 3], r[3, 7] = 5.0, 1.0  # tmin > tmax: miss
    g = scene.trace(r)
    assert g["prim"][0] == 0xFFFFFFFF and g["prim"][2] == 0xFFFFFFFF and g["prim"][3] == 0xFFFFFFFF
    assert g["prim"][1] != 0xFFFFFFFF and abs(g["t"][1] - 0.99) < 1e-5  # the light at y = 0.99


# ------------------------------------------------------------------ photon pass and whole frames
def _cam(srt, cam, w, h, frame):
    pos, yaw, pitch = cam
    return srt.camera_uniform(pos, yaw, pitch, w / h, frame)


def test_photon_emission_matches_oracle(srt, ctx, cornell):
    b, scene, o, cam = cornell
    p = srt.default_params(photons_per_frame=1 << 16)
    r = srt.Renderer(ctx, scene, 16, 16, p)
    r.render(_cam(srt, cam, 16, 16, 4))
    g = r.read_photons()
    op, _ = o.photon_emit(1 << 16, 4)
    # same stored set in the same (emission) order, up to rare FP32-vs-FP64 hit differences
    assert abs(len(g) - len(op)) <= max(3, len(op) // 200)
    m = min(len(g), len(op))
    close = np.all(np.abs(g[:m] - op[:m]) < 1e-3 * np.maximum(1, np.abs(op[:m])), axis=1)
    assert close[: m // 2].mean() > 0.97
    r.close()


# 37 x 23: the camera rays of bounce 0 leave 8 x 4 pixel tiles per warp,
# narrower at the right and bottom edges when the size is no multiple
@pytest.mark.parametrize("which,photons,w,h", [("config1", 1 << 18, 48, 32), ("cornell", 1 << 18, 48, 32),
                                              ("cornell", 1 << 16, 37, 23)])
def test_frame_matches_oracle(srt, ctx, request, which, photons, w, h):
    b, scene, o, cam = request.getfixturevalue(which)
    p = srt.default_params(photons_per_frame=photons)
    r = srt.Renderer(ctx, scene, w, h, p)
    acc_o = np.zeros((h, w, 4), np.float32)
    for f in range(3):
        u = _cam(srt, cam, w, h, f)
        r.render(u)
        acc_o, ldr_o, _, _ = o.render_frame(u, w, h, p, acc_o)
    acc_g = r.read_accum()
    ldr_g = r.read_ldr()
    assert np.all(acc_g[..., 3] == 3) and np.all(acc_o[..., 3] == 3)
    e = rel_err(acc_g[..., :3], acc_o[..., :3], floor=1e-3)
    pix_ok = (e < 1e-3).all(-1)
    assert pix_ok.mean() >= 0.97, pix_ok.mean()
    assert relmse(acc_g[..., :3] / 3, acc_o[..., :3] / 3) < 1e-4
    assert (np.abs(ldr_g.astype(int) - ldr_o.astype(int)) <= 1).mean() > 0.97
    r.close()


def test_accumulation_reset_and_stats(srt, ctx, config1, tmp_path):
    b, scene, o, cam = config1
    w, h = 32, 32
    r = srt.Renderer(ctx, scene, w, h, srt.default_params(photons_per_frame=1 << 14))
    for f in range(4):
        r.render(_cam(srt, cam, w, h, f))
    assert r.frame_count == 4
    assert np.all(r.read_accum()[..., 3] == 4)
    r.render(_cam(srt, cam, w, h, 0))  # frame_count 0 resets (shader.wgsl:803-805)
    assert np.all(r.read_accum()[..., 3] == 1)
    st = r.stats()
    assert st["frames"] == 5 and st["paths"] == 5 * w * h and st["rays_closest"] > st["paths"]
    r.save_screenshot(tmp_path / "s.png")
    assert (tmp_path / "s.png").stat().st_size > 100
    r.save_screenshot_async(tmp_path / "a.png")  # read back now, encoded on the worker thread
    assert srt.screenshot_flush() == 0
    assert (tmp_path / "a.png").read_bytes() == (tmp_path / "s.png").read_bytes()
    r.close()


def test_graph_and_direct_launch_agree(srt, ctx, config1):
    b, scene, o, cam = config1
    w, h = 40, 24
    outs = []
    for flags in (0, srt.FLAG_NO_GRAPH, srt.FLAG_STAGE_TIMING):
        r = srt.Renderer(ctx, scene, w, h, srt.default_params(photons_per_frame=1 << 15, flags=flags))
        for f in range(2):
            r.render(_cam(srt, cam, w, h, f))
        outs.append(r.read_accum())
        r.close()
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])


def test_accumulation_resume_continues_bit_for_bit(srt, ctx, cornell):
    """srt_write_accum_f64: FP64 sums read back after 5 frames and loaded into a
    new renderer continue, frame for frame, exactly as the uninterrupted render."""
    b, scene, o, cam = cornell
    w, h = 32, 24
    p = srt.default_params(photons_per_frame=1 << 14, flags=srt.FLAG_FP64_ACCUM)
    r = srt.Renderer(ctx, scene, w, h, p)
    for f in range(5):
        r.render(_cam(srt, cam, w, h, f))
    saved = r.read_accum64()
    for f in range(5, 9):
        r.render(_cam(srt, cam, w, h, f))
    full = r.read_accum64()
    r2 = srt.Renderer(ctx, scene, w, h, p)
    r2.write_accum64(saved)
    np.testing.assert_array_equal(r2.read_accum64(), saved)
    for f in range(5, 9):
        r2.render(_cam(srt, cam, w, h, f))
    np.testing.assert_array_equal(r2.read_accum64(), full)
    assert np.all(r2.read_accum()[..., 3] == 9)
    plain = srt.Renderer(ctx, scene, w, h, srt.default_params(photons_per_frame=1 << 14))
    with pytest.raises(srt.SrtError):
        plain.write_accum64(saved)  # no FP64 accumulation to load into
    for x in (r, r2, plain):
        x.close()


def test_bounded_wait_timeout_is_reported_and_context_survives(srt, ctx, cornell):
    """A device wait that cannot complete gives up after its poll limit; the
    host gets SRT_ERR_TIMEOUT and the context keeps working."""
    with pytest.raises(srt.SrtError) as e:
        srt.wait_timeout_check(ctx, 1000)
    assert e.value.status == 4  # SRT_ERR_TIMEOUT
    b, scene, o, cam = cornell
    r = srt.Renderer(ctx, scene, 16, 16, srt.default_params(photons_per_frame=1 << 12))
    r.render(_cam(srt, cam, 16, 16, 0))
    assert np.all(r.read_accum()[..., 3] == 1)
    r.close()
