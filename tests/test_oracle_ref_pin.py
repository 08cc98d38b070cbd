"""The oracle pinned to the reference's own shader code.

The reference's hot path is WGSL on a Vulkan ray-query device (no graphics
stack here).  oracle/wgsl_translate.py translates its shader.wgsl,
photon_emit.wgsl and build_grid.wgsl mechanically into C++, and
oracle/ref_harness.cpp runs them on the CPU with their ray queries answered
by the oracle's FP64 query (the part the Vulkan driver answers in the
reference).  Against that run the oracle's hand restatement must be
BIT-EXACT: the shading functions, the camera rays, the stored photons, the
grid's linked lists, the accumulated frames and the rgba8 image.

Two sources:
* tests/golden/ref_wgsl.npz (tests/golden/make_ref_golden.py), outputs of the
  translated shaders stored as fixtures: always checked;
* a live run of the translated shaders on fresh inputs: checked where the
  reference tree is present (it is read only to build oracle/_ref/).
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))

import make_ref_golden as mrg  # noqa: E402

FIX = Path(__file__).resolve().parent / "golden" / "ref_wgsl.npz"
MATH_OPS = (0, 1, 2, 3, 4, 6, 7, 102, 109, 110)


@pytest.fixture(scope="module")
def fx():
    return np.load(FIX)


def _uniform(orc, raw: np.ndarray):
    u = orc.CameraUniform()
    C.memmove(C.addressof(u), raw.ctypes.data, C.sizeof(u))
    return u


def _bits(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a).view(np.uint32)


def _ref_or_skip():
    import ref_binding as ref

    if not ref.available():
        pytest.skip("the reference tree is not present (the fixture tests cover this machine)")
    ref.lib()
    return ref


# ------------------------------------------------------------------ fixtures
@pytest.mark.parametrize("op", MATH_OPS)
def test_oracle_math_matches_reference_fixture(orc, fx, op):
    """Each shading function of the oracle against the reference's function
    on the stored inputs (sample_bsdf over material types 0, 1, 2, 4 with its
    rng draws and final rng state), bit for bit."""
    inp, want = fx[f"math{op}_in"], fx[f"math{op}_out"]
    got = orc.device_math(op, inp)
    assert got.shape == want.shape
    bad = np.nonzero(np.any(_bits(got) != _bits(want), axis=1))[0]
    assert len(bad) == 0, (op, len(bad), inp[bad[:3]], got[bad[:3]], want[bad[:3]])


def test_oracle_camera_rays_match_reference_fixture(orc, fx):
    """shader.wgsl:713-728 (init_rng, the two jitter draws, the inverse
    view-projection) for every pixel of a 64 x 48 view, bit for bit."""
    u = _uniform(orc, fx["camray_uniform"])
    w, h = (int(v) for v in fx["camray_size"])
    pix = fx["camray_pix"]
    seeds = orc.device_math(0, (pix[:, 0] + pix[:, 1] * w + u.frame_count * 927163).astype(np.uint32))[:, 0]
    inp = np.zeros((len(pix), 5), np.uint32)
    inp[:, 0], inp[:, 1], inp[:, 2], inp[:, 3], inp[:, 4] = pix[:, 0], pix[:, 1], w, h, seeds
    got = orc.device_math(8, inp, aux=u)[:, :6]
    assert np.array_equal(_bits(got), _bits(fx["camray_out"]))


@pytest.mark.parametrize("case", [c[0] for c in mrg.FRAME_CASES])
def test_oracle_frames_match_reference_fixture(orc, fx, case):
    """Two frames of the scene as renderer/mod.rs:168-207 records them (2^20
    photon emitters): the photon counter, the stored photons and the grid's
    lists (by SHA-256), the accumulation buffer after each frame and the rgba8
    image — the oracle's own photon pass, grid and camera paths, bit for bit."""
    name, preset, seed, w, h, aspect, edit = next(c for c in mrg.FRAME_CASES if c[0] == case)
    pre, arrays, keep = mrg.scene_arrays(preset, seed, edit)
    o = orc.OracleScene(arrays)
    params = orc.default_params()  # MAX_DEPTH 12, 2^20 photons, the reference's constants
    accum = np.zeros((h, w, 4), np.float32)
    for f in mrg.FRAMES:
        k = f"{name}_f{f}"
        u = _uniform(orc, fx[k + "_uniform"])
        ph, _em = o.photon_emit(mrg.EMITTERS, f, 5)
        assert len(ph) == min(int(fx[k + "_count"][0]), mrg.ref.MAX_PHOTONS)
        assert mrg.sha(ph) == fx[k + "_photons_sha"].tobytes().decode()
        keys, _ranges = orc.photon_grid_build(ph, f)
        head, nxt = mrg.grid_lists_from_sorted(keys)
        assert mrg.sha(head, nxt) == fx[k + "_grid_sha"].tobytes().decode()
        accum, ldr, _, _ = o.render_frame(u, w, h, params, accum)
        assert np.array_equal(_bits(accum), _bits(fx[k + "_accum"])), k
        assert np.array_equal(ldr, fx[k + "_ldr"]), k
    o.close()
    del keep


def test_grid_lists_from_sorted_keys():
    """The sorted-key form and build_grid.wgsl's linked lists hold the same
    cells: a sequential insertion by hand against the conversion."""
    rng = np.random.default_rng(5)
    n, hs = 300, 64
    cells = rng.integers(0, hs + 1, n)  # hs = the sentinel (zero energy)
    keys = np.sort((cells.astype(np.uint64) << np.uint64(32)) | np.arange(n, dtype=np.uint64))
    head, nxt = mrg.grid_lists_from_sorted(keys, n_ids=n, hash_size=hs)
    h2 = np.full(hs, 0xFFFFFFFF, np.uint32)
    n2 = np.zeros(n, np.uint32)
    for i in range(n):  # build_grid.wgsl:55-73, one invocation after another
        if cells[i] == hs:
            continue
        n2[i] = h2[cells[i]]
        h2[cells[i]] = i
    assert np.array_equal(head, h2) and np.array_equal(nxt, n2)


# ------------------------------------------------------------------ live runs
@pytest.mark.parametrize("op", MATH_OPS)
def test_oracle_math_matches_reference_live(orc, op):
    ref = _ref_or_skip()
    inp = mrg.math_inputs(777, 20_000)[op]
    assert np.array_equal(_bits(orc.device_math(op, inp)), _bits(ref.device_math(op, inp)))


def test_oracle_frames_match_reference_live(orc):
    """A size, frame range and photon count the fixtures do not hold: 40 x 30,
    frames 2..4 accumulated, 2^17 emitters (the gather still normalises by the
    shaders' MAX_PHOTON 2^20), on the caustic slab and the prism."""
    ref = _ref_or_skip()
    w, h, n_emit = 40, 30, 1 << 17
    for preset in (4, 1):
        pre = orc.Preset(preset, 0)
        pos, yaw, pitch = pre.camera
        rs = ref.RefScene(pre.arrays())
        o = orc.OracleScene(pre.arrays())
        params = orc.default_params(photons_per_frame=n_emit, photon_norm_count=float(ref.MAX_PHOTONS))
        acc_r = np.zeros((h, w, 4), np.float32)
        acc_o = np.zeros((h, w, 4), np.float32)
        for f in (2, 3, 4):
            u = orc.camera_uniform(pos, yaw, pitch, w / h, f)
            acc_r, ldr_r, ph_r = rs.render_frame(u, w, h, 12, n_emit, accum=acc_r)
            ph_o, _ = o.photon_emit(n_emit, f, 5)
            assert np.array_equal(_bits(ph_o), _bits(ph_r)), (preset, f)
            acc_o, ldr_o, _, _ = o.render_frame(u, w, h, params, acc_o)
            assert np.array_equal(_bits(acc_o), _bits(acc_r)), (preset, f)
            assert np.array_equal(ldr_o, ldr_r), (preset, f)
        rs.close()
        o.close()


def test_translation_keeps_argument_order():
    """WGSL evaluates arguments left to right and C++ does not promise it for a
    call: the translator emits constructors as braced lists (ordered) and
    refuses any other statement that calls functions with side effects twice."""
    import wgsl_translate as wt

    src = """
var<private> s: u32;
fn draw() -> f32 { s = s + 1u; return f32(s); }
fn pair() -> vec2f { return vec2f(draw(), draw()); }
"""
    out = wt.Translator(src, "t").run()
    assert "wgsl_rt::vec2f { draw ( ) , draw ( ) }" in out
    bad = """
var<private> s: u32;
fn draw() -> f32 { s = s + 1u; return f32(s); }
fn sum() -> f32 { return draw() - draw(); }
"""
    with pytest.raises(wt.WgslError):
        wt.Translator(bad, "t").run()
