"""The C ABI library loads and exports every declared entry point; the host
side (scene builder, geometry, presets, camera uniform, screenshot) behaves
like the reference's.  CPU only: no compute call touches a GPU here."""
from __future__ import annotations

import ctypes as C
import math
import re
import struct
import zlib
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "srt.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(srt_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_every_declared_symbol_is_exported(srt):
    names = declared_functions()
    assert len(names) >= 40
    L = C.CDLL(str(srt.LIB_PATH))
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the Python mirror binds each one
    assert set(names) <= set(srt.SIGNATURES), set(names) - set(srt.SIGNATURES)


def test_abi_version_and_record_sizes(srt):
    assert srt.lib().srt_abi_version() == 4
    assert srt.guide_param_count() == 23856
    assert C.sizeof(srt.CameraUniform) == 272 and C.sizeof(srt.Vertex) == 32 and C.sizeof(srt.Light) == 64


def test_params_default_match_reference_constants(srt):
    p = srt.default_params()
    assert p.max_depth == 12  # renderer/compute_pass.rs:26
    assert p.photons_per_frame == 1 << 20  # renderer/mod.rs:18
    assert p.hash_bits == 22  # renderer/mod.rs:19
    assert p.photon_max_bounces == 5 and p.gather_cap == 64
    assert p.cell_size == pytest.approx(0.02) and p.gather_radius0 == pytest.approx(0.02)
    assert p.radius_exponent == pytest.approx(-0.15) and p.spectral_radius == pytest.approx(20.0)


def test_plane_and_cube(srt):
    v, i = srt.geometry("plane")
    assert v.shape == (4, 8) and i.tolist() == [0, 1, 2, 2, 1, 3]
    assert v[:, :4].tolist() == [[-0.5, 0, 0.5, 1], [0.5, 0, 0.5, 1], [-0.5, 0, -0.5, 1], [0.5, 0, -0.5, 1]]
    v, i = srt.geometry("cube")
    assert v.shape == (24, 8) and len(i) == 36
    # every face is wound counter-clockwise seen from outside
    p = v[:, :3]
    for f in range(12):
        a, b, c = p[i[3 * f]], p[i[3 * f + 1]], p[i[3 * f + 2]]
        n = np.cross(b - a, c - a)
        assert np.dot(n, (a + b + c) / 3) > 0


@pytest.mark.parametrize("sub", [0, 1, 2, 4])
def test_icosphere_counts_and_radius(srt, sub):
    v, i = srt.geometry("icosphere", sub)
    assert len(i) // 3 == 20 * 4 ** sub
    assert len(v) == 10 * 4 ** sub + 2
    r = np.linalg.norm(v[:, :3], axis=1)
    np.testing.assert_allclose(r, 0.5, atol=1e-6)
    np.testing.assert_allclose(np.linalg.norm(v[:, 4:7], axis=1), 1.0, atol=1e-6)
    p = v[:, :3]
    a, b, c = p[i[0::3]], p[i[1::3]], p[i[2::3]]
    assert np.all((np.cross(b - a, c - a) * (a + b + c)).sum(1) > 0)


def test_uv_sphere(srt):
    v, i = srt.geometry("uv_sphere", 64, 32)
    assert len(i) // 3 == 4032
    np.testing.assert_allclose(np.linalg.norm(v[:, :3], axis=1), 0.5, atol=1e-6)


def test_light_expansion_matches_builder(srt):
    # builder.rs:101-129: one world-space light triangle per mesh triangle
    b = srt.SceneBuilder()
    pv, pi = srt.geometry("plane")
    m = b.add_mesh(pv, pi)
    mat = b.add_material([6500, 1, 0, 1], [3, 0, 0, 0])
    T = np.eye(4, dtype=np.float32)
    T[:3, 3] = [1, 2, 3]
    b.add_light_instance(m, mat, T, [0, 6500, 1, 0])
    a = b.arrays()
    assert a.n_lights == 2 and a.n_instances == 1
    L = a.lights[0]
    assert list(L.v0) == [-0.5 + 1, 2, 0.5 + 3, 1.0] and list(L.params) == [0, 6500, 1, 0]


@pytest.mark.parametrize("preset,tris", [(0, 10 + 2 + 12 + 5120), (2, 10 + 2 + 4032), (5, 10 + 2 + 2 * 12)])
def test_presets(srt, preset, tris):
    b = srt.SceneBuilder()
    pos, yaw, pitch = b.add_preset(preset)
    a = b.arrays()
    n = 0
    idx_end = [a.mesh_infos[m + 1].index_offset if m + 1 < a.n_meshes else a.n_indices for m in range(a.n_meshes)]
    for k in range(a.n_instances):
        m = a.instances[k].mesh_id
        n += (idx_end[m] - a.mesh_infos[m].index_offset) // 3
    assert n == tris
    assert pos == [0, 0, 3] and yaw == pytest.approx(-math.pi / 2) and a.n_lights == 2


def test_camera_uniform(srt):
    u = srt.camera_uniform([0.0, 0.0, 3.0], -math.pi / 2, 0.0, 16 / 9, 5)
    view = np.array(u.view, np.float64).reshape(4, 4).T
    vinv = np.array(u.view_inverse, np.float64).reshape(4, 4).T
    proj = np.array(u.proj, np.float64).reshape(4, 4).T
    pinv = np.array(u.proj_inverse, np.float64).reshape(4, 4).T
    np.testing.assert_allclose(view @ vinv, np.eye(4), atol=1e-6)
    np.testing.assert_allclose(proj @ pinv, np.eye(4), atol=1e-5)
    np.testing.assert_allclose(vinv[:3, 3], [0, 0, 3], atol=1e-6)  # camera position
    h = 1.0 / math.tan(math.radians(22.5))
    assert proj[1, 1] == pytest.approx(h, rel=1e-6) and proj[0, 0] == pytest.approx(h / (16 / 9), rel=1e-6)
    assert proj[3, 2] == -1 and proj[2, 2] == pytest.approx(100 / (0.1 - 100), rel=1e-6)
    assert u.frame_count == 5


def _read_png(path):
    data = Path(path).read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, w, h = 8, b"", 0, 0
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        typ = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        crc = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]
        assert zlib.crc32(typ + body) & 0xFFFFFFFF == crc
        if typ == b"IHDR":
            w, h = struct.unpack(">II", body[:8])
        elif typ == b"IDAT":
            idat += body
        pos += 12 + n
    raw = zlib.decompress(idat)
    rows = [raw[r * (4 * w + 1) + 1:(r + 1) * (4 * w + 1)] for r in range(h)]
    return np.frombuffer(b"".join(rows), np.uint8).reshape(h, w, 4)


def test_screenshot_flip_and_srgb(srt, tmp_path):
    # screenshot.rs:41-70: rows reversed, sRGB OETF on the 8-bit linear values, alpha 255
    rng = np.random.default_rng(0)
    img = rng.integers(0, 256, (7, 5, 4), dtype=np.uint8)
    p = tmp_path / "shot.png"
    srt.screenshot_write(p, img)
    got = _read_png(p)

    def oetf(c):
        cf = np.float32(c) / np.float32(255.0)
        s = cf * np.float32(12.92) if cf <= 0.0031308 else np.float32(1.055) * np.float32(cf) ** (1 / 2.4) - 0.055
        return int(np.round(np.clip(s, 0, 1) * 255))

    exp = np.zeros_like(img)
    for y in range(7):
        for x in range(5):
            src = img[6 - y, x]
            exp[y, x] = [oetf(src[0]), oetf(src[1]), oetf(src[2]), 255]
    assert np.array_equal(got, exp)


def test_screenshot_worker_writes_the_same_files(srt, tmp_path):
    """srt_screenshot_write_async: PNGs encoded on the library's worker thread are
    byte-identical to the synchronous writer's; the caller's buffer may change
    right after the call; a failed write is counted once by the next flush."""
    rng = np.random.default_rng(1)
    imgs = [rng.integers(0, 256, (9 + k, 6 + 2 * k, 4), dtype=np.uint8) for k in range(4)]
    for k, img in enumerate(imgs):
        srt.screenshot_write(tmp_path / f"sync{k}.png", img)
        srt.screenshot_write_async(tmp_path / f"async{k}.png", img)
        img[:] = 0  # the job holds its own copy
    srt.screenshot_write_async(tmp_path / "no_such_dir" / "x.png", imgs[0])
    assert srt.screenshot_flush() == 1
    assert srt.screenshot_flush() == 0
    for k in range(4):
        assert (tmp_path / f"async{k}.png").read_bytes() == (tmp_path / f"sync{k}.png").read_bytes()
    with pytest.raises(srt.SrtError):
        srt.screenshot_write_async(tmp_path / "bad.png", np.zeros((0, 4, 4), np.uint8))


def test_invalid_arguments_fail_cleanly(srt):
    L = srt.lib()
    assert L.srt_scene_builder_add_instance(None, 0, 0, None) == 1
    b = srt.SceneBuilder()
    with pytest.raises(srt.SrtError):
        b.add_instance(3, 0, np.eye(4))  # no such mesh
    with pytest.raises(srt.SrtError):
        b.add_mesh(np.zeros((3, 8), np.float32), [0, 1, 5])  # index out of range


def test_missing_native_library_fails_loudly(tmp_path):
    """Without the CUDA library the package raises on first use; there is no
    CPU fallback for the product path."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import wgpu_spectral_rt_b200 as srt\n"
            "try:\n    srt.Context(0)\nexcept RuntimeError as e:\n    print('raised:', e)\n")
    env = dict(os.environ, SRT_LIB_PATH=str(tmp_path / "missing.so"), PYTHONPATH=root)
    p = subprocess.run([sys.executable, "-c", code], env=env, cwd=tmp_path, capture_output=True, text=True,
                       timeout=120)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.startswith("raised: native library missing")


def test_no_device_is_reported_as_a_status(srt):
    """On a machine without a CUDA device, context creation returns
    SRT_ERR_NO_DEVICE instead of aborting (skipped where a GPU is present)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(srt.SrtError) as e:
        srt.Context(0)
    assert e.value.status == 6  # SRT_ERR_NO_DEVICE


def test_noalloc_grid_refuses_bad_arguments_before_device_work(srt):
    """srt_photon_grid_build_noalloc checks its arguments before it touches a
    device: a misaligned photon, key or range pointer (the kernels read
    photons as 16-byte vectors and write 8-byte keys and ranges), a count
    above the fixed scratch capacity and an invalid cell size are refused with
    a status.  The pointers below are never dereferenced."""
    L = srt.lib()
    f = L.srt_photon_grid_build_noalloc
    aligned = C.c_void_p(1 << 20)
    st = f(None, C.c_void_p(aligned.value + 8), 10, 0, 0.02, 22, None, None)
    assert srt.STATUS[st] == "INVALID_ARG"
    st = f(None, aligned, 10, 0, 0.02, 22, C.c_void_p(aligned.value + 4), None)
    assert srt.STATUS[st] == "INVALID_ARG"
    st = f(None, aligned, 10, 0, 0.02, 22, None, C.c_void_p(aligned.value + 2))
    assert srt.STATUS[st] == "INVALID_ARG"
    st = f(None, aligned, (1 << 20) + 1, 0, 0.02, 22, None, None)
    assert srt.STATUS[st] == "CAPACITY"
    st = f(None, aligned, 10, 0, 0.0, 22, None, None)
    assert srt.STATUS[st] == "INVALID_ARG"
    st = f(None, None, 10, 0, 0.02, 22, None, None)
    assert srt.STATUS[st] == "INVALID_ARG"
