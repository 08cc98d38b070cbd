"""The headless C++ driver (wgpu_spectral_rt_b200/srt_render): a native
caller of the C ABI that runs the reference engine's loop without a window
(engine.rs:139-244: scene, renderer, per-frame camera uniform with the frame
count, render, screenshot).

CPU: it is built beside the library, links against it and handles its
command line (version, help, bad arguments) without touching a GPU.
GPU: its PNG equals, byte for byte, the screenshot of the same frames rendered
through the Python binding of the same C ABI."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

DRIVER = Path(__file__).resolve().parents[1] / "wgpu_spectral_rt_b200" / "srt_render"


def _run(*args, timeout=120):
    return subprocess.run([str(DRIVER), *map(str, args)], capture_output=True, text=True, timeout=timeout)


def test_driver_is_built_and_parses_its_arguments():
    if not DRIVER.exists():
        from wgpu_spectral_rt_b200 import build

        build.build()
    assert DRIVER.exists()
    p = _run("--version")
    assert p.returncode == 0 and "library ABI 4, header ABI 4" in p.stdout
    p = _run("--help")
    assert p.returncode == 0 and p.stdout.startswith("usage: srt_render")
    for bad in (["--bogus"], ["--width", "0"], ["--preset", "9"], ["--frames"], ["--depth", "x"]):
        p = _run(*bad)
        assert p.returncode == 2, bad
        assert "usage" in p.stderr


@pytest.mark.gpu
def test_driver_png_equals_the_binding_screenshot(srt, ctx, tmp_path):
    w, h, frames = 64, 48, 8
    out = tmp_path / "driver.png"
    p = _run("--preset", 0, "--width", w, "--height", h, "--frames", frames, "--photons", 1 << 16, "--out", out)
    assert p.returncode == 0, p.stderr
    assert f"{w}x{h}, {frames} frames" in p.stdout
    b = srt.SceneBuilder()
    cam = b.add_preset(srt.PRESET_CORNELL_BOX)
    scene = b.build(ctx)
    params = srt.default_params(photons_per_frame=1 << 16)
    r = srt.Renderer(ctx, scene, w, h, params)
    ctl = srt.CameraController(*cam)
    for f in range(frames):
        r.render(ctl.build_uniform(w / h, f))
    ref = tmp_path / "binding.png"
    r.save_screenshot(ref)
    r.close()
    scene.close()
    assert out.read_bytes() == ref.read_bytes()
