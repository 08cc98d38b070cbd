"""Equal-time and equal-sample comparison of guided and plain path tracing.

Both renderers run the same scene and camera without the photon pass (so the
comparison is about the sampling of the diffuse continuation alone).  The
reference image is plain path tracing accumulated in FP64 over `ref_spp`
frames whose sample streams are disjoint from the compared runs (frame
indices offset by 2^30).  The guided renderer learns online: its training
steps run inside its time budget, and its image includes the frames
rendered while the guide was still untrained.

    python -m wgpu_spectral_rt_b200.guide_study --seconds 2 --ref-spp 65536

prints one JSON object: per arm the frames rendered, ms per frame and the
relMSE, mean over pixels and RGB of (x - ref)^2 / (ref^2 + 0.01).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

import wgpu_spectral_rt_b200 as srt

REF_FRAME_OFFSET = 1 << 30


def relmse(x: np.ndarray, ref: np.ndarray) -> float:
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 0.01)))


def _mean_rgb(r: srt.Renderer) -> np.ndarray:
    a = r.read_accum64()
    return a[..., :3] / a[..., 3:4]


def _renderer(ctx, scene, w, h, flags, max_depth):
    p = srt.default_params(photons_per_frame=0, flags=flags | srt.FLAG_FP64_ACCUM, max_depth=max_depth)
    return srt.Renderer(ctx, scene, w, h, p)


def _run_for(ctx, r, ctl, aspect, seconds=None, frames=None, offset=0, chunk=8):
    """Renders until `seconds` of wall time (synchronised every `chunk`
    frames) or `frames` frames; returns (frames, seconds)."""
    ctx.synchronize()
    t0 = time.perf_counter()
    f = 0
    while True:
        for _ in range(chunk):
            r.render(ctl.build_uniform(aspect, offset + f))
            f += 1
            if frames is not None and f >= frames:
                break
        ctx.synchronize()
        el = time.perf_counter() - t0
        if (frames is not None and f >= frames) or (seconds is not None and el >= seconds):
            return f, el


def study(preset=srt.PRESET_INDIRECT_ROOM, width=256, height=192, ref_spp=65536, seconds=2.0, max_depth=12,
          equal_spp=None, lr=None, batch=None):
    ctx = srt.Context(0)
    b = srt.SceneBuilder()
    cam = b.add_preset(preset)
    scene = b.build(ctx)
    ctl = srt.CameraController(*cam)
    aspect = width / height
    out = {"scene_preset": preset, "width": width, "height": height, "max_depth": max_depth, "ref_spp": ref_spp,
           "photons_per_frame": 0, "lr": lr, "batch": batch}

    ref_r = _renderer(ctx, scene, width, height, 0, max_depth)
    f, el = _run_for(ctx, ref_r, ctl, aspect, frames=ref_spp, offset=REF_FRAME_OFFSET, chunk=64)
    ref = _mean_rgb(ref_r)
    out["reference"] = {"frames": f, "seconds": round(el, 3)}
    ref_r.close()

    arms = {"plain": 0, "guided": srt.FLAG_GUIDING}
    for name, flags in arms.items():
        r = _renderer(ctx, scene, width, height, flags, max_depth)
        if flags:
            r.configure_guide(lr, batch)
        # warm-up (graph capture, first-launch costs) on a throwaway renderer state
        _run_for(ctx, r, ctl, aspect, frames=8, offset=REF_FRAME_OFFSET // 2)
        r.close()
        r = _renderer(ctx, scene, width, height, flags, max_depth)
        if flags:
            r.configure_guide(lr, batch)
        f, el = _run_for(ctx, r, ctl, aspect, seconds=seconds)
        img = _mean_rgb(r)
        arm = {"frames": f, "seconds": round(el, 3), "ms_per_frame": round(1e3 * el / f, 4),
               "relmse_equal_time": relmse(img, ref)}
        if equal_spp:
            r2 = _renderer(ctx, scene, width, height, flags, max_depth)
            if flags:
                r2.configure_guide(lr, batch)
            _run_for(ctx, r2, ctl, aspect, frames=equal_spp)
            arm["relmse_equal_spp"] = relmse(_mean_rgb(r2), ref)
            r2.close()
        out[name] = arm
        r.close()
    out["equal_spp"] = equal_spp
    out["relmse_ratio_plain_over_guided_equal_time"] = out["plain"]["relmse_equal_time"] / max(
        out["guided"]["relmse_equal_time"], 1e-30)
    if equal_spp:
        out["relmse_ratio_plain_over_guided_equal_spp"] = out["plain"]["relmse_equal_spp"] / max(
            out["guided"]["relmse_equal_spp"], 1e-30)
    scene.close()
    ctx.close()
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--preset", type=int, default=srt.PRESET_INDIRECT_ROOM)
    ap.add_argument("--width", type=int, default=256)
    ap.add_argument("--height", type=int, default=192)
    ap.add_argument("--ref-spp", type=int, default=65536)
    ap.add_argument("--seconds", type=float, default=2.0)
    ap.add_argument("--max-depth", type=int, default=12)
    ap.add_argument("--equal-spp", type=int, default=0)
    ap.add_argument("--lr", type=float, default=None)
    ap.add_argument("--batch", type=int, default=None, help="training samples per frame")
    a = ap.parse_args()
    print(json.dumps(study(a.preset, a.width, a.height, a.ref_spp, a.seconds, a.max_depth, a.equal_spp or None,
                           a.lr, a.batch)))


if __name__ == "__main__":
    main()
