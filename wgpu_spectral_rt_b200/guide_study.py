"""Equal-time comparison of guided and plain path tracing against an FP64 reference.

Both arms render the same scene, camera, depth and photon pass.  The
reference image is the plain method accumulated in FP64 over `ref_spp`
frames, on sample streams decorrelated from the two arms (a different
`seed`; the progressive photon radius schedule is the arms' one).  The
guided arm learns online: its training steps run inside its time, and its
image includes the frames rendered while the guide was untrained.

Each arm renders for `seconds` of wall time (frames launched back to back,
the stream synchronised at checkpoints; the image read-back for the error
is outside the timed region).  Reported per arm: frames, ms per frame, and
relMSE (mean over pixels and RGB of (x - ref)^2 / (ref^2 + 0.01)) at each
checkpoint; and the time the guided arm needs to reach the plain arm's
final relMSE, as a fraction of the plain arm's time.

    python -m wgpu_spectral_rt_b200.guide_study --preset 4 --width 1920 --height 1080 \\
        --max-depth 16 --batch 262144 --seconds 20 --ref-spp 65536
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

import wgpu_spectral_rt_b200 as srt

REF_SEED = 0x5EED0001


def relmse(x: np.ndarray, ref: np.ndarray) -> float:
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 0.01)))


def _mean_rgb(r: srt.Renderer) -> np.ndarray:
    a = r.read_accum64()
    return a[..., :3] / a[..., 3:4]


def _renderer(ctx, scene, w, h, flags, max_depth, photons, seed=0):
    p = srt.default_params(photons_per_frame=photons, flags=flags | srt.FLAG_FP64_ACCUM, max_depth=max_depth,
                           seed=seed)
    return srt.Renderer(ctx, scene, w, h, p)


def _render(ctx, r, ctl, aspect, first, count):
    for f in range(first, first + count):
        r.render(ctl.build_uniform(aspect, f))
    ctx.synchronize()


def _arm(ctx, r, ctl, aspect, seconds, ref, n_checkpoints=8):
    """Renders for `seconds`; returns (frames, seconds, [(t, frames, relmse)])."""
    # frames per checkpoint from a short timed probe, then geometric checkpoints
    t0 = time.perf_counter()
    _render(ctx, r, ctl, aspect, 0, 4)
    t_probe = time.perf_counter() - t0
    ms = t_probe / 4
    frames, elapsed = 4, t_probe
    curve = []
    targets = [seconds * (2.0 ** (k - n_checkpoints + 1)) for k in range(n_checkpoints)]
    for tgt in targets:
        n = max(1, int((tgt - elapsed) / ms))
        if elapsed >= tgt:
            n = 0
        t0 = time.perf_counter()
        if n:
            _render(ctx, r, ctl, aspect, frames, n)
        dt = time.perf_counter() - t0
        frames += n
        elapsed += dt
        if n:
            ms = dt / n
        curve.append((round(elapsed, 4), frames, relmse(_mean_rgb(r), ref)))
    return frames, elapsed, curve


def _time_to_reach(curve, target):
    """Interpolated (log-log) time at which the error curve reaches `target`."""
    prev = None
    for t, _, e in curve:
        if e <= target:
            if prev is None:
                return t
            t0, e0 = prev
            if e0 <= e or t0 <= 0:
                return t
            a = (np.log(target) - np.log(e0)) / (np.log(e) - np.log(e0))
            return float(np.exp(np.log(t0) + a * (np.log(t) - np.log(t0))))
        prev = (t, e)
    return None


def study(preset=srt.PRESET_CAUSTIC_SLAB, width=1920, height=1080, max_depth=16, photons=1 << 20, ref_spp=65536,
          seconds=20.0, lr=None, batch=None, guide_bounces=None, training=None):
    """Runs the study.  The reference is rendered as two halves on decorrelated
    streams; their difference estimates the reference's own noise, which every
    measured relMSE contains as a constant floor (E (x - ref)^2 = E (x - mu)^2
    + Var ref for independent x and ref).  The time fraction is reported on
    the raw curves and on the curves with that floor subtracted
    ("time_fraction_ref_noise_subtracted"), which a short reference needs."""
    ctx = srt.Context(0)
    b = srt.SceneBuilder()
    cam = b.add_preset(preset)
    scene = b.build(ctx)
    ctl = srt.CameraController(*cam)
    aspect = width / height
    out = {"scene_preset": preset, "width": width, "height": height, "max_depth": max_depth,
           "photons_per_frame": photons, "ref_spp": ref_spp, "lr": lr if lr is not None else 1e-3,
           "batch": batch if batch else 65536, "seconds": seconds}

    t0 = time.perf_counter()
    halves = []
    for k in range(2):
        ref_r = _renderer(ctx, scene, width, height, 0, max_depth, photons, REF_SEED + k)
        n = ref_spp // 2
        for f0 in range(0, n, 256):
            _render(ctx, ref_r, ctl, aspect, f0, min(256, n - f0))
        halves.append(_mean_rgb(ref_r))
        ref_r.close()
    ref = 0.5 * (halves[0] + halves[1])
    # Var(A - B) = 4 Var(ref) for halves A, B of the reference: its noise floor
    floor = float(np.mean((halves[0] - halves[1]) ** 2 / (ref ** 2 + 0.01))) / 4.0
    out["reference"] = {"frames": 2 * (ref_spp // 2), "seconds": round(time.perf_counter() - t0, 2),
                        "accumulation": "fp64", "seed": REF_SEED, "noise_floor_relmse": floor}

    for name, flags in (("plain", 0), ("guided", srt.FLAG_GUIDING)):
        # warm-up (library load, graph capture) on a throwaway renderer
        w = _renderer(ctx, scene, width, height, flags, max_depth, photons, 7)
        _render(ctx, w, ctl, aspect, 0, 4)
        w.close()
        r = _renderer(ctx, scene, width, height, flags, max_depth, photons)
        if flags:
            r.configure_guide(lr, batch)
            if guide_bounces:
                r.set_guide_bounces(guide_bounces)
            if training is not None:
                r.set_guide_training(training)
        frames, el, curve = _arm(ctx, r, ctl, aspect, seconds, ref)
        out[name] = {"frames": frames, "seconds": round(el, 3), "ms_per_frame": round(1e3 * el / frames, 4),
                     "relmse": curve[-1][2], "curve": curve, "tail_first": r.stats()["tail_first"]}
        if flags:
            out[name]["guide"] = r.guide_info()
        r.close()
    target = out["plain"]["relmse"]
    t_g = _time_to_reach(out["guided"]["curve"], target)
    out["guided_time_to_plain_relmse"] = t_g
    out["time_fraction"] = (t_g / out["plain"]["seconds"]) if t_g is not None else None
    out["relmse_ratio_plain_over_guided"] = target / max(out["guided"]["relmse"], 1e-30)
    # the same with the reference's noise floor taken out of both curves
    sub = [(t, f, e - floor) for t, f, e in out["guided"]["curve"]]
    t_s = _time_to_reach(sub, target - floor) if target > floor else None
    out["time_fraction_ref_noise_subtracted"] = (t_s / out["plain"]["seconds"]) if t_s is not None else None
    out["relmse_ratio_ref_noise_subtracted"] = ((target - floor) / max(out["guided"]["relmse"] - floor, 1e-30)
                                                if target > floor else None)
    # per sample: relMSE x frames (noise floor out), guided over plain; the
    # time fraction is about this times the cost ratio of a guided frame
    if target > floor and out["guided"]["relmse"] > floor:
        out["variance_ratio_per_sample_ref_noise_subtracted"] = (
            (out["guided"]["relmse"] - floor) * out["guided"]["frames"] / ((target - floor) * out["plain"]["frames"]))
    out["cost_ratio_guided_over_plain"] = out["guided"]["ms_per_frame"] / out["plain"]["ms_per_frame"]
    out["guide_bounces"] = guide_bounces
    scene.close()
    ctx.close()
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--preset", type=int, default=srt.PRESET_CAUSTIC_SLAB)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--max-depth", type=int, default=16)
    ap.add_argument("--photons", type=int, default=1 << 20)
    ap.add_argument("--ref-spp", type=int, default=65536)
    ap.add_argument("--seconds", type=float, default=20.0)
    ap.add_argument("--lr", type=float, default=None)
    ap.add_argument("--batch", type=int, default=None, help="training samples per frame")
    ap.add_argument("--guide-bounces", type=int, default=None, help="guide bounces < N only (default 8)")
    ap.add_argument("--training", choices=("mma-sync", "tcgen05"), default=None,
                    help="training kernel (default: the library's)")
    a = ap.parse_args()
    training = {None: None, "mma-sync": srt.GUIDE_TRAIN_MMA_SYNC, "tcgen05": srt.GUIDE_TRAIN_TCGEN05}[a.training]
    print(json.dumps(study(a.preset, a.width, a.height, a.max_depth, a.photons, a.ref_spp, a.seconds, a.lr,
                           a.batch, a.guide_bounces, training)))


if __name__ == "__main__":
    main()
