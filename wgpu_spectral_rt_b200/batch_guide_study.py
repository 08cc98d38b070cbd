"""Equal-time comparison of the guided and the plain batched tracer, per scene.

A batch of seeded scenes (the batched-random preset: displaced icospheres
with GGX, thin-film and dielectric spheres; square viewports drawn from
`resolutions`, photons per frame log-uniform in `photons`) is rendered by
two batched renderers for `seconds` of wall time each: the plain method, and
the guided method in which every scene has its own network, trained online
by the grouped training launches and sampled by the grouped tcgen05
inference launch.  Each scene's reference is the plain method accumulated in
FP64 over `ref_spp` iterations on decorrelated sample streams.

Reported per scene: relMSE of each arm (mean over pixels and RGB of
(x - ref)^2 / (ref^2 + 0.01)), their ratio, and the time the guided arm needs
to reach the plain arm's final relMSE as a fraction of the plain arm's time
(interpolated between checkpoints; None when not reached); plus the
iteration times of both arms.

    python -m wgpu_spectral_rt_b200.batch_guide_study --scenes 16 --seconds 20 --ref-spp 1024
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

import wgpu_spectral_rt_b200 as srt
from wgpu_spectral_rt_b200.guide_study import REF_SEED, _time_to_reach, relmse


def _mean_rgb(r) -> np.ndarray:
    a = r.read_accum64()
    return a[..., :3] / a[..., 3:4]


def _workload(n_scenes, resolutions, photons, seed):
    rng = np.random.default_rng(seed)
    sizes, phot = [], []
    for _ in range(n_scenes):
        r = int(rng.choice(resolutions))
        sizes.append((r, r))
        phot.append(int(round(float(np.exp(rng.uniform(np.log(photons[0]), np.log(photons[1])))))))
    return sizes, phot


def study(n_scenes=16, resolutions=(256, 512, 1024, 2048), photons=(1e6, 16e6), max_depth=12, ref_spp=1024,
          seconds=20.0, seed=777, lr=None, batch=None, n_checkpoints=6):
    ctx = srt.Context(0)
    sizes, phot = _workload(n_scenes, resolutions, photons, seed)
    scenes, ctls = [], []
    for s in range(n_scenes):
        b = srt.SceneBuilder()
        cam = b.add_preset(srt.PRESET_BATCH_RANDOM, s)
        scenes.append(b.build(ctx))
        ctls.append(srt.CameraController(*cam))

    def params(flags, seed0):
        return [srt.default_params(photons_per_frame=phot[i], max_depth=max_depth, seed=seed0 + i,
                                   flags=flags | srt.FLAG_FP64_ACCUM) for i in range(n_scenes)]

    def cams(f):
        return [c.build_uniform(w / h, f) for c, (w, h) in zip(ctls, sizes)]

    def render(bt, first, count):
        for f in range(first, first + count):
            bt.render(cams(f))
        ctx.synchronize()

    out = {"scenes": n_scenes, "sizes": [w for w, _ in sizes], "photons_per_frame": phot,
           "triangles": [sc.info()["triangles"] for sc in scenes], "max_depth": max_depth, "ref_spp": ref_spp,
           "seconds": seconds, "lr": lr if lr is not None else 1e-3, "batch": batch if batch else 65536}

    t0 = time.perf_counter()
    ref_b = srt.Batch(ctx, scenes, sizes, params(0, REF_SEED))
    for f0 in range(0, ref_spp, 64):
        render(ref_b, f0, min(64, ref_spp - f0))
    refs = [_mean_rgb(x) for x in ref_b.renderers]
    ref_b.close()
    out["reference"] = {"iterations": ref_spp, "seconds": round(time.perf_counter() - t0, 2),
                        "accumulation": "fp64", "seed": REF_SEED}

    for name, flags in (("plain", 0), ("guided", srt.FLAG_GUIDING)):
        # warm-up (library, graph capture, allocator) on a throwaway batch
        w = srt.Batch(ctx, scenes, sizes, params(flags, 991))
        render(w, 0, 2)
        w.close()
        bt = srt.Batch(ctx, scenes, sizes, params(flags, 0))
        if flags:
            for x in bt.renderers:
                x.configure_guide(lr, batch)
        t0 = time.perf_counter()
        render(bt, 0, 2)
        elapsed = time.perf_counter() - t0
        frames, ms = 2, elapsed / 2
        curve = []
        targets = [seconds * (2.0 ** (k - n_checkpoints + 1)) for k in range(n_checkpoints)]
        for tgt in targets:
            n = max(1, int((tgt - elapsed) / ms)) if elapsed < tgt else 0
            t0 = time.perf_counter()
            if n:
                render(bt, frames, n)
            dt = time.perf_counter() - t0
            frames += n
            elapsed += dt
            if n:
                ms = dt / n
            errs = [relmse(_mean_rgb(x), refs[i]) for i, x in enumerate(bt.renderers)]
            curve.append((round(elapsed, 4), frames, errs))
        out[name] = {"iterations": frames, "seconds": round(elapsed, 3),
                     "ms_per_iteration": round(1e3 * elapsed / frames, 3), "curve": curve}
        if flags:
            out[name]["adam_steps"] = [x.guide_info()["adam_steps"] for x in bt.renderers]
        bt.close()

    per = []
    for i in range(n_scenes):
        e_p = out["plain"]["curve"][-1][2][i]
        e_g = out["guided"]["curve"][-1][2][i]
        t_g = _time_to_reach([(t, f, e[i]) for t, f, e in out["guided"]["curve"]], e_p)
        per.append({"scene": i, "size": sizes[i][0], "triangles": out["triangles"][i], "relmse_plain": e_p,
                    "relmse_guided": e_g, "ratio_plain_over_guided": e_p / max(e_g, 1e-30),
                    "time_fraction": (t_g / out["plain"]["seconds"]) if t_g is not None else None})
    out["per_scene"] = per
    ratios = np.array([p["ratio_plain_over_guided"] for p in per])
    out["geomean_ratio_plain_over_guided"] = float(np.exp(np.mean(np.log(ratios))))
    out["scenes_improved"] = int(np.sum(ratios > 1.0))
    for s in scenes:
        s.close()
    ctx.close()
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--scenes", type=int, default=16)
    ap.add_argument("--resolutions", type=str, default="256,512,1024,2048")
    ap.add_argument("--photons", type=str, default="1e6,16e6", help="log-uniform range of photons per frame")
    ap.add_argument("--max-depth", type=int, default=12)
    ap.add_argument("--ref-spp", type=int, default=1024)
    ap.add_argument("--seconds", type=float, default=20.0)
    ap.add_argument("--seed", type=int, default=777)
    ap.add_argument("--lr", type=float, default=None)
    ap.add_argument("--batch", type=int, default=None, help="training samples per frame and scene")
    a = ap.parse_args()
    res = tuple(int(x) for x in a.resolutions.split(","))
    ph = tuple(float(x) for x in a.photons.split(","))
    print(json.dumps(study(a.scenes, res, ph, a.max_depth, a.ref_spp, a.seconds, a.seed, a.lr, a.batch)))


if __name__ == "__main__":
    main()
