"""Benchmark of the spectral path-tracing hot path on B200.

Workload (default): the plain method at scale — a level-8 displaced
icosphere (1,310,720 triangles) plus 64 thin-film-coated GGX spheres
(4,032 triangles each) in a lit room, 1920x1080, max depth 12, 4M photons
per frame (2^22), 4 hero wavelengths, FP32 transport.  One step = one frame
= one sample per pixel (photon emit -> grid -> wavefront camera paths ->
accumulate + tonemap), so the default 64 steps are the 64-spp image.

Metric: Mpaths/s (camera paths per second, whole job).  Mphotons/s and
Mrays/s are reported beside it.

  value       device time (CUDA events on the library's stream) of K frames
              with every input resident in HBM
  e2e         the same frames through the public C ABI with host buffers:
              the camera uniform is copied from host memory and the RGBA8
              image is read back to host memory every step
  roofline    the closest-hit traversal kernel: algorithmic bytes per
              launch (32 B ray + 16 B hit per ray, 80 B per BVH8 node
              visited, 48 B per triangle tested; visit counts from a
              counting build over the same frames) / its mean CUDA-event
              duration, against the measured HBM copy bandwidth
  cpu_baseline  the CPU oracle (C++ restatement of the reference shader
              math, OpenMP over all host threads) on one whole frame of the
              same workload, with the oracle's own scene generator

Multi-GPU: the path does not shard across GPUs (one frame is one GPU's
work); --gpus N under torchrun runs N replicas, each rendering its own
sample stream (frame offset = rank * steps), value = all ranks' paths / the
max over ranks of the timed region ("scaling": "weak").

--impl reference times the reference's CPU implementation of the path — the
oracle port (the reference itself is Rust + WGSL on a Vulkan ray-query
device and cannot run here) — with all host threads, on the same workload
and metric, one whole frame per timed step; rank 0 only.  It builds its
scene and camera with the oracle's own generator and loads nothing of the
GPU package.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CONFIGS = {
    # name: (preset, width, height, max_depth, photons per frame)
    "config2": ("PRESET_CONFIG2", 1920, 1080, 12, 1 << 22),
    "config1": ("PRESET_CONFIG1", 256, 256, 8, 1 << 18),
}
# srt_preset values (include/srt.h), for the CPU legs that do not load the GPU package
PRESET_IDS = {"PRESET_CONFIG1": 2, "PRESET_CONFIG2": 3}


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic_from_profile(name: str, rays_per_launch: float):
    """DRAM bytes per launch of the traversal kernel: the per-ray DRAM traffic of a
    committed ncu capture scaled to this run's rays per launch (None without one)."""
    p = ROOT / "profiles" / f"{name}.json"
    if p.exists():
        d = json.loads(p.read_text())
        return round(d["dram_bytes_per_ray"] * rays_per_launch), d.get("note")
    return None, None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def rank_frame_offset(rank: int, steps: int, warmup: int) -> int:
    """First frame index of a replica: each rank renders its own sample stream."""
    return rank * (steps + warmup)


def replica_reduce(local_ms: float, local_paths: int, dist=None, device="cpu"):
    """(max over ranks of the timed region in ms, paths summed over ranks).

    Replicas never exchange path data; the only collectives are this timing
    reduction and the barriers around the timed region."""
    if dist is None:
        return local_ms, local_paths
    import torch

    t = torch.tensor([local_ms], dtype=torch.float64, device=device)
    p = torch.tensor([local_paths], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(p, op=dist.ReduceOp.SUM)
    return float(t.item()), int(p.item())


def build_scene(srt, ctx, preset_name: str, seed: int = 0):
    b = srt.SceneBuilder()
    cam = b.add_preset(getattr(srt, preset_name), seed)
    scene = b.build(ctx)
    return b, scene, cam


def _oracle():
    sys.path.insert(0, str(ROOT / "oracle"))
    import binding as orc  # the oracle: timed as the CPU baseline, never part of the GPU path

    return orc


def _cpu_frame(orc, o, preset_cam, w, h, depth, photons, frame, fraction=1):
    """One frame of the oracle port (all host threads): rows y % fraction == 0
    and 1/fraction of the photons (fraction 1 = the whole frame).  Returns
    (seconds, stats [paths, closest rays, shadow rays, emitted, stored])."""
    pos, yaw, pitch = preset_cam
    u = orc.camera_uniform(pos, yaw, pitch, w / h, frame)
    p = orc.default_params(max_depth=depth, photons_per_frame=max(1, photons // fraction),
                           photon_norm_count=float(photons))
    t = time.perf_counter()
    _, _, _, st = o.render_frame(u, w, h, p, row_stride=fraction, row_phase=0, want_ldr=False)
    return time.perf_counter() - t, st


def cpu_baseline(cfg, frames=1):
    """The CPU oracle (the reference's shader math restated in C++, OpenMP over
    all host threads) on whole frames of the same workload: its own scene
    generator and camera, the same sampling as the reference arm's steps."""
    orc = _oracle()
    preset, w, h, depth, photons = cfg
    t0 = time.perf_counter()
    scn = orc.Preset(PRESET_IDS[preset], 0)
    o = orc.OracleScene(scn.arrays())
    build_s = time.perf_counter() - t0
    _cpu_frame(orc, o, scn.camera, w, h, depth, photons, 0, fraction=16)  # warm-up (page-in, thread pool)
    dt_total, paths, st_sum = 0.0, 0, np.zeros(5, np.uint64)
    for f in range(frames):
        dt, st = _cpu_frame(orc, o, scn.camera, w, h, depth, photons, 1 + f)
        dt_total += dt
        paths += int(st[0])
        st_sum += st
    value = paths / dt_total / 1e6
    out = {
        "value": round(value, 4), "unit": "Mpaths/s", "cores": orc.max_threads(), "kind": "port",
        "sample": (f"{frames} whole {w}x{h} frame(s) ({paths} paths, {photons} photons each), "
                   f"{dt_total:.1f} s; oracle scene generator + FP64 BVH build {build_s:.1f} s not timed"),
        "rays_closest": int(st_sum[1]), "rays_shadow": int(st_sum[2]), "seconds": round(dt_total, 3),
    }
    o.close()
    scn.close()
    return out


def reference_shaders_sample(cfg, frames=1):
    """The reference's own WGSL (shader.wgsl, photon_emit.wgsl, build_grid.wgsl),
    translated mechanically to C++ (oracle/_ref, built from the reference tree by
    oracle/wgsl_translate.py), timed on whole frames on all host threads: its
    photon and grid dispatches and its camera pass run their invocations
    concurrently, ray queries answered by the oracle's FP64 BVH.  Its constants
    are its own: 2^20 photons per frame (the shaders fix the dispatch and the
    gather's normalisation) and MAX_DEPTH = the workload's depth; material type
    5, which the reference lacks, is replaced by its GGX, glass and film types.
    None of the GPU package is loaded.  A sample beside the arm's value (the
    oracle port, which takes the workload's photon count), not the value."""
    orc = _oracle()
    import ref_binding as ref

    if not ref.available():
        return {"unavailable": "oracle/_ref/libref_wgsl.so not built here (it is built from the reference tree)"}
    preset, w, h, depth, _photons = cfg
    scn = orc.Preset(PRESET_IDS[preset], 0)
    arrays, keep = ref.reference_materials(scn.arrays())
    rs = ref.RefScene(arrays)
    pos, yaw, pitch = scn.camera
    # warm-up (page-in, thread pool): a small crop with few emitters
    rs.render_frame(orc.camera_uniform(pos, yaw, pitch, w / h, 0), 64, 36, depth, 1 << 14, ordered=False)
    t_total = 0.0
    for f in range(frames):
        u = orc.camera_uniform(pos, yaw, pitch, w / h, 1 + f)
        t0 = time.perf_counter()
        rs.render_frame(u, w, h, depth, ref.MAX_PHOTONS, ordered=False)
        t_total += time.perf_counter() - t0
    rs.close()
    del keep
    return {"value": round(w * h * frames / t_total / 1e6, 4), "unit": "Mpaths/s", "kind": "reference",
            "cores": orc.max_threads(), "frames": frames, "seconds": round(t_total, 2),
            "sample": (f"{frames} whole {w}x{h} frame(s) of the reference's own WGSL translated to C++ "
                       f"(oracle/wgsl_translate.py), its constants: 2^20 photons, MAX_DEPTH {depth}; "
                       f"type-5 materials as reference types; FP64 ray queries")}


def run_reference(args, cfg, rank, world):
    """--impl reference: the CPU port of the reference path (the oracle, with
    its own scene generator and camera; nothing of the GPU package is loaded),
    all host threads, rank 0 only.  A timed step is one whole frame of the
    workload; the untimed warm-up steps render 1/16 of a frame."""
    if rank != 0:
        return 0
    orc = _oracle()
    preset, w, h, depth, photons = cfg
    scn = orc.Preset(PRESET_IDS[preset], 0)
    o = orc.OracleScene(scn.arrays())
    n_tris = o.n_tris
    for k in range(args.warmup):
        _cpu_frame(orc, o, scn.camera, w, h, depth, photons, k, fraction=16)
    total_paths, t_total = 0, 0.0
    for k in range(args.steps):
        dt, st = _cpu_frame(orc, o, scn.camera, w, h, depth, photons, args.warmup + k)
        total_paths += int(st[0])
        t_total += dt
    value = total_paths / t_total / 1e6
    cores = orc.max_threads()
    line = {
        "metric": "Mpaths/s", "value": round(value, 4), "unit": "Mpaths/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * t_total / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (procedural scene, seeded)",
        "impl": "reference",
        "config": {"workload": (f"{args.config}: {n_tris} triangles, {w}x{h}, depth {depth}, {photons} "
                                f"photons/frame, 1 spp per step"),
                   "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": round(value, 4), "unit": "Mpaths/s", "cores": cores, "kind": "port",
                         "sample": (f"per timed step one whole {w}x{h} frame ({photons} photons); warm-up steps "
                                    f"1/16 of a frame")},
        "e2e": {"value": round(value, 4), "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    o.close()
    scn.close()
    if not args.no_cpu_baseline:
        try:
            line["reference_shaders"] = reference_shaders_sample(cfg)
        except Exception as e:  # a sample beside the value: never costs the arm its line
            line["reference_shaders"] = {"unavailable": f"{type(e).__name__}: {e}"[:200]}
    print(json.dumps(line), flush=True)
    return 0


def _pcg(v: int) -> int:
    state = (v * 747796405 + 2891336453) & 0xFFFFFFFF
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & 0xFFFFFFFF
    return ((word >> 22) ^ word) & 0xFFFFFFFF


def batch_seeds(n: int, base: int = 0) -> list[int]:
    """Seeds of the seeded batch scene (PRESET_BATCH_RANDOM) whose triangle
    budgets fall one into each of n equal strata of log [1e4, 2e6].  The
    preset draws its budget from the seed as exp(log 1e4 + u log 200), u the
    first draw of its PCG stream (pcg(pcg(seed * 747796405 + 2891336453)) /
    2^32), so the stratified choice spans the configured range (up to the 2M
    triangles of the largest scenes) instead of leaving its ends to chance."""
    chosen: list[int | None] = [None] * n
    seed = base
    while any(c is None for c in chosen):
        u = _pcg(_pcg((seed * 747796405 + 2891336453) & 0xFFFFFFFF)) / 4294967296.0
        k = min(n - 1, int(u * n))
        if chosen[k] is None:
            chosen[k] = seed
        seed += 1
    return [int(c) for c in chosen]


def batched_section(srt, ctx, stream, n_scenes=32, seed=12345):
    """C3: n seeded scenes with triangle budgets stratified over log [1e4, 2e6],
    square viewports of 256..1024, 1M..8M photons and 16..256 spp each
    (log-uniform): the batched renderer (after autotuning) renders every scene
    to its own spp count, scenes dropping out of the iterations as they finish;
    against the same scenes rendered one after another with single-scene
    renderers."""
    import torch

    rng = np.random.default_rng(seed)
    seeds = batch_seeds(n_scenes)
    scenes, ctls, sizes, params, spp = [], [], [], [], []
    for s in seeds:
        b = srt.SceneBuilder()
        cam = b.add_preset(srt.PRESET_BATCH_RANDOM, s)
        scenes.append(b.build(ctx))
        ctls.append(srt.CameraController(*cam))
        r = int(rng.choice([256, 512, 768, 1024]))
        sizes.append((r, r))
        ph = int(round(float(np.exp(rng.uniform(np.log(1e6), np.log(8e6))))))
        params.append(srt.default_params(photons_per_frame=ph, seed=s))
        spp.append(int(round(float(np.exp(rng.uniform(np.log(16), np.log(256)))))))
    tris = [sc.info()["triangles"] for sc in scenes]
    paths = sum(w * h * k for (w, h), k in zip(sizes, spp))
    photons = sum(p.photons_per_frame * k for p, k in zip(params, spp))
    iters = max(spp)

    def cams(f):
        return [c.build_uniform(w / h, f) for c, (w, h) in zip(ctls, sizes)]

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    singles = [srt.Renderer(ctx, sc, w, h, p) for sc, (w, h), p in zip(scenes, sizes, params)]
    for i, r in enumerate(singles):  # warm-up: graph capture
        r.render(ctls[i].build_uniform(sizes[i][0] / sizes[i][1], 0))

    def seq():
        for i, r in enumerate(singles):
            w, h = sizes[i]
            for f in range(spp[i]):
                r.render(ctls[i].build_uniform(w / h, f))

    ms_seq = timed(seq)
    for r in singles:
        r.close()
    batch = srt.Batch(ctx, scenes, sizes, params)
    tune = batch.autotune(cams(0), iterations=1)
    batch.render(cams(0))
    for k in range(1, 8):  # warm-up of the active sets near the end
        batch.render(cams(0), active=[k * 32 <= x for x in spp])
    for r in batch.renderers:
        r.reset_accumulation()
        r.reset_stats()

    def run():
        for f in range(iters):
            batch.render(cams(f), active=[f < x for x in spp])

    ms_batch = timed(run)
    frames = [r.stats()["frames"] for r in batch.renderers]
    batch.close()
    for sc in scenes:
        sc.close()
    return {"workload": (f"C3: {n_scenes} seeded scenes (budgets stratified over log [1e4, 2e6]), "
                         f"{min(tris)}..{max(tris)} triangles, viewports 256^2..1024^2, {min(spp)}..{max(spp)} spp "
                         f"per scene ({sum(spp)} scene-frames), {paths} paths and {photons} photons in all, depth 12"),
            "iterations": iters, "ms_total": round(ms_batch, 2),
            "mpaths_per_s": round(paths / ms_batch / 1e3, 2), "mphotons_per_s": round(photons / ms_batch / 1e3, 2),
            "sequential_ms_total": round(ms_seq, 2), "speedup_vs_sequential": round(ms_seq / ms_batch, 3),
            "frames_rendered_match_spp": frames[: len(spp)] == spp, "tuning": tune,
            "grid_cell": "0.02, fixed: the cell size changes the photon density estimate (the image), so it is not "
                         "a speed knob of the compatible renderer"}


def config1_section(srt, ctx, stream, cpu=True):
    """C1 as a whole (Cornell walls + 2-triangle light + dispersive UV sphere,
    256x256, 16 spp, depth 8, 2^18 photons per frame): the GPU renderer timed
    with CUDA events after warm-up, and the CPU oracle port on the same 16
    frames (all host threads)."""
    import torch

    preset, w, h, depth, photons = CONFIGS["config1"]
    _, scene, cam = build_scene(srt, ctx, preset)
    pos, yaw, pitch = cam
    r = srt.Renderer(ctx, scene, w, h, srt.default_params(max_depth=depth, photons_per_frame=photons))
    spp = 16
    r.render(srt.camera_uniform(pos, yaw, pitch, w / h, 0))
    ctx.synchronize()
    for k in range(1, 4):
        r.render(srt.camera_uniform(pos, yaw, pitch, w / h, k))
    ctx.synchronize()
    r.reset_stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(spp):
        r.render(srt.camera_uniform(pos, yaw, pitch, w / h, k))
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    st = r.stats()
    rays = st["rays_closest"] + st["rays_shadow"] + st["rays_photon"]
    out = {"workload": f"C1: {scene.info()['triangles']} triangles, {w}x{h}, {spp} spp, depth {depth}, {photons} "
                       f"photons/frame",
           "gpu": {"ms_total": round(ms, 3), "mpaths_per_s": round(w * h * spp / ms / 1e3, 2),
                   "mphotons_per_s": round(photons * spp / ms / 1e3, 2), "mrays_per_s": round(rays / ms / 1e3, 2)}}
    r.close()
    scene.close()
    if cpu:
        c = cpu_baseline(CONFIGS["config1"], frames=spp)
        out["cpu"] = {"mpaths_per_s": c["value"], "cores": c["cores"], "seconds": c["seconds"],
                      "mphotons_per_s": round(photons * spp / c["seconds"] / 1e6, 3),
                      "mrays_per_s": round((c["rays_closest"] + c["rays_shadow"]) / c["seconds"] / 1e6, 3),
                      "kind": "port"}
    return out


def guided_section(seconds=30.0, ref_spp=8192):
    """C4 at full size (1920x1080, depth 16): equal-time relMSE of guided vs
    plain against an FP64 reference of ref_spp frames rendered in two halves
    (their difference measures the reference's own noise, reported and
    subtracted as the constant floor it adds to every relMSE)."""
    from wgpu_spectral_rt_b200 import guide_study

    d = guide_study.study(preset=4, width=1920, height=1080, max_depth=16, photons=1 << 20, ref_spp=ref_spp,
                          seconds=seconds, batch=1 << 18)
    return {"workload": f"C4 1920x1080 (slab + slit light), depth 16, 2^20 photons, 2^18 training samples/frame, "
                        f"Adam lr 1e-3; reference {ref_spp} spp FP64 in two halves, {seconds} s per arm",
            "relmse_plain": round(d["plain"]["relmse"], 6), "relmse_guided": round(d["guided"]["relmse"], 6),
            "reference_noise_floor": round(d["reference"]["noise_floor_relmse"], 6),
            "relmse_ratio_plain_over_guided": round(d["relmse_ratio_plain_over_guided"], 3),
            "time_fraction_to_plain_relmse": (round(d["time_fraction"], 3) if d["time_fraction"] else None),
            "time_fraction_ref_noise_subtracted": (round(d["time_fraction_ref_noise_subtracted"], 3)
                                                   if d["time_fraction_ref_noise_subtracted"] else None),
            "ms_per_frame_plain": d["plain"]["ms_per_frame"], "ms_per_frame_guided": d["guided"]["ms_per_frame"],
            "cost_ratio_guided_over_plain": round(d["cost_ratio_guided_over_plain"], 3),
            "variance_ratio_per_sample_ref_noise_subtracted": (
                round(d["variance_ratio_per_sample_ref_noise_subtracted"], 3)
                if d.get("variance_ratio_per_sample_ref_noise_subtracted") else None),
            "tail_first_plain": d["plain"]["tail_first"], "tail_first_guided": d["guided"]["tail_first"],
            "guided_bounces": d["guide_bounces"] or "0..7 (the library default)"}


def batched_guided_section(seconds=4.0, ref_spp=256):
    """C5 reduced (full-size study: wgpu_spectral_rt_b200.batch_guide_study): 16 seeded scenes, each
    with its own online-trained network, in one batched renderer (grouped guide launches) vs the
    plain batched renderer at equal time, per-scene relMSE against FP64 plain references."""
    from wgpu_spectral_rt_b200 import batch_guide_study

    d = batch_guide_study.study(n_scenes=16, resolutions=(64, 128, 256, 512), photons=(0.25e6, 4e6),
                                max_depth=12, ref_spp=ref_spp, seconds=seconds)
    return {"workload": (f"C5 reduced: 16 scenes ({min(d['triangles'])}..{max(d['triangles'])} triangles), "
                         f"viewports 64^2..512^2, 0.25M..4M photons, depth 12, one network per scene; "
                         f"reference {ref_spp} iterations FP64, {seconds} s per arm"),
            "ms_per_iteration_plain": d["plain"]["ms_per_iteration"],
            "ms_per_iteration_guided": d["guided"]["ms_per_iteration"],
            "geomean_relmse_ratio_plain_over_guided": round(d["geomean_ratio_plain_over_guided"], 3),
            "scenes_improved": d["scenes_improved"]}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=64)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="config2", choices=sorted(CONFIGS))
    ap.add_argument("--width", type=int, default=0)
    ap.add_argument("--height", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-roofline", action="store_true")
    ap.add_argument("--no-config1", action="store_true", help="skip the C1 section (GPU and CPU)")
    ap.add_argument("--no-batched", action="store_true", help="skip the C3 batched-renderer section")
    ap.add_argument("--no-guided", action="store_true", help="skip the C4 guided-vs-plain section")
    ap.add_argument("--no-batched-guided", action="store_true", help="skip the C5 batched-guiding section")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    preset, w, h, depth, photons = CONFIGS[args.config]
    if args.width:
        w = args.width
    if args.height:
        h = args.height
    cfg = (preset, w, h, depth, photons)
    if args.impl == "reference":
        return run_reference(args, cfg, rank, world)

    import torch

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import wgpu_spectral_rt_b200 as srt

    stream = torch.cuda.Stream(device=local_rank)
    ctx = srt.Context(local_rank, stream.cuda_stream)
    b, scene, cam = build_scene(srt, ctx, preset)
    info = scene.info()
    pos, yaw, pitch = cam
    params = srt.default_params(max_depth=depth, photons_per_frame=photons)
    r = srt.Renderer(ctx, scene, w, h, params)
    f0 = rank_frame_offset(rank, args.steps, args.warmup)

    def cam_u(k):
        return srt.camera_uniform(pos, yaw, pitch, w / h, f0 + k)

    for k in range(args.warmup):
        r.render(cam_u(k))
        if k == 0:
            # the renderer picks its tail start from the first frame's path
            # counts; they are back before the second warm-up frame
            ctx.synchronize()
    ctx.synchronize()
    r.reset_stats()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        start.record(stream)
        for k in range(args.steps):
            r.render(cam_u(args.warmup + k))
        end.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = start.elapsed_time(end)
    st = r.stats()
    ms_max, paths_all = replica_reduce(ms, w * h * args.steps, dist, f"cuda:{local_rank}")
    value = paths_all / (ms_max * 1e-3) / 1e6
    photons_all = photons * args.steps * world
    rays_all = (st["rays_closest"] + st["rays_shadow"] + st["rays_photon"]) * world

    # ---- end to end through the C ABI with host buffers: the camera uniform goes
    # in from pinned memory each step, and each step's RGBA8 image comes back to
    # pinned host memory (srt_read_ldr_async); the host waits for frame k's image
    # after launching frame k + 1, and for the last one before the clock stops
    # (at least 48 frames: the host clock over a fraction of a second is jittery)
    e2e_steps = 0 if args.no_e2e else max(48, args.steps // 2)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    checksum = 0
    tickets = []
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        r.render(cam_u(args.warmup + args.steps + k))
        tickets.append(r.read_ldr_async())
        if k >= 1:
            checksum += int(r.ldr_wait(tickets[k - 1])[h // 2, w // 2, 0])
    if e2e_steps:
        checksum += int(r.ldr_wait(tickets[-1])[h // 2, w // 2, 0])
    t1 = time.perf_counter()
    te = torch.tensor([t1 - t0], dtype=torch.float64, device=f"cuda:{local_rank}")
    if dist:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = w * h * e2e_steps * world / float(te.item()) / 1e6 if e2e_steps else None

    # ---- roofline of the closest-hit traversal kernel: timing pass + counting pass
    roof = None
    if rank == 0 and not args.no_roofline:
        rt = srt.Renderer(ctx, scene, w, h, srt.default_params(max_depth=depth, photons_per_frame=photons,
                                                               flags=srt.FLAG_STAGE_TIMING))
        rc = srt.Renderer(ctx, scene, w, h, srt.default_params(max_depth=depth, photons_per_frame=photons,
                                                               flags=srt.FLAG_COUNT_VISITS))
        # one frame first: the renderers choose their tail start from its path counts
        rt.render(cam_u(0))
        rc.render(cam_u(0))
        ctx.synchronize()
        rt.reset_stats()
        rc.reset_stats()
        nf = 4
        for k in range(nf):
            rt.render(cam_u(1 + k))
            rc.render(cam_u(1 + k))
        s1, s2 = rt.stats(), rc.stats()
        bt, bc = rt.bounce_stats(), rc.bounce_stats()
        tail = int(s1["tail_first"])  # bounces >= tail run in the tail kernel
        launches = s1["launches_trace_closest"]  # closest-hit launches of bounces < tail
        ms_launch = s1["ms_trace_closest"] / launches
        rays = int(bc["rays"][0][:tail].sum())
        alg_bytes = rays * (32 + 16) + float(bc["nodes"][0][:tail].sum()) * 80 + float(bc["tris"][0][:tail].sum()) * 48
        bytes_launch = alg_bytes / launches
        achieved = bytes_launch / (ms_launch * 1e-3) / 1e9
        peak, peak_kind = _peaks()
        traffic, tnote = _traffic_from_profile(f"trace_closest_{args.config}", rays / launches)
        roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "kernel": "camera closest-hit traversal: k_trace (bounce 0) and k_trace_pt (bounces 1..tail-1), "
                          "trace_kernels.cu",
                "peak_source": f"{peak_kind} HBM copy bandwidth (MEASURED_PEAKS.json hbm_gbs)",
                "bytes_per_launch": round(bytes_launch), "ms_per_launch": round(ms_launch, 4),
                "nodes_per_ray": round(float(bc["nodes"][0][:tail].sum()) / max(1, rays), 2),
                "tris_per_ray": round(float(bc["tris"][0][:tail].sum()) / max(1, rays), 2),
                "stage_ms_per_frame": {k: round(s1[k] / nf, 3) for k in
                                       ("ms_photon_pass", "ms_raygen", "ms_trace_closest", "ms_shade",
                                        "ms_trace_shadow", "ms_tail", "ms_finalize")}}
        if traffic is not None:
            roof["traffic_note"] = tnote
        # per bounce: rays, algorithmic GB/s of the closest-hit launch, node
        # visits per ray; the bounces from `tail` on run in the tail kernel
        per = []
        for k in range(min(tail, depth)):
            rays_k = float(bc["rays"][0][k]) / nf
            bytes_k = (float(bc["rays"][0][k]) * 48 + float(bc["nodes"][0][k]) * 80 + float(bc["tris"][0][k]) * 48) / nf
            ms_k = float(bt["ms"][0][k]) / nf
            per.append({"bounce": k, "rays": round(rays_k), "ms": round(ms_k, 4),
                        "gbs": round(bytes_k / (ms_k * 1e-3) / 1e9, 1) if ms_k > 0 else None,
                        "nodes_per_ray": round(float(bc["nodes"][0][k]) / max(1.0, float(bc["rays"][0][k])), 2),
                        "shadow_rays": round(float(bc["rays"][1][k]) / nf),
                        "shadow_ms": round(float(bt["ms"][1][k]) / nf, 4)})
        roof["per_bounce_closest"] = per
        if tail < depth:
            # the tail kernel: closest-hit and shadow traversal of the last bounces plus their shading
            tb = sum(float(bc["rays"][0][k]) * 48 + float(bc["nodes"][0][k]) * 80 + float(bc["tris"][0][k]) * 48 +
                     float(bc["rays"][1][k]) * 36 + float(bc["nodes"][1][k]) * 80 + float(bc["tris"][1][k]) * 48
                     for k in range(tail, depth)) / nf
            ms_t = s1["ms_tail"] / nf
            roof["tail_kernel"] = {"first_bounce": tail, "ms": round(ms_t, 4),
                                   "closest_rays": round(float(bc["rays"][0][tail:depth].sum()) / nf),
                                   "shadow_rays": round(float(bc["rays"][1][tail:depth].sum()) / nf),
                                   "traversal_gbs": round(tb / (ms_t * 1e-3) / 1e9, 1) if ms_t > 0 else None}
        rt.close()
        rc.close()

    config1 = None
    if rank == 0 and world == 1 and not args.no_config1:
        config1 = config1_section(srt, ctx, stream, cpu=not args.no_cpu_baseline)
    batched = None
    if rank == 0 and world == 1 and not args.no_batched:
        batched = batched_section(srt, ctx, stream)
    guided = None
    if rank == 0 and world == 1 and not args.no_guided:
        guided = guided_section()
    batched_guided = None
    if rank == 0 and world == 1 and not args.no_batched_guided:
        batched_guided = batched_guided_section()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(cfg)
    if rank == 0:
        clocks = clk.summary()
        line = {
            "metric": "Mpaths/s", "value": round(value, 3), "unit": "Mpaths/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (procedural scene, seeded)",
            "config": {"workload": (f"{args.config}: {info['triangles']} triangles, {w}x{h}, depth {depth}, "
                                    f"{photons} photons/frame, 1 spp per step"),
                       "l2": "inputs larger than L2 (per-frame working set > 1 GB: path state, photons, BVH)",
                       "parallelism": f"replicas x{world}", "bvh_nodes": info["nodes"], "bvh_depth": info["depth"]},
            "mphotons_per_s": round(photons_all / (ms_max * 1e-3) / 1e6, 2),
            "mrays_per_s": round(rays_all / (ms_max * 1e-3) / 1e6, 2),
            "rays_per_path": round((st["rays_closest"] + st["rays_shadow"]) / max(1, st["paths"]), 3),
            "photons_stored_per_frame": round(st["photons_stored"] / max(1, st["frames"])),
            "e2e": {"value": round(e2e_value, 3), "unit": "Mpaths/s", "h2d_bytes_per_step": 272,
                    "d2h_bytes_per_step": w * h * 4, "steps": e2e_steps} if e2e_steps else None,
            "gpu_launches": int(st["kernel_launches"]),
            "roofline": roof,
            "config1": config1,
            "batched": batched,
            "guided": guided,
            "batched_guided": batched_guided,
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    r.close()
    scene.close()
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
