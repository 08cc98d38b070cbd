"""Writes tests/golden/ref_wgsl.npz: outputs of the reference's OWN shader code.

The reference's hot path is WGSL (src/renderer/shaders/shader.wgsl,
photon_emit.wgsl, build_grid.wgsl) run by wgpu on a Vulkan ray-query device,
which this machine cannot run.  oracle/wgsl_translate.py translates those three
files mechanically into C++ and oracle/ref_harness.cpp runs them on the CPU
(make -C oracle ref), answering their ray queries with the oracle's FP64 query
— the part the Vulkan driver answers in the reference.  This script records,
from that run:

* the shading functions one at a time on seeded inputs (the op codes of
  orc_device_math: pcg_hash, sample_cie_xyz, blackbody_radiance,
  rgb_to_spectrum_vec4, fresnel_thin_film, sample_bsdf with its rng draws, the
  grid hash; and photon_emit.wgsl's blackbody and single-wavelength film,
  Schlick's reflectance);
* the camera ray of every pixel of a 64 x 48 view (shader.wgsl:713-728);
* whole frames as renderer/mod.rs:168-207 records them (2^20 photon emitters,
  the grid, the camera pass) for five preset scenes and for the config-2
  geometry with reference material types in place of the coated spheres: per
  frame the photon counter, a SHA-256 of the stored photons and of the grid's
  head/next lists, the accumulation buffer and the rgba8 image, two frames
  each (the second accumulates onto the first).

tests/test_oracle_ref_pin.py checks the oracle against these fixtures (they
travel without the reference tree) and, where the tree is present, against a
live run of the translated shaders on fresh inputs.

Usage: python tests/golden/make_ref_golden.py   (needs the reference tree)
"""
from __future__ import annotations

import hashlib
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))

import binding as orc  # noqa: E402
import ref_binding as ref  # noqa: E402

OUT = Path(__file__).resolve().parent / "ref_wgsl.npz"
N_MATH = 2048

# (name, preset id, scene seed, width, height, camera aspect, material edit)
FRAME_CASES = [
    ("cornell", 0, 0, 32, 24, 32 / 24, None),
    ("prism", 1, 0, 32, 24, 32 / 24, None),
    ("config1", 2, 0, 32, 24, 32 / 24, None),
    ("caustic_slab", 4, 0, 32, 24, 32 / 24, None),
    ("indirect_room", 5, 0, 32, 24, 32 / 24, None),
    ("config2_ref_materials", 3, 0, 64, 36, 16 / 9, "config2_mix"),
]
FRAMES = (0, 1)
EMITTERS = ref.MAX_PHOTONS  # the reference's photon dispatch (renderer/mod.rs MAX_PHOTONS)


def math_inputs(seed: int, n: int) -> dict[int, np.ndarray]:
    """Seeded inputs per op, in the record layouts of orc_device_math."""
    rng = np.random.default_rng(seed)

    def unit(k):
        v = rng.normal(size=(k, 3))
        return v / np.linalg.norm(v, axis=1, keepdims=True)

    lam = rng.uniform(380, 780, n)
    inp = {
        0: rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32),
        1: lam.astype(np.float32),
        2: np.stack([lam, rng.uniform(1000, 9000, n)], 1).astype(np.float32),
        3: np.concatenate([rng.uniform(0, 1, (n, 3)), rng.uniform(380, 780, (n, 4))], 1).astype(np.float32),
        4: np.concatenate([rng.uniform(0, 1, (n, 1)), np.ones((n, 1)), rng.uniform(1.0, 1.8, (n, 2)),
                           rng.uniform(0, 900, (n, 1)), rng.uniform(380, 780, (n, 4))], 1).astype(np.float32),
        102: np.stack([lam, rng.uniform(1000, 9000, n)], 1).astype(np.float32),
        109: np.concatenate([rng.uniform(-1, 1, (n, 1)), np.ones((n, 1)), rng.uniform(1.0, 1.8, (n, 2)),
                             rng.uniform(0, 900, (n, 1)), rng.uniform(380, 780, (n, 1))], 1).astype(np.float32),
        110: np.stack([rng.uniform(-1, 1, n), rng.uniform(0.3, 3, n)], 1).astype(np.float32),
    }
    # sample_bsdf: the reference's material types 0, 1, 2, 4 (type 3 emits and
    # never scatters; type 5 is this project's own)
    rec = np.zeros((n, 24), np.float32)
    rec[:, 0:3] = unit(n)
    rec[:, 3:6] = unit(n)
    mt = rng.choice([0, 1, 2, 4], n)
    rec[:, 6:9] = rng.uniform(0, 1, (n, 3))
    rec[:, 9] = 1.0
    rec[:, 10] = mt
    rec[:, 11] = np.where(mt == 4, rng.uniform(0, 800, n), rng.uniform(0.0, 1, n))
    rec[:, 12] = np.where(mt == 2, rng.uniform(1.3, 1.8, n), rng.uniform(1.0, 1.6, n))
    rec[:, 13] = np.where(mt == 2, rng.uniform(0, 0.02, n), rng.uniform(1.0, 1.6, n))
    rec[:, 14] = rng.integers(0, 2, n)
    rec[:, 15:19] = rng.uniform(380, 780, (n, 4))
    collapsed = rng.uniform(size=(n, 1)) < 0.3
    rec[:, 19:23] = np.where(collapsed, np.array([1.0, 0, 0, 0]), rng.uniform(0, 1, (n, 4)))
    rec[:, 23] = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32).view(np.float32)
    inp[6] = rec
    g = np.zeros((n, 5), np.float32)
    g[:, :3] = rng.uniform(-4, 4, (n, 3))
    g[:, 3] = rng.integers(0, 5000, n).astype(np.uint32).view(np.float32)
    g[:, 4] = 0.02  # the shaders' CELL_SIZE
    inp[7] = g
    return inp


def scene_arrays(preset: int, seed: int, edit: str | None):
    """The oracle generator's preset arrays; edit "config2_mix" gives the 64
    coated spheres of config 2 (material type 5, which the reference lacks)
    reference types instead: a third GGX (roughness from color.w), a third
    dispersive glass (A 1.5, B 0.004), a third Airy film (thickness, n2, n3
    kept).  Returns (preset, arrays, keep-alive)."""
    pre = orc.Preset(preset, seed)
    a = pre.arrays()
    if edit is None:
        return pre, a, None
    assert edit == "config2_mix"
    a2, mats = ref.reference_materials(a)
    return pre, a2, mats


def grid_lists_from_sorted(keys: np.ndarray, n_ids: int = ref.MAX_PHOTONS, hash_size: int = ref.HASH_SIZE):
    """The linked lists build_grid.wgsl leaves after a sequential run (head =
    the highest id of a cell, next = the id inserted before it) from the sorted
    (hash << 32 | id) keys; the sentinel bucket (zero-energy photons) is not
    inserted."""
    head = np.full(hash_size, 0xFFFFFFFF, np.uint32)
    nxt = np.zeros(n_ids, np.uint32)
    hsh = (keys >> np.uint64(32)).astype(np.int64)
    ids = (keys & np.uint64(0xFFFFFFFF)).astype(np.int64)
    keep = hsh < hash_size
    hsh, ids = hsh[keep], ids[keep]
    if len(ids):
        first = np.ones(len(ids), bool)
        first[1:] = hsh[1:] != hsh[:-1]
        prev = np.empty(len(ids), np.int64)
        prev[0] = 0xFFFFFFFF
        prev[1:] = ids[:-1]
        nxt[ids] = np.where(first, 0xFFFFFFFF, prev).astype(np.uint32)
        last = np.ones(len(ids), bool)
        last[:-1] = hsh[1:] != hsh[:-1]
        head[hsh[last]] = ids[last].astype(np.uint32)
    return head, nxt


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main() -> int:
    if not ref.reference_present():
        print("the reference tree is not present; nothing written", file=sys.stderr)
        return 1
    ref.build()
    out: dict[str, np.ndarray] = {}
    for op, a in math_inputs(2024, N_MATH).items():
        out[f"math{op}_in"] = a
        out[f"math{op}_out"] = ref.device_math(op, a)
    pre = orc.Preset(0, 0)
    pos, yaw, pitch = pre.camera
    w, h = 64, 48
    cam = orc.camera_uniform(pos, yaw, pitch, w / h, 3)
    pix = np.stack(np.meshgrid(np.arange(w), np.arange(h)), -1).reshape(-1, 2).astype(np.uint32)
    out["camray_uniform"] = np.frombuffer(bytes(cam), np.uint8).copy()
    out["camray_size"] = np.array([w, h], np.uint32)
    out["camray_pix"] = pix
    out["camray_out"] = ref.camera_rays(cam, w, h, pix)
    names = []
    for name, preset, seed, fw, fh, aspect, edit in FRAME_CASES:
        t0 = time.time()
        _pre, arrays, _keep = scene_arrays(preset, seed, edit)
        rs = ref.RefScene(arrays)
        p3, yaw, pitch = _pre.camera
        accum = None
        for f in FRAMES:
            u = orc.camera_uniform(p3, yaw, pitch, aspect, f)
            buf, count = rs.photon_emit(u, EMITTERS)
            head, nxt = rs.build_grid(u, buf, count)
            accum, ldr = rs.camera_pass(u, fw, fh, 12, buf, head, nxt, accum=accum)
            stored = min(count, ref.MAX_PHOTONS)
            k = f"{name}_f{f}"
            out[k + "_uniform"] = np.frombuffer(bytes(u), np.uint8).copy()
            out[k + "_count"] = np.array([count], np.uint32)
            out[k + "_photons_sha"] = np.frombuffer(sha(buf[:stored]).encode(), np.uint8).copy()
            out[k + "_grid_sha"] = np.frombuffer(sha(head, nxt).encode(), np.uint8).copy()
            out[k + "_accum"] = accum.copy()
            out[k + "_ldr"] = ldr.copy()
        rs.close()
        names.append(name)
        print(f"{name}: {time.time() - t0:.1f} s, {stored} photons in the last frame")
    out["frame_cases"] = np.array(names)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
