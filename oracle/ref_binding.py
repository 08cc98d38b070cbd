"""ctypes binding of oracle/_ref/libref_wgsl.so: the reference's own WGSL
shaders (shader.wgsl, photon_emit.wgsl, build_grid.wgsl), translated to C++ by
oracle/wgsl_translate.py and run on the CPU by oracle/ref_harness.cpp.

TEST INFRASTRUCTURE ONLY: it pins the oracle's restatement (oracle.cpp) to the
reference's code.  The library is built from the reference tree, so it exists
only where that tree does; tests/golden/make_ref_golden.py stores its outputs
as fixtures that travel without it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

import binding as orc  # oracle/binding.py (oracle/ is on sys.path, as the tests put it)

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_ref" / "libref_wgsl.so"
REFERENCE = Path(os.environ.get("SRT_REFERENCE_TREE", "/root/reference"))
SHADERS = REFERENCE / "src" / "renderer" / "shaders"
MAX_PHOTONS = 1 << 20   # renderer/mod.rs: MAX_PHOTONS, the photon dispatch and buffer size
HASH_SIZE = 1 << 22     # HASH_SIZE of shader.wgsl and build_grid.wgsl

_lib = None


def reference_present() -> bool:
    return all((SHADERS / f"{n}.wgsl").is_file() for n in ("shader", "photon_emit", "build_grid"))


def build() -> Path:
    """Translates and compiles the reference's shaders (make -C oracle ref)."""
    orc.build()
    subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={REFERENCE}"], check=True)
    return LIB_PATH


def available() -> bool:
    return LIB_PATH.exists() or reference_present()


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if reference_present():
            build()  # make: a no-op when up to date
        orc.lib()  # loads liboracle.so first (the harness links it)
        L = C.CDLL(str(LIB_PATH))
        P = C.c_void_p
        U32 = C.c_uint32
        L.ref_scene_create.restype = P
        L.ref_scene_create.argtypes = [P]
        L.ref_scene_destroy.argtypes = [P]
        L.ref_photon_emit.restype = U32
        L.ref_photon_emit.argtypes = [P, P, U32, P, C.c_int]
        L.ref_build_grid.argtypes = [P, P, U32, P, P, C.c_int]
        L.ref_camera_pass.argtypes = [P, P, U32, U32, U32, P, P, P, P, P, C.c_int]
        L.ref_camera_rays.argtypes = [P, U32, U32, P, U32, P]
        L.ref_device_math.restype = C.c_int
        L.ref_device_math.argtypes = [C.c_int, U32, P, P]
        _lib = L
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def reference_materials(arrays):
    """The scene with material type 5 (thin-film-coated GGX, this project's own:
    the reference's shaders do not know it) replaced by reference types, a third
    each: GGX (roughness from color.w), dispersive glass (A 1.5, B 0.004), Airy
    film (thickness, n2, n3 kept).  Returns (arrays, materials): keep the second
    alive while the first is used.  Scenes without type 5 come back unchanged."""
    mats = np.ctypeslib.as_array(C.cast(arrays.materials, C.POINTER(C.c_float)), (arrays.n_materials, 8)).copy()
    idx = np.nonzero(mats[:, 4] == 5)[0]
    if len(idx) == 0:
        return arrays, None
    g1, g2, g4 = idx[0::3], idx[1::3], idx[2::3]
    mats[g1, 4] = 1
    mats[g1, 5] = mats[g1, 3]
    mats[g2, 4] = 2
    mats[g2, 6] = 1.5
    mats[g2, 7] = 0.004
    mats[g4, 4] = 4
    a2 = type(arrays)()  # the oracle's or the product's srt_scene_arrays record
    C.pointer(a2)[0] = arrays
    field = dict(type(arrays)._fields_)["materials"]  # c_void_p or a typed pointer
    a2.materials = C.cast(C.c_void_p(mats.ctypes.data), field)
    return a2, mats


# op -> (input bytes, output bytes) per record; the orc_device_math layouts
# plus the photon_emit.wgsl functions and Schlick's reflectance
SIZES = {0: (4, 4), 1: (4, 12), 2: (8, 4), 3: (28, 16), 4: (36, 16), 6: (96, 40), 7: (20, 4), 102: (8, 4),
         109: (24, 4), 110: (8, 4)}


def device_math(op: int, inp: np.ndarray) -> np.ndarray:
    isz, osz = SIZES[op]
    a = np.ascontiguousarray(inp)
    n = a.nbytes // isz
    out = np.zeros(n * osz // 4, np.uint32 if op in (0, 7) else np.float32)
    rc = lib().ref_device_math(op, n, _p(a), _p(out))
    if rc != 0:
        raise ValueError(f"op {op}: the reference has no function for this input")
    return out.reshape(n, osz // 4)


def camera_rays(cam, w: int, h: int, pix: np.ndarray) -> np.ndarray:
    """(n, 6) origin and direction of the camera ray of each (x, y) in pix, as
    the reference's main computes it."""
    p = np.ascontiguousarray(pix, np.uint32).reshape(-1, 2)
    out = np.zeros((len(p), 6), np.float32)
    lib().ref_camera_rays(C.byref(cam), w, h, _p(p), len(p), _p(out))
    return out


class RefScene:
    """One scene's buffers bound the way the reference's passes bind them."""

    def __init__(self, arrays):
        self.h = lib().ref_scene_create(C.byref(arrays))

    def photon_emit(self, cam, n_emit: int = MAX_PHOTONS, threads: int = 1):
        """photon_emit.wgsl over emitter ids [0, n_emit): (the 2^20-record photon
        buffer, the atomic counter).  threads = 1 runs the invocations in id order
        (the deterministic order the oracle reproduces); more (0 = all) run them
        concurrently, the photons landing in the order the atomic hands out."""
        buf = np.zeros((MAX_PHOTONS, 8), np.float32)
        count = lib().ref_photon_emit(self.h, C.byref(cam), n_emit, _p(buf), threads)
        return buf, int(count)

    @staticmethod
    def build_grid(cam, buf: np.ndarray, count: int, threads: int = 1):
        """build_grid.wgsl over the 2^20-id dispatch: (grid_head, grid_next);
        threads as for photon_emit."""
        head = np.zeros(HASH_SIZE, np.uint32)
        nxt = np.zeros(MAX_PHOTONS, np.uint32)
        lib().ref_build_grid(C.byref(cam), _p(buf), count, _p(head), _p(nxt), threads)
        return head, nxt

    def camera_pass(self, cam, w: int, h: int, max_depth: int, buf, head, nxt, accum=None, threads: int = 0):
        """shader.wgsl main over a w x h target: (accumulation, rgba8 image)."""
        if accum is None:
            accum = np.zeros((h, w, 4), np.float32)
        ldr = np.zeros((h, w, 4), np.uint8)
        lib().ref_camera_pass(self.h, C.byref(cam), w, h, max_depth, _p(buf), _p(head), _p(nxt), _p(accum),
                              _p(ldr), threads)
        return accum, ldr

    def render_frame(self, cam, w: int, h: int, max_depth: int = 12, n_emit: int = MAX_PHOTONS, accum=None,
                     threads: int = 0, ordered: bool = True):
        """One frame as renderer/mod.rs:168-207 records it: photon pass, grid,
        camera pass (on `threads` threads, 0 = all).  ordered: the photon and
        grid dispatches run in id order (deterministic), else concurrently.
        Returns (accumulation, rgba8, stored photons)."""
        pt = 1 if ordered else threads
        buf, count = self.photon_emit(cam, n_emit, pt)
        head, nxt = self.build_grid(cam, buf, count, pt)
        accum, ldr = self.camera_pass(cam, w, h, max_depth, buf, head, nxt, accum, threads)
        return accum, ldr, buf[:min(count, MAX_PHOTONS)].copy()

    def close(self):
        if self.h:
            lib().ref_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
