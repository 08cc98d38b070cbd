"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, to check the CUDA path.  The product package never
imports it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

_lib = None


# Record layouts of include/srt.h, declared here so that the oracle runs
# without the product package.
class CameraUniform(C.Structure):  # srt_camera_uniform (camera.rs:4-13), 272 B
    _fields_ = [("view_inverse", C.c_float * 16), ("proj_inverse", C.c_float * 16), ("view", C.c_float * 16),
                ("proj", C.c_float * 16), ("frame_count", C.c_uint32), ("pad", C.c_uint32 * 3)]


class Params(C.Structure):  # srt_params, 52 B
    _fields_ = [("max_depth", C.c_uint32), ("photons_per_frame", C.c_uint32), ("hash_bits", C.c_uint32),
                ("photon_max_bounces", C.c_uint32), ("gather_cap", C.c_uint32), ("flags", C.c_uint32),
                ("cell_size", C.c_float), ("gather_radius0", C.c_float), ("radius_exponent", C.c_float),
                ("spectral_radius", C.c_float), ("photon_norm_count", C.c_float), ("block_size", C.c_uint32),
                ("seed", C.c_uint32)]


class SceneArrays(C.Structure):  # srt_scene_arrays
    _fields_ = [("vertices", C.c_void_p), ("n_vertices", C.c_uint32), ("indices", C.c_void_p),
                ("n_indices", C.c_uint32), ("mesh_infos", C.c_void_p), ("n_meshes", C.c_uint32),
                ("materials", C.c_void_p), ("n_materials", C.c_uint32), ("instances", C.c_void_p),
                ("n_instances", C.c_uint32), ("lights", C.c_void_p), ("n_lights", C.c_uint32)]


assert C.sizeof(CameraUniform) == 272 and C.sizeof(Params) == 52


def default_params(**kw) -> Params:
    """The reference's constants: MAX_DEPTH 12 (renderer/compute_pass.rs:26),
    MAX_PHOTONS 2^20 (renderer/mod.rs:18), HASH_SIZE 2^22 (:19), 5 photon
    bounces (photon_emit.wgsl:219), 64 gathered photons (shader.wgsl:312),
    CELL_SIZE 0.02 (:275), radius 0.02 * (frame + 1)^-0.15 (:302-303),
    spectral radius 20 nm (:279)."""
    p = Params(max_depth=12, photons_per_frame=1 << 20, hash_bits=22, photon_max_bounces=5, gather_cap=64,
               flags=0, cell_size=0.02, gather_radius0=0.02, radius_exponent=-0.15, spectral_radius=20.0,
               photon_norm_count=0.0, block_size=0, seed=0)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def build() -> Path:
    """Compiles the oracle with its Makefile (g++ -fopenmp)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        P = C.c_void_p
        U32 = C.c_uint32
        L.orc_scene_create.restype = P
        L.orc_scene_create.argtypes = [P]
        L.orc_scene_destroy.argtypes = [P]
        L.orc_scene_num_tris.restype = C.c_uint64
        L.orc_scene_num_tris.argtypes = [P]
        L.orc_trace.argtypes = [P, P, U32, C.c_int, C.c_int, P, P, P, P, P]
        L.orc_device_math.restype = C.c_int
        L.orc_device_math.argtypes = [C.c_int, U32, P, P, P]
        L.orc_photon_emit.restype = U32
        L.orc_photon_emit.argtypes = [P, U32, U32, U32, P, P, C.c_int]
        L.orc_photon_grid_build.argtypes = [P, U32, U32, C.c_float, U32, P, P]
        L.orc_photon_gather.argtypes = [P, U32, P, U32, U32, P, P]
        L.orc_render_frame.argtypes = [P, P, U32, U32, P, U32, U32, P, P, P, P, C.c_int]
        L.orc_render_frame_photons.argtypes = [P, P, U32, U32, P, P, U32, U32, U32, P, P, P, P, C.c_int]
        L.orc_tri_probe.argtypes = [P, P, P, U32, P, P, P]
        L.orc_max_threads.restype = C.c_int
        L.orc_preset_create.restype = P
        L.orc_preset_create.argtypes = [C.c_int, U32]
        L.orc_preset_destroy.argtypes = [P]
        L.orc_preset_arrays.argtypes = [P, P, P]
        L.orc_camera_uniform.argtypes = [P, C.c_float, C.c_float, C.c_float, U32, P]
        _lib = L
    return _lib


def _p(a: np.ndarray | None):
    return C.c_void_p(a.ctypes.data) if a is not None else None


class Preset:
    """A preset scene from the oracle's own generator (scenes.cpp): arrays()
    gives an srt_scene_arrays view of it, camera = ([x, y, z], yaw, pitch)."""

    def __init__(self, preset: int, seed: int = 0):
        self.h = lib().orc_preset_create(preset, seed)
        if not self.h:
            raise ValueError(f"unknown preset {preset}")
        self._arrays = SceneArrays()
        cam = (C.c_float * 5)()
        lib().orc_preset_arrays(self.h, C.byref(self._arrays), cam)
        self.camera = ([cam[0], cam[1], cam[2]], cam[3], cam[4])

    def arrays(self) -> SceneArrays:
        return self._arrays

    def n_triangles(self) -> int:
        a = self._arrays
        ends = []
        mi = np.ctypeslib.as_array(C.cast(a.mesh_infos, C.POINTER(C.c_uint32)), (a.n_meshes, 4))
        inst = np.ctypeslib.as_array(C.cast(a.instances, C.POINTER(C.c_uint32)), (a.n_instances, 20))
        for m in range(a.n_meshes):
            ends.append(int(mi[m + 1, 1]) if m + 1 < a.n_meshes else a.n_indices)
        return int(sum((ends[k] - int(mi[k, 1])) // 3 for k in inst[:, 0]))

    def close(self):
        if self.h:
            lib().orc_preset_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def camera_uniform(pos, yaw: float, pitch: float, aspect: float, frame: int) -> CameraUniform:
    """camera.rs:178-194 (the oracle's restatement)."""
    u = CameraUniform()
    p = (C.c_float * 3)(*pos)
    lib().orc_camera_uniform(p, yaw, pitch, aspect, frame, C.byref(u))
    return u


class OracleScene:
    """FP64 ray queries + FP32 shading restatement over one scene's arrays."""

    def __init__(self, arrays):
        # arrays: an srt_scene_arrays structure (the product's SceneBuilder.arrays()
        # or Preset.arrays()), pointers into host memory that outlive this call
        self.h = lib().orc_scene_create(C.byref(arrays))

    @property
    def n_tris(self) -> int:
        return int(lib().orc_scene_num_tris(self.h))

    def trace(self, rays: np.ndarray, any_hit=False, brute=True):
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = len(r)
        t = np.zeros(n, np.float64)
        prim = np.zeros(n, np.uint32)
        u = np.zeros(n, np.float64)
        v = np.zeros(n, np.float64)
        t2 = np.zeros(n, np.float64)
        lib().orc_trace(self.h, _p(r), n, int(any_hit), int(brute), _p(t), _p(prim), _p(u), _p(v), _p(t2))
        return t, prim, u, v, t2

    def photon_emit(self, n_photons: int, frame: int, max_bounces: int = 5, threads: int = 0):
        out = np.zeros((n_photons, 8), np.float32)
        em = np.zeros(n_photons, np.uint32)
        c = lib().orc_photon_emit(self.h, n_photons, frame, max_bounces, _p(out), _p(em), threads)
        return out[:c].copy(), em[:c].copy()

    def tri_probe(self, rays: np.ndarray, prims: np.ndarray, with_cos: bool = False):
        """FP64 (t where each ray's line meets the plane of triangle prims[i],
        distance from that point to the triangle's boundary: > 0 inside[, |cos|
        of the angle between the ray and the plane's normal])."""
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        pr = np.ascontiguousarray(prims, np.uint32)
        t = np.zeros(len(r), np.float64)
        e = np.zeros(len(r), np.float64)
        c = np.zeros(len(r), np.float64)
        lib().orc_tri_probe(self.h, _p(r), _p(pr), len(r), _p(t), _p(e), _p(c))
        return (t, e, c) if with_cos else (t, e)

    def render_frame(self, cam, w: int, h: int, params, accum: np.ndarray | None = None, row_stride=1, row_phase=0,
                     want_ldr=True, want_radiance=False, threads: int = 0, photons: np.ndarray | None = None):
        """One frame; `photons` (n x 8 float32) replaces the oracle's own photon pass."""
        if accum is None:
            accum = np.zeros((h, w, 4), np.float32)
        ldr = np.zeros((h, w, 4), np.uint8) if want_ldr else None
        rad = np.zeros((h, w, 4), np.float32) if want_radiance else None
        stats = np.zeros(5, np.uint64)
        if photons is None:
            lib().orc_render_frame(self.h, C.byref(cam), w, h, C.byref(params), row_stride, row_phase, _p(accum),
                                   _p(ldr), _p(rad), _p(stats), threads)
        else:
            ph = np.ascontiguousarray(photons, np.float32).reshape(-1, 8)
            lib().orc_render_frame_photons(self.h, C.byref(cam), w, h, C.byref(params), _p(ph), len(ph), row_stride,
                                           row_phase, _p(accum), _p(ldr), _p(rad), _p(stats), threads)
        return accum, ldr, rad, stats

    def close(self):
        if self.h:
            lib().orc_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def device_math(op: int, inp: np.ndarray, aux=None) -> np.ndarray:
    sizes = {0: (4, 4), 1: (4, 12), 2: (8, 4), 3: (28, 16), 4: (36, 16), 5: (4, 20), 6: (96, 40), 7: (20, 4),
             8: (20, 28), 102: (8, 4), 109: (24, 4), 110: (8, 4)}
    isz, osz = sizes[op]
    a = np.ascontiguousarray(inp)
    n = a.nbytes // isz
    out = np.zeros(n * osz // 4, np.uint32 if op in (0, 7) else np.float32)
    rc = lib().orc_device_math(op, n, _p(a), _p(out), C.byref(aux) if aux is not None else None)
    assert rc == 0
    return out.reshape(n, osz // 4)


def photon_grid_build(photons: np.ndarray, frame: int, cell: float = 0.02, hash_bits: int = 22):
    p = np.ascontiguousarray(photons, np.float32).reshape(-1, 8)
    keys = np.zeros(len(p), np.uint64)
    ranges = np.zeros((1 << hash_bits, 2), np.uint32)
    lib().orc_photon_grid_build(_p(p), len(p), frame, cell, hash_bits, _p(keys), _p(ranges))
    return keys, ranges


def photon_gather(photons: np.ndarray, queries: np.ndarray, frame: int, params) -> np.ndarray:
    p = np.ascontiguousarray(photons, np.float32).reshape(-1, 8)
    q = np.ascontiguousarray(queries, np.float32).reshape(-1, 10)
    out = np.zeros((len(q), 4), np.float32)
    lib().orc_photon_gather(_p(p), len(p), _p(q), len(q), frame, C.byref(params), _p(out))
    return out


def max_threads() -> int:
    return int(lib().orc_max_threads())
