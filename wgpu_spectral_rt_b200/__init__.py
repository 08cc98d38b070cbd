"""B200-native spectral path tracer: Python mirror of the reference's
scene / renderer API over the C ABI of libsrt_b200.so (include/srt.h).

The classes keep the reference's names and call order:

    builder = SceneBuilder()                       # src/scene/builder.rs:47
    builder.add_material(...); builder.add_mesh(...); builder.add_instance(...)
    scene = builder.build(ctx)                     # builder.rs:131
    renderer = Renderer(ctx, scene, w, h)          # src/renderer/mod.rs:45
    cam = CameraController().build_uniform(w / h, renderer.frame_count)
    renderer.render(cam)                           # renderer/mod.rs:168

Every call goes through the native library; there is no Python or CPU
fallback.  A missing library raises at import of `lib()`.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
# SRT_LIB_PATH selects another build of the same library (e.g. a variant build)
LIB_PATH = Path(os.environ["SRT_LIB_PATH"]) if os.environ.get("SRT_LIB_PATH") else _PKG / "libsrt_b200.so"

# --------------------------------------------------------------------------- records


class Vertex(C.Structure):
    _fields_ = [("pos", C.c_float * 4), ("normal", C.c_float * 4)]


class Material(C.Structure):
    _fields_ = [("color", C.c_float * 4), ("extra", C.c_float * 4)]


class Light(C.Structure):
    _fields_ = [("v0", C.c_float * 4), ("v1", C.c_float * 4), ("v2", C.c_float * 4), ("params", C.c_float * 4)]


class MeshInfo(C.Structure):
    _fields_ = [("vertex_offset", C.c_uint32), ("index_offset", C.c_uint32), ("pad", C.c_uint32 * 2)]


class Instance(C.Structure):
    _fields_ = [("mesh_id", C.c_uint32), ("mat_id", C.c_uint32), ("pad", C.c_uint32 * 2),
                ("transform", C.c_float * 16)]


class CameraUniform(C.Structure):
    _fields_ = [("view_inverse", C.c_float * 16), ("proj_inverse", C.c_float * 16), ("view", C.c_float * 16),
                ("proj", C.c_float * 16), ("frame_count", C.c_uint32), ("pad", C.c_uint32 * 3)]


class Photon(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("wavelength", C.c_float), ("direction", C.c_float * 3),
                ("energy", C.c_float)]


class Ray(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("tmin", C.c_float), ("dir", C.c_float * 3), ("tmax", C.c_float)]


class Hit(C.Structure):
    _fields_ = [("t", C.c_float), ("prim", C.c_uint32), ("u", C.c_float), ("v", C.c_float)]


class Params(C.Structure):
    _fields_ = [("max_depth", C.c_uint32), ("photons_per_frame", C.c_uint32), ("hash_bits", C.c_uint32),
                ("photon_max_bounces", C.c_uint32), ("gather_cap", C.c_uint32), ("flags", C.c_uint32),
                ("cell_size", C.c_float), ("gather_radius0", C.c_float), ("radius_exponent", C.c_float),
                ("spectral_radius", C.c_float), ("photon_norm_count", C.c_float), ("block_size", C.c_uint32),
                ("seed", C.c_uint32)]


class BatchTuning(C.Structure):
    _fields_ = [("blocks_per_sm", C.c_uint32), ("chunk", C.c_uint32), ("ms_per_iteration", C.c_float),
                ("candidates", C.c_uint32), ("bvh_width", C.c_uint32)]


class Stats(C.Structure):
    _fields_ = [("frames", C.c_uint64), ("paths", C.c_uint64), ("rays_closest", C.c_uint64),
                ("rays_shadow", C.c_uint64), ("rays_photon", C.c_uint64), ("photons_emitted", C.c_uint64),
                ("photons_stored", C.c_uint64), ("nodes_visited", C.c_uint64 * 3), ("tris_tested", C.c_uint64 * 3),
                ("ms_photon_pass", C.c_double), ("ms_trace_closest", C.c_double), ("ms_shade", C.c_double),
                ("ms_trace_shadow", C.c_double), ("ms_finalize", C.c_double), ("ms_raygen", C.c_double),
                ("launches_trace_closest", C.c_uint64), ("kernel_launches", C.c_uint64),
                ("ms_guide_train", C.c_double), ("ms_tail", C.c_double), ("tail_first", C.c_uint32),
                ("pad", C.c_uint32)]


class BounceStats(C.Structure):  # srt_bounce_stats
    _fields_ = [("rays", (C.c_uint64 * 32) * 3), ("nodes", (C.c_uint64 * 32) * 3), ("tris", (C.c_uint64 * 32) * 3),
                ("ms", (C.c_double * 32) * 2)]


class SceneArrays(C.Structure):
    _fields_ = [("vertices", C.POINTER(Vertex)), ("n_vertices", C.c_uint32),
                ("indices", C.POINTER(C.c_uint32)), ("n_indices", C.c_uint32),
                ("mesh_infos", C.POINTER(MeshInfo)), ("n_meshes", C.c_uint32),
                ("materials", C.POINTER(Material)), ("n_materials", C.c_uint32),
                ("instances", C.POINTER(Instance)), ("n_instances", C.c_uint32),
                ("lights", C.POINTER(Light)), ("n_lights", C.c_uint32)]


for _t, _n in ((Vertex, 32), (Material, 32), (Light, 64), (MeshInfo, 16), (Instance, 80), (CameraUniform, 272),
               (Photon, 32), (Ray, 32), (Hit, 16), (Params, 52)):
    assert C.sizeof(_t) == _n, (_t, C.sizeof(_t))

FLAG_FP64_ACCUM = 0x1
FLAG_NO_GRAPH = 0x2
FLAG_STAGE_TIMING = 0x4
FLAG_COUNT_VISITS = 0x8
FLAG_RAY_SORT = 0x10
FLAG_GUIDING = 0x20
FLAG_GUIDE_FROZEN = 0x40

PRESET_CORNELL_BOX = 0
PRESET_CUSTOM_PRISM = 1
PRESET_CONFIG1 = 2
PRESET_CONFIG2 = 3
PRESET_CAUSTIC_SLAB = 4
PRESET_INDIRECT_ROOM = 5
PRESET_BATCH_RANDOM = 6

BVH_SAH = 0
BVH_LBVH = 1

GUIDE_INFER_MMA_SYNC = 0
GUIDE_INFER_TCGEN05 = 1
TAIL_AUTO = 0xFFFFFFFF  # srt_renderer_set_tail: chosen from the first frame's path counts
GUIDE_TRAIN_MMA_SYNC = 0
GUIDE_TRAIN_TCGEN05 = 1

STATUS = {0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "CUDA_ERROR", 4: "TIMEOUT", 5: "DEVICE_ASSERT", 6: "NO_DEVICE",
          7: "UNSUPPORTED", 8: "CAPACITY"}

# Every exported entry point with (restype, argtypes).
_P = C.c_void_p
_U32 = C.c_uint32
_F = C.c_float
_I = C.c_int
SIGNATURES = {
    "srt_abi_version": (_U32, []),
    "srt_ctx_create": (_I, [_I, _P, C.POINTER(_P)]),
    "srt_ctx_destroy": (_I, [_P]),
    "srt_get_error_string": (C.c_char_p, [_P]),
    "srt_ctx_stream": (_P, [_P]),
    "srt_ctx_synchronize": (_I, [_P]),
    "srt_ctx_sm_count": (_I, [_P]),
    "srt_scene_builder_create": (_I, [C.POINTER(_P)]),
    "srt_scene_builder_destroy": (_I, [_P]),
    "srt_scene_builder_add_material": (_U32, [_P, C.POINTER(Material)]),
    "srt_scene_builder_add_mesh": (_U32, [_P, C.POINTER(Vertex), _U32, C.POINTER(_U32), _U32]),
    "srt_scene_builder_add_instance": (_I, [_P, _U32, _U32, C.POINTER(_F)]),
    "srt_scene_builder_add_light_instance": (_I, [_P, _U32, _U32, C.POINTER(_F), C.POINTER(_F)]),
    "srt_scene_builder_arrays": (_I, [_P, C.POINTER(SceneArrays)]),
    "srt_scene_builder_build": (_I, [_P, _P, C.POINTER(_P)]),
    "srt_scene_build": (_I, [_P, C.POINTER(SceneArrays), C.POINTER(_P)]),
    "srt_scene_destroy": (_I, [_P]),
    "srt_scene_info": (_I, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(_U32)]),
    "srt_scene_rebuild_bvh": (_I, [_P, _U32]),
    "srt_scene_bvh_width": (_I, [_P, C.POINTER(_U32)]),
    "srt_geometry_plane": (_I, [C.POINTER(Vertex), C.POINTER(_U32), C.POINTER(_U32), C.POINTER(_U32)]),
    "srt_geometry_cube": (_I, [C.POINTER(Vertex), C.POINTER(_U32), C.POINTER(_U32), C.POINTER(_U32)]),
    "srt_geometry_icosphere": (_I, [_U32, C.POINTER(Vertex), C.POINTER(_U32), C.POINTER(_U32), C.POINTER(_U32)]),
    "srt_geometry_uv_sphere": (_I, [_U32, _U32, C.POINTER(Vertex), C.POINTER(_U32), C.POINTER(_U32),
                                    C.POINTER(_U32)]),
    "srt_scene_builder_add_preset": (_I, [_P, _I, _U32, C.POINTER(_F)]),
    "srt_camera_build_uniform": (_I, [C.POINTER(_F), _F, _F, _F, _U32, C.POINTER(CameraUniform)]),
    "srt_params_default": (Params, []),
    "srt_renderer_create": (_I, [_P, _P, _U32, _U32, C.POINTER(Params), C.POINTER(_P)]),
    "srt_renderer_destroy": (_I, [_P]),
    "srt_render_frame": (_I, [_P, C.POINTER(CameraUniform)]),
    "srt_renderer_frame_count": (_U32, [_P]),
    "srt_renderer_set_frame_count": (_I, [_P, _U32]),
    "srt_reset_accumulation": (_I, [_P]),
    "srt_read_accum_f32": (_I, [_P, _P]),
    "srt_read_accum_f64": (_I, [_P, _P]),
    "srt_read_ldr_rgba8": (_I, [_P, _P, _U32]),
    "srt_save_screenshot": (_I, [_P, C.c_char_p]),
    "srt_screenshot_write": (_I, [C.c_char_p, _P, _U32, _U32, _U32]),
    "srt_save_screenshot_async": (_I, [_P, C.c_char_p]),
    "srt_screenshot_write_async": (_I, [C.c_char_p, _P, _U32, _U32, _U32]),
    "srt_screenshot_flush": (_I, [_P]),
    "srt_renderer_get_stats": (_I, [_P, C.POINTER(Stats)]),
    "srt_renderer_get_bounce_stats": (_I, [_P, C.POINTER(BounceStats)]),
    "srt_renderer_set_tail": (_I, [_P, _U32]),
    "srt_renderer_reset_stats": (_I, [_P]),
    "srt_renderer_read_photons": (_I, [_P, _P, _U32, C.POINTER(_U32)]),
    "srt_trace_rays": (_I, [_P, _P, _U32, _P, _I]),
    "srt_photon_grid_build": (_I, [_P, _P, _U32, _U32, _F, _U32, _P, _P]),
    "srt_photon_gather": (_I, [_P, _P, _U32, _P, _U32, _U32, C.POINTER(Params), _P]),
    "srt_photon_grid_build_noalloc": (_I, [_P, _P, _U32, _U32, _F, _U32, _P, _P]),
    "srt_test_device_math": (_I, [_P, _I, _U32, _P, _P, _P]),
    "srt_blit_letterbox": (_I, [_P, _P, _U32, _U32, _U32, _U32, _I, _P]),
    "srt_renderer_blit": (_I, [_P, _U32, _U32, _I, _P]),
    "srt_photon_splat": (_I, [_P, _P, _U32, _P, _U32, _U32, _P]),
    "srt_renderer_splat_photons": (_I, [_P, _P, _U32, _U32, _P]),
    "srt_batch_create": (_I, [_P, _U32, _P, _P, _P, _P, _P]),
    "srt_batch_destroy": (_I, [_P]),
    "srt_batch_size": (_U32, [_P]),
    "srt_batch_renderer": (_P, [_P, _U32]),
    "srt_batch_render": (_I, [_P, _P, _P]),
    "srt_batch_get_tuning": (_I, [_P, _P]),
    "srt_batch_set_tuning": (_I, [_P, _P]),
    "srt_batch_autotune": (_I, [_P, _P, _U32, _P]),
    "srt_scene_update_instances": (_I, [_P, _P, _P, _U32]),
    "srt_scene_read_lights": (_I, [_P, _P, _U32, C.POINTER(_U32)]),
    "srt_scene_read_bvh": (_I, [_P, _P, C.c_uint64, _P, C.c_uint64]),
    "srt_ctx_set_bvh_builder": (_I, [_P, _I]),
    "srt_ctx_set_bvh_width": (_I, [_P, _U32]),
    "srt_ctx_set_bvh_leaf_size": (_I, [_P, _U32]),
    "srt_read_ldr_async": (_I, [_P, C.POINTER(_U32)]),
    "srt_ldr_wait": (_I, [_P, _U32, C.POINTER(C.POINTER(C.c_uint8))]),
    "srt_guide_param_count": (_U32, []),
    "srt_guide_default_weights": (_I, [C.c_uint64, _P, _U32]),
    "srt_renderer_guide_get_weights": (_I, [_P, _P, _U32]),
    "srt_renderer_guide_set_weights": (_I, [_P, _P, _U32]),
    "srt_renderer_guide_info": (_I, [_P, C.POINTER(_U32), C.POINTER(_U32)]),
    "srt_renderer_guide_configure": (_I, [_P, _F, _U32]),
    "srt_guide_test_forward": (_I, [_P, _P, _P, _U32, _P]),
    "srt_guide_test_forward_tc": (_I, [_P, _P, _P, _U32, _P]),
    "srt_renderer_guide_set_inference": (_I, [_P, _I]),
    "srt_renderer_guide_set_training": (_I, [_P, _I]),
    "srt_guide_test_mixture": (_I, [_P, _P, _P, _P, _U32, _P]),
    "srt_guide_test_mixture_tc": (_I, [_P, _P, _P, _P, _U32, _P]),
    "srt_renderer_guide_set_steps": (_I, [_P, _U32]),
    "srt_renderer_guide_set_bounces": (_I, [_P, _U32]),
    "srt_renderer_guide_get_state": (_I, [_P, _P, _P, _P, _P]),
    "srt_renderer_guide_set_state": (_I, [_P, _P, _P, _P, _U32]),
    "srt_write_accum_f64": (_I, [_P, _P]),
    "srt_test_wait_timeout": (_I, [_P, _U32]),
    "srt_guide_test_train": (_I, [_P, _P, _P, _P, _U32, _F, _P, _P, _P, _P, _U32, _P, _P, _P, _P]),
    "srt_guide_test_train_tc": (_I, [_P, _P, _P, _P, _U32, _F, _P, _P, _P, _P, _U32, _P, _P, _P, _P]),
}

_lib = None


def lib() -> C.CDLL:
    """The loaded native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"native library missing: {LIB_PATH} (run python -m wgpu_spectral_rt_b200.build)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class SrtError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


def _check(status: int, ctx=None):
    if status != 0:
        m = lib().srt_get_error_string(ctx)
        raise SrtError(status, m.decode() if m else "")


def ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def default_params(**kw) -> Params:
    p = lib().srt_params_default()
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def params_dict(p: Params) -> dict:
    return {f: getattr(p, f) for f, _ in Params._fields_}


# --------------------------------------------------------------------------- context


class Context:
    """WgpuContext replacement (src/wgpu_ctx.rs:3-82): one CUDA device + stream."""

    def __init__(self, device: int = 0, stream: int | None = None):
        h = C.c_void_p()
        _check(lib().srt_ctx_create(device, C.c_void_p(stream) if stream else None, C.byref(h)), None)
        self.h = h

    @property
    def stream(self) -> int:
        return lib().srt_ctx_stream(self.h) or 0

    @property
    def sm_count(self) -> int:
        return lib().srt_ctx_sm_count(self.h)

    def set_bvh_builder(self, builder: int) -> None:
        """BVH_SAH (default) or BVH_LBVH for the scenes built next."""
        _check(lib().srt_ctx_set_bvh_builder(self.h, builder), self.h)

    def set_bvh_width(self, width: int) -> None:
        """Children per BVH node (2..8, default 8) for the scenes built next."""
        _check(lib().srt_ctx_set_bvh_width(self.h, width), self.h)

    def set_bvh_leaf_size(self, max_triangles: int) -> None:
        """Triangles of the largest BVH leaf (1..3, default 2) for the scenes built next."""
        _check(lib().srt_ctx_set_bvh_leaf_size(self.h, max_triangles), self.h)

    def synchronize(self):
        _check(lib().srt_ctx_synchronize(self.h), self.h)

    def close(self):
        if self.h:
            lib().srt_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------- scene


def _vertices(v) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(v, dtype=np.float32).reshape(-1, 8))
    return a


def geometry(kind: str, *args) -> tuple[np.ndarray, np.ndarray]:
    """Procedural meshes (src/scene/geometry.rs): 'plane', 'cube', 'icosphere' (subdivisions),
    'uv_sphere' (slices, stacks).  Returns (vertices float32 [n, 8], indices uint32)."""
    fn = {"plane": lib().srt_geometry_plane, "cube": lib().srt_geometry_cube,
          "icosphere": lib().srt_geometry_icosphere, "uv_sphere": lib().srt_geometry_uv_sphere}[kind]
    nv, ni = C.c_uint32(0), C.c_uint32(0)
    _check(fn(*args, None, C.byref(nv), None, C.byref(ni)))
    v = np.zeros((nv.value, 8), np.float32)
    i = np.zeros(ni.value, np.uint32)
    _check(fn(*args, v.ctypes.data_as(C.POINTER(Vertex)), C.byref(nv), i.ctypes.data_as(C.POINTER(C.c_uint32)),
              C.byref(ni)))
    return v, i


def material(color, extra) -> Material:
    m = Material()
    m.color[:] = [float(x) for x in color]
    m.extra[:] = [float(x) for x in extra]
    return m


class SceneBuilder:
    """SceneBuilder (src/scene/builder.rs:47-267) on the native host builder."""

    def __init__(self):
        h = C.c_void_p()
        _check(lib().srt_scene_builder_create(C.byref(h)))
        self.h = h

    def add_material(self, color, extra) -> int:
        m = color if isinstance(color, Material) else material(color, extra)
        return int(lib().srt_scene_builder_add_material(self.h, C.byref(m)))

    def add_mesh(self, vertices, indices) -> int:
        v = _vertices(vertices)
        i = np.ascontiguousarray(np.asarray(indices, np.uint32))
        r = lib().srt_scene_builder_add_mesh(self.h, v.ctypes.data_as(C.POINTER(Vertex)), len(v),
                                             i.ctypes.data_as(C.POINTER(C.c_uint32)), len(i))
        if r == 0xFFFFFFFF:
            raise SrtError(1, "invalid mesh")
        return int(r)

    def add_instance(self, mesh_id: int, mat_id: int, transform) -> None:
        t = np.ascontiguousarray(np.asarray(transform, np.float32).reshape(4, 4).T.reshape(16))  # -> column-major
        _check(lib().srt_scene_builder_add_instance(self.h, mesh_id, mat_id, t.ctypes.data_as(C.POINTER(C.c_float))))

    def add_light_instance(self, mesh_id: int, mat_id: int, transform, params) -> None:
        t = np.ascontiguousarray(np.asarray(transform, np.float32).reshape(4, 4).T.reshape(16))
        p = np.ascontiguousarray(np.asarray(params, np.float32).reshape(4))
        _check(lib().srt_scene_builder_add_light_instance(self.h, mesh_id, mat_id, t.ctypes.data_as(C.POINTER(C.c_float)),
                                                          p.ctypes.data_as(C.POINTER(C.c_float))))

    def add_preset(self, preset: int, seed: int = 0) -> tuple[list[float], float, float]:
        """Fills the builder with a preset scene; returns (camera position, yaw, pitch)."""
        cam = (C.c_float * 5)()
        _check(lib().srt_scene_builder_add_preset(self.h, preset, seed, cam))
        return [cam[0], cam[1], cam[2]], cam[3], cam[4]

    def arrays(self) -> SceneArrays:
        a = SceneArrays()
        _check(lib().srt_scene_builder_arrays(self.h, C.byref(a)))
        return a

    def build(self, ctx: Context) -> "Scene":
        h = C.c_void_p()
        _check(lib().srt_scene_builder_build(ctx.h, self.h, C.byref(h)), ctx.h)
        return Scene(ctx, h)

    def close(self):
        if self.h:
            lib().srt_scene_builder_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Scene:
    """SceneResources (builder.rs:30-39): device buffers + the GPU-built BVH8."""

    def __init__(self, ctx: Context, h):
        self.ctx, self.h = ctx, h

    def info(self) -> dict:
        t, n, d, w = C.c_uint64(), C.c_uint64(), C.c_uint32(), C.c_uint32()
        _check(lib().srt_scene_info(self.h, C.byref(t), C.byref(n), C.byref(d)), self.ctx.h)
        _check(lib().srt_scene_bvh_width(self.h, C.byref(w)), self.ctx.h)
        return {"triangles": t.value, "nodes": n.value, "depth": d.value, "width": w.value}

    def rebuild_bvh(self, width: int) -> None:
        """Rebuilds the tree with `width` children per node (renderers pick it up at their next frame)."""
        _check(lib().srt_scene_rebuild_bvh(self.h, width), self.ctx.h)

    def trace(self, rays: np.ndarray, any_hit: bool = False) -> np.ndarray:
        """rays: float32 [n, 8] (origin, tmin, dir, tmax) -> hits structured (t, prim, u, v)."""
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        out = np.zeros(len(r), dtype=[("t", np.float32), ("prim", np.uint32), ("u", np.float32), ("v", np.float32)])
        _check(lib().srt_trace_rays(self.h, ptr(r), len(r), ptr(out), 1 if any_hit else 0), self.ctx.h)
        return out

    def update_instances(self, ids, transforms) -> None:
        """Moves instances: transforms [n, 16] column-major object-to-world (GPU re-transform + BVH refit)."""
        i = np.ascontiguousarray(ids, np.uint32).reshape(-1)
        t = np.ascontiguousarray(transforms, np.float32).reshape(-1, 16)
        _check(lib().srt_scene_update_instances(self.h, ptr(i), ptr(t), len(i)), self.ctx.h)

    def read_lights(self) -> np.ndarray:
        n = C.c_uint32()
        _check(lib().srt_scene_read_lights(self.h, None, 0, C.byref(n)), self.ctx.h)
        out = np.zeros((n.value, 16), np.float32)
        _check(lib().srt_scene_read_lights(self.h, ptr(out), n.value, C.byref(n)), self.ctx.h)
        return out

    def read_bvh(self):
        info = self.info()
        nodes = np.zeros((info["nodes"], 20), np.uint32)
        tris = np.zeros((info["triangles"], 12), np.float32)
        _check(lib().srt_scene_read_bvh(self.h, ptr(nodes), nodes.nbytes, ptr(tris), tris.nbytes), self.ctx.h)
        return nodes, tris

    def close(self):
        if self.h:
            lib().srt_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def camera_uniform(position, yaw: float, pitch: float, aspect: float, frame_count: int) -> CameraUniform:
    """CameraController::build_uniform (src/scene/camera.rs:178-194)."""
    u = CameraUniform()
    p = (C.c_float * 3)(*[float(x) for x in position])
    _check(lib().srt_camera_build_uniform(p, yaw, pitch, aspect, frame_count, C.byref(u)))
    return u


class CameraController:
    """Camera state of src/scene/camera.rs:15-52 (keyboard handling left out)."""

    def __init__(self, position=(0.0, 0.0, 3.0), yaw: float = -math.pi / 2, pitch: float = 0.0):
        self.position = list(position)
        self.yaw = yaw
        self.pitch = pitch

    def build_uniform(self, aspect: float, frame_count: int) -> CameraUniform:
        return camera_uniform(self.position, self.yaw, self.pitch, aspect, frame_count)


# --------------------------------------------------------------------------- renderer


class Renderer:
    """Renderer (src/renderer/mod.rs:21-208): per-frame photon pass, grid, wavefront camera paths."""

    def __init__(self, ctx: Context, scene: Scene, width: int, height: int, params: Params | None = None):
        self.ctx, self.scene = ctx, scene
        self.target_width, self.target_height = int(width), int(height)
        self.params = params if params is not None else default_params()
        h = C.c_void_p()
        _check(lib().srt_renderer_create(ctx.h, scene.h, width, height, C.byref(self.params), C.byref(h)), ctx.h)
        self.h = h

    @property
    def frame_count(self) -> int:
        return int(lib().srt_renderer_frame_count(self.h))

    @frame_count.setter
    def frame_count(self, v: int):
        _check(lib().srt_renderer_set_frame_count(self.h, v), self.ctx.h)

    def render(self, camera: CameraUniform) -> None:
        _check(lib().srt_render_frame(self.h, C.byref(camera)), self.ctx.h)

    def reset_accumulation(self):
        _check(lib().srt_reset_accumulation(self.h), self.ctx.h)

    def read_accum(self) -> np.ndarray:
        out = np.zeros((self.target_height, self.target_width, 4), np.float32)
        _check(lib().srt_read_accum_f32(self.h, ptr(out)), self.ctx.h)
        return out

    def read_accum64(self) -> np.ndarray:
        out = np.zeros((self.target_height, self.target_width, 4), np.float64)
        _check(lib().srt_read_accum_f64(self.h, ptr(out)), self.ctx.h)
        return out

    def write_accum64(self, sums: np.ndarray) -> None:
        """Loads FP64 sums [h, w, 4] (as read_accum64 returns them) to resume an accumulation; the next
        frame must carry the frame count the sums were read at."""
        a = np.ascontiguousarray(sums, np.float64)
        if a.shape != (self.target_height, self.target_width, 4):
            raise ValueError(f"expected shape {(self.target_height, self.target_width, 4)}, got {a.shape}")
        _check(lib().srt_write_accum_f64(self.h, ptr(a)), self.ctx.h)

    def read_ldr(self) -> np.ndarray:
        out = np.zeros((self.target_height, self.target_width, 4), np.uint8)
        _check(lib().srt_read_ldr_rgba8(self.h, ptr(out), 4 * self.target_width), self.ctx.h)
        return out

    def read_ldr_async(self) -> int:
        """Enqueues a read-back of the current image into a pinned slot; returns its ticket."""
        t = C.c_uint32()
        _check(lib().srt_read_ldr_async(self.h, C.byref(t)), self.ctx.h)
        return t.value

    def ldr_wait(self, ticket: int) -> np.ndarray:
        """The image of `ticket` once its copy has landed (a view of the pinned slot, valid
        until the second read_ldr_async after it)."""
        p = C.POINTER(C.c_uint8)()
        _check(lib().srt_ldr_wait(self.h, ticket, C.byref(p)), self.ctx.h)
        return np.ctypeslib.as_array(p, shape=(self.target_height, self.target_width, 4))

    def save_screenshot(self, path: str | os.PathLike):
        _check(lib().srt_save_screenshot(self.h, str(path).encode()), self.ctx.h)

    def save_screenshot_async(self, path: str | os.PathLike):
        """Reads the image back now; the PNG is encoded and written on the library's worker thread
        (screenshot_flush waits for it)."""
        _check(lib().srt_save_screenshot_async(self.h, str(path).encode()), self.ctx.h)

    def stats(self) -> dict:
        s = Stats()
        _check(lib().srt_renderer_get_stats(self.h, C.byref(s)), self.ctx.h)
        return {f: (list(getattr(s, f)) if f in ("nodes_visited", "tris_tested") else getattr(s, f))
                for f, _ in Stats._fields_}

    def bounce_stats(self) -> dict:
        """Per-bounce arrays [kind][bounce] (kind 0 camera closest, 1 shadow, 2 photon): rays, nodes, tris;
        ms [0 closest, 1 shadow][bounce] (SRT_FLAG_STAGE_TIMING)."""
        s = BounceStats()
        _check(lib().srt_renderer_get_bounce_stats(self.h, C.byref(s)), self.ctx.h)
        return {"rays": np.array(s.rays, np.uint64), "nodes": np.array(s.nodes, np.uint64),
                "tris": np.array(s.tris, np.uint64), "ms": np.array(s.ms, np.float64)}

    def set_tail(self, first_bounce: int) -> None:
        """Bounces >= first_bounce in one persistent kernel per frame (0: bounce by bounce; TAIL_AUTO, the
        default: chosen from the first frame's path counts)."""
        _check(lib().srt_renderer_set_tail(self.h, first_bounce), self.ctx.h)

    def reset_stats(self):
        _check(lib().srt_renderer_reset_stats(self.h), self.ctx.h)

    def read_photons(self) -> np.ndarray:
        n = C.c_uint32()
        _check(lib().srt_renderer_read_photons(self.h, None, 0, C.byref(n)), self.ctx.h)
        out = np.zeros((n.value, 8), np.float32)
        _check(lib().srt_renderer_read_photons(self.h, ptr(out), n.value, C.byref(n)), self.ctx.h)
        return out

    def blit(self, window_width: int, window_height: int, srgb_target: bool = False) -> np.ndarray:
        """Headless letterbox blit of the current image into a window-sized RGBA8 array (row 0 on top)."""
        out = np.zeros((window_height, window_width, 4), np.uint8)
        _check(lib().srt_renderer_blit(self.h, window_width, window_height, int(srgb_target), ptr(out)), self.ctx.h)
        return out

    def splat_photons(self, camera: CameraUniform, rgba: np.ndarray) -> np.ndarray:
        """Photon point splat of the last frame's stored photons over rgba [h, w, 4] (returns a copy)."""
        a = np.ascontiguousarray(rgba, np.uint8).copy()
        h, w = a.shape[:2]
        _check(lib().srt_renderer_splat_photons(self.h, C.byref(camera), w, h, ptr(a)), self.ctx.h)
        return a

    # neural path guiding (FLAG_GUIDING)
    def guide_weights(self) -> np.ndarray:
        out = np.zeros(guide_param_count(), np.float32)
        _check(lib().srt_renderer_guide_get_weights(self.h, ptr(out), len(out)), self.ctx.h)
        return out

    def guide_state(self) -> dict:
        """Checkpoint of the guide's training state: weights, Adam moments and step count."""
        n = guide_param_count()
        p, m, v = (np.zeros(n, np.float32) for _ in range(3))
        step = C.c_uint32()
        _check(lib().srt_renderer_guide_get_state(self.h, ptr(p), ptr(m), ptr(v), C.byref(step)), self.ctx.h)
        return {"params": p, "adam_m": m, "adam_v": v, "adam_step": step.value}

    def set_guide_state(self, state: dict) -> None:
        p, m, v = (np.ascontiguousarray(state[k], np.float32) for k in ("params", "adam_m", "adam_v"))
        n = guide_param_count()
        if not (p.size == m.size == v.size == n):
            raise ValueError(f"expected {n} values per array")
        _check(lib().srt_renderer_guide_set_state(self.h, ptr(p), ptr(m), ptr(v), int(state["adam_step"])),
               self.ctx.h)

    def set_guide_inference(self, kind: int) -> None:
        """GUIDE_INFER_MMA_SYNC or GUIDE_INFER_TCGEN05."""
        _check(lib().srt_renderer_guide_set_inference(self.h, kind), self.ctx.h)

    def set_guide_training(self, kind: int) -> None:
        """GUIDE_TRAIN_MMA_SYNC or GUIDE_TRAIN_TCGEN05."""
        _check(lib().srt_renderer_guide_set_training(self.h, kind), self.ctx.h)

    def set_guide_weights(self, w: np.ndarray) -> None:
        a = np.ascontiguousarray(w, np.float32)
        _check(lib().srt_renderer_guide_set_weights(self.h, ptr(a), len(a)), self.ctx.h)

    def guide_info(self) -> dict:
        steps, thr = C.c_uint32(), C.c_uint32()
        _check(lib().srt_renderer_guide_info(self.h, C.byref(steps), C.byref(thr)), self.ctx.h)
        return {"adam_steps": steps.value, "record_threshold": thr.value}

    def set_guide_steps(self, steps: int) -> None:
        """Adam steps per frame, each on a consecutive 1/steps of the frame's training records."""
        _check(lib().srt_renderer_guide_set_steps(self.h, steps), self.ctx.h)

    def set_guide_bounces(self, bounces: int) -> None:
        """Guide the Lambert continuations of bounces < `bounces` only (default 8; later ones sample the
        cosine lobe)."""
        _check(lib().srt_renderer_guide_set_bounces(self.h, bounces), self.ctx.h)

    def configure_guide(self, lr: float | None = None, batch: int | None = None) -> None:
        """Adam learning rate and training samples recorded per frame."""
        _check(lib().srt_renderer_guide_configure(self.h, -1.0 if lr is None else lr, batch or 0), self.ctx.h)

    def close(self):
        if self.h:
            lib().srt_renderer_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------- standalone kernels


def screenshot_write(path, rgba: np.ndarray) -> None:
    """ScreenshotSaver (src/screenshot.rs:27-103): rgba uint8 [h, w, 4], row 0 = bottom."""
    a = np.ascontiguousarray(rgba, np.uint8)
    h, w = a.shape[:2]
    _check(lib().srt_screenshot_write(str(path).encode(), ptr(a), w, h, 4 * w))


def screenshot_write_async(path, rgba: np.ndarray) -> None:
    """screenshot_write on the library's worker thread (the pixels are copied before this returns)."""
    a = np.ascontiguousarray(rgba, np.uint8)
    h, w = a.shape[:2]
    _check(lib().srt_screenshot_write_async(str(path).encode(), ptr(a), w, h, 4 * w))


def screenshot_flush() -> int:
    """Waits for every queued screenshot write; returns how many failed since the previous flush."""
    n = C.c_uint32()
    _check(lib().srt_screenshot_flush(C.byref(n)))
    return n.value


def photon_grid_build(ctx: Context, photons: np.ndarray, frame: int, cell: float = 0.02, hash_bits: int = 22):
    """Cell keys (sorted, u64) and ranges ([2^bits, 2] u32) for a photon set float32 [n, 8]."""
    p = np.ascontiguousarray(photons, np.float32).reshape(-1, 8)
    keys = np.zeros(len(p), np.uint64)
    ranges = np.zeros((1 << hash_bits, 2), np.uint32)
    _check(lib().srt_photon_grid_build(ctx.h, ptr(p), len(p), frame, cell, hash_bits, ptr(keys), ptr(ranges)), ctx.h)
    return keys, ranges


def photon_gather(ctx: Context, photons: np.ndarray, queries: np.ndarray, frame: int, params: Params) -> np.ndarray:
    p = np.ascontiguousarray(photons, np.float32).reshape(-1, 8)
    q = np.ascontiguousarray(queries, np.float32).reshape(-1, 10)
    out = np.zeros((len(q), 4), np.float32)
    _check(lib().srt_photon_gather(ctx.h, ptr(p), len(p), ptr(q), len(q), frame, C.byref(params), ptr(out)), ctx.h)
    return out


MATH_SIZES = {0: (4, 4), 1: (4, 12), 2: (8, 4), 3: (28, 16), 4: (36, 16), 5: (4, 20), 6: (96, 40), 7: (20, 4),
              8: (20, 28)}


def device_math(ctx: Context, op: int, inp: np.ndarray, aux: CameraUniform | None = None) -> np.ndarray:
    """Runs one device unit kernel (srt_test_device_math); inp rows are op records."""
    isz, osz = MATH_SIZES[op]
    a = np.ascontiguousarray(inp)
    n = a.nbytes // isz
    out = np.zeros(n * osz // 4, np.uint32 if op in (0, 7) else np.float32)
    _check(lib().srt_test_device_math(ctx.h, op, n, ptr(a), ptr(out), C.byref(aux) if aux is not None else None), ctx.h)
    return out.reshape(n, osz // 4)


# --------------------------------------------------------------------------- path guiding


def guide_param_count() -> int:
    return int(lib().srt_guide_param_count())


def guide_default_weights(seed: int = 1) -> np.ndarray:
    out = np.zeros(guide_param_count(), np.float32)
    _check(lib().srt_guide_default_weights(seed, ptr(out), len(out)))
    return out


def wait_timeout_check(ctx: Context, polls: int = 1000) -> None:
    """Runs a device wait that cannot complete (bounded by `polls`); raises SrtError with SRT_ERR_TIMEOUT."""
    _check(lib().srt_test_wait_timeout(ctx.h, polls), ctx.h)


def guide_forward(ctx: Context, params: np.ndarray, x: np.ndarray, tcgen05: bool = False) -> np.ndarray:
    """Raw network outputs [n, 48] for inputs x [n, 10] (srt_guide_test_forward[_tc])."""
    w = np.ascontiguousarray(params, np.float32)
    a = np.ascontiguousarray(x, np.float32).reshape(-1, 10)
    out = np.zeros((len(a), 48), np.float32)
    fn = lib().srt_guide_test_forward_tc if tcgen05 else lib().srt_guide_test_forward
    _check(fn(ctx.h, ptr(w), ptr(a), len(a), ptr(out)), ctx.h)
    return out


def guide_mixture(ctx: Context, raw: np.ndarray, omega: np.ndarray, u: np.ndarray, tcgen05: bool = False) -> np.ndarray:
    """[n, 4]: mixture pdf at omega and a direction sampled with u (srt_guide_test_mixture; tcgen05: the
    mixture functions of the tcgen05 inference kernel, srt_guide_test_mixture_tc)."""
    r = np.ascontiguousarray(raw, np.float32).reshape(-1, 48)
    o = np.ascontiguousarray(omega, np.float32).reshape(-1, 3)
    uu = np.ascontiguousarray(u, np.float32).reshape(-1, 3)
    out = np.zeros((len(r), 4), np.float32)
    fn = lib().srt_guide_test_mixture_tc if tcgen05 else lib().srt_guide_test_mixture
    _check(fn(ctx.h, ptr(r), ptr(o), ptr(uu), len(r), ptr(out)), ctx.h)
    return out


def guide_train_step(ctx: Context, params, x, omega, pdf_bsdf, weight, adam_m=None, adam_v=None, adam_step=0,
                     lr=1e-3, adam=True, tcgen05=False):
    """Loss gradients (summed over the samples) and, with adam, the parameters
    and Adam moments after one step (srt_guide_test_train; tcgen05: the fused
    tensor-core training kernel, srt_guide_test_train_tc)."""
    n = len(x)
    w = np.ascontiguousarray(params, np.float32)
    m = None if adam_m is None else np.ascontiguousarray(adam_m, np.float32)
    v = None if adam_v is None else np.ascontiguousarray(adam_v, np.float32)
    xs = np.ascontiguousarray(x, np.float32).reshape(-1, 10)
    om = np.ascontiguousarray(omega, np.float32).reshape(-1, 3)
    pb = np.ascontiguousarray(pdf_bsdf, np.float32).reshape(-1)
    wt = np.ascontiguousarray(weight, np.float32).reshape(-1)
    grad = np.zeros_like(w)
    outs = [np.zeros_like(w) for _ in range(3)] if adam else [None, None, None]
    fn = lib().srt_guide_test_train_tc if tcgen05 else lib().srt_guide_test_train
    _check(fn(ctx.h, ptr(w), ptr(m) if m is not None else None,
                                      ptr(v) if v is not None else None, adam_step, lr, ptr(xs), ptr(om), ptr(pb),
                                      ptr(wt), n, ptr(grad), *(ptr(o) if o is not None else None for o in outs)),
           ctx.h)
    return (grad, *outs) if adam else grad


# --------------------------------------------------------------------------- headless presentation


def blit_letterbox(ctx: Context, src: np.ndarray, window_width: int, window_height: int,
                   srgb_target: bool = False) -> np.ndarray:
    """BlitPass (blit.wgsl, blit_pass.rs:114-154) headless: src RGBA8 [sh, sw, 4] -> window RGBA8."""
    a = np.ascontiguousarray(src, np.uint8)
    sh, sw = a.shape[:2]
    out = np.zeros((window_height, window_width, 4), np.uint8)
    _check(lib().srt_blit_letterbox(ctx.h, ptr(a), sw, sh, window_width, window_height, int(srgb_target), ptr(out)),
           ctx.h)
    return out


def photon_splat(ctx: Context, photons: np.ndarray, camera: CameraUniform, rgba: np.ndarray) -> np.ndarray:
    """DebugPhotonsPass (debug_photons.wgsl) headless: photons float32 [n, 8] over rgba [h, w, 4]."""
    p = np.ascontiguousarray(photons, np.float32).reshape(-1, 8)
    a = np.ascontiguousarray(rgba, np.uint8).copy()
    h, w = a.shape[:2]
    _check(lib().srt_photon_splat(ctx.h, ptr(p), len(p), C.byref(camera), w, h, ptr(a)), ctx.h)
    return a


# --------------------------------------------------------------------------- batched rendering


class _BorrowedRenderer(Renderer):
    """A scene's renderer inside a Batch (read-only use; owned by the batch)."""

    def __init__(self, batch, i, handle, width, height, params):
        self.ctx, self.scene = batch.ctx, batch.scenes[i]
        self.target_width, self.target_height = int(width), int(height)
        self.params = params
        self.h = handle

    def render(self, camera):
        raise SrtError(1, "a batched scene renders through Batch.render")

    def close(self):
        self.h = None


class Batch:
    """Many scenes and viewports per iteration (srt_batch_*): per-scene stages as
    parallel CUDA-graph branches, all scenes' rays traced in shared launches."""

    def __init__(self, ctx: Context, scenes, sizes, params=None):
        self.ctx, self.scenes = ctx, list(scenes)
        n = len(self.scenes)
        self.sizes = [(int(w), int(h)) for w, h in sizes]
        self.params = list(params) if params is not None else [default_params() for _ in range(n)]
        hs = (C.c_void_p * n)(*[s.h.value if isinstance(s.h, C.c_void_p) else s.h for s in self.scenes])
        ws = (C.c_uint32 * n)(*[w for w, _ in self.sizes])
        hh = (C.c_uint32 * n)(*[h for _, h in self.sizes])
        ps = (Params * n)(*self.params)
        h = C.c_void_p()
        _check(lib().srt_batch_create(ctx.h, n, hs, ws, hh, ps, C.byref(h)), ctx.h)
        self.h = h
        self.renderers = [_BorrowedRenderer(self, i, C.c_void_p(lib().srt_batch_renderer(self.h, i)), w, hgt,
                                            self.params[i]) for i, (w, hgt) in enumerate(self.sizes)]

    def __len__(self):
        return len(self.scenes)

    def render(self, cameras, active=None) -> None:
        n = len(self.scenes)
        cams = (CameraUniform * n)(*cameras)
        act = None if active is None else (C.c_uint8 * n)(*[1 if a else 0 for a in active])
        _check(lib().srt_batch_render(self.h, cams, act), self.ctx.h)

    def tuning(self) -> dict:
        t = BatchTuning()
        _check(lib().srt_batch_get_tuning(self.h, C.byref(t)), self.ctx.h)
        return {f: getattr(t, f) for f, _ in BatchTuning._fields_}

    def set_tuning(self, blocks_per_sm: int, chunk: int) -> None:
        t = BatchTuning(blocks_per_sm, chunk, 0.0, 0)
        _check(lib().srt_batch_set_tuning(self.h, C.byref(t)), self.ctx.h)

    def autotune(self, cameras, iterations: int = 2) -> dict:
        n = len(self.scenes)
        cams = (CameraUniform * n)(*cameras)
        t = BatchTuning()
        _check(lib().srt_batch_autotune(self.h, cams, iterations, C.byref(t)), self.ctx.h)
        return {f: getattr(t, f) for f, _ in BatchTuning._fields_}

    def close(self):
        if self.h:
            for r in self.renderers:
                r.h = None
            lib().srt_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
