"""The oracle's own scene generator (oracle/scenes.cpp) against the product's
scene builder, on the CPU: every preset's arrays are equal byte for byte, and
the camera uniforms agree to rounding.  The oracle and the CPU baseline take
their scenes from that generator, so the geometry restatement of the product
(geometry.rs:12-232, cornell_box.rs:6-110, custom.rs:6-116, builder.rs:101-129
and the project's synthetic scenes) is checked by independent code."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

FIELDS = (("vertices", "n_vertices", 32), ("indices", "n_indices", 4), ("mesh_infos", "n_meshes", 16),
          ("materials", "n_materials", 32), ("instances", "n_instances", 80), ("lights", "n_lights", 64))


def _bytes(arrays, name, count, size):
    p = C.cast(getattr(arrays, name), C.c_void_p).value
    n = getattr(arrays, count)
    return C.string_at(p, n * size) if n else b""


@pytest.mark.parametrize("preset,seed", [(0, 0), (1, 0), (2, 0), (3, 0), (4, 0), (5, 0), (6, 0), (6, 3), (6, 7),
                                         (6, 11), (6, 29)])
def test_preset_arrays_equal_the_products(srt, orc, preset, seed):
    mine = orc.Preset(preset, seed)
    b = srt.SceneBuilder()
    cam = b.add_preset(preset, seed)
    a, o = b.arrays(), mine.arrays()
    for name, count, size in FIELDS:
        assert getattr(a, count) == getattr(o, count), name
        assert _bytes(a, name, count, size) == _bytes(o, name, count, size), name
    pos, yaw, pitch = cam
    mpos, myaw, mpitch = mine.camera
    assert list(pos) == list(mpos) and yaw == myaw and pitch == mpitch
    mine.close()


def test_config2_triangle_count(orc):
    # 20 * 4^8 icosphere triangles + 64 spheres of 4,032 + 6 planes of 2
    assert orc.Preset(3, 0).n_triangles() == 1310720 + 64 * 4032 + 12 == 1568780


@pytest.mark.parametrize("pos,yaw,pitch,aspect", [([0.0, 0.0, 3.0], -math.pi / 2, 0.0, 1.0),
                                                  ([0.0, 1.0, 6.0], -math.pi / 2, -0.12, 16 / 9),
                                                  ([0.3, -0.2, 2.0], -1.2, 0.3, 4 / 3)])
def test_camera_uniform_matches_the_products(srt, orc, pos, yaw, pitch, aspect):
    """camera.rs:178-194: the oracle's closed-form inverses and the product's
    agree to FP32 rounding."""
    a = srt.camera_uniform(pos, yaw, pitch, aspect, 9)
    o = orc.camera_uniform(pos, yaw, pitch, aspect, 9)
    for f in ("view", "proj", "view_inverse", "proj_inverse"):
        x = np.array(getattr(a, f), np.float64)
        y = np.array(getattr(o, f), np.float64)
        assert np.abs(x - y).max() <= 2e-6 * max(1.0, np.abs(y).max()), f
    assert a.frame_count == o.frame_count == 9
