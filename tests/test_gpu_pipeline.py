"""Photon-pass pipelining: a frame builds the next frame's photon map on a
branch of its own, beside its camera paths.  The frames must be those of the
serial renderer (stage timing keeps every stage in order and builds each
frame's map inside the frame), bit for bit, also when the frame count jumps
(the map built ahead is for the wrong frame), when the scene moves between
frames (the map built ahead is stale), and without the frame graph; the photon
set read back after a frame is that frame's."""
from __future__ import annotations

import math

import numpy as np
import pytest

from test_gpu_scene_update import CUBE, LIGHT, T0, T1, _build, _colmajor

pytestmark = pytest.mark.gpu


def _renderers(srt, ctx, scene, w, h):
    p = dict(photons_per_frame=1 << 16, max_depth=8)
    return {"graph": srt.Renderer(ctx, scene, w, h, srt.default_params(**p)),
            "direct": srt.Renderer(ctx, scene, w, h, srt.default_params(flags=srt.FLAG_NO_GRAPH, **p)),
            "serial": srt.Renderer(ctx, scene, w, h, srt.default_params(flags=srt.FLAG_STAGE_TIMING, **p))}


def test_pipelined_frames_equal_serial_frames(srt, ctx):
    _, scene = _build(srt, ctx, **T0)
    w, h = 48, 40
    cam = srt.CameraController([0.0, 0.0, 3.0], -math.pi / 2, 0.0)
    rs = _renderers(srt, ctx, scene, w, h)
    # frame counts in order, a jump back to 0 (a reset), then on; the scene
    # moves before the sixth frame
    for i, f in enumerate([0, 1, 2, 3, 0, 1, 2, 5, 6]):
        if i == 5:
            scene.update_instances([LIGHT, CUBE], np.stack([_colmajor(T1["light_t"]), _colmajor(T1["cube_t"])]))
        u = cam.build_uniform(w / h, f)
        for r in rs.values():
            r.render(u)
        ref = rs["serial"].read_accum()
        ref_ph = rs["serial"].read_photons()
        assert ref_ph.shape[0] > 0
        for name in ("graph", "direct"):
            np.testing.assert_array_equal(rs[name].read_accum(), ref, err_msg=f"{name}, frame {i} (count {f})")
            np.testing.assert_array_equal(rs[name].read_photons(), ref_ph, err_msg=f"{name} photons, frame {i}")
    st = {k: r.stats() for k, r in rs.items()}
    for k in ("rays_closest", "rays_shadow", "rays_photon", "paths"):
        assert st["graph"][k] == st["serial"][k] == st["direct"][k], k
    for r in rs.values():
        r.close()
    scene.close()


def test_pipelined_guided_frames_equal_serial_frames(srt, ctx):
    """A guiding renderer (frozen guide: the same network in every renderer):
    the training branch, the photon branch and the camera paths together."""
    b = srt.SceneBuilder()
    cam = srt.CameraController(*b.add_preset(srt.PRESET_CAUSTIC_SLAB))
    scene = b.build(ctx)
    w, h = 40, 24
    p = dict(photons_per_frame=1 << 15, max_depth=12, flags=srt.FLAG_GUIDING | srt.FLAG_GUIDE_FROZEN)
    a = srt.Renderer(ctx, scene, w, h, srt.default_params(**p))
    s = srt.Renderer(ctx, scene, w, h, srt.default_params(**{**p, "flags": p["flags"] | srt.FLAG_STAGE_TIMING}))
    for f in range(5):
        u = cam.build_uniform(w / h, f)
        a.render(u)
        s.render(u)
    np.testing.assert_array_equal(a.read_accum(), s.read_accum())
    a.close()
    s.close()
    scene.close()
