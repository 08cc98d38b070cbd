"""Scene-side GPU ingestion: light instances expanded on the device match the
host builder's expansion bit for bit; moving instances (re-transform on the
GPU + BVH8 refit) gives the same lights, ray hits and frames as building the
moved scene from scratch; a refit without motion leaves the tree unchanged."""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _t(tx=0.0, ty=0.0, tz=0.0, sx=1.0, sy=1.0, sz=1.0, rx=0.0, ry=0.0):
    """Row-major 4x4: translate * rot_y * rot_x * scale."""
    S = np.diag([sx, sy, sz, 1.0])
    cx, sxn = math.cos(rx), math.sin(rx)
    Rx = np.array([[1, 0, 0, 0], [0, cx, -sxn, 0], [0, sxn, cx, 0], [0, 0, 0, 1]])
    cy, syn = math.cos(ry), math.sin(ry)
    Ry = np.array([[cy, 0, syn, 0], [0, 1, 0, 0], [-syn, 0, cy, 0], [0, 0, 0, 1]])
    T = np.eye(4)
    T[:3, 3] = [tx, ty, tz]
    return (T @ Ry @ Rx @ S).astype(np.float32)


WALLS = [_t(0, -1, 0, 2, 2, 2), _t(0, 1, 0, 2, 2, 2, rx=math.pi), _t(0, 0, -1, 2, 2, 2, rx=math.pi / 2)]
LIGHT, CUBE, SPHERE = 3, 4, 5  # instance ids in build order


def _build(srt, ctx, light_t, cube_t, sphere_t):
    b = srt.SceneBuilder()
    white = b.add_material((0.73, 0.73, 0.73, 1), (0, 0, 0, 0))
    light = b.add_material((6500, 4, 0, 1), (3, 0, 0, 0))
    glass = b.add_material((1, 1, 1, 1), (2, 0, 1.5, 0.004))
    plane = b.add_mesh(*srt.geometry("plane"))
    cube = b.add_mesh(*srt.geometry("cube"))
    ball = b.add_mesh(*srt.geometry("icosphere", 3))
    for w in WALLS:
        b.add_instance(plane, white, w)
    b.add_light_instance(plane, light, light_t, (0, 6500, 4, 0))
    b.add_instance(cube, white, cube_t)
    b.add_instance(ball, glass, sphere_t)
    return b, b.build(ctx)


T0 = dict(light_t=_t(0, 0.99, 0, 0.5, 0.5, 0.5, rx=math.pi), cube_t=_t(-0.35, -0.6, -0.3, 0.5, 0.8, 0.5, ry=0.4),
          sphere_t=_t(0.4, -0.64, 0.3, 0.6, 0.6, 0.6))
T1 = dict(light_t=_t(0.2, 0.95, -0.1, 0.4, 0.4, 0.4, rx=math.pi), cube_t=_t(0.25, -0.5, 0.1, 0.5, 1.0, 0.5, ry=1.1),
          sphere_t=T0["sphere_t"])


def _colmajor(t):
    return np.ascontiguousarray(t.T.reshape(16))


def _rays(n, seed):
    rng = np.random.default_rng(seed)
    o = rng.uniform(-0.9, 0.9, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3] = 1e-4
    r[:, 4:7] = d
    r[:, 7] = 100.0
    return r


@pytest.mark.parametrize("preset", [0, 2, 4])
def test_gpu_light_expansion_matches_host(srt, ctx, preset):
    b = srt.SceneBuilder()
    b.add_preset(preset)
    a = b.arrays()
    host = np.ctypeslib.as_array(C_lights(a), shape=(a.n_lights, 16)).copy()
    scene = b.build(ctx)
    np.testing.assert_array_equal(scene.read_lights(), host)
    scene.close()


def C_lights(a):
    import ctypes as C

    return C.cast(a.lights, C.POINTER(C.c_float))


def test_refit_without_motion_keeps_the_tree(srt, ctx):
    _, s = _build(srt, ctx, **T0)
    nodes0, tris0 = s.read_bvh()
    s.update_instances([LIGHT, CUBE, SPHERE], np.stack([_colmajor(T0[k]) for k in ("light_t", "cube_t", "sphere_t")]))
    nodes1, tris1 = s.read_bvh()
    np.testing.assert_array_equal(tris1, tris0)
    np.testing.assert_array_equal(nodes1, nodes0)
    s.close()


def test_moved_instances_match_a_fresh_build(srt, ctx):
    _, moved = _build(srt, ctx, **T0)
    cam = ([0.0, 0.0, 3.0], -math.pi / 2, 0.0)
    w, h = 48, 40
    p = srt.default_params(photons_per_frame=1 << 14)
    r_moved = srt.Renderer(ctx, moved, w, h, p)
    u0 = srt.CameraController(*cam).build_uniform(w / h, 0)
    r_moved.render(u0)  # graph captured before the update
    ctx.synchronize()
    moved.update_instances([LIGHT, CUBE], np.stack([_colmajor(T1["light_t"]), _colmajor(T1["cube_t"])]))
    _, fresh = _build(srt, ctx, **T1)
    np.testing.assert_array_equal(moved.read_lights(), fresh.read_lights())
    rays = _rays(40_000, 5)
    hm, hf = moved.trace(rays), fresh.trace(rays)
    for k in ("prim", "t", "u", "v"):
        np.testing.assert_array_equal(hm[k], hf[k])
    # any-hit: the occlusion answer (its t is whichever hit ended the search)
    np.testing.assert_array_equal(moved.trace(rays, True)["prim"], fresh.trace(rays, True)["prim"])
    r_fresh = srt.Renderer(ctx, fresh, w, h, p)
    r_moved.reset_accumulation()
    for f in range(3):
        u = srt.CameraController(*cam).build_uniform(w / h, f)
        r_moved.render(u)
        r_fresh.render(u)
    np.testing.assert_array_equal(r_moved.read_accum(), r_fresh.read_accum())
    for x in (r_moved, r_fresh, moved, fresh):
        x.close()


def test_update_rejects_bad_input(srt, ctx):
    _, s = _build(srt, ctx, **T0)
    with pytest.raises(srt.SrtError):
        s.update_instances([99], _colmajor(T0["cube_t"])[None])
    with pytest.raises(srt.SrtError):
        s.update_instances([CUBE], np.zeros((1, 16), np.float32))  # singular
    s.close()


@pytest.mark.parametrize("preset", [0, 1, 2, 4, 5])
def test_gpu_light_expansion_matches_oracle_expansion(srt, orc, ctx, preset):
    """The device expansion of light instances (builder.rs:101-129) against the
    oracle's own restatement of the builder (oracle/scenes.cpp), bit for bit."""
    b = srt.SceneBuilder()
    b.add_preset(preset)
    scene = b.build(ctx)
    mine = orc.Preset(preset)
    a = mine.arrays()
    import ctypes as C

    ref = np.ctypeslib.as_array(C.cast(a.lights, C.POINTER(C.c_float)), shape=(a.n_lights, 16)).copy()
    np.testing.assert_array_equal(scene.read_lights(), ref)
    scene.close()
    mine.close()


def test_moved_scene_hits_match_the_oracle(srt, orc, ctx):
    """After srt_scene_update_instances, the moved scene's closest hits against
    the FP64 oracle's brute force over the moved scene's arrays: exact outside
    the named exclusion set."""
    from conftest import closest_hit_parity, report

    _, moved = _build(srt, ctx, **T0)
    moved.update_instances([LIGHT, CUBE], np.stack([_colmajor(T1["light_t"]), _colmajor(T1["cube_t"])]))
    b1, _unused = _build(srt, ctx, **T1)
    o = orc.OracleScene(b1.arrays())
    rays = _rays(40_000, 6)
    d = closest_hit_parity(moved, o, rays, brute=True)
    report("moved scene", d)
    assert len(d["bad"]) == 0
    assert d["max_dt_over_bound"] <= 1.0
    _unused.close()
    moved.close()
    o.close()


def test_tree_rebuild_mid_render_keeps_frames_bit_identical(srt, ctx):
    """srt_scene_rebuild_bvh between frames (4 children per node, then 8
    again): the renderer captures its frame again on the new tree and the
    image equals that of a renderer whose scene was never rebuilt."""
    b = srt.SceneBuilder()
    cam = b.add_preset(srt.PRESET_CONFIG1)
    s1, s2 = b.build(ctx), b.build(ctx)
    w, h = 40, 32
    p = srt.default_params(photons_per_frame=1 << 15)
    r1, r2 = srt.Renderer(ctx, s1, w, h, p), srt.Renderer(ctx, s2, w, h, p)
    ctl = srt.CameraController(*cam)
    for f in range(6):
        if f == 2:
            s1.rebuild_bvh(4)
            assert s1.info()["width"] == 4 and s1.info()["nodes"] > s2.info()["nodes"]
        if f == 4:
            s1.rebuild_bvh(8)
        u = ctl.build_uniform(w / h, f)
        r1.render(u)
        r2.render(u)
    np.testing.assert_array_equal(r1.read_accum(), r2.read_accum())
    for x in (r1, r2, s1, s2):
        x.close()
