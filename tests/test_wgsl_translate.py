"""oracle/wgsl_translate.py and oracle/ref_runtime.h on small inputs: the
translation rules (abstract floats become f32, swizzles, parenthesised
conditions, declarations, refusals of what it does not handle) and, compiled
with g++, the runtime's reading of WGSL built-ins against the formulas of the
WGSL specification (float remainder, reflect, refract, sign, saturating
conversions, column-major matrix products, left-to-right constructor
arguments)."""
from __future__ import annotations

import ctypes as C
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ORACLE = Path(__file__).resolve().parents[1] / "oracle"
sys.path.insert(0, str(ORACLE))

import wgsl_translate as wt  # noqa: E402


def _tr(src: str) -> str:
    return wt.Translator(src, "t").run()


def test_literals_swizzles_and_statements():
    out = _tr("""
struct S { a: vec4f, n: u32, }
const K = 0.5;
fn f(v: vec4f, s: S) -> vec3f {
    let x = 1.0 + 2e-3 + 3u + 4i;
    var y: f32;
    var z = v.xyz * v.r;
    if z.x > 0.0 { y = 1.0; } else if z.y > 0.0 { y = 2.0; } else { y = 3.0; }
    for (var i = 0u; i < s.n; i++) { y += 1.0; }
    return z + vec3f(y) * K;
}
""")
    assert "static const auto K = 0.5f;" in out
    assert "1.0f + 2e-3f + 3u + 4" in out
    assert "float y{};" in out
    assert "v . sw<0,1,2>() * v . x" in out
    assert "if (z . x > 0.0f)" in out and "else if (z . y > 0.0f)" in out
    assert "for (auto i = 0u; i < s . n; i ++)" in out
    assert "wgsl_rt::vec3f { y }" in out  # constructors as braced lists
    assert "vec3f f(vec4f v, S s);" in out  # prototypes before the bodies
    assert "uint32_t n{};" in out


@pytest.mark.parametrize("src", [
    "fn f(x: u32) -> u32 { switch x { default: { return 1u; } } }",
    "fn f() { loop { continuing { } } }",
    "var<private> s: u32;\nfn d() -> u32 { s = s + 1u; return s; }\nfn f() -> u32 { return d() + d(); }",
])
def test_translator_refuses_what_it_cannot_keep(src):
    with pytest.raises(wt.WgslError):
        _tr(src)


PROBE = """
var<private> s: u32;
fn draw() -> f32 { s = s * 3u + 1u; return f32(s); }
fn rem(a: vec4f, b: f32) -> vec4f { return a % b; }
fn refl(i: vec3f, n: vec3f) -> vec3f { return reflect(i, n); }
fn refr(i: vec3f, n: vec3f, e: f32) -> vec3f { return refract(i, n, e); }
fn sgn(x: f32) -> f32 { return sign(x); }
fn conv(x: f32) -> vec2u { return vec2u(u32(x), u32(i32(x))); }
fn mv(a: vec3f, b: vec3f, c: vec3f, v: vec3f) -> vec3f { return mat3x3f(a, b, c) * v; }
fn vm(a: vec3f, b: vec3f, c: vec3f, v: vec3f) -> vec3f { return v * mat3x3f(a, b, c); }
fn order() -> vec2f { s = 1u; return vec2f(draw(), draw()); }
fn sq(x: f32) -> f32 { return pow(x, 2.0); }
"""

GLUE = r"""
#include "ref_runtime.h"
#include "probe.inc"
using namespace wgsl_rt;
extern "C" {
void p_rem(const float* a, float b, float* o) { vec4f r = t::rem(vec4f(a[0], a[1], a[2], a[3]), b); for (int k = 0; k < 4; ++k) o[k] = r[k]; }
void p_refl(const float* i, const float* n, float* o) { vec3f r = t::refl(vec3f(i[0], i[1], i[2]), vec3f(n[0], n[1], n[2])); o[0] = r.x; o[1] = r.y; o[2] = r.z; }
void p_refr(const float* i, const float* n, float e, float* o) { vec3f r = t::refr(vec3f(i[0], i[1], i[2]), vec3f(n[0], n[1], n[2]), e); o[0] = r.x; o[1] = r.y; o[2] = r.z; }
float p_sgn(float x) { return t::sgn(x); }
void p_conv(float x, uint32_t* o) { vec2u r = t::conv(x); o[0] = r.x; o[1] = r.y; }
void p_mv(const float* m, const float* v, float* o, int right) {
    vec3f a(m[0], m[1], m[2]), b(m[3], m[4], m[5]), c(m[6], m[7], m[8]), w(v[0], v[1], v[2]);
    vec3f r = right ? t::vm(a, b, c, w) : t::mv(a, b, c, w); o[0] = r.x; o[1] = r.y; o[2] = r.z; }
void p_order(float* o) { vec2f r = t::order(); o[0] = r.x; o[1] = r.y; }
float p_sq(float x) { return t::sq(x); }
}
"""


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    d = tmp_path_factory.mktemp("wgsl")
    (d / "probe.inc").write_text(_tr(PROBE))
    (d / "glue.cpp").write_text(GLUE)
    so = d / "libprobe.so"
    subprocess.run(["g++", "-O2", "-std=c++20", "-ffp-contract=off", "-fPIC", "-shared", f"-I{ORACLE}", f"-I{d}",
                    "-o", str(so), str(d / "glue.cpp")], check=True)
    L = C.CDLL(str(so))
    F = C.c_float
    P = C.c_void_p
    L.p_rem.argtypes = [P, F, P]
    L.p_refl.argtypes = [P, P, P]
    L.p_refr.argtypes = [P, P, F, P]
    L.p_sgn.argtypes = [F]
    L.p_sgn.restype = F
    L.p_conv.argtypes = [F, P]
    L.p_mv.argtypes = [P, P, P, C.c_int]
    L.p_order.argtypes = [P]
    L.p_sq.argtypes = [F]
    L.p_sq.restype = F
    return L


def _f(*v):
    return np.array(v, np.float32)


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


def test_runtime_builtins_follow_the_specification(probe):
    f32 = np.float32
    # e1 % e2 = e1 - e2 * trunc(e1 / e2), every step in f32
    a = _f(405.5, -7.25, 1199.0, 380.0)
    o = np.zeros(4, np.float32)
    probe.p_rem(_ptr(a), 400.0, _ptr(o))
    want = [f32(x) - f32(400.0) * np.trunc(f32(x) / f32(400.0)) for x in a]
    assert np.array_equal(o, np.array(want, np.float32))
    # reflect(e1, e2) = e1 - 2 dot(e2, e1) e2
    i, n = _f(0.6, -0.8, 0.0), _f(0.0, 1.0, 0.0)
    o3 = np.zeros(3, np.float32)
    probe.p_refl(_ptr(i), _ptr(n), _ptr(o3))
    assert np.allclose(o3, [0.6, 0.8, 0.0])
    # refract: k < 0 gives the zero vector (total internal reflection)
    probe.p_refr(_ptr(_f(0.9, -0.43588989, 0.0)), _ptr(n), 1.5, _ptr(o3))
    assert np.array_equal(o3, np.zeros(3, np.float32))
    probe.p_refr(_ptr(_f(0.0, -1.0, 0.0)), _ptr(n), 0.5, _ptr(o3))
    assert np.allclose(o3, [0.0, -1.0, 0.0])
    # sign(0) = 0
    assert probe.p_sgn(0.0) == 0.0 and probe.p_sgn(-3.0) == -1.0 and probe.p_sgn(2.0) == 1.0
    # conversions truncate and saturate: u32(-2.5) = 0, u32(i32(-2.5)) = bits of -2
    u = np.zeros(2, np.uint32)
    probe.p_conv(-2.5, _ptr(u))
    assert u[0] == 0 and u[1] == np.uint32(2**32 - 2)
    probe.p_conv(5e9, _ptr(u))
    assert u[0] == 0xFFFFFFFF and u[1] == 0x7FFFFFFF
    # column-major: mat3x3f(a, b, c) * v = a v.x + b v.y + c v.z; v * M = (dot(v, a), dot(v, b), dot(v, c))
    m = _f(1, 2, 3, 4, 5, 6, 7, 8, 10)
    v = _f(1, -1, 2)
    probe.p_mv(_ptr(m), _ptr(v), _ptr(o3), 0)
    assert np.allclose(o3, m.reshape(3, 3).T @ v)
    probe.p_mv(_ptr(m), _ptr(v), _ptr(o3), 1)
    assert np.allclose(o3, m.reshape(3, 3) @ v)
    # constructor arguments left to right: s = 1 -> draw() 4, then 13
    o2 = np.zeros(2, np.float32)
    probe.p_order(_ptr(o2))
    assert list(o2) == [4.0, 13.0]
    # pow(x, 2.0) read as x * x (defined for negative x)
    assert probe.p_sq(-3.0) == 9.0
