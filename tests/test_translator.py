"""The WGSL-subset translator: WGSL semantics of the emitted C++ (compiled with g++
and run on the host), the subset's error cases, and the reference formula set."""

import json
import math
import os
import subprocess
import tempfile

import pytest

from numericdream_b200.translator import TranslateError, translate, translate_module
from numericdream_b200.translator.wgsl import TEMPLATE_CONSTS, Parser, lex

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "numericdream_b200", "csrc")

PROBES = r"""
const THIRD = 1.0 / 3.0;
const MASK = 127u;
fn r_round(x: f32) -> f32 { return round(x); }
fn r_fract(x: f32) -> f32 { return fract(x); }
fn r_i32(x: f32) -> i32 { return i32(x); }
fn r_u32(x: f32) -> u32 { return u32(x); }
fn r_sign(x: f32) -> f32 { return sign(x); }
fn r_fmod(x: f32, y: f32) -> f32 { return x % y; }
fn r_select(a: f32, b: f32, c: bool) -> f32 { return select(a, b, c); }
fn r_third() -> f32 { return THIRD; }
fn r_idiv(a: i32, b: i32) -> i32 { return a / b; }
fn r_irem(a: i32, b: i32) -> i32 { return a % b; }
fn r_shl(a: u32, s: u32) -> u32 { return a << s; }
fn r_mask(x: f32) -> u32 { return bitcast<u32>(x) & ~MASK; }
fn r_swz(v: vec3f) -> f32 { let w = v.zyx; return w.x * 100.0 + w.y * 10.0 + w.z; }
fn r_matvec(v: vec3f) -> f32 {
    let m = mat3x3f(vec3f(1.0, 2.0, 3.0), vec3f(4.0, 5.0, 6.0), vec3f(7.0, 8.0, 9.0));
    let a = m * v;
    let b = v * m;
    return a.x + 10.0 * b.x;
}
fn r_arr(k: i32) -> f32 {
    var a: array<f32, 4>;
    for (var i = 0; i < 4; i++) { a[i] = f32(i) * 2.0; }
    return a[k];
}
fn r_var_default() -> f32 { var x: vec3f; return x.x + x.y + x.z; }
fn r_abstract_mix(x: f32) -> f32 { return 2 * x + 1; }
fn r_step(e: f32, x: f32) -> f32 { return step(e, x); }
fn r_mix(a: f32, b: f32, t: f32) -> f32 { return mix(a, b, t); }
const TWO = 2;
fn r_switch(x: i32) -> f32 {
    var d: f32 = 0.5;
    switch x {
        case 1: { d = 10.0; }
        case TWO, 3: { d = 20.0; }
        case 4, default: { d = -1.0; }
    }
    switch x { case 7: { d += 100.0; } }
    return d;
}
fn r_loop(n: i32) -> i32 {
    var s = 0;
    for (var i = 0; i < n; i++) {
        if (i == 2) { continue; }
        if (i == 5) { break; }
        s += i;
    }
    return s;
}
"""

CALLS = [
    ("r_round(2.5f)", 2.0), ("r_round(3.5f)", 4.0), ("r_round(-0.5f)", -0.0), ("r_round(-2.5f)", -2.0),
    ("r_fract(-0.25f)", 0.75), ("r_i32(-2.7f)", -2), ("r_i32(1e10f)", 2147483647), ("r_i32(-1e10f)", -2147483648),
    ("r_u32(-3.0f)", 0), ("r_sign(0.0f)", 0.0), ("r_sign(-3.0f)", -1.0), ("r_fmod(-7.0f, 3.0f)", -1.0),
    ("r_fmod(7.5f, 2.0f)", 1.5), ("r_select(1.0f, 2.0f, true)", 2.0), ("r_select(1.0f, 2.0f, false)", 1.0),
    ("r_third()", float.fromhex("0x1.555556p-2")), ("r_idiv(7, 0)", 7), ("r_idiv(-7, 2)", -3), ("r_irem(-7, 2)", -1),
    ("r_irem(5, 0)", 0), ("r_shl(1u, 33u)", 2), ("r_mask(1.0f)", 0x3F800000 & ~127),
    ("r_swz(ndw::v3<float>(1, 2, 3))", 321.0), ("r_matvec(ndw::v3<float>(1, 0, 0))", 1.0 + 10 * 1.0),
    ("r_matvec(ndw::v3<float>(0, 1, 0))", 4.0 + 10 * 2.0),
    ("r_arr(3)", 6.0), ("r_arr(9)", 6.0), ("r_arr(-1)", 0.0), ("r_var_default()", 0.0), ("r_abstract_mix(1.5f)", 4.0),
    ("r_step(1.0f, 1.0f)", 1.0), ("r_step(1.0f, 0.5f)", 0.0), ("r_mix(2.0f, 4.0f, 0.25f)", 2.5), ("r_loop(10)", 8),
    ("r_switch(1)", 10.0), ("r_switch(2)", 20.0), ("r_switch(3)", 20.0), ("r_switch(4)", -1.0), ("r_switch(9)", -1.0),
    ("r_switch(7)", 99.0),
]


def _run_cpp(module_ns_cpp, calls):
    body = "\n".join(f'  std::printf("%.9g\\n", double(ndt::{c.replace("(", "<float, NoP>(", 1)}));' for c, _ in calls)
    src = ('#include <cstdio>\n#include "nd_helpers.h"\nstruct NoP { float operator[](int) const { return 0; } };\n'
           + module_ns_cpp + "\nint main() {\n" + body + "\n  return 0;\n}\n")
    with tempfile.TemporaryDirectory() as d:
        cpp = os.path.join(d, "t.cpp")
        exe = os.path.join(d, "t")
        with open(cpp, "w") as fh:
            fh.write(src)
        subprocess.run(["g++", "-std=c++17", "-O1", "-ffp-contract=off", "-I", CSRC, cpp, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    return [float(x) for x in out]


def test_wgsl_semantics_on_the_host():
    cpp = translate_module(PROBES, "ndt", contract=False)
    got = _run_cpp(cpp, CALLS)
    for (call, want), g in zip(CALLS, got):
        assert g == want or (math.isclose(g, want, rel_tol=1e-7)), (call, g, want)
        if want == 0.0 and math.copysign(1.0, want) < 0:
            assert math.copysign(1.0, g) < 0, call


@pytest.mark.parametrize("src, msg", [
    ("fn f() -> i32 { loop { break; } return 0; }", "loop"),
    ("fn f(x: i32) -> i32 { for (var i = 0; i < 2; i++) { switch x { default: { break; } } } return 0; }",
     "break inside a switch"),
    ("var<private> g: f32;", "module-scope"),
    ("struct S { a: f32 }", "struct"),
    ("fn f(x: f32) -> f32 { return nosuch(x); }", "unknown function"),
    ("fn f(x: f32) -> f32 { return y; }", "unknown identifier"),
    ("fn f(x: f32) -> f32 { let v = vec3f(1.0); return v.q; }", "swizzle"),
    ("fn f(x: f32) -> i32 { return x; }", "mismatch"),
])
def test_outside_the_subset_is_rejected(src, msg):
    with pytest.raises(TranslateError) as e:
        translate_module(src, "ndt", contract=False)
    assert msg in str(e.value)


def test_contract_is_checked():
    with pytest.raises(TranslateError):
        translate("fn de_iterations(p: Params) -> i32 { return 1; }", "x")
    bad = ("fn de_iterations(p: Params) -> i32 { return 1; }\n"
           "fn de_step(carry: IterCarry, pos: vec3f, p: Params) -> f32 { return 1.0; }\n"
           "fn de_finalize(carry: IterCarry) -> f32 { return 0.0; }\n")
    with pytest.raises(TranslateError) as e:
        translate(bad, "x")
    assert "signature" in str(e.value)


def test_legacy_params_signature_is_accepted():
    src = ("fn de_iterations(p: array<f32, 8>) -> i32 { return i32(p[0]); }\n"
           "fn de_step(carry: IterCarry, pos: vec3f, p: array<f32, 8>) -> IterCarry { return IterCarry(carry.z * p[1] + pos, carry.dr); }\n"
           "fn de_finalize(carry: IterCarry) -> f32 { return length(carry.z) / carry.dr; }\n")
    tf = translate(src, "legacy")
    assert "de_step" in tf.cpp and tf.params == []


def test_template_constants_match_the_reference_values():
    with open(os.path.join(ROOT, "tests", "golden", "template_consts.json")) as fh:
        ref = json.load(fh)
    assert set(ref) <= set(TEMPLATE_CONSTS)
    for name, text in ref.items():
        toks = lex(text)
        tok = toks[0].text
        if tok.lower().startswith("0x"):
            v = int(tok.rstrip("u"), 16)
        elif tok.endswith("u"):
            v = int(tok[:-1])
        else:
            v = float(tok) if any(ch in tok for ch in ".eE") else int(tok)
        assert TEMPLATE_CONSTS[name][0] == v, (name, TEMPLATE_CONSTS[name][0], v)


def test_generated_build_translates_the_formula_set():
    man = os.path.join(ROOT, "numericdream_b200", "_generated", "manifest.json")
    if not os.path.exists(man):
        pytest.skip("library not built")
    with open(man) as fh:
        m = json.load(fh)
    assert len(m["formulas"]) >= 54
    for n in ("mandelbrot", "amazingbox_box", "menger3_ifs", "pseudokleinian_kleinian"):
        assert n in m["formulas"]
    assert set(m["rejected"]) <= {"heightmap_primitive"}


INV_FORMULA = r"""
fn de_iterations(p: Params) -> i32 { return 4; }
fn de_step(carry: IterCarry, pos: vec3f, p: Params) -> IterCarry {
    let julia = vec3f(p[1], p[2], p[3]);
    var z = carry.z * p[0] + pos * p[4] + julia;
    z = z + carry.dr + julia;
    let w = carry.z + pos + julia;
    return IterCarry(z + w, carry.dr * 2.0);
}
fn de_finalize(carry: IterCarry) -> f32 { return length(carry.z) / carry.dr; }
"""


def test_invariant_addends_are_grouped_only_in_de_step():
    # (a + b) + c in de_step with b and c built from pos and the parameters alone is
    # emitted as ndw::add_inv(a, b, c); a sum with an iteration-dependent b is not
    cpp = translate(INV_FORMULA, "ndt_inv").cpp
    lines = [l.strip() for l in cpp.split("\n")]
    grouped = [l for l in lines if "add_inv" in l]
    assert any(l.startswith("ndw::v3<T> z = ndw::add_inv((carry.z * ndw::param(p, int32_t(0)))") for l in grouped), grouped
    assert any("const ndw::v3<T> w = ndw::add_inv(carry.z, pos, julia)" in l for l in grouped), grouped
    assert not any(l.startswith("z = ndw::add_inv") for l in grouped), grouped  # carry.dr is not invariant
    assert "add_inv" not in cpp.split("de_finalize(ndw::IterCarry<T> carry) {")[1]


def test_add_inv_keeps_the_wgsl_order_on_the_host():
    # host code (the oracle's, the op counter's) sums left to right like WGSL
    src = r"""
#include <stdio.h>
#include "nd_wgsl.h"
int main() {
  const float a = 1.0f, b = 1e-8f, c = 1e-8f;
  const ndw::v3<float> v(1.0f, 2.0f, 3.0f), u(1e-8f), w(1e-8f);
  const ndw::v3<float> r = ndw::add_inv(v, u, w);
  printf("%d %d\n", ndw::add_inv(a, b, c) == (a + b) + c, r.x == (1.0f + 1e-8f) + 1e-8f);
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        cpp = os.path.join(d, "t.cpp")
        exe = os.path.join(d, "t")
        with open(cpp, "w") as fh:
            fh.write(src)
        subprocess.run(["g++", "-std=c++17", "-O1", "-ffp-contract=off", "-I", CSRC, cpp, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    assert out == ["1", "1"]
