"""The C-ABI library loads, exports every entry point include/*.h declares, and its
struct layouts match the ctypes mirror (no compute call: runs without a GPU)."""

import ctypes as C
import glob
import os
import re

from numericdream_b200 import abi, formula, runtime

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(nd_[a-z0-9_]+)\s*\(", text, re.M):
            names.add(m.group(1))
    return names


def test_header_declares_the_abi():
    names = declared_functions()
    for must in ("nd_formula_register", "nd_formula_params", "nd_ctx_create", "nd_ctx_destroy",
                 "nd_march_forward", "nd_last_stats", "nd_autotune", "nd_graph_capture", "nd_graph_launch",
                 "nd_march_backward", "nd_march_forward_noalloc", "nd_march_forward_scenes", "nd_accel_grid",
                 "nd_scene_file_load", "nd_scene_file_lite", "nd_shade_lite", "nd_shade_lite_scenes",
                 "nd_graph_capture_scenes"):
        assert must in names


def test_library_exports_every_declared_symbol(ndlib):
    missing = [n for n in declared_functions() if not hasattr(ndlib, n)]
    assert not missing, missing


def test_struct_layouts(ndlib):
    runtime.check_layout(ndlib)
    assert C.sizeof(abi.nd_view_desc) % 8 == 0


def test_registry_has_the_benchmark_formulas(ndlib):
    names = runtime.formula_names()
    for n in ("mandelbrot", "amazingbox_box", "menger3_ifs", "pseudokleinian_kleinian"):
        assert n in names
    assert len(names) >= 50


def test_formula_params_match_the_parser(ndlib):
    from numericdream_b200 import build

    for name in ("amazingbox_box", "menger3_ifs", "pseudokleinian_kleinian", "mandelbrot"):
        path, src = build.formula_sources().get(name, (None, None)) if build.reference_root() else (None, None)
        fid = runtime.find_formula(name)
        ps = runtime.formula_params(fid)
        if src is not None:
            mine = formula.parse_formula_params(src)
            assert [p.name.decode() for p in ps] == [m.name for m in mine]
            assert [p.default_value for p in ps] == [m.default for m in mine]
            assert [bool(p.integral) for p in ps] == [m.integral for m in mine]


def test_register_rejects_bad_sources(ndlib):
    import pytest

    with pytest.raises(runtime.FormulaError) as e:
        runtime.register_formula("fn de_iterations(p: Params) -> i32 { return 1; }")
    assert "de_step" in str(e.value)
    # all three contract functions, but one names a value that does not exist: the
    # translator refuses it and its message comes back
    with pytest.raises(runtime.FormulaError) as e:
        runtime.register_formula(
            "fn de_iterations(p: Params) -> i32 { return 1; }\n"
            "fn de_step(carry: IterCarry, pos: vec3f, p: Params) -> IterCarry { return carry; }\n"
            "fn de_finalize(carry: IterCarry) -> f32 { return undefined_value; }\n")
    assert e.value.status == abi.ND_ERR_COMPILE
    assert "undefined_value" in str(e.value)


def test_register_finds_compiled_sources(ndlib):
    from numericdream_b200 import build

    if not build.reference_root():
        return
    srcs = build.formula_sources()
    path, src = srcs["menger3_ifs"]
    assert runtime.register_formula(src) == runtime.find_formula("menger3_ifs")


def test_status_strings(ndlib):
    assert ndlib.nd_status_string(0) == b"ND_OK"
    assert ndlib.nd_status_string(4) == b"ND_ERR_TIMEOUT"
    assert ndlib.nd_abi_version() == 4


def test_noalloc_rejections_carry_a_message(ndlib):
    # rejected before any CUDA call: runs without a GPU.  The message of the calling
    # thread's last failed call comes back through nd_march_forward_noalloc_stats.
    fid = runtime.find_formula("mandelbrot")
    v = abi.make_view(fid, 8, 8, (0.0, 0.0, -2.5))
    g = abi.nd_gbuffer()
    g.depth = 256  # never dereferenced: the call is rejected first
    err = C.create_string_buffer(256)
    st = abi.nd_stats()
    too_many = (abi.nd_view_desc * 65)(*([v] * 65))
    assert ndlib.nd_march_forward_noalloc(too_many, 65, None, C.byref(g), None) == abi.ND_ERR_INVALID
    ndlib.nd_march_forward_noalloc_stats(None, C.byref(st), err, 256)
    assert b"at most 64" in err.value
    g.trap = 512
    one = (abi.nd_view_desc * 1)(v)
    assert ndlib.nd_march_forward_noalloc(one, 1, None, C.byref(g), None) == abi.ND_ERR_UNSUPPORTED
    ndlib.nd_march_forward_noalloc_stats(None, C.byref(st), err, 256)
    assert b"per-ray scratch" in err.value
