"""Formula sources registered at run time (nd_formula_register with a source the build
did not compile): the library runs the build's translator and nvcc on it, as the
reference compiles an edited formula on its worker thread, loads the result and gives
it the next formula id.  Runs without a GPU (compiling and loading need none)."""

import os

import pytest

from numericdream_b200 import abi, runtime

HERE = os.path.dirname(os.path.abspath(__file__))
BAILOUT = os.path.join(HERE, "..", "numericdream_b200", "formulas", "mandelbulb_bailout.wgsl")


def edited_source():
    # the package's Mandelbulb with another default power: new bytes, so not in the build
    src = open(BAILOUT, newline="").read()
    out = src.replace("// @param Power min=2 max=16 default=8", "// @param Power min=2 max=16 default=7.5")
    assert out != src
    return out


def test_a_new_source_is_compiled_and_registered(ndlib):
    before = runtime.formula_count()
    src = edited_source()
    fid = runtime.register_formula(src)
    assert fid < runtime.formula_count() and runtime.formula_count() >= before
    assert runtime.formula_name(fid).startswith("user_")
    ps = runtime.formula_params(fid)
    assert [p.name.decode() for p in ps] == ["Power", "Iterations", "Bailout"]
    assert [p.default_value for p in ps] == [7.5, 12.0, 2.0]
    assert [bool(p.integral) for p in ps] == [False, True, False]
    # the same bytes again: found by their hash, no second compile
    assert runtime.register_formula(src) == fid
    # defaults of a view of it come from its @param table
    v = runtime.view_defaults(fid)
    assert list(v.params[:3]) == [7.5, 12.0, 2.0]


def test_translator_errors_come_back_as_compile_errors(ndlib):
    bad = edited_source().replace("let power = p[0];", "let power = p[0] +;")
    with pytest.raises(runtime.FormulaError) as e:
        runtime.register_formula(bad)
    assert e.value.status == abi.ND_ERR_COMPILE
    assert "line" in str(e.value)
    unknown = edited_source().replace("let r = length(carry.z);", "let r = no_such_helper(carry.z);")
    with pytest.raises(runtime.FormulaError) as e:
        runtime.register_formula(unknown)
    assert e.value.status == abi.ND_ERR_COMPILE and "no_such_helper" in str(e.value)


def test_the_compile_directory_is_removed(ndlib, tmp_path, monkeypatch):
    # ND_RTC_DIR holds the temporary compile directories; after a compile that failed
    # and one that succeeded (its library loaded), none is left
    monkeypatch.setenv("ND_RTC_DIR", str(tmp_path))
    bad = edited_source().replace("let power = p[0];", "let power = p[0] * ;")
    with pytest.raises(runtime.FormulaError):
        runtime.register_formula(bad)
    assert os.listdir(tmp_path) == []
    src = edited_source().replace("default=7.5", "default=7.25")
    fid = runtime.register_formula(src)
    assert runtime.formula_params(fid)[0].default_value == 7.25
    assert os.listdir(tmp_path) == []
