"""The host mirror of the reference's formula-file parser (src/app/formula.zig)."""

from numericdream_b200 import formula


def test_param_line_basic():
    p = formula.parse_param_line("// @param Scale min=-3 max=3 default=2")
    assert (p.name, p.min, p.max, p.default, p.integral) == ("Scale", -3.0, 3.0, 2.0, False)


def test_param_line_int_and_order():
    p = formula.parse_param_line("// @param Iterations int default=12 max=30 min=1")
    assert (p.name, p.min, p.max, p.default, p.integral) == ("Iterations", 1.0, 30.0, 12.0, True)


def test_param_line_name_with_spaces_keeps_inner_whitespace():
    p = formula.parse_param_line("// @param Twist A min=-180 max=180 default=90")
    assert p.name == "Twist A"
    p = formula.parse_param_line("// @param  Twist\tB  min=0")
    assert p.name == "Twist\tB"


def test_param_line_defaults_and_bad_values():
    p = formula.parse_param_line("// @param Foo min=abc default=0.25")
    assert (p.min, p.max, p.default) == (0.0, 1.0, 0.25)
    assert formula.parse_param_line("// @param min=1 max=2") is None
    assert formula.parse_param_line("no marker here") is None


def test_param_name_cut_to_23_bytes_and_f32_values():
    p = formula.parse_param_line("// @param " + "N" * 40 + " default=0.1")
    assert p.name == "N" * 23
    assert p.default == formula._f32(0.1) != 0.1


def test_parse_formula_params_caps_at_16():
    src = "\n".join(f"// @param P{i} default={i}" for i in range(20))
    ps = formula.parse_formula_params(src)
    assert len(ps) == 16 and ps[-1].name == "P15"
    packed = formula.pack_params(ps[:3])
    assert packed[:4] == [0.0, 1.0, 2.0, 0.0] and len(packed) == 16


def test_contract_check_order_and_image_directive():
    assert formula.missing_contract_fn("") .startswith("fn de_step(")
    assert formula.missing_contract_fn("fn de_step(x)").startswith("fn de_finalize(")
    assert formula.missing_contract_fn("fn de_step(x) fn de_finalize(y)").startswith("fn de_iterations(")
    assert formula.missing_contract_fn("fn de_step( fn de_finalize( fn de_iterations(") is None
    assert formula.image_directive("// @image") == "Image"
    assert formula.image_directive("// @image  Height map \r\n") == "Height map"
    assert formula.image_directive("nothing") is None


def test_builtin_params_and_source_hash():
    ps = formula.builtin_mandelbulb_params()
    assert [p.name for p in ps] == ["Power", "Iterations"] and ps[1].integral
    assert formula.source_hash("abc") == formula.source_hash(b"abc") != formula.source_hash("abd")
