"""Host-side mirror of NumericDream's formula plugin surface.

A formula plugin is one WGSL file that defines three contract functions
(``de_iterations``, ``de_step``, ``de_finalize``) plus ``// @param`` slider lines.
This module restates the reference's own parsing rules so that a formula file
behaves here exactly as it does in the reference app:

* ``parse_param_line``   follows ``src/app/formula.zig:110-146`` (parseParamLine)
* ``make_param``         follows ``src/app/formula.zig:19-33`` (makeParam, 23-char names)
* ``parse_formula_params`` follows ``src/app/formula.zig:147-157``
* ``pack_params``        follows ``src/app/formula.zig:104-108`` (16 floats, declaration order)
* ``image_directive``    follows ``src/app/formula.zig:159-168``
* ``missing_contract_fn`` follows ``src/app/formula.zig:170-181``
* ``builtin_mandelbulb_params`` follows ``src/app/formula.zig:35-40``
"""

from __future__ import annotations

import dataclasses
import struct

MAX_PARAMS = 16          # fractal_renderer.zig:47 (max_params)
MAX_NAME_LEN = 23        # CustomParam.name is [24:0]u8 (formula.zig:7), makeParam keeps 23


@dataclasses.dataclass
class CustomParam:
    """One ``@param`` slider: mirrors ``CustomParam`` (src/app/formula.zig:6-13)."""

    name: str
    min: float
    max: float
    default: float
    integral: bool = False

    @property
    def value(self) -> float:
        return self.default


def _f32(x: float) -> float:
    """Round a Python float to the nearest f32, as Zig's parseFloat(f32, ...) does."""
    return struct.unpack("<f", struct.pack("<f", x))[0]


def make_param(name: str, min_v: float, max_v: float, default: float, integral: bool) -> CustomParam:
    """src/app/formula.zig:19-33: names are cut to 23 bytes."""
    raw = name.encode("utf-8")[:MAX_NAME_LEN]
    return CustomParam(raw.decode("utf-8", errors="ignore"), _f32(min_v), _f32(max_v), _f32(default), integral)


def _parse_float(tok: str):
    """Zig std.fmt.parseFloat accepts decimal/scientific forms, inf and nan."""
    t = tok.strip()
    if not t:
        return None
    low = t.lower().lstrip("+-")
    if low in ("inf", "infinity", "nan"):
        return float(t)
    try:
        if t.lower().startswith(("0x", "-0x", "+0x")):
            return float.fromhex(t)
        return float(t)
    except ValueError:
        return None


def parse_param_line(line: str):
    """src/app/formula.zig:110-146.

    The name is every token before the first token holding ``=`` or equal to
    ``int``; then ``min=``, ``max=``, ``default=`` and a bare ``int`` are read in
    any order.  Unparseable values are skipped (defaults min 0, max 1, default 0).
    """
    marker = "@param"
    idx = line.find(marker)
    if idx < 0:
        return None
    rest = line[idx + len(marker):].strip(" \t")
    tokens = [t for t in rest.replace("\t", " ").split(" ") if t]
    name_tokens = []
    for tok in tokens:
        if "=" in tok or tok == "int":
            break
        name_tokens.append(tok)
    if not name_tokens:
        return None
    # the reference slices the original text from the start up to the end of the
    # last name token, which keeps the original inner whitespace
    last = name_tokens[-1]
    pos = 0
    for tok in name_tokens:
        pos = rest.index(tok, pos) + len(tok)
    name = rest[:pos]
    assert name.endswith(last)
    min_v, max_v, default_v, integral = 0.0, 1.0, 0.0, False
    for tok in tokens:
        if "=" not in tok:
            if tok == "int":
                integral = True
            continue
        key, val = tok.split("=", 1)
        v = _parse_float(val)
        if v is None:
            continue
        if key == "min":
            min_v = v
        elif key == "max":
            max_v = v
        elif key == "default":
            default_v = v
    return make_param(name, min_v, max_v, default_v, integral)


def parse_formula_params(content: str) -> list[CustomParam]:
    """src/app/formula.zig:147-157: at most 16 params, in file order."""
    out: list[CustomParam] = []
    for raw in content.split("\n"):
        if len(out) >= MAX_PARAMS:
            break
        line = raw.strip(" \t\r")
        p = parse_param_line(line)
        if p is not None:
            out.append(p)
    return out


def pack_params(params: list[CustomParam], values=None) -> list[float]:
    """src/app/formula.zig:104-108: p[i] = value of the i-th declared param, rest 0."""
    out = [0.0] * MAX_PARAMS
    for i, prm in enumerate(params[:MAX_PARAMS]):
        v = prm.default if values is None or i >= len(values) else values[i]
        out[i] = _f32(v)
    return out


def image_directive(content: str):
    """src/app/formula.zig:159-168."""
    marker = "@image"
    for line in content.split("\n"):
        idx = line.find(marker)
        if idx < 0:
            continue
        label = line[idx + len(marker):].strip(" \t\r")
        return label if label else "Image"
    return None


def missing_contract_fn(content: str):
    """src/app/formula.zig:170-181: the first missing contract signature, else None."""
    if "fn de_step(" not in content:
        return "fn de_step(carry: IterCarry, pos: vec3f, p: Params) -> IterCarry"
    if "fn de_finalize(" not in content:
        return "fn de_finalize(carry: IterCarry) -> f32"
    if "fn de_iterations(" not in content:
        return "fn de_iterations(p: Params) -> i32"
    return None


def builtin_mandelbulb_params() -> list[CustomParam]:
    """src/app/formula.zig:35-40: the built-in formula's two sliders."""
    return [make_param("Power", 2.0, 16.0, 8.0, False), make_param("Iterations", 2.0, 16.0, 6.0, True)]


def source_hash(source: str | bytes) -> int:
    """64-bit FNV-1a of the formula source bytes.

    The reference keys its formula code table by a 64-bit hash of the exact source
    text (``sourceHash``, fractal_renderer.zig:542-544, Wyhash).  Only the
    "same bytes -> same key" property matters for lookup, so a simpler hash with the
    same width is used; the C runtime computes the identical FNV-1a.
    """
    data = source.encode("utf-8") if isinstance(source, str) else source
    h = 0xCBF29CE484222325
    for b in data:
        h ^= b
        h = (h * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h
