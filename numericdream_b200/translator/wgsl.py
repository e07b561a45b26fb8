"""Build-time translator: the WGSL subset used by formula plugins -> C++.

NumericDream splices each formula file into its WGSL template and renames the
file's top-level names per slot (``appendRenamedFormula``,
src/gpu/fractal_renderer.zig:453-488; legacy ``p: array<f32, 8>`` is accepted as
``p: Params``, fractal_renderer.zig:435-451).  Here each formula file instead
becomes one C++ namespace of ``__host__ __device__`` function templates,
parameterised on the float type ``T`` (f32 on the GPU, f64 for the oracle, a dual
number for the adjoint) and on the parameter-vector type ``P``.  Namespacing plays
the role of the reference's ``_N`` / ``_fN`` renaming.

The pipeline is lexer -> recursive-descent parser -> type checker with WGSL's
abstract-numeric rules (abstract int/float constant expressions are folded in
double precision and converted at their first concrete use, as WGSL does) ->
C++ emitter.  Semantics kept from WGSL: ``round`` is half-to-even, ``select(f, t,
c)`` argument order, ``fract(x) = x - floor(x)``, float->int conversion truncates
and saturates, ``sign(0) = 0``, float ``%`` truncates, out-of-range indices are
clamped, ``var`` without initialiser is zero.
"""

from __future__ import annotations

import dataclasses
import math
import re
from typing import Optional

# ----------------------------------------------------------------------------
# errors


class TranslateError(Exception):
    def __init__(self, msg: str, line: int = 0):
        super().__init__(f"line {line}: {msg}" if line else msg)
        self.line = line
        self.msg = msg


# ----------------------------------------------------------------------------
# lexer

_TOKEN_RE = re.compile(
    r"""
    (?P<ws>[ \t\r\n]+)
  | (?P<comment>//[^\n]*|/\*.*?\*/)
  | (?P<num>0[xX][0-9a-fA-F]+[iu]?|(?:\d+\.\d*|\.\d+|\d+)(?:[eE][+-]?\d+)?[fhiu]?)
  | (?P<ident>[A-Za-z_][A-Za-z0-9_]*)
  | (?P<op>->|<<=|>>=|\+\+|--|&&|\|\||==|!=|<=|>=|<<|>>|\+=|-=|\*=|/=|%=|&=|\|=|\^=|[-+*/%&|^~!<>=(){}\[\];:,.@])
    """,
    re.X | re.S,
)


@dataclasses.dataclass
class Tok:
    kind: str
    text: str
    line: int


def lex(src: str) -> list[Tok]:
    out = []
    pos = 0
    line = 1
    while pos < len(src):
        m = _TOKEN_RE.match(src, pos)
        if not m:
            raise TranslateError(f"unexpected character {src[pos]!r}", line)
        kind = m.lastgroup
        text = m.group(kind)
        if kind not in ("ws", "comment"):
            out.append(Tok(kind, text, line))
        line += text.count("\n")
        pos = m.end()
    out.append(Tok("eof", "", line))
    return out


# ----------------------------------------------------------------------------
# AST


@dataclasses.dataclass
class TypeRef:          # syntactic type
    name: str
    args: list           # list of TypeRef or int/str (array length expression)
    line: int = 0


@dataclasses.dataclass
class Expr:
    line: int


@dataclasses.dataclass
class Num(Expr):
    text: str


@dataclasses.dataclass
class Ident(Expr):
    name: str


@dataclasses.dataclass
class Unary(Expr):
    op: str
    e: Expr


@dataclasses.dataclass
class Binary(Expr):
    op: str
    l: Expr
    r: Expr


@dataclasses.dataclass
class Call(Expr):
    name: str
    targs: Optional[list]   # template args for constructors/bitcast
    args: list


@dataclasses.dataclass
class Index(Expr):
    e: Expr
    idx: Expr


@dataclasses.dataclass
class Member(Expr):
    e: Expr
    name: str


@dataclasses.dataclass
class Stmt:
    line: int


@dataclasses.dataclass
class Decl(Stmt):
    kind: str            # let | var | const
    name: str
    ty: Optional[TypeRef]
    init: Optional[Expr]


@dataclasses.dataclass
class Assign(Stmt):
    lhs: Expr
    op: str
    rhs: Expr


@dataclasses.dataclass
class IncDec(Stmt):
    lhs: Expr
    op: str


@dataclasses.dataclass
class Return(Stmt):
    e: Optional[Expr]


@dataclasses.dataclass
class If(Stmt):
    cond: Expr
    then: list
    els: Optional[list]


@dataclasses.dataclass
class Switch(Stmt):
    sel: Expr
    clauses: list   # [(case expressions, has default, body)]


@dataclasses.dataclass
class For(Stmt):
    init: Optional[Stmt]
    cond: Optional[Expr]
    update: Optional[Stmt]
    body: list


@dataclasses.dataclass
class While(Stmt):
    cond: Expr
    body: list


@dataclasses.dataclass
class Break(Stmt):
    pass


@dataclasses.dataclass
class Continue(Stmt):
    pass


@dataclasses.dataclass
class ExprStmt(Stmt):
    e: Expr


@dataclasses.dataclass
class Block(Stmt):
    body: list


@dataclasses.dataclass
class FnDecl:
    name: str
    params: list          # list of (name, TypeRef)
    ret: Optional[TypeRef]
    body: list
    line: int


@dataclasses.dataclass
class ConstDecl:
    name: str
    ty: Optional[TypeRef]
    init: Expr
    line: int


# ----------------------------------------------------------------------------
# parser

_TEMPLATED = {"array", "vec2", "vec3", "vec4", "mat2x2", "mat3x3", "mat4x4", "bitcast", "ptr", "atomic"}
_ASSIGN_OPS = {"=", "+=", "-=", "*=", "/=", "%=", "&=", "|=", "^=", "<<=", ">>="}
_BINARY_LEVELS = [
    ["||"], ["&&"], ["|"], ["^"], ["&"], ["==", "!="], ["<", ">", "<=", ">="], ["<<", ">>"],
    ["+", "-"], ["*", "/", "%"],
]


class Parser:
    def __init__(self, toks: list[Tok]):
        self.t = toks
        self.i = 0
        self.pending_gt = 0   # a split '>>' closing two template lists

    # helpers
    def peek(self, k=0) -> Tok:
        return self.t[min(self.i + k, len(self.t) - 1)]

    def at(self, text: str) -> bool:
        return self.peek().text == text and self.peek().kind != "eof"

    def eat(self, text: str) -> bool:
        if self.at(text):
            self.i += 1
            return True
        return False

    def expect(self, text: str) -> Tok:
        tok = self.peek()
        if tok.text != text:
            raise TranslateError(f"expected {text!r}, found {tok.text!r}", tok.line)
        self.i += 1
        return tok

    def ident(self) -> str:
        tok = self.peek()
        if tok.kind != "ident":
            raise TranslateError(f"expected identifier, found {tok.text!r}", tok.line)
        self.i += 1
        return tok.text

    def close_template(self):
        if self.pending_gt:
            self.pending_gt -= 1
            return
        tok = self.peek()
        if tok.text == ">":
            self.i += 1
        elif tok.text == ">>":
            self.i += 1
            self.pending_gt += 1
        else:
            raise TranslateError(f"expected '>', found {tok.text!r}", tok.line)

    # module
    def module(self):
        fns, consts = [], []
        while self.peek().kind != "eof":
            tok = self.peek()
            if tok.text == "@":
                raise TranslateError("attributes are not supported in formula files", tok.line)
            if tok.text == "fn":
                fns.append(self.fn_decl())
            elif tok.text == "const":
                self.i += 1
                name = self.ident()
                ty = self.type_ref() if self.eat(":") else None
                self.expect("=")
                init = self.expr()
                self.expect(";")
                consts.append(ConstDecl(name, ty, init, tok.line))
            elif tok.text == ";":
                self.i += 1
            elif tok.text in ("struct", "var", "override", "alias"):
                raise TranslateError(f"module-scope '{tok.text}' is not in the supported subset", tok.line)
            else:
                raise TranslateError(f"unexpected {tok.text!r} at module scope", tok.line)
        return fns, consts

    def type_ref(self) -> TypeRef:
        tok = self.peek()
        name = self.ident()
        args = []
        if name in _TEMPLATED and self.at("<"):
            self.i += 1
            while True:
                if name == "array" and args:
                    e = self.expr_noncomparison()
                    args.append(e)
                else:
                    args.append(self.type_ref())
                if self.pending_gt:
                    break
                if self.eat(","):
                    continue
                break
            self.close_template()
        return TypeRef(name, args, tok.line)

    def fn_decl(self) -> FnDecl:
        line = self.expect("fn").line
        name = self.ident()
        self.expect("(")
        params = []
        while not self.at(")"):
            pname = self.ident()
            self.expect(":")
            params.append((pname, self.type_ref()))
            if not self.eat(","):
                break
        self.expect(")")
        ret = self.type_ref() if self.eat("->") else None
        body = self.block()
        return FnDecl(name, params, ret, body, line)

    def block(self) -> list:
        self.expect("{")
        out = []
        while not self.at("}"):
            if self.peek().kind == "eof":
                raise TranslateError("unterminated block", self.peek().line)
            s = self.statement()
            if s is not None:
                out.append(s)
        self.expect("}")
        return out

    def statement(self):
        tok = self.peek()
        t = tok.text
        if t == ";":
            self.i += 1
            return None
        if t == "{":
            return Block(tok.line, self.block())
        if t in ("let", "var", "const"):
            s = self.decl()
            self.expect(";")
            return s
        if t == "return":
            self.i += 1
            e = None if self.at(";") else self.expr()
            self.expect(";")
            return Return(tok.line, e)
        if t == "if":
            return self.if_stmt()
        if t == "for":
            self.i += 1
            self.expect("(")
            init = None if self.at(";") else self.simple_stmt()
            self.expect(";")
            cond = None if self.at(";") else self.expr()
            self.expect(";")
            update = None if self.at(")") else self.simple_stmt()
            self.expect(")")
            return For(tok.line, init, cond, update, self.block())
        if t == "while":
            self.i += 1
            cond = self.expr()
            return While(tok.line, cond, self.block())
        if t == "break":
            self.i += 1
            self.expect(";")
            return Break(tok.line)
        if t == "continue":
            self.i += 1
            self.expect(";")
            return Continue(tok.line)
        if t == "switch":
            return self.switch_stmt()
        if t in ("loop", "discard"):
            raise TranslateError(f"'{t}' is not in the supported subset", tok.line)
        s = self.simple_stmt()
        self.expect(";")
        return s

    def decl(self):
        tok = self.peek()
        kind = tok.text
        self.i += 1
        if kind == "var" and self.at("<"):
            raise TranslateError("address-space vars are not supported", tok.line)
        name = self.ident()
        ty = self.type_ref() if self.eat(":") else None
        init = self.expr() if self.eat("=") else None
        if init is None and kind != "var":
            raise TranslateError(f"'{kind}' needs an initialiser", tok.line)
        return Decl(tok.line, kind, name, ty, init)

    def simple_stmt(self):
        tok = self.peek()
        if tok.text in ("let", "var", "const"):
            return self.decl()
        if tok.text == "_" and self.peek(1).text == "=":
            self.i += 2
            return ExprStmt(tok.line, self.expr())
        e = self.expr()
        nt = self.peek().text
        if nt in _ASSIGN_OPS:
            self.i += 1
            return Assign(tok.line, e, nt, self.expr())
        if nt in ("++", "--"):
            self.i += 1
            return IncDec(tok.line, e, nt)
        return ExprStmt(tok.line, e)

    def switch_stmt(self):
        # switch sel { case a, b: { ... } case c, default: { ... } default: { ... } }
        line = self.expect("switch").line
        sel = self.expr()
        self.expect("{")
        clauses = []
        while not self.eat("}"):
            cases, dflt = [], False
            if self.eat("default"):
                dflt = True
            else:
                self.expect("case")
                while True:
                    if self.eat("default"):
                        dflt = True
                    else:
                        cases.append(self.expr())
                    if not self.eat(","):
                        break
                    if self.at(":") or self.at("{"):
                        break
            self.eat(":")
            clauses.append((cases, dflt, self.block()))
        return Switch(line, sel, clauses)

    def if_stmt(self):
        line = self.expect("if").line
        cond = self.expr()
        then = self.block()
        els = None
        if self.eat("else"):
            if self.at("if"):
                els = [self.if_stmt()]
            else:
                els = self.block()
        return If(line, cond, then, els)

    # expressions
    def expr(self):
        return self.binary(0)

    def expr_noncomparison(self):
        # array length inside a template list: stop before '>'
        return self.binary(7)

    def binary(self, level):
        if level >= len(_BINARY_LEVELS):
            return self.unary()
        left = self.binary(level + 1)
        while True:
            tok = self.peek()
            if tok.kind == "op" and tok.text in _BINARY_LEVELS[level]:
                self.i += 1
                right = self.binary(level + 1)
                left = Binary(tok.line, tok.text, left, right)
            else:
                return left

    def unary(self):
        tok = self.peek()
        if tok.kind == "op" and tok.text in ("-", "!", "~"):
            self.i += 1
            return Unary(tok.line, tok.text, self.unary())
        if tok.kind == "op" and tok.text in ("&", "*"):
            raise TranslateError("pointers are not in the supported subset", tok.line)
        return self.postfix(self.primary())

    def postfix(self, e):
        while True:
            tok = self.peek()
            if tok.text == "[":
                self.i += 1
                idx = self.expr()
                self.expect("]")
                e = Index(tok.line, e, idx)
            elif tok.text == ".":
                self.i += 1
                e = Member(tok.line, e, self.ident())
            else:
                return e

    def primary(self):
        tok = self.peek()
        if tok.kind == "num":
            self.i += 1
            return Num(tok.line, tok.text)
        if tok.text == "(":
            self.i += 1
            e = self.expr()
            self.expect(")")
            return e
        if tok.kind == "ident":
            if tok.text in ("true", "false"):
                self.i += 1
                return Num(tok.line, tok.text)
            name = tok.text
            self.i += 1
            targs = None
            if name in _TEMPLATED and self.at("<"):
                self.i -= 1
                tr = self.type_ref()
                targs = tr.args
            if self.at("("):
                self.i += 1
                args = []
                while not self.at(")"):
                    args.append(self.expr())
                    if not self.eat(","):
                        break
                self.expect(")")
                return Call(tok.line, name, targs, args)
            if targs is not None:
                raise TranslateError(f"template type {name} used as a value", tok.line)
            return Ident(tok.line, name)
        raise TranslateError(f"unexpected {tok.text!r}", tok.line)


# ----------------------------------------------------------------------------
# types


@dataclasses.dataclass(frozen=True)
class Ty:
    kind: str                 # 's' scalar | 'v' vector | 'm' matrix | 'a' array | 'st' struct | 'params' | 'void'
    scalar: str = ""          # f32 i32 u32 bool AInt AFloat
    n: int = 0                # vector size / matrix columns / array length
    r: int = 0                # matrix rows
    elem: Optional["Ty"] = None
    name: str = ""

    def __str__(self):
        if self.kind == "s":
            return self.scalar
        if self.kind == "v":
            return f"vec{self.n}<{self.scalar}>"
        if self.kind == "m":
            return f"mat{self.n}x{self.r}f"
        if self.kind == "a":
            return f"array<{self.elem},{self.n}>"
        if self.kind == "st":
            return self.name
        return self.kind


def S(s):
    return Ty("s", s)


def V(n, s):
    return Ty("v", s, n)


def M(c, r):
    return Ty("m", "f32", c, r)


F32, I32, U32, BOOL, AINT, AFLOAT = S("f32"), S("i32"), S("u32"), S("bool"), S("AInt"), S("AFloat")
VOID = Ty("void")
PARAMS = Ty("params")
CARRY = Ty("st", name="IterCarry")
IMAGE_INFO = Ty("st", name="ImageInfo")
IMAGE_SAMPLE = Ty("st", name="ImageSample")
# struct types a formula may use: its carry, and the image sampler's records
# (ImageInfo / ImageSample, template.wgsl:1142-1162)
STRUCT_FIELDS = {"IterCarry": {"z": V(3, "f32"), "dr": F32},
                 "ImageInfo": {"base": U32, "size": V(2, "u32"), "slope": V(4, "f32")},
                 "ImageSample": {"value": V(4, "f32"), "near": V(4, "f32"), "far": V(4, "f32")}}

_SHORT_TYPES = {
    "f32": F32, "i32": I32, "u32": U32, "bool": BOOL,
    "vec2f": V(2, "f32"), "vec3f": V(3, "f32"), "vec4f": V(4, "f32"),
    "vec2i": V(2, "i32"), "vec3i": V(3, "i32"), "vec4i": V(4, "i32"),
    "vec2u": V(2, "u32"), "vec3u": V(3, "u32"), "vec4u": V(4, "u32"),
    "mat2x2f": M(2, 2), "mat3x3f": M(3, 3), "mat4x4f": M(4, 4),
    "IterCarry": CARRY, "Params": PARAMS, "ImageInfo": IMAGE_INFO, "ImageSample": IMAGE_SAMPLE,
}

_CPP_SCALAR = {"f32": "T", "i32": "int32_t", "u32": "uint32_t", "bool": "bool"}


def cpp_type(t: Ty) -> str:
    if t.kind == "s":
        return _CPP_SCALAR[t.scalar]
    if t.kind == "v":
        return f"ndw::v{t.n}<{_CPP_SCALAR[t.scalar]}>"
    if t.kind == "m":
        return f"ndw::m{t.n}<T>"
    if t.kind == "a":
        return f"ndw::arr<{cpp_type(t.elem)}, {t.n}>"
    if t.kind == "st":
        return f"ndw::{t.name}<T>"
    if t.kind == "params":
        return "P"
    if t.kind == "void":
        return "void"
    raise TranslateError(f"no C++ type for {t}")


def is_abstract(t: Ty) -> bool:
    return t.kind == "s" and t.scalar in ("AInt", "AFloat")


def is_float_scalar_name(s: str) -> bool:
    return s in ("f32", "AFloat")


def concretize(t: Ty) -> Ty:
    if t == AINT:
        return I32
    if t == AFLOAT:
        return F32
    return t


# ----------------------------------------------------------------------------
# the template-library surface formulas may call (src/gpu/shaders/template.wgsl)

# Constants from template.wgsl:57-90 visible to formula code (value, abstract kind
# or concrete type).  These numbers are part of the plugin interface: a formula
# that names PI or EPSILON_FINE must see the same value it sees in the reference.
TEMPLATE_CONSTS = {
    "PI": (3.14159265, AFLOAT),
    "TAU": (6.28318530718, AFLOAT),
    "SQRT3": (1.7320508, AFLOAT),
    "HALF_SQRT3": (0.8660254, AFLOAT),
    "GOLDEN_RATIO_FRACT": (0.61803399, AFLOAT),
    "INFINITE_DISTANCE": (1e30, AFLOAT),
    "NO_SURFACE_DE": (1e6, AFLOAT),
    "EPSILON": (1e-4, AFLOAT),
    "EPSILON_FINE": (1e-6, AFLOAT),
    "EPSILON_TINY": (1e-12, AFLOAT),
    "UNORM8_MAX": (255.0, AFLOAT),
    "CUBE_CORNERS": (8, AINT),
    "MAX_PARAMS": (16, AINT),
    "U32_MAX": (0xFFFFFFFF, U32),
    "U32_SIGN_BIT": (0x80000000, U32),
    "U32_RANGE": (4294967296.0, AFLOAT),
    "INV_U32_RANGE": (2.3283064365386963e-10, AFLOAT),
    "PCG_MULTIPLIER": (747796405, U32),
    "PCG_INCREMENT": (2891336453, U32),
    "PCG_OUTPUT_MULTIPLIER": (277803737, U32),
    "LCG_MULTIPLIER": (1664525, U32),
    "LCG_INCREMENT": (1013904223, U32),
    "KNUTH_MULTIPLIER": (2654435761, U32),
    "GOLDEN_RATIO_U32": (0x9E3779B9, U32),
    "GOLDEN_RATIO_U16": (40503, U32),
    "SPATIAL_PRIME_X": (73856093, U32),
    "SPATIAL_PRIME_Y": (19349663, U32),
    "SPATIAL_PRIME_Z": (83492791, U32),
    "BULB_BAILOUT": (2.0, AFLOAT),
    "SMOOTH_K_MIN": (0.0001, AFLOAT),
    "IMAGE_SLOPE_RADIUS_NEAR": (8.0, AFLOAT),   # tpl:1124-1125
    "IMAGE_SLOPE_RADIUS_FAR": (64.0, AFLOAT),
}

V3F, V4F, V2F = V(3, "f32"), V(4, "f32"), V(2, "f32")

# Helper functions of the DE library (template.wgsl:945-1109, 1394-1408, 1653-1706)
# with their WGSL signatures; they are implemented by hand in nd_helpers.h.
TEMPLATE_FUNCS = {
    "box_fold": ([V3F, F32], V3F),
    "sphere_fold": ([V3F, F32, F32, F32], V4F),
    "sphere_invert_offset": ([V3F, F32, V3F, F32], V4F),
    "lattice_wrap": ([V3F, F32], V3F),
    "de_finalize_scaled": ([CARRY], F32),
    "de_finalize_plain": ([CARRY], F32),
    "bulb_log_escape": ([CARRY], F32),
    "bulb_power_step": ([CARRY, V3F, F32], CARRY),
    "sort_desc_abs": ([V3F], V3F),
    "tetra_fold": ([V3F], V3F),
    "wrap_angle": ([F32, F32], F32),
    "rotate_xyz_deg": ([V3F, V3F], V3F),
    "primitive_de_iterations": ([], I32),
    "primitive_de_step": ([CARRY, F32], CARRY),
    "rot_x": ([F32], M(3, 3)),
    "rot_y": ([F32], M(3, 3)),
    "rot_z": ([F32], M(3, 3)),
    "smin": ([F32, F32, F32], F32),
    "smax": ([F32, F32, F32], F32),
    "ssub": ([F32, F32, F32], F32),
    "smin_lin": ([F32, F32, F32], F32),
    "smin_nlin": ([F32, F32, F32], F32),
    "smix": ([F32, F32, F32], F32),
}

_FLOAT_UNARY = {"sin", "cos", "tan", "asin", "acos", "atan", "sinh", "cosh", "tanh", "exp", "exp2",
                "log", "log2", "sqrt", "inverseSqrt", "floor", "ceil", "round", "fract", "trunc",
                "radians", "degrees", "saturate"}
_NUM_UNARY = {"abs", "sign"}
_NUM_BINARY = {"min", "max"}
_FLOAT_BINARY = {"pow", "atan2", "step"}

_CPP_RESERVED = {
    "alignas", "alignof", "and", "asm", "auto", "bitand", "bitor", "case", "catch", "char", "class",
    "compl", "concept", "constexpr", "const_cast", "decltype", "default", "delete", "do", "double",
    "dynamic_cast", "enum", "explicit", "export", "extern", "float", "friend", "goto", "inline",
    "int", "long", "mutable", "namespace", "new", "noexcept", "not", "nullptr", "operator", "or",
    "private", "protected", "public", "register", "reinterpret_cast", "requires", "short",
    "signed", "sizeof", "static", "static_assert", "static_cast", "struct", "switch", "template",
    "this", "thread_local", "throw", "try", "typedef", "typeid", "typename", "union", "unsigned",
    "using", "virtual", "void", "volatile", "wchar_t", "xor", "T", "P", "ndw", "std", "near", "far",
    "min", "max", "abs", "sin", "cos", "exp", "log", "pow", "sqrt", "floor", "round", "sign", "dot",
    "length", "cross", "mix", "clamp", "select", "normalize", "fract", "step", "atan2", "acos",
    "tan", "atan", "asin", "ceil", "trunc", "log2", "exp2", "assert", "errno",
}


def cpp_name(name: str) -> str:
    if name in _CPP_RESERVED or name.startswith("__"):
        return name + "_w"
    return name


def _fmt_float(v: float) -> str:
    if math.isinf(v):
        return "(1.0/0.0)" if v > 0 else "(-1.0/0.0)"
    if math.isnan(v):
        return "(0.0/0.0)"
    r = repr(float(v))
    if "e" not in r and "." not in r and "inf" not in r:
        r += ".0"
    return r


# ----------------------------------------------------------------------------
# typed expression


@dataclasses.dataclass
class TE:
    ty: Ty
    code: str
    const: object = None       # folded Python value for abstract/const expressions
    lvalue: bool = False
    inv: bool = False          # de_step: the same in every iteration (no carry in it)


def _wrap_trunc_div(a: int, b: int) -> int:
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


class FormulaCompiler:
    """Type-checks one formula module and emits its C++ namespace."""

    def __init__(self, fns: list[FnDecl], consts: list[ConstDecl], ns: str, helper_ns: str = "ndw"):
        self.helper_ns = helper_ns
        self.fns = {f.name: f for f in fns}
        self.fn_order = [f.name for f in fns]
        self.module_consts_src = {c.name: c for c in consts}
        self.module_consts: dict[str, TE] = {}
        self.ns = ns
        self.scopes: list[dict] = []
        self.fn_sigs: dict[str, tuple] = {}
        self.cur_ret: Ty = VOID
        self.features: set[str] = set()
        self.calls: dict[str, set] = {}
        self.cur_fn = ""
        self.inv_fn = False  # translating de_step: track what is the same in every iteration
        for f in fns:
            if f.name in self.fn_sigs:
                raise TranslateError(f"function {f.name} defined twice", f.line)
            ptys = [(pn, self.resolve_type(pt)) for pn, pt in f.params]
            rty = self.resolve_type(f.ret) if f.ret else VOID
            self.fn_sigs[f.name] = (ptys, rty)

    # ---- type resolution
    def resolve_type(self, tr: TypeRef) -> Ty:
        if tr.name in _SHORT_TYPES and not tr.args:
            return _SHORT_TYPES[tr.name]
        if tr.name in ("vec2", "vec3", "vec4") and tr.args:
            st = self.resolve_type(tr.args[0])
            return V(int(tr.name[3]), st.scalar)
        if tr.name in ("mat2x2", "mat3x3", "mat4x4") and tr.args:
            return M(int(tr.name[3]), int(tr.name[5]))
        if tr.name == "array":
            if len(tr.args) != 2:
                raise TranslateError("runtime-sized arrays are not supported", tr.line)
            elem = self.resolve_type(tr.args[0])
            if elem == F32 and isinstance(tr.args[1], Num) and tr.args[1].text == "8":
                # legacy `p: array<f32, 8>` (fractal_renderer.zig:435-451) is read as Params
                return Ty("a", "", 8, elem=elem)
            n = self.const_int(tr.args[1])
            return Ty("a", "", n, elem=elem)
        raise TranslateError(f"unsupported type {tr.name}", tr.line)

    def const_int(self, e: Expr) -> int:
        te = self.expr(e)
        if te.const is None or not isinstance(te.const, int):
            raise TranslateError("array length must be a constant integer", e.line)
        return int(te.const)

    # ---- scopes
    def push(self):
        self.scopes.append({})

    def pop(self):
        self.scopes.pop()

    def declare(self, name: str, te: TE, line: int):
        if name in self.scopes[-1]:
            raise TranslateError(f"'{name}' redeclared in the same scope", line)
        self.scopes[-1][name] = te

    def lookup(self, name: str, line: int) -> TE:
        for sc in reversed(self.scopes):
            if name in sc:
                return sc[name]
        if name in self.module_consts:
            return self.module_consts[name]
        if name in self.module_consts_src:
            return self.eval_module_const(name)
        if name in TEMPLATE_CONSTS:
            v, t = TEMPLATE_CONSTS[name]
            return self.literal_te(v, t)
        raise TranslateError(f"unknown identifier '{name}'", line)

    def eval_module_const(self, name: str) -> TE:
        c = self.module_consts_src[name]
        if name in getattr(self, "_evaluating", set()):
            raise TranslateError(f"const '{name}' refers to itself", c.line)
        self._evaluating = getattr(self, "_evaluating", set()) | {name}
        saved = self.scopes
        self.scopes = []
        te = self.expr(c.init)
        if c.ty is not None:
            te = self.convert(te, self.resolve_type(c.ty), c.line)
        self.scopes = saved
        self._evaluating.discard(name)
        te = TE(te.ty, f"({te.code})" if te.const is None else te.code, te.const)
        self.module_consts[name] = te
        return te

    # ---- literal helpers
    def literal_te(self, v, t: Ty) -> TE:
        if t == AINT:
            return TE(AINT, str(int(v)), int(v))
        if t == AFLOAT:
            return TE(AFLOAT, _fmt_float(v), float(v))
        if t == U32:
            return TE(U32, f"{int(v) & 0xFFFFFFFF}u", int(v) & 0xFFFFFFFF)
        if t == I32:
            return TE(I32, f"int32_t({int(v)})", int(v))
        if t == F32:
            return TE(F32, f"T({_fmt_float(v)})", float(v))
        if t == BOOL:
            return TE(BOOL, "true" if v else "false", bool(v))
        raise TranslateError(f"bad literal type {t}")

    def num(self, e: Num) -> TE:
        s = e.text
        if s in ("true", "false"):
            return TE(BOOL, s, s == "true")
        if s.lower().startswith("0x"):
            suf = s[-1] if s[-1] in "iu" else ""
            v = int(s[:-1] if suf else s, 16)
            return self.literal_te(v, {"": AINT, "i": I32, "u": U32}[suf])
        suf = s[-1] if s[-1] in "fhiu" else ""
        body = s[:-1] if suf else s
        if suf == "h":
            raise TranslateError("f16 literals are not supported", e.line)
        is_float = suf == "f" or any(c in body for c in ".eE")
        if suf in ("i", "u"):
            return self.literal_te(int(body), I32 if suf == "i" else U32)
        if is_float:
            return self.literal_te(float(body), F32 if suf == "f" else AFLOAT)
        return self.literal_te(int(body), AINT)

    # ---- conversion
    def convert(self, te: TE, target: Ty, line: int) -> TE:
        if te.ty == target:
            return te
        if target.kind == "params" and te.ty.kind == "params":
            return te
        if is_abstract(te.ty):
            if target.kind == "s":
                return self._abstract_to_scalar(te, target.scalar, line)
            raise TranslateError(f"cannot convert {te.ty} to {target}", line)
        if (te.ty.kind == "a" and target.kind == "a" and te.ty.n == target.n
                and te.ty.elem == target.elem):
            return te
        raise TranslateError(f"type mismatch: {te.ty} where {target} is expected", line)

    def _abstract_to_scalar(self, te: TE, scalar: str, line: int) -> TE:
        v = te.const
        if v is None:
            raise TranslateError("abstract value without a constant", line)
        if scalar == "f32":
            return TE(F32, f"T({_fmt_float(float(v))})", float(v))
        if scalar == "AFloat":
            return TE(AFLOAT, _fmt_float(float(v)), float(v))
        if scalar == "i32":
            if te.ty == AFLOAT:
                raise TranslateError("abstract float used where i32 is expected", line)
            return TE(I32, f"int32_t({int(v)})", int(v))
        if scalar == "u32":
            if te.ty == AFLOAT or int(v) < 0:
                raise TranslateError("value not representable as u32", line)
            return TE(U32, f"{int(v)}u", int(v))
        if scalar == "bool":
            raise TranslateError("number used as bool", line)
        raise TranslateError(f"cannot convert abstract to {scalar}", line)

    def unify_scalars(self, tes: list[TE], line: int, default="f32") -> list[TE]:
        """Apply WGSL's automatic conversion of abstract operands to a common type."""
        concrete = None
        for te in tes:
            s = te.ty.scalar if te.ty.kind in ("s", "v") else ("f32" if te.ty.kind == "m" else None)
            if s is None:
                continue
            if s not in ("AInt", "AFloat"):
                if concrete is not None and concrete != s:
                    raise TranslateError(f"mixed operand types {concrete} and {s}", line)
                concrete = s
        if concrete is None:
            kinds = {te.ty.scalar for te in tes if te.ty.kind == "s"}
            if "AFloat" in kinds:
                return [self._abstract_to_scalar(te, "AFloat", line) if te.ty == AINT else te for te in tes]
            return tes
        out = []
        for te in tes:
            if is_abstract(te.ty):
                out.append(self._abstract_to_scalar(te, concrete, line))
            else:
                out.append(te)
        return out

    # ---- expressions
    def expr(self, e: Expr) -> TE:
        m = getattr(self, "e_" + type(e).__name__)
        return m(e)

    def e_Num(self, e):
        return self.num(e)

    def e_Ident(self, e):
        te = self.lookup(e.name, e.line)
        return te

    def e_Unary(self, e):
        a = self.expr(e.e)
        if e.op == "-":
            if a.const is not None and is_abstract(a.ty):
                return self.literal_te(-a.const, a.ty)
            if a.ty.kind in ("s", "v", "m") and a.ty.scalar != "bool":
                c = None if a.const is None or not isinstance(a.const, (int, float)) else -a.const
                if a.ty == F32 and c is not None:
                    return TE(F32, f"T({_fmt_float(c)})", c)
                return TE(a.ty, f"(-{a.code})", None)
            raise TranslateError(f"unary - on {a.ty}", e.line)
        if e.op == "!":
            if a.ty == BOOL:
                return TE(BOOL, f"(!{a.code})")
            if a.ty.kind == "v" and a.ty.scalar == "bool":
                return TE(a.ty, f"ndw::vnot({a.code})")
            raise TranslateError(f"! on {a.ty}", e.line)
        if e.op == "~":
            if a.ty in (AINT,) and a.const is not None:
                return self.literal_te(~a.const, AINT)
            if a.ty == U32 and a.const is not None:
                return self.literal_te((~a.const) & 0xFFFFFFFF, U32)
            if a.ty.scalar in ("i32", "u32"):
                return TE(a.ty, f"(~{a.code})")
            raise TranslateError(f"~ on {a.ty}", e.line)
        raise TranslateError(f"unary {e.op}", e.line)

    def _fold(self, op, a, b, kind, line):
        if kind == "AInt":
            if op == "+":
                return a + b
            if op == "-":
                return a - b
            if op == "*":
                return a * b
            if op == "/":
                if b == 0:
                    raise TranslateError("constant division by zero", line)
                return _wrap_trunc_div(a, b)
            if op == "%":
                if b == 0:
                    raise TranslateError("constant division by zero", line)
                return a - b * _wrap_trunc_div(a, b)
            if op == "<<":
                return a << b
            if op == ">>":
                return a >> b
            if op == "&":
                return a & b
            if op == "|":
                return a | b
            if op == "^":
                return a ^ b
        else:
            a, b = float(a), float(b)
            if op == "+":
                return a + b
            if op == "-":
                return a - b
            if op == "*":
                return a * b
            if op == "/":
                return a / b if b != 0 else (math.copysign(math.inf, a) if a else math.nan)
            if op == "%":
                return math.fmod(a, b)
        return None

    def e_Binary(self, e):
        te = self._e_binary(e)
        # (a + b) + c in de_step with b and c the same in every iteration and a not:
        # ndw::add_inv lets the FP32 DE on the device add b + c first, so that it is
        # computed once per evaluation instead of once per iteration
        if (e.op == "+" and self.inv_fn and isinstance(e.l, Binary) and e.l.op == "+" and
                te.ty.kind in ("s", "v") and te.ty.scalar == "f32" and
                self.is_inv(e.r) and self.is_inv(e.l.r) and not self.is_inv(e.l.l)):
            x, y, z = self.expr(e.l.l), self.expr(e.l.r), self.expr(e.r)
            if all(not is_abstract(t.ty) and t.ty.kind in ("s", "v") and t.ty.scalar == "f32" for t in (x, y, z)):
                return TE(te.ty, f"ndw::add_inv({x.code}, {y.code}, {z.code})")
        return te

    def _e_binary(self, e):
        op = e.op
        a = self.expr(e.l)
        b = self.expr(e.r)
        if op in ("&&", "||"):
            if a.ty != BOOL or b.ty != BOOL:
                raise TranslateError(f"{op} needs bool operands", e.line)
            return TE(BOOL, f"({a.code} {op} {b.code})")
        # abstract constant folding
        if is_abstract(a.ty) and is_abstract(b.ty) and a.const is not None and b.const is not None:
            if op in ("==", "!=", "<", ">", "<=", ">="):
                r = {"==": a.const == b.const, "!=": a.const != b.const, "<": a.const < b.const,
                     ">": a.const > b.const, "<=": a.const <= b.const, ">=": a.const >= b.const}[op]
                return TE(BOOL, "true" if r else "false", r)
            kind = "AInt" if a.ty == AINT and b.ty == AINT else "AFloat"
            v = self._fold(op, a.const, b.const, kind, e.line)
            if v is not None:
                return self.literal_te(v, AINT if kind == "AInt" else AFLOAT)
        if op in ("<<", ">>"):
            if is_abstract(a.ty):
                a = self._abstract_to_scalar(a, "i32", e.line)
            sh_scalar = "u32"
            if b.ty.kind == "s" and is_abstract(b.ty):
                b = self._abstract_to_scalar(b, sh_scalar, e.line)
            if a.ty.scalar not in ("i32", "u32") or b.ty.scalar != "u32":
                raise TranslateError(f"shift of {a.ty} by {b.ty}", e.line)
            if a.ty.kind == "v":
                if b.ty.kind != "v":
                    raise TranslateError("vector shift needs a vector shift amount", e.line)
            return TE(a.ty, f"ndw::sh{'l' if op == '<<' else 'r'}({a.code}, {b.code})")
        a, b = self.unify_scalars([a, b], e.line)
        ta, tb = a.ty, b.ty
        if op in ("==", "!=", "<", ">", "<=", ">="):
            if ta != tb:
                raise TranslateError(f"comparison of {ta} and {tb}", e.line)
            if ta.kind == "s":
                return TE(BOOL, f"({a.code} {op} {b.code})")
            if ta.kind == "v":
                fn = {"==": "veq", "!=": "vne", "<": "vlt", ">": "vgt", "<=": "vle", ">=": "vge"}[op]
                return TE(V(ta.n, "bool"), f"ndw::{fn}({a.code}, {b.code})")
            raise TranslateError(f"comparison of {ta}", e.line)
        if op in ("&", "|", "^"):
            if ta != tb or ta.scalar not in ("i32", "u32", "bool"):
                raise TranslateError(f"bitwise {op} on {ta}, {tb}", e.line)
            if ta.kind == "s" and ta.scalar == "bool":
                return TE(BOOL, f"bool({a.code} {op} {b.code})")
            return TE(ta, f"({a.code} {op} {b.code})")
        if op in ("+", "-", "*", "/", "%"):
            # matrices
            if ta.kind == "m" or tb.kind == "m":
                if op == "*" and ta.kind == "m" and tb.kind == "v":
                    if tb.n != ta.n:
                        raise TranslateError("matrix * vector size mismatch", e.line)
                    return TE(V(ta.r, "f32"), f"ndw::mul({a.code}, {b.code})")
                if op == "*" and ta.kind == "v" and tb.kind == "m":
                    return TE(V(tb.n, "f32"), f"ndw::mul({a.code}, {b.code})")
                if op == "*" and ta.kind == "m" and tb.kind == "m":
                    return TE(M(tb.n, ta.r), f"ndw::mul({a.code}, {b.code})")
                if op in ("*", "/") and ta.kind == "m" and tb.kind == "s":
                    if op == "/":
                        raise TranslateError("matrix / scalar is not WGSL", e.line)
                    return TE(ta, f"({a.code} * {b.code})")
                if op == "*" and ta.kind == "s" and tb.kind == "m":
                    return TE(tb, f"({b.code} * {a.code})")
                if op in ("+", "-") and ta == tb:
                    return TE(ta, f"({a.code} {op} {b.code})")
                raise TranslateError(f"unsupported matrix operation {ta} {op} {tb}", e.line)
            if ta.kind not in ("s", "v") or tb.kind not in ("s", "v"):
                raise TranslateError(f"arithmetic on {ta}, {tb}", e.line)
            if ta.scalar == "bool" or tb.scalar == "bool":
                raise TranslateError("arithmetic on bool", e.line)
            if ta.kind == "v" and tb.kind == "v" and ta != tb:
                raise TranslateError(f"vector size mismatch {ta} {tb}", e.line)
            rty = ta if ta.kind == "v" else tb
            if op == "%" and rty.scalar == "f32":
                return TE(rty, f"ndw::fmod_trunc({a.code}, {b.code})")
            if op in ("/", "%") and rty.scalar in ("i32", "u32"):
                fn = "idiv" if op == "/" else "irem"
                return TE(rty, f"ndw::{fn}({a.code}, {b.code})")
            return TE(rty, f"({a.code} {op} {b.code})")
        raise TranslateError(f"operator {op}", e.line)

    def e_Index(self, e):
        base = self.expr(e.e)
        idx = self.expr(e.idx)
        if is_abstract(idx.ty):
            idx = self._abstract_to_scalar(idx, "i32", e.line)
        if idx.ty.kind != "s" or idx.ty.scalar not in ("i32", "u32"):
            raise TranslateError("index must be an integer", e.line)
        bt = base.ty
        if bt.kind == "params" or (bt.kind == "a" and bt.n == 8 and bt.elem == F32 and base.code == "p"):
            return TE(F32, f"ndw::param({base.code}, {idx.code})")
        if bt.kind == "v":
            return TE(S(bt.scalar), f"{base.code}[{idx.code}]", lvalue=base.lvalue)
        if bt.kind == "m":
            return TE(V(bt.r, "f32"), f"{base.code}[{idx.code}]", lvalue=base.lvalue)
        if bt.kind == "a":
            return TE(bt.elem, f"{base.code}[{idx.code}]", lvalue=base.lvalue)
        raise TranslateError(f"cannot index {bt}", e.line)

    def e_Member(self, e):
        base = self.expr(e.e)
        bt = base.ty
        if bt.kind == "st":
            fields = STRUCT_FIELDS[bt.name]
            if e.name not in fields:
                raise TranslateError(f"{bt.name} has no field {e.name}", e.line)
            return TE(fields[e.name], f"{base.code}.{e.name}", lvalue=base.lvalue)
        if bt.kind == "v":
            sw = e.name
            comp = {"x": 0, "y": 1, "z": 2, "w": 3, "r": 0, "g": 1, "b": 2, "a": 3}
            try:
                ids = [comp[c] for c in sw]
            except KeyError:
                raise TranslateError(f"bad swizzle .{sw}", e.line)
            if any(i >= bt.n for i in ids) or len(ids) > 4:
                raise TranslateError(f"swizzle .{sw} out of range for {bt}", e.line)
            if len(ids) == 1:
                return TE(S(bt.scalar), f"{base.code}.{'xyzw'[ids[0]]}", lvalue=base.lvalue)
            return TE(V(len(ids), bt.scalar), f"ndw::swz<{', '.join(map(str, ids))}>({base.code})")
        raise TranslateError(f"member .{e.name} of {bt}", e.line)

    # ---- calls
    def e_Call(self, e):
        name = e.name
        args = [self.expr(a) for a in e.args]
        line = e.line
        self.calls.setdefault(self.cur_fn, set()).add(name)
        # type constructors and conversions
        if name in ("f32", "i32", "u32", "bool") and e.targs is None:
            return self.scalar_conv(name, args, line)
        ctor_ty = None
        if name in _SHORT_TYPES and e.targs is None and name not in ("Params", "IterCarry", "ImageInfo",
                                                                        "ImageSample"):
            ctor_ty = _SHORT_TYPES[name]
        elif name in ("vec2", "vec3", "vec4"):
            n = int(name[3])
            if e.targs:
                ctor_ty = V(n, self.resolve_type(e.targs[0]).scalar)
            else:
                ctor_ty = ("infer_vec", n)
        elif name in ("mat2x2", "mat3x3", "mat4x4"):
            ctor_ty = M(int(name[3]), int(name[5]))
        elif name == "array":
            return self.array_ctor(e, args)
        if ctor_ty is not None:
            return self.construct(ctor_ty, args, line)
        if name == "IterCarry":
            if len(args) != 2:
                raise TranslateError("IterCarry(z, dr) takes two arguments", line)
            z = self.convert(args[0], V3F, line)
            dr = self.convert(args[1], F32, line) if is_abstract(args[1].ty) else args[1]
            if dr.ty != F32:
                raise TranslateError("IterCarry.dr must be f32", line)
            return TE(CARRY, f"ndw::IterCarry<T>{{{z.code}, {dr.code}}}")
        if name == "ImageSample":
            if len(args) != 3:
                raise TranslateError("ImageSample(value, near, far) takes three arguments", line)
            conv = [self.convert(a, V4F, line) for a in args]
            return TE(IMAGE_SAMPLE, f"ndw::ImageSample<T>{{{', '.join(c.code for c in conv)}}}")
        if name in ("image_info", "image_sample"):
            return self.image_call(name, args, line)
        if name == "bitcast":
            return self.bitcast(e, args)
        if name in self.fn_sigs:
            return self.user_call(name, args, line)
        if name in TEMPLATE_FUNCS:
            ptys, rty = TEMPLATE_FUNCS[name]
            if len(args) != len(ptys):
                raise TranslateError(f"{name} takes {len(ptys)} arguments", line)
            conv = [self.convert(a, t, line) for a, t in zip(args, ptys)]
            self.features.add("helper:" + name)
            if self.helper_ns != "ndw":  # helpers translated from WGSL: <T, P> templates
                return TE(rty, f"{self.helper_ns}::{name}<T, P>({', '.join(c.code for c in conv)})")
            return TE(rty, f"ndw::{name}<T>({', '.join(c.code for c in conv)})")
        return self.builtin(name, args, line)

    def user_call(self, name, args, line):
        ptys, rty = self.fn_sigs[name]
        if len(args) != len(ptys):
            raise TranslateError(f"{name} takes {len(ptys)} arguments", line)
        conv = []
        for a, (pn, pt) in zip(args, ptys):
            if pt.kind == "params" or (pt.kind == "a" and pt.n == 8 and pt.elem == F32 and pn == "p"):
                if a.ty.kind not in ("params", "a"):
                    raise TranslateError(f"argument {pn} of {name} must be Params", line)
                conv.append(a)
            else:
                conv.append(self.convert(a, pt, line))
        return TE(rty, f"{cpp_name(name)}<T, P>({', '.join(c.code for c in conv)})")

    def scalar_conv(self, name, args, line):
        if len(args) != 1:
            raise TranslateError(f"{name}() takes one argument", line)
        a = args[0]
        target = S(name)
        if a.ty.kind != "s":
            raise TranslateError(f"{name}() of {a.ty}", line)
        if is_abstract(a.ty):
            if name == "f32":
                return self._abstract_to_scalar(self.literal_te(float(a.const), AFLOAT), "f32", line)
            if name in ("i32", "u32"):
                v = int(a.const) if a.ty == AINT else int(math.trunc(a.const))
                return self.literal_te(v, target)
            return TE(BOOL, "true" if a.const else "false", bool(a.const))
        src = a.ty.scalar
        if src == name:
            return a
        if name == "f32":
            if src == "bool":
                return TE(F32, f"({a.code} ? T(1) : T(0))")
            return TE(F32, f"T({a.code})")
        if name == "i32":
            if src == "f32":
                return TE(I32, f"ndw::to_i32({a.code})")
            if src == "u32":
                return TE(I32, f"int32_t({a.code})")
            return TE(I32, f"({a.code} ? 1 : 0)")
        if name == "u32":
            if src == "f32":
                return TE(U32, f"ndw::to_u32({a.code})")
            if src == "i32":
                return TE(U32, f"uint32_t({a.code})")
            return TE(U32, f"({a.code} ? 1u : 0u)")
        if name == "bool":
            if src == "f32":
                return TE(BOOL, f"({a.code} != T(0))")
            return TE(BOOL, f"({a.code} != 0)")
        raise TranslateError(f"conversion {name}({src})", line)

    def bitcast(self, e, args):
        if not e.targs or len(args) != 1:
            raise TranslateError("bitcast<T>(x) needs one type and one argument", e.line)
        target = self.resolve_type(e.targs[0])
        a = args[0]
        if is_abstract(a.ty):
            a = self._abstract_to_scalar(a, "i32" if a.ty == AINT else "f32", e.line)
        self.features.add("bitcast")
        if target.kind == "s" and a.ty.kind == "s":
            src, dst = a.ty.scalar, target.scalar
            if src == dst:
                return a
            if dst == "f32":
                return TE(F32, f"T(ndw::bitcast_f32({a.code}))")
            if src == "f32":
                return TE(target, f"ndw::bitcast_{dst}({a.code})")
            return TE(target, f"{_CPP_SCALAR[dst]}({a.code})")
        if target.kind == "v" and a.ty.kind == "v" and target.n == a.ty.n:
            src, dst = a.ty.scalar, target.scalar
            if src == dst:
                return a
            if "f32" in (src, dst):
                return TE(target, f"ndw::vbitcast_{dst}({a.code})")
            return TE(target, f"ndw::vcast<{_CPP_SCALAR[dst]}>({a.code})")
        raise TranslateError(f"bitcast from {a.ty} to {target}", e.line)

    def construct(self, ty, args, line):
        if isinstance(ty, tuple):           # vecN(...) with inferred element type
            n = ty[1]
            if not args:
                raise TranslateError("vecN() without element type", line)
            args_u = self.unify_scalars(args, line)
            s = None
            for a in args_u:
                s = a.ty.scalar
            s = {"AInt": "i32", "AFloat": "f32"}.get(s, s)
            ty = V(n, s)
        if ty.kind == "s":
            return self.scalar_conv(ty.scalar, args, line)
        if ty.kind == "v":
            sc = ty.scalar
            cty = _CPP_SCALAR[sc]
            if not args:
                return TE(ty, f"ndw::v{ty.n}<{cty}>()")
            if len(args) == 1 and args[0].ty.kind == "v":
                a = args[0]
                if a.ty.n != ty.n:
                    raise TranslateError("vector conversion size mismatch", line)
                if a.ty.scalar == sc:
                    return a
                if a.ty.scalar == "f32" and sc in ("i32", "u32"):
                    return TE(ty, f"ndw::vto_{sc}({a.code})")
                if sc == "f32":
                    return TE(ty, f"ndw::vcast<T>({a.code})")
                return TE(ty, f"ndw::vcast<{cty}>({a.code})")
            parts = []
            count = 0
            for a in args:
                if a.ty.kind == "s":
                    c = self.convert(a, S(sc), line) if is_abstract(a.ty) else a
                    if c.ty.scalar != sc:
                        c = self.scalar_conv(sc, [c], line)
                    parts.append(c.code)
                    count += 1
                elif a.ty.kind == "v":
                    c = a
                    if a.ty.scalar != sc:
                        c = self.construct(V(a.ty.n, sc), [a], line)
                    parts.append(c.code)
                    count += a.ty.n
                else:
                    raise TranslateError(f"cannot build {ty} from {a.ty}", line)
            if count == 1 and len(args) == 1:
                return TE(ty, f"ndw::v{ty.n}<{cty}>({parts[0]})")
            if count != ty.n:
                raise TranslateError(f"{ty} built from {count} components", line)
            return TE(ty, f"ndw::v{ty.n}<{cty}>({', '.join(parts)})")
        if ty.kind == "m":
            if not args:
                return TE(ty, f"ndw::m{ty.n}<T>()")
            if all(a.ty.kind == "v" for a in args):
                if len(args) != ty.n or any(a.ty != V(ty.r, "f32") for a in args):
                    raise TranslateError(f"{ty} needs {ty.n} column vectors", line)
                return TE(ty, f"ndw::m{ty.n}<T>({', '.join(a.code for a in args)})")
            if len(args) == 1 and args[0].ty == ty:
                return args[0]
            if len(args) == ty.n * ty.r:
                conv = [self.convert(a, F32, line) for a in args]
                cols = []
                for c in range(ty.n):
                    comps = ", ".join(conv[c * ty.r + r].code for r in range(ty.r))
                    cols.append(f"ndw::v{ty.r}<T>({comps})")
                return TE(ty, f"ndw::m{ty.n}<T>({', '.join(cols)})")
            raise TranslateError(f"unsupported {ty} constructor", line)
        raise TranslateError(f"cannot construct {ty}", line)

    def array_ctor(self, e, args):
        if e.targs:
            elem = self.resolve_type(e.targs[0])
            n = self.const_int(e.targs[1]) if len(e.targs) > 1 else len(args)
        else:
            if not args:
                raise TranslateError("array() needs elements", e.line)
            args = self.unify_scalars(args, e.line)
            elem = concretize(args[0].ty)
            n = len(args)
        if args and len(args) != n:
            raise TranslateError("array constructor length mismatch", e.line)
        conv = [self.convert(a, elem, e.line) for a in args]
        ty = Ty("a", "", n, elem=elem)
        if not args:
            return TE(ty, f"{cpp_type(ty)}()")
        return TE(ty, f"{cpp_type(ty)}{{{{{', '.join(c.code for c in conv)}}}}}")

    def builtin(self, name, args, line):
        def float_args(xs, n):
            if len(xs) != n:
                raise TranslateError(f"{name} takes {n} arguments", line)
            xs = self.unify_scalars(xs, line)
            xs = [self._abstract_to_scalar(x, "f32", line) if is_abstract(x.ty) else x for x in xs]
            return xs

        def ty_of(xs):
            for x in xs:
                if x.ty.kind == "v":
                    return x.ty
            return xs[0].ty

        if name in _FLOAT_UNARY:
            (a,) = float_args(args, 1)
            if a.ty.scalar != "f32":
                raise TranslateError(f"{name} of {a.ty}", line)
            return TE(a.ty, f"ndw::{name}({a.code})")
        if name in _NUM_UNARY:
            if len(args) != 1:
                raise TranslateError(f"{name} takes 1 argument", line)
            a = args[0]
            if is_abstract(a.ty):
                a = self._abstract_to_scalar(a, "i32" if a.ty == AINT else "f32", line)
            return TE(a.ty, f"ndw::{name}({a.code})")
        if name in _NUM_BINARY or name == "clamp":
            n = 3 if name == "clamp" else 2
            if len(args) != n:
                raise TranslateError(f"{name} takes {n} arguments", line)
            xs = self.unify_scalars(args, line)
            if all(is_abstract(x.ty) for x in xs):
                k = "i32" if all(x.ty == AINT for x in xs) else "f32"
                xs = [self._abstract_to_scalar(x, k, line) for x in xs]
            t = ty_of(xs)
            if t.kind == "v":
                xs = [TE(t, f"ndw::v{t.n}<{_CPP_SCALAR[t.scalar]}>({x.code})") if x.ty.kind == "s" and name == "clamp" else x for x in xs]
                if name != "clamp" and any(x.ty != t for x in xs):
                    raise TranslateError(f"{name} of mixed vector/scalar", line)
            return TE(t, f"ndw::{name}({', '.join(x.code for x in xs)})")
        if name in _FLOAT_BINARY:
            a, b = float_args(args, 2)
            if a.ty != b.ty:
                raise TranslateError(f"{name} of {a.ty} and {b.ty}", line)
            return TE(a.ty, f"ndw::{name}({a.code}, {b.code})")
        if name in ("mix", "smoothstep", "fma"):
            a, b, c = float_args(args, 3)
            t = ty_of([a, b, c])
            if name == "smoothstep" and t.kind == "v" and a.ty.kind == "s":
                a = TE(t, f"ndw::v{t.n}<T>({a.code})")
                b = TE(t, f"ndw::v{t.n}<T>({b.code})")
            return TE(t, f"ndw::{name}({a.code}, {b.code}, {c.code})")
        if name in ("length", "normalize"):
            (a,) = float_args(args, 1)
            if a.ty.kind == "s":
                return TE(F32, f"ndw::{'abs' if name == 'length' else 'sign'}({a.code})")
            return TE(F32 if name == "length" else a.ty, f"ndw::{name}({a.code})")
        if name in ("distance", "dot"):
            a, b = float_args(args, 2)
            if a.ty != b.ty:
                raise TranslateError(f"{name} of {a.ty} and {b.ty}", line)
            rt = F32 if a.ty.scalar == "f32" else S(a.ty.scalar)
            if a.ty.kind == "s" and name == "distance":
                return TE(F32, f"ndw::abs({a.code} - {b.code})")
            return TE(rt, f"ndw::{name}({a.code}, {b.code})")
        if name in ("cross", "reflect"):
            a, b = float_args(args, 2)
            return TE(a.ty, f"ndw::{name}({a.code}, {b.code})")
        if name == "transpose":
            (a,) = args
            if a.ty.kind != "m":
                raise TranslateError("transpose of non-matrix", line)
            return TE(M(a.ty.r, a.ty.n), f"ndw::transpose({a.code})")
        if name == "determinant":
            (a,) = args
            return TE(F32, f"ndw::determinant({a.code})")
        if name == "select":
            if len(args) != 3:
                raise TranslateError("select takes 3 arguments", line)
            f, t_, c = args
            f, t_ = self.unify_scalars([f, t_], line)
            if is_abstract(f.ty):
                k = "i32" if f.ty == AINT and t_.ty == AINT else "f32"
                f = self._abstract_to_scalar(f, k, line)
                t_ = self._abstract_to_scalar(t_, k, line)
            if f.ty != t_.ty:
                raise TranslateError(f"select of {f.ty} and {t_.ty}", line)
            if c.ty != BOOL and not (c.ty.kind == "v" and c.ty.scalar == "bool"):
                raise TranslateError("select condition must be bool", line)
            return TE(f.ty, f"ndw::select({f.code}, {t_.code}, {c.code})")
        if name in ("any", "all"):
            (a,) = args
            if a.ty == BOOL:
                return a
            return TE(BOOL, f"ndw::{name}({a.code})")
        if name in ("countOneBits", "reverseBits", "firstLeadingBit", "firstTrailingBit"):
            (a,) = args
            if is_abstract(a.ty):
                a = self._abstract_to_scalar(a, "u32", line)
            return TE(a.ty, f"ndw::{name}({a.code})")
        if name.startswith("image_") or name in ("textureSample", "textureLoad"):
            raise TranslateError(f"'{name}' is not part of the formula image interface", line)
        raise TranslateError(f"unknown function '{name}'", line)

    def image_call(self, name, args, line):
        """The formula image interface (template.wgsl:1126-1191): image_info() and
        image_sample(info, uv).  The reference selects the image through the private
        g_image_slot its wrapper sets; here the image travels with the parameter
        accessor, so the calling function must have its Params parameter in scope."""
        self.features.add("image")
        if name == "image_info":
            if args:
                raise TranslateError("image_info() takes no arguments", line)
            for sc in reversed(self.scopes):
                for te in sc.values():
                    if te.ty.kind == "params":
                        return TE(IMAGE_INFO, f"ndw::image_info<T>({te.code})")
            raise TranslateError("image_info() needs the function's Params parameter in scope", line)
        if len(args) != 2:
            raise TranslateError("image_sample(info, uv) takes two arguments", line)
        if args[0].ty != IMAGE_INFO:
            raise TranslateError("image_sample's first argument must be an ImageInfo", line)
        uv = self.convert(args[1], V(2, "f32"), line)
        return TE(IMAGE_SAMPLE, f"ndw::image_sample<T>({args[0].code}, {uv.code})")

    # ---- statements
    def block(self, stmts, indent) -> list[str]:
        self.push()
        out = []
        for s in stmts:
            out.extend(self.stmt(s, indent))
        self.pop()
        return out

    def decl_code(self, s: Decl) -> str:
        if s.kind == "const":
            te = self.expr(s.init)
            if s.ty is not None:
                te = self.convert(te, self.resolve_type(s.ty), s.line)
            if te.const is not None:
                self.declare(s.name, te, s.line)
                return ""
            # a const bound to a non-constant expression is a let
        ty = self.resolve_type(s.ty) if s.ty is not None else None
        if s.init is not None:
            te = self.expr(s.init)
            if ty is None:
                ty = concretize(te.ty)
            te = self.convert(te, ty, s.line)
            init = te.code
        else:
            init = None
        if ty.kind in ("params", "void"):
            raise TranslateError(f"cannot declare a {ty}", s.line)
        mutable = s.kind == "var"
        cname = cpp_name(s.name)
        inv = self.inv_fn and not mutable and s.init is not None and self.is_inv(s.init)
        self.declare(s.name, TE(ty, cname, None, lvalue=mutable, inv=inv), s.line)
        qual = "" if mutable else "const "
        if init is None:
            return f"{qual}{cpp_type(ty)} {cname}{{}};"
        return f"{qual}{cpp_type(ty)} {cname} = {init};"

    def assign_code(self, s: Assign) -> str:
        lhs = self.expr(s.lhs)
        if not lhs.lvalue:
            raise TranslateError("assignment to a non-variable", s.line)
        rhs = self.expr(s.rhs)
        if s.op == "=":
            rhs = self.convert(rhs, lhs.ty, s.line) if is_abstract(rhs.ty) else rhs
            if rhs.ty != lhs.ty:
                raise TranslateError(f"assigning {rhs.ty} to {lhs.ty}", s.line)
            return f"{lhs.code} = {rhs.code};"
        op = s.op[:-1]
        combined = self.e_Binary(Binary(s.line, op, s.lhs, s.rhs))
        if combined.ty != lhs.ty:
            raise TranslateError(f"compound {s.op} changes type {lhs.ty} -> {combined.ty}", s.line)
        return f"{lhs.code} = {combined.code};"

    def stmt(self, s, ind) -> list[str]:
        pad = "    " * ind
        if isinstance(s, Decl):
            c = self.decl_code(s)
            return [pad + c] if c else []
        if isinstance(s, Assign):
            return [pad + self.assign_code(s)]
        if isinstance(s, IncDec):
            lhs = self.expr(s.lhs)
            if not lhs.lvalue or lhs.ty.scalar not in ("i32", "u32") or lhs.ty.kind != "s":
                raise TranslateError(f"{s.op} needs an integer variable", s.line)
            return [pad + f"{lhs.code}{s.op};"]
        if isinstance(s, Return):
            if s.e is None:
                return [pad + "return;"]
            te = self.expr(s.e)
            if self.cur_ret.kind == "params":
                raise TranslateError("returning Params is not supported", s.line)
            te = self.convert(te, self.cur_ret, s.line) if (is_abstract(te.ty) or te.ty != self.cur_ret) else te
            return [pad + f"return {te.code};"]
        if isinstance(s, If):
            c = self.expr(s.cond)
            if c.ty != BOOL:
                raise TranslateError("if condition must be bool", s.line)
            out = [pad + f"if ({c.code}) {{"] + self.block(s.then, ind + 1)
            if s.els is not None:
                out.append(pad + "} else {")
                out += self.block(s.els, ind + 1)
            out.append(pad + "}")
            return out
        if isinstance(s, For):
            self.push()
            init = ""
            if s.init is not None:
                if isinstance(s.init, Decl):
                    init = self.decl_code(s.init)
                else:
                    init = self.stmt(s.init, 0)[0].strip()
            cond = ""
            if s.cond is not None:
                c = self.expr(s.cond)
                if c.ty != BOOL:
                    raise TranslateError("for condition must be bool", s.line)
                cond = c.code
            upd = ""
            if s.update is not None:
                upd = self.stmt(s.update, 0)[0].strip().rstrip(";")
            init = init.rstrip(";")
            out = [pad + f"for ({init}; {cond}; {upd}) {{"] + self.block(s.body, ind + 1) + [pad + "}"]
            self.pop()
            self.features.add("loop")
            return out
        if isinstance(s, While):
            c = self.expr(s.cond)
            if c.ty != BOOL:
                raise TranslateError("while condition must be bool", s.line)
            self.features.add("loop")
            return [pad + f"while ({c.code}) {{"] + self.block(s.body, ind + 1) + [pad + "}"]
        if isinstance(s, Switch):
            # an if / else-if chain on the selector: WGSL clauses do not fall through;
            # a `break` inside a clause (leave the switch) is outside the subset
            sel = self.expr(s.sel)
            if sel.ty.kind != "s" or sel.ty.scalar not in ("i32", "u32"):
                sel = self.convert(sel, I32, s.line) if is_abstract(sel.ty) else sel
            if sel.ty.kind != "s" or sel.ty.scalar not in ("i32", "u32"):
                raise TranslateError("switch selector must be an integer", s.line)

            def has_break(body):
                for st in body:
                    if isinstance(st, Break):
                        return True
                    if isinstance(st, If) and (has_break(st.then) or (st.els and has_break(st.els))):
                        return True
                    if isinstance(st, Block) and has_break(st.body):
                        return True
                return False

            var = f"sw_{s.line}_{len(self.features)}"
            out = [pad + "{", pad + f"    const {cpp_type(sel.ty)} {var} = {sel.code};"]
            default_body = None
            first = True
            for cases, dflt, body in s.clauses:
                if has_break(body):
                    raise TranslateError("break inside a switch clause is outside the subset", s.line)
                if dflt:
                    default_body = body
                    if not cases:
                        continue
                conds = []
                for c in cases:
                    ce = self.expr(c)
                    ce = self.convert(ce, sel.ty, s.line) if (is_abstract(ce.ty) or ce.ty != sel.ty) else ce
                    conds.append(f"{var} == {ce.code}")
                if dflt:
                    continue  # `case x, default` is the default clause
                out.append(pad + f"    {'if' if first else '} else if'} ({' || '.join(conds)}) {{")
                out += self.block(body, ind + 2)
                first = False
            if default_body is not None:
                if first:
                    out.append(pad + "    {")
                else:
                    out.append(pad + "    } else {")
                out += self.block(default_body, ind + 2)
                out.append(pad + "    }")
            elif not first:
                out.append(pad + "    }")
            out.append(pad + "}")
            return out
        if isinstance(s, Break):
            return [pad + "break;"]
        if isinstance(s, Continue):
            return [pad + "continue;"]
        if isinstance(s, ExprStmt):
            te = self.expr(s.e)
            return [pad + f"(void)({te.code});"]
        if isinstance(s, Block):
            return [pad + "{"] + self.block(s.body, ind + 1) + [pad + "}"]
        raise TranslateError(f"statement {type(s).__name__}", s.line)

    # ---- functions
    def fn_signature(self, f: FnDecl) -> str:
        ptys, rty = self.fn_sigs[f.name]
        params = []
        for (pn, pt) in ptys:
            if pt.kind == "params" or (pt.kind == "a" and pt.n == 8 and pt.elem == F32 and pn == "p"):
                params.append(f"const P& {cpp_name(pn)}")
            else:
                params.append(f"{cpp_type(pt)} {cpp_name(pn)}")
        return (f"template <class T, class P> ND_HD_INLINE {cpp_type(rty)} "
                f"{cpp_name(f.name)}({', '.join(params)})")

    def fn_body(self, f: FnDecl) -> list[str]:
        ptys, rty = self.fn_sigs[f.name]
        self.cur_ret = rty
        self.cur_fn = f.name
        # de_step(carry, pos, p): pos and the parameters are the same in every iteration
        self.inv_fn = f.name == "de_step" and len(ptys) == 3
        self.push()
        for k, (pn, pt) in enumerate(ptys):
            if pt.kind == "a" and pt.n == 8 and pt.elem == F32 and pn == "p":
                pt = PARAMS
            self.declare(pn, TE(pt, cpp_name(pn), None, lvalue=False, inv=self.inv_fn and k > 0), f.line)
        body = []
        for s in f.body:
            body.extend(self.stmt(s, 1))
        self.pop()
        self.inv_fn = False
        return body

    def is_inv(self, e: Expr) -> bool:
        """In de_step: does e have the same value in every iteration (built from pos, the
        parameters, constants and `let`s of those, through pure operations)?"""
        if isinstance(e, Num):
            return True
        if isinstance(e, Ident):
            if e.name in ("true", "false"):
                return True
            for sc in reversed(self.scopes):
                if e.name in sc:
                    te = sc[e.name]
                    return te.inv or te.const is not None
            return e.name in self.module_consts_src or e.name in TEMPLATE_CONSTS
        if isinstance(e, Unary):
            return self.is_inv(e.e)
        if isinstance(e, Binary):
            return self.is_inv(e.l) and self.is_inv(e.r)
        if isinstance(e, Call):
            return all(self.is_inv(a) for a in e.args)
        if isinstance(e, Index):
            return self.is_inv(e.e) and self.is_inv(e.idx)
        if isinstance(e, Member):
            return self.is_inv(e.e)
        return False

    def check_contract(self):
        need = {
            "de_iterations": ([PARAMS], I32),
            "de_step": ([CARRY, V3F, PARAMS], CARRY),
            "de_finalize": ([CARRY], F32),
        }
        for name, (ptys, rty) in need.items():
            if name not in self.fn_sigs:
                raise TranslateError(f"missing contract function {name}")
            have_p, have_r = self.fn_sigs[name]
            have_t = [PARAMS if (t.kind == "a" and t.n == 8 and t.elem == F32) else t for _, t in have_p]
            if have_t != ptys or have_r != rty:
                raise TranslateError(f"contract function {name} has the wrong signature")

    def emit(self, contract: bool = True) -> str:
        if contract:
            self.check_contract()
        lines = [f"namespace {self.ns} {{"]
        for name in self.fn_order:
            lines.append(self.fn_signature(self.fns[name]) + ";")
        for name in self.fn_order:
            f = self.fns[name]
            body = self.fn_body(f)
            lines.append(self.fn_signature(f) + " {")
            lines.extend(body)
            lines.append("}")
        lines.append(f"}}  // namespace {self.ns}")
        return "\n".join(lines)


@dataclasses.dataclass
class TranslatedFormula:
    name: str
    namespace: str
    cpp: str
    params: list
    source_hash: int
    features: set


def _sanitize(name: str) -> str:
    s = re.sub(r"[^A-Za-z0-9_]", "_", name)
    if s and s[0].isdigit():
        s = "_" + s
    return s


def translate(source: str, name: str) -> TranslatedFormula:
    """Translate one formula file.  Raises TranslateError on anything outside the subset."""
    from ..formula import parse_formula_params, source_hash, missing_contract_fn, image_directive

    missing = missing_contract_fn(source)
    if missing is not None:
        raise TranslateError(f"formula is missing `{missing}`")

    toks = lex(source)
    fns, consts = Parser(toks).module()
    ns = "ndf_" + _sanitize(name)
    comp = FormulaCompiler(fns, consts, ns)
    cpp = comp.emit()
    return TranslatedFormula(name, ns, cpp, parse_formula_params(source), source_hash(source), comp.features)


def translate_module(source: str, namespace: str, helper_ns: str = "ndw", contract: bool = True) -> str:
    """Translate a WGSL module into one C++ namespace.  With helper_ns, calls to the
    template helper functions go to that namespace (helpers translated from WGSL)
    instead of the hand-written library; contract=False skips the formula contract
    check (for a module of helpers)."""
    toks = lex(source)
    fns, consts = Parser(toks).module()
    comp = FormulaCompiler(fns, consts, namespace, helper_ns=helper_ns)
    return comp.emit(contract=contract)
