"""Fortran 90 rate expressions and assignments -> C / CUDA text.

KPP mechanisms written for the Fortran 90 target (examples/mcm of KPP) give
their rate constants as Fortran expressions: `1.7E-12*EXP(-940./TEMP)`,
`(TEMP/300.)**(-2.6)`, `J(J_NO2)`, `KRO2NO*0.917`.  This module translates
them into C that computes the same values with the same roundings:

  * literal kinds: a real literal without a D exponent is default REAL
    (single precision) and stays a float literal (`2.7E-12` -> `2.7E-12f`),
    a D exponent makes it double; integer literals stay int.  Mixed
    arithmetic then promotes exactly as Fortran does (int < float < double,
    C's usual arithmetic conversions are the same rules);
  * intrinsics follow the argument kind (`EXP` of a float is `expf`, of a
    double `exp`);
  * `a**b`: integer exponent literals 2..4 expand to products in the base's
    kind; real exponents use `pow`/`powf` in the wider kind of the two
    operands (an integer base takes the exponent's kind);
  * named variables are REAL(dp) (double) unless listed otherwise; `J(k)`
    style indexing maps through a table of integer parameters.

Precedence is Fortran's: `**` binds tightest and right to left, unary minus
applies to a whole multiplicative term (`-a**2` is `-(a**2)`).
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional

INT, F32, F64 = 0, 1, 2
_KIND_NAME = {INT: "int", F32: "float", F64: "double"}

_TOKEN = re.compile(r"""
    (?P<num>(\d+\.\d*|\.\d+|\d+)([EeDd][+-]?\d+)?(_\w+)?)
  | (?P<id>[A-Za-z_][A-Za-z_0-9]*)
  | (?P<pow>\*\*)
  | (?P<op>[-+*/(),])
  | (?P<ws>\s+)
""", re.X)


class FortranError(ValueError):
    pass


@dataclass
class Expr:
    text: str
    kind: int


@dataclass
class Context:
    """How identifiers translate.  `variables` maps a Fortran name (upper
    case) to (C text, kind); `arrays` maps an array name to a function
    turning the translated index into C; `int_params` are integer named
    constants (Fortran PARAMETERs) usable as indices."""
    variables: Dict[str, tuple] = field(default_factory=dict)
    arrays: Dict[str, Callable[[str, "Expr"], str]] = field(default_factory=dict)
    int_params: Dict[str, int] = field(default_factory=dict)
    default_kind: Optional[int] = F64  # undeclared names: REAL(dp) variables

    def variable(self, name: str) -> Expr:
        u = name.upper()
        if u in self.int_params:
            return Expr(str(self.int_params[u]), INT)
        if u in self.variables:
            text, kind = self.variables[u]
            return Expr(text, kind)
        if self.default_kind is None:
            raise FortranError(f"unknown name {name}")
        return Expr(name, self.default_kind)


def tokenize(s: str) -> List[tuple]:
    out, i = [], 0
    while i < len(s):
        m = _TOKEN.match(s, i)
        if not m:
            raise FortranError(f"cannot read {s[i:i + 20]!r}")
        i = m.end()
        if m.lastgroup != "ws":
            out.append((m.lastgroup, m.group()))
    return out


def _literal(text: str) -> Expr:
    t = text.split("_")[0]
    if re.fullmatch(r"\d+", t):
        return Expr(t, INT)
    m = re.fullmatch(r"(\d+\.\d*|\.\d+|\d+)([EeDd]([+-]?\d+))?", t)
    mant, exp = m.group(1), m.group(3)
    if mant.endswith("."):
        mant += "0"
    if mant.startswith("."):
        mant = "0" + mant
    if m.group(2) and m.group(2)[0] in "Dd":
        return Expr(f"{mant}e{exp}", F64)
    return Expr(f"{mant}e{exp}f" if exp is not None else f"{mant}f", F32)


def _cast(e: Expr, kind: int) -> str:
    if e.kind == kind:
        return e.text
    return f"(({_KIND_NAME[kind]})({e.text}))"


_INTRINSICS = {  # name: (float form, double form)
    "EXP": ("expf", "exp"), "LOG": ("logf", "log"), "LOG10": ("log10f", "log10"),
    "SQRT": ("sqrtf", "sqrt"), "COS": ("cosf", "cos"), "SIN": ("sinf", "sin"),
    "TAN": ("tanf", "tan"), "ABS": ("fabsf", "fabs"), "ATAN": ("atanf", "atan"),
    "ACOS": ("acosf", "acos"),
}


class _Parser:
    def __init__(self, tokens, ctx: Context):
        self.t = tokens
        self.i = 0
        self.ctx = ctx

    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else (None, None)

    def take(self, text=None):
        tok = self.peek()
        if tok[0] is None or (text is not None and tok[1] != text):
            raise FortranError(f"expected {text!r}, found {tok[1]!r}")
        self.i += 1
        return tok

    # level-2 expression: [sign] term {(+|-) term}
    def expr(self) -> Expr:
        sign = None
        if self.peek()[1] in ("+", "-"):
            sign = self.take()[1]
        e = self.term()
        if sign == "-":
            e = Expr(f"(-{e.text})", e.kind)
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            r = self.term()
            e = Expr(f"({e.text} {op} {r.text})", max(e.kind, r.kind))
        return e

    def term(self) -> Expr:
        e = self.factor()
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            r = self.factor()
            e = Expr(f"({e.text} {op} {r.text})", max(e.kind, r.kind))
        return e

    def factor(self) -> Expr:
        # a signed operand after * or / (a common extension) binds like -(x**y)
        if self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            e = self.factor()
            return Expr(f"({op}{e.text})", e.kind) if op == "-" else e
        base = self.primary()
        if self.peek()[0] == "pow":
            self.take()
            ex = self.factor()  # right associative, may carry a sign
            return self.power(base, ex)
        return base

    def power(self, b: Expr, e: Expr) -> Expr:
        if e.kind == INT:
            m = re.fullmatch(r"\(*(-?\d+)\)*", e.text.replace(" ", ""))
            n = int(m.group(1)) if m else None
            if n is not None and 2 <= n <= 4 and b.kind != INT:
                x = f"({b.text})"
                prod = {2: f"({x} * {x})", 3: f"(({x} * {x}) * {x})",
                        4: f"(({x} * {x}) * ({x} * {x}))"}[n]
                return Expr(prod, b.kind)
            if b.kind == INT:
                raise FortranError("integer ** integer is not supported")
            fn = "powf" if b.kind == F32 else "pow"
            return Expr(f"{fn}({b.text}, {_cast(e, b.kind)})", b.kind)
        kind = max(b.kind, e.kind) if b.kind != INT else e.kind
        fn = "powf" if kind == F32 else "pow"
        return Expr(f"{fn}({_cast(b, kind)}, {_cast(e, kind)})", kind)

    def primary(self) -> Expr:
        kind, text = self.peek()
        if kind == "num":
            self.take()
            return _literal(text)
        if text == "(":
            self.take("(")
            e = self.expr()
            self.take(")")
            return Expr(f"({e.text})", e.kind)
        if kind == "id":
            self.take()
            u = text.upper()
            if self.peek()[1] == "(":
                self.take("(")
                args = [self.expr()]
                while self.peek()[1] == ",":
                    self.take(",")
                    args.append(self.expr())
                self.take(")")
                return self.call(u, text, args)
            return self.ctx.variable(text)
        raise FortranError(f"unexpected {text!r}")

    def call(self, u: str, name: str, args: List[Expr]) -> Expr:
        if u in self.ctx.arrays:
            if len(args) != 1:
                raise FortranError(f"{name}: one index expected")
            return Expr(self.ctx.arrays[u](name, args[0]), F64)
        if u in _INTRINSICS:
            a = args[0]
            kind = F32 if a.kind == F32 else F64
            if a.kind == INT:
                raise FortranError(f"{name} of an integer")
            fn = _INTRINSICS[u][0 if kind == F32 else 1]
            return Expr(f"{fn}({a.text})", kind)
        if u in ("REAL", "SNGL"):
            return Expr(_cast(args[0], F32), F32)
        if u == "DBLE":
            return Expr(_cast(args[0], F64), F64)
        if u in ("MAX", "MIN"):
            kind = max(a.kind for a in args)
            fn = ("fmaxf" if u == "MAX" else "fminf") if kind == F32 else (
                "fmax" if u == "MAX" else "fmin")
            text = _cast(args[0], kind)
            for a in args[1:]:
                text = f"{fn}({text}, {_cast(a, kind)})"
            return Expr(text, kind)
        raise FortranError(f"unknown function {name}")


def translate_expr(s: str, ctx: Context) -> Expr:
    p = _Parser(tokenize(s), ctx)
    e = p.expr()
    if p.i != len(p.t):
        raise FortranError(f"trailing text in {s!r}: {p.t[p.i:]}")
    return e


def join_continuations(lines: List[str]) -> List[str]:
    """Free-form source lines with `!` comments removed and `&` continuations
    joined."""
    out, cur = [], ""
    for raw in lines:
        line = raw.split("!", 1)[0].rstrip()
        if not line.strip():
            continue
        if line.rstrip().endswith("&"):
            cur += line.rstrip()[:-1] + " "
            continue
        out.append((cur + line).strip())
        cur = ""
    if cur.strip():
        out.append(cur.strip())
    return out


_ASSIGN = re.compile(r"^([A-Za-z_][A-Za-z_0-9]*)\s*(\(\s*([^)]*)\s*\))?\s*=\s*(.+)$")


def translate_assignment(stmt: str, ctx: Context, lhs_kind: int = F64) -> tuple:
    """`NAME = expr` or `ARR(idx) = expr` -> (C statement, target name)."""
    m = _ASSIGN.match(stmt)
    if not m:
        raise FortranError(f"not an assignment: {stmt!r}")
    name, idx, rhs = m.group(1), m.group(3), m.group(4)
    e = translate_expr(rhs, ctx)
    value = _cast(e, lhs_kind)
    if idx is not None:
        u = name.upper()
        if u not in ctx.arrays:
            raise FortranError(f"unknown array {name}")
        target = ctx.arrays[u](name, translate_expr(idx, ctx))
        return f"{target} = {value};", name
    target, _ = ctx.variables.get(name.upper(), (name, lhs_kind))
    return f"{target} = {value};", name
