"""CellML (OpenCOR C export) parser and code emitter.

The reference turns an OpenCOR-exported C file (``initConsts`` / ``computeRates``)
into model code at run time: it parses every assignment line into an expression
tree, substitutes per-instance *parameters* for selected CONSTANTS / ALGEBRAIC
entries, replaces ``pow(x, <int>)`` by integer-power helpers and ``exp`` / ``log`` by
helpers that may be approximated, and then emits vectorised C++
(core/src/cellml/source_code_generator/00_parse_source_code_file.cpp:159-357,
03_generator_vc.cpp:13-302 and :304-617).

This module does the same job for the B200 build, ahead of time:

* :func:`parse_model_file` reads the OpenCOR C file into a :class:`Model`
  (initial states, folded constants, assignment lines as expression trees,
  variable names from the header comments).
* :func:`emit_cuda_model` writes a ``__device__`` right-hand side templated on the
  arithmetic type (``double`` for the FP64 path, ``float`` for FP32 reaction)
  and on a math policy (exact or approximate exp/log).
* :func:`emit_c_model` writes the same right-hand side as scalar C for the CPU
  oracle.
* :func:`emit_cuda_vjp` writes the reverse-mode (vector-Jacobian) product of the
  right-hand side used by the hand-written adjoint.

Parameter substitution follows the reference exactly
(00_parse_source_code_file.cpp:281-323): the assignment line of an algebraic
that is a parameter is dropped and every later read of it becomes
``PARAMS[j]``; a constant that is a parameter is read as
``PARAMS[nAlgebraicParameters + j]`` in the right-hand side lines only, while
the derived constants of ``initConsts`` keep using the file's raw values
(00_source_code_generator_base.cpp:45-113, 03_generator_vc.cpp:937-944).
"""
from __future__ import annotations

import json
import math
import numbers
import os
import re
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

# ----------------------------------------------------------------------------------------------
# tokenizer / parser for the C expression subset used by OpenCOR exports
# ----------------------------------------------------------------------------------------------

_TOKEN_RE = re.compile(r"""
    (?P<num>(?:\d+\.\d*|\.\d+|\d+)(?:[eE][+-]?\d+)?)
  | (?P<arr>(?:STATES|CONSTANTS|ALGEBRAIC|RATES)\s*\[\s*\d+\s*\])
  | (?P<name>[A-Za-z_][A-Za-z_0-9]*)
  | (?P<op>&&|\|\||<=|>=|==|!=|[-+*/<>()?:,!])
  | (?P<ws>\s+)
""", re.VERBOSE)

_KIND = {"STATES": "S", "CONSTANTS": "C", "ALGEBRAIC": "A", "RATES": "R"}


def tokenize(text: str) -> List[Tuple[str, object]]:
    pos = 0
    out: List[Tuple[str, object]] = []
    while pos < len(text):
        m = _TOKEN_RE.match(text, pos)
        if not m:
            raise ValueError(f"cannot tokenize at {text[pos:pos + 30]!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        val = m.group(kind)
        if kind == "arr":
            name, idx = val.split("[")
            out.append(("var", (_KIND[name.strip()], int(idx.strip().rstrip("]").strip()))))
        elif kind == "name":
            if val == "VOI":
                out.append(("var", ("T", 0)))
            else:
                out.append(("name", val))
        else:
            out.append((kind, val))
    out.append(("end", None))
    return out


# binary operator precedence (C): || < && < == != < < <= > >= < + - < * /
_BIN_PREC = {"||": 1, "&&": 2, "==": 3, "!=": 3, "<": 4, "<=": 4, ">": 4, ">=": 4,
             "+": 5, "-": 5, "*": 6, "/": 6}


class _Parser:
    def __init__(self, tokens):
        self.t = tokens
        self.i = 0

    def peek(self):
        return self.t[self.i]

    def take(self, kind=None, val=None):
        tok = self.t[self.i]
        if kind is not None and tok[0] != kind:
            raise ValueError(f"expected {kind} {val} got {tok}")
        if val is not None and tok[1] != val:
            raise ValueError(f"expected {val} got {tok}")
        self.i += 1
        return tok

    def expr(self):
        return self.ternary()

    def ternary(self):
        cond = self.binary(1)
        if self.peek() == ("op", "?"):
            self.take()
            a = self.ternary()
            self.take("op", ":")
            b = self.ternary()
            return ("tern", cond, a, b)
        return cond

    def binary(self, min_prec):
        left = self.unary()
        while True:
            tok = self.peek()
            if tok[0] != "op" or tok[1] not in _BIN_PREC:
                return left
            prec = _BIN_PREC[tok[1]]
            if prec < min_prec:
                return left
            self.take()
            right = self.binary(prec + 1)  # left associative
            left = ("bin", tok[1], left, right)

    def unary(self):
        tok = self.peek()
        if tok == ("op", "-"):
            self.take()
            return ("neg", self.unary())
        if tok == ("op", "+"):
            self.take()
            return ("pos", self.unary())
        if tok == ("op", "!"):
            self.take()
            return ("not", self.unary())
        return self.primary()

    def primary(self):
        tok = self.take()
        if tok[0] == "num":
            return ("num", tok[1], float(tok[1]))
        if tok[0] == "var":
            return ("var",) + tuple(tok[1])
        if tok[0] == "name":
            fname = tok[1]
            self.take("op", "(")
            args = [self.expr()]
            while self.peek() == ("op", ","):
                self.take()
                args.append(self.expr())
            self.take("op", ")")
            return ("call", fname, args)
        if tok == ("op", "("):
            e = self.expr()
            self.take("op", ")")
            return e
        raise ValueError(f"unexpected token {tok}")


def parse_expression(text: str):
    p = _Parser(tokenize(text))
    e = p.expr()
    if p.peek()[0] != "end":
        raise ValueError(f"trailing tokens in {text!r}: {p.t[p.i:]}")
    return e


# ----------------------------------------------------------------------------------------------
# model
# ----------------------------------------------------------------------------------------------

@dataclass
class Model:
    """A parsed OpenCOR C model."""
    name: str
    source: str
    n_states: int
    n_algebraics: int
    n_constants: int
    states_initial: List[float]
    constants: List[float]                      # folded raw values after initConsts
    constant_lines: List[Tuple[int, object]]    # (index, expr) in initConsts order
    lines: List[Tuple[str, int, object]]        # (kind 'A'|'R', index, expr) right-hand side
    state_names: List[str] = field(default_factory=list)
    algebraic_names: List[str] = field(default_factory=list)
    constant_names: List[str] = field(default_factory=list)
    uses_voi: bool = False


def _int_pow_value(x: float, n: int) -> float:
    """Integer power by the reference helper recursion (03_generator_vc.cpp:549-608)."""
    if n < 0:
        return 1.0 / _int_pow_value(x, -n)
    if n == 1:
        return x
    if n == 2:
        return x * x
    e0 = n // 2
    e1 = n - e0
    if e0 == 1:
        return x * _int_pow_value(x, e1)
    return _int_pow_value(x, e0) * _int_pow_value(x, e1)


def eval_expr(e, env) -> float:
    """Evaluate an expression tree in IEEE double (used to fold initConsts)."""
    t = e[0]
    if t == "num":
        return e[2]
    if t == "var":
        return env[e[1]][e[2]] if e[1] != "T" else env["T"]
    if t == "neg":
        return -eval_expr(e[1], env)
    if t == "pos":
        return eval_expr(e[1], env)
    if t == "not":
        return 0.0 if eval_expr(e[1], env) else 1.0
    if t == "bin":
        op = e[1]
        a = eval_expr(e[2], env)
        if op == "&&":
            return 1.0 if (a and eval_expr(e[3], env)) else 0.0
        if op == "||":
            return 1.0 if (a or eval_expr(e[3], env)) else 0.0
        b = eval_expr(e[3], env)
        return {"+": lambda: a + b, "-": lambda: a - b, "*": lambda: a * b, "/": lambda: a / b,
                "<": lambda: float(a < b), "<=": lambda: float(a <= b), ">": lambda: float(a > b),
                ">=": lambda: float(a >= b), "==": lambda: float(a == b),
                "!=": lambda: float(a != b)}[op]()
    if t == "tern":
        return eval_expr(e[2], env) if eval_expr(e[1], env) else eval_expr(e[3], env)
    if t == "call":
        f = e[1]
        args = [eval_expr(a, env) for a in e[2]]
        if f == "exp":
            return math.exp(args[0])
        if f == "log":
            return math.log(args[0])
        if f == "pow":
            return math.pow(args[0], args[1])
        if f == "fabs":
            return abs(args[0])
        if f == "sqrt":
            return math.sqrt(args[0])
        raise ValueError(f"unknown function {f}")
    raise ValueError(f"bad node {e}")


_NAME_RE = re.compile(r"\*\s*(STATES|ALGEBRAIC|CONSTANTS)\[(\d+)\] is (\S+) in component (\S+) \(")


def parse_model_file(path: str, name: Optional[str] = None) -> Model:
    """Parse an OpenCOR C export.

    Line handling follows 00_parse_source_code_file.cpp:183-354: ``void`` is
    joined with the next line, ``STATES[i] = v`` lines before ``computeRates`` give
    initial values, ``CONSTANTS[i] = ...`` lines inside ``initConsts`` are the
    constant assignments, ``ALGEBRAIC`` / ``RATES`` lines after it are the right-hand
    side, and algebraics that are assigned a second time (in
    ``computeVariables``) are skipped.
    """
    with open(path) as f:
        text = f.read()
    header = re.search(r"There are a total of (\d+) entries in the algebraic variable array\.\s*"
                       r"\s*There are a total of (\d+) entries in each of the rate and state variable arrays\.\s*"
                       r"\s*There are a total of (\d+) entries in the constant variable array", text)
    if not header:
        raise ValueError(f"{path}: not an OpenCOR C export (missing size header)")
    n_alg, n_states, n_const = (int(x) for x in header.groups())
    names = {"STATES": [""] * n_states, "ALGEBRAIC": [""] * n_alg, "CONSTANTS": [""] * n_const}
    for m in _NAME_RE.finditer(text):
        arr, idx, var, comp = m.group(1), int(m.group(2)), m.group(3), m.group(4)
        if idx < len(names[arr]):
            names[arr][idx] = f"{comp}/{var}"

    states_init = [0.0] * n_states
    constant_lines: List[Tuple[int, object]] = []
    lines: List[Tuple[str, int, object]] = []
    assigned_alg = set()
    in_init = False
    header_done = False
    uses_voi = False
    raw_lines = text.split("\n")
    i = 0
    while i < len(raw_lines):
        line = raw_lines[i]
        i += 1
        if line == "void" and i < len(raw_lines):
            line = line + " " + raw_lines[i]
            i += 1
        if not header_done and line.startswith("STATES["):
            idx = int(line[7:line.index("]")])
            states_init[idx] = float(line[line.index("= ") + 2:].strip().rstrip(";"))
        if "initConsts" in line:
            in_init = True
            continue
        if "}" in line and in_init:
            in_init = False
            continue
        if line.startswith("CONSTANTS["):
            lhs, rhs = line.split("=", 1)
            idx = int(lhs[lhs.index("[") + 1:lhs.index("]")])
            constant_lines.append((idx, parse_expression(rhs.strip().rstrip(";"))))
            continue
        if "computeRates" in line:
            header_done = True
            continue
        if header_done and (line.startswith("ALGEBRAIC") or line.startswith("RATES")):
            lhs, rhs = line.split("=", 1)
            kind = "A" if lhs.startswith("ALGEBRAIC") else "R"
            idx = int(lhs[lhs.index("[") + 1:lhs.index("]")])
            if kind == "A":
                if idx in assigned_alg:
                    continue
                assigned_alg.add(idx)
            expr = parse_expression(rhs.strip().rstrip(";"))
            if "VOI" in rhs:
                uses_voi = True
            lines.append((kind, idx, expr))

    # fold the constants in initConsts order, in IEEE double
    consts = [0.0] * n_const
    env = {"S": states_init, "C": consts, "A": [], "R": [], "T": 0.0}
    for idx, expr in constant_lines:
        consts[idx] = eval_expr(expr, env)

    return Model(name=name or os.path.splitext(os.path.basename(path))[0], source=path,
                 n_states=n_states, n_algebraics=n_alg, n_constants=n_const,
                 states_initial=states_init, constants=consts, constant_lines=constant_lines,
                 lines=lines, state_names=names["STATES"], algebraic_names=names["ALGEBRAIC"],
                 constant_names=names["CONSTANTS"], uses_voi=uses_voi)


# ----------------------------------------------------------------------------------------------
# parameter substitution
# ----------------------------------------------------------------------------------------------

def substitute_parameters(model: Model, params_alg: Sequence[int], params_const: Sequence[int]):
    """Return the right-hand side lines with parameters substituted.

    Follows 00_parse_source_code_file.cpp:281-323: the line assigning an
    algebraic parameter is dropped, reads of it become PARAMS[j], reads of a
    constant parameter become PARAMS[len(params_alg) + j].
    """
    alg_map = {a: j for j, a in enumerate(params_alg)}
    const_map = {c: len(params_alg) + j for j, c in enumerate(params_const)}

    def sub(e):
        t = e[0]
        if t == "var":
            if e[1] == "A" and e[2] in alg_map:
                return ("var", "P", alg_map[e[2]])
            if e[1] == "C" and e[2] in const_map:
                return ("var", "P", const_map[e[2]])
            return e
        if t in ("num",):
            return e
        if t in ("neg", "pos", "not"):
            return (t, sub(e[1]))
        if t == "bin":
            return ("bin", e[1], sub(e[2]), sub(e[3]))
        if t == "tern":
            return ("tern", sub(e[1]), sub(e[2]), sub(e[3]))
        if t == "call":
            return ("call", e[1], [sub(a) for a in e[2]])
        raise ValueError(e)

    out = []
    for kind, idx, expr in model.lines:
        if kind == "A" and idx in alg_map:
            continue
        out.append((kind, idx, sub(expr)))
    return out


# ----------------------------------------------------------------------------------------------
# emitters
# ----------------------------------------------------------------------------------------------

def _hexf(v: float) -> str:
    """Exact double literal (C99 hex float)."""
    if v == 0.0:
        return "0.0" if math.copysign(1.0, v) > 0 else "-0.0"
    if math.isinf(v) or math.isnan(v):
        raise ValueError("non-finite constant")
    return float.hex(v)


def _int_exponent(e) -> Optional[int]:
    """Integer exponent detection of the reference (03_generator_vc.cpp:68-117):
    a literal made only of digits, sign and dot whose atoi is non-zero."""
    neg = False
    while e[0] in ("neg", "pos"):
        neg ^= e[0] == "neg"
        e = e[1]
    if e[0] != "num":
        return None
    txt = e[1]
    if re.fullmatch(r"[0-9.+-]+", txt) is None:
        return None
    m = re.match(r"\s*[+-]?\d+", txt)
    n = int(m.group(0)) if m else 0
    if n == 0:
        return None
    return -n if neg else n


class _Emitter:
    """Emits an expression tree as C / CUDA source text."""

    def __init__(self, real: str, const_values: List[float], target: str):
        self.real = real            # C type name used for literals and casts
        self.consts = const_values
        self.target = target        # "cuda" or "c"

    def lit(self, v: float) -> str:
        return f"(({self.real}){_hexf(v)})"

    def var(self, kind: str, idx: int) -> str:
        if kind == "S":
            return f"STATES[{idx}]"
        if kind == "C":
            return self.lit(self.consts[idx])
        if kind == "A":
            return f"ALGEBRAIC[{idx}]"
        if kind == "R":
            return f"RATES[{idx}]"
        if kind == "P":
            return f"PARAMS[{idx}]"
        if kind == "T":
            return "VOI"
        raise ValueError(kind)

    def expr(self, e) -> str:
        t = e[0]
        if t == "num":
            return f"(({self.real}){e[1]})"
        if t == "var":
            return self.var(e[1], e[2])
        if t == "neg":
            return f"(-{self.expr(e[1])})"
        if t == "pos":
            return f"(+{self.expr(e[1])})"
        if t == "not":
            return f"(!{self.expr(e[1])})"
        if t == "bin":
            return f"({self.expr(e[2])} {e[1]} {self.expr(e[3])})"
        if t == "tern":
            return f"(({self.expr(e[1])}) ? {self.expr(e[2])} : {self.expr(e[3])})"
        if t == "call":
            f = e[1]
            if f == "pow":
                n = _int_exponent(e[2][1])
                if n is not None:
                    if n > 0:
                        return f"FDM_POW{n}({self.expr(e[2][0])})"
                    return f"(({self.real})1.0/FDM_POW{-n}({self.expr(e[2][0])}))"
                return f"FDM_POWF({self.expr(e[2][0])}, {self.expr(e[2][1])})"
            if f == "exp":
                return f"FDM_EXP({self.expr(e[2][0])})"
            if f == "log":
                return f"FDM_LOG({self.expr(e[2][0])})"
            if f == "fabs":
                return f"FDM_ABS({self.expr(e[2][0])})"
            if f == "sqrt":
                return f"FDM_SQRT({self.expr(e[2][0])})"
            raise ValueError(f"unsupported function {f}")
        raise ValueError(e)


def _collect_int_pows(lines) -> List[int]:
    found = set()

    def walk(e):
        t = e[0]
        if t == "call":
            if e[1] == "pow":
                n = _int_exponent(e[2][1])
                if n is not None:
                    found.add(abs(n))
            for a in e[2]:
                walk(a)
        elif t in ("neg", "pos", "not"):
            walk(e[1])
        elif t == "bin":
            walk(e[2])
            walk(e[3])
        elif t == "tern":
            walk(e[1])
            walk(e[2])
            walk(e[3])
    for _, _, e in lines:
        walk(e)
    # close over the recursion of the helpers
    changed = True
    while changed:
        changed = False
        for n in list(found):
            if n > 2:
                e0 = n // 2
                e1 = n - e0
                for k in (e0, e1):
                    if k > 1 and k not in found:
                        found.add(k)
                        changed = True
    return sorted(found)


def _pow_macro_defs(pows: List[int], prefix: str = "") -> List[str]:
    out = []
    for n in pows:
        if n == 1:
            out.append(f"#define FDM_POW1(x) (x)")
        elif n == 2:
            out.append(f"#define FDM_POW2(x) fdm_pow2(x)")
        else:
            out.append(f"#define FDM_POW{n}(x) fdm_pow{n}(x)")
    return out


def _pow_helpers(pows: List[int], qual: str) -> List[str]:
    """Integer power helpers with the reference's multiplication order
    (03_generator_vc.cpp:549-608): pow2 = x*x; powN = pow_{N/2}*pow_{N-N/2},
    written x*(pow_{N-1}) when N/2 == 1."""
    out = []
    for n in pows:
        if n < 2:
            continue
        if n == 2:
            out.append(f"template<class R> {qual} R fdm_pow2(R x) {{ return x*x; }}")
            continue
        e0 = n // 2
        e1 = n - e0
        if e0 == 1:
            body = f"x*(fdm_pow{e1}(x))"
        else:
            body = f"fdm_pow{e0}(x)*fdm_pow{e1}(x)"
        out.append(f"template<class R> {qual} R fdm_pow{n}(R x) {{ return {body}; }}")
    return out


def variant_tag(params_alg: Sequence[int], params_const: Sequence[int]) -> str:
    a = "_".join(str(x) for x in params_alg) or "none"
    c = "_".join(str(x) for x in params_const) or "none"
    return f"a{a}_c{c}"


def _ident(model: Model) -> str:
    return re.sub(r"[^A-Za-z0-9_]", "_", model.name)


def _affine(e, consts):
    """e as (coefficients {(kind, idx): a}, constant b) if it is affine in STATES/PARAMS/VOI with numeric
    coefficients, else None (CONSTANTS count as numbers: they are folded)."""
    t = e[0]
    if t == "num":
        return {}, e[2]
    if t == "var":
        if e[1] == "C":
            return {}, consts[e[2]]
        if e[1] in ("S", "P", "T"):
            return {(e[1], e[2]): 1.0}, 0.0
        return None
    if t == "neg":
        a = _affine(e[1], consts)
        return None if a is None else ({k: -v for k, v in a[0].items()}, -a[1])
    if t == "pos":
        return _affine(e[1], consts)
    if t == "bin" and e[1] in "+-":
        a = _affine(e[2], consts)
        b = _affine(e[3], consts)
        if a is None or b is None:
            return None
        sg = 1.0 if e[1] == "+" else -1.0
        c = dict(a[0])
        for k, v in b[0].items():
            c[k] = c.get(k, 0.0) + sg * v
        return c, a[1] + sg * b[1]
    if t == "bin" and e[1] in "*/":
        a = _affine(e[2], consts)
        b = _affine(e[3], consts)
        if a is None or b is None:
            return None
        if e[1] == "*":
            if not a[0]:
                return {k: a[1] * v for k, v in b[0].items()}, a[1] * b[1]
            if not b[0]:
                return {k: b[1] * v for k, v in a[0].items()}, b[1] * a[1]
            return None
        if not b[0] and b[1] != 0.0:
            return {k: v / b[1] for k, v in a[0].items()}, a[1] / b[1]
        return None
    return None


def _exp_groups(lines, consts):
    """Exponentials whose arguments are affine in the same variables with the same coefficients, differing
    only by a constant: exp(a.x + b_k) = exp(a.x) * e^{b_k}.  Returns {repr(exp node): (group, b_k)} and the
    list of group (coefficients) of the groups with at least two distinct members."""
    found = {}

    def walk(e):
        t = e[0]
        if t == "call":
            if e[1] == "exp":
                af = _affine(e[2][0], consts)
                if af is not None and af[0]:
                    key = tuple(sorted((k, round(v, 15)) for k, v in af[0].items()))
                    found.setdefault(key, {})[repr(e)] = af[1]
            for a in e[2]:
                walk(a)
        elif t in ("neg", "pos", "not"):
            walk(e[1])
        elif t == "bin":
            walk(e[2])
            walk(e[3])
        elif t == "tern":
            walk(e[1])
            walk(e[2])
            walk(e[3])
    for _, _, e in lines:
        walk(e)
    repl = {}
    groups = []
    for key, members in found.items():
        if len(members) < 2:
            continue
        g = len(groups)
        groups.append(key)
        for r, b in members.items():
            repl[r] = (g, b)
    return repl, groups


_LOG2E = 1.4426950408889634
_LN2 = 0.6931471805599453


def _uses_algebraic(e) -> bool:
    t = e[0]
    if t == "var":
        return e[1] in ("A", "R")
    if t == "call":
        return any(_uses_algebraic(x) for x in e[2])
    if t in ("neg", "pos", "not"):
        return _uses_algebraic(e[1])
    if t == "bin":
        return _uses_algebraic(e[2]) or _uses_algebraic(e[3])
    if t == "tern":
        return any(_uses_algebraic(x) for x in e[1:4])
    return False


def _one_minus_exp(e, consts):
    """(sign, exp node) if e is 1 - exp(u) (sign +1) or exp(u) - 1 (sign -1), else None.  Such a difference is
    exactly 0 in FP32 wherever the SFU exponential rounds to 1 (|u| below about 2^-23): a removable singularity
    of the model (e.g. the Goldman-Hodgkin-Katz flux x / (1 - exp(-a x))) would become 0/0."""
    if e[0] != "bin" or e[1] != "-":
        return None
    for sign, one, ex in ((1, e[2], e[3]), (-1, e[3], e[2])):
        c = _affine(one, consts)
        if c is not None and not c[0] and c[1] == 1.0 and ex[0] == "call" and ex[1] == "exp":
            return sign, ex
    return None


def _unsafe_one_minus_exp(e, consts, repl) -> bool:
    """1 - exp(u) / exp(u) - 1 as the FP32 form would write it with a bare SFU exponential (not a shared
    exponential times a factor other than 1, which is one FMA and never exactly 0): see fdm_1mexp2."""
    om = _one_minus_exp(e, consts)
    if om is None:
        return False
    shared = repl.get(repr(om[1]))
    return shared is None or shared[1] == 0.0


def _batched_denominators(lines, consts, max_group: int = 3, repl=None):
    """Denominators of divisions that depend on states, parameters, time and constants only (no algebraic
    variables) and are not constants, in order of first appearance; grouped by max_group for a batched
    reciprocal (one SFU reciprocal per group, see fdm_rcp_batch)."""
    seen = []

    def walk(e):
        t = e[0]
        if t == "bin":
            if e[1] == "/":
                den = e[3]
                af = _affine(den, consts)
                # an unsafe 1 - exp(u) stays out: near u = 0 it is tiny, and a tiny factor would underflow the
                # group's product
                if (not (af is not None and not af[0]) and not _uses_algebraic(den) and repr(den) not in seen
                        and not _unsafe_one_minus_exp(den, consts, repl or {})):
                    seen.append(repr(den))
                    found.append(den)
            walk(e[2])
            walk(e[3])
        elif t == "call":
            for x in e[2]:
                walk(x)
        elif t in ("neg", "pos", "not"):
            walk(e[1])
        elif t == "tern":
            for x in e[1:4]:
                walk(x)
    found = []
    for _, _, e in lines:
        walk(e)
    groups = [found[i:i + max_group] for i in range(0, len(found), max_group)]
    return [g for g in groups if len(g) >= 2]


class _FastEmitter(_Emitter):
    """FP32 form of the right-hand side, written for the fewest instructions:
      - shared exponentials (see _exp_groups); every exponential one SFU ex2 of an argument whose log2(e)
        scaling and affine coefficients are folded at generation time; a positive constant factor of an
        exponential goes into its argument (c e^u = e^(u + ln c));
      - affine subexpressions c (x + k) as one fused multiply-add (c x + c k);
      - the gate form a (1 - s) - b s as a - (a + b) s;
      - divisions by constants as multiplications, other divisions as a multiplication by a reciprocal;
        denominators free of algebraic variables share one SFU reciprocal per group of up to three
        (fdm_rcp_batch: 1/d_k from 1/(d_0 d_1 d_2) and the other factors)."""

    def __init__(self, real, consts, repl, paired: bool = False, recip=None, alg_defs=None):
        super().__init__(real, consts, "cuda")
        self.repl = repl
        self.paired = paired        # fdm_f2 operands: conditional expressions become per-component selects
        self.recip = recip or {}    # repr(denominator) -> name of its batched reciprocal
        # paired form: definitions of the algebraic variables (index -> expression), for _folded_subtrahend
        self.alg_defs = alg_defs or {}

    def _folded_subtrahend(self, acc_text, b):
        """acc - b for an algebraic variable b defined as F (x + k) with one state or parameter x (a current
        F (V - E)): written F (-k - x) + acc, a packed subtraction and a packed FMA, the negation folded into
        the constant (packed instructions take no negated operand); None if b has no such form.  For HH this
        left the FP32 results bit for bit as they were and took one instruction per current off each
        right-hand side"""
        if not self.paired or b[0] != "var" or b[1] != "A" or b[2] not in self.alg_defs:
            return None
        d = self.alg_defs[b[2]]
        if d[0] != "bin" or d[1] != "*":
            return None
        for f_side, g_side in ((d[2], d[3]), (d[3], d[2])):
            g = _affine(g_side, self.consts)
            if g is None or len(g[0]) != 1 or _affine(f_side, self.consts) is not None:
                continue
            (x_key, coef), = g[0].items()
            if coef not in (1.0, -1.0):
                continue
            x = self.var(x_key[0], x_key[1])
            k = g[1]
            neg_g = (f"((({self.real}){_hexf(-k)}) - {x})" if coef == 1.0
                     else f"({x} + (({self.real}){_hexf(-k)}))")
            return f"(({self.expr(f_side)}) * {neg_g} + {acc_text})"
        return None

    def coef_text(self, v, x):
        if v == 1.0:
            return x
        if v == -1.0:
            return f"(-{x})"
        return f"(({self.real}){_hexf(v)}) * {x}"

    def affine_text(self, coeffs, const, scale):
        terms = [self.coef_text(v * scale, self.var(k[0], k[1])) for k, v in coeffs]
        if const != 0.0:
            terms.append(f"(({self.real}){_hexf(const * scale)})")
        return " + ".join(terms) if terms else f"(({self.real})0)"

    def _positive_const(self, e):
        af = _affine(e, self.consts)
        if af is not None and not af[0] and af[1] > 0.0:
            return af[1]
        return None

    def exp_text(self, e, factor: float = 1.0):
        """factor * exp(arg) for the exp call node e (factor > 0)"""
        if repr(e) in self.repl:
            g, b = self.repl[repr(e)]
            return f"(fdm_e{g} * (({self.real}){_hexf(math.exp(b) * factor)}))"
        af = _affine(e[2][0], self.consts)
        if af is not None:
            return f"fdm_ex2({self.affine_text(sorted(af[0].items()), af[1] + math.log(factor), _LOG2E)})"
        arg = f"(({self.real}){_hexf(_LOG2E)}) * {self.expr(e[2][0])}"
        if factor != 1.0:
            arg = f"{arg} + (({self.real}){_hexf(math.log(factor) * _LOG2E)})"
        return f"fdm_ex2({arg})"

    def expr(self, e):
        t = e[0]
        if t == "call" and e[1] == "exp":
            return self.exp_text(e)
        if t == "call" and e[1] == "log":
            return f"(fdm_lg2({self.expr(e[2][0])}) * (({self.real}){_hexf(_LN2)}))"
        if t == "bin" and e[1] == "*":
            for c_side, x_side in ((e[2], e[3]), (e[3], e[2])):
                c = self._positive_const(c_side)
                if c is not None and x_side[0] == "call" and x_side[1] == "exp":
                    return self.exp_text(x_side, c)
        if (t == "bin" and e[1] in "*/") or t == "neg":
            af = _affine(e, self.consts)
            if af is not None and af[0]:
                return f"({self.affine_text(sorted(af[0].items()), af[1], 1.0)})"
        if t == "neg":
            return self.neg_text(e[1])
        if t == "bin" and e[1] == "-":
            # 1 - exp(u), exp(u) - 1: formed without cancellation and never exactly 0 (fdm_1mexp2), unless the
            # exponential is a shared one with a factor other than 1 (then e * c - 1 is one FMA, not exactly 0)
            if _unsafe_one_minus_exp(e, self.consts, self.repl):
                sign, ex = _one_minus_exp(e, self.consts)
                af = _affine(ex[2][0], self.consts)
                arg = (self.affine_text(sorted(af[0].items()), af[1], _LOG2E) if af is not None
                       else f"(({self.real}){_hexf(_LOG2E)}) * {self.expr(ex[2][0])}")
                return f"fdm_1mexp2({arg})" if sign > 0 else f"(-fdm_1mexp2({arg}))"
        if t == "bin" and e[1] == "-":
            # x - c for a constant c: x + (-c), so that a product x = a b fuses with it
            c = _affine(e[3], self.consts)
            if c is not None and not c[0] and not (e[2][0] == "var" or _affine(e[2], self.consts) is not None):
                return f"({self.expr(e[2])} + (({self.real}){_hexf(-c[1])}))"
        if t == "bin" and e[1] == "-":
            # a (1 - s) - b s  ->  a - (a + b) s, for variables a, b, s
            l, r = e[2], e[3]
            if l[0] == "bin" and l[1] == "*" and r[0] == "bin" and r[1] == "*":
                a, one_minus = l[2], l[3]
                b, s2 = r[2], r[3]
                if (one_minus[0] == "bin" and one_minus[1] == "-" and _affine(one_minus[2], self.consts) == ({}, 1.0)
                        and a[0] == "var" and b[0] == "var" and s2[0] == "var" and repr(one_minus[3]) == repr(s2)):
                    A, B, S = self.expr(a), self.expr(b), self.expr(s2)
                    return f"({A} - ({A} + {B}) * {S})"
            folded = self._folded_subtrahend(self.expr(l), r)
            if folded is not None:
                return folded
        if t == "bin" and e[1] == "/":
            den = _affine(e[3], self.consts)
            if den is not None and not den[0] and den[1] != 0.0:
                if den[1] == 1.0:
                    return self.expr(e[2])
                return f"({self.expr(e[2])} * (({self.real}){_hexf(1.0 / den[1])}))"
            num = _affine(e[2], self.consts)
            inv = self.recip.get(repr(e[3])) or f"fdm_rcp({self.expr(e[3])})"
            if num is not None and not num[0] and num[1] == 1.0:
                return inv
            return f"({self.expr(e[2])} * {inv})"
        if t == "tern" and self.paired:
            return f"fdm_sel({self.expr(e[1])}, {self.expr(e[2])}, {self.expr(e[3])})"
        return super().expr(e)

    def neg_text(self, e):
        """-(e) with the negation pushed through sums to a single leaf: -((a + b) - c) = (-a - b) + c"""
        t = e[0]
        if t == "neg":
            return self.expr(e[1])
        if t == "bin" and e[1] == "+":
            folded = self._folded_subtrahend(self.neg_text(e[2]), e[3])
            if folded is not None:
                return folded
            return f"({self.neg_text(e[2])} - {self.expr(e[3])})"
        if t == "bin" and e[1] == "-":
            return f"({self.neg_text(e[2])} + {self.expr(e[3])})"
        return f"(-{self.expr(e)})"

    def batch_lines(self, groups):
        """Declarations of the batched reciprocals (after the shared exponentials); fills self.recip."""
        out = []
        k = 0
        for g in groups:
            names = []
            for den in g:
                out.append(f"    const R fdm_d{k} = {self.expr(den)};")
                names.append(k)
                k += 1
            out.append("    R " + ", ".join(f"fdm_r{j}" for j in names) + ";")
            args = ", ".join(f"fdm_d{j}" for j in names) + ", " + ", ".join(f"fdm_r{j}" for j in names)
            out.append(f"    fdm_rcp_batch({args});")
            for j, den in zip(names, g):
                self.recip[repr(den)] = f"fdm_r{j}"
        return out


def emit_cuda_model(model: Model, params_alg: Sequence[int], params_const: Sequence[int]) -> str:
    """CUDA device right-hand side for one parameter variant.

    The struct exposes ``rates<R, M>(VOI, STATES, PARAMS, RATES, ALGEBRAIC)``; R is
    the arithmetic type and M a math policy providing exp / log / pow.
    """
    lines = substitute_parameters(model, params_alg, params_const)
    em = _Emitter("R", model.constants, "cuda")
    ident = _ident(model)
    tag = variant_tag(params_alg, params_const)
    pows = _collect_int_pows(lines)
    n_params = len(params_alg) + len(params_const)
    out = []
    out.append("// Generated by opendihu_b200/cellml.py from the OpenCOR C export "
               f"{os.path.basename(model.source)}; do not edit.")
    out.append(f"// parametersUsedAsAlgebraic = {list(params_alg)}, parametersUsedAsConstant = {list(params_const)}")
    out.append("#pragma once")
    out.append('#include "../fdm_math.cuh"')
    out.append("")
    out.append(f"struct fdm_model_{ident}_{tag} {{")
    out.append(f"  static constexpr int nStates = {model.n_states};")
    out.append(f"  static constexpr int nAlgebraics = {model.n_algebraics};")
    out.append(f"  static constexpr int nParameters = {n_params};")
    out.append(f"  static constexpr bool usesTime = {'true' if model.uses_voi else 'false'};")
    out.append(f"  static constexpr const char* name = \"{model.name}\";")
    out.append(f"  static constexpr double statesInitialValues[{model.n_states}] = {{"
               + ", ".join(_hexf(v) for v in model.states_initial) + "};")
    defaults = [0.0] * len(params_alg) + [model.constants[c] for c in params_const]
    out.append(f"  static constexpr double parameterDefaults[{max(n_params, 1)}] = {{"
               + ", ".join(_hexf(v) for v in (defaults or [0.0])) + "};")
    out.extend("  " + s for s in _pow_helpers(pows, "__device__ __forceinline__ static"))
    out.append("  template<class R, class M>")
    out.append("  __device__ __forceinline__ static void rates(const R VOI, const R* __restrict__ STATES,"
               " const R* __restrict__ PARAMS, R* __restrict__ RATES, R* __restrict__ ALGEBRAIC)")
    out.append("  {")
    out.append("    (void)VOI; (void)PARAMS;")
    out.append("#define FDM_EXP(x) M::exp(x)")
    out.append("#define FDM_LOG(x) M::log(x)")
    out.append("#define FDM_POWF(x, y) M::pow(x, y)")
    out.append("#define FDM_ABS(x) fabs(x)")
    out.append("#define FDM_SQRT(x) sqrt(x)")
    out.extend("#define " + s.split("#define ", 1)[1] for s in _pow_macro_defs(pows))
    for kind, idx, expr in lines:
        tgt = f"ALGEBRAIC[{idx}]" if kind == "A" else f"RATES[{idx}]"
        out.append(f"    {tgt} = {em.expr(expr)};")
    for n in pows:
        out.append(f"#undef FDM_POW{n}")
    out.append("#undef FDM_EXP\n#undef FDM_LOG\n#undef FDM_POWF\n#undef FDM_ABS\n#undef FDM_SQRT")
    out.append("  }")
    # FP32 variant with shared exponentials
    repl, groups = _exp_groups(lines, model.constants)
    rgroups = _batched_denominators(lines, model.constants, repl=repl)
    fem = _FastEmitter("R", model.constants, repl)
    out.append("  // FP32 form: exponentials exp(a.x + b_k) that share a.x are evaluated once as exp(a.x) * e^{b_k};")
    out.append("  // exponentials, logarithms and reciprocals as single SFU instructions (fdm_ex2/fdm_lg2/fdm_rcp)")
    out.append(f"  static constexpr int nSharedExponentials = {len(groups)};")
    out.append("  template<class R, class M>")
    out.append("  __device__ __forceinline__ static void rates_fast(const R VOI, const R* __restrict__ STATES,"
               " const R* __restrict__ PARAMS, R* __restrict__ RATES, R* __restrict__ ALGEBRAIC)")
    out.append("  {")
    out.append("    (void)VOI; (void)PARAMS;")
    out.append("#define FDM_EXP(x) M::exp(x)")
    out.append("#define FDM_LOG(x) M::log(x)")
    out.append("#define FDM_POWF(x, y) M::pow(x, y)")
    out.append("#define FDM_ABS(x) fabs(x)")
    out.append("#define FDM_SQRT(x) sqrt(x)")
    out.extend("#define " + s2.split("#define ", 1)[1] for s2 in _pow_macro_defs(pows))
    for g, key in enumerate(groups):
        out.append(f"    const R fdm_e{g} = fdm_ex2({fem.affine_text(list(key), 0.0, _LOG2E)});")
    out.extend(fem.batch_lines(rgroups))
    for kind, idx, expr in lines:
        tgt = f"ALGEBRAIC[{idx}]" if kind == "A" else f"RATES[{idx}]"
        out.append(f"    {tgt} = {fem.expr(expr)};")
    for n in pows:
        out.append(f"#undef FDM_POW{n}")
    out.append("#undef FDM_EXP\n#undef FDM_LOG\n#undef FDM_POWF\n#undef FDM_ABS\n#undef FDM_SQRT")
    out.append("  }")
    # the same FP32 form over node pairs (packed FP32 instructions)
    fem2 = _FastEmitter("R", model.constants, repl, paired=True,
                        alg_defs={idx: expr for kind, idx, expr in lines if kind == "A"})
    out.append("  // paired FP32 form: the FP32 form over two nodes at once (fdm_f2, packed FP32 instructions)")
    out.append("  template<class M>")
    out.append("  __device__ __forceinline__ static void rates_fast2(const fdm_f2 VOI, const fdm_f2* __restrict__ STATES,"
               " const fdm_f2* __restrict__ PARAMS, fdm_f2* __restrict__ RATES, fdm_f2* __restrict__ ALGEBRAIC)")
    out.append("  {")
    out.append("    typedef fdm_f2 R;")
    out.append("    (void)VOI; (void)PARAMS;")
    out.append("#define FDM_POWF(x, y) fdm_powf_pair(x, y)")
    out.append("#define FDM_ABS(x) fabs(x)")
    out.append("#define FDM_SQRT(x) sqrt(x)")
    out.extend("#define " + s2.split("#define ", 1)[1] for s2 in _pow_macro_defs(pows))
    for g, key in enumerate(groups):
        out.append(f"    const R fdm_e{g} = fdm_ex2({fem2.affine_text(list(key), 0.0, _LOG2E)});")
    out.extend(fem2.batch_lines(rgroups))
    for kind, idx, expr in lines:
        tgt = f"ALGEBRAIC[{idx}]" if kind == "A" else f"RATES[{idx}]"
        out.append(f"    {tgt} = {fem2.expr(expr)};")
    for n in pows:
        out.append(f"#undef FDM_POW{n}")
    out.append("#undef FDM_POWF\n#undef FDM_ABS\n#undef FDM_SQRT")
    out.append("  }")
    # the right-hand side split by state (few-node reaction kernel)
    out.append("  // the right-hand side of one state at a time: rates_group<R, M, G> = RATES[G]")
    out.extend(emit_group_rates(model, params_alg, params_const))
    # reverse mode (adjoint)
    out.append("  // vector-Jacobian product: LAM_STATES += J^T LAM_RATES, LAM_PARAMS += (dRATES/dPARAMS)^T LAM_RATES")
    out.extend(emit_cuda_vjp(model, params_alg, params_const))
    out.append("  // the same in the fast form (exact exponentials): shared exponentials, reciprocals")
    out.extend(emit_cuda_vjp(model, params_alg, params_const, fast=True))
    out.append("};")
    out.append("")
    return "\n".join(out)


def _algebraic_reads(e, out: set):
    t = e[0]
    if t == "var":
        if e[1] == "A":
            out.add(e[2])
    elif t in ("neg", "pos", "not"):
        _algebraic_reads(e[1], out)
    elif t == "bin":
        _algebraic_reads(e[2], out)
        _algebraic_reads(e[3], out)
    elif t == "tern":
        for k in (1, 2, 3):
            _algebraic_reads(e[k], out)
    elif t == "call":
        for a in e[2]:
            _algebraic_reads(a, out)


def rate_cone(lines, states: Sequence[int]) -> List[int]:
    """Indices (into lines, in their order) of the lines the rates of the given states need: their RATES lines
    and, transitively, the ALGEBRAIC lines those read."""
    where = {(k, i): n for n, (k, i, _) in enumerate(lines)}
    need, stack = set(), [where[("R", s)] for s in states if ("R", s) in where]
    while stack:
        n = stack.pop()
        if n in need:
            continue
        need.add(n)
        reads = set()
        _algebraic_reads(lines[n][2], reads)
        stack.extend(where[("A", a)] for a in reads if ("A", a) in where)
    return sorted(need)


#: models with at most this many states get the state-group form (one warp per state of the node group)
MAX_GROUP_STATES = 8


def emit_group_rates(model: Model, params_alg: Sequence[int], params_const: Sequence[int]) -> List[str]:
    """The right-hand side split by state: ``rates_group<R, M, G>`` computes RATES[G] only, from the lines its
    cone needs, so that the warps of a node group can each evaluate one state's rate (the reaction kernel for
    few nodes, where one thread per node leaves the SMs short of independent work).  Same expressions as
    ``rates``, so the same values."""
    lines = substitute_parameters(model, params_alg, params_const)
    em = _Emitter("R", model.constants, "cuda")
    pows = _collect_int_pows(lines)
    out = [f"  static constexpr int nGroups = {model.n_states if model.n_states <= MAX_GROUP_STATES else 0};"]
    if model.n_states > MAX_GROUP_STATES:
        return out
    out.append("  template<class R, class M, int G>")
    out.append("  __device__ __forceinline__ static R rates_group(const R VOI, const R* __restrict__ STATES,"
               " const R* __restrict__ PARAMS)")
    out.append("  {")
    out.append("    (void)VOI; (void)PARAMS;")
    out.append(f"    R ALGEBRAIC[{max(model.n_algebraics, 1)}];")
    out.append("    (void)ALGEBRAIC;")
    out.append("#define FDM_EXP(x) M::exp(x)")
    out.append("#define FDM_LOG(x) M::log(x)")
    out.append("#define FDM_POWF(x, y) M::pow(x, y)")
    out.append("#define FDM_ABS(x) fabs(x)")
    out.append("#define FDM_SQRT(x) sqrt(x)")
    out.extend("#define " + s2.split("#define ", 1)[1] for s2 in _pow_macro_defs(pows))
    for g in range(model.n_states):
        out.append(f"    {'if' if g == 0 else 'else if'} constexpr (G == {g}) {{")
        rate = None
        for n in rate_cone(lines, [g]):
            kind, idx, expr = lines[n]
            if kind == "A":
                out.append(f"      ALGEBRAIC[{idx}] = {em.expr(expr)};")
            else:
                rate = em.expr(expr)
        out.append(f"      return {rate if rate is not None else '(R)0'};")
        out.append("    }")
    out.append("    else {")
    out.append("      return (R)0;")
    out.append("    }")
    for n in pows:
        out.append(f"#undef FDM_POW{n}")
    out.append("#undef FDM_EXP\n#undef FDM_LOG\n#undef FDM_POWF\n#undef FDM_ABS\n#undef FDM_SQRT")
    out.append("  }")
    return out


def emit_c_model(model: Model, params_alg: Sequence[int], params_const: Sequence[int]) -> str:
    """Scalar C right-hand side for the CPU oracle (same expression trees)."""
    lines = substitute_parameters(model, params_alg, params_const)
    em = _Emitter("double", model.constants, "c")
    ident = _ident(model)
    tag = variant_tag(params_alg, params_const)
    pows = _collect_int_pows(lines)
    out = []
    out.append("/* Generated by opendihu_b200/cellml.py from the OpenCOR C export "
               f"{os.path.basename(model.source)}; do not edit. */")
    out.append(f"/* parametersUsedAsAlgebraic = {list(params_alg)}, parametersUsedAsConstant = {list(params_const)} */")
    out.append("#pragma once")
    out.append('#include "../oracle_math.h"')
    for n in pows:
        if n < 2:
            continue
        if n == 2:
            out.append(f"static inline double oracle_{ident}_{tag}_pow2(double x) {{ return x*x; }}")
        else:
            e0 = n // 2
            e1 = n - e0
            if e0 == 1:
                body = f"x*(oracle_{ident}_{tag}_pow{e1}(x))"
            else:
                body = f"oracle_{ident}_{tag}_pow{e0}(x)*oracle_{ident}_{tag}_pow{e1}(x)"
            out.append(f"static inline double oracle_{ident}_{tag}_pow{n}(double x) {{ return {body}; }}")
    out.append(f"#define ORACLE_{ident.upper()}_{tag.upper()}_N_STATES {model.n_states}")
    out.append(f"#define ORACLE_{ident.upper()}_{tag.upper()}_N_ALGEBRAICS {model.n_algebraics}")
    out.append(f"#define ORACLE_{ident.upper()}_{tag.upper()}_N_PARAMETERS {len(params_alg) + len(params_const)}")
    out.append(f"static void oracle_{ident}_{tag}_rates(double VOI, const double *STATES, const double *PARAMS,"
               f" double *RATES, double *ALGEBRAIC, int approx)")
    out.append("{")
    out.append("  (void)VOI; (void)PARAMS;")
    out.append("#define FDM_EXP(x) (approx ? oracle_approx_exp(x) : exp(x))")
    out.append("#define FDM_LOG(x) (approx ? oracle_approx_log(x) : log(x))")
    out.append("#define FDM_POWF(x, y) pow(x, y)")
    out.append("#define FDM_ABS(x) fabs(x)")
    out.append("#define FDM_SQRT(x) sqrt(x)")
    for n in pows:
        if n == 1:
            out.append("#define FDM_POW1(x) (x)")
        else:
            out.append(f"#define FDM_POW{n}(x) oracle_{ident}_{tag}_pow{n}(x)")
    for kind, idx, expr in lines:
        tgt = f"ALGEBRAIC[{idx}]" if kind == "A" else f"RATES[{idx}]"
        out.append(f"  {tgt} = {em.expr(expr)};")
    for n in pows:
        out.append(f"#undef FDM_POW{n}")
    out.append("#undef FDM_EXP\n#undef FDM_LOG\n#undef FDM_POWF\n#undef FDM_ABS\n#undef FDM_SQRT")
    out.append("}")
    out.append(f"static const double oracle_{ident}_{tag}_states_initial[{model.n_states}] = {{"
               + ", ".join(_hexf(v) for v in model.states_initial) + "};")
    out.append("")
    return "\n".join(out)


# ----------------------------------------------------------------------------------------------
# the prebuilt variants
# ----------------------------------------------------------------------------------------------

#: (model file basename, parametersUsedAsAlgebraic, parametersUsedAsConstant) compiled into the
#: library.  A settings dict may use any subset of a variant's constant parameters (the unused
#: slots are filled with the constants' raw values, which gives identical arithmetic).
VARIANTS = [
    ("hodgkin_huxley_1952.c", (), (2, 3, 4)),
    ("shorten_ocallaghan_davidson_soboleva_2007.c", (32,), (65,)),
]


def _tree_to_json(e):
    """Expression tree as nested lists (numbers keep their literal text)."""
    if e[0] == "num":
        return ["num", e[1]]
    if e[0] == "var":
        return ["var", e[1], e[2]]
    if e[0] in ("neg", "pos", "not"):
        return [e[0], _tree_to_json(e[1])]
    if e[0] == "bin":
        return ["bin", e[1], _tree_to_json(e[2]), _tree_to_json(e[3])]
    if e[0] == "tern":
        return ["tern", _tree_to_json(e[1]), _tree_to_json(e[2]), _tree_to_json(e[3])]
    if e[0] == "call":
        return ["call", e[1], [_tree_to_json(a) for a in e[2]]]
    raise ValueError(e)


def tree_from_json(j):
    """Inverse of _tree_to_json (numbers get their double value back)."""
    t = j[0]
    if t == "num":
        return ("num", j[1], float(j[1]))
    if t == "var":
        return ("var", j[1], j[2])
    if t in ("neg", "pos", "not"):
        return (t, tree_from_json(j[1]))
    if t == "bin":
        return ("bin", j[1], tree_from_json(j[2]), tree_from_json(j[3]))
    if t == "tern":
        return ("tern", tree_from_json(j[1]), tree_from_json(j[2]), tree_from_json(j[3]))
    if t == "call":
        return ("call", j[1], [tree_from_json(a) for a in j[2]])
    raise ValueError(j)


def model_to_json(model: Model) -> dict:
    """The parsed model (its equations as expression trees, initial values, names) as plain JSON data."""
    return {"name": model.name, "source": os.path.basename(model.source), "n_states": model.n_states,
            "n_algebraics": model.n_algebraics, "n_constants": model.n_constants,
            "states_initial": model.states_initial, "state_names": model.state_names,
            "algebraic_names": model.algebraic_names, "constant_names": model.constant_names,
            "uses_voi": model.uses_voi,
            "constant_lines": [[i, _tree_to_json(e)] for i, e in model.constant_lines],
            "lines": [[k, i, _tree_to_json(e)] for k, i, e in model.lines]}


def model_from_json(j: dict) -> Model:
    """Inverse of model_to_json: the constants are folded again from their assignments, in IEEE double."""
    constant_lines = [(int(i), tree_from_json(e)) for i, e in j["constant_lines"]]
    consts = [0.0] * int(j["n_constants"])
    env = {"S": list(j["states_initial"]), "C": consts, "A": [], "R": [], "T": 0.0}
    for idx, expr in constant_lines:
        consts[idx] = eval_expr(expr, env)
    return Model(name=j["name"], source=j["source"], n_states=int(j["n_states"]),
                 n_algebraics=int(j["n_algebraics"]), n_constants=int(j["n_constants"]),
                 states_initial=[float(x) for x in j["states_initial"]], constants=consts,
                 constant_lines=constant_lines, lines=[(k, int(i), tree_from_json(e)) for k, i, e in j["lines"]],
                 state_names=list(j["state_names"]), algebraic_names=list(j["algebraic_names"]),
                 constant_names=list(j["constant_names"]), uses_voi=bool(j["uses_voi"]))


def builtin_model(name: str) -> Model:
    """A built-in model (one the library carries generated code for), from its generated description."""
    gen = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "generated")
    for fname, pa, pc in VARIANTS:
        if os.path.splitext(fname)[0] == name:
            with open(os.path.join(gen, f"{name}_{variant_tag(pa, pc)}.json")) as f:
                return model_from_json(__import__("json").load(f)["model"])
    raise KeyError(name)


def generate_all(input_dir: str, cuda_dir: str, c_dir: str) -> List[str]:
    """(Re)generate the device and oracle model sources for every prebuilt variant."""
    written = []
    for fname, pa, pc in VARIANTS:
        model = parse_model_file(os.path.join(input_dir, fname))
        tag = variant_tag(pa, pc)
        for text, d, ext in ((emit_cuda_model(model, pa, pc), cuda_dir, ".cuh"),
                             (emit_c_model(model, pa, pc), c_dir, ".h")):
            path = os.path.join(d, f"{_ident(model)}_{tag}{ext}")
            with open(path, "w") as f:
                f.write(text)
            written.append(path)
        # names and initial values, used by the host to describe the model
        meta = os.path.join(cuda_dir, f"{_ident(model)}_{tag}.json")
        import json
        with open(meta, "w") as f:
            json.dump({"name": model.name, "source": fname, "n_states": model.n_states,
                       "n_algebraics": model.n_algebraics, "n_constants": model.n_constants,
                       "parametersUsedAsAlgebraic": list(pa), "parametersUsedAsConstant": list(pc),
                       "states_initial": model.states_initial,
                       "constants": model.constants,
                       "state_names": model.state_names, "algebraic_names": model.algebraic_names,
                       "constant_names": model.constant_names, "uses_time": model.uses_voi,
                       "operations_per_rhs": count_operations(model, pa, pc),
                       "rhs_lines": [[k, i, _tree_to_json(e)] for k, i, e in substitute_parameters(model, pa, pc)],
                       # the model as parsed, before any parameter substitution: other parameter variants are
                       # generated from it at run time (opendihu_b200/models.py)
                       "model": model_to_json(model)},
                      f, indent=1)
        written.append(meta)
    return written


# ----------------------------------------------------------------------------------------------
# operation counts (algorithmic work of one right-hand side evaluation)
# ----------------------------------------------------------------------------------------------

def count_operations(model: Model, params_alg: Sequence[int] = (), params_const: Sequence[int] = ()) -> Dict[str, int]:
    """Arithmetic operations of one right-hand side evaluation: ``flops`` (+, -, *, / and the
    multiplications of integer powers; a negation counts as one) and ``special`` (exp, log, pow
    with a non-integer exponent)."""
    lines = substitute_parameters(model, params_alg, params_const)
    c = {"flops": 0, "div": 0, "special": 0}

    def walk(e):
        t = e[0]
        if t in ("num", "var"):
            return
        if t in ("neg", "pos", "not"):
            c["flops"] += 1 if t == "neg" else 0
            walk(e[1])
            return
        if t == "bin":
            if e[1] in "+-*/":
                c["flops"] += 1
                if e[1] == "/":
                    c["div"] += 1
            walk(e[2])
            walk(e[3])
            return
        if t == "tern":
            walk(e[1])
            walk(e[2])
            walk(e[3])
            return
        if t == "call":
            if e[1] == "pow":
                n = _int_exponent(e[2][1])
                if n is not None:
                    k = abs(n)
                    c["flops"] += max(k - 1, 0) + (1 if n < 0 else 0)
                    if n < 0:
                        c["div"] += 1
                    walk(e[2][0])
                    return
            if e[1] in ("exp", "log", "pow"):
                c["special"] += 1
            for a in e[2]:
                walk(a)
            return
    for _, _, e in lines:
        walk(e)
    return c


# ----------------------------------------------------------------------------------------------
# reverse mode: vector-Jacobian product of the right-hand side (for the hand-written adjoint)
# ----------------------------------------------------------------------------------------------

class _VjpBuilder:
    """Straight-line forward code with one temporary per operation, then the adjoint accumulation in
    reverse order (classic reverse-mode differentiation of the expression DAG)."""

    def __init__(self, consts, real="R", repl=None, groups=None):
        self.consts = consts
        self.real = real
        self.fwd: List[str] = []
        self.ops: List[tuple] = []     # (temp name, op, operands, extra)
        self.alg_temp: Dict[int, str] = {}
        self.rate_temp: Dict[int, str] = {}
        self.n = 0
        self.plain = _Emitter(real, consts, "cuda")
        # fast form (exact exponentials only): shared exponentials exp(a.x + b) = exp(a.x) e^b
        # (repl/groups from _exp_groups), divisions by constants as multiplications, one reciprocal per
        # division by a variable (its derivative -1/d^2 from the same reciprocal)
        self.fast = repl is not None
        self.repl = repl or {}
        self.groups = groups or []
        self.group_temp: Dict[int, tuple] = {}

    def lit(self, v):
        return ("lit", f"(({self.real}){_hexf(v)})", None)

    def leaf(self, e):
        t = e[0]
        if t == "num":
            return ("lit", f"(({self.real}){e[1]})", None)
        k, i = e[1], e[2]
        if k == "C":
            return self.lit(self.consts[i])
        if k == "S":
            return ("ref", f"STATES[{i}]", f"LAM_STATES[{i}]")
        if k == "P":
            return ("ref", f"PARAMS[{i}]", f"LAM_PARAMS[{i}]")
        if k == "T":
            return ("ref", "VOI", None)
        if k == "A":
            tn = self.alg_temp[i]
            return ("ref", tn, "a_" + tn)
        if k == "R":
            tn = self.rate_temp[i]
            return ("ref", tn, "a_" + tn)
        raise ValueError(e)

    def temp(self, op, operands, expr_text, extra=None):
        name = f"t{self.n}"
        self.n += 1
        self.fwd.append(f"    const {self.real} {name} = {expr_text};")
        self.ops.append((name, op, operands, extra))
        return ("ref", name, "a_" + name)

    def build(self, e):
        t = e[0]
        if t in ("num", "var"):
            return self.leaf(e)
        if t == "pos":
            return self.build(e[1])
        if t == "neg":
            a = self.build(e[1])
            return self.temp("neg", [a], f"(-{a[1]})")
        if t == "bin":
            op = e[1]
            if op == "/" and self.fast:
                a = self.build(e[2])
                den = _affine(e[3], self.consts)
                if den is not None and not den[0] and den[1] != 0.0:
                    c = self.lit(1.0 / den[1])
                    return self.temp("*", [a, c], f"({a[1]} * {c[1]})")
                b = self.build(e[3])
                r = self.temp("rcp", [b], f"((({self.real})1) / {b[1]})")
                return self.temp("*", [a, r], f"({a[1]} * {r[1]})")
            if op in "+-*/":
                a = self.build(e[2])
                b = self.build(e[3])
                return self.temp(op, [a, b], f"({a[1]} {op} {b[1]})")
            raise ValueError("comparison outside a condition")
        if t == "tern":
            cond = self.plain.expr(e[1]).replace("ALGEBRAIC[", "ALG[")
            a = self.build(e[2])
            b = self.build(e[3])
            cname = f"c{self.n}"
            self.fwd.append(f"    const bool {cname} = ({cond});")
            return self.temp("tern", [a, b], f"({cname} ? {a[1]} : {b[1]})", cname)
        if t == "call":
            f = e[1]
            if f == "pow":
                n = _int_exponent(e[2][1])
                a = self.build(e[2][0])
                if n is not None:
                    if n > 0:
                        return self.temp(("powi", n), [a], f"FDM_POW{n}({a[1]})")
                    return self.temp(("powi", n), [a], f"(({self.real})1.0/FDM_POW{-n}({a[1]}))")
                b = self.build(e[2][1])
                return self.temp("pow", [a, b], f"M::pow({a[1]}, {b[1]})")
            if f == "exp" and repr(e) in self.repl:
                g, off = self.repl[repr(e)]
                if g not in self.group_temp:
                    arg = None
                    for (kind, idx), coef in self.groups[g]:
                        term = ("bin", "*", ("num", _hexf(coef), coef), ("var", kind, idx))
                        arg = term if arg is None else ("bin", "+", arg, term)
                    x = self.build(arg)
                    self.group_temp[g] = self.temp("exp", [x], f"M::exp({x[1]})")
                ge = self.group_temp[g]
                c = self.lit(math.exp(off))
                return self.temp("*", [ge, c], f"({ge[1]} * {c[1]})")
            a = self.build(e[2][0])
            if f == "exp":
                return self.temp("exp", [a], f"M::exp({a[1]})")
            if f == "log":
                return self.temp("log", [a], f"M::log({a[1]})")
            if f == "fabs":
                return self.temp("fabs", [a], f"fabs({a[1]})")
            if f == "sqrt":
                return self.temp("sqrt", [a], f"sqrt({a[1]})")
        raise ValueError(f"unsupported node {e}")

    def backward(self):
        out = []
        R = self.real
        for name, op, ops, extra in reversed(self.ops):
            a = "a_" + name

            def acc(o, term):
                if o[2] is not None:
                    out.append(f"    {o[2]} += {term};")
            if op == "+":
                acc(ops[0], a)
                acc(ops[1], a)
            elif op == "-":
                acc(ops[0], a)
                acc(ops[1], f"-{a}")
            elif op == "*":
                acc(ops[0], f"{a} * {ops[1][1]}")
                acc(ops[1], f"{a} * {ops[0][1]}")
            elif op == "/":
                acc(ops[0], f"{a} / {ops[1][1]}")
                acc(ops[1], f"-{a} * {name} / {ops[1][1]}")
            elif op == "rcp":
                acc(ops[0], f"-{a} * {name} * {name}")
            elif op == "neg":
                acc(ops[0], f"-{a}")
            elif op == "exp":
                acc(ops[0], f"{a} * M::dexp({ops[0][1]}, {name})")
            elif op == "log":
                acc(ops[0], f"{a} * M::dlog({ops[0][1]}, {name})")
            elif op == "fabs":
                acc(ops[0], f"({ops[0][1]} >= ({R})0 ? {a} : -{a})")
            elif op == "sqrt":
                acc(ops[0], f"{a} * ({R})0.5 / {name}")
            elif op == "pow":
                acc(ops[0], f"{a} * {ops[1][1]} * {name} / {ops[0][1]}")
                acc(ops[1], f"{a} * {name} * M::log({ops[0][1]})")
            elif op == "tern":
                acc(ops[0], f"({extra} ? {a} : ({R})0)")
                acc(ops[1], f"({extra} ? ({R})0 : {a})")
            elif isinstance(op, tuple) and op[0] == "powi":
                n = op[1]
                x = ops[0][1]
                if n > 0:
                    d = f"(({R}){n})" if n == 1 else (f"(({R}){n} * {x})" if n == 2 else f"(({R}){n} * FDM_POW{n - 1}({x}))")
                    if n == 1:
                        d = f"(({R})1)"
                    acc(ops[0], f"{a} * {d}")
                else:
                    acc(ops[0], f"{a} * (({R}){n}) * {name} / {x}")
            else:
                raise ValueError(op)
        return out


def emit_cuda_vjp(model: Model, params_alg: Sequence[int], params_const: Sequence[int], fast: bool = False) -> List[str]:
    """Lines of the member function ``rates_vjp<R, M>`` (to be placed inside the model struct):
    given STATES, PARAMS and LAM_RATES it evaluates the right-hand side and adds J^T LAM_RATES to
    LAM_STATES and (dRATES/dPARAMS)^T LAM_RATES to LAM_PARAMS; ``rates_tape`` / ``rates_vjp_tape``
    split it in a recording forward and a backward.  ``fast``: the same functions with the suffix
    ``_fast`` in the fast form of _VjpBuilder (shared exponentials, reciprocals; exact exponentials)."""
    lines = substitute_parameters(model, params_alg, params_const)
    sfx = "_fast" if fast else ""
    if fast:
        repl, groups = _exp_groups(lines, model.constants)
        b = _VjpBuilder(model.constants, repl=repl, groups=groups)
    else:
        b = _VjpBuilder(model.constants)
    for kind, idx, expr in lines:
        r = b.build(expr)
        if r[0] == "lit" or (r[0] == "ref" and not r[1].startswith("t")):
            r = b.temp("+", [r, b.lit(0.0)], f"({r[1]} + (({b.real})0))")
        if kind == "A":
            b.alg_temp[idx] = r[1]
            b.fwd.append(f"    ALG[{idx}] = {r[1]};")
        else:
            b.rate_temp[idx] = r[1]
    out = []
    out.append("  template<class R, class M>")
    out.append(f"  __device__ __forceinline__ static void rates_vjp{sfx}(const R VOI, const R* __restrict__ STATES,"
               " const R* __restrict__ PARAMS, const R* __restrict__ LAM_RATES, R* __restrict__ LAM_STATES,"
               " R* __restrict__ LAM_PARAMS)")
    out.append("  {")
    out.append("    (void)VOI; (void)PARAMS;")
    pows = _collect_int_pows(lines)
    pows_vjp = sorted(set(pows) | {n - 1 for n in pows if n > 2})
    for n in pows_vjp:
        out.append("#define " + _pow_macro_defs([n])[0].split("#define ", 1)[1])
    out.append(f"    R ALG[{max(model.n_algebraics, 1)}];")
    out.append("    (void)ALG;")
    out.extend(b.fwd)
    for name, *_ in b.ops:
        out.append(f"    R a_{name} = (R)0;")
    for idx, tn in sorted(b.rate_temp.items()):
        out.append(f"    a_{tn} += LAM_RATES[{idx}];")
    bwd = b.backward()
    out.extend(bwd)
    out.append("  }")
    # the same split in two: a forward that records every temporary (and condition) on a tape, and a
    # backward that reads the tape, so that a caller who needs the rates anyway evaluates them only once
    n_tape = b.n
    conds = [ln.split("const bool ", 1)[1].split(" =", 1)[0] for ln in b.fwd if "const bool " in ln]
    out.append(f"  static constexpr int nTape{sfx.title().replace('_', '')} = {n_tape + len(conds)};")
    out.append("  template<class R, class M>")
    out.append(f"  __device__ __forceinline__ static void rates_tape{sfx}(const R VOI, const R* __restrict__ STATES,"
               " const R* __restrict__ PARAMS, R* __restrict__ RATES, R* __restrict__ TAPE)")
    out.append("  {")
    out.append("    (void)VOI; (void)PARAMS;")
    out.append(f"    R ALG[{max(model.n_algebraics, 1)}];")
    out.append("    (void)ALG;")
    ci = {c: n_tape + k for k, c in enumerate(conds)}
    for ln in b.fwd:
        out.append(ln)
        st = ln.strip()
        if st.startswith("const R t"):
            name = st.split()[2]
            out.append(f"    TAPE[{int(name[1:])}] = {name};")
        elif st.startswith("const bool c"):
            name = st.split()[2]
            out.append(f"    TAPE[{ci[name]}] = {name} ? (R)1 : (R)0;")
    for idx, tn in sorted(b.rate_temp.items()):
        out.append(f"    RATES[{idx}] = {tn};")
    out.append("  }")
    out.append("  template<class R, class M>")
    out.append(f"  __device__ __forceinline__ static void rates_vjp_tape{sfx}(const R VOI, const R* __restrict__ STATES,"
               " const R* __restrict__ PARAMS, const R* __restrict__ TAPE, const R* __restrict__ LAM_RATES,"
               " R* __restrict__ LAM_STATES, R* __restrict__ LAM_PARAMS)")
    out.append("  {")
    out.append("    (void)VOI; (void)PARAMS; (void)STATES;")
    for k in range(n_tape):
        out.append(f"    const R t{k} = TAPE[{k}];")
    for c, k in ci.items():
        out.append(f"    const bool {c} = TAPE[{k}] != (R)0;")
    for name, *_ in b.ops:
        out.append(f"    R a_{name} = (R)0;")
    for idx, tn in sorted(b.rate_temp.items()):
        out.append(f"    a_{tn} += LAM_RATES[{idx}];")
    out.extend(bwd)
    out.append("  }")
    for n in pows_vjp:
        out.append(f"#undef FDM_POW{n}")
    return out


# ----------------------------------------------------------------------------------------------
# the "mappings" settings key
# ----------------------------------------------------------------------------------------------

def model_variable_names(model: str) -> Dict[str, List[str]]:
    """Names ("component/variable") of the states, algebraics and constants of a built model, from the
    generator's description next to its CUDA code."""
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "generated")
    for f in sorted(os.listdir(here)):
        if f.startswith(model + "_") and f.endswith(".json"):
            with open(os.path.join(here, f)) as fh:
                d = json.load(fh)
            return {"state": d["state_names"], "algebraic": d["algebraic_names"], "constant": d["constant_names"]}
    raise ValueError(f"no generated description for model {model!r}")


def parse_mappings(mappings: dict, names: Dict[str, List[str]]) -> Dict[str, list]:
    """The CellmlAdapter's ``"mappings"`` key (core/src/cellml/00_cellml_adapter_base.tpp:160-607).

    Keys are ``("parameter", i)``, ``("connectorSlot", i)``, ``("connectorSlot", "slotName")`` (numbered on from
    the last number) or ``(kind, i, "slotName")``; a key that is not a tuple is a parameter number.  Values are
    ``(kind, name or number)`` with kind state / algebraic (or intermediate) / constant / parameter, or a bare
    name, looked up among the algebraics, then the states, then the constants.  Entries are ordered by the
    length of the key's first word and then by number (parameters before connector slots).  Parameters mapped to
    algebraics and constants give parametersUsedAsAlgebraic / parametersUsedAsConstant in that order; connector
    slots give statesForTransfer, algebraicsForTransfer and parametersForTransfer (a constant that is a parameter
    counts as that parameter).  What the reference only logs as an error raises ValueError here."""
    entries = []
    slot_counter = 0
    for key, value in mappings.items():
        if isinstance(key, tuple):
            word = str(key[0])
            if len(key) == 2:
                if isinstance(key[1], numbers.Integral):
                    no, slot = int(key[1]), ""
                    slot_counter = no + 1
                else:
                    no, slot = slot_counter, str(key[1])
                    slot_counter += 1
            elif len(key) == 3:
                no, slot = int(key[1]), str(key[2])
            else:
                raise ValueError(f"mappings: key {key!r} is not a tuple with 2 or 3 entries")
            if word not in ("parameter", "connectorSlot", "outputConnectorSlot"):
                raise ValueError(f"mappings: key {key!r} is not ('parameter', i) or ('connectorSlot', i)")
        else:
            word, no, slot = "parameter", int(key), ""
        if isinstance(value, tuple):
            kind, what = str(value[0]), value[1]
        else:
            what = str(value)
            kind = next((k for k in ("algebraic", "state", "constant") if what in names[k]), None)
            if kind is None:
                raise ValueError(f"mappings: {what!r} is neither a state, an algebraic nor a constant of the model")
        if kind == "intermediate":
            kind = "algebraic"
        entries.append(((word, no, slot), (kind, what)))
    entries.sort(key=lambda e: (len(e[0][0]), e[0][1]))

    def field_no(kind, what):
        if isinstance(what, numbers.Integral) or (isinstance(what, str) and what.isdigit()):
            return int(what)
        if kind not in names or what not in names[kind]:
            raise ValueError(f"mappings: {kind} {what!r} is not a {kind} of the model")
        return names[kind].index(what)

    out = {"parametersUsedAsAlgebraic": [], "parametersUsedAsConstant": [], "statesForTransfer": [],
           "algebraicsForTransfer": [], "parametersForTransfer": [], "slotNames": []}
    slot_names = {"state": [], "algebraic": [], "parameter": []}
    for (word, no, slot), (kind, what) in entries:
        if kind not in ("state", "algebraic", "constant", "parameter"):
            raise ValueError(f"mappings: invalid field {kind!r} (state, algebraic or constant)")
        if kind == "parameter":
            fno = int(what)
        else:
            fno = field_no(kind, what)
        if word == "parameter":
            if kind == "algebraic":
                out["parametersUsedAsAlgebraic"].append(fno)
            elif kind == "constant":
                out["parametersUsedAsConstant"].append(fno)
            else:
                raise ValueError(f"mappings: parameter {no} maps to a {kind}; parameters map to algebraics and "
                                 f"constants only")
        elif kind in ("state", "algebraic", "parameter"):
            out[{"state": "statesForTransfer", "algebraic": "algebraicsForTransfer",
                 "parameter": "parametersForTransfer"}[kind]].append(fno)
            slot_names[kind].append(slot)
        elif fno in out["parametersUsedAsConstant"]:
            out["parametersForTransfer"].append(len(out["parametersUsedAsAlgebraic"]) +
                                                out["parametersUsedAsConstant"].index(fno))
            slot_names["parameter"].append(slot)
        else:
            raise ValueError(f"mappings: connector slot {no} maps to constant {what!r}, which is no parameter")
    out["slotNames"] = slot_names["state"] + slot_names["algebraic"] + slot_names["parameter"]
    return out
