#!/usr/bin/env python3
"""f2c_ref.py — TEST INFRASTRUCTURE: mechanical Fortran-to-C translation of
the reference's hot-path sources, used only to pin the oracle.

The reference (leon-astrophy/CUMPIC) is Fortran 90 and this image has no
Fortran compiler. This script reads the reference's own .f90 files where they
lie (the --reference directory; oracle/Makefile passes it), translates the subset of
Fortran they use (module globals, subroutines and functions with by-reference
arguments, arrays with explicit lower bounds in column-major order, array
sections, DO / DO WHILE / IF / SELECT CASE, the intrinsics on the path) into
one C file, and writes it to oracle/_ref/. oracle/ref_harness.c includes that
file and exposes the same orc_* entry points as the hand-written oracle, so a
test can run either against identical inputs. Nothing here is copied into the
repository: the translation is regenerated from the reference sources and
stays in the git-ignored oracle/_ref/.

Compile-time PARAMETERs of the reference (grid size, boundary flags, CFL,
reconstruction, adiabatic index, ...) become C globals whose values the
harness can override before f2c_init_params() evaluates the declarations in
order, which is how the reference is rebuilt per configuration.

Fixed translation choices (processor-dependent points of Fortran):
  * ALLOCATE returns zeroed memory.
  * SIGN(a, b) = copysign(|a|, b); MIN/MAX use fmin/fmax on reals.
  * x**n with a literal integer n >= 2 is a left-to-right product (x*x)*x...
  * REAL literals without a D exponent are single precision, as in Fortran.
  * Expressions keep Fortran's left-to-right association; compiled with
    -ffp-contract=off.
"""
from __future__ import annotations

import argparse
import os
import re
import sys

SOLVER = ["definition", "setup", "coords", "initial", "rungekutta", "update", "spatial", "reconstruct", "rsolver",
          "flux", "ptou_face", "mhd", "fromrvetou", "ptou", "utop", "boundary"]
MODELS = {m: [f"model/{m}/src/defs.f90", f"model/{m}/src/custom.f90", f"model/{m}/src/eos.f90"]
          for m in ("riemann", "torus_sph", "torus_cyn")}
SKIP_UNITS = {"initial_model", "getgrid"}  # call GET_MODEL / CUSTOM_GRID of model.f90, not translated


class F2CError(Exception):
    pass


# ---------------------------------------------------------------------------
# source preprocessing: cpp conditionals, comments, continuations
# ---------------------------------------------------------------------------
def strip_comment(line: str) -> str:
    q = None
    for i, ch in enumerate(line):
        if q:
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
        elif ch == "!":
            return line[:i]
    return line


def logical_lines(path: str):
    """yield (lineno, statement) with cpp, comments and continuations resolved.
    No preprocessor macro is defined (the reference's default build: no MPI,
    no GPU)."""
    stack = []  # (parent_active, cond)
    active = True
    pending, pend_ln = "", 0
    for ln, raw in enumerate(open(path, encoding="latin-1").read().split("\n"), 1):
        s = raw.strip()
        if s.startswith("#"):
            d = s[1:].strip().lower()
            if d.startswith(("ifdef", "if ", "if(")):
                stack.append((active, False))
                active = False
            elif d.startswith("ifndef"):
                stack.append((active, True))
                active = active and True
            elif d.startswith("else"):
                par, cond = stack[-1]
                stack[-1] = (par, not cond)
                active = par and not cond
            elif d.startswith("endif"):
                par, _ = stack.pop()
                active = par
            continue
        if not active:
            continue
        body = strip_comment(raw).rstrip()
        if not body.strip():
            continue
        if pending:
            b = body.strip()
            if b.startswith("&"):
                b = b[1:]
            body = pending + " " + b
            ln = pend_ln
        else:
            pend_ln = ln
        if body.rstrip().endswith("&"):
            pending = body.rstrip()[:-1]
            continue
        pending = ""
        for part in split_top(body, ";"):
            if part.strip():
                yield ln, part.strip()


def split_top(s: str, sep: str = ","):
    out, depth, cur, q = [], 0, [], None
    i = 0
    while i < len(s):
        ch = s[i]
        if q:
            cur.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            cur.append(ch)
        elif ch == "(":
            depth += 1
            cur.append(ch)
        elif ch == ")":
            depth -= 1
            cur.append(ch)
        elif ch == sep and depth == 0:
            out.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
        i += 1
    out.append("".join(cur))
    return out


# ---------------------------------------------------------------------------
# expressions
# ---------------------------------------------------------------------------
TOKEN = re.compile(r"""
    (?P<ws>\s+)
  | (?P<dotop>\.(?:and|or|not|eq|ne|lt|le|gt|ge|true|false)\.)
  | (?P<num>(?:\d+\.\d*|\.\d+|\d+)(?:[dDeE][+-]?\d+)?)
  | (?P<name>[A-Za-z_]\w*)
  | (?P<str>'[^']*'|"[^"]*")
  | (?P<op>\*\*|==|/=|<=|>=|\(/|/\)|[-+*/<>(),:=%])
""", re.X | re.I)


def tokenize(s: str):
    toks, pos = [], 0
    while pos < len(s):
        m = TOKEN.match(s, pos)
        if not m:
            raise F2CError(f"cannot tokenize {s[pos:]!r} in {s!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        text = m.group(kind)
        if kind in ("name", "dotop"):
            text = text.lower()
        toks.append((kind, text))
    return toks


class Parser:
    PREC = {".or.": 1, ".and.": 2, "==": 4, "/=": 4, "<": 4, "<=": 4, ">": 4, ">=": 4,
            ".eq.": 4, ".ne.": 4, ".lt.": 4, ".le.": 4, ".gt.": 4, ".ge.": 4,
            "+": 5, "-": 5, "*": 6, "/": 6}

    def __init__(self, text: str):
        self.t = tokenize(text)
        self.i = 0

    def peek(self):
        return self.t[self.i] if self.i < len(self.t) else (None, None)

    def take(self, text=None):
        tok = self.peek()
        if text is not None and tok[1] != text:
            raise F2CError(f"expected {text!r}, got {tok!r}")
        self.i += 1
        return tok

    def done(self):
        return self.i >= len(self.t)

    def expr(self, minp=0):
        k, v = self.peek()
        if v == ".not.":
            self.take()
            lhs = ("un", "!", self.expr(3))
        elif v in ("+", "-") and minp <= 5:
            self.take()
            lhs = ("un", v, self.expr(6))
        else:
            lhs = self.power()
        while True:
            k, v = self.peek()
            p = self.PREC.get(v)
            if p is None or p < minp or (p == minp and False):
                break
            if p <= minp - 1:
                break
            self.take()
            rhs = self.expr(p + 1)
            lhs = ("bin", v, lhs, rhs)
        return lhs

    def power(self):
        base = self.primary()
        if self.peek()[1] == "**":
            self.take()
            k, v = self.peek()
            if v in ("+", "-"):
                self.take()
                e = ("un", v, self.power())
            else:
                e = self.power()
            return ("pow", base, e)
        return base

    def primary(self):
        k, v = self.take()
        if k == "num":
            return ("num", v)
        if k == "str":
            return ("str", v)
        if k == "dotop":
            if v in (".true.", ".false."):
                return ("num", "1" if v == ".true." else "0")
            raise F2CError(f"unexpected {v}")
        if v == "(/":
            items = []
            while self.peek()[1] != "/)":
                items.append(self.expr())
                if self.peek()[1] == ",":
                    self.take()
            self.take("/)")
            return ("arr", items)
        if v == "(":
            e = self.expr()
            self.take(")")
            return ("paren", e)
        if k == "name":
            if self.peek()[1] == "(":
                self.take("(")
                args = []
                if self.peek()[1] != ")":
                    while True:
                        args.append(self.arg())
                        if self.peek()[1] == ",":
                            self.take()
                            continue
                        break
                self.take(")")
                return ("ref", v, args)
            return ("name", v)
        raise F2CError(f"unexpected token {v!r}")

    def arg(self):
        # section lo:hi, :, or expression
        if self.peek()[1] == ":":
            self.take()
            hi = None if self.peek()[1] in (",", ")") else self.expr()
            return ("sec", None, hi)
        e = self.expr()
        if self.peek()[1] == ":":
            self.take()
            hi = None if self.peek()[1] in (",", ")") else self.expr()
            return ("sec", e, hi)
        return e


def parse_expr(text: str):
    p = Parser(text)
    e = p.expr()
    if not p.done():
        raise F2CError(f"trailing tokens in {text!r}: {p.t[p.i:]}")
    return e


# ---------------------------------------------------------------------------
# program units and declarations
# ---------------------------------------------------------------------------
TYPE_RE = re.compile(r"^(real\s*\*\s*8|real\s*\*\s*4|double\s+precision|real|integer|logical)(\s*\(\s*\w+\s*\))?"
                     r"(?P<attrs>(\s*,\s*[a-z]+(\s*\([^)]*\))?)*)\s*(::)?\s*(?P<rest>.*)$", re.I)


class Sym:
    def __init__(self, name, typ, kind="scalar", dims=None, param=False, alloc=False, dummy=False, intent=None):
        self.name, self.typ, self.kind, self.dims = name, typ, kind, dims
        self.param, self.alloc, self.dummy, self.intent = param, alloc, dummy, intent
        self.init = None  # initializer expression (PARAMETER or DATA-like)


class Unit:
    def __init__(self, kind, name, args, ret=None, module=None, src=""):
        self.kind, self.name, self.args, self.ret, self.module, self.src = kind, name, args, ret, module, src
        self.syms: dict[str, Sym] = {}
        self.order: list[str] = []
        self.body: list = []  # (ln, stmt)


def base_type(t: str) -> str:
    t = t.lower().replace(" ", "")
    if t.startswith("integer"):
        return "i"
    if t.startswith("logical"):
        return "l"
    if t in ("real*4", "real"):
        return "f"
    return "d"


def parse_units(path: str, label: str):
    units, modvars = [], []
    cur = None
    module = None
    in_contains_sub = 0
    for ln, s in logical_lines(path):
        low = s.lower()
        m = re.match(r"^module\s+(\w+)$", low)
        if m:
            module = Unit("module", m.group(1), [], src=label)
            cur = module
            units.append(module)
            continue
        if re.match(r"^end\s*module\b", low):
            module = None
            cur = None
            continue
        if low == "contains":
            if cur is not None and cur.kind != "module":
                in_contains_sub = 1  # internal procedures of a subroutine: skipped
            continue
        m = re.match(r"^subroutine\s+(\w+)\s*(?:\((.*)\))?$", low)
        mf = re.match(r"^(real\s*\*\s*8|integer|real|double\s+precision)\s+function\s+(\w+)\s*\((.*)\)$", low)
        if (m or mf) and in_contains_sub:
            in_contains_sub += 1
            continue
        if m:
            args = [a.strip() for a in (m.group(2) or "").split(",") if a.strip()]
            cur = Unit("sub", m.group(1), args, module=module.name if module else None, src=label)
            units.append(cur)
            continue
        if mf:
            args = [a.strip() for a in mf.group(3).split(",") if a.strip()]
            cur = Unit("func", mf.group(2), args, ret=base_type(mf.group(1)), module=module.name if module else None,
                       src=label)
            units.append(cur)
            continue
        if re.match(r"^end\s*(subroutine|function)\b", low) or low == "end":
            if in_contains_sub:
                in_contains_sub -= 1
                if in_contains_sub == 0:
                    cur = module
                else:
                    continue
                if low.startswith("end") and in_contains_sub == 0:
                    pass
                continue
            cur = module
            continue
        if in_contains_sub:
            continue
        if cur is None:
            continue
        cur.body.append((ln, s))
    return units


def split_decl(unit: Unit):
    """move declarations out of the unit body into its symbol table"""
    body = []
    for ln, s in unit.body:
        low = s.lower()
        if re.match(r"^(use\b|implicit\b|save$|include\b)", low):
            continue
        m = TYPE_RE.match(low)
        if m and not re.match(r"^(real|integer)[^:]*\bfunction\b", low):
            if m.group(2) and m.group(2).strip(" ()") not in ("8", "4"):
                continue  # e.g. integer(HID_T): HDF5 handles, unused on the path
            typ = base_type(m.group(1))
            attrs = [a.strip() for a in split_top(m.group("attrs"), ",") if a.strip()]
            param = any(a.startswith("parameter") for a in attrs)
            alloc = any(a.startswith("allocatable") for a in attrs)
            dims = None
            intent = None
            for a in attrs:
                dm = re.match(r"dimension\s*\((.*)\)$", a)
                if dm:
                    dims = [d.strip() for d in split_top(dm.group(1))]
                im = re.match(r"intent\s*\((\w+)\)", a)
                if im:
                    intent = im.group(1)
            for item in split_top(m.group("rest")):
                item = item.strip()
                if not item:
                    continue
                init = None
                if "=" in item and not re.match(r"^\w+\s*\([^)]*=", item):
                    name_part, init = item.split("=", 1)
                else:
                    name_part = item
                nm = re.match(r"^(\w+)\s*(?:\((.*)\))?$", name_part.strip())
                name = nm.group(1)
                d = [x.strip() for x in split_top(nm.group(2))] if nm.group(2) else dims
                sym = Sym(name, typ, "array" if d else "scalar", d, param, alloc, name in unit.args, intent)
                if init is not None:
                    sym.init = init.strip()
                if name in unit.syms and unit.kind == "func" and name == unit.name:
                    continue
                unit.syms[name] = sym
                unit.order.append(name)
            continue
        body.append((ln, s))
    unit.body = body


# ---------------------------------------------------------------------------
# C emission
# ---------------------------------------------------------------------------
INTRINSIC_D = {"dsqrt": "sqrt", "sqrt": "sqrt", "dsin": "sin", "sin": "sin", "dcos": "cos", "cos": "cos",
               "dtan": "tan", "tan": "tan", "dexp": "exp", "exp": "exp", "datan": "atan", "atan": "atan",
               "dlog": "log", "log": "log"}


class Emitter:
    def __init__(self, units):
        self.units = units
        self.globals: dict[str, Sym] = {}
        self.procs: dict[str, Unit] = {}
        self.param_order: list[tuple[str, Sym]] = []
        for u in units:
            split_decl(u)
        for u in units:
            if u.kind == "module":
                for n in u.order:
                    s = u.syms[n]
                    self.globals[n] = s
                    if s.param or s.init is not None:
                        self.param_order.append((n, s))
            else:
                if u.name in SKIP_UNITS:
                    continue
                self.procs[u.name] = u
        self.called_missing: set[str] = set()
        self.out: list[str] = []
        self.tmp = 0

    # -- symbol lookup ------------------------------------------------------
    def lookup(self, unit: Unit | None, name: str):
        if unit is not None and name in unit.syms:
            return "local", unit.syms[name]
        if name in self.globals:
            return "global", self.globals[name]
        return None, None

    def cname(self, unit, name):
        where, s = self.lookup(unit, name)
        if where == "global":
            return "f_" + name
        if where == "local":
            if s.dummy:
                return ("v_" if s.kind == "array" else "a_") + name
            return "l_" + name
        if unit is not None and unit.kind == "func" and name == unit.name:
            return "r_ret"
        raise F2CError(f"unknown name {name!r} in {unit.name if unit else '<global>'}")

    # -- typing ---------------------------------------------------------------
    def typ(self, unit, e) -> str:
        k = e[0]
        if k == "num":
            t = e[1].lower()
            if re.search(r"[.de]", t):
                return "f" if "d" not in t else "d"
            return "i"
        if k == "name":
            if unit is not None and unit.kind == "func" and e[1] == unit.name and e[1] not in unit.syms:
                return unit.ret
            where, s = self.lookup(unit, e[1])
            if s is None:
                raise F2CError(f"unknown {e[1]}")
            return s.typ
        if k == "paren":
            return self.typ(unit, e[1])
        if k == "un":
            return "l" if e[1] == "!" else self.typ(unit, e[2])
        if k == "bin":
            if e[1] in (".and.", ".or.") or self.PRED.get(e[1]):
                return "l"
            a, b = self.typ(unit, e[2]), self.typ(unit, e[3])
            if "d" in (a, b):
                return "d"
            if "f" in (a, b):
                return "f"
            return "i"
        if k == "pow":
            return self.typ(unit, e[1])
        if k == "ref":
            name = e[1]
            where, s = self.lookup(unit, name)
            if s is not None and s.kind == "array":
                return s.typ
            if name in self.procs and self.procs[name].kind == "func":
                return self.procs[name].ret
            if name in INTRINSIC_D:
                return "d"
            if name in ("abs", "min", "max", "sign"):
                ts = [self.typ(unit, a) for a in e[2]]
                return "d" if "d" in ts else ("f" if "f" in ts else "i")
            if name in ("dble", "tiny"):
                return "d"
            if name in ("int", "nint"):
                return "i"
            raise F2CError(f"unknown function/array {name}")
        raise F2CError(f"cannot type {e}")

    PRED = {"==": "==", "/=": "!=", "<": "<", "<=": "<=", ">": ">", ">=": ">=", ".eq.": "==", ".ne.": "!=",
            ".lt.": "<", ".le.": "<=", ".gt.": ">", ".ge.": ">="}

    # -- expressions ------------------------------------------------------------
    def num(self, t: str) -> str:
        tl = t.lower()
        if "d" in tl:
            m = re.match(r"^(.*?)d([+-]?\d+)$", tl)
            mant = m.group(1)
            if mant.endswith("."):
                mant += "0"
            if mant.startswith("."):
                mant = "0" + mant
            return f"{mant}e{m.group(2)}"
        if re.search(r"[.e]", tl):
            mant = tl
            if mant.endswith("."):
                mant += "0"
            if mant.startswith("."):
                mant = "0" + mant
            return f"((double){mant}f)"  # single-precision literal, promoted
        return t

    def elem(self, unit, name, idx, sec_map=None):
        """pointer expression to an array element; idx are subscript nodes"""
        where, s = self.lookup(unit, name)
        cn = self.cname(unit, name)
        parts = []
        si = 0
        for a in idx:
            if a[0] == "sec":
                if sec_map is None:
                    raise F2CError(f"section of {name} outside an array assignment")
                var, lhs_lo = sec_map[si]
                lo = self.lbound_expr(unit, name, len(parts)) if a[1] is None else self.ex(unit, a[1])
                parts.append(f"(({lo}) + ({var}) - ({lhs_lo}))")
                si += 1
            else:
                parts.append(self.ex(unit, a))
        while len(parts) < 4:
            parts.append("0")
        fn = "fai_at" if s.typ == "i" else "fad_at"
        return f"{fn}(&{cn}, {', '.join(parts)})"

    def lbound_expr(self, unit, name, dim):
        return f"{self.cname(unit, name)}.lb[{dim}]"

    def ex(self, unit, e, sec_map=None) -> str:
        k = e[0]
        if k == "num":
            return self.num(e[1])
        if k == "str":
            return '"' + e[1][1:-1] + '"'
        if k == "paren":
            return "(" + self.ex(unit, e[1], sec_map) + ")"
        if k == "name":
            where, s = self.lookup(unit, e[1])
            cn = self.cname(unit, e[1])
            if s is not None and s.kind == "array":
                if sec_map is not None:  # whole array in an array assignment
                    return "(*" + self.elem(unit, e[1], [("sec", None, None)] * self.rank(unit, e[1]), sec_map) + ")"
                raise F2CError(f"whole array {e[1]} in a scalar context")
            if cn.startswith("a_"):
                return f"(*{cn})"
            return cn
        if k == "un":
            if e[1] == "!":
                return "(!" + self.ex(unit, e[2], sec_map) + ")"
            return f"({e[1]}" + self.ex(unit, e[2], sec_map) + ")"
        if k == "bin":
            op = e[1]
            a = self.ex(unit, e[2], sec_map)
            b = self.ex(unit, e[3], sec_map)
            if op == ".and.":
                return f"({a} && {b})"
            if op == ".or.":
                return f"({a} || {b})"
            if op in self.PRED:
                return f"({a} {self.PRED[op]} {b})"
            return f"({a} {op} {b})"
        if k == "pow":
            b = self.ex(unit, e[1], sec_map)
            ex = e[2]
            if ex[0] == "num" and re.fullmatch(r"\d+", ex[1]):
                n = int(ex[1])
                if n == 0:
                    return "1.0"
                r = b
                for _ in range(n - 1):
                    r = f"({r} * {b})"
                return r
            return f"pow({b}, {self.ex(unit, ex, sec_map)})"
        if k == "arr":
            raise F2CError("array constructor outside a PARAMETER")
        if k == "ref":
            name, args = e[1], e[2]
            where, s = self.lookup(unit, name)
            if s is not None and s.kind == "array":
                return "(*" + self.elem(unit, name, args, sec_map) + ")"
            if name in self.procs and self.procs[name].kind == "func":
                return self.call_args(unit, self.procs[name], args, func=True)
            if name in INTRINSIC_D:
                return f"{INTRINSIC_D[name]}(" + self.ex(unit, args[0], sec_map) + ")"
            ts = [self.typ(unit, a) for a in args]
            real = "d" in ts or "f" in ts
            xs = [self.ex(unit, a, sec_map) for a in args]
            if name == "abs":
                return f"fabs({xs[0]})" if real else f"abs({xs[0]})"
            if name in ("min", "max"):
                fn = ("fmin" if name == "min" else "fmax") if real else ("f2c_imin" if name == "min" else "f2c_imax")
                r = xs[0]
                for x in xs[1:]:
                    r = f"{fn}({r}, {x})"
                return r
            if name == "sign":
                return f"copysign(fabs({xs[0]}), {xs[1]})" if real else f"f2c_isign({xs[0]}, {xs[1]})"
            if name == "dble":
                return f"((double)({xs[0]}))"
            if name == "tiny":
                return "DBL_MIN"
            if name == "int":
                return f"((int)({xs[0]}))"
            raise F2CError(f"unknown function {name}")
        raise F2CError(f"cannot emit {e}")

    def rank(self, unit, name):
        where, s = self.lookup(unit, name)
        return len(s.dims)

    # -- calls -------------------------------------------------------------------
    def call_args(self, unit, proc: Unit, args, func=False) -> str:
        if len(args) != len(proc.args):
            raise F2CError(f"{proc.name}: {len(args)} actual arguments for {len(proc.args)} dummies")
        cargs = []
        for a, dn in zip(args, proc.args):
            d = proc.syms.get(dn)
            if d is None:
                raise F2CError(f"undeclared dummy {dn} of {proc.name}")
            if d.kind == "array":
                cargs.append(self.array_actual(unit, a))
            else:
                cargs.append(self.scalar_actual(unit, a, d.typ))
        fn = ("ff_" if func else "fs_") + proc.name
        return f"{fn}({', '.join(cargs)})"

    def array_actual(self, unit, a):
        if a[0] == "name":
            return self.cname(unit, a[1]) + ".d"
        if a[0] == "ref":
            where, s = self.lookup(unit, a[1])
            if s is None or s.kind != "array":
                raise F2CError(f"array actual expected, got {a}")
            idx = []
            for x in a[2]:
                if x[0] == "sec":
                    idx.append(("__lb__", len(idx)) if x[1] is None else x[1])
                else:
                    idx.append(x)
            parts = []
            for i, x in enumerate(idx):
                if isinstance(x, tuple) and x[0] == "__lb__":
                    parts.append(self.lbound_expr(unit, a[1], x[1]))
                else:
                    parts.append(self.ex(unit, x))
            while len(parts) < 4:
                parts.append("0")
            fn = "fai_at" if s.typ == "i" else "fad_at"
            return f"{fn}(&{self.cname(unit, a[1])}, {', '.join(parts)})"
        raise F2CError(f"bad array actual {a}")

    def scalar_actual(self, unit, a, dtyp):
        ctype = {"i": "int", "d": "double", "f": "float", "l": "int"}[dtyp]
        if a[0] == "name":
            where, s = self.lookup(unit, a[1])
            if s is not None and s.kind == "scalar" and s.typ == dtyp:
                cn = self.cname(unit, a[1])
                return cn if cn.startswith("a_") else "&" + cn
        if a[0] == "ref":
            where, s = self.lookup(unit, a[1])
            if s is not None and s.kind == "array" and s.typ == dtyp:
                return self.elem(unit, a[1], a[2])
        return f"&({ctype}){{{self.ex(unit, a)}}}"

    # -- statements ---------------------------------------------------------------
    def emit_body(self, unit: Unit):
        lines = []
        ind = 1
        stack = []

        def put(s):
            lines.append("    " * ind + s)

        for ln, s in unit.body:
            low = s.lower()
            where = f"{unit.src}:{ln}"
            try:
                if re.match(r"^(write|print)\b", low):
                    continue
                if re.match(r"^stop\b", low):
                    put(f'f2c_stop("{where}");')
                    continue
                if re.match(r"^return$", low):
                    put("goto f2c_exit;")
                    unit._has_exit = True
                    continue
                m = re.match(r"^do\s+while\s*\((.*)\)$", low)
                if m:
                    put(f"while ({self.ex(unit, parse_expr(m.group(1)))}) {{ /* {where} */")
                    ind += 1
                    stack.append("do")
                    continue
                m = re.match(r"^do\s+(\w+)\s*=\s*(.*)$", low)
                if m:
                    parts = split_top(m.group(2))
                    v = self.cname(unit, m.group(1))
                    lo = self.ex(unit, parse_expr(parts[0]))
                    hi = self.ex(unit, parse_expr(parts[1]))
                    st = self.ex(unit, parse_expr(parts[2])) if len(parts) > 2 else "1"
                    self.tmp += 1
                    t = self.tmp
                    put(f"{{ const int hi{t} = {hi}, st{t} = {st}; for ({v} = {lo}; st{t} > 0 ? {v} <= hi{t} : {v} >= hi{t}; {v} += st{t}) {{ /* {where} */")
                    ind += 1
                    stack.append("dofor")
                    continue
                if re.match(r"^end\s*do$", low):
                    ind -= 1
                    kind = stack.pop()
                    put("}}" if kind == "dofor" else "}")
                    continue
                m = re.match(r"^if\s*\((.*)\)\s*then$", low)
                if m and self.balanced_if(low):
                    put(f"if ({self.ex(unit, parse_expr(m.group(1)))}) {{ /* {where} */")
                    ind += 1
                    stack.append("if")
                    continue
                m = re.match(r"^else\s*if\s*\((.*)\)\s*then$", low)
                if m:
                    ind -= 1
                    put(f"}} else if ({self.ex(unit, parse_expr(m.group(1)))}) {{ /* {where} */")
                    ind += 1
                    continue
                if low == "else":
                    ind -= 1
                    put("} else {")
                    ind += 1
                    continue
                if re.match(r"^end\s*if$", low):
                    ind -= 1
                    stack.pop()
                    put("}")
                    continue
                m = re.match(r"^select\s*case\s*\((.*)\)$", low)
                if m:
                    self.tmp += 1
                    put(f"{{ const long sel{self.tmp} = {self.ex(unit, parse_expr(m.group(1)))}; int first{self.tmp} = 1; (void)first{self.tmp}; /* {where} */")
                    stack.append(("select", self.tmp, False))
                    ind += 1
                    continue
                m = re.match(r"^case\s*\((.*)\)$", low)
                if m or low == "case default":
                    sel = stack[-1]
                    t = sel[1]
                    opened = sel[2]
                    if opened:
                        ind -= 1
                        put("}")
                    if low == "case default":
                        cond = "1"
                    else:
                        vals = [self.ex(unit, parse_expr(v)) for v in split_top(m.group(1))]
                        cond = " || ".join(f"sel{t} == ({v})" for v in vals)
                    put(f"{'if' if not opened else 'else if'} ({cond}) {{")
                    stack[-1] = ("select", t, True)
                    ind += 1
                    continue
                if re.match(r"^end\s*select$", low):
                    sel = stack.pop()
                    if sel[2]:
                        ind -= 1
                        put("}")
                    ind -= 1
                    put("}")
                    continue
                m = re.match(r"^call\s+(\w+)\s*(?:\((.*)\))?$", low)
                if m:
                    name = m.group(1)
                    args = []
                    if m.group(2) is not None and m.group(2).strip():
                        args = [Parser(a).arg() if ":" in a else parse_expr(a) for a in split_top(m.group(2))]
                    if name not in self.procs:
                        self.called_missing.add(name)
                        put(f'f2c_missing("{name}", "{where}");')
                        continue
                    put(self.call_args(unit, self.procs[name], args) + f"; /* {where} */")
                    continue
                m = re.match(r"^allocate\s*\((.*)\)$", low)
                if m:
                    for item in split_top(m.group(1)):
                        nm = re.match(r"^\s*(\w+)\s*\((.*)\)\s*$", item)
                        name = nm.group(1)
                        dims = split_top(nm.group(2))
                        bounds = []
                        for d in dims:
                            if ":" in d:
                                lo, hi = split_top(d, ":")
                            else:
                                lo, hi = "1", d
                            bounds += [self.ex(unit, parse_expr(lo)), self.ex(unit, parse_expr(hi))]
                        where_, s = self.lookup(unit, name)
                        fn = "f2c_alloc_i" if s.typ == "i" else "f2c_alloc_d"
                        put(f"{fn}(&{self.cname(unit, name)}, {len(dims)}, (int[]){{{', '.join(bounds)}}}); /* {where} */")
                    continue
                if re.match(r"^deallocate\b", low):
                    continue
                # single-line IF
                m = re.match(r"^if\s*\(", low)
                if m:
                    cond, rest = self.split_if(s)
                    put(f"if ({self.ex(unit, parse_expr(cond))}) {{ /* {where} */")
                    sub = Unit(unit.kind, unit.name, unit.args, unit.ret, unit.module, unit.src)
                    sub.syms, sub.order = unit.syms, unit.order
                    sub.body = [(ln, rest)]
                    for l2 in self.emit_body(sub):
                        lines.append("    " * ind + l2.strip())
                    put("}")
                    continue
                # assignment
                lhs, rhs = self.split_assign(s)
                lines.extend("    " * ind + x for x in self.assign(unit, lhs, rhs, where))
            except F2CError as err:
                raise F2CError(f"{where}: {err} [{s}]") from None
        return lines

    @staticmethod
    def balanced_if(low):
        # "if (...) then" where the parenthesis closes right before "then"
        depth = 0
        for i, ch in enumerate(low):
            if ch == "(":
                depth += 1
            elif ch == ")":
                depth -= 1
                if depth == 0:
                    return low[i + 1:].strip() == "then"
        return False

    @staticmethod
    def split_if(s):
        i = s.index("(")
        depth = 0
        for j in range(i, len(s)):
            if s[j] == "(":
                depth += 1
            elif s[j] == ")":
                depth -= 1
                if depth == 0:
                    return s[i + 1:j], s[j + 1:].strip()
        raise F2CError("unbalanced IF")

    @staticmethod
    def split_assign(s):
        depth = 0
        for i, ch in enumerate(s):
            if ch == "(":
                depth += 1
            elif ch == ")":
                depth -= 1
            elif ch == "=" and depth == 0 and s[i + 1:i + 2] != "=" and s[i - 1:i] not in "<>/=":
                return s[:i].strip(), s[i + 1:].strip()
        raise F2CError(f"not an assignment: {s}")

    def assign(self, unit, lhs_text, rhs_text, where):
        lhs = Parser(lhs_text).primary()
        rhs = parse_expr(rhs_text)
        name = lhs[1]
        wh, s = self.lookup(unit, name)
        # whole array or section assignment
        secs = []
        if s is not None and s.kind == "array":
            if lhs[0] == "name":
                lhs = ("ref", name, [("sec", None, None)] * len(s.dims))
            for d, a in enumerate(lhs[2]):
                if a[0] == "sec":
                    secs.append(d)
        if not secs:
            if lhs[0] == "name":
                target = self.ex(unit, lhs) if not self.cname(unit, name).startswith("a_") else f"(*{self.cname(unit, name)})"
                if unit.kind == "func" and name == unit.name:
                    target = "r_ret"
            else:
                target = "(*" + self.elem(unit, name, lhs[2]) + ")"
            return [f"{target} = {self.ex(unit, rhs)}; /* {where} */"]
        out = ["{ /* " + where + " */"]
        sec_map = []
        loops = []
        for n_, d in enumerate(secs):
            a = lhs[2][d]
            lo = f"{self.cname(unit, name)}.lb[{d}]" if a[1] is None else self.ex(unit, a[1])
            hi = (f"({self.cname(unit, name)}.lb[{d}] + {self.cname(unit, name)}.n[{d}] - 1)" if a[2] is None
                  else self.ex(unit, a[2]))
            self.tmp += 1
            v = f"s{self.tmp}"
            out.append(f"    const int {v}lo = {lo}, {v}hi = {hi}; int {v};")
            loops.append((v, f"{v}lo", f"{v}hi"))
            sec_map.append((v, f"{v}lo"))
        # loops: first section varies fastest
        body_ind = "    "
        for v, lo, hi in reversed(loops):
            out.append(f"{body_ind}for ({v} = {lo}; {v} <= {hi}; ++{v})")
            body_ind += "    "
        lhs_ptr = self.elem(unit, name, lhs[2], sec_map)
        out.append(f"{body_ind}(*{lhs_ptr}) = {self.ex(unit, rhs, sec_map)};")
        out.append("}")
        return out

    # -- units --------------------------------------------------------------------
    def ctype(self, t):
        return {"i": "int", "d": "double", "f": "float", "l": "int"}[t]

    def proto(self, u: Unit) -> str:
        ps = []
        for a in u.args:
            s = u.syms.get(a)
            if s is None:
                raise F2CError(f"{u.src}: undeclared dummy {a} of {u.name}")
            ps.append(f"{self.ctype(s.typ)}* {'p_' if s.kind == 'array' else 'a_'}{a}")
        ret = "void" if u.kind == "sub" else self.ctype(u.ret)
        pre = "fs_" if u.kind == "sub" else "ff_"
        return f"static {ret} {pre}{u.name}({', '.join(ps) if ps else 'void'})"

    def emit_unit(self, u: Unit):
        o = self.out
        o.append(f"/* {u.src}: {u.kind} {u.name} */")
        o.append(self.proto(u) + " {")
        if u.kind == "func":
            o.append(f"    {self.ctype(u.ret)} r_ret = 0;")
        for n in u.order:
            s = u.syms[n]
            if u.kind == "func" and n == u.name:
                continue
            if s.dummy:
                if s.kind == "array":
                    arrt = "fai" if s.typ == "i" else "fad"
                    bounds = []
                    for d in s.dims:
                        if ":" in d:
                            lo, hi = split_top(d, ":")
                        else:
                            lo, hi = "1", d
                        bounds += [self.ex(u, parse_expr(lo)), self.ex(u, parse_expr(hi))]
                    o.append(f"    {arrt} v_{n}; f2c_view_{'i' if s.typ == 'i' else 'd'}(&v_{n}, p_{n}, {len(s.dims)}, (int[]){{{', '.join(bounds)}}});")
                continue
            if s.kind == "array":
                raise F2CError(f"{u.src}: local array {n} in {u.name} not supported")
            init = f" = {self.ex(u, parse_expr(s.init))}" if s.init else " = 0"
            o.append(f"    {self.ctype(s.typ)} l_{n}{init};")
        u._has_exit = False
        body = self.emit_body(u)
        o.extend(body)
        if getattr(u, "_has_exit", False):
            o.append("f2c_exit: ;")
        if u.kind == "func":
            o.append("    return r_ret;")
        o.append("}")
        o.append("")

    def emit(self) -> str:
        o = self.out
        o.append("/* Generated by oracle/f2c_ref.py from the reference sources; do not edit. */")
        # globals
        o.append("/* ---- module variables and PARAMETERs ---- */")
        for n, s in self.globals.items():
            if s.kind == "array":
                o.append(f"static {'fai' if s.typ == 'i' else 'fad'} f_{n};")
            else:
                o.append(f"static {self.ctype(s.typ)} f_{n};")
        o.append("")
        for u in self.procs.values():
            o.append(self.proto(u) + ";")
        o.append("")
        # parameter init
        o.append("static void f2c_init_params(void) {")
        for n, s in self.globals.items():
            if s.kind == "array" and not s.alloc:
                bounds = []
                for d in s.dims:
                    if ":" in d:
                        lo, hi = split_top(d, ":")
                    else:
                        lo, hi = "1", d
                    bounds += [self.ex(None, parse_expr(lo)), self.ex(None, parse_expr(hi))]
                fn = "f2c_alloc_i" if s.typ == "i" else "f2c_alloc_d"
                o.append(f"    {fn}(&f_{n}, {len(s.dims)}, (int[]){{{', '.join(bounds)}}});")
                if s.init:
                    e = parse_expr(s.init)
                    if e[0] != "arr":
                        raise F2CError(f"array PARAMETER {n} needs (/ ... /)")
                    for i, it in enumerate(e[1]):
                        o.append(f'    f_{n}.d[{i}] = f2c_override_{"i" if s.typ == "i" else "d"}("{n}", {i}, {self.ex(None, it)});')
            elif s.kind == "scalar" and s.init is not None:
                o.append(f'    f_{n} = f2c_override_{"i" if s.typ == "i" else "d"}("{n}", 0, {self.ex(None, parse_expr(s.init))});')
        o.append("}")
        o.append("")
        for u in self.procs.values():
            self.emit_unit(u)
        return "\n".join(o)


RUNTIME = r"""
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double* d; int lb[4]; int n[4]; int rank; } fad;
typedef struct { int* d; int lb[4]; int n[4]; int rank; } fai;

static void f2c_stop(const char* where) { fprintf(stderr, "STOP at %s\n", where); abort(); }
static void f2c_missing(const char* name, const char* where) {
    fprintf(stderr, "call of untranslated %s at %s\n", name, where); abort();
}
static inline int f2c_imin(int a, int b) { return a < b ? a : b; }
static inline int f2c_imax(int a, int b) { return a > b ? a : b; }
static inline int f2c_isign(int a, int b) { int x = a < 0 ? -a : a; return b >= 0 ? x : -x; }

#define F2C_MAX_OVR 64
static struct { const char* name; int idx; double v; } f2c_ovr[F2C_MAX_OVR];
static int f2c_novr = 0;
static void f2c_set_override(const char* name, int idx, double v) {
    for (int i = 0; i < f2c_novr; ++i)
        if (!strcmp(f2c_ovr[i].name, name) && f2c_ovr[i].idx == idx) { f2c_ovr[i].v = v; return; }
    f2c_ovr[f2c_novr].name = name; f2c_ovr[f2c_novr].idx = idx; f2c_ovr[f2c_novr].v = v; ++f2c_novr;
}
static double f2c_override_d(const char* name, int idx, double dflt) {
    for (int i = 0; i < f2c_novr; ++i) if (!strcmp(f2c_ovr[i].name, name) && f2c_ovr[i].idx == idx) return f2c_ovr[i].v;
    return dflt;
}
static int f2c_override_i(const char* name, int idx, int dflt) {
    return (int)f2c_override_d(name, idx, (double)dflt);
}

static void f2c_shape(int* lb, int* n, int rank, const int* b) {
    for (int i = 0; i < 4; ++i) { lb[i] = 0; n[i] = 1; }
    for (int i = 0; i < rank; ++i) { lb[i] = b[2 * i]; n[i] = b[2 * i + 1] - b[2 * i] + 1; }
}
static void f2c_alloc_d(fad* a, int rank, const int* b) {
    free(a->d); a->rank = rank; f2c_shape(a->lb, a->n, rank, b);
    size_t t = 1; for (int i = 0; i < 4; ++i) t *= (size_t)a->n[i];
    a->d = (double*)calloc(t, sizeof(double));
}
static void f2c_alloc_i(fai* a, int rank, const int* b) {
    free(a->d); a->rank = rank; f2c_shape(a->lb, a->n, rank, b);
    size_t t = 1; for (int i = 0; i < 4; ++i) t *= (size_t)a->n[i];
    a->d = (int*)calloc(t, sizeof(int));
}
static void f2c_view_d(fad* a, double* p, int rank, const int* b) { a->d = p; a->rank = rank; f2c_shape(a->lb, a->n, rank, b); }
static void f2c_view_i(fai* a, int* p, int rank, const int* b) { a->d = p; a->rank = rank; f2c_shape(a->lb, a->n, rank, b); }

static inline size_t f2c_off(const int* lb, const int* n, int i0, int i1, int i2, int i3) {
#ifdef F2C_CHECK
    const int ii[4] = {i0, i1, i2, i3};
    for (int q = 0; q < 4; ++q)
        if (ii[q] < lb[q] || ii[q] >= lb[q] + n[q]) { fprintf(stderr, "index %d out of bounds in dim %d\n", ii[q], q); abort(); }
#endif
    return (size_t)(i0 - lb[0]) + (size_t)n[0] * ((size_t)(i1 - lb[1]) + (size_t)n[1] * ((size_t)(i2 - lb[2]) + (size_t)n[2] * (size_t)(i3 - lb[3])));
}
static inline double* fad_at(fad* a, int i0, int i1, int i2, int i3) { return a->d + f2c_off(a->lb, a->n, i0, i1, i2, i3); }
static inline int* fai_at(fai* a, int i0, int i1, int i2, int i3) { return a->d + f2c_off(a->lb, a->n, i0, i1, i2, i3); }
"""


def translate(model: str, ref: str) -> str:
    units = []
    files = [f"solver/{f}.f90" for f in SOLVER] + MODELS[model]
    # the model's PARAMETER module comes first: definition.f90 does not use it
    for f in MODELS[model][:1] + [f for f in files if f not in MODELS[model][:1]]:
        units += parse_units(os.path.join(ref, f), f)
    em = Emitter(units)
    body = em.emit()
    return RUNTIME + "\n" + body + "\n"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--model", default="riemann", choices=sorted(MODELS))
    ap.add_argument("--reference", required=True, help="root of the reference's source tree")
    ap.add_argument("-o", "--output", required=True)
    args = ap.parse_args()
    if not os.path.isdir(os.path.join(args.reference, "solver")):
        print(f"reference sources not found under {args.reference}", file=sys.stderr)
        return 2
    code = translate(args.model, args.reference)
    os.makedirs(os.path.dirname(os.path.abspath(args.output)), exist_ok=True)
    with open(args.output, "w") as f:
        f.write(code)
    return 0


if __name__ == "__main__":
    sys.exit(main())
