#!/usr/bin/env python3
"""Mechanical translation of the reference's hydro-path Fortran into C.

TEST INFRASTRUCTURE ONLY.  No Fortran compiler exists on this image, so the
reference cannot be built as is.  This script reads the reference's own
sources (module global, compparameter, decomposition, q2w, pressure,
coordinates, w2n, press2temp, muscl.f90, riemann.f90, boundary.f90,
hydrostep, cosmostep, updatetime, timestepiteration, thermalstep,
coolstep (chemistry build), conduction.f90, compunits, temp2press, chem, the comoving-time routines of
cosmology.f90 and the shocktube / Kelvin-Helmholtz ICs) and translates the
Fortran 90 subset they use into C, statement by statement, keeping Fortran
semantics:

  * default-real literals (0.5, 1e6, 3.1415927) are C floats, d-exponent
    literals doubles, so mixed-mode promotion is the Fortran one;
  * expressions keep Fortran precedence and left-to-right association
    (a*b*c = (a*b)*c; unary minus binds looser than * and /; ** is right
    associative); x**n with an integer n becomes repeated multiplication as
    gfortran expands it, a real exponent becomes pow;
  * arrays are column-major with their declared lower bounds; array-section
    assignments become loops; actual arguments are passed by reference
    (sections by the address of their first element);
  * MIN/MAX take the next argument when it is smaller/larger;
  * real(8) functions become C functions returning double; an `external`
    dummy procedure becomes a function pointer, and a function named as an
    actual argument is passed as one; `exit` leaves the innermost DO.

The output is compiled with gcc -O2 -ffp-contract=off (gfortran -O3 on x86-64
emits no FMA) together with oracle/ref/harness.c into oracle/_ref/.  Any
construct outside the handled subset aborts the translation.

Usage: f2c.py --ref /root/reference --out oracle/_ref/evora_ref.c
"""
from __future__ import annotations

import argparse
import os
import re
import sys

UNITS = [
    # (file, subroutines to take (None = all), renames)
    ("source/global.f90", None, {}),
    ("source/parameter.f90", ["compparameter"], {}),
    ("source/parallel.f90", ["decomposition"], {}),
    ("source/comp.f90", ["q2w", "pressure", "coordinates", "w2n", "press2temp", "temp2press"], {}),
    ("source/muscl.f90", None, {}),
    ("source/riemann.f90", None, {}),
    ("source/boundary.f90", None, {}),
    ("source/timestep.f90", ["hydrostep", "cosmostep", "updatetime", "timestepiteration", "thermalstep"], {}),
    ("source/cosmology.f90", ["cosmostart", "compcosmo", "expansion", "peebles", "adot2", "dcosmodt", "peeblesint",
                              "rungekutta", "trapezoid"], {}),
    ("source/conduction.f90", None, {}),
    ("source/units.f90", ["compunits"], {}),
    ("source/chemistry.f90", ["chem"], {}),
    ("ic/shocktube.f90", None, {"ic": "ic_shocktube"}),
    ("ic/kevinhelmholtz.f90", None, {"ic": "ic_kevinhelmholtz"}),
]

# Routines called by the translated code but not translated: the harness
# provides them (error stop, MPI broadcast no-ops, the species solvers).
EXTERNAL_STUBS = {"cleanstop", "bcastdouble", "bcastcoef", "cie", "ncie"}

# The CIE build adds the equilibrium chemistry and cooling.
CIE_UNITS = [
    ("source/chemistry.f90", ["initchem", "compbackground", "ncheck"], {}),
    ("source/cie.f90", ["cie", "cieabundance", "implicitcie", "rf_cie", "fne", "cieions"], {}),
    ("source/rates.f90", ["compcoef", "comprates", "cool"], {}),
    ("source/timestep.f90", ["coolstep"], {}),
]


# The non-equilibrium build (-DNONCIE: nq = nf = 12, nw = 11) adds the
# Patankar solver; chem calls both species solvers, so it links the CIE
# routines as well.
NCIE_UNITS = [
    ("source/ncie.f90", ["ncie", "patankarh", "patankarhe"], {}),
]


class F2CError(Exception):
    pass


# --------------------------------------------------------------- lexing ---
# Macros of the build being translated: none for the plain build, {"CIE"}
# for the equilibrium-chemistry build, {"NONCIE"} for the non-equilibrium
# one (global.f90:29-36).
DEFINES: set = set()


def preprocess(text):
    """#ifdef/#elif/#else/#endif with the macros of DEFINES."""
    out, stack = [], []   # stack of (taking, any_taken)
    for line in text.splitlines():
        s = line.strip()
        if s.startswith("#"):
            d = s[1:].split()
            kw = d[0]
            if kw in ("ifdef", "if"):
                on = d[1] in DEFINES
                stack.append([on, on])
            elif kw == "elif":
                top = stack[-1]
                on = (not top[1]) and d[1] in DEFINES
                top[0] = on
                top[1] = top[1] or on
            elif kw == "else":
                top = stack[-1]
                top[0] = not top[1]
                top[1] = True
            elif kw == "endif":
                stack.pop()
            else:
                raise F2CError(f"preprocessor directive {s}")
            out.append("")
            continue
        if all(t[0] for t in stack) or not stack:
            out.append(line)
        else:
            out.append("")
    return out


def strip_comment(line):
    res, q = [], None
    for ch in line:
        if q:
            res.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            res.append(ch)
        elif ch == "!":
            break
        else:
            res.append(ch)
    return "".join(res)


def split_semicolons(line):
    parts, cur, q = [], [], None
    for ch in line:
        if q:
            cur.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            cur.append(ch)
        elif ch == ";":
            parts.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    parts.append("".join(cur))
    return parts


def statements(text):
    lines = preprocess(text)
    stmts, buf = [], ""
    for raw in lines:
        s = strip_comment(raw).rstrip()
        if not s.strip():
            continue
        s = s.strip()
        if buf:
            if s.startswith("&"):
                s = s[1:]
            buf += " " + s
        else:
            buf = s
        if buf.endswith("&"):
            buf = buf[:-1]
            continue
        for part in split_semicolons(buf):
            if part.strip():
                stmts.append(part.strip())
        buf = ""
    return stmts


TOKEN_RE = re.compile(r"""
    (?P<ws>\s+)
  | (?P<str>'[^']*'|"[^"]*")
  | (?P<dotop>\.(?:and|or|not|eqv|neqv|lt|le|gt|ge|eq|ne|true|false)\.)
  | (?P<num>(?:\d+\.(?![a-z])\d*|\.\d+)(?:[ed][+-]?\d+)?|\d+[ed][+-]?\d+|\d+)
  | (?P<name>[a-z_][a-z0-9_]*)
  | (?P<op>\*\*|==|/=|<=|>=|::|[-+*/()<>=,:%])
""", re.X)


def tokenize(s):
    s = s.lower() if "'" not in s and '"' not in s else s
    toks, pos = [], 0
    while pos < len(s):
        m = TOKEN_RE.match(s, pos)
        if not m:
            raise F2CError(f"cannot tokenize: {s[pos:]!r} in {s!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        val = m.group(kind)
        if kind in ("name", "dotop", "num"):
            val = val.lower()
        toks.append((kind, val))
    return toks


# --------------------------------------------------------- expressions ---
class Node:
    pass


class Num(Node):
    def __init__(self, text):
        self.text = text
        if re.fullmatch(r"\d+", text):
            self.type = "int"
        elif "d" in text:
            self.type = "double"
        else:
            self.type = "float"


class Log(Node):
    def __init__(self, v):
        self.v = v
        self.type = "logical"


class Name(Node):
    def __init__(self, name):
        self.name = name


class Ref(Node):
    def __init__(self, name, args):
        self.name = name
        self.args = args


class Range(Node):
    def __init__(self, lo, hi):
        self.lo, self.hi = lo, hi


class Bin(Node):
    def __init__(self, op, a, b):
        self.op, self.a, self.b = op, a, b


class Un(Node):
    def __init__(self, op, a):
        self.op, self.a = op, a


class Parser:
    def __init__(self, toks):
        self.t = toks
        self.i = 0

    def peek(self, k=0):
        return self.t[self.i + k] if self.i + k < len(self.t) else (None, None)

    def take(self, val=None):
        tok = self.peek()
        if val is not None and tok[1] != val:
            raise F2CError(f"expected {val!r}, got {tok!r} in {self.t}")
        self.i += 1
        return tok

    def at(self, val):
        return self.peek()[1] == val

    def done(self):
        return self.i >= len(self.t)

    # precedence climbing, Fortran levels
    def expr(self):
        return self.eqv()

    def eqv(self):
        a = self.or_()
        while self.peek()[1] in (".eqv.", ".neqv."):
            op = self.take()[1]
            a = Bin(op, a, self.or_())
        return a

    def or_(self):
        a = self.and_()
        while self.at(".or."):
            self.take()
            a = Bin(".or.", a, self.and_())
        return a

    def and_(self):
        a = self.not_()
        while self.at(".and."):
            self.take()
            a = Bin(".and.", a, self.not_())
        return a

    def not_(self):
        if self.at(".not."):
            self.take()
            return Un(".not.", self.not_())
        return self.rel()

    REL = {".lt.": "<", "<": "<", ".le.": "<=", "<=": "<=", ".gt.": ">", ">": ">", ".ge.": ">=",
           ">=": ">=", ".eq.": "==", "==": "==", ".ne.": "!=", "/=": "!="}

    def rel(self):
        a = self.add()
        if self.peek()[1] in self.REL:
            op = self.REL[self.take()[1]]
            a = Bin(op, a, self.add())
        return a

    def add(self):
        if self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            a = self.mul()
            a = Un(op, a)
        else:
            a = self.mul()
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            a = Bin(op, a, self.mul())
        return a

    def mul(self):
        a = self.power()
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            a = Bin(op, a, self.power())
        return a

    def power(self):
        a = self.primary()
        if self.at("**"):
            self.take()
            b = self.power_rhs()
            return Bin("**", a, b)
        return a

    def power_rhs(self):
        # right associative; a unary minus may lead the exponent
        if self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            return Un(op, self.power())
        return self.power()

    def primary(self):
        kind, val = self.peek()
        if kind == "num":
            self.take()
            return Num(val)
        if kind == "dotop" and val in (".true.", ".false."):
            self.take()
            return Log(val == ".true.")
        if val == "(":
            self.take()
            e = self.expr()
            self.take(")")
            return e
        if kind == "name":
            self.take()
            if self.at("("):
                self.take()
                args = []
                if not self.at(")"):
                    while True:
                        args.append(self.subscript())
                        if self.at(","):
                            self.take()
                            continue
                        break
                self.take(")")
                return Ref(val, args)
            return Name(val)
        raise F2CError(f"unexpected token {self.peek()} in {self.t}")

    def subscript(self):
        if self.at(":"):
            self.take()
            hi = None if self.peek()[1] in (",", ")") else self.expr()
            return Range(None, hi)
        e = self.expr()
        if self.at(":"):
            self.take()
            hi = None if self.peek()[1] in (",", ")") else self.expr()
            return Range(e, hi)
        return e


def parse_expr(s):
    p = Parser(tokenize(s))
    e = p.expr()
    if not p.done():
        raise F2CError(f"trailing tokens in {s!r}: {p.t[p.i:]}")
    return e


# ------------------------------------------------------------- symbols ---
class Sym:
    def __init__(self, name, ftype, dims=None, param=None, scope="local", dummy=False, external=False):
        self.name = name
        self.external = external    # a procedure (real(8), external :: f)
        self.ftype = ftype          # int, long, double, float, logical, char, complex
        self.dims = dims or []      # list of (lo_node, hi_node)
        self.param = param          # constant expression node for parameters
        self.scope = scope          # module / local
        self.dummy = dummy

    @property
    def is_array(self):
        return bool(self.dims)


CTYPE = {"int": "int", "long": "long long", "double": "double", "float": "float", "logical": "int"}


def parse_type(spec):
    spec = spec.replace(" ", "")
    if spec.startswith("real(8)") or spec.startswith("doubleprecision"):
        return "double"
    if spec.startswith("real"):
        return "float"
    if spec.startswith("integer(8)"):
        return "long"
    if spec.startswith("integer"):
        return "int"
    if spec.startswith("logical"):
        return "logical"
    if spec.startswith("character"):
        return "char"
    if spec.startswith("complex"):
        return "complex"
    raise F2CError(f"type {spec}")


def split_top(s, sep=","):
    out, depth, cur, q = [], 0, [], None
    for ch in s:
        if q:
            cur.append(ch)
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == sep and depth == 0:
            out.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    out.append("".join(cur))
    return [x.strip() for x in out if x.strip()]


def parse_dims(s):
    dims = []
    for d in split_top(s):
        if ":" in d:
            lo, hi = d.split(":", 1)
            dims.append((parse_expr(lo), parse_expr(hi)))
        else:
            dims.append((Num("1"), parse_expr(d)))
    return dims


DECL_RE = re.compile(r"^(integer(\(8\))?|real(\(8\))?|double\s+precision|logical|character(\([^)]*\))?|complex(\(8\))?)(?![a-z0-9_])(.*)$", re.I)


def parse_decl(stmt):
    m = DECL_RE.match(stmt)
    if not m:
        return None
    ftype = parse_type(m.group(1).lower())
    rest = m.group(6)
    if "::" in rest:
        attrs_s, ents_s = rest.split("::", 1)
    else:
        attrs_s, ents_s = "", rest
    attrs = split_top(attrs_s.lstrip(","))
    dims, is_param, is_ext = None, False, False
    for a in attrs:
        a = a.strip().lower()
        if a.startswith("dimension"):
            dims = parse_dims(a[a.index("(") + 1:a.rindex(")")])
        elif a == "parameter":
            is_param = True
        elif a == "external":
            is_ext = True
        elif a.startswith("intent") or a == "allocatable" or a == "save":
            pass
        else:
            raise F2CError(f"attribute {a}")
    ents = []
    for e in split_top(ents_s):
        init = None
        if "=" in e and not e.startswith("("):
            e, init = e.split("=", 1)
            init = init.strip()
        e = e.strip()
        edims = dims
        if "(" in e:
            nm = e[:e.index("(")].strip()
            edims = parse_dims(e[e.index("(") + 1:e.rindex(")")])
        else:
            nm = e
        ents.append((nm.lower(), edims, init))
    return ftype, is_param, ents, is_ext


# ----------------------------------------------------------- emitter ---
class Unit:
    def __init__(self, name, args, body, renames, rtype=None):
        self.name = name
        self.rtype = rtype          # None: subroutine; else the function's result type
        self.args = args
        self.body = body
        self.renames = renames


class Translator:
    def __init__(self):
        self.module = {}         # name -> Sym
        self.units = []          # Unit
        self.unit_names = set()
        self.functions = {}      # function unit name -> result type
        self.arity = {}          # unit name -> number of dummy arguments
        self.out = []
        self.tmp = 0

    # ---- module global
    def load_module(self, stmts):
        inmod = False
        for s in stmts:
            low = s.lower()
            if low.startswith("module "):
                inmod = True
                continue
            if low.startswith("end module"):
                inmod = False
                continue
            if not inmod or low.startswith("implicit") or low.startswith("use "):
                continue
            d = parse_decl(s)
            if not d:
                raise F2CError(f"module statement {s}")
            ftype, is_param, ents, is_ext = d
            if is_ext:
                raise F2CError(f"external in module {s}")
            for nm, dims, init in ents:
                self.module[nm] = Sym(nm, ftype, dims, parse_expr(init) if (is_param and init) else None,
                                      scope="module")
                if init and not is_param:
                    raise F2CError(f"initialised module variable {nm}")

    # ---- units
    def load_units(self, stmts, take, renames):
        i = 0
        while i < len(stmts):
            s = stmts[i]
            m = re.match(r"^(?:(real\(8\)|double\s+precision)\s+)?(subroutine|function)\s+(\w+)\s*(\((.*)\))?\s*$",
                         s, re.I)
            if not m:
                i += 1
                continue
            kind = m.group(2).lower()
            if kind == "function" and not m.group(1):
                raise F2CError(f"function without a real(8) result: {s}")
            rtype = "double" if kind == "function" else None
            name = m.group(3).lower()
            args = [a.strip().lower() for a in (m.group(5) or "").split(",") if a.strip()]
            j = i + 1
            body = []
            while not re.match(r"^end\s*(subroutine|function)\b", stmts[j], re.I) and stmts[j].lower() != "end":
                body.append(stmts[j])
                j += 1
            if take is None or name in take:
                uname = renames.get(name, name)
                self.units.append(Unit(uname, args, body, renames, rtype))
                self.unit_names.add(uname)
                self.arity[uname] = len(args)
                if rtype:
                    self.functions[uname] = rtype
            i = j + 1

    # ---- expression typing / emission
    def sym(self, name, local):
        if name in local:
            return local[name]
        if name in self.module:
            return self.module[name]
        return None

    def const_value(self, node, local):
        """Translation-time value of an integer constant expression."""
        if isinstance(node, Num) and node.type == "int":
            return int(node.text)
        if isinstance(node, Name):
            s = self.sym(node.name, local)
            if s and s.param is not None and s.ftype == "int":
                return self.const_value(s.param, local)
        if isinstance(node, Bin) and node.op in "+-*/":
            a, b = self.const_value(node.a, local), self.const_value(node.b, local)
            if a is None or b is None:
                return None
            return {"+": a + b, "-": a - b, "*": a * b, "/": int(a / b)}[node.op]
        if isinstance(node, Un) and node.op == "-":
            a = self.const_value(node.a, local)
            return None if a is None else -a
        return None

    def etype(self, node, local):
        if isinstance(node, (Num, Log)):
            return node.type
        if isinstance(node, Name):
            s = self.sym(node.name, local)
            if not s:
                raise F2CError(f"unknown name {node.name}")
            return s.ftype
        if isinstance(node, Ref):
            s = self.sym(node.name, local)
            if s and s.is_array:
                return s.ftype
            fn = node.name
            if s and s.external:
                return s.ftype
            if fn in self.functions and not s:
                return self.functions[fn]
            if fn in ("sqrt", "exp", "sin", "cos", "abs"):
                t = self.etype(node.args[0], local)
                return "double" if t in ("double",) else ("float" if t == "float" else t)
            if fn in ("min", "max"):
                return self.promote([self.etype(a, local) for a in node.args])
            if fn == "dble":
                return "double"
            if fn == "maxval":
                return "double"
            if fn == "sum":
                a = node.args[0]
                sa = self.sym(a.name, local) if isinstance(a, (Name, Ref)) else None
                if not sa or not sa.is_array:
                    raise F2CError("sum of a non-array")
                return sa.ftype
            raise F2CError(f"unknown function {fn}")
        if isinstance(node, Un):
            return "logical" if node.op == ".not." else self.etype(node.a, local)
        if isinstance(node, Bin):
            if node.op in (".and.", ".or.", ".eqv.", ".neqv.", "<", "<=", ">", ">=", "==", "!="):
                return "logical"
            if node.op == "**":
                return self.promote([self.etype(node.a, local), self.etype(node.b, local)])
            return self.promote([self.etype(node.a, local), self.etype(node.b, local)])
        raise F2CError(f"type of {node}")

    @staticmethod
    def promote(ts):
        order = ["logical", "int", "long", "float", "double"]
        return max(ts, key=lambda t: order.index(t))

    def index_expr(self, s, subs, loopmap, local):
        """C offset expression for array sym s with subscripts (scalar nodes,
        or Range nodes bound to loop variables via loopmap)."""
        terms = []
        rng = 0
        for k, (lo, hi) in enumerate(s.dims):
            sub = subs[k] if k < len(subs) else Range(None, None)
            if isinstance(sub, Range):
                lo_sub = sub.lo if sub.lo is not None else lo
                var = loopmap[rng] if loopmap is not None else "0"
                rng += 1
                idx = f"(({self.c(lo_sub, local)}) + {var})"
            else:
                idx = f"({self.c(sub, local)})"
            terms.append(f"({idx} - ({self.c(lo, local)}))")
        off = terms[-1]
        for k in range(len(terms) - 2, -1, -1):
            ext = f"(({self.c(s.dims[k][1], local)}) - ({self.c(s.dims[k][0], local)}) + 1)"
            off = f"{terms[k]} + (long)({ext}) * ({off})"
        return off

    def base(self, s):
        if s.scope == "module":
            return f"G_{s.name}"
        return f"v_{s.name}"

    def c(self, node, local, loopmap=None):
        if isinstance(node, Num):
            if node.type == "int":
                return node.text
            t = node.text.replace("d", "e")
            if "." not in t and "e" in t:
                t = t.replace("e", ".0e", 1)
            return t if node.type == "double" else t + "f"
        if isinstance(node, Log):
            return "1" if node.v else "0"
        if isinstance(node, Name):
            s = self.sym(node.name, local)
            if s is None:
                raise F2CError(f"unknown {node.name}")
            if s.is_array:
                raise F2CError(f"whole array {node.name} in scalar context")
            if s.external:
                raise F2CError(f"procedure {node.name} in an expression")
            if s.dummy:
                return f"(*v_{s.name})"
            return self.base(s)
        if isinstance(node, Ref):
            s = self.sym(node.name, local)
            if s and s.is_array:
                ranges = [a for a in node.args if isinstance(a, Range)]
                if ranges and loopmap is None:
                    raise F2CError(f"array section {node.name} in scalar context")
                lm = loopmap[:len(ranges)] if ranges else None
                return f"{self.base(s)}[{self.index_expr(s, node.args, lm, local)}]"
            fn = node.name
            if (s and s.external) or (not s and fn in self.functions):
                return self.fcall(node, local, loopmap)
            if fn == "maxval":
                # MAXVAL of a one-dimensional elementwise array expression
                # (real(8)): a running maximum in element order that takes an
                # element when it is larger, so NaN elements are passed over
                a = self.whole(node.args[0], local)
                sec = self.first_section(a, local)
                if sec is None:
                    raise F2CError("maxval of a scalar")
                ext = self.section_extents(sec, local)
                if len(ext) != 1:
                    raise F2CError("maxval over more than one dimension")
                x = self.c(a, local, ["m_i_"])
                return (f"({{ double m_ = -HUGE_VAL; for (long m_i_ = 0; m_i_ < {ext[0]}; ++m_i_) "
                        f"{{ double x_ = {x}; if (x_ > m_) m_ = x_; }} m_; }})")
            if fn == "sum":
                # SUM of a whole one-dimensional array, accumulated in
                # element order (no reassociation without -ffast-math)
                a = node.args[0]
                sa = self.sym(a.name, local)
                if not isinstance(a, Name) or len(sa.dims) != 1:
                    raise F2CError("sum of an array section")
                lo, hi = sa.dims[0]
                t = CTYPE[sa.ftype]
                ext = f"(({self.c(hi, local)}) - ({self.c(lo, local)}) + 1)"
                return f"({{ {t} acc_ = 0; for (long i_ = 0; i_ < {ext}; ++i_) acc_ += {self.base(sa)}[i_]; acc_; }})"
            args = [self.c(a, local, loopmap) for a in node.args]
            if fn == "sqrt":
                return f"sqrt({args[0]})" if self.etype(node, local) == "double" else f"sqrtf({args[0]})"
            if fn == "exp":
                return f"exp({args[0]})"
            if fn == "sin":
                return f"sin({args[0]})"
            if fn == "abs":
                t = self.etype(node.args[0], local)
                return f"fabs({args[0]})" if t == "double" else (f"fabsf({args[0]})" if t == "float" else f"abs({args[0]})")
            if fn in ("min", "max"):
                t = CTYPE[self.etype(node, local)]
                fname = f"ref_{fn}_{t.replace(' ', '')}"
                acc = f"({t})({args[0]})"
                for a in args[1:]:
                    acc = f"{fname}({acc}, ({t})({a}))"
                return acc
            if fn == "dble":
                return f"((double)({args[0]}))"
            raise F2CError(f"function {fn}")
        if isinstance(node, Un):
            a = self.c(node.a, local, loopmap)
            if node.op == ".not.":
                return f"(!({a}))"
            return f"({node.op}({a}))"
        if isinstance(node, Bin):
            a = self.c(node.a, local, loopmap)
            b = self.c(node.b, local, loopmap)
            op = node.op
            if op == ".and.":
                return f"(({a}) && ({b}))"
            if op == ".or.":
                return f"(({a}) || ({b}))"
            if op == ".eqv.":
                return f"((!({a})) == (!({b})))"
            if op == ".neqv.":
                return f"((!({a})) != (!({b})))"
            if op == "**":
                if isinstance(node.b, Num) and node.b.type == "int":
                    n = int(node.b.text)
                    if n == 2:
                        return f"(({a}) * ({a}))"
                    raise F2CError("integer power other than 2")
                return f"pow({a}, {b})"
            return f"(({a}) {op} ({b}))"
        raise F2CError(f"emit {node}")

    def section_rank(self, node, local):
        if isinstance(node, Ref):
            s = self.sym(node.name, local)
            if s and s.is_array:
                return sum(isinstance(a, Range) for a in node.args) + max(0, len(s.dims) - len(node.args)) \
                    if node.args else len(s.dims)
        return 0

    def whole(self, node, local):
        """Name of an array -> Ref with full ranges."""
        if isinstance(node, Name):
            s = self.sym(node.name, local)
            if s and s.is_array:
                return Ref(node.name, [Range(None, None) for _ in s.dims])
        if isinstance(node, (Bin,)):
            return Bin(node.op, self.whole(node.a, local), self.whole(node.b, local))
        if isinstance(node, Un):
            return Un(node.op, self.whole(node.a, local))
        if isinstance(node, Ref):
            s = self.sym(node.name, local)
            if not (s and s.is_array):
                return Ref(node.name, [self.whole(a, local) for a in node.args])
        return node

    def first_section(self, node, local):
        """The first array section (a Ref to an array with a Range) in node."""
        if isinstance(node, Ref):
            sa = self.sym(node.name, local)
            if sa and sa.is_array and any(isinstance(a, Range) for a in node.args):
                return node
            for a in node.args:
                r = self.first_section(a, local)
                if r is not None:
                    return r
        if isinstance(node, Bin):
            return self.first_section(node.a, local) or self.first_section(node.b, local)
        if isinstance(node, Un):
            return self.first_section(node.a, local)
        return None

    def section_extents(self, ref, local):
        s = self.sym(ref.name, local)
        ext = []
        for k, (lo, hi) in enumerate(s.dims):
            sub = ref.args[k] if k < len(ref.args) else Range(None, None)
            if isinstance(sub, Range):
                l = sub.lo if sub.lo is not None else lo
                h = sub.hi if sub.hi is not None else hi
                ext.append(f"(({self.c(h, local)}) - ({self.c(l, local)}) + 1)")
        return ext

    # ---- statements
    def emit(self, line, ind):
        self.out.append("  " * ind + line)

    def translate_unit(self, u):
        local = {}
        for a in u.args:
            local[a] = None
        decls, execs = [], []
        for s in u.body:
            low = s.lower()
            if low.startswith("use ") or low.startswith("implicit"):
                continue
            if low.startswith("namelist"):
                m = re.match(r"namelist\s*/(\w+)/(.*)", low)
                local[f"__nml_{m.group(1)}"] = [x.strip() for x in m.group(2).split(",")]
                continue
            d = parse_decl(s)
            if d and not execs:
                decls.append(d)
            else:
                execs.append(s)
        nml = {k[6:]: v for k, v in local.items() if k.startswith("__nml_")}
        local = {k: v for k, v in local.items() if not k.startswith("__nml_")}
        for ftype, is_param, ents, is_ext in decls:
            for nm, dims, init in ents:
                local[nm] = Sym(nm, ftype, dims, parse_expr(init) if is_param and init else None,
                                dummy=nm in u.args, external=is_ext)
        if u.rtype and local.get(u.name) is None:
            local[u.name] = Sym(u.name, u.rtype)       # the function's result variable
        for a in u.args:
            if local.get(a) is None:
                raise F2CError(f"undeclared dummy {a} in {u.name}")
        params = []
        for a in u.args:
            s = local[a]
            if s.external:
                params.append(f"{CTYPE[s.ftype]} (*v_{a})()")
            else:
                params.append(f"{CTYPE[s.ftype]} *v_{a}")
        ret = CTYPE[u.rtype] if u.rtype else "void"
        self.emit(f"{ret} ref_{u.name}({', '.join(params) or 'void'}) {{", 0)
        for nm, s in local.items():
            if s.dummy or s.external:
                continue
            if s.ftype == "char":
                continue
            ct = CTYPE[s.ftype]
            if s.param is not None:
                self.emit(f"const {ct} v_{nm} = {self.c(s.param, local)};", 1)
            elif s.is_array:
                n = 1
                for lo, hi in s.dims:
                    lo_v, hi_v = self.const_value(lo, local), self.const_value(hi, local)
                    if lo_v is None or hi_v is None:
                        raise F2CError(f"non-constant local array {nm}")
                    n *= hi_v - lo_v + 1
                self.emit(f"{ct} v_{nm}[{n}];", 1)
            else:
                self.emit(f"{ct} v_{nm};", 1)
        self.block(execs, local, nml, 1)
        if u.rtype:
            self.emit(f"return v_{u.name};", 1)
        self.emit("}", 0)
        self.emit("", 0)

    def block(self, execs, local, nml, ind):
        i = 0
        while i < len(execs):
            s = execs[i]
            low = s.lower()
            m_if = re.match(r"^if\s*\((.*)\)\s*then$", low)
            if m_if or low.startswith("if") and low.rstrip().endswith("then") and re.match(r"^if\s*\(", low):
                cond = self.if_cond(s)
                self.emit(f"if ({self.c(parse_expr(cond), local)}) {{", ind)
                depth, j, seg = 0, i + 1, []
                branches = []
                cur_cond = None
                while True:
                    t = execs[j].lower()
                    if re.match(r"^if\s*\(", t) and t.endswith("then"):
                        depth += 1
                    if depth == 0 and (re.match(r"^else\s*if\s*\(", t) or t == "else"):
                        branches.append((cur_cond, seg))
                        seg = []
                        cur_cond = self.if_cond(execs[j]) if t != "else" else "__else"
                        j += 1
                        continue
                    if re.match(r"^end\s*if$", t):
                        if depth == 0:
                            break
                        depth -= 1
                    seg.append(execs[j])
                    j += 1
                branches.append((cur_cond, seg))
                first = True
                for cnd, body in branches:
                    if not first:
                        if cnd == "__else":
                            self.emit("} else {", ind)
                        else:
                            self.emit(f"}} else if ({self.c(parse_expr(cnd), local)}) {{", ind)
                    first = False
                    self.block(body, local, nml, ind + 1)
                self.emit("}", ind)
                i = j + 1
                continue
            m_do = re.match(r"^do\s+(\w+)\s*=\s*(.*)$", low)
            m_while = re.match(r"^do\s+while\s*\(", low)
            if m_do or m_while:
                depth, j, seg = 0, i + 1, []
                while True:
                    t = execs[j].lower()
                    if re.match(r"^do\s+\w+\s*=", t) or re.match(r"^do\s+while\s*\(", t):
                        depth += 1
                    if re.match(r"^end\s*do$", t):
                        if depth == 0:
                            break
                        depth -= 1
                    seg.append(execs[j])
                    j += 1
                if m_while:
                    cond, rest = self.split_if(s[s.lower().index("while"):].replace("while", "if", 1))
                    if rest:
                        raise F2CError(f"text after do while: {s}")
                    self.emit(f"while ({self.c(parse_expr(cond), local)}) {{", ind)
                else:
                    var = m_do.group(1)
                    lo, hi = split_top(m_do.group(2))
                    v = self.c(Name(var), local)
                    self.emit(f"for ({v} = {self.c(parse_expr(lo), local)}; {v} <= {self.c(parse_expr(hi), local)}; ++{v}) {{",
                              ind)
                self.block(seg, local, nml, ind + 1)
                self.emit("}", ind)
                i = j + 1
                continue
            m_sif = re.match(r"^if\s*\(", low)
            if m_sif:
                cond, rest = self.split_if(s)
                self.emit(f"if ({self.c(parse_expr(cond), local)}) {{", ind)
                self.block([rest], local, nml, ind + 1)
                self.emit("}", ind)
                i += 1
                continue
            self.simple(s, local, nml, ind)
            i += 1

    @staticmethod
    def if_cond(s):
        cond, _ = Translator.split_if(s)
        return cond

    @staticmethod
    def split_if(s):
        k = s.index("(")
        depth = 0
        for j in range(k, len(s)):
            if s[j] == "(":
                depth += 1
            elif s[j] == ")":
                depth -= 1
                if depth == 0:
                    return s[k + 1:j], s[j + 1:].strip()
        raise F2CError(f"unbalanced if {s}")

    def simple(self, s, local, nml, ind):
        low = s.lower()
        if low.startswith("print") or low.startswith("write"):
            self.emit("/* " + s.replace("*/", "* /") + " */", ind)
            return
        if low == "exit":
            self.emit("break;", ind)
            return
        if low == "stop" or low.startswith("stop "):
            self.emit("ref_stop();", ind)
            return
        if low.startswith("open") or low.startswith("close"):
            self.emit("/* " + s + " */", ind)
            return
        m = re.match(r"^read\s*\(\s*\w+\s*,\s*nml\s*=\s*(\w+)\s*\)$", low)
        if m:
            grp = m.group(1)
            args = ", ".join("&" + self.c(Name(v), local) for v in nml[grp])
            self.emit(f"ref_namelist_{grp}({args});", ind)
            return
        m = re.match(r"^call\s+(\w+)\s*(\((.*)\))?$", low)
        if m:
            self.call(m.group(1), m.group(3) or "", local, ind)
            return
        # assignment
        lhs_s, rhs_s = self.split_assign(s)
        lhs = parse_expr(lhs_s)
        rhs = parse_expr(rhs_s)
        if isinstance(lhs, Name):
            sym = self.sym(lhs.name, local)
            if sym and sym.is_array:
                lhs = Ref(lhs.name, [Range(None, None) for _ in sym.dims])
        rank = self.section_rank(lhs, local) if isinstance(lhs, Ref) else 0
        if rank == 0:
            self.emit(f"{self.c(lhs, local)} = {self.c(rhs, local)};", ind)
            return
        ext = self.section_extents(lhs, local)
        rhs = self.whole(rhs, local)
        loops = [f"_i{k}" for k in range(len(ext))]
        for k in range(len(ext) - 1, -1, -1):
            self.emit(f"for (long {loops[k]} = 0; {loops[k]} < {ext[k]}; ++{loops[k]}) {{", ind + (len(ext) - 1 - k))
        depth = ind + len(ext)
        self.emit(f"{self.c(lhs, local, loops)} = {self.c(rhs, local, loops)};", depth)
        for k in range(len(ext)):
            self.emit("}", depth - 1 - k)

    @staticmethod
    def split_assign(s):
        depth = 0
        for j, ch in enumerate(s):
            if ch == "(":
                depth += 1
            elif ch == ")":
                depth -= 1
            elif ch == "=" and depth == 0 and s[j + 1:j + 2] != "=" and s[j - 1:j] not in "<>/=":
                return s[:j], s[j + 1:]
        raise F2CError(f"not an assignment: {s}")

    def call(self, name, argstr, local, ind):
        target = name
        if name in EXTERNAL_STUBS:
            target = name
        elif name not in self.unit_names:
            raise F2CError(f"call to untranslated routine {name}")
        args = []
        pre = []
        for a in split_top(argstr):
            node = parse_expr(a)
            if isinstance(node, Name):
                s = self.sym(node.name, local)
                if s is None:
                    raise F2CError(f"unknown actual {node.name}")
                if s.external:
                    args.append(self.proc(s))
                    continue
                if s.is_array or s.dummy:
                    args.append(self.base(s) if not s.dummy else f"v_{s.name}")
                else:
                    args.append(f"&{self.base(s)}")
                continue
            if isinstance(node, Ref):
                s = self.sym(node.name, local)
                if s and s.is_array:
                    args.append(f"&{self.base(s)}[{self.index_expr(s, node.args, ['0'] * 8, local)}]")
                    continue
            t = CTYPE[self.etype(node, local)]
            tmpn = f"_t{self.tmp}"
            self.tmp += 1
            pre.append(f"{t} {tmpn} = {self.c(node, local)};")
            args.append(f"&{tmpn}")
        # An external procedure has no explicit interface: surplus actual
        # arguments reach the callee, which never reads them (coolstep's
        # cieabundance(q(7:nq,..),chemrate,q(1,..)) against
        # cieabundance(n,chemrate), timestep.f90:127 / cie.f90:62).
        if target in self.arity and len(args) > self.arity[target]:
            args = args[:self.arity[target]]
        if pre:
            self.emit("{", ind)
            for p in pre:
                self.emit(p, ind + 1)
            self.emit(f"ref_{target}({', '.join(args)});", ind + 1)
            self.emit("}", ind)
        else:
            self.emit(f"ref_{target}({', '.join(args)});", ind)

    def proc(self, s):
        """A procedure name as a C function (pointer)."""
        if s.dummy:
            return f"v_{s.name}"
        if s.name not in self.functions:
            raise F2CError(f"external {s.name} is not a translated function")
        return f"ref_{s.name}"

    def fcall(self, node, local, loopmap):
        """A function reference: arguments by address, expressions through
        compound literals (evaluated before the call, as Fortran does)."""
        s = self.sym(node.name, local)
        target = self.proc(s) if s else f"ref_{node.name}"
        args = []
        for a in node.args:
            if isinstance(a, Range):
                raise F2CError(f"array section passed to function {node.name}")
            if isinstance(a, Name):
                sa = self.sym(a.name, local)
                if sa is None:
                    raise F2CError(f"unknown actual {a.name}")
                if sa.external:
                    args.append(self.proc(sa))
                    continue
                if sa.is_array:
                    args.append(self.base(sa))
                    continue
                args.append(f"v_{sa.name}" if sa.dummy else f"&{self.base(sa)}")
                continue
            if isinstance(a, Ref):
                sa = self.sym(a.name, local)
                if sa and sa.is_array:
                    if any(isinstance(x, Range) for x in a.args):
                        raise F2CError(f"array section passed to function {node.name}")
                    args.append(f"&{self.c(a, local, loopmap)}")
                    continue
            t = CTYPE[self.etype(a, local)]
            args.append(f"&({t}){{{self.c(a, local, loopmap)}}}")
        return f"{target}({', '.join(args)})"

    # ---- whole program
    def module_c(self):
        lines = []
        for nm, s in self.module.items():
            if s.ftype in ("char", "complex"):
                continue
            ct = CTYPE[s.ftype]
            if s.param is not None:
                lines.append(f"const {ct} G_{nm} = {self.c(s.param, {})};")
            elif s.is_array:
                n = 1
                for lo, hi in s.dims:
                    n *= self.const_value(hi, {}) - self.const_value(lo, {}) + 1
                lines.append(f"{ct} G_{nm}[{n}];")
            else:
                lines.append(f"{ct} G_{nm};")
        return lines


def translate(ref_root):
    tr = Translator()
    species = "CIE" in DEFINES or "NONCIE" in DEFINES
    units = UNITS + (CIE_UNITS if species else []) + (NCIE_UNITS if "NONCIE" in DEFINES else [])
    if species:
        EXTERNAL_STUBS.discard("cie")
    if "NONCIE" in DEFINES:
        EXTERNAL_STUBS.discard("ncie")
    for rel, take, ren in units:
        text = open(os.path.join(ref_root, rel)).read()
        st = statements(text)
        if rel.endswith("global.f90"):
            tr.load_module(st)
        else:
            tr.load_units(st, take, ren)
    body = []
    tr.out = body
    # prototypes
    protos = []
    for u in tr.units:
        tr.out = []
        tr.translate_unit(u)
        body.extend(tr.out)
        protos.append(tr.out[0].replace(" {", ";"))
    head = [
        "/* GENERATED by oracle/ref/f2c.py from the reference's Fortran sources -- do not edit.",
        " * Test infrastructure: mechanical translation of the hydro path for parity pinning. */",
        "#include <math.h>",
        "#include <stdlib.h>",
        "void ref_stop(void);",
        "void ref_cleanstop(void);",
        "void ref_bcastdouble(double*);",
        "void ref_namelist_ic_para(double*, double*, double*, double*, double*, double*, double*, int*);",
        "static inline double ref_min_double(double a, double b) { return (b < a) ? b : a; }",
        "static inline double ref_max_double(double a, double b) { return (b > a) ? b : a; }",
        "static inline float ref_min_float(float a, float b) { return (b < a) ? b : a; }",
        "static inline float ref_max_float(float a, float b) { return (b > a) ? b : a; }",
        "static inline int ref_min_int(int a, int b) { return (b < a) ? b : a; }",
        "static inline int ref_max_int(int a, int b) { return (b > a) ? b : a; }",
        "",
        "/* module global (global.f90) */",
    ] + tr.module_c() + [""] + protos + [""]
    return "\n".join(head + body) + "\n"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--out", required=True)
    ap.add_argument("--define", action="append", default=[], help="build macro (CIE)")
    a = ap.parse_args()
    DEFINES.update(a.define)
    try:
        src = translate(a.ref)
    except F2CError as e:
        sys.stderr.write(f"f2c: {e}\n")
        return 1
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    with open(a.out, "w") as f:
        f.write(src)
    return 0


if __name__ == "__main__":
    sys.exit(main())
