"""Runs the reference's own Fortran 90 procedures of the hot path in Python.

TEST INFRASTRUCTURE ONLY: used by tests/golden/make_ref_golden.py to produce
golden vectors from the reference's source text in a container that has the
reference tree but no Fortran compiler; the product never imports it.

The reference (yw-choi/DMFT-ED-ZT) is Fortran 90 + MPI + MKL and cannot be
compiled here (no Fortran compiler).  This module translates, statement by
statement, the subset of Fortran 90 that the hot-path files use into Python
functions and runs them: modules and their `use ... only:` scoping,
subroutines and functions with dummy-argument intents, explicit-shape and
allocatable arrays with lower bounds (column-major, 1-based by default),
derived types with allocatable components, do / do while / labelled do,
if / else if / select case, cycle / exit / return, whole-array and section
assignments, the intrinsics used (BTEST, IBSET, IBCLR, mod, abs, min, max,
sqrt, sum, cmplx, dcmplx, dble, huge, allocated) and Fortran's integer
division and default-kind rules (cmplx without a kind is single precision).
I/O statements are skipped.

Outside the translated source, only what the reference takes from external
libraries is supplied here, named and restated:
  * MPI with one rank: mpi_allgather(v) copy, mpi_allreduce identity,
    mpi_bcast / mpi_barrier no-ops, mpi_wtime 0 (the reference's `use mpi`);
  * BLAS daxpy: y(i) = y(i) + a x(i) in index order (Netlib's loop);
  * LAPACK dstevx('V', 'A') and dlamch: all eigenpairs of the symmetric
    tridiagonal matrix through scipy.linalg.eigh_tridiagonal (LAPACK
    dstemr/dstebz; MKL's own dstevx is not available), eigenvectors with the
    sign of their largest component made positive, as LAPACK leaves it free;
  * random_number: the caller's start vector hook, since the reference draws
    from an unseeded generator (src/lanczos_solver.f90:42-46).
Fortran's default integer is 32 bits: the states of nsite 16 overflow in the
reference (src/ed_basis.f90:135), so runs here stay at nsite <= 15.
"""

from __future__ import annotations

import math
import re
import sys
from dataclasses import dataclass, field

import numpy as np

# ---------------------------------------------------------------------------
# runtime: arrays, derived types, intrinsics, external libraries
# ---------------------------------------------------------------------------


class FArray:
    """A Fortran array: column-major flat list `d`, lower bounds `lb`,
    extents `ext`.  Integers are Python ints, reals Python floats."""

    __slots__ = ("d", "lb", "ext", "st", "kind")

    def __init__(self, bounds, kind, fill=None):
        self.lb = [b[0] for b in bounds]
        self.ext = [max(b[1] - b[0] + 1, 0) for b in bounds]
        st, s = [], 1
        for e in self.ext:
            st.append(s)
            s *= e
        self.st = st
        self.kind = kind
        if fill is None:
            fill = {"integer": 0, "real": 0.0, "complex": 0j, "logical": False}.get(kind, 0.0)
        self.d = [fill] * s

    def size(self):
        return len(self.d)

    def off(self, idx):
        o = 0
        for i, l, e, s in zip(idx, self.lb, self.ext, self.st):
            if not (l <= i < l + e):
                raise IndexError(f"index {idx} outside bounds lb={self.lb} ext={self.ext}")
            o += (i - l) * s
        return o

    def section(self, spec):
        """Flat offsets of a section; spec per dimension: int or (lo, hi) or None (all)."""
        ranges = []
        for dim, sp in enumerate(spec):
            l, e = self.lb[dim], self.ext[dim]
            if sp is None:
                ranges.append(range(l, l + e))
            elif isinstance(sp, tuple):
                lo = l if sp[0] is None else sp[0]
                hi = l + e - 1 if sp[1] is None else sp[1]
                ranges.append(range(lo, hi + 1))
            else:
                ranges.append(range(sp, sp + 1))
        return _colmajor_offsets(self, ranges)


def _colmajor_offsets(a, ranges):
    offs = [0]
    for dim, rg in enumerate(ranges):
        s, l = a.st[dim], a.lb[dim]
        offs = [o + s * (i - l) for i in rg for o in offs]
    return offs


class Elems:
    """Values of a whole array or section in column-major order."""

    __slots__ = ("v",)

    def __init__(self, v):
        self.v = v


def _vals(x):
    if isinstance(x, FArray):
        return x.d
    if isinstance(x, Elems):
        return x.v
    return None


def _elemental(op, a, b):
    va, vb = _vals(a), _vals(b)
    if va is None and vb is None:
        return op(a, b)
    if va is None:
        return Elems([op(a, y) for y in vb])
    if vb is None:
        return Elems([op(x, b) for x in va])
    if len(va) != len(vb):
        raise ValueError("non-conformable arrays")
    return Elems([op(x, y) for x, y in zip(va, vb)])


def _neg(a):
    va = _vals(a)
    return Elems([-x for x in va]) if va is not None else -a


def _idiv(a, b):
    """Fortran integer division (truncation toward zero)."""
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


def _div(a, b):
    if isinstance(a, int) and isinstance(b, int) and not isinstance(a, bool):
        return _idiv(a, b)
    return a / b


def _pow(a, b):
    if isinstance(a, int) and isinstance(b, int):
        return a ** b if b >= 0 else _idiv(1, a ** (-b))
    return a ** b


def _mod(a, b):
    if isinstance(a, int) and isinstance(b, int):
        return a - _idiv(a, b) * b
    return math.fmod(a, b)


def _f32(x):
    return float(np.float32(x))


class Ops:
    add = staticmethod(lambda a, b: _elemental(lambda x, y: x + y, a, b))
    sub = staticmethod(lambda a, b: _elemental(lambda x, y: x - y, a, b))
    mul = staticmethod(lambda a, b: _elemental(lambda x, y: x * y, a, b))
    div = staticmethod(lambda a, b: _elemental(_div, a, b))
    pow = staticmethod(lambda a, b: _elemental(_pow, a, b))
    neg = staticmethod(_neg)


def _assign_array(dst: FArray, offs, value):
    vals = _vals(value)
    if vals is None:
        conv = _conv(dst.kind)
        v = conv(value)
        for o in offs:
            dst.d[o] = v
        return
    if len(vals) != len(offs):
        raise ValueError(f"assignment of {len(vals)} values to a section of {len(offs)}")
    conv = _conv(dst.kind)
    vals = list(vals)                     # the whole right side first (Fortran semantics)
    for o, v in zip(offs, vals):
        dst.d[o] = conv(v)


def _conv(kind):
    if kind == "integer":
        return lambda v: int(v) if not isinstance(v, bool) else int(v)
    if kind == "real":
        return lambda v: float(v.real) if isinstance(v, complex) else float(v)
    if kind == "complex":
        return complex
    if kind == "logical":
        return bool
    return lambda v: v


def conv_scalar(kind, v):
    if kind == "integer":
        if isinstance(v, float):
            return int(v)                 # Fortran real -> integer assignment truncates
        return int(v)
    if kind == "real":
        return float(v.real) if isinstance(v, complex) else float(v)
    if kind == "complex":
        return complex(v)
    if kind == "logical":
        return bool(v)
    return v


class Intrinsics:
    """The Fortran intrinsics the hot-path files call."""

    @staticmethod
    def btest(i, pos):
        return ((i >> pos) & 1) == 1

    @staticmethod
    def ibset(i, pos):
        return i | (1 << pos)

    @staticmethod
    def ibclr(i, pos):
        return i & ~(1 << pos)

    @staticmethod
    def mod(a, b):
        return _mod(a, b)

    @staticmethod
    def abs(a):
        return abs(a)

    @staticmethod
    def min(*a):
        return min(a)

    @staticmethod
    def max(*a):
        return max(a)

    @staticmethod
    def sqrt(a):
        return math.sqrt(a) if not isinstance(a, complex) else a ** 0.5

    @staticmethod
    def exp(a):
        return math.exp(a)

    @staticmethod
    def dble(a):
        return float(a.real) if isinstance(a, complex) else float(a)

    @staticmethod
    def real(a):
        return float(a.real) if isinstance(a, complex) else float(a)

    @staticmethod
    def int(a):
        return int(a)

    @staticmethod
    def huge(a):
        return sys.float_info.max if isinstance(a, float) else 2 ** 31 - 1

    @staticmethod
    def cmplx(x, y=0.0):
        """CMPLX without a KIND argument: default (single precision) complex."""
        return complex(_f32(x), _f32(y))

    @staticmethod
    def dcmplx(x, y=0.0):
        return complex(float(x), float(y))

    @staticmethod
    def sum(a):
        s = 0.0
        for v in _vals(a):                # in index order, one rounding per term
            s = s + v
        return s

    @staticmethod
    def allocated(a):
        return a is not None

    @staticmethod
    def size(a, dim=None):
        return a.size() if dim is None else a.ext[dim - 1]


class Externals:
    """MPI (one rank), BLAS daxpy, LAPACK dstevx/dlamch and random_number."""

    def __init__(self):
        self.random_hook = None

    # MPI, one rank: the reference's collectives reduce to copies
    def mpi_allgatherv(self, send, n, t1, recv, counts, displs, t2, comm, ierr):
        for i in range(n):
            recv.d[i] = send.d[i]
        return {}

    def mpi_allgather(self, send, n, t1, recv, n2, t2, comm, ierr):
        return {"recv": send}

    def mpi_allreduce(self, send, recv, n, t, op, comm, ierr):
        return {"recv": send}

    def mpi_bcast(self, *a):
        return {}

    def mpi_barrier(self, *a):
        return {}

    def mpi_wtime(self, *a):
        return 0.0

    def die(self, routine, msg="", *a):
        raise RuntimeError(f"die({routine}, {msg}) in the reference")

    def random_seed(self, *a):
        if self.random_hook is not None:
            self.random_hook("seed")
        return {}

    def random_number(self, r):
        return {"r": self.random_hook("next")}

    def daxpy(self, n, a, x, incx, y, incy):
        # Netlib daxpy with unit strides: dy(i) = dy(i) + da*dx(i)
        xd, yd = x.d, y.d
        for i in range(n):
            yd[i] = yd[i] + a * xd[i]
        return {}

    def dlamch(self, c):
        if c.lower().startswith("s"):
            return sys.float_info.min     # safe minimum (2^-1022)
        if c.lower().startswith("e"):
            return 2.0 ** -53
        raise ValueError(c)

    def dstevx(self, jobz, rng, n, d, e, vl, vu, il, iu, abstol, m, w, z, ldz, work, iwork, ifail, info):
        from scipy.linalg import eigh_tridiagonal
        dd = np.array(d.d[:n], dtype=float)
        ee = np.array(e.d[: max(n - 1, 0)], dtype=float)
        if n == 1:
            vals, vecs = dd.copy(), np.ones((1, 1))
        else:
            vals, vecs = eigh_tridiagonal(dd, ee)
        for j in range(n):
            col = vecs[:, j]
            if col[np.argmax(np.abs(col))] < 0:
                vecs[:, j] = -col
        for j in range(n):
            w.d[j] = float(vals[j])
            for i in range(n):
                z.d[i + ldz * j] = float(vecs[i, j])
        return {"m": n, "info": 0}


# ---------------------------------------------------------------------------
# source: logical statements
# ---------------------------------------------------------------------------


@dataclass
class Stmt:
    text: str          # lower case, comments stripped, continuation joined
    line: int          # first source line
    raw: str


def _strip_comment(line):
    out, q = [], None
    for ch in line:
        if q:
            out.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            out.append(ch)
        elif ch == "!":
            break
        else:
            out.append(ch)
    return "".join(out)


def _lower_code(s):
    out, q = [], None
    for ch in s:
        if q:
            out.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            out.append(ch)
        else:
            out.append(ch.lower())
    return "".join(out)


def statements(src):
    lines = src.split("\n")
    out = []
    buf, start = "", 0
    for no, raw in enumerate(lines, 1):
        s = _strip_comment(raw).rstrip()
        if not s.strip():
            continue
        t = s.strip()
        if buf:
            if t.startswith("&"):
                t = t[1:]
            buf += " " + t
        else:
            buf, start = t, no
        if buf.endswith("&"):
            buf = buf[:-1]
            continue
        for part in _split_semicolons(buf):
            if part.strip():
                out.append(Stmt(_lower_code(part.strip()), start, part.strip()))
        buf = ""
    return out


def _split_semicolons(s):
    parts, cur, q = [], [], None
    for ch in s:
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


# ---------------------------------------------------------------------------
# expressions
# ---------------------------------------------------------------------------

_DOTOPS = {".and.": "and", ".or.": "or", ".not.": "not", ".eq.": "==", ".ne.": "/=", ".lt.": "<",
           ".le.": "<=", ".gt.": ">", ".ge.": ">=", ".eqv.": "eqv", ".neqv.": "neqv", ".true.": "TRUE",
           ".false.": "FALSE"}


def tokenize(s):
    toks, i, n = [], 0, len(s)
    while i < n:
        c = s[i]
        if c.isspace():
            i += 1
            continue
        if c == ".":
            m = re.match(r"\.(and|or|not|eq|ne|lt|le|gt|ge|eqv|neqv|true|false)\.", s[i:])
            if m:
                toks.append(("op", _DOTOPS[m.group(0)]))
                i += len(m.group(0))
                continue
        if c.isdigit() or (c == "." and i + 1 < n and s[i + 1].isdigit()):
            m = re.match(r"\d*\.?\d*([ed][-+]?\d+)?(_\w+)?", s[i:])
            txt = m.group(0)
            # "2.or." : an integer followed by a dot operator
            dm = re.match(r"(\d+)\.(and|or|not|eq|ne|lt|le|gt|ge|eqv|neqv)\.", s[i:])
            if dm:
                txt = dm.group(1)
            toks.append(("num", txt))
            i += len(txt)
            continue
        if c.isalpha() or c == "_":
            m = re.match(r"[a-z_]\w*", s[i:])
            toks.append(("name", m.group(0)))
            i += len(m.group(0))
            continue
        if c in "'\"":
            j = s.index(c, i + 1)
            toks.append(("str", s[i + 1:j]))
            i = j + 1
            continue
        two = s[i:i + 2]
        if two in ("**", "==", "/=", "<=", ">=", "//"):
            toks.append(("op", two))
            i += 2
            continue
        if c in "+-*/()<>,:%=":
            toks.append(("op", c))
            i += 1
            continue
        raise SyntaxError(f"cannot tokenize {s[i:]!r}")
    return toks


class Parser:
    """Pratt parser with Fortran precedence; produces tuples:
    ("num", text) ("str", s) ("bool", v) ("name", n) ("call", name, args)
    ("comp", base, field) ("bin", op, a, b) ("un", op, a) ("range", lo, hi)."""

    PREC = {"eqv": 1, "neqv": 1, "or": 2, "and": 3, "==": 5, "/=": 5, "<": 5, "<=": 5, ">": 5,
            ">=": 5, "//": 6, "+": 7, "-": 7, "*": 8, "/": 8, "**": 10}

    def __init__(self, toks):
        self.t = toks
        self.i = 0

    def peek(self):
        return self.t[self.i] if self.i < len(self.t) else (None, None)

    def take(self, kind=None, val=None):
        tk = self.peek()
        if (kind and tk[0] != kind) or (val and tk[1] != val):
            raise SyntaxError(f"expected {val or kind}, got {tk}")
        self.i += 1
        return tk

    def expr(self, minp=0):
        tk = self.peek()
        if tk == ("op", "-") or tk == ("op", "+"):
            self.i += 1
            a = self.expr(7)             # unary +/- bind like binary +/-
            left = ("un", tk[1], a) if tk[1] == "-" else a
        elif tk == ("op", "not"):
            self.i += 1
            left = ("un", "not", self.expr(4))
        else:
            left = self.primary()
        while True:
            tk = self.peek()
            if tk[0] != "op" or tk[1] not in self.PREC:
                break
            p = self.PREC[tk[1]]
            if p < minp:
                break
            self.i += 1
            right = self.expr(p if tk[1] == "**" else p + 1)
            left = ("bin", tk[1], left, right)
        return left

    def primary(self):
        tk = self.take()
        if tk[0] == "num":
            return ("num", tk[1])
        if tk[0] == "str":
            return ("str", tk[1])
        if tk == ("op", "TRUE"):
            return ("bool", True)
        if tk == ("op", "FALSE"):
            return ("bool", False)
        if tk == ("op", "("):
            e = self.expr()
            self.take("op", ")")
            return e
        if tk[0] == "name":
            node = ("name", tk[1])
            while True:
                nx = self.peek()
                if nx == ("op", "("):
                    self.i += 1
                    args = []
                    if self.peek() != ("op", ")"):
                        while True:
                            args.append(self.arg())
                            if self.peek() == ("op", ","):
                                self.i += 1
                                continue
                            break
                    self.take("op", ")")
                    node = ("call", node, args)
                elif nx == ("op", "%"):
                    self.i += 1
                    f = self.take("name")[1]
                    node = ("comp", node, f)
                else:
                    break
            return node
        raise SyntaxError(f"unexpected {tk}")

    def arg(self):
        # section a:b, :, a:, :b, or keyword=value
        if self.peek() == ("op", ":"):
            self.i += 1
            hi = None if self.peek() in (("op", ","), ("op", ")")) else self.expr()
            return ("range", None, hi)
        if self.peek()[0] == "name" and self.i + 1 < len(self.t) and self.t[self.i + 1] == ("op", "="):
            k = self.take("name")[1]
            self.take("op", "=")
            return ("kw", k, self.expr())
        e = self.expr()
        if self.peek() == ("op", ":"):
            self.i += 1
            hi = None if self.peek() in (("op", ","), ("op", ")")) else self.expr()
            return ("range", e, hi)
        return e


def parse_expr(s):
    p = Parser(tokenize(s))
    e = p.expr()
    if p.i != len(p.t):
        raise SyntaxError(f"trailing tokens in {s!r}: {p.t[p.i:]}")
    return e


# ---------------------------------------------------------------------------
# program structure
# ---------------------------------------------------------------------------


@dataclass
class Var:
    name: str
    kind: str                        # integer, real, complex, logical, char, type:<name>
    dims: list | None = None         # list of (lo_expr, hi_expr) or None; "deferred" for allocatable
    intent: str | None = None
    allocatable: bool = False
    init: str | None = None
    param: bool = False


@dataclass
class Proc:
    name: str
    kind: str                        # subroutine / function
    args: list
    result: str | None
    rtype: str | None
    body: list                       # Stmt list (executable, incl. declarations)
    module: "Module" = None
    vars: dict = field(default_factory=dict)
    uses: list = field(default_factory=list)
    implicit: bool = True


@dataclass
class Module:
    name: str
    uses: list = field(default_factory=list)
    vars: dict = field(default_factory=dict)
    types: dict = field(default_factory=dict)
    procs: dict = field(default_factory=dict)


_TYPE_RE = re.compile(r"^(integer|double precision|double complex|logical|character|real|complex|type\s*\(\s*\w+\s*\))"
                      r"(\s*\([^)]*\))?\s*(,[^:]*)?::?\s*(.*)$")
_TYPE_RE2 = re.compile(r"^(integer|double precision|double complex|logical|real|complex)\s+(\w.*)$")


def _kind_of(t):
    t = t.replace(" ", "")
    if t.startswith("integer"):
        return "integer"
    if t.startswith("doubleprecision") or t.startswith("real"):
        return "real"
    if t.startswith("doublecomplex") or t.startswith("complex"):
        return "complex"
    if t.startswith("logical"):
        return "logical"
    if t.startswith("character"):
        return "char"
    m = re.match(r"type\((\w+)\)", t)
    if m:
        return "type:" + m.group(1)
    raise SyntaxError(t)


def _split_top(s, sep=","):
    parts, depth, cur = [], 0, []
    for ch in s:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == sep and depth == 0:
            parts.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    if cur:
        parts.append("".join(cur))
    return [p.strip() for p in parts]


def parse_decl(text):
    """A type declaration statement -> list of Var, or None."""
    m = _TYPE_RE.match(text)
    if not m:
        m2 = _TYPE_RE2.match(text)
        if not m2 or "::" in text or text.startswith(("integer function", "double precision function",
                                                       "double complex function", "logical function")):
            return None
        tname, attrs, ents = m2.group(1), "", m2.group(2)
    else:
        tname, attrs, ents = m.group(1), (m.group(3) or ""), m.group(4)
        if " function " in " " + ents or ents.startswith("function"):
            return None
    kind = _kind_of(tname)
    intent = None
    alloc = False
    param = False
    dims_attr = None
    for a in _split_top(attrs.lstrip(","), ","):
        a = a.strip()
        if not a:
            continue
        if a.startswith("intent"):
            intent = re.search(r"\((\w+)\)", a).group(1)
        elif a == "allocatable":
            alloc = True
        elif a == "parameter":
            param = True
        elif a.startswith("dimension"):
            dims_attr = a[a.index("(") + 1:a.rindex(")")]
        elif a in ("public", "private", "save", "optional", "target", "pointer"):
            pass
        else:
            raise SyntaxError(f"attribute {a!r}")
    out = []
    for ent in _split_top(ents, ","):
        init = None
        if "=" in ent and "==" not in ent:
            ent, init = ent.split("=", 1)
            ent, init = ent.strip(), init.strip()
        mm = re.match(r"(\w+)\s*(\((.*)\))?$", ent)
        if not mm:
            raise SyntaxError(f"declaration entity {ent!r}")
        nm = mm.group(1)
        dspec = mm.group(3) if mm.group(2) else dims_attr
        dims = None
        if dspec is not None:
            dims = []
            for dd in _split_top(dspec, ","):
                if dd == ":":
                    dims.append("deferred")
                elif ":" in dd:
                    lo, hi = dd.split(":", 1)
                    dims.append((lo.strip(), hi.strip()))
                else:
                    dims.append(("1", dd.strip()))
        out.append(Var(nm, kind, dims, intent, alloc or (dims is not None and "deferred" in dims), init, param))
    return out


def parse_source(src, modules=None):
    """Modules and external procedures of one source file."""
    modules = {} if modules is None else modules
    st = statements(src)
    i = 0
    externals = {}
    while i < len(st):
        s = st[i].text
        m = re.match(r"module (\w+)$", s)
        if m:
            mod = Module(m.group(1))
            i += 1
            i0 = i
            in_type = None
            while not re.match(r"end module", st[i].text) and st[i].text != "contains":
                t = st[i].text
                tm = re.match(r"type(\s*,\s*\w+)?\s*(::)?\s*(\w+)$", t)
                if tm and not t.startswith("type("):
                    in_type = tm.group(3)
                    mod.types[in_type] = {}
                elif t.startswith("end type"):
                    in_type = None
                elif t.startswith("use "):
                    mod.uses.append(_parse_use(t))
                elif in_type is not None:
                    for v in parse_decl(t) or []:
                        mod.types[in_type][v.name] = v
                else:
                    decl = parse_decl(t)
                    if decl:
                        for v in decl:
                            mod.vars[v.name] = v
                i += 1
            mod_implicit = not any(x.text == "implicit none" for x in st[i0:i])
            if st[i].text == "contains":
                i += 1
                while not re.match(r"end module", st[i].text):
                    p, i = _parse_proc(st, i)
                    p.module = mod
                    p.implicit = p.implicit and mod_implicit
                    mod.procs[p.name] = p
            modules[mod.name] = mod
            i += 1
            continue
        if re.match(r"(\w[\w ]*\s)?(subroutine|function) ", s + " "):
            p, i = _parse_proc(st, i)
            externals[p.name] = p
            continue
        i += 1
    return modules, externals


def _parse_use(t):
    m = re.match(r"use\s+(\w+)\s*(,\s*only\s*:\s*(.*))?$", t)
    only = None
    if m.group(3) is not None:
        only = [x.strip() for x in m.group(3).split(",") if x.strip()]
    return (m.group(1), only)


_PROC_RE = re.compile(r"^((?:integer|double precision|double complex|logical|real)\s+)?(subroutine|function)\s+(\w+)"
                      r"\s*(\(([^)]*)\))?\s*(result\s*\(\s*(\w+)\s*\))?$")


def _parse_proc(st, i):
    s = st[i].text
    m = _PROC_RE.match(s)
    if not m:
        raise SyntaxError(f"line {st[i].line}: procedure header {s!r}")
    rtype = _kind_of(m.group(1).strip()) if m.group(1) else None
    kind, name = m.group(2), m.group(3)
    args = [a.strip() for a in (m.group(5) or "").split(",") if a.strip()]
    result = m.group(7) or (name if kind == "function" else None)
    body = []
    i += 1
    depth = 0
    while True:
        t = st[i].text
        if re.match(r"end\s*(subroutine|function)\b", t) or (t == "end" and depth == 0):
            break
        body.append(st[i])
        i += 1
    p = Proc(name, kind, args, result, rtype, body)
    p.implicit = not any(b.text == "implicit none" for b in body)
    for b in body:
        if b.text.startswith("use "):
            p.uses.append(_parse_use(b.text))
        else:
            decl = parse_decl(b.text)
            if decl:
                for v in decl:
                    p.vars[v.name] = v
    if kind == "function" and result not in p.vars:
        p.vars[result] = Var(result, rtype or "real")
    elif kind == "function" and rtype and p.vars[result].kind != rtype:
        p.vars[result].kind = rtype
    return p, i + 1


# ---------------------------------------------------------------------------
# translation
# ---------------------------------------------------------------------------

_INTRINSICS = {"btest", "ibset", "ibclr", "mod", "abs", "min", "max", "sqrt", "exp", "dble", "real", "int",
               "huge", "cmplx", "dcmplx", "sum", "allocated", "size"}
_EXTERNALS = {"mpi_allgatherv", "mpi_allgather", "mpi_allreduce", "mpi_bcast", "mpi_barrier", "mpi_wtime",
              "random_seed", "random_number", "daxpy", "dlamch", "dstevx", "die"}
_SKIP_CALLS = {"timestamp", "print_elapsed_time", "dump_hamiltonian"}


class Program:
    """Translated modules and external procedures, callable from Python."""

    def __init__(self, globals_init=None):
        self.modules = {}
        self.externals = {}
        self.ext = Externals()
        self.intr = type("ProgramIntrinsics", (Intrinsics,), {})   # per-program overrides
        self.O = Ops
        self.scope = {}              # module name -> dict of module variables
        self.funcs = {}              # (module or '', proc name) -> python function
        self.sources = {}

    def load(self, path, only=None):
        src = open(path).read()
        mods, exts = parse_source(src)
        for name, mod in mods.items():
            if only is not None:
                mod.procs = {k: v for k, v in mod.procs.items() if k in only.get(name, ())}
            self.modules[name] = mod
        for name, p in exts.items():
            if only is None or name in only.get("", ()):
                self.externals[name] = p
        self.sources[path] = src

    def module_vars(self, name):
        if name not in self.scope:
            sc = {}
            mod = self.modules.get(name)
            for vn, v in (mod.vars.items() if mod else ()):
                if v.dims is not None:
                    sc[vn] = None                 # allocatable or set by the caller
                elif v.kind.startswith("type:"):
                    sc[vn] = None
                elif v.init is not None:
                    try:
                        sc[vn] = conv_scalar(v.kind, eval(_const_expr(v.init, sc), {"math": math}))
                    except Exception:
                        sc[vn] = None
                else:
                    sc[vn] = conv_scalar(v.kind, 0) if v.kind != "char" else ""
            self.scope[name] = sc
        return self.scope[name]

    # -- name resolution ---------------------------------------------------
    def resolve(self, proc, name):
        """('local', Var) | ('module', modname, Var) | ('proc', key, Proc) | ('intrinsic',) | ('external',)."""
        if name in proc.vars:
            return ("local", proc.vars[name])
        mod = proc.module
        if mod is not None:
            if name in mod.procs:
                return ("proc", (mod.name, name), mod.procs[name])
            if name in mod.vars:
                return ("module", mod.name, mod.vars[name])
        for uses in ([proc.uses] + ([mod.uses] if mod else [])):
            for mname, only in uses:
                if only is not None and name not in only:
                    continue
                r = self._module_name(mname, name)
                if r:
                    return r
        if name in self.externals:
            return ("proc", ("", name), self.externals[name])
        if name in _INTRINSICS:
            return ("intrinsic",)
        if name in _EXTERNALS:
            return ("external",)
        if name in ("mpi_double_precision", "mpi_integer", "mpi_sum", "mpi_comm_world"):
            return ("const", 0)
        return None

    def _module_name(self, mname, name, seen=None):
        mod = self.modules.get(mname)
        if mod is None:
            return None
        if name in mod.procs:
            return ("proc", (mod.name, name), mod.procs[name])
        if name in mod.vars:
            return ("module", mod.name, mod.vars[name])
        seen = seen or set()
        if mname in seen:
            return None
        seen.add(mname)
        for m2, only in mod.uses:
            if only is not None and name not in only:
                continue
            r = self._module_name(m2, name, seen)
            if r:
                return r
        return None

    def init_scopes(self):
        for name in self.modules:
            self.module_vars(name)

    def proc(self, name, module=None):
        key = (module or "", name)
        if key not in self.funcs:
            p = self.modules[module].procs[name] if module else self.externals[name]
            self.funcs[key] = Translator(self, p).build()
        return self.funcs[key]

    def type_fields(self, tname):
        for mod in self.modules.values():
            if tname in mod.types:
                return mod.types[tname]
        raise KeyError(tname)

    def new_type(self, tname):
        obj = DerivedObj()
        for fname, v in self.type_fields(tname).items():
            setattr(obj, fname, None if v.dims is not None else conv_scalar(v.kind, 0))
        obj._type = tname
        return obj


class DerivedObj:
    pass


def _const_expr(text, scope):
    """A parameter's initialisation expression as Python (numbers, names of
    earlier parameters, + - * / ** and parentheses)."""
    out = []
    for kind, val in tokenize(text):
        if kind == "num":
            out.append(repr(float(val.replace("d", "e"))) if re.search(r"[.ed]", val) else val)
        elif kind == "name":
            if val in scope:
                out.append(repr(scope[val]))
            elif val == "atan":
                out.append("math.atan")
            else:
                raise NameError(val)
        elif kind == "str":
            out.append(repr(val))
        else:
            out.append(val)
    return " ".join(out)


class Translator:
    def __init__(self, prog: Program, p: Proc):
        self.prog = prog
        self.p = p
        self.lines = []
        self.tmp = 0
        self.implicit = []

    # -- helpers ----------------------------------------------------------
    def emit(self, depth, s):
        self.lines.append("    " * depth + s)

    def newtmp(self):
        self.tmp += 1
        return f"_t{self.tmp}"

    def var_of(self, name):
        r = self.prog.resolve(self.p, name)
        if r and r[0] == "local":
            return r[1]
        if r and r[0] == "module":
            return r[2]
        return None

    def is_array_name(self, name):
        v = self.var_of(name)
        return v is not None and v.dims is not None

    def ref(self, name):
        r = self.prog.resolve(self.p, name)
        if r is None and self.p.implicit:
            # implicit typing (no `implicit none`): i-n integer, else real
            self.p.vars[name] = Var(name, "integer" if name[0] in "ijklmn" else "real")
            self.implicit.append(name)
            r = self.prog.resolve(self.p, name)
        if r is None:
            raise NameError(f"{self.p.name}: unknown name {name!r}")
        if r[0] == "local":
            return name + "_"
        if r[0] == "module":
            return f"_M[{r[1]!r}][{name!r}]"
        if r[0] == "const":
            return "0"
        raise NameError(f"{self.p.name}: {name!r} is not a variable")

    def comp_field_var(self, node):
        """Declaration of the component a%b%c (for array-ness)."""
        base = node[1]
        if base[0] == "name":
            v = self.var_of(base[1])
            tname = v.kind.split(":", 1)[1]
        elif base[0] == "comp":
            tname = self.comp_field_var(base).kind.split(":", 1)[1]
        else:
            raise SyntaxError(node)
        return self.prog.type_fields(tname)[node[2]]

    def is_array_node(self, node):
        if node[0] == "name":
            return self.is_array_name(node[1])
        if node[0] == "comp":
            return self.comp_field_var(node).dims is not None
        return False

    # -- expressions -------------------------------------------------------
    def x(self, node):
        t = node[0]
        if t == "num":
            txt = node[1]
            if re.match(r"^\d+$", txt):
                return txt
            kind_d = "d" in txt
            val = txt.replace("d", "e")
            if "_" in val:
                val = val.split("_")[0]
            if kind_d:
                return repr(float(val))
            return repr(_f32(float(val)))              # default real literal: single precision
        if t == "str":
            return repr(node[1])
        if t == "bool":
            return repr(node[1])
        if t == "name":
            return self.ref(node[1])
        if t == "comp":
            return f"{self.x(node[1])}.{node[2]}"
        if t == "un":
            if node[1] == "not":
                return f"(not {self.x(node[2])})"
            return f"_O.neg({self.x(node[2])})"
        if t == "bin":
            op, a, b = node[1], self.x(node[2]), self.x(node[3])
            if op == "+":
                return f"_O.add({a}, {b})"
            if op == "-":
                return f"_O.sub({a}, {b})"
            if op == "*":
                return f"_O.mul({a}, {b})"
            if op == "/":
                return f"_O.div({a}, {b})"
            if op == "**":
                return f"_O.pow({a}, {b})"
            if op in ("==", "/=", "<", "<=", ">", ">="):
                py = {"==": "==", "/=": "!=", "<": "<", "<=": "<=", ">": ">", ">=": ">="}[op]
                return f"({a} {py} {b})"
            if op == "and":
                return f"({a} and {b})"
            if op == "or":
                return f"({a} or {b})"
            if op == "eqv":
                return f"(bool({a}) == bool({b}))"
            if op == "neqv":
                return f"(bool({a}) != bool({b}))"
            raise SyntaxError(op)
        if t == "call":
            return self.call_expr(node)
        raise SyntaxError(node)

    def subscripts(self, arr, args):
        """Python for element access or an Elems section."""
        if any(a[0] == "range" for a in args):
            spec = []
            for a in args:
                if a[0] == "range":
                    lo = "None" if a[1] is None else self.x(a[1])
                    hi = "None" if a[2] is None else self.x(a[2])
                    spec.append(f"({lo}, {hi})")
                else:
                    spec.append(self.x(a))
            return f"_sec({arr}, [{', '.join(spec)}])"
        idx = ", ".join(self.x(a) for a in args)
        if len(args) == 1:
            return f"{arr}.d[{self.x(args[0])} - {arr}.lb[0]]"
        return f"{arr}.d[{arr}.off(({idx},))]"

    def call_expr(self, node):
        head, args = node[1], node[2]
        if head[0] == "comp":
            return self.subscripts(self.x(head), args)
        name = head[1]
        r = self.prog.resolve(self.p, name)
        if r is None:
            raise NameError(f"{self.p.name}: unknown {name!r}")
        if r[0] in ("local", "module"):
            return self.subscripts(self.ref(name), args)
        if r[0] == "intrinsic":
            if name == "sum":
                return f"_I.sum({self.arr_value(args[0])})"
            if name == "allocated":
                return f"({self.x(args[0])} is not None)"
            return f"_I.{name}({', '.join(self.x(a) for a in args)})"
        if r[0] == "external":
            return f"_E.{name}({', '.join(self.x(a) for a in args)})"
        if r[0] == "proc":
            callee = r[2]
            return f"_P({name!r}, {r[1][0]!r})({', '.join(self.actual(callee, i, a) for i, a in enumerate(args))})[0]"
        raise NameError(name)

    def arr_value(self, node):
        """A whole array, section or elemental expression as a value."""
        return self.x(node)

    def actual(self, callee, i, node):
        """Actual argument i: arrays and derived objects by reference, the rest by value."""
        if node[0] == "call" and any(a[0] == "range" for a in node[2]):
            return self.x(node)                       # a section: Elems (copy-in)
        return self.x(node)

    # -- statements ---------------------------------------------------------
    def build(self):
        p = self.p
        argl = ", ".join(a + "_" for a in p.args)
        self.emit(0, f"def {p.name}_({argl}):")
        # locals: declarations with initialisation; explicit-shape arrays
        for name, v in p.vars.items():
            if name in p.args:
                continue
            if v.param:
                self.emit(1, f"{name}_ = {self.x(parse_expr(v.init))}")
                continue
            if v.kind.startswith("type:"):
                self.emit(1, f"{name}_ = _newtype({v.kind.split(':', 1)[1]!r})")
            elif v.dims is None:
                init = self.x(parse_expr(v.init)) if v.init else repr(conv_scalar(v.kind, 0))
                self.emit(1, f"{name}_ = {init}")
            elif v.allocatable:
                self.emit(1, f"{name}_ = None")
            else:
                self.emit(1, f"{name}_ = _FArray([{self.bounds(v.dims)}], {v.kind!r})")
        # dummy arrays: explicit shape declared in the procedure (sequence association)
        for a in p.args:
            v = p.vars.get(a)
            if v is not None and v.dims is not None and not v.allocatable:
                self.emit(1, f"{a}_ = _reshape({a}_, [{self.bounds(v.dims)}], {v.kind!r})")
            elif v is not None and v.dims is None and not v.kind.startswith("type:"):
                self.emit(1, f"{a}_ = _scalar_in({a}_, {v.kind!r})")
        head = self.lines
        self.lines = []
        self.block(p.body, 1)
        self.emit(1, "return _ret()")
        body = self.lines
        self.lines = head + [f"    {n}_ = {conv_scalar(p.vars[n].kind, 0)!r}" for n in self.implicit] + body
        # returns: function result first, then every scalar argument (by reference)
        rets = []
        if p.kind == "function":
            rets.append(f"{p.result}_")
        outs = [a for a in p.args if a in p.vars and p.vars[a].dims is None and not p.vars[a].kind.startswith("type:")]
        rets += [f"{a}_" for a in outs]
        src = "\n".join(self.lines)
        src = src.replace("return _ret()", f"return ({', '.join(rets)},)" if rets else "return (None,)")
        self.out_args = outs
        ns = {"_O": Ops, "_I": self.prog.intr, "_E": self.prog.ext, "_FArray": FArray, "_M": self.prog.scope,
              "_P": self.prog.proc, "_sec": _sec, "_sec_offsets": _sec_offsets, "_asg": _assign_array, "_reshape": _reshape,
              "_scalar_in": _scalar_in, "_newtype": self.prog.new_type, "_conv": conv_scalar, "math": math,
              "_alloc": _alloc, "_Exit": _Exit, "_Cycle": _Cycle}
        try:
            code = compile(src, f"<{p.module.name if p.module else ''}:{p.name}>", "exec")
        except SyntaxError as e:
            raise SyntaxError(f"translation of {p.name} failed: {e}\n{src}")
        exec(code, ns)
        fn = ns[f"{p.name}_"]
        fn.out_args = outs
        fn.source = src
        fn.proc = p
        return fn

    def bounds(self, dims):
        parts = []
        for d in dims:
            if d == "deferred":
                raise SyntaxError("deferred shape where explicit shape expected")
            lo, hi = d
            if hi == "*":
                parts.append(f"({self.x(parse_expr(lo))}, None)")
            else:
                parts.append(f"({self.x(parse_expr(lo))}, {self.x(parse_expr(hi))})")
        return ", ".join(parts)

    def block(self, stmts, depth):
        i = 0
        n = len(stmts)
        n0 = len(self.lines)
        while i < n:
            s = stmts[i]
            t = s.text
            if (t.startswith("use ") or t.startswith("implicit") or t.startswith("include")
                    or parse_decl(t) is not None or t in ("private", "public")):
                i += 1
                continue
            m = re.match(r"^(\w+\s*:\s*)?do\b(.*)$", t)
            if m and not re.match(r"^do\s*=", t):
                end = _find_end(stmts, i, "do")
                self.do(stmts[i], stmts[i + 1:end], depth)
                i = end + 1
                continue
            if re.match(r"^if\s*\(.*\)\s*then$", t):
                end, branches = _find_if(stmts, i)
                self.if_block(branches, depth)
                i = end + 1
                continue
            if re.match(r"^select case", t):
                end = _find_end(stmts, i, "select")
                self.select(stmts[i], stmts[i + 1:end], depth)
                i = end + 1
                continue
            self.simple(s, depth)
            i += 1
        if len(self.lines) == n0:
            self.emit(depth, "pass")

    def do(self, head, body, depth):
        t = re.sub(r"^\w+\s*:\s*", "", head.text)
        m = re.match(r"^do\s+(\w+)\s*=\s*(.*)$", t)
        if m:
            var = m.group(1)
            parts = _split_top(m.group(2), ",")
            lo, hi = self.x(parse_expr(parts[0])), self.x(parse_expr(parts[1]))
            step = self.x(parse_expr(parts[2])) if len(parts) > 2 else "1"
            v = self.ref(var)
            tl = self.newtmp()
            self.emit(depth, f"for {tl} in range({lo}, ({hi}) + (1 if ({step}) > 0 else -1), {step}):")
            self.emit(depth + 1, f"{v} = {tl}")
            self.block(body, depth + 1)
            return
        m = re.match(r"^do\s+while\s*\((.*)\)$", t)
        if m:
            cond = m.group(1).strip()
            c = "True" if cond in ("1", ".true.") else self.x(parse_expr(cond))
            self.emit(depth, f"while {c}:")
            self.block(body, depth + 1)
            return
        if t == "do":
            self.emit(depth, "while True:")
            self.block(body, depth + 1)
            return
        raise SyntaxError(head.text)

    def if_block(self, branches, depth):
        first = True
        for cond, body in branches:
            if cond is None:
                self.emit(depth, "else:")
            else:
                self.emit(depth, f"{'if' if first else 'elif'} {self.cond(cond)}:")
            self.block(body, depth + 1)
            first = False

    def cond(self, text):
        return self.x(parse_expr(text))

    def select(self, head, body, depth):
        sel = self.x(parse_expr(re.match(r"^select case\s*\((.*)\)$", head.text).group(1)))
        tv = self.newtmp()
        self.emit(depth, f"{tv} = {sel}")
        cases, cur = [], None
        for s in body:
            m = re.match(r"^case\s*(\((.*)\)|default)$", s.text)
            if m:
                cur = [m.group(2), []]
                cases.append(cur)
            elif cur is not None:
                cur[1].append(s)
        first = True
        for val, stmts in cases:
            if val is None:
                self.emit(depth, "else:" if not first else "if True:")
            else:
                vals = ", ".join(self.x(parse_expr(v)) for v in _split_top(val, ","))
                self.emit(depth, f"{'if' if first else 'elif'} {tv} in ({vals},):")
            self.block(stmts, depth + 1)
            first = False

    def simple(self, s, depth):
        t = s.text
        if t in ("cycle",) or re.match(r"^cycle\s+\w+$", t):
            self.emit(depth, "continue")
            return
        if t == "exit" or re.match(r"^exit\s+\w+$", t):
            self.emit(depth, "break")
            return
        if t == "return":
            self.emit(depth, "return _ret()")
            return
        if t == "stop" or t.startswith("stop "):
            self.emit(depth, "raise RuntimeError('stop in the reference')")
            return
        if re.match(r"^(print|write|open|close|read|flush|format)\b", t) or re.match(r"^\d+\s+format", t):
            return
        m = re.match(r"^if\s*\((.*)\)\s*(\w.*)$", t)
        if m and _balanced_if(t):
            cond, rest = _split_if(t)
            self.emit(depth, f"if {self.cond(cond)}:")
            self.simple(Stmt(rest, s.line, rest), depth + 1)
            return
        if t.startswith("call "):
            self.call_stmt(t[5:].strip(), depth)
            return
        if t.startswith("allocate"):
            for ent in _split_top(t[t.index("(") + 1:t.rindex(")")], ","):
                mm = re.match(r"(.+?)\((.*)\)$", ent)
                target, spec = mm.group(1), mm.group(2)
                node = parse_expr(target)
                dims = []
                for d in _split_top(spec, ","):
                    if ":" in d:
                        lo, hi = d.split(":", 1)
                    else:
                        lo, hi = "1", d
                    dims.append(f"({self.x(parse_expr(lo))}, {self.x(parse_expr(hi))})")
                kind = self.kind_of_node(node)
                self.emit(depth, f"{self.lvalue(node)} = _alloc([{', '.join(dims)}], {kind!r})")
            return
        if t.startswith("deallocate"):
            for ent in _split_top(t[t.index("(") + 1:t.rindex(")")], ","):
                self.emit(depth, f"{self.lvalue(parse_expr(ent))} = None")
            return
        if "=" in t:
            lhs, rhs = _split_assign(t)
            self.assign(lhs, rhs, depth)
            return
        raise SyntaxError(f"{self.p.name} line {s.line}: {s.raw}")

    def kind_of_node(self, node):
        if node[0] == "name":
            return self.var_of(node[1]).kind
        if node[0] == "comp":
            return self.comp_field_var(node).kind
        raise SyntaxError(node)

    def lvalue(self, node):
        if node[0] == "name":
            return self.ref(node[1])
        if node[0] == "comp":
            return f"{self.x(node[1])}.{node[2]}"
        raise SyntaxError(node)

    def assign(self, lhs_txt, rhs_txt, depth):
        lhs = parse_expr(lhs_txt)
        rhs = parse_expr(rhs_txt)
        if lhs[0] == "call":                           # element or section
            head, args = lhs[1], lhs[2]
            arr = self.x(head) if head[0] == "comp" else self.ref(head[1])
            kind = self.kind_of_node(head)
            if any(a[0] == "range" for a in args):
                offs = self.subscripts(arr, args).replace("_sec(", "_sec_offsets(", 1)
                self.emit(depth, f"_asg({arr}, {offs}, {self.x(rhs)})")
                return
            if len(args) == 1:
                self.emit(depth, f"{arr}.d[{self.x(args[0])} - {arr}.lb[0]] = _conv({kind!r}, {self.x(rhs)})")
            else:
                idx = ", ".join(self.x(a) for a in args)
                self.emit(depth, f"{arr}.d[{arr}.off(({idx},))] = _conv({kind!r}, {self.x(rhs)})")
            return
        if self.is_array_node(lhs):                    # whole array
            arr = self.lvalue(lhs)
            self.emit(depth, f"_asg({arr}, range(len({arr}.d)), {self.x(rhs)})")
            return
        kind = self.kind_of_node(lhs) if lhs[0] in ("name", "comp") else None
        if kind and kind.startswith("type:"):
            self.emit(depth, f"{self.lvalue(lhs)} = {self.x(rhs)}")
            return
        self.emit(depth, f"{self.lvalue(lhs)} = _conv({kind!r}, {self.x(rhs)})")

    def call_stmt(self, t, depth):
        node = parse_expr(t) if "(" in t else ("call", ("name", t), [])
        name = node[1][1]
        args = node[2]
        if name in _SKIP_CALLS:
            return
        r = self.prog.resolve(self.p, name)
        if r is None:                 # a procedure that is not loaded: an error only if reached
            self.emit(depth, f"raise RuntimeError({f'{self.p.name}: call to {name}, which is not loaded'!r})")
            return
        if r[0] == "external":
            tv = self.newtmp()
            self.emit(depth, f"{tv} = _E.{name}({', '.join(self.x(a) for a in args)})")
            # outputs the shim returns by dummy name: map onto the actual arguments
            shim = getattr(self.prog.ext, name)
            import inspect
            pnames = list(inspect.signature(shim).parameters)
            for i, a in enumerate(args):
                if i < len(pnames):
                    pn = pnames[i]
                    self.emit(depth, f"if {pn!r} in {tv}: {self._store(a, f'{tv}[{pn!r}]')}")
            return
        if r[0] != "proc":
            raise NameError(f"{name} is not a procedure")
        callee = r[2]
        tv = self.newtmp()
        self.emit(depth, f"{tv} = _P({name!r}, {r[1][0]!r})({', '.join(self.actual(callee, i, a) for i, a in enumerate(args))})")
        # scalar dummies come back: store into scalar actual variables
        outs = [i for i, a in enumerate(callee.args) if a in callee.vars and callee.vars[a].dims is None
                and not callee.vars[a].kind.startswith("type:") and callee.vars[a].intent in ("out", "inout", None)]
        k0 = 1 if callee.kind == "function" else 0
        allouts = [a for a in callee.args if a in callee.vars and callee.vars[a].dims is None
                   and not callee.vars[a].kind.startswith("type:")]
        for i in outs:
            if i >= len(args):
                continue
            pos = allouts.index(callee.args[i]) + k0
            a = args[i]
            if a[0] in ("name", "comp") or (a[0] == "call" and not any(x[0] == "range" for x in a[2])):
                if a[0] == "name" and self.var_of(a[1]) is None:
                    continue
                if a[0] == "name" and self.var_of(a[1]).param:
                    continue
                if a[0] == "call" and a[1][0] == "name" and self.prog.resolve(self.p, a[1][1])[0] == "proc":
                    continue
                self.emit(depth, self._store(a, f"{tv}[{pos}]"))

    def _store(self, node, value):
        if node[0] == "name":
            v = self.var_of(node[1])
            if v is None:
                return "pass"
            if v.dims is not None:
                return f"_asg({self.ref(node[1])}, range(len({self.ref(node[1])}.d)), {value})"
            return f"{self.ref(node[1])} = _conv({v.kind!r}, {value})"
        if node[0] == "comp":
            fv = self.comp_field_var(node)
            if fv.dims is not None:
                return f"{self.lvalue(node)} = {value}"
            return f"{self.lvalue(node)} = _conv({fv.kind!r}, {value})"
        if node[0] == "call":
            head, args = node[1], node[2]
            arr = self.x(head) if head[0] == "comp" else self.ref(head[1])
            kind = self.kind_of_node(head)
            if len(args) == 1:
                return f"{arr}.d[{self.x(args[0])} - {arr}.lb[0]] = _conv({kind!r}, {value})"
            idx = ", ".join(self.x(a) for a in args)
            return f"{arr}.d[{arr}.off(({idx},))] = _conv({kind!r}, {value})"
        return "pass"


class _Exit(Exception):
    pass


class _Cycle(Exception):
    pass


def _alloc(bounds, kind):
    return FArray(bounds, kind)


def _sec(arr, spec):
    return Elems([arr.d[o] for o in arr.section(spec)])


def _sec_offsets(arr, spec):
    return arr.section(spec)


def _reshape(actual, bounds, kind):
    """A dummy array of explicit shape over the actual argument's storage
    (sequence association): the same list when the sizes agree."""
    if isinstance(actual, Elems):
        a = FArray([(1, len(actual.v))], kind)
        a.d = list(actual.v)
        actual = a
    storage = actual.d.base if isinstance(actual.d, _Window) else actual.d
    out = FArray.__new__(FArray)
    lb = [b[0] for b in bounds]
    ext = []
    for b in bounds:
        ext.append(len(actual.d) if b[1] is None else max(b[1] - b[0] + 1, 0))
    st, s = [], 1
    for e in ext:
        st.append(s)
        s *= e
    if s > len(storage):
        raise ValueError(f"dummy array of {s} elements over an actual of {len(storage)}")
    out.lb, out.ext, out.st, out.kind = lb, ext, st, kind
    out.d = storage if s == len(storage) else _Window(storage, s)   # shares storage
    return out


class _Window(list):
    """The leading part of an actual array's storage, written through."""

    def __init__(self, base, n):
        super().__init__()
        self.base = base
        self.n = n

    def __len__(self):
        return self.n

    def __getitem__(self, i):
        if isinstance(i, slice):
            return [self.base[j] for j in range(*i.indices(self.n))]
        if i >= self.n or i < -self.n:
            raise IndexError(i)
        return self.base[i]

    def __setitem__(self, i, v):
        if i >= self.n:
            raise IndexError(i)
        self.base[i] = v

    def __iter__(self):
        return (self.base[i] for i in range(self.n))


def _scalar_in(v, kind):
    if isinstance(v, Elems):
        raise TypeError("array passed to a scalar dummy")
    return conv_scalar(kind, v) if v is not None else v


def _find_end(stmts, i, kind):
    depth = 0
    for j in range(i, len(stmts)):
        t = stmts[j].text
        if kind == "do":
            if re.match(r"^(\w+\s*:\s*)?do\b", t) and not re.match(r"^do\s*=", t):
                depth += 1
            elif re.match(r"^end\s*do\b", t):
                depth -= 1
                if depth == 0:
                    return j
        elif kind == "select":
            if t.startswith("select case"):
                depth += 1
            elif re.match(r"^end\s*select", t):
                depth -= 1
                if depth == 0:
                    return j
    raise SyntaxError(f"unterminated {kind} at line {stmts[i].line}")


def _find_if(stmts, i):
    depth = 0
    branches = []
    cond = _if_cond(stmts[i].text)
    cur = []
    for j in range(i + 1, len(stmts)):
        t = stmts[j].text
        if re.match(r"^if\s*\(.*\)\s*then$", t):
            depth += 1
            cur.append(stmts[j])
            continue
        if re.match(r"^end\s*if\b", t):
            if depth == 0:
                branches.append((cond, cur))
                return j, branches
            depth -= 1
            cur.append(stmts[j])
            continue
        if depth == 0 and re.match(r"^else\s*if\s*\(.*\)\s*then$", t):
            branches.append((cond, cur))
            cond, cur = _if_cond(re.sub(r"^else\s*", "", t)), []
            continue
        if depth == 0 and t == "else":
            branches.append((cond, cur))
            cond, cur = None, []
            continue
        cur.append(stmts[j])
    raise SyntaxError(f"unterminated if at line {stmts[i].line}")


def _if_cond(t):
    t = re.sub(r"^if\s*", "", t)
    t = re.sub(r"\s*then$", "", t)
    assert t.startswith("(") and t.endswith(")")
    return t[1:-1]


def _balanced_if(t):
    cond, rest = _split_if(t)
    return rest is not None and not rest.startswith("then")


def _split_if(t):
    i = t.index("(")
    depth = 0
    for j in range(i, len(t)):
        if t[j] == "(":
            depth += 1
        elif t[j] == ")":
            depth -= 1
            if depth == 0:
                return t[i + 1:j], t[j + 1:].strip() or None
    return None, None


def _split_assign(t):
    depth = 0
    for j, ch in enumerate(t):
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == "=" and depth == 0 and t[j - 1] not in "=/<>" and (j + 1 >= len(t) or t[j + 1] != "="):
            return t[:j].strip(), t[j + 1:].strip()
    raise SyntaxError(t)
