"""Runs T-Flows' own Fortran source for the Native_Mod solver path.

TEST INFRASTRUCTURE ONLY.  Used by tests/golden/make_golden.py and by the
CPU test tests/test_reference_exec.py to pin the C++ oracle (tf_oracle.cpp)
to the reference itself.  It reads the reference's .f90 files, so it works
only where the T-Flows tree is present (this build container, not the GPU
box); nothing in the product, smoke() or bench.py imports it.

No Fortran compiler exists on either machine this project builds or runs on,
so the reference cannot be compiled.  Instead this module translates the
subset of free-form Fortran 2008 that the path's source files use into
Python and executes it:

    Sources/Process/Cpu/Native_Mod/{Solve_Native,Cg,Bicg,Prec_Form,
        Prec_Solve,Residual_Vector,Normalized_Root_Mean_Square,
        Root_Mean_Square}.f90
    Sources/Process/Cpu/Solver_Mod/Set_Singular.f90
    constants from Sources/Shared/Const_Mod.f90 and
        Sources/Process/Cpu/Solver_Mod.f90 (parameter statements)

Semantics kept from the reference's GNU build (makefile: gfortran -O3
-fdefault-real-8, no -ffast-math, no -march): every `real` is an IEEE double,
literals included; expressions are evaluated in source order with no fused
multiply-add (Python floats round every operation); `x**2` with an integer
literal exponent is x*x, as gfortran expands it; loop reductions run in
serial order (the `!$omp` directives are comments; one thread); DO loops
leave their variable at lower + trips * step on normal completion;
assumed-shape dummies start at 1, explicit-shape dummies at their declared
lower bound, pointers keep their target's bounds; scalar dummies are passed
by reference (written back after the call); string comparison ignores
trailing blanks; a real division by zero gives the IEEE infinity or NaN
as the hardware does; MAX/MIN keep their first argument unless a later one
compares greater (smaller), so a NaN first argument stays.  Every array
access is bounds-checked.

The services the path calls are replaced by one-process stand-ins, as the
sequential build's stubs do (Sources/Shared/Comm_Mod/Sequential): the
Global % Sum/Min/Max reductions return their argument, halo exchange does
nothing, Work % Connect_Real_Cell hands out arrays of bounds
(-n_bnd_cells:n_cells) filled with NaN (so a read before a write would
poison the result), Profiler calls do nothing, Message % Error raises.

Anything outside the subset raises FortranSubsetError at translation time.
"""
import math
import os
import re

REF_ROOT = os.environ.get("TFLOWS_REFERENCE", "/root/reference")

PATH_FILES = [
    "Sources/Process/Cpu/Native_Mod/Solve_Native.f90",
    "Sources/Process/Cpu/Native_Mod/Cg.f90",
    "Sources/Process/Cpu/Native_Mod/Bicg.f90",
    "Sources/Process/Cpu/Native_Mod/Prec_Form.f90",
    "Sources/Process/Cpu/Native_Mod/Prec_Solve.f90",
    "Sources/Process/Cpu/Native_Mod/Residual_Vector.f90",
    "Sources/Process/Cpu/Native_Mod/Normalized_Root_Mean_Square.f90",
    "Sources/Process/Cpu/Native_Mod/Root_Mean_Square.f90",
    "Sources/Process/Cpu/Solver_Mod/Set_Singular.f90",
]
CONST_FILES = [
    "Sources/Shared/Const_Mod.f90",
    "Sources/Process/Cpu/Solver_Mod.f90",
]


class FortranSubsetError(Exception):
    pass


class FortranRuntimeError(Exception):
    def __init__(self, code, msg):
        super().__init__(f"Message % Error({code}): {msg}")
        self.code = code


class _Goto(Exception):
    def __init__(self, label):
        self.label = label


class _Return(Exception):
    pass


def available(root=REF_ROOT):
    return all(os.path.exists(os.path.join(root, f)) for f in PATH_FILES + CONST_FILES)


# ---------------------------------------------------------------------------
# Run-time objects
# ---------------------------------------------------------------------------
class FArray:
    """A Fortran array view: element k lives at d[base + k - lo]."""
    __slots__ = ("d", "base", "lo", "n", "o")

    def __init__(self, d, base, lo, n):
        self.d, self.base, self.lo, self.n = d, base, lo, n
        self.o = base - lo

    def g(self, k):
        if not (self.lo <= k < self.lo + self.n):
            raise IndexError(f"index {k} outside ({self.lo}:{self.lo + self.n - 1})")
        return self.d[k + self.o]

    def s(self, k, v):
        if not (self.lo <= k < self.lo + self.n):
            raise IndexError(f"index {k} outside ({self.lo}:{self.lo + self.n - 1})")
        self.d[k + self.o] = v

    def values(self):
        return self.d[self.base:self.base + self.n]


def farray(values, lo=1, real=True):
    vals = [float(v) for v in values] if real else [int(v) for v in values]
    return FArray(vals, 0, lo, len(vals))


def _sec(a, lo, hi):
    if lo is None:
        lo = a.lo
    if hi is None:
        hi = a.lo + a.n - 1
    n = max(0, hi - lo + 1)
    if n and not (a.lo <= lo and hi <= a.lo + a.n - 1):
        raise IndexError(f"section ({lo}:{hi}) outside ({a.lo}:{a.lo + a.n - 1})")
    return FArray(a.d, a.base + (lo - a.lo), 1, n)


def _assumed(a):
    """Assumed-shape dummy: lower bound 1."""
    return a if a is None else FArray(a.d, a.base, 1, a.n)


def _explicit(a, lo, hi):
    """Explicit-shape dummy (lo:hi), sequence-associated with the actual."""
    n = hi - lo + 1
    if a.n < n:
        raise IndexError(f"actual of {a.n} elements for a dummy of ({lo}:{hi})")
    return FArray(a.d, a.base, lo, n)


def _fill(a, v):
    for k in range(a.n):
        a.d[a.base + k] = v


def _trip(lo, hi, st):
    q = hi - lo + st
    if q == 0 or (q > 0) != (st > 0):
        return 0
    return abs(q) // abs(st)


def _idiv(a, b):
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


def _rdiv(a, b):
    """IEEE division (Python raises on a zero divisor, the hardware does not)."""
    try:
        return a / b
    except ZeroDivisionError:
        if a != a or a == 0:
            return math.nan
        return math.copysign(math.inf, a) * math.copysign(1.0, b)


def _div(a, b):
    if isinstance(a, int) and isinstance(b, int):
        return _idiv(a, b)
    return _rdiv(a, b)


def _streq(a, b):
    if isinstance(a, str):
        return a.rstrip() == b.rstrip()
    return a == b


def _fmax(*a):
    m = a[0]
    for v in a[1:]:
        if v > m:
            m = v
    return m


def _fmin(*a):
    m = a[0]
    for v in a[1:]:
        if v < m:
            m = v
    return m


def _int(v):
    return int(v)   # truncation toward zero, as INT()


def _unsupported(name):
    raise FortranSubsetError(f"call of {name} reached (outside the stand-ins)")


class _Obj:
    """A derived-type value (attributes are the lower-case component names)."""

    def __init__(self, **kw):
        self.__dict__.update(kw)


class _Global:
    """Comm_Mod's Global in a one-process run (Sequential/Global stubs)."""

    def sum_real(self, v):
        return v

    def sum_int(self, v):
        return v

    def min_real(self, v):
        return v

    def max_real(self, v):
        return v


class _Profiler:
    def start(self, *a):
        pass

    def stop(self, *a):
        pass


class _Message:
    def error(self, code, msg, **kw):
        raise FortranRuntimeError(code, msg)


class _Grid(_Obj):
    def exchange_cells_real(self, *a):
        pass


class _Work:
    """Work_Mod's pool of cell arrays, bounds (-n_bnd_cells:n_cells)."""

    def __init__(self, nb, nc):
        self.nb, self.nc = nb, nc

    def connect_real_cell(self, count):
        return [FArray([math.nan] * (self.nb + self.nc + 1), 0, -self.nb, self.nb + self.nc + 1)
                for _ in range(count)]

    def disconnect_real_cell(self, *a):
        pass


# ---------------------------------------------------------------------------
# Source reading
# ---------------------------------------------------------------------------
def _strip_comment(line):
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


def logical_lines(text):
    """Free-form source -> [(first line number, statement text)]."""
    out, buf, start = [], "", None
    for no, raw in enumerate(text.splitlines(), 1):
        if raw.lstrip().startswith("#"):
            continue
        s = _strip_comment(raw).strip()
        if not s:
            continue
        if buf and s.startswith("&"):
            s = s[1:].lstrip()
        if start is None:
            start = no
        if s.endswith("&"):
            buf += s[:-1] + " "
            continue
        buf += s
        out.append((start, buf.strip()))
        buf, start = "", None
    return out


# ---------------------------------------------------------------------------
# Expressions
# ---------------------------------------------------------------------------
_TOKEN = re.compile(r"""
    (?P<ws>\s+)
  | (?P<str>'(?:[^']|'')*'|"(?:[^"]|"")*")
  | (?P<dotop>\.(?:eq|ne|lt|le|gt|ge|and|or|not|eqv|neqv|true|false)\.)
  | (?P<real>(?:\d+\.(?!(?:eq|ne|lt|le|gt|ge|and|or|not|eqv|neqv)\.)\d*|\.\d+)(?:[eEdD][+-]?\d+)?
             |\d+[eEdD][+-]?\d+)
  | (?P<int>\d+)
  | (?P<name>[A-Za-z_]\w*)
  | (?P<op>\*\*|//|==|/=|<=|>=|=>|[-+*/()<>=,:%])
""", re.X | re.I)

_PY_KEYWORDS = {"global", "lambda", "pass", "in", "is", "not", "and", "or", "def", "class",
                "from", "import", "return", "if", "else", "elif", "for", "while", "try",
                "except", "raise", "with", "as", "del", "yield", "assert", "break",
                "continue", "finally", "none", "true", "false", "nonlocal", "async",
                "await"}


def pyname(n):
    n = n.lower()
    return n + "_" if n in _PY_KEYWORDS else n


def tokenize(s):
    toks, pos = [], 0
    while pos < len(s):
        m = _TOKEN.match(s, pos)
        if not m:
            raise FortranSubsetError(f"cannot tokenize {s[pos:]!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        toks.append((kind, m.group(kind)))
    return toks


# Types of the derived-type components the path reads
# (Matrix_Type, Grid_Type, Comm_Type, Native_Type, Var_Type, Solver_Type).
_COMPONENTS = {
    "val": ("r", True), "col": ("i", True), "row": ("i", True), "dia": ("i", True),
    "n_cells": ("i", False), "n_bnd_cells": ("i", False), "n_buff_cells": ("i", False),
    "solvers": ("i", False), "pnt_grid": ("o", False), "comm": ("o", False),
    "pnt_matrix": ("o", False),
}

_STUB_OBJECTS = {"global": "global_", "profiler": "profiler", "message": "message",
                 "work": "work"}


class _Expr:
    """Recursive-descent translator of one Fortran expression to Python."""

    def __init__(self, unit, toks):
        self.u, self.t, self.i = unit, toks, 0

    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else (None, None)

    def take(self, val=None):
        tok = self.peek()
        if val is not None and (tok[1] is None or tok[1].lower() != val):
            raise FortranSubsetError(f"expected {val!r}, got {tok!r}")
        self.i += 1
        return tok

    def at(self, *vals):
        v = self.peek()[1]
        return v is not None and v.lower() in vals

    def done(self):
        return self.i >= len(self.t)

    # precedence climbing -------------------------------------------------
    def expr(self):
        return self.p_or()

    def p_or(self):
        c, t = self.p_and()
        while self.at(".or."):
            self.take()
            c2, _ = self.p_and()
            c, t = f"({c} or {c2})", "l"
        return c, t

    def p_and(self):
        c, t = self.p_not()
        while self.at(".and."):
            self.take()
            c2, _ = self.p_not()
            c, t = f"({c} and {c2})", "l"
        return c, t

    def p_not(self):
        if self.at(".not."):
            self.take()
            c, _ = self.p_not()
            return f"(not {c})", "l"
        return self.p_rel()

    _REL = {".eq.": "==", "==": "==", ".ne.": "!=", "/=": "!=", ".lt.": "<", "<": "<",
            ".le.": "<=", "<=": "<=", ".gt.": ">", ">": ">", ".ge.": ">=", ">=": ">="}

    def p_rel(self):
        c, t = self.p_concat()
        v = (self.peek()[1] or "").lower()
        if v in self._REL:
            self.take()
            c2, t2 = self.p_concat()
            op = self._REL[v]
            if op in ("==", "!=") and ("s" in (t, t2) or "?" in (t, t2)):
                e = f"_streq({c}, {c2})"
                return (e if op == "==" else f"(not {e})"), "l"
            return f"({c} {op} {c2})", "l"
        return c, t

    def p_concat(self):
        c, t = self.p_add()
        while self.at("//"):
            self.take()
            c2, _ = self.p_add()
            c, t = f"({c} + {c2})", "s"
        return c, t

    @staticmethod
    def _num(t1, t2):
        if t1 == "r" or t2 == "r":
            return "r"
        if t1 == "i" and t2 == "i":
            return "i"
        return "?"

    def p_add(self):
        if self.at("+", "-"):
            op = self.take()[1]
            c, t = self.p_mul()
            c = f"(-{c})" if op == "-" else c
        else:
            c, t = self.p_mul()
        while self.at("+", "-"):
            op = self.take()[1]
            c2, t2 = self.p_mul()
            c, t = f"({c} {op} {c2})", self._num(t, t2)
        return c, t

    def p_mul(self):
        c, t = self.p_pow()
        while self.at("*", "/"):
            op = self.take()[1]
            c2, t2 = self.p_pow()
            if op == "*":
                c, t = f"({c} * {c2})", self._num(t, t2)
            elif t == "i" and t2 == "i":
                c, t = f"_idiv({c}, {c2})", "i"
            elif "r" in (t, t2):
                c, t = f"_rdiv({c}, {c2})", "r"
            else:
                c, t = f"_div({c}, {c2})", "?"
        return c, t

    def p_pow(self):
        c, t = self.p_unary_primary()
        if self.at("**"):
            self.take()
            if self.peek()[0] == "int" and not self.at_op_after(1, "**"):
                n = int(self.take()[1])
                if n == 2:
                    return f"({c} * {c})", t
                if n == 1:
                    return c, t
                raise FortranSubsetError(f"integer power {n}")
            c2, t2 = self.p_pow()
            return f"({c} ** {c2})", self._num(t, t2)
        return c, t

    def at_op_after(self, k, op):
        return (self.peek(k)[1] or "") == op

    def p_unary_primary(self):
        if self.at("-", "+"):     # gfortran extension: a * -b
            op = self.take()[1]
            c, t = self.p_pow()
            return (f"(-{c})" if op == "-" else c), t
        return self.primary()

    def primary(self):
        kind, v = self.peek()
        if kind is None:
            raise FortranSubsetError("unexpected end of expression")
        if kind == "real":
            self.take()
            s = v.lower().replace("d", "e")
            if s.endswith("."):
                s += "0"
            s = re.sub(r"\.e", ".0e", s)
            return repr(float(s)), "r"
        if kind == "int":
            self.take()
            return str(int(v)), "i"
        if kind == "str":
            self.take()
            q = v[0]
            return repr(v[1:-1].replace(q + q, q)), "s"
        if kind == "dotop":
            if v.lower() in (".true.", ".false."):
                self.take()
                return ("True" if v.lower() == ".true." else "False"), "l"
        if v == "(":
            self.take()
            c, t = self.expr()
            self.take(")")
            return f"({c})", t
        if kind == "name":
            return self.designator()
        raise FortranSubsetError(f"unexpected token {v!r}")

    def arglist(self):
        """After '(' : returns [(kind, payload)] with kind 'sec', 'kw' or 'x'."""
        args = []
        if self.at(")"):
            self.take()
            return args
        while True:
            if self.peek()[0] == "name" and self.at_op_after(1, "=") and \
                    not self.at_op_after(1, "=="):
                kw = self.take()[1].lower()
                self.take("=")
                args.append(("kw", (kw, self.expr())))
            elif self.at(":"):
                self.take()
                hi = None if self.at(",", ")") else self.expr()
                args.append(("sec", (None, hi)))
            else:
                e = self.expr()
                if self.at(":"):
                    self.take()
                    hi = None if self.at(",", ")") else self.expr()
                    args.append(("sec", (e, hi)))
                else:
                    args.append(("x", e))
            if self.at(","):
                self.take()
                continue
            self.take(")")
            return args

    def designator(self):
        """name[(args)] {% name[(args)]} -> (code, type)."""
        parts = []
        while True:
            name = self.take()[1]
            args = None
            if self.at("("):
                self.take()
                args = self.arglist()
            parts.append((name, args))
            if self.at("%"):
                self.take()
                continue
            break
        return self.u.designator_code(parts)


# ---------------------------------------------------------------------------
# Program units
# ---------------------------------------------------------------------------
_DECL = re.compile(r"^(real|integer|logical|character(?:\s*\([^)]*\))?|class\s*\([^)]*\)|"
                   r"type\s*\([^)]*\))\s*(,[^:]*)?::\s*(.*)$", re.I)
_HEAD = re.compile(r"^(?:(real|integer|logical)\s+)?(subroutine|function)\s+(\w+)\s*"
                   r"\(([^)]*)\)\s*$", re.I)


def _split_top(s, sep=","):
    out, depth, cur = [], 0, ""
    q = None
    for ch in s:
        if q:
            cur += ch
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == sep and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


class Var:
    def __init__(self, name, base, shape, attrs):
        self.name, self.base, self.shape, self.attrs = name, base, shape, attrs

    @property
    def is_array(self):
        return self.shape is not None

    @property
    def scalar_type(self):
        return {"real": "r", "integer": "i", "logical": "l", "character": "s"}.get(self.base, "o")


class Unit:
    def __init__(self, name, kind, rtype, dummies, src, lineno):
        self.name, self.kind, self.rtype = name.lower(), kind, rtype
        self.dummies = [d.strip().lower() for d in dummies.split(",") if d.strip()]
        self.src, self.lineno = src, lineno
        self.vars = {}
        self.body = []        # logical lines of the executable part
        self.program = None   # set by Program

    # declarations --------------------------------------------------------
    def declare(self, text):
        m = _DECL.match(text)
        if not m:
            return False
        tspec, attrs, ents = m.group(1).lower(), (m.group(2) or "").lower(), m.group(3)
        base = tspec.split("(")[0].strip()
        base = {"class": "derived", "type": "derived"}.get(base, base)
        attr = [a.strip() for a in _split_top(attrs.lstrip(","))] if attrs else []
        for ent in _split_top(ents):
            mm = re.match(r"^(\w+)\s*(\((.*)\))?\s*(=.*)?$", ent, re.S)
            if not mm:
                raise FortranSubsetError(f"declaration entity {ent!r}")
            name = mm.group(1).lower()
            shape = None
            if mm.group(2):
                shape = []
                for dim in _split_top(mm.group(3)):
                    if ":" in dim and dim.strip() != ":":
                        lo, hi = dim.split(":", 1) if dim.count(":") == 1 else _split_top(dim, ":")
                        shape.append((lo.strip(), hi.strip()))
                    elif dim.strip() == ":":
                        shape.append((None, None))
                    else:
                        shape.append(("1", dim.strip()))
                if len(shape) != 1:
                    raise FortranSubsetError(f"rank {len(shape)} array {name}")
            self.vars[name] = Var(name, base, shape, attr)
        return True

    # expression helpers ---------------------------------------------------
    def expr(self, text_or_toks):
        toks = tokenize(text_or_toks) if isinstance(text_or_toks, str) else text_or_toks
        e = _Expr(self, toks)
        c, t = e.expr()
        if not e.done():
            raise FortranSubsetError(f"trailing tokens in {text_or_toks!r}")
        return c, t

    def var_code(self, name):
        n = name.lower()
        if n in self.vars or n in self.dummies:
            return pyname(n)
        if n == self.name and self.kind == "function":
            return "_result"
        if n in self.program.consts:
            return repr(self.program.consts[n])
        if n in _STUB_OBJECTS:
            return _STUB_OBJECTS[n]
        if n == "__line__":
            return "0"
        if n == "__file__":
            return repr(os.path.basename(self.src))
        raise FortranSubsetError(f"{self.name}: unknown name {name}")

    def var_type(self, name):
        n = name.lower()
        v = self.vars.get(n)
        if v is not None:
            return v.scalar_type, v.is_array
        if n in self.program.consts:
            return ("r" if isinstance(self.program.consts[n], float) else "i"), False
        if n == self.name and self.kind == "function":
            return {"real": "r", "integer": "i"}.get(self.rtype, "?"), False
        if n == "__file__":
            return "s", False
        return "o", False

    def _index_code(self, arr, args):
        if len(args) != 1:
            raise FortranSubsetError("rank-1 arrays only")
        kind, payload = args[0]
        if kind == "sec":
            lo = "None" if payload[0] is None else payload[0][0]
            hi = "None" if payload[1] is None else payload[1][0]
            return f"_sec({arr}, {lo}, {hi})", True
        if kind != "x":
            raise FortranSubsetError("keyword in an array reference")
        return f"{arr}.g({payload[0]})", False

    def designator_code(self, parts):
        name0, args0 = parts[0]
        n0 = name0.lower()
        intr = {"sqrt": ("_sqrt", "r"), "abs": ("abs", None), "max": ("_fmax", None),
                "min": ("_fmin", None), "real": ("float", "r"), "dble": ("float", "r"),
                "int": ("_int", "i"), "trim": (None, "s")}
        if len(parts) == 1:
            if args0 is not None and n0 == "present" and n0 not in self.vars:
                return f"({self.var_code(args0[0][1][0])} is not None)", "l"
            if args0 is not None and n0 in intr and n0 not in self.vars:
                fn, rt = intr[n0]
                cs = [a[1][0] for a in args0 if a[0] == "x"]
                ts = [a[1][1] for a in args0 if a[0] == "x"]
                if n0 == "trim":
                    return f"({cs[0]}).rstrip()", "s"
                if rt is None:
                    rt = "r" if "r" in ts else ("i" if all(t == "i" for t in ts) else "?")
                return f"{fn}({', '.join(cs)})", rt
            if args0 is not None and n0 in self.program.units and n0 not in self.vars:
                return self.program.call_code(self, None, n0, args0, want_value=True)
            base = self.var_code(name0)
            st, is_arr = self.var_type(name0)
            if args0 is None:
                return base, st
            code, sec = self._index_code(base, args0)
            return code, ("a" if sec else st)
        # component chain
        code = self.var_code(name0)
        if args0 is not None:
            code, _ = self._index_code(code, args0)
        st = "o"
        for k, (nm, args) in enumerate(parts[1:], 1):
            n = nm.lower()
            last = k == len(parts) - 1
            if last and n in self.program.units:
                return self.program.call_code(self, code, n, args or [], want_value=True)
            code = f"{code}.{pyname(n)}"
            st, is_arr = _COMPONENTS.get(n, ("o", False))
            if args is not None:
                code, sec = self._index_code(code, args)
                if sec:
                    st = "a"
        return code, st


class Program:
    """All translated units plus the constants they read."""

    def __init__(self, root=REF_ROOT):
        self.root = root
        self.consts = {}
        self.units = {}
        for f in CONST_FILES:
            self._read_consts(os.path.join(root, f))
        for f in PATH_FILES:
            self._read_unit(os.path.join(root, f))
        self.ns = {
            "_sec": _sec, "_assumed": _assumed, "_explicit": _explicit, "_fill": _fill,
            "_trip": _trip, "_idiv": _idiv, "_div": _div, "_rdiv": _rdiv, "_streq": _streq,
            "_fmax": _fmax, "_fmin": _fmin, "_int": _int, "_sqrt": math.sqrt,
            "_Goto": _Goto, "_Return": _Return, "_unsupported": _unsupported,
            "global_": _Global(), "profiler": _Profiler(), "message": _Message(),
            "work": None,
        }
        self.code = {}
        for u in self.units.values():
            src = self._translate(u)
            self.code[u.name] = src
            exec(compile(src, f"<{os.path.basename(u.src)}>", "exec"), self.ns)

    # constants -------------------------------------------------------------
    def _read_consts(self, path):
        with open(path) as fh:
            text = fh.read()
        for _, line in logical_lines(text):
            m = re.match(r"^(real|integer)\s*,\s*parameter\s*::\s*(.*)$", line, re.I)
            if not m:
                continue
            for ent in _split_top(m.group(2)):
                if "=" not in ent:
                    continue
                name, val = ent.split("=", 1)
                name = name.strip().lower()
                toks = tokenize(val.strip())
                if len(toks) == 1 and toks[0][0] in ("real", "int"):
                    v = toks[0][1].lower().replace("d", "e")
                    if m.group(1).lower() == "real":
                        v = v + "0" if v.endswith(".") else re.sub(r"\.e", ".0e", v)
                        self.consts[name] = float(v)
                    else:
                        self.consts[name] = int(v)
                elif len(toks) == 1 and toks[0][0] == "name" and \
                        toks[0][1].lower() in self.consts:
                    self.consts[name] = self.consts[toks[0][1].lower()]

    # units -----------------------------------------------------------------
    def _read_unit(self, path):
        with open(path) as fh:
            lines = logical_lines(fh.read())
        unit = None
        in_decl = True
        for no, text in lines:
            low = text.lower()
            m = _HEAD.match(text)
            if m and unit is None:
                unit = Unit(m.group(3), m.group(2).lower(), (m.group(1) or "").lower(),
                            m.group(4), path, no)
                continue
            if unit is None:
                continue
            if re.match(r"^end\s*(subroutine|function)\b", low):
                self.units[unit.name] = unit
                unit.program = self
                unit = None
                continue
            if in_decl:
                if low == "implicit none" or re.match(r"^unused\s*\(", low):
                    continue
                if unit.declare(text):
                    continue
                in_decl = False
            if re.match(r"^unused\s*\(", low):
                continue
            unit.body.append((no, text))
        if unit is not None:
            raise FortranSubsetError(f"{path}: unterminated unit")

    def call_code(self, unit, obj, name, args, want_value=False):
        """Code that calls translated unit `name` (obj = passed object)."""
        callee = self.units[name]
        actual = [] if obj is None else [obj]
        for kind, payload in args:
            if kind == "kw":
                raise FortranSubsetError(f"keyword argument in a call of {name}")
            if kind == "sec":
                raise FortranSubsetError("bare section as an argument")
            actual.append(payload[0])
        if len(actual) > len(callee.dummies):
            raise FortranSubsetError(f"too many arguments for {name}")
        call = f"P_{name}({', '.join(actual)})"
        if want_value:
            if callee.kind != "function":
                raise FortranSubsetError(f"subroutine {name} used as a value")
            rt = {"real": "r", "integer": "i"}.get(callee.rtype, "?")
            return f"{call}[0]", rt
        return call

    # statements ------------------------------------------------------------
    def _translate(self, u):
        out = []
        ind = "    "
        sig = []
        for d in u.dummies:
            v = u.vars.get(d)
            opt = v is not None and "optional" in v.attrs
            sig.append(f"{pyname(d)}=None" if opt else pyname(d))
        out.append(f"def P_{u.name}({', '.join(sig)}):")
        # dummy arrays take the bounds their declarations give
        for d in u.dummies:
            v = u.vars.get(d)
            if v is None or not v.is_array or "pointer" in v.attrs:
                continue
            lo, hi = v.shape[0]
            if lo is None:
                out.append(f"{ind}{pyname(d)} = _assumed({pyname(d)})")
            else:
                lc, _ = u.expr(lo)
                hc, _ = u.expr(hi)
                out.append(f"{ind}{pyname(d)} = _explicit({pyname(d)}, {lc}, {hc})")
        for name, v in u.vars.items():
            if name not in u.dummies:
                out.append(f"{ind}{pyname(name)} = None")
        out.append(f"{ind}_result = None")
        out.append(f"{ind}try:")
        body = self._block(u, u.body, 2)
        out.extend(body if body else [ind * 2 + "pass"])
        out.append(f"{ind}except _Return:")
        out.append(f"{ind * 2}pass")
        out.append(f"{ind}return [_result, [{', '.join(pyname(d) for d in u.dummies)}]]")
        return "\n".join(out) + "\n"

    def _block(self, u, stmts, depth):
        """Statements at one level, with forward GOTOs to top-level labels."""
        # labels at this level: `N continue`
        labels = [k for k, (_, t) in enumerate(stmts) if re.match(r"^\d+\s+continue$", t, re.I)]
        if labels and depth != 2:
            raise FortranSubsetError("labels inside a block")
        if labels:
            out, prev = [], 0
            # nest: try { seg0 } except goto L0 ; seg1 ...
            lines = []
            for li in labels:
                lab = int(stmts[li][1].split()[0])
                seg = self._seq(u, stmts[prev:li], depth + len(labels) - labels.index(li))
                lines.append((lab, seg))
                prev = li + 1
            ind = "    "
            # innermost first: build text bottom-up
            text = lines[0][1] or [ind * (depth + len(labels)) + "pass"]
            for k, (lab, seg) in enumerate(lines):
                d = depth + len(labels) - k - 1
                block = [ind * d + "try:"] + text + [
                    ind * d + "except _Goto as _g:",
                    ind * (d + 1) + f"if _g.label != {lab}:",
                    ind * (d + 2) + "raise"]
                nxt = lines[k + 1][1] if k + 1 < len(lines) else None
                text = block + (nxt if nxt else [])
            out = text + self._seq(u, stmts[prev:], depth)
            return out
        return self._seq(u, stmts, depth)

    def _seq(self, u, stmts, depth):
        out = []
        ind = "    "
        k = 0
        loops = 0
        while k < len(stmts):
            no, t = stmts[k]
            low = t.lower()
            pad = ind * depth
            m_if = re.match(r"^if\s*\(", low)
            m_do = re.match(r"^do\s+(\w+)\s*=\s*(.*)$", low)
            if m_if:
                cond, rest = self._paren_after(t, "if")
                if rest.lower() == "then":
                    # collect the if-block and its branches
                    branches, k = self._collect_if(stmts, k, cond)
                    first = True
                    for c, blk in branches:
                        if c is None:
                            out.append(pad + "else:")
                        else:
                            cc, _ = u.expr(c)
                            out.append(pad + ("if " if first else "elif ") + cc + ":")
                        first = False
                        body = self._block(u, blk, depth + 1)
                        out.extend(body if body else [pad + ind + "pass"])
                    continue
                cc, _ = u.expr(cond)
                out.append(pad + f"if {cc}:")
                out.extend(self._simple(u, rest, depth + 1, no))
                k += 1
                continue
            if m_do:
                var = m_do.group(1)
                bounds = _split_top(t[t.index("=") + 1:])
                if len(bounds) not in (2, 3):
                    raise FortranSubsetError(f"line {no}: DO bounds {t!r}")
                blk, k = self._collect_do(stmts, k)
                loops += 1
                tag = f"{depth}_{loops}"
                lo, _ = u.expr(bounds[0])
                hi, _ = u.expr(bounds[1])
                st = u.expr(bounds[2])[0] if len(bounds) == 3 else "1"
                v = u.var_code(var)
                out.append(pad + f"_lo{tag} = {lo}; _hi{tag} = {hi}; _st{tag} = {st}")
                out.append(pad + f"for {v} in range(_lo{tag}, _hi{tag} + (1 if _st{tag} > 0 "
                                 f"else -1), _st{tag}):")
                body = self._block(u, blk, depth + 1)
                out.extend(body if body else [pad + ind + "pass"])
                out.append(pad + "else:")
                out.append(pad + ind + f"{v} = _lo{tag} + _trip(_lo{tag}, _hi{tag}, _st{tag})"
                                        f" * _st{tag}")
                continue
            if re.match(r"^(end\s*if|else|end\s*do|enddo)\b", low):
                raise FortranSubsetError(f"line {no}: unmatched {t!r}")
            out.extend(self._simple(u, t, depth, no))
            k += 1
        return out

    @staticmethod
    def _paren_after(t, kw):
        s = t[len(kw):].lstrip()
        if not s.startswith("("):
            raise FortranSubsetError(f"expected '(' after {kw}: {t!r}")
        depth = 0
        for i, ch in enumerate(s):
            depth += ch == "("
            depth -= ch == ")"
            if depth == 0:
                return s[1:i], s[i + 1:].strip()
        raise FortranSubsetError(f"unbalanced: {t!r}")

    def _collect_if(self, stmts, k, cond):
        branches = [[cond, []]]
        depth = 0
        k += 1
        while k < len(stmts):
            no, t = stmts[k]
            low = t.lower()
            opens_if = re.match(r"^if\s*\(", low) and self._paren_after(t, "if")[1].lower() == "then"
            if opens_if or re.match(r"^do\b", low):
                depth += 1
            elif re.match(r"^(end\s*if|end\s*do|enddo)\b", low):
                if depth == 0:
                    if not re.match(r"^end\s*if", low):
                        raise FortranSubsetError(f"line {no}: {t!r} closes an IF")
                    return branches, k + 1
                depth -= 1
            elif depth == 0 and re.match(r"^else\s*if\s*\(", low):
                c, rest = self._paren_after(re.sub(r"^else\s*", "", t, flags=re.I), "if")
                if rest.lower() != "then":
                    raise FortranSubsetError(f"line {no}: {t!r}")
                branches.append([c, []])
                k += 1
                continue
            elif depth == 0 and low == "else":
                branches.append([None, []])
                k += 1
                continue
            branches[-1][1].append(stmts[k])
            k += 1
        raise FortranSubsetError("unterminated IF")

    def _collect_do(self, stmts, k):
        blk, depth = [], 0
        k += 1
        while k < len(stmts):
            no, t = stmts[k]
            low = t.lower()
            opens_if = re.match(r"^if\s*\(", low) and self._paren_after(t, "if")[1].lower() == "then"
            if opens_if or re.match(r"^do\b", low):
                depth += 1
            elif re.match(r"^(end\s*if|end\s*do|enddo)\b", low):
                if depth == 0:
                    if re.match(r"^end\s*if", low):
                        raise FortranSubsetError(f"line {no}: END IF closes a DO")
                    return blk, k + 1
                depth -= 1
            blk.append(stmts[k])
            k += 1
        raise FortranSubsetError("unterminated DO")

    def _simple(self, u, t, depth, no):
        pad = "    " * depth
        low = t.lower().strip()
        if low == "exit":
            return [pad + "break"]
        if low == "cycle":
            return [pad + "continue"]
        if low == "return":
            return [pad + "raise _Return()"]
        m = re.match(r"^go\s*to\s+(\d+)$", low)
        if m:
            return [pad + f"raise _Goto({int(m.group(1))})"]
        if low.startswith("call "):
            return [pad + c for c in self._call(u, t[5:].strip(), no)]
        toks = tokenize(t)
        # assignment / pointer assignment at depth 0 of parentheses
        depth_p, split, op = 0, None, None
        for i, (kind, v) in enumerate(toks):
            if v == "(":
                depth_p += 1
            elif v == ")":
                depth_p -= 1
            elif depth_p == 0 and v in ("=", "=>"):
                split, op = i, v
                break
        if split is None:
            raise FortranSubsetError(f"line {no}: statement {t!r}")
        rhs, rt = u.expr(toks[split + 1:])
        lhs_t = toks[:split]
        if op == "=>":
            e = _Expr(u, lhs_t)
            lc, _ = e.designator()
            return [pad + f"{lc} = {rhs}"]
        # lhs
        if len(lhs_t) == 1:
            name = lhs_t[0][1]
            st, is_arr = u.var_type(name)
            lc = u.var_code(name)
            if is_arr:
                return [pad + f"_fill({lc}, {self._conv(st, rhs, rt)})"]
            return [pad + f"{lc} = {self._conv(st, rhs, rt)}"]
        e = _Expr(u, lhs_t)
        # element store: rewrite the final `.g(idx)` of the designator into `.s(idx, v)`
        code, st = e.designator()
        if not e.done():
            raise FortranSubsetError(f"line {no}: left side {t!r}")
        if code.startswith("_sec("):
            return [pad + f"_fill({code}, {rhs})"]
        split = self._last_access(code)
        if split is None:
            # component scalar store (obj.attr = v)
            return [pad + f"{code} = {rhs}"]
        return [pad + f"{split[0]}.s({split[1]}, {self._conv(st, rhs, rt)})"]

    @staticmethod
    def _last_access(code):
        """'obj.g(idx)' -> ('obj', 'idx') for the access whose ')' ends code."""
        if not code.endswith(")"):
            return None
        for m in re.finditer(r"\.g\(", code):
            depth = 0
            for i in range(m.end() - 1, len(code)):
                depth += code[i] == "("
                depth -= code[i] == ")"
                if depth == 0:
                    break
            if i == len(code) - 1:
                return code[:m.start()], code[m.end():-1]
        return None

    @staticmethod
    def _conv(st, code, rt):
        if st == "r" and rt != "r":
            return f"float({code})"
        if st == "i" and rt != "i":
            return f"_int({code})"
        return code

    def _call(self, u, t, no):
        toks = tokenize(t)
        e = _Expr(u, toks)
        parts = []
        while True:
            name = e.take()[1]
            args = None
            if e.at("("):
                e.take()
                args = e.arglist()
            parts.append((name, args))
            if e.at("%"):
                e.take()
                continue
            break
        if not e.done():
            raise FortranSubsetError(f"line {no}: call {t!r}")
        meth, args = parts[-1][0].lower(), parts[-1][1] or []
        if len(parts) == 1:
            obj = None
            if meth not in self.units:
                return [f"_unsupported({meth!r})"]
        else:
            obj, _ = u.designator_code(parts[:-1])
        if meth in self.units:
            callee = self.units[meth]
            code = ["_r = " + self.call_code(u, obj, meth, args)]
            actual_names = ([None] if obj is not None else []) + [
                self._bare_name(a) for a in args]
            for k, nm in enumerate(actual_names):
                if nm is None or k >= len(callee.dummies):
                    continue
                dv = callee.vars.get(callee.dummies[k])
                if dv is None or dv.is_array or dv.base == "derived":
                    continue
                if any(i in ("intent(in)",) for i in dv.attrs):
                    continue
                lv = u.vars.get(nm)
                if lv is None or lv.is_array:
                    continue
                code.append(f"{pyname(nm)} = _r[1][{k}]")
            return code
        # stand-ins
        xs = [a[1][0] for a in args if a[0] == "x"]
        kws = [f"{a[1][0]}={a[1][1][0]}" for a in args if a[0] == "kw"]
        if any(a[0] == "sec" for a in args):
            raise FortranSubsetError(f"line {no}: bare section argument")
        if meth == "connect_real_cell":
            names = [self._bare_name(a) for a in args]
            if any(n is None for n in names):
                raise FortranSubsetError(f"line {no}: Connect_Real_Cell of non-names")
            return [f"{', '.join(pyname(n) for n in names)}, = "
                    f"{obj}.connect_real_cell({len(names)})"]
        if meth in ("sum_real", "sum_int", "min_real", "max_real"):
            nm = self._bare_name(args[0])
            if nm is None:
                raise FortranSubsetError(f"line {no}: reduction of an expression")
            return [f"{pyname(nm)} = {obj}.{meth}({xs[0]})"]
        return [f"{obj}.{pyname(meth)}({', '.join(xs + kws)})"]

    @staticmethod
    def _bare_name(a):
        if a[0] != "x":
            return None
        code = a[1][0]
        return code.rstrip("_") if re.match(r"^[a-z_]\w*$", code) else None


# ---------------------------------------------------------------------------
# Driver
# ---------------------------------------------------------------------------
_PROGRAM = None


def program():
    global _PROGRAM
    if _PROGRAM is None:
        if not available():
            raise FileNotFoundError("the T-Flows sources are not present")
        _PROGRAM = Program()
    return _PROGRAM


def _system(row, col, dia, val, n_bnd=0):
    n = len(row) - 1
    grid = _Grid(n_cells=n, n_bnd_cells=n_bnd, comm=_Obj(n_buff_cells=0))
    a = _Obj(val=farray(val), col=farray(col, real=False), row=farray(row, real=False),
             dia=farray(dia, real=False), pnt_grid=grid)
    nat = _Obj(pnt_grid=grid)
    return grid, a, nat


def solve_native(solver, prec, row, col, dia, val, x, b, miter, tol, norm=None, n_bnd=2):
    """Native_Type % Solve_Native of the reference source on one system.

    row/col/dia are 1-based (Matrix_Type), x the initial guess x(1:n).
    Returns dict(x, val, b, niter, fin_res) with x, val, b as lists in the
    state the reference leaves them (val and b rescaled, x the solution)."""
    P = program()
    grid, a, nat = _system(row, col, dia, val, n_bnd)
    n = grid.n_cells
    P.ns["work"] = _Work(n_bnd, n)
    # x(-n_bnd:n): boundary entries and x(0) hold a value no solver may read
    xa = FArray([7.0e300] * (n_bnd + 1) + [float(v) for v in x], 0, -n_bnd, n_bnd + 1 + n)
    ba = farray(b)
    prec_s = prec.ljust(80)
    args = [nat, solver, prec_s, a, xa, ba, int(miter), 0, float(tol), 0.0]
    if norm is not None:
        args.append(float(norm))
    r = P.ns["P_solve_native"](*args)
    dummies = P.units["solve_native"].dummies
    fin = dict(zip(dummies, r[1]))
    return dict(x=xa.values()[n_bnd + 1:], val=a.val.values(), b=ba.values(),
                niter=fin["niter"], fin_res=fin["fin_res"])


def set_singular(row, dia, val):
    """Solver_Type % Set_Singular (NATIVE solvers) of the reference source."""
    P = program()
    grid, a, nat = _system(row, [1] * (len(val)), dia, val)
    sol = _Obj(solvers=P.consts.get("native", 1))
    phi = _Obj(pnt_matrix=a)
    P.ns["P_set_singular"](sol, phi)
    return a.val.values()


def nrms(row, dia, val, r, x, norm=None):
    """Nat % Normalized_Root_Mean_Square of the reference source."""
    P = program()
    grid, a, nat = _system(row, [1] * len(val), dia, val)
    args = [nat, grid.n_cells, farray(r), a, farray(x)]
    if norm is not None:
        args.append(float(norm))
    return P.ns["P_normalized_root_mean_square"](*args)[0]


if __name__ == "__main__":
    P = program()
    for name, src in P.code.items():
        print(f"# ---- {name}")
        print(src)
