"""Interpreter for the Fortran 2008 subset the reference program uses.

No Fortran compiler exists in this image, and the reference (2d_mrlbm.f90,
2d_statistics.f90) has no tests or golden vectors.  This module executes the reference's
own source text so its outputs can pin the C++ oracle: it parses the program (free form,
continuation lines, `;` separators, labels), compiles every statement to Python closures
and runs them with Fortran semantics where they matter for the numbers:

  * kinds: default INTEGER, REAL (single precision, emulated with numpy.float32),
    REAL(8)/DOUBLE PRECISION (IEEE double, Python float); mixed operations promote to the
    wider kind; a literal without a d exponent is single precision (so `16.0/36.0` is a
    float32 division, as in 2d_mrlbm.f90:129);
  * expressions evaluate left to right with Fortran precedence, `x**2` is `x*x`, integer
    division truncates toward zero; no operation is fused or re-associated (the x86-64
    gfortran -O3 build the reference uses emits no FMA and does not re-associate without
    -ffast-math); intrinsic SUM accumulates in array-element order;
  * arrays keep their declared lower bounds, column-major; sections are numpy views;
  * dummy arguments are passed by reference (array elements and whole arrays included);
  * file I/O is captured in memory: every WRITE appends a record of values to its file,
    namelist READs parse input.dat, unformatted READs take records supplied by the caller.

It is test infrastructure: only tests/golden/make_golden.py uses it, to write fixtures.
"""
import math
import re

import numpy as np

I4, R4, R8, LOG, CHR = "i", "r4", "r8", "l", "c"
_RANK = {I4: 0, R4: 1, R8: 2}


class FortranStop(Exception):
    pass


class _Exit(Exception):
    pass


class _Cycle(Exception):
    pass


# ---------------------------------------------------------------------------------------
# values
def kind_of(v):
    if isinstance(v, np.ndarray):
        d = v.dtype
        if d == np.float64:
            return R8
        if d == np.float32:
            return R4
        if d == np.bool_:
            return LOG
        if d.kind in "iu":
            return I4
        return CHR
    if isinstance(v, bool) or isinstance(v, np.bool_):
        return LOG
    if isinstance(v, (int, np.integer)):
        return I4
    if isinstance(v, np.float32):
        return R4
    if isinstance(v, float):
        return R8
    if isinstance(v, str):
        return CHR
    raise TypeError(f"no Fortran kind for {type(v)}")


def to_kind(v, k):
    if isinstance(v, np.ndarray):
        if k == R8:
            return v.astype(np.float64, copy=False)
        if k == R4:
            return v.astype(np.float32, copy=False)
        if k == I4:
            return v if v.dtype.kind in "iu" else np.trunc(v).astype(np.int64)
        if k == LOG:
            return v.astype(bool, copy=False)
        return v
    if k == R8:
        return float(v)
    if k == R4:
        return np.float32(v)
    if k == I4:
        return int(v)
    if k == LOG:
        return bool(v)
    return v


def promote(a, b):
    ka, kb = kind_of(a), kind_of(b)
    if ka == kb:
        return a, b, ka
    if ka in _RANK and kb in _RANK:
        k = ka if _RANK[ka] > _RANK[kb] else kb
        return to_kind(a, k), to_kind(b, k), k
    return a, b, ka


def _idiv(a, b):
    if isinstance(a, np.ndarray) or isinstance(b, np.ndarray):
        a = np.asarray(a)
        b = np.asarray(b)
        return np.sign(a) * np.sign(b) * (np.abs(a) // np.abs(b))
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


def arith(op, a, b):
    a, b, k = promote(a, b)
    if op == "+":
        return a + b
    if op == "-":
        return a - b
    if op == "*":
        return a * b
    if op == "/":
        if k == I4:
            return _idiv(a, b)
        return a / b
    if op == "**":
        if kind_of(b) == I4 and not isinstance(b, np.ndarray) and k != I4:
            n = int(b)
            if n == 2:
                return a * a
            r = a
            for _ in range(n - 1):
                r = r * a
            return r
        return a ** b
    raise ValueError(op)


class FArray:
    """A Fortran array: numpy data (column-major) plus per-dimension lower bounds."""

    __slots__ = ("data", "lb")

    def __init__(self, data, lb):
        self.data = data
        self.lb = tuple(lb)

    def index(self, subs):
        out = []
        for d, s in enumerate(subs):
            lb = self.lb[d]
            if isinstance(s, tuple):          # section (lo, hi) with None = bound
                lo = lb if s[0] is None else s[0]
                hi = lb + self.data.shape[d] - 1 if s[1] is None else s[1]
                out.append(slice(lo - lb, hi - lb + 1))
            else:
                out.append(s - lb)
        return tuple(out)


# ---------------------------------------------------------------------------------------
# source preparation
def logical_lines(text):
    """Free-form source -> list of (label, statement) with continuations joined."""
    raw = text.split("\n")
    out, buf = [], ""
    for line in raw:
        s = _strip_comment(line)
        if not s.strip():
            if buf:
                continue
            continue
        st = s.strip()
        if buf:
            if st.startswith("&"):
                st = st[1:]
            buf += " " + st
        else:
            buf = st
        if buf.rstrip().endswith("&"):
            buf = buf.rstrip()[:-1]
            continue
        for part in _split_semicolons(buf):
            part = part.strip()
            if not part:
                continue
            m = re.match(r"^(\d+)\s+(.*)$", part)
            if m:
                out.append((int(m.group(1)), m.group(2).strip()))
            else:
                out.append((None, part))
        buf = ""
    return out


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


def _split_semicolons(s):
    parts, q, cur = [], None, ""
    for ch in s:
        if q:
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
        elif ch == ";":
            parts.append(cur)
            cur = ""
            continue
        cur += ch
    parts.append(cur)
    return parts


# ---------------------------------------------------------------------------------------
# lexer / expression parser
_TOK = re.compile(r"""
   (?P<ws>\s+)
  |(?P<real>(?:\d+\.\d*|\.\d+)(?:[eEdD][+-]?\d+)?|\d+[eEdD][+-]?\d+)
  |(?P<int>\d+)
  |(?P<str>'(?:[^']|'')*'|"(?:[^"]|"")*")
  |(?P<dot>\.(?:and|or|not|eqv|neqv|eq|ne|lt|le|gt|ge|true|false)\.)
  |(?P<op>\*\*|//|==|/=|<=|>=|\(/|/\)|::|[-+*/()=<>,:%])
  |(?P<name>[A-Za-z_]\w*)
""", re.X | re.I)


def tokenize(s):
    toks, pos = [], 0
    while pos < len(s):
        m = _TOK.match(s, pos)
        if not m:
            raise SyntaxError(f"cannot tokenize at {s[pos:pos + 20]!r} in {s!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        v = m.group(kind)
        if kind == "dot":
            v = v.lower()
        if kind == "name":
            v = v.lower()
        toks.append((kind, v))
    return toks


class Parser:
    def __init__(self, toks):
        self.t = toks
        self.i = 0

    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else (None, None)

    def eat(self, v=None):
        tok = self.peek()
        if v is not None and tok[1] != v:
            raise SyntaxError(f"expected {v!r}, got {tok!r} in {self.t}")
        self.i += 1
        return tok

    def at(self, v):
        return self.peek()[1] == v

    def expr(self):
        return self.eqv()

    def eqv(self):
        a = self.or_()
        while self.at(".eqv.") or self.at(".neqv."):
            op = self.eat()[1]
            a = ("bin", op, a, self.or_())
        return a

    def or_(self):
        a = self.and_()
        while self.at(".or."):
            self.eat()
            a = ("bin", ".or.", a, self.and_())
        return a

    def and_(self):
        a = self.not_()
        while self.at(".and."):
            self.eat()
            a = ("bin", ".and.", a, self.not_())
        return a

    def not_(self):
        if self.at(".not."):
            self.eat()
            return ("not", self.not_())
        return self.rel()

    _REL = {"==": "==", "/=": "/=", "<": "<", "<=": "<=", ">": ">", ">=": ">=", ".eq.": "==", ".ne.": "/=",
            ".lt.": "<", ".le.": "<=", ".gt.": ">", ".ge.": ">="}

    def rel(self):
        a = self.concat()
        if self.peek()[1] in self._REL:
            op = self._REL[self.eat()[1]]
            a = ("rel", op, a, self.concat())
        return a

    def concat(self):
        a = self.add()
        while self.at("//"):
            self.eat()
            a = ("cat", a, self.add())
        return a

    def add(self):
        if self.at("-") or self.at("+"):
            op = self.eat()[1]
            t = self.mul()
            a = ("neg", t) if op == "-" else t
        else:
            a = self.mul()
        while self.at("+") or self.at("-"):
            op = self.eat()[1]
            a = ("bin", op, a, self.mul())
        return a

    def mul(self):
        a = self.power()
        while self.at("*") or self.at("/"):
            op = self.eat()[1]
            a = ("bin", op, a, self.power())
        return a

    def power(self):
        a = self.unary_primary()
        if self.at("**"):
            self.eat()
            return ("bin", "**", a, self.power())
        return a

    def unary_primary(self):
        if self.at("-"):
            self.eat()
            return ("neg", self.power())
        return self.primary()

    def primary(self):
        kind, v = self.peek()
        if kind == "real":
            self.eat()
            return ("const", _real_literal(v))
        if kind == "int":
            self.eat()
            return ("const", int(v))
        if kind == "str":
            self.eat()
            q = v[0]
            return ("const", v[1:-1].replace(q + q, q))
        if kind == "dot" and v in (".true.", ".false."):
            self.eat()
            return ("const", v == ".true.")
        if v == "(/":
            self.eat()
            items = []
            while not self.at("/)"):
                items.append(self.expr())
                if self.at(","):
                    self.eat()
            self.eat("/)")
            return ("ctor", items)
        if v == "(":
            self.eat()
            e = self.expr()
            self.eat(")")
            return ("paren", e)
        if kind == "name":
            self.eat()
            if self.at("("):
                self.eat()
                args = []
                while not self.at(")"):
                    args.append(self.subscript())
                    if self.at(","):
                        self.eat()
                self.eat(")")
                return ("call", v, args)
            return ("name", v)
        raise SyntaxError(f"unexpected token {self.peek()} in {self.t}")

    def subscript(self):
        # a:b, :, a:, :b, name=value (keyword argument) or plain expression
        if self.peek()[0] == "name" and self.peek(1)[1] == "=" and self.peek(2)[1] != "=":
            name = self.eat()[1]
            self.eat("=")
            return ("kw", name, self.expr())
        lo = hi = None
        if not self.at(":"):
            lo = self.expr()
            if not self.at(":"):
                return lo
        self.eat(":")
        if not (self.at(",") or self.at(")")):
            hi = self.expr()
        return ("range", lo, hi)


def _real_literal(s):
    t = s.lower()
    if "d" in t:
        return float(t.replace("d", "e"))
    return np.float32(float(t))


def parse_expr(s):
    p = Parser(tokenize(s))
    e = p.expr()
    if p.peek()[0] is not None:
        raise SyntaxError(f"trailing tokens in {s!r}")
    return e


def split_top(s, sep=","):
    """Split on `sep` at parenthesis depth 0, outside strings."""
    parts, depth, q, cur = [], 0, None, ""
    for ch in s:
        if q:
            if ch == q:
                q = None
            cur += ch
            continue
        if ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == sep and depth == 0:
            parts.append(cur)
            cur = ""
            continue
        cur += ch
    parts.append(cur)
    return [p.strip() for p in parts]


def match_paren(s, start):
    """Index of the parenthesis closing the one at s[start]."""
    depth, q = 0, None
    for i in range(start, len(s)):
        ch = s[i]
        if q:
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
            if depth == 0:
                return i
    raise SyntaxError(f"unbalanced parentheses in {s!r}")


# ---------------------------------------------------------------------------------------
# program structure
class Decl:
    def __init__(self, name, ftype, dims, init, intent, parameter):
        self.name, self.ftype, self.dims, self.init = name, ftype, dims, init
        self.intent, self.parameter = intent, parameter


class Unit:
    """The main program or one internal subroutine."""

    def __init__(self, name, args):
        self.name = name
        self.args = args
        self.decls = {}
        self.namelists = {}
        self.body = []          # list of (label, stmt)
        self.formats = {}


def _parse_type(spec):
    s = spec.strip().lower().replace(" ", "")
    if s.startswith("real(8)") or s.startswith("doubleprecision") or s.startswith("real(kind=8)"):
        return R8
    if s.startswith("real"):
        return R4
    if s.startswith("integer(8)"):
        return "i8"
    if s.startswith("integer"):
        return I4
    if s.startswith("logical"):
        return LOG
    if s.startswith("character"):
        return CHR
    raise SyntaxError(spec)


_TYPE_RE = re.compile(r"^(real\s*\(\s*8\s*\)|real|double\s+precision|integer\s*\(\s*8\s*\)|integer|logical|"
                      r"character\s*(?:\(\s*len\s*=\s*\d+\s*\)|\*\d+)?)\s*(.*)$", re.I)


def parse_decl(stmt):
    m = _TYPE_RE.match(stmt)
    if not m or "::" not in stmt:
        return None
    ftype = _parse_type(m.group(1))
    rest = m.group(2)
    attrs_s, names_s = rest.split("::", 1)
    attrs = [a.strip().lower() for a in split_top(attrs_s) if a.strip()]
    dims, intent, parameter = None, None, False
    for a in attrs:
        if a.startswith("dimension"):
            dims = split_top(a[a.index("(") + 1:a.rindex(")")])
        elif a.startswith("intent"):
            intent = a[a.index("(") + 1:a.rindex(")")].strip()
        elif a == "parameter":
            parameter = True
    out = []
    for item in split_top(names_s):
        init = None
        if "=" in item and "==" not in item:
            name_part, init = item.split("=", 1)
            init = init.strip()
        else:
            name_part = item
        name_part = name_part.strip()
        d = dims
        if "(" in name_part:
            d = split_top(name_part[name_part.index("(") + 1:name_part.rindex(")")])
            name_part = name_part[:name_part.index("(")].strip()
        out.append(Decl(name_part.lower(), ftype, d, init, intent, parameter))
    return out


def parse_program(text):
    lines = logical_lines(text)
    units, main, cur, in_contains = {}, None, None, False
    for label, st in lines:
        low = st.lower()
        if re.match(r"^program\s+\w+", low):
            main = cur = Unit(low.split()[1], [])
            continue
        if low.startswith("end program") or low == "end":
            break
        if low == "contains":
            in_contains = True
            continue
        m = re.match(r"^subroutine\s+(\w+)\s*(\((.*)\))?\s*$", low)
        if m:
            args = [a.strip() for a in (m.group(3) or "").split(",") if a.strip()]
            cur = Unit(m.group(1), args)
            units[cur.name] = cur
            continue
        if low.startswith("end subroutine"):
            cur = main
            continue
        if low.startswith("implicit none"):
            continue
        d = parse_decl(st)
        if d is not None:
            for x in d:
                cur.decls[x.name] = x
            continue
        if low.startswith("namelist"):
            for m2 in re.finditer(r"/(\w+)/([^/]*)", st):
                cur.namelists[m2.group(1).lower()] = [n.strip().lower() for n in m2.group(2).split(",") if n.strip()]
            continue
        if re.match(r"^format\s*\(", low):
            cur.formats[label] = st[st.index("(") + 1:st.rindex(")")]
            continue
        cur.body.append((label, st))
    return main, units


# ---------------------------------------------------------------------------------------
# execution
class Frame:
    __slots__ = ("vars", "unit")

    def __init__(self, unit):
        self.vars = {}
        self.unit = unit


class Ref:
    """A scalar dummy argument bound to its actual argument."""

    __slots__ = ("get", "set")

    def __init__(self, get, set_):
        self.get = get
        self.set = set_


class Interpreter:
    def __init__(self, source, files=None, inputs=None):
        self.main, self.units = parse_program(source)
        self.G = {}
        self.files = {} if files is None else files      # name -> list of records
        self.text_inputs = inputs or {}                  # name -> text (namelist files)
        self.unformatted_inputs = {}                     # name -> list of records
        self.units_open = {}                             # unit number -> file name
        self.compiled = {}
        self.stdout = []
        self.history = {}                                # name -> every record written
        self.text_records = {}                           # name -> records of a formatted input file

    # -- declarations ------------------------------------------------------------------
    def _new_scalar(self, ftype):
        return {I4: 0, "i8": 0, R4: np.float32(0), R8: 0.0, LOG: False, CHR: ""}[ftype]

    def _dtype(self, ftype):
        return {I4: np.int32, "i8": np.int64, R4: np.float32, R8: np.float64, LOG: np.bool_, CHR: object}[ftype]

    def _bounds(self, dims, frame):
        lbs, shape = [], []
        for d in dims:
            if ":" in d:
                lo, hi = d.split(":")
                lo = self.eval_str(lo, frame) if lo.strip() else 1
                hi = self.eval_str(hi, frame)
            else:
                lo, hi = 1, self.eval_str(d, frame)
            lbs.append(int(lo))
            shape.append(int(hi) - int(lo) + 1)
        return lbs, shape

    def eval_str(self, s, frame):
        return self.compile_expr(parse_expr(s), frame.unit)(frame)

    def init_unit_vars(self, unit, frame):
        for d in unit.decls.values():
            if d.name in unit.args:
                continue
            if d.dims is not None and all(x.strip() == ":" for x in d.dims):
                frame.vars[d.name] = None                # allocatable, set by ALLOCATE
                continue
            if d.dims is not None:
                lbs, shape = self._bounds(d.dims, frame)
                frame.vars[d.name] = FArray(np.zeros(shape, dtype=self._dtype(d.ftype), order="F"), lbs)
                continue
            v = self._new_scalar(d.ftype)
            if d.init is not None:
                v = to_kind(self.eval_str(d.init, frame), d.ftype if d.ftype != "i8" else I4) \
                    if d.ftype != CHR else self.eval_str(d.init, frame)
            frame.vars[d.name] = v

    # -- name resolution ----------------------------------------------------------------
    def _scope(self, name, unit):
        if unit is not self.main and (name in unit.decls or name in unit.args):
            return "local"
        if name in self.main.decls:
            return "global"
        return None

    def _getter(self, name, unit):
        sc = self._scope(name, unit)
        G = self.G
        if sc == "global":
            return lambda fr: G[name]
        if sc == "local":
            d = unit.decls.get(name)
            is_ref = name in unit.args and d is not None and d.dims is None and d.intent != "in"
            if is_ref:
                return lambda fr: fr.vars[name].get()
            return lambda fr: fr.vars[name]
        raise NameError(f"{name} not declared in {unit.name}")

    def _setter(self, name, unit):
        sc = self._scope(name, unit)
        G = self.G
        d = unit.decls.get(name) if sc == "local" else self.main.decls.get(name)
        ftype = d.ftype if d is not None else None
        k = I4 if ftype == "i8" else ftype

        def conv(v):
            if isinstance(v, np.ndarray):
                return v
            return to_kind(v, k) if k in (I4, R4, R8, LOG) else v
        if sc == "global":
            def s(fr, v):
                cur = G[name]
                if isinstance(cur, FArray):
                    cur.data[...] = v
                else:
                    G[name] = conv(v)
            return s
        if sc == "local":
            is_ref = name in unit.args and d is not None and d.dims is None and d.intent != "in"
            if is_ref:
                return lambda fr, v: fr.vars[name].set(conv(v))

            def s(fr, v):
                cur = fr.vars[name]
                if isinstance(cur, FArray):
                    cur.data[...] = v
                else:
                    fr.vars[name] = conv(v)
            return s
        raise NameError(f"{name} not declared in {unit.name}")

    # -- expressions ---------------------------------------------------------------------
    def compile_expr(self, e, unit):
        t = e[0]
        if t == "const":
            v = e[1]
            return lambda fr: v
        if t == "paren":
            return self.compile_expr(e[1], unit)
        if t == "name":
            g = self._getter(e[1], unit)
            d = unit.decls.get(e[1]) if self._scope(e[1], unit) == "local" else self.main.decls.get(e[1])
            if d is not None and d.dims is not None:       # whole array in an expression
                return lambda fr: g(fr).data
            return g
        if t == "neg":
            f = self.compile_expr(e[1], unit)
            return lambda fr: -f(fr)
        if t == "not":
            f = self.compile_expr(e[1], unit)
            return lambda fr: not f(fr)
        if t == "bin":
            op = e[1]
            a, b = self.compile_expr(e[2], unit), self.compile_expr(e[3], unit)
            if op == ".and.":
                return lambda fr: bool(a(fr)) and bool(b(fr))
            if op == ".or.":
                return lambda fr: bool(a(fr)) or bool(b(fr))
            if op == ".eqv.":
                return lambda fr: bool(a(fr)) == bool(b(fr))
            if op == ".neqv.":
                return lambda fr: bool(a(fr)) != bool(b(fr))

            def f(fr, op=op):
                x, y = a(fr), b(fr)
                if type(x) is float and type(y) is float:        # hot path: both real(8)
                    if op == "+":
                        return x + y
                    if op == "-":
                        return x - y
                    if op == "*":
                        return x * y
                    if op == "/":
                        return x / y
                return arith(op, x, y)
            return f
        if t == "rel":
            op = e[1]
            a, b = self.compile_expr(e[2], unit), self.compile_expr(e[3], unit)
            ops = {"==": lambda x, y: x == y, "/=": lambda x, y: x != y, "<": lambda x, y: x < y,
                   "<=": lambda x, y: x <= y, ">": lambda x, y: x > y, ">=": lambda x, y: x >= y}[op]

            def f(fr):
                x, y = a(fr), b(fr)
                if isinstance(x, str) or isinstance(y, str):
                    return ops(str(x).rstrip(), str(y).rstrip())
                x, y, _ = promote(x, y)
                return ops(x, y)
            return f
        if t == "cat":
            a, b = self.compile_expr(e[1], unit), self.compile_expr(e[2], unit)
            return lambda fr: str(a(fr)) + str(b(fr))
        if t == "ctor":
            items = [self.compile_expr(x, unit) for x in e[1]]

            def f(fr):
                vals = [it(fr) for it in items]
                k = max((kind_of(v) for v in vals), key=lambda q: _RANK.get(q, -1))
                return np.array([to_kind(v, k) for v in vals],
                                dtype={I4: np.int32, R4: np.float32, R8: np.float64}.get(k, object))
            return f
        if t == "call":
            name, args = e[1], e[2]
            if self._scope(name, unit) is not None:
                return self._compile_ref(name, args, unit)
            return self._compile_intrinsic(name, args, unit)
        raise SyntaxError(e)

    def _compile_ref(self, name, args, unit):
        get = self._getter(name, unit)
        subs = []
        scalar = True
        for a in args:
            if a[0] == "range":
                lo = self.compile_expr(a[1], unit) if a[1] is not None else None
                hi = self.compile_expr(a[2], unit) if a[2] is not None else None
                subs.append(("r", lo, hi))
                scalar = False
            else:
                subs.append(("s", self.compile_expr(a, unit)))
        if scalar:
            fs = [s[1] for s in subs]
            if len(fs) == 1:
                f0 = fs[0]
                return lambda fr: (lambda A: A.data[f0(fr) - A.lb[0]])(get(fr))
            if len(fs) == 2:
                f0, f1 = fs

                def g2(fr):
                    A = get(fr)
                    return A.data[f0(fr) - A.lb[0], f1(fr) - A.lb[1]]
                return g2
            if len(fs) == 3:
                f0, f1, f2 = fs

                def g3(fr):
                    A = get(fr)
                    return A.data[f0(fr) - A.lb[0], f1(fr) - A.lb[1], f2(fr) - A.lb[2]]
                return g3

        def gs(fr):
            A = get(fr)
            idx = []
            for s in subs:
                if s[0] == "s":
                    idx.append(s[1](fr))
                else:
                    idx.append((s[1](fr) if s[1] else None, s[2](fr) if s[2] else None))
            return A.data[A.index(idx)]
        return gs

    def _compile_intrinsic(self, name, args, unit):
        cargs = [self.compile_expr(a, unit) if a[0] != "kw" else None for a in args]
        if name == "sum":
            f = cargs[0]

            def s(fr):
                a = np.asarray(f(fr))
                k = kind_of(a)
                flat = a.ravel(order="F")
                if k == I4:
                    return int(flat.sum())
                acc = to_kind(0.0, k)
                for v in flat:
                    acc = acc + (float(v) if k == R8 else v)
                return acc
            return s
        if name == "maxval":
            f = cargs[0]
            return lambda fr: (lambda a: float(a.max()) if a.dtype == np.float64 else a.max())(np.asarray(f(fr)))
        if name == "sqrt":
            f = cargs[0]
            return lambda fr: (lambda x: math.sqrt(x) if type(x) is float else np.sqrt(x))(f(fr))
        if name == "abs":
            f = cargs[0]
            return lambda fr: abs(f(fr))
        if name == "exp":
            f = cargs[0]
            return lambda fr: (lambda x: math.exp(x) if type(x) is float else np.exp(x))(f(fr))
        if name in ("cos", "sin"):
            f = cargs[0]
            fn = math.cos if name == "cos" else math.sin
            return lambda fr: (lambda x: fn(x) if type(x) is float else np.float32(fn(float(x))))(f(fr))
        if name == "atan":
            if len(cargs) == 1:
                f = cargs[0]
                return lambda fr: (lambda x: math.atan(x) if type(x) is float else np.float32(math.atan(float(x))))(f(fr))
            fy, fx = cargs

            def at2(fr):
                y, x, k = promote(fy(fr), fx(fr))
                return math.atan2(y, x) if k == R8 else np.float32(math.atan2(float(y), float(x)))
            return at2
        if name == "floor":
            f = cargs[0]
            return lambda fr: int(math.floor(f(fr)))
        if name == "real":
            f = cargs[0]
            return lambda fr: to_kind(f(fr), R4)
        if name == "sngl":
            f = cargs[0]
            return lambda fr: to_kind(f(fr), R4)
        if name == "dble":
            f = cargs[0]
            return lambda fr: to_kind(f(fr), R8)
        if name == "mod":
            fa, fb = cargs

            def md(fr):
                a, b = fa(fr), fb(fr)
                return a - _idiv(a, b) * b
            return md
        if name == "trim":
            f = cargs[0]
            return lambda fr: str(f(fr)).rstrip()
        if name == "char":
            f = cargs[0]
            return lambda fr: chr(f(fr))
        raise NameError(f"intrinsic {name} not supported")

    # -- statements ----------------------------------------------------------------------
    def compile_block(self, stmts, unit):
        """stmts: list of (label, text).  Returns a list of closures."""
        out, i = [], 0
        while i < len(stmts):
            fn, i = self.compile_stmt(stmts, i, unit)
            if fn is not None:
                out.append(fn)
        return out

    def _find_end(self, stmts, i, openers, closers, mids=()):
        depth, j = 0, i
        marks = []
        while j < len(stmts):
            low = stmts[j][1].lower()
            if j > i and any(o(low) for o in openers):
                depth += 1
            elif any(c(low) for c in closers):
                if depth == 0:
                    return j, marks
                depth -= 1
            elif depth == 0 and j > i and any(mm(low) for mm in mids):
                marks.append(j)
            j += 1
        raise SyntaxError(f"unterminated block at {stmts[i]}")

    def compile_stmt(self, stmts, i, unit):
        label, st = stmts[i]
        low = st.lower().strip()
        # IF blocks
        if re.match(r"^if\s*\(", low) and low.endswith("then"):
            return self._compile_if(stmts, i, unit)
        if re.match(r"^if\s*\(", low):
            close = match_paren(st, st.index("("))
            cond = self.compile_expr(parse_expr(st[st.index("(") + 1:close]), unit)
            body, _ = self.compile_stmt([(None, st[close + 1:].strip())], 0, unit)

            def f(fr):
                if cond(fr):
                    body(fr)
            return f, i + 1
        if re.match(r"^do\b", low):
            return self._compile_do(stmts, i, unit)
        if re.match(r"^select\s+case", low):
            return self._compile_select(stmts, i, unit)
        if low == "exit":
            def f(fr):
                raise _Exit()
            return f, i + 1
        if low == "cycle":
            def f(fr):
                raise _Cycle()
            return f, i + 1
        if low == "stop" or low.startswith("stop "):
            def f(fr):
                raise FortranStop()
            return f, i + 1
        if low == "return":
            raise SyntaxError("RETURN not supported")
        if low.startswith("call "):
            return self._compile_call(st[5:].strip(), unit), i + 1
        if low.startswith("allocate"):
            return self._compile_allocate(st, unit), i + 1
        if re.match(r"^(open|close|inquire)\s*\(", low):
            return self._compile_open_close(st, unit), i + 1
        if re.match(r"^(write|read)\s*\(", low):
            return self._compile_io(st, unit), i + 1
        if re.match(r"^print\b", low):
            return (lambda fr: None), i + 1
        # assignment
        eq = self._assignment_eq(st)
        if eq is None:
            raise SyntaxError(f"unsupported statement: {st!r}")
        return self._compile_assign(st[:eq].strip(), st[eq + 1:].strip(), unit), i + 1

    def _assignment_eq(self, st):
        depth, q = 0, None
        for k, ch in enumerate(st):
            if q:
                if ch == q:
                    q = None
                continue
            if ch in "'\"":
                q = ch
            elif ch == "(":
                depth += 1
            elif ch == ")":
                depth -= 1
            elif ch == "=" and depth == 0:
                nxt = st[k + 1] if k + 1 < len(st) else ""
                prv = st[k - 1] if k > 0 else ""
                if nxt != "=" and prv not in "=/<>":
                    return k
        return None

    def _compile_assign(self, lhs, rhs, unit):
        rv = self.compile_expr(parse_expr(rhs), unit)
        le = parse_expr(lhs)
        if le[0] == "name":
            setv = self._setter(le[1], unit)
            return lambda fr: setv(fr, rv(fr))
        if le[0] == "call":
            name, args = le[1], le[2]
            get = self._getter(name, unit)
            subs = []
            for a in args:
                if a[0] == "range":
                    subs.append(("r", self.compile_expr(a[1], unit) if a[1] else None,
                                 self.compile_expr(a[2], unit) if a[2] else None))
                else:
                    subs.append(("s", self.compile_expr(a, unit)))
            if all(s[0] == "s" for s in subs):
                fs = [s[1] for s in subs]

                def asg(fr):
                    A = get(fr)
                    v = rv(fr)
                    idx = tuple(f(fr) - lb for f, lb in zip(fs, A.lb))
                    A.data[idx] = v
                return asg

            def asg_sec(fr):
                A = get(fr)
                idx = []
                for s in subs:
                    if s[0] == "s":
                        idx.append(s[1](fr))
                    else:
                        idx.append((s[1](fr) if s[1] else None, s[2](fr) if s[2] else None))
                A.data[A.index(idx)] = rv(fr)
            return asg_sec
        raise SyntaxError(lhs)

    def _compile_if(self, stmts, i, unit):
        is_if = lambda s: re.match(r"^if\s*\(", s) is not None and s.endswith("then")
        is_end = lambda s: s in ("end if", "endif")
        is_mid = lambda s: re.match(r"^else\s*if\s*\(", s) is not None or s == "else"
        end, marks = self._find_end(stmts, i, [is_if], [is_end], [is_mid])
        heads = [i] + marks
        branches = []
        for bi, h in enumerate(heads):
            st = stmts[h][1]
            low = st.lower()
            nxt = heads[bi + 1] if bi + 1 < len(heads) else end
            body = self.compile_block(stmts[h + 1:nxt], unit)
            if low.strip() == "else":
                cond = None
            else:
                p0 = st.index("(")
                cond = self.compile_expr(parse_expr(st[p0 + 1:match_paren(st, p0)]), unit)
            branches.append((cond, body))

        def f(fr):
            for cond, body in branches:
                if cond is None or cond(fr):
                    for b in body:
                        b(fr)
                    return
        return f, end + 1

    def _compile_do(self, stmts, i, unit):
        is_do = lambda s: re.match(r"^do\b", s) is not None
        is_end = lambda s: s in ("end do", "enddo")
        end, _ = self._find_end(stmts, i, [is_do], [is_end])
        body = self.compile_block(stmts[i + 1:end], unit)
        st = stmts[i][1]
        m = re.match(r"^do\s+(\w+)\s*=\s*(.*)$", st, re.I)
        if not m:
            def f(fr):
                try:
                    while True:
                        try:
                            for b in body:
                                b(fr)
                        except _Cycle:
                            pass
                except _Exit:
                    pass
            return f, end + 1
        var = m.group(1).lower()
        parts = split_top(m.group(2))
        lo, hi = self.compile_expr(parse_expr(parts[0]), unit), self.compile_expr(parse_expr(parts[1]), unit)
        step = self.compile_expr(parse_expr(parts[2]), unit) if len(parts) > 2 else (lambda fr: 1)
        setv = self._setter(var, unit)

        def f(fr):
            a, b, c = int(lo(fr)), int(hi(fr)), int(step(fr))
            v = a
            try:
                for v in range(a, b + (1 if c > 0 else -1), c):
                    setv(fr, v)
                    try:
                        for bb in body:
                            bb(fr)
                    except _Cycle:
                        pass
                else:
                    setv(fr, (v + c) if b >= a else a)
            except _Exit:
                pass
        return f, end + 1

    def _compile_select(self, stmts, i, unit):
        is_sel = lambda s: re.match(r"^select\s+case", s) is not None
        is_end = lambda s: s in ("end select", "endselect")
        is_case = lambda s: re.match(r"^case\b", s) is not None
        end, marks = self._find_end(stmts, i, [is_sel], [is_end], [is_case])
        st = stmts[i][1]
        p0 = st.index("(")
        sel = self.compile_expr(parse_expr(st[p0 + 1:match_paren(st, p0)]), unit)
        cases = []
        for ci, h in enumerate(marks):
            nxt = marks[ci + 1] if ci + 1 < len(marks) else end
            body = self.compile_block(stmts[h + 1:nxt], unit)
            cst = stmts[h][1].strip()
            if cst.lower() == "case default":
                cases.append((None, body))
            else:
                q0 = cst.index("(")
                vals = [self.compile_expr(parse_expr(v), unit)(None) for v in split_top(cst[q0 + 1:match_paren(cst, q0)])]
                cases.append((vals, body))

        def f(fr):
            v = sel(fr)
            vs = v.rstrip() if isinstance(v, str) else v
            for vals, body in cases:
                if vals is None or any((x.rstrip() if isinstance(x, str) else x) == vs for x in vals):
                    for b in body:
                        b(fr)
                    return
        return f, end + 1

    def _compile_allocate(self, st, unit):
        inner = st[st.index("(") + 1:st.rindex(")")]
        items = []
        for it in split_top(inner):
            name = it[:it.index("(")].strip().lower()
            dims = split_top(it[it.index("(") + 1:it.rindex(")")])
            items.append((name, dims))
        sc_decl = lambda n: unit.decls.get(n) or self.main.decls.get(n)

        def f(fr):
            for name, dims in items:
                lbs, shape = self._bounds(dims, fr)
                d = sc_decl(name)
                arr = FArray(np.zeros(shape, dtype=self._dtype(d.ftype), order="F"), lbs)
                if self._scope(name, unit) == "global":
                    self.G[name] = arr
                else:
                    fr.vars[name] = arr
        return f

    # -- calls ---------------------------------------------------------------------------
    def _compile_call(self, text, unit):
        m = re.match(r"^(\w+)\s*(\((.*)\))?$", text.strip(), re.S)
        name = m.group(1).lower()
        arg_s = m.group(3) or ""
        args = [parse_expr_sub(a) for a in split_top(arg_s)] if arg_s.strip() else []
        if name == "cpu_time":
            setv = self._actual_setter(args[0], unit)
            return lambda fr: setv(fr, 0.0)
        if name in ("omp_set_num_threads", "system", "get_environment_variable"):
            return lambda fr: None
        callee = self.units[name]
        binders = []
        for dname, a in zip(callee.args, args):
            d = callee.decls[dname]
            binders.append((dname, d, self._compile_actual(a, d, unit)))

        def f(fr):
            nf = Frame(callee)
            for dname, d, bind in binders:
                nf.vars[dname] = bind(fr, nf)
            self.run_unit(callee, nf)
        return f

    def _actual_setter(self, a, unit):
        if a[0] == "name":
            return self._setter(a[1], unit)
        if a[0] == "call":
            get = self._getter(a[1], unit)
            fs = [self.compile_expr(x, unit) for x in a[2]]

            def s(fr, v):
                A = get(fr)
                A.data[tuple(f(fr) - lb for f, lb in zip(fs, A.lb))] = v
            return s
        raise SyntaxError(a)

    def _compile_actual(self, a, d, unit):
        """Returns bind(frame, new_frame) -> value for the dummy's slot."""
        if d.dims is not None:                       # array dummy: a view with the declared bounds
            get = self.compile_expr(a, unit) if a[0] != "name" else self._getter(a[1], unit)

            def bind(fr, nf):
                actual = get(fr)
                data = actual.data if isinstance(actual, FArray) else actual
                lbs, shape = self._bounds(d.dims, nf)
                view = data.reshape(shape, order="F") if tuple(shape) != data.shape else data
                return FArray(view, lbs)
            return bind
        if d.intent == "in":
            ev = self.compile_expr(a, unit)
            k = I4 if d.ftype == "i8" else d.ftype
            return lambda fr, nf: (lambda v: to_kind(v, k) if k in (I4, R4, R8) else v)(ev(fr))
        # out / inout scalar: by reference
        getter = self.compile_expr(a, unit)
        setter = self._actual_setter(a, unit)
        return lambda fr, nf: Ref(lambda: getter(fr), lambda v: setter(fr, v))

    def run_unit(self, unit, frame):
        if unit.name not in self.compiled:
            self.compiled[unit.name] = None
            self.compiled[unit.name] = self.compile_block(unit.body, unit)
        # locals (SAVE semantics for initialised locals are not needed by the reference)
        for d in unit.decls.values():
            if d.name in unit.args:
                continue
            if d.dims is not None and not all(x.strip() == ":" for x in d.dims):
                lbs, shape = self._bounds(d.dims, frame)
                frame.vars[d.name] = FArray(np.zeros(shape, dtype=self._dtype(d.ftype), order="F"), lbs)
            elif d.dims is not None:
                frame.vars[d.name] = None
            else:
                v = self._new_scalar(d.ftype)
                if d.init is not None:
                    v = self.eval_str(d.init, frame)
                    if d.ftype in (I4, R4, R8):
                        v = to_kind(v, d.ftype)
                frame.vars[d.name] = v
        for s in self.compiled[unit.name]:
            s(frame)

    # -- I/O -----------------------------------------------------------------------------
    def _kw(self, spec_items):
        pos, kw = [], {}
        for it in spec_items:
            m = re.match(r"^(\w+)\s*=\s*(.*)$", it, re.S)
            if m and m.group(1).lower() in ("unit", "file", "status", "form", "position", "action", "access",
                                             "iostat", "err", "fmt", "exist", "nml"):
                kw[m.group(1).lower()] = m.group(2).strip()
            else:
                pos.append(it)
        return pos, kw

    def _compile_open_close(self, st, unit):
        low = st.lower()
        inner = st[st.index("(") + 1:match_paren(st, st.index("("))]
        pos, kw = self._kw(split_top(inner))
        ustr = kw.get("unit", pos[0] if pos else None)
        uexp = self.compile_expr(parse_expr(ustr), unit)
        if low.startswith("close"):
            def f(fr):
                self.units_open.pop(uexp(fr), None)
            return f
        if low.startswith("inquire"):
            return lambda fr: None
        fexp = self.compile_expr(parse_expr(kw["file"]), unit)
        status = kw.get("status", "'unknown'").strip("'\"").lower()
        position = kw.get("position", "'asis'").strip("'\"").lower()
        access = kw.get("access", "'sequential'").strip("'\"").lower()
        form = kw.get("form", "'formatted'").strip("'\"").lower()

        def f(fr):
            name = str(fexp(fr)).rstrip()
            self.units_open[uexp(fr)] = (name, form, [0])
            append = position == "append" or access == "append"
            if name in self.text_inputs or name in self.text_records or name in self.unformatted_inputs and \
                    status == "old":
                return
            if not append or status == "replace":
                self.files[name] = []
            else:
                self.files.setdefault(name, [])
        return f

    def _compile_io(self, st, unit):
        is_write = st.lower().startswith("write")
        p0 = st.index("(")
        p1 = match_paren(st, p0)
        spec = split_top(st[p0 + 1:p1])
        rest = st[p1 + 1:].strip()
        items = [x for x in split_top(rest)] if rest else []
        ustr = spec[0]
        fmt = spec[1] if len(spec) > 1 and "=" not in spec[1] else None
        if is_write:
            vals = [self._compile_io_item(x, unit) for x in items]
            if ustr.strip() == "*":
                return lambda fr: None
            # internal write to a character variable with a numbered FORMAT
            if fmt is not None and self._scope(ustr.strip().lower(), unit) and (
                    fmt.strip().isdigit() or fmt.strip()[:1] in "'\""):
                if fmt.strip().isdigit():
                    fspec = (unit.formats.get(int(fmt)) or self.main.formats.get(int(fmt)))
                else:
                    fspec = fmt.strip()[1:-1].strip()[1:-1]
                setv = self._setter(ustr.strip().lower(), unit)

                def f(fr):
                    out = []
                    for v in vals:
                        out.extend(v(fr))
                    setv(fr, _format(fspec, out))
                return f
            uexp = self.compile_expr(parse_expr(ustr), unit)

            def f(fr):
                u = uexp(fr)
                rec = []
                for v in vals:
                    rec.extend(v(fr))
                if u in self.units_open:
                    self.files[self.units_open[u][0]].append(rec)
                    self.history.setdefault(self.units_open[u][0], []).append(rec)
            return f
        # READ: namelist from input text, or an unformatted record supplied by the caller
        uexp = self.compile_expr(parse_expr(ustr), unit)
        if fmt is not None and fmt.strip().lower() in {**self.main.namelists, **unit.namelists}:
            group = fmt.strip().lower()
            names = (unit.namelists.get(group) or self.main.namelists[group])
            setters = {n: self._setter(n, unit) for n in names}

            def f(fr):
                name = self.units_open[uexp(fr)][0]
                for k, v in _namelist_group(self.text_inputs[name], group).items():
                    setters[k](fr, v)
            return f
        targets = [self._compile_read_target(x, unit) for x in items]
        kw = dict(self._kw(spec)[1])
        iostat = self._setter(kw["iostat"].strip().lower(), unit) if "iostat" in kw else None
        as_line = fmt is not None and fmt.strip().replace(" ", "").lower() in ("'(a)'", '"(a)"')

        def f(fr):
            name, form, cursor = self.units_open[uexp(fr)]
            recs = self.unformatted_inputs.get(name)
            if recs is None:
                recs = self.text_records.get(name, [])
            if cursor[0] >= len(recs):                 # end of file
                if iostat is None:
                    raise FortranStop(f"end of file on {name}")
                iostat(fr, -1)
                return
            rec = list(recs[cursor[0]])
            cursor[0] += 1
            if as_line:
                rec = [" ".join(str(x) for x in rec)]
            for t in targets:
                t(fr, rec)
            if iostat is not None:
                iostat(fr, 0)
        return f

    def _compile_read_target(self, x, unit):
        x = x.strip()
        if x.startswith("(") and match_paren(x, 0) == len(x) - 1:      # implied-do target list
            parts = split_top(x[1:-1])
            var, lo = parts[-2].split("=", 1)
            lo_e = self.compile_expr(parse_expr(lo), unit)
            hi_e = self.compile_expr(parse_expr(parts[-1]), unit)
            subs = [self._compile_read_target(q, unit) for q in parts[:-2]]
            setv = self._setter(var.strip().lower(), unit)

            def t_do(fr, rec):
                for v in range(int(lo_e(fr)), int(hi_e(fr)) + 1):
                    setv(fr, v)
                    for sb in subs:
                        sb(fr, rec)
            return t_do
        e = parse_expr(x)
        if e[0] == "name":
            get = self._getter(e[1], unit)
            setv = self._setter(e[1], unit)

            def t(fr, rec):
                cur = get(fr)
                if isinstance(cur, FArray):
                    cur.data[...] = np.asarray(rec.pop(0)).reshape(cur.data.shape, order="F")
                else:
                    setv(fr, rec.pop(0))
            return t
        if e[0] == "call":
            setter = self._actual_setter(e, unit)

            def t2(fr, rec):
                setter(fr, rec.pop(0))
            return t2
        raise SyntaxError(x)

    def _compile_io_item(self, x, unit):
        x = x.strip()
        if x.startswith("(") and match_paren(x, 0) == len(x) - 1:
            inner = x[1:-1]
            parts = split_top(inner)
            if len(parts) >= 3 and re.match(r"^\w+\s*=", parts[-2]):
                var, lo = parts[-2].split("=", 1)
                var = var.strip().lower()
                lo_e = self.compile_expr(parse_expr(lo), unit)
                hi_e = self.compile_expr(parse_expr(parts[-1]), unit)
                subs = [self._compile_io_item(p, unit) for p in parts[:-2]]
                setv = self._setter(var, unit)

                def f(fr):
                    out = []
                    for v in range(int(lo_e(fr)), int(hi_e(fr)) + 1):
                        setv(fr, v)
                        for s in subs:
                            out.extend(s(fr))
                    return out
                return f
        ev = self.compile_expr(parse_expr(x), unit)

        def g(fr):
            v = ev(fr)
            if isinstance(v, FArray):
                return [v.data.copy(order="F")]
            if isinstance(v, np.ndarray):
                return [v.copy()]
            return [v]
        return g

    # -- driver --------------------------------------------------------------------------
    def run(self):
        fr = Frame(self.main)
        for d in self.main.decls.values():
            if d.dims is not None and all(x.strip() == ":" for x in d.dims):
                self.G[d.name] = None
            elif d.dims is not None:
                lbs, shape = self._bounds(d.dims, fr)
                self.G[d.name] = FArray(np.zeros(shape, dtype=self._dtype(d.ftype), order="F"), lbs)
            else:
                self.G[d.name] = self._new_scalar(d.ftype)
        for d in self.main.decls.values():       # initialisers (parameters first)
            if d.init is not None and d.dims is None:
                v = self.eval_str(d.init, fr)
                self.G[d.name] = to_kind(v, I4 if d.ftype == "i8" else d.ftype) if d.ftype != CHR else v
        body = self.compile_block(self.main.body, self.main)
        try:
            for s in body:
                s(fr)
        except FortranStop:
            pass
        return self


def parse_expr_sub(s):
    p = Parser(tokenize(s))
    e = p.subscript()
    return e


def _format(spec, values):
    """Edit descriptors A[w] and I[w] (the only ones the reference formats internally)."""
    out, vi = "", 0
    for d in split_top(spec):
        d = d.strip()
        m = re.match(r"^([aAiI])(\d*)$", d)
        if m and m.group(2) == "0":
            m = re.match(r"^([aAiI])()$", d[0])
        if not m:
            continue
        v = values[vi]
        vi += 1
        w = int(m.group(2)) if m.group(2) else None
        if m.group(1).lower() == "a":
            s = str(v)
            out += s if w is None else (s[:w] if len(s) >= w else s.rjust(w))
        else:
            s = str(int(v))
            out += s if w is None else ("*" * w if len(s) > w else s.rjust(w))
    return out


def _namelist_group(text, group):
    m = re.search(r"&" + group + r"\b(.*?)/", text, re.I | re.S)
    if not m:
        raise FortranStop(f"namelist group {group} missing")
    body = re.sub(r"!.*", "", m.group(1))
    out = {}
    for name, val in re.findall(r"(\w+)\s*=\s*([^=\n,]+?)(?=\s*,|\s*\n|\s*$|\s+\w+\s*=)", body, re.S):
        v = val.strip()
        lv = v.lower()
        if lv in (".true.", "t", ".t."):
            out[name.lower()] = True
        elif lv in (".false.", "f", ".f."):
            out[name.lower()] = False
        elif re.match(r"^[+-]?\d+$", v):
            out[name.lower()] = int(v)
        else:
            out[name.lower()] = float(lv.replace("d", "e"))
    return out
