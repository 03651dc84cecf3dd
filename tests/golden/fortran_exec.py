"""Execute routines of the reference's Fortran source in Python, statement
for statement, to make golden fixtures.

Test infrastructure only: it runs where the reference is mounted, at
fixture-generation time (`make_driver_golden.py`), never at test time.

The reference is Fortran 90 and no Fortran compiler exists where this
library is built, so the routines whose results the library must
reproduce are translated into Python functions and executed in IEEE
double precision with Fortran's semantics where they differ from
Python's:

* arrays are 1-based, column-major, with sections `a(lo:hi, j)` and `:`;
  sections are numpy views, so a section passed to a subroutine is written
  in place;
* integer / integer truncates toward zero; assignment to an integer
  variable truncates; integer `**` with a constant exponent is the
  multiplication chain gfortran emits;
* a DO loop's variable ends at max(start, end + 1) after normal completion
  and keeps its value after EXIT; the bounds are evaluated once;
* `sum`, `dot_product` and `maxval` run left to right;
* default-kind REAL literals (no `_double`, no `d` exponent) are rounded to
  single precision;
* `exp`, `sqrt`, `erf`, `log`, `cos`, `sin`, `acos` and `**` with a real
  exponent are the C library's (CPython's `math` calls libm, as gfortran's
  runtime does).

Only the subset the translated routines use is handled: assignments, DO /
DO WHILE, IF blocks and one-line IFs, EXIT, CYCLE, CALL, ALLOCATE,
RETURN, STOP, functions, derived-type components (`%`).  WRITE, FLUSH,
OPEN, CLOSE, REWIND and DEALLOCATE are dropped.  HDF5 and LAPACK calls are
supplied by the caller as Python hooks.
"""

import math
import re

import numpy as np


# ---------------------------------------------------------------- runtime

class Arr:
    """A 1-based Fortran array over a column-major numpy array."""

    def __init__(self, shape, dtype=float):
        if isinstance(shape, int):
            shape = (shape,)
        self.a = np.zeros(tuple(int(s) for s in shape), dtype=dtype, order="F")

    @classmethod
    def wrap(cls, x):
        """A dummy array: the actual argument's storage, 1-based."""
        if isinstance(x, Arr) or x is None:
            return x
        out = cls.__new__(cls)
        out.a = x if isinstance(x, np.ndarray) else np.asarray(x)
        return out

    @classmethod
    def of(cls, values, dtype=float):
        v = np.asarray(values, dtype=dtype)
        out = cls(v.shape, dtype)
        out.a[...] = v
        return out

    def _k(self, k):
        if not isinstance(k, tuple):
            k = (k,)
        if len(k) != self.a.ndim:
            raise IndexError(f"rank {self.a.ndim} array indexed with {len(k)} subscripts")
        out = []
        for d, i in enumerate(k):
            if isinstance(i, slice):
                lo = 1 if i.start is None else int(i.start)
                hi = self.a.shape[d] if i.stop is None else int(i.stop)
                if lo < 1 or hi > self.a.shape[d]:
                    if hi >= lo:
                        raise IndexError(f"section {lo}:{hi} out of 1:{self.a.shape[d]}")
                out.append(slice(lo - 1, max(hi, lo - 1)))
            else:
                i = int(i)
                if not 1 <= i <= self.a.shape[d]:
                    raise IndexError(f"subscript {i} out of 1:{self.a.shape[d]}")
                out.append(i - 1)
        return tuple(out)

    def __getitem__(self, k):
        v = self.a[self._k(k)]
        if isinstance(v, np.ndarray):
            return v
        return v.item() if hasattr(v, "item") else v

    def __setitem__(self, k, v):
        self.a[self._k(k)] = v.a if isinstance(v, Arr) else v

    def whole(self):
        return self.a

    # a whole array named in an expression acts as its values
    def __array__(self, dtype=None, copy=None):
        return self.a if dtype is None else self.a.astype(dtype)

    def __add__(self, o): return self.a + _val(o)
    def __radd__(self, o): return _val(o) + self.a
    def __sub__(self, o): return self.a - _val(o)
    def __rsub__(self, o): return _val(o) - self.a
    def __mul__(self, o): return self.a * _val(o)
    def __rmul__(self, o): return _val(o) * self.a
    def __truediv__(self, o): return self.a / _val(o)
    def __rtruediv__(self, o): return _val(o) / self.a
    def __neg__(self): return -self.a


class Obj:
    """A derived-type value: components as attributes."""

    def __init__(self, **kw):
        self.__dict__.update(kw)


def _is_int(x):
    return isinstance(x, (int, np.integer)) and not isinstance(x, bool)


def _val(x):
    return x.a if isinstance(x, Arr) else x


def f_div(a, b):
    a, b = _val(a), _val(b)
    if _is_int(a) and _is_int(b):
        q = abs(int(a)) // abs(int(b))
        return q if (a >= 0) == (b >= 0) else -q
    return a / b


POWI_TABLE = [0, 1, 1, 2, 2, 3, 3, 4, 4, 6, 5, 6, 6, 10, 7, 9, 8]


def f_powi(x, n):
    """x**n for a constant integer n as gfortran evaluates it: GCC's power
    tree (x^n = x^k x^(n-k), k = POWI_TABLE[n]), or plain repeated
    squaring above the table."""
    x = _val(x)
    if _is_int(x):
        return int(x) ** n
    if n == 0:
        return 1.0 if not isinstance(x, np.ndarray) else np.ones_like(x)
    if n < 0:
        return 1.0 / f_powi(x, -n)
    if n >= len(POWI_TABLE):
        r, b, e = None, x, n
        while e:
            if e & 1:
                r = b if r is None else r * b
            b = b * b
            e >>= 1
        return r
    cache = {1: x}

    def pw(m):
        if m not in cache:
            k = POWI_TABLE[m]
            cache[m] = pw(k) * pw(m - k)
        return cache[m]
    return pw(n)


def f_pow(x, y):
    x, y = _val(x), _val(y)
    if _is_int(y):
        return f_powi(x, int(y))
    if isinstance(x, np.ndarray) or isinstance(y, np.ndarray):
        return np.vectorize(math.pow)(x, y)
    return math.pow(x, y)


def _elementwise(fn):
    def g(x):
        x = _val(x)
        if isinstance(x, np.ndarray):
            return np.vectorize(fn, otypes=[float])(x) if x.size else x.astype(float)
        return fn(float(x))
    return g


f_exp = _elementwise(math.exp)
f_sqrt = _elementwise(math.sqrt)
f_log = _elementwise(math.log)
f_cos = _elementwise(math.cos)
f_sin = _elementwise(math.sin)
f_acos = _elementwise(math.acos)
f_erf = _elementwise(math.erf)


def f_abs(x):
    x = _val(x)
    if isinstance(x, np.ndarray):
        return np.abs(x)
    return abs(x)


def f_sum(x, dim=None):
    x = _val(x)
    if dim is not None:
        raise NotImplementedError("sum(..., dim)")
    x = np.asarray(x).ravel(order="F")
    if x.dtype.kind in "iu":
        return int(x.sum())
    if x.dtype.kind == "c":
        c = 0.0 + 0.0j
        for v in x:
            c = c + complex(v)
        return c
    s = 0.0
    for v in x:
        s = s + float(v)
    return s


def f_dot_product(a, b):
    a, b = np.asarray(_val(a)).ravel(), np.asarray(_val(b)).ravel()
    s = 0.0
    for x, y in zip(a, b):
        s = s + float(x) * float(y)
    return s


def f_maxval(x):
    x = np.asarray(_val(x)).ravel(order="F")
    m = -math.inf
    for v in x:
        if v > m:
            m = float(v)
    return m


def f_minval(x):
    x = np.asarray(_val(x)).ravel(order="F")
    m = math.inf
    for v in x:
        if v < m:
            m = float(v)
    return m


def f_max(*a):
    a = [_val(x) for x in a]
    if any(isinstance(x, np.ndarray) for x in a):
        return np.maximum.reduce(np.broadcast_arrays(*a))
    if all(_is_int(x) for x in a):
        return max(int(x) for x in a)
    return float(max(a))


def f_min(*a):
    a = [_val(x) for x in a]
    if any(isinstance(x, np.ndarray) for x in a):
        return np.minimum.reduce(np.broadcast_arrays(*a))
    if all(_is_int(x) for x in a):
        return min(int(x) for x in a)
    return float(min(a))


def f_real(x, kind=None):
    x = _val(x)
    if isinstance(x, complex):
        x = x.real
    if isinstance(x, np.ndarray) and x.dtype.kind == "c":
        x = x.real
    if isinstance(x, np.ndarray):
        return x.astype(float) if kind is not None else x.astype(np.float32).astype(float)
    return float(x) if kind is not None else float(np.float32(x))


f_dble = lambda x: f_real(x, 8)


def f_int(x, kind=None):
    x = _val(x)
    if isinstance(x, np.ndarray):
        return np.trunc(x).astype(np.int64)
    return int(math.trunc(x))


def f_nint(x):
    x = _val(x)
    return int(math.floor(abs(x) + 0.5)) * (1 if x >= 0 else -1)


def f_ceiling(x):
    return int(math.ceil(_val(x)))


def f_floor(x):
    return int(math.floor(_val(x)))


def f_mod(a, b):
    a, b = _val(a), _val(b)
    if _is_int(a) and _is_int(b):
        r = abs(int(a)) % abs(int(b))
        return r if a >= 0 else -r
    return math.fmod(a, b)


def f_sign(a, b):
    a, b = _val(a), _val(b)
    if _is_int(a) and _is_int(b):
        return abs(a) if b >= 0 else -abs(a)
    return math.copysign(abs(a), b)


def f_size(x, dim=None):
    x = _val(x)
    return int(x.size if dim is None else x.shape[int(dim) - 1])


def f_allocated(x):
    return isinstance(x, Arr)


def f_cmplx(re_, im_=0.0, kind=None):
    re_, im_ = _val(re_), _val(im_)
    if isinstance(re_, np.ndarray) or isinstance(im_, np.ndarray):
        return np.asarray(re_) + 1j * np.asarray(im_)
    return complex(re_, im_)


def f_aimag(x):
    x = _val(x)
    return x.imag if isinstance(x, np.ndarray) else complex(x).imag


def f_conjg(x):
    x = _val(x)
    return np.conj(x) if isinstance(x, np.ndarray) else complex(x).conjugate()


def f_transpose(x):
    return np.asarray(_val(x)).T


def f_ishft(a, n):
    a, n = int(_val(a)), int(_val(n))
    return a << n if n >= 0 else a >> -n


def f_bit_size(x):
    return 64


def f_btest(a, pos):
    return bool((int(_val(a)) >> int(_val(pos))) & 1)


def _signed64(v):
    v &= (1 << 64) - 1
    return v - (1 << 64) if v >= (1 << 63) else v


def f_ibclr(a, pos):
    return _signed64((int(_val(a)) & ((1 << 64) - 1)) & ~(1 << int(_val(pos))))


def f_ibset(a, pos):
    return _signed64((int(_val(a)) & ((1 << 64) - 1)) | (1 << int(_val(pos))))


def f_matmul(a, b):
    return np.asarray(_val(a)) @ np.asarray(_val(b))


def f_log10(x):
    return math.log10(_val(x))


INTRINSICS = {"exp", "sqrt", "log", "cos", "sin", "acos", "erf", "abs", "sum",
              "dot_product", "maxval", "minval", "max", "min", "real", "dble",
              "int", "nint", "ceiling", "floor", "mod", "sign", "size", "allocated",
              "cmplx", "log10", "aimag", "conjg", "transpose", "ishft", "matmul",
              "bit_size", "btest", "ibclr", "ibset"}


class FortranStop(RuntimeError):
    pass


def f_stop(msg=""):
    raise FortranStop(msg)


def runtime_namespace():
    ns = {"Arr": Arr, "Obj": Obj, "f_div": f_div, "f_powi": f_powi, "f_pow": f_pow,
          "f_stop": f_stop, "FortranStop": FortranStop, "np": np, "math": math,
          "f32": lambda s: float(np.float32(float(s))), "double": 8}
    for n in INTRINSICS:
        ns["f_" + n] = globals()["f_" + n]
    return ns


# ------------------------------------------------------------ expressions

TOKEN = re.compile(r"""
    (?P<ws>\s+)
  | (?P<str>'[^']*'|"[^"]*")
  | (?P<dotop>\.(?:and|or|not|eq|ne|lt|le|gt|ge|true|false|eqv|neqv)\.)
  | (?P<real>(?:\d+\.(?![a-zA-Z]{2,}\.)\d*|\.\d+)(?:[eEdD][-+]?\d+)?(?:_\w+)?
             |\d+[eEdD][-+]?\d+(?:_\w+)?)
  | (?P<int>\d+(?:_\w+)?)
  | (?P<name>[A-Za-z]\w*)
  | (?P<op>\*\*|//|==|/=|<=|>=|<|>|\+|-|\*|/|\(|\)|,|:|%|=)
""", re.X | re.I)


def tokenize(s):
    out, pos = [], 0
    while pos < len(s):
        m = TOKEN.match(s, pos)
        if not m:
            raise ValueError(f"cannot tokenize {s[pos:]!r} in {s!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        out.append((kind, m.group(kind)))
    return out


def real_literal(text):
    t = text.lower()
    kind = None
    if "_" in t:
        t, kind = t.split("_", 1)
    if "d" in t:
        return repr(float(t.replace("d", "e")))
    if kind is not None:
        return repr(float(t))
    return f"f32({t!r})"  # default REAL kind: single precision


class ExprParser:
    """Recursive-descent parser of a Fortran expression into Python."""

    def __init__(self, tokens, ctx):
        self.t = tokens
        self.i = 0
        self.ctx = ctx

    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else (None, None)

    def take(self, val=None):
        tok = self.peek()
        if val is not None and (tok[1] is None or tok[1].lower() != val):
            raise ValueError(f"expected {val} at {tok} in {self.t}")
        self.i += 1
        return tok

    def at(self, *vals):
        tok = self.peek()
        return tok[1] is not None and tok[1].lower() in vals

    def parse(self):
        e = self.eqv()
        if self.i != len(self.t):
            raise ValueError(f"trailing tokens {self.t[self.i:]}")
        return e

    def eqv(self):
        e = self.or_()
        while self.at(".eqv.", ".neqv."):
            op = "==" if self.take()[1].lower() == ".eqv." else "!="
            e = f"(bool({e}) {op} bool({self.or_()}))"
        return e

    def or_(self):
        e = self.and_()
        while self.at(".or."):
            self.take()
            e = f"({e} or {self.and_()})"
        return e

    def and_(self):
        e = self.not_()
        while self.at(".and."):
            self.take()
            e = f"({e} and {self.not_()})"
        return e

    def not_(self):
        if self.at(".not."):
            self.take()
            return f"(not {self.not_()})"
        return self.rel()

    REL = {"==": "==", "/=": "!=", "<": "<", "<=": "<=", ">": ">", ">=": ">=",
           ".eq.": "==", ".ne.": "!=", ".lt.": "<", ".le.": "<=", ".gt.": ">",
           ".ge.": ">="}

    def rel(self):
        e = self.add()
        if self.at(*self.REL):
            op = self.REL[self.take()[1].lower()]
            e = f"({e} {op} {self.add()})"
        return e

    def add(self):
        if self.at("-", "+"):
            op = self.take()[1]
            e = f"({op}{self.mul()})"
        else:
            e = self.mul()
        while self.at("+", "-"):
            op = self.take()[1]
            e = f"({e} {op} {self.mul()})"
        return e

    def mul(self):
        e = self.pow_()
        while self.at("*", "/") and not (self.at("/") and self.peek(1)[1] == ")"):
            op = self.take()[1]
            r = self.pow_()
            e = f"({e} * {r})" if op == "*" else f"f_div({e}, {r})"
        return e

    def pow_(self):
        base = self.primary()
        if self.at("**"):
            self.take()
            if self.at("-", "+"):  # a**-n
                op = self.take()[1]
                exp = f"({op}{self.pow_()})"
            else:
                exp = self.pow_()
            if re.fullmatch(r"\d+", exp) or re.fullmatch(r"\(\d+\)", exp):
                return f"f_powi({base}, {exp.strip('()')})"
            return f"f_pow({base}, {exp})"
        return base

    def primary(self):
        kind, val = self.peek()
        if kind == "real":
            self.take()
            return real_literal(val)
        if kind == "int":
            self.take()
            return val.split("_")[0]
        if kind == "str":
            self.take()
            return repr(val[1:-1])
        if kind == "dotop":
            low = val.lower()
            if low in (".true.", ".false."):
                self.take()
                return "True" if low == ".true." else "False"
        if val == "(" and self.peek(1)[1] == "/":
            # array constructor (/ a, b, ... /)
            self.take()
            self.take()
            items = [self.eqv()]
            while self.at(","):
                self.take()
                items.append(self.eqv())
            self.take("/")
            self.take(")")
            return f"np.array([{', '.join(items)}])"
        if val == "(":
            self.take()
            e = self.eqv()
            if self.at(","):  # complex literal (re, im)
                self.take()
                im = self.eqv()
                self.take(")")
                return f"complex({e}, {im})"
            self.take(")")
            return f"({e})"
        if kind == "name":
            return self.designator()
        raise ValueError(f"unexpected {val!r} in {self.t}")

    def designator(self):
        name = self.take()[1]
        low = name.lower()
        out = self.ctx.name(low)
        first = True
        while True:
            if self.at("("):
                self.take()
                if first and low in INTRINSICS:
                    args = self.arglist(subscripts=False)
                    out = f"f_{low}({args})"
                elif first and low in self.ctx.functions:
                    args = self.arglist(subscripts=False)
                    out = f"{self.ctx.name(low)}({args})"
                else:
                    out = f"{out}[{self.arglist(subscripts=True)}]"
                self.take(")")
            elif self.at("%"):
                self.take()
                comp = self.take()[1].lower()
                out = f"{out}.{comp}"
            else:
                return out
            first = False

    def arglist(self, subscripts):
        args = []
        if self.at(")"):
            return ""
        while True:
            args.append(self.subscript() if subscripts else self.argument())
            if self.at(","):
                self.take()
                continue
            return ", ".join(args)

    def argument(self):
        # keyword arguments (kind=...) are dropped
        if self.peek()[0] == "name" and self.peek(1)[1] == "=":
            self.take()
            self.take()
            self.eqv()
            return "8"
        return self.eqv()

    def subscript(self):
        lo = hi = None
        if not self.at(":"):
            lo = self.eqv()
            if not self.at(":"):
                return lo
        self.take(":")
        if not self.at(",", ")"):
            hi = self.eqv()
        return f"{'' if lo is None else lo}:{'' if hi is None else hi}"


LVALUE = re.compile(r"[A-Za-z]\w*(\([^():]*\))?(%[A-Za-z]\w*(\([^():]*\))?)*")


class Ctx:
    """Names known to the translator: functions (called, not indexed),
    renames, and the scalar-dummy positions of translated subroutines."""

    def __init__(self, functions=(), rename=None, types=None):
        self.functions = set(functions)
        self.rename = rename or {}
        self.sigs = {}
        # types of module arrays allocated by the translated routines
        self.types = types or {}

    def name(self, low):
        return self.rename.get(low, low)


def expr(src, ctx):
    return ExprParser(tokenize(src), ctx).parse()


# ------------------------------------------------------------- statements

def preprocess(lines, defined=()):
    """#ifdef / #ifndef / #else / #endif with the given macros defined (the
    reference builds its complex engine without GAMMA)."""
    out, stack = [], []
    for raw in lines:
        t = raw.strip()
        m = re.match(r"#\s*(ifdef|ifndef)\s+(\w+)", t)
        if m:
            on = (m.group(2) in defined) == (m.group(1) == "ifdef")
            stack.append(on)
            continue
        if re.match(r"#\s*else", t):
            stack[-1] = not stack[-1]
            continue
        if re.match(r"#\s*endif", t):
            stack.pop()
            continue
        if all(stack):
            out.append(raw)
    return out


def join_lines(lines):
    """Free-form continuation and comments: one logical statement per item."""
    out, cur = [], ""
    for raw in preprocess(lines):
        code = _strip_comment(raw.rstrip("\n"))
        if cur:
            s = code.lstrip()
            if s.startswith("&"):
                s = s[1:]
            code = s
        if code.rstrip().endswith("&"):
            cur += code.rstrip()[:-1] + " "
            continue
        cur += code
        if cur.strip():
            for part in _split_semicolons(cur.strip()):
                out.append(part)
        cur = ""
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
            cur += ch
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            cur += ch
        elif ch == ";":
            if cur.strip():
                parts.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        parts.append(cur.strip())
    return parts


def extract(lines, kind, name):
    """The statements of `subroutine name` / `function name` from a file's
    lines."""
    start = None
    pat = re.compile(rf"^\s*(?:[\w\s(),=]*\s)?{kind}\s+{name}\b", re.I)
    endp = re.compile(rf"^\s*end\s+{kind}\s+{name}\b", re.I)
    for i, l in enumerate(lines):
        if start is None and pat.match(_strip_comment(l)):
            start = i
        elif start is not None and endp.match(l):
            return join_lines(lines[start:i + 1])
    raise KeyError(f"{kind} {name} not found")


DECL = re.compile(r"^(real|integer|logical|character|complex|type\s*\(\w+\))(.*?)::(.*)$", re.I)
SKIP = re.compile(r"^(use\b|implicit\b|write\b|flush\b|call\s+flush\b|open\b|close\b|"
                  r"rewind\b|deallocate\b|print\b|format\b|contains\b|"
                  r"call\s+timestamp|intrinsic\b|external\b|save\b)", re.I)


def _split_top(s, sep=","):
    parts, depth, cur = [], 0, ""
    for ch in s:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == sep and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        parts.append(cur)
    return [p.strip() for p in parts]


def translate(stmts, ctx, hooks=None, record=False):
    """Python source of one subroutine or function.  hooks: {name: [argument
    positions]} of calls handed to Python callables, which return the final
    values of those (scalar) arguments as a tuple, as translated
    subroutines do for their scalar dummies."""
    hooks = hooks or {}
    head = stmts[0]
    m = re.match(r"^(?:[\w\s(),=]*?\s)?(subroutine|function)\s+(\w+)\s*(?:\(([^)]*)\))?"
                 r"(?:\s*result\s*\((\w+)\))?", head, re.I)
    kind, name = m.group(1).lower(), m.group(2).lower()
    params = [p.strip().lower() for p in (m.group(3) or "").split(",") if p.strip()]
    result = (m.group(4) or name).lower()
    decls = {}
    inits = {}
    body = []
    for s in stmts[1:-1]:
        d = DECL.match(s)
        if d:
            typ = d.group(1).lower()
            attrs = d.group(2).lower()
            if typ == "real" and ("double" not in attrs and "8" not in attrs):
                typ = "real4"
            dim = re.search(r"dimension\s*\(([^)]*)\)", attrs)
            for v in _split_top(d.group(3)):
                init = None
                if "=" in v:
                    v, init = v.split("=", 1)
                v = v.strip()
                vm = re.match(r"(\w+)\s*(?:\((.*)\))?", v)
                vn = vm.group(1).lower()
                vdims = vm.group(2) or (dim.group(1) if dim else None)
                decls[vn] = (typ, vdims)
                if init is not None:
                    inits[vn] = init.strip()
            continue
        body.append(s)
    py = [f"def {ctx.name(name)}({', '.join(params)}):"]
    scalar_dummies = [p for p in params if decls.get(p, ("real", None))[1] is None]
    if kind == "subroutine":
        ctx.sigs[name] = [params.index(p) for p in scalar_dummies]
    ret = "".join(f"{p}, " for p in scalar_dummies)
    local = set(decls) | set(params)
    global_at = len(py)
    for p in params:
        if p in decls and decls[p][1] is not None:
            py.append(f"    {p} = Arr.wrap({p})")
    # local scalars start at zero (the translated routines set them first),
    # fixed-size local arrays are created
    for v, (typ, dims) in decls.items():
        if v in params:
            continue
        if dims is None:
            py.append(f"    {v} = {0 if typ in ('integer', 'logical') else 0.0}")
        elif ":" not in dims:
            shape = ", ".join(f"int({expr(x, ctx)})" for x in _split_top(dims))
            dt = {"integer": "np.int64", "complex": "complex"}.get(typ, "float")
            py.append(f"    {v} = Arr(({shape},), {dt})")
        else:
            py.append(f"    {v} = None")
    for v, init in inits.items():
        typ, dims = decls[v]
        if dims is None:
            py.append(f"    {v} = {expr(init, ctx)}")
        else:
            dt = {"integer": "np.int64", "complex": "complex"}.get(typ, "float")
            py.append(f"    {v} = Arr.of({expr(init, ctx)}, {dt})")
    if kind == "function" and result not in decls:
        py.append(f"    {result} = 0.0")
    ind = 1
    stack = []
    scalar_type = {v: t for v, (t, d) in decls.items() if d is None}

    def emit(line):
        py.append("    " * ind + line)

    def assign(lhs, rhs):
        lhs_py = expr(lhs, ctx)
        base = re.match(r"\w+", lhs).group(0).lower()
        r = expr(rhs, ctx)
        if "(" not in lhs:
            t = scalar_type.get(base) if "%" not in lhs else None
            if t == "integer":
                r = f"f_int({r})"
            elif t == "real":
                r = f"float({r})"
            elif t == "real4":
                r = f"f_real({r})"
            if t is None:
                # a whole array (a local one, or a module or component
                # array) is assigned element by element
                if base in decls and decls[base][1] is not None:
                    emit(f"{lhs_py}.a[...] = {r}")
                else:
                    emit(f"if isinstance({lhs_py}, Arr): {lhs_py}.a[...] = {r}")
                    emit(f"else: {lhs_py} = {r}")
                return
        emit(f"{lhs_py} = {r}")

    def simple(s):
        low = s.lower()
        if SKIP.match(s):
            emit("pass")
            return
        if low == "exit":
            emit("break")
            return
        if low == "cycle":
            emit("continue")
            return
        if low == "return":
            if record:
                emit(f"_record({name!r}, dict(locals()))")
            emit(f"return {result}" if kind == "function" else f"return ({ret})")
            return
        if low.startswith("stop"):
            emit(f"f_stop({s[4:].strip()!r})")
            return
        m = re.match(r"^allocate\s*\((.*)\)$", s, re.I)
        if m:
            for item in _split_top(m.group(1)):
                im = re.match(r"(\w+)\s*\((.*)\)$", item)
                v = im.group(1).lower()
                shape = ", ".join(f"int({expr(x, ctx)})" for x in _split_top(im.group(2)))
                typ = decls.get(v, (ctx.types.get(v, "real"), None))[0]
                dt = {"integer": "np.int64", "complex": "complex"}.get(typ, "float")
                emit(f"{ctx.name(v)} = Arr(({shape},), {dt})")
            return
        m = re.match(r"^call\s+(\w+)\s*(?:\((.*)\))?$", s, re.I)
        if m:
            callee = m.group(1).lower()
            args = _split_top(m.group(2) or "")
            py_args = ", ".join(expr(a, ctx) for a in args)
            outs = hooks.get(callee, ctx.sigs.get(callee))
            if outs is None:
                emit(f"{ctx.name(callee)}({py_args})")
                return
            # Fortran passes scalars by reference: the callee returns the
            # final values of its scalar dummies, written back here to the
            # actual arguments that are variables
            emit(f"_r = {ctx.name(callee)}({py_args})")
            for k, j in enumerate(outs):
                if j < len(args) and LVALUE.fullmatch(args[j].strip()):
                    emit(f"{expr(args[j], ctx)} = _r[{k}]")
            return
        m = re.match(r"^([\w%(),:\s+\-*/]+?)\s*=(?!=)\s*(.*)$", s)
        if m:
            assign(m.group(1), m.group(2))
            return
        raise ValueError(f"{name}: cannot translate: {s}")

    for s in body:
        s = re.sub(r"^\d+\s+", "", s)  # statement labels
        low = s.lower()
        m = re.match(r"^(\w+\s*:\s*)?do\s+(\w+)\s*=\s*(.*)$", s, re.I)
        if m:
            var = m.group(2).lower()
            parts = _split_top(m.group(3))
            lo, hi = expr(parts[0], ctx), expr(parts[1], ctx)
            step = expr(parts[2], ctx) if len(parts) > 2 else "1"
            emit(f"_lo_{var}, _hi_{var}, _st_{var} = int({lo}), int({hi}), int({step})")
            emit(f"for {var} in range(_lo_{var}, _hi_{var} + (1 if _st_{var} > 0 else -1), _st_{var}):")
            stack.append(("do", var))
            ind += 1
            continue
        m = re.match(r"^do\s+while\s*\((.*)\)$", s, re.I)
        if m:
            emit(f"while {expr(m.group(1), ctx)}:")
            stack.append(("while", None))
            ind += 1
            continue
        if re.fullmatch(r"end\s*do(\s+\w+)?", low):
            k, var = stack.pop()
            ind -= 1
            if k == "do":
                emit("else:")
                emit(f"    {var} = _lo_{var} + max(0, (_hi_{var} - _lo_{var} + _st_{var}) // _st_{var}) * _st_{var}")
            continue
        m = re.match(r"^if\s*\((.*)\)\s*then$", s, re.I)
        if m:
            emit(f"if {expr(m.group(1), ctx)}:")
            stack.append(("if", None))
            ind += 1
            continue
        m = re.match(r"^select\s+case\s*\((.*)\)$", s, re.I)
        if m:
            sel = f"_sel{len(stack)}"
            emit(f"{sel} = {expr(m.group(1), ctx)}")
            emit("if False:")
            emit("    pass")
            stack.append(("select", sel))
            ind += 1
            continue
        m = re.match(r"^case\s*(default|\((.*)\))$", s, re.I)
        if m:
            sel = stack[-1][1]
            if m.group(1).lower() == "default":
                py.append("    " * (ind - 1) + "else:")
            else:
                conds = []
                for item in _split_top(m.group(2)):
                    if ":" in item:
                        lo, hi = item.split(":")
                        conds.append(f"({expr(lo, ctx)} <= {sel} <= {expr(hi, ctx)})")
                    else:
                        conds.append(f"({sel} == {expr(item, ctx)})")
                py.append("    " * (ind - 1) + f"elif {' or '.join(conds)}:")
            continue
        if re.fullmatch(r"end\s*select", low):
            stack.pop()
            ind -= 1
            continue
        m = re.match(r"^else\s*if\s*\((.*)\)\s*then$", s, re.I)
        if m:
            py.append("    " * (ind - 1) + f"elif {expr(m.group(1), ctx)}:")
            continue
        if low == "else":
            py.append("    " * (ind - 1) + "else:")
            continue
        if re.fullmatch(r"end\s*if", low):
            stack.pop()
            ind -= 1
            continue
        m = re.match(r"^if\s*\(", s, re.I)
        if m:
            # one-line IF: find the closing parenthesis of the condition
            depth, j = 0, s.index("(")
            for j in range(s.index("("), len(s)):
                if s[j] == "(":
                    depth += 1
                elif s[j] == ")":
                    depth -= 1
                    if depth == 0:
                        break
            emit(f"if {expr(s[s.index('(') + 1:j], ctx)}:")
            ind += 1
            simple(s[j + 1:].strip())
            ind -= 1
            continue
        simple(s)
    if record:
        py.append(f"    _record({name!r}, dict(locals()))")
    if kind == "function":
        py.append(f"    return {result}")
    else:
        py.append(f"    return ({ret})")
    # names assigned here that are not local are module variables
    assigned = set()
    for line in py[1:]:
        a = re.match(r"^\s*(?:else:\s*)?([A-Za-z]\w*(?:\s*,\s*[A-Za-z_]\w*)*)\s*=(?!=)", line)
        if a:
            for nm in re.findall(r"[A-Za-z_]\w*", a.group(1)):
                assigned.add(nm)
        f = re.match(r"^\s*for\s+(\w+)\s+in", line)
        if f:
            assigned.add(f.group(1))
    glob = sorted(v for v in assigned
                  if v not in local and v not in (ctx.name(p) for p in params)
                  and not v.startswith("_") and v != result)
    if glob:
        py.insert(global_at, "    global " + ", ".join(glob))
    return "\n".join(py) + "\n"


def load(path, kind, name, ns, ctx=None, hooks=None, record=False):
    """Translate `kind name` from the Fortran file at `path` and define it
    in namespace `ns` (module variables and hooks live there too).  With
    `record`, the routine's local variables at its return are stored in
    ns["_recorded"][name]."""
    with open(path) as fh:
        lines = fh.readlines()
    ctx = ctx or Ctx()
    ns.setdefault("_recorded", {})
    ns.setdefault("_record", lambda n, d: ns["_recorded"].__setitem__(n, d))
    src = translate(extract(lines, kind, name), ctx, hooks or {}, record)
    try:
        exec(compile(src, f"<{name}>", "exec"), ns)
    except SyntaxError as e:
        raise SyntaxError(f"{e}\n{src}") from None
    return src
