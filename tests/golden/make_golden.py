"""Generate golden primitive-integral vectors by executing the reference's
own generated kernels.

The reference's primitive integrals live in `src/imago/gaussIntegrals.f90`
(overlap2CIntg 26-4420, kinetic2CIntg 4422-11622, massvel2CIntg
39070-49402, electron3CIntg 11624-16023, boys 16080-16221, nuclear3CIntg
16223-23039, momentum2CIntg 23041-39068, dipole3CIntg 49404-65510,
KOverlap2CIntg 129408-135102).  No Fortran compiler exists where this script runs, so the
script transliterates those subroutines statement by statement into Python and executes them with IEEE
double arithmetic, which is what gfortran -O3 (no -ffast-math, no FMA on
x86-64 baseline) evaluates.  Fortran semantics that matter for the values
are kept:

* default-kind REAL literals (no `d` exponent, e.g. `1.5`, `10E-2` and the
  Boys series constants) are rounded to single precision first;
* `sum()` adds left to right;
* `**` with a constant integer exponent is the multiplication chain
  gfortran emits for it; `**` with a real exponent and `exp`/`erf`/`sqrt`
  are the C library's (CPython's `math` module calls libm).

Run in a container that has the reference mounted (it is read here and
nowhere else):

    python tests/golden/make_golden.py <root of the reference checkout>

It writes `tests/golden/primitives.json`, which the tests read.  The
fixture is committed; nothing at test time touches the reference.
"""

import json
import math
import os
import re
import sys

import numpy as np

KERNEL_LINES = {
    "overlap2CIntg": (26, 4420),
    "kinetic2CIntg": (4422, 11622),
    "electron3CIntg": (11624, 16023),
    "boys": (16080, 16221),
    "nuclear3CIntg": (16223, 23039),
    "massvel2CIntg": (39070, 49402),
    "momentum2CIntg": (23041, 39068),
    "dipole3CIntg": (49404, 65510),
}
# Kernels whose local arrays are assigned whole rows or are complex.
NUMPY_KERNELS = {"KOverlap2CIntg": (129408, 135102)}

# Class codes built by integrals.F90:533-536: bit 0..3 for atom 1 (s,p,d,f),
# bit 4..7 for atom 2.
L_OF_NSH = {1: 0, 4: 1, 9: 2, 16: 3}


def f32(x):
    return float(np.float32(x))


class FArr:
    """1-based Fortran array backed by a dict; unset reads raise."""

    def __init__(self, name, dims):
        self.name = name
        self.dims = dims
        self.d = {}

    def _key(self, k):
        if not isinstance(k, tuple):
            k = (k,)
        k = tuple(int(i) for i in k)
        if len(k) != len(self.dims):
            raise IndexError(f"{self.name}{k}")
        for i, n in zip(k, self.dims):
            if not 1 <= i <= n:
                raise IndexError(f"{self.name}{k} out of {self.dims}")
        return k

    def __getitem__(self, k):
        return self.d[self._key(k)]

    def __setitem__(self, k, v):
        self.d[self._key(k)] = float(v)


class NArr:
    """1-based Fortran array backed by numpy, for kernels that assign whole
    rows (`Hn(1,:) = ...`) or hold complex values; `:` is the token ALL."""

    def __init__(self, name, dims, cplx=False):
        self.name = name
        self.a = np.zeros(dims, dtype=complex if cplx else float)

    def _k(self, k):
        if not isinstance(k, tuple):
            k = (k,)
        return tuple(i if isinstance(i, slice) else int(i) - 1 for i in k)

    def __getitem__(self, k):
        v = self.a[self._k(k)]
        return v if isinstance(v, np.ndarray) else v.item()

    def __setitem__(self, k, v):
        self.a[self._k(k)] = v


ALL = slice(None)


def _exp(x):
    return math.exp(x) if isinstance(x, float) else np.exp(x)


def _fsum(x):
    s = 0.0
    for v in x:
        s = s + float(v)
    return s


def _ix(arr, *k):
    if isinstance(arr, (FArr, NArr)):
        return arr[k if len(k) > 1 else k[0]]
    # numpy vector from a whole-array assignment
    assert len(k) == 1
    if isinstance(k[0], slice):
        return arr
    return arr[int(k[0]) - 1].item()


REAL_LIT = re.compile(
    r"(?<![\w.])(\d+\.\d*|\.\d+|\d+)([eEdD][-+]?\d+)?(?![\w.])")


def _lit(m):
    mant, exp = m.group(1), m.group(2)
    if exp is None and "." not in mant:
        return mant  # integer literal
    if exp is not None and exp[0] in "dD":
        return f"float('{mant}e{exp[1:]}')"
    # default REAL kind: single precision
    e = "" if exp is None else "e" + exp[1:]
    return f"f32('{mant}{e}')"


def _powi(x, n):
    """x**n for a constant integer n as gfortran evaluates it
    (gfc_conv_cst_int_power): an addition chain from GCC's power tree,
    x^n = x^k * x^(n-k) with k = POWI_TABLE[n], intermediate powers
    computed once."""
    cache = {1: x}

    def pw(m):
        if m not in cache:
            k = POWI_TABLE[m]
            cache[m] = pw(k) * pw(m - k)
        return cache[m]
    if n == 0:
        return 1.0
    return pw(n)


POWI_TABLE = [0, 1, 1, 2, 2, 3, 3, 4, 4, 6, 5, 6, 6, 10, 7, 9, 8]

INT_POW = re.compile(r"(\b[A-Za-z_]\w*)\s*\*\*\s*(?:\(\s*(\d+)\s*\)|(\d+))(?![\w.])")
SLICE_POW = re.compile(r"(\b[A-Za-z_]\w*)\(:\)\s*\*\*\s*(\d+)(?![\w.])")
PAREN_POW = re.compile(r"\)\s*\*\*\s*(\d+)(?![\w.])")


def _apowi(x, n):
    """Whole-array NAME(:)**n: the same chain per element."""
    if isinstance(x, NArr):
        x = x.a
    return np.array([_powi(v.item() if hasattr(v, "item") else v, n) for v in x])


def _paren_pow(expr):
    """(expr)**n with a constant integer n -> _powi((expr), n)."""
    while True:
        m = PAREN_POW.search(expr)
        if not m:
            return expr
        depth, i = 0, m.start()
        while True:
            if expr[i] == ")":
                depth += 1
            elif expr[i] == "(":
                depth -= 1
                if depth == 0:
                    break
            i -= 1
        # a function call's parentheses belong to the call: keep its name
        j = i
        while j > 0 and (expr[j - 1].isalnum() or expr[j - 1] == "_"):
            j -= 1
        expr = (expr[:j] + "_powi(" + expr[j:m.start() + 1] + ", "
                + m.group(1) + ")" + expr[m.end():])


ALL_INDEX = re.compile(r"(?<=[(,])\s*:\s*(?=[,)])")


def translate_expr(expr, arrays):
    expr = SLICE_POW.sub(lambda m: f"_apowi({m.group(1)}, {m.group(2)})", expr)
    expr = ALL_INDEX.sub("ALL", expr)
    expr = _paren_pow(expr)
    expr = INT_POW.sub(lambda m: f"_powi({m.group(1)}, {m.group(2) or m.group(3)})", expr)
    expr = expr.replace(".eq.", "==").replace(".ne.", "!=")
    expr = expr.replace(".lt.", "<").replace(".le.", "<=")
    expr = expr.replace(".gt.", ">").replace(".ge.", ">=")
    expr = expr.replace(".and.", " and ").replace(".or.", " or ")
    # integer-by-integer division would truncate in Fortran; refuse it.
    if re.search(r"(?<![\w.])\d+\s*/\s*\d+(?![\w.dDeE])", expr):
        raise ValueError("integer division in: " + expr)
    expr = REAL_LIT.sub(_lit, expr)

    def arr_ref(m):
        name, args = m.group(1), m.group(2)
        if name in arrays:
            return f"_ix({name}, {args})"
        return m.group(0)

    prev = None
    while prev != expr:
        prev = expr
        expr = re.sub(r"\b([A-Za-z_]\w*)\(([^()]*)\)", arr_ref, expr)
    return expr


def read_subroutine(lines, start, end):
    body = lines[start - 1:end]
    # Join free-form continuations: trailing '&' then optional leading '&'.
    joined, cur = [], ""
    for raw in body:
        line = raw.rstrip("\n")
        code = line.split("!", 1)[0] if "!" in line else line
        if cur:
            s = code.lstrip()
            if s.startswith("&"):
                s = s[1:]
            code = s
        if code.rstrip().endswith("&"):
            cur += code.rstrip()[:-1]
            continue
        cur += code
        if cur.strip():
            joined.append(cur.strip())
        cur = ""
    return joined


def transpile(name, stmts, numpy_arrays=False):
    """Return python source of a function `name(**kw)` for one subroutine.
    numpy_arrays: local arrays as NArr (whole-row assignments, complex)."""
    arrays = set()
    cplx = set()
    decl_lines = []
    params = None
    py = []
    indent = 1
    for s in stmts:
        low = s.lower()
        if low.startswith("subroutine"):
            params = re.search(r"\((.*)\)", s).group(1).replace(" ", "")
            continue
        if low.startswith("end subroutine") or low.startswith("use ") \
                or low.startswith("implicit"):
            continue
        if low.startswith("real") or low.startswith("integer") or low.startswith("complex"):
            m = re.search(r"dimension\s*\(([^)]*)\)\s*(?:,\s*intent\s*\([^)]*\))?\s*::\s*(.*)$", s)
            if m:
                dims = [int(x) for x in m.group(1).split(",")]
                for v in m.group(2).split(","):
                    v = v.strip()
                    arrays.add(v)
                    decl_lines.append((v, dims))
                    if low.startswith("complex"):
                        cplx.add(v)
            continue
        pad = "    " * indent
        m = re.match(r"(else\s*if|if)\s*\((.*)\)\s*then$", s, re.I)
        if m:
            kw = "elif" if m.group(1).lower().startswith("else") else "if"
            if kw == "elif":
                py.append("    " * (indent - 1) + f"elif {translate_expr(m.group(2), arrays)}:")
            else:
                py.append(pad + f"if {translate_expr(m.group(2), arrays)}:")
                indent += 1
            continue
        if re.fullmatch(r"else", s, re.I):
            py.append("    " * (indent - 1) + "else:")
            continue
        if re.fullmatch(r"end\s*if", s, re.I):
            indent -= 1
            continue
        m = re.match(r"do\s+(\w+)\s*=\s*(.*),(.*)$", s, re.I)
        if m:
            py.append(pad + f"for {m.group(1)} in range(int({translate_expr(m.group(2), arrays)}), int({translate_expr(m.group(3), arrays)}) + 1):")
            indent += 1
            continue
        if re.fullmatch(r"end\s*do", s, re.I):
            indent -= 1
            continue
        m = re.match(r"call\s+(\w+)\s*\((.*)\)$", s, re.I)
        if m:
            py.append(pad + f"{m.group(1)}({m.group(2)})")
            continue
        m = re.match(r"([A-Za-z_]\w*)\s*(\(([^()]*)\))?\s*=\s*(.*)$", s)
        if m:
            lhs, idx, rhs = m.group(1), m.group(3), m.group(4)
            rhs = translate_expr(rhs, arrays)
            if idx is not None:
                idx = ",".join("ALL" if q.strip() == ":" else q for q in idx.split(","))
                idx = translate_expr(idx, arrays)
                py.append(pad + f"{lhs}[{idx}] = {rhs}")
            else:
                py.append(pad + f"{lhs} = {rhs}")
            continue
        raise ValueError(f"{name}: cannot translate: {s}")
    head = [f"def {name}({params}):"]
    for v, dims in decl_lines:
        if v in params.split(","):
            continue
        if numpy_arrays:
            head.append(f"    {v} = NArr('{v}', {dims}, {v in cplx})")
        else:
            head.append(f"    {v} = FArr('{v}', {dims})")
    return "\n".join(head + py) + "\n"


def load_kernels(ref_root):
    path = os.path.join(ref_root, "src", "imago", "gaussIntegrals.f90")
    with open(path) as fh:
        lines = fh.readlines()
    ns = {
        "FArr": FArr, "_ix": _ix, "f32": f32, "pi": 3.141592653589793,
        "_powi": _powi, "_apowi": _apowi, "NArr": NArr, "ALL": ALL,
        "cmplx": lambda re, im, kind=None: complex(re, im), "double": 8,
        # constants.f90:47, a double-kind parameter
        "fineStructure": float("7.2973525693"),
        "exp": _exp, "sqrt": math.sqrt, "erf": math.erf, "sum": _fsum,
        "abs": abs, "float": float,
    }
    for name, (a, b) in KERNEL_LINES.items():
        src = transpile(name, read_subroutine(lines, a, b))
        exec(compile(src, f"<{name}>", "exec"), ns)
    for name, (a, b) in NUMPY_KERNELS.items():
        src = transpile(name, read_subroutine(lines, a, b), numpy_arrays=True)
        exec(compile(src, f"<{name}>", "exec"), ns)
    return ns


def class_code(la, lb):
    return (1 << la) + (16 << lb)


def nsh(l):
    return (l + 1) ** 2


def run_2c(ns, kern, la, lb, a1, a2, A, B):
    sh = FArr("sh", [16, 16])
    ns[kern](a1, a2, np.array(A, float), np.array(B, float),
             class_code(la, lb), sh)
    return [[sh[i, j] for j in range(1, nsh(lb) + 1)]
            for i in range(1, nsh(la) + 1)]


def run_vec(ns, kern, la, lb, a1, a2, A, B, C=None):
    """Kernels with sh(16,16,3): one block per Cartesian component."""
    sh = FArr("sh", [16, 16, 3])
    args = [a1, a2, np.array(A, float), np.array(B, float)]
    if C is not None:
        args.append(np.array(C, float))
    ns[kern](*args, class_code(la, lb), sh)
    return [[[sh[i, j, c] for j in range(1, nsh(lb) + 1)]
             for i in range(1, nsh(la) + 1)] for c in range(1, 4)]


def run_k(ns, la, lb, a1, a2, A, B, dK):
    """KOverlap2CIntg: complex sh(16,16) as [re, im] pairs."""
    sh = NArr("sh", [16, 16], True)
    ns["KOverlap2CIntg"](a1, a2, np.array(A, float), np.array(B, float),
                         np.array(dK, float), class_code(la, lb), sh)
    return [[[sh[i, j].real, sh[i, j].imag] for j in range(1, nsh(lb) + 1)]
            for i in range(1, nsh(la) + 1)]


def run_3c(ns, kern, la, lb, a1, a2, a3, A, B, C):
    sh = FArr("sh", [16, 16])
    ns[kern](a1, a2, a3, np.array(A, float), np.array(B, float),
             np.array(C, float), class_code(la, lb), sh)
    return [[sh[i, j] for j in range(1, nsh(lb) + 1)]
            for i in range(1, nsh(la) + 1)]


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <root of the reference checkout>")
    ref_root = sys.argv[1]
    ns = load_kernels(ref_root)
    rng = np.random.default_rng(20261203)
    records = []
    # Alpha ranges span the configs' even-tempered sets (0.1 .. 1e6) and the
    # potential/nuclear exponents (0.1 .. 1e5, nucAlpha 20).
    for la in range(4):
        for lb in range(4):
            for rep in range(4):
                a1 = float(10 ** rng.uniform(-1, 3 if rep < 3 else 6))
                a2 = float(10 ** rng.uniform(-1, 3 if rep < 2 else 6))
                a3 = float(10 ** rng.uniform(-1, 2))
                # Place the centres so the Gaussian-product exponents
                # xi*|A-B|^2 and mu*|P-C|^2 land in [0, 9]: the values then
                # exercise every term instead of underflowing.
                xi = a1 * a2 / (a1 + a2)
                mu = (a1 + a2) * a3 / (a1 + a2 + a3)
                A = (rng.normal(size=3) * 1.5).tolist()
                u = rng.normal(size=3)
                u = u / np.linalg.norm(u)
                dab = math.sqrt(rng.uniform(0.0, 9.0) / xi)
                B = [A[i] + dab * u[i] for i in range(3)]
                if rep == 3:
                    B = list(A)  # same-centre pair (atom with itself, R=0)
                P = [(a1 * A[i] + a2 * B[i]) / (a1 + a2) for i in range(3)]
                v = rng.normal(size=3)
                v = v / np.linalg.norm(v)
                dpc = math.sqrt(rng.uniform(0.0, 9.0) / mu)
                C = [P[i] + dpc * v[i] for i in range(3)]
                rec = {"la": la, "lb": lb, "a1": a1, "a2": a2, "a3": a3,
                       "A": A, "B": B, "C": C}
                rec["overlap"] = run_2c(ns, "overlap2CIntg", la, lb, a1, a2, A, B)
                rec["kinetic"] = run_2c(ns, "kinetic2CIntg", la, lb, a1, a2, A, B)
                rec["massvel"] = run_2c(ns, "massvel2CIntg", la, lb, a1, a2, A, B)
                rec["momentum"] = run_vec(ns, "momentum2CIntg", la, lb, a1, a2, A, B)
                rec["dipole"] = run_vec(ns, "dipole3CIntg", la, lb, a1, a2, A, B, C)
                # a wave vector of the size of a reciprocal-lattice vector
                # over a k-point count (gaussKOverlap's deltaK)
                dK = (np.sin(np.arange(3) + 7 * la + 3 * lb + rep) * 0.6).tolist()
                rec["dK"] = dK
                rec["koverlap"] = run_k(ns, la, lb, a1, a2, A, B, dK)
                rec["electron3c"] = run_3c(ns, "electron3CIntg", la, lb,
                                           a1, a2, a3, A, B, C)
                rec["nuclear3c"] = run_3c(ns, "nuclear3CIntg", la, lb,
                                          a1, a2, a3, A, B, C)
                records.append(rec)
    # Nuclear records with the nucleus close to the product centre, so the
    # Boys argument falls in the series branch (T <= 0.1f).
    for la in range(4):
        for lb in range(4):
            a1 = float(10 ** rng.uniform(-1, 1))
            a2 = float(10 ** rng.uniform(-1, 1))
            a3 = 20.0
            A = (rng.normal(size=3) * 0.05).tolist()
            B = (rng.normal(size=3) * 0.05).tolist()
            z = a1 + a2 + a3
            G = [(a1 * A[i] + a2 * B[i]) / (a1 + a2) for i in range(3)]
            C = [G[i] + rng.normal() * 0.02 for i in range(3)]
            rec = {"la": la, "lb": lb, "a1": a1, "a2": a2, "a3": a3,
                   "A": A, "B": B, "C": C, "near": True}
            rec["nuclear3c"] = run_3c(ns, "nuclear3CIntg", la, lb,
                                      a1, a2, a3, A, B, C)
            rec["electron3c"] = run_3c(ns, "electron3CIntg", la, lb,
                                       a1, a2, a3, A, B, C)
            records.append(rec)
    # Nuclear records with the Boys argument U = zeta3*|G-C|^2 spread over
    # [0.02, 40], across the series/closed-form switch at 0.1f.
    for la in range(4):
        for lb in range(4):
            for rep in range(2):
                a1 = float(10 ** rng.uniform(-1, 2))
                a2 = float(10 ** rng.uniform(-1, 2))
                a3 = 20.0
                xi = a1 * a2 / (a1 + a2)
                A = (rng.normal(size=3) * 1.5).tolist()
                u = rng.normal(size=3)
                u = u / np.linalg.norm(u)
                dab = math.sqrt(rng.uniform(0.0, 6.0) / xi)
                B = [A[i] + dab * u[i] for i in range(3)]
                z = a1 + a2
                z3 = z + a3
                P = [(a1 * A[i] + a2 * B[i]) / z for i in range(3)]
                U = float(10 ** rng.uniform(math.log10(0.02), math.log10(40.0)))
                v = rng.normal(size=3)
                v = v / np.linalg.norm(v)
                dpc = math.sqrt(U * z3) / z
                C = [P[i] + dpc * v[i] for i in range(3)]
                rec = {"la": la, "lb": lb, "a1": a1, "a2": a2, "a3": a3,
                       "A": A, "B": B, "C": C, "mid": True}
                rec["nuclear3c"] = run_3c(ns, "nuclear3CIntg", la, lb,
                                          a1, a2, a3, A, B, C)
                records.append(rec)
    boys_T = [0.0, 1e-12, 1e-6, 1e-3, 0.05, 0.09999999999, 0.1,
              0.10000000149011611938, 0.1000000015, 0.10000001, 0.11, 0.2,
              0.5, 1.0, 2.0, 5.0, 10.0, 20.0, 33.0, 50.0, 100.0, 700.0]
    boys = []
    for T in boys_T:
        F = FArr("F", [7])
        ns["boys"](float(T), F)
        boys.append({"T": float(T), "F": [F[m] for m in range(1, 8)]})
    out = {
        "source": "src/imago/gaussIntegrals.f90 (overlap2CIntg, kinetic2CIntg,"
                  " electron3CIntg, boys, nuclear3CIntg, massvel2CIntg,"
                  " momentum2CIntg, dipole3CIntg, KOverlap2CIntg)"
                  " executed statement by statement in IEEE double",
        "generator": "tests/golden/make_golden.py",
        "records": records,
        "boys": boys,
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                       "primitives.json")
    with open(dst, "w") as fh:
        json.dump(out, fh, indent=None, separators=(",", ":"))
    print(f"wrote {dst}: {len(records)} records, {len(boys)} boys rows")


if __name__ == "__main__":
    main()
