"""Analytic primitives against numerical quadrature, as the reference
validates its generated integrals: osrecurintg.py in test mode emits a
program comparing each analytic formula with a brute-force 3-D Riemann sum
of the integrand on a cube (src/scripts/osrecurintgnum.py:874-1033,
src/imago/auxiliary/gaussIntgTest.f90:44-117).  Here the oracle's overlap,
kinetic and three-centre overlap primitives are compared with Riemann sums
of the same unnormalised real solid-harmonic Gaussians, in the reference's
harmonic order (src/scripts/osrecurintg.py:332-426).  The nuclear integral
(a 1/r singularity) is checked by the golden vectors only."""

import numpy as np
import pytest

import oracle

# sh components as polynomials: lists of (coefficient, (i, j, k)) for
# x^i y^j z^k, in the reference's order s; x; y; z; xy; xz; yz; xx-yy;
# 2zz-xx-yy; xyz; xxz-yyz; xxx-3yyx; 3xxy-yyy; 2zzz-3xxz-3yyz;
# 4zzx-xxx-yyx; 4zzy-xxy-yyy.
SH = [
    [(1, (0, 0, 0))],
    [(1, (1, 0, 0))], [(1, (0, 1, 0))], [(1, (0, 0, 1))],
    [(1, (1, 1, 0))], [(1, (1, 0, 1))], [(1, (0, 1, 1))],
    [(1, (2, 0, 0)), (-1, (0, 2, 0))],
    [(2, (0, 0, 2)), (-1, (2, 0, 0)), (-1, (0, 2, 0))],
    [(1, (1, 1, 1))],
    [(1, (2, 0, 1)), (-1, (0, 2, 1))],
    [(1, (3, 0, 0)), (-3, (1, 2, 0))],
    [(3, (2, 1, 0)), (-1, (0, 3, 0))],
    [(2, (0, 0, 3)), (-3, (2, 0, 1)), (-3, (0, 2, 1))],
    [(4, (1, 0, 2)), (-1, (3, 0, 0)), (-1, (1, 2, 0))],
    [(4, (0, 1, 2)), (-1, (2, 1, 0)), (-1, (0, 3, 0))],
]
NSH = [1, 4, 9, 16]

H = 0.1
AX = np.arange(-7.0, 7.0 + H / 2, H)
X, Y, Z = np.meshgrid(AX, AX, AX, indexing="ij", sparse=True)


def _poly(terms, dx, dy, dz):
    out = 0.0
    for c, (i, j, k) in terms:
        out = out + c * dx ** i * dy ** j * dz ** k
    return out


def _dpoly(terms, axis):
    out = []
    for c, e in terms:
        if e[axis] > 0:
            e2 = list(e)
            e2[axis] -= 1
            out.append((c * e[axis], tuple(e2)))
    return out


def _functions(l, a, A, grad=False):
    dx, dy, dz = X - A[0], Y - A[1], Z - A[2]
    g = np.exp(-a * (dx * dx + dy * dy + dz * dz))
    fs = []
    for terms in SH[:NSH[l]]:
        p = _poly(terms, dx, dy, dz)
        if not grad:
            fs.append(p * g)
        else:
            d = [(_poly(_dpoly(terms, ax), dx, dy, dz) if _dpoly(terms, ax) else 0.0)
                 - 2.0 * a * (dx, dy, dz)[ax] * p for ax in range(3)]
            fs.append([di * g for di in d])
    return fs


def _quadrature(kind, la, lb, a1, a2, a3, A, B, C):
    out = np.zeros((16, 16))
    w = H ** 3
    if kind == 1:  # <a| -1/2 nabla^2 |b> = 1/2 <grad a | grad b>
        fa, fb = _functions(la, a1, A, True), _functions(lb, a2, B, True)
        for i, gi in enumerate(fa):
            for j, gj in enumerate(fb):
                out[i, j] = 0.5 * w * sum(float(np.sum(gi[x] * gj[x])) for x in range(3))
        return out
    fa, fb = _functions(la, a1, A), _functions(lb, a2, B)
    third = 1.0
    if kind == 2:
        third = np.exp(-a3 * ((X - C[0]) ** 2 + (Y - C[1]) ** 2 + (Z - C[2]) ** 2))
    for i, f in enumerate(fa):
        ft = f * third
        for j, g in enumerate(fb):
            out[i, j] = w * float(np.sum(ft * g))
    return out


CASES = [(0, 0, 1.1, 0.9), (1, 0, 1.3, 0.8), (1, 1, 0.9, 1.2), (2, 1, 1.0, 1.4),
         (2, 2, 1.2, 0.95), (3, 2, 1.5, 1.1)]


@pytest.mark.parametrize("kind", ["overlap", "kinetic", "electron3c"])
@pytest.mark.parametrize("la,lb,a1,a2", CASES)
def test_primitive_matches_riemann_sum(kind, la, lb, a1, a2):
    A = np.array([0.31, -0.42, 0.25])
    B = np.array([-0.55, 0.37, 0.61])
    C = np.array([0.12, 0.48, -0.33])
    a3 = 0.7
    got = oracle.primitive(kind, la, lb, a1, a2, a3, A, B, C)
    code = {"overlap": 0, "kinetic": 1, "electron3c": 2}[kind]
    ref = _quadrature(code, la, lb, a1, a2, a3, A, B, C)[:NSH[la], :NSH[lb]]
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 1e-9 * scale, (got, ref)
