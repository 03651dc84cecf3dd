"""ctypes access to the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA integral path.  It is
imported by tests/, by __graft_entry__.smoke() and by bench.py's CPU
baseline leg, never by the imago_b200 package.  See oracle.h for what it
restates and how its parity is pinned.
"""

import ctypes
import os
import subprocess

import numpy as np

from imago_b200.system import ImagoDimsC

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_D = ctypes.POINTER(ctypes.c_double)


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        for name in ("orc_overlap2c", "orc_kinetic2c", "orc_massvel2c"):
            f = getattr(L, name)
            f.argtypes = [ctypes.c_double, ctypes.c_double, _D, _D,
                          ctypes.c_int, ctypes.c_int, _D]
            f.restype = None
        L.orc_momentum2c.argtypes = [ctypes.c_double, ctypes.c_double, _D, _D,
                                     ctypes.c_int, ctypes.c_int, _D]
        L.orc_momentum2c.restype = None
        L.orc_dipole2c.argtypes = [ctypes.c_double, ctypes.c_double, _D, _D, _D,
                                   ctypes.c_int, ctypes.c_int, _D]
        L.orc_dipole2c.restype = None
        L.orc_koverlap2c.argtypes = [ctypes.c_double, ctypes.c_double, _D, _D, _D,
                                     ctypes.c_int, ctypes.c_int, _D]
        L.orc_koverlap2c.restype = None
        for name in ("orc_electron3c", "orc_nuclear3c"):
            f = getattr(L, name)
            f.argtypes = [ctypes.c_double] * 3 + [_D, _D, _D, ctypes.c_int,
                                                  ctypes.c_int, _D]
            f.restype = None
        L.orc_boys.argtypes = [ctypes.c_double, _D]
        L.orc_boys.restype = None
        L.orc_create.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
        L.orc_create.restype = ctypes.c_int
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_destroy.restype = None
        L.orc_dims.argtypes = [ctypes.c_void_p, ctypes.POINTER(ImagoDimsC)]
        L.orc_set_sampling.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_set_sampling.restype = None
        L.orc_set_skip_ortho.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_set_skip_ortho.restype = None
        L.orc_gauss_overlap_ol.argtypes = [ctypes.c_void_p, _D, _D, _D]
        L.orc_gauss_overlap_ke.argtypes = [ctypes.c_void_p, _D]
        L.orc_gauss_overlap_np.argtypes = [ctypes.c_void_p, _D]
        L.orc_gauss_overlap_mv.argtypes = [ctypes.c_void_p, _D]
        L.orc_gauss_overlap_mm.argtypes = [ctypes.c_void_p, _D]
        L.orc_gauss_overlap_dm.argtypes = [ctypes.c_void_p, _D, _D]
        L.orc_gauss_koverlap.argtypes = [ctypes.c_void_p, _D, _D, _D]
        L.orc_ham_pscf.argtypes = [ctypes.c_void_p, ctypes.c_int, _D,
                                   ctypes.c_int, _D]
        L.orc_elec_pot_gauss_overlap.argtypes = [ctypes.c_void_p, ctypes.c_int,
                                                 ctypes.c_int, _D]
        L.orc_last_times.argtypes = [ctypes.c_void_p, _D, _D]
        L.orc_last_times.restype = None
        L.orc_num_cells.argtypes = [ctypes.c_void_p]
        L.orc_cells.argtypes = [ctypes.c_void_p, _D, _D]
        L.orc_cells.restype = None
        L.orc_kpoints_xyz.argtypes = [ctypes.c_void_p, _D]
        L.orc_kpoints_xyz.restype = None
        L.orc_find_lattice_vector.argtypes = [ctypes.c_void_p, _D, _D]
        L.orc_find_lattice_vector.restype = None
        L.orc_last_counts.argtypes = [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_longlong)] * 3
        L.orc_last_counts.restype = None
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(_D)


def primitive_vec(kind, la, lb, a1, a2, A, B, C=None):
    """Three-component blocks [3, nsh(la), nsh(lb)]: kind momentum
    (momentum2CIntg) or dipole (dipole3CIntg, operator centre C)."""
    L = lib()
    sh = np.zeros(768)
    A = np.ascontiguousarray(A, float)
    B = np.ascontiguousarray(B, float)
    if kind == "momentum":
        L.orc_momentum2c(a1, a2, _p(A), _p(B), la, lb, _p(sh))
    elif kind == "dipole":
        C = np.ascontiguousarray(C, float)
        L.orc_dipole2c(a1, a2, _p(A), _p(B), _p(C), la, lb, _p(sh))
    else:
        raise ValueError(kind)
    n1, n2 = (la + 1) ** 2, (lb + 1) ** 2
    return sh.reshape(3, 16, 16)[:, :n1, :n2].copy()


def primitive_koverlap(la, lb, a1, a2, A, B, dK):
    """<a|exp(-i dK.r)|b> (KOverlap2CIntg) as a complex [nsh(la), nsh(lb)]."""
    sh = np.zeros(512)
    arr = [np.ascontiguousarray(v, float) for v in (A, B, dK)]
    lib().orc_koverlap2c(a1, a2, _p(arr[0]), _p(arr[1]), _p(arr[2]), la, lb, _p(sh))
    c = sh[0::2] + 1j * sh[1::2]
    n1, n2 = (la + 1) ** 2, (lb + 1) ** 2
    return c.reshape(16, 16)[:n1, :n2].copy()


def primitive(kind, la, lb, a1, a2, a3, A, B, C):
    """Reference-layout sh block (nsh(la) x nsh(lb)) from the oracle.
    kind: overlap, kinetic, massvel, electron3c, nuclear3c."""
    L = lib()
    sh = np.zeros(256)
    A = np.ascontiguousarray(A, float)
    B = np.ascontiguousarray(B, float)
    C = np.ascontiguousarray(C, float)
    if kind == "overlap":
        L.orc_overlap2c(a1, a2, _p(A), _p(B), la, lb, _p(sh))
    elif kind == "kinetic":
        L.orc_kinetic2c(a1, a2, _p(A), _p(B), la, lb, _p(sh))
    elif kind == "massvel":
        L.orc_massvel2c(a1, a2, _p(A), _p(B), la, lb, _p(sh))
    elif kind == "electron3c":
        L.orc_electron3c(a1, a2, a3, _p(A), _p(B), _p(C), la, lb, _p(sh))
    elif kind == "nuclear3c":
        L.orc_nuclear3c(a1, a2, a3, _p(A), _p(B), _p(C), la, lb, _p(sh))
    else:
        raise ValueError(kind)
    n1, n2 = (la + 1) ** 2, (lb + 1) ** 2
    return sh.reshape(16, 16)[:n1, :n2].copy()


def boys(T):
    F = np.zeros(7)
    lib().orc_boys(float(T), _p(F))
    return F


class OracleBuild:
    """The reference's four integral builds restated on the CPU."""

    def __init__(self, system, stride=1, nthreads=0):
        self.system = system
        self._cs, self._keep = system.to_c()
        self._ctx = ctypes.c_void_p()
        st = lib().orc_create(ctypes.byref(self._cs), ctypes.byref(self._ctx))
        if st != 0:
            raise RuntimeError(f"orc_create failed with status {st}")
        lib().orc_set_sampling(self._ctx, stride, nthreads)
        d = ImagoDimsC()
        lib().orc_dims(self._ctx, ctypes.byref(d))
        self.vale_dim, self.core_dim = d.vale_dim, d.core_dim
        self.nk, self.pot_dim, self.num_cells = d.num_kpoints, d.pot_dim, d.num_cells
        self.npacked = int(d.packed)

    def close(self):
        if self._ctx:
            lib().orc_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _packed(self, n=1):
        return np.zeros((n, self.nk, self.npacked, 2))

    def _check(self, st, what):
        if st != 0:
            raise RuntimeError(f"{what} failed with status {st}")

    def overlap(self):
        out = self._packed()
        cre = np.zeros((self.nk, self.vale_dim, max(self.core_dim, 1)))
        cim = np.zeros_like(cre)
        self._check(lib().orc_gauss_overlap_ol(self._ctx, _p(out), _p(cre), _p(cim)), "OL")
        return out[0], cre[:, :, :self.core_dim], cim[:, :, :self.core_dim]

    def kinetic(self):
        out = self._packed()
        self._check(lib().orc_gauss_overlap_ke(self._ctx, _p(out)), "KE")
        return out[0]

    def mass_velocity(self):
        out = self._packed()
        self._check(lib().orc_gauss_overlap_mv(self._ctx, _p(out)), "MV")
        return out[0]

    def momentum(self):
        """gaussOverlapMM: [3, nk, np, 2] (x, y, z)."""
        out = self._packed(3)
        self._check(lib().orc_gauss_overlap_mm(self._ctx, _p(out)), "MM")
        return out

    def dipole(self, center):
        """gaussOverlapDM about `center` (xyz): [3, nk, np, 2]."""
        c = np.ascontiguousarray(center, dtype=np.float64)
        out = self._packed(3)
        self._check(lib().orc_gauss_overlap_dm(self._ctx, _p(c), _p(out)), "DM")
        return out

    def koverlap(self, dk):
        """gaussKOverlap for the three wave vectors dk [3, 3] (axis, xyz):
        complex [3, nk, V, V] (row, col)."""
        dk = np.ascontiguousarray(dk, dtype=np.float64).reshape(9)
        nk = self.nk
        V = self.vale_dim
        re = np.zeros((3, nk, V, V))
        im = np.zeros_like(re)
        self._check(lib().orc_gauss_koverlap(self._ctx, _p(dk), _p(re), _p(im)), "KOV")
        # planes are [col][row]: transpose to [row][col]
        return (re + 1j * im).transpose(0, 1, 3, 2)

    def ham_pscf(self, coeffs, rel=False):
        """gaussOverlapHamPSCF: coeffs [potDim] or [potDim, spin] ->
        [spin, nk, np, 2]."""
        coeffs = np.asarray(coeffs, dtype=np.float64)
        if coeffs.ndim == 1:
            coeffs = coeffs[:, None]
        spin = coeffs.shape[1]
        cf = np.ascontiguousarray(coeffs.T)  # potCoeffs(potDim, spin)
        out = self._packed(spin)
        self._check(lib().orc_ham_pscf(self._ctx, spin, _p(cf), 1 if rel else 0,
                                       _p(out)), "HamPSCF")
        return out

    def nuclear(self):
        out = self._packed()
        self._check(lib().orc_gauss_overlap_np(self._ctx, _p(out)), "NP")
        return out[0]

    def elec_pot(self, lo=0, hi=None):
        hi = self.pot_dim if hi is None else hi
        out = self._packed(hi - lo)
        self._check(lib().orc_elec_pot_gauss_overlap(self._ctx, lo, hi, _p(out)), "EP")
        return out

    def set_skip_ortho(self, skip=True):
        """Timing samples only: run the pair loops without the
        orthogonalisation and packing (outputs are left unwritten)."""
        lib().orc_set_skip_ortho(self._ctx, 1 if skip else 0)

    def last_times(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        lib().orc_last_times(self._ctx, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def last_counts(self):
        x = [ctypes.c_longlong() for _ in range(3)]
        lib().orc_last_counts(self._ctx, *[ctypes.byref(v) for v in x])
        return tuple(v.value for v in x)

    def cells(self):
        n = lib().orc_num_cells(self._ctx)
        d, s = np.zeros((n, 3)), np.zeros(n)
        lib().orc_cells(self._ctx, _p(d), _p(s))
        return d, s

    def kpoints_xyz(self):
        k = np.zeros((self.nk, 3))
        lib().orc_kpoints_xyz(self._ctx, _p(k))
        return k

    def nearest_lattice_vector(self, v):
        v = np.ascontiguousarray(v, float)
        o = np.zeros(3)
        lib().orc_find_lattice_vector(self._ctx, _p(v), _p(o))
        return o


def secular_eigenvalues(np_packed, ke_packed, ep_packed, pot_coeffs, ol_packed,
                        mv_packed=None):
    """The secular equation of one SCF step on the CPU, as secularEqnSCF
    (secularEqn.F90:135-186) does it: H = NP + KE (+ MV for a
    scalar-relativistic run) + sum_j w_j EP_j in that
    order with readPackedMatrixAccum's rule (a factor of exactly 0.0 adds
    the matrix unscaled, matrixSubs.F90:369-373), upper triangles unpacked
    (matrixSubs.F90:405-433), then LAPACK's generalised Hermitian solver
    (scipy.linalg.eigh(H, S), the problem of zhegv(1, 'V', 'U')).
    Returns [nk, V] eigenvalues, ascending."""
    import scipy.linalg
    nk, npk = np_packed.shape[0], np_packed.shape[1]
    V = int((int((8 * npk + 1) ** 0.5) - 1) // 2)
    iu = np.triu_indices(V)
    # packed index of (row, col), row <= col: col (col + 1) / 2 + row
    pidx = iu[1] * (iu[1] + 1) // 2 + iu[0]
    out = np.zeros((nk, V))
    for k in range(nk):
        hp = np_packed[k, :, 0] + 1j * np_packed[k, :, 1]
        hp = hp + (ke_packed[k, :, 0] + 1j * ke_packed[k, :, 1])
        if mv_packed is not None:  # rel == 1, secularEqn.F90:157-163
            hp = hp + (mv_packed[k, :, 0] + 1j * mv_packed[k, :, 1])
        for j, w in enumerate(pot_coeffs):
            f = 1.0 if w == 0.0 else w
            hp = hp + (ep_packed[j, k, :, 0] + 1j * ep_packed[j, k, :, 1]) * f
        sp = ol_packed[k, :, 0] + 1j * ol_packed[k, :, 1]
        H = np.zeros((V, V), complex)
        S = np.zeros((V, V), complex)
        H[iu] = hp[pidx]
        S[iu] = sp[pidx]
        out[k] = scipy.linalg.eigh(H, S, lower=False, eigvals_only=True)
    return out


def _secular_hs(np_packed, ke_packed, ep_packed, pot_coeffs, ol_packed, mv_packed, k):
    """H and S of k-point k, upper triangles, as secular_eigenvalues forms them."""
    npk = np_packed.shape[1]
    V = int((int((8 * npk + 1) ** 0.5) - 1) // 2)
    iu = np.triu_indices(V)
    pidx = iu[1] * (iu[1] + 1) // 2 + iu[0]
    hp = np_packed[k, :, 0] + 1j * np_packed[k, :, 1]
    hp = hp + (ke_packed[k, :, 0] + 1j * ke_packed[k, :, 1])
    if mv_packed is not None:
        hp = hp + (mv_packed[k, :, 0] + 1j * mv_packed[k, :, 1])
    for j, w in enumerate(pot_coeffs):
        f = 1.0 if w == 0.0 else w
        hp = hp + (ep_packed[j, k, :, 0] + 1j * ep_packed[j, k, :, 1]) * f
    sp = ol_packed[k, :, 0] + 1j * ol_packed[k, :, 1]
    H = np.zeros((V, V), complex)
    S = np.zeros((V, V), complex)
    H[iu] = hp[pidx]
    S[iu] = sp[pidx]
    return H, S


def populate_standard(eigenvalues, num_electrons, kpoint_weights=None):
    """populateStandard (populate.F90:190-483) statement by statement, with
    Python loops (small cases only): eigenvalues [nk, spin, numStates].
    Returns (population [nk, spin, numStates], occupiedEnergy,
    occupiedEnergyIndex (0-based), bandGap, gapKindCode)."""
    small, metal_gap = 1.0e-8, 1.0e-3    # constants.f90:49, populate.F90
    e = np.asarray(eigenvalues, dtype=np.float64)
    nk, spin, ns = e.shape
    kw = [2.0 / nk] * nk if kpoint_weights is None else list(kpoint_weights)
    temp = [e[i, j, k] for i in range(nk) for j in range(spin) for k in range(ns)]
    n = len(temp)
    index = sorted(range(n), key=lambda i: temp[i])   # stable, ascending
    srt = [temp[i] for i in index]
    wt = lambda idx: kw[idx // (ns * spin)] / float(spin)
    pop = [0.0] * n
    populated = 0.0
    ne = float(num_electrons)
    occ = None
    for i in range(n):
        pop[index[i]] = wt(index[i])
        populated = populated + pop[index[i]]
        if populated > ne:
            pop[index[i]] = wt(index[i]) + ne - populated
            populated = ne
        if abs(ne - populated) < small:
            occ = i
            break
    if occ is None:
        raise ValueError("fewer states than electrons")
    occ_e = srt[occ]
    lo = hi = occ
    degen = pop[index[occ]]
    possible = wt(index[occ])
    while hi + 1 < n and abs(occ_e - srt[hi + 1]) <= small:
        hi += 1
        possible = possible + wt(index[hi])
    while lo > 0 and abs(occ_e - srt[lo - 1]) <= small:
        lo -= 1
        possible = possible + wt(index[lo])
        degen = degen + wt(index[lo])
    for i in range(lo, hi + 1):
        pop[index[i]] = degen / possible * wt(index[i])
    occ = hi
    occ_e = srt[occ]
    if occ >= n - 1:
        gap, kind = 0.0, 0
    else:
        gap = srt[occ + 1] - srt[occ]
        if gap <= metal_gap:
            gap, kind = 0.0, 0
        else:
            vbm, cbm = index[occ] // (ns * spin), index[occ + 1] // (ns * spin)
            kind = 1 if vbm == cbm else 2
    return np.array(pop).reshape(nk, spin, ns), occ_e, occ, gap, kind


def populate_smearing(eigenvalues, num_electrons, thermal_sigma, max_thermal_range,
                      fermi_search_limit, kpoint_weights=None):
    """populateSmearing (populate.F90:486-620) statement by statement with
    Python loops and stepFunction (mathSubs.f90:164-185), after
    populate_standard.  Returns (population, occupiedEnergy, iterations)."""
    import math
    e = np.asarray(eigenvalues, dtype=np.float64)
    nk, spin, ns = e.shape
    _, _, occ, _, _ = populate_standard(e, num_electrons, kpoint_weights)
    kw = [2.0 / nk] * nk if kpoint_weights is None else list(kpoint_weights)
    temp = [e[i, j, k] for i in range(nk) for j in range(spin) for k in range(ns)]
    n = len(temp)
    index = sorted(range(n), key=lambda i: temp[i])
    srt = [temp[i] for i in index]

    def step(x, r):
        if x > r:
            return 0.0
        if x < -r:
            return 1.0
        return 1.0 / (1.0 + math.exp(x))

    lo = srt[occ] - fermi_search_limit
    hi = srt[min(occ + 1, n - 1)] + fermi_search_limit
    ne = float(num_electrons)
    pop = [0.0] * n
    ef, it = 0.0, 0
    for it in range(1, 501):
        ef = 0.5 * (lo + hi)
        charge = 0.0
        pop = [0.0] * n
        for j in range(n):
            f = step((srt[j] - ef) / thermal_sigma, max_thermal_range)
            if f == 0.0:
                break
            pop[index[j]] = (kw[index[j] // (ns * spin)] / float(spin)) * f
            charge = charge + pop[index[j]]
        if abs(charge - ne) < 1.0e-8:
            break
        if charge < ne:
            lo = ef
        else:
            hi = ef
    return np.array(pop).reshape(nk, spin, ns), ef, it


def matrix_element_mult(m1, m2):
    """matrixElementMult (matrixSubs.F90:66-109) on one packed pair
    [nPacked, 2]: off-diagonal re*re + im*im, diagonal re*re / 2, times 2."""
    npk = m1.shape[0]
    V = int((int((8 * npk + 1) ** 0.5) - 1) // 2)
    t = 0.0
    d = 0
    for i in range(1, V + 1):
        seg = slice(d, d + i - 1)
        t += float(np.dot(m1[seg, 0], m2[seg, 0]) + np.dot(m1[seg, 1], m2[seg, 1]))
        d += i
        t += m1[d - 1, 0] * m2[d - 1, 0] / 2.0
    return t * 2.0


def valence_rho(np_packed, ke_packed, ep_packed, ol_packed, pot_coeffs, num_electrons,
                num_states, mv_packed=None, kpoint_weights=None):
    """One step of secularEqnSCF, populateStandard and makeValenceRho's
    traces (valeCharge.F90:34-488) on the CPU: LAPACK's eigh(H, S) per k
    and spin (pot_coeffs [potDim, spin]), rank-one updates of the upper
    triangle per occupied state, packMatrix, matrixElementMult.  Returns a
    dict named as the reference's variables, plus "population"."""
    import scipy.linalg
    w = np.asarray(pot_coeffs, dtype=np.float64)
    if w.ndim == 1:
        w = w[:, None]
    spin = w.shape[1]
    nk = np_packed.shape[0]
    ev = np.zeros((nk, spin, num_states))
    vecs = {}
    for k in range(nk):
        for s in range(spin):
            H, S = _secular_hs(np_packed, ke_packed, ep_packed, w[:, s], ol_packed,
                               mv_packed, k)
            e, c = scipy.linalg.eigh(H, S, lower=False)
            ev[k, s] = e[:num_states]
            vecs[k, s] = c[:, :num_states]
    pop, occ_e, _, gap, kind = populate_standard(ev, num_electrons, kpoint_weights)
    V = vecs[0, 0].shape[0]
    iu = np.triu_indices(V)
    pidx = iu[1] * (iu[1] + 1) // 2 + iu[0]
    order = np.argsort(pidx)
    npk = V * (V + 1) // 2
    mats = {"chargeDensityTrace": ol_packed, "nucPotTrace": np_packed,
            "kineticEnergyTrace": ke_packed}
    if mv_packed is not None:
        mats["massVelocityTrace"] = mv_packed
    res = {key: np.zeros(spin) for key in mats}
    res["potRho"] = np.zeros((ep_packed.shape[0], spin))
    res["electronEnergy"] = np.zeros(spin)
    for k in range(nk):
        rho = []
        for s in range(spin):
            r = np.zeros((V, V), complex)
            for j in range(num_states):
                f = pop[k, :, j]
                if np.abs(f).sum() < 1.0e-8:
                    continue
                res["electronEnergy"][s] += f[s] * ev[k, s, j]
                c = vecs[k, s][:, j]
                r += f[s] * np.outer(c, np.conj(c))
            p = np.zeros((npk, 2))
            p[:, 0] = r[iu][order].real
            p[:, 1] = r[iu][order].imag
            rho.append(p)
        if spin == 2:
            rho = [rho[0] + rho[1], rho[0] - rho[1]]
        for s in range(spin):
            for key, m in mats.items():
                res[key][s] += matrix_element_mult(m[k], rho[s])
            for t in range(ep_packed.shape[0]):
                res["potRho"][t, s] += matrix_element_mult(ep_packed[t, k], rho[s])
    mv = res.get("massVelocityTrace", np.zeros(spin))
    ke, nuc, pr = res["kineticEnergyTrace"], res["nucPotTrace"], res["potRho"]
    if spin == 1:
        res["sumElecEnergy"] = np.array([(w[:, 0] * pr[:, 0]).sum() + ke[0] + mv[0] + nuc[0]])
    else:
        res["sumElecEnergy"] = np.array([
            0.5 * ((w[:, 0] * (pr[:, 0] + pr[:, 1])).sum() + ke[0] + ke[1] + mv[0] + mv[1]
                   + nuc[0] + nuc[1]),
            0.5 * ((w[:, 1] * (pr[:, 0] - pr[:, 1])).sum() + ke[0] - ke[1] + mv[0] - mv[1]
                   + nuc[0] - nuc[1])])
    res["population"] = pop
    res["occupiedEnergy"], res["bandGap"], res["gapKindCode"] = occ_e, gap, kind
    res["eigenvalues"] = ev
    return res
