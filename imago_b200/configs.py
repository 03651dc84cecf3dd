"""Synthetic systems for the workloads this library is measured on.

The reference builds its decks with makeinput.py from the atomic basis
database `src/data/atomicBDB`, which is not available, so the contracted
radial functions here are synthesised: each radial function is a
least-squares fit of a Slater-type orbital r^(n-1) e^(-zeta r) (Slater-rule
style exponents) onto the even-tempered primitives r^l e^(-alpha r^2),
normalised, and Gram-Schmidt orthogonalised against the lower functions of
the same l.  Positions, strains and jitters are drawn from seeded
generators, so every call returns the same system.

Workloads (sizes are the ones the integral path is quoted on):
  diamond_primitive  2 C atoms, fcc a=3.567 A, 1s core + 2s 2p valence,
                     16 even-tempered primitives 0.12..1e6, 16 potential
                     terms 0.12..1e5, 4x4x4 k.
  silicon_cubic8     8 Si, a=5.431 A, jitter N(0, 0.02 A), s,p,d basis of 20
                     primitives 0.10..5e5 (NUM_ALPHA_S_P_D_F 20 20 14 0),
                     1s 2s 2p core + 3s 3p 4s 4p 3d valence, 20 potential
                     terms 0.10..1e5, 8x8x8 k.
  quartz_supercell   alpha-quartz SiO2 3x3x2 (162 atoms), jitter
                     N(0, 0.03 A); Si as above, O 18 primitives 0.12..3e5
                     (18 18 0 0), 1s core + 2s 2p 3s 3p valence; 20 potential
                     terms per element; Gamma or 2x2x2 k.
  graphite_cell      AB graphite a=2.46 A, c=6.71 A.
  batch_cells        64 independent cells of uneven size for the batched
                     stream: Si (8..64 atoms), diamond and graphite (8..216
                     atoms) supercells, each strained by a random symmetric
                     strain with components in +-3% and jittered by
                     N(0, 0.02 A), 2x2x2 k.
"""

import math

import numpy as np

from .system import AtomType, ImagoSystem, PotType, kpoint_mesh, pot_alphas

ANGSTROM = 1.0 / 0.529177210903  # bohr per angstrom (constants.f90:43)


def even_tempered(n, amin, amax):
    return np.array([amin * (amax / amin) ** (i / (n - 1)) for i in range(n)])


def _fit_radial(alphas, l, n, zeta):
    """Coefficients c_i so that sum_i c_i r^l exp(-alpha_i r^2) fits
    r^(n-1) exp(-zeta r) on a radial grid."""
    r = np.exp(np.linspace(math.log(1e-4), math.log(40.0), 1500))
    w = np.sqrt(r ** 3)  # r^2 dr on a log grid
    target = r ** (n - 1) * np.exp(-zeta * r)
    basis = (r[:, None] ** l) * np.exp(-np.outer(r * r, alphas))
    coef, *_ = np.linalg.lstsq(basis * w[:, None], target * w, rcond=1e-12)
    return coef


def _radial_overlap(alphas, l, c1, c2):
    """Integral of R1 R2 r^2 dr with R = sum c r^l exp(-a r^2)."""
    s = alphas[:, None] + alphas[None, :]
    g = math.gamma(l + 1.5) / (2.0 * s ** (l + 1.5))
    return float(c1 @ g @ c2)


def _make_type(element, label, alphas, norb, core, vale):
    """core/vale: lists of (n, l, zeta).  Functions are stored l-major, n
    within l, the order the reference's contracted basis files use
    (src/contract/printResults.f90:71-115)."""
    t = AtomType(element=element, label=label, num_orb_alphas=list(norb),
                 alphas=np.asarray(alphas, float))
    core = sorted(core, key=lambda f: (f[1], f[0]))
    vale = sorted(vale, key=lambda f: (f[1], f[0]))
    done = []
    for kind, lst in (("core", core), ("vale", vale)):
        for (n, l, zeta) in lst:
            a = t.alphas[:norb[l]]
            c = _fit_radial(a, l, n, zeta)
            for (l2, c2) in done:
                if l2 == l:
                    c = c - _radial_overlap(a, l, c, c2) * c2
            c = c / math.sqrt(_radial_overlap(a, l, c, c))
            done.append((l, c))
            if kind == "core":
                t.core_l.append(l)
                t.core_n.append(n)
                t.core_coeffs.append(c)
            else:
                t.vale_l.append(l)
                t.vale_n.append(n)
                t.vale_coeffs.append(c)
    return t


def carbon_type(element=1, label="c1_1", nprim=16, amin=0.12, amax=1.0e6,
                extended=False):
    vale = [(2, 0, 1.608), (2, 1, 1.568)]
    if extended:
        vale += [(3, 0, 0.9), (3, 1, 0.8)]
    return _make_type(element, label, even_tempered(nprim, amin, amax),
                      (nprim, nprim, 0, 0), [(1, 0, 5.673)], vale)


def silicon_type(element=1, label="si1_1", nprim=20, amin=0.10, amax=5.0e5,
                 nd=14):
    core = [(1, 0, 13.575), (2, 0, 4.903), (2, 1, 5.086)]
    vale = [(3, 0, 1.634), (3, 1, 1.428), (4, 0, 0.80), (4, 1, 0.70),
            (3, 2, 1.00)]
    return _make_type(element, label, even_tempered(nprim, amin, amax),
                      (nprim, nprim, nd, 0), core, vale)


def oxygen_type(element=2, label="o1_1", nprim=18, amin=0.12, amax=3.0e5):
    vale = [(2, 0, 2.246), (2, 1, 2.227), (3, 0, 0.95), (3, 1, 0.85)]
    return _make_type(element, label, even_tempered(nprim, amin, amax),
                      (nprim, nprim, 0, 0), [(1, 0, 7.658)], vale)


def _pot(element, label, Z, nterms, amin, amax, nuc_alpha=20.0):
    return PotType(element=element, label=label, nuc_charge=float(Z),
                   nuc_alpha=nuc_alpha, alphas=pot_alphas(nterms, amin, amax))


def _system(rv, types, site_type, pos, pots, pot_site_type, k, convg=1e-16,
            title="", kmesh=None):
    sys_ = ImagoSystem(real_vectors=np.asarray(rv, float), atom_types=types,
                       site_type=np.asarray(site_type, np.int32),
                       site_pos=np.asarray(pos, float), pot_types=pots,
                       pot_site_type=np.asarray(pot_site_type, np.int32),
                       pot_site_pos=np.asarray(pos, float),
                       kpoints_abc=np.asarray(k, float), basis_fn_convg=convg,
                       electro_convg=convg, title=title, kmesh=kmesh)
    sys_.validate()
    return sys_


def _mesh(n, shift):
    return kpoint_mesh(n, shift), (tuple(n), tuple(shift))


def diamond_primitive(kmesh=(4, 4, 4), shift=(0.5, 0.5, 0.5)):
    a = 3.567 * ANGSTROM
    rv = [[0, a / 2, a / 2], [a / 2, 0, a / 2], [a / 2, a / 2, 0]]
    pos = [[0, 0, 0], [a / 4, a / 4, a / 4]]
    t = carbon_type()
    p = _pot(1, "c1_1", 6, 16, 0.12, 1.0e5)
    k, km = _mesh(kmesh, shift)
    return _system(rv, [t], [1, 1], pos, [p], [1, 1], k,
                   title="diamond primitive cell", kmesh=km)


DIAMOND_FRAC = [[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                [.25, .25, .25], [.25, .75, .75], [.75, .25, .75],
                [.75, .75, .25]]


def silicon_cubic8(kmesh=(8, 8, 8), shift=(0.5, 0.5, 0.5), seed=2,
                   jitter=0.02, nd=14, npot=20):
    a = 5.431 * ANGSTROM
    rng = np.random.default_rng(seed)
    rv = np.eye(3) * a
    pos = np.array(DIAMOND_FRAC) @ rv
    pos = pos + rng.normal(0.0, jitter * ANGSTROM, size=pos.shape)
    t = silicon_type(nd=nd)
    p = _pot(1, "si1_1", 14, npot, 0.10, 1.0e5)
    k, km = _mesh(kmesh, shift)
    return _system(rv, [t], [1] * 8, pos, [p], [1] * 8, k,
                   title="silicon conventional cell, jittered", kmesh=km)


def _hex(a, c):
    return np.array([[a, 0, 0], [-a / 2, a * math.sqrt(3) / 2, 0], [0, 0, c]])


def _apply_ops(ops, frac):
    out = []
    for op in ops:
        p = np.array(op(*frac)) % 1.0
        if not any(np.allclose((p - q + 0.5) % 1.0 - 0.5, 0, atol=1e-6)
                   for q in out):
            out.append(p)
    return out


P3121 = [lambda x, y, z: (x, y, z),
         lambda x, y, z: (-y, x - y, z + 1 / 3),
         lambda x, y, z: (-x + y, -x, z + 2 / 3),
         lambda x, y, z: (y, x, -z),
         lambda x, y, z: (x - y, -y, -z + 2 / 3),
         lambda x, y, z: (-x, -x + y, -z + 1 / 3)]


def quartz_supercell(reps=(3, 3, 2), kmesh=(2, 2, 2), shift=(0.5, 0.5, 0.5),
                     seed=3, jitter=0.03, npot=20, gamma=False):
    a, c = 4.913 * ANGSTROM, 5.404 * ANGSTROM
    cell = _hex(a, c)
    si = _apply_ops(P3121, (0.465, 0.0, 1 / 3))
    ox = _apply_ops(P3121, (0.417, 0.278, 0.222))
    rng = np.random.default_rng(seed)
    frac_si, frac_o = [], []
    for i in range(reps[0]):
        for j in range(reps[1]):
            for k in range(reps[2]):
                sh = np.array([i, j, k], float)
                frac_si += [(p + sh) / reps for p in si]
                frac_o += [(p + sh) / reps for p in ox]
    rv = cell * np.array(reps)[:, None]
    pos = np.array(frac_si + frac_o) @ rv
    pos = pos + rng.normal(0.0, jitter * ANGSTROM, size=pos.shape)
    nsi, no = len(frac_si), len(frac_o)
    tsi, to = silicon_type(element=1), oxygen_type(element=2)
    psi = _pot(1, "si1_1", 14, npot, 0.10, 1.0e5)
    po = _pot(2, "o1_1", 8, npot, 0.12, 1.0e5)
    k, km = ((np.zeros((1, 3)), None) if gamma else _mesh(kmesh, shift))
    types = [1] * nsi + [2] * no
    return _system(rv, [tsi, to], types, pos, [psi, po], types, k,
                   title=f"alpha-quartz {reps} supercell, jittered", kmesh=km)


def graphite_cell(reps=(1, 1, 1), kmesh=(2, 2, 2), shift=(0.5, 0.5, 0.5),
                  seed=4, jitter=0.0, strain=None):
    a, c = 2.46 * ANGSTROM, 6.71 * ANGSTROM
    cell = _hex(a, c)
    base = [(0, 0, 0), (0, 0, 0.5), (1 / 3, 2 / 3, 0), (2 / 3, 1 / 3, 0.5)]
    rng = np.random.default_rng(seed)
    frac = []
    for i in range(reps[0]):
        for j in range(reps[1]):
            for k in range(reps[2]):
                frac += [(np.array(p) + [i, j, k]) / reps for p in base]
    rv = cell * np.array(reps)[:, None]
    if strain is not None:
        rv = rv @ (np.eye(3) + np.asarray(strain))
    pos = np.array(frac) @ rv
    if jitter:
        pos = pos + rng.normal(0.0, jitter * ANGSTROM, size=pos.shape)
    t = carbon_type()
    p = _pot(1, "c1_1", 6, 16, 0.12, 1.0e5)
    k, km = _mesh(kmesh, shift)
    n = len(frac)
    return _system(rv, [t], [1] * n, pos, [p], [1] * n, k,
                   title="AB graphite", kmesh=km)


def cubic_supercell(element="si", reps=(1, 1, 1), kmesh=(2, 2, 2),
                    shift=(0.5, 0.5, 0.5), seed=6, jitter=0.02, strain=None):
    """Diamond-structure conventional cell (Si a=5.431 A with the s,p,d
    basis and 20 potential terms, or C a=3.567 A with the 1s/2s2p basis and
    16 terms) repeated reps times, optionally strained (rv <- rv (1 + e))
    and jittered."""
    si = element == "si"
    a = (5.431 if si else 3.567) * ANGSTROM
    rng = np.random.default_rng(seed)
    rv = np.eye(3) * a * np.array(reps)[:, None]
    if strain is not None:
        rv = rv @ (np.eye(3) + np.asarray(strain))
    frac = []
    for i in range(reps[0]):
        for j in range(reps[1]):
            for k in range(reps[2]):
                frac += [(np.array(f) + [i, j, k]) / reps for f in DIAMOND_FRAC]
    pos = np.array(frac) @ rv
    if jitter:
        pos = pos + rng.normal(0.0, jitter * ANGSTROM, size=pos.shape)
    if si:
        t, p = silicon_type(), _pot(1, "si1_1", 14, 20, 0.10, 1.0e5)
    else:
        t, p = carbon_type(), _pot(1, "c1_1", 6, 16, 0.12, 1.0e5)
    k, km = _mesh(kmesh, shift)
    n = len(frac)
    return _system(rv, [t], [1] * n, pos, [p], [1] * n, k,
                   title=f"{'silicon' if si else 'diamond'} {tuple(reps)} supercell",
                   kmesh=km)


# Supercell repetitions of the batched workload by kind (atoms in brackets):
# Si conventional 8 (8..64), diamond conventional 8 (8..216), graphite 4
# (8..216).  Si stops at 64 atoms: its 13 valence and 5 core states per atom
# make a 216-atom cell alone a second-long build.
BATCH_REPS = {
    "si": [(1, 1, 1), (2, 1, 1), (2, 2, 1), (2, 2, 2)],
    "diamond": [(1, 1, 1), (2, 1, 1), (2, 2, 1), (2, 2, 2), (3, 2, 2),
                (3, 3, 2), (3, 3, 3)],
    "graphite": [(2, 1, 1), (2, 2, 1), (2, 2, 2), (3, 3, 1), (4, 4, 1),
                 (3, 3, 2), (4, 4, 2), (6, 6, 1), (6, 3, 3)],
}


def batch_cells(n=64, seed=5, kmesh=(2, 2, 2), jitter=0.02, strain=0.03):
    """The batched multi-cell workload: n cells drawn (seeded) over Si,
    diamond and graphite supercells of BATCH_REPS, each with its own
    symmetric strain (components uniform in +-strain, off-diagonal halved)
    and jitter."""
    rng = np.random.default_rng(seed)
    kinds = ["si", "diamond", "graphite"]
    cells = []
    for i in range(n):
        kind = kinds[int(rng.integers(3))]
        reps = BATCH_REPS[kind][int(rng.integers(len(BATCH_REPS[kind])))]
        e = rng.uniform(-strain, strain, size=(3, 3))
        e = np.diag(np.diag(e)) + 0.25 * (np.triu(e, 1) + np.triu(e, 1).T)
        cseed = int(rng.integers(1 << 30))
        if kind == "graphite":
            cells.append(graphite_cell(reps=reps, kmesh=kmesh, seed=cseed,
                                       jitter=jitter, strain=e))
        else:
            cells.append(cubic_supercell(kind, reps=reps, kmesh=kmesh,
                                         seed=cseed, jitter=jitter, strain=e))
    return cells


def small_test_system(seed=7, kmesh=(2, 2, 1)):
    """A two-element, four-atom cell with every class up to d-p, small
    enough for the CPU oracle in seconds."""
    a = 6.0
    rng = np.random.default_rng(seed)
    rv = np.array([[a, 0.3, 0.0], [0.2, a * 0.9, 0.1], [0.0, 0.4, a * 1.1]])
    frac = np.array([[0.05, 0.1, 0.0], [0.45, 0.55, 0.5], [0.3, 0.2, 0.7],
                     [0.8, 0.6, 0.25]])
    pos = frac @ rv + rng.normal(0, 0.05, size=(4, 3))
    tsi = silicon_type(element=1, nprim=8, amin=0.15, amax=2.0e3, nd=5)
    to = oxygen_type(element=2, nprim=7, amin=0.2, amax=1.0e3)
    psi = _pot(1, "si1_1", 14, 4, 0.15, 1.0e3)
    po = _pot(2, "o1_1", 8, 3, 0.2, 1.0e3)
    types = [1, 2, 2, 1]
    pot_site_type = [1, 1, 2, 2]
    order = [0, 3, 1, 2]  # pot sites grouped by type
    k, km = _mesh(kmesh, (0.5, 0.5, 0.0))
    sys_ = ImagoSystem(real_vectors=rv, atom_types=[tsi, to],
                       site_type=np.array(types, np.int32), site_pos=pos,
                       pot_types=[psi, po],
                       pot_site_type=np.array(pot_site_type, np.int32),
                       pot_site_pos=pos[order], kpoints_abc=k,
                       basis_fn_convg=1e-16, electro_convg=1e-16,
                       title="small two-element test cell", kmesh=km)
    sys_.validate()
    return sys_


def no_core_test_system(kmesh=(2, 2, 2)):
    """Three atoms of a valence-only element (coreDim = 0): the reference
    packs valeVale without orthogonalisation and without the 1e-10 zeroing
    (integrals.F90:3657-3676)."""
    a = 6.5
    rv = np.array([[a, 0.0, 0.2], [0.4, a * 1.1, 0.0], [0.0, 0.3, a * 0.9]])
    pos = np.array([[0.2, 0.1, 0.0], [2.3, 1.9, 1.1], [4.4, 0.5, 3.9]])
    alphas = even_tempered(8, 0.2, 5.0e2)
    t = _make_type(1, "v1_1", alphas, (8, 8, 5, 0), [],
                   [(1, 0, 1.3), (2, 1, 1.1), (3, 2, 0.9)])
    p = _pot(1, "v1_1", 3, 4, 0.2, 1.0e3)
    k, km = _mesh(kmesh, (0.5, 0.5, 0.5))
    return _system(rv, [t], [1, 1, 1], pos, [p], [1, 1, 1], k,
                   title="valence-only test cell", kmesh=km)


def f_test_system(kmesh=(2, 1, 1)):
    """Two atoms of one element with s, p, d and f functions, so every class
    up to f-f appears; small enough for the CPU oracle."""
    a = 7.0
    rv = np.array([[a, 0.0, 0.0], [0.5, a, 0.0], [0.0, 0.3, a]])
    pos = np.array([[0.1, 0.2, 0.3], [2.1, 1.7, 2.6]])
    alphas = even_tempered(6, 0.3, 3.0e2)
    t = _make_type(1, "x1_1", alphas, (6, 6, 5, 4), [(1, 0, 6.0)],
                   [(2, 0, 1.6), (2, 1, 1.5), (3, 2, 1.2), (4, 3, 1.0)])
    p = _pot(1, "x1_1", 10, 3, 0.3, 1.0e3)
    k, km = _mesh(kmesh, (0.5, 0.0, 0.0))
    return _system(rv, [t], [1, 1], pos, [p], [1, 1], k,
                   title="f-class test pair", kmesh=km)
