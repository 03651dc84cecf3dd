"""Host-side description of an Imago system and its C-ABI mirror.

`ImagoSystem` holds the module data that Imago's setupSCF has read before
the integral calls (src/imago/imago.F90:185-258): atom types with their
radial functions (atomicTypes.f90:132-361), atom sites (atomicSites.f90),
potential types and sites (potTypes.f90, potSites.f90), the cell
(lattice.f90 CELL_VECTORS), the k-points (kpoints.f90) and the basis
function cutoff (input.f90:327-346).  `to_c()` packs it into the
`imago_system` struct of include/imago_intg.h.
"""

import ctypes
from dataclasses import dataclass, field
from typing import List

import numpy as np


@dataclass
class AtomType:
    element: int                 # elementID, 1-based
    label: str
    num_orb_alphas: List[int]    # NUM_ALPHA_S_P_D_F
    alphas: np.ndarray           # numOrbAlphas[0] values, ascending
    core_l: List[int] = field(default_factory=list)
    core_coeffs: List[np.ndarray] = field(default_factory=list)
    vale_l: List[int] = field(default_factory=list)
    vale_coeffs: List[np.ndarray] = field(default_factory=list)
    core_n: List[int] = field(default_factory=list)
    vale_n: List[int] = field(default_factory=list)

    @property
    def num_core_states(self):
        return sum(2 * l + 1 for l in self.core_l)

    @property
    def num_vale_states(self):
        return sum(2 * l + 1 for l in self.vale_l)


@dataclass
class PotType:
    element: int
    label: str
    nuc_charge: float
    nuc_alpha: float
    alphas: np.ndarray           # ascending
    covalent_radius: float = 1.0
    coeffs: np.ndarray = None    # starting potential coefficients (fort.8)


@dataclass
class ImagoSystem:
    real_vectors: np.ndarray     # (3 abc, 3 xyz) rows are a, b, c in bohr
    atom_types: List[AtomType]
    site_type: np.ndarray        # 1-based type per atom site
    site_pos: np.ndarray         # (nSites, 3) bohr
    pot_types: List[PotType]
    pot_site_type: np.ndarray    # 1-based
    pot_site_pos: np.ndarray     # (nPotSites, 3)
    kpoints_abc: np.ndarray      # (nk, 3) fractional reciprocal coordinates
    basis_fn_convg: float = 1e-16
    electro_convg: float = 1e-16
    title: str = "imago-b200 system"
    kmesh: tuple = None          # (n, shift) when the k-points are a mesh

    @property
    def vale_dim(self):
        return int(sum(self.atom_types[t - 1].num_vale_states
                       for t in self.site_type))

    @property
    def core_dim(self):
        return int(sum(self.atom_types[t - 1].num_core_states
                       for t in self.site_type))

    @property
    def pot_dim(self):
        return int(sum(len(p.alphas) for p in self.pot_types))

    @property
    def num_kpoints(self):
        return int(len(self.kpoints_abc))

    def validate(self):
        """Checks the reference makes while reading the decks."""
        for t in self.atom_types:
            n = t.num_orb_alphas
            if any(n[i] < n[i + 1] for i in range(3)):
                raise ValueError("Num of alphas not monotonically decreasing.")
            if len(t.alphas) != n[0]:
                raise ValueError("ALPHAS count differs from NUM_ALPHA_S_P_D_F")
            for l, c in zip(t.core_l + t.vale_l, t.core_coeffs + t.vale_coeffs):
                if len(c) != n[l]:
                    raise ValueError("radial function length differs from "
                                     "numOrbAlphas(l+1)")
        pt = np.asarray(self.pot_site_type)
        if np.any(np.diff(pt) < 0):
            raise ValueError("potential sites must be grouped by type in "
                             "ascending order")

    def to_c(self):
        """Return (imago_system struct, keep-alive list)."""
        keep = []

        def arr(a, ctype):
            if ctype is ctypes.c_double:
                x = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())
            else:
                x = np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel())
            keep.append(x)
            return x.ctypes.data_as(ctypes.POINTER(ctype))

        s = ImagoSystemC()
        rv = np.asarray(self.real_vectors, dtype=np.float64)
        for abc in range(3):
            for xyz in range(3):
                s.real_vectors[3 * abc + xyz] = rv[abc, xyz]
        s.basis_fn_convg = self.basis_fn_convg
        s.electro_convg = self.electro_convg
        ts = self.atom_types
        s.num_atom_types = len(ts)
        s.type_element = arr([t.element for t in ts], ctypes.c_int)
        s.type_num_orb_alphas = arr([list(t.num_orb_alphas) for t in ts],
                                    ctypes.c_int)
        s.type_alphas = arr(np.concatenate([np.asarray(t.alphas, float)
                                            for t in ts]), ctypes.c_double)
        s.type_num_core_fns = arr([len(t.core_l) for t in ts], ctypes.c_int)
        s.type_num_vale_fns = arr([len(t.vale_l) for t in ts], ctypes.c_int)
        fl, fc = [], []
        for t in ts:
            fl += list(t.core_l) + list(t.vale_l)
            fc += [np.asarray(c, float) for c in t.core_coeffs + t.vale_coeffs]
        s.fn_l = arr(fl, ctypes.c_int)
        s.fn_coeffs = arr(np.concatenate(fc) if fc else [0.0], ctypes.c_double)
        s.num_atom_sites = len(self.site_type)
        s.site_type = arr(self.site_type, ctypes.c_int)
        s.site_pos = arr(self.site_pos, ctypes.c_double)
        ps = self.pot_types
        s.num_pot_types = len(ps)
        s.pot_type_element = arr([p.element for p in ps], ctypes.c_int)
        s.pot_type_nuc_charge = arr([p.nuc_charge for p in ps], ctypes.c_double)
        s.pot_type_nuc_alpha = arr([p.nuc_alpha for p in ps], ctypes.c_double)
        s.pot_type_num_alphas = arr([len(p.alphas) for p in ps], ctypes.c_int)
        s.pot_type_alphas = arr(np.concatenate([np.asarray(p.alphas, float)
                                                for p in ps]), ctypes.c_double)
        s.num_pot_sites = len(self.pot_site_type)
        s.pot_site_type = arr(self.pot_site_type, ctypes.c_int)
        s.pot_site_pos = arr(self.pot_site_pos, ctypes.c_double)
        s.num_kpoints = len(self.kpoints_abc)
        s.kpoints_abc = arr(self.kpoints_abc, ctypes.c_double)
        return s, keep


class ImagoSystemC(ctypes.Structure):
    """Mirror of `imago_system` in include/imago_intg.h."""
    _fields_ = [
        ("real_vectors", ctypes.c_double * 9),
        ("basis_fn_convg", ctypes.c_double),
        ("electro_convg", ctypes.c_double),
        ("num_atom_types", ctypes.c_int),
        ("type_element", ctypes.POINTER(ctypes.c_int)),
        ("type_num_orb_alphas", ctypes.POINTER(ctypes.c_int)),
        ("type_alphas", ctypes.POINTER(ctypes.c_double)),
        ("type_num_core_fns", ctypes.POINTER(ctypes.c_int)),
        ("type_num_vale_fns", ctypes.POINTER(ctypes.c_int)),
        ("fn_l", ctypes.POINTER(ctypes.c_int)),
        ("fn_coeffs", ctypes.POINTER(ctypes.c_double)),
        ("num_atom_sites", ctypes.c_int),
        ("site_type", ctypes.POINTER(ctypes.c_int)),
        ("site_pos", ctypes.POINTER(ctypes.c_double)),
        ("num_pot_types", ctypes.c_int),
        ("pot_type_element", ctypes.POINTER(ctypes.c_int)),
        ("pot_type_nuc_charge", ctypes.POINTER(ctypes.c_double)),
        ("pot_type_nuc_alpha", ctypes.POINTER(ctypes.c_double)),
        ("pot_type_num_alphas", ctypes.POINTER(ctypes.c_int)),
        ("pot_type_alphas", ctypes.POINTER(ctypes.c_double)),
        ("num_pot_sites", ctypes.c_int),
        ("pot_site_type", ctypes.POINTER(ctypes.c_int)),
        ("pot_site_pos", ctypes.POINTER(ctypes.c_double)),
        ("num_kpoints", ctypes.c_int),
        ("kpoints_abc", ctypes.POINTER(ctypes.c_double)),
    ]


class ImagoDimsC(ctypes.Structure):
    """Mirror of `imago_dims`."""
    _fields_ = [
        ("vale_dim", ctypes.c_int),
        ("core_dim", ctypes.c_int),
        ("num_kpoints", ctypes.c_int),
        ("pot_dim", ctypes.c_int),
        ("num_cells", ctypes.c_int),
        ("packed", ctypes.c_longlong),
        ("num_pair_images", ctypes.c_longlong),
        ("num_shell_pairs", ctypes.c_longlong),
        ("block_elements", ctypes.c_longlong),
    ]


def kpoint_mesh(n, shift=(0.0, 0.0, 0.0)):
    """Fractional k-point mesh of kpoints.f90:896-899 (no symmetry folding):
    k_abc = -1/2 + (i - 1 + shift)/n, a-major loop order."""
    n = [int(x) for x in n]
    pts = []
    for i in range(1, n[0] + 1):
        for j in range(1, n[1] + 1):
            for k in range(1, n[2] + 1):
                idx = (i, j, k)
                pts.append([-0.5 + (idx[a] - 1.0 + shift[a]) * (1.0 / n[a])
                            for a in range(3)])
    return np.array(pts, dtype=np.float64)


def pot_alphas(num, amin, amax):
    """makePotAlphas (potTypes.f90:170-195): geometric series
    alphas(i) = min * ((max/min)**(1/(n-1)))**(i-1), the integer power taken
    by repeated multiplication as gfortran does for a variable exponent."""
    r = (amax / amin) ** (1.0 / float(num - 1))
    out = []
    for i in range(1, num + 1):
        e = i - 1
        p, b = 1.0, r
        while e:  # square-and-multiply
            if e & 1:
                p *= b
            b *= b
            e >>= 1
        out.append(amin * p)
    return np.array(out)
