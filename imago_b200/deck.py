"""Read and write the parts of Imago's input decks the integral setup uses.

Imago reads three text decks (src/imago/input.f90:139-240):

* fort.5 (imago.dat): TITLE, the atom types with their contracted radial
  functions (atomicTypes.f90:132-361), the potential types
  (potTypes.f90:86-169), then control sections; of those the integral setup
  needs BASISFUNCTION_AND_ELECTROSTATIC_CUTOFFS (input.f90:327-346);
* fort.4 (structure.dat): CELL_VECTORS (bohr), the atom sites and the
  potential sites (atomicSites.f90:85-132, potSites.f90:40-86);
* fort.15 (kp-scf.dat): KPOINT_STYLE_CODE 0 (explicit list) or 1 (mesh;
  only the identity point operation is supported here, the P1 case),
  kpoints.f90:195-440.

Values follow Fortran list-directed input: a read starts on a new record,
takes as many records as it needs, and ignores the rest of its last record.
Reading tolerates the control sections it does not use; writing emits the
sections above (a deck for the reference needs the control sections too,
which makeinput.py writes).
"""

import os

import numpy as np

from .system import AtomType, ImagoSystem, PotType, pot_alphas


class DeckError(ValueError):
    pass


class _Records:
    """Fortran list-directed reads over a text file."""

    def __init__(self, path):
        with open(path) as fh:
            self.lines = [ln.rstrip("\n") for ln in fh]
        self.pos = 0
        self.path = path

    def _next_line(self):
        if self.pos >= len(self.lines):
            raise DeckError(f"{self.path}: unexpected end of file")
        ln = self.lines[self.pos]
        self.pos += 1
        return ln

    def label(self, expect):
        """readAndCheckLabel: the first token of the next record."""
        ln = self._next_line()
        got = ln.split()[0] if ln.split() else ""
        if got[:len(expect)] != expect:
            raise DeckError(f"{self.path}: {expect} label not found (line "
                            f"{self.pos}: {ln!r})")

    def values(self, n, conv=float):
        out = []
        while len(out) < n:
            toks = self._next_line().replace(",", " ").split()
            out += toks
        return [conv(_fortran_real(t)) if conv is float else conv(t)
                for t in out[:n]]

    def line(self):
        return self._next_line()

    def seek_label(self, label):
        while self.pos < len(self.lines):
            toks = self.lines[self.pos].split()
            if toks and toks[0] == label:
                return True
            self.pos += 1
        return False


def _fortran_real(t):
    return t.replace("d", "e").replace("D", "E")


def _read_radial_fns(r, num_fns, norb, basis_code):
    ls, ns, coeffs = [], [], []
    if num_fns == 0:
        return ls, ns, coeffs
    r.label("NL_RADIAL_FUNCTIONS")
    for _ in range(num_fns):
        ids = r.values(2, int)
        comp = r.values(5, int)
        n, l = comp[0], comp[1]
        c = r.values(norb[l])
        if ids[1] <= basis_code:
            ls.append(l)
            ns.append(n)
            coeffs.append(np.array(c))
    return ls, ns, coeffs


def read_decks(directory, basis_code=2, fort5="fort.5", fort4="fort.4",
               fort15="fort.15"):
    """Read the integral-setup inputs of an Imago run directory into an
    ImagoSystem.  basis_code: 1 MB, 2 FB, 3 EB (commandLine.f90)."""
    r = _Records(os.path.join(directory, fort5))
    r.label("TITLE")
    title = []
    while True:
        ln = r.line()
        if ln.strip().startswith("END_TITLE"):
            break
        title.append(ln)
    r.label("NUM_ATOM_TYPES")
    ntypes = r.values(1, int)[0]
    types = []
    for i in range(ntypes):
        r.label("ATOM_TYPE_ID__SEQUENTIAL_NUMBER")
        ids = r.values(4, int)
        if ids[3] != i + 1:
            raise DeckError("Types numbered out of order")
        r.label("ATOM_TYPE_LABEL")
        label = r.line().strip()
        r.label("NUM_ALPHA_S_P_D_F")
        norb = r.values(4, int)
        if any(norb[j] < norb[j + 1] for j in range(3)):
            raise DeckError("Num of alphas not monotonically decreasing.")
        r.label("ALPHAS")
        alphas = np.array(r.values(norb[0]))
        r.label("NUM_CORE_RADIAL_FNS")
        ncore = r.values(3, int)
        cl, cn, cc = _read_radial_fns(r, ncore[2], norb, basis_code)
        r.label("NUM_VALE_RADIAL_FNS")
        nvale = r.values(3, int)
        vl, vn, vc = _read_radial_fns(r, nvale[2], norb, basis_code)
        types.append(AtomType(element=ids[0], label=label, num_orb_alphas=norb,
                              alphas=alphas, core_l=cl, core_coeffs=cc,
                              vale_l=vl, vale_coeffs=vc, core_n=cn, vale_n=vn))
    r.label("NUM_POTENTIAL_TYPES")
    npt = r.values(1, int)[0]
    pots = []
    for i in range(npt):
        r.label("POTENTIAL_TYPE_ID__SEQUENTIAL_NUMBER")
        ids = r.values(4, int)
        if ids[3] != i + 1:
            raise DeckError("Types numbered out of order")
        r.label("POTENTIAL_TYPE_LABEL")
        label = r.line().strip()
        r.label("NUCLEAR_CHARGE__ALPHA")
        z, nuc = r.values(2)
        r.label("COVALENT_RADIUS")
        cov = r.values(1)[0]
        r.label("NUM_ALPHAS")
        na = r.values(1, int)[0]
        r.label("ALPHAS")
        amin, amax = r.values(2)
        pots.append(PotType(element=ids[0], label=label, nuc_charge=z,
                            nuc_alpha=nuc, alphas=pot_alphas(na, amin, amax),
                            covalent_radius=cov))
    if not r.seek_label("SHARED_INPUT_DATA"):
        raise DeckError("SHARED_INPUT_DATA label not found.")
    r.label("SHARED_INPUT_DATA")
    r.label("SPACE_GROUP")
    r.values(2, int)
    r.label("BASISFUNCTION_AND_ELECTROSTATIC_CUTOFFS")
    bf, es = r.values(2)
    if not (0.0 < bf <= 1.0) or not (0.0 < es <= 1.0):
        raise DeckError("Wave Fn Convergence value is not in (0,1]")

    s = _Records(os.path.join(directory, fort4))
    s.label("CELL_VECTORS")
    rv = np.array([s.values(3) for _ in range(3)])
    s.label("NUM_ATOM_SITES")
    nsites = s.values(1, int)[0]
    s.label("NUM_TYPE_X_Y_Z_ELEM")
    st, sp = [], []
    for i in range(nsites):
        toks = s.line().split()
        if int(toks[0]) != i + 1:
            raise DeckError(f"Atom site list is out of order at i = {i + 1}")
        st.append(int(toks[1]))
        sp.append([float(_fortran_real(x)) for x in toks[2:5]])
    s.label("NUM_POTENTIAL_SITES")
    npsites = s.values(1, int)[0]
    s.label("NUM_TYPE_X_Y_Z_ELEM")
    pst, psp = [], []
    for i in range(npsites):
        toks = s.line().split()
        if int(toks[0]) != i + 1:
            raise DeckError(f"Potential site list is out of order at i = {i + 1}")
        pst.append(int(toks[1]))
        psp.append([float(_fortran_real(x)) for x in toks[2:5]])

    k = _Records(os.path.join(directory, fort15))
    k.label("KPOINT_STYLE_CODE")
    style = k.values(1, int)[0]
    k.label("KPOINT_INTG_CODE")
    k.values(1, int)
    kmesh = None
    if style == 0:
        k.label("NUM_BLOCH_VECTORS")
        nk = k.values(1, int)[0]
        k.label("NUM_AXIAL_KPOINTS")
        k.values(3, int)
        k.label("NUM_WEIGHT_KA_KB_KC")
        kp = []
        for _ in range(nk):
            v = k.values(5)
            kp.append(v[2:5])
        kpts = np.array(kp)
    elif style == 1:
        k.label("NUM_KP_A_B_C")
        n = k.values(3, int)
        k.label("KP_SHIFT_A_B_C")
        shift = k.values(3)
        k.label("NUM_POINT_OPS")
        nops = k.values(1, int)[0]
        if nops != 1:
            raise DeckError("only the identity point operation (P1) is "
                            "supported for KPOINT_STYLE_CODE 1")
        from .system import kpoint_mesh
        kpts = kpoint_mesh(n, shift)
        kmesh = (tuple(n), tuple(shift))
    else:
        raise DeckError(f"KPOINT_STYLE_CODE {style} is not supported")
    sys_ = ImagoSystem(real_vectors=rv, atom_types=types,
                       site_type=np.array(st, np.int32), site_pos=np.array(sp),
                       pot_types=pots, pot_site_type=np.array(pst, np.int32),
                       pot_site_pos=np.array(psp), kpoints_abc=kpts,
                       basis_fn_convg=bf, electro_convg=es,
                       title="\n".join(title), kmesh=kmesh)
    sys_.validate()
    return sys_


def _fmt(vals, per=4, f=" {:.16e}"):
    out = []
    for i in range(0, len(vals), per):
        out.append("".join(f.format(v) for v in vals[i:i + per]))
    return "\n".join(out) + "\n"


def write_decks(system, directory, kpoint_style=None):
    """Write fort.5 (integral-setup sections), fort.4 and fort.15 for
    `system` in the reference's formats."""
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, "fort.5"), "w") as f:
        f.write("TITLE\n" + system.title + "\nEND_TITLE\n")
        f.write(f"NUM_ATOM_TYPES\n{len(system.atom_types)}\n")
        for i, t in enumerate(system.atom_types):
            f.write("ATOM_TYPE_ID__SEQUENTIAL_NUMBER\n")
            f.write(f"{t.element:<5d} 1     {i + 1:<5d}     {i + 1}\n")
            f.write(f"ATOM_TYPE_LABEL\n{t.label}\n")
            f.write("NUM_ALPHA_S_P_D_F\n" + " ".join(str(x) for x in t.num_orb_alphas) + "\n")
            f.write("ALPHAS\n" + _fmt(list(t.alphas)))
            for kind, ls, ns, cs in (("CORE", t.core_l, t.core_n, t.core_coeffs),
                                     ("VALE", t.vale_l, t.vale_n, t.vale_coeffs)):
                n = len(ls)
                f.write(f"NUM_{kind}_RADIAL_FNS\n{n} {n} {n}\n")
                if n == 0 and kind == "CORE":
                    continue
                f.write("NL_RADIAL_FUNCTIONS\n")
                for l, nq, c in zip(ls, ns or [l + 1] * n, cs):
                    f.write("1 1\n")
                    f.write(f"{nq} {l} {2 * l} {2 * (2 * l + 1)} 1\n")
                    f.write(_fmt(list(c)))
        f.write(f"NUM_POTENTIAL_TYPES\n{len(system.pot_types)}\n")
        for i, p in enumerate(system.pot_types):
            f.write("POTENTIAL_TYPE_ID__SEQUENTIAL_NUMBER\n")
            f.write(f"{p.element:<5d} 1     {i + 1:<5d}     {i + 1}\n")
            f.write(f"POTENTIAL_TYPE_LABEL\n{p.label}\n")
            f.write(f"NUCLEAR_CHARGE__ALPHA\n{p.nuc_charge:.10f} {p.nuc_alpha:.10f}\n")
            f.write(f"COVALENT_RADIUS\n{p.covalent_radius:.10f}\n")
            f.write(f"NUM_ALPHAS\n{len(p.alphas)}\n")
            f.write(f"ALPHAS\n{p.alphas[0]:.17e} {p.alphas[-1]:.17e}\n")
        f.write("SHARED_INPUT_DATA\nSPACE_GROUP\n1 1\n")
        f.write("BASISFUNCTION_AND_ELECTROSTATIC_CUTOFFS\n")
        f.write(f"{system.basis_fn_convg:.8e} {system.electro_convg:.8e}\n")
    with open(os.path.join(directory, "fort.4"), "w") as f:
        f.write("CELL_VECTORS\n")
        for abc in range(3):
            f.write("".join(f"{v:26.18f}" for v in system.real_vectors[abc]) + "\n")
        for kind, types, pos in (("ATOM", system.site_type, system.site_pos),
                                 ("POTENTIAL", system.pot_site_type,
                                  system.pot_site_pos)):
            f.write(f"NUM_{kind}_SITES\n{len(types):<5d}\nNUM_TYPE_X_Y_Z_ELEM\n")
            for i, (t, p) in enumerate(zip(types, pos)):
                f.write(f"{i + 1:5d} {int(t):5d} {p[0]:26.18f} {p[1]:26.18f} "
                        f"{p[2]:26.18f} xx\n")
    style = kpoint_style if kpoint_style is not None else (1 if system.kmesh else 0)
    with open(os.path.join(directory, "fort.15"), "w") as f:
        f.write(f"KPOINT_STYLE_CODE\n{style}\nKPOINT_INTG_CODE\n0\n")
        if style == 1:
            n, shift = system.kmesh
            f.write("NUM_KP_A_B_C\n" + " ".join(str(x) for x in n) + "\n")
            f.write("KP_SHIFT_A_B_C\n" + " ".join(f"{x:.17g}" for x in shift) + "\n")
            f.write("NUM_POINT_OPS\n1\nPOINT_OPS\n1 0 0\n0 1 0\n0 0 1\n0 0 0\n")
            f.write("CONV_LATTICE\n1 0 0\n0 1 0\n0 0 1\nCELL_MODE\nfull\n")
        else:
            nk = len(system.kpoints_abc)
            f.write(f"NUM_BLOCH_VECTORS\n{nk}\nNUM_AXIAL_KPOINTS\n1 1 1\n")
            f.write("NUM_WEIGHT_KA_KB_KC\n")
            w = 2.0 / nk
            for i, kp in enumerate(system.kpoints_abc):
                f.write(f"{i + 1} {w:.17g} {kp[0]:.17g} {kp[1]:.17g} {kp[2]:.17g}\n")
