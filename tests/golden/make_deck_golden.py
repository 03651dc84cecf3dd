"""Decks written by the reference's own makeinput.py, for the deck reader.

The reference's input generator (src/scripts/makeinput.py) is Python, so its
writer functions run here as they stand:

  _print_imago_input   imago.dat (fort.5): title, the atom types (each type's
                       contracted basis file copied in, its state counts
                       parsed back), the potential types from the potential
                       database (src/data/atomicPDB.tgz, pot1/coeff1), the
                       exchange-correlation mesh, NUM_STATES_TO_USE and
                       NUM_ELECTRONS as the generator counts them, the
                       cutoffs and every control section; also scfV.dat
  _print_structure     structure.dat (fort.4)
  _write_mesh_kp_file  kp-scf.dat (fort.15), KPOINT_STYLE_CODE 1

Supplied here: the generator's settings and structure objects (plain
namespaces holding the values its command line and skeleton file would
give; the numeric controls that do not bear on the integral setup are left
at 0), and the contracted basis files, whose database (atomicBDB) is not in
the reference mount: they are written in the layout the generator parses,
from the synthetic two-element cell of imago_b200.configs.

Fixtures: tests/golden/decks/ (fort.5, fort.4, fort.15, scfV.dat) and
tests/golden/decks/expected.json (what the generator was given).

Run where the reference is mounted:

    python tests/golden/make_deck_golden.py <root of the reference checkout>
"""
import json
import os
import shutil
import sys
import tarfile
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from imago_b200 import configs, deck  # noqa: E402

ELEMENTS = ("si", "o")


class Settings:
    """The generator's ScriptSettings: the values given, 0 for the rest."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return 0


def _basis_files(system, work):
    """Each atom type's section of a deck written by imago_b200.deck, from
    NUM_ALPHA_S_P_D_F to the end of its valence functions: the contracted
    basis file layout (the generator copies the file after the type's
    label and parses its state counts from it)."""
    tmp = os.path.join(work, "ours")
    deck.write_decks(system, tmp)
    lines = open(os.path.join(tmp, "fort.5")).read().split("\n")
    out, cur = [], None
    for ln in lines:
        if ln.startswith("NUM_ALPHA_S_P_D_F"):
            cur = [ln]
            out.append(cur)
        elif ln.startswith("ATOM_TYPE_ID") or ln.startswith("NUM_POTENTIAL_TYPES"):
            cur = None
        elif cur is not None:
            cur.append(ln)
    return ["\n".join(c) + "\n" for c in out]


def main(ref):
    sys.path.insert(0, os.path.join(ref, "src", "scripts"))
    import makeinput as mi

    s = configs.small_test_system()
    assert [t.label for t in s.atom_types] == ["si1_1", "o1_1"]
    work = tempfile.mkdtemp()
    cwd = os.getcwd()
    try:
        basis = _basis_files(s, work)
        os.chdir(work)
        os.makedirs(mi.INPUT_TEMP)
        os.makedirs(mi.INPUTS_DIR)
        with tarfile.open(os.path.join(ref, "src", "data", "sybdDB.tgz")) as tf:
            data = tf.extractfile("sybdDB/tric1a").read()
        os.makedirs("sybdDB")
        with open(os.path.join("sybdDB", "tric1a"), "wb") as fh:
            fh.write(data)
        with tarfile.open(os.path.join(ref, "src", "data", "atomicPDB.tgz")) as tf:
            for el in ELEMENTS:
                for f in ("pot1", "coeff1"):
                    data = tf.extractfile(f"atomicPDB/{el}/{f}").read()
                    with open(os.path.join(mi.INPUT_TEMP, f"{el}_{f}"), "wb") as fh:
                        fh.write(data)
        for el, text in zip(ELEMENTS, basis):
            with open(os.path.join(mi.INPUT_TEMP, f"{el}_basis"), "w") as fh:
                fh.write(text)

        natoms = len(s.site_type)
        count = [None] + [int(np.sum(s.site_type == t + 1)) for t in range(2)]
        settings = Settings(
            num_elements=2, num_species=[None, 1, 1],
            num_types=[[None, [None, 1], [None, 1]]],
            element_list=[None, "si", "o"],
            basis_files=[None, [None, "si_basis"], [None, "o_basis"]],
            pot_files=[None, [None, "si_pot1"], [None, "o_pot1"]],
            coeff_files=[None, [None, "si_coeff1"], [None, "o_coeff1"]],
            max_num_atom_alphas=0, xanes=0, mod_element_name="", mod_pot=0,
            num_samp_vectors=100, xc_in_weight=0.5, xc_out_weight=0.5,
            xc_in_samp=0.1, xc_out_samp=3.5, xc_spacing_samp=0.8,
            space_group_num=1, space_group_sub_num=1, bf_cutoff=16, es_cutoff=16,
            state_factor=1.0, num_atoms=natoms, xc_code=100, num_iter_main=50,
            converg_main=0.0001, spin_main=1, kp_mesh_pscf=[None, 1, 1, 1],
            sybd_db="sybdDB", sybd_path="tric1a", print_bz=0)
        rv = np.asarray(s.real_vectors)
        mag = [float(np.linalg.norm(rv[a])) for a in range(3)]
        ang = [float(np.arccos(rv[b] @ rv[c] / (mag[b] * mag[c])))
               for b, c in ((1, 2), (0, 2), (0, 1))]
        sc = types.SimpleNamespace(
            system_title=[None, "two-element", "test", "cell"],
            real_lattice=[None] + [[None] + list(rv[a]) for a in range(3)],
            full_cell_mag=[None] + mag, full_cell_angle=[None] + ang)
        # the generator sorts the atoms by element before writing (its
        # sorted_* arrays); here the same order, stable within an element
        order = np.argsort(s.site_type, kind="stable")
        st, sp = np.asarray(s.site_type)[order], np.asarray(s.site_pos)[order]
        elem = [None] + [int(t) for t in st]
        ones = [None] + [1] * natoms
        xyz = [None] + [[None] + list(p) for p in sp]
        cum = [None, [None, 0], [None, 1]]
        mi._print_imago_input(settings, sc, 0, elem, ones, ones, [0], cum, 2, count)
        mi._print_structure(settings, sc, 0, elem, ones, ones, xyz, cum, 2)
        eye = [[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]]
        conv = [None] + [[None] + list(rv[a]) for a in range(3)]
        mi._write_mesh_kp_file(os.path.join(mi.INPUTS_DIR, "kp-scf.dat"), [None, 2, 2, 2],
                               "0.5 0.5 0.5", [eye], [[0.0, 0.0, 0.0]], conv, "full", 0)
        dst = os.path.join(HERE, "decks")
        os.makedirs(dst, exist_ok=True)
        for src, name in ((mi.IMAGO_DAT, "fort.5"), (mi.STRUCTURE, "fort.4"),
                          ("kp-scf.dat", "fort.15"), (mi.POTENTIAL, "scfV.dat")):
            shutil.copy(os.path.join(mi.INPUTS_DIR, src), os.path.join(dst, name))
        with open(os.path.join(dst, "expected.json"), "w") as fh:
            json.dump({"site_type": [int(x) for x in st], "site_pos": sp.tolist(),
                       "real_vectors": rv.tolist(), "kmesh": [2, 2, 2],
                       "kshift": [0.5, 0.5, 0.5]}, fh, indent=1)
    finally:
        os.chdir(cwd)
        shutil.rmtree(work, ignore_errors=True)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_deck_golden.py <root of the reference checkout>")
    main(sys.argv[1])
