"""The deck reader (imago_b200/deck.py) against decks written by the
reference's own input generator: tests/golden/make_deck_golden.py ran
makeinput.py's _print_imago_input, _print_structure and _write_mesh_kp_file
(src/scripts/makeinput.py:5215-5505, 5148-5212, 3961-4066) with the
potential database entries of Si and O (src/data/atomicPDB.tgz) and the
two-element test cell's atom types, and committed what they wrote."""
import json
import os

import numpy as np

from conftest import ROOT
from imago_b200 import configs, deck, scf
from imago_b200.system import kpoint_mesh

DECKS = os.path.join(ROOT, "tests", "golden", "decks")


def _read():
    return deck.read_decks(DECKS)


def _label_value(name, n=1):
    lines = open(os.path.join(DECKS, "fort.5")).read().split("\n")
    i = next(k for k, ln in enumerate(lines) if ln.startswith(name))
    return lines[i + 1].split()[:n]


def test_atom_types_are_the_basis_files_the_generator_copied():
    s, ref = _read(), configs.small_test_system()
    assert len(s.atom_types) == len(ref.atom_types)
    for a, b in zip(s.atom_types, ref.atom_types):
        assert a.label == b.label and list(a.num_orb_alphas) == list(b.num_orb_alphas)
        assert np.allclose(a.alphas, b.alphas, rtol=1e-15, atol=0)
        assert list(a.core_l) == list(b.core_l) and list(a.vale_l) == list(b.vale_l)
        for x, y in zip(a.core_coeffs + a.vale_coeffs, b.core_coeffs + b.vale_coeffs):
            assert np.allclose(x, y, rtol=1e-15, atol=0)


def test_potential_types_from_the_database():
    # the database's even-tempered exponents: the reader's alphas (from
    # NUM_ALPHAS and the ALPHAS range) equal the exponents the database's
    # coefficient files list, which the generator copied into scfV.dat
    s = _read()
    assert [p.nuc_charge for p in s.pot_types] == [14.0, 8.0]
    lines = open(os.path.join(DECKS, "scfV.dat")).read().split("\n")
    i = lines.index(" TOTAL__OR__SPIN_UP") + 1
    for p in s.pot_types:
        n = int(lines[i])
        listed = np.array([float(lines[i + 1 + j].split()[1]) for j in range(n)])
        assert n == len(p.alphas)
        assert np.allclose(p.alphas, listed, rtol=5e-10, atol=0)
        i += n + 1


def test_structure_and_kpoints():
    s = _read()
    exp = json.load(open(os.path.join(DECKS, "expected.json")))
    assert np.abs(s.real_vectors - np.array(exp["real_vectors"])).max() < 1e-14
    assert list(s.site_type) == exp["site_type"]
    assert np.abs(s.site_pos - np.array(exp["site_pos"])).max() < 1e-13
    # makeinput writes the potential sites as the atom sites
    assert list(s.pot_site_type) == exp["site_type"]
    assert np.array_equal(s.pot_site_pos, s.site_pos)
    assert s.kmesh == (tuple(exp["kmesh"]), tuple(exp["kshift"]))
    assert np.array_equal(s.kpoints_abc, kpoint_mesh(exp["kmesh"], exp["kshift"]))
    assert s.basis_fn_convg == 1e-16 and s.electro_convg == 1e-16


def test_electron_count_agrees_with_the_generator():
    # NUM_ELECTRONS as makeinput counts it (the database's nuclear charges
    # less two electrons per core state, _get_elec_and_states) against the
    # library's count on the deck it read
    s = _read()
    assert float(_label_value("NUM_ELECTRONS")[0]) == scf.valence_electrons(s)
