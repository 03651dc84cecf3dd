"""Deck reading and writing in the reference's input formats."""
import numpy as np

from imago_b200 import configs, deck


def _same(a, b):
    assert np.array_equal(a.real_vectors, b.real_vectors)
    assert np.array_equal(a.site_type, b.site_type)
    assert np.array_equal(a.site_pos, b.site_pos)
    assert np.array_equal(a.pot_site_type, b.pot_site_type)
    assert np.array_equal(a.kpoints_abc, b.kpoints_abc)
    assert a.basis_fn_convg == b.basis_fn_convg
    for t, u in zip(a.atom_types, b.atom_types):
        assert t.num_orb_alphas == u.num_orb_alphas
        assert np.array_equal(t.alphas, u.alphas)
        assert t.core_l == u.core_l and t.vale_l == u.vale_l
        for c, d in zip(t.core_coeffs + t.vale_coeffs, u.core_coeffs + u.vale_coeffs):
            assert np.array_equal(c, d)
    for p, q in zip(a.pot_types, b.pot_types):
        assert p.nuc_charge == q.nuc_charge and p.nuc_alpha == q.nuc_alpha
        assert np.allclose(p.alphas, q.alphas, rtol=1e-15)


def test_round_trip_mesh(tmp_path):
    s = configs.small_test_system()
    deck.write_decks(s, tmp_path)
    _same(s, deck.read_decks(tmp_path))


def test_round_trip_explicit_kpoints(tmp_path):
    s = configs.f_test_system()
    deck.write_decks(s, tmp_path, kpoint_style=0)
    _same(s, deck.read_decks(tmp_path))


def test_reader_skips_control_sections(tmp_path):
    s = configs.diamond_primitive(kmesh=(2, 2, 2))
    deck.write_decks(s, tmp_path)
    f5 = tmp_path / "fort.5"
    txt = f5.read_text()
    # control sections the integral path does not use sit between the
    # potential types and SHARED_INPUT_DATA in a full deck
    txt = txt.replace("SHARED_INPUT_DATA", "EXCHANGE_CORRELATION\n1 2 3\n"
                      "RADIAL_SAMPLE-IN_OUT_SPACING\n0.1 0.2 0.3\nSHARED_INPUT_DATA", 1)
    f5.write_text(txt)
    _same(s, deck.read_decks(tmp_path))


def test_basis_code_selects_functions(tmp_path):
    s = configs.small_test_system()
    deck.write_decks(s, tmp_path)
    f5 = tmp_path / "fort.5"
    lines = f5.read_text().split("\n")
    # tag the first valence function of type 1 as extended-basis only (3)
    i = lines.index("NUM_VALE_RADIAL_FNS")
    assert lines[i + 2] == "NL_RADIAL_FUNCTIONS"
    lines[i + 3] = "1 3"
    f5.write_text("\n".join(lines))
    fb = deck.read_decks(tmp_path, basis_code=2)
    eb = deck.read_decks(tmp_path, basis_code=3)
    assert len(fb.atom_types[0].vale_l) == len(s.atom_types[0].vale_l) - 1
    assert len(eb.atom_types[0].vale_l) == len(s.atom_types[0].vale_l)
