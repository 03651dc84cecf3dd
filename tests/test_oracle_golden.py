"""The CPU oracle's primitives against the reference's own generated
kernels (tests/golden/primitives.json, made by executing
src/imago/gaussIntegrals.f90 statement by statement)."""
import numpy as np
import pytest

import oracle
from conftest import massvel_scale, momentum_scale

KINDS = ("overlap", "kinetic", "electron3c", "nuclear3c")
# Relative to the largest element of the block.  The oracle uses its own
# recursions, so the two agree to rounding; 1e-12 leaves room for the
# nuclear higher classes (observed <= 1.2e-13).
RTOL = 1e-12


@pytest.mark.parametrize("kind", KINDS)
def test_primitives_match_reference_kernels(golden, kind):
    n = 0
    for r in golden["records"]:
        if kind not in r:
            continue
        ref = np.array(r[kind])
        got = oracle.primitive(kind, r["la"], r["lb"], r["a1"], r["a2"],
                               r["a3"], r["A"], r["B"], r["C"])
        scale = max(np.abs(ref).max(), 1e-300)
        assert np.abs(got - ref).max() <= RTOL * scale, (kind, r["la"], r["lb"])
        n += 1
    assert n >= 64


def test_boys_bit_exact_with_reference(golden):
    # Same branch structure, same single-precision series constants and the
    # same operation order as gaussIntegrals.f90:16080-16221.
    for row in golden["boys"]:
        F = oracle.boys(row["T"])
        assert np.array_equal(F, np.array(row["F"])), row["T"]


def test_boys_reference_deviation_from_exact():
    # The reference's series constants are single precision, so F_6(0) is
    # not 1/13; the oracle keeps that.
    F = oracle.boys(0.0)
    assert abs(F[6] - 1.0 / 13.0) > 1e-9
    assert abs(F[6] - 1.0 / 13.0) < 1e-7


def test_closed_forms_s_s():
    a1, a2, a3 = 0.7, 1.9, 3.1
    A, B, C = np.array([0.1, 0.2, -0.3]), np.array([1.0, -0.4, 0.5]), np.array([0.3, 0.9, 0.2])
    z, xi = a1 + a2, a1 * a2 / (a1 + a2)
    d2 = ((A - B) ** 2).sum()
    S = (np.pi / z) ** 1.5 * np.exp(-xi * d2)
    assert oracle.primitive("overlap", 0, 0, a1, a2, 0, A, B, C)[0, 0] == pytest.approx(S, rel=1e-14)
    assert oracle.primitive("kinetic", 0, 0, a1, a2, 0, A, B, C)[0, 0] == pytest.approx(
        xi * (3 - 2 * xi * d2) * S, rel=1e-13)
    z3 = z + a3
    P = (a1 * A + a2 * B) / z
    E = (np.pi / z3) ** 1.5 * np.exp(-xi * d2 - z * a3 / z3 * ((P - C) ** 2).sum())
    assert oracle.primitive("electron3c", 0, 0, a1, a2, a3, A, B, C)[0, 0] == pytest.approx(E, rel=1e-14)


def test_massvel_matches_reference_kernel(golden):
    n = 0
    for r in golden["records"]:
        if "massvel" not in r:
            continue
        ref = np.array(r["massvel"])
        got = oracle.primitive("massvel", r["la"], r["lb"], r["a1"], r["a2"],
                               0.0, r["A"], r["B"], r["C"])
        # observed <= 2.3e-13 of the scale over all 16 classes
        assert np.abs(got - ref).max() <= 1e-12 * massvel_scale(r), (r["la"], r["lb"])
        n += 1
    assert n == 64


def test_massvel_s_s_against_50_digit_value(golden):
    # The closed s-s form in 50-digit arithmetic: the oracle's symmetric
    # <nabla^2 a|nabla^2 b> keeps 1e-10 relative accuracy where the
    # reference's seed has cancelled (a1 << a2), and agrees with the
    # reference to rounding elsewhere.
    mp = pytest.importorskip("mpmath")
    mp.mp.dps = 50
    fs = mp.mpf("7.2973525693") * mp.mpf("0.001")
    n = 0
    for r in golden["records"]:
        if r["la"] or r["lb"] or "massvel" not in r:
            continue
        a1, a2 = mp.mpf(r["a1"]), mp.mpf(r["a2"])
        A = [mp.mpf(x) for x in r["A"]]
        B = [mp.mpf(x) for x in r["B"]]
        z = a1 + a2
        PB = [(a1 * A[i] + a2 * B[i]) / z - B[i] for i in range(3)]
        d2 = sum((A[i] - B[i]) ** 2 for i in range(3))
        S = (mp.pi / z) ** mp.mpf(1.5) * mp.exp(-a1 * a2 / z * d2)
        p2 = sum(x ** 2 for x in PB)
        r4 = (sum(x ** 4 for x in PB) + 3 * p2 / z + mp.mpf(9) / (4 * z ** 2)
              + 2 * ((PB[0] * PB[1]) ** 2 + (PB[0] * PB[2]) ** 2
                     + (PB[1] * PB[2]) ** 2 + p2 / z + mp.mpf(3) / (4 * z ** 2)))
        exact = fs ** 2 / 8 * (16 * a2 ** 4 * r4 - 80 * a2 ** 3 * (p2 + 3 / (2 * z))
                               + 60 * a2 ** 2) * S
        got = oracle.primitive("massvel", 0, 0, r["a1"], r["a2"], 0.0, r["A"],
                               r["B"], r["C"])[0, 0]
        assert abs(got - float(exact)) <= 1e-10 * abs(float(exact))
        n += 1
    assert n >= 4


def test_momentum_and_dipole_match_reference_kernels(golden):
    # three components each; momentum at the size the reference's own seed
    # rounds at (observed <= 3.1e-16 of it), dipole at 1e-12 of the block
    n = 0
    for r in golden["records"]:
        if "momentum" not in r:
            continue
        ref = np.array(r["momentum"])
        got = oracle.primitive_vec("momentum", r["la"], r["lb"], r["a1"], r["a2"],
                                   r["A"], r["B"])
        scale = max(np.abs(ref).max(), momentum_scale(r))
        assert np.abs(got - ref).max() <= 1e-12 * scale, (r["la"], r["lb"])
        ref = np.array(r["dipole"])
        got = oracle.primitive_vec("dipole", r["la"], r["lb"], r["a1"], r["a2"],
                                   r["A"], r["B"], r["C"])
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), (r["la"], r["lb"])
        n += 1
    assert n == 64


def test_koverlap_matches_reference_kernel(golden):
    # <a|exp(-i dK.r)|b>, complex, at random wave vectors of |dK| ~ 1
    # bohr^-1 (a few times the reference's recipVectors / numAxialKPoints)
    n = 0
    for r in golden["records"]:
        if "koverlap" not in r:
            continue
        ref = np.array(r["koverlap"])
        ref = ref[..., 0] + 1j * ref[..., 1]
        got = oracle.primitive_koverlap(r["la"], r["lb"], r["a1"], r["a2"],
                                        r["A"], r["B"], r["dK"])
        assert got.shape == ref.shape
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), (r["la"], r["lb"])
        n += 1
    assert n == 64


def test_koverlap_at_zero_wave_vector_is_the_overlap():
    # exp(-i 0.r) = 1: the plane-wave overlap of dK = 0 is the orthogonalised
    # overlap itself, here unpacked from its Hermitian upper triangle
    from imago_b200 import configs
    s = configs.small_test_system()
    ob = oracle.OracleBuild(s)
    ol = ob.overlap()[0]
    kov = ob.koverlap(np.zeros((3, 3)))
    V = ob.vale_dim
    iu = np.triu_indices(V)
    for k in range(ob.nk):
        full = np.zeros((V, V), complex)
        p = ol[k, :, 0] + 1j * ol[k, :, 1]
        # packed column-major upper triangle: index col (col + 1) / 2 + row
        cols, rows = iu[1], iu[0]
        order = np.argsort(cols * (cols + 1) // 2 + rows)
        full[rows[order], cols[order]] = p
        full = full + np.conj(np.triu(full, 1)).T
        for ax in range(3):
            # the packed overlap zeroes entries below 1e-10; the full planes
            # do not
            assert np.abs(kov[ax, k] - full).max() <= 1e-10


def test_oracle_driver_matches_reference_driver_executed():
    # the oracle's restatement of the integral driver against the
    # reference's own driver executed statement for statement
    # (tests/golden/make_driver_golden.py): OL with coreValeOL, KE, NP and
    # the 16 EP terms on the diamond primitive cell at 2x2x2 k
    import os
    import numpy as np
    import oracle
    from conftest import ROOT, packed_mismatch
    from imago_b200 import configs
    g = np.load(os.path.join(ROOT, "tests", "golden", "driver_diamond.npz"))
    ob = oracle.OracleBuild(configs.diamond_primitive(kmesh=(2, 2, 2)))
    ol, cre, cim = ob.overlap()
    ke = ob.kinetic()
    npk = ob.nuclear()
    ep = ob.elec_pot()
    assert np.array_equal(ob.kpoints_xyz(), g["kPointsXYZ"])
    assert ep.shape == g["ep_packed"].shape
    for a, b in ((ol, g["ol_packed"]), (ke, g["ke_packed"]), (cre, g["ol_cv_re"]),
                 (cim, g["ol_cv_im"]), (npk, g["np_packed"]), (ep, g["ep_packed"])):
        assert packed_mismatch(a, b, atol=1e-13)[1] == 0


def test_oracle_cell_list_gives_the_reference_phase_factors():
    # computePhaseFactors (kpoints.f90:578-609) executed over the
    # reference's own cell list (initializeLattice): the oracle's integral
    # cell list, in its order, reproduces every exp(i k.R) of it
    import os
    import numpy as np
    import oracle
    from conftest import ROOT
    from imago_b200 import configs
    g = np.load(os.path.join(ROOT, "tests", "golden", "driver_diamond.npz"))
    ob = oracle.OracleBuild(configs.diamond_primitive(kmesh=(2, 2, 2)))
    cells, _ = ob.cells()
    assert cells.shape[0] == g["phaseFactor"].shape[0]
    ph = np.exp(1j * (cells @ ob.kpoints_xyz().T))
    assert np.abs(ph - g["phaseFactor"]).max() < 1e-14
