"""The SCF set-up and potential update (include/imago_scf.h) against the
reference's own routines executed statement for statement
(tests/golden/make_scf_golden.py: lattice.f90, elecStat.f90, exchCorr.f90,
coreCharge.f90, potentialUpdate.F90), and against the numpy oracle
(oracle/scf.py).

Tolerances: the lattice lists are exact; the electrostatic operators and
the mesh agree within 1e-12 relative to the largest element (the device's
exp and the order of the sums over site pairs); the core charge fit and the
next potential coefficients come out of ill-conditioned Gaussian fits
(condition numbers near 1e10), so they are compared at 1e-9 relative, the
convergence measure (a norm of the difference of two coefficient sets) at
1e-7 relative plus 1e-10, and what the physics depends on, the energies,
at 1e-9 Hartree per iteration and 1e-7 Hartree at convergence.
"""
import os

import numpy as np
import pytest

from conftest import ROOT
from imago_b200 import configs

GOLD = os.path.join(ROOT, "tests", "golden")


def _gold(name):
    return np.load(os.path.join(GOLD, name))


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


SYSTEMS = {"scf_diamond.npz": (lambda: configs.diamond_primitive(kmesh=(2, 2, 2)), 20),
           "scf_two_type.npz": (configs.small_test_system, 8)}


def _check_setup(g, cells, csize, rcells, rcsize, arr, site_points, weights, op):
    assert np.array_equal(csize, g["cellSizesReal"])
    assert np.array_equal(cells, g["cellDimsReal"])
    assert np.array_equal(rcsize, g["cellSizesRecip"])
    assert np.array_equal(rcells, g["cellDimsRecip"])
    for key, ref in (("potAlphaOverlap", "potalphaoverlap"),
                     ("nonLocalNeutQPot", "nonlocalneutqpot"),
                     ("localNeutQPot", "localneutqpot"), ("nonLocalNucQPot", "nonlocalnucqpot"),
                     ("localNucQPot", "localnucqpot"),
                     ("nonLocalResidualQ", "nonlocalresidualq")):
        assert _rel(arr[key], g[ref]) < 1e-12, key
    assert _rel(arr["coreChargeDensity"], g["coreChargeDensity"]) < 1e-9
    assert np.array_equal(site_points, g["numPoints"])
    assert _rel(weights, g["radialWeight"]) < 1e-13
    assert _rel(op, g["exchRhoOp"]) < 1e-12
    assert _rel(arr["exchCorrOverlap"], g["exchCorrOverlap"]) < 1e-12


@pytest.mark.parametrize("fixture", sorted(SYSTEMS))
def test_oracle_setup_matches_reference_routines(fixture):
    from oracle import scf as oscf
    make, nsv = SYSTEMS[fixture]
    g = _gold(fixture)
    o = oscf.ScfOracle(make(), num_sample_vectors=nsv)
    arr = {"potAlphaOverlap": o.pot_ol, "nonLocalNeutQPot": o.nl_neut,
           "localNeutQPot": o.l_neut, "nonLocalNucQPot": o.nl_nuc, "localNucQPot": o.l_nuc,
           "nonLocalResidualQ": o.nl_res, "coreChargeDensity": o.core,
           "exchCorrOverlap": o.xc_ol}
    _check_setup(g, o.cells, o.csize, o.rcells, o.rcsize, arr, o.site_points, o.weights, o.op)


def _replay(update, g):
    """Feed each recorded iteration's valence charge to `update` and compare
    its outputs with the reference's makeSCFPot."""
    for it in range(len(g["scf_totalEnergy"])):
        nxt, r = update(g["scf_potRho"][it], g["scf_nucPotTrace"][it],
                        g["scf_kineticEnergyTrace"][it], g["scf_used"][it])
        for key in ("totalEnergy", "kineticEnergy", "elecStatEnergy", "exchCorrEnergy"):
            assert abs(r[key] - g["scf_" + key][it]) < 1e-9, (it, key)
        assert abs(r["electronDiff"] - g["scf_electronDiff"][it]) < 1e-9
        # testableDelta is a norm of (new - used) coefficients, which cancel
        # near convergence: its absolute error is that of the coefficients
        # (1e-9 relative of their size, O(1..100)) times the mesh operator
        assert abs(r["testableDelta"] - g["scf_testableDelta"][it]) <= \
            1e-7 * g["scf_testableDelta"][it] + 1e-10
        assert r["converged"] == g["scf_converged"][it]
        assert _rel(nxt, g["scf_next"][it]) < 1e-9, it


def test_oracle_update_matches_reference_make_scf_pot():
    from imago_b200 import scf
    from oracle import scf as oscf
    g = _gold("scf_diamond.npz")
    s = configs.diamond_primitive(kmesh=(2, 2, 2))
    o = oscf.ScfOracle(s, num_sample_vectors=20)
    o.reset()
    ne = scf.valence_electrons(s)
    _replay(lambda pr, nuc, kin, c: o.make_scf_pot(pr, nuc, kin, c, ne), g)
    # the recorded run converged by the reference's own test
    assert g["scf_converged"][-1] == 1


def test_atomic_start_is_the_recorded_start():
    from imago_b200 import scf
    g = _gold("scf_diamond.npz")
    assert np.array_equal(scf.atomic_start(configs.diamond_primitive(kmesh=(2, 2, 2))),
                          g["scf_used"][0])


# ------------------------------------------------------------------- GPU

@pytest.mark.gpu
@pytest.mark.parametrize("fixture", sorted(SYSTEMS))
def test_library_setup_matches_reference_routines(imago_lib, fixture):
    from imago_b200 import scf
    make, nsv = SYSTEMS[fixture]
    g = _gold(fixture)
    with scf.ScfSetup(make(), scf.ScfParams(num_sample_vectors=nsv)) as st:
        cells, csize, rcells, rcsize = st.lattice()
        n, w, op = st.mesh()
        _check_setup(g, cells, csize, rcells, rcsize, st.setup_arrays(), n, w, op)


@pytest.mark.gpu
def test_library_update_matches_reference_make_scf_pot(imago_lib):
    from imago_b200 import scf
    g = _gold("scf_diamond.npz")
    s = configs.diamond_primitive(kmesh=(2, 2, 2))
    with scf.ScfSetup(s, scf.ScfParams(num_sample_vectors=20)) as st:
        _replay(st.pot_update, g)


@pytest.mark.gpu
def test_gpu_scf_converges_to_the_reference_energy(imago_lib):
    # the whole loop on the GPU (integrals, secular equation, populations,
    # density traces, makeSCFPot) from the atomic-superposition start: the
    # reference's convergence test ends it at the recorded iteration, on the
    # recorded total energy
    from imago_b200 import scf
    g = _gold("scf_diamond.npz")
    s = configs.diamond_primitive(kmesh=(2, 2, 2))
    p = scf.ScfParams(num_sample_vectors=20, energy_tol=0.0)
    r = scf.run_scf(s, scf.atomic_start(s), p)
    n = len(g["scf_totalEnergy"])
    assert r["converged"] and r["iterations"] == n
    assert np.abs(np.array(r["energies"]) - g["scf_totalEnergy"]).max() < 1e-7
    assert abs(r["energies"][-1] - g["scf_totalEnergy"][-1]) < 1e-7


@pytest.mark.gpu
def test_gpu_setup_matches_oracle_on_si8(imago_lib):
    # a cell the reference was not run on: the jittered Si8 cell (one type,
    # 8 sites, 20 terms) with 12 sample vectors, library against oracle
    from imago_b200 import scf
    from oracle import scf as oscf
    s = configs.silicon_cubic8(kmesh=(1, 1, 1))
    o = oscf.ScfOracle(s, num_sample_vectors=12)
    with scf.ScfSetup(s, scf.ScfParams(num_sample_vectors=12)) as st:
        cells, csize, rcells, rcsize = st.lattice()
        assert np.array_equal(csize, o.csize) and np.array_equal(rcsize, o.rcsize)
        a = st.setup_arrays()
        for key, ref in (("potAlphaOverlap", o.pot_ol), ("nonLocalNeutQPot", o.nl_neut),
                         ("localNeutQPot", o.l_neut), ("nonLocalNucQPot", o.nl_nuc),
                         ("localNucQPot", o.l_nuc), ("nonLocalResidualQ", o.nl_res),
                         ("exchCorrOverlap", o.xc_ol)):
            assert _rel(a[key], ref) < 1e-12, key
        assert _rel(a["coreChargeDensity"], o.core) < 1e-9
        n, w, op = st.mesh()
        assert np.array_equal(n, o.site_points)
        assert _rel(op, o.op) < 1e-12


@pytest.mark.gpu
def test_gpu_scf_matches_the_oracle_loop_on_si8_2x2x2(imago_lib):
    # the whole SCF on the jittered Si8 cell at 2x2x2 k (8 k-points, one
    # type, 20 terms), GPU against the CPU oracle's loop (the oracle's
    # integrals, LAPACK eigh(H, S), populateStandard, makeValenceRho's
    # traces and makeSCFPot restated): the same iterations, every total
    # energy within 1e-7 Ha, and the last iteration's eigenvalues within
    # 1e-8 Ha
    import oracle
    from oracle import scf as oscf
    from imago_b200 import scf, secular
    s = configs.silicon_cubic8(kmesh=(2, 2, 2))
    nsv = 12
    ne = scf.valence_electrons(s)
    ob = oracle.OracleBuild(s)
    ol, _, _ = ob.overlap()
    ke, npk, ep = ob.kinetic(), ob.nuclear(), ob.elec_pot()
    o = oscf.ScfOracle(s, num_sample_vectors=nsv)
    o.reset()
    coeffs = scf.atomic_start(s)
    V = ol.shape[1]
    V = int((int((8 * V + 1) ** 0.5) - 1) // 2)
    energies, last_ev = [], None
    for _ in range(30):
        r = oracle.valence_rho(npk, ke, ep, ol, coeffs, ne, V)
        last_ev = r["eigenvalues"][:, 0, :]
        coeffs, res = o.make_scf_pot(r["potRho"][:, 0], r["nucPotTrace"][0],
                                     r["kineticEnergyTrace"][0], coeffs, ne)
        energies.append(res["totalEnergy"])
        if res["converged"]:
            break
    p = scf.ScfParams(num_sample_vectors=nsv, energy_tol=0.0)
    ints, _ = scf.device_integrals(s)
    g = scf.run_scf(s, scf.atomic_start(s), p, integrals=ints)
    assert g["converged"] and g["iterations"] == len(energies)
    assert np.abs(np.array(g["energies"]) - np.array(energies)).max() < 1e-7
    ev = secular.secular_eigenvalues(ints, g["pot_coeffs"]).cpu().numpy()
    assert np.abs(ev - last_ev).max() < 1e-8
