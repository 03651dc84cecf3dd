"""The valence charge of one SCF step (imago_b200.charge): the standard
population (populateStandard) against the oracle's statement-by-statement
loops, and the density traces of makeValenceRho on the GPU (the library's
trace kernel) against the oracle (LAPACK eigenvectors, rank-one updates,
matrixElementMult) on the same integral matrices."""

import numpy as np
import pytest

import oracle
from imago_b200 import charge, configs

# traces: the eigenvectors come from cuSOLVER on the GPU and LAPACK on the
# CPU, so the densities agree to the solvers' rounding, not bit for bit
TRACE_RTOL = 1e-9


def _spectrum(rng, nk, spin, ns, degenerate=False):
    e = np.sort(rng.normal(size=(nk, spin, ns)), axis=-1)
    if degenerate:
        # the same levels at every k-point and spin: whole shells are
        # degenerate across k, the population must share them
        e[:] = np.round(e[0, 0], 1)
    return e


@pytest.mark.parametrize("seed", range(6))
def test_populate_matches_oracle(seed):
    rng = np.random.default_rng(seed)
    nk, spin, ns = int(rng.integers(1, 6)), int(rng.integers(1, 3)), int(rng.integers(4, 12))
    e = _spectrum(rng, nk, spin, ns, degenerate=seed % 2 == 1)
    kw = rng.uniform(0.5, 1.5, nk)
    kw *= 2.0 / kw.sum()
    for ne in (1, 2, 3, int(ns * 0.7) + 1):
        got = charge.populate_standard(e, ne, kw)
        pop, occ_e, occ, gap, kind = oracle.populate_standard(e, ne, kw)
        assert np.allclose(got["population"], pop, rtol=0, atol=1e-14), (seed, ne)
        assert got["occupied_energy"] == occ_e and got["occupied_index"] == occ
        assert got["band_gap"] == gap and got["gap_kind"] == kind
        assert abs(got["population"].sum() - ne) < 1e-12


def test_populate_shares_a_degenerate_level():
    # two k-points, one spin: levels -1, 0, 0 at both; three electrons fill
    # -1 (two electrons) and leave one for the four-fold level 0 (weight 1/2
    # per state per k... i.e. 1/4 of its capacity each)
    e = np.array([[[-1.0, 0.0, 0.0]], [[-1.0, 0.0, 0.0]]])
    got = charge.populate_standard(e, 3)
    assert np.allclose(got["population"][:, 0, 0], 1.0)
    assert np.allclose(got["population"][:, 0, 1:], 0.25)
    assert got["band_gap"] == 0.0 and got["gap_kind"] == 0
    # insulators: the top of the valence band and the bottom of the
    # conduction band at the same k-point (direct) or not (indirect)
    e = np.array([[[-1.0, 0.0]], [[-1.25, 0.5]]])
    got = charge.populate_standard(e, 2)
    assert got["band_gap"] == 1.0 and got["gap_kind"] == 1
    e = np.array([[[-1.0, 0.5]], [[-1.25, 0.25]]])
    got = charge.populate_standard(e, 2)
    assert got["band_gap"] == 1.25 and got["gap_kind"] == 2
    with pytest.raises(ValueError):
        charge.populate_standard(e, 9)


@pytest.mark.parametrize("seed", range(5))
def test_smearing_matches_oracle(seed):
    # thermal smearing: sigma from 0.01 to 0.5 eV, in Hartree
    rng = np.random.default_rng(50 + seed)
    nk, spin, ns = int(rng.integers(1, 5)), int(rng.integers(1, 3)), int(rng.integers(5, 14))
    e = _spectrum(rng, nk, spin, ns, degenerate=seed == 4) * 0.3
    kw = rng.uniform(0.5, 1.5, nk)
    kw *= 2.0 / kw.sum()
    hartree = 27.21138386
    for sigma_ev in (0.01, 0.1, 0.5):
        ne = int(rng.integers(1, ns))
        args = (e, ne, sigma_ev / hartree, 20.0, 1.0 / hartree)
        got = charge.populate_smearing(*args, kpoint_weights=kw)
        pop, ef, it = oracle.populate_smearing(*args, kpoint_weights=kw)
        assert got["iterations"] == it and got["fermi_energy"] == ef, (seed, sigma_ev)
        assert np.allclose(got["population"], pop, rtol=0, atol=1e-14)
        assert abs(got["population"].sum() - ne) < 1e-8
        both = charge.populate_states(e, ne, kw, *args[2:])
        assert np.array_equal(both["population"], got["population"])


def test_smearing_tends_to_the_standard_population():
    # a gapped spectrum and a sigma far below the gap: the Fermi function
    # is a step at the gap, so the smeared population is the standard one
    e = np.array([[[-1.0, -0.5, 0.5]], [[-0.9, -0.4, 0.6]]])
    std = charge.populate_standard(e, 4)
    sm = charge.populate_smearing(e, 4, 0.001, 50.0, 0.05)
    assert np.allclose(sm["population"], std["population"], atol=1e-12)
    assert -0.4 < sm["fermi_energy"] < 0.5


def test_oracle_charge_trace_counts_the_electrons():
    # Tr(rho S) = sum_j f_j c_j^H S c_j = sum_j f_j = numElectrons
    s = configs.small_test_system()
    ob = oracle.OracleBuild(s)
    ol = ob.overlap()[0]
    ke, npm, ep = ob.kinetic(), ob.nuclear(), ob.elec_pot()
    w = -np.abs(np.random.default_rng(1).normal(0.5, 0.3, ep.shape[0]))
    r = oracle.valence_rho(npm, ke, ep, ol, w, 8, ob.vale_dim)
    assert abs(r["chargeDensityTrace"][0] - 8.0) < 1e-9


def _device_case(name, spin, rel):
    import torch
    from imago_b200 import intg
    s = (configs.small_test_system() if name == "small"
         else configs.silicon_cubic8(kmesh=(2, 2, 2)))
    dev = torch.device("cuda", 0)
    with intg.IntegralSetup(s) as g:
        which = intg.IMAGO_OL | intg.IMAGO_KE | intg.IMAGO_NP | intg.IMAGO_EP
        host = g.build(which | (intg.IMAGO_MV if rel else 0))
        V, P = g.vale_dim, g.pot_dim
    rng = np.random.default_rng(7)
    w = -np.abs(rng.normal(0.5, 0.3, (P, spin)))
    if spin == 2:
        w[:, 1] *= 1.1
    out = {k: torch.as_tensor(v, device=dev) for k, v in host.items()}
    return s, host, out, w, V


@pytest.mark.gpu
@pytest.mark.parametrize("name,spin,rel", [("small", 1, False), ("si8", 1, False),
                                           ("small", 2, True)])
def test_valence_rho_matches_oracle(imago_lib, name, spin, rel):
    from imago_b200 import secular
    s, host, out, w, V = _device_case(name, spin, rel)
    ns = V
    ne = 16 if name == "si8" else 8
    ref = oracle.valence_rho(host["np_packed"], host["ke_packed"], host["ep_packed"],
                             host["ol_packed"], w, ne, ns,
                             mv_packed=host.get("mv_packed") if rel else None)
    evs, vecs = [], []
    for sp in range(spin):
        e, c = secular.secular_eigensystem(out, w[:, sp], ns)
        evs.append(e)
        vecs.append(c)
    ev = np.stack([e.cpu().numpy() for e in evs], axis=1)
    assert np.abs(ev - ref["eigenvalues"]).max() <= 1e-8
    pop = charge.populate_standard(ev, ne)
    assert np.allclose(pop["population"], ref["population"], atol=1e-12)
    got = charge.valence_rho(out, evs, vecs, pop["population"], w, rel=rel)
    keys = ["chargeDensityTrace", "nucPotTrace", "kineticEnergyTrace", "potRho",
            "electronEnergy", "sumElecEnergy"] + (["massVelocityTrace"] if rel else [])
    for k in keys:
        scale = max(1.0, np.abs(ref[k]).max())
        assert np.abs(got[k] - ref[k]).max() <= TRACE_RTOL * scale, (k, got[k], ref[k])
    assert abs(got["chargeDensityTrace"][0] - ne) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("V,nk,nmat,nrho", [(7, 3, 2, 1), (91, 2, 3, 2), (140, 1, 5, 2)])
def test_packed_traces_kernel(imago_lib, V, nk, nmat, nrho):
    # against matrixElementMult on random packed data; V = 91 and 140 put
    # chunk boundaries (4096 elements) inside columns
    import torch
    rng = np.random.default_rng(V)
    npk = V * (V + 1) // 2
    mats = rng.normal(size=(nmat, nk, npk, 2))
    rho = rng.normal(size=(nrho, nk, npk, 2))
    got = charge.packed_traces(torch.as_tensor(mats, device="cuda"),
                               torch.as_tensor(rho, device="cuda"), nk, V).cpu().numpy()
    for m in range(nmat):
        for s in range(nrho):
            ref = sum(oracle.matrix_element_mult(mats[m, k], rho[s, k]) for k in range(nk))
            assert abs(got[m, s] - ref) <= 1e-12 * max(1.0, abs(ref)), (m, s)
