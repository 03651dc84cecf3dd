"""The secular equation of one SCF step (secularEqnSCF) from the integral
builds: H = NP + KE + sum_j w_j EP_j and S = OL unpacked and solved as the
generalised Hermitian problem.  Eigenvalues on the GPU (the library's
assembly and Cholesky-reduction kernels, then cuSOLVER's batched solver or
the library's Jacobi kernel) against the CPU oracle (numpy assembly,
LAPACK), within the 1e-8 Hartree of the target."""

import numpy as np
import pytest

import oracle
from imago_b200 import configs, intg

EV_TOL = 1e-8  # Hartree


def _coefficients(pot_dim, seed=1):
    # synthetic potential coefficients (the reference reads them from the
    # SCF potential file); one is exactly 0.0, which the reference's
    # accumulation adds with weight one
    rng = np.random.default_rng(seed)
    w = -np.abs(rng.normal(0.5, 0.3, pot_dim))
    w[1] = 0.0
    return w


def test_zero_factor_adds_the_matrix_unscaled():
    s = configs.small_test_system()
    ob = oracle.OracleBuild(s)
    ol = ob.overlap()[0]
    ke, npm, ep = ob.kinetic(), ob.nuclear(), ob.elec_pot()
    w = _coefficients(ep.shape[0])
    w1 = w.copy()
    w1[1] = 1.0
    a = oracle.secular_eigenvalues(npm, ke, ep, w, ol)
    b = oracle.secular_eigenvalues(npm, ke, ep, w1, ol)
    assert np.array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("name,rel", [("small", False), ("si8_2x2x2", False),
                                      ("small", True)])
def test_secular_eigenvalues_match_oracle(imago_lib, name, rel):
    # rel: a scalar-relativistic step, the mass velocity added after KE
    import torch
    from imago_b200 import secular
    s = (configs.small_test_system() if name == "small"
         else configs.silicon_cubic8(kmesh=(2, 2, 2)))
    ob = oracle.OracleBuild(s)
    ol = ob.overlap()[0]
    ke, npm, ep = ob.kinetic(), ob.nuclear(), ob.elec_pot()
    mv = ob.mass_velocity() if rel else None
    w = _coefficients(ep.shape[0])
    ref = oracle.secular_eigenvalues(npm, ke, ep, w, ol, mv_packed=mv)
    dev = torch.device("cuda", 0)
    with intg.IntegralSetup(s, outputs_on_device=True) as g:
        C = max(g.core_dim, 1)
        shapes = {"ol_packed": (g.nk, g.npacked, 2), "ol_cv_re": (g.nk, g.vale_dim, C),
                  "ol_cv_im": (g.nk, g.vale_dim, C), "ke_packed": (g.nk, g.npacked, 2),
                  "np_packed": (g.nk, g.npacked, 2),
                  "ep_packed": (g.pot_dim, g.nk, g.npacked, 2)}
        if rel:
            shapes["mv_packed"] = (g.nk, g.npacked, 2)
        out = {k: torch.empty(v, dtype=torch.float64, device=dev) for k, v in shapes.items()}
        which = intg.IMAGO_OL | intg.IMAGO_KE | intg.IMAGO_NP | intg.IMAGO_EP
        g.build(which | (intg.IMAGO_MV if rel else 0), out=out)
        ev = secular.secular_eigenvalues(out, w).cpu().numpy()
    assert ev.shape == ref.shape
    assert np.abs(ev - ref).max() <= EV_TOL, np.abs(ev - ref).max()


@pytest.fixture(params=["jacobi", "batched"])
def eigensolver(request):
    # each solver behind imago_hermitian_eigvals/eigh in turn, the default
    # restored after the test
    from imago_b200 import secular
    before = secular.eigensolver()
    secular.set_eigensolver(request.param)
    yield request.param
    secular.set_eigensolver(before)


def test_eigensolver_choice_is_validated(imago_lib):
    from imago_b200 import secular
    assert secular.eigensolver() == "auto"
    with pytest.raises(ValueError):
        secular.set_eigensolver("qr")
    assert imago_lib.imago_hermitian_set_solver(3) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 5, 33, 104, 112])
def test_batched_jacobi_eigenvalues(imago_lib, eigensolver, n):
    # imago_hermitian_eigvals against LAPACK, including degenerate spectra
    import torch
    from imago_b200 import secular
    rng = np.random.default_rng(n)
    b = 7
    x = rng.normal(size=(b, n, n)) + 1j * rng.normal(size=(b, n, n))
    h = (x + np.conj(np.swapaxes(x, 1, 2))) / 2
    h[0] = np.eye(n) * 2.5                       # fully degenerate
    h[1] = np.diag(np.arange(n, dtype=float))    # already diagonal
    ref = np.linalg.eigvalsh(h)
    got = secular.hermitian_eigvals(torch.as_tensor(h, device="cuda")).cpu().numpy()
    scale = max(1.0, np.abs(ref).max())
    assert np.abs(got - ref).max() <= 1e-12 * scale


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 5, 33, 104, 112])
def test_batched_jacobi_eigenvectors(imago_lib, eigensolver, n):
    # imago_hermitian_eigh: A V = V diag(w), V unitary, w as LAPACK's, on
    # random and degenerate spectra
    import torch
    from imago_b200 import secular
    rng = np.random.default_rng(100 + n)
    b = 6
    x = rng.normal(size=(b, n, n)) + 1j * rng.normal(size=(b, n, n))
    h = (x + np.conj(np.swapaxes(x, 1, 2))) / 2
    h[0] = np.eye(n) * 2.5
    if n > 3:  # a three-fold level inside a random spectrum
        q, _ = np.linalg.qr(x[1])
        d = np.sort(rng.normal(size=n))
        d[1:4] = d[1]
        h[1] = (q * d) @ np.conj(q.T)
    w, v = secular.hermitian_eigh(torch.as_tensor(h, device="cuda"))
    w, v = w.cpu().numpy(), v.cpu().numpy()
    scale = max(1.0, np.abs(h).max())
    assert np.abs(w - np.linalg.eigvalsh(h)).max() <= 1e-12 * scale * n
    for i in range(b):
        assert np.abs(h[i] @ v[i] - v[i] * w[i]).max() <= 1e-11 * scale * n
        assert np.abs(np.conj(v[i].T) @ v[i] - np.eye(n)).max() <= 1e-12 * n


def test_oracle_pscf_hamiltonian_is_the_combination_of_its_parts():
    # gaussOverlapHamPSCF sums kinetic, nuclear, potCoeffs-weighted
    # potential terms and (rel) minus mass velocity per alpha pair; every
    # later step is linear, so it equals the same combination of the
    # separate builds up to rounding and the screen radius's evaluation
    # order (an ulp of the radius)
    s = configs.small_test_system()
    ob = oracle.OracleBuild(s)
    ob.overlap()
    rng = np.random.default_rng(3)
    w = rng.normal(size=(ob.pot_dim, 2))
    h = ob.ham_pscf(w, rel=True)
    lin = (ob.kinetic() + ob.nuclear() + ob.mass_velocity()
           + np.tensordot(w.T, ob.elec_pot(), axes=1))
    assert h.shape == lin.shape
    assert np.abs(h - lin).max() <= 1e-12 * np.abs(lin).max()


def test_mass_velocity_shifts_the_oracle_eigenvalues():
    # rel adds -p^4/8c^2: every eigenvalue moves down, by a few per cent
    # at most (the most at the highest states, where p^4 is largest)
    s = configs.small_test_system()
    ob = oracle.OracleBuild(s)
    ol = ob.overlap()[0]
    ke, npm, ep, mv = ob.kinetic(), ob.nuclear(), ob.elec_pot(), ob.mass_velocity()
    w = _coefficients(ep.shape[0])
    a = oracle.secular_eigenvalues(npm, ke, ep, w, ol)
    b = oracle.secular_eigenvalues(npm, ke, ep, w, ol, mv_packed=mv)
    assert np.all(b <= a + 1e-12)
    assert np.all(a - b <= 0.05 * (np.abs(a) + 1.0))


@pytest.mark.gpu
@pytest.mark.parametrize("n", [113, 208])
def test_batched_eigensolver_beyond_the_jacobi_kernel(imago_lib, n):
    # above n = 112 imago_hermitian_eigh hands the batch to cuSOLVER's
    # batched solver under the same contract: ascending eigenvalues equal to
    # LAPACK's, unit eigenvectors in columns with A V = V diag(w)
    import torch
    from imago_b200 import secular
    rng = np.random.default_rng(n)
    x = rng.normal(size=(3, n, n)) + 1j * rng.normal(size=(3, n, n))
    a = (x + np.conj(np.transpose(x, (0, 2, 1)))) / 2
    at = torch.tensor(a, device="cuda")
    w, v = secular.hermitian_eigh(at)
    w, v = w.cpu().numpy(), v.cpu().numpy()
    ref = np.linalg.eigvalsh(a)
    assert np.abs(w - ref).max() < 1e-10 * np.abs(ref).max()
    for b in range(3):
        r = a[b] @ v[b] - v[b] * w[b][None, :]
        assert np.abs(r).max() < 1e-10 * np.abs(ref[b]).max()
        assert np.abs(np.conj(v[b].T) @ v[b] - np.eye(n)).max() < 1e-10
    assert np.abs(secular.hermitian_eigvals(at).cpu().numpy() - ref).max() < \
        1e-10 * np.abs(ref).max()
