"""The library's Cholesky reduction, back-transformation and packed density
(imago_secular_reduce / imago_secular_back / imago_packed_density, the
zpotrf + zhegst, ztrsm and zher steps of one SCF step) against numpy's
LAPACK on seeded matrices, every size class of the kernels (n up to 128,
one to four rows per lane), and zpotrf's failure report."""

import numpy as np
import pytest
import scipy.linalg

torch = pytest.importorskip("torch")

SIZES = [1, 5, 31, 32, 33, 64, 97, 104, 112, 128]


def _hermitian_pair(n, nk, seed):
    """Per k-point a Hermitian H and a well-conditioned Hermitian positive
    definite S, as the secular equation gives them."""
    rng = np.random.default_rng(seed)
    h = rng.normal(size=(nk, n, n)) + 1j * rng.normal(size=(nk, n, n))
    h = 0.5 * (h + h.conj().transpose(0, 2, 1))
    b = (rng.normal(size=(nk, n, n)) + 1j * rng.normal(size=(nk, n, n))) / np.sqrt(n)
    s = b @ b.conj().transpose(0, 2, 1) + np.eye(n)
    for k in range(nk):
        np.fill_diagonal(s[k], s[k].diagonal().real)
        np.fill_diagonal(h[k], h[k].diagonal().real)
    return h, s


def _storage(m):
    """Column-major per k-point, as imago_secular_matrices writes."""
    return torch.as_tensor(np.ascontiguousarray(m.transpose(0, 2, 1)), device="cuda")


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("n", SIZES)
def test_reduce_matches_lapack(n):
    from imago_b200 import secular
    nk = 3
    h, s = _hermitian_pair(n, nk, seed=n)
    a, lfac, info = secular.cholesky_reduce(_storage(h), _storage(s), factor=True)
    secular._check_info(info)
    lo = np.linalg.cholesky(s)
    li = np.linalg.inv(lo)
    ref = li @ h @ li.conj().transpose(0, 2, 1)
    assert _rel(a.cpu().numpy(), ref) < 1e-12
    # the factor, column by column from the diagonal down
    got = lfac.cpu().numpy()
    rows, cols = np.tril_indices(n)
    order = np.lexsort((rows, cols))
    assert _rel(got, lo[:, rows[order], cols[order]]) < 1e-13
    assert np.all(got[:, [j * n - j * (j - 1) // 2 for j in range(n)]].imag == 0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 33, 104, 128])
def test_back_transform_matches_lapack(n):
    from imago_b200 import secular
    nk, ns = 2, max(1, n // 3)
    h, s = _hermitian_pair(n, nk, seed=100 + n)
    _, lfac, _ = secular.cholesky_reduce(_storage(h), _storage(s), factor=True)
    rng = np.random.default_rng(n)
    vec = rng.normal(size=(nk, n, n)) + 1j * rng.normal(size=(nk, n, n))
    c = secular.back_transform(lfac, torch.as_tensor(vec, device="cuda"), ns)
    assert tuple(c.shape) == (nk, n, ns)
    lo = np.linalg.cholesky(s)
    ref = np.linalg.solve(lo.conj().transpose(0, 2, 1), vec[:, :, :ns])
    assert _rel(c.cpu().numpy(), ref) < 1e-12


@pytest.mark.gpu
def test_generalised_eigenvectors_are_s_normalised():
    # zhegv's normalisation: c^H S c = 1, and H c = E S c
    from imago_b200 import secular
    n, nk = 104, 2
    h, s = _hermitian_pair(n, nk, seed=7)
    a, lfac, info = secular.cholesky_reduce(_storage(h), _storage(s), factor=True)
    ev, vec = secular.hermitian_eigh(a)
    c = secular.back_transform(lfac, vec, n).cpu().numpy()
    secular._check_info(info)
    ev = ev.cpu().numpy()
    for k in range(nk):
        g = c[k].conj().T @ s[k] @ c[k]
        assert np.abs(g - np.eye(n)).max() < 1e-10
        assert np.abs(h[k] @ c[k] - s[k] @ c[k] * ev[k]).max() < 1e-9
        ref = scipy.linalg.eigh(h[k], s[k], eigvals_only=True)
        assert np.abs(ref - ev[k]).max() < 1e-9


@pytest.mark.gpu
def test_reduce_reports_the_leading_minor_that_is_not_positive_definite():
    from imago_b200 import secular
    n, nk = 40, 3
    h, s = _hermitian_pair(n, nk, seed=3)
    s[1] = np.eye(n)
    s[1][17, 17] = -1.0          # leading minor of order 18 is not positive definite
    a, _, info = secular.cholesky_reduce(_storage(h), _storage(s))
    got = info.cpu().numpy()
    assert got.tolist() == [0, 18, 0]
    assert np.all(a[1].cpu().numpy() == 0.0)
    with pytest.raises(ValueError, match="k-point 1"):
        secular._check_info(info)


@pytest.mark.gpu
@pytest.mark.parametrize("n,ns,used", [(1, 1, 1), (40, 20, 7), (104, 104, 16), (150, 90, 61)])
def test_packed_density_matches_zher(n, ns, used):
    from imago_b200 import charge
    nk = 3
    rng = np.random.default_rng(n + ns)
    c = rng.normal(size=(nk, n, ns)) + 1j * rng.normal(size=(nk, n, ns))
    f = np.zeros((nk, ns))
    f[:, :used] = rng.uniform(0.0, 2.0 / nk, size=(nk, used))
    f[0, used - 1] = 0.0                 # a gap inside the occupied range
    full = np.einsum("kis,ks,kjs->kij", c, f, c.conj())
    rows, cols = np.triu_indices(n)
    order = np.lexsort((rows, cols))
    ref = full[:, rows[order], cols[order]]
    # state-major storage (secular_eigensystem's) and a plain [nk, V, ns]
    # tensor; host populations (the unpopulated tail not read) and device ones
    ct = torch.as_tensor(np.ascontiguousarray(c.transpose(0, 2, 1)), device="cuda")
    cases = [(ct.transpose(-2, -1), f), (torch.as_tensor(c, device="cuda"), f),
             (ct.transpose(-2, -1), torch.as_tensor(f, device="cuda"))]
    for cv, fv in cases:
        rho = charge.packed_density(cv, fv).cpu().numpy()
        got = rho[..., 0] + 1j * rho[..., 1]
        assert _rel(got, ref) < 1e-13
        diag = [q * (q + 1) // 2 + q for q in range(n)]
        assert np.all(rho[:, diag, 1] == 0.0)


@pytest.mark.gpu
def test_packed_density_of_no_occupied_state_is_zero():
    from imago_b200 import charge
    c = torch.ones((2, 9, 4), dtype=torch.complex128, device="cuda")
    rho = charge.packed_density(c, np.zeros((2, 4)))
    assert rho.shape == (2, 45, 2)
    assert torch.count_nonzero(rho).item() == 0


def test_packed_density_checks_its_arguments(imago_lib):
    # shape and type errors surface before any device work
    from imago_b200 import charge
    c = torch.zeros((2, 5, 3), dtype=torch.complex128)
    with pytest.raises(ValueError, match="population shape"):
        charge.packed_density(c, np.zeros((2, 4)))
    with pytest.raises(TypeError):
        charge.packed_density(c.to(torch.complex64), np.zeros((2, 3)))
