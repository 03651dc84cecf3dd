"""The secular equation of one SCF step, on the GPU, from the integral
builds (secularEqnSCF, src/imago/secularEqn.F90:37-330).

    eigenvalues = secular_eigenvalues(out, pot_coeffs)

`out` holds the device-resident packed matrices of an IntegralSetup build
(np_packed, ke_packed, ep_packed, ol_packed as CUDA tensors); pot_coeffs are
the potDim coefficients of the current SCF potential (potCoeffs in the
reference).  H and S are assembled and unpacked on the device by
imago_secular_matrices, then the generalised Hermitian problem
H c = E S c, which the reference hands to LAPACK zhegv(1, 'V', 'U')
(interfaces.F90:73-120), is reduced by the Cholesky factor of S and the
eigenvalues of the reduced matrices come from the library's batched Jacobi
kernel or cuSOLVER's batched solver (set_eigensolver).  Up to n = 128 the
reduction and the back-transformation of the vectors are the library's own
kernels (imago_secular_reduce / _back, one CTA per k-point); beyond,
cuSOLVER through torch.linalg.  Eigenvalues come back ascending per
k-point, in Hartree.
"""

import ctypes

import torch

from . import intg


def secular_matrices(out, pot_coeffs, stream=None):
    """Full Hermitian H and S [nk, V, V] (complex128, CUDA) for every k;
    with out["mv_packed"] (a scalar-relativistic run) H includes the mass
    velocity, added after KE as the reference does."""
    h, s = _secular_storage(out, pot_coeffs, stream)
    # stored [k][col][row]: the matrix is the transpose of each slice
    return h.transpose(-2, -1), s.transpose(-2, -1)


def _secular_storage(out, pot_coeffs, stream=None):
    """H and S as imago_secular_matrices_rel writes them: contiguous
    [nk, V, V], column-major per k-point."""
    npk = out["np_packed"]
    nk, npacked = npk.shape[0], npk.shape[1]
    V = int((int((8 * npacked + 1) ** 0.5) - 1) // 2)
    if V * (V + 1) // 2 != npacked:
        raise ValueError("packed length is not V(V+1)/2")
    ep = out.get("ep_packed")
    P = 0 if ep is None else ep.shape[0]
    w = torch.as_tensor(pot_coeffs, dtype=torch.float64, device=npk.device).contiguous()
    if w.numel() != P:
        raise ValueError(f"{w.numel()} coefficients for {P} potential terms")
    h = torch.empty((nk, V, V), dtype=torch.complex128, device=npk.device)
    s = torch.empty_like(h)
    mv = out.get("mv_packed")
    L = intg.lib()
    L.imago_secular_matrices_rel.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p] * 9
    L.imago_secular_matrices_rel.restype = ctypes.c_int
    st = torch.cuda.current_stream().cuda_stream if stream is None else stream
    rc = L.imago_secular_matrices_rel(
        V, nk, P, npk.data_ptr(), out["ke_packed"].data_ptr(),
        mv.data_ptr() if mv is not None else None,
        ep.data_ptr() if P else None, w.data_ptr() if P else None,
        out["ol_packed"].data_ptr(), h.data_ptr(), s.data_ptr(), st)
    if rc:
        raise intg.ImagoError(rc, "imago_secular_matrices_rel")
    return h, s


REDUCE_MAX_N = 128


def cholesky_reduce(h_store, s_store, factor=False):
    """imago_secular_reduce: A = L^-1 H L^-H [nk, n, n] (row-major,
    complex128) with S = L L^H, from H and S stored column-major per k-point
    (_secular_storage); with factor, also L packed by columns [nk,
    n(n+1)/2] for back_transform.  Raises ValueError, as zhegv stops, when S
    of some k-point is not positive definite."""
    nk, n = h_store.shape[0], h_store.shape[-1]
    a = torch.empty_like(h_store)
    lfac = (torch.empty((nk, n * (n + 1) // 2), dtype=torch.complex128, device=h_store.device)
            if factor else None)
    info = torch.zeros(nk, dtype=torch.int32, device=h_store.device)
    L = intg.lib()
    L.imago_secular_reduce.argtypes = [ctypes.c_int] * 2 + [ctypes.c_void_p] * 6
    L.imago_secular_reduce.restype = ctypes.c_int
    rc = L.imago_secular_reduce(n, nk, h_store.data_ptr(), s_store.data_ptr(), a.data_ptr(),
                                lfac.data_ptr() if factor else None, info.data_ptr(),
                                torch.cuda.current_stream().cuda_stream)
    if rc:
        raise intg.ImagoError(rc, "imago_secular_reduce")
    return a, lfac, info


def _check_info(info):
    bad = torch.nonzero(info).flatten()
    if bad.numel():
        k = int(bad[0])
        raise ValueError(f"overlap matrix of k-point {k} is not positive definite "
                         f"(leading minor {int(info[k])})")


def back_transform(lfac, vec, num_states):
    """imago_secular_back: c = L^-H y for the first num_states columns of vec
    [nk, n, n] (hermitian_eigh's eigenvectors); returns [nk, n, num_states]
    as a view of state-major storage [nk, num_states, n]."""
    nk, n = vec.shape[0], vec.shape[-1]
    ct = torch.empty((nk, num_states, n), dtype=torch.complex128, device=vec.device)
    L = intg.lib()
    L.imago_secular_back.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p] * 4
    L.imago_secular_back.restype = ctypes.c_int
    rc = L.imago_secular_back(n, nk, num_states, lfac.data_ptr(), vec.contiguous().data_ptr(),
                              ct.data_ptr(), torch.cuda.current_stream().cuda_stream)
    if rc:
        raise intg.ImagoError(rc, "imago_secular_back")
    return ct.transpose(-2, -1)


JACOBI_MAX_N = 112
_ERR_RANGE = 8  # IMAGO_ERR_RANGE
_SOLVERS = {"auto": 0, "jacobi": 1, "batched": 2}


def set_eigensolver(name):
    """The solver behind hermitian_eigvals / hermitian_eigh for the whole
    process (imago_hermitian_set_solver): "auto" (the default) cuSOLVER's
    batched Hermitian solver where it loads, else the library's Jacobi
    kernel; "jacobi" the Jacobi kernel up to n = 112; "batched" the batched
    solver only."""
    L = intg.lib()
    L.imago_hermitian_set_solver.argtypes = [ctypes.c_int]
    L.imago_hermitian_set_solver.restype = ctypes.c_int
    if name not in _SOLVERS:
        raise ValueError(f"eigensolver must be one of {sorted(_SOLVERS)}")
    rc = L.imago_hermitian_set_solver(_SOLVERS[name])
    if rc:
        raise intg.ImagoError(rc, "imago_hermitian_set_solver")


def eigensolver():
    """The name set by set_eigensolver."""
    L = intg.lib()
    L.imago_hermitian_solver.argtypes = [ctypes.c_void_p]
    L.imago_hermitian_solver.restype = ctypes.c_int
    m = ctypes.c_int(0)
    rc = L.imago_hermitian_solver(ctypes.byref(m))
    if rc:
        raise intg.ImagoError(rc, "imago_hermitian_solver")
    return {v: k for k, v in _SOLVERS.items()}[m.value]


def hermitian_eigvals(a):
    """Ascending eigenvalues of a batch of Hermitian matrices [b, n, n]
    (complex128, CUDA): imago_hermitian_eigvals, cuSOLVER's batched solver
    through the library or the library's Jacobi kernel (one CTA per matrix,
    cyclic Jacobi in shared memory, n up to 112) as set_eigensolver chooses
    (torch's eigvalsh beyond n = 112 if the batched solver is absent)."""
    b, n = a.shape[0], a.shape[-1]
    a = a.contiguous()
    w = torch.empty((b, n), dtype=torch.float64, device=a.device)
    L = intg.lib()
    L.imago_hermitian_eigvals.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p]
    L.imago_hermitian_eigvals.restype = ctypes.c_int
    rc = L.imago_hermitian_eigvals(n, b, a.data_ptr(), w.data_ptr(),
                                   torch.cuda.current_stream().cuda_stream)
    if rc == _ERR_RANGE and n > JACOBI_MAX_N:  # no batched cuSOLVER in the process
        return torch.linalg.eigvalsh(a)
    if rc:
        raise intg.ImagoError(rc, "imago_hermitian_eigvals")
    return w


_EIGH_LANES = 8
_EIGH_POOL = None
_EIGH_STREAMS = {}


def _eigh_lanes(a):
    """torch.linalg.eigh (cuSOLVER syevd) of each matrix of the batch, the
    matrices dealt to _EIGH_LANES host threads with a CUDA stream each:
    syevd synchronises with the host inside every call, so one stream runs
    the batch one matrix at a time.  Measured on one B200 for 64 matrices:
    n = 832 743 -> 577 ms, n = 256 190 -> 124 ms, n = 208 161 -> 102 ms."""
    global _EIGH_POOL
    import concurrent.futures
    b = a.shape[0]
    lanes = min(_EIGH_LANES, b)
    dev = a.device
    if _EIGH_POOL is None:
        _EIGH_POOL = concurrent.futures.ThreadPoolExecutor(_EIGH_LANES)
    streams = _EIGH_STREAMS.setdefault(dev, [torch.cuda.Stream(dev)
                                             for _ in range(_EIGH_LANES)])
    w = torch.empty(a.shape[:-1], dtype=torch.float64, device=dev)
    v = torch.empty_like(a)
    cur = torch.cuda.current_stream(dev)
    ready = torch.cuda.Event()
    ready.record(cur)

    def lane(i):
        st = streams[i]
        st.wait_event(ready)
        with torch.cuda.device(dev), torch.cuda.stream(st):
            for j in range(i, b, lanes):
                wj, vj = torch.linalg.eigh(a[j])
                w[j].copy_(wj)
                v[j].copy_(vj)

    list(_EIGH_POOL.map(lane, range(lanes)))
    for st in streams[:lanes]:
        cur.wait_stream(st)
    return w, v


def hermitian_eigh(a):
    """Ascending eigenvalues [b, n] and unit eigenvectors [b, n, n] (in
    columns) of a batch of Hermitian matrices [b, n, n] (complex128, CUDA):
    imago_hermitian_eigh, cuSOLVER's batched solver through the library (one
    call for the batch) or the Jacobi kernel accumulating its rotations (n
    up to 112) as set_eigensolver chooses; _eigh_lanes beyond n = 112 if the
    process has no batched solver."""
    b, n = a.shape[0], a.shape[-1]
    a = a.contiguous()
    w = torch.empty((b, n), dtype=torch.float64, device=a.device)
    v = torch.empty((b, n, n), dtype=torch.complex128, device=a.device)
    L = intg.lib()
    L.imago_hermitian_eigh.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 4
    L.imago_hermitian_eigh.restype = ctypes.c_int
    rc = L.imago_hermitian_eigh(n, b, a.data_ptr(), w.data_ptr(), v.data_ptr(),
                                torch.cuda.current_stream().cuda_stream)
    if rc == _ERR_RANGE and n > JACOBI_MAX_N:  # no batched cuSOLVER in the process
        return _eigh_lanes(a) if b > 1 else torch.linalg.eigh(a)
    if rc:
        raise intg.ImagoError(rc, "imago_hermitian_eigh")
    return w, v


def secular_eigenvalues(out, pot_coeffs, num_states=None):
    """Eigenvalues of H c = E S c per k-point, ascending, [nk, num_states]:
    the Cholesky factor L of S, A = L^-1 H L^-H (cholesky_reduce up to n =
    128, cuSOLVER through torch.linalg beyond), and the eigenvalues of A
    (hermitian_eigvals)."""
    hs, ss = _secular_storage(out, pot_coeffs)
    if hs.shape[-1] <= REDUCE_MAX_N:
        a, _, info = cholesky_reduce(hs, ss)
        ev = hermitian_eigvals(a)
        _check_info(info)
    else:
        h, s = hs.transpose(-2, -1), ss.transpose(-2, -1)
        lo = torch.linalg.cholesky(s)
        y = torch.linalg.solve_triangular(lo, h, upper=False)          # L^-1 H
        a = torch.linalg.solve_triangular(lo, y.mH, upper=False)       # L^-1 H L^-H
        ev = hermitian_eigvals(a)
    return ev if num_states is None else ev[:, :num_states]


def secular_eigensystem(out, pot_coeffs, num_states=None):
    """Eigenvalues [nk, num_states] (ascending) and eigenvectors
    [nk, V, num_states] of H c = E S c per k-point, the vectors normalised
    as zhegv(1, 'V', 'U') returns them (c^H S c = 1): A = L^-1 H L^-H is
    diagonalised by hermitian_eigh and the vectors taken back by
    c = L^-H y (cholesky_reduce and back_transform up to n = 128, the
    vectors then a view of state-major storage; cuSOLVER through
    torch.linalg beyond)."""
    hs, ss = _secular_storage(out, pot_coeffs)
    n = hs.shape[-1]
    if n <= REDUCE_MAX_N:
        a, lfac, info = cholesky_reduce(hs, ss, factor=True)
        ev, vec = hermitian_eigh(a)
        ns = n if num_states is None else num_states
        c = back_transform(lfac, vec, ns)
        _check_info(info)
        return ev[:, :ns], c
    h, s = hs.transpose(-2, -1), ss.transpose(-2, -1)
    lo = torch.linalg.cholesky(s)
    y = torch.linalg.solve_triangular(lo, h, upper=False)
    a = torch.linalg.solve_triangular(lo, y.mH, upper=False)
    ev, vec = hermitian_eigh(a)
    c = torch.linalg.solve_triangular(lo.mH, vec, upper=True)
    if num_states is not None:
        ev, c = ev[:, :num_states], c[:, :, :num_states]
    return ev, c
