"""The valence charge of one SCF step: the state populations and the
traces of the density matrix against the integral matrices.

    pop = populate_standard(eigenvalues, num_electrons)
    rho = valence_rho(out, eigenvalues, eigenvectors, pop["population"],
                      pot_coeffs)

populate_standard is populateStandard (populate.F90:190-483, the
population without thermal smearing): host work over the sorted
eigenvalues, as in the reference.  valence_rho is the trace part of
makeValenceRho (valeCharge.F90:34-526): per k-point the density
rho = sum_j f_j c_j c_j^H of the occupied states (a batched complex GEMM,
cuBLAS through torch), packed like the integrals, and its traces against
the packed OL, NP, KE, MV and every EP_j matrix by the library's trace
kernel (imago_packed_traces), which reads each integral matrix once from
HBM.  Energies in Hartree.
"""

import ctypes

import numpy as np
import torch

from . import intg

SMALL_THRESH = 1.0e-8      # smallThresh, constants.f90:49
METAL_GAP_THRESH = 1.0e-3  # populate.F90 metalGapThresh


def populate_standard(eigenvalues, num_electrons, kpoint_weights=None):
    """populateStandard (populate.F90:190-483) for eigenvalues [nk, spin,
    numStates] (energyEigenValues(state, k, spin) in the reference).  Every
    state takes kPointWeight(k) / spin electrons in ascending energy until
    numElectrons are placed, the last one the remainder; the states within
    smallThresh of that energy then share the degenerate charge in
    proportion to their weights.  kpoint_weights default to 2 / nk (the
    mesh weights, kpoints.f90:816).  Returns {"population": [nk, spin,
    numStates], "occupied_energy", "occupied_index" (0-based, into the
    sorted list), "band_gap", "gap_kind" (0 metal, 1 direct, 2 indirect)}."""
    e = np.asarray(eigenvalues, dtype=np.float64)
    nk, spin, ns = e.shape
    kw = (np.full(nk, 2.0 / nk) if kpoint_weights is None
          else np.asarray(kpoint_weights, dtype=np.float64))
    flat = e.reshape(-1)        # (k, spin, state), state fastest
    n = flat.size
    order = np.argsort(flat, kind="stable")
    srt = flat[order]
    w = kw[order // (ns * spin)] / float(spin)
    ne = float(num_electrons)
    pop = np.zeros(n)
    # the running total, added in the reference's order
    run = np.cumsum(w)
    hit = np.nonzero((run > ne) | (np.abs(ne - run) < SMALL_THRESH))[0]
    if hit.size == 0:
        raise ValueError("fewer states than electrons")
    occ = int(hit[0])
    pop[order[:occ + 1]] = w[:occ + 1]
    if run[occ] > ne:
        pop[order[occ]] = w[occ] + ne - run[occ]
    occ_e = srt[occ]
    lo = hi = occ
    degen = pop[order[occ]]
    possible = w[occ]
    while hi + 1 < n and abs(occ_e - srt[hi + 1]) <= SMALL_THRESH:
        hi += 1
        possible += w[hi]
    while lo > 0 and abs(occ_e - srt[lo - 1]) <= SMALL_THRESH:
        lo -= 1
        possible += w[lo]
        degen += w[lo]
    pop[order[lo:hi + 1]] = degen / possible * w[lo:hi + 1]
    occ = hi
    occ_e = srt[occ]
    gap, kind = 0.0, 0
    if occ < n - 1:
        gap = srt[occ + 1] - srt[occ]
        if gap <= METAL_GAP_THRESH:
            gap = 0.0
        else:
            vbm, cbm = order[occ] // (ns * spin), order[occ + 1] // (ns * spin)
            kind = 1 if vbm == cbm else 2
    return {"population": pop.reshape(nk, spin, ns), "occupied_energy": float(occ_e),
            "occupied_index": occ, "band_gap": float(gap), "gap_kind": kind}


def step_function(x, step_range):
    """stepFunction (mathSubs.f90:164-185): 0 above the range, 1 below it,
    the Fermi function 1 / (1 + e^x) between."""
    x = np.asarray(x, dtype=np.float64)
    with np.errstate(over="ignore"):
        f = 1.0 / (1.0 + np.exp(np.minimum(x, step_range)))
    return np.where(x > step_range, 0.0, np.where(x < -step_range, 1.0, f))


def populate_smearing(eigenvalues, num_electrons, thermal_sigma, max_thermal_range,
                      fermi_search_limit, kpoint_weights=None, standard=None):
    """populateSmearing (populate.F90:486-620): the Fermi level bisected
    (at most 500 steps) between the standard population's highest occupied
    state minus fermi_search_limit and the next state plus it, every state
    taking weight x stepFunction((E - E_F) / thermal_sigma,
    max_thermal_range) until the charge is within smallThresh of
    numElectrons.  Energies in Hartree (the reference divides its eV inputs
    by hartree, input.f90:369-383).  `standard` is populate_standard's
    result for the same arguments (computed when absent).  Returns
    {"population", "fermi_energy", "iterations", "charge"}."""
    e = np.asarray(eigenvalues, dtype=np.float64)
    nk, spin, ns = e.shape
    if standard is None:
        standard = populate_standard(e, num_electrons, kpoint_weights)
    kw = (np.full(nk, 2.0 / nk) if kpoint_weights is None
          else np.asarray(kpoint_weights, dtype=np.float64))
    flat = e.reshape(-1)
    order = np.argsort(flat, kind="stable")
    srt = flat[order]
    w = kw[order // (ns * spin)] / float(spin)
    occ = standard["occupied_index"]
    lo = srt[occ] - fermi_search_limit
    hi = srt[min(occ + 1, srt.size - 1)] + fermi_search_limit
    ne = float(num_electrons)
    pop = np.zeros(srt.size)
    ef, charge, it = 0.5 * (lo + hi), 0.0, 0
    for it in range(1, 501):
        ef = 0.5 * (lo + hi)
        f = step_function((srt - ef) / thermal_sigma, max_thermal_range)
        p = w * f
        # the reference's loop stops at the first state the step function
        # zeroes; the energies ascend, so every later one is zero too
        charge = float(np.cumsum(p)[-1])
        pop = np.zeros(srt.size)
        pop[order] = p
        if abs(charge - ne) < SMALL_THRESH:
            break
        if charge < ne:
            lo = ef
        else:
            hi = ef
    return {"population": pop.reshape(nk, spin, ns), "fermi_energy": float(ef),
            "iterations": it, "charge": charge}


def populate_states(eigenvalues, num_electrons, kpoint_weights=None, thermal_sigma=0.0,
                    max_thermal_range=0.0, fermi_search_limit=0.0):
    """populateStates (populate.F90:150-187): the standard population, then
    the thermal smearing when thermal_sigma is not zero.  The XANES/ELNES
    core-hole correction (excitedQN_n) is not part of this step."""
    std = populate_standard(eigenvalues, num_electrons, kpoint_weights)
    if thermal_sigma == 0.0:
        return std
    sm = populate_smearing(eigenvalues, num_electrons, thermal_sigma, max_thermal_range,
                           fermi_search_limit, kpoint_weights, standard=std)
    out = dict(std)
    out["population"] = sm["population"]
    out["occupied_energy"] = sm["fermi_energy"]
    out["smearing_iterations"] = sm["iterations"]
    return out


_PACK_CACHE = {}


def _pack_index(V, device):
    key = (V, str(device))
    if key not in _PACK_CACHE:
        cols = torch.repeat_interleave(torch.arange(V), torch.arange(1, V + 1))
        starts = cols * (cols + 1) // 2
        rows = torch.arange(V * (V + 1) // 2) - starts
        _PACK_CACHE[key] = (rows.to(device), cols.to(device))
    return _PACK_CACHE[key]


def packed_density(eigenvectors, population):
    """rho = sum_j f_j c_j c_j^H per k-point (the zher updates of
    valeCharge.F90:187-192) for populations [nk, numStates], packed as
    packMatrix does (matrixSubs.F90:506-533): [nk, V(V+1)/2, 2]."""
    c = eigenvectors
    f = torch.as_tensor(population, dtype=torch.float64, device=c.device)
    full = (c * f[:, None, :].to(c.dtype)) @ c.mH
    rows, cols = _pack_index(c.shape[1], c.device)
    return torch.view_as_real(full[:, rows, cols].contiguous()).contiguous()


def packed_traces(mats, rho, nk, V):
    """imago_packed_traces: [nmat, nrho] traces of packed matrices
    [nmat, nk, nPacked, 2] against packed densities [nrho, nk, nPacked, 2],
    both CUDA float64."""
    mats = mats.contiguous()
    rho = rho.contiguous()
    nmat, nrho = mats.shape[0], rho.shape[0]
    out = torch.empty((nmat, nrho), dtype=torch.float64, device=rho.device)
    L = intg.lib()
    L.imago_packed_traces.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p, ctypes.c_int] + \
        [ctypes.c_void_p] * 3
    L.imago_packed_traces.restype = ctypes.c_int
    rc = L.imago_packed_traces(V, nk, nmat, mats.data_ptr(), nrho, rho.data_ptr(),
                               out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    if rc:
        raise intg.ImagoError(rc, "imago_packed_traces")
    return out


def valence_rho(out, eigenvalues, eigenvectors, population, pot_coeffs, rel=False):
    """The traces of makeValenceRho (valeCharge.F90:218-291) and its energy
    sums (valeCharge.F90:427-488).

    out: the device-resident packed matrices of the step (ol_packed,
    np_packed, ke_packed, ep_packed, and mv_packed when rel);
    eigenvalues [spin][nk, numStates] and eigenvectors [spin][nk, V,
    numStates] (CUDA tensors, one entry per spin); population [nk, spin,
    numStates] from populate_standard; pot_coeffs [potDim] or [potDim,
    spin].  For spin 2 the traces are taken against the total and the
    difference densities, as the reference forms them.  Returns numpy
    arrays named as the reference's variables: chargeDensityTrace,
    nucPotTrace, kineticEnergyTrace, massVelocityTrace (rel), potRho
    [potDim, spin], electronEnergy and sumElecEnergy [spin]."""
    spin = len(eigenvectors)
    pop = np.asarray(population, dtype=np.float64)
    # a state whose populations over the spins sum below smallThresh is
    # skipped (valeCharge.F90:181-183)
    pop = np.where((np.abs(pop).sum(axis=1) < SMALL_THRESH)[:, None, :], 0.0, pop)
    nk, V = eigenvectors[0].shape[0], eigenvectors[0].shape[1]
    rho = torch.stack([packed_density(eigenvectors[s], pop[:, s, :]) for s in range(spin)])
    if spin == 2:
        rho = torch.stack([rho[0] + rho[1], rho[0] - rho[1]])
    res = {}
    one = lambda key: packed_traces(out[key][None], rho, nk, V)[0].cpu().numpy()
    res["chargeDensityTrace"] = one("ol_packed")
    res["nucPotTrace"] = one("np_packed")
    res["kineticEnergyTrace"] = one("ke_packed")
    if rel:
        res["massVelocityTrace"] = one("mv_packed")
    res["potRho"] = packed_traces(out["ep_packed"], rho, nk, V).cpu().numpy()
    res["electronEnergy"] = np.array(
        [float((pop[:, s, :] * eigenvalues[s].cpu().numpy()).sum()) for s in range(spin)])
    w = np.asarray(pot_coeffs, dtype=np.float64).reshape(res["potRho"].shape[0], -1)
    ke, nuc, pr = res["kineticEnergyTrace"], res["nucPotTrace"], res["potRho"]
    mv = res.get("massVelocityTrace", np.zeros(spin))
    if spin == 1:
        res["sumElecEnergy"] = np.array([float((w[:, 0] * pr[:, 0]).sum() + ke[0] + mv[0]
                                               + nuc[0])])
    else:
        up = 0.5 * ((w[:, 0] * (pr[:, 0] + pr[:, 1])).sum() + ke[0] + ke[1] + mv[0] + mv[1]
                    + nuc[0] + nuc[1])
        dn = 0.5 * ((w[:, 1] * (pr[:, 0] - pr[:, 1])).sum() + ke[0] - ke[1] + mv[0] - mv[1]
                    + nuc[0] - nuc[1])
        res["sumElecEnergy"] = np.array([up, dn])
    return res
