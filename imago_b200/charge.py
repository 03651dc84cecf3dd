"""The valence charge of one SCF step: the state populations and the
traces of the density matrix against the integral matrices.

    pop = populate_standard(eigenvalues, num_electrons)
    rho = valence_rho(out, eigenvalues, eigenvectors, pop["population"],
                      pot_coeffs)

populate_states is populateStates (populate.F90:150-620: the standard
population and the thermal smearing) in the library's host code
(imago_populate_states), over the sorted eigenvalues as in the reference.  valence_rho is the trace part of
makeValenceRho (valeCharge.F90:34-526): per k-point the density
rho = sum_j f_j c_j c_j^H of the occupied states (the library's packed
density kernel, imago_packed_density), packed like the integrals, and its
traces against
the packed OL, NP, KE, MV and every EP_j matrix by the library's trace
kernel (imago_packed_traces), which reads each integral matrix once from
HBM.  Energies in Hartree.
"""

import ctypes

import numpy as np
import torch

from . import intg

SMALL_THRESH = 1.0e-8      # smallThresh, constants.f90:49


def populate_states(eigenvalues, num_electrons, kpoint_weights=None, thermal_sigma=0.0,
                    max_thermal_range=0.0, fermi_search_limit=0.0):
    """populateStates (populate.F90:150-620) through imago_populate_states:
    populateStandard and, when thermal_sigma is not zero, populateSmearing,
    for eigenvalues [nk, spin, numStates] (energyEigenValues(state, k, spin)
    in the reference; Hartree).  Every state takes kPointWeight(k) / spin
    electrons in ascending energy until numElectrons are placed, the last
    one the remainder, and the states within smallThresh of that energy
    share the degenerate charge; with smearing, the Fermi level is bisected
    and each state takes its weight times the clipped Fermi function.
    kpoint_weights default to 2 / nk (the mesh weights, kpoints.f90:816);
    thermal_sigma and fermi_search_limit in Hartree (the reference divides
    its eV inputs by hartree, input.f90:369-383).  The XANES/ELNES core-hole
    correction (excitedQN_n) is not part of this step.  Returns
    {"population": [nk, spin, numStates], "occupied_energy" (the Fermi level
    when smearing), "occupied_index" (0-based, into the sorted list),
    "band_gap", "gap_kind" (0 metal, 1 direct, 2 indirect),
    "smearing_iterations"}."""
    e = np.ascontiguousarray(eigenvalues, dtype=np.float64)
    nk, spin, ns = e.shape
    kw = None if kpoint_weights is None else np.ascontiguousarray(kpoint_weights,
                                                                  dtype=np.float64)
    pop = np.zeros_like(e)
    info = np.zeros(5)
    L = intg.lib()
    L.imago_populate_states.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p] * 2 + \
        [ctypes.c_double] * 4 + [ctypes.c_void_p] * 2
    L.imago_populate_states.restype = ctypes.c_int
    dp = lambda a: None if a is None else a.ctypes.data
    rc = L.imago_populate_states(nk, spin, ns, dp(e), dp(kw), float(num_electrons),
                                 float(thermal_sigma), float(max_thermal_range),
                                 float(fermi_search_limit), dp(pop), dp(info))
    if rc == 8:
        raise ValueError("fewer states than electrons")
    if rc:
        raise intg.ImagoError(rc, "imago_populate_states")
    return {"population": pop, "occupied_energy": float(info[0]),
            "occupied_index": int(info[3]), "band_gap": float(info[1]),
            "gap_kind": int(info[2]), "smearing_iterations": int(info[4])}


def populate_standard(eigenvalues, num_electrons, kpoint_weights=None):
    """populateStandard (populate.F90:190-483): populate_states without
    thermal smearing."""
    return populate_states(eigenvalues, num_electrons, kpoint_weights)


def populate_smearing(eigenvalues, num_electrons, thermal_sigma, max_thermal_range,
                      fermi_search_limit, kpoint_weights=None):
    """populateSmearing (populate.F90:486-620) after populateStandard:
    {"population", "fermi_energy", "iterations", "charge"}."""
    if thermal_sigma == 0.0:
        raise ValueError("thermal_sigma must not be zero")
    r = populate_states(eigenvalues, num_electrons, kpoint_weights, thermal_sigma,
                        max_thermal_range, fermi_search_limit)
    return {"population": r["population"], "fermi_energy": r["occupied_energy"],
            "iterations": r["smearing_iterations"],
            "charge": float(r["population"].sum())}


def packed_density(eigenvectors, population):
    """rho = sum_j f_j c_j c_j^H per k-point (the zher updates of
    valeCharge.F90:187-192, in state order, the diagonal real) for
    eigenvectors [nk, V, numStates] (complex128, CUDA; state-major storage,
    as secular_eigensystem returns it, is read in place) and populations
    [nk, numStates], packed as packMatrix does (matrixSubs.F90:506-533):
    [nk, V(V+1)/2, 2], by imago_packed_density.  With host populations
    (numpy, as populate_states returns them) the states after the last one
    populated at any k-point are not read and the call does not wait for
    the device; device populations are used as they are (every state read,
    the unpopulated ones adding nothing)."""
    c = eigenvectors
    if c.dtype != torch.complex128:
        raise TypeError("eigenvectors must be complex128")
    nk, V, ns = c.shape
    ct = c.transpose(-2, -1)
    if not ct.is_contiguous():
        ct = ct.contiguous()
    shape = tuple(population.shape) if hasattr(population, "shape") else np.shape(population)
    if tuple(shape) != (nk, ns):
        raise ValueError(f"population shape {tuple(shape)} for {nk} k-points x {ns} states")
    if isinstance(population, torch.Tensor):
        f = population.to(device=c.device, dtype=torch.float64).contiguous()
        used = ns
    else:
        fh = np.ascontiguousarray(population, dtype=np.float64)
        occ = np.flatnonzero((fh != 0).any(axis=0))
        used = int(occ[-1]) + 1 if len(occ) else 0
        f = torch.from_numpy(fh).pin_memory().to(c.device, non_blocking=True)
    rho = torch.empty((nk, V * (V + 1) // 2, 2), dtype=torch.float64, device=c.device)
    L = intg.lib()
    L.imago_packed_density.argtypes = [ctypes.c_int] * 4 + [ctypes.c_void_p] * 4
    L.imago_packed_density.restype = ctypes.c_int
    rc = L.imago_packed_density(V, nk, ns, used, ct.data_ptr(), f.data_ptr(), rho.data_ptr(),
                                torch.cuda.current_stream().cuda_stream)
    if rc:
        raise intg.ImagoError(rc, "imago_packed_density")
    return rho


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
