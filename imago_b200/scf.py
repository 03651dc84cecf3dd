"""The SCF loop of Imago on the GPU: mainSCF (src/imago/imago.F90:420-540).

    result = run_scf(system, start_coeffs)

Every iteration runs, as the reference does:

  secularEqnSCF   H = NP + KE + sum_j potCoeffs_j EP_j and S = OL from the
                  device-resident integral builds, the Cholesky reduction,
                  the batched eigensolver and the back-transformation
                  (imago_b200.secular);
  populateStates  the populations (imago_populate_states, host);
  makeValenceRho  the density of the occupied states and its traces
                  against OL, NP, KE and every EP_j (imago_b200.charge);
  makeSCFPot      the charge fit, the electrostatic and exchange-correlation
                  potentials, the total energy, the Anderson mixing and the
                  convergence measure (imago_scf_pot_update, the mesh work
                  on the device).

The reference stops when the real-space change of the potential
(testableDelta) falls below CONVERGENCE_TEST or after LAST_ITERATION
iterations.  With `energy_tol` > 0 the run goes on until, besides that
test, the last two total energies agree within energy_tol Hartree: the SCF
"to 1e-6 Ha" this library is measured with (a deviation: the reference has
no energy test).  The energy test alone would stop runs whose small
Anderson steps change the energy by less than 1e-6 Ha while the potential
is still moving (the plain start of the 64-atom Si cell, 1e-5 Ha from its
fixed point); with energy_tol = 0 the reference's test alone decides.

`ScfSetup` wraps the C ABI of include/imago_scf.h: the set-up after the
integrals (lattice lists, exchange-correlation mesh, core charge,
electrostatic operators) and the per-iteration update.
"""

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np

from . import intg

_D = ctypes.POINTER(ctypes.c_double)


class ScfParamsC(ctypes.Structure):
    """Mirror of `imago_scf_params` in include/imago_scf.h."""
    _fields_ = [
        ("xc_code", ctypes.c_int),
        ("feedback_level", ctypes.c_int),
        ("relax_factor", ctypes.c_double),
        ("convergence_test", ctypes.c_double),
        ("num_sample_vectors", ctypes.c_int),
        ("ang_weights", ctypes.c_double * 2),
        ("r_sample", ctypes.c_double * 3),
        ("num_electrons", ctypes.c_double),
        ("covalent_radius", _D),
    ]


class ScfDimsC(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("pot_dim", "num_pot_types", "num_pot_sites",
                                             "num_cells_real", "num_cells_recip",
                                             "num_mesh_points")]


@dataclass
class ScfParams:
    """MAIN_INPUT_DATA and the exchange-correlation mesh of the control deck,
    with makeinput.py's defaults (src/scripts/makeinputrc.py: xc_code 100,
    50 iterations, convergence 1e-4, 100 sample vectors, weights 0.5/0.5,
    radial sampling 0.1/3.5/0.8; FEEDBACK_LEVEL 2 and RELAXATION_FACTOR 0.2 as
    makeinput.py writes them)."""
    xc_code: int = 100
    feedback_level: int = 2
    relax_factor: float = 0.2
    convergence_test: float = 1.0e-4
    last_iteration: int = 50
    num_sample_vectors: int = 100
    ang_weights: tuple = (0.5, 0.5)
    r_sample: tuple = (0.1, 3.5, 0.8)
    num_electrons: float = None        # default: the valence electrons of the sites
    num_states: int = None             # default: every valence state
    energy_tol: float = 1.0e-6         # also require |E_n - E_(n-1)| < energy_tol
    covalent_radius: list = field(default=None)


def valence_electrons(system):
    """NUM_ELECTRONS as makeinput.py counts it: nuclear charge less two
    electrons per core state, over the atom sites."""
    n = 0.0
    for t, z in zip(system.site_type, system.pot_site_type):
        at = system.atom_types[int(t) - 1]
        n += system.pot_types[int(z) - 1].nuc_charge - 2 * at.num_core_states
    return n


def _lib():
    L = intg.lib()
    if not hasattr(L, "_scf_ready"):
        vp = ctypes.c_void_p
        L.imago_scf_create.argtypes = [vp, ctypes.POINTER(ScfParamsC), ctypes.c_int, vp,
                                       ctypes.POINTER(vp)]
        L.imago_scf_create.restype = ctypes.c_int
        L.imago_scf_destroy.argtypes = [vp]
        L.imago_scf_destroy.restype = None
        L.imago_scf_get_dims.argtypes = [vp, ctypes.POINTER(ScfDimsC)]
        L.imago_scf_setup_arrays.argtypes = [vp] + [_D] * 9
        L.imago_scf_mesh.argtypes = [vp, ctypes.POINTER(ctypes.c_int), _D, _D]
        L.imago_scf_lattice.argtypes = [vp, _D, _D, _D, _D]
        L.imago_scf_pot_update.argtypes = [vp, _D, ctypes.c_double, ctypes.c_double, _D, _D]
        L.imago_scf_reset_history.argtypes = [vp]
        L.imago_scf_timings.argtypes = [vp, _D]
        L._scf_ready = True
    return L


def _p(a):
    return a.ctypes.data_as(_D)


class ScfSetup:
    """The SCF set-up of one system on one GPU and its potential update
    (include/imago_scf.h)."""

    def __init__(self, system, params=None, device=0, stream=None):
        self.params = params or ScfParams()
        p = self.params
        self.system = system
        self._cs, self._keep = system.to_c()
        cr = np.ascontiguousarray(
            p.covalent_radius if p.covalent_radius is not None
            else [t.covalent_radius for t in system.pot_types], dtype=np.float64)
        self._cr = cr
        ne = valence_electrons(system) if p.num_electrons is None else p.num_electrons
        self.num_electrons = float(ne)
        c = ScfParamsC(p.xc_code, p.feedback_level, p.relax_factor, p.convergence_test,
                       p.num_sample_vectors, (ctypes.c_double * 2)(*p.ang_weights),
                       (ctypes.c_double * 3)(*p.r_sample), self.num_electrons, _p(cr))
        self._ctx = ctypes.c_void_p()
        L = _lib()
        st = L.imago_scf_create(ctypes.byref(self._cs), ctypes.byref(c), device, stream,
                                ctypes.byref(self._ctx))
        if st:
            raise intg.ImagoError(st, "imago_scf_create")
        d = ScfDimsC()
        L.imago_scf_get_dims(self._ctx, ctypes.byref(d))
        self.pot_dim = d.pot_dim
        self.num_pot_types = d.num_pot_types
        self.num_pot_sites = d.num_pot_sites
        self.num_cells_real = d.num_cells_real
        self.num_cells_recip = d.num_cells_recip
        self.num_mesh_points = d.num_mesh_points

    def close(self):
        if self._ctx:
            _lib().imago_scf_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def setup_arrays(self):
        """The set-up datasets, named as the reference's arrays."""
        P, T = self.pot_dim, self.num_pot_types
        m = {k: np.zeros((P, P)) for k in ("potAlphaOverlap", "nonLocalNeutQPot",
                                            "localNeutQPot", "exchCorrOverlap")}
        v = {k: np.zeros(P) for k in ("nonLocalNucQPot", "localNucQPot",
                                      "coreChargeDensity", "intgConsts")}
        res = np.zeros((P, T))
        st = _lib().imago_scf_setup_arrays(
            self._ctx, _p(m["potAlphaOverlap"]), _p(m["nonLocalNeutQPot"]),
            _p(m["localNeutQPot"]), _p(v["nonLocalNucQPot"]), _p(v["localNucQPot"]), _p(res),
            _p(v["coreChargeDensity"]), _p(m["exchCorrOverlap"]), _p(v["intgConsts"]))
        if st:
            raise intg.ImagoError(st, "imago_scf_setup_arrays")
        # column-major (r, c) at [c][r]: transpose to row-major
        out = {k: a.T.copy() for k, a in m.items()}
        out.update(v)
        out["nonLocalResidualQ"] = res.T.copy()   # (numPotTypes, potDim)
        return out

    def mesh(self):
        """(numRayPoints per site, radialWeight [points], exchRhoOp
        [points, potDim])."""
        n = np.zeros(self.num_pot_sites, np.int32)
        w = np.zeros(self.num_mesh_points)
        op = np.zeros((self.num_mesh_points, self.pot_dim))
        st = _lib().imago_scf_mesh(self._ctx, n.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                   _p(w), _p(op))
        if st:
            raise intg.ImagoError(st, "imago_scf_mesh")
        return n, w, op

    def lattice(self):
        rd = np.zeros((self.num_cells_real, 3))
        rs = np.zeros(self.num_cells_real)
        gd = np.zeros((self.num_cells_recip, 3))
        gs = np.zeros(self.num_cells_recip)
        _lib().imago_scf_lattice(self._ctx, _p(rd), _p(rs), _p(gd), _p(gs))
        return rd, rs, gd, gs

    def pot_update(self, pot_rho, nuc_trace, kin_trace, coeffs):
        """makeSCFPot: returns (next coefficients, {totalEnergy,
        kineticEnergy, elecStatEnergy, exchCorrEnergy, electronDiff,
        testableDelta, converged, currIteration})."""
        c = np.ascontiguousarray(coeffs, dtype=np.float64).copy()
        pr = np.ascontiguousarray(pot_rho, dtype=np.float64)
        res = np.zeros(8)
        st = _lib().imago_scf_pot_update(self._ctx, _p(pr), float(nuc_trace), float(kin_trace),
                                         _p(c), _p(res))
        out = {"totalEnergy": res[0], "kineticEnergy": res[1], "elecStatEnergy": res[2],
               "exchCorrEnergy": res[3], "electronDiff": res[4]}
        if st:
            raise intg.ImagoError(st, "imago_scf_pot_update")
        out.update(testableDelta=res[5], converged=int(res[6]), currIteration=int(res[7]))
        return c, out

    def reset_history(self):
        _lib().imago_scf_reset_history(self._ctx)

    def timings(self):
        ms = np.zeros(3)
        _lib().imago_scf_timings(self._ctx, _p(ms))
        return {"electrostatics_ms": ms[0], "mesh_ms": ms[1], "update_ms": ms[2]}


def device_integrals(system, device=0, stream=None):
    """Build OL, KE, NP and every EP term into device memory (torch tensors)
    with imago_intg_build; returns (tensors, setup seconds)."""
    import torch
    t0 = time.perf_counter()
    dev = torch.device("cuda", device)
    with intg.IntegralSetup(system, device=device, outputs_on_device=True,
                            stream=stream) as g:
        nk, npk, V, C, P = g.nk, g.npacked, g.vale_dim, g.core_dim, g.pot_dim
        f64 = torch.float64
        bufs = {"ol_packed": torch.empty((nk, npk, 2), dtype=f64, device=dev),
                "ol_cv_re": torch.empty((nk, V, max(C, 1)), dtype=f64, device=dev),
                "ol_cv_im": torch.empty((nk, V, max(C, 1)), dtype=f64, device=dev),
                "ke_packed": torch.empty((nk, npk, 2), dtype=f64, device=dev),
                "np_packed": torch.empty((nk, npk, 2), dtype=f64, device=dev),
                "ep_packed": torch.empty((P, nk, npk, 2), dtype=f64, device=dev)}
        g.build(out={k: v.data_ptr() for k, v in bufs.items()})
    torch.cuda.synchronize(dev)
    return bufs, time.perf_counter() - t0


def run_scf(system, start_coeffs, params=None, device=0, integrals=None, setup=None,
            keep_history=False):
    """mainSCF on the GPU from the potential coefficients `start_coeffs`
    (initPotCoeffs' potCoeffs(:,1)).  `integrals` (device tensors from
    device_integrals) and `setup` (an ScfSetup) are built when not given.
    Returns a dict: energies (total energy per iteration), deltas
    (testableDelta), iterations, converged (the reference's test),
    energy_converged (the last two energies within energy_tol), done (both,
    or the reference's test alone with energy_tol = 0), pot_coeffs (the last used), timings (seconds: integrals,
    scf set-up, loop), and the last iteration's populations' Fermi level and
    gap."""
    import torch

    from . import charge, secular
    p = params or ScfParams()
    t_start = time.perf_counter()
    t_int = 0.0
    if integrals is None:
        integrals, t_int = device_integrals(system, device)
    t0 = time.perf_counter()
    own = setup is None
    if own:
        setup = ScfSetup(system, p, device)
    else:
        setup.reset_history()
    torch.cuda.synchronize(device)
    t_setup = time.perf_counter() - t0
    ne = setup.num_electrons
    out = {k: integrals[k] for k in ("np_packed", "ke_packed", "ep_packed", "ol_packed")}
    coeffs = np.asarray(start_coeffs, dtype=np.float64).copy()
    energies, deltas, history = [], [], []
    converged = energy_converged = False
    t1 = time.perf_counter()
    it = 0
    res = None
    while True:
        it += 1
        used = coeffs.copy()
        e, c = secular.secular_eigensystem(out, used, p.num_states)
        pop = charge.populate_standard(e.cpu().numpy()[:, None, :], ne)
        r = charge.valence_rho(out, [e], [c], pop["population"], used)
        try:
            coeffs, res = setup.pot_update(r["potRho"][:, 0], r["nucPotTrace"][0],
                                           r["kineticEnergyTrace"][0], used)
        except intg.ImagoError as err:
            if err.status != 9:
                raise
            res = None
            break
        energies.append(res["totalEnergy"])
        deltas.append(res["testableDelta"])
        history.append(used)
        converged = bool(res["converged"])
        energy_converged = len(energies) > 1 and \
            abs(energies[-1] - energies[-2]) < p.energy_tol
        done = converged and (p.energy_tol <= 0.0 or energy_converged)
        if done or it >= p.last_iteration:
            break
    torch.cuda.synchronize(device)
    t_loop = time.perf_counter() - t1
    if own:
        setup.close()
    return {"energies": energies, "deltas": deltas, "iterations": it,
            "converged": converged, "energy_converged": energy_converged,
            "done": bool(converged and (p.energy_tol <= 0.0 or energy_converged)),
            "positive_energy": res is None, "pot_coeffs": history[-1] if history else coeffs,
            "next_coeffs": coeffs, "fermi_energy": pop["occupied_energy"],
            "band_gap": pop["band_gap"],
            "timings": {"integrals_s": t_int, "setup_s": t_setup, "loop_s": t_loop,
                        "total_s": time.perf_counter() - t_start}}


_START = None


def atomic_start(system):
    """initPotCoeffs' plain start: the atomic-superposition potential of
    each potential type's element (imago_b200/data/initial_potentials.json,
    the database potentials projected onto these exponents), concatenated
    in potential-term order."""
    import json
    import os
    global _START
    if _START is None:
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                            "initial_potentials.json")
        with open(path) as fh:
            _START = json.load(fh)["potentials"]
    out = []
    for p in system.pot_types:
        for e in _START:
            a = np.asarray(e["alphas"])
            if int(e["z"]) == int(round(p.nuc_charge)) and len(a) == len(p.alphas) and \
                    np.allclose(a, p.alphas, rtol=1e-12):
                out.append(np.asarray(e["coeffs"]))
                break
        else:
            raise ValueError(f"no starting potential for Z={p.nuc_charge} with "
                             f"{len(p.alphas)} terms {p.alphas[0]}..{p.alphas[-1]}")
    return np.concatenate(out)
