"""Golden integral matrices made by executing the reference's own integral
driver (tests/golden/fortran_exec.py), end to end: the lattice, the k-points
and phase factors, the basis renormalisation, the screening tables, the
pair / image / alpha-pair loops, the contraction, the Bloch phases, the
origin shift, the block savers, the core orthogonalisation and the packing.

Executed from src/imago, statement for statement:

  lattice.f90          getRecipCellVectors, setCutoffThresh, initializeLattice
                       (getNumCells, makeLattice, cellBorderCheck; sortSubs'
                       mergeSort)
  kpoints.f90          convertKPointsToXYZ, computePhaseFactors
  basis.f90            renormalizeBasis, initializeAtomSite, initializePotSite
  gaussRelations.f90   makeAlphaDist, makeAlphaNucDist, makeAlphaPotDist
  integrals.F90        gaussOverlapOL, orthoOL, gaussOverlapKE, gaussOverlapNP,
                       nuclearPE, elecPotGaussOverlap, gaussOverlapEP,
                       electronicPE, checkElecPotInteraction, ortho
  intgSaving.F90       multWithBasisFn1, applyPhaseFactors,
                       kPointLatticeOriginShift, saveCurrentPair and its
                       block savers
  intgOrtho.F90        valeCoreCoreValeOL, valeCoreCoreVale, coreValeCoreCore,
                       makeValeVale
  gaussIntegrals.f90   overlap2CIntg, kinetic2CIntg, nuclear3CIntg,
                       electron3CIntg (through make_golden.py's transliteration)

Supplied by this script: the module data of the synthetic systems
(imago_b200.configs), findLatticeVector (a nearest lattice vector; the
image loop covers the whole sphere around it, so which of two equidistant
vectors is used only reorders terms), the HDF5 writes (a dictionary), and
LAPACK's zherk / zher2k (their definitions on the upper triangle in numpy,
the diagonal's imaginary part set to zero as the routines specify).

Fixture: driver_diamond.npz, the diamond primitive cell at 2x2x2 k: the
packed OL, KE, NP and every EP term per k-point and coreValeOL, as the
reference hands them to HDF5.

Run where the reference is mounted:

    python tests/golden/make_driver_golden.py <root of the reference checkout>
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)

import fortran_exec as fe  # noqa: E402
import make_golden  # noqa: E402
import make_scf_golden as msg  # noqa: E402


def zherk(uplo, trans, n, k, alpha, A, lda, beta, C, ldc):
    """C := alpha A^H A + beta C on the upper triangle (uplo 'U', trans 'C');
    the diagonal comes out real."""
    a = np.asarray(fe._val(A))[:k, :n]
    c = fe._val(C)
    upd = alpha * (a.conj().T @ a) + beta * c[:n, :n]
    iu = np.triu_indices(n)
    c[:n, :n][iu] = upd[iu]
    d = np.arange(n)
    c[d, d] = c[d, d].real
    return ()


def zher2k(uplo, trans, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
    """C := alpha A^H B + conj(alpha) B^H A + beta C on the upper triangle
    (uplo 'U', trans 'C'); the diagonal comes out real."""
    a = np.asarray(fe._val(A))[:k, :n]
    b = np.asarray(fe._val(B))[:k, :n]
    c = fe._val(C)
    upd = alpha * (a.conj().T @ b) + np.conj(alpha) * (b.conj().T @ a) + beta * c[:n, :n]
    iu = np.triu_indices(n)
    c[:n, :n][iu] = upd[iu]
    d = np.arange(n)
    c[d, d] = c[d, d].real
    return ()


def kernel_hook(kns, name):
    """overlap2CIntg / kinetic2CIntg(a1, a2, A, B, code, sh) through the
    transliterated generated kernel."""
    def call(a1, a2, A, B, code, sh):
        f = make_golden.FArr("sh", [16, 16])
        kns[name](float(a1), float(a2), np.array(fe._val(A), float),
                  np.array(fe._val(B), float), int(code), f)
        out = fe._val(sh)
        out[...] = 0.0
        for (i, j), v in f.d.items():
            out[i - 1, j - 1] = v
        return ()
    return call


def kernel3c_hook(kns, name):
    """nuclear3CIntg / electron3CIntg(a1, a2, a3, A, B, C, code, sh) through
    the transliterated generated kernel."""
    def call(a1, a2, a3, A, B, C, code, sh):
        f = make_golden.FArr("sh", [16, 16])
        kns[name](float(a1), float(a2), float(a3), np.array(fe._val(A), float),
                  np.array(fe._val(B), float), np.array(fe._val(C), float), int(code), f)
        out = fe._val(sh)
        out[...] = 0.0
        for (i, j), v in f.d.items():
            out[i - 1, j - 1] = v
        return ()
    return call


def module_state(s, store, kns):
    ns = msg.module_state(s, store, 20)
    # atom sites and types (atomicSites.f90, atomicTypes.f90)
    ats = []
    for t in s.atom_types:
        nc, nv = len(t.core_l), len(t.vale_l)
        na = t.num_orb_alphas[0]
        cr = np.zeros((na, max(nc, 1)))
        vr = np.zeros((na, max(nv, 1)))
        for k, c in enumerate(t.core_coeffs):
            cr[:len(c), k] = c
        for k, c in enumerate(t.vale_coeffs):
            vr[:len(c), k] = c
        ats.append(fe.Obj(elementid=t.element, numorbalphas=fe.Arr.of(t.num_orb_alphas, np.int64),
                          alphas=fe.Arr.of(t.alphas), numcorestates=t.num_core_states,
                          numvalestates=t.num_vale_states, numcoreradialfns=nc,
                          numvaleradialfns=nv,
                          coreqn_llist=fe.Arr.of(list(t.core_l) or [0], np.int64),
                          valeqn_llist=fe.Arr.of(list(t.vale_l) or [0], np.int64),
                          coreradialfns=fe.Arr.of(cr), valeradialfns=fe.Arr.of(vr)))
    ns["atomtypes"] = msg.objs(ats)
    ns["numatomtypes"] = len(ats)
    ns["numelements"] = max(t.element for t in s.atom_types)
    ns["maxnumatomalphas"] = max(t.num_orb_alphas[0] for t in s.atom_types)
    ns["maxnumstates"] = max(t.num_core_states + t.num_vale_states for t in s.atom_types)
    sites = []
    cv = cc = 0
    for t, pos in zip(s.site_type, s.site_pos):
        at = s.atom_types[int(t) - 1]
        sites.append(fe.Obj(atomtypeassn=int(t), cartpos=fe.Arr.of(pos), cumulvalestates=cv,
                            cumulcorestates=cc))
        cv += at.num_vale_states
        cc += at.num_core_states
    ns["atomsites"] = msg.objs(sites)
    ns["numatomsites"] = len(sites)
    ns["valedim"], ns["coredim"] = cv, cc
    nk = len(s.kpoints_abc)
    ns["numkpoints"] = nk
    ns["kpoints"] = fe.Arr.of(np.asarray(s.kpoints_abc, float).T)
    for v in ("lmindex", "lmalphaindex", "basis", "phasefactor", "alphadist", "alphacenter",
              "numelementatomicalphas", "elementatomicalphas"):
        ns[v] = None
    V, C = cv, max(cc, 1)
    ns["valevale"] = fe.Arr((V, V, nk), complex)
    ns["corevaleol"] = fe.Arr((C, V, nk), complex)
    ns["corecore"] = fe.Arr((C, C, nk), complex)
    ns["corevale"] = None
    ns["valecore"] = None
    ns.update(zherk=zherk, zher2k=zher2k, overlap2cintg=kernel_hook(kns, "overlap2CIntg"),
              kinetic2cintg=kernel_hook(kns, "kinetic2CIntg"),
              nuclear3cintg=kernel3c_hook(kns, "nuclear3CIntg"),
              electron3cintg=kernel3c_hook(kns, "electron3CIntg"))
    for v in ("alphanucdist", "elementnucalpha", "alphapotdist", "anyelecpotinteraction",
              "hsize_t_bitsize", "matrixindex", "cellindex", "currpottypenumber",
              "curralphanumber", "currpotalpha", "currpotnumber", "currpotelement",
              "currmultiplicity", "numelementpotalphas", "elementpotalphas"):
        ns[v] = None
    ns["elecpotinteraction"] = 0
    return ns


ROUTINES = msg.ROUTINES[:9] + [
    ("kpoints.f90", "subroutine", "convertKPointsToXYZ"),
    ("kpoints.f90", "subroutine", "computePhaseFactors"),
    ("basis.f90", "subroutine", "renormalizeBasis"),
    ("basis.f90", "subroutine", "initializeAtomSite"),
    ("gaussRelations.f90", "subroutine", "makeAlphaDist"),
    ("intgSaving.F90", "subroutine", "multWithBasisFn1"),
    ("intgSaving.F90", "subroutine", "applyPhaseFactors"),
    ("intgSaving.F90", "subroutine", "kPointLatticeOriginShift"),
    ("intgSaving.F90", "subroutine", "valeValeSaving"),
    ("intgSaving.F90", "subroutine", "coreValeSaving"),
    ("intgSaving.F90", "subroutine", "coreCoreSaving"),
    ("intgSaving.F90", "subroutine", "saveCurrentPair"),
    ("intgOrtho.F90", "subroutine", "valeCoreCoreValeOL"),
    ("intgOrtho.F90", "subroutine", "valeCoreCoreVale"),
    ("intgOrtho.F90", "subroutine", "coreValeCoreCore"),
    ("intgOrtho.F90", "subroutine", "makeValeVale"),
    ("integrals.F90", "subroutine", "orthoOL"),
    ("integrals.F90", "subroutine", "ortho"),
    ("integrals.F90", "subroutine", "gaussOverlapOL"),
    ("integrals.F90", "subroutine", "gaussOverlapKE"),
    ("gaussRelations.f90", "subroutine", "makeAlphaNucDist"),
    ("basis.f90", "subroutine", "initializePotSite"),
    ("integrals.F90", "subroutine", "nuclearPE"),
    ("integrals.F90", "subroutine", "gaussOverlapNP"),
    ("gaussRelations.f90", "subroutine", "makeAlphaPotDist"),
    ("integrals.F90", "function", "checkElecPotInteraction"),
    ("integrals.F90", "subroutine", "electronicPE"),
    ("integrals.F90", "subroutine", "gaussOverlapEP"),
    ("integrals.F90", "subroutine", "elecPotGaussOverlap"),
]


def run(s, ref, with_ep=True):
    store = msg.Store()
    kns = make_golden.load_kernels(ref)
    ns = module_state(s, store, kns)
    ctx = fe.Ctx(functions=["error_fn", "checkelecpotinteraction"],
                 types={"phasefactor": "complex", "corevale": "complex",
                        "valecore": "complex", "lmindex": "integer",
                        "lmalphaindex": "integer", "numelementatomicalphas": "integer",
                        "anyelecpotinteraction": "integer",
                        "numelementpotalphas": "integer"})
    src = os.path.join(ref, "src", "imago")
    hooks = dict(msg.HOOK_ARGS)
    hooks.update({"zherk": [], "zher2k": [], "overlap2cintg": [], "kinetic2cintg": [],
                  "nuclear3cintg": [], "electron3cintg": []})
    for f, k, n in ROUTINES:
        fe.load(os.path.join(src, f), k, n, ns, ctx, hooks)
    ns["findlatticevector"] = msg.nearest_lattice(ns)
    ns["setcutoffthresh"](s.basis_fn_convg, s.electro_convg)
    ns["getrecipcellvectors"]()
    ns["initializelattice"](1)
    ns["convertkpointstoxyz"]()
    ns["computephasefactors"]()
    ns["renormalizebasis"]()
    ns["makealphadist"]()
    nk = ns["numkpoints"]
    did = msg.names("ol", nk)
    cvdid = fe.Arr.of(np.array([[f"olcv_re_{k + 1}", f"olcv_im_{k + 1}"] for k in range(nk)],
                               dtype=object).T, dtype=object)
    t0 = time.time()
    ns["gaussoverlapol"](2, None, None, did, cvdid, "ol_aid")
    print(f"  OL executed in {time.time() - t0:.1f} s", flush=True)
    # gaussOverlapKE allocates its own coreVale (integrals.F90:775)
    t0 = time.time()
    ns["gaussoverlapke"](None, msg.names("ke", nk), "ke_aid")
    print(f"  KE executed in {time.time() - t0:.1f} s", flush=True)
    ns["makealphanucdist"]()
    t0 = time.time()
    ns["gaussoverlapnp"](None, msg.names("np", nk), "np_aid")
    print(f"  NP executed in {time.time() - t0:.1f} s", flush=True)
    if with_ep:
        ns["makealphapotdist"]()
        P = ns["potdim"]
        didp = fe.Arr.of(np.array([[f"ep_{t + 1}_{k + 1}" for t in range(P)] for k in range(nk)],
                                  dtype=object), dtype=object)
        t0 = time.time()
        ns["elecpotgaussoverlap"](None, didp, msg.names("ep_aid", P))
        print(f"  EP executed in {time.time() - t0:.1f} s", flush=True)
    V = ns["valedim"]
    npk = V * (V + 1) // 2

    def packed(prefix):
        return np.stack([np.asarray(store.d[f"{prefix}_{k + 1}"]).reshape(2, npk).T
                         for k in range(nk)])
    out = {"ol_packed": packed("ol"), "ke_packed": packed("ke"), "np_packed": packed("np")}
    if with_ep:
        out["ep_packed"] = np.stack([packed(f"ep_{t + 1}") for t in range(ns["potdim"])])
    if ns["coredim"]:
        out["ol_cv_re"] = np.stack([np.asarray(store.d[f"olcv_re_{k + 1}"]).T
                                    for k in range(nk)])
        out["ol_cv_im"] = np.stack([np.asarray(store.d[f"olcv_im_{k + 1}"]).T
                                    for k in range(nk)])
    out["phaseFactor"] = ns["phasefactor"].a.T.copy()     # [cell][k]
    out["kPointsXYZ"] = ns["kpoints"].a.T.copy()
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_driver_golden.py <root of the reference checkout>")
    from imago_b200 import configs
    s = configs.diamond_primitive(kmesh=(2, 2, 2))
    print("diamond 2x2x2", flush=True)
    np.savez_compressed(os.path.join(HERE, "driver_diamond.npz"), **run(s, sys.argv[1]))


if __name__ == "__main__":
    main()
