"""Golden fixtures of the SCF set-up and potential update, made by executing
the reference's own Fortran routines (tests/golden/fortran_exec.py).

Executed from src/imago, statement for statement:

  lattice.f90      getRecipCellVectors, setCutoffThresh, initializeLattice,
                   getNumCells, makeLattice, cellBorderCheck
  sortSubs.f90     mergeSort, mergeLists
  mathSubs.f90     error_fn
  elecStat.f90     neutralAndNuclearQPot, residualQ
  exchCorr.f90     makeSampleVectors, getECMeshParameters, makeECMeshAndOverlap
  coreCharge.f90   makeCoreRho
  potentialUpdate.F90  makeSCFPot and the LDA functionals it calls

Supplied by this script: the module data (from the same synthetic systems
the tests build, imago_b200.configs), findLatticeVector (any nearest lattice
vector: the routines sum over the whole lattice list, so which of two
equidistant vectors is taken only reorders terms), HDF5 reads and writes
(a dictionary), solveDPOSVX (LAPACK's dposvx('E', 'U') through scipy, the
routine the reference calls), and, for the SCF trajectory, the valence
charge of each iteration from the oracle (oracle.valence_rho: eigh(H, S),
populateStandard, the density traces).

Fixtures (npz, under tests/golden/):

  scf_diamond.npz   the diamond primitive cell at 2x2x2 k with 20 angular
                    sample vectors: lattice lists, electrostatic operators,
                    core charge, the mesh and its overlap, and makeSCFPot's
                    inputs and outputs over the iterations of a whole SCF
                    run from the atomic-superposition start (Wigner,
                    feedback 2, relaxation 0.2)
  scf_two_type.npz  the small two-element cell (potential types of 4 and 3
                    terms, sites reordered by type): lattice lists,
                    electrostatic operators, core charge, mesh (8 vectors)

Run where the reference is mounted:

    python tests/golden/make_scf_golden.py <root of the reference checkout>
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

HOOK_ARGS = {"h5dwrite_f": [4], "h5dread_f": [2, 4], "h5aread_f": [2, 4],
             "h5awrite_f": [4], "h5aclose_f": [1], "solvedposvx": [5]}


class Store:
    """The HDF5 datasets the routines write and read back."""

    def __init__(self):
        self.d = {}

    def write(self, did, typ, buf, dims, err):
        self.d[did] = np.array(fe._val(buf), copy=True)
        return (0,)

    def read(self, did, typ, buf, dims, err):
        v = self.d[did]
        if isinstance(buf, (fe.Arr, np.ndarray)):
            a = fe._val(buf)
            a[...] = np.asarray(v).reshape(a.shape) if np.size(v) == a.size else v
            return (buf, 0)
        return (np.asarray(v).item(), 0)


def solve_dposvx(N, NRHS, A, LD, B, INFO):
    from scipy.linalg import lapack
    a = np.array(fe._val(A), float)[:N, :N]
    b = fe._val(B)
    b2 = b.reshape(b.shape[0], -1)
    x = lapack.dposvx(a, np.array(b2[:N, :NRHS], float), fact="E", lower=0)
    b2[:N, :NRHS] = x[5]
    return (x[9],)


def nearest_lattice(ns):
    def find(v, out):
        rv = ns["realvectors"].a  # (xyz, abc)
        v = np.asarray(fe._val(v), float)
        base = np.round(np.linalg.solve(rv, v))
        best, bd = None, None
        for d in np.ndindex(3, 3, 3):
            L = rv @ (base + np.array(d) - 1)
            dist = ((v - L) ** 2).sum()
            if bd is None or dist < bd * (1 - 1e-12):
                best, bd = L, dist
        fe._val(out)[...] = best
        return ()
    return find


def objs(items):
    a = np.empty(len(items), dtype=object)
    a[:] = items
    return fe.Arr.of(a, dtype=object)


def names(prefix, n):
    return objs([f"{prefix}_{i + 1}" for i in range(n)])


def module_state(s, store, nsv):
    ns = fe.runtime_namespace()
    ns.update(dim3=3, pi=3.141592653589793, smallthresh=1.0e-8, bigthresh=1.0e20,
              langmomcount=4, h5t_native_double=0, h5t_native_integer=1,
              h5dwrite_f=store.write, h5dread_f=store.read,
              h5aread_f=lambda aid, t, st, d, e: (0, 0), h5awrite_f=lambda *a: (0,),
              h5aclose_f=lambda *a: (0,), timestampstart=lambda *a: (),
              timestampend=lambda *a: (), solvedposvx=solve_dposvx)
    ns["realvectors"] = fe.Arr.of(np.asarray(s.real_vectors).T)
    for v in ("recipvectors", "invrealvectors"):
        ns[v] = fe.Arr((3, 3))
    ns["recipmag"] = fe.Arr(3)
    for v in ("realcellvolume", "recipcellvolume", "numcellsreal", "numcellsrecip",
              "negliglimitreal", "negliglimitrecip", "logbasisfnthresh", "logelecthresh"):
        ns[v] = 0
    ns["primrepsreal"] = fe.Arr(3, np.int64)
    ns["primrepsrecip"] = fe.Arr(3, np.int64)
    ns["minatomicalpha"] = min(100.0, *[t.alphas[0] for t in s.atom_types])
    ns["minpotalpha"] = min(10000.0, *[p.alphas[0] for p in s.pot_types])
    pst = np.asarray(s.pot_site_type)
    pts, cum = [], 0
    for ti, p in enumerate(s.pot_types):
        pts.append(fe.Obj(numalphas=len(p.alphas), alphas=fe.Arr.of(p.alphas),
                          nucalpha=p.nuc_alpha, nuccharge=p.nuc_charge,
                          multiplicity=int((pst == ti + 1).sum()), cumulalphasum=cum,
                          elementid=p.element, covalentradius=p.covalent_radius))
        cum += len(p.alphas)
    ns["pottypes"] = objs(pts)
    ns["numpottypes"] = len(pts)
    ns["potdim"] = cum
    ns["maxnumpotalphas"] = max(len(p.alphas) for p in s.pot_types)
    sites, last = [], 0
    for t, pos in zip(pst, s.pot_site_pos):
        sites.append(fe.Obj(pottypeassn=int(t), cartpos=fe.Arr.of(pos),
                            firstpottype=int(t != last)))
        last = t
    ns["potsites"] = objs(sites)
    ns["numpotsites"] = len(sites)
    ats = []
    for t in s.atom_types:
        nc = len(t.core_l)
        cr = np.zeros((t.num_orb_alphas[0], max(nc, 1)))
        for k, c in enumerate(t.core_coeffs):
            cr[:len(c), k] = c
        ats.append(fe.Obj(numorbalphas=fe.Arr.of(t.num_orb_alphas, np.int64),
                          alphas=fe.Arr.of(t.alphas), numcoreradialfns=nc,
                          coreqn_llist=fe.Arr.of(list(t.core_l) or [0], np.int64),
                          coreradialfns=fe.Arr.of(cr), maxcoreqn_l=max(t.core_l) if nc else -1,
                          numcorestates=t.num_core_states))
    ns["atomtypes"] = objs(ats)
    ns["maxnumatomalphas"] = max(t.num_orb_alphas[0] for t in s.atom_types)
    ns["maxnumcoreradialfns"] = max(len(t.core_l) for t in s.atom_types)
    ns["coredim"] = s.core_dim
    n = len(sites)
    ns.update(printxcmesh=0, numsamplevectors=nsv, angsampleweights=fe.Arr.of([0.5, 0.5]),
              rsamplein=0.1, rsampleout=3.5, rsamplespace=0.8, gga=0, numraypoints=0,
              maxnumraypoints=0, numpoints_did=names("numPoints", n),
              radialweight_did=names("radialWeight", n), exchrhoop_did=names("exchRhoOp", n),
              exchcorroverlap_did="exchCorrOverlap", exchcorrgroup_aid="xc",
              corechargedensity_did="coreChargeDensity")
    for v in ("potalphaoverlap", "nonlocalneutqpot", "nonlocalnucqpot", "localneutqpot",
              "localnucqpot", "nonlocalresidualq"):
        ns[v + "_did"] = v
        ns[v] = None
    for v in ("potolandlocalq_aid", "nonlocalresidualq_aid", "potpot", "pot", "pottypespot",
              "numpoints", "points", "potpoints", "angsamplevectors", "potlatticesep",
              "sitesamplemaxradius", "radialweight", "exchrhoop", "exchcorroverlap",
              "corechargedensity"):
        ns[v] = None
    return ns


ROUTINES = [
    ("sortSubs.f90", "subroutine", "mergeLists"), ("sortSubs.f90", "subroutine", "mergeSort"),
    ("lattice.f90", "subroutine", "cellBorderCheck"), ("lattice.f90", "subroutine", "getNumCells"),
    ("lattice.f90", "subroutine", "makeLattice"),
    ("lattice.f90", "subroutine", "getRecipCellVectors"),
    ("lattice.f90", "subroutine", "setCutoffThresh"),
    ("lattice.f90", "subroutine", "initializeLattice"),
    ("mathSubs.f90", "function", "error_fn"),
    ("elecStat.f90", "subroutine", "neutralAndNuclearQPot"),
    ("elecStat.f90", "subroutine", "residualQ"),
    ("exchCorr.f90", "subroutine", "makeSampleVectors"),
    ("exchCorr.f90", "subroutine", "getECMeshParameters"),
    ("exchCorr.f90", "subroutine", "makeECMeshAndOverlap"),
    ("coreCharge.f90", "subroutine", "makeCoreRho"),
    ("potentialUpdate.F90", "subroutine", "wignerXC"),
    ("potentialUpdate.F90", "subroutine", "wignerXCEnergy"),
    ("potentialUpdate.F90", "subroutine", "ceperleyAlderXC"),
    ("potentialUpdate.F90", "subroutine", "ceperleyAlderXCEnergy"),
    ("potentialUpdate.F90", "subroutine", "hedinLundqvistXC"),
    ("potentialUpdate.F90", "subroutine", "hedinLundqvistXCEnergy"),
    ("potentialUpdate.F90", "subroutine", "makeSCFPot"),
]


def setup(s, ref_root, nsv):
    """Run the reference's set-up routines for system s; returns the
    namespace and the dataset store."""
    store = Store()
    ns = module_state(s, store, nsv)
    ctx = fe.Ctx(functions=["error_fn"])
    src = os.path.join(ref_root, "src", "imago")
    for f, k, n in ROUTINES:
        fe.load(os.path.join(src, f), k, n, ns, ctx, HOOK_ARGS, record=(n == "makeSCFPot"))
    ns["findlatticevector"] = nearest_lattice(ns)
    ns["setcutoffthresh"](s.basis_fn_convg, s.electro_convg)
    ns["getrecipcellvectors"]()
    ns["initializelattice"](1)
    t0 = time.time()
    ns["neutralandnuclearqpot"]()
    ns["residualq"]()
    ns["makesamplevectors"]()
    ns["getecmeshparameters"]()
    ns["makeecmeshandoverlap"]()
    if s.core_dim:
        ns["makecorerho"]()
    else:
        store.d["coreChargeDensity"] = np.zeros(ns["potdim"])
    print(f"  set-up executed in {time.time() - t0:.1f} s", flush=True)
    return ns, store


def setup_arrays(ns, store):
    n = ns["numpotsites"]
    out = {"cellDimsReal": ns["celldimsreal"].a.T.copy(),
           "cellSizesReal": ns["cellsizesreal"].a.copy(),
           "cellDimsRecip": ns["celldimsrecip"].a.T.copy(),
           "cellSizesRecip": ns["cellsizesrecip"].a.copy(),
           "realCellVolume": np.array(ns["realcellvolume"])}
    # potDim x potDim datasets as the reference holds them: (row, col)
    for k in ("potalphaoverlap", "nonlocalneutqpot", "localneutqpot", "nonlocalnucqpot",
              "localnucqpot", "nonlocalresidualq"):
        out[k] = np.asarray(store.d[k])
    out["exchCorrOverlap"] = np.asarray(store.d["exchCorrOverlap"])
    out["coreChargeDensity"] = np.asarray(store.d["coreChargeDensity"])
    out["numPoints"] = np.array([int(store.d[f"numPoints_{i + 1}"]) for i in range(n)])
    out["radialWeight"] = np.concatenate(
        [store.d[f"radialWeight_{i + 1}"][:out["numPoints"][i]] for i in range(n)])
    out["exchRhoOp"] = np.concatenate(
        [store.d[f"exchRhoOp_{i + 1}"][:, :out["numPoints"][i], 0].T for i in range(n)])
    return out


def scf_trajectory(s, ns, store, start, max_iter=40):
    """mainSCF with the reference's makeSCFPot: each iteration's valence
    charge from the oracle, then the executed update."""
    import oracle
    ob = oracle.OracleBuild(s)
    olp = ob.overlap()[0]
    kep = ob.kinetic()
    npp = ob.nuclear()
    epp = ob.elec_pot()
    ob.close()
    from imago_b200 import scf as pyscf
    ne = pyscf.valence_electrons(s)
    P = ns["potdim"]
    ic = np.zeros(P)
    for p in ns["pottypes"].a:
        for j in range(p.numalphas):
            ic[p.cumulalphasum + j] = p.multiplicity * np.pi ** 1.5 / p.alphas[j + 1] ** 1.5
    nk = len(s.kpoints_abc)
    ns.update(numelectrons=ne, numkpoints=nk, rel=0, spin=1, intgconsts=fe.Arr.of(ic),
              spinsplitfactor=fe.Arr.of(np.zeros(P)),
              potalphas=fe.Arr.of(np.concatenate([p.alphas for p in s.pot_types])),
              potcoeffs=fe.Arr.of(np.asarray(start)[:, None]), curriteration=1,
              lastiteration=max_iter, feedbacklevel=2, relaxfactor=0.2, xccode=100,
              converged=0, convgtest=1.0e-4, numplusujatoms=0,
              plusujatomid=fe.Arr((1,), np.int64), plusuj=fe.Arr((7, 1, 1, nk)),
              massvelocitytrace=None, xl0=None, xl1=None, xl2=None, yl0=None, yl1=None,
              yl2=None, potcoeffs_did=objs([[f"potCoeffs_{i}_1"] for i in range(1, 200)]),
              totalrhocoeffs_did=names("totalRho", 200), valerhocoeffs_did=names("valeRho", 200),
              spindiffrhocoeffs_did=None, alphas_did="alphas", terms=None)
    ns["potcoeffs_did"] = fe.Arr.of(np.array([[f"potCoeffs_{i}_1"] for i in range(1, 200)],
                                             dtype=object), dtype=object)
    ns["points"] = fe.Arr.of([ns["maxnumraypoints"]], np.int64)
    rows = {k: [] for k in ("used", "potRho", "nucPotTrace", "kineticEnergyTrace", "next",
                            "totalEnergy", "kineticEnergy", "elecStatEnergy",
                            "exchCorrEnergy", "electronDiff", "testableDelta", "converged")}
    for it in range(max_iter):
        used = ns["potcoeffs"].a[:, 0].copy()
        r = oracle.valence_rho(npp, kep, epp, olp, used, ne, s.vale_dim)
        ns["occupiedenergy"] = r["occupiedEnergy"]
        ns["bandgap"] = r["bandGap"]
        ns["gapkindcode"] = r["gapKindCode"]
        ns["potrho"] = fe.Arr.of(r["potRho"])
        ns["chargedensitytrace"] = fe.Arr.of(r["chargeDensityTrace"])
        ns["nucpottrace"] = fe.Arr.of(r["nucPotTrace"])
        ns["kineticenergytrace"] = fe.Arr.of(r["kineticEnergyTrace"])
        (etot,) = ns["makescfpot"](0.0)
        loc = ns["_recorded"]["makescfpot"]
        rows["used"].append(used)
        rows["potRho"].append(r["potRho"][:, 0])
        rows["nucPotTrace"].append(r["nucPotTrace"][0])
        rows["kineticEnergyTrace"].append(r["kineticEnergyTrace"][0])
        rows["next"].append(ns["potcoeffs"].a[:, 0].copy())
        rows["totalEnergy"].append(etot)
        rows["kineticEnergy"].append(loc["kineticenergy"])
        rows["elecStatEnergy"].append(loc["elecstatenergy"])
        rows["exchCorrEnergy"].append(loc["exchcorrenergy"])
        rows["electronDiff"].append(loc["electrondiff"])
        rows["testableDelta"].append(loc["testabledelta"])
        rows["converged"].append(ns["converged"])
        print(f"  iteration {it + 1}: E = {etot:.10f}  delta = {loc['testabledelta']:.3e}",
              flush=True)
        if ns["converged"]:
            break
    return {"scf_" + k: np.asarray(v) for k, v in rows.items()}


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_scf_golden.py <root of the reference checkout>")
    ref = sys.argv[1]
    from imago_b200 import configs, scf as pyscf
    s = configs.diamond_primitive(kmesh=(2, 2, 2))
    print("diamond 2x2x2", flush=True)
    ns, store = setup(s, ref, 20)
    out = setup_arrays(ns, store)
    out.update(scf_trajectory(s, ns, store, pyscf.atomic_start(s)))
    np.savez_compressed(os.path.join(HERE, "scf_diamond.npz"), **out)
    s = configs.small_test_system()
    print("two-type cell", flush=True)
    ns, store = setup(s, ref, 8)
    np.savez_compressed(os.path.join(HERE, "scf_two_type.npz"), **setup_arrays(ns, store))


if __name__ == "__main__":
    main()
