"""Integral-build benchmark: Imago's SCF integral setup on B200.

Workload (one "step", default --workload si8): the full integral setup of
the jittered 8-atom silicon conventional cell with an s,p,d basis of 20
even-tempered primitives, 20 potential terms and an 8x8x8 k-mesh: the
overlap, kinetic, nuclear and all 20 electronic-potential matrices,
lattice-summed, Bloch-phased onto 512 k-points, core-orthogonalised and
packed as the reference hands them to SCF.  Inputs are synthetic (seeded
positions and synthesised contraction coefficients; the reference's basis
database is not available).  --workload quartz-gamma / quartz-222 runs the
162-atom alpha-quartz supercell instead (Gamma only, or a 2x2x2 mesh); the
default run also reports the quartz Gamma build as "silica_162".

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
                    [--workload si8|quartz-gamma|quartz-222]

Our arm times K builds on the device (CUDA events on the library's stream,
L2 flushed between steps, outputs resident in HBM), then the same build end
to end through the C ABI with host buffers (create + build + copies into
pinned host memory, wall clock).  The reference arm times the CPU
restatement of the reference's algorithm (oracle/, all host threads) on a
bounded sample of the same workload and scales it to one build.
Under torchrun each rank builds its own independently jittered cell (weak
scaling, no collective on the data path).
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

UNIT = "s"
WORKLOADS = {
    "si8": {
        "metric": "integral build time (OL+KE+NP+20 EP, 512 k-points)",
        "desc": ("Si8 conventional cell, jitter N(0,0.02 A), s,p,d basis 20 "
                 "primitives (20/20/14/0), 20 potential terms, 8x8x8 k"),
        # the oracle runs the whole build when it is this cheap
        "cpu_stride": 1,
    },
    "quartz-gamma": {
        "metric": "integral build time (OL+KE+NP+40 EP, Gamma)",
        "desc": ("alpha-quartz SiO2 3x3x2 supercell, 162 atoms, jitter "
                 "N(0,0.03 A), Si s,p,d (20/20/14) and O s,p (18/18) "
                 "primitives, 20+20 potential terms, Gamma"),
        "cpu_stride": 8,
    },
    "batch64": {
        "metric": "batched integral build time, 64 cells (OL+KE+NP+all EP each, 2x2x2 k)",
        "desc": ("64 independent cells of uneven size (Si 8..64 atoms, diamond "
                 "and graphite 8..216 atoms), random symmetric strain within "
                 "+-3%, jitter N(0,0.02 A), bases and potentials as the diamond "
                 "and Si8 workloads, 2x2x2 k, one CUDA graph with a branch per "
                 "cell"),
        "cpu_stride": 4,
    },
    "quartz-222": {
        "metric": "integral build time (OL+KE+NP+40 EP, 8 k-points)",
        "desc": ("alpha-quartz SiO2 3x3x2 supercell, 162 atoms, jitter "
                 "N(0,0.03 A), Si s,p,d (20/20/14) and O s,p (18/18) "
                 "primitives, 20+20 potential terms, 2x2x2 k (shift 1/2)"),
        "cpu_stride": 8,
    },
}


def system_for(workload, rank=0, kmesh=(8, 8, 8)):
    from imago_b200 import configs
    if workload == "batch64":
        return configs.batch_cells(seed=5 + rank)
    if workload == "si8":
        return configs.silicon_cubic8(seed=2 + rank, kmesh=tuple(kmesh))
    if workload == "quartz-gamma":
        return configs.quartz_supercell(seed=3 + rank, gamma=True)
    return configs.quartz_supercell(seed=3 + rank, kmesh=(2, 2, 2))


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


# ---------------------------------------------------------------- clocks --
class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------ algorithmic --
def algorithmic_flops(g):
    """Per-build FLOPs of the dense stages, from the screened work counts:
    lattice-to-k sum: 4 flops per (k, unit block element), per matrix;
    orthogonalisation: Y = X_cv - X_cc S/2 (8 C^2 V per k) and the packed
    update S^H Y + Y^H S (16 C per packed element per k), per matrix."""
    nmat = 3 + g.pot_dim
    V, C, nk = g.vale_dim, g.core_dim, g.nk
    m_elems = g.block_elements
    bloch = 4.0 * nk * m_elems * nmat
    ortho = nk * (8.0 * C * C * V + 16.0 * C * g.npacked) * nmat
    return {"bloch": bloch, "ortho": ortho}


# DRAM bytes (read + write) per (k-point, matrix) of the fused
# orthogonalisation, from one ncu capture of its Si8 4x4x4 EP launch: 243.66 MB
# read and 83.76 MB written for 64 k x 20 terms.  The kernel's traffic grows
# in proportion to the (k, matrix) pairs, so the build's figure is this times
# nk x (3 + potDim).
ORTHO_FUSED_BYTES_PER_KMAT = (243.658496e6 + 83.760128e6) / 1280


def fp64_peak_tflops(torch):
    """Measured FP64 dense throughput of this GPU (cuBLAS DGEMM 8192^3)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


# ------------------------------------------------------------- CPU legs --
def oracle_build_time(system, nthreads, pair_stride=1, ep_ortho_sampled=False):
    """Seconds the oracle takes for the pair loops and the
    orthogonalisation of OL, KE, NP and every EP term.  With pair_stride > 1
    every pair_stride-th atom pair runs and the pair loops are scaled up.
    With ep_ortho_sampled the EP terms run their pair loops only and their
    orthogonalisation (the same Hermitian rank-2k update for every term) is
    the mean of the KE and NP ones."""
    import oracle
    ob = oracle.OracleBuild(system, stride=pair_stride, nthreads=nthreads)
    loops = ortho = 0.0
    zher2k = []
    for call in (ob.overlap, ob.kinetic, ob.nuclear):
        call()
        lo, ot = ob.last_times()
        loops += lo
        ortho += ot
        if call != ob.overlap:
            zher2k.append(ot)
    ob.set_skip_ortho(ep_ortho_sampled)
    for t in range(ob.pot_dim):
        ob.elec_pot(t, t + 1)
        lo, ot = ob.last_times()
        loops += lo
        ortho += float(np.mean(zher2k)) if ep_ortho_sampled else ot
    ob.close()
    return pair_stride * loops + ortho


def k_subset(system, k_stride):
    import copy
    s = copy.copy(system)
    s.kpoints_abc = system.kpoints_abc[::k_stride].copy()
    return s


def cpu_baseline(system, nthreads, workload, limit_s=40.0):
    """The oracle on the host cores, scaled to one build of the workload.
    Si8: a quick probe (every 8th atom pair, every 16th k-point) estimates
    the full build; when that is within limit_s the full build is timed,
    otherwise every 4th atom pair.  Quartz: every cpu_stride-th atom pair,
    the EP orthogonalisations sampled."""
    t0 = time.perf_counter()
    stride = WORKLOADS[workload]["cpu_stride"]
    if workload == "batch64":
        # the cells are independent draws: every 8th cell, scaled by 8
        cells = system[::8]
        value = 8 * sum(oracle_build_time(c, nthreads, pair_stride=stride,
                                          ep_ortho_sampled=True) for c in cells)
        sample = (f"every 8th cell ({len(cells)} of {len(system)}, scaled by 8), "
                  f"every {stride}th atom pair (pair loops scaled by {stride}), "
                  f"EP orthogonalisation timed on KE and NP")
        return value, time.perf_counter() - t0, sample
    if stride > 1:
        value = oracle_build_time(system, nthreads, pair_stride=stride,
                                  ep_ortho_sampled=True)
        sample = (f"every {stride}th atom pair (pair loops scaled by {stride}), "
                  f"EP orthogonalisation timed on KE and NP")
        return value, time.perf_counter() - t0, sample
    est = 16 * oracle_build_time(k_subset(system, 16), nthreads, pair_stride=8)
    if est <= limit_s:
        value, sample = oracle_build_time(system, nthreads), "the full build"
    else:
        value = oracle_build_time(system, nthreads, pair_stride=4)
        sample = "every 4th atom pair at all k-points, pair loops scaled by 4"
    return value, time.perf_counter() - t0, sample


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle  # noqa: F401
    wl = WORKLOADS[args.workload]
    system = system_for(args.workload, 0, args.kmesh)
    nthreads = os.cpu_count() or 1
    times, walls = [], []
    probe = system[0] if args.workload == "batch64" else k_subset(system, 16)
    for _ in range(args.warmup):  # warm caches and pages on a small probe
        oracle_build_time(probe, nthreads, pair_stride=16, ep_ortho_sampled=True)
    what = ""
    for _ in range(args.steps):
        v, wall, what = cpu_baseline(system, nthreads, args.workload, limit_s=30.0)
        times.append(v)
        walls.append(wall)
    value = float(np.mean(times))
    sample = (f"CPU restatement of the reference path (oracle/, C, OpenMP over "
              f"atom pairs, {nthreads} threads): {what}; "
              f"{np.mean(walls):.1f} s of CPU work per step")
    line = {
        "impl": "reference", "metric": wl["metric"], "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": value * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": wl["desc"]},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads,
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if args.workload == "si8" and list(args.kmesh) != [8, 8, 8]:
        line["note"] = f"k-mesh {args.kmesh} (profiling case, not the measured workload)"
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------- our arm --
def device_outputs(g, torch, dev):
    nk, npk, V, C, P = g.nk, g.npacked, g.vale_dim, g.core_dim, g.pot_dim
    f64 = torch.float64
    return {
        "ol_packed": torch.empty((nk, npk, 2), dtype=f64, device=dev),
        "ol_cv_re": torch.empty((nk, V, max(C, 1)), dtype=f64, device=dev),
        "ol_cv_im": torch.empty((nk, V, max(C, 1)), dtype=f64, device=dev),
        "ke_packed": torch.empty((nk, npk, 2), dtype=f64, device=dev),
        "np_packed": torch.empty((nk, npk, 2), dtype=f64, device=dev),
        "ep_packed": torch.empty((P, nk, npk, 2), dtype=f64, device=dev),
    }


def time_device_builds(g, bufs, stream, steps, flush, torch):
    """Device seconds of each build (outputs in HBM) replayed from the
    context's CUDA graph (imago_intg_build_graph, captured in the warm-up;
    the four kinds run concurrently), with 512 MiB written between builds
    to flush L2.  The kernel-stage milliseconds come from the same number
    of plain builds with the kinds serialised, so that each stage's time is
    its own."""
    out = {k: v.data_ptr() for k, v in bufs.items()}
    step_s, kms, launches = [], np.zeros(4), 0
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record(stream)
        g.build_graph(out)
        e.record(stream)
        e.synchronize()
        step_s.append(s.elapsed_time(e) / 1e3)
        launches += g.kernel_stats()[1]
    g.set_serial(True)  # stage times of each kernel without the overlap
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        g.build(out=out)
        kms += g.kernel_stats()[0]
    g.set_serial(False)
    return step_s, kms, launches


# Algorithmic FP64 flops of one primitive three-centre evaluation by class
# (l_a, l_b), larger l first: the binary + - * of the reference's generated
# recursions (src/imago/gaussIntegrals.f90 electron3CIntg / nuclear3CIntg
# class blocks, counted over the statements; ranges between the two orders
# taken at their middle), prefactor exp / erf / pow not included.
EP_FLOPS = {(0, 0): 0, (1, 0): 3, (1, 1): 21, (2, 0): 19, (2, 1): 91, (2, 2): 320,
            (3, 0): 54, (3, 1): 248, (3, 2): 819, (3, 3): 2022}
NP_FLOPS = {(0, 0): 0, (1, 0): 9, (1, 1): 63, (2, 0): 49, (2, 1): 241, (2, 2): 797,
            (3, 0): 137, (3, 1): 610, (3, 2): 1916, (3, 3): 4499}


def prim3c_roofline(g, bufs, stream, flush, torch, peak, steps=3):
    """FP64 roofline of the three-centre primitive stage: the screened
    (shell pair, site, image) triples of the NP build and every EP term per
    class (imago_intg_count_triples) times the per-class flops above, over
    the k_prim3c time of NP + EP builds run alone (kinds serialised, L2
    flushed before each), against the measured FP64 peak."""
    from imago_b200 import intg
    cnp = g.count_triples(intg.IMAGO_NP)
    cep = g.count_triples(intg.IMAGO_EP)
    if (cnp < 0).any() or (cep < 0).any():
        return None
    flops = 0.0
    for la in range(4):
        for lb in range(4):
            key = (max(la, lb), min(la, lb))
            flops += cnp[la, lb] * NP_FLOPS[key] + cep[la, lb] * EP_FLOPS[key]
    out = {k: v.data_ptr() for k, v in bufs.items()}
    g.set_serial(True)
    ms = 0.0
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        g.build(which=intg.IMAGO_NP | intg.IMAGO_EP, out=out)
        ms += g.kernel_stats()[0][0]
    g.set_serial(False)
    ms /= steps
    achieved = flops / (ms / 1e3) / 1e12
    return {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if peak else None, "kernel": "k_prim3c (NP + EP)",
            "kernel_ms": ms, "algorithmic_flops": flops,
            "triples_np": int(cnp.sum()), "triples_ep": int(cep.sum()),
            "flops_source": "reference recursion flops per class x screened triples"}


def time_e2e(system, local, stream, bufs, steps, torch):
    """End to end through the C ABI with host buffers, wall clock: create
    (host set-up, H2D of the system, device tables) + one build of every
    matrix into pinned host memory (the call returns once the copies have
    landed).  The first of steps + 1 runs is a warm-up; the median run is
    reported, the host being shared."""
    from imago_b200 import intg
    pinned = {k: torch.empty(v.shape, dtype=v.dtype, pin_memory=True)
              for k, v in bufs.items()}
    tot, cre = [], []
    for i in range(steps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g2 = intg.IntegralSetup(system, device=local, outputs_on_device=False,
                                stream=stream.cuda_stream)
        t1 = time.perf_counter()
        g2.build(out={k: v.data_ptr() for k, v in pinned.items()})
        t2 = time.perf_counter()
        g2.close()
        if i > 0:
            tot.append(t2 - t0)
            cre.append(t1 - t0)
    d2h = sum(v.numel() * 8 for v in pinned.values())
    i = int(np.argsort(tot)[len(tot) // 2])  # the median run
    return {"value": float(tot[i]), "unit": UNIT,
            "h2d_bytes_per_step": _system_bytes(system), "d2h_bytes_per_step": d2h,
            "create_s": float(cre[i]), "build_and_copy_s": float(tot[i] - cre[i]),
            "stat": f"median of {len(tot)} runs (mean {np.mean(tot):.4f} s)"}


def time_secular(bufs, pot_dim, stream, torch, steps=3):
    """Device seconds of one SCF step's secular equation from the resident
    builds: H and S assembled for every k and the generalised eigenvalues
    (imago_b200.secular), with synthetic potential coefficients."""
    from imago_b200 import secular
    w = -0.5 * np.ones(pot_dim)
    out = {k: bufs[k] for k in ("np_packed", "ke_packed", "ep_packed", "ol_packed")}
    with torch.cuda.stream(stream):
        secular.secular_eigenvalues(out, w)
        ts = []
        for _ in range(steps):
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record(stream)
            secular.secular_eigenvalues(out, w)
            e.record(stream)
            e.synchronize()
            ts.append(s.elapsed_time(e) / 1e3)
    return float(np.median(ts))


def _event_ms(fn, stream, torch, steps=3):
    fn()
    ts = []
    for _ in range(steps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts))


def time_reduction(out, w, pop, stream, torch):
    """Device milliseconds (median of 3, CUDA events) of the library's
    Cholesky reduction (A = L^-1 H L^-H), back-transformation (c = L^-H y for
    the populated states' count of vectors) and packed density for every
    k-point, each beside the cuSOLVER / cuBLAS calls through torch that do
    the same work (batched Cholesky and triangular solves; a complex GEMM
    and the packing gather), on the same matrices."""
    from imago_b200 import charge, secular
    hs, ss = secular._secular_storage(out, w)
    nk, n = hs.shape[0], hs.shape[-1]
    h, s = hs.transpose(-2, -1), ss.transpose(-2, -1)
    f = torch.as_tensor(pop, dtype=torch.float64, device=hs.device)
    ns = int(torch.nonzero((f != 0).any(dim=0)).flatten()[-1]) + 1
    res = {"n": n, "num_kpoints": nk, "states": ns}
    with torch.cuda.stream(stream):
        a, lfac, _ = secular.cholesky_reduce(hs, ss, factor=True)
        _, vec = secular.hermitian_eigh(a)
        res["reduce_ms"] = _event_ms(lambda: secular.cholesky_reduce(hs, ss, factor=True),
                                     stream, torch)

        def lib_reduce():
            lo = torch.linalg.cholesky(s)
            y = torch.linalg.solve_triangular(lo, h, upper=False)
            return lo, torch.linalg.solve_triangular(lo, y.mH, upper=False)
        res["cusolver_reduce_ms"] = _event_ms(lib_reduce, stream, torch)
        lo, _ = lib_reduce()
        res["back_ms"] = _event_ms(lambda: secular.back_transform(lfac, vec, ns), stream, torch)
        res["cusolver_back_ms"] = _event_ms(
            lambda: torch.linalg.solve_triangular(lo.mH, vec[:, :, :ns], upper=True),
            stream, torch)
        c = secular.back_transform(lfac, vec, ns)
        fs = f[:, :ns].contiguous()
        ph = np.ascontiguousarray(np.asarray(pop, dtype=np.float64)[:, :ns])
        res["density_ms"] = _event_ms(lambda: charge.packed_density(c, ph), stream, torch)
        cols = torch.repeat_interleave(torch.arange(n), torch.arange(1, n + 1)).to(hs.device)
        rows = torch.arange(n * (n + 1) // 2, device=hs.device) - cols * (cols + 1) // 2
        cc = c.contiguous()

        def lib_density():
            full = (cc * fs[:, None, :].to(cc.dtype)) @ cc.mH
            return torch.view_as_real(full[:, rows, cols].contiguous())
        res["cublas_density_ms"] = _event_ms(lib_density, stream, torch)
        res["density_max_diff"] = float((charge.packed_density(c, ph) - lib_density())
                                        .abs().max())
    return res


def time_valence_rho(bufs, pot_dim, stream, torch, steps=3):
    """One SCF step's valence charge from the resident builds
    (imago_b200.charge): eigenvalues and eigenvectors, the populations (host,
    half as many electrons as valence states), and the density traces
    against OL, NP, KE and every EP term; median wall seconds of the step
    with the device synchronised on both sides.  Then the trace kernel alone
    over the EP terms (device events): its time and HBM bandwidth, the
    algorithmic bytes being the EP matrices read once (potDim x nk x
    nPacked x 16)."""
    import time
    from imago_b200 import charge, secular
    w = -0.5 * np.ones(pot_dim)
    out = {k: bufs[k] for k in ("np_packed", "ke_packed", "ep_packed", "ol_packed")}
    nk, npk = out["np_packed"].shape[0], out["np_packed"].shape[1]
    V = int((int((8 * npk + 1) ** 0.5) - 1) // 2)
    ne = V // 2
    ts = []
    with torch.cuda.stream(stream):
        for rep in range(steps + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e, c = secular.secular_eigensystem(out, w)
            pop = charge.populate_standard(e.cpu().numpy()[:, None, :], ne)
            r = charge.valence_rho(out, [e], [c], pop["population"], w)
            torch.cuda.synchronize()
            if rep:
                ts.append(time.perf_counter() - t0)
        rho = charge.packed_density(c, pop["population"][:, 0, :])[None]
        reduction = time_reduction(out, w, pop["population"][:, 0, :], stream, torch)
        charge.packed_traces(out["ep_packed"], rho, nk, V)
        kt = []
        for _ in range(steps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            charge.packed_traces(out["ep_packed"], rho, nk, V)
            b.record(stream)
            b.synchronize()
            kt.append(a.elapsed_time(b))
    nbytes = pot_dim * nk * npk * 16
    kms = float(np.median(kt))
    return {"valence_step_s": float(np.median(ts)), "num_electrons": ne,
            "charge_trace": float(r["chargeDensityTrace"][0]),
            "trace_kernel_ms": kms, "trace_bytes": nbytes,
            "trace_gbs": nbytes / (kms * 1e-3) / 1e9,
            "reduction": reduction,
            "stat": f"median of {steps}"}


def adjacent_builds(g, bufs, stream, torch, dev, reps=5, ham_mode="auto"):
    """Device milliseconds (median of `reps`, CUDA events on the library's
    stream, outputs resident in HBM) of the builds beside the SCF set on the
    same system: mass velocity, the momentum and dipole matrices (three
    each), the plane-wave overlaps for the three wave vectors
    b_c / n_c (reciprocal lattice vector over the k-mesh divisions; b_c at
    Gamma), the PSCF Hamiltonian for one spin and for two spins with mass
    velocity (synthetic potential coefficients), and KE + NP + all EP terms,
    the matrices the Hamiltonian combines, for comparison.  The overlap of
    the main run is resident, as these builds need."""
    from imago_b200 import intg
    n = g.nk * g.npacked * 2
    z = lambda m: torch.empty(m * n, dtype=torch.float64, device=dev)
    mv, v3, h1, h2 = z(1), z(3), z(1), z(2)
    w = np.random.default_rng(1).normal(scale=0.5, size=(g.pot_dim, 2))
    parts = {k: bufs[k].data_ptr() for k in ("ke_packed", "np_packed", "ep_packed")}
    nvv = 3 * g.nk * g.vale_dim * g.vale_dim
    kre, kim = (torch.empty(nvv, dtype=torch.float64, device=dev) for _ in range(2))
    dk = intg.koverlap_wave_vectors(g.system)
    g.set_ham_mode(ham_mode)
    cases = {
        "mass_velocity": lambda: g.build(intg.IMAGO_MV, {"mv_packed": mv.data_ptr()}),
        "momentum_xyz": lambda: g.gauss_overlap_mm(out=v3),
        "dipole_xyz": lambda: g.gauss_overlap_dm([0.5, 0.5, 0.5], out=v3),
        "plane_wave_xyz": lambda: g.gauss_koverlap(dk, re=kre, im=kim),
        "ham_pscf_spin1": lambda: g.ham_pscf(w[:, :1], out=h1),
        "ham_pscf_spin2_rel": lambda: g.ham_pscf(w, rel=True, out=h2),
        "ke_np_ep_separate": lambda: g.build(intg.IMAGO_KE | intg.IMAGO_NP | intg.IMAGO_EP,
                                             parts),
    }
    out = {}
    for name, fn in cases.items():
        fn()
        ts = []
        for _ in range(reps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ts.append(a.elapsed_time(b))
        out[name + "_ms"] = float(np.median(ts))
    out["stat"] = f"median of {reps}, device events on the library's stream"
    out["ham_mode"] = ham_mode
    g.set_ham_mode("auto")
    return out


def scf_headline(local, torch, systems=("si8", "si64", "graphite64")):
    """The metric's SCF half: Imago's SCF loop on the GPU (imago_b200.scf:
    integrals, set-up, then secular equation / populations / density traces
    / makeSCFPot per iteration) run until the reference's convergence test
    (testableDelta below 1e-5, a decade under makeinput.py's default) holds
    and two total energies agree within 1e-6 Ha, from the
    plain atomic-superposition start and from the learned start
    (imago_b200.learned, the network in imago_b200/data/learned_start.npz
    trained on the GPU by the library's own kernels).  Wall seconds with the
    device synchronised; the learned start is kept only when it reaches the
    plain start's energy within 1e-6 Ha in no more iterations.
    si8: the benched Si8 cell at 8x8x8 k (plain start only, after one
    untimed run);
    si64 / graphite64: the learned start's test cells at 4x4x4 k."""
    from imago_b200 import learned, scf
    out = {}
    weights = os.path.join(ROOT, "imago_b200", "data", "learned_start.npz")
    ls = learned.LearnedStart.load(weights, device=local) if os.path.exists(weights) else None
    for name in systems:
        s = system_for("si8") if name == "si8" else learned.test_system(name, (4, 4, 4))
        if ls is None or name == "si8":
            # one untimed run first: the process's first SCF pays one-time
            # costs (kernel loading, pool growth) that a user's steady state
            # does not
            scf.run_scf(s, scf.atomic_start(s), learned.metric_params(), device=local)
            torch.cuda.synchronize(local)
            t0 = time.perf_counter()
            r = scf.run_scf(s, scf.atomic_start(s), learned.metric_params(), device=local)
            torch.cuda.synchronize(local)
            out[name] = {"atoms": int(len(s.pot_site_type)), "kpoints": int(len(s.kpoints_abc)),
                         "plain_iterations": r["iterations"],
                         "plain_energy": r["energies"][-1],
                         "plain_converged": bool(r["done"]),
                         "integrals_s": r["timings"]["integrals_s"],
                         "setup_s": r["timings"]["setup_s"],
                         "plain_loop_s": r["timings"]["loop_s"],
                         "plain_total_s": time.perf_counter() - t0}
            continue
        r = learned.compare(s, ls, device=local)
        p, q = r["plain"], r["learned"]
        shared = r["integrals_s"] + r["setup_s"]
        lt = q["timings"]["loop_s"] + r["inference_s"]
        out[name] = {
            "atoms": int(len(s.pot_site_type)), "kpoints": int(len(s.kpoints_abc)),
            "integrals_s": r["integrals_s"], "setup_s": r["setup_s"],
            "plain_iterations": p["iterations"], "learned_iterations": q["iterations"],
            "plain_energy": p["energies"][-1], "learned_energy": q["energies"][-1],
            "plain_loop_s": p["timings"]["loop_s"], "learned_loop_s": lt,
            "inference_s": r["inference_s"], "kept": r["kept"],
            "plain_total_s": shared + p["timings"]["loop_s"],
            "learned_total_s": shared + lt,
            "learned_over_plain_total": (shared + lt) / (shared + p["timings"]["loop_s"]),
            "learned_over_plain_loop": lt / p["timings"]["loop_s"]}
    return out


def silica_headline(args, local, stream, torch):
    """The 162-atom alpha-quartz build at Gamma (device time, end to end,
    the builds beside the SCF set, and the oracle on the host cores),
    reported beside the main line."""
    from imago_b200 import intg
    wl = "quartz-gamma"
    system = system_for(wl)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=local)
    g = intg.IntegralSetup(system, device=local, outputs_on_device=True,
                           stream=stream.cuda_stream)
    bufs = device_outputs(g, torch, dev)
    flush = torch.empty(512 * 1024 * 1024 // 8, dtype=torch.float64, device=dev)
    for _ in range(2):
        g.build_graph({k: v.data_ptr() for k, v in bufs.items()})
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        step_s, kms, launches = time_device_builds(g, bufs, stream, 5, flush, torch)
    out = {"workload": WORKLOADS[wl]["desc"], "metric": WORKLOADS[wl]["metric"],
           "value": float(np.mean(step_s)), "unit": UNIT,
           "stage_ms": dict(zip(STAGES, [float(x) / 5 for x in kms])),
           "vale_dim": g.vale_dim, "core_dim": g.core_dim, "pot_terms": g.pot_dim,
           "pair_images": g.num_pair_images, "shell_pairs": g.num_shell_pairs,
           "gpu_launches": int(launches), "clocks": clk.summary(),
           "schedule": schedules(g, bufs, stream, flush, torch),
           "contract": g.contract_tuning(),
           "prim3c_roofline": prim3c_roofline(g, bufs, stream, flush, torch,
                                              fp64_peak_tflops(torch))}
    if not args.no_adjacent:
        out["adjacent_builds"] = adjacent_builds(g, bufs, stream, torch, dev, reps=3,
                                                 ham_mode=args.ham_mode)
    g.close()
    out["e2e"] = time_e2e(system, local, stream, bufs, 3, torch)
    del bufs, flush
    torch.cuda.empty_cache()
    if not args.skip_cpu:
        ncores = os.cpu_count() or 1
        v, wall, what = cpu_baseline(system, ncores, wl)
        out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": ncores,
                               "kind": "port",
                               "sample": (f"oracle (CPU restatement, OpenMP over "
                                          f"atom pairs): {what}; {wall:.1f} s wall")}
        if not args.no_full_cpu:
            # the same build run once in full: every atom pair, every EP
            # term's own orthogonalisation
            t0 = time.perf_counter()
            full = oracle_build_time(system, ncores)
            out["cpu_full"] = {"value": full, "unit": UNIT, "cores": ncores, "kind": "port",
                               "sample": "the full build, run once",
                               "wall_s": time.perf_counter() - t0,
                               "sampled_over_full": v / full}
            out["speedup_vs_cpu_full"] = {"device": full / out["value"],
                                          "e2e": full / out["e2e"]["value"]}
    out["quartz_222"] = quartz_222(args, local, torch)
    return out


def schedules(g, bufs, stream, flush, torch, steps=3):
    """The three-centre stage's schedules on the context's build: per-class
    launches, the persistent work-queue launch and per-class launches with
    two EP terms per thread (device seconds of
    whole builds replayed from graphs, and the primitive stage's ms with the
    kinds serialised), the measured choice the context made, and back to
    the measured choice."""
    out = {"chosen": g.schedule()}
    for mode in ("per_class", "queue", "pairs"):
        g.set_schedule(mode)
        g.build_graph({k: v.data_ptr() for k, v in bufs.items()})
        torch.cuda.synchronize()
        step_s, kms, _ = time_device_builds(g, bufs, stream, steps, flush, torch)
        out[mode] = {"build_s": float(np.mean(step_s)), "prim_ms": float(kms[0]) / steps}
    g.set_schedule(out["chosen"]["schedule"])
    return out


def quartz_222(args, local, torch):
    """The same cell at 2x2x2 k (8 k-points): device time of the graph
    replay, end to end, and the oracle on the host cores (sampled as for
    Gamma: every 8th atom pair, the EP orthogonalisations timed on KE and
    NP)."""
    from imago_b200 import intg
    wl = "quartz-222"
    system = system_for(wl)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=local)
    g = intg.IntegralSetup(system, device=local, outputs_on_device=True,
                           stream=stream.cuda_stream)
    bufs = device_outputs(g, torch, dev)
    flush = torch.empty(512 * 1024 * 1024 // 8, dtype=torch.float64, device=dev)
    for _ in range(2):
        g.build_graph({k: v.data_ptr() for k, v in bufs.items()})
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        step_s, kms, launches = time_device_builds(g, bufs, stream, 3, flush, torch)
    out = {"workload": WORKLOADS[wl]["desc"], "value": float(np.mean(step_s)), "unit": UNIT,
           "stage_ms": dict(zip(STAGES, [float(x) / 3 for x in kms])),
           "gpu_launches": int(launches), "clocks": clk.summary(),
           "schedule": schedules(g, bufs, stream, flush, torch)}
    g.close()
    out["e2e"] = time_e2e(system, local, stream, bufs, 2, torch)
    del bufs, flush
    torch.cuda.empty_cache()
    if not args.skip_cpu:
        ncores = os.cpu_count() or 1
        v, wall, what = cpu_baseline(system, ncores, wl)
        out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": ncores, "kind": "port",
                               "sample": (f"oracle (CPU restatement, OpenMP over "
                                          f"atom pairs): {what}; {wall:.1f} s wall")}
        out["speedup_vs_cpu"] = {"device": v / out["value"], "e2e": v / out["e2e"]["value"]}
    return out


STAGES = ["prim", "contract", "bloch", "ortho"]


def run_batch(args):
    """The batched workload on one GPU: all cells' builds as one CUDA graph
    (imago_batch_build), outputs resident in HBM."""
    import torch
    from imago_b200 import intg
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    wl = WORKLOADS["batch64"]
    cells = system_for("batch64", rank)
    stream = torch.cuda.Stream()
    dev = torch.device("cuda", local)
    b = intg.IntegralBatch(cells, device=local, stream=stream.cuda_stream)
    outs = [{k: torch.empty(v, dtype=torch.float64, device=dev)
             for k, v in b.output_shapes(i).items()} for i in range(len(b))]
    out_bytes = [sum(t.numel() * 8 for t in o.values()) for o in outs]
    flush = torch.empty(512 * 1024 * 1024 // 8, dtype=torch.float64, device=dev)
    t0 = time.perf_counter()
    b.build(outs)  # eager build of every cell + graph capture
    first = time.perf_counter() - t0
    for _ in range(args.warmup):
        b.build(outs)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    step_s = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                s = torch.cuda.Event(enable_timing=True)
                e = torch.cuda.Event(enable_timing=True)
                s.record(stream)
            b.build(outs)
            e.record(stream)
            e.synchronize()
            step_s.append(s.elapsed_time(e) / 1e3)
    total = float(np.sum(step_s))
    if world > 1:
        t = torch.tensor([total], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total = float(t.item())
    value = total / args.steps
    launches = b.graph_launches()
    b.close()
    del outs, flush
    torch.cuda.empty_cache()

    # end to end: create the batch (host set-up and staging of 64 cells),
    # build (eager + capture) and copy every output into pinned host memory
    stage = torch.empty(max(out_bytes) // 8, dtype=torch.float64, pin_memory=True)
    e2e = []
    for i in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b2 = intg.IntegralBatch(cells, device=local, stream=stream.cuda_stream)
        o2 = [{k: torch.empty(v, dtype=torch.float64, device=dev)
               for k, v in b2.output_shapes(j).items()} for j in range(len(b2))]
        b2.build(o2)
        for o in o2:
            off = 0
            for t in o.values():
                n = t.numel()
                stage[off:off + n].copy_(t.reshape(-1))
                off += n
        torch.cuda.synchronize()
        if i > 0:
            e2e.append(time.perf_counter() - t0)
        b2.close()
        del o2
        torch.cuda.empty_cache()
    if rank == 0:
        cpu = None
        if world == 1 and not args.skip_cpu:
            ncores = os.cpu_count() or 1
            v, wall, what = cpu_baseline(cells, ncores, "batch64")
            cpu = {"value": v, "unit": UNIT, "cores": ncores, "kind": "port",
                   "sample": (f"oracle (CPU restatement, OpenMP over atom "
                              f"pairs): {what}; {wall:.1f} s wall")}
        atoms = [len(c.site_type) for c in cells]
        line = {
            "metric": wl["metric"], "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": value * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded strain and jitter, synthesised contraction coefficients)",
            "config": {"workload": wl["desc"], "l2": "512 MiB flush between steps",
                       "cells": len(cells), "atoms_min": min(atoms),
                       "atoms_max": max(atoms), "atoms_total": int(sum(atoms)),
                       "output_bytes": int(sum(out_bytes))},
            "e2e": {"value": float(np.mean(e2e)), "unit": UNIT,
                    "h2d_bytes_per_step": int(sum(_system_bytes(c) for c in cells)),
                    "d2h_bytes_per_step": int(sum(out_bytes))},
            "first_build_s": first,
            "gpu_launches": int(launches),
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def run_sharded(args):
    """--shard terms: one system's build spread over the ranks
    (imago_b200.shard): every rank builds the overlap and its block of the
    KE, NP and EP matrices, then one gather brings all of them to rank 0.
    Strong scaling: the work of the whole job is fixed."""
    import datetime
    import torch
    import torch.distributed as dist
    from imago_b200 import intg, shard
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", "29517")
    dist.init_process_group("nccl" if world > 1 else "gloo", rank=rank,
                            world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    wl = WORKLOADS[args.workload]
    system = system_for(args.workload, 0, args.kmesh)  # the same cell everywhere
    stream = torch.cuda.Stream(device=local)
    g = intg.IntegralSetup(system, device=local, outputs_on_device=True,
                           stream=stream.cuda_stream)
    sb = shard.ShardedBuild.from_setup(g)
    for _ in range(args.warmup):
        sb.build()
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    step_s = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record(stream)
            with torch.cuda.stream(stream):
                sb.build()
            e.record(stream)
            e.synchronize()
            step_s.append(s.elapsed_time(e) / 1e3)
    torch.cuda.synchronize()
    dist.barrier()
    t = torch.tensor([float(np.sum(step_s))], dtype=torch.float64,
                     device=torch.device("cuda", local) if world > 1 else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    value = float(t.item()) / args.steps
    if rank == 0:
        line = {
            "metric": wl["metric"], "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3,
            "higher_is_better": False, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded jitter, synthesised contraction coefficients)",
            "config": {"workload": wl["desc"], "parallelism": f"terms{world}",
                       "shard": "overlap on every rank, KE/NP/EP matrices in "
                                "contiguous blocks per rank, one gather to rank 0",
                       "parts": shard.partition(g.pot_dim, world)},
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    g.close()
    dist.destroy_process_group()


def run_ours(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from imago_b200 import intg

    wl = WORKLOADS[args.workload]
    system = system_for(args.workload, rank, args.kmesh)
    # the library runs on this stream, and the timing events are recorded on
    # it, so they bracket exactly the build's work
    stream = torch.cuda.Stream(device=local)
    g = intg.IntegralSetup(system, device=local, outputs_on_device=True,
                           stream=stream.cuda_stream,
                           scratch_bytes=args.scratch_mb << 20)
    nk, V, C, P = g.nk, g.vale_dim, g.core_dim, g.pot_dim
    dev = torch.device("cuda", local)
    bufs = device_outputs(g, torch, dev)
    flush = torch.empty(512 * 1024 * 1024 // 8, dtype=torch.float64, device=dev)

    for _ in range(args.warmup):  # the first also captures the graph
        g.build_graph({k: v.data_ptr() for k, v in bufs.items()})
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        step_s, kms, launches = time_device_builds(g, bufs, stream, args.steps,
                                                   flush, torch)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    total = float(np.sum(step_s))
    if world > 1:
        t = torch.tensor([total], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total = float(t.item())
    value = total / args.steps
    kms /= args.steps

    tuning = g.tuning()
    tuning["prim3c"] = g.schedule()
    tuning["ortho"] = g.ortho_schedule()
    tuning["contract"] = g.contract_tuning()
    secular_s = time_secular(bufs, P, stream, torch)
    # the valence-charge step as measured on the Si8 mesh (V = 104, within
    # the library's reduction kernels); the SCF cells beyond are in `scf`
    valence = time_valence_rho(bufs, P, stream, torch) if args.workload == "si8" else None
    adjacent = None
    if world == 1 and args.workload == "si8" and not args.no_adjacent:
        adjacent = adjacent_builds(g, bufs, stream, torch, dev, ham_mode=args.ham_mode)
    e2e = time_e2e(system, local, stream, bufs, 5, torch)

    flops = algorithmic_flops(g)
    fp64 = fp64_peak_tflops(torch) if rank == 0 else None
    prim3c = prim3c_roofline(g, bufs, stream, flush, torch, fp64) if rank == 0 else None
    top = int(np.argmax(kms))
    top_name = STAGES[top]
    roofline = None
    if top_name in flops and fp64:
        achieved = flops[top_name] / (kms[top] / 1e3) / 1e12
        traffic = None
        if top_name == "ortho" and args.workload == "si8":
            traffic = ORTHO_FUSED_BYTES_PER_KMAT * nk * (3 + P)
        roofline = {"bound": "tensor", "achieved": achieved, "peak": fp64,
                    "unit": "TFLOP/s", "frac": achieved / fp64, "traffic": traffic,
                    "traffic_unit": "bytes per build (ncu, scaled by (k, matrix) pairs)",
                    "kernel": top_name,
                    "peak_source": "measured cuBLAS DGEMM 8192^3 in this run "
                                   "(MEASURED_PEAKS.json has no FP64 figure)"}
    if rank == 0:
        cpu = None
        if world == 1 and not args.skip_cpu:
            ncores = os.cpu_count() or 1
            v, wall, what = cpu_baseline(system, ncores, args.workload)
            cpu = {"value": v, "unit": UNIT, "cores": ncores, "kind": "port",
                   "sample": (f"oracle (CPU restatement, OpenMP over atom "
                              f"pairs): {what}; {wall:.1f} s wall")}
        line = {
            "metric": wl["metric"], "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": value * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded jitter, synthesised contraction coefficients)",
            "config": {"workload": wl["desc"], "l2": "512 MiB flush between steps",
                       "launch": "one CUDA graph per build (imago_intg_build_graph)",
                       "vale_dim": V, "core_dim": C, "kpoints": nk, "pot_terms": P,
                       "pair_images": g.num_pair_images,
                       "shell_pairs": g.num_shell_pairs},
            "e2e": e2e,
            "gpu_launches": int(launches),
            "stage_ms": dict(zip(STAGES, [float(x) for x in kms])),
            "shell_pairs_per_s": g.num_shell_pairs * (3 + P) / value,
            "roofline": roofline,
            "prim3c_roofline": prim3c if rank == 0 else None,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "tuning": tuning,
            "secular_step_s": secular_s,
            **({"valence_rho": valence} if valence else {}),
        }
        if adjacent:
            line["adjacent_builds"] = adjacent
        if args.workload == "si8" and list(args.kmesh) != [8, 8, 8]:
            line["note"] = (f"k-mesh {args.kmesh} (profiling case, not the "
                            f"measured workload)")
        g.close()
        del bufs, flush
        torch.cuda.empty_cache()
        if world == 1 and args.workload == "si8" and not args.no_silica:
            line["silica_162"] = silica_headline(args, local, stream, torch)
        if world == 1 and args.workload == "si8" and not args.no_scf:
            torch.cuda.synchronize(local)
            torch.cuda.empty_cache()
            line["scf"] = scf_headline(local, torch)
        print(json.dumps(line), flush=True)
    g.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def _system_bytes(system):
    s, keep = system.to_c()
    return int(sum(a.nbytes for a in keep)) + 9 * 8


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--workload", default="si8", choices=sorted(WORKLOADS))
    ap.add_argument("--kmesh", type=int, nargs=3, default=[8, 8, 8],
                    help="k-mesh of the Si8 cell; the measured workload is 8 8 8, "
                         "smaller meshes are for profiling captures")
    ap.add_argument("--scratch-mb", type=int, default=0,
                    help="device scratch budget of the EP chunks (0: a quarter "
                         "of free memory); small budgets are for profiling")
    ap.add_argument("--shard", default="none", choices=["none", "terms"],
                    help="under torchrun: 'none' builds an independent cell per "
                         "rank (weak scaling); 'terms' spreads one cell's "
                         "matrices over the ranks (strong scaling)")
    ap.add_argument("--no-silica", action="store_true",
                    help="skip the 162-atom quartz report of the default run")
    ap.add_argument("--ham-mode", default="auto",
                    choices=["auto", "blocks", "fused", "fused1"],
                    help="how the PSCF Hamiltonian of the adjacent builds sums "
                         "its potential terms (profiling the fused kernel on a "
                         "small case)")
    ap.add_argument("--no-full-cpu", action="store_true",
                    help="skip the one unsampled oracle run of the quartz Gamma "
                         "build in the default line")
    ap.add_argument("--no-scf", action="store_true",
                    help="skip the SCF runs (plain and learned start) of the "
                         "default line")
    ap.add_argument("--no-adjacent", action="store_true",
                    help="skip the timings of the mass-velocity, momentum, "
                         "dipole and PSCF Hamiltonian builds")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch64":
        run_batch(args)
    elif args.shard == "terms":
        run_sharded(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
