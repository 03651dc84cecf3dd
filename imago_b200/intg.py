"""Python mirror of the integral-setup calls in Imago's setupSCF.

The four builds keep the reference's names and meaning
(src/imago/imago.F90:262-293):

    gauss_overlap_ol()       -> gaussOverlapOL       (integrals.F90:151)
    gauss_overlap_ke()       -> gaussOverlapKE       (integrals.F90:656)
    gauss_overlap_np()       -> gaussOverlapNP       (integrals.F90:1531)
    elec_pot_gauss_overlap() -> elecPotGaussOverlap  (integrals.F90:2357)

Each returns the packed valence-valence matrices exactly as the reference
writes them to HDF5: an array [nk, valeDim*(valeDim+1)/2, 2] of (re, im)
per packed upper-triangle element (EP: one such array per potential term).
The overlap also returns coreValeOL as (re, im) arrays [nk, valeDim,
coreDim].  Where the reference would `stop`, these raise ImagoError with
the reference's message.

All work runs in libimago_b200.so on a compute-capability 10.0 GPU; there
is no CPU path.
"""

import ctypes
import os

import numpy as np

from .system import ImagoDimsC

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libimago_b200.so")

IMAGO_OL, IMAGO_KE, IMAGO_NP, IMAGO_EP, IMAGO_MV = 1, 2, 4, 8, 16
IMAGO_ERR_NO_DEVICE = 7

_LIB = None
_D = ctypes.POINTER(ctypes.c_double)


class ImagoError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = lib().imago_strerror(status).decode()
        super().__init__(f"{what}: {msg} (status {status})" if what else msg)


class ImagoOptsC(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("stream", ctypes.c_void_p),
                ("outputs_on_device", ctypes.c_int),
                ("scratch_bytes", ctypes.c_size_t)]


class ImagoOutC(ctypes.Structure):
    _fields_ = [("ol_packed", _D), ("ol_cv_re", _D), ("ol_cv_im", _D),
                ("ke_packed", _D), ("np_packed", _D), ("ep_packed", _D),
                ("mv_packed", _D)]


def lib():
    """Load libimago_b200.so; raise if it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m imago_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        L.imago_intg_create.argtypes = [ctypes.c_void_p, ctypes.POINTER(ImagoOptsC),
                                        ctypes.POINTER(ctypes.c_void_p)]
        L.imago_intg_create.restype = ctypes.c_int
        L.imago_intg_dims.argtypes = [ctypes.c_void_p, ctypes.POINTER(ImagoDimsC)]
        L.imago_intg_dims.restype = ctypes.c_int
        L.imago_gauss_overlap_ol.argtypes = [ctypes.c_void_p, _D, _D, _D]
        L.imago_gauss_overlap_ol.restype = ctypes.c_int
        for n in ("imago_gauss_overlap_ke", "imago_gauss_overlap_np", "imago_gauss_overlap_mv",
                  "imago_gauss_overlap_mm",
                  "imago_elec_pot_gauss_overlap"):
            getattr(L, n).argtypes = [ctypes.c_void_p, _D]
            getattr(L, n).restype = ctypes.c_int
        L.imago_gauss_overlap_dm.argtypes = [ctypes.c_void_p, _D, _D]
        L.imago_gauss_overlap_dm.restype = ctypes.c_int
        L.imago_gauss_koverlap.argtypes = [ctypes.c_void_p, _D, _D, _D]
        L.imago_gauss_koverlap.restype = ctypes.c_int
        L.imago_intg_set_ham_mode.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.imago_intg_set_ham_mode.restype = ctypes.c_int
        L.imago_ham_pscf.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, ctypes.c_int, _D]
        L.imago_ham_pscf.restype = ctypes.c_int
        L.imago_elec_pot_gauss_overlap_range.argtypes = [ctypes.c_void_p, ctypes.c_int,
                                                         ctypes.c_int, _D]
        L.imago_elec_pot_gauss_overlap_range.restype = ctypes.c_int
        L.imago_intg_build.argtypes = [ctypes.c_void_p, ctypes.c_uint,
                                       ctypes.POINTER(ImagoOutC)]
        L.imago_intg_build.restype = ctypes.c_int
        L.imago_intg_stage_ms.argtypes = [ctypes.c_void_p, _D]
        L.imago_intg_stage_ms.restype = ctypes.c_int
        L.imago_intg_kernel_stats.argtypes = [ctypes.c_void_p, _D,
                                              ctypes.POINTER(ctypes.c_longlong)]
        L.imago_intg_kernel_stats.restype = ctypes.c_int
        L.imago_intg_destroy.argtypes = [ctypes.c_void_p]
        L.imago_intg_destroy.restype = None
        L.imago_intg_set_serial.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.imago_intg_set_serial.restype = ctypes.c_int
        L.imago_intg_tuning.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), _D]
        L.imago_intg_tuning.restype = ctypes.c_int
        L.imago_intg_set_schedule.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.imago_intg_set_schedule.restype = ctypes.c_int
        L.imago_intg_schedule.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), _D]
        L.imago_intg_schedule.restype = ctypes.c_int
        L.imago_intg_set_ortho_schedule.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.imago_intg_set_ortho_schedule.restype = ctypes.c_int
        L.imago_intg_ortho_schedule.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                                _D]
        L.imago_intg_ortho_schedule.restype = ctypes.c_int
        L.imago_trim_memory.argtypes = [ctypes.c_int]
        L.imago_trim_memory.restype = ctypes.c_int
        L.imago_intg_contract_tuning.argtypes = [ctypes.c_void_p,
                                                 ctypes.POINTER(ctypes.c_int), _D]
        L.imago_intg_contract_tuning.restype = ctypes.c_int
        L.imago_intg_count_triples.argtypes = [ctypes.c_void_p, ctypes.c_uint,
                                               ctypes.POINTER(ctypes.c_longlong)]
        L.imago_intg_count_triples.restype = ctypes.c_int
        L.imago_wait_check.argtypes = [ctypes.c_int, ctypes.c_double,
                                       ctypes.POINTER(ctypes.c_int)]
        L.imago_wait_check.restype = ctypes.c_int
        L.imago_intg_build_graph.argtypes = [ctypes.c_void_p, ctypes.c_uint,
                                             ctypes.POINTER(ImagoOutC)]
        L.imago_intg_build_graph.restype = ctypes.c_int
        L.imago_batch_create.argtypes = [ctypes.c_int, ctypes.c_void_p,
                                         ctypes.POINTER(ImagoOptsC),
                                         ctypes.POINTER(ctypes.c_void_p)]
        L.imago_batch_create.restype = ctypes.c_int
        L.imago_batch_size.argtypes = [ctypes.c_void_p]
        L.imago_batch_size.restype = ctypes.c_int
        L.imago_batch_dims.argtypes = [ctypes.c_void_p, ctypes.c_int,
                                       ctypes.POINTER(ImagoDimsC)]
        L.imago_batch_dims.restype = ctypes.c_int
        L.imago_batch_build.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p]
        L.imago_batch_build.restype = ctypes.c_int
        L.imago_batch_launches.argtypes = [ctypes.c_void_p,
                                           ctypes.POINTER(ctypes.c_longlong)]
        L.imago_batch_launches.restype = ctypes.c_int
        L.imago_batch_destroy.argtypes = [ctypes.c_void_p]
        L.imago_batch_destroy.restype = None
        L.imago_strerror.argtypes = [ctypes.c_int]
        L.imago_strerror.restype = ctypes.c_char_p
        L.imago_kpoint_mesh.argtypes = [ctypes.POINTER(ctypes.c_int), _D, _D]
        L.imago_kpoint_mesh.restype = ctypes.c_int
        L.imago_prim_eval.argtypes = [ctypes.c_int, ctypes.c_int, _D,
                                      ctypes.POINTER(ctypes.c_int), _D]
        L.imago_prim_eval.restype = ctypes.c_int
        L.imago_prim_eval_static.argtypes = [ctypes.c_int, ctypes.c_int, _D,
                                             ctypes.POINTER(ctypes.c_int), _D]
        L.imago_prim_eval_static.restype = ctypes.c_int
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(_D)


def _check(st, what):
    if st != 0:
        raise ImagoError(st, what)


def trim_memory(device=0):
    """Hand the unused memory of the library's device pool back to the
    driver (contexts keep taking scratch from the pool afterwards)."""
    _check(lib().imago_trim_memory(device), "imago_trim_memory")


def wait_check(device=0, limit_ms=5.0):
    """The library's bounded device wait run out on purpose
    (imago_wait_check): a barrier that nothing completes, given up after
    limit_ms.  Returns the status the kernel recorded (IMAGO_ERR_TIMEOUT, 6,
    when the bound works)."""
    st = ctypes.c_int(-1)
    _check(lib().imago_wait_check(device, float(limit_ms), ctypes.byref(st)),
           "imago_wait_check")
    return st.value


def kpoint_mesh(n, shift=(0.0, 0.0, 0.0)):
    """k-point mesh made by the library (kpoints.f90:896-899, no folding)."""
    n3 = (ctypes.c_int * 3)(*[int(x) for x in n])
    sh = np.ascontiguousarray(shift, dtype=np.float64)
    out = np.zeros((int(np.prod(n)), 3))
    _check(lib().imago_kpoint_mesh(n3, _p(sh), _p(out)), "imago_kpoint_mesh")
    return out


PRIM_KINDS = {"overlap": 0, "kinetic": 1, "electron3c": 2, "nuclear3c": 3,
              "boys": 4, "massvel": 5,
              "momentum_x": 6, "momentum_y": 7, "momentum_z": 8,
              "dipole_x": 9, "dipole_y": 10, "dipole_z": 11}


def prim_eval(kind, params, cls=None):
    """Evaluate primitive integrals on the GPU.  params: [n, 12] rows
    (a1, a2, a3, A, B, C); cls: [n, 2] (l of atom 1, l of atom 2).
    Returns [n, 16, 16] in the reference's sh layout."""
    params = np.ascontiguousarray(params, dtype=np.float64).reshape(-1, 12)
    n = len(params)
    c = (np.ascontiguousarray(cls, dtype=np.int32).reshape(-1, 2) if cls is not None
         else np.zeros((n, 2), np.int32))
    out = np.zeros((n, 256))
    st = lib().imago_prim_eval(PRIM_KINDS[kind], n, _p(params),
                               c.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                               _p(out))
    _check(st, "imago_prim_eval")
    return out.reshape(n, 16, 16)


PRIM_STATIC_MAX_RECORDS = 512


def prim_eval_static(kind, params, cls=None):
    """prim_eval through imago_prim_eval_static, which stages the records in
    a fixed device array instead of allocating: for callers that must not
    call cudaMalloc (a GPU shared under a fixed memory budget, device memory
    owned by a pool allocator, or a loop that cannot afford the
    synchronisation of cudaMalloc/cudaFree).  At most
    PRIM_STATIC_MAX_RECORDS records per call; calls must not overlap on the
    GPU, since they share the array."""
    params = np.ascontiguousarray(params, dtype=np.float64).reshape(-1, 12)
    n = len(params)
    c = (np.ascontiguousarray(cls, dtype=np.int32).reshape(-1, 2) if cls is not None
         else np.zeros((n, 2), np.int32))
    out = np.zeros((n, 256))
    st = lib().imago_prim_eval_static(PRIM_KINDS[kind], n, _p(params),
                                      c.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                      _p(out))
    _check(st, "imago_prim_eval_static")
    return out.reshape(n, 16, 16)


_OUT_NAMES = ("ol_packed", "ol_cv_re", "ol_cv_im", "ke_packed", "np_packed",
              "ep_packed", "mv_packed")


def _out_struct(out):
    s = ImagoOutC()
    for name in _OUT_NAMES:
        v = out.get(name)
        if v is None:
            setattr(s, name, _D())
        elif isinstance(v, int):
            setattr(s, name, ctypes.cast(ctypes.c_void_p(v), _D))
        elif hasattr(v, "data_ptr"):
            setattr(s, name, ctypes.cast(ctypes.c_void_p(v.data_ptr()), _D))
        else:
            setattr(s, name, _p(v))
    return s


def koverlap_wave_vectors(system, num_axial=None):
    """The wave vectors of the reference's gaussKOverlap
    (integrals3Terms.F90:1293-1297): recipVectors(:, c) / numAxialKPoints(c)
    as rows c of a [3, 3] array (bohr^-1), recipVectors as
    initializeLattice forms them (lattice.f90:200-214).  num_axial
    defaults to the system's k-point mesh, else one point per axis."""
    a = np.asarray(system.real_vectors, dtype=np.float64)
    recip = 2.0 * np.pi * np.linalg.inv(a).T
    if num_axial is None:
        num_axial = system.kmesh[0] if system.kmesh is not None else (1, 1, 1)
    return recip / np.asarray(num_axial, dtype=np.float64)[:, None]


class IntegralSetup:
    """One system staged on the GPU: imago_intg_create .. imago_intg_destroy.

    outputs_on_device=True makes the build methods take torch CUDA tensors
    (or raw device pointers) instead of returning numpy arrays."""

    def __init__(self, system, device=0, outputs_on_device=False,
                 scratch_bytes=0, stream=None):
        self.system = system
        self._cs, self._keep = system.to_c()
        opts = ImagoOptsC(device, stream, 1 if outputs_on_device else 0,
                          scratch_bytes)
        self._ctx = ctypes.c_void_p()
        st = lib().imago_intg_create(ctypes.byref(self._cs), ctypes.byref(opts),
                                     ctypes.byref(self._ctx))
        _check(st, "imago_intg_create")
        d = ImagoDimsC()
        lib().imago_intg_dims(self._ctx, ctypes.byref(d))
        self.vale_dim, self.core_dim = d.vale_dim, d.core_dim
        self.nk, self.pot_dim, self.num_cells = d.num_kpoints, d.pot_dim, d.num_cells
        self.npacked = int(d.packed)
        self.num_pair_images = int(d.num_pair_images)
        self.num_shell_pairs = int(d.num_shell_pairs)
        self.block_elements = int(d.block_elements)
        self.outputs_on_device = outputs_on_device

    def close(self):
        if self._ctx:
            lib().imago_intg_destroy(self._ctx)
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

    # -- host-output builds (reference layout, numpy) --
    def _device_only(self, out, what):
        """A device-output context's kernels write straight through the
        output pointers, so host (numpy) memory there, or no output at all,
        is refused before the library is called."""
        if self.outputs_on_device and (out is None or isinstance(out, np.ndarray)):
            raise ValueError(f"{what}: this context writes device memory; pass CUDA "
                             "tensors or device pointers")

    def _packed(self, n=None):
        self._device_only(None, "a host output")
        shape = (self.nk, self.npacked, 2) if n is None else (n, self.nk, self.npacked, 2)
        return np.zeros(shape)

    def gauss_overlap_ol(self):
        out = self._packed()
        c = max(self.core_dim, 1)
        re = np.zeros((self.nk, self.vale_dim, c))
        im = np.zeros_like(re)
        _check(lib().imago_gauss_overlap_ol(self._ctx, _p(out), _p(re), _p(im)),
               "gaussOverlapOL")
        return out, re[:, :, :self.core_dim], im[:, :, :self.core_dim]

    def gauss_overlap_ke(self):
        out = self._packed()
        _check(lib().imago_gauss_overlap_ke(self._ctx, _p(out)), "gaussOverlapKE")
        return out

    def gauss_overlap_np(self):
        out = self._packed()
        _check(lib().imago_gauss_overlap_np(self._ctx, _p(out)), "gaussOverlapNP")
        return out

    def gauss_overlap_mv(self):
        """Mass velocity (imago_gauss_overlap_mv), the scalar-relativistic
        term of rel = 1 runs; needs the overlap first when coreDim > 0."""
        out = self._packed()
        _check(lib().imago_gauss_overlap_mv(self._ctx, _p(out)), "gaussOverlapMV")
        return out

    def _ptr(self, out):
        self._device_only(out, "an output")
        if isinstance(out, int):
            return ctypes.cast(ctypes.c_void_p(out), _D)
        if hasattr(out, "data_ptr"):
            return ctypes.cast(ctypes.c_void_p(out.data_ptr()), _D)
        return _p(out)

    def set_schedule(self, mode):
        """How the three-centre primitive stage schedules its classes
        (imago_intg_set_schedule): "auto" (all measured on the first EP
        build, the fastest kept), "per_class" (one launch per class),
        "queue" (one persistent launch fed by a device work queue) or
        "pairs" (one launch per class, two EP terms of a type per thread)."""
        m = {"auto": -1, "per_class": 0, "queue": 1, "pairs": 2}[mode]
        _check(lib().imago_intg_set_schedule(self._ctx, m), "imago_intg_set_schedule")

    def schedule(self):
        """{"schedule": "per_class" | "queue" | "pairs",
        "trial_ms": [per class, queue, pairs]}"""
        s = ctypes.c_int()
        ms = np.zeros(3)
        _check(lib().imago_intg_schedule(self._ctx, ctypes.byref(s), _p(ms)),
               "imago_intg_schedule")
        return {"schedule": ("per_class", "queue", "pairs")[s.value], "trial_ms": ms.tolist()}

    def set_ortho_schedule(self, mode):
        """How EP builds of several terms run the core orthogonalisation
        (imago_intg_set_ortho_schedule): "auto" (both measured on the first
        EP build, the faster kept), "per_item" (one CTA per k-point and
        term) or "piped" (one persistent CTA per SM, the overlap block
        resident, the next term's block brought in by TMA meanwhile)."""
        m = {"auto": -1, "per_item": 0, "piped": 1}[mode]
        _check(lib().imago_intg_set_ortho_schedule(self._ctx, m),
               "imago_intg_set_ortho_schedule")

    def ortho_schedule(self):
        """{"schedule": "per_item" | "piped", "trial_ms": [per item, piped]}"""
        s = ctypes.c_int()
        ms = np.zeros(2)
        _check(lib().imago_intg_ortho_schedule(self._ctx, ctypes.byref(s), _p(ms)),
               "imago_intg_ortho_schedule")
        return {"schedule": ("per_item", "piped")[s.value], "trial_ms": ms.tolist()}

    def contract_tuning(self):
        """{"terms_per_cta": 4 | 8, "trial_ms": [4, 8]}: the contraction's
        measured terms per CTA (imago_intg_contract_tuning)."""
        n = ctypes.c_int()
        ms = np.zeros(2)
        _check(lib().imago_intg_contract_tuning(self._ctx, ctypes.byref(n), _p(ms)),
               "imago_intg_contract_tuning")
        return {"terms_per_cta": n.value, "trial_ms": ms.tolist()}

    def count_triples(self, which):
        """Screened primitive triples (shell pair, site, image) per class of
        the NP build (which=IMAGO_NP) or of every EP term (IMAGO_EP), as an
        int64 [4, 4] array indexed (l_a, l_b); -1 for f classes present."""
        c = np.zeros(16, dtype=np.int64)
        _check(lib().imago_intg_count_triples(
            self._ctx, which, c.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))),
            "imago_intg_count_triples")
        return c.reshape(4, 4)

    def set_ham_mode(self, mode):
        """How ham_pscf sums the potential terms (imago_intg_set_ham_mode):
        "auto", "blocks" (per-term blocks added with their weights),
        "fused" (all terms of a shell pair in registers, a pass per spin,
        four lanes per shell pair on small systems) or "fused1" (one lane)."""
        m = {"auto": 0, "blocks": 1, "fused": 2, "fused1": 3}[mode]
        _check(lib().imago_intg_set_ham_mode(self._ctx, m), "imago_intg_set_ham_mode")

    def gauss_overlap_mm(self, out=None):
        """Momentum matrices -i<a|d/dx_c|b>, c = x, y, z
        (imago_gauss_overlap_mm): [3, nk, nPacked, 2]."""
        if out is None:
            out = self._packed(3)
        _check(lib().imago_gauss_overlap_mm(self._ctx, self._ptr(out)), "gaussOverlapMM")
        return out

    def gauss_overlap_dm(self, center, out=None):
        """Dipole matrices <a|(r - center)_c|b> (imago_gauss_overlap_dm):
        [3, nk, nPacked, 2]."""
        c = np.ascontiguousarray(center, dtype=np.float64).reshape(3)
        if out is None:
            out = self._packed(3)
        _check(lib().imago_gauss_overlap_dm(self._ctx, _p(c), self._ptr(out)),
               "gaussOverlapDM")
        return out

    def gauss_koverlap(self, dk, re=None, im=None):
        """The overlap with a plane wave <a|exp(-i dK_c . r)|b> for three
        wave vectors dk [3, 3] (row c is dK_c, bohr^-1)
        (imago_gauss_koverlap): full complex matrices, returned as real and
        imaginary planes [3, nk, V, V] indexed [c, k, col, row]."""
        q = np.ascontiguousarray(dk, dtype=np.float64).reshape(9)
        shape = (3, self.nk, self.vale_dim, self.vale_dim)
        if re is None:
            self._device_only(None, "gauss_koverlap re")
            re = np.zeros(shape)
        if im is None:
            self._device_only(None, "gauss_koverlap im")
            im = np.zeros(shape)
        _check(lib().imago_gauss_koverlap(self._ctx, _p(q), self._ptr(re), self._ptr(im)),
               "gaussKOverlap")
        return re, im

    def ham_pscf(self, coeffs, rel=False, out=None):
        """The PSCF Hamiltonian (imago_ham_pscf): coeffs [potDim] or
        [potDim, spin] -> [spin, nk, nPacked, 2]; kinetic + nuclear +
        coefficient-weighted potential terms, minus mass velocity when rel.
        `out` a device pointer/tensor for outputs_on_device contexts."""
        c = np.asarray(coeffs, dtype=np.float64)
        if c.ndim == 1:
            c = c[:, None]
        if c.shape[0] != self.pot_dim or c.shape[1] not in (1, 2):
            raise ValueError("coeffs must be [potDim] or [potDim, spin]")
        spin = c.shape[1]
        cf = np.ascontiguousarray(c.T)  # potCoeffs(potDim, spin) column-major
        if out is None:
            out = self._packed(spin)
        self._device_only(out, "ham_pscf")
        ptr = (ctypes.cast(ctypes.c_void_p(out), _D) if isinstance(out, int) else
               ctypes.cast(ctypes.c_void_p(out.data_ptr()), _D) if hasattr(out, "data_ptr")
               else _p(out))
        _check(lib().imago_ham_pscf(self._ctx, spin, _p(cf), 1 if rel else 0, ptr),
               "gaussOverlapHamPSCF")
        return out

    def elec_pot_gauss_overlap(self):
        out = self._packed(self.pot_dim)
        _check(lib().imago_elec_pot_gauss_overlap(self._ctx, _p(out)),
               "elecPotGaussOverlap")
        return out

    def elec_pot_gauss_overlap_range(self, first, count, out=None):
        """EP terms first .. first+count-1 (imago_elec_pot_gauss_overlap_range);
        `out` a device pointer/tensor for outputs_on_device contexts."""
        if out is None:
            out = self._packed(count)
        self._device_only(out, "elec_pot_gauss_overlap_range")
        ptr = (ctypes.cast(ctypes.c_void_p(out), _D) if isinstance(out, int) else
               ctypes.cast(ctypes.c_void_p(out.data_ptr()), _D) if hasattr(out, "data_ptr")
               else _p(out))
        _check(lib().imago_elec_pot_gauss_overlap_range(self._ctx, first, count, ptr),
               "elecPotGaussOverlap terms")
        return out

    # -- all matrices in one call --
    def build(self, which=IMAGO_OL | IMAGO_KE | IMAGO_NP | IMAGO_EP, out=None):
        """Run the selected builds.  `out` maps ol_packed, ol_cv_re, ol_cv_im,
        ke_packed, np_packed, ep_packed (and mv_packed with IMAGO_MV) to
        numpy arrays (host outputs) or integer device pointers
        (outputs_on_device).  Returns `out`."""
        if out is None:
            out = {}
            if which & IMAGO_OL:
                out["ol_packed"] = self._packed()
                c = max(self.core_dim, 1)
                out["ol_cv_re"] = np.zeros((self.nk, self.vale_dim, c))
                out["ol_cv_im"] = np.zeros((self.nk, self.vale_dim, c))
            if which & IMAGO_KE:
                out["ke_packed"] = self._packed()
            if which & IMAGO_NP:
                out["np_packed"] = self._packed()
            if which & IMAGO_EP:
                out["ep_packed"] = self._packed(self.pot_dim)
            if which & IMAGO_MV:
                out["mv_packed"] = self._packed()
        for k, v in out.items():
            self._device_only(v, k)
        s = _out_struct(out)
        _check(lib().imago_intg_build(self._ctx, which, ctypes.byref(s)),
               "imago_intg_build")
        return out

    def build_graph(self, out, which=IMAGO_OL | IMAGO_KE | IMAGO_NP | IMAGO_EP):
        """imago_intg_build_graph: the same builds replayed from a CUDA
        graph (outputs_on_device contexts; `out` maps names to device
        pointers or CUDA tensors).  The first call for an output set builds
        eagerly and captures, later calls replay."""
        for k, v in out.items():
            self._device_only(v, k)
        s = _out_struct(out)
        _check(lib().imago_intg_build_graph(self._ctx, which, ctypes.byref(s)),
               "imago_intg_build_graph")
        return out

    def set_serial(self, serial=True):
        """Run the build kinds one after another on the context's stream
        (per-kernel timing) instead of concurrently (imago_intg_set_serial)."""
        _check(lib().imago_intg_set_serial(self._ctx, 1 if serial else 0),
               "imago_intg_set_serial")

    def tuning(self):
        """The phase-sum column width the context measured fastest and the
        trial milliseconds of widths 32, 48, 64 (imago_intg_tuning)."""
        w = ctypes.c_int()
        ms = np.zeros(3)
        _check(lib().imago_intg_tuning(self._ctx, ctypes.byref(w), _p(ms)),
               "imago_intg_tuning")
        return {"bloch_width": w.value, "trial_ms": [float(x) for x in ms]}

    def stage_ms(self):
        ms = np.zeros(4)
        lib().imago_intg_stage_ms(self._ctx, _p(ms))
        return ms

    def kernel_stats(self):
        """(ms by stage [prim, contract, bloch, ortho], kernel launches) of
        the last build call."""
        ms = np.zeros(4)
        n = ctypes.c_longlong()
        lib().imago_intg_kernel_stats(self._ctx, _p(ms), ctypes.byref(n))
        return ms, n.value

    def output_bytes(self, which=IMAGO_OL | IMAGO_KE | IMAGO_NP | IMAGO_EP):
        per = 16 * self.nk * self.npacked
        n = 0
        if which & IMAGO_OL:
            n += per + 16 * self.nk * self.vale_dim * self.core_dim
        if which & IMAGO_KE:
            n += per
        if which & IMAGO_NP:
            n += per
        if which & IMAGO_EP:
            n += per * self.pot_dim
        if which & IMAGO_MV:
            n += per
        return n


class IntegralBatch:
    """Independent cells built together (imago_batch_*): one context per
    cell, outputs on the device, the builds of all cells captured as one
    CUDA graph on their first call and replayed afterwards."""

    def __init__(self, systems, device=0, scratch_bytes=0, stream=None):
        from .system import ImagoSystemC
        self.systems = list(systems)
        conv = [s.to_c() for s in self.systems]
        self._keep = conv
        arr = (ImagoSystemC * len(conv))(*[c for c, _ in conv])
        self._arr = arr
        opts = ImagoOptsC(device, stream, 1, scratch_bytes)
        self._b = ctypes.c_void_p()
        _check(lib().imago_batch_create(len(conv), ctypes.cast(arr, ctypes.c_void_p),
                                        ctypes.byref(opts), ctypes.byref(self._b)),
               "imago_batch_create")
        self.dims = []
        for i in range(len(conv)):
            d = ImagoDimsC()
            _check(lib().imago_batch_dims(self._b, i, ctypes.byref(d)), "imago_batch_dims")
            self.dims.append(d)

    def __len__(self):
        return len(self.dims)

    def output_shapes(self, i):
        d = self.dims[i]
        nk, npk, V, C, P = (d.num_kpoints, int(d.packed), d.vale_dim,
                            max(d.core_dim, 1), d.pot_dim)
        return {"ol_packed": (nk, npk, 2), "ol_cv_re": (nk, V, C),
                "ol_cv_im": (nk, V, C), "ke_packed": (nk, npk, 2),
                "np_packed": (nk, npk, 2), "ep_packed": (P, nk, npk, 2),
                "mv_packed": (nk, npk, 2)}

    def build(self, outs, which=IMAGO_OL | IMAGO_KE | IMAGO_NP | IMAGO_EP):
        """`outs[i]` maps output names of cell i to device pointers or CUDA
        tensors."""
        if len(outs) != len(self.dims):
            raise ValueError("one output set per cell")
        arr = (ImagoOutC * len(outs))(*[_out_struct(o) for o in outs])
        _check(lib().imago_batch_build(self._b, which, ctypes.cast(arr, ctypes.c_void_p)),
               "imago_batch_build")
        return outs

    def graph_launches(self):
        n = ctypes.c_longlong()
        _check(lib().imago_batch_launches(self._b, ctypes.byref(n)), "imago_batch_launches")
        return n.value

    def close(self):
        if self._b:
            lib().imago_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
