"""The C ABI library: it loads, exports what include/imago_intg.h
declares, and its host-only entry points behave (no GPU needed)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, has_gpu
from imago_b200 import configs, intg
from imago_b200.system import kpoint_mesh, pot_alphas


def declared_symbols():
    names = []
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            txt = open(os.path.join(inc, f)).read()
            names += re.findall(r"IMAGO_API\s+[\w\s\*]*?\b(imago_\w+)\s*\(", txt)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(imago_lib):
    names = declared_symbols()
    assert len(names) >= 12
    out = subprocess.run(["nm", "-D", "--defined-only", intg.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (imago_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        assert hasattr(imago_lib, n)


def test_strerror_messages(imago_lib):
    assert imago_lib.imago_strerror(0) == b"success"
    assert b"More lattice points" in imago_lib.imago_strerror(2)
    assert imago_lib.imago_strerror(12345) == b"unknown status"


def test_kpoint_mesh_matches_reference_formula(imago_lib):
    for n, sh in [((4, 4, 4), (0.5, 0.5, 0.5)), ((3, 2, 5), (0.0, 0.5, 0.25)),
                  ((1, 1, 1), (0.0, 0.0, 0.0))]:
        got = intg.kpoint_mesh(n, sh)
        assert np.array_equal(got, kpoint_mesh(n, sh))
        # kpoints.f90:896-899 : -1/2 + (i - 1 + shift) / n, a-major
        i = np.arange(n[0])
        assert np.allclose(np.unique(got[:, 0]), -0.5 + (i + sh[0]) / n[0])


def test_kpoint_mesh_rejects_bad_sizes(imago_lib):
    n3 = (ctypes.c_int * 3)(0, 2, 2)
    sh = np.zeros(3)
    out = np.zeros(3)
    st = imago_lib.imago_kpoint_mesh(n3, sh.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                     out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert st == 8


def test_pot_alphas_geometric_series():
    a = pot_alphas(16, 0.12, 1.0e5)
    assert a[0] == 0.12
    assert abs(a[-1] - 1.0e5) < 1e-8 * 1.0e5
    assert np.allclose(a[1:] / a[:-1], (1.0e5 / 0.12) ** (1 / 15), rtol=1e-12)


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_create_without_device_fails_loudly(imago_lib):
    with pytest.raises(intg.ImagoError) as e:
        intg.IntegralSetup(configs.diamond_primitive())
    assert e.value.status == intg.IMAGO_ERR_NO_DEVICE


def test_system_validation():
    s = configs.diamond_primitive()
    s.atom_types[0].num_orb_alphas = [16, 8, 12, 0]
    with pytest.raises(ValueError):
        s.validate()


def test_added_entry_points_reject_bad_arguments(imago_lib):
    # argument checks come before any device work, so they hold without a GPU
    L = imago_lib
    vp = ctypes.c_void_p
    L.imago_intg_set_serial.argtypes = [vp, ctypes.c_int]
    assert L.imago_intg_set_serial(None, 1) == 1
    L.imago_intg_build_graph.argtypes = [vp, ctypes.c_uint, vp]
    assert L.imago_intg_build_graph(None, 15, None) == 1
    L.imago_intg_tuning.argtypes = [vp, vp, vp]
    assert L.imago_intg_tuning(None, None, None) == 1
    L.imago_elec_pot_gauss_overlap_range.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp]
    assert L.imago_elec_pot_gauss_overlap_range(None, 0, 1, None) == 1
    out = vp()
    L.imago_batch_create.argtypes = [ctypes.c_int, vp, vp, ctypes.POINTER(vp)]
    assert L.imago_batch_create(0, None, None, ctypes.byref(out)) == 1
    assert not out.value
    L.imago_batch_build.argtypes = [vp, ctypes.c_uint, vp]
    assert L.imago_batch_build(None, 15, None) == 1
    L.imago_batch_size.argtypes = [vp]
    assert L.imago_batch_size(None) == 0
    L.imago_hermitian_eigvals.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp, vp]
    assert L.imago_hermitian_eigvals(0, 1, None, None, None) == 1
    L.imago_secular_matrices.argtypes = [ctypes.c_int] * 3 + [vp] * 8
    assert L.imago_secular_matrices(0, 1, 0, *([None] * 8)) == 1
    L.imago_gauss_overlap_mv.argtypes = [vp, vp]
    assert L.imago_gauss_overlap_mv(None, None) == 1
    L.imago_ham_pscf.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, vp]
    assert L.imago_ham_pscf(None, 1, None, 0, None) == 1
    L.imago_gauss_overlap_mm.argtypes = [vp, vp]
    assert L.imago_gauss_overlap_mm(None, None) == 1
    L.imago_gauss_overlap_dm.argtypes = [vp, vp, vp]
    assert L.imago_gauss_overlap_dm(None, None, None) == 1
    L.imago_gauss_koverlap.argtypes = [vp] * 4
    assert L.imago_gauss_koverlap(None, None, None, None) == 1
    L.imago_hermitian_eigh.argtypes = [ctypes.c_int, ctypes.c_int] + [vp] * 4
    assert L.imago_hermitian_eigh(0, 1, None, None, None, None) == 1
    L.imago_populate_states.argtypes = [ctypes.c_int] * 3 + [vp] * 2 + \
        [ctypes.c_double] * 4 + [vp] * 2
    assert L.imago_populate_states(0, 1, 1, None, None, 0.0, 0.0, 0.0, 0.0, None, None) == 1
    L.imago_packed_traces.argtypes = [ctypes.c_int] * 3 + [vp, ctypes.c_int] + [vp] * 3
    assert L.imago_packed_traces(0, 1, 1, None, 1, None, None, None) == 1
    L.imago_intg_set_ham_mode.argtypes = [vp, ctypes.c_int]
    assert L.imago_intg_set_ham_mode(None, 0) == 1
    L.imago_secular_matrices_rel.argtypes = [ctypes.c_int] * 3 + [vp] * 9
    assert L.imago_secular_matrices_rel(0, 1, 0, *([None] * 9)) == 1
    L.imago_secular_reduce.argtypes = [ctypes.c_int] * 2 + [vp] * 6
    assert L.imago_secular_reduce(0, 1, *([None] * 6)) == 1
    dummy = [vp(16), vp(32), vp(48)]
    # one CTA per k-point holds the factor: n above 128 is out of range
    assert L.imago_secular_reduce(129, 1, *dummy, None, None, None) == 8
    # the reduced matrix may not overwrite H or S
    assert L.imago_secular_reduce(8, 1, dummy[0], dummy[1], dummy[0], None, None, None) == 1
    L.imago_secular_back.argtypes = [ctypes.c_int] * 3 + [vp] * 4
    assert L.imago_secular_back(0, 1, 1, *([None] * 4)) == 1
    assert L.imago_secular_back(8, 1, 9, *dummy, None) == 1
    assert L.imago_secular_back(129, 1, 4, *dummy, None) == 8
    L.imago_packed_density.argtypes = [ctypes.c_int] * 4 + [vp] * 4
    assert L.imago_packed_density(0, 1, 1, 1, *([None] * 4)) == 1
    assert L.imago_packed_density(8, 1, 2, 3, *dummy, None) == 1


def test_device_output_context_refuses_host_outputs():
    # a context whose kernels write through the output pointers takes no
    # numpy array (the check runs before the library is called, so an
    # instance without a context shows it on the CPU)
    import ctypes
    import numpy as np
    from imago_b200 import intg
    g = object.__new__(intg.IntegralSetup)
    g._ctx = ctypes.c_void_p()
    g.outputs_on_device = True
    g.nk, g.npacked, g.vale_dim, g.core_dim, g.pot_dim = 2, 3, 2, 0, 1
    calls = [lambda: g.gauss_overlap_ke(), lambda: g.gauss_overlap_mm(),
             lambda: g.gauss_overlap_dm([0.0, 0.0, 0.0]),
             lambda: g.gauss_overlap_mm(out=np.zeros((3, 2, 3, 2))),
             lambda: g.gauss_koverlap(np.zeros((3, 3))),
             lambda: g.ham_pscf(np.zeros(1)),
             lambda: g.elec_pot_gauss_overlap_range(0, 1, np.zeros((1, 2, 3, 2))),
             lambda: g.build(intg.IMAGO_KE, {"ke_packed": np.zeros((2, 3, 2))}),
             lambda: g.build(intg.IMAGO_KE)]
    for call in calls:
        with pytest.raises(ValueError):
            call()
