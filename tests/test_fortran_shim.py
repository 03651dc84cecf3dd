"""The Fortran shim (fortran/imago_b200_bind.F90) against the C ABI it
binds, and the populate outputs it hands to the reference's module data.

No Fortran compiler exists where these tests run, so the shim's interface
blocks are read as text: every `bind(C, name=...)` function must name a
symbol that include/imago_intg.h declares, with the same number of
arguments, passed by value where the C prototype takes a scalar and by reference
(or as a c_ptr value) where it takes a pointer.
When gfortran is on the PATH the shim's interface module is also compiled
(syntax only)."""
import ctypes
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from imago_b200 import charge, intg

F90 = os.path.join(ROOT, "fortran", "imago_b200_bind.F90")
HDR = os.path.join(ROOT, "include", "imago_intg.h")


def _c_prototypes():
    txt = open(HDR).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    protos = {}
    for m in re.finditer(r"IMAGO_API\s+[\w\s\*]*?\b(imago_\w+)\s*\(([^)]*)\)", txt):
        args = [a.strip() for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        protos[m.group(1)] = args
    return protos


def _fortran_interfaces():
    src = open(F90).read()
    src = re.sub(r"&\s*\n\s*&?", " ", src)  # join continuation lines
    out = {}
    for m in re.finditer(r"(?:function|subroutine)\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)"
                         r"(.*?)end (?:function|subroutine)", src, flags=re.S | re.I):
        dummies = [a.strip().lower() for a in m.group(2).split(",") if a.strip()]
        body = m.group(4)
        value, ptr = set(), set()
        for decl in re.finditer(r"^\s*([^!\n]*?)::\s*([^\n!]*)", body, flags=re.M):
            attrs = decl.group(1).lower()
            names = [re.sub(r"\(.*", "", v).strip().lower()
                     for v in re.sub(r"\([^)]*\)", "", decl.group(2)).split(",")]
            if "value" in attrs:
                value.update(names)
            if "c_ptr" in attrs:
                ptr.update(names)
        out[m.group(3)] = (dummies, value, ptr)
    return out


def test_every_bound_function_matches_its_c_prototype():
    protos = _c_prototypes()
    ifaces = _fortran_interfaces()
    assert len(ifaces) >= 10
    for name, (dummies, value, ptr) in ifaces.items():
        assert name in protos, f"{name} is bound but not declared in imago_intg.h"
        cargs = protos[name]
        assert len(dummies) == len(cargs), (name, dummies, cargs)
        for d, c in zip(dummies, cargs):
            c_scalar = "*" not in c and "[" not in c
            if c_scalar:
                # a C scalar is passed by value, and is not a pointer
                assert d in value and d not in ptr, (name, d, c)
            else:
                # a C pointer is a Fortran reference, or a c_ptr by value
                assert d not in value or d in ptr, (name, d, c)


def test_populate_call_fills_the_sorted_module_arrays():
    src = open(F90).read()
    body = src[src.index("subroutine b200PopulateStates"):
               src.index("end subroutine b200PopulateStates")]
    # cleanUpPopulation deallocates both every SCF iteration
    # (populate.F90:1230-1231), so the shim must allocate them
    assert "allocate (sortedEnergyEigenValues(n))" in body
    assert "allocate (indexEnergyEigenValues(n))" in body
    assert "imago_populate_states_sorted" in body
    assert "indexEnergyEigenValues(:) = idx(:) + 1" in body


def test_sorted_outputs_are_the_stable_sort(imago_lib):
    rng = np.random.default_rng(4)
    nk, spin, ns = 5, 2, 7
    e = np.round(rng.normal(size=(nk, spin, ns)), 2)  # ties on purpose
    L = intg.lib()
    vp = ctypes.c_void_p
    L.imago_populate_states_sorted.argtypes = [ctypes.c_int] * 3 + [vp] * 2 + \
        [ctypes.c_double] * 4 + [vp] * 4
    L.imago_populate_states_sorted.restype = ctypes.c_int
    pop = np.zeros_like(e)
    info = np.zeros(5)
    srt = np.zeros(e.size)
    idx = np.zeros(e.size, np.int32)
    rc = L.imago_populate_states_sorted(nk, spin, ns, e.ctypes.data, None, 10.0, 0.0,
                                        0.0, 0.0, pop.ctypes.data, info.ctypes.data,
                                        srt.ctypes.data, idx.ctypes.data)
    assert rc == 0
    flat = e.ravel()
    order = np.argsort(flat, kind="stable")
    assert np.array_equal(idx, order)
    assert np.array_equal(srt, flat[order])
    ref = charge.populate_states(e, 10.0)
    assert np.array_equal(pop, ref["population"])
    assert int(info[3]) == ref["occupied_index"]
    # both outputs are optional
    assert L.imago_populate_states_sorted(nk, spin, ns, e.ctypes.data, None, 10.0, 0.0,
                                          0.0, 0.0, pop.ctypes.data, info.ctypes.data,
                                          None, None) == 0


@pytest.mark.skipif(shutil.which("gfortran") is None, reason="no Fortran compiler")
def test_shim_interface_block_compiles(tmp_path):
    src = open(F90).read()
    start = src.index("   interface")
    end = src.index("   end interface") + len("   end interface")
    mod = ("module b200_iface_check\n   use, intrinsic :: iso_c_binding\n   implicit none\n"
           + src[start:end] + "\nend module b200_iface_check\n")
    f = tmp_path / "iface.f90"
    f.write_text(mod)
    r = subprocess.run(["gfortran", "-fsyntax-only", str(f)], capture_output=True, text=True,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stderr
