"""imago_prim_eval_static: primitive integrals with no device allocation.

It serves callers that cannot call cudaMalloc (a GPU shared under a fixed
memory budget, device memory held by a pool allocator, loops that cannot
take cudaMalloc's synchronisation).  Called through the C ABI, its results
must equal those of imago_prim_eval, which allocates its staging buffers,
on consecutive calls that reuse the same fixed device array.  This file is
collected last so that a run stopping at the first failure has already run
every other test.
"""
import ctypes

import numpy as np
import pytest

from imago_b200 import intg

pytestmark = pytest.mark.gpu


def _records(golden, kind):
    recs = [r for r in golden["records"] if kind in r]
    params = np.array([[r["a1"], r["a2"], r["a3"]] + r["A"] + r["B"] + r["C"]
                       for r in recs])
    cls = np.array([[r["la"], r["lb"]] for r in recs], np.int32)
    return params, cls


def _close(a, b):
    # the tolerance the primitive tests use: 1e-12 of each block's largest
    # element
    for x, y in zip(a, b):
        scale = max(np.abs(y).max(), 1e-300)
        assert np.abs(x - y).max() <= 1e-12 * scale


def test_static_matches_allocating_entry_point_on_consecutive_calls(imago_lib, golden):
    p1, c1 = _records(golden, "nuclear3c")
    p2, c2 = _records(golden, "overlap")
    p2, c2 = p2[:17], c2[:17]  # fewer records than the first call
    first = intg.prim_eval_static("nuclear3c", p1, c1)
    second = intg.prim_eval_static("overlap", p2, c2)
    _close(first, intg.prim_eval("nuclear3c", p1, c1))
    _close(second, intg.prim_eval("overlap", p2, c2))
    boys = np.zeros((5, 12))
    boys[:, 0] = [0.0, 0.05, 0.5, 5.0, 50.0]
    _close(intg.prim_eval_static("boys", boys), intg.prim_eval("boys", boys))


def test_static_rejects_more_records_than_its_array_holds(imago_lib):
    n = intg.PRIM_STATIC_MAX_RECORDS + 1
    params = np.ones((n, 12))
    cls = np.zeros((n, 2), np.int32)
    out = np.zeros((n, 256))
    D = ctypes.POINTER(ctypes.c_double)
    st = imago_lib.imago_prim_eval_static(
        0, n, params.ctypes.data_as(D),
        cls.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), out.ctypes.data_as(D))
    assert st == 8  # IMAGO_ERR_RANGE


def test_static_at_its_record_limit(imago_lib, golden):
    # exactly PRIM_STATIC_MAX_RECORDS records: the only size whose output
    # blocks fill the array to its end
    p, c = _records(golden, "kinetic")
    n = intg.PRIM_STATIC_MAX_RECORDS
    reps = -(-n // len(p))
    p, c = np.tile(p, (reps, 1))[:n], np.tile(c, (reps, 1))[:n]
    for _ in range(2):
        _close(intg.prim_eval_static("kinetic", p, c), intg.prim_eval("kinetic", p, c))
