import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA device of compute capability 10.0")


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "primitives.json")) as fh:
        return json.load(fh)


@pytest.fixture(scope="session")
def imago_lib():
    """The product library, built in-tree when missing."""
    from imago_b200 import build, intg
    if not os.path.exists(intg.LIB_PATH):
        build.build()
    return intg.lib()


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


# Matrix elements must agree within 1e-10 absolute.  The reference zeroes
# packed elements with |x| < 1e-10 when coreDim > 0 (intgOrtho.F90:185-190),
# so a value that sits on that threshold may be zeroed on one side only; such
# a pair differs by at most the threshold plus the tolerance.
ATOL = 1e-10
ZERO_THRESH = 1e-10


def packed_mismatch(got, ref, atol=ATOL):
    """Largest |got - ref| that is not explained by the 1e-10 zeroing, and
    the count of elements beyond atol."""
    got = np.asarray(got)
    ref = np.asarray(ref)
    d = np.abs(got - ref)
    flip = ((got == 0.0) & (np.abs(ref) < ZERO_THRESH + atol)) | \
           ((ref == 0.0) & (np.abs(got) < ZERO_THRESH + atol))
    d = np.where(flip, 0.0, d)
    return float(d.max()) if d.size else 0.0, int((d > atol).sum())


FINE_STRUCTURE = 7.2973525693e-3  # constants.f90:47 (stored there x 1000)


def massvel_scale(r):
    """The size the reference's own massvel2CIntg rounds at.  It seeds its
    recursion with 16 a2^4 <r_B^4> - 80 a2^3 <r_B^2> + 60 a2^2
    (gaussIntegrals.f90:39118-39120), terms of order alpha^2/8 a^2 S that
    cancel to a value of order a1 a2 when a1 << a2, so its rounding is
    relative to alpha^2/8 max(a1, a2)^2 |S|, not to the result."""
    import oracle
    S = oracle.primitive("overlap", r["la"], r["lb"], r["a1"], r["a2"], 0.0,
                         r["A"], r["B"], r["B"])
    return FINE_STRUCTURE ** 2 / 8 * max(r["a1"], r["a2"]) ** 2 * np.abs(S).max()


def momentum_scale(r):
    """The size the reference's momentum2CIntg rounds at: it seeds with
    2 a1 PA S (gaussIntegrals.f90:23080-23082), PA = P - A formed from
    coordinates of size |A|, |B|, which cancels when a2 << a1."""
    import oracle
    S = oracle.primitive("overlap", r["la"], r["lb"], r["a1"], r["a2"], 0.0,
                         r["A"], r["B"], r["B"])
    coord = max(np.abs(r["A"]).max(), np.abs(r["B"]).max(), 1.0)
    return 2 * max(r["a1"], r["a2"]) * coord * np.abs(S).max()
