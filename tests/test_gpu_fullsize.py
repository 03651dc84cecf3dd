"""The benched configurations, compared element by element with the oracle
at their full sizes (1e-10 absolute, the 1e-10 zeroing allowance of
`packed_mismatch`):

* the jittered Si8 conventional cell at 8x8x8 k (512 k-points): every one of
  its 23 matrices (OL with coreValeOL, KE, NP and the 20 EP terms), the
  only case that runs the tensor-core phase sum over 16 k tiles;
* the 162-atom alpha-quartz 3x3x2 supercell at Gamma: OL, KE, NP and all 40
  EP terms;
* the same cell at 2x2x2 k: OL, KE, NP and the first and last EP term of
  each element.

The oracle runs the reference's loop nest on all host cores (OpenMP over
atom pairs); these are the slowest tests of the suite (the quartz Gamma
oracle takes about a minute and a half on 16 cores).
"""
import numpy as np
import pytest

import oracle
from conftest import packed_mismatch
from imago_b200 import configs, intg

pytestmark = pytest.mark.gpu


def _bad(res):
    return {k: v for k, v in res.items() if v[1] != 0}


def test_silicon8_8x8x8_all_matrices(imago_lib):
    s = configs.silicon_cubic8()
    assert s.num_kpoints == 512
    ob = oracle.OracleBuild(s)
    ref_ol, ref_cre, ref_cim = ob.overlap()
    ref = {"ol_packed": ref_ol, "ol_cv_re": ref_cre, "ol_cv_im": ref_cim,
           "ke_packed": ob.kinetic(), "np_packed": ob.nuclear(),
           "ep_packed": ob.elec_pot()}
    ob.close()
    with intg.IntegralSetup(s) as g:
        got = g.build()
    assert got["ep_packed"].shape[0] == 20
    res = {k: packed_mismatch(got[k], ref[k]) for k in ref}
    for t in range(20):
        res[f"EP{t}"] = packed_mismatch(got["ep_packed"][t], ref["ep_packed"][t])
    assert not _bad(res), res


def test_quartz_gamma_all_forty_potential_terms(imago_lib):
    s = configs.quartz_supercell(gamma=True)
    ob = oracle.OracleBuild(s)
    ref_ol = ob.overlap()[0]
    ref = {"OL": ref_ol, "KE": ob.kinetic(), "NP": ob.nuclear()}
    ref_ep = ob.elec_pot()
    ob.close()
    with intg.IntegralSetup(s) as g:
        out = g.build()
    assert out["ep_packed"].shape[0] == 40 == ref_ep.shape[0]
    res = {"OL": packed_mismatch(out["ol_packed"], ref["OL"]),
           "KE": packed_mismatch(out["ke_packed"], ref["KE"]),
           "NP": packed_mismatch(out["np_packed"], ref["NP"])}
    for t in range(40):
        res[f"EP{t}"] = packed_mismatch(out["ep_packed"][t], ref_ep[t])
    assert not _bad(res), res


def test_quartz_2x2x2(imago_lib):
    s = configs.quartz_supercell(kmesh=(2, 2, 2))
    assert s.num_kpoints == 8
    ob = oracle.OracleBuild(s)
    ref = {"OL": ob.overlap()[0], "KE": ob.kinetic(), "NP": ob.nuclear()}
    terms = (0, 19, 20, 39)  # first and last term of Si, then of O
    for t in terms:
        ref[f"EP{t}"] = ob.elec_pot(t, t + 1)[0]
    ob.close()
    with intg.IntegralSetup(s) as g:
        got = {"OL": g.gauss_overlap_ol()[0], "KE": g.gauss_overlap_ke(),
               "NP": g.gauss_overlap_np()}
        for t in terms:
            got[f"EP{t}"] = g.elec_pot_gauss_overlap_range(t, 1)[0]
    res = {k: packed_mismatch(got[k], ref[k]) for k in ref}
    assert not _bad(res), res
