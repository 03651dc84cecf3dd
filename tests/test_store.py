"""The checkpointed on-disk store (imago_b200.store): the reference's
group/dataset/status layout, skipping of finished groups, and resumption
after an interruption.  A fake builder stands in for the GPU here; the
real builds go through it in test_gpu_parity.py."""

import os

import numpy as np
import pytest

from imago_b200 import store as st


class FakeSetup:
    """Deterministic packed matrices; counts the builds it runs."""

    def __init__(self, nk=3, V=4, C=2, P=5):
        from imago_b200 import configs
        self.nk, self.V, self.C, self.P = nk, V, C, P
        self.system = configs.silicon_cubic8(kmesh=(2, 2, 3))
        self.np = V * (V + 1) // 2
        self.calls = []

    def _mat(self, tag):
        x = np.arange(self.nk * self.np * 2, dtype=float).reshape(self.nk, self.np, 2)
        return x + 1000.0 * tag

    def gauss_overlap_ol(self):
        self.calls.append("OL")
        re = np.full((self.nk, self.V, self.C), 1.5)
        return self._mat(0), re, -re

    def gauss_overlap_ke(self):
        self.calls.append("KE")
        return self._mat(1)

    def gauss_overlap_mv(self):
        self.calls.append("MV")
        return self._mat(3)

    def gauss_overlap_dm(self, center):
        self.calls.append(("DM", tuple(center)))
        return np.stack([self._mat(20 + c) for c in range(3)])

    def gauss_overlap_mm(self):
        self.calls.append("MM")
        return np.stack([self._mat(30 + c) for c in range(3)])

    def gauss_overlap_np(self):
        self.calls.append("NP")
        return self._mat(2)

    def gauss_koverlap(self, dk):
        self.calls.append(("KOV", np.asarray(dk).round(12).tobytes()))
        x = np.arange(3 * self.nk * self.V * self.V, dtype=float)
        x = x.reshape(3, self.nk, self.V, self.V)
        return x + 40000.0, -x

    def elec_pot_gauss_overlap_range(self, first, count):
        self.calls.append(("EP", first, count))
        return np.stack([self._mat(10 + t) for t in range(first, first + count)])


def _store(tmp_path, f):
    return st.IntegralStore(str(tmp_path), f.nk, f.np, f.P, f.V, f.C)


def test_layout_and_complete_build(tmp_path):
    f = FakeSetup()
    s = _store(tmp_path, f)
    written = st.build_checkpointed(f, s)
    assert written == [st.OL, st.KE, st.NP] + [s.ep_group(t) for t in range(f.P)]
    root = os.path.join(str(tmp_path), st.GROUP)
    assert os.path.exists(os.path.join(root, "atomOverlap", "0000001.npy"))
    assert os.path.exists(os.path.join(root, "atomOverlapCV", "imag0000003.npy"))
    assert os.path.exists(os.path.join(root, "atomPotOverlap", "0000005", "0000002.npy"))
    out = st.read_all(s)
    assert np.array_equal(out["ke_packed"], f._mat(1))
    assert np.array_equal(out["ep_packed"][4], f._mat(14))
    assert np.array_equal(out["ol_cv_im"], -out["ol_cv_re"])
    # a second run finds everything done and builds nothing
    f2 = FakeSetup()
    assert st.build_checkpointed(f2, _store(tmp_path, f2)) == []
    assert f2.calls == []


def test_resume_after_interruption(tmp_path):
    f = FakeSetup(P=7)
    s = _store(tmp_path, f)

    def stop(group):
        if group == s.ep_group(2):
            raise KeyboardInterrupt

    with pytest.raises(KeyboardInterrupt):
        st.build_checkpointed(f, s, ep_batch=2, on_group=stop)
    # terms 0..2 are recorded; term 3 was built in the same run but its
    # status never set, so it is built again
    f2 = FakeSetup(P=7)
    written = st.build_checkpointed(f2, _store(tmp_path, f2), ep_batch=8)
    assert written == [s.ep_group(t) for t in range(3, 7)]
    # coreDim > 0: the overlap is rebuilt for the orthogonalisation, not
    # written again
    assert f2.calls == ["OL", ("EP", 3, 4)]
    out = st.read_all(s)
    for t in range(7):
        assert np.array_equal(out["ep_packed"][t], f._mat(10 + t))


def test_store_refuses_another_system(tmp_path):
    f = FakeSetup()
    _store(tmp_path, f)
    with pytest.raises(ValueError):
        st.IntegralStore(str(tmp_path), f.nk, f.np, f.P + 1, f.V, f.C)


def test_relativistic_run_adds_mass_velocity_in_order(tmp_path):
    f = FakeSetup()
    s = _store(tmp_path, f)
    written = st.build_checkpointed(f, s, rel=True)
    assert written[:4] == [st.OL, st.KE, st.MV, st.NP]
    assert f.calls[:4] == ["OL", "KE", "MV", "NP"]
    assert np.array_equal(st.read_all(s, rel=True)["mv_packed"], f._mat(3))
    # a later non-relativistic store of the same system skips MV entirely
    f2 = FakeSetup()
    assert st.build_checkpointed(f2, _store(tmp_path, f2)) == []


def test_dipole_and_momentum_groups(tmp_path):
    # atomDMOverlap/<axis>/<k> and atomMMOverlap/<axis>/<k>, one status
    # each, built after the potential terms
    f = FakeSetup(P=2)
    s = _store(tmp_path, f)
    written = st.build_checkpointed(f, s, dipole_center=(0.5, 0.0, 0.0), momentum=True)
    assert written[-2:] == [st.DM, st.MM]
    assert f.calls[-2:] == [("DM", (0.5, 0.0, 0.0)), "MM"]
    root = os.path.join(str(tmp_path), st.GROUP)
    assert os.path.exists(os.path.join(root, "atomDMOverlap", "0000003", "0000002.npy"))
    out = st.read_all(s, dipole=True, momentum=True)
    assert np.array_equal(out["dm_packed"][1], f._mat(21))
    assert np.array_equal(out["mm_packed"][2], f._mat(32))
    # a rerun with everything recorded builds nothing, the overlap included
    f2 = FakeSetup(P=2)
    assert st.build_checkpointed(f2, _store(tmp_path, f2), dipole_center=(0.5, 0.0, 0.0),
                                 momentum=True) == []
    assert f2.calls == []


def test_plane_wave_groups(tmp_path):
    # atomKOverlap/<axis>/real<k>, imag<k> and the same matrices in
    # atomKOverlapPlusG, from one build with dK_c = b_c / n_c, after the
    # momentum matrices; a rerun builds nothing
    from imago_b200 import intg
    f = FakeSetup(P=1)
    s = _store(tmp_path, f)
    written = st.build_checkpointed(f, s, momentum=True, plane_wave=True)
    assert written[-3:] == [st.MM, st.KOV, st.KOVG]
    kov = [c for c in f.calls if isinstance(c, tuple) and c[0] == "KOV"]
    assert len(kov) == 1
    dk = intg.koverlap_wave_vectors(f.system)
    assert kov[0][1] == dk.round(12).tobytes()
    # b_c . a_c = 2 pi, so dK_c . a_c = 2 pi / n_c
    a = np.asarray(f.system.real_vectors)
    assert np.allclose(np.einsum("cx,cx->c", dk, a), 2 * np.pi / np.array([2, 2, 3]))
    root = os.path.join(str(tmp_path), st.GROUP)
    for g in ("atomKOverlap", "atomKOverlapPlusG"):
        assert os.path.exists(os.path.join(root, g, "0000003", "imag0000003.npy"))
    out = st.read_all(s, momentum=True, plane_wave=True)
    re, im = f.gauss_koverlap(dk)
    assert np.array_equal(out["kov_re"], re) and np.array_equal(out["kov_im"], im)
    assert np.array_equal(s.read_planes(st.KOVG)[1], im)
    f2 = FakeSetup(P=1)
    assert st.build_checkpointed(f2, _store(tmp_path, f2), momentum=True,
                                 plane_wave=True) == []
    assert f2.calls == []


def test_wave_vectors_follow_the_reference_reciprocal_lattice():
    # recipVectors(:, i) = 2 pi (a_{i+1} x a_{i+2}) / (a_i . a_{i+1} x a_{i+2})
    # with cyclic indices (lattice.f90:200-214), on a skewed cell, divided
    # by numAxialKPoints(i)
    from imago_b200 import configs, intg
    s = configs.silicon_cubic8(kmesh=(2, 3, 4))
    a = np.array([[10.2, 0.3, -0.4], [1.1, 9.7, 0.2], [-0.6, 0.8, 11.3]])
    s.real_vectors = a
    ref = np.zeros((3, 3))
    for i in range(3):
        b = np.cross(a[(i + 1) % 3], a[(i + 2) % 3])
        ref[i] = 2.0 * np.pi * b / np.dot(a[i], b) / (2, 3, 4)[i]
    got = intg.koverlap_wave_vectors(s)
    assert np.allclose(got, ref, rtol=1e-14, atol=0)
    # the reciprocal vectors themselves with one point per axis
    assert np.allclose(intg.koverlap_wave_vectors(s, num_axial=(1, 1, 1)),
                       ref * [[2], [3], [4]], rtol=1e-14, atol=0)
