"""Checkpointed integral builds on disk, in the group layout of the
reference's SCF integral file.

The reference writes its integrals to HDF5 (hdf5SCFIntg.F90:188-460): a
group atomIntgGroup holding atomOverlap, atomOverlapCV (when coreDim > 0),
atomKEOverlap, atomMVOverlap (scalar-relativistic runs), atomNPOverlap,
atomPotOverlap/<term>, and atomDMOverlap/<axis> and atomMMOverlap/<axis>
(dipole and momentum matrices, axes x, y, z as 1..3, one status for the
three; hdf5SCFIntg.F90:227-267, 383-396), atomKOverlap/<axis> and
atomKOverlapPlusG/<axis> (the plane-wave overlaps, full valence matrices
as "real%07d" and "imag%07d"; hdf5SCFIntg.F90:235-275, 398-423), one
dataset per
k-point named by its 1-based index ("%07d"; coreValeOL as "real%07d" and
"imag%07d"), and an integer attribute "status" on each group that is set
to 1 once the group's datasets are written.  setupSCF skips every matrix
whose status is already 1 (imago.F90:262-293), which is how an interrupted
run resumes.

No HDF5 library is available here, so this container keeps the same tree
as directories: one .npy file per dataset (packed matrices as
[V(V+1)/2, 2] per k, the memory layout of the reference's (2, ...) Fortran
datasets; coreValeOL as [V, C]) and a file "status" per group, written
atomically after the group's datasets.  build_checkpointed() runs the
builds the store is missing and nothing else.
"""

import json
import os

import numpy as np

GROUP = "atomIntgGroup"
OL, CV, KE, MV, NP, EP = ("atomOverlap", "atomOverlapCV", "atomKEOverlap",
                          "atomMVOverlap", "atomNPOverlap", "atomPotOverlap")
DM, MM = "atomDMOverlap", "atomMMOverlap"
KOV, KOVG = "atomKOverlap", "atomKOverlapPlusG"


def _name(i):
    return f"{i + 1:07d}"


class IntegralStore:
    """A directory tree of packed integral datasets with per-group status."""

    def __init__(self, root, nk, npacked, pot_dim, vale_dim, core_dim):
        self.root = os.path.join(root, GROUP)
        self.nk, self.npacked, self.pot_dim = nk, npacked, pot_dim
        self.vale_dim, self.core_dim = vale_dim, core_dim
        os.makedirs(self.root, exist_ok=True)
        meta = {"nk": nk, "npacked": npacked, "pot_dim": pot_dim,
                "vale_dim": vale_dim, "core_dim": core_dim}
        path = os.path.join(self.root, "dims.json")
        if os.path.exists(path):
            with open(path) as f:
                old = json.load(f)
            if old != meta:
                raise ValueError(f"store holds another system: {old} != {meta}")
        else:
            self._atomic(path, json.dumps(meta))

    @classmethod
    def for_setup(cls, root, setup):
        """The store for an IntegralSetup's system."""
        return cls(root, setup.nk, setup.npacked, setup.pot_dim,
                   setup.vale_dim, setup.core_dim)

    @staticmethod
    def ep_group(term):
        return f"{EP}/{_name(term)}"

    def _dir(self, group):
        d = os.path.join(self.root, *group.split("/"))
        os.makedirs(d, exist_ok=True)
        return d

    @staticmethod
    def _atomic(path, text):
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            f.write(text)
            f.flush()
            os.fsync(f.fileno())
        os.replace(tmp, path)

    def status(self, group):
        path = os.path.join(self.root, *group.split("/"), "status")
        if not os.path.exists(path):
            return 0
        with open(path) as f:
            return int(f.read().strip() or 0)

    def set_status(self, group, value=1):
        self._atomic(os.path.join(self._dir(group), "status"), str(int(value)))

    def write_packed(self, group, packed):
        """packed [nk, V(V+1)/2, 2]: one dataset per k-point."""
        packed = np.asarray(packed)
        assert packed.shape == (self.nk, self.npacked, 2), packed.shape
        d = self._dir(group)
        for k in range(self.nk):
            np.save(os.path.join(d, _name(k) + ".npy"), packed[k])

    def read_packed(self, group):
        d = os.path.join(self.root, *group.split("/"))
        return np.stack([np.load(os.path.join(d, _name(k) + ".npy"))
                         for k in range(self.nk)])

    def write_xyz(self, group, packed3):
        """packed3 [3, nk, V(V+1)/2, 2]: the x, y, z matrices in subgroups
        1..3 of `group`."""
        packed3 = np.asarray(packed3)
        assert packed3.shape == (3, self.nk, self.npacked, 2), packed3.shape
        for c in range(3):
            self.write_packed(f"{group}/{_name(c)}", packed3[c])

    def read_xyz(self, group):
        return np.stack([self.read_packed(f"{group}/{_name(c)}") for c in range(3)])

    def write_planes(self, group, re, im):
        """re, im [3, nk, V, V] indexed (axis, k, col, row), the memory
        order of the reference's (valeDim, valeDim) Fortran datasets: the
        full matrices of each axis in subgroups 1..3 of `group`."""
        shape = (3, self.nk, self.vale_dim, self.vale_dim)
        assert np.shape(re) == shape and np.shape(im) == shape, np.shape(re)
        for c in range(3):
            d = self._dir(f"{group}/{_name(c)}")
            for k in range(self.nk):
                np.save(os.path.join(d, "real" + _name(k) + ".npy"), np.asarray(re[c][k]))
                np.save(os.path.join(d, "imag" + _name(k) + ".npy"), np.asarray(im[c][k]))

    def read_planes(self, group):
        def part(name):
            return np.stack([np.stack([
                np.load(os.path.join(self.root, group, _name(c), name + _name(k) + ".npy"))
                for k in range(self.nk)]) for c in range(3)])
        return part("real"), part("imag")

    def write_cv(self, re, im):
        d = self._dir(CV)
        for k in range(self.nk):
            np.save(os.path.join(d, "real" + _name(k) + ".npy"), np.asarray(re[k]))
            np.save(os.path.join(d, "imag" + _name(k) + ".npy"), np.asarray(im[k]))

    def read_cv(self):
        d = os.path.join(self.root, CV)
        re = np.stack([np.load(os.path.join(d, "real" + _name(k) + ".npy"))
                       for k in range(self.nk)])
        im = np.stack([np.load(os.path.join(d, "imag" + _name(k) + ".npy"))
                       for k in range(self.nk)])
        return re, im


def build_checkpointed(setup, store, ep_batch=8, on_group=None, rel=False,
                       dipole_center=None, momentum=False, plane_wave=False):
    """Run, in the reference's order (imago.F90:260-323: OL, KE, MV when
    rel, NP, EP, then the dipole matrices about `dipole_center`, the
    momentum matrices and the plane-wave overlaps when asked for), the
    builds whose status in `store` is not yet 1, writing each group's
    datasets and then its status.  The plane-wave overlaps fill
    atomKOverlap and atomKOverlapPlusG with the same matrices, as the
    reference does (its plusG argument does not enter the integrals,
    integrals3Terms.F90:1287-1298).

    `setup` is an IntegralSetup with host outputs (or anything with its
    gauss_overlap_ol / _ke / _mv / _np and elec_pot_gauss_overlap_range
    methods).
    The overlap is rebuilt on the device whenever a later matrix still has
    to be built and coreDim > 0 (their orthogonalisation needs its
    coreValeOL), but written only if its own status is 0.  EP terms missing
    from the store are built in runs of at most `ep_batch` terms, so an
    interruption loses at most one run.  `on_group(group)` is called after
    each status is set.  Returns the groups written."""
    written = []

    def done(group):
        store.set_status(group)
        written.append(group)
        if on_group:
            on_group(group)

    ep_todo = [t for t in range(store.pot_dim) if store.status(store.ep_group(t)) == 0]
    singles = [(KE, setup.gauss_overlap_ke)]
    if rel:
        singles.append((MV, setup.gauss_overlap_mv))
    singles.append((NP, setup.gauss_overlap_np))
    triples = []
    if dipole_center is not None:
        triples.append((DM, lambda: setup.gauss_overlap_dm(dipole_center)))
    if momentum:
        triples.append((MM, setup.gauss_overlap_mm))
    planes = [g for g in ((KOV, KOVG) if plane_wave else ()) if store.status(g) == 0]
    later = (any(store.status(g) == 0 for g, _ in singles + triples)
             or bool(ep_todo) or bool(planes))
    if store.status(OL) == 0 or (later and store.core_dim > 0):
        ol, re, im = setup.gauss_overlap_ol()
        if store.status(OL) == 0:
            store.write_packed(OL, ol)
            if store.core_dim > 0:
                store.write_cv(re, im)
            done(OL)
    for group, call in singles:
        if store.status(group) == 0:
            store.write_packed(group, call())
            done(group)
    i = 0
    while i < len(ep_todo):
        first = ep_todo[i]
        count = 1
        while (i + count < len(ep_todo) and count < ep_batch
               and ep_todo[i + count] == first + count):
            count += 1
        mats = setup.elec_pot_gauss_overlap_range(first, count)
        for j in range(count):
            store.write_packed(store.ep_group(first + j), mats[j])
            done(store.ep_group(first + j))
        i += count
    for group, call in triples:
        if store.status(group) == 0:
            store.write_xyz(group, call())
            done(group)
    if planes:
        from imago_b200.intg import koverlap_wave_vectors
        re, im = setup.gauss_koverlap(koverlap_wave_vectors(setup.system))
        for group in planes:
            store.write_planes(group, re, im)
            done(group)
    return written


def read_all(store, rel=False, dipole=False, momentum=False, plane_wave=False):
    """Every matrix of a complete store: {"ol_packed", "ol_cv_re",
    "ol_cv_im", "ke_packed", "np_packed", "ep_packed"}, and "mv_packed"
    when rel, "dm_packed" / "mm_packed" ([3, ...]) and "kov_re" /
    "kov_im" ([3, nk, V, V], from atomKOverlap) when asked for, as numpy
    arrays."""
    out = {"ol_packed": store.read_packed(OL), "ke_packed": store.read_packed(KE),
           "np_packed": store.read_packed(NP),
           "ep_packed": np.stack([store.read_packed(store.ep_group(t))
                                  for t in range(store.pot_dim)])}
    if store.core_dim > 0:
        out["ol_cv_re"], out["ol_cv_im"] = store.read_cv()
    if rel:
        out["mv_packed"] = store.read_packed(MV)
    if dipole:
        out["dm_packed"] = store.read_xyz(DM)
    if momentum:
        out["mm_packed"] = store.read_xyz(MM)
    if plane_wave:
        out["kov_re"], out["kov_im"] = store.read_planes(KOV)
    return out
