"""One system's integral build spread over the ranks of a process group.

The matrices after the overlap are independent: KE, NP and the potDim EP
terms (integrals.F90:656-2486).  Every rank builds the overlap, whose
coreValeOL orthogonalises the others (integrals.F90:3686), then its own
contiguous block of the remaining 2 + potDim matrices; one gather brings
every packed matrix to the destination rank (point-to-point sends over
NVLink with NCCL, or gloo on the host), in the reference's order.  No
other exchange is needed: each matrix is complete on the rank that built
it.
"""

import torch
import torch.distributed as dist

# matrix ids after the overlap: 0 = KE, 1 = NP, 2 + j = EP term j
KE, NP = 0, 1


def partition(pot_dim, world):
    """Contiguous blocks of the 2 + pot_dim matrices after the overlap,
    one per rank, sizes differing by at most one: [(lo, hi), ...]."""
    n = 2 + pot_dim
    base, extra = divmod(n, world)
    out, lo = [], 0
    for r in range(world):
        hi = lo + base + (1 if r < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


class ShardedBuild:
    """build() runs this rank's share and gathers all matrices on `dst`.

    `builder(ids, shape)` returns one tensor [len(ids), *shape] holding the
    packed matrices of the ids (KE, NP, EP terms); `overlap()` returns the
    rank's overlap output dict.  `from_setup` wires them to an
    IntegralSetup with outputs on the device."""

    def __init__(self, pot_dim, shape, builder, overlap, dst=0, group=None,
                 device=None):
        self.pot_dim = pot_dim
        self.shape = tuple(shape)
        self.builder = builder
        self.overlap = overlap
        self.dst = dst
        self.group = group
        self.device = device
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.parts = partition(pot_dim, self.world)

    @classmethod
    def from_setup(cls, setup, dst=0, group=None):
        from . import intg
        dev = torch.device("cuda", torch.cuda.current_device())
        shape = (setup.nk, setup.npacked, 2)

        def overlap():
            C = max(setup.core_dim, 1)
            out = {"ol_packed": torch.empty(shape, dtype=torch.float64, device=dev),
                   "ol_cv_re": torch.empty((setup.nk, setup.vale_dim, C),
                                           dtype=torch.float64, device=dev),
                   "ol_cv_im": torch.empty((setup.nk, setup.vale_dim, C),
                                           dtype=torch.float64, device=dev)}
            setup.build(which=intg.IMAGO_OL, out=out)
            return out

        def builder(ids, shp):
            t = torch.empty((len(ids),) + tuple(shp), dtype=torch.float64, device=dev)
            for i, m in enumerate(ids):
                if m == KE:
                    setup.build(which=intg.IMAGO_KE, out={"ke_packed": t[i]})
                elif m == NP:
                    setup.build(which=intg.IMAGO_NP, out={"np_packed": t[i]})
            eps = [m - 2 for m in ids if m >= 2]
            if eps:
                j0 = ids.index(eps[0] + 2)
                setup.elec_pot_gauss_overlap_range(eps[0], len(eps), t[j0])
            return t

        return cls(setup.pot_dim, shape, builder, overlap, dst, group, dev)

    def build(self):
        """On `dst`: {"ol": overlap dict, "ke": ..., "np": ..., "ep": [potDim,
        ...]}; on the other ranks None."""
        ol = self.overlap()
        lo, hi = self.parts[self.rank]
        mine = self.builder(list(range(lo, hi)), self.shape)
        if self.rank != self.dst:
            if hi > lo:
                dist.send(mine.contiguous(), self.dst, group=self.group)
            return None
        full = torch.empty((2 + self.pot_dim,) + self.shape, dtype=mine.dtype,
                           device=mine.device)
        full[lo:hi] = mine
        for r, (a, b) in enumerate(self.parts):
            if r != self.dst and b > a:
                dist.recv(full[a:b], r, group=self.group)
        return {"ol": ol, "ke": full[KE], "np": full[NP], "ep": full[2:]}
