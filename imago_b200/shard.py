"""One system's integral build spread over the ranks of a process group.

The matrices after the overlap are independent: KE, NP and the potDim EP
terms (integrals.F90:656-2486).  Every rank builds the overlap, whose
coreValeOL orthogonalises the others (integrals.F90:3686), then its own
contiguous block of the remaining 2 + potDim matrices, the blocks balanced
by an estimate of each matrix's cost (matrix_costs); one gather brings
every packed matrix to the destination rank (point-to-point sends over
NVLink with NCCL, or gloo on the host), in the reference's order.  No
other exchange is needed: each matrix is complete on the rank that built
it.
"""

import torch
import torch.distributed as dist

# matrix ids after the overlap: 0 = KE, 1 = NP, 2 + j = EP term j
KE, NP = 0, 1


def matrix_costs(system):
    """Relative cost of the matrices after the overlap, in the order KE, NP,
    EP terms: a two-centre build counts 1; a three-centre build counts the
    potential sites it sums over (NP every site, integrals.F90:2533-2698;
    an EP term the sites of its type, integrals.F90:2700-2858), each site
    weighted like a two-centre build because a site's image sum costs about
    as much as the shell pairs' own image sum."""
    import numpy as np
    types = np.asarray(system.pot_site_type)
    costs = [1.0, float(len(types))]
    for t, p in enumerate(system.pot_types):
        costs += [float((types == t + 1).sum())] * len(p.alphas)
    return costs


def partition(pot_dim, world, costs=None):
    """Contiguous blocks of the 2 + pot_dim matrices after the overlap, one
    per rank: [(lo, hi), ...].  Without costs the sizes differ by at most
    one; with costs (one per matrix, matrix_costs) each block ends where its
    cumulative cost is nearest its share of the total, every rank keeping
    at least one matrix while there are matrices left."""
    n = 2 + pot_dim
    if costs is None:
        base, extra = divmod(n, world)
        out, lo = [], 0
        for r in range(world):
            hi = lo + base + (1 if r < extra else 0)
            out.append((lo, hi))
            lo = hi
        return out
    if len(costs) != n:
        raise ValueError(f"{len(costs)} costs for {n} matrices")
    total = float(sum(costs))
    out, lo, acc = [], 0, 0.0
    for r in range(world):
        if r == world - 1:
            hi = n
        else:
            target = total * (r + 1) / world
            hi = lo
            # leave one matrix for each rank after this one, if possible
            limit = max(lo, n - (world - 1 - r))
            while hi < limit and (hi == lo or acc + costs[hi] / 2 <= target):
                acc += costs[hi]
                hi += 1
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
                 device=None, costs=None):
        self.pot_dim = pot_dim
        self.shape = tuple(shape)
        self.builder = builder
        self.overlap = overlap
        self.dst = dst
        self.group = group
        self.device = device
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.parts = partition(pot_dim, self.world, costs)

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

        costs = matrix_costs(setup.system) if getattr(setup, "system", None) else None
        return cls(setup.pot_dim, shape, builder, overlap, dst, group, dev, costs)

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
