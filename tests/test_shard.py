"""Term sharding of one system's build (imago_b200.shard) on two gloo ranks
on the CPU: every matrix is built by exactly one rank and the gather puts
each at its place on the destination rank.  Fake builders stand in for the
GPU builds; the GPU path itself runs in test_gpu_parity.py."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from imago_b200 import shard


def test_partition_covers_every_matrix_once():
    for pot_dim in (0, 1, 5, 20, 40):
        for world in (1, 2, 3, 8):
            parts = shard.partition(pot_dim, world)
            assert parts[0][0] == 0 and parts[-1][1] == 2 + pot_dim
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            sizes = [hi - lo for lo, hi in parts]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, pot_dim, dst, results):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    shape = (3, 5, 2)
    built = []

    def builder(ids, shp):
        built.extend(ids)
        t = torch.empty((len(ids),) + tuple(shp), dtype=torch.float64)
        for i, m in enumerate(ids):
            t[i] = 100.0 * m + torch.arange(t[i].numel(), dtype=torch.float64).reshape(shp)
        return t

    def overlap():
        return {"ol_packed": torch.full(shape, float(rank), dtype=torch.float64)}

    sb = shard.ShardedBuild(pot_dim, shape, builder, overlap, dst=dst)
    out = sb.build()
    ok = True
    if rank == dst:
        full = torch.stack([out["ke"], out["np"]] + list(out["ep"]))
        for m in range(2 + pot_dim):
            ref = 100.0 * m + torch.arange(full[m].numel(), dtype=torch.float64).reshape(shape)
            ok &= bool(torch.equal(full[m], ref))
    else:
        ok &= out is None
    lo, hi = shard.partition(pot_dim, world)[rank]
    ok &= built == list(range(lo, hi))
    results[rank] = ok
    dist.destroy_process_group()


@pytest.mark.parametrize("pot_dim,dst", [(5, 0), (20, 1), (0, 0)])
def test_two_ranks_gather_every_matrix(pot_dim, dst):
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    results = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, pot_dim, dst, results))
             for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert results[0] and results[1]


def test_cost_partition_balances_the_three_centre_builds():
    from imago_b200 import configs
    s = configs.quartz_supercell(gamma=True)
    costs = shard.matrix_costs(s)
    assert len(costs) == 2 + s.pot_dim
    for world in (1, 2, 3, 4, 8):
        parts = shard.partition(s.pot_dim, world, costs)
        assert parts[0][0] == 0 and parts[-1][1] == 2 + s.pot_dim
        assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
        assert all(hi > lo for lo, hi in parts)
        loads = [sum(costs[lo:hi]) for lo, hi in parts]
        # no rank above its share by more than its largest single matrix
        assert max(loads) <= sum(costs) / world + max(costs)


def _oracle_rank_main(rank, world, port, results):
    # real builders on the CPU: the oracle's restatement of the driver
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import numpy as np
    import oracle
    from imago_b200 import configs
    s = configs.small_test_system()
    ob = oracle.OracleBuild(s, nthreads=1)

    def overlap():
        return {"ol_packed": torch.as_tensor(ob.overlap()[0])}

    def builder(ids, shp):
        out = torch.empty((len(ids),) + tuple(shp), dtype=torch.float64)
        for i, m in enumerate(ids):
            if m == shard.KE:
                out[i] = torch.as_tensor(ob.kinetic())
            elif m == shard.NP:
                out[i] = torch.as_tensor(ob.nuclear())
            else:
                out[i] = torch.as_tensor(ob.elec_pot(m - 2, m - 1)[0])
        return out

    shape = ob.overlap()[0].shape
    sb = shard.ShardedBuild(s.pot_dim, shape, builder, overlap, dst=0,
                            costs=shard.matrix_costs(s))
    got = sb.build()
    if rank == 0:
        ok = bool(np.array_equal(got["ke"].numpy(), ob.kinetic()))
        ok &= bool(np.array_equal(got["np"].numpy(), ob.nuclear()))
        ok &= bool(np.array_equal(got["ep"].numpy(), ob.elec_pot()))
        results[rank] = ok
    else:
        results[rank] = got is None
    ob.close()
    dist.destroy_process_group()


def test_two_ranks_with_oracle_builders_reproduce_the_single_build():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    results = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_oracle_rank_main, args=(r, 2, port, results))
             for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    assert results[0] and results[1]
