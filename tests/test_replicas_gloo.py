"""Multi-rank host logic on CPU with the gloo backend (world size 2): the
bench's max/sum over ranks and the ensemble sharding every rank computes
identically."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from lowmachmixtures_b200 import ensemble
        mx = bench.max_over_ranks(world, 10.0 + rank)
        sm = bench.sum_over_ranks(world, 1.0 + rank)
        sizes = ensemble.instance_sizes(64, seed=3)
        parts = ensemble.shard([n * n for n in sizes], world)
        mine = parts[rank]
        # every rank gathers the others' shards to check the partition
        got = [None] * world
        dist.all_gather_object(got, mine)
        out[rank] = (mx, sm, got)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_reductions_and_sharding():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    (mx0, sm0, g0), (mx1, sm1, g1) = out[0], out[1]
    assert mx0 == mx1 == 11.0 and sm0 == sm1 == 3.0
    assert g0 == g1
    allidx = sorted(i for part in g0 for i in part)
    assert allidx == list(range(64))


def test_shard_balances_cost():
    from lowmachmixtures_b200 import ensemble
    sizes = ensemble.instance_sizes(512, seed=0)
    costs = [n * n for n in sizes]
    for world in (1, 2, 4, 8):
        parts = ensemble.shard(costs, world)
        loads = [sum(costs[i] for i in p) for p in parts]
        assert sorted(i for p in parts for i in p) == list(range(512))
        assert max(loads) - min(loads) <= max(costs)


def test_instance_cost_weights_cells_by_expected_iterations():
    """A 2D instance's expected work grows with its cells and with the log of
    its viscosity contrast (the iteration count measured on the oracle)."""
    from lowmachmixtures_b200 import ensemble
    assert abs(ensemble.expected_iterations(10.0) - 12.7) < 1e-12
    assert abs(ensemble.expected_iterations(1000.0) - (12.7 + 21.2)) < 1e-9
    assert ensemble.instance_cost(128, 100.0) > ensemble.instance_cost(128, 10.0)
    assert ensemble.instance_cost(128, 10.0) == 4 * ensemble.instance_cost(64, 10.0)
    sizes = ensemble.instance_sizes(512, seed=0)
    costs = [ensemble.instance_cost(n, ensemble.instance_contrast(i)) for i, n in enumerate(sizes)]
    parts = ensemble.shard(costs, 4)
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= 1.01 * min(loads)
