"""The multi-rank host path on CPU: two gloo ranks split an uneven site table
by cost, step nothing on the device, reduce a timing with MAX and gather
per-site rows on rank 0 (the exchanges bench.py makes after a run)."""
import os
import socket

import numpy as np
import pytest

from casim_b200 import configs, dist as cdist


def test_partition_is_disjoint_complete_and_balanced():
    _, sites = configs.config2(n_sites=256)
    cost = cdist.site_cost(sites, 25 ** 3)
    for world in (1, 2, 4, 8):
        parts = cdist.partition(cost, world)
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(256))
        loads = [cost[p].sum() for p in parts]
        assert max(loads) - min(loads) <= cost.max()


def test_shard_keeps_channel_rows():
    _, sites = configs.config2(n_sites=12)
    idx = np.array([3, 7, 11])
    sub = cdist.shard(sites, idx)
    off = np.concatenate([[0], np.cumsum(sites["n_ch"])])
    assert np.array_equal(sub["nx"], sites["nx"][idx])
    want = np.concatenate([sites["ch_x"][off[i]:off[i + 1]] for i in idx])
    assert np.array_equal(sub["ch_x"], want)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        _, sites = configs.config2(n_sites=10)
        parts = cdist.partition(cdist.site_cost(sites), world)
        mine = parts[rank]
        rows = np.stack([sites["nx"][mine], sites["n_ch"][mine]], axis=1).astype(np.int64)
        t = cdist.max_over_ranks(1.5 + rank)
        full = cdist.gather_sites(rows, mine, 10)
        if rank == 0:
            q.put((t, full.tolist(), np.stack([sites["nx"], sites["n_ch"]], axis=1).tolist()))
        else:
            q.put(t)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_and_gather():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    full = [r for r in res if isinstance(r, tuple)][0]
    other = [r for r in res if not isinstance(r, tuple)][0]
    assert full[0] == pytest.approx(2.5) and other == pytest.approx(2.5)
    assert full[1] == full[2]


def _oracle_batch(params, sites):
    from oracle import oracle
    return oracle.OracleSim(params, sites)


def _oracle_run(sim, sites):
    sim.start(sites["first_channel"])
    sim.step(30)


def _bench_rank(rank, world, port, q):
    import sys
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        sys.path.insert(0, ROOT)
        import bench
        params, sites = configs.small_mixed(n_sites=7, seed=13, dim=3, cytosol="RD3D")
        _, mine, _, full = bench.sharded_run(params, sites, world, rank, _oracle_batch, _oracle_run)
        q.put((rank, len(mine["nx"]), None if full is None else full.tolist()))
    finally:
        dist.destroy_process_group()


ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_rank_entry_two_gloo_ranks_equal_one():
    """bench.sharded_run, the rank body of `bench.py --gpus N`, on two gloo ranks:
    each rank steps its cost-balanced share of one global table (the oracle stands in
    for the device batch here), and the per-site outputs gathered on rank 0 equal a
    one-rank run of the whole table."""
    import sys
    import torch.multiprocessing as mp
    sys.path.insert(0, ROOT)
    import bench
    params, sites = configs.small_mixed(n_sites=7, seed=13, dim=3, cytosol="RD3D")
    _, _, _, one = bench.sharded_run(params, sites, 1, 0, _oracle_batch, _oracle_run)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bench_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=120) for _ in range(2)])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] + res[1][1] == 7 and min(res[0][1], res[1][1]) >= 2
    assert res[1][2] is None
    assert np.array_equal(np.asarray(res[0][2]), one)
    assert np.all(one[:, 2] > 0)  # every site consumed draws
