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
