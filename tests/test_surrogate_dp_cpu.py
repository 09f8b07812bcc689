"""Data-parallel surrogate training on CPU: two gloo ranks, each taking half of every
global mini-batch, average their gradients by an all-reduce and apply the same Adam
step; their parameters stay identical and equal a one-rank run on whole batches. The
MLP oracle (the numpy restatement of the device network) stands in for the device
gradients here."""
import os
import socket

import numpy as np

from casim_b200 import surrogate as sg
from oracle import mlp_oracle

N_IN, N_OUT, WIDTH, DEPTH = 8, 4, 16, 2
SHAPES = [(WIDTH, N_IN)] + [(WIDTH, WIDTH)] * (DEPTH - 1) + [(N_OUT, WIDTH)]


def _unflatten(p):
    out, off = [], 0
    for dout, din in SHAPES:
        w = p[off:off + dout * din].reshape(dout, din)
        off += dout * din
        out.append((w, p[off:off + dout]))
        off += dout
    return out


def _grad_fn(p, x, y):
    loss, grads = mlp_oracle.gradients(_unflatten(p), x, y, N_IN, N_OUT)
    return loss, np.concatenate([np.concatenate([gw.ravel(), gb.ravel()]) for gw, gb in grads]).astype(np.float32)


def _data():
    rng = np.random.default_rng(4)
    X = rng.standard_normal((512, N_IN)).astype(np.float32)
    Y = np.tanh(X[:, :N_OUT] * 0.5).astype(np.float32)
    p0 = np.concatenate([np.concatenate([(rng.standard_normal(dout * din) / np.sqrt(din)).astype(np.float32),
                                         np.zeros(dout, np.float32)]) for dout, din in SHAPES])
    return X, Y, p0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        X, Y, p0 = _data()
        p, hist = sg.data_parallel_train(_grad_fn, p0, X, Y, steps=6, batch=128, lr=3e-3, seed=2)
        q.put((rank, p.tolist(), hist))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_train_as_one():
    import torch.multiprocessing as mp
    X, Y, p0 = _data()
    p1, h1 = sg.data_parallel_train(_grad_fn, p0, X, Y, steps=6, batch=128, lr=3e-3, seed=2)
    assert h1[-1] < h1[0]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = sorted([q.get(timeout=120) for _ in range(2)])
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    pa, pb = np.array(res[0][1], np.float32), np.array(res[1][1], np.float32)
    assert np.array_equal(pa, pb)  # the ranks' parameters stay identical
    assert np.allclose(pa, p1, rtol=1e-5, atol=1e-7)
    assert np.allclose(res[0][2], h1, rtol=1e-5)
