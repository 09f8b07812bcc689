"""The surrogate MLP on the tensor cores: the tcgen05 GEMM against an FP64
product of the same BF16 operands, the gradients of a full forward/backward
pass against the CPU oracle (oracle/mlp_oracle.py, same BF16 rounding points),
and training on the device lowering the loss.

Tolerances: GEMM 1e-5 of the largest |C| (FP32 accumulation order only);
gradients 2e-2 relative per layer (a different FP32 summation order can flip
an individual BF16 rounding of an activation)."""
import numpy as np
import pytest

from casim_b200 import surrogate as sg
from oracle import mlp_oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(128, 16, 64), (256, 64, 64), (128, 128, 256), (384, 256, 256), (256, 256, 1024)])
def test_tcgen05_gemm_matches_fp64(cuda_device, M, N, K):
    import torch
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    a = torch.randn((M, K), generator=g, device="cuda").to(torch.bfloat16)
    b = torch.randn((N, K), generator=g, device="cuda").to(torch.bfloat16)
    c = sg.gemm(a, b).cpu().numpy().astype(np.float64)
    ref = a.double().cpu().numpy() @ b.double().cpu().numpy().T
    err = np.max(np.abs(c - ref)) / np.max(np.abs(ref))
    assert err <= 1e-5, err


def test_gemm_rejects_unsupported_shapes(cuda_device):
    import torch
    from casim_b200 import CasimError
    a = torch.zeros((100, 64), dtype=torch.bfloat16, device="cuda")
    b = torch.zeros((16, 64), dtype=torch.bfloat16, device="cuda")
    with pytest.raises(CasimError):
        sg.gemm(a, b)  # M not a multiple of 128


def test_gradients_match_oracle(cuda_device):
    import torch
    n_in, n_out, B = 63, 20, 256
    net = sg.Surrogate(n_in, n_out, seed=7)
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, size=(B, n_in)).astype(np.float32)
    t = rng.normal(size=(B, n_out)).astype(np.float32)
    loss, g = net.gradients(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda())
    layers = net.unflatten(net.get_params())
    ref_loss, ref = mlp_oracle.gradients(layers, x, t, n_in, n_out)
    assert abs(loss - ref_loss) <= 1e-3 * abs(ref_loss)
    for l, ((gw, gb), (rw, rb)) in enumerate(zip(net.unflatten(g), ref)):
        ew = np.linalg.norm(gw - rw) / np.linalg.norm(rw)
        eb = np.linalg.norm(gb - rb) / max(np.linalg.norm(rb), 1e-30)
        assert ew <= 2e-2 and eb <= 2e-2, (l, ew, eb)
    net.close()


def test_forward_matches_oracle(cuda_device):
    import torch
    n_in, n_out, B = 40, 30, 128
    net = sg.Surrogate(n_in, n_out, width=128, depth=2, seed=11)
    x = np.random.default_rng(5).uniform(-2, 2, size=(B, n_in)).astype(np.float32)
    y = net.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    ref, _, _ = mlp_oracle.forward(net.unflatten(net.get_params()), x, n_in)
    err = np.max(np.abs(y - ref[:, :n_out])) / np.max(np.abs(ref[:, :n_out]))
    assert err <= 2e-2, err
    net.close()


def test_training_lowers_loss(cuda_device):
    import torch
    n_in, n_out, B = 16, 8, 1024
    rng = np.random.default_rng(0)
    x = rng.uniform(-1, 1, size=(B, n_in)).astype(np.float32)
    w = rng.normal(size=(n_in, n_out)).astype(np.float32)
    t = np.sin(x @ w).astype(np.float32)
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    net = sg.Surrogate(n_in, n_out, width=128, depth=3, seed=1)
    first = net.train_step(xd, td, 1e-3)
    for _ in range(300):
        last = net.train_step(xd, td, 1e-3)
    assert last < 0.1 * first, (first, last)
    assert np.all(np.isfinite(net.get_params()))
    net.close()


def test_data_parallel_training_on_the_device(cuda_device):
    """data_parallel_train with the device gradients (one rank here; the all-reduce over
    ranks is tested on gloo): the loss falls and the parameters stay finite."""
    n_in, n_out = 16, 8
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, size=(2048, n_in)).astype(np.float32)
    w = rng.normal(size=(n_in, n_out)).astype(np.float32)
    t = np.sin(x @ w).astype(np.float32)
    net = sg.Surrogate(n_in, n_out, width=128, depth=3, seed=5)
    p0 = net.get_params()
    p, hist = sg.data_parallel_train(sg.device_grad_fn(net), p0, x, t, steps=150, batch=512, lr=1e-3, seed=1)
    assert np.mean(hist[-10:]) < 0.6 * np.mean(hist[:10]), (hist[:10], hist[-10:])
    assert np.all(np.isfinite(p))
    net.close()


def test_surrogate_learns_rd_snapshots_and_beats_rd_cost(cuda_device):
    """Snapshots of the plain RD method (frozen open sets, 0.25 ms relaxation)
    train the network on the device; on held-out sites it predicts the mouth
    Ca at a small fraction of the RD cost."""
    import time
    import torch
    X, Y, rd_s = sg.rd_snapshots(8192, seed=100)
    Xv, Yv, _ = sg.rd_snapshots(1024, seed=999)
    net = sg.Surrogate(X.shape[1], Y.shape[1], seed=3)
    hist = sg.train(net, X, Y, 1500, batch=4096, lr=2e-3)
    assert np.mean(hist[-50:]) < 0.01 * hist[0]
    P = sg.predict(net, Xv)
    rel = np.abs(10.0 ** P - 10.0 ** Yv) / 10.0 ** Yv
    assert np.median(rel) < 0.10, np.median(rel)
    xd = torch.zeros((4096, X.shape[1]), dtype=torch.float32, device="cuda")
    net.forward(xd)
    torch.cuda.synchronize()
    t0 = time.time()
    for _ in range(10):
        net.forward(xd)
    torch.cuda.synchronize()
    per_site_nn = (time.time() - t0) / 10 / 4096
    per_site_rd = rd_s / 8192
    assert per_site_nn * 100 < per_site_rd, (per_site_nn, per_site_rd)
    net.close()


_NET = []


def _config1_net():
    """A network trained on 32768 frozen-open-set RD snapshots of config-1 geometry
    (trained once per test module)."""
    if not _NET:
        Xs, Ys = [], []
        for b in range(8):
            X, Y, _ = sg.rd_snapshots(4096, seed=200 + b)
            Xs.append(X)
            Ys.append(Y)
        net = sg.Surrogate(Xs[0].shape[1], Ys[0].shape[1], seed=5)
        sg.train(net, np.concatenate(Xs), np.concatenate(Ys), 3000, batch=8192, lr=2e-3)
        _NET.append(net)
    return _NET[0]


def test_surrogate_gating_tracks_rd_open_counts_faster(cuda_device):
    """Sites of config-1 geometry run 1 ms from one open RyR with RD gating
    and with surrogate gating (network every 1 us, no RD step): the mean
    number of open RyRs at 1 ms agrees within 15 % and the surrogate run is
    faster. (The quasi-steady surrogate recruits neighbours earlier than the
    RD transient does, so the counts differ more at 0.5 ms.)"""
    import time
    import torch
    import casim_b200 as cb
    from casim_b200 import configs
    net = _config1_net()
    S, T = 2048, 19800
    p, s = configs.config1(n_sites=S)
    first = np.random.default_rng(5).integers(0, 20, size=S).astype(np.int32)
    res = {}
    for mode in ("rd", "surrogate"):
        sim = cb.ReleaseSiteBatch(p, s, precision="fp32", path="auto")
        sim.start(first)
        gate = sg.SurrogateGating(net, sim, window=20) if mode == "surrogate" else None
        (sim.step if gate is None else gate.step)(200)  # warm-up: plans, graph capture
        sim.synchronize()
        torch.cuda.synchronize()
        t0 = time.time()
        (sim.step if gate is None else gate.step)(T)
        sim.synchronize()
        res[mode] = (time.time() - t0, sim.all_states().reshape(S, 20).sum(1).mean())
        sim.close()
    (t_rd, n_rd), (t_sg, n_sg) = res["rd"], res["surrogate"]
    assert abs(n_sg - n_rd) <= 0.15 * n_rd, (n_rd, n_sg)
    assert t_sg < t_rd, (t_rd, t_sg)


def test_warp_gating_matches_one_thread_gating(cuda_device):
    """Surrogate-driven gating runs one warp per site while every site has at
    most 256 RyRs and one thread per site otherwise; both consume each site's
    MRG32k3a stream in the reference's order, so the same sites under the same
    held mouth Ca follow identical RyR trajectories and draw counts."""
    import ctypes
    import torch
    import casim_b200 as cb
    from casim_b200 import configs
    p, s = configs.config1(n_sites=8)
    rng = np.random.default_rng(4)
    xs, ys = configs.lattice(300, 63 * 5.0, 63 * 5.0, rng, jitter=0.0)
    big = {k: (np.concatenate([v, v[:1]]) if isinstance(v, np.ndarray) and v.shape[:1] == (8,) else v) for k, v in s.items()}
    big["n_ch"] = np.concatenate([s["n_ch"], [300]]).astype(np.int32)
    big["ch_x"] = np.concatenate([s["ch_x"], xs])
    big["ch_y"] = np.concatenate([s["ch_y"], ys])
    big["first_channel"] = np.concatenate([s["first_channel"], [0]]).astype(np.int32)
    y = torch.from_numpy(rng.uniform(1.0, 2.5, size=(128, 300)).astype(np.float32)).cuda()
    out = []
    for table in (s, big):
        sim = cb.ReleaseSiteBatch(p, table, precision="fp32", path="plain")
        sim.start(table["first_channel"])
        sim._ck(cb.lib().casim_b200_sg_set_mouth(sim.h, ctypes.c_void_p(y.data_ptr()), 300, 1.0))
        sim._ck(cb.lib().casim_b200_sg_gate_steps(sim.h, 4000))
        sim.synchronize()
        st = sim.all_states()[:160].reshape(8, 20)
        out.append((st, [sim.draws(k) for k in range(8)]))
        sim.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1]
    assert sum(out[0][1]) > 8 * 20 * 4000  # transitions happened


def test_hybrid_run_corrects_and_falls_back(cuda_device):
    """Surrogate gating with a full-RD correction (20 steps) after every 10 windows and a
    residual check at the open RyRs: with an unreachable tolerance every period after the
    first falls back to the RD method and the run keeps the RD method's open-RyR and
    release distributions; with no check it never falls back; with a 20 % tolerance on at
    most 20 % of the sites it mixes both, runs faster than the RD method and keeps its
    open-RyR distribution (the surrogate alone releases about 20 % more Ca)."""
    import time
    import torch
    from scipy.stats import ks_2samp
    import casim_b200 as cb
    from casim_b200 import configs
    net = _config1_net()
    S, T = 2048, 19800
    p, s = configs.config1(n_sites=S)
    first = np.random.default_rng(5).integers(0, 20, size=S).astype(np.int32)
    out = {}
    for mode, hp in (("rd", None), ("strict", (10, 20, 0.01, 0.0)), ("none", (10, 20, 1e9, 0.0)), ("mixed", (10, 20, 0.2, 0.2))):
        sim = cb.ReleaseSiteBatch(p, s, precision="fp32", path="auto")
        sim.start(first)
        gate = sg.SurrogateGating(net, sim, window=20)
        run = sim.step if hp is None else (lambda n, hp=hp, gate=gate: gate.hybrid_step(n, *hp))
        run(220)  # warm-up: plans, graph capture
        sim.synchronize()
        torch.cuda.synchronize()
        t0 = time.time()
        stats = run(T)
        sim.synchronize()
        out[mode] = (time.time() - t0, sim.all_states().reshape(S, 20).sum(1), np.array([sim.release(k) for k in range(S)]), stats)
        sim.close()
    t_rd, o_rd, r_rd, _ = out["rd"]
    st = out["strict"][3]
    assert st["checks"] == 90 and st["fallbacks"] == 90 and st["surrogate_steps"] == 200
    assert ks_2samp(out["strict"][1], o_rd).pvalue > 0.05 and ks_2samp(out["strict"][2], r_rd).pvalue > 0.05
    st = out["none"][3]
    assert st["fallbacks"] == 0 and st["surrogate_steps"] == 18000 and st["rd_steps"] == 1800
    t_mx, o_mx, r_mx, st = out["mixed"]
    assert 0 < st["fallbacks"] < st["checks"], st
    assert t_mx < t_rd, (t_rd, t_mx)
    assert ks_2samp(o_mx, o_rd).pvalue > 0.05
    assert abs(r_mx.mean() / r_rd.mean() - 1) < 0.1
