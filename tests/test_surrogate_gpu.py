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
