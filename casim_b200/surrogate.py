"""Surrogate of the quasi-steady Ca at the RyR mouths (host side).

The network, its forward and backward passes and the Adam update run in
libcasim_b200.so on the tensor cores (tcgen05, BF16 operands, FP32
accumulation); this module binds the casim_b200_sg_* entry points of
include/casim_b200.h and builds the training set from the plain RD solver of
the same library: each snapshot is one site held at a fixed set of open RyRs
(gating frozen) until the cleft Ca has relaxed, then read at every mouth.

Features of a site (config-1 layout, built on the device from the site's
current state so that training and use see the same values; padded RyR slots
are zero): per RyR slot its open flag and grid position scaled to [-1, 1] by
the cleft half-widths; then jSR Ca / 1000 uM; then each buffer total / its
config value.
Targets: log10(mouth Ca / 1 uM) per RyR slot (zero for empty slots).

Device data are torch tensors (torch is the device-memory plumbing here).
"""
import ctypes

import numpy as np

from . import CasimError, lib

WIDTH, DEPTH = 256, 4


def _ck(st, h=None):
    if st != 0:
        msg = ""
        if h:
            buf = ctypes.create_string_buffer(1024)
            lib().casim_b200_sg_last_error(h, buf, 1024)
            msg = buf.value.decode()
        raise CasimError(st, msg or "surrogate call failed")


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class Surrogate:
    """MLP n_in -> depth x width (GELU) -> n_out on the device."""

    def __init__(self, n_in, n_out, width=WIDTH, depth=DEPTH, seed=1234):
        self.n_in, self.n_out, self.width, self.depth = n_in, n_out, width, depth
        self.h = ctypes.c_void_p()
        _ck(lib().casim_b200_sg_create(n_in, n_out, width, depth, seed, ctypes.byref(self.h)))

    def close(self):
        if self.h:
            lib().casim_b200_sg_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr):
        _ck(lib().casim_b200_sg_set_stream(self.h, ctypes.c_void_p(stream_ptr)), self.h)

    def num_params(self):
        n = ctypes.c_int64()
        _ck(lib().casim_b200_sg_num_params(self.h, ctypes.byref(n)), self.h)
        return n.value

    def layer_shapes(self):
        """(dout, din) of each layer, padded as the library stores them."""
        in_pad = (self.n_in + 63) // 64 * 64
        out_pad = (self.n_out + 127) // 128 * 128
        dims = [in_pad] + [self.width] * self.depth + [out_pad]
        return [(dims[i + 1], dims[i]) for i in range(self.depth + 1)]

    def get_params(self):
        out = np.zeros(self.num_params(), np.float32)
        _ck(lib().casim_b200_sg_get_params(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))), self.h)
        return out

    def set_params(self, flat):
        flat = np.ascontiguousarray(flat, np.float32)
        assert flat.size == self.num_params()
        _ck(lib().casim_b200_sg_set_params(self.h, flat.ctypes.data_as(ctypes.POINTER(ctypes.c_float))), self.h)

    def unflatten(self, flat):
        """[(W [dout][din], b [dout]) per layer] views of a flat parameter vector."""
        out, off = [], 0
        for dout, din in self.layer_shapes():
            w = flat[off:off + dout * din].reshape(dout, din)
            off += dout * din
            b = flat[off:off + dout]
            off += dout
            out.append((w, b))
        return out

    def forward(self, x):
        """x: float32 CUDA tensor [batch, n_in], batch a multiple of 128."""
        import torch
        y = torch.empty((x.shape[0], self.n_out), dtype=torch.float32, device=x.device)
        _ck(lib().casim_b200_sg_forward(self.h, _ptr(x), int(x.shape[0]), _ptr(y)), self.h)
        return y

    def gradients(self, x, t):
        loss = ctypes.c_float()
        g = np.zeros(self.num_params(), np.float32)
        _ck(lib().casim_b200_sg_gradients(self.h, _ptr(x), _ptr(t), int(x.shape[0]), ctypes.byref(loss),
                                          g.ctypes.data_as(ctypes.POINTER(ctypes.c_float))), self.h)
        return float(loss.value), g

    def train_step(self, x, t, lr):
        loss = ctypes.c_float()
        _ck(lib().casim_b200_sg_train_step(self.h, _ptr(x), _ptr(t), int(x.shape[0]), float(lr), ctypes.byref(loss)), self.h)
        return float(loss.value)

    def launches(self):
        n = ctypes.c_int64()
        _ck(lib().casim_b200_sg_launches(self.h, ctypes.byref(n)), self.h)
        return n.value


def gemm(a_bf16, b_bf16):
    """C = A . B^T on the tensor cores; a [M, K], b [N, K] bfloat16 CUDA tensors."""
    import torch
    M, K = a_bf16.shape
    N = b_bf16.shape[0]
    c = torch.empty((M, N), dtype=torch.float32, device=a_bf16.device)
    _ck(lib().casim_b200_sg_gemm(_ptr(a_bf16), _ptr(b_bf16), M, N, K, _ptr(c)))
    return c


def n_features(max_ch, n_buf=2):
    return 3 * max_ch + 1 + n_buf


def device_features(sim, max_ch):
    """Features of every site of a ReleaseSiteBatch from its current RyR states and
    jSR Ca, built on the device (casim_b200_sg_features); a CUDA tensor
    [S padded to a multiple of 128, n_features]."""
    import torch
    ld = n_features(max_ch, int(sim.info.n_buffers))
    X = torch.zeros(((sim.S + 127) // 128 * 128, ld), dtype=torch.float32, device="cuda")
    # the batch runs on its own stream unless one was set: order the zero fill
    # (torch's stream) before the kernel and the kernel before any later reader
    torch.cuda.current_stream().synchronize()
    sim._ck(lib().casim_b200_sg_features(sim.h, max_ch, ld, _ptr(X)))
    sim.synchronize()
    return X


# ---------------------------------------------------------------- snapshots
RELAX_STEPS = 5000  # 0.25 ms at dt = 50 ns: the time a frozen open set is held before the mouths are read
CA_REF_UM = 1.0     # targets are log10(mouth Ca / CA_REF_UM)


def snapshot_batch(n_sites, seed=0, n_ryr=20, max_open=20, jsr_range=(100.0, 1500.0)):
    """Config-1 sites (2D 64 x 64, 20 RyRs on the jittered 31 nm lattice) with a
    random frozen open set of 1..max_open RyRs and a constant jSR Ca per site.
    Returns (params, sites, open_mask [S, n_ryr], jsr [S])."""
    from . import configs
    frozen = {"kopen0": 0.0, "ncaopen": 2.5, "kopenmax": 1e15, "kclose0": 0.0, "ncaclose": 0.0}
    p = configs.base_params(dim=2, nx=64, ny=64, gating=frozen)
    p["jSR"]["Constant"] = True
    p = configs._clean(p)
    rng = np.random.default_rng(seed)
    xs, ys, seeds = [], [], []
    jsr = rng.uniform(jsr_range[0], jsr_range[1], size=n_sites)
    mask = np.zeros((n_sites, n_ryr), np.float32)
    for k in range(n_sites):
        x, y = configs.lattice(n_ryr, 63 * 5.0, 63 * 5.0, rng)
        xs += x
        ys += y
        seeds.append([int(v) for v in rng.integers(1, 4294944443, size=6)])
        n_open = int(rng.integers(1, min(max_open, n_ryr) + 1))
        mask[k, rng.choice(n_ryr, size=n_open, replace=False)] = 1.0
    sites = configs.sites_table([64] * n_sites, [64] * n_sites, [1] * n_sites, [n_ryr] * n_sites, xs, ys, seeds,
                                jsr_init=jsr.reshape(-1, 1))
    return p, sites, mask, jsr


def rd_snapshots(n_sites, seed=0, relax_steps=RELAX_STEPS, precision="fp32", n_ryr=20, max_open=20):
    """Features and targets of n_sites snapshots computed by the plain RD method
    of this library: reset, open the frozen set, relax_steps RD steps, read the
    Ca at every mouth. Returns (X [S, F], Y [S, n_ryr], seconds of RD device time)."""
    from . import ReleaseSiteBatch
    p, s, mask, jsr = snapshot_batch(n_sites, seed, n_ryr, max_open)
    sim = ReleaseSiteBatch(p, s, precision=precision, path="auto")
    sim.reset()
    sim.set_all_states(mask.astype(np.int32).reshape(-1))
    sim.update()
    sim.step(relax_steps)
    sim.synchronize()
    secs = sim.last_step_ms() / 1e3
    st = sim.all_states().reshape(n_sites, n_ryr)
    assert np.array_equal(st, mask.astype(np.int32)), "gating was not frozen"
    ca = sim.all_mouth(0).reshape(n_sites, n_ryr)
    X = device_features(sim, n_ryr)[:n_sites].cpu().numpy()
    sim.close()
    Y = np.log10(np.maximum(ca, 1e-6) / CA_REF_UM).astype(np.float32)
    return X, Y, secs


def dynamic_snapshots(n_sites, seed=0, every=1000, samples=20, precision="fp32"):
    """Features and targets read from the plain RD method while it gates: config-1 sites
    started from one random open RyR, sampled every `every` steps (`samples` times), so the
    training set holds the open sets, jSR depletion and transient mouth Ca of real runs.
    Returns (X [n_sites * samples, F], Y [n_sites * samples, 20])."""
    from . import ReleaseSiteBatch
    from . import configs
    p, s = configs.config1(n_sites=n_sites, seed0=1000 + seed)
    first = np.random.default_rng(seed).integers(0, 20, size=n_sites).astype(np.int32)
    sim = ReleaseSiteBatch(p, s, precision=precision, path="auto")
    sim.start(first)
    Xs, Ys = [], []
    for _ in range(samples):
        sim.step(every)
        sim.synchronize()
        ca = sim.all_mouth(0).reshape(n_sites, 20)
        Xs.append(device_features(sim, 20)[:n_sites].cpu().numpy())
        Ys.append(np.log10(np.maximum(ca, 1e-6) / CA_REF_UM).astype(np.float32))
    sim.close()
    return np.concatenate(Xs), np.concatenate(Ys)


def train(net, X, Y, steps, batch=4096, lr=1e-3, seed=0, lr_decay=True):
    """Adam on random mini-batches of (X, Y) held on the device; returns the loss history."""
    import torch
    xd = torch.from_numpy(np.ascontiguousarray(X, np.float32)).cuda()
    yd = torch.from_numpy(np.ascontiguousarray(Y, np.float32)).cuda()
    g = torch.Generator(device="cuda").manual_seed(seed)
    n = xd.shape[0]
    batch = min(batch, n // 128 * 128)
    hist = []
    for k in range(steps):
        idx = torch.randint(0, n, (batch,), device="cuda", generator=g)
        rate = lr * (0.5 * (1 + np.cos(np.pi * k / steps)) if lr_decay else 1.0) + 1e-6
        hist.append(net.train_step(xd[idx].contiguous(), yd[idx].contiguous(), rate))
    return hist


def predict(net, X):
    """Network output for X (host array), padding the batch to a multiple of 128."""
    import torch
    n = X.shape[0]
    npad = (n + 127) // 128 * 128
    xp = np.zeros((npad, X.shape[1]), np.float32)
    xp[:n] = X
    return net.forward(torch.from_numpy(xp).cuda()).cpu().numpy()[:n]


class SurrogateGating:
    """Gating of a ReleaseSiteBatch (pool cytosol) driven by the surrogate's
    mouth Ca instead of the RD step: every `window` time steps the network is
    evaluated on the features of the current open sets and jSR Ca and the mouth
    Ca replaced; in between, gating, the jSR and pool ODEs and the RyR currents
    run with the mouth values held. The whole loop runs on the batch's stream
    (casim_b200_sg_run, one captured window replayed as a CUDA graph)."""

    def __init__(self, net, sim, max_ch=20, window=20):
        self.net, self.sim, self.max_ch, self.window = net, sim, max_ch, window

    def step(self, n):
        self.sim._ck(lib().casim_b200_sg_run(self.sim.h, self.net.h, self.max_ch, int(n), self.window, CA_REF_UM))

    def hybrid_step(self, n, windows_per_check=10, rd_steps=20, tol=0.01, max_fail_fraction=0.0):
        """n steps alternating surrogate periods (windows_per_check windows) with a
        full-RD correction of rd_steps steps, a residual check of the network against
        it (relative mouth-Ca error tol per site) and a fallback to the full RD method
        for the next period when more than max_fail_fraction of the sites fail
        (casim_b200_sg_hybrid_run). Returns the run's statistics."""
        from . import HybridStats
        st = HybridStats()
        self.sim._ck(lib().casim_b200_sg_hybrid_run(self.sim.h, self.net.h, self.max_ch, int(n), self.window, int(windows_per_check),
                                                    int(rd_steps), float(tol), float(max_fail_fraction), CA_REF_UM,
                                                    ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in HybridStats._fields_}


def data_parallel_train(grad_fn, params, X, Y, steps, batch=4096, lr=1e-3, seed=0, group=None):
    """Data-parallel training over the ranks of a torch.distributed process group (NCCL
    between GPUs, gloo on CPU; one rank when no group is initialised): every step all
    ranks draw the same global mini-batch of `batch` rows of (X, Y), each takes its equal
    share, grad_fn(params, x, y) -> (loss, flat gradients) gives the mean-square loss
    gradient of that share (a Surrogate's `gradients` on the device, see
    `device_grad_fn`), the shares' gradients are averaged by an all-reduce, and every
    rank applies the same Adam step (beta 0.9 / 0.999, eps 1e-8) to its FP32 copy of
    the parameters, which therefore stay identical on all ranks. Returns (params, the
    averaged loss per step)."""
    import torch
    import torch.distributed as tdist
    world = tdist.get_world_size(group) if tdist.is_available() and tdist.is_initialized() else 1
    rank = tdist.get_rank(group) if world > 1 else 0
    n = X.shape[0]
    share = batch // world
    if share < 1:
        raise ValueError("batch smaller than the number of ranks")
    p = np.array(params, dtype=np.float32, copy=True)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    b1, b2, eps = 0.9, 0.999, 1e-8
    hist = []
    for k in range(steps):
        idx = np.random.default_rng(seed + k).integers(0, n, size=share * world)
        mine = idx[rank * share:(rank + 1) * share]
        loss, g = grad_fn(p, X[mine], Y[mine])
        buf = torch.from_numpy(np.concatenate([np.asarray(g, np.float32), np.float32([loss])]))
        if world > 1:
            tdist.all_reduce(buf, op=tdist.ReduceOp.SUM, group=group)
            buf /= world
        g = buf[:-1].numpy()
        hist.append(float(buf[-1]))
        m = b1 * m + (1 - b1) * g
        v = b2 * v + (1 - b2) * g * g
        mh = m / (1 - b1 ** (k + 1))
        vh = v / (1 - b2 ** (k + 1))
        p = (p - lr * mh / (np.sqrt(vh) + eps)).astype(np.float32)
    return p, hist


def device_grad_fn(net):
    """grad_fn of data_parallel_train for a Surrogate on this rank's GPU: the parameters
    and this rank's share of the batch go to the device, the gradients come back (the
    device kernels take batches of a multiple of 128 rows, so each share must be one)."""
    import torch

    def fn(params, x, y):
        if x.shape[0] % 128:
            raise ValueError("each rank's share of the batch must be a multiple of 128 rows")
        net.set_params(params)
        xd = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
        yd = torch.from_numpy(np.ascontiguousarray(y, np.float32)).cuda()
        return net.gradients(xd, yd)
    return fn
