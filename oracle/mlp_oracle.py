"""CPU oracle of the surrogate MLP (test infrastructure only: imported by tests/,
never by the library).

Restates, in numpy, the computation of casim_b200/csrc/surrogate.cu with the
same rounding points: inputs, hidden activations and backward pre-activation
gradients are rounded to BF16 (round to nearest even), weights are the BF16
copies of the FP32 masters, products accumulate in FP64 here (FP32 on the
device), GELU is the erf form. The surrogate has no counterpart in the
reference, so this oracle is pinned only by its own definition.
"""
import numpy as np
from scipy.special import erf


def bf16(a):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(layers, x, n_in):
    """layers: [(W [dout][din] fp32, b [dout])]; x [B][n_in]. Returns (Y, Zs, Hs)."""
    B = x.shape[0]
    din0 = layers[0][0].shape[1]
    h = np.zeros((B, din0), np.float32)
    h[:, :n_in] = x
    h = bf16(h).astype(np.float64)
    Zs, Hs = [], [h]
    for l, (W, b) in enumerate(layers):
        Wb = bf16(W).astype(np.float64)
        z = (h @ Wb.T + b.astype(np.float64)).astype(np.float32)
        if l + 1 < len(layers):
            Zs.append(z)
            h = bf16(gelu(z.astype(np.float64)).astype(np.float32)).astype(np.float64)
            Hs.append(h)
        else:
            return z, Zs, Hs


def gradients(layers, x, t, n_in, n_out):
    """Mean-square loss and [(dW, db)] per layer, as the device computes them."""
    Y, Zs, Hs = forward(layers, x, n_in)
    B = x.shape[0]
    d = Y[:, :n_out].astype(np.float64) - t.astype(np.float64)
    loss = float(np.mean(d * d))
    g = np.zeros_like(Y, dtype=np.float32)
    g[:, :n_out] = (2.0 * d / (B * n_out)).astype(np.float32)
    dz = bf16(g).astype(np.float64)
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W = bf16(layers[l][0]).astype(np.float64)
        grads[l] = ((dz.T @ Hs[l]).astype(np.float32), dz.sum(axis=0).astype(np.float32))
        if l > 0:
            dh = (dz @ W).astype(np.float32)
            dz = bf16((dh.astype(np.float64) * gelu_grad(Zs[l - 1].astype(np.float64))).astype(np.float32)).astype(np.float64)
    return loss, grads
