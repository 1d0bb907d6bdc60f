"""CPU restatement of the learned warm start's network, FP64 (numpy). TEST INFRASTRUCTURE ONLY: the checker the
tensor-core forward / backward kernels are compared against; only tests/ import it.

The network is the library's own (the reference has no counterpart; it replaces the initial guess of
ThreeD/Forging3DSolver.cs:854-869): per node 16 inputs -> 128 -> 128 -> 128 (GELU, erf form) -> 3, mean squared
error over normalised targets. ``bf16=True`` rounds to bfloat16 exactly where the GPU path stores BF16 (inputs,
hidden weights, hidden activations and their gradients), so that the remaining difference is FP32 accumulation
order; ``bf16=False`` is the exact FP64 network at the same parameters.

Parameter layout (flat FP32, as ifea_mlp_get_params): W1 [128][16], b1, W2 [128][128], b2, W3 [128][128], b3,
W4 [3][128], b4.
"""
import numpy as np
from scipy.special import erf

NIN, HID, NOUT = 16, 128, 3
SHAPES = [("W1", (HID, NIN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (HID, HID)), ("b3", (HID,)),
          ("W4", (NOUT, HID)), ("b4", (NOUT,))]
NPAR = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(flat):
    out, k = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(flat[k:k + n], np.float64).reshape(shape)
        k += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in SHAPES])


def to_bf16(a):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_d(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(flat, x, bf16=False):
    """Outputs (in normalised target units) and the intermediates, for normalised inputs x [n][16]."""
    p = unpack(flat)
    r = to_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))
    h0 = r(x)
    z1 = h0 @ r(p["W1"]).T + p["b1"]
    h1 = r(gelu(z1))
    z2 = h1 @ r(p["W2"]).T + p["b2"]
    h2 = r(gelu(z2))
    z3 = h2 @ r(p["W3"]).T + p["b3"]
    h3 = r(gelu(z3))
    y = h3 @ p["W4"].T + p["b4"]
    return y, (h0, z1, h1, z2, h2, z3, h3)


def loss_and_gradients(flat, x, t, bf16=False):
    """Mean squared error over n x 3 outputs and its gradient (flat, NPAR values)."""
    p = unpack(flat)
    r = to_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))
    y, (h0, z1, h1, z2, h2, z3, h3) = forward(flat, x, bf16)
    n = len(x)
    e = y - t
    loss = float((e * e).sum() / (n * NOUT))
    dy = 2.0 * e / (n * NOUT)
    g = {"W4": dy.T @ h3, "b4": dy.sum(0)}
    dz3 = r((dy @ p["W4"]) * gelu_d(z3))
    g["W3"], g["b3"] = dz3.T @ h2, dz3.sum(0)
    dz2 = r((dz3 @ r(p["W3"])) * gelu_d(z2))
    g["W2"], g["b2"] = dz2.T @ h1, dz2.sum(0)
    dz1 = r((dz2 @ r(p["W2"])) * gelu_d(z1))
    g["W1"], g["b1"] = dz1.T @ h0, dz1.sum(0)
    return loss, pack(g)


def adam_step(w, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (Kingma and Ba 2015) in FP32, as the GPU applies it; returns (w, m, v)."""
    w, g, m, v = (np.asarray(a, np.float32) for a in (w, g, m, v))
    m = np.float32(b1) * m + np.float32(1 - b1) * g
    v = np.float32(b2) * v + np.float32(1 - b2) * g * g
    bc1, bc2 = np.float32(1 - b1 ** t), np.float32(1 - b2 ** t)
    w = w - np.float32(lr) * (m / bc1) / (np.sqrt(v / bc2) + np.float32(eps))
    return w, m, v
