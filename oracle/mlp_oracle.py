"""Oracle (test infrastructure only): float64 restatement of the warm-start network, its training
loss and its gradients, optionally with the bf16 roundings the tensor-core kernels apply.

The network is the one the learned warm start uses: 24 features -> 64 -> SiLU -> 64 -> SiLU -> 3,
features normalised by (x - in_mean) * in_scale, targets by 1 / out_scale. The loss over n rows is
L = sum (y - t / out_scale)^2 / (3 n); its gradients are those of plain back-propagation.

With round_bf16=True every value that the device feeds to a tensor-core MMA is rounded to bf16
(round to nearest even) at the same point as on the device: the weights, the normalised inputs,
the hidden activations, and the back-propagated errors dy, dz2, dz1 that the backward and
weight-gradient MMAs consume. Biases, pre-activations (z1, z2, kept in FP32 for the SiLU
derivatives) and the output error e stay unrounded. What then separates the device from this
restatement is FP32 accumulation order, the fast exponential in SiLU, and values that sit next
to a bf16 rounding boundary.

Nothing in the library imports this module; tests do.
"""
import numpy as np


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def _ident(x):
    return np.asarray(x, np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(W, x, round_bf16=True):
    """Network output in target units (n x 3)."""
    q = bf16 if round_bf16 else _ident
    f = {k: np.asarray(v, np.float64) for k, v in W.items()}
    xn = q(((np.asarray(x, np.float32) - W["in_mean"]) * W["in_scale"]).astype(np.float32))
    h1 = q(silu(xn @ q(W["w1"]).T + f["b1"]))
    h2 = q(silu(h1 @ q(W["w2"]).T + f["b2"]))
    return (h2 @ q(W["w3"]).T + f["b3"]) * f["out_scale"]


def loss_and_gradients(W, x, t, round_bf16=True):
    """(loss, {w1, b1, w2, b2, w3, b3}) over the rows of x (n x 24) and t (n x 3)."""
    q = bf16 if round_bf16 else _ident
    f = {k: np.asarray(v, np.float64) for k, v in W.items()}
    w1, w2, w3 = q(W["w1"]), q(W["w2"]), q(W["w3"])
    xn32 = ((np.asarray(x, np.float32) - W["in_mean"]) * W["in_scale"]).astype(np.float32)
    xn = q(xn32)
    z1 = xn @ w1.T + f["b1"]
    h1 = q(silu(z1))
    z2 = h1 @ w2.T + f["b2"]
    h2 = q(silu(z2))
    y = h2 @ w3.T + f["b3"]
    tn = (np.asarray(t, np.float32) / W["out_scale"]).astype(np.float32).astype(np.float64)
    e = y - tn
    n = len(x)
    loss = float((e * e).sum() / (3 * n))
    dy = q(2.0 * e / (3 * n))
    g = {"w3": dy.T @ h2, "b3": dy.sum(0)}
    dz2 = q((dy @ w3) * dsilu(z2))
    g["w2"], g["b2"] = dz2.T @ h1, dz2.sum(0)
    dz1 = q((dz2 @ w2) * dsilu(z1))
    g["w1"], g["b1"] = dz1.T @ xn, dz1.sum(0)
    return loss, g
