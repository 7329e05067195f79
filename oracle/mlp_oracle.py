"""Test infrastructure: NumPy restatement of the learned-bias network of
metad-toy_b200/csrc/mlp.cu, used only by tests/ to check the device forward,
input gradient and parameter gradient.  The reference has no learned bias,
so this pins the device code to the network's definition, not to reference
outputs.

The device rounds W1, W2, w3 to BF16 for the forward pass and rounds the
tensor-core operands h1 and dL/dz2 to BF16; this restatement applies the same
roundings and otherwise works in FP64.
"""
import numpy as np

H = 128
IN = 4
O_W1 = 0
O_B1 = O_W1 + H * IN
O_W2 = O_B1 + H
O_B2 = O_W2 + H * H
O_W3 = O_B2 + H
O_B3 = O_W3 + H
NP = O_B3 + 1


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    a = np.asarray(x, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    r = ((b >> 16) & 1) + 0x7FFF
    out = ((b + r) & 0xFFFF0000).astype(np.uint32).view(np.float32)
    return out.astype(np.float64)


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    return (w[O_W1:O_B1].reshape(H, IN), w[O_B1:O_W2], w[O_W2:O_B2].reshape(H, H), w[O_B2:O_W3],
            w[O_W3:O_B3], w[O_B3])


def normalise(pts, lo, hi):
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    u = np.zeros((pts.shape[0], IN))
    u[:, :pts.shape[1]] = (2.0 * (pts - lo) / (hi - lo) - 1.0).astype(np.float32)
    return u


def _silu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return z * s, s * (1.0 + z * (1.0 - s))


def forward(w, u):
    W1, b1, W2, b2, w3, b3 = unpack(w)
    W1b, W2b, w3b = bf16(W1), bf16(W2), bf16(w3)
    z1 = u @ W1b.T + b1
    h1, d1 = _silu(z1)
    h1b = bf16(h1)
    z2 = h1b @ W2b.T + b2
    h2, d2 = _silu(z2)
    y = h2 @ w3b + b3
    return dict(W1b=W1b, W2b=W2b, w3b=w3b, z1=z1, d1=d1, h1b=h1b, z2=z2, h2=h2, d2=d2, y=y)


def input_grad(w, u):
    """dy/du per point (D <= 4 slots)."""
    f = forward(w, u)
    dz2 = bf16(f["w3b"][None, :] * f["d2"])
    dh1 = dz2 @ f["W2b"]
    dz1 = dh1 * f["d1"]
    return f["y"], dz1 @ f["W1b"]


def loss_grad(w, u, t):
    """Gradient of sum_i (y_i - t_i)^2 / n over the flat parameters."""
    n = u.shape[0]
    f = forward(w, u)
    dy = 2.0 / n * (f["y"] - t)
    g = np.zeros(NP)
    dz2 = dy[:, None] * f["w3b"][None, :] * f["d2"]
    dz2b = bf16(dz2)
    g[O_B2:O_W3] = dz2.sum(0)
    g[O_W3:O_B3] = (dy[:, None] * f["h2"]).sum(0)
    g[O_B3] = dy.sum()
    g[O_W2:O_B2] = (dz2b.T @ f["h1b"]).reshape(-1)
    dh1 = dz2b @ f["W2b"]
    dz1 = dh1 * f["d1"]
    g[O_B1:O_W2] = dz1.sum(0)
    g[O_W1:O_B1] = (dz1.T @ u).reshape(-1)
    return g, float(np.mean((f["y"] - t) ** 2))


def hill_sum(pts, centers, heights, sigmas):
    """Exact FP64 sum of isotropic Gaussians and its gradient."""
    pts = np.asarray(pts, dtype=np.float64)
    V = np.zeros(pts.shape[0])
    dV = np.zeros_like(pts)
    for c, h, s in zip(centers, heights, sigmas):
        d = pts - c
        e = h * np.exp(-(d * d).sum(1) / (2.0 * s * s))
        V += e
        dV -= e[:, None] * d / (s * s)
    return V, dV
