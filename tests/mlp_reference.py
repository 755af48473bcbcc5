"""FP64 numpy forward/backward of the seed MLP — the CPU check of the GPU training kernels.

Same network as ecogen_b200/csrc/ecg_mlp_train.cu: nin -> 64 -> 64 -> nout (1 or 2), tanh-approximated
GELU, loss the sum over outputs of the mean squared error.
"""
import numpy as np

C = 0.7978845608028654


def gelu(z):
    u = C * (z + 0.044715 * z ** 3)
    th = np.tanh(u)
    d = 0.5 * (1 + th) + 0.5 * z * (1 - th ** 2) * C * (1 + 3 * 0.044715 * z ** 2)
    return 0.5 * z * (1 + th), d


def forward_backward(p, x, y):
    """p: w1 (H, I), b1, w2 (H, H), b2, w3 (H,) or (O, H), b3 scalar or (O,); y: (n,) or (n, O)."""
    x = x.astype(np.float64)
    one = np.ndim(y) == 1
    y2 = np.asarray(y, dtype=np.float64).reshape(len(y), -1)
    w3 = np.asarray(p["w3"], dtype=np.float64).reshape(y2.shape[1], -1)
    b3 = np.atleast_1d(np.asarray(p["b3"], dtype=np.float64))
    n = len(y2)
    z1 = x @ p["w1"].T.astype(np.float64) + p["b1"]
    h1, d1 = gelu(z1)
    z2 = h1 @ p["w2"].T.astype(np.float64) + p["b2"]
    h2, d2 = gelu(z2)
    yh = h2 @ w3.T + b3
    e = yh - y2
    loss = np.sum(np.mean(e ** 2, axis=0))
    dy = 2 * e / n
    g = {"b3": dy.sum(0), "w3": dy.T @ h2}
    dz2 = (dy @ w3) * d2
    g["w2"] = dz2.T @ h1
    g["b2"] = dz2.sum(0)
    dh1 = dz2 @ p["w2"].astype(np.float64)
    dz1 = dh1 * d1
    g["w1"] = dz1.T @ x
    g["b1"] = dz1.sum(0)
    if one:
        g["b3"], g["w3"], yh = float(g["b3"][0]), g["w3"][0], yh[:, 0]
    return loss, g, yh
