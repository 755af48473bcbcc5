"""FP64 numpy forward/backward of the seed MLP — the CPU check of the GPU training kernels.

Same network as ecogen_b200/csrc/ecg_mlp_train.cu: nin -> 64 -> 64 -> 1, tanh-approximated GELU,
mean squared error.
"""
import numpy as np

C = 0.7978845608028654


def gelu(z):
    u = C * (z + 0.044715 * z ** 3)
    th = np.tanh(u)
    d = 0.5 * (1 + th) + 0.5 * z * (1 - th ** 2) * C * (1 + 3 * 0.044715 * z ** 2)
    return 0.5 * z * (1 + th), d


def forward_backward(p, x, y):
    x = x.astype(np.float64)
    y = y.astype(np.float64)
    n = len(y)
    z1 = x @ p["w1"].T.astype(np.float64) + p["b1"]
    h1, d1 = gelu(z1)
    z2 = h1 @ p["w2"].T.astype(np.float64) + p["b2"]
    h2, d2 = gelu(z2)
    yh = h2 @ p["w3"].astype(np.float64) + p["b3"]
    e = yh - y
    loss = np.mean(e ** 2)
    dy = 2 * e / n
    g = {"b3": dy.sum(), "w3": h2.T @ dy}
    dz2 = np.outer(dy, p["w3"]) * d2
    g["w2"] = dz2.T @ h1
    g["b2"] = dz2.sum(0)
    dh1 = dz2 @ p["w2"].astype(np.float64)
    dz1 = dh1 * d1
    g["w1"] = dz1.T @ x
    g["b1"] = dz1.sum(0)
    return loss, g, yh
