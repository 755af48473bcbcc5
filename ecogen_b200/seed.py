"""Learned initial guess of the pressure-relaxation Newton iteration: record, train, install.

1. ``record``: run the plain solver on training cases and let the step kernels record, for every
   converged relaxation, the features (alpha_k, log rho_k, asinh(p_k/1e5) per phase) and the
   position of the relaxed pressure inside the bracket of the phase pressures.
2. ``train``: fit the 3N -> 64 -> 64 -> 1 GELU MLP with the library's own CUDA training kernels
   (forward, backward and AdamW in ecg_mlp_train.cu).
3. ``SeedModel.install(ctx)``: copy the weights into a context; the step kernels then make the
   plain first Newton evaluation for every cell and, in warps where it leaves a cell unconverged,
   evaluate the network with BF16 tensor-core MMA inside the fused update and restart those cells
   from its output.  Newton still iterates to |f| <= 1e-10, so the plain iteration stays the judge
   of convergence.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile
from typing import List, Sequence, Tuple

import numpy as np

from . import api


class SeedModel:
    def __init__(self, mlp: api.Mlp, arrays):
        self.mlp = mlp
        self._arrays = arrays  # keep the weight buffers alive

    def install(self, ctx: api.Context):
        ctx.set_seed_model(self.mlp)

    def install_batch(self, batch_handle):
        api.check(api.lib().ecg_batch_set_seed_model(batch_handle, C.byref(self.mlp)), "ecg_batch_set_seed_model")

    def save(self, path: str):
        w1, b1, w2, b2, w3 = self._arrays
        m = self.mlp
        nout = max(1, m.n_out)
        np.savez(path, w1=w1, b1=b1, w2=w2, b2=b2, w3=w3,
                 b3=np.array([m.b3, m.b3_1][:nout], dtype=np.float32),
                 in_shift=np.array(m.in_shift[:m.n_in], dtype=np.float32),
                 in_scale=np.array(m.in_scale[:m.n_in], dtype=np.float32),
                 out_shift=np.array([m.out_shift, m.out_shift_1][:nout], dtype=np.float32),
                 out_scale=np.array([m.out_scale, m.out_scale_1][:nout], dtype=np.float32))

    @staticmethod
    def load(path: str) -> "SeedModel":
        d = np.load(path)
        return make_model(d["w1"], d["b1"], d["w2"], d["b2"], d["w3"], d["b3"], d["in_shift"], d["in_scale"],
                          d["out_shift"], d["out_scale"])


def make_model(w1, b1, w2, b2, w3, b3, in_shift, in_scale, out_shift, out_scale) -> SeedModel:
    """A model record from its arrays; b3 / out_shift / out_scale hold one value per output (a scalar
    reads as one output)."""
    arrays = [np.ascontiguousarray(a, dtype=np.float32) for a in (w1, b1, w2, b2, w3)]
    b3, osh, osc = (np.atleast_1d(np.asarray(v, dtype=np.float32)) for v in (b3, out_shift, out_scale))
    m = api.Mlp()
    m.n_in = int(len(in_shift))
    m.hidden = api.MLP_HIDDEN
    m.n_out = int(len(b3))
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    m.w1, m.b1, m.w2, m.b2, m.w3 = (fp(a) for a in arrays)
    m.b3 = float(b3[0])
    for i in range(m.n_in):
        m.in_shift[i] = float(in_shift[i])
        m.in_scale[i] = float(in_scale[i])
    m.out_shift = float(osh[0])
    m.out_scale = float(osc[0])
    if m.n_out == 2:
        m.b3_1, m.out_shift_1, m.out_scale_1 = float(b3[1]), float(osh[1]), float(osc[1])
    return SeedModel(m, arrays)


def record(case_specs: Sequence, steps: int, max_pairs: int = 2_000_000, warm: int = 0, min_evals: int = 2
           ) -> Tuple[np.ndarray, np.ndarray]:
    """Run each case on the GPU and collect (features, target) pairs of its relaxations.

    Each case first runs `warm` steps unrecorded, then records during `steps` steps the
    relaxations that took at least `min_evals` Newton evaluations (the seeded kernels ask the
    network only for those); the pair budget is shared evenly between the cases.
    """
    xs, ys = [], []
    per_case = max(1, max_pairs // max(1, len(case_specs)))
    for spec in case_specs:
        with tempfile.TemporaryDirectory() as tmp:
            d = spec.write(tmp)
            inp = api.Input(d, os.path.join(tmp, "libEOS"))
            ctx = api.Context(inp.case)
            ctx.upload(inp.fill())
            if warm:
                ctx.step(warm)
            ctx.record_pairs(per_case, min_evals)
            ctx.step(steps)
            x, y = ctx.fetch_pairs()
            ctx.close()
        xs.append(x)
        ys.append(y)
    if not xs:
        return np.zeros((0, 0), np.float32), np.zeros(0, np.float32)
    return np.concatenate(xs), np.concatenate(ys)


class Trainer:
    """The library's GPU trainer (ecg_trainer_*)."""

    def __init__(self, n_in: int, seed: int = 0, n_out: int = 1):
        h = C.c_void_p()
        api.check(api.lib().ecg_trainer_create_n(n_in, n_out, api.MLP_HIDDEN, seed, C.byref(h)),
                  "ecg_trainer_create_n")
        self.h = h
        self.n_in = n_in
        self.n_out = n_out

    def set_norm(self, in_shift, in_scale, out_shift, out_scale):
        """out_shift / out_scale: one value per output."""
        a = np.ascontiguousarray(in_shift, dtype=np.float32)
        b = np.ascontiguousarray(in_scale, dtype=np.float32)
        osh, osc = np.atleast_1d(out_shift), np.atleast_1d(out_scale)
        api.check(api.lib().ecg_trainer_set_norm(self.h, a.ctypes.data_as(C.POINTER(C.c_float)),
                                                 b.ctypes.data_as(C.POINTER(C.c_float)), float(osh[0]),
                                                 float(osc[0])), "ecg_trainer_set_norm")
        if self.n_out == 2:
            api.check(api.lib().ecg_trainer_set_norm_out1(self.h, float(osh[1]), float(osc[1])),
                      "ecg_trainer_set_norm_out1")

    def epoch(self, x: np.ndarray, y: np.ndarray, batch: int = 4096, lr: float = 1e-3, wd: float = 1e-5) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        loss = C.c_float()
        api.check(api.lib().ecg_trainer_epoch(self.h, x.ctypes.data_as(C.POINTER(C.c_float)),
                                              y.ctypes.data_as(C.POINTER(C.c_float)), len(x), batch, lr, wd,
                                              C.byref(loss)), "ecg_trainer_epoch")
        return loss.value

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.zeros((len(x), self.n_out) if self.n_out > 1 else len(x), dtype=np.float32)
        api.check(api.lib().ecg_trainer_forward(self.h, x.ctypes.data_as(C.POINTER(C.c_float)), len(x),
                                                out.ctypes.data_as(C.POINTER(C.c_float))), "ecg_trainer_forward")
        return out

    def grad(self, x: np.ndarray, y: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        H, I, O = api.MLP_HIDDEN, self.n_in, self.n_out
        g = {"w1": np.zeros((H, I), np.float32), "b1": np.zeros(H, np.float32), "w2": np.zeros((H, H), np.float32),
             "b2": np.zeros(H, np.float32), "w3": np.zeros(H * O, np.float32)}
        gb3 = np.zeros(O, np.float32)
        loss = C.c_float()
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        api.check(api.lib().ecg_trainer_grad(self.h, fp(x), fp(y), len(x), C.byref(loss), fp(g["w1"]), fp(g["b1"]),
                                             fp(g["w2"]), fp(g["b2"]), fp(g["w3"]), fp(gb3)), "ecg_trainer_grad")
        if O > 1:
            g["w3"] = g["w3"].reshape(O, H)
            g["b3"] = gb3
        else:
            g["b3"] = float(gb3[0])
        return loss.value, g

    def params(self):
        m = api.Mlp()
        api.check(api.lib().ecg_trainer_export(self.h, C.byref(m)), "ecg_trainer_export")
        H, I, O = api.MLP_HIDDEN, m.n_in, max(1, m.n_out)
        arr = lambda p, n: np.ctypeslib.as_array(p, shape=(n,)).copy()
        out = {"w1": arr(m.w1, H * I).reshape(H, I), "b1": arr(m.b1, H), "w2": arr(m.w2, H * H).reshape(H, H),
               "b2": arr(m.b2, H), "w3": arr(m.w3, H * O), "b3": m.b3,
               "in_shift": np.array(m.in_shift[:I]), "in_scale": np.array(m.in_scale[:I]),
               "out_shift": m.out_shift, "out_scale": m.out_scale}
        if O == 2:
            out["b3"] = np.array([m.b3, m.b3_1], np.float32)
            out["out_shift"] = np.array([m.out_shift, m.out_shift_1], np.float32)
            out["out_scale"] = np.array([m.out_scale, m.out_scale_1], np.float32)
        return out

    def model(self) -> SeedModel:
        p = self.params()
        return make_model(p["w1"], p["b1"], p["w2"], p["b2"], p["w3"], p["b3"], p["in_shift"], p["in_scale"],
                          p["out_shift"], p["out_scale"])

    def close(self):
        if getattr(self, "h", None):
            api.lib().ecg_trainer_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def train(x: np.ndarray, y: np.ndarray, epochs: int = 20, batch: int = 4096, lr: float = 2e-3, seed: int = 0,
          log=None) -> Tuple[SeedModel, List[float]]:
    """Normalise the features and the targets (y: n, or n x 2 for a two-output network), then fit the
    MLP on the GPU."""
    shift = x.mean(axis=0)
    scale = 1.0 / np.maximum(x.std(axis=0), 1e-6)
    xn = ((x - shift) * scale).astype(np.float32)
    nout = 1 if y.ndim == 1 else y.shape[1]
    ysh = y.mean(axis=0)
    ysc = np.maximum(y.std(axis=0), 1e-6)
    yn = ((y - ysh) / ysc).astype(np.float32)
    if nout == 1:
        ysh, ysc = float(ysh), float(ysc)
    tr = Trainer(x.shape[1], seed=seed, n_out=nout)
    tr.set_norm(shift, scale, ysh, ysc)
    rng = np.random.default_rng(seed)
    losses = []
    for ep in range(epochs):
        perm = rng.permutation(len(yn))
        l = tr.epoch(xn[perm], yn[perm], batch=batch, lr=lr * (0.5 ** (ep // max(1, epochs // 3))))
        losses.append(l)
        if log:
            log(f"epoch {ep}: loss {l:.4e}")
    m = tr.model()
    tr.close()
    return m, losses
