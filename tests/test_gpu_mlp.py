"""Learned relaxation seed: GPU training kernels vs the FP64 CPU check, and what the seed gains."""
import numpy as np
import pytest

from ecogen_b200 import api, cases, seed
from tests.conftest import rel_l1
from tests.helpers import gpu_run
from tests.mlp_reference import forward_backward


@pytest.mark.gpu
def test_training_gradients_match_cpu_reference():
    rng = np.random.default_rng(3)
    tr = seed.Trainer(9, seed=11)
    x = rng.normal(size=(300, 9)).astype(np.float32)
    y = rng.normal(size=300).astype(np.float32)
    loss, g = tr.grad(x, y)
    p = tr.params()
    ref_loss, rg, _ = forward_backward(p, x, y)
    assert loss == pytest.approx(ref_loss, rel=1e-4)
    for k in ("w1", "b1", "w2", "b2", "w3"):
        err = np.abs(g[k] - rg[k]).max() / max(np.abs(rg[k]).max(), 1e-12)
        assert err < 2e-4, (k, err)
    assert g["b3"] == pytest.approx(rg["b3"], rel=1e-4, abs=1e-7)
    yh = tr.forward(x)
    assert np.allclose(yh, forward_backward(p, x, y)[2], rtol=1e-4, atol=1e-5)
    tr.close()


@pytest.mark.gpu
def test_training_reduces_loss():
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, size=(20000, 6)).astype(np.float32)
    y = (np.tanh(x[:, 0] * 2 + x[:, 1]) * 0.5 + 0.5).astype(np.float32)
    model, losses = seed.train(x, y, epochs=12, batch=1024, lr=3e-3)
    assert losses[-1] < 0.1 * losses[0]


def _run(case, tmp, model=None):
    import os
    d = case.write(str(tmp))
    inp = api.Input(d, os.path.join(str(tmp), "libEOS"))
    ctx = api.Context(inp.case)
    ctx.upload(inp.fill())
    if model is not None:
        model.install(ctx)
    st = ctx.step(case.iterations)
    out = ctx.download_dict()
    ctx.close()
    return out, st


@pytest.mark.gpu
def test_seeded_relaxation_same_residual_fewer_iterations(tmp_path):
    train_cases = [cases.cavity_collapse_3d(n=24, iterations=6, seed=100 + s, ninclusions=10, radius_cells=(2.0, 5.0))
                   for s in range(4)]
    x, y = seed.record(train_cases, steps=6, max_pairs=400000)
    assert len(y) > 10000 and np.all(np.isfinite(x)) and np.all((y >= -1e-3) & (y <= 1.001))
    model, losses = seed.train(x, y, epochs=15, batch=2048, lr=2e-3)
    test_case = cases.cavity_collapse_3d(n=24, iterations=6, seed=999, ninclusions=10, radius_cells=(2.0, 5.0))
    plain, st0 = _run(test_case, tmp_path / "plain")
    seeded, st1 = _run(test_case, tmp_path / "seeded", model)
    # the network is asked only for cells the plain first evaluation leaves unconverged
    assert 0 < st1.seeded + st1.seed_rejected < st1.relax_calls
    assert st1.newton_fallback == 0
    # same residual: Newton stops at |f| <= 1e-10 from either start, so fields agree to that level
    for name in ("alpha", "rho", "p", "E"):
        assert rel_l1(seeded[name], plain[name]) < 1e-8, name
    # the trained seed needs no more Newton evaluations than the plain start
    assert st1.newton_evals <= st0.newton_evals
