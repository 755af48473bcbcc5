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
def test_training_gradients_match_cpu_reference_two_outputs():
    """The 8 -> 64 -> 64 -> 2 network of the p-T-mu seed: both heads' gradients and outputs."""
    rng = np.random.default_rng(4)
    tr = seed.Trainer(8, seed=12, n_out=2)
    x = rng.normal(size=(257, 8)).astype(np.float32)
    y = rng.normal(size=(257, 2)).astype(np.float32)
    loss, g = tr.grad(x, y)
    p = tr.params()
    ref_loss, rg, yref = forward_backward(p, x, y)
    assert loss == pytest.approx(ref_loss, rel=1e-4)
    for k in ("w1", "b1", "w2", "b2", "w3", "b3"):
        err = np.abs(g[k] - rg[k]).max() / max(np.abs(rg[k]).max(), 1e-12)
        assert err < 2e-4, (k, err)
    assert np.allclose(tr.forward(x), yref, rtol=1e-4, atol=1e-5)
    tr.close()


@pytest.mark.gpu
def test_training_reduces_loss():
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, size=(20000, 6)).astype(np.float32)
    y = (np.tanh(x[:, 0] * 2 + x[:, 1]) * 0.5 + 0.5).astype(np.float32)
    model, losses = seed.train(x, y, epochs=12, batch=1024, lr=3e-3)
    assert losses[-1] < 0.1 * losses[0]


def _run(case, tmp, model=None, ptmu_mode=None):
    import os
    os.makedirs(str(tmp), exist_ok=True)
    d = case.write(str(tmp))
    inp = api.Input(d, os.path.join(str(tmp), "libEOS"))
    ctx = api.Context(inp.case)
    ctx.upload(inp.fill())
    if model is not None:
        model.install(ctx)
    if ptmu_mode is not None:
        ctx.set_ptmu_seed(ptmu_mode)
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
    # what training buys: an untrained network (random weights, same normalisation) asked about the same
    # hard cells needs more Newton evaluations than the trained one (the trained seed lands about as
    # close to p* as the plain first iterate, so against the plain start it gains nothing measurable)
    tr = seed.Trainer(x.shape[1], seed=7)
    untrained = tr.model()
    um = untrained.mlp
    for i in range(x.shape[1]):
        um.in_shift[i], um.in_scale[i] = model.mlp.in_shift[i], model.mlp.in_scale[i]
    um.out_shift, um.out_scale = model.mlp.out_shift, model.mlp.out_scale
    _, st2 = _run(test_case, tmp_path / "untrained", untrained)
    tr.close()
    assert st1.seeded > 0 and st2.seeded > 0
    assert st1.newton_evals < st2.newton_evals, (st1.newton_evals, st2.newton_evals)


@pytest.mark.gpu
def test_ptmu_seed_fewer_saturation_iterations_same_residual(tmp_path):
    """The (p*, T) network of the p-T-mu saturation solve, trained on expansion tubes unlike the test case.

    Its T starts the T_sat(p) Newton solves (the reference starts every one cold at 0.1 B / C, far from
    T_sat), so they must take far fewer iterations, while the saturation Newton on p* keeps the plain
    start (sum_k alpha_k p_k, already within one or two iterations) and its iteration count.  An untrained
    network asked the same must do worse than the trained one, and starting p* from the network as well
    (ECG_PTMU_SEED_P_T) is the measured alternative: it converges to the same residual with more p*
    iterations.  Fields stay within the spread the solves' own 1e-10 residuals allow."""
    train_cases = [cases.expansion_tube_2d(n=48, iterations=10, velocity=v, alpha_vap=a, name=f"trainPTMu{i}")
                   for i, (v, a) in enumerate([(300.0, 5e-3), (700.0, 2e-2), (400.0, 1.5e-2)])]
    x, y = seed.record(train_cases, steps=10, max_pairs=200000, min_evals=1)
    assert x.shape[1] == 8 and y.shape[1] == 2 and len(y) > 10000
    assert np.all(np.isfinite(x)) and np.all(np.isfinite(y))
    model, losses = seed.train(x, y, epochs=15, batch=2048, lr=2e-3)
    assert losses[-1] < 0.05 * losses[0]
    test_case = cases.expansion_tube_2d(n=48, iterations=10, name="testPTMu")
    plain, st0 = _run(test_case, tmp_path / "plain")
    seeded, st1 = _run(test_case, tmp_path / "seeded", model)
    assert st0.ptmu_seeded == 0 and st1.ptmu_seeded > 0.9 * st1.ptmu_solves
    assert st1.ptmu_errors == 0 and st1.nonfinite_cells == 0 and st1.newton_fallback == st0.newton_fallback
    # the pure-phase tests decide as the plain iteration does; states that differ at the solves' residual
    # level may flip a borderline cell
    assert abs(st1.ptmu_solves - st0.ptmu_solves) <= 0.01 * st0.ptmu_solves
    assert st1.ptmu_tsat_iters < 0.5 * st0.ptmu_tsat_iters, (st1.ptmu_tsat_iters, st0.ptmu_tsat_iters)
    assert abs(st1.ptmu_outer_iters - st0.ptmu_outer_iters) <= 0.02 * st0.ptmu_outer_iters
    for name in ("alpha", "rho", "E"):
        assert rel_l1(seeded[name], plain[name]) < 1e-8, name
    assert rel_l1(seeded["p"], plain["p"]) < 1e-6
    # what training buys: random weights with the same normalisation give worse T starts
    tr = seed.Trainer(8, seed=7, n_out=2)
    untrained = tr.model()
    um = untrained.mlp
    for i in range(8):
        um.in_shift[i], um.in_scale[i] = model.mlp.in_shift[i], model.mlp.in_scale[i]
    um.out_shift, um.out_scale = model.mlp.out_shift, model.mlp.out_scale
    um.out_shift_1, um.out_scale_1 = model.mlp.out_shift_1, model.mlp.out_scale_1
    _, st2 = _run(test_case, tmp_path / "untrained", untrained)
    tr.close()
    assert st2.ptmu_errors == 0
    assert st1.ptmu_tsat_iters < st2.ptmu_tsat_iters, (st1.ptmu_tsat_iters, st2.ptmu_tsat_iters)
    # p* from the network too: same residual, not fewer p* iterations than the plain start
    both, st3 = _run(test_case, tmp_path / "both", model, ptmu_mode=api.PTMU_SEED_P_T)
    assert st3.ptmu_errors == 0 and st3.ptmu_seeded > 0.9 * st3.ptmu_solves
    assert st3.ptmu_outer_iters >= st0.ptmu_outer_iters
    for name in ("alpha", "rho", "E"):
        assert rel_l1(both[name], plain[name]) < 1e-8, name
