"""p-T-mu warm start without a network: each cell's T_sat(p) solves start from its previous solve.

Mixture::computeTsat (src/Models/Mixture.cpp:59-100) starts every solve cold at 0.1 B / C.  With the warm
start on, the context keeps the T_sat of each cell's last saturation solve and the next solve starts
there; the saturation Newton on p* keeps the reference's start.  Both Newton loops still stop at
|f| <= 1e-10, so the fields agree with the plain solve to that residual level; with the warm start off
the step is the reference's, bit for bit.
"""
import os

import numpy as np
import pytest

from ecogen_b200 import api, cases
from tests.conftest import rel_l1


def _run(case, tmp, warm, toggle=False):
    os.makedirs(str(tmp), exist_ok=True)
    d = case.write(str(tmp))
    inp = api.Input(d, os.path.join(str(tmp), "libEOS"))
    ctx = api.Context(inp.case)
    ctx.upload(inp.fill())
    if toggle:  # on, then off again before any step: the reference's starts
        ctx.set_ptmu_warm_start(True)
        ctx.set_ptmu_warm_start(False)
    if warm:
        ctx.set_ptmu_warm_start(True)
    st = ctx.step(case.iterations)
    out = ctx.download_dict()
    ctx.close()
    return out, st


@pytest.mark.gpu
def test_warm_start_fewer_tsat_iterations_same_residual(tmp_path):
    case = cases.expansion_tube_2d(n=64, iterations=20, name="warmPTMu")
    plain, st0 = _run(case, tmp_path / "plain", False)
    warm, st1 = _run(case, tmp_path / "warm", True)
    assert st0.ptmu_seeded == 0 and st1.ptmu_seeded > 0
    assert st1.ptmu_errors == 0 and st1.nonfinite_cells == 0
    assert abs(st1.ptmu_solves - st0.ptmu_solves) <= 0.01 * st0.ptmu_solves
    assert st1.ptmu_tsat_iters < 0.4 * st0.ptmu_tsat_iters, (st1.ptmu_tsat_iters, st0.ptmu_tsat_iters)
    # the p* Newton keeps its start; cells whose plain start already meets |f| <= 1e-10 to within the T_sat
    # solves' own residual may stop one iteration earlier or later, so the count moves a little (measured:
    # fewer), never up by more than that
    assert st1.ptmu_outer_iters <= 1.02 * st0.ptmu_outer_iters
    for name in ("alpha", "rho", "E"):
        assert rel_l1(warm[name], plain[name]) < 1e-8, name
    assert rel_l1(warm["p"], plain["p"]) < 1e-6


@pytest.mark.gpu
def test_warm_start_off_is_the_reference_path(tmp_path):
    case = cases.expansion_tube_2d(n=40, iterations=8, name="warmOff")
    plain, st0 = _run(case, tmp_path / "plain", False)
    again, st1 = _run(case, tmp_path / "toggled", False, toggle=True)
    for name in ("alpha", "rho", "p", "u", "E"):
        assert np.array_equal(plain[name], again[name]), name
    assert st0.ptmu_tsat_iters == st1.ptmu_tsat_iters and st1.ptmu_seeded == 0


@pytest.mark.gpu
def test_warm_start_needs_ptmu(tmp_path):
    case = cases.shock_bubble_2d(n=16, iterations=2, name="warmNoPTMu")
    d = case.write(str(tmp_path))
    ctx = api.Context(api.Input(d, os.path.join(str(tmp_path), "libEOS")).case)
    with pytest.raises(api.EcgError):
        ctx.set_ptmu_warm_start(True)
    ctx.set_ptmu_warm_start(False)
    ctx.close()
