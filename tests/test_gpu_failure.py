"""Failure detection on the GPU path without a GPU fault.

The reference's step has no runtime physics error: a pressure-relaxation Newton that does not
converge within its cap falls back to the interface pressure (src/Relaxations/RelaxationPInfinite.cpp,
the `iteration > 100` branch) and non-finite values propagate.  The device path reproduces that
and reports both through ecg_step_stats, so a caller can detect them after every step:
 * newton_fallback counts relaxations that hit the cap,
 * nonfinite_cells counts cells whose updated state is not finite.
"""
import numpy as np
import pytest

from ecogen_b200 import api, cases

from tests.helpers import write_case

pytestmark = pytest.mark.gpu


def _ctx(case, tmp):
    d, eosdir = write_case(case, tmp)
    inp = api.Input(d, eosdir)
    ctx = api.Context(inp.case)
    fields = inp.fill()
    return ctx, fields


def test_newton_cap_forces_counted_fallback(tmp_path):
    case = cases.shock_bubble_2d(n=48, iterations=6)
    ctx, fields = _ctx(case, tmp_path / "a")
    ctx.upload(fields)
    st = ctx.step(6)
    assert st.newton_fallback == 0 and st.relax_calls > 0
    ctx.close()

    ctx, fields = _ctx(case, tmp_path / "b")
    ctx.set_newton_cap(1)
    ctx.upload(fields)
    st = ctx.step(6)
    assert st.newton_fallback > 0
    assert st.newton_max <= 1
    assert st.nonfinite_cells == 0
    ctx.close()


def test_newton_cap_is_validated(tmp_path):
    case = cases.shock_tube_1d(ncells=40, iterations=2)
    ctx, _ = _ctx(case, tmp_path)
    with pytest.raises(api.EcgError):
        ctx.set_newton_cap(0)
    ctx.close()


def test_nonfinite_cells_are_counted_not_fatal(tmp_path):
    case = cases.shock_tube_1d(ncells=64, iterations=3)
    ctx, fields = _ctx(case, tmp_path)
    k = 2  # two phases: alpha0, alpha1, rho0, rho1, p, ...
    fields[2 * k][10] = np.nan  # mixture pressure of cell 10
    ctx.upload(fields)
    st = ctx.step(1)
    assert st.nonfinite_cells > 0
    out = ctx.download_dict()
    # cells away from the planted value (more than two stencil widths) are untouched by it
    assert np.all(np.isfinite(out["p"][30:]))
    ctx.close()
