"""ecg_step_noalloc: a time step on caller-owned device buffers that allocates no device memory.

Callers such as codes that hand out all device memory from their own pool, or that must not
allocate inside their time loop, cannot let the library call cudaMalloc.  This test drives the
no-allocation entry point through the C ABI on device buffers owned by the test (torch tensors),
twice in a row, and checks each result against the context-based entry point (ecg_step) on the
same input, within the tolerance of the other parity tests.  This file is collected last so that a
run stopping at the first failure has already run every other test.
"""
import ctypes as C
import os

import numpy as np
import pytest

from ecogen_b200 import api, cases
from tests.conftest import rel_l1

TOL = 1e-12


def _device_state(fields, case_rec, dim):
    """ABI host fields -> the device layout (what ecg_upload_prim stores)."""
    import torch
    k = case_rec.nphases
    sel = list(range(2 * k + 1)) + [2 * k + 1 + d for d in range(dim)] + [2 * k + 4]
    return torch.tensor(np.stack([fields[i] for i in sel]), dtype=torch.float64, device="cuda").contiguous()


@pytest.mark.gpu
@pytest.mark.parametrize("order", ["vanleer", None])
def test_noalloc_step_matches_context_step(order, tmp_path):
    import torch
    case = cases.shock_bubble_2d(n=40, iterations=2, limiter=order)
    d = case.write(str(tmp_path))
    inp = api.Input(d, os.path.join(str(tmp_path), "libEOS"))
    rec = inp.case
    fields = inp.fill()
    k, n, dim = rec.nphases, inp.ncells, 2

    ctx = api.Context(rec)
    ctx.upload(fields)

    s_in = _device_state(fields, rec, dim)
    s_out = torch.empty_like(s_in)
    dt = 1e-15
    for call in range(2):
        dt_next = C.c_double()
        st = api.StepStats()
        api.check(api.lib().ecg_step_noalloc(C.byref(rec), C.c_void_p(s_in.data_ptr()), C.c_void_p(s_out.data_ptr()),
                                             dt, C.byref(dt_next), C.byref(st), None), "ecg_step_noalloc")
        ref_st = ctx.step(1)
        ref = ctx.download_dict()
        assert dt_next.value == pytest.approx(ctx.dt.value, rel=TOL)
        out = s_out.cpu().numpy()
        got = {"alpha": out[:k], "rho": out[k:2 * k], "u": out[2 * k + 1:2 * k + 1 + dim], "E": out[2 * k + 1 + dim]}
        # the stored pressure is the mixture-EOS pressure; the reference writes sum_k alpha_k p_k
        pinf = [rec.eos[j].pinf for j in range(k)]
        pk = [np.where(out[2 * k] <= -(1 - 1e-15) * pinf[j] + 1e-15, -(1 - 1e-15) * pinf[j] + 1e-15, out[2 * k])
              if rec.eos[j].type != 0 else np.maximum(out[2 * k], 1e-8) for j in range(k)]
        got["p"] = sum(out[j] * pk[j] for j in range(k))
        for name in ("alpha", "rho", "p", "E"):
            assert rel_l1(got[name], ref[name]) <= TOL, (call, name)
        assert rel_l1(got["u"], ref["u"][:dim]) <= TOL, call
        assert st.relax_calls == ref_st.relax_calls and st.newton_evals == ref_st.newton_evals
        s_in, s_out = s_out, s_in
        dt = dt_next.value
    ctx.close()


@pytest.mark.gpu
def test_noalloc_refuses_cases_above_its_maximum():
    import torch
    case = cases.shock_bubble_2d(n=300, iterations=1)  # 90000 cells > 65536
    rec = api.case_from_spec(case)
    buf = torch.zeros(8, 16, dtype=torch.float64, device="cuda")
    st = api.lib().ecg_step_noalloc(C.byref(rec), C.c_void_p(buf.data_ptr()), C.c_void_p(buf[4:].data_ptr()), 1e-15,
                                    None, None, None)
    assert st == 7  # ECG_ERR_TOO_LARGE
