"""ecg_step_noalloc: a time step on caller-owned device buffers that allocates no device memory.

Some callers cannot let the library call cudaMalloc: codes that hand out all device memory from
their own pool or allocator, and codes that must not allocate inside their time loop (an allocation
can synchronise the device and stall their other streams).  The no-allocation entry point keeps its
scratch in a fixed-size array of the library instead.  These tests drive it through the C ABI on
device buffers the test owns (torch tensors), two calls in a row, and check each result against
the context-based entry point (ecg_step) on the same input -- and once against the oracle -- within
the tolerance of the other parity tests.  They cover the Kapila model in 1D, 2D (first order and
MUSCL) and 3D with three phases near the scratch's cell maximum, and the Euler model.  This file is
collected last so that a run stopping at the first failure has already run every other test.
"""
import ctypes as C
import os

import numpy as np
import pytest

from ecogen_b200 import api, cases
from tests.conftest import rel_l1

TOL = 1e-12
ERR_INVALID, ERR_UNSUPPORTED, ERR_TOO_LARGE = 1, 2, 7


def _dim(rec):
    return sum(1 for a in range(3) if rec.ncells[a] != 1)


def _device_state(fields, rec):
    """ABI host fields -> the device layout (what ecg_upload_prim stores)."""
    import torch
    dim = _dim(rec)
    pre = 2 if rec.model == api.MODEL_EULER else 2 * rec.nphases + 1  # fields up to and including p
    sel = list(range(pre)) + [pre + d for d in range(dim)] + [pre + 3]
    return torch.tensor(np.stack([fields[i] for i in sel]), dtype=torch.float64, device="cuda").contiguous()


def _as_dict(out, rec):
    """Device-layout state -> the fields ecg_download_prim returns (Kapila p = sum_k alpha_k p_k)."""
    dim = _dim(rec)
    if rec.model == api.MODEL_EULER:
        return {"rho": out[0:1], "p": out[1], "u": out[2:2 + dim], "E": out[2 + dim]}
    k = rec.nphases
    got = {"alpha": out[:k], "rho": out[k:2 * k], "u": out[2 * k + 1:2 * k + 1 + dim], "E": out[2 * k + 1 + dim]}
    pk = []
    for j in range(k):  # phase pressures: the stored mixture-EOS pressure clamped by each phase's EOS
        q = rec.eos[j]
        if q.type == 0:
            pk.append(np.maximum(out[2 * k], 1e-8))
        else:
            floor = -(1 - 1e-15) * q.pinf + 1e-15
            pk.append(np.where(out[2 * k] <= floor, floor, out[2 * k]))
    got["p"] = sum(out[j] * pk[j] for j in range(k))
    return got


def _noalloc(rec, s_in, s_out, dt):
    dt_next = C.c_double()
    st = api.StepStats()
    api.check(api.lib().ecg_step_noalloc(C.byref(rec), C.c_void_p(s_in.data_ptr()), C.c_void_p(s_out.data_ptr()),
                                         dt, C.byref(dt_next), C.byref(st), None), "ecg_step_noalloc")
    return dt_next.value, st


NOALLOC_CASES = {
    "kapila2d_muscl": lambda: cases.shock_bubble_2d(n=40, iterations=2, limiter="vanleer"),
    "kapila2d_o1": lambda: cases.shock_bubble_2d(n=40, iterations=2, limiter=None),
    "kapila1d_tube": lambda: cases.shock_tube_1d(ncells=1000, iterations=2, total_time=None),
    "euler1d_muscl": lambda: cases.euler_shock_tube(ncells=400, iterations=2, order="vanleer"),
    # 40^3 = 64,000 cells: three phases and MUSCL fill every half-step field of the scratch close to
    # its 65,536-cell maximum
    "kapila3d_3phase_muscl": lambda: cases.cavity_collapse_3d(n=40, iterations=2),
}


@pytest.mark.gpu
@pytest.mark.parametrize("key", list(NOALLOC_CASES))
def test_noalloc_step_matches_context_step(key, tmp_path):
    case = NOALLOC_CASES[key]()
    d = case.write(str(tmp_path))
    inp = api.Input(d, os.path.join(str(tmp_path), "libEOS"))
    rec = inp.case
    fields = inp.fill()
    dim = _dim(rec)

    ctx = api.Context(rec)
    ctx.upload(fields)

    import torch
    s_in = _device_state(fields, rec)
    s_out = torch.empty_like(s_in)
    dt = 1e-15
    for call in range(2):
        dt_next, st = _noalloc(rec, s_in, s_out, dt)
        ref_st = ctx.step(1)
        ref = ctx.download_dict()
        assert dt_next == pytest.approx(ctx.dt.value, rel=TOL)
        got = _as_dict(s_out.cpu().numpy(), rec)
        for name in got:
            want = ref[name][:dim] if name == "u" else ref[name]
            assert rel_l1(got[name], want) <= TOL, (key, call, name)
        assert st.relax_calls == ref_st.relax_calls and st.newton_evals == ref_st.newton_evals
        assert st.nonfinite_cells == 0
        s_in, s_out = s_out, s_in
        dt = dt_next
    ctx.close()


@pytest.mark.gpu
def test_noalloc_matches_oracle_and_allocates_nothing(tmp_path):
    """Two calls against the oracle's two steps; the device's free memory does not change across them."""
    import torch

    from oracle import oracle
    case = cases.shock_bubble_2d(n=48, iterations=2)
    d = case.write(str(tmp_path))
    inp = api.Input(d, os.path.join(str(tmp_path), "libEOS"))
    rec = inp.case
    fields = inp.fill()
    s0 = _device_state(fields, rec)
    a, b = torch.empty_like(s0), torch.empty_like(s0)
    _noalloc(rec, s0, a, 1e-15)  # first call on this device: set-up (module load, scratch address)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    dt, _ = _noalloc(rec, s0, a, 1e-15)
    _noalloc(rec, a, b, dt)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    sim = oracle.Sim(case)
    sim.step(2)
    o = sim.fields()
    got = _as_dict(b.cpu().numpy(), rec)
    for name in ("alpha", "rho", "p", "E"):
        assert rel_l1(got[name], o[name]) <= TOL, name
    assert rel_l1(got["u"], o["u"][:2]) <= TOL


@pytest.mark.gpu
def test_noalloc_refuses_cases_above_its_maximum():
    import torch
    case = cases.shock_bubble_2d(n=300, iterations=1)  # 90000 cells > 65536
    rec = api.case_from_spec(case)
    buf = torch.zeros(8, 16, dtype=torch.float64, device="cuda")
    st = api.lib().ecg_step_noalloc(C.byref(rec), C.c_void_p(buf.data_ptr()), C.c_void_p(buf[4:].data_ptr()), 1e-15,
                                    None, None, None)
    assert st == ERR_TOO_LARGE


# ---- argument checks: they return before any CUDA call, so they run without a GPU too

def _status(rec, a, b):
    return api.lib().ecg_step_noalloc(C.byref(rec), C.c_void_p(a), C.c_void_p(b), 1e-15, None, None, None)


def test_noalloc_rejects_what_ecg_create_rejects():
    base = api.case_from_spec(cases.shock_bubble_2d(n=16, iterations=1))
    n = 16 * 16
    a, b = 1 << 20, (1 << 20) + 8 * 8 * n * 4  # disjoint (fake) device addresses; never dereferenced
    bad = api.Case.from_buffer_copy(base)
    bad.ncells[0], bad.ncells[1] = 1, 16  # a 1 x N mesh (x must have more than one cell)
    assert _status(bad, a, b) == ERR_INVALID
    bad = api.Case.from_buffer_copy(base)
    bad.limiter[0] = 42
    assert _status(bad, a, b) == ERR_INVALID
    bad = api.Case.from_buffer_copy(base)
    bad.nphases = 4
    assert _status(bad, a, b) in (ERR_INVALID, ERR_UNSUPPORTED)
    bad = api.Case.from_buffer_copy(base)
    bad.ptmu, bad.ptmu_liquid, bad.ptmu_vapor = 1, 0, 7  # phase index out of range
    assert _status(bad, a, b) == ERR_INVALID


def test_noalloc_rejects_ptueq_and_overlapping_buffers():
    ptueq = api.case_from_spec(cases.ptueq_bubble_2d(n=16, iterations=1))
    assert _status(ptueq, 1 << 20, 1 << 24) == ERR_UNSUPPORTED
    base = api.case_from_spec(cases.shock_bubble_2d(n=16, iterations=1))
    a = 1 << 20
    assert _status(base, a, a) == ERR_INVALID
    assert _status(base, a, a + 8 * 16 * 16) == ERR_INVALID  # output starts one field into the input
    assert _status(base, a + 8 * 16 * 16 * 3, a) == ERR_INVALID
