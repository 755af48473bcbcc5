"""Temperature-pressure-velocity equilibrium model (ECOGEN's PTUEq, src/Models/PTUEq).

CPU: the C ABI reads PTUEq cases (mixture pressure and temperature, phase volume fractions), fills the
initial state as the reference does (phase densities computeDensity(p, T), total energy of the mixture),
and refuses what the reference cannot run: NASG phases (MixPTUEq::computePressure), passive transports
(no transport Riemann solver, src/Models/Model.h:185), MUSCL symmetry sides (Phase::setU on PhasePTUEq).
GPU: the step kernels match the reference fixtures and the oracle within 1e-12 relative L1 per field,
and the ecogen-b200 driver writes the reference's PTUEq arrays.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from ecogen_b200 import api, cases
from oracle import oracle, refrun
from tests.conftest import load_golden, rel_l1
from tests.helpers import ROOT, gpu_run, write_case

TOL = 1e-12
KEYS = ["ptueq_tube_o2", "ptueq_tube_o1", "ptueq_tube_wall_o1", "ptueq_bubble2d_o2", "ptueq_bubble2d_o1_sym",
        "ptueq_bubble2d_thinc", "ptueq_bubble3d_o2"]


def _input(case, tmp):
    d, eosdir = write_case(case, tmp)
    return api.Input(d, eosdir)


def test_ptueq_layout_and_fill_match_oracle(tmp_path):
    case = cases.ptueq_bubble_2d(n=24, iterations=10)
    inp = _input(case, tmp_path)
    assert inp.case.model == api.MODEL_PTUEQ and inp.case.nphases == 2
    f = inp.fill()
    assert len(f) == api.nfields(inp.case) == 10
    _, g = load_golden("ptueq_bubble2d_o2")
    assert np.array_equal(np.stack(f[0:2]), g["init_alpha"])
    assert np.array_equal(np.stack(f[2:4]), g["init_rho"])
    assert np.array_equal(f[4], g["init_p"])
    assert np.array_equal(f[9], g["init_Tm"])
    o = oracle.Sim(case).fields()
    assert np.array_equal(f[8], o["E"])  # Cell::completeFulfillState (MixPTUEq::computeTotalEnergy)


def test_ptueq_restart_fill_recomputes_densities_and_energy(tmp_path):
    case = cases.ptueq_bubble_2d(n=12, iterations=2)
    inp = _input(case, tmp_path)
    f = inp.fill()
    ref = [a.copy() for a in f]
    f[2][:] = 0.0  # densities and energy are rebuilt from (alpha_k, p, T, u)
    f[3][:] = -1.0
    f[8][:] = 0.0
    api.check(api.lib().ecg_restart_fill(C.byref(inp.case), api._field_ptrs(f), case.ncells), "ecg_restart_fill")
    for i in (2, 3, 8):
        assert np.array_equal(f[i], ref[i])


@pytest.mark.parametrize("what", ["nasg", "transport", "relaxation"])
def test_ptueq_input_refusals(what, tmp_path):
    case = cases.ptueq_shock_tube_1d(ncells=20, iterations=2)
    if what == "nasg":
        case.eos = [cases.AIR_IG, cases.WATER_NASG]
    elif what == "transport":
        case.transports = ["color"]
    else:
        case.pt_relaxation = True
    d, eosdir = write_case(case, tmp_path)
    h = C.c_void_p()
    st = api.lib().ecg_input_read(d.encode(), eosdir.encode(), C.byref(h))
    assert st == 2  # ECG_ERR_UNSUPPORTED


def test_ptueq_muscl_symmetry_side_is_refused(tmp_path):
    case = cases.ptueq_shock_tube_1d(ncells=20, iterations=2, boundaries=["wall", "nonReflecting"])
    inp = _input(case, tmp_path)
    h = C.c_void_p()
    assert api.lib().ecg_create(C.byref(inp.case), C.byref(h)) == 2  # refused before any device work


def test_ptueq_oracle_refuses_what_the_reference_cannot_run():
    case = cases.ptueq_shock_tube_1d(ncells=20, iterations=2, boundaries=["wall", "nonReflecting"])
    with pytest.raises(ValueError):
        oracle.Sim(case)
    case = cases.ptueq_shock_tube_1d(ncells=20, iterations=2, transports=["color"])
    with pytest.raises(ValueError):
        oracle.Sim(case)


def _compare(key, out, g):
    for name in ("alpha", "rho", "p", "u"):
        err = rel_l1(out[name], g["final_" + name])
        assert err <= TOL, f"{key}: {name} rel L1 {err:.3e}"
    err = rel_l1(out["Tm"], g["final_Tm"])
    assert err <= TOL, f"{key}: temperature rel L1 {err:.3e}"


@pytest.mark.gpu
@pytest.mark.parametrize("key", KEYS)
def test_gpu_ptueq_matches_reference_golden(key, golden_cases, tmp_path):
    meta, g = load_golden(key)
    out = gpu_run(golden_cases[key], tmp_path)
    assert out["iteration"] == meta["iterations_done"]
    _compare(key, out, g)


def _oracle_compare(case, steps, tmp_path):
    out = gpu_run(case, tmp_path)
    sim = oracle.Sim(case)
    sim.step(steps)
    o = sim.fields()
    for name in ("alpha", "rho", "p", "u", "E"):
        assert rel_l1(out[name], o[name]) <= TOL, name
    assert rel_l1(out["Tm"], o["T"][0]) <= TOL
    assert out["dt"] == pytest.approx(sim.dt.value, rel=1e-12)
    assert out["t"] == pytest.approx(sim.t.value, rel=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("limiter,vf", [("vanleer", None), ("minmod", "THINC"), (None, None)])
def test_gpu_ptueq_matches_oracle_2d(limiter, vf, tmp_path):
    """Meshes of several tiles per axis (ragged in y), MUSCL with and without THINC, and first order."""
    case = cases.ptueq_bubble_2d(n=70, ny=45, iterations=25, limiter=limiter, name="ptueqBubble70")
    case.interface_vf_limiter = vf
    if limiter is None:
        case.boundaries = ["wall", "nonReflecting", "symmetry", "symmetry"]
    _oracle_compare(case, 25, tmp_path)


@pytest.mark.gpu
@pytest.mark.parametrize("limiter", ["vanleer", None])
def test_gpu_ptueq_matches_oracle_3d_ragged(limiter, tmp_path):
    case = cases.ptueq_bubble_2d(n=13, ny=9, nz=7, iterations=4, limiter=limiter, name="ptueqBubble3D")
    if limiter is None:
        case.boundaries = ["symmetry", "nonReflecting", "wall", "symmetry", "nonReflecting", "wall"]
    _oracle_compare(case, 4, tmp_path)


@pytest.mark.gpu
@pytest.mark.parametrize("key", ["ptueq_tube_o2", "ptueq_bubble2d_o2"])
def test_driver_writes_ptueq_results(key, golden_cases, tmp_path):
    """ecogen-b200 writes the reference's PTUEq arrays (phase Alpha, Density; mixture Density, Pressure,
    Temperature, Velocity_Mixture_norm; gradRho)."""
    meta, g = load_golden(key)
    case = golden_cases[key]
    d = case.write(str(tmp_path))
    cases.write_ecogen_list(str(tmp_path), [d])
    r = subprocess.run([os.path.join(ROOT, "ecogen_b200", "ecogen-b200"), str(tmp_path) + "/"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    raw = refrun.read_vtr(refrun.result_files(str(tmp_path), case.name)[-1])
    got = refrun.reference_prim(raw, case.nphases)
    for name in ("alpha", "rho", "p", "u", "rho_mix"):
        assert rel_l1(got[name], g["final_" + name]) <= TOL, name
    assert rel_l1(got["Tm"], g["final_Tm"]) <= TOL
    assert rel_l1(raw["gradRho"], g["final_gradRho"]) <= 1e-9
