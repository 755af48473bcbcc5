"""C ABI: the library loads without a GPU, exports every declared symbol, reads case inputs."""
import os
import re

import numpy as np
import pytest

from ecogen_b200 import api, cases
from oracle import oracle
from tests.conftest import ROOT, display, load_golden


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "ecogen_b200.h")).read()
    return sorted(set(re.findall(r"\b(ecg_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = api.lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    assert len(declared_symbols()) >= 30


@pytest.mark.parametrize("key", ["tube1d_o1_full", "bubble2d_o2", "cavity3d_o2", "expansion2d_ptmu", "euler1d_o1"])
def test_xml_input_fill_matches_reference_initial_state(key, golden_cases, tmp_path):
    _, g = load_golden(key)
    case = golden_cases[key]
    d = case.write(str(tmp_path))
    inp = api.Input(d, os.path.join(str(tmp_path), "libEOS"))
    f = inp.fill()
    k = case.nphases
    if case.model.upper() == "EULER":
        assert np.array_equal(f[0], g["init_rho"][0])
        assert np.array_equal(f[1], g["init_p"])
    else:
        assert np.array_equal(display(np.stack(f[:k]), "alpha"), g["init_alpha"])
        assert np.array_equal(np.stack(f[k:2 * k]), g["init_rho"])
        # E is the total energy of Cell::completeFulfillState
        assert np.array_equal(f[2 * k + 4], g["init_E"])
    sim = oracle.Sim(case)
    assert np.array_equal(f[-1], sim.fields()["E"])


def test_case_record_from_xml(tmp_path):
    case = cases.shock_bubble_2d(n=16, iterations=5)
    case.interface_limiter = "superbee"
    d = case.write(str(tmp_path))
    inp = api.Input(d, os.path.join(str(tmp_path), "libEOS"))
    c = inp.case
    assert (c.model, c.nphases, c.order) == (api.MODEL_KAPILA, 2, 2)
    assert list(c.limiter) == [2, 4, 2, 4]
    assert list(c.ncells) == [16, 16, 1] and c.cfl == 0.6
    assert c.time_iterations == 1 and c.max_iterations == 5
    assert c.eos[0].type == 1 and c.eos[0].pinf == 6e8 and c.eos[1].type == 0
    assert inp.run_name == "shockBubble2D"


def _expect(status, fn):
    with pytest.raises(api.EcgError) as ei:
        fn()
    assert ei.value.status == status


def test_malformed_inputs_are_input_errors(tmp_path):
    # reference non-regression error cases: a missing element and a missing attribute
    case = cases.shock_tube_1d(ncells=50, iterations=3)
    d = case.write(str(tmp_path))
    eosdir = os.path.join(str(tmp_path), "libEOS")
    main = open(os.path.join(d, "main.xml")).read()
    open(os.path.join(d, "main.xml"), "w").write(main.replace("<run>shockTube1D</run>", ""))
    _expect(4, lambda: api.Input(d, eosdir))
    open(os.path.join(d, "main.xml"), "w").write(main)
    mesh = open(os.path.join(d, "mesh.xml")).read()
    open(os.path.join(d, "mesh.xml"), "w").write(mesh.replace(' y="1"', ""))
    _expect(4, lambda: api.Input(d, eosdir))
    open(os.path.join(d, "mesh.xml"), "w").write(mesh.replace("<numberCells", "<numberCells").replace("</mesh>", ""))
    _expect(4, lambda: api.Input(d, eosdir))  # unterminated root


def test_unsupported_inputs_are_refused(tmp_path):
    case = cases.shock_tube_1d(ncells=50, iterations=3)
    d = case.write(str(tmp_path))
    eosdir = os.path.join(str(tmp_path), "libEOS")
    mesh = open(os.path.join(d, "mesh.xml")).read()
    open(os.path.join(d, "mesh.xml"), "w").write(
        mesh.replace("</cartesianMesh>", '<AMR lvlMax="1" criteriaVar="0.1" varRho="true" varP="false" '
                                          'varU="false" varAlpha="false" xiSplit="0.1" xiJoin="0.1"/></cartesianMesh>'))
    _expect(2, lambda: api.Input(d, eosdir))
    open(os.path.join(d, "mesh.xml"), "w").write(mesh)
    ic = open(os.path.join(d, "initialConditions.xml")).read()
    open(os.path.join(d, "initialConditions.xml"), "w").write(ic.replace('type="nonReflecting" number="1"',
                                                                          'type="outletPressure" number="1"'))
    _expect(2, lambda: api.Input(d, eosdir))


def test_boundary_sides_read_in_order(tmp_path):
    """The i-th boundCond is side i (Xm, Xp, Ym, Yp, ...); wall and symmetry are the same side type."""
    case = cases.shock_bubble_2d(n=8, iterations=2)
    case.boundaries = ["wall", "nonReflecting", "symmetry", "wall"]
    d = case.write(str(tmp_path))
    inp = api.Input(d, os.path.join(str(tmp_path), "libEOS"))
    assert list(inp.case.bc) == [1, 0, 1, 1, 0, 0]
    assert list(api.case_from_spec(case).bc) == [1, 0, 1, 1, 0, 0]


def test_create_rejects_bad_cases_without_gpu_work():
    c = api.Case()
    c.model, c.nphases, c.order = 0, 4, 1
    c.ncells[0], c.ncells[1], c.ncells[2] = 10, 1, 1
    c.length[0] = c.length[1] = c.length[2] = 1.0
    h = api.C.c_void_p()
    st = api.lib().ecg_create(api.C.byref(c), api.C.byref(h))
    assert st == 2 and not h.value
    c.nphases, c.ncells[0] = 2, 1
    assert api.lib().ecg_create(api.C.byref(c), api.C.byref(h)) == 1


def test_transports_read_and_filled(tmp_path):
    """numberTransports, <transport name> of model.xml and the per-state values (0 when absent)."""
    case = cases.shock_tube_1d(ncells=20, iterations=2)
    case.transports = ["color", "marker"]
    case.states[0].transports = {"color": 1.0, "marker": 0.25}
    case.states[1].transports = {"marker": 2.0, "unknown": 7.0}
    d = case.write(str(tmp_path))
    inp = api.Input(d, os.path.join(str(tmp_path), "libEOS"))
    assert inp.case.ntransports == 2
    f = inp.fill()
    assert len(f) == 2 * 2 + 5 + 2
    ref = oracle.initial_fields(case)["tr"]
    assert np.array_equal(np.stack(f[-2:]), ref)
    assert set(np.unique(f[-2])) <= {0.0, 1.0} and set(np.unique(f[-1])) <= {0.25, 2.0}


def test_stretched_mesh_read_and_filled(tmp_path):
    """mesh.xml meshStretching: zones per axis (Input::inputMesh :460-520), the axis' cells their sum,
    and the initial fill at the stretched cell centres (the oracle's restatement of
    MeshCartesian::meshStretching, pinned on the reference's own fixtures)."""
    from tests.golden.make_golden import stretched_cases
    for key, case in stretched_cases().items():
        d = case.write(str(tmp_path / key))
        inp = api.Input(d, os.path.join(str(tmp_path / key), "libEOS"))
        assert list(inp.case.ncells) == [int(v) for v in case.cells], key
        for a, ax in enumerate("xyz"):
            zones = (case.stretch or {}).get(ax) or []
            assert inp.case.nstretch[a] == len(zones), key
            for z, (s0, s1, f, m) in enumerate(zones):
                zr = inp.case.stretch[a][z]
                assert (zr.start, zr.end, zr.factor, zr.ncells) == (s0, s1, f, m)
        f = inp.fill()
        ini = oracle.initial_fields(case)
        if case.model.upper() == "EULER":
            assert np.array_equal(f[0], np.ravel(ini["rho"])), key
        else:
            assert np.array_equal(np.stack(f[:case.nphases]), ini["alpha"]), key
            assert np.array_equal(np.stack(f[case.nphases:2 * case.nphases]), ini["rho"]), key


def test_stretch_zones_are_checked_without_gpu_work():
    """Zones that do not start at 0, leave gaps, miss the axis length or the axis' cells are refused
    (stretchZone::verifyStretching src/Meshes/stretchZone.cpp:74-93) before any device work."""
    base = api.case_from_spec(cases.shock_tube_1d(ncells=100, iterations=1, order="vanleer"))
    h = api.C.c_void_p()

    def zones(*zs):
        c = api.Case.from_buffer_copy(base)
        c.nstretch[0] = len(zs)
        for i, z in enumerate(zs):
            c.stretch[0][i] = api.StretchZone(*z)
        return api.lib().ecg_create(api.C.byref(c), api.C.byref(h))

    assert zones((0.1, 1.0, 1.0, 100)) == 1               # does not start at 0
    assert zones((0.0, 0.5, 1.0, 50), (0.6, 1.0, 1.0, 50)) == 1  # gap
    assert zones((0.0, 0.9, 1.0, 100)) == 1               # does not reach the length
    assert zones((0.0, 1.0, 1.05, 90)) == 1               # 90 cells on a 100-cell axis
    assert not h.value


def test_context_settings_refuse_a_null_context():
    """The GPU-side settings check their context before any device work (no GPU needed)."""
    L = api.lib()
    assert L.ecg_set_step_form(None, api.FORM_SPLIT) == 1
    assert L.ecg_set_face_staging(None, api.STAGING_TMA) == 1
    assert L.ecg_set_ptmu_seed(None, api.PTMU_SEED_T) == 1
    assert L.ecg_set_ptmu_warm_start(None, 1) == 1
    assert L.ecg_set_newton_cap_mode(None, api.CAP_ACCEPT) == 1
    assert L.ecg_set_newton_cap(None, 3) == 1
    assert L.ecg_step_form(None) == api.FORM_FUSED
    assert L.ecg_face_staging(None) == api.STAGING_PLAIN
