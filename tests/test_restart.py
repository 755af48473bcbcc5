"""Restart from a result file (Run::restartSimulation src/Run.cpp:345).

Fixture tests/golden/restart2d.*: the reference's ASCII result file 2 (17 digits) and infoCalcul.out of a
30-iteration 2D run printed every 10 iterations, and the final file of the reference restarted from
file 2 (tests/golden/make_golden.py restart2d).

CPU: ecg_restart_fill completes the read fields as the reference does (phase corrections, total energy),
and the oracle advanced from them with the infoCalcul.out time and next dt ends bit for bit on the
reference's restarted run.  GPU: the ecogen-b200 driver restarts from the same files (written here in
the reference's layout) and ends within the parity tolerance.
"""
import ctypes as C
import json
import os
import subprocess

import numpy as np
import pytest

from ecogen_b200 import api, cases
from oracle import oracle, refrun
from tests.conftest import display, rel_l1
from tests.golden.make_golden import restart_case, restart_case_ptueq

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _fixture(key="restart2d"):
    with open(os.path.join(HERE, "golden", key + ".json")) as f:
        meta = json.load(f)
    g = dict(np.load(os.path.join(HERE, "golden", key + ".npz")))
    arrays = [g[f"in{i:02d}"] for i in range(len(meta["names"]))]
    return meta, g, arrays


def _abi_fields(case, arrays):
    """ABI layout (alpha_k, rho_k, p, u_x, u_y, u_z, E) from the arrays a restart reads, in file order:
    per phase alpha, density, temperature, mass fraction; mixture density, pressure, energy, velocity."""
    k = case.nphases
    f = [arrays[4 * i] for i in range(k)] + [arrays[4 * i + 1] for i in range(k)]
    f.append(arrays[4 * k + 1])
    vel = arrays[4 * k + 3].reshape(-1, 3)
    f += [vel[:, d] for d in range(3)]
    f.append(arrays[4 * k + 2])
    return [np.ascontiguousarray(x, dtype=np.float64) for x in f]


def _abi_fields_ptueq(case, arrays):
    """PTUEq ABI layout (alpha_k, rho_k, p, u_x, u_y, u_z, E, T) from a PTUEq result file in file order:
    per phase alpha, density; mixture density, pressure, temperature, velocity.  E is left to
    ecg_restart_fill."""
    f = [arrays[0], arrays[2], arrays[1], arrays[3], arrays[5]]
    vel = arrays[7].reshape(-1, 3)
    f += [vel[:, d] for d in range(3)]
    f += [np.zeros(case.ncells), arrays[6]]
    return [np.ascontiguousarray(x, dtype=np.float64) for x in f]


def _info(meta):
    parts = meta["info_lines"][meta["restart_file"] + 1].split()
    return int(parts[1]), float(parts[2]), float(parts[3])


def test_restart_fill_and_oracle_match_reference_restart():
    meta, g, arrays = _fixture()
    case = restart_case()
    f = _abi_fields(case, arrays)
    api.check(api.lib().ecg_restart_fill(C.byref(api.case_from_spec(case)), api._field_ptrs(f), case.ncells),
              "ecg_restart_fill")
    k = case.nphases
    sim = oracle.Sim(case, {"alpha": np.stack(f[:k]), "rho": np.stack(f[k:2 * k]), "p": f[2 * k],
                            "u": np.stack(f[2 * k + 1:2 * k + 4])})
    # the total energy ecg_restart_fill rebuilt is the oracle's (Cell::completeFulfillState)
    assert np.array_equal(sim.fields()["E"], f[2 * k + 4])
    it, t, dt = _info(meta)
    assert it == 20
    sim.t.value, sim.dt.value = t, dt
    sim.step(10)
    o = sim.fields()
    for name in ("alpha", "rho", "p", "u", "E"):
        ref = g["final_" + name]
        assert np.array_equal(display(o[name], name), ref), name


def test_restart_fill_rejects_bad_arguments():
    case = restart_case()
    c = api.case_from_spec(case)
    f = [np.zeros(case.ncells) for _ in range(api.nfields(c))]
    assert api.lib().ecg_restart_fill(C.byref(c), api._field_ptrs(f), case.ncells + 1) == 1
    assert api.lib().ecg_restart_fill(None, api._field_ptrs(f), case.ncells) == 1


def _write_reference_layout(path, names, arrays, case):
    """A result file laid out as the reference writes ASCII ones (OutputXML::writeResultsXML)."""
    nx, ny, nz = case.cells
    with open(path, "w") as fh:
        fh.write('<?xml version="1.0"?>\n<VTKFile type="RectilinearGrid" version="0.1" byte_order="LittleEndian">\n')
        fh.write(f'  <RectilinearGrid WholeExtent="0 {nx} 0 {ny} 0 {nz}">\n    <Piece Extent="0 {nx} 0 {ny} 0 {nz}">\n')
        fh.write("      <CellData>\n")
        for name, a in zip(names, arrays):
            comp = ' NumberOfComponents="3"' if a.ndim == 2 else ""
            fh.write(f'        <DataArray type="Float64" Name="{name}"{comp} format="ascii">\n')
            fh.write(" ".join("%.17g" % x for x in a.ravel()) + " \n        </DataArray>\n")
        fh.write("      </CellData>\n    </Piece>\n  </RectilinearGrid>\n</VTKFile>\n")


@pytest.mark.gpu
def test_driver_restart_matches_reference_restart(tmp_path):
    meta, g, arrays = _fixture()
    case = restart_case(meta["restart_file"])
    work = str(tmp_path)
    d = case.write(work)
    cases.write_ecogen_list(work, [d])
    res = os.path.join(work, "results", case.name)
    os.makedirs(os.path.join(res, "datasets"))
    with open(os.path.join(res, "infoCalcul.out"), "w") as fh:
        fh.write("\n".join(meta["info_lines"]) + "\n")
    _write_reference_layout(refrun.result_file(work, case.name, 2, binary=False), meta["names"], arrays, case)
    exe = os.path.join(ROOT, "ecogen_b200", "ecogen-b200")
    r = subprocess.run([exe, work + "/"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    got = refrun.reference_prim(refrun.read_vtr(refrun.result_file(work, case.name, 3, binary=False)), case.nphases)
    for name in ("alpha", "rho", "p", "u", "E"):
        assert rel_l1(got[name], g["final_" + name]) <= 1e-12, name
    with open(os.path.join(res, "infoCalcul.out")) as fh:
        lines = [ln.split() for ln in fh if ln.strip()]
    assert [ln[0] for ln in lines] == ["1", "0", "1", "2", "3"]
    assert lines[-1][1] == "30"


def test_ptueq_restart_fill_and_oracle_match_reference_restart():
    """PTUEq restart (fixture restart_ptueq): densities from (p, T) and the total energy rebuilt by
    ecg_restart_fill, then the oracle continues bit for bit on the reference's restarted run."""
    meta, g, arrays = _fixture("restart_ptueq")
    assert meta["names"][:2] == ["F0_Alpha_IG_air", "F0_Density_IG_air"]
    case = restart_case_ptueq()
    f = _abi_fields_ptueq(case, arrays)
    api.check(api.lib().ecg_restart_fill(C.byref(api.case_from_spec(case)), api._field_ptrs(f), case.ncells),
              "ecg_restart_fill")
    assert np.array_equal(f[2], arrays[1]) and np.array_equal(f[3], arrays[3])  # computeDensity(p, T)
    sim = oracle.Sim(case, {"alpha": np.stack(f[:2]), "rho": np.stack(f[2:4]), "p": f[4], "T": f[9],
                            "u": np.stack(f[5:8])})
    assert np.array_equal(sim.fields()["E"], f[8])
    it, t, dt = _info(meta)
    assert it == 20
    sim.t.value, sim.dt.value = t, dt
    sim.step(10)
    o = sim.fields()
    for name in ("alpha", "rho", "p", "u"):
        assert np.array_equal(o[name], g["final_" + name]), name
    assert np.array_equal(o["T"][0], g["final_Tm"])


@pytest.mark.gpu
def test_driver_ptueq_restart_matches_reference_restart(tmp_path):
    meta, g, arrays = _fixture("restart_ptueq")
    case = restart_case_ptueq(meta["restart_file"])
    work = str(tmp_path)
    d = case.write(work)
    cases.write_ecogen_list(work, [d])
    res = os.path.join(work, "results", case.name)
    os.makedirs(os.path.join(res, "datasets"))
    with open(os.path.join(res, "infoCalcul.out"), "w") as fh:
        fh.write("\n".join(meta["info_lines"]) + "\n")
    _write_reference_layout(refrun.result_file(work, case.name, 2, binary=False), meta["names"], arrays, case)
    exe = os.path.join(ROOT, "ecogen_b200", "ecogen-b200")
    r = subprocess.run([exe, work + "/"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    got = refrun.reference_prim(refrun.read_vtr(refrun.result_file(work, case.name, 3, binary=False)), case.nphases)
    for name in ("alpha", "rho", "p", "u", "Tm"):
        assert rel_l1(got[name], g["final_" + name]) <= 1e-12, name
