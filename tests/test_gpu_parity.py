"""GPU path vs the reference's golden outputs and vs the oracle, through the C ABI.

Tolerance: 1e-12 relative L1 per field (sum|gpu - ref| / sum|ref|) after N steps.  The kernels
are built without multiply-add contraction and divide with the IEEE-exact ddiv, so the only
differences come from last-ulp differences of pow (ecg::epow, about 1 call in 1000) and exp against
glibc's, propagated through the scheme.
"""
import numpy as np
import pytest

from oracle import oracle
from tests.conftest import display, load_golden, rel_l1
from tests.helpers import gpu_run

TOL = 1e-12
KAPILA_KEYS = ["tube1d_o1_full", "tube1d_o2_vanleer", "tube1d_alphanull", "tube1d_nasg_o2", "bubble2d_o2",
               "bubble2d_limiters", "bubble2d_vanalbada", "bubble2d_o1", "cavity3d_o2", "cavity3d_o1",
               "expansion2d_ptmu", "tube1d_wall_o1", "tube1d_wall_o2", "bubble2d_sym_o2", "bubble2d_sym_o1",
               "cavity3d_wall_o2", "tube1d_thinc_o2", "bubble2d_thinc", "tube1d_transport_o2", "bubble2d_transport",
               "tube1d_transport_o1", "tube1d_pt_o1", "bubble2d_pt",
               "tube1d_stretch_o2", "tube1d_stretch_o1", "bubble2d_stretch_o2", "cavity3d_stretch_o2"]
EULER_KEYS = ["euler1d_o1", "euler1d_o2", "euler1d_wall_o2", "euler1d_transport_o2", "euler2d_o2_walls", "euler2d_o1",
              "euler3d_o2", "euler2d_stretch_o2"]


def _compare(key, got, g):
    for name in ("alpha", "rho", "p", "u", "E", "tr"):
        ref = g.get("final_" + name)
        if ref is None:
            continue
        v = display(got[name], name)
        err = rel_l1(v, ref)
        assert err <= TOL, f"{key}: {name} rel L1 {err:.3e} > {TOL}"


@pytest.mark.gpu
@pytest.mark.parametrize("key", KAPILA_KEYS + EULER_KEYS)
def test_gpu_matches_reference_golden(key, golden_cases, tmp_path):
    meta, g = load_golden(key)
    case = golden_cases[key]
    out = gpu_run(case, tmp_path)
    assert out["iteration"] == meta["iterations_done"]
    assert out["stats"]["nonfinite_cells"] == 0
    _compare(key, out, g)


@pytest.mark.gpu
@pytest.mark.parametrize("size", [(64, 30), (100, 20)])
def test_gpu_matches_oracle_2d(size, tmp_path):
    from ecogen_b200 import cases
    n, it = size
    case = cases.shock_bubble_2d(n=n, iterations=it)
    out = gpu_run(case, tmp_path)
    sim = oracle.Sim(case)
    sim.step(it)
    o = sim.fields()
    for name in ("alpha", "rho", "p", "u", "E"):
        assert rel_l1(out[name], o[name]) <= TOL, name
    assert out["dt"] == pytest.approx(sim.dt.value, rel=1e-12)
    assert out["t"] == pytest.approx(sim.t.value, rel=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("sides", [None, ["wall", "nonReflecting", "symmetry", "symmetry", "nonReflecting", "wall"]])
def test_gpu_matches_oracle_3d_ragged(sides, tmp_path):
    # non-multiple-of-tile sizes in every direction
    from ecogen_b200 import cases
    case = cases.cavity_collapse_3d(n=19, iterations=3, ninclusions=5, radius_cells=(2.0, 4.0))
    case.cells = (19, 7, 5)
    case.boundaries = sides
    out = gpu_run(case, tmp_path)
    sim = oracle.Sim(case)
    sim.step(3)
    o = sim.fields()
    for name in ("alpha", "rho", "p", "u", "E"):
        assert rel_l1(out[name], o[name]) <= TOL, name


@pytest.mark.gpu
@pytest.mark.parametrize("order", [None, "vanleer", "minmod"])
def test_gpu_symmetry_sides_match_oracle_2d(order, tmp_path):
    """Symmetry / wall sides on a mesh of several tiles per axis (tile edges next to the sides)."""
    from ecogen_b200 import cases
    case = cases.shock_bubble_2d(n=70, iterations=30, limiter=order, shock_x=6e-3, name="bubbleWalls")
    case.boundaries = ["wall", "symmetry", "symmetry", "wall"]
    out = gpu_run(case, tmp_path)
    sim = oracle.Sim(case)
    sim.step(30)
    o = sim.fields()
    for name in ("alpha", "rho", "p", "u", "E"):
        assert rel_l1(out[name], o[name]) <= TOL, name
    assert out["dt"] == pytest.approx(sim.dt.value, rel=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("vf", [("THINC", "THINC"), (None, "THINC")])
def test_gpu_thinc_matches_oracle_2d(vf, tmp_path):
    """THINC volume-fraction reconstruction on a mesh of several tiles per axis."""
    from ecogen_b200 import cases
    case = cases.shock_bubble_2d(n=64, iterations=25, limiter="vanleer", name="bubbleTHINC64")
    case.vf_limiter, case.interface_vf_limiter = vf
    case.boundaries = ["wall", "nonReflecting", "symmetry", "symmetry"]
    out = gpu_run(case, tmp_path)
    sim = oracle.Sim(case)
    sim.step(25)
    o = sim.fields()
    for name in ("alpha", "rho", "p", "u", "E"):
        assert rel_l1(out[name], o[name]) <= TOL, name


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
def test_gpu_transports_match_oracle(dim, tmp_path):
    """Two passive transports on meshes of several tiles per axis, with symmetry and open sides."""
    from ecogen_b200 import cases
    if dim == 2:
        case = cases.shock_bubble_2d(n=60, iterations=20, limiter="vanleer", name="bubbleTransport60")
        case.boundaries = ["wall", "nonReflecting", "symmetry", "nonReflecting"]
        steps = 20
    else:
        case = cases.cavity_collapse_3d(n=14, iterations=4, ninclusions=5, radius_cells=(2.0, 4.0), name="cavityTr")
        case.cells = (14, 9, 7)
        case.boundaries = ["wall", "nonReflecting", "symmetry", "symmetry", "nonReflecting", "wall"]
        steps = 4
    case.transports = ["color", "marker"]
    for i, st in enumerate(case.states):
        st.transports = {"color": float(i % 2), "marker": 0.5 * i}
    out = gpu_run(case, tmp_path)
    sim = oracle.Sim(case)
    sim.step(steps)
    o = sim.fields()
    for name in ("alpha", "rho", "p", "u", "E", "tr"):
        assert rel_l1(out[name], o[name]) <= TOL, name


@pytest.mark.gpu
def test_gpu_pt_relaxation_matches_oracle_2d(tmp_path):
    """Analytic p-T relaxation after the pressure one, on a mesh of several tiles per axis."""
    from ecogen_b200 import cases
    case = cases.shock_bubble_2d(n=64, iterations=20, limiter="vanleer", name="bubblePT64")
    case.pt_relaxation = True
    case.boundaries = ["wall", "nonReflecting", "symmetry", "symmetry"]
    out = gpu_run(case, tmp_path)
    sim = oracle.Sim(case)
    sim.step(20)
    o = sim.fields()
    for name in ("alpha", "rho", "p", "u", "E"):
        assert rel_l1(out[name], o[name]) <= TOL, name


@pytest.mark.gpu
def test_newton_stats_match_oracle(tmp_path):
    from ecogen_b200 import cases
    case = cases.cavity_collapse_3d(n=16, iterations=3, ninclusions=6, radius_cells=(2.0, 4.0))
    out = gpu_run(case, tmp_path)
    sim = oracle.Sim(case)
    sim.step(3)
    assert out["stats"]["relax_calls"] == sim.stats.relax_calls
    assert out["stats"]["newton_evals"] == sim.stats.newton_evals
    assert sum(out["stats"]["newton_hist"]) == sim.stats.relax_calls


@pytest.mark.gpu
@pytest.mark.parametrize("key", ["tube1d_o1_full", "bubble2d_o2", "euler1d_o2", "bubble2d_sym_o2"])
def test_driver_writes_reference_results(key, golden_cases, tmp_path):
    """ecogen-b200 <work> runs ECOGEN.xml's cases and writes reference-format VTK results."""
    import subprocess
    import os
    from ecogen_b200 import cases
    from oracle import refrun
    from tests.helpers import ROOT
    meta, g = load_golden(key)
    case = golden_cases[key]
    d = case.write(str(tmp_path))
    cases.write_ecogen_list(str(tmp_path), [d])
    exe = os.path.join(ROOT, "ecogen_b200", "ecogen-b200")
    r = subprocess.run([exe, str(tmp_path) + "/"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    files = refrun.result_files(str(tmp_path), case.name)
    assert len(files) >= 2
    raw = refrun.read_vtr(files[-1])
    got = refrun.reference_prim(raw, case.nphases)
    for name in ("alpha", "rho", "p", "u", "E"):
        ref = g.get("final_" + name)
        if ref is None or got.get(name) is None:
            continue
        assert rel_l1(got[name], ref) <= TOL, name
    # |grad rho| of the output (finite differences of the density: differences amplify the 1e-12)
    assert rel_l1(raw["gradRho"], g["final_gradRho"]) <= 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
def test_gpu_euler_matches_oracle_multid(dim, tmp_path):
    """Euler model on meshes of several tiles per axis (ragged), symmetry and open sides."""
    from ecogen_b200 import cases
    if dim == 2:
        case = cases.euler_blast_2d(n=70, ny=45, iterations=20, name="eulerBlast70",
                                    boundaries=["wall", "nonReflecting", "symmetry", "nonReflecting"])
    else:
        case = cases.euler_blast_2d(n=13, ny=9, nz=7, iterations=5, name="eulerBlast13",
                                    boundaries=["nonReflecting", "wall", "symmetry", "nonReflecting", "wall", "wall"])
    out = gpu_run(case, tmp_path)
    sim = oracle.Sim(case)
    sim.step(case.iterations)
    o = sim.fields()
    for name in ("rho", "p", "u", "E"):
        assert rel_l1(out[name], o[name]) <= TOL, name
    assert out["dt"] == pytest.approx(sim.dt.value, rel=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", ["2d", "3d"])
def test_gpu_matches_oracle_stretched(shape, tmp_path):
    """Stretched meshes over many tiles: per-cell CFL lengths and surface / volume ratios, MUSCL
    distances of unequal cells, symmetry sides."""
    from ecogen_b200 import cases
    if shape == "2d":
        case = cases.shock_bubble_2d(n=24, iterations=15, name="stretchBubbleTiles")
        case.cells = (90, 70, 1)
        case.stretch = {"x": [(0.0, 0.003, 0.96, 30), (0.003, 0.007, 1.0, 40), (0.007, 0.01, 1.05, 20)],
                        "y": [(0.0, 0.005, 1.0, 40), (0.005, 0.01, 1.04, 30)]}
        case.boundaries = ["wall", "nonReflecting", "symmetry", "nonReflecting"]
    else:
        case = cases.cavity_collapse_3d(n=16, iterations=5, ninclusions=8, radius_cells=(2.0, 4.0),
                                        name="stretchCavityTiles")
        case.cells = (19, 16, 14)
        case.stretch = {"x": [(0.0, 0.01, 1.03, 19)], "z": [(0.0, 0.004, 1.0, 6), (0.004, 0.01, 1.08, 8)]}
    out = gpu_run(case, tmp_path)
    sim = oracle.Sim(case)
    sim.step(case.iterations)
    o = sim.fields()
    for name in ("alpha", "rho", "p", "u", "E"):
        assert rel_l1(out[name], o[name]) <= TOL, name
    assert out["dt"] == pytest.approx(sim.dt.value, rel=1e-12)
