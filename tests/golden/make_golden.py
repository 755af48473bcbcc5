"""Generates the golden fixtures of tests/golden/ by running the reference ECOGEN solver.

The reference is built from its own sources by ``make -C oracle ref`` (single-rank MPI stand-in,
``oracle/Makefile``).  Each fixture is the final state the reference writes (base64 Float64 VTK,
read back exactly by oracle/refrun.py) for one small case from ecogen_b200/cases.py, plus the
initial state (result file 0).  Run from the repository root:

    python tests/golden/make_golden.py [key ...]
"""
from __future__ import annotations

import json
import os
import shutil
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from ecogen_b200 import cases  # noqa: E402
from oracle import refrun  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def golden_cases():
    """Name -> case.  Small versions of every workload family plus edge cases."""
    g = {}
    g["tube1d_o1_full"] = cases.shock_tube_1d(ncells=1000)  # 1000 cells to t = 240 us (797 steps)
    g["tube1d_o2_vanleer"] = cases.shock_tube_1d(ncells=200, iterations=60, order="vanleer")
    g["tube1d_alphanull"] = cases.shock_tube_1d(ncells=120, iterations=40, alpha_floor=0.0, alpha_null=True,
                                                name="tubeAlphaNull")
    g["tube1d_nasg_o2"] = cases.shock_tube_1d(ncells=150, iterations=30, order="minmod", liquid=cases.WATER_NASG,
                                              name="tubeNASG")
    g["bubble2d_o2"] = cases.shock_bubble_2d(n=32, iterations=12)
    c = cases.shock_bubble_2d(n=24, iterations=8, limiter="vanleer", name="bubbleLimiters")
    c.interface_limiter, c.vf_limiter, c.interface_vf_limiter = "superbee", "minmod", "mc"
    g["bubble2d_limiters"] = c
    g["bubble2d_vanalbada"] = cases.shock_bubble_2d(n=20, iterations=6, limiter="vanalbada", name="bubbleVanAlbada")
    g["bubble2d_o1"] = cases.shock_bubble_2d(n=24, iterations=8, limiter=None, name="bubbleO1")
    g["cavity3d_o2"] = cases.cavity_collapse_3d(n=12, iterations=4, ninclusions=6, radius_cells=(2.0, 4.0))
    g["cavity3d_o1"] = cases.cavity_collapse_3d(n=10, iterations=3, ninclusions=4, radius_cells=(2.0, 3.0),
                                                limiter=None, name="cavityO1")
    g["expansion2d_ptmu"] = cases.expansion_tube_2d(n=24, iterations=8)
    g["euler1d_o1"] = cases.euler_shock_tube(ncells=200, iterations=40)
    # symmetry / wall sides (reflecting boundaries)
    c = cases.shock_tube_1d(ncells=120, iterations=120, x_interface=0.75, name="tubeWallO1")
    c.boundaries = ["symmetry", "wall"]
    g["tube1d_wall_o1"] = c
    c = cases.shock_tube_1d(ncells=120, iterations=120, x_interface=0.75, order="vanleer", name="tubeWallO2")
    c.boundaries = ["wall", "symmetry"]
    g["tube1d_wall_o2"] = c
    c = cases.shock_bubble_2d(n=24, iterations=10, name="bubbleSym")
    c.boundaries = ["wall", "nonReflecting", "symmetry", "symmetry"]
    g["bubble2d_sym_o2"] = c
    c = cases.shock_bubble_2d(n=20, iterations=8, limiter=None, name="bubbleSymO1")
    c.boundaries = ["symmetry", "nonReflecting", "symmetry", "wall"]
    g["bubble2d_sym_o1"] = c
    c = cases.cavity_collapse_3d(n=10, iterations=4, ninclusions=5, radius_cells=(2.0, 3.0), name="cavityWall")
    c.boundaries = ["wall"] * 6
    g["cavity3d_wall_o2"] = c
    c = cases.euler_shock_tube(ncells=100, iterations=80, order="vanleer", name="eulerWall")
    c.boundaries = ["wall", "symmetry"]
    g["euler1d_wall_o2"] = c
    # THINC volume-fraction reconstruction (everywhere, and at interfaces only)
    c = cases.shock_tube_1d(ncells=200, iterations=60, order="vanleer", name="tubeTHINC")
    c.vf_limiter, c.interface_vf_limiter = "THINC", "THINC"
    g["tube1d_thinc_o2"] = c
    c = cases.shock_bubble_2d(n=24, iterations=10, limiter="minmod", name="bubbleTHINC")
    c.interface_vf_limiter = "THINC"
    c.boundaries = ["wall", "nonReflecting", "symmetry", "symmetry"]
    g["bubble2d_thinc"] = c
    # passive transports (a colour function of the bubble and a second marker)
    c = cases.shock_tube_1d(ncells=150, iterations=50, order="vanleer", name="tubeTransport")
    c.transports = ["color", "marker"]
    c.states[0].transports = {"color": 1.0, "marker": 0.25}
    c.states[1].transports = {"color": 0.0}
    c.boundaries = ["nonReflecting", "wall"]
    g["tube1d_transport_o2"] = c
    c = cases.shock_bubble_2d(n=24, iterations=10, limiter="vanleer", name="bubbleTransport")
    c.transports = ["color"]
    for st in c.states:
        st.transports = {"color": 1.0 if st.phases[0].alpha < 0.5 else 0.0}
    c.interface_vf_limiter = "THINC"
    c.boundaries = ["wall", "nonReflecting", "symmetry", "symmetry"]
    g["bubble2d_transport"] = c
    c = cases.shock_tube_1d(ncells=120, iterations=40, name="tubeTransportO1")
    c.transports = ["color"]
    c.states[0].transports = {"color": 1.0}
    g["tube1d_transport_o1"] = c
    c = cases.euler_shock_tube(ncells=100, iterations=40, order="minmod", name="eulerTransport")
    c.transports = ["color"]
    c.states[1].transports = {"color": 1.0}
    g["euler1d_transport_o2"] = c
    # analytic pressure-temperature relaxation after the pressure relaxation (RelaxationPT)
    c = cases.shock_tube_1d(ncells=100, iterations=40, name="tubePT")
    c.pt_relaxation = True
    g["tube1d_pt_o1"] = c
    c = cases.shock_bubble_2d(n=20, iterations=8, limiter="vanleer", name="bubblePT")
    c.pt_relaxation = True
    g["bubble2d_pt"] = c
    g["euler1d_o2"] = cases.euler_shock_tube(ncells=200, iterations=40, order="vanleer", name="eulerO2")
    # Euler model on 2D and 3D meshes
    g["euler2d_o2_walls"] = cases.euler_blast_2d(n=24, ny=20, iterations=12,
                                                 boundaries=["nonReflecting", "wall", "symmetry", "nonReflecting"])
    g["euler2d_o1"] = cases.euler_blast_2d(n=20, iterations=10, order=None, name="eulerBlastO1")
    g["euler3d_o2"] = cases.euler_blast_2d(n=10, ny=8, nz=6, iterations=5, order="minmod", name="eulerBlast3D",
                                           boundaries=["wall", "nonReflecting", "nonReflecting", "symmetry",
                                                       "wall", "nonReflecting"])
    # temperature-pressure-velocity equilibrium model (ModPTUEq)
    g["ptueq_tube_o2"] = cases.ptueq_shock_tube_1d(ncells=200, iterations=60)
    g["ptueq_tube_o1"] = cases.ptueq_shock_tube_1d(ncells=300, iterations=None, total_time=1.0e-4, order=None,
                                                   name="ptueqTubeO1")
    g["ptueq_tube_wall_o1"] = cases.ptueq_shock_tube_1d(ncells=120, iterations=150, order=None, x_interface=0.75,
                                                        name="ptueqTubeWall", boundaries=["wall", "symmetry"])
    g["ptueq_bubble2d_o2"] = cases.ptueq_bubble_2d(n=24, iterations=10)
    g["ptueq_bubble2d_o1_sym"] = cases.ptueq_bubble_2d(n=20, ny=16, iterations=8, limiter=None, name="ptueqBubbleSym",
                                                       boundaries=["symmetry", "nonReflecting", "wall", "symmetry"])
    c = cases.ptueq_bubble_2d(n=20, iterations=8, limiter="minmod", name="ptueqBubbleTHINC")
    c.interface_limiter, c.interface_vf_limiter = "superbee", "THINC"
    g["ptueq_bubble2d_thinc"] = c
    g["ptueq_bubble3d_o2"] = cases.ptueq_bubble_2d(n=10, nz=6, iterations=4, name="ptueqBubble3D")
    # stretched meshes (mesh.xml meshStretching, MeshCartesian::meshStretching / stretchZone::stretching):
    # a uniform zone then a geometric one (and the reverse), per axis
    g.update(stretched_cases())
    return g


def stretched_cases():
    g = {}
    c = cases.shock_tube_1d(ncells=100, iterations=60, order="vanleer", name="tubeStretch")
    c.stretch = {"x": [(0.0, 0.6, 1.0, 60), (0.6, 1.0, 1.04, 40)]}
    g["tube1d_stretch_o2"] = c
    c = cases.shock_tube_1d(ncells=90, iterations=40, name="tubeStretchO1")
    c.stretch = {"x": [(0.0, 0.3, 0.95, 30), (0.3, 1.0, 1.0, 60)]}
    g["tube1d_stretch_o1"] = c
    c = cases.shock_bubble_2d(n=24, iterations=10, name="bubbleStretch")
    c.cells = (28, 26, 1)
    c.stretch = {"x": [(0.0, 0.004, 1.0, 12), (0.004, 0.01, 1.05, 16)],
                 "y": [(0.0, 0.003, 0.93, 8), (0.003, 0.007, 1.0, 10), (0.007, 0.01, 1.08, 8)]}
    c.boundaries = ["wall", "nonReflecting", "symmetry", "nonReflecting"]
    g["bubble2d_stretch_o2"] = c
    c = cases.cavity_collapse_3d(n=10, iterations=4, ninclusions=5, radius_cells=(2.0, 3.0), name="cavityStretch")
    c.cells = (10, 11, 12)
    c.stretch = {"y": [(0.0, 0.005, 1.0, 5), (0.005, 0.01, 1.1, 6)], "z": [(0.0, 0.01, 0.95, 12)]}
    g["cavity3d_stretch_o2"] = c
    c = cases.euler_blast_2d(n=20, iterations=12, name="eulerStretch")
    c.cells = (22, 20, 1)
    c.stretch = {"x": [(0.0, c.lengths[0] / 2, 1.0, 10), (c.lengths[0] / 2, c.lengths[0], 1.06, 12)]}
    g["euler2d_stretch_o2"] = c
    return g


def case_meta(c) -> dict:
    return {"name": c.name, "cells": list(c.cells), "lengths": list(c.lengths), "nphases": c.nphases,
            "model": c.model, "iterations": c.iterations, "total_time": c.total_time, "cfl": c.cfl,
            "order": c.second_order, "limiters": [c.interface_limiter, c.vf_limiter, c.interface_vf_limiter]}


def main():
    if not refrun.available():
        sys.exit("reference binary missing: run `make -C oracle ref` first")
    work = tempfile.mkdtemp(prefix="ecg_golden_")
    only = set(sys.argv[1:])
    for key, c in golden_cases().items():
        if only and key not in only:
            continue
        w = os.path.join(work, key)
        shutil.rmtree(w, ignore_errors=True)
        d = c.write(w)
        cases.write_ecogen_list(w, [d])
        r = refrun.run(w)
        if r.returncode != 0:
            raise SystemExit(f"{key}: reference failed\n{r.stdout[-3000:]}")
        files = refrun.result_files(w, c.name)
        f0 = refrun.reference_prim(refrun.read_vtr(files[0]), c.nphases)
        raw1 = refrun.read_vtr(files[-1])
        f1 = refrun.reference_prim(raw1, c.nphases)
        f1["gradRho"] = raw1.get("gradRho")
        it, t, dt = refrun.info(w, c.name)
        arrays = {}
        for tag, f in (("init", f0), ("final", f1)):
            for name, v in f.items():
                if v is not None:
                    arrays[f"{tag}_{name}"] = np.asarray(v)
        np.savez_compressed(os.path.join(OUT, f"{key}.npz"), **arrays)
        meta = case_meta(c)
        meta.update({"iterations_done": it, "time6": t, "dt6": dt})
        with open(os.path.join(OUT, f"{key}.json"), "w") as fh:
            json.dump(meta, fh, indent=1)
        print(key, "iterations", it, "t", t)
    shutil.rmtree(work, ignore_errors=True)


def restart_case(restart_file=None):
    """2D shock-bubble printed every 10 iterations as ASCII with 17 digits (a restart reads ASCII files)."""
    c = cases.shock_bubble_2d(n=20, iterations=30, name="restartBubble")
    c.boundaries = ["wall", "nonReflecting", "symmetry", "nonReflecting"]
    c.output_binary, c.output_precision, c.print_freq, c.restart_file = False, 17, 10, restart_file
    return c


def restart_case_ptueq(restart_file=None):
    """2D PTUEq bubble printed every 10 iterations as ASCII with 17 digits."""
    c = cases.ptueq_bubble_2d(n=20, ny=16, iterations=30, name="restartPTUEq")
    c.output_binary, c.output_precision, c.print_freq, c.restart_file = False, 17, 10, restart_file
    return c


def make_restart_golden(key="restart2d", make_case=None):
    """<key>.npz/.json: the reference's result file 2 and infoCalcul.out of a 30-iteration run, and the
    final file of the reference restarted from file 2 (Run::restartSimulation src/Run.cpp:345)."""
    make_case = make_case or restart_case
    work = tempfile.mkdtemp(prefix=f"ecg_golden_{key}_")
    c = make_case()
    d = c.write(work)
    cases.write_ecogen_list(work, [d])
    r = refrun.run(work)
    if r.returncode != 0:
        raise SystemExit(key + ": reference failed\n" + r.stdout[-3000:])
    with open(os.path.join(work, "results", c.name, "infoCalcul.out")) as f:
        info_lines = [ln.rstrip("\n") for ln in f if ln.strip()]
    src = refrun.read_vtr_ordered(refrun.result_file(work, c.name, 2, binary=False))
    c2 = make_case(2)
    d = c2.write(work)  # same case folder, now restarting from file 2
    r = refrun.run(work)
    if r.returncode != 0:
        raise SystemExit(key + ": reference restart failed\n" + r.stdout[-3000:])
    fin = refrun.read_vtr(refrun.result_file(work, c.name, 3, binary=False))
    arrays = {f"in{i:02d}": np.asarray(a) for i, (_, a) in enumerate(src)}
    arrays.update({"final_" + k: np.asarray(v) for k, v in
                   refrun.reference_prim(fin, c.nphases).items() if v is not None})
    np.savez_compressed(os.path.join(OUT, key + ".npz"), **arrays)
    with open(os.path.join(OUT, key + ".json"), "w") as fh:
        json.dump({"info_lines": info_lines[:4], "names": [n for n, _ in src], "restart_file": 2,
                   "case": case_meta(c)}, fh, indent=1)
    print(key, info_lines[:4])
    shutil.rmtree(work, ignore_errors=True)


if __name__ == "__main__":
    if sys.argv[1:] == ["restart2d"]:
        make_restart_golden()
    elif sys.argv[1:] == ["restart_ptueq"]:
        make_restart_golden("restart_ptueq", restart_case_ptueq)
    else:
        main()
