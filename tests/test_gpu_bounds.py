"""The bounds-checked build (libecg_bounds.so, -DECG_BOUNDS_CHECK): no device access leaves its buffer.

Every state, face-array and staged-cell index of the step kernels is checked in that build; an index
outside its buffer would be counted in ecg_step_stats.bounds_violations and the access skipped (never a
trap).  A separate process loads the bounds-checked library (ECG_LIB) and runs small cases of each
kernel family -- split and fused forms, first order and MUSCL, walls, stretched meshes, ragged meshes
that leave partial tiles, 1D to 3D, the allocation-free step -- and must see no violation and the
oracle's fields within 1e-12.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "ecogen_b200", "libecg_bounds.so")

SCRIPT = r'''
import json, os, sys, tempfile
sys.path.insert(0, sys.argv[1])
import numpy as np
from ecogen_b200 import api, cases
from oracle import oracle

def rel(a, b):
    d = np.abs(b).sum()
    return float(np.abs(a - b).sum() / d) if d else float(np.abs(a - b).sum())

def run(case, form):
    with tempfile.TemporaryDirectory() as tmp:
        d = case.write(tmp)
        inp = api.Input(d, os.path.join(tmp, "libEOS"))
        ctx = api.Context(inp.case)
        if form is not None:
            ctx.set_step_form(form)
        ctx.upload(inp.fill())
        st = ctx.step(case.iterations)
        out = ctx.download_dict()
        ctx.close()
    return out, st

def walls(c, b):
    c.boundaries = b
    return c

def stretched(c, cells, st):
    c.cells, c.stretch = cells, st
    return c

CASES = [
    ("bubble2d_ragged", lambda: cases.shock_bubble_2d(n=37, iterations=6, name="bBubble")),
    ("bubble2d_walls_o1", lambda: walls(cases.shock_bubble_2d(n=29, iterations=5, limiter=None, name="bWalls"),
                                         ["symmetry", "wall", "nonReflecting", "symmetry"])),
    ("cavity3d_walls", lambda: walls(cases.cavity_collapse_3d(n=13, iterations=3, ninclusions=4,
                                                              radius_cells=(2.0, 3.0), name="bCavity"),
                                     ["wall", "symmetry", "nonReflecting", "symmetry", "wall", "nonReflecting"])),
    ("bubble2d_stretched", lambda: stretched(cases.shock_bubble_2d(n=20, iterations=5, name="bStretch"), (33, 21, 1),
                                             {"x": [(0.0, 0.004, 1.0, 13), (0.004, 0.01, 1.05, 20)]})),
    ("expansion_ptmu", lambda: cases.expansion_tube_2d(n=26, iterations=4, name="bPTMu")),
    ("tube1d", lambda: cases.shock_tube_1d(ncells=300, iterations=20, order="vanleer", name="bTube")),
    ("euler2d", lambda: cases.euler_blast_2d(n=23, iterations=5, name="bEuler")),
]
res = {}
for key, make in CASES:
    case = make()
    sim = oracle.Sim(case)
    sim.step(case.iterations)
    o = sim.fields()
    forms = [None] if case.dim < 2 or case.model.upper() == "EULER" else [api.FORM_SPLIT, api.FORM_FUSED]
    for form in forms:
        out, st = run(case, form)
        err = max(rel(out[k], o[k]) for k in ("alpha", "rho", "p", "u", "E"))
        res[f"{key}/{form}"] = {"violations": st.bounds_violations, "err": err}
print(json.dumps(res))
'''


@pytest.mark.gpu
def test_bounds_checked_build_sees_no_violation():
    assert os.path.exists(LIB), "libecg_bounds.so is not built (python -m ecogen_b200.build bounds)"
    env = dict(os.environ, ECG_LIB=LIB)
    r = subprocess.run([sys.executable, "-c", SCRIPT, ROOT], env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-4000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res
    for key, v in res.items():
        assert v["violations"] == 0, (key, v)
        assert v["err"] <= 1e-12, (key, v)
