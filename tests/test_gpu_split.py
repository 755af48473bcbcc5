"""Split form (per-axis face-flux kernels + cell kernel) against the fused form, bit for bit.

Both forms compute every face flux with the same device functions and accumulate the fluxes of a
cell in the reference's face order, so after N steps every field, dt, t and every relaxation counter
must be identical -- not merely close.  The cases cover the kernel variants the split form runs:
EOS types and limiter compiled in (the benchmark's), generic EOS with THINC, symmetry / wall sides
in MUSCL and first order, three phases in 3D, p-T-mu relaxation, the learned seed, and meshes whose
sizes are not multiples of the face-kernel blocks.  The face kernels stage their tiles by TMA tensor
copies where the mesh allows (an even number of x cells) and by their own loads elsewhere; both stagings
must give the same bits too.
"""
import os

import numpy as np
import pytest

from ecogen_b200 import api, cases


def _thinc():
    c = cases.shock_bubble_2d(n=40, iterations=12, limiter="minmod", name="splitTHINC")
    c.interface_limiter, c.interface_vf_limiter = "superbee", "THINC"
    return c


def _walls2d():
    c = cases.shock_bubble_2d(n=37, iterations=15, name="splitWalls")
    c.boundaries = ["wall", "nonReflecting", "symmetry", "symmetry"]
    return c


def _walls2d_o1():
    c = cases.shock_bubble_2d(n=29, iterations=10, limiter=None, name="splitWallsO1")
    c.boundaries = ["symmetry", "wall", "nonReflecting", "symmetry"]
    return c


def _walls3d():
    c = cases.cavity_collapse_3d(n=14, iterations=6, ninclusions=5, radius_cells=(2.0, 4.0), name="splitWalls3D")
    c.boundaries = ["wall", "symmetry", "nonReflecting", "symmetry", "wall", "nonReflecting"]
    return c


def _stretched():
    c = cases.shock_bubble_2d(n=24, iterations=12, name="splitStretch")
    c.cells = (50, 44, 1)
    c.stretch = {"x": [(0.0, 0.005, 1.0, 20), (0.005, 0.01, 1.04, 30)], "y": [(0.0, 0.01, 0.97, 44)]}
    c.boundaries = ["symmetry", "nonReflecting", "wall", "nonReflecting"]
    return c


SPLIT_CASES = {
    "bubble2d_stretched_walls": _stretched,
    "bubble2d_vanleer_ragged": lambda: cases.shock_bubble_2d(n=70, iterations=20, name="splitBubble"),
    "bubble2d_thinc_generic": _thinc,
    "bubble2d_walls_o2": _walls2d,
    "bubble2d_walls_o1": _walls2d_o1,
    "cavity3d_3phase_minmod": lambda: cases.cavity_collapse_3d(n=23, iterations=8, ninclusions=12,
                                                               radius_cells=(2.0, 5.0), name="splitCavity"),
    "cavity3d_walls": _walls3d,
    "expansion2d_ptmu": lambda: cases.expansion_tube_2d(n=48, iterations=10, name="splitPTMu"),
}


def _run(case, tmp, form, steps, model=None, staging=None):
    d = case.write(str(tmp))
    inp = api.Input(d, os.path.join(str(tmp), "libEOS"))
    ctx = api.Context(inp.case)
    assert ctx.step_form == api.FORM_SPLIT  # the default for 2D / 3D Kapila cases
    # TMA staging is the default wherever the x rows allow a tensor copy (even number of x cells)
    assert ctx.face_staging == (api.STAGING_TMA if case.cells[0] % 2 == 0 else api.STAGING_PLAIN)
    ctx.set_step_form(form)
    if staging is not None:
        ctx.set_face_staging(staging)
    ctx.upload(inp.fill())
    if model is not None:
        model.install(ctx)
    st = ctx.step(steps)
    out = ctx.download_dict()
    res = (out, st.as_dict(), ctx.dt.value, ctx.t.value)
    ctx.close()
    return res


def _same(a, b):
    out_a, st_a, dt_a, t_a = a
    out_b, st_b, dt_b, t_b = b
    for name in ("alpha", "rho", "p", "u", "E"):
        assert np.array_equal(out_a[name], out_b[name]), name
    assert dt_a == dt_b and t_a == t_b
    for k in ("relax_calls", "newton_evals", "newton_fallback", "newton_max", "nonfinite_cells", "ptmu_errors",
              "seeded", "seed_rejected"):
        assert st_a[k] == st_b[k], k


@pytest.mark.gpu
@pytest.mark.parametrize("key", list(SPLIT_CASES))
def test_split_form_equals_fused_form(key, tmp_path):
    case = SPLIT_CASES[key]()
    steps = case.iterations
    (tmp_path / "s").mkdir()
    (tmp_path / "f").mkdir()
    split = _run(case, tmp_path / "s", api.FORM_SPLIT, steps)
    fused = _run(case, tmp_path / "f", api.FORM_FUSED, steps)
    _same(split, fused)


@pytest.mark.gpu
def test_split_form_equals_fused_form_seeded(tmp_path):
    from ecogen_b200 import seed as seedmod
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "ecogen_b200", "models",
                        "seed_np3.npz")
    model = seedmod.SeedModel.load(path)
    case = cases.cavity_collapse_3d(n=20, iterations=6, ninclusions=10, radius_cells=(2.0, 5.0), name="splitSeed")
    (tmp_path / "s").mkdir()
    (tmp_path / "f").mkdir()
    split = _run(case, tmp_path / "s", api.FORM_SPLIT, 6, model)
    fused = _run(case, tmp_path / "f", api.FORM_FUSED, 6, model)
    _same(split, fused)
    assert split[1]["seeded"] + split[1]["seed_rejected"] > 0


@pytest.mark.gpu
def test_split_form_is_refused_where_it_does_not_apply(tmp_path):
    """1D cases run fused only: asking for the split form is an error, not a silent fallback."""
    case = cases.shock_tube_1d(ncells=64, iterations=2, order="vanleer")
    d = case.write(str(tmp_path))
    inp = api.Input(d, os.path.join(str(tmp_path), "libEOS"))
    ctx = api.Context(inp.case)
    assert ctx.step_form == api.FORM_FUSED
    with pytest.raises(api.EcgError):
        ctx.set_step_form(api.FORM_SPLIT)
    ctx.close()


TMA_CASES = {
    "bubble2d_vanleer": lambda: cases.shock_bubble_2d(n=70, iterations=12, name="tmaBubble"),
    "bubble2d_walls_o1": lambda: _walls_o1_even(),
    "bubble2d_stretched_walls": _stretched,
    "cavity3d_3phase_minmod": lambda: cases.cavity_collapse_3d(n=26, iterations=6, ninclusions=12,
                                                               radius_cells=(2.0, 5.0), name="tmaCavity"),
    "cavity3d_walls": _walls3d,
    "expansion2d_ptmu": lambda: cases.expansion_tube_2d(n=48, iterations=8, name="tmaPTMu"),
}


def _walls_o1_even():
    c = cases.shock_bubble_2d(n=34, iterations=10, limiter=None, name="tmaWallsO1")
    c.boundaries = ["symmetry", "wall", "nonReflecting", "symmetry"]
    return c


@pytest.mark.gpu
@pytest.mark.parametrize("key", list(TMA_CASES))
def test_tma_staging_equals_plain_staging(key, tmp_path):
    """Tensor-copy staging of the face kernels' tiles against the kernels' own loads: the same bits, on
    meshes whose sizes are not multiples of the blocks (partial boxes at the ends of the lines, zero-filled
    cells outside the mesh), with walls, first order and MUSCL, 2D and 3D."""
    case = TMA_CASES[key]()
    assert case.cells[0] % 2 == 0
    steps = case.iterations
    (tmp_path / "t").mkdir()
    (tmp_path / "p").mkdir()
    tma = _run(case, tmp_path / "t", api.FORM_SPLIT, steps, staging=api.STAGING_TMA)
    plain = _run(case, tmp_path / "p", api.FORM_SPLIT, steps, staging=api.STAGING_PLAIN)
    _same(tma, plain)
    assert tma[1]["staging_timeouts"] == 0


@pytest.mark.gpu
def test_staging_setting_and_odd_rows(tmp_path):
    """An odd number of x cells leaves no 16-byte row stride for a tensor map: the context reports plain
    staging and runs it; the fused form has no face kernels to stage for."""
    case = cases.shock_bubble_2d(n=37, iterations=2, name="tmaOdd")
    d = case.write(str(tmp_path))
    inp = api.Input(d, os.path.join(str(tmp_path), "libEOS"))
    ctx = api.Context(inp.case)
    assert ctx.face_staging == api.STAGING_PLAIN
    ctx.set_face_staging(api.STAGING_TMA)  # accepted, but no maps exist for this mesh
    assert ctx.face_staging == api.STAGING_PLAIN
    ctx.close()
    even = cases.shock_bubble_2d(n=38, iterations=2, name="tmaEven")
    d = even.write(str(tmp_path / "e"))
    inp = api.Input(d, os.path.join(str(tmp_path / "e"), "libEOS"))
    ctx = api.Context(inp.case)
    assert ctx.face_staging == api.STAGING_TMA
    ctx.set_face_staging(api.STAGING_PLAIN)
    assert ctx.face_staging == api.STAGING_PLAIN
    ctx.set_face_staging(api.STAGING_TMA)
    ctx.set_step_form(api.FORM_FUSED)
    assert ctx.face_staging == api.STAGING_PLAIN
    with pytest.raises(api.EcgError):
        ctx.set_face_staging(7)
    ctx.close()
