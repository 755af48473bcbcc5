"""Batched mode: many independent 1D cases in one persistent launch equal independent runs."""
import numpy as np
import pytest

from ecogen_b200 import api, cases
from oracle import oracle
from tests.conftest import rel_l1

TOL = 1e-12


def _batch_inputs(cs, tmp):
    import os
    recs, fields = [], []
    for i, c in enumerate(cs):
        d = c.write(str(tmp), subdir=f"c{i}")
        inp = api.Input(d, os.path.join(str(tmp), "libEOS"))
        recs.append(inp.case)
        fields.append(inp.fill())
    arr = (api.Case * len(recs))(*recs)
    cat = [np.concatenate([f[k] for f in fields]) for k in range(len(fields[0]))]
    return arr, cat


@pytest.mark.gpu
@pytest.mark.parametrize("order", [None, "vanleer"])
def test_batch_equals_independent_oracle_runs(order, tmp_path):
    cs = cases.batch_shock_tubes(ncases=12, seed=7, cells_range=(40, 700), iterations=15, limiter=order)
    arr, cat = _batch_inputs(cs, tmp_path)
    h = api.C.c_void_p()
    api.check(api.lib().ecg_batch_create(arr, len(cs), api.C.byref(h)), "ecg_batch_create")
    total = int(api.lib().ecg_batch_total_cells(h))
    assert total == sum(c.ncells for c in cs)
    api.check(api.lib().ecg_batch_upload_prim(h, api._field_ptrs(cat), total), "upload")
    tile, th = api.C.c_int32(), api.C.c_int32()
    api.check(api.lib().ecg_batch_autotune(h, api.C.byref(tile), api.C.byref(th)), "autotune")
    assert tile.value in (64, 128, 256)
    dt = np.full(len(cs), 1e-15)
    t = np.zeros(len(cs))
    st = api.StepStats()
    api.check(api.lib().ecg_batch_step(h, 15, dt.ctypes.data_as(api.C.POINTER(api.C.c_double)),
                                       t.ctypes.data_as(api.C.POINTER(api.C.c_double)), api.C.byref(st)), "step")
    out = [np.zeros(total) for _ in range(len(cat))]
    api.check(api.lib().ecg_batch_download_prim(h, api._field_ptrs(out), total), "download")
    api.lib().ecg_batch_destroy(h)
    off = 0
    for i, c in enumerate(cs):
        sim = oracle.Sim(c)
        sim.step(15)
        o = sim.fields()
        n = c.ncells
        k = c.nphases
        got = {"alpha": np.stack([out[j][off:off + n] for j in range(k)]),
               "rho": np.stack([out[k + j][off:off + n] for j in range(k)]),
               "p": out[2 * k][off:off + n], "u": out[2 * k + 1][off:off + n], "E": out[2 * k + 4][off:off + n]}
        for name in ("alpha", "rho", "p", "E"):
            assert rel_l1(got[name], o[name]) <= TOL, (i, name)
        assert rel_l1(got["u"], o["u"][0]) <= TOL
        assert dt[i] == pytest.approx(sim.dt.value, rel=1e-12)
        assert t[i] == pytest.approx(sim.t.value, rel=1e-12)
        off += n
    assert st.cell_updates == 15 * total


@pytest.mark.gpu
@pytest.mark.parametrize("tile", [64, 128, 256])
def test_batch_every_tile_equals_oracle(tile, tmp_path):
    """Each tile shape, on cases whose cell counts straddle the item size (tile - 1 cells per item)."""
    sizes = [40, 63, 64, 65, 127, 128, 254, 255, 256, 511]
    cs = cases.batch_shock_tubes(ncases=len(sizes), seed=11, cells_range=(40, 600), iterations=8, limiter="vanleer")
    for c, n in zip(cs, sizes):
        c.cells = (n, 1, 1)
    arr, cat = _batch_inputs(cs, tmp_path)
    h = api.C.c_void_p()
    api.check(api.lib().ecg_batch_create(arr, len(cs), api.C.byref(h)), "ecg_batch_create")
    total = int(api.lib().ecg_batch_total_cells(h))
    api.check(api.lib().ecg_batch_upload_prim(h, api._field_ptrs(cat), total), "upload")
    api.check(api.lib().ecg_batch_set_shape(h, tile, tile), "set_shape")
    st = api.StepStats()
    api.check(api.lib().ecg_batch_step(h, 8, None, None, api.C.byref(st)), "step")
    out = [np.zeros(total) for _ in range(len(cat))]
    api.check(api.lib().ecg_batch_download_prim(h, api._field_ptrs(out), total), "download")
    api.lib().ecg_batch_destroy(h)
    off = 0
    for i, c in enumerate(cs):
        sim = oracle.Sim(c)
        sim.step(8)
        o = sim.fields()
        n, k = c.ncells, c.nphases
        for j, name in ((0, "alpha"), (k, "rho")):
            assert rel_l1(np.stack([out[j + q][off:off + n] for q in range(k)]), o[name]) <= TOL, (i, name)
        assert rel_l1(out[2 * k][off:off + n], o["p"]) <= TOL, (i, "p")
        assert rel_l1(out[2 * k + 4][off:off + n], o["E"]) <= TOL, (i, "E")
        off += n
