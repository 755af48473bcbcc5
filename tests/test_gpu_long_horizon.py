"""Parity of the benchmarked kernels at mid sizes and long horizons.

The other parity tests run tens of steps on meshes of up to 100^2 cells; the benchmark quotes the
workloads at 2048^2 (2000 steps), 256^3 and 1024^2.  A 1e-12 relative L1 bar after N steps could
hold at 30 steps and fail at 300 if branch decisions (interface detector, limiter thresholds,
velocity zeroing, Newton stopping tests) flip on last-ulp differences and the flips accumulate.
These tests run the exact kernel variants of the benchmark (EOS types and limiter compiled in) for
hundreds of steps:

* against the oracle (the C restatement, pinned bit for bit on the reference's fixtures):
  2D shock-bubble 512^2 x 200 steps, 3D three-phase cavity 64^3 x 20 steps, 2D p-T-mu expansion
  256^2 x 50 steps;
* against the reference solver itself (oracle/_ref/ECOGEN, built from the reference sources):
  2D shock-bubble 128^2 x 300 steps, 3D cavity 32^3 x 30 steps, 2D p-T-mu expansion 128^2 x 100 steps.

The CPU runs start together in a process pool (spawned, so no GPU state is inherited) before any GPU
work of this module and take about three minutes; the GPU runs take seconds.

The p-T-mu workload is the exception to a fixed 1e-12 bar, and the tests measure why.  Its
saturation Newton (RelaxationPTMu, Mixture::computeTsat) stops at a loose residual, so a last-ulp
difference of ln or pow in one cell changes that cell's Newton path and moves its pressure by up to
~1e-6; the changes spread.  Run on the CPU alone, the oracle with a correctly rounded ln instead of
the host libm's (they differ in about 1 call in 600,000) differs from the stock oracle after 50 steps
on 256^2 by 1.6e-12 relative L1 in alpha and 4.5e-9 in p.  That spread -- the envelope -- is
measured in the same run (oracle/ecg_crlog.h, libecg_oracle_crlog.so) and the GPU, which uses a
correctly rounded ln and CUDA's pow, must stay within 3x of it per field (or 1e-12, whichever is
larger).  The 2D and 3D pressure-relaxation workloads carry such differences no further than
~1e-14 (1-ulp pow changes in 10 % of calls over 300 steps), and are held to 1e-12.
"""
import concurrent.futures as cf
import multiprocessing as mp
import os
import shutil
import tempfile

import numpy as np
import pytest

from ecogen_b200 import cases
from tests.conftest import display, rel_l1
from tests.helpers import gpu_run

TOL = 1e-12


def _c2(n, it):
    return cases.shock_bubble_2d(n=n, iterations=it, name=f"longBubble{n}")


def _c3(n, it):
    return cases.cavity_collapse_3d(n=n, iterations=it, name=f"longCavity{n}")


def _c5(n, it):
    return cases.expansion_tube_2d(n=n, iterations=it, name=f"longExpansion{n}")


# key -> (checker, case builder, mesh, steps)
LONG = {
    "c2_512_oracle": ("oracle", _c2, 512, 200),
    "c3_64_oracle": ("oracle", _c3, 64, 20),
    "c5_256_oracle": ("oracle", _c5, 256, 50),
    "c2_128_reference": ("reference", _c2, 128, 300),
    "c3_32_reference": ("reference", _c3, 32, 30),
    "c5_128_reference": ("reference", _c5, 128, 100),
}


def _case(key):
    _, build, n, it = LONG[key]
    return build(n, it)


ENVELOPE_FACTOR = 3.0


def _ptmu(key):
    return LONG[key][1] is _c5


def _cpu_job(key, crlog=False):
    """Runs one checker (in a spawned worker) and returns its final fields; with crlog, the oracle
    built with a correctly rounded ln (the sensitivity variant) on the checker's case."""
    kind = LONG[key][0]
    case = _case(key)
    if kind == "oracle" or crlog:
        from oracle import oracle
        sim = oracle.Sim(case, crlog=crlog)
        sim.step(case.iterations)
        f = sim.fields()
        return {"fields": {k: np.asarray(f[k]) for k in ("alpha", "rho", "p", "u", "E")},
                "t": sim.t.value, "dt": sim.dt.value, "iterations": case.iterations}
    from oracle import refrun
    work = tempfile.mkdtemp(prefix=f"ecg_long_{key}_")
    try:
        d = case.write(work)
        cases.write_ecogen_list(work, [d])
        r = refrun.run(work)
        if r.returncode != 0:
            raise RuntimeError(f"reference failed on {key}: {r.stdout[-2000:]}")
        f = refrun.reference_prim(refrun.final_fields(work, case.name), case.nphases)
        it, t, _ = refrun.info(work, case.name)
        return {"fields": {k: np.asarray(v) for k, v in f.items() if k in ("alpha", "rho", "p", "u", "E")
                           and v is not None}, "t": t, "iterations": it}
    finally:
        shutil.rmtree(work, ignore_errors=True)


@pytest.fixture(scope="module")
def cpu_results():
    from oracle import refrun
    keys = [k for k in LONG if LONG[k][0] == "oracle" or refrun.available()]
    jobs = [(k, False) for k in keys] + [(k, True) for k in keys if _ptmu(k)]
    ex = cf.ProcessPoolExecutor(max_workers=min(len(jobs), max(1, len(os.sched_getaffinity(0)))),
                                mp_context=mp.get_context("spawn"))
    futs = {(k, crl): ex.submit(_cpu_job, k, crl) for k, crl in jobs}
    yield futs
    ex.shutdown(wait=False, cancel_futures=True)


@pytest.mark.gpu
@pytest.mark.parametrize("key", list(LONG))
def test_long_horizon(key, cpu_results, tmp_path):
    kind = LONG[key][0]
    if (key, False) not in cpu_results:
        pytest.skip("reference binary oracle/_ref/ECOGEN not built")
    case = _case(key)
    out = gpu_run(case, tmp_path, steps=case.iterations)
    assert out["stats"]["nonfinite_cells"] == 0
    assert out["stats"]["ptmu_errors"] == 0
    ref = cpu_results[(key, False)].result(timeout=1800)
    env = cpu_results[(key, True)].result(timeout=1800)["fields"] if _ptmu(key) else None
    assert out["iteration"] == ref["iterations"]
    for name, want in ref["fields"].items():
        got = out[name]
        if kind == "reference":
            got = display(got, name)  # the clamps the reference applies when it writes a field
        err = rel_l1(got, want)
        tol = TOL
        if env is not None:  # p-T-mu: the spread of the checker itself under a last-ulp change of ln
            e = rel_l1(display(env[name], name) if kind == "reference" else env[name], want)
            tol = max(TOL, ENVELOPE_FACTOR * e)
        assert err <= tol, f"{key}: {name} rel L1 {err:.3e} after {case.iterations} steps (bound {tol:.3e})"
    if kind == "oracle":
        cpu = cpu_results[(key, True)].result() if _ptmu(key) else None
        for q in ("dt", "t"):
            tol = TOL if cpu is None else max(TOL, ENVELOPE_FACTOR * abs(cpu[q] - ref[q]) / abs(ref[q]))
            assert out[q] == pytest.approx(ref[q], rel=tol), q
    else:  # infoCalcul.out holds t with 6 significant digits
        assert out["t"] == pytest.approx(ref["t"], rel=1e-5)
