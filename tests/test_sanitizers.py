"""Host code under AddressSanitizer and UndefinedBehaviorSanitizer (CPU only).

The reference builds with -Wall -Wextra only (its Makefile); this build checks the host side of its
own C ABI and its oracle with the sanitizers: any out-of-bounds access, use after free, leak, signed
overflow, misaligned load or other undefined behaviour aborts the harness, and the test fails.

* tests/sanitize/host_harness.cpp links the host translation units that need no GPU -- the XML
  reader (ecg_xml.cpp), the case reader, initial fill and restart fill (ecg_input.cpp), the case checks
  (ecg_case.cpp) -- and runs them over every golden case folder (1D to 3D, Kapila, Euler, PTUEq, walls,
  THINC, transports, p-T-mu, stretched meshes) and over malformed folders that must be refused.  The
  filled fields must equal the regular build's, bit for bit.
* tests/sanitize/oracle_harness.c runs the oracle (oracle/ecg_oracle.c) for a few steps of small cases
  of each physics family; the result must equal the regular oracle build's.
"""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from ecogen_b200 import api, cases
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "ecogen_b200", "csrc")
SAN = ["-fsanitize=address,undefined", "-fno-sanitize-recover=all", "-fno-omit-frame-pointer", "-g", "-O1"]
ENV = dict(os.environ, ASAN_OPTIONS="abort_on_error=0:halt_on_error=1:detect_leaks=1",
           UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1")


@pytest.fixture(scope="module")
def harnesses():
    if not shutil.which("g++") or not shutil.which("gcc"):
        pytest.skip("no host compiler")
    out = tempfile.mkdtemp(prefix="ecg_san_")
    host = os.path.join(out, "host_harness")
    cmd = ["g++", "-std=c++17", "-ffp-contract=off"] + SAN + ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
                                                               os.path.join(ROOT, "tests", "sanitize", "host_harness.cpp"),
                                                               os.path.join(CSRC, "ecg_input.cpp"),
                                                               os.path.join(CSRC, "ecg_xml.cpp"),
                                                               os.path.join(CSRC, "ecg_case.cpp"), "-o", host]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    orc = os.path.join(out, "oracle_harness")
    cmd = ["gcc", "-std=c11", "-ffp-contract=off"] + SAN + ["-I" + os.path.join(ROOT, "oracle"),
                                                            os.path.join(ROOT, "tests", "sanitize", "oracle_harness.c"),
                                                            os.path.join(ROOT, "oracle", "ecg_oracle.c"), "-lm", "-o", orc]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    yield {"host": host, "oracle": orc, "dir": out}
    shutil.rmtree(out, ignore_errors=True)


def _run(exe, *args):
    r = subprocess.run([exe, *args], capture_output=True, text=True, env=ENV, timeout=600)
    assert "Sanitizer" not in r.stderr and "runtime error" not in r.stderr, r.stderr[-4000:]
    return r


def test_case_input_under_sanitizers(harnesses, golden_cases, tmp_path):
    for key, case in golden_cases.items():
        d = case.write(str(tmp_path / key))
        eos = os.path.join(str(tmp_path / key), "libEOS")
        out = str(tmp_path / f"{key}.bin")
        r = _run(harnesses["host"], "ok", d, eos, out)
        assert r.returncode == 0 and r.stdout.startswith("ok"), (key, r.stdout, r.stderr[-2000:])
        inp = api.Input(d, eos)
        assert int(r.stdout.split()[1]) == inp.ncells, key
        got = np.fromfile(out, dtype=np.float64)
        assert np.array_equal(got, np.concatenate(inp.fill())), key  # the regular build's fill, bit for bit
        if key in ("bubble2d_o2", "ptueq_bubble2d_o2", "euler2d_o1", "bubble2d_stretch_o2"):
            r = _run(harnesses["host"], "restart", d, eos, out)
            assert r.returncode == 0 and r.stdout.startswith("ok"), (key, r.stdout)


def _break(case_dir, name, old, new):
    p = os.path.join(case_dir, name)
    with open(p) as f:
        txt = f.read()
    assert old in txt, (name, old)
    with open(p, "w") as f:
        f.write(txt.replace(old, new))


def test_malformed_input_refused_under_sanitizers(harnesses, tmp_path):
    """Malformed XML (truncated files, missing elements and attributes, bad values) is refused with a
    status, not a crash -- the reference's own error cases (nonreg/nonregTests/errors) included."""
    base = cases.shock_bubble_2d(n=8, iterations=2, name="broken")
    stretched = cases.shock_tube_1d(ncells=40, iterations=2, name="brokenStretch")
    stretched.stretch = {"x": [(0.0, 0.5, 1.0, 20), (0.5, 1.0, 1.05, 20)]}
    edits = [
        ("mesh.xml", '<numberCells x="8"', '<numberCells x="1"'),
        ("mesh.xml", "<dimensions", "<dimension"),
        ("main.xml", "<computationControl", "<computationContro"),
        ("model.xml", 'name="PressureVelocityEq"', 'name="NoSuchModel"'),
        ("model.xml", "</model>", ""),
        ("initialConditions.xml", "</CI>", "<physicalDomains>"),
        ("mesh.xml", 'structure="cartesian"', 'structure="unStructured"'),
    ]
    for i, (name, old, new) in enumerate(edits):
        d = base.write(str(tmp_path / f"b{i}"))
        _break(d, name, old, new)
        r = _run(harnesses["host"], "refuse", d, os.path.join(str(tmp_path / f"b{i}"), "libEOS"))
        assert r.returncode == 0, (name, old, r.stdout, r.stderr[-2000:])
    for i, (old, new) in enumerate([('endAt="0.5"', 'endAt="0.4"'), ('startAt="0.0"', 'startAt="0.1"'),
                                    ('endAt="1.0"', 'endAt="0.9"')]):
        d = stretched.write(str(tmp_path / f"s{i}"))
        _break(d, "mesh.xml", old, new)
        r = _run(harnesses["host"], "refuse", d, os.path.join(str(tmp_path / f"s{i}"), "libEOS"))
        assert r.returncode == 0, (old, r.stdout, r.stderr[-2000:])


def _blob(case, path):
    c = oracle.make_case(case)
    f = oracle.initial_fields(case)
    n = case.ncells
    with open(path, "wb") as fh:
        fh.write(bytes(c))
        fh.write(np.int64(n).tobytes())
        for name in ("alpha", "rho", "p", "u"):
            fh.write(np.ascontiguousarray(f[name], dtype=np.float64).tobytes())


SAN_CASES = {
    "bubble2d_walls": lambda: _walls(cases.shock_bubble_2d(n=14, iterations=3, name="sanBubble")),
    "cavity3d": lambda: cases.cavity_collapse_3d(n=8, iterations=2, ninclusions=3, radius_cells=(1.5, 2.5)),
    "expansion_ptmu": lambda: cases.expansion_tube_2d(n=12, iterations=3),
    "tube_stretched": lambda: _stretch(cases.shock_tube_1d(ncells=50, iterations=5, order="vanleer")),
}


def _walls(c):
    c.boundaries = ["wall", "nonReflecting", "symmetry", "nonReflecting"]
    return c


def _stretch(c):
    c.stretch = {"x": [(0.0, 0.6, 1.0, 30), (0.6, 1.0, 1.05, 20)]}
    return c


@pytest.mark.parametrize("key", list(SAN_CASES))
def test_oracle_under_sanitizers(harnesses, key, tmp_path):
    case = SAN_CASES[key]()
    blob = str(tmp_path / "case.bin")
    _blob(case, blob)
    steps = case.iterations
    r = _run(harnesses["oracle"], blob, str(steps))
    assert r.returncode == 0, r.stderr[-3000:]
    total, dt = (float(v) for v in r.stdout.split())  # sums in another order than numpy's: approx
    sim = oracle.Sim(case)
    sim.step(steps)
    o = sim.fields()
    ref = float(np.sum(o["alpha"]) + np.sum(o["rho"]) + np.sum(o["p"]) + np.sum(o["E"]) + np.sum(o["u"]))
    assert total == pytest.approx(ref, rel=1e-14)
    assert dt == sim.dt.value
