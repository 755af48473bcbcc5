"""CPU-side checks of the benchmark script.

* Every name a function of bench.py (or __graft_entry__.py) reads resolves: a local, an enclosing
  function's, a module-level name or a builtin.  A name left over from an edit would otherwise surface
  only on the GPU box, in the bench line of one workload.
* The reference arm (`bench.py --impl reference`, the reference's own CPU solver timed on the host
  cores) prints one JSON line with the keys of the bench contract, or its `unavailable` line when the
  reference binary is not built.
"""
import builtins
import json
import os
import subprocess
import sys
import symtable

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _unresolved(path):
    src = open(path).read()
    top = symtable.symtable(src, path, "exec")
    module_names = {s.get_name() for s in top.get_symbols() if s.is_assigned() or s.is_imported()}
    module_names |= {c.get_name() for c in top.get_children()}
    bad = []

    def walk(table):
        for sym in table.get_symbols():
            # an implicit global: read in this scope, bound in no enclosing function
            if sym.is_referenced() and sym.is_global() and not sym.is_declared_global():
                name = sym.get_name()
                if name not in module_names and not hasattr(builtins, name):
                    bad.append(f"{table.get_name()}: {name}")
        for child in table.get_children():
            walk(child)

    for child in top.get_children():
        walk(child)
    return bad


@pytest.mark.parametrize("name", ["bench.py", "__graft_entry__.py"])
def test_every_name_resolves(name):
    assert _unresolved(os.path.join(ROOT, name)) == []


def test_reference_arm_prints_the_contract_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--config", "c1", "--steps", "1",
                        "--warmup", "0"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    if "unavailable" in line:
        pytest.skip(line["unavailable"])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling", "dtype",
                "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["value"] > 0 and line["higher_is_better"] is True
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
