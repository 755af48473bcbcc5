"""Shared helpers of the test-suite: run a case on the GPU through the C ABI."""
import os
import shutil

import numpy as np

from ecogen_b200 import api, cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def write_case(case, tmp):
    d = case.write(str(tmp))
    return d, os.path.join(str(tmp), "libEOS")


def gpu_run(case, tmp, steps=None, mode="auto"):
    """Read the case from its XML files, fill, upload, advance, download (all through the C ABI)."""
    d, eosdir = write_case(case, tmp)
    inp = api.Input(d, eosdir)
    ctx = api.Context(inp.case)
    ctx.upload(inp.fill())
    if steps is not None:
        st = ctx.step(steps)
    elif mode == "auto":
        st = ctx.run()
    out = ctx.download_dict()
    out["stats"] = st.as_dict()
    out["t"] = ctx.t.value
    out["dt"] = ctx.dt.value
    out["iteration"] = ctx.iteration
    ctx.close()
    return out
