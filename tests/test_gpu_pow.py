"""The table-driven pow and log of the step kernels (ecogen_b200/csrc/ecg_pow.cuh) on the GPU equal the same
source built for the host bit for bit (the host build is checked against glibc and 300-bit arithmetic in
tests/test_pow.py).  The device values come from the probe library (ecogen_b200/libecg_probe.so,
ecg_probe_epow)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROBE = os.path.join(ROOT, "ecogen_b200", "libecg_probe.so")
P = C.POINTER(C.c_double)

pytestmark = pytest.mark.gpu


def test_device_epow_equals_host_build(tmp_path):
    if not os.path.exists(PROBE):
        pytest.fail(f"{PROBE} is missing: build it with python -m ecogen_b200.build")
    so = str(tmp_path / "pow_host.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-o", so,
                    os.path.join(ROOT, "tests", "pow", "pow_host.cpp")], check=True)
    host = C.CDLL(so)
    host.host_epow.argtypes = [P, P, P, C.c_long]
    dev = C.CDLL(PROBE)
    dev.ecg_probe_epow.argtypes = [P, P, P, C.c_long]
    dev.ecg_probe_epow.restype = C.c_int
    rng = np.random.default_rng(2024)
    parts = [np.exp(rng.uniform(np.log(lo), np.log(hi), 1 << 20))
             for lo, hi in ((0.996, 1.0), (0.999, 1.001), (0.9, 1.1), (0.2, 5.0), (1e-17, 1e17))]
    x = np.concatenate(parts + [np.array([0.0, -0.0, -2.0, np.inf, np.nan, 1.0, 0.5, 2.0])])
    y = rng.choice([4.4, 1.4, 1.67, 2.35, 1.43, 7.15], size=x.size)
    a = np.empty_like(x)
    b = np.empty_like(x)
    assert dev.ecg_probe_epow(x.ctypes.data_as(P), y.ctypes.data_as(P), a.ctypes.data_as(P), x.size) == 0
    host.host_epow(x.ctypes.data_as(P), y.ctypes.data_as(P), b.ctypes.data_as(P), x.size)
    same = (a.view(np.int64) == b.view(np.int64)) | (np.isnan(a) & np.isnan(b))
    assert same.all(), f"{np.count_nonzero(~same)} of {x.size} device values differ from the host build"


def test_device_elog_equals_host_build(tmp_path):
    if not os.path.exists(PROBE):
        pytest.fail(f"{PROBE} is missing: build it with python -m ecogen_b200.build")
    so = str(tmp_path / "pow_host.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-o", so,
                    os.path.join(ROOT, "tests", "pow", "pow_host.cpp")], check=True)
    host = C.CDLL(so)
    host.host_elog.argtypes = [P, P, C.c_long]
    dev = C.CDLL(PROBE)
    dev.ecg_probe_elog.argtypes = [P, P, C.c_long]
    dev.ecg_probe_elog.restype = C.c_int
    rng = np.random.default_rng(77)
    x = np.concatenate([np.exp(rng.uniform(np.log(lo), np.log(hi), 1 << 20))
                        for lo, hi in ((50.0, 2000.0), (1e3, 1e10), (0.5, 2.0), (1e-300, 1e300))] +
                       [np.array([0.0, -1.0, np.inf, np.nan, 1.0, 2.0])])
    a = np.empty_like(x)
    b = np.empty_like(x)
    assert dev.ecg_probe_elog(x.ctypes.data_as(P), a.ctypes.data_as(P), x.size) == 0
    host.host_elog(x.ctypes.data_as(P), b.ctypes.data_as(P), x.size)
    same = (a.view(np.int64) == b.view(np.int64)) | (np.isnan(a) & np.isnan(b))
    assert same.all(), f"{np.count_nonzero(~same)} of {x.size} device values differ from the host build"
