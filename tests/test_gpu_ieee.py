"""The step kernels' branch-free division and square root (ecogen_b200/csrc/ecg_ieee.cuh) against
CUDA's correctly rounded `/` and `sqrt()`, bit for bit.

The step kernels divide with ecg::ddiv and take square roots with ecg::dsqrt: straight-line
Newton-Markstein sequences that return the IEEE round-to-nearest result without the branch CUDA's own
sequence takes for operands it cannot handle.  The check runs in the probe library
(ecogen_b200/libecg_probe.so, ecg_probe_ieee_check) over hashed operands of random significand, sign
and exponent, with exact quotients, all-ones-significand divisors and zero / infinite / NaN operands
mixed in.  Parity of the step itself is covered by every parity test, which compares the kernels'
fields with the oracle (host IEEE division).
"""
import ctypes as C
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROBE = os.path.join(ROOT, "ecogen_b200", "libecg_probe.so")

pytestmark = pytest.mark.gpu


def _lib():
    if not os.path.exists(PROBE):
        pytest.fail(f"{PROBE} is missing: build it with python -m ecogen_b200.build")
    lib = C.CDLL(PROBE)
    lib.ecg_probe_ieee_check.argtypes = [C.c_ulonglong, C.c_int, C.c_int, C.c_int, C.c_int,
                                         C.POINTER(C.c_ulonglong)]
    lib.ecg_probe_ieee_check.restype = C.c_int
    return lib


@pytest.mark.parametrize("emin,emax", [(0, 0), (-4, 4), (-60, 60), (-500, 500)])
def test_division_and_sqrt_equal_cuda_bit_for_bit(emin, emax):
    lib = _lib()
    counts = (C.c_ulonglong * 3)()
    rc = lib.ecg_probe_ieee_check(0x5EED0000 + emax, emin, emax, 148 * 8, 256, counts)
    assert rc == 0, f"probe returned {rc}"
    checked, bad_div, bad_sqrt = counts[0], counts[1], counts[2]
    assert checked == 148 * 8 * 256 * 256
    assert bad_div == 0, f"{bad_div} of {checked} divisions differ from CUDA's a / b"
    assert bad_sqrt == 0, f"{bad_sqrt} of {checked} square roots differ from CUDA's sqrt"


def test_check_refuses_exponents_outside_the_normal_range():
    lib = _lib()
    counts = (C.c_ulonglong * 3)()
    assert lib.ecg_probe_ieee_check(1, -600, 0, 1, 1, counts) == -1
    assert lib.ecg_probe_ieee_check(1, 0, 0, 0, 1, counts) == -1
