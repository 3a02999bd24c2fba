"""The PML kernels' quotient by a divisor known before the launch (dh, 1 + omega) is
the IEEE quotient for every float dividend: fd3d_check_division compares the two on
all 2^32 bit patterns per divisor on the GPU."""
import ctypes as C

import numpy as np
import pytest

from fd3d_tsn_b200 import abi, configs
from fd3d_tsn_b200.solver import lib

pytestmark = pytest.mark.gpu


def pml_divisors(m):
    """1 + omega for every profile value of init_pml (fd3d_deriv.f90:1319-1493), in FP32
    with the reference's operation order."""
    f = np.float32
    dt, dh, nabc = f(m["dt"]), f(m["dh"]), m["nabc"]
    omega_m = f(m["pml_fact"]) * f(m["pml_vp"]) / (f(2) * dh * f(nabc - 1))
    n = nabc - 1
    out = set()
    for i in range(1, n + 1):
        r, rm = f(i) / f(n), (f(i) - f(0.5)) / f(n)
        for q in (r, rm):
            om = f(0.5) * dt * omega_m * ((q * q) * (q * q))
            out.add(float(f(1) + om))
    return sorted(out)


def test_division_matches_ieee_on_every_dividend(gpu_available):
    if not gpu_available:
        pytest.skip("no CUDA device")
    divs = set()
    for m in (configs.sw_small(), configs.sw_large(), configs.fvw_medium(), configs.tiny_sw()):
        divs.add(float(np.float32(m["dh"])))
        divs.update(pml_divisors(m))
    rng = np.random.default_rng(7)
    # significands near 1, sqrt 2 and 2, powers of two, both ends of the fast range
    extra = [1.0, 2.0, 0.5, 1.0000001, 1.4142135, 1.9999999, 1.99999988, 3.0, 7.0, 1e-6, 2.0 ** -20,
             2.0 ** 20, 1e6, 2.0 ** 21, 2.0 ** -21, 12.5, 37.5,
             -3.0, -1.0, 0.0]   # outside the checked range: every quotient by the FP64 path
    divs.update(float(np.float32(x)) for x in extra)
    divs.update(float(np.float32(x)) for x in rng.uniform(1.0, 2.0, 8))
    divs = sorted(divs)
    arr = (C.c_float * len(divs))(*divs)
    bad = (C.c_ulonglong * len(divs))()
    first = (C.c_uint * len(divs))()
    rc = lib().fd3d_check_division(arr, len(divs), bad, first)
    assert rc == 0, abi.ERRORS.get(rc, rc)
    failures = {d: (bad[k], hex(first[k])) for k, d in enumerate(divs) if bad[k]}
    assert not failures, failures
