"""Failure detection without a GPU fault: the device waits of the library are bounded.
A wait that nothing completes (an mbarrier phase without an arrival, a grid barrier one
CTA never reaches) gives up after its bound, records the timeout bit in the status word,
and the context that runs next still computes the oracle's results."""
import ctypes as C
import time

import numpy as np
import pytest

from fd3d_tsn_b200 import configs
from fd3d_tsn_b200.solver import Solver, lib
from oracle.oracle import MIXED, Oracle

pytestmark = pytest.mark.gpu

ST_TIMEOUT = 4


def test_bounded_waits_give_up_and_device_stays_usable():
    mb, gb = C.c_int(-1), C.c_int(-1)
    t0 = time.perf_counter()
    assert lib().fd3d_check_waits(C.byref(mb), C.byref(gb)) == 0
    elapsed = time.perf_counter() - t0
    assert mb.value == ST_TIMEOUT and gb.value == ST_TIMEOUT
    assert elapsed < 60.0
    m = configs.tiny_sw(nsteps=20)
    oh, _ = Oracle(m, MIXED).step(20)
    s = Solver(m)
    s.run(20)
    s.sync()
    np.testing.assert_array_equal(s.history(0), oh[:, 0])
    s.close()
