"""fd3d_run_noalloc against fd3d_run, through the C ABI.

fd3d_run_noalloc is for hosts that cannot let the library allocate device memory once
their run has started, for instance a Fortran host whose device arrays belong to the
OpenACC runtime, or a service that reserved its HBM up front.  It runs the fault
boundary condition as separate launches whose scratch comes from a fixed device array
of the library instead of memory the library allocates.  Its results must equal
fd3d_run's (whose fused fault-boundary kernel keeps that scratch in shared memory) bit
for bit, over two calls in a row.

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from fd3d_tsn_b200 import configs
from fd3d_tsn_b200.solver import Solver, lib

pytestmark = pytest.mark.gpu


def _noalloc(s, n):
    fn = lib().fd3d_run_noalloc
    fn.argtypes = [C.c_void_p, C.c_int]
    fn.restype = C.c_int
    return fn(s.h, int(n))


@pytest.mark.parametrize("maker,prec", [(configs.tiny_sw, "f32"), (configs.tiny_sw, "f64"),
                                        (configs.tiny_fvw, "f32")])
def test_noalloc_equals_run_two_calls(maker, prec):
    m = maker(nsteps=40, precision=prec)
    ref = Solver(m)
    new = Solver(m)
    for call in range(2):
        ref.run(20)
        ref.sync()
        assert _noalloc(new, 20) == 0
        new.sync()
        n = ref.history_records()
        assert new.history_records() == n == 20 * (call + 1)
        for f in range(ref.nf):
            np.testing.assert_array_equal(new.history(f), ref.history(f), err_msg=f"call {call} field {f}")
        for name in ("u", "w", "xz"):
            np.testing.assert_array_equal(new.field(name), ref.field(name), err_msg=f"call {call} {name}")
        for name in ("tx", "tz", "slipX", "ruptime"):
            np.testing.assert_array_equal(new.plane(name), ref.plane(name), err_msg=f"call {call} {name}")


def test_noalloc_rejects_planes_over_the_limit():
    # nxt*nzt = 1120*1012 > 2^20 fault-plane nodes
    m = configs.tiny_sw(nxT=1100, nyT=4, nzT=1000, nsteps=1, nstations=0)
    s = Solver(m)
    assert _noalloc(s, 1) == -1
    assert s.steps_done() == 0


def test_noalloc_leaves_device_memory_unchanged():
    """A call after set-up allocates no device memory: the device's free memory is the same
    before and after it (measured around the second call, after the first has loaded the
    kernels it launches), and fd3d_run afterwards still agrees with a context that only
    ever ran fd3d_run."""
    import torch
    m = configs.tiny_sw(nsteps=60)
    ref = Solver(m)
    new = Solver(m)
    assert _noalloc(new, 20) == 0
    new.sync()
    torch.cuda.mem_get_info(0)      # the first query sets up the caller's view of the device
    free0, _ = torch.cuda.mem_get_info(0)
    assert _noalloc(new, 20) == 0
    new.sync()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)
    new.run(20)
    new.sync()
    ref.run(60)
    ref.sync()
    for f in range(ref.nf):
        np.testing.assert_array_equal(new.history(f), ref.history(f), err_msg=f"field {f}")
    for name in ("tx", "tz", "slipX", "distX", "ruptime"):
        np.testing.assert_array_equal(new.plane(name), ref.plane(name), err_msg=name)
