"""Grid shapes away from the workloads' (PML thickness nabc, sizes that fill no tile, the
FSPACE strip on an odd grid, a strided history ring that wraps): the FP32 build against
the oracle, bit for bit, fields and histories."""
import numpy as np
import pytest

from fd3d_tsn_b200 import configs
from fd3d_tsn_b200.solver import Solver
from oracle.oracle import MIXED, Oracle

pytestmark = pytest.mark.gpu

CASES = [
    dict(nabc=4, nxT=33, nyT=9, nzT=17),
    dict(nabc=7, nxT=45, nyT=12, nzT=21),
    dict(nabc=13, nxT=30, nyT=10, nzT=19),
    dict(nabc=6, nxT=35, nyT=11, nzT=18, fspace=True),
    dict(nabc=10, nxT=65, nyT=9, nzT=33, stride=3),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_edge_grid_bitwise(case):
    steps = 45
    m = configs.tiny_sw(seed=23, nsteps=steps, **case)
    stride = case.get("stride", 1)
    m["history_capacity"] = 7 if stride > 1 else steps  # wraps when strided
    o = Oracle(m, MIXED)
    oh, os_ = o.step(steps)
    s = Solver(m)
    s.run(steps)
    s.sync()
    assert np.abs(oh[:, 0]).max() > 0.05, "the model must slip"
    nrec = steps // stride
    keep = min(nrec, m["history_capacity"])
    recs = [stride * (r + 1) - 1 for r in range(nrec - keep, nrec)]
    for f in range(4):
        np.testing.assert_array_equal(s.history(f, rec0=nrec - keep, nrec=keep), oh[recs, f], err_msg=f"field {f}")
    for name in ("u", "v", "w", "xx", "yy", "zz", "xy", "yz", "xz"):
        np.testing.assert_array_equal(s.field(name), o.field(name), err_msg=name)
    fo, fg = o.final(), s.final()
    for k in fo:
        np.testing.assert_array_equal(fg[k], fo[k], err_msg=k)
    s.close()
