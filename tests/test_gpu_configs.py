"""The workloads at their own sizes.

* The small slip-weakening model (160 x 80 x 120 cells, h = 200 m, 8 s = 960 steps):
  the whole run against the oracle, bit for bit in FP32, and the FP32 build against the
  FP64 oracle at the stated accuracy (relative L2 <= 1e-3 on the slip-rate and traction
  histories, final slip <= 1e-4, rupture time within 2 dt).
* The production model (1000 x 400 x 500 cells, 214 M padded): the first 24 steps bit
  for bit against the oracle (histories, stations, wave fields, fault planes), and
  properties that hold at any size -- a run repeated after fd3d_reset is the same bits,
  and the FP64 build of the same kernels agrees with the FP32 build at the stated
  accuracy.
* The rate-and-state model (600 x 300 x 400 cells, 79 M padded, histories every 5
  steps): 50 steps against the oracle within 1e-5 relative L2 (CUDA's and libm's
  exp/log/sinh/asinh differ in the last bits).
* A rate-and-state model that ruptures (48 x 14 x 32 cells, 250 steps): the FP32 build
  against the FP64 oracle at the stated accuracy, rupture time included.
"""
import numpy as np
import pytest

from fd3d_tsn_b200 import configs
from fd3d_tsn_b200.solver import Solver
from oracle.oracle import F64, MIXED, Oracle

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(900)]


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def test_small_model_full_run_bitwise():
    m = configs.sw_small()
    chunk = 96
    m["history_capacity"] = chunk
    steps = m["ntfd"]
    assert steps == 960
    o = Oracle(m, MIXED)
    s = Solver(m)
    for c0 in range(0, steps, chunk):
        n = min(chunk, steps - c0)
        oh, os_ = o.step(n)
        s.run(n)
        s.sync()
        for f in range(4):
            np.testing.assert_array_equal(s.history(f, rec0=c0, nrec=n), oh[:, f], err_msg=f"step {c0} field {f}")
        np.testing.assert_array_equal(s.stations(rec0=c0, nrec=n), os_)
    fo, fg = o.final(), s.final()
    for k in fo:
        np.testing.assert_array_equal(fg[k], fo[k], err_msg=k)
    assert (fo["ruptime"] < 1e4).sum() > 1000, "the small model must rupture"


def test_small_model_fp32_against_fp64_oracle():
    m = configs.sw_small()
    chunk = 96
    m["history_capacity"] = chunk
    steps = m["ntfd"]
    o = Oracle(m, F64)
    s = Solver(m)
    num = np.zeros(4)
    den = np.zeros(4)
    for c0 in range(0, steps, chunk):
        n = min(chunk, steps - c0)
        oh, _ = o.step(n)
        s.run(n)
        s.sync()
        for f in range(4):
            g = s.history(f, rec0=c0, nrec=n)
            num[f] += np.sum((g - oh[:, f]) ** 2)
            den[f] += np.sum(oh[:, f] ** 2)
    assert np.all(np.sqrt(num / den) <= 1e-3), np.sqrt(num / den)
    fo, fg = o.final(), s.final()
    assert rel_l2(fg["slipX"], fo["slipX"]) <= 1e-4
    ruptured = fo["ruptime"] < 1e4
    assert np.all((fg["ruptime"] < 1e4) == ruptured)
    assert np.abs(fg["ruptime"][ruptured] - fo["ruptime"][ruptured]).max() <= 2 * m["dt"]


def test_production_model_bitwise_against_oracle():
    """214 M padded cells, 5 layers, 800 x 400 frictional nodes: the FP32 build against
    the oracle's FP32-field / FP64-accumulator variant over 24 steps, compared one
    array at a time to bound the host memory (each 3-D field is 1.7 GB in FP64)."""
    steps = 24
    m = configs.sw_large(ntfd=steps)
    m["history_capacity"] = steps
    o = Oracle(m, MIXED)
    oh, os_ = o.step(steps)
    s = Solver(m)
    s.run(steps)
    s.sync()
    assert np.abs(oh[:, 0]).max() > 0.1, "the nucleation patch must slip"
    for f in range(4):
        np.testing.assert_array_equal(s.history(f), oh[:, f], err_msg=f"history field {f}")
    np.testing.assert_array_equal(s.stations(), os_)
    del oh
    for name in ("u", "w", "xz", "yy"):
        np.testing.assert_array_equal(s.field(name), o.field(name), err_msg=name)
    for name in ("tx", "tz", "distX", "distZ", "slipX", "slipZ", "ruptime", "rise", "sliptime"):
        np.testing.assert_array_equal(s.plane(name), o.plane(name), err_msg=name)
    s.close()
    o.close()


def test_fvw_medium_against_oracle():
    """600 x 300 x 400 cells, rate-and-state friction, FP64 state and Newton solve at the
    fault, nucleation ramp on, histories every 5 steps: 50 steps against the oracle."""
    steps = 50
    m = configs.fvw_medium(ntfd=steps)
    assert m["history_stride"] == 5
    m["history_capacity"] = steps // 5
    o = Oracle(m, MIXED)
    oh, os_ = o.step(steps)
    s = Solver(m)
    s.run(steps)
    s.sync()
    nrec = steps // 5
    assert s.history_records() == nrec
    ohr = oh[4::5]   # the oracle returns every step; the records are steps 5, 10, ...
    for f in range(5):
        assert rel_l2(s.history(f), ohr[:, f]) <= 1e-5, (f, rel_l2(s.history(f), ohr[:, f]))
    assert rel_l2(s.stations(), os_[4::5]) <= 1e-5
    for name in ("psiX", "psiZ", "slipX", "slipZ", "T0X"):   # T0X carries the nucleation ramp
        assert rel_l2(s.plane(name), o.plane(name)) <= 1e-5, name
    s.close()
    o.close()


def test_fvw_fp32_against_fp64_oracle():
    """Rate-and-state friction, FP32 wave field with the FP64 per-node state and slip-rate
    solve, against the all-FP64 oracle at the stated accuracy: relative L2 <= 1e-3 on the
    slip-rate, traction and state histories, final slip <= 1e-4, and rupture time within
    2 dt on the same set of ruptured nodes."""
    steps = 250
    m = configs.tiny_fvw(nsteps=steps, nxT=48, nzT=32)
    m["history_capacity"] = steps
    o = Oracle(m, F64)
    oh, _ = o.step(steps)
    s = Solver(m)
    s.run(steps)
    s.sync()
    for f in range(5):
        assert rel_l2(s.history(f), oh[:, f]) <= 1e-3, (f, rel_l2(s.history(f), oh[:, f]))
    fo, fg = o.final(), s.final()
    assert rel_l2(fg["slipX"], fo["slipX"]) <= 1e-4
    assert rel_l2(fg["slipZ"], fo["slipZ"]) <= 1e-4
    ruptured = fo["ruptime"] < 1e4
    assert ruptured.sum() > 100, "the model must rupture beyond its nucleation"
    assert np.all((fg["ruptime"] < 1e4) == ruptured)
    assert np.abs(fg["ruptime"][ruptured] - fo["ruptime"][ruptured]).max() <= 2 * m["dt"]
    s.close()


def test_production_model_repeatable_and_fp64_consistent():
    steps = 40
    m = configs.sw_large(ntfd=steps)
    m["history_capacity"] = steps
    s = Solver(m)
    s.run(steps)
    s.sync()
    h1 = np.stack([s.history(f, real_kind=4) for f in range(4)])
    fin1 = s.final()
    assert np.abs(h1[0]).max() > 0.1, "the nucleation patch must slip"
    s.reset()
    s.run(steps)
    s.sync()
    np.testing.assert_array_equal(np.stack([s.history(f, real_kind=4) for f in range(4)]), h1)
    for k, v in s.final().items():
        np.testing.assert_array_equal(v, fin1[k], err_msg=k)
    s.close()
    d = Solver(dict(m, precision="f64"))
    d.run(steps)
    d.sync()
    for f in range(4):
        assert rel_l2(h1[f], d.history(f)) <= 1e-3, f
    assert rel_l2(fin1["slipX"], d.final()["slipX"]) <= 1e-4
    d.close()
