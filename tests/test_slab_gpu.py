"""One model over several contexts (z-slabs) against the same model in one context.

The slabs of a model update disjoint planes and exchange two halo planes (or
fault-plane rows) after each phase of a step, so every cell update reads the same
values as in one context: the merged histories, stations, wave fields and fault planes
must be the same bits.  All slabs run on one GPU here (each a context with its own
stream; the exchange is stream-ordered, nothing spins), which is the same code path as
slabs on several GPUs with the copies crossing NVLink.  The slab boundaries fall inside
the z-low PML strip, on its top plane and in the interior, and the top slab owns the
free surface or the FSPACE strip.
"""
import numpy as np
import pytest

from fd3d_tsn_b200 import abi, configs
from fd3d_tsn_b200.slab import SlabSolver, plan
from fd3d_tsn_b200.solver import Solver

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "xx", "yy", "zz", "xy", "yz", "xz")
PLANES = ("tx", "tz", "slipX", "slipZ", "ruptime", "rise", "sliptime", "distX", "distZ")


def compare(m, steps, ranges=None, nslabs=2, chunks=(None,), medium3d=False, fvw=False):
    m["history_capacity"] = steps
    ref = Solver(m, medium3d=medium3d)
    sl = SlabSolver(m, nslabs=nslabs, ranges=ranges, medium3d=medium3d)
    done = 0
    for c in chunks:
        n = steps - done if c is None else c
        ref.run(n)
        sl.run(n)
        done += n
    ref.sync()
    sl.sync()
    assert sl.steps_done() == steps
    assert np.abs(ref.history(0)).max() > 0.05, "the model must slip"
    for f in range(ref.nf):
        np.testing.assert_array_equal(sl.history(f), ref.history(f), err_msg=f"history field {f}")
    np.testing.assert_array_equal(sl.stations(), ref.stations())
    for name in FIELDS:
        np.testing.assert_array_equal(sl.field(name), ref.field(name), err_msg=name)
    planes = PLANES + (("psiX", "psiZ", "T0X") if fvw else ())
    for name in planes:
        np.testing.assert_array_equal(sl.plane(name), ref.plane(name), err_msg=name)
    fr, fs = ref.final(), sl.final()
    for k in fr:
        np.testing.assert_array_equal(fs[k], fr[k], err_msg=k)
    ref.close()
    sl.close()


@pytest.mark.parametrize("nslabs", [2, 3, 4])
def test_slabs_match_one_context_sw(nslabs):
    m = configs.tiny_sw(seed=71, nsteps=120)
    rng = plan(m, nslabs)
    assert rng[0][0] == 1 and rng[-1][1] == m["nzt"] and len(rng) == nslabs
    compare(m, 120, nslabs=nslabs, chunks=(37, 64, None))


def test_slab_boundaries_at_the_pml_and_fault_edges():
    """A slab of z-PML planes only (1 .. nabc-1), one that starts on the strip's top plane
    (nabc) and holds the lowest fault rows, and a top slab that starts 12 planes down."""
    m = configs.tiny_sw(seed=72, nsteps=80)
    nab, nzt = m["nabc"], m["nzt"]
    ranges = [(1, nab - 1), (nab, nab + 5), (nab + 6, nzt - 12), (nzt - 11, nzt)]
    compare(m, 80, ranges=ranges)


def test_slabs_match_one_context_fvw_with_nucleation():
    m = configs.tiny_fvw(seed=73, nsteps=100)
    compare(m, 100, nslabs=3, fvw=True)


def test_slabs_match_one_context_fspace():
    m = configs.tiny_sw(seed=74, nsteps=90, fspace=True)
    compare(m, 90, nslabs=3)


def test_slabs_match_one_context_3d_medium_fp64():
    m = configs.tiny_sw(seed=75, nsteps=60, precision="f64")
    compare(m, 60, nslabs=2, medium3d=True)


def test_slabs_history_stride_and_wrapping_ring():
    """Records every 3 steps into a ring of 8 records, read back in chunks as the run goes:
    the merged records are the same bits as one context's."""
    m = configs.tiny_sw(seed=77, nsteps=96, stride=3)
    m["history_capacity"] = 8
    ref = Solver(m)
    sl = SlabSolver(m, nslabs=3)
    for c in range(4):
        ref.run(24)
        sl.run(24)
        ref.sync()
        sl.sync()
        rec0 = 8 * c        # 24 steps = 8 records per chunk, all still in the ring
        for f in range(ref.nf):
            np.testing.assert_array_equal(sl.history(f, rec0=rec0, nrec=8), ref.history(f, rec0=rec0, nrec=8),
                                          err_msg=f"chunk {c} field {f}")
        np.testing.assert_array_equal(sl.stations(rec0=rec0, nrec=8), ref.stations(rec0=rec0, nrec=8))
    assert sl.history_records() == ref.history_records() == 32
    ref.close()
    sl.close()


def test_slab_context_refuses_whole_model_calls():
    m = configs.tiny_sw(seed=76, nsteps=10)
    (a, b), _ = plan(m, 2)
    s = Solver(m, slab=(a, b))
    with pytest.raises(abi.Fd3dError):
        s.run(1)            # a slab steps in its group only
    with pytest.raises(abi.Fd3dError):
        s.post_process()    # sums over the whole fault plane
    s.close()
