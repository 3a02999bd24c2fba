"""The FSPACE build (fspace = 1) on the GPU against the oracle, through the C ABI.

FSPACE replaces the free surface by a fifth PML strip of nabc cells above the model
(nfs = nabc, fd3d_init.f90:161-165): pml_uvw/pml_xyz gain the top strip
(fd3d_deriv.f90:2223-2293, 2996-3143), fuvw and fres are not called, the top fault row
takes the interior traction formula and the xz/yz split components are not zeroed at
the strips' top rows.  The slip-weakening path stays bit-identical to the oracle.
"""
import numpy as np
import pytest

from fd3d_tsn_b200 import configs
from fd3d_tsn_b200.batch import Batch
from fd3d_tsn_b200.solver import Solver
from oracle.oracle import F64, MIXED, Oracle

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "xx", "yy", "zz", "xy", "yz", "xz")
PLANES = ("tx", "tz", "slipX", "slipZ", "ruptime", "rise", "sliptime", "distX", "distZ")


def model(precision="f32", nsteps=90, **kw):
    m = configs.tiny_sw(seed=31, nsteps=nsteps, precision=precision, fspace=True, **kw)
    m["history_capacity"] = nsteps
    return m


@pytest.mark.parametrize("precision,variant", [("f32", MIXED), ("f64", F64)])
def test_fspace_bitwise(precision, variant):
    m = model(precision)
    assert m["nfs"] == m["nabc"]
    o = Oracle(m, variant)
    oh, os_ = o.step(90)
    s = Solver(m)
    s.run(90)
    s.sync()
    assert np.abs(oh[:, 0]).max() > 0.1, "the model must rupture"
    for f in range(4):
        np.testing.assert_array_equal(s.history(f), oh[:, f], err_msg=f"history field {f}")
    np.testing.assert_array_equal(s.stations(), os_)
    for name in FIELDS:
        np.testing.assert_array_equal(s.field(name), o.field(name), err_msg=name)
    for name in PLANES:
        np.testing.assert_array_equal(s.plane(name), o.plane(name), err_msg=name)
    # the top strip is live: waves reached it and were damped there, not reflected
    ks = m["nzt"] - m["nfs"]
    assert np.abs(s.field("u")[:, :, ks + 1:]).max() > 0
    s.close()


def test_fspace_layered_and_heterogeneous_media_bitwise():
    """Both interior sweep variants (profile table for the layered medium, 3-D arrays
    for a perturbed one) next to the top strip."""
    lay = configs.layered(np.random.default_rng(41), 3, 40 * 200.0)
    m = model(nsteps=50, layers=lay)
    lam, mu, d = configs.medium_3d(m)
    rng = np.random.default_rng(5)
    pert = tuple(np.asfortranarray(a * (1.0 + 0.05 * rng.uniform(-1.0, 1.0, a.shape))) for a in (lam, mu, d))
    for arrays in (tuple(np.asfortranarray(a) for a in (lam, mu, d)), pert):
        o = Oracle(m, MIXED)
        o.set_medium_arrays(*arrays)
        oh, _ = o.step(50)
        s = Solver(m)
        s.upload_medium_arrays(*arrays, real_kind=8)
        s.run(50)
        s.sync()
        np.testing.assert_array_equal(np.stack([s.history(f) for f in range(4)], axis=1), oh[:, :4])
        for name in ("u", "w", "xx", "xz", "yz"):
            np.testing.assert_array_equal(s.field(name), o.field(name), err_msg=name)
        s.close()
        o.close()


@pytest.mark.parametrize("schedule", ["graph", "persistent"])
def test_fspace_model_in_a_batch(schedule):
    """An FSPACE model next to free-surface models in one batch: the same bits as alone."""
    steps = 30
    ms = [model(nsteps=steps), configs.tiny_sw(seed=32, nsteps=steps), model(nsteps=steps, nxT=36, nzT=24)]
    for q in ms:
        q["history_capacity"] = steps
    b = Batch(1 << 30, 8)
    b.set_schedule(schedule)
    slots = [b.add(q) for q in ms]
    b.run(steps)
    b.sync()
    for q, slot in zip(ms, slots):
        s = Solver(q)
        s.run(steps)
        s.sync()
        fb, fs = b.final(slot), s.final()
        for k in fb:
            np.testing.assert_array_equal(fb[k], fs[k], err_msg=k)
        np.testing.assert_array_equal(b.history(slot, 0, 0, steps), s.history(0, 0, steps))
        s.close()


@pytest.mark.parametrize("precision,variant,tol", [("f32", MIXED, 1e-5), ("f64", F64, 1e-9)])
def test_fspace_fvw_matches_oracle(precision, variant, tol):
    """Rate-and-state friction with the top PML strip (the fault reaches the top row)."""
    m = configs.tiny_fvw(nsteps=60, precision=precision, fspace=True)
    o = Oracle(m, variant)
    oh, _ = o.step(60)
    s = Solver(m)
    s.run(60)
    s.sync()
    assert np.abs(oh[:, 0]).max() > 1e-3
    for f in range(5):
        g = s.history(f)
        assert np.linalg.norm(g - oh[:, f]) <= tol * max(np.linalg.norm(oh[:, f]), 1e-30), f
    s.close()
