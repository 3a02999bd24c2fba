"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

* FP32 build vs the oracle's FP32-field/FP64-accumulator variant and FP64 build vs
  the oracle's FP64 variant: same operations in the same order, so slip-weakening
  runs agree to the last bit; FVW runs (CUDA vs libm transcendentals) agree within
  1e-5 (FP32) / 1e-9 (FP64) relative L2.
* FP32 build vs the FP64 oracle at the stated accuracy: relative L2 <= 1e-3 on the
  slip-rate and traction histories, final slip <= 1e-4 (relative L2), rupture time
  within 2*dt.
"""
import os

import numpy as np
import pytest

from fd3d_tsn_b200 import configs
from fd3d_tsn_b200.abi import Fd3dError
from fd3d_tsn_b200.solver import Solver
from oracle.oracle import F64, MIXED, Oracle

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def run_both(model, nsteps, variant):
    o = Oracle(model, variant)
    oh, os_ = o.step(nsteps)
    s = Solver(model)
    s.run(nsteps)
    s.sync()
    gh = np.stack([s.history(f) for f in range(s.nf)], axis=1)
    gs = s.stations()
    return o, oh, os_, s, gh, gs


@pytest.fixture(scope="module")
def sw32():
    m = configs.tiny_sw(nsteps=90)
    return (m,) + run_both(m, 90, MIXED)


def test_sw_f32_history_bitwise(sw32):
    m, o, oh, os_, s, gh, gs = sw32
    assert gh.shape == (90, 4, s.nzT, s.nxT)
    assert np.abs(oh[:, 0]).max() > 0.1, "the tiny model must rupture"
    for f in range(4):
        np.testing.assert_array_equal(gh[:, f], oh[:, f], err_msg=f"history field {f}")
    np.testing.assert_array_equal(gs, os_)


def test_sw_f32_state_bitwise(sw32):
    m, o, oh, os_, s, gh, gs = sw32
    for name in ("u", "v", "w", "xx", "yy", "zz", "xy", "yz", "xz"):
        np.testing.assert_array_equal(s.field(name), o.field(name), err_msg=name)
    for name in ("tx", "tz", "slipX", "slipZ", "ruptime", "rise", "sliptime", "distX", "distZ"):
        np.testing.assert_array_equal(s.plane(name), o.plane(name), err_msg=name)


def test_sw_f64_bitwise():
    m = configs.tiny_sw(nsteps=60, precision="f64")
    o, oh, os_, s, gh, gs = run_both(m, 60, F64)
    for f in range(4):
        np.testing.assert_array_equal(gh[:, f], oh[:, f], err_msg=f"history field {f}")
    for name in ("u", "w", "xx", "xz"):
        np.testing.assert_array_equal(s.field(name), o.field(name), err_msg=name)


@pytest.mark.parametrize("prec,variant,tol", [("f32", MIXED, 1e-5), ("f64", F64, 1e-9)])
def test_fvw_matches_oracle(prec, variant, tol):
    m = configs.tiny_fvw(nsteps=60, precision=prec)
    o, oh, os_, s, gh, gs = run_both(m, 60, variant)
    assert np.abs(oh[:, 0]).max() > 1e-3, "the nucleation must start slip"
    for f in range(5):
        assert rel_l2(gh[:, f], oh[:, f]) <= tol, (f, rel_l2(gh[:, f], oh[:, f]))
    for name in ("psiX", "psiZ", "slipX", "slipZ"):
        assert rel_l2(s.plane(name), o.plane(name)) <= tol, name


def test_f32_vs_f64_oracle_accuracy():
    """The production FP32 build against the FP64 oracle at the stated tolerances."""
    m = configs.tiny_sw(nsteps=150, nxT=48, nzT=32)
    o = Oracle(m, F64)
    oh, _ = o.step(150)
    s = Solver(m)
    s.run(150)
    s.sync()
    for f in range(4):
        assert rel_l2(s.history(f), oh[:, f]) <= 1e-3, f
    fo, fg = o.final(), s.final()
    assert rel_l2(fg["slipX"], fo["slipX"]) <= 1e-4
    assert rel_l2(fg["slipZ"], fo["slipZ"]) <= 1e-4 or np.abs(fo["slipZ"]).max() < 1e-6
    ruptured = fo["ruptime"] < 1e4
    assert ruptured.sum() > 50
    assert np.all((fg["ruptime"] < 1e4) == ruptured)
    assert np.abs(fg["ruptime"][ruptured] - fo["ruptime"][ruptured]).max() <= 2 * m["dt"]


def test_odd_sizes_and_partial_tiles():
    m = configs.tiny_sw(nxT=37, nyT=11, nzT=23, nsteps=40)
    o, oh, os_, s, gh, gs = run_both(m, 40, MIXED)
    for f in range(4):
        np.testing.assert_array_equal(gh[:, f], oh[:, f])


def test_graph_chunks_equal_single_steps():
    m = configs.tiny_sw(nsteps=40)
    a = Solver(m)
    a.run(40)   # two 16-step graphs + 8 eager steps
    a.sync()
    b = Solver(m)
    for _ in range(40):
        b.run(1)
    b.sync()
    np.testing.assert_array_equal(a.history(0), b.history(0))
    np.testing.assert_array_equal(a.field("xz"), b.field("xz"))


def test_reset_reproduces():
    m = configs.tiny_fvw(nsteps=30)
    s = Solver(m)
    s.run(30)
    s.sync()
    h1 = s.history(0)
    s.reset()
    s.run(30)
    s.sync()
    np.testing.assert_array_equal(s.history(0), h1)


@pytest.mark.parametrize("variant,kchunk", [("tiled", 64), ("pipe", 64), ("pipe", 5), ("point", 1), ("point", 3),
                                            ("tma", 32), ("tma", 5), ("tma", 2), ("tma", 1)])
def test_interior_variants_identical(variant, kchunk):
    """Every interior sweep variant computes the same bits as the per-point kernel."""
    m = configs.tiny_sw(nxT=70, nyT=20, nzT=36, nsteps=30)
    os.environ["FD3D_INTERIOR"] = "point"
    os.environ["FD3D_KCHUNK"] = "4"
    try:
        a = Solver(m)
        os.environ["FD3D_INTERIOR"] = variant
        os.environ["FD3D_KCHUNK"] = str(kchunk)
        b = Solver(m)
    finally:
        del os.environ["FD3D_INTERIOR"]
        del os.environ["FD3D_KCHUNK"]
    for s in (a, b):
        s.run(30)
        s.sync()
    for name in ("u", "v", "w", "xx", "yy", "zz", "xy", "yz", "xz"):
        np.testing.assert_array_equal(a.field(name), b.field(name), err_msg=name)


def test_history_stride_and_ring():
    m = configs.tiny_sw(nsteps=40, stride=4)
    m["history_capacity"] = 4
    s = Solver(m)
    s.run(40)
    s.sync()
    assert s.history_records() == 10
    o = Oracle(m, MIXED)
    oh, _ = o.step(40)
    last = s.history(0, rec0=6, nrec=4)          # the ring keeps the last 4 records
    np.testing.assert_array_equal(last, oh[[27, 31, 35, 39], 0])
    # the same records in the field type: copied straight out of the ring (which wraps here)
    np.testing.assert_array_equal(s.history(0, rec0=6, nrec=4, real_kind=4), oh[[27, 31, 35, 39], 0].astype(np.float32))
    with pytest.raises(Fd3dError):
        s.history(0, rec0=0, nrec=1)             # overwritten


def test_nonfinite_input_is_reported():
    m = configs.tiny_sw(nsteps=10)
    m["fault"]["striniX"] = m["fault"]["striniX"].copy()
    m["fault"]["striniX"][25, 20] = np.nan
    s = Solver(m)
    s.run(10)
    with pytest.raises(Fd3dError) as e:
        s.sync()
    assert "NONFINITE" in str(e.value)


def test_write_results_files(tmp_path):
    m = configs.tiny_sw(nsteps=20)
    s = Solver(m)
    s.run(12)
    s.sync()
    s.write_results(str(tmp_path), 4)
    s.run(8)
    s.sync()
    s.write_results(str(tmp_path), 4)
    raw = np.fromfile(tmp_path / "sliprateX.res", dtype=np.float32)
    assert raw.size == 20 * s.nxT * s.nzT
    np.testing.assert_array_equal(raw.reshape(20, s.nzT, s.nxT), s.history(0).astype(np.float32))
    st = np.loadtxt(tmp_path / "stan0.txt")
    assert st.shape == (20, 3)
    np.testing.assert_allclose(st, s.stations()[:, 0], rtol=1e-14, atol=0)
    rt = np.loadtxt(tmp_path / "ruptime.res")
    assert rt.size == s.nxT * s.nzT
    fin = s.final()["ruptime"][m["nabc"]:m["nxt"] - m["nabc"], m["nabc"]:m["nzt"] - m["nfs"]]
    np.testing.assert_allclose(rt, fin.ravel(order="F"), rtol=1e-14)


def test_heterogeneous_medium_bitwise():
    """A medium that varies in x and y as well (every cell perturbed) runs the sweeps
    that read the 3-D arrays; a layered medium uploaded as 3-D arrays is detected as
    layered.  Both agree with the oracle to the last bit."""
    m = configs.tiny_sw(seed=21, nsteps=40)
    lam, mu, d = configs.medium_3d(m)
    rng = np.random.default_rng(3)
    lam3, mu3, d3 = (np.asfortranarray(a * (1.0 + 0.05 * rng.uniform(-1.0, 1.0, a.shape))) for a in (lam, mu, d))
    for arrays in ((lam3, mu3, d3), tuple(np.asfortranarray(a) for a in (lam, mu, d))):
        o = Oracle(m, MIXED)
        o.set_medium_arrays(*arrays)
        oh, os_ = o.step(40)
        s = Solver(m)
        s.upload_medium_arrays(*arrays, real_kind=8)
        s.run(40)
        s.sync()
        gh = np.stack([s.history(f) for f in range(s.nf)], axis=1)
        np.testing.assert_array_equal(gh, oh[:, :s.nf])
        for name in ("u", "w", "xx", "xz", "yz"):
            np.testing.assert_array_equal(s.field(name), o.field(name), err_msg=name)
        s.close()
        o.close()


@pytest.mark.parametrize("precision,variant", [("f32", MIXED), ("f64", F64)])
def test_moment_rate_and_post_loop_match_oracle(precision, variant, tmp_path):
    """Moment rate per step and the post-loop block (rupture velocity, cohesive zone,
    average rupture speed, seismic moment, stress drop) on the device against the
    oracle's sequential loops: the per-node planes agree to the last bit, the sums up to
    their summation order."""
    m = configs.tiny_sw(seed=8, nsteps=70, precision=precision)
    o = Oracle(m, variant)
    o.step(70, history=False)
    s = Solver(m)
    s.run(70)
    s.sync()
    mr = s.moment_rate()
    assert mr.shape == (70,) and mr.max() > 0
    np.testing.assert_allclose(mr, o.moment_rate(), rtol=1e-12, atol=0)
    got = s.post_process()
    ref, rv, cz = o.post()
    np.testing.assert_array_equal(got["rvel"], rv)
    np.testing.assert_array_equal(got["czone"], cz)
    assert got["area"] == 0.0
    np.testing.assert_allclose([got["rupture_speed"], got["moment"], got["stress_drop"]], ref[[0, 1, 3]],
                               rtol=1e-12)
    s.write_results(str(tmp_path), 8 if precision == "f64" else 4)
    c = np.loadtxt(tmp_path / "contour.res", skiprows=1)
    assert c.shape == (s.nxT * s.nzT, 3)
    inner = (slice(m["nabc"], m["nxt"] - m["nabc"]), slice(m["nabc"], m["nzt"] - m["nfs"]))
    np.testing.assert_allclose(np.loadtxt(tmp_path / "rvel.res"), rv[inner].ravel(order="F"), rtol=1e-14)
    np.testing.assert_allclose(np.loadtxt(tmp_path / "czone.res"), cz[inner].ravel(order="F"), rtol=1e-14)


@pytest.mark.parametrize("dipslip", [False, True])
def test_fault_from_inversion_control_points(dipslip):
    """The control points of forwardmodel.dat interpolated onto the fault plane on the
    device (inversion_modeltofd3d + interp_fric) give the oracle's fault and, after a
    run, its histories, to the last bit."""
    m = configs.tiny_sw(seed=31, nsteps=40)
    rng = np.random.default_rng(5)
    nli, nwi = 7, 5
    T0I = rng.uniform(20e6, 30e6, (nli, nwi))
    TsI = rng.uniform(0.6, 0.7, (nli, nwi))
    TsI[3, 2] = 0.02  # a weak spot in the middle breaks at once
    DcI = rng.uniform(0.2, 0.5, (nli, nwi))
    o = Oracle(m, MIXED)
    o.set_fault_model(T0I, TsI, DcI, dip=75.0, dipslip=dipslip)
    oh, _ = o.step(40)
    s = Solver(m)
    s.upload_fault_model(T0I, TsI, DcI, dip=75.0, dipslip=dipslip)
    for name in ("T0X", "T0Z"):
        np.testing.assert_array_equal(s.plane(name), o.plane(name), err_msg=name)
    s.run(40)
    s.sync()
    gh = np.stack([s.history(f) for f in range(s.nf)], axis=1)
    assert np.abs(oh[:, 0:2]).max() > 0, "the weak spot must slip"
    np.testing.assert_array_equal(gh, oh[:, :s.nf])
    np.testing.assert_array_equal(s.final()["slipX"], o.plane("slipX"))


def test_history_read_while_next_run_is_queued():
    """fd3d_fetch_history waits only for the run that made the records it reads: the
    records of one run come back while the next run is still queued, and both sets are
    the oracle's."""
    m = configs.tiny_sw(seed=19, nsteps=60)
    m["history_capacity"] = 40
    oh, os_ = Oracle(m, MIXED).step(60)
    s = Solver(m)
    s.run(20)
    s.run(20)                       # queued behind the first run
    first = np.stack([s.history(f, rec0=0, nrec=20) for f in range(4)], axis=1)
    st = s.stations(rec0=0, nrec=20)
    s.run(20)
    second = np.stack([s.history(f, rec0=20, nrec=20) for f in range(4)], axis=1)
    s.sync()
    third = np.stack([s.history(f, rec0=40, nrec=20) for f in range(4)], axis=1)
    np.testing.assert_array_equal(np.concatenate([first, second, third]), oh[:, :4])
    np.testing.assert_array_equal(st, os_[:20])
    s.close()


def test_medium_upload_paths_agree():
    """fd3d_upload_medium stages the host arrays in the still-zero wave field (before the
    first step) or copies them row by row into the padded arrays (after steps, when the wave
    field is live): FP32 and FP64 host arrays, before and after steps, give the same run."""
    m = configs.tiny_sw(seed=17, nxT=37, nyT=13, nzT=25, nsteps=30)
    lam, mu, d = configs.medium_3d(m)
    rng = np.random.default_rng(8)
    arrs = [np.asfortranarray((a * (1.0 + 0.05 * rng.uniform(-1.0, 1.0, a.shape))).astype(np.float32))
            for a in (lam, mu, d)]
    runs = []
    for rk in (4, 8):
        s = Solver(m)
        s.upload_medium_arrays(*(a if rk == 4 else a.astype(np.float64) for a in arrs), real_kind=rk)
        s.run(30)
        s.sync()
        runs.append((s.history(0), s.field("xz")))
        s.close()
    s = Solver(m)                      # medium replaced mid-run with the same values
    s.upload_medium_arrays(*arrs, real_kind=4)
    s.run(10)
    s.sync()
    s.upload_medium_arrays(*arrs, real_kind=4)
    s.run(20)
    s.sync()
    runs.append((s.history(0), s.field("xz")))
    s.close()
    for h, xz in runs[1:]:
        np.testing.assert_array_equal(h, runs[0][0])
        np.testing.assert_array_equal(xz, runs[0][1])
    o = Oracle(m, MIXED)
    o.set_medium_arrays(*(a.astype(np.float64) for a in arrs))
    oh, _ = o.step(30)
    np.testing.assert_array_equal(runs[0][0], oh[:, 0])


@pytest.mark.parametrize("case", ["tiny_sw_f32", "tiny_sw_f64", "tiny_sw_fspace_f32"])
def test_gpu_matches_golden_fixture(case):
    """The CUDA path against the committed fixture (digests of the oracle's outputs on seeded
    small models, tests/golden/make_golden.py): histories, stations, wave fields and fault
    planes bit for bit, with no oracle run on the GPU box."""
    import json
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "golden"))
    import make_golden as mg
    with open(os.path.join(here, "golden", "oracle_tiny.json")) as f:
        g = json.load(f)
    m, _ = mg.cases()[case]
    steps = g["steps"]
    m["history_capacity"] = steps
    s = Solver(m)
    s.run(steps)
    s.sync()
    hist = np.stack([s.history(f) for f in range(4)], axis=1)
    got = mg.outputs_digests(hist, s.stations(), s.field, s.plane)
    s.close()
    want = g["cases"][case]
    for k, v in got.items():
        assert v == want[k], k
