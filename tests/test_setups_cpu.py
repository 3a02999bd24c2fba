"""The reference's SCEC set-ups (forwardspecialTPV5/8/9/103/104, src/fd3d_init.f90:283-783)
restated on the host in fd3d_tsn_b200.configs, checked on decks written here in the
reference's file format and, where the reference's example directories are present, on
those.  The oracle runs a few steps of each to show the fault they build behaves as the
set-up intends (dip slip for TPV9, strike slip for TPV5/8, the rate-and-state
nucleation ramp for TPV103/104)."""
import os

import numpy as np
import pytest

from fd3d_tsn_b200 import configs
from oracle.oracle import F64, Oracle

# the reference's examples/ directory (input decks), when a copy is at hand
REF_EXAMPLES = os.environ.get("FD3D_REFERENCE_EXAMPLES", "")


def write_sw_scec(path, no0, hx0, hz0, hdelta, T0, T0n, sn, mus, muso, mud, d0h):
    """scecmodel.dat of TPV5/8/9: the two side patches of TPV5 are placed off the grid."""
    with open(path, "w") as f:
        f.write(f"{no0} {hx0!r} {hz0!r} -1e9 -1e9 -1e9 -1e9\n{hdelta!r}\n{T0!r} {T0n!r} {T0!r} {T0!r}\n{sn!r}\n")
        f.write(f"{mus!r} {muso!r}\n{mud!r}\n{d0h!r}\n0. 0.\n")


def write_fvw_scec(path, wfx, wfz, hx0t, hz0t, trans, fringe, tini=40e6, perturb=45e6, rr=1200.0, tt=0.1):
    vals = [0.6, 1e-6, 0.01, 0.014, 0.4, 0.2, 0.1, 0.9, 0.5e-16, tini, 120e6, perturb, rr, tt]
    with open(path, "w") as f:
        f.write(f"{wfx!r} {wfz!r} {hx0t!r} {hz0t!r} {trans!r} {fringe!r}\n")
        for v in vals:
            f.write(f"{v!r}\n")


def synthetic_deck(tmp_path, setup, dt=None, nxT=40, nyT=14, nzT=28, h=200.0):
    """A small deck directory for one SCEC set-up (homogeneous medium, 2 stations)."""
    lay = dict(depth=[0.0], vp=[6000.0], vs=[3464.0], rho=[2670.0])
    m = configs.sw_model(nxT, nyT, nzT, h, 1.0, 4, layers=lay, nstations=2, ntfd=60)
    if dt is not None:
        m["dt"] = dt
    d = str(tmp_path / setup)
    configs.write_deck(m, d, lay)
    scec = os.path.join(d, "scecmodel.dat")
    nab = m["nabc"]
    if setup in ("TPV5", "TPV8", "TPV9"):
        # nucleation square centred in the fault plane, fault border of 3 nodes
        cx = (nab + nxT // 2 - 1) * h
        cz = (nab + nzT // 2 - 1) * h
        if setup == "TPV5":
            write_sw_scec(scec, nab + 3, cx, cz, 1600.0, 70e6, 81.6e6 * 1.02, 120e6, 0.677, 1e4, 0.525, 0.4)
        else:  # TPV8/9 stresses scale with depth: T0 and T0n are ratios
            write_sw_scec(scec, nab + 3, cx, cz, 1600.0, 0.55, 1.02, 7378.0, 0.76, 1e4, 0.448, 0.5)
    else:
        write_fvw_scec(scec, nxT * h / 3, nzT * h / 3, nxT * h / 2 - 600.0, nzT * h / 2 - 600.0, 600.0, 600.0)
    return d


@pytest.mark.parametrize("setup", ["TPV5", "TPV8", "TPV9"])
def test_sw_setups_slip_in_their_direction(tmp_path, setup):
    d = synthetic_deck(tmp_path, setup)
    m = configs.reference_example(d, setup)
    f = m["fault"]
    nzt = m["nzt"]
    if setup != "TPV5":
        assert np.all(f["coh"] == 1e6)
        # depth-dependent normal stress: strength grows with depth below the surface row
        col = f["peak_xz"][m["nxt"] // 2, :]
        assert col[nzt // 2] > col[nzt - 4] > 0
    pre = f["striniZ"] if setup == "TPV9" else f["striniX"]
    other = f["striniX"] if setup == "TPV9" else f["striniZ"]
    assert np.all(other == 0) and pre.max() > 0
    np.testing.assert_array_equal(f["peak_xz"][:, nzt - 2], f["peak_xz"][:, nzt - 3])  # ghost rows
    sign = -1 if setup != "TPV5" else 1
    np.testing.assert_array_equal(pre[:, nzt - 1], sign * pre[:, nzt - 4])
    o = Oracle(m, F64)
    h, _ = o.step(40)
    assert np.isfinite(h).all()
    sx, sz = np.abs(h[:, 0]).max(), np.abs(h[:, 1]).max()
    if setup == "TPV9":
        assert sz > 0.1 and sx < 0.05 * sz
    else:
        assert sx > 0.1 and sz < 0.05 * sx


@pytest.mark.parametrize("variant", ["TPV103", "TPV104"])
def test_fvw_setups_nucleate(tmp_path, variant):
    d = synthetic_deck(tmp_path, variant, dt=0.004)
    m = configs.reference_example(d, variant)
    m["history_stride"] = 1
    f = m["fault"]
    assert f["nucleation"] == 1 and f["strinixI"] == 40e6
    assert np.all((f["a"] >= 0.01 - 1e-15) & (f["a"] <= 0.02 + 1e-15))
    assert f["a"].min() == 0.01 and f["a"].max() == 0.02  # velocity-strengthening outside the box
    assert np.isfinite(f["psi"]).all() and np.isfinite(f["psiX"]).all()
    if variant == "TPV104":  # one-sided taper: nothing above the hypocentre is strengthened
        k0 = int(f["hz0"] / m["dh"])
        assert np.all(f["a"][:, k0:] == f["a"][:, k0:k0 + 1])
    o = Oracle(m, F64)
    h, _ = o.step(40)
    assert np.isfinite(h).all() and o.last_rc == 0
    assert np.abs(h[:, 0]).max() > 1e-6  # the ramp starts slip
    assert o.plane("T0X").max() > 40e6


@pytest.mark.skipif(not (REF_EXAMPLES and os.path.isdir(REF_EXAMPLES)),
                    reason="FD3D_REFERENCE_EXAMPLES does not name the reference's examples directory")
@pytest.mark.parametrize("deck,setup", [("TPV5", "TPV5"), ("TPV9", "TPV9"), ("TPV104", "TPV104")])
def test_reference_example_decks_build(deck, setup):
    m = configs.reference_example(os.path.join(REF_EXAMPLES, deck), setup)
    f = m["fault"]
    for k, v in f.items():
        if isinstance(v, np.ndarray):
            assert v.shape == (m["nxt"], m["nzt"]) and np.isfinite(v).all(), k
    if setup == "TPV9":
        assert np.all(f["striniX"] == 0) and f["striniZ"].max() > 0
    if setup == "TPV104":
        assert f["law"] == "fvw" and f["hx0"] > m["nabc"] * m["dh"]


def write_forward_model(d, T0I, TsI, DcI):
    nli, nwi = T0I.shape
    with open(os.path.join(d, "inputinv.dat"), "w") as f:
        f.write(f"0\n{nli} {nwi}\n-123\n1\n0. 1.e8\n")
    vals = [19.7, 0.6] + [float(x) for a in (T0I, TsI, DcI) for x in a.ravel(order="F")]
    with open(os.path.join(d, "forwardmodel.dat"), "w") as f:
        f.write(" ".join(f"{v:.5E}" for v in vals) + "\n")


def test_inversion_deck_reads_control_points(tmp_path):
    d = synthetic_deck(tmp_path, "TPV5")
    rng = np.random.default_rng(9)
    T0I, TsI, DcI = rng.uniform(1e6, 5e6, (6, 4)), rng.uniform(0.5, 0.7, (6, 4)), rng.uniform(0.2, 0.4, (6, 4))
    write_forward_model(d, T0I, TsI, DcI)
    m = configs.inversion_example(d, dipslip=True)
    fm = m["fault_model"]
    for got, want in zip((fm["T0I"], fm["TsI"], fm["DcI"]), (T0I, TsI, DcI)):
        np.testing.assert_allclose(got, want, rtol=1e-5)
    assert fm["dipslip"] and "fault" not in m
    o = Oracle(m, F64)  # takes the fault from the control points
    assert np.abs(o.plane("T0Z")).max() > 0 and np.all(o.plane("T0X") == 0)


@pytest.mark.skipif(not (REF_EXAMPLES and os.path.isdir(REF_EXAMPLES)),
                    reason="FD3D_REFERENCE_EXAMPLES does not name the reference's examples directory")
def test_reference_inversion_example_reads():
    m = configs.inversion_example(os.path.join(REF_EXAMPLES, "Amatrice2016"), dipslip=True)
    fm = m["fault_model"]
    assert fm["T0I"].shape == (13, 8) and np.isfinite(fm["DcI"]).all() and fm["DcI"].min() > 0


def test_fspace_variant_keeps_the_model_below_the_top():
    m = configs.tiny_sw(nsteps=10)
    f = configs.fspace_variant(m)
    nab, ks = m["nabc"], m["nzt"] - m["nfs"]
    assert f["fspace"] and f["nfs"] == nab and f["nzt"] == m["nzt"] + nab - m["nfs"]
    assert f["nzt"] - f["nfs"] == ks                          # the former free-surface row
    for a, b in zip(m["medium"], f["medium"]):
        np.testing.assert_array_equal(b[:m["nzt"]], a)
    for k, v in m["fault"].items():
        if isinstance(v, np.ndarray):
            np.testing.assert_array_equal(f["fault"][k][:, :m["nzt"]], v)
            assert f["fault"][k].flags.f_contiguous


def test_reference_example_in_the_fspace_build(tmp_path):
    d = synthetic_deck(tmp_path, "TPV5")
    a = configs.reference_example(d, "TPV5")
    b = configs.reference_example(d, "TPV5", fspace=True)
    assert b["nfs"] == b["nabc"] and b["nzt"] - b["nfs"] == a["nzt"] - a["nfs"]
    np.testing.assert_array_equal(b["medium"][1][:a["nzt"] - a["nfs"]], a["medium"][1][:a["nzt"] - a["nfs"]])
