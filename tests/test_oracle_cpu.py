"""The CPU oracle on its own: physics invariants and agreement of its precision variants.

Parity of the oracle with the reference's own output is unpinned (no golden outputs
ship with the reference and no Fortran compiler exists here); these invariants are
what pins it instead.
"""
import numpy as np
import pytest

from fd3d_tsn_b200 import configs
from oracle.oracle import F32, F64, MIXED, Oracle


def test_rest_state_stays_at_rest():
    m = configs.tiny_sw(nsteps=30)
    m["fault"]["striniX"] = np.zeros_like(m["fault"]["striniX"])
    o = Oracle(m, F64)
    h, s = o.step(30)
    assert np.all(h == 0) and np.all(s == 0)
    for f in ("u", "v", "w", "xx", "yy", "zz", "xy", "yz", "xz"):
        assert np.all(o.field(f) == 0), f


def test_sw_rupture_grows_and_stays_finite():
    m = configs.tiny_sw(nsteps=120)
    o = Oracle(m, F64)
    h, _ = o.step(120)
    assert np.isfinite(h).all()
    fin = o.final()
    rupt = fin["ruptime"] < 1e4
    assert rupt.sum() > 100
    # rupture times increase away from the nucleation patch
    nab = m["nabc"]
    i = np.arange(m["nxt"])[:, None] + 1
    k = np.arange(m["nzt"])[None, :] + 1
    ic = nab + 1 + (m["nxt"] - 2 * nab) // 2
    kc = nab + 1 + (m["nzt"] - m["nfs"] - nab) // 2
    r = np.hypot(i - ic, k - kc)
    near = rupt & (r < 4)
    far = rupt & (r > 8)
    assert far.any()
    assert fin["ruptime"][near].mean() < fin["ruptime"][far].mean()
    # right-lateral slip sign: the prestress drives negative u on the fault side
    assert (fin["slipX"][rupt] > 0).mean() > 0.95


def test_precision_variants_agree():
    m = configs.tiny_sw(nsteps=80)
    hm, _ = Oracle(m, MIXED).step(80)
    hd, _ = Oracle(m, F64).step(80)
    hs, _ = Oracle(m, F32).step(80)
    for f in range(4):
        ref = np.linalg.norm(hd[:, f])
        assert np.linalg.norm(hm[:, f] - hd[:, f]) / ref < 1e-4
        assert np.linalg.norm(hs[:, f] - hd[:, f]) / ref < 1e-3


def test_pml_absorbs_radiated_energy():
    """After the rupture stops at its barrier, kinetic energy leaves through the PML."""
    m = configs.tiny_sw(nsteps=500, nxT=40, nzT=28)
    f = m["fault"]
    f["peak_xz"] = f["peak_xz"].copy()
    nab = m["nabc"]
    # a small patch only: rupture dies quickly
    f["peak_xz"][:, :] = 120e6 * 10000.0
    ic, kc = nab + 20, nab + 14
    f["peak_xz"][ic - 5:ic + 5, kc - 5:kc + 5] = 0.68 * 120e6
    o = Oracle(m, F64)
    energies = []
    for _ in range(25):
        o.step(20, history=False)
        e = sum(float((o.field(c) ** 2).sum()) for c in ("u", "v", "w"))
        energies.append(e)
    peak = max(energies)
    assert energies[-1] < 0.05 * peak, (energies[-1], peak)


def test_fvw_nucleation_and_state():
    m = configs.tiny_fvw(nsteps=80)
    o = Oracle(m, F64)
    h, _ = o.step(80)
    assert np.isfinite(h).all()
    assert o.last_rc == 0
    assert np.abs(h[:, 0]).max() > 1e-3
    psi0 = m["fault"]["psi"]
    psi = o.plane("psiZ")
    nab = m["nabc"]
    sl = (slice(nab, m["nxt"] - nab), slice(nab, m["nzt"] - m["nfs"]))
    assert np.abs(psi[sl] - psi0[sl]).max() > 0
    # the ramp raised T0X near the hypocentre
    t0 = o.plane("T0X")
    assert t0.max() > m["fault"]["striniX"].max()


@pytest.mark.parametrize("variant", [MIXED, F64])
def test_reset_is_exact(variant):
    m = configs.tiny_fvw(nsteps=20)
    o = Oracle(m, variant)
    h1, _ = o.step(20)
    from oracle import oracle as om
    om.lib().oracle_reset(o.h)
    h2, _ = o.step(20)
    np.testing.assert_array_equal(h1, h2)


def _fspace_pair(nsteps):
    m = configs.sw_model(40, 14, 40, 200.0, 1.0, 7, patch_nodes=(8, 8), nstations=2, ntfd=nsteps, corr_m=600.0)
    return m, configs.fspace_variant(m)


def test_fspace_equals_free_surface_until_the_waves_reach_the_top():
    """The FSPACE build (PML strip above instead of the free surface) runs the same
    arithmetic below the top: its histories follow the free-surface build's until the
    waves from the patch (16 cells below the top) reach it, and part ways afterwards."""
    m, mf = _fspace_pair(200)
    assert mf["nzt"] == m["nzt"] + m["nabc"] - 2 and mf["nfs"] == m["nabc"]
    a, b = Oracle(m, MIXED), Oracle(mf, MIXED)
    ha, _ = a.step(40)
    hb, _ = b.step(40)
    assert np.abs(ha[:, 0]).max() > 0.1, "the patch must slip"
    for f in range(4):
        assert np.linalg.norm(ha[:, f] - hb[:, f]) <= 1e-8 * np.linalg.norm(ha[:, f]), f
    a.step(110, history=False)
    b.step(110, history=False)
    ha, _ = a.step(50)
    hb, _ = b.step(50)
    assert np.linalg.norm(ha[:, 0] - hb[:, 0]) > 0.05 * np.linalg.norm(ha[:, 0])


@pytest.mark.parametrize("fspace", [False, True])
def test_top_boundary_energy(fspace):
    """A rupture confined to a small patch radiates; with the FSPACE strip the energy
    leaves through all sides, and it never grows without bound in either build."""
    m, mf = _fspace_pair(500)
    o = Oracle(mf if fspace else m, F64)
    energies, top = [], 0.0
    ks = m["nzt"] - m["nfs"]
    for _ in range(25):
        o.step(20, history=False)
        u = o.field("u")
        energies.append(sum(float((o.field(c) ** 2).sum()) for c in ("u", "v", "w")))
        top = max(top, float(np.abs(u[:, :, ks + 1:]).max()))  # k >= ks+2: u of the top strip / never set
    peak = max(energies)
    assert np.isfinite(energies).all()
    assert energies[-1] < 0.05 * peak, (fspace, energies[-1], peak)
    if fspace:
        assert top > 1e-3  # the top strip carries the wave field it absorbs
    else:
        assert top == 0.0  # fuvw sets u on the first ghost row only


def test_symmetric_setup_gives_symmetric_rupture():
    """A homogeneous model with uniform prestress and friction and a nucleation square
    centred in x ruptures symmetrically: the rupture times on the Z nodes mirror exactly
    about the centre of the interior plane."""
    m = configs.tiny_sw(nsteps=120, nxT=40, nzT=28)
    f = m["fault"]
    nab, nxt, nzt = m["nabc"], m["nxt"], m["nzt"]
    T = np.full((nxt, nzt), 70e6)
    T[nab + 16:nab + 24, nab + 10:nab + 18] = 0.68 * 120e6 * 1.02   # nodes nab+17..nab+24 in x
    plane = lambda v: np.asfortranarray(np.full((nxt, nzt), v))
    f.update(striniX=np.asfortranarray(T), peak_xz=plane(0.68 * 120e6), dyn_xz=plane(0.52 * 120e6), Dc=plane(0.4),
             coh=plane(0.0))
    o = Oracle(m, F64)
    o.step(120)
    rt = o.final()["ruptime"][nab:nxt - nab, nab:nzt - m["nfs"]]
    assert (rt < 1e4).sum() > 100
    np.testing.assert_array_equal(rt, rt[::-1, :])


def _golden():
    import json
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "oracle_tiny.json")
    with open(path) as f:
        return json.load(f)


@pytest.mark.parametrize("case", ["tiny_sw_f32", "tiny_sw_f64", "tiny_sw_fspace_f32"])
def test_oracle_matches_its_golden_fixture(case):
    """The committed fixture (tests/golden/make_golden.py, digests of the oracle's own outputs on
    seeded small models) still holds: the restatement has not drifted.  The fixture is made by
    the oracle, not by the reference, whose Fortran build cannot run here."""
    import sys
    import os
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_golden as mg
    g = _golden()
    m, var = mg.cases()[case]
    want = g["cases"][case]
    o = Oracle(m, {"MIXED": MIXED, "F64": F64}[var])
    hist, seis = o.step(g["steps"])
    got = mg.outputs_digests(hist, seis, o.field, o.plane)
    o.close()
    assert want["max_slip_rate"] > 0.1, "the fixture's model must slip"
    for k, v in got.items():
        assert v == want[k], k
