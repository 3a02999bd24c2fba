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
