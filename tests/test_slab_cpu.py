"""The z-slab plan and the slab arguments, on the host (no device needed).

fd3d_slab_plan splits planes 1..nzt into slabs of about equal cost; every slab must
own at least 4 planes and the top slab the two planes below the free surface (its fres
and fuvw rows then stay out of every neighbour's halo).  fd3d_ctx_create_slab checks a
range before it looks for a device.
"""
import ctypes as C

import pytest

from fd3d_tsn_b200 import abi, configs
from fd3d_tsn_b200.slab import plan
from fd3d_tsn_b200.solver import lib


def _valid(m, ranges):
    nzt, ks = m["nzt"], m["nzt"] - m["nfs"]
    assert ranges[0][0] == 1 and ranges[-1][1] == nzt
    for r, (a, b) in enumerate(ranges):
        assert b - a + 1 >= 4
        if r:
            assert a == ranges[r - 1][1] + 1
    assert ranges[-1][0] <= ks - 2


@pytest.mark.parametrize("name", ["tiny_sw", "sw_small", "sw_large", "fvw_medium"])
@pytest.mark.parametrize("n", [1, 2, 3, 4, 8])
def test_plan_covers_the_model(name, n):
    m = getattr(configs, name)()
    ranges = plan(m, n)
    assert len(ranges) == n
    _valid(m, ranges)


def test_plan_balances_cost():
    m = configs.sw_large()
    ranges = plan(m, 8)
    sizes = [b - a + 1 for a, b in ranges]
    # the bottom slab holds the z-PML planes (2.2x the cost of an interior plane each)
    assert sizes[0] < sizes[1]
    assert max(sizes[1:]) - min(sizes[1:]) <= 2


def test_plan_fspace():
    m = configs.tiny_sw(fspace=True)
    _valid(m, plan(m, 4))


def test_plan_refuses_too_many_slabs():
    m = configs.tiny_sw()
    with pytest.raises(abi.Fd3dError):
        plan(m, 12)   # 40 planes cannot give 12 slabs of 4 with the top rule


@pytest.mark.parametrize("rng", [(0, 10), (1, 2), (37, 40), (1, 37)])
def test_invalid_slab_ranges_refused_before_any_device(rng):
    """(0,10): k_lo < 1; (1,2): fewer than 4 planes; (37,40) with nzt=40, ks=38: top slab
    starts above ks-2; (1,37): a slab that is not the top ends inside ks-2 .. ks."""
    m = configs.tiny_sw()
    p = abi.make_params(m)
    h = C.c_void_p()
    assert lib().fd3d_ctx_create_slab(C.byref(p), rng[0], rng[1], C.byref(h)) == -1  # FD3D_ERR_ARG
    assert not h.value


def _halo(k_lo, k_hi, side):
    s, r = C.c_int(), C.c_int()
    assert lib().fd3d_slab_halo_plan(k_lo, k_hi, side, C.byref(s), C.byref(r)) == 0
    return s.value, r.value


@pytest.mark.parametrize("name,n", [("tiny_sw", 4), ("sw_small", 8), ("sw_large", 8), ("fvw_medium", 3)])
def test_halo_plan_pairs_every_receive_with_the_neighbours_send(name, n):
    """Both transports (the in-process pull and the NCCL send/receive pairs) take their
    planes from fd3d_slab_halo_plan: what a slab receives on one side is exactly what its
    neighbour sends on the other, two of the neighbour's own planes, landing in the
    receiver's halo (stored, not owned)."""
    m = getattr(configs, name)()
    ranges = plan(m, n)
    for (a_lo, a_hi), (b_lo, b_hi) in zip(ranges, ranges[1:]):
        a_send_up, a_recv_up = _halo(a_lo, a_hi, 1)
        b_send_dn, b_recv_dn = _halo(b_lo, b_hi, 0)
        assert a_recv_up == b_send_dn and b_recv_dn == a_send_up
        for k in (b_send_dn, b_send_dn + 1):
            assert b_lo <= k <= b_hi and a_hi < k <= a_hi + 3      # B's own, A's halo
        for k in (a_send_up, a_send_up + 1):
            assert a_lo <= k <= a_hi and b_lo - 3 <= k < b_lo      # A's own, B's halo
