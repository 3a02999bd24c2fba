"""Models built by the SCEC set-ups (decks in the reference's format, written here) on
the GPU against the oracle: TPV9's dip-slip fault with cohesion and depth-dependent
normal stress bit for bit, TPV104's rate-and-state fault with its nucleation ramp
within the FVW tolerance (CUDA's exp/log/sinh/asinh against libm)."""
import numpy as np
import pytest

from fd3d_tsn_b200 import configs
from fd3d_tsn_b200.solver import Solver
from oracle.oracle import MIXED, Oracle
from test_setups_cpu import synthetic_deck, write_forward_model

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0)


@pytest.mark.parametrize("setup", ["TPV8", "TPV9"])
def test_scec_sw_setup_bitwise(tmp_path, setup):
    m = configs.reference_example(synthetic_deck(tmp_path, setup), setup)
    m["history_capacity"] = 60
    o = Oracle(m, MIXED)
    oh, os_ = o.step(60)
    s = Solver(m)
    s.run(60)
    s.sync()
    comp = 1 if setup == "TPV9" else 0
    assert np.abs(oh[:, comp]).max() > 0.1
    for f in range(4):
        np.testing.assert_array_equal(s.history(f), oh[:, f], err_msg=f"history field {f}")
    np.testing.assert_array_equal(s.stations(), os_)
    fo, fg = o.final(), s.final()
    for k in fo:
        np.testing.assert_array_equal(fg[k], fo[k], err_msg=k)
    s.close()


def test_tpv104_setup_matches_oracle(tmp_path):
    m = configs.reference_example(synthetic_deck(tmp_path, "TPV104", dt=0.004), "TPV104")
    m["history_capacity"] = 60
    o = Oracle(m, MIXED)
    oh, _ = o.step(60)
    s = Solver(m)
    s.run(60)
    s.sync()
    assert np.abs(oh[:, 0]).max() > 1e-3
    for f in range(5):
        assert rel_l2(s.history(f), oh[:, f]) <= 1e-5, f
    for name in ("psiX", "psiZ", "slipX", "T0X"):
        assert rel_l2(s.plane(name), o.plane(name)) <= 1e-5, name
    s.close()


def test_inversion_deck_model_bitwise(tmp_path):
    """A deck with forwardmodel.dat (dynamicsolver without -DSCEC): Solver and oracle both
    take the fault from the control points; histories agree to the last bit."""
    d = synthetic_deck(tmp_path, "TPV5")
    rng = np.random.default_rng(12)
    T0I = rng.uniform(20e6, 30e6, (7, 5))
    TsI = rng.uniform(0.6, 0.7, (7, 5))
    TsI[3, 2] = 0.02
    DcI = rng.uniform(0.2, 0.5, (7, 5))
    write_forward_model(d, T0I, TsI, DcI)
    m = configs.inversion_example(d, dipslip=False)
    m["history_capacity"] = 40
    oh, _ = Oracle(m, MIXED).step(40)
    s = Solver(m)
    s.run(40)
    s.sync()
    assert np.abs(oh[:, 0]).max() > 0
    np.testing.assert_array_equal(np.stack([s.history(f) for f in range(4)], axis=1), oh[:, :4])
    s.close()
