"""Checkpoint and resume through the C ABI: a run saved after some steps and resumed in a
new context continues bit for bit (wave field, PML state, fault state, step counter and
history ring), for slip weakening and for rate-and-state friction with its nucleation ramp."""
import numpy as np
import pytest

from fd3d_tsn_b200 import abi, configs
from fd3d_tsn_b200.solver import Solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["sw", "fvw", "sw_f64"])
def test_resume_continues_bitwise(tmp_path, kind):
    if kind == "fvw":
        m = configs.tiny_fvw(nsteps=40)
    else:
        m = configs.tiny_sw(nsteps=40, precision="f64" if kind == "sw_f64" else "f32")
    m["history_capacity"] = 40
    path = str(tmp_path / "run.ckpt")
    a = Solver(m)
    a.run(17)
    a.checkpoint(path)
    a.run(23)
    a.sync()
    b = Solver.restore(path, m)
    assert b.steps_done() == 17
    b.run(23)
    b.sync()
    assert b.steps_done() == 40
    for f in range(a.nf):
        np.testing.assert_array_equal(b.history(f, rec0=17, nrec=23), a.history(f, rec0=17, nrec=23), err_msg=str(f))
    np.testing.assert_array_equal(b.history(0, rec0=0, nrec=17), a.history(0, rec0=0, nrec=17))  # the saved ring
    for name in ("u", "w", "xz", "yz"):
        np.testing.assert_array_equal(b.field(name), a.field(name), err_msg=name)
    fa, fb = a.final(), b.final()
    for k in fa:
        np.testing.assert_array_equal(fb[k], fa[k], err_msg=k)
    a.close()
    b.close()


def test_restore_rejects_other_files(tmp_path):
    p = tmp_path / "not.ckpt"
    p.write_bytes(b"something else entirely")
    with pytest.raises(abi.Fd3dError) as e:
        Solver.restore(str(p), configs.tiny_sw())
    assert e.value.code == -8
