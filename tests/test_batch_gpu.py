"""The batched schedules against the single-model path, through the C ABI.

Every model in a batch must produce the same bits as the same model solved alone
with fd3d_run (the per-item device bodies are the single-model kernels' bodies), no
matter which other models share the launch, when it joined, which schedule runs the
batch (one persistent cooperative kernel, or graphs of per-region kernels) or which
tile shape the autotuner picked.  Models of the batched workload's own size are also
checked against the oracle directly, in both schedules.
"""
import numpy as np
import pytest

from fd3d_tsn_b200 import configs
from fd3d_tsn_b200.batch import Batch, bytes_needed
from fd3d_tsn_b200.solver import Solver
from oracle.oracle import MIXED, Oracle

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0)


def small_models(n, seed0=100, steps=30):
    rng = np.random.default_rng(seed0)
    out = []
    for q in range(n):
        nxT = int(rng.integers(30, 60))
        nzT = int(rng.integers(20, 40))
        m = configs.tiny_sw(seed=seed0 + q, nxT=nxT, nyT=int(rng.integers(12, 18)), nzT=nzT, nsteps=steps)
        m["history_capacity"] = steps
        out.append(m)
    return out


def alone(m, steps):
    s = Solver(m)
    s.run(steps)
    s.sync()
    return s


def same(b, slot, s, steps):
    fb, fs = b.final(slot), s.final()
    for k in fb:
        np.testing.assert_array_equal(fb[k], fs[k], err_msg=k)
    for name in ("tx", "tz", "slipX"):
        np.testing.assert_array_equal(b.plane(slot, name), s.plane(name), err_msg=name)
    np.testing.assert_array_equal(b.history(slot, 0, 0, steps), s.history(0, 0, steps))


SCHEDULES = pytest.mark.parametrize("schedule", ["graph", "persistent"])


@SCHEDULES
def test_batch_equals_single_model_runs(schedule):
    models = small_models(5, steps=30)
    b = Batch(2 << 30, 16)
    b.set_schedule(schedule)
    slots = [b.add(m) for m in models]
    b.run(30)
    b.sync()
    for m, slot in zip(models, slots):
        assert b.steps_done(slot) == 30
        same(b, slot, alone(m, 30), 30)


@SCHEDULES
def test_batch_mixed_laws_and_uneven_lengths(schedule):
    sw = small_models(2, seed0=7, steps=24)
    fvw = configs.tiny_fvw(nsteps=18)
    fvw["history_capacity"] = 18
    b = Batch(2 << 30, 8)
    b.set_schedule(schedule)
    s0, s1, s2 = b.add(sw[0]), b.add(fvw), b.add(sw[1])
    b.run(16)
    b.run(16)   # each model stops at its own ntfd
    b.sync()
    assert b.steps_done(s1) == 18 and b.steps_done(s0) == 24
    same(b, s0, alone(sw[0], 24), 24)
    same(b, s2, alone(sw[1], 24), 24)
    ref = alone(fvw, 18)
    for k in ("slipX", "slipZ"):
        np.testing.assert_array_equal(b.final(s1)[k], ref.final()[k])


@SCHEDULES
def test_models_joining_later_and_leaving(schedule):
    """Continuous batching: a model admitted while others run gets its own answer."""
    ms = small_models(4, seed0=40, steps=40)
    b = Batch(2 << 30, 8)
    b.set_schedule(schedule)
    a0, a1 = b.add(ms[0]), b.add(ms[1])
    b.run(10)
    a2 = b.add(ms[2])        # joins at another model's step 10
    b.run(10)
    b.remove(a1)             # leaves early
    a3 = b.add(ms[3])        # reuses arena space
    b.run(40)
    b.sync()
    for m, slot in ((ms[0], a0), (ms[2], a2), (ms[3], a3)):
        assert b.steps_done(slot) == 40
        same(b, slot, alone(m, 40), 40)


def test_arena_admission():
    m = small_models(1)[0]
    need = bytes_needed(m)
    b = Batch(need * 2 + (1 << 20), 8)
    assert b.try_add(m) is not None
    assert b.try_add(m) is not None
    assert b.try_add(m) is None          # arena full
    n, used = b.live()
    assert n == 2 and used >= 2 * need - 512


def test_autotune_keeps_results(tmp_path):
    models = small_models(3, seed0=70, steps=20)
    b = Batch(2 << 30, 8)
    slots = [b.add(m) for m in models]
    t = b.autotune(steps=5, cache_path=str(tmp_path / "tune.jsonl"), key="test3")
    assert t["kchunk"] in (4, 8, 16, 32) and t["schedule"] in ("graph", "persistent")
    assert (tmp_path / "tune.jsonl").read_text().count("test3") == 1
    b.run(20)
    b.sync()
    for m, slot in zip(models, slots):
        same(b, slot, alone(m, 20), 20)
    b2 = Batch(1 << 30, 4)
    b2.add(models[0])
    assert b2.autotune(steps=5, cache_path=str(tmp_path / "tune.jsonl"), key="test3") == {**t, "max_ctas_per_sm": t["max_ctas_per_sm"]}


def batch_size_fvw(steps):
    """A rate-and-state model of the batched workload's size (h = 200 m, 140 x 30 x 70
    simulated cells, a 16 x 8 km fault, nucleation ramp on)."""
    m = configs.fvw_model(140, 30, 70, 200.0, 1.0, 88, fault_m=(16e3, 8e3), dt=0.008, ntfd=steps,
                          history_stride=1, border_m=2000.0, R=2000.0, TT=0.1)
    m["history_capacity"] = steps
    return m


@SCHEDULES
def test_batch_models_against_oracle(schedule):
    """Models of the batched workload's distribution (fault 8-24 x 6-14 km, h = 200 m,
    grids of 0.35-0.9 M cells) plus a rate-and-state model of the same size, in one
    batch, each against the oracle: slip weakening bit for bit (histories, final planes,
    tractions, slip path), rate-and-state within 1e-5 relative
    L2 on all five history fields and the state planes."""
    steps = 40
    models = configs.batch_set(4, seed=515, ntfd=steps)
    for m in models:
        m["history_capacity"] = steps
    fvw = batch_size_fvw(steps)
    b = Batch(4 << 30, 8)
    b.set_schedule(schedule)
    slots = [b.add(m) for m in models]
    fslot = b.add(fvw)
    b.run(steps)
    b.sync()
    for m, slot in zip(models, slots):
        assert b.steps_done(slot) == steps
        o = Oracle(m, MIXED)
        oh, _ = o.step(steps)
        assert np.abs(oh[:, 0]).max() > 0.1, "the nucleation patch must slip"
        for f in range(4):
            np.testing.assert_array_equal(b.history(slot, f, 0, steps), oh[:, f], err_msg=f"field {f}")
        fo, fb = o.final(), b.final(slot)
        for k in fo:
            np.testing.assert_array_equal(fb[k], fo[k], err_msg=k)
        for name in ("tx", "tz", "distZ"):
            np.testing.assert_array_equal(b.plane(slot, name), o.plane(name), err_msg=name)
        o.close()
    o = Oracle(fvw, MIXED)
    oh, _ = o.step(steps)
    assert np.abs(oh[:, 0]).max() > 1e-3, "the nucleation must start slip"
    for f in range(5):
        assert rel_l2(b.history(fslot, f, 0, steps), oh[:, f]) <= 1e-5, f
    for name in ("psiX", "psiZ", "slipX", "slipZ"):
        assert rel_l2(b.plane(fslot, name), o.plane(name)) <= 1e-5, name
    b.close()
