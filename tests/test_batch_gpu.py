"""The batched schedules against the single-model path, through the C ABI.

Every model in a batch must produce the same bits as the same model solved alone
with fd3d_run (the per-item device bodies are the single-model kernels' bodies), no
matter which other models share the launch, when it joined, which schedule runs the
batch (one persistent cooperative kernel, or graphs of per-region kernels) or which
tile shape the autotuner picked.
"""
import numpy as np
import pytest

from fd3d_tsn_b200 import configs
from fd3d_tsn_b200.batch import Batch, bytes_needed
from fd3d_tsn_b200.solver import Solver

pytestmark = pytest.mark.gpu


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
