"""The continuous-batching request loop: requests of mixed size arrive while others
are on the GPU, are admitted as arena space frees up (their set-up overlapping the
running chunk), and each result is the same bits as the request solved alone and as the
oracle's solve of it."""
import numpy as np
import pytest

from fd3d_tsn_b200 import configs
from fd3d_tsn_b200.batch import bytes_needed
from fd3d_tsn_b200.serve import plain, pretune, serve
from oracle.oracle import MIXED, Oracle

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(300)]


def stream(n, seed=11):
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(0.01, size=n))
    out = []
    for q in range(n):
        m = configs.tiny_sw(seed=300 + q, nxT=int(rng.integers(30, 64)), nyT=int(rng.integers(12, 18)),
                            nzT=int(rng.integers(20, 40)), nsteps=int(rng.integers(20, 70)))
        m["history_capacity"] = 16
        m["request"] = q
        out.append((float(t[q]), m))
    return out


def check(results, ref):
    assert {r.request for r in results} == set(ref)
    for r in results:
        for k in ("slipX", "slipZ", "ruptime", "rise", "sliptime"):
            np.testing.assert_array_equal(r.final[k], ref[r.request][k], err_msg=f"{r.request} {k}")


def test_serve_results_equal_plain_solves():
    s = stream(24)
    ref, _ = plain([m for _, m in s])
    # a budget of about four models forces waiting, admission into freed space and reuse
    budget = 4 * max(bytes_needed(m) for _, m in s)
    results, stats = serve(s, budget, chunk=8)
    assert stats["requests"] == len(s) and stats["rejected"] == 0
    assert 1 < stats["peak_resident"] < len(s)  # several at once, never all: requests waited
    assert all(r.latency >= 0 for r in results)
    check(results, ref)


def test_serve_with_pretuned_schedule(tmp_path):
    s = stream(10, seed=12)
    ref, _ = plain([m for _, m in s])
    t = pretune([m for _, m in s[:4]], cache_path=str(tmp_path / "t.jsonl"), key="serve-test", steps=4)
    results, stats = serve([(0.0, m) for _, m in s], 1 << 30, chunk=16, tuning=t)
    assert stats["requests"] == len(s)
    check(results, ref)


def test_oversized_request_is_rejected_not_queued_forever():
    small = [m for _, m in stream(2, seed=13)]
    big = configs.tiny_sw(seed=399, nxT=120, nyT=30, nzT=80, nsteps=10)
    big["request"] = 2
    s = [(0.0, small[0]), (0.0, big), (0.0, small[1])]
    budget = bytes_needed(small[0]) + bytes_needed(small[1]) + (4 << 20)
    assert bytes_needed(big) > budget
    results, stats = serve(s, budget, chunk=8)
    assert stats["rejected"] == 1 and stats["requests"] == 2
    assert {r.request for r in results} == {small[0]["request"], small[1]["request"]}


def test_served_results_against_oracle():
    """Requests of the batched workload's size (h = 200 m, 0.35-0.9 M cells) through the
    request loop, two of them checked against the oracle directly, bit for bit."""
    steps = 30
    models = configs.batch_set(6, seed=616, ntfd=steps)
    s = []
    for q, m in enumerate(models):
        m["request"] = q
        m["history_capacity"] = 8
        s.append((0.002 * q, m))
    budget = 3 * max(bytes_needed(m) for m in models)
    results, stats = serve(s, budget, chunk=8)
    assert stats["requests"] == len(models) and stats["rejected"] == 0
    byreq = {r.request: r for r in results}
    for q in (0, 5):
        o = Oracle(models[q], MIXED)
        o.step(steps)
        fo = o.final()
        assert np.abs(fo["slipX"]).max() > 0, "the request must slip"
        for k in fo:
            np.testing.assert_array_equal(byreq[q].final[k], fo[k], err_msg=f"request {q} {k}")
        o.close()
