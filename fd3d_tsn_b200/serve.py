"""Continuous-batching request loop over the batched C ABI.

Requests (forward solves of mixed size) arrive on a clock.  The loop admits every
arrived request whose model fits the device arena (the HBM budget) into the running
batch, advances all resident models together for a chunk of time steps in one
persistent launch, retires the models that reached their last step (their final
planes are read back and their arena space freed) and admits waiting requests into
the freed space at the next chunk boundary.  Requests that arrive while others are on
the GPU therefore share the launches with them.

Latency of a request = completion time - arrival time (wall clock of the loop).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from .batch import Batch, bytes_needed
from .solver import Solver


@dataclass
class Result:
    request: int
    arrival: float
    admitted: float
    done: float
    final: dict = field(repr=False)

    @property
    def latency(self):
        return self.done - self.arrival


def serve(stream, hbm_budget_bytes: int, chunk: int = 32, max_models: int = 1024, autotune_key: str | None = None,
          tune_cache: str | None = None, keep_final=None, clock=time.perf_counter):
    """Runs the request stream [(arrival_s, model), ...] (sorted by arrival).

    keep_final(request) -> bool selects the requests whose final planes are kept in
    the results (all if None).  Returns (results, stats)."""
    b = Batch(hbm_budget_bytes, max_models)
    need = {id(m): bytes_needed(m) for _, m in stream}
    waiting = []           # (arrival, model) arrived but not admitted
    resident = {}          # slot -> (arrival, admitted, model)
    results = []
    nxt = 0
    t0 = clock()
    busy = 0.0
    launches = 0
    peak_resident = 0
    tuned = False
    while nxt < len(stream) or waiting or resident:
        now = clock() - t0
        while nxt < len(stream) and stream[nxt][0] <= now:
            waiting.append(stream[nxt])
            nxt += 1
        # admission by HBM budget: first come first served, skip what does not fit yet
        still = []
        for arr, m in waiting:
            slot = b.try_add(m) if need[id(m)] <= hbm_budget_bytes else None
            if slot is None:
                still.append((arr, m))
            else:
                resident[slot] = (arr, clock() - t0, m)
        waiting = still
        peak_resident = max(peak_resident, len(resident))
        if not resident:
            if nxt < len(stream):  # idle until the next arrival
                time.sleep(max(0.0, min(0.01, stream[nxt][0] - (clock() - t0))))
            continue
        if autotune_key and not tuned and all(b.steps_done(s) == 0 for s in resident):
            b.autotune(steps=8, cache_path=tune_cache, key=autotune_key)
            tuned = True
        b.run(chunk)
        b.sync()
        launches += 1
        busy += b.last_run_ms() / 1e3
        for slot in list(resident):
            arr, adm, m = resident[slot]
            if b.steps_done(slot) >= m["ntfd"]:
                fin = b.final(slot) if (keep_final is None or keep_final(m["request"])) else None
                results.append(Result(m["request"], arr, adm, clock() - t0, fin))
                b.remove(slot)
                del resident[slot]
    makespan = clock() - t0
    b.close()
    lat = np.array([r.latency for r in results])
    stats = dict(requests=len(results), makespan_s=makespan, solves_per_s=len(results) / makespan,
                 p50_latency_s=float(np.percentile(lat, 50)), p99_latency_s=float(np.percentile(lat, 99)),
                 mean_latency_s=float(lat.mean()), gpu_busy_s=busy, launches=launches, chunk_steps=chunk,
                 peak_resident=peak_resident, hbm_budget_bytes=hbm_budget_bytes)
    return results, stats


def plain(models, keep_final=None, clock=time.perf_counter):
    """One-at-a-time solves through the single-model path (create, upload, run, read
    back, destroy).  Returns (finals by request, seconds)."""
    t0 = clock()
    out = {}
    for m in models:
        s = Solver(m)
        s.run(m["ntfd"])
        s.sync()
        if keep_final is None or keep_final(m["request"]):
            out[m["request"]] = s.final()
        else:
            s.final()
        s.close()
    return out, clock() - t0
