"""Continuous-batching request loop over the batched C ABI.

Requests (forward solves of mixed size) arrive on a clock.  The loop admits every
arrived request whose model fits the device arena (the HBM budget) into the batch,
advances all resident models together for a chunk of time steps in one batch run,
retires the models that reached their last step (their final planes are read back
and their arena space freed) and admits waiting requests into the freed space.
Admission happens while the previous chunk runs on the GPU, and the new models join
at the next chunk, so requests that arrive while others are on the GPU share the
launches with them.

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


def pretune(models, cache_path: str | None = None, key: str | None = None, steps: int = 8):
    """Tile shape and schedule for a request mix, picked before serving starts: a scratch
    batch of the given sample models is autotuned (and cached under key), then dropped.
    Returns the tuning dict."""
    arena = int(sum(bytes_needed(m) for m in models) * 1.05) + (64 << 20)
    b = Batch(arena, len(models) + 4)
    for m in models:
        b.add(m)
    t = b.autotune(steps=steps, cache_path=cache_path, key=key)
    b.close()
    return t


def serve(stream, hbm_budget_bytes: int, chunk: int = 32, max_models: int = 1024, tuning: dict | None = None,
          keep_final=None, clock=time.perf_counter):
    """Runs the request stream [(arrival_s, model), ...] (sorted by arrival).

    Each pass launches one batch run of `chunk` steps over the resident models
    (asynchronous), admits the requests that arrived meanwhile while that run is on the
    GPU (their set-up goes on the batch's own set-up stream), then waits for the run
    and retires the models that reached their last step.  tuning (from pretune) fixes
    the schedule and tile shape.  keep_final(request) -> bool selects the requests whose
    final planes are kept in the results (all if None).  Returns (results, stats)."""
    b = Batch(hbm_budget_bytes, max_models)
    if tuning:
        b.set_schedule(tuning["schedule"])
        b.set_tuning(tuning["kchunk"], tuning["ctas_per_sm"] if tuning["schedule"] == "persistent" else 0)
    need = {id(m): bytes_needed(m) for _, m in stream}
    waiting = []           # (arrival, model) arrived but not admitted
    resident = {}          # slot -> (arrival, admitted, model)
    results = []
    nxt = 0
    t0 = clock()
    busy = 0.0
    launches = 0
    peak_resident = 0
    rejected = []

    def admit():
        nonlocal waiting, nxt
        now = clock() - t0
        while nxt < len(stream) and stream[nxt][0] <= now:
            waiting.append(stream[nxt])
            nxt += 1
        still = []
        for arr, m in waiting:  # first come first served by HBM budget; what does not fit waits
            if need[id(m)] > hbm_budget_bytes:  # can never fit: rejected, not queued forever
                rejected.append(m["request"])
                continue
            slot = b.try_add(m)
            if slot is not None:
                resident[slot] = (arr, clock() - t0, m)
            elif not resident and not b.live()[0]:  # does not fit even an empty arena
                rejected.append(m["request"])
            else:
                still.append((arr, m))
        waiting = still

    while nxt < len(stream) or waiting or resident:
        running = list(resident)
        if running:
            b.run(chunk)       # asynchronous: the admissions below overlap it
            launches += 1
        admit()
        peak_resident = max(peak_resident, len(resident))
        if not running:
            if not resident and nxt < len(stream):  # idle until the next arrival
                time.sleep(max(0.0, min(0.01, stream[nxt][0] - (clock() - t0))))
            continue
        b.sync()
        busy += b.last_run_ms() / 1e3
        for slot in running:
            arr, adm, m = resident[slot]
            if b.steps_done(slot) >= m["ntfd"]:
                fin = b.final(slot) if (keep_final is None or keep_final(m["request"])) else None
                results.append(Result(m["request"], arr, adm, clock() - t0, fin))
                b.remove(slot)
                del resident[slot]
    makespan = clock() - t0
    b.close()
    lat = np.array([r.latency for r in results])
    pct = (lambda q: float(np.percentile(lat, q))) if len(lat) else (lambda q: None)
    stats = dict(requests=len(results), makespan_s=makespan, solves_per_s=len(results) / makespan,
                 p50_latency_s=pct(50), p99_latency_s=pct(99), mean_latency_s=float(lat.mean()) if len(lat) else None,
                 gpu_busy_s=busy, launches=launches, chunk_steps=chunk,
                 peak_resident=peak_resident, hbm_budget_bytes=hbm_budget_bytes, rejected=len(rejected))
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
