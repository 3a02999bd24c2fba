#!/usr/bin/env python3
"""Throughput of the FD3D_TSN time step on B200.

Default workload: the slip-weakening production model (1000 x 400 x 500 simulated cells,
1020 x 410 x 512 padded = 214.1 M cells, h = 50 m, 5 seeded layers, FP32 wave field
with FP64 slip / rupture-time accumulators).  A *step* is one pass of the time loop
(velocity + stress sweeps, PML strips, free surface, fault boundary condition and the
history planes) over the whole grid.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line.  value = padded cells x steps x N / max-over-ranks device time.
The same line carries, as "batch" and "serve", the batched workload (256 models of
uneven size, 8 s simulated, against the same models solved one at a time) and the
serving workload (a mixed-size request stream through the continuous-batching loop:
capacity solves/s, p50 / p99 latency at 70% of that capacity, against one-at-a-time
solves), both measured after the timed region.  With N > 1 every rank runs its own
independent replicas (the path has no exchange step), so scaling is weak; --gpus N
started without torchrun starts N ranks under torch.distributed.run itself.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

B_ALG_STEP = 120          # algorithmic FP32 bytes per cell per step (velocity 52 + stress 68)
B_ALG_STR = 68            # stress sweep: 3 v + lam + mu + 6 sigma loads, 6 sigma stores
B_ALG_VEL = 52            # velocity sweep: 6 sigma + rho + 3 v loads, 3 v stores
# The workloads' media are 1-D layered (as readcrustalmodel builds them), and the interior
# sweeps then read one lam/mu/rho value per plane instead of per cell: the bytes they must
# move are 4 B less per medium array (velocity 48, stress 60, step 108).  The roofline of
# the dominant kernel is quoted against those; the step figure keeps the 120 B convention.
B_ALG_STR_LAYERED = 60
B_ALG_VEL_LAYERED = 48
FALLBACK_HBM_GBS = 6650.0


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev: int):
        self.dev = dev
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.flush()
        self.out.seek(0)
        rows = [r.split(",") for r in self.out.read().splitlines() if r.strip()]
        os.unlink(self.out.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() in ("active", "1"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(ngpus, backend=None):
    """One process per GPU under torchrun: the process group carries only the barrier
    around the timed region and the max-over-ranks reduction of the timings (replicas,
    no data-path collective).  backend "gloo" (FD3D_BENCH_BACKEND) runs the same
    plumbing on CPU tensors."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    backend = backend or os.environ.get("FD3D_BENCH_BACKEND", "nccl")
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def _on_gpu(pg):
    return pg is not None and pg.get_backend() == "nccl"


def barrier(pg, local):
    if pg is not None:
        import torch
        if _on_gpu(pg):
            pg.barrier(device_ids=[local])
            torch.cuda.synchronize()
        else:
            pg.barrier()


def max_over_ranks(pg, local, v):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{local}" if _on_gpu(pg) else "cpu")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, world, seconds_max):
    """Weak scaling over replicas: every rank processed units_per_rank; the job took the
    slowest rank's time."""
    return units_per_rank * world / seconds_max


def workload(name):
    from fd3d_tsn_b200 import configs
    if name == "sw_large":
        return configs.sw_large()
    if name == "sw_small":
        return configs.sw_small()
    if name == "sw_mid":   # 400x200x200 cells: larger than L2, small enough for ncu captures
        return configs.sw_model(400, 200, 200, 100.0, 1.0, 4, patch_nodes=(300, 150), ntfd=1000)
    if name == "fvw_medium":
        return configs.fvw_medium()
    raise SystemExit(f"unknown workload {name}")


def describe(name, m):
    nab = m["nabc"]
    return {"workload": name,
            "grid_sim": [m["nxt"] - 2 * nab, m["nyt"] - nab, m["nzt"] - nab - m["nfs"]],
            "grid_padded": [m["nxt"], m["nyt"], m["nzt"]],
            "cells_padded": m["nxt"] * m["nyt"] * m["nzt"],
            "h_m": m["dh"], "dt_s": m["dt"], "law": m.get("law", "sw"),
            "fields": "fp32", "accumulators": "fp64", "medium": "1-D layered",
            "history_stride": m.get("history_stride", 1),
            "l2": "inputs larger than L2 (wave field ~10 GB >> 126 MB)"}


def cpu_baseline(m, seconds_target=15.0, threads=None):
    """The oracle (a loop-by-loop CPU restatement of the reference) on the host cores,
    FP32 like the reference built without -r8, on whole steps of the same model."""
    from oracle import oracle as om
    if threads:
        om.set_threads(threads)
    o = om.Oracle(m, om.F32)
    o.step(1, history=False)  # first touch of the 11 GB of state
    t0 = time.perf_counter()
    n = 0
    while True:
        o.step(1, history=False)
        n += 1
        if time.perf_counter() - t0 > seconds_target:
            break
    dt = time.perf_counter() - t0
    cells = m["nxt"] * m["nyt"] * m["nzt"]
    o.close()
    return {"value": cells * n / dt / 1e9, "unit": "GCell-updates/s", "cores": om.num_threads(),
            "kind": "port", "sample": f"{n} whole time steps of the same model after 1 untimed step ({dt:.1f} s)"}


def run_reference(args, world, rank, local, pg):
    if rank != 0:
        return
    m = workload(args.workload)
    from oracle import oracle as om
    o = om.Oracle(m, om.F32)
    o.step(1, history=True)  # first touch of the state; the CPU path has nothing else to warm
    # whole time steps of the same model, at most args.steps and about a minute of CPU work
    n, dt = 0, 0.0
    t0 = time.perf_counter()
    while n < args.steps and (n < 2 or dt < args.ref_seconds):
        o.step(1, history=True)
        n += 1
        dt = time.perf_counter() - t0
    cells = m["nxt"] * m["nyt"] * m["nzt"]
    v = cells * n / dt / 1e9
    line = {"impl": "reference", "metric": "GCell-updates/s", "value": v, "unit": "GCell-updates/s",
            "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / n * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": describe(args.workload, m),
            "cpu_baseline": {"value": v, "unit": "GCell-updates/s", "cores": om.num_threads(), "kind": "port",
                             "sample": f"{n} whole time steps of the {m['nxt']}x{m['nyt']}x{m['nzt']} model with "
                                       f"history planes ({dt:.1f} s) after 1 untimed step, all host threads; the "
                                       f"CPU restatement of the reference in FP32 (no Fortran compiler here)"},
            "e2e": {"value": v, "unit": "GCell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_b200(args, world, rank, local, pg):
    from fd3d_tsn_b200 import abi
    from fd3d_tsn_b200.solver import Solver, lib
    lib().fd3d_set_device(local)
    m = workload(args.workload)
    cells = m["nxt"] * m["nyt"] * m["nzt"]
    nab = m["nabc"]
    nxT, nzT = m["nxt"] - 2 * nab, m["nzt"] - nab - m["nfs"]
    interior = nxT * (m["nyt"] - 2 - nab) * nzT
    s = Solver(m)
    s.run(args.warmup)
    s.sync()
    clocks = ClockSampler(local)
    barrier(pg, local)
    clocks.start()
    time.sleep(0.3)
    s.run(args.steps)
    s.sync()
    ms = s.last_run_ms()          # CUDA events on the stream the steps are launched on
    ck = clocks.stop()
    ms_max = max_over_ranks(pg, local, ms)
    value = whole_job_rate(cells * args.steps, world, ms_max / 1e3) / 1e9

    # per-kernel times (CUDA events around each launch) over a few extra steps
    s.set_profiling(True)
    nprof = max(3, min(10, args.steps))
    s.run(nprof)
    s.sync()
    kt = s.kernel_times()
    s.set_profiling(False)
    peak, peak_kind = measured_peak()
    kstr_ms = kt["str_interior"][0] / max(kt["str_interior"][1], 1)
    kvel_ms = kt["vel_interior"][0] / max(kt["vel_interior"][1], 1)
    dom, dom_ms, dom_bytes = ("str_interior", kstr_ms, B_ALG_STR_LAYERED * interior) if kstr_ms >= kvel_ms else \
        ("vel_interior", kvel_ms, B_ALG_VEL_LAYERED * interior)
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    step_gbs = cells * B_ALG_STEP / (ms / args.steps / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic_dram_bytes.txt")   # ncu DRAM bytes per launch
    if os.path.exists(tpath):
        with open(tpath) as f:
            for line in f:
                w = line.split()
                if len(w) == 3 and not w[0].startswith("#") and w[0] == args.workload and w[1] == dom:
                    traffic = int(w[2])
    info = s.info()
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "interior_variant": info["interior_variant"], "layered_medium": info["layered_medium"],
                "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                "algorithmic_bytes_per_launch": dom_bytes, "avg_launch_ms": dom_ms,
                "step_frac": step_gbs / peak, "step_gbs": step_gbs,
                "kernel_ms_per_step": {k: (v[0] / max(v[1], 1)) for k, v in kt.items()}}
    s.close()

    # end to end through the C ABI with host buffers: medium + fault upload from pinned
    # host memory, K steps, and every step's history planes and station samples read back
    e2e = None
    if args.e2e:
        e2e = end_to_end(m, args.steps, local)
        e2e_v = max_over_ranks(pg, local, e2e.pop("_seconds"))
        e2e["value"] = whole_job_rate(cells * args.steps, world, e2e_v) / 1e9

    # the batched and serving workloads, after the timed region of the production model
    batch = batch_section(args, world, rank, local, pg) if args.batch and args.workload == "sw_large" else None
    serving = serve_section(args, world, rank, local, pg) if args.serve and args.workload == "sw_large" else None

    cpu = None
    if rank == 0 and world == 1 and args.cpu_baseline > 0:
        cpu = cpu_baseline(m, args.cpu_baseline)
    if rank == 0:
        line = {"metric": "GCell-updates/s", "value": value, "unit": "GCell-updates/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": describe(args.workload, m), "roofline": roofline,
                "cpu_baseline": cpu, "e2e": e2e, "clocks": ck,
                "gpu_launches": gpu_launches(m, args.steps),
                "hbm_roofline_frac_step": step_gbs / peak}
        if batch is not None:
            line["batch"] = batch
        if serving is not None:
            line["serve"] = serving
        print(json.dumps(line), flush=True)


def gpu_launches(m, steps):
    # vel interior, fault band, PML, free surface; stress interior, fault band, PML; fres +
    # fault boundary condition (one fused launch); the nucleation ramp of rate-and-state runs
    per_step = 8 - (1 if m.get("fspace") else 0) + (1 if m.get("law") == "fvw" and m["fault"].get("nucleation") else 0)
    return per_step * steps


def pinned(shape, dtype, order="F"):
    """Page-locked host array (cudaHostAlloc through torch)."""
    import torch
    t = torch.empty(int(np.prod(shape)), dtype=torch.float32 if dtype == np.float32 else torch.float64,
                    pin_memory=True)
    return t.numpy().reshape(shape, order=order), t


def end_to_end(m, steps, local):
    import ctypes as C
    from fd3d_tsn_b200 import abi
    from fd3d_tsn_b200.solver import Solver, lib
    shp = (m["nxt"], m["nyt"], m["nzt"])
    keep = []
    host = []
    for a in m["medium"]:
        arr, t = pinned(shp, np.float32)
        arr[...] = np.asarray(a, dtype=np.float32)[None, None, :]
        host.append(arr)
        keep.append(t)
    nab = m["nabc"]
    plane = (m["nxt"] - 2 * nab) * (m["nzt"] - nab - m["nfs"])
    nf = 5 if m.get("law") == "fvw" else 4   # slip rates, shear tractions (+ psi for FVW)
    stride = max(1, int(m.get("history_stride", 1)))
    nrec = steps // stride
    hist, th = pinned((nf, max(nrec, 1), plane), np.float32, order="C")
    keep.append(th)
    nst = len(m.get("stations", []))
    seis = np.empty((max(nrec, 1), max(nst, 1), 3))
    chunk = 16              # history records are read back every chunk of steps
    m = dict(m, history_capacity=2 * chunk)
    s = Solver(m)           # context + fault; its medium is replaced inside the timed region
    s.run(0)
    s.sync()
    s.reset()
    t0 = time.perf_counter()
    s.upload_medium_arrays(*host, real_kind=4)
    s.upload_fault(m["fault"])
    # Chunks of steps are enqueued one ahead: the records of a chunk are read back while
    # the next chunk runs (a read waits only for the run that made its records).
    done = got = 0
    ready = 0                    # steps of the chunks enqueued before the latest one
    while got < nrec or done < steps:
        if done < steps:
            n = min(chunk, steps - done)
            s.run(n)
            done += n
        else:
            ready = done
        have = ready // stride
        if have > got:
            for f in range(nf):
                rc = lib().fd3d_fetch_history(s.h, f, got, have - got, hist[f, got:have].ctypes.data, 4)
                if rc:
                    raise abi.Fd3dError(rc, "fd3d_fetch_history")
            if nst:
                rc = lib().fd3d_fetch_stations(s.h, got, have - got,
                                               seis[got:have].ctypes.data_as(C.POINTER(C.c_double)))
                if rc:
                    raise abi.Fd3dError(rc, "fd3d_fetch_stations")
            got = have
        ready = done
    s.sync()
    dt = time.perf_counter() - t0
    s.close()
    fault_bytes = 6 * m["nxt"] * m["nzt"] * 8
    h2d = 3 * int(np.prod(shp)) * 4 + fault_bytes
    d2h = (nf * plane * 4 + nst * 3 * 8) * nrec
    return {"unit": "GCell-updates/s", "h2d_bytes_per_step": h2d / steps, "d2h_bytes_per_step": d2h / steps,
            "_seconds": dt, "includes": f"medium (fp32, pinned) + fault upload, K steps, the {nrec} history records "
                                        f"({nf} planes each, every {stride} steps) + stations read back; wall clock"}


def _same_finals(a, b):
    return all(np.array_equal(a[k], b[k]) for k in ("slipX", "slipZ", "ruptime", "rise", "sliptime"))


def pml_cells(m):
    """Cells of the PML strips' u/w loop ranges (init_pml, src/fd3d_deriv.f90:1319-1410):
    x-low and x-high (nabc-1 wide, j up to nyt, interior k), y-low (nabc-1 rows), z-low
    (nabc-1 planes) and, under FSPACE, the top strip."""
    nxt, nyt, nzt, nab, nfs = m["nxt"], m["nyt"], m["nzt"], m["nabc"], m["nfs"]
    nk = nzt - nfs - nab
    n = 2 * (nab - 1) * (nyt - nab) * nk + (nxt - 2) * (nab - 1) * nk + (nxt - 2) * (nyt - 1) * (nab - 1)
    if m.get("fspace"):
        n += (nxt - 2) * (nyt - 1) * (nab - 1)
    return n


def interior_cells(m):
    nab = m["nabc"]
    return (m["nxt"] - 2 * nab) * (m["nyt"] - 2 - nab) * (m["nzt"] - nab - m["nfs"])


# algorithmic bytes of one step of a layered-medium model: 108 B per interior cell (velocity
# 48 + stress 60) and 264 B per PML cell (108 + 156: fields plus the split components)
B_INTERIOR_LAYERED = B_ALG_VEL_LAYERED + B_ALG_STR_LAYERED
B_PML_LAYERED = 108 + 156


def step_bytes(m):
    return interior_cells(m) * B_INTERIOR_LAYERED + pml_cells(m) * B_PML_LAYERED


def batch_section(args, world, rank, local, pg):
    """The batched workload: args.models slip-weakening models of uneven size (fault 8-24 x
    6-14 km, h = 200 m, 8 s simulated) in one batch, the schedule and tile shape tuned on
    the live batch first, against the same models solved one at a time through the
    single-model path (create, upload, run, read back, destroy).  Solves/s and cell
    updates/s are wall clock over the whole run; the HBM fraction is the batch's
    algorithmic bytes (PML split components counted) over its GPU time."""
    from fd3d_tsn_b200 import configs
    from fd3d_tsn_b200.batch import Batch, bytes_needed
    from fd3d_tsn_b200.solver import lib
    from fd3d_tsn_b200.serve import plain
    lib().fd3d_set_device(local)
    models = configs.batch_set(args.models, seed=2024 + rank)
    for q, m in enumerate(models):
        m["request"] = q
    cells = sum(m["nxt"] * m["nyt"] * m["nzt"] * m["ntfd"] for m in models)
    alg_bytes = sum(step_bytes(m) * m["ntfd"] for m in models)
    arena = int(sum(bytes_needed(m) for m in models) * 1.05) + (64 << 20)
    t_setup = time.perf_counter()
    b = Batch(arena, len(models) + 8)
    slots = [b.add(m) for m in models]
    if args.batch_schedule == "auto":
        tune = b.autotune(steps=10, cache_path=os.path.join(tempfile.gettempdir(), "fd3d_batch_tune.jsonl"),
                          key=f"batch{len(models)}-seed{2024 + rank}")
    else:  # a fixed schedule at its usual tile depth, no tuning launches
        b.set_schedule(args.batch_schedule)
        b.set_tuning(32 if args.batch_schedule == "graph" else 8, 3 if args.batch_schedule == "persistent" else 0)
        tune = b.tuning()
    t_setup = time.perf_counter() - t_setup
    barrier(pg, local)
    t0 = time.perf_counter()
    gpu = 0.0
    nmax = max(m["ntfd"] for m in models)
    done = 0
    while done < nmax:
        b.run(64)
        b.sync()
        gpu += b.last_run_ms() / 1e3
        done += 64
    finals = {q: b.final(s) for q, s in zip(range(len(models)), slots)}
    wall = time.perf_counter() - t0
    b.close()
    wall_max = max_over_ranks(pg, local, wall)
    ref, t_plain = plain(models)
    t_plain_max = max_over_ranks(pg, local, t_plain)
    identical = all(_same_finals(finals[q], ref[q]) for q in ref)
    peak, peak_kind = measured_peak()
    rate = whole_job_rate(len(models), world, wall_max)
    plain_rate = whole_job_rate(len(models), world, t_plain_max)
    return {"metric": "batched solves/s", "value": rate, "unit": "solves/s",
            "config": {"workload": "batch", "models": len(models), "h_m": 200.0, "sim_s": 8.0,
                       "cells_x_steps": cells, "fault_km": [[8, 24], [6, 14]]},
            "gcell_updates_per_s": cells * world / wall_max / 1e9, "wall_s": wall_max, "gpu_s": gpu,
            "setup_s": t_setup,
            "hbm": {"algorithmic_bytes": alg_bytes, "gbs_on_gpu_time": alg_bytes / gpu / 1e9,
                    "frac": alg_bytes / gpu / 1e9 / peak, "peak": peak, "peak_source": peak_kind,
                    "bytes_per_cell": "108 B per interior cell, 264 B per PML cell (split components counted)"},
            "tuning": tune,
            "plain": {"solves_per_s": plain_rate, "wall_s": t_plain_max,
                      "gcell_updates_per_s": cells * world / t_plain_max / 1e9},
            "speedup_vs_plain": rate / plain_rate,
            "results_identical_to_plain": identical}


def serve_section(args, world, rank, local, pg):
    """Continuous batching of a Poisson stream of mixed-size requests (95% batch-size
    models, 5% large h = 100 m models, args.sim_time simulated seconds each).  The
    schedule and tile shape are tuned once on a sample of the mix before traffic (a
    server warms up before it takes requests).  Two runs of the same stream: every
    request arriving at once (capacity: the reported solves/s) and Poisson arrivals at
    args.load of that capacity (p50 / p99 latency under load), against one-at-a-time
    plain solves of a sample of the stream."""
    from fd3d_tsn_b200 import configs
    from fd3d_tsn_b200.serve import plain, pretune, serve
    from fd3d_tsn_b200.solver import lib
    lib().fd3d_set_device(local)
    stream = configs.serving_stream(args.requests, seed=4242 + rank, rate=1.0, sim_time=args.sim_time)
    sample = set(range(0, len(stream), max(1, len(stream) // args.plain_sample)))
    budget = int(args.hbm_gb * (1 << 30))
    t_tune = time.perf_counter()
    tuning = pretune([m for _, m in stream[:64]],
                     cache_path=os.path.join(tempfile.gettempdir(), "fd3d_batch_tune.jsonl"),
                     key=f"serve-{args.sim_time}-{args.requests}-{rank}")
    t_tune = time.perf_counter() - t_tune
    burst = [(0.0, m) for _, m in stream]
    barrier(pg, local)
    _, cap = serve(burst, budget, chunk=32, tuning=tuning, keep_final=lambda r: False)
    cap_max = max_over_ranks(pg, local, cap["makespan_s"])
    capacity = whole_job_rate(cap["requests"], world, cap_max)
    # the same requests arriving as a Poisson stream at args.load of the measured capacity
    rate = args.load * cap["requests"] / cap_max
    gaps = np.random.default_rng(4243 + rank).exponential(1.0 / rate, size=len(stream))
    timed = [(float(t), m) for t, (_, m) in zip(np.cumsum(gaps), stream)]
    results, stats = serve(timed, budget, chunk=32, tuning=tuning, keep_final=lambda r: r in sample)
    byreq = {r.request: r for r in results}
    ref, t_plain = plain([m for q, (_, m) in enumerate(stream) if q in sample], keep_final=lambda r: True)
    identical = all(_same_finals(byreq[q].final, ref[q]) for q in ref)
    plain_rate = len(ref) / max_over_ranks(pg, local, t_plain) * world
    nlarge = sum(1 for _, m in stream if m["dh"] == 100.0)
    return {"metric": "serving solves/s", "value": capacity, "unit": "solves/s",
            "config": {"workload": "serve", "requests": len(stream), "large_requests": nlarge,
                       "large_fraction": 0.05, "sim_s": args.sim_time, "hbm_budget_gb": args.hbm_gb,
                       "offered_rate_per_s": rate, "offered_load_of_capacity": args.load},
            "p50_latency_s": stats["p50_latency_s"], "p99_latency_s": stats["p99_latency_s"],
            "offered_load": stats, "capacity": cap, "tuning": tuning, "tuning_s": t_tune,
            "plain": {"solves_per_s": plain_rate, "sample": len(ref), "wall_s": t_plain},
            "speedup_vs_plain": capacity / plain_rate,
            "results_identical_to_plain": identical}


def _line(sec, world):
    out = dict(sec)
    out.update(n_gpus=world, higher_is_better=True, scaling="weak", dtype="f32", data="synthetic")
    return out


def run_batch_bench(args, world, rank, local, pg):
    sec = batch_section(args, world, rank, local, pg)
    if rank == 0:
        print(json.dumps(_line(sec, world)), flush=True)


def run_serve_bench(args, world, rank, local, pg):
    sec = serve_section(args, world, rank, local, pg)
    if rank == 0:
        print(json.dumps(_line(sec, world)), flush=True)


def _free_port():
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def relaunch(ngpus):
    """bench.py --gpus N started as a plain process: run it again as N ranks under
    torch.distributed.run (one process per GPU, rendezvous on 127.0.0.1)."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(ngpus),
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.abspath(__file__),
           *sys.argv[1:]]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--models", type=int, default=256, help="batched workload: number of models")
    ap.add_argument("--batch-schedule", default="auto", choices=["auto", "graph", "persistent"],
                    help="batched workload: tune the schedule on the live batch, or fix it")
    ap.add_argument("--requests", type=int, default=500, help="serving workload: number of requests")
    ap.add_argument("--load", type=float, default=0.7,
                    help="serving workload: offered Poisson rate as a fraction of the measured capacity")
    ap.add_argument("--sim-time", type=float, default=8.0, help="serving workload: simulated seconds per request")
    ap.add_argument("--plain-sample", type=int, default=32, help="serving workload: plain solves timed")
    ap.add_argument("--hbm-gb", type=float, default=120.0, help="serving workload: arena (HBM budget) in GB")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="sw_large")
    ap.add_argument("--cpu-baseline", type=float, default=15.0, help="seconds of oracle time (0 = skip)")
    ap.add_argument("--ref-seconds", type=float, default=60.0, help="reference arm: CPU seconds to time")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-batch", dest="batch", action="store_false",
                    help="leave the batched workload out of the default line")
    ap.add_argument("--no-serve", dest="serve", action="store_false",
                    help="leave the serving workload out of the default line")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    ws = os.environ.get("WORLD_SIZE")
    if ws is None and args.gpus > 1:
        sys.exit(relaunch(args.gpus))
    if ws is not None and int(ws) != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={ws}", file=sys.stderr)
        sys.exit(2)
    world, rank, local, pg = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank, local, pg)
        elif args.workload == "batch":
            run_batch_bench(args, world, rank, local, pg)
        elif args.workload == "serve":
            run_serve_bench(args, world, rank, local, pg)
        else:
            run_b200(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
