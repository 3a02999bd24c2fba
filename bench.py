#!/usr/bin/env python3
"""Throughput of the FD3D_TSN time step on B200.

Default workload: the slip-weakening production model (1000 x 400 x 500 simulated cells,
1020 x 410 x 512 padded = 214.1 M cells, h = 50 m, 5 seeded layers, FP32 wave field
with FP64 slip / rupture-time accumulators).  A *step* is one pass of the time loop
(velocity + stress sweeps, PML strips, free surface, fault boundary condition and the
history planes) over the whole grid.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line.  value = padded cells x steps x N / max-over-ranks device time.
Under torchrun (N>1) every rank runs its own independent model (replicas; the path has
no exchange step), so scaling is weak.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

B_ALG_STEP = 120          # algorithmic FP32 bytes per cell per step (velocity 52 + stress 68)
B_ALG_STR = 68            # stress sweep: 3 v + lam + mu + 6 sigma loads, 6 sigma stores
B_ALG_VEL = 52            # velocity sweep: 6 sigma + rho + 3 v loads, 3 v stores
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


def dist_setup(ngpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def barrier(pg, local):
    if pg is not None:
        import torch
        pg.barrier(device_ids=[local])
        torch.cuda.synchronize()


def max_over_ranks(pg, local, v):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{local}")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


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
            "fields": "fp32", "accumulators": "fp64",
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
    for _ in range(args.warmup):
        o.step(1, history=True)
    t0 = time.perf_counter()
    o.step(args.steps, history=True)
    dt = time.perf_counter() - t0
    cells = m["nxt"] * m["nyt"] * m["nzt"]
    v = cells * args.steps / dt / 1e9
    line = {"impl": "reference", "metric": "GCell-updates/s", "value": v, "unit": "GCell-updates/s",
            "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": describe(args.workload, m),
            "cpu_baseline": {"value": v, "unit": "GCell-updates/s", "cores": om.num_threads(), "kind": "port",
                             "sample": f"{args.steps} whole time steps with history planes, all host threads"},
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
    value = cells * args.steps * world / (ms_max / 1e3) / 1e9

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
    dom, dom_ms, dom_bytes = ("str_interior", kstr_ms, B_ALG_STR * interior) if kstr_ms >= kvel_ms else \
        ("vel_interior", kvel_ms, B_ALG_VEL * interior)
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    step_gbs = cells * B_ALG_STEP / (ms / args.steps / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get(args.workload, {}).get(dom)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
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
        e2e["value"] = cells * args.steps * world / e2e_v / 1e9

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
        print(json.dumps(line), flush=True)


def gpu_launches(m, steps):
    per_step = 11 + (1 if m.get("law") == "fvw" and m["fault"].get("nucleation") else 0)
    return per_step * steps


def pinned(shape, dtype):
    """Page-locked host array (cudaHostAlloc through torch)."""
    import torch
    t = torch.empty(int(np.prod(shape)), dtype=torch.float32 if dtype == np.float32 else torch.float64,
                    pin_memory=True)
    return t.numpy().reshape(shape, order="F"), t


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
    nf = 4
    hist, th = pinned((steps, nf, plane), np.float32)
    keep.append(th)
    nst = len(m.get("stations", []))
    seis = np.empty((steps, max(nst, 1), 3))
    s = Solver(m)           # context + fault; its medium is replaced inside the timed region
    s.run(0)
    s.sync()
    s.reset()
    t0 = time.perf_counter()
    s.upload_medium_arrays(*host, real_kind=4)
    s.upload_fault(m["fault"])
    s.run(steps)
    s.sync()
    for f in range(nf):
        rc = lib().fd3d_fetch_history(s.h, f, 0, steps, hist[:, f].ctypes.data, 4)
        if rc:
            raise abi.Fd3dError(rc, "fd3d_fetch_history")
    if nst:
        lib().fd3d_fetch_stations(s.h, 0, steps, seis.ctypes.data_as(C.POINTER(C.c_double)))
    dt = time.perf_counter() - t0
    s.close()
    fault_bytes = 6 * m["nxt"] * m["nzt"] * 8
    h2d = 3 * int(np.prod(shp)) * 4 + fault_bytes
    d2h = nf * plane * 4 + nst * 3 * 8
    return {"unit": "GCell-updates/s", "h2d_bytes_per_step": h2d / steps, "d2h_bytes_per_step": d2h,
            "_seconds": dt, "includes": "medium (fp32, pinned) + fault upload, K steps, K history records of 4 "
                                        "planes + stations read back; wall clock"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="sw_large")
    ap.add_argument("--cpu-baseline", type=float, default=15.0, help="seconds of oracle time (0 = skip)")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local, pg = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank, local, pg)
        else:
            run_b200(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
