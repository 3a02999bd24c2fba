"""Multi-process plumbing of bench.py on CPU (gloo, world size 2).

The path shards only as replicas: the process group carries the barrier around the
timed region and the max-over-ranks reduction of the timings, nothing else.  These
tests run that plumbing with the gloo backend and check the whole-job aggregate, and
run the reference arm under torchrun, where rank 0 alone works and prints, and as a plain
process with --gpus 2, which starts the two ranks itself.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank), FD3D_BENCH_BACKEND="gloo")
    sys.path.insert(0, ROOT)
    import bench
    w, r, local, pg = bench.dist_setup(world)
    try:
        bench.barrier(pg, local)
        # rank r "took" 1 + r seconds for its replica of 1000 units
        t = bench.max_over_ranks(pg, local, 1.0 + r)
        out.put((r, w, t, bench.whole_job_rate(1000, w, t)))
    finally:
        pg.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(world))
    for r, w, t, rate in got:
        assert w == world
        assert t == 2.0                      # the slower rank's time
        assert rate == pytest.approx(1000.0)  # 2 ranks x 1000 units / 2 s


def test_reference_arm_under_torchrun_prints_once():
    port = _free_port()
    env = dict(os.environ, FD3D_BENCH_BACKEND="gloo", FD3D_ORACLE_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--workload", "sw_small", "--steps", "2", "--warmup", "3", "--ref-seconds", "1"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference"
    assert line["metric"] == "GCell-updates/s" and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["value"] > 0


def test_gpus_flag_starts_the_ranks_itself():
    """bench.py --gpus 2 run as a plain process (no WORLD_SIZE) relaunches itself as two
    ranks under torch.distributed.run, and rank 0 alone prints the line."""
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    env.update(FD3D_BENCH_BACKEND="gloo", FD3D_ORACLE_THREADS="2")
    cmd = [sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--workload", "sw_small",
           "--steps", "2", "--warmup", "3", "--ref-seconds", "1"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1 and lines[0]["impl"] == "reference"


def test_gpus_flag_must_match_the_rank_count():
    env = dict(os.environ, WORLD_SIZE="2", RANK="0", LOCAL_RANK="0", FD3D_BENCH_BACKEND="gloo")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--gpus", "3"], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 2 and "WORLD_SIZE=2" in r.stderr


def _slab_rank_main(rank, world, port, out):
    """The host side of z-slabs in separate processes: every rank gets its own plane
    range and the id rank 0 made (the NCCL call itself needs GPUs; a fixed id stands
    in for ncclGetUniqueId here)."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from fd3d_tsn_b200 import configs
    from fd3d_tsn_b200.slab import rank_setup
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = configs.sw_small()
        rng, uid = rank_setup(m, rank, world, lambda o: dist.broadcast_object_list(o, src=0),
                              make_id=lambda: bytes(range(128)))
        out.put((rank, rng, uid))
    finally:
        dist.destroy_process_group()


def test_slab_ranks_get_their_planes_and_one_id():
    world = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_slab_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(world))
    assert all(uid == bytes(range(128)) for _, _, uid in got)
    ranges = [rng for _, rng, _ in got]
    assert ranges[0][0] == 1 and ranges[-1][1] == 132          # sw_small: nzt = 132
    assert all(ranges[r][0] == ranges[r - 1][1] + 1 for r in range(1, world))
