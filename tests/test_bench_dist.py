"""Multi-rank plumbing of bench.py on CPU (gloo, world_size 2).

With N GPUs every rank factors and solves its own replica of the workload
(the single-GPU path has no exchange step), so the only collectives are the
barriers around the timed region and the max of the per-rank times.  These
tests run that host logic as two gloo ranks, and the reference arm under
torchrun, where rank 0 alone works and prints.
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


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist = bench.dist_init("gloo")
    try:
        bench.barrier(dist)
        # per-rank "step times": the job time is the slowest replica's
        mx = bench.max_over_ranks(10.0 + 7.5 * rank, dist)
        mn = -bench.max_over_ranks(-(10.0 + 7.5 * rank), dist)
        bench.barrier(dist)
        q.put((rank, bench.rank_env(), mx, mn))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=5) for _ in range(world))
    for rank, (r, w, local), mx, mn in got:
        assert (r, w, local) == (rank, world, rank)
        assert mx == 17.5 and mn == 10.0


def test_single_process_plumbing():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.dist_init("gloo") is None
    assert bench.max_over_ranks(3.25, None) == 3.25
    bench.barrier(None)


def test_reference_arm_torchrun_two_ranks():
    """`bench.py --impl reference` under torchrun: rank 0 prints one JSON line, rank 1 exits 0 without work."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--grid", "14",
           "--nrhs", "2", "--cutoff", "64", "--cpu-budget", "0.2"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["higher_is_better"] is False and line["unit"] == "s"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
