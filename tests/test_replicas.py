"""The multi-GPU run's host logic on CPU: two ranks over gloo (127.0.0.1).
Each rank is a replica with its own query stream; the job's time is the
largest per-rank time, counts add up, and the reference arm does its work on
rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from ahead_b200.replicas import Replicas
    g = Replicas("gloo", timeout_s=60)
    g.barrier()
    t = g.max(1.5 + rank)          # per-rank elapsed times
    n = g.sum(64 * (rank + 1))     # queries each replica answered
    q.put((rank, g.seed(1), t, n))
    g.close()


def test_two_replicas_over_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[1] for g in got] == [1, 1001]           # different query streams per replica
    assert all(g[2] == 2.5 for g in got)              # the job's time: the slowest rank
    assert all(g[3] == 64 * 3 for g in got)           # counts summed over ranks


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    from ahead_b200.replicas import Replicas
    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK") if k in os.environ}
    try:
        g = Replicas("gloo")
        assert g.world == 1 and g.max(3.0) == 3.0 and g.sum(2) == 2.0
        g.barrier()
        g.close()
    finally:
        os.environ.update(env)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
