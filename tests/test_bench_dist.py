"""Multi-process plumbing of bench.py on CPU (gloo, world size 2): the max-over-ranks
timing reduction, the barrier, and the reference arm's rank-0-only rule.  The GPU replicas
use the same helpers over NCCL."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist = bench.init_dist(ws, "gloo")
    try:
        got_ws, got_rank, _ = bench.dist_env()
        bench.barrier(dist)
        # each rank's "timed region" differs; every rank must see the maximum
        m = bench.max_over_ranks(10.0 + 5.0 * rank, dist)
        bench.barrier(dist)
        q.put((rank, got_ws, got_rank, m))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_barrier_gloo_ws2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [(0, 2, 0, 15.0), (1, 2, 1, 15.0)]


def test_single_process_helpers_are_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25, None) == 3.25
    bench.barrier(None)


@pytest.mark.parametrize("rank", [1])
def test_reference_arm_non_zero_rank_exits_without_work(rank):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
