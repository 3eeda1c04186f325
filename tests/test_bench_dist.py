"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (torchrun's
environment, rendezvous on 127.0.0.1).  Every rank runs its own replica of
the workload; the reported time is the slowest rank's, and under
--impl reference only rank 0 works and prints."""
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


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        got = bench.max_over_ranks([1.0 + rank, 5.0 - rank, 3.0], ws)
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0] == res[1] == [2.0, 5.0, 3.0]


def test_max_over_ranks_single_rank():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([1.5, 2.5], 1) == [1.5, 2.5]


def test_reference_arm_other_ranks_exit_without_work():
    """Under torchrun with N > 1, ranks other than 0 of the reference arm exit
    0 at once and print nothing."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
