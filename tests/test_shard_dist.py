"""The exchange of the sharded brute-force gravity (ncorpion_b200/shard.py) on
CPU: two and three gloo ranks, each holding its part of the field the way
ncgpu_vector_field_part writes it (its targets' rows, -0.0 elsewhere, +0.0
for empty slots from part 0).  The all-reduce sum must give every rank the
full field bit for bit, signed zeros included.  The field itself comes from
the oracle here (CPU ranks); the GPU test of the parts is in
tests/test_shard_gpu.py."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def full_field():
    """A brute-force field from the oracle with holes, plus signed zeros
    planted in some rows (the combine must keep the sign of every value)."""
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    from conftest import make_params
    from ncorpion_b200 import disks
    n = 301
    b = disks.gravity_disk(n, seed=5)
    rng = np.random.default_rng(5)
    ex = (rng.random(n) > 0.1).astype(np.int32)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    acc, cma = oracle.Port().vector_field(b, ex, cm, make_params(softening_parameter=0.5))
    live = np.flatnonzero(ex)
    acc[live[7], 1] = -0.0
    acc[live[8], 2] = 0.0
    acc[ex == 0] = 0.0
    return acc, cma, ex


def part_rows(acc, ex, part, nparts):
    """What part `part` of `nparts` holds in the exact mode."""
    from ncorpion_b200.shard import part_slice
    live = np.flatnonzero(ex)
    lo, hi = part_slice(len(live), part, nparts)
    out = np.full_like(acc, -0.0)
    out[live[lo:hi]] = acc[live[lo:hi]]
    if part == 0:
        out[ex == 0] = 0.0
    return out


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    from ncorpion_b200.shard import ShardedField
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        acc, cma, ex = full_field()

        def compute(part, nparts, d_acc, d_cma):
            d_acc.copy_(torch.from_numpy(part_rows(acc, ex, part, nparts)))
            d_cma.copy_(torch.from_numpy(cma))

        sf = ShardedField(compute=compute)
        assert (sf.rank, sf.world) == (rank, ws)
        d_acc = torch.empty(acc.shape, dtype=torch.float64)
        d_cma = torch.empty(3, dtype=torch.float64)
        sf.vector_field(None, None, None, 0, d_acc, d_cma)
        got = d_acc.numpy()
        q.put((rank, bool(np.array_equal(got.view(np.int64), acc.view(np.int64))),
               bool(np.array_equal(d_cma.numpy(), cma))))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ws", [2, 3])
def test_sharded_field_sum_is_the_full_field(ws):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = dict((r, (a, c)) for r, a, c in (q.get(timeout=180) for _ in range(ws)))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(res[r] == (True, True) for r in range(ws)), res


def test_part_slices_cover_every_item_once():
    sys.path.insert(0, ROOT)
    from ncorpion_b200.shard import part_slice
    for n in (0, 1, 7, 128, 1000):
        for nparts in (1, 2, 3, 8):
            s = [part_slice(n, p, nparts) for p in range(nparts)]
            assert s[0][0] == 0 and s[-1][1] == n
            assert all(s[i][1] == s[i + 1][0] for i in range(nparts - 1))


def test_negative_zero_is_the_identity_of_the_sum():
    """The property the exchange rests on: x + (-0.0) == x bit for bit for
    every double x, signed zeros included, in any order of the additions."""
    xs = np.array([0.0, -0.0, 1.5, -2.25e-300, 5e-324, np.inf], dtype=np.float64)
    for x in xs:
        for y in (x + -0.0, -0.0 + x, (-0.0 + -0.0) + x):
            assert np.float64(y).view(np.int64) == np.float64(x).view(np.int64)
