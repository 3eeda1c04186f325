"""GPU: the parts of the sharded brute-force gravity (ncgpu_vector_field_part)
on one GPU.  Every part of a split is evaluated in turn; the sum of their
outputs must be the full field (bit for bit in the exact mode, where each
part computes its targets exactly as the whole does), each existing body's
row must come from exactly one part (-0.0 in all the others), and CM_acc
must be the full one in every part.  FP64 / mixed: the parts split the
Morton-ordered target blocks, whose source chunking then differs from the
whole's, so their sum is compared within the modes' tolerances (relative
1e-12 and 2e-6)."""
import ctypes as C

import numpy as np
import pytest

from conftest import make_params

pytestmark = pytest.mark.gpu

NEG0 = np.float64(-0.0).view(np.int64)


def _run(lib, api, torch, b, ex, cm, mode, part, nparts):
    n = b.shape[0]
    d_b = torch.from_numpy(b).cuda()
    d_ex = torch.from_numpy(ex).cuda()
    d_acc = torch.full((n, 3), np.nan, dtype=torch.float64, device="cuda")
    d_cma = torch.full((3,), np.nan, dtype=torch.float64, device="cuda")
    st = lib.ncgpu_vector_field_part(C.c_void_p(d_b.data_ptr()), C.c_void_p(d_ex.data_ptr()), n - 1, api.ptr(cm),
                                     part, nparts, C.c_void_p(d_acc.data_ptr()), C.c_void_p(d_cma.data_ptr()),
                                     mode, None)
    api.check(st, "ncgpu_vector_field_part")
    torch.cuda.synchronize()
    return d_acc.cpu().numpy(), d_cma.cpu().numpy()


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("n", [129, 5000])
def test_parts_sum_to_the_full_field(lib, mode, n):
    import torch
    from ncorpion_b200 import api, disks
    b = disks.gravity_disk(n, seed=n)
    rng = np.random.default_rng(n)
    ex = (rng.random(n) > 0.05).astype(np.int32)
    cm = np.array([1e-6, 0.0, -1e-6, 0, 0, 0, 1.0, 1.0])
    api.init(n, make_params(softening_parameter=0.5, gravity_mode=mode))
    try:
        full, cma_full = _run(lib, api, torch, b, ex, cm, mode, 0, 1)
        live = ex == 1
        for nparts in (2, 3, 7, 64):
            tot = np.full_like(full, -0.0)
            owners = np.zeros(n, np.int32)
            for part in range(nparts):
                acc, cma = _run(lib, api, torch, b, ex, cm, mode, part, nparts)
                assert np.array_equal(cma, cma_full) if mode == 0 else np.allclose(cma, cma_full, rtol=1e-12)
                mine = ~(acc.view(np.int64) == NEG0).all(axis=1)
                owners += mine & live
                if part > 0:
                    assert (acc[~live].view(np.int64) == NEG0).all()
                tot = tot + acc
            assert (owners[live] == 1).all(), "a body's row must come from exactly one part"
            assert not tot[~live].any() and not np.signbit(tot[~live]).any()
            if mode == 0:
                assert np.array_equal(tot.view(np.int64), full.view(np.int64))
            else:
                rel = np.linalg.norm(tot[live] - full[live], axis=1) / np.linalg.norm(full[live], axis=1)
                assert rel.max() <= (1e-12 if mode == 1 else 2e-6)
    finally:
        api.finalize()


def test_sharded_field_single_rank_is_the_whole(lib):
    """ShardedField without a process group: part 0 of 1, no exchange."""
    import torch
    from ncorpion_b200 import api, disks
    from ncorpion_b200.shard import ShardedField
    n = 3000
    b = disks.gravity_disk(n, seed=3)
    ex = np.ones(n, np.int32)
    cm = np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])
    api.init(n, make_params(softening_parameter=0.5))
    try:
        full, cma_full = _run(lib, api, torch, b, ex, cm, 0, 0, 1)
        sf = ShardedField()
        assert (sf.rank, sf.world) == (0, 1)
        d_acc = torch.empty((n, 3), dtype=torch.float64, device="cuda")
        d_cma = torch.empty(3, dtype=torch.float64, device="cuda")
        stream = torch.cuda.Stream()
        with torch.cuda.stream(stream):
            sf.vector_field(torch.from_numpy(b).cuda(), torch.from_numpy(ex).cuda(), cm, 0, d_acc, d_cma, stream)
        torch.cuda.synchronize()
        assert np.array_equal(d_acc.cpu().numpy(), full) and np.array_equal(d_cma.cpu().numpy(), cma_full)
    finally:
        api.finalize()


def test_part_arguments_checked(lib):
    import torch
    from ncorpion_b200 import api
    api.init(16, make_params())
    try:
        b = np.zeros((4, 8))
        ex = np.ones(4, np.int32)
        for part, nparts in ((0, 0), (2, 2), (-1, 3)):
            d_b = torch.from_numpy(b).cuda()
            d_ex = torch.from_numpy(ex).cuda()
            out = torch.zeros((4, 3), dtype=torch.float64, device="cuda")
            cma = torch.zeros(3, dtype=torch.float64, device="cuda")
            st = lib.ncgpu_vector_field_part(C.c_void_p(d_b.data_ptr()), C.c_void_p(d_ex.data_ptr()), 3,
                                             api.ptr(np.array([0, 0, 0, 0, 0, 0, 1.0, 1.0])), part, nparts,
                                             C.c_void_p(out.data_ptr()), C.c_void_p(cma.data_ptr()), 0, None)
            assert st == api.E_ARG
    finally:
        api.finalize()


def test_bench_two_ranks_share_one_gpu():
    """bench.py's multi-rank path (the gravity headline split over the ranks,
    one all-reduce per step) with two ranks on one GPU over gloo: it runs to
    the end and reports the whole field's accuracy unchanged.  (NCCL needs one
    GPU per rank; the collective here goes through the host.)"""
    import json
    import os
    import socket
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), os.path.join(root, "bench.py"), "--gpus", "2", "--steps", "3",
           "--warmup", "3", "--dist-backend", "gloo", "--no-mesh", "--no-frag", "--no-bf", "--no-adjoint",
           "--no-central", "--no-output", "--no-cpu-baseline"]
    r = subprocess.run(cmd, cwd=root, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    out = json.loads(lines[0])
    assert out["n_gpus"] == 2 and out["scaling"] == "strong"
    assert out["accuracy"]["mutual_rel_err_max"] < 1e-6
    assert out["accuracy"]["total_rel_err_max"] < 1e-8
