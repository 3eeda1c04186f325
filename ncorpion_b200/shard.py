"""Brute-force gravity with its targets split over several GPUs.

One process per GPU (torch.distributed, NCCL over NVLink between the GPUs).
Every rank holds the whole body state -- the reference's own data model, in
which every body sees every other -- and evaluates the field of its part of
the targets with ``ncgpu_vector_field_part``: the part-th slice of the
existing bodies in slot order in the exact mode, of the Morton-ordered
128-body target blocks in the FP64 and mixed modes.  The rows of the other
targets hold -0.0, the identity of IEEE addition, so one all-reduce sum of the
3 doubles per body assembles on every rank the field a single GPU computes,
bit for bit (each element receives exactly one value that is not -0.0).
CM_acc needs no exchange: every part computes the full one from the O(N)
central terms.  That all-reduce is the path's only exchange step; the kick and
drift that follow are replicated (identical on every rank).
"""
from __future__ import annotations

import ctypes as C

from . import api


def part_slice(n: int, part: int, nparts: int) -> tuple[int, int]:
    """[lo, hi) of the part-th of nparts slices of n items, the split the
    library uses for compacted bodies (exact) and for target blocks (tiled)."""
    return n * part // nparts, n * (part + 1) // nparts


class ShardedField:
    """vector_field over the ranks of a process group.

    ``compute(part, nparts, d_acc, d_cm_acc)`` may replace the library call
    (tests of the exchange on CPU ranks); by default it is
    ``ncgpu_vector_field_part`` on the given device buffers.
    """

    def __init__(self, group=None, compute=None):
        import torch.distributed as dist
        self.group = group
        self.distributed = dist.is_available() and dist.is_initialized()
        self.rank = dist.get_rank(group) if self.distributed else 0
        self.world = dist.get_world_size(group) if self.distributed else 1
        self.compute = compute

    def _library_part(self, d_bodies, d_exists, cm, mode, d_acc, d_cm_acc, stream):
        lib = api.load()
        n = d_bodies.shape[0]
        sp = C.c_void_p(stream.cuda_stream) if stream is not None else None
        st = lib.ncgpu_vector_field_part(C.c_void_p(d_bodies.data_ptr()), C.c_void_p(d_exists.data_ptr()), n - 1,
                                         api.ptr(cm), self.rank, self.world, C.c_void_p(d_acc.data_ptr()),
                                         C.c_void_p(d_cm_acc.data_ptr()), mode, sp)
        api.check(st, "ncgpu_vector_field_part")

    def vector_field(self, d_bodies, d_exists, cm, mode, d_acc, d_cm_acc, stream=None):
        """Accelerations of all bodies into d_acc (n x 3) and CM_acc into
        d_cm_acc (3), on every rank.  d_bodies: n x 8 (struct moonlet layout),
        d_exists: n int32, cm: 8 doubles (host numpy).  The library work is
        ordered on `stream` and the all-reduce follows it on the current torch
        stream, so call this inside ``torch.cuda.stream(stream)``."""
        if self.compute is not None:
            self.compute(self.rank, self.world, d_acc, d_cm_acc)
        else:
            self._library_part(d_bodies, d_exists, cm, mode, d_acc, d_cm_acc, stream)
        if self.world > 1:
            import torch.distributed as dist
            dist.all_reduce(d_acc, op=dist.ReduceOp.SUM, group=self.group)
        return d_acc, d_cm_acc
