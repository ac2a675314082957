"""Process-group plumbing of multi-GPU runs: one process per GPU.

A single mesh does not shard across GPUs here (replicas only); ensemble members do:
``shard`` deals members to ranks round-robin with no data-path collective.  The only
collectives are the barrier around a timed region and the maximum of the ranks' times.
NCCL on GPUs, gloo on CPU (the tests).
"""
from __future__ import annotations

import os
from datetime import timedelta


class Dist:
    def __init__(self, world, rank, local, pg, backend):
        self.world, self.rank, self.local, self.pg, self.backend = world, rank, local, pg, backend

    def _dev(self):
        return "cuda:%d" % self.local if self.backend == "nccl" else "cpu"

    def reduce_max(self, x):
        if self.pg is None:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self._dev())
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def barrier(self):
        if self.pg is None:
            return
        if self.backend == "nccl":
            import torch
            torch.cuda.synchronize(self.local)
        self.pg.barrier()

    def close(self):
        if self.pg is not None:
            self.pg.destroy_process_group()
            self.pg = None


def setup(backend=None, timeout_s=600):
    """Join the process group described by RANK / WORLD_SIZE / LOCAL_RANK / MASTER_*."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world <= 1:
        return Dist(1, 0, local, None, None)
    import torch
    import torch.distributed as dist
    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return Dist(world, rank, local, dist, backend)


def shard(items, rank, world):
    """Round-robin share of ``items`` for ``rank`` of ``world``."""
    return [x for i, x in enumerate(items) if i % world == rank]
