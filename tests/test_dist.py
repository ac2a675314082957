"""The multi-process path on CPU: two gloo ranks join, agree on the maximum of their
timings, pass barriers, and shard ensemble members disjointly and completely."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from myfvcomcode_b200 import dist, ensemble
    d = dist.setup(backend="gloo", timeout_s=60)
    m = d.reduce_max(1.5 + rank)
    d.barrier()
    specs = ensemble.perturbed_members(None, 11, seed=2)
    mine = dist.shard(list(range(len(specs))), d.rank, d.world)
    d.barrier()
    d.close()
    q.put((rank, m, mine))


def test_two_gloo_ranks_reduce_and_shard():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][1] == out[1][1] == 2.5
    a, b = set(out[0][2]), set(out[1][2])
    assert not (a & b) and (a | b) == set(range(11))
