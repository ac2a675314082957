"""The multi-process path on CPU: two gloo ranks join, agree on the maximum of their
timings, pass barriers, and shard ensemble members disjointly and completely; and each
rank steps its own shard of perturbed members (one union model per rank, on the oracle,
as ``bench.py --workload ensemble`` does on GPUs), every member ending bitwise equal to
the same member stepped alone in one process."""
import hashlib
import os
import socket

import numpy as np
import pytest

MEMBER_FIELDS = ("el", "ua", "va", "u", "v", "t1", "s1", "q2", "km")


def _small_coastal():
    from myfvcomcode_b200 import cases
    return cases.coastal_mesh(npts=1500, kb=7, lx=20000.0, ly=10000.0, seed=7, IRAMP=20)


def _digest(arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


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


def _member_rank(rank, world, port, q, nmem, steps):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from myfvcomcode_b200 import dist, ensemble
    from oracle.oracle import Oracle, set_threads
    set_threads(1)
    d = dist.setup(backend="gloo", timeout_s=60)
    base = _small_coastal()
    specs = ensemble.perturbed_members(base, nmem, seed=4)
    mine = dist.shard(list(range(nmem)), d.rank, d.world)
    out = {}
    peak = 0.0
    if mine:
        u = ensemble.union_case(base, [specs[m] for m in mine])
        o = Oracle(u)
        o.run(steps)
        for j, m in enumerate(mine):
            out[m] = _digest([ensemble.member_slice(u, j, f, o) for f in MEMBER_FIELDS])
        peak = float(np.abs(o.get("el")).max())
        o.close()
    d.barrier()
    peak = d.reduce_max(peak)
    d.close()
    q.put((rank, out, peak))


def test_two_gloo_ranks_step_their_member_shards():
    """Each of two ranks steps its shard of three perturbed members as one union model
    for two internal steps; every member is bitwise equal to the member stepped alone."""
    import torch.multiprocessing as mp
    from myfvcomcode_b200 import ensemble
    from oracle.oracle import Oracle
    nmem, steps = 3, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_member_rank, args=(r, 2, port, q, nmem, steps)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=300) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    got = {}
    for _, out, _ in res:
        assert not (set(out) & set(got))
        got.update(out)
    assert sorted(got) == list(range(nmem))
    base = _small_coastal()
    specs = ensemble.perturbed_members(base, nmem, seed=4)
    peak = 0.0
    for m, sp in enumerate(specs):
        o = Oracle(ensemble.member_case(base, sp))
        o.run(steps)
        assert got[m] == _digest([o.get(f) for f in MEMBER_FIELDS]), m
        peak = max(peak, float(np.abs(o.get("el")).max()))
        o.close()
    assert res[0][2] == res[1][2] == peak
