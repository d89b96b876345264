"""Multi-rank host logic on CPU (gloo, world size 2): cage sharding, the
max-over-ranks timing reduction, and a rank that fails between steps.

The refinement itself is per cage (no exchange between cages), so a sharded
batch must give, cage by cage, the unsharded result: each rank refines its
shard with the oracle and rank 0 compares the gathered digests with a
one-process run.
"""
import hashlib
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _cages():
    from halfedgecatmullclark_b200 import configs
    return configs.batch_cages(count=10, fmin=8, fmax=40, dmin=1, dmax=2, seed=9)


def _digest(w):
    from oracle import oracle
    he, cr, pts = oracle.refine(w.cage, w.depth, "scatter")
    h = hashlib.sha256()
    for a in (he, cr, pts):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def _init(rank, world, port, timeout_s=30):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=timeout_s))


def _shard_worker(rank, world, port, out):
    import torch.distributed as dist
    from halfedgecatmullclark_b200 import shard
    _init(rank, world, port)
    ws = _cages()
    work = [shard.cage_work(w.cage, w.depth) for w in ws]
    mine = shard.shard(work, world)[rank]
    digests = {i: _digest(ws[i]) for i in mine}
    gathered = [None] * world
    dist.all_gather_object(gathered, digests)
    t = shard.max_over_ranks(10.0 + rank, world, device="cpu")
    s = shard.sum_over_ranks(float(len(mine)), world, device="cpu")
    if rank == 0:
        out.put({"gathered": gathered, "max": t, "sum": s})
    dist.barrier()
    dist.destroy_process_group()


def _failing_worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    _init(rank, world, port, timeout_s=5)
    dist.barrier()                           # step 0 completes on both ranks
    if rank == 1:
        os._exit(3)                          # leaves between steps, nothing in flight
    try:
        t = torch.ones(1)
        dist.all_reduce(t)                   # step 1: the peer is gone
        out.put("no error")
    except Exception as exc:                 # noqa: BLE001 - any transport error is the signal
        out.put("error: %s" % type(exc).__name__)


def _run(fn, world=2):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=fn, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return res, [p.exitcode for p in procs]


def test_shard_covers_every_cage_once_and_balances():
    from halfedgecatmullclark_b200 import configs, shard
    ws = configs.batch_cages(count=512)
    work = [shard.cage_work(w.cage, w.depth) for w in ws]
    for world in (1, 2, 3, 8):
        parts = shard.shard(work, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(ws)))
        ld = shard.loads(work, parts)
        lower = max(sum(work) / world, max(work))      # no assignment beats this
        assert ld.max() <= 4.0 / 3.0 * lower + 1
        assert shard.shard(work, world) == parts          # every rank computes the same split


def test_sharded_refinement_equals_unsharded():
    res, codes = _run(_shard_worker)
    assert codes == [0, 0]
    ws = _cages()
    merged = {}
    for d in res["gathered"]:
        assert not (set(d) & set(merged))
        merged.update(d)
    assert sorted(merged) == list(range(len(ws)))
    for i, w in enumerate(ws):
        assert merged[i] == _digest(w), i
    assert res["max"] == 11.0
    assert res["sum"] == len(ws)


def test_rank_leaving_between_steps_is_reported():
    res, codes = _run(_failing_worker)
    assert codes[1] == 3
    assert res.startswith("error"), res
