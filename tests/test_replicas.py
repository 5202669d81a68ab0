"""Multi-GPU replica logic on CPU ranks (gloo, world_size 2).

The GPU path shards nothing: every rank runs independent pairs and the job time is the max over
ranks.  This checks the host logic of that scheme with two real processes: the assignment is a
partition, each rank's results equal a single-process run of the same items, and the max / sum
collectives give the whole-job figures.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _work(item):
    # stand-in for one pair: a deterministic per-item computation (the oracle's FNV over bytes)
    rng = np.random.default_rng(item)
    a = rng.integers(0, 256, 4096, dtype=np.uint8)
    h = 14695981039346656037
    for b in a.tobytes():
        h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def _rank_main(rank, world, port, items, out):
    import torch.distributed as dist
    from apg_sgm_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = replicas.run_replica(items, _work, rank, world)
        t = 1.0 + rank  # this rank's "device time"
        tmax = replicas.max_over_ranks(t, dist)
        units = replicas.sum_over_ranks(len(res), dist)
        dist.barrier()
        out[rank] = (res, tmax, units)
    finally:
        dist.destroy_process_group()


def test_replicas_two_ranks_gloo():
    from apg_sgm_b200 import replicas
    items = list(range(11))
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, items, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        got = dict(out)
    merged = {}
    for r in range(world):
        res, tmax, units = got[r]
        assert tmax == 2.0          # max over ranks of (1, 2)
        assert units == len(items)  # all items processed exactly once
        assert not (set(res) & set(merged))
        merged.update(res)
    assert sorted(merged) == items
    for i in items:
        assert merged[i] == _work(i)
    assert replicas.throughput([6, 5], [1.0, 2.0]) == pytest.approx(5.5)
    assert replicas.assign(5, 1, 2) == [1, 3]
    with pytest.raises(ValueError):
        replicas.assign(5, 2, 2)
