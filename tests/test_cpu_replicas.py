"""The N>1 path (replicas over DM trials) with world_size 2 on CPU (gloo):
sharding covers every trial once, the step time reduces to the maximum over
ranks, and candidate lists gather to rank 0 in trial order."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from presto_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ntrials = 7
        mine = replicas.shard(ntrials, rank, world)
        # a stand-in search result per trial: (power, sigma, numharm, r, z, w)
        res = [(t, [(10.0 + t, 3.0, 1, 100.0 * t, 0.0, 0.0)]) for t in mine]
        tmax = replicas.max_over_ranks(1.5 + rank, dist)
        allres = replicas.gather_to_rank0(res, dist)
        if rank == 0:
            merged = replicas.merge_candidates(allres, list(range(ntrials)))
            q.put((tmax, merged))
        else:
            q.put((tmax, None))
    finally:
        dist.destroy_process_group()


def test_shard_partitions():
    for world in (1, 2, 3, 8):
        seen = sorted(i for r in range(world) for i in replicas.shard(13, r, world))
        assert seen == list(range(13))
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


def test_two_rank_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    outs = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(o[0] == 2.5 for o in outs)
    merged = [o[1] for o in outs if o[1] is not None][0]
    assert [c[0][3] for c in merged] == [100.0 * t for t in range(7)]
