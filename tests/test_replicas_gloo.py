"""The N > 1 path (independent replicas) with two gloo ranks on CPU: the
max-over-ranks timing and the whole-job aggregate the bench reports, and the
cloud sharding of a batched ensemble."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from sph_3_b200 import replicas
    try:
        r, w = replicas.world()
        ms = 10.0 + 5.0 * rank
        mx = replicas.max_over_ranks(ms)
        rate = replicas.whole_job_rate(1000.0 * (rank + 1), ms / 1e3)
        out.put((r, w, mx, rate))
    finally:
        dist.destroy_process_group()


def test_two_rank_aggregation():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, mx, rate in res:
        assert w == 2
        assert mx == 15.0
        assert rate == pytest.approx(3000.0 / 0.015)


def test_shard_clouds_partition():
    from sph_3_b200 import replicas
    counts = np.array([5, 100, 3, 40, 40, 7, 900, 1])
    for nr in (1, 2, 3, 4, 8):
        spans = [replicas.shard_clouds(counts, r, nr) for r in range(nr)]
        assert spans[0][0] == 0 and spans[-1][1] == len(counts)
        for a, b in zip(spans, spans[1:]):
            assert a[1] == b[0]
