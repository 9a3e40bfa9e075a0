"""The multi-rank replica path on CPU: two gloo ranks, each with its own
seeded grid, reduce their timings to the slowest rank's."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    from arcos_b200 import workloads
    from arcos_b200.replicas import barrier, job_throughput, max_over_ranks, rank_info
    info = rank_info()
    pb = workloads.plain(nr=16, nz=32, noise=1e-6, seed=info.rank)
    barrier()
    slowest = max_over_ranks(1.0 + info.rank, "cpu")
    out.put((info.rank, info.world, slowest, float(pb.dens[0][0].sum()),
             job_throughput(16 * 32 * 2, info.world, slowest)))
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_to_the_slowest():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1] and all(r[1] == 2 for r in res)
    assert all(r[2] == 2.0 for r in res)               # max over ranks
    assert res[0][3] != res[1][3]                      # independent seeded replicas
    assert res[0][4] == pytest.approx(2 * 16 * 32 * 2 / 2.0)


def test_single_rank_is_identity():
    from arcos_b200.replicas import max_over_ranks, rank_info
    assert rank_info().world >= 1
    assert max_over_ranks(3.5, "cpu") == 3.5
