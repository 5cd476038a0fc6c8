"""The N > 1 path of bench.py on CPU: two gloo ranks (replicas, no data-path
collective) combine their device times as the max over ranks, and the job
throughput counts every rank's bytes."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    r, w, _ = bench.dist_env()
    ms = bench.max_over_ranks(torch, 10.0 + 5.0 * rank, torch.device("cpu"))
    out.put((r, w, ms, bench.job_gbs(w, 1e9, ms)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_max_time():
    import socket
    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r for r, *_ in res] == [0, 1] and all(w == 2 for _, w, _, _ in res)
    assert all(ms == pytest.approx(15.0) for _, _, ms, _ in res)        # the slower rank's time
    assert all(v == pytest.approx(2 * 1e9 / 15e-3 / 1e9) for *_, v in res)
