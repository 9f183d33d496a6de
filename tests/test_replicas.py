"""Multi-GPU is replicas only (no data-path collective): the bench's cross-rank
timing reduction and whole-job aggregation, run as world_size-2 gloo ranks on CPU."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = [10.0 + rank * 5.0, 2.0 - rank]  # per-rank device ms, e2e seconds
        got = bench.max_over_ranks(mine)
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_value():
    import bench

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res[0] == res[1] == [15.0, 2.0]
    # 2 replicas x 518400 rays in 15 ms -> 69.12 Mrays/s
    assert abs(bench.replica_value(518400, 2, 0.015) - 69.12) < 1e-9
