"""World-size-2 CPU test (gloo) of the multi-GPU plumbing in vfd.dist: rank
sharding, max-over-ranks timing and the whole-job aggregate."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(ws), "LOCAL_RANK": str(rank)})
    from vfd import dist as vd
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        env = vd.env()
        mine = vd.shard(32, rank, ws)
        elapsed = 1.0 + 0.5 * rank           # ranks finish at different times
        m = vd.max_over_ranks(elapsed)
        rate = vd.aggregate_rate(1000.0, m, ws)
        out[rank] = (env, mine, m, rate)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_plumbing():
    ws = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(ws, port, out), nprocs=ws, join=True)
        res = dict(out)
    (e0, s0, m0, r0), (e1, s1, m1, r1) = res[0], res[1]
    assert e0 == (2, 0, 0) and e1 == (2, 1, 1)
    assert sorted(s0 + s1) == list(range(32)) and not set(s0) & set(s1)
    assert m0 == m1 == 1.5                    # max over ranks
    assert r0 == r1 == 2 * 1000.0 / 1.5       # whole-job aggregate
