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


def _shard_worker(rank, ws, port, out):
    """Diffuses this rank's share of an ensemble of small worlds (unit i on
    rank i % ws) with the FP32 CPU port, gathers every rank's results."""
    import datetime

    import numpy as np
    import torch.distributed as dist
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(ws), "LOCAL_RANK": str(rank)})
    import oracle
    from vfd import dist as vd
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        local = {}
        for i in vd.shard(len(_ENSEMBLE), rank, ws):
            local[i] = _diffuse_world(i, oracle, np)
        merged = vd.gather_units(local)
        out[rank] = {k: v.tobytes() for k, v in merged.items()}
        dist.barrier()
    finally:
        dist.destroy_process_group()


# (grid nx, ny, nz; sigma per field; decay per field): an uneven ensemble
_ENSEMBLE = [((24, 20, 16), (1.1, 0.7), (0.05, 0.02)), ((32, 16, 12), (0.9, 1.4), (0.01, 0.03)),
             ((20, 20, 20), (1.3, 0.8), (0.04, 0.05)), ((28, 12, 18), (0.6, 1.0), (0.02, 0.02)),
             ((16, 24, 14), (1.2, 1.2), (0.06, 0.01))]


def _diffuse_world(i, oracle, np):
    (nx, ny, nz), sig, dec = _ENSEMBLE[i]
    rng = np.random.default_rng(100 + i)
    outs = []
    for f in range(2):
        u = (rng.random((nz, ny, nx), dtype=np.float32) * np.float32(1e-3)).astype(np.float32)
        idx = rng.integers(0, u.size, 40, dtype=np.int32)
        amt = rng.lognormal(-6.0, 1.0, 40).astype(np.float32)
        r = oracle.radius_of(sig[f])
        for _ in range(3):
            oracle.port_substep(u, (sig[f],) * 3, (r,) * 3, dec[f], nthreads=1)
        oracle.port_deposit_total(u, idx, amt)
        outs.append(u)
    return np.stack(outs)


@pytest.mark.timeout(180)
def test_sharded_ensemble_equals_single_rank():
    """Two gloo ranks each diffuse their share of the worlds (the ensemble's
    partition, no exchange on the data path); the gathered results equal a
    one-rank run of every world, bit for bit."""
    import numpy as np

    import oracle
    ws = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_shard_worker, args=(ws, port, out), nprocs=ws, join=True)
        res = dict(out)
    assert res[0] == res[1]
    assert sorted(res[0]) == list(range(len(_ENSEMBLE)))
    for i in range(len(_ENSEMBLE)):
        single = _diffuse_world(i, oracle, np)
        assert res[0][i] == single.tobytes(), i
