"""GPU tests of the serving loop (vfd_server_*): continuous batching keeps
each request's result equal to its result alone, admission respects the HBM
budget and the slot count, and later arrivals join while others are resident."""
import time

import numpy as np
import pytest

import oracle
import vfd
from vfd import configs

pytestmark = pytest.mark.gpu


def params_for(nf, scale=1.0):
    return [vfd.field_params(configs.SIGMA0[f] * scale, configs.DECAY0[f]) for f in range(nf)]


def req(server, grid, world, ticks, nf=3, n_src=300, with_result=True):
    nx, ny, nz = grid
    srcs = [vfd.synth_sources(7, world, f, n_src, nx * ny * nz) for f in range(nf)]
    res = [np.empty((nz, ny, nx), np.float32) for _ in range(nf)] if with_result else None
    rid = server.submit(grid, params_for(nf), ticks, synth=(7, world, 0.0, 1e-3), sources=srcs, result=res)
    return rid, res, srcs


def test_device_generator_matches_host(gpu):
    import torch
    n = 1 << 20
    t = torch.empty(n, dtype=torch.float32, device="cuda")
    st = vfd.lib().vfd_synth_field_device(3, 2, 1, 0.0, 1e-3, t.data_ptr(), n, None)
    assert st == 0
    torch.cuda.synchronize()
    host = vfd.synth_field(3, 2, 1, (n,))
    np.testing.assert_array_equal(t.cpu().numpy(), host)


def test_request_alone_equals_request_in_mix(gpu):
    grid_a = (64, 48, 40)
    with vfd.Server(8 << 30, max_active=4) as s:
        rid, alone, _ = req(s, grid_a, 0, 5)
        info_alone = s.wait(rid)
    assert info_alone["status"] == 0
    with vfd.Server(8 << 30, max_active=4) as s:
        r_b, _, _ = req(s, (96, 64, 64), 1, 8, with_result=False)
        r_c, _, _ = req(s, (40, 40, 40), 2, 3, with_result=False)
        rid, mixed, _ = req(s, grid_a, 0, 5)
        r_d, _, _ = req(s, (128, 96, 96), 3, 6, with_result=False)
        info = s.wait(rid)
        for r in (r_b, r_c, r_d):
            assert s.wait(r)["status"] == 0
    for f in range(3):
        np.testing.assert_array_equal(mixed[f], alone[f])
    assert info["mass"][0]["total"] == pytest.approx(info_alone["mass"][0]["total"], rel=1e-12)


def test_server_result_matches_oracle(gpu):
    grid = (48, 40, 32)
    nx, ny, nz = grid
    with vfd.Server(4 << 30, max_active=2) as s:
        rid, res, srcs = req(s, grid, 5, 3, nf=2)
        s.wait(rid)
    for f in range(2):
        u = vfd.synth_field(7, 5, f, (nz, ny, nx))
        ref = u.astype(np.float64)
        for _ in range(3):
            ref = oracle.tick(ref, configs.SIGMA0[f], configs.DECAY0[f], 1, *srcs[f])
        err = np.sqrt(((res[f] - ref) ** 2).sum() / (ref ** 2).sum())
        assert err <= 1e-5


def test_budget_and_slots(gpu):
    grid = (64, 64, 64)
    one = 3 * 64 ** 3 * 4
    # a budget that fits one request at a time: all complete, never two resident
    with vfd.Server(int(one * 1.5), max_active=8) as s:
        ids = [req(s, grid, w, 4, with_result=False)[0] for w in range(3)]
        infos = [s.wait(i) for i in ids]
        st = s.stats()
    assert all(i["status"] == 0 for i in infos)
    for a, b in zip(infos, infos[1:]):
        assert b["t_admit"] >= a["t_done"] - 1e-3
    assert st["completed"] == 3 and st["hbm_peak"] <= one * 1.5
    # larger than the whole budget: rejected with VFD_ERR_BUDGET
    with vfd.Server(one // 2, max_active=8) as s:
        rid = req(s, grid, 9, 2, with_result=False)[0]
        with pytest.raises(vfd.VfdError) as e:
            s.wait(rid)
        assert e.value.status == 3


def test_continuous_batching_overlaps_requests(gpu):
    """A request submitted while another is resident is admitted before the
    first one finishes (it joins the running rounds)."""
    with vfd.Server(8 << 30, max_active=4) as s:
        r1 = req(s, (256, 128, 192), 0, 400, with_result=False)[0]
        t_end = time.time() + 30
        while s.stats()["admitted"] < 1 and time.time() < t_end:
            time.sleep(0.001)
        r2 = req(s, (64, 64, 32), 1, 5, with_result=False)[0]
        i1, i2 = s.wait(r1), s.wait(r2)
        st = s.stats()
    assert i1["t_admit"] < i2["t_admit"] < i1["t_done"]
    assert i2["t_done"] < i1["t_done"]
    assert st["p99_latency_s"] >= st["p50_latency_s"] > 0
