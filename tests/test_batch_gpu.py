"""GPU tests of the batched ensemble form (vfd_batch_*): every world's result
equals its own single-world tick (pairing of lines into complex FFTs may
differ, so within FP32 rounding) and the FP64 oracle."""
import numpy as np
import pytest

import oracle
import vfd
from vfd import configs

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def make_world(grid, sig, dec, seed, w_index, n_src=200, nf=3):
    nx, ny, nz = grid
    params = [vfd.field_params(s, d) for s, d in zip(sig[:nf], dec[:nf])]
    w = vfd.World(nx, ny, nz, params)
    ins = configs.field_inputs(seed, w_index, grid, n_src, n_fields=nf)
    for f, (u, idx, amt) in enumerate(ins):
        w.upload(f, u)
        w.set_sources(f, idx, amt)
    return w, ins


def test_batch_matches_single_worlds_and_oracle(gpu):
    specs = [((96, 64, 64), [1.0, 2.1, 0.6]), ((70, 33, 41), [1.7, 0.5, 1.2]),
             ((128, 96, 96), [0.9, 1.3, 2.4])]
    dec = [0.05, 0.01, 0.03]
    worlds, singles, inputs = [], [], []
    for i, (g, sig) in enumerate(specs):
        w, ins = make_world(g, sig, dec, 0, i)
        s, _ = make_world(g, sig, dec, 0, i)
        worlds.append(w)
        singles.append(s)
        inputs.append(ins)
    with vfd.Batch(worlds) as b:
        b.tick(3)
        b.tick(3)  # graph replay
    for s in singles:
        s.tick(3)
        s.tick(3)
    errs = []
    for i, (g, sig) in enumerate(specs):
        for f in range(3):
            got = worlds[i].download(f)
            ref_single = singles[i].download(f)
            u, idx, amt = inputs[i][f]
            ref = oracle.tick(oracle.tick(u, sig[f], dec[f], 3, idx, amt), sig[f], dec[f], 3, idx, amt)
            errs.append((i, f, rel_l2(got, ref_single), rel_l2(got, ref), rel_l2(ref_single, ref)))
    for e in errs:
        assert e[2] <= 1e-6 and e[3] <= 1e-5 and e[4] <= 1e-5, errs
    for w in worlds:
        m = w.mass()
        for f in range(3):
            s_ = w.download(f).astype(np.float64).sum()
            assert abs(m[f]["total"] - s_) <= 1e-6 * abs(s_)
    for w in worlds + singles:
        w.close()


def test_batch_recaptures_when_sources_change(gpu):
    w1, _ = make_world((40, 30, 20), [1.0, 1.0, 1.0], [0.0, 0.0, 0.0], 1, 0, n_src=0, nf=1)
    w2, _ = make_world((40, 30, 20), [1.0, 1.0, 1.0], [0.0, 0.0, 0.0], 1, 0, n_src=0, nf=1)
    before = [w1.download(0).astype(np.float64).sum()]
    # direct, captured, replayed; sources change; direct, captured, replayed
    with vfd.Batch([w1]) as b:
        for _ in range(3):
            b.tick(1)
        w1.set_sources(0, np.array([7], np.int32), np.array([2.0], np.float32))
        for _ in range(3):
            b.tick(1)
    for _ in range(3):
        w2.tick(1)
    w2.set_sources(0, np.array([7], np.int32), np.array([2.0], np.float32))
    for _ in range(3):
        w2.tick(1)
    np.testing.assert_allclose(w1.download(0), w2.download(0), rtol=1e-5, atol=1e-9)
    assert w1.mass()[0]["sources"] == pytest.approx(2.0)
    del before
    w1.close()
    w2.close()


@pytest.mark.parametrize("grid,sig", [((128, 96, 96), (0.9, 1.3, 2.4)), ((96, 64, 64), (1.0, 2.1, 0.6)),
                                      ((512, 64, 40), (1.8, 1.8, 1.8))])
def test_single_world_is_deterministic(gpu, grid, sig):
    """No sources (atomics aside, every output is computed by one thread):
    two runs on identical inputs are bitwise equal."""
    outs = []
    for _ in range(2):
        w, _ = make_world(grid, sig, [0.05, 0.01, 0.03], 4, 0, n_src=0)
        w.tick(3)
        outs.append([w.download(f) for f in range(3)])
        w.close()
    for f in range(3):
        np.testing.assert_array_equal(outs[0][f], outs[1][f])


def test_batch_autotune_keeps_fields_and_results(gpu):
    """vfd_batch_autotune times the pass candidates on the worlds' own fields
    and restores them: ticks after tuning equal ticks of untuned single worlds."""
    specs = [((96, 64, 64), [1.0, 2.1, 0.6]), ((70, 33, 41), [1.7, 0.5, 1.2]), ((128, 96, 96), [0.9, 1.3, 2.4])]
    dec = [0.05, 0.01, 0.03]
    worlds, singles = [], []
    for i, (g, sig) in enumerate(specs):
        worlds.append(make_world(g, sig, dec, 2, i)[0])
        singles.append(make_world(g, sig, dec, 2, i)[0])
    before = [w.download(0).copy() for w in worlds]
    with vfd.Batch(worlds) as b:
        tuning = b.autotune(reps=2)
        assert len(tuning) == 3 and all(t["ms"] > 0 for t in tuning)
        for w, u in zip(worlds, before):
            np.testing.assert_array_equal(w.download(0), u)
        for _ in range(3):
            b.tick(2)
    for s in singles:
        for _ in range(3):
            s.tick(2)
    for w, s in zip(worlds, singles):
        for f in range(3):
            assert rel_l2(w.download(f), s.download(f)) <= 1e-6
    for w in worlds + singles:
        w.close()
