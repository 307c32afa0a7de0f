"""GPU tests of the per-shape pass tuning (vfd_autotune, vfd_autotune_set,
vfd_world_tuning): the tuner's choice is cached and applied, and every pass
it can choose -- register FFT, overlap-save at 3 or 4 CTAs per SM, full-line
FFT with either radix order and each kernel variant -- gives the FP64
oracle's result (relative L2 <= 1e-5 per field), alone and in a batch."""
import numpy as np
import pytest

import oracle
import vfd
from vfd import configs

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5
GRID = (96, 70, 33)
SIGMAS = [0.6, 1.3]      # radii 2 and 4
DECAY = [0.03, 0.05]


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def params():
    return [vfd.field_params(s, d) for s, d in zip(SIGMAS, DECAY)]


def run_and_check(world, substeps=2, seed=5):
    ins = configs.field_inputs(seed, 0, GRID, 64, n_fields=len(SIGMAS))
    for f, (u, idx, amt) in enumerate(ins):
        world.upload(f, u)
        world.set_sources(f, idx, amt)
    world.tick(substeps)
    for f, (u, idx, amt) in enumerate(ins):
        ref = oracle.tick(u, SIGMAS[f], DECAY[f], substeps, idx, amt)
        e = rel_l2(world.download(f), ref)
        assert e <= REL_L2, (f, e, world.tuning())


@pytest.fixture
def clean_cache():
    vfd.autotune_clear()
    yield
    vfd.autotune_clear()


def test_autotune_choice_is_cached_and_applied(gpu, clean_cache):
    nx, ny, nz = GRID
    with vfd.World(nx, ny, nz, params()) as w:
        untuned = w.tuning()
    assert all(t["ms"] == 0.0 for t in untuned)
    best = vfd.autotune(nx, ny, nz, params(), reps=2)
    assert len(best) == 3
    for t in best:
        assert t["method"] in ("register_fft", "overlap_save", "full_line")
        assert t["ms"] > 0.0
        if t["method"] == "overlap_save":
            assert t["ctas_per_sm"] in (3, 4)
        if t["method"] == "full_line":
            assert t["fft_len"] >= max(GRID) // 3 and t["variant"] >= 0
    with vfd.World(nx, ny, nz, params()) as w:
        got = w.tuning()
        for a in range(3):
            for k in ("method", "ctas_per_sm", "fft_len", "radix_order", "variant"):
                assert got[a][k] == best[a][k], (a, k, got, best)
            assert got[a]["ms"] == pytest.approx(best[a]["ms"])
        run_and_check(w)
    vfd.autotune_clear()
    with vfd.World(nx, ny, nz, params()) as w:
        assert all(t["ms"] == 0.0 for t in w.tuning())


PINS = [
    ("register_fft", {"method": "register_fft"}),
    ("overlap_save_3", {"method": "overlap_save", "ctas_per_sm": 3}),
    ("overlap_save_4", {"method": "overlap_save", "ctas_per_sm": 4}),
    ("full_line_order0", {"method": "full_line", "radix_order": 0}),
    ("full_line_order1", {"method": "full_line", "radix_order": 1}),
] + [(f"full_line_variant{v}", {"method": "full_line", "variant": v}) for v in range(6)]


@pytest.mark.parametrize("name,pin", PINS, ids=[p[0] for p in PINS])
def test_pinned_pass_against_oracle(gpu, clean_cache, name, pin):
    nx, ny, nz = GRID
    vfd.autotune_set(nx, ny, nz, params(), [pin] * 3)
    with vfd.World(nx, ny, nz, params()) as w:
        got = w.tuning()
        for a in range(3):
            assert got[a]["method"] == pin["method"], (a, got)
            if pin["method"] == "overlap_save":
                assert got[a]["ctas_per_sm"] == pin["ctas_per_sm"]
            if pin["method"] == "full_line":
                assert got[a]["radix_order"] == pin.get("radix_order", 0)
        run_and_check(w)


def test_full_line_lengths_and_mixed_axes(gpu, clean_cache):
    # x: FFT length 112 (radices 8 7 2 / 4 4 7), y: overlap-save at 4 CTAs/SM,
    # z: register FFT
    nx, ny, nz = GRID
    for order in (0, 1):
        pin = [{"method": "full_line", "fft_len": 112, "radix_order": order},
               {"method": "overlap_save", "ctas_per_sm": 4},
               {"method": "register_fft"}]
        vfd.autotune_set(nx, ny, nz, params(), pin)
        with vfd.World(nx, ny, nz, params()) as w:
            t = w.tuning()
            assert w.fft_dims()[0] == 112
            assert [x["method"] for x in t] == ["full_line", "overlap_save", "register_fft"]
            assert t[0]["radix_order"] == order and t[1]["ctas_per_sm"] == 4
            run_and_check(w, seed=7 + order)


def test_pin_rejects_bad_choices(gpu, clean_cache):
    nx, ny, nz = GRID
    with pytest.raises(vfd.VfdError):
        vfd.autotune_set(nx, ny, nz, params(), [{"method": "full_line", "fft_len": 97}] * 3)  # < n + r
    with pytest.raises(vfd.VfdError):
        vfd.autotune_set(nx, ny, nz, params(), [{"method": "full_line", "fft_len": 101}] * 3)  # not 7-smooth
    with pytest.raises(vfd.VfdError):
        vfd.autotune_set(nx, ny, nz, params(), [{"method": "overlap_save", "ctas_per_sm": 5}] * 3)
    with pytest.raises(vfd.VfdError):
        vfd.autotune_set(nx, ny, nz, params(), [{"method": 7}] * 3)


def test_batch_of_pinned_worlds_matches_single_worlds(gpu, clean_cache):
    nx, ny, nz = GRID
    pin = [{"method": "overlap_save", "ctas_per_sm": 4}, {"method": "full_line", "radix_order": 1},
           {"method": "overlap_save", "ctas_per_sm": 4}]
    vfd.autotune_set(nx, ny, nz, params(), pin)
    worlds, singles, ins = [], [], []
    for i in range(2):
        w = vfd.World(nx, ny, nz, params())
        s = vfd.World(nx, ny, nz, params())
        x = configs.field_inputs(3, i, GRID, 64, n_fields=len(SIGMAS))
        for f, (u, idx, amt) in enumerate(x):
            for t in (w, s):
                t.upload(f, u)
                t.set_sources(f, idx, amt)
        worlds.append(w)
        singles.append(s)
        ins.append(x)
    with vfd.Batch(worlds) as b:
        b.tick(2)
    for s in singles:
        s.tick(2)
    for i in range(2):
        for f, (u, idx, amt) in enumerate(ins[i]):
            got = worlds[i].download(f)
            assert rel_l2(got, singles[i].download(f)) <= 1e-6
            assert rel_l2(got, oracle.tick(u, SIGMAS[f], DECAY[f], 2, idx, amt)) <= REL_L2
    for w in worlds + singles:
        w.close()
