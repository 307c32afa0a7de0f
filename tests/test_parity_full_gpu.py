"""Full-size parity of every field against the FP64 oracle, per field:
the human-scale world (512x256x384 x 8 fields, one tick of 10 substeps,
200k sources per field), the large-world stress grid (768x384x576 x 8
fields, 10 substeps, 1M sources) and the 32-world batched ensemble (8 fields
per world, sigma and decay x U[0.5, 2], 500 sources, three ticks of 10
substeps through one batch, the second and third replayed from its CUDA
graph).

Per field: relative L2 <= 1e-5 and max-abs error <= 1e-5 of the field's
largest value against the FP64 oracle (oracle.tick_mt: the separable direct
sums in FP64, equal to the FFT linear convolution on any grid F >= n + r);
mass identity of the last substep and the reported FP64 total within 1e-6
relative.  The per-field figures are printed (pytest -s shows them)."""
import numpy as np
import pytest

import oracle
import vfd
from vfd import configs

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5
MAX_ABS_REL = 1e-5
MASS_REL = 1e-6


def errors(got, ref):
    g = np.asarray(got, np.float64)
    d = g - ref
    rel = float(np.sqrt((d * d).sum() / max((ref * ref).sum(), 1e-300)))
    mx = float(np.abs(d).max())
    return rel, mx, float(np.abs(ref).max())


def check_field(name, f, got, ref, m, keep, V):
    rel, mx, scale = errors(got, ref)
    s = got.astype(np.float64).sum()
    mass_err = abs(m["total"] - s) / max(abs(s), 1e-30)
    ident = abs(m["input_sum"] - m["conv_sum"] - sum(m["leaked"])) / max(abs(m["input_sum"]), abs(s), 1e-30)
    print(f"{name} field {f}: rel_l2 {rel:.3e} max_abs {mx:.3e} (max |ref| {scale:.3e}) "
          f"mass {mass_err:.1e} identity {ident:.1e}")
    assert rel <= REL_L2, (name, f, rel)
    assert mx <= MAX_ABS_REL * scale, (name, f, mx, scale)
    assert mass_err <= MASS_REL, (name, f, mass_err)
    assert ident <= MASS_REL, (name, f, ident)
    assert abs(m["total"] - (keep * (m["conv_sum"] + 0.0 * V) + m["sources"])) <= MASS_REL * max(abs(s), 1e-30)


def _one_world(c):
    nx, ny, nz = c["grid"]
    V = nx * ny * nz
    params = [vfd.field_params(s, d) for s, d in zip(c["sigma"], c["decay"])]
    srcs = []
    with vfd.World(nx, ny, nz, params) as w:
        for f in range(8):
            u = vfd.synth_field(c["seed"], 0, f, (nz, ny, nx))
            idx, amt = vfd.synth_sources(c["seed"], 0, f, c["n_sources"], V)
            w.upload(f, u)
            w.set_sources(f, idx, amt)
            srcs.append((idx, amt))
            del u
        w.tick(c["substeps"])
        mass = w.mass()
        for f in range(8):
            got = w.download(f)
            u = vfd.synth_field(c["seed"], 0, f, (nz, ny, nx))
            ref, _ = oracle.tick_mt(u, c["sigma"][f], c["decay"][f], c["substeps"], *srcs[f])
            del u
            check_field(c["name"], f, got, ref, mass[f], 1 - c["decay"][f], V)
            del got, ref


def test_cfg1_every_field_full_size(gpu):
    _one_world(configs.CFG1)


def test_cfg4_every_field_full_size(gpu):
    _one_world(configs.CFG4)


def test_cfg2_ensemble_batched_every_field(gpu):
    c = configs.CFG2
    specs = configs.cfg2_worlds(c["n_worlds"], c["seed"])
    ticks = 3
    worlds, inputs = [], []
    for sp in specs:
        nx, ny, nz = sp["grid"]
        params = [vfd.field_params(s_, d_) for s_, d_ in zip(sp["sigma"], sp["decay"])]
        w = vfd.World(nx, ny, nz, params)
        ins = configs.field_inputs(c["seed"], sp["world"], sp["grid"], sp["n_sources"])
        for f, (u, idx, amt) in enumerate(ins):
            w.upload(f, u)
            w.set_sources(f, idx, amt)
        worlds.append(w)
        inputs.append(ins)
    with vfd.Batch(worlds) as b:
        for _ in range(ticks):
            b.tick(c["substeps"])
    for i, sp in enumerate(specs):
        nx, ny, nz = sp["grid"]
        m = worlds[i].mass()
        for f, (u, idx, amt) in enumerate(inputs[i]):
            ref = np.asarray(u, np.float64)
            for _ in range(ticks):
                ref, _ = oracle.tick_mt(ref, sp["sigma"][f], sp["decay"][f], c["substeps"], idx, amt)
            check_field(f"cfg2 world {i} {sp['grid']}", f, worlds[i].download(f), ref, m[f],
                        1 - sp["decay"][f], nx * ny * nz)
        worlds[i].close()
