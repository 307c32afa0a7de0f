"""GPU parity of the product path (libvfd.so through its C ABI) against the
FP64 oracle.

Bar (per field): relative L2 <= 1e-5 against the FP64 oracle; mass identity
(input = kept + leaked) and the reported FP64 totals within 1e-6 relative.
"""
import numpy as np
import pytest

import oracle
import vfd
from vfd import configs

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5
MASS_REL = 1e-6


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def run_world(grid, sigmas, decays, inputs, substeps=1, pad_mode=vfd.PAD_ZERO, epi=0,
              baselines=None, fft=(0, 0, 0)):
    nx, ny, nz = grid
    params = [vfd.field_params(s, d, baseline=(baselines[f] if baselines else 0.0))
              for f, (s, d) in enumerate(zip(sigmas, decays))]
    with vfd.World(nx, ny, nz, params, pad_mode=pad_mode, epi_boundary=epi, fft=fft) as w:
        for f, (u, idx, amt) in enumerate(inputs):
            w.upload(f, u)
            w.set_sources(f, idx, amt)
        w.tick(substeps)
        outs = [w.download(f) for f in range(len(inputs))]
        mass = w.mass()
        dims = w.fft_dims()
    return outs, mass, dims


def check_mass(out, m, keep, b, V):
    s = out.astype(np.float64).sum()
    scale = max(abs(m["input_sum"]), abs(s), 1e-30)
    # identity of the last substep: sum(M (u-b)) = kept + leaked
    assert abs(m["input_sum"] - m["conv_sum"] - sum(m["leaked"])) <= MASS_REL * scale
    # reported total equals the field's sum
    assert abs(m["total"] - s) <= MASS_REL * max(abs(s), 1e-30)
    # total = keep * (conv + b V) + sources
    assert abs(m["total"] - (keep * (m["conv_sum"] + b * V) + m["sources"])) <= MASS_REL * max(abs(s), 1e-30)


def test_cfg0_all_fields_against_oracle(gpu):
    c = configs.CFG0
    inputs = configs.field_inputs(c["seed"], 0, c["grid"], c["n_sources"])
    outs, mass, _ = run_world(c["grid"], c["sigma"], c["decay"], inputs)
    V = configs.voxels(c["grid"])
    for f, (u, idx, amt) in enumerate(inputs):
        ref = oracle.tick(u, c["sigma"][f], c["decay"][f], 1, idx, amt)
        e = rel_l2(outs[f], ref)
        assert e <= REL_L2, (f, e)
        check_mass(outs[f], mass[f], 1 - c["decay"][f], 0.0, V)
        assert abs(mass[f]["sources"] - amt.astype(np.float64).sum()) <= 1e-6 * amt.sum()


def test_cfg0_against_committed_fixture(gpu):
    import os
    from conftest import ROOT
    g = np.load(os.path.join(ROOT, "tests", "golden", "cfg0_oracle.npz"))
    c = configs.CFG0
    inputs = configs.field_inputs(c["seed"], 0, c["grid"], c["n_sources"])
    outs, _, _ = run_world(c["grid"], c["sigma"], c["decay"], inputs)
    for f in range(8):
        got = outs[f].ravel()[g["sample_idx"]]
        assert rel_l2(got, g["sample"][f]) <= REL_L2
        assert abs(outs[f].astype(np.float64).sum() - g["sums"][f]) <= MASS_REL * g["sums"][f]


@pytest.mark.parametrize("grid", [(1, 1, 1), (2, 3, 1), (3, 5, 7), (33, 17, 9), (70, 37, 50),
                                  (31, 64, 33), (129, 2, 65)])
def test_ragged_grids(gpu, grid):
    nx, ny, nz = grid
    sig = [(1.0, 0.7, 1.3), 2.2]
    dec = [0.05, 0.0]
    inputs = []
    for f in range(2):
        u = vfd.synth_field(3, 1, f, (nz, ny, nx))
        idx, amt = vfd.synth_sources(3, 1, f, 17, nx * ny * nz)
        inputs.append((u, idx, amt))
    outs, mass, _ = run_world(grid, sig, dec, inputs)
    for f, (u, idx, amt) in enumerate(inputs):
        ref = oracle.tick(u, sig[f], dec[f], 1, idx, amt)
        assert rel_l2(outs[f], ref) <= REL_L2, (grid, f)
        check_mass(outs[f], mass[f], 1 - dec[f], 0.0, nx * ny * nz)


def test_constant_vf_padding_rule(gpu):
    """The reference's padDataConstantVF3D boundary: interior 0<z<D-1,
    0<y<H-1, 0<x<epi keeps u; everything else holds the baseline."""
    grid = (48, 40, 36)
    nx, ny, nz = grid
    sig = [1.2, 0.9]
    dec = [0.05, 0.01]
    base = [4e-4, 7e-4]
    inputs = []
    for f in range(2):
        u = vfd.synth_field(5, 0, f, (nz, ny, nx))
        inputs.append((u, np.zeros(0, np.int32), np.zeros(0, np.float32)))
    epi = 37
    outs, mass, _ = run_world(grid, sig, dec, inputs, pad_mode=vfd.PAD_CONSTANT_VF, epi=epi,
                              baselines=base)
    for f, (u, idx, amt) in enumerate(inputs):
        ref = oracle.tick(u, sig[f], dec[f], 1, idx, amt, b=float(np.float32(base[f])), pad_mode=1, epi=epi)
        assert rel_l2(outs[f], ref) <= REL_L2
        check_mass(outs[f], mass[f], 1 - dec[f], float(np.float32(base[f])), nx * ny * nz)


# The pass a world uses depends on its shape and radii: the register-FFT pass
# for radius <= 8 (x with 16-byte tiles when nx is a multiple of 4, else the
# overlap-save x pass), the overlap-save pass for radius 9..16.  Tiles of 64
# lines end partly filled and with an odd line count on these grids.
PATH_GRIDS = [(96, 70, 33), (70, 33, 41), (37, 65, 29), (132, 9, 66)]
SIGMAS_RF = [0.3, 0.6, 1.0, 1.3, 1.6, 2.0, 2.3, 2.6]   # radii 1..8
SIGMAS_OS = [0.6, 3.2, 4.0]                            # radii 2, 10, 12


@pytest.mark.parametrize("grid", PATH_GRIDS)
@pytest.mark.parametrize("sigmas", [SIGMAS_RF, SIGMAS_OS], ids=["r1-8", "r2-12"])
def test_pass_paths_against_oracle(gpu, grid, sigmas):
    nx, ny, nz = grid
    dec = [0.03] * len(sigmas)
    inputs = configs.field_inputs(11, 2, grid, 64, n_fields=len(sigmas))
    outs, mass, _ = run_world(grid, sigmas, dec, inputs, substeps=2)
    for f, (u, idx, amt) in enumerate(inputs):
        ref = oracle.tick(u, sigmas[f], dec[f], 2, idx, amt)
        assert rel_l2(outs[f], ref) <= REL_L2, (grid, sigmas[f])
        check_mass(outs[f], mass[f], 1 - dec[f], 0.0, nx * ny * nz)


@pytest.mark.parametrize("sigmas", [[0.3, 0.6], [1.6, 2.0], [1.0, 2.3, 2.6]])
def test_constant_vf_padding_every_x_block_offset(gpu, sigmas):
    # radii 1, 2, 5, 6 start the x pass's FFT input 2 positions into its
    # window, radii 3, 4, 7, 8 at the window start; the constant-VF rule is
    # applied to the staged x samples in both cases
    grid = (48, 40, 36)
    nx, ny, nz = grid
    dec = [0.02] * len(sigmas)
    base = [3e-4 * (f + 1) for f in range(len(sigmas))]
    inputs = []
    for f in range(len(sigmas)):
        u = vfd.synth_field(6, 1, f, (nz, ny, nx))
        idx, amt = vfd.synth_sources(6, 1, f, 40, nx * ny * nz)
        inputs.append((u, idx, amt))
    outs, mass, _ = run_world(grid, sigmas, dec, inputs, substeps=2, pad_mode=vfd.PAD_CONSTANT_VF, epi=29,
                              baselines=base)
    for f, (u, idx, amt) in enumerate(inputs):
        ref = oracle.tick(u, sigmas[f], dec[f], 2, idx, amt, b=float(np.float32(base[f])), pad_mode=1, epi=29)
        assert rel_l2(outs[f], ref) <= REL_L2, sigmas[f]
        check_mass(outs[f], mass[f], 1 - dec[f], float(np.float32(base[f])), nx * ny * nz)


def test_constant_field_fixed_point(gpu):
    c = 5e-4
    grid = (40, 30, 20)
    u = np.full((20, 30, 40), c, np.float32)
    outs, _, _ = run_world(grid, [1.3], [0.1], [(u, np.zeros(0, np.int32), np.zeros(0, np.float32))],
                           pad_mode=vfd.PAD_CONSTANT_VF, epi=40, baselines=[c])
    np.testing.assert_allclose(outs[0], 0.9 * np.float32(c), rtol=2e-6)


def test_ten_substeps_against_fp64_oracle(gpu):
    grid = (96, 64, 64)
    nx, ny, nz = grid
    sig = [1.8, 0.6, 2.4]
    dec = [0.05, 0.01, 0.03]
    inputs = []
    for f in range(3):
        u = vfd.synth_field(0, 9, f, (nz, ny, nx))
        idx, amt = vfd.synth_sources(0, 9, f, 500, nx * ny * nz)
        inputs.append((u, idx, amt))
    outs, mass, _ = run_world(grid, sig, dec, inputs, substeps=10)
    for f, (u, idx, amt) in enumerate(inputs):
        ref = oracle.tick(u, sig[f], dec[f], 10, idx, amt)
        assert rel_l2(outs[f], ref) <= REL_L2, f
        check_mass(outs[f], mass[f], 1 - dec[f], 0.0, nx * ny * nz)


def test_fft_length_does_not_change_result(gpu):
    grid = (40, 24, 18)
    nx, ny, nz = grid
    u = vfd.synth_field(1, 0, 0, (nz, ny, nx))
    inp = [(u, np.zeros(0, np.int32), np.zeros(0, np.float32))]
    r = 4
    base, _, _ = run_world(grid, [1.2], [0.0], inp)
    # n + r = (44, 28, 22) are not all 7-smooth; these are (and >= n + r)
    for fft in [(45, 28, 24), (64, 32, 32), (48, 35, 28), (49, 30, 42)]:
        o, _, dims = run_world(grid, [1.2], [0.0], inp, fft=fft)
        assert tuple(dims) == fft
        assert rel_l2(o[0], base[0]) <= 2e-6
    with pytest.raises(vfd.VfdError) as e:
        run_world(grid, [1.2], [0.0], inp, fft=(nx + r - 1, 0, 0))
    assert e.value.status == 1
    with pytest.raises(vfd.VfdError) as e:
        run_world(grid, [1.2], [0.0], inp, fft=(nx + 13, 0, 0))  # 53 is prime
    assert e.value.status == 7


def test_host_buffer_entry_matches_resident_tick(gpu):
    """vfd_diffuse_host (the diffuseChemGPU drop-in) == upload + tick + download."""
    c = configs.CFG0
    inputs = configs.field_inputs(c["seed"], 2, c["grid"], 300)
    outs, _, _ = run_world(c["grid"], c["sigma"], c["decay"], inputs, substeps=2)
    nx, ny, nz = c["grid"]
    params = [vfd.field_params(s, d) for s, d in zip(c["sigma"], c["decay"])]
    with vfd.World(nx, ny, nz, params) as w:
        for f, (u, idx, amt) in enumerate(inputs):
            w.set_sources(f, idx, amt)
        host_in = [u.copy() for (u, _, _) in inputs]
        host_out = [np.empty_like(u) for u in host_in]
        w.diffuse_host(host_in, host_out, 2)
    # same kernels; duplicate sources may be summed in another order (the
    # warp grouping of the deposit differs), so equal to FP32 rounding
    for f in range(8):
        np.testing.assert_allclose(host_out[f], outs[f], rtol=1e-6, atol=1e-12)


def test_duplicate_sources_accumulate(gpu):
    grid = (16, 16, 16)
    u = np.zeros((16, 16, 16), np.float32)
    idx = np.array([5, 5, 5, 9, 5, 4095, 0] * 40, np.int32)
    amt = np.arange(idx.size, dtype=np.float32) * 1e-3
    outs, mass, _ = run_world(grid, [1.0], [0.0], [(u, idx, amt)])
    ref = np.zeros(u.size)
    np.add.at(ref, idx, amt.astype(np.float64))
    np.testing.assert_allclose(outs[0].ravel(), ref, rtol=1e-6, atol=1e-9)
    assert abs(mass[0]["sources"] - amt.astype(np.float64).sum()) <= 1e-6 * amt.sum()


def test_errors_are_status_codes(gpu):
    with vfd.World(8, 8, 8, [vfd.field_params(1.0, 0.1)]) as w:
        with pytest.raises(vfd.VfdError) as e:
            w.set_sources(0, np.array([512], np.int32), np.array([1.0], np.float32))
        assert e.value.status == 1
        with pytest.raises(vfd.VfdError) as e:
            w.set_sources(3, np.array([1], np.int32), np.array([1.0], np.float32))
        assert e.value.status == 1
        with pytest.raises(vfd.VfdError) as e:
            w.tick(0)
        assert e.value.status == 1
        w.tick(1)  # still usable


@pytest.mark.parametrize("sigma", [(6.0, 1.0, 5.5), 6.2])
def test_wide_kernel_uses_full_line_path(gpu, sigma):
    """Radius above the overlap-save limit (16) on some axes: those passes run
    the full-line shared-memory FFT; results still match the oracle."""
    grid = (80, 50, 44)
    nx, ny, nz = grid
    u = vfd.synth_field(8, 0, 0, (nz, ny, nx))
    idx, amt = vfd.synth_sources(8, 0, 0, 50, nx * ny * nz)
    outs, mass, _ = run_world(grid, [sigma], [0.03], [(u, idx, amt)], substeps=2)
    ref = oracle.tick(u, sigma, 0.03, 2, idx, amt)
    assert rel_l2(outs[0], ref) <= REL_L2
    check_mass(outs[0], mass[0], 0.97, 0.0, nx * ny * nz)


def test_bounded_wait_reports_timeout(gpu):
    """Failure detection without a GPU fault: the passes' bounded wait for a
    bulk copy, run against a barrier that nothing completes, gives up after
    its limit (2e6 cycles, about 1 ms) and the library reports
    VFD_ERR_TIMEOUT; the context stays usable (a world ticks afterwards)."""
    st = vfd.lib().vfd_check_wait_timeout(0, 2_000_000)
    assert st == 5, vfd.lib().vfd_last_error(None).decode()
    with vfd.World(32, 24, 16, [vfd.field_params(1.0, 0.1)]) as w:
        w.upload(0, vfd.synth_field(1, 0, 0, (16, 24, 32)))
        w.tick(1)
        m = w.mass()
        assert m[0]["total"] > 0
