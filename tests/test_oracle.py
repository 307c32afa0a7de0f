"""CPU tests of the FP64 oracle: its three tiers agree with each other, it
matches the reference's own CPU gold routine, and it satisfies the
known-answer properties of the diffusion path.

The reference ships no golden vectors for this path (no test suite; only the
|sum(w) - 1| <= 1e-3 kernel check behind TEST_KERNEL, Diffusion.cu:1438-1454),
so the pins are: the reference's convolutionClampToBorderCPU
(convolutionFFT_gold.cpp:22-58) compiled from the reference tree into
oracle/_ref, the committed fixtures in tests/golden, and the properties below.
"""
import os

import numpy as np
import pytest

import oracle

RNG = np.random.default_rng(12345)


def _sep_window(sig3, r3):
    tx, ty, tz = (oracle.gauss_taps(s, r) for s, r in zip(sig3, r3))
    return np.einsum("z,y,x->zyx", tz, ty, tx)


def test_gauss_taps_normalised_and_symmetric():
    for s in (0.45, 0.8, 1.2, 1.95, 2.6):
        t = oracle.gauss_taps(s)
        assert len(t) == 2 * int(np.ceil(3 * s)) + 1
        assert abs(t.sum() - 1.0) < 1e-15
        np.testing.assert_array_equal(t, t[::-1])


def test_spectrum_dc_is_one_and_matches_dft():
    t = oracle.gauss_taps(1.3)
    F = 70
    spec = oracle.gauss_spectrum(t, F)
    r = (len(t) - 1) // 2
    wrapped = np.zeros(F)
    for j in range(-r, r + 1):
        wrapped[j % F] += t[j + r]
    np.testing.assert_allclose(spec, np.fft.fft(wrapped).real, atol=1e-15)
    assert abs(spec[0] - 1.0) < 1e-15


@pytest.mark.parametrize("n", [1, 2, 7, 30, 64, 105, 243, 392, 525])
def test_fft_matches_numpy(n):
    x = RNG.standard_normal(n) + 1j * RNG.standard_normal(n)
    np.testing.assert_allclose(oracle.fft(x), np.fft.fft(x), atol=1e-11 * max(1, n))
    np.testing.assert_allclose(oracle.fft(x, inverse=True), np.fft.ifft(x) * n, atol=1e-11 * max(1, n))


def test_tiers_agree_direct3d_separable_fft():
    """O1 (literal 3D sum) == O2 (separable direct) == O3 (FP64 FFT) for F >= n + r."""
    nz, ny, nx = 9, 11, 13
    sig = (1.1, 0.8, 1.4)
    r = tuple(int(np.ceil(3 * s)) for s in sig)
    v = RNG.random((nz, ny, nx))
    w = _sep_window(sig, r)
    o1 = oracle.conv_direct3d(v, w, (r[2], r[1], r[0]))
    o2 = v.copy()
    tx, ty, tz = (oracle.gauss_taps(s, rr) for s, rr in zip(sig, r))
    lk = np.zeros(3)
    L = oracle.lib()
    L.vfo_conv_sep_direct(nx, ny, nz, oracle._p(o2), oracle._p(tx), r[0], oracle._p(ty), r[1],
                          oracle._p(tz), r[2], oracle._p(lk))
    np.testing.assert_allclose(o2, o1, rtol=0, atol=1e-14)
    for F in [(nx + r[0], ny + r[1], nz + r[2]), (32, 24, 20), (nx + 2 * r[0], 30, 27)]:
        spec = [oracle.gauss_spectrum(oracle.gauss_taps(s, rr), f) for s, rr, f in zip(sig, r, F)]
        o3, full = oracle.conv_fft3d(v, F, spec3=spec)
        np.testing.assert_allclose(o3, o1, rtol=0, atol=1e-13)
        # mass identity: the full circular result carries the whole input mass
        assert abs(full - v.sum()) < 1e-12 * v.sum()
        # per-axis leak of O2 + kept mass = input mass
        assert abs(o2.sum() + lk.sum() - v.sum()) < 1e-12 * v.sum()
    # a grid shorter than n + r wraps mass around: must differ
    F = (nx + r[0] - 2, ny + r[1], nz + r[2])
    spec = [oracle.gauss_spectrum(oracle.gauss_taps(s, rr), f) for s, rr, f in zip(sig, r, F)]
    o3, _ = oracle.conv_fft3d(v, F, spec3=spec)
    assert np.abs(o3 - o1).max() > 1e-6


def test_dense_window_fft_matches_direct():
    """Window path of O3 (padKernel3D wrap + complex multiply) == O1, asymmetric window."""
    nz, ny, nx = 8, 10, 12
    v = RNG.random((nz, ny, nx))
    w = RNG.random((3, 5, 4))
    centre = (1, 2, 1)
    o1 = oracle.conv_direct3d(v, w, centre)
    o3, _ = oracle.conv_fft3d(v, (nx + 4, ny + 5, nz + 3), window=w, centre=centre)
    np.testing.assert_allclose(o3, o1, atol=1e-13)


@pytest.mark.skipif(not oracle.ref_gold_available(), reason="oracle/_ref not built (make -C oracle ref)")
def test_pin_against_reference_gold_2d():
    """The oracle's direct sum uses the reference's kernel orientation: it
    equals the reference's own convolutionClampToBorderCPU."""
    h, w = 23, 31
    data = RNG.random((h, w)).astype(np.float32)
    for (kh, kw, cy, cx) in [(5, 7, 2, 3), (3, 3, 1, 1), (4, 6, 1, 4)]:
        ker = RNG.random((kh, kw)).astype(np.float32)
        ref = oracle.ref_conv_clamp2d(data, ker, (cy, cx))
        mine = oracle.conv_clamp2d(data, ker, (cy, cx))
        np.testing.assert_allclose(mine, ref.astype(np.float64), rtol=2e-6, atol=1e-6)


def test_delta_returns_kernel():
    nz, ny, nx = 15, 15, 15
    u = np.zeros((nz, ny, nx), np.float32)
    u[7, 7, 7] = 1.0
    out, m = oracle.substep(u, (1.0, 0.9, 1.2), 0.0)
    r = (3, 3, 4)
    w = _sep_window((1.0, 0.9, 1.2), r)
    np.testing.assert_allclose(out[7 - r[2]:8 + r[2], 7 - r[1]:8 + r[1], 7 - r[0]:8 + r[0]], w, atol=1e-16)
    assert abs(out.sum() - 1.0) < 1e-14


def test_constant_field_constant_padding_is_fixed_point():
    """Constant field c with the constant-VF rule at b = c returns keep * c."""
    c = 3.5e-4
    u = np.full((10, 12, 14), c, np.float32)
    out, _ = oracle.substep(u, 1.3, 0.05, b=float(np.float32(c)), pad_mode=1, epi=9)
    np.testing.assert_allclose(out, 0.95 * float(np.float32(c)), rtol=1e-14)


def test_linearity_and_translation():
    a = RNG.random((12, 13, 14)).astype(np.float32)
    b = RNG.random((12, 13, 14)).astype(np.float32)
    oa, _ = oracle.substep(a, 1.1, 0.02)
    ob, _ = oracle.substep(b, 1.1, 0.02)
    oab, _ = oracle.substep(a + 2 * b, 1.1, 0.02)
    np.testing.assert_allclose(oab, oa + 2 * ob, atol=1e-14)
    # translation invariance away from the boundary
    u = np.zeros((20, 20, 20), np.float32)
    u[8, 9, 10] = 1
    s = np.roll(u, (1, -2, 3), axis=(0, 1, 2))
    ou, _ = oracle.substep(u, 1.0, 0.0)
    os_, _ = oracle.substep(s, 1.0, 0.0)
    np.testing.assert_allclose(np.roll(ou, (1, -2, 3), axis=(0, 1, 2)), os_, atol=1e-16)


def test_fft_method_matches_direct_method_with_padding_rule():
    u = RNG.random((10, 9, 11)).astype(np.float32)
    kw = dict(b=2e-4, pad_mode=1, epi=8)
    o_dir, m_dir = oracle.substep(u, (1.2, 0.7, 1.0), 0.03, **kw)
    o_fft, m_fft = oracle.substep(u, (1.2, 0.7, 1.0), 0.03, method=1, fft3=(15, 12, 14), **kw)
    np.testing.assert_allclose(o_fft, o_dir, atol=1e-15)
    assert abs(m_fft[0] - m_dir[0]) < 1e-15
    assert abs(m_fft[1] - m_dir[1]) < 1e-12 * abs(m_dir[0])


def test_stencil_power_is_heat_kernel():
    """Reference-mode kernel: the 7-point stencil to the power n (centre
    1 - 6 lambda - gamma dt, arms lambda; Diffusion.cu:1182-1195) sums to 1 at
    gamma = 0 and has per-axis variance 2 lambda n."""
    lam, n, R = 0.1333, 20, 20  # window wide enough to hold the whole support
    w = oracle.stencil_power(lam, 0.0, n, R)
    assert abs(w.sum() - 1.0) < 1e-9
    z = np.arange(-R, R + 1)
    var_x = (w.sum(axis=(0, 1)) * z * z).sum()
    assert abs(var_x - 2 * lam * n) < 1e-6
    # spectrum of S^n = (1 - 6 lam + 2 lam (cos kx + cos ky + cos kz))^n
    F = 2 * R + 1
    wrapped = np.roll(w, (-R, -R, -R), axis=(0, 1, 2))
    spec = np.fft.fftn(wrapped).real
    k = 2 * np.pi * np.arange(F) / F
    s1 = 1 - 6 * lam + 2 * lam * (np.cos(k)[:, None, None] + np.cos(k)[None, :, None] + np.cos(k)[None, None, :])
    np.testing.assert_allclose(spec, s1 ** n, atol=1e-9)


def test_update_restates_whchemical():
    t = RNG.random(1000).astype(np.float32)
    d = RNG.random(1000).astype(np.float32)
    p, d_after, total = oracle.update(t, d, 0.319)
    np.testing.assert_array_equal(p, (d.astype(np.float64) + t.astype(np.float64) * 0.319).astype(np.float32))
    assert not d_after.any()
    assert abs(total - p.astype(np.float64).sum()) < 1e-9


def test_tick_deposit_accumulates_duplicates():
    u = np.zeros((4, 4, 4), np.float32)
    idx = np.array([5, 5, 7, 5], np.int32)
    amt = np.array([1.0, 2.0, 4.0, 8.0], np.float32)
    out = oracle.tick(u, 1.0, 0.0, 1, idx, amt)
    assert out.flat[5] == 11.0 and out.flat[7] == 4.0


GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLDEN, "cfg0_oracle.npz")), reason="no fixture")
def test_oracle_against_committed_cfg0_fixture():
    """The oracle reproduces the committed seed-0 config-0 fixture."""
    import golden_cfg
    g = np.load(os.path.join(GOLDEN, "cfg0_oracle.npz"))
    fields = golden_cfg.cfg0_inputs()
    for f in range(8):
        u, idx, amt = fields[f]
        out = golden_cfg.cfg0_oracle_field(f, u, idx, amt)
        np.testing.assert_allclose(out.ravel()[g["sample_idx"]], g["sample"][f], rtol=1e-12, atol=1e-18)
        assert abs(out.sum() - g["sums"][f]) <= 1e-12 * abs(g["sums"][f])
        assert abs(np.sqrt((out ** 2).sum()) - g["l2"][f]) <= 1e-12 * g["l2"][f]


@pytest.mark.parametrize("pad_mode", [0, 1])
def test_cpu_port_matches_fp64_oracle(pad_mode):
    # the FP32 OpenMP port timed as the CPU baseline computes the same step:
    # relative L2 within 1e-5 of the FP64 oracle, deposit totals exact in FP64
    nx, ny, nz = 37, 24, 19
    rng = np.random.default_rng(3)
    u = rng.uniform(0.0, 1e-3, (nz, ny, nx)).astype(np.float32)
    idx = rng.integers(0, nx * ny * nz, 300).astype(np.int32)
    amt = rng.lognormal(-6.0, 1.0, 300).astype(np.float32)
    sig, rate, b, epi = (1.3, 0.8, 2.1), 0.04, (2e-4 if pad_mode else 0.0), 30
    rad = tuple(oracle.radius_of(s) for s in sig)
    ref = oracle.tick(u, sig, rate, 1, idx, amt, b=b, pad_mode=pad_mode, epi=epi)
    got = u.copy()
    oracle.port_substep(got, sig, rad, rate, b=b, pad_mode=pad_mode, epi=epi, nthreads=2)
    total = oracle.port_deposit_total(got, idx, amt)
    err = np.sqrt(((got.astype(np.float64) - ref) ** 2).sum() / (ref ** 2).sum())
    assert err <= 1e-5, err
    assert abs(total - got.astype(np.float64).sum()) <= 1e-9 * abs(total)  # FP64 total of the field


def test_multithreaded_oracle_equals_serial_oracle():
    """oracle.tick_mt (the OpenMP, column-blocked separable sums used for the
    full-size parity tests) gives the serial O2 oracle's result."""
    rng = np.random.default_rng(3)
    u = rng.random((23, 30, 141)).astype(np.float32)
    idx = rng.integers(0, u.size, 50).astype(np.int32)
    amt = rng.random(50).astype(np.float32)
    for sig in [(1.3, 0.8, 2.1), 0.4, (6.0, 1.0, 5.5)]:
        a = oracle.tick(u, sig, 0.05, 3, idx, amt)
        b, lk = oracle.tick_mt(u, sig, 0.05, 3, idx, amt)
        assert float(np.abs(a - b).max()) <= 1e-15 * float(np.abs(a).max())
        assert lk.shape == (3,)


@pytest.mark.parametrize("lam,n,R,G", [(0.1333, 30, 12, 96), (0.0667, 60, 14, 80), (0.1, 7, 9, 32)])
def test_spectral_stencil_oracle_equals_explicit_iteration(lam, n, R, G):
    """The FP64 spectral form of the stencil power (used at the reference's
    894-step size, where explicit iteration is out of reach) equals the
    explicit 7-point iteration."""
    a = oracle.stencil_power(lam, 0.0, n, R)
    b = oracle.stencil_power_spectral(lam, 0.0, n, R, G)
    assert float(np.abs(a - b).max()) <= 1e-14 * float(a.max())
