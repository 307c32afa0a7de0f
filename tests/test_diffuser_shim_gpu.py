"""GPU test of the C++ drop-in for the reference's Diffuser
(vf-version_7_3_b200/host/vfd_diffuser.hpp), built against the reference's
own c_ctx (src/Diffusion/convolutionFFT_common.h) by oracle/Makefile into
oracle/_ref/libref_shim.so, and driven with the reference's allocation
pattern: kernel spectra in chem_cctx->h_kernelspectrum[ic] (one per
chemical, made by the reference's padKernel3D + cuFFT), the kernel context a
dead local with one shared window buffer per GPU by the first call.

Each chemical's output is compared with the reference's own fftDiffuse3D
kernels + cuFFT (oracle/_ref/libref_replay.so) on the same input, window,
FFT grid, epiBoundary and baseline: <= 1e-5 relative L2 per chemical."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
import vfd
from conftest import ROOT

pytestmark = pytest.mark.gpu

SHIM = os.path.join(ROOT, "oracle", "_ref", "libref_shim.so")
# eight chemicals with distinct stencil weights (the reference's lambda =
# D dt / dx^2 per cytokine, woundHealingWorld.cpp:954-961)
LAMBDAS = [0.1333, 0.0667, 0.1, 0.12, 0.05, 0.0833, 0.1111, 0.0909]
# the reference's retention factors (woundHealingWorld.cpp:2640-2648)
DECAY = [0.319, 3.052e-5, 0.67, 0.2, 0.2, 0.7937, 0.9284, 0.2]


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def snap_transform_size(n):
    """The reference's FFT length rule (snapTransformSize, Diffusion.cu:39-70):
    align to 16, then the next power of two."""
    n = (n + 15) // 16 * 16
    p = 1
    while p < n:
        p *= 2
    return p


def _setup(nx, ny, nz, R, steps):
    k = 2 * R + 1
    wins = [oracle.stencil_power(l, 0.0, steps, R).astype(np.float32) for l in LAMBDAS]
    fft = [snap_transform_size(n + k - 1) for n in (nx, ny, nz)]
    base = np.array([2e-4, 5e-4, 1e-4, 3e-4, 4e-4, 1.5e-4, 2.5e-4, 3.5e-4], np.float32)
    ins = [vfd.synth_field(4, 0, c, (nz, ny, nx)) for c in range(8)]
    return k, wins, fft, base, ins


def _run(nx, ny, nz, wins, k, fft, base, ins, epi, calls, decay=None, dins=None, lambdas=None, n_steps=0):
    lib = C.CDLL(SHIM)
    f = lib.shim_harness_run
    P = C.c_void_p
    f.argtypes = [C.c_int] * 4 + [P, C.c_int, P, P, P, P, C.c_int, C.c_int, P, P, P, P, C.c_int, P, C.c_int]
    f.restype = C.c_int
    arr = lambda xs: (P * len(xs))(*[x.ctypes.data for x in xs])
    outs = [np.empty_like(u) for u in ins]
    totals = np.zeros(8, np.float32)
    err = C.create_string_buffer(512)
    fft3 = np.array(fft, np.int32)
    lam = None if lambdas is None else np.asarray(lambdas, np.float32)
    rc = f(nx, ny, nz, 8, arr(wins), k, fft3.ctypes.data, base.ctypes.data, arr(ins), arr(outs), epi, calls,
           None if decay is None else np.asarray(decay, np.float32).ctypes.data,
           None if dins is None else arr(dins), totals.ctypes.data,
           None if lam is None else lam.ctypes.data, n_steps, err, 512)
    assert rc == 0, err.value.decode()
    return outs, totals


@pytest.mark.skipif(not os.path.exists(SHIM), reason="oracle/_ref/libref_shim.so not built (no reference tree)")
@pytest.mark.parametrize("reference_grid", [False, True])
def test_diffuser_dropin_with_reference_cctx(gpu, reference_grid, monkeypatch):
    """diffuseChemGPU x2 on 8 chemicals: each equals the reference's own
    kernels + cuFFT with that chemical's spectrum (not another chemical's
    window, and not the freed kernel context's); on the cheapest grid with
    the windows recovered from the spectra (default) and on the reference's
    own grid (VFD_SHIM_REFERENCE_GRID=1)."""
    monkeypatch.setenv("VFD_SHIM_REFERENCE_GRID", "1" if reference_grid else "0")
    nx, ny, nz, R = 40, 34, 28, 6
    epi = 33
    k, wins, fft, base, ins = _setup(nx, ny, nz, R, 12)
    outs, _ = _run(nx, ny, nz, wins, k, fft, base, ins, epi, calls=2)
    for c in range(8):
        ref = oracle.ref_replay(ins[c], fft, wins[c], (R, R, R), epi, float(base[c]))
        assert rel_l2(outs[c], ref) <= 1e-5, (c, rel_l2(outs[c], ref))
    # chemicals that share the reference's per-GPU window buffer (ic, ic + 2)
    # still get their own kernels
    assert rel_l2(outs[0], outs[2]) > 1e-3


@pytest.mark.skipif(not os.path.exists(SHIM), reason="oracle/_ref/libref_shim.so not built (no reference tree)")
def test_diffuser_dropin_device_update(gpu):
    """diffuseAndUpdateChemGPU x2: p = d + t * cytokineDecay, d = 0 on the
    device (WHChemical::update, WHChemical.cpp:420-450), chained over two
    ticks; the FP64 totals match the updated fields."""
    nx, ny, nz, R = 36, 30, 26, 5
    epi = 30
    k, wins, fft, base, ins = _setup(nx, ny, nz, R, 10)
    dins = [vfd.synth_field(5, 0, c, (nz, ny, nx), 0.0, 1e-4) for c in range(8)]
    outs, totals = _run(nx, ny, nz, wins, k, fft, base, ins, epi, calls=2, decay=DECAY, dins=dins)
    for c in range(8):
        p = ins[c]
        for _ in range(2):
            t = oracle.ref_replay(p, fft, wins[c], (R, R, R), epi, float(base[c]))
            p, _, _ = oracle.update(t, dins[c], DECAY[c])
        assert rel_l2(outs[c], p) <= 1e-5, (c, rel_l2(outs[c], p))
        s = outs[c].astype(np.float64).sum()
        assert abs(float(totals[c]) - s) <= 1e-6 * abs(s) + 1e-30, c


@pytest.mark.skipif(not os.path.exists(SHIM), reason="oracle/_ref/libref_shim.so not built (no reference tree)")
def test_diffuser_dropin_with_own_kernel_preparation(gpu):
    """vfd::prepKernelSpectra in place of the reference's prepKernel: the
    stencil window and its spectrum computed with this library (no cuFFT);
    each chemical's diffusion still equals the reference's kernels + cuFFT
    fed the same stencil window (the FP64 oracle's)."""
    nx, ny, nz, R = 40, 34, 28, 6
    epi = 33
    steps = 12
    k, wins, fft, base, ins = _setup(nx, ny, nz, R, steps)
    outs, _ = _run(nx, ny, nz, wins, k, fft, base, ins, epi, calls=1, lambdas=LAMBDAS, n_steps=steps)
    for c in range(8):
        ref = oracle.ref_replay(ins[c], fft, wins[c], (R, R, R), epi, float(base[c]))
        assert rel_l2(outs[c], ref) <= 1e-5, (c, rel_l2(outs[c], ref))
