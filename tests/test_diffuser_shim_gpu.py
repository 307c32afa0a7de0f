"""GPU test of the C++ drop-in for the reference's Diffuser
(vf-version_7_3_b200/host/vfd_diffuser.hpp): constructed from c_ctx /
WHChemical-shaped contexts and called as diffuseChemGPU(rightWallIndex), it
reproduces fftDiffuse3D's output per chemical (reference-mode window,
padDataConstantVF3D boundary, no decay)."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
import vfd
from conftest import PKG

pytestmark = pytest.mark.gpu

SHIM = os.path.join(PKG, "lib", "libvfd_shim_selftest.so")


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def reference_field(u, w, base, epi):
    """b * sum(w) + conv(M (u - b)) -- fftDiffuse3D with padDataConstantVF3D."""
    nz, ny, nx = u.shape
    R = w.shape[0] // 2
    v = u.astype(np.float64) - np.float64(np.float32(base))
    mask = np.zeros_like(v, bool)
    mask[1:nz - 1, 1:ny - 1, 1:min(epi, nx)] = True
    v[~mask] = 0.0
    w64 = w.astype(np.float64)
    return oracle.conv_direct3d(v, w64, (R, R, R)) + np.float64(np.float32(base)) * w64.sum()


def test_diffuser_dropin(gpu):
    lib = C.CDLL(SHIM)
    f = lib.vfd_shim_selftest
    f.restype = C.c_int
    nx, ny, nz, nchem = 40, 34, 28, 3
    R = 6
    epi = 33
    lams = [0.1333, 0.0667, 0.1]
    wins = [oracle.stencil_power(l, 0.0, 12, R).astype(np.float32) for l in lams]
    base = np.array([2e-4, 5e-4, 1e-4], np.float32)
    ins = [vfd.synth_field(4, 0, c, (nz, ny, nx)) for c in range(nchem)]
    outs = [np.empty_like(u) for u in ins]
    P = C.c_void_p
    arr = lambda xs: (P * len(xs))(*[x.ctypes.data for x in xs])
    err = C.create_string_buffer(256)
    k = 2 * R + 1
    rc = f(nx, ny, nz, nchem, arr(ins), arr(outs), arr(wins), k, k, k, base.ctypes.data_as(P), epi, 2,
           err, 256)
    assert rc == 0, err.value
    for c in range(nchem):
        ref = reference_field(ins[c], wins[c], base[c], epi)
        assert rel_l2(outs[c], ref) <= 1e-5, c
