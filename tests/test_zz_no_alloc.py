"""GPU test of the allocation-free entry point vfd_fft_diffuse3d_noalloc.

It serves callers that cannot call cudaMalloc -- code that owns all device
memory in its own arena or pool, or that must not cause the device-wide
synchronisation of cudaMalloc / cudaFree inside a per-tick loop.  The test
allocates the field and the kernel spectrum itself (here with torch) and
checks, on two calls in a row, that the result equals the library's regular
entry point (a VFD_METHOD_FFT3D world with the same window) and the FP64
oracle's direct 3D convolution, within the tolerance of the other parity
tests, on FFT grids with radix-8 and odd lengths.  This file is collected last
so that a run stopping at the first failure has run every other test before
it.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
import vfd

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def oracle_substep(u, win, R, pad_mode, base, epi, keep):
    """keep * (b * sum(w) + conv(M (u - b))) in FP64 (zero padding: b = 0, M = 1)."""
    nz, ny, nx = u.shape
    b = np.float64(np.float32(base)) if pad_mode == vfd.PAD_CONSTANT_VF else 0.0
    v = u.astype(np.float64) - b
    if pad_mode == vfd.PAD_CONSTANT_VF:
        mask = np.zeros_like(v, bool)
        mask[1:nz - 1, 1:ny - 1, 1:min(epi, nx)] = True
        v[~mask] = 0.0
    w64 = win.astype(np.float64)
    return keep * (oracle.conv_direct3d(v, w64, (R, R, R)) + b * w64.sum())


@pytest.mark.parametrize("pad_mode,grid,fft", [
    (vfd.PAD_ZERO, (40, 36, 30), (56, 48, 42)),          # even x, 7-smooth, >= n + R
    (vfd.PAD_CONSTANT_VF, (40, 36, 30), (56, 48, 42)),
    (vfd.PAD_CONSTANT_VF, (40, 36, 28), (64, 45, 35)),   # radix-8 x, odd y and z lengths
])
def test_noalloc_matches_regular_entry_point(gpu, pad_mode, grid, fft):
    import torch
    nx, ny, nz = grid
    R = 6
    fx, fy, fz = fft
    base, epi, keep = 3e-4, 33, 0.95
    win = oracle.stencil_power(0.1333, 0.0, 12, R).astype(np.float32)
    u = vfd.synth_field(21, 0, 0, (nz, ny, nx))

    # regular entry point: a world with the same window, two substeps
    params = [vfd.field_params(1.0, 1.0 - keep, radius=R, baseline=base)]
    with vfd.World(nx, ny, nz, params, pad_mode=pad_mode, epi_boundary=epi, fft=(fx, fy, fz),
                   method=vfd.METHOD_FFT3D) as w:
        w.set_window(0, win, (R, R, R))
        w.upload(0, u)
        w.tick(1)
        ref1 = w.download(0)
        w.tick(1)
        ref2 = w.download(0)

    # the same window's spectrum, made by the caller (layout [fz][fy][fx/2+1])
    wrapped = np.zeros((fz, fy, fx), np.float64)
    for z in range(2 * R + 1):
        for y in range(2 * R + 1):
            for x in range(2 * R + 1):
                wrapped[(z - R) % fz, (y - R) % fy, (x - R) % fx] += win[z, y, x]
    spec = np.fft.rfftn(wrapped).astype(np.complex64)
    kspec = torch.from_numpy(np.ascontiguousarray(spec).view(np.float32)).cuda()
    field = torch.from_numpy(u.copy()).cuda()
    ksum = float(spec[0, 0, 0].real)
    lib = vfd.lib()
    outs = []
    for _ in range(2):
        st = lib.vfd_fft_diffuse3d_noalloc(C.c_void_p(field.data_ptr()), C.c_void_p(kspec.data_ptr()),
                                           nx, ny, nz, fx, fy, fz, pad_mode, epi, base, ksum, keep, None)
        assert st == 0
        torch.cuda.synchronize()
        outs.append(field.cpu().numpy().copy())
    assert rel_l2(outs[0], ref1) <= 1e-5
    assert rel_l2(outs[1], ref2) <= 1e-5
    # and against the FP64 oracle, two substeps chained
    o1 = oracle_substep(u, win, R, pad_mode, base, epi, keep)
    o2 = oracle_substep(o1, win, R, pad_mode, base, epi, keep)
    assert rel_l2(outs[0], o1) <= 1e-5
    assert rel_l2(outs[1], o2) <= 1e-5


def test_noalloc_rejects_sizes_beyond_the_static_scratch(gpu):
    import torch
    f = torch.zeros(8, device="cuda")
    # 1024 x 512 x 512 needs ~1 GiB of spectrum scratch: beyond the 32 MiB array
    st = vfd.lib().vfd_fft_diffuse3d_noalloc(C.c_void_p(f.data_ptr()), C.c_void_p(f.data_ptr()),
                                             1000, 500, 500, 1024, 512, 512, 0, 0, 0.0, 1.0, 1.0, None)
    assert st == 1
