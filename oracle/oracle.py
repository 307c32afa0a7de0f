"""ctypes wrapper of the FP64 oracle (liboracle.so) and of the reference
builds under oracle/_ref.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py.  The product library never uses it.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_GOLD = os.path.join(HERE, "_ref", "libref_gold.so")
REF_REPLAY = os.path.join(HERE, "_ref", "libref_replay.so")

_lib = None
_P = C.c_void_p


def _p(a):
    return C.c_void_p(a.ctypes.data)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise ImportError(f"oracle not built: run `make -C {HERE}`")
        L = C.CDLL(LIB)
        L.vfo_gauss_taps.argtypes = [C.c_double, C.c_int, _P]
        L.vfo_gauss_taps.restype = C.c_int
        L.vfo_gauss_spectrum.argtypes = [_P, C.c_int, C.c_int, _P]
        L.vfo_fft.argtypes = [C.c_int, _P, _P, C.c_int]
        L.vfo_prepare.argtypes = [C.c_int, C.c_int, C.c_int, _P, C.c_double, C.c_int, C.c_int, _P]
        L.vfo_conv_sep_direct.argtypes = [C.c_int, C.c_int, C.c_int, _P, _P, C.c_int, _P, C.c_int,
                                          _P, C.c_int, _P]
        L.vfo_conv_sep_direct_mt.argtypes = L.vfo_conv_sep_direct.argtypes
        L.vfo_conv_fft3d.argtypes = [C.c_int] * 6 + [_P, _P, _P, _P, _P] + [C.c_int] * 6 + [_P]
        L.vfo_conv_fft3d.restype = C.c_int
        L.vfo_conv_direct3d.argtypes = [C.c_int] * 3 + [_P, _P, _P] + [C.c_int] * 6
        L.vfo_conv_clamp2d.argtypes = [C.c_int, C.c_int, _P, _P, C.c_int, C.c_int, C.c_int, C.c_int, _P]
        L.vfo_stencil_power.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int, _P]
        L.vfo_stencil_power.restype = C.c_int
        L.vfo_stencil_power_spectral.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, _P]
        L.vfo_stencil_power_spectral.restype = C.c_int
        L.vfo_substep.argtypes = ([C.c_int] * 3 + [_P, _P] + [C.c_double] * 3 + [C.c_int] * 3 +
                                  [C.c_double, C.c_double, C.c_int, C.c_int, C.c_int] +
                                  [C.c_int] * 3 + [_P])
        L.vfo_substep.restype = C.c_int
        L.vfo_deposit.argtypes = [_P, C.c_size_t, _P, _P, C.c_int64]
        L.vfo_deposit.restype = C.c_int
        L.vfo_update.argtypes = [C.c_size_t, _P, _P, _P, C.c_double]
        L.vfo_update.restype = C.c_double
        L.vfo_sum.argtypes = [_P, C.c_size_t]
        L.vfo_sum.restype = C.c_double
        L.vfp_substep.argtypes = ([C.c_int] * 3 + [_P, _P, _P, C.c_double, C.c_float] +
                                  [C.c_int] * 3)
        L.vfp_substep.restype = C.c_int
        L.vfp_deposit_total.argtypes = [_P, C.c_size_t, _P, _P, C.c_int64]
        L.vfp_deposit_total.restype = C.c_double
        L.vfp_max_threads.restype = C.c_int
        _lib = L
    return _lib


def radius_of(sigma):
    return int(np.ceil(3.0 * sigma))


def gauss_taps(sigma, r=None):
    r = radius_of(sigma) if r is None else r
    t = np.empty(2 * r + 1, np.float64)
    assert lib().vfo_gauss_taps(float(sigma), r, _p(t)) == 0
    return t


def gauss_spectrum(taps, F):
    r = (len(taps) - 1) // 2
    t = np.ascontiguousarray(taps, np.float64)
    s = np.empty(F, np.float64)
    lib().vfo_gauss_spectrum(_p(t), r, F, _p(s))
    return s


def fft(x, inverse=False):
    re = np.ascontiguousarray(np.real(x), np.float64).copy()
    im = np.ascontiguousarray(np.imag(x), np.float64).copy()
    lib().vfo_fft(len(re), _p(re), _p(im), 1 if inverse else -1)
    return re + 1j * im


def substep(u, sigma3, rate, radius3=None, b=0.0, pad_mode=0, epi=0, method=0, fft3=None):
    """One substep on field u (nz, ny, nx) float32; returns (out float64, [sum_v, leaked])."""
    u = np.ascontiguousarray(u, np.float32)
    nz, ny, nx = u.shape
    s = [float(sigma3)] * 3 if np.isscalar(sigma3) else [float(v) for v in sigma3]
    r = [radius_of(v) for v in s] if radius3 is None else (
        [int(radius3)] * 3 if np.isscalar(radius3) else [int(v) for v in radius3])
    F = fft3 if fft3 is not None else (0, 0, 0)
    out = np.empty(u.shape, np.float64)
    m = np.zeros(3, np.float64)
    rc = lib().vfo_substep(nx, ny, nz, _p(u), _p(out), s[0], s[1], s[2], r[0], r[1], r[2],
                           float(rate), float(b), int(pad_mode), int(epi), int(method),
                           int(F[0]), int(F[1]), int(F[2]), _p(m))
    assert rc == 0
    return out, m[:2].copy()


def tick(u, sigma3, rate, n_substeps, idx, amt, **kw):
    """n substeps in FP64 (separable direct method), then the deposit."""
    out = np.asarray(u, np.float64)
    for _ in range(n_substeps):
        out = _substep64(out, sigma3, rate, **kw)
    return deposit(np.ascontiguousarray(out), idx, amt)


def _substep64(u64, sigma3, rate, radius3=None, b=0.0, pad_mode=0, epi=0):
    """FP64-input substep through the separable direct path (O2) in numpy."""
    nz, ny, nx = u64.shape
    s = [float(sigma3)] * 3 if np.isscalar(sigma3) else [float(v) for v in sigma3]
    r = [radius_of(v) for v in s] if radius3 is None else (
        [int(radius3)] * 3 if np.isscalar(radius3) else [int(v) for v in radius3])
    v = np.array(u64, np.float64, copy=True) - b
    if pad_mode == 1:
        mask = np.zeros_like(v, dtype=bool)
        mask[1:nz - 1, 1:ny - 1, 1:min(epi, nx)] = True
        v[~mask] = 0.0
    v = np.ascontiguousarray(v)
    tx, ty, tz = gauss_taps(s[0], r[0]), gauss_taps(s[1], r[1]), gauss_taps(s[2], r[2])
    lk = np.zeros(3, np.float64)
    lib().vfo_conv_sep_direct(nx, ny, nz, _p(v), _p(tx), r[0], _p(ty), r[1], _p(tz), r[2], _p(lk))
    return (1.0 - rate) * (b + v)


def tick_mt(u, sigma3, rate, n_substeps, idx, amt, radius3=None):
    """oracle.tick with the separable direct sums spread over OpenMP threads
    (vfo_conv_sep_direct_mt): FP64 throughout, zero padding; for the
    full-size grids.  Returns (out float64, leaked [x, y, z] of the last substep)."""
    nz, ny, nx = np.shape(u)
    s = [float(sigma3)] * 3 if np.isscalar(sigma3) else [float(v) for v in sigma3]
    r = [radius_of(v) for v in s] if radius3 is None else (
        [int(radius3)] * 3 if np.isscalar(radius3) else [int(v) for v in radius3])
    tx, ty, tz = gauss_taps(s[0], r[0]), gauss_taps(s[1], r[1]), gauss_taps(s[2], r[2])
    v = np.array(u, np.float64, copy=True, order="C")
    lk = np.zeros(3, np.float64)
    for _ in range(n_substeps):
        lib().vfo_conv_sep_direct_mt(nx, ny, nz, _p(v), _p(tx), r[0], _p(ty), r[1], _p(tz), r[2], _p(lk))
        v *= (1.0 - rate)
    return deposit(v, idx, amt), lk


def deposit(u64, idx, amt):
    i = np.ascontiguousarray(idx, np.int32)
    a = np.ascontiguousarray(amt, np.float32)
    assert lib().vfo_deposit(_p(u64), u64.size, _p(i), _p(a), i.size) == 0
    return u64


def conv_direct3d(v, w, centre):
    v = np.ascontiguousarray(v, np.float64)
    w = np.ascontiguousarray(w, np.float64)
    nz, ny, nx = v.shape
    kd, kh, kw = w.shape
    out = np.empty_like(v)
    lib().vfo_conv_direct3d(nx, ny, nz, _p(v), _p(out), _p(w), kw, kh, kd,
                            centre[2], centre[1], centre[0])
    return out


def conv_fft3d(v, fft3, spec3=None, window=None, centre=None):
    """FFT convolution on grid fft3=(Fx,Fy,Fz); returns (cropped, full-grid sum)."""
    v = np.array(v, np.float64, copy=True, order="C")
    nz, ny, nx = v.shape
    fs = np.zeros(1, np.float64)
    if window is not None:
        w = np.ascontiguousarray(window, np.float64)
        kd, kh, kw = w.shape
        rc = lib().vfo_conv_fft3d(nx, ny, nz, fft3[0], fft3[1], fft3[2], _p(v), None, None, None,
                                  _p(w), kw, kh, kd, centre[2], centre[1], centre[0], _p(fs))
    else:
        sx, sy, sz = [np.ascontiguousarray(s, np.float64) for s in spec3]
        rc = lib().vfo_conv_fft3d(nx, ny, nz, fft3[0], fft3[1], fft3[2], _p(v), _p(sx), _p(sy),
                                  _p(sz), None, 0, 0, 0, 0, 0, 0, _p(fs))
    assert rc == 0
    return v, float(fs[0])


def conv_clamp2d(data, ker, centre):
    d = np.ascontiguousarray(data, np.float64)
    k = np.ascontiguousarray(ker, np.float64)
    out = np.empty_like(d)
    lib().vfo_conv_clamp2d(d.shape[0], d.shape[1], _p(d), _p(k), k.shape[0], k.shape[1],
                           centre[0], centre[1], _p(out))
    return out


def stencil_power(lam, gamma_dt, n_steps, R):
    w = np.empty((2 * R + 1,) * 3, np.float64)
    assert lib().vfo_stencil_power(float(lam), float(gamma_dt), int(n_steps), int(R), _p(w)) == 0
    return w


def stencil_power_spectral(lam, gamma_dt, n_steps, R, G):
    """The same window from the stencil's spectrum on a periodic G^3 grid (FP64)."""
    w = np.empty((2 * R + 1,) * 3, np.float64)
    assert lib().vfo_stencil_power_spectral(float(lam), float(gamma_dt), int(n_steps), int(R), int(G), _p(w)) == 0
    return w


def ref_compute_kernel3d(lam, gamma_dt, kernel_radius, niter, F, window):
    """The reference's computeKernel3D (its own kernels + cuFFT, GPU)."""
    L = C.CDLL(REF_REPLAY)
    f = L.ref_compute_kernel3d
    f.argtypes = [C.c_float, C.c_float, C.c_int, C.c_int, C.c_int, C.c_int, _P]
    f.restype = C.c_int
    L.ref_replay_error.restype = C.c_char_p
    out = np.empty((window,) * 3, np.float32)
    rc = f(float(lam), float(gamma_dt), int(kernel_radius), int(niter), int(F), int(window), _p(out))
    if rc != 0:
        raise RuntimeError("ref computeKernel3D replay failed: " + L.ref_replay_error().decode())
    return out


def update(t, d, decay):
    """WHChemical::update restated: returns (p, d_after, total)."""
    t = np.ascontiguousarray(t, np.float32)
    d = np.array(d, np.float32, copy=True)
    p = np.empty_like(t)
    s = lib().vfo_update(t.size, _p(t), _p(d), _p(p), float(decay))
    return p, d, s


# ---- FP32 OpenMP CPU port (timed baseline) --------------------------------
def port_substep(u, sigma3, radius3, rate, b=0.0, pad_mode=0, epi=0, nthreads=0):
    """In place on float32 u (nz, ny, nx)."""
    assert u.dtype == np.float32 and u.flags.c_contiguous
    nz, ny, nx = u.shape
    s = (C.c_double * 3)(*sigma3)
    r = (C.c_int * 3)(*radius3)
    rc = lib().vfp_substep(nx, ny, nz, _p(u), s, r, float(rate), float(b), int(pad_mode), int(epi),
                           int(nthreads))
    assert rc == 0


def port_deposit_total(u, idx, amt):
    i = np.ascontiguousarray(idx, np.int32)
    a = np.ascontiguousarray(amt, np.float32)
    return lib().vfp_deposit_total(_p(u), u.size, _p(i), _p(a), i.size)


def port_threads():
    return int(lib().vfp_max_threads())


# ---- reference builds (oracle/_ref) ---------------------------------------
def ref_gold_available():
    return os.path.exists(REF_GOLD)


def ref_conv_clamp2d(data, ker, centre):
    """The reference's convolutionClampToBorderCPU (convolutionFFT_gold.cpp:22-58)."""
    L = C.CDLL(REF_GOLD)
    f = L.convolutionClampToBorderCPU
    f.argtypes = [_P, _P, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
    d = np.ascontiguousarray(data, np.float32)
    k = np.ascontiguousarray(ker, np.float32)
    out = np.empty_like(d)
    f(_p(out), _p(d), _p(k), d.shape[0], d.shape[1], k.shape[0], k.shape[1], centre[0], centre[1])
    return out


def ref_replay_available():
    return os.path.exists(REF_REPLAY)


def ref_replay(u, fft3, window, centre, epi, base):
    """The reference's own kernels + cuFFT in fftDiffuse3D's order (GPU)."""
    L = C.CDLL(REF_REPLAY)
    f = L.ref_replay_fft_diffuse3d
    f.argtypes = [_P, _P] + [C.c_int] * 6 + [_P] + [C.c_int] * 7 + [C.c_float]
    f.restype = C.c_int
    L.ref_replay_error.restype = C.c_char_p
    u = np.ascontiguousarray(u, np.float32)
    w = np.ascontiguousarray(window, np.float32)
    nz, ny, nx = u.shape
    kd, kh, kw = w.shape
    out = np.empty_like(u)
    rc = f(_p(u), _p(out), nz, ny, nx, fft3[2], fft3[1], fft3[0], _p(w), kd, kh, kw,
           centre[0], centre[1], centre[2], int(epi), float(base))
    if rc != 0:
        raise RuntimeError("ref replay failed: " + L.ref_replay_error().decode())
    return out
