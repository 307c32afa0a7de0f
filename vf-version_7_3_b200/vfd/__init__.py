"""ctypes binding of libvfd.so (include/vfd.h) for tests and benchmarks.

The library is the product: every call here goes through its C ABI.  There
is no Python or CPU fallback -- importing this module raises if libvfd.so
is missing, and world creation raises if no CUDA device is visible.

The `World` class mirrors the reference's diffusion surface
(src/Diffusion/Diffuser.h:24-70, Diffuser::diffuseChemGPU and the
WHChemical update it feeds): per-world fields resident on the device, one
`tick()` per simulation tick, `diffuse_host()` for the reference's
host-buffer-in / host-buffer-out contract.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libvfd.so")

PAD_ZERO = 0
PAD_CONSTANT_VF = 1

METHOD_SEPARABLE = 0
METHOD_FFT3D = 1
METHOD_PLAIN = 2

STATUS = {
    0: "VFD_OK", 1: "VFD_ERR_INVALID_ARG", 2: "VFD_ERR_OUT_OF_MEMORY",
    3: "VFD_ERR_BUDGET", 4: "VFD_ERR_CUDA", 5: "VFD_ERR_TIMEOUT",
    6: "VFD_ERR_DEVICE_FAULT", 7: "VFD_ERR_NOT_SUPPORTED", 8: "VFD_ERR_NO_DEVICE",
}

# Every symbol include/vfd.h declares (checked by the CPU test suite).
EXPORTED = [
    "vfd_world_create", "vfd_world_destroy", "vfd_world_fft_dims",
    "vfd_world_device_bytes", "vfd_upload_field", "vfd_download_field",
    "vfd_field_device_ptr", "vfd_set_sources", "vfd_tick", "vfd_read_mass",
    "vfd_diffuse_host", "vfd_status_string", "vfd_last_error",
    "vfd_kernel_launch_count", "vfd_synth_field", "vfd_synth_sources",
    "vfd_world_set_profiling", "vfd_read_profile",
    "vfd_batch_create", "vfd_batch_tick", "vfd_batch_destroy", "vfd_batch_last_error",
    "vfd_set_window", "vfd_synth_field_device", "vfd_stencil_window",
    "vfd_server_create", "vfd_server_submit", "vfd_server_wait", "vfd_server_drain",
    "vfd_server_get_stats", "vfd_server_clock", "vfd_server_destroy",
    "vfd_fft_diffuse3d_noalloc", "vfd_update_gradients", "vfd_sample_field", "vfd_write_vtk",
    "vfd_autotune", "vfd_world_tuning", "vfd_autotune_set", "vfd_autotune_clear",
    "vfd_set_spectrum", "vfd_set_boundary", "vfd_tick_update", "vfd_diffuse_update_host",
    "vfd_batch_autotune", "vfd_window_spectrum", "vfd_write_raw_normalized", "vfd_write_csv",
    "vfd_check_wait_timeout", "vfd_spectrum_window",
]

PASS_METHODS = {0: "register_fft", 1: "overlap_save", 2: "full_line"}


class VfdError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class FieldParams(C.Structure):
    _fields_ = [("sigma", C.c_double * 3), ("radius", C.c_int * 3),
                ("decay_rate", C.c_double), ("baseline", C.c_float)]


class WorldDesc(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("n_fields", C.c_int), ("fields", C.POINTER(FieldParams)),
                ("pad_mode", C.c_int), ("epi_boundary", C.c_int),
                ("fft", C.c_int * 3), ("method", C.c_int)]


class Mass(C.Structure):
    _fields_ = [("input_sum", C.c_double), ("leaked", C.c_double * 3),
                ("conv_sum", C.c_double), ("total", C.c_double),
                ("sources", C.c_double), ("reserved", C.c_double)]

    def as_dict(self):
        return {"input_sum": self.input_sum, "leaked": list(self.leaked),
                "conv_sum": self.conv_sum, "total": self.total,
                "sources": self.sources}


class RequestDesc(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("n_fields", C.c_int),
                ("fields", C.POINTER(FieldParams)), ("pad_mode", C.c_int), ("epi_boundary", C.c_int),
                ("ticks", C.c_int), ("init", C.POINTER(C.c_void_p)), ("synth_seed", C.c_uint64),
                ("synth_world", C.c_int), ("synth_lo", C.c_float), ("synth_hi", C.c_float),
                ("src_idx", C.POINTER(C.c_void_p)), ("src_amt", C.POINTER(C.c_void_p)),
                ("n_src", C.POINTER(C.c_int64)), ("result", C.POINTER(C.c_void_p)),
                ("mass", C.POINTER(Mass))]


class RequestInfo(C.Structure):
    _fields_ = [("id", C.c_uint64), ("status", C.c_int), ("t_submit", C.c_double),
                ("t_admit", C.c_double), ("t_done", C.c_double), ("voxel_steps", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("admitted", C.c_int64), ("completed", C.c_int64),
                ("rejected", C.c_int64), ("active", C.c_int64), ("queued", C.c_int64),
                ("rounds", C.c_int64), ("busy_s", C.c_double), ("voxel_steps_done", C.c_double),
                ("p50_latency_s", C.c_double), ("p99_latency_s", C.c_double),
                ("mean_latency_s", C.c_double), ("hbm_in_use", C.c_size_t), ("hbm_peak", C.c_size_t),
                ("device_s", C.c_double), ("p50_completed_s", C.c_double), ("p99_completed_s", C.c_double),
                ("censored", C.c_int64), ("host_batch_s", C.c_double), ("host_admit_s", C.c_double),
                ("host_wait_s", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class AxisTuning(C.Structure):
    _fields_ = [("method", C.c_int), ("ctas_per_sm", C.c_int), ("fft_len", C.c_int),
                ("radix_order", C.c_int), ("variant", C.c_int), ("ms", C.c_float)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["method"] = PASS_METHODS.get(self.method, self.method)
        return d


def load(path=LIB_PATH):
    if not os.path.exists(path):
        raise ImportError(f"libvfd.so not built at {path}; run `make` in "
                          f"{os.path.dirname(path)}/.. or __graft_entry__.build()")
    lib = C.CDLL(path)
    P = C.c_void_p
    lib.vfd_world_create.argtypes = [C.POINTER(WorldDesc), C.c_int, C.POINTER(P)]
    lib.vfd_world_destroy.argtypes = [P]
    lib.vfd_world_fft_dims.argtypes = [P, C.POINTER(C.c_int)]
    lib.vfd_world_device_bytes.argtypes = [P, C.POINTER(C.c_size_t)]
    lib.vfd_upload_field.argtypes = [P, C.c_int, P, P]
    lib.vfd_download_field.argtypes = [P, C.c_int, P, P]
    lib.vfd_field_device_ptr.argtypes = [P, C.c_int, C.POINTER(P)]
    lib.vfd_set_sources.argtypes = [P, C.c_int, P, P, C.c_int64]
    lib.vfd_tick.argtypes = [P, C.c_int, P]
    lib.vfd_read_mass.argtypes = [P, C.POINTER(Mass), P]
    lib.vfd_diffuse_host.argtypes = [P, C.POINTER(P), C.POINTER(P), C.c_int]
    lib.vfd_world_set_profiling.argtypes = [P, C.c_int]
    lib.vfd_read_profile.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_int64)]
    lib.vfd_set_window.argtypes = [P, C.c_int, P] + [C.c_int] * 6
    lib.vfd_set_spectrum.argtypes = [P, C.c_int, P, C.c_int, C.c_int, C.c_int]
    lib.vfd_window_spectrum.argtypes = [P] + [C.c_int] * 9 + [P, C.c_int]
    lib.vfd_spectrum_window.argtypes = [P] + [C.c_int] * 9 + [P, C.c_int]
    lib.vfd_set_boundary.argtypes = [P, C.c_int, P]
    lib.vfd_tick_update.argtypes = [P, C.c_int, C.POINTER(P), P, P]
    lib.vfd_diffuse_update_host.argtypes = [P, C.POINTER(P), C.POINTER(P), P, C.c_int]
    lib.vfd_batch_create.argtypes = [C.POINTER(P), C.c_int, C.POINTER(P)]
    lib.vfd_batch_tick.argtypes = [P, C.c_int, P]
    lib.vfd_batch_autotune.argtypes = [P, C.c_int, P]
    lib.vfd_batch_destroy.argtypes = [P]
    lib.vfd_batch_last_error.argtypes = [P]
    lib.vfd_batch_last_error.restype = C.c_char_p
    lib.vfd_fft_diffuse3d_noalloc.argtypes = [P, P] + [C.c_int] * 8 + [C.c_float] * 3 + [P]
    lib.vfd_update_gradients.argtypes = [P, P, P, P, P, P, P]
    lib.vfd_sample_field.argtypes = [P, C.c_int, C.c_int, C.c_float, P, P]
    lib.vfd_write_vtk.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_char_p]
    lib.vfd_write_raw_normalized.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_int]
    lib.vfd_write_csv.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_char_p]
    lib.vfd_check_wait_timeout.argtypes = [C.c_int, C.c_longlong]
    lib.vfd_stencil_window.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int, P, C.c_int]
    lib.vfd_synth_field_device.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_float, C.c_float, P,
                                           C.c_size_t, P]
    lib.vfd_server_create.argtypes = [C.c_int, C.c_size_t, C.c_int, C.c_int, C.POINTER(P)]
    lib.vfd_server_submit.argtypes = [P, C.POINTER(RequestDesc), C.POINTER(C.c_uint64)]
    lib.vfd_server_wait.argtypes = [P, C.c_uint64, C.c_double, C.POINTER(RequestInfo)]
    lib.vfd_server_drain.argtypes = [P, C.c_double]
    lib.vfd_server_get_stats.argtypes = [P, C.POINTER(ServerStats)]
    lib.vfd_server_clock.argtypes = [P]
    lib.vfd_server_clock.restype = C.c_double
    lib.vfd_server_destroy.argtypes = [P]
    lib.vfd_status_string.argtypes = [C.c_int]
    lib.vfd_status_string.restype = C.c_char_p
    lib.vfd_last_error.argtypes = [P]
    lib.vfd_last_error.restype = C.c_char_p
    lib.vfd_kernel_launch_count.argtypes = []
    lib.vfd_kernel_launch_count.restype = C.c_uint64
    lib.vfd_synth_field.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_float, C.c_float, P, C.c_size_t]
    lib.vfd_synth_sources.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int64, C.c_int64,
                                      C.c_double, C.c_double, P, P]
    for name in EXPORTED:
        if name not in ("vfd_status_string", "vfd_last_error", "vfd_kernel_launch_count",
                        "vfd_batch_last_error", "vfd_server_clock"):
            getattr(lib, name).restype = C.c_int
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = load()
    return _lib


def _check(status, world_ptr=None):
    if status != 0:
        msg = lib().vfd_last_error(world_ptr).decode()
        raise VfdError(status, msg)


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


def synth_field(seed, world, field, shape_zyx, lo=0.0, hi=1e-3):
    out = np.empty(shape_zyx, dtype=np.float32)
    _check(lib().vfd_synth_field(seed, world, field, lo, hi, _ptr(out), out.size))
    return out


def synth_sources(seed, world, field, n, n_voxels, mu=-6.0, sigma=1.0):
    idx = np.empty(n, dtype=np.int32)
    amt = np.empty(n, dtype=np.float32)
    _check(lib().vfd_synth_sources(seed, world, field, n, n_voxels, mu, sigma,
                                   _ptr(idx), _ptr(amt)))
    return idx, amt


def field_params(sigma, decay_rate, radius=None, baseline=0.0):
    """sigma: scalar or (sx, sy, sz); radius: None (ceil(3 sigma)) or int / triple."""
    p = FieldParams()
    s = [float(sigma)] * 3 if np.isscalar(sigma) else [float(v) for v in sigma]
    r = [0, 0, 0] if radius is None else ([int(radius)] * 3 if np.isscalar(radius)
                                         else [int(v) for v in radius])
    for a in range(3):
        p.sigma[a] = s[a]
        p.radius[a] = r[a]
    p.decay_rate = float(decay_rate)
    p.baseline = float(baseline)
    return p


def _world_desc(nx, ny, nz, params, pad_mode, epi_boundary, fft, method):
    """WorldDesc and the FieldParams array it points to (keep both alive)."""
    arr = (FieldParams * len(params))(*params)
    d = WorldDesc()
    d.nx, d.ny, d.nz, d.n_fields = nx, ny, nz, len(params)
    d.fields = C.cast(arr, C.POINTER(FieldParams))
    d.pad_mode, d.epi_boundary = pad_mode, epi_boundary
    for a in range(3):
        d.fft[a] = int(fft[a])
    d.method = int(method)
    return d, arr


def autotune(nx, ny, nz, params, pad_mode=PAD_ZERO, epi_boundary=0, fft=(0, 0, 0),
             device=0, reps=3):
    """Times every axis pass candidate for this shape on temporary worlds,
    caches the fastest (later worlds of the shape use it) and returns one
    dict per axis (x, y, z)."""
    d, _arr = _world_desc(nx, ny, nz, params, pad_mode, epi_boundary, fft, METHOD_SEPARABLE)
    out = (AxisTuning * 3)()
    _check(lib().vfd_autotune(C.byref(d), device, int(reps), out))
    return [out[a].as_dict() for a in range(3)]


def autotune_set(nx, ny, nz, params, tuning, pad_mode=PAD_ZERO, epi_boundary=0,
                 fft=(0, 0, 0), device=0):
    """Pins a per-axis choice (dicts as autotune returns) for this shape."""
    d, _arr = _world_desc(nx, ny, nz, params, pad_mode, epi_boundary, fft, METHOD_SEPARABLE)
    inv = {v: k for k, v in PASS_METHODS.items()}
    arr = (AxisTuning * 3)()
    for a in range(3):
        t = tuning[a]
        m = t.get("method", "register_fft")
        arr[a].method = inv.get(m, m)
        arr[a].ctas_per_sm = int(t.get("ctas_per_sm", 0))
        arr[a].fft_len = int(t.get("fft_len", 0))
        arr[a].radix_order = int(t.get("radix_order", 0))
        arr[a].variant = int(t.get("variant", -1))
        arr[a].ms = float(t.get("ms", 0.0))
    _check(lib().vfd_autotune_set(C.byref(d), device, arr))


def autotune_clear():
    _check(lib().vfd_autotune_clear())


class World:
    """One world of `n_fields` fields on an nx*ny*nz grid (x fastest)."""

    def __init__(self, nx, ny, nz, params, pad_mode=PAD_ZERO, epi_boundary=0,
                 fft=(0, 0, 0), device=0, method=METHOD_SEPARABLE):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.nf = len(params)
        d, self._params = _world_desc(nx, ny, nz, params, pad_mode, epi_boundary, fft, method)
        h = C.c_void_p()
        _check(lib().vfd_world_create(C.byref(d), device, C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            lib().vfd_world_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx)

    def fft_dims(self):
        a = (C.c_int * 3)()
        _check(lib().vfd_world_fft_dims(self._h, a), self._h)
        return tuple(a)

    def device_bytes(self):
        b = C.c_size_t()
        _check(lib().vfd_world_device_bytes(self._h, C.byref(b)), self._h)
        return b.value

    def tuning(self):
        """The pass each axis runs, one dict per axis (x, y, z)."""
        out = (AxisTuning * 3)()
        _check(lib().vfd_world_tuning(self._h, out), self._h)
        return [out[a].as_dict() for a in range(3)]

    def upload(self, field, arr, stream=None):
        a = np.ascontiguousarray(arr, dtype=np.float32)
        assert a.size == self.nx * self.ny * self.nz
        # pageable source: the call returns once the buffer has been staged
        _check(lib().vfd_upload_field(self._h, field, _ptr(a), stream), self._h)
        return a

    def download(self, field, out=None, stream=None):
        if out is None:
            out = np.empty(self.shape, dtype=np.float32)
        _check(lib().vfd_download_field(self._h, field, _ptr(out), stream), self._h)
        return out

    def device_ptr(self, field):
        p = C.c_void_p()
        _check(lib().vfd_field_device_ptr(self._h, field, C.byref(p)), self._h)
        return p.value

    def set_sources(self, field, idx, amt):
        i = np.ascontiguousarray(idx, dtype=np.int32)
        a = np.ascontiguousarray(amt, dtype=np.float32)
        assert i.size == a.size
        _check(lib().vfd_set_sources(self._h, field, _ptr(i), _ptr(a), i.size), self._h)

    def set_window(self, field, window, centre=None):
        """Dense real window (kd, kh, kw) as this field's kernel; centre (cz, cy, cx)."""
        w = np.ascontiguousarray(window, dtype=np.float32)
        kd, kh, kw = w.shape
        cz, cy, cx = centre if centre is not None else (kd // 2, kh // 2, kw // 2)
        _check(lib().vfd_set_window(self._h, field, _ptr(w), kw, kh, kd, cx, cy, cz), self._h)

    def set_spectrum(self, field, spec):
        """Stored kernel spectrum, complex (Fz, Fy, Fx/2 + 1) on the world's FFT grid
        (the reference's h_kernelspectrum[ic] layout)."""
        a = np.ascontiguousarray(spec, dtype=np.complex64)
        fz, fy, fxh = a.shape
        fx = self.fft_dims()[0]
        assert fxh == fx // 2 + 1
        _check(lib().vfd_set_spectrum(self._h, field, _ptr(a), fx, fy, fz), self._h)

    def set_boundary(self, epi_boundary, baselines=None):
        b = None
        if baselines is not None:
            b = np.ascontiguousarray(baselines, dtype=np.float32)
            assert b.size == self.nf
        _check(lib().vfd_set_boundary(self._h, int(epi_boundary), None if b is None else _ptr(b)), self._h)

    def tick(self, n_substeps=1, stream=None):
        _check(lib().vfd_tick(self._h, n_substeps, stream), self._h)

    def tick_update(self, decay, dchem_ptrs=None, n_substeps=1, stream=None):
        """One tick whose last substep stores p = d + decay * t, d = 0 (device
        pointers of the fields' dChem arrays, or None: d = 0)."""
        dec = np.ascontiguousarray(decay, dtype=np.float32)
        assert dec.size == self.nf
        dp = None
        if dchem_ptrs is not None:
            dp = (C.c_void_p * self.nf)(*[p or None for p in dchem_ptrs])
        _check(lib().vfd_tick_update(self._h, n_substeps, dp, _ptr(dec), stream), self._h)

    def diffuse_update_host(self, host_p, host_d, decay, n_substeps=1):
        """vfd_diffuse_update_host: host pChem in/out, host dChem in (zeroed)."""
        dec = np.ascontiguousarray(decay, dtype=np.float32)
        ps = (C.c_void_p * self.nf)(*[a.ctypes.data for a in host_p])
        ds = None if host_d is None else (C.c_void_p * self.nf)(*[a.ctypes.data for a in host_d])
        _check(lib().vfd_diffuse_update_host(self._h, ps, ds, _ptr(dec), n_substeps), self._h)

    def mass(self, stream=None):
        m = (Mass * self.nf)()
        _check(lib().vfd_read_mass(self._h, m, stream), self._h)
        return [x.as_dict() for x in m]

    def update_gradients(self, collagen=0, elastin=0, fib=0, neu=0, mac=0, stream=None):
        """Device pointers (ints, 0 = NULL) of nx*ny*nz float arrays."""
        _check(lib().vfd_update_gradients(self._h, collagen or None, elastin or None, fib or None,
                                          neu or None, mac or None, stream), self._h)

    def sample(self, field, stride, scale, out_ptr, stream=None):
        _check(lib().vfd_sample_field(self._h, field, stride, scale, out_ptr, stream), self._h)

    def set_profiling(self, enable=True):
        _check(lib().vfd_world_set_profiling(self._h, int(bool(enable))), self._h)

    def read_profile(self):
        """{kind: (ms_total, launches)} for kinds x, y, z, deposit since the last read."""
        ms = (C.c_double * 4)()
        n = (C.c_int64 * 4)()
        _check(lib().vfd_read_profile(self._h, ms, n), self._h)
        return {k: (ms[i], n[i]) for i, k in enumerate(("x", "y", "z", "deposit"))}

    def diffuse_host(self, host_in, host_out, n_substeps=1):
        ins = (C.c_void_p * self.nf)(*[a.ctypes.data for a in host_in])
        outs = (C.c_void_p * self.nf)(*[a.ctypes.data for a in host_out])
        _check(lib().vfd_diffuse_host(self._h, ins, outs, n_substeps), self._h)


class Batch:
    """Many worlds ticked together: one launch per axis pass per substep for
    all their fields, the tick captured in a CUDA graph (vfd_batch_*)."""

    def __init__(self, worlds):
        self.worlds = list(worlds)
        arr = (C.c_void_p * len(self.worlds))(*[w.handle.value for w in self.worlds])
        h = C.c_void_p()
        _check(lib().vfd_batch_create(arr, len(self.worlds), C.byref(h)))
        self._h = h

    def set_window(self, field, window, centre=None):
        """Dense real window (kd, kh, kw) as this field's kernel; centre (cz, cy, cx)."""
        w = np.ascontiguousarray(window, dtype=np.float32)
        kd, kh, kw = w.shape
        cz, cy, cx = centre if centre is not None else (kd // 2, kh // 2, kw // 2)
        _check(lib().vfd_set_window(self._h, field, _ptr(w), kw, kh, kd, cx, cy, cz), self._h)

    def tick(self, n_substeps=1, stream=None):
        st = lib().vfd_batch_tick(self._h, n_substeps, stream)
        if st != 0:
            raise VfdError(st, lib().vfd_batch_last_error(self._h).decode())

    def autotune(self, reps=3):
        """Times each axis pass candidate over the whole batch and keeps the
        fastest; returns one dict per axis (x, y, z)."""
        out = (AxisTuning * 3)()
        st = lib().vfd_batch_autotune(self._h, int(reps), out)
        if st != 0:
            raise VfdError(st, lib().vfd_batch_last_error(self._h).decode())
        return [out[a].as_dict() for a in range(3)]

    def close(self):
        if getattr(self, "_h", None):
            lib().vfd_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def write_vtk(field, path):
    """Legacy-VTK ASCII file of a (nz, ny, nx) float32 field."""
    a = np.ascontiguousarray(field, np.float32)
    nz, ny, nx = a.shape
    _check(lib().vfd_write_vtk(_ptr(a), nx, ny, nz, str(path).encode()))


def window_spectrum(window, fft, centre=None, device=0):
    """Unscaled R2C spectrum (complex64, (Fz, Fy, Fx/2 + 1)) of the window
    wrapped with its centre at index 0 on the fft = (Fx, Fy, Fz) grid."""
    w = np.ascontiguousarray(window, dtype=np.float32)
    kd, kh, kw = w.shape
    cz, cy, cx = centre if centre is not None else (kd // 2, kh // 2, kw // 2)
    fx, fy, fz = fft
    out = np.empty((fz, fy, fx // 2 + 1), np.complex64)
    _check(lib().vfd_window_spectrum(_ptr(w), kw, kh, kd, cx, cy, cz, fx, fy, fz, _ptr(out), device))
    return out


def write_raw_normalized(field, path, append=False):
    """8-bit normalised volume of a (nz, ny, nx) float32 field (the
    reference's writeNormalizedFloatRaw / ...Frames)."""
    a = np.ascontiguousarray(field, np.float32)
    nz, ny, nx = a.shape
    _check(lib().vfd_write_raw_normalized(_ptr(a), nx, ny, nz, str(path).encode(), int(bool(append))))


def write_csv(field, path):
    """Comma-separated values of a (nz, ny, nx) float32 field (writeFloatCsv)."""
    a = np.ascontiguousarray(field, np.float32)
    nz, ny, nx = a.shape
    _check(lib().vfd_write_csv(_ptr(a), nx, ny, nz, str(path).encode()))


def spectrum_window(spec, fx, window_shape, centre=None, device=0):
    """The window (kd, kh, kw) whose wrapped copy has the R2C spectrum spec
    (complex (Fz, Fy, Fx/2 + 1)) on the fx x Fy x Fz grid."""
    a = np.ascontiguousarray(spec, dtype=np.complex64)
    fz, fy, _ = a.shape
    kd, kh, kw = window_shape
    cz, cy, cx = centre if centre is not None else (kd // 2, kh // 2, kw // 2)
    out = np.empty((kd, kh, kw), np.float32)
    _check(lib().vfd_spectrum_window(_ptr(a), fx, fy, fz, kw, kh, kd, cx, cy, cz, _ptr(out), device))
    return out


def stencil_window(lam, gamma_dt, n_steps, R, device=0):
    """The reference's kernel window: 7-point stencil to the power n_steps,
    centred (2R+1)^3 window, computed on the device."""
    w = np.empty((2 * R + 1,) * 3, np.float32)
    _check(lib().vfd_stencil_window(lam, gamma_dt, n_steps, R, _ptr(w), device))
    return w


class Server:
    """Request loop with continuous batching (vfd_server_*)."""

    def __init__(self, hbm_budget_bytes, max_active, substeps_per_tick=1, device=0):
        h = C.c_void_p()
        _check(lib().vfd_server_create(device, int(hbm_budget_bytes), int(max_active),
                                       int(substeps_per_tick), C.byref(h)))
        self._h = h
        self._keep = {}

    def submit(self, grid, params, ticks, init=None, synth=None, sources=None, result=None,
               pad_mode=PAD_ZERO, epi_boundary=0):
        """grid (nx, ny, nz); params: list of FieldParams; init: list of host arrays or None;
        synth: (seed, world, lo, hi) when init is None; sources: list of (idx, amt) per field;
        result: list of host arrays receiving the final fields.  Returns the request id."""
        nx, ny, nz = grid
        nf = len(params)
        keep = []
        d = RequestDesc()
        d.nx, d.ny, d.nz, d.n_fields = nx, ny, nz, nf
        fp = (FieldParams * nf)(*params)
        keep.append(fp)
        d.fields = C.cast(fp, C.POINTER(FieldParams))
        d.pad_mode, d.epi_boundary, d.ticks = pad_mode, epi_boundary, int(ticks)
        if init is not None:
            arrs = [np.ascontiguousarray(a, np.float32) for a in init]
            keep.append(arrs)
            ip = (C.c_void_p * nf)(*[a.ctypes.data for a in arrs])
            keep.append(ip)
            d.init = C.cast(ip, C.POINTER(C.c_void_p))
        else:
            seed, world, lo, hi = synth
            d.synth_seed, d.synth_world, d.synth_lo, d.synth_hi = seed, world, lo, hi
        if sources is not None:
            idxs = [np.ascontiguousarray(i, np.int32) for i, _ in sources]
            amts = [np.ascontiguousarray(a, np.float32) for _, a in sources]
            ns = (C.c_int64 * nf)(*[i.size for i in idxs])
            pi = (C.c_void_p * nf)(*[i.ctypes.data for i in idxs])
            pa = (C.c_void_p * nf)(*[a.ctypes.data for a in amts])
            keep += [idxs, amts, ns, pi, pa]
            d.src_idx = C.cast(pi, C.POINTER(C.c_void_p))
            d.src_amt = C.cast(pa, C.POINTER(C.c_void_p))
            d.n_src = C.cast(ns, C.POINTER(C.c_int64))
        if result is not None:
            rp = (C.c_void_p * nf)(*[a.ctypes.data for a in result])
            keep += [result, rp]
            d.result = C.cast(rp, C.POINTER(C.c_void_p))
        m = (Mass * nf)()
        keep.append(m)
        d.mass = C.cast(m, C.POINTER(Mass))
        rid = C.c_uint64()
        _check(lib().vfd_server_submit(self._h, C.byref(d), C.byref(rid)))
        self._keep[rid.value] = (keep, m)
        return rid.value

    def wait(self, rid, timeout_s=600.0):
        info = RequestInfo()
        st = lib().vfd_server_wait(self._h, rid, timeout_s, C.byref(info))
        if st != 0:
            raise VfdError(st, f"request {rid}")
        keep, m = self._keep.pop(rid)
        out = {k: getattr(info, k) for k, _ in info._fields_}
        out["mass"] = [x.as_dict() for x in m]
        return out

    def drain(self, timeout_s=600.0):
        _check(lib().vfd_server_drain(self._h, timeout_s))

    def stats(self):
        st = ServerStats()
        _check(lib().vfd_server_get_stats(self._h, C.byref(st)))
        return st.as_dict()

    def clock(self):
        return lib().vfd_server_clock(self._h)

    def close(self):
        if getattr(self, "_h", None):
            lib().vfd_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def launch_count():
    return int(lib().vfd_kernel_launch_count())
