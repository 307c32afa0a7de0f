"""Times the reference's own GPU diffusion (its convolutionFFT.cu kernels +
cuFFT, built into oracle/_ref/libref_replay.so) beside this library on the
human-scale world (512x256x384, one field, Gaussian sigma 1.95, radius 6).

TEST/MEASUREMENT INFRASTRUCTURE ONLY (run on a B200):
    python oracle/ref_timing.py [--iters 5]
Prints one JSON line: voxel-steps/s of one field-substep for
  * the reference path with its power-of-two FFT grid (snapTransformSize,
    Diffusion.cu:39-70) -- kernels only, and as called each tick (plans and
    buffers re-created per call, Diffuser.cpp:273-274, Diffusion.cu:1686-1687);
  * the same reference kernels on this library's 7-smooth grid;
  * this library's separable path (one field, one substep, resident).
"""
import argparse
import ctypes as C
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "vf-version_7_3_b200"))

import oracle  # noqa: E402


def pow2_snap(n):
    n16 = (n + 15) // 16 * 16
    p = 1
    while p < n16:
        p *= 2
    return p


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--iters", type=int, default=5)
    args = ap.parse_args()
    import torch

    import vfd
    nx, ny, nz = 512, 256, 384
    sigma = 1.3 * 1.5
    r = int(np.ceil(3 * sigma))
    t = oracle.gauss_taps(sigma, r)
    win = np.ascontiguousarray(np.einsum("z,y,x->zyx", t, t, t).astype(np.float32))
    k = 2 * r + 1
    L = C.CDLL(oracle.REF_REPLAY)
    f = L.ref_replay_time
    f.argtypes = [C.c_int] * 6 + [C.c_void_p] + [C.c_int] * 7 + [C.c_float, C.c_int, C.c_void_p]
    f.restype = C.c_int
    V = nx * ny * nz
    res = {"workload": "one field of the 512x256x384 world, one substep (fftDiffuse3D)", "voxels": V}
    grids = {"reference_pow2": (pow2_snap(nx + k - 1), pow2_snap(ny + k - 1), pow2_snap(nz + k - 1))}
    with vfd.World(nx, ny, nz, [vfd.field_params(sigma, 0.0)]) as w:
        grids["library_7smooth"] = tuple(vfd.World(nx, ny, nz, [vfd.field_params(sigma, 0.0)],
                                                   method=vfd.METHOD_FFT3D).fft_dims())
        w.upload(0, np.zeros((nz, ny, nx), np.float32))
        w.tick(1)
        st = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.iters):
            w.tick(1, stream=st.cuda_stream)
        e1.record(st)
        torch.cuda.synchronize()
        res["library_separable"] = {"ms": e0.elapsed_time(e1) / args.iters}
    for name, (fx, fy, fz) in grids.items():
        ms = (C.c_double * 2)()
        rc = f(nz, ny, nx, fz, fy, fx, win.ctypes.data, k, k, k, r, r, r, nx, 0.0, args.iters, ms)
        if rc != 0:
            res[name] = {"error": L.ref_replay_error().decode() if hasattr(L, "ref_replay_error") else rc}
            continue
        res[name] = {"fft": [fx, fy, fz], "ms_kernels": ms[0], "ms_as_called": ms[1]}
    for key, v in res.items():
        if isinstance(v, dict) and "ms" in v:
            v["voxel_steps_per_s"] = V / (v["ms"] / 1e3)
        if isinstance(v, dict) and "ms_kernels" in v:
            v["voxel_steps_per_s_kernels"] = V / (v["ms_kernels"] / 1e3)
            v["voxel_steps_per_s_as_called"] = V / (v["ms_as_called"] / 1e3)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
