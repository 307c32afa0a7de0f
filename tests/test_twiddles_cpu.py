"""CPU test of the register FFT engine's compile-time twiddles.

The small DFTs of the general path (csrc/vfd_tpr.cuh) take w_N^e as FP32
immediates whose values the compiler computes in FP64 (tpr_trig2pi: integer
quadrant reduction, then Taylor series).  This compiles that header's host
side with nvcc (no GPU needed) and checks every cos / sin of 2 pi e / n for
n <= 64 against numpy's FP64 values: within 2e-15, and identical once
rounded to FP32 (the immediates the kernels use).
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import PKG

NMAX = 64

SRC = r"""
#include <cstdio>
#include "vfd_tpr.cuh"
int main()
{
    for (int n = 2; n <= %d; ++n)
        for (int e = 0; e < n; ++e)
            std::printf("%%d %%d %%.17g %%.17g\n", n, e, vfd::tpr_trig2pi(e, n, false), vfd::tpr_trig2pi(e, n, true));
    return 0;
}
""" % NMAX


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not on PATH")
def test_immediate_twiddles_match_fp64(tmp_path):
    src = tmp_path / "tw.cu"
    exe = tmp_path / "tw"
    src.write_text(SRC)
    subprocess.run(["nvcc", "-std=c++17", "-Wno-deprecated-gpu-targets", "-I", os.path.join(PKG, "csrc"),
                    str(src), "-o", str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    a = np.array(out, dtype=np.float64).reshape(-1, 4)
    n, e, c, s = a[:, 0], a[:, 1], a[:, 2], a[:, 3]
    assert len(a) == sum(range(2, NMAX + 1))
    ang = 2.0 * np.pi * e / n
    rc, rs = np.cos(ang), np.sin(ang)
    # the exact zeros of the quarter turns are exact here; numpy's are ~1e-16
    rc[np.abs(rc) < 1e-15] = 0.0
    rs[np.abs(rs) < 1e-15] = 0.0
    # numpy evaluates at the FP64-rounded angle (error up to ~1e-15 near the zeros)
    assert np.max(np.abs(c - rc)) < 2e-15
    assert np.max(np.abs(s - rs)) < 2e-15
    assert np.array_equal(c.astype(np.float32), rc.astype(np.float32))
    assert np.array_equal(s.astype(np.float32), rs.astype(np.float32))
    # quarter turns exact
    q = (4 * e) % n == 0
    assert np.all(np.isin(c[q], [-1.0, 0.0, 1.0])) and np.all(np.isin(s[q], [-1.0, 0.0, 1.0]))
