"""CPU tests of bench.py's pure helpers (no device): the byte count of the
canonical 5-sweep FFT convolution that the bench line reports beside its
own roofline."""
import importlib.util
import os

import pytest

from conftest import ROOT


def test_bench_fft_contract_bytes():
    # the canonical 5-sweep FFT-convolution byte count per voxel-step the
    # bench line reports beside its own roofline: 56.7 / 43.0 / 42.5 B for
    # the small, human-scale and large worlds
    from vfd import configs
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    got = [b.fft_contract_bytes(c) for c in (configs.CFG0, configs.CFG1, configs.CFG4)]
    assert got == pytest.approx([56.77, 42.99, 42.50], abs=0.02)
