"""CPU tests of the tuning cache's host side (vfd_autotune_set /
vfd_autotune_clear): a stored choice is validated against the shape before
it is cached, and nothing here touches a device."""
import pytest

import vfd

GRID = (96, 70, 33)


def params(sigmas=(0.6, 1.3)):
    return [vfd.field_params(s, 0.05) for s in sigmas]


@pytest.fixture(autouse=True)
def clean_cache():
    vfd.autotune_clear()
    yield
    vfd.autotune_clear()


def test_valid_choices_are_stored():
    nx, ny, nz = GRID
    vfd.autotune_set(nx, ny, nz, params(), [{"method": "register_fft"}] * 3)
    vfd.autotune_set(nx, ny, nz, params(), [{"method": "overlap_save", "ctas_per_sm": 4}] * 3)
    # full line: 7-smooth lengths >= n + r (radius 4): x 100, y 75, z 40; both radix orders
    vfd.autotune_set(nx, ny, nz, params(),
                     [{"method": "full_line", "fft_len": 100, "radix_order": 1},
                      {"method": "full_line", "fft_len": 75},
                      {"method": "full_line", "fft_len": 0, "variant": 2}])


@pytest.mark.parametrize("bad", [
    {"method": "full_line", "fft_len": 97},                 # shorter than n + r = 100
    {"method": "full_line", "fft_len": 101},                # prime: no 7-smooth plan
    {"method": "full_line", "radix_order": 2},              # two radix orders
    {"method": "full_line", "variant": 99},                 # no such kernel variant
    {"method": "overlap_save", "ctas_per_sm": 5},           # 3 or 4 CTAs per SM
    {"method": 7},                                          # unknown pass
])
def test_invalid_choices_are_rejected(bad):
    nx, ny, nz = GRID
    with pytest.raises(vfd.VfdError) as e:
        vfd.autotune_set(nx, ny, nz, params(), [bad, {"method": "register_fft"}, {"method": "register_fft"}])
    assert e.value.status == 1  # VFD_ERR_INVALID_ARG


def test_general_methods_are_not_tuned():
    nx, ny, nz = GRID
    L = vfd.lib()
    import ctypes as C
    d, arr = vfd._world_desc(nx, ny, nz, params(), vfd.PAD_ZERO, 0, (0, 0, 0), vfd.METHOD_FFT3D)
    t = (vfd.AxisTuning * 3)()
    assert L.vfd_autotune_set(C.byref(d), 0, t) == 7  # VFD_ERR_NOT_SUPPORTED
    assert L.vfd_autotune_set(None, 0, t) == 1
    assert L.vfd_world_tuning(None, t) == 1

