"""CPU tests of the C ABI: libvfd.so loads, exports every function that
include/vfd.h declares, reports errors as status codes, and its input
generator is deterministic (pinned by the committed fixture)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import vfd
from conftest import ROOT, has_gpu

HEADER = os.path.join(ROOT, "include", "vfd.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(vfd_[a-z0-9_]+)\s*\(", src)))


def test_header_and_binding_agree():
    assert sorted(vfd.EXPORTED) == declared_functions()


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(vfd.LIB_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_status_strings():
    L = vfd.lib()
    for s in range(9):
        assert L.vfd_status_string(s).decode()
    assert L.vfd_status_string(99).decode() == "unknown status"


def test_create_rejects_bad_arguments_without_touching_a_device():
    L = vfd.lib()
    h = C.c_void_p()
    assert L.vfd_world_create(None, 0, C.byref(h)) == 1
    d = vfd.WorldDesc()
    d.nx, d.ny, d.nz, d.n_fields = 0, 4, 4, 1
    p = (vfd.FieldParams * 1)(vfd.field_params(1.0, 0.1))
    d.fields = C.cast(p, C.POINTER(vfd.FieldParams))
    assert L.vfd_world_create(C.byref(d), 0, C.byref(h)) == 1
    assert "dims" in L.vfd_last_error(None).decode()
    d.nx = 4
    d.pad_mode = 7
    assert L.vfd_world_create(C.byref(d), 0, C.byref(h)) == 1
    assert L.vfd_world_destroy(None) == 1
    assert L.vfd_tick(None, 1, None) == 1
    assert L.vfd_set_spectrum(None, 0, None, 8, 8, 8) == 1
    assert L.vfd_set_boundary(None, 0, None) == 1
    assert L.vfd_tick_update(None, 1, None, None, None) == 1
    assert L.vfd_diffuse_update_host(None, None, None, None, 1) == 1


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_create_without_device_reports_no_device():
    with pytest.raises(vfd.VfdError) as e:
        vfd.World(8, 8, 8, [vfd.field_params(1.0, 0.1)])
    assert e.value.status == 8


def test_generator_deterministic_and_in_range():
    a = vfd.synth_field(0, 0, 3, (4, 5, 6))
    b = vfd.synth_field(0, 0, 3, (4, 5, 6))
    c = vfd.synth_field(0, 0, 4, (4, 5, 6))
    np.testing.assert_array_equal(a, b)
    assert not np.array_equal(a, c)
    assert a.min() >= 0.0 and a.max() < 1e-3
    idx, amt = vfd.synth_sources(0, 0, 1, 10000, 1000)
    assert idx.min() >= 0 and idx.max() < 1000
    # lognormal(-6, 1): median exp(-6)
    assert abs(np.log(np.median(amt)) + 6.0) < 0.05
    assert abs(np.std(np.log(amt)) - 1.0) < 0.05


def test_generator_matches_committed_fixture():
    g = np.load(os.path.join(ROOT, "tests", "golden", "cfg0_oracle.npz"))
    from vfd import configs
    c = configs.CFG0
    nx, ny, nz = c["grid"]
    for f in range(8):
        u = vfd.synth_field(c["seed"], 0, f, (nz, ny, nx))
        idx, amt = vfd.synth_sources(c["seed"], 0, f, c["n_sources"], nx * ny * nz)
        np.testing.assert_array_equal(u.ravel()[:16], g["gen_u"][f])
        np.testing.assert_array_equal(idx[:16], g["gen_idx"][f])
        np.testing.assert_array_equal(amt[:16], g["gen_amt"][f])


def test_header_is_plain_c(tmp_path):
    # the boundary is a C ABI: the header compiles as strict C99 and every
    # struct a binding mirrors has the size the ctypes mirror assumes
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "h.c"
    src.write_text('#include "vfd.h"\n#include <stdio.h>\n'
                   'int main(void) { printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(vfd_field_params), '
                   'sizeof(vfd_world_desc), sizeof(vfd_mass), sizeof(vfd_axis_tuning), '
                   'sizeof(vfd_request_desc), sizeof(vfd_request_info), sizeof(vfd_server_stats)); '
                   'return 0; }\n')
    exe = tmp_path / "h"
    subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                    "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    sizes = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True,
                                            text=True).stdout.split()]
    assert sizes == [C.sizeof(vfd.FieldParams), C.sizeof(vfd.WorldDesc), C.sizeof(vfd.Mass),
                     C.sizeof(vfd.AxisTuning), C.sizeof(vfd.RequestDesc), C.sizeof(vfd.RequestInfo),
                     C.sizeof(vfd.ServerStats)]
