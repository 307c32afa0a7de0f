"""The steps either side of the path: attractant gradients (F1), the compute
part of sampleChem (F3), the field writers (F4: legacy VTK, the 8-bit
normalised raw volume and the CSV dump of output_utils.h)."""
import numpy as np
import pytest

import vfd

SCALES = [5e4, 1e4, 1e6, 100.0, 1e4, 1e5, 1e5, 1e4]


def test_vtk_writer_layout(tmp_path):
    f = (np.arange(4 * 3 * 2, dtype=np.float32) * 0.25).reshape(2, 3, 4)
    p = tmp_path / "f.vtk"
    vfd.write_vtk(f, p)
    lines = p.read_text().splitlines()
    assert lines[0] == "# vtk DataFile Version 2.0"
    assert lines[2] == "ASCII" and lines[3] == "DATASET STRUCTURED_POINTS"
    assert lines[4] == "DIMENSIONS 4 3 2" and lines[7] == "POINT_DATA 24"
    assert lines[8] == "SCALARS Color float 1" and lines[9] == "LOOKUP_TABLE default"
    rows = [list(map(float, ln.split())) for ln in lines[10:]]
    assert len(rows) == 6 and all(len(r) == 4 for r in rows)
    np.testing.assert_array_equal(np.array(rows, np.float32).reshape(2, 3, 4), f)


def test_raw_normalized_writer(tmp_path):
    """writeNormalizedFloatRaw (output_utils.h:86-103): 255 at or above 1, 0 at
    or below 0, else floor(256 v); the frames variant appends."""
    f = np.array([-1.0, 0.0, 0.001, 0.5, 0.999, 1.0, 2.0, 0.25, 0.75, 0.1, 0.3, 0.0039],
                 np.float32).reshape(2, 2, 3)
    p = tmp_path / "f.raw"
    vfd.write_raw_normalized(f, p)
    got = np.frombuffer(p.read_bytes(), np.uint8)
    v = f.ravel()
    ref = np.where(v >= 1.0, 255, np.where(v <= 0.0, 0, np.floor(v * np.float32(256.0)))).astype(np.uint8)
    np.testing.assert_array_equal(got, ref)
    vfd.write_raw_normalized(f, p, append=True)
    assert p.read_bytes() == ref.tobytes() * 2


def test_csv_writer_layout(tmp_path):
    """writeFloatCsv (output_utils.h:41-66): one line per row, each value
    followed by ", ", an empty line after each z plane."""
    f = (np.arange(3 * 2 * 2, dtype=np.float32) * 0.125).reshape(2, 2, 3)
    p = tmp_path / "f.csv"
    vfd.write_csv(f, p)
    lines = p.read_text().split("\n")
    assert lines[0] == "0, 0.125, 0.25, " and lines[1] == "0.375, 0.5, 0.625, " and lines[2] == ""
    assert lines[3] == "0.75, 0.875, 1, " and lines[5] == ""
    vals = [float(x) for ln in lines if ln for x in ln.split(", ") if x]
    np.testing.assert_array_equal(np.array(vals, np.float32), f.ravel())


@pytest.mark.gpu
def test_gradients_and_sampling(gpu):
    import torch
    nx, ny, nz = 37, 20, 14
    params = [vfd.field_params(1.0, 0.0) for _ in range(8)]
    with vfd.World(nx, ny, nz, params) as w:
        fields = [vfd.synth_field(2, 0, f, (nz, ny, nx)) for f in range(8)]
        for f in range(8):
            w.upload(f, fields[f])
        col = torch.rand(nz, ny, nx, device="cuda")
        ela = torch.rand(nz, ny, nx, device="cuda")
        fib, neu, mac = (torch.empty(nz, ny, nx, device="cuda") for _ in range(3))
        w.update_gradients(col.data_ptr(), ela.data_ptr(), fib.data_ptr(), neu.data_ptr(), mac.data_ptr())
        torch.cuda.synchronize()
        TNF, TGF, FGF, MMP8, IL1, IL6, IL8, IL10 = fields
        grad = IL1 + TNF + TGF + FGF + col.cpu().numpy()
        np.testing.assert_allclose(fib.cpu().numpy(), TGF)
        np.testing.assert_allclose(neu.cpu().numpy(), grad + IL6 + IL8, rtol=1e-6)
        np.testing.assert_allclose(mac.cpu().numpy(), grad + ela.cpu().numpy(), rtol=1e-6)
        for f in (0, 2, 3):
            out = torch.empty(nz // 3, ny // 3, nx // 3, device="cuda")
            w.sample(f, 3, SCALES[f], out.data_ptr())
            torch.cuda.synchronize()
            ref = np.minimum(fields[f][::3, ::3, ::3][:nz // 3, :ny // 3, :nx // 3] * np.float32(SCALES[f]), 1.0)
            np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-6)
