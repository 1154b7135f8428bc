"""HDF5 grid output from device-resident grids: values held as CUDA tensors are staged through
two pinned buffers on a side stream (the copy of one chunk overlaps the write of the previous
one); the file must equal, byte for byte, the file written from the same values on the host."""
import numpy as np
import pytest

import distorteddustydiscanalysistoolkits_b200 as pb
from distorteddustydiscanalysistoolkits_b200 import gridio

pytestmark = pytest.mark.gpu


def test_device_grids_stream_to_the_same_file(tmp_path, monkeypatch):
    torch = pytest.importorskip("torch")
    g = np.random.default_rng(7)
    n = 100_003   # not a multiple of the chunk: a partial last chunk
    coor = tuple(g.normal(size=n) for _ in range(3))
    vals = [g.normal(size=n) for _ in range(3)]
    params = {"dtype": "Float64", "grid_type": "PointSamples", "note": "device"}
    host = pb.GridBundle([pb.PointSamples(v, coor) for v in vals], ["a", "b", "c"])
    pb.write_GridDataset(pb.GridDataset(host, params), tmp_path / "host.h5")
    dcoor = tuple(torch.from_numpy(c).cuda() for c in coor)
    dev = pb.GridBundle([pb.PointSamples(torch.from_numpy(v).cuda(), dcoor) for v in vals], ["a", "b", "c"])
    monkeypatch.setattr(gridio, "CHUNK_BYTES", 4096)   # many chunks through both staging buffers
    pb.write_GridDataset(pb.GridDataset(dev, params), tmp_path / "dev.h5")
    assert (tmp_path / "dev.h5").read_bytes() == (tmp_path / "host.h5").read_bytes()
    back = pb.read_GridDataset(tmp_path / "dev.h5")
    for a, v in zip(back.data.grids, vals):
        assert np.array_equal(a.grid, v)


def test_interpolated_bundle_written_from_the_device(tmp_path, backend):
    torch = pytest.importorskip("torch")
    from distorteddustydiscanalysistoolkits_b200 import synthetic
    p = synthetic.disc(20000, seed=5)
    cols = ("rho", "vz")
    inp = pb.InterpolationInput(p["x"].copy(), p["y"].copy(), p["z"].copy(), p["m"].copy(), p["h"].copy(),
                                p["rho"].copy(), tuple(p[c].copy() for c in cols), smoothed_kernel=pb.M4_spline)
    cat = pb.InterpolationCatalog(cols, scalars=cols)
    flat = pb.flatten(pb.Cartesian, synthetic.cartesian_box_grid(p, n=12))
    out = pb.PointSamples_interpolation(backend, flat, inp, cat, pb.itpGather, precision=pb.FP64)
    dev = pb.GridBundle([pb.PointSamples(torch.from_numpy(g.grid).cuda(), out.grids[0].coor) for g in out.grids],
                        out.names)
    units = {"umass": 1.0, "udist": 1.0, "utime": 1.0, "umagfd": 1.0}
    pb.write_GridBundle(dev, tmp_path / "interp.h5", code_units=units, operation_name="interp")
    back = pb.read_GridDataset(tmp_path / "interp.h5")
    assert list(back.data.names) == list(out.names)
    for a, b in zip(back.data.grids, out.grids):
        assert np.array_equal(a.grid.view(np.uint64), np.asarray(b.grid).view(np.uint64))
