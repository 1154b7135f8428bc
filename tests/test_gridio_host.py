"""HDF5 grid output (write_GridDataset / write_GridBundle, write_grids.jl:29-215) and its reader
(read_grids.jl:29-80) on the host: the lookup3 checksum against its published test values, round
trips of point and structured bundles (values bit for bit, names, metadata, HDF5 dimensions of
column-major grids), the file's structural invariants, checksum verification and the reference's
error cases."""
import struct

import numpy as np
import pytest

import distorteddustydiscanalysistoolkits_b200 as pb
from distorteddustydiscanalysistoolkits_b200 import gridio

UNITS = {"umass": 1.989e33, "udist": 1.496e13, "utime": 5.0226e6, "umagfd": 1.0}


def test_lookup3_published_values():
    # Bob Jenkins' lookup3.c driver values for hashlittle
    assert gridio.lookup3(b"") == 0xDEADBEEF
    assert gridio.lookup3(b"", 0xDEADBEEF) == 0xBD5B7DDE
    assert gridio.lookup3(b"Four score and seven years ago", 0) == 0x17770551
    assert gridio.lookup3(b"Four score and seven years ago", 1) == 0xCD628161


def _points(n=1000, seed=0):
    g = np.random.default_rng(seed)
    coor = tuple(g.normal(size=n) for _ in range(3))
    grids = [pb.PointSamples(g.normal(size=n), coor) for _ in range(4)]
    return pb.GridBundle(grids, ["rho", "vx", "vy", "vz"])


def test_point_bundle_round_trip(tmp_path):
    gb = _points()
    path = tmp_path / "points.h5"
    pb.write_GridBundle(gb, path, code_units=UNITS, operation_name="test", params={"note": "x", "n": 3, "on": True})
    gd = pb.read_GridDataset(path)
    assert list(gd.data.names) == ["rho", "vx", "vy", "vz"]
    for a, b in zip(gd.data.grids, gb.grids):
        assert np.array_equal(a.grid.view(np.uint64), b.grid.view(np.uint64))
    for d in range(3):
        assert np.array_equal(gd.data.grids[0].coor[d], gb.grids[0].coor[d])
        assert gd.data.grids[3].coor[d] is gd.data.grids[0].coor[d]
    p = gd.params
    assert p["schema_name"] == "GridDataset" and p["schema_id"] == "GridDataset.v1"
    assert p["dtype"] == "Float64" and p["grid_type"] == "PointSamples"
    assert p["umass"] == UNITS["umass"] and p["umagfd"] == 1.0
    assert p["note"] == "x" and p["n"] == 3 and p["on"] is True
    assert p["file_identifier"].startswith("FT:Partia:%s (test): " % pb.__version__)


def test_structured_bundle_round_trip_and_column_major_dims(tmp_path):
    axes = (np.linspace(0, 1, 5), np.linspace(-1, 1, 7), np.linspace(2, 3, 3))
    g = np.random.default_rng(1)
    grids = [pb.StructuredGrid(g.normal(size=(5, 7, 3)), axes) for _ in range(2)]
    gb = pb.GridBundle(grids, ["a", "b"])
    path = tmp_path / "struct.h5"
    pb.write_GridBundle(gb, path, code_units=UNITS)
    gd = pb.read_GridDataset(path)
    assert gd.params["grid_type"] == "StructuredGrid"
    for a, b in zip(gd.data.grids, grids):
        assert a.size == (5, 7, 3) and np.array_equal(a.grid, b.grid)
    # HDF5 dimensions are the Julia size reversed, over the same column-major bytes
    tree = gridio._open_tree(memoryview(path.read_bytes()))
    raw = tree["data"]["grids"]["1"]
    assert raw.shape == (3, 7, 5)
    assert np.array_equal(raw.reshape(-1), grids[0].grid.reshape(-1, order="F"))


def test_file_structure(tmp_path):
    path = tmp_path / "s.h5"
    pb.write_GridBundle(_points(37), path, code_units=UNITS)
    raw = path.read_bytes()
    assert raw[:8] == b"\x89HDF\r\n\x1a\n" and raw[8] == 2 and raw[9] == 8 and raw[10] == 8
    base, ext, eof, root = struct.unpack_from("<QQQQ", raw, 12)
    assert base == 0 and ext == gridio.UNDEF and eof == len(raw) and root == 48
    # every dataset's values start on an 8-byte boundary inside the file
    gd = pb.GridDataset(_points(37), {"dtype": "Float64", "grid_type": "PointSamples"})
    root_node = gridio._Group()
    d = root_node.add("v", gridio._vector(gd.data.grids[0].grid))
    nodes, end = gridio._layout(root_node)
    assert d.data_addr % 8 == 0 and end == d.data_addr + 8 * 37


def test_checksums_are_verified(tmp_path):
    path = tmp_path / "c.h5"
    pb.write_GridBundle(_points(10), path, code_units=UNITS)
    raw = bytearray(path.read_bytes())
    bad = tmp_path / "bad.h5"
    raw[60] ^= 0xFF   # inside the root group's object header
    bad.write_bytes(bytes(raw))
    with pytest.raises(pb.ArgumentError, match="checksum"):
        pb.read_GridDataset(bad)
    raw[60] ^= 0xFF
    raw[20] ^= 0x01   # superblock
    bad.write_bytes(bytes(raw))
    with pytest.raises(pb.ArgumentError, match="checksum"):
        pb.read_GridDataset(bad)


def test_reference_errors(tmp_path):
    gb = _points(10)
    with pytest.raises(pb.ArgumentError, match="code_units missing required keys"):
        pb.write_GridBundle(gb, tmp_path / "e.h5", code_units={"umass": 1.0})
    other = pb.GridBundle([gb.grids[0], pb.PointSamples(gb.grids[1].grid, tuple(c.copy() for c in gb.grids[1].coor))],
                          ["a", "b"])
    with pytest.raises(pb.ArgumentError, match="not shared: grid=2 dim=1"):
        pb.write_GridDataset(pb.GridDataset(other, {}), tmp_path / "e.h5")
    with pytest.raises(pb.ArgumentError, match="String, Int, Bool or Float64"):
        pb.write_GridDataset(pb.GridDataset(gb, {"bad": [1, 2]}), tmp_path / "e.h5")
    lines = pb.GridBundle([pb.LineSamples(np.zeros(2), (np.zeros(2),) * 3, (np.ones(2),) * 3)], ["c"])
    with pytest.raises(pb.ArgumentError, match="no method"):
        pb.write_GridBundle(lines, tmp_path / "e.h5", code_units=UNITS)
    pb.write_GridDataset(pb.GridDataset(gb, {"grid_type": "PointSamples"}), tmp_path / "nodtype.h5")
    with pytest.raises(pb.ArgumentError, match="params missing :dtype"):
        pb.read_GridDataset(tmp_path / "nodtype.h5")


def test_two_dimensional_grids_and_value_types(tmp_path):
    g = np.random.default_rng(3)
    coor = (g.normal(size=50), g.normal(size=50))
    pts = pb.GridBundle([pb.PointSamples(g.normal(size=50), coor)], ["Σρ"])   # a UTF-8 name
    params = {"empty": "", "big": 2 ** 62, "neg": -7, "tiny": 5e-324, "off": False}
    pb.write_GridDataset(pb.GridDataset(pts, dict(params, dtype="Float64", grid_type="PointSamples")),
                         tmp_path / "p2.h5")
    gd = pb.read_GridDataset(tmp_path / "p2.h5")
    assert list(gd.data.names) == ["Σρ"] and len(gd.data.grids[0].coor) == 2
    for k, v in params.items():
        assert gd.params[k] == v and type(gd.params[k]) is type(v)
    tree = gridio._open_tree(memoryview((tmp_path / "p2.h5").read_bytes()))
    assert list(tree["data"]["coord"].keys()) == ["x", "y"]
    axes = (np.linspace(0, 1, 4), np.linspace(0, 2, 6))
    st = pb.GridBundle([pb.StructuredGrid(g.normal(size=(4, 6)), axes)], ["s"])
    pb.write_GridBundle(st, tmp_path / "s2.h5", code_units=UNITS)
    back = pb.read_GridDataset(tmp_path / "s2.h5")
    assert back.data.grids[0].size == (4, 6) and np.array_equal(back.data.grids[0].grid, st.grids[0].grid)
    assert back.params["file_identifier"].startswith("FT:Partia:%s (CommonOutput): " % pb.__version__)
