"""Phantom dump ingest and ParticleIO's build_input on the host (no GPU).

read_phantom (ParticleIO.jl/src/julia/IO/phantomIO/read_phantom.jl) on dumps written by
tests/golden/phantom_dump.py: both default integer and real sizes, typed header blocks with
repeated names, typed particle arrays, the sinks block, inactive particles, particle-type
separation and the error paths; add_rho! (add_quantities.jl:308-345) and build_input
(build_input.jl:44-160) with mass from a column and from params, and its missing-column error.
"""
import numpy as np
import pytest

import distorteddustydiscanalysistoolkits_b200 as pb
from distorteddustydiscanalysistoolkits_b200 import phantom
from golden.phantom_dump import write_dump


def _disc_dump(path, def_int=np.int32, def_real=np.float64, n_gas=600, n_dust=200, seed=3, sinks=True):
    g = np.random.default_rng(seed)
    n = n_gas + n_dust
    x, y = g.uniform(-50, 50, (2, n))
    z = g.normal(0, 2, n)
    h = g.uniform(0.5, 3.0, n).astype(np.float32)
    h[[5, 17]] = -h[[5, 17]]   # accreted particles: negative h
    v = g.normal(0, 1, (3, n)).astype(np.float32)
    itype = np.array([1] * n_gas + [2] * n_dust, np.int8)
    blocks = [(n, [("x", x, "def_real"), ("y", y, "def_real"), ("z", z, "def_real"), ("h", h, "float32"),
                   ("vx", v[0], "float32"), ("vy", v[1], "float32"), ("vz", v[2], "float32"),
                   ("itype", itype, "int8")])]
    if sinks:
        blocks.append((2, [("x", [0.0, 30.0], "def_real"), ("y", [0.0, -5.0], "def_real"),
                           ("z", [0.0, 0.1], "def_real"), ("m", [1.0, 1e-3], "def_real"),
                           ("h", [1.0, 0.5], "def_real")]))
    header = [("nparttot", n, "def_int"), ("ntypes", 2, "def_int"), ("isink", 1, "int32"),
              ("massoftype", 1e-6, "def_real"), ("massoftype", 1e-8, "def_real"), ("massoftype", 0.0, "def_real"),
              ("time", 12.5, "def_real"), ("hfact", 1.2, "def_real"), ("udist", 1.496e13, "float64")]
    write_dump(str(path), blocks, header, def_int=def_int, def_real=def_real)
    return dict(x=x, y=y, z=z, h=h, vx=v[0], vy=v[1], vz=v[2], itype=itype)


@pytest.mark.parametrize("def_int,def_real", [(np.int32, np.float64), (np.int32, np.float32)])
def test_read_phantom_sinks_and_types(tmp_path, def_int, def_real):
    src = _disc_dump(tmp_path / "d_00000", def_int, def_real)
    df, sinks = phantom.read_phantom(str(tmp_path / "d_00000"))
    keep = src["h"] > 0
    assert df.npart == keep.sum() == len(src["h"]) - 2
    assert np.array_equal(df["x"], np.asarray(src["x"], def_real)[keep])
    assert df["x"].dtype == np.dtype(def_real) and df["h"].dtype == np.float32 and df["itype"].dtype == np.int8
    assert np.array_equal(df["vz"], src["vz"][keep])
    p = df.params
    assert p["massoftype"] == pytest.approx(1e-6) and p["massoftype_2"] == pytest.approx(1e-8)
    assert "massoftype_3" in p and p["hfact"] == pytest.approx(1.2) and p["udist"] == 1.496e13
    assert p["nparttot"] == 800 and p["isink"] == 1 and p["default_Int"] == np.dtype(def_int).name
    assert p["file_identifier"] == "FT:Phantom test dump" and p["mass"] is None
    assert sinks.npart == 2 and np.array_equal(sinks["m"], np.array([1.0, 1e-3], def_real))


def test_read_phantom_separate_all_and_none(tmp_path):
    src = _disc_dump(tmp_path / "d_00001")
    gas, dust, sinks = phantom.read_phantom(str(tmp_path / "d_00001"), separate_types="all")
    keep = src["h"] > 0
    assert gas.npart == (keep & (src["itype"] == 1)).sum() and dust.npart == (keep & (src["itype"] == 2)).sum()
    assert gas.params["mass"] == pytest.approx(1e-6) and dust.params["mass"] == pytest.approx(1e-8)
    assert gas.params["itype"] == 1 and dust.params["itype"] == 2 and sinks.npart == 2
    (one,) = phantom.read_phantom(str(tmp_path / "d_00001"), separate_types=None)
    assert one.npart == keep.sum() + 2
    assert np.isnan(one["vx"][-2:]).all() and np.array_equal(one["m"][-2:], [1.0, 1e-3])
    (allp,) = phantom.read_phantom(str(tmp_path / "d_00001"), separate_types=None, ignore_inactive=False)
    assert allp.npart == 802
    _disc_dump(tmp_path / "nosink", sinks=False)
    (only,) = phantom.read_phantom(str(tmp_path / "nosink"))
    assert only.npart == keep.sum()


def test_read_phantom_eight_byte_default_int_is_refused_as_in_the_reference(tmp_path):
    # the capture check reads the first integer as int*4 first, which matches the low half of a
    # little-endian int*8 60769; the following real then fails the check (read_phantom.jl:40-62)
    _disc_dump(tmp_path / "i8", def_int=np.int64, def_real=np.float64)
    with pytest.raises(pb.ArgumentError, match="CapturePattern"):
        phantom.read_phantom(str(tmp_path / "i8"))


def test_read_phantom_errors(tmp_path):
    bad = tmp_path / "bad"
    bad.write_bytes(b"\x14\x00\x00\x00" + b"\x00" * 40)
    with pytest.raises(pb.ArgumentError, match="CapturePattern"):
        phantom.read_phantom(str(bad))
    g = np.random.default_rng(0)
    write_dump(str(tmp_path / "tags"), [(3, [("x", g.random(3), "def_real")])], [], swap_tail=True)
    with pytest.raises(pb.ArgumentError, match="tags"):
        phantom.read_phantom(str(tmp_path / "tags"))
    raw = (tmp_path / "tags").read_bytes()
    (tmp_path / "short").write_bytes(raw[:60])
    with pytest.raises(pb.ArgumentError):
        phantom.read_phantom(str(tmp_path / "short"))


def test_add_rho_and_build_input(tmp_path):
    _disc_dump(tmp_path / "d")
    gas, dust, sinks = phantom.read_phantom(str(tmp_path / "d"), separate_types="all")
    phantom.add_rho(gas)
    m, hf = 1e-6, 1.2
    h = gas["h"].astype(np.float64)
    exp = (m * hf * hf * hf) * ((1.0 / h) * (1.0 / h) * (1.0 / h))
    assert np.array_equal(gas["rho"], exp)
    with pytest.raises(KeyError):
        phantom.add_rho(sinks)   # no per-type mass in the sinks frame
    inp, cat = phantom.build_input(gas, phantom.MassFromParams("mass"), scalars=("rho",), divergences=("v",))
    assert cat.ordered_names[0] == "rho" and cat.L == 2
    assert np.array_equal(inp.m, np.full(gas.npart, 1e-6)) and np.array_equal(inp.h, h)
    assert [q.dtype for q in inp.quant] == [np.float64] * 4
    assert np.array_equal(inp.quant[1], gas["vx"].astype(np.float64))
    gas["mcol"] = np.full(gas.npart, 2e-6, np.float32)
    inp2, _ = phantom.build_input(gas, phantom.MassFromColumn("mcol"), scalars=("vz",))
    assert np.array_equal(inp2.m, np.full(gas.npart, np.float64(np.float32(2e-6))))
    with pytest.raises(pb.ArgumentError, match="Missing columns"):
        phantom.build_input(gas, phantom.MassFromParams("mass"), scalars=("T",))
    with pytest.raises(pb.ArgumentError, match="Missing parameter"):
        phantom.build_input(gas, phantom.MassFromParams("nope"), scalars=("rho",))
