"""build_input on the device from a Phantom dump (pb_column_to_f64, pb_fill_f64,
pb_density_from_h) against ParticleIO's host build_input + add_rho!: every column bit for bit,
and the interpolation of the device-built input equal to the host-built one's and to the
oracle's (FP64)."""
import numpy as np
import pytest

import distorteddustydiscanalysistoolkits_b200 as pb
from distorteddustydiscanalysistoolkits_b200 import phantom, synthetic
from golden.phantom_dump import write_dump
import oracle

pytestmark = pytest.mark.gpu


def _dump_from_disc(path, n=30000, seed=12):
    p = synthetic.disc(n, seed=seed)
    hfact = 1.2
    # h as a dump stores it (real*4); the columns a Phantom gas dump carries
    h32 = p["h"].astype(np.float32)
    blocks = [(n, [("x", p["x"], "def_real"), ("y", p["y"], "def_real"), ("z", p["z"], "def_real"),
                   ("h", h32, "float32"), ("vx", p["vx"].astype(np.float32), "float32"),
                   ("vy", p["vy"].astype(np.float32), "float32"), ("vz", p["vz"].astype(np.float32), "float32"),
                   ("itype", np.ones(n, np.int8), "int8")])]
    header = [("nparttot", n, "def_int"), ("massoftype", 1e-6, "def_real"), ("hfact", hfact, "def_real")]
    write_dump(str(path), blocks, header)
    (df,) = phantom.read_phantom(str(path), separate_types=None)
    df.params["mass"] = df.params["massoftype"]
    return df


def test_build_input_device_matches_host(backend, tmp_path):
    torch = pytest.importorskip("torch")
    df = _dump_from_disc(tmp_path / "disc_00000")
    kw = dict(scalars=("rho", "vz"), gradients=("rho",), divergences=("v",), curls=("v",),
              smoothed_kernel=pb.M4_spline)
    dinp, dcat = phantom.build_input_device(df, phantom.MassFromParams("mass"), backend, rho_from_h=True, **kw)
    hdf = phantom.add_rho(phantom.ParticleDataFrame(df.columns, df.params))
    hinp, hcat = phantom.build_input(hdf, phantom.MassFromParams("mass"), **kw)
    assert dcat.ordered_names == hcat.ordered_names
    for a, b in [(dinp.coord[k], hinp.coord[k]) for k in range(3)] + [(dinp.m, hinp.m), (dinp.h, hinp.h),
                                                                      (dinp.rho, hinp.rho)]:
        assert a.dtype == torch.float64 and np.array_equal(a.cpu().numpy(), b)
    for a, b in zip(dinp.quant, hinp.quant):
        assert np.array_equal(a.cpu().numpy(), b)
    # mass from a float32 column, widened on the device
    df["mcol"] = np.full(df.npart, 2e-6, np.float32)
    d2, _ = phantom.build_input_device(df, phantom.MassFromColumn("mcol"), backend, scalars=("vz",), rho_from_h=True)
    assert np.array_equal(d2.m.cpu().numpy(), df["mcol"].astype(np.float64))
    # the same interpolation from either input; FP64 equals the oracle bit for bit
    flat = pb.flatten(pb.Cartesian, synthetic.cartesian_box_grid(
        {"x": hinp.coord[0], "y": hinp.coord[1], "z": hinp.coord[2]}, n=10))
    ref = oracle.OracleLBVH(hinp.coord[0], hinp.coord[1], hinp.coord[2], hinp.h).attach(
        hinp.m, hinp.rho, list(hinp.quant), "M4_spline").interp_points(hcat.oracle_dict(), *flat.coor,
                                                                      strategy="itpSymmetric")
    hout = pb.PointSamples_interpolation(backend, flat, hinp, hcat, pb.itpSymmetric, precision=pb.FP64)
    dout = pb.PointSamples_interpolation(backend, flat, dinp, dcat, pb.itpSymmetric, precision=pb.FP64)
    got_h = np.stack([g.grid for g in hout.grids])
    got_d = np.stack([g.grid for g in dout.grids])
    ok = ~np.isnan(ref)
    assert np.array_equal(np.isnan(got_d), ~ok) and np.array_equal(got_d[ok], ref[ok])
    assert np.array_equal(np.isnan(got_h), ~ok) and np.array_equal(got_h[ok], ref[ok])
