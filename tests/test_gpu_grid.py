"""Sample points generated on the device (pb_grid_points) against the host's coordinate_grid +
flatten (StructuredGrid.jl:126-204, transform.jl:53-66), StructuredGrid_interpolation with
device-generated points against the host path, and image lines generated on the device
(pb_line_image) against the host's LineSamples construction (LineSamples.jl:391-403)."""
import numpy as np
import pytest

import distorteddustydiscanalysistoolkits_b200 as pb
from distorteddustydiscanalysistoolkits_b200 import synthetic
from distorteddustydiscanalysistoolkits_b200.interpolation import grid_points_device
import oracle


def _input(p, cols):
    return pb.InterpolationInput(p["x"].copy(), p["y"].copy(), p["z"].copy(), p["m"].copy(), p["h"].copy(),
                                 p["rho"].copy(), tuple(p[c].copy() for c in cols), smoothed_kernel=pb.M4_spline)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("coord,grid,exact", [
    (pb.Cartesian, lambda: pb.StructuredGrid.cartesian((-3.0, 2.5, 7), (0.1, 4.0, 5), (-1.0, 1.0, 3)), True),
    (pb.Cylindrical, lambda: synthetic.log_cylindrical_grid(9, 8, 5), False),
    (pb.Spherical, lambda: pb.StructuredGrid.spherical((0.5, 3.0, 6), (0.0, 6.0, 7), (0.1, 3.0, 5)), False),
])
def test_device_points_match_host(backend, coord, grid, exact):
    g = grid()
    host = pb.flatten(coord, g).coor
    dev = [t.cpu().numpy() for t in grid_points_device(backend, coord, g)]
    for h, d in zip(host, dev):
        if exact:
            assert np.array_equal(h, d)
        else:   # the device's sin/cos against the host's: a few ulp of the coordinate scale
            scale = np.abs(h).max()
            assert np.abs(h - d).max() <= 8 * np.finfo(np.float64).eps * scale


def test_structured_grid_interpolation_with_device_points(backend):
    p = synthetic.disc(20000, seed=31)
    cols = ("rho", "vx", "vy", "vz")
    cat = pb.InterpolationCatalog(cols, **synthetic.C2_CATALOG)

    def inp():
        return pb.InterpolationInput(p["x"].copy(), p["y"].copy(), p["z"].copy(), p["m"].copy(), p["h"].copy(),
                                     p["rho"].copy(), tuple(p[c].copy() for c in cols))

    g = synthetic.cartesian_box_grid(p, n=12)
    a = pb.StructuredGrid_interpolation(backend, pb.Cartesian, g, inp(), cat, pb.itpSymmetric, precision=pb.FP64)
    b = pb.StructuredGrid_interpolation(backend, pb.Cartesian, g, inp(), cat, pb.itpSymmetric, precision=pb.FP64,
                                        points_on_device=True)
    for x, y in zip(a.grids, b.grids):
        assert x.grid.shape == y.grid.shape
        assert np.array_equal(x.grid.view(np.uint64), y.grid.view(np.uint64))
    g = synthetic.log_cylindrical_grid(10, 8, 6)
    a = pb.StructuredGrid_interpolation(backend, pb.Cylindrical, g, inp(), cat, pb.itpSymmetric, precision=pb.FP64)
    b = pb.StructuredGrid_interpolation(backend, pb.Cylindrical, g, inp(), cat, pb.itpSymmetric, precision=pb.FP64,
                                        points_on_device=True)
    for x, y in zip(a.grids, b.grids):
        ok = ~np.isnan(x.grid)
        assert np.array_equal(ok, ~np.isnan(y.grid))
        scale = np.abs(x.grid[ok]).max()
        assert np.abs(x.grid[ok] - y.grid[ok]).max() <= 1e-9 * scale


def test_line_image_on_device_matches_host_lines(backend):
    """pb_line_image builds the face-on image's lines exactly as the host does
    (synthetic.face_on_lines), and column densities from device-resident lines equal those from
    host lines bit for bit."""
    torch = pytest.importorskip("torch")
    p = synthetic.disc(30000, seed=41)
    host = synthetic.face_on_lines(p, npix=64)
    x = pb.grids.linrange(float(np.min(p["x"])), float(np.max(p["x"])), 64)
    y = pb.grids.linrange(float(np.min(p["y"])), float(np.max(p["y"])), 64)
    dev = pb.LineSamples_image(backend, x, y)
    for d in range(3):
        assert np.array_equal(dev.origin[d].cpu().numpy(), host.origin[d])
        assert np.array_equal(dev.direction[d].cpu().numpy(), host.direction[d])
    cat = pb.InterpolationCatalog(("rho", "vz"), scalars=("rho", "vz"))
    ref = pb.LineSamples_interpolation(backend, host, _input(p, ("rho", "vz")), cat, pb.itpScatter)
    got = pb.LineSamples_interpolation(backend, dev, _input(p, ("rho", "vz")), cat, pb.itpScatter)
    for a, b in zip(got.grids, ref.grids):
        a = a.grid.cpu().numpy() if hasattr(a.grid, "cpu") else a.grid
        assert np.array_equal(np.isnan(a), np.isnan(b.grid)) and np.array_equal(a[~np.isnan(a)], b.grid[~np.isnan(a)])
    # an oblique image plane: per-component (c + u e1) + v e2 in the host's order
    c, e1, e2 = (1.0, -2.0, 0.5), (0.6, 0.8, 0.0), (0.0, 0.6, 0.8)
    d = np.cross(e1, e2)
    d /= np.linalg.norm(d)
    obl = pb.LineSamples_image(backend, x[:7], y[:5], c, e1, e2, tuple(d), on_device=False)
    U, V = np.meshgrid(x[:7], y[:5], indexing="ij")
    U, V = U.reshape(-1, order="F"), V.reshape(-1, order="F")
    for k in range(3):
        assert np.array_equal(obl.origin[k], (c[k] + U * e1[k]) + V * e2[k])
        assert (obl.direction[k] == d[k]).all()
    with pytest.raises(pb.ArgumentError):
        pb.LineSamples_image(backend, x, y, direction=(0.0, 0.0, 2.0))


def test_lines_256_image_against_oracle(backend):
    """A 256^2 face-on column-density image of a two-species disc against the oracle:
    FP64 bit-exact, FP32C within 1e-5 of each field's magnitude."""
    gas, dust = synthetic.dusty_disc(90000, 30000, seed=8)
    cat = pb.InterpolationCatalog(("rho", "vz"), scalars=("rho", "vz"))
    for p in (gas, dust):
        x = pb.grids.linrange(float(np.min(p["x"])), float(np.max(p["x"])), 256)
        y = pb.grids.linrange(float(np.min(p["y"])), float(np.max(p["y"])), 256)
        lines = pb.LineSamples_image(backend, x, y, on_device=False)
        exp = oracle.OracleLBVH(p["x"], p["y"], p["z"], p["h"]).attach(
            p["m"], p["rho"], [p["rho"], p["vz"]], "M4_spline").interp_lines(cat.oracle_dict(), lines.origin,
                                                                             lines.direction)
        out = pb.LineSamples_interpolation(backend, lines, _input(p, ("rho", "vz")), cat, pb.itpScatter,
                                           precision=pb.FP64)
        got = np.stack([g.grid for g in out.grids])
        assert np.array_equal(np.isnan(got), np.isnan(exp))
        assert np.array_equal(got[~np.isnan(exp)], exp[~np.isnan(exp)])
        out = pb.LineSamples_interpolation(backend, lines, _input(p, ("rho", "vz")), cat, pb.itpScatter,
                                           precision=pb.FP32C)
        got = np.stack([g.grid for g in out.grids])
        scale = np.nanmax(np.abs(exp), axis=1, keepdims=True)
        assert np.nanmax(np.abs(got - exp) / scale) <= 1e-5
