"""Sample points generated on the device (pb_grid_points) against the host's coordinate_grid +
flatten (StructuredGrid.jl:126-204, transform.jl:53-66), and StructuredGrid_interpolation with
device-generated points against the host path."""
import numpy as np
import pytest

import distorteddustydiscanalysistoolkits_b200 as pb
from distorteddustydiscanalysistoolkits_b200 import synthetic
from distorteddustydiscanalysistoolkits_b200.interpolation import grid_points_device

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
