"""Host-side API mirror and C-ABI library checks (no GPU needed).

Catalog construction and naming (InterpolationCatalog.jl:71-225), input validation
(InterpolationInput.jl:85-109), grid geometry and flatten/restore
(Partia.jl/test/structured_grid_interpolation_tests.jl), error classes of the entry points
that are decided on the host, and the shared library: it loads, exports every function
declared in include/partia_b200.h, and refuses to run without a CUDA device (no CPU
fallback).
"""
import ctypes
import os
import re

import numpy as np
import pytest

import distorteddustydiscanalysistoolkits_b200 as pb
from distorteddustydiscanalysistoolkits_b200 import _lib

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_catalog_names_slots_and_shepard_flags():
    cat = pb.InterpolationCatalog(("rho", "vx", "vy", "vz", "T"), scalars=("rho", "T"), gradients=("rho",),
                                  divergences=("v",), curls=("v",))
    assert cat.scalar_slots == (0, 4)
    assert cat.scalar_snormalization == (False, True)
    assert cat.grad_slots == (0,)
    assert cat.div_slots == ((1, 2, 3),)
    assert cat.ordered_names == ("rho", "T", "∇rhoˣ", "∇rhoʸ", "∇rhoᶻ", "∇⋅v", "∇×vˣ", "∇×vʸ", "∇×vᶻ")
    assert cat.L == 9
    assert pb.InterpolationCatalog(("ρ",), scalars=("ρ",)).scalar_snormalization == (False,)


def test_catalog_errors():
    with pytest.raises(KeyError):
        pb.InterpolationCatalog(("a",), scalars=("b",))
    with pytest.raises(KeyError):
        pb.InterpolationCatalog(("vx", "vy"), divergences=("v",))
    with pytest.raises(pb.ArgumentError):
        pb.InterpolationCatalog(("a", "a"), scalars=("a",))
    with pytest.raises(pb.DimensionMismatch):
        pb.InterpolationCatalog.from_slots(scalar_names=("a",), scalar_slots=())


def test_catalog_from_slots_density_gradient():
    cat = pb.InterpolationCatalog.from_slots(scalar_names=("rho",), scalar_slots=(1,), grad_names=("ρ",),
                                             grad_slots=(0,))
    assert cat.grad_slots == (-1,)
    assert cat.scalar_slots == (0,)
    d = cat.oracle_dict()
    assert d["grad_cols"] == [-1] and d["scalar_shepard"] == [0]


def test_input_validation():
    z3 = np.zeros(3)
    with pytest.raises(pb.DimensionMismatch):
        pb.InterpolationInput(z3, z3, np.zeros(2), z3, z3, z3)
    with pytest.raises(pb.DimensionMismatch):
        pb.InterpolationInput(z3, z3, z3, z3, z3, z3, (np.zeros(4),))
    with pytest.raises(pb.ArgumentError):
        pb.InterpolationInput(z3, z3, z3, z3, z3, z3, smoothed_kernel=int)
    with pytest.raises(pb.ArgumentError):
        pb.InterpolationInput(np.zeros(3, np.float32), z3, z3, z3, z3, z3)
    inp, cat = pb.build_input([0.0, 1.0], [0, 1], [0, 1], [1, 1], [0.1, 0.1], [1, 1], ([5, 6],),
                              column_names=("T",), scalars=("T",), smoothed_kernel=pb.C4_Wendland)
    assert inp.Npart == 2 and inp.smoothed_kernel is pb.C4_Wendland and cat.L == 1


def test_linrange_and_steprange():
    r = pb.grids.linrange(0.2, 0.7, 3)
    assert r[0] == 0.2 and r[-1] == 0.7 and abs(r[1] - 0.45) < 1e-15
    s = pb.grids.steprange(0.0, 2 * np.pi / 4, 4)
    assert np.allclose(s, [0, np.pi / 2, np.pi, 3 * np.pi / 2])


@pytest.mark.parametrize("coord,grid", [
    (pb.Cartesian, lambda: pb.StructuredGrid.cartesian((0.2, 0.7, 3), (0.25, 0.55, 2), (0.3, 0.6, 2))),
    (pb.Cylindrical, lambda: pb.StructuredGrid.cylindrical((0.25, 0.55, 3), (0.3, 1.1, 2), (0.2, 0.5, 2))),
    (pb.Spherical, lambda: pb.StructuredGrid.spherical((0.5, 0.7, 2), (0.35, 0.85, 2), (0.8, 1.1, 2))),
])
def test_flatten_restore_roundtrip(coord, grid):
    g = grid()
    g.grid[...] = np.arange(len(g)).reshape(g.size, order="F")
    flat = pb.flatten(coord, g)
    assert len(flat) == len(g)
    assert np.array_equal(flat.grid, np.arange(len(g)))
    back = pb.restore_struct(coord, flat, g.axes)
    assert np.array_equal(back.grid, g.grid)
    # column-major: first axis fastest
    if coord is pb.Cartesian:
        assert flat.coor[0][1] == g.axes[0][1] and flat.coor[1][1] == g.axes[1][0]


def test_restore_struct_rejects_mismatched_coordinates():
    g = pb.StructuredGrid.cartesian((0.0, 1.0, 3), (0.0, 1.0, 3), (0.0, 1.0, 3))
    flat = pb.flatten(pb.Cartesian, g)
    flat.coor[0][0] += 1.0
    with pytest.raises(pb.ArgumentError):
        pb.restore_struct(pb.Cartesian, flat, g.axes)


def test_cylindrical_grid_argument_checks():
    with pytest.raises(pb.ArgumentError):
        pb.StructuredGrid.cylindrical((0.5, 0.2, 3), (0.0, 1.0, 2), (0.0, 1.0, 2))
    with pytest.raises(pb.ArgumentError):
        pb.StructuredGrid.cylindrical((0.1, 0.2, 3), (0.0, 7.0, 2), (0.0, 1.0, 2))


def test_line_samples_validation_and_strategy_error():
    with pytest.raises(pb.ArgumentError):
        pb.LineSamples(np.zeros(2), (np.zeros(2), np.zeros(2), np.zeros(1)), (np.zeros(2),) * 3)
    lines = pb.LineSamples.from_arrays(*(np.zeros(2),) * 6)
    inp = pb.InterpolationInput(*(np.zeros(2),) * 6)
    cat = pb.InterpolationCatalog((), scalars=())
    for s in (pb.itpGather, pb.itpSymmetric):
        with pytest.raises(pb.ArgumentError):   # decided before any device work
            pb.LineSamples_interpolation(pb.CUDAComputeBackend(), lines, inp, cat, s)


def _declared_functions():
    hdr = open(os.path.join(REPO, "include", "partia_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int32_t|int64_t|void)\s+(pb_\w+)\s*\(", hdr, re.M)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = _declared_functions()
    assert len(names) >= 19
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_lib.EXPORTED)


def test_no_cpu_fallback_without_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(pb.DeviceError):
        pb.CUDAComputeBackend(0).handle


def test_noalloc_rejects_host_pointers_and_oversize():
    lib = _lib.load()
    a = np.zeros(4)
    out = np.zeros(4, np.int64)
    rc = lib.pb_morton_sort_noalloc(a.ctypes.data, a.ctypes.data, a.ctypes.data, 4, out.ctypes.data,
                                    out.ctypes.data, None)
    assert rc == _lib.PB_ERR_INVALID
    rc = lib.pb_morton_sort_noalloc(a.ctypes.data, a.ctypes.data, a.ctypes.data, 262145, out.ctypes.data,
                                    out.ctypes.data, None)
    assert rc == _lib.PB_ERR_CAPACITY
