"""Sample containers and structured-grid geometry on the host (numpy).

Mirrors Partia's grid layer (Partia.jl/src/julia/Grids/): ``PointSamples``
(grids/PointSamples.jl:25-39), ``LineSamples`` (grids/LineSamples.jl:31-47),
``StructuredGrid`` with Cartesian/Polar/Cylindrical/Spherical constructors
(grids/StructuredGrid.jl:42-46,262-400), ``coordinate_grid`` (StructuredGrid.jl:126-204),
``flatten``/``restore_struct`` (grids/transform.jl:53-116) and ``GridBundle``
(griddataset/GridBundle.jl:1-4).  Flattening is column-major (first axis fastest), as
Julia's ``vec``.
"""
import numpy as np

from ._lib import ArgumentError


class Cartesian:
    pass


class Polar:          # (s, phi)
    pass


class Cylindrical:    # (s, phi, z)
    pass


class Spherical:      # (r, phi, theta)
    pass


def _f64(a):
    """float64, contiguous; a torch tensor (e.g. sample coordinates on the device) stays a tensor."""
    if hasattr(a, "data_ptr") and hasattr(a, "is_contiguous"):
        if str(a.dtype) != "torch.float64":
            a = a.double()
        return a.contiguous()
    return np.ascontiguousarray(a, dtype=np.float64)


class PointSamples:
    """Unstructured sample points: values ``grid`` (N,) and SoA coordinates ``coor`` (D arrays)."""

    def __init__(self, grid, coor):
        grid = _f64(grid)
        coor = tuple(_f64(c) for c in coor)
        for d, c in enumerate(coor):
            if len(c) != len(grid):
                raise ArgumentError("coor[%d] length mismatch" % (d + 1))
        self.grid = grid
        self.coor = coor

    def __len__(self):
        return len(self.grid)

    def similar(self):
        return PointSamples(np.zeros_like(self.grid), self.coor)


class LineSamples:
    """Line samples: values ``grid`` (N,), SoA ``origin`` and unit ``direction`` (3 arrays each)."""

    def __init__(self, grid, origin, direction):
        grid = _f64(grid)
        origin = tuple(_f64(c) for c in origin)
        direction = tuple(_f64(c) for c in direction)
        for d in range(len(origin)):
            if len(origin[d]) != len(grid):
                raise ArgumentError("origin[%d] length mismatch" % (d + 1))
            if len(direction[d]) != len(grid):
                raise ArgumentError("direction[%d] length mismatch" % (d + 1))
        self.grid = grid
        self.origin = origin
        self.direction = direction

    @classmethod
    def from_arrays(cls, xo, yo, zo, xd, yd, zd):
        return cls(np.zeros(len(xo)), (xo, yo, zo), (xd, yd, zd))

    def __len__(self):
        return len(self.grid)

    def similar(self):
        return LineSamples(np.zeros_like(self.grid), self.origin, self.direction)


def linrange(a, b, n):
    """Julia LinRange{Float64}(a, b, n): element j is (1-t)*a + t*b with t = j/(n-1)."""
    if n == 1:
        return np.array([float(a)])
    j = np.arange(n, dtype=np.float64)
    t = j / (n - 1)
    return (1.0 - t) * a + t * b


def steprange(a, step, n):
    """range(a, step=step, length=n) with the step accumulated in extended precision."""
    k = np.arange(n, dtype=np.longdouble)
    return np.asarray(np.longdouble(a) + k * np.longdouble(step), dtype=np.float64)


class StructuredGrid:
    """Tensor-product grid: values ``grid`` of shape ``size`` (column-major) and 1D ``axes``."""

    def __init__(self, grid, axes, size=None):
        axes = tuple(_f64(a) for a in axes)
        size = tuple(len(a) for a in axes) if size is None else tuple(size)
        self.axes = axes
        self.size = size
        self.grid = np.asarray(grid, dtype=np.float64).reshape(size, order="F") if grid is not None \
            else np.zeros(size, order="F")

    @classmethod
    def cartesian(cls, *params):
        axes = [linrange(a, b, n) for (a, b, n) in params]
        return cls(None, axes)

    @classmethod
    def polar(cls, sparams, phiparams):
        (smin, smax, ns), (pmin, pmax, npf) = sparams, phiparams
        _check_radial(smin, smax)
        _check_phi(pmin, pmax)
        return cls(None, [linrange(smin, smax, ns), steprange(pmin, (pmax - pmin) / npf, npf)])

    @classmethod
    def cylindrical(cls, sparams, phiparams, zparams):
        (smin, smax, ns), (pmin, pmax, npf), (zmin, zmax, nz) = sparams, phiparams, zparams
        if min(ns, npf, nz) < 1:
            raise ArgumentError("ns, nphi, nz must be >= 1")
        _check_radial(smin, smax)
        _check_phi(pmin, pmax)
        if not zmax > zmin:
            raise ArgumentError("axial range must satisfy zmin < zmax")
        return cls(None, [linrange(smin, smax, ns), steprange(pmin, (pmax - pmin) / npf, npf),
                          linrange(zmin, zmax, nz)])

    @classmethod
    def spherical(cls, rparams, phiparams, thetaparams):
        return cls(None, [linrange(*rparams), linrange(*phiparams), linrange(*thetaparams)])

    def __len__(self):
        return int(np.prod(self.size))


def _check_radial(smin, smax):
    if not (smin >= 0.0 and smax > smin):
        raise ArgumentError("radial range must satisfy 0 <= smin < smax")


def _check_phi(pmin, pmax):
    if not (pmin >= 0.0 and (pmax <= 2 * np.pi or np.isclose(pmax, 2 * np.pi)) and pmax > pmin):
        raise ArgumentError("angular range must satisfy 0 <= phimin < phimax <= 2pi")


def _mesh(grid):
    return np.meshgrid(*grid.axes, indexing="ij")


def coordinate_grid(coord, grid):
    """Cartesian coordinates of every grid point, column-major linear order (StructuredGrid.jl:126-204)."""
    m = [a.reshape(-1, order="F") for a in _mesh(grid)]
    if coord is Cartesian:
        return tuple(np.ascontiguousarray(a) for a in m)
    if coord is Polar:
        s, p = m
        return (s * np.cos(p), s * np.sin(p))
    if coord is Cylindrical:
        s, p, z = m
        return (s * np.cos(p), s * np.sin(p), np.ascontiguousarray(z))
    if coord is Spherical:
        r, p, t = m
        st = np.sin(t)
        return (r * st * np.cos(p), r * st * np.sin(p), r * np.cos(t))
    raise ArgumentError("unknown coordinate system %r" % (coord,))


def flatten(coord, grid):
    """StructuredGrid -> PointSamples (grids/transform.jl:53-66)."""
    return PointSamples(grid.grid.reshape(-1, order="F"), coordinate_grid(coord, grid))


def restore_struct(coord, samples, axes, atol=1.0e-8, rtol=1.0e-8):
    """PointSamples -> StructuredGrid after checking the coordinates (grids/transform.jl:107-116)."""
    size = tuple(len(a) for a in axes)
    template = StructuredGrid(None, axes, size)
    expected = coordinate_grid(coord, template)
    for a, e in zip(samples.coor, expected):
        if len(a) != len(e) or not np.allclose(a, e, atol=atol, rtol=rtol):
            raise ArgumentError("PointSamples coordinates do not match the provided axes under %s dispatch"
                                % coord.__name__)
    return StructuredGrid(samples.grid, axes, size)


class GridBundle:
    """Output bundle: ``grids`` (one per output quantity) and ``names`` (catalog.ordered_names)."""

    def __init__(self, grids, names):
        self.grids = tuple(grids)
        self.names = tuple(names)

    def __getitem__(self, name):
        return self.grids[self.names.index(name)]

    def __len__(self):
        return len(self.grids)
