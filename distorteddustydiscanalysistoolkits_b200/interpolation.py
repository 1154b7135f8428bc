"""Partia's interpolation entry points, executed by the B200 library.

Host-side mirror of the reference interface for the hot path, with the same names,
argument meaning and error behaviour:

  InterpolationInput      Partia.jl/src/julia/KernelInterpolation/interpolation_setup/InterpolationInput.jl:43-109
  InterpolationCatalog    .../interpolation_setup/InterpolationCatalog.jl:9-225
  build_input             .../interpolation_setup/constructor.jl:69-137
  itpGather/itpScatter/itpSymmetric   .../interpolation_setup/InterpolationStrategy.jl:1-5
  CUDAComputeBackend      Partia.jl/src/julia/ExtDummy/CUDAExtDummy.jlh:12
  PointSamples_interpolation   Partia.jl/ext/CUDAExt/KernelInterpolation/grid_interpolation/PointSamples_interpolation.jl:12-29
  LineSamples_interpolation    Partia.jl/ext/CUDAExt/KernelInterpolation/grid_interpolation/LineSamples_interpolation.jl:11-34
  StructuredGrid_interpolation .../grid_interpolation/StructuredGrid_interpolation.jl:46-64

Every call goes through the C ABI of libpartia_b200.so; arrays may be numpy (host)
or torch CUDA tensors (device).  Like the reference, interpolation permutes the
particle columns of ``input`` in place into Morton order (InterpolationInput.jl:211-219).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import ArgumentError, DimensionMismatch, PBCatalog, PBInput, ptr
from .grids import GridBundle, LineSamples, PointSamples, StructuredGrid, flatten, restore_struct


# ---- kernels (Partia.jl/src/julia/KernelInterpolation/kernel_function/kernels/) ----
class _Kernel:
    code = -1
    valid = 2.0


class M4_spline(_Kernel):
    code, valid = 0, 2.0


class M5_spline(_Kernel):
    code, valid = 1, 2.5


class M6_spline(_Kernel):
    code, valid = 2, 3.0


class C2_Wendland(_Kernel):
    code, valid = 3, 2.0


class C4_Wendland(_Kernel):
    code, valid = 4, 2.0


class C6_Wendland(_Kernel):
    code, valid = 5, 2.0


KERNELS = (M4_spline, M5_spline, M6_spline, C2_Wendland, C4_Wendland, C6_Wendland)


def KernelFunctionValid(K):
    """Support radius in units of h (kernels/*.jl: KernelFunctionValid)."""
    return K.valid


# ---- strategies ----
class itpGather:
    code = 0


class itpScatter:
    code = 1


class itpSymmetric:
    code = 2


FP64 = "fp64"
FP32C = "fp32c"


def _precision(p):
    if p in (FP64, _lib.PB_FP64):
        return _lib.PB_FP64
    if p in (FP32C, _lib.PB_FP32C, "fp32"):
        return _lib.PB_FP32C
    raise ArgumentError("unknown precision %r" % (p,))


class CUDAComputeBackend:
    """Execution backend tag of Partia's CUDA extension.  Holds one library handle (the
    device buffers of the last particle set stay resident between calls)."""

    def __init__(self, device=0):
        self.device = int(device)
        self._handle = None

    @property
    def handle(self):
        if self._handle is None:
            self._handle = _lib.Handle(self.device)
        return self._handle

    def close(self):
        if self._handle is not None:
            self._handle.close()
            self._handle = None


def Greeting_CUDA(backend=None):
    """Print the CUDA device the extension runs on (CUDAExt.jl Greeting_CUDA)."""
    import torch
    d = backend.device if backend is not None else 0
    print("Hello from the B200 CUDA extension: %s (cc %d.%d)" % ((torch.cuda.get_device_name(d),)
                                                                   + torch.cuda.get_device_capability(d)))


def _is_array(a):
    return isinstance(a, np.ndarray) or hasattr(a, "data_ptr")


def _len(a):
    return int(a.shape[0])


def _as_f64(a):
    if hasattr(a, "data_ptr"):
        import torch
        if a.dtype != torch.float64 or not a.is_contiguous():
            raise ArgumentError("particle columns must be contiguous float64 tensors")
        return a
    a = np.asarray(a)
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise ArgumentError("particle columns must be contiguous float64 arrays "
                            "(in-place Morton permutation needs the caller's own buffer)")
    return a


class InterpolationInput:
    """SoA particle container: coord (x, y, z), m, h, rho and NCOLUMN quantity columns."""

    def __init__(self, x, y, z, m, h, rho, quant=(), smoothed_kernel=M5_spline):
        cols = [_as_f64(c) for c in (x, y, z, m, h, rho)]
        quant = tuple(_as_f64(q) for q in quant)
        n = _len(cols[3])
        for d, c in enumerate(cols[:3]):
            if _len(c) != n:
                raise DimensionMismatch("coord[%d] length %d != Nparticles %d" % (d + 1, _len(c), n))
        if _len(cols[4]) != n:
            raise DimensionMismatch("h length %d != Nparticles %d" % (_len(cols[4]), n))
        if _len(cols[5]) != n:
            raise DimensionMismatch("rho length %d != Nparticles %d" % (_len(cols[5]), n))
        for j, q in enumerate(quant):
            if _len(q) != n:
                raise DimensionMismatch("quant[%d] length %d != Nparticles %d" % (j + 1, _len(q), n))
        if not (isinstance(smoothed_kernel, type) and issubclass(smoothed_kernel, _Kernel)):
            raise ArgumentError("smoothed_kernel must be one of %s" % ", ".join(k.__name__ for k in KERNELS))
        self.Npart = n
        self.smoothed_kernel = smoothed_kernel
        self.coord = tuple(cols[:3])
        self.m, self.h, self.rho = cols[3], cols[4], cols[5]
        self.quant = quant

    def __len__(self):
        return self.Npart

    def _c_struct(self):
        qarr = (ctypes.c_void_p * max(len(self.quant), 1))(*[ptr(q) for q in self.quant])
        s = PBInput(self.Npart, ptr(self.coord[0]), ptr(self.coord[1]), ptr(self.coord[2]), ptr(self.m),
                    ptr(self.h), ptr(self.rho), len(self.quant),
                    ctypes.cast(qarr, ctypes.POINTER(ctypes.c_void_p)), self.smoothed_kernel.code)
        s._keep = qarr
        return s


_NO_NORM = ("ρ", "rho")
_DERIV = ("ˣ", "ʸ", "ᶻ")


class InterpolationCatalog:
    """Output catalog: scalar, gradient, divergence and curl targets resolved to 0-based
    quantity columns.  A gradient slot of -1 is the density gradient (the reference's slot 0).
    Shepard normalisation is off exactly for the scalar names rho/ρ (InterpolationCatalog.jl:222-225)."""

    def __init__(self, column_names=None, scalars=(), gradients=(), divergences=(), curls=()):
        if column_names is None:
            column_names = ()
        column_names = tuple(column_names)
        if len(set(column_names)) != len(column_names):
            raise ArgumentError("column_names must be unique")
        index = {name: i for i, name in enumerate(column_names)}

        def col(name):
            if name not in index:
                raise KeyError(name)
            return index[name]

        self._init(tuple(scalars), tuple(col(s) for s in scalars),
                   tuple(gradients), tuple(col(g) for g in gradients),
                   tuple(divergences), tuple(tuple(col(c) for c in _components(d)) for d in divergences),
                   tuple(curls), tuple(tuple(col(c) for c in _components(c)) for c in curls))

    @classmethod
    def from_slots(cls, scalar_names=(), scalar_slots=(), grad_names=(), grad_slots=(), div_names=(),
                   div_slots=(), curl_names=(), curl_slots=()):
        """Explicit-slot constructor (InterpolationCatalog.jl:71-102); slots are 1-based as in
        Julia and grad slot 0 selects the density gradient."""
        for a, b, what in ((scalar_names, scalar_slots, "scalar"), (grad_names, grad_slots, "grad"),
                           (div_names, div_slots, "div"), (curl_names, curl_slots, "curl")):
            if len(a) != len(b):
                raise DimensionMismatch("%s_slots length %d != %s_names length %d" % (what, len(b), what, len(a)))
        self = cls.__new__(cls)
        self._init(tuple(scalar_names), tuple(s - 1 for s in scalar_slots),
                   tuple(grad_names), tuple(-1 if s == 0 else s - 1 for s in grad_slots),
                   tuple(div_names), tuple(tuple(c - 1 for c in t) for t in div_slots),
                   tuple(curl_names), tuple(tuple(c - 1 for c in t) for t in curl_slots))
        return self

    def _init(self, sn, ss, gn, gs, dn, ds, cn, cs):
        self.scalar_names, self.scalar_slots = sn, ss
        self.scalar_snormalization = tuple(name not in _NO_NORM for name in sn)
        self.grad_names, self.grad_slots = gn, gs
        self.div_names, self.div_slots = dn, ds
        self.curl_names, self.curl_slots = cn, cs
        names = list(sn)
        for b in gn:
            names += ["∇" + b + s for s in _DERIV]
        for b in dn:
            names.append("∇⋅" + b)
        for b in cn:
            names += ["∇×" + b + s for s in _DERIV]
        self.ordered_names = tuple(names)
        self.L = len(names)

    def oracle_dict(self):
        """The catalog as plain column lists (the form the CPU oracle takes)."""
        return {"scalar_cols": list(self.scalar_slots), "scalar_shepard": [int(f) for f in self.scalar_snormalization],
                "grad_cols": list(self.grad_slots), "div_cols": [list(t) for t in self.div_slots],
                "curl_cols": [list(t) for t in self.curl_slots]}

    def _c_struct(self):
        arrs = [np.ascontiguousarray(a, np.int32).reshape(-1) for a in
                (self.scalar_slots, [int(f) for f in self.scalar_snormalization], self.grad_slots,
                 [c for t in self.div_slots for c in t], [c for t in self.curl_slots for c in t])]
        arrs = [a if len(a) else np.zeros(1, np.int32) for a in arrs]
        P = ctypes.POINTER(ctypes.c_int32)
        s = PBCatalog(len(self.scalar_slots), arrs[0].ctypes.data_as(P), arrs[1].ctypes.data_as(P),
                      len(self.grad_slots), arrs[2].ctypes.data_as(P), len(self.div_slots), arrs[3].ctypes.data_as(P),
                      len(self.curl_slots), arrs[4].ctypes.data_as(P))
        s._keep = arrs
        return s


def _components(name):
    return (name + "x", name + "y", name + "z")


def build_input(x, y, z, m, h, rho, quantity_columns=(), column_names=(), scalars=(), gradients=(),
                divergences=(), curls=(), smoothed_kernel=M5_spline):
    """InterpolationInput + InterpolationCatalog from materialised columns (constructor.jl:69-137)."""
    if len(quantity_columns) != len(column_names):
        raise DimensionMismatch("column_names must correspond one-to-one with quantity_columns")

    def f64(a):
        return a if hasattr(a, "data_ptr") else np.array(a, dtype=np.float64)

    inp = InterpolationInput(f64(x), f64(y), f64(z), f64(m), f64(h), f64(rho),
                             tuple(f64(q) for q in quantity_columns), smoothed_kernel=smoothed_kernel)
    cat = InterpolationCatalog(column_names, scalars=scalars, gradients=gradients, divergences=divergences,
                               curls=curls)
    return inp, cat


def _out_arrays(n, L, like=None):
    if like is not None and hasattr(like, "data_ptr") and like.is_cuda:
        import torch
        return [torch.empty(n, dtype=torch.float64, device=like.device) for _ in range(L)]
    return [np.empty(n, dtype=np.float64) for _ in range(L)]


def _ptr_array(arrs):
    return (ctypes.c_void_p * max(len(arrs), 1))(*[ptr(a) for a in arrs])


def _strategy(s):
    if s in (itpGather, itpScatter, itpSymmetric):
        return s.code
    raise ArgumentError("unknown interpolation strategy %r" % (s,))


def PointSamples_interpolation(backend, grid_template, input, catalog, itp_strategy=itpSymmetric, precision=FP64,
                               out=None):
    """Build the LBVH of ``input`` (permuting it in place) and interpolate the catalog at every
    point of ``grid_template``.  Returns a GridBundle of PointSamples sharing the template's
    coordinates, one per catalog.ordered_names entry (written into ``out`` when given)."""
    if not isinstance(backend, CUDAComputeBackend):
        raise ArgumentError("backend must be a CUDAComputeBackend")
    if not isinstance(grid_template, PointSamples):
        raise ArgumentError("grid_template must be PointSamples")
    H = backend.handle
    n = len(grid_template)
    outs = out if out is not None else _out_arrays(n, catalog.L)
    if len(outs) != catalog.L:
        raise DimensionMismatch("out must hold %d arrays" % catalog.L)
    cin, ccat = input._c_struct(), catalog._c_struct()
    optrs = _ptr_array(outs)
    qx, qy, qz = grid_template.coor
    rc = H.lib.pb_point_samples_interpolation(H.h, ctypes.byref(cin), ctypes.byref(ccat), n, ptr(qx), ptr(qy),
                                              ptr(qz), _strategy(itp_strategy), _precision(precision), optrs,
                                              _lib.PB_PERMUTE_CALLER)
    H.check(rc, "PointSamples_interpolation")
    return GridBundle([PointSamples(o, grid_template.coor) for o in outs], catalog.ordered_names)


def LineSamples_interpolation(backend, grid_template, input, catalog, itp_strategy=itpScatter, precision=FP64):
    """Line-integrated (column) interpolation along every line of ``grid_template``; only
    itpScatter is defined (LineSamples_interpolation.jl:48-52)."""
    if not isinstance(backend, CUDAComputeBackend):
        raise ArgumentError("backend must be a CUDAComputeBackend")
    if itp_strategy is not itpScatter:
        raise ArgumentError("LineSamples_interpolation only supports itpScatter. Line-integrated samples do not "
                            "have a well-defined query smoothing length ha, so itpGather and itpSymmetric are "
                            "not supported.")
    if not isinstance(grid_template, LineSamples):
        raise ArgumentError("grid_template must be LineSamples")
    if len(catalog.grad_slots) or len(catalog.div_slots) or len(catalog.curl_slots):
        raise TypeError("LineSamples_interpolation takes a scalar-only catalog (MethodError in the reference)")
    H = backend.handle
    n = len(grid_template)
    o, d = grid_template.origin, grid_template.direction
    outs = _out_arrays(n, catalog.L, like=o[0])
    cin, ccat = input._c_struct(), catalog._c_struct()
    rc = H.lib.pb_line_samples_interpolation(H.h, ctypes.byref(cin), ctypes.byref(ccat), n, ptr(o[0]), ptr(o[1]),
                                             ptr(o[2]), ptr(d[0]), ptr(d[1]), ptr(d[2]), itpScatter.code,
                                             _precision(precision), _ptr_array(outs), _lib.PB_PERMUTE_CALLER)
    H.check(rc, "LineSamples_interpolation")
    return GridBundle([LineSamples(v, o, d) for v in outs], catalog.ordered_names)


def LineSamples_image(backend, a0, a1, center=(0.0, 0.0, 0.0), e1=(1.0, 0.0, 0.0), e2=(0.0, 1.0, 0.0),
                      direction=(0.0, 0.0, 1.0), on_device=True):
    """The lines of an image, generated on the backend's device (pb_line_image): line
    i + len(a0) * j starts at (center + a0[i] e1) + a1[j] e2 and runs along the unit vector
    ``direction`` -- the LineSamples(xo, yo, zo, xd, yd, zd) a caller would build for a
    column-density map (LineSamples.jl:391-403), without a host-to-device copy of 48 B per line
    when ``on_device`` (origins and directions are then CUDA float64 tensors)."""
    a0 = np.ascontiguousarray(a0, np.float64)
    a1 = np.ascontiguousarray(a1, np.float64)
    n = len(a0) * len(a1)
    frame = np.ascontiguousarray(np.concatenate([center, e1, e2, direction]), np.float64)
    if frame.shape != (12,):
        raise ArgumentError("center, e1, e2 and direction must each have 3 components")
    if on_device:
        import torch
        out = [torch.empty(n, dtype=torch.float64, device="cuda:%d" % backend.device) for _ in range(6)]
    else:
        out = [np.empty(n) for _ in range(6)]
    H = backend.handle
    H.check(H.lib.pb_line_image(H.h, ptr(a0), len(a0), ptr(a1), len(a1), ptr(frame), *[ptr(x) for x in out]),
            "LineSamples_image")
    vals = out[0].new_zeros(n) if on_device else np.zeros(n)
    return LineSamples(vals, tuple(out[:3]), tuple(out[3:]))


_COORD_CODE = {"Cartesian": 0, "Cylindrical": 2, "Spherical": 3}


def grid_points_device(backend, coord, grid_template):
    """The flattened sample points of a 3D StructuredGrid, generated on the backend's device
    (pb_grid_points): three CUDA float64 tensors in column-major order (first axis fastest)."""
    import torch
    code = _COORD_CODE.get(coord.__name__)
    if code is None or len(grid_template.axes) != 3:
        raise ArgumentError("device grid points need a 3D Cartesian, Cylindrical or Spherical grid")
    axes = [np.ascontiguousarray(a, np.float64) for a in grid_template.axes]
    n = int(np.prod([len(a) for a in axes]))
    out = [torch.empty(n, dtype=torch.float64, device="cuda:%d" % backend.device) for _ in range(3)]
    H = backend.handle
    H.check(H.lib.pb_grid_points(H.h, code, ptr(axes[0]), len(axes[0]), ptr(axes[1]), len(axes[1]), ptr(axes[2]),
                                 len(axes[2]), out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr()), "grid_points")
    return out


def StructuredGrid_interpolation(backend, coord, grid_template, input, catalog, itp_strategy=itpSymmetric,
                                 precision=FP64, points_on_device=False):
    """flatten -> PointSamples_interpolation -> restore_struct (StructuredGrid_interpolation.jl:46-64).

    With ``points_on_device`` the sample points are generated on the device (grid_points_device)
    and never copied from the host; the outputs are reshaped directly (the generated points
    follow the axes by construction)."""
    if not isinstance(grid_template, StructuredGrid):
        raise ArgumentError("grid_template must be a StructuredGrid")
    if points_on_device:
        q = grid_points_device(backend, coord, grid_template)
        H = backend.handle
        n = len(q[0])
        outs = _out_arrays(n, catalog.L)
        cin, ccat = input._c_struct(), catalog._c_struct()
        rc = H.lib.pb_point_samples_interpolation(H.h, ctypes.byref(cin), ctypes.byref(ccat), n, q[0].data_ptr(),
                                                  q[1].data_ptr(), q[2].data_ptr(), _strategy(itp_strategy),
                                                  _precision(precision), _ptr_array(outs), _lib.PB_PERMUTE_CALLER)
        H.check(rc, "StructuredGrid_interpolation")
        size = tuple(len(a) for a in grid_template.axes)
        grids = [StructuredGrid(np.asarray(o).reshape(size, order="F"), grid_template.axes, size) for o in outs]
        return GridBundle(grids, catalog.ordered_names)
    flat = flatten(coord, grid_template)
    bundle = PointSamples_interpolation(backend, flat, input, catalog, itp_strategy, precision)
    grids = [restore_struct(coord, g, grid_template.axes) for g in bundle.grids]
    return GridBundle(grids, bundle.names)


def interpolate_points(lbvh, catalog, points, itp_strategy=itpSymmetric, precision=FP64, out=None):
    """The per-point loop of PointSamples_interpolation on an already built LinearBVH
    (several grids per particle snapshot).  ``points`` is (x, y, z); returns L arrays."""
    H = lbvh.handle
    qx, qy, qz = points
    n = _len(qx)
    outs = out if out is not None else _out_arrays(n, catalog.L, qx)
    ccat = catalog._c_struct()
    rc = H.lib.pb_interpolate_points(H.h, ctypes.byref(ccat), n, ptr(qx), ptr(qy), ptr(qz),
                                     _strategy(itp_strategy), _precision(precision), _ptr_array(outs))
    H.check(rc, "interpolate_points")
    return outs


def interpolate_lines(lbvh, catalog, origin, direction, precision=FP64, out=None, itp_strategy=itpScatter):
    """The per-line loop of LineSamples_interpolation on an already built LinearBVH."""
    H = lbvh.handle
    n = _len(origin[0])
    outs = out if out is not None else _out_arrays(n, catalog.L, origin[0])
    ccat = catalog._c_struct()
    rc = H.lib.pb_interpolate_lines(H.h, ctypes.byref(ccat), n, ptr(origin[0]), ptr(origin[1]), ptr(origin[2]),
                                    ptr(direction[0]), ptr(direction[1]), ptr(direction[2]),
                                    _strategy(itp_strategy), _precision(precision), _ptr_array(outs))
    H.check(rc, "interpolate_lines")
    return outs
