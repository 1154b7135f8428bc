"""ctypes binding of libpartia_b200.so (the C ABI declared in include/partia_b200.h).

The library is built in-tree by ``_build.py``.  Loading fails loudly when it is missing
or when no CUDA device is usable: there is no CPU fallback for the hot path.
"""
import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libpartia_b200.so")

PB_OK = 0
PB_ERR_INVALID = -1
PB_ERR_CAPACITY = -2
PB_ERR_CUDA = -3
PB_ERR_STATE = -4
PB_ERR_INTERNAL = -6
PB_ERR_KEY = -7
PB_ERR_DIMENSION = -8
PB_FP64 = 0
PB_FP32C = 1
PB_PERMUTE_CALLER = 1
PB_BUILD_ASYNC = 2
PB_BATCH_ASYNC = 1

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_lp = ctypes.POINTER(ctypes.c_int64)
_up = ctypes.POINTER(ctypes.c_uint64)
_vp = ctypes.c_void_p


class ArgumentError(ValueError):
    """Julia's ArgumentError (invalid argument values)."""


class DimensionMismatch(ValueError):
    """Julia's DimensionMismatch (length mismatch between columns)."""


class CapacityError(ArgumentError):
    """n exceeds the Int32 node-id capacity (n <= 2^30)."""


class DeviceError(RuntimeError):
    """CUDA runtime failure or a failed device-side consistency check."""


class PBInput(ctypes.Structure):
    _fields_ = [("npart", ctypes.c_int64),
                ("x", _vp), ("y", _vp), ("z", _vp), ("m", _vp), ("h", _vp), ("rho", _vp),
                ("ncolumn", ctypes.c_int32), ("quant", ctypes.POINTER(_vp)), ("kernel", ctypes.c_int32)]


class PBCatalog(ctypes.Structure):
    _fields_ = [("n_scalar", ctypes.c_int32), ("scalar_cols", _ip), ("scalar_shepard", _ip),
                ("n_grad", ctypes.c_int32), ("grad_cols", _ip),
                ("n_div", ctypes.c_int32), ("div_cols", _ip),
                ("n_curl", ctypes.c_int32), ("curl_cols", _ip)]


EXPORTED = ["pb_create", "pb_destroy", "pb_last_error", "pb_set_stream", "pb_set_option", "pb_linear_bvh",
            "pb_export_encoding", "pb_export_tree", "pb_find_nearest_h", "pb_query_count", "pb_query_neighbors",
            "pb_probe_neighbors", "pb_traversal_stats",
            "pb_interpolate_points", "pb_interpolate_lines", "pb_point_samples_interpolation",
            "pb_line_samples_interpolation", "pb_launch_count", "pb_last_timings", "pb_morton_sort_noalloc",
            "pb_last_schedule", "pb_last_pair_split", "pb_scheduler_features", "pb_scheduler_set", "pb_scheduler_get",
            "pb_scheduler_predict", "pb_scheduler_gradients", "pb_scheduler_train", "pb_grid_points", "pb_line_image",
            "pb_column_to_f64", "pb_fill_f64", "pb_density_from_h", "pb_batch_points", "pb_batch_check"]

SCHED_FEATURES = 16
SCHED_PARAMS = 5313

_lib = None


def load():
    """Load the shared library and declare every entry point's signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libpartia_b200.so is not built (run distorteddustydiscanalysistoolkits_b200/_build.py); "
                          "the CUDA path has no CPU fallback")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    sig = {
        "pb_create": (ctypes.c_int32, [P(_vp), ctypes.c_int32]),
        "pb_destroy": (None, [_vp]),
        "pb_last_error": (ctypes.c_int32, [_vp, ctypes.c_char_p, ctypes.c_int64]),
        "pb_set_stream": (ctypes.c_int32, [_vp, _vp]),
        "pb_set_option": (ctypes.c_int32, [_vp, ctypes.c_char_p, ctypes.c_int64]),
        "pb_linear_bvh": (ctypes.c_int32, [_vp, P(PBInput), ctypes.c_int32]),
        "pb_export_encoding": (ctypes.c_int32, [_vp, _vp, _vp]),
        "pb_export_tree": (ctypes.c_int32, [_vp] + [_vp] * 7 + [_ip]),
        "pb_find_nearest_h": (ctypes.c_int32, [_vp, ctypes.c_int64, _vp, _vp, _vp, _vp, _vp]),
        "pb_query_count": (ctypes.c_int32, [_vp, ctypes.c_int64, _vp, _vp, _vp, _vp, _vp]),
        "pb_query_neighbors": (ctypes.c_int32, [_vp, ctypes.c_int64, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
        "pb_probe_neighbors": (ctypes.c_int32, [_vp, ctypes.c_int64, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
        "pb_traversal_stats": (ctypes.c_int32, [_vp, ctypes.c_int64, _vp, _vp, _vp, ctypes.c_int32, _vp]),
        "pb_interpolate_points": (ctypes.c_int32, [_vp, P(PBCatalog), ctypes.c_int64, _vp, _vp, _vp,
                                                   ctypes.c_int32, ctypes.c_int32, P(_vp)]),
        "pb_interpolate_lines": (ctypes.c_int32, [_vp, P(PBCatalog), ctypes.c_int64] + [_vp] * 6 +
                                 [ctypes.c_int32, ctypes.c_int32, P(_vp)]),
        "pb_point_samples_interpolation": (ctypes.c_int32, [_vp, P(PBInput), P(PBCatalog), ctypes.c_int64,
                                                            _vp, _vp, _vp, ctypes.c_int32, ctypes.c_int32,
                                                            P(_vp), ctypes.c_int32]),
        "pb_line_samples_interpolation": (ctypes.c_int32, [_vp, P(PBInput), P(PBCatalog), ctypes.c_int64] +
                                          [_vp] * 6 + [ctypes.c_int32, ctypes.c_int32, P(_vp), ctypes.c_int32]),
        "pb_launch_count": (ctypes.c_int64, [_vp]),
        "pb_last_timings": (ctypes.c_int32, [_vp, _dp, _dp, _lp]),
        "pb_last_schedule": (ctypes.c_int32, [_vp, _lp, _lp, _lp, _dp]),
        "pb_last_pair_split": (ctypes.c_int32, [_vp, _lp, _lp, _lp, _lp]),
        "pb_grid_points": (ctypes.c_int32, [_vp, ctypes.c_int32, _vp, ctypes.c_int64, _vp, ctypes.c_int64, _vp,
                                            ctypes.c_int64, _vp, _vp, _vp]),
        "pb_line_image": (ctypes.c_int32, [_vp, _vp, ctypes.c_int64, _vp, ctypes.c_int64, _vp] + [_vp] * 6),
        "pb_batch_points": (ctypes.c_int32, [P(_vp), ctypes.c_int32, P(PBCatalog), _vp, _vp, _vp, _vp, _vp,
                                             ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
        "pb_batch_check": (ctypes.c_int32, [P(_vp), ctypes.c_int32]),
        "pb_column_to_f64": (ctypes.c_int32, [_vp, _vp, ctypes.c_int32, ctypes.c_int64, _vp]),
        "pb_fill_f64": (ctypes.c_int32, [_vp, ctypes.c_double, ctypes.c_int64, _vp]),
        "pb_density_from_h": (ctypes.c_int32, [_vp, _vp, ctypes.c_int64, ctypes.c_double, ctypes.c_double, _vp]),
        "pb_scheduler_features": (ctypes.c_int32, [_vp, ctypes.c_int64, _vp, _vp, _vp, _vp]),
        "pb_scheduler_set": (ctypes.c_int32, [_vp, _vp, _vp, ctypes.c_float, ctypes.c_int32]),
        "pb_scheduler_get": (ctypes.c_int32, [_vp, _vp]),
        "pb_scheduler_predict": (ctypes.c_int32, [_vp, _vp, ctypes.c_int64, _vp]),
        "pb_scheduler_gradients": (ctypes.c_int32, [_vp, _vp, _vp, ctypes.c_int64, _vp, _vp]),
        "pb_scheduler_train": (ctypes.c_int32, [_vp, _vp, _vp, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                                ctypes.c_float, ctypes.c_uint64, _vp]),
        "pb_morton_sort_noalloc": (ctypes.c_int32, [_vp, _vp, _vp, ctypes.c_int64, _vp, _vp, _vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def ptr(a):
    """Address of a contiguous float64/int array (numpy, or a torch tensor on any device)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr") and hasattr(a, "is_contiguous"):
        if not a.is_contiguous():
            raise ArgumentError("tensor must be contiguous")
        return a.data_ptr()
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ArgumentError("array must be C-contiguous")
        return a.ctypes.data
    raise ArgumentError("unsupported array type %r" % type(a))


class Handle:
    """Owns one pb_handle (device buffers of one particle set stay resident between calls)."""

    def __init__(self, device=0):
        self.lib = load()
        h = _vp()
        rc = self.lib.pb_create(ctypes.byref(h), int(device))
        if rc != PB_OK:
            raise DeviceError("pb_create(device=%d) failed (%d): no usable CUDA device" % (device, rc))
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            self.lib.pb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def error(self):
        buf = ctypes.create_string_buffer(4096)
        self.lib.pb_last_error(self.h, buf, 4096)
        return buf.value.decode(errors="replace")

    def check(self, rc, what):
        if rc == PB_OK:
            return
        msg = "%s: %s" % (what, self.error())
        if rc == PB_ERR_CAPACITY:
            raise CapacityError(msg)
        if rc == PB_ERR_KEY:
            raise KeyError(msg)
        if rc == PB_ERR_DIMENSION:
            raise DimensionMismatch(msg)
        if rc == PB_ERR_INVALID:
            raise ArgumentError(msg)
        if rc == PB_ERR_STATE:
            raise ArgumentError(msg)
        raise DeviceError(msg)

    def set_option(self, name, value):
        self.check(self.lib.pb_set_option(self.h, name.encode(), int(value)), "pb_set_option")

    def set_stream(self, stream_ptr):
        self.check(self.lib.pb_set_stream(self.h, stream_ptr), "pb_set_stream")

    def launch_count(self):
        return self.lib.pb_launch_count(self.h)

    def timings(self):
        b, i, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
        self.lib.pb_last_timings(self.h, ctypes.byref(b), ctypes.byref(i), ctypes.byref(n))
        return b.value, i.value, n.value

    def schedule(self):
        """(walk rounds, deferred queries, pool chunks) of the last FP32-compensated point call."""
        r, d, c = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        self.lib.pb_last_schedule(self.h, ctypes.byref(r), ctypes.byref(d), ctypes.byref(c), None)
        return r.value, d.value, c.value

    def pair_split(self):
        """(heavy queries, light queries, heavy pairs, light pairs) of the last point call: heavy
        queries were summed by the FP32-compensated pair kernel, light ones by the FP64 one."""
        v = [ctypes.c_int64() for _ in range(4)]
        self.lib.pb_last_pair_split(self.h, *[ctypes.byref(x) for x in v])
        return tuple(x.value for x in v)

    def phase_times(self):
        """Device ms of the nearest search, walk and pair sums, summed over slices and rounds (option "timing")."""
        t = (ctypes.c_double * 3)()
        self.lib.pb_last_schedule(self.h, None, None, None, t)
        return tuple(t)
