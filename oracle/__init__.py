"""CPU oracle for the Partia LBVH build + SPH grid interpolation path.

TEST INFRASTRUCTURE ONLY.  A ctypes wrapper over ``libpartia_oracle.so`` (plain C,
FP64, OpenMP), the restatement of the reference algorithm that the tests and the
CPU-baseline leg of ``bench.py`` use as the checker.  The product path never imports
this package.  See ``partia_oracle.c`` for the reference files each part follows and
for the pinning status of the restatement.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libpartia_oracle.so")
_lib = None

KERNELS = {"M4_spline": 0, "M5_spline": 1, "M6_spline": 2, "C2_Wendland": 3, "C4_Wendland": 4, "C6_Wendland": 5}
STRATEGIES = {"itpGather": 0, "itpScatter": 1, "itpSymmetric": 2}

_dp = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u64p = ctypes.POINTER(ctypes.c_uint64)


class _Tree(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("root", ctypes.c_int32),
                ("x", _dp), ("y", _dp), ("z", _dp), ("h", _dp),
                ("left", _i32p), ("right", _i32p), ("escape", _i32p),
                ("bmin", _dp), ("bmax", _dp), ("hmax", _dp),
                ("m", _dp), ("rho", _dp), ("ncol", ctypes.c_int32),
                ("quant", ctypes.POINTER(_dp)), ("kernel", ctypes.c_int32)]


class _Catalog(ctypes.Structure):
    _fields_ = [("n_scalar", ctypes.c_int32), ("scalar_cols", _i32p), ("scalar_shepard", _i32p),
                ("n_grad", ctypes.c_int32), ("grad_cols", _i32p),
                ("n_div", ctypes.c_int32), ("div_cols", _i32p),
                ("n_curl", ctypes.c_int32), ("curl_cols", _i32p)]


def build_library():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build_library()
        L = ctypes.CDLL(_LIB)
        for name in ("orc_kernel_f", "orc_kernel_df"):
            getattr(L, name).restype = ctypes.c_double
            getattr(L, name).argtypes = [ctypes.c_int32, ctypes.c_double]
        for name in ("orc_kernel_norm3", "orc_kernel_valid"):
            getattr(L, name).restype = ctypes.c_double
            getattr(L, name).argtypes = [ctypes.c_int32]
        L.orc_W.restype = ctypes.c_double
        L.orc_W.argtypes = [ctypes.c_int32, ctypes.c_double, ctypes.c_double]
        L.orc_line_W.restype = ctypes.c_double
        L.orc_line_W.argtypes = [ctypes.c_int32, ctypes.c_double, ctypes.c_double]
        L.orc_gradW.restype = None
        L.orc_gradW.argtypes = [ctypes.c_int32] + [ctypes.c_double] * 4 + [_dp]
        L.orc_jl_pow.restype = ctypes.c_double
        L.orc_jl_pow.argtypes = [ctypes.c_double, ctypes.c_int64]
        L.orc_build.restype = ctypes.c_int
        L.orc_build.argtypes = [ctypes.c_int64] + [_dp] * 4 + [_u64p, _i64p] + [_dp] * 4 + [_i32p] * 4 + [_dp] * 3 + [_i32p]
        L.orc_find_nearest_h.restype = ctypes.c_double
        L.orc_find_nearest_h.argtypes = [ctypes.POINTER(_Tree)] + [ctypes.c_double] * 3 + [_i64p]
        L.orc_query.restype = ctypes.c_int64
        L.orc_query.argtypes = [ctypes.POINTER(_Tree)] + [ctypes.c_double] * 4 + [_i64p, ctypes.c_int64, _i64p]
        L.orc_probe_neighbors.restype = ctypes.c_int64
        L.orc_probe_neighbors.argtypes = [ctypes.POINTER(_Tree)] + [ctypes.c_double] * 4 + [_i64p, _dp]
        L.orc_interp_points.restype = None
        L.orc_interp_points.argtypes = [ctypes.POINTER(_Tree), ctypes.POINTER(_Catalog), ctypes.c_int64,
                                        _dp, _dp, _dp, ctypes.c_int32, _dp, ctypes.c_int32, _i64p]
        L.orc_interp_lines.restype = None
        L.orc_interp_lines.argtypes = [ctypes.POINTER(_Tree), ctypes.POINTER(_Catalog), ctypes.c_int64,
                                       _dp, _dp, _dp, _dp, _dp, _dp, _dp, ctypes.c_int32, _i64p]
        L.orc_max_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ---------------------------------------------------------------------------------------
# kernel functions
def kernel_f(k, q):
    return lib().orc_kernel_f(KERNELS.get(k, k), float(q))


def kernel_df(k, q):
    return lib().orc_kernel_df(KERNELS.get(k, k), float(q))


def kernel_norm3(k):
    return lib().orc_kernel_norm3(KERNELS.get(k, k))


def kernel_valid(k):
    return lib().orc_kernel_valid(KERNELS.get(k, k))


def W(k, r, h):
    return lib().orc_W(KERNELS.get(k, k), float(r), float(h))


def line_W(k, r, h):
    return lib().orc_line_W(KERNELS.get(k, k), float(r), float(h))


def gradW(k, dx, dy, dz, h):
    g = np.zeros(3)
    lib().orc_gradW(KERNELS.get(k, k), float(dx), float(dy), float(dz), float(h), _p(g))
    return tuple(g)


def jl_pow(x, n):
    return lib().orc_jl_pow(float(x), int(n))


# ---------------------------------------------------------------------------------------
class OracleLBVH:
    """Result of the oracle build: sorted codes/order, topology, boxes (reference layout)."""

    def __init__(self, x, y, z, h):
        x, y, z, h = (_f64(a) for a in (x, y, z, h))
        n = len(x)
        self.n = n
        self.codes = np.zeros(n, np.uint64)
        self.order = np.zeros(n, np.int64)
        self.x, self.y, self.z, self.h = (np.zeros(n) for _ in range(4))
        nt = max(2 * n - 1, 1)
        self.left, self.right, self.escape, self.parent = (np.zeros(nt, np.int32) for _ in range(4))
        nin = max(n - 1, 1)
        self.bmin = np.zeros(3 * nin)
        self.bmax = np.zeros(3 * nin)
        self.hmax = np.zeros(nin)
        root = ctypes.c_int32(0)
        rc = lib().orc_build(n, _p(x), _p(y), _p(z), _p(h), _p(self.codes, _u64p), _p(self.order, _i64p),
                             _p(self.x), _p(self.y), _p(self.z), _p(self.h),
                             _p(self.left, _i32p), _p(self.right, _i32p), _p(self.escape, _i32p),
                             _p(self.parent, _i32p), _p(self.bmin), _p(self.bmax), _p(self.hmax),
                             ctypes.byref(root))
        if rc != 0:
            raise RuntimeError("oracle build failed (%d)" % rc)
        self.root = root.value
        self._fields = None

    def attach(self, m, rho, quant, kernel="M4_spline"):
        """Permute particle fields by the build order (LinearBVH! side effect) and keep them."""
        o = self.order
        self.m = _f64(np.asarray(m)[o])
        self.rho = _f64(np.asarray(rho)[o])
        self.quant = [_f64(np.asarray(q)[o]) for q in quant]
        self.kernel = KERNELS.get(kernel, kernel)
        return self

    def _tree(self):
        qarr = (_dp * max(len(self.quant), 1))(*[_p(q) for q in self.quant])
        t = _Tree(self.n, self.root, _p(self.x), _p(self.y), _p(self.z), _p(self.h),
                  _p(self.left, _i32p), _p(self.right, _i32p), _p(self.escape, _i32p),
                  _p(self.bmin), _p(self.bmax), _p(self.hmax), _p(self.m), _p(self.rho),
                  len(self.quant), ctypes.cast(qarr, ctypes.POINTER(_dp)), self.kernel)
        t._keep = qarr
        return t

    def _geom_tree(self):
        if not hasattr(self, "m"):
            z = np.zeros(self.n)
            self.attach(z, np.ones(self.n), [], 0)
        return self._tree()

    def find_nearest_h(self, p):
        best = ctypes.c_int64(-1)
        t = self._geom_tree()
        hv = lib().orc_find_nearest_h(ctypes.byref(t), float(p[0]), float(p[1]), float(p[2]), ctypes.byref(best))
        return hv, best.value

    def query(self, p, radius):
        t = self._geom_tree()
        pool = np.zeros(self.n, np.int64)
        nearest = ctypes.c_int64(-1)
        cnt = lib().orc_query(ctypes.byref(t), float(p[0]), float(p[1]), float(p[2]), float(radius),
                              _p(pool, _i64p), self.n, ctypes.byref(nearest))
        return pool[:cnt].copy(), nearest.value

    def probe_neighbors(self, p, radius):
        """LBVH_probe_neighbors: (count, closest 0-based index or -1, closest d2 or +Inf)."""
        t = self._geom_tree()
        ci = ctypes.c_int64(-1)
        cd = ctypes.c_double(0.0)
        cnt = lib().orc_probe_neighbors(ctypes.byref(t), float(p[0]), float(p[1]), float(p[2]), float(radius),
                                        ctypes.byref(ci), ctypes.byref(cd))
        return cnt, ci.value, cd.value

    def interp_points(self, catalog, qx, qy, qz, strategy="itpSymmetric", nthreads=0, stats=False):
        qx, qy, qz = _f64(qx), _f64(qy), _f64(qz)
        npts = len(qx)
        c, keep = _catalog(catalog)
        L = catalog_L(catalog)
        out = np.zeros((L, npts))
        st = np.zeros((npts, 5), np.int64) if stats else None
        t = self._tree()
        lib().orc_interp_points(ctypes.byref(t), ctypes.byref(c), npts, _p(qx), _p(qy), _p(qz),
                                STRATEGIES.get(strategy, strategy), _p(out), int(nthreads),
                                _p(st, _i64p) if stats else None)
        return (out, st) if stats else out

    def interp_lines(self, catalog, origin, direction, nthreads=0, stats=False):
        o = [_f64(a) for a in origin]
        d = [_f64(a) for a in direction]
        nl = len(o[0])
        c, keep = _catalog(catalog)
        out = np.zeros((len(catalog["scalar_cols"]), nl))
        st = np.zeros((nl, 3), np.int64) if stats else None
        t = self._tree()
        lib().orc_interp_lines(ctypes.byref(t), ctypes.byref(c), nl, _p(o[0]), _p(o[1]), _p(o[2]),
                               _p(d[0]), _p(d[1]), _p(d[2]), _p(out), int(nthreads),
                               _p(st, _i64p) if stats else None)
        return (out, st) if stats else out


def catalog_L(cat):
    return (len(cat["scalar_cols"]) + 3 * len(cat.get("grad_cols", ())) + len(cat.get("div_cols", ()))
            + 3 * len(cat.get("curl_cols", ())))


def _catalog(cat):
    """cat: dict with scalar_cols, scalar_shepard, grad_cols (-1 = density), div_cols [(cx,cy,cz)],
    curl_cols [(cx,cy,cz)]; all column indices 0-based."""
    sc = np.ascontiguousarray(cat["scalar_cols"], np.int32).reshape(-1)
    sh = np.ascontiguousarray(cat.get("scalar_shepard", [1] * len(sc)), np.int32).reshape(-1)
    gc = np.ascontiguousarray(cat.get("grad_cols", []), np.int32).reshape(-1)
    dc = np.ascontiguousarray(cat.get("div_cols", []), np.int32).reshape(-1)
    cc = np.ascontiguousarray(cat.get("curl_cols", []), np.int32).reshape(-1)
    keep = [np.zeros(1, np.int32) if len(a) == 0 else a for a in (sc, sh, gc, dc, cc)]
    c = _Catalog(len(sc), _p(keep[0], _i32p), _p(keep[1], _i32p), len(gc), _p(keep[2], _i32p),
                 len(dc) // 3, _p(keep[3], _i32p), len(cc) // 3, _p(keep[4], _i32p))
    return c, keep


def max_threads():
    return lib().orc_max_threads()
