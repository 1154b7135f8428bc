"""Partia's neighbour-search entry points on the device-resident LBVH.

  LinearBVH_build(input)   LinearBVH!(input, Val(3))  InterpolationInput.jl:203-223
  LinearBVH.encoding()     MortonEncoding codes/order MortonCode.jl:8-13,38-45
  LinearBVH.tree()         BinaryRadixTree + LinearBVH arrays  BinaryRadixTree.jl:8-15, LinearBVH.jl:20-26
  LBVH_find_nearest_h      LinearBVHQueries.jl:118-140 (batched)
  LBVH_find_nearest        LinearBVHQueries.jl:79-95 (batched; leaf index)
  LBVH_query               LBVH_query! LinearBVHQueries.jl:183-211 + NeighborSelection.jl:1-23 (batched)
  LBVH_probe_neighbors     LinearBVHQueries.jl:22-42 (batched)

Indices are 0-based (Julia's are 1-based); node ids keep the reference's unified
1-based id space.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import ArgumentError, ptr
from .interpolation import CUDAComputeBackend, InterpolationInput


class NeighborSelection:
    """Accepted 0-based sorted leaf indices (DFS order), their count and the nearest one (-1 if none)."""

    def __init__(self, pool, count, nearest):
        self.pool = pool
        self.count = int(count)
        self.nearest = int(nearest)

    def __len__(self):
        return self.count

    def valid_indices(self):
        return self.pool[:self.count]

    def nearest_index(self):
        return self.nearest


class LinearBVH:
    """Handle on the LBVH last built by LinearBVH_build on a backend."""

    def __init__(self, backend, n):
        self.backend = backend
        self.handle = backend.handle
        self.nleaf = int(n)

    def encoding(self):
        n = self.nleaf
        codes = np.empty(n, np.uint64)
        order = np.empty(n, np.int64)
        H = self.handle
        H.check(H.lib.pb_export_encoding(H.h, codes.ctypes.data, order.ctypes.data), "export_encoding")
        return codes, order

    def tree(self):
        n = self.nleaf
        nt, nin = 2 * n - 1, max(n - 1, 1)
        out = {k: np.zeros(nt, np.int32) for k in ("left", "right", "escape", "parent")}
        out["bmin"] = np.zeros(3 * nin)
        out["bmax"] = np.zeros(3 * nin)
        out["hmax"] = np.zeros(nin)
        root = ctypes.c_int32()
        H = self.handle
        rc = H.lib.pb_export_tree(H.h, *[out[k].ctypes.data for k in ("left", "right", "escape", "parent", "bmin",
                                                                      "bmax", "hmax")], ctypes.byref(root))
        H.check(rc, "export_tree")
        out["root"] = root.value
        return out


def LinearBVH_build(input, backend=None, permute_input=True):
    """LinearBVH!(input, Val(3)): build the LBVH on the device; with ``permute_input`` the
    caller's particle columns are permuted in place into Morton order, as the reference does."""
    if backend is None:
        backend = CUDAComputeBackend()
    if not isinstance(input, InterpolationInput):
        raise ArgumentError("input must be an InterpolationInput")
    H = backend.handle
    cin = input._c_struct()
    H.check(H.lib.pb_linear_bvh(H.h, ctypes.byref(cin), _lib.PB_PERMUTE_CALLER if permute_input else 0),
            "LinearBVH!")
    return LinearBVH(backend, input.Npart)


def MortonEncoding(x, y, z, h=None, backend=None):
    """Sorted Morton codes (after the duplicate bump) and the 0-based sorting order."""
    x = np.ascontiguousarray(x, np.float64)
    n = len(x)
    h = np.zeros(n) if h is None else np.ascontiguousarray(h, np.float64)
    one = np.ones(n)
    inp = InterpolationInput(x.copy(), np.ascontiguousarray(y, np.float64).copy(),
                             np.ascontiguousarray(z, np.float64).copy(), one.copy(), h.copy(), one.copy(), ())
    return LinearBVH_build(inp, backend, permute_input=False).encoding()


def _pts(points):
    return [np.ascontiguousarray(p, np.float64) if not hasattr(p, "data_ptr") else p for p in points]


def LBVH_find_nearest_h(lbvh, points):
    """Smoothing length of the nearest leaf to every point (NaN only for an empty tree)."""
    qx, qy, qz = _pts(points)
    n = len(qx)
    hout = np.empty(n)
    H = lbvh.handle
    H.check(H.lib.pb_find_nearest_h(H.h, n, ptr(qx), ptr(qy), ptr(qz), hout.ctypes.data, None), "LBVH_find_nearest_h")
    return hout


def LBVH_find_nearest(lbvh, points):
    """0-based sorted leaf index of the nearest leaf to every point (ties: smallest index)."""
    qx, qy, qz = _pts(points)
    n = len(qx)
    idx = np.empty(n, np.int64)
    H = lbvh.handle
    H.check(H.lib.pb_find_nearest_h(H.h, n, ptr(qx), ptr(qy), ptr(qz), None, idx.ctypes.data), "LBVH_find_nearest")
    return idx


def traversal_stats(lbvh, points, itp_strategy):
    """Per-point event counts of the reference traversal (nearest internal visits, nearest leaf
    tests, main internal visits, main leaf tests, accepted neighbours) as an (N, 5) int64 array."""
    qx, qy, qz = _pts(points)
    n = len(qx)
    st = np.empty((n, 5), np.int64)
    H = lbvh.handle
    H.check(H.lib.pb_traversal_stats(H.h, n, ptr(qx), ptr(qy), ptr(qz), itp_strategy.code, st.ctypes.data),
            "traversal_stats")
    return st


def LBVH_query(lbvh, points, radius):
    """Batched LBVH_query!: one NeighborSelection per point (radius scalar or per point)."""
    qx, qy, qz = _pts(points)
    n = len(qx)
    r = np.broadcast_to(np.asarray(radius, np.float64), (n,)).copy()
    counts = np.empty(n, np.int64)
    H = lbvh.handle
    H.check(H.lib.pb_query_count(H.h, n, ptr(qx), ptr(qy), ptr(qz), r.ctypes.data, counts.ctypes.data), "LBVH_query!")
    offsets = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=offsets[1:])
    pool = np.empty(max(int(offsets[-1]), 1), np.int64)
    nearest = np.empty(n, np.int64)
    H.check(H.lib.pb_query_neighbors(H.h, n, ptr(qx), ptr(qy), ptr(qz), r.ctypes.data, offsets.ctypes.data,
                                     pool.ctypes.data, nearest.ctypes.data), "LBVH_query!")
    return [NeighborSelection(pool[offsets[i]:offsets[i + 1]], counts[i], nearest[i]) for i in range(n)]


def LBVH_probe_neighbors(lbvh, points, radius):
    """Batched LBVH_probe_neighbors: for every point the number of leaves within ``radius``
    (d2 <= radius^2), the 0-based index of the closest of them (-1 if none; the reference's 0)
    and its squared distance (+Inf if none; the reference's typemax).  Returns three arrays."""
    qx, qy, qz = _pts(points)
    n = len(qx)
    r = np.broadcast_to(np.asarray(radius, np.float64), (n,)).copy()
    count = np.empty(n, np.int64)
    idx = np.empty(n, np.int64)
    d2 = np.empty(n)
    H = lbvh.handle
    H.check(H.lib.pb_probe_neighbors(H.h, n, ptr(qx), ptr(qy), ptr(qz), r.ctypes.data, count.ctypes.data,
                                     idx.ctypes.data, d2.ctypes.data), "LBVH_probe_neighbors")
    return count, idx, d2
