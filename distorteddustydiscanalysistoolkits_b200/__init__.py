"""B200-native (sm_100a) implementation of Partia.jl's LBVH build + SPH grid interpolation path.

The hot path runs in libpartia_b200.so (hand-written CUDA kernels behind a C ABI, see
include/partia_b200.h).  This package is the host-side mirror of Partia's interface for
that path: grids, interpolation inputs/catalogs, the CUDA backend's interpolation entry
points and the neighbour-search queries.
"""
__version__ = "0.2.0"

from ._lib import ArgumentError, CapacityError, DeviceError, DimensionMismatch
from .grids import (Cartesian, Cylindrical, GridBundle, LineSamples, PointSamples, Polar, Spherical,
                    StructuredGrid, coordinate_grid, flatten, restore_struct)
from .interpolation import (C2_Wendland, C4_Wendland, C6_Wendland, CUDAComputeBackend, FP32C, FP64,
                            Greeting_CUDA, InterpolationCatalog, InterpolationInput, KernelFunctionValid, M4_spline,
                            M5_spline, M6_spline, LineSamples_image, LineSamples_interpolation, PointSamples_interpolation,
                            StructuredGrid_interpolation, build_input, interpolate_lines, interpolate_points,
                            itpGather, itpScatter, itpSymmetric)
from .neighbor import (LBVH_find_nearest, LBVH_find_nearest_h, LBVH_probe_neighbors, LBVH_query, LinearBVH,
                       LinearBVH_build,
                       MortonEncoding, NeighborSelection, traversal_stats)

from . import phantom
from .phantom import MassFromColumn, MassFromParams, ParticleDataFrame, add_rho, read_phantom
from . import gridio
from .gridio import GridDataset, read_GridDataset, write_GridBundle, write_GridDataset

__all__ = [n for n in dir() if not n.startswith("_")]
