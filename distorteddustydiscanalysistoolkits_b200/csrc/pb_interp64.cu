// pb_interp64.cu -- FP64 point/line interpolation kernels (reference arithmetic).
// Compiled with -fmad=false so that every expression is the IEEE result of the
// reference's operation order (no FMA contraction).
#include "line_tables.h"
#include "pb_internal.h"
#include "pb_interp_impl.cuh"

namespace pb {

__device__ const double g_line_inorm64[6][PB_LINE_NTAB] = PB_LINE_INORM_INIT;

cudaError_t launch_points_fp64(Handle *H, const DevTree &T, const DevCatalog &C, int strategy, int64_t nq,
                               const double *qx, const double *qy, const double *qz, const uint32_t *perm)
{
    int bs = 128;
    int grid = grid_for(nq, bs, 1 << 30);
    switch (strategy) {
    case GATHER: k_points<Exact64, GATHER><<<grid, bs, 0, H->stream>>>(T, C, nq, qx, qy, qz, perm); break;
    case SCATTER: k_points<Exact64, SCATTER><<<grid, bs, 0, H->stream>>>(T, C, nq, qx, qy, qz, perm); break;
    default: k_points<Exact64, SYMMETRIC><<<grid, bs, 0, H->stream>>>(T, C, nq, qx, qy, qz, perm); break;
    }
    H->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_lines_fp64(Handle *H, const DevTree &T, const DevCatalog &C, int64_t nl, const double *ox,
                              const double *oy, const double *oz, const double *dx, const double *dy,
                              const double *dz, const uint32_t *perm)
{
    const double *tab = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&tab, g_line_inorm64);
    if (e) return e;
    int bs = 128;
    k_lines<double><<<grid_for(nl, bs, 1 << 30), bs, 0, H->stream>>>(T, C, nl, ox, oy, oz, dx, dy, dz, perm, tab);
    H->launches += 1;
    return cudaGetLastError();
}

}  // namespace pb
