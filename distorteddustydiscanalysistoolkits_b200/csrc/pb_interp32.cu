// pb_interp32.cu -- FP32-compensated point/line interpolation kernels (same neighbour
// sets as the FP64 path; FP32 kernel sums with TwoSum compensation and offsets).
#include "line_tables.h"
#include "pb_internal.h"
#include "pb_interp_impl.cuh"

namespace pb {

__device__ const float g_line_inorm32[6][PB_LINE_NTAB] = PB_LINE_INORM_INIT;

cudaError_t launch_points_fp32(Handle *H, const DevTree &T, const DevCatalog &C, int strategy, int64_t nq,
                               const double *qx, const double *qy, const double *qz, const uint32_t *perm)
{
    int bs = 128;
    int grid = grid_for(nq, bs, 1 << 30);
    switch (strategy) {
    case GATHER: k_points<Comp32, GATHER><<<grid, bs, 0, H->stream>>>(T, C, nq, qx, qy, qz, perm); break;
    case SCATTER: k_points<Comp32, SCATTER><<<grid, bs, 0, H->stream>>>(T, C, nq, qx, qy, qz, perm); break;
    default: k_points<Comp32, SYMMETRIC><<<grid, bs, 0, H->stream>>>(T, C, nq, qx, qy, qz, perm); break;
    }
    H->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_lines_fp32(Handle *H, const DevTree &T, const DevCatalog &C, int64_t nl, const double *ox,
                              const double *oy, const double *oz, const double *dx, const double *dy,
                              const double *dz, const uint32_t *perm)
{
    const float *tab = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&tab, g_line_inorm32);
    if (e) return e;
    int bs = 128;
    k_lines<float><<<grid_for(nl, bs, 1 << 30), bs, 0, H->stream>>>(T, C, nl, ox, oy, oz, dx, dy, dz, perm, tab);
    H->launches += 1;
    return cudaGetLastError();
}

}  // namespace pb
