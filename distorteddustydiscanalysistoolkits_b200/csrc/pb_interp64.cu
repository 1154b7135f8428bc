// pb_interp64.cu -- FP64 point/line interpolation kernels (reference arithmetic).
// Compiled with -fmad=false so that every expression is the IEEE result of the
// reference's operation order (no FMA contraction).
#include "line_tables.h"
#include "pb_internal.h"
#include "pb_fp64_impl.cuh"

namespace pb {

__device__ const double g_line_inorm64[6][PB_LINE_NTAB] = PB_LINE_INORM_INIT;


template <int STRAT>
__global__ void __launch_bounds__(128) k_points64w(DevTree T, DevCatalog C, int64_t nq, const double *__restrict__ qx,
                                                   const double *__restrict__ qy, const double *__restrict__ qz,
                                                   const uint32_t *__restrict__ perm, int64_t npts,
                                                   unsigned long long *counter)
{
    __shared__ double sterm[4][32][NT + 1];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    for (;;) {
        int64_t j = next_query(counter, lane);
        if (j >= nq) break;
        int64_t qi = perm ? (int64_t)__ldg(perm + j) : j;
        if (qi >= npts) continue;
        const double px = __ldg(qx + qi), py = __ldg(qy + qi), pz = __ldg(qz + qi);
        const int64_t bnear = STRAT != SCATTER ? nearest_leaf(T, px, py, pz) : -1;
        points64_query<STRAT>(T, C, px, py, pz, bnear, qi, &sterm[wib][0][0], lane, 1);
    }
}

// Two-phase form: the warp reads the walked query's runs (deal_runs) instead of walking, with
// the same per-slot terms and the same in-order column sums, so the values are those of
// k_points64w bit for bit.
template <int STRAT>
__global__ void __launch_bounds__(128) k_pairs64w(DevTree T, DevCatalog C, RunPool P, int64_t m,
                                                  const uint32_t *__restrict__ ql, const uint32_t *__restrict__ order,
                                                  const double *__restrict__ qx, const double *__restrict__ qy,
                                                  const double *__restrict__ qz, unsigned long long *counter)
{
    __shared__ double sterm[4][32][NT + 1];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    // the next query's position in the order is fetched (lane 0's atomic) while the current
    // one is summed, so the counter's latency overlaps the work; which warp sums a query does
    // not change its value
    unsigned long long nxt = 0;
    if (lane == 0) nxt = atomicAdd(counter, 1ULL);
    int64_t t = (int64_t)__shfl_sync(0xffffffffu, nxt, 0);
    while (t < m) {
        if (lane == 0) nxt = atomicAdd(counter, 1ULL);
        const int64_t j = order ? (int64_t)__ldg(order + t) : t;
        if (!__ldg(P.qflag + j)) {
            const int64_t qi = __ldg(ql + j);
            const double px = __ldg(qx + qi), py = __ldg(qy + qi), pz = __ldg(qz + qi);
            pairs64_query<STRAT>(T, C, P, j, qi, px, py, pz, STRAT != SCATTER ? (int64_t)__ldg(P.bnear + j) : -1,
                                 &sterm[wib][0][0], lane);
        }
        t = (int64_t)__shfl_sync(0xffffffffu, nxt, 0);
    }
}

static int persistent_grid(const void *kern, int bs)
{
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, bs, 0);
    return sms * (per > 0 ? per : 1);
}

cudaError_t launch_points_fp64(Handle *H, const DevTree &T, const DevCatalog &C, int strategy, int64_t nq,
                               const double *qx, const double *qy, const double *qz, const uint32_t *perm,
                               int64_t npts)
{
    int bs = 128;
    cudaError_t e = H->counter.reserve(sizeof(unsigned long long));
    if (e) return e;
    unsigned long long *ctr = H->counter.as<unsigned long long>();
    cudaMemsetAsync(ctr, 0, sizeof(unsigned long long), H->stream);
    switch (strategy) {
    case GATHER:
        k_points64w<GATHER><<<persistent_grid((const void *)k_points64w<GATHER>, bs), bs, 0, H->stream>>>(
            T, C, nq, qx, qy, qz, perm, npts, ctr);
        break;
    case SCATTER:
        k_points64w<SCATTER><<<persistent_grid((const void *)k_points64w<SCATTER>, bs), bs, 0, H->stream>>>(
            T, C, nq, qx, qy, qz, perm, npts, ctr);
        break;
    default:
        k_points64w<SYMMETRIC><<<persistent_grid((const void *)k_points64w<SYMMETRIC>, bs), bs, 0, H->stream>>>(
            T, C, nq, qx, qy, qz, perm, npts, ctr);
        break;
    }
    H->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_pairs_fp64(Handle *H, const DevTree &T, const DevCatalog &C, int strategy, const RunPool &P,
                              int64_t m, const uint32_t *ql, const uint32_t *order, const double *qx,
                              const double *qy, const double *qz)
{
    int bs = 128;
    cudaError_t e = H->counter.reserve(sizeof(unsigned long long));
    if (e) return e;
    unsigned long long *ctr = H->counter.as<unsigned long long>();
    cudaMemsetAsync(ctr, 0, sizeof(unsigned long long), H->stream);
    switch (strategy) {
    case GATHER:
        k_pairs64w<GATHER><<<persistent_grid((const void *)k_pairs64w<GATHER>, bs), bs, 0, H->stream>>>(
            T, C, P, m, ql, order, qx, qy, qz, ctr);
        break;
    case SCATTER:
        k_pairs64w<SCATTER><<<persistent_grid((const void *)k_pairs64w<SCATTER>, bs), bs, 0, H->stream>>>(
            T, C, P, m, ql, order, qx, qy, qz, ctr);
        break;
    default:
        k_pairs64w<SYMMETRIC><<<persistent_grid((const void *)k_pairs64w<SYMMETRIC>, bs), bs, 0, H->stream>>>(
            T, C, P, m, ql, order, qx, qy, qz, ctr);
        break;
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
