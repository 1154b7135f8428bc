// pb_interp32.cu -- FP32-compensated interpolation kernels.
//
// Same neighbour sets as the FP64 path: the nearest search, the node pruning and every
// per-leaf acceptance test run in FP64 exactly as there, and accepted neighbours are
// processed in the same DFS order.  Per pair, the kernel values and the accumulated terms
// are FP32:
//   * a per-call particle payload (built once per launch) holds the position as double-float
//     pairs, 1/h_b, m_b/rho_b and every quantity column as a (hi, lo) float pair, so the pair
//     needs no division and no FP64 column arithmetic (sigma h_b^-3 and sigma h_b^-4 are
//     formed from 1/h_b);
//   * kernel shapes are evaluated branch-free (selects between pieces written so that nothing
//     cancels near q = 0), templated on the kernel type;
//   * every quantity enters as an offset A_b - A_hat (A_hat = the nearest particle's value,
//     or the first accepted neighbour's for scatter, as a double-float) so that
//     gradient/divergence/curl F - A B cancels as little as possible;
//   * each lane sums its terms in plain FP32 over chunks of 32 full batches of 32 pairs (32 of
//     its own pairs) and adds each chunk sum, converted exactly, to an FP64 accumulator.
// Line integrals are not here: both precision modes use the FP64 line kernel (pb_interp64.cu).
// The per-query arithmetic depends only on the query and the tree (chunks are counted over
// the query's own accepted-neighbour sequence), never on the launch shape or schedule.
#include "pb_internal.h"
#include "pb_fp32_impl.cuh"

namespace pb {

// Fused form: the warp walks the query's tree itself (warp-uniform next_item) and deals the
// accepted leaves to its lanes.  Used for queries the run pool could not hold.
template <int STRAT, int KT>
__global__ void __launch_bounds__(128) k_points32w(DevTree T, DevCatalog C, const float4 *__restrict__ pay, int stride,
                                                   int64_t nq, const double *__restrict__ qx,
                                                   const double *__restrict__ qy, const double *__restrict__ qz,
                                                   const uint32_t *__restrict__ perm, int64_t npts,
                                                   unsigned long long *counter)
{
    __shared__ double s_acc[ACC_SLOTS * ACC_STRIDE];   // FP64 sums, slot k of thread t at [k * 128 + t]
    const int lane = threadIdx.x & 31;
    for (;;) {
        int64_t j = next_query(counter, lane);
        if (j >= nq) break;
        int64_t qi = perm ? (int64_t)__ldg(perm + j) : j;
        if (qi >= npts) continue;
        const double px = __ldg(qx + qi), py = __ldg(qy + qi), pz = __ldg(qz + qi);
        const int64_t bnear = STRAT != SCATTER ? nearest_leaf(T, px, py, pz) : -1;
        points32_query<STRAT, KT>(T, C, pay, stride, px, py, pz, bnear, qi, s_acc, lane, 1);
    }
}

// Pair kernel of the two-phase path: a warp takes a walked query (heaviest first), reads the
// runs of its (query, subtree) items in subtree order, chunk by chunk, and deals the accepted
// leaves to its lanes in DFS order -- the k-th accepted leaf to lane k mod 32, exactly as the
// fused kernel does, so both produce the same bits.  Within a chunk, lane l finds the run
// holding its leaf by a binary search over the inclusive prefix sums of the run lengths
// held one per lane.
template <int STRAT, int KT, int CAT>
__global__ void __launch_bounds__(128, 5) k_pairs32w(DevTree T, DevCatalog C, const float4 *__restrict__ pay, int stride,
                                                  RunPool P, int64_t m, const uint32_t *__restrict__ ql,
                                                  const uint32_t *__restrict__ order, const double *__restrict__ qx,
                                                  const double *__restrict__ qy, const double *__restrict__ qz,
                                                  unsigned long long *counter)
{
    __shared__ double s_acc[ACC_SLOTS * ACC_STRIDE];   // FP64 sums, slot k of thread t at [k * 128 + t]
    const int lane = threadIdx.x & 31;
    for (;;) {
        int64_t t = next_query(counter, lane);
        if (t >= m) break;
        const int64_t j = order ? (int64_t)__ldg(order + t) : t;
        if (__ldg(P.qflag + j)) continue;
        const int64_t qi = __ldg(ql + j);
        const double px = __ldg(qx + qi), py = __ldg(qy + qi), pz = __ldg(qz + qi);
        pairs32_query<STRAT, KT, CAT>(T, C, pay, stride, P, j, qi, px, py, pz,
                                      STRAT != SCATTER ? (int64_t)__ldg(P.bnear + j) : -1, s_acc, lane);
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

template <int STRAT, int KT>
static void launch_one(Handle *H, const DevTree &T, const DevCatalog &C, const float4 *pay, int stride, int64_t nq,
                       const double *qx, const double *qy, const double *qz, const uint32_t *perm, int64_t npts,
                       unsigned long long *ctr)
{
    const int bs = 128;
    k_points32w<STRAT, KT><<<persistent_grid((const void *)k_points32w<STRAT, KT>, bs), bs, 0, H->stream>>>(
        T, C, pay, stride, nq, qx, qy, qz, perm, npts, ctr);
}

template <int STRAT>
static void launch_kt(Handle *H, const DevTree &T, const DevCatalog &C, const float4 *pay, int stride, int64_t nq,
                      const double *qx, const double *qy, const double *qz, const uint32_t *perm, int64_t npts,
                      unsigned long long *ctr)
{
    switch (T.kernel) {
    case 0: launch_one<STRAT, 0>(H, T, C, pay, stride, nq, qx, qy, qz, perm, npts, ctr); break;
    case 1: launch_one<STRAT, 1>(H, T, C, pay, stride, nq, qx, qy, qz, perm, npts, ctr); break;
    case 2: launch_one<STRAT, 2>(H, T, C, pay, stride, nq, qx, qy, qz, perm, npts, ctr); break;
    case 3: launch_one<STRAT, 3>(H, T, C, pay, stride, nq, qx, qy, qz, perm, npts, ctr); break;
    case 4: launch_one<STRAT, 4>(H, T, C, pay, stride, nq, qx, qy, qz, perm, npts, ctr); break;
    default: launch_one<STRAT, 5>(H, T, C, pay, stride, nq, qx, qy, qz, perm, npts, ctr); break;
    }
}

cudaError_t launch_points_fp32(Handle *H, const DevTree &T, const DevCatalog &C, int strategy, int64_t nq,
                               const double *qx, const double *qy, const double *qz, const uint32_t *perm,
                               int64_t npts)
{
    int stride = payload_stride(C.nU);
    cudaError_t e = H->payload.reserve(sizeof(float4) * payload_float4s(T.n, stride));
    if (e) return e;
    e = H->counter.reserve(sizeof(unsigned long long));
    if (e) return e;
    float4 *pay = H->payload.as<float4>();
    unsigned long long *ctr = H->counter.as<unsigned long long>();
    k_payload<<<grid_for(T.n, 256), 256, 0, H->stream>>>(T.n, T, C, pay, stride);
    cudaMemsetAsync(ctr, 0, sizeof(unsigned long long), H->stream);
    switch (strategy) {
    case GATHER: launch_kt<GATHER>(H, T, C, pay, stride, nq, qx, qy, qz, perm, npts, ctr); break;
    case SCATTER: launch_kt<SCATTER>(H, T, C, pay, stride, nq, qx, qy, qz, perm, npts, ctr); break;
    default: launch_kt<SYMMETRIC>(H, T, C, pay, stride, nq, qx, qy, qz, perm, npts, ctr); break;
    }
    H->launches += 2;
    return cudaGetLastError();
}

template <int STRAT, int KT, int CAT>
static void launch_pairs_one(Handle *H, const DevTree &T, const DevCatalog &C, const float4 *pay, int stride,
                             const RunPool &P, int64_t m, const uint32_t *ql, const uint32_t *order, const double *qx,
                             const double *qy, const double *qz, unsigned long long *ctr)
{
    const int bs = 128;
    k_pairs32w<STRAT, KT, CAT><<<persistent_grid((const void *)k_pairs32w<STRAT, KT, CAT>, bs), bs, 0, H->stream>>>(
        T, C, pay, stride, P, m, ql, order, qx, qy, qz, ctr);
}

template <int STRAT, int KT>
static void launch_pairs_cat(Handle *H, const DevTree &T, const DevCatalog &C, const float4 *pay, int stride,
                             const RunPool &P, int64_t m, const uint32_t *ql, const uint32_t *order, const double *qx,
                             const double *qy, const double *qz, unsigned long long *ctr)
{
    switch (catalog_shape(C)) {
    case CAT_GDC4: launch_pairs_one<STRAT, KT, CAT_GDC4>(H, T, C, pay, stride, P, m, ql, order, qx, qy, qz, ctr); break;
    case CAT_C4: launch_pairs_one<STRAT, KT, CAT_C4>(H, T, C, pay, stride, P, m, ql, order, qx, qy, qz, ctr); break;
    case CAT_S1: launch_pairs_one<STRAT, KT, CAT_S1>(H, T, C, pay, stride, P, m, ql, order, qx, qy, qz, ctr); break;
    case CAT_SG1: launch_pairs_one<STRAT, KT, CAT_SG1>(H, T, C, pay, stride, P, m, ql, order, qx, qy, qz, ctr); break;
    default: launch_pairs_one<STRAT, KT, CAT_ANY>(H, T, C, pay, stride, P, m, ql, order, qx, qy, qz, ctr); break;
    }
}

template <int STRAT>
static void launch_pairs_kt(Handle *H, const DevTree &T, const DevCatalog &C, const float4 *pay, int stride,
                            const RunPool &P, int64_t m, const uint32_t *ql, const uint32_t *order, const double *qx,
                            const double *qy, const double *qz, unsigned long long *ctr)
{
    switch (T.kernel) {
    case 0: launch_pairs_cat<STRAT, 0>(H, T, C, pay, stride, P, m, ql, order, qx, qy, qz, ctr); break;
    case 1: launch_pairs_cat<STRAT, 1>(H, T, C, pay, stride, P, m, ql, order, qx, qy, qz, ctr); break;
    case 2: launch_pairs_cat<STRAT, 2>(H, T, C, pay, stride, P, m, ql, order, qx, qy, qz, ctr); break;
    case 3: launch_pairs_cat<STRAT, 3>(H, T, C, pay, stride, P, m, ql, order, qx, qy, qz, ctr); break;
    case 4: launch_pairs_cat<STRAT, 4>(H, T, C, pay, stride, P, m, ql, order, qx, qy, qz, ctr); break;
    default: launch_pairs_cat<STRAT, 5>(H, T, C, pay, stride, P, m, ql, order, qx, qy, qz, ctr); break;
    }
}

cudaError_t launch_pairs_fp32(Handle *H, const DevTree &T, const DevCatalog &C, int strategy, const RunPool &P,
                              int64_t m, const uint32_t *ql, const uint32_t *order, const double *qx,
                              const double *qy, const double *qz)
{
    int stride = payload_stride(C.nU);
    cudaError_t e = H->payload.reserve(sizeof(float4) * payload_float4s(T.n, stride));
    if (e) return e;
    e = H->counter.reserve(sizeof(unsigned long long));
    if (e) return e;
    float4 *pay = H->payload.as<float4>();
    unsigned long long *ctr = H->counter.as<unsigned long long>();
    k_payload<<<grid_for(T.n, 256), 256, 0, H->stream>>>(T.n, T, C, pay, stride);
    cudaMemsetAsync(ctr, 0, sizeof(unsigned long long), H->stream);
    switch (strategy) {
    case GATHER: launch_pairs_kt<GATHER>(H, T, C, pay, stride, P, m, ql, order, qx, qy, qz, ctr); break;
    case SCATTER: launch_pairs_kt<SCATTER>(H, T, C, pay, stride, P, m, ql, order, qx, qy, qz, ctr); break;
    default: launch_pairs_kt<SYMMETRIC>(H, T, C, pay, stride, P, m, ql, order, qx, qy, qz, ctr); break;
    }
    H->launches += 2;
    return cudaGetLastError();
}

}  // namespace pb
