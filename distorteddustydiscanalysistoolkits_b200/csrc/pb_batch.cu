// pb_batch.cu -- the point interpolation of many snapshots (discs) at once, each disc with its
// own LBVH, particles, grid and outputs.  The sample points of all discs form one index space
// (disc after disc, in the processing order the host chose), cut into slices of a fixed size.
// Per slice, two persistent launches cover every disc:
//   1. k_batch_walk: one thread per sample point finds its disc (binary search over the discs'
//      first indices), its nearest particle, and walks the disc's tree, appending the accepted
//      leaves as runs to a shared pool (the walk of the single-disc path, whole tree per point);
//   2. k_batch_pairs: one warp per sample point sums its runs with the bodies of the single-disc
//      pair kernels -- FP64 (the reference's arithmetic) for FP64 mode and for FP32C points of at
//      most light_max accepted neighbours, FP32-compensated for heavier ones -- and a point whose
//      runs did not fit the pool is summed by the fused walk-and-sum bodies instead.
// Every decision is taken on the device and the number of launches depends only on the number
// of sample points, so a step (the discs' builds and these launches) can be captured in a CUDA
// graph.  The bodies are the single-disc kernels' (pb_fp32_impl.cuh, pb_fp64_impl.cuh, compiled
// with -fmad=false here as there), so every value equals a separate call's bit for bit.
#include "pb_internal.h"
#include "pb_fp32_impl.cuh"
#include "pb_fp64_impl.cuh"
#include "pb_walk_impl.cuh"

namespace pb {

// number of accepted leaves of a query: the warp-uniform walk of the sum, without the sums
template <int STRAT>
__device__ __forceinline__ int64_t count_accepted(const DevTree &T, double px, double py, double pz, int64_t bnear,
                                                  int leaf_size)
{
    const double K = kernel_valid(T.kernel);
    double ha = 0.0;
    if (STRAT != SCATTER) ha = bnear < 0 ? __longlong_as_double(0x7ff8000000000000LL) : ldg4(T.leaf + bnear).w;
    const double ra = __dmul_rn(K, ha), r2a = __dmul_rn(ra, ra);
    if (T.root == 0) {
        double4 L;
        double d2;
        return single_leaf_accepted<STRAT>(T, px, py, pz, K, r2a, L, d2) ? 1 : 0;
    }
    Walk w{T.root, 1, 0, 0, 4 * T.n + 64};
    int64_t lo, hi, cnt = 0;
    while (next_item<STRAT>(T, w, px, py, pz, K, r2a, lo, hi, leaf_size)) cnt += hi - lo + 1;
    return cnt;
}

constexpr int BATCH_WARPS = 4;   // warps per block of the pair kernel (128 threads: the Acc32 slot layout)

// processing slot of global index j: the last slot whose first index is at most j
__device__ __forceinline__ int batch_slot(const int64_t *__restrict__ starts, int ndisc, int64_t j)
{
    int lo = 0, hi = ndisc - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(starts + mid) <= j) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <int STRAT>
__global__ void __launch_bounds__(128) k_batch_walk(const BatchDisc *__restrict__ discs,
                                                    const int64_t *__restrict__ starts,
                                                    const uint32_t *__restrict__ slot_disc, int ndisc, int64_t s0,
                                                    int64_t m, RunPool P)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = s0 + t;
        const int lo = batch_slot(starts, ndisc, j);
        const BatchDisc &D = discs[__ldg(slot_disc + lo)];
        const DevTree T = D.T;
        const int64_t qi = j - __ldg(starts + lo);
        const double px = __ldg(D.qx + qi), py = __ldg(D.qy + qi), pz = __ldg(D.qz + qi);
        const int64_t bnear = STRAT != SCATTER ? nearest_leaf(T, px, py, pz) : -1;
        P.bnear[t] = (int)bnear;
        walk_item_at<STRAT>(T, P, t, 0, (uint32_t)t, px, py, pz, kernel_valid(T.kernel));
    }
}

template <int STRAT, int KT>
__global__ void __launch_bounds__(128) k_batch_pairs(const BatchDisc *__restrict__ discs,
                                                     const int64_t *__restrict__ starts,
                                                     const uint32_t *__restrict__ slot_disc, int ndisc, int64_t s0,
                                                     int64_t m, RunPool P, int fp64_only, unsigned light_max,
                                                     int leaf_size, unsigned long long *counter)
{
    __shared__ double s_acc[ACC_SLOTS * ACC_STRIDE];
    __shared__ double s_term[BATCH_WARPS][32 * (NT + 1)];
    __shared__ BatchDisc s_desc[BATCH_WARPS];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int cur = -1;   // disc whose descriptor this warp's slot holds
    for (;;) {
        const int64_t t = next_query(counter, lane);
        if (t >= m) break;
        const int64_t j = s0 + t;
        const int lo = batch_slot(starts, ndisc, j);
        const int k = (int)__ldg(slot_disc + lo);
        if (k != cur) {   // warp-uniform: copy the disc's descriptor into the warp's slot
            __syncwarp();
            const unsigned long long *src = reinterpret_cast<const unsigned long long *>(discs + k);
            unsigned long long *dst = reinterpret_cast<unsigned long long *>(&s_desc[wib]);
            for (int w = lane; w < (int)(sizeof(BatchDisc) / 8); w += 32) dst[w] = __ldg(src + w);
            __syncwarp();
            cur = k;
        }
        const BatchDisc &D = s_desc[wib];
        const DevTree T = D.T;
        const int64_t qi = j - __ldg(starts + lo);
        const double px = __ldg(D.qx + qi), py = __ldg(D.qy + qi), pz = __ldg(D.qz + qi);
        const int64_t bnear = STRAT != SCATTER ? (int64_t)__ldg(P.bnear + t) : -1;
        if (__ldg(P.qflag + t)) {   // runs did not fit the pool: the fused bodies walk again
            const bool fp64 = fp64_only || count_accepted<STRAT>(T, px, py, pz, bnear, leaf_size) <= (int64_t)light_max;
            if (fp64) points64_query<STRAT>(T, D.C64, px, py, pz, bnear, qi, s_term[wib], lane, leaf_size);
            else points32_query<STRAT, KT>(T, D.C32, D.pay, D.stride, px, py, pz, bnear, qi, s_acc, lane, leaf_size);
        } else if (fp64_only || __ldg(P.qacc + t) <= light_max) {
            pairs64_query<STRAT>(T, D.C64, P, t, qi, px, py, pz, bnear, s_term[wib], lane);
        } else {
            pairs32_query<STRAT, KT, CAT_ANY>(T, D.C32, D.pay, D.stride, P, t, qi, px, py, pz, bnear, s_acc, lane);
        }
    }
}

template <int STRAT>
static void launch_batch_kt(Handle *H, int kernel, int grid, const BatchDisc *discs, const int64_t *starts,
                            const uint32_t *slot_disc, int ndisc, int64_t s0, int64_t m, const RunPool &P,
                            int fp64_only, unsigned light_max, int leaf_size, unsigned long long *ctr)
{
#define PB_BATCH_LAUNCH(KT)                                                                                        \
    k_batch_pairs<STRAT, KT><<<grid, 128, 0, H->stream>>>(discs, starts, slot_disc, ndisc, s0, m, P, fp64_only,     \
                                                          light_max, leaf_size, ctr)
    switch (kernel) {
    case 0: PB_BATCH_LAUNCH(0); break;
    case 1: PB_BATCH_LAUNCH(1); break;
    case 2: PB_BATCH_LAUNCH(2); break;
    case 3: PB_BATCH_LAUNCH(3); break;
    case 4: PB_BATCH_LAUNCH(4); break;
    default: PB_BATCH_LAUNCH(5); break;
    }
#undef PB_BATCH_LAUNCH
}

template <int STRAT>
static int batch_blocks_per_sm()
{
    int per = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void *)k_batch_pairs<STRAT, 0>, 128, 0);
    return per > 0 ? per : 1;
}

template <int STRAT>
static void launch_walk_batch(Handle *H, const BatchDisc *discs, const int64_t *starts, const uint32_t *slot_disc,
                              int ndisc, int64_t s0, int64_t m, const RunPool &P)
{
    k_batch_walk<STRAT><<<grid_for(m, 128, 1 << 30), 128, 0, H->stream>>>(discs, starts, slot_disc, ndisc, s0, m, P);
}

// one slice [s0, s0 + m) of the batch's sample points: the walk, then the sums
cudaError_t launch_batch_slice(Handle *H, int strategy, int kernel, const BatchDisc *discs, const int64_t *starts,
                               const uint32_t *slot_disc, int ndisc, int64_t s0, int64_t m, const RunPool &P,
                               int fp64_only, unsigned light_max, int leaf_size, int blocks_per_sm,
                               unsigned long long *ctr)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int per;
    switch (strategy) {   // the occupancy of the M4 instance stands for all kernels of a strategy
    case GATHER: per = batch_blocks_per_sm<GATHER>(); break;
    case SCATTER: per = batch_blocks_per_sm<SCATTER>(); break;
    default: per = batch_blocks_per_sm<SYMMETRIC>(); break;
    }
    if (blocks_per_sm > 0 && blocks_per_sm < per) per = blocks_per_sm;
    const int grid = sms * per;
    cudaError_t e = cudaMemsetAsync(ctr, 0, sizeof(unsigned long long), H->stream);
    if (e) return e;
    switch (strategy) {
    case GATHER:
        launch_walk_batch<GATHER>(H, discs, starts, slot_disc, ndisc, s0, m, P);
        launch_batch_kt<GATHER>(H, kernel, grid, discs, starts, slot_disc, ndisc, s0, m, P, fp64_only, light_max,
                                leaf_size, ctr);
        break;
    case SCATTER:
        launch_walk_batch<SCATTER>(H, discs, starts, slot_disc, ndisc, s0, m, P);
        launch_batch_kt<SCATTER>(H, kernel, grid, discs, starts, slot_disc, ndisc, s0, m, P, fp64_only, light_max,
                                 leaf_size, ctr);
        break;
    default:
        launch_walk_batch<SYMMETRIC>(H, discs, starts, slot_disc, ndisc, s0, m, P);
        launch_batch_kt<SYMMETRIC>(H, kernel, grid, discs, starts, slot_disc, ndisc, s0, m, P, fp64_only, light_max,
                                   leaf_size, ctr);
        break;
    }
    H->launches += 2;
    return cudaGetLastError();
}

// the FP32-compensated payload of one disc (the single-disc launchers build it the same way)
cudaError_t launch_batch_payload(Handle *H, const DevTree &T, const DevCatalog &C, float4 **pay, int *stride)
{
    const int s = payload_stride(C.nU);
    cudaError_t e = H->payload.reserve(sizeof(float4) * payload_float4s(T.n, s));
    if (e) return e;
    *pay = H->payload.as<float4>();
    *stride = s;
    k_payload<<<grid_for(T.n, 256), 256, 0, H->stream>>>(T.n, T, C, *pay, s);
    H->launches += 1;
    return cudaGetLastError();
}

}  // namespace pb
