// pb_batch.cu -- one persistent launch over the sample points of many snapshots (discs), each
// with its own LBVH, particles, grid and outputs.  The queries of all discs form one index
// space (disc after disc, in the processing order the host chose); a warp takes the next
// query from a global counter, finds its disc by binary search over the discs' first query
// indices, copies that disc's descriptor into the warp's shared slot when it changes, and
// sums the query with the fused bodies of the single-disc kernels:
//   * FP64: points64_query (the reference's arithmetic);
//   * FP32C: the accepted leaves are first counted with the same warp-uniform walk, then a
//     query with at most light_max of them is summed by points64_query and a heavier one by
//     points32_query -- the routing of the two-phase path, decided on the device, so a
//     batch needs no host decision between its phases and can be captured in a CUDA graph.
// The bodies are the ones the single-disc kernels run (pb_fp32_impl.cuh, pb_fp64_impl.cuh,
// -fmad=false here as there), so every value equals a separate call's bit for bit.
#include "pb_internal.h"
#include "pb_fp32_impl.cuh"
#include "pb_fp64_impl.cuh"

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

constexpr int BATCH_WARPS = 4;   // warps per block (128 threads: the Acc32 slot layout)

template <int STRAT, int KT>
__global__ void __launch_bounds__(128) k_batch_points(const BatchDisc *__restrict__ discs,
                                                      const int64_t *__restrict__ starts,
                                                      const uint32_t *__restrict__ slot_disc, int ndisc,
                                                      int64_t qtotal, int fp64_only, unsigned light_max,
                                                      int leaf_size, unsigned long long *counter)
{
    __shared__ double s_acc[ACC_SLOTS * ACC_STRIDE];
    __shared__ double s_term[BATCH_WARPS][32 * (NT + 1)];
    __shared__ BatchDisc s_desc[BATCH_WARPS];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int cur = -1;   // disc whose descriptor this warp's slot holds
    for (;;) {
        const int64_t j = next_query(counter, lane);
        if (j >= qtotal) break;
        int lo = 0, hi = ndisc - 1;   // processing slot: the last one starting at or before j
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(starts + mid) <= j) lo = mid;
            else hi = mid - 1;
        }
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
        const int64_t bnear = STRAT != SCATTER ? nearest_leaf(T, px, py, pz) : -1;
        bool fp64 = fp64_only != 0;
        if (!fp64) fp64 = count_accepted<STRAT>(T, px, py, pz, bnear, leaf_size) <= (int64_t)light_max;
        if (fp64) points64_query<STRAT>(T, D.C64, px, py, pz, bnear, qi, s_term[wib], lane, leaf_size);
        else points32_query<STRAT, KT>(T, D.C32, D.pay, D.stride, px, py, pz, bnear, qi, s_acc, lane, leaf_size);
    }
}

template <int STRAT>
static void launch_batch_kt(Handle *H, int kernel, int grid, const BatchDisc *discs, const int64_t *starts,
                            const uint32_t *slot_disc, int ndisc, int64_t qtotal, int fp64_only, unsigned light_max,
                            int leaf_size, unsigned long long *ctr)
{
#define PB_BATCH_LAUNCH(KT)                                                                                        \
    k_batch_points<STRAT, KT><<<grid, 128, 0, H->stream>>>(discs, starts, slot_disc, ndisc, qtotal, fp64_only,     \
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

template <int STRAT, int KT>
static int batch_blocks_per_sm()
{
    int per = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void *)k_batch_points<STRAT, KT>, 128, 0);
    return per > 0 ? per : 1;
}

cudaError_t launch_batch_points(Handle *H, int strategy, int kernel, const BatchDisc *discs, const int64_t *starts,
                                const uint32_t *slot_disc, int ndisc, int64_t qtotal, int fp64_only,
                                unsigned light_max, int leaf_size, int blocks_per_sm, unsigned long long *ctr)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int per;
    switch (strategy) {   // the occupancy of the M4 instance stands for all kernels of a strategy
    case GATHER: per = batch_blocks_per_sm<GATHER, 0>(); break;
    case SCATTER: per = batch_blocks_per_sm<SCATTER, 0>(); break;
    default: per = batch_blocks_per_sm<SYMMETRIC, 0>(); break;
    }
    if (blocks_per_sm > 0 && blocks_per_sm < per) per = blocks_per_sm;
    const int grid = sms * per;
    cudaError_t e = cudaMemsetAsync(ctr, 0, sizeof(unsigned long long), H->stream);
    if (e) return e;
    switch (strategy) {
    case GATHER:
        launch_batch_kt<GATHER>(H, kernel, grid, discs, starts, slot_disc, ndisc, qtotal, fp64_only, light_max, leaf_size, ctr);
        break;
    case SCATTER:
        launch_batch_kt<SCATTER>(H, kernel, grid, discs, starts, slot_disc, ndisc, qtotal, fp64_only, light_max, leaf_size, ctr);
        break;
    default:
        launch_batch_kt<SYMMETRIC>(H, kernel, grid, discs, starts, slot_disc, ndisc, qtotal, fp64_only, light_max, leaf_size, ctr);
        break;
    }
    H->launches += 1;
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
