// pb_batch.cu -- the point interpolation of many snapshots (discs) at once, each disc with its
// own LBVH, particles, grid and outputs.  The sample points of all discs form one index space
// (disc after disc, in the processing order the host chose), cut into slices of a fixed size.
// Per slice, these launches cover every disc:
//   1. k_batch_nearest, k_batch_filter (count, bucket scan, emit) and k_batch_walk_list: one
//      thread per sample point finds its disc (binary search over the discs' first indices)
//      and its nearest particle; every disc's tree is cut into subtrees on the device after
//      its build, the (point, subtree) items whose subtree root survives the walk's first test
//      are listed grouped by (disc, subtree), and warps walk that list, appending the
//      accepted leaves as runs to a shared pool (the single-disc path's prefiltered walk);
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

// per point of the slice: its disc's processing slot and, for gather/symmetric, its nearest
// particle (LBVH_find_nearest_h)
template <int STRAT>
__global__ void __launch_bounds__(128) k_batch_nearest(const BatchDisc *__restrict__ discs,
                                                       const int64_t *__restrict__ starts,
                                                       const uint32_t *__restrict__ slot_disc, int ndisc, int64_t s0,
                                                       int64_t m, RunPool P, int *slot_of)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = s0 + t;
        const int lo = batch_slot(starts, ndisc, j);
        slot_of[t] = lo;
        int64_t bnear = -1;
        if (STRAT != SCATTER) {
            const BatchDisc &D = discs[__ldg(slot_disc + lo)];
            const int64_t qi = j - __ldg(starts + lo);
            bnear = nearest_leaf(D.T, __ldg(D.qx + qi), __ldg(D.qy + qi), __ldg(D.qz + qi));
        }
        P.bnear[t] = (int)bnear;
    }
}

// Prefilter of the walk items (the single-disc k_item_filter for many discs): item (t, s) is
// walked only if the walk would not prune the root of subtree s of point t's disc at its first
// step; the others (and every s past the disc's cut) get an empty record here.  Walked items
// are counted per bucket (disc slot, subtree) and, with EMIT, listed bucket by bucket at
// off[bucket] + cursor, so that the lanes of a walk warp share a disc and a subtree; points are
// taken in `order` (the Morton walk order of the slice; NULL: slice order), so a bucket lists
// neighbouring points next to each other.  The atomics are aggregated over the lanes of a warp
// with equal buckets.
template <int STRAT, bool EMIT>
__global__ void __launch_bounds__(128) k_batch_filter(const BatchDisc *__restrict__ discs,
                                                      const int64_t *__restrict__ starts,
                                                      const uint32_t *__restrict__ slot_disc,
                                                      const int *__restrict__ slot_of, int64_t s0, int64_t m,
                                                      RunPool P, const uint32_t *__restrict__ order, unsigned *cnt,
                                                      const unsigned *__restrict__ off, uint2 *list)
{
    const int ns = P.ns;
    const int lane = threadIdx.x & 31;
    const int64_t mw = (m + 31) & ~int64_t(31);   // whole warps, so every lane reaches the votes
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < mw; p += (int64_t)gridDim.x * blockDim.x) {
        const bool live = p < m;
        const int64_t t = live && order ? (int64_t)__ldg(order + p) : p;   // the point at walk position p
        int lo = 0, nc = 0;
        const BatchDisc *D = nullptr;
        QBox q{};
        float r2a_up = 0.f, Kf = 0.f;
        if (live) {
            lo = __ldg(slot_of + t);
            D = discs + __ldg(slot_disc + lo);
            nc = min(__ldg(D->ncut), ns);   // the cut holds at most ns subtrees
            const int64_t qi = s0 + t - __ldg(starts + lo);
            const double px = __ldg(D->qx + qi), py = __ldg(D->qy + qi), pz = __ldg(D->qz + qi);
            const double K = kernel_valid(D->T.kernel);
            double ha = 0.0;
            if (STRAT != SCATTER) {
                const int b = P.bnear[t];
                ha = b < 0 ? __longlong_as_double(0x7ff8000000000000LL) : ldg4(D->T.leaf + b).w;
            }
            const double ra = __dmul_rn(K, ha);
            r2a_up = __double2float_ru(__dmul_rn(ra, ra));
            Kf = (float)K;
            q = make_qbox(px, py, pz);
        }
        const int smax = __reduce_max_sync(0xffffffffu, nc);
        for (int s = 0; s < smax; ++s) {
            bool walk = false;
            if (s < nc) {
                const DevTree &T = D->T;
                const int node = __ldg(&D->cut[s].x);
                walk = true;
                if (T.root != 0 && node < T.n)
                    walk = !node_pruned<STRAT>(T, load_node(T.node + (node - 1)), node, q, Kf, r2a_up);
                if (!walk && !EMIT) P.items[t * ns + s] = make_int2(-1, 0);
            }
            const unsigned key = (unsigned)lo * (unsigned)ns + (unsigned)s;
            const unsigned act = __ballot_sync(0xffffffffu, walk);
            if (walk) {
                const unsigned grp = __match_any_sync(act, key);
                const int leader = __ffs(grp) - 1;
                const unsigned rank = __popc(grp & ((1u << lane) - 1u));
                unsigned base = 0;
                if (lane == leader) base = atomicAdd(cnt + key, (unsigned)__popc(grp));
                base = __shfl_sync(grp, base, leader);
                if (EMIT) list[off[key] + base + rank] = make_uint2((unsigned)t, (unsigned)s);
            }
        }
        if (live && !EMIT)
            for (int s = nc; s < ns; ++s) P.items[t * ns + s] = make_int2(-1, 0);
    }
}

// the walk over the prefiltered list: nlist = off[nb - 1] + cnt[nb - 1], read on the device
template <int STRAT>
__global__ void __launch_bounds__(128) k_batch_walk_list(const BatchDisc *__restrict__ discs,
                                                         const int64_t *__restrict__ starts,
                                                         const uint32_t *__restrict__ slot_disc,
                                                         const int *__restrict__ slot_of, int64_t s0, RunPool P,
                                                         const unsigned *__restrict__ cnt,
                                                         const unsigned *__restrict__ off, int nb,
                                                         const uint2 *__restrict__ list, unsigned long long *counter)
{
    const int lane = threadIdx.x & 31;
    const int64_t nlist = (int64_t)__ldg(off + nb - 1) + __ldg(cnt + nb - 1);
    for (;;) {
        unsigned long long wi = 0;
        if (lane == 0) wi = atomicAdd(counter, 1ULL);
        wi = __shfl_sync(0xffffffffu, wi, 0);
        if ((int64_t)wi * 32 >= nlist) break;
        const int64_t k = (int64_t)wi * 32 + lane;
        if (k >= nlist) continue;
        const uint2 it = __ldg(list + k);
        const int64_t t = it.x;
        const int lo = __ldg(slot_of + t);
        const BatchDisc &D = discs[__ldg(slot_disc + lo)];
        const DevTree &T = D.T;
        const int64_t qi = s0 + t - __ldg(starts + lo);
        walk_item_at<STRAT>(T, P, D.cut, t, (int)it.y, (uint32_t)t, __ldg(D.qx + qi), __ldg(D.qy + qi),
                            __ldg(D.qz + qi), kernel_valid(T.kernel));
    }
}

// Sort keys of a slice's pair order: class (FP32C points, then FP64 points, then points whose
// runs overflowed the pool), then the disc's processing slot, then descending accepted count
// (clipped to the count bits left after the slot's).  Grouping a class by disc keeps the
// points that run at the same time on one disc's tree and payload, so the L2 holds one disc's
// working set instead of all of them; heaviest first inside a disc keeps the tail short.
__global__ void k_batch_keys(int64_t m, const unsigned *__restrict__ qacc, const int *__restrict__ qflag,
                             const int *__restrict__ slot_of, const uint32_t *__restrict__ order, unsigned light_max,
                             int slot_bits, uint32_t *keys, uint32_t *vals)
{
    const int cbits = 30 - slot_bits;
    const unsigned cmask = cbits >= 32 ? 0xffffffffu : ((1u << cbits) - 1u);
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < m; p += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = order[p];   // laid out in walk order: the stable sort keeps it among equal keys
        const unsigned a = qacc[t];
        const unsigned cls = qflag[t] ? 2u : (a > light_max ? 0u : 1u);
        const unsigned slot = (unsigned)slot_of[t];
        keys[p] = (cls << 30) | (slot << cbits) | (cmask - (a > cmask ? cmask : a));
        vals[p] = (uint32_t)t;
    }
}

// Per-warp copy of the descriptor of the disc of global point j (warp-uniform).
struct DescCache {
    int cur = -1;
    __device__ __forceinline__ const BatchDisc &get(const BatchDisc *__restrict__ discs, BatchDisc &slot, int k, int lane)
    {
        if (k != cur) {
            __syncwarp();
            const unsigned long long *src = reinterpret_cast<const unsigned long long *>(discs + k);
            unsigned long long *dst = reinterpret_cast<unsigned long long *>(&slot);
            for (int w = lane; w < (int)(sizeof(BatchDisc) / 8); w += 32) dst[w] = __ldg(src + w);
            __syncwarp();
            cur = k;
        }
        return slot;
    }
};

// the slice's points in pair order (k_batch_keys): positions [0, nheavy)
// are FP32C points, [nheavy, m - nover) FP64 points, [m - nover, m) points whose runs did not
// fit the pool; ord[t] is the slice-local point
struct SliceOrder {
    const uint32_t *ord;
    const int *slot_of;          // processing slot of every point (k_batch_nearest)
    const unsigned *nheavy;      // device counters of the slice
    const unsigned *nover;
};

template <int STRAT, int KT, int CAT>
__global__ void __launch_bounds__(128, 5) k_batch_pairs32(const BatchDisc *__restrict__ discs,
                                                          const int64_t *__restrict__ starts,
                                                          const uint32_t *__restrict__ slot_disc, int ndisc, int64_t s0,
                                                          RunPool P, SliceOrder O, unsigned long long *counter)
{
    __shared__ double s_acc[ACC_SLOTS * ACC_STRIDE];
    __shared__ BatchDisc s_desc[BATCH_WARPS];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t end = *O.nheavy;
    DescCache dc;
    for (;;) {
        const int64_t pos = next_query(counter, lane);
        if (pos >= end) break;
        const int64_t t = __ldg(O.ord + pos), j = s0 + t;
        const int lo = __ldg(O.slot_of + t);
        const BatchDisc &D = dc.get(discs, s_desc[wib], (int)__ldg(slot_disc + lo), lane);
        const DevTree &T = D.T;
        const int64_t qi = j - __ldg(starts + lo);
        const double px = __ldg(D.qx + qi), py = __ldg(D.qy + qi), pz = __ldg(D.qz + qi);
        pairs32_query<STRAT, KT, CAT>(T, D.C32, D.pay, D.stride, P, t, qi, px, py, pz,
                                      STRAT != SCATTER ? (int64_t)__ldg(P.bnear + t) : -1, s_acc, lane);
    }
}

template <int STRAT>
__global__ void __launch_bounds__(128) k_batch_pairs64(const BatchDisc *__restrict__ discs,
                                                       const int64_t *__restrict__ starts,
                                                       const uint32_t *__restrict__ slot_disc, int ndisc, int64_t s0,
                                                       int64_t m, RunPool P, SliceOrder O, unsigned long long *counter)
{
    __shared__ double s_term[BATCH_WARPS][32 * (NT + 1)];
    __shared__ BatchDisc s_desc[BATCH_WARPS];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t first = *O.nheavy, end = m - (int64_t)*O.nover;
    DescCache dc;
    // the next point's position is fetched while the current one is summed (k_pairs64w)
    unsigned long long nxt = 0;
    if (lane == 0) nxt = atomicAdd(counter, 1ULL);
    int64_t pos = first + (int64_t)__shfl_sync(0xffffffffu, nxt, 0);
    for (; pos < end; pos = first + (int64_t)__shfl_sync(0xffffffffu, nxt, 0)) {
        if (lane == 0) nxt = atomicAdd(counter, 1ULL);
        const int64_t t = __ldg(O.ord + pos), j = s0 + t;
        const int lo = __ldg(O.slot_of + t);
        const BatchDisc &D = dc.get(discs, s_desc[wib], (int)__ldg(slot_disc + lo), lane);
        const DevTree &T = D.T;
        const int64_t qi = j - __ldg(starts + lo);
        const double px = __ldg(D.qx + qi), py = __ldg(D.qy + qi), pz = __ldg(D.qz + qi);
        pairs64_query<STRAT>(T, D.C64, P, t, qi, px, py, pz, STRAT != SCATTER ? (int64_t)__ldg(P.bnear + t) : -1,
                             s_term[wib], lane);
    }
}

// points whose runs did not fit the pool: the fused walk-and-sum bodies, routed by a counting walk
template <int STRAT, int KT>
__global__ void __launch_bounds__(128) k_batch_over(const BatchDisc *__restrict__ discs,
                                                    const int64_t *__restrict__ starts,
                                                    const uint32_t *__restrict__ slot_disc, int ndisc, int64_t s0,
                                                    int64_t m, RunPool P, SliceOrder O, int fp64_only,
                                                    unsigned light_max, int leaf_size, unsigned long long *counter)
{
    __shared__ double s_acc[ACC_SLOTS * ACC_STRIDE];
    __shared__ double s_term[BATCH_WARPS][32 * (NT + 1)];
    __shared__ BatchDisc s_desc[BATCH_WARPS];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t first = m - (int64_t)*O.nover;
    DescCache dc;
    for (;;) {
        const int64_t pos = first + next_query(counter, lane);
        if (pos >= m) break;
        const int64_t t = __ldg(O.ord + pos), j = s0 + t;
        const int lo = __ldg(O.slot_of + t);
        const BatchDisc &D = dc.get(discs, s_desc[wib], (int)__ldg(slot_disc + lo), lane);
        const DevTree &T = D.T;
        const int64_t qi = j - __ldg(starts + lo);
        const double px = __ldg(D.qx + qi), py = __ldg(D.qy + qi), pz = __ldg(D.qz + qi);
        const int64_t bnear = STRAT != SCATTER ? (int64_t)__ldg(P.bnear + t) : -1;
        const bool fp64 = fp64_only || count_accepted<STRAT>(T, px, py, pz, bnear, leaf_size) <= (int64_t)light_max;
        if (fp64) points64_query<STRAT>(T, D.C64, px, py, pz, bnear, qi, s_term[wib], lane, leaf_size);
        else points32_query<STRAT, KT>(T, D.C32, D.pay, D.stride, px, py, pz, bnear, qi, s_acc, lane, leaf_size);
    }
}

template <typename KERN>
static int persistent_blocks_of(KERN kern, int cap)
{
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void *)kern, 128, 0);
    if (per < 1) per = 1;
    if (cap > 0 && cap < per) per = cap;
    return sms * per;
}

template <int STRAT, int KT>
static void launch_slice_pairs(Handle *H, int cat, const BatchDisc *discs, const int64_t *starts, const uint32_t *slot_disc,
                               int ndisc, int64_t s0, int64_t m, const RunPool &P, const SliceOrder &O, int fp64_only,
                               unsigned light_max, int leaf_size, int blocks_per_sm, unsigned long long *ctr)
{
    if (!fp64_only) {
#define PB_PAIRS32(CAT)                                                                                            \
    k_batch_pairs32<STRAT, KT, CAT><<<persistent_blocks_of(k_batch_pairs32<STRAT, KT, CAT>, blocks_per_sm), 128, 0,     \
                                      H->stream>>>(discs, starts, slot_disc, ndisc, s0, P, O, ctr)
        switch (cat) {
        case CAT_GDC4: PB_PAIRS32(CAT_GDC4); break;
        case CAT_C4: PB_PAIRS32(CAT_C4); break;
        case CAT_S1: PB_PAIRS32(CAT_S1); break;
        case CAT_SG1: PB_PAIRS32(CAT_SG1); break;
        default: PB_PAIRS32(CAT_ANY); break;
        }
#undef PB_PAIRS32
    }
    k_batch_pairs64<STRAT><<<persistent_blocks_of(k_batch_pairs64<STRAT>, blocks_per_sm), 128, 0, H->stream>>>(
        discs, starts, slot_disc, ndisc, s0, m, P, O, ctr + 1);
    k_batch_over<STRAT, KT><<<persistent_blocks_of(k_batch_over<STRAT, KT>, blocks_per_sm), 128, 0, H->stream>>>(
        discs, starts, slot_disc, ndisc, s0, m, P, O, fp64_only, light_max, leaf_size, ctr + 2);
}

// nearest particles, the Morton walk order (*worder), prefilter (count, bucket scan, emit) and
// the walk of a slice
template <int STRAT>
static cudaError_t launch_walk_batch(Handle *H, const BatchDisc *discs, const int64_t *starts,
                                     const uint32_t *slot_disc, int ndisc, int64_t s0, int64_t m, const RunPool &P,
                                     int *slot_of, int slot_bits, const uint32_t **worder,
                                     unsigned long long *counter)
{
    const int64_t nb = (int64_t)ndisc * P.ns;
    cudaError_t e;
    if ((e = H->batch_bcnt.reserve(sizeof(unsigned) * nb)) || (e = H->batch_boff.reserve(sizeof(unsigned) * nb)) ||
        (e = H->batch_bcur.reserve(sizeof(unsigned) * nb)) || (e = H->batch_list.reserve(sizeof(uint2) * m * P.ns)))
        return e;
    unsigned *cnt = H->batch_bcnt.as<unsigned>(), *off = H->batch_boff.as<unsigned>(), *cur = H->batch_bcur.as<unsigned>();
    uint2 *list = H->batch_list.as<uint2>();
    if ((e = cudaMemsetAsync(cnt, 0, sizeof(unsigned) * nb, H->stream)) ||
        (e = cudaMemsetAsync(cur, 0, sizeof(unsigned) * nb, H->stream)))
        return e;
    k_batch_nearest<STRAT><<<grid_for(m, 128, 1 << 30), 128, 0, H->stream>>>(discs, starts, slot_disc, ndisc, s0, m, P,
                                                                          slot_of);
    // walk order: disc by disc (processing slot), Morton order of the points inside a disc
    if ((e = H->batch_mk.reserve(sizeof(uint64_t) * m)) || (e = H->batch_mka.reserve(sizeof(uint64_t) * m)) ||
        (e = H->batch_mv.reserve(sizeof(uint32_t) * m)) || (e = H->batch_mva.reserve(sizeof(uint32_t) * m)))
        return e;
    uint64_t *mk = H->batch_mk.as<uint64_t>();
    uint32_t *mv = H->batch_mv.as<uint32_t>();
    if ((e = launch_batch_query_codes(H, m, discs, starts, slot_disc, slot_of, s0, mk, mv))) return e;
    if ((e = sort_pairs_u64(H, mk, mv, H->batch_mka.as<uint64_t>(), H->batch_mva.as<uint32_t>(), m, 32 + slot_bits)))
        return e;
    *worder = mv;
    k_batch_filter<STRAT, false><<<grid_for(m, 128, 1 << 30), 128, 0, H->stream>>>(
        discs, starts, slot_disc, slot_of, s0, m, P, nullptr, cnt, nullptr, nullptr);
    if ((e = launch_exclusive_scan_u32(H, cnt, off, nb))) return e;
    k_batch_filter<STRAT, true><<<grid_for(m, 128, 1 << 30), 128, 0, H->stream>>>(discs, starts, slot_disc, slot_of,
                                                                                s0, m, P, mv, cur, off, list);
    k_batch_walk_list<STRAT><<<persistent_blocks_of(k_batch_walk_list<STRAT>, 0), 128, 0, H->stream>>>(
        discs, starts, slot_disc, slot_of, s0, P, cnt, off, (int)nb, list, counter);
    H->launches += 4;
    return cudaGetLastError();
}

template <int STRAT>
static void launch_slice_strat(Handle *H, int kernel, int cat, const BatchDisc *discs, const int64_t *starts,
                               const uint32_t *slot_disc, int ndisc, int64_t s0, int64_t m, const RunPool &P,
                               const SliceOrder &O, int fp64_only, unsigned light_max, int leaf_size,
                               int blocks_per_sm, unsigned long long *ctr)
{
#define PB_SLICE(KT)                                                                                               \
    launch_slice_pairs<STRAT, KT>(H, cat, discs, starts, slot_disc, ndisc, s0, m, P, O, fp64_only, light_max,       \
                                  leaf_size, blocks_per_sm, ctr)
    switch (kernel) {
    case 0: PB_SLICE(0); break;
    case 1: PB_SLICE(1); break;
    case 2: PB_SLICE(2); break;
    case 3: PB_SLICE(3); break;
    case 4: PB_SLICE(4); break;
    default: PB_SLICE(5); break;
    }
#undef PB_SLICE
}

// One slice [s0, s0 + m) of the batch's sample points: nearest particles, the walk over
// (point, subtree) items, the pair order (by class, then disc, with the FP32C/FP64 split
// counted on the device), then the sums.  slot_of holds m ints.
// ctr: [0..2] persistent pair-kernel counters, [3..4] pair split sums, [5] heavy count (low
// word), [6] walk queue.
cudaError_t launch_batch_slice(Handle *H, int strategy, int kernel, int cat, const BatchDisc *discs,
                               const int64_t *starts, const uint32_t *slot_disc, int ndisc, int64_t s0, int64_t m,
                               const RunPool &P, int fp64_only, unsigned light_max, int leaf_size, int blocks_per_sm,
                               int *slot_of, unsigned long long *ctr)
{
    cudaError_t e = cudaMemsetAsync(ctr, 0, 7 * sizeof(unsigned long long), H->stream);
    if (e) return e;
    int slot_bits = 0;
    while ((1 << slot_bits) < ndisc && slot_bits < 30) ++slot_bits;
    const uint32_t *worder = nullptr;
    switch (strategy) {
    case GATHER:
        e = launch_walk_batch<GATHER>(H, discs, starts, slot_disc, ndisc, s0, m, P, slot_of, slot_bits, &worder, ctr + 6);
        break;
    case SCATTER:
        e = launch_walk_batch<SCATTER>(H, discs, starts, slot_disc, ndisc, s0, m, P, slot_of, slot_bits, &worder,
                                       ctr + 6);
        break;
    default:
        e = launch_walk_batch<SYMMETRIC>(H, discs, starts, slot_disc, ndisc, s0, m, P, slot_of, slot_bits, &worder,
                                         ctr + 6);
        break;
    }
    if (e) return e;
    // pair order: FP32C points, FP64 points, overflowed points; by disc inside a class
    if ((e = H->lpt_k.reserve(4 * m)) || (e = H->lpt_v.reserve(4 * m)) || (e = H->lpt_ka.reserve(4 * m)) ||
        (e = H->lpt_va.reserve(4 * m)))
        return e;
    k_batch_keys<<<grid_for(m, 256), 256, 0, H->stream>>>(m, P.qacc, P.qflag, slot_of, worder,
                                                          fp64_only ? 0xffffffffu : light_max, slot_bits,
                                                          H->lpt_k.as<uint32_t>(), H->lpt_v.as<uint32_t>());
    H->launches += 1;
    if ((e = sort_pairs_u32(H, H->lpt_k.as<uint32_t>(), H->lpt_v.as<uint32_t>(), H->lpt_ka.as<uint32_t>(),
                            H->lpt_va.as<uint32_t>(), m, 32)))
        return e;
    const uint32_t *ord = H->lpt_v.as<uint32_t>();
    unsigned *nheavy = reinterpret_cast<unsigned *>(ctr + 5);
    if ((e = launch_count_heavy(H, P, m, fp64_only ? 0xffffffffu : light_max, nheavy, ctr + 3))) return e;
    SliceOrder O{ord, slot_of, nheavy, P.n_deferred};
    switch (strategy) {
    case GATHER:
        launch_slice_strat<GATHER>(H, kernel, cat, discs, starts, slot_disc, ndisc, s0, m, P, O, fp64_only, light_max,
                                   leaf_size, blocks_per_sm, ctr);
        break;
    case SCATTER:
        launch_slice_strat<SCATTER>(H, kernel, cat, discs, starts, slot_disc, ndisc, s0, m, P, O, fp64_only, light_max,
                                    leaf_size, blocks_per_sm, ctr);
        break;
    default:
        launch_slice_strat<SYMMETRIC>(H, kernel, cat, discs, starts, slot_disc, ndisc, s0, m, P, O, fp64_only,
                                      light_max, leaf_size, blocks_per_sm, ctr);
        break;
    }
    H->launches += 3;
    return cudaGetLastError();
}

// compile-time catalog shape of the batch's FP32C pair kernel (the host-side view of the catalog)
int batch_catalog_shape(const DevCatalog &C32) { return catalog_shape(C32); }

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
