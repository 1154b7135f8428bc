// pb_walk_impl.cuh -- the per-item walk of the two-phase point path: a thread walks one
// (query, subtree) item with the flat walk (walk_subtree) and appends the accepted leaves, merged
// into runs of consecutive sorted indices, to chunks drawn from a shared pool.  Shared by the
// walk kernels (pb_walk.cu) and the batched walk (pb_batch.cu).
#pragma once
#include <cooperative_groups.h>

#include "pb_interp_impl.cuh"

namespace pb {

namespace cg = cooperative_groups;

// one chunk per calling thread; threads that arrive together share one atomic
__device__ __forceinline__ int alloc_chunk(const RunPool &P)
{
    cg::coalesced_group g = cg::coalesced_threads();
    unsigned long long base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(P.used, (unsigned long long)g.size());
    base = g.shfl(base, 0);
    unsigned long long c = base + g.thread_rank();
    return c < P.cap ? (int)c : -1;
}

struct RunWriter {
    int first = -1, cur = -1, k = 0;
    int nruns = 0;
    int64_t nacc = 0;
    int64_t olo = -1, ohi = -1;   // open run

    __device__ __forceinline__ bool store(const RunPool &P)
    {
        if (P.count_only) {
            ++nruns;
            return true;
        }
        if (cur < 0 || k == RUN_CHUNK) {
            int c = alloc_chunk(P);
            if (c < 0) return false;
            P.next[c] = -1;
            if (cur >= 0) P.next[cur] = c;
            else first = c;
            cur = c;
            k = 0;
        }
        P.runs[(int64_t)cur * RUN_CHUNK + k] = make_uint2((unsigned)olo, (unsigned)(ohi - olo + 1));
        ++k;
        ++nruns;
        return true;
    }
    __device__ __forceinline__ bool emit(const RunPool &P, int64_t lo, int64_t hi)
    {
        nacc += hi - lo + 1;
        if (olo >= 0 && lo == ohi + 1) {
            ohi = hi;
            return true;
        }
        bool ok = olo < 0 || store(P);
        olo = lo;
        ohi = hi;
        return ok;
    }
    __device__ __forceinline__ bool close(const RunPool &P) { return olo < 0 || store(P); }
};

// One (query, subtree) item: walk subtree s of the cut `cut` (P.cut for a single tree) for the
// j-th listed query (sample point qi at px, py, pz; nearest sorted leaf P.bnear[j]) and write
// its runs.
template <int STRAT>
__device__ __forceinline__ void walk_item_at(const DevTree &T, const RunPool &P, const int2 *__restrict__ cut,
                                             int64_t j, int s, uint32_t qi, double px, double py, double pz, double K)
{
    bool ok = P.count_only || (*(volatile unsigned long long *)P.used < P.cap &&
                               *(volatile int *)(P.qflag + j) == 0);   // pool exhausted or query deferred
    RunWriter R;
    if (ok) {
        double ha = 0.0;
        if (STRAT != SCATTER) {
            const int b = P.bnear[j];
            ha = b < 0 ? __longlong_as_double(0x7ff8000000000000LL) : ldg4(T.leaf + b).w;
        }
        const double ra = __dmul_rn(K, ha), r2a = __dmul_rn(ra, ra);
        if (T.root == 0) {
            double4 L;
            double d2;
            if (single_leaf_accepted<STRAT>(T, px, py, pz, K, r2a, L, d2)) ok = R.emit(P, 0, 0);
        } else {
            const int2 c = __ldg(cut + s);
            auto emit = [&](int64_t lo, int64_t hi) { return R.emit(P, lo, hi); };
            ok = walk_subtree<STRAT>(T, c.x, c.y, px, py, pz, K, r2a, emit, P.leaf_size);
        }
        if (ok) ok = R.close(P);
    }
    const int64_t it = j * P.ns + s;
    if (P.count_only) {
        if (R.nacc > 0) atomicAdd(P.qacc + j, (unsigned)R.nacc);
        return;
    }
    if (!ok) {
        P.items[it] = make_int2(RUN_DEFERRED, 0);
        if (atomicExch(P.qflag + j, 1) == 0) {
            unsigned d = atomicAdd(P.n_deferred, 1u);
            P.deferred[d] = qi;
        }
        return;
    }
    P.items[it] = make_int2(R.first, R.nruns);
    if (R.nacc > 0) atomicAdd(P.qacc + j, (unsigned)R.nacc);
}

template <int STRAT>
__device__ __forceinline__ void walk_item(const DevTree &T, const RunPool &P, int64_t j, int s,
                                          const uint32_t *__restrict__ ql, const double *__restrict__ qx,
                                          const double *__restrict__ qy, const double *__restrict__ qz, double K)
{
    const uint32_t qi = __ldg(ql + j);
    walk_item_at<STRAT>(T, P, P.cut, j, s, qi, __ldg(qx + qi), __ldg(qy + qi), __ldg(qz + qi), K);
}

}  // namespace pb
