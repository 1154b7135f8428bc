// pb_walk.cu -- the traversal half of the two-phase point interpolation.
//
// 1. k_nearest_list: the nearest particle of every query (gather/symmetric strategies;
//    LBVH_find_nearest_h, LinearBVHQueries.jl:118-140), one thread per query.
// 2. k_cut_mark / k_cut_order: a cut of the tree into ns subtrees of at most ceil(n/ns_target)
//    leaves each (every node whose subtree is small enough while its parent's is not),
//    listed in DFS order.  Their leaf ranges partition 0..n-1 in ascending order.
// 3. k_walk_items: one thread per (query, subtree) item.  A warp walks one subtree for 32
//    consecutive queries of the (Morton-ordered) list, so its lanes follow nearby paths, and
//    a heavy query is spread over ns independent walks.  The walk is next_item<STRAT> of
//    pb_interp_impl.cuh (the reference's acceptance predicate,
//    LinearBVHTraversalMacros.jl:26-371) started at the subtree root and stopped at the node
//    that follows the subtree in DFS order; accepted leaves are emitted as runs of consecutive
//    sorted indices into a chunked pool.
// The pair kernels read a query's items in subtree order, which is the reference's DFS order
// of its accepted leaves.
#include "pb_internal.h"
#include "pb_walk_impl.cuh"

namespace pb {

__global__ void __launch_bounds__(128) k_nearest_list(DevTree T, int64_t m, const uint32_t *__restrict__ ql,
                                                      const double *__restrict__ qx, const double *__restrict__ qy,
                                                      const double *__restrict__ qz, int *bnear)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t qi = __ldg(ql + j);
        bnear[j] = (int)nearest_leaf(T, __ldg(qx + qi), __ldg(qy + qi), __ldg(qz + qi));
    }
}

__device__ __forceinline__ int64_t subtree_size(const DevTree &T, int id)
{
    if (id >= T.n) return 1;
    int2 r = __ldg(T.range + (id - 1));
    return (int64_t)r.y - r.x + 1;
}

// cut nodes: size <= tsz < size(parent) (the root alone when n <= tsz)
__global__ void k_cut_mark(DevTree T, const int *__restrict__ parent, int64_t tsz, int2 *cut, int *count, int cap)
{
    const int64_t ntot = T.root ? 2 * T.n - 1 : 1;
    for (int64_t id = 1 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; id <= ntot;
         id += (int64_t)gridDim.x * blockDim.x) {
        if (subtree_size(T, (int)id) > tsz) continue;
        const int p = T.root ? parent[id - 1] : 0;
        if (p != 0 && subtree_size(T, p) <= tsz) continue;
        const int stop = id >= T.n ? __ldg(T.leaf_escape + (id - T.n)) : T.node[id - 1].escape;
        int k = atomicAdd(count, 1);
        if (k < cap) cut[k] = make_int2((int)id, stop);
    }
}

// one block: order the cut nodes by the first sorted leaf of their subtrees (rank sort)
__global__ void k_cut_order(DevTree T, const int2 *__restrict__ in, const int *count, int cap, int2 *out)
{
    const int k = min(*count, cap);
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const int2 a = in[i];
        const int la = a.x >= T.n ? (int)(a.x - T.n) : T.range[a.x - 1].x;
        int rank = 0;
        for (int t = 0; t < k; ++t) {
            const int2 b = in[t];
            const int lb = b.x >= T.n ? (int)(b.x - T.n) : T.range[b.x - 1].x;
            rank += lb < la;
        }
        out[rank] = a;
    }
}

// warp items: (block of 32 list positions, subtree), query blocks outermost
template <int STRAT>
__global__ void __launch_bounds__(128) k_walk_items(DevTree T, RunPool P, int64_t m, const uint32_t *__restrict__ ql,
                                                    const double *__restrict__ qx, const double *__restrict__ qy,
                                                    const double *__restrict__ qz, unsigned long long *counter)
{
    const int lane = threadIdx.x & 31;
    const int ns = P.ns;
    const int64_t nitems = ((m + 31) / 32) * ns;
    const double K = kernel_valid(T.kernel);
    for (;;) {
        unsigned long long wi = 0;
        if (lane == 0) wi = atomicAdd(counter, 1ULL);
        wi = __shfl_sync(0xffffffffu, wi, 0);
        if ((int64_t)wi >= nitems) break;
        const int64_t j = (int64_t)(wi / ns) * 32 + lane;
        const int s = (int)(wi % ns);
        if (j >= m) continue;
        walk_item<STRAT>(T, P, j, s, ql, qx, qy, qz, K);
    }
}

// Subtree prefilter: an item whose subtree root the walk would prune at its first step gets
// an empty record here and no walk; the others are counted (cnt[j]) and, with emit, listed
// as (subtree, query) pairs at off[j].  The root test is the walk's own (node_pruned).
template <int STRAT, bool EMIT>
__global__ void __launch_bounds__(128) k_item_filter(DevTree T, RunPool P, int64_t m, const uint32_t *__restrict__ ql,
                                                     const double *__restrict__ qx, const double *__restrict__ qy,
                                                     const double *__restrict__ qz, uint32_t *cnt,
                                                     const uint32_t *__restrict__ off, uint32_t *ws, uint32_t *wj)
{
    const double K = kernel_valid(T.kernel);
    const float Kf = (float)K;
    const int ns = P.ns;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t qi = __ldg(ql + j);
        const double px = __ldg(qx + qi), py = __ldg(qy + qi), pz = __ldg(qz + qi);
        double ha = 0.0;
        if (STRAT != SCATTER) {
            const int b = P.bnear[j];
            ha = b < 0 ? __longlong_as_double(0x7ff8000000000000LL) : ldg4(T.leaf + b).w;
        }
        const double ra = __dmul_rn(K, ha), r2a = __dmul_rn(ra, ra);
        const QBox q = make_qbox(px, py, pz);
        const float r2a_up = __double2float_ru(r2a);
        uint32_t k = 0, base = EMIT ? off[j] : 0;
        for (int s = 0; s < ns; ++s) {
            const int node = __ldg(&P.cut[s].x);
            bool walk = true;
            if (T.root != 0 && node < T.n) walk = !node_pruned<STRAT>(T, load_node(T.node + (node - 1)), node, q, Kf, r2a_up);
            if (walk) {
                if (EMIT) {
                    ws[base + k] = (uint32_t)s;
                    wj[base + k] = (uint32_t)j;
                }
                ++k;
            } else if (!EMIT) {
                P.items[j * ns + s] = make_int2(-1, 0);
            }
        }
        if (!EMIT) cnt[j] = k;
    }
}

// walk over a (subtree, query) work list grouped by subtree: the lanes of a warp walk the same
// subtree for neighbouring queries
template <int STRAT>
__global__ void __launch_bounds__(128) k_walk_list(DevTree T, RunPool P, int64_t nlist, const uint32_t *__restrict__ ws,
                                                   const uint32_t *__restrict__ wj, const uint32_t *__restrict__ ql,
                                                   const double *__restrict__ qx, const double *__restrict__ qy,
                                                   const double *__restrict__ qz, unsigned long long *counter)
{
    const int lane = threadIdx.x & 31;
    const double K = kernel_valid(T.kernel);
    for (;;) {
        unsigned long long wi = 0;
        if (lane == 0) wi = atomicAdd(counter, 1ULL);
        wi = __shfl_sync(0xffffffffu, wi, 0);
        const int64_t k = (int64_t)wi * 32 + lane;
        if ((int64_t)wi * 32 >= nlist) break;
        if (k >= nlist) continue;
        walk_item<STRAT>(T, P, (int64_t)__ldg(wj + k), (int)__ldg(ws + k), ql, qx, qy, qz, K);
    }
}

// descending accepted count first (deferred queries last): the heaviest queries start first
__global__ void k_lpt_keys(int64_t m, const unsigned *__restrict__ qacc, const int *__restrict__ qflag,
                           uint32_t *keys, uint32_t *vals)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
        unsigned a = qflag[j] ? 0u : qacc[j];
        keys[j] = 0x7fffffffu - (a > 0x7fffffffu ? 0x7fffffffu : a);
        vals[j] = (uint32_t)j;
    }
}

// queries (not deferred) with more than `light_max` accepted leaves, and the accepted pairs of
// the heavy and of the light queries (pairs[0], pairs[1]); one set of atomics per block
__global__ void k_count_heavy(int64_t m, const unsigned *__restrict__ qacc, const int *__restrict__ qflag,
                              unsigned light_max, unsigned *count, unsigned long long *pairs)
{
    __shared__ unsigned long long s_pairs[2];
    __shared__ unsigned s_count;
    if (threadIdx.x == 0) {
        s_pairs[0] = s_pairs[1] = 0ULL;
        s_count = 0u;
    }
    __syncthreads();
    unsigned c = 0;
    unsigned long long ph = 0, pl = 0;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
        if (qflag[j]) continue;
        const unsigned a = qacc[j];
        if (a > light_max) {
            ++c;
            ph += a;
        } else {
            pl += a;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        c += __shfl_down_sync(0xffffffffu, c, off);
        ph += __shfl_down_sync(0xffffffffu, ph, off);
        pl += __shfl_down_sync(0xffffffffu, pl, off);
    }
    if ((threadIdx.x & 31) == 0) {
        if (c) atomicAdd(&s_count, c);
        if (ph) atomicAdd(&s_pairs[0], ph);
        if (pl) atomicAdd(&s_pairs[1], pl);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_count) atomicAdd(count, s_count);
        if (s_pairs[0]) atomicAdd(pairs, s_pairs[0]);
        if (s_pairs[1]) atomicAdd(pairs + 1, s_pairs[1]);
    }
}

// plain schedule: a stable partition, heavy queries first, input order kept in each part
__global__ void k_heavy_keys(int64_t m, const unsigned *__restrict__ qacc, const int *__restrict__ qflag,
                             unsigned light_max, uint32_t *keys, uint32_t *vals)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
        keys[j] = (!qflag[j] && qacc[j] > light_max) ? 0u : 1u;
        vals[j] = (uint32_t)j;
    }
}

__global__ void k_iota(int64_t m, uint32_t *out)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x)
        out[j] = (uint32_t)j;
}

static int persistent_blocks(const void *kern, int bs)
{
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, bs, 0);
    return sms * (per > 0 ? per : 1);
}

cudaError_t launch_cut(Handle *H, const DevTree &T, int target, int *ns_out)
{
    const int64_t n = T.n;
    int64_t tsz = (n + target - 1) / target;
    if (tsz < 1) tsz = 1;
    const int cap = 4 * target + 8;
    cudaError_t e;
    if ((e = H->cut.reserve(sizeof(int2) * 2 * cap + 16))) return e;
    int2 *raw = H->cut.as<int2>();
    int2 *sorted = raw + cap;
    int *count = reinterpret_cast<int *>(raw + 2 * cap);
    if ((e = cudaMemsetAsync(count, 0, sizeof(int), H->stream))) return e;
    const int64_t ntot = T.root ? 2 * n - 1 : 1;
    k_cut_mark<<<grid_for(ntot, 256), 256, 0, H->stream>>>(T, H->parent.as<int>(), tsz, raw, count, cap);
    k_cut_order<<<1, 1024, 0, H->stream>>>(T, raw, count, cap, sorted);
    H->launches += 2;
    if ((e = cudaGetLastError())) return e;
    int k = 0;
    if ((e = cudaMemcpyAsync(&k, count, sizeof(int), cudaMemcpyDeviceToHost, H->stream))) return e;
    if ((e = cudaStreamSynchronize(H->stream))) return e;
    if (k < 1 || k > cap) return cudaErrorInvalidValue;
    *ns_out = k;
    return cudaSuccess;
}

// a device-made cut that overflowed its capacity flags the tree's status word (the host
// path returns an error instead)
__global__ void k_cut_check(const int *count, int cap, int *status)
{
    if (*count > cap) atomicOr(status, ST_CUT);
}

cudaError_t launch_cut_device(Handle *H, const DevTree &T, int target, const int2 **cut, const int **count)
{
    const int64_t n = T.n;
    int64_t tsz = (n + target - 1) / target;
    if (tsz < 1) tsz = 1;
    const int cap = 4 * target + 8;
    cudaError_t e;
    if ((e = H->cut.reserve(sizeof(int2) * 2 * cap + 16))) return e;
    int2 *raw = H->cut.as<int2>();
    int2 *sorted = raw + cap;
    int *cnt = reinterpret_cast<int *>(raw + 2 * cap);
    if ((e = cudaMemsetAsync(cnt, 0, sizeof(int), H->stream))) return e;
    const int64_t ntot = T.root ? 2 * n - 1 : 1;
    k_cut_mark<<<grid_for(ntot, 256), 256, 0, H->stream>>>(T, H->parent.as<int>(), tsz, raw, cnt, cap);
    k_cut_order<<<1, 1024, 0, H->stream>>>(T, raw, cnt, cap, sorted);
    k_cut_check<<<1, 1, 0, H->stream>>>(cnt, cap, T.status);
    H->launches += 3;
    *cut = sorted;
    *count = cnt;
    return cudaGetLastError();
}

cudaError_t launch_nearest_list(Handle *H, const DevTree &T, int64_t m, const uint32_t *ql, const double *qx,
                                const double *qy, const double *qz, int *bnear)
{
    k_nearest_list<<<grid_for(m, 128, 1 << 30), 128, 0, H->stream>>>(T, m, ql, qx, qy, qz, bnear);
    H->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_walk(Handle *H, const DevTree &T, int strategy, const RunPool &P, int64_t m, const uint32_t *ql,
                        const double *qx, const double *qy, const double *qz, unsigned long long *counter)
{
    const int bs = 128;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), H->stream);
    if (e) return e;
    switch (strategy) {
    case GATHER:
        k_walk_items<GATHER><<<persistent_blocks((const void *)k_walk_items<GATHER>, bs), bs, 0, H->stream>>>(
            T, P, m, ql, qx, qy, qz, counter);
        break;
    case SCATTER:
        k_walk_items<SCATTER><<<persistent_blocks((const void *)k_walk_items<SCATTER>, bs), bs, 0, H->stream>>>(
            T, P, m, ql, qx, qy, qz, counter);
        break;
    default:
        k_walk_items<SYMMETRIC><<<persistent_blocks((const void *)k_walk_items<SYMMETRIC>, bs), bs, 0, H->stream>>>(
            T, P, m, ql, qx, qy, qz, counter);
        break;
    }
    H->launches += 1;
    return cudaGetLastError();
}

template <int STRAT>
static cudaError_t walk_list_strat(Handle *H, const DevTree &T, const RunPool &P, int64_t m, const uint32_t *ql,
                                   const double *qx, const double *qy, const double *qz, unsigned long long *counter)
{
    cudaError_t e;
    if ((e = H->wl_cnt.reserve(sizeof(uint32_t) * (m + 1)))) return e;
    if ((e = H->wl_off.reserve(sizeof(uint32_t) * (m + 1)))) return e;
    uint32_t *cnt = H->wl_cnt.as<uint32_t>(), *off = H->wl_off.as<uint32_t>();
    k_item_filter<STRAT, false><<<grid_for(m, 128, 1 << 30), 128, 0, H->stream>>>(T, P, m, ql, qx, qy, qz, cnt,
                                                                                 nullptr, nullptr, nullptr);
    if ((e = launch_exclusive_scan_u32(H, cnt, off, m))) return e;
    uint32_t last[2] = {0, 0};
    if ((e = cudaMemcpyAsync(&last[0], off + (m - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, H->stream))) return e;
    if ((e = cudaMemcpyAsync(&last[1], cnt + (m - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, H->stream))) return e;
    if ((e = cudaStreamSynchronize(H->stream))) return e;
    const int64_t nlist = (int64_t)last[0] + last[1];
    H->launches += 1;
    if (nlist == 0) return cudaSuccess;
    if ((e = H->wl_s.reserve(sizeof(uint32_t) * nlist))) return e;
    if ((e = H->wl_j.reserve(sizeof(uint32_t) * nlist))) return e;
    if ((e = H->wl_sa.reserve(sizeof(uint32_t) * nlist))) return e;
    if ((e = H->wl_ja.reserve(sizeof(uint32_t) * nlist))) return e;
    uint32_t *ws = H->wl_s.as<uint32_t>(), *wj = H->wl_j.as<uint32_t>();
    k_item_filter<STRAT, true><<<grid_for(m, 128, 1 << 30), 128, 0, H->stream>>>(T, P, m, ql, qx, qy, qz, nullptr,
                                                                                off, ws, wj);
    H->launches += 1;
    int bits = 1;
    while ((1 << bits) < P.ns) ++bits;
    if ((e = sort_pairs_u32(H, ws, wj, H->wl_sa.as<uint32_t>(), H->wl_ja.as<uint32_t>(), nlist, bits))) return e;
    if ((e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), H->stream))) return e;
    const int bs = 128;
    k_walk_list<STRAT><<<persistent_blocks((const void *)k_walk_list<STRAT>, bs), bs, 0, H->stream>>>(
        T, P, nlist, ws, wj, ql, qx, qy, qz, counter);
    H->launches += 1;
    return cudaGetLastError();
}

// the walk of a slice through the prefiltered (subtree, query) work list
cudaError_t launch_walk_list(Handle *H, const DevTree &T, int strategy, const RunPool &P, int64_t m,
                             const uint32_t *ql, const double *qx, const double *qy, const double *qz,
                             unsigned long long *counter)
{
    if (m <= 0) return cudaSuccess;
    switch (strategy) {
    case GATHER: return walk_list_strat<GATHER>(H, T, P, m, ql, qx, qy, qz, counter);
    case SCATTER: return walk_list_strat<SCATTER>(H, T, P, m, ql, qx, qy, qz, counter);
    default: return walk_list_strat<SYMMETRIC>(H, T, P, m, ql, qx, qy, qz, counter);
    }
}

cudaError_t launch_lpt_order(Handle *H, const RunPool &P, int64_t m, uint32_t **order)
{
    cudaError_t e;
    if ((e = H->lpt_k.reserve(4 * m))) return e;
    if ((e = H->lpt_v.reserve(4 * m))) return e;
    if ((e = H->lpt_ka.reserve(4 * m))) return e;
    if ((e = H->lpt_va.reserve(4 * m))) return e;
    k_lpt_keys<<<grid_for(m, 256), 256, 0, H->stream>>>(m, P.qacc, P.qflag, H->lpt_k.as<uint32_t>(),
                                                        H->lpt_v.as<uint32_t>());
    H->launches += 1;
    if ((e = cudaGetLastError())) return e;
    if ((e = sort_pairs_u32(H, H->lpt_k.as<uint32_t>(), H->lpt_v.as<uint32_t>(), H->lpt_ka.as<uint32_t>(),
                            H->lpt_va.as<uint32_t>(), m, 31)))
        return e;
    *order = H->lpt_v.as<uint32_t>();
    return cudaSuccess;
}

// pair order of a walked slice and the number of heavy queries at its front: heaviest first
// (LPT) unless `plain`, where it is the stable heavy/light partition of the walk order; the
// accepted pairs of the heavy and the light queries are added to pairs[0], pairs[1]
cudaError_t launch_split_order(Handle *H, const RunPool &P, int64_t m, unsigned light_max, bool plain,
                               uint32_t **order, int64_t *m_heavy, unsigned long long *pairs)
{
    cudaError_t e;
    if (!plain) {
        if ((e = launch_lpt_order(H, P, m, order))) return e;
    } else {
        if ((e = H->lpt_k.reserve(4 * m))) return e;
        if ((e = H->lpt_v.reserve(4 * m))) return e;
        if ((e = H->lpt_ka.reserve(4 * m))) return e;
        if ((e = H->lpt_va.reserve(4 * m))) return e;
        k_heavy_keys<<<grid_for(m, 256), 256, 0, H->stream>>>(m, P.qacc, P.qflag, light_max, H->lpt_k.as<uint32_t>(),
                                                             H->lpt_v.as<uint32_t>());
        H->launches += 1;
        if ((e = cudaGetLastError())) return e;
        if ((e = sort_pairs_u32(H, H->lpt_k.as<uint32_t>(), H->lpt_v.as<uint32_t>(), H->lpt_ka.as<uint32_t>(),
                                H->lpt_va.as<uint32_t>(), m, 1)))
            return e;
        *order = H->lpt_v.as<uint32_t>();
    }
    unsigned *cnt = reinterpret_cast<unsigned *>(P.n_deferred) + 1;
    if ((e = cudaMemsetAsync(cnt, 0, sizeof(unsigned), H->stream))) return e;
    k_count_heavy<<<grid_for(m, 256), 256, 0, H->stream>>>(m, P.qacc, P.qflag, light_max, cnt, pairs);
    H->launches += 1;
    if ((e = cudaGetLastError())) return e;
    unsigned hcount = 0;
    if ((e = cudaMemcpyAsync(&hcount, cnt, sizeof(unsigned), cudaMemcpyDeviceToHost, H->stream))) return e;
    if ((e = cudaStreamSynchronize(H->stream))) return e;
    *m_heavy = hcount;
    return cudaSuccess;
}

// the FP32C/FP64 split of a walked slice, left on the device: *count (zeroed here) = queries
// with more than light_max accepted leaves, pairs[0..1] += their pairs / the other queries' pairs
cudaError_t launch_count_heavy(Handle *H, const RunPool &P, int64_t m, unsigned light_max, unsigned *count,
                               unsigned long long *pairs)
{
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(unsigned), H->stream);
    if (e) return e;
    k_count_heavy<<<grid_for(m, 256), 256, 0, H->stream>>>(m, P.qacc, P.qflag, light_max, count, pairs);
    H->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_iota(Handle *H, int64_t m, uint32_t *out)
{
    k_iota<<<grid_for(m, 256), 256, 0, H->stream>>>(m, out);
    H->launches += 1;
    return cudaGetLastError();
}

}  // namespace pb
