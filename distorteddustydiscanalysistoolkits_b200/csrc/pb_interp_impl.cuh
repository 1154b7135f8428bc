// pb_interp_impl.cuh -- the traversal building blocks shared by the interpolation units:
// nearest-h search, the stackless left/escape DFS of the ball query
// (LinearBVHTraversalMacros.jl:26-371) in its warp-uniform (next_item) and flat per-thread
// (walk_subtree) forms, the dealing of a query's accepted runs to the lanes of a warp
// (deal_runs), the FP64 accumulator of the reference's arithmetic and the line kernel.
//
// Included by pb_interp64.cu (-fmad=false; FP64 terms in the reference's expressions and
// order, bit-exact with the FP64 oracle), pb_interp32.cu (FP32 per-pair terms with double-float
// offsets, FP64 accumulation of FP32 chunk sums; the FP32 line kernel uses TwoSum) and
// pb_walk.cu (the walk kernels).
//
// Accepted neighbours are visited in ascending sorted-leaf order (DFS preorder), exactly as
// in the reference, so the per-query summation order does not depend on the launch shape.
// Node pruning uses FP32 boxes rounded outward: it visits a superset of the reference's
// nodes and accepts exactly the same leaves.
#pragma once
#include "pb_device.cuh"

namespace pb {

template <int N, typename T>
__device__ __forceinline__ T pick(const T (&a)[N], int i)
{
    T r = a[0];
#pragma unroll
    for (int k = 1; k < N; ++k)
        if (i == k) r = a[k];
    return r;
}

__device__ __forceinline__ void flag(int *status, int bit) { atomicOr(status, bit); }

__device__ __forceinline__ NodeF load_node(const NodeF *p)
{
    const float4 *q = reinterpret_cast<const float4 *>(p);
    float4 a = __ldg(q), c = __ldg(q + 1);
    NodeF nd;
    nd.lox = a.x; nd.loy = a.y; nd.loz = a.z; nd.left = __float_as_int(a.w);
    nd.hix = c.x; nd.hiy = c.y; nd.hiz = c.z; nd.escape = __float_as_int(c.w);
    return nd;
}

// --------------------------------------------------------------------------------------
// FP32 box tests with directed rounding.  The query point is kept as round-down/round-up
// floats; gaps, squares and sums are rounded toward the safe side, so `lower` never exceeds
// the exact box distance^2 and `upper` is never below the exact farthest-corner distance^2.
// Decisions then carry a relative margin of 2^-20, far above FP64 rounding (2^-53), so a
// subtree is pruned only if every leaf in it fails its FP64 acceptance test and is
// bulk-accepted only if every leaf passes it -- exactly the decisions of the FP64 walk.
struct QBox {
    float dn[3], up[3];
};

__device__ __forceinline__ QBox make_qbox(double px, double py, double pz)
{
    QBox q;
    q.dn[0] = __double2float_rd(px); q.up[0] = __double2float_ru(px);
    q.dn[1] = __double2float_rd(py); q.up[1] = __double2float_ru(py);
    q.dn[2] = __double2float_rd(pz); q.up[2] = __double2float_ru(pz);
    return q;
}

constexpr float MARGIN_UP = 1.0f + 9.5367431640625e-07f;   // 1 + 2^-20
constexpr float MARGIN_DN = 1.0f - 9.5367431640625e-07f;

__device__ __forceinline__ float box_lower(const QBox &q, const NodeF &nd)
{
    float gx = fmaxf(fmaxf(__fsub_rd(nd.lox, q.up[0]), __fsub_rd(q.dn[0], nd.hix)), 0.f);
    float gy = fmaxf(fmaxf(__fsub_rd(nd.loy, q.up[1]), __fsub_rd(q.dn[1], nd.hiy)), 0.f);
    float gz = fmaxf(fmaxf(__fsub_rd(nd.loz, q.up[2]), __fsub_rd(q.dn[2], nd.hiz)), 0.f);
    return __fadd_rd(__fadd_rd(__fmul_rd(gx, gx), __fmul_rd(gy, gy)), __fmul_rd(gz, gz));
}

__device__ __forceinline__ float box_upper(const QBox &q, const NodeF &nd)
{
    float fx = fmaxf(__fsub_ru(q.up[0], nd.lox), __fsub_ru(nd.hix, q.dn[0]));
    float fy = fmaxf(__fsub_ru(q.up[1], nd.loy), __fsub_ru(nd.hiy, q.dn[1]));
    float fz = fmaxf(__fsub_ru(q.up[2], nd.loz), __fsub_ru(nd.hiz, q.dn[2]));
    return __fadd_ru(__fadd_ru(__fmul_ru(fx, fx), __fmul_ru(fy, fy)), __fmul_ru(fz, fz));
}

// (K h)^2 rounded up, for a node's hmax (already rounded up) or the query radius
__device__ __forceinline__ float sq_up(float K, float h)
{
    float r = __fmul_ru(K, h);
    return __fmul_ru(r, r);
}

// LBVH_find_nearest_h (LinearBVHQueries.jl:118-140).  The reference walks the tree in DFS
// order with a shrinking radius and keeps the first strictly closer leaf, i.e. it returns
// the minimum squared distance and, among equal distances, the smallest sorted leaf index.
// This search visits the nearer child first (explicit stack) and applies exactly that
// rule, so it returns the same leaf while visiting far fewer nodes.  Boxes are the FP32
// outward-rounded ones (never farther than any leaf inside), and a subtree is skipped only
// when its box distance is strictly greater than the best distance.
constexpr int NN_STACK = 64;

__device__ __forceinline__ float child_dist(const DevTree &T, const QBox &q, int id, double px, double py,
                                            double pz, double &best, int64_t &bi)
{
    const int64_t n = T.n;
    if (id >= n) {
        int64_t b = id - n;
        double d2 = d2_point(px, py, pz, ldg4(T.leaf + b));
        if (d2 < best || (d2 == best && b < bi)) { best = d2; bi = b; }
        return INFINITY;   // a leaf needs no further visit
    }
    return box_lower(q, load_node(T.node + (id - 1)));
}

__device__ __forceinline__ int64_t nearest_leaf(const DevTree &T, double px, double py, double pz)
{
    double best = INFINITY;
    int64_t bi = -1;
    if (T.root == 0) {
        double d2 = d2_point(px, py, pz, ldg4(T.leaf));
        return d2 < best ? 0 : -1;
    }
    const QBox q = make_qbox(px, py, pz);
    int sn[NN_STACK];
    float sd[NN_STACK];
    int sp = 0;
    int node = T.root;
    int64_t guard = 0, limit = 4 * T.n + 64;
    // a subtree is skipped only when its lower bound exceeds the best distance by the margin
    auto visit = [&](float d) { return d <= __fmul_ru(__double2float_ru(best), MARGIN_UP); };
    for (;;) {
        if (++guard > limit) { atomicOr(T.status, ST_TRAVERSAL); break; }
        int2 ch = __ldg(T.child + (node - 1));
        float dl = child_dist(T, q, ch.x, px, py, pz, best, bi);
        float dr = child_dist(T, q, ch.y, px, py, pz, best, bi);
        bool vl = visit(dl), vr = visit(dr);
        if (vl && vr) {
            bool lf = dl <= dr;
            int far = lf ? ch.y : ch.x;
            float fd = lf ? dr : dl;
            if (sp < NN_STACK) { sn[sp] = far; sd[sp] = fd; ++sp; }
            else { atomicOr(T.status, ST_TRAVERSAL); }
            node = lf ? ch.x : ch.y;
            continue;
        }
        if (vl) { node = ch.x; continue; }
        if (vr) { node = ch.y; continue; }
        node = 0;
        while (sp > 0) {
            --sp;
            if (visit(sd[sp])) { node = sn[sp]; break; }
        }
        if (node == 0) break;
    }
    return bi;
}

// Largest squared distance from the point to any point of the (outward-rounded) box,
// with the rounding sequence of d2_point: every leaf inside has d2_point <= this value.
__device__ __forceinline__ double far_d2_box(double px, double py, double pz, const NodeF &nd)
{
    double ax = fmax(fabs(__dsub_rn(px, (double)nd.lox)), fabs(__dsub_rn(px, (double)nd.hix)));
    double ay = fmax(fabs(__dsub_rn(py, (double)nd.loy)), fabs(__dsub_rn(py, (double)nd.hiy)));
    double az = fmax(fabs(__dsub_rn(pz, (double)nd.loz)), fabs(__dsub_rn(pz, (double)nd.hiz)));
    double s = __dmul_rn(ax, ax);
    s = __dadd_rn(s, __dmul_rn(ay, ay));
    s = __dadd_rn(s, __dmul_rn(az, az));
    return s;
}


// --------------------------------------------------------------------------------------
// DFS walker of the main pass ("while-while" form): each call advances the stackless
// left/escape traversal (LinearBVHTraversalMacros.jl:135-371) until the next accepted leaf
// and returns it, so all lanes of a warp evaluate their pair terms together.  A subtree
// lying entirely inside the query's radius is turned into a cursor over its contiguous
// sorted-leaf range, which is exactly the DFS order of its leaves.  The sequence of
// accepted leaves is therefore the reference's.
struct Walk {
    int node;
    int64_t cur, end, guard, limit;
    int stop = 0;   // node where the walk ends: 0 for the whole tree, a subtree's escape target for a subtree
};

template <int STRAT>
__device__ __forceinline__ int64_t next_accepted(const DevTree &T, Walk &w, double px, double py, double pz,
                                                 double K, double r2a, double4 &L, double &d2)
{
    const int64_t n = T.n;
    for (;;) {
        if (w.cur <= w.end) {
            int64_t b = w.cur++;
            L = ldg4(T.leaf + b);
            d2 = d2_point(px, py, pz, L);
            return b;
        }
        if (w.node == 0) return -1;
        if (++w.guard > w.limit) { flag(T.status, ST_TRAVERSAL); w.node = 0; return -1; }
        const int node = w.node;
        if (node >= n) {
            int64_t b = node - n;
            L = ldg4(T.leaf + b);
            w.node = __ldg(T.leaf_escape + b);
            double r2;
            if (STRAT == GATHER) r2 = r2a;
            else {
                double r = __dmul_rn(K, L.w);
                double rr = __dmul_rn(r, r);
                r2 = STRAT == SCATTER ? rr : (r2a > rr ? r2a : rr);
            }
            d2 = d2_point(px, py, pz, L);
            if (d2 <= r2) return b;
            continue;
        }
        NodeF nd = load_node(T.node + (node - 1));
        double r2;
        if (STRAT == GATHER) r2 = r2a;
        else {
            double r = __dmul_rn(K, (double)__ldg(T.node_hmax + (node - 1)));
            double rr = __dmul_rn(r, r);
            r2 = STRAT == SCATTER ? rr : (r2a > rr ? r2a : rr);
        }
        if (d2_box(px, py, pz, nd) > r2) { w.node = nd.escape; continue; }
        if (STRAT != SCATTER && far_d2_box(px, py, pz, nd) <= r2a) {
            int2 rg = __ldg(T.range + (node - 1));
            w.cur = rg.x;
            w.end = rg.y;
            w.node = nd.escape;
            continue;
        }
        w.node = nd.left;
    }
}

// The walk's pruning decision for internal node `node` (box `nd`): FP32 box distance with
// directed rounding against the node radius (query radius and/or K * hmax) with the 2^-20
// margin.  Shared by the walk and by the subtree prefilter so both decide alike.
template <int STRAT>
__device__ __forceinline__ bool node_pruned(const DevTree &T, const NodeF &nd, int node, const QBox &q, float Kf,
                                            float r2a_up)
{
    float r2n;
    if (STRAT == GATHER) r2n = r2a_up;
    else {
        float rr = sq_up(Kf, __ldg(T.node_hmax + (node - 1)));
        r2n = STRAT == SCATTER ? rr : fmaxf(r2a_up, rr);
    }
    return box_lower(q, nd) > __fmul_ru(r2n, MARGIN_UP);
}

// Warp-uniform form of the same walk for the warp-per-query kernels: returns the next
// accepted item in DFS order, either a single leaf (lo == hi) or the whole contiguous leaf
// range of a subtree that lies inside the query radius.  With leaf_size > 1, a subtree of at
// most leaf_size leaves that is neither pruned nor accepted whole is scanned leaf by leaf in
// sorted order with the exact FP64 test instead of being descended: the accepted leaves and
// their order -- hence every sum -- are the same, only the node visits change.
template <int STRAT>
__device__ __forceinline__ bool next_item(const DevTree &T, Walk &w, double px, double py, double pz, double K,
                                          double r2a, int64_t &lo, int64_t &hi, int leaf_size = 1)
{
    const int64_t n = T.n;
    const QBox q = make_qbox(px, py, pz);
    const float Kf = (float)K;
    const float r2a_up = __double2float_ru(r2a);
    const float bulk_lim = __fmul_rd(__double2float_rd(r2a), MARGIN_DN);
    for (;;) {
        if (w.cur <= w.end) {   // linear scan of a small subtree's leaves
            if (++w.guard > w.limit) { flag(T.status, ST_TRAVERSAL); w.cur = 1; w.end = 0; w.node = w.stop; return false; }
            const int64_t b = w.cur++;
            const double4 L = ldg4(T.leaf + b);
            double r2;
            if (STRAT == GATHER) r2 = r2a;
            else {
                double r = __dmul_rn(K, L.w);
                double rr = __dmul_rn(r, r);
                r2 = STRAT == SCATTER ? rr : (r2a > rr ? r2a : rr);
            }
            if (d2_point(px, py, pz, L) <= r2) { lo = hi = b; return true; }
            continue;
        }
        if (w.node == w.stop) return false;
        if (++w.guard > w.limit) { flag(T.status, ST_TRAVERSAL); w.node = w.stop; return false; }
        const int node = w.node;
        if (node >= n) {
            int64_t b = node - n;
            double4 L = ldg4(T.leaf + b);
            w.node = __ldg(T.leaf_escape + b);
            double r2;
            if (STRAT == GATHER) r2 = r2a;
            else {
                double r = __dmul_rn(K, L.w);
                double rr = __dmul_rn(r, r);
                r2 = STRAT == SCATTER ? rr : (r2a > rr ? r2a : rr);
            }
            if (d2_point(px, py, pz, L) <= r2) { lo = hi = b; return true; }
            continue;
        }
        NodeF nd = load_node(T.node + (node - 1));
        if (node_pruned<STRAT>(T, nd, node, q, Kf, r2a_up)) { w.node = nd.escape; continue; }
        if (STRAT != SCATTER && box_upper(q, nd) <= bulk_lim) {
            int2 rg = __ldg(T.range + (node - 1));
            lo = rg.x;
            hi = rg.y;
            w.node = nd.escape;
            return true;
        }
        if (leaf_size > 1) {
            const int2 rg = __ldg(T.range + (node - 1));
            if (rg.y - rg.x < leaf_size) {   // scan this subtree's leaves, then continue after it
                w.cur = rg.x;
                w.end = rg.y;
                w.node = nd.escape;
                continue;
            }
        }
        w.node = nd.left;
    }
}

// Flat form of the same walk for one thread, over the subtree entered at `start` and left at
// `stop`: one node step per loop iteration, and every accepted item (a single leaf, or the
// whole leaf range of a subtree inside the query radius) passed to emit(lo, hi) in DFS order.
// The decisions are next_item's, step for step (with the same leaf_size cutoff: a small
// subtree's leaves tested in sorted order); a warp running this loop reconverges once per node
// step instead of once per accepted item.  Returns false if emit refused an item.
template <int STRAT, typename EMIT>
__device__ __forceinline__ bool walk_subtree(const DevTree &T, int start, int stop, double px, double py, double pz,
                                             double K, double r2a, EMIT &emit, int leaf_size = 1)
{
    const int64_t n = T.n;
    const QBox q = make_qbox(px, py, pz);
    const float Kf = (float)K;
    const float r2a_up = __double2float_ru(r2a);
    const float bulk_lim = __fmul_rd(__double2float_rd(r2a), MARGIN_DN);
    const int64_t limit = 4 * n + 64;
    int64_t guard = 0;
    int node = start;
    while (node != stop) {
        if (++guard > limit) {
            flag(T.status, ST_TRAVERSAL);
            break;
        }
        int64_t lo = -1, hi = -1;
        if (node >= n) {
            const int64_t b = node - n;
            const double4 L = ldg4(T.leaf + b);
            node = __ldg(T.leaf_escape + b);
            double r2;
            if (STRAT == GATHER) r2 = r2a;
            else {
                const double r = __dmul_rn(K, L.w);
                const double rr = __dmul_rn(r, r);
                r2 = STRAT == SCATTER ? rr : (r2a > rr ? r2a : rr);
            }
            if (d2_point(px, py, pz, L) <= r2) lo = hi = b;
        } else {
            const NodeF nd = load_node(T.node + (node - 1));
            if (node_pruned<STRAT>(T, nd, node, q, Kf, r2a_up)) {
                node = nd.escape;
            } else if (STRAT != SCATTER && box_upper(q, nd) <= bulk_lim) {
                const int2 rg = __ldg(T.range + (node - 1));
                lo = rg.x;
                hi = rg.y;
                node = nd.escape;
            } else if (leaf_size > 1 && __ldg(&T.range[node - 1].y) - __ldg(&T.range[node - 1].x) < leaf_size) {
                const int2 rg = __ldg(T.range + (node - 1));
                for (int64_t b = rg.x; b <= rg.y; ++b) {   // the subtree's leaves in sorted order
                    if (++guard > limit) {
                        flag(T.status, ST_TRAVERSAL);
                        return true;
                    }
                    const double4 L = ldg4(T.leaf + b);
                    double r2;
                    if (STRAT == GATHER) r2 = r2a;
                    else {
                        const double r = __dmul_rn(K, L.w);
                        const double rr = __dmul_rn(r, r);
                        r2 = STRAT == SCATTER ? rr : (r2a > rr ? r2a : rr);
                    }
                    if (d2_point(px, py, pz, L) <= r2 && !emit(b, b)) return false;
                }
                node = nd.escape;
            } else {
                node = nd.left;
            }
        }
        if (lo >= 0 && !emit(lo, hi)) return false;
    }
    return true;
}

// Slot filler shared by the warp-per-query kernels: accepted leaves, in DFS order, are
// dealt to the 32 lanes (the k-th accepted leaf goes to lane k mod 32); PROC(fill) is
// called whenever 32 slots are full and once more for the remainder.
struct Slots {
    int fill;
    int64_t mine;   // this lane's leaf in the current batch (-1 if none)
};

template <typename PROC>
__device__ __forceinline__ void deal(Slots &S, int lane, int64_t lo, int64_t hi, PROC &proc)
{
    while (lo <= hi) {
        int64_t t = hi - lo + 1;
        int room = 32 - S.fill;
        if (t > room) t = room;
        if (lane >= S.fill && lane < S.fill + (int)t) S.mine = lo + (lane - S.fill);
        S.fill += (int)t;
        lo += t;
        if (S.fill == 32) {
            proc(32);
            S.fill = 0;
            S.mine = -1;
        }
    }
}

// query scheduling: warps take queries in the given order from a global counter
__device__ __forceinline__ int64_t next_query(unsigned long long *counter, int lane)
{
    unsigned long long q = 0;
    if (lane == 0) q = atomicAdd(counter, 1ULL);
    return (int64_t)__shfl_sync(0xffffffffu, q, 0);
}

// --------------------------------------------------------------------------------------
// Dealing of a walked query's accepted leaves (its items in subtree order, the runs of each
// item chunk by chunk) to the 32 lanes in DFS order: the k-th accepted leaf goes to lane
// k mod 32.  first(b) is called with the first leaf of every non-empty item (the callee uses
// the very first one); one(mine) for every full batch (every lane holds a leaf); two(m1) for
// two consecutive full batches inside one run (lane leaves m1 and m1 + 32) when cantwo()
// allows it, and four(m1) for four of them (m1, m1 + 32, m1 + 64, m1 + 96) when canfour()
// does.  Within a chunk, lane l finds the run holding its leaf through a uniform run cursor,
// or a binary search over the inclusive prefix sums of the run lengths held one per lane
// when a batch spans several runs.  Leaf indices are 32-bit (n <= 2^30), and so is every
// count: an item's accepted leaves lie in one subtree.  Returns the fill of the last,
// partial batch, whose leaves are left in `mine` (-1 on empty lanes).
template <typename FIRST, typename ONE, typename TWO, typename CANTWO, typename FOUR, typename CANFOUR>
__device__ __forceinline__ int deal_runs(const RunPool &P, int64_t j, int lane, FIRST &first, ONE &one, TWO &two,
                                         CANTWO &cantwo, FOUR &four, CANFOUR &canfour, int &mine)
{
    const int ns = P.ns;
    int fill = 0;
    mine = -1;
    for (int s0 = 0; s0 < ns; s0 += 32) {
        const int2 itm = s0 + lane < ns ? __ldg(P.items + j * ns + s0 + lane) : make_int2(-1, 0);
        unsigned nonempty = __ballot_sync(0xffffffffu, itm.y > 0);
        while (nonempty) {
            const int l = __ffs(nonempty) - 1;
            nonempty &= nonempty - 1;
            int c = __shfl_sync(0xffffffffu, itm.x, l);
            int left = __shfl_sync(0xffffffffu, itm.y, l);
            first((int)__ldg(&P.runs[(int64_t)c * RUN_CHUNK].x));
            while (left > 0) {
                const int cnt = left < RUN_CHUNK ? left : RUN_CHUNK;
                const uint2 rn = lane < cnt ? __ldg(P.runs + (int64_t)c * RUN_CHUNK + lane) : make_uint2(0u, 0u);
                const int nextc = left > RUN_CHUNK ? __ldg(P.next + c) : -1;
                int inc = (int)rn.y;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    int v = __shfl_up_sync(0xffffffffu, inc, o);
                    if (lane >= o) inc += v;
                }
                const int tot = __shfl_sync(0xffffffffu, inc, 31);
                const int ex_own = inc - (int)rn.y;
                int tb = -fill;
                // uniform cursor: run r0 holds leaf position max(tb, 0) of the chunk; a batch
                // inside one run needs no search
                int r0 = -1, rc = -1;
                int end0 = 0, lo0 = 0, ex0 = 0;
                for (;;) {
                    // t0 < tot = inc[cnt - 1], so the cursor stops at a run of this chunk
                    const int t0 = tb <= 0 ? 0 : (tb < tot ? tb : tot - 1);
                    while (end0 <= t0 && r0 < 31) {
                        ++r0;
                        end0 = __shfl_sync(0xffffffffu, inc, r0);
                    }
                    if (tb >= 0 && tb + 64 <= end0) {
                        if (rc != r0) {
                            lo0 = __shfl_sync(0xffffffffu, (int)rn.x, r0);
                            ex0 = __shfl_sync(0xffffffffu, ex_own, r0);
                            rc = r0;
                        }
                        const int m1 = lo0 + (tb - ex0) + lane;
                        if (tb + 128 <= end0 && canfour()) {   // four full batches inside one run
                            four(m1);
                            tb += 128;
                            continue;
                        }
                        if (cantwo()) {   // two full batches inside one run
                            two(m1);
                            tb += 64;
                            continue;   // the next pass assigns or closes what is left of the chunk
                        }
                    }
                    if (tb >= 0 && tb + 32 <= end0) {
                        if (rc != r0) {
                            lo0 = __shfl_sync(0xffffffffu, (int)rn.x, r0);
                            ex0 = __shfl_sync(0xffffffffu, ex_own, r0);
                            rc = r0;
                        }
                        mine = lo0 + (tb - ex0) + lane;
                    } else {
                        const int tl = tb + lane;
                        const bool here = tl >= 0 && tl < tot;
                        const int tt = here ? tl : 0;
                        int r = 0;
#pragma unroll
                        for (int sh = 16; sh > 0; sh >>= 1) {
                            int v = __shfl_sync(0xffffffffu, inc, r + sh - 1);
                            if (v <= tt) r += sh;
                        }
                        const int lo = __shfl_sync(0xffffffffu, (int)rn.x, r);
                        const int ex = __shfl_sync(0xffffffffu, ex_own, r);
                        if (here) mine = lo + (tt - ex);
                    }
                    if (tb + 31 < tot) {
                        one(mine);   // full batch
                        mine = -1;
                        tb += 32;
                    } else {
                        fill = tot - tb;
                        break;
                    }
                }
                left -= cnt;
                c = nextc;
            }
        }
    }
    return fill;
}

// the n == 1 tree has no internal node: its single leaf is tested directly
template <int STRAT>
__device__ __forceinline__ bool single_leaf_accepted(const DevTree &T, double px, double py, double pz, double K,
                                                     double r2a, double4 &L, double &d2)
{
    L = ldg4(T.leaf);
    double r = __dmul_rn(K, L.w), rr = __dmul_rn(r, r);
    double r2 = STRAT == GATHER ? r2a : (STRAT == SCATTER ? rr : (r2a > rr ? r2a : rr));
    d2 = d2_point(px, py, pz, L);
    return d2 <= r2;
}

// --------------------------------------------------------------------------------------
// Exact FP64 accumulator (the reference's arithmetic)
template <int STRAT>
struct Exact64 {
    double S1;
    double SA[MAXU];
    double Bq[3];
    double Fg[MAXG][3];
    double Bd[3], Sd;
    double D[MAXD];
    double Cc[MAXC][3];

    __device__ __forceinline__ void init()
    {
        S1 = 0.0;
#pragma unroll
        for (int u = 0; u < MAXU; ++u) SA[u] = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) { Bq[d] = 0.0; Bd[d] = 0.0; }
        Sd = 0.0;
#pragma unroll
        for (int j = 0; j < MAXG; ++j) Fg[j][0] = Fg[j][1] = Fg[j][2] = 0.0;
#pragma unroll
        for (int j = 0; j < MAXD; ++j) D[j] = 0.0;
#pragma unroll
        for (int j = 0; j < MAXC; ++j) Cc[j][0] = Cc[j][1] = Cc[j][2] = 0.0;
    }

    __device__ __forceinline__ void add(const DevTree &T, const DevCatalog &C, bool need_grad, double px, double py,
                                        double pz, const double4 &L, int64_t b, double d2, double ha, double hb)
    {
        const int k = T.kernel;
        double dx = px - L.x, dy = py - L.y, dz = pz - L.z;
        double dr = sqrt(d2);
        double mb = __ldg(T.m + b), rb = __ldg(T.rho + b);
        double W;
        if (STRAT == SYMMETRIC) W = 0.5 * (Wfun<double>(k, dr, ha) + Wfun<double>(k, dr, hb));
        else W = Wfun<double>(k, dr, STRAT == GATHER ? ha : hb);
        double w = mb * W / rb;
        S1 += w;
        double A[MAXU];
#pragma unroll
        for (int u = 0; u < MAXU; ++u) {
            A[u] = (u < C.nU) ? __ldg(C.ucol[u] + b) : 0.0;
            if (u < C.nU) SA[u] += A[u] * w;
        }
        if (!need_grad) return;
        double gx, gy, gz;
        if (STRAT == SYMMETRIC) {
            double ax, ay, az, bx, by, bz;
            gradW<double>(k, dx, dy, dz, dr, ha, ax, ay, az);
            gradW<double>(k, dx, dy, dz, dr, hb, bx, by, bz);
            gx = 0.5 * (ax + bx); gy = 0.5 * (ay + by); gz = 0.5 * (az + bz);
        } else {
            gradW<double>(k, dx, dy, dz, dr, STRAT == GATHER ? ha : hb, gx, gy, gz);
        }
        double invrb = 1.0 / rb;
        double ml = mb * invrb;
        double qx = ml * gx, qy = ml * gy, qz = ml * gz;
        Bq[0] += qx; Bq[1] += qy; Bq[2] += qz;
#pragma unroll
        for (int j = 0; j < MAXG; ++j) {
            if (j < C.n_grad) {
                int u = C.g_u[j];
                if (u < 0) {   // density gradient (gradient_accumulation.jl:160-182)
                    double mx = mb * gx, my = mb * gy, mz = mb * gz;
                    Fg[j][0] += mx; Fg[j][1] += my; Fg[j][2] += mz;
                    Bd[0] += mx * invrb; Bd[1] += my * invrb; Bd[2] += mz * invrb;
                    Sd += mb * W;
                } else {
                    double a = pick<MAXU>(A, u);
                    Fg[j][0] += qx * a; Fg[j][1] += qy * a; Fg[j][2] += qz * a;
                }
            }
        }
#pragma unroll
        for (int j = 0; j < MAXD; ++j) {
            if (j < C.n_div) {
                double ax = pick<MAXU>(A, C.d_u[j][0]), ay = pick<MAXU>(A, C.d_u[j][1]), az = pick<MAXU>(A, C.d_u[j][2]);
                D[j] += qx * ax + qy * ay + qz * az;
            }
        }
#pragma unroll
        for (int j = 0; j < MAXC; ++j) {
            if (j < C.n_curl) {
                double ax = pick<MAXU>(A, C.c_u[j][0]), ay = pick<MAXU>(A, C.c_u[j][1]), az = pick<MAXU>(A, C.c_u[j][2]);
                Cc[j][0] += ay * qz - az * qy;
                Cc[j][1] += az * qx - ax * qz;
                Cc[j][2] += ax * qy - ay * qx;
            }
        }
    }

    __device__ __forceinline__ void finalize(const DevCatalog &C, int64_t qi) const
    {
        int l = 0;
        if (S1 == 0.0) {
            for (int o = 0; o < C.L; ++o) C.out[o][qi] = __longlong_as_double(0x7ff8000000000000LL);
            return;
        }
        double inv = 1.0 / S1;
#pragma unroll
        for (int j = 0; j < MAXS; ++j) {
            if (j < C.n_scalar) {
                double s = pick<MAXU>(SA, C.s_u[j]);
                C.out[l++][qi] = C.s_shep[j] ? s * inv : s;
            }
        }
#pragma unroll
        for (int j = 0; j < MAXG; ++j) {
            if (j < C.n_grad) {
                int u = C.g_u[j];
                if (u < 0) {
                    double a = Sd * inv;
                    C.out[l++][qi] = Fg[j][0] - Bd[0] * a;
                    C.out[l++][qi] = Fg[j][1] - Bd[1] * a;
                    C.out[l++][qi] = Fg[j][2] - Bd[2] * a;
                } else {
                    double a = pick<MAXU>(SA, u) * inv;
                    C.out[l++][qi] = Fg[j][0] - Bq[0] * a;
                    C.out[l++][qi] = Fg[j][1] - Bq[1] * a;
                    C.out[l++][qi] = Fg[j][2] - Bq[2] * a;
                }
            }
        }
#pragma unroll
        for (int j = 0; j < MAXD; ++j) {
            if (j < C.n_div) {
                double ax = pick<MAXU>(SA, C.d_u[j][0]) * inv;
                double ay = pick<MAXU>(SA, C.d_u[j][1]) * inv;
                double az = pick<MAXU>(SA, C.d_u[j][2]) * inv;
                double bb = ax * Bq[0] + ay * Bq[1] + az * Bq[2];
                C.out[l++][qi] = D[j] - bb;
            }
        }
#pragma unroll
        for (int j = 0; j < MAXC; ++j) {
            if (j < C.n_curl) {
                double ax = pick<MAXU>(SA, C.c_u[j][0]) * inv;
                double ay = pick<MAXU>(SA, C.c_u[j][1]) * inv;
                double az = pick<MAXU>(SA, C.c_u[j][2]) * inv;
                double bx = ay * Bq[2] - az * Bq[1];
                double by = az * Bq[0] - ax * Bq[2];
                double bz = ax * Bq[1] - ay * Bq[0];
                C.out[l++][qi] = -(Cc[j][0] - bx);
                C.out[l++][qi] = -(Cc[j][1] - by);
                C.out[l++][qi] = -(Cc[j][2] - bz);
            }
        }
    }
};

// --------------------------------------------------------------------------------------
// FP32 compensated accumulator
template <int STRAT>
struct Comp32 {
    CSum S1;
    CSum SA[MAXU];
    CSum Bq[3];
    CSum Fg[MAXG][3];
    CSum D[MAXD];
    CSum Cc[MAXC][3];
    double Ahat[MAXU];
    bool have;

    __device__ __forceinline__ void init()
    {
        S1.zero();
#pragma unroll
        for (int u = 0; u < MAXU; ++u) { SA[u].zero(); Ahat[u] = 0.0; }
#pragma unroll
        for (int d = 0; d < 3; ++d) Bq[d].zero();
#pragma unroll
        for (int j = 0; j < MAXG; ++j) { Fg[j][0].zero(); Fg[j][1].zero(); Fg[j][2].zero(); }
#pragma unroll
        for (int j = 0; j < MAXD; ++j) D[j].zero();
#pragma unroll
        for (int j = 0; j < MAXC; ++j) { Cc[j][0].zero(); Cc[j][1].zero(); Cc[j][2].zero(); }
        have = false;
    }

    __device__ __forceinline__ void add(const DevTree &T, const DevCatalog &C, bool need_grad, double px, double py,
                                        double pz, const double4 &L, int64_t b, double d2, double ha, double hb)
    {
        const int k = T.kernel;
        float dx = (float)(px - L.x), dy = (float)(py - L.y), dz = (float)(pz - L.z);
        float dr = sqrtf((float)d2);
        float mb = (float)__ldg(T.m + b), rb = (float)__ldg(T.rho + b);
        float fha = (float)ha, fhb = (float)hb;
        float W;
        if (STRAT == SYMMETRIC) W = 0.5f * (Wfun<float>(k, dr, fha) + Wfun<float>(k, dr, fhb));
        else W = Wfun<float>(k, dr, STRAT == GATHER ? fha : fhb);
        float w = mb * W / rb;
        S1.add(w);
        float a[MAXU];
#pragma unroll
        for (int u = 0; u < MAXU; ++u) {
            double A = (u < C.nU) ? __ldg(C.ucol[u] + b) : 0.0;
            if (!have) Ahat[u] = A;
            a[u] = (float)(A - Ahat[u]);
            if (u < C.nU) SA[u].add(a[u] * w);
        }
        have = true;
        if (!need_grad) return;
        float gx, gy, gz;
        if (STRAT == SYMMETRIC) {
            float ax, ay, az, bx, by, bz;
            gradW<float>(k, dx, dy, dz, dr, fha, ax, ay, az);
            gradW<float>(k, dx, dy, dz, dr, fhb, bx, by, bz);
            gx = 0.5f * (ax + bx); gy = 0.5f * (ay + by); gz = 0.5f * (az + bz);
        } else {
            gradW<float>(k, dx, dy, dz, dr, STRAT == GATHER ? fha : fhb, gx, gy, gz);
        }
        float ml = mb / rb;
        float qx = ml * gx, qy = ml * gy, qz = ml * gz;
        Bq[0].add(qx); Bq[1].add(qy); Bq[2].add(qz);
#pragma unroll
        for (int j = 0; j < MAXG; ++j) {
            if (j < C.n_grad) {
                float av = pick<MAXU>(a, C.g_u[j]);
                Fg[j][0].add(qx * av); Fg[j][1].add(qy * av); Fg[j][2].add(qz * av);
            }
        }
#pragma unroll
        for (int j = 0; j < MAXD; ++j) {
            if (j < C.n_div) {
                float ax = pick<MAXU>(a, C.d_u[j][0]), ay = pick<MAXU>(a, C.d_u[j][1]), az = pick<MAXU>(a, C.d_u[j][2]);
                D[j].add(qx * ax + qy * ay + qz * az);
            }
        }
#pragma unroll
        for (int j = 0; j < MAXC; ++j) {
            if (j < C.n_curl) {
                float ax = pick<MAXU>(a, C.c_u[j][0]), ay = pick<MAXU>(a, C.c_u[j][1]), az = pick<MAXU>(a, C.c_u[j][2]);
                Cc[j][0].add(ay * qz - az * qy);
                Cc[j][1].add(az * qx - ax * qz);
                Cc[j][2].add(ax * qy - ay * qx);
            }
        }
    }

    __device__ __forceinline__ void finalize(const DevCatalog &C, int64_t qi) const
    {
        int l = 0;
        double S = S1.val();
        if (S == 0.0) {
            for (int o = 0; o < C.L; ++o) C.out[o][qi] = __longlong_as_double(0x7ff8000000000000LL);
            return;
        }
        double abar[MAXU];
#pragma unroll
        for (int u = 0; u < MAXU; ++u) abar[u] = SA[u].val() / S;
        double B[3] = {Bq[0].val(), Bq[1].val(), Bq[2].val()};
#pragma unroll
        for (int j = 0; j < MAXS; ++j) {
            if (j < C.n_scalar) {
                int u = C.s_u[j];
                double ah = pick<MAXU>(Ahat, u);
                C.out[l++][qi] = C.s_shep[j] ? ah + pick<MAXU>(abar, u) : ah * S + pick<MAXU>(abar, u) * S;
            }
        }
#pragma unroll
        for (int j = 0; j < MAXG; ++j) {
            if (j < C.n_grad) {
                double a = pick<MAXU>(abar, C.g_u[j]);
                C.out[l++][qi] = Fg[j][0].val() - a * B[0];
                C.out[l++][qi] = Fg[j][1].val() - a * B[1];
                C.out[l++][qi] = Fg[j][2].val() - a * B[2];
            }
        }
#pragma unroll
        for (int j = 0; j < MAXD; ++j) {
            if (j < C.n_div) {
                double ax = pick<MAXU>(abar, C.d_u[j][0]), ay = pick<MAXU>(abar, C.d_u[j][1]),
                       az = pick<MAXU>(abar, C.d_u[j][2]);
                C.out[l++][qi] = D[j].val() - (ax * B[0] + ay * B[1] + az * B[2]);
            }
        }
#pragma unroll
        for (int j = 0; j < MAXC; ++j) {
            if (j < C.n_curl) {
                double ax = pick<MAXU>(abar, C.c_u[j][0]), ay = pick<MAXU>(abar, C.c_u[j][1]),
                       az = pick<MAXU>(abar, C.c_u[j][2]);
                double bx = ay * B[2] - az * B[1];
                double by = az * B[0] - ax * B[2];
                double bz = ax * B[1] - ay * B[0];
                C.out[l++][qi] = -(Cc[j][0].val() - bx);
                C.out[l++][qi] = -(Cc[j][1].val() - by);
                C.out[l++][qi] = -(Cc[j][2].val() - bz);
            }
        }
    }
};

// --------------------------------------------------------------------------------------
// point-sample kernel: one thread per (Morton-ordered) sample point
template <template <int> class ACC, int STRAT>
__global__ void __launch_bounds__(128) k_points(DevTree T, DevCatalog C, int64_t nq, const double *__restrict__ qx,
                                                const double *__restrict__ qy, const double *__restrict__ qz,
                                                const uint32_t *__restrict__ perm)
{
    const int64_t n = T.n;
    const double K = kernel_valid(T.kernel);
    const bool need_grad = (C.n_grad + C.n_div + C.n_curl) > 0;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nq; j += (int64_t)gridDim.x * blockDim.x) {
        int64_t qi = perm ? (int64_t)__ldg(perm + j) : j;
        if (qi >= nq) continue;   // unreachable for a valid permutation
        double px = __ldg(qx + qi), py = __ldg(qy + qi), pz = __ldg(qz + qi);
        double ha = 0.0;
        if (STRAT != SCATTER) {
            int64_t b = nearest_leaf(T, px, py, pz);
            ha = b < 0 ? __longlong_as_double(0x7ff8000000000000LL) : ldg4(T.leaf + b).w;
        }
        double ra = __dmul_rn(K, ha);
        double r2a = __dmul_rn(ra, ra);
        ACC<STRAT> acc;
        acc.init();
        double4 L;
        double d2;
        if (T.root == 0) {
            if (single_leaf_accepted<STRAT>(T, px, py, pz, K, r2a, L, d2))
                acc.add(T, C, need_grad, px, py, pz, L, 0, d2, ha, L.w);
        } else {
            Walk w{T.root, 1, 0, 0, 4 * n + 64};
            int64_t b;
            while ((b = next_accepted<STRAT>(T, w, px, py, pz, K, r2a, L, d2)) >= 0)
                acc.add(T, C, need_grad, px, py, pz, L, b, d2, ha, L.w);
        }
        acc.finalize(C, qi);
    }
}

// --------------------------------------------------------------------------------------
// line-sample kernel (itpScatter): one thread per line
template <typename R>
__device__ __forceinline__ R line_lut(const R *__restrict__ I, R qmax, R q)
{
    const R dq = qmax / R(PB_LINE_NTAB_DEV - 1);
    R idxf = q / dq + R(1);
    int i = (int)idxf;
    i = i < 1 ? 1 : (i > PB_LINE_NTAB_DEV - 1 ? PB_LINE_NTAB_DEV - 1 : i);
    R t = idxf - R(i);
    return __ldg(I + i - 1) * (R(1) - t) + __ldg(I + i) * t;
}

// FP32 table, index and interpolation fraction formed in FP64 from an FP64 q: near the support
// edge the line-integrated kernel is small and steep, and an FP32 q / dq would move the
// fraction by ~4e-4 of a table step
__device__ __forceinline__ float line_lut_q64(const float *__restrict__ I, double qmax, double q)
{
    const double dq = qmax / double(PB_LINE_NTAB_DEV - 1);
    const double idxf = q / dq + 1.0;
    int i = (int)idxf;
    i = i < 1 ? 1 : (i > PB_LINE_NTAB_DEV - 1 ? PB_LINE_NTAB_DEV - 1 : i);
    const float t = (float)(idxf - (double)i);
    return __ldg(I + i - 1) * (1.f - t) + __ldg(I + i) * t;
}

template <typename R>
__global__ void __launch_bounds__(128) k_lines(DevTree T, DevCatalog C, int64_t nl, const double *__restrict__ ox,
                                               const double *__restrict__ oy, const double *__restrict__ oz,
                                               const double *__restrict__ mx, const double *__restrict__ my,
                                               const double *__restrict__ mz, const uint32_t *__restrict__ perm,
                                               const R *__restrict__ table)
{
    const int64_t n = T.n;
    const int k = T.kernel;
    const double K = kernel_valid(k);
    const R qmax = (R)K;
    const R *I = table + (int64_t)k * PB_LINE_NTAB_DEV;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nl; j += (int64_t)gridDim.x * blockDim.x) {
        int64_t li = perm ? (int64_t)__ldg(perm + j) : j;
        if (li >= nl) continue;
        double o[3] = {__ldg(ox + li), __ldg(oy + li), __ldg(oz + li)};
        double m[3] = {__ldg(mx + li), __ldg(my + li), __ldg(mz + li)};
        // FP64 mode: plain sums in the reference order; FP32 mode: compensated with offsets
        double S1 = 0.0, acc[MAXS];
        CSum cS1, cacc[MAXS];
        double Ahat[MAXS];
        bool have = false;
        cS1.zero();
#pragma unroll
        for (int s = 0; s < MAXS; ++s) { acc[s] = 0.0; cacc[s].zero(); Ahat[s] = 0.0; }
        int node = T.root;
        int64_t bi = 0, guard = 0, limit = 4 * n + 64;
        bool brute = (node == 0);
        while (brute ? (bi < n) : (node != 0)) {
            if (++guard > limit) { flag(T.status, ST_TRAVERSAL); break; }
            bool leafnode = brute || node >= n;
            if (leafnode) {
                int64_t b = brute ? bi++ : (int64_t)(node - n);
                double4 L = ldg4(T.leaf + b);
                int esc = brute ? 0 : __ldg(T.leaf_escape + b);
                double r = __dmul_rn(K, L.w);
                double r2 = __dmul_rn(r, r);
                double d2 = d2_line(L.x, L.y, L.z, o, m);
                if (d2 <= r2) {
                    double mb = __ldg(T.m + b), rb = __ldg(T.rho + b);
                    if (sizeof(R) == 8) {
                        // line_integrated_kernel_function (line_integrated_kernel.jl:132-137)
                        double dr = sqrt(d2 > 0.0 ? d2 : 0.0);
                        double invh = 1.0 / L.w;
                        double q = dr * invh;
                        double Iq = (q >= K) ? 0.0 : (double)line_lut<R>(I, qmax, (R)q);
                        double W = invh * Iq;
                        double w = mb * W / rb;
                        S1 += w;
#pragma unroll
                        for (int s = 0; s < MAXS; ++s)
                            if (s < C.n_scalar) acc[s] += __ldg(C.ucol[C.s_u[s]] + b) * w;
                    } else {
                        // the line distance and q in FP64 (the pair-distance part), the kernel
                        // value and the sums in FP32
                        const double q = sqrt(d2 > 0.0 ? d2 : 0.0) * (1.0 / L.w);
                        const float invh = (float)(1.0 / L.w);
                        float Iq = (q >= K) ? 0.f : line_lut_q64(reinterpret_cast<const float *>(I), K, q);
                        float w = (float)mb * (invh * Iq) / (float)rb;
                        cS1.add(w);
#pragma unroll
                        for (int s = 0; s < MAXS; ++s) {
                            if (s < C.n_scalar) {
                                double A = __ldg(C.ucol[C.s_u[s]] + b);
                                if (!have) Ahat[s] = A;
                                cacc[s].add((float)(A - Ahat[s]) * w);
                            }
                        }
                        have = true;
                    }
                }
                if (!brute) node = esc;
            } else {
                NodeF nd = load_node(T.node + (node - 1));
                double r = __dmul_rn(K, (double)__ldg(T.node_hmax + (node - 1)));
                double r2 = __dmul_rn(r, r);
                node = (d2_line_box_lower(o, m, nd) > r2) ? nd.escape : nd.left;
            }
        }
        double S = (sizeof(R) == 8) ? S1 : cS1.val();
        int l = 0;
#pragma unroll
        for (int s = 0; s < MAXS; ++s) {
            if (s < C.n_scalar) {
                double v;
                if (S == 0.0) v = __longlong_as_double(0x7ff8000000000000LL);
                else if (sizeof(R) == 8) v = C.s_shep[s] ? acc[s] * (1.0 / S) : acc[s];
                else v = C.s_shep[s] ? Ahat[s] + cacc[s].val() / S : Ahat[s] * S + cacc[s].val();
                C.out[l++][li] = v;
            }
        }
    }
}

}  // namespace pb
