// pb_fp64_impl.cuh -- the FP64 per-pair terms with the reference's expressions and the
// in-order column sums of the warp-per-query kernels, and the fused per-query body.  Shared by
// pb_interp64.cu and the batched kernel (pb_batch.cu); both are compiled with -fmad=false, so
// the values are the reference's FP64 results bit for bit in either.
#pragma once
#include "pb_interp_impl.cuh"

namespace pb {

// ------------------------------------------------------------------------------------
// Warp-per-query FP64 kernel.  Accepted leaves are dealt to the 32 lanes in DFS order;
// each lane computes its pair's terms with the reference's expressions, the terms go to
// shared memory, and lane a then adds term a of every slot, in slot (= DFS) order, to its
// accumulator -- the reference's sequential sums, bit for bit, with the per-pair work
// spread over the warp.
constexpr int NT = 19;   // S1, SA[4], Bq[3], Fg[3], Bd[3], Sd, D, Cc[3]

template <int STRAT>
__device__ __forceinline__ void terms64(const DevTree &T, const DevCatalog &C, bool need_grad, double px, double py,
                                        double pz, int64_t b, double ha, double *t)
{
    const int k = T.kernel;
    double4 L = ldg4(T.leaf + b);
    double hb = L.w;
    double d2 = d2_point(px, py, pz, L);
    double dx = px - L.x, dy = py - L.y, dz = pz - L.z;
    double dr = sqrt(d2);
    double mb = __ldg(T.m + b), rb = __ldg(T.rho + b);
    double W;
    if (STRAT == SYMMETRIC) W = 0.5 * (Wfun<double>(k, dr, ha) + Wfun<double>(k, dr, hb));
    else W = Wfun<double>(k, dr, STRAT == GATHER ? ha : hb);
    double w = mb * W / rb;
    t[0] = w;
    double A[MAXU];
#pragma unroll
    for (int u = 0; u < MAXU; ++u) {
        A[u] = (u < C.nU) ? __ldg(C.ucol[u] + b) : 0.0;
        t[1 + u] = A[u] * w;
    }
#pragma unroll
    for (int a = 5; a < NT; ++a) t[a] = 0.0;
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
    t[5] = qx; t[6] = qy; t[7] = qz;
    if (C.n_grad > 0) {
        int u = C.g_u[0];
        if (u < 0) {
            double mx = mb * gx, my = mb * gy, mz = mb * gz;
            t[8] = mx; t[9] = my; t[10] = mz;
            t[11] = mx * invrb; t[12] = my * invrb; t[13] = mz * invrb;
            t[14] = mb * W;
        } else {
            double a = pick<MAXU>(A, u);
            t[8] = qx * a; t[9] = qy * a; t[10] = qz * a;
        }
    }
    if (C.n_div > 0) {
        double ax = pick<MAXU>(A, C.d_u[0][0]), ay = pick<MAXU>(A, C.d_u[0][1]), az = pick<MAXU>(A, C.d_u[0][2]);
        t[15] = qx * ax + qy * ay + qz * az;
    }
    if (C.n_curl > 0) {
        double ax = pick<MAXU>(A, C.c_u[0][0]), ay = pick<MAXU>(A, C.c_u[0][1]), az = pick<MAXU>(A, C.c_u[0][2]);
        t[16] = ay * qz - az * qy;
        t[17] = az * qx - ax * qz;
        t[18] = ax * qy - ay * qx;
    }
}

__device__ __forceinline__ void finalize64(const double *v, const DevCatalog &C, int64_t qi)
{
    Exact64<SYMMETRIC> A;   // the finalisation does not depend on the strategy
    A.S1 = v[0];
#pragma unroll
    for (int u = 0; u < MAXU; ++u) A.SA[u] = v[1 + u];
    A.Bq[0] = v[5]; A.Bq[1] = v[6]; A.Bq[2] = v[7];
    A.Fg[0][0] = v[8]; A.Fg[0][1] = v[9]; A.Fg[0][2] = v[10];
    A.Bd[0] = v[11]; A.Bd[1] = v[12]; A.Bd[2] = v[13];
    A.Sd = v[14];
    A.D[0] = v[15];
    A.Cc[0][0] = v[16]; A.Cc[0][1] = v[17]; A.Cc[0][2] = v[18];
    A.finalize(C, qi);
}

// The fused FP64 sum of one query: the warp walks the tree (warp-uniform next_item), deals the
// accepted leaves to its lanes, each lane computes its pair's terms into the warp's slot array
// sterm ([32][NT + 1] doubles), and lane a adds term a of every slot in DFS order.  bnear is
// the nearest sorted leaf (-1 for itpScatter); leaf_size the walk's linear-scan cutoff.
template <int STRAT>
__device__ __forceinline__ void points64_query(const DevTree &T, const DevCatalog &C, double px, double py, double pz,
                                               int64_t bnear, int64_t qi, double *sterm, int lane, int leaf_size)
{
    const int64_t n = T.n;
    const double K = kernel_valid(T.kernel);
    const bool need_grad = (C.n_grad + C.n_div + C.n_curl) > 0;
    double ha = 0.0;
    if (STRAT != SCATTER) ha = bnear < 0 ? __longlong_as_double(0x7ff8000000000000LL) : ldg4(T.leaf + bnear).w;
    const double ra = __dmul_rn(K, ha), r2a = __dmul_rn(ra, ra);
    double acc = 0.0;   // lane a < NT owns accumulator a
    Slots S{0, -1};
    auto proc = [&](int fill) {
        if (S.mine >= 0) {
            double t[NT];
            terms64<STRAT>(T, C, need_grad, px, py, pz, S.mine, ha, t);
#pragma unroll
            for (int a = 0; a < NT; ++a) sterm[lane * (NT + 1) + a] = t[a];
        }
        __syncwarp();
        if (lane < NT)
            for (int s = 0; s < fill; ++s) acc += sterm[s * (NT + 1) + lane];
        __syncwarp();
    };
    if (T.root == 0) {
        double4 L;
        double d2;
        if (single_leaf_accepted<STRAT>(T, px, py, pz, K, r2a, L, d2)) deal(S, lane, 0, 0, proc);
    } else {
        Walk w{T.root, 1, 0, 0, 4 * n + 64};
        int64_t lo, hi;
        while (next_item<STRAT>(T, w, px, py, pz, K, r2a, lo, hi, leaf_size)) deal(S, lane, lo, hi, proc);
    }
    if (S.fill > 0) proc(S.fill);
    double v[NT];
#pragma unroll
    for (int a = 0; a < NT; ++a) v[a] = __shfl_sync(0xffffffffu, acc, a);
    if (lane == 0) finalize64(v, C, qi);
}

// The two-phase FP64 sum of one walked query j (its runs in the pool P) at sample point qi:
// the accepted leaves dealt in DFS order, the terms and in-order sums of points64_query.
template <int STRAT>
__device__ __forceinline__ void pairs64_query(const DevTree &T, const DevCatalog &C, const RunPool &P, int64_t j,
                                              int64_t qi, double px, double py, double pz, int64_t bnear,
                                              double *sterm, int lane)
{
    const bool need_grad = (C.n_grad + C.n_div + C.n_curl) > 0;
    double ha = 0.0;
    if (STRAT != SCATTER) ha = bnear < 0 ? __longlong_as_double(0x7ff8000000000000LL) : ldg4(T.leaf + bnear).w;
    double acc = 0.0;   // lane a < NT owns accumulator a
    auto proc = [&](int fill, int64_t b) {
        if (b >= 0) {
            double tv[NT];
            terms64<STRAT>(T, C, need_grad, px, py, pz, b, ha, tv);
#pragma unroll
            for (int a = 0; a < NT; ++a) sterm[lane * (NT + 1) + a] = tv[a];
        }
        __syncwarp();
        if (lane < NT)
            for (int s = 0; s < fill; ++s) acc += sterm[s * (NT + 1) + lane];
        __syncwarp();
    };
    auto first = [&](int64_t) {};
    auto one = [&](int64_t b) { proc(32, b); };
    auto cantwo = [&]() { return false; };
    // never called (cantwo and canfour are false): empty bodies keep the kernels free of a
    // stack frame, which a multi-batch body here would force on the per-pair term array
    auto two = [&](int64_t) {};
    auto four = [&](int64_t) {};
    int mine = -1;
    const int fill = deal_runs(P, j, lane, first, one, two, cantwo, four, cantwo, mine);
    if (fill > 0) proc(fill, mine);
    double v[NT];
#pragma unroll
    for (int a = 0; a < NT; ++a) v[a] = __shfl_sync(0xffffffffu, acc, a);
    if (lane == 0) finalize64(v, C, qi);
}

}  // namespace pb
