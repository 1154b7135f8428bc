// pb_device.cuh -- device-side data layout and arithmetic shared by the LBVH build,
// the traversal/interpolation kernels and the neighbour-query kernels.
//
// Layout in HBM (one particle set per handle, Morton-sorted):
//   leaf[n]        double4 {x, y, z, h}            one 32-byte sector per leaf test
//   leaf_escape[n] int32 unified escape id of each leaf
//   node[n-1]      NodeF {lo.xyz, left | hi.xyz, escape}, 32 bytes, FP32 boxes rounded
//                  outward so every pruning test is conservative against the FP64 tree
//   node_hmax[n-1] float, max smoothing length of the subtree, rounded up
//   m, rho, quant  FP64 particle columns in sorted order
// Unified ids follow the reference (BinaryRadixTree.jl:36-51): internal 1..n-1,
// leaf n..2n-1, 0 = none.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pb {

enum Strategy { GATHER = 0, SCATTER = 1, SYMMETRIC = 2 };

#define PB_LINE_NTAB_DEV 4096

// per-launch catalog limits; larger catalogs are split into several launches
constexpr int MAXU = 4;   // unique quantity columns read per neighbour
constexpr int MAXS = 4;   // scalar outputs
constexpr int MAXG = 1;   // gradient outputs (3 values each)
constexpr int MAXD = 1;   // divergence outputs
constexpr int MAXC = 1;   // curl outputs (3 values each)
constexpr int MAXL = MAXS + 3 * MAXG + MAXD + 3 * MAXC;

// device status word bits (host turns them into error codes)
constexpr int ST_NONFINITE = 1;     // non-finite particle coordinate or smoothing length
constexpr int ST_REFIT = 2;         // an internal node was not combined exactly twice
constexpr int ST_TRAVERSAL = 4;     // a traversal exceeded its iteration bound (corrupt tree)
constexpr int ST_POOL = 8;          // neighbour pool too small for a query
constexpr int ST_CUT = 16;          // a walk cut made on the device had more subtrees than its capacity

struct __align__(16) NodeF {
    float lox, loy, loz;
    int left;
    float hix, hiy, hiz;
    int escape;
};

struct DevTree {
    int64_t n;
    int root;
    const double4 *leaf;
    const int *leaf_escape;
    const NodeF *node;
    const float *node_hmax;
    const int2 *child;      // (left, right) unified ids of each internal node
    const int2 *range;      // 0-based sorted leaf range [lo, hi] of each internal node's subtree
    const double *m;
    const double *rho;
    int kernel;
    int *status;
};

// Accepted-neighbour run lists written by the walk kernel and read by the pair kernels.
// The tree is cut into ns disjoint subtrees whose leaf ranges follow one another in DFS
// order; every (query, subtree) item is walked separately.  A run is a maximal interval of
// consecutive sorted leaves accepted by one item, stored as (first leaf, length); an item's
// runs are kept in DFS (= ascending leaf) order in a linked list of fixed-size chunks drawn
// from one pool, and items[j * ns + s] = (first chunk, number of runs).  Concatenating a
// query's items in subtree order gives its accepted leaves in the reference's DFS order.
constexpr int RUN_CHUNK = 32;
constexpr int RUN_DEFERRED = -2;

struct RunPool {
    uint2 *runs;                  // cap * RUN_CHUNK (first leaf, length)
    int *next;                    // cap chunk links (-1 ends a list)
    unsigned long long *used;     // chunks handed out (may run past cap)
    unsigned long long cap;       // chunks in the pool
    int ns;                       // subtrees of the cut
    const int2 *cut;              // (subtree root, node after the subtree in DFS order) per subtree
    int2 *items;                  // m * ns item heads
    int *bnear;                   // nearest sorted leaf per walked query (-1: none / not needed)
    unsigned *qacc;               // accepted leaves per walked query
    int *qflag;                   // 1: some item of the query found the pool full (deferred)
    unsigned *n_deferred;         // queries deferred in this walk
    uint32_t *deferred;           // their query indices
    int count_only;               // 1: only count accepted leaves (qacc); no runs, no items
    int leaf_size;                // walk cutoff: subtrees of at most this many leaves are scanned
};

// Catalog of one launch.  ucol[] are the unique sorted quantity columns read per
// neighbour; outputs index into them.  g_u == -1 is the density gradient (the
// reference's grad slot 0, general_interpolation.jl:76-81).
struct DevCatalog {
    int nU;
    const double *ucol[MAXU];
    int n_scalar;
    int s_u[MAXS];
    int s_shep[MAXS];
    int n_grad;
    int g_u[MAXG];
    int n_div;
    int d_u[MAXD][3];
    int n_curl;
    int c_u[MAXC][3];
    int L;
    double *out[MAXL];
};

// read-only 32-byte leaf record as two 16-byte loads
__device__ __forceinline__ double4 ldg4(const double4 *p)
{
    const double2 *q = reinterpret_cast<const double2 *>(p);
    double2 a = __ldg(q), b = __ldg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

__host__ __device__ inline double kernel_valid(int k) { return k == 1 ? 2.5 : (k == 2 ? 3.0 : 2.0); }

// ---------------------------------------------------------------------------------
// Squared distances.  Explicit round-to-nearest intrinsics keep these free of FMA
// contraction so that (a) the leaf test reproduces the reference's FP64 value bit for
// bit (LinearBVHTraversalMacros.jl:800-814) and (b) the box bound computed with the same
// operation sequence is never larger than the leaf distance of any leaf inside the box.
__device__ __forceinline__ double d2_point(double px, double py, double pz, const double4 &L)
{
    double dx = __dsub_rn(px, L.x);
    double dy = __dsub_rn(py, L.y);
    double dz = __dsub_rn(pz, L.z);
    double s = __dmul_rn(dx, dx);
    s = __dadd_rn(s, __dmul_rn(dy, dy));
    s = __dadd_rn(s, __dmul_rn(dz, dz));
    return s;
}

__device__ __forceinline__ double axis_gap(double p, double a, double b)
{
    return p < a ? __dsub_rn(a, p) : (p > b ? __dsub_rn(p, b) : 0.0);
}

__device__ __forceinline__ double d2_box(double px, double py, double pz, const NodeF &nd)
{
    double tx = axis_gap(px, (double)nd.lox, (double)nd.hix);
    double ty = axis_gap(py, (double)nd.loy, (double)nd.hiy);
    double tz = axis_gap(pz, (double)nd.loz, (double)nd.hiz);
    double s = __dmul_rn(tx, tx);
    s = __dadd_rn(s, __dmul_rn(ty, ty));
    s = __dadd_rn(s, __dmul_rn(tz, tz));
    return s;
}

// infinite-line distance: Delta2 - (Delta.m)^2 with Delta = p - o (LinearBVHTraversalMacros.jl:859-876)
__device__ __forceinline__ double d2_line(double px, double py, double pz, const double o[3], const double m[3])
{
    double ax = __dsub_rn(px, o[0]), ay = __dsub_rn(py, o[1]), az = __dsub_rn(pz, o[2]);
    double D2 = __dmul_rn(ax, ax);
    double Dm = __dmul_rn(ax, m[0]);
    D2 = __dadd_rn(D2, __dmul_rn(ay, ay));
    Dm = __dadd_rn(Dm, __dmul_rn(ay, m[1]));
    D2 = __dadd_rn(D2, __dmul_rn(az, az));
    Dm = __dadd_rn(Dm, __dmul_rn(az, m[2]));
    return __dsub_rn(D2, __dmul_rn(Dm, Dm));
}

// Conservative lower bound of the line-to-box squared distance, minus a slack that covers
// the cancellation error of d2_line for any point of the box, so that pruning never drops
// a leaf whose computed d2_line passes the acceptance test.
__device__ __forceinline__ double d2_line_box_lower(const double o[3], const double m[3], const NodeF &nd)
{
    double a[3] = {(double)nd.lox, (double)nd.loy, (double)nd.loz};
    double b[3] = {(double)nd.hix, (double)nd.hiy, (double)nd.hiz};
    double tmin = -INFINITY, tmax = INFINITY;
    bool hit = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (m[d] == 0.0) {
            if (o[d] < a[d] || o[d] > b[d]) hit = false;
        } else {
            double t0 = (a[d] - o[d]) / m[d];
            double t1 = (b[d] - o[d]) / m[d];
            double lo = fmin(t0, t1), hi = fmax(t0, t1);
            tmin = fmax(tmin, lo);
            tmax = fmin(tmax, hi);
        }
    }
    if (hit && tmin <= tmax) return 0.0;
    double c[3], r2 = 0.0, oc2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        c[d] = 0.5 * (a[d] + b[d]);
        double hh = 0.5 * (b[d] - a[d]);
        r2 += hh * hh;
        double q = c[d] - o[d];
        oc2 += q * q;
    }
    double dc2 = d2_line(c[0], c[1], c[2], o, m);
    double R = sqrt(r2);
    double far = sqrt(oc2) + R;
    double slack = 1e-12 * far * far + 1e-300;
    if (dc2 <= r2) return 0.0;
    double dl = sqrt(dc2) - R;
    double bound = dl * dl * (1.0 - 1e-12) - slack;
    return bound > 0.0 ? bound : 0.0;
}

// ---------------------------------------------------------------------------------
// Kernel shapes (Partia.jl/src/julia/KernelInterpolation/kernel_function/kernels/*.jl).
// FP64: Julia Float64 semantics -- literal ^2/^3 are plain products, other integer
// powers use Base.Math's compensated power-by-squaring, restated below.
__device__ __forceinline__ double jl_pow(double x, int n)
{
    if (n == 2) return x * x;
    if (n == 3) return x * x * x;
    double y = 1.0, xnlo = -0.0, ynlo = 0.0;
    while (n > 1) {
        if (n & 1) {
            double err = fma(y, xnlo, x * ynlo);
            double p = x * y;
            double lo = fma(x, y, -p);
            y = p;
            ynlo = lo + err;
        }
        double err = x * 2.0 * xnlo;
        double p = x * x;
        double lo = fma(x, x, -p);
        x = p;
        xnlo = lo + err;
        n >>= 1;
    }
    double err = fma(y, xnlo, x * ynlo);
    return (isfinite(x) && isfinite(err)) ? fma(x, y, err) : x * y;
}

__device__ __forceinline__ float jl_pow(float x, int n)
{
    float y = x;
#pragma unroll
    for (int i = 1; i < 8; ++i)
        if (i < n) y *= x;
    return y;
}

template <typename R>
__device__ __forceinline__ R kshape(int k, R q)
{
    if (q < R(0)) return R(NAN);
    switch (k) {
    case 0:
        if (R(0) <= q && q < R(1)) return R(0.25) * jl_pow(R(2) - q, 3) - jl_pow(R(1) - q, 3);
        if (R(1) <= q && q < R(2)) return R(0.25) * jl_pow(R(2) - q, 3);
        return R(0);
    case 1:
        if (R(0) <= q && q < R(0.5))
            return jl_pow(R(2.5) - q, 4) - R(5) * jl_pow(R(1.5) - q, 4) + R(10) * jl_pow(R(0.5) - q, 4);
        if (R(0.5) <= q && q < R(1.5)) return jl_pow(R(2.5) - q, 4) - R(5) * jl_pow(R(1.5) - q, 4);
        if (R(1.5) <= q && q < R(2.5)) return jl_pow(R(2.5) - q, 4);
        return R(0);
    case 2:
        if (R(0) <= q && q < R(1))
            return jl_pow(R(3) - q, 5) - R(6) * jl_pow(R(2) - q, 5) + R(15) * jl_pow(R(1) - q, 5);
        if (R(1) <= q && q < R(2)) return jl_pow(R(3) - q, 5) - R(6) * jl_pow(R(2) - q, 5);
        if (R(2) <= q && q < R(3)) return jl_pow(R(3) - q, 5);
        return R(0);
    case 3:
        if (q < R(2)) return jl_pow(R(1) - R(0.5) * q, 4) * (R(2) * q + R(1));
        return R(0);
    case 4:
        if (q < R(2)) return jl_pow(R(1) - R(0.5) * q, 6) * ((R(35) / R(12)) * (q * q) + R(3) * q + R(1));
        return R(0);
    default:
        if (q < R(2))
            return jl_pow(R(1) - R(0.5) * q, 8) * (R(4) * (q * q * q) + R(6.25) * (q * q) + R(4) * q + R(1));
        return R(0);
    }
}

template <typename R>
__device__ __forceinline__ R kdshape(int k, R q)
{
    if (q < R(0)) return R(NAN);
    switch (k) {
    case 0:
        if (R(0) <= q && q < R(1)) return R(-0.75) * jl_pow(R(2) - q, 2) + R(3) * jl_pow(R(1) - q, 2);
        if (R(1) <= q && q < R(2)) return R(-0.75) * jl_pow(R(2) - q, 2);
        return R(0);
    case 1:
        if (R(0) <= q && q < R(0.5))
            return R(-4) * jl_pow(R(2.5) - q, 3) + R(20) * jl_pow(R(1.5) - q, 3) - R(40) * jl_pow(R(0.5) - q, 3);
        if (R(0.5) <= q && q < R(1.5)) return -R(4) * jl_pow(R(2.5) - q, 3) + R(20) * jl_pow(R(1.5) - q, 3);
        if (R(1.5) <= q && q < R(2.5)) return R(-4) * jl_pow(R(2.5) - q, 3);
        return R(0);
    case 2:
        if (R(0) <= q && q < R(1))
            return R(-5) * jl_pow(R(3) - q, 4) + R(30) * jl_pow(R(2) - q, 4) - R(75) * jl_pow(R(1) - q, 4);
        if (R(1) <= q && q < R(2)) return R(-5) * jl_pow(R(3) - q, 4) + R(30) * jl_pow(R(2) - q, 4);
        if (R(2) <= q && q < R(3)) return R(-5) * jl_pow(R(3) - q, 4);
        return R(0);
    case 3:
        if (q < R(2)) return jl_pow(R(1) - R(0.5) * q, 4) * R(2) - jl_pow(R(1) - R(0.5) * q, 3) * (R(4) * q + R(2));
        return R(0);
    case 4:
        if (q < R(2))
            return jl_pow(R(1) - R(0.5) * q, 6) * ((R(35) / R(6)) * q + R(3)) -
                   jl_pow(R(1) - R(0.5) * q, 5) * ((R(35) / R(4)) * (q * q) + R(9) * q + R(3));
        return R(0);
    default:
        if (q < R(2))
            return jl_pow(R(1) - R(0.5) * q, 8) * (R(12) * (q * q) + R(12.5) * q + R(4)) -
                   jl_pow(R(1) - R(0.5) * q, 7) * (R(16) * (q * q * q) + R(25) * (q * q) + R(16) * q + R(4));
        return R(0);
    }
}

// KernelFunctionnorm(K, Val(3), T): T(a)/(T(b)*T(pi)) evaluated in T
template <typename R>
__device__ __forceinline__ R knorm3(int k)
{
    const R pi = R(3.141592653589793);
    switch (k) {
    case 0: return R(1) / pi;
    case 1: return R(0.05) / pi;
    case 2: return R(1) / (R(120) * pi);
    case 3: return R(21) / (R(16) * pi);
    case 4: return R(495) / (R(256) * pi);
    default: return R(1365) / (R(512) * pi);
    }
}

// Smoothed_kernel_function(K, r, h, Val(3)) -- kernel.jl:152-157
template <typename R>
__device__ __forceinline__ R Wfun(int k, R r, R h)
{
    R invh = R(1) / h;
    R inv_hD = invh * invh * invh;
    R q = r * invh;
    return inv_hD * (knorm3<R>(k) * kshape<R>(k, q));
}

// Smoothed_gradient_kernel_function(K, dx, dy, dz, h) -- kernel.jl:284-296,371-376.
// Only the scalar coefficient is returned: grad = coeff * (dx, dy, dz) with
// coeff = inv_hDp1 * (dW(q)*norm*invr); the reference forms inv_hDp1 * (dx*coeff') per
// component, so the exact path multiplies in that order itself.
template <typename R>
__device__ __forceinline__ void gradW(int k, R dx, R dy, R dz, R r, R h, R &gx, R &gy, R &gz)
{
    R invh = R(1) / h;
    R inv_hDp1 = invh * invh * invh * invh;
    R cx = R(0), cy = R(0), cz = R(0);
    R r2 = dx * dx + dy * dy + dz * dz;
    if (r2 != R(0)) {
        R invr = R(1) / r;
        R q = r / h;
        R coeff = kdshape<R>(k, q) * knorm3<R>(k) * invr;
        cx = dx * coeff;
        cy = dy * coeff;
        cz = dz * coeff;
    }
    gx = inv_hDp1 * cx;
    gy = inv_hDp1 * cy;
    gz = inv_hDp1 * cz;
}

// error-free transformation accumulator (Knuth TwoSum with a running compensation term)
struct CSum {
    float s, c;
    __device__ __forceinline__ void zero() { s = 0.f; c = 0.f; }
    __device__ __forceinline__ void add(float x)
    {
        float t = __fadd_rn(s, x);
        float bp = __fsub_rn(t, s);
        float e = __fadd_rn(__fsub_rn(s, __fsub_rn(t, bp)), __fsub_rn(x, bp));
        s = t;
        c = __fadd_rn(c, e);
    }
    __device__ __forceinline__ double val() const { return (double)s + (double)c; }
};

}  // namespace pb
