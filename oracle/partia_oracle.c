/*
 * partia_oracle.c -- CPU oracle (FP64 restatement) of Partia's LBVH build and SPH grid
 * interpolation path.
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA library and the timed
 * CPU baseline.  The product path never links or calls it.
 *
 * Parity pinning: the reference is Julia and cannot run in this environment, so this
 * restatement is pinned against (a) the known-answer kernel values, normalisations
 * and support radii of Partia.jl/test/kernel_function_tests.jl, (b) the structural
 * invariants and brute-force neighbour checks of Partia.jl/test/neighbor_search_tests.jl
 * on the same deterministic prime-hash coordinates, (c) the brute-force interpolation
 * evaluators of Partia.jl/test/interpolation_test_common.jl on the fixtures of
 * Partia.jl/test/grid_interpolation_test_common.jl, and (d) the reference's tabulated
 * line-integrated kernel (Partia.jl/src/julia/KernelInterpolation/table/
 * line_integrated_kernel_tables.jl, read at test time only).  Field values are
 * otherwise "parity partially pinned": no reference output exists to compare with.
 *
 * Every floating-point expression follows the reference's operation order; compile
 * with -ffp-contract=off (no FMA contraction) so that the results are the IEEE
 * results of that order.
 */
#include "partia_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "line_tables.h"
static const double PB_LINE_INORM[6][PB_LINE_NTAB] = PB_LINE_INORM_INIT;

/* ------------------------------------------------------------------------------------ */
/* Julia's Float64 ^ Int: literal ^2 and ^3 are plain products (Base.literal_pow); other  */
/* integer powers use Base.Math's compensated power-by-squaring (pow_body), restated here. */
double orc_jl_pow(double x, int64_t n)
{
    if (n == 0) return 1.0;
    if (n == 1) return x;
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
#define P(x, n) orc_jl_pow((x), (n))

/* Kernel shapes: Partia.jl/src/julia/KernelInterpolation/kernel_function/kernels/{M4,M5,M6}_spline.jl:9-33,
   {C2,C4,C6}_Wendland.jl:9-33. */
double orc_kernel_f(int32_t k, double q)
{
    if (q < 0.0) return NAN;
    switch (k) {
    case 0:
        if (0.0 <= q && q < 1.0) return 0.25 * P(2.0 - q, 3) - P(1.0 - q, 3);
        if (1.0 <= q && q < 2.0) return 0.25 * P(2.0 - q, 3);
        return 0.0;
    case 1:
        if (0.0 <= q && q < 0.5) return P(2.5 - q, 4) - 5.0 * P(1.5 - q, 4) + 10.0 * P(0.5 - q, 4);
        if (0.5 <= q && q < 1.5) return P(2.5 - q, 4) - 5.0 * P(1.5 - q, 4);
        if (1.5 <= q && q < 2.5) return P(2.5 - q, 4);
        return 0.0;
    case 2:
        if (0.0 <= q && q < 1.0) return P(3.0 - q, 5) - 6.0 * P(2.0 - q, 5) + 15.0 * P(1.0 - q, 5);
        if (1.0 <= q && q < 2.0) return P(3.0 - q, 5) - 6.0 * P(2.0 - q, 5);
        if (2.0 <= q && q < 3.0) return P(3.0 - q, 5);
        return 0.0;
    case 3:
        if (q < 2.0) return P(1.0 - 0.5 * q, 4) * (2.0 * q + 1.0);
        return 0.0;
    case 4:
        if (q < 2.0) return P(1.0 - 0.5 * q, 6) * ((35.0 / 12.0) * P(q, 2) + 3.0 * q + 1.0);
        return 0.0;
    case 5:
        if (q < 2.0) return P(1.0 - 0.5 * q, 8) * (4.0 * P(q, 3) + 6.25 * P(q, 2) + 4.0 * q + 1.0);
        return 0.0;
    }
    return NAN;
}

double orc_kernel_df(int32_t k, double q)
{
    if (q < 0.0) return NAN;
    switch (k) {
    case 0:
        if (0.0 <= q && q < 1.0) return -0.75 * P(2.0 - q, 2) + 3.0 * P(1.0 - q, 2);
        if (1.0 <= q && q < 2.0) return -0.75 * P(2.0 - q, 2);
        return 0.0;
    case 1:
        if (0.0 <= q && q < 0.5) return -4.0 * P(2.5 - q, 3) + 20.0 * P(1.5 - q, 3) - 40.0 * P(0.5 - q, 3);
        if (0.5 <= q && q < 1.5) return -4.0 * P(2.5 - q, 3) + 20.0 * P(1.5 - q, 3);
        if (1.5 <= q && q < 2.5) return -4.0 * P(2.5 - q, 3);
        return 0.0;
    case 2:
        if (0.0 <= q && q < 1.0) return -5.0 * P(3.0 - q, 4) + 30.0 * P(2.0 - q, 4) - 75.0 * P(1.0 - q, 4);
        if (1.0 <= q && q < 2.0) return -5.0 * P(3.0 - q, 4) + 30.0 * P(2.0 - q, 4);
        if (2.0 <= q && q < 3.0) return -5.0 * P(3.0 - q, 4);
        return 0.0;
    case 3:
        if (q < 2.0) return P(1.0 - 0.5 * q, 4) * 2.0 - P(1.0 - 0.5 * q, 3) * (4.0 * q + 2.0);
        return 0.0;
    case 4:
        if (q < 2.0)
            return P(1.0 - 0.5 * q, 6) * ((35.0 / 6.0) * q + 3.0) -
                   P(1.0 - 0.5 * q, 5) * ((35.0 / 4.0) * P(q, 2) + 9.0 * q + 3.0);
        return 0.0;
    case 5:
        if (q < 2.0)
            return P(1.0 - 0.5 * q, 8) * (12.0 * P(q, 2) + 12.5 * q + 4.0) -
                   P(1.0 - 0.5 * q, 7) * (16.0 * P(q, 3) + 25.0 * P(q, 2) + 16.0 * q + 4.0);
        return 0.0;
    }
    return NAN;
}

/* KernelFunctionnorm(K, Val(3), Float64) and KernelFunctionValid (kernels/ directory). */
double orc_kernel_norm3(int32_t k)
{
    switch (k) {
    case 0: return 1.0 / M_PI;
    case 1: return 0.05 / M_PI;
    case 2: return 1.0 / (120.0 * M_PI);
    case 3: return 21.0 / (16.0 * M_PI);
    case 4: return 495.0 / (256.0 * M_PI);
    case 5: return 1365.0 / (512.0 * M_PI);
    }
    return NAN;
}

double orc_kernel_valid(int32_t k)
{
    switch (k) {
    case 1: return 2.5;
    case 2: return 3.0;
    default: return 2.0;
    }
}

/* Smoothed_kernel_function(K, r, h, Val(3)): kernel.jl:152-157 */
double orc_W(int32_t k, double r, double h)
{
    double invh = 1.0 / h;
    double inv_hD = invh * invh * invh;
    double q = r * invh;
    return inv_hD * (orc_kernel_norm3(k) * orc_kernel_f(k, q));
}

/* Smoothed_gradient_kernel_function(K, dx, dy, dz, h): kernel.jl:284-296,371-376 */
void orc_gradW(int32_t k, double dx, double dy, double dz, double h, double *g3)
{
    double invh = 1.0 / h;
    double inv_hDp1 = invh * invh * invh * invh;
    double r2 = dx * dx + dy * dy + dz * dz;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    if (r2 != 0.0) {
        double r = sqrt(r2);
        double invr = 1.0 / r;
        double q = r / h;
        double coeff = orc_kernel_df(k, q) * orc_kernel_norm3(k) * invr;
        gx = dx * coeff;
        gy = dy * coeff;
        gz = dz * coeff;
    }
    g3[0] = inv_hDp1 * gx;
    g3[1] = inv_hDp1 * gy;
    g3[2] = inv_hDp1 * gz;
}

/* _lin_lut + line_integrated_kernel_function: line_integrated_kernel.jl:13-19,90-94,132-137 */
static double lin_lut(int32_t k, double q)
{
    const double *I = PB_LINE_INORM[k];
    double dq = 1.0 * PB_LINE_QMAX[k] / (double)(PB_LINE_NTAB - 1) - 0.0;
    double idxf = q / dq + 1.0;
    int32_t i = (int32_t)idxf;
    if (i < 1) i = 1;
    if (i > PB_LINE_NTAB - 1) i = PB_LINE_NTAB - 1;
    double t = idxf - (double)i;
    return I[i - 1] * (1.0 - t) + I[i] * t;
}

double orc_line_W(int32_t k, double r, double h)
{
    double invh = 1.0 / h;
    double q = r * invh;
    double I = (q >= orc_kernel_valid(k)) ? 0.0 : lin_lut(k, q);
    return invh * I;
}

/* ------------------------------------------------------------------------------------ */
/* Morton encoding: MortonCode.jl:209-217,275-305,426-498                               */
static inline uint64_t expand_bits3(uint64_t x)
{
    x = (x | (x << 32)) & 0x1f00000000ffffULL;
    x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
    x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
    x = (x | (x << 2)) & 0x1249249249249249ULL;
    return x;
}

/* The per-particle loops of the build run on all host threads, as the reference's
   Threads.@threads loops do (MortonCode.jl:301,484; BinaryRadixTree.jl:106-118); the
   min/max reductions are exact, so the results do not depend on the thread count. */
static void quantize_axis(int64_t n, const double *v, uint64_t *iv)
{
    double vmin = v[0], vmax = v[0];
#pragma omp parallel for reduction(min : vmin) reduction(max : vmax) schedule(static)
    for (int64_t i = 1; i < n; ++i) {
        if (v[i] < vmin) vmin = v[i];
        if (v[i] > vmax) vmax = v[i];
    }
    double dv = vmax - vmin;
    const double scale = 2097151.0; /* exp2(21) - 1 */
    if (dv == 0.0) {
        for (int64_t i = 0; i < n; ++i) iv[i] = (uint64_t)floor(scale * 0.5);
        return;
    }
    double inv = 1.0 / dv;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double f = (v[i] - vmin) * inv;
        iv[i] = (uint64_t)floor(scale * f);
    }
}

/* Stable LSD radix sort of (code, index): equivalent to Julia's sortperm, whose Perm
   ordering breaks ties by index (MortonCode.jl:182). */
static void stable_sort_codes(int64_t n, uint64_t *codes, int64_t *idx)
{
    uint64_t *kt = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n);
    int64_t *it = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    for (int pass = 0; pass < 8; ++pass) {
        int shift = pass * 8;
        int64_t cnt[257];
        memset(cnt, 0, sizeof(cnt));
        for (int64_t i = 0; i < n; ++i) cnt[((codes[i] >> shift) & 0xff) + 1]++;
        int trivial = 0;
        for (int b = 1; b <= 256; ++b)
            if (cnt[b] == n) trivial = 1;
        if (trivial) continue;
        for (int b = 0; b < 256; ++b) cnt[b + 1] += cnt[b];
        for (int64_t i = 0; i < n; ++i) {
            int64_t d = (int64_t)((codes[i] >> shift) & 0xff);
            int64_t o = cnt[d]++;
            kt[o] = codes[i];
            it[o] = idx[i];
        }
        memcpy(codes, kt, sizeof(uint64_t) * (size_t)n);
        memcpy(idx, it, sizeof(int64_t) * (size_t)n);
    }
    free(kt);
    free(it);
}

/* ------------------------------------------------------------------------------------ */
/* Binary radix tree: BinaryRadixTree.jl:81-281 (1-based indices throughout)             */
static inline int64_t lcp(const uint64_t *c1, int64_t i, int64_t j) /* c1 is 1-based */
{
    uint64_t a = c1[i], b = c1[j];
    uint64_t x = (a == b) ? ((uint64_t)i ^ (uint64_t)j) : (a ^ b);
    return x == 0 ? 64 : (int64_t)__builtin_clzll(x);
}

static void find_range(const uint64_t *c1, int64_t n, int64_t i, int64_t *lo, int64_t *hi)
{
    int64_t dL = (i > 1) ? lcp(c1, i, i - 1) : -1;
    int64_t dR = (i < n) ? lcp(c1, i, i + 1) : -1;
    int64_t d = (dR - dL > 0) ? 1 : ((dR - dL < 0) ? -1 : 1);
    int64_t dmin = (1 <= i - d && i - d <= n) ? lcp(c1, i, i - d) : -1;
    int64_t lmax = 2;
    for (;;) {
        int64_t j = i + lmax * d;
        if (j < 1 || j > n) break;
        if (lcp(c1, i, j) <= dmin) break;
        lmax *= 2;
    }
    int64_t l = 0;
    for (int64_t t = lmax >> 1; t > 0; t >>= 1) {
        int64_t j = i + (l + t) * d;
        if (j >= 1 && j <= n && lcp(c1, i, j) > dmin) l += t;
    }
    int64_t j = i + l * d;
    *lo = i < j ? i : j;
    *hi = i < j ? j : i;
}

static int64_t split_position(const uint64_t *c1, int64_t first, int64_t last)
{
    if (c1[first] == c1[last]) {
        int64_t s = (first + last) >> 1;
        if (s < first) s = first;
        if (s > last - 1) s = last - 1;
        return s;
    }
    int64_t pfl = lcp(c1, first, last);
    int64_t split = first, step = last - first;
    while (step > 1) {
        step = (step + 1) >> 1;
        int64_t ns = split + step;
        if (ns < last && lcp(c1, first, ns) > pfl) split = ns;
    }
    return split;
}

int orc_build(int64_t n, const double *x, const double *y, const double *z, const double *h,
              uint64_t *codes, int64_t *order,
              double *sx, double *sy, double *sz, double *sh,
              int32_t *left, int32_t *right, int32_t *escape, int32_t *parent,
              double *bmin, double *bmax, double *hmax, int32_t *root_out)
{
    if (n < 1 || n > 1073741824LL) return -1;
    uint64_t *ix = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n);
    uint64_t *iy = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n);
    uint64_t *iz = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n);
    quantize_axis(n, x, ix);
    quantize_axis(n, y, iy);
    quantize_axis(n, z, iz);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        codes[i] = (expand_bits3(ix[i]) << 2) | (expand_bits3(iy[i]) << 1) | expand_bits3(iz[i]);
        order[i] = i;
    }
    free(ix); free(iy); free(iz);
    stable_sort_codes(n, codes, order);
    /* sequential duplicate bump (MortonCode.jl:189-193) */
    for (int64_t i = 1; i < n; ++i)
        if (codes[i] <= codes[i - 1]) codes[i] = codes[i - 1] + 1;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        int64_t o = order[i];
        sx[i] = x[o]; sy[i] = y[o]; sz[i] = z[o]; sh[i] = h[o];
    }

    int64_t ntot = 2 * n - 1;
    memset(left, 0, sizeof(int32_t) * (size_t)ntot);
    memset(right, 0, sizeof(int32_t) * (size_t)ntot);
    memset(escape, 0, sizeof(int32_t) * (size_t)ntot);
    memset(parent, 0, sizeof(int32_t) * (size_t)ntot);
    int32_t root = (n >= 2) ? 1 : 0;
    *root_out = root;
    if (n < 2) return 0;

    const uint64_t *c1 = codes - 1; /* 1-based view */
    int32_t *L = left - 1, *R = right - 1, *E = escape - 1, *Pa = parent - 1; /* id-indexed */
    int64_t nin = n - 1, off = n - 1;
    int32_t *range_hi = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nin + 1));
    int32_t *adj = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
#pragma omp parallel for schedule(static)
    for (int64_t i = 1; i <= nin; ++i) {
        int64_t lo, hi;
        find_range(c1, n, i, &lo, &hi);
        range_hi[i] = (int32_t)hi;
        int64_t s = split_position(c1, lo, hi);
        int64_t li = (s == lo) ? lo + off : s;
        L[i] = (int32_t)li; Pa[li] = (int32_t)i;
        int64_t ri = (s + 1 == hi) ? hi + off : s + 1;
        R[i] = (int32_t)ri; Pa[ri] = (int32_t)i;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 1; i <= n - 1; ++i) adj[i] = (int32_t)lcp(c1, i, i + 1);
    adj[n] = 2147483647;
#pragma omp parallel for schedule(static)
    for (int64_t i = 1; i <= nin; ++i) {
        int64_t hi = range_hi[i];
        if (hi == n) E[i] = 0;
        else if (hi == n - 1) E[i] = (int32_t)(off + n);
        else {
            int64_t nx = hi + 1;
            E[i] = (adj[nx] < adj[nx - 1]) ? (int32_t)(off + nx) : (int32_t)nx;
        }
    }
    /* leaf escapes read only internal escapes, which are final here */
#pragma omp parallel for schedule(static)
    for (int64_t id = n; id <= ntot; ++id) {
        int32_t p = Pa[id];
        if (p == 0) { E[id] = 0; continue; }
        E[id] = (L[p] == (int32_t)id) ? R[p] : E[p];
    }
    free(range_hi);
    free(adj);

    /* Karras refit with second-arrival counters: LinearBVH.jl:55-156 */
    uint32_t *visited = (uint32_t *)calloc((size_t)(nin + 1), sizeof(uint32_t));
    const double *leaf[3] = {sx, sy, sz};
    for (int64_t startid = n; startid <= ntot; ++startid) {
        int64_t p = Pa[startid];
        while (p != 0) {
            if (++visited[p] != 2) break;
            int64_t l = L[p], r = R[p];
            int lleaf = l >= n, rleaf = r >= n;
            double hl = lleaf ? sh[l - n] : hmax[l - 1];
            double hr = rleaf ? sh[r - n] : hmax[r - 1];
            hmax[p - 1] = (hl > hr) ? hl : hr;
            for (int d = 0; d < 3; ++d) {
                double lmn = lleaf ? leaf[d][l - n] : bmin[d * nin + l - 1];
                double rmn = rleaf ? leaf[d][r - n] : bmin[d * nin + r - 1];
                double lmx = lleaf ? leaf[d][l - n] : bmax[d * nin + l - 1];
                double rmx = rleaf ? leaf[d][r - n] : bmax[d * nin + r - 1];
                bmin[d * nin + p - 1] = (lmn < rmn) ? lmn : rmn;
                bmax[d * nin + p - 1] = (lmx > rmx) ? lmx : rmx;
            }
            p = Pa[p];
        }
    }
    int ok = 1;
    for (int64_t i = 1; i <= nin; ++i)
        if (visited[i] < 2) ok = 0;
    free(visited);
    return ok ? 0 : -2;
}

/* ------------------------------------------------------------------------------------ */
/* Traversal helpers: LinearBVHTraversalMacros.jl:800-953                                */
static inline double d2_point(const orc_tree *t, double px, double py, double pz, int64_t b)
{
    double s = 0.0, dd;
    dd = px - t->x[b]; s += dd * dd;
    dd = py - t->y[b]; s += dd * dd;
    dd = pz - t->z[b]; s += dd * dd;
    return s;
}

static inline double d2_box(const orc_tree *t, double px, double py, double pz, int64_t i0)
{
    int64_t nin = t->n - 1;
    double p[3] = {px, py, pz};
    double s = 0.0;
    for (int d = 0; d < 3; ++d) {
        double a = t->bmin[d * nin + i0], b = t->bmax[d * nin + i0];
        double tt = p[d] < a ? (a - p[d]) : (p[d] > b ? (p[d] - b) : 0.0);
        s += tt * tt;
    }
    return s;
}

static inline double d2_line_point(const double p[3], const double o[3], const double m[3])
{
    double D2 = 0.0, Dm = 0.0;
    for (int d = 0; d < 3; ++d) {
        double D = p[d] - o[d];
        D2 += D * D;
        Dm += D * m[d];
    }
    return D2 - Dm * Dm;
}

static inline int line_hits_box(const double o[3], const double m[3], const double a[3], const double b[3])
{
    double tmin = -INFINITY, tmax = INFINITY;
    for (int d = 0; d < 3; ++d) {
        if (m[d] == 0.0) {
            if (o[d] < a[d] || o[d] > b[d]) return 0;
        } else {
            double t0 = (a[d] - o[d]) / m[d];
            double t1 = (b[d] - o[d]) / m[d];
            if (t0 > t1) { double tt = t0; t0 = t1; t1 = tt; }
            tmin = (t0 > tmin) ? t0 : tmin;
            tmax = (t1 < tmax) ? t1 : tmax;
            if (tmin > tmax) return 0;
        }
    }
    return 1;
}

static inline double d2_line_box(const orc_tree *t, const double o[3], const double m[3], int64_t i0)
{
    int64_t nin = t->n - 1;
    double a[3], b[3];
    for (int d = 0; d < 3; ++d) { a[d] = t->bmin[d * nin + i0]; b[d] = t->bmax[d * nin + i0]; }
    if (line_hits_box(o, m, a, b)) return 0.0;
    double c[3], r2 = 0.0;
    for (int d = 0; d < 3; ++d) c[d] = (a[d] + b[d]) * 0.5;
    for (int d = 0; d < 3; ++d) { double hh = (b[d] - a[d]) * 0.5; r2 += hh * hh; }
    double dc2 = d2_line_point(c, o, m);
    if (dc2 <= r2) return 0.0;
    double dl = sqrt(dc2) - sqrt(r2);
    return dl * dl;
}

/* LBVH_find_nearest_h: LinearBVHQueries.jl:118-140 over @LBVH_gather_point_traversal */
static double nearest_h_impl(const orc_tree *t, double px, double py, double pz, int64_t *best_out,
                             int64_t *nvis, int64_t *nleaf)
{
    double best = INFINITY;
    int64_t bi = -1, n = t->n, vis = 0, lt = 0;
    if (t->root == 0) {
        for (int64_t b = 0; b < n; ++b) {
            double d2 = d2_point(t, px, py, pz, b);
            ++lt;
            if (d2 <= best && d2 < best) { best = d2; bi = b; }
        }
    } else {
        int64_t node = t->root;
        while (node != 0) {
            if (node >= n) {
                int64_t b = node - n;
                double d2 = d2_point(t, px, py, pz, b);
                ++lt;
                if (d2 <= best && d2 < best) { best = d2; bi = b; }
                node = t->escape[node - 1];
                continue;
            }
            ++vis;
            if (d2_box(t, px, py, pz, node - 1) > best) { node = t->escape[node - 1]; continue; }
            node = t->left[node - 1];
        }
    }
    if (best_out) *best_out = bi;
    if (nvis) *nvis += vis;
    if (nleaf) *nleaf += lt;
    return bi < 0 ? NAN : t->h[bi];
}

double orc_find_nearest_h(const orc_tree *t, double px, double py, double pz, int64_t *best)
{
    return nearest_h_impl(t, px, py, pz, best, NULL, NULL);
}

/* LBVH_query! (LinearBVHQueries.jl:183-205) and LBVH_probe_neighbors (LinearBVHQueries.jl:22-42):
   the gather traversal with r2 = radius * radius; the closest accepted leaf is the first
   strictly closer one in DFS order. */
static int64_t query_impl(const orc_tree *t, double px, double py, double pz, double radius,
                          int64_t *pool, int64_t cap, int64_t *nearest, double *nearest_d2)
{
    double r2 = radius * radius, cd = INFINITY;
    int64_t count = 0, ci = -1, n = t->n;
    int64_t node = t->root;
    if (node == 0) {
        for (int64_t b = 0; b < n; ++b) {
            double d2 = d2_point(t, px, py, pz, b);
            if (d2 <= r2) {
                if (count < cap) pool[count] = b;
                ++count;
                if (d2 < cd) { cd = d2; ci = b; }
            }
        }
    } else {
        while (node != 0) {
            if (node >= n) {
                int64_t b = node - n;
                double d2 = d2_point(t, px, py, pz, b);
                if (d2 <= r2) {
                    if (count < cap) pool[count] = b;
                    ++count;
                    if (d2 < cd) { cd = d2; ci = b; }
                }
                node = t->escape[node - 1];
                continue;
            }
            if (d2_box(t, px, py, pz, node - 1) > r2) { node = t->escape[node - 1]; continue; }
            node = t->left[node - 1];
        }
    }
    if (nearest) *nearest = ci;
    if (nearest_d2) *nearest_d2 = cd;
    return count;
}

int64_t orc_query(const orc_tree *t, double px, double py, double pz, double radius,
                  int64_t *pool, int64_t cap, int64_t *nearest)
{
    return query_impl(t, px, py, pz, radius, pool, cap, nearest, NULL);
}

int64_t orc_probe_neighbors(const orc_tree *t, double px, double py, double pz, double radius,
                            int64_t *closest, double *closest_d2)
{
    return query_impl(t, px, py, pz, radius, NULL, 0, closest, closest_d2);
}

/* ------------------------------------------------------------------------------------ */
/* Fused per-point interpolation: general_interpolation.jl:1-669 with the accumulators of */
/* single_point_interpolation/accumulations/ files.                                        */
#define MAXQ 64

typedef struct {
    double S1;
    double sc[MAXQ];
    double gf[MAXQ][3], gb[MAXQ][3], gs[MAXQ];
    double df[MAXQ], db[MAXQ][3], ds[MAXQ][3];
    double cf[MAXQ][3], cb[MAXQ][3], cs[MAXQ][3];
} acc_t;

static void acc_zero(const orc_catalog *c, acc_t *A)
{
    A->S1 = 0.0;
    memset(A->sc, 0, sizeof(double) * (size_t)c->n_scalar);
    memset(A->gf, 0, sizeof(double) * 3 * (size_t)c->n_grad);
    memset(A->gb, 0, sizeof(double) * 3 * (size_t)c->n_grad);
    memset(A->gs, 0, sizeof(double) * (size_t)c->n_grad);
    memset(A->df, 0, sizeof(double) * (size_t)c->n_div);
    memset(A->db, 0, sizeof(double) * 3 * (size_t)c->n_div);
    memset(A->ds, 0, sizeof(double) * 3 * (size_t)c->n_div);
    memset(A->cf, 0, sizeof(double) * 3 * (size_t)c->n_curl);
    memset(A->cb, 0, sizeof(double) * 3 * (size_t)c->n_curl);
    memset(A->cs, 0, sizeof(double) * 3 * (size_t)c->n_curl);
}

static inline double Wsel(int32_t k, int32_t strategy, double r, double ha, double hb)
{
    if (strategy == 2) return 0.5 * (orc_W(k, r, ha) + orc_W(k, r, hb));
    return orc_W(k, r, strategy == 0 ? ha : hb);
}

static inline void gWsel(int32_t k, int32_t strategy, double dx, double dy, double dz, double ha, double hb,
                         double g[3])
{
    if (strategy == 2) {
        double ga[3], gb[3];
        orc_gradW(k, dx, dy, dz, ha, ga);
        orc_gradW(k, dx, dy, dz, hb, gb);
        g[0] = 0.5 * (ga[0] + gb[0]);
        g[1] = 0.5 * (ga[1] + gb[1]);
        g[2] = 0.5 * (ga[2] + gb[2]);
    } else {
        orc_gradW(k, dx, dy, dz, strategy == 0 ? ha : hb, g);
    }
}

static void accumulate_pair(const orc_tree *t, const orc_catalog *c, int32_t strategy, acc_t *A,
                            double xa, double ya, double za, double ha, int64_t b, double d2, double hb)
{
    int32_t k = t->kernel;
    double dx = xa - t->x[b], dy = ya - t->y[b], dz = za - t->z[b];
    double dr = sqrt(d2);
    double mb = t->m[b], rb = t->rho[b];
    double W = Wsel(k, strategy, dr, ha, hb);
    double w = mb * W / rb; /* (mb*W)/rho_b */
    A->S1 += w;
    for (int j = 0; j < c->n_scalar; ++j) A->sc[j] += t->quant[c->scalar_cols[j]][b] * w;
    if (c->n_grad + c->n_div + c->n_curl == 0) return;
    double g[3];
    gWsel(k, strategy, dx, dy, dz, ha, hb, g);
    double invrb = 1.0 / rb;
    double ml = mb * invrb;
    double gx = ml * g[0], gy = ml * g[1], gz = ml * g[2];
    for (int j = 0; j < c->n_grad; ++j) {
        int32_t col = c->grad_cols[j];
        if (col < 0) {
            double mx = mb * g[0], my = mb * g[1], mz = mb * g[2];
            A->gf[j][0] += mx; A->gf[j][1] += my; A->gf[j][2] += mz;
            A->gb[j][0] += mx * invrb; A->gb[j][1] += my * invrb; A->gb[j][2] += mz * invrb;
            A->gs[j] += mb * W;
        } else {
            double Ab = t->quant[col][b];
            A->gf[j][0] += gx * Ab; A->gf[j][1] += gy * Ab; A->gf[j][2] += gz * Ab;
            A->gb[j][0] += gx; A->gb[j][1] += gy; A->gb[j][2] += gz;
            A->gs[j] += Ab * w;
        }
    }
    for (int j = 0; j < c->n_div; ++j) {
        double Ax = t->quant[c->div_cols[3 * j]][b];
        double Ay = t->quant[c->div_cols[3 * j + 1]][b];
        double Az = t->quant[c->div_cols[3 * j + 2]][b];
        A->df[j] += gx * Ax + gy * Ay + gz * Az;
        A->db[j][0] += gx; A->db[j][1] += gy; A->db[j][2] += gz;
        A->ds[j][0] += Ax * w; A->ds[j][1] += Ay * w; A->ds[j][2] += Az * w;
    }
    for (int j = 0; j < c->n_curl; ++j) {
        double Ax = t->quant[c->curl_cols[3 * j]][b];
        double Ay = t->quant[c->curl_cols[3 * j + 1]][b];
        double Az = t->quant[c->curl_cols[3 * j + 2]][b];
        A->cf[j][0] += Ay * gz - Az * gy;
        A->cf[j][1] += Az * gx - Ax * gz;
        A->cf[j][2] += Ax * gy - Ay * gx;
        A->cb[j][0] += gx; A->cb[j][1] += gy; A->cb[j][2] += gz;
        A->cs[j][0] += Ax * w; A->cs[j][1] += Ay * w; A->cs[j][2] += Az * w;
    }
}

static int64_t catalog_L(const orc_catalog *c)
{
    return c->n_scalar + 3 * c->n_grad + c->n_div + 3 * c->n_curl;
}

static void finalize(const orc_catalog *c, const acc_t *A, double *o /* L values */)
{
    int64_t L = catalog_L(c), q = 0;
    if (A->S1 == 0.0) {
        for (int64_t l = 0; l < L; ++l) o[l] = NAN;
        return;
    }
    double inv = 1.0 / A->S1;
    for (int j = 0; j < c->n_scalar; ++j) o[q++] = c->scalar_shepard[j] ? A->sc[j] * inv : A->sc[j];
    for (int j = 0; j < c->n_grad; ++j) {
        double a = A->gs[j] * inv;
        for (int d = 0; d < 3; ++d) o[q++] = A->gf[j][d] - A->gb[j][d] * a;
    }
    for (int j = 0; j < c->n_div; ++j) {
        double ax = A->ds[j][0] * inv, ay = A->ds[j][1] * inv, az = A->ds[j][2] * inv;
        double b = ax * A->db[j][0] + ay * A->db[j][1] + az * A->db[j][2];
        o[q++] = A->df[j] - b;
    }
    for (int j = 0; j < c->n_curl; ++j) {
        double ax = A->cs[j][0] * inv, ay = A->cs[j][1] * inv, az = A->cs[j][2] * inv;
        double bx = ay * A->cb[j][2] - az * A->cb[j][1];
        double by = az * A->cb[j][0] - ax * A->cb[j][2];
        double bz = ax * A->cb[j][1] - ay * A->cb[j][0];
        o[q++] = -(A->cf[j][0] - bx);
        o[q++] = -(A->cf[j][1] - by);
        o[q++] = -(A->cf[j][2] - bz);
    }
}

static void interp_one_point(const orc_tree *t, const orc_catalog *c, int32_t strategy,
                             double xa, double ya, double za, double *o, int64_t *st)
{
    int64_t n = t->n;
    int32_t k = t->kernel;
    double K = orc_kernel_valid(k);
    double ha = 0.0;
    int64_t nv = 0, nl = 0, mv = 0, ml = 0, acc = 0;
    if (strategy != 1) ha = nearest_h_impl(t, xa, ya, za, NULL, &nv, &nl);
    double radius = K * ha;
    double radius2 = radius * radius;
    acc_t A;
    acc_zero(c, &A);
    int64_t node = t->root;
    if (node == 0) {
        for (int64_t b = 0; b < n; ++b) {
            double hb = t->h[b], r2;
            if (strategy == 0) r2 = radius2;
            else {
                double r = K * hb;
                double rr = r * r;
                r2 = (strategy == 2) ? (radius2 > rr ? radius2 : rr) : rr;
            }
            double d2 = d2_point(t, xa, ya, za, b);
            ++ml;
            if (d2 <= r2) { ++acc; accumulate_pair(t, c, strategy, &A, xa, ya, za, ha, b, d2, hb); }
        }
    } else {
        while (node != 0) {
            if (node >= n) {
                int64_t b = node - n;
                double hb = t->h[b], r2;
                if (strategy == 0) r2 = radius2;
                else {
                    double r = K * hb;
                    double rr = r * r;
                    r2 = (strategy == 2) ? (radius2 > rr ? radius2 : rr) : rr;
                }
                double d2 = d2_point(t, xa, ya, za, b);
                ++ml;
                if (d2 <= r2) { ++acc; accumulate_pair(t, c, strategy, &A, xa, ya, za, ha, b, d2, hb); }
                node = t->escape[node - 1];
                continue;
            }
            ++mv;
            double r2;
            if (strategy == 0) r2 = radius2;
            else {
                double r = K * t->hmax[node - 1];
                double rr = r * r;
                r2 = (strategy == 2) ? (radius2 > rr ? radius2 : rr) : rr;
            }
            if (d2_box(t, xa, ya, za, node - 1) > r2) { node = t->escape[node - 1]; continue; }
            node = t->left[node - 1];
        }
    }
    finalize(c, &A, o);
    if (st) { st[0] = nv; st[1] = nl; st[2] = mv; st[3] = ml; st[4] = acc; }
}

void orc_interp_points(const orc_tree *t, const orc_catalog *cat, int64_t npts,
                       const double *qx, const double *qy, const double *qz,
                       int32_t strategy, double *out, int32_t nthreads, int64_t *stats)
{
    int64_t L = catalog_L(cat);
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    /* one point per dispatch: the per-point work is heavy-tailed and neighbouring points are
       alike, so larger chunks leave one thread finishing a run of heavy points alone */
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
    for (int64_t i = 0; i < npts; ++i) {
        double o[4 * MAXQ + 4 * MAXQ];
        interp_one_point(t, cat, strategy, qx[i], qy[i], qz[i], o, stats ? stats + 5 * i : NULL);
        for (int64_t l = 0; l < L; ++l) out[l * npts + i] = o[l];
    }
    (void)nthreads;
}

/* Line-integrated scatter interpolation: line_integrated_scalar_interpolation.jl:123-166 over
   @LBVH_scatter_line_traversal (LinearBVHTraversalMacros.jl:539-644). */
static void interp_one_line(const orc_tree *t, const orc_catalog *c, const double o[3], const double m[3],
                            double *out, int64_t *st)
{
    int64_t n = t->n;
    int32_t k = t->kernel;
    double K = orc_kernel_valid(k);
    double S1 = 0.0, acc[MAXQ];
    int64_t nv = 0, nl = 0, na = 0;
    for (int j = 0; j < c->n_scalar; ++j) acc[j] = 0.0;
    int64_t node = t->root;
    int64_t b = -1;
    int brute = (node == 0);
    int64_t bi = 0;
    while (brute ? (bi < n) : (node != 0)) {
        int is_leaf;
        if (brute) { b = bi++; is_leaf = 1; }
        else { is_leaf = node >= n; b = node - n; }
        if (is_leaf) {
            double hb = t->h[b];
            double r = K * hb, r2 = r * r;
            double p[3] = {t->x[b], t->y[b], t->z[b]};
            double d2 = d2_line_point(p, o, m);
            ++nl;
            if (d2 <= r2) {
                /* Julia's sqrt raises DomainError for d2 < 0 (rounding); clamp instead. */
                double dr = sqrt(d2 > 0.0 ? d2 : 0.0);
                double mb = t->m[b], rb = t->rho[b];
                double W = orc_line_W(k, dr, hb);
                double w = mb * W / rb;
                S1 += w;
                for (int j = 0; j < c->n_scalar; ++j) acc[j] += t->quant[c->scalar_cols[j]][b] * w;
                ++na;
            }
            if (!brute) node = t->escape[node - 1];
            continue;
        }
        ++nv;
        double r = K * t->hmax[node - 1], r2 = r * r;
        if (d2_line_box(t, o, m, node - 1) > r2) { node = t->escape[node - 1]; continue; }
        node = t->left[node - 1];
    }
    if (S1 == 0.0) {
        for (int j = 0; j < c->n_scalar; ++j) out[j] = NAN;
    } else {
        double inv = 1.0 / S1;
        for (int j = 0; j < c->n_scalar; ++j) out[j] = c->scalar_shepard[j] ? acc[j] * inv : acc[j];
    }
    if (st) { st[0] = nv; st[1] = nl; st[2] = na; }
}

void orc_interp_lines(const orc_tree *t, const orc_catalog *cat, int64_t nlines,
                      const double *ox, const double *oy, const double *oz,
                      const double *dx, const double *dy, const double *dz,
                      double *out, int32_t nthreads, int64_t *stats)
{
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
    for (int64_t i = 0; i < nlines; ++i) {
        double o[3] = {ox[i], oy[i], oz[i]}, m[3] = {dx[i], dy[i], dz[i]}, v[MAXQ];
        interp_one_line(t, cat, o, m, v, stats ? stats + 3 * i : NULL);
        for (int j = 0; j < cat->n_scalar; ++j) out[j * nlines + i] = v[j];
    }
    (void)nthreads;
}

int orc_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
