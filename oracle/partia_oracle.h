/*
 * partia_oracle.h -- CPU oracle for the Partia LBVH build + SPH grid interpolation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C, FP64 restatement of the reference
 * algorithm (Partia.jl, weishansu011017/DistortedDustyDiscAnalysisToolkits) used as
 * the parity checker for the CUDA library and as the timed CPU baseline.  Nothing in
 * the product path links or calls it.
 *
 * Conventions follow the reference exactly:
 *   - kernels:    0 M4_spline, 1 M5_spline, 2 M6_spline, 3 C2_Wendland, 4 C4_Wendland, 5 C6_Wendland
 *   - strategies: 0 itpGather, 1 itpScatter, 2 itpSymmetric
 *   - tree ids:   unified 1-based ids (internal 1..n-1, leaf n..2n-1, 0 = none);
 *                 id k is stored at array index k-1 of left/right/escape/parent.
 *   - boxes:      bmin/bmax are [3][n-1] (axis-major), hmax is [n-1].
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int64_t n;
    int32_t root;
    const double *x, *y, *z, *h;      /* sorted leaf coordinates / smoothing lengths */
    const int32_t *left, *right, *escape;
    const double *bmin, *bmax, *hmax;
    const double *m, *rho;            /* sorted particle masses / densities */
    int32_t ncol;
    const double *const *quant;       /* ncol sorted quantity columns */
    int32_t kernel;
} orc_tree;

typedef struct {
    int32_t n_scalar;  const int32_t *scalar_cols; const int32_t *scalar_shepard;
    int32_t n_grad;    const int32_t *grad_cols;   /* -1 = density gradient */
    int32_t n_div;     const int32_t *div_cols;    /* 3 per entry */
    int32_t n_curl;    const int32_t *curl_cols;   /* 3 per entry */
} orc_catalog;

/* kernel functions (Partia.jl/src/julia/KernelInterpolation/kernel_function/ directory) */
double orc_kernel_f(int32_t k, double q);
double orc_kernel_df(int32_t k, double q);
double orc_kernel_norm3(int32_t k);
double orc_kernel_valid(int32_t k);
double orc_W(int32_t k, double r, double h);
void   orc_gradW(int32_t k, double dx, double dy, double dz, double h, double *g3);
double orc_line_W(int32_t k, double r, double h);
double orc_jl_pow(double x, int64_t n);

/* LBVH build (MortonEncoding + BinaryRadixTree + LinearBVH).  order[] is 0-based. */
int orc_build(int64_t n, const double *x, const double *y, const double *z, const double *h,
              uint64_t *codes, int64_t *order,
              double *sx, double *sy, double *sz, double *sh,
              int32_t *left, int32_t *right, int32_t *escape, int32_t *parent,
              double *bmin, double *bmax, double *hmax, int32_t *root);

/* LBVH_find_nearest_h; best is the 0-based sorted leaf index (-1 if none). */
double orc_find_nearest_h(const orc_tree *t, double px, double py, double pz, int64_t *best);

/* LBVH_query!: accepted 0-based leaf indices in DFS order; returns count (pool may be
   shorter than count: only the first cap entries are written). */
int64_t orc_query(const orc_tree *t, double px, double py, double pz, double radius,
                  int64_t *pool, int64_t cap, int64_t *nearest);

/* LBVH_probe_neighbors: number of leaves within radius, the closest one (0-based, -1 if none)
   and its squared distance (+Inf if none). */
int64_t orc_probe_neighbors(const orc_tree *t, double px, double py, double pz, double radius,
                            int64_t *closest, double *closest_d2);

/* PointSamples interpolation on a built tree.  out is [L][npts].  stats (optional) is
   [npts][5]: nearest internal visits, nearest leaf tests, main internal visits,
   main leaf tests, accepted neighbours. */
void orc_interp_points(const orc_tree *t, const orc_catalog *cat, int64_t npts,
                       const double *qx, const double *qy, const double *qz,
                       int32_t strategy, double *out, int32_t nthreads, int64_t *stats);

/* LineSamples interpolation (itpScatter only), out is [n_scalar][nlines].
   stats (optional) is [nlines][3]: internal visits, leaf tests, accepted. */
void orc_interp_lines(const orc_tree *t, const orc_catalog *cat, int64_t nlines,
                      const double *ox, const double *oy, const double *oz,
                      const double *dx, const double *dy, const double *dz,
                      double *out, int32_t nthreads, int64_t *stats);

int orc_max_threads(void);

#ifdef __cplusplus
}
#endif
