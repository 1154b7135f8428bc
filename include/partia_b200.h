/*
 * partia_b200.h -- C ABI of libpartia_b200.so, the B200 (sm_100a) implementation of
 * Partia.jl's LBVH build + SPH grid interpolation path.
 *
 * This is the boundary that Partia's CUDA package extension binds through `ccall`
 * (Partia.jl/ext/CUDAExt.jl, Partia.jl/src/julia/ExtDummy/CUDAExtDummy.jlh:12).  All
 * arguments are plain pointers and sizes.  Every pointer may refer to host memory or to
 * device memory of the handle's device; the library detects which
 * (cudaPointerGetAttributes) and copies host buffers in and out itself.  Calls are
 * synchronous, like the reference extension (`CUDA.synchronize()` in
 * Partia.jl/ext/CUDAExt/KernelInterpolation/grid_interpolation/PointSamples_interpolation.jl:23),
 * and a handle must be used by one host thread at a time.  No exceptions cross the ABI:
 * every entry point returns PB_OK or a negative error class, and pb_last_error() holds a
 * message.  There is no CPU fallback: without a usable CUDA device pb_create fails.
 *
 * Conventions (reference -> ABI):
 *   - indices are 0-based (the Julia shim subtracts 1);
 *   - tree node ids keep the reference's unified 1-based id space (internal 1..n-1,
 *     leaf n..2n-1, 0 = none; BinaryRadixTree.jl:36-51); id k is at array index k-1;
 *   - catalog gradient slot 0 (density gradient, general_interpolation.jl:76-81) is -1;
 *   - kernels: 0 M4_spline, 1 M5_spline, 2 M6_spline, 3 C2_Wendland, 4 C4_Wendland,
 *     5 C6_Wendland; strategies: 0 itpGather, 1 itpScatter, 2 itpSymmetric
 *     (InterpolationStrategy.jl:1-5);
 *   - precision: PB_FP64 reproduces the reference's Float64 arithmetic in the reference's
 *     operation order; PB_FP32C evaluates the per-pair kernel terms in FP32 (double-float
 *     pair offsets) and accumulates FP32 chunk sums in FP64, with the same neighbour sets.
 */
#ifndef PARTIA_B200_H
#define PARTIA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PB_OK 0
#define PB_ERR_INVALID (-1)   /* ArgumentError: bad value, bad enum, non-finite coordinate, n = 0 */
#define PB_ERR_CAPACITY (-2)  /* n > 2^30 (BinaryRadixTree.jl:89-90) */
#define PB_ERR_CUDA (-3)      /* CUDA runtime error (message in pb_last_error) */
#define PB_ERR_STATE (-4)     /* query before pb_linear_bvh */
#define PB_ERR_INTERNAL (-6)  /* device consistency check failed (refit counters, traversal bound) */
#define PB_ERR_KEY (-7)       /* KeyError: a catalog column that the input does not have
                                 (InterpolationCatalog.jl:161-176) */
#define PB_ERR_DIMENSION (-8) /* DimensionMismatch: array lengths that do not agree (a neighbour
                                 pool shorter than a query's count; InterpolationInput.jl:87-98) */

#define PB_FP64 0
#define PB_FP32C 1

/* flags for pb_linear_bvh / pb_*_samples_interpolation */
#define PB_PERMUTE_CALLER 1   /* permute the caller's particle arrays in place, as LinearBVH! does */
#define PB_BUILD_ASYNC 2      /* pb_linear_bvh: enqueue the build without waiting for it; its status is
                                 checked by the next synchronous call on the handle or pb_batch_check */
/* flags for pb_batch_points */
#define PB_BATCH_ASYNC 1      /* enqueue only; pb_batch_check waits and checks every disc's status */

typedef struct pb_handle pb_handle;

/* InterpolationInput{3,Float64} (Partia.jl/src/julia/KernelInterpolation/interpolation_setup/InterpolationInput.jl:43-51) */
typedef struct {
    int64_t npart;
    const double *x, *y, *z, *m, *h, *rho;
    int32_t ncolumn;
    const double *const *quant;   /* ncolumn column pointers, each npart long */
    int32_t kernel;
} pb_input;

/* InterpolationCatalogConcise (InterpolationCatalog.jl:26-32), 0-based columns */
typedef struct {
    int32_t n_scalar;
    const int32_t *scalar_cols;
    const int32_t *scalar_shepard;   /* 0 for :rho / :ρ (InterpolationCatalog.jl:222-225) */
    int32_t n_grad;
    const int32_t *grad_cols;        /* -1 = density gradient */
    int32_t n_div;
    const int32_t *div_cols;         /* 3 per divergence */
    int32_t n_curl;
    const int32_t *curl_cols;        /* 3 per curl */
} pb_catalog;

/* Create a handle on CUDA device `device` (CUDAComputeBackend, CUDAExtDummy.jlh:12). */
int32_t pb_create(pb_handle **out, int32_t device);
void pb_destroy(pb_handle *h);
/* Copy the last error message (NUL terminated) into buf; returns its full length. */
int32_t pb_last_error(const pb_handle *h, char *buf, int64_t size);
/* Launch on this stream (a cudaStream_t of the handle's device); NULL = the handle's own. */
int32_t pb_set_stream(pb_handle *h, void *cuda_stream);
/* Options: "timing" (record CUDA events around build/traversal), "sort_queries"
   (Morton-order queries before traversal; schedule only), "block_size", "walk_split" (target
   number of subtrees each FP32-compensated point walk is split into, 1..4096; schedule only),
   "schedule" (FP32-compensated points: 0 plain = input order, one walk per query, no
   ordering; 1 tuned = Morton order, split walks, heaviest first (default); 2 learned = tuned
   plus binning by predicted work; results are identical), "slice_queries" (queries per
   walk/sum slice, default 2^22). */
int32_t pb_set_option(pb_handle *h, const char *name, int64_t value);

/* LinearBVH!(input, Val(3)) (InterpolationInput.jl:203-223): MortonEncoding
   (MortonCode.jl:38-45), BinaryRadixTree (BinaryRadixTree.jl:81-132) and LinearBVH
   (LinearBVH.jl:55-87), built on the device; the particle columns are kept on the device
   in sorted order.  With PB_PERMUTE_CALLER the caller's x,y,z,m,h,rho,quant buffers are
   permuted in place like the reference. */
int32_t pb_linear_bvh(pb_handle *h, const pb_input *in, int32_t flags);

/* MortonEncoding.codes/.order of the last build (MortonCode.jl:8-13); order is 0-based. */
int32_t pb_export_encoding(pb_handle *h, uint64_t *codes, int64_t *order);
/* BinaryRadixTree left/right/escape/parent (2n-1 each), LinearBVH node_aabb min/max
   ([3][n-1] axis-major) and node_hmax (n-1) of the last build (LinearBVH.jl:20-26). */
int32_t pb_export_tree(pb_handle *h, int32_t *left, int32_t *right, int32_t *escape, int32_t *parent,
                       double *bmin, double *bmax, double *hmax, int32_t *root);

/* LBVH_find_nearest_h / LBVH_find_nearest (LinearBVHQueries.jl:79-140), batched:
   h_out[i] = smoothing length of the nearest leaf, idx_out[i] = its 0-based sorted leaf
   index (either output may be NULL). */
int32_t pb_find_nearest_h(pb_handle *h, int64_t npts, const double *qx, const double *qy, const double *qz,
                          double *h_out, int64_t *idx_out);
/* LBVH_query! (LinearBVHQueries.jl:183-211), batched in two steps: pb_query_count gives
   counts[i]; pb_query_neighbors writes each query's accepted 0-based sorted leaf indices in
   DFS order at pool[offsets[i] ...] and the nearest accepted leaf (-1 if none). */
int32_t pb_query_count(pb_handle *h, int64_t npts, const double *qx, const double *qy, const double *qz,
                       const double *radius, int64_t *counts);
int32_t pb_query_neighbors(pb_handle *h, int64_t npts, const double *qx, const double *qy, const double *qz,
                           const double *radius, const int64_t *offsets, int64_t *pool, int64_t *nearest);
/* LBVH_probe_neighbors (LinearBVHQueries.jl:22-42), batched: the gather traversal with
   r2 = radius^2 counts the accepted leaves (count[i]) and keeps the first strictly closer one
   in DFS order, i.e. the minimum squared distance and among equal distances the smallest
   sorted index: closest_idx[i] (0-based; -1 if none, the reference's 0) and closest_d2[i]
   (+Inf if none, the reference's typemax).  Any output may be NULL. */
int32_t pb_probe_neighbors(pb_handle *h, int64_t npts, const double *qx, const double *qy, const double *qz,
                           const double *radius, int64_t *count, int64_t *closest_idx, double *closest_d2);

/* Event counts of the reference traversal algorithm on the last build (leaf size 1, Karras
   tree, left-first DFS, FP64 boxes; LinearBVHTraversalMacros.jl:26-371 driven as in
   PointSamples_interpolation.jl:118-133).  stats is [npts][5]: nearest-pass internal visits,
   nearest-pass leaf tests, main-pass internal visits, main-pass leaf tests, accepted
   neighbours.  These define the algorithmic-bytes model of the traversal and are the exact
   per-query work labels of the learned schedule. */
int32_t pb_traversal_stats(pb_handle *h, int64_t npts, const double *qx, const double *qy, const double *qz,
                           int32_t strategy, int64_t *stats);

/* Per-point kernel loop of PointSamples_interpolation on the last build
   (Partia.jl/src/julia/KernelInterpolation/grid_interpolation/PointSamples_interpolation.jl:99-184):
   LBVH_find_nearest_h + _general_quantity_interpolate_kernel (general_interpolation.jl:1-669).
   out holds L = n_scalar + 3 n_grad + n_div + 3 n_curl pointers of npts doubles, in the
   catalog's ordered_names order. */
int32_t pb_interpolate_points(pb_handle *h, const pb_catalog *cat, int64_t npts, const double *qx,
                              const double *qy, const double *qz, int32_t strategy, int32_t precision,
                              double *const *out);

/* Per-line kernel loop of LineSamples_interpolation on the last build (LineSamples_interpolation.jl:47-99,
   line_integrated_scalar_interpolation.jl:123-166).  Only itpScatter is accepted (others:
   PB_ERR_INVALID, the reference's ArgumentError).  Directions must be unit vectors. */
int32_t pb_interpolate_lines(pb_handle *h, const pb_catalog *cat, int64_t nlines, const double *ox,
                             const double *oy, const double *oz, const double *dx, const double *dy,
                             const double *dz, int32_t strategy, int32_t precision, double *const *out);

/* Partia.PointSamples_interpolation(::CUDAComputeBackend, grid, input, catalog, strategy)
   (Partia.jl/ext/CUDAExt/KernelInterpolation/grid_interpolation/PointSamples_interpolation.jl:12-29):
   build + interpolate in one call. */
int32_t pb_point_samples_interpolation(pb_handle *h, const pb_input *in, const pb_catalog *cat, int64_t npts,
                                       const double *qx, const double *qy, const double *qz, int32_t strategy,
                                       int32_t precision, double *const *out, int32_t flags);

/* Partia.LineSamples_interpolation(::CUDAComputeBackend, lines, input, catalog, itpScatter)
   (Partia.jl/ext/CUDAExt/KernelInterpolation/grid_interpolation/LineSamples_interpolation.jl:11-34).
   Both precision modes sum the line integrals in FP64 (the reference's arithmetic). */
int32_t pb_line_samples_interpolation(pb_handle *h, const pb_input *in, const pb_catalog *cat, int64_t nlines,
                                      const double *ox, const double *oy, const double *oz, const double *dx,
                                      const double *dy, const double *dz, int32_t strategy, int32_t precision,
                                      double *const *out, int32_t flags);

/* Batched PointSamples interpolation over many snapshots (the reference interpolates one
   snapshot per call, PointSamples_interpolation.jl:12-29; this batches calls).  discs[k] is a
   handle on which pb_linear_bvh has built disc k (PB_BUILD_ASYNC allowed); npts[k] sample
   points at qx[k], qy[k], qz[k] and the L = n_scalar + 3 n_grad + n_div + 3 n_curl outputs
   out[k * L + l] are device memory.  Every disc's tree is cut into subtrees on the device; one
   walk launch covers every disc's (point, subtree) items and persistent kernels sum every
   disc's points (FP64: the reference's arithmetic; FP32C: queries with at most fp64_light_max
   neighbours in FP64, the rest FP32-compensated, decided on the device), with values equal to
   separate pb_interpolate_points calls bit for bit.  Every handle must use the first one's
   device, stream (pb_set_stream) and kernel; the catalog must fit one launch.  Options of
   discs[0]: "leaf_size" (walk cutoff), "batch_walk_split" (target subtrees per disc, 1..1024,
   default 16), "batch_order" (0 given, 1 most work first) and "batch_blocks_per_sm" (0 = all
   that fit) change the schedule only.  With device pointers, no
   synchronisation and all buffers already sized by an earlier identical call, the builds with
   PB_BUILD_ASYNC and this call with PB_BATCH_ASYNC can be captured in a CUDA graph. */
int32_t pb_batch_points(pb_handle *const *discs, int32_t ndiscs, const pb_catalog *cat, const int64_t *npts,
                        const double *const *qx, const double *const *qy, const double *const *qz, double *const *out,
                        int32_t strategy, int32_t precision, int32_t flags);
/* Wait for the batch's stream and check every disc's device status word (build and traversal). */
int32_t pb_batch_check(pb_handle *const *discs, int32_t ndiscs);

/* Morton encode + stable radix sort + duplicate bump of the LBVH build (the sorted
   MortonEncoding codes and the 0-based sorting order) without allocating any device memory.
   This entry point has no counterpart in the reference: it exists for callers that cannot
   call cudaMalloc -- applications that own all device memory through their own pool, or
   pipelines that cannot take the synchronisation an allocation may imply.  Its sort scratch
   is one fixed static device array (about 6.3 MB per GPU, held until exit) shared by every
   call: n <= PB_NOALLOC_MAX_N (larger n returns PB_ERR_CAPACITY), calls whose GPU work
   overlaps race on it, and the first call on a device (which looks up the array's address)
   should come before any stream capture.  x, y, z, codes_out, order_out are device pointers;
   the call is synchronous on `cuda_stream` (NULL = the default stream). */
#define PB_NOALLOC_MAX_N 262144
int32_t pb_morton_sort_noalloc(const double *x, const double *y, const double *z, int64_t n, uint64_t *codes_out,
                               int64_t *order_out, void *cuda_stream);

/* Diagnostics: kernels launched by this handle so far; build / traversal device time of
   the last call in ms (needs option "timing"); traversal kernel launches of the last call. */
int64_t pb_launch_count(const pb_handle *h);
int32_t pb_last_timings(const pb_handle *h, double *build_ms, double *interp_ms, int64_t *interp_launches);

/* Sample points of a structured grid generated on the device: coordinate_grid + flatten
   (Partia.jl/src/julia/Grids/grids/StructuredGrid.jl:126-204, grids/transform.jl:53-66),
   column-major (first axis fastest).  coord: 0 Cartesian (axes x, y, z), 2 cylindrical
   (s, phi, z), 3 spherical (r, phi, theta).  Axes may be host or device arrays; when x, y, z
   are device arrays the points never leave the device (no host-to-device copy of sample
   coordinates).  Trigonometric values are the device's libm, within 2 ulp of the host's. */
int32_t pb_grid_points(pb_handle *h, int32_t coord, const double *a0, int64_t n0, const double *a1, int64_t n1,
                       const double *a2, int64_t n2, double *x, double *y, double *z);

/* Lines of an image generated on the device: the LineSamples(xo, yo, zo, xd, yd, zd) a caller
   builds for a column-density image (Partia.jl/src/julia/Grids/grids/LineSamples.jl:391-403;
   the CUDA extension copies those host arrays to the device,
   Partia.jl/ext/CUDAExt/Grids/grids/LineSamples.jl:1-7).  Line k = i + n0 * j (the first
   axis fastest, as flatten orders a grid) starts at (c + a0[i] e1) + a1[j] e2 and runs along d,
   evaluated per component without FMA.  frame holds 12 doubles (host memory): c, e1, e2, d;
   d must be a unit vector (|d| within 1e-12 of 1; else PB_ERR_INVALID).  The face-on image of a
   disc is c = (0, 0, z0), e1 = (1, 0, 0), e2 = (0, 1, 0), d = (0, 0, 1).  Axes may be host or
   device arrays; with device outputs the lines never cross PCIe. */
int32_t pb_line_image(pb_handle *h, const double *a0, int64_t n0, const double *a1, int64_t n1, const double *frame,
                      double *ox, double *oy, double *oz, double *dx, double *dy, double *dz);

/* build_input on the device (ParticleIO.jl/src/julia/PartiaAdapter/build_input.jl:44-160):
   the interpolation input's FP64 columns made from a snapshot's columns where they will be
   used, so they cross PCIe in the width the dump stores them in (Phantom writes h and most
   per-particle quantities as real*4).  All arrays are device memory of the handle's device.
   pb_column_to_f64: dst[i] = src[i] widened to double (src_type 0 = float64, 1 = float32).
   pb_fill_f64: dst[i] = value (a mass given once for all particles, MassFromParams).
   pb_density_from_h: rho[i] = (mass hfact^3) (1/h[i])^3, add_rho! in 3D
   (ParticleIO.jl/src/julia/Particles/add_quantities.jl:308-345), in its operation order. */
int32_t pb_column_to_f64(pb_handle *h, const void *src, int32_t src_type, int64_t n, double *dst);
int32_t pb_fill_f64(pb_handle *h, double value, int64_t n, double *dst);
int32_t pb_density_from_h(pb_handle *h, const double *hsml, int64_t n, double mass, double hfact, double *rho);

/* Learned work prediction for the FP32-compensated point schedule (no counterpart in the
   reference; the reference runs queries in input order).  A 3-layer MLP of width 64 with
   BF16 weights and activations (PB_SCHED_FEATURES inputs, PB_SCHED_PARAMS parameters laid out
   W1[64][F], b1[64], W2[64][64], b2[64], W3[64], b3) predicts log2(1 + accepted neighbours) of
   a sample point; option "schedule" = 2 then walks the queries binned by predicted work
   (class = floor(prediction / bin_width), heaviest first).  Outputs do not depend on it.
   pb_scheduler_features: the npts x F features of sample points on the last build.
   pb_scheduler_set: weights, input normalisation norm[2F] = (mean[F], 1/std[F]), bins.
   pb_scheduler_train: Adam on the device (own forward/backward kernels), minibatches drawn
   with `seed`, starting from the current weights; losses[steps] (may be NULL) = batch MSE.
   pb_scheduler_gradients: gradient of the mean squared error over all n samples.
   Arrays may be host or device memory. */
#define PB_SCHED_FEATURES 16
#define PB_SCHED_PARAMS 5313
int32_t pb_scheduler_features(pb_handle *h, int64_t npts, const double *qx, const double *qy, const double *qz,
                              float *feat);
int32_t pb_scheduler_set(pb_handle *h, const float *params, const float *norm, float bin_width, int32_t nclass);
int32_t pb_scheduler_get(pb_handle *h, float *params);
int32_t pb_scheduler_predict(pb_handle *h, const float *X, int64_t n, float *out);
int32_t pb_scheduler_gradients(pb_handle *h, const float *X, const float *y, int64_t n, float *grads, float *loss);
int32_t pb_scheduler_train(pb_handle *h, const float *X, const float *y, int64_t n, int32_t steps, int32_t batch,
                           float lr, uint64_t seed, float *losses);

/* Diagnostics of the last FP32-compensated point call (no counterpart in the reference):
   walk rounds taken, queries deferred because the accepted-run pool was full (they are walked
   again, or finished by the fused kernel), the pool size in chunks of 32 runs, and (with
   option "timing") the device time in ms of the phases, summed over slices and walk rounds,
   in phase_ms[3]: nearest search (with the learned binning), walk (with the prefilter and the
   pair ordering), pair sums.  The pool follows
   PB_RUN_POOL_MB (MiB) or PB_RUN_POOL_CHUNKS from the environment when set. */
int32_t pb_last_schedule(const pb_handle *h, int64_t *walk_rounds, int64_t *deferred, int64_t *pool_chunks,
                         double *phase_ms);
/* Diagnostics of the last point call (no counterpart in the reference): how the queries and
   their accepted pairs were split between the FP32-compensated pair kernel (queries with more
   than option "fp64_light_max" accepted neighbours; heavy) and the FP64 pair kernel (light).
   In PB_FP64 mode every query is light.  Any output may be NULL. */
int32_t pb_last_pair_split(const pb_handle *h, int64_t *heavy_queries, int64_t *light_queries, int64_t *heavy_pairs,
                           int64_t *light_pairs);

#ifdef __cplusplus
}
#endif

#endif /* PARTIA_B200_H */
