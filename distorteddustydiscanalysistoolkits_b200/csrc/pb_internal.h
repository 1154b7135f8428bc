// pb_internal.h -- host-side handle and the launchers shared between translation units.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "pb_device.cuh"

namespace pb {

// One disc of a batched launch (pb_batch.cu): its tree, the FP32C and FP64 catalogs of its
// columns and outputs, its FP32C payload, and its sample points.
struct QuantParams;

struct BatchDisc {
    DevTree T;
    DevCatalog C32, C64;
    const float4 *pay;
    const double *qx, *qy, *qz;
    const int2 *cut;     // the disc's walk cut (subtree root, node after it), in DFS order
    const int *ncut;     // its number of subtrees (device-resident: the cut is made on the device)
    const QuantParams *qp;   // the disc's quantisation frame (Morton order of its sample points)
    int64_t nq;
    int stride;
    int pad;
};
static_assert(sizeof(BatchDisc) % 8 == 0, "batch descriptors are copied in 8-byte words");

// grow-only device buffer
struct DBuf {
    void *p = nullptr;
    size_t bytes = 0;
    cudaError_t reserve(size_t b)
    {
        if (b <= bytes) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, b < 256 ? 256 : b);
        if (e == cudaSuccess) bytes = b < 256 ? 256 : b;
        return e;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <typename T> T *as() const { return static_cast<T *>(p); }
};

// learned schedule: MLP of SCHED_F features -> SCHED_H -> SCHED_H -> 1
constexpr int SCHED_F = 16;
constexpr int SCHED_H = 64;
constexpr int SCHED_NPARAM = SCHED_H * SCHED_F + SCHED_H + SCHED_H * SCHED_H + SCHED_H + SCHED_H + 1;

struct QuantParams {
    double vmin[3];
    double inv[3];
    int flat[3];   // axis with zero extent: every particle gets f = 0.5
    int pad;
};

struct Handle {
    int device = 0;
    cudaStream_t stream = nullptr;       // where launches go
    cudaStream_t own_stream = nullptr;   // created by pb_create
    std::string err;
    int64_t launches = 0;

    // built particle set
    bool built = false;
    int64_t n = 0;
    int ncol = 0;
    int kernel = 0;

    DBuf in_x, in_y, in_z, in_h, in_m, in_rho;    // staging for host inputs
    std::vector<DBuf> in_cols;
    DBuf codes, codes_alt, idx, idx_alt, scan_tmp, scan_part, hist;
    DBuf bbox_part, qparams, status;
    DBuf leaf, leaf_escape, node, node_hmax, node_child, node_range;
    DBuf payload;       // per-call FP32 particle payload of the FP32-compensated path
    DBuf counter;       // work-queue counter of the warp-per-query kernels
    DBuf left, right, escape, parent;
    DBuf bmin64, bmax64, hmax64, counters;
    DBuf m_s, rho_s;
    std::vector<DBuf> cols_s;
    DBuf col_ptrs;      // device array of sorted column pointers

    // run lists of the two-phase point path (walk kernel -> pair kernels)
    DBuf grid_ax, grid_out;   // axes / points of pb_grid_points
    DBuf wl_cnt, wl_off, wl_s, wl_j, wl_sa, wl_ja;   // (query, subtree) work list of the walk
    DBuf pool_runs, pool_next, pool_ctr, items, wbnear, qacc, qflag, cut, defer_a, defer_b, lpt_k, lpt_v, lpt_ka,
        lpt_va, iota;
    int walk_split = 64;   // target number of subtrees each query's walk is split into
    int sched = 1;         // 0 plain (input order, one walk per query, no ordering), 1 tuned, 2 learned
    int64_t light_max = 4096;   // FP32C: queries with at most this many neighbours are summed in FP64
    int64_t slice = int64_t(1) << 22;   // queries per two-phase slice
    double pool_cpq = 0.0;   // largest pool chunks per completed query seen by the last call (0: none)
    // learned work prediction (pb_sched.cu)
    DBuf mlp_w, mlp_m, mlp_v, mlp_g, mlp_norm, mlp_scr, mlp_idx, mlp_x, mlp_y, mlp_loss, sched_feat, sched_pred,
        sched_ql, sched_tmp;
    bool mlp_ready = false;
    float sched_width = 1.f;
    int sched_nclass = 16;
    unsigned long long pool_cap = 0;
    int64_t walk_rounds = 0, deferred_total = 0;
    // queries and accepted pairs of the last point call summed by the FP32C (heavy) and the
    // FP64 (light) pair kernels
    int64_t split_hq = 0, split_lq = 0, split_hp = 0, split_lp = 0;

    // batched launch (pb_batch_points): descriptors, processing-order starts, pinned staging
    DBuf batch_desc, batch_starts, batch_slots, batch_ctr;
    void *batch_host = nullptr;
    size_t batch_host_bytes = 0;
    int leaf_size = 1;       // warp-uniform walk: subtrees of at most this many leaves are scanned
    int batch_order = 0;     // 0: discs in the given order, 1: discs with the most work first
    int batch_blocks = 0;    // blocks per SM of the batched pair kernel (0: as many as fit)
    int64_t batch_slice = 0; // sample points per slice the batch's run pool was sized for
    int batch_ns = 0;        // subtrees per point the batch's item records were sized for
    int batch_walk_split = 16;   // target number of subtrees per disc of the batched walk
    DBuf batch_slot_of;      // processing slot of every point of a slice
    DBuf batch_bcnt, batch_boff, batch_bcur, batch_list;   // walk prefilter: buckets and item list
    DBuf batch_mk, batch_mka, batch_mv, batch_mva;         // Morton walk order of a slice

    // query-side scratch
    DBuf q_x, q_y, q_z, q_keys, q_keys_alt, q_perm, q_perm_alt, q_out, q_aux;
    std::vector<DBuf> q_outs;

    // timing (CUDA events around the build and the traversal launches)
    bool timing = false;
    cudaEvent_t ev[8] = {};
    float t_build_ms = 0.f, t_interp_ms = 0.f;
    float t_phase_ms[3] = {0.f, 0.f, 0.f};   // nearest search, walk (+ ordering), pairs; all slices and rounds
    int64_t interp_launches = 0;
    int sort_queries = 1;
    int block_size = 128;

    ~Handle();
};

// ---- launchers (pb_build.cu) ----
cudaError_t launch_bbox(Handle *H, int64_t n, const double *x, const double *y, const double *z, const double *h);
cudaError_t launch_encode(Handle *H, int64_t n, const double *x, const double *y, const double *z);
cudaError_t sort_pairs_u64(Handle *H, uint64_t *keys, uint32_t *vals, uint64_t *kalt, uint32_t *valt, int64_t n,
                           int bits);
cudaError_t sort_pairs_u32(Handle *H, uint32_t *keys, uint32_t *vals, uint32_t *kalt, uint32_t *valt, int64_t n,
                           int bits);
cudaError_t launch_exclusive_scan_u32(Handle *H, const uint32_t *in, uint32_t *out, int64_t m);
// per point t of a batch slice: key (processing slot << 32) | Morton code of the point in its
// disc's quantisation frame, value t
cudaError_t launch_batch_query_codes(Handle *H, int64_t m, const BatchDisc *discs, const int64_t *starts,
                                     const uint32_t *slot_disc, const int *slot_of, int64_t s0, uint64_t *keys,
                                     uint32_t *vals);
cudaError_t launch_dedupe(Handle *H, uint64_t *codes, int64_t n);
cudaError_t launch_gather(Handle *H, int64_t n, const double *x, const double *y, const double *z, const double *h,
                          const double *m, const double *rho, const std::vector<const double *> &cols);
cudaError_t launch_topology(Handle *H, int64_t n);
cudaError_t launch_query_codes(Handle *H, int64_t nq, const double *qx, const double *qy, const double *qz,
                               uint32_t *keys, uint32_t *perm);
cudaError_t launch_permute_back(Handle *H, int64_t n, const uint32_t *idx, const double *src, double *dst);

// ---- launchers (pb_walk.cu) ----
cudaError_t launch_cut(Handle *H, const DevTree &T, int target, int *ns_out);
// launch_cut without the read-back: the ordered cut and its size stay on the device
cudaError_t launch_cut_device(Handle *H, const DevTree &T, int target, const int2 **cut, const int **count);
cudaError_t launch_nearest_list(Handle *H, const DevTree &T, int64_t m, const uint32_t *ql, const double *qx,
                                const double *qy, const double *qz, int *bnear);
cudaError_t launch_walk(Handle *H, const DevTree &T, int strategy, const RunPool &P, int64_t m, const uint32_t *ql,
                        const double *qx, const double *qy, const double *qz, unsigned long long *counter);
cudaError_t launch_walk_list(Handle *H, const DevTree &T, int strategy, const RunPool &P, int64_t m,
                             const uint32_t *ql, const double *qx, const double *qy, const double *qz,
                             unsigned long long *counter);
cudaError_t launch_lpt_order(Handle *H, const RunPool &P, int64_t m, uint32_t **order);
cudaError_t launch_split_order(Handle *H, const RunPool &P, int64_t m, unsigned light_max, bool plain,
                               uint32_t **order, int64_t *m_heavy, unsigned long long *pairs);
cudaError_t launch_iota(Handle *H, int64_t m, uint32_t *out);
cudaError_t launch_count_heavy(Handle *H, const RunPool &P, int64_t m, unsigned light_max, unsigned *count,
                               unsigned long long *pairs);
int batch_catalog_shape(const DevCatalog &C32);

// ---- launchers (pb_sched.cu) ----
cudaError_t launch_sched_features(Handle *H, const DevTree &T, int64_t m, const uint32_t *ql, const double *qx,
                                  const double *qy, const double *qz, const int *bnear, float *feat);
cudaError_t launch_mlp_predict(Handle *H, int64_t n, const float *X, float *y);
cudaError_t launch_mlp_grad(Handle *H, int64_t nb, const float *X, const float *T, const int64_t *idx, float *loss);
const float *mlp_last_sq(Handle *H, int64_t nb);
cudaError_t launch_mlp_adam(Handle *H, float lr, int64_t step);
cudaError_t launch_draw(Handle *H, int64_t nb, int64_t n, unsigned long long seed, unsigned long long step,
                        int64_t *idx);
cudaError_t launch_sched_order(Handle *H, int64_t m, const float *pred, float width, int nclass, uint32_t *order);
cudaError_t launch_gather_u32(Handle *H, int64_t m, const uint32_t *order, const uint32_t *src, uint32_t *dst);
cudaError_t launch_gather_i32(Handle *H, int64_t m, const uint32_t *order, const int *src, int *dst);

// ---- launchers (pb_interp64.cu / pb_interp32.cu / pb_query.cu) ----
cudaError_t launch_pairs_fp32(Handle *H, const DevTree &T, const DevCatalog &C, int strategy, const RunPool &P,
                              int64_t m, const uint32_t *ql, const uint32_t *order, const double *qx,
                              const double *qy, const double *qz);
cudaError_t launch_points_fp64(Handle *H, const DevTree &T, const DevCatalog &C, int strategy, int64_t nq,
                               const double *qx, const double *qy, const double *qz, const uint32_t *perm,
                               int64_t npts);
cudaError_t launch_pairs_fp64(Handle *H, const DevTree &T, const DevCatalog &C, int strategy, const RunPool &P,
                              int64_t m, const uint32_t *ql, const uint32_t *order, const double *qx,
                              const double *qy, const double *qz);
cudaError_t launch_points_fp32(Handle *H, const DevTree &T, const DevCatalog &C, int strategy, int64_t nq,
                               const double *qx, const double *qy, const double *qz, const uint32_t *perm,
                               int64_t npts);
cudaError_t launch_lines_fp64(Handle *H, const DevTree &T, const DevCatalog &C, int64_t nl, const double *ox,
                              const double *oy, const double *oz, const double *dx, const double *dy,
                              const double *dz, const uint32_t *perm);
cudaError_t launch_nearest(Handle *H, const DevTree &T, int64_t nq, const double *qx, const double *qy,
                           const double *qz, double *h_out, int64_t *idx_out);
cudaError_t launch_query(Handle *H, const DevTree &T, int64_t nq, const double *qx, const double *qy,
                         const double *qz, const double *radius, const int64_t *offsets, int64_t *counts,
                         int64_t *pool, int64_t *nearest, double *nearest_d2);
cudaError_t launch_grid_points(Handle *H, int coord, const double *a0, int64_t n0, const double *a1, int64_t n1,
                               const double *a2, int64_t n2, double *x, double *y, double *z);
cudaError_t launch_stats(Handle *H, const DevTree &T, int strategy, int64_t nq, const double *qx, const double *qy,
                         const double *qz, int64_t *stats);
// image plane of pb_line_image: origin c, axes e1 and e2, line direction d
struct LineFrame {
    double c[3], e1[3], e2[3], d[3];
};
cudaError_t launch_batch_slice(Handle *H, int strategy, int kernel, int cat, const BatchDisc *discs,
                               const int64_t *starts, const uint32_t *slot_disc, int ndisc, int64_t s0, int64_t m,
                               const RunPool &P, int fp64_only, unsigned light_max, int leaf_size, int blocks_per_sm,
                               int *slot_of, unsigned long long *ctr);
cudaError_t launch_batch_payload(Handle *H, const DevTree &T, const DevCatalog &C, float4 **pay, int *stride);
cudaError_t launch_line_image(Handle *H, const double *a0, int64_t n0, const double *a1, int64_t n1, const LineFrame &F,
                              double *ox, double *oy, double *oz, double *dx, double *dy, double *dz);

inline int grid_for(int64_t n, int block, int cap = 148 * 32)
{
    int64_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}

}  // namespace pb

// the opaque handle of the C ABI (include/partia_b200.h)
struct pb_handle {
    pb::Handle H;
};
