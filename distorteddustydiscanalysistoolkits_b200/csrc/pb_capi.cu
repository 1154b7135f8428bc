// pb_capi.cu -- the extern "C" boundary of libpartia_b200.so (declared in include/partia_b200.h).
//
// Host orchestration only: argument validation with the reference's error classes,
// host/device pointer detection and staging, catalog planning (a catalog larger than one
// launch's register budget is split into several traversal launches), device status
// checks, and optional CUDA-event timing of the build and traversal stages.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "partia_b200.h"
#include "pb_internal.h"

using namespace pb;


pb::Handle::~Handle()
{
    DBuf *all[] = {&in_x, &in_y, &in_z, &in_h, &in_m, &in_rho, &codes, &codes_alt, &idx, &idx_alt, &scan_tmp,
                   &scan_part, &hist, &bbox_part, &qparams, &status, &leaf, &leaf_escape, &node, &node_hmax, &node_child, &node_range, &payload, &counter, &left,
                   &right, &escape, &parent, &bmin64, &bmax64, &hmax64, &counters, &m_s, &rho_s, &col_ptrs,
                   &q_x, &q_y, &q_z, &q_keys, &q_keys_alt, &q_perm, &q_perm_alt, &q_out, &q_aux,
                   &pool_runs, &pool_next, &pool_ctr, &items, &wbnear, &qacc, &qflag, &cut, &defer_a, &defer_b,
                   &lpt_k, &lpt_v, &lpt_ka, &lpt_va, &iota, &grid_ax, &grid_out, &wl_cnt, &wl_off, &wl_s, &wl_j, &wl_sa, &wl_ja, &mlp_w, &mlp_m, &mlp_v, &mlp_g, &mlp_norm,
                   &mlp_scr, &mlp_idx, &mlp_x, &mlp_y, &mlp_loss, &sched_feat, &sched_pred, &sched_ql, &sched_tmp};
    for (DBuf *b : all) b->release();
    batch_desc.release();
    batch_starts.release();
    batch_slots.release();
    batch_ctr.release();
    if (batch_host) cudaFreeHost(batch_host);
    for (auto &b : in_cols) b.release();
    for (auto &b : cols_s) b.release();
    for (auto &b : q_outs) b.release();
    for (auto &e : ev)
        if (e) cudaEventDestroy(e);
    if (own_stream) cudaStreamDestroy(own_stream);
}

namespace {

int fail(Handle &H, int code, const std::string &msg)
{
    H.err = msg;
    return code;
}

#define CK(expr)                                                                                     \
    do {                                                                                             \
        cudaError_t _e = (expr);                                                                     \
        if (_e != cudaSuccess)                                                                       \
            return fail(H, PB_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e));         \
    } while (0)

// Where a caller pointer lives: 0 host memory (pageable or pinned), 1 device memory of the
// handle's device or managed memory, 2 device memory of another GPU (rejected: the kernels
// would read it without peer access).
int ptr_place(const Handle &H, const void *p)
{
    if (!p) return 0;
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (a.type == cudaMemoryTypeManaged) return 1;
    if (a.type == cudaMemoryTypeDevice) return a.device == H.device ? 1 : 2;
    return 0;
}

bool is_device_ptr(const Handle &H, const void *p) { return ptr_place(H, p) == 1; }

// device view of a caller array: the array itself if it lives on the device, else a staged copy
cudaError_t stage_in(Handle &H, DBuf &buf, const void *p, size_t bytes, const void **out)
{
    const int place = ptr_place(H, p);
    if (place == 2) return cudaErrorInvalidDevice;
    if (place == 1) {
        *out = p;
        return cudaSuccess;
    }
    cudaError_t e = buf.reserve(bytes);
    if (e) return e;
    e = cudaMemcpyAsync(buf.p, p, bytes, cudaMemcpyHostToDevice, H.stream);
    *out = buf.p;
    return e;
}

int check_status(Handle &H)
{
    int st = 0;
    CK(cudaMemcpyAsync(&st, H.status.p, sizeof(int), cudaMemcpyDeviceToHost, H.stream));
    CK(cudaStreamSynchronize(H.stream));
    if (st & ST_NONFINITE) return fail(H, PB_ERR_INVALID, "non-finite particle coordinate or smoothing length");
    if (st & ST_REFIT) return fail(H, PB_ERR_INTERNAL, "LBVH refit: an internal node was not combined exactly twice");
    if (st & ST_TRAVERSAL) return fail(H, PB_ERR_INTERNAL, "traversal exceeded its iteration bound");
    if (st & ST_POOL)
        return fail(H, PB_ERR_DIMENSION, "neighbour pool offsets too small for a query (DimensionMismatch)");
    if (st & ST_CUT) return fail(H, PB_ERR_INTERNAL, "walk cut larger than its capacity (raise batch_walk_split)");
    return PB_OK;
}

DevTree make_tree(Handle &H)
{
    DevTree T;
    T.n = H.n;
    T.root = H.n >= 2 ? 1 : 0;
    T.leaf = H.leaf.as<double4>();
    T.leaf_escape = H.leaf_escape.as<int>();
    T.node = H.node.as<NodeF>();
    T.node_hmax = H.node_hmax.as<float>();
    T.child = H.node_child.as<int2>();
    T.range = H.node_range.as<int2>();
    T.m = H.m_s.as<double>();
    T.rho = H.rho_s.as<double>();
    T.kernel = H.kernel;
    T.status = H.status.as<int>();
    return T;
}

void ev_record(Handle &H, int i)
{
    if (!H.timing) return;
    if (!H.ev[i]) cudaEventCreate(&H.ev[i]);
    cudaEventRecord(H.ev[i], H.stream);
}

float ev_ms(Handle &H, int a, int b)
{
    if (!H.timing || !H.ev[a] || !H.ev[b]) return 0.f;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, H.ev[a], H.ev[b]);
    return ms;
}

// ---------------------------------------------------------------------------------------
// catalog planning
struct Item {
    int kind;          // 0 scalar, 1 grad, 2 div, 3 curl
    int cols[3];       // column ids (-1 = density for grads, -2 = rho pseudo column in FP32 mode)
    int ncols;
    int shep;
    int out0;          // first global output index
};

int validate_catalog(Handle &H, const pb_catalog *c, bool lines)
{
    if (!c) return fail(H, PB_ERR_INVALID, "catalog is NULL");
    if (c->n_scalar < 0 || c->n_grad < 0 || c->n_div < 0 || c->n_curl < 0)
        return fail(H, PB_ERR_INVALID, "negative catalog count");
    if (lines && (c->n_grad || c->n_div || c->n_curl))
        return fail(H, PB_ERR_INVALID, "LineSamples interpolation takes scalar quantities only");
    auto okcol = [&](int col) { return col >= 0 && col < H.ncol; };
    for (int i = 0; i < c->n_scalar; ++i)
        if (!okcol(c->scalar_cols[i])) return fail(H, PB_ERR_KEY, "scalar column out of range (KeyError)");
    for (int i = 0; i < c->n_grad; ++i)
        if (c->grad_cols[i] != -1 && !okcol(c->grad_cols[i]))
            return fail(H, PB_ERR_KEY, "gradient column out of range (KeyError)");
    for (int i = 0; i < 3 * c->n_div; ++i)
        if (!okcol(c->div_cols[i])) return fail(H, PB_ERR_KEY, "divergence column out of range (KeyError)");
    for (int i = 0; i < 3 * c->n_curl; ++i)
        if (!okcol(c->curl_cols[i])) return fail(H, PB_ERR_KEY, "curl column out of range (KeyError)");
    return PB_OK;
}

std::vector<Item> items_of(const pb_catalog *c, bool fp32)
{
    std::vector<Item> it;
    int o = 0;
    for (int i = 0; i < c->n_scalar; ++i) {
        Item x{0, {c->scalar_cols[i], 0, 0}, 1, c->scalar_shepard ? (c->scalar_shepard[i] != 0) : 1, o};
        it.push_back(x);
        o += 1;
    }
    for (int i = 0; i < c->n_grad; ++i) {
        int col = c->grad_cols[i];
        Item x{1, {col, 0, 0}, col == -1 ? 0 : 1, 0, o};
        if (col == -1 && fp32) { x.cols[0] = -2; x.ncols = 1; }
        it.push_back(x);
        o += 3;
    }
    for (int i = 0; i < c->n_div; ++i) {
        Item x{2, {c->div_cols[3 * i], c->div_cols[3 * i + 1], c->div_cols[3 * i + 2]}, 3, 0, o};
        it.push_back(x);
        o += 1;
    }
    for (int i = 0; i < c->n_curl; ++i) {
        Item x{3, {c->curl_cols[3 * i], c->curl_cols[3 * i + 1], c->curl_cols[3 * i + 2]}, 3, 0, o};
        it.push_back(x);
        o += 3;
    }
    return it;
}

struct Launch {
    std::vector<int> ucols;   // column of each slot u
    std::vector<Item> items;
    int cnt[4] = {0, 0, 0, 0};
};

constexpr int PB_COL_NONE = -100;

// Fixed slot layout of a launch: the gradient's column in slot 0, the divergence/curl vector
// in slots 1..3 (one vector per launch), scalars in the slots left over or in the slot that
// already holds their column.  The pair kernels then read every term's operands from fixed
// slots.  Returns false when the items do not fit MAXU slots.
bool layout(const std::vector<Item> &items, std::vector<int> &slots)
{
    std::vector<int> u(MAXU, PB_COL_NONE);
    bool vec = false;
    for (const Item &x : items) {
        if (x.kind == 1 && x.ncols > 0) {
            if (u[0] != PB_COL_NONE && u[0] != x.cols[0]) return false;
            u[0] = x.cols[0];
        }
        if (x.kind >= 2) {
            for (int d = 0; d < 3; ++d) {
                if (u[1 + d] != PB_COL_NONE && u[1 + d] != x.cols[d]) return false;
                u[1 + d] = x.cols[d];
            }
            vec = true;
        }
    }
    for (const Item &x : items) {
        if (x.kind != 0) continue;
        if (std::find(u.begin(), u.end(), x.cols[0]) != u.end()) continue;
        auto it = std::find(u.begin(), u.end(), PB_COL_NONE);
        if (it == u.end()) return false;
        *it = x.cols[0];
    }
    // slot 0 is read whenever a vector is present: it then holds a real column
    if (vec && u[0] == PB_COL_NONE) u[0] = u[1];
    int used = 0;
    for (int k = 0; k < MAXU; ++k)
        if (u[k] != PB_COL_NONE) used = k + 1;
    for (int k = 0; k < used; ++k)
        if (u[k] == PB_COL_NONE) u[k] = u[0] != PB_COL_NONE ? u[0] : u[1];
    u.resize(used);
    slots = u;
    return true;
}

std::vector<Launch> plan(const std::vector<Item> &items)
{
    const int lim[4] = {MAXS, MAXG, MAXD, MAXC};
    std::vector<Launch> out;
    Launch cur;
    for (const Item &x : items) {
        std::vector<Item> trial = cur.items;
        trial.push_back(x);
        std::vector<int> u;
        bool fits = cur.cnt[x.kind] < lim[x.kind] && layout(trial, u);
        if (!fits) {
            out.push_back(cur);
            cur = Launch();
            trial.assign(1, x);
            layout(trial, u);
        }
        cur.ucols = u;
        cur.items.push_back(x);
        cur.cnt[x.kind]++;
    }
    if (!cur.items.empty()) out.push_back(cur);
    return out;
}

int uidx(const Launch &L, int col)
{
    for (size_t i = 0; i < L.ucols.size(); ++i)
        if (L.ucols[i] == col) return (int)i;
    return -1;
}

DevCatalog dev_catalog(Handle &H, const Launch &L, double *const *outs)
{
    DevCatalog C;
    memset(&C, 0, sizeof(C));
    C.nU = (int)L.ucols.size();
    for (int u = 0; u < C.nU; ++u) {
        int col = L.ucols[u];
        C.ucol[u] = col == -2 ? H.rho_s.as<double>() : H.cols_s[col].as<double>();
    }
    int l = 0;
    // kernel writes scalars, grads, divs, curls in that order
    for (int kind = 0; kind < 4; ++kind) {
        for (const Item &x : L.items) {
            if (x.kind != kind) continue;
            if (kind == 0) {
                C.s_u[C.n_scalar] = uidx(L, x.cols[0]);
                C.s_shep[C.n_scalar] = x.shep;
                C.n_scalar++;
                C.out[l++] = outs[x.out0];
            } else if (kind == 1) {
                C.g_u[C.n_grad] = x.cols[0] == -1 ? -1 : 0;
                C.n_grad++;
                for (int d = 0; d < 3; ++d) C.out[l++] = outs[x.out0 + d];
            } else if (kind == 2) {
                for (int d = 0; d < 3; ++d) C.d_u[C.n_div][d] = 1 + d;
                C.n_div++;
                C.out[l++] = outs[x.out0];
            } else {
                for (int d = 0; d < 3; ++d) C.c_u[C.n_curl][d] = 1 + d;
                C.n_curl++;
                for (int d = 0; d < 3; ++d) C.out[l++] = outs[x.out0 + d];
            }
        }
    }
    C.L = l;
    return C;
}

int64_t catalog_L(const pb_catalog *c) { return c->n_scalar + 3 * c->n_grad + c->n_div + 3 * c->n_curl; }

// stage output pointers: device outputs are written in place, host outputs via staging
int stage_outputs(Handle &H, int64_t L, int64_t npts, double *const *out, std::vector<double *> &dev,
                  std::vector<int> &is_host)
{
    dev.assign(L, nullptr);
    is_host.assign(L, 0);
    if ((int64_t)H.q_outs.size() < L) H.q_outs.resize(L);
    for (int64_t l = 0; l < L; ++l) {
        if (!out || !out[l]) return fail(H, PB_ERR_INVALID, "output pointer is NULL");
        if (ptr_place(H, out[l]) == 2) return fail(H, PB_ERR_INVALID, "output is device memory of another GPU");
        if (is_device_ptr(H, out[l])) dev[l] = out[l];
        else {
            CK(H.q_outs[l].reserve(sizeof(double) * npts));
            dev[l] = H.q_outs[l].as<double>();
            is_host[l] = 1;
        }
    }
    return PB_OK;
}

int finish_outputs(Handle &H, int64_t L, int64_t npts, double *const *out, const std::vector<double *> &dev,
                   const std::vector<int> &is_host)
{
    for (int64_t l = 0; l < L; ++l)
        if (is_host[l]) CK(cudaMemcpyAsync(out[l], dev[l], sizeof(double) * npts, cudaMemcpyDeviceToHost, H.stream));
    return check_status(H);
}

int stage_queries(Handle &H, int64_t nq, const double *qx, const double *qy, const double *qz, const double **dx,
                  const double **dy, const double **dz)
{
    const void *a, *b, *c;
    CK(stage_in(H, H.q_x, qx, sizeof(double) * nq, &a));
    CK(stage_in(H, H.q_y, qy, sizeof(double) * nq, &b));
    CK(stage_in(H, H.q_z, qz, sizeof(double) * nq, &c));
    *dx = (const double *)a;
    *dy = (const double *)b;
    *dz = (const double *)c;
    return PB_OK;
}

// Morton order of the queries (a schedule only; each result goes to its own slot)
int query_order(Handle &H, int64_t nq, const double *dx, const double *dy, const double *dz, const uint32_t **perm)
{
    *perm = nullptr;
    if (!H.sort_queries || nq < 2) return PB_OK;
    CK(H.q_keys.reserve(sizeof(uint32_t) * nq));
    CK(H.q_keys_alt.reserve(sizeof(uint32_t) * nq));
    CK(H.q_perm.reserve(sizeof(uint32_t) * nq));
    CK(H.q_perm_alt.reserve(sizeof(uint32_t) * nq));
    CK(launch_query_codes(&H, nq, dx, dy, dz, H.q_keys.as<uint32_t>(), H.q_perm.as<uint32_t>()));
    CK(sort_pairs_u32(&H, H.q_keys.as<uint32_t>(), H.q_perm.as<uint32_t>(), H.q_keys_alt.as<uint32_t>(),
                      H.q_perm_alt.as<uint32_t>(), nq, 30));
    *perm = H.q_perm.as<uint32_t>();
    return PB_OK;
}

int do_build(Handle &H, const pb_input *in, int32_t flags)
{
    if (!in) return fail(H, PB_ERR_INVALID, "input is NULL");
    if ((flags & PB_BUILD_ASYNC) && (flags & PB_PERMUTE_CALLER))
        return fail(H, PB_ERR_INVALID, "PB_BUILD_ASYNC cannot permute the caller's arrays (that needs the sorted order)");
    int64_t n = in->npart;
    if (n < 1) return fail(H, PB_ERR_INVALID, "BinaryRadixTree: enc.codes must be non-empty (got n=0)");
    if (n > 1073741824LL) return fail(H, PB_ERR_CAPACITY, "n exceeds the Int32 node-id capacity (n <= 2^30)");
    if (in->kernel < 0 || in->kernel > 5) return fail(H, PB_ERR_INVALID, "unknown kernel id");
    if (in->ncolumn < 0 || (in->ncolumn > 0 && !in->quant)) return fail(H, PB_ERR_INVALID, "bad quantity columns");
    if (!in->x || !in->y || !in->z || !in->m || !in->h || !in->rho)
        return fail(H, PB_ERR_INVALID, "particle column pointer is NULL");
    for (int c = 0; c < in->ncolumn; ++c)
        if (!in->quant[c]) return fail(H, PB_ERR_INVALID, "quantity column pointer is NULL");
    CK(cudaSetDevice(H.device));
    H.built = false;
    const size_t nb = sizeof(double) * n;
    const void *x, *y, *z, *h, *m, *rho;
    CK(stage_in(H, H.in_x, in->x, nb, &x));
    CK(stage_in(H, H.in_y, in->y, nb, &y));
    CK(stage_in(H, H.in_z, in->z, nb, &z));
    CK(stage_in(H, H.in_h, in->h, nb, &h));
    CK(stage_in(H, H.in_m, in->m, nb, &m));
    CK(stage_in(H, H.in_rho, in->rho, nb, &rho));
    if ((int)H.in_cols.size() < in->ncolumn) H.in_cols.resize(in->ncolumn);
    if ((int)H.cols_s.size() < in->ncolumn) H.cols_s.resize(in->ncolumn);
    std::vector<const double *> cols(in->ncolumn);
    for (int c = 0; c < in->ncolumn; ++c) {
        const void *p;
        CK(stage_in(H, H.in_cols[c], in->quant[c], nb, &p));
        cols[c] = (const double *)p;
        CK(H.cols_s[c].reserve(nb));
    }
    int64_t nin = n > 1 ? n - 1 : 1, ntot = 2 * n - 1;
    CK(H.codes.reserve(8 * n));
    CK(H.codes_alt.reserve(8 * n));
    CK(H.idx.reserve(4 * n));
    CK(H.idx_alt.reserve(4 * n));
    CK(H.leaf.reserve(32 * n));
    CK(H.leaf_escape.reserve(4 * n));
    CK(H.node.reserve(sizeof(NodeF) * nin));
    CK(H.node_hmax.reserve(4 * nin));
    CK(H.node_child.reserve(8 * nin));
    CK(H.node_range.reserve(8 * nin));
    CK(H.left.reserve(4 * nin));
    CK(H.right.reserve(4 * nin));
    CK(H.escape.reserve(4 * ntot));
    CK(H.parent.reserve(4 * ntot));
    CK(H.bmin64.reserve(24 * nin));
    CK(H.bmax64.reserve(24 * nin));
    CK(H.hmax64.reserve(8 * nin));
    CK(H.counters.reserve(4 * nin));
    CK(H.m_s.reserve(nb));
    CK(H.rho_s.reserve(nb));
    CK(H.qparams.reserve(sizeof(QuantParams)));
    CK(H.status.reserve(sizeof(int)));
    CK(cudaMemsetAsync(H.status.p, 0, sizeof(int), H.stream));
    ev_record(H, 0);
    CK(launch_bbox(&H, n, (const double *)x, (const double *)y, (const double *)z, (const double *)h));
    CK(launch_encode(&H, n, (const double *)x, (const double *)y, (const double *)z));
    CK(sort_pairs_u64(&H, H.codes.as<uint64_t>(), H.idx.as<uint32_t>(), H.codes_alt.as<uint64_t>(),
                      H.idx_alt.as<uint32_t>(), n, 63));
    CK(launch_dedupe(&H, H.codes.as<uint64_t>(), n));
    CK(launch_gather(&H, n, (const double *)x, (const double *)y, (const double *)z, (const double *)h,
                     (const double *)m, (const double *)rho, cols));
    CK(launch_topology(&H, n));
    ev_record(H, 1);
    H.n = n;
    H.ncol = in->ncolumn;
    H.kernel = in->kernel;
    if (flags & PB_BUILD_ASYNC) {
        // no synchronisation: the status word is checked by a later synchronous call
        // (pb_batch_check, or any query or interpolation entry point)
        H.built = true;
        return PB_OK;
    }
    int rc = check_status(H);
    if (rc) return rc;
    H.t_build_ms = ev_ms(H, 0, 1);
    if (flags & PB_PERMUTE_CALLER) {
        // the reference permutes the caller's columns in place (InterpolationInput.jl:211-219)
        CK(H.q_aux.reserve(nb));
        const double *srcs[6] = {(const double *)x, (const double *)y, (const double *)z,
                                 (const double *)m, (const double *)h, (const double *)rho};
        const double *dsts[6] = {in->x, in->y, in->z, in->m, in->h, in->rho};
        for (int a = 0; a < 6 + in->ncolumn; ++a) {
            const double *s = a < 6 ? srcs[a] : cols[a - 6];
            double *d = const_cast<double *>(a < 6 ? dsts[a] : in->quant[a - 6]);
            CK(launch_permute_back(&H, n, H.idx.as<uint32_t>(), s, H.q_aux.as<double>()));
            CK(cudaMemcpyAsync(d, H.q_aux.p, nb, cudaMemcpyDefault, H.stream));
        }
        CK(cudaStreamSynchronize(H.stream));
    }
    H.built = true;
    return PB_OK;
}

// Run pool of the two-phase point path.  Its size follows the number of queries (24 chunks
// of 32 runs per query), bounded by half of the free device memory (at most 64 GiB), by
// PB_RUN_POOL_MB, or set exactly in chunks by PB_RUN_POOL_CHUNKS; it never drops below what
// one query can need (n/2 runs) unless one of the two variables asks for less.  Buffers only
// grow; the cap of a call is what it may use.
int reserve_pool(Handle &H, int64_t m, int ns)
{
    const unsigned long long per_chunk = sizeof(uint2) * RUN_CHUNK + sizeof(int);
    const unsigned long long min_chunks =
        (unsigned long long)((H.n / 2 + 1 + RUN_CHUNK - 1) / RUN_CHUNK) + (unsigned long long)ns + 64;
    unsigned long long want = (unsigned long long)m * 24ULL;
    if (want < min_chunks) want = min_chunks;
    const char *env = getenv("PB_RUN_POOL_MB");
    const char *envc = getenv("PB_RUN_POOL_CHUNKS");
    long long env_mb = env ? atoll(env) : 0, env_chunks = envc ? atoll(envc) : 0;
    unsigned long long budget;
    if (env_mb > 0) budget = (unsigned long long)env_mb << 20;
    else {
        // half of the free memory plus what the pool already holds, at most 64 GiB
        size_t fr = 0, tot = 0;
        CK(cudaMemGetInfo(&fr, &tot));
        budget = (fr + H.pool_runs.bytes + H.pool_next.bytes) / 2;
        if (budget > (64ULL << 30)) budget = 64ULL << 30;
    }
    unsigned long long cap = budget / per_chunk;
    if (cap > want) cap = want;
    if (env_mb <= 0 && cap < min_chunks) cap = min_chunks;
    // a pool an earlier call grew (grow_pool) is kept: its memory is already held
    const unsigned long long held = std::min<unsigned long long>(H.pool_runs.bytes / (sizeof(uint2) * RUN_CHUNK),
                                                                 H.pool_next.bytes / sizeof(int));
    if (env_mb <= 0 && held > cap) cap = held;
    if (env_chunks > 0) cap = (unsigned long long)env_chunks;
    if (cap < 1) cap = 1;
    if (cap > 0x7fffffffULL) cap = 0x7fffffffULL;
    for (;;) {
        cudaError_t e1 = H.pool_runs.reserve(sizeof(uint2) * RUN_CHUNK * cap);
        cudaError_t e2 = e1 ? e1 : H.pool_next.reserve(sizeof(int) * cap);
        if (e2 == cudaSuccess) break;
        cudaGetLastError();
        if (e2 != cudaErrorMemoryAllocation || cap / 2 < min_chunks)
            return fail(H, PB_ERR_CUDA, std::string("run pool allocation failed: ") + cudaGetErrorString(e2));
        H.pool_runs.release();
        H.pool_next.release();
        cap /= 2;
    }
    H.pool_cap = cap;
    CK(H.pool_ctr.reserve(64));   // [0] chunks used, [1] deferred | heavy count, [2] walk queue, [4..5] pair split
    CK(H.items.reserve(sizeof(int2) * m * ns));
    CK(H.wbnear.reserve(sizeof(int) * m));
    CK(H.qacc.reserve(sizeof(unsigned) * m));
    CK(H.qflag.reserve(sizeof(int) * m));
    CK(H.defer_a.reserve(sizeof(uint32_t) * m));
    CK(H.defer_b.reserve(sizeof(uint32_t) * m));
    return PB_OK;
}

// Fused walk-and-sum for the queries a full pool left over (P.deferred[0..nd)).  Their exact
// accepted counts come from a counting walk, so the light ones get the FP64 kernel and the
// heavy ones the FP32-compensated one, exactly as in the two-phase path.
int fused_fallback(Handle &H, const DevTree &T, const std::vector<Launch> &launches,
                   const std::vector<Launch> &launches64, std::vector<double *> &dev, int strategy, int64_t npts,
                   const double *dx, const double *dy, const double *dz, RunPool P, int64_t nd)
{
    std::vector<uint32_t> list(nd), heavy, light;
    std::vector<unsigned> acc(nd);
    uint32_t *lst = reinterpret_cast<uint32_t *>(H.sched_tmp.p);
    CK(H.sched_tmp.reserve(sizeof(uint32_t) * 2 * nd));
    lst = H.sched_tmp.as<uint32_t>();
    CK(cudaMemcpyAsync(lst, P.deferred, sizeof(uint32_t) * nd, cudaMemcpyDeviceToDevice, H.stream));
    CK(cudaMemsetAsync(P.qacc, 0, sizeof(unsigned) * nd, H.stream));
    CK(cudaMemsetAsync(P.qflag, 0, sizeof(int) * nd, H.stream));
    P.count_only = 1;
    if (strategy != SCATTER) CK(launch_nearest_list(&H, T, nd, lst, dx, dy, dz, P.bnear));
    unsigned long long *ctr = H.pool_ctr.as<unsigned long long>();
    CK(launch_walk(&H, T, strategy, P, nd, lst, dx, dy, dz, ctr + 2));
    CK(cudaMemcpyAsync(list.data(), lst, sizeof(uint32_t) * nd, cudaMemcpyDeviceToHost, H.stream));
    CK(cudaMemcpyAsync(acc.data(), P.qacc, sizeof(unsigned) * nd, cudaMemcpyDeviceToHost, H.stream));
    CK(cudaStreamSynchronize(H.stream));
    for (int64_t k = 0; k < nd; ++k) {
        const bool hv = acc[k] > (unsigned)H.light_max;
        (hv ? heavy : light).push_back(list[k]);
        (hv ? H.split_hp : H.split_lp) += acc[k];
    }
    H.split_hq += (int64_t)heavy.size();
    H.split_lq += (int64_t)light.size();
    uint32_t *hl = lst, *ll = lst + heavy.size();
    if (!heavy.empty())
        CK(cudaMemcpyAsync(hl, heavy.data(), sizeof(uint32_t) * heavy.size(), cudaMemcpyHostToDevice, H.stream));
    if (!light.empty())
        CK(cudaMemcpyAsync(ll, light.data(), sizeof(uint32_t) * light.size(), cudaMemcpyHostToDevice, H.stream));
    if (!heavy.empty())
        for (const Launch &Lc : launches) {
            DevCatalog C = dev_catalog(H, Lc, dev.data());
            CK(launch_points_fp32(&H, T, C, strategy, (int64_t)heavy.size(), dx, dy, dz, hl, npts));
            H.interp_launches++;
        }
    if (!light.empty())
        for (const Launch &Lc : launches64) {
            DevCatalog C = dev_catalog(H, Lc, dev.data());
            CK(launch_points_fp64(&H, T, C, strategy, (int64_t)light.size(), dx, dy, dz, ll, npts));
            H.interp_launches++;
        }
    CK(cudaStreamSynchronize(H.stream));
    return PB_OK;
}

// Doubles the run pool (within the budget of reserve_pool) after a round that deferred
// queries; the pool is empty between rounds, so nothing is lost.  Returns false if it cannot
// grow (at the budget, fixed by PB_RUN_POOL_CHUNKS, or out of memory).
bool grow_pool(Handle &H)
{
    if (getenv("PB_RUN_POOL_CHUNKS") || getenv("PB_RUN_POOL_MB")) return false;
    const unsigned long long per_chunk = sizeof(uint2) * RUN_CHUNK + sizeof(int);
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return false;
    unsigned long long budget = (fr + H.pool_runs.bytes + H.pool_next.bytes) / 2;
    if (budget > (64ULL << 30)) budget = 64ULL << 30;
    unsigned long long cap = std::min<unsigned long long>(2 * H.pool_cap, budget / per_chunk);
    if (cap > 0x7fffffffULL) cap = 0x7fffffffULL;
    if (cap <= H.pool_cap) return false;
    H.pool_runs.release();
    H.pool_next.release();
    if (H.pool_runs.reserve(sizeof(uint2) * RUN_CHUNK * cap) || H.pool_next.reserve(sizeof(int) * cap)) {
        cudaGetLastError();
        H.pool_runs.release();
        H.pool_next.release();
        cap = H.pool_cap;   // fall back to the old size
        if (H.pool_runs.reserve(sizeof(uint2) * RUN_CHUNK * cap) || H.pool_next.reserve(sizeof(int) * cap)) {
            cudaGetLastError();
            H.pool_cap = 0;
        }
        return false;
    }
    H.pool_cap = cap;
    return true;
}

// FP32-compensated points in two phases: the walk kernels write every (query, subtree) item's
// accepted runs, the pair kernel evaluates them (once per catalog launch).  Queries go through
// in slices of H.slice (Morton order when sorted), which bounds the item and pool memory.
// Queries that found the pool full are walked again in another round with an emptied pool;
// if a round completes fewer than 1/8 of its queries, the fused walk-and-sum kernel takes the
// rest.  Both kernels produce identical bits for a query.
//
// Schedule modes (H.sched), all with identical results:
//   0 plain:   queries in input order, one walk item per query, pairs in walk order;
//   1 tuned:   Morton order, walk split into ~walk_split subtrees, pairs heaviest first;
//   2 learned: as tuned, with the walk order binned by the MLP's predicted work
//              (heaviest class first, Morton order inside a class).
int two_phase_points(Handle &H, const DevTree &T, const std::vector<Launch> &launches,
                     const std::vector<Launch> &launches64, std::vector<double *> &dev, int strategy, int64_t npts,
                     const double *dx, const double *dy, const double *dz, const uint32_t *perm)
{
    if (npts > 0x7fffffffLL) return fail(H, PB_ERR_CAPACITY, "more than 2^31-1 sample points in one call");
    const int mode = H.sched;
    if (mode == 2 && !H.mlp_ready) return fail(H, PB_ERR_STATE, "learned schedule requested but no scheduler weights set");
    int ns = 1;
    CK(launch_cut(&H, T, mode == 0 ? 1 : H.walk_split, &ns));
    // a slice holds at most 2^31 - 1 (query, subtree) items: the work-list offsets are 32-bit
    const int64_t S_items = std::max<int64_t>(1024, (int64_t)0x7fffffff / std::max(ns, 1));
    const int64_t S = std::min<int64_t>(std::min<int64_t>(H.slice > 0 ? H.slice : npts, npts), S_items);
    int rc = reserve_pool(H, S, ns);
    if (rc) return rc;
    const uint32_t *ql_all = mode == 0 ? nullptr : perm;
    if (!ql_all) {
        CK(H.iota.reserve(sizeof(uint32_t) * npts));
        CK(launch_iota(&H, npts, H.iota.as<uint32_t>()));
        ql_all = H.iota.as<uint32_t>();
    }
    if (mode == 2) {
        CK(H.sched_feat.reserve(sizeof(float) * SCHED_F * S));
        CK(H.sched_pred.reserve(sizeof(float) * S));
        CK(H.sched_ql.reserve(sizeof(uint32_t) * S));
        CK(H.sched_tmp.reserve(sizeof(uint32_t) * S));
        CK(H.lpt_k.reserve(4 * S));
        CK(H.lpt_v.reserve(4 * S));
        CK(H.lpt_ka.reserve(4 * S));
        CK(H.lpt_va.reserve(4 * S));
    }
    uint32_t *lists[2] = {H.defer_a.as<uint32_t>(), H.defer_b.as<uint32_t>()};
    unsigned long long *ctr = H.pool_ctr.as<unsigned long long>();
    H.walk_rounds = 0;
    H.deferred_total = 0;
    for (int k = 0; k < 3; ++k) H.t_phase_ms[k] = 0.f;
    // slice size, adapted to the pool use seen so far; the first slice is sized from the largest
    // per-query pool use of the handle's previous call, when there was one
    int64_t Snext = S;
    if (H.pool_cpq > 0.0)
        Snext = std::max<int64_t>(1024, std::min<int64_t>(S, (int64_t)(0.85 * (double)H.pool_cap / H.pool_cpq)));
    double cpq_max = 0.0;
    for (int64_t s0 = 0; s0 < npts;) {
        const uint32_t *ql = ql_all + s0;
        int64_t m = std::min<int64_t>(Snext, npts - s0);
        s0 += m;
        for (int round = 0;; ++round) {
            CK(cudaMemsetAsync(ctr, 0, 16, H.stream));
            CK(cudaMemsetAsync(ctr + 4, 0, 16, H.stream));
            CK(cudaMemsetAsync(H.qacc.p, 0, sizeof(unsigned) * m, H.stream));
            CK(cudaMemsetAsync(H.qflag.p, 0, sizeof(int) * m, H.stream));
            RunPool P;
            P.runs = H.pool_runs.as<uint2>();
            P.next = H.pool_next.as<int>();
            P.used = ctr;
            P.cap = H.pool_cap;
            P.ns = ns;
            P.cut = H.cut.as<int2>() + (4 * (mode == 0 ? 1 : H.walk_split) + 8);
            P.items = H.items.as<int2>();
            P.bnear = H.wbnear.as<int>();
            P.qacc = H.qacc.as<unsigned>();
            P.qflag = H.qflag.as<int>();
            P.n_deferred = reinterpret_cast<unsigned *>(ctr + 1);
            P.deferred = lists[round & 1];
            P.count_only = 0;
            P.leaf_size = H.leaf_size;
            ev_record(H, 4);
            if (strategy != SCATTER || mode == 2) {
                CK(launch_nearest_list(&H, T, m, ql, dx, dy, dz, P.bnear));
                H.interp_launches++;
            }
            if (mode == 2) {
                // predicted work -> class-major walk order (Morton order kept inside a class)
                float *feat = H.sched_feat.as<float>(), *pred = H.sched_pred.as<float>();
                uint32_t *order = H.lpt_v.as<uint32_t>();
                CK(launch_sched_features(&H, T, m, ql, dx, dy, dz, P.bnear, feat));
                CK(launch_mlp_predict(&H, m, feat, pred));
                CK(launch_sched_order(&H, m, pred, H.sched_width, H.sched_nclass, order));
                uint32_t *qn = H.sched_ql.as<uint32_t>();
                CK(launch_gather_u32(&H, m, order, ql, qn));
                int *bt = reinterpret_cast<int *>(H.sched_tmp.as<uint32_t>());
                CK(launch_gather_i32(&H, m, order, P.bnear, bt));
                CK(cudaMemcpyAsync(P.bnear, bt, sizeof(int) * m, cudaMemcpyDeviceToDevice, H.stream));
                ql = qn;
                H.interp_launches += 4;
            }
            ev_record(H, 5);
            if (mode == 0 || ns == 1) CK(launch_walk(&H, T, strategy, P, m, ql, dx, dy, dz, ctr + 2));
            else CK(launch_walk_list(&H, T, strategy, P, m, ql, dx, dy, dz, ctr + 2));
            H.interp_launches++;
            uint32_t *order = nullptr;
            int64_t m_heavy = 0;
            CK(launch_split_order(&H, P, m, (unsigned)H.light_max, mode == 0, &order, &m_heavy, ctr + 4));
            ev_record(H, 6);
            if (m_heavy > 0)
                for (const Launch &Lc : launches) {
                    DevCatalog C = dev_catalog(H, Lc, dev.data());
                    CK(launch_pairs_fp32(&H, T, C, strategy, P, m_heavy, ql, order, dx, dy, dz));
                    H.interp_launches++;
                }
            if (m_heavy < m)
                for (const Launch &Lc : launches64) {   // light queries: FP64, the reference's arithmetic
                    DevCatalog C = dev_catalog(H, Lc, dev.data());
                    CK(launch_pairs_fp64(&H, T, C, strategy, P, m - m_heavy, ql, order + m_heavy, dx, dy, dz));
                    H.interp_launches++;
                }
            ev_record(H, 7);
            unsigned long long used_nd[6] = {0, 0, 0, 0, 0, 0};
            CK(cudaMemcpyAsync(used_nd, ctr, 6 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, H.stream));
            CK(cudaStreamSynchronize(H.stream));
            const unsigned nd = (unsigned)(used_nd[1] & 0xffffffffULL);
            H.split_hq += m_heavy;
            H.split_lq += m - (int64_t)nd - m_heavy;
            H.split_hp += (int64_t)used_nd[4];
            H.split_lp += (int64_t)used_nd[5];
            if (round == 0) {
                // next slice: the queries that 85 % of the pool holds at this slice's chunks per query
                const unsigned long long used = std::min<unsigned long long>(used_nd[0], H.pool_cap);
                const int64_t done = m - (int64_t)nd;
                if (done > 0 && used > 0) {
                    const double per = (double)used / (double)done;
                    cpq_max = std::max(cpq_max, per);
                    Snext = std::max<int64_t>(1024, std::min<int64_t>(S, (int64_t)(0.85 * (double)H.pool_cap / per)));
                } else if (nd > 0) {
                    Snext = std::max<int64_t>(1024, Snext / 2);
                }
            }
            for (int k = 0; k < 3; ++k) H.t_phase_ms[k] += ev_ms(H, 4 + k, 5 + k);   // every slice and round
            H.walk_rounds = std::max<int64_t>(H.walk_rounds, round + 1);
            if (nd == 0) break;
            H.deferred_total += nd;
            const bool grew = grow_pool(H);
            if (grew) {
                // the bigger pool holds proportionally more of a slice
                Snext = std::min<int64_t>(S, Snext * 2);
            } else if (H.pool_cap == 0) {
                return fail(H, PB_ERR_CUDA, "run pool could not be reallocated");
            }
            if (!grew && (int64_t)nd > m - m / 8) {   // under 1/8 completed, pool at its limit: finish fused
                int rc2 = fused_fallback(H, T, launches, launches64, dev, strategy, npts, dx, dy, dz, P, nd);
                if (rc2) return rc2;
                break;
            }
            // the deferred list is walked next; in learned mode it is binned again
            if (mode == 2) {
                CK(cudaMemcpyAsync(H.sched_tmp.p, P.deferred, sizeof(uint32_t) * nd, cudaMemcpyDeviceToDevice,
                                   H.stream));
                ql = H.sched_tmp.as<uint32_t>();
            } else {
                ql = P.deferred;
            }
            m = nd;
        }
    }
    if (cpq_max > 0.0) H.pool_cpq = cpq_max;
    return PB_OK;
}

int do_points(Handle &H, const pb_catalog *cat, int64_t npts, const double *qx, const double *qy,
              const double *qz, int32_t strategy, int32_t precision, double *const *out)
{
    if (!H.built) return fail(H, PB_ERR_STATE, "no LBVH has been built on this handle");
    if (strategy < 0 || strategy > 2) return fail(H, PB_ERR_INVALID, "unknown interpolation strategy");
    if (precision != PB_FP64 && precision != PB_FP32C) return fail(H, PB_ERR_INVALID, "unknown precision mode");
    int rc = validate_catalog(H, cat, false);
    if (rc) return rc;
    if (npts < 0) return fail(H, PB_ERR_INVALID, "negative number of sample points");
    H.interp_launches = 0;
    H.t_interp_ms = 0.f;
    H.split_hq = H.split_lq = H.split_hp = H.split_lp = 0;
    int64_t L = catalog_L(cat);
    if (npts == 0 || L == 0) return PB_OK;
    if (!qx || !qy || !qz) return fail(H, PB_ERR_INVALID, "sample coordinate pointer is NULL");
    CK(cudaSetDevice(H.device));
    CK(cudaMemsetAsync(H.status.p, 0, sizeof(int), H.stream));
    const double *dx, *dy, *dz;
    if ((rc = stage_queries(H, npts, qx, qy, qz, &dx, &dy, &dz))) return rc;
    std::vector<double *> dev;
    std::vector<int> is_host;
    if ((rc = stage_outputs(H, L, npts, out, dev, is_host))) return rc;
    DevTree T = make_tree(H);
    std::vector<Launch> launches = plan(items_of(cat, precision == PB_FP32C));
    std::vector<Launch> launches64 = plan(items_of(cat, false));
    ev_record(H, 2);   // the query ordering is part of the timed interpolation
    const uint32_t *perm;
    if ((rc = query_order(H, npts, dx, dy, dz, &perm))) return rc;
    if (precision == PB_FP64) {
        // every query summed by the FP64 pair kernel (the fused kernel's arithmetic, bit for bit)
        const int64_t keep = H.light_max;
        H.light_max = 0x7fffffffLL;
        rc = two_phase_points(H, T, launches64, launches64, dev, strategy, npts, dx, dy, dz, perm);
        H.light_max = keep;
        if (rc) return rc;
    } else if ((rc = two_phase_points(H, T, launches, launches64, dev, strategy, npts, dx, dy, dz, perm))) {
        return rc;
    }
    ev_record(H, 3);
    if ((rc = finish_outputs(H, L, npts, out, dev, is_host))) return rc;
    H.t_interp_ms = ev_ms(H, 2, 3);
    return PB_OK;
}

int do_lines(Handle &H, const pb_catalog *cat, int64_t nl, const double *ox, const double *oy, const double *oz,
             const double *mx, const double *my, const double *mz, int32_t strategy, int32_t precision,
             double *const *out)
{
    if (!H.built) return fail(H, PB_ERR_STATE, "no LBVH has been built on this handle");
    if (strategy != SCATTER)
        return fail(H, PB_ERR_INVALID,
                    "LineSamples_interpolation only supports itpScatter (ArgumentError in the reference)");
    if (precision != PB_FP64 && precision != PB_FP32C) return fail(H, PB_ERR_INVALID, "unknown precision mode");
    int rc = validate_catalog(H, cat, true);
    if (rc) return rc;
    if (nl < 0) return fail(H, PB_ERR_INVALID, "negative number of lines");
    H.interp_launches = 0;
    H.t_interp_ms = 0.f;
    int64_t L = cat->n_scalar;
    if (nl == 0 || L == 0) return PB_OK;
    if (!ox || !oy || !oz || !mx || !my || !mz) return fail(H, PB_ERR_INVALID, "line pointer is NULL");
    CK(cudaSetDevice(H.device));
    CK(cudaMemsetAsync(H.status.p, 0, sizeof(int), H.stream));
    const double *dox, *doy, *doz;
    if ((rc = stage_queries(H, nl, ox, oy, oz, &dox, &doy, &doz))) return rc;
    const void *a, *b, *c;
    CK(H.q_out.reserve(sizeof(double) * 3 * nl));
    // directions: device views or staged into q_out (3 * nl doubles)
    double *stage = H.q_out.as<double>();
    const double *dirs[3] = {mx, my, mz};
    const void *dv[3];
    for (int d = 0; d < 3; ++d) {
        if (ptr_place(H, dirs[d]) == 2) return fail(H, PB_ERR_INVALID, "direction is device memory of another GPU");
        if (is_device_ptr(H, dirs[d])) dv[d] = dirs[d];
        else {
            CK(cudaMemcpyAsync(stage + d * nl, dirs[d], sizeof(double) * nl, cudaMemcpyHostToDevice, H.stream));
            dv[d] = stage + d * nl;
        }
    }
    a = dv[0]; b = dv[1]; c = dv[2];
    std::vector<double *> dev;
    std::vector<int> is_host;
    if ((rc = stage_outputs(H, L, nl, out, dev, is_host))) return rc;
    DevTree T = make_tree(H);
    // Both precision modes take the FP64 line kernel.  An FP32-compensated line sum needs its
    // projected distances and table indices in FP64 too (FP32 ones miss the 1e-5 tolerance on
    // 256^2 images), so only its accumulation would be cheaper, and that did not pay: the whole
    // C3 image took 433 ms with FP32C accumulation against 388 ms in FP64.
    std::vector<Launch> launches = plan(items_of(cat, false));
    ev_record(H, 2);   // the line ordering is part of the timed interpolation
    const uint32_t *perm;
    if ((rc = query_order(H, nl, dox, doy, doz, &perm))) return rc;
    for (const Launch &Lc : launches) {
        DevCatalog C = dev_catalog(H, Lc, dev.data());
        CK(launch_lines_fp64(&H, T, C, nl, dox, doy, doz, (const double *)a, (const double *)b, (const double *)c, perm));
        H.interp_launches++;
    }
    ev_record(H, 3);
    if ((rc = finish_outputs(H, L, nl, out, dev, is_host))) return rc;
    H.t_interp_ms = ev_ms(H, 2, 3);
    return PB_OK;
}

}  // namespace

// =========================================================================================
extern "C" {

int32_t pb_create(pb_handle **out, int32_t device)
{
    if (!out) return PB_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return PB_ERR_CUDA;
    }
    if (device < 0 || device >= ndev) return PB_ERR_INVALID;
    pb_handle *p = new pb_handle();
    p->H.device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&p->H.own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete p;
        return PB_ERR_CUDA;
    }
    p->H.stream = p->H.own_stream;
    *out = p;
    return PB_OK;
}

void pb_destroy(pb_handle *h)
{
    if (!h) return;
    cudaSetDevice(h->H.device);
    if (h->H.stream) cudaStreamSynchronize(h->H.stream);
    delete h;
}

int32_t pb_last_error(const pb_handle *h, char *buf, int64_t size)
{
    if (!h) return 0;
    const std::string &e = h->H.err;
    if (buf && size > 0) {
        int64_t k = std::min<int64_t>(size - 1, (int64_t)e.size());
        memcpy(buf, e.data(), k);
        buf[k] = 0;
    }
    return (int32_t)e.size();
}

int32_t pb_set_stream(pb_handle *h, void *s)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    H.stream = s ? (cudaStream_t)s : H.own_stream;
    return PB_OK;
}

int32_t pb_set_option(pb_handle *h, const char *name, int64_t value)
{
    if (!h || !name) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (!strcmp(name, "timing")) H.timing = value != 0;
    else if (!strcmp(name, "sort_queries")) H.sort_queries = (int)value;
    else if (!strcmp(name, "block_size")) H.block_size = (int)value;
    else if (!strcmp(name, "schedule")) {
        if (value < 0 || value > 2) return fail(H, PB_ERR_INVALID, "schedule must be 0 (plain), 1 (tuned) or 2 (learned)");
        H.sched = (int)value;
    } else if (!strcmp(name, "fp64_light_max")) {
        if (value < 0 || value > 0x7fffffffLL) return fail(H, PB_ERR_INVALID, "fp64_light_max out of range");
        H.light_max = value;
    } else if (!strcmp(name, "slice_queries")) {
        if (value < 1024) return fail(H, PB_ERR_INVALID, "slice_queries must be >= 1024");
        H.slice = value;
    } else if (!strcmp(name, "leaf_size")) {
        if (value < 1 || value > 64) return fail(H, PB_ERR_INVALID, "leaf_size must be in 1..64");
        H.leaf_size = (int)value;
    } else if (!strcmp(name, "batch_order")) {
        if (value < 0 || value > 1) return fail(H, PB_ERR_INVALID, "batch_order must be 0 (given) or 1 (most work first)");
        H.batch_order = (int)value;
    } else if (!strcmp(name, "batch_blocks_per_sm")) {
        if (value < 0 || value > 32) return fail(H, PB_ERR_INVALID, "batch_blocks_per_sm must be in 0..32");
        H.batch_blocks = (int)value;
    } else if (!strcmp(name, "batch_walk_split")) {
        if (value < 1 || value > 1024) return fail(H, PB_ERR_INVALID, "batch_walk_split must be in 1..1024");
        H.batch_walk_split = (int)value;
    } else if (!strcmp(name, "walk_split")) {
        if (value < 1 || value > 4096) return fail(H, PB_ERR_INVALID, "walk_split must be in 1..4096");
        H.walk_split = (int)value;
    }
    else return fail(H, PB_ERR_INVALID, std::string("unknown option ") + name);
    return PB_OK;
}

int32_t pb_linear_bvh(pb_handle *h, const pb_input *in, int32_t flags)
{
    if (!h) return PB_ERR_INVALID;
    return do_build(h->H, in, flags);
}

int32_t pb_export_encoding(pb_handle *h, uint64_t *codes, int64_t *order)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (!H.built) return fail(H, PB_ERR_STATE, "no LBVH has been built on this handle");
    CK(cudaSetDevice(H.device));
    int64_t n = H.n;
    if (codes) CK(cudaMemcpyAsync(codes, H.codes.p, 8 * n, cudaMemcpyDefault, H.stream));
    if (order) {
        std::vector<uint32_t> tmp(n);
        CK(cudaMemcpyAsync(tmp.data(), H.idx.p, 4 * n, cudaMemcpyDeviceToHost, H.stream));
        CK(cudaStreamSynchronize(H.stream));
        std::vector<int64_t> w(tmp.begin(), tmp.end());
        CK(cudaMemcpy(order, w.data(), 8 * n, cudaMemcpyDefault));
    }
    CK(cudaStreamSynchronize(H.stream));
    return PB_OK;
}

int32_t pb_export_tree(pb_handle *h, int32_t *left, int32_t *right, int32_t *escape, int32_t *parent, double *bmin,
                       double *bmax, double *hmax, int32_t *root)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (!H.built) return fail(H, PB_ERR_STATE, "no LBVH has been built on this handle");
    CK(cudaSetDevice(H.device));
    int64_t n = H.n, nin = n - 1, ntot = 2 * n - 1;
    if (root) *root = n >= 2 ? 1 : 0;
    std::vector<int32_t> z(ntot, 0);
    if (left) {
        CK(cudaMemcpy(left, z.data(), 4 * ntot, cudaMemcpyDefault));
        if (nin > 0) CK(cudaMemcpyAsync(left, H.left.p, 4 * nin, cudaMemcpyDefault, H.stream));
    }
    if (right) {
        CK(cudaMemcpy(right, z.data(), 4 * ntot, cudaMemcpyDefault));
        if (nin > 0) CK(cudaMemcpyAsync(right, H.right.p, 4 * nin, cudaMemcpyDefault, H.stream));
    }
    if (escape) CK(cudaMemcpyAsync(escape, H.escape.p, 4 * ntot, cudaMemcpyDefault, H.stream));
    if (parent) CK(cudaMemcpyAsync(parent, H.parent.p, 4 * ntot, cudaMemcpyDefault, H.stream));
    if (nin > 0) {
        if (bmin) CK(cudaMemcpyAsync(bmin, H.bmin64.p, 24 * nin, cudaMemcpyDefault, H.stream));
        if (bmax) CK(cudaMemcpyAsync(bmax, H.bmax64.p, 24 * nin, cudaMemcpyDefault, H.stream));
        if (hmax) CK(cudaMemcpyAsync(hmax, H.hmax64.p, 8 * nin, cudaMemcpyDefault, H.stream));
    }
    CK(cudaStreamSynchronize(H.stream));
    return PB_OK;
}

int32_t pb_find_nearest_h(pb_handle *h, int64_t npts, const double *qx, const double *qy, const double *qz,
                          double *h_out, int64_t *idx_out)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (!H.built) return fail(H, PB_ERR_STATE, "no LBVH has been built on this handle");
    if (npts <= 0) return npts == 0 ? PB_OK : fail(H, PB_ERR_INVALID, "negative npts");
    CK(cudaSetDevice(H.device));
    CK(cudaMemsetAsync(H.status.p, 0, sizeof(int), H.stream));
    const double *dx, *dy, *dz;
    int rc = stage_queries(H, npts, qx, qy, qz, &dx, &dy, &dz);
    if (rc) return rc;
    CK(H.q_out.reserve(16 * npts));
    double *hd = H.q_out.as<double>();
    int64_t *id = reinterpret_cast<int64_t *>(hd + npts);
    CK(launch_nearest(&H, make_tree(H), npts, dx, dy, dz, hd, id));
    if (h_out) CK(cudaMemcpyAsync(h_out, hd, 8 * npts, cudaMemcpyDefault, H.stream));
    if (idx_out) CK(cudaMemcpyAsync(idx_out, id, 8 * npts, cudaMemcpyDefault, H.stream));
    return check_status(H);
}

int32_t pb_query_count(pb_handle *h, int64_t npts, const double *qx, const double *qy, const double *qz,
                       const double *radius, int64_t *counts)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (!H.built) return fail(H, PB_ERR_STATE, "no LBVH has been built on this handle");
    if (npts <= 0) return npts == 0 ? PB_OK : fail(H, PB_ERR_INVALID, "negative npts");
    if (!radius || !counts) return fail(H, PB_ERR_INVALID, "NULL radius/counts");
    CK(cudaSetDevice(H.device));
    CK(cudaMemsetAsync(H.status.p, 0, sizeof(int), H.stream));
    const double *dx, *dy, *dz;
    int rc = stage_queries(H, npts, qx, qy, qz, &dx, &dy, &dz);
    if (rc) return rc;
    const void *r;
    CK(stage_in(H, H.q_aux, radius, 8 * npts, &r));
    CK(H.q_out.reserve(8 * npts));
    CK(launch_query(&H, make_tree(H), npts, dx, dy, dz, (const double *)r, nullptr, H.q_out.as<int64_t>(), nullptr,
                    nullptr, nullptr));
    CK(cudaMemcpyAsync(counts, H.q_out.p, 8 * npts, cudaMemcpyDefault, H.stream));
    return check_status(H);
}

int32_t pb_query_neighbors(pb_handle *h, int64_t npts, const double *qx, const double *qy, const double *qz,
                           const double *radius, const int64_t *offsets, int64_t *pool, int64_t *nearest)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (!H.built) return fail(H, PB_ERR_STATE, "no LBVH has been built on this handle");
    if (npts <= 0) return npts == 0 ? PB_OK : fail(H, PB_ERR_INVALID, "negative npts");
    if (!radius || !offsets || !pool) return fail(H, PB_ERR_INVALID, "NULL radius/offsets/pool");
    CK(cudaSetDevice(H.device));
    CK(cudaMemsetAsync(H.status.p, 0, sizeof(int), H.stream));
    const double *dx, *dy, *dz;
    int rc = stage_queries(H, npts, qx, qy, qz, &dx, &dy, &dz);
    if (rc) return rc;
    const void *r, *o;
    CK(stage_in(H, H.q_aux, radius, 8 * npts, &r));
    CK(stage_in(H, H.q_keys, offsets, 8 * (npts + 1), &o));
    int64_t total = 0;
    CK(cudaStreamSynchronize(H.stream));
    CK(cudaMemcpy(&total, (const int64_t *)o + npts, 8, cudaMemcpyDefault));
    if (total < 0) return fail(H, PB_ERR_INVALID, "negative pool size");
    bool pool_dev = is_device_ptr(H, pool);
    int64_t *dpool = pool;
    if (!pool_dev) {
        CK(H.q_perm_alt.reserve(8 * (total + 1)));
        dpool = H.q_perm_alt.as<int64_t>();
    }
    CK(H.q_out.reserve(8 * npts));
    CK(launch_query(&H, make_tree(H), npts, dx, dy, dz, (const double *)r, (const int64_t *)o, nullptr, dpool,
                    H.q_out.as<int64_t>(), nullptr));
    if (!pool_dev && total > 0) CK(cudaMemcpyAsync(pool, dpool, 8 * total, cudaMemcpyDeviceToHost, H.stream));
    if (nearest) CK(cudaMemcpyAsync(nearest, H.q_out.p, 8 * npts, cudaMemcpyDefault, H.stream));
    return check_status(H);
}

int32_t pb_probe_neighbors(pb_handle *h, int64_t npts, const double *qx, const double *qy, const double *qz,
                           const double *radius, int64_t *count, int64_t *closest_idx, double *closest_d2)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (!H.built) return fail(H, PB_ERR_STATE, "no LBVH has been built on this handle");
    if (npts <= 0) return npts == 0 ? PB_OK : fail(H, PB_ERR_INVALID, "negative npts");
    if (!radius) return fail(H, PB_ERR_INVALID, "NULL radius");
    CK(cudaSetDevice(H.device));
    CK(cudaMemsetAsync(H.status.p, 0, sizeof(int), H.stream));
    const double *dx, *dy, *dz;
    int rc = stage_queries(H, npts, qx, qy, qz, &dx, &dy, &dz);
    if (rc) return rc;
    const void *r;
    CK(stage_in(H, H.q_aux, radius, 8 * npts, &r));
    CK(H.q_out.reserve(24 * npts));
    int64_t *dc = H.q_out.as<int64_t>(), *di = dc + npts;
    double *dd = reinterpret_cast<double *>(di + npts);
    CK(launch_query(&H, make_tree(H), npts, dx, dy, dz, (const double *)r, nullptr, dc, nullptr, di, dd));
    if (count) CK(cudaMemcpyAsync(count, dc, 8 * npts, cudaMemcpyDefault, H.stream));
    if (closest_idx) CK(cudaMemcpyAsync(closest_idx, di, 8 * npts, cudaMemcpyDefault, H.stream));
    if (closest_d2) CK(cudaMemcpyAsync(closest_d2, dd, 8 * npts, cudaMemcpyDefault, H.stream));
    return check_status(H);
}

int32_t pb_traversal_stats(pb_handle *h, int64_t npts, const double *qx, const double *qy, const double *qz,
                           int32_t strategy, int64_t *stats)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (!H.built) return fail(H, PB_ERR_STATE, "no LBVH has been built on this handle");
    if (strategy < 0 || strategy > 2) return fail(H, PB_ERR_INVALID, "unknown interpolation strategy");
    if (npts <= 0) return npts == 0 ? PB_OK : fail(H, PB_ERR_INVALID, "negative npts");
    if (!stats) return fail(H, PB_ERR_INVALID, "NULL stats");
    CK(cudaSetDevice(H.device));
    CK(cudaMemsetAsync(H.status.p, 0, sizeof(int), H.stream));
    const double *dx, *dy, *dz;
    int rc = stage_queries(H, npts, qx, qy, qz, &dx, &dy, &dz);
    if (rc) return rc;
    int64_t *ds = stats;
    bool dev = is_device_ptr(H, stats);
    if (!dev) {
        CK(H.q_aux.reserve(40 * npts));
        ds = H.q_aux.as<int64_t>();
    }
    CK(launch_stats(&H, make_tree(H), strategy, npts, dx, dy, dz, ds));
    if (!dev) CK(cudaMemcpyAsync(stats, ds, 40 * npts, cudaMemcpyDeviceToHost, H.stream));
    return check_status(H);
}

int32_t pb_interpolate_points(pb_handle *h, const pb_catalog *cat, int64_t npts, const double *qx, const double *qy,
                              const double *qz, int32_t strategy, int32_t precision, double *const *out)
{
    if (!h) return PB_ERR_INVALID;
    return do_points(h->H, cat, npts, qx, qy, qz, strategy, precision, out);
}

int32_t pb_interpolate_lines(pb_handle *h, const pb_catalog *cat, int64_t nlines, const double *ox, const double *oy,
                             const double *oz, const double *dx, const double *dy, const double *dz, int32_t strategy,
                             int32_t precision, double *const *out)
{
    if (!h) return PB_ERR_INVALID;
    return do_lines(h->H, cat, nlines, ox, oy, oz, dx, dy, dz, strategy, precision, out);
}

int32_t pb_point_samples_interpolation(pb_handle *h, const pb_input *in, const pb_catalog *cat, int64_t npts,
                                       const double *qx, const double *qy, const double *qz, int32_t strategy,
                                       int32_t precision, double *const *out, int32_t flags)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (strategy < 0 || strategy > 2) return fail(H, PB_ERR_INVALID, "unknown interpolation strategy");
    int rc = do_build(H, in, flags);
    if (rc) return rc;
    return do_points(H, cat, npts, qx, qy, qz, strategy, precision, out);
}

int32_t pb_line_samples_interpolation(pb_handle *h, const pb_input *in, const pb_catalog *cat, int64_t nlines,
                                      const double *ox, const double *oy, const double *oz, const double *dx,
                                      const double *dy, const double *dz, int32_t strategy, int32_t precision,
                                      double *const *out, int32_t flags)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (strategy != SCATTER)
        return fail(H, PB_ERR_INVALID,
                    "LineSamples_interpolation only supports itpScatter (ArgumentError in the reference)");
    int rc = do_build(H, in, flags);
    if (rc) return rc;
    return do_lines(H, cat, nlines, ox, oy, oz, dx, dy, dz, strategy, precision, out);
}

int64_t pb_launch_count(const pb_handle *h) { return h ? h->H.launches : 0; }

int32_t pb_grid_points(pb_handle *h, int32_t coord, const double *a0, int64_t n0, const double *a1, int64_t n1,
                       const double *a2, int64_t n2, double *x, double *y, double *z)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (coord != 0 && coord != 2 && coord != 3)
        return fail(H, PB_ERR_INVALID, "coordinate system must be 0 (Cartesian), 2 (cylindrical) or 3 (spherical)");
    if (!a0 || !a1 || !a2 || !x || !y || !z || n0 < 1 || n1 < 1 || n2 < 1)
        return fail(H, PB_ERR_INVALID, "grid axes / outputs: bad arguments");
    const int64_t n = n0 * n1 * n2;
    CK(cudaSetDevice(H.device));
    CK(H.grid_ax.reserve(sizeof(double) * (n0 + n1 + n2)));
    double *ax = H.grid_ax.as<double>();
    CK(cudaMemcpyAsync(ax, a0, sizeof(double) * n0, cudaMemcpyDefault, H.stream));
    CK(cudaMemcpyAsync(ax + n0, a1, sizeof(double) * n1, cudaMemcpyDefault, H.stream));
    CK(cudaMemcpyAsync(ax + n0 + n1, a2, sizeof(double) * n2, cudaMemcpyDefault, H.stream));
    double *outs[3] = {x, y, z};
    double *dst[3];
    const bool dev = is_device_ptr(H, x) && is_device_ptr(H, y) && is_device_ptr(H, z);
    if (!dev) {
        CK(H.grid_out.reserve(sizeof(double) * 3 * n));
        for (int d = 0; d < 3; ++d) dst[d] = H.grid_out.as<double>() + d * n;
    } else {
        for (int d = 0; d < 3; ++d) dst[d] = outs[d];
    }
    CK(launch_grid_points(&H, coord, ax, n0, ax + n0, n1, ax + n0 + n1, n2, dst[0], dst[1], dst[2]));
    if (!dev)
        for (int d = 0; d < 3; ++d)
            CK(cudaMemcpyAsync(outs[d], dst[d], sizeof(double) * n, cudaMemcpyDeviceToHost, H.stream));
    CK(cudaStreamSynchronize(H.stream));
    return PB_OK;
}

int32_t pb_line_image(pb_handle *h, const double *a0, int64_t n0, const double *a1, int64_t n1, const double *frame,
                      double *ox, double *oy, double *oz, double *dx, double *dy, double *dz)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (!a0 || !a1 || !frame || !ox || !oy || !oz || !dx || !dy || !dz || n0 < 1 || n1 < 1)
        return fail(H, PB_ERR_INVALID, "line image axes / outputs: bad arguments");
    LineFrame F;
    for (int d = 0; d < 3; ++d) {
        F.c[d] = frame[d];
        F.e1[d] = frame[3 + d];
        F.e2[d] = frame[6 + d];
        F.d[d] = frame[9 + d];
    }
    for (int k = 0; k < 12; ++k)
        if (!std::isfinite(frame[k])) return fail(H, PB_ERR_INVALID, "line image frame is not finite");
    const double dn = std::sqrt(F.d[0] * F.d[0] + F.d[1] * F.d[1] + F.d[2] * F.d[2]);
    if (std::fabs(dn - 1.0) > 1e-12) return fail(H, PB_ERR_INVALID, "line direction must be a unit vector");
    const int64_t n = n0 * n1;
    CK(cudaSetDevice(H.device));
    CK(H.grid_ax.reserve(sizeof(double) * (n0 + n1)));
    double *ax = H.grid_ax.as<double>();
    CK(cudaMemcpyAsync(ax, a0, sizeof(double) * n0, cudaMemcpyDefault, H.stream));
    CK(cudaMemcpyAsync(ax + n0, a1, sizeof(double) * n1, cudaMemcpyDefault, H.stream));
    double *outs[6] = {ox, oy, oz, dx, dy, dz};
    double *dst[6];
    bool dev = true;
    for (int k = 0; k < 6; ++k) {
        if (ptr_place(H, outs[k]) == 2) return fail(H, PB_ERR_INVALID, "output is device memory of another GPU");
        dev = dev && is_device_ptr(H, outs[k]);
    }
    if (!dev) {
        CK(H.grid_out.reserve(sizeof(double) * 6 * n));
        for (int k = 0; k < 6; ++k) dst[k] = H.grid_out.as<double>() + k * n;
    } else {
        for (int k = 0; k < 6; ++k) dst[k] = outs[k];
    }
    CK(launch_line_image(&H, ax, n0, ax + n0, n1, F, dst[0], dst[1], dst[2], dst[3], dst[4], dst[5]));
    if (!dev)
        for (int k = 0; k < 6; ++k)
            CK(cudaMemcpyAsync(outs[k], dst[k], sizeof(double) * n, cudaMemcpyDeviceToHost, H.stream));
    CK(cudaStreamSynchronize(H.stream));
    return PB_OK;
}

// ---- learned work prediction ----
namespace {
// device view of a float array given as host or device memory (staged into `buf`)
int stage_f32(Handle &H, DBuf &buf, const float *src, int64_t n, const float **out)
{
    if (is_device_ptr(H, src)) {
        *out = src;
        return PB_OK;
    }
    CK(buf.reserve(sizeof(float) * (n > 0 ? n : 1)));
    CK(cudaMemcpyAsync(buf.p, src, sizeof(float) * n, cudaMemcpyHostToDevice, H.stream));
    *out = buf.as<float>();
    return PB_OK;
}

int copy_out_f32(Handle &H, float *dst, const float *src, int64_t n)
{
    CK(cudaMemcpyAsync(dst, src, sizeof(float) * n, cudaMemcpyDefault, H.stream));
    CK(cudaStreamSynchronize(H.stream));
    return PB_OK;
}

int mlp_reserve(Handle &H)
{
    CK(H.mlp_w.reserve(sizeof(float) * SCHED_NPARAM));
    CK(H.mlp_m.reserve(sizeof(float) * SCHED_NPARAM));
    CK(H.mlp_v.reserve(sizeof(float) * SCHED_NPARAM));
    CK(H.mlp_g.reserve(sizeof(float) * SCHED_NPARAM));
    CK(H.mlp_norm.reserve(sizeof(float) * 2 * SCHED_F));
    return PB_OK;
}
}  // namespace

int32_t pb_scheduler_features(pb_handle *h, int64_t npts, const double *qx, const double *qy, const double *qz,
                              float *feat)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (!H.built) return fail(H, PB_ERR_STATE, "no LBVH has been built on this handle");
    if (npts < 0 || !feat) return fail(H, PB_ERR_INVALID, "bad arguments");
    if (npts == 0) return PB_OK;
    CK(cudaSetDevice(H.device));
    const double *dx, *dy, *dz;
    int rc = stage_queries(H, npts, qx, qy, qz, &dx, &dy, &dz);
    if (rc) return rc;
    float *out = feat;
    if (!is_device_ptr(H, feat)) {
        CK(H.sched_feat.reserve(sizeof(float) * SCHED_F * npts));
        out = H.sched_feat.as<float>();
    }
    DevTree T = make_tree(H);
    CK(launch_sched_features(&H, T, npts, nullptr, dx, dy, dz, nullptr, out));
    if (out != feat) return copy_out_f32(H, feat, out, SCHED_F * npts);
    CK(cudaStreamSynchronize(H.stream));
    return PB_OK;
}

int32_t pb_scheduler_set(pb_handle *h, const float *params, const float *norm, float bin_width, int32_t nclass)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (!params || !norm || !(bin_width > 0.f) || nclass < 1 || nclass > 1024)
        return fail(H, PB_ERR_INVALID, "scheduler weights: bad arguments");
    CK(cudaSetDevice(H.device));
    int rc = mlp_reserve(H);
    if (rc) return rc;
    CK(cudaMemcpyAsync(H.mlp_w.p, params, sizeof(float) * SCHED_NPARAM, cudaMemcpyDefault, H.stream));
    CK(cudaMemcpyAsync(H.mlp_norm.p, norm, sizeof(float) * 2 * SCHED_F, cudaMemcpyDefault, H.stream));
    CK(cudaStreamSynchronize(H.stream));
    H.sched_width = bin_width;
    H.sched_nclass = nclass;
    H.mlp_ready = true;
    return PB_OK;
}

int32_t pb_scheduler_get(pb_handle *h, float *params)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (!H.mlp_ready) return fail(H, PB_ERR_STATE, "no scheduler weights set");
    CK(cudaSetDevice(H.device));
    return copy_out_f32(H, params, H.mlp_w.as<float>(), SCHED_NPARAM);
}

int32_t pb_scheduler_predict(pb_handle *h, const float *X, int64_t n, float *out)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (!H.mlp_ready) return fail(H, PB_ERR_STATE, "no scheduler weights set");
    if (n < 0 || !X || !out) return fail(H, PB_ERR_INVALID, "bad arguments");
    if (n == 0) return PB_OK;
    CK(cudaSetDevice(H.device));
    const float *dX;
    int rc = stage_f32(H, H.mlp_x, X, n * SCHED_F, &dX);
    if (rc) return rc;
    CK(H.sched_pred.reserve(sizeof(float) * n));
    CK(launch_mlp_predict(&H, n, dX, H.sched_pred.as<float>()));
    return copy_out_f32(H, out, H.sched_pred.as<float>(), n);
}

int32_t pb_scheduler_gradients(pb_handle *h, const float *X, const float *y, int64_t n, float *grads, float *loss)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (!H.mlp_ready) return fail(H, PB_ERR_STATE, "no scheduler weights set");
    if (n < 1 || !X || !y || !grads) return fail(H, PB_ERR_INVALID, "bad arguments");
    CK(cudaSetDevice(H.device));
    const float *dX, *dy;
    int rc = stage_f32(H, H.mlp_x, X, n * SCHED_F, &dX);
    if (!rc) rc = stage_f32(H, H.mlp_y, y, n, &dy);
    if (rc) return rc;
    CK(launch_mlp_grad(&H, n, dX, dy, nullptr, nullptr));
    if ((rc = copy_out_f32(H, grads, H.mlp_g.as<float>(), SCHED_NPARAM))) return rc;
    if (loss) {
        std::vector<float> sq(n);
        if ((rc = copy_out_f32(H, sq.data(), mlp_last_sq(&H, n), n))) return rc;
        double acc = 0.0;
        for (float v : sq) acc += v;
        *loss = (float)(acc / (double)n);
    }
    return PB_OK;
}

int32_t pb_scheduler_train(pb_handle *h, const float *X, const float *y, int64_t n, int32_t steps, int32_t batch,
                           float lr, uint64_t seed, float *losses)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (!H.mlp_ready) return fail(H, PB_ERR_STATE, "set initial scheduler weights first (pb_scheduler_set)");
    if (n < 1 || !X || !y || steps < 0 || batch < 1) return fail(H, PB_ERR_INVALID, "bad arguments");
    CK(cudaSetDevice(H.device));
    const float *dX, *dy;
    int rc = stage_f32(H, H.mlp_x, X, n * SCHED_F, &dX);
    if (!rc) rc = stage_f32(H, H.mlp_y, y, n, &dy);
    if (rc) return rc;
    CK(cudaMemsetAsync(H.mlp_m.p, 0, sizeof(float) * SCHED_NPARAM, H.stream));
    CK(cudaMemsetAsync(H.mlp_v.p, 0, sizeof(float) * SCHED_NPARAM, H.stream));
    CK(H.mlp_idx.reserve(sizeof(int64_t) * batch));
    std::vector<float> sq(losses ? batch : 0);
    for (int32_t t = 0; t < steps; ++t) {
        CK(launch_draw(&H, batch, n, seed, (unsigned long long)t, H.mlp_idx.as<int64_t>()));
        CK(launch_mlp_grad(&H, batch, dX, dy, H.mlp_idx.as<int64_t>(), nullptr));
        CK(launch_mlp_adam(&H, lr, t + 1));
        if (losses) {
            if ((rc = copy_out_f32(H, sq.data(), mlp_last_sq(&H, batch), batch))) return rc;
            double acc = 0.0;
            for (float v : sq) acc += v;
            losses[t] = (float)(acc / (double)batch);
        }
    }
    CK(cudaStreamSynchronize(H.stream));
    return PB_OK;
}

int32_t pb_last_schedule(const pb_handle *h, int64_t *walk_rounds, int64_t *deferred, int64_t *pool_chunks,
                         double *phase_ms)
{
    if (!h) return PB_ERR_INVALID;
    if (phase_ms)
        for (int k = 0; k < 3; ++k) phase_ms[k] = h->H.t_phase_ms[k];
    if (walk_rounds) *walk_rounds = h->H.walk_rounds;
    if (deferred) *deferred = h->H.deferred_total;
    if (pool_chunks) *pool_chunks = (int64_t)h->H.pool_cap;
    return PB_OK;
}

namespace {

int batch_fail(pb_handle *h, int code, const std::string &msg)
{
    if (h) h->H.err = msg;
    return code;
}

int check_statuses(pb_handle *const *discs, int32_t ndiscs)
{
    Handle &H0 = discs[0]->H;
    if (cudaStreamSynchronize(H0.stream) != cudaSuccess) {
        cudaError_t e = cudaGetLastError();
        return batch_fail(discs[0], PB_ERR_CUDA, std::string("batched launch: ") + cudaGetErrorString(e));
    }
    for (int32_t k = 0; k < ndiscs; ++k) {
        int rc = check_status(discs[k]->H);
        if (rc) return batch_fail(discs[0], rc, "disc " + std::to_string(k) + ": " + discs[k]->H.err);
    }
    return PB_OK;
}

}  // namespace

int32_t pb_batch_points(pb_handle *const *discs, int32_t ndiscs, const pb_catalog *cat, const int64_t *npts,
                        const double *const *qx, const double *const *qy, const double *const *qz, double *const *out,
                        int32_t strategy, int32_t precision, int32_t flags)
{
    if (!discs || ndiscs < 1 || !discs[0]) return PB_ERR_INVALID;
    pb_handle *h0 = discs[0];
    Handle &H = h0->H;
    if (ndiscs > 65536) return batch_fail(h0, PB_ERR_INVALID, "at most 65536 discs per batch");
    if (strategy < 0 || strategy > 2) return batch_fail(h0, PB_ERR_INVALID, "unknown interpolation strategy");
    if (precision != PB_FP64 && precision != PB_FP32C) return batch_fail(h0, PB_ERR_INVALID, "unknown precision mode");
    if (!cat || !npts || !qx || !qy || !qz || !out) return batch_fail(h0, PB_ERR_INVALID, "NULL argument");
    const int64_t L = catalog_L(cat);
    if (L < 1) return batch_fail(h0, PB_ERR_INVALID, "empty catalog");
    for (int32_t k = 0; k < ndiscs; ++k) {
        if (!discs[k]) return batch_fail(h0, PB_ERR_INVALID, "NULL disc handle");
        Handle &Hk = discs[k]->H;
        if (!Hk.built) return batch_fail(h0, PB_ERR_STATE, "disc " + std::to_string(k) + " has no LBVH");
        if (Hk.device != H.device || Hk.stream != H.stream)
            return batch_fail(h0, PB_ERR_INVALID, "every disc handle must use the first one's device and stream");
        if (Hk.kernel != H.kernel) return batch_fail(h0, PB_ERR_INVALID, "every disc must use the same kernel");
        int rc = validate_catalog(Hk, cat, false);
        if (rc) return batch_fail(h0, rc, "disc " + std::to_string(k) + ": " + Hk.err);
        if (npts[k] < 0) return batch_fail(h0, PB_ERR_INVALID, "negative number of sample points");
        if (npts[k] > 0 && (!is_device_ptr(H, qx[k]) || !is_device_ptr(H, qy[k]) || !is_device_ptr(H, qz[k])))
            return batch_fail(h0, PB_ERR_INVALID, "batched sample points must be device memory of the handles' device");
        for (int64_t l = 0; l < L; ++l)
            if (npts[k] > 0 && !is_device_ptr(H, out[k * L + l]))
                return batch_fail(h0, PB_ERR_INVALID, "batched outputs must be device memory of the handles' device");
    }
    const std::vector<Launch> p32 = plan(items_of(cat, true)), p64 = plan(items_of(cat, false));
    if (p32.size() != 1 || p64.size() != 1)
        return batch_fail(h0, PB_ERR_INVALID, "catalog needs more than one launch: not supported by the batched path");
    CK(cudaSetDevice(H.device));
    // processing order of the discs: given, or the most work (points x particles^(1/3)) first
    std::vector<uint32_t> order(ndiscs);
    for (int32_t k = 0; k < ndiscs; ++k) order[k] = (uint32_t)k;
    if (H.batch_order == 1) {
        std::vector<double> work(ndiscs);
        for (int32_t k = 0; k < ndiscs; ++k) work[k] = (double)npts[k] * std::cbrt((double)discs[k]->H.n);
        std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return work[a] > work[b]; });
    }
    // pinned staging: descriptors, starts (processing order) and slot -> disc
    const size_t desc_bytes = sizeof(BatchDisc) * ndiscs, start_bytes = sizeof(int64_t) * (ndiscs + 1),
                 slot_bytes = sizeof(uint32_t) * ndiscs;
    const size_t host_bytes = desc_bytes + start_bytes + slot_bytes;
    if (H.batch_host_bytes < host_bytes) {
        if (H.batch_host) cudaFreeHost(H.batch_host);
        H.batch_host = nullptr;
        H.batch_host_bytes = 0;
        CK(cudaMallocHost(&H.batch_host, host_bytes));
        H.batch_host_bytes = host_bytes;
    }
    CK(H.batch_desc.reserve(desc_bytes));
    CK(H.batch_starts.reserve(start_bytes));
    CK(H.batch_slots.reserve(slot_bytes));
    CK(H.batch_ctr.reserve(8 * sizeof(unsigned long long)));
    BatchDisc *hd = static_cast<BatchDisc *>(H.batch_host);
    int64_t *hs = reinterpret_cast<int64_t *>(static_cast<char *>(H.batch_host) + desc_bytes);
    uint32_t *ho = reinterpret_cast<uint32_t *>(static_cast<char *>(H.batch_host) + desc_bytes + start_bytes);
    int64_t qtotal = 0;
    for (int32_t i = 0; i < ndiscs; ++i) {
        hs[i] = qtotal;
        ho[i] = order[i];
        qtotal += npts[order[i]];
    }
    hs[ndiscs] = qtotal;
    for (int32_t k = 0; k < ndiscs; ++k) {
        Handle &Hk = discs[k]->H;
        BatchDisc D;
        memset(&D, 0, sizeof(D));
        D.T = make_tree(Hk);
        D.C32 = dev_catalog(Hk, p32[0], out + k * L);
        D.C64 = dev_catalog(Hk, p64[0], out + k * L);
        D.qx = qx[k];
        D.qy = qy[k];
        D.qz = qz[k];
        D.nq = npts[k];
        // the disc's walk cut, made on the device from the tree just built
        CK(launch_cut_device(&Hk, D.T, H.batch_walk_split, &D.cut, &D.ncut));
        D.qp = Hk.qparams.as<QuantParams>();
        if (precision == PB_FP32C) {
            float4 *pay = nullptr;
            int stride = 0;
            CK(launch_batch_payload(&Hk, D.T, D.C32, &pay, &stride));
            D.pay = pay;
            D.stride = stride;
        }
        hd[k] = D;
    }
    const int cat_shape = batch_catalog_shape(hd[0].C32);
    CK(cudaMemcpyAsync(H.batch_desc.p, H.batch_host, desc_bytes, cudaMemcpyHostToDevice, H.stream));
    CK(cudaMemcpyAsync(H.batch_starts.p, hs, start_bytes, cudaMemcpyHostToDevice, H.stream));
    CK(cudaMemcpyAsync(H.batch_slots.p, ho, slot_bytes, cudaMemcpyHostToDevice, H.stream));
    // slices of a fixed size share one run pool, sized once (a call that reuses it allocates
    // nothing, which is what lets a step be captured in a CUDA graph)
    // (point, subtree) item records per point: the largest cut launch_cut_device can make
    const int NS = 4 * H.batch_walk_split + 8;
    const int64_t S = std::max<int64_t>(1, std::min<int64_t>(H.slice > 0 ? H.slice : qtotal, qtotal));
    if (qtotal > 0 && (H.pool_cap == 0 || H.batch_slice < S || H.batch_ns < NS)) {
        int rc = reserve_pool(H, S, NS);
        if (rc) return rc;
        H.batch_slice = S;
        H.batch_ns = NS;
    }
    if (qtotal > 0) {
        CK(H.batch_slot_of.reserve(sizeof(int) * H.batch_slice));
        unsigned long long *ctr = H.pool_ctr.as<unsigned long long>();
        RunPool P;
        P.runs = H.pool_runs.as<uint2>();
        P.next = H.pool_next.as<int>();
        P.used = ctr;
        P.cap = H.pool_cap;
        P.ns = NS;
        P.cut = nullptr;   // every disc's own cut is in its descriptor
        P.items = H.items.as<int2>();
        P.bnear = H.wbnear.as<int>();
        P.qacc = H.qacc.as<unsigned>();
        P.qflag = H.qflag.as<int>();
        P.n_deferred = reinterpret_cast<unsigned *>(ctr + 1);
        P.deferred = H.defer_a.as<uint32_t>();
        P.count_only = 0;
        P.leaf_size = H.leaf_size;
        for (int64_t s0 = 0; s0 < qtotal; s0 += S) {
            const int64_t m = std::min<int64_t>(S, qtotal - s0);
            CK(cudaMemsetAsync(ctr, 0, 16, H.stream));
            CK(cudaMemsetAsync(P.qacc, 0, sizeof(unsigned) * m, H.stream));
            CK(cudaMemsetAsync(P.qflag, 0, sizeof(int) * m, H.stream));
            CK(launch_batch_slice(&H, strategy, H.kernel, cat_shape, H.batch_desc.as<BatchDisc>(),
                                  H.batch_starts.as<int64_t>(), H.batch_slots.as<uint32_t>(), ndiscs, s0, m, P,
                                  precision == PB_FP64 ? 1 : 0, (unsigned)H.light_max, H.leaf_size, H.batch_blocks,
                                  H.batch_slot_of.as<int>(), H.batch_ctr.as<unsigned long long>()));
        }
    }
    if (flags & PB_BATCH_ASYNC) return PB_OK;
    return check_statuses(discs, ndiscs);
}

int32_t pb_batch_check(pb_handle *const *discs, int32_t ndiscs)
{
    if (!discs || ndiscs < 1 || !discs[0]) return PB_ERR_INVALID;
    for (int32_t k = 0; k < ndiscs; ++k)
        if (!discs[k]) return batch_fail(discs[0], PB_ERR_INVALID, "NULL disc handle");
    return check_statuses(discs, ndiscs);
}

int32_t pb_last_pair_split(const pb_handle *h, int64_t *heavy_queries, int64_t *light_queries, int64_t *heavy_pairs,
                           int64_t *light_pairs)
{
    if (!h) return PB_ERR_INVALID;
    if (heavy_queries) *heavy_queries = h->H.split_hq;
    if (light_queries) *light_queries = h->H.split_lq;
    if (heavy_pairs) *heavy_pairs = h->H.split_hp;
    if (light_pairs) *light_pairs = h->H.split_lp;
    return PB_OK;
}

int32_t pb_last_timings(const pb_handle *h, double *build_ms, double *interp_ms, int64_t *interp_launches)
{
    if (!h) return PB_ERR_INVALID;
    if (build_ms) *build_ms = h->H.t_build_ms;
    if (interp_ms) *interp_ms = h->H.t_interp_ms;
    if (interp_launches) *interp_launches = h->H.interp_launches;
    return PB_OK;
}

}  // extern "C"
