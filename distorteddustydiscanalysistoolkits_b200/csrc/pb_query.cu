// pb_query.cu -- batched neighbour-search entry points on a built LBVH:
//   LBVH_find_nearest_h / LBVH_find_nearest (LinearBVHQueries.jl:79-140)
//   LBVH_query! (LinearBVHQueries.jl:183-211) as count + fill passes (CSR output)
// These are the bit-exact probes of the neighbour sets: the traversal is the same
// conservative stackless DFS as the interpolation kernels, so accepted leaves appear in
// ascending sorted-leaf order exactly as in the reference.
#include "pb_internal.h"
#include "pb_interp_impl.cuh"

namespace pb {

__global__ void k_nearest(DevTree T, int64_t nq, const double *__restrict__ qx, const double *__restrict__ qy,
                          const double *__restrict__ qz, double *h_out, int64_t *idx_out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nq; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t b = nearest_leaf(T, qx[i], qy[i], qz[i]);
        if (h_out) h_out[i] = b < 0 ? __longlong_as_double(0x7ff8000000000000LL) : T.leaf[b].w;
        if (idx_out) idx_out[i] = b;
    }
}

// gather predicate d2 <= radius^2 (LinearBVHTraversalMacros.jl:26-108); pool == nullptr counts only.
// The closest accepted leaf is the first strictly closer one in DFS order (LinearBVHQueries.jl:33-39,
// 196-203): nearest[i] its index (-1 if none), nearest_d2[i] its squared distance (+Inf if none).
__global__ void k_query(DevTree T, int64_t nq, const double *__restrict__ qx, const double *__restrict__ qy,
                        const double *__restrict__ qz, const double *__restrict__ radius,
                        const int64_t *__restrict__ offsets, int64_t *counts, int64_t *pool, int64_t *nearest,
                        double *nearest_d2)
{
    const int64_t n = T.n;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nq; i += (int64_t)gridDim.x * blockDim.x) {
        double px = qx[i], py = qy[i], pz = qz[i];
        double r = radius[i];
        double r2 = __dmul_rn(r, r);
        int64_t cnt = 0, ci = -1;
        double cd = INFINITY;
        int64_t base = pool ? offsets[i] : 0;
        int64_t cap = pool ? offsets[i + 1] - offsets[i] : 0;
        int node = T.root;
        int64_t bi = 0, guard = 0, limit = 4 * n + 64;
        bool brute = (node == 0);
        while (brute ? (bi < n) : (node != 0)) {
            if (++guard > limit) { flag(T.status, ST_TRAVERSAL); break; }
            if (brute || node >= n) {
                int64_t b = brute ? bi++ : (int64_t)(node - n);
                double4 L = ldg4(T.leaf + b);
                double d2 = d2_point(px, py, pz, L);
                if (d2 <= r2) {
                    if (pool) {
                        if (cnt < cap) pool[base + cnt] = b;
                        else flag(T.status, ST_POOL);
                    }
                    ++cnt;
                    if (d2 < cd) { cd = d2; ci = b; }
                }
                if (!brute) node = __ldg(T.leaf_escape + b);
            } else {
                NodeF nd = load_node(T.node + (node - 1));
                node = (d2_box(px, py, pz, nd) > r2) ? nd.escape : nd.left;
            }
        }
        if (counts) counts[i] = cnt;
        if (nearest) nearest[i] = ci;
        if (nearest_d2) nearest_d2[i] = cd;
    }
}

// Event counts of the reference algorithm itself (leaf size 1, Karras tree, left-first DFS,
// FP64 boxes and the reference's pruning tests, LinearBVHTraversalMacros.jl:26-371): per
// query [nearest-pass internal visits, nearest-pass leaf tests, main-pass internal visits,
// main-pass leaf tests, accepted neighbours].  Used for the algorithmic-bytes roofline model
// and as exact per-query work labels.
struct Tree64 {
    const double *bmin, *bmax, *hmax;
};

__device__ __forceinline__ double d2_box64(const Tree64 &B, int64_t nin, int64_t i0, double px, double py, double pz)
{
    double p[3] = {px, py, pz};
    double s = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double a = B.bmin[d * nin + i0], b = B.bmax[d * nin + i0];
        double t = p[d] < a ? __dsub_rn(a, p[d]) : (p[d] > b ? __dsub_rn(p[d], b) : 0.0);
        s = __dadd_rn(s, __dmul_rn(t, t));
    }
    return s;
}

__global__ void k_stats(DevTree T, Tree64 B, int strategy, int64_t nq, const double *__restrict__ qx,
                        const double *__restrict__ qy, const double *__restrict__ qz, int64_t *stats)
{
    const int64_t n = T.n, nin = n - 1;
    const double K = kernel_valid(T.kernel);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nq; i += (int64_t)gridDim.x * blockDim.x) {
        double px = qx[i], py = qy[i], pz = qz[i];
        int64_t nv = 0, nl = 0, mv = 0, ml = 0, acc = 0;
        int64_t guard, limit = 4 * n + 64;
        double ha = 0.0;
        if (strategy != SCATTER) {
            double best = INFINITY;
            int64_t bi = -1;
            if (T.root == 0) {
                double d2 = d2_point(px, py, pz, ldg4(T.leaf));
                ++nl;
                if (d2 < best) bi = 0;
            } else {
                int node = T.root;
                guard = 0;
                while (node != 0) {
                    if (++guard > limit) { flag(T.status, ST_TRAVERSAL); break; }
                    if (node >= n) {
                        int64_t b = node - n;
                        double d2 = d2_point(px, py, pz, ldg4(T.leaf + b));
                        ++nl;
                        if (d2 < best) { best = d2; bi = b; }
                        node = __ldg(T.leaf_escape + b);
                    } else {
                        ++nv;
                        NodeF nd = load_node(T.node + (node - 1));
                        node = (d2_box64(B, nin, node - 1, px, py, pz) > best) ? nd.escape : nd.left;
                    }
                }
            }
            ha = bi < 0 ? __longlong_as_double(0x7ff8000000000000LL) : T.leaf[bi].w;
        }
        double ra = __dmul_rn(K, ha), r2a = __dmul_rn(ra, ra);
        int node = T.root;
        int64_t bi = 0;
        bool brute = (node == 0);
        guard = 0;
        while (brute ? (bi < n) : (node != 0)) {
            if (++guard > limit) { flag(T.status, ST_TRAVERSAL); break; }
            if (brute || node >= n) {
                int64_t b = brute ? bi++ : (int64_t)(node - n);
                double4 L = ldg4(T.leaf + b);
                double r = __dmul_rn(K, L.w), rr = __dmul_rn(r, r);
                double r2 = strategy == GATHER ? r2a : (strategy == SCATTER ? rr : (r2a > rr ? r2a : rr));
                ++ml;
                if (d2_point(px, py, pz, L) <= r2) ++acc;
                if (!brute) node = __ldg(T.leaf_escape + b);
            } else {
                ++mv;
                NodeF nd = load_node(T.node + (node - 1));
                double r = __dmul_rn(K, B.hmax[node - 1]), rr = __dmul_rn(r, r);
                double r2 = strategy == GATHER ? r2a : (strategy == SCATTER ? rr : (r2a > rr ? r2a : rr));
                node = (d2_box64(B, nin, node - 1, px, py, pz) > r2) ? nd.escape : nd.left;
            }
        }
        int64_t *s = stats + 5 * i;
        s[0] = nv; s[1] = nl; s[2] = mv; s[3] = ml; s[4] = acc;
    }
}

cudaError_t launch_stats(Handle *H, const DevTree &T, int strategy, int64_t nq, const double *qx, const double *qy,
                         const double *qz, int64_t *stats)
{
    Tree64 B{H->bmin64.as<double>(), H->bmax64.as<double>(), H->hmax64.as<double>()};
    k_stats<<<grid_for(nq, 128, 1 << 30), 128, 0, H->stream>>>(T, B, strategy, nq, qx, qy, qz, stats);
    H->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_nearest(Handle *H, const DevTree &T, int64_t nq, const double *qx, const double *qy,
                           const double *qz, double *h_out, int64_t *idx_out)
{
    k_nearest<<<grid_for(nq, 128, 1 << 30), 128, 0, H->stream>>>(T, nq, qx, qy, qz, h_out, idx_out);
    H->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_query(Handle *H, const DevTree &T, int64_t nq, const double *qx, const double *qy,
                         const double *qz, const double *radius, const int64_t *offsets, int64_t *counts,
                         int64_t *pool, int64_t *nearest, double *nearest_d2)
{
    k_query<<<grid_for(nq, 128, 1 << 30), 128, 0, H->stream>>>(T, nq, qx, qy, qz, radius, offsets, counts, pool,
                                                                nearest, nearest_d2);
    H->launches += 1;
    return cudaGetLastError();
}

// Sample points of a structured grid, generated on the device (coordinate_grid + flatten,
// StructuredGrid.jl:126-204, transform.jl:53-66): column-major linear order, the first axis
// fastest; coord 0 Cartesian (a0, a1, a2), 2 cylindrical (s cos phi, s sin phi, z), 3 spherical
// (r sin(theta) cos(phi), r sin(theta) sin(phi), r cos(theta)) with the host's operation order.
__global__ void k_grid_points(int coord, const double *__restrict__ a0, int64_t n0, const double *__restrict__ a1,
                              int64_t n1, const double *__restrict__ a2, int64_t n2, double *x, double *y, double *z)
{
    const int64_t n = n0 * n1 * n2;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i0 = i % n0, i1 = (i / n0) % n1, i2 = i / (n0 * n1);
        const double u = a0[i0], v = a1[i1], w = a2[i2];
        if (coord == 2) {
            x[i] = __dmul_rn(u, cos(v));
            y[i] = __dmul_rn(u, sin(v));
            z[i] = w;
        } else if (coord == 3) {
            const double st = sin(w);
            x[i] = __dmul_rn(__dmul_rn(u, st), cos(v));
            y[i] = __dmul_rn(__dmul_rn(u, st), sin(v));
            z[i] = __dmul_rn(u, cos(w));
        } else {
            x[i] = u;
            y[i] = v;
            z[i] = w;
        }
    }
}

cudaError_t launch_grid_points(Handle *H, int coord, const double *a0, int64_t n0, const double *a1, int64_t n1,
                               const double *a2, int64_t n2, double *x, double *y, double *z)
{
    k_grid_points<<<grid_for(n0 * n1 * n2, 256), 256, 0, H->stream>>>(coord, a0, n0, a1, n1, a2, n2, x, y, z);
    H->launches += 1;
    return cudaGetLastError();
}

// Lines of an image (LineSamples of a column-density map): line k = i + n0 * j starts at
// (c + a0[i] e1) + a1[j] e2 and runs along d; no FMA, so the values equal the host's
// per-component expression.
__global__ void k_line_image(const double *__restrict__ a0, int64_t n0, const double *__restrict__ a1, int64_t n1,
                             LineFrame F, double *ox, double *oy, double *oz, double *dx, double *dy, double *dz)
{
    const int64_t n = n0 * n1;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const double u = a0[k % n0], v = a1[k / n0];
        ox[k] = __dadd_rn(__dadd_rn(F.c[0], __dmul_rn(u, F.e1[0])), __dmul_rn(v, F.e2[0]));
        oy[k] = __dadd_rn(__dadd_rn(F.c[1], __dmul_rn(u, F.e1[1])), __dmul_rn(v, F.e2[1]));
        oz[k] = __dadd_rn(__dadd_rn(F.c[2], __dmul_rn(u, F.e1[2])), __dmul_rn(v, F.e2[2]));
        dx[k] = F.d[0];
        dy[k] = F.d[1];
        dz[k] = F.d[2];
    }
}

cudaError_t launch_line_image(Handle *H, const double *a0, int64_t n0, const double *a1, int64_t n1, const LineFrame &F,
                              double *ox, double *oy, double *oz, double *dx, double *dy, double *dz)
{
    k_line_image<<<grid_for(n0 * n1, 256), 256, 0, H->stream>>>(a0, n0, a1, n1, F, ox, oy, oz, dx, dy, dz);
    H->launches += 1;
    return cudaGetLastError();
}

}  // namespace pb
