// pb_sched.cu -- learned work prediction for the point-interpolation schedule.
//
// A small MLP (SCHED_F inputs -> 64 -> 64 -> 1, ReLU) predicts log2(1 + accepted neighbours)
// of a sample point from features that are cheap to compute before the walk: the nearest
// particle's smoothing length and distance, the point's position in the particle set's box,
// and the smoothing-length maximum and size of the nearest leaf's ancestor subtrees at five
// scales.  Queries are then binned by predicted work (heaviest class first, Morton order kept
// inside a class) so that the 32 queries of a walk warp have similar work.  Only the order
// changes: every query's arithmetic, and so every output bit, is the same as without it.
//
// The network is BF16: weights and the inputs of every layer are rounded to bfloat16
// (round to nearest even), products are accumulated in FP32.  Training keeps FP32 master
// weights and runs on the GPU with the kernels below: forward, per-sample backward, a
// deterministic per-parameter gradient reduction (fixed sample order) and Adam.  The MLP is a
// few thousand parameters and well under a millisecond per million queries, so it uses plain
// FP32 FMAs rather than tensor cores.
#include <cuda_bf16.h>

#include "pb_internal.h"
#include "pb_interp_impl.cuh"

namespace pb {

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// parameter offsets in the flat array
__host__ __device__ constexpr int off_w1() { return 0; }
__host__ __device__ constexpr int off_b1() { return SCHED_H * SCHED_F; }
__host__ __device__ constexpr int off_w2() { return off_b1() + SCHED_H; }
__host__ __device__ constexpr int off_b2() { return off_w2() + SCHED_H * SCHED_H; }
__host__ __device__ constexpr int off_w3() { return off_b2() + SCHED_H; }
__host__ __device__ constexpr int off_b3() { return off_w3() + SCHED_H; }
static_assert(off_b3() + 1 == SCHED_NPARAM, "parameter layout");

// ------------------------------------------------------------------------------------
// features

__device__ __forceinline__ float flog2(double v) { return (float)log2(v > 1e-300 ? v : 1e-300); }

__global__ void k_sched_features(DevTree T, const int *__restrict__ parent, const QuantParams *__restrict__ qp,
                                 int64_t m, const uint32_t *__restrict__ ql, const double *__restrict__ qx,
                                 const double *__restrict__ qy, const double *__restrict__ qz,
                                 const int *__restrict__ bnear_in, float *feat)
{
    const QuantParams q = *qp;
    double ext = 0.0, cen[3];
    for (int d = 0; d < 3; ++d) {
        double e = q.flat[d] ? 0.0 : 1.0 / q.inv[d];
        cen[d] = q.vmin[d] + 0.5 * e;
        ext = fmax(ext, 0.5 * e);
    }
    if (!(ext > 0.0)) ext = 1.0;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t qi = ql ? __ldg(ql + j) : (uint32_t)j;
        const double px = qx[qi], py = qy[qi], pz = qz[qi];
        int64_t b = bnear_in ? bnear_in[j] : nearest_leaf(T, px, py, pz);
        float f[SCHED_F];
        double4 L = b >= 0 ? ldg4(T.leaf + b) : make_double4(px, py, pz, 1.0);
        double dn = sqrt(d2_point(px, py, pz, L));
        f[0] = flog2(L.w);
        f[1] = flog2(dn / ext + 1e-12);
        const double u0 = (px - cen[0]) / ext, u1 = (py - cen[1]) / ext, u2 = (pz - cen[2]) / ext;
        f[2] = (float)u0;
        f[3] = (float)u1;
        f[4] = (float)u2;
        f[5] = flog2(sqrt(u0 * u0 + u1 * u1 + u2 * u2) + 1e-6);
        // ancestors of the nearest leaf whose subtrees hold >= 2^4, 2^8, ..., 2^20 leaves
        int id = b >= 0 ? (int)(T.n + b) : T.root;
        int lev = 0;
        const int64_t guard_max = 4 * T.n + 64;
        int64_t guard = 0;
        while (lev < 5) {
            const int64_t need = (int64_t)1 << (4 + 4 * lev);
            int64_t size = 1;
            if (id >= 1 && id < T.n) {
                int2 r = T.range[id - 1];
                size = (int64_t)r.y - r.x + 1;
            }
            const int p = (id >= 1 && T.root) ? parent[id - 1] : 0;
            if (size < need && p != 0 && ++guard < guard_max) {
                id = p;
                continue;
            }
            float hm, hd;
            if (id >= 1 && id < T.n) {
                NodeF nd = T.node[id - 1];
                hm = T.node_hmax[id - 1];
                double dx = nd.hix - nd.lox, dy = nd.hiy - nd.loy, dz = nd.hiz - nd.loz;
                hd = flog2(0.5 * sqrt(dx * dx + dy * dy + dz * dz) / ext + 1e-12);
            } else {
                hm = (float)L.w;
                hd = flog2(1e-12);
            }
            f[6 + 2 * lev] = flog2(hm);
            f[7 + 2 * lev] = hd;
            ++lev;
        }
        for (int k = 0; k < SCHED_F; ++k) feat[j * SCHED_F + k] = f[k];
    }
}

// ------------------------------------------------------------------------------------
// MLP forward (shared by inference and training)

struct MlpSmem {
    float w1[SCHED_H * SCHED_F], b1[SCHED_H], w2[SCHED_H * SCHED_H], b2[SCHED_H], w3[SCHED_H], b3;
    float mu[SCHED_F], isd[SCHED_F];
};

__device__ void load_mlp(MlpSmem &S, const float *params, const float *norm)
{
    for (int i = threadIdx.x; i < SCHED_NPARAM; i += blockDim.x) {
        float v = bf16r(params[i]);
        if (i < off_b1()) S.w1[i] = v;
        else if (i < off_w2()) S.b1[i - off_b1()] = v;
        else if (i < off_b2()) S.w2[i - off_w2()] = v;
        else if (i < off_w3()) S.b2[i - off_b2()] = v;
        else if (i < off_b3()) S.w3[i - off_w3()] = v;
        else S.b3 = v;
    }
    for (int i = threadIdx.x; i < SCHED_F; i += blockDim.x) {
        S.mu[i] = norm[i];
        S.isd[i] = norm[SCHED_F + i];
    }
    __syncthreads();
}

// one sample: returns the prediction; optionally stores the layer inputs (bf16-rounded)
// and pre-activation signs for the backward pass
__device__ __forceinline__ float mlp_forward(const MlpSmem &S, const float *x_raw, float *xin, float *a1, float *a2,
                                             unsigned long long *m1, unsigned long long *m2)
{
    float x[SCHED_F];
#pragma unroll
    for (int k = 0; k < SCHED_F; ++k) x[k] = bf16r((x_raw[k] - S.mu[k]) * S.isd[k]);
    if (xin)
        for (int k = 0; k < SCHED_F; ++k) xin[k] = x[k];
    float h1[SCHED_H];
    unsigned long long mask1 = 0, mask2 = 0;
#pragma unroll 4
    for (int i = 0; i < SCHED_H; ++i) {
        float z = S.b1[i];
#pragma unroll
        for (int k = 0; k < SCHED_F; ++k) z = fmaf(S.w1[i * SCHED_F + k], x[k], z);
        if (z > 0.f) mask1 |= 1ULL << i;
        h1[i] = bf16r(fmaxf(z, 0.f));
    }
    float y = S.b3;
    for (int i = 0; i < SCHED_H; ++i) {
        float z = S.b2[i];
#pragma unroll 8
        for (int k = 0; k < SCHED_H; ++k) z = fmaf(S.w2[i * SCHED_H + k], h1[k], z);
        if (z > 0.f) mask2 |= 1ULL << i;
        const float h = bf16r(fmaxf(z, 0.f));
        if (a2) a2[i] = h;
        y = fmaf(S.w3[i], h, y);
    }
    if (a1)
        for (int k = 0; k < SCHED_H; ++k) a1[k] = h1[k];
    if (m1) *m1 = mask1;
    if (m2) *m2 = mask2;
    return y;
}

__global__ void __launch_bounds__(128) k_mlp_predict(const float *__restrict__ params, const float *__restrict__ norm,
                                                     int64_t n, const float *__restrict__ X, float *y)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MlpSmem &S = *reinterpret_cast<MlpSmem *>(smem_raw);
    load_mlp(S, params, norm);
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x)
        y[s] = mlp_forward(S, X + s * SCHED_F, nullptr, nullptr, nullptr, nullptr, nullptr);
}

// training, step 1: forward + per-sample backward.  Loss = mean over the batch of (y - t)^2.
// Per sample it stores the bf16 layer inputs (x, a1, a2) and the backpropagated deltas
// (d1, d2 at the two hidden pre-activations, g at the output).
__global__ void __launch_bounds__(128) k_mlp_fwd_bwd(const float *__restrict__ params, const float *__restrict__ norm,
                                                     int64_t nb, const float *__restrict__ X,
                                                     const float *__restrict__ T, const int64_t *__restrict__ idx,
                                                     float *xin, float *a1, float *a2, float *d1, float *d2, float *g,
                                                     float *sq)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MlpSmem &S = *reinterpret_cast<MlpSmem *>(smem_raw);
    load_mlp(S, params, norm);
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < nb; s += (int64_t)gridDim.x * blockDim.x) {
        const int64_t src = idx ? idx[s] : s;
        unsigned long long m1, m2;
        const float y = mlp_forward(S, X + src * SCHED_F, xin + s * SCHED_F, a1 + s * SCHED_H, a2 + s * SCHED_H, &m1, &m2);
        const float e = y - T[src];
        const float gy = 2.f * e / (float)nb;
        g[s] = gy;
        sq[s] = e * e;
        float dd2[SCHED_H];
        for (int i = 0; i < SCHED_H; ++i) {
            dd2[i] = ((m2 >> i) & 1ULL) ? gy * S.w3[i] : 0.f;
            d2[s * SCHED_H + i] = dd2[i];
        }
        for (int k = 0; k < SCHED_H; ++k) {
            float acc = 0.f;
            if ((m1 >> k) & 1ULL)
                for (int i = 0; i < SCHED_H; ++i) acc = fmaf(dd2[i], S.w2[i * SCHED_H + k], acc);
            d1[s * SCHED_H + k] = acc;
        }
    }
}

// training, step 2: one thread per parameter sums its gradient over the batch in sample order
__global__ void k_mlp_reduce(int64_t nb, const float *__restrict__ xin, const float *__restrict__ a1,
                             const float *__restrict__ a2, const float *__restrict__ d1,
                             const float *__restrict__ d2, const float *__restrict__ g, float *grad)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= SCHED_NPARAM) return;
    float acc = 0.f;
    if (p < off_b1()) {
        const int i = p / SCHED_F, k = p % SCHED_F;
        for (int64_t s = 0; s < nb; ++s) acc = fmaf(d1[s * SCHED_H + i], xin[s * SCHED_F + k], acc);
    } else if (p < off_w2()) {
        const int i = p - off_b1();
        for (int64_t s = 0; s < nb; ++s) acc += d1[s * SCHED_H + i];
    } else if (p < off_b2()) {
        const int i = (p - off_w2()) / SCHED_H, k = (p - off_w2()) % SCHED_H;
        for (int64_t s = 0; s < nb; ++s) acc = fmaf(d2[s * SCHED_H + i], a1[s * SCHED_H + k], acc);
    } else if (p < off_w3()) {
        const int i = p - off_b2();
        for (int64_t s = 0; s < nb; ++s) acc += d2[s * SCHED_H + i];
    } else if (p < off_b3()) {
        const int i = p - off_w3();
        for (int64_t s = 0; s < nb; ++s) acc = fmaf(g[s], a2[s * SCHED_H + i], acc);
    } else {
        for (int64_t s = 0; s < nb; ++s) acc += g[s];
    }
    grad[p] = acc;
}

__global__ void k_adam(float *w, const float *__restrict__ g, float *m, float *v, float lr, float b1, float b2,
                       float eps, float c1, float c2)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= SCHED_NPARAM) return;
    const float gp = g[p];
    const float mp = b1 * m[p] + (1.f - b1) * gp;
    const float vp = b2 * v[p] + (1.f - b2) * gp * gp;
    m[p] = mp;
    v[p] = vp;
    w[p] -= lr * (mp / c1) / (sqrtf(vp / c2) + eps);
}

// batch sampling: a fixed-seed permutation-free draw (splitmix64 per step and slot)
__global__ void k_draw(int64_t nb, int64_t n, unsigned long long seed, unsigned long long step, int64_t *idx)
{
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < nb; s += (int64_t)gridDim.x * blockDim.x) {
        unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * (step * 1315423911ULL + (unsigned long long)s + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        idx[s] = (int64_t)(z % (unsigned long long)n);
    }
}

// ------------------------------------------------------------------------------------
// binning keys: heaviest predicted class first; a stable sort keeps the Morton order inside
__global__ void k_sched_keys(int64_t m, const float *__restrict__ pred, float width, int nclass, uint32_t *keys,
                             uint32_t *vals)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
        float p = pred[j];
        int c = (p == p) ? (int)floorf(p / width) : 0;
        c = c < 0 ? 0 : (c >= nclass ? nclass - 1 : c);
        keys[j] = (uint32_t)(nclass - 1 - c);
        vals[j] = (uint32_t)j;
    }
}

__global__ void k_gather_u32(int64_t m, const uint32_t *__restrict__ order, const uint32_t *__restrict__ src,
                             uint32_t *dst)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x)
        dst[j] = src[order[j]];
}

__global__ void k_gather_i32(int64_t m, const uint32_t *__restrict__ order, const int *__restrict__ src, int *dst)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x)
        dst[j] = src[order[j]];
}

// ------------------------------------------------------------------------------------
// launchers

static size_t mlp_smem() { return sizeof(MlpSmem); }

cudaError_t launch_sched_features(Handle *H, const DevTree &T, int64_t m, const uint32_t *ql, const double *qx,
                                  const double *qy, const double *qz, const int *bnear, float *feat)
{
    k_sched_features<<<grid_for(m, 128, 1 << 30), 128, 0, H->stream>>>(T, H->parent.as<int>(),
                                                                     H->qparams.as<QuantParams>(), m, ql, qx, qy,
                                                                     qz, bnear, feat);
    H->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_mlp_predict(Handle *H, int64_t n, const float *X, float *y)
{
    const size_t sm = mlp_smem();
    cudaError_t e = cudaFuncSetAttribute(k_mlp_predict, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e) return e;
    k_mlp_predict<<<grid_for(n, 128), 128, sm, H->stream>>>(H->mlp_w.as<float>(), H->mlp_norm.as<float>(), n, X, y);
    H->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_mlp_grad(Handle *H, int64_t nb, const float *X, const float *T, const int64_t *idx, float *loss)
{
    cudaError_t e;
    const size_t sm = mlp_smem();
    if ((e = cudaFuncSetAttribute(k_mlp_fwd_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm))) return e;
    if ((e = H->mlp_scr.reserve(sizeof(float) * nb * (SCHED_F + 4 * SCHED_H + 2)))) return e;
    float *xin = H->mlp_scr.as<float>();
    float *a1 = xin + nb * SCHED_F, *a2 = a1 + nb * SCHED_H, *d1 = a2 + nb * SCHED_H, *d2 = d1 + nb * SCHED_H;
    float *g = d2 + nb * SCHED_H, *sq = g + nb;
    k_mlp_fwd_bwd<<<grid_for(nb, 128), 128, sm, H->stream>>>(H->mlp_w.as<float>(), H->mlp_norm.as<float>(), nb, X, T,
                                                           idx, xin, a1, a2, d1, d2, g, sq);
    k_mlp_reduce<<<(SCHED_NPARAM + 127) / 128, 128, 0, H->stream>>>(nb, xin, a1, a2, d1, d2, g,
                                                                   H->mlp_g.as<float>());
    H->launches += 2;
    if (loss) *loss = 0.f;
    (void)sq;
    return cudaGetLastError();
}

const float *mlp_last_sq(Handle *H, int64_t nb)
{
    return H->mlp_scr.as<float>() + nb * (SCHED_F + 4 * SCHED_H) + nb;
}

cudaError_t launch_mlp_adam(Handle *H, float lr, int64_t step)
{
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_adam<<<(SCHED_NPARAM + 127) / 128, 128, 0, H->stream>>>(H->mlp_w.as<float>(), H->mlp_g.as<float>(),
                                                             H->mlp_m.as<float>(), H->mlp_v.as<float>(), lr, b1, b2,
                                                             1e-8f, c1, c2);
    H->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_draw(Handle *H, int64_t nb, int64_t n, unsigned long long seed, unsigned long long step,
                        int64_t *idx)
{
    k_draw<<<grid_for(nb, 256), 256, 0, H->stream>>>(nb, n, seed, step, idx);
    H->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_sched_order(Handle *H, int64_t m, const float *pred, float width, int nclass, uint32_t *order)
{
    cudaError_t e;
    uint32_t *k = H->lpt_k.as<uint32_t>(), *ka = H->lpt_ka.as<uint32_t>(), *va = H->lpt_va.as<uint32_t>();
    k_sched_keys<<<grid_for(m, 256), 256, 0, H->stream>>>(m, pred, width, nclass, k, order);
    H->launches += 1;
    if ((e = cudaGetLastError())) return e;
    int bits = 1;
    while ((1 << bits) < nclass) ++bits;
    return sort_pairs_u32(H, k, order, ka, va, m, bits);
}

cudaError_t launch_gather_u32(Handle *H, int64_t m, const uint32_t *order, const uint32_t *src, uint32_t *dst)
{
    k_gather_u32<<<grid_for(m, 256), 256, 0, H->stream>>>(m, order, src, dst);
    H->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_gather_i32(Handle *H, int64_t m, const uint32_t *order, const int *src, int *dst)
{
    k_gather_i32<<<grid_for(m, 256), 256, 0, H->stream>>>(m, order, src, dst);
    H->launches += 1;
    return cudaGetLastError();
}

}  // namespace pb
