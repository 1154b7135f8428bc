// pb_build.cu -- LBVH build on the device, bit-exact against the reference.
//
//   bbox      per-axis min/max (exact in any order)           MortonCode.jl:443-456
//   encode    FP64 (v-vmin)*inv(dv), floor(2097151*f), interleave   MortonCode.jl:209-217,275-305,473-498
//   sort      stable LSD radix sort of (code, index)          == sortperm's index-tie order, MortonCode.jl:182
//   dedupe    c'[i] = i + max_{j<=i}(c[j]-j)                  == the sequential bump, MortonCode.jl:189-193
//   gather    permuted leaves and particle columns            InterpolationInput.jl:211-219, LinearBVH.jl:89-96
//   topology  Karras range/split + internal escapes           BinaryRadixTree.jl:140-260
//   refit     leaf escapes + bottom-up AABB/hmax refit         BinaryRadixTree.jl:262-281, LinearBVH.jl:98-156
//
// Compiled with -fmad=false: the quantisation must be the IEEE result of the reference's
// operation order.
#include <cstdio>

#include "pb_internal.h"

namespace pb {

constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;   // 4096 keys per block
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_CHUNK = SCAN_THREADS * SCAN_ITEMS;

// ------------------------------------------------------------------------------------
// bounding box
__global__ void k_bbox_partial(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                               const double *__restrict__ z, const double *__restrict__ h, double *part,
                               int *status)
{
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    int bad = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double v[3] = {x[i], y[i], z[i]};
        if (!isfinite(h[i])) bad = 1;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (!isfinite(v[d])) bad = 1;
            if (v[d] < mn[d]) mn[d] = v[d];
            if (v[d] > mx[d]) mx[d] = v[d];
        }
    }
    if (bad) atomicOr(status, ST_NONFINITE);
    __shared__ double s[6][32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        for (int o = 16; o > 0; o >>= 1) {
            double a = __shfl_down_sync(0xffffffffu, mn[d], o);
            double b = __shfl_down_sync(0xffffffffu, mx[d], o);
            if (a < mn[d]) mn[d] = a;
            if (b > mx[d]) mx[d] = b;
        }
    }
    if (lane == 0)
        for (int d = 0; d < 3; ++d) { s[d][w] = mn[d]; s[3 + d][w] = mx[d]; }
    __syncthreads();
    if (threadIdx.x < 6) {
        int d = threadIdx.x;
        double r = s[d][0];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
            double v = s[d][k];
            if (d < 3 ? (v < r) : (v > r)) r = v;
        }
        part[blockIdx.x * 6 + d] = r;
    }
}

__global__ void k_bbox_final(int nparts, const double *part, QuantParams *qp)
{
    if (threadIdx.x >= 3) return;
    int d = threadIdx.x;
    double mn = part[d], mx = part[3 + d];
    for (int b = 1; b < nparts; ++b) {
        double a = part[b * 6 + d], c = part[b * 6 + 3 + d];
        if (a < mn) mn = a;
        if (c > mx) mx = c;
    }
    double dv = mx - mn;
    qp->vmin[d] = mn;
    qp->flat[d] = (dv == 0.0);
    qp->inv[d] = (dv == 0.0) ? 0.0 : 1.0 / dv;
}

cudaError_t launch_bbox(Handle *H, int64_t n, const double *x, const double *y, const double *z, const double *h)
{
    int grid = grid_for(n, 256, 148 * 4);
    cudaError_t e = H->bbox_part.reserve(sizeof(double) * 6 * grid);
    if (e) return e;
    k_bbox_partial<<<grid, 256, 0, H->stream>>>(n, x, y, z, h, H->bbox_part.as<double>(), H->status.as<int>());
    k_bbox_final<<<1, 32, 0, H->stream>>>(grid, H->bbox_part.as<double>(), H->qparams.as<QuantParams>());
    H->launches += 2;
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// quantise + Morton encode
__device__ __forceinline__ uint64_t expand_bits3(uint64_t x)
{
    x = (x | (x << 32)) & 0x1f00000000ffffULL;
    x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
    x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
    x = (x | (x << 2)) & 0x1249249249249249ULL;
    return x;
}

__device__ __forceinline__ uint64_t quantize21(double v, double vmin, double inv, int flat)
{
    const double scale = 2097151.0;   // exp2(21) - 1 (MortonCode.jl:426-434)
    double f = flat ? 0.5 : __dmul_rn(__dsub_rn(v, vmin), inv);
    return (uint64_t)floor(__dmul_rn(scale, f));
}

__global__ void k_encode(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                         const double *__restrict__ z, const QuantParams *__restrict__ qp, uint64_t *codes,
                         uint32_t *idx)
{
    QuantParams q = *qp;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t ix = quantize21(x[i], q.vmin[0], q.inv[0], q.flat[0]);
        uint64_t iy = quantize21(y[i], q.vmin[1], q.inv[1], q.flat[1]);
        uint64_t iz = quantize21(z[i], q.vmin[2], q.inv[2], q.flat[2]);
        codes[i] = (expand_bits3(ix) << 2) | (expand_bits3(iy) << 1) | expand_bits3(iz);
        idx[i] = (uint32_t)i;
    }
}

cudaError_t launch_encode(Handle *H, int64_t n, const double *x, const double *y, const double *z)
{
    k_encode<<<grid_for(n, 256), 256, 0, H->stream>>>(n, x, y, z, H->qparams.as<QuantParams>(),
                                                       H->codes.as<uint64_t>(), H->idx.as<uint32_t>());
    H->launches += 1;
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// device-wide exclusive sum of uint32 (radix-sort offsets)
__device__ __forceinline__ uint32_t block_exclusive_sum(uint32_t v, uint32_t *total)
{
    __shared__ uint32_t ws[32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) ws[w] = inc;
    __syncthreads();
    if (w == 0) {
        uint32_t s = lane < nw ? ws[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += t;
        }
        ws[lane] = s;
    }
    __syncthreads();
    uint32_t before = (w > 0 ? ws[w - 1] : 0) + inc - v;
    if (total) *total = ws[nw - 1];
    __syncthreads();
    return before;
}

__global__ void k_scan_reduce(int64_t m, const uint32_t *in, uint32_t *part)
{
    int64_t base = (int64_t)blockIdx.x * SCAN_CHUNK;
    uint32_t s = 0;
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        int64_t i = base + k * SCAN_THREADS + threadIdx.x;
        if (i < m) s += in[i];
    }
    uint32_t tot;
    block_exclusive_sum(s, &tot);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

__global__ void k_scan_partials(int np, uint32_t *part)
{
    uint32_t carry = 0;
    for (int base = 0; base < np; base += SCAN_THREADS) {
        int i = base + threadIdx.x;
        uint32_t v = i < np ? part[i] : 0;
        uint32_t tot;
        uint32_t ex = block_exclusive_sum(v, &tot);
        if (i < np) part[i] = carry + ex;
        carry += tot;
    }
}

__global__ void k_scan_apply(int64_t m, const uint32_t *in, uint32_t *out, const uint32_t *part)
{
    int64_t base = (int64_t)blockIdx.x * SCAN_CHUNK + (int64_t)threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS], s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        int64_t i = base + k;
        v[k] = i < m ? in[i] : 0;
        s += v[k];
    }
    uint32_t ex = block_exclusive_sum(s, nullptr) + part[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        int64_t i = base + k;
        if (i < m) out[i] = ex;
        ex += v[k];
    }
}

static cudaError_t exclusive_scan_u32(Handle *H, const uint32_t *in, uint32_t *out, int64_t m)
{
    int nb = (int)((m + SCAN_CHUNK - 1) / SCAN_CHUNK);
    cudaError_t e = H->scan_part.reserve(sizeof(uint32_t) * (nb + 1));
    if (e) return e;
    uint32_t *part = H->scan_part.as<uint32_t>();
    k_scan_reduce<<<nb, SCAN_THREADS, 0, H->stream>>>(m, in, part);
    k_scan_partials<<<1, SCAN_THREADS, 0, H->stream>>>(nb, part);
    k_scan_apply<<<nb, SCAN_THREADS, 0, H->stream>>>(m, in, out, part);
    H->launches += 3;
    return cudaGetLastError();
}

cudaError_t launch_exclusive_scan_u32(Handle *H, const uint32_t *in, uint32_t *out, int64_t m)
{
    return exclusive_scan_u32(H, in, out, m);
}

// ------------------------------------------------------------------------------------
// stable LSD radix sort, 8-bit digits
template <typename K>
__global__ void k_rs_hist(int64_t n, const K *__restrict__ keys, int shift, uint32_t *hist, int nblocks)
{
    __shared__ uint32_t sh[256];
    sh[threadIdx.x] = 0;
    __syncthreads();
    int64_t base = (int64_t)blockIdx.x * RS_TILE;
    for (int k = 0; k < RS_ITEMS; ++k) {
        int64_t i = base + k * RS_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&sh[(unsigned)(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * nblocks + blockIdx.x] = sh[threadIdx.x];
}

// Each warp owns 512 consecutive keys of the tile and ranks them in order, 32 at a time,
// with __match_any_sync; per-warp digit counts are then prefix-summed across warps, so the
// output position of every key preserves the input order among equal digits (stability).
template <typename K>
__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(int64_t n, const K *__restrict__ kin,
                                                          const uint32_t *__restrict__ vin, K *kout, uint32_t *vout,
                                                          int shift, const uint32_t *__restrict__ offs, int nblocks)
{
    __shared__ uint32_t wcnt[RS_WARPS][256];
    __shared__ uint32_t boff[256];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = threadIdx.x; k < RS_WARPS * 256; k += RS_THREADS) (&wcnt[0][0])[k] = 0;
    boff[threadIdx.x] = offs[(int64_t)threadIdx.x * nblocks + blockIdx.x];
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    K key[RS_ITEMS];
    uint32_t val[RS_ITEMS], rank[RS_ITEMS];
    int64_t base = (int64_t)blockIdx.x * RS_TILE + w * (RS_TILE / RS_WARPS);
#pragma unroll
    for (int c = 0; c < RS_ITEMS; ++c) {
        int64_t i = base + c * 32 + lane;
        bool valid = i < n;
        key[c] = valid ? kin[i] : K(0);
        val[c] = valid ? vin[i] : 0u;
        unsigned d = (unsigned)(key[c] >> shift) & 255u;
        unsigned mask = __ballot_sync(0xffffffffu, valid);
        unsigned peers = 0;
        if (valid) {
            peers = __match_any_sync(mask, d);
            rank[c] = wcnt[w][d] + __popc(peers & lt);
        }
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) wcnt[w][d] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {
        uint32_t run = 0;
        for (int ww = 0; ww < RS_WARPS; ++ww) {
            uint32_t t = wcnt[ww][threadIdx.x];
            wcnt[ww][threadIdx.x] = run;
            run += t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < RS_ITEMS; ++c) {
        int64_t i = base + c * 32 + lane;
        if (i < n) {
            unsigned d = (unsigned)(key[c] >> shift) & 255u;
            uint32_t pos = boff[d] + wcnt[w][d] + rank[c];
            if (pos < (uint64_t)n) {   // always true for consistent offsets; never write out of bounds
                kout[pos] = key[c];
                vout[pos] = val[c];
            }
        }
    }
}

template <typename K>
static cudaError_t sort_pairs(Handle *H, K *keys, uint32_t *vals, K *kalt, uint32_t *valt, int64_t n, int bits)
{
    if (n <= 1) return cudaSuccess;
    int nblocks = (int)((n + RS_TILE - 1) / RS_TILE);
    int64_t m = (int64_t)256 * nblocks;
    cudaError_t e = H->hist.reserve(sizeof(uint32_t) * 2 * m);
    if (e) return e;
    uint32_t *hist = H->hist.as<uint32_t>();
    uint32_t *offs = hist + m;
    K *src = keys, *dst = kalt;
    uint32_t *vs = vals, *vd = valt;
    int passes = (bits + 7) / 8;
    for (int p = 0; p < passes; ++p) {
        int shift = 8 * p;
        k_rs_hist<K><<<nblocks, RS_THREADS, 0, H->stream>>>(n, src, shift, hist, nblocks);
        H->launches += 1;
        e = exclusive_scan_u32(H, hist, offs, m);
        if (e) return e;
        k_rs_scatter<K><<<nblocks, RS_THREADS, 0, H->stream>>>(n, src, vs, dst, vd, shift, offs, nblocks);
        H->launches += 1;
        K *tk = src; src = dst; dst = tk;
        uint32_t *tv = vs; vs = vd; vd = tv;
    }
    if (src != keys) {
        cudaMemcpyAsync(keys, src, sizeof(K) * n, cudaMemcpyDeviceToDevice, H->stream);
        cudaMemcpyAsync(vals, vs, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, H->stream);
    }
    return cudaGetLastError();
}

cudaError_t sort_pairs_u64(Handle *H, uint64_t *keys, uint32_t *vals, uint64_t *kalt, uint32_t *valt, int64_t n,
                           int bits)
{
    return sort_pairs<uint64_t>(H, keys, vals, kalt, valt, n, bits);
}

cudaError_t sort_pairs_u32(Handle *H, uint32_t *keys, uint32_t *vals, uint32_t *kalt, uint32_t *valt, int64_t n,
                           int bits)
{
    return sort_pairs<uint32_t>(H, keys, vals, kalt, valt, n, bits);
}

// ------------------------------------------------------------------------------------
// duplicate bump as an inclusive max-scan of d[i] = c[i] - i
constexpr int DD_THREADS = 1024, DD_ITEMS = 8, DD_CHUNK = DD_THREADS * DD_ITEMS;

__device__ __forceinline__ int64_t block_inclusive_max(int64_t v, int64_t *total)
{
    __shared__ int64_t ws[32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int64_t inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        int64_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o && t > inc) inc = t;
    }
    if (lane == 31) ws[w] = inc;
    __syncthreads();
    if (w == 0) {
        int64_t s = lane < nw ? ws[lane] : INT64_MIN;
        for (int o = 1; o < 32; o <<= 1) {
            int64_t t = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o && t > s) s = t;
        }
        ws[lane] = s;
    }
    __syncthreads();
    int64_t r = inc;
    if (w > 0 && ws[w - 1] > r) r = ws[w - 1];
    if (total) *total = ws[nw - 1];
    __syncthreads();
    return r;
}

__global__ void k_dd_partial(int64_t n, const uint64_t *__restrict__ c, int64_t *part)
{
    int64_t base = (int64_t)blockIdx.x * DD_CHUNK;
    int64_t mx = INT64_MIN;
    for (int k = 0; k < DD_ITEMS; ++k) {
        int64_t i = base + k * DD_THREADS + threadIdx.x;
        if (i < n) {
            int64_t d = (int64_t)c[i] - i;
            if (d > mx) mx = d;
        }
    }
    int64_t tot;
    block_inclusive_max(mx, &tot);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

__global__ void k_dd_scan(int np, int64_t *part)
{
    // exclusive max-scan over chunk maxima (carry into each chunk)
    int64_t carry = INT64_MIN;
    for (int base = 0; base < np; base += DD_THREADS) {
        int i = base + threadIdx.x;
        int64_t v = i < np ? part[i] : INT64_MIN;
        int64_t tot;
        int64_t inc = block_inclusive_max(v, &tot);
        int64_t prev = __shfl_up_sync(0xffffffffu, inc, 1);
        __shared__ int64_t wlast[32];
        int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (lane == 31) wlast[w] = inc;
        __syncthreads();
        int64_t ex = (lane > 0) ? prev : (w > 0 ? wlast[w - 1] : INT64_MIN);
        if (carry > ex) ex = carry;
        __syncthreads();
        if (i < np) part[i] = ex;
        if (tot > carry) carry = tot;
    }
}

__global__ void k_dd_apply(int64_t n, uint64_t *c, const int64_t *__restrict__ carry)
{
    int64_t base = (int64_t)blockIdx.x * DD_CHUNK + (int64_t)threadIdx.x * DD_ITEMS;
    int64_t d[DD_ITEMS];
    int64_t run = INT64_MIN;
#pragma unroll
    for (int k = 0; k < DD_ITEMS; ++k) {
        int64_t i = base + k;
        d[k] = i < n ? (int64_t)c[i] - i : INT64_MIN;
        if (d[k] > run) run = d[k];
        d[k] = run;   // inclusive within the thread
    }
    // exclusive prefix of thread maxima
    int64_t inc = block_inclusive_max(run, nullptr);
    int64_t prev = __shfl_up_sync(0xffffffffu, inc, 1);
    __shared__ int64_t wl[32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 31) wl[w] = inc;
    __syncthreads();
    int64_t ex = (lane > 0) ? prev : (w > 0 ? wl[w - 1] : INT64_MIN);
    int64_t cin = carry[blockIdx.x];
    if (cin > ex) ex = cin;
#pragma unroll
    for (int k = 0; k < DD_ITEMS; ++k) {
        int64_t i = base + k;
        if (i < n) {
            int64_t v = d[k] > ex ? d[k] : ex;
            c[i] = (uint64_t)v + (uint64_t)i;
        }
    }
}

cudaError_t launch_dedupe(Handle *H, uint64_t *codes, int64_t n)
{
    if (n <= 1) return cudaSuccess;
    int nb = (int)((n + DD_CHUNK - 1) / DD_CHUNK);
    cudaError_t e = H->scan_tmp.reserve(sizeof(int64_t) * (nb + 1));
    if (e) return e;
    int64_t *part = H->scan_tmp.as<int64_t>();
    k_dd_partial<<<nb, DD_THREADS, 0, H->stream>>>(n, codes, part);
    k_dd_scan<<<1, DD_THREADS, 0, H->stream>>>(nb, part);
    k_dd_apply<<<nb, DD_THREADS, 0, H->stream>>>(n, codes, part);
    H->launches += 3;
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// permuted leaves and particle columns
__global__ void k_gather(int64_t n, const uint32_t *__restrict__ idx, const double *__restrict__ x,
                         const double *__restrict__ y, const double *__restrict__ z, const double *__restrict__ h,
                         const double *__restrict__ m, const double *__restrict__ rho, double4 *leaf, double *ms,
                         double *rhos)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t o = idx[i];
        if (o >= (uint64_t)n) o = 0;   // unreachable for a valid permutation; keeps reads in bounds
        leaf[i] = make_double4(x[o], y[o], z[o], h[o]);
        ms[i] = m[o];
        rhos[i] = rho[o];
    }
}

__global__ void k_gather_col(int64_t n, const uint32_t *__restrict__ idx, const double *__restrict__ src, double *dst)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t o = idx[i];
        dst[i] = src[o < (uint64_t)n ? o : 0];
    }
}

cudaError_t launch_gather(Handle *H, int64_t n, const double *x, const double *y, const double *z, const double *h,
                          const double *m, const double *rho, const std::vector<const double *> &cols)
{
    const uint32_t *idx = H->idx.as<uint32_t>();
    k_gather<<<grid_for(n, 256), 256, 0, H->stream>>>(n, idx, x, y, z, h, m, rho, H->leaf.as<double4>(),
                                                       H->m_s.as<double>(), H->rho_s.as<double>());
    H->launches += 1;
    for (size_t c = 0; c < cols.size(); ++c) {
        k_gather_col<<<grid_for(n, 256), 256, 0, H->stream>>>(n, idx, cols[c], H->cols_s[c].as<double>());
        H->launches += 1;
    }
    return cudaGetLastError();
}

__global__ void k_permute_back(int64_t n, const uint32_t *__restrict__ idx, const double *__restrict__ src, double *dst)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t o = idx[i];
        dst[i] = src[o < (uint64_t)n ? o : 0];
    }
}

cudaError_t launch_permute_back(Handle *H, int64_t n, const uint32_t *idx, const double *src, double *dst)
{
    k_permute_back<<<grid_for(n, 256), 256, 0, H->stream>>>(n, idx, src, dst);
    H->launches += 1;
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// Karras topology (1-based, unified ids) with internal escapes
__device__ __forceinline__ int lcp(const uint64_t *__restrict__ c1, int64_t i, int64_t j)
{
    uint64_t a = c1[i], b = c1[j];
    uint64_t x = (a == b) ? ((uint64_t)i ^ (uint64_t)j) : (a ^ b);
    return x == 0 ? 64 : __clzll((long long)x);
}

__global__ void k_karras(int64_t n, const uint64_t *__restrict__ codes, int *left, int *right, int *parent,
                         int *escape, int2 *child, int2 *range)
{
    const uint64_t *c1 = codes - 1;
    const int64_t off = n - 1;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n - 1; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = t + 1;
        // _range_direction / _find_range (BinaryRadixTree.jl:140-179)
        int dL = (i > 1) ? lcp(c1, i, i - 1) : -1;
        int dR = (i < n) ? lcp(c1, i, i + 1) : -1;
        int64_t d = (dR - dL >= 0) ? 1 : -1;
        int dmin = (1 <= i - d && i - d <= n) ? lcp(c1, i, i - d) : -1;
        int64_t lmax = 2;
        for (;;) {
            int64_t j = i + lmax * d;
            if (j < 1 || j > n) break;
            if (lcp(c1, i, j) <= dmin) break;
            lmax *= 2;
        }
        int64_t l = 0;
        for (int64_t s = lmax >> 1; s > 0; s >>= 1) {
            int64_t j = i + (l + s) * d;
            if (j >= 1 && j <= n && lcp(c1, i, j) > dmin) l += s;
        }
        int64_t j = i + l * d;
        int64_t lo = i < j ? i : j, hi = i < j ? j : i;
        // _split_position (BinaryRadixTree.jl:181-202)
        int64_t split;
        if (c1[lo] == c1[hi]) {
            split = (lo + hi) >> 1;
            if (split < lo) split = lo;
            if (split > hi - 1) split = hi - 1;
        } else {
            int pfl = lcp(c1, lo, hi);
            split = lo;
            int64_t step = hi - lo;
            while (step > 1) {
                step = (step + 1) >> 1;
                int64_t ns = split + step;
                if (ns < hi && lcp(c1, lo, ns) > pfl) split = ns;
            }
        }
        int64_t li = (split == lo) ? lo + off : split;
        int64_t ri = (split + 1 == hi) ? hi + off : split + 1;
        left[i - 1] = (int)li;
        right[i - 1] = (int)ri;
        child[i - 1] = make_int2((int)li, (int)ri);
        range[i - 1] = make_int2((int)(lo - 1), (int)(hi - 1));   // 0-based sorted leaf range of the subtree
        parent[li - 1] = (int)i;
        parent[ri - 1] = (int)i;
        // internal escape (BinaryRadixTree.jl:245-260); adj[k] = lcp(k, k+1), adj[n] = +inf
        int e;
        if (hi == n) e = 0;
        else if (hi == n - 1) e = (int)(off + n);
        else {
            int64_t nx = hi + 1;
            int anx = (nx < n) ? lcp(c1, nx, nx + 1) : 0x7fffffff;
            int apv = lcp(c1, nx - 1, nx);
            e = (anx < apv) ? (int)(off + nx) : (int)nx;
        }
        escape[i - 1] = e;
    }
}

// Leaf escapes (BinaryRadixTree.jl:262-281) and the Karras bottom-up refit with atomic
// second arrival (LinearBVH.jl:98-156).  Min/max are order independent, so the FP64
// boxes and hmax are bit-identical to a sequential refit.  Children written by other
// threads in this launch are read through L2 (__ldcg) after the acquiring fence.
__global__ void k_refit(int64_t n, const int *__restrict__ parent, const int *__restrict__ left,
                        const int *__restrict__ right, int *escape, const double4 *__restrict__ leaf, NodeF *node,
                        float *node_hmax, double *bmin, double *bmax, double *hmax, unsigned *counters,
                        int *leaf_escape, int *status)
{
    const int64_t nin = n - 1;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        int64_t id = n + k;
        int p = parent[id - 1];
        int e = 0;
        if (p != 0) e = (left[p - 1] == (int)id) ? right[p - 1] : escape[p - 1];
        leaf_escape[k] = e;
        escape[id - 1] = e;
        int64_t depth = 0;
        while (p != 0) {
            // a valid tree has depth < n and ids in range; anything else is reported, not followed
            if (++depth > n || p < 0 || p > nin) { atomicOr(status, ST_REFIT); break; }
            __threadfence();
            unsigned old = atomicAdd(&counters[p - 1], 1u);
            if (old == 0) break;
            __threadfence();
            int l = left[p - 1], r = right[p - 1];
            if (l < 1 || l > 2 * n - 1 || r < 1 || r > 2 * n - 1) { atomicOr(status, ST_REFIT); break; }
            double lmn[3], lmx[3], rmn[3], rmx[3], hl, hr;
            if (l >= n) {
                double4 L = leaf[l - n];
                lmn[0] = lmx[0] = L.x; lmn[1] = lmx[1] = L.y; lmn[2] = lmx[2] = L.z; hl = L.w;
            } else {
                for (int d = 0; d < 3; ++d) { lmn[d] = __ldcg(&bmin[d * nin + l - 1]); lmx[d] = __ldcg(&bmax[d * nin + l - 1]); }
                hl = __ldcg(&hmax[l - 1]);
            }
            if (r >= n) {
                double4 R = leaf[r - n];
                rmn[0] = rmx[0] = R.x; rmn[1] = rmx[1] = R.y; rmn[2] = rmx[2] = R.z; hr = R.w;
            } else {
                for (int d = 0; d < 3; ++d) { rmn[d] = __ldcg(&bmin[d * nin + r - 1]); rmx[d] = __ldcg(&bmax[d * nin + r - 1]); }
                hr = __ldcg(&hmax[r - 1]);
            }
            double hm = (hl > hr) ? hl : hr;
            double mn[3], mx[3];
            for (int d = 0; d < 3; ++d) {
                mn[d] = (lmn[d] < rmn[d]) ? lmn[d] : rmn[d];
                mx[d] = (lmx[d] > rmx[d]) ? lmx[d] : rmx[d];
                bmin[d * nin + p - 1] = mn[d];
                bmax[d * nin + p - 1] = mx[d];
            }
            hmax[p - 1] = hm;
            NodeF nd;
            nd.lox = __double2float_rd(mn[0]); nd.loy = __double2float_rd(mn[1]); nd.loz = __double2float_rd(mn[2]);
            nd.hix = __double2float_ru(mx[0]); nd.hiy = __double2float_ru(mx[1]); nd.hiz = __double2float_ru(mx[2]);
            nd.left = l;
            nd.escape = escape[p - 1];
            node[p - 1] = nd;
            node_hmax[p - 1] = __double2float_ru(hm);
            p = parent[p - 1];
        }
    }
}

__global__ void k_check_counters(int64_t nin, const unsigned *__restrict__ counters, int *status)
{
    int bad = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nin; i += (int64_t)gridDim.x * blockDim.x)
        if (counters[i] != 2u) bad = 1;
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(status, ST_REFIT);
}

cudaError_t launch_topology(Handle *H, int64_t n)
{
    if (n < 2) {
        cudaMemsetAsync(H->escape.p, 0, sizeof(int), H->stream);
        cudaMemsetAsync(H->parent.p, 0, sizeof(int), H->stream);
        cudaMemsetAsync(H->leaf_escape.p, 0, sizeof(int), H->stream);
        return cudaGetLastError();
    }
    int64_t ntot = 2 * n - 1;
    cudaMemsetAsync(H->parent.p, 0, sizeof(int) * ntot, H->stream);
    cudaMemsetAsync(H->counters.p, 0, sizeof(unsigned) * (n - 1), H->stream);
    k_karras<<<grid_for(n - 1, 256), 256, 0, H->stream>>>(n, H->codes.as<uint64_t>(), H->left.as<int>(),
                                                          H->right.as<int>(), H->parent.as<int>(), H->escape.as<int>(),
                                                          H->node_child.as<int2>(), H->node_range.as<int2>());
    k_refit<<<grid_for(n, 256, 1 << 30), 256, 0, H->stream>>>(
        n, H->parent.as<int>(), H->left.as<int>(), H->right.as<int>(), H->escape.as<int>(), H->leaf.as<double4>(),
        H->node.as<NodeF>(), H->node_hmax.as<float>(), H->bmin64.as<double>(), H->bmax64.as<double>(),
        H->hmax64.as<double>(), H->counters.as<unsigned>(), H->leaf_escape.as<int>(), H->status.as<int>());
    k_check_counters<<<grid_for(n - 1, 256), 256, 0, H->stream>>>(n - 1, H->counters.as<unsigned>(),
                                                                  H->status.as<int>());
    H->launches += 3;
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// Morton order of query points (schedule only: outputs are written back to their own slot)
// 30-bit Morton code of a sample point in a tree's quantisation frame (10 bits per axis,
// clamped to the particles' box): only an ordering key, not the build's codes
__device__ __forceinline__ uint32_t query_code30(const QuantParams &q, double x, double y, double z)
{
    const double p[3] = {x, y, z};
    uint32_t c[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double f = q.flat[d] ? 0.5 : (p[d] - q.vmin[d]) * q.inv[d];
        f = fmin(fmax(f, 0.0), 1.0);
        if (!(f == f)) f = 0.0;
        c[d] = (uint32_t)(f * 1023.0);
    }
    return ((uint32_t)expand_bits3(c[0]) << 2) | ((uint32_t)expand_bits3(c[1]) << 1) | (uint32_t)expand_bits3(c[2]);
}

__global__ void k_query_codes(int64_t nq, const double *__restrict__ qx, const double *__restrict__ qy,
                              const double *__restrict__ qz, const QuantParams *__restrict__ qp, uint32_t *keys,
                              uint32_t *perm)
{
    const QuantParams q = *qp;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nq; i += (int64_t)gridDim.x * blockDim.x) {
        keys[i] = query_code30(q, qx[i], qy[i], qz[i]);
        perm[i] = (uint32_t)i;
    }
}

__global__ void k_batch_query_codes(int64_t m, const BatchDisc *__restrict__ discs, const int64_t *__restrict__ starts,
                                    const uint32_t *__restrict__ slot_disc, const int *__restrict__ slot_of,
                                    int64_t s0, uint64_t *keys, uint32_t *vals)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
        const int lo = slot_of[t];
        const BatchDisc &D = discs[slot_disc[lo]];
        const int64_t qi = s0 + t - starts[lo];
        keys[t] = ((uint64_t)(uint32_t)lo << 32) | query_code30(*D.qp, D.qx[qi], D.qy[qi], D.qz[qi]);
        vals[t] = (uint32_t)t;
    }
}

cudaError_t launch_batch_query_codes(Handle *H, int64_t m, const BatchDisc *discs, const int64_t *starts,
                                     const uint32_t *slot_disc, const int *slot_of, int64_t s0, uint64_t *keys,
                                     uint32_t *vals)
{
    k_batch_query_codes<<<grid_for(m, 256), 256, 0, H->stream>>>(m, discs, starts, slot_disc, slot_of, s0, keys, vals);
    H->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_query_codes(Handle *H, int64_t nq, const double *qx, const double *qy, const double *qz,
                               uint32_t *keys, uint32_t *perm)
{
    k_query_codes<<<grid_for(nq, 256), 256, 0, H->stream>>>(nq, qx, qy, qz, H->qparams.as<QuantParams>(), keys, perm);
    H->launches += 1;
    return cudaGetLastError();
}

}  // namespace pb
