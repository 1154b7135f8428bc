// pb_noalloc.cu -- pb_morton_sort_noalloc: the Morton encode + stable radix sort + duplicate
// bump of the LBVH build, for callers that cannot allocate device memory.
//
// Who needs it: an application that owns all device memory through its own pool (and
// forbids allocations behind its back), or a caller that cannot afford the device-wide
// synchronisation that cudaMalloc/cudaFree can imply in the middle of its own pipeline.
// The regular entry points keep grow-only scratch buffers per handle and may call
// cudaMalloc; this one calls no allocator at all.  Its sort scratch (the second key and
// both index buffers, per-block digit histograms and their offsets, a status word) lives
// in one file-scope static __device__ array of fixed size, which every GPU that loads the
// library holds until the process exits.
//
// Limits and sharing rules:
//   * n <= PB_NOALLOC_MAX_N (262,144 particles); larger n is rejected with PB_ERR_CAPACITY.
//   * All calls share the one scratch array per device and it keeps the last call's
//     contents; every buffer a call reads is written by that call first (the status word
//     is cleared at the start).  Calls whose GPU work overlaps -- two streams, two host
//     threads, or one call launched while another is still running -- race on the
//     scratch array and give undefined results.  Serialise them.
//   * The first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current); make that first
//     call before any stream capture is started on the device.
//   * Inputs and outputs are device pointers of the current device, supplied by the caller.
//   * A CUDA error still pending from the caller's own earlier work makes the call return
//     PB_ERR_CUDA before it launches anything; the error is left for the caller to read.
#include <cstdint>
#include <mutex>

#include <cuda_runtime.h>

#include "partia_b200.h"

namespace {

constexpr int64_t NA_MAX_N = PB_NOALLOC_MAX_N;
constexpr int NA_THREADS = 256;
constexpr int NA_ITEMS = 16;
constexpr int NA_TILE = NA_THREADS * NA_ITEMS;                  // keys per sort block
constexpr int NA_MAX_BLOCKS = (int)(NA_MAX_N / NA_TILE);        // 64
constexpr int NA_WARPS = NA_THREADS / 32;

// byte offsets inside the scratch array (all 256-byte aligned)
constexpr size_t OFF_KEYS = 0;                                           // uint64 [MAX_N]
constexpr size_t OFF_VALS = OFF_KEYS + 8 * NA_MAX_N;                     // uint32 [MAX_N]
constexpr size_t OFF_VALS_ALT = OFF_VALS + 4 * NA_MAX_N;                 // uint32 [MAX_N]
constexpr size_t OFF_HIST = OFF_VALS_ALT + 4 * NA_MAX_N;                 // uint32 [256*MAX_BLOCKS]
constexpr size_t OFF_OFFS = OFF_HIST + 4 * 256 * NA_MAX_BLOCKS;          // uint32 [256*MAX_BLOCKS]
constexpr size_t OFF_QUANT = OFF_OFFS + 4 * 256 * NA_MAX_BLOCKS;         // double vmin[3], inv[3]; int flat[3]
constexpr size_t OFF_STATUS = OFF_QUANT + 256;                           // int
constexpr size_t SCRATCH_BYTES = OFF_STATUS + 256;                       // ~6.3 MB

static __device__ __align__(256) unsigned char g_noalloc_scratch[SCRATCH_BYTES];

struct QP {
    double vmin[3];
    double inv[3];
    int flat[3];
};

// per-axis min/max in one block (order independent: exact comparisons), reduced with warp
// shuffles and one value per warp in shared memory, then the quantisation parameters of
// MortonCode.jl:443-456; non-finite coordinates set the status word
__global__ void k_na_bbox(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                          const double *__restrict__ z, QP *qp, int *status)
{
    __shared__ double smin[3][32], smax[3][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = (blockDim.x + 31) >> 5;
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    int bad = 0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        double v[3] = {x[i], y[i], z[i]};
        for (int d = 0; d < 3; ++d) {
            if (!isfinite(v[d])) bad = 1;
            if (v[d] < mn[d]) mn[d] = v[d];
            if (v[d] > mx[d]) mx[d] = v[d];
        }
    }
    if (bad) atomicOr(status, 1);
    for (int off = 16; off > 0; off >>= 1)
        for (int d = 0; d < 3; ++d) {
            const double a = __shfl_xor_sync(0xffffffffu, mn[d], off), b = __shfl_xor_sync(0xffffffffu, mx[d], off);
            if (a < mn[d]) mn[d] = a;
            if (b > mx[d]) mx[d] = b;
        }
    if (lane == 0)
        for (int d = 0; d < 3; ++d) { smin[d][warp] = mn[d]; smax[d][warp] = mx[d]; }
    __syncthreads();
    if (warp != 0) return;
    for (int d = 0; d < 3; ++d) {
        mn[d] = lane < nwarps ? smin[d][lane] : INFINITY;
        mx[d] = lane < nwarps ? smax[d][lane] : -INFINITY;
    }
    for (int off = 16; off > 0; off >>= 1)
        for (int d = 0; d < 3; ++d) {
            const double a = __shfl_xor_sync(0xffffffffu, mn[d], off), b = __shfl_xor_sync(0xffffffffu, mx[d], off);
            if (a < mn[d]) mn[d] = a;
            if (b > mx[d]) mx[d] = b;
        }
    if (lane == 0)
        for (int d = 0; d < 3; ++d) {
            const double dv = mx[d] - mn[d];
            qp->vmin[d] = mn[d];
            qp->flat[d] = (dv == 0.0);
            qp->inv[d] = (dv == 0.0) ? 0.0 : 1.0 / dv;
        }
}

__device__ __forceinline__ uint64_t na_expand(uint64_t v)
{
    v = (v | (v << 32)) & 0x1f00000000ffffULL;
    v = (v | (v << 16)) & 0x1f0000ff0000ffULL;
    v = (v | (v << 8)) & 0x100f00f00f00f00fULL;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ULL;
    v = (v | (v << 2)) & 0x1249249249249249ULL;
    return v;
}

__device__ __forceinline__ uint64_t na_quant(double v, double vmin, double inv, int flat)
{
    double f = flat ? 0.5 : __dmul_rn(__dsub_rn(v, vmin), inv);
    return (uint64_t)floor(__dmul_rn(2097151.0, f));
}

__global__ void k_na_encode(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                            const double *__restrict__ z, const QP *__restrict__ qp, uint64_t *keys, uint32_t *vals)
{
    QP q = *qp;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        keys[i] = (na_expand(na_quant(x[i], q.vmin[0], q.inv[0], q.flat[0])) << 2) |
                  (na_expand(na_quant(y[i], q.vmin[1], q.inv[1], q.flat[1])) << 1) |
                  na_expand(na_quant(z[i], q.vmin[2], q.inv[2], q.flat[2]));
        vals[i] = (uint32_t)i;
    }
}

__global__ void k_na_hist(int64_t n, const uint64_t *__restrict__ keys, int shift, uint32_t *hist, int nblocks)
{
    __shared__ uint32_t sh[256];
    sh[threadIdx.x] = 0;
    __syncthreads();
    int64_t base = (int64_t)blockIdx.x * NA_TILE;
    for (int k = 0; k < NA_ITEMS; ++k) {
        int64_t i = base + k * NA_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&sh[(unsigned)(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * nblocks + blockIdx.x] = sh[threadIdx.x];
}

// exclusive scan of the digit-major histogram (at most 256 * 64 entries) in one block
__global__ void k_na_scan(int m, const uint32_t *__restrict__ hist, uint32_t *offs)
{
    __shared__ uint32_t part[1024];
    const int per = (m + 1023) / 1024;
    int b0 = threadIdx.x * per;
    uint32_t s = 0;
    for (int k = 0; k < per; ++k)
        if (b0 + k < m) s += hist[b0 + k];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        uint32_t v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = part[threadIdx.x] - s;
    for (int k = 0; k < per; ++k)
        if (b0 + k < m) {
            offs[b0 + k] = run;
            run += hist[b0 + k];
        }
}

// stable scatter: each warp ranks its 512 consecutive keys in order (match_any), warp
// counts are prefix-summed across warps so equal digits keep their input order
__global__ void k_na_scatter(int64_t n, const uint64_t *__restrict__ kin, const uint32_t *__restrict__ vin,
                             uint64_t *kout, uint32_t *vout, int shift, const uint32_t *__restrict__ offs, int nblocks)
{
    __shared__ uint32_t wcnt[NA_WARPS][256];
    __shared__ uint32_t boff[256];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = threadIdx.x; k < NA_WARPS * 256; k += NA_THREADS) (&wcnt[0][0])[k] = 0;
    boff[threadIdx.x] = offs[threadIdx.x * nblocks + blockIdx.x];
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    uint64_t key[NA_ITEMS];
    uint32_t val[NA_ITEMS], rank[NA_ITEMS];
    int64_t base = (int64_t)blockIdx.x * NA_TILE + w * (NA_TILE / NA_WARPS);
    for (int c = 0; c < NA_ITEMS; ++c) {
        int64_t i = base + c * 32 + lane;
        bool valid = i < n;
        key[c] = valid ? kin[i] : 0;
        val[c] = valid ? vin[i] : 0;
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
        for (int ww = 0; ww < NA_WARPS; ++ww) {
            uint32_t t = wcnt[ww][threadIdx.x];
            wcnt[ww][threadIdx.x] = run;
            run += t;
        }
    }
    __syncthreads();
    for (int c = 0; c < NA_ITEMS; ++c) {
        int64_t i = base + c * 32 + lane;
        if (i < n) {
            unsigned d = (unsigned)(key[c] >> shift) & 255u;
            uint32_t pos = boff[d] + wcnt[w][d] + rank[c];
            if (pos < (uint64_t)n) {
                kout[pos] = key[c];
                vout[pos] = val[c];
            }
        }
    }
}

// duplicate bump c'[i] = i + max_{j<=i}(c[j] - j) (MortonCode.jl:189-193) in one block,
// then the 0-based order as int64
__global__ void k_na_dedupe(int64_t n, uint64_t *keys, const uint32_t *__restrict__ vals, int64_t *order)
{
    __shared__ int64_t part[1024];
    const int64_t per = (n + 1023) / 1024;
    int64_t b0 = threadIdx.x * per;
    int64_t run = INT64_MIN;
    for (int64_t k = 0; k < per && b0 + k < n; ++k) {
        int64_t d = (int64_t)keys[b0 + k] - (b0 + k);
        if (d > run) run = d;
    }
    part[threadIdx.x] = run;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        int64_t v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : INT64_MIN;
        __syncthreads();
        if (v > part[threadIdx.x]) part[threadIdx.x] = v;
        __syncthreads();
    }
    int64_t carry = threadIdx.x > 0 ? part[threadIdx.x - 1] : INT64_MIN;
    for (int64_t k = 0; k < per && b0 + k < n; ++k) {
        int64_t i = b0 + k;
        int64_t d = (int64_t)keys[i] - i;
        if (d > carry) carry = d;
        keys[i] = (uint64_t)carry + (uint64_t)i;
        order[i] = (int64_t)vals[i];
    }
}

// The GPU a pointer's memory belongs to: its device id for device memory, -2 for managed
// memory (usable from any device), -1 for host memory or an unknown pointer.
int device_of(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    if (a.type == cudaMemoryTypeManaged) return -2;
    return a.type == cudaMemoryTypeDevice ? a.device : -1;
}

std::mutex g_setup_mutex;
unsigned char *g_scratch_ptr[64] = {};

}  // namespace

extern "C" int32_t pb_morton_sort_noalloc(const double *x, const double *y, const double *z, int64_t n,
                                          uint64_t *codes_out, int64_t *order_out, void *cuda_stream)
{
    if (n < 1 || !x || !y || !z || !codes_out || !order_out) return PB_ERR_INVALID;
    if (n > NA_MAX_N) return PB_ERR_CAPACITY;
    const void *ptrs[5] = {x, y, z, codes_out, order_out};
    int owner[5];
    for (int k = 0; k < 5; ++k)
        if ((owner[k] = device_of(ptrs[k])) == -1) return PB_ERR_INVALID;   // host memory
    // an error still pending from the caller's earlier work is left in place for the caller
    // and reported before any launch, so that it is not taken for one of this call's
    if (cudaPeekAtLastError() != cudaSuccess) return PB_ERR_CUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return PB_ERR_CUDA;
    // memory of another GPU is refused: the kernels would read it without peer access
    for (int k = 0; k < 5; ++k)
        if (owner[k] >= 0 && owner[k] != dev) return PB_ERR_INVALID;
    unsigned char *base;
    {
        // once per device, with that device current: the device address of the static array
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_ptr[dev]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
                cudaGetLastError();
                return PB_ERR_CUDA;
            }
            g_scratch_ptr[dev] = static_cast<unsigned char *>(p);
        }
        base = g_scratch_ptr[dev];
    }
    cudaStream_t s = (cudaStream_t)cuda_stream;
    uint64_t *keys_alt = reinterpret_cast<uint64_t *>(base + OFF_KEYS);
    uint32_t *vals = reinterpret_cast<uint32_t *>(base + OFF_VALS);
    uint32_t *vals_alt = reinterpret_cast<uint32_t *>(base + OFF_VALS_ALT);
    uint32_t *hist = reinterpret_cast<uint32_t *>(base + OFF_HIST);
    uint32_t *offs = reinterpret_cast<uint32_t *>(base + OFF_OFFS);
    QP *qp = reinterpret_cast<QP *>(base + OFF_QUANT);
    int *status = reinterpret_cast<int *>(base + OFF_STATUS);

    if (cudaMemsetAsync(status, 0, sizeof(int), s) != cudaSuccess) return PB_ERR_CUDA;
    k_na_bbox<<<1, 1024, 0, s>>>(n, x, y, z, qp, status);
    k_na_encode<<<(int)((n + 255) / 256), 256, 0, s>>>(n, x, y, z, qp, codes_out, vals);
    int nblocks = (int)((n + NA_TILE - 1) / NA_TILE);
    uint64_t *ka = codes_out, *kb = keys_alt;
    uint32_t *va = vals, *vb = vals_alt;
    for (int pass = 0; pass < 8; ++pass) {   // 8 even passes: the result ends in codes_out/vals
        k_na_hist<<<nblocks, NA_THREADS, 0, s>>>(n, ka, 8 * pass, hist, nblocks);
        k_na_scan<<<1, 1024, 0, s>>>(256 * nblocks, hist, offs);
        k_na_scatter<<<nblocks, NA_THREADS, 0, s>>>(n, ka, va, kb, vb, 8 * pass, offs, nblocks);
        uint64_t *tk = ka; ka = kb; kb = tk;
        uint32_t *tv = va; va = vb; vb = tv;
    }
    k_na_dedupe<<<1, 1024, 0, s>>>(n, codes_out, vals, order_out);
    if (cudaGetLastError() != cudaSuccess) return PB_ERR_CUDA;
    int st = 0;
    if (cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return PB_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PB_ERR_CUDA;
    return st ? PB_ERR_INVALID : PB_OK;
}
