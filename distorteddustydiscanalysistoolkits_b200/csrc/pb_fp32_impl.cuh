// pb_fp32_impl.cuh -- the FP32-compensated per-pair arithmetic: kernel shapes, the particle
// payload, the FP32 chunk sums with FP64 accumulation and the finalisation, and the fused
// per-query body (warp-uniform walk + dealing + sums).  Shared by pb_interp32.cu and the batched
// kernel (pb_batch.cu); both units are compiled with -fmad=false, so a query's bits do not
// depend on which kernel summed it.
#pragma once
#include "pb_interp_impl.cuh"

namespace pb {

constexpr int CHUNK = 32;
static_assert(CHUNK % 4 == 0, "groups of two or four batches must not straddle a flush");

// ---- kernel shapes f(q), f'(q) for q >= 0 (kernels/*.jl) in FP32 ----
// Algebraically identical to the reference's piecewise forms but arranged so that nothing
// cancels near q = 0 (where f'(q) -> 0): the innermost piece of every spline and every
// Wendland derivative is expanded into a polynomial with an explicit factor q, e.g. M4
// f'(q) = -0.75 (2-q)^2 + 3 (1-q)^2 = q (2.25 q - 3) for q < 1, and C4
// f'(q) = t^5 (t (35/6 q + 3) - (35/4 q^2 + 9 q + 3)) = -(14/3) q (1 + 2.5 q) t^5, t = 1 - q/2.
// Pieces are chosen with selects, so lanes never diverge.
template <int KT>
__device__ __forceinline__ void shape(float q, float &f, float &df)
{
    if (KT == 0) {   // M4
        const float a = fmaxf(2.f - q, 0.f), a2 = a * a;
        const float fi = fmaf(q * q, fmaf(0.75f, q, -1.5f), 1.f), di = q * fmaf(2.25f, q, -3.f);
        const float fo = (0.25f * a2) * a, dO = -0.75f * a2;
        const bool in = q < 1.f;
        f = in ? fi : fo;
        df = in ? di : dO;
    } else if (KT == 1) {   // M5
        const float a = fmaxf(2.5f - q, 0.f), b = fmaxf(1.5f - q, 0.f), c = fmaxf(0.5f - q, 0.f);
        const float a2 = a * a, b2 = b * b, c2 = c * c;
        f = fmaf(10.f * c2, c2, fmaf(-5.f * b2, b2, a2 * a2));
        const float di = q * fmaf(24.f, q * q, -30.f);
        const float dO = fmaf(20.f * b2, b, -4.f * a2 * a);
        df = q < 0.5f ? di : dO;
    } else if (KT == 2) {   // M6
        const float a = fmaxf(3.f - q, 0.f), b = fmaxf(2.f - q, 0.f), c = fmaxf(1.f - q, 0.f);
        const float a4 = (a * a) * (a * a), b4 = (b * b) * (b * b), c4 = (c * c) * (c * c);
        f = fmaf(15.f * c4, c, fmaf(-6.f * b4, b, a4 * a));
        const float di = q * fmaf(q * q, fmaf(-50.f, q, 120.f), -120.f);
        const float dO = fmaf(30.f, b4, -5.f * a4);
        df = q < 1.f ? di : dO;
    } else if (KT == 3) {   // C2
        const float t = fmaxf(fmaf(-0.5f, q, 1.f), 0.f);
        const float t3 = t * t * t;
        f = (t3 * t) * fmaf(2.f, q, 1.f);
        df = (-5.f * q) * t3;
    } else if (KT == 4) {   // C4
        const float t = fmaxf(fmaf(-0.5f, q, 1.f), 0.f);
        const float t5 = (t * t) * (t * t) * t;
        f = (t5 * t) * fmaf(fmaf(35.f / 12.f, q, 3.f), q, 1.f);
        df = ((-14.f / 3.f) * q) * fmaf(2.5f, q, 1.f) * t5;
    } else {   // C6
        const float t = fmaxf(fmaf(-0.5f, q, 1.f), 0.f);
        const float t7 = (t * t) * (t * t) * (t * t) * t;
        f = (t7 * t) * fmaf(fmaf(fmaf(4.f, q, 6.25f), q, 4.f), q, 1.f);
        df = (-5.5f * q) * fmaf(fmaf(4.f, q, 3.5f), q, 1.f) * t7;
    }
}

__device__ __forceinline__ float ldexp_norm3(int k)
{
    const float pi = 3.14159265358979f;
    switch (k) {
    case 0: return 1.f / pi;
    case 1: return 0.05f / pi;
    case 2: return 1.f / (120.f * pi);
    case 3: return 21.f / (16.f * pi);
    case 4: return 495.f / (256.f * pi);
    default: return 1365.f / (512.f * pi);
    }
}

// payload: record of `stride` float4 fields per sorted particle
//   [0] = {x_hi, y_hi, z_hi, 1/h}, [1] = {x_lo, y_lo, z_lo, m/rho}, [2..] = the (hi, lo) pairs of the
//   columns, two per field (64 bytes for four columns).  The kernel factors sigma h^-3 and
//   sigma h^-4 are formed from 1/h in the pair loop: four multiplies cost less than the load.  Coordinates are double-float pairs, so the pair
//   offset x_a - x_b is formed in FP32 as (xa_hi - xb_hi) + (xa_lo - xb_lo) without FP64 loads.
// Layout: blocks of 32 consecutive particles, field-major inside a block -- field k of particle
// b is float4 number ((b / 32) * stride + k) * 32 + b % 32.  The lanes of a warp read 32
// consecutive particles (the common case: a batch inside one accepted run), so every field
// load of the warp is one contiguous 512-byte segment.
__host__ __device__ inline int payload_stride(int nU) { return 2 + (2 * nU + 3) / 4; }
constexpr int PAY_BLOCK = 32;   // particles per payload block; field k is at rec[k * PAY_BLOCK]

__host__ __device__ inline int64_t payload_float4s(int64_t n, int stride)
{
    return ((n + PAY_BLOCK - 1) / PAY_BLOCK) * PAY_BLOCK * stride;
}

// field 0 of particle b's record (b < n <= 2^30: 32-bit index arithmetic, one wide multiply)
__device__ __forceinline__ const float4 *rec_of(const float4 *pay, int stride, uint32_t b)
{
    return pay + (uint64_t)(b >> 5) * (uint32_t)(stride * PAY_BLOCK) + (b & (PAY_BLOCK - 1));
}

// Compile-time shape of a launch's catalog, for the pair kernels.  CAT 0 reads everything from
// the DevCatalog at run time; 1: four columns, gradient + divergence + curl; 2: four columns,
// curl only; 3: one column, scalars only.  A specialised kernel performs exactly the
// operations, in the same order, that the generic one performs for such a catalog.
constexpr int CAT_ANY = 0, CAT_GDC4 = 1, CAT_C4 = 2, CAT_S1 = 3, CAT_SG1 = 4;   // SG1: one column, scalar + gradient

template <int CAT>
struct CatShape {
    __device__ static __forceinline__ int nu(const DevCatalog &C)
    {
        return (CAT == CAT_GDC4 || CAT == CAT_C4) ? 4 : ((CAT == CAT_S1 || CAT == CAT_SG1) ? 1 : C.nU);
    }
    __device__ static __forceinline__ bool grad(const DevCatalog &C)
    {
        return (CAT == CAT_GDC4 || CAT == CAT_SG1) ? true : (CAT == CAT_ANY ? C.n_grad > 0 : false);
    }
    __device__ static __forceinline__ bool div(const DevCatalog &C)
    {
        return CAT == CAT_GDC4 ? true : (CAT == CAT_ANY ? C.n_div > 0 : false);
    }
    __device__ static __forceinline__ bool curl(const DevCatalog &C)
    {
        return (CAT == CAT_GDC4 || CAT == CAT_C4) ? true : (CAT == CAT_ANY ? C.n_curl > 0 : false);
    }
    __device__ static __forceinline__ bool any(const DevCatalog &C) { return grad(C) || div(C) || curl(C); }
    __device__ static __forceinline__ int stride(int s)
    {
        return (CAT == CAT_GDC4 || CAT == CAT_C4) ? 4 : ((CAT == CAT_S1 || CAT == CAT_SG1) ? 3 : s);
    }
};

inline int catalog_shape(const DevCatalog &C)
{
    if (C.nU == 4 && C.n_grad == 1 && C.g_u[0] == 0 && C.n_div == 1 && C.n_curl == 1) return CAT_GDC4;
    if (C.nU == 4 && C.n_grad == 0 && C.n_div == 0 && C.n_curl == 1) return CAT_C4;
    if (C.nU == 1 && C.n_grad == 0 && C.n_div == 0 && C.n_curl == 0) return CAT_S1;
    if (C.nU == 1 && C.n_grad == 1 && C.g_u[0] == 0 && C.n_div == 0 && C.n_curl == 0) return CAT_SG1;
    return CAT_ANY;
}

// internal linkage: each unit that includes this header gets its own copy of the kernel
static __global__ void k_payload(int64_t n, DevTree T, DevCatalog C, float4 *pay, int stride)
{
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < n; b += (int64_t)gridDim.x * blockDim.x) {
        double4 L = T.leaf[b];
        double ih = 1.0 / L.w;
        float xh = (float)L.x, yh = (float)L.y, zh = (float)L.z;
        float4 *rec = const_cast<float4 *>(rec_of(pay, stride, (uint32_t)b));
        rec[0] = make_float4(xh, yh, zh, (float)ih);
        rec[PAY_BLOCK] = make_float4((float)(L.x - (double)xh), (float)(L.y - (double)yh), (float)(L.z - (double)zh),
                                     (float)(T.m[b] / T.rho[b]));
        float v[2 * MAXU + 4];
#pragma unroll
        for (int u = 0; u < MAXU; ++u) {
            double a = (u < C.nU) ? C.ucol[u][b] : 0.0;
            float hi = (float)a;
            v[2 * u] = hi;
            v[2 * u + 1] = (float)(a - (double)hi);
        }
        v[2 * MAXU] = v[2 * MAXU + 1] = v[2 * MAXU + 2] = v[2 * MAXU + 3] = 0.f;
        for (int k = 2; k < stride; ++k)
            rec[k * PAY_BLOCK] = make_float4(v[4 * k - 8], v[4 * k - 7], v[4 * k - 6], v[4 * k - 5]);
    }
}

// The 15 FP64 sums of a thread live in shared memory (slot k at sa[k * ACC_STRIDE]): the pair
// loop touches them once every CHUNK batches, so they need not hold registers.  Slots: 0 S1,
// 1-4 SA, 5-7 B, 8-10 F, 11 D, 12-14 curl.
constexpr int ACC_STRIDE = 128;   // threads per block of the kernels that use Acc32
constexpr int ACC_SLOTS = 15;

struct Acc32 {
    float pS1, pSA[MAXU], pB[3], pF[MAXG][3], pD[MAXD], pC[MAXC][3];
    float hh[MAXU], hl[MAXU];
    double *sa;
    bool have;

    __device__ __forceinline__ void addk(int k, float x)
    {
        double &d = sa[k * ACC_STRIDE];
        d = __dadd_rn(d, (double)x);
    }
    __device__ __forceinline__ double getk(int k) const { return sa[k * ACC_STRIDE]; }

    __device__ __forceinline__ void zero_partials()
    {
        pS1 = 0.f;
#pragma unroll
        for (int u = 0; u < MAXU; ++u) pSA[u] = 0.f;
#pragma unroll
        for (int d = 0; d < 3; ++d) pB[d] = 0.f;
#pragma unroll
        for (int j = 0; j < MAXG; ++j) pF[j][0] = pF[j][1] = pF[j][2] = 0.f;
#pragma unroll
        for (int j = 0; j < MAXD; ++j) pD[j] = 0.f;
#pragma unroll
        for (int j = 0; j < MAXC; ++j) pC[j][0] = pC[j][1] = pC[j][2] = 0.f;
    }

    __device__ __forceinline__ void init(double *slots)
    {
        sa = slots;
        zero_partials();
#pragma unroll
        for (int k = 0; k < ACC_SLOTS; ++k) sa[k * ACC_STRIDE] = 0.0;
#pragma unroll
        for (int u = 0; u < MAXU; ++u) { hh[u] = 0.f; hl[u] = 0.f; }
        have = false;
    }

    template <int CAT>
    __device__ __forceinline__ void flush(const DevCatalog &C)
    {
        using S = CatShape<CAT>;
        addk(0, pS1);
#pragma unroll
        for (int u = 0; u < MAXU; ++u)
            if (u < S::nu(C)) addk(1 + u, pSA[u]);
        if (S::any(C)) {
#pragma unroll
            for (int d = 0; d < 3; ++d) addk(5 + d, pB[d]);
            if (S::grad(C)) { addk(8, pF[0][0]); addk(9, pF[0][1]); addk(10, pF[0][2]); }
            if (S::div(C)) addk(11, pD[0]);
            if (S::curl(C)) { addk(12, pC[0][0]); addk(13, pC[0][1]); addk(14, pC[0][2]); }
        }
        zero_partials();
    }
};

struct Query32 {
    float ih, cw, cg, sig;   // 1/h_a, sigma h_a^-3, sigma h_a^-4, sigma
    float ph[3], pl[3]; // query position as double-float pairs
};

// column value pairs (hi, lo) of a record
template <int CAT>
__device__ __forceinline__ void load_cols(const float4 *rec, int stride, float *ch, float *cl)
{
    stride = CatShape<CAT>::stride(stride);
    float v[8];
#pragma unroll
    for (int k = 2; k < 4; ++k) {
        float4 c = (k < stride) ? __ldg(rec + k * PAY_BLOCK) : make_float4(0.f, 0.f, 0.f, 0.f);
        v[4 * k - 8] = c.x; v[4 * k - 7] = c.y; v[4 * k - 6] = c.z; v[4 * k - 5] = c.w;
    }
#pragma unroll
    for (int u = 0; u < MAXU; ++u) { ch[u] = v[2 * u]; cl[u] = v[2 * u + 1]; }
}

// per-pair terms: weight m_b/rho_b W, quantity offsets a_u, weighted kernel gradient
struct Terms32 {
    float w, a[MAXU], gx, gy, gz;
};

// the terms of the pair with the particle whose record (field 0) is `rec`
template <int STRAT, int KT, int CAT>
__device__ __forceinline__ void terms32(const Acc32 &A, const DevCatalog &C, const Query32 &Q,
                                        const float4 *__restrict__ rec, int stride, Terms32 &t)
{
    stride = CatShape<CAT>::stride(stride);
    const bool need_grad = CatShape<CAT>::any(C);
    const float4 p0 = __ldg(rec), p1 = __ldg(rec + PAY_BLOCK);
    const float dx = (Q.ph[0] - p0.x) + (Q.pl[0] - p1.x);
    const float dy = (Q.ph[1] - p0.y) + (Q.pl[1] - p1.y);
    const float dz = (Q.ph[2] - p0.z) + (Q.pl[2] - p1.z);
    float ch[MAXU], cl[MAXU];
    load_cols<CAT>(rec, stride, ch, cl);
    const float cWb = ((Q.sig * p0.w) * p0.w) * p0.w, cGb = cWb * p0.w;
    const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    // the SFU's reciprocal square root without the subnormal-input path of rsqrtf (the
    // approximation is the same for normal inputs); a pair closer than 1e-15 (r2 <= 1e-30)
    // counts as coincident, as r2 = 0 does: no gradient term, W at q = 0
    float rs;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(rs) : "f"(r2));
    const float rinv = r2 > 1e-30f ? rs : 0.f;
    const float r = r2 * rinv;
    float W, G;
    if (STRAT == SYMMETRIC) {
        float fa, dfa;
        shape<KT>(r * Q.ih, fa, dfa);
        // W(r, h_b) and its derivative: every piece of a shape clamps to zero outside the
        // neighbour's own support, so there the h_b term adds zeros; it is evaluated on every
        // lane (a warp vote to skip it costs more issue slots than it saves)
        float fb, dfb;
        shape<KT>(r * p0.w, fb, dfb);
        const float Wb = cWb * fb, Gb = cGb * dfb;
        W = 0.5f * fmaf(Q.cw, fa, Wb);
        G = (0.5f * fmaf(Q.cg, dfa, Gb)) * rinv;
    } else if (STRAT == GATHER) {
        float f, df;
        shape<KT>(r * Q.ih, f, df);
        W = Q.cw * f;
        G = (Q.cg * df) * rinv;
    } else {
        float f, df;
        shape<KT>(r * p0.w, f, df);
        W = cWb * f;
        G = (cGb * df) * rinv;
    }
    const float mrho = p1.w;
    t.w = mrho * W;
#pragma unroll
    for (int u = 0; u < MAXU; ++u) t.a[u] = u < CatShape<CAT>::nu(C) ? (ch[u] - A.hh[u]) + (cl[u] - A.hl[u]) : 0.f;
    if (need_grad) {
        const float gq = mrho * G;
        t.gx = gq * dx;
        t.gy = gq * dy;
        t.gz = gq * dz;
    }
}

// fixed slots: the gradient's column in slot 0, the div/curl vector in slots 1..3
template <int CAT>
__device__ __forceinline__ void accum32(Acc32 &A, const DevCatalog &C, const Terms32 &t)
{
    using S = CatShape<CAT>;
    A.pS1 += t.w;
#pragma unroll
    for (int u = 0; u < MAXU; ++u)
        if (u < S::nu(C)) A.pSA[u] = fmaf(t.a[u], t.w, A.pSA[u]);
    if (S::any(C)) {
        A.pB[0] += t.gx; A.pB[1] += t.gy; A.pB[2] += t.gz;
        if (S::grad(C)) {
            A.pF[0][0] = fmaf(t.gx, t.a[0], A.pF[0][0]);
            A.pF[0][1] = fmaf(t.gy, t.a[0], A.pF[0][1]);
            A.pF[0][2] = fmaf(t.gz, t.a[0], A.pF[0][2]);
        }
        if (S::div(C)) A.pD[0] = fmaf(t.gz, t.a[3], fmaf(t.gy, t.a[2], fmaf(t.gx, t.a[1], A.pD[0])));
        if (S::curl(C)) {
            A.pC[0][0] = fmaf(t.a[2], t.gz, fmaf(-t.a[3], t.gy, A.pC[0][0]));
            A.pC[0][1] = fmaf(t.a[3], t.gx, fmaf(-t.a[1], t.gz, A.pC[0][1]));
            A.pC[0][2] = fmaf(t.a[1], t.gy, fmaf(-t.a[2], t.gx, A.pC[0][2]));
        }
    }
}

template <int STRAT, int KT, int CAT>
__device__ __forceinline__ void pair32(Acc32 &A, const DevCatalog &C, const Query32 &Q,
                                       const float4 *__restrict__ pay, int stride, int b)
{
    Terms32 t;
    terms32<STRAT, KT, CAT>(A, C, Q, rec_of(pay, CatShape<CAT>::stride(stride), b), stride, t);
    accum32<CAT>(A, C, t);
}

// two pairs of one lane, with particles b and b + 32 (the same lane of two consecutive full
// batches inside one run; r1 is b's record, so b + 32's is one payload block further):
// independent terms, then accumulated in order -- the same arithmetic as two pair32 calls,
// with twice the independent work
template <int STRAT, int KT, int CAT>
__device__ __forceinline__ void pair32x2(Acc32 &A, const DevCatalog &C, const Query32 &Q,
                                         const float4 *__restrict__ r1, int stride)
{
    Terms32 t1, t2;
    terms32<STRAT, KT, CAT>(A, C, Q, r1, stride, t1);
    terms32<STRAT, KT, CAT>(A, C, Q, r1 + CatShape<CAT>::stride(stride) * PAY_BLOCK, stride, t2);
    accum32<CAT>(A, C, t1);
    accum32<CAT>(A, C, t2);
}

__device__ __forceinline__ void finalize32w(const double *v, const Acc32 &A, const DevCatalog &C, int64_t qi)
{
    int l = 0;
    double S = v[0];
    if (S == 0.0) {
        for (int o = 0; o < C.L; ++o) C.out[o][qi] = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    double abar[MAXU], ah[MAXU], sav[MAXU];
#pragma unroll
    for (int u = 0; u < MAXU; ++u) {
        sav[u] = v[1 + u];
        abar[u] = sav[u] / S;
        ah[u] = (double)A.hh[u] + (double)A.hl[u];
    }
    const double B[3] = {v[5], v[6], v[7]};
#pragma unroll
    for (int j = 0; j < MAXS; ++j) {
        if (j < C.n_scalar) {
            int u = C.s_u[j];
            double h0 = pick<MAXU>(ah, u);
            C.out[l++][qi] = C.s_shep[j] ? h0 + pick<MAXU>(abar, u) : h0 * S + pick<MAXU>(sav, u);
        }
    }
    if (C.n_grad > 0) {
        double a = pick<MAXU>(abar, C.g_u[0]);
        C.out[l++][qi] = v[8] - a * B[0];
        C.out[l++][qi] = v[9] - a * B[1];
        C.out[l++][qi] = v[10] - a * B[2];
    }
    if (C.n_div > 0) {
        double ax = pick<MAXU>(abar, C.d_u[0][0]), ay = pick<MAXU>(abar, C.d_u[0][1]), az = pick<MAXU>(abar, C.d_u[0][2]);
        C.out[l++][qi] = v[11] - (ax * B[0] + ay * B[1] + az * B[2]);
    }
    if (C.n_curl > 0) {
        double ax = pick<MAXU>(abar, C.c_u[0][0]), ay = pick<MAXU>(abar, C.c_u[0][1]), az = pick<MAXU>(abar, C.c_u[0][2]);
        double bx = ay * B[2] - az * B[1];
        double by = az * B[0] - ax * B[2];
        double bz = ax * B[1] - ay * B[0];
        C.out[l++][qi] = -(v[12] - bx);
        C.out[l++][qi] = -(v[13] - by);
        C.out[l++][qi] = -(v[14] - bz);
    }
}

// per-query constants: kernel scale factors at h_a, the query position as double-float
// pairs, and the quantity offsets (nearest particle, else the first accepted neighbour)
template <int STRAT, int CAT>
__device__ __forceinline__ void setup32(const DevTree &T, float sig, double px, double py, double pz, int64_t bnear,
                                        Query32 &Q, Acc32 &A, const float4 *pay, int stride, double *slots)
{
    Q = Query32{};
    Q.sig = sig;
    if (STRAT != SCATTER) {
        double ha = bnear < 0 ? __longlong_as_double(0x7ff8000000000000LL) : ldg4(T.leaf + bnear).w;
        float ih = (float)(1.0 / ha);
        Q.ih = ih;
        Q.cw = sig * ih * ih * ih;
        Q.cg = Q.cw * ih;
    }
    Q.ph[0] = (float)px; Q.pl[0] = (float)(px - (double)Q.ph[0]);
    Q.ph[1] = (float)py; Q.pl[1] = (float)(py - (double)Q.ph[1]);
    Q.ph[2] = (float)pz; Q.pl[2] = (float)(pz - (double)Q.ph[2]);
    A.init(slots);
    if (bnear >= 0) {
        // quantities enter as offsets from the nearest particle's values, which are close
        // to the kernel-weighted means, so gradient/divergence/curl sums cancel far less
        load_cols<CAT>(rec_of(pay, CatShape<CAT>::stride(stride), (uint32_t)bnear), stride, A.hh, A.hl);
        A.have = true;
    }
}

template <int CAT>
__device__ __forceinline__ void offsets_from(Acc32 &A, const float4 *pay, int stride, int b0)
{
    load_cols<CAT>(rec_of(pay, CatShape<CAT>::stride(stride), b0), stride, A.hh, A.hl);
    A.have = true;
}

// flush, fixed-tree FP64 reduction of the 32 lane sums, lane 0 finalises
template <int CAT>
__device__ __forceinline__ void reduce_finalize32(Acc32 &A, const DevCatalog &C, int64_t qi, int lane)
{
    A.flush<CAT>(C);
    double v[15];
#pragma unroll
    for (int k = 0; k < ACC_SLOTS; ++k) v[k] = A.getk(k);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
        for (int a = 0; a < 15; ++a) v[a] += __shfl_down_sync(0xffffffffu, v[a], off);
    }
    if (lane == 0) finalize32w(v, A, C, qi);
}


// The fused FP32-compensated sum of one query (the warp walks the query's tree itself with the
// warp-uniform next_item and deals the accepted leaves to its lanes); bnear is the nearest
// sorted leaf (-1 for itpScatter), s_acc the block's FP64 slot array (ACC_SLOTS x 128), and
// leaf_size the walk's linear-scan cutoff (1: none).  Every lane of the warp calls it.
template <int STRAT, int KT>
__device__ __forceinline__ void points32_query(const DevTree &T, const DevCatalog &C, const float4 *__restrict__ pay,
                                               int stride, double px, double py, double pz, int64_t bnear,
                                               int64_t qi, double *s_acc, int lane, int leaf_size)
{
    const int64_t n = T.n;
    const double K = kernel_valid(KT);
    const float sig = ldexp_norm3(KT);
    double ha = 0.0;
    if (STRAT != SCATTER) ha = bnear < 0 ? __longlong_as_double(0x7ff8000000000000LL) : ldg4(T.leaf + bnear).w;
    const double ra = __dmul_rn(K, ha), r2a = __dmul_rn(ra, ra);
    Query32 Q;
    Acc32 A;
    setup32<STRAT, CAT_ANY>(T, sig, px, py, pz, bnear, Q, A, pay, stride, s_acc + threadIdx.x);
    Slots S{0, -1};
    int nb = 0;   // full batches since the last flush (warp-uniform)
    auto proc = [&](int fill) {
        if (!A.have) offsets_from<CAT_ANY>(A, pay, stride, (int)__shfl_sync(0xffffffffu, S.mine, 0));
        if (S.mine >= 0) pair32<STRAT, KT, CAT_ANY>(A, C, Q, pay, stride, (int)S.mine);
        if (fill == 32 && ++nb == CHUNK) {
            A.flush<CAT_ANY>(C);
            nb = 0;
        }
    };
    if (T.root == 0) {
        double4 L;
        double d2;
        if (single_leaf_accepted<STRAT>(T, px, py, pz, K, r2a, L, d2)) deal(S, lane, 0, 0, proc);
    } else {
        Walk w{T.root, 1, 0, 0, 4 * n + 64};
        int64_t lo, hi;
        while (next_item<STRAT>(T, w, px, py, pz, K, r2a, lo, hi, leaf_size)) deal(S, lane, lo, hi, proc);
    }
    if (S.fill > 0) proc(S.fill);
    reduce_finalize32<CAT_ANY>(A, C, qi, lane);
}


// The two-phase FP32-compensated sum of one walked query j (its runs in the pool P) at sample
// point qi: the k-th accepted leaf to lane k mod 32, in DFS order, exactly as the fused body
// deals them, so both give the same bits.  Every lane of the warp calls it.
template <int STRAT, int KT, int CAT>
__device__ __forceinline__ void pairs32_query(const DevTree &T, const DevCatalog &C, const float4 *__restrict__ pay,
                                              int stride, const RunPool &P, int64_t j, int64_t qi, double px,
                                              double py, double pz, int64_t bnear, double *s_acc, int lane)
{
    const float sig = ldexp_norm3(KT);
    Query32 Q;
    Acc32 A;
    setup32<STRAT, CAT>(T, sig, px, py, pz, bnear, Q, A, pay, stride, s_acc + threadIdx.x);
    int nb = 0;   // full batches since the last flush (warp-uniform)
    int mine = -1;
    auto first = [&](int b0) {
        if (!A.have) offsets_from<CAT>(A, pay, stride, b0);
    };
    auto one = [&](int b) {
        pair32<STRAT, KT, CAT>(A, C, Q, pay, stride, b);
        if (++nb == CHUNK) {
            A.flush<CAT>(C);
            nb = 0;
        }
    };
    const int S = CatShape<CAT>::stride(stride);
    auto two = [&](int m1) {   // flush boundary after the second batch (nb is even here)
        pair32x2<STRAT, KT, CAT>(A, C, Q, rec_of(pay, S, m1), stride);
        nb += 2;
        if (nb == CHUNK) {
            A.flush<CAT>(C);
            nb = 0;
        }
    };
    auto four = [&](int m1) {   // flush boundary after the fourth batch (nb is a multiple of 4 here)
        const float4 *r1 = rec_of(pay, S, m1);   // m1 + 64 is two payload blocks further
        pair32x2<STRAT, KT, CAT>(A, C, Q, r1, stride);
        pair32x2<STRAT, KT, CAT>(A, C, Q, r1 + 2 * S * PAY_BLOCK, stride);
        nb += 4;
        if (nb == CHUNK) {
            A.flush<CAT>(C);
            nb = 0;
        }
    };
    auto cantwo = [&]() { return (nb & 1) == 0; };
    auto canfour = [&]() { return (nb & 3) == 0; };
    deal_runs(P, j, lane, first, one, two, cantwo, four, canfour, mine);
    if (mine >= 0) pair32<STRAT, KT, CAT>(A, C, Q, pay, stride, mine);
    reduce_finalize32<CAT>(A, C, qi, lane);
}

}  // namespace pb
