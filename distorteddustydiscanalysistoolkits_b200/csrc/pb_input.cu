// pb_input.cu -- ParticleIO's build_input on the device (ParticleIO.jl/src/julia/PartiaAdapter/
// build_input.jl:44-160): particle columns arrive in the type a dump stores them in (Phantom
// writes h and most per-particle quantities as real*4) and are widened to the FP64 columns of
// the interpolation input here, a constant particle mass is broadcast, and the density is
// derived from h as add_rho! does (ParticleIO.jl/src/julia/Particles/add_quantities.jl:308-345),
// so a snapshot's input is built where it will be used and crosses PCIe in its stored width.
#include <cmath>
#include <cstring>

#include "partia_b200.h"
#include "pb_internal.h"

namespace pb {

__global__ void k_f32_to_f64(int64_t n, const float *__restrict__ src, double *dst)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = (double)src[i];
}

__global__ void k_fill_f64(int64_t n, double v, double *dst)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = v;
}

// rho_i = (m hfact^3) * ((1/h_i)^3): mhfactd is formed on the host as m * hfact * hfact * hfact,
// the reference's left-to-right order; 1/h_i is the correctly rounded quotient (Julia inv)
__global__ void k_density_from_h(int64_t n, const double *__restrict__ h, double mhfactd, double *rho)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double inv = __ddiv_rn(1.0, h[i]);
        rho[i] = __dmul_rn(mhfactd, __dmul_rn(__dmul_rn(inv, inv), inv));
    }
}

}  // namespace pb

using namespace pb;


namespace {

int fail_in(Handle &H, int code, const char *msg)
{
    H.err = msg;
    return code;
}

bool on_device(const Handle &H, const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice && a.device == H.device) || a.type == cudaMemoryTypeManaged;
}

int finish(Handle &H, const char *what)
{
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(H.stream);
    if (e != cudaSuccess) {
        H.err = std::string(what) + ": " + cudaGetErrorString(e);
        return PB_ERR_CUDA;
    }
    return PB_OK;
}

}  // namespace

extern "C" {

int32_t pb_column_to_f64(pb_handle *h, const void *src, int32_t src_type, int64_t n, double *dst)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (n < 0 || !src || !dst || (src_type != 0 && src_type != 1))
        return fail_in(H, PB_ERR_INVALID, "pb_column_to_f64: bad arguments (src_type 0 = float64, 1 = float32)");
    if (!on_device(H, src) || !on_device(H, dst))
        return fail_in(H, PB_ERR_INVALID, "pb_column_to_f64: src and dst must be device memory of the handle's device");
    if (n == 0) return PB_OK;
    if (cudaSetDevice(H.device) != cudaSuccess) return fail_in(H, PB_ERR_CUDA, "cudaSetDevice failed");
    if (src_type == 0) {
        if (src != dst && cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToDevice, H.stream) != cudaSuccess)
            return finish(H, "pb_column_to_f64");
    } else {
        k_f32_to_f64<<<grid_for(n, 256), 256, 0, H.stream>>>(n, static_cast<const float *>(src), dst);
        H.launches += 1;
    }
    return finish(H, "pb_column_to_f64");
}

int32_t pb_fill_f64(pb_handle *h, double value, int64_t n, double *dst)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (n < 0 || !dst) return fail_in(H, PB_ERR_INVALID, "pb_fill_f64: bad arguments");
    if (!on_device(H, dst)) return fail_in(H, PB_ERR_INVALID, "pb_fill_f64: dst must be device memory of the handle's device");
    if (n == 0) return PB_OK;
    if (cudaSetDevice(H.device) != cudaSuccess) return fail_in(H, PB_ERR_CUDA, "cudaSetDevice failed");
    k_fill_f64<<<grid_for(n, 256), 256, 0, H.stream>>>(n, value, dst);
    H.launches += 1;
    return finish(H, "pb_fill_f64");
}

int32_t pb_density_from_h(pb_handle *h, const double *hsml, int64_t n, double mass, double hfact, double *rho)
{
    if (!h) return PB_ERR_INVALID;
    Handle &H = h->H;
    if (n < 0 || !hsml || !rho || !std::isfinite(mass) || !std::isfinite(hfact))
        return fail_in(H, PB_ERR_INVALID, "pb_density_from_h: bad arguments");
    if (!on_device(H, hsml) || !on_device(H, rho))
        return fail_in(H, PB_ERR_INVALID, "pb_density_from_h: h and rho must be device memory of the handle's device");
    if (n == 0) return PB_OK;
    if (cudaSetDevice(H.device) != cudaSuccess) return fail_in(H, PB_ERR_CUDA, "cudaSetDevice failed");
    volatile double mh = mass * hfact;   // m * hfact * hfact * hfact, left to right, no contraction
    mh = mh * hfact;
    mh = mh * hfact;
    k_density_from_h<<<grid_for(n, 256), 256, 0, H.stream>>>(n, hsml, (double)mh, rho);
    H.launches += 1;
    return finish(H, "pb_density_from_h");
}

}  // extern "C"
