// swpc_prec.cu -- reduced-precision storage of the 3D stress and
// memory-variable arrays.
//
// Three storage forms share the FP32 arithmetic of the kernels:
//   SWPC_PREC_F32     : S and R in FP32 (the reference's MP = SP build)
//   SWPC_PREC_BF16_R  : the 18 memory variables R in BF16 (2 bytes)
//   SWPC_PREC_F16_R   : the memory variables R in FP16 with per-array
//                       power-of-two scales as below, S in FP32
//   SWPC_PREC_F16_SR  : the 6 stresses S and the memory variables R in FP16,
//                       each array with its own power-of-two scale s = 2^e:
//                       value = stored * s.  swpc_rescale moves e so that
//                       every array's largest magnitude sits near 2^7 in
//                       storage, far from the FP16 overflow at 65504 and from
//                       its subnormal range; scaling by a power of two is
//                       exact, so rescaling adds no rounding.  The time loop
//                       (swpc_run, swpc_step, swpc_step_half) calls it before
//                       every step whose index is a multiple of
//                       kRescaleEvery, so growth between two calls stays far
//                       below the headroom.
// This file holds the conversion kernels used by the field transfers and the
// rescaling pass.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "swpc_ctx.h"

namespace swpc {
int graph_invalidate(swpc_ctx *c);
}

using namespace swpc;

namespace {

__global__ void to_f32_kernel(const void *src, int kind, float s, float *dst, long long n) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        dst[q] = kind == 1 ? __bfloat162float(reinterpret_cast<const __nv_bfloat16 *>(src)[q])
                           : __half2float(reinterpret_cast<const __half *>(src)[q]) * s;
}

__global__ void from_f32_kernel(const float *src, int kind, float is, void *dst, long long n) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        if (kind == 1) reinterpret_cast<__nv_bfloat16 *>(dst)[q] = __float2bfloat16_rn(src[q]);
        else reinterpret_cast<__half *>(dst)[q] = __float2half_rn(src[q] * is);
    }
}

// max |stored| of one FP16 array into out (float bits, atomicMax)
__global__ void absmax_half_kernel(const __half *p, long long n, unsigned int *out) {
    unsigned int m = 0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        m = max(m, __float_as_uint(fabsf(__half2float(p[q]))));
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// stored *= f (a power of two)
__global__ void rescale_half_kernel(__half *p, long long n, float f) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        p[q] = __float2half_rn(__half2float(p[q]) * f);
}

constexpr int kGrid = 148 * 8;

}  // namespace

namespace swpc {

// storage of a field id: 0 FP32, 1 BF16, 2 FP16
int field_storage(const swpc_ctx *c, int field) {
    if (field >= SWPC_F_SXX && field <= SWPC_F_SXY) return c->prec == SWPC_PREC_F16_SR ? 2 : 0;
    if (field >= SWPC_F_R && field < SWPC_F_R + 18)
        return (c->prec == SWPC_PREC_F16_SR || c->prec == SWPC_PREC_F16_R) ? 2 : (c->prec == SWPC_PREC_BF16_R ? 1 : 0);
    return 0;
}

float field_scale(const swpc_ctx *c, int field) {
    if (field >= SWPC_F_SXX && field <= SWPC_F_SXY) return std::ldexp(1.0f, c->eS[field - SWPC_F_SXX]);
    if (field >= SWPC_F_R && field < SWPC_F_R + 18) return std::ldexp(1.0f, c->eR[field - SWPC_F_R]);
    return 1.0f;
}

// Converts a reduced-precision field to / from a temporary FP32 copy on the
// device, so that the FP32 box transfer can move it.
int prec_to_f32(swpc_ctx *c, int field, const float *stored, float **tmp) {
    *tmp = nullptr;
    cudaError_t e = cudaMalloc((void **)tmp, sizeof(float) * c->g.ncell);
    if (e != cudaSuccess) return set_err(c, SWPC_ERR_NOMEM, "cudaMalloc of the conversion buffer failed");
    to_f32_kernel<<<kGrid, 256, 0, c->stream>>>(stored, field_storage(c, field), field_scale(c, field), *tmp,
                                               c->g.ncell);
    return cuda_check(c, cudaGetLastError(), "to_f32_kernel");
}

int prec_from_f32(swpc_ctx *c, int field, const float *tmp, float *stored) {
    from_f32_kernel<<<kGrid, 256, 0, c->stream>>>(tmp, field_storage(c, field), 1.0f / field_scale(c, field),
                                                 stored, c->g.ncell);
    return cuda_check(c, cudaGetLastError(), "from_f32_kernel");
}

}  // namespace swpc

extern "C" int swpc_rescale(swpc_ctx *c, int *changed) {
    if (!c) return SWPC_ERR_ARG;
    if (changed) *changed = 0;
    if (c->prec != SWPC_PREC_F16_SR && c->prec != SWPC_PREC_F16_R) return SWPC_OK;
    if (cudaSetDevice(c->device) != cudaSuccess) return set_err(c, SWPC_ERR_CUDA, "cudaSetDevice failed");
    const bool with_s = c->prec == SWPC_PREC_F16_SR;   // F16_R keeps S in FP32
    const int nf = (with_s ? 6 : 0) + 6 * c->d.nm;
    std::vector<float *> fields;
    std::vector<int *> expo;
    if (with_s)
        for (int q = 0; q < 6; q++) { fields.push_back(c->S[q]); expo.push_back(&c->eS[q]); }
    for (int comp = 0; comp < 6; comp++)
        for (int m = 0; m < c->d.nm; m++) { fields.push_back(c->R[comp * 3 + m]); expo.push_back(&c->eR[comp * 3 + m]); }
    unsigned int *d_max = nullptr;
    if (cudaMalloc((void **)&d_max, sizeof(unsigned int) * nf) != cudaSuccess)
        return set_err(c, SWPC_ERR_NOMEM, "cudaMalloc failed");
    int rc = cuda_check(c, cudaMemsetAsync(d_max, 0, sizeof(unsigned int) * nf, c->stream), "cudaMemsetAsync");
    for (int q = 0; q < nf && !rc; q++) {
        absmax_half_kernel<<<kGrid, 256, 0, c->stream>>>(reinterpret_cast<const __half *>(fields[q]), c->g.ncell,
                                                         d_max + q);
        rc = cuda_check(c, cudaGetLastError(), "absmax_half_kernel");
    }
    std::vector<unsigned int> h(nf, 0);
    if (!rc) rc = cuda_check(c, cudaMemcpyAsync(h.data(), d_max, sizeof(unsigned int) * nf, cudaMemcpyDeviceToHost,
                                                c->stream), "cudaMemcpyAsync");
    if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    cudaFree(d_max);
    if (rc) return rc;
    int nchg = 0;
    for (int q = 0; q < nf; q++) {
        float m;
        memcpy(&m, &h[q], sizeof(float));
        if (!(m > 0.0f) || !std::isfinite(m)) continue;
        // stored max in [2^3, 2^10) is kept; otherwise move it to [2^7, 2^8),
        // which leaves at least 64x (after a move 256x) headroom below the
        // FP16 overflow for growth between two calls: a wave front can
        // multiply an array's maximum by ~40 in 10 steps while the source
        // starts up
        const int ex = std::ilogb(m);   // m = f * 2^ex, 1 <= f < 2
        if (ex >= 3 && ex < 10) continue;
        const int shift = ex - 7;       // stored /= 2^shift, e += shift
        rescale_half_kernel<<<kGrid, 256, 0, c->stream>>>(reinterpret_cast<__half *>(fields[q]), c->g.ncell,
                                                          std::ldexp(1.0f, -shift));
        rc = cuda_check(c, cudaGetLastError(), "rescale_half_kernel");
        if (rc) return rc;
        *expo[q] += shift;
        nchg++;
    }
    if (changed) *changed = nchg;
    // the kernels read the scales from device memory: no new launch arguments
    if (nchg) return upload_scales(c);
    return cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
}
