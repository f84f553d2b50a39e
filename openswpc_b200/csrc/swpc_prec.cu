// swpc_prec.cu -- reduced-precision storage of the 3D stress and
// memory-variable arrays.
//
// The storage forms share the FP32 arithmetic of the kernels:
//   SWPC_PREC_F32     : S and R in FP32 (the reference's MP = SP build)
//   SWPC_PREC_BF16_R  : the 18 memory variables R in BF16 (2 bytes)
//   SWPC_PREC_F16_R   : the memory variables R in FP16 with a power-of-two
//                       scale as below, S in FP32
//   SWPC_PREC_F16_SR  : the 6 stresses S and the memory variables R in FP16,
//                       with a power-of-two scale s = 2^e per stress array
//                       and one for the memory variables: value = stored * s.
// Re-centring the FP16 scales, on the device inside the step's launch
// sequence (and so inside the captured graph), without the host: before the
// stress update of every step whose index is a multiple of kRescaleEvery, one
// small-grid kernel takes the largest stored magnitude of each unit (each
// stress array; the memory variables together) and a one-thread kernel moves
// the exponent of a unit whose maximum left [2^3, 2^10) so that it sits near
// 2^7 (at least 64x headroom below the FP16 overflow at 65504, far from the
// subnormal range).  The stress update reads with the old scale and writes
// with the new one, which converts every value it rewrites (a power of two:
// exact), and a one-thread kernel then makes the new scale the read scale.
// Between measurements the kernels return at once.  swpc_rescale does the
// same between steps, converting the data with a pass of its own.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "swpc_ctx.h"

using namespace swpc;

namespace {


// s: the array's scale (FP16) in device memory, read once
__global__ void to_f32_kernel(const void *src, int kind, const float *s, float *dst, long long n) {
    const float sc = kind == 1 ? 1.0f : *s;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        dst[q] = kind == 1 ? __bfloat162float(reinterpret_cast<const __nv_bfloat16 *>(src)[q])
                           : __half2float(reinterpret_cast<const __half *>(src)[q]) * sc;
}

__global__ void from_f32_kernel(const float *src, int kind, const float *is, void *dst, long long n) {
    const float isc = kind == 1 ? 1.0f : *is;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        if (kind == 1) reinterpret_cast<__nv_bfloat16 *>(dst)[q] = __float2bfloat16_rn(src[q]);
        else reinterpret_cast<__half *>(dst)[q] = __float2half_rn(src[q] * isc);
    }
}

constexpr int kRescaleEvery = 8;   // the time loop measures before every step whose index is a multiple of this

// the FP16 arrays of a context: the stresses (F16_SR) first, then the
// memory variables.  Units: each stress array (0..5) and the memory
// variables as one (6).
struct RescaleArgs {
    __half *p[24];
    int ns, nf;           // stress arrays, all arrays
    long long n8;         // 16-byte words per array (ncell / 8)
    const int *d_it;      // step counter of graph replays (null: it)
    int it;
    int force;            // measure now, whatever the step
    unsigned int *d_max;  // 7 unit maxima of stored magnitudes (float bits), zero between uses
    int *d_exp;           // 7 unit exponents
    float *d_scale;       // the scales the kernels read (swpc_kernels.cuh sc_sS)
    float *d_factor;      // 7 unit factors 2^-shift of this re-centring, 1 if none
    int *d_changed;       // arrays moved (swpc_rescale's count)
};

__device__ __forceinline__ bool measure_now(const RescaleArgs &r) {
    return r.force || (r.d_it ? *r.d_it : r.it) % kRescaleEvery == 0;
}

// Largest stored magnitude of each unit (8 halves a thread per load, a
// grid-stride walk over every array); returns at once between measurements
__global__ void __launch_bounds__(256) rescale_max_kernel(const RescaleArgs r) {
    if (!measure_now(r)) return;
    const long long total = r.n8 * r.nf;
    unsigned int mu[7] = {0, 0, 0, 0, 0, 0, 0};   // per unit: stress arrays 0..5, memory variables 6
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < total;
         w += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(w / r.n8);
        const uint4 v4 = __ldcs(reinterpret_cast<const uint4 *>(r.p[y]) + (w - (long long)y * r.n8));
        const unsigned int v[4] = {v4.x, v4.y, v4.z, v4.w};
        unsigned int m = 0;
#pragma unroll
        for (int h = 0; h < 4; h++) {
            const float2 f = __half22float2(*reinterpret_cast<const __half2 *>(&v[h]));
            m = max(m, max(__float_as_uint(fabsf(f.x)), __float_as_uint(fabsf(f.y))));
        }
        const int u = y < r.ns ? y : 6;
#pragma unroll
        for (int q = 0; q < 7; q++)
            if (q == u) mu[q] = max(mu[q], m);
    }
#pragma unroll
    for (int q = 0; q < 7; q++) {
        unsigned int m = mu[q];
        for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0 && m) atomicMax(r.d_max + q, m);
    }
}

// From the unit maxima (then cleared): a unit whose stored maximum left
// [2^3, 2^10) gets the exponent that puts it near 2^7 (at least 64x headroom
// below 65504), in the scales that the next stress update writes with.  One
// thread; returns at once between measurements.
__global__ void rescale_decide_kernel(const RescaleArgs r) {
    if (!measure_now(r)) return;
    for (int u = 0; u < 7; u++) {
        const float m = __uint_as_float(r.d_max[u]);
        r.d_max[u] = 0u;
        float factor = 1.0f;
        const bool present = u < 6 ? u < r.ns : r.nf > r.ns;
        if (present && m > 0.0f && isfinite(m)) {
            const int ex = ilogbf(m);   // m = f 2^ex, 1 <= f < 2
            if (ex < 3 || ex >= 10) {
                const int shift = ex - 7;   // stored /= 2^shift, e += shift
                const int e = r.d_exp[u] + shift;
                r.d_exp[u] = e;
                if (u < 6) { r.d_scale[7 + u] = ldexpf(1.0f, e); r.d_scale[13 + u] = ldexpf(1.0f, -e); }
                else { r.d_scale[19] = ldexpf(1.0f, e); r.d_scale[20] = ldexpf(1.0f, -e); }
                factor = ldexpf(1.0f, -shift);
                *r.d_changed += u < 6 ? 1 : r.nf - r.ns;
            }
        }
        r.d_factor[u] = factor;
    }
}

// stored *= factor (a power of two) in the moved units: a re-centring asked
// for between steps converts the data itself
__global__ void __launch_bounds__(256) rescale_apply_kernel(const RescaleArgs r) {
    const long long total = r.n8 * r.nf;
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < total;
         w += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(w / r.n8);
        const float f = r.d_factor[y < r.ns ? y : 6];
        if (f == 1.0f) continue;
        uint4 *p = reinterpret_cast<uint4 *>(r.p[y]) + (w - (long long)y * r.n8);
        uint4 v4 = *p;
        unsigned int *v = reinterpret_cast<unsigned int *>(&v4);
#pragma unroll
        for (int h = 0; h < 4; h++) {
            const float2 x = __half22float2(*reinterpret_cast<const __half2 *>(&v[h]));
            const __half2 o = __floats2half2_rn(x.x * f, x.y * f);
            v[h] = *reinterpret_cast<const unsigned int *>(&o);
        }
        *p = v4;
    }
}

// what the stored values mean from now on (sc_sS_in, sc_sR_in)
__global__ void rescale_commit_kernel(float *d_scale) {
    for (int f = 0; f < 6; f++) d_scale[f] = d_scale[7 + f];
    d_scale[6] = d_scale[19];
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

// the device addresses of a field's scale (stored -> value) and inverse
static const float *field_scale(const swpc_ctx *c, int field, bool inverse) {
    if (field >= SWPC_F_SXX && field <= SWPC_F_SXY) return c->d_scale + (inverse ? 13 : 7) + (field - SWPC_F_SXX);
    if (field >= SWPC_F_R && field < SWPC_F_R + 18) return c->d_scale + (inverse ? 20 : 19);
    return c->d_scale;   // unused (FP32 or BF16)
}

// Converts a reduced-precision field to / from a temporary FP32 copy on the
// device, so that the FP32 box transfer can move it.
int prec_to_f32(swpc_ctx *c, int field, const float *stored, float **tmp) {
    *tmp = nullptr;
    cudaError_t e = cudaMalloc((void **)tmp, sizeof(float) * c->g.ncell);
    if (e != cudaSuccess) return set_err(c, SWPC_ERR_NOMEM, "cudaMalloc of the conversion buffer failed");
    to_f32_kernel<<<kGrid, 256, 0, c->stream>>>(stored, field_storage(c, field), field_scale(c, field, false), *tmp,
                                               c->g.ncell);
    return cuda_check(c, cudaGetLastError(), "to_f32_kernel");
}

int prec_from_f32(swpc_ctx *c, int field, const float *tmp, float *stored) {
    from_f32_kernel<<<kGrid, 256, 0, c->stream>>>(tmp, field_storage(c, field), field_scale(c, field, true),
                                                 stored, c->g.ncell);
    return cuda_check(c, cudaGetLastError(), "from_f32_kernel");
}

}  // namespace swpc

namespace swpc {
static RescaleArgs rescale_args(swpc_ctx *c, int it, const int *d_it, bool force) {
    RescaleArgs r;
    memset(&r, 0, sizeof(r));
    if (c->prec == SWPC_PREC_F16_SR)
        for (int q = 0; q < 6; q++) r.p[r.nf++] = reinterpret_cast<__half *>(c->S[q]);
    r.ns = r.nf;
    for (int comp = 0; comp < 6; comp++)
        for (int m = 0; m < c->d.nm; m++) r.p[r.nf++] = reinterpret_cast<__half *>(c->R[comp * 3 + m]);
    r.n8 = c->g.ncell / 8;   // ncell is a multiple of 8 (Kp is)
    r.d_it = d_it; r.it = it; r.force = force ? 1 : 0;
    r.d_max = c->d_rmax; r.d_exp = c->d_exp; r.d_scale = c->d_scale;
    r.d_factor = c->d_rfactor; r.d_changed = c->d_rchanged;
    return r;
}

static bool fp16_form(const swpc_ctx *c) { return c->prec == SWPC_PREC_F16_SR || c->prec == SWPC_PREC_F16_R; }

// Around each step's stress update (FP16 forms): before it, every
// kRescaleEvery steps, the largest stored magnitudes and from them new write
// scales (the update converts every value it rewrites); after it, the read
// scales follow.  Small grids: between measurements the kernels return at once.
int rescale_before_stress(swpc_ctx *c, int it, const int *d_it) {
    if (!fp16_form(c)) return SWPC_OK;
    const RescaleArgs r = rescale_args(c, it, d_it, false);
    if (r.nf == 0) return SWPC_OK;
    rescale_max_kernel<<<148 * 2, 256, 0, c->stream>>>(r);
    rescale_decide_kernel<<<1, 1, 0, c->stream>>>(r);
    return cuda_check(c, cudaGetLastError(), "rescale kernels");
}
int rescale_after_stress(swpc_ctx *c) {
    if (!fp16_form(c)) return SWPC_OK;
    rescale_commit_kernel<<<1, 1, 0, c->stream>>>(c->d_scale);
    return cuda_check(c, cudaGetLastError(), "rescale_commit_kernel");
}
}  // namespace swpc

extern "C" int swpc_rescale(swpc_ctx *c, int *changed) {
    if (!c) return SWPC_ERR_ARG;
    if (changed) *changed = 0;
    if (!fp16_form(c)) return SWPC_OK;
    if (cudaSetDevice(c->device) != cudaSuccess) return set_err(c, SWPC_ERR_CUDA, "cudaSetDevice failed");
    const RescaleArgs r = rescale_args(c, 0, nullptr, true);
    int rc = cuda_check(c, cudaMemsetAsync(c->d_rchanged, 0, sizeof(int), c->stream), "cudaMemsetAsync");
    if (!rc) rc = cuda_check(c, cudaMemsetAsync(c->d_rmax, 0, 7 * sizeof(unsigned int), c->stream), "cudaMemsetAsync");
    if (!rc && r.nf > 0) {
        rescale_max_kernel<<<148 * 4, 256, 0, c->stream>>>(r);
        rescale_decide_kernel<<<1, 1, 0, c->stream>>>(r);
        rescale_apply_kernel<<<148 * 4, 256, 0, c->stream>>>(r);
        rescale_commit_kernel<<<1, 1, 0, c->stream>>>(c->d_scale);
        rc = cuda_check(c, cudaGetLastError(), "rescale kernels");
    }
    int n = 0;
    if (!rc) rc = cuda_check(c, cudaMemcpyAsync(&n, c->d_rchanged, sizeof(int), cudaMemcpyDeviceToHost, c->stream),
                             "cudaMemcpyAsync");
    if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    if (rc) return rc;
    if (changed) *changed = n;
    return SWPC_OK;
}
