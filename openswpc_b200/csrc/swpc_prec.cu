// swpc_prec.cu -- reduced-precision storage of the 3D stress and
// memory-variable arrays.
//
// The storage forms share the FP32 arithmetic of the kernels:
//   SWPC_PREC_F32     : S and R in FP32 (the reference's MP = SP build)
//   SWPC_PREC_BF16_R  : the 18 memory variables R in BF16 (2 bytes)
//   SWPC_PREC_F16_R   : the memory variables R in FP16 with a power-of-two
//                       scale as below, S in FP32
//   SWPC_PREC_F16_SR  : the 6 stresses S and the memory variables R in FP16,
//                       with a power-of-two scale s = 2^e per group (the
//                       stresses, the memory variables): value = stored * s.
// Re-centring the FP16 scales runs on the device, inside every step's launch
// sequence (and so inside the captured graph): before each step whose index is
// a multiple of kRescaleEvery, one kernel takes the largest stored magnitude of
// every FP16 array, one single-warp kernel moves e so that a group whose
// maximum left [2^3, 2^10) has it near 2^7 again (at least 64x headroom below
// the FP16 overflow at 65504, far from the subnormal range) and writes the new
// scales where the kernels read them, and one kernel multiplies the stored
// values of the moved arrays by the power of two (exact).  On other steps the
// three kernels return at once.  The host never waits for them.
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

constexpr int kRescaleEvery = 8;   // re-centre before every step whose index is a multiple of this

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

// the FP16 arrays of a context and the exponent slot of each: 0..5 the
// stresses, 6 + component * 3 + m the memory variables
struct RescaleArgs {
    __half *p[24];
    int slot[24];
    int nf;
    long long n;          // halves per array (a multiple of 8)
    const int *d_it;      // step counter of graph replays (null: it)
    int it;
    int force;            // re-centre now, whatever the step
    unsigned int *d_max;  // per array, zero between re-centrings
    int *d_exp;           // exponent per slot (24)
    float *d_scale;       // the 48 scales the kernels read (swpc_kernels.cuh)
    float *d_factor;      // per array: 2^-shift of this re-centring, 1 if none
    int *d_changed;       // arrays moved (swpc_rescale's count)
};

__device__ __forceinline__ bool rescale_now(const RescaleArgs &r) {
    return r.force || (r.d_it ? *r.d_it : r.it) % kRescaleEvery == 0;
}

// max |stored| of every FP16 array (blockIdx.y) into d_max (float bits,
// atomicMax), 8 halves a thread per load
__global__ void rescale_max_kernel(const RescaleArgs r) {
    if (!rescale_now(r)) return;
    const uint4 *p8 = reinterpret_cast<const uint4 *>(r.p[blockIdx.y]);
    unsigned int m = 0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < r.n / 8;
         q += (long long)gridDim.x * blockDim.x) {
        const uint4 w = __ldcs(p8 + q);
        const unsigned int v[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int h = 0; h < 4; h++) {
            const float2 f = __half22float2(*reinterpret_cast<const __half2 *>(&v[h]));
            m = max(m, max(__float_as_uint(fabsf(f.x)), __float_as_uint(fabsf(f.y))));
        }
    }
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(r.d_max + blockIdx.y, m);
}

// the new exponent and scales of each group (stresses: slots 0-5, memory
// variables: slots 6-23), from the largest stored magnitude over its arrays;
// one warp, thread y owns array y
__global__ void rescale_decide_kernel(const RescaleArgs r) {
    if (!rescale_now(r)) return;
    const int y = threadIdx.x;
    const bool mine = y < r.nf;
    const unsigned int mb = mine ? r.d_max[y] : 0u;
    if (mine) r.d_max[y] = 0u;
    const bool is_r = mine && r.slot[y] >= 6;
    // group maxima (bit patterns of non-negative floats order like the values)
    unsigned int ms = (mine && !is_r) ? mb : 0u, mr = is_r ? mb : 0u;
    for (int o = 16; o > 0; o >>= 1) {
        ms = max(ms, __shfl_xor_sync(0xffffffffu, ms, o));
        mr = max(mr, __shfl_xor_sync(0xffffffffu, mr, o));
    }
    float gfac[2] = {1.0f, 1.0f};
#pragma unroll
    for (int g = 0; g < 2; g++) {
        const float m = __uint_as_float(g == 0 ? ms : mr);
        if (!(m > 0.0f) || !isfinite(m)) continue;
        const int ex = ilogbf(m);   // m = f 2^ex, 1 <= f < 2
        if (ex >= 3 && ex < 10) continue;
        const int shift = ex - 7;   // stored /= 2^shift, e += shift
        const int e = r.d_exp[g == 0 ? 0 : 6] + shift;   // every thread reads before thread 0 writes
        gfac[g] = ldexpf(1.0f, -shift);
        __syncwarp();
        if (y == 0) {
            r.d_exp[g == 0 ? 0 : 6] = e;
            const float sc = ldexpf(1.0f, e), inv = ldexpf(1.0f, -e);
            const int base = g == 0 ? 0 : 12, n = g == 0 ? 6 : 18;
            for (int q = 0; q < n; q++) { r.d_scale[base + q] = sc; r.d_scale[base + n + q] = inv; }
        }
    }
    if (mine) {
        const float f = gfac[is_r ? 1 : 0];
        r.d_factor[y] = f;
        if (f != 1.0f) atomicAdd(r.d_changed, 1);
    }
}

// stored *= factor (a power of two) for the moved arrays
__global__ void rescale_apply_kernel(const RescaleArgs r) {
    if (!rescale_now(r)) return;
    const float f = r.d_factor[blockIdx.y];
    if (f == 1.0f) return;
    uint4 *p8 = reinterpret_cast<uint4 *>(r.p[blockIdx.y]);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < r.n / 8;
         q += (long long)gridDim.x * blockDim.x) {
        uint4 w = p8[q];
        unsigned int *v = reinterpret_cast<unsigned int *>(&w);
#pragma unroll
        for (int h = 0; h < 4; h++) {
            const float2 x = __half22float2(*reinterpret_cast<const __half2 *>(&v[h]));
            const __half2 o = __floats2half2_rn(x.x * f, x.y * f);
            v[h] = *reinterpret_cast<const unsigned int *>(&o);
        }
        p8[q] = w;
    }
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
    if (field >= SWPC_F_SXX && field <= SWPC_F_SXY) return c->d_scale + (inverse ? 6 : 0) + (field - SWPC_F_SXX);
    if (field >= SWPC_F_R && field < SWPC_F_R + 18) return c->d_scale + (inverse ? 30 : 12) + (field - SWPC_F_R);
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
// the three re-centring kernels, on the context's stream (it or d_it: the
// step about to run; force: now)
int rescale_launch(swpc_ctx *c, int it, const int *d_it, bool force) {
    if (c->prec != SWPC_PREC_F16_SR && c->prec != SWPC_PREC_F16_R) return SWPC_OK;
    RescaleArgs r;
    memset(&r, 0, sizeof(r));
    if (c->prec == SWPC_PREC_F16_SR)
        for (int q = 0; q < 6; q++) { r.p[r.nf] = reinterpret_cast<__half *>(c->S[q]); r.slot[r.nf++] = q; }
    for (int comp = 0; comp < 6; comp++)
        for (int m = 0; m < c->d.nm; m++) {
            r.p[r.nf] = reinterpret_cast<__half *>(c->R[comp * 3 + m]);
            r.slot[r.nf++] = 6 + comp * 3 + m;
        }
    if (r.nf == 0) return SWPC_OK;
    r.n = c->g.ncell;
    r.d_it = d_it; r.it = it; r.force = force ? 1 : 0;
    r.d_max = c->d_rmax; r.d_exp = c->d_exp; r.d_scale = c->d_scale; r.d_factor = c->d_rfactor;
    r.d_changed = c->d_rchanged;
    const dim3 grid(148 * 2, r.nf);
    rescale_max_kernel<<<grid, 256, 0, c->stream>>>(r);
    rescale_decide_kernel<<<1, 32, 0, c->stream>>>(r);   // nf <= 24: one warp
    rescale_apply_kernel<<<grid, 256, 0, c->stream>>>(r);
    return cuda_check(c, cudaGetLastError(), "rescale kernels");
}
}  // namespace swpc

extern "C" int swpc_rescale(swpc_ctx *c, int *changed) {
    if (!c) return SWPC_ERR_ARG;
    if (changed) *changed = 0;
    if (c->prec != SWPC_PREC_F16_SR && c->prec != SWPC_PREC_F16_R) return SWPC_OK;
    if (cudaSetDevice(c->device) != cudaSuccess) return set_err(c, SWPC_ERR_CUDA, "cudaSetDevice failed");
    int rc = cuda_check(c, cudaMemsetAsync(c->d_rchanged, 0, sizeof(int), c->stream), "cudaMemsetAsync");
    if (!rc) rc = rescale_launch(c, 0, nullptr, true);
    int n = 0;
    if (!rc) rc = cuda_check(c, cudaMemcpyAsync(&n, c->d_rchanged, sizeof(int), cudaMemcpyDeviceToHost, c->stream),
                             "cudaMemcpyAsync");
    if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    if (rc) return rc;
    if (changed) *changed = n;
    return SWPC_OK;
}
