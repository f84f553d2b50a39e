// swpc_rmedia.cu -- random media in HBM: rmedia__3dgen / rmedia__2dgen
// (src/shared/m_rmedia.f90:176-307, :424-) and the cyclic mapping of the
// volume onto the memory box that rdrmed__3d does when the reference reads
// the generated file back (src/shared/m_rdrmed.f90:73-134).
//
// The method is the reference's (Roth and Korn 1993):
//   1. a volume of uniform random numbers in [0, 1),
//   2. its spectrum (forward FFT),
//   3. whitening: every coefficient divided by its modulus,
//   4. filtering by sqrt(psdf(|m|) * N * dV) for the Gaussian, exponential or
//      von Karman power spectral density (m_rmedia.f90:530-679),
//   5. the DC coefficient set to zero and the inverse FFT,
//   6. the mean removed and the field scaled to an rms of epsil.
// The random numbers come from a counter-based generator (splitmix64 of the
// seed and the cell index), so a realisation depends on the seed alone and
// not on the launch shape; gfortran's random_number stream of the reference
// cannot be reproduced, so realisations differ from the reference's files
// while their spectrum and rms follow the same rule.  The FFTs are cuFFT's
// (setup work, not the time step); reductions accumulate in FP64.
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>

#include "../../include/swpc_gpu.h"
#include "../../include/swpc_setup.h"

namespace {

constexpr int kThreads = 256;
constexpr int kGrid = 148 * 8;

__device__ __forceinline__ float uniform01(unsigned long long seed, unsigned long long q) {
    // splitmix64 finaliser of (seed, q); the top 24 bits give a float in [0, 1)
    unsigned long long z = seed + (q + 1ull) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (float)(z >> 40) * (1.0f / 16777216.0f);
}

__global__ void uniform_kernel(float *r, long long n, unsigned long long seed) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        r[q] = uniform01(seed, (unsigned long long)q);
}

struct FilterArgs {
    int ptype, two_d;
    int n1, n2, n3;          // FFT extents, slowest to fastest: (ny, nx, nz) in 3D, (1, nx, nz) in 2D
    float d1, d2, d3;        // spacings along them
    float a, epsil, kappa;
    float gk, gk15;          // gamma(kappa), gamma(kappa + 1.5) (3D von Karman)
    float norm;              // sqrt(N * dV) / (N * dV): filter factor and the inverse transform's 1 / (N dV)
};

// wavenumber of FFT index q of n points at spacing d (fk__x2k: non-negative
// up to n/2, negative above)
__device__ __forceinline__ float wavenumber(int q, int n, float d) {
    const float two_pi = 6.28318530717958647692f;
    return q <= n / 2 ? two_pi * (float)q / ((float)n * d) : -two_pi * (float)(n - q) / ((float)n * d);
}

__device__ float psdf(const FilterArgs &f, float m) {
    const float pi = 3.14159265358979323846f;
    const float e2 = f.epsil * f.epsil, am2 = f.a * f.a * m * m;
    if (f.two_d) {
        if (f.ptype == SWPC_RMEDIA_GAUSS) return e2 * f.a * f.a * pi * expf(-m * m * f.a * f.a * 0.25f);
        if (f.ptype == SWPC_RMEDIA_EXP) return (2 * e2 * f.a * f.a * pi) / powf(1 + am2, 1.5f);
        return (4 * pi * f.a * f.a * e2 * f.kappa) / powf(1 + am2, 1 + f.kappa);
    }
    if (f.ptype == SWPC_RMEDIA_GAUSS)
        return e2 * (f.a * f.a * f.a) * powf(pi, 1.5f) * expf(-m * m * f.a * f.a * 0.25f);
    if (f.ptype == SWPC_RMEDIA_EXP) {
        const float wk = 1.0f + am2;
        return (8 * e2 * f.a * f.a * f.a * pi) / (wk * wk);
    }
    return (8 * powf(pi, 1.5f) * e2 * f.a * f.a * f.a * f.gk15) / (f.gk * powf(1 + am2, f.kappa + 1.5f));
}

// whitening and filtering of the half spectrum (n1, n2, n3/2 + 1)
__global__ void filter_kernel(cufftComplex *c, FilterArgs f) {
    const int h3 = f.n3 / 2 + 1;
    const long long n = (long long)f.n1 * f.n2 * h3;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(q % h3);
        const int i = (int)((q / h3) % f.n2);
        const int j = (int)(q / ((long long)h3 * f.n2));
        const float k1 = f.n1 > 1 ? wavenumber(j, f.n1, f.d1) : 0.0f;
        const float k2 = wavenumber(i, f.n2, f.d2);
        const float k3 = wavenumber(k, f.n3, f.d3);
        const float m = sqrtf(k1 * k1 + k2 * k2 + k3 * k3);
        cufftComplex b = c[q];
        const float mod = hypotf(b.x, b.y);
        if (q == 0 || !(mod > 0.0f)) {   // the DC coefficient, or no phase to keep
            c[q] = make_cuFloatComplex(0.0f, 0.0f);
            continue;
        }
        const float g = sqrtf(psdf(f, m)) * f.norm / mod;
        c[q] = make_cuFloatComplex(b.x * g, b.y * g);
    }
}

// sum (pass 0) or centred sum of squares (pass 1) in FP64
__global__ void moments_kernel(const float *r, long long n, double mean, int pass, double *out) {
    double s = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const double v = (double)r[q] - mean;
        s += pass ? v * v : v;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ double sh[kThreads / 32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kThreads / 32; w++) t += sh[w];
        atomicAdd(out, t);
    }
}

__device__ __forceinline__ int wrap(int q, int n) {   // periodic index in 1..n (m_rdrmed.f90:111-119, 128-132)
    int r = q % n;
    return r <= 0 ? r + n : r;
}

// the volume, centred and scaled, over the memory box of the caller
__global__ void scatter_kernel(const float *r, int nx, int ny, int nz, int two_d, float mean, float scale,
                               float *xi, long long ld_k, long long ld_i) {
    const long long bk = nz + 6, bi = nx + 6, bj = two_d ? 1 : ny + 6;
    const long long n = bk * bi * bj;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(q % bk) - 2;
        const int i = (int)((q / bk) % bi) - 2;
        const int j = two_d ? 1 : (int)(q / (bk * bi)) - 2;
        const int kk = wrap(k, nz), ii = wrap(i, nx), jj = two_d ? 1 : wrap(j, ny);
        const long long src = ((long long)(jj - 1) * nx + (ii - 1)) * nz + (kk - 1);
        const long long dst = two_d ? (long long)(i + 2) * ld_k + (k + 2)
                                    : ((long long)(j + 2) * ld_i + (i + 2)) * ld_k + (k + 2);
        xi[dst] = (r[src] - mean) * scale;
    }
}

}  // namespace

extern "C" int swpc_rmedia_generate(const swpc_rmedia_desc *d, float *xi, int ld_k, int ld_i, void *stream) {
    if (!d || !xi) return SWPC_ERR_ARG;
    const bool two_d = d->ny == 1;
    if (d->nx < 2 || d->nz < 2 || d->ny < 1 || d->dx <= 0 || d->dz <= 0 || (!two_d && d->dy <= 0)) return SWPC_ERR_ARG;
    if (d->ptype != SWPC_RMEDIA_GAUSS && d->ptype != SWPC_RMEDIA_EXP && d->ptype != SWPC_RMEDIA_VONKARMAN)
        return SWPC_ERR_ARG;
    if (!(d->a > 0) || !(d->epsil >= 0) || (d->ptype == SWPC_RMEDIA_VONKARMAN && !(d->kappa > 0))) return SWPC_ERR_ARG;
    if (ld_k < d->nz + 6 || (!two_d && ld_i < d->nx + 6)) return SWPC_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int n1 = two_d ? 1 : d->ny, n2 = d->nx, n3 = d->nz;
    const long long n = (long long)n1 * n2 * n3;
    const long long nc = (long long)n1 * n2 * (n3 / 2 + 1);
    float *r = nullptr;
    cufftComplex *c = nullptr;
    double *mom = nullptr;
    cufftHandle fwd = 0, inv = 0;
    bool have_fwd = false, have_inv = false;
    int rc = SWPC_OK;
    if (cudaMalloc((void **)&r, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&c, nc * sizeof(cufftComplex)) != cudaSuccess ||
        cudaMalloc((void **)&mom, 2 * sizeof(double)) != cudaSuccess)
        rc = SWPC_ERR_NOMEM;
    if (!rc) {
        const cufftResult e1 = two_d ? cufftPlan2d(&fwd, n2, n3, CUFFT_R2C) : cufftPlan3d(&fwd, n1, n2, n3, CUFFT_R2C);
        have_fwd = e1 == CUFFT_SUCCESS;
        const cufftResult e2 = two_d ? cufftPlan2d(&inv, n2, n3, CUFFT_C2R) : cufftPlan3d(&inv, n1, n2, n3, CUFFT_C2R);
        have_inv = e2 == CUFFT_SUCCESS;
        if (!have_fwd || !have_inv) rc = (e1 == CUFFT_ALLOC_FAILED || e2 == CUFFT_ALLOC_FAILED) ? SWPC_ERR_NOMEM
                                                                                               : SWPC_ERR_CUDA;
    }
    if (!rc && (cufftSetStream(fwd, st) != CUFFT_SUCCESS || cufftSetStream(inv, st) != CUFFT_SUCCESS)) rc = SWPC_ERR_CUDA;
    if (!rc) {
        uniform_kernel<<<kGrid, kThreads, 0, st>>>(r, n, d->seed);
        if (cudaGetLastError() != cudaSuccess || cufftExecR2C(fwd, r, c) != CUFFT_SUCCESS) rc = SWPC_ERR_CUDA;
    }
    if (!rc) {
        FilterArgs f;
        f.ptype = d->ptype; f.two_d = two_d;
        f.n1 = n1; f.n2 = n2; f.n3 = n3;
        f.d1 = two_d ? 1.0f : d->dy; f.d2 = d->dx; f.d3 = d->dz;
        f.a = d->a; f.epsil = d->epsil; f.kappa = d->kappa;
        f.gk = d->ptype == SWPC_RMEDIA_VONKARMAN ? tgammaf(d->kappa) : 1.0f;
        f.gk15 = d->ptype == SWPC_RMEDIA_VONKARMAN ? tgammaf(d->kappa + 1.5f) : 1.0f;
        const double ndv = (double)n * d->dx * d->dz * (two_d ? 1.0 : d->dy);
        f.norm = (float)(std::sqrt(ndv) / ndv);
        filter_kernel<<<kGrid, kThreads, 0, st>>>(c, f);
        if (cudaGetLastError() != cudaSuccess || cufftExecC2R(inv, c, r) != CUFFT_SUCCESS) rc = SWPC_ERR_CUDA;
    }
    double h[2] = {0.0, 0.0};
    if (!rc) {
        cudaMemsetAsync(mom, 0, 2 * sizeof(double), st);
        moments_kernel<<<kGrid, kThreads, 0, st>>>(r, n, 0.0, 0, mom);
        if (cudaMemcpyAsync(h, mom, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            rc = SWPC_ERR_CUDA;
    }
    const double mean = h[0] / (double)n;
    if (!rc) {
        moments_kernel<<<kGrid, kThreads, 0, st>>>(r, n, mean, 1, mom + 1);
        if (cudaMemcpyAsync(h + 1, mom + 1, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            rc = SWPC_ERR_CUDA;
    }
    if (!rc) {
        const double rms = std::sqrt(h[1] / (double)n);
        const float scale = rms > 0 ? (float)(d->epsil / rms) : 0.0f;
        scatter_kernel<<<kGrid, kThreads, 0, st>>>(r, n2, n1, n3, two_d, (float)mean, scale, xi, ld_k, ld_i);
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) rc = SWPC_ERR_CUDA;
    }
    if (have_fwd) cufftDestroy(fwd);
    if (have_inv) cufftDestroy(inv);
    if (r) cudaFree(r);
    if (c) cudaFree(c);
    if (mom) cudaFree(mom);
    return rc;
}
