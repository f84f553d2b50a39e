// swpc2d_kernels.cu -- 2D P-SV and SH time-step kernels for sm_100a.
//
// Every launch works on a table of models and a list of 32 (k) x (TI*RI) (i)
// tiles covering all of them (a block of 32 x TI threads, RI rows per thread), walked by a persistent grid: one model is the
// single-run case, many models of uneven size are the batched ensemble, and
// both run the same code.  Per cell the kernels restate
//   P-SV: src/swpc_psv/m_kernel.f90:76-306 (interior) and
//         src/swpc_psv/m_absorb_p.f90:180-230, 337-385 (ADE-CFS PML),
//   SH:   src/swpc_sh/m_kernel.f90:77-221 and src/swpc_sh/m_absorb_p.f90,
// in the reference's expression order; the file is compiled with
// -fmad=false so the FP32 results are bitwise identical to the oracle.
#include <cuda_runtime.h>

#include "swpc_ctx.h"
#include "swpc2d.cuh"

namespace swpc {

namespace {
constexpr float EPSL = 1.1920929e-07f;   // epsilon(1.0)
__device__ __forceinline__ float lds(const float *p) { return __ldcs(p); }
__device__ __forceinline__ void sts(float *p, float v) { __stcs(p, v); }

// The block's copy of the model descriptor of the current tile.  Shared
// memory does not alias the fields the kernel stores to, so the descriptor
// is read once per tile instead of after every store, and consecutive tiles
// of the same model reuse it.  Uniform over the block.
__device__ __forceinline__ const Model2D &tile_model(const Model2D *__restrict__ models, int model, Model2D &sM,
                                                     int &cached) {
    if (model != cached) {
        __syncthreads();   // every thread is done with the previous copy
        const int nw = (int)(sizeof(Model2D) / sizeof(int));
        const int *src = reinterpret_cast<const int *>(models + model);
        int *dst = reinterpret_cast<int *>(&sM);
        for (int w = threadIdx.y * blockDim.x + threadIdx.x; w < nw; w += blockDim.x * blockDim.y) dst[w] = __ldg(src + w);
        __syncthreads();
        cached = model;
    }
    return sM;
}
}  // namespace

// ---------------------------------------------------------------------------
// P-SV stress: kernel__update_stress + absorb_p__update_stress
// ---------------------------------------------------------------------------
template <int NM>
__global__ void __launch_bounds__(256) psv_stress_kernel(const Model2D *__restrict__ models,
                                                         const Tile2D *__restrict__ tiles, int ntiles, int mask,
        int ri) {
    __shared__ Model2D sM;
    int cached = -1;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const Tile2D tl = tiles[t];
        const Model2D &M = tile_model(models, tl.model, sM, cached);
        // ri rows of the tile per thread: the tile and model descriptors are
        // fetched once for ri cells
        for (int r = 0; r < ri; r++) {
            const int k = tl.k0 + threadIdx.x, i = tl.i0 + threadIdx.y + r * (int)blockDim.y;
            if (k > M.nz || i > M.nx) continue;
            const long long PI = M.Kp;
            const long long e = (long long)(i + 2) * PI + (k - 1 + KH);
            const float *__restrict__ Vx = M.V0;
            const float *__restrict__ Vz = M.V1;
            const float dt = M.dt;
            if (i >= M.ibk && i <= M.iek && k <= M.kek) {
                if (!(mask & 1)) continue;
                const int4 bd = __ldg(&M.band[i + 2]);
                const int p1 = (k - bd.x) * (bd.y - k), p2 = (k - bd.z) * (bd.w - k);
                const int s = ((p1 > p2 ? p1 : p2) >= 0) ? 1 : 0;
                const float re40x = M.e40[0][s], re41x = M.e41[0][s], re40z = M.e40[1][s], re41z = M.e41[1][s];
                float r[3][NM > 0 ? NM : 1];
    #pragma unroll
                for (int c = 0; c < 3; c++)
    #pragma unroll
                    for (int m = 0; m < NM; m++) r[c][m] = lds(&M.R[c * 3 + m][e]);
                const float sxx = lds(&M.S0[e]), szz = lds(&M.S1[e]), sxz = lds(&M.S2[e]);
                const float mu = lds(&M.mu[e]), lam = lds(&M.lam[e]), taup1 = lds(&M.taup[e]), taus1 = lds(&M.taus[e]);
                const float pnn = __ldg(&M.mu[e + 1]), npn = __ldg(&M.mu[e + PI]), ppn = __ldg(&M.mu[e + 1 + PI]);
                const float vx0 = __ldg(&Vx[e]), vz0 = __ldg(&Vz[e]);
                const float dxVx = (vx0 - __ldg(&Vx[e - PI])) * re40x - (__ldg(&Vx[e + PI]) - __ldg(&Vx[e - 2 * PI])) * re41x;
                const float dzVz = (vz0 - __ldg(&Vz[e - 1])) * re40z - (__ldg(&Vz[e + 1]) - __ldg(&Vz[e - 2])) * re41z;
                const float dxVz = (__ldg(&Vz[e + PI]) - vz0) * re40x - (__ldg(&Vz[e + 2 * PI]) - __ldg(&Vz[e - PI])) * re41x;
                const float dzVx = (__ldg(&Vx[e + 1]) - vx0) * re40z - (__ldg(&Vx[e + 2]) - __ldg(&Vx[e - 1])) * re41z;
                // normal components (src/swpc_psv/m_kernel.f90:191-227)
                const float mu2 = 2 * mu;
                const float lam2mu = lam + mu2;
                const float d2v2 = dxVx + dzVz;
                const float f_Rxx = lam2mu * taup1 * d2v2 - mu2 * taus1 * dzVz;
                const float f_Rzz = lam2mu * taup1 * d2v2 - mu2 * taus1 * dxVx;
                float Rxx_n = 0.0f, Rzz_n = 0.0f;
    #pragma unroll
                for (int m = 0; m < NM; m++) {
                    r[0][m] = M.c1[m] * r[0][m] - M.c2[m] * f_Rxx * dt;
                    r[1][m] = M.c1[m] * r[1][m] - M.c2[m] * f_Rzz * dt;
                    Rxx_n = Rxx_n + M.d1[m] * r[0][m];
                    Rzz_n = Rzz_n + M.d1[m] * r[1][m];
                }
                const float taup_plus1 = 1 + taup1 * (1 + M.d2);
                const float taus_plus1 = 1 + taus1 * (1 + M.d2);
                sts(&M.S0[e], sxx + (lam2mu * taup_plus1 * d2v2 - mu2 * taus_plus1 * dzVz + Rxx_n) * dt);
                sts(&M.S1[e], szz + (lam2mu * taup_plus1 * d2v2 - mu2 * taus_plus1 * dxVx + Rzz_n) * dt);
                // shear component (src/swpc_psv/m_kernel.f90:270-300)
                const float nnn = mu;
                const float mu_xz = 4 * nnn * pnn * npn * ppn / (nnn * pnn * npn + nnn * pnn * ppn + nnn * npn * ppn + pnn * npn * ppn + EPSL);
                const float dxVz_dzVx = dxVz + dzVx;
                const float f_Rxz = mu_xz * taus1 * dxVz_dzVx;
                float Rxz_n = 0.0f;
    #pragma unroll
                for (int m = 0; m < NM; m++) {
                    r[2][m] = M.c1[m] * r[2][m] - M.c2[m] * f_Rxz * dt;
                    Rxz_n = Rxz_n + M.d1[m] * r[2][m];
                }
                sts(&M.S2[e], sxz + (mu_xz * taus_plus1 * dxVz_dzVx + Rxz_n) * dt);
    #pragma unroll
                for (int c = 0; c < 3; c++)
    #pragma unroll
                    for (int m = 0; m < NM; m++) sts(&M.R[c * 3 + m][e], r[c][m]);
                continue;
            }
            if (!(mask & 2)) continue;
            // absorber (src/swpc_psv/m_absorb_p.f90:337-385)
            const int2 pc = __ldg(&M.pmlcol[i + 2]);
            const long long q = (long long)pc.y + (k - pc.x);
            float *__restrict__ axVx = M.aux[0];
            float *__restrict__ azVx = M.aux[1];
            float *__restrict__ axVz = M.aux[2];
            float *__restrict__ azVz = M.aux[3];
            const float vaxVx = lds(&axVx[q]), vazVx = lds(&azVx[q]), vaxVz = lds(&axVz[q]), vazVz = lds(&azVz[q]);
            const float sxx = lds(&M.S0[e]), szz = lds(&M.S1[e]), sxz = lds(&M.S2[e]);
            const float mu = lds(&M.mu[e]), lam = lds(&M.lam[e]);
            const float pnn = __ldg(&M.mu[e + 1]), npn = __ldg(&M.mu[e + PI]), ppn = __ldg(&M.mu[e + 1 + PI]);
            const float vx0 = __ldg(&Vx[e]), vz0 = __ldg(&Vz[e]);
            const float4 gxc = __ldg(&M.gxc[i - 1]), gxe = __ldg(&M.gxe[i - 1]);
            const float4 gzc = __ldg(&M.gzc[k - 1]), gze = __ldg(&M.gze[k - 1]);
            const float dxVx = (vx0 - __ldg(&Vx[e - PI])) * M.r20[0];
            const float dzVz = (vz0 - __ldg(&Vz[e - 1])) * M.r20[1];
            const float lam2mu_R = lam + 2 * mu;
            const float lam_R = lam2mu_R - 2 * mu;
            const float dxVx_ade = gxc.x * dxVx + gxc.y * vaxVx;
            const float dzVz_ade = gzc.x * dzVz + gzc.y * vazVz;
            sts(&M.S0[e], sxx + (lam2mu_R * dxVx_ade + lam_R * dzVz_ade) * dt);
            sts(&M.S1[e], szz + (lam2mu_R * dzVz_ade + lam_R * dxVx_ade) * dt);
            sts(&axVx[q], gxc.z * vaxVx + gxc.w * dxVx * dt);
            sts(&azVz[q], gzc.z * vazVz + gzc.w * dzVz * dt);
            const float dzVx = (__ldg(&Vx[e + 1]) - vx0) * M.r20[1];
            const float dxVz = (__ldg(&Vz[e + PI]) - vz0) * M.r20[0];
            const float nnn = mu;
            const float muxz = 4 * nnn * pnn * npn * ppn / (nnn * pnn * npn + nnn * pnn * ppn + nnn * npn * ppn + pnn * npn * ppn + EPSL);
            sts(&M.S2[e], sxz + muxz * (gxe.x * dxVz + gze.x * dzVx + gxe.y * vaxVz + gze.y * vazVx) * dt);
            sts(&azVx[q], gze.z * vazVx + gze.w * dzVx * dt);
            sts(&axVz[q], gxe.z * vaxVz + gxe.w * dxVz * dt);
        }
    }
}

// ---------------------------------------------------------------------------
// P-SV velocity: kernel__update_vel + absorb_p__update_vel
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) psv_vel_kernel(const Model2D *__restrict__ models,
                                                      const Tile2D *__restrict__ tiles, int ntiles, int mask,
        int ri) {
    __shared__ Model2D sM;
    int cached = -1;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const Tile2D tl = tiles[t];
        const Model2D &M = tile_model(models, tl.model, sM, cached);
        // ri rows of the tile per thread: the tile and model descriptors are
        // fetched once for ri cells
        for (int r = 0; r < ri; r++) {
            const int k = tl.k0 + threadIdx.x, i = tl.i0 + threadIdx.y + r * (int)blockDim.y;
            if (k > M.nz || i > M.nx) continue;
            const long long PI = M.Kp;
            const long long e = (long long)(i + 2) * PI + (k - 1 + KH);
            const float *__restrict__ Sxx = M.S0;
            const float *__restrict__ Szz = M.S1;
            const float *__restrict__ Sxz = M.S2;
            const float dt = M.dt;
            const float vx = lds(&M.V0[e]), vz = lds(&M.V1[e]);
            const float rho0 = __ldg(&M.rho[e]), rhoi = __ldg(&M.rho[e + PI]), rhok = __ldg(&M.rho[e + 1]);
            const float bx = 2.0f / (rho0 + rhoi);
            const float bz = 2.0f / (rho0 + rhok);
            if (i >= M.ibk && i <= M.iek && k <= M.kek) {
                if (!(mask & 1)) continue;
                const int4 bd = __ldg(&M.band[i + 2]);
                const int p1 = (k - bd.x) * (bd.y - k), p2 = (k - bd.z) * (bd.w - k);
                const int s = ((p1 > p2 ? p1 : p2) >= 0) ? 1 : 0;
                const float re40x = M.e40[0][s], re41x = M.e41[0][s], re40z = M.e40[1][s], re41z = M.e41[1][s];
                const float dxSxx = (__ldg(&Sxx[e + PI]) - __ldg(&Sxx[e])) * re40x - (__ldg(&Sxx[e + 2 * PI]) - __ldg(&Sxx[e - PI])) * re41x;
                const float dzSzz = (__ldg(&Szz[e + 1]) - __ldg(&Szz[e])) * re40z - (__ldg(&Szz[e + 2]) - __ldg(&Szz[e - 1])) * re41z;
                const float dxSxz = (__ldg(&Sxz[e]) - __ldg(&Sxz[e - PI])) * re40x - (__ldg(&Sxz[e + PI]) - __ldg(&Sxz[e - 2 * PI])) * re41x;
                const float dzSxz = (__ldg(&Sxz[e]) - __ldg(&Sxz[e - 1])) * re40z - (__ldg(&Sxz[e + 1]) - __ldg(&Sxz[e - 2])) * re41z;
                sts(&M.V0[e], vx + bx * (dxSxx + dzSxz) * dt);
                sts(&M.V1[e], vz + bz * (dxSxz + dzSzz) * dt);
                continue;
            }
            if (!(mask & 2)) continue;
            const int2 pc = __ldg(&M.pmlcol[i + 2]);
            const long long q = (long long)pc.y + (k - pc.x);
            float *__restrict__ axSxx = M.aux[4];
            float *__restrict__ azSxz = M.aux[5];
            float *__restrict__ axSxz = M.aux[6];
            float *__restrict__ azSzz = M.aux[7];
            const float vxSxx = lds(&axSxx[q]), vzSxz = lds(&azSxz[q]), vxSxz = lds(&axSxz[q]), vzSzz = lds(&azSzz[q]);
            const float4 gxc = __ldg(&M.gxc[i - 1]), gxe = __ldg(&M.gxe[i - 1]);
            const float4 gzc = __ldg(&M.gzc[k - 1]), gze = __ldg(&M.gze[k - 1]);
            const float dxSxx = (__ldg(&Sxx[e + PI]) - __ldg(&Sxx[e])) * M.r20[0];
            const float dzSzz = (__ldg(&Szz[e + 1]) - __ldg(&Szz[e])) * M.r20[1];
            const float dxSxz = (__ldg(&Sxz[e]) - __ldg(&Sxz[e - PI])) * M.r20[0];
            const float dzSxz = (__ldg(&Sxz[e]) - __ldg(&Sxz[e - 1])) * M.r20[1];
            sts(&M.V0[e], vx + bx * (gxe.x * dxSxx + gzc.x * dzSxz + gxe.y * vxSxx + gzc.y * vzSxz) * dt);
            sts(&M.V1[e], vz + bz * (gxc.x * dxSxz + gze.x * dzSzz + gxc.y * vxSxz + gze.y * vzSzz) * dt);
            sts(&axSxx[q], gxe.z * vxSxx + gxe.w * dxSxx * dt);
            sts(&azSxz[q], gzc.z * vzSxz + gzc.w * dzSxz * dt);
            sts(&axSxz[q], gxc.z * vxSxz + gxc.w * dxSxz * dt);
            sts(&azSzz[q], gze.z * vzSzz + gze.w * dzSzz * dt);
        }
    }
}

// ---------------------------------------------------------------------------
// SH stress: kernel__update_stress + absorb_p__update_stress
// ---------------------------------------------------------------------------
template <int NM>
__global__ void __launch_bounds__(256) sh_stress_kernel(const Model2D *__restrict__ models,
                                                        const Tile2D *__restrict__ tiles, int ntiles, int mask,
        int ri) {
    __shared__ Model2D sM;
    int cached = -1;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const Tile2D tl = tiles[t];
        const Model2D &M = tile_model(models, tl.model, sM, cached);
        // ri rows of the tile per thread: the tile and model descriptors are
        // fetched once for ri cells
        for (int r = 0; r < ri; r++) {
            const int k = tl.k0 + threadIdx.x, i = tl.i0 + threadIdx.y + r * (int)blockDim.y;
            if (k > M.nz || i > M.nx) continue;
            const long long PI = M.Kp;
            const long long e = (long long)(i + 2) * PI + (k - 1 + KH);
            const float *__restrict__ Vy = M.V0;
            const float dt = M.dt;
            const float syz = lds(&M.S0[e]), sxy = lds(&M.S1[e]);
            const float nnn = lds(&M.mu[e]), pnn = __ldg(&M.mu[e + 1]), npn = __ldg(&M.mu[e + PI]);
            const float vy0 = __ldg(&Vy[e]);
            const float mu_xy = 2 * nnn * npn / (nnn + npn + EPSL);
            const float mu_yz = 2 * nnn * pnn / (nnn + pnn + EPSL);
            if (i >= M.ibk && i <= M.iek && k <= M.kek) {
                if (!(mask & 1)) continue;
                float r[2][NM > 0 ? NM : 1];
    #pragma unroll
                for (int c = 0; c < 2; c++)
    #pragma unroll
                    for (int m = 0; m < NM; m++) r[c][m] = lds(&M.R[c * 3 + m][e]);
                const float taus1 = lds(&M.taus[e]);
                const int4 bd = __ldg(&M.band[i + 2]);
                const int p1 = (k - bd.x) * (bd.y - k), p2 = (k - bd.z) * (bd.w - k);
                const int s = ((p1 > p2 ? p1 : p2) >= 0) ? 1 : 0;
                const float re40x = M.e40[0][s], re41x = M.e41[0][s], re40z = M.e40[1][s], re41z = M.e41[1][s];
                const float dxVy = (__ldg(&Vy[e + PI]) - vy0) * re40x - (__ldg(&Vy[e + 2 * PI]) - __ldg(&Vy[e - PI])) * re41x;
                const float dzVy = (__ldg(&Vy[e + 1]) - vy0) * re40z - (__ldg(&Vy[e + 2]) - __ldg(&Vy[e - 1])) * re41z;
                const float f_Ryz = mu_yz * taus1 * dzVy;
                const float f_Rxy = mu_xy * taus1 * dxVy;
                float Ryz_n = 0.0f, Rxy_n = 0.0f;
    #pragma unroll
                for (int m = 0; m < NM; m++) {
                    r[0][m] = M.c1[m] * r[0][m] - M.c2[m] * f_Ryz * dt;
                    r[1][m] = M.c1[m] * r[1][m] - M.c2[m] * f_Rxy * dt;
                    Ryz_n = Ryz_n + M.d1[m] * r[0][m];
                    Rxy_n = Rxy_n + M.d1[m] * r[1][m];
                }
                const float taus_plus1 = 1 + taus1 * (1 + M.d2);
                sts(&M.S0[e], syz + (mu_yz * taus_plus1 * dzVy + Ryz_n) * dt);
                sts(&M.S1[e], sxy + (mu_xy * taus_plus1 * dxVy + Rxy_n) * dt);
    #pragma unroll
                for (int c = 0; c < 2; c++)
    #pragma unroll
                    for (int m = 0; m < NM; m++) sts(&M.R[c * 3 + m][e], r[c][m]);
                continue;
            }
            if (!(mask & 2)) continue;
            const int2 pc = __ldg(&M.pmlcol[i + 2]);
            const long long q = (long long)pc.y + (k - pc.x);
            float *__restrict__ axVy = M.aux[0];
            float *__restrict__ azVy = M.aux[1];
            const float4 gxe = __ldg(&M.gxe[i - 1]);
            const float4 gze = __ldg(&M.gze[k - 1]);
            const float dxVy = (__ldg(&Vy[e + PI]) - vy0) * M.r20[0];
            const float dzVy = (__ldg(&Vy[e + 1]) - vy0) * M.r20[1];
            // the auxiliaries are advanced first and then used (src/swpc_sh/m_absorb_p.f90)
            const float ax = gxe.z * lds(&axVy[q]) + gxe.w * dxVy * dt;
            const float az = gze.z * lds(&azVy[q]) + gze.w * dzVy * dt;
            sts(&axVy[q], ax);
            sts(&azVy[q], az);
            sts(&M.S0[e], syz + mu_yz * (gze.x * dzVy + gze.y * az) * dt);
            sts(&M.S1[e], sxy + mu_xy * (gxe.x * dxVy + gxe.y * ax) * dt);
        }
    }
}

// ---------------------------------------------------------------------------
// SH velocity: kernel__update_vel + absorb_p__update_vel
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) sh_vel_kernel(const Model2D *__restrict__ models,
                                                     const Tile2D *__restrict__ tiles, int ntiles, int mask,
        int ri) {
    __shared__ Model2D sM;
    int cached = -1;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const Tile2D tl = tiles[t];
        const Model2D &M = tile_model(models, tl.model, sM, cached);
        // ri rows of the tile per thread: the tile and model descriptors are
        // fetched once for ri cells
        for (int r = 0; r < ri; r++) {
            const int k = tl.k0 + threadIdx.x, i = tl.i0 + threadIdx.y + r * (int)blockDim.y;
            if (k > M.nz || i > M.nx) continue;
            const long long PI = M.Kp;
            const long long e = (long long)(i + 2) * PI + (k - 1 + KH);
            const float *__restrict__ Syz = M.S0;
            const float *__restrict__ Sxy = M.S1;
            const float dt = M.dt;
            const float vy = lds(&M.V0[e]);
            const float by = 1.0f / lds(&M.rho[e]);
            if (i >= M.ibk && i <= M.iek && k <= M.kek) {
                if (!(mask & 1)) continue;
                const int4 bd = __ldg(&M.band[i + 2]);
                const int p1 = (k - bd.x) * (bd.y - k), p2 = (k - bd.z) * (bd.w - k);
                const int s = ((p1 > p2 ? p1 : p2) >= 0) ? 1 : 0;
                const float re40x = M.e40[0][s], re41x = M.e41[0][s], re40z = M.e40[1][s], re41z = M.e41[1][s];
                const float dzSyz = (__ldg(&Syz[e]) - __ldg(&Syz[e - 1])) * re40z - (__ldg(&Syz[e + 1]) - __ldg(&Syz[e - 2])) * re41z;
                const float dxSxy = (__ldg(&Sxy[e]) - __ldg(&Sxy[e - PI])) * re40x - (__ldg(&Sxy[e + PI]) - __ldg(&Sxy[e - 2 * PI])) * re41x;
                sts(&M.V0[e], vy + by * (dxSxy + dzSyz) * dt);
                continue;
            }
            if (!(mask & 2)) continue;
            const int2 pc = __ldg(&M.pmlcol[i + 2]);
            const long long q = (long long)pc.y + (k - pc.x);
            float *__restrict__ axSxy = M.aux[2];
            float *__restrict__ azSyz = M.aux[3];
            const float vxSxy = lds(&axSxy[q]), vzSyz = lds(&azSyz[q]);
            const float4 gxc = __ldg(&M.gxc[i - 1]);
            const float4 gzc = __ldg(&M.gzc[k - 1]);
            const float dzSyz = (__ldg(&Syz[e]) - __ldg(&Syz[e - 1])) * M.r20[1];
            const float dxSxy = (__ldg(&Sxy[e]) - __ldg(&Sxy[e - PI])) * M.r20[0];
            sts(&M.V0[e], vy + by * (gxc.x * dxSxy + gzc.x * dzSyz + gxc.y * vxSxy + gzc.y * vzSyz) * dt);
            sts(&axSxy[q], gxc.z * vxSxy + gxc.w * dxSxy * dt);
            sts(&azSyz[q], gzc.z * vzSyz + gzc.w * dzSyz * dt);
        }
    }
}

// ---------------------------------------------------------------------------
// recorder (src/swpc_psv/m_wav.f90:170-260, src/swpc_sh/m_wav.f90:170-250)
// and vmax (src/swpc_psv/m_kernel.f90:308-324)
// ---------------------------------------------------------------------------
__global__ void wav2d_kernel(const Wav2Args *__restrict__ list, int nlist, int it_arg, const int *d_it) {
    const int it = d_it ? *d_it : it_arg;
    for (int b = blockIdx.y; b < nlist; b += gridDim.y) {
        const Wav2Args &a = list[b];
        for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < a.nst; n += gridDim.x * blockDim.x) {
            const int i = a.st[2 * n], k = a.st[2 * n + 1];
            const long long PI = a.Kp;
            const long long e = (long long)(i + 2) * PI + (k - 1 + KH);
            const float dt = a.dt;
            if (a.what & SWPC_WAV_U) {
                if (a.psv) {
                    a.uacc[2 * n] = a.uacc[2 * n] + (a.V0[e] + a.V0[e - PI]) * 0.5f * dt;
                    a.uacc[2 * n + 1] = a.uacc[2 * n + 1] - (a.V1[e] + a.V1[e - 1]) * 0.5f * dt;
                } else {
                    a.uacc[2 * n] = a.uacc[2 * n] + a.V0[e] * dt;
                }
            }
            if (it < 1 || (it - 1) % a.ntdec_w != 0) continue;
            const int itw = (it - 1) / a.ntdec_w + 1;
            if (itw > a.ntw) continue;
            const long long ntw = a.ntw;
            const int nc = a.psv ? 2 : 1;
            const float M0 = a.M0, UC = a.UC;
            if (a.what & SWPC_WAV_V) {
                float *w = a.wav_v + (long long)n * nc * ntw + (itw - 1);
                if (a.psv) {
                    w[0] = (a.V0[e] + a.V0[e - PI]) / 2.0f * M0 * UC * 1e9f;
                    w[ntw] = -(a.V1[e] + a.V1[e - 1]) / 2.0f * M0 * UC * 1e9f;
                } else {
                    w[0] = a.V0[e] * M0 * UC * 1e9f;
                }
            }
            if (a.what & SWPC_WAV_U) {
                float *w = a.wav_u + (long long)n * nc * ntw + (itw - 1);
                w[0] = a.uacc[2 * n] * M0 * UC * 1e9f;
                if (a.psv) w[ntw] = a.uacc[2 * n + 1] * M0 * UC * 1e9f;
            }
        }
    }
}

__global__ void vmax2d_kernel(const float *V0, const float *V1, const int *kob, int Kp, int i0, int i1,
                              unsigned int *out) {
    unsigned int a = 0, b = 0;
    for (int i = i0 + blockIdx.x * blockDim.x + threadIdx.x; i <= i1; i += gridDim.x * blockDim.x) {
        const int k = kob[i + 2] + 1;
        const long long e = (long long)(i + 2) * Kp + (k - 1 + KH);
        a = max(a, __float_as_uint(fabsf(V0[e])));
        if (V1) b = max(b, __float_as_uint(fabsf(V1[e])));
    }
    for (int o = 16; o > 0; o >>= 1) {
        a = max(a, __shfl_xor_sync(0xffffffffu, a, o));
        b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&out[0], a);
        atomicMax(&out[1], b);
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int persistent_grid(int ntiles, int blocks_per_sm) {
    // 148 SMs x blocks_per_sm resident blocks, never more blocks than tiles;
    // blocks_per_sm = 0: one block per tile
    const int g = blocks_per_sm > 0 ? 148 * blocks_per_sm : ntiles;
    return ntiles < g ? (ntiles > 0 ? ntiles : 1) : g;
}

void launch_stress2d(int kind, int nm, const Model2D *models, const Tile2D *tiles, int ntiles, int mask,
                     TileShape ts, cudaStream_t st) {
    const dim3 block(32, ts.ti);
    const int grid = persistent_grid(ntiles, ts.blocks_per_sm);
    if (kind == SWPC_KIND_PSV) {
        switch (nm) {
        case 0: psv_stress_kernel<0><<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri); break;
        case 1: psv_stress_kernel<1><<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri); break;
        case 2: psv_stress_kernel<2><<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri); break;
        default: psv_stress_kernel<3><<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri); break;
        }
    } else {
        switch (nm) {
        case 0: sh_stress_kernel<0><<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri); break;
        case 1: sh_stress_kernel<1><<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri); break;
        case 2: sh_stress_kernel<2><<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri); break;
        default: sh_stress_kernel<3><<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri); break;
        }
    }
}

void launch_vel2d(int kind, const Model2D *models, const Tile2D *tiles, int ntiles, int mask, TileShape ts,
                  cudaStream_t st) {
    const dim3 block(32, ts.ti);
    const int grid = persistent_grid(ntiles, ts.blocks_per_sm);
    if (kind == SWPC_KIND_PSV) psv_vel_kernel<<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri);
    else sh_vel_kernel<<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri);
}

void launch_wav2d(const Wav2Args *list, int nlist, int max_nst, int it, const int *d_it, cudaStream_t st) {
    if (nlist <= 0 || max_nst <= 0) return;
    const int threads = 128;
    const dim3 grid((max_nst + threads - 1) / threads, nlist < 65535 ? nlist : 65535);
    wav2d_kernel<<<grid, threads, 0, st>>>(list, nlist, it, d_it);
}

void launch_vmax2d(const float *V0, const float *V1, const int *kob, int Kp, int i0, int i1, unsigned int *out,
                   cudaStream_t st) {
    vmax2d_kernel<<<8, 256, 0, st>>>(V0, V1, kob, Kp, i0, i1, out);
}

}  // namespace swpc
