// swpc_kernels.cuh -- launch argument blocks of the device kernels.
#pragma once

#include <cuda_runtime.h>

#include "swpc_ctx.h"

namespace swpc {

enum InjMode { INJ_GLUT = 0, INJ_GLUT4 = 1, INJ_GLUT2 = 2, INJ_BF3 = 3, INJ_GREEN = 4, INJ_BFPSV = 5, INJ_BFSH = 6 };

// Power-of-two scales of the FP16 storage forms, in device memory (so that
// re-centring them needs no new launch arguments): value = stored * sS[f]
// for stress array f, stored = value * iS[f], and sR, iR for the memory
// variables, which share one scale (FP16 keeps 11 significant bits over 29
// binades, so arrays that differ by orders of magnitude lose nothing by
// sharing it, and the stress kernel reads it from one read-only address).
// Layout: [0..5] sS_in, [6] sR_in (what the stored values meant before this
// step's stress update: only the stress kernel reads them), [7..12] sS,
// [13..18] iS, [19] sR, [20] iR (what it writes, and what every other kernel
// and transfer uses).  A re-centring changes the latter before the stress
// update, which converts every value as it rewrites it; the former follow
// after it.  FP32 storage keeps them 1.
constexpr int kScaleFloats = 48;
__device__ __forceinline__ float sc_sS_in(const float *s, int f) { return __ldg(s + f); }
__device__ __forceinline__ float sc_sR_in(const float *s) { return __ldg(s + 6); }
__device__ __forceinline__ float sc_sS(const float *s, int f) { return __ldg(s + 7 + f); }
__device__ __forceinline__ float sc_iS(const float *s, int f) { return __ldg(s + 13 + f); }
__device__ __forceinline__ float sc_sR(const float *s, int) { return __ldg(s + 19); }
__device__ __forceinline__ float sc_iR(const float *s, int) { return __ldg(s + 20); }

struct Vel3Args {
    Geo g;
    int ibk, iek, jbk, jek, kek;
    float *Vx, *Vy, *Vz;
    const float *Sxx, *Syy, *Szz, *Syz, *Sxz, *Sxy;
    const float *bx, *by, *bz;
    const int4 *band;
    const int2 *pmlcol;
    float *aS[9];   // axSxx aySxy azSxz axSxy aySyy azSyz axSxz aySyz azSzz
    const float4 *gxc, *gxe, *gyc, *gye, *gzc, *gze;
    float e40[3][2], e41[3][2];
    float r20[3];
    float dt;
    int mask;       // bit 0: interior cells, bit 1: absorber cells
    const float *scale;   // FP16 scales in device memory (see sc_sS)
    // where not null, the interior cells also store their stress divergences (the gradient's kept steps): field c
    // of cell (k, i, j) at divo[c * dn + ((j - dj0) * dIp + (i - di0)) * dKp + k - 1 + KH]
    float *divo;
    int dKp, dIp, di0, dj0;
    long long dn;
};

struct Str3Args {
    Geo g;
    int ibk, iek, jbk, jek, kek;
    const float *Vx, *Vy, *Vz;
    float *Sxx, *Syy, *Szz, *Syz, *Sxz, *Sxy;
    float *R[18];
    const float *lam, *mu, *taup, *taus, *muyz, *muxz, *muxy;
    const int4 *band;
    const int2 *pmlcol;
    float *aV[9];   // axVx ayVx azVx axVy ayVy azVy axVz ayVz azVz
    const float4 *gxc, *gxe, *gyc, *gye, *gzc, *gze;
    float e40[3][2], e41[3][2];
    float r20[3];
    float c1[NM_MAX], c2[NM_MAX], d1[NM_MAX], d2;
    float dt;
    int mask;
    const float *scale;     // FP16 stress and memory-variable scales in device memory (see sc_sS)
};

struct InjArgs {
    const InjEntry *list;
    int n;
    int serial;
    int it;              // used when d_it is null
    const int *d_it;     // step counter for graph replays
    int nt;
    int nsrc;
    const float *stime;  // (nt, nsrc)
    const float *mo;     // (nsrc) for stress glut
    float dt_dxyz;
    float *fields[9];    // V (0..2) and S (3..8) by SWPC_F_* id
    const float *bfields[3];
    const long long *rho_cell;   // (nsrc) density cell of 2D body forces
    int s_half;          // S stored in FP16 (SWPC_PREC_F16_SR)
    const float *scale;  // its scales in device memory (see sc_sS)
};

struct Wav3Args {
    Geo g;
    int nst, ntw, ntdec_w, what;
    int it;
    const int *d_it;
    const int *st;       // (3, nst) i j k
    const float *Vx, *Vy, *Vz;
    const float *Sxx, *Syy, *Szz, *Syz, *Sxz, *Sxy;
    float *uacc, *eacc;
    float *wav_v, *wav_u, *wav_s, *wav_e;
    float M0, UC, dt;
    float r40[3], r41[3];
    int s_half;          // S stored in FP16 (SWPC_PREC_F16_SR)
    const float *scale;
};

struct VmaxArgs {
    Geo g;
    int i0, i1, j0, j1;
    const int *kob;
    const float *Vx, *Vy, *Vz;
    unsigned int *out;
};

void launch_vel3d(const Vel3Args &a, int minb, int prec, dim3 grid, dim3 block, cudaStream_t st);
void launch_stress3d(const Str3Args &a, int nm, int minb, int prec, dim3 grid, dim3 block, cudaStream_t st);
void launch_stress3d_march(const Str3Args &a, int nm, int minb, int jc, cudaStream_t st);
void launch_vel3d_march(const Vel3Args &a, int minb, int jc, cudaStream_t st);
void launch_vel3d_vec(const Vel3Args &a, int minb, dim3 block, cudaStream_t st);
void launch_inject(const InjArgs &a, cudaStream_t st);
void launch_inject_multi(const InjArgs *list, int nlist, int max_n, const int *d_it, int it, cudaStream_t st);
void launch_wav3d(const Wav3Args &a, cudaStream_t st);
void launch_vmax3d(const VmaxArgs &a, cudaStream_t st);
void launch_advance_it(int *d_it, cudaStream_t st);

}  // namespace swpc
