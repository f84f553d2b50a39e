// swpc3d_cell.cuh -- per-cell device routines shared by the 3D kernels.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "swpc_ctx.h"
#include "swpc_kernels.cuh"

namespace swpc {

// streaming accesses: every value below is touched once per launch, so they
// are loaded and stored with the evict-first hint and leave L2 to the
// stencil operands that neighbouring blocks re-read
__device__ __forceinline__ float lds(const float *p) { return __ldcs(p); }
__device__ __forceinline__ void sts(float *p, float v) { __stcs(p, v); }

// Storage precision of the stress (S) and memory-variable (R) arrays; the
// arithmetic is FP32 in every form.
//   PREC_F32   : S and R in FP32 (the reference's MP = SP build)
//   PREC_BF16_R: R stored in BF16
//   PREC_F16_SR: S and R stored in FP16, each array with its own power-of-two
//                scale: value = stored * s, stored = value * (1 / s) (exact)
enum { PREC_F32 = 0, PREC_BF16_R = 1, PREC_F16_SR = 2 };

template <int PREC>
__device__ __forceinline__ float ldS(const float *p, long long e, float s) {
    if constexpr (PREC == PREC_F16_SR) return __half2float(__ldcs(reinterpret_cast<const __half *>(p) + e)) * s;
    else return __ldcs(p + e);
}
template <int PREC>
__device__ __forceinline__ float ldgS(const float *p, long long e, float s) {
    if constexpr (PREC == PREC_F16_SR) return __half2float(__ldg(reinterpret_cast<const __half *>(p) + e)) * s;
    else return __ldg(p + e);
}
template <int PREC>
__device__ __forceinline__ void stS(float *p, long long e, float v, float is) {
    if constexpr (PREC == PREC_F16_SR) __stcs(reinterpret_cast<__half *>(p) + e, __float2half_rn(v * is));
    else __stcs(p + e, v);
}
template <int PREC>
__device__ __forceinline__ float ldR(const float *p, long long e, float s) {
    if constexpr (PREC == PREC_F16_SR) return __half2float(__ldcs(reinterpret_cast<const __half *>(p) + e)) * s;
    else if constexpr (PREC == PREC_BF16_R)
        return __bfloat162float(__ldcs(reinterpret_cast<const __nv_bfloat16 *>(p) + e));
    else return __ldcs(p + e);
}
template <int PREC>
__device__ __forceinline__ void stR(float *p, long long e, float v, float is) {
    if constexpr (PREC == PREC_F16_SR) __stcs(reinterpret_cast<__half *>(p) + e, __float2half_rn(v * is));
    else if constexpr (PREC == PREC_BF16_R) __stcs(reinterpret_cast<__nv_bfloat16 *>(p) + e, __float2bfloat16_rn(v));
    else __stcs(p + e, v);
}

// ---------------------------------------------------------------------------
// velocity: kernel__update_vel (m_kernel.f90:75-140) +
//           absorb_p__update_vel (m_absorb_p.f90:248-309)
// ---------------------------------------------------------------------------
// One cell (k, i, j) of the fused velocity update.  All loads of the cell are
// issued before its first store: the arrays never alias, and with every
// operand in flight at once the update is limited by HBM bandwidth instead of
// by load latency.
template <int PREC>
__device__ __forceinline__ void vel_cell(const Vel3Args &a, int k, int i, int j) {
    const Geo g = a.g;
    const long long col = col_index(g, i, j);
    const long long e = col * g.Kp + (k - 1 + KH);
    const long long PI = g.Kp;
    const long long PJ = (long long)g.Kp * g.Ip;
    const float *__restrict__ Sxx = a.Sxx;
    const float *__restrict__ Syy = a.Syy;
    const float *__restrict__ Szz = a.Szz;
    const float *__restrict__ Syz = a.Syz;
    const float *__restrict__ Sxz = a.Sxz;
    const float *__restrict__ Sxy = a.Sxy;
    float *__restrict__ Vx = a.Vx;
    float *__restrict__ Vy = a.Vy;
    float *__restrict__ Vz = a.Vz;
    const float dt = a.dt;

    if (i >= a.ibk && i <= a.iek && j >= a.jbk && j <= a.jek && k <= a.kek) {
        if (!(a.mask & 1)) return;
        const float vx = lds(&Vx[e]), vy = lds(&Vy[e]), vz = lds(&Vz[e]);
        const float bx = lds(&a.bx[e]), by = lds(&a.by[e]), bz = lds(&a.bz[e]);
        const float xx0 = ldgS<PREC>(Sxx, e, a.sS[0]), xxp = ldgS<PREC>(Sxx, e + PI, a.sS[0]), xxp2 = ldgS<PREC>(Sxx, e + 2 * PI, a.sS[0]), xxm = ldgS<PREC>(Sxx, e - PI, a.sS[0]);
        const float yy0 = ldgS<PREC>(Syy, e, a.sS[1]), yyp = ldgS<PREC>(Syy, e + PJ, a.sS[1]), yyp2 = ldgS<PREC>(Syy, e + 2 * PJ, a.sS[1]), yym = ldgS<PREC>(Syy, e - PJ, a.sS[1]);
        const float zz0 = ldgS<PREC>(Szz, e, a.sS[2]), zzp = ldgS<PREC>(Szz, e + 1, a.sS[2]), zzp2 = ldgS<PREC>(Szz, e + 2, a.sS[2]), zzm = ldgS<PREC>(Szz, e - 1, a.sS[2]);
        const float xy0 = ldgS<PREC>(Sxy, e, a.sS[5]);
        const float xyjm = ldgS<PREC>(Sxy, e - PJ, a.sS[5]), xyjp = ldgS<PREC>(Sxy, e + PJ, a.sS[5]), xyjm2 = ldgS<PREC>(Sxy, e - 2 * PJ, a.sS[5]);
        const float xyim = ldgS<PREC>(Sxy, e - PI, a.sS[5]), xyip = ldgS<PREC>(Sxy, e + PI, a.sS[5]), xyim2 = ldgS<PREC>(Sxy, e - 2 * PI, a.sS[5]);
        const float xz0 = ldgS<PREC>(Sxz, e, a.sS[4]);
        const float xzkm = ldgS<PREC>(Sxz, e - 1, a.sS[4]), xzkp = ldgS<PREC>(Sxz, e + 1, a.sS[4]), xzkm2 = ldgS<PREC>(Sxz, e - 2, a.sS[4]);
        const float xzim = ldgS<PREC>(Sxz, e - PI, a.sS[4]), xzip = ldgS<PREC>(Sxz, e + PI, a.sS[4]), xzim2 = ldgS<PREC>(Sxz, e - 2 * PI, a.sS[4]);
        const float yz0 = ldgS<PREC>(Syz, e, a.sS[3]);
        const float yzkm = ldgS<PREC>(Syz, e - 1, a.sS[3]), yzkp = ldgS<PREC>(Syz, e + 1, a.sS[3]), yzkm2 = ldgS<PREC>(Syz, e - 2, a.sS[3]);
        const float yzjm = ldgS<PREC>(Syz, e - PJ, a.sS[3]), yzjp = ldgS<PREC>(Syz, e + PJ, a.sS[3]), yzjm2 = ldgS<PREC>(Syz, e - 2 * PJ, a.sS[3]);
        const int4 bd = __ldg(&a.band[col]);
        const int p1 = (k - bd.x) * (bd.y - k);
        const int p2 = (k - bd.z) * (bd.w - k);
        const int s = ((p1 > p2 ? p1 : p2) >= 0) ? 1 : 0;   // isign = +1 -> 2nd-order band
        const float re40x = a.e40[0][s], re41x = a.e41[0][s];
        const float re40y = a.e40[1][s], re41y = a.e41[1][s];
        const float re40z = a.e40[2][s], re41z = a.e41[2][s];

        const float d3Sx3 = (xxp - xx0) * re40x - (xxp2 - xxm) * re41x
                          + (xy0 - xyjm) * re40y - (xyjp - xyjm2) * re41y
                          + (xz0 - xzkm) * re40z - (xzkp - xzkm2) * re41z;
        const float d3Sy3 = (xy0 - xyim) * re40x - (xyip - xyim2) * re41x
                          + (yyp - yy0) * re40y - (yyp2 - yym) * re41y
                          + (yz0 - yzkm) * re40z - (yzkp - yzkm2) * re41z;
        const float d3Sz3 = (xz0 - xzim) * re40x - (xzip - xzim2) * re41x
                          + (yz0 - yzjm) * re40y - (yzjp - yzjm2) * re41y
                          + (zzp - zz0) * re40z - (zzp2 - zzm) * re41z;
        sts(&Vx[e], vx + bx * d3Sx3 * dt);
        sts(&Vy[e], vy + by * d3Sy3 * dt);
        sts(&Vz[e], vz + bz * d3Sz3 * dt);
        return;
    }

    // absorber cell: k >= kbeg_a(i, j) holds for every cell outside the kernel box
    if (!(a.mask & 2)) return;
    const int2 pc = __ldg(&a.pmlcol[col]);
    const long long q = (long long)pc.y + (k - pc.x);
    float *__restrict__ axSxx = a.aS[0];
    float *__restrict__ aySxy = a.aS[1];
    float *__restrict__ azSxz = a.aS[2];
    float *__restrict__ axSxy = a.aS[3];
    float *__restrict__ aySyy = a.aS[4];
    float *__restrict__ azSyz = a.aS[5];
    float *__restrict__ axSxz = a.aS[6];
    float *__restrict__ aySyz = a.aS[7];
    float *__restrict__ azSzz = a.aS[8];
    const float vxSxx = lds(&axSxx[q]), vySxy = lds(&aySxy[q]), vzSxz = lds(&azSxz[q]);
    const float vxSxy = lds(&axSxy[q]), vySyy = lds(&aySyy[q]), vzSyz = lds(&azSyz[q]);
    const float vxSxz = lds(&axSxz[q]), vySyz = lds(&aySyz[q]), vzSzz = lds(&azSzz[q]);
    const float vx = lds(&Vx[e]), vy = lds(&Vy[e]), vz = lds(&Vz[e]);
    const float bx = lds(&a.bx[e]), by = lds(&a.by[e]), bz = lds(&a.bz[e]);
    const float xx0 = ldgS<PREC>(Sxx, e, a.sS[0]), xxp = ldgS<PREC>(Sxx, e + PI, a.sS[0]);
    const float yy0 = ldgS<PREC>(Syy, e, a.sS[1]), yyp = ldgS<PREC>(Syy, e + PJ, a.sS[1]);
    const float zz0 = ldgS<PREC>(Szz, e, a.sS[2]), zzp = ldgS<PREC>(Szz, e + 1, a.sS[2]);
    const float yz0 = ldgS<PREC>(Syz, e, a.sS[3]), yzjm = ldgS<PREC>(Syz, e - PJ, a.sS[3]), yzkm = ldgS<PREC>(Syz, e - 1, a.sS[3]);
    const float xz0 = ldgS<PREC>(Sxz, e, a.sS[4]), xzim = ldgS<PREC>(Sxz, e - PI, a.sS[4]), xzkm = ldgS<PREC>(Sxz, e - 1, a.sS[4]);
    const float xy0 = ldgS<PREC>(Sxy, e, a.sS[5]), xyim = ldgS<PREC>(Sxy, e - PI, a.sS[5]), xyjm = ldgS<PREC>(Sxy, e - PJ, a.sS[5]);
    const float4 gxc = __ldg(&a.gxc[i - 1]), gxe = __ldg(&a.gxe[i - 1]);
    const float4 gyc = __ldg(&a.gyc[j - 1]), gye = __ldg(&a.gye[j - 1]);
    const float4 gzc = __ldg(&a.gzc[k - 1]), gze = __ldg(&a.gze[k - 1]);
    const float r20x = a.r20[0], r20y = a.r20[1], r20z = a.r20[2];
    const float dxSxx = (xxp - xx0) * r20x;
    const float dySyy = (yyp - yy0) * r20y;
    const float dzSzz = (zzp - zz0) * r20z;
    const float dySyz = (yz0 - yzjm) * r20y;
    const float dzSyz = (yz0 - yzkm) * r20z;
    const float dxSxz = (xz0 - xzim) * r20x;
    const float dzSxz = (xz0 - xzkm) * r20z;
    const float dxSxy = (xy0 - xyim) * r20x;
    const float dySxy = (xy0 - xyjm) * r20y;

    sts(&Vx[e], vx + bx * (gxe.x * dxSxx + gyc.x * dySxy + gzc.x * dzSxz
                           + gxe.y * vxSxx + gyc.y * vySxy + gzc.y * vzSxz) * dt);
    sts(&Vy[e], vy + by * (gxc.x * dxSxy + gye.x * dySyy + gzc.x * dzSyz
                           + gxc.y * vxSxy + gye.y * vySyy + gzc.y * vzSyz) * dt);
    sts(&Vz[e], vz + bz * (gxc.x * dxSxz + gyc.x * dySyz + gze.x * dzSzz
                           + gxc.y * vxSxz + gyc.y * vySyz + gze.y * vzSzz) * dt);

    sts(&axSxx[q], gxe.z * vxSxx + gxe.w * dxSxx * dt);
    sts(&aySxy[q], gyc.z * vySxy + gyc.w * dySxy * dt);
    sts(&azSxz[q], gzc.z * vzSxz + gzc.w * dzSxz * dt);
    sts(&axSxy[q], gxc.z * vxSxy + gxc.w * dxSxy * dt);
    sts(&aySyy[q], gye.z * vySyy + gye.w * dySyy * dt);
    sts(&azSyz[q], gzc.z * vzSyz + gzc.w * dzSyz * dt);
    sts(&axSxz[q], gxc.z * vxSxz + gxc.w * dxSxz * dt);
    sts(&aySyz[q], gyc.z * vySyz + gyc.w * dySyz * dt);
    sts(&azSzz[q], gze.z * vzSzz + gze.w * dzSzz * dt);
}


}  // namespace swpc
