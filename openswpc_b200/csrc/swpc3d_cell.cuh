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
//   PREC_F16_SR: S and R stored in FP16, with a power-of-two scale per
//                stress array and one for the memory variables: value =
//                stored * s, stored = value * (1 / s) (exact)
//   PREC_F16_R : R stored in FP16 with its scale, S in FP32
enum { PREC_F32 = 0, PREC_BF16_R = 1, PREC_F16_SR = 2, PREC_F16_R = 3 };
// the forms whose R lives in the 2-byte slab and S in the FP32 one
template <int PREC>
__host__ __device__ constexpr bool r_only_half() { return PREC == PREC_BF16_R || PREC == PREC_F16_R; }

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
    if constexpr (PREC == PREC_F16_SR || PREC == PREC_F16_R)
        return __half2float(__ldcs(reinterpret_cast<const __half *>(p) + e)) * s;
    else if constexpr (PREC == PREC_BF16_R)
        return __bfloat162float(__ldcs(reinterpret_cast<const __nv_bfloat16 *>(p) + e));
    else return __ldcs(p + e);
}
template <int PREC>
__device__ __forceinline__ void stR(float *p, long long e, float v, float is) {
    if constexpr (PREC == PREC_F16_SR || PREC == PREC_F16_R)
        __stcs(reinterpret_cast<__half *>(p) + e, __float2half_rn(v * is));
    else if constexpr (PREC == PREC_BF16_R) __stcs(reinterpret_cast<__nv_bfloat16 *>(p) + e, __float2bfloat16_rn(v));
    else __stcs(p + e, v);
}

// 2nd-order band of the free surface / ocean bottom (m_kernel.f90:103-108):
// isign = sign(1, max(...)) = +1 -> index 1 of the coefficient pairs
__device__ __forceinline__ int band_sign_of(const int4 *band, long long col, int k) {
    const int4 bd = __ldg(&band[col]);
    const int p1 = (k - bd.x) * (bd.y - k);
    const int p2 = (k - bd.z) * (bd.w - k);
    return ((p1 > p2 ? p1 : p2) >= 0) ? 1 : 0;
}

// Operands of the interior updates.  The one-cell kernels read them from
// global memory (GVelOps, GStrOps); the staged kernels (swpc3d_tma.cu) from
// the tiles that TMA copied to shared memory.  s(f, dk, di, dj) is stress
// component f (xx yy zz yz xz xy) at (k+dk, i+di, j+dj), v(c, ...) velocity
// component c (x y z).
template <int PREC>
struct GVelOps {
    const Vel3Args &a;
    long long e, PI, PJ;
    const float *S[6];
    const float *V[3];
    __device__ __forceinline__ float v(int c) const { return lds(&V[c][e]); }
    __device__ __forceinline__ float b(int c) const { return lds(&(c == 0 ? a.bx : c == 1 ? a.by : a.bz)[e]); }
    __device__ __forceinline__ float s(int f, int dk, int di, int dj) const {
        return ldgS<PREC>(S[f], e + dk + di * PI + dj * PJ, sc_sS(a.scale, f));
    }
};

// kernel__update_vel (m_kernel.f90:103-125) for one interior cell
template <int PREC, class Ops>
__device__ __forceinline__ void vel_interior(const Vel3Args &a, const Ops &o, int s, float *Vx, float *Vy, float *Vz,
                                             long long e) {
    const float dt = a.dt;
    const float vx = o.v(0), vy = o.v(1), vz = o.v(2);
    const float bx = o.b(0), by = o.b(1), bz = o.b(2);
    const float xx0 = o.s(0, 0, 0, 0), xxp = o.s(0, 0, 1, 0), xxp2 = o.s(0, 0, 2, 0), xxm = o.s(0, 0, -1, 0);
    const float yy0 = o.s(1, 0, 0, 0), yyp = o.s(1, 0, 0, 1), yyp2 = o.s(1, 0, 0, 2), yym = o.s(1, 0, 0, -1);
    const float zz0 = o.s(2, 0, 0, 0), zzp = o.s(2, 1, 0, 0), zzp2 = o.s(2, 2, 0, 0), zzm = o.s(2, -1, 0, 0);
    const float xy0 = o.s(5, 0, 0, 0);
    const float xyjm = o.s(5, 0, 0, -1), xyjp = o.s(5, 0, 0, 1), xyjm2 = o.s(5, 0, 0, -2);
    const float xyim = o.s(5, 0, -1, 0), xyip = o.s(5, 0, 1, 0), xyim2 = o.s(5, 0, -2, 0);
    const float xz0 = o.s(4, 0, 0, 0);
    const float xzkm = o.s(4, -1, 0, 0), xzkp = o.s(4, 1, 0, 0), xzkm2 = o.s(4, -2, 0, 0);
    const float xzim = o.s(4, 0, -1, 0), xzip = o.s(4, 0, 1, 0), xzim2 = o.s(4, 0, -2, 0);
    const float yz0 = o.s(3, 0, 0, 0);
    const float yzkm = o.s(3, -1, 0, 0), yzkp = o.s(3, 1, 0, 0), yzkm2 = o.s(3, -2, 0, 0);
    const float yzjm = o.s(3, 0, 0, -1), yzjp = o.s(3, 0, 0, 1), yzjm2 = o.s(3, 0, 0, -2);
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
    if (a.divo) {
        const long long col = e / a.g.Kp;
        const int kd = (int)(e - col * a.g.Kp), ic = (int)(col % a.g.Ip), jc = (int)(col / a.g.Ip);
        const long long es = ((long long)(jc - 2 - a.dj0) * a.dIp + (ic - 2 - a.di0)) * a.dKp + kd;
        __stcs(a.divo + es, d3Sx3);
        __stcs(a.divo + a.dn + es, d3Sy3);
        __stcs(a.divo + 2 * a.dn + es, d3Sz3);
    }
}

template <int NM, int PREC>
struct GStrOps {
    const Str3Args &a;
    long long e, PI, PJ, so;
    const float *V[3];
    const float *S[6];
    __device__ __forceinline__ float v(int c, int dk, int di, int dj) const {
        return __ldg(&V[c][e + dk + di * PI + dj * PJ]);
    }
    __device__ __forceinline__ float sown(int f) const { return ldS<PREC>(S[f], e, sc_sS_in(a.scale, f)); }
    __device__ __forceinline__ float r(int q) const { return ldR<PREC>(a.R[q] + so, e, sc_sR_in(a.scale)); }
    // 0 mu, 1 lam, 2 taup, 3 taus, 4 muyz, 5 muxz, 6 muxy
    __device__ __forceinline__ float med(int m) const {
        const float *p = m == 0 ? a.mu : m == 1 ? a.lam : m == 2 ? a.taup : m == 3 ? a.taus
                       : m == 4 ? a.muyz : m == 5 ? a.muxz : a.muxy;
        return lds(&p[e]);
    }
};

// kernel__update_stress (m_kernel.f90:176-321) for one interior cell: every
// operand first (see vel_cell), then the normal and shear components and the
// memory variables, stored at e of the given arrays
template <int NM, int PREC, class Ops>
__device__ __forceinline__ void stress_interior(const Str3Args &a, const Ops &o, int s, float *const (&S)[6],
                                                long long e, long long so) {
    const float dt = a.dt;
    float r[6][NM > 0 ? NM : 1];
#pragma unroll
    for (int c = 0; c < 6; c++)
#pragma unroll
        for (int m = 0; m < NM; m++) r[c][m] = o.r(c * 3 + m);
    const float sxx = o.sown(0), syy = o.sown(1), szz = o.sown(2);
    const float syz = o.sown(3), sxz = o.sown(4), sxy = o.sown(5);
    const float mu = o.med(0), lam = o.med(1);
    const float taup1 = o.med(2), taus1 = o.med(3);
    const float muyz = o.med(4), muxz = o.med(5), muxy = o.med(6);
    const float vx0 = o.v(0, 0, 0, 0), vy0 = o.v(1, 0, 0, 0), vz0 = o.v(2, 0, 0, 0);
    const float vxim = o.v(0, 0, -1, 0), vxip = o.v(0, 0, 1, 0), vxim2 = o.v(0, 0, -2, 0);
    const float vxjp = o.v(0, 0, 0, 1), vxjp2 = o.v(0, 0, 0, 2), vxjm = o.v(0, 0, 0, -1);
    const float vxkp = o.v(0, 1, 0, 0), vxkp2 = o.v(0, 2, 0, 0), vxkm = o.v(0, -1, 0, 0);
    const float vyjm = o.v(1, 0, 0, -1), vyjp = o.v(1, 0, 0, 1), vyjm2 = o.v(1, 0, 0, -2);
    const float vyip = o.v(1, 0, 1, 0), vyip2 = o.v(1, 0, 2, 0), vyim = o.v(1, 0, -1, 0);
    const float vykp = o.v(1, 1, 0, 0), vykp2 = o.v(1, 2, 0, 0), vykm = o.v(1, -1, 0, 0);
    const float vzkm = o.v(2, -1, 0, 0), vzkp = o.v(2, 1, 0, 0), vzkm2 = o.v(2, -2, 0, 0);
    const float vzip = o.v(2, 0, 1, 0), vzip2 = o.v(2, 0, 2, 0), vzim = o.v(2, 0, -1, 0);
    const float vzjp = o.v(2, 0, 0, 1), vzjp2 = o.v(2, 0, 0, 2), vzjm = o.v(2, 0, 0, -1);
    const float re40x = a.e40[0][s], re41x = a.e41[0][s];
    const float re40y = a.e40[1][s], re41y = a.e41[1][s];
    const float re40z = a.e40[2][s], re41z = a.e41[2][s];

    // normal components (m_kernel.f90:195-235)
    const float dxVx = (vx0 - vxim) * re40x - (vxip - vxim2) * re41x;
    const float dyVy = (vy0 - vyjm) * re40y - (vyjp - vyjm2) * re41y;
    const float dzVz = (vz0 - vzkm) * re40z - (vzkp - vzkm2) * re41z;
    const float mu2 = 2 * mu;
    const float lam2mu = lam + mu2;
    const float d3v3 = dxVx + dyVy + dzVz;
    const float dyVy_dzVz = dyVy + dzVz;
    const float dxVx_dzVz = dxVx + dzVz;
    const float dxVx_dyVy = dxVx + dyVy;
    float Rxx_n = 0.0f, Ryy_n = 0.0f, Rzz_n = 0.0f;
#pragma unroll
    for (int m = 0; m < NM; m++) {
        r[0][m] = a.c1[m] * r[0][m] - a.c2[m] * (lam2mu * taup1 * d3v3 - mu2 * taus1 * dyVy_dzVz) * dt;
        r[1][m] = a.c1[m] * r[1][m] - a.c2[m] * (lam2mu * taup1 * d3v3 - mu2 * taus1 * dxVx_dzVz) * dt;
        r[2][m] = a.c1[m] * r[2][m] - a.c2[m] * (lam2mu * taup1 * d3v3 - mu2 * taus1 * dxVx_dyVy) * dt;
        Rxx_n = Rxx_n + a.d1[m] * r[0][m];
        Ryy_n = Ryy_n + a.d1[m] * r[1][m];
        Rzz_n = Rzz_n + a.d1[m] * r[2][m];
    }
    const float taup_plus1 = 1 + taup1 * (1 + a.d2);
    const float taus_plus1 = 1 + taus1 * (1 + a.d2);
    stS<PREC>(S[0], e, sxx + (lam2mu * taup_plus1 * d3v3 - mu2 * taus_plus1 * dyVy_dzVz + Rxx_n) * dt, sc_iS(a.scale, 0));
    stS<PREC>(S[1], e, syy + (lam2mu * taup_plus1 * d3v3 - mu2 * taus_plus1 * dxVx_dzVz + Ryy_n) * dt, sc_iS(a.scale, 1));
    stS<PREC>(S[2], e, szz + (lam2mu * taup_plus1 * d3v3 - mu2 * taus_plus1 * dxVx_dyVy + Rzz_n) * dt, sc_iS(a.scale, 2));

    // shear components (m_kernel.f90:282-311)
    const float dxVy_dyVx = (vyip - vy0) * re40x - (vyip2 - vyim) * re41x
                          + (vxjp - vx0) * re40y - (vxjp2 - vxjm) * re41y;
    const float dxVz_dzVx = (vzip - vz0) * re40x - (vzip2 - vzim) * re41x
                          + (vxkp - vx0) * re40z - (vxkp2 - vxkm) * re41z;
    const float dyVz_dzVy = (vzjp - vz0) * re40y - (vzjp2 - vzjm) * re41y
                          + (vykp - vy0) * re40z - (vykp2 - vykm) * re41z;
    float Ryz_n = 0.0f, Rxz_n = 0.0f, Rxy_n = 0.0f;
#pragma unroll
    for (int m = 0; m < NM; m++) {
        r[3][m] = a.c1[m] * r[3][m] - a.c2[m] * muyz * taus1 * dyVz_dzVy * dt;
        r[4][m] = a.c1[m] * r[4][m] - a.c2[m] * muxz * taus1 * dxVz_dzVx * dt;
        r[5][m] = a.c1[m] * r[5][m] - a.c2[m] * muxy * taus1 * dxVy_dyVx * dt;
        Ryz_n = Ryz_n + a.d1[m] * r[3][m];
        Rxz_n = Rxz_n + a.d1[m] * r[4][m];
        Rxy_n = Rxy_n + a.d1[m] * r[5][m];
    }
    stS<PREC>(S[3], e, syz + (muyz * taus_plus1 * dyVz_dzVy + Ryz_n) * dt, sc_iS(a.scale, 3));
    stS<PREC>(S[4], e, sxz + (muxz * taus_plus1 * dxVz_dzVx + Rxz_n) * dt, sc_iS(a.scale, 4));
    stS<PREC>(S[5], e, sxy + (muxy * taus_plus1 * dxVy_dyVx + Rxy_n) * dt, sc_iS(a.scale, 5));
#pragma unroll
    for (int c = 0; c < 6; c++)
#pragma unroll
        for (int m = 0; m < NM; m++) stR<PREC>(a.R[c * 3 + m] + so, e, r[c][m], sc_iR(a.scale, c * 3 + m));
}

// absorb_p__update_vel (m_absorb_p.f90:248-309) for one absorber cell: the
// auxiliaries (compact, per absorber column) from global memory, the other
// operands through the accessor
// The nine auxiliaries of an absorber cell (compact, per absorber column:
// m_absorb_p.f90:96-116), loaded ahead of the rest of the cell's operands.
struct Aux9 {
    long long q;   // index of the cell in the compact arrays (without the member offset)
    float v[9];
};
__device__ __forceinline__ Aux9 aux_load(float *const *aux, long long ao, const int2 *pmlcol, const Geo &g, int k,
                                         int i, int j) {
    Aux9 r;
    const int2 pc = __ldg(&pmlcol[col_index(g, i, j)]);
    r.q = (long long)pc.y + (k - pc.x);
#pragma unroll
    for (int n = 0; n < 9; n++) r.v[n] = lds(&aux[n][ao + r.q]);
    return r;
}

template <int PREC, class Ops>
__device__ __forceinline__ void vel_absorber(const Vel3Args &a, const Ops &o, const Aux9 &x, int k, int i, int j,
                                             long long e, long long ao, float *Vx, float *Vy, float *Vz) {
    const float dt = a.dt;
    const long long q = x.q;
    float *__restrict__ axSxx = a.aS[0] + ao;
    float *__restrict__ aySxy = a.aS[1] + ao;
    float *__restrict__ azSxz = a.aS[2] + ao;
    float *__restrict__ axSxy = a.aS[3] + ao;
    float *__restrict__ aySyy = a.aS[4] + ao;
    float *__restrict__ azSyz = a.aS[5] + ao;
    float *__restrict__ axSxz = a.aS[6] + ao;
    float *__restrict__ aySyz = a.aS[7] + ao;
    float *__restrict__ azSzz = a.aS[8] + ao;
    const float vxSxx = x.v[0], vySxy = x.v[1], vzSxz = x.v[2];
    const float vxSxy = x.v[3], vySyy = x.v[4], vzSyz = x.v[5];
    const float vxSxz = x.v[6], vySyz = x.v[7], vzSzz = x.v[8];
    const float vx = o.v(0), vy = o.v(1), vz = o.v(2);
    const float bx = o.b(0), by = o.b(1), bz = o.b(2);
    const float xx0 = o.s(0, 0, 0, 0), xxp = o.s(0, 0, 1, 0);
    const float yy0 = o.s(1, 0, 0, 0), yyp = o.s(1, 0, 0, 1);
    const float zz0 = o.s(2, 0, 0, 0), zzp = o.s(2, 1, 0, 0);
    const float yz0 = o.s(3, 0, 0, 0), yzjm = o.s(3, 0, 0, -1), yzkm = o.s(3, -1, 0, 0);
    const float xz0 = o.s(4, 0, 0, 0), xzim = o.s(4, 0, -1, 0), xzkm = o.s(4, -1, 0, 0);
    const float xy0 = o.s(5, 0, 0, 0), xyim = o.s(5, 0, -1, 0), xyjm = o.s(5, 0, 0, -1);
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

// absorb_p__update_stress (m_absorb_p.f90:445-491) for one absorber cell: the
// auxiliaries from global memory, the other operands through the accessor
template <int PREC, class Ops>
__device__ __forceinline__ void stress_absorber(const Str3Args &a, const Ops &o, const Aux9 &x, int k, int i, int j,
                                                long long e, long long ao, float *const (&S)[6]) {
    const float dt = a.dt;
    const long long q = x.q;
    float *__restrict__ axVx = a.aV[0] + ao;
    float *__restrict__ ayVx = a.aV[1] + ao;
    float *__restrict__ azVx = a.aV[2] + ao;
    float *__restrict__ axVy = a.aV[3] + ao;
    float *__restrict__ ayVy = a.aV[4] + ao;
    float *__restrict__ azVy = a.aV[5] + ao;
    float *__restrict__ axVz = a.aV[6] + ao;
    float *__restrict__ ayVz = a.aV[7] + ao;
    float *__restrict__ azVz = a.aV[8] + ao;
    // aux order of a.aV: axVx ayVx azVx axVy ayVy azVy axVz ayVz azVz
    const float vaxVx = x.v[0], vayVy = x.v[4], vazVz = x.v[8];
    const float vayVx = x.v[1], vazVx = x.v[2], vaxVy = x.v[3];
    const float vazVy = x.v[5], vaxVz = x.v[6], vayVz = x.v[7];
    const float sxx = o.sown(0), syy = o.sown(1), szz = o.sown(2);
    const float syz = o.sown(3), sxz = o.sown(4), sxy = o.sown(5);
    const float mu = o.med(0), lam = o.med(1);
    const float muyz = o.med(4), muxz = o.med(5), muxy = o.med(6);
    const float vx0 = o.v(0, 0, 0, 0), vy0 = o.v(1, 0, 0, 0), vz0 = o.v(2, 0, 0, 0);
    const float vxim = o.v(0, 0, -1, 0), vyjm = o.v(1, 0, 0, -1), vzkm = o.v(2, -1, 0, 0);
    const float vyip = o.v(1, 0, 1, 0), vzip = o.v(2, 0, 1, 0);
    const float vxjp = o.v(0, 0, 0, 1), vzjp = o.v(2, 0, 0, 1);
    const float vxkp = o.v(0, 1, 0, 0), vykp = o.v(1, 1, 0, 0);
    const float4 gxc = __ldg(&a.gxc[i - 1]), gxe = __ldg(&a.gxe[i - 1]);
    const float4 gyc = __ldg(&a.gyc[j - 1]), gye = __ldg(&a.gye[j - 1]);
    const float4 gzc = __ldg(&a.gzc[k - 1]), gze = __ldg(&a.gze[k - 1]);
    const float r20x = a.r20[0], r20y = a.r20[1], r20z = a.r20[2];

    const float dxVx = (vx0 - vxim) * r20x;
    const float dyVy = (vy0 - vyjm) * r20y;
    const float dzVz = (vz0 - vzkm) * r20z;
    const float lam2mu_R = (lam + 2 * mu);
    const float lam_R = lam2mu_R - 2 * mu;
    const float dxVx_ade = gxc.x * dxVx + gxc.y * vaxVx;
    const float dyVy_ade = gyc.x * dyVy + gyc.y * vayVy;
    const float dzVz_ade = gzc.x * dzVz + gzc.y * vazVz;
    stS<PREC>(S[0], e, sxx + (lam2mu_R * dxVx_ade + lam_R * (dyVy_ade + dzVz_ade)) * dt, sc_iS(a.scale, 0));
    stS<PREC>(S[1], e, syy + (lam2mu_R * dyVy_ade + lam_R * (dxVx_ade + dzVz_ade)) * dt, sc_iS(a.scale, 1));
    stS<PREC>(S[2], e, szz + (lam2mu_R * dzVz_ade + lam_R * (dxVx_ade + dyVy_ade)) * dt, sc_iS(a.scale, 2));
    sts(&axVx[q], gxc.z * vaxVx + gxc.w * dxVx * dt);
    sts(&ayVy[q], gyc.z * vayVy + gyc.w * dyVy * dt);
    sts(&azVz[q], gzc.z * vazVz + gzc.w * dzVz * dt);

    const float dxVy = (vyip - vy0) * r20x;
    const float dxVz = (vzip - vz0) * r20x;
    const float dyVx = (vxjp - vx0) * r20y;
    const float dyVz = (vzjp - vz0) * r20y;
    const float dzVx = (vxkp - vx0) * r20z;
    const float dzVy = (vykp - vy0) * r20z;
    stS<PREC>(S[3], e, syz + muyz * (gye.x * dyVz + gze.x * dzVy + gye.y * vayVz + gze.y * vazVy) * dt, sc_iS(a.scale, 3));
    stS<PREC>(S[4], e, sxz + muxz * (gxe.x * dxVz + gze.x * dzVx + gxe.y * vaxVz + gze.y * vazVx) * dt, sc_iS(a.scale, 4));
    stS<PREC>(S[5], e, sxy + muxy * (gxe.x * dxVy + gye.x * dyVx + gxe.y * vaxVy + gye.y * vayVx) * dt, sc_iS(a.scale, 5));
    sts(&ayVx[q], gye.z * vayVx + gye.w * dyVx * dt);
    sts(&azVx[q], gze.z * vazVx + gze.w * dzVx * dt);
    sts(&axVy[q], gxe.z * vaxVy + gxe.w * dxVy * dt);
    sts(&azVy[q], gze.z * vazVy + gze.w * dzVy * dt);
    sts(&axVz[q], gxe.z * vaxVz + gxe.w * dxVz * dt);
    sts(&ayVz[q], gye.z * vayVz + gye.w * dyVz * dt);
}

// ---------------------------------------------------------------------------
// velocity: kernel__update_vel (m_kernel.f90:75-140) +
//           absorb_p__update_vel (m_absorb_p.f90:248-309)
// ---------------------------------------------------------------------------
// One cell (k, i, j) of the fused velocity update.  All loads of the cell are
// issued before its first store: the arrays never alias, and with every
// operand in flight at once the update is limited by HBM bandwidth instead of
// by load latency.
// so / ao: offset of the state arrays (V, S) / PML auxiliaries, for a member
// of a batch that keeps its wavefields one after another (0 for a single run)
template <int PREC>
__device__ __forceinline__ void vel_cell(const Vel3Args &a, int k, int i, int j, long long so = 0, long long ao = 0) {
    const Geo g = a.g;
    const long long col = col_index(g, i, j);
    const long long e = col * g.Kp + (k - 1 + KH);
    const long long PI = g.Kp;
    const long long PJ = (long long)g.Kp * g.Ip;
    const float *__restrict__ Sxx = a.Sxx + so;
    const float *__restrict__ Syy = a.Syy + so;
    const float *__restrict__ Szz = a.Szz + so;
    const float *__restrict__ Syz = a.Syz + so;
    const float *__restrict__ Sxz = a.Sxz + so;
    const float *__restrict__ Sxy = a.Sxy + so;
    float *__restrict__ Vx = a.Vx + so;
    float *__restrict__ Vy = a.Vy + so;
    float *__restrict__ Vz = a.Vz + so;
    const float dt = a.dt;

    if (i >= a.ibk && i <= a.iek && j >= a.jbk && j <= a.jek && k <= a.kek) {
        if (!(a.mask & 1)) return;
        const GVelOps<PREC> o{a, e, PI, PJ, {Sxx, Syy, Szz, Syz, Sxz, Sxy}, {Vx, Vy, Vz}};
        vel_interior<PREC>(a, o, band_sign_of(a.band, col, k), Vx, Vy, Vz, e);
        return;
    }

    // absorber cell: k >= kbeg_a(i, j) holds for every cell outside the kernel box
    if (!(a.mask & 2)) return;
    const Aux9 x = aux_load(a.aS, ao, a.pmlcol, g, k, i, j);
    const GVelOps<PREC> o{a, e, PI, PJ, {Sxx, Syy, Szz, Syz, Sxz, Sxy}, {Vx, Vy, Vz}};
    vel_absorber<PREC>(a, o, x, k, i, j, e, ao, Vx, Vy, Vz);
}

// ---------------------------------------------------------------------------
// stress: kernel__update_stress (m_kernel.f90:142-326) +
//         absorb_p__update_stress (m_absorb_p.f90:424-503)
// ---------------------------------------------------------------------------
// One cell (k, i, j) of the fused stress and memory-variable update; like
// vel_cell, every load of the cell is issued before its first store.
template <int NM, int PREC>
__device__ __forceinline__ void stress_cell(const Str3Args &a, int k, int i, int j, long long so = 0,
                                            long long ao = 0) {
    const Geo g = a.g;
    const long long col = col_index(g, i, j);
    const long long e = col * g.Kp + (k - 1 + KH);
    const long long PI = g.Kp;
    const long long PJ = (long long)g.Kp * g.Ip;
    const float *__restrict__ Vx = a.Vx + so;
    const float *__restrict__ Vy = a.Vy + so;
    const float *__restrict__ Vz = a.Vz + so;
    float *__restrict__ Sxx = a.Sxx + so;
    float *__restrict__ Syy = a.Syy + so;
    float *__restrict__ Szz = a.Szz + so;
    float *__restrict__ Syz = a.Syz + so;
    float *__restrict__ Sxz = a.Sxz + so;
    float *__restrict__ Sxy = a.Sxy + so;
    const float dt = a.dt;

    if (i >= a.ibk && i <= a.iek && j >= a.jbk && j <= a.jek && k <= a.kek) {
        if (!(a.mask & 1)) return;
        const GStrOps<NM, PREC> o{a, e, PI, PJ, so, {Vx, Vy, Vz}, {Sxx, Syy, Szz, Syz, Sxz, Sxy}};
        float *const Sp[6] = {Sxx, Syy, Szz, Syz, Sxz, Sxy};
        stress_interior<NM, PREC>(a, o, band_sign_of(a.band, col, k), Sp, e, so);
        return;
    }

    // absorber cell (m_absorb_p.f90:445-491)
    if (!(a.mask & 2)) return;
    const Aux9 x = aux_load(a.aV, ao, a.pmlcol, g, k, i, j);
    const GStrOps<NM, PREC> o{a, e, PI, PJ, so, {Vx, Vy, Vz}, {Sxx, Syy, Szz, Syz, Sxz, Sxy}};
    float *const Sp[6] = {Sxx, Syy, Szz, Syz, Sxz, Sxy};
    stress_absorber<PREC>(a, o, x, k, i, j, e, ao, Sp);
}

// ---------------------------------------------------------------------------
// wav__store (m_wav.f90:433-620) for station n
// ---------------------------------------------------------------------------
__device__ __forceinline__ void wav_station(const Wav3Args &a, int n) {
    const int it = a.d_it ? *a.d_it : a.it;
    const Geo g = a.g;
    const int i = a.st[3 * n], j = a.st[3 * n + 1], k = a.st[3 * n + 2];
    const long long e = cell_index(g, k, i, j);
    const long long PI = g.Kp, PJ = (long long)g.Kp * g.Ip;
    const float *Vx = a.Vx, *Vy = a.Vy, *Vz = a.Vz;
    const float dt = a.dt;
    if (a.what & SWPC_WAV_U) {
        a.uacc[3 * n + 0] = a.uacc[3 * n + 0] + (Vx[e] + Vx[e - PI]) * 0.5f * dt;
        a.uacc[3 * n + 1] = a.uacc[3 * n + 1] + (Vy[e] + Vy[e - PJ]) * 0.5f * dt;
        a.uacc[3 * n + 2] = a.uacc[3 * n + 2] - (Vz[e] + Vz[e - 1]) * 0.5f * dt;
    }
    if (a.what & SWPC_WAV_STRAIN) {
        const float r40x = a.r40[0], r40y = a.r40[1], r40z = a.r40[2];
        const float r41x = a.r41[0], r41y = a.r41[1], r41z = a.r41[2];
        // m_wav.f90:468-500
        const float dxVx = (Vx[e] - Vx[e - PI]) * r40x - (Vx[e + PI] - Vx[e - 2 * PI]) * r41x;
        const float dyVy = (Vy[e] - Vy[e - PJ]) * r40y - (Vy[e + PJ] - Vy[e - 2 * PJ]) * r41y;
        const float dzVz = (Vz[e] - Vz[e - 1]) * r40z - (Vz[e + 1] - Vz[e - 2]) * r41z;
        const long long m = e - PJ;   // (k, i, j-1)
        const float dxVy = ((Vy[e + PI] - Vy[e]) * r40x - (Vy[e + 2 * PI] - Vy[e - PI]) * r41x
                          + (Vy[m + PI] - Vy[m]) * r40x - (Vy[m + 2 * PI] - Vy[m - PI]) * r41x
                          + (Vy[e] - Vy[e - PI]) * r40x - (Vy[e + PI] - Vy[e - 2 * PI]) * r41x
                          + (Vy[m] - Vy[m - PI]) * r40x - (Vy[m + PI] - Vy[m - 2 * PI]) * r41x) / 4.0f;
        const long long u = e - 1;    // (k-1, i, j)
        const float dxVz = ((Vz[e + PI] - Vz[e]) * r40x - (Vz[e + 2 * PI] - Vz[e - PI]) * r41x
                          + (Vz[u + PI] - Vz[u]) * r40x - (Vz[u + 2 * PI] - Vz[u - PI]) * r41x
                          + (Vz[e] - Vz[e - PI]) * r40x - (Vz[e + PI] - Vz[e - 2 * PI]) * r41x
                          + (Vz[u] - Vz[u - PI]) * r40x - (Vz[u + PI] - Vz[u - 2 * PI]) * r41x) / 4.0f;
        const long long w = e - PI;   // (k, i-1, j)
        const float dyVx = ((Vx[e + PJ] - Vx[e]) * r40y - (Vx[e + 2 * PJ] - Vx[e - PJ]) * r41y
                          + (Vx[w + PJ] - Vx[w]) * r40y - (Vx[w + 2 * PJ] - Vx[w - PJ]) * r41y
                          + (Vx[e] - Vx[e - PJ]) * r40y - (Vx[e + PJ] - Vx[e - 2 * PJ]) * r41y
                          + (Vx[w] - Vx[w - PJ]) * r40y - (Vx[w + PJ] - Vx[w - 2 * PJ]) * r41y) / 4.0f;
        const float dyVz = ((Vz[e + PJ] - Vz[e]) * r40y - (Vz[e + 2 * PJ] - Vz[e - PJ]) * r41y
                          + (Vz[u + PJ] - Vz[u]) * r40y - (Vz[u + 2 * PJ] - Vz[u - PJ]) * r41y
                          + (Vz[e] - Vz[e - PJ]) * r40y - (Vz[e + PJ] - Vz[e - 2 * PJ]) * r41y
                          + (Vz[u] - Vz[u - PJ]) * r40y - (Vz[u + PJ] - Vz[u - 2 * PJ]) * r41y) / 4.0f;
        const float dzVx = ((Vx[e + 1] - Vx[e]) * r40z - (Vx[e + 2] - Vx[e - 1]) * r41z
                          + (Vx[w + 1] - Vx[w]) * r40z - (Vx[w + 2] - Vx[w - 1]) * r41z
                          + (Vx[e] - Vx[e - 1]) * r40z - (Vx[e + 1] - Vx[e - 2]) * r41z
                          + (Vx[w] - Vx[w - 1]) * r40z - (Vx[w + 1] - Vx[w - 2]) * r41z) / 4.0f;
        const float dzVy = ((Vy[e + 1] - Vy[e]) * r40z - (Vy[e + 2] - Vy[e - 1]) * r41z
                          + (Vy[m + 1] - Vy[m]) * r40z - (Vy[m + 2] - Vy[m - 1]) * r41z
                          + (Vy[e] - Vy[e - 1]) * r40z - (Vy[e + 1] - Vy[e - 2]) * r41z
                          + (Vy[m] - Vy[m - 1]) * r40z - (Vy[m + 1] - Vy[m - 2]) * r41z) / 4.0f;
        float *ea = a.eacc + 6 * n;
        ea[0] = ea[0] + dxVx * dt;
        ea[1] = ea[1] + dyVy * dt;
        ea[2] = ea[2] + dzVz * dt;
        ea[3] = ea[3] + (dyVz + dzVy) / 2.0f * dt;
        ea[4] = ea[4] + (dxVz + dzVx) / 2.0f * dt;
        ea[5] = ea[5] + (dxVy + dyVx) / 2.0f * dt;
    }
    if ((it - 1) % a.ntdec_w != 0) return;
    const int itw = (it - 1) / a.ntdec_w + 1;
    if (itw > a.ntw) return;
    const float M0 = a.M0, UC = a.UC;
    const long long ntw = a.ntw;
    if (a.what & SWPC_WAV_V) {
        float *w = a.wav_v + (long long)n * 3 * ntw + (itw - 1);
        w[0 * ntw] = (Vx[e] + Vx[e - PI]) / 2.0f * M0 * UC * 1e9f;
        w[1 * ntw] = (Vy[e] + Vy[e - PJ]) / 2.0f * M0 * UC * 1e9f;
        w[2 * ntw] = -(Vz[e] + Vz[e - 1]) / 2.0f * M0 * UC * 1e9f;
    }
    if (a.what & SWPC_WAV_U) {
        float *w = a.wav_u + (long long)n * 3 * ntw + (itw - 1);
        w[0 * ntw] = a.uacc[3 * n + 0] * M0 * UC * 1e9f;
        w[1 * ntw] = a.uacc[3 * n + 1] * M0 * UC * 1e9f;
        w[2 * ntw] = a.uacc[3 * n + 2] * M0 * UC * 1e9f;
    }
    if (a.what & SWPC_WAV_STRESS) {
        float *w = a.wav_s + (long long)n * 6 * ntw + (itw - 1);
        if (a.s_half) {
            // FP16 stress arrays: the same expressions on the scaled values
            auto S = [&](const float *p, int c, long long q) {
                return __half2float(reinterpret_cast<const __half *>(p)[q]) * sc_sS(a.scale, c);
            };
            w[0 * ntw] = S(a.Sxx, 0, e) * M0 * UC * 1e6f;
            w[1 * ntw] = S(a.Syy, 1, e) * M0 * UC * 1e6f;
            w[2 * ntw] = S(a.Szz, 2, e) * M0 * UC * 1e6f;
            w[3 * ntw] = (S(a.Syz, 3, e) + S(a.Syz, 3, e - PJ) + S(a.Syz, 3, e - 1) + S(a.Syz, 3, e - 1 - PJ)) / 4.0f
                         * M0 * UC * 1e6f;
            w[4 * ntw] = (S(a.Sxz, 4, e) + S(a.Sxz, 4, e - PI) + S(a.Sxz, 4, e - 1) + S(a.Sxz, 4, e - 1 - PI)) / 4.0f
                         * M0 * UC * 1e6f;
            w[5 * ntw] = (S(a.Sxy, 5, e) + S(a.Sxy, 5, e - PJ) + S(a.Sxy, 5, e - PI) + S(a.Sxy, 5, e - PI - PJ)) / 4.0f
                         * M0 * UC * 1e6f;
        } else {
        const float *Sxx = a.Sxx, *Syy = a.Syy, *Szz = a.Szz, *Syz = a.Syz, *Sxz = a.Sxz, *Sxy = a.Sxy;
        w[0 * ntw] = Sxx[e] * M0 * UC * 1e6f;
        w[1 * ntw] = Syy[e] * M0 * UC * 1e6f;
        w[2 * ntw] = Szz[e] * M0 * UC * 1e6f;
        w[3 * ntw] = (Syz[e] + Syz[e - PJ] + Syz[e - 1] + Syz[e - 1 - PJ]) / 4.0f * M0 * UC * 1e6f;
        w[4 * ntw] = (Sxz[e] + Sxz[e - PI] + Sxz[e - 1] + Sxz[e - 1 - PI]) / 4.0f * M0 * UC * 1e6f;
        w[5 * ntw] = (Sxy[e] + Sxy[e - PJ] + Sxy[e - PI] + Sxy[e - PI - PJ]) / 4.0f * M0 * UC * 1e6f;
        }
    }
    if (a.what & SWPC_WAV_STRAIN) {
        float *w = a.wav_e + (long long)n * 6 * ntw + (itw - 1);
        for (int c = 0; c < 6; c++) w[c * ntw] = a.eacc[6 * n + c] * M0 * UC * 1e-3f;
    }
}

}  // namespace swpc
