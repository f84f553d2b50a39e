// swpc2d_cell.cuh -- the per-cell arithmetic of the 2D P-SV and SH updates,
// shared by the tile-walking kernels (operands from global memory,
// swpc2d_kernels.cu) and the TMA-staged kernels (operands from shared
// memory, swpc2d_tma.cu).
//
// Per cell the functions restate
//   P-SV: src/swpc_psv/m_kernel.f90:76-306 (interior) and
//         src/swpc_psv/m_absorb_p.f90:180-230, 337-385 (ADE-CFS PML),
//   SH:   src/swpc_sh/m_kernel.f90:77-221 and src/swpc_sh/m_absorb_p.f90,
// in the reference's expression order.  An operand source `o` supplies the
// values: o.v(c, dk, di) velocity component c at (k+dk, i+di); o.s(c) the
// cell's own stress component; o.sn(c, dk, di) a stress neighbour; o.r(c, m)
// memory variable m of component c; o.lam() o.taup() o.taus() the cell's
// medium; o.mu(dk, di) and o.rho(dk, di) the rigidity and density that the
// averaged moduli and buoyancies read.  Stores go to global memory.  Both
// translation units are compiled with -fmad=false, so every operand source
// gives bitwise the same results (and those of the oracle).
//   P-SV: v 0 Vx, 1 Vz; s / sn 0 Sxx, 1 Szz, 2 Sxz; r c = xx zz xz
//   SH:   v 0 Vy;       s / sn 0 Syz, 1 Sxy;          r c = yz xy
#pragma once

#include <cuda_runtime.h>

#include "swpc2d.cuh"

namespace swpc {

constexpr float EPSL2D = 1.1920929e-07f;   // epsilon(1.0)

__device__ __forceinline__ float ld2s(const float *p) { return __ldcs(p); }
__device__ __forceinline__ void st2s(float *p, float v) { __stcs(p, v); }

// 4th-order band sign of cell (k, i): 1 inside the 2nd-order bands around the
// free surface and the ocean bottom
__device__ __forceinline__ int band_sign2d(const Model2D &M, int k, int i) {
    const int4 bd = __ldg(&M.band[i + 2]);
    const int p1 = (k - bd.x) * (bd.y - k), p2 = (k - bd.z) * (bd.w - k);
    return ((p1 > p2 ? p1 : p2) >= 0) ? 1 : 0;
}

// operands of a cell read from global memory
struct G2Ops {
    const Model2D &M;
    long long e, PI;
    __device__ __forceinline__ const float *vf(int c) const { return c ? M.V1 : M.V0; }
    __device__ __forceinline__ const float *sf(int c) const { return c == 0 ? M.S0 : c == 1 ? M.S1 : M.S2; }
    __device__ __forceinline__ float v(int c, int dk, int di) const { return __ldg(&vf(c)[e + dk + di * PI]); }
    __device__ __forceinline__ float vown(int c) const { return ld2s(&vf(c)[e]); }
    __device__ __forceinline__ float s(int c) const { return ld2s(&sf(c)[e]); }
    __device__ __forceinline__ float sn(int c, int dk, int di) const { return __ldg(&sf(c)[e + dk + di * PI]); }
    __device__ __forceinline__ float r(int c, int m) const { return ld2s(&M.R[c * 3 + m][e]); }
    __device__ __forceinline__ float lam() const { return ld2s(&M.lam[e]); }
    __device__ __forceinline__ float taup() const { return ld2s(&M.taup[e]); }
    __device__ __forceinline__ float taus() const { return ld2s(&M.taus[e]); }
    __device__ __forceinline__ float mu(int dk, int di) const {
        return (dk | di) ? __ldg(&M.mu[e + dk + di * PI]) : ld2s(&M.mu[e]);
    }
    __device__ __forceinline__ float rho(int dk, int di) const { return __ldg(&M.rho[e + dk + di * PI]); }
};

// ---------------------------------------------------------------------------
// P-SV
// ---------------------------------------------------------------------------
template <int NM, class O>
__device__ __forceinline__ void psv_stress_interior(const Model2D &M, const O &o, int s, long long e) {
    const float dt = M.dt;
    const float re40x = M.e40[0][s], re41x = M.e41[0][s], re40z = M.e40[1][s], re41z = M.e41[1][s];
    float r[3][NM > 0 ? NM : 1];
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int m = 0; m < NM; m++) r[c][m] = o.r(c, m);
    const float sxx = o.s(0), szz = o.s(1), sxz = o.s(2);
    const float mu = o.mu(0, 0), lam = o.lam(), taup1 = o.taup(), taus1 = o.taus();
    const float pnn = o.mu(1, 0), npn = o.mu(0, 1), ppn = o.mu(1, 1);
    const float vx0 = o.v(0, 0, 0), vz0 = o.v(1, 0, 0);
    const float dxVx = (vx0 - o.v(0, 0, -1)) * re40x - (o.v(0, 0, 1) - o.v(0, 0, -2)) * re41x;
    const float dzVz = (vz0 - o.v(1, -1, 0)) * re40z - (o.v(1, 1, 0) - o.v(1, -2, 0)) * re41z;
    const float dxVz = (o.v(1, 0, 1) - vz0) * re40x - (o.v(1, 0, 2) - o.v(1, 0, -1)) * re41x;
    const float dzVx = (o.v(0, 1, 0) - vx0) * re40z - (o.v(0, 2, 0) - o.v(0, -1, 0)) * re41z;
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
    st2s(&M.S0[e], sxx + (lam2mu * taup_plus1 * d2v2 - mu2 * taus_plus1 * dzVz + Rxx_n) * dt);
    st2s(&M.S1[e], szz + (lam2mu * taup_plus1 * d2v2 - mu2 * taus_plus1 * dxVx + Rzz_n) * dt);
    // shear component (src/swpc_psv/m_kernel.f90:270-300)
    const float nnn = mu;
    const float mu_xz =
        4 * nnn * pnn * npn * ppn / (nnn * pnn * npn + nnn * pnn * ppn + nnn * npn * ppn + pnn * npn * ppn + EPSL2D);
    const float dxVz_dzVx = dxVz + dzVx;
    const float f_Rxz = mu_xz * taus1 * dxVz_dzVx;
    float Rxz_n = 0.0f;
#pragma unroll
    for (int m = 0; m < NM; m++) {
        r[2][m] = M.c1[m] * r[2][m] - M.c2[m] * f_Rxz * dt;
        Rxz_n = Rxz_n + M.d1[m] * r[2][m];
    }
    st2s(&M.S2[e], sxz + (mu_xz * taus_plus1 * dxVz_dzVx + Rxz_n) * dt);
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int m = 0; m < NM; m++) st2s(&M.R[c * 3 + m][e], r[c][m]);
}

// absorber cell (src/swpc_psv/m_absorb_p.f90:337-385)
template <class O>
__device__ __forceinline__ void psv_stress_absorber(const Model2D &M, const O &o, int k, int i, long long e) {
    const float dt = M.dt;
    const int2 pc = __ldg(&M.pmlcol[i + 2]);
    const long long q = (long long)pc.y + (k - pc.x);
    float *__restrict__ axVx = M.aux[0];
    float *__restrict__ azVx = M.aux[1];
    float *__restrict__ axVz = M.aux[2];
    float *__restrict__ azVz = M.aux[3];
    const float vaxVx = ld2s(&axVx[q]), vazVx = ld2s(&azVx[q]), vaxVz = ld2s(&axVz[q]), vazVz = ld2s(&azVz[q]);
    const float sxx = o.s(0), szz = o.s(1), sxz = o.s(2);
    const float mu = o.mu(0, 0), lam = o.lam();
    const float pnn = o.mu(1, 0), npn = o.mu(0, 1), ppn = o.mu(1, 1);
    const float vx0 = o.v(0, 0, 0), vz0 = o.v(1, 0, 0);
    const float4 gxc = __ldg(&M.gxc[i - 1]), gxe = __ldg(&M.gxe[i - 1]);
    const float4 gzc = __ldg(&M.gzc[k - 1]), gze = __ldg(&M.gze[k - 1]);
    const float dxVx = (vx0 - o.v(0, 0, -1)) * M.r20[0];
    const float dzVz = (vz0 - o.v(1, -1, 0)) * M.r20[1];
    const float lam2mu_R = lam + 2 * mu;
    const float lam_R = lam2mu_R - 2 * mu;
    const float dxVx_ade = gxc.x * dxVx + gxc.y * vaxVx;
    const float dzVz_ade = gzc.x * dzVz + gzc.y * vazVz;
    st2s(&M.S0[e], sxx + (lam2mu_R * dxVx_ade + lam_R * dzVz_ade) * dt);
    st2s(&M.S1[e], szz + (lam2mu_R * dzVz_ade + lam_R * dxVx_ade) * dt);
    st2s(&axVx[q], gxc.z * vaxVx + gxc.w * dxVx * dt);
    st2s(&azVz[q], gzc.z * vazVz + gzc.w * dzVz * dt);
    const float dzVx = (o.v(0, 1, 0) - vx0) * M.r20[1];
    const float dxVz = (o.v(1, 0, 1) - vz0) * M.r20[0];
    const float nnn = mu;
    const float muxz =
        4 * nnn * pnn * npn * ppn / (nnn * pnn * npn + nnn * pnn * ppn + nnn * npn * ppn + pnn * npn * ppn + EPSL2D);
    st2s(&M.S2[e], sxz + muxz * (gxe.x * dxVz + gze.x * dzVx + gxe.y * vaxVz + gze.y * vazVx) * dt);
    st2s(&azVx[q], gze.z * vazVx + gze.w * dzVx * dt);
    st2s(&axVz[q], gxe.z * vaxVz + gxe.w * dxVz * dt);
}

// velocity: interior (s >= 0: band sign) or absorber (s < 0) cell
template <class O>
__device__ __forceinline__ void psv_vel_cell(const Model2D &M, const O &o, int k, int i, long long e, int s) {
    const float dt = M.dt;
    const float vx = o.vown(0), vz = o.vown(1);
    const float rho0 = o.rho(0, 0), rhoi = o.rho(0, 1), rhok = o.rho(1, 0);
    const float bx = 2.0f / (rho0 + rhoi);
    const float bz = 2.0f / (rho0 + rhok);
    if (s >= 0) {
        const float re40x = M.e40[0][s], re41x = M.e41[0][s], re40z = M.e40[1][s], re41z = M.e41[1][s];
        const float dxSxx = (o.sn(0, 0, 1) - o.sn(0, 0, 0)) * re40x - (o.sn(0, 0, 2) - o.sn(0, 0, -1)) * re41x;
        const float dzSzz = (o.sn(1, 1, 0) - o.sn(1, 0, 0)) * re40z - (o.sn(1, 2, 0) - o.sn(1, -1, 0)) * re41z;
        const float dxSxz = (o.sn(2, 0, 0) - o.sn(2, 0, -1)) * re40x - (o.sn(2, 0, 1) - o.sn(2, 0, -2)) * re41x;
        const float dzSxz = (o.sn(2, 0, 0) - o.sn(2, -1, 0)) * re40z - (o.sn(2, 1, 0) - o.sn(2, -2, 0)) * re41z;
        st2s(&M.V0[e], vx + bx * (dxSxx + dzSxz) * dt);
        st2s(&M.V1[e], vz + bz * (dxSxz + dzSzz) * dt);
        return;
    }
    // absorber (src/swpc_psv/m_absorb_p.f90:180-230)
    const int2 pc = __ldg(&M.pmlcol[i + 2]);
    const long long q = (long long)pc.y + (k - pc.x);
    float *__restrict__ axSxx = M.aux[4];
    float *__restrict__ azSxz = M.aux[5];
    float *__restrict__ axSxz = M.aux[6];
    float *__restrict__ azSzz = M.aux[7];
    const float vxSxx = ld2s(&axSxx[q]), vzSxz = ld2s(&azSxz[q]), vxSxz = ld2s(&axSxz[q]), vzSzz = ld2s(&azSzz[q]);
    const float4 gxc = __ldg(&M.gxc[i - 1]), gxe = __ldg(&M.gxe[i - 1]);
    const float4 gzc = __ldg(&M.gzc[k - 1]), gze = __ldg(&M.gze[k - 1]);
    const float dxSxx = (o.sn(0, 0, 1) - o.sn(0, 0, 0)) * M.r20[0];
    const float dzSzz = (o.sn(1, 1, 0) - o.sn(1, 0, 0)) * M.r20[1];
    const float dxSxz = (o.sn(2, 0, 0) - o.sn(2, 0, -1)) * M.r20[0];
    const float dzSxz = (o.sn(2, 0, 0) - o.sn(2, -1, 0)) * M.r20[1];
    st2s(&M.V0[e], vx + bx * (gxe.x * dxSxx + gzc.x * dzSxz + gxe.y * vxSxx + gzc.y * vzSxz) * dt);
    st2s(&M.V1[e], vz + bz * (gxc.x * dxSxz + gze.x * dzSzz + gxc.y * vxSxz + gze.y * vzSzz) * dt);
    st2s(&axSxx[q], gxe.z * vxSxx + gxe.w * dxSxx * dt);
    st2s(&azSxz[q], gzc.z * vzSxz + gzc.w * dzSxz * dt);
    st2s(&axSxz[q], gxc.z * vxSxz + gxc.w * dxSxz * dt);
    st2s(&azSzz[q], gze.z * vzSzz + gze.w * dzSzz * dt);
}

// ---------------------------------------------------------------------------
// SH
// ---------------------------------------------------------------------------
// interior (s >= 0) or absorber (s < 0) stress cell
template <int NM, class O>
__device__ __forceinline__ void sh_stress_cell(const Model2D &M, const O &o, int k, int i, long long e, int s) {
    const float dt = M.dt;
    const float syz = o.s(0), sxy = o.s(1);
    const float nnn = o.mu(0, 0), pnn = o.mu(1, 0), npn = o.mu(0, 1);
    const float vy0 = o.v(0, 0, 0);
    const float mu_xy = 2 * nnn * npn / (nnn + npn + EPSL2D);
    const float mu_yz = 2 * nnn * pnn / (nnn + pnn + EPSL2D);
    if (s >= 0) {
        float r[2][NM > 0 ? NM : 1];
#pragma unroll
        for (int c = 0; c < 2; c++)
#pragma unroll
            for (int m = 0; m < NM; m++) r[c][m] = o.r(c, m);
        const float taus1 = o.taus();
        const float re40x = M.e40[0][s], re41x = M.e41[0][s], re40z = M.e40[1][s], re41z = M.e41[1][s];
        const float dxVy = (o.v(0, 0, 1) - vy0) * re40x - (o.v(0, 0, 2) - o.v(0, 0, -1)) * re41x;
        const float dzVy = (o.v(0, 1, 0) - vy0) * re40z - (o.v(0, 2, 0) - o.v(0, -1, 0)) * re41z;
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
        st2s(&M.S0[e], syz + (mu_yz * taus_plus1 * dzVy + Ryz_n) * dt);
        st2s(&M.S1[e], sxy + (mu_xy * taus_plus1 * dxVy + Rxy_n) * dt);
#pragma unroll
        for (int c = 0; c < 2; c++)
#pragma unroll
            for (int m = 0; m < NM; m++) st2s(&M.R[c * 3 + m][e], r[c][m]);
        return;
    }
    const int2 pc = __ldg(&M.pmlcol[i + 2]);
    const long long q = (long long)pc.y + (k - pc.x);
    float *__restrict__ axVy = M.aux[0];
    float *__restrict__ azVy = M.aux[1];
    const float4 gxe = __ldg(&M.gxe[i - 1]);
    const float4 gze = __ldg(&M.gze[k - 1]);
    const float dxVy = (o.v(0, 0, 1) - vy0) * M.r20[0];
    const float dzVy = (o.v(0, 1, 0) - vy0) * M.r20[1];
    // the auxiliaries are advanced first and then used (src/swpc_sh/m_absorb_p.f90)
    const float ax = gxe.z * ld2s(&axVy[q]) + gxe.w * dxVy * dt;
    const float az = gze.z * ld2s(&azVy[q]) + gze.w * dzVy * dt;
    st2s(&axVy[q], ax);
    st2s(&azVy[q], az);
    st2s(&M.S0[e], syz + mu_yz * (gze.x * dzVy + gze.y * az) * dt);
    st2s(&M.S1[e], sxy + mu_xy * (gxe.x * dxVy + gxe.y * ax) * dt);
}

template <class O>
__device__ __forceinline__ void sh_vel_cell(const Model2D &M, const O &o, int k, int i, long long e, int s) {
    const float dt = M.dt;
    const float vy = o.vown(0);
    const float by = 1.0f / o.rho(0, 0);
    if (s >= 0) {
        const float re40x = M.e40[0][s], re41x = M.e41[0][s], re40z = M.e40[1][s], re41z = M.e41[1][s];
        const float dzSyz = (o.sn(0, 0, 0) - o.sn(0, -1, 0)) * re40z - (o.sn(0, 1, 0) - o.sn(0, -2, 0)) * re41z;
        const float dxSxy = (o.sn(1, 0, 0) - o.sn(1, 0, -1)) * re40x - (o.sn(1, 0, 1) - o.sn(1, 0, -2)) * re41x;
        st2s(&M.V0[e], vy + by * (dxSxy + dzSyz) * dt);
        return;
    }
    const int2 pc = __ldg(&M.pmlcol[i + 2]);
    const long long q = (long long)pc.y + (k - pc.x);
    float *__restrict__ axSxy = M.aux[2];
    float *__restrict__ azSyz = M.aux[3];
    const float vxSxy = ld2s(&axSxy[q]), vzSyz = ld2s(&azSyz[q]);
    const float4 gxc = __ldg(&M.gxc[i - 1]);
    const float4 gzc = __ldg(&M.gzc[k - 1]);
    const float dzSyz = (o.sn(0, 0, 0) - o.sn(0, -1, 0)) * M.r20[1];
    const float dxSxy = (o.sn(1, 0, 0) - o.sn(1, 0, -1)) * M.r20[0];
    st2s(&M.V0[e], vy + by * (gxc.x * dxSxy + gzc.x * dzSyz + gxc.y * vxSxy + gzc.y * vzSyz) * dt);
    st2s(&axSxy[q], gxc.z * vxSxy + gxc.w * dxSxy * dt);
    st2s(&azSyz[q], gzc.z * vzSyz + gzc.w * dzSyz * dt);
}

}  // namespace swpc
