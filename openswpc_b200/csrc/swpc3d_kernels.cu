// swpc3d_kernels.cu -- fused sm_100a kernels of the 3D viscoelastic step.
//
// One launch per half step covers the whole domain: cells of the interior
// kernel region (m_global.f90:349-378) run the 4th-order viscoelastic update
// of src/swpc_3d/m_kernel.f90, the remaining cells (k >= kbeg_a(i,j),
// m_global.f90:336-345) run the 2nd-order ADE-CFS PML update of
// src/swpc_3d/m_absorb_p.f90.  The two regions are disjoint and neither pass
// reads what the other writes within a half step, so the fused launch gives
// exactly the result of the two reference routines run one after the other.
//
// Arithmetic: every expression keeps the reference's left-to-right order and
// this file is compiled with -fmad=false, so each product and sum is rounded
// separately exactly as the single-precision (MP = SP) Fortran build spells
// it out; the results are bitwise identical to the CPU oracle.
//
// Thread mapping: a warp owns 32 consecutive k of one (i, j) column (one
// coalesced 128-byte row per field); block = 32 x BI x BJ columns.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "swpc_ctx.h"
#include "swpc_kernels.cuh"
#include "swpc3d_cell.cuh"

namespace swpc {

// ---------------------------------------------------------------------------
// velocity: one thread per cell (vel_cell in swpc3d_cell.cuh)
// ---------------------------------------------------------------------------
template <int MINB, int PREC>
__global__ void __launch_bounds__(256, MINB) vel3d_kernel(const Vel3Args a) {
    const Geo g = a.g;
    const int k = 1 + blockIdx.x * 32 + threadIdx.x;
    const int i = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int j = 1 + blockIdx.z * blockDim.z + threadIdx.z;
    if (k > g.nz || i > g.nx || j > g.ny) return;
    vel_cell<PREC>(a, k, i, j);
}

// ---------------------------------------------------------------------------
// stress: kernel__update_stress (m_kernel.f90:142-326) +
//         absorb_p__update_stress (m_absorb_p.f90:424-503)
// ---------------------------------------------------------------------------
template <int NM, int MINB, int PREC>
__global__ void __launch_bounds__(256, MINB) stress3d_kernel(const Str3Args a) {
    const Geo g = a.g;
    const int k = 1 + blockIdx.x * 32 + threadIdx.x;
    const int i = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int j = 1 + blockIdx.z * blockDim.z + threadIdx.z;
    if (k > g.nz || i > g.nx || j > g.ny) return;
    const long long col = col_index(g, i, j);
    const long long e = col * g.Kp + (k - 1 + KH);
    const long long PI = g.Kp;
    const long long PJ = (long long)g.Kp * g.Ip;
    const float *__restrict__ Vx = a.Vx;
    const float *__restrict__ Vy = a.Vy;
    const float *__restrict__ Vz = a.Vz;
    float *__restrict__ Sxx = a.Sxx;
    float *__restrict__ Syy = a.Syy;
    float *__restrict__ Szz = a.Szz;
    float *__restrict__ Syz = a.Syz;
    float *__restrict__ Sxz = a.Sxz;
    float *__restrict__ Sxy = a.Sxy;
    const float dt = a.dt;

    if (i >= a.ibk && i <= a.iek && j >= a.jbk && j <= a.jek && k <= a.kek) {
        if (!(a.mask & 1)) return;
        // every operand of the cell first (see the velocity kernel)
        float r[6][NM > 0 ? NM : 1];
#pragma unroll
        for (int c = 0; c < 6; c++)
#pragma unroll
            for (int m = 0; m < NM; m++) r[c][m] = ldR<PREC>(a.R[c * 3 + m], e, a.sR[c * 3 + m]);
        const float sxx = ldS<PREC>(Sxx, e, a.sS[0]), syy = ldS<PREC>(Syy, e, a.sS[1]), szz = ldS<PREC>(Szz, e, a.sS[2]);
        const float syz = ldS<PREC>(Syz, e, a.sS[3]), sxz = ldS<PREC>(Sxz, e, a.sS[4]), sxy = ldS<PREC>(Sxy, e, a.sS[5]);
        const float mu = lds(&a.mu[e]), lam = lds(&a.lam[e]);
        const float taup1 = lds(&a.taup[e]), taus1 = lds(&a.taus[e]);
        const float muyz = lds(&a.muyz[e]), muxz = lds(&a.muxz[e]), muxy = lds(&a.muxy[e]);
        const float vx0 = __ldg(&Vx[e]), vy0 = __ldg(&Vy[e]), vz0 = __ldg(&Vz[e]);
        const float vxim = __ldg(&Vx[e - PI]), vxip = __ldg(&Vx[e + PI]), vxim2 = __ldg(&Vx[e - 2 * PI]);
        const float vxjp = __ldg(&Vx[e + PJ]), vxjp2 = __ldg(&Vx[e + 2 * PJ]), vxjm = __ldg(&Vx[e - PJ]);
        const float vxkp = __ldg(&Vx[e + 1]), vxkp2 = __ldg(&Vx[e + 2]), vxkm = __ldg(&Vx[e - 1]);
        const float vyjm = __ldg(&Vy[e - PJ]), vyjp = __ldg(&Vy[e + PJ]), vyjm2 = __ldg(&Vy[e - 2 * PJ]);
        const float vyip = __ldg(&Vy[e + PI]), vyip2 = __ldg(&Vy[e + 2 * PI]), vyim = __ldg(&Vy[e - PI]);
        const float vykp = __ldg(&Vy[e + 1]), vykp2 = __ldg(&Vy[e + 2]), vykm = __ldg(&Vy[e - 1]);
        const float vzkm = __ldg(&Vz[e - 1]), vzkp = __ldg(&Vz[e + 1]), vzkm2 = __ldg(&Vz[e - 2]);
        const float vzip = __ldg(&Vz[e + PI]), vzip2 = __ldg(&Vz[e + 2 * PI]), vzim = __ldg(&Vz[e - PI]);
        const float vzjp = __ldg(&Vz[e + PJ]), vzjp2 = __ldg(&Vz[e + 2 * PJ]), vzjm = __ldg(&Vz[e - PJ]);
        const int4 bd = __ldg(&a.band[col]);
        const int p1 = (k - bd.x) * (bd.y - k);
        const int p2 = (k - bd.z) * (bd.w - k);
        const int s = ((p1 > p2 ? p1 : p2) >= 0) ? 1 : 0;
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
        stS<PREC>(Sxx, e, sxx + (lam2mu * taup_plus1 * d3v3 - mu2 * taus_plus1 * dyVy_dzVz + Rxx_n) * dt, a.iS[0]);
        stS<PREC>(Syy, e, syy + (lam2mu * taup_plus1 * d3v3 - mu2 * taus_plus1 * dxVx_dzVz + Ryy_n) * dt, a.iS[1]);
        stS<PREC>(Szz, e, szz + (lam2mu * taup_plus1 * d3v3 - mu2 * taus_plus1 * dxVx_dyVy + Rzz_n) * dt, a.iS[2]);

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
        stS<PREC>(Syz, e, syz + (muyz * taus_plus1 * dyVz_dzVy + Ryz_n) * dt, a.iS[3]);
        stS<PREC>(Sxz, e, sxz + (muxz * taus_plus1 * dxVz_dzVx + Rxz_n) * dt, a.iS[4]);
        stS<PREC>(Sxy, e, sxy + (muxy * taus_plus1 * dxVy_dyVx + Rxy_n) * dt, a.iS[5]);
#pragma unroll
        for (int c = 0; c < 6; c++)
#pragma unroll
            for (int m = 0; m < NM; m++) stR<PREC>(a.R[c * 3 + m], e, r[c][m], a.iR[c * 3 + m]);
        return;
    }

    // absorber cell (m_absorb_p.f90:445-491)
    if (!(a.mask & 2)) return;
    const int2 pc = __ldg(&a.pmlcol[col]);
    const long long q = (long long)pc.y + (k - pc.x);
    float *__restrict__ axVx = a.aV[0];
    float *__restrict__ ayVx = a.aV[1];
    float *__restrict__ azVx = a.aV[2];
    float *__restrict__ axVy = a.aV[3];
    float *__restrict__ ayVy = a.aV[4];
    float *__restrict__ azVy = a.aV[5];
    float *__restrict__ axVz = a.aV[6];
    float *__restrict__ ayVz = a.aV[7];
    float *__restrict__ azVz = a.aV[8];
    const float vaxVx = lds(&axVx[q]), vayVy = lds(&ayVy[q]), vazVz = lds(&azVz[q]);
    const float vayVx = lds(&ayVx[q]), vazVx = lds(&azVx[q]), vaxVy = lds(&axVy[q]);
    const float vazVy = lds(&azVy[q]), vaxVz = lds(&axVz[q]), vayVz = lds(&ayVz[q]);
    const float sxx = ldS<PREC>(Sxx, e, a.sS[0]), syy = ldS<PREC>(Syy, e, a.sS[1]), szz = ldS<PREC>(Szz, e, a.sS[2]);
    const float syz = ldS<PREC>(Syz, e, a.sS[3]), sxz = ldS<PREC>(Sxz, e, a.sS[4]), sxy = ldS<PREC>(Sxy, e, a.sS[5]);
    const float mu = lds(&a.mu[e]), lam = lds(&a.lam[e]);
    const float muyz = lds(&a.muyz[e]), muxz = lds(&a.muxz[e]), muxy = lds(&a.muxy[e]);
    const float vx0 = __ldg(&Vx[e]), vy0 = __ldg(&Vy[e]), vz0 = __ldg(&Vz[e]);
    const float vxim = __ldg(&Vx[e - PI]), vyjm = __ldg(&Vy[e - PJ]), vzkm = __ldg(&Vz[e - 1]);
    const float vyip = __ldg(&Vy[e + PI]), vzip = __ldg(&Vz[e + PI]);
    const float vxjp = __ldg(&Vx[e + PJ]), vzjp = __ldg(&Vz[e + PJ]);
    const float vxkp = __ldg(&Vx[e + 1]), vykp = __ldg(&Vy[e + 1]);
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
    stS<PREC>(Sxx, e, sxx + (lam2mu_R * dxVx_ade + lam_R * (dyVy_ade + dzVz_ade)) * dt, a.iS[0]);
    stS<PREC>(Syy, e, syy + (lam2mu_R * dyVy_ade + lam_R * (dxVx_ade + dzVz_ade)) * dt, a.iS[1]);
    stS<PREC>(Szz, e, szz + (lam2mu_R * dzVz_ade + lam_R * (dxVx_ade + dyVy_ade)) * dt, a.iS[2]);
    sts(&axVx[q], gxc.z * vaxVx + gxc.w * dxVx * dt);
    sts(&ayVy[q], gyc.z * vayVy + gyc.w * dyVy * dt);
    sts(&azVz[q], gzc.z * vazVz + gzc.w * dzVz * dt);

    const float dxVy = (vyip - vy0) * r20x;
    const float dxVz = (vzip - vz0) * r20x;
    const float dyVx = (vxjp - vx0) * r20y;
    const float dyVz = (vzjp - vz0) * r20y;
    const float dzVx = (vxkp - vx0) * r20z;
    const float dzVy = (vykp - vy0) * r20z;
    stS<PREC>(Syz, e, syz + muyz * (gye.x * dyVz + gze.x * dzVy + gye.y * vayVz + gze.y * vazVy) * dt, a.iS[3]);
    stS<PREC>(Sxz, e, sxz + muxz * (gxe.x * dxVz + gze.x * dzVx + gxe.y * vaxVz + gze.y * vazVx) * dt, a.iS[4]);
    stS<PREC>(Sxy, e, sxy + muxy * (gxe.x * dxVy + gye.x * dyVx + gxe.y * vaxVy + gye.y * vayVx) * dt, a.iS[5]);
    sts(&ayVx[q], gye.z * vayVx + gye.w * dyVx * dt);
    sts(&azVx[q], gze.z * vazVx + gze.w * dzVx * dt);
    sts(&axVy[q], gxe.z * vaxVy + gxe.w * dxVy * dt);
    sts(&azVy[q], gze.z * vazVy + gze.w * dzVy * dt);
    sts(&axVz[q], gxe.z * vaxVz + gxe.w * dxVz * dt);
    sts(&ayVz[q], gye.z * vayVz + gye.w * dyVz * dt);
}

// MINB (minimum resident blocks per SM) trades registers for occupancy; the
// launch table picks it per kernel (swpc_set_launch)
template <int PREC>
static void vel_minb(const Vel3Args &a, int minb, dim3 grid, dim3 block, cudaStream_t st) {
    switch (minb) {
    case 1: vel3d_kernel<1, PREC><<<grid, block, 0, st>>>(a); break;
    case 2: vel3d_kernel<2, PREC><<<grid, block, 0, st>>>(a); break;
    case 3: vel3d_kernel<3, PREC><<<grid, block, 0, st>>>(a); break;
    default: vel3d_kernel<4, PREC><<<grid, block, 0, st>>>(a); break;
    }
}

void launch_vel3d(const Vel3Args &a, int minb, int prec, dim3 grid, dim3 block, cudaStream_t st) {
    // S is read in FP16 only by the PREC_F16_SR form; the others share the FP32 kernel
    if (prec == PREC_F16_SR) vel_minb<PREC_F16_SR>(a, minb, grid, block, st);
    else vel_minb<PREC_F32>(a, minb, grid, block, st);
}

template <int NM, int PREC>
static void stress_minb(const Str3Args &a, int minb, dim3 grid, dim3 block, cudaStream_t st) {
    switch (minb) {
    case 1: stress3d_kernel<NM, 1, PREC><<<grid, block, 0, st>>>(a); break;
    case 2: stress3d_kernel<NM, 2, PREC><<<grid, block, 0, st>>>(a); break;
    case 3: stress3d_kernel<NM, 3, PREC><<<grid, block, 0, st>>>(a); break;
    default: stress3d_kernel<NM, 4, PREC><<<grid, block, 0, st>>>(a); break;
    }
}

template <int PREC>
static void stress_nm(const Str3Args &a, int nm, int minb, dim3 grid, dim3 block, cudaStream_t st) {
    switch (nm) {
    case 0: stress_minb<0, PREC>(a, minb, grid, block, st); break;
    case 1: stress_minb<1, PREC>(a, minb, grid, block, st); break;
    case 2: stress_minb<2, PREC>(a, minb, grid, block, st); break;
    default: stress_minb<3, PREC>(a, minb, grid, block, st); break;
    }
}

void launch_stress3d(const Str3Args &a, int nm, int minb, int prec, dim3 grid, dim3 block, cudaStream_t st) {
    switch (prec) {
    case PREC_BF16_R: stress_nm<PREC_BF16_R>(a, nm, minb, grid, block, st); break;
    case PREC_F16_SR: stress_nm<PREC_F16_SR>(a, nm, minb, grid, block, st); break;
    default: stress_nm<PREC_F32>(a, nm, minb, grid, block, st); break;
    }
}

// ---------------------------------------------------------------------------
// point sources: source__stressglut (m_source.f90:798-826),
// source__bodyforce (:854-870), green__source (m_green.f90:615-627).
// Entries are applied in list order; when no two entries touch the same
// cell the host marks the list parallel and each entry gets a thread.
// ---------------------------------------------------------------------------
// S -= coef * sdrop / div on an FP16 stress array (SWPC_PREC_F16_SR)
__device__ __forceinline__ void glut_half(const InjArgs &a, const InjEntry &en, float sdrop, int div) {
    __half *h = reinterpret_cast<__half *>(a.fields[en.field]);
    const int c = en.field - SWPC_F_SXX;
    const float v = __half2float(h[en.cell]) * a.sS[c];
    const float w = div == 1 ? v - en.coef * sdrop : v - en.coef * sdrop / div;
    h[en.cell] = __float2half_rn(w * a.iS[c]);
}

__device__ __forceinline__ void apply_entry(const InjArgs &a, const InjEntry &en, int it) {
    float *f = a.fields[en.field];
    const float st = a.stime[(long long)(it - 1) * a.nsrc + en.src];
    if (a.s_half && en.field >= SWPC_F_SXX && en.mode <= INJ_GLUT2) {
        const float sdrop = a.mo[en.src] * st * a.dt_dxyz;
        glut_half(a, en, sdrop, en.mode == INJ_GLUT ? 1 : (en.mode == INJ_GLUT4 ? 4 : 2));
        return;
    }
    switch (en.mode) {
    case INJ_GLUT: {        // S -= m * sdrop, sdrop = mo * stime * dt_dxyz
        const float sdrop = a.mo[en.src] * st * a.dt_dxyz;
        f[en.cell] = f[en.cell] - en.coef * sdrop;
        break;
    }
    case INJ_GLUT4: {       // S -= m * sdrop / 4 (3D and P-SV shear cells)
        const float sdrop = a.mo[en.src] * st * a.dt_dxyz;
        f[en.cell] = f[en.cell] - en.coef * sdrop / 4;
        break;
    }
    case INJ_GLUT2: {       // S -= m * sdrop / 2 (SH, src/swpc_sh/m_source.f90:583-587)
        const float sdrop = a.mo[en.src] * st * a.dt_dxyz;
        f[en.cell] = f[en.cell] - en.coef * sdrop / 2;
        break;
    }
    case INJ_BF3: {         // V += b * f * stime * dt_dxyz / 2 (m_source.f90:863-868)
        const float b = a.bfields[en.bfield][en.cell];
        f[en.cell] = f[en.cell] + b * en.coef * st * a.dt_dxyz / 2;
        break;
    }
    case INJ_GREEN: {       // fx = fx1 * dt_dxyz * stf ; V += b * fx / 2 (m_green.f90:617-627)
        const float fv = en.coef * a.dt_dxyz * st;
        const float b = a.bfields[en.bfield][en.cell];
        f[en.cell] = f[en.cell] + b * fv / 2;
        break;
    }
    case INJ_BFPSV: {       // V += f / rho(kk,ii) * stime * dt_dxz / 2 (src/swpc_psv/m_source.f90:640-645)
        const float rho = a.bfields[0][a.rho_cell[en.src]];
        f[en.cell] = f[en.cell] + en.coef / rho * st * a.dt_dxyz / 2;
        break;
    }
    case INJ_BFSH: {        // Vy += f / rho(kk,ii) * stime * dt_dxz (src/swpc_sh/m_source.f90:621)
        const float rho = a.bfields[0][a.rho_cell[en.src]];
        f[en.cell] = f[en.cell] + en.coef / rho * st * a.dt_dxyz;
        break;
    }
    default: break;
    }
}

__global__ void inject_kernel(const InjArgs a) {
    const int it = a.d_it ? *a.d_it : a.it;
    if (it < 1 || it > a.nt) return;
    if (a.serial) {
        if (blockIdx.x == 0 && threadIdx.x == 0)
            for (int n = 0; n < a.n; n++) apply_entry(a, a.list[n], it);
        return;
    }
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < a.n) apply_entry(a, a.list[n], it);
}

// many injection lists in one launch (batched ensembles): blockIdx.y picks
// the list; each list keeps its own serial / parallel mode
__global__ void inject_multi_kernel(const InjArgs *__restrict__ list, int nlist, const int *d_it, int it_arg) {
    const int it = d_it ? *d_it : it_arg;
    for (int b = blockIdx.y; b < nlist; b += gridDim.y) {
        const InjArgs &a = list[b];
        if (it < 1 || it > a.nt) continue;
        if (a.serial) {
            if (blockIdx.x == 0 && threadIdx.x == 0)
                for (int n = 0; n < a.n; n++) apply_entry(a, a.list[n], it);
            continue;
        }
        for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < a.n; n += gridDim.x * blockDim.x)
            apply_entry(a, a.list[n], it);
    }
}

void launch_inject_multi(const InjArgs *list, int nlist, int max_n, const int *d_it, int it, cudaStream_t st) {
    if (!list || nlist <= 0 || max_n <= 0) return;
    const int threads = 128;
    const dim3 grid((max_n + threads - 1) / threads, nlist < 65535 ? nlist : 65535);
    inject_multi_kernel<<<grid, threads, 0, st>>>(list, nlist, d_it, it);
}

void launch_inject(const InjArgs &a, cudaStream_t st) {
    if (a.n <= 0) return;
    const int threads = 128;
    const int blocks = a.serial ? 1 : (a.n + threads - 1) / threads;
    inject_kernel<<<blocks, threads, 0, st>>>(a);
}

// ---------------------------------------------------------------------------
// wav__store (m_wav.f90:433-620): one thread per station
// ---------------------------------------------------------------------------
__global__ void wav3d_kernel(const Wav3Args a) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.nst) return;
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
                return __half2float(reinterpret_cast<const __half *>(p)[q]) * a.sS[c];
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

void launch_wav3d(const Wav3Args &a, cudaStream_t st) {
    if (a.nst <= 0) return;
    const int threads = 128;
    wav3d_kernel<<<(a.nst + threads - 1) / threads, threads, 0, st>>>(a);
}

// ---------------------------------------------------------------------------
// kernel__vmax (m_kernel.f90:328-352): max |V(kob+1, i, j)|; |x| of a finite
// float orders like its bit pattern, so the max is an atomicMax on the bits.
// ---------------------------------------------------------------------------
__global__ void vmax3d_kernel(const VmaxArgs a) {
    const int ni = a.i1 - a.i0 + 1, nj = a.j1 - a.j0 + 1;
    const long long n = (long long)ni * nj;
    unsigned int mx = 0, my = 0, mz = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = a.i0 + (int)(t % ni), j = a.j0 + (int)(t / ni);
        const long long col = col_index(a.g, i, j);
        const int k = a.kob[col] + 1;
        const long long e = col * a.g.Kp + (k - 1 + KH);
        const unsigned int bx = __float_as_uint(fabsf(a.Vx[e]));
        const unsigned int by = __float_as_uint(fabsf(a.Vy[e]));
        const unsigned int bz = __float_as_uint(fabsf(a.Vz[e]));
        mx = max(mx, bx);
        my = max(my, by);
        mz = max(mz, bz);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        my = max(my, __shfl_xor_sync(0xffffffffu, my, o));
        mz = max(mz, __shfl_xor_sync(0xffffffffu, mz, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&a.out[0], mx);
        atomicMax(&a.out[1], my);
        atomicMax(&a.out[2], mz);
    }
}

void launch_vmax3d(const VmaxArgs &a, cudaStream_t st) {
    vmax3d_kernel<<<148, 256, 0, st>>>(a);
}

__global__ void advance_it_kernel(int *d_it) { *d_it = *d_it + 1; }
void launch_advance_it(int *d_it, cudaStream_t st) { advance_it_kernel<<<1, 1, 0, st>>>(d_it); }

}  // namespace swpc
