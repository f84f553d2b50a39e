// swpc3d_march.cu -- 2.5D marching variants of the fused 3D kernels.
//
// A block owns a 32 (k) x BI (i) tile of columns and walks along j over a
// chunk of JC planes.  The stencil operands come from on-chip storage:
//   - j-neighbours live in per-thread register windows that shift by one
//     plane per step (one new coalesced load per field per step);
//   - k- and i-neighbours come from a shared-memory copy of the current
//     (k, i) plane with a 2-cell halo, filled by the block each step.
// Every global element of the stencil fields is then read about once from
// L2/HBM (plus the i-halo), instead of once per neighbouring cell, and the
// per-cell load count drops from ~58 to ~36 (the pointwise streams).
//
// The arithmetic is the expression-for-expression copy of swpc3d_kernels.cu
// (same operand order, -fmad=false), so results are bitwise identical to the
// flat kernels and to the oracle; only where operands are read from changes.
#include <cuda_runtime.h>

#include "swpc_ctx.h"
#include "swpc_kernels.cuh"

namespace swpc {

namespace {

__device__ __forceinline__ float lds(const float *p) { return __ldcs(p); }
__device__ __forceinline__ void sts(float *p, float v) { __stcs(p, v); }

// plane tile: [field][i + 2][k + 2], k fastest (lane-consecutive, no bank
// conflicts); 36 = 32 + 2 + 2 k rows
constexpr int TK = 36;

}  // namespace

// ---------------------------------------------------------------------------
// stress (m_kernel.f90:142-326 + m_absorb_p.f90:424-503)
// ---------------------------------------------------------------------------
template <int NM, int BI, int MINB>
__global__ void __launch_bounds__(32 * BI, MINB) stress3d_march_kernel(const Str3Args a, int JC) {
    const Geo g = a.g;
    const int lane = threadIdx.x, ty = threadIdx.y;
    const int k0 = 1 + blockIdx.x * 32, i0 = 1 + blockIdx.y * BI;
    const int k = k0 + lane, i = i0 + ty;
    const int jb = 1 + blockIdx.z * JC;
    const int je = min(jb + JC - 1, g.ny);
    const long long PI = g.Kp, PJ = (long long)g.Kp * g.Ip;
    // cells inside the memory box can be read; cells inside the domain are updated
    const bool ld_ok = (k <= g.nz + 3) && (i <= g.nx + 3);
    const bool act = (k <= g.nz) && (i <= g.nx);
    __shared__ float tv[3][BI + 4][TK];

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

    // halo roles of this thread: k-halo rows (lane < 4), i-halo columns (ty < 4)
    const int kh = lane < 2 ? k0 - 2 + lane : k0 + 30 + lane;       // lanes 2,3 -> k0+32, k0+33
    const int kh_row = lane < 2 ? lane : 32 + lane;                 // 0,1,34,35
    const bool kh_ok = (lane < 4) && (kh <= g.nz + 3) && (i <= g.nx + 3);
    const int ih = ty < 2 ? i0 - 2 + ty : i0 + BI - 2 + ty;         // ty 2,3 -> i0+BI, i0+BI+1
    const int ih_col = ty < 2 ? ty : BI + ty;                       // 0,1,BI+2,BI+3
    const bool ih_ok = (ty < 4) && (ih <= g.nx + 3) && (k <= g.nz + 3);

    long long e = cell_index(g, k, i, jb);
    // register windows (j-neighbours): Vx j-1..j+2, Vy j-2..j+1, Vz j-1..j+2
    float x_m1 = 0, x_0 = 0, x_p1 = 0, x_p2 = 0, y_m2 = 0, y_m1 = 0, y_0 = 0, y_p1 = 0;
    float z_m1 = 0, z_0 = 0, z_p1 = 0, z_p2 = 0;
    if (ld_ok) {
        x_m1 = __ldg(&Vx[e - PJ]); x_0 = __ldg(&Vx[e]); x_p1 = __ldg(&Vx[e + PJ]);
        y_m2 = __ldg(&Vy[e - 2 * PJ]); y_m1 = __ldg(&Vy[e - PJ]); y_0 = __ldg(&Vy[e]);
        z_m1 = __ldg(&Vz[e - PJ]); z_0 = __ldg(&Vz[e]); z_p1 = __ldg(&Vz[e + PJ]);
    }
    for (int j = jb; j <= je; j++, e += PJ) {
        if (j > jb) {
            x_m1 = x_0; x_0 = x_p1; x_p1 = x_p2;
            y_m2 = y_m1; y_m1 = y_0; y_0 = y_p1;
            z_m1 = z_0; z_0 = z_p1; z_p1 = z_p2;
        }
        if (ld_ok) {
            x_p2 = __ldg(&Vx[e + 2 * PJ]);
            y_p1 = __ldg(&Vy[e + PJ]);
            z_p2 = __ldg(&Vz[e + 2 * PJ]);
        }
        const long long col = col_index(g, i, j);
        const bool inner = act && i >= a.ibk && i <= a.iek && j >= a.jbk && j <= a.jek && k <= a.kek;
        const bool pml = act && !inner;
        // pointwise operands of this cell, issued before the tile exchange
        float r[6][NM > 0 ? NM : 1];
        float sxx = 0, syy = 0, szz = 0, syz = 0, sxz = 0, sxy = 0;
        float mu = 0, lam = 0, taup1 = 0, taus1 = 0, muyz = 0, muxz = 0, muxy = 0;
        float va[9];
        int4 bd = make_int4(0, 0, 0, 0);
        long long q = 0;
        if (act) {
            sxx = lds(&Sxx[e]); syy = lds(&Syy[e]); szz = lds(&Szz[e]);
            syz = lds(&Syz[e]); sxz = lds(&Sxz[e]); sxy = lds(&Sxy[e]);
            mu = lds(&a.mu[e]); lam = lds(&a.lam[e]);
            muyz = lds(&a.muyz[e]); muxz = lds(&a.muxz[e]); muxy = lds(&a.muxy[e]);
        }
        if (inner) {
#pragma unroll
            for (int c = 0; c < 6; c++)
#pragma unroll
                for (int m = 0; m < NM; m++) r[c][m] = lds(&a.R[c * 3 + m][e]);
            taup1 = lds(&a.taup[e]);
            taus1 = lds(&a.taus[e]);
            bd = __ldg(&a.band[col]);
        }
        if (pml && (a.mask & 2)) {
            const int2 pc = __ldg(&a.pmlcol[col]);
            q = (long long)pc.y + (k - pc.x);
#pragma unroll
            for (int n = 0; n < 9; n++) va[n] = lds(&a.aV[n][q]);
        }
        // the (k, i) plane of V at j with its 2-cell halo
        __syncthreads();
        tv[0][ty + 2][lane + 2] = x_0;
        tv[1][ty + 2][lane + 2] = y_0;
        tv[2][ty + 2][lane + 2] = z_0;
        if (lane < 4) {
            const long long eh = e + (kh - k);
            float hx = 0, hy = 0, hz = 0;
            if (kh_ok) { hx = __ldg(&Vx[eh]); hy = __ldg(&Vy[eh]); hz = __ldg(&Vz[eh]); }
            tv[0][ty + 2][kh_row] = hx; tv[1][ty + 2][kh_row] = hy; tv[2][ty + 2][kh_row] = hz;
        }
        if (ty < 4) {
            const long long eh = e + (long long)(ih - i) * PI;
            float hx = 0, hy = 0, hz = 0;
            if (ih_ok) { hx = __ldg(&Vx[eh]); hy = __ldg(&Vy[eh]); hz = __ldg(&Vz[eh]); }
            tv[0][ih_col][lane + 2] = hx; tv[1][ih_col][lane + 2] = hy; tv[2][ih_col][lane + 2] = hz;
        }
        __syncthreads();
        if (!act) continue;
        const int c0 = ty + 2, r0 = lane + 2;
        const float vx0 = x_0, vy0 = y_0, vz0 = z_0;

        if (inner) {
            if (!(a.mask & 1)) continue;
            const float vxim = tv[0][c0 - 1][r0], vxip = tv[0][c0 + 1][r0], vxim2 = tv[0][c0 - 2][r0];
            const float vxkp = tv[0][c0][r0 + 1], vxkp2 = tv[0][c0][r0 + 2], vxkm = tv[0][c0][r0 - 1];
            const float vyip = tv[1][c0 + 1][r0], vyip2 = tv[1][c0 + 2][r0], vyim = tv[1][c0 - 1][r0];
            const float vykp = tv[1][c0][r0 + 1], vykp2 = tv[1][c0][r0 + 2], vykm = tv[1][c0][r0 - 1];
            const float vzip = tv[2][c0 + 1][r0], vzip2 = tv[2][c0 + 2][r0], vzim = tv[2][c0 - 1][r0];
            const float vzkm = tv[2][c0][r0 - 1], vzkp = tv[2][c0][r0 + 1], vzkm2 = tv[2][c0][r0 - 2];
            const float vxjp = x_p1, vxjp2 = x_p2, vxjm = x_m1;
            const float vyjm = y_m1, vyjp = y_p1, vyjm2 = y_m2;
            const float vzjp = z_p1, vzjp2 = z_p2, vzjm = z_m1;
            const int p1 = (k - bd.x) * (bd.y - k);
            const int p2 = (k - bd.z) * (bd.w - k);
            const int s = ((p1 > p2 ? p1 : p2) >= 0) ? 1 : 0;
            const float re40x = a.e40[0][s], re41x = a.e41[0][s];
            const float re40y = a.e40[1][s], re41y = a.e41[1][s];
            const float re40z = a.e40[2][s], re41z = a.e41[2][s];

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
            sts(&Sxx[e], sxx + (lam2mu * taup_plus1 * d3v3 - mu2 * taus_plus1 * dyVy_dzVz + Rxx_n) * dt);
            sts(&Syy[e], syy + (lam2mu * taup_plus1 * d3v3 - mu2 * taus_plus1 * dxVx_dzVz + Ryy_n) * dt);
            sts(&Szz[e], szz + (lam2mu * taup_plus1 * d3v3 - mu2 * taus_plus1 * dxVx_dyVy + Rzz_n) * dt);

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
            sts(&Syz[e], syz + (muyz * taus_plus1 * dyVz_dzVy + Ryz_n) * dt);
            sts(&Sxz[e], sxz + (muxz * taus_plus1 * dxVz_dzVx + Rxz_n) * dt);
            sts(&Sxy[e], sxy + (muxy * taus_plus1 * dxVy_dyVx + Rxy_n) * dt);
#pragma unroll
            for (int c = 0; c < 6; c++)
#pragma unroll
                for (int m = 0; m < NM; m++) sts(&a.R[c * 3 + m][e], r[c][m]);
            continue;
        }

        // absorber cell (m_absorb_p.f90:445-491)
        if (!(a.mask & 2)) continue;
        const float vaxVx = va[0], vayVx = va[1], vazVx = va[2], vaxVy = va[3], vayVy = va[4];
        const float vazVy = va[5], vaxVz = va[6], vayVz = va[7], vazVz = va[8];
        const float vxim = tv[0][c0 - 1][r0], vyjm = y_m1, vzkm = tv[2][c0][r0 - 1];
        const float vyip = tv[1][c0 + 1][r0], vzip = tv[2][c0 + 1][r0];
        const float vxjp = x_p1, vzjp = z_p1;
        const float vxkp = tv[0][c0][r0 + 1], vykp = tv[1][c0][r0 + 1];
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
        sts(&Sxx[e], sxx + (lam2mu_R * dxVx_ade + lam_R * (dyVy_ade + dzVz_ade)) * dt);
        sts(&Syy[e], syy + (lam2mu_R * dyVy_ade + lam_R * (dxVx_ade + dzVz_ade)) * dt);
        sts(&Szz[e], szz + (lam2mu_R * dzVz_ade + lam_R * (dxVx_ade + dyVy_ade)) * dt);
        sts(&a.aV[0][q], gxc.z * vaxVx + gxc.w * dxVx * dt);
        sts(&a.aV[4][q], gyc.z * vayVy + gyc.w * dyVy * dt);
        sts(&a.aV[8][q], gzc.z * vazVz + gzc.w * dzVz * dt);

        const float dxVy = (vyip - vy0) * r20x;
        const float dxVz = (vzip - vz0) * r20x;
        const float dyVx = (vxjp - vx0) * r20y;
        const float dyVz = (vzjp - vz0) * r20y;
        const float dzVx = (vxkp - vx0) * r20z;
        const float dzVy = (vykp - vy0) * r20z;
        sts(&Syz[e], syz + muyz * (gye.x * dyVz + gze.x * dzVy + gye.y * vayVz + gze.y * vazVy) * dt);
        sts(&Sxz[e], sxz + muxz * (gxe.x * dxVz + gze.x * dzVx + gxe.y * vaxVz + gze.y * vazVx) * dt);
        sts(&Sxy[e], sxy + muxy * (gxe.x * dxVy + gye.x * dyVx + gxe.y * vaxVy + gye.y * vayVx) * dt);
        sts(&a.aV[1][q], gye.z * vayVx + gye.w * dyVx * dt);
        sts(&a.aV[2][q], gze.z * vazVx + gze.w * dzVx * dt);
        sts(&a.aV[3][q], gxe.z * vaxVy + gxe.w * dxVy * dt);
        sts(&a.aV[5][q], gze.z * vazVy + gze.w * dzVy * dt);
        sts(&a.aV[6][q], gxe.z * vaxVz + gxe.w * dxVz * dt);
        sts(&a.aV[7][q], gye.z * vayVz + gye.w * dyVz * dt);
    }
}

// ---------------------------------------------------------------------------
// velocity (m_kernel.f90:75-140 + m_absorb_p.f90:248-309)
// ---------------------------------------------------------------------------
template <int BI, int MINB>
__global__ void __launch_bounds__(32 * BI, MINB) vel3d_march_kernel(const Vel3Args a, int JC) {
    const Geo g = a.g;
    const int lane = threadIdx.x, ty = threadIdx.y;
    const int k0 = 1 + blockIdx.x * 32, i0 = 1 + blockIdx.y * BI;
    const int k = k0 + lane, i = i0 + ty;
    const int jb = 1 + blockIdx.z * JC;
    const int je = min(jb + JC - 1, g.ny);
    const long long PI = g.Kp, PJ = (long long)g.Kp * g.Ip;
    const bool ld_ok = (k <= g.nz + 3) && (i <= g.nx + 3);
    const bool act = (k <= g.nz) && (i <= g.nx);
    // tiles: 0 Sxx (i), 1 Sxy (i), 2 Sxz (i, k), 3 Syz (k), 4 Szz (k)
    __shared__ float ts[5][BI + 4][TK];

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

    const int kh = lane < 2 ? k0 - 2 + lane : k0 + 30 + lane;
    const int kh_row = lane < 2 ? lane : 32 + lane;
    const bool kh_ok = (lane < 4) && (kh <= g.nz + 3) && (i <= g.nx + 3);
    const int ih = ty < 2 ? i0 - 2 + ty : i0 + BI - 2 + ty;
    const int ih_col = ty < 2 ? ty : BI + ty;
    const bool ih_ok = (ty < 4) && (ih <= g.nx + 3) && (k <= g.nz + 3);

    long long e = cell_index(g, k, i, jb);
    // windows: Sxy j-2..j+1, Syy j-1..j+2, Syz j-2..j+1
    float xy_m2 = 0, xy_m1 = 0, xy_0 = 0, xy_p1 = 0, yy_m1 = 0, yy_0 = 0, yy_p1 = 0, yy_p2 = 0;
    float yz_m2 = 0, yz_m1 = 0, yz_0 = 0, yz_p1 = 0;
    if (ld_ok) {
        xy_m2 = __ldg(&Sxy[e - 2 * PJ]); xy_m1 = __ldg(&Sxy[e - PJ]); xy_0 = __ldg(&Sxy[e]);
        yy_m1 = __ldg(&Syy[e - PJ]); yy_0 = __ldg(&Syy[e]); yy_p1 = __ldg(&Syy[e + PJ]);
        yz_m2 = __ldg(&Syz[e - 2 * PJ]); yz_m1 = __ldg(&Syz[e - PJ]); yz_0 = __ldg(&Syz[e]);
    }
    for (int j = jb; j <= je; j++, e += PJ) {
        if (j > jb) {
            xy_m2 = xy_m1; xy_m1 = xy_0; xy_0 = xy_p1;
            yy_m1 = yy_0; yy_0 = yy_p1; yy_p1 = yy_p2;
            yz_m2 = yz_m1; yz_m1 = yz_0; yz_0 = yz_p1;
        }
        float xx_0 = 0, xz_0 = 0, zz_0 = 0;
        if (ld_ok) {
            xy_p1 = __ldg(&Sxy[e + PJ]);
            yy_p2 = __ldg(&Syy[e + 2 * PJ]);
            yz_p1 = __ldg(&Syz[e + PJ]);
            xx_0 = __ldg(&Sxx[e]);
            xz_0 = __ldg(&Sxz[e]);
            zz_0 = __ldg(&Szz[e]);
        }
        const long long col = col_index(g, i, j);
        const bool inner = act && i >= a.ibk && i <= a.iek && j >= a.jbk && j <= a.jek && k <= a.kek;
        const bool pml = act && !inner;
        float vx = 0, vy = 0, vz = 0, bx = 0, by = 0, bz = 0;
        float va[9];
        int4 bd = make_int4(0, 0, 0, 0);
        long long q = 0;
        if (act) {
            vx = lds(&Vx[e]); vy = lds(&Vy[e]); vz = lds(&Vz[e]);
            bx = lds(&a.bx[e]); by = lds(&a.by[e]); bz = lds(&a.bz[e]);
        }
        if (inner) bd = __ldg(&a.band[col]);
        if (pml && (a.mask & 2)) {
            const int2 pc = __ldg(&a.pmlcol[col]);
            q = (long long)pc.y + (k - pc.x);
#pragma unroll
            for (int n = 0; n < 9; n++) va[n] = lds(&a.aS[n][q]);
        }
        __syncthreads();
        ts[0][ty + 2][lane + 2] = xx_0;
        ts[1][ty + 2][lane + 2] = xy_0;
        ts[2][ty + 2][lane + 2] = xz_0;
        ts[3][ty + 2][lane + 2] = yz_0;
        ts[4][ty + 2][lane + 2] = zz_0;
        if (lane < 4) {
            const long long eh = e + (kh - k);
            float h2 = 0, h3 = 0, h4 = 0;
            if (kh_ok) { h2 = __ldg(&Sxz[eh]); h3 = __ldg(&Syz[eh]); h4 = __ldg(&Szz[eh]); }
            ts[2][ty + 2][kh_row] = h2; ts[3][ty + 2][kh_row] = h3; ts[4][ty + 2][kh_row] = h4;
        }
        if (ty < 4) {
            const long long eh = e + (long long)(ih - i) * PI;
            float h0 = 0, h1 = 0, h2 = 0;
            if (ih_ok) { h0 = __ldg(&Sxx[eh]); h1 = __ldg(&Sxy[eh]); h2 = __ldg(&Sxz[eh]); }
            ts[0][ih_col][lane + 2] = h0; ts[1][ih_col][lane + 2] = h1; ts[2][ih_col][lane + 2] = h2;
        }
        __syncthreads();
        if (!act) continue;
        const int c0 = ty + 2, r0 = lane + 2;

        if (inner) {
            if (!(a.mask & 1)) continue;
            const float xx0 = xx_0, xxp = ts[0][c0 + 1][r0], xxp2 = ts[0][c0 + 2][r0], xxm = ts[0][c0 - 1][r0];
            const float yy0 = yy_0, yyp = yy_p1, yyp2 = yy_p2, yym = yy_m1;
            const float zz0 = zz_0, zzp = ts[4][c0][r0 + 1], zzp2 = ts[4][c0][r0 + 2], zzm = ts[4][c0][r0 - 1];
            const float xy0 = xy_0, xyjm = xy_m1, xyjp = xy_p1, xyjm2 = xy_m2;
            const float xyim = ts[1][c0 - 1][r0], xyip = ts[1][c0 + 1][r0], xyim2 = ts[1][c0 - 2][r0];
            const float xz0 = xz_0, xzkm = ts[2][c0][r0 - 1], xzkp = ts[2][c0][r0 + 1], xzkm2 = ts[2][c0][r0 - 2];
            const float xzim = ts[2][c0 - 1][r0], xzip = ts[2][c0 + 1][r0], xzim2 = ts[2][c0 - 2][r0];
            const float yz0 = yz_0, yzkm = ts[3][c0][r0 - 1], yzkp = ts[3][c0][r0 + 1], yzkm2 = ts[3][c0][r0 - 2];
            const float yzjm = yz_m1, yzjp = yz_p1, yzjm2 = yz_m2;
            const int p1 = (k - bd.x) * (bd.y - k);
            const int p2 = (k - bd.z) * (bd.w - k);
            const int s = ((p1 > p2 ? p1 : p2) >= 0) ? 1 : 0;
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
            continue;
        }

        if (!(a.mask & 2)) continue;
        const float vxSxx = va[0], vySxy = va[1], vzSxz = va[2], vxSxy = va[3], vySyy = va[4];
        const float vzSyz = va[5], vxSxz = va[6], vySyz = va[7], vzSzz = va[8];
        const float4 gxc = __ldg(&a.gxc[i - 1]), gxe = __ldg(&a.gxe[i - 1]);
        const float4 gyc = __ldg(&a.gyc[j - 1]), gye = __ldg(&a.gye[j - 1]);
        const float4 gzc = __ldg(&a.gzc[k - 1]), gze = __ldg(&a.gze[k - 1]);
        const float r20x = a.r20[0], r20y = a.r20[1], r20z = a.r20[2];
        const float dxSxx = (ts[0][c0 + 1][r0] - xx_0) * r20x;
        const float dySyy = (yy_p1 - yy_0) * r20y;
        const float dzSzz = (ts[4][c0][r0 + 1] - zz_0) * r20z;
        const float dySyz = (yz_0 - yz_m1) * r20y;
        const float dzSyz = (yz_0 - ts[3][c0][r0 - 1]) * r20z;
        const float dxSxz = (xz_0 - ts[2][c0 - 1][r0]) * r20x;
        const float dzSxz = (xz_0 - ts[2][c0][r0 - 1]) * r20z;
        const float dxSxy = (xy_0 - ts[1][c0 - 1][r0]) * r20x;
        const float dySxy = (xy_0 - xy_m1) * r20y;
        sts(&Vx[e], vx + bx * (gxe.x * dxSxx + gyc.x * dySxy + gzc.x * dzSxz
                               + gxe.y * vxSxx + gyc.y * vySxy + gzc.y * vzSxz) * dt);
        sts(&Vy[e], vy + by * (gxc.x * dxSxy + gye.x * dySyy + gzc.x * dzSyz
                               + gxc.y * vxSxy + gye.y * vySyy + gzc.y * vzSyz) * dt);
        sts(&Vz[e], vz + bz * (gxc.x * dxSxz + gyc.x * dySyz + gze.x * dzSzz
                               + gxc.y * vxSxz + gyc.y * vySyz + gze.y * vzSzz) * dt);
        sts(&a.aS[0][q], gxe.z * vxSxx + gxe.w * dxSxx * dt);
        sts(&a.aS[1][q], gyc.z * vySxy + gyc.w * dySxy * dt);
        sts(&a.aS[2][q], gzc.z * vzSxz + gzc.w * dzSxz * dt);
        sts(&a.aS[3][q], gxc.z * vxSxy + gxc.w * dxSxy * dt);
        sts(&a.aS[4][q], gye.z * vySyy + gye.w * dySyy * dt);
        sts(&a.aS[5][q], gzc.z * vzSyz + gzc.w * dzSyz * dt);
        sts(&a.aS[6][q], gxc.z * vxSxz + gxc.w * dxSxz * dt);
        sts(&a.aS[7][q], gyc.z * vySyz + gyc.w * dySyz * dt);
        sts(&a.aS[8][q], gze.z * vzSzz + gze.w * dzSzz * dt);
    }
}

// launch helpers: BI is fixed to 8 (a 32 x 8 plane tile, 256 threads)
template <int NM>
static void stress_march_minb(const Str3Args &a, int minb, int jc, dim3 grid, cudaStream_t st) {
    const dim3 block(32, 8, 1);
    switch (minb) {
    case 1: stress3d_march_kernel<NM, 8, 1><<<grid, block, 0, st>>>(a, jc); break;
    case 2: stress3d_march_kernel<NM, 8, 2><<<grid, block, 0, st>>>(a, jc); break;
    case 3: stress3d_march_kernel<NM, 8, 3><<<grid, block, 0, st>>>(a, jc); break;
    default: stress3d_march_kernel<NM, 8, 4><<<grid, block, 0, st>>>(a, jc); break;
    }
}

void launch_stress3d_march(const Str3Args &a, int nm, int minb, int jc, cudaStream_t st) {
    const dim3 grid((a.g.nz + 31) / 32, (a.g.nx + 7) / 8, (a.g.ny + jc - 1) / jc);
    switch (nm) {
    case 0: stress_march_minb<0>(a, minb, jc, grid, st); break;
    case 1: stress_march_minb<1>(a, minb, jc, grid, st); break;
    case 2: stress_march_minb<2>(a, minb, jc, grid, st); break;
    default: stress_march_minb<3>(a, minb, jc, grid, st); break;
    }
}

void launch_vel3d_march(const Vel3Args &a, int minb, int jc, cudaStream_t st) {
    const dim3 grid((a.g.nz + 31) / 32, (a.g.nx + 7) / 8, (a.g.ny + jc - 1) / jc);
    const dim3 block(32, 8, 1);
    switch (minb) {
    case 1: vel3d_march_kernel<8, 1><<<grid, block, 0, st>>>(a, jc); break;
    case 2: vel3d_march_kernel<8, 2><<<grid, block, 0, st>>>(a, jc); break;
    case 3: vel3d_march_kernel<8, 3><<<grid, block, 0, st>>>(a, jc); break;
    default: vel3d_march_kernel<8, 4><<<grid, block, 0, st>>>(a, jc); break;
    }
}

}  // namespace swpc
