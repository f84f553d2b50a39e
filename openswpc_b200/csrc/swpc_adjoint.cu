// swpc_adjoint.cu -- discrete adjoint of the 3D viscoelastic step and the
// gradient of an L2 velocity-waveform misfit with respect to the medium.
//
// The forward step (kernel__update_stress + absorb_p__update_stress, then
// kernel__update_vel + absorb_p__update_vel; src/swpc_3d/m_kernel.f90:75-326,
// src/swpc_3d/m_absorb_p.f90:126-505) is linear in the wavefield state
// (V, S, R, PML auxiliaries).  This file applies its exact transpose, in the
// reverse order, as two kinds of passes per half step:
//   weights: per cell, the adjoint of that cell's own update -- memory
//            variables and PML auxiliaries in place, and for each of the
//            nine (field, axis) difference operators the two weights that
//            multiply the 4th-order coefficient pair (2nd-order difference
//            r20 and zero in absorber cells);
//   gather:  per cell, the transposed stencil: every neighbour that read this
//            cell adds its weight with the sign of the difference.
// Receiver residuals enter as sources at the transposed recorder cells
// (wav__store, src/swpc_3d/m_wav.f90:530-535).  The gradient imaging
// condition pairs the adjoint with the forward derivatives of the same step;
// each step's term is formed in FP64 and added into an FP32 partial sum that
// covers one checkpoint segment (at most ckpt steps), and every segment's
// partials are folded into the FP64 totals (blocked summation: the FP32 sums
// hold ckpt terms, the FP64 ones the segments).  It is formed on the interior
// kernel region, whose cells are the model parameters (absorber cells copy the
// medium of the interior edge and are not parameters).  swpc_gradient runs
// the forward with checkpoints every `ckpt` steps, then per segment
// recomputes the forward from its checkpoint, keeping V and the stress
// divergences of every step, and steps the adjoint back through it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "swpc_ctx.h"
#include "swpc_kernels.cuh"
#include "swpc_tma.h"
#include "swpc_tma_ptx.cuh"
#include "swpc_tma_tile.cuh"

namespace swpc {
int graph_invalidate(swpc_ctx *c);
int copy_box(swpc_ctx *c, float *dev, const float *host_in, float *host_out, int ld_k, int ld_i);
int aux_transfer_ptr(swpc_ctx *c, float *dev, float *out, const float *in, int ld_k, int ld_i);
}  // namespace swpc

using namespace swpc;

// adjoint state of a context
struct swpc_adj_state {
    float *lV[3] = {}, *lS[6] = {}, *lR[18] = {}, *laux[18] = {};
    float *slab = nullptr;               // lV, lS, lR in the forward slab's field order (V, S, R)
    int slab_nf = 0;
    swpc::TmaMaps *maps = nullptr;       // staged stress-phase weights: state, s6 (adjoint slab), med, vh (slots)
    float *w40[9] = {}, *w41[9] = {};    // difference-operator weights of the stress phase
    float *w40v[9] = {}, *w41v[9] = {};  // and of the velocity phase (formed while the stress-phase ones are read)
    unsigned char *srcmask = nullptr;    // cells whose lambda_V a receiver residual changes
    int *srccells = nullptr;             // the same cells: (k, i, j) triplets, then nsrc + 1 offsets into the
                                         // contributions (station << 2 | component), in station order
    int nsrc = 0, nsrc_contrib = 0;
    double *grad[8] = {};                // lam mu muyz muxz muxy bx by bz: FP64 totals
    float *gpart[8] = {};                // the same, FP32 partial sums of the current segment
    float *res = nullptr;                // receiver residuals (nst, 3, ntw)
    int ckpt = 0, nseg = 0;
    float *ckpool = nullptr;             // checkpoints: V S R aux per segment
    float *slots = nullptr;              // V and the stress divergences after each step of a segment, or of
                                         // the trailing segments kept from the first forward pass
    size_t ck_floats = 0, slot_cap = 0;  // floats per checkpoint; slots allocated
    long long slot_budget = 0;           // bytes the kept steps of trailing segments may take (0: recompute all)
    int ntail = 0;                       // trailing segments whose steps the forward pass keeps
    float *keep = nullptr;               // kept segments: V of each segment's first state, then per kept step the
    size_t keep_floats = 0;              //   divergences and V on the slot box's shell (or the whole box)
    int *shell = nullptr;                // slot-box indices of the shell cells (slot box less the interior)
    int nshell = 0;
    long long bytes = 0;
};

namespace {

constexpr int kThreadsK = 32;

// Layout of a recompute slot: the box of the kernel region with a two-cell
// halo in i and j (i0 = ibk - 2, j0 = jbk - 2) over k up to kek + 2, the part
// of V the imaging condition reads (the stress-phase gradient takes V at
// i-2..i+2, j-2..j+2, k-2..k+2 of interior cells) and of the divergences it
// needs (interior cells).  Cell (k, i, j) at ((j - j0) * Ip + (i - i0)) * Kp +
// (k - 1 + KH): the k origin of the memory box, so TMA boxes keep their x.
struct SlotGeo {
    int Kp, Ip, Jp, i0, j0;
    long long n;
};
__host__ __device__ __forceinline__ long long slot_index(const SlotGeo &s, int k, int i, int j) {
    return ((long long)(j - s.j0) * s.Ip + (i - s.i0)) * s.Kp + (k - 1 + KH);
}

struct AdjVelArgs {
    Geo g;
    int ibk, iek, jbk, jek, kek;
    const float *lV[3];
    const float *b[3];
    const int4 *band;
    const int2 *pmlcol;
    float *laS[9];               // adjoint of the velocity-phase PML auxiliaries
    const float4 *gxc, *gxe, *gyc, *gye, *gzc, *gze;
    float e40[3][2], e41[3][2], r20[3], dt;
    float *w40[9], *w41[9];
    const float *divS[3];        // forward stress divergences after the stress update (gradient, slot layout)
    float *gb[3];                // segment partials of the bx, by, bz gradient (null: none)
    SlotGeo sg;
};

struct AdjStrArgs {
    Geo g;
    int ibk, iek, jbk, jek, kek, nm;
    const float *lS[6];
    float *lR[18];
    const float *lam, *mu, *taup, *taus, *muyz, *muxz, *muxy;
    const int4 *band;
    const int2 *pmlcol;
    float *laV[9];               // adjoint of the stress-phase PML auxiliaries
    const float4 *gxc, *gxe, *gyc, *gye, *gzc, *gze;
    float e40[3][2], e41[3][2], r20[3], dt;
    float c1[NM_MAX], c2[NM_MAX], d1[NM_MAX], d2;
    float *w40[9], *w41[9];
    const float *V[3];           // forward V before the stress update (gradient, slot layout)
    float *gm[5];                // segment partials of the lam, mu, muyz, muxz, muxy gradient (null: none)
    SlotGeo sg;
};

struct GatherArgs {
    Geo g;
    float *dst[6];
    const float *w40[9], *w41[9];
};

__device__ __forceinline__ bool cell_of(const Geo &g, int &k, int &i, int &j) {
    k = 1 + blockIdx.x * kThreadsK + threadIdx.x;
    i = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    j = 1 + blockIdx.z * blockDim.z + threadIdx.z;
    return k <= g.nz && i <= g.nx && j <= g.ny;
}

// axis of the difference operator of stress-phase pair q (x 0, y 1, z 2)
__device__ __forceinline__ int qaxis(int q) { return (q == 0 || q == 3 || q == 5) ? 0 : (q == 1 || q == 4 || q == 7) ? 1 : 2; }

__device__ __forceinline__ int band_sign(const int4 bd, int k) {
    const int p1 = (k - bd.x) * (bd.y - k);
    const int p2 = (k - bd.z) * (bd.w - k);
    return ((p1 > p2 ? p1 : p2) >= 0) ? 1 : 0;
}

// tiles of the staged adjoint kernels: 32 x 4 x 4 cells, one thread per cell
namespace adjt {
using namespace tma;
constexpr int BI = 4, BJ = 4, NT = KT * BI * BJ;
}  // namespace adjt

// ---------------------------------------------------------------------------
// transpose of the velocity update: weights
// pairs p: 0 (Vx,Sxx,x) 1 (Vx,Sxy,y) 2 (Vx,Sxz,z) 3 (Vy,Sxy,x) 4 (Vy,Syy,y)
//          5 (Vy,Syz,z) 6 (Vz,Sxz,x) 7 (Vz,Syz,y) 8 (Vz,Szz,z)
// ---------------------------------------------------------------------------
// Operands of one cell: lV(c) the adjoint velocity, b(c) the buoyancy.
struct GAdjVelOps {
    const AdjVelArgs &a;
    long long e;
    __device__ __forceinline__ float lV(int c) const { return a.lV[c][e]; }
    __device__ __forceinline__ float b(int c) const { return a.b[c][e]; }
};

// The stress divergences of the velocity update, d3Sx3 d3Sy3 d3Sz3 of an
// interior cell (m_kernel.f90:103-125) on S(f, dk, di, dj), the forward stress
// after the stress update (f: xx yy zz yz xz xy), with the coefficient pairs
// of band sign s.
template <class F>
__device__ __forceinline__ void stress_divergence(const float (&e40)[3][2], const float (&e41)[3][2], int s, const F &S,
                                                  float (&d)[3]) {
    const float re40x = e40[0][s], re41x = e41[0][s], re40y = e40[1][s], re41y = e41[1][s];
    const float re40z = e40[2][s], re41z = e41[2][s];
    d[0] = (S(0, 0, 1, 0) - S(0, 0, 0, 0)) * re40x - (S(0, 0, 2, 0) - S(0, 0, -1, 0)) * re41x
         + (S(5, 0, 0, 0) - S(5, 0, 0, -1)) * re40y - (S(5, 0, 0, 1) - S(5, 0, 0, -2)) * re41y
         + (S(4, 0, 0, 0) - S(4, -1, 0, 0)) * re40z - (S(4, 1, 0, 0) - S(4, -2, 0, 0)) * re41z;
    d[1] = (S(5, 0, 0, 0) - S(5, 0, -1, 0)) * re40x - (S(5, 0, 1, 0) - S(5, 0, -2, 0)) * re41x
         + (S(1, 0, 0, 1) - S(1, 0, 0, 0)) * re40y - (S(1, 0, 0, 2) - S(1, 0, 0, -1)) * re41y
         + (S(3, 0, 0, 0) - S(3, -1, 0, 0)) * re40z - (S(3, 1, 0, 0) - S(3, -2, 0, 0)) * re41z;
    d[2] = (S(4, 0, 0, 0) - S(4, 0, -1, 0)) * re40x - (S(4, 0, 1, 0) - S(4, 0, -2, 0)) * re41x
         + (S(3, 0, 0, 0) - S(3, 0, 0, -1)) * re40y - (S(3, 0, 0, 1) - S(3, 0, 0, -2)) * re41y
         + (S(2, 1, 0, 0) - S(2, 0, 0, 0)) * re40z - (S(2, 2, 0, 0) - S(2, -1, 0, 0)) * re41z;
}

struct Gb3 {
    float v[3];
};
__device__ __forceinline__ Gb3 gb_load(const AdjVelArgs &a, long long e) {
    Gb3 g;
#pragma unroll
    for (int q = 0; q < 3; q++) g.v[q] = a.gb[q][e];
    return g;
}

// interior (s >= 0: band sign) or absorber (s < 0) cell
template <class O>
__device__ __forceinline__ void adj_vel_cell(const AdjVelArgs &a, const O &o, long long col, int k, int i, int j,
                                             long long e, int s, const Gb3 &g0) {
    const float dt = a.dt;
    const float l[3] = {o.lV(0), o.lV(1), o.lV(2)};
    const float u[3] = {o.b(0) * dt * l[0], o.b(1) * dt * l[1], o.b(2) * dt * l[2]};
    if (s >= 0) {
#pragma unroll
        for (int p = 0; p < 9; p++) {
            const int c = p / 3, ax = p % 3;
            a.w40[p][e] = a.e40[ax][s] * u[c];
            a.w41[p][e] = a.e41[ax][s] * u[c];
        }
        if (a.gb[0]) {
            // d(Vx)/d(bx) = d3Sx3 * dt, the divergences of the forward S after
            // the stress update (formed once per step of the recompute)
#pragma unroll
            const long long es = slot_index(a.sg, k, i, j);
            for (int q = 0; q < 3; q++) a.gb[q][e] = (float)(g0.v[q] + (double)l[q] * __ldcs(a.divS[q] + es) * dt);
        }
        return;
    }
    // absorber cell: V += b * (g.x * D + g.y * aux_old) * dt, aux = g.z * aux + g.w * D * dt
    const int2 pc = __ldg(&a.pmlcol[col]);
    const long long q = (long long)pc.y + (k - pc.x);
    const float4 gp[9] = {__ldg(&a.gxe[i - 1]), __ldg(&a.gyc[j - 1]), __ldg(&a.gzc[k - 1]),
                          __ldg(&a.gxc[i - 1]), __ldg(&a.gye[j - 1]), __ldg(&a.gzc[k - 1]),
                          __ldg(&a.gxc[i - 1]), __ldg(&a.gyc[j - 1]), __ldg(&a.gze[k - 1])};
#pragma unroll
    for (int p = 0; p < 9; p++) {
        const int c = p / 3, ax = p % 3;
        const float la = a.laS[p][q];
        const float lD = u[c] * gp[p].x + gp[p].w * dt * la;
        a.laS[p][q] = gp[p].z * la + u[c] * gp[p].y;
        a.w40[p][e] = a.r20[ax] * lD;
        a.w41[p][e] = 0.0f;
    }
}

__global__ void __launch_bounds__(128) adj_vel_weights_kernel(const AdjVelArgs a) {
    const Geo g = a.g;
    int k, i, j;
    if (!cell_of(g, k, i, j)) return;
    const long long col = col_index(g, i, j);
    const long long e = col * g.Kp + (k - 1 + KH);
    const GAdjVelOps o{a, e};
    const bool interior = i >= a.ibk && i <= a.iek && j >= a.jbk && j <= a.jek && k <= a.kek;
    const int s = interior ? band_sign(__ldg(&a.band[col]), k) : -1;
    const Gb3 g0 = (interior && a.gb[0]) ? gb_load(a, e) : Gb3{};
    adj_vel_cell(a, o, col, k, i, j, e, s, g0);
}

__global__ void mark_cells_kernel(Geo g, const int *cells, int n, unsigned char *mask) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) mask[cell_index(g, cells[3 * q], cells[3 * q + 1], cells[3 * q + 2])] = 1;
}

// transpose of a forward difference (f[e+P] - f[e]) * A40 - (f[e+2P] - f[e-P]) * A41
__device__ __forceinline__ float tfwd(const float *w40, const float *w41, long long f, long long P) {
    return w40[f - P] - w40[f] - w41[f - 2 * P] + w41[f + P];
}
// transpose of a backward difference (f[e] - f[e-P]) * A40 - (f[e+P] - f[e-2P]) * A41
__device__ __forceinline__ float tbwd(const float *w40, const float *w41, long long f, long long P) {
    return w40[f] - w40[f + P] - w41[f - P] + w41[f + 2 * P];
}

// lambda_S += D_S^T weights (dst = lS: xx yy zz yz xz xy)
__global__ void __launch_bounds__(128) adj_vel_gather_kernel(const GatherArgs a) {
    const Geo g = a.g;
    int k, i, j;
    if (!cell_of(g, k, i, j)) return;
    const long long f = cell_index(g, k, i, j);
    const long long PI = g.Kp, PJ = (long long)g.Kp * g.Ip;
    a.dst[0][f] += tfwd(a.w40[0], a.w41[0], f, PI);
    a.dst[1][f] += tfwd(a.w40[4], a.w41[4], f, PJ);
    a.dst[2][f] += tfwd(a.w40[8], a.w41[8], f, 1);
    a.dst[3][f] += tbwd(a.w40[5], a.w41[5], f, 1) + tbwd(a.w40[7], a.w41[7], f, PJ);
    a.dst[4][f] += tbwd(a.w40[2], a.w41[2], f, 1) + tbwd(a.w40[6], a.w41[6], f, PI);
    a.dst[5][f] += tbwd(a.w40[1], a.w41[1], f, PJ) + tbwd(a.w40[3], a.w41[3], f, PI);
}

// ---------------------------------------------------------------------------
// transpose of the stress update: weights
// pairs q: 0 (Vx,x,bwd) 1 (Vy,y,bwd) 2 (Vz,z,bwd) 3 (Vy,x,fwd) 4 (Vx,y,fwd)
//          5 (Vz,x,fwd) 6 (Vx,z,fwd) 7 (Vz,y,fwd) 8 (Vy,z,fwd)
// ---------------------------------------------------------------------------
// Operands of one cell: lS(c) the adjoint stress, lR(q) the adjoint memory
// variable q = component * 3 + m, med(m) the medium (0 mu, 1 lam, 2 taup,
// 3 taus, 4 muyz, 5 muxz, 6 muxy), V(c, dk, di, dj) the forward velocity
// before the stress update.  The one-cell kernel reads them from global
// memory, the staged kernel from the tiles TMA copied to shared memory.
struct GAdjStrOps {
    const AdjStrArgs &a;
    long long e, es, PI, PJ;     // es, PI, PJ: V in the slot layout
    __device__ __forceinline__ float lS(int c) const { return a.lS[c][e]; }
    __device__ __forceinline__ float lR(int q) const { return a.lR[q][e]; }
    __device__ __forceinline__ float med(int m) const {
        const float *p = m == 0 ? a.mu : m == 1 ? a.lam : m == 2 ? a.taup : m == 3 ? a.taus
                       : m == 4 ? a.muyz : m == 5 ? a.muxz : a.muxy;
        return p[e];
    }
    __device__ __forceinline__ float V(int c, int dk, int di, int dj) const {
        return a.V[c][es + dk + di * PI + dj * PJ];
    }
};

// the five imaging accumulators of a cell before this step (read early by
// the staged kernel)
struct Gm5 {
    float v[5];
};
__device__ __forceinline__ Gm5 gm_load(const AdjStrArgs &a, long long e) {
    Gm5 g;
#pragma unroll
    for (int q = 0; q < 5; q++) g.v[q] = a.gm[q][e];
    return g;
}

// interior cell (s: band sign)
template <int NM, class O>
__device__ __forceinline__ void adj_stress_interior(const AdjStrArgs &a, const O &o, int s, long long e, const Gm5 &g0) {
    const float dt = a.dt;
    float al[6];
#pragma unroll
    for (int c = 0; c < 6; c++) al[c] = o.lS(c) * dt;
    const float mu = o.med(0), lam = o.med(1);
    const float taup1 = o.med(2), taus1 = o.med(3);
    const float muc[3] = {o.med(4), o.med(5), o.med(6)};
    const float mu2 = 2 * mu;
    const float lam2mu = lam + mu2;
    const float taup_plus1 = 1 + taup1 * (1 + a.d2);
    const float taus_plus1 = 1 + taus1 * (1 + a.d2);
    // memory variables: R' = c1 R - c2 F dt; S' = S + (G + sum d1 R') dt
    float lF[6];
#pragma unroll
    for (int c = 0; c < 6; c++) {
        lF[c] = 0.0f;
#pragma unroll
        for (int m = 0; m < NM; m++) {
            const float L = o.lR(c * 3 + m) + a.d1[m] * al[c];
            a.lR[c * 3 + m][e] = a.c1[m] * L;
            lF[c] = lF[c] + L * (-a.c2[m] * dt);
        }
    }
    // normal: G_c = lam2mu taup+ d3v3 - mu2 taus+ X_c, F_c likewise with taup, taus
    float ld3 = 0.0f, lX[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        ld3 = ld3 + lam2mu * taup_plus1 * al[c] + lam2mu * taup1 * lF[c];
        lX[c] = -(mu2 * taus_plus1 * al[c] + mu2 * taus1 * lF[c]);
    }
    float ld[9];
    ld[0] = ld3 + lX[1] + lX[2];   // dxVx appears in X_yy and X_zz
    ld[1] = ld3 + lX[0] + lX[2];
    ld[2] = ld3 + lX[0] + lX[1];
    // shear: G = mu_c taus+ D, F = mu_c taus D (c = yz xz xy)
    const float lyz = muc[0] * taus_plus1 * al[3] + muc[0] * taus1 * lF[3];
    const float lxz = muc[1] * taus_plus1 * al[4] + muc[1] * taus1 * lF[4];
    const float lxy = muc[2] * taus_plus1 * al[5] + muc[2] * taus1 * lF[5];
    ld[3] = lxy; ld[4] = lxy; ld[5] = lxz; ld[6] = lxz; ld[7] = lyz; ld[8] = lyz;
#pragma unroll
    for (int q = 0; q < 9; q++) {
        a.w40[q][e] = a.e40[qaxis(q)][s] * ld[q];
        a.w41[q][e] = a.e41[qaxis(q)][s] * ld[q];
    }
    if (a.gm[0]) {
        // forward strain rates on V before the stress update
        const float re40x = a.e40[0][s], re41x = a.e41[0][s], re40y = a.e40[1][s], re41y = a.e41[1][s];
        const float re40z = a.e40[2][s], re41z = a.e41[2][s];
        const float vx0 = o.V(0, 0, 0, 0), vy0 = o.V(1, 0, 0, 0), vz0 = o.V(2, 0, 0, 0);
        const float dxVx = (vx0 - o.V(0, 0, -1, 0)) * re40x - (o.V(0, 0, 1, 0) - o.V(0, 0, -2, 0)) * re41x;
        const float dyVy = (vy0 - o.V(1, 0, 0, -1)) * re40y - (o.V(1, 0, 0, 1) - o.V(1, 0, 0, -2)) * re41y;
        const float dzVz = (vz0 - o.V(2, -1, 0, 0)) * re40z - (o.V(2, 1, 0, 0) - o.V(2, -2, 0, 0)) * re41z;
        const float sxy = (o.V(1, 0, 1, 0) - vy0) * re40x - (o.V(1, 0, 2, 0) - o.V(1, 0, -1, 0)) * re41x
                        + (o.V(0, 0, 0, 1) - vx0) * re40y - (o.V(0, 0, 0, 2) - o.V(0, 0, 0, -1)) * re41y;
        const float sxz = (o.V(2, 0, 1, 0) - vz0) * re40x - (o.V(2, 0, 2, 0) - o.V(2, 0, -1, 0)) * re41x
                        + (o.V(0, 1, 0, 0) - vx0) * re40z - (o.V(0, 2, 0, 0) - o.V(0, -1, 0, 0)) * re41z;
        const float syz = (o.V(2, 0, 0, 1) - vz0) * re40y - (o.V(2, 0, 0, 2) - o.V(2, 0, 0, -1)) * re41y
                        + (o.V(1, 1, 0, 0) - vy0) * re40z - (o.V(1, 2, 0, 0) - o.V(1, -1, 0, 0)) * re41z;
        const double d3 = (double)dxVx + dyVy + dzVz;
        const double X[3] = {(double)dyVy + dzVz, (double)dxVx + dzVz, (double)dxVx + dyVy};
        double glam = 0.0, gmu = 0.0;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            glam += (double)al[c] * taup_plus1 * d3 + (double)lF[c] * taup1 * d3;
            gmu += (double)al[c] * (2.0 * taup_plus1 * d3 - 2.0 * taus_plus1 * X[c])
                 + (double)lF[c] * (2.0 * taup1 * d3 - 2.0 * taus1 * X[c]);
        }
        a.gm[0][e] = (float)(g0.v[0] + glam);
        a.gm[1][e] = (float)(g0.v[1] + gmu);
        a.gm[2][e] = (float)(g0.v[2] + ((double)al[3] * taus_plus1 + (double)lF[3] * taus1) * syz);
        a.gm[3][e] = (float)(g0.v[3] + ((double)al[4] * taus_plus1 + (double)lF[4] * taus1) * sxz);
        a.gm[4][e] = (float)(g0.v[4] + ((double)al[5] * taus_plus1 + (double)lF[5] * taus1) * sxy);
    }
}

// absorber cell (m_absorb_p.f90:445-491)
template <class O>
__device__ __forceinline__ void adj_stress_absorber(const AdjStrArgs &a, const O &o, long long col, int k, int i,
                                                    int j, long long e) {
    const float dt = a.dt;
    float al[6];
#pragma unroll
    for (int c = 0; c < 6; c++) al[c] = o.lS(c) * dt;
    const float mu = o.med(0), lam = o.med(1);
    const int2 pc = __ldg(&a.pmlcol[col]);
    const long long q = (long long)pc.y + (k - pc.x);
    const float4 gxc = __ldg(&a.gxc[i - 1]), gxe = __ldg(&a.gxe[i - 1]);
    const float4 gyc = __ldg(&a.gyc[j - 1]), gye = __ldg(&a.gye[j - 1]);
    const float4 gzc = __ldg(&a.gzc[k - 1]), gze = __ldg(&a.gze[k - 1]);
    const float lam2mu_R = lam + 2 * mu;
    const float lam_R = lam2mu_R - 2 * mu;
    const float lA[3] = {lam2mu_R * al[0] + lam_R * (al[1] + al[2]), lam2mu_R * al[1] + lam_R * (al[0] + al[2]),
                         lam2mu_R * al[2] + lam_R * (al[0] + al[1])};
    float ld[9];
    // normal: D_ade = g.x D + g.y aux, aux' = g.z aux + g.w D dt (aux axVx ayVy azVz = laV 0 4 8)
    {
        const float4 gg[3] = {gxc, gyc, gzc};
        const int ia[3] = {0, 4, 8};
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const float la = a.laV[ia[c]][q];
            ld[c] = gg[c].x * lA[c] + gg[c].w * dt * la;
            a.laV[ia[c]][q] = gg[c].z * la + gg[c].y * lA[c];
        }
    }
    // shear: S' = S + mu_c (g1.x D1 + g2.x D2 + g1.y aux1 + g2.y aux2) dt
    {
        const float byz = o.med(4) * dt * o.lS(3);
        const float bxz = o.med(5) * dt * o.lS(4);
        const float bxy = o.med(6) * dt * o.lS(5);
        // (q, profile, aux index, beta): 3 dxVy gxe axVy; 4 dyVx gye ayVx; 5 dxVz gxe axVz;
        // 6 dzVx gze azVx; 7 dyVz gye ayVz; 8 dzVy gze azVy
        const float4 gg[6] = {gxe, gye, gxe, gze, gye, gze};
        const int ia[6] = {3, 1, 6, 2, 7, 5};
        const float bb[6] = {bxy, bxy, bxz, bxz, byz, byz};
#pragma unroll
        for (int n = 0; n < 6; n++) {
            const float la = a.laV[ia[n]][q];
            ld[3 + n] = gg[n].x * bb[n] + gg[n].w * dt * la;
            a.laV[ia[n]][q] = gg[n].z * la + gg[n].y * bb[n];
        }
    }
#pragma unroll
    for (int qq = 0; qq < 9; qq++) {
        a.w40[qq][e] = a.r20[qaxis(qq)] * ld[qq];
        a.w41[qq][e] = 0.0f;
    }
}

template <int NM>
__global__ void __launch_bounds__(128) adj_stress_weights_kernel(const AdjStrArgs a) {
    const Geo g = a.g;
    int k, i, j;
    if (!cell_of(g, k, i, j)) return;
    const long long col = col_index(g, i, j);
    const long long e = col * g.Kp + (k - 1 + KH);
    const GAdjStrOps o{a, e, slot_index(a.sg, k, i, j), (long long)a.sg.Kp, (long long)a.sg.Kp * a.sg.Ip};
    if (i >= a.ibk && i <= a.iek && j >= a.jbk && j <= a.jek && k <= a.kek) {
        const Gm5 g0 = a.gm[0] ? gm_load(a, e) : Gm5{};
        adj_stress_interior<NM>(a, o, band_sign(__ldg(&a.band[col]), k), e, g0);
    } else {
        adj_stress_absorber(a, o, col, k, i, j, e);
    }
}

// The staged form (see swpc3d_tma.cu for the design): a CTA per tile of
// 32 x 4 x 4 cells whose medium (the context's slab), adjoint S and R (the
// adjoint slab, S alone in tiles without interior cells) and, for the
// gradient, the forward V with its halo (one slot of the recompute) arrive
// by bulk tensor copies; the imaging accumulators and band signs are read
// while the copies travel.
namespace adjt {
template <int NM>
struct Boxes {
    static constexpr int n = NT;
    static constexpr int nMed = 7 * n, nState = (6 + 6 * NM) * n, nV = 3 * (BJ + 4) * (BI + 4) * KB;
    static constexpr int oState = up32(nMed), oV = oState + up32(nState), total = oV + up32(nV);
    __host__ __device__ static constexpr unsigned bytes(bool with_r, bool grad) {
        return 4u * (unsigned)(nMed + (with_r ? nState : 6 * n) + (grad ? nV : 0));
    }
};
template <int NM>
struct SOps {
    const float *sm;
    int tx, ty, tz;
    using L = Boxes<NM>;
    __device__ __forceinline__ int at(int f) const { return ((f * BJ + tz) * BI + ty) * KT + tx; }
    __device__ __forceinline__ float lS(int c) const { return sm[L::oState + at(c)]; }
    __device__ __forceinline__ float lR(int q) const { return sm[L::oState + at(6 + (q / 3) * NM + q % 3)]; }
    // medium box: lam mu taup taus muyz muxz muxy
    __device__ __forceinline__ float med(int m) const { return sm[at(m == 0 ? 1 : m == 1 ? 0 : m)]; }
    __device__ __forceinline__ float V(int c, int dk, int di, int dj) const {
        return sm[L::oV + ((c * (BJ + 4) + tz + 2 + dj) * (BI + 4) + ty + 2 + di) * KB + tx + 4 + dk];
    }
};
}  // namespace adjt

template <int NM, bool GRAD>
__global__ void __launch_bounds__(adjt::NT, (tma::blocks_per_sm<adjt::Boxes<NM>::total, adjt::NT>()))
    adj_stress_tma_kernel(const __grid_constant__ CUtensorMap tm_state, const __grid_constant__ CUtensorMap tm_s,
                          const __grid_constant__ CUtensorMap tm_med, const __grid_constant__ CUtensorMap tm_v,
                          const AdjStrArgs a, const TmaTiles t, int fv) {
    using namespace adjt;
    using L = Boxes<NM>;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ unsigned long long limit;
    float *sm = aligned128(smraw);
    const Geo g = a.g;
    const Tile T = tile_of<1>(t, BI, BJ);
    const int tx = threadIdx.x, ty = threadIdx.y, tz = threadIdx.z;
    const bool with_r = tile_has_interior(T, BI, BJ, a.ibk, a.iek, a.jbk, a.jek, a.kek);
    if (tx == 0 && ty == 0 && tz == 0) {
        // the copies go out first; the error word is read while they travel
        stage_init(&bar, L::bytes(with_r, GRAD));
        const int x0 = T.k0 - 1 + KH;
        load_4d(sm, &tm_med, x0, T.i0 + 2, T.j0 + 2, t.f_med, &bar);
        load_4d(sm + L::oState, with_r ? &tm_state : &tm_s, x0, T.i0 + 2, T.j0 + 2, t.f_state, &bar);
        // V with its halo from the slot: the box starts at cell (k0 - 4, i0 - 2, j0 - 2); tiles of the absorber
        // may reach outside the slot box, where the copy fills zeros that no interior cell reads
        if (GRAD) load_4d(sm + L::oV, &tm_v, x0 - 4, T.i0 - 2 - a.sg.i0, T.j0 - 2 - a.sg.j0, fv, &bar);
        limit = wait_limit(t.err);
    }
    const int k = T.k0 + tx, i = T.i0 + ty, j = T.j0 + tz;
    const bool mine = k <= g.nz && i <= g.nx && j <= g.ny;
    const bool interior = i >= a.ibk && i <= a.iek && j >= a.jbk && j <= a.jek && k <= a.kek;
    const long long col = col_index(g, i, j);
    const long long e = col * g.Kp + (k - 1 + KH);
    const int sgn = (mine && interior) ? band_sign(__ldg(&a.band[col]), k) : 0;
    const Gm5 g0 = (GRAD && mine && interior) ? gm_load(a, e) : Gm5{};
    __syncthreads();   // barrier initialised, wait limit set
    if (!wait_tiles(&bar, t.err, limit) || !mine) return;   // the copy failed, or no cell here
    const SOps<NM> o{sm, tx, ty, tz};
    if (interior) adj_stress_interior<NM>(a, o, sgn, e, g0);
    else adj_stress_absorber(a, o, col, k, i, j, e);
}

// lambda_V += D_V^T weights (dst = lV: x y z)
__global__ void __launch_bounds__(128) adj_stress_gather_kernel(const GatherArgs a) {
    const Geo g = a.g;
    int k, i, j;
    if (!cell_of(g, k, i, j)) return;
    const long long f = cell_index(g, k, i, j);
    const long long PI = g.Kp, PJ = (long long)g.Kp * g.Ip;
    a.dst[0][f] += tbwd(a.w40[0], a.w41[0], f, PI) + tfwd(a.w40[4], a.w41[4], f, PJ) + tfwd(a.w40[6], a.w41[6], f, 1);
    a.dst[1][f] += tbwd(a.w40[1], a.w41[1], f, PJ) + tfwd(a.w40[3], a.w41[3], f, PI) + tfwd(a.w40[8], a.w41[8], f, 1);
    a.dst[2][f] += tbwd(a.w40[2], a.w41[2], f, 1) + tfwd(a.w40[5], a.w41[5], f, PI) + tfwd(a.w40[7], a.w41[7], f, PJ);
}

// Operands of the fused kernel below: lambda_V from registers, b from memory.
struct RAdjVelOps {
    const AdjVelArgs &a;
    long long e;
    float l[3];
    __device__ __forceinline__ float lV(int c) const { return l[c]; }
    __device__ __forceinline__ float b(int c) const { return a.b[c][e]; }
};

// lambda_V += D_V^T weights as adj_stress_gather_kernel, then, from the new
// lambda_V of the cell, the velocity-phase weights of the next adjoint step
// (the cell-local transpose of the velocity update, adj_vel_cell), so that
// lambda_V is read once for both and the weights need no launch of their
// own.  Cells of `mask` (when given: a step whose receiver residuals still
// change their lambda_V) leave their weights to adj_source_cells_kernel.
__global__ void __launch_bounds__(128) adj_stress_gather_vel_kernel(const GatherArgs a, const AdjVelArgs v,
                                                                     const unsigned char *mask) {
    const Geo g = a.g;
    int k, i, j;
    if (!cell_of(g, k, i, j)) return;
    const long long f = cell_index(g, k, i, j);
    const long long PI = g.Kp, PJ = (long long)g.Kp * g.Ip;
    const float l0 = a.dst[0][f] + (tbwd(a.w40[0], a.w41[0], f, PI) + tfwd(a.w40[4], a.w41[4], f, PJ) +
                                    tfwd(a.w40[6], a.w41[6], f, 1));
    const float l1 = a.dst[1][f] + (tbwd(a.w40[1], a.w41[1], f, PJ) + tfwd(a.w40[3], a.w41[3], f, PI) +
                                    tfwd(a.w40[8], a.w41[8], f, 1));
    const float l2 = a.dst[2][f] + (tbwd(a.w40[2], a.w41[2], f, 1) + tfwd(a.w40[5], a.w41[5], f, PI) +
                                    tfwd(a.w40[7], a.w41[7], f, PJ));
    a.dst[0][f] = l0;
    a.dst[1][f] = l1;
    a.dst[2][f] = l2;
    if (mask && mask[f]) return;
    const long long col = col_index(g, i, j);
    const bool interior = i >= v.ibk && i <= v.iek && j >= v.jbk && j <= v.jek && k <= v.kek;
    const int s = interior ? band_sign(__ldg(&v.band[col]), k) : -1;
    const Gb3 g0 = (interior && v.gb[0]) ? gb_load(v, f) : Gb3{};
    const RAdjVelOps o{v, f, {l0, l1, l2}};
    adj_vel_cell(v, o, col, k, i, j, f, s, g0);
}

// transpose of the velocity recorder (m_wav.f90:530-535): residuals as
// sources.  A recorder averages two cells per component (Vx at i and i-1, Vy
// at j and j-1, Vz at k and k-1, the latter with the sign of an upward z), so
// its residual r enters both; one thread per receiving cell adds the
// residuals of its stations in station order (cells that several stations
// share get the same bits in every run).  With WEIGHTS the thread then forms
// the velocity-phase weights of the next adjoint step for its cell from the
// new lambda_V (the cells the fused gather left out).
struct SrcArgs {
    Geo g;
    const int *cells;       // (k, i, j) per receiving cell
    const int *offs;        // n + 1 offsets into contrib
    const int *contrib;     // station << 2 | component
    int n, ntw, itw;
    const float *res;
    float scale;
    float *lV[3];
};

template <bool WEIGHTS>
__global__ void __launch_bounds__(128) adj_source_cells_kernel(const SrcArgs a, const AdjVelArgs v) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.n) return;
    const Geo g = a.g;
    const int k = a.cells[3 * q], i = a.cells[3 * q + 1], j = a.cells[3 * q + 2];
    const long long e = cell_index(g, k, i, j);
    float l[3] = {a.lV[0][e], a.lV[1][e], a.lV[2][e]};
    for (int t = a.offs[q]; t < a.offs[q + 1]; t++) {
        const int w = a.contrib[t], n = w >> 2, c = w & 3;
        const float r = a.res[((long long)n * 3 + c) * a.ntw + a.itw - 1] * a.scale;
        l[c] = l[c] + (c == 2 ? -r : r);
    }
#pragma unroll
    for (int c = 0; c < 3; c++) a.lV[c][e] = l[c];
    if (!WEIGHTS || k < 1 || k > g.nz || i < 1 || i > g.nx || j < 1 || j > g.ny) return;
    const long long col = col_index(g, i, j);
    const bool interior = i >= v.ibk && i <= v.iek && j >= v.jbk && j <= v.jek && k <= v.kek;
    const int s = interior ? band_sign(__ldg(&v.band[col]), k) : -1;
    const Gb3 g0 = (interior && v.gb[0]) ? gb_load(v, e) : Gb3{};
    const RAdjVelOps o{v, e, {l[0], l[1], l[2]}};
    adj_vel_cell(v, o, col, k, i, j, e, s, g0);
}

__global__ void zero_double_kernel(double *p, long long n) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        p[q] = 0.0;
}

// one slot of the recompute: the stress divergences of the interior cells,
// on the forward S just after the stress update of that step
struct SlotDivArgs {
    Geo g;
    int ibk, iek, jbk, jek, kek;
    const float *S[6];
    const int4 *band;
    float e40[3][2], e41[3][2];
    float *divS[3];              // slot layout
    SlotGeo sg;
};
__global__ void __launch_bounds__(128) slot_div_kernel(const SlotDivArgs a) {
    const Geo g = a.g;
    int k, i, j;
    if (!cell_of(g, k, i, j)) return;
    if (!(i >= a.ibk && i <= a.iek && j >= a.jbk && j <= a.jek && k <= a.kek)) return;
    const long long col = col_index(g, i, j);
    const long long e = col * g.Kp + (k - 1 + KH);
    const long long PI = g.Kp, PJ = (long long)g.Kp * g.Ip;
    const auto S = [&](int f, int dk, int di, int dj) { return a.S[f][e + dk + di * PI + dj * PJ]; };
    float d[3];
    stress_divergence(a.e40, a.e41, band_sign(__ldg(&a.band[col]), k), S, d);
#pragma unroll
    const long long es = slot_index(a.sg, k, i, j);
#pragma unroll
    for (int q = 0; q < 3; q++) __stcs(a.divS[q] + es, d[q]);
}

// V over the slot box into a slot (float4 along k: both pitches are multiples
// of 8 floats and the slot's k extent is not larger than the memory box's)
__global__ void slot_v_kernel(Geo g, SlotGeo sg, const float *vx, const float *vy, const float *vz, float *dst) {
    const int k4 = sg.Kp / 4;
    const long long per = (long long)sg.Jp * sg.Ip * k4;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 3 * per;
         t += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(t / per);
        const long long r = t - c * per;
        const int kq = (int)(r % k4);
        const long long colq = r / k4;
        const int is = (int)(colq % sg.Ip), js = (int)(colq / sg.Ip);
        const float *src = c == 0 ? vx : c == 1 ? vy : vz;
        const long long from = col_index(g, is + sg.i0, js + sg.j0) * g.Kp + 4LL * kq;
        const long long to = (long long)c * sg.n + colq * sg.Kp + 4LL * kq;
        __stcs(reinterpret_cast<float4 *>(dst + to), __ldcs(reinterpret_cast<const float4 *>(src + from)));
    }
}

// V of the shell cells of the slot box (slot-box indices `shell`) into a kept
// step: dst[c * n + q] = V_c at shell cell q
__global__ void shell_save_kernel(Geo g, SlotGeo sg, const float *vx, const float *vy, const float *vz,
                                  const int *shell, int n, float *dst) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 3LL * n;
         t += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(t / n), q = (int)(t - (long long)c * n);
        const long long es = shell[q];
        const int kd = (int)(es % sg.Kp);
        const long long cs = es / sg.Kp;
        const int is = (int)(cs % sg.Ip), js = (int)(cs / sg.Ip);
        const float *src = c == 0 ? vx : c == 1 ? vy : vz;
        dst[t] = src[col_index(g, is + sg.i0, js + sg.j0) * g.Kp + kd];
    }
}

// the shell values of kept steps 1..len into the V of slots 1..len (slot
// stride sstride floats, kept-step stride kstride floats)
__global__ void shell_load_kernel(const float *keep1, size_t kstride, const int *shell, int n, int len, long long ns,
                                  float *slot1, size_t sstride) {
    const long long per = 3LL * n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < per * len;
         t += (long long)gridDim.x * blockDim.x) {
        const int m = (int)(t / per);
        const long long r = t - m * per;
        const int c = (int)(r / n), q = (int)(r - (long long)c * n);
        slot1[m * sstride + c * ns + shell[q]] = keep1[m * kstride + r];
    }
}

// V of the interior cells through a kept segment: the velocity update of an
// interior cell is V + b * d * dt with d its stress divergence
// (kernel__update_vel, m_kernel.f90:103-125, the expression of vel_interior),
// so from V of slot 0 and the kept divergences d(1..len) the V of slots
// 1..len follow with the update's own rounding
struct ReconArgs {
    Geo g;
    SlotGeo sg;
    int ibk, iek, jbk, jek, kek, len;
    const float *b[3];
    float dt;
    const float *div1;      // divergences of kept step 1 (field c at div1 + c * sg.n)
    size_t kstride;         // floats between kept steps
    float *slot0;           // V of slot 0 (field c at slot0 + c * sg.n), slots every sstride floats
    size_t sstride;
};
__global__ void recon_kernel(const ReconArgs a) {
    const int ni = a.iek - a.ibk + 1, nj = a.jek - a.jbk + 1;
    const long long n = (long long)a.kek * ni * nj;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = 1 + (int)(t % a.kek);
        const long long r = t / a.kek;
        const int i = a.ibk + (int)(r % ni), j = a.jbk + (int)(r / ni);
        const long long es = slot_index(a.sg, k, i, j), e = cell_index(a.g, k, i, j);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const float b = a.b[c][e], dt = a.dt;
            float v = a.slot0[c * a.sg.n + es];
            for (int m = 1; m <= a.len; m++) {
                const float d = __ldcs(a.div1 + (m - 1) * a.kstride + c * a.sg.n + es);
                v = v + b * d * dt;
                __stcs(a.slot0 + m * a.sstride + c * a.sg.n + es, v);
            }
        }
    }
}

// the segment's FP32 partial sums into the FP64 totals; the partials restart from zero
struct FoldArgs {
    double *total[8];
    float *part[8];
};
__global__ void fold_gradient_kernel(const FoldArgs a, long long n) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int f = 0; f < 8; f++) {
            a.total[f][q] += (double)a.part[f][q];
            a.part[f][q] = 0.0f;
        }
    }
}

// ---------------------------------------------------------------------------
// chain rule from the medium arrays to per-cell vp, vs, rho (Q fixed)
//
// The medium of a cell follows from its vp, vs, rho as vmodel_lhm, then
// relaxed_medium and averaged_medium compute it (m_vmodel_lhm.f90:158-160,
// m_medium.f90:234-274, 432-465):
//   mu  = rho vs^2 / chi_s^2,   lam + 2 mu = rho vp^2 / chi_p^2,
// with chi fixed by Q, so d mu/d vs = 2 mu/vs, d mu/d rho = mu/rho and the
// same for lam + 2 mu; b_x(e) = 2/(rho(e) + rho(e+i)) (d/d rho = -b^2/2 for
// both cells); mu_xz(e) = 4 abcd/(abc + abd + acd + bcd + eps) over the four
// cells (e, e+k, e+i, e+k+i), and likewise mu_xy (i, j) and mu_yz (k, j).
// ---------------------------------------------------------------------------
struct ModelGradArgs {
    Geo g;
    const double *gm[8];           // lam mu muyz muxz muxy bx by bz
    const float *lam, *mu, *b[3];  // relaxed medium, buoyancies
    const float *vp, *vs, *rho;    // the model (device layout)
    double *out[3];                // d misfit / d vp, vs, rho
};

// sum over the four entries of a 4-point harmonic mean that contain cell e
// (entry E averages E, E+o1, E+o2, E+o1+o2) of g(E) * d mean(E) / d mu(e)
__device__ double hmean_adjoint(const double *gf, const float *mu, long long e, long long o1, long long o2) {
    const long long offs[4] = {0, o1, o2, o1 + o2};
    double acc = 0.0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const long long E = e - offs[q];
        const double gE = gf[E];
        if (gE == 0.0) continue;
        double m[4];
#pragma unroll
        for (int r = 0; r < 4; r++) m[r] = (double)mu[E + offs[r]];
        // the three values other than the one at e (position q)
        double o[3];
        int n = 0;
#pragma unroll
        for (int r = 0; r < 4; r++)
            if (r != q) o[n++] = m[r];
        const double x = m[q];
        const double p3 = o[0] * o[1] * o[2];
        const double s2 = o[0] * o[1] + o[0] * o[2] + o[1] * o[2];
        const double D = x * s2 + p3 + (double)1.1920929e-07f;
        const double N = 4.0 * x * p3;
        acc += gE * (4.0 * p3 * D - N * s2) / (D * D);
    }
    return acc;
}

__global__ void __launch_bounds__(128) model_grad_kernel(const ModelGradArgs a) {
    const Geo g = a.g;
    int k, i, j;
    if (!cell_of(g, k, i, j)) return;
    const long long e = cell_index(g, k, i, j);
    const long long PI = g.Kp, PJ = (long long)g.Kp * g.Ip;
    const double glam = a.gm[0][e];
    const double gmu = a.gm[1][e] + hmean_adjoint(a.gm[2], a.mu, e, 1, PJ) + hmean_adjoint(a.gm[3], a.mu, e, 1, PI) +
                       hmean_adjoint(a.gm[4], a.mu, e, PI, PJ);
    double grho = 0.0;
    const long long boff[3] = {PI, PJ, 1};
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const double b0 = a.b[q][e], b1 = a.b[q][e - boff[q]];
        grho += a.gm[5 + q][e] * (-0.5 * b0 * b0) + a.gm[5 + q][e - boff[q]] * (-0.5 * b1 * b1);
    }
    const double lam = a.lam[e], mu = a.mu[e];
    const double vp = a.vp[e], vs = a.vs[e], rho = a.rho[e];
    const double m2 = lam + 2.0 * mu;
    a.out[0][e] = vp > 0.0 ? glam * 2.0 * m2 / vp : 0.0;
    a.out[1][e] = vs > 0.0 ? (gmu - 2.0 * glam) * 2.0 * mu / vs : 0.0;
    a.out[2][e] = grho + (rho > 0.0 ? (glam * lam + gmu * mu) / rho : 0.0);
}

dim3 cell_grid(const Geo &g, dim3 block) {
    return dim3((g.nz + kThreadsK - 1) / kThreadsK, (g.nx + block.y - 1) / block.y, (g.ny + block.z - 1) / block.z);
}

int err(swpc_ctx *c, int code, const char *m) { return set_err(c, code, m); }

}  // namespace

#define ACK(call)                                            \
    do {                                                     \
        int _rc = cuda_check(c, (call), #call);              \
        if (_rc) return _rc;                                 \
    } while (0)

static int adj_alloc(swpc_ctx *c) {
    if (c->adj) return SWPC_OK;
    auto *s = new swpc_adj_state();
    c->adj = s;
    const long long n = c->g.ncell;
    // adjoint state slab: 0-2 lV, 3-8 lS, 9.. lR (component-major), as the forward slab
    s->slab_nf = 9 + 6 * c->d.nm;
    {
        int rc = dalloc(c, &s->slab, (size_t)s->slab_nf * n);
        if (rc) return rc;
    }
    for (int q = 0; q < 3; q++) s->lV[q] = s->slab + (size_t)q * n;
    for (int q = 0; q < 6; q++) s->lS[q] = s->slab + (size_t)(3 + q) * n;
    for (int comp = 0; comp < 6; comp++)
        for (int m = 0; m < c->d.nm; m++) s->lR[comp * 3 + m] = s->slab + (size_t)(9 + comp * c->d.nm + m) * n;
    s->maps = new TmaMaps();
    const TmaSlabs sl{s->slab, s->slab_nf, c->slab, c->slab_nf, nullptr, 0};
    if (!tma_encode_stress(*s->maps, sl, c->g, c->d.nm, adjt::BI, adjt::BJ))
        return set_err(c, SWPC_ERR_CUDA, "cuTensorMapEncodeTiled failed for the adjoint slab");
    if (c->npml > 0)
        for (int q = 0; q < 18; q++) { int rc = dalloc(c, &s->laux[q], c->npml); if (rc) return rc; }
    for (int q = 0; q < 9; q++) {
        int rc = dalloc(c, &s->w40[q], n);
        if (!rc) rc = dalloc(c, &s->w41[q], n);
        if (!rc) rc = dalloc(c, &s->w40v[q], n);
        if (!rc) rc = dalloc(c, &s->w41v[q], n);
        if (rc) return rc;
    }
    for (int q = 0; q < 8; q++) { int rc = dalloc(c, &s->grad[q], n); if (rc) return rc; }
    for (int q = 0; q < 8; q++) { int rc = dalloc(c, &s->gpart[q], n); if (rc) return rc; }
    return SWPC_OK;
}

namespace swpc {
void adj_free(swpc_ctx *c) {
    swpc_adj_state *s = c->adj;
    if (!s) return;
    if (s->slab) cudaFree(s->slab);   // lV, lS, lR
    delete s->maps;
    for (auto p : s->laux) if (p) cudaFree(p);
    for (auto p : s->w40) if (p) cudaFree(p);
    for (auto p : s->w41) if (p) cudaFree(p);
    for (auto p : s->w40v) if (p) cudaFree(p);
    for (auto p : s->w41v) if (p) cudaFree(p);
    if (s->srcmask) cudaFree(s->srcmask);
    if (s->srccells) cudaFree(s->srccells);
    for (auto p : s->grad) if (p) cudaFree(p);
    for (auto p : s->gpart) if (p) cudaFree(p);
    if (s->res) cudaFree(s->res);
    if (s->ckpool) cudaFree(s->ckpool);
    if (s->slots) cudaFree(s->slots);
    if (s->keep) cudaFree(s->keep);
    if (s->shell) cudaFree(s->shell);
    delete s;
    c->adj = nullptr;
}
}  // namespace swpc

static int adj_ready(swpc_ctx *c) {
    if (!c) return SWPC_ERR_ARG;
    if (c->kind != SWPC_KIND_3D) return err(c, SWPC_ERR_ARG, "the adjoint is implemented for the 3D solver");
    if (c->prec != SWPC_PREC_F32) return err(c, SWPC_ERR_ARG, "the adjoint needs FP32 storage");
    if (c->abc != 0) return err(c, SWPC_ERR_STATE, "the adjoint is implemented for the PML (not the Cerjan sponge)");
    if (c->pw_mode) return err(c, SWPC_ERR_STATE, "the adjoint is not implemented for the plane-wave mode");
    if (!c->medium_ready || !c->kernel_ready || (c->d.na > 0 && !c->absorb_ready))
        return err(c, SWPC_ERR_STATE, "medium, kernel and absorber setup must precede the adjoint");
    ACK(cudaSetDevice(c->device));
    return adj_alloc(c);
}

// staged stress-phase weights over the whole grid; fv: field of the forward V
// in the slots buffer (gradient), or -1
template <int NM>
static cudaError_t adj_stress_tma(const swpc_adj_state *s, const AdjStrArgs &a, const TmaTiles &t, int fv,
                                  cudaStream_t st) {
    constexpr int bytes = adjt::Boxes<NM>::total * 4 + 128;
    static unsigned long long devices = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(devices >> dev & 1ull)) {
        cudaError_t e0 = cudaFuncSetAttribute(adj_stress_tma_kernel<NM, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e0 == cudaSuccess)
            e0 = cudaFuncSetAttribute(adj_stress_tma_kernel<NM, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e0 != cudaSuccess) return e0;
        devices |= 1ull << dev;
    }
    const TmaMaps &m = *s->maps;
    auto map = [](const unsigned char *p) -> const CUtensorMap & { return *reinterpret_cast<const CUtensorMap *>(p); };
    const unsigned nblk = (unsigned)((long long)t.nkt * t.nit * t.njt);
    const dim3 block(tma::KT, adjt::BI, adjt::BJ);
    if (fv >= 0)
        adj_stress_tma_kernel<NM, true><<<nblk, block, bytes, st>>>(map(m.state), map(m.s6), map(m.med), map(m.vh), a, t, fv);
    else
        adj_stress_tma_kernel<NM, false><<<nblk, block, bytes, st>>>(map(m.state), map(m.s6), map(m.med), map(m.vh), a, t, 0);
    return cudaGetLastError();
}

static SlotGeo slot_geo(const swpc_ctx *c) {
    SlotGeo sg;
    sg.i0 = c->ibk - 2;
    sg.j0 = c->jbk - 2;
    sg.Ip = c->iek - c->ibk + 5;
    sg.Jp = c->jek - c->jbk + 5;
    sg.Kp = ((c->kek + 3 + KH) + 7) / 8 * 8;
    sg.n = (long long)sg.Kp * sg.Ip * sg.Jp;
    return sg;
}

// Arguments of the velocity-phase weights: from lambda_V into the
// velocity-phase weight arrays, with the gradient of b when divS (the forward
// stress divergences of that step) is given.
static AdjVelArgs vel_args(swpc_ctx *c, const float *const *divS) {
    swpc_adj_state *s = c->adj;
    AdjVelArgs a;
    memset(&a, 0, sizeof(a));
    a.g = c->g; a.ibk = c->ibk; a.iek = c->iek; a.jbk = c->jbk; a.jek = c->jek; a.kek = c->kek;
    for (int q = 0; q < 3; q++) { a.lV[q] = s->lV[q]; a.b[q] = c->med[5 + q]; }
    a.band = c->band; a.pmlcol = c->pmlcol;
    for (int q = 0; q < 9; q++) a.laS[q] = s->laux[9 + q];
    a.gxc = c->gx[0]; a.gxe = c->gx[1]; a.gyc = c->gy[0]; a.gye = c->gy[1]; a.gzc = c->gz[0]; a.gze = c->gz[1];
    memcpy(a.e40, c->e40, sizeof(a.e40)); memcpy(a.e41, c->e41, sizeof(a.e41)); memcpy(a.r20, c->r20, sizeof(a.r20));
    a.dt = c->d.dt;
    a.sg = slot_geo(c);
    for (int q = 0; q < 9; q++) { a.w40[q] = s->w40v[q]; a.w41[q] = s->w41v[q]; }
    if (divS) {
        for (int q = 0; q < 3; q++) a.divS[q] = divS[q];
        for (int q = 0; q < 3; q++) a.gb[q] = s->gpart[5 + q];
    }
    return a;
}

// What the stress-phase gather of a step also does: form the velocity-phase
// weights of the next adjoint step (on = true), with that step's forward
// stress divergences divS (gradient) and leaving the cells that receiver
// residuals change this step to the injection (skip_src).
struct AdjNext {
    bool on = false, skip_src = false;
    const float *const *divS = nullptr;
};

// one transposed step: vel^T then stress^T; with gradient when S_after /
// V_before are given (for the staged stress-phase weights, V_before is field
// fv of the slots buffer); vel_done: the velocity-phase weights were formed
// by the previous step's stress-phase gather
static int adj_step(swpc_ctx *c, const float *const *divS_after, const float *const *V_before, int fv,
                    bool vel_done = false, const AdjNext &next = AdjNext()) {
    swpc_adj_state *s = c->adj;
    const dim3 block(kThreadsK, 2, 2);
    const dim3 grid = cell_grid(c->g, block);
    const bool grad = divS_after != nullptr;
    {
        if (!vel_done) {
            // one cell per thread: the kernel is bound by its 18 weight stores, and
            // staging its few loads (a TMA-staged form was tried) made it slower
            adj_vel_weights_kernel<<<grid, block, 0, c->stream>>>(vel_args(c, grad ? divS_after : nullptr));
            ACK(cudaGetLastError());
        }
        GatherArgs ga;
        ga.g = c->g;
        for (int q = 0; q < 6; q++) ga.dst[q] = s->lS[q];
        for (int q = 0; q < 9; q++) { ga.w40[q] = s->w40v[q]; ga.w41[q] = s->w41v[q]; }
        adj_vel_gather_kernel<<<grid, block, 0, c->stream>>>(ga);
        ACK(cudaGetLastError());
    }
    {
        AdjStrArgs a;
        memset(&a, 0, sizeof(a));
        a.g = c->g; a.ibk = c->ibk; a.iek = c->iek; a.jbk = c->jbk; a.jek = c->jek; a.kek = c->kek; a.nm = c->d.nm;
        for (int q = 0; q < 6; q++) a.lS[q] = s->lS[q];
        for (int q = 0; q < 18; q++) a.lR[q] = s->lR[q];
        a.lam = c->med[1]; a.mu = c->med[2]; a.taup = c->med[3]; a.taus = c->med[4];
        a.muyz = c->med[8]; a.muxz = c->med[9]; a.muxy = c->med[10];
        a.band = c->band; a.pmlcol = c->pmlcol;
        for (int q = 0; q < 9; q++) a.laV[q] = s->laux[q];
        a.gxc = c->gx[0]; a.gxe = c->gx[1]; a.gyc = c->gy[0]; a.gye = c->gy[1]; a.gzc = c->gz[0]; a.gze = c->gz[1];
        memcpy(a.e40, c->e40, sizeof(a.e40)); memcpy(a.e41, c->e41, sizeof(a.e41)); memcpy(a.r20, c->r20, sizeof(a.r20));
        a.dt = c->d.dt;
        memcpy(a.c1, c->c1, sizeof(a.c1)); memcpy(a.c2, c->c2, sizeof(a.c2)); memcpy(a.d1, c->d1, sizeof(a.d1));
        a.d2 = c->d2;
        a.sg = slot_geo(c);
        for (int q = 0; q < 9; q++) { a.w40[q] = s->w40[q]; a.w41[q] = s->w41[q]; }
        if (grad) {
            for (int q = 0; q < 3; q++) a.V[q] = V_before[q];
            for (int q = 0; q < 5; q++) a.gm[q] = s->gpart[q];
        }
        if (c->adj_tma && (!grad || fv >= 0)) {
            const TmaTiles t = tma_tiles(c, adjt::BI, adjt::BJ, 1, 1, kStressFields(c), 1);
            const int f = grad ? fv : -1;
            switch (c->d.nm) {
            case 0: ACK(adj_stress_tma<0>(s, a, t, f, c->stream)); break;
            case 1: ACK(adj_stress_tma<1>(s, a, t, f, c->stream)); break;
            case 2: ACK(adj_stress_tma<2>(s, a, t, f, c->stream)); break;
            default: ACK(adj_stress_tma<3>(s, a, t, f, c->stream)); break;
            }
        } else {
            switch (c->d.nm) {
            case 0: adj_stress_weights_kernel<0><<<grid, block, 0, c->stream>>>(a); break;
            case 1: adj_stress_weights_kernel<1><<<grid, block, 0, c->stream>>>(a); break;
            case 2: adj_stress_weights_kernel<2><<<grid, block, 0, c->stream>>>(a); break;
            default: adj_stress_weights_kernel<3><<<grid, block, 0, c->stream>>>(a); break;
            }
            ACK(cudaGetLastError());
        }
        GatherArgs ga;
        ga.g = c->g;
        for (int q = 0; q < 3; q++) ga.dst[q] = s->lV[q];
        for (int q = 3; q < 6; q++) ga.dst[q] = nullptr;
        for (int q = 0; q < 9; q++) { ga.w40[q] = s->w40[q]; ga.w41[q] = s->w41[q]; }
        if (next.on)
            adj_stress_gather_vel_kernel<<<grid, block, 0, c->stream>>>(ga, vel_args(c, next.divS),
                                                                         next.skip_src ? s->srcmask : nullptr);
        else
            adj_stress_gather_kernel<<<grid, block, 0, c->stream>>>(ga);
        ACK(cudaGetLastError());
    }
    return SWPC_OK;
}

// whether adj_source injects receiver residuals at step it
static bool source_at(const swpc_ctx *c, int it) {
    const swpc_adj_state *s = c->adj;
    if (!s->res || c->nst <= 0 || !(c->wav_what & SWPC_WAV_V)) return false;
    if ((it - 1) % c->ntdec_w != 0) return false;
    return (it - 1) / c->ntdec_w + 1 <= c->ntw;
}

// residuals of step it into lambda_V; with divS_next (the fused path) the
// receiving cells also form the velocity-phase weights of step it - 1
static int adj_source(swpc_ctx *c, int it, const float *const *divS_next = nullptr, bool weights = false) {
    swpc_adj_state *s = c->adj;
    if (!source_at(c, it) || s->nsrc <= 0) return SWPC_OK;
    SrcArgs a;
    a.g = c->g;
    a.cells = s->srccells;
    a.offs = s->srccells + 3 * s->nsrc;
    a.contrib = a.offs + s->nsrc + 1;
    a.n = s->nsrc;
    a.ntw = c->ntw;
    a.itw = (it - 1) / c->ntdec_w + 1;
    a.res = s->res;
    // d(trace)/dV = 0.5 M0 UC 1e9 per cell of the two-cell average
    a.scale = 0.5f * c->M0 * c->UC * 1e9f;
    for (int q = 0; q < 3; q++) a.lV[q] = s->lV[q];
    const unsigned nb = (unsigned)((s->nsrc + 127) / 128);
    if (weights) adj_source_cells_kernel<true><<<nb, 128, 0, c->stream>>>(a, vel_args(c, divS_next));
    else adj_source_cells_kernel<false><<<nb, 128, 0, c->stream>>>(a, AdjVelArgs{});
    return cuda_check(c, cudaGetLastError(), "adj_source_cells_kernel");
}

// The cells whose lambda_V adj_source changes (both cells of each recorder's
// two-cell averages, inside the memory box or not), with the residuals each
// receives in station order, and the mask of those cells.
static int source_cells(swpc_ctx *c) {
    swpc_adj_state *s = c->adj;
    const Geo &g = c->g;
    std::vector<int> st(3 * (size_t)std::max(c->nst, 0));
    if (c->nst > 0) {
        ACK(cudaMemcpyAsync(st.data(), c->st_ijk, st.size() * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        ACK(cudaStreamSynchronize(c->stream));
    }
    struct Contrib { long long e; int k, i, j, n, cmp; };
    std::vector<Contrib> all;
    for (int n = 0; n < c->nst; n++) {
        const int i = st[3 * n], j = st[3 * n + 1], k = st[3 * n + 2];
        const int nb[6][4] = {{k, i, j, 0}, {k, i - 1, j, 0}, {k, i, j, 1}, {k, i, j - 1, 1}, {k, i, j, 2},
                              {k - 1, i, j, 2}};
        for (auto &q : nb) all.push_back({cell_index(g, q[0], q[1], q[2]), q[0], q[1], q[2], n, q[3]});
    }
    // by cell, then station: the order of each cell's sums
    std::stable_sort(all.begin(), all.end(), [](const Contrib &a, const Contrib &b) {
        return a.e != b.e ? a.e < b.e : a.n < b.n;
    });
    std::vector<int> cells, offs, contrib;
    for (size_t t = 0; t < all.size(); t++) {
        if (t == 0 || all[t].e != all[t - 1].e) {
            cells.insert(cells.end(), {all[t].k, all[t].i, all[t].j});
            offs.push_back((int)t);
        }
        contrib.push_back(all[t].n << 2 | all[t].cmp);
    }
    offs.push_back((int)all.size());
    const int ncell = (int)cells.size() / 3;
    std::vector<int> packed(cells);
    packed.insert(packed.end(), offs.begin(), offs.end());
    packed.insert(packed.end(), contrib.begin(), contrib.end());
    if (s->srccells) { cudaFree(s->srccells); s->srccells = nullptr; }
    s->nsrc = s->nsrc_contrib = 0;
    if (!s->srcmask && cudaMalloc((void **)&s->srcmask, (size_t)g.ncell) != cudaSuccess) {
        cudaGetLastError();
        s->srcmask = nullptr;
        return err(c, SWPC_ERR_NOMEM, "no room for the receiver cell mask");
    }
    ACK(cudaMemsetAsync(s->srcmask, 0, (size_t)g.ncell, c->stream));
    if (ncell > 0) {
        ACK(cudaMalloc((void **)&s->srccells, packed.size() * sizeof(int)));
        ACK(cudaMemcpyAsync(s->srccells, packed.data(), packed.size() * sizeof(int), cudaMemcpyHostToDevice,
                            c->stream));
        s->nsrc = ncell;
        s->nsrc_contrib = (int)contrib.size();
        mark_cells_kernel<<<(ncell + 127) / 128, 128, 0, c->stream>>>(g, s->srccells, ncell, s->srcmask);
        ACK(cudaGetLastError());
        ACK(cudaStreamSynchronize(c->stream));   // the host list goes out of scope
    }
    return SWPC_OK;
}

static int zero_adjoint(swpc_ctx *c) {
    swpc_adj_state *s = c->adj;
    const size_t n = sizeof(float) * c->g.ncell;
    for (auto p : s->lV) if (p) ACK(cudaMemsetAsync(p, 0, n, c->stream));
    for (auto p : s->lS) if (p) ACK(cudaMemsetAsync(p, 0, n, c->stream));
    for (auto p : s->lR) if (p) ACK(cudaMemsetAsync(p, 0, n, c->stream));
    for (auto p : s->laux) if (p) ACK(cudaMemsetAsync(p, 0, sizeof(float) * c->npml, c->stream));
    for (auto p : s->grad) {
        zero_double_kernel<<<148 * 4, 256, 0, c->stream>>>(p, c->g.ncell);
        ACK(cudaGetLastError());
    }
    for (auto p : s->gpart) ACK(cudaMemsetAsync(p, 0, n, c->stream));
    return SWPC_OK;
}

static int fold_gradient(swpc_ctx *c) {
    FoldArgs a;
    for (int q = 0; q < 8; q++) { a.total[q] = c->adj->grad[q]; a.part[q] = c->adj->gpart[q]; }
    fold_gradient_kernel<<<148 * 4, 256, 0, c->stream>>>(a, c->g.ncell);
    return cuda_check(c, cudaGetLastError(), "fold_gradient_kernel");
}

// the adjoint array of a field id (V, S, R, PML auxiliaries)
static float *adj_field(swpc_ctx *c, int field, bool *compact) {
    swpc_adj_state *s = c->adj;
    *compact = false;
    if (field >= SWPC_F_VX && field <= SWPC_F_VZ) return s->lV[field - SWPC_F_VX];
    if (field >= SWPC_F_SXX && field <= SWPC_F_SXY) return s->lS[field - SWPC_F_SXX];
    if (field >= SWPC_F_R && field < SWPC_F_R + 18) return s->lR[field - SWPC_F_R];
    if (field >= SWPC_F_AUX && field < SWPC_F_AUX + 18) { *compact = true; return s->laux[field - SWPC_F_AUX]; }
    return nullptr;
}

extern "C" int swpc_adj_reset(swpc_ctx *c) {
    int rc = adj_ready(c);
    if (rc) return rc;
    rc = zero_adjoint(c);
    if (rc) return rc;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
}

extern "C" int swpc_adj_step_linear(swpc_ctx *c) {
    int rc = adj_ready(c);
    if (rc) return rc;
    rc = adj_step(c, nullptr, nullptr, -1);
    if (rc) return rc;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
}

extern "C" int swpc_adj_download(swpc_ctx *c, int field, float *out, int ld_k, int ld_i) {
    if (!out) return SWPC_ERR_ARG;
    int rc = adj_ready(c);
    if (rc) return rc;
    bool compact;
    float *p = adj_field(c, field, &compact);
    if (!p) return err(c, SWPC_ERR_ARG, "unknown or unallocated adjoint field");
    ACK(cudaStreamSynchronize(c->stream));
    return compact ? aux_transfer_ptr(c, p, out, nullptr, ld_k, ld_i) : copy_box(c, p, nullptr, out, ld_k, ld_i);
}

extern "C" int swpc_adj_upload(swpc_ctx *c, int field, const float *in, int ld_k, int ld_i) {
    if (!in) return SWPC_ERR_ARG;
    int rc = adj_ready(c);
    if (rc) return rc;
    bool compact;
    float *p = adj_field(c, field, &compact);
    if (!p) return err(c, SWPC_ERR_ARG, "unknown or unallocated adjoint field");
    ACK(cudaStreamSynchronize(c->stream));
    return compact ? aux_transfer_ptr(c, p, nullptr, in, ld_k, ld_i) : copy_box(c, p, in, nullptr, ld_k, ld_i);
}

// ---------------------------------------------------------------------------
// checkpointed gradient
// ---------------------------------------------------------------------------
static std::vector<float *> state_arrays(swpc_ctx *c, std::vector<size_t> *sizes) {
    std::vector<float *> v;
    for (int q = 0; q < 3; q++) { v.push_back(c->V[q]); sizes->push_back(c->g.ncell); }
    for (int q = 0; q < 6; q++) { v.push_back(c->S[q]); sizes->push_back(c->g.ncell); }
    for (int q = 0; q < 18; q++)
        if (c->R[q]) { v.push_back(c->R[q]); sizes->push_back(c->g.ncell); }
    if (c->npml > 0)
        for (int q = 0; q < 18; q++) { v.push_back(c->aux[q]); sizes->push_back(c->npml); }
    return v;
}

static int copy_state(swpc_ctx *c, float *ck, bool save) {
    std::vector<size_t> sz;
    auto arr = state_arrays(c, &sz);
    size_t off = 0;
    for (size_t n = 0; n < arr.size(); n++) {
        if (save) ACK(cudaMemcpyAsync(ck + off, arr[n], sz[n] * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
        else ACK(cudaMemcpyAsync(arr[n], ck + off, sz[n] * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
        off += sz[n];
    }
    return SWPC_OK;
}

// Slot `slot` of the recompute: V over the slot box (read with its halo by
// the stress-phase weights) and the stress divergences of the interior cells
// (the velocity-phase gradient), kSlotFields fields in the slot layout.
constexpr int kSlotFields = 6;
static int save_slot(swpc_ctx *c, int slot) {
    const SlotGeo sg = slot_geo(c);
    float *base = c->adj->slots + (size_t)slot * kSlotFields * sg.n;
    slot_v_kernel<<<148 * 8, 256, 0, c->stream>>>(c->g, sg, c->V[0], c->V[1], c->V[2], base);
    ACK(cudaGetLastError());
    SlotDivArgs a;
    a.g = c->g; a.ibk = c->ibk; a.iek = c->iek; a.jbk = c->jbk; a.jek = c->jek; a.kek = c->kek;
    for (int q = 0; q < 6; q++) a.S[q] = c->S[q];
    a.band = c->band;
    memcpy(a.e40, c->e40, sizeof(a.e40)); memcpy(a.e41, c->e41, sizeof(a.e41));
    for (int q = 0; q < 3; q++) a.divS[q] = base + (3 + q) * sg.n;
    a.sg = sg;
    const dim3 block(kThreadsK, 2, 2);
    slot_div_kernel<<<cell_grid(c->g, block), block, 0, c->stream>>>(a);
    return cuda_check(c, cudaGetLastError(), "slot_div_kernel");
}

static int zero_state(swpc_ctx *c) {
    std::vector<size_t> sz;
    auto arr = state_arrays(c, &sz);
    for (size_t n = 0; n < arr.size(); n++) ACK(cudaMemsetAsync(arr[n], 0, sz[n] * sizeof(float), c->stream));
    // recorder totals start from zero at it = 1 as the reference allocates them (m_wav.f90 displacement and
    // strain sums; m_green.f90:409-425 dxUx..uz); snapshot accumulators and maxima likewise
    if (c->uacc) ACK(cudaMemsetAsync(c->uacc, 0, 3 * sizeof(float) * std::max(c->nst, 1), c->stream));
    if (c->eacc) ACK(cudaMemsetAsync(c->eacc, 0, 6 * sizeof(float) * std::max(c->nst, 1), c->stream));
    if (c->g_acc) ACK(cudaMemsetAsync(c->g_acc, 0, 12 * sizeof(float) * std::max(c->ng, 1), c->stream));
    return snap_clear(c);
}

extern "C" int swpc_reset_state(swpc_ctx *c) {
    if (!c) return SWPC_ERR_ARG;
    if (c->kind != SWPC_KIND_3D) return err(c, SWPC_ERR_ARG, "swpc_reset_state is implemented for the 3D solver");
    ACK(cudaSetDevice(c->device));
    int rc = zero_state(c);
    if (rc) return rc;
    // a state from rest replaces any wavefield a failed tile copy left undefined
    if (c->d_err) ACK(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    return cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
}

extern "C" int swpc_gradient_set_slot_memory(swpc_ctx *c, long long bytes) {
    int rc = adj_ready(c);
    if (rc) return rc;
    if (bytes < 0) return err(c, SWPC_ERR_ARG, "slot memory must be >= 0 bytes");
    c->adj->slot_budget = bytes;
    return SWPC_OK;
}

// Whether a kept step may hold V on the shell of the slot box only: with no
// injection into V (body forces, green__source) the interior V of every step
// follows from the kept divergences (recon_kernel).
static bool keeps_shell(const swpc_ctx *c) { return c->ninj_bf == 0 && !c->green; }

// cells of the shell: slot-box cells with k = -1 .. kek + 2 outside the interior
static std::vector<int> shell_cells(const swpc_ctx *c, const SlotGeo &sg) {
    std::vector<int> out;
    for (int js = 0; js < sg.Jp; js++)
        for (int is = 0; is < sg.Ip; is++) {
            const int i = is + sg.i0, j = js + sg.j0;
            const bool col_in = i >= c->ibk && i <= c->iek && j >= c->jbk && j <= c->jek;
            for (int k = -1; k <= c->kek + 2; k++)
                if (!(col_in && k >= 1 && k <= c->kek)) out.push_back((int)slot_index(sg, k, i, j));
        }
    return out;
}

// floats of one kept step (divergences, then V of the shell or the slot box) and of a kept segment's first V
static void keep_sizes(const swpc_ctx *c, size_t *step, size_t *seg, int *nshell) {
    const SlotGeo sg = slot_geo(c);
    int ns = 0;
    if (keeps_shell(c)) {
        const int ni = c->iek - c->ibk + 1, nj = c->jek - c->jbk + 1;
        ns = (int)((long long)sg.Ip * sg.Jp * (c->kek + 4) - (long long)ni * nj * c->kek);
    }
    *step = 3 * (size_t)sg.n + (keeps_shell(c) ? 3 * (size_t)ns : 3 * (size_t)sg.n);
    *seg = 3 * (size_t)sg.n;
    if (nshell) *nshell = ns;
}

extern "C" int swpc_gradient_memory(swpc_ctx *c, long long *ckpt_bytes, long long *slot_bytes) {
    if (!c || !ckpt_bytes || !slot_bytes) return SWPC_ERR_ARG;
    if (c->kind != SWPC_KIND_3D) return err(c, SWPC_ERR_ARG, "the adjoint is implemented for the 3D solver");
    std::vector<size_t> sz;
    state_arrays(c, &sz);
    long long ckf = 0;
    for (size_t v : sz) ckf += (long long)v;
    size_t step, seg;
    keep_sizes(c, &step, &seg, nullptr);
    *ckpt_bytes = ckf * (long long)sizeof(float);
    *slot_bytes = (long long)(step * sizeof(float));
    return SWPC_OK;
}

extern "C" int swpc_gradient_segment_bytes(swpc_ctx *c, long long *seg_bytes, long long *work_bytes, int ckpt) {
    if (!c || !seg_bytes || !work_bytes || ckpt < 1) return SWPC_ERR_ARG;
    if (c->kind != SWPC_KIND_3D) return err(c, SWPC_ERR_ARG, "the adjoint is implemented for the 3D solver");
    size_t step, seg;
    keep_sizes(c, &step, &seg, nullptr);
    *seg_bytes = (long long)(seg * sizeof(float));
    *work_bytes = (long long)((size_t)kSlotFields * slot_geo(c).n * (ckpt + 1) * sizeof(float));
    return SWPC_OK;
}

// Trailing segments whose kept steps (step floats each) and first V (seg floats each) fit in `budget` floats;
// their steps in *steps.
static int tail_segments(int nt, int ckpt, int nseg, long long budget, size_t step, size_t seg, long long *steps) {
    int ntail = 0;
    long long n = 0;
    while (ntail < nseg) {
        const int it0 = (nseg - 1 - ntail) * ckpt + 1, len = std::min(ckpt, nt - it0 + 1);
        if ((long long)((n + len) * step + (ntail + 1) * seg) > budget) break;
        n += len;
        ntail++;
    }
    *steps = n;
    return ntail;
}

// Kept step it of the trailing segments: the three divergences after step it
// in the slot layout (unless the velocity update stored them, div_done), then
// V of the shell (or of the slot box).
static int save_kept(swpc_ctx *c, float *dst, bool div_done) {
    swpc_adj_state *s = c->adj;
    const SlotGeo sg = slot_geo(c);
    if (div_done) goto vpart;
    {
    SlotDivArgs a;
    a.g = c->g; a.ibk = c->ibk; a.iek = c->iek; a.jbk = c->jbk; a.jek = c->jek; a.kek = c->kek;
    for (int q = 0; q < 6; q++) a.S[q] = c->S[q];
    a.band = c->band;
    memcpy(a.e40, c->e40, sizeof(a.e40)); memcpy(a.e41, c->e41, sizeof(a.e41));
    for (int q = 0; q < 3; q++) a.divS[q] = dst + q * sg.n;
    a.sg = sg;
    const dim3 block(kThreadsK, 2, 2);
    slot_div_kernel<<<cell_grid(c->g, block), block, 0, c->stream>>>(a);
    ACK(cudaGetLastError());
    }
vpart:
    if (keeps_shell(c))
        shell_save_kernel<<<148 * 4, 256, 0, c->stream>>>(c->g, sg, c->V[0], c->V[1], c->V[2], s->shell, s->nshell,
                                                          dst + 3 * sg.n);
    else
        slot_v_kernel<<<148 * 8, 256, 0, c->stream>>>(c->g, sg, c->V[0], c->V[1], c->V[2], dst + 3 * sg.n);
    return cuda_check(c, cudaGetLastError(), "save_kept");
}

extern "C" int swpc_gradient(swpc_ctx *c, const float *obs, int ckpt, double *misfit) {
    int rc = adj_ready(c);
    if (rc) return rc;
    if (!obs || !misfit || ckpt < 1) return err(c, SWPC_ERR_ARG, "observed traces, misfit and ckpt >= 1 required");
    if (c->nst <= 0 || !(c->wav_what & SWPC_WAV_V)) return err(c, SWPC_ERR_STATE, "velocity recorder not set up");
    swpc_adj_state *s = c->adj;
    const int nt = c->d.nt;
    const int nseg = (nt + ckpt - 1) / ckpt;
    std::vector<size_t> sz;
    state_arrays(c, &sz);
    size_t ckf = 0;
    for (size_t v : sz) ckf += v;
    const SlotGeo sg = slot_geo(c);
    const size_t n = (size_t)sg.n, slot_floats = (size_t)kSlotFields * n;
    // the trailing segments whose steps fit the budget keep them from the first forward pass (the divergences
    // and V of the shell every step, V of the first state): they are neither checkpointed nor recomputed, and
    // their V is rebuilt into the working slots; the earlier segments are recomputed into the working slots
    size_t kstep, kseg;
    int nshell = 0;
    keep_sizes(c, &kstep, &kseg, &nshell);
    long long tail_steps = 0;
    const int ntail = tail_segments(nt, ckpt, nseg, s->slot_budget / (long long)sizeof(float), kstep, kseg,
                                    &tail_steps);
    const int gT = nseg - ntail, itT0 = gT * ckpt + 1;
    const size_t cap = (size_t)ckpt + 1;
    const size_t need_ck = ckf * std::max(gT, 1), need_keep = (size_t)tail_steps * kstep + (size_t)ntail * kseg;
    if (s->ckpt != ckpt || s->nseg != nseg || s->ck_floats != ckf || s->slot_cap != cap || s->ntail != ntail ||
        s->keep_floats != need_keep) {
        if (s->ckpool) cudaFree(s->ckpool);
        if (s->slots) cudaFree(s->slots);
        if (s->keep) cudaFree(s->keep);
        s->ckpool = s->slots = s->keep = nullptr;
        s->ckpt = s->nseg = s->ntail = 0;
        s->ck_floats = s->slot_cap = s->keep_floats = 0;
        if (cudaMalloc((void **)&s->ckpool, need_ck * sizeof(float)) != cudaSuccess ||
            cudaMalloc((void **)&s->slots, slot_floats * cap * sizeof(float)) != cudaSuccess ||
            (need_keep && cudaMalloc((void **)&s->keep, need_keep * sizeof(float)) != cudaSuccess)) {
            cudaGetLastError();
            return err(c, SWPC_ERR_NOMEM, "no room for the checkpoints and slots (raise ckpt, lower the slot "
                                          "memory or shrink the grid)");
        }
        s->ckpt = ckpt; s->nseg = nseg; s->ck_floats = ckf; s->slot_cap = cap; s->ntail = ntail;
        s->keep_floats = need_keep;
        // the staged stress-phase weights read the forward V of a slot with its halo
        Geo gs = c->g;
        gs.Kp = sg.Kp; gs.Ip = sg.Ip; gs.Jp = sg.Jp; gs.ncell = sg.n;
        if (!tma_encode_box(s->maps->vh, s->slots, gs, (long long)kSlotFields * cap, tma::KB, adjt::BI + 4, adjt::BJ + 4, 3))
            return err(c, SWPC_ERR_CUDA, "cuTensorMapEncodeTiled failed for the recompute slots");
    }
    if (ntail > 0 && keeps_shell(c) && s->nshell != nshell) {
        const std::vector<int> sh = shell_cells(c, sg);
        if (s->shell) cudaFree(s->shell);
        s->shell = nullptr;
        s->nshell = 0;
        ACK(cudaMalloc((void **)&s->shell, sh.size() * sizeof(int)));
        ACK(cudaMemcpy(s->shell, sh.data(), sh.size() * sizeof(int), cudaMemcpyHostToDevice));
        s->nshell = (int)sh.size();
    }
    // kept segment g >= gT: its first V at keep + (g - gT) * kseg, its steps after all first Vs
    auto kept_first = [&](int g) { return s->keep + (size_t)(g - gT) * kseg; };
    auto kept_step = [&](int it) { return s->keep + (size_t)ntail * kseg + (size_t)(it - itT0) * kstep; };
    const size_t nres = (size_t)c->nst * 3 * c->ntw;
    if (!s->res) ACK(cudaMalloc((void **)&s->res, nres * sizeof(float)));
    // 1. forward from rest with a checkpoint before every recomputed segment; the trailing segments keep their
    //    steps instead (the recorders run in both)
    rc = zero_state(c);
    if (rc) return rc;
    for (int g = 0; g < nseg && !rc; g++) {
        const int it0 = g * ckpt + 1, len = std::min(ckpt, nt - it0 + 1);
        if (g < gT) {
            rc = copy_state(c, s->ckpool + (size_t)g * ckf, true);
            if (!rc) rc = swpc_run(c, it0, len);
            continue;
        }
        slot_v_kernel<<<148 * 8, 256, 0, c->stream>>>(c->g, sg, c->V[0], c->V[1], c->V[2], kept_first(g));
        rc = cuda_check(c, cudaGetLastError(), "slot_v_kernel");
        // the staged and the one-cell velocity kernels store the divergences as they update V (their own
        // values, so the same bits as slot_div_kernel); the other variants leave them to slot_div_kernel
        const bool in_vel = !c->vel_march && !c->vel_vec;
        for (int it = it0; it < it0 + len && !rc; it++) {
            if (in_vel) {
                c->div_out = kept_step(it);
                c->div_geo[0] = sg.Kp; c->div_geo[1] = sg.Ip; c->div_geo[2] = sg.i0; c->div_geo[3] = sg.j0;
                c->div_n = sg.n;
                rc = swpc_step(c, it);
                c->div_out = nullptr;
            } else {
                rc = swpc_run(c, it, 1);
            }
            if (!rc) rc = save_kept(c, kept_step(it), in_vel);
        }
    }
    if (rc) return rc;
    // 2. residuals and misfit
    std::vector<float> syn(nres);
    ACK(cudaMemcpyAsync(syn.data(), c->wav[0], nres * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    ACK(cudaStreamSynchronize(c->stream));
    double J = 0.0;
    for (size_t q = 0; q < nres; q++) {
        syn[q] = syn[q] - obs[q];
        J += 0.5 * (double)syn[q] * (double)syn[q];
    }
    *misfit = J;
    ACK(cudaMemcpyAsync(s->res, syn.data(), nres * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    // 3. adjoint, segment by segment from the last
    rc = source_cells(c);
    if (!rc) rc = zero_adjoint(c);
    if (rc) return rc;
    for (int g = nseg - 1; g >= 0; g--) {
        const int it0 = g * ckpt + 1, it1 = std::min(it0 + ckpt - 1, nt), len = it1 - it0 + 1;
        // the forward V of the segment in the working slots 0..len, and where the divergences of each step are
        const bool kept = g >= gT;
        if (kept) {
            ACK(cudaMemcpyAsync(s->slots, kept_first(g), 3 * n * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
            if (keeps_shell(c)) {
                ReconArgs ra;
                ra.g = c->g; ra.sg = sg; ra.ibk = c->ibk; ra.iek = c->iek; ra.jbk = c->jbk; ra.jek = c->jek;
                ra.kek = c->kek; ra.len = len;
                for (int q = 0; q < 3; q++) ra.b[q] = c->med[5 + q];
                ra.dt = c->d.dt;
                ra.div1 = kept_step(it0);
                ra.kstride = kstep;
                ra.slot0 = s->slots;
                ra.sstride = slot_floats;
                recon_kernel<<<148 * 8, 256, 0, c->stream>>>(ra);
                ACK(cudaGetLastError());
                shell_load_kernel<<<148 * 4, 256, 0, c->stream>>>(kept_step(it0) + 3 * n, kstep, s->shell, s->nshell,
                                                                  len, sg.n, s->slots + slot_floats, slot_floats);
                ACK(cudaGetLastError());
            } else {
                for (int m = 1; m <= len; m++)
                    ACK(cudaMemcpyAsync(s->slots + m * slot_floats, kept_step(it0 + m - 1) + 3 * n,
                                        3 * n * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
            }
        } else {
            rc = copy_state(c, s->ckpool + (size_t)g * ckf, false);
            if (!rc) rc = save_slot(c, 0);
            // the recompute advances the wavefield only: the recorders already hold these steps
            for (int it = it0; it <= it1 && !rc; it++) {
                rc = step_state(c, it);
                if (!rc) rc = save_slot(c, it - it0 + 1);
            }
        }
        // divergences after step it: the kept step, or the working slot
        auto divs = [&](int it, const float **D) {
            const float *base = kept ? kept_step(it) : s->slots + (size_t)(it - it0 + 1) * slot_floats + 3 * n;
            for (int q = 0; q < 3; q++) D[q] = base + q * n;
        };
        // within a segment each stress-phase gather also forms the velocity-phase weights of the step before
        // (kernel 9 of swpc_set_launch); the first step of a segment forms its own
        bool vel_done = false;
        for (int it = it1; it >= it0 && !rc; it--) {
            const size_t sb = (size_t)(it - it0);
            const float *Da[3], *Vb[3], *Dn[3] = {nullptr, nullptr, nullptr};
            divs(it, Da);
            for (int q = 0; q < 3; q++) Vb[q] = s->slots + sb * slot_floats + q * n;
            if (it > it0) divs(it - 1, Dn);   // divergences of step it - 1
            AdjNext nx;
            nx.on = c->adj_fuse && it > it0;
            nx.skip_src = source_at(c, it);
            nx.divS = Dn;
            rc = adj_step(c, Da, Vb, (int)(sb * kSlotFields), vel_done, nx);
            if (!rc) rc = adj_source(c, it, Dn, nx.on);
            vel_done = nx.on;
        }
        if (!rc) rc = fold_gradient(c);
        if (rc) return rc;
    }
    return cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
}

// device double array -> host memory box
static int fetch_double(swpc_ctx *c, const double *dev, double *out, int ld_k, int ld_i) {
    const Geo &g = c->g;
    std::vector<double> h((size_t)g.ncell);
    ACK(cudaMemcpyAsync(h.data(), dev, g.ncell * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ACK(cudaStreamSynchronize(c->stream));
    for (int j = -2; j <= g.ny + 3; j++)
        for (int i = -2; i <= g.nx + 3; i++)
            for (int k = -2; k <= g.nz + 3; k++)
                out[((long long)(j + 2) * ld_i + (i + 2)) * ld_k + (k + 2)] = h[cell_index(g, k, i, j)];
    return SWPC_OK;
}

extern "C" int swpc_gradient_fetch(swpc_ctx *c, int which, double *out, int ld_k, int ld_i) {
    if (!c || !out || which < 0 || which > 7) return SWPC_ERR_ARG;
    if (!c->adj) return err(c, SWPC_ERR_STATE, "swpc_gradient not called");
    const Geo &g = c->g;
    if (ld_k < g.nz + 6 || ld_i < g.nx + 6) return err(c, SWPC_ERR_ARG, "leading extents smaller than the memory box");
    ACK(cudaSetDevice(c->device));
    return fetch_double(c, c->adj->grad[which], out, ld_k, ld_i);
}

// device double array -> device memory box (leading extents ld_k, ld_i)
__global__ void unpack_double_kernel(Geo g, const double *__restrict__ src, double *dst, int ld_k, int ld_i) {
    const int nkb = g.nz + 6, nib = g.nx + 6;
    const long long n = (long long)nkb * nib * (g.ny + 6);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int kb = (int)(t % nkb);
        const long long col = t / nkb;
        const int ib = (int)(col % nib), jb = (int)(col / nib);
        dst[((long long)jb * ld_i + ib) * ld_k + kb] = src[cell_index(g, kb - 2, ib - 2, jb - 2)];
    }
}

static bool is_device_array(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

static int gradient_model(swpc_ctx *c, const float *vp, const float *vs, const float *rho, int ld_k, int ld_i,
                          double *gvp, double *gvs, double *grho, bool on_device);

extern "C" int swpc_gradient_model(swpc_ctx *c, const float *vp, const float *vs, const float *rho, int ld_k,
                                   int ld_i, double *gvp, double *gvs, double *grho) {
    return gradient_model(c, vp, vs, rho, ld_k, ld_i, gvp, gvs, grho, false);
}

extern "C" int swpc_gradient_model_device(swpc_ctx *c, const float *vp, const float *vs, const float *rho, int ld_k,
                                          int ld_i, double *gvp, double *gvs, double *grho) {
    return gradient_model(c, vp, vs, rho, ld_k, ld_i, gvp, gvs, grho, true);
}

static int gradient_model(swpc_ctx *c, const float *vp, const float *vs, const float *rho, int ld_k, int ld_i,
                          double *gvp, double *gvs, double *grho, bool on_device) {
    if (!c || !vp || !vs || !rho || !gvp || !gvs || !grho) return SWPC_ERR_ARG;
    if (on_device)
        for (const void *p : {(const void *)vp, (const void *)vs, (const void *)rho, (const void *)gvp,
                              (const void *)gvs, (const void *)grho})
            if (!is_device_array(p)) return err(c, SWPC_ERR_ARG, "swpc_gradient_model_device takes device arrays");
    if (!c->adj) return err(c, SWPC_ERR_STATE, "swpc_gradient not called");
    const Geo &g = c->g;
    if (ld_k < g.nz + 6 || ld_i < g.nx + 6) return err(c, SWPC_ERR_ARG, "leading extents smaller than the memory box");
    ACK(cudaSetDevice(c->device));
    float *dm[3] = {};
    double *dg[3] = {};
    int rc = SWPC_OK;
    const float *hm[3] = {vp, vs, rho};
    for (int q = 0; q < 3 && !rc; q++) {
        rc = dalloc(c, &dm[q], g.ncell);
        if (!rc) rc = dalloc(c, &dg[q], g.ncell);
        if (!rc) rc = on_device ? copy_box_from_device(c, dm[q], hm[q], ld_k, ld_i)
                                : copy_box(c, dm[q], hm[q], nullptr, ld_k, ld_i);
    }
    if (!rc) {
        ModelGradArgs a;
        a.g = g;
        for (int q = 0; q < 8; q++) a.gm[q] = c->adj->grad[q];
        a.lam = c->med[1]; a.mu = c->med[2];
        for (int q = 0; q < 3; q++) a.b[q] = c->med[5 + q];
        a.vp = dm[0]; a.vs = dm[1]; a.rho = dm[2];
        for (int q = 0; q < 3; q++) a.out[q] = dg[q];
        const dim3 block(kThreadsK, 2, 2);
        model_grad_kernel<<<cell_grid(g, block), block, 0, c->stream>>>(a);
        rc = cuda_check(c, cudaGetLastError(), "model_grad_kernel");
    }
    double *ho[3] = {gvp, gvs, grho};
    for (int q = 0; q < 3 && !rc; q++) {
        if (on_device) {
            unpack_double_kernel<<<148 * 8, 256, 0, c->stream>>>(g, dg[q], ho[q], ld_k, ld_i);
            rc = cuda_check(c, cudaGetLastError(), "unpack_double_kernel");
        } else {
            rc = fetch_double(c, dg[q], ho[q], ld_k, ld_i);
        }
    }
    cudaStreamSynchronize(c->stream);
    for (int q = 0; q < 3; q++) {
        if (dm[q]) { cudaFree(dm[q]); c->bytes -= (long long)g.ncell * sizeof(float); }
        if (dg[q]) { cudaFree(dg[q]); c->bytes -= (long long)g.ncell * sizeof(double); }
    }
    return rc;
}
