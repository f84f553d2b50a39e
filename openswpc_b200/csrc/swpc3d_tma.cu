// swpc3d_tma.cu -- the fused 3D stress and velocity updates with their
// operands staged in shared memory by TMA (kernel__update_stress /
// kernel__update_vel, src/swpc_3d/m_kernel.f90:75-326).
//
// The one-cell-per-thread kernels keep every operand of a cell in registers
// while its loads are in flight, so the register file bounds the bytes in
// flight per SM and the kernels stall on load latency below the HBM roofline.
// Here a CTA owns a tile of 32 (k) x BI (i) x BJ (j) cells and one thread
// issues bulk tensor copies for the whole tile: the medium of the tile (one
// box over consecutive medium fields), and per wavefield member the fields the
// update reads once (S and R, or V) and the stencil fields with their halos
// (the stress kernel: V over k-2..k+2, i-2..i+2, j-2..j+2; the velocity
// kernel: one box per stress component with the halo of its own difference).
// The copies land in shared memory and complete on an mbarrier; several CTAs
// per SM keep well over a hundred KB per SM in flight without holding
// registers.  Each thread then updates its cell from shared memory with the
// arithmetic of the one-cell kernels (stress_interior / vel_interior, the same
// expression order), so the results are bitwise identical.  Absorber cells
// read the tile too (stress_absorber / vel_absorber); only their compact PML
// auxiliaries come from global memory.  A stress tile without interior cells
// copies S without R.  The tensor boxes may reach past the grid at
// its edges: TMA fills those elements with zeros and they are never used.
//
// The lead thread issues the copies first and only then reads the launch's
// error word, while the copies travel; the other threads meanwhile read the
// band signs and the absorber auxiliaries of their cells.  The tile wait is
// bounded (swpc_tma_ptx.cuh).
//
// A CTA serves M members that share the medium (M = 1 for a single run; the
// reciprocity batch, swpc_fbatch.cu, groups its members): the medium box is
// copied once and each member's boxes follow, so the medium crosses HBM once
// per M member updates.  The launch order of tiles and member groups is
// tile_of's (swpc_tma_tile.cuh).
//
// Field order of the state slab (per member): 0-2 V, 3-8 S, 9.. R
// (component-major, nm per component).  Medium slab: lam mu taup taus muyz
// muxz muxy, then bx by bz, from field f_med (the context's slab holds both,
// see swpc_create).  The reduced storage forms keep S (F16_SR) and R in a
// second slab of 2-byte fields (template parameter PREC).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include "swpc3d_cell.cuh"
#include "swpc_tma.h"
#include "swpc_tma_ptx.cuh"
#include "swpc_tma_tile.cuh"

namespace swpc {

namespace {

using namespace tma;

// ---------------------------------------------------------------------------
// stress
// ---------------------------------------------------------------------------
// Shared-memory layout (floats): medium [7][BJ][BI][KT], then per member the
// state region and V [3][BJ+4][BI+4][KB].  The state region by storage form:
//   PREC_F32:    [6 + 6 NM][BJ][BI][KT] floats (S xx..xy, then R)
//   PREC_BF16_R: S [6][BJ][BI][KT] floats, then R [6 NM][BJ][BI][KT] BF16 at oR
//   PREC_F16_SR: [6 + 6 NM][BJ][BI][KT] FP16 (S, then R; stored values)
template <int NM, int BI, int BJ, int M, int PREC = PREC_F32>
struct StrBoxes {
    static constexpr int n = BJ * BI * KT;   // cells of a tile
    static constexpr int nMed = 7 * n;
    static constexpr int nState = PREC == PREC_F32 ? (6 + 6 * NM) * n
                                : r_only_half<PREC>() ? up32(6 * n) + 3 * NM * n : (3 + 3 * NM) * n;
    static constexpr int oR = up32(6 * n);   // 2-byte R box within the state region (BF16_R, F16_R)
    static constexpr int nV = 3 * (BJ + 4) * (BI + 4) * KB;
    static constexpr int member = up32(nState) + up32(nV);
    static constexpr int total = up32(nMed) + M * member;
    __host__ __device__ static constexpr int oMem(int mm) { return up32(nMed) + mm * member; }
    // bytes a member's state copies bring (S alone in tiles without interior cells)
    __host__ __device__ static constexpr int state_bytes(bool with_r) {
        return PREC == PREC_F32 ? 4 * (with_r ? 6 + 6 * NM : 6) * n
             : r_only_half<PREC>() ? 4 * 6 * n + (with_r ? 2 * 6 * NM * n : 0) : 2 * (with_r ? 6 + 6 * NM : 6) * n;
    }
    __host__ __device__ static constexpr int bytes(int nmem, bool with_r) {
        return 4 * nMed + nmem * (state_bytes(with_r) + 4 * nV);
    }
};

template <int NM, int BI, int BJ, int PREC = PREC_F32>
struct SStrOps {
    const float *ss;   // member's state region
    const float *sv;   // member's V box
    const float *sm;   // medium box: lam mu taup taus muyz muxz muxy
    int tx, ty, tz;
    const Str3Args &a;   // FP16 scales of S and R (PREC_F16_SR)
    __device__ __forceinline__ int at(int f) const { return ((f * BJ + tz) * BI + ty) * KT + tx; }
    __device__ __forceinline__ float v(int c, int dk, int di, int dj) const {
        return sv[((c * (BJ + 4) + tz + 2 + dj) * (BI + 4) + ty + 2 + di) * KB + tx + 4 + dk];
    }
    __device__ __forceinline__ float sown(int f) const {
        if constexpr (PREC == PREC_F16_SR) return __half2float(reinterpret_cast<const __half *>(ss)[at(f)]) * sc_sS_in(a.scale, f);
        else return ss[at(f)];
    }
    __device__ __forceinline__ float r(int q) const {
        const int f = (q / 3) * NM + q % 3;
        if constexpr (PREC == PREC_F16_SR) return __half2float(reinterpret_cast<const __half *>(ss)[at(6 + f)]) * sc_sR_in(a.scale);
        else if constexpr (PREC == PREC_BF16_R)
            return __bfloat162float(reinterpret_cast<const __nv_bfloat16 *>(ss + StrBoxes<NM, BI, BJ, 1, PREC>::oR)[at(f)]);
        else if constexpr (PREC == PREC_F16_R)
            return __half2float(reinterpret_cast<const __half *>(ss + StrBoxes<NM, BI, BJ, 1, PREC>::oR)[at(f)]) * sc_sR_in(a.scale);
        else return ss[at(6 + f)];
    }
    // 0 mu, 1 lam, 2 taup, 3 taus, 4 muyz, 5 muxz, 6 muxy
    __device__ __forceinline__ float med(int m) const { return sm[at(m == 0 ? 1 : m == 1 ? 0 : m)]; }
};

// Maps by storage form: tm_state = S and R (F32 slab; F16_SR: the 2-byte
// slab) or R alone (BF16_R: the 2-byte slab); tm_s = S alone (the slab that
// holds S).
template <int NM, int BI, int BJ, int M, int PREC>
__global__ void __launch_bounds__(KT * BI * BJ,
                                  (blocks_per_sm<StrBoxes<NM, BI, BJ, M, PREC>::total, KT * BI * BJ>()))
    stress3d_tma_kernel(const __grid_constant__ CUtensorMap tm_state, const __grid_constant__ CUtensorMap tm_s,
                        const __grid_constant__ CUtensorMap tm_med, const __grid_constant__ CUtensorMap tm_v,
                        const Str3Args a, const TmaTiles t) {
    static_assert(PREC == PREC_F32 || M == 1, "reduced storage forms run single members");
    using L = StrBoxes<NM, BI, BJ, M, PREC>;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ unsigned long long limit;
    float *sm = aligned128(smraw);
    const Geo g = a.g;
    const Tile T = tile_of<M>(t, BI, BJ);
    const int tx = threadIdx.x, ty = threadIdx.y, tz = threadIdx.z;
    const bool lead = tx == 0 && ty == 0 && tz == 0;
    // cells of this launch in the tile: interior ones need S, R and the medium, absorber ones S and the medium
    const bool with_r = (a.mask & 1) && tile_has_interior(T, BI, BJ, a.ibk, a.iek, a.jbk, a.jek, a.kek);
    const bool staged =
        with_r || ((a.mask & 2) && tile_has_absorber(T, BI, BJ, g, a.ibk, a.iek, a.jbk, a.jek, a.kek));
    if (!staged) return;   // nothing of this launch here (uniform over the CTA)
    if (lead) {
        // the copies go out first; the error word is read while they travel
        stage_init(&bar, (unsigned)L::bytes(T.nmem, with_r));
        const int x0 = T.k0 - 1 + KH;
        load_4d(sm, &tm_med, x0, T.i0 + 2, T.j0 + 2, t.f_med, &bar);
        for (int mm = 0; mm < T.nmem; mm++) {
            const int fm = (T.m0 + mm) * t.f_member;
            float *p = sm + L::oMem(mm);
            if constexpr (r_only_half<PREC>()) {
                load_4d(p, &tm_s, x0, T.i0 + 2, T.j0 + 2, t.f_state, &bar);
                if (with_r && NM > 0) load_4d(p + L::oR, &tm_state, x0, T.i0 + 2, T.j0 + 2, t.f_h, &bar);
            } else if constexpr (PREC == PREC_F16_SR) {
                load_4d(p, with_r ? &tm_state : &tm_s, x0, T.i0 + 2, T.j0 + 2, t.f_h, &bar);
            } else {
                load_4d(p, with_r ? &tm_state : &tm_s, x0, T.i0 + 2, T.j0 + 2, t.f_state + fm, &bar);
            }
            load_4d(p + up32(L::nState), &tm_v, x0 - 4, T.i0, T.j0, t.f_v + fm, &bar);
        }
        limit = wait_limit(t.err);
    }
    const int k = T.k0 + tx, i = T.i0 + ty, j = T.j0 + tz;
    const bool interior = i >= a.ibk && i <= a.iek && j >= a.jbk && j <= a.jek && k <= a.kek;
    const bool mine = k <= g.nz && i <= g.nx && j <= g.ny && (a.mask & (interior ? 1 : 2));
    const long long col = col_index(g, i, j);
    const long long e = col * g.Kp + (k - 1 + KH);
    // the band sign of an interior cell and the auxiliaries of an absorber
    // cell (up to two members) are read while the tiles travel
    const int sgn = (mine && interior) ? band_sign_of(a.band, col, k) : 0;
    constexpr bool PRE = M <= 2;
    Aux9 xs[PRE ? M : 1];
    if (PRE && mine && !interior) {
#pragma unroll
        for (int mm = 0; mm < (PRE ? M : 1); mm++)
            if (mm < T.nmem) xs[mm] = aux_load(a.aV, (long long)(T.m0 + mm) * t.ao, a.pmlcol, g, k, i, j);
    }
    __syncthreads();   // barrier initialised, wait limit set
    if (!wait_tiles(&bar, t.err, limit) || !mine) return;   // the copy failed, or no cell of this launch here
#pragma unroll
    for (int mm = 0; mm < M; mm++) {
        if (mm >= T.nmem) break;
        const long long so = (long long)(T.m0 + mm) * t.so, ao = (long long)(T.m0 + mm) * t.ao;
        const float *p = sm + L::oMem(mm);
        const SStrOps<NM, BI, BJ, PREC> o{p, p + up32(L::nState), sm, tx, ty, tz, a};
        float *const Sp[6] = {a.Sxx + so, a.Syy + so, a.Szz + so, a.Syz + so, a.Sxz + so, a.Sxy + so};
        if (interior) {
            stress_interior<NM, PREC>(a, o, sgn, Sp, e, so);
        } else {
            const Aux9 x = PRE ? xs[PRE ? mm : 0] : aux_load(a.aV, ao, a.pmlcol, g, k, i, j);
            stress_absorber<PREC>(a, o, x, k, i, j, e, ao, Sp);
        }
    }
}

// ---------------------------------------------------------------------------
// velocity
// ---------------------------------------------------------------------------
// Shared-memory layout (floats): b [3][BJ][BI][KT], then per member V
// [3][BJ][BI][KT] and one box per stress component with only the halo its
// difference needs: Sxx i-1..i+2, Syy j-1..j+2, Szz k-1..k+2, Syz j-2..j+1 /
// k-2..k+1, Sxz i-2..i+1 / k-2..k+1, Sxy i-2..i+1 / j-2..j+1.  PREC_F16_SR
// keeps the stress boxes as stored FP16; their k halo then starts 8 cells
// below the tile (a 2-byte box must start on a 16-byte boundary).
template <int BI, int BJ, int M, int PREC = PREC_F32>
struct VelBoxes {
    static constexpr bool H = PREC == PREC_F16_SR;
    static constexpr int KS = H ? KT + 16 : KB;              // k extent of a stress box with k halo
    static constexpr int KO = H ? 8 : 4;                     // its first cell, below k0
    __host__ __device__ static constexpr int fl(int n) { return H ? n / 2 : n; }   // stress elements -> floats
    static constexpr int nB3 = 3 * BJ * BI * KT;            // bx by bz; V of a member likewise
    static constexpr int nA = BJ * (BI + 3) * KT;            // Sxx
    static constexpr int nBy = (BJ + 3) * BI * KT;           // Syy
    static constexpr int nC = BJ * BI * KS;                  // Szz
    static constexpr int nF = (BJ + 3) * BI * KS;            // Syz
    static constexpr int nE = BJ * (BI + 3) * KS;            // Sxz
    static constexpr int nD = (BJ + 3) * (BI + 3) * KT;      // Sxy
    // offsets within a member (floats)
    static constexpr int oV = 0, oA = up32(nB3), oBy = oA + up32(fl(nA)), oC = oBy + up32(fl(nBy)),
                         oF = oC + up32(fl(nC)), oE = oF + up32(fl(nF)), oD = oE + up32(fl(nE)),
                         member = oD + up32(fl(nD));
    static constexpr int total = up32(nB3) + M * member;
    __host__ __device__ static constexpr int oMem(int mm) { return up32(nB3) + mm * member; }
    __host__ __device__ static constexpr int bytes(int nmem) {
        return 4 * nB3 + nmem * (4 * nB3 + (H ? 2 : 4) * (nA + nBy + nC + nF + nE + nD));
    }
};

template <int BI, int BJ, int PREC = PREC_F32>
struct SVelOps {
    const float *mem;   // member's boxes
    const float *sb;    // bx by bz
    int tx, ty, jj;
    const Vel3Args &a;  // FP16 scales of S (PREC_F16_SR)
    using L = VelBoxes<BI, BJ, 1, PREC>;
    __device__ __forceinline__ int at(int c) const { return ((c * BJ + jj) * BI + ty) * KT + tx; }
    __device__ __forceinline__ float v(int c) const { return mem[L::oV + at(c)]; }
    __device__ __forceinline__ float b(int c) const { return sb[at(c)]; }
    // element q of the box at float offset o
    __device__ __forceinline__ float el(int f, int o, int q) const {
        if constexpr (L::H) return __half2float(reinterpret_cast<const __half *>(mem + o)[q]) * sc_sS(a.scale, f);
        else return mem[o + q];
    }
    __device__ __forceinline__ float s(int f, int dk, int di, int dj) const {
        constexpr int KS = L::KS, KO = L::KO;
        switch (f) {
        case 0: return el(0, L::oA, (jj * (BI + 3) + ty + 1 + di) * KT + tx);
        case 1: return el(1, L::oBy, ((jj + 1 + dj) * BI + ty) * KT + tx);
        case 2: return el(2, L::oC, (jj * BI + ty) * KS + tx + KO + dk);
        case 3: return el(3, L::oF, ((jj + 2 + dj) * BI + ty) * KS + tx + KO + dk);
        case 4: return el(4, L::oE, (jj * (BI + 3) + ty + 2 + di) * KS + tx + KO + dk);
        default: return el(5, L::oD, ((jj + 2 + dj) * (BI + 3) + ty + 2 + di) * KT + tx);
        }
    }
};

// One CTA per tile of KT x BI x BJ cells and member group, with KT x BI
// threads; each thread updates its (k, i) for the BJ planes j0 .. j0+BJ-1 of
// every member of the group.  The stress maps tm_a .. tm_d cover the slab that
// holds S (PREC_F16_SR: the 2-byte slab, S from field t.f_h).
template <int BI, int BJ, int M, int PREC>
__global__ void __launch_bounds__(KT * BI, (blocks_per_sm<VelBoxes<BI, BJ, M, PREC>::total, KT * BI>()))
    vel3d_tma_kernel(const __grid_constant__ CUtensorMap tm_own, const __grid_constant__ CUtensorMap tm_b,
                     const __grid_constant__ CUtensorMap tm_a, const __grid_constant__ CUtensorMap tm_by,
                     const __grid_constant__ CUtensorMap tm_c, const __grid_constant__ CUtensorMap tm_f,
                     const __grid_constant__ CUtensorMap tm_e, const __grid_constant__ CUtensorMap tm_d,
                     const Vel3Args a, const TmaTiles t) {
    static_assert(PREC == PREC_F32 || M == 1, "reduced storage forms run single members");
    using L = VelBoxes<BI, BJ, M, PREC>;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ unsigned long long limit;
    float *sm = aligned128(smraw);
    const Geo g = a.g;
    const Tile T = tile_of<M>(t, BI, BJ);
    const int tx = threadIdx.x, ty = threadIdx.y;
    const bool lead = tx == 0 && ty == 0;
    const bool staged = ((a.mask & 1) && tile_has_interior(T, BI, BJ, a.ibk, a.iek, a.jbk, a.jek, a.kek)) ||
                        ((a.mask & 2) && tile_has_absorber(T, BI, BJ, g, a.ibk, a.iek, a.jbk, a.jek, a.kek));
    if (!staged) return;   // nothing of this launch here (uniform over the CTA)
    if (lead) {
        // the copies go out first; the error word is read while they travel
        stage_init(&bar, (unsigned)L::bytes(T.nmem));
        const int x0 = T.k0 - 1 + KH, ic = T.i0 + 2, jc = T.j0 + 2;
        load_4d(sm, &tm_b, x0, ic, jc, t.f_b, &bar);
        for (int mm = 0; mm < T.nmem; mm++) {
            const int f = t.f_v + (T.m0 + mm) * t.f_member;   // Vx of the member
            const int fs = L::H ? t.f_h : f + 3;               // Sxx of the member
            float *p = sm + L::oMem(mm);
            load_4d(p + L::oV, &tm_own, x0, ic, jc, f, &bar);
            load_4d(p + L::oA, &tm_a, x0, ic - 1, jc, fs, &bar);
            load_4d(p + L::oBy, &tm_by, x0, ic, jc - 1, fs + 1, &bar);
            load_4d(p + L::oC, &tm_c, x0 - L::KO, ic, jc, fs + 2, &bar);
            load_4d(p + L::oF, &tm_f, x0 - L::KO, ic, jc - 2, fs + 3, &bar);
            load_4d(p + L::oE, &tm_e, x0 - L::KO, ic - 2, jc, fs + 4, &bar);
            load_4d(p + L::oD, &tm_d, x0, ic - 2, jc - 2, fs + 5, &bar);
        }
        limit = wait_limit(t.err);
    }
    const int k = T.k0 + tx, i = T.i0 + ty;
    const bool col_ok = k <= g.nz && i <= g.nx;
    // read while the tiles travel: the band signs of this thread's interior
    // cells, and the auxiliaries of its absorber cells (up to two cells: BJ
    // planes x M members)
    int sgn[BJ];
#pragma unroll
    for (int jj = 0; jj < BJ; jj++) {
        const int j = T.j0 + jj;
        const bool interior = i >= a.ibk && i <= a.iek && j >= a.jbk && j <= a.jek && k <= a.kek;
        sgn[jj] = (col_ok && interior && (a.mask & 1)) ? band_sign_of(a.band, col_index(g, i, j), k) : 0;
    }
    constexpr bool PRE = BJ * M <= 2;
    Aux9 xs[PRE ? M : 1][PRE ? BJ : 1];
    if (PRE && col_ok && (a.mask & 2)) {
#pragma unroll
        for (int mm = 0; mm < (PRE ? M : 1); mm++)
#pragma unroll
            for (int jj = 0; jj < (PRE ? BJ : 1); jj++) {
                const int j = T.j0 + jj;
                if (mm < T.nmem && j <= g.ny && !(i >= a.ibk && i <= a.iek && j >= a.jbk && j <= a.jek && k <= a.kek))
                    xs[mm][jj] = aux_load(a.aS, (long long)(T.m0 + mm) * t.ao, a.pmlcol, g, k, i, j);
            }
    }
    __syncthreads();   // barrier initialised, wait limit set
    if (!wait_tiles(&bar, t.err, limit) || !col_ok) return;   // the copy failed, or no cell of this launch here
#pragma unroll
    for (int mm = 0; mm < M; mm++) {
        if (mm >= T.nmem) break;
        const long long so = (long long)(T.m0 + mm) * t.so, ao = (long long)(T.m0 + mm) * t.ao;
#pragma unroll
        for (int jj = 0; jj < BJ; jj++) {
            const int j = T.j0 + jj;
            if (j > g.ny) break;
            const bool interior = i >= a.ibk && i <= a.iek && j >= a.jbk && j <= a.jek && k <= a.kek;
            if (!(a.mask & (interior ? 1 : 2))) continue;
            const SVelOps<BI, BJ, PREC> o{sm + L::oMem(mm), sm, tx, ty, jj, a};
            const long long e = col_index(g, i, j) * g.Kp + (k - 1 + KH);
            if (interior) {
                vel_interior<PREC>(a, o, sgn[jj], a.Vx + so, a.Vy + so, a.Vz + so, e);
            } else {
                const Aux9 x = PRE ? xs[PRE ? mm : 0][PRE ? jj : 0] : aux_load(a.aS, ao, a.pmlcol, g, k, i, j);
                vel_absorber<PREC>(a, o, x, k, i, j, e, ao, a.Vx + so, a.Vy + so, a.Vz + so);
            }
        }
    }
}

template <typename K>
cudaError_t smem_attr(K kernel, int bytes, unsigned long long &devices) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (devices >> dev & 1ull) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) devices |= 1ull << dev;
    return e;
}

inline const CUtensorMap &map(const unsigned char *p) { return *reinterpret_cast<const CUtensorMap *>(p); }

template <int NM, int BI, int BJ, int M, int PREC>
cudaError_t run_stress(const TmaMaps &m, const Str3Args &a, const TmaTiles &t, cudaStream_t st) {
    constexpr int bytes = StrBoxes<NM, BI, BJ, M, PREC>::total * 4 + 128;
    static unsigned long long devices = 0;   // devices on which the attribute is set
    cudaError_t e = smem_attr(stress3d_tma_kernel<NM, BI, BJ, M, PREC>, bytes, devices);
    if (e != cudaSuccess) return e;
    const unsigned nblk = (unsigned)((long long)t.nkt * t.nit * t.njt * t.mgroups);
    stress3d_tma_kernel<NM, BI, BJ, M, PREC><<<nblk, dim3(KT, BI, BJ), bytes, st>>>(map(m.state), map(m.s6),
                                                                                     map(m.med), map(m.vh), a, t);
    return cudaGetLastError();
}

template <int BI, int BJ, int M, int PREC>
cudaError_t run_vel(const TmaMaps &m, const Vel3Args &a, const TmaTiles &t, cudaStream_t st) {
    constexpr int bytes = VelBoxes<BI, BJ, M, PREC>::total * 4 + 128;
    static unsigned long long devices = 0;
    cudaError_t e = smem_attr(vel3d_tma_kernel<BI, BJ, M, PREC>, bytes, devices);
    if (e != cudaSuccess) return e;
    const unsigned nblk = (unsigned)((long long)t.nkt * t.nit * t.njt * t.mgroups);
    vel3d_tma_kernel<BI, BJ, M, PREC><<<nblk, dim3(KT, BI, 1), bytes, st>>>(map(m.own3), map(m.b3), map(m.va),
                                                                            map(m.vb), map(m.vc), map(m.vf),
                                                                            map(m.ve), map(m.vd), a, t);
    return cudaGetLastError();
}

template <int BI, int BJ, int M, int PREC = PREC_F32>
cudaError_t stress_nm(const TmaMaps &m, const Str3Args &a, const TmaTiles &t, int nm, cudaStream_t st) {
    switch (nm) {
    case 0: return run_stress<0, BI, BJ, M, PREC>(m, a, t, st);
    case 1: return run_stress<1, BI, BJ, M, PREC>(m, a, t, st);
    case 2: return run_stress<2, BI, BJ, M, PREC>(m, a, t, st);
    default: return run_stress<3, BI, BJ, M, PREC>(m, a, t, st);
    }
}

// compiled (bi, bj, members per CTA); the reduced storage forms run (4, 4) and
// (4, 2) with one member
constexpr int kStressShapes[][3] = {{4, 4, 1}, {2, 4, 1}, {4, 2, 1}, {4, 2, 2}, {2, 4, 2}, {2, 2, 2}, {2, 2, 4}, {4, 1, 4}};
constexpr int kVelShapes[][3] = {{4, 4, 1}, {4, 2, 1}, {2, 2, 1}, {4, 2, 2}, {2, 2, 2}, {4, 1, 2}, {2, 2, 4}, {4, 1, 4}};

}  // namespace

bool tma_shape_ok(int bi, int bj, int mpc, int prec) {
    if (prec != PREC_F32) return bi == 4 && (bj == 4 || bj == 2) && mpc == 1;
    for (auto &v : kStressShapes)
        if (v[0] == bi && v[1] == bj && v[2] == mpc) return true;
    return false;
}

bool tma_vel_shape_ok(int bi, int bj, int mpc, int prec) {
    if (prec != PREC_F32) return bi == 4 && (bj == 4 || bj == 2) && mpc == 1;
    for (auto &v : kVelShapes)
        if (v[0] == bi && v[1] == bj && v[2] == mpc) return true;
    return false;
}

cudaError_t launch_stress3d_tma(const TmaMaps &m, const Str3Args &a, const TmaTiles &t, int nm, int bi, int bj, int mpc,
                                cudaStream_t st, int prec) {
    if (prec == PREC_BF16_R)
        return bj == 2 ? stress_nm<4, 2, 1, PREC_BF16_R>(m, a, t, nm, st) : stress_nm<4, 4, 1, PREC_BF16_R>(m, a, t, nm, st);
    if (prec == PREC_F16_R)
        return bj == 2 ? stress_nm<4, 2, 1, PREC_F16_R>(m, a, t, nm, st) : stress_nm<4, 4, 1, PREC_F16_R>(m, a, t, nm, st);
    if (prec == PREC_F16_SR)
        return bj == 2 ? stress_nm<4, 2, 1, PREC_F16_SR>(m, a, t, nm, st) : stress_nm<4, 4, 1, PREC_F16_SR>(m, a, t, nm, st);
    if (mpc == 4) {
        if (bi == 4 && bj == 1) return stress_nm<4, 1, 4>(m, a, t, nm, st);
        return stress_nm<2, 2, 4>(m, a, t, nm, st);
    }
    if (mpc == 2) {
        if (bi == 2 && bj == 4) return stress_nm<2, 4, 2>(m, a, t, nm, st);
        if (bi == 2 && bj == 2) return stress_nm<2, 2, 2>(m, a, t, nm, st);
        return stress_nm<4, 2, 2>(m, a, t, nm, st);
    }
    if (bi == 2 && bj == 4) return stress_nm<2, 4, 1>(m, a, t, nm, st);
    if (bi == 4 && bj == 2) return stress_nm<4, 2, 1>(m, a, t, nm, st);
    return stress_nm<4, 4, 1>(m, a, t, nm, st);
}

cudaError_t launch_vel3d_tma(const TmaMaps &m, const Vel3Args &a, const TmaTiles &t, int bi, int bj, int mpc,
                             cudaStream_t st, int prec) {
    // BF16_R keeps S in FP32: its velocity update is the FP32 one
    if (prec == PREC_F16_SR)
        return bj == 2 ? run_vel<4, 2, 1, PREC_F16_SR>(m, a, t, st) : run_vel<4, 4, 1, PREC_F16_SR>(m, a, t, st);
    if (mpc == 4) {
        if (bi == 4 && bj == 1) return run_vel<4, 1, 4, PREC_F32>(m, a, t, st);
        return run_vel<2, 2, 4, PREC_F32>(m, a, t, st);
    }
    if (mpc == 2) {
        if (bi == 2 && bj == 2) return run_vel<2, 2, 2, PREC_F32>(m, a, t, st);
        if (bi == 4 && bj == 1) return run_vel<4, 1, 2, PREC_F32>(m, a, t, st);
        return run_vel<4, 2, 2, PREC_F32>(m, a, t, st);
    }
    if (bi == 4 && bj == 4) return run_vel<4, 4, 1, PREC_F32>(m, a, t, st);
    if (bi == 2 && bj == 2) return run_vel<2, 2, 1, PREC_F32>(m, a, t, st);
    return run_vel<4, 2, 1, PREC_F32>(m, a, t, st);
}

// ---------------------------------------------------------------------------
// tensor maps
// ---------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled encode_fn() {
    static PFN_cuTensorMapEncodeTiled fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(p);
    }
    return fn;
}

// 4D map (k, i, j, field) over a slab of nf fields with the given box;
// elements of 4 bytes (FP32) or 2 bytes (dtype BF16 / FP16).  The copies
// promote their L2 fills to 256-byte blocks: a box row (32 or 40 k values)
// and the start of the next k tile's row of the same column come in one fill
// (c1 step 27.27 against 27.40 ms with 128-byte fills; 64-byte fills 28.51 ms,
// none 27.40 ms).
static bool encode(unsigned char *out, void *slab, const Geo &g, long long nf, unsigned bk, unsigned bi, unsigned bj,
                   unsigned bf, CUtensorMapDataType dtype = CU_TENSOR_MAP_DATA_TYPE_FLOAT32) {
    PFN_cuTensorMapEncodeTiled fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t es = dtype == CU_TENSOR_MAP_DATA_TYPE_FLOAT32 ? 4 : 2;
    const cuuint64_t dims[4] = {(cuuint64_t)g.Kp, (cuuint64_t)g.Ip, (cuuint64_t)g.Jp, (cuuint64_t)nf};
    const cuuint64_t strides[3] = {(cuuint64_t)g.Kp * es, (cuuint64_t)g.Kp * g.Ip * es, (cuuint64_t)g.ncell * es};
    const cuuint32_t box[4] = {bk, bi, bj, bf};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = fn(reinterpret_cast<CUtensorMap *>(out), dtype, 4, slab, dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool tma_encode_box(unsigned char *out, float *slab, const Geo &g, long long nf, unsigned bk, unsigned bi, unsigned bj,
                    unsigned bf) {
    return encode(out, slab, g, nf, bk, bi, bj, bf);
}

bool tma_encode_stress(TmaMaps &m, const TmaSlabs &s, const Geo &g, int nm, int bi, int bj, int prec) {
    bool ok = encode(m.med, s.med, g, s.nf_med, KT, bi, bj, 7) &&
              encode(m.vh, s.state, g, s.nf_state, KB, bi + 4, bj + 4, 3);
    if (prec == PREC_BF16_R || prec == PREC_F16_R)   // S in the FP32 slab, R in the 2-byte slab
        return ok && encode(m.s6, s.state, g, s.nf_state, KT, bi, bj, 6) &&
               (nm == 0 || encode(m.state, s.half, g, s.nf_half, KT, bi, bj, 6 * nm,
                                  prec == PREC_BF16_R ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                      : CU_TENSOR_MAP_DATA_TYPE_FLOAT16));
    if (prec == PREC_F16_SR)   // S and R in the 2-byte slab
        return ok && encode(m.s6, s.half, g, s.nf_half, KT, bi, bj, 6, CU_TENSOR_MAP_DATA_TYPE_FLOAT16) &&
               encode(m.state, s.half, g, s.nf_half, KT, bi, bj, 6 + 6 * nm, CU_TENSOR_MAP_DATA_TYPE_FLOAT16);
    return ok && encode(m.state, s.state, g, s.nf_state, KT, bi, bj, 6 + 6 * nm) &&
           encode(m.s6, s.state, g, s.nf_state, KT, bi, bj, 6);
}

bool tma_encode_vel(TmaMaps &m, const TmaSlabs &s, const Geo &g, int bi, int bj, int prec) {
    const long long n = s.nf_state;
    bool ok = encode(m.own3, s.state, g, n, KT, bi, bj, 3) && encode(m.b3, s.med, g, s.nf_med, KT, bi, bj, 3);
    if (prec == PREC_F16_SR) {   // the stress boxes from the 2-byte slab, k halos from k0-8
        const CUtensorMapDataType h = CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
        const long long nh = s.nf_half;
        constexpr unsigned KS = KT + 16;
        return ok && encode(m.va, s.half, g, nh, KT, bi + 3, bj, 1, h) && encode(m.vb, s.half, g, nh, KT, bi, bj + 3, 1, h) &&
               encode(m.vc, s.half, g, nh, KS, bi, bj, 1, h) && encode(m.vf, s.half, g, nh, KS, bi, bj + 3, 1, h) &&
               encode(m.ve, s.half, g, nh, KS, bi + 3, bj, 1, h) &&
               encode(m.vd, s.half, g, nh, KT, bi + 3, bj + 3, 1, h);
    }
    return ok && encode(m.va, s.state, g, n, KT, bi + 3, bj, 1) && encode(m.vb, s.state, g, n, KT, bi, bj + 3, 1) &&
           encode(m.vc, s.state, g, n, KB, bi, bj, 1) && encode(m.vf, s.state, g, n, KB, bi, bj + 3, 1) &&
           encode(m.ve, s.state, g, n, KB, bi + 3, bj, 1) && encode(m.vd, s.state, g, n, KT, bi + 3, bj + 3, 1);
}

}  // namespace swpc
