// swpc3d_tma.cu -- the fused 3D stress and velocity updates with their
// operands staged in shared memory by TMA (kernel__update_stress /
// kernel__update_vel, src/swpc_3d/m_kernel.f90:75-326).
//
// The one-cell-per-thread kernels keep every operand of a cell in registers
// while its loads are in flight, so the register file bounds the bytes in
// flight per SM and the kernels stall on load latency below the HBM roofline.
// Here a CTA owns a tile of 32 (k) x BI (i) x BJ (j) cells and one thread
// issues two bulk tensor copies for the whole tile: the fields the update
// reads once (a box over consecutive fields of the context's field slab) and
// the stencil fields with their halos (the stress kernel: V over k-2..k+2,
// i-2..i+2, j-2..j+2; the velocity kernel: one box per stress component with
// the halo of its own difference, and each thread walks BJ planes of j).  The copies
// land in shared memory and complete on an mbarrier; several CTAs per SM keep
// well over a hundred KB per SM in flight without holding registers.  Each
// thread then updates its cell from shared memory with the arithmetic of the
// one-cell kernels (stress_interior / vel_interior, the same expression order),
// so the results are bitwise identical.  Absorber cells of a tile take the
// one-cell path (stress_cell / vel_cell); tiles without interior cells copy
// nothing.  The tensor boxes may reach past the grid at its edges: TMA fills
// those elements with zeros and they are never used.
//
// Slab field order (swpc_create): 0-2 V, 3-8 S, 9-15 lam mu taup taus muyz
// muxz muxy, 16.. R (component-major, nm per component), then bx by bz.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include "swpc3d_cell.cuh"
#include "swpc_tma.h"

namespace swpc {

namespace {

constexpr unsigned long long kWaitNs = 100000000ull;   // 100 ms: a tile copy takes microseconds

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_barrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned phase) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}
// tiled 4D tensor copy global -> shared, completion counted on bar (no multicast)
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *tm, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

// first 128-byte aligned address of the dynamic shared memory (TMA
// destinations); the launches reserve 128 bytes for the shift
__device__ __forceinline__ float *aligned128(unsigned char *p) {
    const unsigned a = smem_u32(p);
    return reinterpret_cast<float *>(p + ((128u - (a & 127u)) & 127u));
}

__device__ __forceinline__ unsigned long long gtime() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for the tile copies.  After kWaitNs the kernel raises the
// context's error word, waits once more (bounded) for its copies in flight,
// and the caller skips the staged cells; CTAs that start after the error
// copy nothing (see stage_begin).
__device__ __forceinline__ bool wait_tiles(uint64_t *bar, int *err) {
    const unsigned long long t0 = gtime();
    while (!mbar_try_wait(bar, 0)) {
        if (gtime() - t0 > kWaitNs) {
            atomicExch(err, 1);
            const unsigned long long t1 = gtime();
            while (!mbar_try_wait(bar, 0) && gtime() - t1 < kWaitNs) {
            }
            return false;
        }
    }
    return true;
}

// barrier set-up of a staged CTA; false when an earlier tile copy of the
// launch failed (nothing is copied then)
__device__ __forceinline__ bool stage_begin(uint64_t *bar, int *flag, const int *err, bool lead) {
    if (lead) {
        *flag = *reinterpret_cast<const volatile int *>(err) == 0;
        if (*flag) {
            mbar_init(bar, 1);
            fence_barrier_init();
        }
    }
    __syncthreads();
    return *flag != 0;
}

// tile of this CTA: k fastest, then i, then j
struct Tile {
    int k0, i0, j0;
};
template <int KT>
__device__ __forceinline__ Tile tile_of(const TmaTiles &t, int bi, int bj) {
    const int b = blockIdx.x;
    const int kt = b % t.nkt, it = (b / t.nkt) % t.nit, jt = b / (t.nkt * t.nit);
    return Tile{1 + KT * kt, 1 + bi * it, 1 + bj * jt};
}

__device__ __forceinline__ bool tile_has_interior(const Tile &T, int bi, int bj, int ibk, int iek, int jbk, int jek,
                                                  int kek) {
    return T.k0 <= kek && T.i0 <= iek && T.i0 + bi - 1 >= ibk && T.j0 <= jek && T.j0 + bj - 1 >= jbk;
}

// operands of the interior stress update in the staged tiles (tiles of KT
// cells along k; a halo box spans k0-4 .. k0+KT+3, KT + 8 cells, so that its
// start stays 16-byte aligned)
template <int NM, int KT, int BI, int BJ>
struct SStrOps {
    const float *ss;   // [13 + 6 NM][BJ][BI][KT]: S xx..xy, lam mu taup taus muyz muxz muxy, R
    const float *sv;   // [3][BJ+4][BI+4][KT+8]: Vx Vy Vz around the tile
    int tx, ty, tz;
    __device__ __forceinline__ float own(int f) const { return ss[((f * BJ + tz) * BI + ty) * KT + tx]; }
    __device__ __forceinline__ float v(int c, int dk, int di, int dj) const {
        return sv[((c * (BJ + 4) + tz + 2 + dj) * (BI + 4) + ty + 2 + di) * (KT + 8) + tx + 4 + dk];
    }
    __device__ __forceinline__ float sown(int f) const { return own(f); }
    __device__ __forceinline__ float r(int q) const { return own(13 + (q / 3) * NM + q % 3); }
    // 0 mu, 1 lam, 2 taup, 3 taus, 4 muyz, 5 muxz, 6 muxy (slab order lam mu taup taus muyz muxz muxy)
    __device__ __forceinline__ float med(int m) const { return own(m == 0 ? 7 : m == 1 ? 6 : 6 + m); }
};

// Velocity tiles: own V and b, and one box per stress component with only the
// halo its difference needs: Sxx i-1..i+2, Syy j-1..j+2, Szz k-1..k+2,
// Syz j-2..j+1 / k-2..k+1, Sxz i-2..i+1 / k-2..k+1, Sxy i-2..i+1 / j-2..j+1.
// Offsets in floats, each a multiple of 32 floats (128-byte TMA destinations).
__host__ __device__ constexpr int up32(int n) { return (n + 31) / 32 * 32; }
template <int KT, int BI, int BJ>
struct VelBoxes {
    static constexpr int KB = KT + 8;
    static constexpr int own = 3 * BJ * BI * KT;                 // V, then b
    static constexpr int nA = (BJ) * (BI + 3) * KT;              // Sxx
    static constexpr int nB = (BJ + 3) * (BI) * KT;              // Syy
    static constexpr int nC = (BJ) * (BI) * KB;                  // Szz
    static constexpr int nF = (BJ + 3) * (BI) * KB;              // Syz
    static constexpr int nE = (BJ) * (BI + 3) * KB;              // Sxz
    static constexpr int nD = (BJ + 3) * (BI + 3) * KT;          // Sxy
    static constexpr int oV = 0, oB = own, oA = 2 * own, oBy = up32(oA + nA), oC = up32(oBy + nB),
                         oF = up32(oC + nC), oE = up32(oF + nF), oD = up32(oE + nE), total = up32(oD + nD);
    static constexpr int bytes = 4 * (2 * own + nA + nB + nC + nF + nE + nD);   // copied bytes
};

template <int KT, int BI, int BJ>
struct SVelOps {
    const float *sm;
    int tx, ty, jj;
    using L = VelBoxes<KT, BI, BJ>;
    static constexpr int KB = L::KB;
    __device__ __forceinline__ float v(int c) const { return sm[L::oV + ((c * BJ + jj) * BI + ty) * KT + tx]; }
    __device__ __forceinline__ float b(int c) const { return sm[L::oB + ((c * BJ + jj) * BI + ty) * KT + tx]; }
    __device__ __forceinline__ float s(int f, int dk, int di, int dj) const {
        switch (f) {
        case 0: return sm[L::oA + (jj * (BI + 3) + ty + 1 + di) * KT + tx];
        case 1: return sm[L::oBy + ((jj + 1 + dj) * BI + ty) * KT + tx];
        case 2: return sm[L::oC + (jj * BI + ty) * KB + tx + 4 + dk];
        case 3: return sm[L::oF + ((jj + 2 + dj) * BI + ty) * KB + tx + 4 + dk];
        case 4: return sm[L::oE + (jj * (BI + 3) + ty + 2 + di) * KB + tx + 4 + dk];
        default: return sm[L::oD + ((jj + 2 + dj) * (BI + 3) + ty + 2 + di) * KT + tx];
        }
    }
};

template <int NM, int KT, int BI, int BJ>
__host__ __device__ constexpr int stress_smem_floats() {
    return (13 + 6 * NM) * BJ * BI * KT + 3 * (BJ + 4) * (BI + 4) * (KT + 8);
}
template <int SMEM_FLOATS, int THREADS>
__host__ __device__ constexpr int blocks_per_sm() {
    constexpr int by_smem = (227 * 1024) / (SMEM_FLOATS * 4 + 128 + 1024);
    constexpr int by_threads = 1024 / THREADS;   // at least 64 registers a thread
    constexpr int n = by_smem < by_threads ? by_smem : by_threads;
    return n < 1 ? 1 : n;
}

template <int NM, int KT, int BI, int BJ>
__global__ void __launch_bounds__(KT * BI * BJ, (blocks_per_sm<stress_smem_floats<NM, KT, BI, BJ>(), KT * BI * BJ>()))
    stress3d_tma_kernel(const __grid_constant__ CUtensorMap tm_str, const __grid_constant__ CUtensorMap tm_v,
                        const Str3Args a, const TmaTiles t) {
    constexpr int NF = 13 + 6 * NM;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ __align__(8) uint64_t bar;
    float *sm = aligned128(smraw);
    float *ss = sm;
    float *sv = sm + NF * BJ * BI * KT;
    const Geo g = a.g;
    const Tile T = tile_of<KT>(t, BI, BJ);
    const int tx = threadIdx.x, ty = threadIdx.y, tz = threadIdx.z;
    const bool lead = tx == 0 && ty == 0 && tz == 0;
    const bool staged = (a.mask & 1) && tile_has_interior(T, BI, BJ, a.ibk, a.iek, a.jbk, a.jek, a.kek);
    __shared__ int go;
    bool ok = true;
    if (staged && !stage_begin(&bar, &go, t.err, lead)) ok = false;
    else if (staged) {
        if (lead) {
            mbar_expect_tx(&bar, (unsigned)(stress_smem_floats<NM, KT, BI, BJ>() * 4));
            const int x0 = T.k0 - 1 + KH;
            tma_load_4d(ss, &tm_str, x0, T.i0 + 2, T.j0 + 2, 3, &bar);
            tma_load_4d(sv, &tm_v, x0 - 4, T.i0, T.j0, 0, &bar);
        }
        ok = wait_tiles(&bar, t.err);
    }
    const int k = T.k0 + tx, i = T.i0 + ty, j = T.j0 + tz;
    if (k > g.nz || i > g.nx || j > g.ny) return;
    if (!(i >= a.ibk && i <= a.iek && j >= a.jbk && j <= a.jek && k <= a.kek)) {
        stress_cell<NM, PREC_F32>(a, k, i, j);   // absorber cell
        return;
    }
    if (!staged || !ok) return;   // interior cells not in this launch (mask), or the copy failed
    const SStrOps<NM, KT, BI, BJ> o{ss, sv, tx, ty, tz};
    const long long col = col_index(g, i, j);
    const long long e = col * g.Kp + (k - 1 + KH);
    float *const Sp[6] = {a.Sxx, a.Syy, a.Szz, a.Syz, a.Sxz, a.Sxy};
    stress_interior<NM, PREC_F32>(a, o, band_sign_of(a.band, col, k), Sp, e, 0);
}

// One CTA per tile of KT x BI x BJ cells with KT x BI threads; each thread
// updates its (k, i) for the BJ planes j0 .. j0+BJ-1.
template <int KT, int BI, int BJ>
__global__ void __launch_bounds__(KT * BI, (blocks_per_sm<VelBoxes<KT, BI, BJ>::total, KT * BI>()))
    vel3d_tma_kernel(const __grid_constant__ CUtensorMap tm_own, const __grid_constant__ CUtensorMap tm_a,
                     const __grid_constant__ CUtensorMap tm_b, const __grid_constant__ CUtensorMap tm_c,
                     const __grid_constant__ CUtensorMap tm_f, const __grid_constant__ CUtensorMap tm_e,
                     const __grid_constant__ CUtensorMap tm_d, const Vel3Args a, const TmaTiles t) {
    using L = VelBoxes<KT, BI, BJ>;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int go;
    float *sm = aligned128(smraw);
    const Geo g = a.g;
    const Tile T = tile_of<KT>(t, BI, BJ);
    const int tx = threadIdx.x, ty = threadIdx.y;
    const bool lead = tx == 0 && ty == 0;
    const bool staged = (a.mask & 1) && tile_has_interior(T, BI, BJ, a.ibk, a.iek, a.jbk, a.jek, a.kek);
    bool ok = true;
    if (staged && !stage_begin(&bar, &go, t.err, lead)) ok = false;
    else if (staged) {
        if (lead) {
            mbar_expect_tx(&bar, (unsigned)L::bytes);
            const int x0 = T.k0 - 1 + KH, ic = T.i0 + 2, jc = T.j0 + 2;
            tma_load_4d(sm + L::oV, &tm_own, x0, ic, jc, 0, &bar);
            tma_load_4d(sm + L::oB, &tm_own, x0, ic, jc, t.b_field, &bar);
            tma_load_4d(sm + L::oA, &tm_a, x0, ic - 1, jc, 3, &bar);
            tma_load_4d(sm + L::oBy, &tm_b, x0, ic, jc - 1, 4, &bar);
            tma_load_4d(sm + L::oC, &tm_c, x0 - 4, ic, jc, 5, &bar);
            tma_load_4d(sm + L::oF, &tm_f, x0 - 4, ic, jc - 2, 6, &bar);
            tma_load_4d(sm + L::oE, &tm_e, x0 - 4, ic - 2, jc, 7, &bar);
            tma_load_4d(sm + L::oD, &tm_d, x0, ic - 2, jc - 2, 8, &bar);
        }
        ok = wait_tiles(&bar, t.err);
    }
    const int k = T.k0 + tx, i = T.i0 + ty;
    if (k > g.nz || i > g.nx) return;
#pragma unroll 1
    for (int jj = 0; jj < BJ; jj++) {
        const int j = T.j0 + jj;
        if (j > g.ny) break;
        if (!(i >= a.ibk && i <= a.iek && j >= a.jbk && j <= a.jek && k <= a.kek)) {
            vel_cell<PREC_F32>(a, k, i, j);   // absorber cell
            continue;
        }
        if (!staged || !ok) continue;   // interior cells not in this launch (mask), or the copy failed
        const SVelOps<KT, BI, BJ> o{sm, tx, ty, jj};
        const long long col = col_index(g, i, j);
        const long long e = col * g.Kp + (k - 1 + KH);
        vel_interior<PREC_F32>(a, o, band_sign_of(a.band, col, k), a.Vx, a.Vy, a.Vz, e);
    }
}

template <int NM, int KT, int BI, int BJ>
cudaError_t run_stress(const TmaMaps &m, const Str3Args &a, const TmaTiles &t, cudaStream_t st) {
    constexpr int bytes = stress_smem_floats<NM, KT, BI, BJ>() * 4 + 128;
    static unsigned long long devices = 0;   // devices on which the attribute is set
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(devices >> dev & 1ull)) {
        cudaError_t e = cudaFuncSetAttribute(stress3d_tma_kernel<NM, KT, BI, BJ>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) return e;
        devices |= 1ull << dev;
    }
    const unsigned nblk = (unsigned)((long long)t.nkt * t.nit * t.njt);
    stress3d_tma_kernel<NM, KT, BI, BJ><<<nblk, dim3(KT, BI, BJ), bytes, st>>>(
        *reinterpret_cast<const CUtensorMap *>(m.str), *reinterpret_cast<const CUtensorMap *>(m.v3h), a, t);
    return cudaGetLastError();
}

template <int KT, int BI, int BJ>
cudaError_t run_vel(const TmaMaps &m, const Vel3Args &a, const TmaTiles &t, cudaStream_t st) {
    constexpr int bytes = VelBoxes<KT, BI, BJ>::total * 4 + 128;
    static unsigned long long devices = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(devices >> dev & 1ull)) {
        cudaError_t e = cudaFuncSetAttribute(vel3d_tma_kernel<KT, BI, BJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             bytes);
        if (e != cudaSuccess) return e;
        devices |= 1ull << dev;
    }
    const unsigned nblk = (unsigned)((long long)t.nkt * t.nit * t.njt);
    auto M = [&](const unsigned char *p) { return *reinterpret_cast<const CUtensorMap *>(p); };
    vel3d_tma_kernel<KT, BI, BJ><<<nblk, dim3(KT, BI, 1), bytes, st>>>(M(m.own3), M(m.va), M(m.vb), M(m.vc), M(m.vf),
                                                                       M(m.ve), M(m.vd), a, t);
    return cudaGetLastError();
}

template <int KT, int BI, int BJ>
cudaError_t stress_nm(const TmaMaps &m, const Str3Args &a, const TmaTiles &t, int nm, cudaStream_t st) {
    switch (nm) {
    case 0: return run_stress<0, KT, BI, BJ>(m, a, t, st);
    case 1: return run_stress<1, KT, BI, BJ>(m, a, t, st);
    case 2: return run_stress<2, KT, BI, BJ>(m, a, t, st);
    default: return run_stress<3, KT, BI, BJ>(m, a, t, st);
    }
}

}  // namespace

// tile shapes (k extent, i, j) with compiled kernels
bool tma_shape_ok(int kt, int bi, int bj) {
    const int s[][3] = {{32, 4, 4}, {32, 2, 4}, {32, 4, 2}, {64, 4, 2}, {64, 2, 2}, {64, 2, 4}, {64, 4, 1}};
    for (auto &v : s)
        if (v[0] == kt && v[1] == bi && v[2] == bj) return true;
    return false;
}

bool tma_vel_shape_ok(int kt, int bi, int bj) {
    const int s[][3] = {{32, 4, 2}, {32, 4, 4}, {32, 2, 2}, {64, 4, 2}, {64, 2, 2}, {64, 4, 1}, {64, 2, 4}, {64, 4, 4}};
    for (auto &v : s)
        if (v[0] == kt && v[1] == bi && v[2] == bj) return true;
    return false;
}

cudaError_t launch_stress3d_tma(const TmaMaps &m, const Str3Args &a, const TmaTiles &t, int nm, int kt, int bi, int bj,
                                cudaStream_t st) {
    if (kt == 64) {
        if (bi == 2 && bj == 2) return stress_nm<64, 2, 2>(m, a, t, nm, st);
        if (bi == 2 && bj == 4) return stress_nm<64, 2, 4>(m, a, t, nm, st);
        if (bi == 4 && bj == 1) return stress_nm<64, 4, 1>(m, a, t, nm, st);
        return stress_nm<64, 4, 2>(m, a, t, nm, st);
    }
    if (bi == 2 && bj == 4) return stress_nm<32, 2, 4>(m, a, t, nm, st);
    if (bi == 4 && bj == 2) return stress_nm<32, 4, 2>(m, a, t, nm, st);
    return stress_nm<32, 4, 4>(m, a, t, nm, st);
}

cudaError_t launch_vel3d_tma(const TmaMaps &m, const Vel3Args &a, const TmaTiles &t, int kt, int bi, int bj,
                             cudaStream_t st) {
    if (kt == 64) {
        if (bi == 2 && bj == 2) return run_vel<64, 2, 2>(m, a, t, st);
        if (bi == 4 && bj == 1) return run_vel<64, 4, 1>(m, a, t, st);
        if (bi == 2 && bj == 4) return run_vel<64, 2, 4>(m, a, t, st);
        if (bi == 4 && bj == 4) return run_vel<64, 4, 4>(m, a, t, st);
        return run_vel<64, 4, 2>(m, a, t, st);
    }
    if (bi == 4 && bj == 4) return run_vel<32, 4, 4>(m, a, t, st);
    if (bi == 2 && bj == 2) return run_vel<32, 2, 2>(m, a, t, st);
    return run_vel<32, 4, 2>(m, a, t, st);
}

// ---------------------------------------------------------------------------
// tensor maps over the field slab
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

// 4D map (k, i, j, field) over the slab with the given box
static bool encode(void *out, float *slab, const Geo &g, int nf, unsigned bk, unsigned bi, unsigned bj, unsigned bf) {
    PFN_cuTensorMapEncodeTiled fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)g.Kp, (cuuint64_t)g.Ip, (cuuint64_t)g.Jp, (cuuint64_t)nf};
    const cuuint64_t strides[3] = {(cuuint64_t)g.Kp * 4, (cuuint64_t)g.Kp * g.Ip * 4, (cuuint64_t)g.ncell * 4};
    const cuuint32_t box[4] = {bk, bi, bj, bf};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = fn(reinterpret_cast<CUtensorMap *>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, slab, dims, strides,
                          box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool tma_encode_stress(TmaMaps &m, float *slab, const Geo &g, int nf, int nm, int kt, int bi, int bj) {
    return encode(m.str, slab, g, nf, kt, bi, bj, 13 + 6 * nm) &&
           encode(m.v3h, slab, g, nf, kt + 8, bi + 4, bj + 4, 3);
}

bool tma_encode_vel(TmaMaps &m, float *slab, const Geo &g, int nf, int kt, int bi, int bj) {
    const unsigned kb = kt + 8;
    return encode(m.own3, slab, g, nf, kt, bi, bj, 3) && encode(m.va, slab, g, nf, kt, bi + 3, bj, 1) &&
           encode(m.vb, slab, g, nf, kt, bi, bj + 3, 1) && encode(m.vc, slab, g, nf, kb, bi, bj, 1) &&
           encode(m.vf, slab, g, nf, kb, bi, bj + 3, 1) && encode(m.ve, slab, g, nf, kb, bi + 3, bj, 1) &&
           encode(m.vd, slab, g, nf, kt, bi + 3, bj + 3, 1);
}

}  // namespace swpc
