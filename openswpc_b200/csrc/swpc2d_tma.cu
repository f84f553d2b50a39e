// swpc2d_tma.cu -- the 2D P-SV and SH stress and velocity updates with their
// operands staged in shared memory by TMA (kernel__update_stress /
// kernel__update_vel with absorb_p__update_stress / absorb_p__update_vel of
// src/swpc_psv and src/swpc_sh).
//
// One CTA per tile of 32 (k) x 16 (i) cells of one model; a batch of models
// of uneven size is one tile list over all of them (Tile2D: model, first
// cell, and whether the tile holds interior and absorber cells).  The lead
// thread issues one bulk tensor copy per box through the model's tensor maps,
// which travel as a kernel parameter (one model for a single run, a group of
// up to kGroup2D models per launch for a batch); the other threads meanwhile
// copy the model descriptor into shared memory.  The boxes:
//   stress: S and R (S alone in tiles without interior cells), the medium of
//           the cells, mu over k..k+1 / i..i+1 (the averaged rigidities) and
//           V over k-2..k+2 / i-2..i+2;
//   velocity: V, rho over k..k+1 / i..i+1 (P-SV buoyancies; SH reads its own
//           cell), and one box per stress component with the halo of its own
//           difference.
// Each thread then updates RI = 16 / TI rows of its k column from shared
// memory with the arithmetic of swpc2d_cell.cuh, so the results are bitwise
// those of the tile-walking kernels and of the oracle.  The boxes may reach
// past the grid at its edges: TMA fills those elements with zeros and they
// are never used.
//
// Field order of a 2D model's slab (see create_2d): V (P-SV Vx Vz, SH Vy),
// S (P-SV Sxx Szz Sxz, SH Syz Sxy), R (component-major, nm per component),
// then lam taup taus mu rho.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>
#include <string.h>

#include "swpc2d.cuh"
#include "swpc2d_cell.cuh"
#include "swpc_tma_ptx.cuh"

namespace swpc {

namespace {

using namespace tma;

constexpr int KT = 32;        // tile extent along k
constexpr int BI = kTileI2D;  // tile extent along i
constexpr int KB = KT + 8;    // k extent of a box over k0-4 .. k0+35 (16-byte aligned start)
constexpr int KM = KT + 4;    // k extent of a box over k0 .. k0+35 (mu, rho)

// tensor-map slots of a model's stress and velocity sets (MapSet2D)
enum { ST_STATE, ST_S, ST_MED, ST_MU, ST_V };
enum { VE_OWN, VE_RHO, VE_A, VE_C, VE_E };

// the maps of the G models of a launch (kernel parameter)
template <int G>
struct MapGroup {
    MapSet2D set[G];
};

__device__ __forceinline__ const CUtensorMap *set_maps(const MapSet2D &s) {
    return reinterpret_cast<const CUtensorMap *>(&s);
}

// the block's copy of the model descriptor
__device__ __forceinline__ void copy_model(const Model2D *__restrict__ models, int model, Model2D &sM) {
    const int nw = (int)(sizeof(Model2D) / sizeof(int));
    const int *src = reinterpret_cast<const int *>(models + model);
    int *dst = reinterpret_cast<int *>(&sM);
    for (int w = threadIdx.y * blockDim.x + threadIdx.x; w < nw; w += blockDim.x * blockDim.y) dst[w] = __ldg(src + w);
}

// ---------------------------------------------------------------------------
// shared-memory layouts (floats) and operand sources
// ---------------------------------------------------------------------------
// stress: state [NS + NS NM][BI][KT] (S, R), medium [NMED][BI][KT], mu
// [BI+1][KM], V [NV][BI+4][KB]
template <int KIND, int NM>
struct StrBox {
    static constexpr int NV = KIND == 0 ? 2 : 1, NS = KIND == 0 ? 3 : 2, NMED = KIND == 0 ? 3 : 1;
    static constexpr int nState = (NS + NS * NM) * BI * KT, nS = NS * BI * KT, nMed = NMED * BI * KT;
    static constexpr int nMu = (BI + 1) * KM, nV = NV * (BI + 4) * KB;
    static constexpr int oState = 0, oMed = up32(nState), oMu = oMed + up32(nMed), oV = oMu + up32(nMu);
    static constexpr int total = oV + up32(nV);
    __host__ __device__ static constexpr unsigned bytes(bool with_r) {
        return 4u * (unsigned)((with_r ? nState : nS) + nMed + nMu + nV);
    }
};

template <int KIND, int NM>
struct SStr2 {
    using L = StrBox<KIND, NM>;
    const float *sm;
    int row, tx;
    __device__ __forceinline__ int at(int f) const { return (f * BI + row) * KT + tx; }
    __device__ __forceinline__ float s(int c) const { return sm[L::oState + at(c)]; }
    __device__ __forceinline__ float r(int c, int m) const { return sm[L::oState + at(L::NS + c * NM + m)]; }
    // P-SV medium box: lam taup taus; SH: taus
    __device__ __forceinline__ float lam() const { return sm[L::oMed + at(0)]; }
    __device__ __forceinline__ float taup() const { return sm[L::oMed + at(1)]; }
    __device__ __forceinline__ float taus() const { return sm[L::oMed + at(KIND == 0 ? 2 : 0)]; }
    __device__ __forceinline__ float mu(int dk, int di) const { return sm[L::oMu + (row + di) * KM + tx + dk]; }
    __device__ __forceinline__ float v(int c, int dk, int di) const {
        return sm[L::oV + (c * (BI + 4) + row + 2 + di) * KB + tx + 4 + dk];
    }
};

// velocity: V [NV][BI][KT], rho (P-SV [BI+1][KM], SH [BI][KT]), and
//   P-SV: Sxx [BI+3][KT] over i-1..i+2, Szz [BI][KB] over k-1..k+2 (box
//         k0-4 ..), Sxz [BI+3][KB] over i-2..i+1 / k-2..k+1;
//   SH:   Sxy [BI+3][KT] over i-2..i+1, Syz [BI][KB] over k-2..k+1.
template <int KIND>
struct VelBox {
    static constexpr int NV = KIND == 0 ? 2 : 1;
    static constexpr int nOwn = NV * BI * KT, nRho = KIND == 0 ? (BI + 1) * KM : BI * KT;
    static constexpr int nA = (BI + 3) * KT, nC = BI * KB, nE = KIND == 0 ? (BI + 3) * KB : 0;
    static constexpr int oOwn = 0, oRho = up32(nOwn), oA = oRho + up32(nRho), oC = oA + up32(nA), oE = oC + up32(nC);
    static constexpr int total = oE + up32(nE);
    __host__ __device__ static constexpr unsigned bytes() { return 4u * (unsigned)(nOwn + nRho + nA + nC + nE); }
};

template <int KIND>
struct SVel2 {
    using L = VelBox<KIND>;
    const float *sm;
    int row, tx;
    __device__ __forceinline__ float vown(int c) const { return sm[L::oOwn + (c * BI + row) * KT + tx]; }
    __device__ __forceinline__ float rho(int dk, int di) const {
        return KIND == 0 ? sm[L::oRho + (row + di) * KM + tx + dk] : sm[L::oRho + row * KT + tx];
    }
    __device__ __forceinline__ float sn(int c, int dk, int di) const {
        if (KIND == 0) {
            if (c == 0) return sm[L::oA + (row + 1 + di) * KT + tx];                // Sxx
            if (c == 1) return sm[L::oC + row * KB + tx + 4 + dk];                  // Szz
            return sm[L::oE + (row + 2 + di) * KB + tx + 4 + dk];                   // Sxz
        }
        if (c == 0) return sm[L::oC + row * KB + tx + 4 + dk];                      // Syz
        return sm[L::oA + (row + 2 + di) * KT + tx];                                // Sxy
    }
};

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
template <int KIND, int NM, int TI, int G>
__global__ void __launch_bounds__(32 * TI) stress2d_tma_kernel(const __grid_constant__ MapGroup<G> pm, int model0,
                                                               const Model2D *__restrict__ models,
                                                               const Tile2D *__restrict__ tiles, int mask,
                                                               Fields2D f, int *err) {
    using L = StrBox<KIND, NM>;
    constexpr int RI = BI / TI;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ Model2D sM;
    __shared__ __align__(8) uint64_t bar;
    __shared__ unsigned long long limit;
    float *sm = aligned128(smraw);
    const Tile2D tl = tiles[blockIdx.x];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const bool lead = tx == 0 && ty == 0;
    // interior cells need S, R and the medium, absorber cells S and the medium
    const bool with_r = (mask & 1) && (tl.flags & kTileInterior);
    if (!with_r && !((mask & 2) && (tl.flags & kTileAbsorber))) return;   // nothing of this launch here
    if (lead) {
        // the copies go out first; the error word is read while they travel
        stage_init(&bar, L::bytes(with_r));
        const CUtensorMap *mp = set_maps(pm.set[tl.model - model0]);
        const int x0 = tl.k0 - 1 + KH, ic = tl.i0 + 2;
        load_3d(sm + L::oState, with_r ? &mp[ST_STATE] : &mp[ST_S], x0, ic, f.s, &bar);
        load_3d(sm + L::oMed, &mp[ST_MED], x0, ic, KIND == 0 ? f.med : f.med + 2, &bar);   // lam taup taus / taus
        load_3d(sm + L::oMu, &mp[ST_MU], x0, ic, f.med + 3, &bar);
        load_3d(sm + L::oV, &mp[ST_V], x0 - 4, ic - 2, f.v, &bar);
        limit = wait_limit(err);
    }
    copy_model(models, tl.model, sM);
    __syncthreads();   // barrier initialised, wait limit and model descriptor set
    const Model2D &M = sM;
    // the band signs of this thread's cells are read while the tiles travel
    int sg[RI];
#pragma unroll
    for (int r = 0; r < RI; r++) {
        const int k = tl.k0 + tx, i = tl.i0 + ty + r * TI;
        const bool interior = i >= M.ibk && i <= M.iek && k <= M.kek;
        sg[r] = (interior && k <= M.nz && (mask & 1)) ? band_sign2d(M, k, i) : -1;
    }
    if (!wait_tiles(&bar, err, limit)) return;   // the copy did not complete
#pragma unroll
    for (int r = 0; r < RI; r++) {
        const int row = ty + r * TI;
        const int k = tl.k0 + tx, i = tl.i0 + row;
        if (k > M.nz || i > M.nx) continue;
        const bool interior = i >= M.ibk && i <= M.iek && k <= M.kek;
        if (!(mask & (interior ? 1 : 2))) continue;
        const long long e = (long long)(i + 2) * M.Kp + (k - 1 + KH);
        const SStr2<KIND, NM> o{sm, row, tx};
        const int s = sg[r];
        if (KIND == 0) {
            if (interior) psv_stress_interior<NM>(M, o, s, e);
            else psv_stress_absorber(M, o, k, i, e);
        } else {
            sh_stress_cell<NM>(M, o, k, i, e, s);
        }
    }
}

template <int KIND, int TI, int G>
__global__ void __launch_bounds__(32 * TI) vel2d_tma_kernel(const __grid_constant__ MapGroup<G> pm, int model0,
                                                            const Model2D *__restrict__ models,
                                                            const Tile2D *__restrict__ tiles, int mask, Fields2D f,
                                                            int *err) {
    using L = VelBox<KIND>;
    constexpr int RI = BI / TI;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ Model2D sM;
    __shared__ __align__(8) uint64_t bar;
    __shared__ unsigned long long limit;
    float *sm = aligned128(smraw);
    const Tile2D tl = tiles[blockIdx.x];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const bool lead = tx == 0 && ty == 0;
    if (!((mask & 1) && (tl.flags & kTileInterior)) && !((mask & 2) && (tl.flags & kTileAbsorber))) return;
    if (lead) {
        // the copies go out first; the error word is read while they travel
        stage_init(&bar, L::bytes());
        const CUtensorMap *mp = set_maps(pm.set[tl.model - model0]);
        const int x0 = tl.k0 - 1 + KH, ic = tl.i0 + 2;
        load_3d(sm + L::oOwn, &mp[VE_OWN], x0, ic, f.v, &bar);
        load_3d(sm + L::oRho, &mp[VE_RHO], x0, ic, f.med + 4, &bar);
        if (KIND == 0) {
            load_3d(sm + L::oA, &mp[VE_A], x0, ic - 1, f.s, &bar);            // Sxx
            load_3d(sm + L::oC, &mp[VE_C], x0 - 4, ic, f.s + 1, &bar);        // Szz
            load_3d(sm + L::oE, &mp[VE_E], x0 - 4, ic - 2, f.s + 2, &bar);    // Sxz
        } else {
            load_3d(sm + L::oA, &mp[VE_A], x0, ic - 2, f.s + 1, &bar);        // Sxy
            load_3d(sm + L::oC, &mp[VE_C], x0 - 4, ic, f.s, &bar);            // Syz
        }
        limit = wait_limit(err);
    }
    copy_model(models, tl.model, sM);
    __syncthreads();   // barrier initialised, wait limit and model descriptor set
    const Model2D &M = sM;
    // the band signs of this thread's cells are read while the tiles travel
    int sg[RI];
#pragma unroll
    for (int r = 0; r < RI; r++) {
        const int k = tl.k0 + tx, i = tl.i0 + ty + r * TI;
        const bool interior = i >= M.ibk && i <= M.iek && k <= M.kek;
        sg[r] = (interior && k <= M.nz && (mask & 1)) ? band_sign2d(M, k, i) : -1;
    }
    if (!wait_tiles(&bar, err, limit)) return;   // the copy did not complete
#pragma unroll
    for (int r = 0; r < RI; r++) {
        const int row = ty + r * TI;
        const int k = tl.k0 + tx, i = tl.i0 + row;
        if (k > M.nz || i > M.nx) continue;
        const bool interior = i >= M.ibk && i <= M.iek && k <= M.kek;
        if (!(mask & (interior ? 1 : 2))) continue;
        const long long e = (long long)(i + 2) * M.Kp + (k - 1 + KH);
        const SVel2<KIND> o{sm, row, tx};
        const int s = sg[r];
        if (KIND == 0) psv_vel_cell(M, o, k, i, e, s);
        else sh_vel_cell(M, o, k, i, e, s);
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

// A launch's maps: nset models from model0 (nset = 1: a single run; up to
// kGroup2D: a group of a batch), copied into the kernel parameter.
struct MapArgs {
    const MapSet2D *sets;
    int nset, model0;
};

template <int G>
MapGroup<G> group_of(const MapArgs &ma) {
    MapGroup<G> g;
    memset(&g, 0, sizeof(g));
    for (int q = 0; q < ma.nset && q < G; q++) g.set[q] = ma.sets[q];
    return g;
}

template <int KIND, int NM, int TI, int G>
cudaError_t run_stress(const MapArgs &ma, const Model2D *models, const Tile2D *tiles, int ntiles, int mask,
                       Fields2D f, int *err, cudaStream_t st) {
    constexpr int bytes = StrBox<KIND, NM>::total * 4 + 128;
    static unsigned long long devices = 0;
    cudaError_t e = smem_attr(stress2d_tma_kernel<KIND, NM, TI, G>, bytes, devices);
    if (e != cudaSuccess) return e;
    stress2d_tma_kernel<KIND, NM, TI, G><<<ntiles, dim3(32, TI), bytes, st>>>(group_of<G>(ma), ma.model0, models, tiles,
                                                                              mask, f, err);
    return cudaGetLastError();
}

template <int KIND, int TI, int G>
cudaError_t run_vel(const MapArgs &ma, const Model2D *models, const Tile2D *tiles, int ntiles, int mask,
                    Fields2D f, int *err, cudaStream_t st) {
    constexpr int bytes = VelBox<KIND>::total * 4 + 128;
    static unsigned long long devices = 0;
    cudaError_t e = smem_attr(vel2d_tma_kernel<KIND, TI, G>, bytes, devices);
    if (e != cudaSuccess) return e;
    vel2d_tma_kernel<KIND, TI, G><<<ntiles, dim3(32, TI), bytes, st>>>(group_of<G>(ma), ma.model0, models, tiles, mask,
                                                                       f, err);
    return cudaGetLastError();
}

template <int KIND, int NM, int TI>
cudaError_t stress_g(const MapArgs &ma, const Model2D *models, const Tile2D *tiles, int ntiles, int mask, Fields2D f,
                     int *err, cudaStream_t st) {
    if (ma.nset > 1) return run_stress<KIND, NM, TI, kGroup2D>(ma, models, tiles, ntiles, mask, f, err, st);
    return run_stress<KIND, NM, TI, 1>(ma, models, tiles, ntiles, mask, f, err, st);
}

template <int KIND, int NM>
cudaError_t stress_ti(int ti, const MapArgs &ma, const Model2D *models, const Tile2D *tiles, int ntiles, int mask,
                      Fields2D f, int *err, cudaStream_t st) {
    if (ti == 4) return stress_g<KIND, NM, 4>(ma, models, tiles, ntiles, mask, f, err, st);
    if (ti == 16) return stress_g<KIND, NM, 16>(ma, models, tiles, ntiles, mask, f, err, st);
    return stress_g<KIND, NM, 8>(ma, models, tiles, ntiles, mask, f, err, st);
}

template <int KIND>
cudaError_t stress_nm(int nm, int ti, const MapArgs &ma, const Model2D *models, const Tile2D *tiles, int ntiles,
                      int mask, Fields2D f, int *err, cudaStream_t st) {
    switch (nm) {
    case 0: return stress_ti<KIND, 0>(ti, ma, models, tiles, ntiles, mask, f, err, st);
    case 1: return stress_ti<KIND, 1>(ti, ma, models, tiles, ntiles, mask, f, err, st);
    case 2: return stress_ti<KIND, 2>(ti, ma, models, tiles, ntiles, mask, f, err, st);
    default: return stress_ti<KIND, 3>(ti, ma, models, tiles, ntiles, mask, f, err, st);
    }
}

template <int KIND, int TI>
cudaError_t vel_g(const MapArgs &ma, const Model2D *models, const Tile2D *tiles, int ntiles, int mask, Fields2D f,
                  int *err, cudaStream_t st) {
    if (ma.nset > 1) return run_vel<KIND, TI, kGroup2D>(ma, models, tiles, ntiles, mask, f, err, st);
    return run_vel<KIND, TI, 1>(ma, models, tiles, ntiles, mask, f, err, st);
}

template <int KIND>
cudaError_t vel_ti(int ti, const MapArgs &ma, const Model2D *models, const Tile2D *tiles, int ntiles, int mask,
                   Fields2D f, int *err, cudaStream_t st) {
    if (ti == 4) return vel_g<KIND, 4>(ma, models, tiles, ntiles, mask, f, err, st);
    if (ti == 16) return vel_g<KIND, 16>(ma, models, tiles, ntiles, mask, f, err, st);
    return vel_g<KIND, 8>(ma, models, tiles, ntiles, mask, f, err, st);
}

// 3D map (k, i, field) over a model's slab with the given box; L2 fills of
// 256 bytes, as the 3D maps (c2A batch 1.394 against 1.400 ms per step with
// 128-byte fills)
bool encode(unsigned char *out, float *slab, const Geo &g, int nf, unsigned bk, unsigned bi, unsigned bf) {
    static PFN_cuTensorMapEncodeTiled fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return false;
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(p);
    }
    const cuuint64_t dims[3] = {(cuuint64_t)g.Kp, (cuuint64_t)g.Ip, (cuuint64_t)nf};
    const cuuint64_t strides[2] = {(cuuint64_t)g.Kp * 4, (cuuint64_t)g.ncell * 4};
    const cuuint32_t box[3] = {bk, bi, bf};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = fn(reinterpret_cast<CUtensorMap *>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, slab, dims, strides,
                          box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace

Fields2D fields2d(int kind, int nm) {
    const bool psv = kind == SWPC_KIND_PSV;
    const int nv = psv ? 2 : 1, ns = psv ? 3 : 2;
    return Fields2D{0, nv, nv + ns + ns * nm};
}

int slab_fields2d(int kind, int nm) { return fields2d(kind, nm).med + 5; }

bool staged2d_ti_ok(int ti) { return ti == 4 || ti == 8 || ti == 16; }

bool encode_maps2d(Maps2D &m, int kind, int nm, float *slab, const Geo &g) {
    const int nf = slab_fields2d(kind, nm);
    unsigned char(*S)[128] = m.str.m;
    unsigned char(*V)[128] = m.vel.m;
    if (kind == SWPC_KIND_PSV) {
        return encode(S[ST_STATE], slab, g, nf, KT, BI, 3 + 3 * nm) && encode(S[ST_S], slab, g, nf, KT, BI, 3) &&
               encode(S[ST_MED], slab, g, nf, KT, BI, 3) && encode(S[ST_MU], slab, g, nf, KM, BI + 1, 1) &&
               encode(S[ST_V], slab, g, nf, KB, BI + 4, 2) && encode(V[VE_OWN], slab, g, nf, KT, BI, 2) &&
               encode(V[VE_RHO], slab, g, nf, KM, BI + 1, 1) && encode(V[VE_A], slab, g, nf, KT, BI + 3, 1) &&
               encode(V[VE_C], slab, g, nf, KB, BI, 1) && encode(V[VE_E], slab, g, nf, KB, BI + 3, 1);
    }
    // SH: the last velocity slot stays unused (zero)
    return encode(S[ST_STATE], slab, g, nf, KT, BI, 2 + 2 * nm) && encode(S[ST_S], slab, g, nf, KT, BI, 2) &&
           encode(S[ST_MED], slab, g, nf, KT, BI, 1) && encode(S[ST_MU], slab, g, nf, KM, BI + 1, 1) &&
           encode(S[ST_V], slab, g, nf, KB, BI + 4, 1) && encode(V[VE_OWN], slab, g, nf, KT, BI, 1) &&
           encode(V[VE_RHO], slab, g, nf, KT, BI, 1) && encode(V[VE_A], slab, g, nf, KT, BI + 3, 1) &&
           encode(V[VE_C], slab, g, nf, KB, BI, 1);
}

cudaError_t launch_stress2d_tma(int kind, int nm, int ti, const MapSet2D *sets, int nset, int model0,
                                const Model2D *models, const Tile2D *tiles, int ntiles, int mask, Fields2D f, int *err,
                                cudaStream_t st) {
    if (ntiles <= 0) return cudaSuccess;
    if (nset < 1 || nset > kGroup2D) return cudaErrorInvalidValue;
    const MapArgs ma{sets, nset, model0};
    if (kind == SWPC_KIND_PSV) return stress_nm<0>(nm, ti, ma, models, tiles, ntiles, mask, f, err, st);
    return stress_nm<1>(nm, ti, ma, models, tiles, ntiles, mask, f, err, st);
}

cudaError_t launch_vel2d_tma(int kind, int ti, const MapSet2D *sets, int nset, int model0, const Model2D *models,
                             const Tile2D *tiles, int ntiles, int mask, Fields2D f, int *err, cudaStream_t st) {
    if (ntiles <= 0) return cudaSuccess;
    if (nset < 1 || nset > kGroup2D) return cudaErrorInvalidValue;
    const MapArgs ma{sets, nset, model0};
    if (kind == SWPC_KIND_PSV) return vel_ti<0>(ti, ma, models, tiles, ntiles, mask, f, err, st);
    return vel_ti<1>(ti, ma, models, tiles, ntiles, mask, f, err, st);
}

}  // namespace swpc
