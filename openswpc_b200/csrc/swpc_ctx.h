// swpc_ctx.h -- device context shared by the 3D, P-SV and SH solvers.
//
// Device layout (all solvers): every full-grid field is one float array over
// the reference memory box i in [-2, nx+3], j in [-2, ny+3] and
// k in [1-KH, nz+3(+pad)] with k fastest.  Cell (k,i,j) sits at
//     e = ((j+2) * Ip + (i+2)) * Kp + (k - 1 + KH),  Ip = nx + 6,
// Kp a multiple of 8 floats, KH = 8, so k = 1 starts every column on a
// 32-byte sector and a warp of 32 consecutive k reads exactly 4 sectors.
// For the 2D codes ny = 1 and j is fixed to 1.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/swpc_gpu.h"

namespace swpc {

constexpr int KH = 8;      // device halo below k = 1
constexpr int NM_MAX = 3;  // reference NM (m_global.f90:31)

struct Geo {
    int nx, ny, nz;
    int Kp;                // k pitch in floats
    int Ip;                // i pitch in columns (nx + 6)
    int Jp;                // j extent in columns (ny + 6, or 1 for 2D)
    long long ncell;       // Kp * Ip * Jp
};

__host__ __device__ inline long long col_index(const Geo &g, int i, int j) {
    return (long long)(j + 2) * g.Ip + (i + 2);
}
__host__ __device__ inline long long cell_index(const Geo &g, int k, int i, int j) {
    return col_index(g, i, j) * g.Kp + (k - 1 + KH);
}

// One entry of the per-step point-source injection list (stress glut, body
// force, reciprocity force).  Entries are applied in list order.
struct InjEntry {
    long long cell;   // device cell index
    int field;        // target field id (SWPC_F_*)
    int src;          // source index into the stime / weight tables
    float coef;       // moment-tensor component or force component
    int mode;         // 0: S -= coef*sdrop ; 1: S -= coef*sdrop/4 ;
                      // 2: V += b*coef*stime*dt_dxyz/2 ; 3: V += b*f/2 (green)
    int bfield;       // buoyancy field for modes 2-3 (index into med[])
    int pad;
};

struct Model2D;
struct Tile2D;
struct Wav2Args;

}  // namespace swpc

struct swpc_snap_state;
struct swpc_adj_state;

struct swpc_ctx {
    int kind;
    swpc::Geo g;
    swpc_desc d;
    int prec = SWPC_PREC_F32;   // storage of S and R (3D)
    // FP16 forms: the scales 2^e, 2^-e of the stresses and memory variables
    // (swpc_kernels.cuh sc_sS) and the exponents, in device memory, where the
    // re-centring kernels of swpc_prec.cu keep them
    float *d_scale = nullptr;
    float h_scale[48];
    int *d_exp = nullptr;                  // exponents: each stress array, the memory variables
    unsigned int *d_rmax = nullptr;        // re-centring scratch: maxima, factors, moved count
    float *d_rfactor = nullptr;
    int *d_rchanged = nullptr;
    int device;
    cudaStream_t stream;
    std::string err;

    // kernel region (m_global.f90:349-378)
    int ibk, iek, jbk, jek, kbk, kek;
    // subdomain of a decomposed grid (m_global.f90:236-303): the global
    // extents and this box's offsets (nxg = nx, ioff = 0 on a single domain)
    int nxg = 0, nyg = 0, ioff = 0, joff = 0;
    bool sub = false;
    bool na_wide = false;   // 2 na >= nx or ny of a single domain: refused at the medium upload

    // full-grid fields
    float *V[3] = {nullptr, nullptr, nullptr};          // Vx Vy Vz (2D: Vx Vz / Vy)
    float *S[6] = {nullptr};                           // Sxx Syy Szz Syz Sxz Sxy
    float *R[18] = {nullptr};                          // component*3 + m
    // medium: 0 rho 1 lam 2 mu 3 taup 4 taus 5 bx 6 by 7 bz 8 muyz 9 muxz 10 muxy
    float *med[11] = {nullptr};
    int4 *band = nullptr;     // per column: kfs_top kfs_bot kob_top kob_bot
    int2 *pmlcol = nullptr;   // per column: kbeg_a, aux base (-1 = no absorber cell)
    int *kob = nullptr, *kfs = nullptr;   // per column
    std::vector<int> h_kbeg_a;            // host copy (columns, device indexing)

    // absorber: 0 ADE-CFS PML, 1 Cerjan sponge (abc_type, m_absorb.f90:25-75)
    int abc = 0;
    // plane-wave mode (pw_mode, m_source.f90:67-79): zero-derivative side boundary of the PML updates
    int pw_mode = 0;
    float *cj = nullptr;   // Cerjan factors: gx_c gx_b (nx) gy_c gy_b (ny) gz_c gz_b (nz)
    // PML
    bool absorb_ready = false;
    long long npml = 0;
    float *aux[18] = {nullptr};
    float4 *gx[2] = {nullptr, nullptr};   // c, e  indexed [i-1]
    float4 *gy[2] = {nullptr, nullptr};
    float4 *gz[2] = {nullptr, nullptr};

    // coefficients
    bool kernel_ready = false;
    bool medium_ready = false;
    bool vmodel_ready = false;   // a per-cell model waits in the medium arrays (swpc_medium.cu)
    float e40[3][2], e41[3][2];   // [axis][0: 4th order (isign=-1), 1: 2nd order band]
    float r20[3];
    float c1[swpc::NM_MAX], c2[swpc::NM_MAX], d1[swpc::NM_MAX], d2;
    float ts[swpc::NM_MAX];

    // sources
    int nsrc_glut = 0, nsrc_bf = 0;
    swpc::InjEntry *inj_glut = nullptr; int ninj_glut = 0; bool glut_serial = false;
    swpc::InjEntry *inj_bf = nullptr; int ninj_bf = 0; bool bf_serial = false;
    float *stime_glut = nullptr;   // (nt, nsrc) moment rate at tbeg+(it-0.5)dt
    float *mo_glut = nullptr;      // (nsrc)
    float *stime_bf = nullptr;     // (nt, nsrc) at tbeg + it*dt
    long long *rho_cell_bf = nullptr;   // 2D body force: density cell per source
    float dt_dxyz = 0.f;
    // green's function source
    bool green = false;
    swpc::InjEntry *inj_green = nullptr; int ninj_green = 0;
    float *stf_green = nullptr;    // (nt)
    float green_dt_dxyz = 0.f;
    float green_f[3] = {0, 0, 0};

    // recorder
    int nst = 0, ntw = 0, ntdec_w = 1, wav_what = 0;
    float M0 = 1.f, UC = 1e-15f;
    int *st_ijk = nullptr;        // (3, nst)
    float *wav[4] = {nullptr};    // v, u, stress, strain: (ntw, ncmp, nst)
    float *uacc = nullptr;        // (3, nst)
    float *eacc = nullptr;        // (6, nst)
    float r40[3], r41[3];         // m_wav.f90:130-135

    // snapshot planes (swpc_snap.cu)
    swpc_snap_state *snp = nullptr;
    // adjoint state and checkpoints (swpc_adjoint.cu)
    swpc_adj_state *adj = nullptr;
    // green__store points (swpc_green.cu): ng grid points, accumulated
    // displacement derivatives (and displacements) and the sampled output
    int ng = 0, ng_cmp = 0, ng_ntw = 0, ng_ntdec = 1;
    int *g_ijk = nullptr;     // (3, ng)
    float *g_acc = nullptr;   // (12, ng): dxUx dxUy dxUz dyUx dyUy dyUz dzUx dzUy dzUz ux uy uz
    float *g_out = nullptr;   // gf(ntw, ncmp*ng), column-major as the reference
    long long g_bytes = 0;    // device bytes of the three arrays (counted in `bytes`)

    // vmax
    unsigned int *vmax_buf = nullptr;
    unsigned int *h_vmax = nullptr;   // pinned

    // graph
    int *d_it = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_key = -1;

    // 2D solvers: device model descriptor, tile list, recorder descriptor
    swpc::Model2D *d_model2d = nullptr;
    swpc::Tile2D *d_tiles2d = nullptr;
    int ntiles2d = 0;
    swpc::Wav2Args *d_wav2d = nullptr;
    int nm2d_aux = 0;
    bool desc_dirty = true;   // device descriptors must be refreshed before the next launch
    void *maps2d = nullptr;   // tensor maps of the model (swpc::Maps2D): a kernel parameter of the staged kernels

    // launch shape (swpc_set_launch): block = 32 x bi x bj threads; minb =
    // minimum resident blocks per SM the kernels are compiled for
    int bi = 2, bj = 1, vbi = 2, vbj = 2;
    int stress_minb = 2, vel_minb = 4;
    // 2.5D marching variants (32 x 8 plane tile walking jc planes along j)
    bool stress_march = false, vel_march = false;
    int stress_jc = 8, vel_jc = 8, stress_mminb = 2, vel_mminb = 2;
    // velocity kernel with four consecutive k per thread (swpc3d_vec.cu)
    bool vel_vec = false;
    int vel_vminb = 2, vel_vbi = 2, vel_vbj = 2;
    // TMA-staged kernels (swpc3d_tma.cu): tile 32 x bi x bj; tensor maps over
    // the field slab, encoded for the shapes in tma_key.  2D contexts
    // (swpc2d_tma.cu): tiles 32 x 16 with stress_tbi / vel_tbi threads along i
    bool stress_tma = false, vel_tma = false;
    int stress_tbi = 4, stress_tbj = 4, vel_tbi = 4, vel_tbj = 4;
    bool adj_tma = true;          // staged stress-phase adjoint weights (swpc_adjoint.cu)
    bool adj_fuse = true;         // velocity-phase adjoint weights formed by the stress-phase gather before
    float *div_out = nullptr;     // the gradient's kept step: the velocity update stores the stress divergences here
    int div_geo[4] = {0, 0, 0, 0};   // its layout: Kp, Ip, i0, j0 (Vel3Args divo)
    long long div_n = 0;
    int tile_jblock = 0;          // j tiles per block of the staged launch order (0: by size, see tma_tiles)
    void *tmaps = nullptr;        // swpc::TmaMaps
    int tma_key[4] = {-1, -1, -1, -1};
    int *d_err = nullptr;         // device error word of the staged kernels

    // FP32 storage: V, S, R and the medium in one allocation, so that tensor
    // maps cover them.  3D field order: 0-2 V, 3-8 S, 9.. R component-major,
    // then lam mu taup taus muyz muxz muxy and bx by bz; 2D: V, S, R, then
    // lam taup taus mu rho
    float *slab = nullptr;
    float *stage = nullptr;       // staging buffer of host uploads (copy_box), allocated on first use
    long long stage_floats = 0;
    int slab_nf = 0;
    // reduced-precision 3D storage: the 2-byte fields (S for F16_SR, then R
    // component-major) in a second slab of ncell-element fields
    unsigned short *hslab = nullptr;
    int hslab_nf = 0;
    int nfbatch = 0;   // reciprocity batches that borrow this context (swpc_fbatch.cu)

    long long bytes = 0;
};

// helpers shared by the translation units
namespace swpc {
int set_err(swpc_ctx *c, int code, const std::string &msg);
// 2 na must fit the grid across x and y (the whole grid for a block of a
// decomposed one); refused when the medium arrives
int upload_scales(swpc_ctx *c);   // swpc_api.cu
int rescale_before_stress(swpc_ctx *c, int it, const int *d_it);   // swpc_prec.cu
int rescale_after_stress(swpc_ctx *c);
inline int check_na_wide(swpc_ctx *c) {
    return c->na_wide ? set_err(c, SWPC_ERR_ARG, "absorber thickness na too large for the grid") : SWPC_OK;
}
int snap_launch(swpc_ctx *c, int it, const int *d_it);   // swpc_snap.cu
void snap_free(swpc_ctx *c);
int snap_clear(swpc_ctx *c);   // frames, displacement accumulators and maxima back to zero
// one time step of the wavefield alone, without recorders (swpc_api.cu): the
// recompute of a checkpointed segment must not record a step twice
int step_state(swpc_ctx *c, int it);
void adj_free(swpc_ctx *c);   // swpc_adjoint.cu
int green_store_launch(swpc_ctx *c, int it, const int *d_it);   // swpc_green.cu
// plane-wave mode (swpc_pw.cu): the ghost planes of V (which = 0) or S (1) extrapolated from inside, and the
// ghost planes global__comm_vel / global__comm_stress zero on a single domain
int pw_fill(swpc_ctx *c, int which);
int pw_comm_zero(swpc_ctx *c, int which);
// the same for nmem wavefields at V[q] + m * vstride (reciprocity batch), with
// per-member accumulators (12 ng each) and outputs (ntw ncmp ng each)
int green_store_members(swpc_ctx *c, float *const *V, long long vstride, int nmem, float *acc, float *out, int it,
                        const int *d_it);
void green_free(swpc_ctx *c);
int field_storage(const swpc_ctx *c, int field);   // swpc_prec.cu
float field_scale(const swpc_ctx *c, int field);
int prec_to_f32(swpc_ctx *c, int field, const float *stored, float **tmp);
int prec_from_f32(swpc_ctx *c, int field, const float *tmp, float *stored);
int cuda_check(swpc_ctx *c, cudaError_t e, const char *what);
// host Fortran box (leading extents ld_k, ld_i) <-> device columns (swpc_api.cu)
int copy_box(swpc_ctx *c, float *dev, const float *host_in, float *host_out, int ld_k, int ld_i);
// the same from a device array in the Fortran box layout, on the context stream
int copy_box_from_device(swpc_ctx *c, float *dev, const float *src, int ld_k, int ld_i);
// averaged_medium on the device from rho (held in the muyz array) and mu (swpc_api.cu)
int average_medium(swpc_ctx *c);
template <typename T>
int dalloc(swpc_ctx *c, T **p, size_t n) {
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        return set_err(c, SWPC_ERR_NOMEM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
    }
    c->bytes += (long long)(n * sizeof(T));
    e = cudaMemsetAsync(*p, 0, n * sizeof(T), c->stream);
    if (e != cudaSuccess) return cuda_check(c, e, "cudaMemsetAsync");
    return 0;
}
}  // namespace swpc
