// swpc2d_api.cu -- 2D P-SV / SH contexts and the batched 2D ensemble.
//
// A 2D context owns one model (one Model2D descriptor and its tile list).
// A batch (swpc_batch_*) joins the descriptors and tiles of many 2D contexts
// of the same kind into one table, so that a single persistent launch per
// half step advances every member; the per-step sequence is captured once
// into a CUDA graph and replayed.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "swpc2d.cuh"
#include "swpc_ctx.h"
#include "swpc_kernels.cuh"

namespace swpc {

int copy_box(swpc_ctx *c, float *dev, const float *host_in, float *host_out, int ld_k, int ld_i);

#define CK(call)                                        \
    do {                                                \
        int _rc = cuda_check(c, (call), #call);         \
        if (_rc) return _rc;                            \
    } while (0)
#define RC(call)             \
    do {                     \
        int _rc = (call);    \
        if (_rc) return _rc; \
    } while (0)

// ctx slots of the 2D fields (3D field ids are reused: P-SV Vx Vz / Sxx Szz
// Sxz, SH Vy / Syz Sxy; memory variables at SWPC_F_R + 3*c + m)
static const int PSV_V[2] = {0, 2}, PSV_S[3] = {0, 2, 4}, PSV_R[3] = {0, 2, 4};
static const int SH_V[1] = {1}, SH_S[2] = {3, 5}, SH_R[2] = {3, 5};

// flags of the 32 x ni tile at (k0, i0): interior and absorber cells present
int tile2d_flags(const swpc_ctx *c, int k0, int i0, int ni) {
    const Geo &g = c->g;
    const int i1 = std::min(i0 + ni - 1, g.nx), k1 = std::min(k0 + 31, g.nz);
    int f = 0;
    if (k0 <= c->kek && i0 <= c->iek && i1 >= c->ibk) f |= kTileInterior;
    if (i0 < c->ibk || i1 > c->iek || k1 > c->kek) f |= kTileAbsorber;
    return f;
}

int build_tiles_2d(swpc_ctx *c);

int create_2d(swpc_ctx *c) {
    const Geo &g = c->g;
    const bool psv = c->kind == SWPC_KIND_PSV;
    int rc = 0;
    const int nv = psv ? 2 : 1, ns = psv ? 3 : 2, nm = c->d.nm;
    // one slab: V, S, R (component-major), then lam taup taus mu rho
    const int nf = slab_fields2d(c->kind, nm);
    rc = dalloc(c, &c->slab, (size_t)nf * g.ncell);
    if (rc) return rc;
    c->slab_nf = nf;
    auto F = [&](int f) { return c->slab + (size_t)f * g.ncell; };
    for (int q = 0; q < nv; q++) c->V[psv ? PSV_V[q] : SH_V[q]] = F(q);
    for (int q = 0; q < ns; q++) c->S[psv ? PSV_S[q] : SH_S[q]] = F(nv + q);
    for (int q = 0; q < ns; q++)
        for (int m = 0; m < nm; m++) c->R[(psv ? PSV_R[q] : SH_R[q]) * 3 + m] = F(nv + ns + q * nm + m);
    const int mb = fields2d(c->kind, nm).med;
    c->med[1] = F(mb);       // lam
    c->med[3] = F(mb + 1);   // taup
    c->med[4] = F(mb + 2);   // taus
    c->med[2] = F(mb + 3);   // mu
    c->med[0] = F(mb + 4);   // rho
    if (!rc) rc = dalloc(c, &c->band, g.Ip);
    if (!rc) rc = dalloc(c, &c->pmlcol, g.Ip);
    if (!rc) rc = dalloc(c, &c->kob, g.Ip);
    if (!rc) rc = dalloc(c, &c->kfs, g.Ip);
    if (!rc) rc = dalloc(c, &c->d_model2d, 1);
    if (!rc) rc = dalloc(c, &c->d_wav2d, 1);
    if (!rc) rc = dalloc(c, &c->d_err, 1);
    c->nm2d_aux = psv ? 8 : 4;
    if (rc) return rc;
    // tensor maps of the staged kernels over the slab; the staged kernels are
    // the default launch
    Maps2D *mp = new Maps2D();
    memset(mp, 0, sizeof(Maps2D));
    c->maps2d = mp;
    if (!encode_maps2d(*mp, c->kind, nm, c->slab, g))
        return set_err(c, SWPC_ERR_CUDA, "cuTensorMapEncodeTiled failed for the 2D field slab");
    c->stress_tma = c->vel_tma = true;
    c->stress_tbi = c->vel_tbi = 8;
    return build_tiles_2d(c);
}

// tile list: 32 (k) x 16 (i), flagged by the kernel region
int build_tiles_2d(swpc_ctx *c) {
    const Geo &g = c->g;
    std::vector<Tile2D> tiles;
    const int ni = kDefaultTiles.ti * kDefaultTiles.ri;
    for (int i0 = 1; i0 <= g.nx; i0 += ni)
        for (int k0 = 1; k0 <= g.nz; k0 += 32) tiles.push_back(Tile2D{0, k0, i0, tile2d_flags(c, k0, i0, ni)});
    if (!c->d_tiles2d) RC(dalloc(c, &c->d_tiles2d, tiles.size()));
    c->ntiles2d = (int)tiles.size();
    CK(cudaMemcpyAsync(c->d_tiles2d, tiles.data(), tiles.size() * sizeof(Tile2D), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SWPC_OK;
}

// absorb_c__setup of the 2D codes (src/swpc_psv/m_absorb_c.f90:27-88,
// src/swpc_sh/m_absorb_c.f90:27-80) with the kernel region of abc_type =
// 'cerjan' (src/swpc_psv/m_global.f90:281-303: the whole domain)
int cerjan_setup_2d(swpc_ctx *c, const float *gx_c, const float *gx_b, const float *gz_c, const float *gz_b) {
    const Geo &g = c->g;
    if (!gx_c || !gx_b || !gz_c || !gz_b) return set_err(c, SWPC_ERR_ARG, "sponge profile missing");
    const size_t n = 2 * (size_t)(g.nx + g.nz);
    if (!c->cj) RC(dalloc(c, &c->cj, n));
    std::vector<float> h(n);
    std::copy(gx_c, gx_c + g.nx, h.begin());
    std::copy(gx_b, gx_b + g.nx, h.begin() + g.nx);
    std::copy(gz_c, gz_c + g.nz, h.begin() + 2 * g.nx);
    std::copy(gz_b, gz_b + g.nz, h.begin() + 2 * g.nx + g.nz);
    CK(cudaMemcpyAsync(c->cj, h.data(), n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    c->abc = 1;
    c->ibk = 1; c->iek = g.nx; c->kbk = 1; c->kek = g.nz;
    RC(build_tiles_2d(c));
    c->desc_dirty = true;
    c->absorb_ready = true;
    return SWPC_OK;
}

// absorb_c__update_stress / _vel of P-SV (src/swpc_psv/m_absorb_c.f90:
// 90-160) and SH (src/swpc_sh/m_absorb_c.f90:82-135) in the reference's
// product order; cells with both factors 1 are not visited (same bits)
__global__ void cerjan2d_kernel(int psv, int phase, int nx, int nz, int na, int ioff, int nxg, int Kp,
                                const float *__restrict__ cj, float *f0, float *f1, float *f2) {
    const float *gxc = cj, *gxb = cj + nx, *gzc = cj + 2 * nx, *gzb = gzc + nz;
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    // one warp per column, lanes along k: every k of the side columns, the
    // bottom na cells of the others
    for (int i = 1 + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i <= nx; i += nw) {
        const bool side = i + ioff <= na || i + ioff > nxg - na;   // global column
        const float xc = gxc[i - 1], xb = gxb[i - 1];
        for (int k = (side ? 1 : nz - na + 1) + lane; k <= nz; k += 32) {
            const long long e = (long long)(i + 2) * Kp + (k - 1 + KH);
            const float zc = gzc[k - 1], zb = gzb[k - 1];
            if (psv) {
                if (phase == 0) {
                    const float gc = __fmul_rn(xc, zc), gb = __fmul_rn(xb, zb);
                    f0[e] = __fmul_rn(f0[e], gc);
                    f1[e] = __fmul_rn(f1[e], gc);
                    f2[e] = __fmul_rn(f2[e], gb);
                } else {
                    f0[e] = __fmul_rn(__fmul_rn(f0[e], xb), zc);
                    f1[e] = __fmul_rn(__fmul_rn(f1[e], xc), zb);
                }
            } else if (phase == 0) {
                f0[e] = __fmul_rn(__fmul_rn(f0[e], xc), zb);
                f1[e] = __fmul_rn(__fmul_rn(f1[e], xb), zc);
            } else {
                f0[e] = __fmul_rn(__fmul_rn(f0[e], xc), zc);
            }
        }
    }
}

static int launch_cerjan2d(swpc_ctx *c, int phase, cudaStream_t stream) {
    const bool psv = c->kind == SWPC_KIND_PSV;
    float *f0, *f1 = nullptr, *f2 = nullptr;
    if (phase == 0) {
        f0 = psv ? c->S[0] : c->S[3];
        f1 = psv ? c->S[2] : c->S[5];
        f2 = psv ? c->S[4] : nullptr;
    } else {
        f0 = psv ? c->V[0] : c->V[1];
        f1 = psv ? c->V[2] : nullptr;
    }
    cerjan2d_kernel<<<148 * 4, 256, 0, stream>>>(psv ? 1 : 0, phase, c->g.nx, c->g.nz, c->d.na, c->ioff, c->nxg,
                                                  c->g.Kp, c->cj, f0, f1, f2);
    return cuda_check(c, cudaGetLastError(), "cerjan2d launch");
}

void destroy_2d(swpc_ctx *c) {
    if (c->d_model2d) cudaFree(c->d_model2d);
    delete static_cast<Maps2D *>(c->maps2d);
    c->maps2d = nullptr;
    if (c->d_tiles2d) cudaFree(c->d_tiles2d);
    if (c->d_wav2d) cudaFree(c->d_wav2d);
    if (c->rho_cell_bf) cudaFree(c->rho_cell_bf);
}

int upload_medium_2d(swpc_ctx *c, const swpc_medium_view *m) {
    const Geo &g = c->g;
    const float *src[5] = {m->rho, m->lam, m->mu, m->taup, m->taus};
    for (int q = 0; q < 5; q++) {
        if (!src[q]) return set_err(c, SWPC_ERR_ARG, "2D medium field missing (rho, lam, mu, taup, taus)");
        RC(copy_box(c, c->med[q], src[q], nullptr, m->ld_k, m->ld_i));
    }
    if (!m->kfs || !m->kob || !m->kfs_top || !m->kfs_bot || !m->kob_top || !m->kob_bot || !m->kbeg_a)
        return set_err(c, SWPC_ERR_ARG, "integer map missing");
    std::vector<int4> band(g.Ip);
    std::vector<int> kob(g.Ip), kfs(g.Ip);
    c->h_kbeg_a.assign(g.Ip, 0);
    for (int i = -2; i <= g.nx + 3; i++) {
        band[i + 2] = make_int4(m->kfs_top[i + 2], m->kfs_bot[i + 2], m->kob_top[i + 2], m->kob_bot[i + 2]);
        kob[i + 2] = m->kob[i + 2];
        kfs[i + 2] = m->kfs[i + 2];
        c->h_kbeg_a[i + 2] = m->kbeg_a[i + 2];
    }
    for (int i = 1; i <= g.nx && c->abc == 0; i++) {
        const int want = (i >= c->ibk && i <= c->iek) ? c->kek + 1 : 1;
        if (c->h_kbeg_a[i + 2] != want)
            return set_err(c, SWPC_ERR_ARG, "kbeg_a map does not match the absorber layout (src/swpc_psv/m_global.f90:271-278)");
    }
    CK(cudaMemcpyAsync(c->band, band.data(), g.Ip * sizeof(int4), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->kob, kob.data(), g.Ip * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->kfs, kfs.data(), g.Ip * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->medium_ready = true;
    return SWPC_OK;
}

static int upload_profile(swpc_ctx *c, float4 **dst, const float *g4, int n) {
    if (!g4) return set_err(c, SWPC_ERR_ARG, "damping profile missing");
    if (!*dst) RC(dalloc(c, dst, n));
    std::vector<float4> v(n);
    for (int q = 0; q < n; q++) v[q] = make_float4(g4[4 * q], g4[4 * q + 1], g4[4 * q + 2], g4[4 * q + 3]);
    CK(cudaMemcpyAsync(*dst, v.data(), n * sizeof(float4), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SWPC_OK;
}

int absorb_setup_2d(swpc_ctx *c, const float *gxc, const float *gxe, const float *gzc, const float *gze) {
    const Geo &g = c->g;
    RC(upload_profile(c, &c->gx[0], gxc, g.nx));
    RC(upload_profile(c, &c->gx[1], gxe, g.nx));
    RC(upload_profile(c, &c->gz[0], gzc, g.nz));
    RC(upload_profile(c, &c->gz[1], gze, g.nz));
    std::vector<int2> pc(g.Ip, make_int2(1, -1));
    long long base = 0;
    for (int i = 1; i <= g.nx; i++) {
        const int kb = c->h_kbeg_a[i + 2];
        const int len = g.nz - kb + 1;
        if (len <= 0) continue;
        pc[i + 2] = make_int2(kb, (int)base);
        base += (len + 7) / 8 * 8;
    }
    c->npml = base;
    for (int q = 0; q < c->nm2d_aux; q++) {
        if (c->aux[q]) { cudaFree(c->aux[q]); c->aux[q] = nullptr; }
        RC(dalloc(c, &c->aux[q], (size_t)std::max<long long>(base, 1)));
    }
    CK(cudaMemcpyAsync(c->pmlcol, pc.data(), g.Ip * sizeof(int2), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->absorb_ready = true;
    return SWPC_OK;
}

// host image of the model descriptor of a 2D context
Model2D model_of(const swpc_ctx *c) {
    Model2D m;
    memset(&m, 0, sizeof(m));
    const bool psv = c->kind == SWPC_KIND_PSV;
    m.nx = c->g.nx; m.nz = c->g.nz; m.Kp = c->g.Kp; m.nm = c->d.nm;
    m.ibk = c->ibk; m.iek = c->iek; m.kek = c->kek; m.dt = c->d.dt;
    if (psv) {
        m.V0 = c->V[0]; m.V1 = c->V[2];
        m.S0 = c->S[0]; m.S1 = c->S[2]; m.S2 = c->S[4];
        for (int q = 0; q < 3; q++)
            for (int k = 0; k < 3; k++) m.R[q * 3 + k] = c->R[PSV_R[q] * 3 + k];
    } else {
        m.V0 = c->V[1];
        m.S0 = c->S[3]; m.S1 = c->S[5];
        for (int q = 0; q < 2; q++)
            for (int k = 0; k < 3; k++) m.R[q * 3 + k] = c->R[SH_R[q] * 3 + k];
    }
    m.rho = c->med[0]; m.lam = c->med[1]; m.mu = c->med[2]; m.taup = c->med[3]; m.taus = c->med[4];
    m.band = c->band; m.pmlcol = c->pmlcol;
    for (int q = 0; q < 8; q++) m.aux[q] = c->aux[q];
    m.gxc = c->gx[0]; m.gxe = c->gx[1]; m.gzc = c->gz[0]; m.gze = c->gz[1];
    for (int s = 0; s < 2; s++) {
        m.e40[0][s] = c->e40[0][s]; m.e41[0][s] = c->e41[0][s];
        m.e40[1][s] = c->e40[2][s]; m.e41[1][s] = c->e41[2][s];
    }
    m.r20[0] = c->r20[0]; m.r20[1] = c->r20[2];
    for (int q = 0; q < NM_MAX; q++) { m.c1[q] = c->c1[q]; m.c2[q] = c->c2[q]; m.d1[q] = c->d1[q]; }
    m.d2 = c->d2;
    return m;
}

int update_stress_2d_kernel(swpc_ctx *c, int mask);
int update_vel_2d_kernel(swpc_ctx *c, int mask);

int update_stress_2d(swpc_ctx *c, int mask) {
    if (c->abc == 1) {
        // Cerjan: the interior update over the whole domain, then the sponge
        if (mask & 1) RC(update_stress_2d_kernel(c, 1));
        if (mask & 2) RC(launch_cerjan2d(c, 0, c->stream));
        return SWPC_OK;
    }
    return update_stress_2d_kernel(c, mask);
}

int update_stress_2d_kernel(swpc_ctx *c, int mask) {
    const int m = (c->d.na > 0 && c->abc == 0) ? mask : (mask & 1);
    if (c->stress_tma)
        return cuda_check(c, launch_stress2d_tma(c->kind, c->d.nm, c->stress_tbi, &static_cast<Maps2D *>(c->maps2d)->str,
                                                 1, 0, c->d_model2d, c->d_tiles2d, c->ntiles2d, m,
                                                 fields2d(c->kind, c->d.nm), c->d_err, c->stream),
                          "stress2d_tma launch");
    launch_stress2d(c->kind, c->d.nm, c->d_model2d, c->d_tiles2d, c->ntiles2d, m, kDefaultTiles, c->stream);
    return cuda_check(c, cudaGetLastError(), "stress2d launch");
}

int update_vel_2d(swpc_ctx *c, int mask) {
    if (c->abc == 1) {
        if (mask & 1) RC(update_vel_2d_kernel(c, 1));
        if (mask & 2) RC(launch_cerjan2d(c, 1, c->stream));
        return SWPC_OK;
    }
    return update_vel_2d_kernel(c, mask);
}

int update_vel_2d_kernel(swpc_ctx *c, int mask) {
    const int m = (c->d.na > 0 && c->abc == 0) ? mask : (mask & 1);
    if (c->vel_tma)
        return cuda_check(c, launch_vel2d_tma(c->kind, c->vel_tbi, &static_cast<Maps2D *>(c->maps2d)->vel, 1, 0,
                                              c->d_model2d, c->d_tiles2d, c->ntiles2d, m, fields2d(c->kind, c->d.nm),
                                              c->d_err, c->stream),
                          "vel2d_tma launch");
    launch_vel2d(c->kind, c->d_model2d, c->d_tiles2d, c->ntiles2d, m, kDefaultTiles, c->stream);
    return cuda_check(c, cudaGetLastError(), "vel2d launch");
}

Wav2Args wav_of(const swpc_ctx *c) {
    Wav2Args a;
    memset(&a, 0, sizeof(a));
    const bool psv = c->kind == SWPC_KIND_PSV;
    a.Kp = c->g.Kp; a.nst = c->nst; a.ntw = c->ntw; a.ntdec_w = c->ntdec_w; a.what = c->wav_what; a.psv = psv;
    a.st = c->st_ijk;
    a.V0 = psv ? c->V[0] : c->V[1];
    a.V1 = psv ? c->V[2] : nullptr;
    a.uacc = c->uacc; a.wav_v = c->wav[0]; a.wav_u = c->wav[1];
    a.M0 = c->M0; a.UC = c->UC; a.dt = c->d.dt;
    return a;
}

int wav_store_2d(swpc_ctx *c, int it, const int *d_it) {
    launch_wav2d(c->d_wav2d, 1, c->nst, it, d_it, c->stream);
    return cuda_check(c, cudaGetLastError(), "wav2d launch");
}

// upload the model and recorder descriptors after any setup change; called
// outside stream capture, before launches
int refresh_2d(swpc_ctx *c) {
    if (!c->desc_dirty) return SWPC_OK;
    const Model2D m = model_of(c);
    const Wav2Args w = wav_of(c);
    CK(cudaMemcpyAsync(c->d_model2d, &m, sizeof(m), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_wav2d, &w, sizeof(w), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->desc_dirty = false;
    return SWPC_OK;
}

int vmax_2d(swpc_ctx *c, float *out) {
    const bool psv = c->kind == SWPC_KIND_PSV;
    CK(cudaMemsetAsync(c->vmax_buf, 0, 4 * sizeof(unsigned int), c->stream));
    launch_vmax2d(psv ? c->V[0] : c->V[1], psv ? c->V[2] : nullptr, c->kob, c->g.Kp, c->ibk, c->iek, c->vmax_buf,
                  c->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->h_vmax, c->vmax_buf, 2 * sizeof(unsigned int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    memcpy(&out[0], &c->h_vmax[0], sizeof(float));
    memcpy(&out[1], &c->h_vmax[1], sizeof(float));
    out[2] = 0.0f;
    return SWPC_OK;
}

}  // namespace swpc

// ---------------------------------------------------------------------------
// batched 2D ensemble
// ---------------------------------------------------------------------------
using namespace swpc;

struct swpc_batch {
    std::vector<swpc_ctx *> members;
    int kind = 0, nm = 0, nt = 0, device = 0;
    cudaStream_t stream = nullptr;
    Model2D *d_models = nullptr;
    Tile2D *d_tiles = nullptr;
    int ntiles = 0;
    TileShape shape = kDefaultTiles;
    bool tuned = false;
    Wav2Args *d_wav = nullptr;
    int max_nst = 0;
    InjArgs *d_inj = nullptr;
    int ninj = 0, max_inj = 0;
    int *d_it = nullptr;
    cudaGraphExec_t graph = nullptr;
    bool psv_bf_split = false;
    // TMA-staged kernels: threads along i of the stress / velocity CTAs (4, 8
    // or 16; 0 = the tile-walking kernels); the members' tensor-map sets in
    // member order; one staged launch per group of consecutive members
    // (first member of each group, and the end); the first tile of every
    // member (and the end); the error word of the staged copies
    int sti = 8, vti = 8;
    std::vector<MapSet2D> str_sets, vel_sets;
    std::vector<int> group_first, tile_first;
    int *d_err = nullptr;
    std::string err;
};

namespace swpc {
void launch_inject_multi(const InjArgs *list, int nlist, int max_n, const int *d_it, int it, cudaStream_t st);
InjArgs glut_args(swpc_ctx *c, int it, const int *d_it);
InjArgs bf_args(swpc_ctx *c, int it, const int *d_it);
}  // namespace swpc

static int berr(swpc_batch *b, int code, const std::string &m) {
    b->err = m;
    return code;
}

extern "C" const char *swpc_batch_last_error(const swpc_batch *b) { return b ? b->err.c_str() : "null batch"; }

extern "C" int swpc_batch_destroy(swpc_batch *b) {
    if (!b) return SWPC_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    void *ps[] = {b->d_models, b->d_tiles, b->d_wav, b->d_inj, b->d_it, b->d_err};
    for (void *p : ps) if (p) cudaFree(p);
    delete b;
    return SWPC_OK;
}

#define RCB(call)            \
    do {                     \
        int _rc = (call);    \
        if (_rc) return _rc; \
    } while (0)

#define BCK(call)                                                                                            \
    do {                                                                                                     \
        cudaError_t _e = (call);                                                                             \
        if (_e != cudaSuccess) return berr(b, SWPC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorName(_e)); \
    } while (0)

// tile list of every member for tiles of 32 (k) x (ts.ti * ts.ri) (i)
static int set_tiles(swpc_batch *b, TileShape ts) {
    std::vector<Tile2D> tiles;
    b->tile_first.clear();
    for (int q = 0; q < (int)b->members.size(); q++) {
        const swpc_ctx *c = b->members[q];
        b->tile_first.push_back((int)tiles.size());
        const int ni = ts.ti * ts.ri;
        for (int i0 = 1; i0 <= c->g.nx; i0 += ni)
            for (int k0 = 1; k0 <= c->g.nz; k0 += 32) tiles.push_back(Tile2D{q, k0, i0, tile2d_flags(c, k0, i0, ni)});
    }
    b->tile_first.push_back((int)tiles.size());
    if (b->d_tiles && (int)tiles.size() > b->ntiles) {
        BCK(cudaFree(b->d_tiles));
        b->d_tiles = nullptr;
    }
    if (!b->d_tiles) BCK(cudaMalloc(&b->d_tiles, tiles.size() * sizeof(Tile2D)));
    BCK(cudaMemcpy(b->d_tiles, tiles.data(), tiles.size() * sizeof(Tile2D), cudaMemcpyHostToDevice));
    b->ntiles = (int)tiles.size();
    b->shape = ts;
    // the staged kernels work on tiles of 32 x 16
    if (ts.ti * ts.ri != kTileI2D) b->sti = b->vti = 0;
    return SWPC_OK;
}

extern "C" int swpc_batch_create(swpc_ctx *const *members, int n, swpc_batch **out) {
    if (!members || n < 1 || !out) return SWPC_ERR_ARG;
    swpc_batch *b = new swpc_batch();
    *out = b;
    b->members.assign(members, members + n);
    swpc_ctx *c0 = members[0];
    b->kind = c0->kind; b->nm = c0->d.nm; b->nt = c0->d.nt; b->device = c0->device;
    if (b->kind == SWPC_KIND_3D) return berr(b, SWPC_ERR_ARG, "batches join 2D (P-SV or SH) contexts");
    for (auto *c : b->members) {
        if (c->kind != b->kind || c->d.nm != b->nm || c->device != b->device)
            return berr(b, SWPC_ERR_ARG, "batch members must share kind, nm and device");
        if (!c->medium_ready || !c->kernel_ready || (!c->absorb_ready && c->d.na > 0))
            return berr(b, SWPC_ERR_STATE, "batch member not fully set up");
        b->nt = std::min(b->nt, c->d.nt);
        if (c->kind == SWPC_KIND_PSV && c->ninj_bf > 0) b->psv_bf_split = true;
    }
    BCK(cudaSetDevice(b->device));
    BCK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    for (auto *c : b->members) BCK(cudaStreamSynchronize(c->stream));
    std::vector<Model2D> models;
    std::vector<Wav2Args> wavs;
    std::vector<InjArgs> injs;
    for (int q = 0; q < n; q++) {
        swpc_ctx *c = b->members[q];
        models.push_back(model_of(c));
        if (c->nst > 0 && c->wav_what) {
            wavs.push_back(wav_of(c));
            b->max_nst = std::max(b->max_nst, c->nst);
        }
    }
    BCK(cudaMalloc(&b->d_models, models.size() * sizeof(Model2D)));
    {
        for (int q = 0; q < n; q++) {
            if (!b->members[q]->maps2d) return berr(b, SWPC_ERR_STATE, "batch member without tensor maps");
            b->str_sets.push_back(static_cast<const Maps2D *>(b->members[q]->maps2d)->str);
            b->vel_sets.push_back(static_cast<const Maps2D *>(b->members[q]->maps2d)->vel);
        }
        // groups of consecutive members of nearly equal count, at most kGroup2D each
        const int ng = (n + kGroup2D - 1) / kGroup2D;
        for (int g = 0; g <= ng; g++) b->group_first.push_back((int)((long long)n * g / ng));
        BCK(cudaMalloc(&b->d_err, sizeof(int)));
        BCK(cudaMemset(b->d_err, 0, sizeof(int)));
    }
    {
        int rc = set_tiles(b, kDefaultTiles);
        if (rc) return rc;
    }
    BCK(cudaMalloc(&b->d_wav, std::max<size_t>(wavs.size(), 1) * sizeof(Wav2Args)));
    BCK(cudaMalloc(&b->d_it, sizeof(int)));
    BCK(cudaMemcpy(b->d_models, models.data(), models.size() * sizeof(Model2D), cudaMemcpyHostToDevice));
    if (!wavs.empty()) BCK(cudaMemcpy(b->d_wav, wavs.data(), wavs.size() * sizeof(Wav2Args), cudaMemcpyHostToDevice));
    b->max_nst = wavs.empty() ? 0 : b->max_nst;
    // injection: stress glut lists then body-force lists of every member
    std::vector<InjArgs> glut, bf;
    for (auto *c : b->members) {
        if (c->ninj_glut > 0) glut.push_back(glut_args(c, 0, b->d_it));
        if (c->ninj_bf > 0) bf.push_back(bf_args(c, 0, b->d_it));
    }
    injs = glut;
    injs.insert(injs.end(), bf.begin(), bf.end());
    b->ninj = (int)glut.size();    // stress-glut lists come first in d_inj
    b->max_inj = (int)bf.size();   // then the body-force lists
    BCK(cudaMalloc(&b->d_inj, std::max<size_t>(injs.size(), 1) * sizeof(InjArgs)));
    if (!injs.empty()) BCK(cudaMemcpy(b->d_inj, injs.data(), injs.size() * sizeof(InjArgs), cudaMemcpyHostToDevice));
    return SWPC_OK;
}

static int batch_step(swpc_batch *b, int it, const int *d_it) {
    int nwav = 0, max_inj_n = 0;
    for (auto *c : b->members) {
        if (c->nst > 0 && c->wav_what) nwav++;
        max_inj_n = std::max(max_inj_n, std::max(c->ninj_glut, c->ninj_bf));
    }
    const int mask_all = 3;
    const Fields2D f = fields2d(b->kind, b->nm);
    // staged: one launch per member group over that group's tiles
    const int ng = (int)b->group_first.size() - 1;
    auto stress = [&](int mask) {
        if (!b->sti) {
            launch_stress2d(b->kind, b->nm, b->d_models, b->d_tiles, b->ntiles, mask, b->shape, b->stream);
            return cudaGetLastError();
        }
        for (int g = 0; g < ng; g++) {
            const int m0 = b->group_first[g], m1 = b->group_first[g + 1];
            const int t0 = b->tile_first[m0], t1 = b->tile_first[m1];
            const cudaError_t e = launch_stress2d_tma(b->kind, b->nm, b->sti, &b->str_sets[m0], m1 - m0, m0,
                                                      b->d_models, b->d_tiles + t0, t1 - t0, mask, f, b->d_err,
                                                      b->stream);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    auto vel = [&](int mask) {
        if (!b->vti) {
            launch_vel2d(b->kind, b->d_models, b->d_tiles, b->ntiles, mask, b->shape, b->stream);
            return cudaGetLastError();
        }
        for (int g = 0; g < ng; g++) {
            const int m0 = b->group_first[g], m1 = b->group_first[g + 1];
            const int t0 = b->tile_first[m0], t1 = b->tile_first[m1];
            const cudaError_t e = launch_vel2d_tma(b->kind, b->vti, &b->vel_sets[m0], m1 - m0, m0, b->d_models,
                                                   b->d_tiles + t0, t1 - t0, mask, f, b->d_err, b->stream);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    // the Cerjan sponge of the members that run it (absorb__update_*), after
    // the batched update of the phase; their tiles hold no PML cells
    auto sponge = [&](int phase) {
        for (auto *c : b->members)
            if (c->abc == 1) {
                const int rc = launch_cerjan2d(c, phase, b->stream);
                if (rc) return rc;
            }
        return (int)SWPC_OK;
    };
    launch_wav2d(b->d_wav, nwav, b->max_nst, it, d_it, b->stream);
    BCK(stress(mask_all));
    RC(sponge(0));
    launch_inject_multi(b->d_inj, b->ninj, max_inj_n, d_it, it, b->stream);
    if (b->kind == SWPC_KIND_PSV && b->psv_bf_split) {
        // P-SV applies body forces between the interior and absorber velocity
        // updates (src/swpc_psv/main.f90:106-110)
        BCK(vel(1));
        launch_inject_multi(b->d_inj + b->ninj, b->max_inj, max_inj_n, d_it, it, b->stream);
        BCK(vel(2));
        RC(sponge(1));
    } else {
        BCK(vel(mask_all));
        RC(sponge(1));
        launch_inject_multi(b->d_inj + b->ninj, b->max_inj, max_inj_n, d_it, it, b->stream);
    }
    BCK(cudaGetLastError());
    return SWPC_OK;
}

extern "C" int swpc_batch_step(swpc_batch *b, int it) {
    if (!b) return SWPC_ERR_ARG;
    if (it < 1 || it > b->nt) return berr(b, SWPC_ERR_ARG, "time step index outside 1..nt");
    BCK(cudaSetDevice(b->device));
    return batch_step(b, it, nullptr);
}

extern "C" int swpc_batch_run(swpc_batch *b, int it0, int nsteps) {
    if (!b) return SWPC_ERR_ARG;
    if (nsteps <= 0) return SWPC_OK;
    if (it0 < 1 || it0 + nsteps - 1 > b->nt) return berr(b, SWPC_ERR_ARG, "time steps outside 1..nt");
    BCK(cudaSetDevice(b->device));
    if (!b->graph) {
        cudaGraph_t g;
        BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        int rc = batch_step(b, 0, b->d_it);
        if (!rc) launch_advance_it(b->d_it, b->stream);
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (rc) return rc;
        BCK(e);
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        BCK(e);
    }
    BCK(cudaMemcpyAsync(b->d_it, &it0, sizeof(int), cudaMemcpyHostToDevice, b->stream));
    for (int s = 0; s < nsteps; s++) BCK(cudaGraphLaunch(b->graph, b->stream));
    return SWPC_OK;
}

extern "C" int swpc_batch_sync(swpc_batch *b) {
    if (!b) return SWPC_ERR_ARG;
    BCK(cudaStreamSynchronize(b->stream));
    int h = 0;
    BCK(cudaMemcpy(&h, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) return berr(b, SWPC_ERR_CUDA, "a staged tile copy did not complete (TMA wait timed out)");
    return SWPC_OK;
}

static int drop_graph(swpc_batch *b) {
    BCK(cudaSetDevice(b->device));
    BCK(cudaStreamSynchronize(b->stream));
    if (b->graph) {
        BCK(cudaGraphExecDestroy(b->graph));
        b->graph = nullptr;
    }
    return SWPC_OK;
}

extern "C" int swpc_batch_set_staged(swpc_batch *b, int stress_ti, int vel_ti) {
    if (!b) return SWPC_ERR_ARG;
    if ((stress_ti && !staged2d_ti_ok(stress_ti)) || (vel_ti && !staged2d_ti_ok(vel_ti)))
        return berr(b, SWPC_ERR_ARG, "staged kernels take 4, 8 or 16 threads along i (0: tile-walking kernels)");
    RCB(drop_graph(b));
    if ((stress_ti || vel_ti) && b->shape.ti * b->shape.ri != kTileI2D) RCB(set_tiles(b, kDefaultTiles));
    b->sti = stress_ti;
    b->vti = vel_ti;
    return SWPC_OK;
}

extern "C" int swpc_batch_get_launch(const swpc_batch *b, int *out) {
    if (!b || !out) return SWPC_ERR_ARG;
    out[0] = b->shape.ti; out[1] = b->shape.ri; out[2] = b->shape.blocks_per_sm;
    out[3] = b->sti; out[4] = b->vti;
    return SWPC_OK;
}

extern "C" int swpc_batch_set_shape(swpc_batch *b, int ti, int ri, int bps) {
    if (!b) return SWPC_ERR_ARG;
    if (ti < 1 || ri < 1 || bps < 0 || 32 * ti > 256 || ri > 64 || bps > 64)
        return berr(b, SWPC_ERR_ARG, "tile shape out of range (32*ti <= 256, 1 <= ri <= 64, 0 <= bps <= 64)");
    RCB(drop_graph(b));
    return set_tiles(b, TileShape{ti, ri, bps});
}

extern "C" int swpc_batch_autotune(swpc_batch *b, int it0, int reps, int *used, int *best_ti, int *best_ri,
                                   int *best_bps) {
    // candidates: staged kernels (threads along i of the stress and velocity
    // CTAs) on 32 x 16 tiles, then tile-walking kernels of several shapes
    struct Cand {
        TileShape ts;
        int sti, vti;
    };
    static const Cand cand[] = {{{4, 4, 0}, 8, 8},  {{4, 4, 0}, 4, 4},  {{4, 4, 0}, 16, 16}, {{4, 4, 0}, 8, 4},
                                {{4, 4, 0}, 4, 8},  {{4, 4, 0}, 16, 8}, {{4, 4, 0}, 0, 0},   {{4, 2, 0}, 0, 0},
                                {{4, 8, 0}, 0, 0},  {{2, 8, 0}, 0, 0},  {{8, 4, 0}, 0, 0},   {{4, 1, 16}, 0, 0}};
    const int ncand = (int)(sizeof(cand) / sizeof(cand[0]));
    if (!b || !used || reps < 1) return SWPC_ERR_ARG;
    if (it0 < 1 || it0 + ncand * reps - 1 > b->nt) return berr(b, SWPC_ERR_ARG, "not enough time steps left to tune");
    RCB(drop_graph(b));
    cudaEvent_t e0, e1;
    BCK(cudaEventCreate(&e0));
    BCK(cudaEventCreate(&e1));
    float best = 0.f;
    Cand pick = cand[0];
    int it = it0, rc = SWPC_OK;
    for (int n = 0; n < ncand && !rc; n++) {
        rc = set_tiles(b, cand[n].ts);
        if (rc) break;
        b->sti = cand[n].sti;
        b->vti = cand[n].vti;
        cudaStreamSynchronize(b->stream);
        cudaEventRecord(e0, b->stream);
        for (int r = 0; r < reps && !rc; r++) rc = batch_step(b, it++, nullptr);
        cudaEventRecord(e1, b->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) { rc = berr(b, SWPC_ERR_CUDA, "autotune step failed"); break; }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (n == 0 || ms < best) { best = ms; pick = cand[n]; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    RCB(set_tiles(b, pick.ts));
    b->sti = pick.sti;
    b->vti = pick.vti;
    b->tuned = true;
    *used = it - it0;
    if (best_ti) *best_ti = pick.ts.ti;
    if (best_ri) *best_ri = pick.ts.ri;
    if (best_bps) *best_bps = pick.ts.blocks_per_sm;
    return SWPC_OK;
}

extern "C" int swpc_batch_time_steps(swpc_batch *b, int it0, int nsteps, float *ms) {
    if (!b || !ms) return SWPC_ERR_ARG;
    BCK(cudaSetDevice(b->device));
    cudaEvent_t e0, e1;
    BCK(cudaEventCreate(&e0));
    BCK(cudaEventCreate(&e1));
    BCK(cudaStreamSynchronize(b->stream));
    BCK(cudaEventRecord(e0, b->stream));
    int rc = swpc_batch_run(b, it0, nsteps);
    BCK(cudaEventRecord(e1, b->stream));
    BCK(cudaEventSynchronize(e1));
    BCK(cudaEventElapsedTime(ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}
