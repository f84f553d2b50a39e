// swpc_fbatch.cu -- reciprocity batch: many independent 3D wavefields, each
// driven by its own single force (green__source, m_green.f90:597-632), over
// the one medium of a context.
//
// Every member runs exactly the reference step of a green-mode run
// (src/swpc_3d/main.f90:125-144 with green__source after the velocity
// update): the same per-cell routines as the single-run kernels
// (stress_cell, vel_cell, wav_station), so a member is bitwise equal to a
// run of its own.  What the batch changes is the launch: one launch per half
// step covers all members, and consecutive blocks of the launch take the
// same cell tile of consecutive members, so the medium of a tile is read from
// HBM once and served from L2 to the other members.  The tile order walks
// i-strips of `strip` cells along j (strip by strip), which keeps the
// velocity / stress planes that the j-stencil re-reads resident in L2 even
// with all members in flight.  That is the flat form; by default the batch
// runs the TMA-staged kernels of swpc3d_tma.cu, whose CTAs copy the medium of a
// tile once and then the boxes of a group of members (members per CTA and
// tile chosen by swpc_fbatch_set_launch / swpc_fbatch_autotune).
//
// Layout: one slab of nmem member blocks, each block the member's V, S and R
// (nfs = 9 + 6 nm fields of the context's cell count, the order of the
// context's slab), so member m's copy of a field sits at m * stride (stride =
// nfs cells); the PML auxiliaries are one array per auxiliary with the
// members at m * astride (the context's compact PML cell count).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "swpc_ctx.h"
#include "swpc_kernels.cuh"
#include "swpc3d_cell.cuh"
#include "swpc_tma.h"

namespace swpc {
int stime_table(swpc_ctx *c, float **dst, int nsrc, const float *srcprm, int stftype, bool half);
bool green_entries(const swpc_ctx *c, int isrc, int jsrc, int ksrc, char cmp, std::vector<InjEntry> &v);
int copy_box(swpc_ctx *c, float *dev, const float *host_in, float *host_out, int ld_k, int ld_i);
}  // namespace swpc

using namespace swpc;

struct swpc_fbatch {
    swpc_ctx *c = nullptr;
    int nmem = 0;
    long long stride = 0, astride = 0;
    float *slab = nullptr;
    int nfs = 0;
    float *V[3] = {}, *S[6] = {}, *R[18] = {}, *aux[18] = {};   // member 0 (V, S, R inside the slab)
    float *wav[4] = {};            // per kind: nmem blocks of (nst, ncmp, ntw)
    float *uacc = nullptr, *eacc = nullptr;
    // green__store of every member at the context's green table (when set up)
    float *g_acc = nullptr, *g_out = nullptr;
    int g_ng = 0;
    // green sources: entries tagged with their member, forces per member
    std::vector<std::vector<InjEntry>> h_inj;
    std::vector<float> h_prm;      // (2, nmem) tbeg, trise
    std::vector<int> h_stf;        // stftype per member (-1: no source)
    InjEntry *inj = nullptr;
    int *inj_mem = nullptr;
    int ninj = 0;
    float *stf = nullptr;          // (nt, nmem)
    bool src_dirty = true;
    int strip = 0;                 // i-strip width in cells (0: automatic), flat kernels
    bool staged = false;           // TMA-staged kernels (FP32 contexts with a field slab)
    int sbi = 4, sbj = 2, smpc = 2, vbi = 4, vbj = 2, vmpc = 2;   // staged tiles and members per CTA
    int tiles_first = 0;           // staged launch order (see swpc3d_tma.cu tile_of)
    void *tmaps = nullptr;         // swpc::TmaMaps over the batch slab and the context's medium
    int tma_key[4] = {-1, -1, -1, -1};
    int *d_it = nullptr;
    cudaGraphExec_t graph = nullptr;
    long long bytes = 0;
};

namespace {

struct BatchGrid {
    int nmem, nkb, nib, njb, sw;   // members, k / i / j blocks, strip width in i-blocks
    long long stride, astride;
};

// block -> (member, cell): member fastest, then k-block, then i within the
// strip, then j, then the strip
__device__ __forceinline__ bool batch_cell(const BatchGrid &bg, const Geo &g, int &m, int &k, int &i, int &j) {
    long long b = blockIdx.x;
    m = (int)(b % bg.nmem);
    b /= bg.nmem;
    const int kb = (int)(b % bg.nkb);
    b /= bg.nkb;
    const long long per = (long long)bg.sw * bg.njb;
    const int s = (int)(b / per);
    const int r = (int)(b % per);
    const int w = min(bg.sw, bg.nib - s * bg.sw);
    const int ib = s * bg.sw + r % w, jb = r / w;
    k = 1 + kb * 32 + threadIdx.x;
    i = 1 + ib * blockDim.y + threadIdx.y;
    j = 1 + jb * blockDim.z + threadIdx.z;
    return k <= g.nz && i <= g.nx && j <= g.ny;
}

template <int NM>
__global__ void __launch_bounds__(256, 2) stress3d_batch_kernel(const Str3Args a, const BatchGrid bg) {
    int m, k, i, j;
    if (!batch_cell(bg, a.g, m, k, i, j)) return;
    stress_cell<NM, PREC_F32>(a, k, i, j, m * bg.stride, m * bg.astride);
}

__global__ void __launch_bounds__(256, 3) vel3d_batch_kernel(const Vel3Args a, const BatchGrid bg) {
    int m, k, i, j;
    if (!batch_cell(bg, a.g, m, k, i, j)) return;
    vel_cell<PREC_F32>(a, k, i, j, m * bg.stride, m * bg.astride);
}

// wav__store for every member: blockIdx.y = member
__global__ void wav3d_batch_kernel(const Wav3Args a, long long stride, int ncv, int ncs) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.nst) return;
    const int m = blockIdx.y;
    const long long so = m * stride;
    const long long w3 = (long long)m * a.nst * ncv * a.ntw, w6 = (long long)m * a.nst * ncs * a.ntw;
    Wav3Args b = a;
    b.Vx = a.Vx + so; b.Vy = a.Vy + so; b.Vz = a.Vz + so;
    b.Sxx = a.Sxx + so; b.Syy = a.Syy + so; b.Szz = a.Szz + so;
    b.Syz = a.Syz + so; b.Sxz = a.Sxz + so; b.Sxy = a.Sxy + so;
    b.uacc = a.uacc + (long long)m * 3 * a.nst;
    b.eacc = a.eacc + (long long)m * 6 * a.nst;
    b.wav_v = a.wav_v + w3; b.wav_u = a.wav_u + w3;
    b.wav_s = a.wav_s + w6; b.wav_e = a.wav_e + w6;
    wav_station(b, n);
}

// green__source of every member (m_green.f90:615-627): fv = f * dt_dxyz *
// stf ; V += b * fv / 2, on the member's copy of V
struct GreenArgs {
    const InjEntry *list;
    const int *mem;
    int n, nt, nmem;
    int it;
    const int *d_it;
    const float *stf;     // (nt, nmem)
    float dt_dxyz;
    float *V[3];
    const float *b[3];
    long long stride;
};

__global__ void green_batch_kernel(const GreenArgs a) {
    const int it = a.d_it ? *a.d_it : a.it;
    if (it < 1 || it > a.nt) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.n) return;
    const InjEntry en = a.list[n];
    const int m = a.mem[n];
    const float st = a.stf[(long long)(it - 1) * a.nmem + m];
    float *f = (en.field == 0 ? a.V[0] : en.field == 1 ? a.V[1] : a.V[2]) + m * a.stride;
    const float fv = en.coef * a.dt_dxyz * st;
    const float b = (en.bfield == 0 ? a.b[0] : en.bfield == 1 ? a.b[1] : a.b[2])[en.cell];
    f[en.cell] = f[en.cell] + b * fv / 2;
}

__global__ void fb_advance_it_kernel(int *d_it) { *d_it = *d_it + 1; }

int ferr(swpc_fbatch *b, int code, const std::string &m) { return set_err(b->c, code, m); }

}  // namespace

#define FCK(call)                                              \
    do {                                                       \
        int _rc = cuda_check(b->c, (call), #call);             \
        if (_rc) return _rc;                                   \
    } while (0)
#define FRC(call)                \
    do {                         \
        int _rc = (call);        \
        if (_rc) return _rc;     \
    } while (0)

template <typename T>
static int falloc(swpc_fbatch *b, T **p, size_t n) {
    int rc = dalloc(b->c, p, n);
    if (!rc) b->bytes += (long long)(n * sizeof(T));
    return rc;
}

static void fb_free(swpc_fbatch *b) {
    auto f = [](void *p) { if (p) cudaFree(p); };
    f(b->slab);
    for (auto p : b->aux) f(p);
    delete static_cast<TmaMaps *>(b->tmaps);
    for (auto p : b->wav) f(p);
    f(b->uacc); f(b->eacc); f(b->inj); f(b->inj_mem); f(b->stf); f(b->d_it); f(b->g_acc); f(b->g_out);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->c) b->c->bytes -= b->bytes;
}

static int wav_ncmp(int q) { return q < 2 ? 3 : 6; }

extern "C" int swpc_fbatch_create(swpc_ctx *c, int nmem, swpc_fbatch **out) {
    if (!c || !out || nmem < 1) return SWPC_ERR_ARG;
    *out = nullptr;
    if (c->kind != SWPC_KIND_3D) return set_err(c, SWPC_ERR_ARG, "the reciprocity batch is a 3D feature");
    if (c->prec != SWPC_PREC_F32) return set_err(c, SWPC_ERR_ARG, "the reciprocity batch needs FP32 storage");
    if (c->abc != 0) return set_err(c, SWPC_ERR_STATE, "the reciprocity batch runs with the PML");
    if (c->pw_mode) return set_err(c, SWPC_ERR_STATE, "the reciprocity batch has no plane-wave mode");
    if (!c->medium_ready || !c->kernel_ready || (c->d.na > 0 && !c->absorb_ready))
        return set_err(c, SWPC_ERR_STATE, "medium, kernel and absorber setup must precede swpc_fbatch_create");
    if (cudaSetDevice(c->device) != cudaSuccess) return set_err(c, SWPC_ERR_CUDA, "cudaSetDevice failed");
    auto *b = new swpc_fbatch();
    b->c = c;
    b->nmem = nmem;
    b->nfs = 9 + 6 * c->d.nm;
    b->stride = (long long)b->nfs * c->g.ncell;
    b->astride = c->npml;
    int rc = falloc(b, &b->slab, (size_t)b->stride * nmem);
    if (!rc) {
        auto F = [&](int f) { return b->slab + (size_t)f * c->g.ncell; };
        for (int q = 0; q < 3; q++) b->V[q] = F(q);
        for (int q = 0; q < 6; q++) b->S[q] = F(3 + q);
        for (int comp = 0; comp < 6; comp++)
            for (int m = 0; m < c->d.nm; m++) b->R[comp * 3 + m] = F(9 + comp * c->d.nm + m);
        b->staged = c->slab != nullptr;
    }
    if (c->npml > 0)
        for (int q = 0; q < 18 && !rc; q++) rc = falloc(b, &b->aux[q], (size_t)c->npml * nmem);
    const int nst = std::max(c->nst, 1);
    for (int q = 0; q < 4 && !rc; q++)
        if (c->wav_what & (1 << q)) rc = falloc(b, &b->wav[q], (size_t)c->ntw * wav_ncmp(q) * nst * nmem);
    if (!rc) rc = falloc(b, &b->uacc, (size_t)3 * nst * nmem);
    if (!rc) rc = falloc(b, &b->eacc, (size_t)6 * nst * nmem);
    if (!rc) rc = falloc(b, &b->d_it, 1);
    if (!rc && c->ng > 0) {
        // green__store for every member at the context's green table
        b->g_ng = c->ng;
        rc = falloc(b, &b->g_acc, (size_t)12 * c->ng * nmem);
        if (!rc) rc = falloc(b, &b->g_out, (size_t)c->ng_ntw * c->ng_cmp * c->ng * nmem);
    }
    if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    if (rc) {
        fb_free(b);
        delete b;
        return rc;
    }
    c->nfbatch++;
    b->h_inj.assign(nmem, {});
    b->h_prm.assign(2 * (size_t)nmem, 0.f);
    b->h_stf.assign(nmem, -1);
    *out = b;
    return SWPC_OK;
}

extern "C" int swpc_fbatch_destroy(swpc_fbatch *b) {
    if (!b) return SWPC_OK;
    cudaSetDevice(b->c->device);
    cudaStreamSynchronize(b->c->stream);
    b->c->nfbatch--;
    fb_free(b);
    delete b;
    return SWPC_OK;
}

extern "C" int swpc_fbatch_green_source(swpc_fbatch *b, int member, int isrc, int jsrc, int ksrc, char cmp,
                                        float green_tbeg, float green_trise, int stftype) {
    if (!b) return SWPC_ERR_ARG;
    if (member < 0 || member >= b->nmem) return ferr(b, SWPC_ERR_ARG, "member index outside 0..nmem-1");
    if (cmp != 'x' && cmp != 'y' && cmp != 'z') return ferr(b, SWPC_ERR_ARG, "green_cmp must be x, y or z");
    std::vector<InjEntry> v;
    if (!green_entries(b->c, isrc, jsrc, ksrc, cmp, v))
        return ferr(b, SWPC_ERR_ARG, "green source cell outside the memory box");
    b->h_inj[member] = v;
    b->h_prm[2 * member] = green_tbeg;
    b->h_prm[2 * member + 1] = green_trise;
    b->h_stf[member] = stftype;
    b->src_dirty = true;
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
    return SWPC_OK;
}

extern "C" int swpc_fbatch_set_launch(swpc_fbatch *b, int kernel, int mpc, int bi, int bj) {
    if (!b) return SWPC_ERR_ARG;
    if (kernel == 0) {
        b->staged = false;
    } else if (kernel == 5 || kernel == 6) {
        if (!b->c->slab) return ferr(b, SWPC_ERR_ARG, "staged kernels need an FP32 context");
        if (!(kernel == 5 ? tma_shape_ok(bi, bj, mpc) : tma_vel_shape_ok(bi, bj, mpc)))
            return ferr(b, SWPC_ERR_ARG, "no compiled staged kernel for this tile and member count");
        b->staged = true;
        if (kernel == 5) { b->sbi = bi; b->sbj = bj; b->smpc = mpc; }
        else { b->vbi = bi; b->vbj = bj; b->vmpc = mpc; }
    } else if (kernel == 7) {
        b->tiles_first = mpc != 0;
    } else {
        return ferr(b, SWPC_ERR_ARG, "kernel must be 0 (flat), 5 (staged stress), 6 (staged velocity) or 7 (order)");
    }
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
    return SWPC_OK;
}

extern "C" int swpc_fbatch_set_strip(swpc_fbatch *b, int strip_cells) {
    if (!b || strip_cells < 0) return SWPC_ERR_ARG;
    b->strip = strip_cells;
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
    return SWPC_OK;
}

static int upload_sources(swpc_fbatch *b) {
    if (!b->src_dirty) return SWPC_OK;
    swpc_ctx *c = b->c;
    std::vector<InjEntry> all;
    std::vector<int> mem;
    for (int m = 0; m < b->nmem; m++)
        for (auto &e : b->h_inj[m]) { all.push_back(e); mem.push_back(m); }
    if (b->inj) { cudaFree(b->inj); b->inj = nullptr; }
    if (b->inj_mem) { cudaFree(b->inj_mem); b->inj_mem = nullptr; }
    FRC(dalloc(c, &b->inj, all.size()));
    FRC(dalloc(c, &b->inj_mem, mem.size()));
    if (!all.empty()) {
        FCK(cudaMemcpyAsync(b->inj, all.data(), all.size() * sizeof(InjEntry), cudaMemcpyHostToDevice, c->stream));
        FCK(cudaMemcpyAsync(b->inj_mem, mem.data(), mem.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    }
    b->ninj = (int)all.size();
    // one table per source-time function code: members without a source keep zeros
    const int nt = c->d.nt;
    std::vector<float> tab((size_t)nt * b->nmem, 0.f);
    for (int m = 0; m < b->nmem; m++) {
        if (b->h_stf[m] < 0) continue;
        float *one = nullptr;
        FRC(stime_table(c, &one, 1, &b->h_prm[2 * m], b->h_stf[m], false));
        std::vector<float> h(nt);
        cudaError_t e = cudaMemcpy(h.data(), one, nt * sizeof(float), cudaMemcpyDeviceToHost);
        cudaFree(one);
        c->bytes -= (long long)nt * sizeof(float);
        FCK(e);
        for (int it = 0; it < nt; it++) tab[(size_t)it * b->nmem + m] = h[it];
    }
    if (b->stf) { cudaFree(b->stf); b->stf = nullptr; }
    FRC(dalloc(c, &b->stf, tab.size()));
    FCK(cudaMemcpyAsync(b->stf, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    FCK(cudaStreamSynchronize(c->stream));
    b->src_dirty = false;
    return SWPC_OK;
}

static BatchGrid batch_grid(const swpc_fbatch *b, int bi, int bj) {
    const swpc_ctx *c = b->c;
    BatchGrid bg;
    bg.nmem = b->nmem;
    bg.nkb = (c->g.nz + 31) / 32;
    bg.nib = (c->g.nx + bi - 1) / bi;
    bg.njb = (c->g.ny + bj - 1) / bj;
    int strip = b->strip;
    if (strip <= 0) {
        // the V planes j-2..j+1 of all members in one strip: about 40 MB of L2
        const double per_cell = 4.0 * 3 * 4 * c->g.nz * (double)b->nmem;
        strip = (int)std::max(32.0, std::min((double)c->g.nx, 40e6 / per_cell));
    }
    bg.sw = std::max(1, std::min(bg.nib, (strip + bi - 1) / bi));
    bg.stride = b->stride;
    bg.astride = b->astride;
    return bg;
}

// tensor maps of the staged kernels: member state over the batch slab, the
// medium over the context's slab
static int fb_tma_ready(swpc_fbatch *b) {
    const int key[4] = {b->sbi, b->sbj, b->vbi, b->vbj};
    if (b->tmaps && std::equal(key, key + 4, b->tma_key)) return SWPC_OK;
    if (!b->tmaps) b->tmaps = new TmaMaps();
    TmaMaps &m = *static_cast<TmaMaps *>(b->tmaps);
    swpc_ctx *c = b->c;
    const TmaSlabs s{b->slab, (long long)b->nfs * b->nmem, c->slab, c->slab_nf};
    if (!tma_encode_stress(m, s, c->g, c->d.nm, key[0], key[1]) || !tma_encode_vel(m, s, c->g, key[2], key[3]))
        return ferr(b, SWPC_ERR_CUDA, "cuTensorMapEncodeTiled failed for the batch slab");
    std::copy(key, key + 4, b->tma_key);
    return SWPC_OK;
}

static TmaTiles fb_tiles(const swpc_fbatch *b, int bi, int bj, int mpc, int nfields) {
    // tiles fastest: one member group's tiles run at a time; else all groups of a tile
    TmaTiles t = tma_tiles(b->c, bi, bj, b->nmem, mpc, nfields, b->tiles_first ? mpc : b->nmem);
    t.f_member = b->nfs;
    t.so = b->stride;
    t.ao = b->astride;
    t.tiles_first = b->tiles_first;
    return t;
}

static int fb_step_body(swpc_fbatch *b, int it, const int *d_it) {
    swpc_ctx *c = b->c;
    const Geo &g = c->g;
    // wav__store
    if (c->nst > 0 && c->wav_what) {
        Wav3Args a;
        memset(&a, 0, sizeof(a));
        a.g = g; a.nst = c->nst; a.ntw = c->ntw; a.ntdec_w = c->ntdec_w; a.what = c->wav_what;
        a.it = it; a.d_it = d_it; a.st = c->st_ijk;
        a.Vx = b->V[0]; a.Vy = b->V[1]; a.Vz = b->V[2];
        a.Sxx = b->S[0]; a.Syy = b->S[1]; a.Szz = b->S[2]; a.Syz = b->S[3]; a.Sxz = b->S[4]; a.Sxy = b->S[5];
        a.uacc = b->uacc; a.eacc = b->eacc;
        a.wav_v = b->wav[0]; a.wav_u = b->wav[1]; a.wav_s = b->wav[2]; a.wav_e = b->wav[3];
        a.M0 = c->M0; a.UC = c->UC; a.dt = c->d.dt;
        memcpy(a.r40, c->r40, sizeof(a.r40)); memcpy(a.r41, c->r41, sizeof(a.r41));
        a.scale = c->d_scale;   // FP32 storage: every scale 1
        const bool sample = d_it || (it - 1) % c->ntdec_w == 0 || (c->wav_what & (SWPC_WAV_U | SWPC_WAV_STRAIN));
        if (sample) {
            wav3d_batch_kernel<<<dim3((c->nst + 127) / 128, b->nmem), 128, 0, c->stream>>>(a, b->stride, 3, 6);
            FCK(cudaGetLastError());
        }
    }
    // green__store beside wav__store, as the context's step
    if (b->g_ng > 0) {
        if (c->ng != b->g_ng) return ferr(b, SWPC_ERR_STATE, "the context's green table changed after the batch");
        FRC(green_store_members(c, b->V, b->stride, b->nmem, b->g_acc, b->g_out, it, d_it));
    }
    const int mask = c->d.na > 0 ? 3 : 1;
    // stress (kernel__update_stress + absorb_p__update_stress)
    {
        Str3Args a;
        memset(&a, 0, sizeof(a));
        a.g = g; a.ibk = c->ibk; a.iek = c->iek; a.jbk = c->jbk; a.jek = c->jek; a.kek = c->kek;
        a.Vx = b->V[0]; a.Vy = b->V[1]; a.Vz = b->V[2];
        a.Sxx = b->S[0]; a.Syy = b->S[1]; a.Szz = b->S[2]; a.Syz = b->S[3]; a.Sxz = b->S[4]; a.Sxy = b->S[5];
        for (int q = 0; q < 18; q++) a.R[q] = b->R[q];
        a.lam = c->med[1]; a.mu = c->med[2]; a.taup = c->med[3]; a.taus = c->med[4];
        a.muyz = c->med[8]; a.muxz = c->med[9]; a.muxy = c->med[10];
        a.band = c->band; a.pmlcol = c->pmlcol;
        for (int q = 0; q < 9; q++) a.aV[q] = b->aux[q];
        a.gxc = c->gx[0]; a.gxe = c->gx[1]; a.gyc = c->gy[0]; a.gye = c->gy[1]; a.gzc = c->gz[0]; a.gze = c->gz[1];
        memcpy(a.e40, c->e40, sizeof(a.e40)); memcpy(a.e41, c->e41, sizeof(a.e41)); memcpy(a.r20, c->r20, sizeof(a.r20));
        memcpy(a.c1, c->c1, sizeof(a.c1)); memcpy(a.c2, c->c2, sizeof(a.c2)); memcpy(a.d1, c->d1, sizeof(a.d1));
        a.d2 = c->d2;
        a.dt = c->d.dt;
        a.mask = mask;
        a.scale = c->d_scale;   // FP32 storage: every scale 1
        if (b->staged) {
            FRC(fb_tma_ready(b));
            const TmaTiles t = fb_tiles(b, b->sbi, b->sbj, b->smpc, kStressFields(b->c));
            FCK(launch_stress3d_tma(*static_cast<TmaMaps *>(b->tmaps), a, t, c->d.nm, b->sbi, b->sbj, b->smpc,
                                    c->stream));
        } else {
        const BatchGrid bg = batch_grid(b, c->bi, c->bj);
        const long long nblk = (long long)bg.nmem * bg.nkb * bg.nib * bg.njb;
        if (nblk > 0x7fffffffLL) return ferr(b, SWPC_ERR_LIMIT, "batch grid above 2^31-1 blocks");
        const dim3 block(32, c->bi, c->bj);
        switch (c->d.nm) {
        case 0: stress3d_batch_kernel<0><<<(unsigned)nblk, block, 0, c->stream>>>(a, bg); break;
        case 1: stress3d_batch_kernel<1><<<(unsigned)nblk, block, 0, c->stream>>>(a, bg); break;
        case 2: stress3d_batch_kernel<2><<<(unsigned)nblk, block, 0, c->stream>>>(a, bg); break;
        default: stress3d_batch_kernel<3><<<(unsigned)nblk, block, 0, c->stream>>>(a, bg); break;
        }
        FCK(cudaGetLastError());
        }
    }
    // velocity (kernel__update_vel + absorb_p__update_vel)
    {
        Vel3Args a;
        memset(&a, 0, sizeof(a));
        a.g = g; a.ibk = c->ibk; a.iek = c->iek; a.jbk = c->jbk; a.jek = c->jek; a.kek = c->kek;
        a.Vx = b->V[0]; a.Vy = b->V[1]; a.Vz = b->V[2];
        a.Sxx = b->S[0]; a.Syy = b->S[1]; a.Szz = b->S[2]; a.Syz = b->S[3]; a.Sxz = b->S[4]; a.Sxy = b->S[5];
        a.bx = c->med[5]; a.by = c->med[6]; a.bz = c->med[7];
        a.band = c->band; a.pmlcol = c->pmlcol;
        for (int q = 0; q < 9; q++) a.aS[q] = b->aux[9 + q];
        a.gxc = c->gx[0]; a.gxe = c->gx[1]; a.gyc = c->gy[0]; a.gye = c->gy[1]; a.gzc = c->gz[0]; a.gze = c->gz[1];
        memcpy(a.e40, c->e40, sizeof(a.e40)); memcpy(a.e41, c->e41, sizeof(a.e41)); memcpy(a.r20, c->r20, sizeof(a.r20));
        a.dt = c->d.dt;
        a.mask = mask;
        a.scale = c->d_scale;   // FP32 storage: every scale 1
        if (b->staged) {
            FRC(fb_tma_ready(b));
            const TmaTiles t = fb_tiles(b, b->vbi, b->vbj, b->vmpc, kVelFields);
            FCK(launch_vel3d_tma(*static_cast<TmaMaps *>(b->tmaps), a, t, b->vbi, b->vbj, b->vmpc, c->stream));
        } else {
            const BatchGrid bg = batch_grid(b, c->vbi, c->vbj);
            const long long nblk = (long long)bg.nmem * bg.nkb * bg.nib * bg.njb;
            if (nblk > 0x7fffffffLL) return ferr(b, SWPC_ERR_LIMIT, "batch grid above 2^31-1 blocks");
            vel3d_batch_kernel<<<(unsigned)nblk, dim3(32, c->vbi, c->vbj), 0, c->stream>>>(a, bg);
            FCK(cudaGetLastError());
        }
    }
    // green__source of every member
    if (b->ninj > 0) {
        GreenArgs a;
        a.list = b->inj; a.mem = b->inj_mem; a.n = b->ninj; a.nt = c->d.nt; a.nmem = b->nmem;
        a.it = it; a.d_it = d_it; a.stf = b->stf;
        a.dt_dxyz = c->d.dt / (c->d.dx * c->d.dy * c->d.dz);
        for (int q = 0; q < 3; q++) { a.V[q] = b->V[q]; a.b[q] = c->med[5 + q]; }
        a.stride = b->stride;
        green_batch_kernel<<<(b->ninj + 127) / 128, 128, 0, c->stream>>>(a);
        FCK(cudaGetLastError());
    }
    return SWPC_OK;
}

extern "C" int swpc_fbatch_step(swpc_fbatch *b, int it) {
    if (!b) return SWPC_ERR_ARG;
    if (it < 1 || it > b->c->d.nt) return ferr(b, SWPC_ERR_ARG, "time step index outside 1..nt");
    FCK(cudaSetDevice(b->c->device));
    FRC(upload_sources(b));
    return fb_step_body(b, it, nullptr);
}

static int fb_graph(swpc_fbatch *b) {
    if (b->graph) return SWPC_OK;
    swpc_ctx *c = b->c;
    FRC(upload_sources(b));
    cudaGraph_t graph;
    FCK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = fb_step_body(b, 0, b->d_it);
    if (!rc) fb_advance_it_kernel<<<1, 1, 0, c->stream>>>(b->d_it);
    cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    if (rc) return rc;
    FCK(e);
    e = cudaGraphInstantiate(&b->graph, graph, 0);
    cudaGraphDestroy(graph);
    FCK(e);
    return SWPC_OK;
}

extern "C" int swpc_fbatch_run(swpc_fbatch *b, int it0, int nsteps) {
    if (!b) return SWPC_ERR_ARG;
    if (nsteps <= 0) return SWPC_OK;
    if (it0 < 1 || it0 + nsteps - 1 > b->c->d.nt) return ferr(b, SWPC_ERR_ARG, "time steps outside 1..nt");
    FCK(cudaSetDevice(b->c->device));
    FRC(fb_graph(b));
    FCK(cudaMemcpyAsync(b->d_it, &it0, sizeof(int), cudaMemcpyHostToDevice, b->c->stream));
    for (int n = 0; n < nsteps; n++) FCK(cudaGraphLaunch(b->graph, b->c->stream));
    return SWPC_OK;
}

extern "C" int swpc_fbatch_time_steps(swpc_fbatch *b, int it0, int nsteps, float *ms) {
    if (!b || !ms) return SWPC_ERR_ARG;
    swpc_ctx *c = b->c;
    FCK(cudaSetDevice(c->device));
    FRC(fb_graph(b));
    cudaEvent_t e0, e1;
    FCK(cudaEventCreate(&e0));
    FCK(cudaEventCreate(&e1));
    FCK(cudaStreamSynchronize(c->stream));
    FCK(cudaEventRecord(e0, c->stream));
    int rc = swpc_fbatch_run(b, it0, nsteps);
    FCK(cudaEventRecord(e1, c->stream));
    FCK(cudaEventSynchronize(e1));
    FCK(cudaEventElapsedTime(ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

// time `reps` steps of the current launch after one untimed replay of the
// (re)built graph; advances *it by 2 reps
static int fb_time(swpc_fbatch *b, int *it, int reps, float *ms) {
    FRC(swpc_fbatch_run(b, *it, reps));
    *it += reps;
    FRC(swpc_fbatch_time_steps(b, *it, reps, ms));
    *it += reps;
    return SWPC_OK;
}

extern "C" int swpc_fbatch_autotune(swpc_fbatch *b, int it0, int reps, int *steps_used, int *strip_out) {
    if (!b || reps < 1) return SWPC_ERR_ARG;
    int it = it0;
    const int nt = b->c->d.nt;
    if (b->staged) {
        // staged kernels: members per CTA and tile of the stress kernel, then of the velocity kernel
        // launch order with the current shapes, then the shapes
        {
            int best = 0;
            float best_ms = 1e30f;
            for (int q = 0; q < 2 && it + 2 * reps - 1 <= nt; q++) {
                FRC(swpc_fbatch_set_launch(b, 7, q, 0, 0));
                float ms = 0.f;
                FRC(fb_time(b, &it, reps, &ms));
                if (ms < best_ms) { best_ms = ms; best = q; }
            }
            FRC(swpc_fbatch_set_launch(b, 7, best, 0, 0));
        }
        const int sc[][3] = {{4, 2, 2}, {4, 4, 1}, {2, 4, 2}, {2, 2, 2}, {2, 2, 4}, {4, 1, 4}};
        const int vc[][3] = {{4, 2, 2}, {4, 4, 1}, {4, 2, 1}, {2, 2, 2}, {2, 2, 4}, {4, 1, 4}};
        for (int kernel = 5; kernel <= 6; kernel++) {
            const int(*cand)[3] = kernel == 5 ? sc : vc;
            int best = 0;
            float best_ms = 1e30f;
            for (int q = 0; q < 6; q++) {
                if (it + 2 * reps - 1 > nt) break;
                FRC(swpc_fbatch_set_launch(b, kernel, cand[q][2], cand[q][0], cand[q][1]));
                float ms = 0.f;
                FRC(fb_time(b, &it, reps, &ms));
                if (ms < best_ms) { best_ms = ms; best = q; }
            }
            FRC(swpc_fbatch_set_launch(b, kernel, cand[best][2], cand[best][0], cand[best][1]));
        }
        if (strip_out) *strip_out = 0;
    } else {
        const int nx = b->c->g.nx;
        std::vector<int> cand = {32, 64, 128, 256, 512};
        cand.erase(std::remove_if(cand.begin(), cand.end(), [&](int w) { return w > nx; }), cand.end());
        cand.push_back(nx);
        int best = cand[0];
        float best_ms = 1e30f;
        for (int w : cand) {
            if (it + 2 * reps - 1 > nt) break;
            FRC(swpc_fbatch_set_strip(b, w));
            float ms = 0.f;
            FRC(fb_time(b, &it, reps, &ms));
            if (ms < best_ms) { best_ms = ms; best = w; }
        }
        FRC(swpc_fbatch_set_strip(b, best));
        if (strip_out) *strip_out = best;
    }
    if (steps_used) *steps_used = it - it0;
    return SWPC_OK;
}

extern "C" int swpc_fbatch_get_launch(const swpc_fbatch *b, int *out) {
    if (!b || !out) return SWPC_ERR_ARG;
    const int v[9] = {b->staged ? 1 : 0, b->strip, b->sbi, b->sbj, b->smpc, b->vbi, b->vbj, b->vmpc, b->tiles_first};
    std::copy(v, v + 9, out);
    return SWPC_OK;
}

extern "C" int swpc_fbatch_sync(swpc_fbatch *b) {
    if (!b) return SWPC_ERR_ARG;
    FCK(cudaSetDevice(b->c->device));
    FCK(cudaStreamSynchronize(b->c->stream));
    return SWPC_OK;
}

extern "C" int swpc_fbatch_wav_fetch(swpc_fbatch *b, int member, int what, float *out) {
    if (!b || !out) return SWPC_ERR_ARG;
    if (member < 0 || member >= b->nmem) return ferr(b, SWPC_ERR_ARG, "member index outside 0..nmem-1");
    const int q = what == SWPC_WAV_V ? 0 : what == SWPC_WAV_U ? 1 : what == SWPC_WAV_STRESS ? 2
                : what == SWPC_WAV_STRAIN ? 3 : -1;
    if (q < 0 || !b->wav[q]) return ferr(b, SWPC_ERR_ARG, "recorder component not recorded");
    swpc_ctx *c = b->c;
    const size_t n = (size_t)c->ntw * wav_ncmp(q) * c->nst;
    FCK(cudaSetDevice(c->device));
    FCK(cudaMemcpyAsync(out, b->wav[q] + n * member, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    FCK(cudaStreamSynchronize(c->stream));
    return SWPC_OK;
}

extern "C" int swpc_fbatch_download_field(swpc_fbatch *b, int member, int field, float *out, int ld_k, int ld_i) {
    if (!b || !out) return SWPC_ERR_ARG;
    if (member < 0 || member >= b->nmem) return ferr(b, SWPC_ERR_ARG, "member index outside 0..nmem-1");
    float *base = nullptr;
    if (field >= SWPC_F_VX && field <= SWPC_F_VZ) base = b->V[field - SWPC_F_VX];
    else if (field >= SWPC_F_SXX && field <= SWPC_F_SXY) base = b->S[field - SWPC_F_SXX];
    else if (field >= SWPC_F_R && field < SWPC_F_R + 18) base = b->R[field - SWPC_F_R];
    if (!base) return ferr(b, SWPC_ERR_ARG, "unknown or unallocated field (V, S or R)");
    FCK(cudaSetDevice(b->c->device));
    FCK(cudaStreamSynchronize(b->c->stream));
    return copy_box(b->c, base + b->stride * member, nullptr, out, ld_k, ld_i);
}

extern "C" int swpc_fbatch_green_fetch(swpc_fbatch *b, int member, float *out) {
    if (!b || !out) return SWPC_ERR_ARG;
    swpc_ctx *c = b->c;
    if (member < 0 || member >= b->nmem) return ferr(b, SWPC_ERR_ARG, "member index out of range");
    if (b->g_ng <= 0) return ferr(b, SWPC_ERR_STATE, "the context had no green table when the batch was created");
    FCK(cudaSetDevice(c->device));
    const size_t n = (size_t)c->ng_ntw * c->ng_cmp * b->g_ng;
    FCK(cudaMemcpyAsync(out, b->g_out + n * member, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    FCK(cudaStreamSynchronize(c->stream));
    return SWPC_OK;
}

extern "C" long long swpc_fbatch_device_bytes(const swpc_fbatch *b) { return b ? b->bytes : 0; }
