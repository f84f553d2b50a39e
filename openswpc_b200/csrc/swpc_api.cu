// swpc_api.cu -- C-ABI implementation (include/swpc_gpu.h) for the 3D solver.
//
// Host orchestration only: allocation, uploads, coefficient setup in the
// reference's single-precision expression order, the per-step launch
// sequence of main.f90:125-144 and its CUDA-graph capture.  No arithmetic of
// the time step runs on the host.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <set>
#include <string>
#include <utility>
#include <vector>

#include "swpc2d.cuh"
#include "swpc_ctx.h"
#include "swpc_host.h"
#include "swpc_kernels.cuh"
#include "swpc_tma.h"

using namespace swpc;

namespace swpc {

int set_err(swpc_ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_check(swpc_ctx *c, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return 0;
    return set_err(c, SWPC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

// extern "C" implementations for the 2D codes live in swpc2d_api.cu
int create_2d(swpc_ctx *c);
int upload_medium_2d(swpc_ctx *c, const swpc_medium_view *m);
int absorb_setup_2d(swpc_ctx *c, const float *gxc, const float *gxe, const float *gzc, const float *gze);
int update_stress_2d(swpc_ctx *c, int mask);
int update_vel_2d(swpc_ctx *c, int mask);
int wav_store_2d(swpc_ctx *c, int it, const int *d_it);
int vmax_2d(swpc_ctx *c, float *out);
void destroy_2d(swpc_ctx *c);
int refresh_2d(swpc_ctx *c);
int cerjan_setup_2d(swpc_ctx *c, const float *gx_c, const float *gx_b, const float *gz_c, const float *gz_b);

}  // namespace swpc

#define CK(call)                                               \
    do {                                                       \
        int _rc = cuda_check(c, (call), #call);                \
        if (_rc) return _rc;                                   \
    } while (0)
#define RC(call)             \
    do {                     \
        int _rc = (call);    \
        if (_rc) return _rc; \
    } while (0)

static bool is3d(const swpc_ctx *c) { return c->kind == SWPC_KIND_3D; }

static void invalidate_graph(swpc_ctx *c) {
    c->desc_dirty = true;
    if (c->graph_exec) {
        cudaGraphExecDestroy(c->graph_exec);
        c->graph_exec = nullptr;
    }
}
namespace swpc {
int graph_invalidate(swpc_ctx *c) {
    invalidate_graph(c);
    return SWPC_OK;
}
// the FP16 scales 2^eS, 2^-eS, 2^eR, 2^-eR to device memory, where the kernels
// read them (no launch argument changes when they are re-centred)
int upload_scales(swpc_ctx *c) {
    for (int q = 0; q < 48; q++) c->h_scale[q] = 1.0f;   // exponents 0 (dalloc zeroes d_exp)
    CK(cudaMemcpyAsync(c->d_scale, c->h_scale, sizeof(c->h_scale), cudaMemcpyHostToDevice, c->stream));
    return cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
}
}  // namespace swpc

// ---------------------------------------------------------------------------
// lifetime
// ---------------------------------------------------------------------------
extern "C" int swpc_create(const swpc_desc *d, swpc_ctx **out) {
    if (!d || !out) return SWPC_ERR_ARG;
    *out = nullptr;
    swpc_ctx *c = new swpc_ctx();
    c->d = *d;
    c->kind = d->kind;
    c->device = d->device;
    auto fail = [&](int rc) {
        // keep the context so that swpc_last_error can report the reason
        *out = c;
        return rc;
    };
    if (d->kind != SWPC_KIND_3D && d->kind != SWPC_KIND_PSV && d->kind != SWPC_KIND_SH)
        return fail(set_err(c, SWPC_ERR_ARG, "unknown solver kind"));
    if (d->nx < 4 || d->nz < 4 || (d->kind == SWPC_KIND_3D && d->ny < 4))
        return fail(set_err(c, SWPC_ERR_ARG, "grid must be at least 4 cells per dimension"));
    if (d->nm < 0 || d->nm > NM_MAX) return fail(set_err(c, SWPC_ERR_ARG, "nm must be 0..3"));
    if (d->na < 0 || d->na >= d->nz) return fail(set_err(c, SWPC_ERR_ARG, "absorber thickness na too large for the grid"));
    // across x and y the absorber is checked against the whole grid: this
    // one, or the global one of swpc_set_subdomain (a block may be narrower
    // than two absorbers)
    c->na_wide = 2 * d->na >= d->nx || (d->kind == SWPC_KIND_3D && 2 * d->na >= d->ny);
    if (d->nt < 1) return fail(set_err(c, SWPC_ERR_ARG, "nt must be positive"));
    if (d->precision < SWPC_PREC_F32 || d->precision > SWPC_PREC_F16_R ||
        (d->kind != SWPC_KIND_3D && d->precision != SWPC_PREC_F32))
        return fail(set_err(c, SWPC_ERR_ARG,
                            "precision must be SWPC_PREC_F32/BF16_R/F16_SR/F16_R (3D) or SWPC_PREC_F32"));
    c->prec = d->precision;
    if (!(d->dx > 0) || !(d->dz > 0) || !(d->dt > 0) || (d->kind == SWPC_KIND_3D && !(d->dy > 0)))
        return fail(set_err(c, SWPC_ERR_ARG, "dx, dy, dz, dt must be positive"));
    {
        int rc = cuda_check(c, cudaSetDevice(d->device), "cudaSetDevice");
        if (rc) return fail(rc);
        rc = cuda_check(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        if (rc) return fail(rc);
    }
    const int nx = d->nx, ny = d->kind == SWPC_KIND_3D ? d->ny : 1, nz = d->nz, na = d->na;
    // kernel region (m_global.f90:349-378) for a single node 1..n
    c->ibk = (1 <= na) ? na + 1 : 1;
    c->iek = (nx >= nx - na + 1) ? nx - na : nx;
    c->jbk = (1 <= na) ? na + 1 : 1;
    c->jek = (ny >= ny - na + 1) ? ny - na : ny;
    if (d->kind != SWPC_KIND_3D) { c->jbk = 1; c->jek = 1; }
    c->kbk = 1;
    c->kek = nz - na;
    c->nxg = nx; c->nyg = ny;
    Geo &g = c->g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.Kp = ((nz + 3 + KH) + 7) / 8 * 8;
    g.Ip = nx + 6;
    g.Jp = d->kind == SWPC_KIND_3D ? ny + 6 : 1;
    g.ncell = (long long)g.Kp * g.Ip * g.Jp;
    int rc = 0;
    if (is3d(c) && c->prec == SWPC_PREC_F32) {
        // one slab: 0-2 V, 3-8 S, R (6 nm), lam mu taup taus muyz muxz muxy, bx by bz
        const int nf = 3 + 6 + 6 * d->nm + 7 + 3;
        rc = dalloc(c, &c->slab, (size_t)nf * g.ncell);
        if (!rc) {
            auto F = [&](int f) { return c->slab + (size_t)f * g.ncell; };
            for (int q = 0; q < 3; q++) c->V[q] = F(q);
            for (int q = 0; q < 6; q++) c->S[q] = F(3 + q);
            for (int comp = 0; comp < 6; comp++)
                for (int m = 0; m < d->nm; m++) c->R[comp * 3 + m] = F(9 + comp * d->nm + m);
            const int mq[7] = {1, 2, 3, 4, 8, 9, 10};
            for (int q = 0; q < 7; q++) c->med[mq[q]] = F(9 + 6 * d->nm + q);
            for (int q = 0; q < 3; q++) c->med[5 + q] = F(16 + 6 * d->nm + q);
            c->slab_nf = nf;
            // the TMA-staged kernels are the default launch of FP32 3D contexts
            c->stress_tma = true;
            c->vel_tma = true;
        }
        const long long ncol = (long long)g.Ip * g.Jp;
        if (!rc) rc = dalloc(c, &c->band, ncol);
        if (!rc) rc = dalloc(c, &c->pmlcol, ncol);
        if (!rc) rc = dalloc(c, &c->kob, ncol);
        if (!rc) rc = dalloc(c, &c->kfs, ncol);
        if (!rc) rc = dalloc(c, &c->d_err, 1);
    } else if (is3d(c)) {
        // reduced-precision storage: the FP32 fields in one slab (V, then S
        // for BF16_R, then lam mu taup taus muyz muxz muxy and bx by bz) and
        // the 2-byte fields in a second (S for F16_SR, then R component-major)
        const bool h_s = c->prec == SWPC_PREC_F16_SR;
        const int nf = 3 + (h_s ? 0 : 6) + 7 + 3;
        const int nh = (h_s ? 6 : 0) + 6 * d->nm;
        rc = dalloc(c, &c->slab, (size_t)nf * g.ncell);
        // g.ncell is even (Kp is a multiple of 8), so every 2-byte field starts on a 4-byte boundary
        if (!rc) rc = dalloc(c, &c->hslab, (size_t)std::max(nh, 1) * g.ncell);
        if (!rc) {
            auto F = [&](int f) { return c->slab + (size_t)f * g.ncell; };
            auto H = [&](int f) { return reinterpret_cast<float *>(c->hslab + (size_t)f * g.ncell); };
            for (int q = 0; q < 3; q++) c->V[q] = F(q);
            for (int q = 0; q < 6; q++) c->S[q] = h_s ? H(q) : F(3 + q);
            for (int comp = 0; comp < 6; comp++)
                for (int m = 0; m < d->nm; m++) c->R[comp * 3 + m] = H((h_s ? 6 : 0) + comp * d->nm + m);
            const int mb = h_s ? 3 : 9;
            const int mq[7] = {1, 2, 3, 4, 8, 9, 10};
            for (int q = 0; q < 7; q++) c->med[mq[q]] = F(mb + q);
            for (int q = 0; q < 3; q++) c->med[5 + q] = F(mb + 7 + q);
            c->slab_nf = nf;
            c->hslab_nf = nh;
            // the staged kernels are the default launch; the 2-byte forms move
            // fewer bytes a tile, and their stress update runs faster on 4 x 2
            // tiles (more CTAs, hence more tiles in flight, per SM)
            c->stress_tma = true;
            c->vel_tma = true;
            c->stress_tbj = 2;
        }
        const long long ncol = (long long)g.Ip * g.Jp;
        if (!rc) rc = dalloc(c, &c->band, ncol);
        if (!rc) rc = dalloc(c, &c->pmlcol, ncol);
        if (!rc) rc = dalloc(c, &c->kob, ncol);
        if (!rc) rc = dalloc(c, &c->kfs, ncol);
        if (!rc) rc = dalloc(c, &c->d_err, 1);
    } else {
        rc = create_2d(c);
    }
    if (!rc) rc = dalloc(c, &c->vmax_buf, 4);
    if (!rc) rc = dalloc(c, &c->d_it, 1);
    if (!rc) rc = dalloc(c, &c->d_scale, kScaleFloats);
    if (!rc) rc = dalloc(c, &c->d_exp, 24);
    if (!rc) rc = dalloc(c, &c->d_rmax, 24);
    if (!rc) rc = dalloc(c, &c->d_rfactor, 24);
    if (!rc) rc = dalloc(c, &c->d_rchanged, 1);
    if (!rc) rc = upload_scales(c);
    if (!rc) rc = cuda_check(c, cudaMallocHost((void **)&c->h_vmax, 4 * sizeof(unsigned int)), "cudaMallocHost");
    if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    if (rc) return fail(rc);
    *out = c;
    return SWPC_OK;
}

extern "C" int swpc_destroy(swpc_ctx *c) {
    if (!c) return SWPC_OK;
    if (c->nfbatch > 0) return set_err(c, SWPC_ERR_STATE, "destroy the reciprocity batches over this context first");
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    invalidate_graph(c);
    snap_free(c);
    adj_free(c);
    green_free(c);
    if (!is3d(c)) destroy_2d(c);
    if (c->slab) {
        // the slabs hold V, S, R and the medium fields
        cudaFree(c->slab);
        if (c->hslab) cudaFree(c->hslab);
        for (auto &p : c->V) p = nullptr;
        for (auto &p : c->S) p = nullptr;
        for (auto &p : c->R) p = nullptr;
        for (auto &p : c->med) p = nullptr;
    }
    if (c->d_err) cudaFree(c->d_err);
    for (void *p : {(void *)c->d_scale, (void *)c->d_exp, (void *)c->d_rmax, (void *)c->d_rfactor, (void *)c->d_rchanged})
        if (p) cudaFree(p);
    if (c->stage) cudaFree(c->stage);
    if (c->cj) cudaFree(c->cj);
    delete static_cast<TmaMaps *>(c->tmaps);
    void *ps[] = {c->V[0], c->V[1], c->V[2], c->band, c->pmlcol, c->kob, c->kfs, c->inj_glut, c->inj_bf,
                  c->stime_glut, c->mo_glut, c->stime_bf, c->inj_green, c->stf_green, c->st_ijk, c->wav[0],
                  c->wav[1], c->wav[2], c->wav[3], c->uacc, c->eacc, c->vmax_buf, c->d_it};
    for (void *p : ps) if (p) cudaFree(p);
    for (auto p : c->S) if (p) cudaFree(p);
    for (auto p : c->R) if (p) cudaFree(p);
    for (auto p : c->med) if (p) cudaFree(p);
    for (auto p : c->aux) if (p) cudaFree(p);
    for (int q = 0; q < 2; q++) {
        if (c->gx[q]) cudaFree(c->gx[q]);
        if (c->gy[q]) cudaFree(c->gy[q]);
        if (c->gz[q]) cudaFree(c->gz[q]);
    }
    if (c->h_vmax) cudaFreeHost(c->h_vmax);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return SWPC_OK;
}

extern "C" const char *swpc_last_error(const swpc_ctx *c) { return c ? c->err.c_str() : "null context"; }
extern "C" void *swpc_stream(swpc_ctx *c) { return c ? (void *)c->stream : nullptr; }
extern "C" long long swpc_device_bytes(const swpc_ctx *c) { return c ? c->bytes : 0; }

extern "C" int swpc_set_launch(swpc_ctx *c, int kernel, int minb, int bi, int bj) {
    if (!c) return SWPC_ERR_ARG;
    if (!is3d(c)) {
        // 2D: kernels 0 / 1 the tile-walking stress / velocity kernels, 5 / 6
        // the staged ones with bi = 4, 8 or 16 threads along i (bj = 1)
        if (!(kernel == 0 || kernel == 1 || kernel == 5 || kernel == 6) ||
            (kernel >= 5 && (!staged2d_ti_ok(bi) || bj != 1 || minb != 1)))
            return set_err(c, SWPC_ERR_ARG, "2D launch: kernel 0, 1, or 5, 6 with minb 1, bi 4/8/16, bj 1");
        invalidate_graph(c);
        if (kernel == 0) c->stress_tma = false;
        else if (kernel == 1) c->vel_tma = false;
        else if (kernel == 5) { c->stress_tma = true; c->stress_tbi = bi; }
        else { c->vel_tma = true; c->vel_tbi = bi; }
        return SWPC_OK;
    }
    if (kernel == 8) {
        // adjoint stress-phase weights: bi = 1 staged, 0 one cell per thread
        if (!is3d(c) || (bi != 0 && bi != 1)) return set_err(c, SWPC_ERR_ARG, "kernel 8 (3D): bi = 0 or 1");
        c->adj_tma = bi == 1;
        return SWPC_OK;
    }
    if (kernel == 9) {
        // adjoint velocity-phase weights: bi = 1 formed by the stress-phase gather of the step before (the
        // gradient's default), 0 by their own kernel
        if (!is3d(c) || (bi != 0 && bi != 1)) return set_err(c, SWPC_ERR_ARG, "kernel 9 (3D): bi = 0 or 1");
        c->adj_fuse = bi == 1;
        return SWPC_OK;
    }
    if (kernel == 7) {
        // launch order of the staged kernels: blocks of bi j tiles (0: chosen by size)
        if (bi < 0 || bi > 1024) return set_err(c, SWPC_ERR_ARG, "kernel 7: bi = j tiles per block, 0..1024");
        invalidate_graph(c);
        c->tile_jblock = bi;
        return SWPC_OK;
    }
    if (kernel < 0 || kernel > 6 || minb < 1 || minb > 4 || bi < 1 || bj < 1 ||
        ((kernel < 2 || kernel == 4) && 32 * bi * bj > 256))
        return set_err(c, SWPC_ERR_ARG, "launch shape out of range (kernel 0..6, minb 1..4, 32*bi*bj <= 256)");
    if (kernel >= 2 && kernel <= 4 && c->prec != SWPC_PREC_F32)
        return set_err(c, SWPC_ERR_ARG, "reduced-precision storage runs the kernels 0, 1, 5 and 6 only");
    // staged kernels: minb is unused (pass 1); the tile must be compiled
    if (kernel >= 5 && (!c->slab || minb != 1 ||
                        !(kernel == 5 ? tma_shape_ok(bi, bj, 1, c->prec) : tma_vel_shape_ok(bi, bj, 1, c->prec))))
        return set_err(c, SWPC_ERR_ARG, "staged kernels: minb 1 and a compiled tile (bi, bj)");
    invalidate_graph(c);
    switch (kernel) {
    case 0: c->stress_march = false; c->stress_tma = false; c->stress_minb = minb; c->bi = bi; c->bj = bj; break;
    case 1:
        c->vel_march = false; c->vel_vec = false; c->vel_tma = false; c->vel_minb = minb; c->vbi = bi; c->vbj = bj;
        break;
    case 2: c->stress_march = true; c->stress_tma = false; c->stress_mminb = minb; c->stress_jc = bj; break;
    case 3: c->vel_march = true; c->vel_vec = false; c->vel_tma = false; c->vel_mminb = minb; c->vel_jc = bj; break;
    case 4:
        c->vel_march = false; c->vel_vec = true; c->vel_tma = false; c->vel_vminb = minb; c->vel_vbi = bi;
        c->vel_vbj = bj;
        break;
    case 5: c->stress_march = false; c->stress_tma = true; c->stress_tbi = bi; c->stress_tbj = bj; break;
    default:
        c->vel_march = false; c->vel_vec = false; c->vel_tma = true; c->vel_tbi = bi; c->vel_tbj = bj;
        break;
    }
    return SWPC_OK;
}

extern "C" int swpc_sync(swpc_ctx *c) {
    if (!c) return SWPC_ERR_ARG;
    CK(cudaStreamSynchronize(c->stream));
    if (c->d_err) {
        int h = 0;
        CK(cudaMemcpy(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (h) return set_err(c, SWPC_ERR_CUDA, "a staged tile copy did not complete (TMA wait timed out)");
    }
    return SWPC_OK;
}

// The error word of the staged kernels: raised by a tile wait that ran out, it
// stays up (every later swpc_sync reports it) until the caller has restored
// the fields and clears it.
extern "C" int swpc_clear_error(swpc_ctx *c) {
    if (!c) return SWPC_ERR_ARG;
    if (!c->d_err) return SWPC_OK;
    CK(cudaSetDevice(c->device));
    CK(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SWPC_OK;
}

// host-side failure injection for error-path tests of a driver: the word a
// timed-out tile wait raises, set from the host (no kernel waits or faults)
extern "C" int swpc_raise_copy_error(swpc_ctx *c) {
    if (!c) return SWPC_ERR_ARG;
    if (!c->d_err) return set_err(c, SWPC_ERR_STATE, "this context has no error word");
    CK(cudaSetDevice(c->device));
    const int one = 1;
    CK(cudaMemcpy(c->d_err, &one, sizeof(int), cudaMemcpyHostToDevice));
    return SWPC_OK;
}

// ---------------------------------------------------------------------------
// layout conversion between the Fortran memory box and the device columns
// ---------------------------------------------------------------------------
namespace swpc {

// host (k, i, j) Fortran array over k in [-2, nz+3+], i in [-2, nx+3+], j in
// [-2, ny+3+] with leading extents ld_k, ld_i  <->  device column layout.
// chunk of nj planes of the host box (rows of ld_k k values, ld_i rows a
// plane) in the staging buffer -> the device columns of planes j0 ..
__global__ void repack_box_kernel(const float *__restrict__ stage, float *__restrict__ dev, int nkb, int nib, int nj,
                                  int ld_k, int ld_i, int Kp, int Ip, int j0, int koff) {
    const long long n = (long long)nkb * nib * nj;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int kk = (int)(q % nkb);
        const long long r = q / nkb;
        const int ii = (int)(r % nib), jj = (int)(r / nib);
        dev[((long long)(j0 + jj) * Ip + ii) * Kp + koff + kk] = stage[((long long)jj * ld_i + ii) * ld_k + kk];
    }
}

int copy_box(swpc_ctx *c, float *dev, const float *host_in, float *host_out, int ld_k, int ld_i) {
    const Geo &g = c->g;
    const int nkb = g.nz + 6;             // k = -2 .. nz+3
    const int nib = g.nx + 6;             // i = -2 .. nx+3
    const int njb = is3d(c) ? g.ny + 6 : 1;
    if (ld_k < nkb || ld_i < nib) return set_err(c, SWPC_ERR_ARG, "leading extents smaller than the memory box");
    const int koff = -2 - 1 + KH;         // device offset of k = -2 within a column
    const long long plane = (long long)ld_i * ld_k;   // floats of a host plane
    if (host_in && plane * njb >= (1LL << 16)) {
        // an upload of 256 KB or more: contiguous chunks of host planes at full
        // link speed into a staging buffer (at most 16 MB), each repacked into
        // the device columns on the device (the strided copy of short rows is
        // several times slower)
        const int nj = (int)std::max<long long>(1, std::min<long long>(njb, (16LL << 20) / plane));
        if (c->stage_floats < plane * nj) {
            if (c->stage) cudaFree(c->stage);
            c->bytes -= c->stage_floats * (long long)sizeof(float);
            c->stage = nullptr;
            c->stage_floats = 0;
            if (cudaMalloc((void **)&c->stage, plane * nj * sizeof(float)) != cudaSuccess)
                return set_err(c, SWPC_ERR_NOMEM, "no room for the upload staging buffer");
            c->stage_floats = plane * nj;
            c->bytes += c->stage_floats * (long long)sizeof(float);
        }
        for (int j0 = 0; j0 < njb; j0 += nj) {
            const int n = std::min(nj, njb - j0);
            CK(cudaMemcpyAsync(c->stage, host_in + (long long)j0 * plane, (size_t)(plane * n) * sizeof(float),
                               cudaMemcpyHostToDevice, c->stream));
            repack_box_kernel<<<148 * 8, 256, 0, c->stream>>>(c->stage, dev, nkb, nib, n, ld_k, ld_i, g.Kp, g.Ip, j0,
                                                             koff);
            CK(cudaGetLastError());
        }
        return cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    }
    // one pitched 3D copy for the whole box: rows of nkb k values, nib rows
    // (i) a plane, njb planes (j); the host box has row pitch ld_k and ld_i
    // rows a plane, the device Kp and Ip
    cudaMemcpy3DParms q = {};
    const cudaPitchedPtr hp = make_cudaPitchedPtr(const_cast<float *>(host_in ? host_in : host_out),
                                                  (size_t)ld_k * sizeof(float), (size_t)nkb, (size_t)ld_i);
    const cudaPitchedPtr dp = make_cudaPitchedPtr(dev + koff, (size_t)g.Kp * sizeof(float), (size_t)nkb, (size_t)g.Ip);
    q.srcPtr = host_in ? hp : dp;
    q.dstPtr = host_in ? dp : hp;
    q.extent = make_cudaExtent((size_t)nkb * sizeof(float), (size_t)nib, (size_t)njb);
    q.kind = host_in ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
    const cudaError_t e = cudaMemcpy3DAsync(&q, c->stream);
    if (e != cudaSuccess) return cuda_check(c, e, "cudaMemcpy3DAsync");
    return cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
}

// 4 a b c d / (a b c + a b d + a c d + b c d + epsilon(1.0)), every product and
// sum rounded left to right without contraction, as the host restatement of
// averaged_medium (m_medium.f90:451-459) evaluates it
__device__ __forceinline__ float harmonic4(float a, float b, float c, float d) {
    const float num = __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(4.0f, a), b), c), d);
    float den = __fmul_rn(__fmul_rn(a, b), c);
    den = __fadd_rn(den, __fmul_rn(__fmul_rn(a, b), d));
    den = __fadd_rn(den, __fmul_rn(__fmul_rn(a, c), d));
    den = __fadd_rn(den, __fmul_rn(__fmul_rn(b, c), d));
    den = __fadd_rn(den, 1.1920929e-07f);
    return __fdiv_rn(num, den);
}

// averaged_medium (m_medium.f90:432-465) over the memory box, on the device:
// buoyancies 2 / (rho + rho') at the velocity points and 4-point harmonic
// means of mu at the shear-stress points for k, i, j in [1, n], zero on the
// rest of the box.  The host sends rho into the muyz array; pass 0 forms bx,
// by, bz, muxz, muxy from it and mu, then pass 1 forms muyz over it.
__global__ void average_medium_kernel(Geo g, const float *rho, const float *__restrict__ mu, float *bx, float *by,
                                      float *bz, float *muyz, float *muxz, float *muxy, int pass) {
    const int nkb = g.nz + 6, nib = g.nx + 6;
    const long long n = (long long)nkb * nib * (g.ny + 6);
    const long long pk = 1, pi = g.Kp, pj = (long long)g.Ip * g.Kp;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(q % nkb) - 2;
        const long long r = q / nkb;
        const int i = (int)(r % nib) - 2, j = (int)(r / nib) - 2;
        const long long e = cell_index(g, k, i, j);
        const bool in = k >= 1 && k <= g.nz && i >= 1 && i <= g.nx && j >= 1 && j <= g.ny;
        const float nnn = in ? mu[e] : 0.0f;
        const float pnn = in ? mu[e + pk] : 0.0f, npn = in ? mu[e + pi] : 0.0f, nnp = in ? mu[e + pj] : 0.0f;
        if (pass == 0) {
            float vx = 0.0f, vy = 0.0f, vz = 0.0f, vxz = 0.0f, vxy = 0.0f;
            if (in) {
                const float r0 = rho[e];
                vx = __fdiv_rn(2.0f, __fadd_rn(r0, rho[e + pi]));
                vy = __fdiv_rn(2.0f, __fadd_rn(r0, rho[e + pj]));
                vz = __fdiv_rn(2.0f, __fadd_rn(r0, rho[e + pk]));
                vxz = harmonic4(nnn, pnn, npn, mu[e + pk + pi]);
                vxy = harmonic4(nnn, npn, nnp, mu[e + pi + pj]);
            }
            bx[e] = vx; by[e] = vy; bz[e] = vz; muxz[e] = vxz; muxy[e] = vxy;
        } else {
            muyz[e] = in ? harmonic4(nnn, pnn, nnp, mu[e + pk + pj]) : 0.0f;
        }
    }
}

int copy_box_from_device(swpc_ctx *c, float *dev, const float *src, int ld_k, int ld_i) {
    const Geo &g = c->g;
    const int nkb = g.nz + 6, nib = g.nx + 6, njb = is3d(c) ? g.ny + 6 : 1;
    if (ld_k < nkb || ld_i < nib) return set_err(c, SWPC_ERR_ARG, "leading extents smaller than the memory box");
    repack_box_kernel<<<148 * 8, 256, 0, c->stream>>>(src, dev, nkb, nib, njb, ld_k, ld_i, g.Kp, g.Ip, 0,
                                                     -2 - 1 + KH);
    CK(cudaGetLastError());
    return SWPC_OK;
}

int average_medium(swpc_ctx *c) {
    for (int pass = 0; pass < 2; pass++) {
        average_medium_kernel<<<148 * 8, 256, 0, c->stream>>>(c->g, c->med[8], c->med[2], c->med[5], c->med[6],
                                                             c->med[7], c->med[8], c->med[9], c->med[10], pass);
        CK(cudaGetLastError());
    }
    return SWPC_OK;
}

}  // namespace swpc

// ---------------------------------------------------------------------------
// medium, coefficients, absorber
// ---------------------------------------------------------------------------
extern "C" int swpc_upload_medium(swpc_ctx *c, const swpc_medium_view *m) {
    if (!c || !m) return SWPC_ERR_ARG;
    RC(check_na_wide(c));
    CK(cudaSetDevice(c->device));
    invalidate_graph(c);
    if (!is3d(c)) return upload_medium_2d(c, m);
    const Geo &g = c->g;
    const float *src[11] = {m->rho, m->lam, m->mu, m->taup, m->taus, m->bx, m->by, m->bz, m->muyz, m->muxz, m->muxy};
    // rho without the six averaged fields: form them in HBM (half the bytes
    // over the host link)
    const bool average = m->rho && !m->bx && !m->by && !m->bz && !m->muyz && !m->muxz && !m->muxy;
    for (int q = 1; q < (average ? 5 : 11); q++) {
        if (!src[q]) return set_err(c, SWPC_ERR_ARG, "medium field missing");
        RC(copy_box(c, c->med[q], src[q], nullptr, m->ld_k, m->ld_i));
    }
    if (average) {
        RC(copy_box(c, c->med[8], m->rho, nullptr, m->ld_k, m->ld_i));
        RC(average_medium(c));
    }
    if (!m->kfs || !m->kob || !m->kfs_top || !m->kfs_bot || !m->kob_top || !m->kob_bot || !m->kbeg_a)
        return set_err(c, SWPC_ERR_ARG, "integer map missing");
    if (m->ld_i2 < g.nx + 6) return set_err(c, SWPC_ERR_ARG, "ld_i2 smaller than the memory box");
    const long long ncol = (long long)g.Ip * g.Jp;
    std::vector<int4> band(ncol, make_int4(0, 0, 0, 0));
    std::vector<int> kob(ncol, 0), kfs(ncol, 0);
    c->h_kbeg_a.assign(ncol, 0);
    for (int j = -2; j <= g.ny + 3; j++)
        for (int i = -2; i <= g.nx + 3; i++) {
            const long long h = (long long)(j + 2) * m->ld_i2 + (i + 2);
            const long long cc = col_index(g, i, j);
            band[cc] = make_int4(m->kfs_top[h], m->kfs_bot[h], m->kob_top[h], m->kob_bot[h]);
            kob[cc] = m->kob[h];
            kfs[cc] = m->kfs[h];
            c->h_kbeg_a[cc] = m->kbeg_a[h];
        }
    // the fused kernels assume kbeg_a = 1 on side columns and kend_k + 1 under
    // the interior box (m_global.f90:336-345); reject anything else.
    for (int j = 1; j <= g.ny && c->abc == 0; j++)
        for (int i = 1; i <= g.nx; i++) {
            const bool inner = i >= c->ibk && i <= c->iek && j >= c->jbk && j <= c->jek;
            const int want = inner ? c->kek + 1 : 1;
            if (c->h_kbeg_a[col_index(g, i, j)] != want)
                return set_err(c, SWPC_ERR_ARG, "kbeg_a map does not match the absorber layout of m_global.f90:336-345");
        }
    CK(cudaMemcpyAsync(c->band, band.data(), ncol * sizeof(int4), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->kob, kob.data(), ncol * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->kfs, kfs.data(), ncol * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->medium_ready = true;
    return SWPC_OK;
}

extern "C" int swpc_kernel_setup(swpc_ctx *c, const float *ts) {
    if (!c) return SWPC_ERR_ARG;
    if (c->d.nm > 0 && !ts) return set_err(c, SWPC_ERR_ARG, "ts required for nm > 0");
    invalidate_graph(c);
    // m_kernel.f90:43-54 in real(MP) = single precision
    const float dd[3] = {c->d.dx, is3d(c) ? c->d.dy : c->d.dx, c->d.dz};
    for (int ax = 0; ax < 3; ax++) {
        const float rc40 = 17.0f / 16.0f / dd[ax];
        const float rc41 = 1.0f / 48.0f / dd[ax];
        const float rd40 = -1.0f / 16.0f / dd[ax];
        const float rd41 = -1.0f / 48.0f / dd[ax];
        // isign = -1 (4th order) and +1 (2nd-order band): rc + isign*rd
        c->e40[ax][0] = rc40 + (-1.0f) * rd40;
        c->e41[ax][0] = rc41 + (-1.0f) * rd41;
        c->e40[ax][1] = rc40 + (1.0f) * rd40;
        c->e41[ax][1] = rc41 + (1.0f) * rd41;
        c->r20[ax] = 1.0f / dd[ax];                       // m_absorb_p.f90:70-72
        c->r40[ax] = 9.0f / 8.0f / dd[ax];                // m_wav.f90:130-135
        c->r41[ax] = 1.0f / 24.0f / dd[ax];
    }
    // m_kernel.f90:58-67 in real(SP)
    const int nm = c->d.nm;
    const float dt = c->d.dt;
    for (int m = 0; m < NM_MAX; m++) { c->c1[m] = c->c2[m] = c->d1[m] = 0.f; c->ts[m] = 0.f; }
    c->d2 = 0.f;
    if (nm > 0) {
        for (int m = 0; m < nm; m++) {
            c->ts[m] = ts[m];
            c->c1[m] = (2 * ts[m] - dt) / (2 * ts[m] + dt);
            c->c2[m] = (2) / (2 * ts[m] + dt) / nm;
        }
        float d2 = 0.0f;
        for (int m = 0; m < nm; m++) d2 = d2 + dt / (2 * ts[m] - dt);
        c->d2 = d2 / nm;
        for (int m = 0; m < nm; m++) c->d1[m] = 2 * ts[m] / (2 * ts[m] - dt);
    }
    c->kernel_ready = true;
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

extern "C" int swpc_absorb_setup(swpc_ctx *c, const float *gxc, const float *gxe, const float *gyc, const float *gye,
                                 const float *gzc, const float *gze) {
    if (!c) return SWPC_ERR_ARG;
    CK(cudaSetDevice(c->device));
    invalidate_graph(c);
    if (!c->medium_ready) return set_err(c, SWPC_ERR_STATE, "swpc_upload_medium must precede swpc_absorb_setup");
    if (c->abc != 0) return set_err(c, SWPC_ERR_STATE, "the context runs the Cerjan sponge (abc_type = 'cerjan')");
    if (!is3d(c)) return absorb_setup_2d(c, gxc, gxe, gzc, gze);
    const Geo &g = c->g;
    RC(upload_profile(c, &c->gx[0], gxc, g.nx));
    RC(upload_profile(c, &c->gx[1], gxe, g.nx));
    RC(upload_profile(c, &c->gy[0], gyc, g.ny));
    RC(upload_profile(c, &c->gy[1], gye, g.ny));
    RC(upload_profile(c, &c->gz[0], gzc, g.nz));
    RC(upload_profile(c, &c->gz[1], gze, g.nz));
    // compact auxiliary storage: one contiguous k-run per absorber column,
    // each run starting on a 32-byte boundary
    const long long ncol = (long long)g.Ip * g.Jp;
    std::vector<int2> pc(ncol, make_int2(1, -1));
    long long base = 0;
    for (int j = 1; j <= g.ny; j++)
        for (int i = 1; i <= g.nx; i++) {
            const long long cc = col_index(g, i, j);
            const int kb = c->h_kbeg_a[cc];
            const int len = g.nz - kb + 1;
            if (len <= 0) continue;
            if (base + len > 0x7fffffffLL) return set_err(c, SWPC_ERR_ARG, "absorber region too large");
            pc[cc] = make_int2(kb, (int)base);
            base += (len + 7) / 8 * 8;
        }
    c->npml = base;
    for (int q = 0; q < 18; q++) {
        if (c->aux[q]) { cudaFree(c->aux[q]); c->aux[q] = nullptr; }
        RC(dalloc(c, &c->aux[q], (size_t)std::max<long long>(base, 1)));
    }
    CK(cudaMemcpyAsync(c->pmlcol, pc.data(), ncol * sizeof(int2), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->absorb_ready = true;
    return SWPC_OK;
}

// absorb_c__setup (src/swpc_3d/m_absorb_c.f90:27-103) with the kernel region
// of abc_type = 'cerjan' (m_global.f90:349-378: the whole domain, so the
// interior update covers every cell and no PML cell remains)
extern "C" int swpc_absorb_setup_cerjan(swpc_ctx *c, const float *gx_c, const float *gx_b, const float *gy_c,
                                        const float *gy_b, const float *gz_c, const float *gz_b) {
    if (!c) return SWPC_ERR_ARG;
    if (c->prec != SWPC_PREC_F32) return set_err(c, SWPC_ERR_ARG, "the Cerjan sponge runs with FP32 storage");
    if (c->abc == 0 && c->absorb_ready)
        return set_err(c, SWPC_ERR_STATE, "the context already runs the PML (abc_type = 'pml')");
    CK(cudaSetDevice(c->device));
    invalidate_graph(c);
    if (!is3d(c)) return cerjan_setup_2d(c, gx_c, gx_b, gz_c, gz_b);
    if (!gx_c || !gx_b || !gy_c || !gy_b || !gz_c || !gz_b) return set_err(c, SWPC_ERR_ARG, "sponge profile missing");
    const Geo &g = c->g;
    const size_t n = 2 * (size_t)(g.nx + g.ny + g.nz);
    if (!c->cj) RC(dalloc(c, &c->cj, n));
    std::vector<float> h(n);
    std::copy(gx_c, gx_c + g.nx, h.begin());
    std::copy(gx_b, gx_b + g.nx, h.begin() + g.nx);
    std::copy(gy_c, gy_c + g.ny, h.begin() + 2 * g.nx);
    std::copy(gy_b, gy_b + g.ny, h.begin() + 2 * g.nx + g.ny);
    std::copy(gz_c, gz_c + g.nz, h.begin() + 2 * (g.nx + g.ny));
    std::copy(gz_b, gz_b + g.nz, h.begin() + 2 * (g.nx + g.ny) + g.nz);
    CK(cudaMemcpyAsync(c->cj, h.data(), n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->abc = 1;
    c->ibk = 1; c->iek = g.nx; c->jbk = 1; c->jek = g.ny; c->kbk = 1; c->kek = g.nz;
    c->absorb_ready = true;
    return SWPC_OK;
}

// absorb_c__update_stress / absorb_c__update_vel (m_absorb_c.f90:105-198):
// each field times the factors of its staggered position, after the
// interior update.  Only the sponge is visited, one warp per column with
// lanes along k: every k of the side columns, the bottom na cells of the
// others.  The cells skipped have all factors 1, and a product with 1
// leaves the bits unchanged.
__global__ void cerjan3d_kernel(Geo g, int na, int ioff, int joff, int nxg, int nyg, int phase,
                                const float *__restrict__ cj, float *f0, float *f1, float *f2, float *f3, float *f4,
                                float *f5) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const float *gxc = cj, *gxb = cj + nx, *gyc = cj + 2 * nx, *gyb = gyc + ny, *gzc = gyc + 2 * ny, *gzb = gzc + nz;
    const int lane = threadIdx.x & 31;
    const long long ncol = (long long)nx * ny;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; w < ncol; w += nw) {
        const int i = 1 + (int)(w % nx), j = 1 + (int)(w / nx);
        const int ig = i + ioff, jg = j + joff;   // global column
        const bool side = ig <= na || ig > nxg - na || jg <= na || jg > nyg - na;
        const float xc = gxc[i - 1], xb = gxb[i - 1], yc = gyc[j - 1], yb = gyb[j - 1];
        for (int k = (side ? 1 : nz - na + 1) + lane; k <= nz; k += 32) {
            const long long e = cell_index(g, k, i, j);
            const float zc = gzc[k - 1], zb = gzb[k - 1];
            if (phase == 0) {
                const float gcc = __fmul_rn(__fmul_rn(xc, yc), zc);
                f0[e] = __fmul_rn(f0[e], gcc);
                f1[e] = __fmul_rn(f1[e], gcc);
                f2[e] = __fmul_rn(f2[e], gcc);
                f3[e] = __fmul_rn(__fmul_rn(__fmul_rn(f3[e], xc), yb), zb);
                f4[e] = __fmul_rn(__fmul_rn(__fmul_rn(f4[e], xb), yc), zb);
                f5[e] = __fmul_rn(__fmul_rn(__fmul_rn(f5[e], xb), yb), zc);
            } else {
                f0[e] = __fmul_rn(__fmul_rn(__fmul_rn(f0[e], xb), yc), zc);
                f1[e] = __fmul_rn(__fmul_rn(__fmul_rn(f1[e], xc), yb), zc);
                f2[e] = __fmul_rn(__fmul_rn(__fmul_rn(f2[e], xc), yc), zb);
            }
        }
    }
}

static int launch_cerjan(swpc_ctx *c, int phase) {
    float *const *f = phase == 0 ? c->S : c->V;
    cerjan3d_kernel<<<148 * 8, 256, 0, c->stream>>>(c->g, c->d.na, c->ioff, c->joff, c->nxg, c->nyg, phase, c->cj,
                                                     f[0], f[1], f[2],
                                                     phase == 0 ? f[3] : nullptr, phase == 0 ? f[4] : nullptr,
                                                     phase == 0 ? f[5] : nullptr);
    return cuda_check(c, cudaGetLastError(), "cerjan3d launch");
}

// ---------------------------------------------------------------------------
// sources
// ---------------------------------------------------------------------------
// ghost cells that global__comm_stress / global__comm_vel overwrite with zero
// on a single node (m_global.f90:460-490, 571-603)
static bool comm_zeroed(const swpc_ctx *c, int field, int k, int i, int j) {
    const int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz;
    if (k < 1 || k > nz) return false;
    auto in1 = [](int v, std::initializer_list<int> s) { return std::find(s.begin(), s.end(), v) != s.end(); };
    if (c->kind == SWPC_KIND_PSV) {   // src/swpc_psv/m_global.f90:356-361, 409-414
        switch (field) {
        case SWPC_F_VX: return in1(i, {-1, 0, nx + 1});
        case SWPC_F_VZ: return in1(i, {0, nx + 1, nx + 2});
        case SWPC_F_SXX: return in1(i, {0, nx + 1, nx + 2});
        case SWPC_F_SXZ: return in1(i, {-1, 0, nx + 1});
        default: return false;
        }
    }
    if (c->kind == SWPC_KIND_SH) {    // src/swpc_sh/m_global.f90:340-342, 386-388
        switch (field) {
        case SWPC_F_VY: return in1(i, {0, nx + 1, nx + 2});
        case SWPC_F_SXY: return in1(i, {-1, 0, nx + 1});
        default: return false;
        }
    }
    const bool jin = (j >= 1 && j <= ny), iin = (i >= 1 && i <= nx);
    auto in = [](int v, std::initializer_list<int> s) { return std::find(s.begin(), s.end(), v) != s.end(); };
    switch (field) {
    case SWPC_F_VX: return (jin && in(i, {-1, 0, nx + 1})) || (iin && in(j, {0, ny + 1, ny + 2}));
    case SWPC_F_VY: return (jin && in(i, {0, nx + 1, nx + 2})) || (iin && in(j, {-1, 0, ny + 1}));
    case SWPC_F_VZ: return (jin && in(i, {0, nx + 1, nx + 2})) || (iin && in(j, {0, ny + 1, ny + 2}));
    case SWPC_F_SXX: return jin && in(i, {0, nx + 1, nx + 2});
    case SWPC_F_SYY: return iin && in(j, {0, ny + 1, ny + 2});
    case SWPC_F_SXY: return (jin && in(i, {-1, 0, nx + 1})) || (iin && in(j, {-1, 0, ny + 1}));
    case SWPC_F_SXZ: return jin && in(i, {-1, 0, nx + 1});
    case SWPC_F_SYZ: return iin && in(j, {-1, 0, ny + 1});
    default: return false;
    }
}

static int build_list(swpc_ctx *c, std::vector<InjEntry> &v, InjEntry **dptr, int *nout, bool *serial) {
    std::set<std::pair<int, long long>> seen;
    bool dup = false;
    for (auto &e : v)
        if (!seen.insert({e.field, e.cell}).second) dup = true;
    *serial = dup;
    *nout = (int)v.size();
    if (*dptr) { cudaFree(*dptr); *dptr = nullptr; }
    RC(dalloc(c, dptr, v.size()));
    if (!v.empty()) CK(cudaMemcpyAsync(*dptr, v.data(), v.size() * sizeof(InjEntry), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SWPC_OK;
}

static bool in_box(const swpc_ctx *c, int k, int i, int j) {
    const Geo &g = c->g;
    const int jlo = is3d(c) ? -2 : 1, jhi = is3d(c) ? g.ny + 3 : 1;
    return k >= 1 - KH + 1 && k <= g.nz + 3 && i >= -2 && i <= g.nx + 3 && j >= jlo && j <= jhi;
}

static void add_entry(const swpc_ctx *c, std::vector<InjEntry> &v, int field, int k, int i, int j, int src, float coef,
                      int mode, int bfield, bool *bad) {
    if (!in_box(c, k, i, j)) { *bad = true; return; }
    if (comm_zeroed(c, field, k, i, j)) return;   // zeroed before anything reads it
    InjEntry e;
    e.cell = is3d(c) ? cell_index(c->g, k, i, j) : (long long)(i + 2) * c->g.Kp + (k - 1 + KH);
    e.field = field; e.src = src; e.coef = coef; e.mode = mode; e.bfield = bfield; e.pad = 0;
    v.push_back(e);
}

namespace swpc {
int stime_table(swpc_ctx *c, float **dst, int nsrc, const float *srcprm, int stftype, bool half) {
    const int nt = c->d.nt;
    std::vector<float> t((size_t)nt * std::max(nsrc, 1), 0.f);
    for (int it = 1; it <= nt; it++) {
        // m_source.f90:800 (half step) and :857
        const float tt = half ? c->d.tbeg + ((float)it - 0.5f) * c->d.dt : c->d.tbeg + (float)it * c->d.dt;
        for (int s = 0; s < nsrc; s++) t[(size_t)(it - 1) * nsrc + s] = momentrate(tt, stftype, srcprm[2 * s], srcprm[2 * s + 1]);
    }
    if (*dst) { cudaFree(*dst); *dst = nullptr; }
    RC(dalloc(c, dst, t.size()));
    CK(cudaMemcpyAsync(*dst, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SWPC_OK;
}

// the six velocity cells of green__source (m_green.f90:615-627) for a unit
// force along cmp at (ksrc, isrc, jsrc); false when a cell is outside the box
bool green_entries(const swpc_ctx *c, int isrc, int jsrc, int ksrc, char cmp, std::vector<InjEntry> &v) {
    // m_green.f90:146-154
    const float f1[3] = {cmp == 'x' ? 1.0f : 0.0f, cmp == 'y' ? 1.0f : 0.0f, cmp == 'z' ? 1.0f : 0.0f};
    bool bad = false;
    add_entry(c, v, SWPC_F_VX, ksrc, isrc, jsrc, 0, f1[0], INJ_GREEN, 0, &bad);
    add_entry(c, v, SWPC_F_VX, ksrc, isrc - 1, jsrc, 0, f1[0], INJ_GREEN, 0, &bad);
    add_entry(c, v, SWPC_F_VY, ksrc, isrc, jsrc, 0, f1[1], INJ_GREEN, 1, &bad);
    add_entry(c, v, SWPC_F_VY, ksrc, isrc, jsrc - 1, 0, f1[1], INJ_GREEN, 1, &bad);
    add_entry(c, v, SWPC_F_VZ, ksrc, isrc, jsrc, 0, f1[2], INJ_GREEN, 2, &bad);
    add_entry(c, v, SWPC_F_VZ, ksrc - 1, isrc, jsrc, 0, f1[2], INJ_GREEN, 2, &bad);
    return !bad;
}
}  // namespace swpc

extern "C" int swpc_source_setup(swpc_ctx *c, int nsrc, const int *isrc, const int *jsrc, const int *ksrc,
                                 const float *srcprm, const float *mo, const float *m6, int stftype) {
    if (!c || nsrc < 0) return SWPC_ERR_ARG;
    if (nsrc > 0 && (!isrc || !ksrc || !srcprm || !mo || !m6 || (is3d(c) && !jsrc)))
        return set_err(c, SWPC_ERR_ARG, "source arrays missing");
    CK(cudaSetDevice(c->device));
    invalidate_graph(c);
    std::vector<InjEntry> v;
    bool bad = false;
    for (int s = 0; s < nsrc; s++) {
        const int ii = isrc[s], jj = is3d(c) ? jsrc[s] : 1, kk = ksrc[s];
        const float *mm = m6 + 6 * s;   // xx yy zz yz xz xy
        if (is3d(c)) {
            // m_source.f90:807-824
            add_entry(c, v, SWPC_F_SXX, kk, ii, jj, s, mm[0], INJ_GLUT, 0, &bad);
            add_entry(c, v, SWPC_F_SYY, kk, ii, jj, s, mm[1], INJ_GLUT, 0, &bad);
            add_entry(c, v, SWPC_F_SZZ, kk, ii, jj, s, mm[2], INJ_GLUT, 0, &bad);
            add_entry(c, v, SWPC_F_SXY, kk, ii, jj, s, mm[5], INJ_GLUT4, 0, &bad);
            add_entry(c, v, SWPC_F_SXY, kk, ii, jj - 1, s, mm[5], INJ_GLUT4, 0, &bad);
            add_entry(c, v, SWPC_F_SXY, kk, ii - 1, jj, s, mm[5], INJ_GLUT4, 0, &bad);
            add_entry(c, v, SWPC_F_SXY, kk, ii - 1, jj - 1, s, mm[5], INJ_GLUT4, 0, &bad);
            add_entry(c, v, SWPC_F_SXZ, kk, ii, jj, s, mm[4], INJ_GLUT4, 0, &bad);
            add_entry(c, v, SWPC_F_SXZ, kk - 1, ii, jj, s, mm[4], INJ_GLUT4, 0, &bad);
            add_entry(c, v, SWPC_F_SXZ, kk, ii - 1, jj, s, mm[4], INJ_GLUT4, 0, &bad);
            add_entry(c, v, SWPC_F_SXZ, kk - 1, ii - 1, jj, s, mm[4], INJ_GLUT4, 0, &bad);
            add_entry(c, v, SWPC_F_SYZ, kk, ii, jj, s, mm[3], INJ_GLUT4, 0, &bad);
            add_entry(c, v, SWPC_F_SYZ, kk - 1, ii, jj, s, mm[3], INJ_GLUT4, 0, &bad);
            add_entry(c, v, SWPC_F_SYZ, kk, ii, jj - 1, s, mm[3], INJ_GLUT4, 0, &bad);
            add_entry(c, v, SWPC_F_SYZ, kk - 1, ii, jj - 1, s, mm[3], INJ_GLUT4, 0, &bad);
        } else if (c->kind == SWPC_KIND_PSV) {
            // src/swpc_psv/m_source.f90:601-606: Sxx, Szz, and Sxz at 4 cells
            add_entry(c, v, SWPC_F_SXX, kk, ii, 1, s, mm[0], INJ_GLUT, 0, &bad);
            add_entry(c, v, SWPC_F_SZZ, kk, ii, 1, s, mm[2], INJ_GLUT, 0, &bad);
            add_entry(c, v, SWPC_F_SXZ, kk, ii, 1, s, mm[4], INJ_GLUT4, 0, &bad);
            add_entry(c, v, SWPC_F_SXZ, kk - 1, ii, 1, s, mm[4], INJ_GLUT4, 0, &bad);
            add_entry(c, v, SWPC_F_SXZ, kk, ii - 1, 1, s, mm[4], INJ_GLUT4, 0, &bad);
            add_entry(c, v, SWPC_F_SXZ, kk - 1, ii - 1, 1, s, mm[4], INJ_GLUT4, 0, &bad);
        } else {
            // src/swpc_sh/m_source.f90:583-587: Sxy and Syz at 2 cells each
            add_entry(c, v, SWPC_F_SXY, kk, ii, 1, s, mm[5], INJ_GLUT2, 0, &bad);
            add_entry(c, v, SWPC_F_SXY, kk, ii - 1, 1, s, mm[5], INJ_GLUT2, 0, &bad);
            add_entry(c, v, SWPC_F_SYZ, kk, ii, 1, s, mm[3], INJ_GLUT2, 0, &bad);
            add_entry(c, v, SWPC_F_SYZ, kk - 1, ii, 1, s, mm[3], INJ_GLUT2, 0, &bad);
        }
    }
    if (bad) return set_err(c, SWPC_ERR_ARG, "source cell outside the memory box");
    RC(build_list(c, v, &c->inj_glut, &c->ninj_glut, &c->glut_serial));
    c->nsrc_glut = nsrc;
    RC(stime_table(c, &c->stime_glut, nsrc, srcprm, stftype, true));
    if (c->mo_glut) { cudaFree(c->mo_glut); c->mo_glut = nullptr; }
    RC(dalloc(c, &c->mo_glut, std::max(nsrc, 1)));
    if (nsrc > 0) CK(cudaMemcpyAsync(c->mo_glut, mo, nsrc * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    // dt_dxyz = dt / (dx * dy * dz) (m_source.f90:305); 2D: dt / (dx * dz)
    c->dt_dxyz = is3d(c) ? c->d.dt / (c->d.dx * c->d.dy * c->d.dz) : c->d.dt / (c->d.dx * c->d.dz);
    return SWPC_OK;
}

extern "C" int swpc_bodyforce_setup(swpc_ctx *c, int nsrc, const int *isrc, const int *jsrc, const int *ksrc,
                                    const float *srcprm, const float *f3, int stftype) {
    if (!c || nsrc < 0) return SWPC_ERR_ARG;
    if (nsrc > 0 && (!isrc || !ksrc || !srcprm || !f3 || (is3d(c) && !jsrc)))
        return set_err(c, SWPC_ERR_ARG, "body-force arrays missing");
    CK(cudaSetDevice(c->device));
    invalidate_graph(c);
    std::vector<InjEntry> v;
    bool bad = false;
    if (!is3d(c)) {
        // src/swpc_psv/m_source.f90:642-645 and src/swpc_sh/m_source.f90:621:
        // V += f / rho(kk, ii) * stime * dt_dxz (/2 for P-SV)
        std::vector<long long> rc(std::max(nsrc, 1), 0);
        for (int s = 0; s < nsrc; s++) {
            const int ii = isrc[s], kk = ksrc[s];
            const float *f = f3 + 3 * s;
            if (!in_box(c, kk, ii, 1)) bad = true;
            rc[s] = (long long)(ii + 2) * c->g.Kp + (kk - 1 + KH);
            if (c->kind == SWPC_KIND_PSV) {
                add_entry(c, v, SWPC_F_VX, kk, ii, 1, s, f[0], INJ_BFPSV, 0, &bad);
                add_entry(c, v, SWPC_F_VX, kk, ii - 1, 1, s, f[0], INJ_BFPSV, 0, &bad);
                add_entry(c, v, SWPC_F_VZ, kk, ii, 1, s, f[2], INJ_BFPSV, 0, &bad);
                add_entry(c, v, SWPC_F_VZ, kk - 1, ii, 1, s, f[2], INJ_BFPSV, 0, &bad);
            } else {
                add_entry(c, v, SWPC_F_VY, kk, ii, 1, s, f[1], INJ_BFSH, 0, &bad);
            }
        }
        if (bad) return set_err(c, SWPC_ERR_ARG, "body-force cell outside the memory box");
        RC(build_list(c, v, &c->inj_bf, &c->ninj_bf, &c->bf_serial));
        c->nsrc_bf = nsrc;
        RC(stime_table(c, &c->stime_bf, nsrc, srcprm, stftype, false));
        if (c->rho_cell_bf) { cudaFree(c->rho_cell_bf); c->rho_cell_bf = nullptr; }
        RC(dalloc(c, &c->rho_cell_bf, rc.size()));
        CK(cudaMemcpyAsync(c->rho_cell_bf, rc.data(), rc.size() * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        c->dt_dxyz = c->d.dt / (c->d.dx * c->d.dz);
        return SWPC_OK;
    }
    for (int s = 0; s < nsrc; s++) {
        const int ii = isrc[s], jj = jsrc[s], kk = ksrc[s];
        const float *f = f3 + 3 * s;
        // m_source.f90:863-868 (buoyancy slots: 0 bx, 1 by, 2 bz)
        add_entry(c, v, SWPC_F_VX, kk, ii, jj, s, f[0], INJ_BF3, 0, &bad);
        add_entry(c, v, SWPC_F_VX, kk, ii - 1, jj, s, f[0], INJ_BF3, 0, &bad);
        add_entry(c, v, SWPC_F_VY, kk, ii, jj, s, f[1], INJ_BF3, 1, &bad);
        add_entry(c, v, SWPC_F_VY, kk, ii, jj - 1, s, f[1], INJ_BF3, 1, &bad);
        add_entry(c, v, SWPC_F_VZ, kk, ii, jj, s, f[2], INJ_BF3, 2, &bad);
        add_entry(c, v, SWPC_F_VZ, kk - 1, ii, jj, s, f[2], INJ_BF3, 2, &bad);
    }
    if (bad) return set_err(c, SWPC_ERR_ARG, "body-force cell outside the memory box");
    RC(build_list(c, v, &c->inj_bf, &c->ninj_bf, &c->bf_serial));
    c->nsrc_bf = nsrc;
    RC(stime_table(c, &c->stime_bf, nsrc, srcprm, stftype, false));
    c->dt_dxyz = c->d.dt / (c->d.dx * c->d.dy * c->d.dz);
    return SWPC_OK;
}

extern "C" int swpc_green_setup(swpc_ctx *c, int isrc, int jsrc, int ksrc, char cmp, float green_tbeg,
                                float green_trise, int stftype) {
    if (!c) return SWPC_ERR_ARG;
    if (!is3d(c)) return set_err(c, SWPC_ERR_ARG, "green mode is a 3D feature (m_green.f90)");
    if (cmp != 'x' && cmp != 'y' && cmp != 'z') return set_err(c, SWPC_ERR_ARG, "green_cmp must be x, y or z");
    CK(cudaSetDevice(c->device));
    invalidate_graph(c);
    std::vector<InjEntry> v;
    if (!green_entries(c, isrc, jsrc, ksrc, cmp, v))
        return set_err(c, SWPC_ERR_ARG, "green source cell outside the memory box");
    bool serial;
    RC(build_list(c, v, &c->inj_green, &c->ninj_green, &serial));
    const float prm[2] = {green_tbeg, green_trise};
    RC(stime_table(c, &c->stf_green, 1, prm, stftype, false));
    c->green_dt_dxyz = c->d.dt / (c->d.dx * c->d.dy * c->d.dz);
    c->green = true;
    return SWPC_OK;
}

// ---------------------------------------------------------------------------
// recorder
// ---------------------------------------------------------------------------
extern "C" int swpc_wav_setup(swpc_ctx *c, int nst, const int *ist, const int *jst, const int *kst, int ntdec_w,
                              int what, float M0, float UC) {
    if (!c || nst < 0 || ntdec_w < 1) return SWPC_ERR_ARG;
    if (nst > 0 && (!ist || !kst || (is3d(c) && !jst))) return set_err(c, SWPC_ERR_ARG, "station arrays missing");
    CK(cudaSetDevice(c->device));
    invalidate_graph(c);
    const Geo &g = c->g;
    if (!is3d(c) && (what & (SWPC_WAV_STRESS | SWPC_WAV_STRAIN)))
        return set_err(c, SWPC_ERR_ARG, "2D recorders support velocity and displacement");
    const int per = is3d(c) ? 3 : 2;
    std::vector<int> st(per * (size_t)std::max(nst, 1), 0);
    for (int n = 0; n < nst; n++) {
        const int i = ist[n], j = is3d(c) ? jst[n] : 1, k = kst[n];
        // stencils of wav__store reach i-2..i+2, j-2..j+2, k-2..k+2
        if (i < 1 || i > g.nx || k < 1 || k > g.nz || (is3d(c) && (j < 1 || j > g.ny)))
            return set_err(c, SWPC_ERR_ARG, "station cell outside the domain");
        if (is3d(c)) { st[3 * n] = i; st[3 * n + 1] = j; st[3 * n + 2] = k; }
        else { st[2 * n] = i; st[2 * n + 1] = k; }
    }
    c->nst = nst;
    c->ntdec_w = ntdec_w;
    c->wav_what = what;
    c->M0 = M0;
    c->UC = UC;
    // ntw = floor(real(nt-1)/real(ntdec_w) + 1.0) (m_wav.f90:92)
    c->ntw = (int)floorf((float)(c->d.nt - 1) / (float)ntdec_w + 1.0f);
    if (c->st_ijk) { cudaFree(c->st_ijk); c->st_ijk = nullptr; }
    RC(dalloc(c, &c->st_ijk, st.size()));
    CK(cudaMemcpyAsync(c->st_ijk, st.data(), st.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    const int nc2 = c->kind == SWPC_KIND_PSV ? 2 : 1;
    const int ncmp[4] = {is3d(c) ? 3 : nc2, is3d(c) ? 3 : nc2, 6, 6};
    for (int q = 0; q < 4; q++) {
        if (c->wav[q]) { cudaFree(c->wav[q]); c->wav[q] = nullptr; }
        RC(dalloc(c, &c->wav[q], (size_t)c->ntw * ncmp[q] * std::max(nst, 1)));
    }
    if (c->uacc) { cudaFree(c->uacc); c->uacc = nullptr; }
    if (c->eacc) { cudaFree(c->eacc); c->eacc = nullptr; }
    RC(dalloc(c, &c->uacc, 3 * (size_t)std::max(nst, 1)));
    RC(dalloc(c, &c->eacc, 6 * (size_t)std::max(nst, 1)));
    CK(cudaStreamSynchronize(c->stream));
    return SWPC_OK;
}

extern "C" int swpc_wav_dims(const swpc_ctx *c, int *ntw, int *nst) {
    if (!c) return SWPC_ERR_ARG;
    if (ntw) *ntw = c->ntw;
    if (nst) *nst = c->nst;
    return SWPC_OK;
}

extern "C" int swpc_wav_fetch(swpc_ctx *c, int what, float *out) {
    if (!c || !out) return SWPC_ERR_ARG;
    int q = what == SWPC_WAV_V ? 0 : what == SWPC_WAV_U ? 1 : what == SWPC_WAV_STRESS ? 2 : what == SWPC_WAV_STRAIN ? 3 : -1;
    if (q < 0) return set_err(c, SWPC_ERR_ARG, "unknown recorder component");
    if (!c->wav[q]) return set_err(c, SWPC_ERR_STATE, "swpc_wav_setup not called");
    const int nc2 = c->kind == SWPC_KIND_PSV ? 2 : 1;
    const int ncmp[4] = {is3d(c) ? 3 : nc2, is3d(c) ? 3 : nc2, 6, 6};
    CK(cudaMemcpyAsync(out, c->wav[q], (size_t)c->ntw * ncmp[q] * c->nst * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SWPC_OK;
}

// ---------------------------------------------------------------------------
// the time step
// ---------------------------------------------------------------------------
static int check_ready(swpc_ctx *c) {
    RC(check_na_wide(c));
    if (!c->medium_ready) return set_err(c, SWPC_ERR_STATE, "swpc_upload_medium not called");
    if (!c->kernel_ready) return set_err(c, SWPC_ERR_STATE, "swpc_kernel_setup not called");
    if (!c->absorb_ready && c->d.na > 0) return set_err(c, SWPC_ERR_STATE, "swpc_absorb_setup not called");
    return SWPC_OK;
}

static void fill_geo_common(const swpc_ctx *c, Geo &g, int &ibk, int &iek, int &jbk, int &jek, int &kek) {
    g = c->g; ibk = c->ibk; iek = c->iek; jbk = c->jbk; jek = c->jek; kek = c->kek;
}

// tensor maps of the staged kernels for the selected tile shapes
static int tma_ready(swpc_ctx *c) {
    const int key[4] = {c->stress_tbi, c->stress_tbj, c->vel_tbi, c->vel_tbj};
    if (c->tmaps && std::equal(key, key + 4, c->tma_key)) return SWPC_OK;
    if (!c->tmaps) c->tmaps = new TmaMaps();
    TmaMaps &m = *static_cast<TmaMaps *>(c->tmaps);
    const TmaSlabs s{c->slab, c->slab_nf, c->slab, c->slab_nf, c->hslab, c->hslab_nf};
    if (!tma_encode_stress(m, s, c->g, c->d.nm, key[0], key[1], c->prec) ||
        !tma_encode_vel(m, s, c->g, key[2], key[3], c->prec))
        return set_err(c, SWPC_ERR_CUDA, "cuTensorMapEncodeTiled failed for the field slab");
    std::copy(key, key + 4, c->tma_key);
    return SWPC_OK;
}

namespace swpc {
// tiles of a staged launch over the whole grid for nmem members grouped by
// mpc; the medium fields come from the context's slab
TmaTiles tma_tiles(const swpc_ctx *c, int bi, int bj, int nmem, int mpc, int nfields, int live) {
    TmaTiles t;
    t.nkt = (c->g.nz + 31) / 32;
    t.nit = (c->g.nx + bi - 1) / bi;
    t.njt = (c->g.ny + bj - 1) / bj;
    t.nmem = nmem;
    t.mgroups = (nmem + mpc - 1) / mpc;
    t.tiles_first = 0;
    // launch order: blocks of j tiles once a j plane of tiles (the fields the
    // kernel reads over bj planes, for the members whose tiles interleave in
    // the launch order) outgrows half of the L2
    const double plane = (double)nfields * live * c->g.Kp * c->g.Ip * bj * 4.0;
    const int jb = c->tile_jblock > 0 ? c->tile_jblock : (plane > 64e6 ? 16 : 1);
    t.jblock = std::max(1, std::min(jb, t.njt));
    // slab field order: FP32 V S R medium b; BF16_R V S medium b (R in the
    // 2-byte slab); F16_SR V medium b (S and R in the 2-byte slab)
    t.f_v = 0;
    t.f_state = 3;
    t.f_member = 0;
    t.f_med = c->prec == SWPC_PREC_F32 ? 9 + 6 * c->d.nm
            : (c->prec == SWPC_PREC_BF16_R || c->prec == SWPC_PREC_F16_R) ? 9 : 3;
    t.f_b = t.f_med + 7;
    t.f_h = 0;
    t.so = 0;
    t.ao = 0;
    t.err = c->d_err;
    return t;
}
}  // namespace swpc

static int launch_stress_kernel(swpc_ctx *c, int mask);
static int launch_vel_kernel(swpc_ctx *c, int mask);

static int launch_stress(swpc_ctx *c, int mask) {
    RC(check_ready(c));
    if (!is3d(c)) return update_stress_2d(c, mask);
    if (mask & 2) RC(pw_fill(c, 0));   // plane-wave side boundary before the absorber update
    if (c->abc == 1) {
        // Cerjan: the interior update over the whole domain, then the sponge
        // (absorb__update_stress's dispatch, m_absorb.f90:43-58)
        if (mask & 1) RC(launch_stress_kernel(c, 1));
        if (mask & 2) RC(launch_cerjan(c, 0));
        return SWPC_OK;
    }
    return launch_stress_kernel(c, mask);
}

static int launch_stress_kernel(swpc_ctx *c, int mask) {
    Str3Args a;
    memset(&a, 0, sizeof(a));
    fill_geo_common(c, a.g, a.ibk, a.iek, a.jbk, a.jek, a.kek);
    a.Vx = c->V[0]; a.Vy = c->V[1]; a.Vz = c->V[2];
    a.Sxx = c->S[0]; a.Syy = c->S[1]; a.Szz = c->S[2]; a.Syz = c->S[3]; a.Sxz = c->S[4]; a.Sxy = c->S[5];
    for (int q = 0; q < 18; q++) a.R[q] = c->R[q];
    a.lam = c->med[1]; a.mu = c->med[2]; a.taup = c->med[3]; a.taus = c->med[4];
    a.muyz = c->med[8]; a.muxz = c->med[9]; a.muxy = c->med[10];
    a.band = c->band; a.pmlcol = c->pmlcol;
    for (int q = 0; q < 9; q++) a.aV[q] = c->aux[q];
    a.gxc = c->gx[0]; a.gxe = c->gx[1]; a.gyc = c->gy[0]; a.gye = c->gy[1]; a.gzc = c->gz[0]; a.gze = c->gz[1];
    memcpy(a.e40, c->e40, sizeof(a.e40)); memcpy(a.e41, c->e41, sizeof(a.e41)); memcpy(a.r20, c->r20, sizeof(a.r20));
    memcpy(a.c1, c->c1, sizeof(a.c1)); memcpy(a.c2, c->c2, sizeof(a.c2)); memcpy(a.d1, c->d1, sizeof(a.d1));
    a.d2 = c->d2;
    a.dt = c->d.dt;
    a.mask = (c->d.na > 0 && c->abc == 0) ? mask : (mask & 1);
    a.scale = c->d_scale;
    dim3 block(32, c->bi, c->bj);
    dim3 grid((c->g.nz + 31) / 32, (c->g.nx + c->bi - 1) / c->bi, (c->g.ny + c->bj - 1) / c->bj);
    if (c->stress_tma && c->slab) {
        RC(tma_ready(c));
        const TmaTiles t = tma_tiles(c, c->stress_tbi, c->stress_tbj, 1, 1, kStressFields(c), 1);
        return cuda_check(c, launch_stress3d_tma(*static_cast<TmaMaps *>(c->tmaps), a, t, c->d.nm, c->stress_tbi,
                                                 c->stress_tbj, 1, c->stream, c->prec), "stress3d_tma launch");
    }
    if (c->stress_march && c->prec == SWPC_PREC_F32)
        launch_stress3d_march(a, c->d.nm, c->stress_mminb, c->stress_jc, c->stream);
    else launch_stress3d(a, c->d.nm, c->stress_minb, c->prec, grid, block, c->stream);
    return cuda_check(c, cudaGetLastError(), "stress3d launch");
}

static int launch_vel(swpc_ctx *c, int mask) {
    RC(check_ready(c));
    if (!is3d(c)) return update_vel_2d(c, mask);
    if (mask & 2) RC(pw_fill(c, 1));
    if (c->abc == 1) {
        // Cerjan (absorb__update_vel's dispatch, m_absorb.f90:60-75)
        if (mask & 1) RC(launch_vel_kernel(c, 1));
        if (mask & 2) RC(launch_cerjan(c, 1));
        return SWPC_OK;
    }
    return launch_vel_kernel(c, mask);
}

static int launch_vel_kernel(swpc_ctx *c, int mask) {
    Vel3Args a;
    memset(&a, 0, sizeof(a));
    fill_geo_common(c, a.g, a.ibk, a.iek, a.jbk, a.jek, a.kek);
    a.Vx = c->V[0]; a.Vy = c->V[1]; a.Vz = c->V[2];
    a.Sxx = c->S[0]; a.Syy = c->S[1]; a.Szz = c->S[2]; a.Syz = c->S[3]; a.Sxz = c->S[4]; a.Sxy = c->S[5];
    a.bx = c->med[5]; a.by = c->med[6]; a.bz = c->med[7];
    a.band = c->band; a.pmlcol = c->pmlcol;
    for (int q = 0; q < 9; q++) a.aS[q] = c->aux[9 + q];
    a.gxc = c->gx[0]; a.gxe = c->gx[1]; a.gyc = c->gy[0]; a.gye = c->gy[1]; a.gzc = c->gz[0]; a.gze = c->gz[1];
    memcpy(a.e40, c->e40, sizeof(a.e40)); memcpy(a.e41, c->e41, sizeof(a.e41)); memcpy(a.r20, c->r20, sizeof(a.r20));
    a.dt = c->d.dt;
    a.mask = (c->d.na > 0 && c->abc == 0) ? mask : (mask & 1);
    a.divo = c->div_out;
    a.dKp = c->div_geo[0]; a.dIp = c->div_geo[1]; a.di0 = c->div_geo[2]; a.dj0 = c->div_geo[3];
    a.dn = c->div_n;
    dim3 block(32, c->vbi, c->vbj);
    dim3 grid((c->g.nz + 31) / 32, (c->g.nx + c->vbi - 1) / c->vbi, (c->g.ny + c->vbj - 1) / c->vbj);
    a.scale = c->d_scale;
    if (c->vel_tma && c->slab) {
        RC(tma_ready(c));
        const TmaTiles t = tma_tiles(c, c->vel_tbi, c->vel_tbj, 1, 1, kVelFields, 1);
        return cuda_check(c, launch_vel3d_tma(*static_cast<TmaMaps *>(c->tmaps), a, t, c->vel_tbi, c->vel_tbj, 1,
                                              c->stream, c->prec), "vel3d_tma launch");
    }
    if (c->prec != SWPC_PREC_F32) launch_vel3d(a, c->vel_minb, c->prec, grid, block, c->stream);
    else if (c->vel_vec) launch_vel3d_vec(a, c->vel_vminb, dim3(32, c->vel_vbi, c->vel_vbj), c->stream);
    else if (c->vel_march) launch_vel3d_march(a, c->vel_mminb, c->vel_jc, c->stream);
    else launch_vel3d(a, c->vel_minb, SWPC_PREC_F32, grid, block, c->stream);
    return cuda_check(c, cudaGetLastError(), "vel3d launch");
}

static void fill_inj_fields(swpc_ctx *c, InjArgs &a) {
    for (int q = 0; q < 3; q++) a.fields[q] = c->V[q];
    for (int q = 0; q < 6; q++) a.fields[3 + q] = c->S[q];
    a.s_half = c->prec == SWPC_PREC_F16_SR;
    a.scale = c->d_scale;
    if (is3d(c)) { a.bfields[0] = c->med[5]; a.bfields[1] = c->med[6]; a.bfields[2] = c->med[7]; }
    else { a.bfields[0] = c->med[0]; a.bfields[1] = c->med[0]; a.bfields[2] = c->med[0]; }
}

namespace swpc {
InjArgs glut_args(swpc_ctx *c, int it, const int *d_it) {
    InjArgs a;
    memset(&a, 0, sizeof(a));
    a.list = c->inj_glut; a.n = c->ninj_glut; a.serial = c->glut_serial ? 1 : 0;
    a.it = it; a.d_it = d_it; a.nt = c->d.nt; a.nsrc = c->nsrc_glut;
    a.stime = c->stime_glut; a.mo = c->mo_glut; a.dt_dxyz = c->dt_dxyz;
    fill_inj_fields(c, a);
    return a;
}

InjArgs bf_args(swpc_ctx *c, int it, const int *d_it) {
    InjArgs a;
    memset(&a, 0, sizeof(a));
    a.list = c->inj_bf; a.n = c->ninj_bf; a.serial = c->bf_serial ? 1 : 0;
    a.it = it; a.d_it = d_it; a.nt = c->d.nt; a.nsrc = c->nsrc_bf;
    a.stime = c->stime_bf; a.dt_dxyz = c->dt_dxyz;
    a.rho_cell = c->rho_cell_bf;
    fill_inj_fields(c, a);
    return a;
}
}  // namespace swpc

static int launch_glut(swpc_ctx *c, int it, const int *d_it) {
    if (c->ninj_glut <= 0) return SWPC_OK;
    launch_inject(glut_args(c, it, d_it), c->stream);
    return cuda_check(c, cudaGetLastError(), "stressglut launch");
}

static int launch_bf(swpc_ctx *c, int it, const int *d_it) {
    if (c->ninj_bf <= 0) return SWPC_OK;
    launch_inject(bf_args(c, it, d_it), c->stream);
    return cuda_check(c, cudaGetLastError(), "bodyforce launch");
}

static int launch_green(swpc_ctx *c, int it, const int *d_it) {
    if (!c->green || c->ninj_green <= 0) return SWPC_OK;
    InjArgs a;
    memset(&a, 0, sizeof(a));
    a.list = c->inj_green; a.n = c->ninj_green; a.serial = 0;
    a.it = it; a.d_it = d_it; a.nt = c->d.nt; a.nsrc = 1;
    a.stime = c->stf_green; a.dt_dxyz = c->green_dt_dxyz;
    fill_inj_fields(c, a);
    launch_inject(a, c->stream);
    return cuda_check(c, cudaGetLastError(), "green launch");
}

static int launch_wav(swpc_ctx *c, int it, const int *d_it) {
    if (c->nst <= 0 || c->wav_what == 0) return SWPC_OK;
    if (!is3d(c)) return wav_store_2d(c, it, d_it);
    Wav3Args a;
    memset(&a, 0, sizeof(a));
    a.g = c->g; a.nst = c->nst; a.ntw = c->ntw; a.ntdec_w = c->ntdec_w; a.what = c->wav_what;
    a.it = it; a.d_it = d_it; a.st = c->st_ijk;
    a.Vx = c->V[0]; a.Vy = c->V[1]; a.Vz = c->V[2];
    a.Sxx = c->S[0]; a.Syy = c->S[1]; a.Szz = c->S[2]; a.Syz = c->S[3]; a.Sxz = c->S[4]; a.Sxy = c->S[5];
    a.uacc = c->uacc; a.eacc = c->eacc;
    a.wav_v = c->wav[0]; a.wav_u = c->wav[1]; a.wav_s = c->wav[2]; a.wav_e = c->wav[3];
    a.M0 = c->M0; a.UC = c->UC; a.dt = c->d.dt;
    memcpy(a.r40, c->r40, sizeof(a.r40)); memcpy(a.r41, c->r41, sizeof(a.r41));
    a.s_half = c->prec == SWPC_PREC_F16_SR;
    a.scale = c->d_scale;
    // outside sampling steps the kernel only integrates u / strain
    if (!d_it && (it - 1) % c->ntdec_w != 0 && !(c->wav_what & (SWPC_WAV_U | SWPC_WAV_STRAIN))) return SWPC_OK;
    launch_wav3d(a, c->stream);
    return cuda_check(c, cudaGetLastError(), "wav launch");
}

static int prepare(swpc_ctx *c) {
    if (!c) return SWPC_ERR_ARG;
    CK(cudaSetDevice(c->device));
    if (!is3d(c)) RC(refresh_2d(c));
    return SWPC_OK;
}
#define PREP(c) do { int _rc = prepare(c); if (_rc) return _rc; } while (0)

extern "C" int swpc_kernel_update_stress(swpc_ctx *c) { PREP(c); return launch_stress(c, 1); }
extern "C" int swpc_absorb_update_stress(swpc_ctx *c) { PREP(c); return launch_stress(c, 2); }
extern "C" int swpc_kernel_update_vel(swpc_ctx *c) { PREP(c); return launch_vel(c, 1); }
extern "C" int swpc_absorb_update_vel(swpc_ctx *c) { PREP(c); return launch_vel(c, 2); }
extern "C" int swpc_update_stress(swpc_ctx *c) { PREP(c); return launch_stress(c, 3); }
extern "C" int swpc_update_vel(swpc_ctx *c) { PREP(c); return launch_vel(c, 3); }
extern "C" int swpc_source_stressglut(swpc_ctx *c, int it) { return c ? launch_glut(c, it, nullptr) : SWPC_ERR_ARG; }
extern "C" int swpc_source_bodyforce(swpc_ctx *c, int it) { return c ? launch_bf(c, it, nullptr) : SWPC_ERR_ARG; }
extern "C" int swpc_green_source(swpc_ctx *c, int it) { return c ? launch_green(c, it, nullptr) : SWPC_ERR_ARG; }
// single domain: the exchange only zeroes ghost planes, which no kernel writes except in plane-wave mode
extern "C" int swpc_comm_stress(swpc_ctx *c) {
    if (!c) return SWPC_ERR_ARG;
    if (!c->pw_mode) return SWPC_OK;
    PREP(c);
    return pw_comm_zero(c, 1);
}
extern "C" int swpc_comm_vel(swpc_ctx *c) {
    if (!c) return SWPC_ERR_ARG;
    if (!c->pw_mode) return SWPC_OK;
    PREP(c);
    return pw_comm_zero(c, 0);
}
extern "C" int swpc_wav_store(swpc_ctx *c, int it) { PREP(c); return launch_wav(c, it, nullptr); }

// main.f90:125-144 loop body (report__progress is driven by the caller
// between steps) in two halves: up to global__comm_stress (half 0) and from
// there up to global__comm_vel (half 1); with record = false the wavefield
// advances without wav__store, green__store and snap__write
static int step_half0(swpc_ctx *c, int it, const int *d_it, bool record) {
    if (record) {
        RC(launch_wav(c, it, d_it));
        RC(green_store_launch(c, it, d_it));
        RC(snap_launch(c, it, d_it));
    }
    RC(rescale_before_stress(c, it, d_it));   // FP16 forms: re-centre the scales, on the device (swpc_prec.cu)
    RC(launch_stress(c, 3));
    RC(rescale_after_stress(c));
    return launch_glut(c, it, d_it);
}
static int step_half1(swpc_ctx *c, int it, const int *d_it) {
    if (c->kind == SWPC_KIND_PSV && c->ninj_bf > 0) {
        // P-SV applies body forces between the interior and absorber velocity
        // updates (src/swpc_psv/main.f90:106-110)
        RC(launch_vel(c, 1));
        RC(launch_bf(c, it, d_it));
        RC(launch_vel(c, 2));
    } else {
        RC(launch_vel(c, 3));
        RC(launch_bf(c, it, d_it));
    }
    return launch_green(c, it, d_it);
}

static int step_body(swpc_ctx *c, int it, const int *d_it, bool record = true) {
    RC(step_half0(c, it, d_it, record));
    RC(pw_comm_zero(c, 1));   // global__comm_stress (no-op outside plane-wave mode)
    RC(step_half1(c, it, d_it));
    RC(pw_comm_zero(c, 0));   // global__comm_vel
    return SWPC_OK;
}

extern "C" int swpc_step_half(swpc_ctx *c, int it, int half) {
    if (!c) return SWPC_ERR_ARG;
    if (it < 1 || it > c->d.nt) return set_err(c, SWPC_ERR_ARG, "time step index outside 1..nt");
    if (half != 0 && half != 1) return set_err(c, SWPC_ERR_ARG, "half must be 0 (stress) or 1 (velocity)");
    if (c->pw_mode) return set_err(c, SWPC_ERR_STATE, "the plane-wave mode steps whole steps (swpc_step)");
    PREP(c);
    return half == 0 ? step_half0(c, it, nullptr, true) : step_half1(c, it, nullptr);
}

extern "C" int swpc_step(swpc_ctx *c, int it) {
    if (!c) return SWPC_ERR_ARG;
    if (it < 1 || it > c->d.nt) return set_err(c, SWPC_ERR_ARG, "time step index outside 1..nt");
    PREP(c);
    return step_body(c, it, nullptr);
}

namespace swpc {
int step_state(swpc_ctx *c, int it) {
    if (!c) return SWPC_ERR_ARG;
    if (it < 1 || it > c->d.nt) return set_err(c, SWPC_ERR_ARG, "time step index outside 1..nt");
    PREP(c);
    return step_body(c, it, nullptr, false);
}
}  // namespace swpc

static int build_graph(swpc_ctx *c) {
    if (c->graph_exec) return SWPC_OK;
    RC(check_ready(c));
    PREP(c);
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = step_body(c, 0, c->d_it);
    if (!rc) launch_advance_it(c->d_it, c->stream);
    cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    if (rc) return rc;
    CK(e);
    e = cudaGraphInstantiate(&c->graph_exec, graph, 0);
    cudaGraphDestroy(graph);
    CK(e);
    return SWPC_OK;
}

extern "C" int swpc_run(swpc_ctx *c, int it0, int nsteps) {
    if (!c) return SWPC_ERR_ARG;
    if (nsteps <= 0) return SWPC_OK;
    if (it0 < 1 || it0 + nsteps - 1 > c->d.nt) return set_err(c, SWPC_ERR_ARG, "time steps outside 1..nt");
    CK(cudaSetDevice(c->device));
    RC(build_graph(c));
    CK(cudaMemcpyAsync(c->d_it, &it0, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    for (int n = 0; n < nsteps; n++) CK(cudaGraphLaunch(c->graph_exec, c->stream));
    return SWPC_OK;
}

extern "C" int swpc_time_steps(swpc_ctx *c, int it0, int nsteps, float *ms) {
    if (!c || !ms) return SWPC_ERR_ARG;
    CK(cudaSetDevice(c->device));
    RC(build_graph(c));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaEventRecord(e0, c->stream));
    int rc = swpc_run(c, it0, nsteps);
    CK(cudaEventRecord(e1, c->stream));
    CK(cudaEventSynchronize(e1));
    CK(cudaEventElapsedTime(ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

// ---------------------------------------------------------------------------
// report: kernel__vmax + divergence check (m_report.f90:134-152)
// ---------------------------------------------------------------------------
extern "C" int swpc_vmax(swpc_ctx *c, float out[3]) {
    if (!c || !out) return SWPC_ERR_ARG;
    CK(cudaSetDevice(c->device));
    if (!c->medium_ready) return set_err(c, SWPC_ERR_STATE, "swpc_upload_medium not called");
    if (!is3d(c)) {
        RC(vmax_2d(c, out));
    } else {
        const int margin = 5, na = c->d.na;
        VmaxArgs a;
        a.g = c->g;
        // global bounds of m_kernel.f90:343-344 in this box's coordinates
        a.j0 = std::max(na + margin + 1 - c->joff, c->jbk);
        a.j1 = std::min(c->nyg - na - margin - c->joff, c->jek);
        a.i0 = std::max(na + margin + 1 - c->ioff, c->ibk);
        a.i1 = std::min(c->nxg - na - margin - c->ioff, c->iek);
        a.kob = c->kob;
        a.Vx = c->V[0]; a.Vy = c->V[1]; a.Vz = c->V[2];
        a.out = c->vmax_buf;
        CK(cudaMemsetAsync(c->vmax_buf, 0, 4 * sizeof(unsigned int), c->stream));
        if (a.i1 >= a.i0 && a.j1 >= a.j0) {
            launch_vmax3d(a, c->stream);
            CK(cudaGetLastError());
        }
        CK(cudaMemcpyAsync(c->h_vmax, c->vmax_buf, 3 * sizeof(unsigned int), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (int q = 0; q < 3; q++) memcpy(&out[q], &c->h_vmax[q], sizeof(float));
    }
    float mx = std::max(out[0], std::max(out[1], out[2]));
    if (!(mx * c->UC <= 1e5f))   // also catches NaN
        return set_err(c, SWPC_ERR_DIVERGED, "numerical divergence detected (max |V| * UC > 1e5)");
    return SWPC_OK;
}

// ---------------------------------------------------------------------------
// field transfer
// ---------------------------------------------------------------------------
static float *field_ptr(swpc_ctx *c, int field) {
    if (field >= SWPC_F_VX && field <= SWPC_F_VZ) return c->V[field - SWPC_F_VX];
    if (field >= SWPC_F_SXX && field <= SWPC_F_SXY) return c->S[field - SWPC_F_SXX];
    if (field >= SWPC_F_R && field < SWPC_F_R + 18) return c->R[field - SWPC_F_R];
    return nullptr;
}

namespace swpc {
// PML auxiliary array `dev` (compact per column) <-> Fortran memory box
int aux_transfer_ptr(swpc_ctx *c, float *dev, float *out, const float *in, int ld_k, int ld_i);
}

static int aux_transfer(swpc_ctx *c, int q, float *out, const float *in, int ld_k, int ld_i) {
    if (!c->absorb_ready || !c->aux[q]) return set_err(c, SWPC_ERR_STATE, "swpc_absorb_setup not called");
    return aux_transfer_ptr(c, c->aux[q], out, in, ld_k, ld_i);
}

int swpc::aux_transfer_ptr(swpc_ctx *c, float *dev, float *out, const float *in, int ld_k, int ld_i) {
    const Geo &g = c->g;
    if (!is3d(c)) {
        std::vector<float> buf((size_t)std::max<long long>(c->npml, 1));
        std::vector<int2> pc(g.Ip);
        CK(cudaMemcpyAsync(pc.data(), c->pmlcol, pc.size() * sizeof(int2), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(buf.data(), dev, c->npml * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (int i = -2; i <= g.nx + 3; i++) {
            const long long h = (long long)(i + 2) * ld_k;
            const int2 p = (i >= 1 && i <= g.nx) ? pc[i + 2] : make_int2(1, -1);
            for (int k = -2; k <= g.nz + 3; k++) {
                const bool has = p.y >= 0 && k >= p.x && k <= g.nz;
                if (out) out[h + (k + 2)] = has ? buf[(size_t)p.y + (k - p.x)] : 0.0f;
                else if (has) buf[(size_t)p.y + (k - p.x)] = in[h + (k + 2)];
            }
        }
        if (in) {
            CK(cudaMemcpyAsync(dev, buf.data(), c->npml * sizeof(float), cudaMemcpyHostToDevice, c->stream));
            CK(cudaStreamSynchronize(c->stream));
        }
        return SWPC_OK;
    }
    std::vector<float> buf((size_t)std::max<long long>(c->npml, 1));
    std::vector<int2> pc((size_t)g.Ip * g.Jp);
    CK(cudaMemcpyAsync(pc.data(), c->pmlcol, pc.size() * sizeof(int2), cudaMemcpyDeviceToHost, c->stream));
    if (in == nullptr || true)
        CK(cudaMemcpyAsync(buf.data(), dev, c->npml * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int j = -2; j <= g.ny + 3; j++)
        for (int i = -2; i <= g.nx + 3; i++) {
            const long long h = ((long long)(j + 2) * ld_i + (i + 2)) * ld_k;
            const bool dom = i >= 1 && i <= g.nx && j >= 1 && j <= g.ny;
            const int2 p = dom ? pc[col_index(g, i, j)] : make_int2(1, -1);
            for (int k = -2; k <= g.nz + 3; k++) {
                const bool has = p.y >= 0 && k >= p.x && k <= g.nz;
                if (out) out[h + (k + 2)] = has ? buf[(size_t)p.y + (k - p.x)] : 0.0f;
                else if (has) buf[(size_t)p.y + (k - p.x)] = in[h + (k + 2)];
            }
        }
    if (in) {
        CK(cudaMemcpyAsync(dev, buf.data(), c->npml * sizeof(float), cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return SWPC_OK;
}

extern "C" int swpc_download_field(swpc_ctx *c, int field, float *out, int ld_k, int ld_i) {
    if (!c || !out) return SWPC_ERR_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    if (field >= SWPC_F_AUX && field < SWPC_F_AUX + 18) return aux_transfer(c, field - SWPC_F_AUX, out, nullptr, ld_k, ld_i);
    if (field > SWPC_F_MED && field <= SWPC_F_MED + 10) {
        if (!is3d(c)) return set_err(c, SWPC_ERR_ARG, "medium field ids address the 3D medium");
        return copy_box(c, c->med[field - SWPC_F_MED], nullptr, out, ld_k, ld_i);
    }
    float *p = field_ptr(c, field);
    if (!p) return set_err(c, SWPC_ERR_ARG, "unknown or unallocated field id");
    if (field_storage(c, field) != 0) {
        // reduced-precision storage: widen to FP32 on the device first
        float *tmp = nullptr;
        int rc = prec_to_f32(c, field, p, &tmp);
        if (!rc) rc = copy_box(c, tmp, nullptr, out, ld_k, ld_i);
        cudaStreamSynchronize(c->stream);
        if (tmp) cudaFree(tmp);
        return rc;
    }
    return copy_box(c, p, nullptr, out, ld_k, ld_i);
}

extern "C" int swpc_upload_field(swpc_ctx *c, int field, const float *in, int ld_k, int ld_i) {
    if (!c || !in) return SWPC_ERR_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    if (field >= SWPC_F_AUX && field < SWPC_F_AUX + 18) return aux_transfer(c, field - SWPC_F_AUX, nullptr, in, ld_k, ld_i);
    float *p = field_ptr(c, field);
    if (!p) return set_err(c, SWPC_ERR_ARG, "unknown or unallocated field id");
    if (field_storage(c, field) != 0) {
        // reduced-precision storage: round the FP32 upload on the device
        float *tmp = nullptr;
        int rc = prec_to_f32(c, field, p, &tmp);   // keeps the cells outside the box
        if (!rc) rc = copy_box(c, tmp, in, nullptr, ld_k, ld_i);
        if (!rc) rc = prec_from_f32(c, field, tmp, p);
        cudaStreamSynchronize(c->stream);
        if (tmp) cudaFree(tmp);
        return rc;
    }
    return copy_box(c, p, in, nullptr, ld_k, ld_i);
}
