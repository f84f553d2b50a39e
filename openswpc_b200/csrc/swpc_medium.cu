// swpc_medium.cu -- the layered model and medium__setup of the 3D code on
// the device.
//
// The reference builds the medium on the host before the time loop:
// vmodel_lhm with the lhm_rmed perturbation (src/swpc_3d/m_vmodel_lhm.f90:
// 21-169, m_vmodel_lhm_rmed.f90:187-195, vcheck src/shared/m_fdtool.f90:
// 15-48), then medium__setup (src/swpc_3d/m_medium.f90:36-467).  Here every
// per-cell step of both runs in HBM, with explicit round-to-nearest
// intrinsics in the operation order of the host restatement (swpc_host.cpp,
// compiled without contraction), so the fields and the integer maps equal
// swpc_vmodel_lhm + swpc_setup_medium bit for bit.  The scalars (layer
// table, relaxation times, zeta, the relaxation constant) come from the host
// routines themselves.
//
// Between the model and the setup the per-cell arrays live in the
// context's medium arrays: lam and mu in their own, Qp in taup, Qs in taus
// and rho in muyz (the 3D slab keeps no rho); the last pass of
// averaged_medium replaces it with muyz.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <vector>

#include "swpc_ctx.h"
#include "swpc_host.h"

using namespace swpc;

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

namespace {

constexpr float kEpsF = 1.1920929e-07f;   // epsilon(1.0)

// the layered model at one depth row k: the last layer l with z(k) >= depth(l)
struct KRow {
    float r0, p0, s0, qa, qb;
    int kind;   // 0 air (z < depth(1), z < 0), 1 layer with vcheck (vp, vs > 0), 2 layer without,
                // 3 seawater (0 <= z < depth(1); p0 holds its lam)
};

void drop_graph(swpc_ctx *c) {
    c->desc_dirty = true;
    if (c->graph_exec) {
        cudaGraphExecDestroy(c->graph_exec);
        c->graph_exec = nullptr;
    }
}

// the memory box k, i, j in [-2, n+3] of the grid-stride index q
__device__ __forceinline__ void box_cell(const Geo &g, long long q, int &k, int &i, int &j) {
    const int nkb = g.nz + 6, nib = g.nx + 6;
    k = (int)(q % nkb) - 2;
    const long long r = q / nkb;
    i = (int)(r % nib) - 2;
    j = (int)(r / nib) - 2;
}

__device__ __forceinline__ long long box_cells(const Geo &g) { return (long long)(g.nz + 6) * (g.nx + 6) * (g.ny + 6); }

// vcheck (m_fdtool.f90:15-48)
__device__ __forceinline__ void vcheck_dev(float &vp, float &vs, float &rho, float xi, float vmin, float vmax,
                                           float rhomin) {
    float gamma = __fdiv_rn(vp, vs);
    if (gamma < kEpsF) gamma = __fsqrt_rn(3.0f);
    if (vp > vmax || vs > vmax) {
        const float xi2 = __fsub_rn(__fdiv_rn(__fmul_rn(__fadd_rn(1.0f, xi), vmax), vp), 1.0f);
        vp = vmax;
        vs = __fdiv_rn(vmax, gamma);
        rho = __fdiv_rn(__fmul_rn(rho, __fadd_rn(1.0f, __fmul_rn(0.8f, xi2))), __fadd_rn(1.0f, __fmul_rn(0.8f, xi)));
    }
    if (vp < vmin || vs < vmin) {
        vs = vmin;
        vp = __fmul_rn(vmin, gamma);
    }
    if (rho < rhomin) rho = rhomin;
}

// vmodel_lhm / lhm_rmed per cell.  With has_xi the rho array holds the
// perturbation xi on entry; each cell reads its own xi before writing rho.
__global__ void vmodel_kernel(Geo g, const KRow *__restrict__ rows, int has_xi, float vcut, float vmax_r, float rhomin,
                              float *rho, float *lam, float *mu, float *qp, float *qs) {
    const long long n = box_cells(g);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        int k, i, j;
        box_cell(g, q, k, i, j);
        const long long e = cell_index(g, k, i, j);
        const KRow r = rows[k + 2];
        if (r.kind == 0) {
            rho[e] = 0.001f; mu[e] = 0.0f; lam[e] = 0.0f; qp[e] = 10.0f; qs[e] = 10.0f;
            continue;
        }
        if (r.kind == 3) {
            rho[e] = 1.0f; mu[e] = 0.0f; lam[e] = r.p0; qp[e] = 1000000.0f; qs[e] = 1000000.0f;
            continue;
        }
        float rho1 = r.r0, vp1 = r.p0, vs1 = r.s0;
        if (has_xi) {
            const float x = rho[e];
            rho1 = __fmul_rn(r.r0, __fadd_rn(1.0f, __fmul_rn(0.8f, x)));
            vp1 = __fmul_rn(__fmul_rn(1.0f, r.p0), __fadd_rn(1.0f, x));
            vs1 = __fmul_rn(__fmul_rn(1.0f, r.s0), __fadd_rn(1.0f, x));
            if (r.kind == 1) vcheck_dev(vp1, vs1, rho1, x, vcut, vmax_r, rhomin);
        }
        rho[e] = rho1;
        mu[e] = __fmul_rn(__fmul_rn(rho1, vs1), vs1);
        lam[e] = __fmul_rn(rho1, __fsub_rn(__fmul_rn(vp1, vp1), __fmul_rn(__fmul_rn(2.0f, vs1), vs1)));
        qp[e] = r.qa;
        qs[e] = r.qb;
    }
}

// stabilize_absorber (m_medium.f90:276-340), one thread per column i, j in
// [0, n+1]: from the first absorber depth within two columns (kbeg_a,
// m_global.f90:336-345) down, a low-velocity layer of at most 20 cells takes
// the medium of the cell above it, then shear velocities below 0.4 vmax are
// raised to it with vp = sqrt(3) vs.  The walk down a column is sequential,
// as each cell compares with the (possibly replaced) cell above.
__global__ void stabilize_kernel(Geo g, int na, float vmax, float *rho, float *lam, float *mu, float *taup,
                                 float *taus) {
    const int ni = g.nx + 2, nj = g.ny + 2;
    const long long ncol = (long long)ni * nj;
    const float vmin_pml = vmax * 0.4f;
    const int lv_thick = 20;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncol; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % ni), j = (int)(q / ni);
        // min of kbeg_a over i-2..i+2, j-2..j+2: 1 when a side absorber column is among them
        const bool side = i - 2 <= na || g.nx - na + 1 <= i + 2 || j - 2 <= na || g.ny - na + 1 <= j + 2;
        const int k0 = side ? 1 : g.nz - na + 1;
        for (int k = k0; k <= g.nz; k++) {
            const long long e = cell_index(g, k, i, j), u = cell_index(g, k - 1, i, j);
            if (lam[e] < lam[u] || mu[e] < mu[u]) {
                int k2 = k + 1;
                for (; k2 <= g.nz; k2++) {
                    const long long e2 = cell_index(g, k2, i, j), u2 = cell_index(g, k2 - 1, i, j);
                    if (lam[e2] > lam[u2] || mu[e2] > mu[u2]) break;
                }
                if (k2 - k <= lv_thick) {
                    rho[e] = rho[u]; lam[e] = lam[u]; mu[e] = mu[u]; taup[e] = taup[u]; taus[e] = taus[u];
                    k = k2 - 1;
                }
            }
        }
        for (int k = k0; k <= g.nz; k++) {
            const long long e = cell_index(g, k, i, j);
            float vp = __fsqrt_rn(__fdiv_rn(__fadd_rn(lam[e], __fmul_rn(2.0f, mu[e])), rho[e]));
            float vs = __fsqrt_rn(__fdiv_rn(mu[e], rho[e]));
            if (vs < kEpsF) continue;   // ocean and air
            const float gamma = __fsqrt_rn(3.0f);
            if (vs < vmin_pml) {
                vs = vmin_pml;
                vp = __fmul_rn(vs, gamma);
                lam[e] = __fmul_rn(rho[e], __fsub_rn(__fmul_rn(vp, vp), __fmul_rn(2.0f, __fmul_rn(vs, vs))));
                mu[e] = __fmul_rn(rho[e], __fmul_rn(vs, vs));
            }
        }
    }
}

// absorber homogenisation (m_medium.f90:124-190): the x sides copy column
// na+1 / nx-na, then the y sides row na+1 / ny-na, then the bottom layer
// nz-na.  The three passes compose to one gather from the clamped cell,
// which is a fixed point of the clamp and so is never written here.
__global__ void homogenise_kernel(Geo g, int na, float *f0, float *f1, float *f2, float *f3, float *f4) {
    const long long n = box_cells(g);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        int k, i, j;
        box_cell(g, q, k, i, j);
        const int ci = i <= na ? na + 1 : (i >= g.nx - na + 1 ? g.nx - na : i);
        const int cj = j <= na ? na + 1 : (j >= g.ny - na + 1 ? g.ny - na : j);
        const int ck = k >= g.nz - na + 1 ? g.nz - na : k;
        if (ci == i && cj == j && ck == k) continue;
        const long long e = cell_index(g, k, i, j), s = cell_index(g, ck, ci, cj);
        f0[e] = f0[s]; f1[e] = f1[s]; f2[e] = f2[s]; f3[e] = f3[s]; f4[e] = f4[s];
    }
}

// hypot in single precision from the exact double squares: one rounding of
// the sum, the square root in double, one rounding to float
__device__ __forceinline__ float hypot_sp(float x, float y) {
    const double xx = __dmul_rn((double)x, (double)x), yy = __dmul_rn((double)y, (double)y);
    return __double2float_rn(__dsqrt_rn(__dadd_rn(xx, yy)));
}

// tau method (m_medium.f90:193-207) and relaxed_medium (m_medium.f90:234-274)
__global__ void tau_relax_kernel(Geo g, float nmz, int relax, float ccr, float cci, float *lam, float *mu, float *taup,
                                 float *taus) {
    const long long n = box_cells(g);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        int k, i, j;
        box_cell(g, q, k, i, j);
        const long long e = cell_index(g, k, i, j);
        const float tp = __fdiv_rn(nmz, taup[e]), ts = __fdiv_rn(nmz, taus[e]);
        taup[e] = tp;
        taus[e] = ts;
        if (!relax) continue;
        const float rb2 = mu[e];
        const float ra2 = __fadd_rn(lam[e], __fmul_rn(2.0f, mu[e]));
        const float tt[2] = {ts, tp};
        float chi[2];
#pragma unroll
        for (int m = 0; m < 2; m++) {
            const float zr = __fsub_rn(1.0f, __fmul_rn(ccr, tt[m]));
            const float zi = __fsub_rn(0.0f, __fmul_rn(cci, tt[m]));
            const float wr = __fsqrt_rn(__fmul_rn(0.5f, __fadd_rn(hypot_sp(zr, zi), zr)));
            const float wi = __fmul_rn(0.5f, __fdiv_rn(zi, wr));
            chi[m] = __fdiv_rn(1.0f, __fdiv_rn(wr, __fadd_rn(__fmul_rn(wr, wr), __fmul_rn(wi, wi))));
        }
        const float mu1 = __fdiv_rn(rb2, __fmul_rn(chi[0], chi[0]));
        mu[e] = mu1;
        lam[e] = __fsub_rn(__fdiv_rn(ra2, __fmul_rn(chi[1], chi[1])), __fmul_rn(2.0f, mu1));
    }
}

// surface_detection, first part (m_medium.f90:342-370): per column i, j in
// [0, n+2] the last k in [1, nz-1] with |f(k)| < eps < |f(k+1)|, for f = lam
// (kfs) and mu (kob); 0 where none.  One warp per column, lanes along k.
__global__ void surface_kernel(Geo g, const float *__restrict__ lam, const float *__restrict__ mu, int *kfs,
                               int *kob) {
    const int lane = threadIdx.x & 31;
    const long long ncol = (long long)(g.nx + 3) * (g.ny + 3);
    const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long w = w0; w < ncol; w += nw) {
        const int i = (int)(w % (g.nx + 3)), j = (int)(w / (g.nx + 3));
        const long long col = col_index(g, i, j);
        int f = 0, o = 0;
        for (int k0 = 1; k0 <= g.nz - 1; k0 += 32) {
            const int k = k0 + lane;
            if (k <= g.nz - 1) {
                const long long e = col * g.Kp + (k - 1 + KH);
                if (fabsf(mu[e]) < kEpsF && fabsf(mu[e + 1]) > kEpsF) o = k;
                if (fabsf(lam[e]) < kEpsF && fabsf(lam[e + 1]) > kEpsF) f = k;
            }
        }
        f = __reduce_max_sync(0xffffffffu, f);
        o = __reduce_max_sync(0xffffffffu, o);
        if (lane == 0) {
            kfs[col] = f;
            kob[col] = o;
        }
    }
}

// surface_detection, second part (m_medium.f90:372-397): the 2nd-order band
// of each column i, j in [1, n] from the extremes over its 6 x 6
// neighbourhood
__global__ void band_kernel(Geo g, const int *__restrict__ kfs, const int *__restrict__ kob, int4 *band) {
    const long long ncol = (long long)g.nx * g.ny;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncol; q += (long long)gridDim.x * blockDim.x) {
        const int i = 1 + (int)(q % g.nx), j = 1 + (int)(q / g.nx);
        int fmn = 1 << 30, fmx = -(1 << 30), omn = 1 << 30, omx = -(1 << 30);
        for (int jj = j - 2; jj <= j + 3; jj++)
            for (int ii = i - 2; ii <= i + 3; ii++) {
                const long long cc = col_index(g, ii, jj);
                const int f = kfs[cc], o = kob[cc];
                fmn = min(fmn, f); fmx = max(fmx, f);
                omn = min(omn, o); omx = max(omx, o);
            }
        band[col_index(g, i, j)] = make_int4(max(fmn - 2, 1), min(fmx + 2, g.nz), max(omn - 2, 1), min(omx + 2, g.nz));
    }
}

// velocity_minmax (m_medium.f90:399-430) below the free surface of each
// column: out[0] = bits of max vp + 1 (0: no cell), out[1] = bits of min
// vs >= eps (all ones: none).  NaN values are skipped, as the host's
// comparisons skip them.
__global__ void vminmax_kernel(Geo g, const float *__restrict__ rho, const float *__restrict__ lam,
                               const float *__restrict__ mu, const int *__restrict__ kfs, unsigned *out) {
    const long long n = (long long)g.nz * g.nx * g.ny;
    unsigned mx = 0u, mn = 0xffffffffu;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int k = 1 + (int)(q % g.nz);
        const long long r = q / g.nz;
        const int i = 1 + (int)(r % g.nx), j = 1 + (int)(r / g.nx);
        const long long col = col_index(g, i, j);
        if (k < kfs[col] + 1) continue;
        const long long e = col * g.Kp + (k - 1 + KH);
        const float rr = rho[e], l = lam[e], m = mu[e];
        const float vp = __fsqrt_rn(__fdiv_rn(__fadd_rn(l, __fmul_rn(2.0f, m)), rr));
        const float vs = __fsqrt_rn(__fdiv_rn(m, rr));
        if (!isnan(vp)) mx = max(mx, __float_as_uint(vp == 0.0f ? 0.0f : vp) + 1u);
        if (!isnan(vs) && !(vs < kEpsF)) mn = min(mn, __float_as_uint(vs));
    }
    mx = __reduce_max_sync(0xffffffffu, mx);
    mn = __reduce_min_sync(0xffffffffu, mn);
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&out[0], mx);
        atomicMin(&out[1], mn);
    }
}

swpc_grid grid_of(const swpc_ctx *c, float zbeg) {
    swpc_grid g = {};
    g.nx = c->d.nx; g.ny = c->d.ny; g.nz = c->d.nz; g.na = c->d.na; g.nm = c->d.nm;
    g.dx = c->d.dx; g.dy = c->d.dy; g.dz = c->d.dz; g.dt = c->d.dt;
    g.zbeg = zbeg; g.tbeg = c->d.tbeg;
    return g;
}

bool device_pointer(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

constexpr int kGrid = 148 * 8, kBlock = 256;

}  // namespace

extern "C" int swpc_vmodel_lhm_device(swpc_ctx *c, int nlayer, const float *depth, const float *rho0,
                                      const float *vp0, const float *vs0, const float *qp0, const float *qs0,
                                      float vcut, float rhomin, float zbeg, const float *xi, int ld_k, int ld_i) {
    return swpc_vmodel_lhm_device_opt(c, nlayer, depth, rho0, vp0, vs0, qp0, qs0, vcut, rhomin, zbeg, xi, ld_k, ld_i,
                                      0);
}

extern "C" int swpc_vmodel_lhm_device_opt(swpc_ctx *c, int nlayer, const float *depth, const float *rho0,
                                          const float *vp0, const float *vs0, const float *qp0, const float *qs0,
                                          float vcut, float rhomin, float zbeg, const float *xi, int ld_k, int ld_i,
                                          int munk_profile) {
    if (!c) return SWPC_ERR_ARG;
    if (c->kind != SWPC_KIND_3D) return set_err(c, SWPC_ERR_ARG, "the device medium setup is for the 3D code");
    RC(check_na_wide(c));
    if (nlayer < 1 || !depth || !rho0 || !vp0 || !vs0 || !qp0 || !qs0)
        return set_err(c, SWPC_ERR_ARG, "layer table missing");
    CK(cudaSetDevice(c->device));
    drop_graph(c);
    c->medium_ready = false;
    c->vmodel_ready = false;
    const Geo &g = c->g;
    const swpc_grid sg = grid_of(c, zbeg);
    std::vector<float> r0(nlayer), p0(nlayer), s0(nlayer), qa(nlayer), qb(nlayer);
    float vmax_r = 0.0f;
    lhm_layers(&sg, nlayer, depth, rho0, vp0, vs0, qp0, qs0, vcut, r0.data(), p0.data(), s0.data(), qa.data(),
               qb.data(), &vmax_r);
    // the layer of each depth row, with the host's comparisons on the host's z
    std::vector<KRow> rows(g.nz + 6);
    for (int k = -2; k <= g.nz + 3; k++) {
        const float zs = swpc_i2x(k, zbeg, sg.dz);
        KRow r = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0};
        if (zs < depth[0] && !(zs < 0.0f)) {   // seawater, lam = 1.0 * vp * vp (m_vmodel_lhm.f90:123-133)
            const float vp1 = 1.0f * swpc_seawater_vel(zs, munk_profile);
            r = {1.0f, 1.0f * vp1 * vp1, 0.0f, 1000000.0f, 1000000.0f, 3};
        }
        if (!(zs < depth[0])) {
            for (int l = 0; l < nlayer; l++)
                if (zs >= depth[l]) {
                    r = {r0[l], p0[l], s0[l], qa[l], qb[l], (p0[l] > 0 && s0[l] > 0) ? 1 : 2};
                }
        }
        rows[k + 2] = r;
    }
    KRow *d_rows = nullptr;
    CK(cudaMalloc((void **)&d_rows, rows.size() * sizeof(KRow)));
    int rc = cuda_check(c, cudaMemcpyAsync(d_rows, rows.data(), rows.size() * sizeof(KRow), cudaMemcpyHostToDevice,
                                           c->stream), "cudaMemcpyAsync");
    if (!rc && xi) rc = device_pointer(xi) ? copy_box_from_device(c, c->med[8], xi, ld_k, ld_i)
                                           : copy_box(c, c->med[8], xi, nullptr, ld_k, ld_i);
    if (!rc) {
        vmodel_kernel<<<kGrid, kBlock, 0, c->stream>>>(g, d_rows, xi ? 1 : 0, vcut, vmax_r, rhomin, c->med[8],
                                                        c->med[1], c->med[2], c->med[3], c->med[4]);
        rc = cuda_check(c, cudaGetLastError(), "vmodel_kernel");
    }
    if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    cudaFree(d_rows);
    if (!rc) c->vmodel_ready = true;
    return rc;
}

extern "C" int swpc_vmodel_upload(swpc_ctx *c, const float *rho, const float *lam, const float *mu, const float *qp,
                                  const float *qs, int ld_k, int ld_i) {
    if (!c) return SWPC_ERR_ARG;
    if (c->kind != SWPC_KIND_3D) return set_err(c, SWPC_ERR_ARG, "the device medium setup is for the 3D code");
    RC(check_na_wide(c));
    if (!rho || !lam || !mu || !qp || !qs) return set_err(c, SWPC_ERR_ARG, "model array missing");
    CK(cudaSetDevice(c->device));
    drop_graph(c);
    c->medium_ready = false;
    c->vmodel_ready = false;
    RC(copy_box(c, c->med[8], rho, nullptr, ld_k, ld_i));
    RC(copy_box(c, c->med[1], lam, nullptr, ld_k, ld_i));
    RC(copy_box(c, c->med[2], mu, nullptr, ld_k, ld_i));
    RC(copy_box(c, c->med[3], qp, nullptr, ld_k, ld_i));
    RC(copy_box(c, c->med[4], qs, nullptr, ld_k, ld_i));
    c->vmodel_ready = true;
    return SWPC_OK;
}

// Moduli of per-cell velocities over the memory box, in the expression order
// of vmodel_lhm (m_vmodel_lhm.f90:146-148): mu = rho vs vs, lam = rho (vp vp -
// 2 vs vs).  On entry lam holds vp and mu holds vs.
__global__ void moduli_kernel(Geo g, const float *__restrict__ rho, float *lam, float *mu) {
    const int nkb = g.nz + 6, nib = g.nx + 6;
    const long long n = (long long)nkb * nib * (g.ny + 6);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % nkb) - 2;
        const long long col = t / nkb;
        const int i = (int)(col % nib) - 2, j = (int)(col / nib) - 2;
        const long long e = cell_index(g, k, i, j);
        const float r = rho[e], vp = lam[e], vs = mu[e];
        mu[e] = r * vs * vs;
        lam[e] = r * (vp * vp - 2.0f * vs * vs);
    }
}

extern "C" int swpc_vmodel_velocity_device(swpc_ctx *c, const float *vp, const float *vs, const float *rho,
                                           const float *qp, const float *qs, int ld_k, int ld_i) {
    if (!c) return SWPC_ERR_ARG;
    if (c->kind != SWPC_KIND_3D) return set_err(c, SWPC_ERR_ARG, "the device medium setup is for the 3D code");
    RC(check_na_wide(c));
    if (!vp || !vs || !rho || !qp || !qs) return set_err(c, SWPC_ERR_ARG, "model array missing");
    for (const float *p : {vp, vs, rho, qp, qs})
        if (!device_pointer(p)) return set_err(c, SWPC_ERR_ARG, "swpc_vmodel_velocity_device takes device arrays");
    if (ld_k < c->g.nz + 6 || ld_i < c->g.nx + 6) return set_err(c, SWPC_ERR_ARG, "leading extents smaller than the memory box");
    CK(cudaSetDevice(c->device));
    drop_graph(c);
    c->medium_ready = false;
    c->vmodel_ready = false;
    RC(copy_box_from_device(c, c->med[8], rho, ld_k, ld_i));
    RC(copy_box_from_device(c, c->med[1], vp, ld_k, ld_i));
    RC(copy_box_from_device(c, c->med[2], vs, ld_k, ld_i));
    RC(copy_box_from_device(c, c->med[3], qp, ld_k, ld_i));
    RC(copy_box_from_device(c, c->med[4], qs, ld_k, ld_i));
    moduli_kernel<<<148 * 8, 256, 0, c->stream>>>(c->g, c->med[8], c->med[1], c->med[2]);
    CK(cudaGetLastError());
    c->vmodel_ready = true;
    return SWPC_OK;
}

extern "C" int swpc_medium_setup_device(swpc_ctx *c, float fq_min, float fq_max, float fq_ref, float *ts,
                                        float *scal, int *kfs, int *kob, int *kfs_top, int *kfs_bot, int *kob_top,
                                        int *kob_bot, int *kbeg_a, int ld_i2) {
    return swpc_medium_setup_device_opt(c, fq_min, fq_max, fq_ref, ts, scal, kfs, kob, kfs_top, kfs_bot, kob_top,
                                        kob_bot, kbeg_a, ld_i2, 0);
}

extern "C" int swpc_medium_setup_device_opt(swpc_ctx *c, float fq_min, float fq_max, float fq_ref, float *ts,
                                            float *scal, int *kfs, int *kob, int *kfs_top, int *kfs_bot,
                                            int *kob_top, int *kob_bot, int *kbeg_a, int ld_i2, int stabilize_pml) {
    if (!c) return SWPC_ERR_ARG;
    if (c->kind != SWPC_KIND_3D) return set_err(c, SWPC_ERR_ARG, "the device medium setup is for the 3D code");
    if (!c->vmodel_ready) return set_err(c, SWPC_ERR_STATE, "no model on the device (swpc_vmodel_lhm_device or swpc_vmodel_upload)");
    if (!ts || !scal) return set_err(c, SWPC_ERR_ARG, "ts and scal are required");
    const Geo &g = c->g;
    const int nx = g.nx, ny = g.ny, na = c->d.na, nm = c->d.nm;
    const bool maps = kfs || kob || kfs_top || kfs_bot || kob_top || kob_bot || kbeg_a;
    if (maps && ld_i2 < nx + 6) return set_err(c, SWPC_ERR_ARG, "ld_i2 smaller than the memory box");
    if (2 * na >= nx || 2 * na >= ny || na >= g.nz) return set_err(c, SWPC_ERR_ARG, "absorber wider than the grid");
    CK(cudaSetDevice(c->device));
    drop_graph(c);
    c->medium_ready = false;
    float *rho = c->med[8], *lam = c->med[1], *mu = c->med[2], *taup = c->med[3], *taus = c->med[4];
    homogenise_kernel<<<kGrid, kBlock, 0, c->stream>>>(g, na, rho, lam, mu, taup, taus);
    CK(cudaGetLastError());
    float zeta = 0.0f;
    swpc_visco_setup(nm, fq_min, fq_max, ts, &zeta);
    float ccr = 0.0f, cci = 0.0f;
    if (nm > 0) relaxed_cc(nm, ts, fq_ref, &ccr, &cci);
    tau_relax_kernel<<<kGrid, kBlock, 0, c->stream>>>(g, (float)nm * zeta, nm > 0 ? 1 : 0, ccr, cci, lam, mu, taup,
                                                       taus);
    CK(cudaGetLastError());
    const long long ncol = (long long)g.Ip * g.Jp;
    CK(cudaMemsetAsync(c->kfs, 0, ncol * sizeof(int), c->stream));
    CK(cudaMemsetAsync(c->kob, 0, ncol * sizeof(int), c->stream));
    CK(cudaMemsetAsync(c->band, 0, ncol * sizeof(int4), c->stream));
    surface_kernel<<<kGrid, kBlock, 0, c->stream>>>(g, lam, mu, c->kfs, c->kob);
    CK(cudaGetLastError());
    band_kernel<<<kGrid, kBlock, 0, c->stream>>>(g, c->kfs, c->kob, c->band);
    CK(cudaGetLastError());
    // the two words of the velocity range reduction
    unsigned *d_mm = nullptr;
    CK(cudaMalloc((void **)&d_mm, 2 * sizeof(unsigned)));
    const unsigned init[2] = {0u, 0xffffffffu};
    unsigned mm[2] = {0u, 0xffffffffu};
    int rc = cuda_check(c, cudaMemcpyAsync(d_mm, init, sizeof(init), cudaMemcpyHostToDevice, c->stream),
                        "cudaMemcpyAsync");
    if (!rc) {
        vminmax_kernel<<<kGrid, kBlock, 0, c->stream>>>(g, rho, lam, mu, c->kfs, d_mm);
        rc = cuda_check(c, cudaGetLastError(), "vminmax_kernel");
    }
    if (!rc) rc = cuda_check(c, cudaMemcpyAsync(mm, d_mm, sizeof(mm), cudaMemcpyDeviceToHost, c->stream),
                             "cudaMemcpyAsync");
    if (!rc && stabilize_pml) {
        // stabilize_pml (m_medium.f90:219-222) with the velocity maximum of velocity_minmax
        rc = cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
        float vmx = -1.0f;
        if (mm[0] != 0u) {
            const unsigned b = mm[0] - 1u;
            memcpy(&vmx, &b, sizeof(float));
        }
        if (!rc) {
            stabilize_kernel<<<kGrid, kBlock, 0, c->stream>>>(g, na, vmx, rho, lam, mu, taup, taus);
            rc = cuda_check(c, cudaGetLastError(), "stabilize_kernel");
        }
    }
    if (!rc) rc = average_medium(c);
    if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    cudaFree(d_mm);
    if (rc) return rc;
    float vmax1 = -1.0f, vmin1 = 1e30f;
    if (mm[0] != 0u) {
        const unsigned b = mm[0] - 1u;
        memcpy(&vmax1, &b, sizeof(float));
    }
    if (mm[1] != 0xffffffffu) memcpy(&vmin1, &mm[1], sizeof(float));
    scal[0] = zeta;
    scal[1] = vmin1;
    scal[2] = vmax1;
    // the absorber start map (m_global.f90:336-345) on the host, as the upload keeps it
    const swpc_grid sg = grid_of(c, 0.0f);
    std::vector<int> ka((size_t)ncol, 0);
    swpc_kbeg_a(&sg, ka.data());
    c->h_kbeg_a = ka;
    if (maps) {
        std::vector<int> hf(ncol), ho(ncol);
        std::vector<int4> hb(ncol);
        CK(cudaMemcpy(hf.data(), c->kfs, ncol * sizeof(int), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(ho.data(), c->kob, ncol * sizeof(int), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(hb.data(), c->band, ncol * sizeof(int4), cudaMemcpyDeviceToHost));
        for (int j = -2; j <= ny + 3; j++)
            for (int i = -2; i <= nx + 3; i++) {
                const long long cc = col_index(g, i, j), h = (long long)(j + 2) * ld_i2 + (i + 2);
                if (kfs) kfs[h] = hf[cc];
                if (kob) kob[h] = ho[cc];
                if (kfs_top) kfs_top[h] = hb[cc].x;
                if (kfs_bot) kfs_bot[h] = hb[cc].y;
                if (kob_top) kob_top[h] = hb[cc].z;
                if (kob_bot) kob_bot[h] = hb[cc].w;
                if (kbeg_a) kbeg_a[h] = ka[cc];
            }
    }
    c->vmodel_ready = false;
    c->medium_ready = true;
    return SWPC_OK;
}
