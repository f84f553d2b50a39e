// swpc_host.cpp -- host setup routines (include/swpc_setup.h).
//
// Single-precision restatements of the reference's setup arithmetic; the
// per-cell loops are OpenMP-parallel (every cell is independent, so results
// do not depend on the thread count).  Compiled with -ffp-contract=off so
// that each operation rounds as the reference's expression spells it.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/swpc_gpu.h"
#include "../../include/swpc_setup.h"
#include "swpc_host.h"

namespace {

const double kPi = 3.141592653589793238462643383279502884;   // m_std.f90:14
const float kEps = 1.1920929e-07f;                             // epsilon(1.0)

struct Box {
    long nk, ni, nj;
    int nx, ny, nz;
    long idx(int k, int i, int j) const { return ((long)(j + 2) * ni + (i + 2)) * nk + (k + 2); }
    long col(int i, int j) const { return (long)(j + 2) * ni + (i + 2); }
};

Box make_box(const swpc_grid *g) {
    Box b;
    b.nx = g->nx; b.ny = g->ny; b.nz = g->nz;
    b.nk = g->nz + 6; b.ni = g->nx + 6; b.nj = g->ny > 1 ? g->ny + 6 : 1;
    return b;
}

}  // namespace

namespace swpc {

void relaxed_cc(int nm, const float *ts, float fq_ref, float *ccr_out, float *cci_out) {
    const float omega = (float)(2 * kPi * (double)fq_ref);
    float ccr = 0.0f, cci = 0.0f;
    for (int m = 0; m < nm; m++) {
        const double a = (double)omega * (double)ts[m];
        const double den = 1.0 + a * a;
        ccr = ccr + (float)(-(a * a) / den);
        cci = cci + (float)(a / den);
    }
    *ccr_out = ccr / nm;
    *cci_out = cci / nm;
}

void lhm_layers(const swpc_grid *g, int nlayer, const float *depth, const float *rho0_in, const float *vp0_in,
                const float *vs0_in, const float *qp0_in, const float *qs0_in, float vcut, float *r0, float *p0,
                float *s0, float *qa, float *qb, float *vmax_r) {
    for (int l = 0; l < nlayer; l++) {
        r0[l] = rho0_in[l]; p0[l] = vp0_in[l]; s0[l] = vs0_in[l]; qa[l] = qp0_in[l]; qb[l] = qs0_in[l];
    }
    // velocity cut-off (m_vmodel_lhm.f90:93-101)
    for (int l = nlayer - 2; l >= 0; l--)
        if ((p0[l] < vcut || s0[l] < vcut) && (p0[l] > 0 && s0[l] > 0)) {
            p0[l] = p0[l + 1]; s0[l] = s0[l + 1]; r0[l] = r0[l + 1]; qa[l] = qa[l + 1]; qb[l] = qb[l + 1];
        }
    // velocity bounds of lhm_rmed (m_vmodel_lhm_rmed.f90:95-98)
    const float dh = 1.0f / sqrtf(1.0f / (g->dx * g->dx) + 1.0f / (g->dy * g->dy) + 1.0f / (g->dz * g->dz));
    *vmax_r = 6.0f / 7.0f * dh / g->dt;
}

float momentrate(float t, int stftype, float ts, float tr) {
    switch (stftype) {
    case SWPC_STF_BOXCAR:
        if (ts <= t && t <= ts + tr) return 1.0f / tr;
        return 0.0f;
    case SWPC_STF_TRIANGLE:
        if (ts <= t && t <= ts + tr / 2) return 4 * (t - ts) / (tr * tr);
        if (ts + tr / 2 < t && t <= ts + tr) return -4 * (t - ts - tr) / (tr * tr);
        return 0.0f;
    case SWPC_STF_HERRMANN: {
        const float t1 = ts + tr / 4;
        const float t2 = ts + 3 * tr / 4;
        if (ts <= t && t < t1) {
            const float a = t - ts;
            return 16 * (a * a) / (tr * tr * tr);
        }
        if (t1 <= t && t < t2) return -2 * (8 * (t * t + tr * ts + ts * ts - t * tr - 2 * t * ts) + tr * tr) / (tr * tr * tr);
        if (t2 <= t && t <= ts + tr) {
            const float a = ts + tr - t;
            return 16 * (a * a) / (tr * tr * tr);
        }
        return 0.0f;
    }
    case SWPC_STF_COSINE:
        if (ts <= t && t <= ts + tr) return (float)((1.0 - cos(2 * kPi * (double)(t - ts) / (double)tr)) / (double)tr);
        return 0.0f;
    case SWPC_STF_TEXP:
        if (ts <= t) {
            const float tt = t - ts;
            const double tp = 2 * kPi;
            return (float)(tp * tp * (double)tt / (double)(tr * tr) * exp(-2 * kPi * (double)tt / (double)tr));
        }
        return 0.0f;
    default:   // kupper (m_fdtool.f90:339-353)
        if (ts <= t && t <= ts + tr) {
            const double s = sin(kPi * (double)(t - ts) / (double)tr);
            return (float)(3.0 * kPi * (s * s * s) / (double)(4.0f * tr));
        }
        return 0.0f;
    }
}

}  // namespace swpc

extern "C" {

int swpc_x2i(float x, float beg, float d) {
    volatile float t = (x - beg) / d;
    return (int)ceilf(t);
}

float swpc_i2x(int i, float beg, float d) {
    volatile float a = (float)i - 0.5f;
    volatile float b = a * d;
    return beg + b;
}

float swpc_momentrate(float t, int stftype, float ts, float tr) { return swpc::momentrate(t, stftype, ts, tr); }

void swpc_sdr2moment(float strike, float dip, float rake, float *m6) {
    const float d2r = (float)(kPi / 180.0);
    const float sind = sinf(dip * d2r), cosd = cosf(dip * d2r);
    const float sin2d = sinf((2 * dip) * d2r), cos2d = cosf((2 * dip) * d2r);
    const float sinl = sinf(rake * d2r), cosl = cosf(rake * d2r);
    const float sf = sinf(strike * d2r), cf = cosf(strike * d2r);
    const float sin2f = sinf((2 * strike) * d2r), cos2f = cosf((2 * strike) * d2r);
    m6[0] = -(sind * cosl * sin2f + sin2d * sinl * sf * sf);   // mxx
    m6[1] = (sind * cosl * sin2f - sin2d * sinl * cf * cf);    // myy
    m6[2] = (sin2d * sinl);                                    // mzz
    m6[3] = -(cosd * cosl * sf - cos2d * sinl * cf);           // myz
    m6[4] = -(cosd * cosl * cf + cos2d * sinl * sf);           // mxz
    m6[5] = (sind * cosl * cos2f + sin2d * sinl * sin2f / 2);  // mxy
}

void swpc_visco_setup(int nm, float fq_min, float fq_max, float *ts, float *zeta) {
    // visco_set_relaxtime (m_fdtool.f90:691-727)
    const float oa = (float)(2 * kPi * (double)fq_min);
    const float ob = (float)(2 * kPi * (double)fq_max);
    if (nm == 1) {
        ts[0] = 1.0f / sqrtf(oa * ob);
    } else if (nm > 1) {
        for (int m = 0; m < nm; m++) {
            const double p = pow((double)(ob / oa), (double)m / (double)(nm - 1));
            ts[m] = 1.0f / (float)((double)oa * p);
        }
    }
    // visco_constq_zeta (m_fdtool.f90:756-812)
    if (nm == 0) { *zeta = 0.0f; return; }
    float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f;
    std::vector<float> i0(nm), i1(nm);
    for (int m = 0; m < nm; m++) {
        const float t = ts[m];
        i0[m] = (logf(1.0f + (ob * ob) * (t * t)) - logf(1.0f + (oa * oa) * (t * t))) / (2 * t);
        const float pb = atanf(ob * t) - ob * t / (1 + (ob * ob) * (t * t));
        const float pa = atanf(oa * t) - oa * t / (1 + (oa * oa) * (t * t));
        i1[m] = (pb - pa) / (2 * t);
    }
    for (int m = 0; m < nm; m++) s0 += i0[m];
    for (int m = 0; m < nm; m++) s1 += i1[m];
    for (int m = 0; m < nm - 1; m++)
        for (int q = m + 1; q < nm; q++) {
            const float w1 = atanf(ob * ts[m]) / ts[m] - atanf(ob * ts[q]) / ts[q];
            const float w2 = atanf(oa * ts[m]) / ts[m] - atanf(oa * ts[q]) / ts[q];
            s2 = s2 + ts[m] * ts[q] / (ts[q] * ts[q] - ts[m] * ts[m]) * (w1 - w2);
        }
    *zeta = s0 / (s1 + 2 * s2);
}

void swpc_kbeg_a(const swpc_grid *g, int *kbeg_a) {
    const Box b = make_box(g);
    const int jlo = g->ny > 1 ? -2 : 1, jhi = g->ny > 1 ? g->ny + 3 : 1;
    for (int j = jlo; j <= jhi; j++)
        for (int i = -2; i <= g->nx + 3; i++) {
            const bool side = i <= g->na || g->nx - g->na + 1 <= i ||
                              (g->ny > 1 && (j <= g->na || g->ny - g->na + 1 <= j));
            const long c = g->ny > 1 ? b.col(i, j) : (long)(i + 2);
            kbeg_a[c] = side ? 1 : g->nz - g->na + 1;
        }
}

static void vcheck(float &vp, float &vs, float &rho, float xi, float vmin, float vmax, float rhomin) {
    // m_fdtool.f90:15-48
    float gamma = vp / vs;
    if (gamma < kEps) gamma = sqrtf(3.0f);
    if (vp > vmax || vs > vmax) {
        const float xi2 = (1 + xi) * vmax / vp - 1;
        vp = vmax;
        vs = vmax / gamma;
        rho = rho * (1 + 0.8f * xi2) / (1 + 0.8f * xi);
    }
    if (vp < vmin || vs < vmin) {
        vs = vmin;
        vp = vmin * gamma;
    }
    if (rho < rhomin) rho = rhomin;
}

// seawater__vel (src/shared/m_seawater.f90:19-49): Munk's profile (eps = 0.00737) of depth z [km], or 1.5 km/s
// without it, evaluated in double as the reference does
float swpc_seawater_vel(float z, int munk_profile) {
    const double eps = munk_profile ? 0.00737 : 0.0;
    const double zc = 1300.0;
    const double zb = 2 * ((double)z * 1000. - zc) / zc;
    return (float)(1.5 * (1.0 + eps * (zb - 1.0 + std::exp(-zb))));
}

int swpc_vmodel_lhm(const swpc_grid *g, int nlayer, const float *depth, const float *rho0_in, const float *vp0_in,
                    const float *vs0_in, const float *qp0_in, const float *qs0_in, float vcut, const float *xi,
                    float rhomin, float *rho, float *lam, float *mu, float *qp, float *qs) {
    return swpc_vmodel_lhm_opt(g, nlayer, depth, rho0_in, vp0_in, vs0_in, qp0_in, qs0_in, vcut, xi, rhomin, rho, lam,
                               mu, qp, qs, 0);
}

int swpc_vmodel_lhm_opt(const swpc_grid *g, int nlayer, const float *depth, const float *rho0_in,
                        const float *vp0_in, const float *vs0_in, const float *qp0_in, const float *qs0_in, float vcut,
                        const float *xi, float rhomin, float *rho, float *lam, float *mu, float *qp, float *qs,
                        int munk_profile) {
    if (nlayer < 1) return SWPC_ERR_ARG;
    std::vector<float> r0(nlayer), p0(nlayer), s0(nlayer), qa(nlayer), qb(nlayer);
    float vmax_r;
    swpc::lhm_layers(g, nlayer, depth, rho0_in, vp0_in, vs0_in, qp0_in, qs0_in, vcut, r0.data(), p0.data(),
                     s0.data(), qa.data(), qb.data(), &vmax_r);
    const Box b = make_box(g);
    const int jlo = g->ny > 1 ? -2 : 0, jhi = g->ny > 1 ? g->ny + 3 : 0;
#pragma omp parallel for schedule(static)
    for (int k = -2; k <= g->nz + 3; k++) {
        const float zs = swpc_i2x(k, g->zbeg, g->dz);
        for (int j = jlo; j <= jhi; j++)
            for (int i = -2; i <= g->nx + 3; i++) {
                const long e = g->ny > 1 ? b.idx(k, i, j) : ((long)(i + 2) * b.nk + (k + 2));
                if (zs < depth[0]) {
                    if (zs < 0.0f) {   // air column (m_vmodel_lhm.f90:110-121)
                        rho[e] = 0.001f; mu[e] = 0.0f; lam[e] = 0.0f; qp[e] = 10.0f; qs[e] = 10.0f;
                    } else {           // seawater above depth(1) (:123-133)
                        const float vp1 = 1.0f * swpc_seawater_vel(zs, munk_profile);
                        rho[e] = 1.0f; mu[e] = 0.0f; lam[e] = 1.0f * vp1 * vp1; qp[e] = 1000000.0f; qs[e] = 1000000.0f;
                    }
                    continue;
                }
                float rho1 = 0, vp1 = 0, vs1 = 0, qp1 = 0, qs1 = 0;
                for (int l = 0; l < nlayer; l++) {
                    if (zs >= depth[l]) {
                        if (xi) {
                            const float x = xi[e];
                            rho1 = r0[l] * (1 + 0.8f * x);
                            vp1 = 1.0f * p0[l] * (1 + x);
                            vs1 = 1.0f * s0[l] * (1 + x);
                            if (p0[l] > 0 && s0[l] > 0) vcheck(vp1, vs1, rho1, x, vcut, vmax_r, rhomin);
                        } else {
                            rho1 = r0[l]; vp1 = 1.0f * p0[l]; vs1 = 1.0f * s0[l];
                        }
                        qp1 = qa[l]; qs1 = qb[l];
                    }
                }
                rho[e] = rho1;
                mu[e] = rho1 * vs1 * vs1;
                lam[e] = rho1 * (vp1 * vp1 - 2 * vs1 * vs1);
                qp[e] = qp1;
                qs[e] = qs1;
            }
    }
    return SWPC_OK;
}

int swpc_setup_medium(const swpc_grid *g, float fq_min, float fq_max, float fq_ref, float *rho, float *lam, float *mu,
                      const float *qp, const float *qs, float *taup, float *taus, float *bx, float *by, float *bz,
                      float *muyz, float *muxz, float *muxy, int *kfs, int *kob, int *kfs_top, int *kfs_bot,
                      int *kob_top, int *kob_bot, float *ts, float *scal) {
    return swpc_setup_medium_opt(g, fq_min, fq_max, fq_ref, rho, lam, mu, qp, qs, taup, taus, bx, by, bz, muyz, muxz,
                                 muxy, kfs, kob, kfs_top, kfs_bot, kob_top, kob_bot, ts, scal, 0);
}

// stabilize_absorber (m_medium.f90:276-340): in each column around the
// absorber, thin low-velocity layers (at most 20 cells) take the medium of
// the cell above, then shear velocities below 0.4 vmax are raised to it
// with vp = sqrt(3) vs
static void stabilize_absorber(const swpc_grid *g, const Box &b, float *rho, float *lam, float *mu, float *taup,
                               float *taus, float vmax) {
    const float vmin_pml = vmax * 0.4f;
    const int lv_thick = 20;
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    std::vector<int> ka((size_t)b.ni * b.nj);
    swpc_kbeg_a(g, ka.data());
    auto kstart = [&](int i, int j) {
        int m = 1 << 30;
        for (int jj = j - 2; jj <= j + 2; jj++)
            for (int ii = i - 2; ii <= i + 2; ii++) m = std::min(m, ka[b.col(ii, jj)]);
        return m;
    };
#pragma omp parallel for schedule(static)
    for (int j = 0; j <= ny + 1; j++)
        for (int i = 0; i <= nx + 1; i++) {
            int k = kstart(i, j);
            while (k <= nz) {
                const long e = b.idx(k, i, j), u = b.idx(k - 1, i, j);
                if (lam[e] < lam[u] || mu[e] < mu[u]) {
                    int k2 = k + 1;
                    for (; k2 <= nz; k2++) {
                        const long e2 = b.idx(k2, i, j), u2 = b.idx(k2 - 1, i, j);
                        if (lam[e2] > lam[u2] || mu[e2] > mu[u2]) break;
                    }
                    if (k2 - k <= lv_thick) {
                        rho[e] = rho[u]; lam[e] = lam[u]; mu[e] = mu[u]; taup[e] = taup[u]; taus[e] = taus[u];
                        k = k2 - 1;
                    }
                }
                k++;
            }
        }
#pragma omp parallel for schedule(static)
    for (int j = 0; j <= ny + 1; j++)
        for (int i = 0; i <= nx + 1; i++)
            for (int k = kstart(i, j); k <= nz; k++) {
                const long e = b.idx(k, i, j);
                float vp = sqrtf((lam[e] + 2 * mu[e]) / rho[e]);
                float vs = sqrtf(mu[e] / rho[e]);
                if (vs < kEps) continue;   // ocean and air
                const float gamma = sqrtf(3.0f);
                if (vs < vmin_pml) {
                    vs = vmin_pml;
                    vp = vs * gamma;
                    lam[e] = rho[e] * (vp * vp - 2 * (vs * vs));
                    mu[e] = rho[e] * (vs * vs);
                }
            }
}

int swpc_setup_medium_opt(const swpc_grid *g, float fq_min, float fq_max, float fq_ref, float *rho, float *lam,
                          float *mu, const float *qp, const float *qs, float *taup, float *taus, float *bx, float *by,
                          float *bz, float *muyz, float *muxz, float *muxy, int *kfs, int *kob, int *kfs_top,
                          int *kfs_bot, int *kob_top, int *kob_bot, float *ts, float *scal, int stabilize_pml) {
    if (g->ny <= 1) return SWPC_ERR_ARG;
    const Box b = make_box(g);
    const int nx = g->nx, ny = g->ny, nz = g->nz, na = g->na, nm = g->nm;
    const long n3 = b.nk * b.ni * b.nj;
    memcpy(taup, qp, sizeof(float) * n3);
    memcpy(taus, qs, sizeof(float) * n3);
    auto copy_cell = [&](long d, long s) {
        rho[d] = rho[s]; lam[d] = lam[s]; mu[d] = mu[s]; taup[d] = taup[s]; taus[d] = taus[s];
    };
    // absorber homogenisation (m_medium.f90:124-190), in the reference order
#pragma omp parallel for schedule(static)
    for (int j = -2; j <= ny + 3; j++)
        for (int i = -2; i <= na; i++)
            for (int k = -2; k <= nz + 3; k++) copy_cell(b.idx(k, i, j), b.idx(k, na + 1, j));
#pragma omp parallel for schedule(static)
    for (int j = -2; j <= ny + 3; j++)
        for (int i = nx - na + 1; i <= nx + 3; i++)
            for (int k = -2; k <= nz + 3; k++) copy_cell(b.idx(k, i, j), b.idx(k, nx - na, j));
    for (int j = -2; j <= na; j++)
#pragma omp parallel for schedule(static)
        for (int i = -2; i <= nx + 3; i++)
            for (int k = -2; k <= nz + 3; k++) copy_cell(b.idx(k, i, j), b.idx(k, i, na + 1));
    for (int j = ny - na + 1; j <= ny + 3; j++)
#pragma omp parallel for schedule(static)
        for (int i = -2; i <= nx + 3; i++)
            for (int k = -2; k <= nz + 3; k++) copy_cell(b.idx(k, i, j), b.idx(k, i, ny - na));
#pragma omp parallel for schedule(static)
    for (int j = -2; j <= ny + 3; j++)
        for (int i = -2; i <= nx + 3; i++)
            for (int k = nz - na + 1; k <= nz + 3; k++) copy_cell(b.idx(k, i, j), b.idx(nz - na, i, j));
    // tau method (m_medium.f90:193-207)
    float zeta = 0.0f;
    swpc_visco_setup(nm, fq_min, fq_max, ts, &zeta);
#pragma omp parallel for schedule(static)
    for (long e = 0; e < n3; e++) {
        taup[e] = nm * zeta / taup[e];
        taus[e] = nm * zeta / taus[e];
    }
    // relaxed_medium (m_medium.f90:234-274): chi = 1 / Re(1/sqrt(1 - cc*tau)),
    // cc = mean over m of (i w ts)/(1 - i w ts)
    if (nm > 0) {
        float ccr, cci;
        swpc::relaxed_cc(nm, ts, fq_ref, &ccr, &cci);
#pragma omp parallel for schedule(static)
        for (long e = 0; e < n3; e++) {
            const float rb2 = mu[e];
            const float ra2 = lam[e] + 2 * mu[e];
            float chi[2];
            const float tt[2] = {taus[e], taup[e]};
            for (int q = 0; q < 2; q++) {
                const float zr = 1.0f - ccr * tt[q];
                const float zi = 0.0f - cci * tt[q];
                const float wr = sqrtf(0.5f * (hypotf(zr, zi) + zr));
                const float wi = 0.5f * (zi / wr);
                chi[q] = 1.0f / (wr / (wr * wr + wi * wi));
            }
            mu[e] = rb2 / (chi[0] * chi[0]);
            lam[e] = ra2 / (chi[1] * chi[1]) - 2 * mu[e];
        }
    }
    // surface_detection (m_medium.f90:342-397)
    for (long c = 0; c < b.ni * b.nj; c++) { kfs[c] = 0; kob[c] = 0; }
#pragma omp parallel for schedule(static)
    for (int j = 0; j <= ny + 2; j++)
        for (int i = 0; i <= nx + 2; i++) {
            int f = 0, o = 0;
            for (int k = 1; k <= nz - 1; k++) {
                if (fabsf(mu[b.idx(k, i, j)]) < kEps && fabsf(mu[b.idx(k + 1, i, j)]) > kEps) o = k;
                if (fabsf(lam[b.idx(k, i, j)]) < kEps && fabsf(lam[b.idx(k + 1, i, j)]) > kEps) f = k;
            }
            kfs[b.col(i, j)] = f;
            kob[b.col(i, j)] = o;
        }
    for (long c = 0; c < b.ni * b.nj; c++) { kfs_top[c] = 0; kfs_bot[c] = 0; kob_top[c] = 0; kob_bot[c] = 0; }
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
            int fmn = 1 << 30, fmx = -(1 << 30), omn = 1 << 30, omx = -(1 << 30);
            for (int jj = j - 2; jj <= j + 3; jj++)
                for (int ii = i - 2; ii <= i + 3; ii++) {
                    const int f = kfs[b.col(ii, jj)], o = kob[b.col(ii, jj)];
                    fmn = std::min(fmn, f); fmx = std::max(fmx, f);
                    omn = std::min(omn, o); omx = std::max(omx, o);
                }
            kfs_top[b.col(i, j)] = std::max(fmn - 2, 1);
            kfs_bot[b.col(i, j)] = std::min(fmx + 2, nz);
            kob_top[b.col(i, j)] = std::max(omn - 2, 1);
            kob_bot[b.col(i, j)] = std::min(omx + 2, nz);
        }
    // velocity_minmax (m_medium.f90:399-430)
    float vmax1 = -1.0f, vmin1 = 1e30f;
    for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++)
            for (int k = kfs[b.col(i, j)] + 1; k <= nz; k++) {
                const long e = b.idx(k, i, j);
                const float vp = sqrtf((lam[e] + 2 * mu[e]) / rho[e]);
                const float vs = sqrtf(mu[e] / rho[e]);
                vmax1 = std::max(vmax1, vp);
                if (vs < kEps) continue;
                vmin1 = std::min(vmin1, vs);
            }
    // stabilize_pml (m_medium.f90:219-222)
    if (stabilize_pml) stabilize_absorber(g, b, rho, lam, mu, taup, taus, vmax1);
    // averaged_medium (m_medium.f90:432-465)
    memset(bx, 0, sizeof(float) * n3); memset(by, 0, sizeof(float) * n3); memset(bz, 0, sizeof(float) * n3);
    memset(muyz, 0, sizeof(float) * n3); memset(muxz, 0, sizeof(float) * n3); memset(muxy, 0, sizeof(float) * n3);
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++)
            for (int k = 1; k <= nz; k++) {
                const long e = b.idx(k, i, j);
                bx[e] = 2.0f / (rho[e] + rho[b.idx(k, i + 1, j)]);
                by[e] = 2.0f / (rho[e] + rho[b.idx(k, i, j + 1)]);
                bz[e] = 2.0f / (rho[e] + rho[b.idx(k + 1, i, j)]);
                const float nnn = mu[e], pnn = mu[b.idx(k + 1, i, j)], npn = mu[b.idx(k, i + 1, j)];
                const float ppn = mu[b.idx(k + 1, i + 1, j)], nnp = mu[b.idx(k, i, j + 1)];
                const float npp = mu[b.idx(k, i + 1, j + 1)], pnp = mu[b.idx(k + 1, i, j + 1)];
                muxz[e] = 4 * nnn * pnn * npn * ppn / (nnn * pnn * npn + nnn * pnn * ppn + nnn * npn * ppn + pnn * npn * ppn + kEps);
                muxy[e] = 4 * nnn * npn * nnp * npp / (nnn * npn * nnp + nnn * npn * npp + nnn * nnp * npp + npn * nnp * npp + kEps);
                muyz[e] = 4 * nnn * pnn * nnp * pnp / (nnn * pnn * nnp + nnn * pnn * pnp + nnn * nnp * pnp + pnn * nnp * pnp + kEps);
            }
    scal[0] = zeta;
    scal[1] = vmin1;
    scal[2] = vmax1;
    return SWPC_OK;
}

// visco_chi (m_fdtool.f90:730-753): cc = mean_m (1 - i w ts (1+tau)) / (1 - i w ts)
// with each term in complex DP and the running sum in complex SP;
// chi = 1 / Re(cc**(-0.5)) with the principal power taken in SP
static float visco_chi(int nm, const float *ts, float tau, float f) {
    const float omega = (float)(2 * kPi * (double)f);
    float ccr = 0.0f, cci = 0.0f;
    for (int m = 0; m < nm; m++) {
        const double a = (double)omega * (double)ts[m];
        const double ni = -(a * (1.0 + (double)tau)), di = -a;
        const double den = 1.0 * 1.0 + di * di;
        const double re = (1.0 * 1.0 + ni * di) / den;
        const double im = (ni * 1.0 - 1.0 * di) / den;
        ccr = (float)((double)ccr + re);
        cci = (float)((double)cci + im);
    }
    ccr = ccr / nm;
    cci = cci / nm;
    const float r = hypotf(ccr, cci);
    const float th = atan2f(cci, ccr);
    return 1.0f / (cosf(-0.5f * th) / sqrtf(r));
}

int swpc_setup_medium_2d(const swpc_grid *g, float fq_min, float fq_max, float fq_ref, float *rho, float *lam,
                         float *mu, const float *qp, const float *qs, float *taup, float *taus, int *kfs, int *kob,
                         int *kfs_top, int *kfs_bot, int *kob_top, int *kob_bot, float *ts, float *scal) {
    return swpc_setup_medium_2d_opt(g, fq_min, fq_max, fq_ref, rho, lam, mu, qp, qs, taup, taus, kfs, kob, kfs_top,
                                    kfs_bot, kob_top, kob_bot, ts, scal, 0);
}

int swpc_setup_medium_2d_opt(const swpc_grid *g, float fq_min, float fq_max, float fq_ref, float *rho, float *lam,
                             float *mu, const float *qp, const float *qs, float *taup, float *taus, int *kfs,
                             int *kob, int *kfs_top, int *kfs_bot, int *kob_top, int *kob_bot, float *ts,
                             float *scal, int stabilize_pml) {
    const int nx = g->nx, nz = g->nz, na = g->na, nm = g->nm;
    const long nk = nz + 6, ni = nx + 6;
    auto id = [&](int k, int i) { return (long)(i + 2) * nk + (k + 2); };
    memcpy(taup, qp, sizeof(float) * nk * ni);
    memcpy(taus, qs, sizeof(float) * nk * ni);
    auto cp = [&](long d, long s) {
        rho[d] = rho[s]; lam[d] = lam[s]; mu[d] = mu[s]; taup[d] = taup[s]; taus[d] = taus[s];
    };
    for (int i = -2; i <= na; i++)
        for (int k = -2; k <= nz + 3; k++) cp(id(k, i), id(k, na + 1));
    for (int i = nx - na + 1; i <= nx + 3; i++)
        for (int k = -2; k <= nz + 3; k++) cp(id(k, i), id(k, nx - na));
    for (int i = -2; i <= nx + 3; i++)
        for (int k = nz - na + 1; k <= nz + 3; k++) cp(id(k, i), id(nz - na, i));
    float zeta = 0.0f;
    swpc_visco_setup(nm, fq_min, fq_max, ts, &zeta);
    for (long e = 0; e < nk * ni; e++) {
        taup[e] = nm * zeta / taup[e];
        taus[e] = nm * zeta / taus[e];
    }
    if (nm > 0)
#pragma omp parallel for schedule(static)
        for (int i = -2; i <= nx + 3; i++) {
            // chi is a function of tau alone, and a column holds runs of equal
            // tau (layers): reuse the last value of each (same bits)
            float ls = 0.0f, lp = 0.0f, cs = 0.0f, cp = 0.0f;
            bool hs = false, hp = false;
            for (int k = -2; k <= nz + 3; k++) {
                const long e = id(k, i);
                const float rb2 = mu[e], ra2 = lam[e] + 2 * mu[e];
                if (!hs || memcmp(&ls, &taus[e], sizeof(float)) != 0) {
                    ls = taus[e]; cs = visco_chi(nm, ts, ls, fq_ref); hs = true;
                }
                const float cm = cs;
                mu[e] = rb2 / (cm * cm);
                if (!hp || memcmp(&lp, &taup[e], sizeof(float)) != 0) {
                    lp = taup[e]; cp = visco_chi(nm, ts, lp, fq_ref); hp = true;
                }
                const float cl = cp;
                lam[e] = ra2 / (cl * cl) - 2 * mu[e];
            }
        }
    for (int i = -2; i <= nx + 3; i++) { kfs[i + 2] = 0; kob[i + 2] = 0; kfs_top[i + 2] = kfs_bot[i + 2] = kob_top[i + 2] = kob_bot[i + 2] = 0; }
    for (int i = 0; i <= nx + 2; i++)
        for (int k = 1; k <= nz - 1; k++) {
            if (fabsf(mu[id(k, i)]) < kEps && fabsf(mu[id(k + 1, i)]) > kEps) kob[i + 2] = k;
            if (fabsf(lam[id(k, i)]) < kEps && fabsf(lam[id(k + 1, i)]) > kEps) kfs[i + 2] = k;
        }
    for (int i = 1; i <= nx; i++) {
        int fmn = 1 << 30, fmx = -(1 << 30), omn = 1 << 30, omx = -(1 << 30);
        for (int ii = i - 2; ii <= i + 3; ii++) {
            fmn = std::min(fmn, kfs[ii + 2]); fmx = std::max(fmx, kfs[ii + 2]);
            omn = std::min(omn, kob[ii + 2]); omx = std::max(omx, kob[ii + 2]);
        }
        kfs_top[i + 2] = std::max(fmn - 2, 1);
        kfs_bot[i + 2] = std::min(fmx + 2, nz);
        kob_top[i + 2] = std::max(omn - 2, 1);
        kob_bot[i + 2] = std::min(omx + 2, nz);
    }
    float vmax1 = -1.0f, vmin1 = 1e30f;
    for (int i = 1; i <= nx; i++)
        for (int k = kfs[i + 2] + 1; k <= nz; k++) {
            const long e = id(k, i);
            const float vp = sqrtf((lam[e] + 2 * mu[e]) / rho[e]);
            vmax1 = std::max(vmax1, vp);
            const float vs = sqrtf(mu[e] / rho[e]);
            if (vs < kEps) continue;
            vmin1 = std::min(vmin1, vs);
        }
    scal[0] = zeta; scal[1] = vmin1; scal[2] = vmax1;
    if (stabilize_pml) {
        // stabilize_absorber of the 2D codes (src/swpc_psv/m_medium.f90:309-365,
        // src/swpc_sh/m_medium.f90:301-357): unlike the 3D routine, a thin
        // low-velocity layer takes the medium above it over its whole thickness
        std::vector<int> ka((size_t)ni);
        swpc_kbeg_a(g, ka.data());
        const float vmin_pml = vmax1 * 0.4f;
        for (int i = 0; i <= nx + 1; i++) {
            int k0 = 1 << 30;
            for (int ii = i - 2; ii <= i + 2; ii++) k0 = std::min(k0, ka[ii + 2]);
            int k = k0;
            while (k <= nz) {
                if (lam[id(k, i)] < lam[id(k - 1, i)] || mu[id(k, i)] < mu[id(k - 1, i)]) {
                    int k2 = k + 1;
                    for (; k2 <= nz; k2++)
                        if (lam[id(k2, i)] > lam[id(k2 - 1, i)] || mu[id(k2, i)] > mu[id(k2 - 1, i)]) break;
                    if (k2 - k <= 20) {
                        const long u = id(k - 1, i);
                        for (int kk = k; kk <= k2 - 1; kk++) {
                            const long e = id(kk, i);
                            rho[e] = rho[u]; lam[e] = lam[u]; mu[e] = mu[u]; taup[e] = taup[u]; taus[e] = taus[u];
                        }
                        k = k2 - 1;
                    }
                }
                k++;
            }
            for (k = k0; k <= nz; k++) {
                const long e = id(k, i);
                float vp = sqrtf((lam[e] + 2 * mu[e]) / rho[e]);
                float vs = sqrtf(mu[e] / rho[e]);
                if (vs < kEps) continue;
                const float gamma = sqrtf(3.0f);
                if (vs < vmin_pml) {
                    vs = vmin_pml;
                    vp = vs * gamma;
                    lam[e] = rho[e] * (vp * vp - 2 * (vs * vs));
                    mu[e] = rho[e] * (vs * vs);
                }
            }
        }
    }
    return SWPC_OK;
}

static void damping_profile(float x, float H, float beg, float end, int na, float fcut, float dt, float *gp) {
    // m_absorb_p.f90:507-547 (pd = pa = 1, pb = 2, cp = 6)
    const float R0 = powf(10.0f, -(log10f((float)na) - 1) / log10f(2.0f) - 3.0f);
    const float d0 = -(1.0f / (2.0f * H)) * (1 + 1) * 6.0f * logf(R0);
    const float b0 = 7.0f;
    const float a0 = (float)(kPi * (double)fcut);
    float xx;
    if (x <= beg + H) xx = (beg + H) - x;
    else if (x >= end - H) xx = x - (end - H);
    else xx = 0.0f;
    const float r = fabsf(xx / H);
    const float d = d0 * r;
    const float a = a0 * (1.0f - r);
    const float bb = 1.0f + (b0 - 1.0f) * (r * r);
    const float h = dt / 2.0f;
    gp[0] = ((1.0f + h * a) / bb) / (1.0f + h * (a + d / bb));
    gp[1] = (-1.0f / bb) / (1.0f + h * (a + d / bb));
    gp[2] = (1.0f - h * (a + d / bb)) / (1.0f + h * (a + d / bb));
    gp[3] = (d / bb) / (1.0f + h * (a + d / bb));
}

void swpc_damping_profiles(const swpc_grid *g, float fcut, float *gxc, float *gxe, float *gyc, float *gye, float *gzc,
                           float *gze) {
    // absorb_p__setup (m_absorb_p.f90:79-93); xend = xbeg + nx*dx (m_global.f90:205-207)
    const float xend = g->xbeg + g->nx * g->dx, yend = g->ybeg + g->ny * g->dy, zend = g->zbeg + g->nz * g->dz;
    const float hx = g->na * g->dx, hy = g->na * g->dy, hz = g->na * g->dz;
    for (int i = 1; i <= g->nx; i++) {
        const float xc = swpc_i2x(i, g->xbeg, g->dx);
        damping_profile(xc, hx, g->xbeg, xend, g->na, fcut, g->dt, gxc + 4 * (i - 1));
        damping_profile(xc + g->dx / 2.0f, hx, g->xbeg, xend, g->na, fcut, g->dt, gxe + 4 * (i - 1));
    }
    if (gyc && gye)
        for (int j = 1; j <= g->ny; j++) {
            const float yc = swpc_i2x(j, g->ybeg, g->dy);
            damping_profile(yc, hy, g->ybeg, yend, g->na, fcut, g->dt, gyc + 4 * (j - 1));
            damping_profile(yc + g->dy / 2.0f, hy, g->ybeg, yend, g->na, fcut, g->dt, gye + 4 * (j - 1));
        }
    for (int k = 1; k <= g->nz; k++) {
        const float zc = swpc_i2x(k, g->zbeg, g->dz);
        damping_profile(zc, hz, g->zbeg, zend, g->na, fcut, g->dt, gzc + 4 * (k - 1));
        damping_profile(zc + g->dz / 2.0f, hz, g->zbeg, zend, g->na, fcut, g->dt, gze + 4 * (k - 1));
    }
}

// one axis of absorb_c__setup (src/swpc_3d/m_absorb_c.f90:48-85): inside
// the na cells at the low end (when `low`) and at the high end, exp(-alpha
// (1 - x/L)^2) with x the distance from the edge at the cell centre (c) and
// at its +d/2 boundary (b); 1 elsewhere
static void cerjan_axis(int n, int na, float d, bool low, float *gc, float *gb) {
    const float alpha = 0.09f;
    const float L = na * d;
    for (int i = 1; i <= n; i++) {
        float c = 1.0f, b = 1.0f;
        if (low && i <= na) {
            const float x = swpc_i2x(i, 0.0f, d);
            const float uc = 1.0f - x / L, ub = 1.0f - (x + d / 2) / L;
            c = expf(-alpha * (uc * uc));
            b = expf(-alpha * (ub * ub));
        } else if (i >= n - na + 1) {
            const float x = swpc_i2x(i, n * d, -d);
            const float uc = 1.0f - (x + d / 2) / L, ub = 1.0f - x / L;
            c = expf(-alpha * (uc * uc));
            b = expf(-alpha * (ub * ub));
        }
        gc[i - 1] = c;
        gb[i - 1] = b;
    }
}

void swpc_cerjan_profiles(const swpc_grid *g, float *gx_c, float *gx_b, float *gy_c, float *gy_b, float *gz_c,
                          float *gz_b) {
    cerjan_axis(g->nx, g->na, g->dx, true, gx_c, gx_b);
    if (gy_c && gy_b) cerjan_axis(g->ny, g->na, g->dy, true, gy_c, gy_b);
    // the free surface side (k <= na) is not damped (m_absorb_c.f90:73-80)
    cerjan_axis(g->nz, g->na, g->dz, false, gz_c, gz_b);
}

}  // extern "C"

// pw_setup (src/swpc_3d/m_source.f90:315-465): the plane-wave initial condition.  Every cell of the memory box
// whose wave speed reaches epsilon(1.0) gets the velocities and stresses of a plane P or S wave travelling along
// the direction (strike, dip), shaped by the moment-rate function over the rotated coordinate (zeta, length
// pw_zlen, front at depth pw_ztop); velocities are evaluated half a time step ahead on their staggered points.
// Single precision with the reference's expression order; fcut from the wave speed at the grid centre and depth
// pw_ztop (:443-462).
extern "C" int swpc_pw_setup(const swpc_grid *g, const float *rho, const float *lam, const float *mu, float pw_ztop,
                  float pw_zlen, int ps, float strike, float dip, float rake, int stftype, float *vx, float *vy,
                  float *vz, float *sxx, float *syy, float *szz, float *syz, float *sxz, float *sxy, float *fcut) {
    if (g->ny <= 1 || !(pw_zlen > 0.0f) || (ps != 0 && ps != 1)) return SWPC_ERR_ARG;
    const Box b = make_box(g);
    auto rad = [](float deg) { return (float)(kPi / 180.0 * (double)deg); };   // std__deg2rad (m_std.f90:132-139)
    const float tf = rad(strike), td = rad(dip), tl = rad(rake);
    const float sd = sinf(td), cd = cosf(td), sf = sinf(tf), cf = cosf(tf);
    const float sl = sinf(tl), cl = cosf(tl), c2d = cosf(2 * td), c2f = cosf(2 * tf);
    const float dx = g->dx, dy = g->dy, dz = g->dz;
    auto speed = [&](long e) {
        return ps == 0 ? sqrtf((lam[e] + 2 * mu[e]) / rho[e]) : sqrtf(mu[e] / rho[e]);
    };
#pragma omp parallel for schedule(static)
    for (int j = -2; j <= g->ny + 3; j++)
        for (int i = -2; i <= g->nx + 3; i++)
            for (int k = -2; k <= g->nz + 3; k++) {
                const long e = b.idx(k, i, j);
                const float v = speed(e);
                if (v < kEps) continue;
                const float x0 = g->xbeg + (i - 0.5f) * dx, y0 = g->ybeg + (j - 0.5f) * dy;
                const float z0 = g->zbeg + (k - 0.5f) * dz - pw_ztop;
                const float x1 = x0 + dx / 2.0f, y1 = y0 + dy / 2.0f, z1 = z0 + dz / 2.0f;
                const float ahead = g->dt / 2.0f * v;
                auto stf = [&](float x, float y, float z, float shift) {
                    const float zeta = sd * sf * x - sd * cf * y + cd * z;
                    return swpc::momentrate(shift != 0.0f ? zeta + shift : zeta, stftype, 0.0f, pw_zlen);
                };
                const float s_ii = stf(x0, y0, z0, 0.0f);
                const float s_vx = stf(x1, y0, z0, ahead), s_vy = stf(x0, y1, z0, ahead), s_vz = stf(x0, y0, z1, ahead);
                const float s_yz = stf(x0, y1, z1, 0.0f), s_xz = stf(x1, y0, z1, 0.0f), s_xy = stf(x1, y1, z0, 0.0f);
                const float la0 = lam[e], mu0 = mu[e];
                if (ps == 0) {
                    vx[e] = -sd * sf * s_vx;
                    vy[e] = sd * cf * s_vy;
                    vz[e] = -cd * s_vz;
                    sxx[e] = -(la0 + 2 * mu0 * sd * sd * sf * sf) * s_ii / v;
                    syy[e] = -(la0 + 2 * mu0 * sd * sd * cf * cf) * s_ii / v;
                    szz[e] = -(la0 + 2 * mu0 * cd * cd) * s_ii / v;
                    syz[e] = 2 * mu0 * sd * cd * cf * s_yz / v;
                    sxz[e] = -2 * mu0 * sd * cd * sf * s_xz / v;
                    sxy[e] = 2 * mu0 * sd * cd * sf * s_xy / v;
                } else {
                    const float ax = cl * cf + sl * cd * sf, ay = cl * sf - sl * cd * cf;
                    vx[e] = ax * s_vx;
                    vy[e] = ay * s_vy;
                    vz[e] = -sl * sd * s_vz;
                    sxx[e] = 2 * mu0 * sd * sf * ax * s_ii / v;
                    syy[e] = -2 * mu0 * sd * cf * ay * s_ii / v;
                    szz[e] = -2 * mu0 * cd * sl * sd * s_ii / v;
                    syz[e] = mu0 * (cl * cd * sf - sl * c2d * cf) * s_yz / v;
                    sxz[e] = mu0 * (cl * cd * cf + sl * c2d * sf) * s_xz / v;
                    sxy[e] = -mu0 * (cl * sd * c2f + 2 * sl * sd * cd * sf * cf) * s_xy / v;
                }
            }
    const float xend = g->xbeg + g->nx * dx, yend = g->ybeg + g->ny * dy;
    const int ic = swpc_x2i((g->xbeg + xend) / 2, g->xbeg, dx), jc = swpc_x2i((g->ybeg + yend) / 2, g->ybeg, dy);
    const int kc = swpc_x2i(pw_ztop, g->zbeg, dz);
    if (ic < -2 || ic > g->nx + 3 || jc < -2 || jc > g->ny + 3 || kc < -2 || kc > g->nz + 3) return SWPC_ERR_ARG;
    *fcut = speed(b.idx(kc, ic, jc)) / pw_zlen;
    return SWPC_OK;
}
