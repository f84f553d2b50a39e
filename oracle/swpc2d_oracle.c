/*
 * swpc2d_oracle.c -- CPU restatement of OpenSWPC's 2D P-SV and SH
 * viscoelastic staggered-grid velocity-stress FDM time step.
 *
 * TEST INFRASTRUCTURE ONLY (see swpc3d_oracle.c): used by tests/, the smoke
 * check and bench.py's CPU baseline, never by the product path.
 *
 * Kinds: 2 = P-SV (src/swpc_psv), 1 = SH (src/swpc_sh).  Same precision
 * macros as the 3D oracle (MPR for V/S and FD coefficients, SPR for memory
 * variables, medium and PML coefficients), built f32 / mixed / f64, compiled
 * with -ffp-contract=off.
 *
 * Two places where the reference's behaviour is undefined are restated with
 * the intended semantics of the 3D code:
 *   - surface_detection (src/swpc_psv/m_medium.f90:241-242,
 *     src/swpc_sh/m_medium.f90:247-248) assigns kfs_top twice and leaves
 *     kfs_bot uninitialised; here kfs_top = max(min(kfs)-2, kbeg) and
 *     kfs_bot = min(max(kfs)+2, kend) as in src/swpc_3d/m_medium.f90:382-383.
 *   - the SH absorber velocity update (src/swpc_sh/m_absorb_p.f90, Vy update)
 *     indexes gzc with i instead of k, reading outside gzc when nx > nz; here
 *     gzc(:, k) as in the P-SV and 3D codes.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef MPR
#define MPR float
#endif
#ifndef SPR
#define SPR float
#endif

#define NM_MAX 3
static const double PI_D = 3.141592653589793238462643383279502884;
static const float EPSL = 1.1920929e-07f;

typedef struct o2d {
    int kind, nx, nz, na, nm, nt;
    MPR dx, dz;
    float dt, xbeg, zbeg, tbeg, xend, zend;
    float fcut, vmin, vmax, UC, M0, zeta;
    int ibeg, iend, kbeg, kend, ibeg_m, iend_m, kbeg_m, kend_m;
    int ibeg_k, iend_k, kbeg_k, kend_k;
    long nk, ni;
    float *xc, *zc;
    int *kbeg_a;
    /* P-SV: V0 = Vx, V1 = Vz; S0 = Sxx, S1 = Szz, S2 = Sxz; R0..2 = Rxx Rzz Rxz
     * SH:   V0 = Vy;           S0 = Syz, S1 = Sxy;          R0..1 = Ryz Rxy */
    MPR *V[2], *S[3];
    SPR *R[3];                     /* (nm, memory box) */
    float *frho, *flam, *fmu, *ftaup, *ftaus;
    SPR *rho, *lam, *mu, *taup, *taus;
    float ts[NM_MAX];
    int *kfs, *kob, *kfs_top, *kfs_bot, *kob_top, *kob_bot;
    float *bddep;                /* (i, 0:NBD2) boundary depths (src/swpc_psv/m_global.f90 bddep) */
    int sdep_fit1;               /* sdep_fit: 0 'asis', 1 + n for 'bd<n>' (src/swpc_psv/m_source.f90:85) */
    int munk;                    /* munk_profile of the ocean column */
    SPR c1[NM_MAX], c2[NM_MAX], d1[NM_MAX], d2;
    MPR rc40x, rc41x, rc40z, rc41z, rd40x, rd41x, rd40z, rd41z;
    float *fgxc, *fgxe, *fgzc, *fgze;
    SPR *gxc, *gxe, *gzc, *gze;
    SPR *aux[8];   /* P-SV: axVx azVx axVz azVz axSxx azSxz axSxz azSzz; SH: axVy azVy axSxy azSyz */
    MPR r20x, r20z;
    int kbeg_min;
    long nka;
    int cerjan;                  /* abc_type = 'cerjan' (m_absorb_c.f90) */
    int stabilize_pml;           /* input-file switch (src/swpc_psv/m_medium.f90:175) */
    SPR *cgx_c, *cgx_b, *cgz_c, *cgz_b;   /* sponge factors, indexed [i - 1] */
    int bf_mode, stftype, nsrc;
    int *isrc, *ksrc;
    float *srcprm;
    MPR *mo, *mxx, *mzz, *mxz, *myz, *mxy, *fx, *fy, *fz;
    MPR dt_dxz;
    int nst, ntdec_w, ntw, sw_v, sw_u;
    int *ist, *kst;
    float *wav_vel, *wav_disp;
    SPR *ux, *uz;
    int threads;
} o2d;

#define NBD2 9
#define I2(o, k, i) ((((long)(i)) - (o)->ibeg_m) * (o)->nk + ((long)(k) - (o)->kbeg_m))
#define IA(o, k, i) ((((long)(i)) - (o)->ibeg) * (o)->nka + ((long)(k) - (o)->kbeg_min))
#define A(arr, k, i) (arr)[I2(o, k, i)]
#define IM(o, i) ((long)(i) - (o)->ibeg_m)
#define GX(arr, n, i) (arr)[4 * ((i) - o->ibeg) + (n) - 1]
#define GZ(arr, n, k) (arr)[4 * ((k) - o->kbeg) + (n) - 1]

static void *zalloc(size_t n) { return calloc(n ? n : 1, 1); }

static int x2i(float x, float beg, float d) {
    volatile float t = (x - beg) / d;
    return (int)ceilf(t);
}
static float i2x(int i, float beg, float d) {
    volatile float a = (float)i - 0.5f;
    volatile float b = a * d;
    return beg + b;
}

/* moment-rate functions, identical to swpc3d_oracle.c (m_fdtool.f90:339-497) */
static float stf(float t, int type, float ts, float tr) {
    switch (type) {
    case 1: return (ts <= t && t <= ts + tr) ? 1.0f / tr : 0.0f;
    case 2:
        if (ts <= t && t <= ts + tr / 2) return 4 * (t - ts) / (tr * tr);
        if (ts + tr / 2 < t && t <= ts + tr) return -4 * (t - ts - tr) / (tr * tr);
        return 0.0f;
    case 3: {
        float t1 = ts + tr / 4, t2 = ts + 3 * tr / 4;
        if (ts <= t && t < t1) { float a = t - ts; return 16 * (a * a) / (tr * tr * tr); }
        if (t1 <= t && t < t2) return -2 * (8 * (t * t + tr * ts + ts * ts - t * tr - 2 * t * ts) + tr * tr) / (tr * tr * tr);
        if (t2 <= t && t <= ts + tr) { float a = ts + tr - t; return 16 * (a * a) / (tr * tr * tr); }
        return 0.0f;
    }
    case 4:
        if (ts <= t && t <= ts + tr) return (float)((1.0 - cos(2 * PI_D * (double)(t - ts) / (double)tr)) / (double)tr);
        return 0.0f;
    case 5:
        if (ts <= t) {
            float tt = t - ts;
            double tp = 2 * PI_D;
            return (float)(tp * tp * (double)tt / (double)(tr * tr) * exp(-2 * PI_D * (double)tt / (double)tr));
        }
        return 0.0f;
    default:
        if (ts <= t && t <= ts + tr) {
            double s = sin(PI_D * (double)(t - ts) / (double)tr);
            return (float)(3.0 * PI_D * (s * s * s) / (double)(4.0f * tr));
        }
        return 0.0f;
    }
}

static void visco(int nm, float *ts, float fmin, float fmax, float *zeta_out) {
    /* visco_set_relaxtime + visco_constq_zeta (m_fdtool.f90:691-812), as in the 3D oracle */
    float oa = (float)(2 * PI_D * (double)fmin), ob = (float)(2 * PI_D * (double)fmax);
    if (nm == 1) ts[0] = 1.0f / sqrtf(oa * ob);
    else if (nm > 1)
        for (int m = 0; m < nm; m++) {
            double p = pow((double)(ob / oa), (double)m / (double)(nm - 1));
            ts[m] = 1.0f / (float)((double)oa * p);
        }
    if (nm == 0) { *zeta_out = 0.0f; return; }
    float i0[NM_MAX], i1[NM_MAX], s0 = 0.0f, s1 = 0.0f, s2 = 0.0f;
    for (int m = 0; m < nm; m++) {
        float t = ts[m];
        i0[m] = (logf(1.0f + (ob * ob) * (t * t)) - logf(1.0f + (oa * oa) * (t * t))) / (2 * t);
        float p = atanf(ob * t) - ob * t / (1 + (ob * ob) * (t * t));
        float q = atanf(oa * t) - oa * t / (1 + (oa * oa) * (t * t));
        i1[m] = (p - q) / (2 * t);
    }
    for (int m = 0; m < nm; m++) s0 += i0[m];
    for (int m = 0; m < nm; m++) s1 += i1[m];
    for (int m = 0; m < nm - 1; m++)
        for (int q = m + 1; q < nm; q++) {
            float w1 = atanf(ob * ts[m]) / ts[m] - atanf(ob * ts[q]) / ts[q];
            float w2 = atanf(oa * ts[m]) / ts[m] - atanf(oa * ts[q]) / ts[q];
            s2 = s2 + ts[m] * ts[q] / (ts[q] * ts[q] - ts[m] * ts[m]) * (w1 - w2);
        }
    *zeta_out = s0 / (s1 + 2 * s2);
}

/* visco_chi (m_fdtool.f90:730-753):
 * cc = mean_m (1 - i w ts (1+tau)) / (1 - i w ts) (terms in complex DP, sum in
 * complex SP); chi = 1 / Re(cc**(-0.5)) with the principal power in SP */
float o2d_visco_chi(int nm, const float *ts, float tau, float f) {
    float omega = (float)(2 * PI_D * (double)f);
    float ccr = 0.0f, cci = 0.0f;
    for (int m = 0; m < nm; m++) {
        double a = (double)omega * (double)ts[m];
        double ni = -(a * (1.0 + (double)tau)), di = -a;
        double den = 1.0 * 1.0 + di * di;
        double re = (1.0 * 1.0 + ni * di) / den;
        double im = (ni * 1.0 - 1.0 * di) / den;
        ccr = (float)((double)ccr + re);
        cci = (float)((double)cci + im);
    }
    ccr = ccr / nm;
    cci = cci / nm;
    float r = hypotf(ccr, cci);
    float th = atan2f(cci, ccr);
    float pr = cosf(-0.5f * th) / sqrtf(r);
    return 1.0f / pr;
}

o2d *o2d_create(int kind, int nx, int nz, int na, int nm, int nt, double dx, double dz, float dt, float xbeg,
                float zbeg, float tbeg, int threads) {
    o2d *o = (o2d *)zalloc(sizeof(o2d));
    o->kind = kind; o->nx = nx; o->nz = nz; o->na = na; o->nm = nm; o->nt = nt;
    o->dx = (MPR)dx; o->dz = (MPR)dz; o->dt = dt; o->xbeg = xbeg; o->zbeg = zbeg; o->tbeg = tbeg;
    o->threads = threads;
    o->xend = xbeg + nx * (float)o->dx;
    o->zend = zbeg + nz * (float)o->dz;
    o->UC = 1.0e-15f; o->M0 = 1.0f;
    o->ibeg = 1; o->iend = nx; o->kbeg = 1; o->kend = nz;
    o->ibeg_m = -2; o->iend_m = nx + 3; o->kbeg_m = -2; o->kend_m = nz + 3;
    o->nk = nz + 6; o->ni = nx + 6;
    o->xc = (float *)zalloc(sizeof(float) * o->ni);
    o->zc = (float *)zalloc(sizeof(float) * o->nk);
    for (int i = -2; i <= nx + 3; i++) o->xc[i + 2] = i2x(i, xbeg, (float)o->dx);
    for (int k = -2; k <= nz + 3; k++) o->zc[k + 2] = i2x(k, zbeg, (float)o->dz);
    o->kbeg_a = (int *)zalloc(sizeof(int) * o->ni);
    for (int i = -2; i <= nx + 3; i++) o->kbeg_a[i + 2] = (i <= na || nx - na + 1 <= i) ? 1 : nz - na + 1;
    o->ibeg_k = (1 <= na) ? na + 1 : 1;
    o->iend_k = (nx >= nx - na + 1) ? nx - na : nx;
    o->kbeg_k = 1;
    o->kend_k = nz - na;
    long n2 = o->nk * o->ni;
    for (int q = 0; q < 2; q++) o->V[q] = (MPR *)zalloc(sizeof(MPR) * n2);
    for (int q = 0; q < 3; q++) o->S[q] = (MPR *)zalloc(sizeof(MPR) * n2);
    for (int q = 0; q < 3; q++) o->R[q] = (SPR *)zalloc(sizeof(SPR) * n2 * (nm > 0 ? nm : 1));
#define AL(p, T) p = (T *)zalloc(sizeof(T) * n2)
    AL(o->frho, float); AL(o->flam, float); AL(o->fmu, float); AL(o->ftaup, float); AL(o->ftaus, float);
    AL(o->rho, SPR); AL(o->lam, SPR); AL(o->mu, SPR); AL(o->taup, SPR); AL(o->taus, SPR);
#undef AL
    o->kfs = (int *)zalloc(sizeof(int) * o->ni); o->kob = (int *)zalloc(sizeof(int) * o->ni);
    o->kfs_top = (int *)zalloc(sizeof(int) * o->ni); o->kfs_bot = (int *)zalloc(sizeof(int) * o->ni);
    o->kob_top = (int *)zalloc(sizeof(int) * o->ni); o->kob_bot = (int *)zalloc(sizeof(int) * o->ni);
    o->bddep = (float *)zalloc(sizeof(float) * o->ni * (NBD2 + 1));
    return o;
}

/* boundary depths of a model that carries its own; vmodel_lhm fills depth(1) and -9999 */
void o2d_set_bddep(o2d *o, const float *bd) { memcpy(o->bddep, bd, sizeof(float) * o->ni * (NBD2 + 1)); }

/* sdep_fit: -1 for 'asis', n for 'bd<n>'; set before o2d_source_setup */
void o2d_set_sdep_fit(o2d *o, int n) { o->sdep_fit1 = (n >= 0 && n <= NBD2) ? n + 1 : 0; }

void o2d_destroy(o2d *o) {
    if (!o) return;
    void *ps[] = {o->xc, o->zc, o->kbeg_a, o->V[0], o->V[1], o->S[0], o->S[1], o->S[2], o->R[0], o->R[1], o->R[2],
                  o->frho, o->flam, o->fmu, o->ftaup, o->ftaus, o->rho, o->lam, o->mu, o->taup, o->taus, o->kfs,
                  o->kob, o->kfs_top, o->kfs_bot, o->kob_top, o->kob_bot, o->fgxc, o->fgxe, o->fgzc, o->fgze,
                  o->gxc, o->gxe, o->gzc, o->gze, o->aux[0], o->aux[1], o->aux[2], o->aux[3], o->aux[4], o->aux[5],
                  o->aux[6], o->aux[7], o->isrc, o->ksrc, o->srcprm, o->mo, o->mxx, o->mzz, o->mxz, o->myz,
                  o->mxy, o->fx, o->fy, o->fz, o->ist, o->kst, o->wav_vel, o->wav_disp, o->ux, o->uz,
                  o->cgx_c, o->cgx_b, o->cgz_c, o->cgz_b, o->bddep};
    for (size_t n = 0; n < sizeof(ps) / sizeof(ps[0]); n++) free(ps[n]);
    free(o);
}

/* seawater__vel (src/shared/m_seawater.f90:36-49) */
static float o2d_seawater_vel(float z, int munk) {
    double eps = munk ? 0.00737 : 0.0;
    double zc = 1300.0;
    double zb = 2 * ((double)z * 1000. - zc) / zc;
    return (float)(1.5 * (1.0 + eps * (zb - 1.0 + exp(-zb))));
}

/* munk_profile switch; set before o2d_vmodel_lhm */
void o2d_set_munk(o2d *o, int munk) { o->munk = munk; }

/* vmodel_lhm in 2D (src/swpc_psv/m_vmodel_lhm.f90; same rule as 3D) with
 * the optional lhm_rmed perturbation (vcheck for P-SV, vcheck_sh for SH). */
void o2d_vmodel_lhm(o2d *o, int nlayer, const float *depth, const float *rho0, const float *vp0, const float *vs0,
                    const float *qp0, const float *qs0, float vcut, const float *xi, float rhomin, float *qp,
                    float *qs) {
    float r0[64], p0[64], s0[64], a0[64], b0[64];
    for (int l = 0; l < nlayer; l++) { r0[l] = rho0[l]; p0[l] = vp0[l]; s0[l] = vs0[l]; a0[l] = qp0[l]; b0[l] = qs0[l]; }
    for (int l = nlayer - 2; l >= 0; l--)
        if ((p0[l] < vcut || s0[l] < vcut) && (p0[l] > 0 && s0[l] > 0)) {
            p0[l] = p0[l + 1]; s0[l] = s0[l + 1]; r0[l] = r0[l + 1]; a0[l] = a0[l + 1]; b0[l] = b0[l + 1];
        }
    float ddx = (float)o->dx, ddz = (float)o->dz;
    /* topography shape and dummy boundary depths (src/swpc_psv/m_vmodel_lhm.f90, as m_vmodel_lhm.f90:104, 161) */
    for (int i = 0; i < o->ni; i++) {
        o->bddep[i * (NBD2 + 1)] = depth[0];
        for (int n = 1; n <= NBD2; n++) o->bddep[i * (NBD2 + 1) + n] = -9999.0f;
    }
    float dh = 1.0f / sqrtf(1.0f / (ddx * ddx) + 1.0f / (ddz * ddz));
    float vmax_r = 6.0f / 7.0f * dh / o->dt;
    for (int i = -2; i <= o->nx + 3; i++)
        for (int k = -2; k <= o->nz + 3; k++) {
            long e = I2(o, k, i);
            float zs = o->zc[k + 2];
            if (zs < depth[0]) {
                /* air (zs < 0) or seawater: src/swpc_psv/m_vmodel_lhm.f90:102-121, lam = rho (vp^2 - 2 vs^2) */
                if (zs < 0.0f) {
                    o->frho[e] = 0.001f; o->fmu[e] = 0.0f; o->flam[e] = 0.0f; qp[e] = 10.0f; qs[e] = 10.0f;
                } else {
                    float rho1 = 1.0f, vp1 = 1.0f * o2d_seawater_vel(zs, o->munk), vs1 = 0.0f;
                    o->frho[e] = rho1; o->fmu[e] = rho1 * vs1 * vs1; o->flam[e] = rho1 * (vp1 * vp1 - 2 * vs1 * vs1);
                    qp[e] = 1000000.0f; qs[e] = 1000000.0f;
                }
                continue;
            }
            float rho1 = 0, vp1 = 0, vs1 = 0, q1 = 0, q2 = 0;
            for (int l = 0; l < nlayer; l++) {
                if (zs >= depth[l]) {
                    if (xi) {
                        float x = xi[e];
                        rho1 = r0[l] * (1 + 0.8f * x);
                        vp1 = 1.0f * p0[l] * (1 + x);
                        vs1 = 1.0f * s0[l] * (1 + x);
                        if (p0[l] > 0 && s0[l] > 0) {
                            float gamma = vp1 / vs1;
                            if (gamma < EPSL) gamma = sqrtf(3.0f);
                            if (vp1 > vmax_r || vs1 > vmax_r) {
                                float xi2 = (1 + x) * vmax_r / vp1 - 1;
                                vp1 = vmax_r; vs1 = vmax_r / gamma;
                                rho1 = rho1 * (1 + 0.8f * xi2) / (1 + 0.8f * x);
                            }
                            if (vp1 < vcut || vs1 < vcut) { vs1 = vcut; vp1 = vcut * gamma; }
                            if (rho1 < rhomin) rho1 = rhomin;
                        }
                    } else {
                        rho1 = r0[l]; vp1 = 1.0f * p0[l]; vs1 = 1.0f * s0[l];
                    }
                    q1 = a0[l]; q2 = b0[l];
                }
            }
            o->frho[e] = rho1;
            o->fmu[e] = rho1 * vs1 * vs1;
            o->flam[e] = rho1 * (vp1 * vp1 - 2 * vs1 * vs1);
            qp[e] = q1;
            qs[e] = q2;
        }
}

/* medium__setup after the vmodel (src/swpc_psv/m_medium.f90:124-281) */
void o2d_medium_setup(o2d *o, const float *qp, const float *qs, float fq_min, float fq_max, float fq_ref) {
    int na = o->na, nx = o->nx, nz = o->nz;
    float *rho = o->frho, *lam = o->flam, *mu = o->fmu, *taup = o->ftaup, *taus = o->ftaus;
    long n2 = o->nk * o->ni;
    memcpy(taup, qp, sizeof(float) * n2);
    memcpy(taus, qs, sizeof(float) * n2);
#define CP(d, s) do { rho[d] = rho[s]; lam[d] = lam[s]; mu[d] = mu[s]; taup[d] = taup[s]; taus[d] = taus[s]; } while (0)
    for (int i = -2; i <= na; i++)
        for (int k = -2; k <= nz + 3; k++) CP(I2(o, k, i), I2(o, k, na + 1));
    for (int i = nx - na + 1; i <= nx + 3; i++)
        for (int k = -2; k <= nz + 3; k++) CP(I2(o, k, i), I2(o, k, nx - na));
    for (int i = -2; i <= nx + 3; i++)
        for (int k = nz - na + 1; k <= nz + 3; k++) CP(I2(o, k, i), I2(o, nz - na, i));
#undef CP
    visco(o->nm, o->ts, fq_min, fq_max, &o->zeta);
    for (long e = 0; e < n2; e++) {
        taup[e] = o->nm * o->zeta / taup[e];
        taus[e] = o->nm * o->zeta / taus[e];
    }
    if (o->nm > 0)
        for (int i = -2; i <= nx + 3; i++)
            for (int k = -2; k <= nz + 3; k++) {
                long e = I2(o, k, i);
                float rb2 = mu[e], ra2 = lam[e] + 2 * mu[e];
                float cm = o2d_visco_chi(o->nm, o->ts, taus[e], fq_ref);
                mu[e] = rb2 / (cm * cm);
                float cl = o2d_visco_chi(o->nm, o->ts, taup[e], fq_ref);
                lam[e] = ra2 / (cl * cl) - 2 * mu[e];
            }
    /* surface_detection (intended semantics, see the file header) */
    for (int i = -2; i <= nx + 3; i++) { o->kfs[i + 2] = 0; o->kob[i + 2] = 0; }
    for (int i = 0; i <= nx + 2; i++)
        for (int k = 1; k <= nz - 1; k++) {
            if (fabsf(mu[I2(o, k, i)]) < EPSL && fabsf(mu[I2(o, k + 1, i)]) > EPSL) o->kob[i + 2] = k;
            if (fabsf(lam[I2(o, k, i)]) < EPSL && fabsf(lam[I2(o, k + 1, i)]) > EPSL) o->kfs[i + 2] = k;
        }
    for (int i = 1; i <= nx; i++) {
        int fmn = 1 << 30, fmx = -(1 << 30), omn = 1 << 30, omx = -(1 << 30);
        for (int ii = i - 2; ii <= i + 3; ii++) {
            int f = o->kfs[ii + 2], b = o->kob[ii + 2];
            if (f < fmn) fmn = f;
            if (f > fmx) fmx = f;
            if (b < omn) omn = b;
            if (b > omx) omx = b;
        }
        o->kfs_top[i + 2] = fmn - 2 > 1 ? fmn - 2 : 1;
        o->kfs_bot[i + 2] = fmx + 2 < nz ? fmx + 2 : nz;
        o->kob_top[i + 2] = omn - 2 > 1 ? omn - 2 : 1;
        o->kob_bot[i + 2] = omx + 2 < nz ? omx + 2 : nz;
    }
    float vmax1 = -1, vmin1 = 1e30f;
    for (int i = 1; i <= nx; i++)
        for (int k = o->kfs[i + 2] + 1; k <= nz; k++) {
            long e = I2(o, k, i);
            float vp = sqrtf((lam[e] + 2 * mu[e]) / rho[e]);
            if (vp > vmax1) vmax1 = vp;
            float vs = sqrtf(mu[e] / rho[e]);
            if (vs < EPSL) continue;
            if (vs < vmin1) vmin1 = vs;
        }
    o->vmax = vmax1; o->vmin = vmin1;
    /* stabilize_absorber: src/swpc_psv/m_medium.f90:175-178, 309-365 */
    if (o->stabilize_pml) {
        const float vmin_pml = vmax1 * 0.4f;
        for (int i = o->ibeg - 1; i <= o->iend + 1; i++) {
            int k0 = 1 << 30;
            for (int ii = i - 2; ii <= i + 2; ii++)
                if (o->kbeg_a[IM(o, ii)] < k0) k0 = o->kbeg_a[IM(o, ii)];
            int k = k0;
            while (k <= o->kend) {
                if (A(lam, k, i) < A(lam, k - 1, i) || A(mu, k, i) < A(mu, k - 1, i)) {
                    int k2;
                    for (k2 = k + 1; k2 <= o->kend; k2++)
                        if (A(lam, k2, i) > A(lam, k2 - 1, i) || A(mu, k2, i) > A(mu, k2 - 1, i)) break;
                    if (k2 - k <= 20) {
                        for (int kk = k; kk <= k2 - 1; kk++) {
                            A(rho, kk, i) = A(rho, k - 1, i); A(lam, kk, i) = A(lam, k - 1, i);
                            A(mu, kk, i) = A(mu, k - 1, i); A(taup, kk, i) = A(taup, k - 1, i);
                            A(taus, kk, i) = A(taus, k - 1, i);
                        }
                        k = k2 - 1;
                    }
                }
                k = k + 1;
            }
            for (k = k0; k <= o->kend; k++) {
                float vp = sqrtf((A(lam, k, i) + 2 * A(mu, k, i)) / A(rho, k, i));
                float vs = sqrtf(A(mu, k, i) / A(rho, k, i));
                if (vs < EPSL) continue;
                float gamma = sqrtf(3.0f);
                if (vs < vmin_pml) {
                    vs = vmin_pml;
                    vp = vs * gamma;
                    A(lam, k, i) = A(rho, k, i) * (vp * vp - 2 * (vs * vs));
                    A(mu, k, i) = A(rho, k, i) * (vs * vs);
                }
            }
        }
    }
    for (long e = 0; e < n2; e++) {
        o->rho[e] = (SPR)rho[e]; o->lam[e] = (SPR)lam[e]; o->mu[e] = (SPR)mu[e];
        o->taup[e] = (SPR)taup[e]; o->taus[e] = (SPR)taus[e];
    }
}

/* kernel__setup (src/swpc_psv/m_kernel.f90:30-73) */
void o2d_kernel_setup(o2d *o) {
    o->rc40x = (MPR)17.0 / (MPR)16.0 / o->dx; o->rc40z = (MPR)17.0 / (MPR)16.0 / o->dz;
    o->rc41x = (MPR)1.0 / (MPR)48.0 / o->dx; o->rc41z = (MPR)1.0 / (MPR)48.0 / o->dz;
    o->rd40x = (MPR)-1.0 / (MPR)16.0 / o->dx; o->rd40z = (MPR)-1.0 / (MPR)16.0 / o->dz;
    o->rd41x = (MPR)-1.0 / (MPR)48.0 / o->dx; o->rd41z = (MPR)-1.0 / (MPR)48.0 / o->dz;
    if (o->nm > 0) {
        float dt = o->dt, fd2 = 0.0f;
        for (int m = 0; m < o->nm; m++) {
            o->c1[m] = (2 * o->ts[m] - dt) / (2 * o->ts[m] + dt);
            o->c2[m] = (float)((2) / (2 * o->ts[m] + dt) / o->nm);
        }
        for (int m = 0; m < o->nm; m++) fd2 = fd2 + dt / (2 * o->ts[m] - dt);
        o->d2 = fd2 / o->nm;
        for (int m = 0; m < o->nm; m++) o->d1[m] = 2 * o->ts[m] / (2 * o->ts[m] - dt);
    }
}

static void damping_profile(float x, float H, float beg, float end, int na, float fcut, float dt, float *g) {
    float R0 = powf(10.0f, -(log10f((float)na) - 1) / log10f(2.0f) - 3.0f);
    float d0 = -(1.0f / (2.0f * H)) * (1 + 1) * 6.0f * logf(R0);
    float a0 = (float)(PI_D * (double)fcut);
    float xx;
    if (x <= beg + H) xx = (beg + H) - x;
    else if (x >= end - H) xx = x - (end - H);
    else xx = 0.0f;
    float r = fabsf(xx / H);
    float d = d0 * r, a = a0 * (1.0f - r), b = 1.0f + (7.0f - 1.0f) * (r * r), h = dt / 2.0f;
    g[0] = ((1.0f + h * a) / b) / (1.0f + h * (a + d / b));
    g[1] = (-1.0f / b) / (1.0f + h * (a + d / b));
    g[2] = (1.0f - h * (a + d / b)) / (1.0f + h * (a + d / b));
    g[3] = (d / b) / (1.0f + h * (a + d / b));
}

/* absorb_p__setup (src/swpc_psv/m_absorb_p.f90:60-104) */
void o2d_absorb_setup(o2d *o, float fcut) {
    o->fcut = fcut;
    o->r20x = (MPR)(float)(1.0 / (double)o->dx);   /* real(1.0 / dx) */
    o->r20z = (MPR)(float)(1.0 / (double)o->dz);
    int nx = o->nx, nz = o->nz;
    o->fgxc = (float *)zalloc(16 * nx); o->fgxe = (float *)zalloc(16 * nx);
    o->fgzc = (float *)zalloc(16 * nz); o->fgze = (float *)zalloc(16 * nz);
    float hx = o->na * (float)o->dx, hz = o->na * (float)o->dz;
    for (int i = 1; i <= nx; i++) {
        float xc = o->xc[i + 2];
        damping_profile(xc, hx, o->xbeg, o->xend, o->na, fcut, o->dt, &o->fgxc[4 * (i - 1)]);
        damping_profile(xc + (float)o->dx / 2.0f, hx, o->xbeg, o->xend, o->na, fcut, o->dt, &o->fgxe[4 * (i - 1)]);
    }
    for (int k = 1; k <= nz; k++) {
        float zc = o->zc[k + 2];
        damping_profile(zc, hz, o->zbeg, o->zend, o->na, fcut, o->dt, &o->fgzc[4 * (k - 1)]);
        damping_profile(zc + (float)o->dz / 2.0f, hz, o->zbeg, o->zend, o->na, fcut, o->dt, &o->fgze[4 * (k - 1)]);
    }
    o->gxc = (SPR *)zalloc(sizeof(SPR) * 4 * nx); o->gxe = (SPR *)zalloc(sizeof(SPR) * 4 * nx);
    o->gzc = (SPR *)zalloc(sizeof(SPR) * 4 * nz); o->gze = (SPR *)zalloc(sizeof(SPR) * 4 * nz);
    for (int q = 0; q < 4 * nx; q++) { o->gxc[q] = (SPR)o->fgxc[q]; o->gxe[q] = (SPR)o->fgxe[q]; }
    for (int q = 0; q < 4 * nz; q++) { o->gzc[q] = (SPR)o->fgzc[q]; o->gze[q] = (SPR)o->fgze[q]; }
    int kmin = 1 << 30;
    for (int i = 0; i < o->ni; i++) if (o->kbeg_a[i] < kmin) kmin = o->kbeg_a[i];
    o->kbeg_min = kmin;
    o->nka = nz - kmin + 1;
    for (int q = 0; q < 8; q++) o->aux[q] = (SPR *)zalloc(sizeof(SPR) * o->nka * nx);
}

#define ISIGN(o, k, i)                                                                   \
    ({                                                                                   \
        int a_ = ((k) - (o)->kfs_top[(i) + 2]) * ((o)->kfs_bot[(i) + 2] - (k));          \
        int b_ = ((k) - (o)->kob_top[(i) + 2]) * ((o)->kob_bot[(i) + 2] - (k));          \
        ((a_ > b_ ? a_ : b_) >= 0) ? 1 : -1;                                             \
    })

/* ---------------------------------------------------------------- P-SV */
static void psv_update_vel(o2d *o) {
    MPR *Vx = o->V[0], *Vz = o->V[1], *Sxx = o->S[0], *Szz = o->S[1], *Sxz = o->S[2];
    float dt = o->dt;
    for (int i = o->ibeg_k; i <= o->iend_k; i++)
        for (int k = o->kbeg_k; k <= o->kend_k; k++) {
            int isign = ISIGN(o, k, i);
            MPR re40x = o->rc40x + isign * o->rd40x, re41x = o->rc41x + isign * o->rd41x;
            MPR re40z = o->rc40z + isign * o->rd40z, re41z = o->rc41z + isign * o->rd41z;
            MPR dxSxx = (A(Sxx, k, i + 1) - A(Sxx, k, i)) * re40x - (A(Sxx, k, i + 2) - A(Sxx, k, i - 1)) * re41x;
            MPR dzSzz = (A(Szz, k + 1, i) - A(Szz, k, i)) * re40z - (A(Szz, k + 2, i) - A(Szz, k - 1, i)) * re41z;
            MPR dxSxz = (A(Sxz, k, i) - A(Sxz, k, i - 1)) * re40x - (A(Sxz, k, i + 1) - A(Sxz, k, i - 2)) * re41x;
            MPR dzSxz = (A(Sxz, k, i) - A(Sxz, k - 1, i)) * re40z - (A(Sxz, k + 1, i) - A(Sxz, k - 2, i)) * re41z;
            SPR bx = 2.0f / (A(o->rho, k, i) + A(o->rho, k, i + 1));
            SPR bz = 2.0f / (A(o->rho, k, i) + A(o->rho, k + 1, i));
            A(Vx, k, i) = A(Vx, k, i) + bx * (dxSxx + dzSxz) * dt;
            A(Vz, k, i) = A(Vz, k, i) + bz * (dxSxz + dzSzz) * dt;
        }
}

static void psv_update_stress(o2d *o) {
    MPR *Vx = o->V[0], *Vz = o->V[1];
    float dt = o->dt;
    int nm = o->nm;
    for (int i = o->ibeg_k; i <= o->iend_k; i++)
        for (int k = o->kbeg_k; k <= o->kend_k; k++) {
            int isign = ISIGN(o, k, i);
            MPR re40x = o->rc40x + isign * o->rd40x, re41x = o->rc41x + isign * o->rd41x;
            MPR re40z = o->rc40z + isign * o->rd40z, re41z = o->rc41z + isign * o->rd41z;
            MPR dxVx = (A(Vx, k, i) - A(Vx, k, i - 1)) * re40x - (A(Vx, k, i + 1) - A(Vx, k, i - 2)) * re41x;
            MPR dzVz = (A(Vz, k, i) - A(Vz, k - 1, i)) * re40z - (A(Vz, k + 1, i) - A(Vz, k - 2, i)) * re41z;
            long e = I2(o, k, i);
            SPR mu2 = 2 * o->mu[e], lam2mu = o->lam[e] + mu2, taup1 = o->taup[e], taus1 = o->taus[e];
            SPR d2v2 = (SPR)(dxVx + dzVz);
            SPR f_Rxx = (SPR)(lam2mu * taup1 * d2v2 - mu2 * taus1 * dzVz);
            SPR f_Rzz = (SPR)(lam2mu * taup1 * d2v2 - mu2 * taus1 * dxVx);
            SPR Rxx_n = 0.0f, Rzz_n = 0.0f;
            for (int m = 0; m < nm; m++) {
                SPR *rx = &o->R[0][e * nm + m], *rz = &o->R[1][e * nm + m];
                *rx = o->c1[m] * *rx - o->c2[m] * f_Rxx * dt;
                *rz = o->c1[m] * *rz - o->c2[m] * f_Rzz * dt;
                Rxx_n = Rxx_n + o->d1[m] * *rx;
                Rzz_n = Rzz_n + o->d1[m] * *rz;
            }
            SPR taup_plus1 = 1 + taup1 * (1 + o->d2), taus_plus1 = 1 + taus1 * (1 + o->d2);
            o->S[0][e] = o->S[0][e] + (lam2mu * taup_plus1 * d2v2 - mu2 * taus_plus1 * dzVz + Rxx_n) * dt;
            o->S[1][e] = o->S[1][e] + (lam2mu * taup_plus1 * d2v2 - mu2 * taus_plus1 * dxVx + Rzz_n) * dt;
        }
    for (int i = o->ibeg_k; i <= o->iend_k; i++)
        for (int k = o->kbeg_k; k <= o->kend_k; k++) {
            int isign = ISIGN(o, k, i);
            MPR re40x = o->rc40x + isign * o->rd40x, re41x = o->rc41x + isign * o->rd41x;
            MPR re40z = o->rc40z + isign * o->rd40z, re41z = o->rc41z + isign * o->rd41z;
            MPR dxVz = (A(Vz, k, i + 1) - A(Vz, k, i)) * re40x - (A(Vz, k, i + 2) - A(Vz, k, i - 1)) * re41x;
            MPR dzVx = (A(Vx, k + 1, i) - A(Vx, k, i)) * re40z - (A(Vx, k + 2, i) - A(Vx, k - 1, i)) * re41z;
            long e = I2(o, k, i);
            SPR taus1 = o->taus[e];
            SPR nnn = o->mu[e], pnn = A(o->mu, k + 1, i), npn = A(o->mu, k, i + 1), ppn = A(o->mu, k + 1, i + 1);
            SPR mu_xz = 4 * nnn * pnn * npn * ppn / (nnn * pnn * npn + nnn * pnn * ppn + nnn * npn * ppn + pnn * npn * ppn + EPSL);
            SPR dxVz_dzVx = (SPR)(dxVz + dzVx);
            SPR f_Rxz = mu_xz * taus1 * dxVz_dzVx;
            SPR Rxz_n = 0.0f;
            for (int m = 0; m < nm; m++) {
                SPR *r = &o->R[2][e * nm + m];
                *r = o->c1[m] * *r - o->c2[m] * f_Rxz * dt;
                Rxz_n = Rxz_n + o->d1[m] * *r;
            }
            SPR taus_plus1 = 1 + taus1 * (1 + o->d2);
            o->S[2][e] = o->S[2][e] + (mu_xz * taus_plus1 * dxVz_dzVx + Rxz_n) * dt;
        }
}

/* absorb_c__setup of the 2D codes (src/swpc_psv/m_absorb_c.f90:27-88,
 * src/swpc_sh/m_absorb_c.f90:27-80) and the kernel region of abc_type =
 * 'cerjan' (src/swpc_psv/m_global.f90:281-303: the whole domain) */
static void cerjan_axis2d(SPR *gc, SPR *gb, int n, int na, float d, int low) {
    const float alpha = 0.09f;
    const float L = na * d;
    for (int i = 1; i <= n; i++) {
        float c = 1.0f, b = 1.0f;
        if (low && i <= na) {
            const float x = i2x(i, 0.0f, d);
            const float yc = 1.0f - x / L, yb = 1.0f - (x + d / 2) / L;
            c = expf(-alpha * (yc * yc));
            b = expf(-alpha * (yb * yb));
        } else if (i >= n - na + 1) {
            const float x = i2x(i, n * d, -d);
            const float yc = 1.0f - (x + d / 2) / L, yb = 1.0f - x / L;
            c = expf(-alpha * (yc * yc));
            b = expf(-alpha * (yb * yb));
        }
        gc[i - 1] = c;
        gb[i - 1] = b;
    }
}

void o2d_set_stabilize(o2d *o, int on) { o->stabilize_pml = on; }

void o2d_cerjan_setup(o2d *o) {
    o->cerjan = 1;
    o->cgx_c = (SPR *)zalloc(sizeof(SPR) * o->nx); o->cgx_b = (SPR *)zalloc(sizeof(SPR) * o->nx);
    o->cgz_c = (SPR *)zalloc(sizeof(SPR) * o->nz); o->cgz_b = (SPR *)zalloc(sizeof(SPR) * o->nz);
    cerjan_axis2d(o->cgx_c, o->cgx_b, o->nx, o->na, (float)o->dx, 1);
    cerjan_axis2d(o->cgz_c, o->cgz_b, o->nz, o->na, (float)o->dz, 0);   /* free surface undamped */
    o->ibeg_k = o->ibeg; o->iend_k = o->iend; o->kbeg_k = o->kbeg; o->kend_k = o->kend;
}

/* absorb_c__update_stress / _vel (src/swpc_psv/m_absorb_c.f90:90-160) */
static void cerjan_psv(o2d *o, int stress) {
    for (int i = o->ibeg; i <= o->iend; i++)
        for (int k = o->kbeg; k <= o->kend; k++) {
            const SPR xc = o->cgx_c[i - 1], xb = o->cgx_b[i - 1], zc = o->cgz_c[k - 1], zb = o->cgz_b[k - 1];
            if (stress) {
                const SPR gc = xc * zc, gb = xb * zb;
                A(o->S[0], k, i) = A(o->S[0], k, i) * gc;
                A(o->S[1], k, i) = A(o->S[1], k, i) * gc;
                A(o->S[2], k, i) = A(o->S[2], k, i) * gb;
            } else {
                A(o->V[0], k, i) = A(o->V[0], k, i) * xb * zc;
                A(o->V[1], k, i) = A(o->V[1], k, i) * xc * zb;
            }
        }
}

/* absorb_c__update_stress / _vel (src/swpc_sh/m_absorb_c.f90:82-135) */
static void cerjan_sh(o2d *o, int stress) {
    for (int i = o->ibeg; i <= o->iend; i++)
        for (int k = o->kbeg; k <= o->kend; k++) {
            const SPR xc = o->cgx_c[i - 1], xb = o->cgx_b[i - 1], zc = o->cgz_c[k - 1], zb = o->cgz_b[k - 1];
            if (stress) {
                A(o->S[0], k, i) = A(o->S[0], k, i) * xc * zb;
                A(o->S[1], k, i) = A(o->S[1], k, i) * xb * zc;
            } else {
                A(o->V[0], k, i) = A(o->V[0], k, i) * xc * zc;
            }
        }
}

static void psv_absorb_vel(o2d *o) {
    if (o->cerjan) { cerjan_psv(o, 0); return; }
    MPR *Vx = o->V[0], *Vz = o->V[1], *Sxx = o->S[0], *Szz = o->S[1], *Sxz = o->S[2];
    SPR *axSxx = o->aux[4], *azSxz = o->aux[5], *axSxz = o->aux[6], *azSzz = o->aux[7];
    float dt = o->dt;
    for (int i = o->ibeg; i <= o->iend; i++)
        for (int k = o->kbeg_a[i + 2]; k <= o->kend; k++) {
            MPR dxSxx = (A(Sxx, k, i + 1) - A(Sxx, k, i)) * o->r20x;
            MPR dzSzz = (A(Szz, k + 1, i) - A(Szz, k, i)) * o->r20z;
            MPR dxSxz = (A(Sxz, k, i) - A(Sxz, k, i - 1)) * o->r20x;
            MPR dzSxz = (A(Sxz, k, i) - A(Sxz, k - 1, i)) * o->r20z;
            SPR bx = 2.0f / (A(o->rho, k, i) + A(o->rho, k, i + 1));
            SPR bz = 2.0f / (A(o->rho, k, i) + A(o->rho, k + 1, i));
            long q = IA(o, k, i), e = I2(o, k, i);
            Vx[e] = Vx[e] + bx * (GX(o->gxe, 1, i) * dxSxx + GZ(o->gzc, 1, k) * dzSxz
                                  + GX(o->gxe, 2, i) * axSxx[q] + GZ(o->gzc, 2, k) * azSxz[q]) * dt;
            Vz[e] = Vz[e] + bz * (GX(o->gxc, 1, i) * dxSxz + GZ(o->gze, 1, k) * dzSzz
                                  + GX(o->gxc, 2, i) * axSxz[q] + GZ(o->gze, 2, k) * azSzz[q]) * dt;
            axSxx[q] = (SPR)(GX(o->gxe, 3, i) * axSxx[q] + GX(o->gxe, 4, i) * dxSxx * dt);
            azSxz[q] = (SPR)(GZ(o->gzc, 3, k) * azSxz[q] + GZ(o->gzc, 4, k) * dzSxz * dt);
            axSxz[q] = (SPR)(GX(o->gxc, 3, i) * axSxz[q] + GX(o->gxc, 4, i) * dxSxz * dt);
            azSzz[q] = (SPR)(GZ(o->gze, 3, k) * azSzz[q] + GZ(o->gze, 4, k) * dzSzz * dt);
        }
}

static void psv_absorb_stress(o2d *o) {
    if (o->cerjan) { cerjan_psv(o, 1); return; }
    MPR *Vx = o->V[0], *Vz = o->V[1];
    SPR *axVx = o->aux[0], *azVx = o->aux[1], *axVz = o->aux[2], *azVz = o->aux[3];
    float dt = o->dt;
    for (int i = o->ibeg; i <= o->iend; i++) {
        for (int k = o->kbeg_a[i + 2]; k <= o->kend; k++) {
            MPR dxVx = (A(Vx, k, i) - A(Vx, k, i - 1)) * o->r20x;
            MPR dzVz = (A(Vz, k, i) - A(Vz, k - 1, i)) * o->r20z;
            long q = IA(o, k, i), e = I2(o, k, i);
            SPR lam2mu_R = o->lam[e] + 2 * o->mu[e];
            SPR lam_R = lam2mu_R - 2 * o->mu[e];
            SPR dxVx_ade = (SPR)(GX(o->gxc, 1, i) * dxVx + GX(o->gxc, 2, i) * axVx[q]);
            SPR dzVz_ade = (SPR)(GZ(o->gzc, 1, k) * dzVz + GZ(o->gzc, 2, k) * azVz[q]);
            o->S[0][e] = o->S[0][e] + (lam2mu_R * dxVx_ade + lam_R * dzVz_ade) * dt;
            o->S[1][e] = o->S[1][e] + (lam2mu_R * dzVz_ade + lam_R * dxVx_ade) * dt;
            axVx[q] = (SPR)(GX(o->gxc, 3, i) * axVx[q] + GX(o->gxc, 4, i) * dxVx * dt);
            azVz[q] = (SPR)(GZ(o->gzc, 3, k) * azVz[q] + GZ(o->gzc, 4, k) * dzVz * dt);
        }
        for (int k = o->kbeg_a[i + 2]; k <= o->kend; k++) {
            MPR dzVx = (A(Vx, k + 1, i) - A(Vx, k, i)) * o->r20z;
            MPR dxVz = (A(Vz, k, i + 1) - A(Vz, k, i)) * o->r20x;
            long q = IA(o, k, i), e = I2(o, k, i);
            SPR nnn = o->mu[e], pnn = A(o->mu, k + 1, i), npn = A(o->mu, k, i + 1), ppn = A(o->mu, k + 1, i + 1);
            SPR muxz = 4 * nnn * pnn * npn * ppn / (nnn * pnn * npn + nnn * pnn * ppn + nnn * npn * ppn + pnn * npn * ppn + EPSL);
            o->S[2][e] = o->S[2][e] + muxz * (GX(o->gxe, 1, i) * dxVz + GZ(o->gze, 1, k) * dzVx
                                              + GX(o->gxe, 2, i) * axVz[q] + GZ(o->gze, 2, k) * azVx[q]) * dt;
            azVx[q] = (SPR)(GZ(o->gze, 3, k) * azVx[q] + GZ(o->gze, 4, k) * dzVx * dt);
            axVz[q] = (SPR)(GX(o->gxe, 3, i) * axVz[q] + GX(o->gxe, 4, i) * dxVz * dt);
        }
    }
}

/* ---------------------------------------------------------------- SH */
static void sh_update_vel(o2d *o) {
    MPR *Vy = o->V[0], *Syz = o->S[0], *Sxy = o->S[1];
    float dt = o->dt;
    for (int i = o->ibeg_k; i <= o->iend_k; i++)
        for (int k = o->kbeg_k; k <= o->kend_k; k++) {
            int isign = ISIGN(o, k, i);
            MPR re40x = o->rc40x + isign * o->rd40x, re41x = o->rc41x + isign * o->rd41x;
            MPR re40z = o->rc40z + isign * o->rd40z, re41z = o->rc41z + isign * o->rd41z;
            MPR dzSyz = (A(Syz, k, i) - A(Syz, k - 1, i)) * re40z - (A(Syz, k + 1, i) - A(Syz, k - 2, i)) * re41z;
            MPR dxSxy = (A(Sxy, k, i) - A(Sxy, k, i - 1)) * re40x - (A(Sxy, k, i + 1) - A(Sxy, k, i - 2)) * re41x;
            SPR by = 1.0f / A(o->rho, k, i);
            A(Vy, k, i) = A(Vy, k, i) + by * (dxSxy + dzSyz) * dt;
        }
}

static void sh_update_stress(o2d *o) {
    MPR *Vy = o->V[0];
    float dt = o->dt;
    int nm = o->nm;
    for (int i = o->ibeg_k; i <= o->iend_k; i++)
        for (int k = o->kbeg_k; k <= o->kend_k; k++) {
            int isign = ISIGN(o, k, i);
            MPR re40x = o->rc40x + isign * o->rd40x, re41x = o->rc41x + isign * o->rd41x;
            MPR re40z = o->rc40z + isign * o->rd40z, re41z = o->rc41z + isign * o->rd41z;
            MPR dxVy = (A(Vy, k, i + 1) - A(Vy, k, i)) * re40x - (A(Vy, k, i + 2) - A(Vy, k, i - 1)) * re41x;
            MPR dzVy = (A(Vy, k + 1, i) - A(Vy, k, i)) * re40z - (A(Vy, k + 2, i) - A(Vy, k - 1, i)) * re41z;
            long e = I2(o, k, i);
            SPR nnn = o->mu[e], pnn = A(o->mu, k + 1, i), npn = A(o->mu, k, i + 1);
            SPR mu_xy = 2 * nnn * npn / (nnn + npn + EPSL);
            SPR mu_yz = 2 * nnn * pnn / (nnn + pnn + EPSL);
            SPR taus1 = o->taus[e];
            SPR f_Ryz = (SPR)(mu_yz * taus1 * dzVy);
            SPR f_Rxy = (SPR)(mu_xy * taus1 * dxVy);
            SPR Ryz_n = 0.0f, Rxy_n = 0.0f;
            for (int m = 0; m < nm; m++) {
                SPR *ry = &o->R[0][e * nm + m], *rx = &o->R[1][e * nm + m];
                *ry = o->c1[m] * *ry - o->c2[m] * f_Ryz * dt;
                *rx = o->c1[m] * *rx - o->c2[m] * f_Rxy * dt;
                Ryz_n = Ryz_n + o->d1[m] * *ry;
                Rxy_n = Rxy_n + o->d1[m] * *rx;
            }
            SPR taus_plus1 = 1 + taus1 * (1 + o->d2);
            o->S[0][e] = o->S[0][e] + (mu_yz * taus_plus1 * dzVy + Ryz_n) * dt;
            o->S[1][e] = o->S[1][e] + (mu_xy * taus_plus1 * dxVy + Rxy_n) * dt;
        }
}

static void sh_absorb_vel(o2d *o) {
    if (o->cerjan) { cerjan_sh(o, 0); return; }
    MPR *Vy = o->V[0], *Syz = o->S[0], *Sxy = o->S[1];
    SPR *axSxy = o->aux[2], *azSyz = o->aux[3];
    float dt = o->dt;
    for (int i = o->ibeg; i <= o->iend; i++)
        for (int k = o->kbeg_a[i + 2]; k <= o->kend; k++) {
            MPR dzSyz = (A(Syz, k, i) - A(Syz, k - 1, i)) * o->r20z;
            MPR dxSxy = (A(Sxy, k, i) - A(Sxy, k, i - 1)) * o->r20x;
            SPR by = 1.0f / A(o->rho, k, i);
            long q = IA(o, k, i), e = I2(o, k, i);
            Vy[e] = Vy[e] + by * (GX(o->gxc, 1, i) * dxSxy + GZ(o->gzc, 1, k) * dzSyz
                                  + GX(o->gxc, 2, i) * axSxy[q] + GZ(o->gzc, 2, k) * azSyz[q]) * dt;
            axSxy[q] = GX(o->gxc, 3, i) * axSxy[q] + GX(o->gxc, 4, i) * dxSxy * dt;
            azSyz[q] = GZ(o->gzc, 3, k) * azSyz[q] + GZ(o->gzc, 4, k) * dzSyz * dt;
        }
}

static void sh_absorb_stress(o2d *o) {
    if (o->cerjan) { cerjan_sh(o, 1); return; }
    MPR *Vy = o->V[0];
    SPR *axVy = o->aux[0], *azVy = o->aux[1];
    float dt = o->dt;
    for (int i = o->ibeg; i <= o->iend; i++)
        for (int k = o->kbeg_a[i + 2]; k <= o->kend; k++) {
            MPR dxVy = (A(Vy, k, i + 1) - A(Vy, k, i)) * o->r20x;
            MPR dzVy = (A(Vy, k + 1, i) - A(Vy, k, i)) * o->r20z;
            long q = IA(o, k, i), e = I2(o, k, i);
            SPR nnn = o->mu[e], pnn = A(o->mu, k + 1, i), npn = A(o->mu, k, i + 1);
            SPR muxy = 2 * nnn * npn / (nnn + npn + EPSL);
            SPR muyz = 2 * nnn * pnn / (nnn + pnn + EPSL);
            axVy[q] = GX(o->gxe, 3, i) * axVy[q] + GX(o->gxe, 4, i) * dxVy * dt;
            azVy[q] = GZ(o->gze, 3, k) * azVy[q] + GZ(o->gze, 4, k) * dzVy * dt;
            o->S[0][e] = o->S[0][e] + muyz * (GZ(o->gze, 1, k) * dzVy + GZ(o->gze, 2, k) * azVy[q]) * dt;
            o->S[1][e] = o->S[1][e] + muxy * (GX(o->gxe, 1, i) * dxVy + GX(o->gxe, 2, i) * axVy[q]) * dt;
        }
}

/* ------------------------------------------------ comm (one node: zeros) */
static void zero_col(o2d *o, MPR *f, int i) {
    for (int k = 1; k <= o->nz; k++) A(f, k, i) = 0;
}
static void comm_stress(o2d *o) {
    int ib = o->ibeg, ie = o->iend;
    if (o->kind == 2) {   /* src/swpc_psv/m_global.f90:409-414 */
        zero_col(o, o->S[0], ib - 1); zero_col(o, o->S[2], ib - 2); zero_col(o, o->S[2], ib - 1);
        zero_col(o, o->S[0], ie + 1); zero_col(o, o->S[0], ie + 2); zero_col(o, o->S[2], ie + 1);
    } else {              /* src/swpc_sh/m_global.f90:386-388 */
        zero_col(o, o->S[1], ie + 1); zero_col(o, o->S[1], ib - 2); zero_col(o, o->S[1], ib - 1);
    }
}
static void comm_vel(o2d *o) {
    int ib = o->ibeg, ie = o->iend;
    if (o->kind == 2) {   /* src/swpc_psv/m_global.f90:356-361 */
        zero_col(o, o->V[0], ib - 2); zero_col(o, o->V[0], ib - 1); zero_col(o, o->V[1], ib - 1);
        zero_col(o, o->V[0], ie + 1); zero_col(o, o->V[1], ie + 1); zero_col(o, o->V[1], ie + 2);
    } else {              /* src/swpc_sh/m_global.f90:340-342 */
        zero_col(o, o->V[0], ie + 1); zero_col(o, o->V[0], ie + 2); zero_col(o, o->V[0], ib - 1);
    }
}

/* ------------------------------------------------------------- sources */
/* m6 = (xx yy zz yz xz xy) ; f3 = (fx fy fz) */
int o2d_source_setup(o2d *o, int bf_mode, int n_g, const float *sx, const float *sz, const float *prm, const float *mo_g,
                     const float *m6, const float *f3, int stftype) {
    o->bf_mode = bf_mode; o->stftype = stftype;
    float fcut = 0.0f;
    for (int i = 0; i < n_g; i++) { float f = 1 / prm[2 * i + 1]; if (f > fcut) fcut = f; }
    o->fcut = fcut;
    if (bf_mode) {
        float s = 0.0f;
        if (o->kind == 2) {
            for (int i = 0; i < n_g; i++) s += f3[3 * i] * f3[3 * i] + f3[3 * i + 2] * f3[3 * i + 2];
            o->M0 = sqrtf(s);
        } else {
            for (int i = 0; i < n_g; i++) s += f3[3 * i + 1];
            o->M0 = sqrtf(s * s);
        }
        o->UC = o->UC * 1000.0f;
    } else {
        float s = 0.0f;
        for (int i = 0; i < n_g; i++) s += mo_g[i];
        o->M0 = s;
    }
    int n = 0;
    int *is = (int *)zalloc(sizeof(int) * n_g), *ks = (int *)zalloc(sizeof(int) * n_g);
    int *in = (int *)zalloc(sizeof(int) * n_g);
    for (int i = 0; i < n_g; i++) {
        is[i] = x2i(sx[i], o->xbeg, (float)o->dx);
        ks[i] = x2i(sz[i], o->zbeg, (float)o->dz);
        if (o->ibeg - 2 <= is[i] && is[i] <= o->iend + 3 && o->kbeg - 2 <= ks[i] && ks[i] <= o->kend + 3) { in[i] = 1; n++; }
    }
    o->nsrc = n;
    o->isrc = (int *)zalloc(sizeof(int) * n); o->ksrc = (int *)zalloc(sizeof(int) * n);
    o->srcprm = (float *)zalloc(sizeof(float) * 2 * n);
    o->mo = (MPR *)zalloc(sizeof(MPR) * n); o->mxx = (MPR *)zalloc(sizeof(MPR) * n); o->mzz = (MPR *)zalloc(sizeof(MPR) * n);
    o->mxz = (MPR *)zalloc(sizeof(MPR) * n); o->myz = (MPR *)zalloc(sizeof(MPR) * n); o->mxy = (MPR *)zalloc(sizeof(MPR) * n);
    o->fx = (MPR *)zalloc(sizeof(MPR) * n); o->fy = (MPR *)zalloc(sizeof(MPR) * n); o->fz = (MPR *)zalloc(sizeof(MPR) * n);
    int nn = 0;
    for (int i = 0; i < n_g; i++) {
        if (!in[i]) continue;
        o->isrc[nn] = is[i]; o->ksrc[nn] = ks[i];
        /* sdep_fit = 'bd<n>' (src/swpc_psv/m_source.f90:227-236), inside FDM space (:242-245) */
        if (o->sdep_fit1 > 0) {
            float szb = o->bddep[(is[i] + 2) * (NBD2 + 1) + (o->sdep_fit1 - 1)];
            o->ksrc[nn] = x2i(szb, o->zbeg, (float)o->dz);
            if (!(o->zbeg <= szb && szb <= o->zend)) { free(is); free(ks); free(in); return -1; }
        }
        o->srcprm[2 * nn] = prm[2 * i]; o->srcprm[2 * nn + 1] = prm[2 * i + 1];
        o->mo[nn] = (MPR)(bf_mode ? 0.0f : mo_g[i]);
        o->mxx[nn] = (MPR)m6[6 * i]; o->mzz[nn] = (MPR)m6[6 * i + 2]; o->myz[nn] = (MPR)m6[6 * i + 3];
        o->mxz[nn] = (MPR)m6[6 * i + 4]; o->mxy[nn] = (MPR)m6[6 * i + 5];
        o->fx[nn] = (MPR)f3[3 * i]; o->fy[nn] = (MPR)f3[3 * i + 1]; o->fz[nn] = (MPR)f3[3 * i + 2];
        nn++;
    }
    free(is); free(ks); free(in);
    for (int i = 0; i < n; i++) {
        if (bf_mode) { o->fx[i] = o->fx[i] / o->M0; o->fy[i] = o->fy[i] / o->M0; o->fz[i] = o->fz[i] / o->M0; }
        else o->mo[i] = o->mo[i] / o->M0;
    }
    o->dt_dxz = o->dt / (o->dx * o->dz);
    return n;
}

static void stressglut(o2d *o, int it) {
    if (o->bf_mode) return;
    for (int i = 0; i < o->nsrc; i++) {
        float t = o->tbeg + ((float)it - 0.5f) * o->dt;
        MPR stime = stf(t, o->stftype, o->srcprm[2 * i], o->srcprm[2 * i + 1]);
        MPR sdrop = o->mo[i] * stime * o->dt_dxz;
        int ii = o->isrc[i], kk = o->ksrc[i];
        if (o->kind == 2) {   /* src/swpc_psv/m_source.f90:601-606 */
            A(o->S[0], kk, ii) = A(o->S[0], kk, ii) - o->mxx[i] * sdrop;
            A(o->S[1], kk, ii) = A(o->S[1], kk, ii) - o->mzz[i] * sdrop;
            A(o->S[2], kk, ii) = A(o->S[2], kk, ii) - o->mxz[i] * sdrop / 4;
            A(o->S[2], kk - 1, ii) = A(o->S[2], kk - 1, ii) - o->mxz[i] * sdrop / 4;
            A(o->S[2], kk, ii - 1) = A(o->S[2], kk, ii - 1) - o->mxz[i] * sdrop / 4;
            A(o->S[2], kk - 1, ii - 1) = A(o->S[2], kk - 1, ii - 1) - o->mxz[i] * sdrop / 4;
        } else {              /* src/swpc_sh/m_source.f90:583-587 */
            A(o->S[1], kk, ii) = A(o->S[1], kk, ii) - o->mxy[i] * sdrop / 2;
            A(o->S[1], kk, ii - 1) = A(o->S[1], kk, ii - 1) - o->mxy[i] * sdrop / 2;
            A(o->S[0], kk, ii) = A(o->S[0], kk, ii) - o->myz[i] * sdrop / 2;
            A(o->S[0], kk - 1, ii) = A(o->S[0], kk - 1, ii) - o->myz[i] * sdrop / 2;
        }
    }
}

static void bodyforce(o2d *o, int it) {
    if (!o->bf_mode) return;
    for (int i = 0; i < o->nsrc; i++) {
        MPR stime = stf(o->tbeg + (float)it * o->dt, o->stftype, o->srcprm[2 * i], o->srcprm[2 * i + 1]);
        int ii = o->isrc[i], kk = o->ksrc[i];
        SPR rho = A(o->rho, kk, ii);
        if (o->kind == 2) {   /* src/swpc_psv/m_source.f90:642-645 */
            A(o->V[0], kk, ii) = A(o->V[0], kk, ii) + o->fx[i] / rho * stime * o->dt_dxz / 2;
            A(o->V[0], kk, ii - 1) = A(o->V[0], kk, ii - 1) + o->fx[i] / rho * stime * o->dt_dxz / 2;
            A(o->V[1], kk, ii) = A(o->V[1], kk, ii) + o->fz[i] / rho * stime * o->dt_dxz / 2;
            A(o->V[1], kk - 1, ii) = A(o->V[1], kk - 1, ii) + o->fz[i] / rho * stime * o->dt_dxz / 2;
        } else {              /* src/swpc_sh/m_source.f90:621 */
            A(o->V[0], kk, ii) = A(o->V[0], kk, ii) + o->fy[i] / rho * stime * o->dt_dxz;
        }
    }
}

/* ----------------------------------------------------- stations / vmax */
int o2d_wav_setup(o2d *o, int n_g, const float *xs, const float *zs, const int *zsw, int ntdec_w, int sw_v, int sw_u) {
    o->ntdec_w = ntdec_w; o->sw_v = sw_v; o->sw_u = sw_u;
    o->ntw = (int)floorf((float)(o->nt - 1) / (float)ntdec_w + 1.0f);
    o->ist = (int *)zalloc(sizeof(int) * (n_g ? n_g : 1));
    o->kst = (int *)zalloc(sizeof(int) * (n_g ? n_g : 1));
    int n = 0;
    float ddx = (float)o->dx, ddz = (float)o->dz;
    for (int s = 0; s < n_g; s++) {
        int i = x2i(xs[s], o->xbeg, ddx), k = x2i(zs[s], o->zbeg, ddz);
        if (!(i2x(1, o->xbeg, ddx) < xs[s] && xs[s] < i2x(o->nx, o->xbeg, ddx) && o->kbeg < k && k < o->kend)) continue;
        if (!(o->ibeg <= i && i <= o->iend)) continue;
        if (zsw[s] == 1) k = o->kfs[i + 2] + 1;
        else if (zsw[s] == 2) k = o->kob[i + 2] + 1;
        else if (zsw[s] == 3) k = o->kob[i + 2] - 1;
        else if (zsw[s] >= 10 && zsw[s] <= 10 + NBD2)   /* bd0-bd9 (src/swpc_psv/m_wav.f90:511-520) */
            k = x2i(o->bddep[(i + 2) * (NBD2 + 1) + (zsw[s] - 10)], o->zbeg, ddz);
        else k = x2i(zs[s], o->zbeg, ddz);
        if (k > o->kend) k = o->kend - 1;
        if (k < o->kbeg) k = o->kbeg + 1;
        o->ist[n] = i; o->kst[n] = k; n++;
    }
    o->nst = n;
    int nc = o->kind == 2 ? 2 : 1;
    o->wav_vel = (float *)zalloc(sizeof(float) * (size_t)o->ntw * nc * (n ? n : 1));
    o->wav_disp = (float *)zalloc(sizeof(float) * (size_t)o->ntw * nc * (n ? n : 1));
    o->ux = (SPR *)zalloc(sizeof(SPR) * (n ? n : 1));
    o->uz = (SPR *)zalloc(sizeof(SPR) * (n ? n : 1));
    return n;
}

static void wav_store(o2d *o, int it) {
    if (o->nst == 0) return;
    float dt = o->dt, M0 = o->M0, UC = o->UC;
    int nc = o->kind == 2 ? 2 : 1;
    if (o->sw_u)
        for (int n = 0; n < o->nst; n++) {
            int i = o->ist[n], k = o->kst[n];
            if (o->kind == 2) {   /* src/swpc_psv/m_wav.f90:177-178 */
                o->ux[n] = o->ux[n] + (float)(A(o->V[0], k, i) + A(o->V[0], k, i - 1)) * 0.5f * dt;
                o->uz[n] = o->uz[n] - (float)(A(o->V[1], k, i) + A(o->V[1], k - 1, i)) * 0.5f * dt;
            } else {              /* src/swpc_sh/m_wav.f90:175 */
                o->ux[n] = o->ux[n] + (float)A(o->V[0], k, i) * dt;
            }
        }
    if ((it - 1) % o->ntdec_w != 0) return;
    int itw = (it - 1) / o->ntdec_w + 1;
    for (int n = 0; n < o->nst; n++) {
        int i = o->ist[n], k = o->kst[n];
        float *w = o->wav_vel + (long)n * nc * o->ntw + (itw - 1);
        float *u = o->wav_disp + (long)n * nc * o->ntw + (itw - 1);
        if (o->kind == 2) {
            if (o->sw_v) {
                w[0] = (float)(A(o->V[0], k, i) + A(o->V[0], k, i - 1)) / 2.0f * M0 * UC * 1e9f;
                w[o->ntw] = -(float)(A(o->V[1], k, i) + A(o->V[1], k - 1, i)) / 2.0f * M0 * UC * 1e9f;
            }
            if (o->sw_u) { u[0] = (float)o->ux[n] * M0 * UC * 1e9f; u[o->ntw] = (float)o->uz[n] * M0 * UC * 1e9f; }
        } else {
            if (o->sw_v) w[0] = (float)A(o->V[0], k, i) * M0 * UC * 1e9f;
            if (o->sw_u) u[0] = (float)o->ux[n] * M0 * UC * 1e9f;
        }
    }
}

void o2d_vmax(o2d *o, float *out) {
    float a = 0.0f, b = 0.0f;
    for (int i = o->ibeg_k; i <= o->iend_k; i++) {
        int k = o->kob[i + 2] + 1;
        float x = fabsf((float)A(o->V[0], k, i));
        if (x > a) a = x;
        if (o->kind == 2) { float z = fabsf((float)A(o->V[1], k, i)); if (z > b) b = z; }
    }
    out[0] = a; out[1] = b;
}

/* main loops: src/swpc_psv/main.f90:95-114, src/swpc_sh/main.f90:95-116 */
void o2d_step(o2d *o, int it) {
    wav_store(o, it);
    if (o->kind == 2) {
        psv_update_stress(o); psv_absorb_stress(o); stressglut(o, it); comm_stress(o);
        psv_update_vel(o); bodyforce(o, it); psv_absorb_vel(o); comm_vel(o);
    } else {
        sh_update_stress(o); sh_absorb_stress(o); stressglut(o, it); comm_stress(o);
        sh_update_vel(o); sh_absorb_vel(o); bodyforce(o, it); comm_vel(o);
    }
}

void o2d_dims(const o2d *o, long *out) {
    out[0] = o->nk; out[1] = o->ni; out[2] = o->nka; out[3] = o->kbeg_min; out[4] = o->nst; out[5] = o->ntw;
    out[6] = o->nsrc; out[7] = o->ibeg_k; out[8] = o->iend_k; out[9] = o->kend_k;
}
void o2d_scalars(const o2d *o, float *out) {
    out[0] = o->M0; out[1] = o->UC; out[2] = o->fcut; out[3] = o->vmin; out[4] = o->vmax; out[5] = o->zeta;
    for (int m = 0; m < NM_MAX; m++) out[6 + m] = o->ts[m];
}
int o2d_mpr_size(void) { return (int)sizeof(MPR); }
int o2d_spr_size(void) { return (int)sizeof(SPR); }

/* ids: 0,1 V ; 2..4 S ; 10..12 R (nm, box) ; 20 rho 21 lam 22 mu 23 taup 24 taus (SPR);
 * 30..34 float copies ; 50 kfs 51 kob 52 kfs_top 53 kfs_bot 54 kob_top 55 kob_bot 56 kbeg_a ;
 * 60..67 aux ; 80..83 profiles gxc gxe gzc gze ; 90 wav_vel 91 wav_disp ; 95 ist 96 kst ; 98 isrc 99 ksrc */
void *o2d_ptr(o2d *o, int id) {
    if (id >= 0 && id <= 1) return o->V[id];
    if (id >= 2 && id <= 4) return o->S[id - 2];
    if (id >= 10 && id <= 12) return o->R[id - 10];
    if (id >= 60 && id <= 67) return o->aux[id - 60];
    switch (id) {
    case 20: return o->rho; case 21: return o->lam; case 22: return o->mu; case 23: return o->taup; case 24: return o->taus;
    case 30: return o->frho; case 31: return o->flam; case 32: return o->fmu; case 33: return o->ftaup; case 34: return o->ftaus;
    case 50: return o->kfs; case 51: return o->kob; case 52: return o->kfs_top; case 53: return o->kfs_bot;
    case 54: return o->kob_top; case 55: return o->kob_bot; case 56: return o->kbeg_a;
    case 80: return o->fgxc; case 81: return o->fgxe; case 82: return o->fgzc; case 83: return o->fgze;
    case 110: return o->cgx_c; case 111: return o->cgx_b; case 114: return o->cgz_c; case 115: return o->cgz_b;
    case 90: return o->wav_vel; case 91: return o->wav_disp; case 95: return o->ist; case 96: return o->kst;
    case 98: return o->isrc; case 99: return o->ksrc;
    default: return 0;
    }
}
