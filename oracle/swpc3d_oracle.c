/*
 * swpc3d_oracle.c -- CPU restatement of OpenSWPC's 3D viscoelastic
 * staggered-grid velocity-stress FDM time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: only tests/,
 * the package smoke check and bench.py's cpu_baseline leg load it, and only
 * as the checker / CPU baseline.  The product path never links it.
 *
 * Each routine restates one reference routine, cited as
 * file:line within the OpenSWPC source tree.  The loops keep the reference's
 * index order and its per-variable kinds:
 *     MPR = real(MP) (velocity, stress, FD coefficients, dx)
 *     SPR = real(SP) (memory variables, medium, Zener and PML coefficients)
 * The file is compiled three times:
 *     f32   : MPR = float,  SPR = float   (the MP = SP build)
 *     mixed : MPR = double, SPR = float   (the reference default MP = DP)
 *     f64   : MPR = double, SPR = double  (all-double error reference)
 * Setup arithmetic (medium, Zener relaxation, PML profiles, maps) stays in
 * single precision as in the reference and is promoted when stored.
 *
 * Floating-point expressions are written in the reference's left-to-right
 * evaluation order and the file is compiled with -ffp-contract=off, so the
 * f32 build performs exactly the IEEE single-precision operations that the
 * Fortran source spells out.
 *
 * Parity status: the reference (Fortran + MPI + NetCDF) cannot be compiled
 * here, so this restatement is pinned only by the reference's single
 * recorded run (example/example.out, max surface |V| at 3 significant
 * digits) through the GPU known-answer test; everything else is "parity
 * unpinned" against the reference binary itself.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef MPR
#define MPR float
#endif
#ifndef SPR
#define SPR float
#endif

#define NM_MAX 3
#define NBD 9
static const double PI_D = 3.141592653589793238462643383279502884;

/* ------------------------------------------------------------------------ */
/* model state                                                              */
/* ------------------------------------------------------------------------ */

typedef struct o3d {
    /* parameters (m_global.f90:54-66) */
    int nx, ny, nz, na, nm, nt;
    MPR dx, dy, dz;
    float dt, xbeg, ybeg, zbeg, tbeg, xend, yend, zend;
    float fcut, fmax, vmin, vmax;
    float UC, M0;
    /* ranges (m_global.f90:276-378), single MPI node */
    int ibeg, iend, jbeg, jend, kbeg, kend;
    int ibeg_m, iend_m, jbeg_m, jend_m, kbeg_m, kend_m;
    int ibeg_k, iend_k, jbeg_k, jend_k, kbeg_k, kend_k;
    long nk, ni, nj;            /* memory-box extents */
    long nkk, nik, njk;         /* kernel-region extents (memory variables) */
    float *xc, *yc, *zc;
    int *kbeg_a;
    /* wavefield (m_global.f90:34-38) */
    MPR *Vx, *Vy, *Vz, *Sxx, *Syy, *Szz, *Syz, *Sxz, *Sxy;
    SPR *Rxx, *Ryy, *Rzz, *Ryz, *Rxz, *Rxy;
    /* medium (m_global.f90:39-43): raw vmodel output is kept in float */
    float *frho, *flam, *fmu, *ftaup, *ftaus;      /* setup-time (SP) */
    float *fbx, *fby, *fbz, *fmuyz, *fmuxz, *fmuxy;
    SPR *lam, *mu, *taup, *taus, *bx, *by, *bz, *muyz, *muxz, *muxy;
    float ts[NM_MAX];
    float zeta;
    int *kfs, *kob, *kfs_top, *kfs_bot, *kob_top, *kob_bot;
    float *bddep;               /* (i, j, 0:NBD) */
    int sdep_fit1;              /* sdep_fit: 0 'asis', 1 + n for 'bd<n>' (m_source.f90:99) */
    int munk;                   /* munk_profile of the ocean column (m_vmodel_lhm.f90:53-54) */
    int pw_mode;                /* plane-wave mode (m_source.f90:67-79) */
    /* kernel coefficients (m_kernel.f90:23-26) */
    SPR c1[NM_MAX], c2[NM_MAX], d1[NM_MAX], d2;
    MPR rc40x, rc41x, rc40y, rc41y, rc40z, rc41z;
    MPR rd40x, rd41x, rd40y, rd41y, rd40z, rd41z;
    /* PML (m_absorb_p.f90:43-56) */
    float *fgxc, *fgxe, *fgyc, *fgye, *fgzc, *fgze;
    SPR *gxc, *gxe, *gyc, *gye, *gzc, *gze;
    SPR *axVx, *ayVx, *azVx, *axVy, *ayVy, *azVy, *axVz, *ayVz, *azVz;
    SPR *axSxx, *aySxy, *azSxz, *axSxy, *aySyy, *azSyz, *axSxz, *aySyz, *azSzz;
    MPR r20x, r20y, r20z;
    int kbeg_min;
    /* Cerjan sponge (m_absorb_c.f90:19-20), indexed [i - 1] */
    int cerjan;
    SPR *cgx_c, *cgx_b, *cgy_c, *cgy_b, *cgz_c, *cgz_b;
    int stabilize_pml;          /* input-file switch (m_medium.f90:219) */
    /* green__store (m_green.f90:389-534) */
    int ng, ng_cmp, ng_ntw, ng_ntdec;
    int *gi, *gj, *gk;
    float *gacc;                /* (12, ng) */
    float *gf;                  /* gf(ntw, ncmp*ng), column-major */
    long nka;                   /* PML aux k extent */
    /* sources (m_source.f90:26-36) */
    int bf_mode, stftype, nsrc;
    int *isrc, *jsrc, *ksrc;
    float *srcprm;              /* (2, nsrc) */
    MPR *mo, *mxx, *myy, *mzz, *myz, *mxz, *mxy, *fx, *fy, *fz;
    MPR dt_dxyz;
    /* green's function source (m_green.f90:597-632) */
    int green_mode, green_is_src, gisrc, gjsrc, gksrc;
    float green_fx1, green_fy1, green_fz1, green_tbeg, green_trise;
    float green_dt_dxyz;
    /* stations (m_wav.f90) */
    int nst, ntdec_w, ntw, sw_v, sw_u, sw_stress, sw_strain;
    int *ist, *jst, *kst;
    float *wav_vel, *wav_disp, *wav_stress, *wav_strain;   /* (ntw, ncmp, nst) */
    SPR *ux, *uy, *uz, *exx, *eyy, *ezz, *eyz, *exz, *exy;
    MPR r40x, r40y, r40z, r41x, r41y, r41z;                /* m_wav.f90:130-135 */
    /* snapshots (m_snap.f90:30-90); plane = 3 * section + quantity with
     * sections yz xz xy fs ob and quantities ps v u */
    int snp_planes, idec, jdec, kdec, ntdec_s, i0_yz, j0_xz, k0_xy;
    int nxs, nys, nzs, is0, is1, js0, js1, ks0, ks1, nframes;
    MPR sr20x, sr20y, sr20z;
    float *snp[15];             /* frames (nframes, nvar, n2, n1) */
    float *sbuf[15];            /* current buffer (nvar, n2, n1): the `save` buf of each wbuf_* */
    float *maxv[4];             /* max_fs_v, max_fs_u, max_ob_v, max_ob_u (3, nys, nxs) */
    int threads;
} o3d;

#define IDX3(o, k, i, j) \
    ((((long)(j) - (o)->jbeg_m) * (o)->ni + ((long)(i) - (o)->ibeg_m)) * (o)->nk + ((long)(k) - (o)->kbeg_m))
#define IDX2(o, i, j) (((long)(j) - (o)->jbeg_m) * (o)->ni + ((long)(i) - (o)->ibeg_m))
#define IDXR(o, m, k, i, j)                                                                   \
    (((((long)(j) - (o)->jbeg_k) * (o)->nik + ((long)(i) - (o)->ibeg_k)) * (o)->nkk +           \
      ((long)(k) - (o)->kbeg_k)) * (o)->nm + ((m) - 1))
#define IDXA(o, k, i, j) \
    ((((long)(j) - (o)->jbeg) * (long)((o)->iend - (o)->ibeg + 1) + ((long)(i) - (o)->ibeg)) * (o)->nka + ((long)(k) - (o)->kbeg_min))

#define A3(arr, k, i, j) (arr)[IDX3(o, k, i, j)]
#define A2(arr, i, j) (arr)[IDX2(o, i, j)]

static void *zalloc(size_t n) { return calloc(n ? n : 1, 1); }

/* ------------------------------------------------------------------------ */
/* m_fdtool.f90 helpers                                                     */
/* ------------------------------------------------------------------------ */

/* x2i/y2j/z2k: m_fdtool.f90:600-636 -- ceiling((x - xbeg) / dx) in SP */
int o3d_x2i(float x, float xbeg, float dx) {
    volatile float t = (x - xbeg) / dx;
    return (int)ceilf(t);
}
/* i2x/j2y/k2z: m_fdtool.f90:639-675 -- xbeg + (i - 0.5) * dx in SP */
float o3d_i2x(int i, float xbeg, float dx) {
    volatile float a = (float)i - 0.5f;
    volatile float b = a * dx;
    return xbeg + b;
}

/* Kupper and the other moment-rate functions: m_fdtool.f90:339-497.
 * PI is real(DP) (m_std.f90:14), so mixed expressions promote to double. */
static float stf_kupper(float t, float ts, float tr) {
    if (ts <= t && t <= ts + tr) {
        double s = sin(PI_D * (double)(t - ts) / (double)tr);
        return (float)(3.0 * PI_D * (s * s * s) / (double)(4.0f * tr));
    }
    return 0.0f;
}
static float stf_boxcar(float t, float ts, float tr) {
    if (ts <= t && t <= ts + tr) return 1.0f / tr;
    return 0.0f;
}
static float stf_triangle(float t, float ts, float tr) {
    if (ts <= t && t <= ts + tr / 2) return 4 * (t - ts) / (tr * tr);
    if (ts + tr / 2 < t && t <= ts + tr) return -4 * (t - ts - tr) / (tr * tr);
    return 0.0f;
}
static float stf_herrmann(float t, float ts, float tr) {
    float t1 = ts + tr / 4;
    float t2 = ts + 3 * tr / 4;
    if (ts <= t && t < t1) {
        float a = t - ts;
        return 16 * (a * a) / (tr * tr * tr);
    } else if (t1 <= t && t < t2) {
        return -2 * (8 * (t * t + tr * ts + ts * ts - t * tr - 2 * t * ts) + tr * tr) / (tr * tr * tr);
    } else if (t2 <= t && t <= ts + tr) {
        float a = ts + tr - t;
        return 16 * (a * a) / (tr * tr * tr);
    }
    return 0.0f;
}
static float stf_cosine(float t, float ts, float tr) {
    if (ts <= t && t <= ts + tr) return (float)((1.0 - cos(2 * PI_D * (double)(t - ts) / (double)tr)) / (double)tr);
    return 0.0f;
}
static float stf_texp(float t, float ts, float tr) {
    if (ts <= t) {
        float tt = t - ts;
        double tp = 2 * PI_D;
        return (float)(tp * tp * (double)tt / (double)(tr * tr) * exp(-2 * PI_D * (double)tt / (double)tr));
    }
    return 0.0f;
}
/* stftype codes: 0 kupper, 1 boxcar, 2 triangle, 3 herrmann, 4 cosine, 5 texp */
float o3d_momentrate(float t, int stftype, float ts, float tr) {
    switch (stftype) {
    case 1: return stf_boxcar(t, ts, tr);
    case 2: return stf_triangle(t, ts, tr);
    case 3: return stf_herrmann(t, ts, tr);
    case 4: return stf_cosine(t, ts, tr);
    case 5: return stf_texp(t, ts, tr);
    default: return stf_kupper(t, ts, tr);
    }
}

/* sdr2moment: m_fdtool.f90:307-336 (SP, std__deg2rad in SP) */
void o3d_sdr2moment(float strike, float dip, float rake, float *m6 /* xx yy zz yz xz xy */) {
    const float d2r = (float)(PI_D / 180.0);
    float sind = sinf(dip * d2r), cosd = cosf(dip * d2r);
    float sin2d = sinf((2 * dip) * d2r), cos2d = cosf((2 * dip) * d2r);
    float sinl = sinf(rake * d2r), cosl = cosf(rake * d2r);
    float sinf_ = sinf(strike * d2r), cosf_ = cosf(strike * d2r);
    float sin2f = sinf((2 * strike) * d2r), cos2f = cosf((2 * strike) * d2r);
    float mxx = -(sind * cosl * sin2f + sin2d * sinl * sinf_ * sinf_);
    float mxy = (sind * cosl * cos2f + sin2d * sinl * sin2f / 2);
    float mxz = -(cosd * cosl * cosf_ + cos2d * sinl * sinf_);
    float myy = (sind * cosl * sin2f - sin2d * sinl * cosf_ * cosf_);
    float myz = -(cosd * cosl * sinf_ - cos2d * sinl * cosf_);
    float mzz = (sin2d * sinl);
    m6[0] = mxx; m6[1] = myy; m6[2] = mzz; m6[3] = myz; m6[4] = mxz; m6[5] = mxy;
}

/* visco_set_relaxtime: m_fdtool.f90:691-727 */
void o3d_visco_set_relaxtime(int nm, float *ts, float fmin, float fmax) {
    float omega_a = (float)(2 * PI_D * (double)fmin);
    float omega_b = (float)(2 * PI_D * (double)fmax);
    if (nm == 1) {
        float omega = sqrtf(omega_a * omega_b);
        ts[0] = 1.0f / omega;
    } else if (nm > 1) {
        for (int im = 1; im <= nm; im++) {
            float ratio = omega_b / omega_a;
            double p = pow((double)ratio, (double)(im - 1) / (double)(nm - 1));
            float omega = (float)((double)omega_a * p);
            ts[im - 1] = 1.0f / omega;
        }
    }
}

/* visco_constq_zeta: m_fdtool.f90:756-812 (SP arithmetic) */
float o3d_visco_constq_zeta(int nm, float fmin, float fmax, const float *ts) {
    if (nm == 0) return 0.0f;
    float om_a = (float)(2 * PI_D * (double)fmin);
    float om_b = (float)(2 * PI_D * (double)fmax);
    float i0[NM_MAX], i1[NM_MAX], i2[NM_MAX][NM_MAX];
    for (int im = 0; im < nm; im++) {
        float t = ts[im];
        float a = logf(1.0f + (om_b * om_b) * (t * t));
        float b = logf(1.0f + (om_a * om_a) * (t * t));
        i0[im] = (a - b) / (2 * t);
        float p = atanf(om_b * t) - om_b * t / (1 + (om_b * om_b) * (t * t));
        float q = atanf(om_a * t) - om_a * t / (1 + (om_a * om_a) * (t * t));
        i1[im] = (p - q) / (2 * t);
    }
    for (int im = 0; im < nm - 1; im++) {
        for (int km = im + 1; km < nm; km++) {
            float wk1 = atanf(om_b * ts[im]) / ts[im] - atanf(om_b * ts[km]) / ts[km];
            float wk2 = atanf(om_a * ts[im]) / ts[im] - atanf(om_a * ts[km]) / ts[km];
            i2[km][im] = ts[im] * ts[km] / (ts[km] * ts[km] - ts[im] * ts[im]) * (wk1 - wk2);
        }
    }
    float i0sum = 0.0f, i1sum = 0.0f, i2sum = 0.0f;
    for (int im = 0; im < nm; im++) i0sum += i0[im];
    for (int im = 0; im < nm; im++) i1sum += i1[im];
    for (int im = 0; im < nm - 1; im++)
        for (int km = im + 1; km < nm; km++) i2sum = i2sum + i2[km][im];
    return i0sum / (i1sum + 2 * i2sum);
}

/* vcheck: m_fdtool.f90:15-48 */
static void vcheck(float *vp, float *vs, float *rho, float xi, float vmin, float vmax, float rhomin) {
    float gamma = *vp / *vs;
    if (gamma < 1.1920929e-07f) gamma = sqrtf(3.0f);
    if (*vp > vmax || *vs > vmax) {
        float xi2 = (1 + xi) * vmax / *vp - 1;
        *vp = vmax;
        *vs = vmax / gamma;
        *rho = *rho * (1 + 0.8f * xi2) / (1 + 0.8f * xi);
    }
    if (*vp < vmin || *vs < vmin) {
        *vs = vmin;
        *vp = vmin * gamma;
    }
    if (*rho < rhomin) *rho = rhomin;
}

/* ------------------------------------------------------------------------ */
/* create / ranges: m_global.f90:221-378 (nproc = 1)                        */
/* ------------------------------------------------------------------------ */

o3d *o3d_create(int nx, int ny, int nz, int na, int nm, int nt, double dx, double dy, double dz, float dt,
                float xbeg, float ybeg, float zbeg, float tbeg, int threads) {
    o3d *o = (o3d *)zalloc(sizeof(o3d));
    o->nx = nx; o->ny = ny; o->nz = nz; o->na = na; o->nm = nm; o->nt = nt;
    o->dx = (MPR)dx; o->dy = (MPR)dy; o->dz = (MPR)dz; o->dt = dt;
    o->xbeg = xbeg; o->ybeg = ybeg; o->zbeg = zbeg; o->tbeg = tbeg;
    o->threads = threads;
    /* global__setup: m_global.f90:205-208 */
    o->xend = xbeg + nx * (float)o->dx;
    o->yend = ybeg + ny * (float)o->dy;
    o->zend = zbeg + nz * (float)o->dz;
    o->UC = 1.0e-15f;
    o->M0 = 1.0f;
    o->ibeg = 1; o->iend = nx; o->jbeg = 1; o->jend = ny; o->kbeg = 1; o->kend = nz;
    o->ibeg_m = o->ibeg - 3; o->iend_m = o->iend + 3;
    o->jbeg_m = o->jbeg - 3; o->jend_m = o->jend + 3;
    o->kbeg_m = o->kbeg - 3; o->kend_m = o->kend + 3;
    o->nk = o->kend_m - o->kbeg_m + 1;
    o->ni = o->iend_m - o->ibeg_m + 1;
    o->nj = o->jend_m - o->jbeg_m + 1;
    o->xc = (float *)zalloc(sizeof(float) * o->ni);
    o->yc = (float *)zalloc(sizeof(float) * o->nj);
    o->zc = (float *)zalloc(sizeof(float) * o->nk);
    for (int i = o->ibeg_m; i <= o->iend_m; i++) o->xc[i - o->ibeg_m] = o3d_i2x(i, xbeg, (float)o->dx);
    for (int j = o->jbeg_m; j <= o->jend_m; j++) o->yc[j - o->jbeg_m] = o3d_i2x(j, ybeg, (float)o->dy);
    for (int k = o->kbeg_m; k <= o->kend_m; k++) o->zc[k - o->kbeg_m] = o3d_i2x(k, zbeg, (float)o->dz);
    /* absorber map kbeg_a: m_global.f90:336-345 */
    o->kbeg_a = (int *)zalloc(sizeof(int) * o->ni * o->nj);
    for (int j = o->jbeg_m; j <= o->jend_m; j++)
        for (int i = o->ibeg_m; i <= o->iend_m; i++) {
            if (i <= na || nx - na + 1 <= i || j <= na || ny - na + 1 <= j) A2(o->kbeg_a, i, j) = o->kbeg;
            else A2(o->kbeg_a, i, j) = o->kend - na + 1;
        }
    /* kernel region: m_global.f90:349-378 (abc_type = 'pml') */
    o->ibeg_k = o->ibeg; o->iend_k = o->iend; o->jbeg_k = o->jbeg; o->jend_k = o->jend;
    o->kbeg_k = o->kbeg; o->kend_k = o->kend;
    if (o->iend <= na) o->ibeg_k = o->iend + 1;
    else if (o->ibeg <= na) o->ibeg_k = na + 1;
    if (o->ibeg >= nx - na + 1) o->iend_k = o->ibeg - 1;
    else if (o->iend >= nx - na + 1) o->iend_k = nx - na;
    if (o->jend <= na) o->jbeg_k = o->jend + 1;
    else if (o->jbeg <= na) o->jbeg_k = na + 1;
    if (o->jbeg >= ny - na + 1) o->jend_k = o->jbeg - 1;
    else if (o->jend >= ny - na + 1) o->jend_k = ny - na;
    o->kend_k = nz - na;
    o->nkk = o->kend_k - o->kbeg_k + 1;
    o->nik = o->iend_k - o->ibeg_k + 1;
    o->njk = o->jend_k - o->jbeg_k + 1;

    long n3 = o->nk * o->ni * o->nj, n2 = o->ni * o->nj;
#define AL(p, T, n) p = (T *)zalloc(sizeof(T) * (size_t)(n))
    AL(o->Vx, MPR, n3); AL(o->Vy, MPR, n3); AL(o->Vz, MPR, n3);
    AL(o->Sxx, MPR, n3); AL(o->Syy, MPR, n3); AL(o->Szz, MPR, n3);
    AL(o->Syz, MPR, n3); AL(o->Sxz, MPR, n3); AL(o->Sxy, MPR, n3);
    long nr = (long)nm * o->nkk * o->nik * o->njk;
    if (nr < 0) nr = 0;
    AL(o->Rxx, SPR, nr); AL(o->Ryy, SPR, nr); AL(o->Rzz, SPR, nr);
    AL(o->Ryz, SPR, nr); AL(o->Rxz, SPR, nr); AL(o->Rxy, SPR, nr);
    AL(o->frho, float, n3); AL(o->flam, float, n3); AL(o->fmu, float, n3);
    AL(o->ftaup, float, n3); AL(o->ftaus, float, n3);
    AL(o->fbx, float, n3); AL(o->fby, float, n3); AL(o->fbz, float, n3);
    AL(o->fmuyz, float, n3); AL(o->fmuxz, float, n3); AL(o->fmuxy, float, n3);
    AL(o->lam, SPR, n3); AL(o->mu, SPR, n3); AL(o->taup, SPR, n3); AL(o->taus, SPR, n3);
    AL(o->bx, SPR, n3); AL(o->by, SPR, n3); AL(o->bz, SPR, n3);
    AL(o->muyz, SPR, n3); AL(o->muxz, SPR, n3); AL(o->muxy, SPR, n3);
    AL(o->kfs, int, n2); AL(o->kob, int, n2); AL(o->kfs_top, int, n2); AL(o->kfs_bot, int, n2);
    AL(o->kob_top, int, n2); AL(o->kob_bot, int, n2);
    AL(o->bddep, float, n2 * (NBD + 1));
#undef AL
    return o;
}

void o3d_destroy(o3d *o) {
    if (!o) return;
    void *ps[] = {o->xc, o->yc, o->zc, o->kbeg_a, o->Vx, o->Vy, o->Vz, o->Sxx, o->Syy, o->Szz, o->Syz, o->Sxz,
                  o->Sxy, o->Rxx, o->Ryy, o->Rzz, o->Ryz, o->Rxz, o->Rxy, o->frho, o->flam, o->fmu, o->ftaup,
                  o->ftaus, o->fbx, o->fby, o->fbz, o->fmuyz, o->fmuxz, o->fmuxy, o->lam, o->mu, o->taup,
                  o->taus, o->bx, o->by, o->bz, o->muyz, o->muxz, o->muxy, o->kfs, o->kob, o->kfs_top,
                  o->kfs_bot, o->kob_top, o->kob_bot, o->bddep, o->fgxc, o->fgxe, o->fgyc, o->fgye, o->fgzc,
                  o->fgze, o->gxc, o->gxe, o->gyc, o->gye, o->gzc, o->gze, o->axVx, o->ayVx, o->azVx, o->axVy,
                  o->ayVy, o->azVy, o->axVz, o->ayVz, o->azVz, o->axSxx, o->aySxy, o->azSxz, o->axSxy,
                  o->aySyy, o->azSyz, o->axSxz, o->aySyz, o->azSzz, o->isrc, o->jsrc, o->ksrc, o->srcprm,
                  o->mo, o->mxx, o->myy, o->mzz, o->myz, o->mxz, o->mxy, o->fx, o->fy, o->fz, o->ist, o->jst,
                  o->kst, o->wav_vel, o->wav_disp, o->wav_stress, o->wav_strain, o->ux, o->uy, o->uz,
                  o->exx, o->eyy, o->ezz, o->eyz, o->exz, o->exy, o->cgx_c, o->cgx_b, o->cgy_c, o->cgy_b,
                  o->cgz_c, o->cgz_b, o->gi, o->gj, o->gk, o->gacc, o->gf};
    for (size_t n = 0; n < sizeof(ps) / sizeof(ps[0]); n++) free(ps[n]);
    for (int q = 0; q < 15; q++) { free(o->snp[q]); free(o->sbuf[q]); }
    for (int q = 0; q < 4; q++) free(o->maxv[q]);
    free(o);
}

/* ------------------------------------------------------------------------ */
/* vmodel_lhm / vmodel_lhm_rmed: m_vmodel_lhm.f90:21-169,                   */
/* m_vmodel_lhm_rmed.f90:84-227 (no ocean column, no earth flattening)      */
/* xi: optional perturbation over the memory box (NULL = lhm)               */
/* ------------------------------------------------------------------------ */
/* seawater__vel: src/shared/m_seawater.f90:19-49 (Munk's profile in DP; eps = 0 gives 1.5 km/s) */
float o3d_seawater_vel(float z, int munk) {
    double eps = munk ? 0.00737 : 0.0;
    double zc = 1300.0;
    double zb = 2 * ((double)z * 1000. - zc) / zc;
    return (float)(1.5 * (1.0 + eps * (zb - 1.0 + exp(-zb))));
}

/* munk_profile switch of the ocean column; set before o3d_vmodel_lhm */
void o3d_set_munk(o3d *o, int munk) { o->munk = munk; }

void o3d_vmodel_lhm(o3d *o, int nlayer, const float *depth, const float *rho0_in, const float *vp0_in,
                    const float *vs0_in, const float *qp0_in, const float *qs0_in, float vcut, const float *xi,
                    float rhomin, float *qp, float *qs) {
    float *rho0 = (float *)zalloc(sizeof(float) * nlayer), *vp0 = (float *)zalloc(sizeof(float) * nlayer);
    float *vs0 = (float *)zalloc(sizeof(float) * nlayer), *q0p = (float *)zalloc(sizeof(float) * nlayer);
    float *q0s = (float *)zalloc(sizeof(float) * nlayer);
    memcpy(rho0, rho0_in, sizeof(float) * nlayer); memcpy(vp0, vp0_in, sizeof(float) * nlayer);
    memcpy(vs0, vs0_in, sizeof(float) * nlayer); memcpy(q0p, qp0_in, sizeof(float) * nlayer);
    memcpy(q0s, qs0_in, sizeof(float) * nlayer);
    /* velocity cut-off: m_vmodel_lhm.f90:93-101 */
    for (int l = nlayer - 2; l >= 0; l--) {
        if ((vp0[l] < vcut || vs0[l] < vcut) && (vp0[l] > 0 && vs0[l] > 0)) {
            vp0[l] = vp0[l + 1]; vs0[l] = vs0[l + 1]; rho0[l] = rho0[l + 1];
            q0p[l] = q0p[l + 1]; q0s[l] = q0s[l + 1];
        }
    }
    /* lhm_rmed velocity bounds: m_vmodel_lhm_rmed.f90:95-98 */
    float vmin_r = vcut;
    float ddx = (float)o->dx, ddy = (float)o->dy, ddz = (float)o->dz;
    float dh = 1.0f / sqrtf(1.0f / (ddx * ddx) + 1.0f / (ddy * ddy) + 1.0f / (ddz * ddz));
    float cc = 6.0f / 7.0f;
    float vmax_r = cc * dh / o->dt;
    for (int j = o->jbeg_m; j <= o->jend_m; j++)
        for (int i = o->ibeg_m; i <= o->iend_m; i++) {
            o->bddep[IDX2(o, i, j) * (NBD + 1) + 0] = depth[0];
            for (int n = 1; n <= NBD; n++) o->bddep[IDX2(o, i, j) * (NBD + 1) + n] = -9999.0f;
        }
    for (int k = o->kbeg_m; k <= o->kend_m; k++) {
        float zs = o->zc[k - o->kbeg_m];
        if (zs < depth[0]) {
            /* air column (zs < 0) or seawater (0 <= zs < depth(1)): m_vmodel_lhm.f90:108-138 */
            float vpw = 1.0f * o3d_seawater_vel(zs, o->munk);
            for (int j = o->jbeg_m; j <= o->jend_m; j++)
                for (int i = o->ibeg_m; i <= o->iend_m; i++) {
                    long e = IDX3(o, k, i, j);
                    if (zs < 0.0f) {
                        o->frho[e] = 0.001f; o->fmu[e] = 0.0f; o->flam[e] = 0.0f;
                        qp[e] = 10.0f; qs[e] = 10.0f;
                    } else {
                        o->frho[e] = 1.0f; o->fmu[e] = 0.0f; o->flam[e] = 1.0f * vpw * vpw;
                        qp[e] = 1000000.0f; qs[e] = 1000000.0f;
                    }
                }
            continue;
        }
        for (int j = o->jbeg_m; j <= o->jend_m; j++)
            for (int i = o->ibeg_m; i <= o->iend_m; i++) {
                long e = IDX3(o, k, i, j);
                float rho1 = 0, vp1 = 0, vs1 = 0, qp1 = 0, qs1 = 0;
                for (int l = 0; l < nlayer; l++) {
                    if (zs >= depth[l]) {
                        if (xi) {
                            float x = xi[e];
                            rho1 = rho0[l] * (1 + 0.8f * x);
                            vp1 = 1.0f * vp0[l] * (1 + x);
                            vs1 = 1.0f * vs0[l] * (1 + x);
                            if (vp0[l] > 0 && vs0[l] > 0) vcheck(&vp1, &vs1, &rho1, x, vmin_r, vmax_r, rhomin);
                        } else {
                            rho1 = rho0[l];
                            vp1 = 1.0f * vp0[l];
                            vs1 = 1.0f * vs0[l];
                        }
                        qp1 = q0p[l];
                        qs1 = q0s[l];
                    }
                }
                o->frho[e] = rho1;
                o->fmu[e] = rho1 * vs1 * vs1;
                o->flam[e] = rho1 * (vp1 * vp1 - 2 * vs1 * vs1);
                qp[e] = qp1;
                qs[e] = qs1;
            }
    }
    free(rho0); free(vp0); free(vs0); free(q0p); free(q0s);
}

/* ------------------------------------------------------------------------ */
/* medium__setup after the vmodel: m_medium.f90:124-225, 234-274, 342-465   */
/* taup_in/taus_in hold Qp/Qs on entry (vmodel output).                     */
/* ------------------------------------------------------------------------ */
void o3d_medium_setup(o3d *o, const float *qp, const float *qs, float fq_min, float fq_max, float fq_ref) {
    int na = o->na, nx = o->nx, ny = o->ny, nz = o->nz;
    float *rho = o->frho, *lam = o->flam, *mu = o->fmu, *taup = o->ftaup, *taus = o->ftaus;
    long n3 = o->nk * o->ni * o->nj;
    memcpy(taup, qp, sizeof(float) * n3);
    memcpy(taus, qs, sizeof(float) * n3);
    /* homogenize absorber region: m_medium.f90:124-190 */
    for (int i = o->ibeg_m; i <= na; i++)
        for (int j = o->jbeg_m; j <= o->jend_m; j++)
            for (int k = o->kbeg_m; k <= o->kend_m; k++) {
                long d = IDX3(o, k, i, j), s = IDX3(o, k, na + 1, j);
                rho[d] = rho[s]; lam[d] = lam[s]; mu[d] = mu[s]; taup[d] = taup[s]; taus[d] = taus[s];
            }
    for (int i = nx - na + 1; i <= o->iend_m; i++)
        for (int j = o->jbeg_m; j <= o->jend_m; j++)
            for (int k = o->kbeg_m; k <= o->kend_m; k++) {
                long d = IDX3(o, k, i, j), s = IDX3(o, k, nx - na, j);
                rho[d] = rho[s]; lam[d] = lam[s]; mu[d] = mu[s]; taup[d] = taup[s]; taus[d] = taus[s];
            }
    for (int j = o->jbeg_m; j <= na; j++)
        for (int i = o->ibeg_m; i <= o->iend_m; i++)
            for (int k = o->kbeg_m; k <= o->kend_m; k++) {
                long d = IDX3(o, k, i, j), s = IDX3(o, k, i, na + 1);
                rho[d] = rho[s]; lam[d] = lam[s]; mu[d] = mu[s]; taup[d] = taup[s]; taus[d] = taus[s];
            }
    for (int j = ny - na + 1; j <= o->jend_m; j++)
        for (int i = o->ibeg_m; i <= o->iend_m; i++)
            for (int k = o->kbeg_m; k <= o->kend_m; k++) {
                long d = IDX3(o, k, i, j), s = IDX3(o, k, i, ny - na);
                rho[d] = rho[s]; lam[d] = lam[s]; mu[d] = mu[s]; taup[d] = taup[s]; taus[d] = taus[s];
            }
    for (int j = o->jbeg_m; j <= o->jend_m; j++)
        for (int i = o->ibeg_m; i <= o->iend_m; i++)
            for (int k = nz - na + 1; k <= o->kend_m; k++) {
                long d = IDX3(o, k, i, j), s = IDX3(o, nz - na, i, j);
                rho[d] = rho[s]; lam[d] = lam[s]; mu[d] = mu[s]; taup[d] = taup[s]; taus[d] = taus[s];
            }
    /* tau-method: m_medium.f90:193-207 */
    o3d_visco_set_relaxtime(o->nm, o->ts, fq_min, fq_max);
    float zeta = o3d_visco_constq_zeta(o->nm, fq_min, fq_max, o->ts);
    o->zeta = zeta;
    for (long e = 0; e < n3; e++) {
        taup[e] = o->nm * zeta / taup[e];
        taus[e] = o->nm * zeta / taus[e];
    }
    /* relaxed_medium: m_medium.f90:234-274.  Complex SP arithmetic written
     * out: cc = sum_m (i w ts)/(1 - i w ts) / nm. */
    if (o->nm > 0) {
        float omega = (float)(2 * PI_D * (double)fq_ref);
        float ccr = 0.0f, cci = 0.0f;
        for (int im = 0; im < o->nm; im++) {
            /* (i a) / (1 - i a) = (-a^2 + i a) / (1 + a^2), a = omega*ts, in DP */
            double a = (double)omega * (double)o->ts[im];
            double den = 1.0 + a * a;
            ccr = ccr + (float)(-(a * a) / den);
            cci = cci + (float)(a / den);
        }
        ccr = ccr / o->nm;
        cci = cci / o->nm;
        for (long e = 0; e < n3; e++) {
            float rho_beta2 = mu[e];
            float rho_alpha2 = lam[e] + 2 * mu[e];
            float chi[2];
            float tt[2] = {taus[e], taup[e]};
            for (int q = 0; q < 2; q++) {
                /* z = 1 - cc * tau ; w = sqrt(z) ; chi = 1 / Re(1 / w) */
                float zr = 1.0f - ccr * tt[q];
                float zi = 0.0f - cci * tt[q];
                /* principal square root for Re z > 0: r = sqrt((|z| + x)/2), s = y / (2 r) */
                float wr = sqrtf(0.5f * (hypotf(zr, zi) + zr));
                float wi = 0.5f * (zi / wr);
                /* Re(1 / w) with the unscaled quotient used under -ffast-math */
                float re_inv = wr / (wr * wr + wi * wi);
                chi[q] = 1.0f / re_inv;
            }
            float chi_mu = chi[0], chi_lam = chi[1];
            mu[e] = rho_beta2 / (chi_mu * chi_mu);
            lam[e] = rho_alpha2 / (chi_lam * chi_lam) - 2 * mu[e];
        }
    }
    /* surface_detection: m_medium.f90:342-397 */
    const float epsl = 1.1920929e-07f;
    for (int j = o->jbeg_m; j <= o->jend_m; j++)
        for (int i = o->ibeg_m; i <= o->iend_m; i++) {
            A2(o->kfs, i, j) = o->kbeg - 1;
            A2(o->kob, i, j) = o->kbeg - 1;
        }
    for (int j = o->jbeg - 1; j <= o->jend + 2; j++)
        for (int i = o->ibeg - 1; i <= o->iend + 2; i++)
            for (int k = o->kbeg; k <= o->kend - 1; k++) {
                if (fabsf(A3(mu, k, i, j)) < epsl && fabsf(A3(mu, k + 1, i, j)) > epsl) A2(o->kob, i, j) = k;
                if (fabsf(A3(lam, k, i, j)) < epsl && fabsf(A3(lam, k + 1, i, j)) > epsl) A2(o->kfs, i, j) = k;
            }
    for (int j = o->jbeg; j <= o->jend; j++)
        for (int i = o->ibeg; i <= o->iend; i++) {
            int fmin = 1 << 30, fmax = -(1 << 30), bmin = 1 << 30, bmax = -(1 << 30);
            for (int jj = j - 2; jj <= j + 3; jj++)
                for (int ii = i - 2; ii <= i + 3; ii++) {
                    int f = A2(o->kfs, ii, jj), b = A2(o->kob, ii, jj);
                    if (f < fmin) fmin = f;
                    if (f > fmax) fmax = f;
                    if (b < bmin) bmin = b;
                    if (b > bmax) bmax = b;
                }
            A2(o->kfs_top, i, j) = (fmin - 2 > o->kbeg) ? fmin - 2 : o->kbeg;
            A2(o->kfs_bot, i, j) = (fmax + 2 < o->kend) ? fmax + 2 : o->kend;
            A2(o->kob_top, i, j) = (bmin - 2 > o->kbeg) ? bmin - 2 : o->kbeg;
            A2(o->kob_bot, i, j) = (bmax + 2 < o->kend) ? bmax + 2 : o->kend;
        }
    /* velocity_minmax: m_medium.f90:399-430 */
    float vmax1 = -1, vmin1 = 1e30f;
    for (int j = o->jbeg; j <= o->jend; j++)
        for (int i = o->ibeg; i <= o->iend; i++)
            for (int k = A2(o->kfs, i, j) + 1; k <= o->kend; k++) {
                long e = IDX3(o, k, i, j);
                float vp = sqrtf((lam[e] + 2 * mu[e]) / rho[e]);
                float vs = sqrtf(mu[e] / rho[e]);
                if (vp > vmax1) vmax1 = vp;
                if (vs < epsl) continue;
                if (vs < vmin1) vmin1 = vs;
            }
    o->vmax = vmax1;
    o->vmin = vmin1;
    /* stabilize_absorber: m_medium.f90:219-222, 276-340 */
    if (o->stabilize_pml) {
        const float vmin_pml = vmax1 * 0.4f;
        for (int j = o->jbeg - 1; j <= o->jend + 1; j++)
            for (int i = o->ibeg - 1; i <= o->iend + 1; i++) {
                int k0 = 1 << 30;
                for (int jj = j - 2; jj <= j + 2; jj++)
                    for (int ii = i - 2; ii <= i + 2; ii++)
                        if (A2(o->kbeg_a, ii, jj) < k0) k0 = A2(o->kbeg_a, ii, jj);
                int k = k0;
                while (k <= o->kend) {
                    long e = IDX3(o, k, i, j), u = IDX3(o, k - 1, i, j);
                    if (lam[e] < lam[u] || mu[e] < mu[u]) {
                        int k2;
                        for (k2 = k + 1; k2 <= o->kend; k2++)
                            if (A3(lam, k2, i, j) > A3(lam, k2 - 1, i, j) || A3(mu, k2, i, j) > A3(mu, k2 - 1, i, j))
                                break;
                        if (k2 - k <= 20) {
                            rho[e] = rho[u]; lam[e] = lam[u]; mu[e] = mu[u]; taup[e] = taup[u]; taus[e] = taus[u];
                            k = k2 - 1;
                        }
                    }
                    k = k + 1;
                }
                for (k = k0; k <= o->kend; k++) {
                    long e = IDX3(o, k, i, j);
                    float vp = sqrtf((lam[e] + 2 * mu[e]) / rho[e]);
                    float vs = sqrtf(mu[e] / rho[e]);
                    if (vs < epsl) continue;
                    float gamma = sqrtf(3.0f);
                    if (vs < vmin_pml) {
                        vs = vmin_pml;
                        vp = vs * gamma;
                        lam[e] = rho[e] * (vp * vp - 2 * (vs * vs));
                        mu[e] = rho[e] * (vs * vs);
                    }
                }
            }
    }
    /* averaged_medium: m_medium.f90:432-465 */
    for (int j = o->jbeg; j <= o->jend; j++)
        for (int i = o->ibeg; i <= o->iend; i++)
            for (int k = o->kbeg; k <= o->kend; k++) {
                long e = IDX3(o, k, i, j);
                o->fbx[e] = 2.0f / (rho[e] + A3(rho, k, i + 1, j));
                o->fby[e] = 2.0f / (rho[e] + A3(rho, k, i, j + 1));
                o->fbz[e] = 2.0f / (rho[e] + A3(rho, k + 1, i, j));
                float nnn = mu[e], pnn = A3(mu, k + 1, i, j), npn = A3(mu, k, i + 1, j);
                float ppn = A3(mu, k + 1, i + 1, j), nnp = A3(mu, k, i, j + 1);
                float npp = A3(mu, k, i + 1, j + 1), pnp = A3(mu, k + 1, i, j + 1);
                o->fmuxz[e] = 4 * nnn * pnn * npn * ppn /
                              (nnn * pnn * npn + nnn * pnn * ppn + nnn * npn * ppn + pnn * npn * ppn + epsl);
                o->fmuxy[e] = 4 * nnn * npn * nnp * npp /
                              (nnn * npn * nnp + nnn * npn * npp + nnn * nnp * npp + npn * nnp * npp + epsl);
                o->fmuyz[e] = 4 * nnn * pnn * nnp * pnp /
                              (nnn * pnn * nnp + nnn * pnn * pnp + nnn * nnp * pnp + pnn * nnp * pnp + epsl);
            }
    /* promote to the kernel kinds */
    for (long e = 0; e < n3; e++) {
        o->lam[e] = (SPR)lam[e]; o->mu[e] = (SPR)mu[e]; o->taup[e] = (SPR)taup[e]; o->taus[e] = (SPR)taus[e];
        o->bx[e] = (SPR)o->fbx[e]; o->by[e] = (SPR)o->fby[e]; o->bz[e] = (SPR)o->fbz[e];
        o->muyz[e] = (SPR)o->fmuyz[e]; o->muxz[e] = (SPR)o->fmuxz[e]; o->muxy[e] = (SPR)o->fmuxy[e];
    }
}

/* Replace the derived medium with externally prepared arrays (memory-box,
 * Fortran order).  Used to feed the oracle and the GPU identical inputs. */
void o3d_set_medium(o3d *o, const float *lam, const float *mu, const float *taup, const float *taus,
                    const float *bx, const float *by, const float *bz, const float *muyz, const float *muxz,
                    const float *muxy, const float *ts) {
    long n3 = o->nk * o->ni * o->nj;
    for (long e = 0; e < n3; e++) {
        o->flam[e] = lam[e]; o->fmu[e] = mu[e]; o->ftaup[e] = taup[e]; o->ftaus[e] = taus[e];
        o->fbx[e] = bx[e]; o->fby[e] = by[e]; o->fbz[e] = bz[e];
        o->fmuyz[e] = muyz[e]; o->fmuxz[e] = muxz[e]; o->fmuxy[e] = muxy[e];
        o->lam[e] = (SPR)lam[e]; o->mu[e] = (SPR)mu[e]; o->taup[e] = (SPR)taup[e]; o->taus[e] = (SPR)taus[e];
        o->bx[e] = (SPR)bx[e]; o->by[e] = (SPR)by[e]; o->bz[e] = (SPR)bz[e];
        o->muyz[e] = (SPR)muyz[e]; o->muxz[e] = (SPR)muxz[e]; o->muxy[e] = (SPR)muxy[e];
    }
    for (int m = 0; m < o->nm; m++) o->ts[m] = ts[m];
}

void o3d_set_maps(o3d *o, const int *kfs, const int *kob, const int *kfs_top, const int *kfs_bot,
                  const int *kob_top, const int *kob_bot) {
    long n2 = o->ni * o->nj;
    memcpy(o->kfs, kfs, sizeof(int) * n2); memcpy(o->kob, kob, sizeof(int) * n2);
    memcpy(o->kfs_top, kfs_top, sizeof(int) * n2); memcpy(o->kfs_bot, kfs_bot, sizeof(int) * n2);
    memcpy(o->kob_top, kob_top, sizeof(int) * n2); memcpy(o->kob_bot, kob_bot, sizeof(int) * n2);
}

/* ------------------------------------------------------------------------ */
/* kernel__setup: m_kernel.f90:30-73                                        */
/* ------------------------------------------------------------------------ */
void o3d_kernel_setup(o3d *o) {
    o->rc40x = (MPR)17.0 / (MPR)16.0 / o->dx; o->rc40y = (MPR)17.0 / (MPR)16.0 / o->dy;
    o->rc40z = (MPR)17.0 / (MPR)16.0 / o->dz;
    o->rc41x = (MPR)1.0 / (MPR)48.0 / o->dx; o->rc41y = (MPR)1.0 / (MPR)48.0 / o->dy;
    o->rc41z = (MPR)1.0 / (MPR)48.0 / o->dz;
    o->rd40x = (MPR)-1.0 / (MPR)16.0 / o->dx; o->rd40y = (MPR)-1.0 / (MPR)16.0 / o->dy;
    o->rd40z = (MPR)-1.0 / (MPR)16.0 / o->dz;
    o->rd41x = (MPR)-1.0 / (MPR)48.0 / o->dx; o->rd41y = (MPR)-1.0 / (MPR)48.0 / o->dy;
    o->rd41z = (MPR)-1.0 / (MPR)48.0 / o->dz;
    if (o->nm > 0) {
        /* c1, c2, d1, d2 are real(SP); ts and dt are real(SP) */
        float fc1[NM_MAX], fc2[NM_MAX], fd1[NM_MAX], fd2 = 0.0f;
        float dt = o->dt;
        for (int m = 0; m < o->nm; m++) {
            fc1[m] = (2 * o->ts[m] - dt) / (2 * o->ts[m] + dt);
            fc2[m] = (2) / (2 * o->ts[m] + dt) / o->nm;
        }
        for (int m = 0; m < o->nm; m++) fd2 = fd2 + dt / (2 * o->ts[m] - dt);
        fd2 = fd2 / o->nm;
        for (int m = 0; m < o->nm; m++) fd1[m] = 2 * o->ts[m] / (2 * o->ts[m] - dt);
        for (int m = 0; m < o->nm; m++) { o->c1[m] = fc1[m]; o->c2[m] = fc2[m]; o->d1[m] = fd1[m]; }
        o->d2 = fd2;
    }
}

/* ------------------------------------------------------------------------ */
/* absorb_p__setup + damping_profile: m_absorb_p.f90:60-124, 507-547         */
/* ------------------------------------------------------------------------ */
static void damping_profile(float x, float H, float xbeg0, float xend0, int na, float fcut, float dt, float *g) {
    float R0 = powf(10.0f, -(log10f((float)na) - 1) / log10f(2.0f) - 3.0f);
    float d0 = -(1.0f / (2.0f * H)) * (1 + 1) * 6.0f * logf(R0);
    float b0 = 7.0f;
    float a0 = (float)(PI_D * (double)fcut);
    float xx;
    if (x <= xbeg0 + H) xx = (xbeg0 + H) - x;
    else if (x >= xend0 - H) xx = x - (xend0 - H);
    else xx = 0.0f;
    float r = fabsf(xx / H);
    float d = d0 * r;
    float a = a0 * (1.0f - r);
    float b = 1.0f + (b0 - 1.0f) * (r * r);
    float h = dt / 2.0f;
    g[0] = ((1.0f + h * a) / b) / (1.0f + h * (a + d / b));
    g[1] = (-1.0f / b) / (1.0f + h * (a + d / b));
    g[2] = (1.0f - h * (a + d / b)) / (1.0f + h * (a + d / b));
    g[3] = (d / b) / (1.0f + h * (a + d / b));
}

void o3d_absorb_setup(o3d *o, float fcut) {
    o->fcut = fcut;
    o->r20x = (MPR)1.0 / o->dx; o->r20y = (MPR)1.0 / o->dy; o->r20z = (MPR)1.0 / o->dz;
    int nxl = o->iend - o->ibeg + 1, nyl = o->jend - o->jbeg + 1, nzl = o->kend - o->kbeg + 1;
    o->fgxc = (float *)zalloc(sizeof(float) * 4 * nxl); o->fgxe = (float *)zalloc(sizeof(float) * 4 * nxl);
    o->fgyc = (float *)zalloc(sizeof(float) * 4 * nyl); o->fgye = (float *)zalloc(sizeof(float) * 4 * nyl);
    o->fgzc = (float *)zalloc(sizeof(float) * 4 * nzl); o->fgze = (float *)zalloc(sizeof(float) * 4 * nzl);
    float hx = o->na * (float)o->dx, hy = o->na * (float)o->dy, hz = o->na * (float)o->dz;
    for (int i = o->ibeg; i <= o->iend; i++) {
        float xc = o->xc[i - o->ibeg_m];
        damping_profile(xc, hx, o->xbeg, o->xend, o->na, fcut, o->dt, &o->fgxc[4 * (i - o->ibeg)]);
        damping_profile(xc + (float)o->dx / 2.0f, hx, o->xbeg, o->xend, o->na, fcut, o->dt, &o->fgxe[4 * (i - o->ibeg)]);
    }
    for (int j = o->jbeg; j <= o->jend; j++) {
        float yc = o->yc[j - o->jbeg_m];
        damping_profile(yc, hy, o->ybeg, o->yend, o->na, fcut, o->dt, &o->fgyc[4 * (j - o->jbeg)]);
        damping_profile(yc + (float)o->dy / 2.0f, hy, o->ybeg, o->yend, o->na, fcut, o->dt, &o->fgye[4 * (j - o->jbeg)]);
    }
    for (int k = o->kbeg; k <= o->kend; k++) {
        float zc = o->zc[k - o->kbeg_m];
        damping_profile(zc, hz, o->zbeg, o->zend, o->na, fcut, o->dt, &o->fgzc[4 * (k - o->kbeg)]);
        damping_profile(zc + (float)o->dz / 2.0f, hz, o->zbeg, o->zend, o->na, fcut, o->dt, &o->fgze[4 * (k - o->kbeg)]);
    }
#define PROMOTE(dst, src, n) do { dst = (SPR *)zalloc(sizeof(SPR) * (n)); for (long q = 0; q < (n); q++) dst[q] = (SPR)src[q]; } while (0)
    PROMOTE(o->gxc, o->fgxc, 4 * nxl); PROMOTE(o->gxe, o->fgxe, 4 * nxl);
    PROMOTE(o->gyc, o->fgyc, 4 * nyl); PROMOTE(o->gye, o->fgye, 4 * nyl);
    PROMOTE(o->gzc, o->fgzc, 4 * nzl); PROMOTE(o->gze, o->fgze, 4 * nzl);
#undef PROMOTE
    int kmin = 1 << 30;
    for (long q = 0; q < o->ni * o->nj; q++)
        if (o->kbeg_a[q] < kmin) kmin = o->kbeg_a[q];
    o->kbeg_min = kmin;
    o->nka = o->kend - kmin + 1;
    long na3 = o->nka * nxl * nyl;
#define AL(p) p = (SPR *)zalloc(sizeof(SPR) * na3)
    AL(o->axVx); AL(o->ayVx); AL(o->azVx); AL(o->axVy); AL(o->ayVy); AL(o->azVy);
    AL(o->axVz); AL(o->ayVz); AL(o->azVz); AL(o->axSxx); AL(o->aySxy); AL(o->azSxz);
    AL(o->axSxy); AL(o->aySyy); AL(o->azSyz); AL(o->axSxz); AL(o->aySyz); AL(o->azSzz);
#undef AL
}

/* Override the PML profiles (4, n) with external values. */
void o3d_set_profiles(o3d *o, const float *gxc, const float *gxe, const float *gyc, const float *gye,
                      const float *gzc, const float *gze) {
    int nxl = o->iend - o->ibeg + 1, nyl = o->jend - o->jbeg + 1, nzl = o->kend - o->kbeg + 1;
    for (int q = 0; q < 4 * nxl; q++) { o->gxc[q] = (SPR)gxc[q]; o->gxe[q] = (SPR)gxe[q]; o->fgxc[q] = gxc[q]; o->fgxe[q] = gxe[q]; }
    for (int q = 0; q < 4 * nyl; q++) { o->gyc[q] = (SPR)gyc[q]; o->gye[q] = (SPR)gye[q]; o->fgyc[q] = gyc[q]; o->fgye[q] = gye[q]; }
    for (int q = 0; q < 4 * nzl; q++) { o->gzc[q] = (SPR)gzc[q]; o->gze[q] = (SPR)gze[q]; o->fgzc[q] = gzc[q]; o->fgze[q] = gze[q]; }
}

#define GX(arr, n, i) (arr)[4 * ((i) - o->ibeg) + (n) - 1]
#define GY(arr, n, j) (arr)[4 * ((j) - o->jbeg) + (n) - 1]
#define GZ(arr, n, k) (arr)[4 * ((k) - o->kbeg) + (n) - 1]

/* ------------------------------------------------------------------------ */
/* kernel__update_vel: m_kernel.f90:75-140                                  */
/* ------------------------------------------------------------------------ */
void o3d_update_vel(o3d *o) {
    const SPR *bx = o->bx, *by = o->by, *bz = o->bz;
    const float dt = o->dt;
#pragma omp parallel for schedule(static) num_threads(o->threads)
    for (int j = o->jbeg_k; j <= o->jend_k; j++)
        for (int i = o->ibeg_k; i <= o->iend_k; i++)
            for (int k = o->kbeg_k; k <= o->kend_k; k++) {
                int a = (k - A2(o->kfs_top, i, j)) * (A2(o->kfs_bot, i, j) - k);
                int b = (k - A2(o->kob_top, i, j)) * (A2(o->kob_bot, i, j) - k);
                int isign = ((a > b ? a : b) >= 0) ? 1 : -1;
                MPR re40x = o->rc40x + isign * o->rd40x, re41x = o->rc41x + isign * o->rd41x;
                MPR re40y = o->rc40y + isign * o->rd40y, re41y = o->rc41y + isign * o->rd41y;
                MPR re40z = o->rc40z + isign * o->rd40z, re41z = o->rc41z + isign * o->rd41z;
                MPR *Sxx = o->Sxx, *Syy = o->Syy, *Szz = o->Szz, *Syz = o->Syz, *Sxz = o->Sxz, *Sxy = o->Sxy;
                MPR d3Sx3 = (A3(Sxx, k, i + 1, j) - A3(Sxx, k, i, j)) * re40x - (A3(Sxx, k, i + 2, j) - A3(Sxx, k, i - 1, j)) * re41x
                          + (A3(Sxy, k, i, j) - A3(Sxy, k, i, j - 1)) * re40y - (A3(Sxy, k, i, j + 1) - A3(Sxy, k, i, j - 2)) * re41y
                          + (A3(Sxz, k, i, j) - A3(Sxz, k - 1, i, j)) * re40z - (A3(Sxz, k + 1, i, j) - A3(Sxz, k - 2, i, j)) * re41z;
                MPR d3Sy3 = (A3(Sxy, k, i, j) - A3(Sxy, k, i - 1, j)) * re40x - (A3(Sxy, k, i + 1, j) - A3(Sxy, k, i - 2, j)) * re41x
                          + (A3(Syy, k, i, j + 1) - A3(Syy, k, i, j)) * re40y - (A3(Syy, k, i, j + 2) - A3(Syy, k, i, j - 1)) * re41y
                          + (A3(Syz, k, i, j) - A3(Syz, k - 1, i, j)) * re40z - (A3(Syz, k + 1, i, j) - A3(Syz, k - 2, i, j)) * re41z;
                MPR d3Sz3 = (A3(Sxz, k, i, j) - A3(Sxz, k, i - 1, j)) * re40x - (A3(Sxz, k, i + 1, j) - A3(Sxz, k, i - 2, j)) * re41x
                          + (A3(Syz, k, i, j) - A3(Syz, k, i, j - 1)) * re40y - (A3(Syz, k, i, j + 1) - A3(Syz, k, i, j - 2)) * re41y
                          + (A3(Szz, k + 1, i, j) - A3(Szz, k, i, j)) * re40z - (A3(Szz, k + 2, i, j) - A3(Szz, k - 1, i, j)) * re41z;
                long e = IDX3(o, k, i, j);
                o->Vx[e] = o->Vx[e] + bx[e] * d3Sx3 * dt;
                o->Vy[e] = o->Vy[e] + by[e] * d3Sy3 * dt;
                o->Vz[e] = o->Vz[e] + bz[e] * d3Sz3 * dt;
            }
}

/* ------------------------------------------------------------------------ */
/* kernel__update_stress: m_kernel.f90:142-326                              */
/* ------------------------------------------------------------------------ */
void o3d_update_stress(o3d *o) {
    const float dt = o->dt;
    const int nm = o->nm;
    const SPR d2 = o->d2;
    MPR *Vx = o->Vx, *Vy = o->Vy, *Vz = o->Vz;
    /* normal components: m_kernel.f90:176-239 */
#pragma omp parallel for schedule(static) num_threads(o->threads)
    for (int j = o->jbeg_k; j <= o->jend_k; j++)
        for (int i = o->ibeg_k; i <= o->iend_k; i++)
            for (int k = o->kbeg_k; k <= o->kend_k; k++) {
                int a = (k - A2(o->kfs_top, i, j)) * (A2(o->kfs_bot, i, j) - k);
                int b = (k - A2(o->kob_top, i, j)) * (A2(o->kob_bot, i, j) - k);
                int isign = ((a > b ? a : b) >= 0) ? 1 : -1;
                MPR re40x = o->rc40x + isign * o->rd40x, re41x = o->rc41x + isign * o->rd41x;
                MPR re40y = o->rc40y + isign * o->rd40y, re41y = o->rc41y + isign * o->rd41y;
                MPR re40z = o->rc40z + isign * o->rd40z, re41z = o->rc41z + isign * o->rd41z;
                MPR dxVx = (A3(Vx, k, i, j) - A3(Vx, k, i - 1, j)) * re40x - (A3(Vx, k, i + 1, j) - A3(Vx, k, i - 2, j)) * re41x;
                MPR dyVy = (A3(Vy, k, i, j) - A3(Vy, k, i, j - 1)) * re40y - (A3(Vy, k, i, j + 1) - A3(Vy, k, i, j - 2)) * re41y;
                MPR dzVz = (A3(Vz, k, i, j) - A3(Vz, k - 1, i, j)) * re40z - (A3(Vz, k + 1, i, j) - A3(Vz, k - 2, i, j)) * re41z;
                long e = IDX3(o, k, i, j);
                SPR mu2 = 2 * o->mu[e];
                SPR lam2mu = o->lam[e] + mu2;
                SPR taup1 = o->taup[e];
                SPR taus1 = o->taus[e];
                SPR d3v3 = (SPR)(dxVx + dyVy + dzVz);
                SPR dyVy_dzVz = (SPR)(dyVy + dzVz);
                SPR dxVx_dzVz = (SPR)(dxVx + dzVz);
                SPR dxVx_dyVy = (SPR)(dxVx + dyVy);
                SPR Rxx_n = 0.0f, Ryy_n = 0.0f, Rzz_n = 0.0f;
                for (int m = 1; m <= nm; m++) {
                    long r = IDXR(o, m, k, i, j);
                    o->Rxx[r] = o->c1[m - 1] * o->Rxx[r] - o->c2[m - 1] * (lam2mu * taup1 * d3v3 - mu2 * taus1 * dyVy_dzVz) * dt;
                    o->Ryy[r] = o->c1[m - 1] * o->Ryy[r] - o->c2[m - 1] * (lam2mu * taup1 * d3v3 - mu2 * taus1 * dxVx_dzVz) * dt;
                    o->Rzz[r] = o->c1[m - 1] * o->Rzz[r] - o->c2[m - 1] * (lam2mu * taup1 * d3v3 - mu2 * taus1 * dxVx_dyVy) * dt;
                    Rxx_n = Rxx_n + o->d1[m - 1] * o->Rxx[r];
                    Ryy_n = Ryy_n + o->d1[m - 1] * o->Ryy[r];
                    Rzz_n = Rzz_n + o->d1[m - 1] * o->Rzz[r];
                }
                SPR taup_plus1 = 1 + taup1 * (1 + d2);
                SPR taus_plus1 = 1 + taus1 * (1 + d2);
                o->Sxx[e] = o->Sxx[e] + (lam2mu * taup_plus1 * d3v3 - mu2 * taus_plus1 * dyVy_dzVz + Rxx_n) * dt;
                o->Syy[e] = o->Syy[e] + (lam2mu * taup_plus1 * d3v3 - mu2 * taus_plus1 * dxVx_dzVz + Ryy_n) * dt;
                o->Szz[e] = o->Szz[e] + (lam2mu * taup_plus1 * d3v3 - mu2 * taus_plus1 * dxVx_dyVy + Rzz_n) * dt;
            }
    /* shear components: m_kernel.f90:263-315 */
#pragma omp parallel for schedule(static) num_threads(o->threads)
    for (int j = o->jbeg_k; j <= o->jend_k; j++)
        for (int i = o->ibeg_k; i <= o->iend_k; i++)
            for (int k = o->kbeg_k; k <= o->kend_k; k++) {
                int a = (k - A2(o->kfs_top, i, j)) * (A2(o->kfs_bot, i, j) - k);
                int b = (k - A2(o->kob_top, i, j)) * (A2(o->kob_bot, i, j) - k);
                int isign = ((a > b ? a : b) >= 0) ? 1 : -1;
                MPR re40x = o->rc40x + isign * o->rd40x, re41x = o->rc41x + isign * o->rd41x;
                MPR re40y = o->rc40y + isign * o->rd40y, re41y = o->rc41y + isign * o->rd41y;
                MPR re40z = o->rc40z + isign * o->rd40z, re41z = o->rc41z + isign * o->rd41z;
                MPR dxVy_dyVx = (A3(Vy, k, i + 1, j) - A3(Vy, k, i, j)) * re40x - (A3(Vy, k, i + 2, j) - A3(Vy, k, i - 1, j)) * re41x
                              + (A3(Vx, k, i, j + 1) - A3(Vx, k, i, j)) * re40y - (A3(Vx, k, i, j + 2) - A3(Vx, k, i, j - 1)) * re41y;
                MPR dxVz_dzVx = (A3(Vz, k, i + 1, j) - A3(Vz, k, i, j)) * re40x - (A3(Vz, k, i + 2, j) - A3(Vz, k, i - 1, j)) * re41x
                              + (A3(Vx, k + 1, i, j) - A3(Vx, k, i, j)) * re40z - (A3(Vx, k + 2, i, j) - A3(Vx, k - 1, i, j)) * re41z;
                MPR dyVz_dzVy = (A3(Vz, k, i, j + 1) - A3(Vz, k, i, j)) * re40y - (A3(Vz, k, i, j + 2) - A3(Vz, k, i, j - 1)) * re41y
                              + (A3(Vy, k + 1, i, j) - A3(Vy, k, i, j)) * re40z - (A3(Vy, k + 2, i, j) - A3(Vy, k - 1, i, j)) * re41z;
                long e = IDX3(o, k, i, j);
                SPR taus1 = o->taus[e];
                SPR muyz = o->muyz[e], muxz = o->muxz[e], muxy = o->muxy[e];
                SPR Ryz_n = 0.0f, Rxz_n = 0.0f, Rxy_n = 0.0f;
                for (int m = 1; m <= nm; m++) {
                    long r = IDXR(o, m, k, i, j);
                    o->Ryz[r] = o->c1[m - 1] * o->Ryz[r] - o->c2[m - 1] * muyz * taus1 * dyVz_dzVy * dt;
                    o->Rxz[r] = o->c1[m - 1] * o->Rxz[r] - o->c2[m - 1] * muxz * taus1 * dxVz_dzVx * dt;
                    o->Rxy[r] = o->c1[m - 1] * o->Rxy[r] - o->c2[m - 1] * muxy * taus1 * dxVy_dyVx * dt;
                    Ryz_n = Ryz_n + o->d1[m - 1] * o->Ryz[r];
                    Rxz_n = Rxz_n + o->d1[m - 1] * o->Rxz[r];
                    Rxy_n = Rxy_n + o->d1[m - 1] * o->Rxy[r];
                }
                SPR taus_plus1 = 1 + taus1 * (1 + d2);
                o->Syz[e] = o->Syz[e] + (muyz * taus_plus1 * dyVz_dzVy + Ryz_n) * dt;
                o->Sxz[e] = o->Sxz[e] + (muxz * taus_plus1 * dxVz_dzVx + Rxz_n) * dt;
                o->Sxy[e] = o->Sxy[e] + (muxy * taus_plus1 * dxVy_dyVx + Rxy_n) * dt;
            }
}

/* ------------------------------------------------------------------------ */
/* absorb_c__setup: m_absorb_c.f90:27-103, with the kernel region of          */
/* abc_type = 'cerjan' (m_global.f90:349-378: the whole domain)              */
/* ------------------------------------------------------------------------ */
static void cerjan_axis(SPR *gc, SPR *gb, int n, int na, float d, int low) {
    const float alpha = 0.09f;
    const float L = na * d;
    for (int i = 1; i <= n; i++) {
        float c = 1.0f, b = 1.0f;
        if (low && i <= na) {
            /* m_absorb_c.f90:56-58 */
            const float x = o3d_i2x(i, 0.0f, d);
            const float yc = 1.0f - x / L, yb = 1.0f - (x + d / 2) / L;
            c = expf(-alpha * (yc * yc));
            b = expf(-alpha * (yb * yb));
        } else if (i >= n - na + 1) {
            /* m_absorb_c.f90:59-61 */
            const float x = o3d_i2x(i, n * d, -d);
            const float yc = 1.0f - (x + d / 2) / L, yb = 1.0f - x / L;
            c = expf(-alpha * (yc * yc));
            b = expf(-alpha * (yb * yb));
        }
        gc[i - 1] = c;
        gb[i - 1] = b;
    }
}

void o3d_set_stabilize(o3d *o, int on) { o->stabilize_pml = on; }

void o3d_cerjan_setup(o3d *o) {
    o->cerjan = 1;
    o->cgx_c = (SPR *)zalloc(sizeof(SPR) * o->nx); o->cgx_b = (SPR *)zalloc(sizeof(SPR) * o->nx);
    o->cgy_c = (SPR *)zalloc(sizeof(SPR) * o->ny); o->cgy_b = (SPR *)zalloc(sizeof(SPR) * o->ny);
    o->cgz_c = (SPR *)zalloc(sizeof(SPR) * o->nz); o->cgz_b = (SPR *)zalloc(sizeof(SPR) * o->nz);
    cerjan_axis(o->cgx_c, o->cgx_b, o->nx, o->na, (float)o->dx, 1);
    cerjan_axis(o->cgy_c, o->cgy_b, o->ny, o->na, (float)o->dy, 1);
    cerjan_axis(o->cgz_c, o->cgz_b, o->nz, o->na, (float)o->dz, 0);   /* free surface undamped (:73-80) */
    o->ibeg_k = o->ibeg; o->iend_k = o->iend; o->jbeg_k = o->jbeg; o->jend_k = o->jend;
    o->kbeg_k = o->kbeg; o->kend_k = o->kend;
    o->nkk = o->kend_k - o->kbeg_k + 1;
    o->nik = o->iend_k - o->ibeg_k + 1;
    o->njk = o->jend_k - o->jbeg_k + 1;
    const long nr = (long)o->nm * o->nkk * o->nik * o->njk;
    SPR **R[6] = {&o->Rxx, &o->Ryy, &o->Rzz, &o->Ryz, &o->Rxz, &o->Rxy};
    for (int q = 0; q < 6; q++) {
        free(*R[q]);
        *R[q] = (SPR *)zalloc(sizeof(SPR) * (size_t)nr);
    }
}

/* absorb_c__update_stress: m_absorb_c.f90:105-167 */
static void cerjan_update_stress(o3d *o) {
#pragma omp parallel for schedule(dynamic) num_threads(o->threads)
    for (int j = o->jbeg; j <= o->jend; j++)
        for (int i = o->ibeg; i <= o->iend; i++)
            for (int k = o->kbeg; k <= o->kend_k; k++) {
                const SPR gxc = o->cgx_c[i - 1], gxb = o->cgx_b[i - 1], gyc = o->cgy_c[j - 1], gyb = o->cgy_b[j - 1];
                const SPR gzc = o->cgz_c[k - 1], gzb = o->cgz_b[k - 1];
                const SPR gcc = gxc * gyc * gzc;
                A3(o->Sxx, k, i, j) = A3(o->Sxx, k, i, j) * gcc;
                A3(o->Syy, k, i, j) = A3(o->Syy, k, i, j) * gcc;
                A3(o->Szz, k, i, j) = A3(o->Szz, k, i, j) * gcc;
                A3(o->Syz, k, i, j) = A3(o->Syz, k, i, j) * gxc * gyb * gzb;
                A3(o->Sxz, k, i, j) = A3(o->Sxz, k, i, j) * gxb * gyc * gzb;
                A3(o->Sxy, k, i, j) = A3(o->Sxy, k, i, j) * gxb * gyb * gzc;
            }
}

/* absorb_c__update_vel: m_absorb_c.f90:169-198 */
static void cerjan_update_vel(o3d *o) {
#pragma omp parallel for schedule(dynamic) num_threads(o->threads)
    for (int j = o->jbeg; j <= o->jend; j++)
        for (int i = o->ibeg; i <= o->iend; i++)
            for (int k = o->kbeg; k <= o->kend; k++) {
                const SPR gxc = o->cgx_c[i - 1], gxb = o->cgx_b[i - 1], gyc = o->cgy_c[j - 1], gyb = o->cgy_b[j - 1];
                const SPR gzc = o->cgz_c[k - 1], gzb = o->cgz_b[k - 1];
                A3(o->Vx, k, i, j) = A3(o->Vx, k, i, j) * gxb * gyc * gzc;
                A3(o->Vy, k, i, j) = A3(o->Vy, k, i, j) * gxc * gyb * gzc;
                A3(o->Vz, k, i, j) = A3(o->Vz, k, i, j) * gxc * gyc * gzb;
            }
}

/* absorb_p__update_vel: m_absorb_p.f90:126-311 (pw_mode off); the dispatch
 * of absorb__update_vel (m_absorb.f90:60-75) picks the sponge instead */
/* ------------------------------------------------------------------------ */
/* horizontal zero-derivative boundary of the plane-wave mode (m_absorb_p.f90:136-243, 324-431): the ghost
   planes i = 0, nx+1 (j = jbeg..jend) and j = 0, ny+1 (i = ibeg..iend), k = 1..nz, of each field extrapolated
   linearly from the two cells inside */
static void pw_ghosts(o3d *o, MPR **f, int nf) {
    for (int q = 0; q < nf; q++) {
        MPR *a = f[q];
        for (int j = o->jbeg; j <= o->jend; j++)
            for (int k = 1; k <= o->nz; k++) {
                A3(a, k, 0, j) = 2 * A3(a, k, 1, j) - A3(a, k, 2, j);
                A3(a, k, o->nx + 1, j) = 2 * A3(a, k, o->nx, j) - A3(a, k, o->nx - 1, j);
            }
    }
    for (int q = 0; q < nf; q++) {
        MPR *a = f[q];
        for (int i = o->ibeg; i <= o->iend; i++)
            for (int k = 1; k <= o->nz; k++) {
                A3(a, k, i, 0) = 2 * A3(a, k, i, 1) - A3(a, k, i, 2);
                A3(a, k, i, o->ny + 1) = 2 * A3(a, k, i, o->ny) - A3(a, k, i, o->ny - 1);
            }
    }
}

void o3d_absorb_update_vel(o3d *o) {
    if (o->cerjan) {
        cerjan_update_vel(o);
        return;
    }
    if (o->pw_mode) {
        MPR *f[6] = {o->Sxx, o->Syy, o->Szz, o->Syz, o->Sxz, o->Sxy};
        pw_ghosts(o, f, 6);
    }
    const float dt = o->dt;
    MPR *Sxx = o->Sxx, *Syy = o->Syy, *Szz = o->Szz, *Syz = o->Syz, *Sxz = o->Sxz, *Sxy = o->Sxy;
#pragma omp parallel for schedule(dynamic) num_threads(o->threads)
    for (int j = o->jbeg; j <= o->jend; j++)
        for (int i = o->ibeg; i <= o->iend; i++)
            for (int k = A2(o->kbeg_a, i, j); k <= o->kend; k++) {
                MPR dxSxx = (A3(Sxx, k, i + 1, j) - A3(Sxx, k, i, j)) * o->r20x;
                MPR dySyy = (A3(Syy, k, i, j + 1) - A3(Syy, k, i, j)) * o->r20y;
                MPR dzSzz = (A3(Szz, k + 1, i, j) - A3(Szz, k, i, j)) * o->r20z;
                MPR dySyz = (A3(Syz, k, i, j) - A3(Syz, k, i, j - 1)) * o->r20y;
                MPR dzSyz = (A3(Syz, k, i, j) - A3(Syz, k - 1, i, j)) * o->r20z;
                MPR dxSxz = (A3(Sxz, k, i, j) - A3(Sxz, k, i - 1, j)) * o->r20x;
                MPR dzSxz = (A3(Sxz, k, i, j) - A3(Sxz, k - 1, i, j)) * o->r20z;
                MPR dxSxy = (A3(Sxy, k, i, j) - A3(Sxy, k, i - 1, j)) * o->r20x;
                MPR dySxy = (A3(Sxy, k, i, j) - A3(Sxy, k, i, j - 1)) * o->r20y;
                long e = IDX3(o, k, i, j), q = IDXA(o, k, i, j);
                o->Vx[e] = o->Vx[e] + o->bx[e] * (SPR)(GX(o->gxe, 1, i) * dxSxx + GY(o->gyc, 1, j) * dySxy + GZ(o->gzc, 1, k) * dzSxz
                                                   + GX(o->gxe, 2, i) * o->axSxx[q] + GY(o->gyc, 2, j) * o->aySxy[q] + GZ(o->gzc, 2, k) * o->azSxz[q]) * dt;
                o->Vy[e] = o->Vy[e] + o->by[e] * (SPR)(GX(o->gxc, 1, i) * dxSxy + GY(o->gye, 1, j) * dySyy + GZ(o->gzc, 1, k) * dzSyz
                                                   + GX(o->gxc, 2, i) * o->axSxy[q] + GY(o->gye, 2, j) * o->aySyy[q] + GZ(o->gzc, 2, k) * o->azSyz[q]) * dt;
                o->Vz[e] = o->Vz[e] + o->bz[e] * (SPR)(GX(o->gxc, 1, i) * dxSxz + GY(o->gyc, 1, j) * dySyz + GZ(o->gze, 1, k) * dzSzz
                                                   + GX(o->gxc, 2, i) * o->axSxz[q] + GY(o->gyc, 2, j) * o->aySyz[q] + GZ(o->gze, 2, k) * o->azSzz[q]) * dt;
                o->axSxx[q] = GX(o->gxe, 3, i) * o->axSxx[q] + GX(o->gxe, 4, i) * (SPR)dxSxx * dt;
                o->aySxy[q] = GY(o->gyc, 3, j) * o->aySxy[q] + GY(o->gyc, 4, j) * (SPR)dySxy * dt;
                o->azSxz[q] = GZ(o->gzc, 3, k) * o->azSxz[q] + GZ(o->gzc, 4, k) * (SPR)dzSxz * dt;
                o->axSxy[q] = GX(o->gxc, 3, i) * o->axSxy[q] + GX(o->gxc, 4, i) * (SPR)dxSxy * dt;
                o->aySyy[q] = GY(o->gye, 3, j) * o->aySyy[q] + GY(o->gye, 4, j) * (SPR)dySyy * dt;
                o->azSyz[q] = GZ(o->gzc, 3, k) * o->azSyz[q] + GZ(o->gzc, 4, k) * (SPR)dzSyz * dt;
                o->axSxz[q] = GX(o->gxc, 3, i) * o->axSxz[q] + GX(o->gxc, 4, i) * (SPR)dxSxz * dt;
                o->aySyz[q] = GY(o->gyc, 3, j) * o->aySyz[q] + GY(o->gyc, 4, j) * (SPR)dySyz * dt;
                o->azSzz[q] = GZ(o->gze, 3, k) * o->azSzz[q] + GZ(o->gze, 4, k) * (SPR)dzSzz * dt;
            }
}

/* ------------------------------------------------------------------------ */
/* absorb_p__update_stress: m_absorb_p.f90:313-505 (pw_mode off); the
 * dispatch of absorb__update_stress (m_absorb.f90:43-58) picks the sponge
 * instead */
/* ------------------------------------------------------------------------ */
void o3d_absorb_update_stress(o3d *o) {
    if (o->cerjan) {
        cerjan_update_stress(o);
        return;
    }
    if (o->pw_mode) {
        MPR *f[3] = {o->Vx, o->Vy, o->Vz};
        pw_ghosts(o, f, 3);
    }
    const float dt = o->dt;
    MPR *Vx = o->Vx, *Vy = o->Vy, *Vz = o->Vz;
#pragma omp parallel for schedule(dynamic) num_threads(o->threads)
    for (int j = o->jbeg; j <= o->jend; j++)
        for (int i = o->ibeg; i <= o->iend; i++) {
            for (int k = A2(o->kbeg_a, i, j); k <= o->kend; k++) {
                MPR dxVx = (A3(Vx, k, i, j) - A3(Vx, k, i - 1, j)) * o->r20x;
                MPR dyVy = (A3(Vy, k, i, j) - A3(Vy, k, i, j - 1)) * o->r20y;
                MPR dzVz = (A3(Vz, k, i, j) - A3(Vz, k - 1, i, j)) * o->r20z;
                long e = IDX3(o, k, i, j), q = IDXA(o, k, i, j);
                SPR lam2mu_R = (o->lam[e] + 2 * o->mu[e]);
                SPR lam_R = lam2mu_R - 2 * o->mu[e];
                SPR dxVx_ade = GX(o->gxc, 1, i) * (SPR)dxVx + GX(o->gxc, 2, i) * o->axVx[q];
                SPR dyVy_ade = GY(o->gyc, 1, j) * (SPR)dyVy + GY(o->gyc, 2, j) * o->ayVy[q];
                SPR dzVz_ade = GZ(o->gzc, 1, k) * (SPR)dzVz + GZ(o->gzc, 2, k) * o->azVz[q];
                o->Sxx[e] = o->Sxx[e] + (lam2mu_R * dxVx_ade + lam_R * (dyVy_ade + dzVz_ade)) * dt;
                o->Syy[e] = o->Syy[e] + (lam2mu_R * dyVy_ade + lam_R * (dxVx_ade + dzVz_ade)) * dt;
                o->Szz[e] = o->Szz[e] + (lam2mu_R * dzVz_ade + lam_R * (dxVx_ade + dyVy_ade)) * dt;
                o->axVx[q] = GX(o->gxc, 3, i) * o->axVx[q] + GX(o->gxc, 4, i) * (SPR)dxVx * dt;
                o->ayVy[q] = GY(o->gyc, 3, j) * o->ayVy[q] + GY(o->gyc, 4, j) * (SPR)dyVy * dt;
                o->azVz[q] = GZ(o->gzc, 3, k) * o->azVz[q] + GZ(o->gzc, 4, k) * (SPR)dzVz * dt;
            }
            for (int k = A2(o->kbeg_a, i, j); k <= o->kend; k++) {
                MPR dxVy = (A3(Vy, k, i + 1, j) - A3(Vy, k, i, j)) * o->r20x;
                MPR dxVz = (A3(Vz, k, i + 1, j) - A3(Vz, k, i, j)) * o->r20x;
                MPR dyVx = (A3(Vx, k, i, j + 1) - A3(Vx, k, i, j)) * o->r20y;
                MPR dyVz = (A3(Vz, k, i, j + 1) - A3(Vz, k, i, j)) * o->r20y;
                MPR dzVx = (A3(Vx, k + 1, i, j) - A3(Vx, k, i, j)) * o->r20z;
                MPR dzVy = (A3(Vy, k + 1, i, j) - A3(Vy, k, i, j)) * o->r20z;
                long e = IDX3(o, k, i, j), q = IDXA(o, k, i, j);
                o->Syz[e] = o->Syz[e] + o->muyz[e] * (GY(o->gye, 1, j) * dyVz + GZ(o->gze, 1, k) * dzVy
                                                      + GY(o->gye, 2, j) * o->ayVz[q] + GZ(o->gze, 2, k) * o->azVy[q]) * dt;
                o->Sxz[e] = o->Sxz[e] + o->muxz[e] * (GX(o->gxe, 1, i) * dxVz + GZ(o->gze, 1, k) * dzVx
                                                      + GX(o->gxe, 2, i) * o->axVz[q] + GZ(o->gze, 2, k) * o->azVx[q]) * dt;
                o->Sxy[e] = o->Sxy[e] + o->muxy[e] * (GX(o->gxe, 1, i) * dxVy + GY(o->gye, 1, j) * dyVx
                                                      + GX(o->gxe, 2, i) * o->axVy[q] + GY(o->gye, 2, j) * o->ayVx[q]) * dt;
                o->ayVx[q] = GY(o->gye, 3, j) * o->ayVx[q] + GY(o->gye, 4, j) * (SPR)dyVx * dt;
                o->azVx[q] = GZ(o->gze, 3, k) * o->azVx[q] + GZ(o->gze, 4, k) * (SPR)dzVx * dt;
                o->axVy[q] = GX(o->gxe, 3, i) * o->axVy[q] + GX(o->gxe, 4, i) * (SPR)dxVy * dt;
                o->azVy[q] = GZ(o->gze, 3, k) * o->azVy[q] + GZ(o->gze, 4, k) * (SPR)dzVy * dt;
                o->axVz[q] = GX(o->gxe, 3, i) * o->axVz[q] + GX(o->gxe, 4, i) * (SPR)dxVz * dt;
                o->ayVz[q] = GY(o->gye, 3, j) * o->ayVz[q] + GY(o->gye, 4, j) * (SPR)dyVz * dt;
            }
        }
}

/* ------------------------------------------------------------------------ */
/* global__comm_stress / global__comm_vel with one rank: every neighbour is */
/* MPI_PROC_NULL, so the unpack writes zeros (m_global.f90:460-490,571-603) */
/* ------------------------------------------------------------------------ */
static void zero_iplane(o3d *o, MPR *f, int i) {
    for (int j = o->jbeg; j <= o->jend; j++)
        for (int k = 1; k <= o->nz; k++) A3(f, k, i, j) = 0;
}
static void zero_jplane(o3d *o, MPR *f, int j) {
    for (int i = o->ibeg; i <= o->iend; i++)
        for (int k = 1; k <= o->nz; k++) A3(f, k, i, j) = 0;
}
void o3d_comm_vel(o3d *o) {
    int ib = o->ibeg, ie = o->iend, jb = o->jbeg, je = o->jend;
    zero_iplane(o, o->Vx, ib - 2); zero_iplane(o, o->Vx, ib - 1); zero_iplane(o, o->Vy, ib - 1);
    zero_iplane(o, o->Vz, ib - 1); zero_iplane(o, o->Vx, ie + 1); zero_iplane(o, o->Vy, ie + 1);
    zero_iplane(o, o->Vy, ie + 2); zero_iplane(o, o->Vz, ie + 1); zero_iplane(o, o->Vz, ie + 2);
    zero_jplane(o, o->Vx, jb - 1); zero_jplane(o, o->Vy, jb - 2); zero_jplane(o, o->Vy, jb - 1);
    zero_jplane(o, o->Vz, jb - 1); zero_jplane(o, o->Vx, je + 1); zero_jplane(o, o->Vx, je + 2);
    zero_jplane(o, o->Vy, je + 1); zero_jplane(o, o->Vz, je + 1); zero_jplane(o, o->Vz, je + 2);
}
void o3d_comm_stress(o3d *o) {
    int ib = o->ibeg, ie = o->iend, jb = o->jbeg, je = o->jend;
    zero_iplane(o, o->Sxx, ib - 1); zero_iplane(o, o->Sxy, ib - 2); zero_iplane(o, o->Sxy, ib - 1);
    zero_iplane(o, o->Sxz, ib - 2); zero_iplane(o, o->Sxz, ib - 1); zero_iplane(o, o->Sxx, ie + 1);
    zero_iplane(o, o->Sxx, ie + 2); zero_iplane(o, o->Sxy, ie + 1); zero_iplane(o, o->Sxz, ie + 1);
    zero_jplane(o, o->Syy, jb - 1); zero_jplane(o, o->Sxy, jb - 2); zero_jplane(o, o->Sxy, jb - 1);
    zero_jplane(o, o->Syz, jb - 2); zero_jplane(o, o->Syz, jb - 1); zero_jplane(o, o->Syy, je + 1);
    zero_jplane(o, o->Syy, je + 2); zero_jplane(o, o->Sxy, je + 1); zero_jplane(o, o->Syz, je + 1);
}

/* ------------------------------------------------------------------------ */
/* source__setup (grid assignment, normalisation): m_source.f90:181-305     */
/* returns the number of sources kept inside the (single) node              */
/* ------------------------------------------------------------------------ */
int o3d_source_setup(o3d *o, int bf_mode, int nsrc_g, const float *sx, const float *sy, const float *sz,
                     const float *srcprm /* (2,n) */, const float *mo_g, const float *m6 /* (6,n) xx yy zz yz xz xy */,
                     const float *f3 /* (3,n) */, int stftype) {
    o->bf_mode = bf_mode;
    o->stftype = stftype;
    float fcut = 0.0f;
    for (int i = 0; i < nsrc_g; i++) {
        float f = 1 / srcprm[2 * i + 1];
        if (f > fcut) fcut = f;
    }
    o->fcut = fcut;
    o->fmax = 2 * fcut;
    if (bf_mode) {
        float s = 0.0f;
        for (int i = 0; i < nsrc_g; i++) s += f3[3 * i] * f3[3 * i] + f3[3 * i + 1] * f3[3 * i + 1] + f3[3 * i + 2] * f3[3 * i + 2];
        o->M0 = sqrtf(s);
        o->UC = o->UC * 1000.0f;
    } else {
        float s = 0.0f;
        for (int i = 0; i < nsrc_g; i++) s += mo_g[i];
        o->M0 = s;
    }
    int n = 0;
    int *is = (int *)zalloc(sizeof(int) * nsrc_g), *js = (int *)zalloc(sizeof(int) * nsrc_g);
    int *ks = (int *)zalloc(sizeof(int) * nsrc_g), *in = (int *)zalloc(sizeof(int) * nsrc_g);
    for (int i = 0; i < nsrc_g; i++) {
        is[i] = o3d_x2i(sx[i], o->xbeg, (float)o->dx);
        js[i] = o3d_x2i(sy[i], o->ybeg, (float)o->dy);
        ks[i] = o3d_x2i(sz[i], o->zbeg, (float)o->dz);
        if (o->ibeg - 2 <= is[i] && is[i] <= o->iend + 3 && o->jbeg - 2 <= js[i] && js[i] <= o->jend + 3 &&
            o->kbeg - 2 <= ks[i] && ks[i] <= o->kend + 3) {
            in[i] = 1;
            n++;
        }
    }
    o->nsrc = n;
    o->isrc = (int *)zalloc(sizeof(int) * n); o->jsrc = (int *)zalloc(sizeof(int) * n);
    o->ksrc = (int *)zalloc(sizeof(int) * n); o->srcprm = (float *)zalloc(sizeof(float) * 2 * n);
    o->mo = (MPR *)zalloc(sizeof(MPR) * n);
    o->mxx = (MPR *)zalloc(sizeof(MPR) * n); o->myy = (MPR *)zalloc(sizeof(MPR) * n);
    o->mzz = (MPR *)zalloc(sizeof(MPR) * n); o->myz = (MPR *)zalloc(sizeof(MPR) * n);
    o->mxz = (MPR *)zalloc(sizeof(MPR) * n); o->mxy = (MPR *)zalloc(sizeof(MPR) * n);
    o->fx = (MPR *)zalloc(sizeof(MPR) * n); o->fy = (MPR *)zalloc(sizeof(MPR) * n);
    o->fz = (MPR *)zalloc(sizeof(MPR) * n);
    int nn = 0;
    for (int i = 0; i < nsrc_g; i++) {
        if (!in[i]) continue;
        o->isrc[nn] = is[i]; o->jsrc[nn] = js[i]; o->ksrc[nn] = ks[i];
        o->srcprm[2 * nn] = srcprm[2 * i]; o->srcprm[2 * nn + 1] = srcprm[2 * i + 1];
        /* sdep_fit = 'bd<n>': the source depth becomes the n-th boundary depth of its column
           (m_source.f90:262-270), and FDM space must contain it (m_source.f90:276-280) */
        if (o->sdep_fit1 > 0) {
            float szb = o->bddep[IDX2(o, is[i], js[i]) * (NBD + 1) + (o->sdep_fit1 - 1)];
            o->ksrc[nn] = o3d_x2i(szb, o->zbeg, (float)o->dz);
            if (!(o->zbeg <= szb && szb <= o->zend)) { free(is); free(js); free(ks); free(in); return -1; }
        }
        if (bf_mode) {
            o->fx[nn] = (MPR)f3[3 * i]; o->fy[nn] = (MPR)f3[3 * i + 1]; o->fz[nn] = (MPR)f3[3 * i + 2];
        } else {
            o->mo[nn] = (MPR)mo_g[i];
            o->mxx[nn] = (MPR)m6[6 * i + 0]; o->myy[nn] = (MPR)m6[6 * i + 1]; o->mzz[nn] = (MPR)m6[6 * i + 2];
            o->myz[nn] = (MPR)m6[6 * i + 3]; o->mxz[nn] = (MPR)m6[6 * i + 4]; o->mxy[nn] = (MPR)m6[6 * i + 5];
        }
        nn++;
    }
    free(is); free(js); free(ks); free(in);
    /* normalisation: m_source.f90:296-302 */
    for (int i = 0; i < n; i++) {
        if (bf_mode) {
            o->fx[i] = o->fx[i] / o->M0; o->fy[i] = o->fy[i] / o->M0; o->fz[i] = o->fz[i] / o->M0;
        } else {
            o->mo[i] = o->mo[i] / o->M0;
        }
    }
    /* dt_dxyz = dt / (dx * dy * dz): m_source.f90:305 */
    o->dt_dxyz = o->dt / (o->dx * o->dy * o->dz);
    return n;
}

/* pw_setup: m_source.f90:315-465.  The plane-wave initial condition over the memory box from the medium after
   medium__setup (every cell whose vp -- vs for an S wave -- reaches epsilon(1.0)), the cut-off frequency at the
   grid centre and depth pw_ztop, no source grid, and the fictitious moment M0 = 1 / UC (m_source.f90:72-79).
   ps: 0 P wave, 1 S wave; angles in degrees. */
void o3d_pw_setup(o3d *o, float pw_ztop, float pw_zlen, int ps, float strike, float dip, float rake, int stftype) {
    const float d2r_strike = (float)(PI_D / 180.0 * (double)strike);
    const float d2r_dip = (float)(PI_D / 180.0 * (double)dip);
    const float d2r_rake = (float)(PI_D / 180.0 * (double)rake);
    const float sd = sinf(d2r_dip), cd = cosf(d2r_dip), sf = sinf(d2r_strike), cf = cosf(d2r_strike);
    const float sl = sinf(d2r_rake), cl = cosf(d2r_rake), c2d = cosf(2 * d2r_dip), c2f = cosf(2 * d2r_strike);
    const float eps = 1.1920929e-07f;
    o->pw_mode = 1;
    o->stftype = stftype;
    for (int j = o->jbeg_m; j <= o->jend_m; j++)
        for (int i = o->ibeg_m; i <= o->iend_m; i++)
            for (int k = o->kbeg_m; k <= o->kend_m; k++) {
                const long e = IDX3(o, k, i, j);
                const float rho = o->frho[e], la0 = o->flam[e], mu0 = o->fmu[e];
                const float v = ps == 0 ? sqrtf((la0 + 2 * mu0) / rho) : sqrtf(mu0 / rho);
                if (v < eps) continue;
                const float x0 = (float)(o->xbeg + (MPR)(i - 0.5f) * o->dx);
                const float y0 = (float)(o->ybeg + (MPR)(j - 0.5f) * o->dy);
                const float z0 = (float)(o->zbeg + (MPR)(k - 0.5f) * o->dz - pw_ztop);
                const float x1 = (float)(x0 + o->dx / (MPR)2);
                const float y1 = (float)(y0 + o->dy / (MPR)2);
                const float z1 = (float)(z0 + o->dz / (MPR)2);
                const float hv = o->dt / 2.f * v;
                const float s_ii = o3d_momentrate(sd * sf * x0 - sd * cf * y0 + cd * z0, stftype, 0.0f, pw_zlen);
                const float s_vx = o3d_momentrate(sd * sf * x1 - sd * cf * y0 + cd * z0 + hv, stftype, 0.0f, pw_zlen);
                const float s_vy = o3d_momentrate(sd * sf * x0 - sd * cf * y1 + cd * z0 + hv, stftype, 0.0f, pw_zlen);
                const float s_vz = o3d_momentrate(sd * sf * x0 - sd * cf * y0 + cd * z1 + hv, stftype, 0.0f, pw_zlen);
                const float s_yz = o3d_momentrate(sd * sf * x0 - sd * cf * y1 + cd * z1, stftype, 0.0f, pw_zlen);
                const float s_xz = o3d_momentrate(sd * sf * x1 - sd * cf * y0 + cd * z1, stftype, 0.0f, pw_zlen);
                const float s_xy = o3d_momentrate(sd * sf * x1 - sd * cf * y1 + cd * z0, stftype, 0.0f, pw_zlen);
                if (ps == 0) {
                    A3(o->Vx, k, i, j) = -sd * sf * s_vx;
                    A3(o->Vy, k, i, j) = sd * cf * s_vy;
                    A3(o->Vz, k, i, j) = -cd * s_vz;
                    A3(o->Sxx, k, i, j) = -(la0 + 2 * mu0 * sd * sd * sf * sf) * s_ii / v;
                    A3(o->Syy, k, i, j) = -(la0 + 2 * mu0 * sd * sd * cf * cf) * s_ii / v;
                    A3(o->Szz, k, i, j) = -(la0 + 2 * mu0 * cd * cd) * s_ii / v;
                    A3(o->Syz, k, i, j) = 2 * mu0 * sd * cd * cf * s_yz / v;
                    A3(o->Sxz, k, i, j) = -2 * mu0 * sd * cd * sf * s_xz / v;
                    A3(o->Sxy, k, i, j) = 2 * mu0 * sd * cd * sf * s_xy / v;
                } else {
                    A3(o->Vx, k, i, j) = (cl * cf + sl * cd * sf) * s_vx;
                    A3(o->Vy, k, i, j) = (cl * sf - sl * cd * cf) * s_vy;
                    A3(o->Vz, k, i, j) = -sl * sd * s_vz;
                    A3(o->Sxx, k, i, j) = 2 * mu0 * sd * sf * (cl * cf + sl * cd * sf) * s_ii / v;
                    A3(o->Syy, k, i, j) = -2 * mu0 * sd * cf * (cl * sf - sl * cd * cf) * s_ii / v;
                    A3(o->Szz, k, i, j) = -2 * mu0 * cd * sl * sd * s_ii / v;
                    A3(o->Syz, k, i, j) = mu0 * (cl * cd * sf - sl * c2d * cf) * s_yz / v;
                    A3(o->Sxz, k, i, j) = mu0 * (cl * cd * cf + sl * c2d * sf) * s_xz / v;
                    A3(o->Sxy, k, i, j) = -mu0 * (cl * sd * c2f + 2 * sl * sd * cd * sf * cf) * s_xy / v;
                }
            }
    /* wavelength condition: m_source.f90:443-462 */
    const int ic = o3d_x2i((o->xbeg + o->xend) / 2, o->xbeg, (float)o->dx);
    const int jc = o3d_x2i((o->ybeg + o->yend) / 2, o->ybeg, (float)o->dy);
    const int kc = o3d_x2i(pw_ztop, o->zbeg, (float)o->dz);
    const long e = IDX3(o, kc, ic, jc);
    const float rho = o->frho[e], la0 = o->flam[e], mu0 = o->fmu[e];
    const float v = ps == 0 ? sqrtf((la0 + 2 * mu0) / rho) : sqrtf(mu0 / rho);
    o->fcut = v / pw_zlen;
    o->fmax = o->fcut * 2.0f;
    o->nsrc = 0;
    o->M0 = 1.0f / o->UC;
}

/* sdep_fit (m_source.f90:99): -1 for 'asis', n for 'bd<n>'; set before o3d_source_setup */
void o3d_set_sdep_fit(o3d *o, int n) { o->sdep_fit1 = (n >= 0 && n <= NBD) ? n + 1 : 0; }

/* boundary depths bddep(i, j, 0:NBD) of a velocity model that carries its own (vmodel_grd / vmodel_user,
   m_vmodel_grd.f90:258-270); vmodel_lhm fills depth(1) and -9999 (m_vmodel_lhm.f90:104, 161) */
void o3d_set_bddep(o3d *o, const float *bd) {
    memcpy(o->bddep, bd, sizeof(float) * o->ni * o->nj * (NBD + 1));
}

/* source__stressglut: m_source.f90:775-833 */
void o3d_stressglut(o3d *o, int it) {
    if (o->bf_mode) return;
    MPR *Sxx = o->Sxx, *Syy = o->Syy, *Szz = o->Szz, *Syz = o->Syz, *Sxz = o->Sxz, *Sxy = o->Sxy;
    for (int i = 0; i < o->nsrc; i++) {
        float t = o->tbeg + ((float)it - 0.5f) * o->dt;
        float stime = o3d_momentrate(t, o->stftype, o->srcprm[2 * i], o->srcprm[2 * i + 1]);
        MPR sdrop = o->mo[i] * stime * o->dt_dxyz;
        int ii = o->isrc[i], jj = o->jsrc[i], kk = o->ksrc[i];
        A3(Sxx, kk, ii, jj) = A3(Sxx, kk, ii, jj) - o->mxx[i] * sdrop;
        A3(Syy, kk, ii, jj) = A3(Syy, kk, ii, jj) - o->myy[i] * sdrop;
        A3(Szz, kk, ii, jj) = A3(Szz, kk, ii, jj) - o->mzz[i] * sdrop;
        A3(Sxy, kk, ii, jj) = A3(Sxy, kk, ii, jj) - o->mxy[i] * sdrop / 4;
        A3(Sxy, kk, ii, jj - 1) = A3(Sxy, kk, ii, jj - 1) - o->mxy[i] * sdrop / 4;
        A3(Sxy, kk, ii - 1, jj) = A3(Sxy, kk, ii - 1, jj) - o->mxy[i] * sdrop / 4;
        A3(Sxy, kk, ii - 1, jj - 1) = A3(Sxy, kk, ii - 1, jj - 1) - o->mxy[i] * sdrop / 4;
        A3(Sxz, kk, ii, jj) = A3(Sxz, kk, ii, jj) - o->mxz[i] * sdrop / 4;
        A3(Sxz, kk - 1, ii, jj) = A3(Sxz, kk - 1, ii, jj) - o->mxz[i] * sdrop / 4;
        A3(Sxz, kk, ii - 1, jj) = A3(Sxz, kk, ii - 1, jj) - o->mxz[i] * sdrop / 4;
        A3(Sxz, kk - 1, ii - 1, jj) = A3(Sxz, kk - 1, ii - 1, jj) - o->mxz[i] * sdrop / 4;
        A3(Syz, kk, ii, jj) = A3(Syz, kk, ii, jj) - o->myz[i] * sdrop / 4;
        A3(Syz, kk - 1, ii, jj) = A3(Syz, kk - 1, ii, jj) - o->myz[i] * sdrop / 4;
        A3(Syz, kk, ii, jj - 1) = A3(Syz, kk, ii, jj - 1) - o->myz[i] * sdrop / 4;
        A3(Syz, kk - 1, ii, jj - 1) = A3(Syz, kk - 1, ii, jj - 1) - o->myz[i] * sdrop / 4;
    }
}

/* source__bodyforce: m_source.f90:835-876 */
void o3d_bodyforce(o3d *o, int it) {
    if (!o->bf_mode) return;
    for (int i = 0; i < o->nsrc; i++) {
        float t = o->tbeg + (float)it * o->dt;
        float stime = o3d_momentrate(t, o->stftype, o->srcprm[2 * i], o->srcprm[2 * i + 1]);
        int ii = o->isrc[i], jj = o->jsrc[i], kk = o->ksrc[i];
        A3(o->Vx, kk, ii, jj) = A3(o->Vx, kk, ii, jj) + A3(o->bx, kk, ii, jj) * o->fx[i] * stime * o->dt_dxyz / 2;
        A3(o->Vx, kk, ii - 1, jj) = A3(o->Vx, kk, ii - 1, jj) + A3(o->bx, kk, ii - 1, jj) * o->fx[i] * stime * o->dt_dxyz / 2;
        A3(o->Vy, kk, ii, jj) = A3(o->Vy, kk, ii, jj) + A3(o->by, kk, ii, jj) * o->fy[i] * stime * o->dt_dxyz / 2;
        A3(o->Vy, kk, ii, jj - 1) = A3(o->Vy, kk, ii, jj - 1) + A3(o->by, kk, ii, jj - 1) * o->fy[i] * stime * o->dt_dxyz / 2;
        A3(o->Vz, kk, ii, jj) = A3(o->Vz, kk, ii, jj) + A3(o->bz, kk, ii, jj) * o->fz[i] * stime * o->dt_dxyz / 2;
        A3(o->Vz, kk - 1, ii, jj) = A3(o->Vz, kk - 1, ii, jj) + A3(o->bz, kk - 1, ii, jj) * o->fz[i] * stime * o->dt_dxyz / 2;
    }
}

/* green__setup (the parts green__source needs): m_green.f90:127-159 */
void o3d_green_setup(o3d *o, int isrc, int jsrc, int ksrc, char cmp, float green_tbeg, float green_trise,
                     int stftype) {
    o->green_mode = 1;
    o->green_is_src = 1;
    o->gisrc = isrc; o->gjsrc = jsrc; o->gksrc = ksrc;
    o->green_fx1 = (cmp == 'x') ? 1.0f : 0.0f;
    o->green_fy1 = (cmp == 'y') ? 1.0f : 0.0f;
    o->green_fz1 = (cmp == 'z') ? 1.0f : 0.0f;
    o->green_tbeg = green_tbeg;
    o->green_trise = green_trise;
    o->stftype = stftype;
    o->M0 = 1.0f;
    o->green_dt_dxyz = (float)(o->dt / (o->dx * o->dy * o->dz));
}

/* green__source: m_green.f90:597-632 */
void o3d_green_source(o3d *o, int it) {
    if (!o->green_mode || !o->green_is_src) return;
    float stf = o3d_momentrate(o->tbeg + (float)it * o->dt, o->stftype, o->green_tbeg, o->green_trise);
    float fx = o->green_fx1 * o->green_dt_dxyz * stf;
    float fy = o->green_fy1 * o->green_dt_dxyz * stf;
    float fz = o->green_fz1 * o->green_dt_dxyz * stf;
    int ii = o->gisrc, jj = o->gjsrc, kk = o->gksrc;
    A3(o->Vx, kk, ii, jj) = A3(o->Vx, kk, ii, jj) + A3(o->bx, kk, ii, jj) * fx / 2;
    A3(o->Vx, kk, ii - 1, jj) = A3(o->Vx, kk, ii - 1, jj) + A3(o->bx, kk, ii - 1, jj) * fx / 2;
    A3(o->Vy, kk, ii, jj) = A3(o->Vy, kk, ii, jj) + A3(o->by, kk, ii, jj) * fy / 2;
    A3(o->Vy, kk, ii, jj - 1) = A3(o->Vy, kk, ii, jj - 1) + A3(o->by, kk, ii, jj - 1) * fy / 2;
    A3(o->Vz, kk, ii, jj) = A3(o->Vz, kk, ii, jj) + A3(o->bz, kk, ii, jj) * fz / 2;
    A3(o->Vz, kk - 1, ii, jj) = A3(o->Vz, kk - 1, ii, jj) + A3(o->bz, kk - 1, ii, jj) * fz / 2;
}

/* ------------------------------------------------------------------------ */
/* wav__setup / set_stinfo / wav__store: m_wav.f90:76-142, 144-274, 400-628 */
/* zsw codes: 0 dep, 1 fsb, 2 obb, 3 oba, 10+n bd<n>                        */
/* ------------------------------------------------------------------------ */
int o3d_wav_setup(o3d *o, int nst_g, const float *xst, const float *yst, const float *zst, const int *zsw,
                  int ntdec_w, int sw_v, int sw_u, int sw_stress, int sw_strain, int *ist_out, int *jst_out,
                  int *kst_out) {
    o->ntdec_w = ntdec_w;
    o->sw_v = sw_v; o->sw_u = sw_u; o->sw_stress = sw_stress; o->sw_strain = sw_strain;
    o->ntw = (int)floorf((float)(o->nt - 1) / (float)ntdec_w + 1.0f);
    o->ist = (int *)zalloc(sizeof(int) * (nst_g ? nst_g : 1));
    o->jst = (int *)zalloc(sizeof(int) * (nst_g ? nst_g : 1));
    o->kst = (int *)zalloc(sizeof(int) * (nst_g ? nst_g : 1));
    int nst = 0;
    float ddx = (float)o->dx, ddy = (float)o->dy, ddz = (float)o->dz;
    for (int n = 0; n < nst_g; n++) {
        int ist = o3d_x2i(xst[n], o->xbeg, ddx), jst = o3d_x2i(yst[n], o->ybeg, ddy);
        int kst = o3d_x2i(zst[n], o->zbeg, ddz);
        if (o3d_i2x(1, o->xbeg, ddx) < xst[n] && xst[n] < o3d_i2x(o->nx, o->xbeg, ddx) &&
            o3d_i2x(1, o->ybeg, ddy) < yst[n] && yst[n] < o3d_i2x(o->ny, o->ybeg, ddy) && o->kbeg < kst &&
            kst < o->kend) {
            if (o->ibeg <= ist && ist <= o->iend && o->jbeg <= jst && jst <= o->jend) {
                int z = zsw[n];
                if (z == 1) kst = A2(o->kfs, ist, jst) + 1;
                else if (z == 2) kst = A2(o->kob, ist, jst) + 1;
                else if (z == 3) kst = A2(o->kob, ist, jst) - 1;
                else if (z >= 10 && z <= 10 + NBD)
                    kst = o3d_x2i(o->bddep[IDX2(o, ist, jst) * (NBD + 1) + (z - 10)], o->zbeg, ddz);
                else kst = o3d_x2i(zst[n], o->zbeg, ddz);
                if (kst > o->kend) kst = o->kend - 1;
                if (kst < o->kbeg) kst = o->kbeg + 1;
                o->ist[nst] = ist; o->jst[nst] = jst; o->kst[nst] = kst;
                nst++;
            }
        }
    }
    o->nst = nst;
    if (ist_out) for (int n = 0; n < nst; n++) { ist_out[n] = o->ist[n]; jst_out[n] = o->jst[n]; kst_out[n] = o->kst[n]; }
    long nw = (long)o->ntw * nst;
    o->wav_vel = (float *)zalloc(sizeof(float) * 3 * nw);
    o->wav_disp = (float *)zalloc(sizeof(float) * 3 * nw);
    o->wav_stress = (float *)zalloc(sizeof(float) * 6 * nw);
    o->wav_strain = (float *)zalloc(sizeof(float) * 6 * nw);
    o->ux = (SPR *)zalloc(sizeof(SPR) * nst); o->uy = (SPR *)zalloc(sizeof(SPR) * nst);
    o->uz = (SPR *)zalloc(sizeof(SPR) * nst);
    o->exx = (SPR *)zalloc(sizeof(SPR) * nst); o->eyy = (SPR *)zalloc(sizeof(SPR) * nst);
    o->ezz = (SPR *)zalloc(sizeof(SPR) * nst); o->eyz = (SPR *)zalloc(sizeof(SPR) * nst);
    o->exz = (SPR *)zalloc(sizeof(SPR) * nst); o->exy = (SPR *)zalloc(sizeof(SPR) * nst);
    o->r40x = (MPR)9.0 / (MPR)8.0 / o->dx; o->r40y = (MPR)9.0 / (MPR)8.0 / o->dy; o->r40z = (MPR)9.0 / (MPR)8.0 / o->dz;
    o->r41x = (MPR)1.0 / (MPR)24.0 / o->dx; o->r41y = (MPR)1.0 / (MPR)24.0 / o->dy; o->r41z = (MPR)1.0 / (MPR)24.0 / o->dz;
    return nst;
}

#define WAV(buf, ncmp, itw, c, n) (buf)[((long)(n) * (ncmp) + (c)) * o->ntw + (itw) - 1]

void o3d_wav_store(o3d *o, int it) {
    if (o->nst == 0) return;
    const float dt = o->dt;
    MPR *Vx = o->Vx, *Vy = o->Vy, *Vz = o->Vz;
    if (o->sw_u) {
        for (int n = 0; n < o->nst; n++) {
            int i = o->ist[n], j = o->jst[n], k = o->kst[n];
            o->ux[n] = o->ux[n] + (float)(A3(Vx, k, i, j) + A3(Vx, k, i - 1, j)) * 0.5f * dt;
            o->uy[n] = o->uy[n] + (float)(A3(Vy, k, i, j) + A3(Vy, k, i, j - 1)) * 0.5f * dt;
            o->uz[n] = o->uz[n] - (float)(A3(Vz, k, i, j) + A3(Vz, k - 1, i, j)) * 0.5f * dt;
        }
    }
    if (o->sw_strain) {
        MPR r40x = o->r40x, r40y = o->r40y, r40z = o->r40z, r41x = o->r41x, r41y = o->r41y, r41z = o->r41z;
        for (int n = 0; n < o->nst; n++) {
            int i = o->ist[n], j = o->jst[n], k = o->kst[n];
            MPR dxVx = (A3(Vx, k, i, j) - A3(Vx, k, i - 1, j)) * r40x - (A3(Vx, k, i + 1, j) - A3(Vx, k, i - 2, j)) * r41x;
            MPR dyVy = (A3(Vy, k, i, j) - A3(Vy, k, i, j - 1)) * r40y - (A3(Vy, k, i, j + 1) - A3(Vy, k, i, j - 2)) * r41y;
            MPR dzVz = (A3(Vz, k, i, j) - A3(Vz, k - 1, i, j)) * r40z - (A3(Vz, k + 1, i, j) - A3(Vz, k - 2, i, j)) * r41z;
            MPR dxVy = ((A3(Vy, k, i + 1, j) - A3(Vy, k, i, j)) * r40x - (A3(Vy, k, i + 2, j) - A3(Vy, k, i - 1, j)) * r41x
                      + (A3(Vy, k, i + 1, j - 1) - A3(Vy, k, i, j - 1)) * r40x - (A3(Vy, k, i + 2, j - 1) - A3(Vy, k, i - 1, j - 1)) * r41x
                      + (A3(Vy, k, i, j) - A3(Vy, k, i - 1, j)) * r40x - (A3(Vy, k, i + 1, j) - A3(Vy, k, i - 2, j)) * r41x
                      + (A3(Vy, k, i, j - 1) - A3(Vy, k, i - 1, j - 1)) * r40x - (A3(Vy, k, i + 1, j - 1) - A3(Vy, k, i - 2, j - 1)) * r41x) / (MPR)4.0;
            MPR dxVz = ((A3(Vz, k, i + 1, j) - A3(Vz, k, i, j)) * r40x - (A3(Vz, k, i + 2, j) - A3(Vz, k, i - 1, j)) * r41x
                      + (A3(Vz, k - 1, i + 1, j) - A3(Vz, k - 1, i, j)) * r40x - (A3(Vz, k - 1, i + 2, j) - A3(Vz, k - 1, i - 1, j)) * r41x
                      + (A3(Vz, k, i, j) - A3(Vz, k, i - 1, j)) * r40x - (A3(Vz, k, i + 1, j) - A3(Vz, k, i - 2, j)) * r41x
                      + (A3(Vz, k - 1, i, j) - A3(Vz, k - 1, i - 1, j)) * r40x - (A3(Vz, k - 1, i + 1, j) - A3(Vz, k - 1, i - 2, j)) * r41x) / (MPR)4.0;
            MPR dyVx = ((A3(Vx, k, i, j + 1) - A3(Vx, k, i, j)) * r40y - (A3(Vx, k, i, j + 2) - A3(Vx, k, i, j - 1)) * r41y
                      + (A3(Vx, k, i - 1, j + 1) - A3(Vx, k, i - 1, j)) * r40y - (A3(Vx, k, i - 1, j + 2) - A3(Vx, k, i - 1, j - 1)) * r41y
                      + (A3(Vx, k, i, j) - A3(Vx, k, i, j - 1)) * r40y - (A3(Vx, k, i, j + 1) - A3(Vx, k, i, j - 2)) * r41y
                      + (A3(Vx, k, i - 1, j) - A3(Vx, k, i - 1, j - 1)) * r40y - (A3(Vx, k, i - 1, j + 1) - A3(Vx, k, i - 1, j - 2)) * r41y) / (MPR)4.0;
            MPR dyVz = ((A3(Vz, k, i, j + 1) - A3(Vz, k, i, j)) * r40y - (A3(Vz, k, i, j + 2) - A3(Vz, k, i, j - 1)) * r41y
                      + (A3(Vz, k - 1, i, j + 1) - A3(Vz, k - 1, i, j)) * r40y - (A3(Vz, k - 1, i, j + 2) - A3(Vz, k - 1, i, j - 1)) * r41y
                      + (A3(Vz, k, i, j) - A3(Vz, k, i, j - 1)) * r40y - (A3(Vz, k, i, j + 1) - A3(Vz, k, i, j - 2)) * r41y
                      + (A3(Vz, k - 1, i, j) - A3(Vz, k - 1, i, j - 1)) * r40y - (A3(Vz, k - 1, i, j + 1) - A3(Vz, k - 1, i, j - 2)) * r41y) / (MPR)4.0;
            MPR dzVx = ((A3(Vx, k + 1, i, j) - A3(Vx, k, i, j)) * r40z - (A3(Vx, k + 2, i, j) - A3(Vx, k - 1, i, j)) * r41z
                      + (A3(Vx, k + 1, i - 1, j) - A3(Vx, k, i - 1, j)) * r40z - (A3(Vx, k + 2, i - 1, j) - A3(Vx, k - 1, i - 1, j)) * r41z
                      + (A3(Vx, k, i, j) - A3(Vx, k - 1, i, j)) * r40z - (A3(Vx, k + 1, i, j) - A3(Vx, k - 2, i, j)) * r41z
                      + (A3(Vx, k, i - 1, j) - A3(Vx, k - 1, i - 1, j)) * r40z - (A3(Vx, k + 1, i - 1, j) - A3(Vx, k - 2, i - 1, j)) * r41z) / (MPR)4.0;
            MPR dzVy = ((A3(Vy, k + 1, i, j) - A3(Vy, k, i, j)) * r40z - (A3(Vy, k + 2, i, j) - A3(Vy, k - 1, i, j)) * r41z
                      + (A3(Vy, k + 1, i, j - 1) - A3(Vy, k, i, j - 1)) * r40z - (A3(Vy, k + 2, i, j - 1) - A3(Vy, k - 1, i, j - 1)) * r41z
                      + (A3(Vy, k, i, j) - A3(Vy, k - 1, i, j)) * r40z - (A3(Vy, k + 1, i, j) - A3(Vy, k - 2, i, j)) * r41z
                      + (A3(Vy, k, i, j - 1) - A3(Vy, k - 1, i, j - 1)) * r40z - (A3(Vy, k + 1, i, j - 1) - A3(Vy, k - 2, i, j - 1)) * r41z) / (MPR)4.0;
            o->exx[n] = o->exx[n] + (float)dxVx * dt;
            o->eyy[n] = o->eyy[n] + (float)dyVy * dt;
            o->ezz[n] = o->ezz[n] + (float)dzVz * dt;
            o->eyz[n] = o->eyz[n] + (float)(dyVz + dzVy) / 2.0f * dt;
            o->exz[n] = o->exz[n] + (float)(dxVz + dzVx) / 2.0f * dt;
            o->exy[n] = o->exy[n] + (float)(dxVy + dyVx) / 2.0f * dt;
        }
    }
    if ((it - 1) % o->ntdec_w == 0) {
        int itw = (it - 1) / o->ntdec_w + 1;
        float M0 = o->M0, UC = o->UC;
        for (int n = 0; n < o->nst; n++) {
            int i = o->ist[n], j = o->jst[n], k = o->kst[n];
            if (o->sw_v) {
                WAV(o->wav_vel, 3, itw, 0, n) = (float)(A3(Vx, k, i, j) + A3(Vx, k, i - 1, j)) / 2.0f * M0 * UC * 1e9f;
                WAV(o->wav_vel, 3, itw, 1, n) = (float)(A3(Vy, k, i, j) + A3(Vy, k, i, j - 1)) / 2.0f * M0 * UC * 1e9f;
                WAV(o->wav_vel, 3, itw, 2, n) = -(float)(A3(Vz, k, i, j) + A3(Vz, k - 1, i, j)) / 2.0f * M0 * UC * 1e9f;
            }
            if (o->sw_u) {
                WAV(o->wav_disp, 3, itw, 0, n) = (float)o->ux[n] * M0 * UC * 1e9f;
                WAV(o->wav_disp, 3, itw, 1, n) = (float)o->uy[n] * M0 * UC * 1e9f;
                WAV(o->wav_disp, 3, itw, 2, n) = (float)o->uz[n] * M0 * UC * 1e9f;
            }
            if (o->sw_stress) {
                MPR *Sxx = o->Sxx, *Syy = o->Syy, *Szz = o->Szz, *Syz = o->Syz, *Sxz = o->Sxz, *Sxy = o->Sxy;
                WAV(o->wav_stress, 6, itw, 0, n) = (float)A3(Sxx, k, i, j) * M0 * UC * 1e6f;
                WAV(o->wav_stress, 6, itw, 1, n) = (float)A3(Syy, k, i, j) * M0 * UC * 1e6f;
                WAV(o->wav_stress, 6, itw, 2, n) = (float)A3(Szz, k, i, j) * M0 * UC * 1e6f;
                WAV(o->wav_stress, 6, itw, 3, n) = (float)(A3(Syz, k, i, j) + A3(Syz, k, i, j - 1) + A3(Syz, k - 1, i, j) + A3(Syz, k - 1, i, j - 1)) / 4.0f * M0 * UC * 1e6f;
                WAV(o->wav_stress, 6, itw, 4, n) = (float)(A3(Sxz, k, i, j) + A3(Sxz, k, i - 1, j) + A3(Sxz, k - 1, i, j) + A3(Sxz, k - 1, i - 1, j)) / 4.0f * M0 * UC * 1e6f;
                WAV(o->wav_stress, 6, itw, 5, n) = (float)(A3(Sxy, k, i, j) + A3(Sxy, k, i, j - 1) + A3(Sxy, k, i - 1, j) + A3(Sxy, k, i - 1, j - 1)) / 4.0f * M0 * UC * 1e6f;
            }
            if (o->sw_strain) {
                WAV(o->wav_strain, 6, itw, 0, n) = (float)o->exx[n] * M0 * UC * 1e-3f;
                WAV(o->wav_strain, 6, itw, 1, n) = (float)o->eyy[n] * M0 * UC * 1e-3f;
                WAV(o->wav_strain, 6, itw, 2, n) = (float)o->ezz[n] * M0 * UC * 1e-3f;
                WAV(o->wav_strain, 6, itw, 3, n) = (float)o->eyz[n] * M0 * UC * 1e-3f;
                WAV(o->wav_strain, 6, itw, 4, n) = (float)o->exz[n] * M0 * UC * 1e-3f;
                WAV(o->wav_strain, 6, itw, 5, n) = (float)o->exy[n] * M0 * UC * 1e-3f;
            }
        }
    }
}

/* kernel__vmax: m_kernel.f90:328-352 */
void o3d_vmax(o3d *o, float *out) {
    const int margin = 5;
    float xm = 0.0f, ym = 0.0f, zm = 0.0f;
    int j0 = o->na + margin + 1 > o->jbeg_k ? o->na + margin + 1 : o->jbeg_k;
    int j1 = o->ny - o->na - margin < o->jend_k ? o->ny - o->na - margin : o->jend_k;
    int i0 = o->na + margin + 1 > o->ibeg_k ? o->na + margin + 1 : o->ibeg_k;
    int i1 = o->nx - o->na - margin < o->iend_k ? o->nx - o->na - margin : o->iend_k;
    for (int j = j0; j <= j1; j++)
        for (int i = i0; i <= i1; i++) {
            int k = A2(o->kob, i, j) + 1;
            float ax = fabsf((float)A3(o->Vx, k, i, j)), ay = fabsf((float)A3(o->Vy, k, i, j));
            float az = fabsf((float)A3(o->Vz, k, i, j));
            if (ax > xm) xm = ax;
            if (ay > ym) ym = ay;
            if (az > zm) zm = az;
        }
    out[0] = xm; out[1] = ym; out[2] = zm;
}

/* ------------------------------------------------------------------------ */
/* snapshots: snap__setup (m_snap.f90:95-322) and the wbuf_* routines of     */
/* snap__write (m_snap.f90:911-2185) for a single MPI node; the file output  */
/* is replaced by frames kept in memory                                      */
/* ------------------------------------------------------------------------ */
static void snap_dims(const o3d *o, int plane, int *nvar, int *n1, int *n2) {
    int sec = plane / 3, q = plane % 3;
    *nvar = q == 0 ? 4 : 3;
    if (sec == 0) { *n1 = o->nys; *n2 = o->nzs; }
    else if (sec == 1) { *n1 = o->nxs; *n2 = o->nzs; }
    else { *n1 = o->nxs; *n2 = o->nys; }
}

int o3d_snap_setup(o3d *o, int planes, int idec, int jdec, int kdec, int ntdec_s, float x0_yz, float y0_xz,
                   float z0_xy) {
    o->snp_planes = planes; o->idec = idec; o->jdec = jdec; o->kdec = kdec; o->ntdec_s = ntdec_s;
    /* m_snap.f90:128-131 */
    o->nxs = (o->nx + idec / 2) / idec;
    o->nys = (o->ny + jdec / 2) / jdec;
    o->nzs = (o->nz + kdec / 2) / kdec;
    /* m_snap.f90:149-154 */
    o->is0 = (int)ceilf((float)(o->ibeg + idec / 2) / (float)idec);
    o->is1 = (int)floorf((float)(o->iend + idec / 2) / (float)idec);
    o->js0 = (int)ceilf((float)(o->jbeg + jdec / 2) / (float)jdec);
    o->js1 = (int)floorf((float)(o->jend + jdec / 2) / (float)jdec);
    o->ks0 = (int)ceilf((float)(o->kbeg + kdec / 2) / (float)kdec);
    o->ks1 = (int)floorf((float)(o->kend + kdec / 2) / (float)kdec);
    /* m_snap.f90:157-159 */
    o->k0_xy = o3d_x2i(z0_xy, o->zbeg, (float)o->dz);
    o->i0_yz = o3d_x2i(x0_yz, o->xbeg, (float)o->dx);
    o->j0_xz = o3d_x2i(y0_xz, o->ybeg, (float)o->dy);
    /* m_snap.f90:311-313 */
    o->sr20x = (MPR)1.0 / o->dx;
    o->sr20y = (MPR)1.0 / o->dy;
    o->sr20z = (MPR)1.0 / o->dz;
    o->nframes = (o->nt - 1) / ntdec_s + 1;
    for (int p = 0; p < 15; p++) {
        if (!(planes >> p & 1)) continue;
        int nv, n1, n2;
        snap_dims(o, p, &nv, &n1, &n2);
        o->snp[p] = (float *)zalloc(sizeof(float) * (size_t)o->nframes * nv * n1 * n2);
        o->sbuf[p] = (float *)zalloc(sizeof(float) * (size_t)nv * n1 * n2);
    }
    for (int q = 0; q < 4; q++) o->maxv[q] = (float *)zalloc(sizeof(float) * 3 * (size_t)o->nxs * o->nys);
    return o->nframes;
}

/* grid cell of snapshot sample (a, b) of a section (m_snap.f90 wbuf_*) */
static void snap_cell(const o3d *o, int sec, int a, int b, int *k, int *i, int *j) {
    switch (sec) {
    case 0: *i = o->i0_yz; *j = a * o->jdec - o->jdec / 2; *k = b * o->kdec - o->kdec / 2; break;
    case 1: *i = a * o->idec - o->idec / 2; *j = o->j0_xz; *k = b * o->kdec - o->kdec / 2; break;
    case 2: *i = a * o->idec - o->idec / 2; *j = b * o->jdec - o->jdec / 2; *k = o->k0_xy; break;
    case 3: *i = a * o->idec - o->idec / 2; *j = b * o->jdec - o->jdec / 2; *k = A2(o->kfs, *i, *j) + 1; break;
    default: *i = a * o->idec - o->idec / 2; *j = b * o->jdec - o->jdec / 2; *k = A2(o->kob, *i, *j) + 1; break;
    }
}

static float fmax_f(float a, float b) { return a > b ? a : b; }

/* one wbuf_<section>_<quantity> call (m_snap.f90:973-2185) */
static void snap_plane(o3d *o, int p, int it) {
    const int sec = p / 3, q = p % 3;
    int nv, n1, n2;
    snap_dims(o, p, &nv, &n1, &n2);
    const long ns = (long)n1 * n2;
    const int a0 = sec == 0 ? o->js0 : o->is0, a1 = sec == 0 ? o->js1 : o->is1;
    const int b0 = sec <= 1 ? o->ks0 : o->js0, b1 = sec <= 1 ? o->ks1 : o->js1;
    const int snap_step = ((it - 1) % o->ntdec_s == 0) || (it > o->nt);
    const int every_step = q == 2 || sec >= 3;   /* u planes and fs/ob v feed running sums / maxima */
    float *buf = o->sbuf[p];
    const float UC = o->UC, M0 = o->M0;
    const float eps = 1.1920929e-07f;            /* epsilon(1.0) */
    MPR *Vx = o->Vx, *Vy = o->Vy, *Vz = o->Vz;
    if (q == 0 && !snap_step) return;
    if (q == 1 && !snap_step && !(sec >= 3)) return;
    if (q == 1 && sec == 0) memset(buf, 0, sizeof(float) * 3 * ns);   /* wbuf_yz_v: buf = 0.0 */
    for (int b = b0; b <= b1; b++)
        for (int a = a0; a <= a1; a++) {
            int k, i, j;
            snap_cell(o, sec, a, b, &k, &i, &j);
            long e = (long)(b - 1) * n1 + (a - 1);
            if (q == 0) {
                const MPR r20x = o->sr20x, r20y = o->sr20y, r20z = o->sr20z;
                SPR div = (SPR)((A3(Vx, k, i, j) - A3(Vx, k, i - 1, j)) * r20x
                              + (A3(Vy, k, i, j) - A3(Vy, k, i, j - 1)) * r20y
                              + (A3(Vz, k, i, j) - A3(Vz, k - 1, i, j)) * r20z);
                SPR rot_x = (SPR)((A3(Vz, k, i, j + 1) - A3(Vz, k, i, j)) * r20y
                                - (A3(Vy, k + 1, i, j) - A3(Vy, k, i, j)) * r20z);
                SPR rot_y = (SPR)((A3(Vx, k + 1, i, j) - A3(Vx, k, i, j)) * r20z
                                - (A3(Vz, k, i + 1, j) - A3(Vz, k, i, j)) * r20x);
                SPR rot_z = (SPR)((A3(Vy, k, i + 1, j) - A3(Vy, k, i, j)) * r20x
                                - (A3(Vx, k, i, j + 1) - A3(Vx, k, i, j)) * r20y);
                SPR lam = A3(o->lam, k, i, j), muyz = A3(o->muyz, k, i, j);
                SPR muxz = A3(o->muxz, k, i, j), muxy = A3(o->muxy, k, i, j);
                div = div * lam / (SPR)fabs(lam + (SPR)eps);
                rot_x = rot_x * muyz / (SPR)fabs(muyz + (SPR)eps);
                rot_y = rot_y * muxz / (SPR)fabs(muxz + (SPR)eps);
                rot_z = rot_z * muxy / (SPR)fabs(muxy + (SPR)eps);
                buf[0 * ns + e] = (float)(div * UC * M0 * 1e-3f);
                buf[1 * ns + e] = (float)(rot_x * UC * M0 * 1e-3f);
                buf[2 * ns + e] = (float)(rot_y * UC * M0 * 1e-3f);
                buf[3 * ns + e] = (float)(rot_z * UC * M0 * 1e-3f);
            } else if (q == 1) {
                buf[0 * ns + e] = (float)(A3(Vx, k, i, j) * (MPR)UC * (MPR)M0);
                buf[1 * ns + e] = (float)(A3(Vy, k, i, j) * (MPR)UC * (MPR)M0);
                buf[2 * ns + e] = (float)(A3(Vz, k, i, j) * (MPR)UC * (MPR)M0);
            } else {
                const MPR dt = (MPR)o->dt;
                buf[0 * ns + e] = (float)((MPR)buf[0 * ns + e] + A3(Vx, k, i, j) * (MPR)UC * (MPR)M0 * dt);
                buf[1 * ns + e] = (float)((MPR)buf[1 * ns + e] + A3(Vy, k, i, j) * (MPR)UC * (MPR)M0 * dt);
                buf[2 * ns + e] = (float)((MPR)buf[2 * ns + e] + A3(Vz, k, i, j) * (MPR)UC * (MPR)M0 * dt);
            }
        }
    if (sec >= 3 && q >= 1) {
        /* running maxima of wbuf_fs_v / _ob_v / _fs_u / _ob_u (m_snap.f90:1691-1703) */
        float *mx = o->maxv[(sec - 3) * 2 + (q - 1)];
        for (int b = b0; b <= b1; b++)
            for (int a = a0; a <= a1; a++) {
                long e = (long)(b - 1) * n1 + (a - 1);
                float b1v = buf[e], b2v = buf[ns + e], b3v = buf[2 * ns + e];
                mx[e] = fmax_f(mx[e], fabsf(b3v));
                mx[ns + e] = fmax_f(mx[ns + e], sqrtf(b1v * b1v + b2v * b2v));
                mx[2 * ns + e] = sqrtf(mx[e] * mx[e] + mx[ns + e] * mx[ns + e]);
            }
    }
    (void)every_step;
    if (snap_step && it <= o->nt) {
        long f = (it - 1) / o->ntdec_s;
        memcpy(o->snp[p] + f * nv * ns, buf, sizeof(float) * nv * ns);
    }
}

/* snap__write (m_snap.f90:911-939): the reference's call order */
void o3d_snap_write(o3d *o, int it) {
    static const int order[15] = {3, 6, 9, 12, 0, 1, 4, 7, 10, 13, 2, 5, 8, 11, 14};
    if (!o->snp_planes) return;
    for (int n = 0; n < 15; n++)
        if (o->snp_planes >> order[n] & 1) snap_plane(o, order[n], it);
}

void o3d_snap_dims(const o3d *o, int *out) {
    out[0] = o->nxs; out[1] = o->nys; out[2] = o->nzs; out[3] = o->nframes;
    out[4] = o->i0_yz; out[5] = o->j0_xz; out[6] = o->k0_xy;
}
float *o3d_snap_frames(o3d *o, int plane) { return (plane >= 0 && plane < 15) ? o->snp[plane] : 0; }
float *o3d_snap_max(o3d *o, int which) { return (which >= 0 && which < 4) ? o->maxv[which] : 0; }

/* one pass of the main.f90:125-144 loop body (report__progress excluded) */
/* green__store: m_green.f90:389-534 (green table points given as grid cells) */
void o3d_green_store_setup(o3d *o, int ng, const int *ig, const int *jg, const int *kg, int bforce, int ntdec) {
    o->ng = ng;
    o->ng_cmp = bforce ? 9 : 6;
    o->ng_ntdec = ntdec;
    o->ng_ntw = (o->nt - 1) / ntdec + 1;
    o->gi = (int *)zalloc(sizeof(int) * ng); o->gj = (int *)zalloc(sizeof(int) * ng); o->gk = (int *)zalloc(sizeof(int) * ng);
    for (int n = 0; n < ng; n++) { o->gi[n] = ig[n]; o->gj[n] = jg[n]; o->gk[n] = kg[n]; }
    o->gacc = (float *)zalloc(sizeof(float) * 12 * (size_t)ng);
    o->gf = (float *)zalloc(sizeof(float) * (size_t)o->ng_ntw * o->ng_cmp * ng);
}

void o3d_green_store(o3d *o, int it) {
    if (o->ng <= 0) return;
    const MPR r40x = (MPR)(9.0 / 8.0) / o->dx, r40y = (MPR)(9.0 / 8.0) / o->dy, r40z = (MPR)(9.0 / 8.0) / o->dz;
    const MPR r41x = (MPR)(1.0 / 24.0) / o->dx, r41y = (MPR)(1.0 / 24.0) / o->dy, r41z = (MPR)(1.0 / 24.0) / o->dz;
    const float dt = o->dt;
    MPR *Vx = o->Vx, *Vy = o->Vy, *Vz = o->Vz;
    const int ng = o->ng;
#define V_(f, k, i, j) A3(f, k, i, j)
#define DF(f, k, i, j, dk, di, dj, r0, r1)                                                                 \
    ((V_(f, (k) + (dk), (i) + (di), (j) + (dj)) - V_(f, k, i, j)) * (r0) -                                 \
     (V_(f, (k) + 2 * (dk), (i) + 2 * (di), (j) + 2 * (dj)) - V_(f, (k) - (dk), (i) - (di), (j) - (dj))) * (r1))
#define DB(f, k, i, j, dk, di, dj, r0, r1)                                                                 \
    ((V_(f, k, i, j) - V_(f, (k) - (dk), (i) - (di), (j) - (dj))) * (r0) -                                 \
     (V_(f, (k) + (dk), (i) + (di), (j) + (dj)) - V_(f, (k) - 2 * (dk), (i) - 2 * (di), (j) - 2 * (dj))) * (r1))
    for (int n = 0; n < ng; n++) {
        const int ii = o->gi[n], jj = o->gj[n], kk = o->gk[n];
        MPR dxVx = DB(Vx, kk, ii, jj, 0, 1, 0, r40x, r41x);
        MPR dyVy = DB(Vy, kk, ii, jj, 0, 0, 1, r40y, r41y);
        MPR dzVz = DB(Vz, kk, ii, jj, 1, 0, 0, r40z, r41z);
        MPR dxVy = (DF(Vy, kk, ii, jj, 0, 1, 0, r40x, r41x) + DF(Vy, kk, ii, jj - 1, 0, 1, 0, r40x, r41x) +
                    DB(Vy, kk, ii, jj, 0, 1, 0, r40x, r41x) + DB(Vy, kk, ii, jj - 1, 0, 1, 0, r40x, r41x)) * 0.25f;
        MPR dxVz = (DF(Vz, kk, ii, jj, 0, 1, 0, r40x, r41x) + DF(Vz, kk - 1, ii, jj, 0, 1, 0, r40x, r41x) +
                    DB(Vz, kk, ii, jj, 0, 1, 0, r40x, r41x) + DB(Vz, kk - 1, ii, jj, 0, 1, 0, r40x, r41x)) * 0.25f;
        MPR dyVx = (DF(Vx, kk, ii, jj, 0, 0, 1, r40y, r41y) + DF(Vx, kk, ii - 1, jj, 0, 0, 1, r40y, r41y) +
                    DB(Vx, kk, ii, jj, 0, 0, 1, r40y, r41y) + DB(Vx, kk, ii - 1, jj, 0, 0, 1, r40y, r41y)) * 0.25f;
        MPR dyVz = (DF(Vz, kk, ii, jj, 0, 0, 1, r40y, r41y) + DF(Vz, kk - 1, ii, jj, 0, 0, 1, r40y, r41y) +
                    DB(Vz, kk, ii, jj, 0, 0, 1, r40y, r41y) + DB(Vz, kk - 1, ii, jj, 0, 0, 1, r40y, r41y)) * 0.25f;
        MPR dzVx = (DF(Vx, kk, ii, jj, 1, 0, 0, r40z, r41z) + DF(Vx, kk, ii - 1, jj, 1, 0, 0, r40z, r41z) +
                    DB(Vx, kk, ii, jj, 1, 0, 0, r40z, r41z) + DB(Vx, kk, ii - 1, jj, 1, 0, 0, r40z, r41z)) * 0.25f;
        MPR dzVy = (DF(Vy, kk, ii, jj, 1, 0, 0, r40z, r41z) + DF(Vy, kk, ii, jj - 1, 1, 0, 0, r40z, r41z) +
                    DB(Vy, kk, ii, jj, 1, 0, 0, r40z, r41z) + DB(Vy, kk, ii, jj - 1, 1, 0, 0, r40z, r41z)) * 0.25f;
        const MPR d[9] = {dxVx, dxVy, dxVz, dyVx, dyVy, dyVz, dzVx, dzVy, dzVz};
        for (int q = 0; q < 9; q++) o->gacc[q * ng + n] = o->gacc[q * ng + n] + (float)(d[q] * dt);
        if (o->ng_cmp == 9) {
            o->gacc[9 * ng + n] = o->gacc[9 * ng + n] + 0.5f * (float)(V_(Vx, kk, ii, jj) + V_(Vx, kk, ii - 1, jj)) * dt;
            o->gacc[10 * ng + n] = o->gacc[10 * ng + n] + 0.5f * (float)(V_(Vy, kk, ii, jj) + V_(Vy, kk, ii, jj - 1)) * dt;
            o->gacc[11 * ng + n] = o->gacc[11 * ng + n] + 0.5f * (float)(V_(Vz, kk, ii, jj) + V_(Vz, kk - 1, ii, jj)) * dt;
        }
    }
#undef DF
#undef DB
#undef V_
    if ((it - 1) % o->ng_ntdec != 0) return;
    const int itw = (it - 1) / o->ng_ntdec + 1;
    if (itw > o->ng_ntw) return;
    const float uc = 1e-15f, ub = 1e-12f;   /* UC_DERIV, UC_BF (m_green.f90:31-32) */
    for (int n = 0; n < ng; n++) {
        const float *u = o->gacc;
        float *g = o->gf + (size_t)n * o->ng_cmp * o->ng_ntw + (itw - 1);
        const long w = o->ng_ntw;
        g[0 * w] = u[0 * ng + n] * uc * 1e9f;
        g[1 * w] = u[4 * ng + n] * uc * 1e9f;
        g[2 * w] = u[8 * ng + n] * uc * 1e9f;
        g[3 * w] = (u[5 * ng + n] + u[7 * ng + n]) * uc * 1e9f;
        g[4 * w] = (u[2 * ng + n] + u[6 * ng + n]) * uc * 1e9f;
        g[5 * w] = (u[1 * ng + n] + u[3 * ng + n]) * uc * 1e9f;
        if (o->ng_cmp == 9)
            for (int q = 0; q < 3; q++) g[(6 + q) * w] = u[(9 + q) * ng + n] * ub * 1e9f;
    }
}

void o3d_step(o3d *o, int it) {
    o3d_wav_store(o, it);
    o3d_green_store(o, it);
    o3d_snap_write(o, it);
    o3d_update_stress(o);
    o3d_absorb_update_stress(o);
    o3d_stressglut(o, it);
    o3d_comm_stress(o);
    o3d_update_vel(o);
    o3d_absorb_update_vel(o);
    o3d_bodyforce(o, it);
    o3d_green_source(o, it);
    o3d_comm_vel(o);
}

/* ------------------------------------------------------------------------ */
/* accessors for the ctypes wrapper                                         */
/* ------------------------------------------------------------------------ */
void o3d_dims(const o3d *o, long *out) {
    out[0] = o->nk; out[1] = o->ni; out[2] = o->nj;
    out[3] = o->nkk; out[4] = o->nik; out[5] = o->njk; out[6] = o->nka;
    out[7] = o->ibeg_k; out[8] = o->iend_k; out[9] = o->jbeg_k; out[10] = o->jend_k;
    out[11] = o->kbeg_k; out[12] = o->kend_k; out[13] = o->kbeg_min; out[14] = o->nst; out[15] = o->ntw;
    out[16] = o->nsrc;
}
void o3d_scalars(const o3d *o, float *out) {
    out[0] = o->M0; out[1] = o->UC; out[2] = o->fcut; out[3] = o->fmax; out[4] = o->vmin; out[5] = o->vmax;
    out[6] = o->zeta; out[7] = o->xend; out[8] = o->yend; out[9] = o->zend;
    for (int m = 0; m < NM_MAX; m++) out[10 + m] = o->ts[m];
}
int o3d_mpr_size(void) { return (int)sizeof(MPR); }
int o3d_spr_size(void) { return (int)sizeof(SPR); }

/* field ids: 0..8 V/S (MPR), 10..15 R (SPR), 20..29 medium (SPR) lam mu taup
 * taus bx by bz muyz muxz muxy, 30.. float setup copies rho lam mu taup taus
 * bx by bz muyz muxz muxy, 50..55 int maps kfs kob kfs_top kfs_bot kob_top
 * kob_bot, 56 kbeg_a, 57 bddep (float, (i, j, 0:NBD)), 60..77 PML aux (SPR), 80..85 float profiles gxc gxe
 * gyc gye gzc gze, 90..93 wav buffers */
void *o3d_ptr(o3d *o, int id) {
    switch (id) {
    case 0: return o->Vx; case 1: return o->Vy; case 2: return o->Vz;
    case 3: return o->Sxx; case 4: return o->Syy; case 5: return o->Szz;
    case 6: return o->Syz; case 7: return o->Sxz; case 8: return o->Sxy;
    case 10: return o->Rxx; case 11: return o->Ryy; case 12: return o->Rzz;
    case 13: return o->Ryz; case 14: return o->Rxz; case 15: return o->Rxy;
    case 20: return o->lam; case 21: return o->mu; case 22: return o->taup; case 23: return o->taus;
    case 24: return o->bx; case 25: return o->by; case 26: return o->bz;
    case 27: return o->muyz; case 28: return o->muxz; case 29: return o->muxy;
    case 30: return o->frho; case 31: return o->flam; case 32: return o->fmu; case 33: return o->ftaup;
    case 34: return o->ftaus; case 35: return o->fbx; case 36: return o->fby; case 37: return o->fbz;
    case 38: return o->fmuyz; case 39: return o->fmuxz; case 40: return o->fmuxy;
    case 50: return o->kfs; case 51: return o->kob; case 52: return o->kfs_top; case 53: return o->kfs_bot;
    case 54: return o->kob_top; case 55: return o->kob_bot; case 56: return o->kbeg_a;
    case 57: return o->bddep;
    case 60: return o->axVx; case 61: return o->ayVx; case 62: return o->azVx;
    case 63: return o->axVy; case 64: return o->ayVy; case 65: return o->azVy;
    case 66: return o->axVz; case 67: return o->ayVz; case 68: return o->azVz;
    case 69: return o->axSxx; case 70: return o->aySxy; case 71: return o->azSxz;
    case 72: return o->axSxy; case 73: return o->aySyy; case 74: return o->azSyz;
    case 75: return o->axSxz; case 76: return o->aySyz; case 77: return o->azSzz;
    case 80: return o->fgxc; case 81: return o->fgxe; case 82: return o->fgyc;
    case 83: return o->fgye; case 84: return o->fgzc; case 85: return o->fgze;
    case 90: return o->wav_vel; case 91: return o->wav_disp; case 92: return o->wav_stress;
    case 93: return o->wav_strain;
    case 95: return o->ist; case 96: return o->jst; case 97: return o->kst;
    case 98: return o->isrc; case 99: return o->jsrc; case 100: return o->ksrc;
    case 120: return o->gf;
    case 110: return o->cgx_c; case 111: return o->cgx_b; case 112: return o->cgy_c;
    case 113: return o->cgy_b; case 114: return o->cgz_c; case 115: return o->cgz_b;
    default: return 0;
    }
}
