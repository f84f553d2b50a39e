/*
 * swpc_setup.h -- host-side setup routines of the B200 OpenSWPC library.
 *
 * In the reference these run once before the time loop, inside the Fortran
 * modules m_global, m_medium, m_vmodel_lhm(_rmed), m_absorb_p, m_source and
 * m_wav.  A Fortran driver keeps its own setup and only needs swpc_gpu.h;
 * these entry points serve drivers that do not have the Fortran setup (the
 * Python host layer of this package, C/C++ drivers).  Every routine computes
 * in single precision with the reference's expression order so that the
 * integer maps are bit-identical and the float fields reproducible.
 *
 * Arrays follow the reference layout: 3D fields over the memory box
 * (kbeg_m:kend_m, ibeg_m:iend_m, jbeg_m:jend_m) = (-2:nz+3, -2:nx+3, -2:ny+3),
 * k fastest; 2D maps over (-2:nx+3, -2:ny+3).  For the 2D codes pass ny = 1
 * and arrays over (-2:nz+3, -2:nx+3).
 */
#ifndef SWPC_SETUP_H
#define SWPC_SETUP_H

#ifdef __cplusplus
extern "C" {
#endif

/* Grid geometry shared by the setup routines (m_global.f90:54-66). */
typedef struct swpc_grid {
    int nx, ny, nz, na, nm;
    float dx, dy, dz, dt;
    float xbeg, ybeg, zbeg, tbeg;
} swpc_grid;

/* x2i / y2j / z2k (src/shared/m_fdtool.f90:600-636): ceiling((x-beg)/d). */
int swpc_x2i(float x, float beg, float d);
/* i2x / j2y / k2z (src/shared/m_fdtool.f90:639-675): beg + (i-0.5)*d. */
float swpc_i2x(int i, float beg, float d);

/* momentrate (src/shared/m_fdtool.f90:472-497) with SWPC_STF_* codes. */
float swpc_momentrate(float t, int stftype, float ts, float tr);

/* sdr2moment (src/shared/m_fdtool.f90:307-336); m6 = xx yy zz yz xz xy. */
void swpc_sdr2moment(float strike, float dip, float rake, float *m6);

/* visco_set_relaxtime + visco_constq_zeta (m_fdtool.f90:691-812). */
void swpc_visco_setup(int nm, float fq_min, float fq_max, float *ts, float *zeta);

/* kbeg_a absorber map (src/swpc_3d/m_global.f90:336-345) over the memory
 * box columns. */
void swpc_kbeg_a(const swpc_grid *g, int *kbeg_a);

/* vmodel_lhm (src/swpc_3d/m_vmodel_lhm.f90:21-169); with xi != NULL the
 * lhm_rmed perturbation (m_vmodel_lhm_rmed.f90:187-195, vcheck
 * m_fdtool.f90:15-48).  depth/rho/vp/vs/qp/qs per layer; outputs over the
 * memory box: rho, lam, mu, qp, qs.  Air above depth(1) with z < 0, seawater of
 * 1.5 km/s above depth(1) with z >= 0. */
int swpc_vmodel_lhm(const swpc_grid *g, int nlayer, const float *depth, const float *rho0, const float *vp0,
                    const float *vs0, const float *qp0, const float *qs0, float vcut, const float *xi, float rhomin,
                    float *rho, float *lam, float *mu, float *qp, float *qs);
/* The same with the input-file switch munk_profile (m_vmodel_lhm.f90:53-54):
 * cells with 0 <= z < depth(1) are seawater (rho 1, mu 0, Q 1e6) whose
 * P velocity is 1.5 km/s, or Munk's profile when munk_profile != 0
 * (seawater__vel, src/shared/m_seawater.f90:36-49).  swpc_vmodel_lhm is
 * this call with munk_profile = 0. */
int swpc_vmodel_lhm_opt(const swpc_grid *g, int nlayer, const float *depth, const float *rho0, const float *vp0,
                        const float *vs0, const float *qp0, const float *qs0, float vcut, const float *xi,
                        float rhomin, float *rho, float *lam, float *mu, float *qp, float *qs, int munk_profile);
/* seawater__vel (src/shared/m_seawater.f90:36-49): the P velocity [km/s] of
 * seawater at depth z [km]. */
float swpc_seawater_vel(float z, int munk_profile);

/* medium__setup after the vmodel (src/swpc_3d/m_medium.f90:124-225 and its
 * contained routines): absorber homogenisation, tau-method (taup/taus from
 * qp/qs), relaxed moduli, free-surface/ocean-bottom detection, velocity
 * range, averaged buoyancy and rigidities.  rho/lam/mu are updated in
 * place, qp/qs are read; outputs: taup, taus, bx, by, bz, muyz, muxz, muxy
 * (3D fields), kfs, kob, kfs_top, kfs_bot, kob_top, kob_bot (2D maps),
 * ts(nm), scal = {zeta, vmin, vmax}.  3D only (see swpc_setup_medium_2d). */
int swpc_setup_medium(const swpc_grid *g, float fq_min, float fq_max, float fq_ref, float *rho, float *lam, float *mu,
                      const float *qp, const float *qs, float *taup, float *taus, float *bx, float *by, float *bz,
                      float *muyz, float *muxz, float *muxy, int *kfs, int *kob, int *kfs_top, int *kfs_bot,
                      int *kob_top, int *kob_bot, float *ts, float *scal);
/* The same with the input-file switch stabilize_pml (m_medium.f90:219-222,
 * stabilize_absorber :276-340) applied before the averaged medium. */
int swpc_setup_medium_opt(const swpc_grid *g, float fq_min, float fq_max, float fq_ref, float *rho, float *lam,
                          float *mu, const float *qp, const float *qs, float *taup, float *taus, float *bx, float *by,
                          float *bz, float *muyz, float *muxz, float *muxy, int *kfs, int *kob, int *kfs_top,
                          int *kfs_bot, int *kob_top, int *kob_bot, float *ts, float *scal, int stabilize_pml);

/* medium__setup of the 2D codes after the vmodel (src/swpc_psv/m_medium.f90:124-281,
 * src/swpc_sh/m_medium.f90): absorber homogenisation in x and at the bottom,
 * tau-method, relaxed moduli through visco_chi (m_fdtool.f90:730-753),
 * free-surface / ocean-bottom detection and velocity range.  Arrays over
 * (-2:nz+3, -2:nx+3); maps over (-2:nx+3).  The 2nd-order band is formed as
 * in the 3D code (kfs_top = max(min-2, 1), kfs_bot = min(max+2, nz)): the 2D
 * reference assigns kfs_top twice and leaves kfs_bot undefined
 * (src/swpc_psv/m_medium.f90:241-242, src/swpc_sh/m_medium.f90:247-248). */
int swpc_setup_medium_2d(const swpc_grid *g, float fq_min, float fq_max, float fq_ref, float *rho, float *lam,
                         float *mu, const float *qp, const float *qs, float *taup, float *taus, int *kfs, int *kob,
                         int *kfs_top, int *kfs_bot, int *kob_top, int *kob_bot, float *ts, float *scal);
/* The same with stabilize_pml (src/swpc_psv/m_medium.f90:175-178, 309-365)
 * applied last. */
int swpc_setup_medium_2d_opt(const swpc_grid *g, float fq_min, float fq_max, float fq_ref, float *rho, float *lam,
                             float *mu, const float *qp, const float *qs, float *taup, float *taus, int *kfs,
                             int *kob, int *kfs_top, int *kfs_bot, int *kob_top, int *kob_bot, float *ts,
                             float *scal, int stabilize_pml);

/* damping_profile (src/swpc_3d/m_absorb_p.f90:507-547) for the six profiles
 * of absorb_p__setup (:79-93); each output is g(4, n). */
void swpc_damping_profiles(const swpc_grid *g, float fcut, float *gxc, float *gxe, float *gyc, float *gye, float *gzc,
                           float *gze);

/* absorb_c__setup (src/swpc_3d/m_absorb_c.f90:27-103): the Cerjan sponge
 * factors at cell centres (_c) and +d/2 boundaries (_b), n values per axis
 * indexed [i-1]; the free surface (k <= na) is undamped.  For the 2D codes
 * gy_c and gy_b may be NULL. */
void swpc_cerjan_profiles(const swpc_grid *g, float *gx_c, float *gx_b, float *gy_c, float *gy_b, float *gz_c,
                          float *gz_b);

/* pw_setup (src/swpc_3d/m_source.f90:315-465): the initial wavefield of the
 * plane-wave mode (pw_mode = .true.) from the medium after medium__setup
 * (rho, lam, mu over the memory box).  ps = 0 for a P wave, 1 for an S wave;
 * the front lies at depth pw_ztop with length pw_zlen [km] along the
 * direction of strike and dip (rake: polarisation of the S wave) [deg],
 * shaped by the moment-rate function stftype (SWPC_STF_*).  Writes V and S
 * over the memory box (cells whose wave speed is below epsilon(1.0) are left
 * as they are) and the cut-off frequency fcut of the PML profiles
 * (:443-462).  The run then has no source grid, its output moment is
 * M0 = 1 / UC (:72-79), and swpc_set_pw_mode switches on the zero-derivative
 * side boundary of the absorber. */
int swpc_pw_setup(const swpc_grid *g, const float *rho, const float *lam, const float *mu, float pw_ztop,
                  float pw_zlen, int ps, float strike, float dip, float rake, int stftype, float *vx, float *vy,
                  float *vz, float *sxx, float *syy, float *szz, float *syz, float *sxz, float *sxy, float *fcut);

/* Random media (src/shared/m_rmedia.f90): rmedia__3dgen (:176-307) for
 * ny > 1 and rmedia__2dgen (:424-) for ny = 1, generated on the current CUDA
 * device.  Uniform random numbers in [0, 1) over nx x ny x nz cells, their
 * spectrum whitened and filtered by the Gaussian (ptype 1), exponential (2)
 * or von Karman (3) power spectral density of correlation distance a, rms
 * epsil and order kappa (rmedia__psdf_*, :530-679), DC removed, mean removed
 * and scaled to rms epsil.  The volume is written to the device array xi over
 * the memory box -- (-2:nz+3, -2:nx+3, -2:ny+3) with leading extents ld_k,
 * ld_i, or (-2:nz+3, -2:nx+3) for ny = 1 -- with the cyclic wrap rdrmed__3d
 * uses for cells outside 1..n (src/shared/m_rdrmed.f90:111-132), ready for
 * swpc_vmodel_lhm_device or swpc_vmodel_lhm.  The random numbers are a
 * counter-based stream of `seed` (gfortran's random_number stream of the
 * reference cannot be reproduced), so a realisation depends on the seed
 * alone.  Runs on `stream` (a cudaStream_t; NULL = the default stream) and
 * blocks until xi is written; allocates about 2.1 x 4 B x nx ny nz of
 * temporary device memory (volume, half spectrum, FFT plans) and frees it
 * before it returns.  Returns SWPC_ERR_ARG, SWPC_ERR_NOMEM or SWPC_ERR_CUDA
 * on failure. */
#define SWPC_RMEDIA_GAUSS 1
#define SWPC_RMEDIA_EXP 2
#define SWPC_RMEDIA_VONKARMAN 3
typedef struct swpc_rmedia_desc {
    int ptype;
    int nx, ny, nz;
    float dx, dy, dz;
    float a, epsil, kappa;
    unsigned long long seed;
} swpc_rmedia_desc;
int swpc_rmedia_generate(const swpc_rmedia_desc *d, float *xi, int ld_k, int ld_i, void *stream);

#ifdef __cplusplus
}
#endif
#endif
