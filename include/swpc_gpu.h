/*
 * swpc_gpu.h -- C ABI of the B200 time-step library for OpenSWPC.
 *
 * The library replaces the hot routines of OpenSWPC's time loop
 * (src/swpc_3d/main.f90:125-144, src/swpc_psv/main.f90:95-114,
 * src/swpc_sh/main.f90:95-116).  In the reference those routines are
 * argument-less Fortran module procedures acting on module-global arrays;
 * here every routine takes an opaque context that owns the device copies of
 * those arrays.  A Fortran caller keeps one `type(c_ptr)` per run and binds
 * each entry point with ISO_C_BINDING: one interface block per function,
 * bind(C) with the C name, scalars by value, arrays by reference.
 *
 * Conventions
 *   - every function returns an int status: 0 = OK, otherwise an
 *     SWPC_ERR_* code; swpc_last_error() gives the message.  The Fortran
 *     shim maps a nonzero status to `call assert(.false.)`, the reference's
 *     error path (src/shared/m_debug.h:7, src/shared/m_pdebug.f90:223-240).
 *   - arrays cross the boundary in the reference's Fortran layout:
 *     3D fields (kbeg_m:kend_m, ibeg_m:iend_m, jbeg_m:jend_m), k fastest,
 *     with the memory box of m_global.f90:297-302 (lower bound 1-3, upper
 *     bound n+3+pad); 2D maps (ibeg_m:iend_m, jbeg_m:jend_m).  ld_k and ld_i
 *     are the leading extents of the caller's arrays.
 *   - the context owns all device memory; host pointers are only read or
 *     written during the call that receives them.
 *   - calls on one context are not thread-safe (one host thread per context,
 *     like the reference's one thread per MPI rank).  All calls are
 *     stream-ordered on the context's stream; *_fetch, swpc_vmax,
 *     swpc_download_* and swpc_sync block.
 *   - precision: velocity, stress, memory variables and medium are FP32
 *     (the reference built with MP = SP, src/swpc_3d/m_global.f90:30).
 */
#ifndef SWPC_GPU_H
#define SWPC_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define SWPC_OK 0
#define SWPC_ERR_ARG 1        /* invalid argument or size                    */
#define SWPC_ERR_CUDA 2       /* CUDA runtime error (message has the name)   */
#define SWPC_ERR_STATE 3      /* call out of order (e.g. step before setup)  */
#define SWPC_ERR_DIVERGED 4   /* max |V| * UC > 1e5 (m_report.f90:142-152)   */
#define SWPC_ERR_NOMEM 5      /* device allocation failed                    */
#define SWPC_ERR_LIMIT 6      /* size above a fixed limit of swpc_vmax_noalloc */

/* solver kinds */
#define SWPC_KIND_3D 3
#define SWPC_KIND_PSV 2
#define SWPC_KIND_SH 1

/* source-time-function codes (m_fdtool.f90:472-497 `momentrate`) */
#define SWPC_STF_KUPPER 0
#define SWPC_STF_BOXCAR 1
#define SWPC_STF_TRIANGLE 2
#define SWPC_STF_HERRMANN 3
#define SWPC_STF_COSINE 4
#define SWPC_STF_TEXP 5

/* field ids for swpc_upload_field / swpc_download_field */
#define SWPC_F_VX 0
#define SWPC_F_VY 1
#define SWPC_F_VZ 2
#define SWPC_F_SXX 3
#define SWPC_F_SYY 4
#define SWPC_F_SZZ 5
#define SWPC_F_SYZ 6
#define SWPC_F_SXZ 7
#define SWPC_F_SXY 8
/* memory variables: SWPC_F_R + 3*c + (m-1), c = 0..5 for xx yy zz yz xz xy */
#define SWPC_F_R 10
/* PML auxiliaries (m_absorb_p.f90:47-52), 18 in the order
 * axVx ayVx azVx axVy ayVy azVy axVz ayVz azVz
 * axSxx aySxy azSxz axSxy aySyy azSyz axSxz aySyz azSzz */
#define SWPC_F_AUX 40
/* 3D medium arrays, swpc_download_field only: SWPC_F_MED + q, q = 1..10 in
 * the field order of the medium view: lam mu taup taus bx by bz muyz muxz
 * muxy (rho is not kept) */
#define SWPC_F_MED 60

/* wave-field recorder components (m_wav.f90:31-34) */
#define SWPC_WAV_V 1
#define SWPC_WAV_U 2
#define SWPC_WAV_STRESS 4
#define SWPC_WAV_STRAIN 8

typedef struct swpc_ctx swpc_ctx;

/* Grid description: the parameters global__readprm / global__setup2 fix
 * (m_global.f90:126-179, 221-390) for a single node covering the whole
 * domain.  For the 2D codes ny = 1 (P-SV: x-z, SH: x-z with Vy). */
typedef struct swpc_desc {
    int kind;        /* SWPC_KIND_3D / _PSV / _SH                                 */
    int nx, ny, nz;  /* global grid size                                          */
    int na;          /* absorber thickness in cells (abc_type = 'pml')            */
    int nm;          /* Zener memory variables, 0..3 (reference NM = 3)           */
    int nt;          /* number of time steps (sizes the source/recorder tables)   */
    float dx, dy, dz;/* grid spacing [km] (real(MP), MP = SP)                     */
    float dt;        /* time step [s]                                             */
    float tbeg;      /* start time [s]                                            */
    int device;      /* CUDA device ordinal                                       */
    int precision;   /* SWPC_PREC_*: storage of stress and memory variables (3D)  */
} swpc_desc;

/* Storage precision of the 3D stress (S) and memory-variable (R) arrays; the
 * arithmetic is FP32 in every form.  F32 is the reference's MP = SP build;
 * BF16_R stores R in BF16; F16_R stores R in FP16 and F16_SR stores S and R
 * in FP16, with a power-of-two scale per stress array and one for the memory
 * variables (see swpc_rescale).  Every form runs the
 * TMA-staged kernels by default (swpc_set_launch kernels 5 and 6); the
 * one-cell-per-thread kernels 0 and 1 stay selectable. */
#define SWPC_PREC_F32 0
#define SWPC_PREC_BF16_R 1
#define SWPC_PREC_F16_SR 2
#define SWPC_PREC_F16_R 3

/* Medium and integer maps as produced by medium__setup
 * (src/swpc_3d/m_medium.f90:36-467).  Float fields are 3D Fortran arrays
 * over the memory box; the 2D int maps cover (ibeg_m:iend_m, jbeg_m:jend_m).
 * For P-SV only lam, mu, taup, taus, rho are read (b and mu_xz are formed
 * inside the kernels as in src/swpc_psv/m_kernel.f90:118-119, 270-274);
 * for SH only mu, taus, rho. */
typedef struct swpc_medium_view {
    const float *rho, *lam, *mu, *taup, *taus;
    const float *bx, *by, *bz, *muyz, *muxz, *muxy;
    int ld_k, ld_i;                        /* extents of the 3D arrays             */
    const int *kfs, *kob;                  /* free-surface / ocean-bottom k        */
    const int *kfs_top, *kfs_bot;          /* 2nd-order band (m_medium.f90:382-386)*/
    const int *kob_top, *kob_bot;
    const int *kbeg_a;                     /* absorber start (m_global.f90:336-345)*/
    int ld_i2;                             /* leading extent of the 2D maps        */
} swpc_medium_view;

/* ---- lifetime ---------------------------------------------------------- */

/* Allocates every device array of the run (zero-filled).  Replaces the
 * allocations of m_kernel.f90:354-378, m_medium.f90:477-500 and the
 * `!$acc enter data` block of main.f90:80-119. */
int swpc_create(const swpc_desc *desc, swpc_ctx **out);
int swpc_destroy(swpc_ctx *ctx);
const char *swpc_last_error(const swpc_ctx *ctx);
/* cudaStream_t of the context, as void*. */
void *swpc_stream(swpc_ctx *ctx);
/* Waits for the context's stream.  Returns SWPC_ERR_CUDA when a staged
 * kernel's tile copy did not complete within its bounded wait (the kernel
 * then skipped its cells and raised the context's error word).  The fields
 * that launch and every later launch wrote are then undefined, and every
 * later swpc_sync reports the error until the caller restores the state --
 * swpc_reset_state (a run from rest, which also clears the word) or uploads
 * of every field followed by swpc_clear_error.  No counterpart in the
 * reference. */
int swpc_sync(swpc_ctx *ctx);
int swpc_clear_error(swpc_ctx *ctx);
/* Failure injection for the error paths of a driver: raises the error word
 * from the host exactly as a timed-out tile wait does (no kernel waits, no
 * device fault).  No counterpart in the reference. */
int swpc_raise_copy_error(swpc_ctx *ctx);

/* ---- setup ------------------------------------------------------------- */

/* Copies the medium and maps to HBM (the `!$acc enter data copyin` of
 * main.f90:97-119).  3D: with rho given and bx, by, bz, muyz, muxz, muxy all
 * NULL, the six averaged fields are formed in HBM from rho and mu as
 * averaged_medium (m_medium.f90:432-465) forms them, bitwise equal to the
 * fields of swpc_setup_medium; the host then sends 5 arrays instead of 10. */
int swpc_upload_medium(swpc_ctx *ctx, const swpc_medium_view *m);

/* ---- medium built on the device (3D) ------------------------------------
 * The alternative to the host setup + swpc_upload_medium: the per-cell model
 * and medium__setup (src/swpc_3d/m_medium.f90:36-467) run in HBM, bitwise
 * equal to swpc_vmodel_lhm + swpc_setup_medium (swpc_setup.h) on the same
 * inputs, and the context ends in the state swpc_upload_medium leaves.
 *
 * Step 1, one of:
 *   swpc_vmodel_lhm_device: vmodel_lhm (m_vmodel_lhm.f90:21-169) from the
 *     layer table; with xi != NULL the lhm_rmed perturbation
 *     (m_vmodel_lhm_rmed.f90:187-195, vcheck m_fdtool.f90:15-48).  xi is a
 *     host or a device array over the memory box (leading extents ld_k,
 *     ld_i); zbeg is the top of the grid (m_global.f90 zbeg).
 *   swpc_vmodel_upload: rho, lam, mu, qp, qs of any host-side model.
 * Step 2, swpc_medium_setup_device: absorber homogenisation, tau method,
 *   relaxed moduli, surface detection, velocity range and averaged medium.
 *   Returns ts(1:nm) and scal = {zeta, vmin, vmax} as swpc_setup_medium does,
 *   and, where the pointers are not NULL, the integer maps over
 *   (-2:nx+3, -2:ny+3) with leading extent ld_i2 (kbeg_a as swpc_kbeg_a). */
int swpc_vmodel_lhm_device(swpc_ctx *ctx, int nlayer, const float *depth, const float *rho0, const float *vp0,
                           const float *vs0, const float *qp0, const float *qs0, float vcut, float rhomin, float zbeg,
                           const float *xi, int ld_k, int ld_i);
/* The same with munk_profile (m_vmodel_lhm.f90:53-54): the seawater above
 * depth(1) takes Munk's profile instead of 1.5 km/s (swpc_vmodel_lhm_opt). */
int swpc_vmodel_lhm_device_opt(swpc_ctx *ctx, int nlayer, const float *depth, const float *rho0, const float *vp0,
                               const float *vs0, const float *qp0, const float *qs0, float vcut, float rhomin,
                               float zbeg, const float *xi, int ld_k, int ld_i, int munk_profile);
int swpc_vmodel_upload(swpc_ctx *ctx, const float *rho, const float *lam, const float *mu, const float *qp,
                       const float *qs, int ld_k, int ld_i);
/* Step 1 from device memory: per-cell vp, vs, rho, qp, qs as device arrays
 * over the memory box (leading extents ld_k, ld_i), the moduli formed on the
 * device as vmodel_lhm forms them (m_vmodel_lhm.f90:146-148, mu = rho vs vs,
 * lam = rho (vp vp - 2 vs vs)); bitwise swpc_vmodel_upload of the moduli a
 * host computes in that order.  For models that already live on the GPU. */
int swpc_vmodel_velocity_device(swpc_ctx *ctx, const float *vp, const float *vs, const float *rho, const float *qp,
                                const float *qs, int ld_k, int ld_i);
int swpc_medium_setup_device(swpc_ctx *ctx, float fq_min, float fq_max, float fq_ref, float *ts, float *scal,
                             int *kfs, int *kob, int *kfs_top, int *kfs_bot, int *kob_top, int *kob_bot, int *kbeg_a,
                             int ld_i2);
/* The same with the input-file switch stabilize_pml (m_medium.f90:219-222,
 * stabilize_absorber :276-340) applied in HBM before the averaged medium, as
 * swpc_setup_medium_opt does on the host. */
int swpc_medium_setup_device_opt(swpc_ctx *ctx, float fq_min, float fq_max, float fq_ref, float *ts, float *scal,
                                 int *kfs, int *kob, int *kfs_top, int *kfs_bot, int *kob_top, int *kob_bot,
                                 int *kbeg_a, int ld_i2, int stabilize_pml);

/* kernel__setup (src/swpc_3d/m_kernel.f90:30-73): FD coefficients from dx,
 * dy, dz and the Zener coefficients c1, c2, d1, d2 from ts(1:nm) and dt,
 * computed in single precision with the reference's expression order. */
int swpc_kernel_setup(swpc_ctx *ctx, const float *ts);

/* absorb_p__setup (src/swpc_3d/m_absorb_p.f90:60-124): the caller passes
 * the damping profiles g(4, n) from damping_profile (:507-547) at cell
 * centres (c) and edges (e) for x (nx), y (ny) and z (nz).  The 18
 * auxiliary fields are allocated only for absorber cells. */
int swpc_absorb_setup(swpc_ctx *ctx, const float *gxc, const float *gxe, const float *gyc, const float *gye,
                      const float *gzc, const float *gze);

/* absorb_c__setup (src/swpc_3d/m_absorb_c.f90:27-103), abc_type = 'cerjan',
 * in place of swpc_absorb_setup: the sponge factors at cell centres (_c) and
 * +d/2 boundaries (_b), n values per axis (swpc_cerjan_profiles).  The
 * interior update then covers the whole domain (m_global.f90:349-378) and
 * the absorber updates multiply by the factors (m_absorb_c.f90:105-198).
 * FP32 storage.  The 2D codes pass gy_c = gy_b = NULL
 * (src/swpc_psv/m_absorb_c.f90, src/swpc_sh/m_absorb_c.f90); a 2D batch
 * applies the sponge of such members after each batched update.  The adjoint
 * and the reciprocity batch refuse such a context. */
int swpc_absorb_setup_cerjan(swpc_ctx *ctx, const float *gx_c, const float *gx_b, const float *gy_c,
                             const float *gy_b, const float *gz_c, const float *gz_b);

/* source__setup (src/swpc_3d/m_source.f90:41-313) after grid assignment and
 * normalisation: nsrc sources at grid (isrc, jsrc, ksrc), srcprm(2, nsrc) =
 * (start time, rise time), mo(nsrc) already divided by M0, m6(6, nsrc) =
 * (mxx, myy, mzz, myz, mxz, mxy).  dt_dxyz = dt / (dx*dy*dz).  The
 * moment-rate function is tabulated for it = 1..nt at t = tbeg + (it-0.5)dt
 * (m_source.f90:800). */
int swpc_source_setup(swpc_ctx *ctx, int nsrc, const int *isrc, const int *jsrc, const int *ksrc,
                      const float *srcprm, const float *mo, const float *m6, int stftype);

/* Body-force mode (bf_mode, m_source.f90:134-137, 835-876): f3(3, nsrc) =
 * (fx, fy, fz) already divided by M0; stime at t = tbeg + it*dt. */
int swpc_bodyforce_setup(swpc_ctx *ctx, int nsrc, const int *isrc, const int *jsrc, const int *ksrc,
                         const float *srcprm, const float *f3, int stftype);

/* Reciprocity source of green__source (src/swpc_3d/m_green.f90:597-632):
 * unit force along cmp ('x','y','z') at one station cell. */
int swpc_green_setup(swpc_ctx *ctx, int isrc, int jsrc, int ksrc, char cmp, float green_tbeg, float green_trise,
                     int stftype);

/* green__store (src/swpc_3d/m_green.f90:389-534): the reciprocity Green's
 * functions at ng grid points (ig, jg, kg in 1..n; the cells of the green
 * table after green__setup's grid assignment).  Each step integrates the
 * nine velocity derivatives (and with bforce the velocities) and every
 * ntdec_w steps samples them into gf(ntw, ncmp*ng), ncmp = 6 (mxx myy mzz
 * myz mxz mxy) or 9 (+ fx fy fz), in the reference's units.  The reference
 * never calls green__store from its main loop; swpc_step and swpc_run call
 * it beside wav__store once this setup has run, and swpc_green_store runs
 * it alone.  swpc_green_fetch copies gf out (column-major, as the reference
 * holds it; green__export's sign flip for green_cmp = 'z' stays with the
 * caller).  FP32 storage. */
int swpc_green_store_setup(swpc_ctx *ctx, int ng, const int *ig, const int *jg, const int *kg, int bforce,
                           int ntdec_w);
int swpc_green_store(swpc_ctx *ctx, int it);
int swpc_green_fetch(swpc_ctx *ctx, float *gf);

/* wav__setup / set_stinfo (src/swpc_3d/m_wav.f90:76-142, 144-274): station
 * cells, decimation, and output scaling M0, UC; what = OR of SWPC_WAV_*. */
int swpc_wav_setup(swpc_ctx *ctx, int nst, const int *ist, const int *jst, const int *kst, int ntdec_w,
                   int what, float M0, float UC);

/* ---- the time step (names follow the reference routines) --------------- */

int swpc_kernel_update_stress(swpc_ctx *ctx);   /* m_kernel.f90:142-326      */
int swpc_absorb_update_stress(swpc_ctx *ctx);   /* m_absorb_p.f90:313-505    */
int swpc_kernel_update_vel(swpc_ctx *ctx);      /* m_kernel.f90:75-140       */
int swpc_absorb_update_vel(swpc_ctx *ctx);      /* m_absorb_p.f90:126-311    */
/* Fused interior + absorber passes: one launch covers the whole domain and
 * computes exactly what kernel__update_* followed by absorb__update_* do. */
int swpc_update_stress(swpc_ctx *ctx);
int swpc_update_vel(swpc_ctx *ctx);
int swpc_source_stressglut(swpc_ctx *ctx, int it);  /* m_source.f90:775-833  */
int swpc_source_bodyforce(swpc_ctx *ctx, int it);   /* m_source.f90:835-876  */
int swpc_green_source(swpc_ctx *ctx, int it);       /* m_green.f90:597-632   */
/* global__comm_stress / global__comm_vel (m_global.f90:393-609): with one
 * domain per GPU every neighbour is MPI_PROC_NULL and the unpack writes
 * zeros into ghost planes that no kernel writes, so these are no-ops kept
 * for call-order fidelity. */
int swpc_comm_stress(swpc_ctx *ctx);
int swpc_comm_vel(swpc_ctx *ctx);

/* ---- decomposed grids (m_global.f90:236-303, 349-378, 393-609) ----------
 * A context becomes one block of a grid split over nproc_x x nproc_y
 * blocks (nproc_x for P-SV and SH): desc.nx / desc.ny are the block's
 * extents, nx_global / ny_global the grid's, and the block's first cell is
 * global cell (ioff + 1, joff + 1); the caller sizes the blocks as
 * global__setup2 does (m_global.f90:236-300).  Call it right after
 * swpc_create, before any medium, kernel or absorber setup: the kernel
 * region then follows the global absorber layout, and the medium, absorber
 * profiles, sources and stations are passed in block coordinates (the
 * medium over the block's memory box, which includes the 3-cell sleeve;
 * source cells anywhere in the sleeve, entries outside the block dropped as
 * the sleeve exchange would overwrite them).  Not with the plane-wave mode,
 * the adjoint or the batches. */
int swpc_set_subdomain(swpc_ctx *ctx, int nx_global, int ny_global, int ioff, int joff);
/* One step of a block: half 0 runs main.f90:125-136 up to
 * global__comm_stress (wav__store, green__store, snapshots, the stress
 * update, absorber, stress glut), half 1 the rest up to global__comm_vel.
 * Between the halves and after half 1 the caller trades the halos. */
int swpc_step_half(swpc_ctx *ctx, int it, int half);
/* Halo exchange after half `half` (0: stress, 1: velocity) with the
 * neighbour on side `side` (0 -x, 1 +x, 2 -y, 3 +y): the planes
 * global__comm_* sends that way (m_global.f90:413-490, 521-603; P-SV and SH
 * from their own m_global.f90) as one flat message of *count floats.
 * swpc_halo_pack writes the message that the neighbour on `side` receives to
 * dst (any device memory this GPU can store to, a peer-mapped buffer
 * included), swpc_halo_unpack writes the message that neighbour sent into
 * this block's sleeve; both are asynchronous on the context's stream.  A
 * side without a neighbour is left alone (its sleeve stays zero, as
 * MPI_PROC_NULL leaves it). */
int swpc_halo_count(swpc_ctx *ctx, int half, int side, long long *count);
int swpc_halo_pack(swpc_ctx *ctx, int half, int side, float *dst);
int swpc_halo_unpack(swpc_ctx *ctx, int half, int side, const float *src);
/* Lets kernels on `device` store to memory of `peer` (cudaDeviceEnablePeerAccess),
 * so that swpc_halo_pack can write a message straight into the receive buffer
 * of a neighbour on another GPU of this process (NVLink peer stores).
 * SWPC_ERR_CUDA when the pair has no peer access. */
int swpc_enable_peer_access(int device, int peer);
/* Plane-wave mode (pw_mode, src/swpc_3d/m_source.f90:67-79): with on != 0
 * the absorber updates first extrapolate the ghost planes of the four side
 * faces from inside (V before the stress update, S before the velocity
 * update; m_absorb_p.f90:136-243, 324-431), and swpc_comm_stress /
 * swpc_comm_vel (and swpc_step, swpc_run) zero the ghost planes that
 * global__comm_stress / global__comm_vel zero on a single domain.  The
 * initial wavefield comes from swpc_pw_setup (swpc_setup.h) through
 * swpc_upload_field.  FP32 storage and the PML only. */
int swpc_set_pw_mode(swpc_ctx *ctx, int on);
int swpc_wav_store(swpc_ctx *ctx, int it);          /* m_wav.f90:400-628     */
/* kernel__vmax (m_kernel.f90:328-352): max |V| one cell below the ocean
 * bottom; blocks.  Sets SWPC_ERR_DIVERGED when max*UC > 1e5
 * (m_report.f90:142-152). */
int swpc_vmax(swpc_ctx *ctx, float out[3]);

/* The same maximum for callers that may not allocate device memory: a solver
 * that keeps Vx, Vy, Vz and kob in device arrays of its own (an OpenACC build
 * of the reference holds them resident for the whole run) and has its device
 * memory claimed up front, so it has no context and cannot have the library
 * call cudaMalloc or cudaFree (which waits for the whole device) at every
 * report.  No counterpart in the reference: it has one kernel__vmax over
 * module arrays.  vx, vy, vz are device arrays over the memory box, k
 * fastest, with leading extents ld_k (>= nz+6) and ld_i (>= nx+6); kob is a
 * device map over (ibeg_m:iend_m, jbeg_m:jend_m) with leading extent ld_i.
 * The range and the result are those of swpc_vmax, and
 * SWPC_ERR_DIVERGED is returned when max*uc > 1e5 or a maximum is NaN.  Work
 * runs on `stream` (a cudaStream_t; NULL = the default stream) of the calling
 * thread's current device, and the call blocks until out[3] (host) is set.
 * Allocates nothing: its scratch is a fixed device array of the library,
 * 3 words per row j, held by every GPU that loads the library until exit, so
 * ny above SWPC_NOALLOC_MAX_NY returns SWPC_ERR_LIMIT.  Every call looks the
 * array's device address up on the current device (nothing is cached, so a
 * cudaDeviceReset between calls is harmless); the first call on a device may
 * load the library's device code, so make it before any stream capture.  All
 * calls on a device share the array: calls that overlap on the GPU (other
 * streams or threads) race and must be serialised. */
#define SWPC_NOALLOC_MAX_NY 16384
int swpc_vmax_noalloc(const float *vx, const float *vy, const float *vz, const int *kob, int nx, int ny, int nz,
                      int na, int ld_k, int ld_i, float uc, void *stream, float out[3]);

/* ---- adjoint and gradient (3D, FP32 storage) ---------------------------- */

/* Discrete adjoint of the step: the exact transpose of update_stress +
 * update_vel (interior, memory variables, ADE-CFS PML, free-surface band).
 * No counterpart in the reference.  The adjoint state uses the field ids of
 * swpc_upload_field (V, S, R, PML auxiliaries).
 *   swpc_adj_reset        zero the adjoint state and the gradients
 *   swpc_adj_step_linear  adjoint <- (one step)^T adjoint, sources off
 *   swpc_adj_upload / _download  adjoint fields in the Fortran memory box
 * swpc_gradient: misfit = 0.5 sum (v_syn - v_obs)^2 over the velocity traces
 * (obs laid out as swpc_wav_fetch's SWPC_WAV_V buffer) of a run from rest over
 * steps 1..nt, and its gradient with respect to the medium arrays of the
 * kernel region.  It runs the forward with a checkpoint every `ckpt` steps,
 * then per segment recomputes the forward from the checkpoint and steps the
 * adjoint back through it, summing each segment's imaging terms in FP32 and
 * folding them into FP64 totals.  Device memory: one checkpoint of the state
 * per recomputed segment, ckpt + 1 working slots (V and the three stress
 * divergences after a step) and the kept steps below.  Every
 * recorder (traces, green__store, snapshots) records the forward run once:
 * the recompute advances the wavefield without them, so what they hold after
 * the call equals a plain run of steps 1..nt from rest.
 * swpc_gradient_set_slot_memory: bytes of HBM that the kept steps of
 * trailing segments may take (default 0).  The first forward pass then keeps,
 * for as many trailing segments as the bytes hold, V of each segment's first
 * state and per step the stress divergences and V on the shell around the
 * kernel region (V of the whole slot box where body forces or green__source
 * write V); those segments are neither checkpointed nor recomputed, their
 * interior V is rebuilt from the divergences with the velocity update's own
 * expression, and only the segments before them are recomputed.  The
 * gradient, the misfit and the recorders are bitwise those of the default.
 * The setting holds for the later swpc_gradient calls of the context.
 * swpc_gradient_memory: bytes of one checkpoint and of one kept step;
 * swpc_gradient_segment_bytes: bytes of a kept segment's first V and of the
 * working slots of a given ckpt; for sizing that budget (free memory from
 * cudaMemGetInfo, say, less the working slots and the checkpoints of the
 * recomputed segments).
 * swpc_gradient_fetch: which = 0 lam, 1 mu, 2 muyz, 3 muxz, 4 muxy, 5 bx,
 * 6 by, 7 bz; out = double array over the memory box. */
int swpc_adj_reset(swpc_ctx *ctx);
/* Zero the forward state (V, S, R, PML auxiliaries) and every recorder total
 * (displacement and strain sums of the stations, green__store's sums,
 * snapshot frames, sums and maxima) for another run from rest on the same
 * context.  No
 * counterpart in the reference, which allocates zeroed arrays once per run
 * (m_kernel.f90:354-378, m_absorb_p.f90:96-116). */
int swpc_reset_state(swpc_ctx *ctx);
int swpc_adj_step_linear(swpc_ctx *ctx);
int swpc_adj_upload(swpc_ctx *ctx, int field, const float *in, int ld_k, int ld_i);
int swpc_adj_download(swpc_ctx *ctx, int field, float *out, int ld_k, int ld_i);
int swpc_gradient(swpc_ctx *ctx, const float *obs, int ckpt, double *misfit);
int swpc_gradient_set_slot_memory(swpc_ctx *ctx, long long bytes);
int swpc_gradient_memory(swpc_ctx *ctx, long long *ckpt_bytes, long long *slot_bytes);
int swpc_gradient_segment_bytes(swpc_ctx *ctx, long long *seg_bytes, long long *work_bytes, int ckpt);
int swpc_gradient_fetch(swpc_ctx *ctx, int which, double *out, int ld_k, int ld_i);
/* The gradient of the last swpc_gradient with respect to per-cell vp, vs and
 * rho with Q held fixed: the chain rule through vmodel_lhm's moduli
 * (src/swpc_3d/m_vmodel_lhm.f90:158-160), relaxed_medium
 * (m_medium.f90:234-274) and averaged_medium's buoyancies and 4-point
 * harmonic rigidities (m_medium.f90:432-465), in FP64 on the device.  No
 * counterpart in the reference.  vp, vs, rho: the model the medium was set up
 * from, over the memory box (host arrays, leading extents ld_k, ld_i);
 * outputs likewise.  The parameters are the cells of the kernel region:
 * absorber cells copy the medium of the region's edge (m_medium.f90:124-190)
 * and their medium is held fixed, so a cell within one cell of the absorber
 * lacks the terms of averaged entries that fall in the absorber. */
int swpc_gradient_model(swpc_ctx *ctx, const float *vp, const float *vs, const float *rho, int ld_k, int ld_i,
                        double *gvp, double *gvs, double *grho);
/* The same with vp, vs, rho and the three gradients as device arrays over
 * the memory box (no host copies). */
int swpc_gradient_model_device(swpc_ctx *ctx, const float *vp, const float *vs, const float *rho, int ld_k, int ld_i,
                               double *gvp, double *gvs, double *grho);

/* ---- reciprocity batch (3D) ---------------------------------------------- */

/* nmem independent wavefields over the medium of one context, each driven by
 * its own single force as green__source drives a green-mode run
 * (src/swpc_3d/m_green.f90:597-632; green__setup :146-154).  No counterpart
 * in the reference, which runs one force per job.  Each member is bitwise
 * the run a context in green mode gives for its force: the step is
 * main.f90:125-144 (wav__store, stress, velocity, green__source), every half
 * step one launch for all members, with the medium of each cell tile read
 * from HBM once for all members.
 *   swpc_fbatch_create        needs medium, kernel and absorber setup on ctx;
 *                             members record at ctx's stations
 *                             (swpc_wav_setup) into their own buffers; the
 *                             batch allocates nmem copies of V, S, R and the
 *                             PML auxiliaries (zero-filled)
 *   swpc_fbatch_green_source  the force of member m (≙ green__setup): unit
 *                             force along cmp ('x','y','z') at cell
 *                             (ksrc, isrc, jsrc), Kupper etc. time function
 *                             from green_tbeg / green_trise
 *   swpc_fbatch_step / _run   one step / nsteps graph replays of all members
 *   swpc_fbatch_set_strip     i-strip width in cells of the flat launch
 *                             order (0 = from the L2 size); _autotune times
 *                             the candidates over steps it0.. and keeps the
 *                             best (see swpc_fbatch_set_launch)
 *   swpc_fbatch_wav_fetch     traces of member m, layout of swpc_wav_fetch
 *   swpc_fbatch_download_field  V, S or R of member m in the memory box
 * The batch borrows ctx, which must outlive it: swpc_destroy refuses a
 * context that still has batches (SWPC_ERR_STATE); ctx's own state and
 * sources are untouched. */
typedef struct swpc_fbatch swpc_fbatch;
int swpc_fbatch_create(swpc_ctx *ctx, int nmem, swpc_fbatch **out);
int swpc_fbatch_destroy(swpc_fbatch *b);
int swpc_fbatch_green_source(swpc_fbatch *b, int member, int isrc, int jsrc, int ksrc, char cmp, float green_tbeg,
                             float green_trise, int stftype);
int swpc_fbatch_set_strip(swpc_fbatch *b, int strip_cells);
/* Launch form of the batch: kernel 0 = the flat one-cell kernels in strip
 * order (swpc_fbatch_set_strip); kernel 5 / 6 = the TMA-staged stress /
 * velocity kernels with tile (bi, bj) and mpc members per CTA, whose CTAs copy
 * the medium of a tile once for the mpc members (FP32 contexts; the default,
 * stress (4,2) and velocity (4,2) with 2 members per CTA).  Compiled stress
 * (bi, bj, mpc): (4,4,1) (2,4,1) (4,2,1) (4,2,2) (2,4,2) (2,2,2) (2,2,4)
 * (4,1,4); velocity: (4,2,1) (4,4,1) (2,2,1) (4,2,2) (2,2,2) (4,1,2) (2,2,4)
 * (4,1,4).  kernel 7 sets the staged launch order: mpc = 0 member groups
 * fastest (the medium of a tile is re-read from L2), 1 tiles fastest (the
 * halos of neighbouring tiles are).  swpc_fbatch_autotune tunes the form in
 * use (strip widths, or the staged order and the shapes of stress then
 * velocity); swpc_fbatch_get_launch writes {staged, strip, stress bi, bj,
 * mpc, velocity bi, bj, mpc, tiles first} to out[9]. */
int swpc_fbatch_set_launch(swpc_fbatch *b, int kernel, int mpc, int bi, int bj);
int swpc_fbatch_get_launch(const swpc_fbatch *b, int *out);
int swpc_fbatch_autotune(swpc_fbatch *b, int it0, int reps, int *steps_used, int *strip);
int swpc_fbatch_step(swpc_fbatch *b, int it);
int swpc_fbatch_run(swpc_fbatch *b, int it0, int nsteps);
int swpc_fbatch_time_steps(swpc_fbatch *b, int it0, int nsteps, float *ms);
int swpc_fbatch_sync(swpc_fbatch *b);
int swpc_fbatch_wav_fetch(swpc_fbatch *b, int member, int what, float *out);
int swpc_fbatch_download_field(swpc_fbatch *b, int member, int field, float *out, int ld_k, int ld_i);
/* green__store of one member: the context's green table (set up before
 * swpc_fbatch_create) is recorded for every member; gf as swpc_green_fetch. */
int swpc_fbatch_green_fetch(swpc_fbatch *b, int member, float *gf);
long long swpc_fbatch_device_bytes(const swpc_fbatch *b);

/* ---- snapshots (3D) ------------------------------------------------------ */

/* Snapshot planes of snap__setup (src/swpc_3d/m_snap.f90:95-322): a plane is
 * a section (yz at i0_yz, xz at j0_xz, xy at k0_xy, fs one cell below the
 * free surface, ob one cell below the ocean bottom) times a quantity (ps:
 * div, rot_x, rot_y, rot_z masked by lam/mu; v: Vx, Vy, Vz; u: displacement),
 * bit SWPC_SNP_BIT(section, quantity) of `planes`.  Samples are decimated by
 * idec/jdec/kdec (nxs = (nx + idec/2)/idec, ...); frames are taken at
 * it = 1, 1 + ntdec_s, ... <= nt.  i0_yz, j0_xz, k0_xy are grid indices
 * (x2i / y2j / z2k of x0_yz, y0_xz, z0_xy, m_snap.f90:157-159).  M0 and UC
 * scale to physical units as wav__store does.  The frames stay in HBM for the
 * run; the file writers (native .snp / NetCDF) stay with the caller. */
#define SWPC_SNP_YZ 0
#define SWPC_SNP_XZ 1
#define SWPC_SNP_XY 2
#define SWPC_SNP_FS 3
#define SWPC_SNP_OB 4
#define SWPC_SNP_PS 0
#define SWPC_SNP_V 1
#define SWPC_SNP_U 2
#define SWPC_SNP_BIT(section, quantity) (1 << (3 * (section) + (quantity)))
typedef struct swpc_snap_desc {
    int planes;                 /* OR of SWPC_SNP_BIT(...)                     */
    int idec, jdec, kdec;       /* spatial decimation                          */
    int ntdec_s;                /* time decimation                             */
    int i0_yz, j0_xz, k0_xy;    /* section positions (grid indices)            */
    float M0, UC;               /* output scaling (m_snap.f90:1022-1025)       */
} swpc_snap_desc;
int swpc_snap_setup(swpc_ctx *ctx, const swpc_snap_desc *d);
/* snap__write (m_snap.f90:911-939) for step it (1..nt; nt+1 updates the
 * displacement sums and maxima once more, as snap__closefiles does before the
 * NetCDF maxima are written).  swpc_step / swpc_run call it after wav__store
 * once snapshots are set up. */
int swpc_snap_write(swpc_ctx *ctx, int it);
/* plane = 3*section + quantity: buffer (n1, n2, nvar) per frame in Fortran
 * order, n1 fastest (yz: nys x nzs, xz: nxs x nzs, xy/fs/ob: nxs x nys). */
int swpc_snap_dims(const swpc_ctx *ctx, int plane, int *nvar, int *n1, int *n2, int *nframes);
/* All frames of a plane: out(n1, n2, nvar, nframes), Fortran order; blocks. */
int swpc_snap_fetch(swpc_ctx *ctx, int plane, float *out);
/* Running maxima max_fs_v, max_fs_u, max_ob_v, max_ob_u (which = 0..3) as
 * (nxs, nys, 3): vertical, horizontal, vector (m_snap.f90:1691-1703,
 * output__put_maxval :2291-2344); needs the matching fs/ob v or u plane. */
int swpc_snap_fetch_max(swpc_ctx *ctx, int which, float *out);

/* One full step in main.f90 order: wav__store, snap__write, update_stress
 * (fused), stressglut, comm, update_vel (fused), bodyforce, green, comm. */
int swpc_step(swpc_ctx *ctx, int it);
/* Steps it0 .. it0+nsteps-1 as replays of a captured CUDA graph. */
int swpc_run(swpc_ctx *ctx, int it0, int nsteps);
/* Device time of `nsteps` steps from it0 (CUDA events on the context's
 * stream); result in milliseconds. */
int swpc_time_steps(swpc_ctx *ctx, int it0, int nsteps, float *ms);

/* ---- data movement ------------------------------------------------------ */

/* wav buffers in the reference layout wav_*(ntw, ncmp, nst) (m_wav.f90:37-38). */
int swpc_wav_fetch(swpc_ctx *ctx, int what, float *out);
int swpc_wav_dims(const swpc_ctx *ctx, int *ntw, int *nst);
/* One field in the Fortran memory-box layout (ld_k, ld_i as above).  Uploads
 * of a box of 256 KB or more (here and in swpc_upload_medium) travel in
 * contiguous chunks of planes through a staging buffer of the context (about
 * 16 MB, allocated by the first such upload and kept until swpc_destroy;
 * counted by swpc_device_bytes); pinned host memory makes them fastest. */
int swpc_download_field(swpc_ctx *ctx, int field, float *out, int ld_k, int ld_i);
int swpc_upload_field(swpc_ctx *ctx, int field, const float *in, int ld_k, int ld_i);
/* Memory-variable and PML-auxiliary fields are defined only on their
 * regions; outside them download writes 0 and upload ignores the input. */

/* SWPC_PREC_F16_SR and SWPC_PREC_F16_R (a no-op otherwise): re-centre the
 * power-of-two scale of every FP16 stress and memory-variable array now, so
 * that its largest stored magnitude lies in [2^7, 2^8) whenever it has left
 * [2^3, 2^10); that leaves at least 64x headroom below the FP16 overflow.
 * Scaling by a power of two is exact.  The time step does the same on the
 * device every 8 steps (swpc_run, swpc_step, swpc_step_half: a measuring
 * kernel before the stress update, which converts the values as it rewrites
 * them; inside the captured graph, without the host), so a caller need not;
 * *changed (may be NULL) = arrays moved.  Blocks.  No counterpart in the
 * reference. */
int swpc_rescale(swpc_ctx *ctx, int *changed);

/* Device bytes held by the context. */
long long swpc_device_bytes(const swpc_ctx *ctx);

/* Launch variant of the fused kernels.  kernel 0 / 1 select the flat stress /
 * velocity kernels (one thread per cell, block = 32 (k) x bi (i) x bj (j)
 * threads, 32*bi*bj <= 256); kernel 2 / 3 select the 2.5D marching stress /
 * velocity kernels (a 32 x 8 (k, i) tile walking bj planes along j; bi is
 * ignored).  minb = minimum resident blocks per SM the variant is compiled
 * for (1..4; fewer blocks leave more registers for operands in flight).
 * kernel 4 selects the velocity kernel with four k per thread.  kernel 5 / 6
 * select the TMA-staged stress / velocity kernels (FP32 3D contexts): a CTA
 * per tile of 32 (k) x bi (i) x bj (j) cells whose operands arrive in shared
 * memory by bulk tensor copies; minb must be 1, and the compiled tiles
 * (bi, bj) are stress (4,4) (2,4) (4,2), velocity (4,4) (4,2) (2,2); the
 * reduced storage forms (BF16_R, F16_SR) compile (4,4) and (4,2) for both.
 * 3D contexts start with kernels 5 (4,4) and 6 (4,4); the reduced storage
 * forms with kernel 5 on (4,2).
 * kernel 7 (3D) sets the launch order of the staged kernels: tiles run k
 * fastest, then over (i, j) in blocks of bi consecutive j tiles (j fastest
 * within a block), so that a tile's j-halo is still in L2; bi = 1 runs i then
 * j, bi = 0 (the default) takes 16 when a j plane of tiles outgrows half of
 * the L2 and 1 otherwise.
 * kernel 8 (3D) selects the stress-phase weights kernel of the adjoint step
 * (swpc_adj_*, swpc_gradient): bi = 1 the TMA-staged kernel (default), 0 the
 * one-cell-per-thread kernel.
 * kernel 9 (3D) selects how swpc_gradient forms the velocity-phase weights
 * of the adjoint step: bi = 1 (default) inside the stress-phase gather of the
 * step before, from the lambda_V it has just summed (the cells whose
 * lambda_V receiver residuals change afterwards are formed again after the
 * injection), 0 by a kernel of their own in every step.
 * 2D contexts (P-SV, SH) take kernels 0 / 1 (the tile-walking stress /
 * velocity kernels) and 5 / 6 (the staged ones: a CTA per 32 x 16 tile with
 * bi = 4, 8 or 16 threads along i, minb 1, bj 1); they start with kernels
 * 5 and 6 at bi = 8.
 * The defaults come from sweeps on B200.  No counterpart in the reference
 * (its OpenMP/OpenACC schedules are fixed at compile time); results are
 * bitwise independent of the variant. */
int swpc_set_launch(swpc_ctx *ctx, int kernel, int minb, int bi, int bj);

/* ---- batched 2D ensemble ----------------------------------------------- */

/* Many independent 2D runs (P-SV or SH, same nm and device, each a fully set
 * up context with its own medium, sources and stations) advanced together:
 * every half step is ONE persistent launch over the tiles of all members,
 * and swpc_batch_run replays the captured step as a CUDA graph.  This
 * replaces the reference's one-process-per-run ensemble loop
 * (work/auto_chengyu.py:68-110) and has no counterpart inside the solver.
 * The batch snapshots its members at creation: set every member up first.
 * Batch work runs on the batch's own stream; call swpc_batch_sync before
 * reading a member's fields or traces (it also reports a staged tile copy
 * that did not complete, SWPC_ERR_CUDA). */
typedef struct swpc_batch swpc_batch;
int swpc_batch_create(swpc_ctx *const *members, int n, swpc_batch **out);
int swpc_batch_step(swpc_batch *b, int it);
int swpc_batch_run(swpc_batch *b, int it0, int nsteps);
int swpc_batch_sync(swpc_batch *b);
int swpc_batch_time_steps(swpc_batch *b, int it0, int nsteps, float *ms);
/* Autotuner of the batched launch.  Candidates: the TMA-staged kernels on
 * tiles of 32 (k) x 16 (i) cells with 4, 8 or 16 threads along i in the
 * stress and velocity CTAs, and the tile-walking kernels on tiles of 32 (k) x
 * (ti*ri) (i) cells, a block of 32 x ti threads with ri rows per thread, a
 * persistent grid of 148 x bps blocks (bps = 0: one block per tile).  It
 * advances the batch by real time steps from it0 -- every candidate runs
 * `reps` steps timed with CUDA events (12 candidates) -- and keeps the
 * fastest; the results do not depend on the launch, so these are ordinary
 * steps of the run.  *used = steps taken (it0 .. it0 + *used - 1); *best_ti,
 * *best_ri, *best_bps (may be NULL) = the tile shape of the pick (see
 * swpc_batch_get_launch for the whole pick).  No counterpart in the
 * reference. */
int swpc_batch_autotune(swpc_batch *b, int it0, int reps, int *used, int *best_ti, int *best_ri, int *best_bps);
/* Sets the tile shape directly (ti threads in i per block, 32*ti <= 256;
 * ri rows per thread; bps blocks per SM of the persistent grid, 0 = one block
 * per tile).  A shape with ti*ri != 16 selects the tile-walking kernels. */
int swpc_batch_set_shape(swpc_batch *b, int ti, int ri, int bps);
/* Selects the TMA-staged kernels (stress_ti / vel_ti = 4, 8 or 16 threads
 * along i of the stress / velocity CTA) or the tile-walking kernels (0) per
 * phase; staged kernels switch the tiles to 32 x 16.  A new batch starts
 * with both phases staged at 8. */
int swpc_batch_set_staged(swpc_batch *b, int stress_ti, int vel_ti);
/* The current launch: out[5] = ti, ri, bps, stress_ti, vel_ti. */
int swpc_batch_get_launch(const swpc_batch *b, int *out);
const char *swpc_batch_last_error(const swpc_batch *b);
int swpc_batch_destroy(swpc_batch *b);

#ifdef __cplusplus
}
#endif
#endif
