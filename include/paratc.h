/*
 * paratc.h -- C ABI of the B200-native ParaTC per-RK3-substep hot path.
 *
 * The hot path of ParaTC (GongZheng-Justin/ParaTC) is the explicit 4th-order
 * staggered right-hand side (src/m_TScheme.f90), the implicit wall-normal
 * Helmholtz tridiagonal solves (src/m_TScheme.f90:365-506 with
 * src/m_Tools.f90:224-251), the FFT-tridiagonal pressure Poisson solve
 * (src/m_Poisson.f90) and the wall/periodic boundary treatment
 * (src/m_BC_and_Halo.f90).  In the reference these are Fortran module
 * procedures called in a fixed order by ChannelIterate
 * (src/m_ChannelSystem.f90:80-187); here they are one library whose entry
 * points take plain pointers and sizes and return an int status.
 *
 * Conventions
 *  - Every entry point returns PARATC_OK (0) or a negative PARATC_ERR_* code.
 *    The reference aborts instead (MainLog%CheckForError(ErrT_Abort, ...),
 *    src/m_LogInfo.f90; MPI_ABORT in src/m_Decomp2d.f90); a Fortran caller
 *    maps a non-zero status to ErrT_Abort to keep that behaviour.
 *  - Host arrays are FP64, Fortran order (x fastest, then y, then z).
 *    PARATC_LAYOUT_INTERIOR: nxc*nyc*nzc values, indices ic=1..nxc,
 *    jc=1..nyc, kc=1..nzc (the y1 pencil of one rank, y1start..y1end).
 *    PARATC_LAYOUT_HALO: (nxc+4)*(nyc+2)*(nzc+4) values with the bounds
 *    mb1%xmm:xpm = -1:nxc+2, ymm:ypm = 0:nyp, zmm:zpm = -1:nzc+2 that
 *    myallocate gives the field arrays (src/m_Variables.f90:47-50,
 *    src/m_Decomp2d.f90:1479-1549).
 *  - A context is bound to one CUDA device and one stream. Calls on one
 *    context must not run concurrently; different contexts are independent.
 *  - The library owns all device memory of a context.
 */
#ifndef PARATC_H
#define PARATC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define PARATC_OK              0
#define PARATC_ERR_BAD_ARG    -1  /* invalid size, option or pointer             */
#define PARATC_ERR_OOM        -2  /* device or host allocation failed            */
#define PARATC_ERR_CUDA       -3  /* a CUDA runtime call failed                  */
#define PARATC_ERR_NONFINITE  -4  /* NaN/Inf found in a field                    */
#define PARATC_ERR_DIV_LIMIT  -5  /* max|div u| > div_limit (ChannelIterate:143) */
#define PARATC_ERR_VEL_LIMIT  -6  /* min(max|u_i|) > vel_limit (ChannelIterate:145) */
#define PARATC_ERR_TIMEOUT    -7  /* a bounded device wait gave up; the context
                                     keeps reporting it: destroy and recreate it */
#define PARATC_ERR_IO         -8  /* restart file missing, short or wrong size   */
#define PARATC_ERR_NO_DEVICE  -9  /* no CUDA device / library built without one  */
#define PARATC_ERR_NUMERIC   -10  /* lambda2 met complex roots (Clc_lamda2 stops) */

/* ---- option values (same numbers as src/m_Parameters.f90) ------------ */
#define PARATC_FT_CH 1          /* FT_CH: channel, no-slip top and bottom   */
#define PARATC_FT_HC 2          /* FT_HC: half channel, free-slip top       */
#define PARATC_AB2   1          /* FI_AB2 */
#define PARATC_RK2   2          /* FI_RK2 */
#define PARATC_RK3   3          /* FI_RK3 */

#define PARATC_LAYOUT_INTERIOR 0
#define PARATC_LAYOUT_HALO     1

/*
 * Run-time parameters. The values are the ones the module m_Parameters holds
 * after ReadAndInitParameters (src/m_Parameters.f90:112-188): uCRF is 0 unless
 * IsUseCRF, uxBcValue already has uCRF subtracted, the scalar vectors are
 * GravityEffVec = GravityDir*GravityEff and FallingVelVec = GravityDir*FallingVel
 * (+uCRF in x), SDiffCoe = xnu/SchmidtNumber.  paratc_params_from_namelist()
 * fills the struct from a ParaTC input file exactly that way.
 */
typedef struct paratc_params {
    int32_t nxc, nyc, nzc;      /* cell counts: nxp-1, nyp-1, nzp-1            */
    int32_t flow_type;          /* PARATC_FT_CH | PARATC_FT_HC                 */
    int32_t ischeme;            /* PARATC_AB2 | PARATC_RK2 | PARATC_RK3        */
    int32_t icfl;               /* 1: dt from CFLc, 2: dt = dtMax              */
    int32_t is_ux_const;        /* IsUxConst: constant flow-rate forcing       */
    int32_t scalar_on;          /* built with -DScalarFlow in the reference    */
    double  xlx, yly, zlz;      /* domain lengths                              */
    double  xnu;                /* kinematic viscosity                         */
    double  ubulk;              /* bulk velocity                               */
    double  ucrf;               /* uCRF (0 when IsUseCRF is false)             */
    double  dt_max;             /* dtMax                                       */
    double  cflc;               /* CFLc                                        */
    double  gravity[3];         /* constant body force                         */
    double  ux_bc[6], uy_bc[6], uz_bc[6];   /* u?BcValue, index 0..5 = x-,x+,y-,y+,z-,z+ */
    double  vel_limit, div_limit;
    /* ScalarFlow options (ignored when scalar_on == 0) */
    double  sdiff;              /* SDiffCoe                                    */
    double  gravity_eff_vec[3]; /* GravityEffVec                               */
    double  falling_vel_vec[3]; /* FallingVelVec                               */
    int32_t scalar_bc_option[2];/* -1 Dirichlet, -2 Neumann, -3 Robin; y-, y+  */
    double  scalar_bc_values[4];/* F_b, F_t, S_b, S_t                          */
    double  scalar_init_value;  /* Scalar_InitValue                            */
} paratc_params;

/* Per-step diagnostics, the numbers ChannelIterate logs
 * (src/m_ChannelSystem.f90:172-183). */
typedef struct paratc_diag {
    double dt;            /* time step used by this step                       */
    double cfl;           /* cflmp = uddxmax*dt_prev (ChannelIterate:93-94)    */
    double sim_time;      /* SimTime after the step                            */
    double divmax_src;    /* divmax1: max|div u*| seen by the last clcPrSrc    */
    double divmax;        /* divmax2: CheckDivergence after the step           */
    double vmax[3];       /* CalcVmax                                          */
    double pr_grad_aver;  /* PrGradAver (mean pressure gradient of the step)   */
    double ux_mean;       /* CalcUxAver / ClcMeanValue(1)                      */
    double sc_mean;       /* ClcMeanValue(2) (0 without scalar)                */
    double sc2_mean;      /* ClcMeanValue(3) raw mean of c^2 (0 without scalar)*/
} paratc_diag;

typedef struct paratc_ctx paratc_ctx;

/* ---- set-up ------------------------------------------------------------ */

/* clcYcoord for every section (src/m_MeshAndMetries.f90:143-181,340-408):
 * fills yp[0..nyp-1] = yp(1..nyp) from the &MeshOptions arrays. */
int paratc_mesh_ycoord(int nsection, const double* section_length,
                       const double* section_cstret, const int32_t* nyc_section,
                       const int32_t* stret_type, const int32_t* stret_option,
                       double yly, double* yp_out);

/* Reads &BasicParam, &MeshSection, &MeshOptions and (when scalar_on != 0)
 * &ScalarFlowOptions from a ParaTC input file and applies the derivations
 * of ReadAndInitParameters (src/m_Parameters.f90:112-188).  yp_out may be
 * NULL (pass nyp_cap = 0); otherwise it receives yp(1..nyp). */
int paratc_params_from_namelist(const char* path, int scalar_on,
                                paratc_params* out, double* yp_out, int nyp_cap);

/* Run control of &BasicParam that main.f90 / ChannelIterate use around the
 * hot path (src/main.f90:31-33, src/m_ChannelSystem.f90:150-183). */
typedef struct paratc_run_options {
    int32_t ifirst, ilast;      /* iteration range                             */
    int32_t restart_flag;       /* RestartFlag                                 */
    int32_t backup_freq;        /* BackupFreq                                  */
    int32_t cmd_lfile_freq;     /* Cmd_LFile_Freq                              */
    char run_name[64];          /* RunName                                     */
    char res_dir[256];          /* Res_Dir                                     */
    char restart_dir[256];      /* RestartDir                                  */
} paratc_run_options;
int paratc_run_options_from_namelist(const char* path, paratc_run_options* out);

/* ChannelInitialize minus IO (src/m_ChannelSystem.f90:26-75): metrics
 * (InitMeshAndMetries), wavenumbers (InitPoissonSolver:36-48), field storage
 * (AllocateVariables, all zero, scalar = Scalar_InitValue).  yp has nyp
 * entries yp(1..nyp).  device < 0 means the current device. */
int paratc_create(const paratc_params* prm, const double* yp, int device,
                  paratc_ctx** out);
int paratc_destroy(paratc_ctx* ctx);

/* The CUDA stream of the context (a cudaStream_t), for callers that order
 * their own work or events against it. */
void* paratc_stream(paratc_ctx* ctx);

/* ---- state in / out ---------------------------------------------------- */

/* Loads ux, uy, uz, p (c when scalar_on) and the explicit histories
 * HistX/Y/Z(/C) (NULL = zero), then applies SetBC_and_UpdateHalo,
 * SetBC_and_UpdateHalo_pr and SetBC_and_UpdateHalo_scalar as
 * ChannelInitialize does (src/m_ChannelSystem.f90:63-68).  ux is the
 * velocity in the computing frame (the restart file holds ux+uCRF). */
int paratc_set_fields(paratc_ctx* ctx, const double* ux, const double* uy,
                      const double* uz, const double* p, const double* c,
                      const double* hx, const double* hy, const double* hz,
                      const double* hc, int layout);
/* Any output pointer may be NULL. */
int paratc_get_fields(paratc_ctx* ctx, double* ux, double* uy, double* uz,
                      double* p, double* c, double* hx, double* hy, double* hz,
                      double* hc, int layout);

/* Same as the pair above with device pointers (interior layout). */
int paratc_set_fields_device(paratc_ctx* ctx, const double* ux, const double* uy,
                             const double* uz, const double* p, const double* c,
                             const double* hx, const double* hy, const double* hz,
                             const double* hc);
int paratc_get_fields_device(paratc_ctx* ctx, double* ux, double* uy, double* uz,
                             double* p, double* c, double* hx, double* hy,
                             double* hz, double* hc);

/* Asynchronous forms: the copies (and the boundary / ghost refresh of
 * set_fields) are queued on the context's stream and the call returns at
 * once; the host arrays must stay valid, and should be page-locked, until
 * paratc_sync (or a synchronous call) returns.  Independent contexts used this
 * way overlap one context's transfers with another's steps. */
int paratc_set_fields_async(paratc_ctx* ctx, const double* ux, const double* uy, const double* uz,
                            const double* p, const double* c, const double* hx, const double* hy,
                            const double* hz, const double* hc, int layout);
int paratc_get_fields_async(paratc_ctx* ctx, double* ux, double* uy, double* uz, double* p, double* c,
                            double* hx, double* hy, double* hz, double* hc, int layout);
/* Waits for everything queued on the context's stream. */
int paratc_sync(paratc_ctx* ctx);

/* SimTime and dt of the context (m_Parameters globals).  After a step,
 * paratc_get_time reports the dt that step used (the device already holds
 * the next step's dt, computed from the same velocity by the step's end
 * kernel).  paratc_set_time makes the next step recompute its CFL. */
int paratc_set_time(paratc_ctx* ctx, double sim_time, double dt);
int paratc_get_time(paratc_ctx* ctx, double* sim_time, double* dt);

/* ---- the hot path ------------------------------------------------------- */

/* One time step = ChannelIterate without statistics/visu/restart IO
 * (src/m_ChannelSystem.f90:80-187): CFL -> dt, iadvance substeps,
 * CheckDivergence / CalcVmax and their limits.  diag may be NULL.
 * Returns PARATC_ERR_DIV_LIMIT / PARATC_ERR_VEL_LIMIT where the reference
 * aborts; the fields then hold the state after the step. */
int paratc_step(paratc_ctx* ctx, paratc_diag* diag);

/* n steps back to back; diag (may be NULL) receives the last step's numbers.
 * The per-step guard readback is done once at the end. */
int paratc_steps(paratc_ctx* ctx, int n, paratc_diag* diag);

/* Enqueues n steps on the context's stream and returns without waiting;
 * the guards are evaluated on the device.  paratc_last_diag() (or any
 * synchronising call) then reports the diagnostics and the first failing
 * guard of the steps enqueued since the previous paratc_last_diag. */
int paratc_steps_async(paratc_ctx* ctx, int n);
int paratc_last_diag(paratc_ctx* ctx, paratc_diag* diag);

/* One substep ns (1..iadvance) with time step dt: PMcoeUpdate(ns) and the body
 * of the ns loop (src/m_ChannelSystem.f90:102-140). divmax_src may be NULL. */
int paratc_substep(paratc_ctx* ctx, int ns, double dt, double* divmax_src);

/* Inspection: the substep above stopped after stage stop_stage (1 clcRhsXYZ
 * with the flow-rate constraint, 2 the Helmholtz solves clcU1Hat/clcU2Hat/
 * clcU3Hat/clcScalar, 3 clcPrSrc, 4 clcPPE, 5 complete), so that each
 * reference routine can be compared on its own. */
int paratc_substep_stage(paratc_ctx* ctx, int ns, double dt, int stop_stage,
                         double* divmax_src);

/* Inspection: copies a work array in interior layout to host memory:
 * 0 RhsX (with the flow-rate term), 1 RhsY, 2 RhsZ, 3 RhsC, 4 prsrc, 5 phi.
 * The Rhs arrays hold the right-hand sides after a substep stopped at stage 1
 * (the Helmholtz forward sweep overwrites them, as InverseTridiagonal
 * overwrites its right-hand side in the reference); prsrc is filled by a
 * substep stopped at stage 3. */
int paratc_get_work(paratc_ctx* ctx, int which, double* out);

/* clcPPE (src/m_Poisson.f90:352-452, choice 1 on one rank): solves
 * Lap4(phi) = src with 4th-order modified wavenumbers in x/z, the 2nd-order
 * Neumann y operator, phi_hat(kx=0,kz=0,jc=1) = 0, scaled by 1/(nxc*nzc).
 * src and phi are host arrays in interior layout (phi may equal src). */
int paratc_poisson(paratc_ctx* ctx, const double* src, double* phi);
/* Same with device pointers (interior layout, nxc*nyc*nzc doubles). */
int paratc_poisson_device(paratc_ctx* ctx, const double* d_src, double* d_phi);
/* As paratc_poisson_device, but returns once the solve is queued on the
 * context's stream (paratc_stream), without waiting for it. */
int paratc_poisson_device_async(paratc_ctx* ctx, const double* d_src, double* d_phi);

/* clcPPE by FP32 solves with FP64 iterative refinement.  No counterpart in
 * the reference (its solve is FP64).  The first solve takes the FP64 source
 * d_src through a spectrum stored in FP32 (the transform and Thomas passes
 * compute in FP64) into d_phi; each correction computes the FP64 residual
 * r = src - L phi of the discrete operator the spectral solve inverts
 * (4th-order D4 D4 in x and z, the Neumann y operator), solves L d = r the
 * same way and adds d to phi.  Stops when max|r| <= rtol * max|src| or after
 * max_corr corrections; ncorr and relres (may be NULL) receive the count and
 * the final max|r| / max|src|.  The source must have zero mean (the gauge
 * phi_hat(0,0,1) = 0 of the FP64 solve is kept).  Device pointers, compact
 * interior layout, d_src != d_phi; needs compile-time-length transforms. */
int paratc_poisson_refined(paratc_ctx* ctx, const double* d_src, double* d_phi, double rtol, int max_corr,
                           int* ncorr, double* relres);
/* The same with exactly ncorr corrections, queued on the context's stream
 * without reading the residual back (for timing). */
int paratc_poisson_refined_async(paratc_ctx* ctx, const double* d_src, double* d_phi, int ncorr);

/* Poisson solve that allocates no memory.  No counterpart in the reference:
 * it exists for callers that cannot call cudaMalloc (a loop with a fixed
 * memory budget, a host code whose allocator owns all device memory, a
 * caller that cannot keep a context alive between calls).  It solves the same
 * system as paratc_poisson_device() for the grid of *prm and the y-grid yp
 * (yp(1..nyp)), d_src -> d_phi (device pointers, interior layout), on
 * `stream` (a cudaStream_t, NULL = default), and waits for the stream.
 * Working memory is one fixed device array inside the library of
 * PARATC_NOALLOC_SCRATCH_DOUBLES doubles (16 MiB, held by every GPU that
 * loads the library until exit): grids needing more than
 * 2*(nxc/2+1)*nyc*nzc + O(nxc+nyc+nzc) doubles, or nxc/nzc > 1024, nyc > 256,
 * are rejected with PARATC_ERR_BAD_ARG.  The first call on a device looks up
 * the array's device address (once per device, safe from several host
 * threads; cudaDeviceReset after it is not supported).  The call must not be
 * made while `stream` is being captured into a CUDA graph: it copies tables
 * from its stack frame (about 68 KB at the largest sizes) and waits for the
 * stream, and returns PARATC_ERR_BAD_ARG during capture.  All calls share the
 * array: calls that overlap on the GPU race. */
#define PARATC_NOALLOC_SCRATCH_DOUBLES (2 * 1024 * 1024)
int paratc_poisson_noalloc(const paratc_params* prm, const double* yp,
                           const double* d_src, double* d_phi, void* stream);

/* Makes the current velocity field discretely solenoidal with one pressure-free
 * projection (u -= grad(phi), Lap4(phi) = div u), the same operators as a
 * substep; used to prepare seeded initial fields. divmax_out may be NULL. */
int paratc_project(paratc_ctx* ctx, double* divmax_out);

/* Reductions of src/m_Tools.f90 on the current fields. */
int paratc_diagnostics(paratc_ctx* ctx, paratc_diag* diag);

/* x profile of a field averaged over the depth and the span,
 * out[i] = sum_kc sum_jc q(ic, jc, kc) dyp(jc) / (nzc yly), ic = i+1, for
 * field 0 ux, 1 uy, 2 uz, 3 p, 4 scalar (out: nxc doubles).  No counterpart
 * in the reference; it is the depth-averaged concentration from which a
 * gravity current's front is read. */
int paratc_xprofile(paratc_ctx* ctx, int field, double* out);
/* Front (nose) of a gravity current released from a lock ending at x_from:
 * the furthest cell centre (ic-0.5)*dx to the right of x_from, within half
 * the periodic domain, where the depth-averaged scalar is at least `level`,
 * moved to the level's linear crossing between that cell and the next;
 * -1 when no cell there reaches `level`.  Not in the reference (a
 * builder-defined diagnostic of the lock-exchange case). */
int paratc_front_position(paratc_ctx* ctx, double x_from, double level, double* x_front);

/* ---- restart files (src/m_IOAndVisu.f90:408-512) ----------------------- */
/* Raw FP64, headerless, Fortran order: ux+uCRF, uy, uz, p, [c],
 * [HistX, HistY, HistZ, [HistC]] (histories only when with_hist != 0). */
int paratc_write_restart(paratc_ctx* ctx, const char* path, int with_hist);
int paratc_read_restart(paratc_ctx* ctx, const char* path);

/* ---- errors -------------------------------------------------------------- */
const char* paratc_strerror(int status);
/* Text of the last failure on this context (empty when none). */
const char* paratc_last_error(paratc_ctx* ctx);

/* Number of kernel launches issued by this context since creation. */
int64_t paratc_launch_count(paratc_ctx* ctx);

/* ---- per-kernel timing (CUDA events around every launch, off by default) */
#define PARATC_PROF_NKERNELS 16
/* on != 0 starts recording (and clears the totals), 0 stops. */
int paratc_profile_enable(paratc_ctx* ctx, int on);
/* Device time (ms, summed) and launch count of kernel class k in
 * [0, PARATC_PROF_NKERNELS) since the last enable; the pending events are
 * resolved first (this synchronises the stream). */
int paratc_profile_get(paratc_ctx* ctx, int k, double* total_ms, int64_t* launches);
/* Name of kernel class k ("rhs", "helmholtz", "fft_x_fwd", ...). */
const char* paratc_profile_name(int k);

/* ---- bounded device waits.  No counterpart in the reference (its MPI calls
 * block).  Every pipeline wait of the TMA-fed kernels (z transforms, x
 * transforms, divergence-fed x transform) polls its
 * mbarrier at most 2^22 times; a CTA whose wait runs out records the failure,
 * waits (with the full limit) for its own copies still in flight and returns,
 * and the next synchronising call reports PARATC_ERR_TIMEOUT.  This sets the
 * poll limit of those pipeline waits on this context: polls >= 0 allows that
 * many polls (0: give up at the first wait), polls < 0 restores the default.
 * It exists so that tests can drive the timeout path without stalling a GPU. */
int paratc_set_wait_limit(paratc_ctx* ctx, long long polls);

/* ---- precision of the step.  PARATC_PREC_FP64 (the default) is the
 * reference's arithmetic.  PARATC_PREC_MIXED computes the explicit
 * right-hand side (clcRhsXYZ's stencils, interpolations and products) in
 * FP32 arithmetic from the FP64 state and writes it in FP64; the state, the
 * explicit histories, the Helmholtz and Poisson solves, the projection, the
 * flow-rate constraint sum (s3tot) and every reduction stay FP64, so the
 * divergence after a step is at the FP64 level while the fields differ from
 * the FP64 path by the FP32 rounding of one explicit term per substep.
 * PARATC_PREC_FP32 is the FP32 storage form: u, v, w, the scalar, the
 * explicit histories, the right-hand sides, the spectrum of the Poisson
 * solve and the potential are stored in FP32 (half the bytes of every pass
 * over them); the pressure stays FP64.  The right-hand side is computed in
 * FP32 arithmetic; the Helmholtz sweeps, the transforms, the spectral y-solve
 * (with its kx = kz = 0 mean mode) and the projection in FP64 arithmetic on
 * values loaded from FP32; the flow-rate constraint, the guards and the
 * statistics in FP64.  The divergence of the FP32-stored velocity is limited
 * by its rounding (about 1e-7 of |u|/dx), not by the solves.  Switching to or
 * from FP32 converts the state; statistics, spectra, visualisation, restart
 * and get_fields read an FP64 copy refreshed from it.  The FP32 form needs
 * nxc % 4 == 0 and compile-time-length transforms for nxc/2 and nzc (else
 * PARATC_ERR_BAD_ARG) and runs the plane or separate x/z transform kernels of the context's
 * schedule (the TMA-fed variants stay FP64). */
#define PARATC_PREC_FP64  0
#define PARATC_PREC_MIXED 1
#define PARATC_PREC_FP32  2
int paratc_set_precision(paratc_ctx* ctx, int prec);
int paratc_get_precision(paratc_ctx* ctx, int* prec);

/* ---- Poisson schedule auto-tuning (the four-choice search of
 * InitPoissonSolver, src/m_Poisson.f90:50-175, which times 15 solves of each
 * transpose/solver variant and keeps the fastest).  The schedules here:
 * choice = 2*s + y, s = 0 fused y-plane transforms (grids whose plane fits
 * one CTA), 1 separate compile-time-length x and z transforms, 2 generic
 * mixed-radix transforms (any 2^a 3^b 5^c size), 3 as 1 with the z
 * transforms fed by TMA (persistent CTAs, two shared-memory stages; nz in
 * 128, 256, 512, 768, 1024), 4 as 1 with the divergence source computed by
 * producer warps into the stages of the forward x transform
 * (warp-specialised, one CTA per SM), 5 as 4 with the z transforms of 3;
 * y = 0 staged (one-warp CTAs, cp.async
 * row staging), 1 streaming (a thread per column) spectral y-solve.  The x
 * transforms of the separate-transform schedules are fed by bulk copies
 * where the rows are 16-byte aligned.
 * paratc_create picks a schedule by rule; paratc_autotune times nrep solves
 * in the step's form (divergence source, transforms, y-solve, inverse with
 * the Neumann ghosts; the state is not touched; in the context's storage
 * form, so an FP32-storage context times the float2 solve and skips the
 * generic transforms) for every supported choice,
 * in three interleaved rounds (each choice keeps its fastest round, so a
 * clock that drifts during the search favours none), writes the times (ms
 * for nrep solves, -1 where unsupported) to
 * times_ms[PARATC_SCHED_NCHOICES] (may be NULL) and keeps the fastest.  All
 * choices solve the same system; results differ by rounding only. */
#define PARATC_SCHED_NCHOICES 12
int paratc_autotune(paratc_ctx* ctx, int nrep, int* choice, double* times_ms);
int paratc_get_schedule(paratc_ctx* ctx, int* choice);
/* pin a choice (PARATC_ERR_BAD_ARG when this grid has no such kernels) */
int paratc_set_schedule(paratc_ctx* ctx, int choice);

/* ---- Tuning of the launch shapes, with a cache.  The reference tunes only
 * its Poisson variant (InitPoissonSolver, src/m_Poisson.f90:50-175, four
 * choices timed at every start).  paratc_autotune_all first runs
 * paratc_autotune (the Poisson schedule), then times whole steps from the
 * current state for every compiled launch shape of the right-hand side
 * (FP64: rows prefetched 1 or 2 ahead, 2 or 1 cells per thread; FP32
 * storage: 1 or 2 cells per thread) and of the Helmholtz sweeps (8 or 4
 * rows per register chunk; FP32 storage also float-arithmetic sweeps), puts
 * the state back
 * and keeps the fastest.  With cache_path != NULL the picks are written to
 * that JSON file under a key naming the GPU, the grid, the scalar, the
 * precision and the flow type, and a later call (or paratc_create, when the
 * environment variable PARATC_TUNE_CACHE names the file) that finds its key
 * there applies the picks without searching (from_cache = 1).  All choices
 * compute the same step; results differ by rounding only. */
typedef struct paratc_tuning {
    int32_t schedule;    /* Poisson schedule, as paratc_autotune               */
    int32_t rhs_var;     /* right-hand-side launch shape                        */
    int32_t helm_var;    /* Helmholtz launch shape                              */
    int32_t from_cache;  /* 1 when the picks were read from the cache           */
    double  step_ms;     /* ms per step of the picks when they were timed       */
} paratc_tuning;
int paratc_autotune_all(paratc_ctx* ctx, int nrep, const char* cache_path, paratc_tuning* out);
int paratc_get_tuning(paratc_ctx* ctx, paratc_tuning* out);
/* pin a combination (PARATC_ERR_BAD_ARG when one of its parts does not exist here) */
int paratc_set_tuning(paratc_ctx* ctx, const paratc_tuning* t);

/* ---- Statistics (clcStat, src/m_FlowCase.f90:257-428).  FP64 accumulators
 * on the device: SumStat(k, jc) += <q_k>_xz for the 35 moments of clcStat (40
 * with the scalar) at rows jc = 1..nyc and the three top-wall moments at
 * jc = nyp, PrGradsum += PrGradAver, nfstime += 1.  The caller decides the
 * cadence (every ivstats steps in the reference, :191).  The accumulators start
 * at zero when the context is created. */
int paratc_stats_reset(paratc_ctx* ctx);
int paratc_stats_accumulate(paratc_ctx* ctx);
/* SumStat in the reference's memory order (k fastest: sumstat[(jc-1)*nstat +
 * k-1], nyp*nstat doubles; may be NULL), the moment count, nfstime and
 * PrGradsum. */
int paratc_stats_get(paratc_ctx* ctx, double* sumstat, int* nstat, int* nfstime, double* prgradsum);

/* ---- 1-D spectra (clcStat's spectra section, src/m_FlowCase.f90:430-806,
 * with clcEnergySpectraX/Z, clcLTS_x/z_real/imag and clcCospectraX/Z at
 * :954-1180).  FP64 accumulators on the device, EnergySpecX(kx, jc, m) and
 * EnergySpecZ(kz, jc, m), m = 1..8 (9 with the scalar) in the reference's
 * order: ux+uCRF, uy, uz, p, the cospectra <ux uy_c> and <ux_c uy_c> (uy and
 * ux interpolated to the cell centre), the real and imaginary linear
 * coherence spectrum of ux against the row jForLCS (mirrored to
 * nyc+1-jForLCS in the upper half of a channel) [, scalar].  One accumulate
 * call is one spectra step of the reference (every ivSpec steps, :431) and
 * adds EgyX*normEgy and EgyZ*normEgy; nSpectime counts the calls.  nx and nz
 * must be lengths the transform kernels are built for (2^a 3^b 5^c, listed
 * in k_spectra.cu), else PARATC_ERR_BAD_ARG.  The accumulators are created
 * and zeroed on first use. */
int paratc_spectra_reset(paratc_ctx* ctx);
/* jlcs: jForLCS of &SpectraOptions, 1..nyc. */
int paratc_spectra_accumulate(paratc_ctx* ctx, int jlcs);
/* spec_x[(m-1)*nyc*(nxc/2+1) + (jc-1)*(nxc/2+1) + kx] (the reference's
 * Fortran order of EnergySpecX(nxhp, nyc, m)), spec_z likewise with nzc/2+1
 * modes; either may be NULL.  nspec: 8 or 9; nspectime: samples summed (the
 * reference divides by it when it writes SpecX/SpecZ, :841-884). */
int paratc_spectra_get(paratc_ctx* ctx, double* spec_x, double* spec_z, int* nspec, int* nspectime);

/* ---- 2-D spectra (clcStat's 2-D section, src/m_FlowCase.f90:780-803, with
 * clcEnergySpectra2D and clcCosSpectra2D at :1186-1375).  Each field is
 * transformed R2HC along x and then R2HC along z (a halfcomplex-of-
 * halfcomplex array, as the reference does, not a complex 2-D transform);
 * at the rows iySpec2D the squares are added with normEgy = (1/(nxc nzc))^2,
 * halved in a channel, where the mirrored row is added too (nyp+1-jct for
 * the uy faces, nyc+1-jct otherwise).  Spectra m = 1..5 (6 with the scalar):
 * ux (without uCRF), uy, uz, p, the cospectrum of ux at the cell centre
 * (+uCRF) with uy at the cell centre (minus the mirrored product), scalar.
 * setup takes &Spectra2DOpt's iySpec2D (nsel = nySpec2D rows; 2..nyc/2 in a
 * channel, 2..nyc otherwise, as InitStatVar checks, :220-232, else
 * PARATC_ERR_BAD_ARG) and zeroes the accumulators; accumulate is one spectra
 * step. */
int paratc_spectra2d_setup(paratc_ctx* ctx, int nsel, const int* iy);
int paratc_spectra2d_reset(paratc_ctx* ctx);
int paratc_spectra2d_accumulate(paratc_ctx* ctx);
/* out[((m-1)*nzc + kc)*nsel*nxc + (q-1)*nxc + ic] (EnergySpec2D(nxc, nySpec2D,
 * nzc, m) in Fortran order; may be NULL), nspec: 5 or 6, nsel, nspectime. */
int paratc_spectra2d_get(paratc_ctx* ctx, double* out, int* nspec, int* nsel, int* nspectime);

/* ---- visualisation dumps (dump_visu, src/m_IOAndVisu.f90:182-385, and the
 * XDMF index of InitVisu, :29-175) ---------------------------------------- */
#define PARATC_VISU_UX      0   /* (ux_i + ux_i+1)/2 + uCRF; node: ux + uCRF   */
#define PARATC_VISU_UY      1   /* (uy_j + uy_j+1)/2;        node: uy          */
#define PARATC_VISU_UZ      2   /* (uz_k + uz_k+1)/2;        node: uz          */
#define PARATC_VISU_PR      3   /* pressure                                    */
#define PARATC_VISU_WX      4   /* vorticity components (2nd-order, :264-330)  */
#define PARATC_VISU_WY      5
#define PARATC_VISU_WZ      6
#define PARATC_VISU_WMAG    7   /* |vorticity|                                 */
#define PARATC_VISU_Q       8   /* Q criterion (Clc_Q_vor)                     */
#define PARATC_VISU_LAMDA2  9   /* lambda2 (Clc_lamda2)                        */
#define PARATC_VISU_SCALAR 10   /* scalar (scalar_on only)                     */
#define PARATC_VISU_NQ     11

/* One quantity at the points decomp_2d_write_every keeps with from1 = .true.
 * (src/m_Decomp2d.f90:1232-1389): global indices 1, 1+skip, ... in each
 * direction, nxo = ceil(nxc/iskip) (likewise y, z) values in Fortran order
 * (x fastest), FP64.  node != 0 selects the SaveNode build (staggered
 * velocities instead of cell-centre averages).  count (may be NULL) gets
 * nxo*nyo*nzo; out may be NULL to query it.  Returns PARATC_ERR_NUMERIC
 * (after filling out) when lambda2 met a point whose cubic has complex
 * roots, where the reference stops. */
int paratc_visu_quantity(paratc_ctx* ctx, int q, int iskip, int jskip, int kskip, int node, double* out,
                         int64_t* count);
/* The same into device memory d_out (nxo*nyo*nzo doubles), asynchronous on
 * the context's stream; the count of lambda2 points with complex roots is
 * added to the device counter *d_nbad (NULL: an internal counter). */
int paratc_visu_quantity_device(paratc_ctx* ctx, int q, int iskip, int jskip, int kskip, int node, double* d_out,
                                unsigned int* d_nbad);
/* Name of quantity q as it appears in the file names ("ux", ..., "wMag",
 * "Q", "lamda2", "scalar"). */
const char* paratc_visu_name(int q);
/* dump_visu: for every q with bit q of save_mask set, writes
 * res_dir + "VisuFor" + run_name + "_" + name + "_" + ntime (10 digits,
 * zero padded): the kept points in Fortran order as REAL(8), or REAL(4)
 * when single != 0 (the SAVE_SINGLE build). */
int paratc_dump_visu(paratc_ctx* ctx, const char* res_dir, const char* run_name, int ntime, int save_mask, int iskip,
                     int jskip, int kskip, int node, int single);
/* InitVisu's XDMF index res_dir + "VisuFor" + run_name + ".xmf": the
 * rectilinear grid (XDMF_SET_TYPE 0: cell corners x = (i-1) dx, yp, z; 1:
 * cell centres) and one temporal entry per ifld = ifirst-1, ifirst-1 +
 * save_visu, ..., ilast with a binary attribute per quantity in save_mask.
 * yp: yp(1..nyp). */
int paratc_write_xdmf(const paratc_params* prm, const double* yp, const char* res_dir, const char* run_name,
                      int ifirst, int ilast, int save_visu, int save_mask, int xdmf_set_type, int single);

/* &IO_Options (+ &SaveScalarOption), &SpectraOptions + &Spectra2DOpt and the
 * output cadences of &BasicParam (src/m_IOAndVisu.f90:37-41,
 * src/m_FlowCase.f90:140-151,209-214, src/m_Parameters.f90:118-121). */
#define PARATC_MAX_SPEC2D 64
typedef struct paratc_io_options {
    int32_t ivstats, save_stat, save_visu;           /* &BasicParam            */
    int32_t iskip, jskip, kskip, xdmf_set_type;      /* &IO_Options            */
    int32_t save_mask;                               /* bit PARATC_VISU_* set when save_<name> = T */
    int32_t write_hist_old, read_hist_old;
    int32_t clc_spectra1d, iv_spec, j_for_lcs;       /* &SpectraOptions        */
    int32_t clc_spectra2d, ny_spec2d;
    int32_t iy_spec2d[PARATC_MAX_SPEC2D];            /* &Spectra2DOpt          */
} paratc_io_options;
int paratc_io_options_from_namelist(const char* path, int scalar_on, paratc_io_options* out);

/* ---- Ensembles.  No counterpart in the reference, which advances one case
 * per MPI job; this is the batched form of ChannelIterate
 * (src/m_ChannelSystem.f90:119-226) for many independent channel instances of
 * uneven grid sizes and parameters on one device.  Every member is an ordinary
 * context (create / set / get through paratc_batch_member) with its own
 * stream; a step of the batch advances every member by one ChannelIterate,
 * the members' kernels running concurrently.  With use_graph != 0 the
 * members' steps are captured once into one CUDA graph (fork/join over the
 * member streams) and every further step of the batch is one graph launch;
 * a member whose state was changed since (set_fields, project, substep, a dt
 * change) first takes one ordinary step, so the graph never replays a step
 * whose clcCFL or Helmholtz pivots are stale.  Calls on one batch must not be
 * concurrent; members must not be stepped on their own while a batch call
 * runs. */
typedef struct paratc_batch paratc_batch;

/* n members; prm[i] and yp[i] (nyc+1 y-faces) as for paratc_create. */
int paratc_batch_create(int n, const paratc_params* prm, const double* const* yp, int device,
                        paratc_batch** out);
int paratc_batch_destroy(paratc_batch* b);
/* The context of member i (owned by the batch: do not paratc_destroy it). */
int paratc_batch_member(paratc_batch* b, int i, paratc_ctx** ctx);
/* nsteps steps of every member; diag (n entries, may be NULL) receives each
 * member's last step.  Returns the first failing member's status. */
int paratc_batch_steps(paratc_batch* b, int nsteps, int use_graph, paratc_diag* diag);
/* Kernels one graph launch of the batch runs (0 before the first capture). */
int64_t paratc_batch_graph_kernels(paratc_batch* b);
/* How a batch step launches its kernels.
 * PARATC_BATCH_STREAMS (the default): every member enqueues its own step on
 * its own stream, one kernel per stage and member (the members' kernels run
 * concurrently).
 * PARATC_BATCH_GROUPED: every stage of the step is ONE launch per kernel
 * instantiation over all members that share it, on the batch's stream: each
 * member's CTAs run that member's launch shape on its own fields, reading
 * its arguments from a device table (so a member computes exactly what its
 * own launches compute).  Members sharing precision, scalar flag and launch
 * shapes share the right-hand side, Helmholtz, y-solve, projection and
 * end-of-step launches; the x transforms are grouped by nxc, the z
 * transforms by nzc.  The batch sets every member's Poisson schedule to the
 * separate compile-time-length transforms (paratc_set_schedule choice 2 or
 * 3, keeping the y-solve kind); a member without them (nxc/2 or nzc not a
 * compiled length) makes the call fail with PARATC_ERR_BAD_ARG.  The tables
 * are rebuilt when a member's schedule, precision or launch shapes change.
 * Both modes take the ordinary step first where a member is not steady
 * (see above), and capture the rest in one graph with use_graph != 0. */
#define PARATC_BATCH_STREAMS 0
#define PARATC_BATCH_GROUPED 1
int paratc_batch_set_mode(paratc_batch* b, int mode);
/* ---- z-slab Poisson solve over several GPUs.  Replaces clcPPE_x1
 * (src/m_Poisson.f90:352-452) with its six pencil transposes
 * (transpose_y1_to_x1 ... transpose_x1_to_y1, src/m_Decomp2d.f90:585-1000,
 * MPI_ALLTOALLW) on a 1-D slab decomposition: rank r of G owns the planes
 * kc in [k0_r, k0_r + nzl_r) in physical space and the modes kx in
 * [kx0_r, kx0_r + nxl_r) of the x spectrum (0 <= kx <= nxc/2) after the
 * first exchange.  One solve is
 *   paratc_slab_forward   x R2HC of the local planes, packed by destination
 *   caller: all-to-all    send -> xslab (counts from paratc_slab_counts)
 *   paratc_slab_middle    z transform, y-Thomas, inverse z transform, in place
 *   caller: all-to-all    xslab -> recv (the counts swapped)
 *   paratc_slab_backward  unpack, inverse x transform, scaled by 1/(nxc nzc)
 * The exchanges are the caller's (NCCL all-to-all between GPUs, through
 * torch.distributed or ncclSend/ncclRecv; MPI_Alltoallv in a host code), so
 * the library links no communicator.  Buffers are device arrays of doubles
 * (complex values as (re, im) pairs): d_send and d_recv hold
 * 2*nzl*nyc*(nxc/2+1), d_xslab 2*nzc*nyc*nxl doubles.  Every call makes
 * the plan's device current, queues its kernels on `stream` (a cudaStream_t,
 * NULL = default) and returns.  Calls on one plan must not run concurrently;
 * the plan's buffers are reused by every solve. */
typedef struct paratc_slab paratc_slab;
/* The balanced split of n items over nranks: rank `rank` gets [*start,
 * *start + *count), the first n % nranks ranks one item more.  Needs no
 * device. */
int paratc_slab_partition(int n, int nranks, int rank, int* start, int* count);
/* A rank's plan on `device`: planes and modes from paratc_slab_partition over
 * nzc and nxc/2+1 (nranks <= PARATC_SLAB_MAX_RANKS, at most one rank per
 * plane and per mode); needs nxc/2 and nzc with factors 2, 3 and 5 only and
 * 3 <= nyc <= 256. */
#define PARATC_SLAB_MAX_RANKS 64
int paratc_slab_create(const paratc_params* prm, const double* yp, int device, int rank, int nranks,
                       paratc_slab** out);
int paratc_slab_destroy(paratc_slab* s);
/* Per-peer counts of the forward exchange, in doubles (nranks entries each):
 * send[q] goes from this rank to rank q, recv[q] comes from rank q.  The
 * backward exchange sends recv[q] and receives send[q].  Either may be NULL. */
int paratc_slab_counts(const paratc_slab* s, int64_t* send, int64_t* recv);
/* d_src: the local planes, nzl*nyc*nxc doubles (interior layout). */
int paratc_slab_forward(paratc_slab* s, const double* d_src, double* d_send, void* stream);
int paratc_slab_middle(paratc_slab* s, double* d_xslab, void* stream);
/* d_phi: the local planes of phi, nzl*nyc*nxc doubles (interior layout). */
int paratc_slab_backward(paratc_slab* s, const double* d_recv, double* d_phi, void* stream);
/* Peer form: no collective library; replaces the same transposes as the
 * all-to-all form (src/m_Decomp2d.f90:585-1000).  Each plan owns an x-slab
 * (paratc_slab_xslab, 2*nzc*nyc*nxl doubles); xslabs[q] (nranks device
 * pointers, host array) is rank q's, this rank's own included, mapped here
 * with paratc_ipc_open when q is another process.  forward_peers transforms
 * the local planes and stores every value straight into its owner's x-slab
 * (plain stores over NVLink); backward_peers loads the rank's planes back
 * from all x-slabs and transforms them.  The caller orders the ranks: every
 * rank's forward_peers completes before any rank's paratc_slab_middle (on
 * its own x-slab), every middle before any backward_peers, every
 * backward_peers before the next forward_peers (a stream synchronisation
 * and a barrier of the processes at each point).  Ranks in one process on
 * one stream need no barrier. */
double* paratc_slab_xslab(paratc_slab* s);
int paratc_slab_forward_peers(paratc_slab* s, const double* d_src, const double* const* xslabs, void* stream);
int paratc_slab_backward_peers(paratc_slab* s, const double* const* xslabs, double* d_phi, void* stream);
/* CUDA IPC of a device allocation's base address (cudaIpcGetMemHandle /
 * cudaIpcOpenMemHandle with lazy peer access): the handle is
 * PARATC_IPC_HANDLE_BYTES opaque bytes to send to the other processes.  No
 * counterpart in the reference, whose ranks exchange only through MPI. */
#define PARATC_IPC_HANDLE_BYTES 64
int paratc_ipc_get_handle(const void* d_ptr, void* handle);
int paratc_ipc_open(const void* handle, void** d_ptr);
int paratc_ipc_close(void* d_ptr);
/* Waits for `stream`; PARATC_ERR_TIMEOUT if a bulk-copy-fed transform of
 * this plan gave up a bounded wait since the plan was created (its results
 * are then not to be used). */
int paratc_slab_sync(paratc_slab* s, void* stream);
int paratc_batch_get_mode(paratc_batch* b, int* mode);
/* Kernel launches of one steady step of the batch in its mode (grouped: the
 * plan's launches; streams: the last captured graph's kernels, 0 before). */
int64_t paratc_batch_step_launches(paratc_batch* b);
/* The stream the batch's graph is launched on (cudaStream_t); work queued on
 * it before paratc_batch_steps precedes the steps, work queued after them
 * follows them. */
void* paratc_batch_stream(paratc_batch* b);

#ifdef __cplusplus
}
#endif
#endif /* PARATC_H */
