/*
 * blgpu.h -- C ABI of the B200 step path of the boundary-layer DNS solver.
 *
 * Drop-in for the per-step hot path of ms-alvaro/boundary-layer-gpu: the
 * staggered second-order RHS (equations.f90), the Euler/RK2/RK3 substeps
 * (time_integration.f90), the boundary-condition pass of the GPU build
 * (boundary_conditions.f90:127-262) and the fractional-step projection
 * (projection.f90).  Plain C types only, so a Fortran host binds it with
 * ISO_C_BINDING and Python with ctypes.
 *
 * Conventions
 *  - Every entry point returns 0 on success and a negative BLGPU_E* code on
 *    failure; blgpu_last_error() then returns a message.  Nothing aborts.
 *  - Host arrays use the reference's Fortran layout and bounds (column-major,
 *    i fastest):  U(nx,nyg,nzg)  V(nxg,ny,nzg)  W(nxg,nyg,nz)  P(nxg,nyg,nzg)
 *    with nxg = nx+1, nyg = ny+1, nzg = nz+1 (global.f90:86-88 at nprocs=1).
 *  - The context owns all device memory, allocated in blgpu_create; state
 *    crosses the host boundary only in blgpu_upload_state/download_state,
 *    i.e. where the reference has its !$acc data copy / update self
 *    (main.f90:61-81,99-101).
 *  - One context = one box on one GPU, work in issue order on one stream.
 */
#ifndef BLGPU_H
#define BLGPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define BLGPU_OK 0
#define BLGPU_EINVAL (-1)   /* bad argument or size */
#define BLGPU_ECUDA (-2)    /* CUDA runtime error */
#define BLGPU_ESTATE (-3)   /* call out of order (e.g. no grid yet) */
#define BLGPU_EDEVICE (-4)  /* device-side check failed (NaN, wait limit) */

#define BLGPU_FP64 0   /* bit-faithful FP64 form */
#define BLGPU_MIXED 1  /* FP32 fields/RHS/transforms, FP64 Thomas and mean mode */

#define BLGPU_LES_HOST (-1)  /* les_model: nu_t supplied by the host (blgpu_set_nu_t) */

#define BLGPU_POISSON_NATIVE 0  /* hand-written DCT/DFT/Thomas kernels */
#define BLGPU_POISSON_CUFFT 1   /* cuFFT comparison path (FP64 only) */

typedef struct blgpu_ctx blgpu_ctx;

/* Run parameters: the .turbb keys of the path (params.f90:119-207). */
typedef struct blgpu_config {
  int nx, ny, nz;     /* nxyz: face points (params.f90:131) */
  double nu;          /* nu (params.f90:119) */
  double cfl;         /* CFL; < 0 means fixed dt = -CFL (time_integration.f90:539) */
  double dpdx, dpdz;  /* dPdx, dPdz (params.f90:152-153) */
  int rk_scheme;      /* RKscheme: 1 Euler, 2 RK2, 3 RK3 (params.f90:195) */
  int les_model;      /* LES, nu_t computed on the device before every substep: 0 DNS;
                         1 constant-coefficient Smagorinsky (subgrid.f90:609-730); 2 dynamic
                         Smagorinsky, coefficient averaged in z (subgrid.f90:261-414); 3 dynamic
                         Smagorinsky, pointwise (subgrid.f90:420-583); 2 and 3 hold 29 FP64
                         work arrays of nxg*nyg*nzg.  BLGPU_LES_HOST: eddy viscosity given by
                         blgpu_set_nu_t and held fixed */
  int precision;      /* BLGPU_FP64 | BLGPU_MIXED */
  int poisson;        /* BLGPU_POISSON_NATIVE | BLGPU_POISSON_CUFFT */
  int device;         /* CUDA device ordinal */
} blgpu_config;

/* initialize/allocation part of initialization.f90:25-759 and
 * cufft_init_plans (cufft_solver.f90:26) */
int blgpu_create(const blgpu_config *cfg, blgpu_ctx **out);
/* finalize (finalization.f90:6-38) */
int blgpu_destroy(blgpu_ctx *ctx);
/* message of the last failure (global one when ctx is NULL) */
const char *blgpu_last_error(const blgpu_ctx *ctx);

/* face grids x(nx), y(ny), z(nz); centres, ghosts, modified wavenumbers,
 * Dyy and interpolation weights are derived as in initialization.f90:174-222,
 * 329-344, 395-425, 482-484 */
int blgpu_set_grid(blgpu_ctx *ctx, const double *x, const double *y, const double *z);

/* inflow/top vectors of compute_blasius_solution_for_bc /
 * compute_turbulent_solution_for_bc (boundary_conditions.f90:1371-1797):
 * U_inlet(nyg) V_inlet(ny) W_inlet(nyg) U_top(nx) V_top(nxg) W_top(nxg) */
int blgpu_set_boundary(blgpu_ctx *ctx, const double *U_inlet, const double *V_inlet, const double *W_inlet,
                       const double *U_top, const double *V_top, const double *W_top);

/* temporal inflow modes (boundary_conditions.f90:1720-1797): zmode(n) and
 * tmode(m) already scaled by beta/omega; qu(nyg,n,m), qv(ny,n,m),
 * qw(nyg,n,m) as interleaved (re,im) doubles */
int blgpu_set_inflow_modes(blgpu_ctx *ctx, int n_modes, int m_modes, const double *zmode, const double *tmode,
                           const double *qu, const double *qv, const double *qw);

/* Lund recycling/rescaling inflow (rescaled_inlet_bc.f90:60-345), the
 * inflow_flag 3 / 5 branches of apply_boundary_conditions
 * (boundary_conditions.f90:35-43, 512-597).  mode 0 = off (inflow modes as
 * above), 3 = the rescaled plane replaces the inlet plane, 5 = the rescaled
 * fluctuations are added to U_inlet/V_inlet/W_inlet.  The plane is computed
 * once per step on the device from the step's starting fields at
 * x-index i_rescale (Lund_ix, 2..nx); delta_inlet = Lund_deltai, T_resc =
 * Lund_T.  The running means start from the current device state
 * (initialization.f90:636-664), or from Umean0(nyg)/Vmean0(ny) -- the
 * .mean.rescaling restart means -- when Umean0 is non-null and sums above
 * 1e-4.  Requires grid and state; replaces the GPU routine's inflow plane
 * (boundary_conditions.f90:182-190), which the reference leaves undefined
 * for these flags. */
int blgpu_set_rescaling(blgpu_ctx *ctx, int mode, int i_rescale, double delta_inlet, double T_resc,
                        const double *Umean0, const double *Vmean0);
/* one evaluation of compute_rescaled_inflow from the current state, with the
 * current dt (what a step does before its first boundary pass) */
int blgpu_rescaled_inflow(blgpu_ctx *ctx);
/* running means Umean_resc_T(nyg), Vmean_resc_T(ny), Umean_inlet_T(nyg),
 * Vmean_inlet_T(ny); the last planes Ut_inlet(nyg,nzg), Vt_inlet(ny,nzg),
 * Wt_inlet(nyg,nz); diag[8] = Uinf, delta_resc, delta99 at the inlet,
 * theta_resc, theta_inlet, utau_resc, utau_inlet, gamma; err != 0 when
 * interp_vel met its 'j==1' stop (rescaled_inlet_bc.f90:334).  Any pointer
 * may be NULL. */
int blgpu_get_rescaling(blgpu_ctx *ctx, double *Umean_resc, double *Vmean_resc, double *Umean_inlet,
                        double *Vmean_inlet, double *Lu, double *Lv, double *Lw, double *diag, int *err);

/* eddy viscosity nu_t(nxg,nyg,nzg) supplied by the host (les_model = BLGPU_LES_HOST) */
int blgpu_set_nu_t(blgpu_ctx *ctx, const double *nu_t);

/* box sizes and viscosity of a context; the face grids given to set_grid */
int blgpu_box(const blgpu_ctx *ctx, int *nx, int *ny, int *nz, double *nu);
int blgpu_get_grid(blgpu_ctx *ctx, double *x, double *y, double *z);

/* state in/out (main.f90:61-81 copy-in; main.f90:99-101 update self).
 * Upload also sets Uo = U as read_input_data does (input_output.f90:476-478).
 * A NaN or an infinity in the host arrays is rejected with BLGPU_EDEVICE
 * (the context then holds no state); blgpu_set_nu_t and blgpu_compute_rhs
 * check their host arrays the same way. */
int blgpu_upload_state(blgpu_ctx *ctx, const double *U, const double *V, const double *W, double t);
int blgpu_download_state(blgpu_ctx *ctx, double *U, double *V, double *W, double *P, double *t);
/* Streamed variants for passing a sequence of states through the solver:
 * they return at once; the host-to-device copies run on their own stream,
 * the device-to-host copies on another, each through its own device staging
 * buffers, ordered against the context's compute stream by events, so that
 * the upload of the next state, the steps of the current one and the
 * download of the previous one overlap (PCIe is full duplex).  Host arrays
 * must be pinned for the copies to be asynchronous and must not be touched
 * until blgpu_sync returns; the state semantics are those of
 * blgpu_upload_state / blgpu_download_state (U, V, W; no pressure, no time);
 * a NaN or an infinity in a streamed upload is reported by the next
 * blgpu_sync as BLGPU_EDEVICE. */
int blgpu_upload_state_async(blgpu_ctx *ctx, const double *U, const double *V, const double *W, double t);
int blgpu_download_state_async(blgpu_ctx *ctx, double *U, double *V, double *W);

/* compute_dt (time_integration.f90:528-591): device reduction, no host copy
 * of the fields; the resulting dt is returned and kept on the device */
int blgpu_compute_dt(blgpu_ctx *ctx, double *dt);
int blgpu_set_dt(blgpu_ctx *ctx, double dt);
int blgpu_get_time(blgpu_ctx *ctx, double *t, double *dt);

/* one step of the main loop body (main.f90:87-96): compute_dt, then
 * compute_time_step_{Euler,RK2,RK3}; repeated nsteps times, replayed from a
 * captured CUDA graph */
int blgpu_advance(blgpu_ctx *ctx, int nsteps);

/* compute_time_step_RK3 / _RK2 / _Euler (time_integration.f90:305,145,24):
 * one step with the current dt, no compute_dt */
int blgpu_time_step(blgpu_ctx *ctx);

/* compute_rhs_u/v/w (equations.f90:24,163,301) on host arrays; outputs are
 * the reference's compact interior arrays rhs_u(2:nx-1,2:nyg-1,2:nzg-1),
 * rhs_v(2:nxg-1,2:ny-1,2:nzg-1), rhs_w(2:nxg-1,2:nyg-1,2:nz-1) */
int blgpu_compute_rhs(blgpu_ctx *ctx, const double *U, const double *V, const double *W, double *rhs_u,
                      double *rhs_v, double *rhs_w);

/* apply_boundary_conditions_gpu (boundary_conditions.f90:127) on the
 * resident state, with the outflow factor rk_t(rk_step) */
int blgpu_apply_bc(blgpu_ctx *ctx, int rk_step);

/* compute_projection_step (projection.f90:21) on the resident state;
 * rk_step == 1 also stores P (projection.f90:75-85) */
int blgpu_projection(blgpu_ctx *ctx, int rk_step);

/* rhs_p(2:nxg-1,2:nyg-1,2:nzg) of the last projection (projection.f90 array) */
int blgpu_get_rhs_p(blgpu_ctx *ctx, double *rhs_p);

/* check_divergence (projection.f90:391-413) */
int blgpu_max_divergence(blgpu_ctx *ctx, double *max_div);

/* wait for all queued work */
int blgpu_sync(blgpu_ctx *ctx);

/* device bytes held by the context */
long long blgpu_device_bytes(const blgpu_ctx *ctx);

/* Per-phase device time of nsteps eager steps (compute_dt + time step),
 * measured with CUDA events on the context stream -- the B200 counterpart of
 * the reference's RK2 phase timers (time_integration.f90:149-155,194-236,
 * 283-298).  ms[p] and kernels[p] accumulate over the steps for the phases
 *   0 RHS+RK update  1 boundary conditions  2 divergence+DCT-x  3 DFT-z
 *   4 Thomas-y  5 inverse DFT-z  6 inverse DCT-x  7 velocity correction
 *   8 compute_dt  9 time bookkeeping
 * nphase must be >= 10; kernels may be NULL. */
int blgpu_phase_times(blgpu_ctx *ctx, int nsteps, double *ms, long long *kernels, int nphase);

/* the context's LES model on the resident state.  LES = 1: sgs_Smagorinsky
 * (subgrid.f90:609-730), nu_t on the interior i=2..nxg-1, j=2..nyg-1,
 * k=2..nzg-1 (Cs = 0.11, f = 1).  LES = 2, 3: the dynamic model
 * (subgrid.f90:261-583), nu_t on the whole (nxg,nyg,nzg) array after clipping
 * and the Neumann y ghosts. */
int blgpu_eddy_viscosity(blgpu_ctx *ctx);
/* nu_t(nxg,nyg,nzg); zeros for a context created with LES = 0 */
int blgpu_get_nu_t(blgpu_ctx *ctx, double *nu_t);

/* compute_statistics (statistics.f90:26-201) on the device, FP64
 * accumulators: means = Umean,Vmean,Wmean,U2mean,V2mean,W2mean,UVmean,
 * Pmean,P2mean as 9 consecutive (nx,ny) arrays; nu_t_mean(nxg,nyg); Cf(nx);
 * dUdy_wall(nx); scalars = theta_inlet, delta99_inlet, Re_x, Re_theta,
 * Re_delta.  Any output may be NULL. */
int blgpu_statistics(blgpu_ctx *ctx, double *means, double *nu_t_mean, double *Cf, double *dUdy_wall,
                     double *scalars);

/* compute_law_of_the_wall_model (wallmodel.f90:1951-1985) with
 * Newton_iter_solver (Newton_solver.f90:13-79): utau(nx) is the initial
 * guess on entry and utau_model on exit; *iters_max = largest iteration
 * count (30 = not converged) */
int blgpu_law_of_wall(blgpu_ctx *ctx, double *utau, int *iters_max);

/* blgpu_advance(ctx, nsteps) bracketed by CUDA events on the context
 * stream; *ms = device time of the nsteps (graph captured beforehand) */
int blgpu_advance_timed(blgpu_ctx *ctx, int nsteps, double *ms);

/* Test hook of the failure path, no counterpart in the reference: the
 * number of mbarrier polls the tiled y-solve's CTAs make before a tile copy
 * counts as lost (polls < 0 restores the built-in limit of 2^24).  A wait
 * that gives up sets bit 4 of the device flag; the CTA still waits, with the
 * built-in limit, for its copy to land before it leaves, and the next
 * blgpu_sync / blgpu_advance_timed reports BLGPU_EDEVICE (once; the flag is
 * cleared when reported).  The state of such a step is not valid. */
int blgpu_set_wait_limit(blgpu_ctx *ctx, int polls);

/* number of kernels this context has launched (graph replays included) */
long long blgpu_kernel_launches(const blgpu_ctx *ctx);

/* check_divergence on device arrays the caller owns, with no device
 * allocation: no counterpart in the reference.  For hosts that cannot call
 * cudaMalloc (an OpenACC program passing its data-region arrays by device
 * address, or code under a pool allocator / in a no-allocation region).
 * U(nx,nyg,nzg), V(nxg,ny,nzg), W(nxg,nyg,nz), x(nx), y(ny), z(nz) and the
 * result *max_div are device addresses in the reference layout; stream may be
 * NULL.  Scratch is a fixed 512 KiB __device__ array: (ny-1)*(nz-1) must be
 * <= 65536 (else BLGPU_EINVAL); the first call on a device sets it up and
 * should come before any stream capture; calls that overlap on the GPU race.
 * The result is ready when the stream reaches the call. */
int blgpu_check_divergence_noalloc(const double *U, const double *V, const double *W, const double *x,
                                   const double *y, const double *z, int nx, int ny, int nz, double *max_div,
                                   void *stream);

/* ---- launch shapes and the autotuner ----
 * tiles[5 to 10] = rhs_kc (k-planes per CTA of the RHS kernel), rhs_by (RHS
 * block 32 x rhs_by), dct_nw (complex lines per CTA of the forward DCT, up
 * to 16 in the mixed form (8 with the two-pass x transforms) and 8 in FP64),
 * dftz_rk (z wavenumbers per warp of the z-DFT, 4 or 8), proj_by (projection
 * block 32 x proj_by), zdft (mixed form, where M/2+1 <= 96: 1 = FP32 direct
 * sums, 2 = mma.sync TF32 tensor cores, 3 = tcgen05 tensor cores with the
 * accumulators in tensor memory), rhs_pts (mixed-form DNS RHS: 1 = one
 * x-point per thread, 2 = two, 3 = two in packed FP32x2 instructions, 4 = as
 * 3 with every plane staged in shared memory by TMA, rhs_by then fixed at
 * 8; FP64 DNS, all bit-identical: 1 = one point, global loads, 4 = one point,
 * TMA-fed planes, 2 = two points in a register window),
 * thomas (y-solve: 1 = register ring,
 * 2 = TMA-fed tiles where ny-1 <= 256, one thread per mode, 3 = the same
 * tiles with each mode's rows split over 16 threads; the built-in choice
 * is 3 where ny-1 <= 256, else 1), idct_nw (lines per CTA of the
 * inverse DCT), xfft (x transforms: 1 = Stockham mixed-radix FFT in shared
 * memory, any N; 2 = two-pass register FFT, built for N = nx-2 = 812
 * (29 x 28; both precisions), 510 (17 x 30), 190 (19 x 10) and 126 (14 x 9)
 * (mixed form));
 * 0 = the built-in choice.
 * Values not passed keep their current setting.  All but zdft, rhs_pts,
 * xfft and thomas 3 leave results unchanged; those change them at rounding
 * level.  No counterpart in the
 * reference (its OpenACC loops take compiler-chosen gangs). */
int blgpu_set_tiles(blgpu_ctx *ctx, const int *tiles, int n);
int blgpu_get_tiles(const blgpu_ctx *ctx, int *tiles, int n);
/* Coordinate search over the tile candidates, timing `steps` graph-replayed
 * steps per candidate on the device; keeps the fastest.  The fields, time,
 * dt and Lund means are restored afterwards.  ms_default / ms_best (may be
 * NULL) receive the per-step times of the starting and the chosen tiles. */
int blgpu_autotune(blgpu_ctx *ctx, int steps, double *ms_default, double *ms_best);

/* ---- ensembles of independent boxes (no counterpart in the reference) ----
 * Boxes are ordinary contexts on one device, created and loaded by the
 * caller (grid, boundary, state, Lund); the ensemble does not own them.
 * blgpu_ensemble_advance runs each step of every box as ONE CUDA-graph launch
 * whose branches (one per box) run concurrently; results equal those of
 * blgpu_advance on each box.  Boxes must be at the same buffer rotation
 * (advanced the same number of RK3 steps since their last upload). */
typedef struct blgpu_ensemble blgpu_ensemble;
int blgpu_ensemble_create(blgpu_ctx *const *boxes, int nbox, blgpu_ensemble **ens);
int blgpu_ensemble_destroy(blgpu_ensemble *ens);
const char *blgpu_ensemble_last_error(const blgpu_ensemble *ens);
int blgpu_ensemble_advance(blgpu_ensemble *ens, int nsteps);
/* the same steps with one box at a time (the sequential baseline) */
int blgpu_ensemble_advance_sequential(blgpu_ensemble *ens, int nsteps);
/* device time (CUDA events on the ensemble stream) of nsteps steps, graph
 * capture excluded; sequential != 0 times the sequential baseline */
int blgpu_ensemble_time(blgpu_ensemble *ens, int nsteps, int sequential, double *ms);
int blgpu_ensemble_sync(blgpu_ensemble *ens);
long long blgpu_ensemble_launches(const blgpu_ensemble *ens);
/* blgpu_autotune on the first box of each distinct shape; the others of
 * that shape take its tiles.  ntuned (may be NULL) = shapes tuned. */
int blgpu_ensemble_autotune(blgpu_ensemble *ens, int steps, int *ntuned);

/* ---- learned wall model (no counterpart in the reference) ----
 * A 4 -> 64 -> 64 -> 64 -> 2 GELU network evaluated and trained on the
 * tensor cores (BF16 operands, FP32 accumulation).  Parameters are FP32 in
 * the order W0[64][4] b0[64] W1[64][64] b1[64] W2[64][64] b2[64] W3[2][64]
 * b3[2] (blgpu_mlp_nparams() = 8770).  Inputs per wall point: u and w at the
 * sampling row jh, ln(h |u| / nu) / 10 and 100 h dP/dx (h = yg(jh));
 * outputs: 1000 tau_x, 1000 tau_z.  Loss: mean over samples of the summed
 * squared output error. */
typedef struct blgpu_mlp blgpu_mlp;
int blgpu_mlp_nparams(void);
int blgpu_mlp_create(int device, unsigned long long seed, blgpu_mlp **net); /* Glorot init */
int blgpu_mlp_destroy(blgpu_mlp *net);
const char *blgpu_mlp_last_error(const blgpu_mlp *net);
int blgpu_mlp_set_params(blgpu_mlp *net, const float *params, int n); /* resets the Adam state */
int blgpu_mlp_get_params(blgpu_mlp *net, float *params, int n);
/* host arrays X[rows][4] -> Y[rows][2] */
int blgpu_mlp_forward(blgpu_mlp *net, const float *X, int rows, float *Y);
/* loss and its gradient (8770 values) over host samples X[rows][4], T[rows][2] */
int blgpu_mlp_gradient(blgpu_mlp *net, const float *X, const float *T, int rows, float *grad, float *loss);
/* the device training set */
int blgpu_mlp_add_data(blgpu_mlp *net, const float *X, const float *T, int rows);
int blgpu_mlp_sample(blgpu_mlp *net, blgpu_ctx *ctx, int jh); /* wall samples of the solver state */
int blgpu_mlp_clear_data(blgpu_mlp *net);
int blgpu_mlp_num_samples(const blgpu_mlp *net);
int blgpu_mlp_get_data(blgpu_mlp *net, float *X, float *T, int rows);
/* `steps` Adam steps (lr, betas 0.9 / 0.999) on minibatches of `batch`
 * samples in a shuffled order; loss_last = loss of the last batch */
int blgpu_mlp_train(blgpu_mlp *net, int steps, int batch, float lr, float *loss_last);
int blgpu_mlp_steps(blgpu_mlp *net, long long *steps);
int blgpu_mlp_loss_history(blgpu_mlp *net, float *hist, int n);
int blgpu_mlp_eval(blgpu_mlp *net, float *loss); /* loss over the whole training set */

/* Wall model of the step, evaluated at the start of every substep
 * (time_integration.f90:341-346) from the substep's fields and applied as
 * the non-zero Neumann condition U(:,1,:) = U(:,2,:) - tau/nu_w (yg(2)-yg(1))
 * (boundary_conditions.f90:359-372), nu_w the viscosity of the wall flux (nu
 * plus the interpolated eddy viscosity with LES).  mode 0: no-slip (the
 * reference GPU routine); 1: law of the wall (wallmodel.f90:1951-1985) at
 * row jh, tau = u_tau(x)^2, V and W no-slip; 2: the network at row jh,
 * tau_x on U and tau_z on W. */
int blgpu_set_wall_model(blgpu_ctx *ctx, int mode, int jh, const blgpu_mlp *net);
/* the model's stress on the current state at i = 2..nx-1 (fastest),
 * k = 2..nzg-2: (nx-2)(nzg-3) values each */
int blgpu_wall_stress(blgpu_ctx *ctx, double *tau_x, double *tau_z);

/* ---- the reference's files: .turbb parameters, snapshots, Lund means ----
 * Host code only (no device needed); messages of these calls come from
 * blgpu_io_last_error(). */

/* Every key initparams reads (params.f90:119-197), in its order; bit q of
 * `found` is set when the q-th key was present (BLGPU_PARAM_*).  Keys not
 * given keep 0 (init_step: -45, "not given", input_output.f90:33). */
typedef struct blgpu_params {
  double nu, cfl, vmax, x0, sigma, phi;       /* nu CFL Vmax x0 sigma phi */
  int nsteps, nsave, nstats, nmonitor;
  int nxyz[3];
  double boxsize[4];                         /* Lx Ly Lz alpha */
  int inflow_flag, top_flag;
  char inflow_file[201];
  int lund_ix;
  double lund_deltai, lund_T;
  double dpdx, dpdz;
  int les, wm, tauw_model, nut_bc, wm_nut_flag;  /* LES WM TauwModel nutBC WMnutflag */
  double wm_nut, amplitude;                  /* WMnut Amplitude */
  int init_step, init_rand;
  char filein[201], fileout[201], timeinflow_file[201];
  int rk_scheme;                             /* RKscheme */
  double alphas[5];
  unsigned long long found;
} blgpu_params;
enum {
  BLGPU_PARAM_NU, BLGPU_PARAM_CFL, BLGPU_PARAM_VMAX, BLGPU_PARAM_X0, BLGPU_PARAM_SIGMA, BLGPU_PARAM_PHI,
  BLGPU_PARAM_NSTEPS, BLGPU_PARAM_NSAVE, BLGPU_PARAM_NSTATS, BLGPU_PARAM_NMONITOR, BLGPU_PARAM_NXYZ,
  BLGPU_PARAM_BOXSIZE, BLGPU_PARAM_INFLOW_FLAG, BLGPU_PARAM_TOP_FLAG, BLGPU_PARAM_INFLOW_FILE, BLGPU_PARAM_LUND_IX,
  BLGPU_PARAM_LUND_DELTAI, BLGPU_PARAM_LUND_T, BLGPU_PARAM_DPDX, BLGPU_PARAM_DPDZ, BLGPU_PARAM_LES, BLGPU_PARAM_WM,
  BLGPU_PARAM_TAUWMODEL, BLGPU_PARAM_NUTBC, BLGPU_PARAM_WMNUTFLAG, BLGPU_PARAM_WMNUT, BLGPU_PARAM_AMPLITUDE,
  BLGPU_PARAM_INIT_STEP, BLGPU_PARAM_INIT_RAND, BLGPU_PARAM_FILEIN, BLGPU_PARAM_FILEOUT,
  BLGPU_PARAM_TIMEINFLOW_FILE, BLGPU_PARAM_RKSCHEME, BLGPU_PARAM_ALPHAS
};
const char *blgpu_io_last_error(void);
/* initparams through getvar (miscel.f90:13-262): a line matches a key when
 * the text before its first '=' is the key; the value runs to a '!'; the
 * first match wins.  BLGPU_EINVAL for a missing file, an unreadable value,
 * no inflow_file, or init_rand = 1 with a filein (params.f90:136-139,166-169). */
int blgpu_read_params(const char *path, blgpu_params *p);
/* the blgpu_config fields a .turbb sets (sizes, nu, CFL, dPdx, dPdz,
 * RKscheme, LES); the others are left as they are */
int blgpu_params_config(const blgpu_params *p, blgpu_config *cfg);

/* Snapshot: t, nu; -73 and the step; x, y, z, xm, ym, zm with their sizes;
 * then U, V, W, nu_t, P, each after its 3 dims (input_output.f90:521-636).
 * One process writes n3-1 planes of U, V, W and nu_t and all planes of P
 * (the layout of the reference's GPU runs and of its plotting scripts); a
 * file assembled from several processes holds every plane.  The reader
 * accepts both, and files that end after W (then nu_t and P read as 0); a
 * plane left out is filled as the z-periodic boundary pass fills it. */
typedef struct blgpu_snapshot_info {
  double t, nu;
  int step;          /* -1 when the file has no magic number */
  int nx, ny, nz;
  int full_planes;   /* 1: every plane stored; 0: the one-process layout */
  int has_nu_t_p;
} blgpu_snapshot_info;
int blgpu_snapshot_info_read(const char *path, blgpu_snapshot_info *h);
/* any output pointer may be NULL; U(nx,nyg,nzg) V(nxg,ny,nzg) W(nxg,nyg,nz)
 * nu_t, P (nxg,nyg,nzg) as everywhere in this header */
int blgpu_read_snapshot(const char *path, blgpu_snapshot_info *h, double *x, double *y, double *z, double *U,
                        double *V, double *W, double *nu_t, double *P);
/* writes the one-process layout; nu_t and P may be NULL (zeros) */
int blgpu_write_snapshot(const char *path, int nx, int ny, int nz, double t, double nu, int step, const double *x,
                         const double *y, const double *z, const double *U, const double *V, const double *W,
                         const double *nu_t, const double *P);
/* <snapshot>.mean.rescaling: nyg, Umean_resc(nyg), Vmean_resc(ny); written
 * in native byte order, read in either (the reference writes native and
 * reads big-endian, input_output.f90:445,671) */
int blgpu_read_rescaling(const char *path, int nyg, int ny, double *Umean, double *Vmean);
int blgpu_write_rescaling(const char *path, int nyg, int ny, const double *Umean, const double *Vmean);
/* inflow_file of inflow flags 2 and 5 (boundary_conditions.f90:1405-1413,
 * 1550-1558; written by the reference's generate_inflow scripts): ny
 * (int32), U_inlet(ny+1) at the centres yg, V_inlet(ny) at the faces y,
 * in either byte order (told apart by the file size); the _info call
 * returns the file's ny, the read refuses a ny other than the grid's
 * ("Profile doesnt match dimensions"). */
int blgpu_read_inflow_profile_info(const char *path, int *ny);
int blgpu_read_inflow_profile(const char *path, int ny, double *U_inlet, double *V_inlet);
/* output_statistics (input_output.f90:685-746): <name>.stats.txt in the
 * reference's text layout ('%', t, nu as F15.8; nx, ny, nz, istep as I8;
 * Cf and x as one record of nx F15.8 values; y as one of ny; then Umean,
 * Vmean, Wmean, U2mean, V2mean, W2mean, Pmean, P2mean as nx records of ny).
 * means: the nine (nx,ny) arrays of blgpu_statistics, in its order.  The
 * context form computes the statistics on the device and names the file
 * fileout.<istep+nstep_init, 8 digits>.stats.txt, with istep in the header,
 * as the reference does. */
int blgpu_write_statistics(const char *path, double t, double nu, int nx, int ny, int nz, int istep,
                           const double *Cf, const double *x, const double *y, const double *means);
int blgpu_output_statistics(blgpu_ctx *ctx, const char *fileout, int istep, int nstep_init);
/* fileout.%08d (input_output.f90:516-518) */
int blgpu_snapshot_name(const char *fileout, int step, char *name, int cap);
/* output_data (input_output.f90:496-680) for a context: downloads the state,
 * writes fileout.<step>, points fileout.restart at it and, when rescaling
 * != 0, writes the Lund means to fileout.<step>.mean.rescaling.  Creates the
 * directory of fileout if missing (params.f90:177-191). */
int blgpu_output_data(blgpu_ctx *ctx, const char *fileout, int step, int rescaling);
/* read_input_data (input_output.f90:288-487) for a context: size checks,
 * the file's grid replaces the context's (blgpu_set_grid), U, V, W and t are
 * uploaded; *step (may be NULL) = the file's step or -1.  The Lund means of
 * filein.mean.rescaling go to blgpu_set_rescaling through
 * blgpu_read_rescaling. */
int blgpu_read_input_data(blgpu_ctx *ctx, const char *filein, int *step);

/* Temporal inflow modes of the transition case (inflow_flag = 1): the binary
 * mode file read by compute_blasius_solution_for_bc
 * (boundary_conditions.f90:1652-1797), a native-order stream of ny_inlet,
 * n, m (int32), beta, omega (f64), ymesh(ny_inlet), zmode(n), tmode(m) and
 * the real and imaginary parts of qu, qv, qw (ny_inlet, n, m).  The info
 * call reads the header and checks the file size against it. */
typedef struct blgpu_modes_info {
  int ny_inlet, n_modes, m_modes;
  double beta, omega;
} blgpu_modes_info;
int blgpu_read_temporal_modes_info(const char *path, blgpu_modes_info *h);
/* The modes on the solver's mesh, ready for blgpu_set_inflow_modes:
 * zmode(n) = beta * file zmode, tmode(m) = omega * file tmode; qu(nyg,n,m)
 * and qw(nyg,n,m) interpolated linearly to the cell centres yg, qv(ny,n,m)
 * to the faces y (the face grid y(ny) is given; centres and ghosts as in
 * initialization.f90:174-222); rows at or above the file's last ymesh point
 * are zero, as in the reference.  Complex values as interleaved (re, im)
 * doubles; ymesh (may be NULL) receives the file's mesh. */
int blgpu_read_temporal_modes(const char *path, int ny, const double *y, double *zmode, double *tmode, double *qu,
                              double *qv, double *qw, double *ymesh);

#ifdef __cplusplus
}
#endif
#endif
