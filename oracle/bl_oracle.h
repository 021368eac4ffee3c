/*
 * bl_oracle.h -- CPU restatement of the boundary-layer DNS time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity oracle: it restates,
 * in plain C99 FP64, the step path of the reference CPU build (Makefile.cpu)
 * of ms-alvaro/boundary-layer-gpu so that the CUDA path can be checked
 * against it.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it; the product never does.
 *
 * Arrays crossing this interface use the reference's Fortran layout
 * (column-major, i fastest) with the reference's bounds:
 *   U(nx ,nyg,nzg)  V(nxg,ny ,nzg)  W(nxg,nyg,nz )  P(nxg,nyg,nzg)
 * with nxg=nx+1, nyg=ny+1, nzg=nz+1 (global.f90:86-88, initialization.f90:
 * 118-121 at nprocs=1).
 */
#ifndef BL_ORACLE_H
#define BL_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct blo blo_t;

/* poisson_variant: 0 = solve_poisson_cpu (4N embedding + zgtsv,
 * projection.f90:210-288), 1 = solve_poisson_gpu semantics (2N symmetric
 * extension + DCT twiddle + precomputed Thomas, projection.f90:93-204). */
blo_t *blo_create(int nx, int ny, int nz, double nu, double cfl, double dpdx,
                  double dpdz, int rk_scheme, int poisson_variant);
void blo_destroy(blo_t *o);
void blo_set_threads(int n);

/* faces x(nx), y(ny), z(nz); derives centres/ghosts/operators like
 * initialization.f90:174-222,329-344,395-469,482-484 */
int blo_set_grid(blo_t *o, const double *x, const double *y, const double *z);
/* U_inlet(nyg) V_inlet(ny) W_inlet(nyg) U_top(nx) V_top(nxg) W_top(nxg) */
void blo_set_bc(blo_t *o, const double *U_inlet, const double *V_inlet,
                const double *W_inlet, const double *U_top,
                const double *V_top, const double *W_top);
/* temporal inflow modes (boundary_conditions.f90:1740-1797): zmode(n),
 * tmode(m) already multiplied by beta/omega; q*(ny?,n,m) complex interleaved */
void blo_set_modes(blo_t *o, int n_modes, int m_modes, const double *zmode,
                   const double *tmode, const double *qu, const double *qv,
                   const double *qw);
void blo_set_state(blo_t *o, const double *U, const double *V,
                   const double *W, double t);
void blo_get_state(const blo_t *o, double *U, double *V, double *W,
                   double *P, double *t);
void blo_set_nu_t(blo_t *o, const double *nu_t, int les_model);
void blo_set_les(blo_t *o, int les_model); /* 1: Smagorinsky before every substep */

double blo_compute_dt(blo_t *o);  /* time_integration.f90:528-591 */
void blo_set_dt(blo_t *o, double dt);
double blo_get_dt(const blo_t *o);
void blo_step(blo_t *o);          /* one Euler/RK2/RK3 step */
void blo_rk3_stage(blo_t *o, int stage); /* one RK3 substep, stage 1..3 */

/* kernel-level entry points (equations.f90) -- host arrays, Fortran layout */
void blo_rhs_u(blo_t *o, const double *U, const double *V, const double *W,
               double *rhs_u);
void blo_rhs_v(blo_t *o, const double *U, const double *V, const double *W,
               double *rhs_v);
void blo_rhs_w(blo_t *o, const double *U, const double *V, const double *W,
               double *rhs_w);
void blo_apply_bc(blo_t *o, int rk_step);  /* boundary_conditions.f90:127 */
void blo_projection(blo_t *o, int rk_step); /* projection.f90:21 */
double blo_max_divergence(const blo_t *o);  /* projection.f90:391 */
/* rhs_p(2:nxg-1,2:nyg-1,2:nzg) after the last projection */
void blo_get_rhs_p(const blo_t *o, double *rhs_p);

/* models and diagnostics */
void blo_smagorinsky(blo_t *o);          /* subgrid.f90:609-730 */
void blo_dynamic_smagorinsky(blo_t *o);  /* subgrid.f90:261-583, LES = 2 or 3 from blo_set_les */
void blo_get_nu_t(const blo_t *o, double *nu_t);
void blo_statistics(const blo_t *o, double *means, double *nu_t_mean, double *Cf,
                    double *dUdy_wall, double *sc); /* statistics.f90:26-201 */
int blo_law_of_wall(const blo_t *o, double *utau); /* wallmodel.f90:1951-1985 */

/* Lund recycling/rescaling inflow (rescaled_inlet_bc.f90:60-345); mode 0 off,
 * 3 = whole inlet plane (inflow flag 3), 5 = fluctuations added to the inlet
 * profile (flag 5).  Umean0(nyg)/Vmean0(ny): restart means or NULL. */
int blo_set_rescaling(blo_t *o, int mode, int i_rescale, double delta_inlet, double T_resc,
                      const double *Umean0, const double *Vmean0);
void blo_rescaled_inflow(blo_t *o);
/* diag: Uinf, delta_resc, delta_inlet, theta_resc, theta_inlet, utau_resc,
 * utau_inlet, gamma */
void blo_get_rescaling(const blo_t *o, double *Umean_resc, double *Vmean_resc, double *Umean_inlet,
                       double *Vmean_inlet, double *Lu, double *Lv, double *Lw, double *diag, int *err);

/* wall-stress network (mlp_oracle.c): params[8770] in the device order;
 * exact = 0 rounds like the BF16 tensor-core kernels, 1 is plain FP64 */
int blo_mlp_nparams(void);
void blo_mlp_forward(const double *params, const float *X, int rows, float *Y, int exact);
double blo_mlp_gradient(const double *params, const float *X, const float *T, int rows, double *grad, int exact);

/* wall model of the step (mode 0 no-slip, 1 law of the wall at row jh,
 * 2 the network at row jh with params[8770]), evaluated at the start of
 * every substep and applied as U(:,1,:) = U(:,2,:) - tau/nu_w (yg(2)-yg(1)) */
int blo_set_wall_model(blo_t *o, int mode, int jh, const double *params);
/* the model's stress on the current state: (nx-2)(nzg-3) values each */
void blo_wall_stress(blo_t *o, double *tau_x, double *tau_z);

/* test hooks for the transform and the tridiagonal solver */
void blo_fft(int n, double *data, int inverse);
int blo_zgtsv(int n, double *dl, double *d, double *du, double *b);
void blo_dct2(int n, const double *f, double *c);

#ifdef __cplusplus
}
#endif
#endif
