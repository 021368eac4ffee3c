/*
 * bl_oracle.c -- CPU restatement of the boundary-layer DNS step path.
 *
 * TEST INFRASTRUCTURE ONLY (parity oracle, CPU baseline).  Never linked into
 * or called by the product library.  Each routine cites the reference
 * Fortran it restates (paths relative to the ms-alvaro/boundary-layer-gpu
 * source tree).  Compile with -O2 -ffp-contract=off so that every FP64
 * expression is evaluated in the order the Fortran source writes it, without
 * fused multiply-adds (the reference CPU build, gfortran -O2 on x86-64, has
 * none either).
 *
 * Third-party arithmetic that the reference takes from libraries is restated
 * here from the published algorithms:
 *   - FFTW 3 complex DFT (projection.f90:233,277): a recursive mixed-radix
 *     Cooley-Tukey transform, with Bluestein's chirp-z algorithm for lengths
 *     with a prime factor above 64;
 *   - LAPACK ZGTSV (projection.f90:253): Gaussian elimination with partial
 *     pivoting for a tridiagonal system, as in the LAPACK reference routine.
 */
#include "bl_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

/* ------------------------------------------------------------------------ */
/* FFT: recursive decimation in time, arbitrary length                      */
/* ------------------------------------------------------------------------ */

typedef struct fft_plan {
  int n;
  int nfac;
  int fac[64]; /* pairs (p, m) like the recursion consumes them */
  cplx *tw;    /* tw[j] = exp(-2 pi i j / n) */
  /* Bluestein */
  int blue;
  int m;
  cplx *chirp;  /* exp(-i pi j^2 / n), j = 0..n-1 */
  cplx *bfft;   /* FFT_m of the conjugate chirp, wrapped */
  struct fft_plan *sub;
} fft_plan;

static int largest_prime_factor(int n) {
  int lp = 1;
  for (int p = 2; p * p <= n; ++p)
    while (n % p == 0) { lp = p; n /= p; }
  if (n > 1) lp = n > lp ? n : lp;
  return lp;
}

static fft_plan *fft_plan_create(int n);
static void fft_exec(const fft_plan *pl, cplx *data, cplx *work);
static size_t fft_work_size(const fft_plan *pl);

static void fft_plan_free(fft_plan *p) {
  if (!p) return;
  free(p->tw);
  free(p->chirp);
  free(p->bfft);
  fft_plan_free(p->sub);
  free(p);
}

static fft_plan *fft_plan_create(int n) {
  fft_plan *p = (fft_plan *)calloc(1, sizeof(fft_plan));
  p->n = n;
  p->tw = (cplx *)malloc(sizeof(cplx) * (size_t)n);
  for (int j = 0; j < n; ++j) {
    double a = -2.0 * M_PI * (double)j / (double)n;
    p->tw[j] = cos(a) + I * sin(a);
  }
  if (n > 64 && largest_prime_factor(n) > 64) {
    /* Bluestein: X_k = c_k * sum_j (x_j c_j) conj(c_{k-j}), c_j = e^{-i pi j^2/n} */
    p->blue = 1;
    int m = 1;
    while (m < 2 * n - 1) m <<= 1;
    p->m = m;
    p->chirp = (cplx *)malloc(sizeof(cplx) * (size_t)n);
    for (int j = 0; j < n; ++j) {
      long long jj = ((long long)j * j) % (2LL * n);
      double a = -M_PI * (double)jj / (double)n;
      p->chirp[j] = cos(a) + I * sin(a);
    }
    p->sub = fft_plan_create(m);
    p->bfft = (cplx *)calloc((size_t)m, sizeof(cplx));
    p->bfft[0] = conj(p->chirp[0]);
    for (int j = 1; j < n; ++j) {
      p->bfft[j] = conj(p->chirp[j]);
      p->bfft[m - j] = conj(p->chirp[j]);
    }
    {
      cplx *w = (cplx *)malloc(sizeof(cplx) * fft_work_size(p->sub));
      fft_exec(p->sub, p->bfft, w);
      free(w);
    }
    return p;
  }
  /* factorisation: 4s first, then 2, 3, 5, ... */
  int rem = n, k = 0;
  while (rem > 1) {
    int f;
    if (rem % 4 == 0) f = 4;
    else if (rem % 2 == 0) f = 2;
    else {
      f = 3;
      while (rem % f) f += 2;
    }
    rem /= f;
    p->fac[k++] = f;
    p->fac[k++] = rem;
  }
  p->nfac = k / 2;
  return p;
}

/* one level of the recursion: out[0..p*m) from in with stride */
static void fft_work(const fft_plan *pl, cplx *out, const cplx *in,
                     size_t fstride, size_t istride, const int *fac,
                     cplx *scratch) {
  const int p = fac[0], m = fac[1];
  if (m == 1) {
    for (int q = 0; q < p; ++q) out[q] = in[(size_t)q * fstride * istride];
  } else {
    for (int q = 0; q < p; ++q)
      fft_work(pl, out + (size_t)q * m, in + (size_t)q * fstride * istride,
               fstride * (size_t)p, istride, fac + 2, scratch);
  }
  const int n = pl->n;
  const cplx *tw = pl->tw;
  if (p == 2) {
    for (int u = 0; u < m; ++u) {
      cplx t = out[u + m] * tw[(size_t)u * fstride];
      out[u + m] = out[u] - t;
      out[u] = out[u] + t;
    }
    return;
  }
  if (p == 4) {
    for (int u = 0; u < m; ++u) {
      cplx a0 = out[u];
      cplx a1 = out[u + m] * tw[(size_t)u * fstride];
      cplx a2 = out[u + 2 * m] * tw[(size_t)2 * u * fstride];
      cplx a3 = out[u + 3 * m] * tw[(size_t)3 * u * fstride];
      cplx s0 = a0 + a2, s1 = a0 - a2, s2 = a1 + a3, s3 = a1 - a3;
      cplx s3j = cimag(s3) - I * creal(s3); /* -i * s3 */
      out[u] = s0 + s2;
      out[u + 2 * m] = s0 - s2;
      out[u + m] = s1 + s3j;
      out[u + 3 * m] = s1 - s3j;
    }
    return;
  }
  /* generic odd radix */
  for (int u = 0; u < m; ++u) {
    for (int q = 0; q < p; ++q) scratch[q] = out[u + q * m];
    for (int q1 = 0; q1 < p; ++q1) {
      size_t k = (size_t)u + (size_t)q1 * m;
      cplx acc = scratch[0];
      size_t idx = 0, step = fstride * k % (size_t)n;
      for (int q = 1; q < p; ++q) {
        idx += step;
        if (idx >= (size_t)n) idx -= (size_t)n;
        acc += scratch[q] * tw[idx];
      }
      out[k] = acc;
    }
  }
}

/* forward (e^{-i}) unnormalised DFT, in place on data[0..n) */
static void fft_exec(const fft_plan *pl, cplx *data, cplx *work) {
  const int n = pl->n;
  if (n == 1) return;
  if (pl->blue) {
    const int m = pl->m;
    cplx *a = work;           /* m */
    cplx *w2 = work + m;      /* m + sub work */
    for (int j = 0; j < n; ++j) a[j] = data[j] * pl->chirp[j];
    for (int j = n; j < m; ++j) a[j] = 0;
    fft_exec(pl->sub, a, w2);
    for (int j = 0; j < m; ++j) a[j] *= pl->bfft[j];
    /* inverse via conjugation */
    for (int j = 0; j < m; ++j) a[j] = conj(a[j]);
    fft_exec(pl->sub, a, w2);
    const double inv = 1.0 / (double)m;
    for (int j = 0; j < n; ++j) data[j] = conj(a[j]) * inv * pl->chirp[j];
    return;
  }
  cplx *out = work;
  cplx *scratch = work + n;
  fft_work(pl, out, data, 1, 1, pl->fac, scratch);
  memcpy(data, out, sizeof(cplx) * (size_t)n);
}

static size_t fft_work_size(const fft_plan *pl) {
  if (pl->blue) return (size_t)pl->m + fft_work_size(pl->sub);
  return (size_t)pl->n + (size_t)pl->n + 8;
}

static void fft_exec_dir(const fft_plan *pl, cplx *data, cplx *work,
                         int inverse) {
  if (!inverse) {
    fft_exec(pl, data, work);
    return;
  }
  for (int j = 0; j < pl->n; ++j) data[j] = conj(data[j]);
  fft_exec(pl, data, work);
  for (int j = 0; j < pl->n; ++j) data[j] = conj(data[j]);
}

void blo_fft(int n, double *data, int inverse) {
  fft_plan *pl = fft_plan_create(n);
  cplx *work = (cplx *)malloc(sizeof(cplx) * fft_work_size(pl));
  fft_exec_dir(pl, (cplx *)data, work, inverse);
  free(work);
  fft_plan_free(pl);
}

/* unnormalised DCT-II, c_k = sum_m f_m cos(pi k (2m+1) / 2n), via the 4n
 * odd-slot embedding of projection.f90:221-233 (returns half of that DFT) */
void blo_dct2(int n, const double *f, double *c) {
  fft_plan *pl = fft_plan_create(4 * n);
  cplx *g = (cplx *)calloc((size_t)4 * n, sizeof(cplx));
  cplx *work = (cplx *)malloc(sizeof(cplx) * fft_work_size(pl));
  for (int m = 0; m < n; ++m) {
    g[2 * m + 1] = f[m];
    g[4 * n - 1 - 2 * m] = f[m];
  }
  fft_exec(pl, g, work);
  for (int k = 0; k < n; ++k) c[k] = 0.5 * creal(g[k]);
  free(g);
  free(work);
  fft_plan_free(pl);
}

/* ------------------------------------------------------------------------ */
/* ZGTSV restated: LAPACK's tridiagonal solve with partial pivoting.         */
/* dl(n-1), d(n), du(n-1), b(n) complex; returns info like LAPACK.           */
/* ------------------------------------------------------------------------ */
static double cabs1(cplx z) { return fabs(creal(z)) + fabs(cimag(z)); }

static int zgtsv_c(int n, cplx *dl, cplx *d, cplx *du, cplx *b) {
  if (n <= 0) return 0;
  for (int k = 0; k < n - 1; ++k) {
    if (dl[k] == 0) {
      if (d[k] == 0) return k + 1;
    } else if (cabs1(d[k]) >= cabs1(dl[k])) {
      cplx mult = dl[k] / d[k];
      d[k + 1] = d[k + 1] - mult * du[k];
      b[k + 1] = b[k + 1] - mult * b[k];
      if (k < n - 2) dl[k] = 0;
    } else {
      cplx mult = d[k] / dl[k];
      d[k] = dl[k];
      cplx temp = d[k + 1];
      d[k + 1] = du[k] - mult * temp;
      if (k < n - 2) {
        dl[k] = du[k + 1];
        du[k + 1] = -mult * dl[k];
      }
      du[k] = temp;
      temp = b[k];
      b[k] = b[k + 1];
      b[k + 1] = temp - mult * b[k + 1];
    }
  }
  if (d[n - 1] == 0) return n;
  b[n - 1] = b[n - 1] / d[n - 1];
  if (n > 1) b[n - 2] = (b[n - 2] - du[n - 2] * b[n - 1]) / d[n - 2];
  for (int k = n - 3; k >= 0; --k)
    b[k] = (b[k] - du[k] * b[k + 1] - dl[k] * b[k + 2]) / d[k];
  return 0;
}

int blo_zgtsv(int n, double *dl, double *d, double *du, double *b) {
  return zgtsv_c(n, (cplx *)dl, (cplx *)d, (cplx *)du, (cplx *)b);
}

/* ------------------------------------------------------------------------ */
/* solver state                                                              */
/* ------------------------------------------------------------------------ */

struct blo {
  int nx, ny, nz, nxg, nyg, nzg;
  int nxp, nzp, nm;
  double nu, cfl, dpdx, dpdz;
  int rk_scheme, variant, les;
  /* grids, 1-based (index 0 unused) */
  double *x, *y, *z, *xm, *ym, *zm, *xg, *yg, *zg, *wy0, *wy1;
  double dxmin, dymin, dzmin, dx, dz;
  double *kxx, *kzz;               /* 0-based */
  double *Dd, *Dl, *Du;            /* Dyy(j,j), Dyy(j+1,j), Dyy(j,j+1), j=2..nyg-1 stored at [j] */
  /* fields, Fortran layout */
  double *U, *V, *W, *P, *Uo, *Vo, *Wo;
  double *Fu[3], *Fv[3], *Fw[3];
  double *rhs_p;                   /* (2:nxg-1, 2:nyg-1, 2:nzg) */
  double *nu_t;                    /* (nxg, nyg, nzg) */
  /* boundary data */
  double *U_inlet, *V_inlet, *W_inlet, *U_top, *V_top, *W_top;
  double *Ut, *Vt, *Wt;            /* (nyg,nzg) (ny,nzg) (nyg,nz) */
  int n_modes, m_modes;
  double *zmode, *tmode;
  cplx *qu, *qv, *qw;
  double t, dt;
  int rk_step;
  /* RK tables (initialization.f90:504-530) */
  double rk_t[4], rk_coef[3][3], rk2_t[3], rk2_coef[2][2];
  /* projection work */
  fft_plan *pl_x, *pl_z;           /* 4N (variant 0) or 2N (variant 1); nzp */
  cplx *rhs_hat;                   /* (0:nxp-1, nm, 0:nzp-1) */
  cplx *th_dl, *th_dp, *th_du;     /* variant 1 factors (nxp, nzp, nm) */
  cplx *twid;                      /* DCT twiddle, 0..nxp-1 */
  /* Lund recycling/rescaling inflow (rescaled_inlet_bc.f90) */
  int resc_mode, i_rescale, lund_err;  /* mode 0 off, 3 full plane, 5 fluctuations */
  double delta_inlet, T_resc;
  double *Umr, *Vmr, *Umi, *Vmi;   /* Umean_resc_T(nyg) Vmean_resc_T(ny) Umean_inlet_T Vmean_inlet_T, 1-based */
  double *Lu, *Lv, *Lw;            /* Ut_inlet(nyg,nzg) Vt_inlet(ny,nzg) Wt_inlet(nyg,nz) */
  double lund_diag[8];
  /* wall model */
  int wm, wm_jh;
  double *wm_ax, *wm_az, *utau_wm, *mlp_params;
};

static int nthreads_req = 1;
void blo_set_threads(int n) {
  nthreads_req = n > 0 ? n : 1;
#ifdef _OPENMP
  omp_set_num_threads(nthreads_req);
#endif
}

/* Fortran-layout index helpers, 1-based indices as in the source */
#define IX3(i, j, k, n1, n2) \
  (((size_t)((k)-1) * (size_t)(n2) + (size_t)((j)-1)) * (size_t)(n1) + (size_t)((i)-1))
#define AU(a, i, j, k) (a)[IX3(i, j, k, o->nx, o->nyg)]
#define AV(a, i, j, k) (a)[IX3(i, j, k, o->nxg, o->ny)]
#define AW(a, i, j, k) (a)[IX3(i, j, k, o->nxg, o->nyg)]
#define AP(a, i, j, k) (a)[IX3(i, j, k, o->nxg, o->nyg)]
/* rhs arrays with lower bound 2 in every dimension */
#define RU(a, i, j, k) (a)[IX3((i)-1, (j)-1, (k)-1, o->nx - 2, o->nyg - 2)]
#define RV(a, i, j, k) (a)[IX3((i)-1, (j)-1, (k)-1, o->nxg - 2, o->ny - 2)]
#define RW(a, i, j, k) (a)[IX3((i)-1, (j)-1, (k)-1, o->nxg - 2, o->nyg - 2)]
#define RP(a, i, j, k) (a)[IX3((i)-1, (j)-1, (k)-1, o->nxg - 2, o->nyg - 2)]

static double *dalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

blo_t *blo_create(int nx, int ny, int nz, double nu, double cfl, double dpdx,
                  double dpdz, int rk_scheme, int poisson_variant) {
  if (nx < 4 || ny < 4 || nz < 4) return NULL;
  blo_t *o = (blo_t *)calloc(1, sizeof(blo_t));
  o->nx = nx; o->ny = ny; o->nz = nz;
  o->nxg = nx + 1; o->nyg = ny + 1; o->nzg = nz + 1;
  o->nxp = nx - 2; o->nzp = nz - 2; o->nm = ny - 1;
  o->nu = nu; o->cfl = cfl; o->dpdx = dpdx; o->dpdz = dpdz;
  o->rk_scheme = rk_scheme; o->variant = poisson_variant;
  o->x = dalloc(nx + 1); o->y = dalloc(ny + 1); o->z = dalloc(nz + 1);
  o->xm = dalloc(nx); o->ym = dalloc(ny); o->zm = dalloc(nz);
  o->xg = dalloc(nx + 2); o->yg = dalloc(ny + 2); o->zg = dalloc(nz + 2);
  o->wy0 = dalloc(ny + 1); o->wy1 = dalloc(ny + 1);
  o->kxx = dalloc(o->nxp); o->kzz = dalloc(o->nzp);
  o->Dd = dalloc(o->nyg + 1); o->Dl = dalloc(o->nyg + 1); o->Du = dalloc(o->nyg + 1);
  size_t su = (size_t)nx * o->nyg * o->nzg, sv = (size_t)o->nxg * ny * o->nzg,
         sw = (size_t)o->nxg * o->nyg * nz, sp = (size_t)o->nxg * o->nyg * o->nzg;
  o->U = dalloc(su); o->V = dalloc(sv); o->W = dalloc(sw); o->P = dalloc(sp);
  o->Uo = dalloc(su); o->Vo = dalloc(sv); o->Wo = dalloc(sw);
  o->nu_t = dalloc(sp);
  size_t fu = (size_t)(nx - 2) * (o->nyg - 2) * (o->nzg - 2),
         fv = (size_t)(o->nxg - 2) * (ny - 2) * (o->nzg - 2),
         fw = (size_t)(o->nxg - 2) * (o->nyg - 2) * (nz - 2);
  for (int s = 0; s < 3; ++s) {
    o->Fu[s] = dalloc(fu); o->Fv[s] = dalloc(fv); o->Fw[s] = dalloc(fw);
  }
  o->rhs_p = dalloc((size_t)(o->nxg - 2) * (o->nyg - 2) * (o->nzg - 1));
  o->U_inlet = dalloc(o->nyg + 1); o->V_inlet = dalloc(ny + 1); o->W_inlet = dalloc(o->nyg + 1);
  o->U_top = dalloc(nx + 1); o->V_top = dalloc(o->nxg + 1); o->W_top = dalloc(o->nxg + 1);
  o->Ut = dalloc((size_t)o->nyg * o->nzg); o->Vt = dalloc((size_t)ny * o->nzg);
  o->Wt = dalloc((size_t)o->nyg * nz);
  o->Umr = dalloc(o->nyg + 1); o->Vmr = dalloc(ny + 1);
  o->Umi = dalloc(o->nyg + 1); o->Vmi = dalloc(ny + 1);
  o->Lu = dalloc((size_t)o->nyg * o->nzg); o->Lv = dalloc((size_t)ny * o->nzg);
  o->Lw = dalloc((size_t)o->nyg * nz);
  o->wm_ax = dalloc((size_t)(nx - 2) * (o->nzg - 3));
  o->wm_az = dalloc((size_t)(nx - 2) * (o->nzg - 3));
  o->utau_wm = dalloc(nx);
  o->mlp_params = dalloc(blo_mlp_nparams());
  o->rk_t[0] = 0.0; o->rk_t[1] = 8.0 / 15.0; o->rk_t[2] = 2.0 / 3.0; o->rk_t[3] = 1.0;
  memset(o->rk_coef, 0, sizeof(o->rk_coef));
  o->rk_coef[0][0] = 8.0 / 15.0;
  o->rk_coef[1][0] = 1.0 / 4.0; o->rk_coef[1][1] = 5.0 / 12.0;
  o->rk_coef[2][0] = 1.0 / 4.0; o->rk_coef[2][1] = 0.0; o->rk_coef[2][2] = 3.0 / 4.0;
  o->rk2_t[0] = 0.0; o->rk2_t[1] = 1.0 / 2.0; o->rk2_t[2] = 1.0;
  o->rk2_coef[0][0] = 1.0 / 2.0; o->rk2_coef[0][1] = 0.0;
  o->rk2_coef[1][0] = 0.0; o->rk2_coef[1][1] = 1.0;
  o->rhs_hat = (cplx *)calloc((size_t)o->nxp * o->nm * o->nzp, sizeof(cplx));
  o->pl_z = fft_plan_create(o->nzp);
  o->pl_x = fft_plan_create(poisson_variant ? 2 * o->nxp : 4 * o->nxp);
  return o;
}

void blo_destroy(blo_t *o) {
  if (!o) return;
  double *arrs[] = {o->x, o->y, o->z, o->xm, o->ym, o->zm, o->xg, o->yg, o->zg,
                    o->wy0, o->wy1, o->kxx, o->kzz, o->Dd, o->Dl, o->Du, o->U,
                    o->V, o->W, o->P, o->Uo, o->Vo, o->Wo, o->nu_t, o->rhs_p,
                    o->U_inlet, o->V_inlet, o->W_inlet, o->U_top, o->V_top,
                    o->W_top, o->Ut, o->Vt, o->Wt, o->zmode, o->tmode,
                    o->Umr, o->Vmr, o->Umi, o->Vmi, o->Lu, o->Lv, o->Lw, o->wm_ax, o->wm_az,
                    o->utau_wm, o->mlp_params};
  for (size_t q = 0; q < sizeof(arrs) / sizeof(arrs[0]); ++q) free(arrs[q]);
  for (int s = 0; s < 3; ++s) { free(o->Fu[s]); free(o->Fv[s]); free(o->Fw[s]); }
  free(o->qu); free(o->qv); free(o->qw);
  free(o->rhs_hat); free(o->th_dl); free(o->th_dp); free(o->th_du); free(o->twid);
  fft_plan_free(o->pl_x); fft_plan_free(o->pl_z);
  free(o);
}

/* initialization.f90:174-222 (centres, ghosts, minimum spacing),
 * 254-259 (dx, dz), 329-344 (modified wavenumbers), 395-425 (Dyy),
 * 428-469 (Thomas factors, variant 1), 482-484 (weights), 316-320 (twiddle) */
int blo_set_grid(blo_t *o, const double *x, const double *y, const double *z) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  const int nxm = nx - 1, nym = ny - 1, nzm = nz - 1;
  for (int i = 1; i <= nx; ++i) o->x[i] = x[i - 1];
  for (int j = 1; j <= ny; ++j) o->y[j] = y[j - 1];
  for (int k = 1; k <= nz; ++k) o->z[k] = z[k - 1];
  for (int i = 1; i <= nxm; ++i) o->xm[i] = 0.5 * (o->x[i] + o->x[i + 1]);
  for (int j = 1; j <= nym; ++j) o->ym[j] = 0.5 * (o->y[j] + o->y[j + 1]);
  for (int k = 1; k <= nzm; ++k) o->zm[k] = 0.5 * (o->z[k] + o->z[k + 1]);
  for (int i = 1; i <= nxm; ++i) o->xg[i + 1] = o->xm[i];
  o->xg[1] = o->xm[1] - 2.0 * (o->xm[1] - o->x[1]);
  o->xg[nxm + 2] = o->xm[nxm] + 2.0 * (o->x[nx] - o->xm[nxm]);
  for (int j = 1; j <= nym; ++j) o->yg[j + 1] = o->ym[j];
  o->yg[1] = o->ym[1] - 2.0 * (o->ym[1] - o->y[1]);
  o->yg[nym + 2] = o->ym[nym] + 2.0 * (o->y[ny] - o->ym[nym]);
  for (int k = 1; k <= nzm; ++k) o->zg[k + 1] = o->zm[k];
  o->zg[1] = o->zm[1] - 2.0 * (o->zm[1] - o->z[1]);
  o->zg[nzm + 2] = o->zm[nzm] + 2.0 * (o->z[nz] - o->zm[nzm]);
  double mn;
  mn = INFINITY;
  for (int i = 2; i <= o->nxg; ++i) { double d = o->xg[i] - o->xg[i - 1]; if (d < mn) mn = d; }
  o->dxmin = mn;
  mn = INFINITY;
  for (int j = 2; j <= o->nyg; ++j) { double d = o->yg[j] - o->yg[j - 1]; if (d < mn) mn = d; }
  o->dymin = mn;
  mn = INFINITY;
  for (int k = 2; k <= o->nzg; ++k) { double d = o->zg[k] - o->zg[k - 1]; if (d < mn) mn = d; }
  o->dzmin = mn;
  o->dx = o->dxmin;
  o->dz = o->dzmin;
  const double pi = 4.0 * atan(1.0);
  const int nxp = o->nxp, nzp = o->nzp;
  for (int i = 0; i < nxp; ++i)
    o->kxx[i] = 2.0 * (cos(pi * (double)i / (double)nxp) - 1.0) / (o->dx * o->dx);
  int half = (int)ceil((double)nzp / 2.0);
  for (int k = 0; k <= half && k < nzp; ++k)
    o->kzz[k] = 2.0 * (cos(2.0 * pi * (double)k / (double)nzp) - 1.0) / (o->dz * o->dz);
  for (int k = half + 1; k < nzp; ++k)
    o->kzz[k] = 2.0 * (cos(2.0 * pi * (double)(-nzp + k) / (double)nzp) - 1.0) / (o->dz * o->dz);
  /* Dyy: rows j = 2..nyg-1 */
  const double *yy = o->y, *yg = o->yg;
  const int nyg = o->nyg;
  for (int j = 2; j <= nyg - 1; ++j) {
    double a = 1.0 / (yy[j] - yy[j - 1]) / (yg[j + 1] - yg[j]);
    double b = 1.0 / (yy[j] - yy[j - 1]) * (-1.0 / (yg[j + 1] - yg[j]) - 1.0 / (yg[j] - yg[j - 1]));
    double c = 1.0 / (yy[j] - yy[j - 1]) / (yg[j] - yg[j - 1]);
    o->Du[j] = a;  /* Dyy(j,j+1) */
    o->Dl[j] = c;  /* Dyy(j,j-1) (sub-diagonal entry of row j) */
    o->Dd[j] = b;
    if (j == 2) o->Dd[j] = b + c;
    if (j == nyg - 1) o->Dd[j] = a + b;
  }
  /* weights: weight_y_0(j) = (yg(j+1)-y(j))/(yg(j+1)-yg(j)), j = 1..ny */
  for (int j = 1; j <= ny; ++j) {
    o->wy0[j] = (yg[j + 1] - yy[j]) / (yg[j + 1] - yg[j]);
    o->wy1[j] = 1.0 - o->wy0[j];
  }
  if (o->variant == 1) {
    const int nm = o->nm;
    free(o->th_dl); free(o->th_dp); free(o->th_du); free(o->twid);
    o->th_dl = (cplx *)calloc((size_t)nxp * nzp * nm, sizeof(cplx));
    o->th_dp = (cplx *)calloc((size_t)nxp * nzp * nm, sizeof(cplx));
    o->th_du = (cplx *)calloc((size_t)nm, sizeof(cplx));
    o->twid = (cplx *)calloc((size_t)nxp, sizeof(cplx));
    /* thomas_du(jj) = Dyy(jj+1, jj+2), jj = 1..nm-1 */
    for (int jj = 1; jj <= nm - 1; ++jj) o->th_du[jj - 1] = o->Du[jj + 1];
    o->th_du[nm - 1] = 0;
#define TH(a, ii, kk, jj) (a)[((size_t)((jj)-1) * nzp + (size_t)((kk)-1)) * nxp + (size_t)((ii)-1)]
    for (int kk = 1; kk <= nzp; ++kk)
      for (int ii = 1; ii <= nxp; ++ii) {
        int ig = ii - 1, kg = kk - 1;
        for (int jj = 1; jj <= nm; ++jj)
          TH(o->th_dp, ii, kk, jj) = o->Dd[jj + 1] + o->kxx[ig] + o->kzz[kg];
        /* thomas_dl_fact(jj) = Dyy(jj+2, jj+1): sub-diagonal of row jj+2 */
        for (int jj = 1; jj <= nm - 1; ++jj) TH(o->th_dl, ii, kk, jj) = o->Dl[jj + 2];
        TH(o->th_dl, ii, kk, nm) = 0;
        if (ig == 0 && kg == 0) TH(o->th_dp, ii, kk, 1) = 3.0 / 2.0 * TH(o->th_dp, ii, kk, 1);
        for (int jj = 2; jj <= nm; ++jj) {
          cplx dd = TH(o->th_dl, ii, kk, jj - 1) / TH(o->th_dp, ii, kk, jj - 1);
          TH(o->th_dl, ii, kk, jj - 1) = dd;
          TH(o->th_dp, ii, kk, jj) = TH(o->th_dp, ii, kk, jj) - dd * o->th_du[jj - 2];
        }
        for (int jj = 1; jj <= nm; ++jj) TH(o->th_dp, ii, kk, jj) = 1.0 / TH(o->th_dp, ii, kk, jj);
      }
#undef TH
    for (int i = 0; i < nxp; ++i) {
      double a = -pi * (double)i / (2.0 * (double)nxp);
      o->twid[i] = cos(a) + I * sin(a);
    }
  }
  return 0;
}

void blo_set_bc(blo_t *o, const double *U_inlet, const double *V_inlet,
                const double *W_inlet, const double *U_top, const double *V_top,
                const double *W_top) {
  for (int j = 1; j <= o->nyg; ++j) o->U_inlet[j] = U_inlet[j - 1];
  for (int j = 1; j <= o->ny; ++j) o->V_inlet[j] = V_inlet[j - 1];
  for (int j = 1; j <= o->nyg; ++j) o->W_inlet[j] = W_inlet[j - 1];
  for (int i = 1; i <= o->nx; ++i) o->U_top[i] = U_top[i - 1];
  for (int i = 1; i <= o->nxg; ++i) o->V_top[i] = V_top[i - 1];
  for (int i = 1; i <= o->nxg; ++i) o->W_top[i] = W_top[i - 1];
}

void blo_set_modes(blo_t *o, int n_modes, int m_modes, const double *zmode,
                   const double *tmode, const double *qu, const double *qv,
                   const double *qw) {
  free(o->zmode); free(o->tmode); free(o->qu); free(o->qv); free(o->qw);
  o->n_modes = n_modes; o->m_modes = m_modes;
  o->zmode = dalloc(n_modes); o->tmode = dalloc(m_modes);
  memcpy(o->zmode, zmode, sizeof(double) * (size_t)n_modes);
  memcpy(o->tmode, tmode, sizeof(double) * (size_t)m_modes);
  size_t nu_ = (size_t)o->nyg * n_modes * m_modes, nv_ = (size_t)o->ny * n_modes * m_modes;
  o->qu = (cplx *)malloc(sizeof(cplx) * nu_);
  o->qv = (cplx *)malloc(sizeof(cplx) * nv_);
  o->qw = (cplx *)malloc(sizeof(cplx) * nu_);
  memcpy(o->qu, qu, sizeof(cplx) * nu_);
  memcpy(o->qv, qv, sizeof(cplx) * nv_);
  memcpy(o->qw, qw, sizeof(cplx) * nu_);
}

void blo_set_state(blo_t *o, const double *U, const double *V, const double *W,
                   double t) {
  size_t su = (size_t)o->nx * o->nyg * o->nzg, sv = (size_t)o->nxg * o->ny * o->nzg,
         sw = (size_t)o->nxg * o->nyg * o->nz;
  memcpy(o->U, U, su * sizeof(double));
  memcpy(o->V, V, sv * sizeof(double));
  memcpy(o->W, W, sw * sizeof(double));
  /* read_input_data sets Uo = U (input_output.f90:476-478) */
  memcpy(o->Uo, U, su * sizeof(double));
  memcpy(o->Vo, V, sv * sizeof(double));
  memcpy(o->Wo, W, sw * sizeof(double));
  o->t = t;
}

void blo_get_state(const blo_t *o, double *U, double *V, double *W, double *P,
                   double *t) {
  size_t su = (size_t)o->nx * o->nyg * o->nzg, sv = (size_t)o->nxg * o->ny * o->nzg,
         sw = (size_t)o->nxg * o->nyg * o->nz, sp = (size_t)o->nxg * o->nyg * o->nzg;
  if (U) memcpy(U, o->U, su * sizeof(double));
  if (V) memcpy(V, o->V, sv * sizeof(double));
  if (W) memcpy(W, o->W, sw * sizeof(double));
  if (P) memcpy(P, o->P, sp * sizeof(double));
  if (t) *t = o->t;
}

void blo_set_nu_t(blo_t *o, const double *nu_t, int les_model) {
  memcpy(o->nu_t, nu_t, sizeof(double) * (size_t)o->nxg * o->nyg * o->nzg);
  o->les = les_model;
}

void blo_set_dt(blo_t *o, double dt) { o->dt = dt; }
double blo_get_dt(const blo_t *o) { return o->dt; }

/* ------------------------------------------------------------------------ */
/* RHS: equations.f90:24-415 (DNS branch and LES branch)                     */
/* ------------------------------------------------------------------------ */

#define NUT(i, j, k) o->nu_t[IX3(i, j, k, o->nxg, o->nyg)]

static void rhs_u_impl(blo_t *o, const double *U_, const double *V_,
                       const double *W_, double *rhs) {
  const double *x = o->x, *xg = o->xg, *y = o->y, *yg = o->yg, *z = o->z,
               *zg = o->zg, *w0 = o->wy0, *w1 = o->wy1;
  const double nu = o->nu, dPdx = o->dpdx;
  const int nx = o->nx, nyg = o->nyg, nzg = o->nzg;
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= nzg - 1; ++k)
    for (int j = 2; j <= nyg - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i) {
        /* equations.f90:53-64 */
        double a = 0.5 * (AU(U_, i, j, k) + AU(U_, i + 1, j, k));
        double b = 0.5 * (AU(U_, i - 1, j, k) + AU(U_, i, j, k));
        double r = -(a * a - b * b) / (xg[i + 1] - xg[i]);
        double t1 = (w0[j] * AU(U_, i, j, k) + w1[j] * AU(U_, i, j + 1, k)) * 0.5 *
                    (AV(V_, i, j, k) + AV(V_, i + 1, j, k));
        double t2 = (w0[j - 1] * AU(U_, i, j - 1, k) + w1[j - 1] * AU(U_, i, j, k)) * 0.5 *
                    (AV(V_, i, j - 1, k) + AV(V_, i + 1, j - 1, k));
        r = r - (t1 - t2) / (y[j] - y[j - 1]);
        double t3 = 0.5 * (AU(U_, i, j, k) + AU(U_, i, j, k + 1)) * 0.5 *
                    (AW(W_, i, j, k) + AW(W_, i + 1, j, k));
        double t4 = 0.5 * (AU(U_, i, j, k - 1) + AU(U_, i, j, k)) * 0.5 *
                    (AW(W_, i, j, k - 1) + AW(W_, i + 1, j, k - 1));
        r = r - (t3 - t4) / (z[k] - z[k - 1]);
        double dx_1 = x[i] - x[i - 1], dx_2 = x[i + 1] - x[i], dx_3 = xg[i + 1] - xg[i];
        double dy_3 = y[j] - y[j - 1];
        double dz_1 = zg[k] - zg[k - 1], dz_2 = zg[k + 1] - zg[k], dz_3 = z[k] - z[k - 1];
        double uc = AU(U_, i, j, k);
        if (o->les == 0) {
          /* equations.f90:88-91 */
          double vx = (1.0 / dx_2 * (AU(U_, i + 1, j, k) - uc) - 1.0 / dx_1 * (uc - AU(U_, i - 1, j, k))) / dx_3;
          double vy = ((AU(U_, i, j + 1, k) - uc) / (yg[j + 1] - yg[j]) -
                       (uc - AU(U_, i, j - 1, k)) / (yg[j] - yg[j - 1])) / dy_3;
          double vz = (1.0 / dz_2 * (AU(U_, i, j, k + 1) - uc) - 1.0 / dz_1 * (uc - AU(U_, i, j, k - 1))) / dz_3;
          r = r + dPdx + nu * (vx + vy + vz);
        } else {
          /* equations.f90:98-129 */
          double nu_x1 = nu + NUT(i, j, k);
          double nu_x2 = nu + NUT(i + 1, j, k);
          double nu_y1 = nu + 0.5 * (w0[j - 1] * NUT(i, j - 1, k) + w1[j - 1] * NUT(i, j, k) +
                                     w0[j - 1] * NUT(i + 1, j - 1, k) + w1[j - 1] * NUT(i + 1, j, k));
          double nu_y2 = nu + 0.5 * (w0[j] * NUT(i, j, k) + w1[j] * NUT(i, j + 1, k) +
                                     w0[j] * NUT(i + 1, j, k) + w1[j] * NUT(i + 1, j + 1, k));
          double nu_z1 = nu + 0.25 * (NUT(i, j, k) + NUT(i, j, k - 1) + NUT(i + 1, j, k) + NUT(i + 1, j, k - 1));
          double nu_z2 = nu + 0.25 * (NUT(i, j, k) + NUT(i, j, k + 1) + NUT(i + 1, j, k) + NUT(i + 1, j, k + 1));
          double t2p = (AU(U_, i, j + 1, k) - uc) / (yg[j + 1] - yg[j]);
          double t2m = (uc - AU(U_, i, j - 1, k)) / (yg[j] - yg[j - 1]);
          r = r + dPdx +
              (nu_x2 / dx_2 * (AU(U_, i + 1, j, k) - uc) - nu_x1 / dx_1 * (uc - AU(U_, i - 1, j, k))) / dx_3 +
              (nu_y2 * t2p - nu_y1 * t2m) / dy_3 +
              (nu_z2 / dz_2 * (AU(U_, i, j, k + 1) - uc) - nu_z1 / dz_1 * (uc - AU(U_, i, j, k - 1))) / dz_3;
        }
        RU(rhs, i, j, k) = r;
      }
  /* equations.f90:149-154 */
  for (int k = 2; k <= nzg - 1; ++k)
    for (int j = 2; j <= nyg - 1; ++j) RU(rhs, nx - 1, j, k) = 0.0;
}

static void rhs_v_impl(blo_t *o, const double *U_, const double *V_,
                       const double *W_, double *rhs) {
  const double *x = o->x, *xg = o->xg, *y = o->y, *yg = o->yg, *z = o->z,
               *zg = o->zg, *w0 = o->wy0, *w1 = o->wy1;
  const double nu = o->nu;
  const int nxg = o->nxg, ny = o->ny, nzg = o->nzg;
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= nzg - 1; ++k)
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nxg - 1; ++i) {
        /* equations.f90:188-201 */
        double a = 0.5 * (AV(V_, i, j, k) + AV(V_, i, j + 1, k));
        double b = 0.5 * (AV(V_, i, j - 1, k) + AV(V_, i, j, k));
        double r = -(a * a - b * b) / (yg[j + 1] - yg[j]);
        double t1 = (w0[j] * AU(U_, i, j, k) + w1[j] * AU(U_, i, j + 1, k)) * 0.5 *
                    (AV(V_, i, j, k) + AV(V_, i + 1, j, k));
        double t2 = (w0[j] * AU(U_, i - 1, j, k) + w1[j] * AU(U_, i - 1, j + 1, k)) * 0.5 *
                    (AV(V_, i - 1, j, k) + AV(V_, i, j, k));
        r = r - (t1 - t2) / (x[i] - x[i - 1]);
        double t3 = 0.5 * (AV(V_, i, j, k) + AV(V_, i, j, k + 1)) *
                    (w0[j] * AW(W_, i, j, k) + w1[j] * AW(W_, i, j + 1, k));
        double t4 = 0.5 * (AV(V_, i, j, k - 1) + AV(V_, i, j, k)) *
                    (w0[j] * AW(W_, i, j, k - 1) + w1[j] * AW(W_, i, j + 1, k - 1));
        r = r - (t3 - t4) / (z[k] - z[k - 1]);
        double dx_1 = xg[i] - xg[i - 1], dx_2 = xg[i + 1] - xg[i], dx_3 = x[i] - x[i - 1];
        double dy_1 = y[j] - y[j - 1], dy_2 = y[j + 1] - y[j], dy_3 = yg[j + 1] - yg[j];
        double dz_1 = zg[k] - zg[k - 1], dz_2 = zg[k + 1] - zg[k], dz_3 = z[k] - z[k - 1];
        double vc = AV(V_, i, j, k);
        if (o->les == 0) {
          /* equations.f90:224-227 */
          double vx = (1.0 / dx_2 * (AV(V_, i + 1, j, k) - vc) - 1.0 / dx_1 * (vc - AV(V_, i - 1, j, k))) / dx_3;
          double vy = (1.0 / dy_2 * (AV(V_, i, j + 1, k) - vc) - 1.0 / dy_1 * (vc - AV(V_, i, j - 1, k))) / dy_3;
          double vz = (1.0 / dz_2 * (AV(V_, i, j, k + 1) - vc) - 1.0 / dz_1 * (vc - AV(V_, i, j, k - 1))) / dz_3;
          r = r + nu * (vx + vy + vz);
        } else {
          /* equations.f90:238-266 */
          double nu_x1 = nu + 0.5 * (w0[j] * NUT(i - 1, j, k) + w1[j] * NUT(i - 1, j + 1, k) +
                                     w0[j] * NUT(i, j, k) + w1[j] * NUT(i, j + 1, k));
          double nu_x2 = nu + 0.5 * (w0[j] * NUT(i, j, k) + w1[j] * NUT(i, j + 1, k) +
                                     w0[j] * NUT(i + 1, j, k) + w1[j] * NUT(i + 1, j + 1, k));
          double nu_y1 = nu + NUT(i, j, k);
          double nu_y2 = nu + NUT(i, j + 1, k);
          double nu_z1 = nu + 0.5 * (w0[j] * NUT(i, j, k - 1) + w1[j] * NUT(i, j + 1, k - 1) +
                                     w0[j] * NUT(i, j, k) + w1[j] * NUT(i, j + 1, k));
          double nu_z2 = nu + 0.5 * (w0[j] * NUT(i, j, k) + w1[j] * NUT(i, j + 1, k) +
                                     w0[j] * NUT(i, j, k + 1) + w1[j] * NUT(i, j + 1, k + 1));
          r = r +
              1.0 / dx_3 * (nu_x2 * 1.0 / dx_2 * (AV(V_, i + 1, j, k) - vc) - nu_x1 * 1.0 / dx_1 * (vc - AV(V_, i - 1, j, k))) +
              1.0 / dy_3 * (nu_y2 * 1.0 / dy_2 * (AV(V_, i, j + 1, k) - vc) - nu_y1 * 1.0 / dy_1 * (vc - AV(V_, i, j - 1, k))) +
              1.0 / dz_3 * (nu_z2 * 1.0 / dz_2 * (AV(V_, i, j, k + 1) - vc) - nu_z1 * 1.0 / dz_1 * (vc - AV(V_, i, j, k - 1)));
        }
        RV(rhs, i, j, k) = r;
      }
  /* equations.f90:287-292 */
  for (int k = 2; k <= nzg - 1; ++k)
    for (int j = 2; j <= ny - 1; ++j) RV(rhs, nxg - 1, j, k) = 0.0;
}

static void rhs_w_impl(blo_t *o, const double *U_, const double *V_,
                       const double *W_, double *rhs) {
  const double *x = o->x, *xg = o->xg, *y = o->y, *yg = o->yg, *z = o->z,
               *zg = o->zg, *w0 = o->wy0, *w1 = o->wy1;
  const double nu = o->nu, dPdz = o->dpdz;
  const int nxg = o->nxg, nyg = o->nyg, nz = o->nz;
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= nz - 1; ++k)
    for (int j = 2; j <= nyg - 1; ++j)
      for (int i = 2; i <= nxg - 1; ++i) {
        /* equations.f90:328-339 */
        double a = 0.5 * (AW(W_, i, j, k) + AW(W_, i, j, k + 1));
        double b = 0.5 * (AW(W_, i, j, k - 1) + AW(W_, i, j, k));
        double r = -(a * a - b * b) / (zg[k + 1] - zg[k]);
        double t1 = 0.5 * (AU(U_, i, j, k) + AU(U_, i, j, k + 1)) * 0.5 *
                    (AW(W_, i, j, k) + AW(W_, i + 1, j, k));
        double t2 = 0.5 * (AU(U_, i - 1, j, k) + AU(U_, i - 1, j, k + 1)) * 0.5 *
                    (AW(W_, i - 1, j, k) + AW(W_, i, j, k));
        r = r - (t1 - t2) / (x[i] - x[i - 1]);
        double t3 = 0.5 * (AV(V_, i, j, k) + AV(V_, i, j, k + 1)) *
                    (w0[j] * AW(W_, i, j, k) + w1[j] * AW(W_, i, j + 1, k));
        double t4 = 0.5 * (AV(V_, i, j - 1, k) + AV(V_, i, j - 1, k + 1)) *
                    (w0[j - 1] * AW(W_, i, j - 1, k) + w1[j - 1] * AW(W_, i, j, k));
        r = r - (t3 - t4) / (y[j] - y[j - 1]);
        double dx_1 = xg[i] - xg[i - 1], dx_2 = xg[i + 1] - xg[i], dx_3 = x[i] - x[i - 1];
        double dy_3 = y[j] - y[j - 1];
        double dz_1 = z[k] - z[k - 1], dz_2 = z[k + 1] - z[k], dz_3 = zg[k + 1] - zg[k];
        double wc = AW(W_, i, j, k);
        if (o->les == 0) {
          /* equations.f90:360-363 */
          double vx = (1.0 / dx_2 * (AW(W_, i + 1, j, k) - wc) - 1.0 / dx_1 * (wc - AW(W_, i - 1, j, k))) / dx_3;
          double vy = ((AW(W_, i, j + 1, k) - wc) / (yg[j + 1] - yg[j]) -
                       (wc - AW(W_, i, j - 1, k)) / (yg[j] - yg[j - 1])) / dy_3;
          double vz = (1.0 / dz_2 * (AW(W_, i, j, k + 1) - wc) - 1.0 / dz_1 * (wc - AW(W_, i, j, k - 1))) / dz_3;
          r = r + dPdz + nu * (vx + vy + vz);
        } else {
          /* equations.f90:370-401 */
          double nu_x1 = nu + 0.25 * (NUT(i, j, k) + NUT(i, j, k + 1) + NUT(i - 1, j, k) + NUT(i - 1, j, k + 1));
          double nu_x2 = nu + 0.25 * (NUT(i, j, k) + NUT(i, j, k + 1) + NUT(i + 1, j, k) + NUT(i + 1, j, k + 1));
          double nu_y1 = nu + 0.5 * (w0[j - 1] * NUT(i, j - 1, k) + w1[j - 1] * NUT(i, j, k) +
                                     w0[j - 1] * NUT(i, j - 1, k + 1) + w1[j - 1] * NUT(i, j, k + 1));
          double nu_y2 = nu + 0.5 * (w0[j] * NUT(i, j, k) + w1[j] * NUT(i, j + 1, k) +
                                     w0[j] * NUT(i, j, k + 1) + w1[j] * NUT(i, j + 1, k + 1));
          double nu_z1 = nu + NUT(i, j, k);
          double nu_z2 = nu + NUT(i, j, k + 1);
          double t2p = (AW(W_, i, j + 1, k) - wc) / (yg[j + 1] - yg[j]);
          double t2m = (wc - AW(W_, i, j - 1, k)) / (yg[j] - yg[j - 1]);
          r = r + dPdz +
              (nu_x2 / dx_2 * (AW(W_, i + 1, j, k) - wc) - nu_x1 / dx_1 * (wc - AW(W_, i - 1, j, k))) / dx_3 +
              (nu_y2 * t2p - nu_y1 * t2m) / dy_3 +
              (nu_z2 / dz_2 * (AW(W_, i, j, k + 1) - wc) - nu_z1 / dz_1 * (wc - AW(W_, i, j, k - 1))) / dz_3;
        }
        RW(rhs, i, j, k) = r;
      }
  /* equations.f90:408-413 */
  for (int k = 2; k <= nz - 1; ++k)
    for (int j = 2; j <= nyg - 1; ++j) RW(rhs, nxg - 1, j, k) = 0.0;
}

void blo_rhs_u(blo_t *o, const double *U, const double *V, const double *W, double *r) { rhs_u_impl(o, U, V, W, r); }
void blo_rhs_v(blo_t *o, const double *U, const double *V, const double *W, double *r) { rhs_v_impl(o, U, V, W, r); }
void blo_rhs_w(blo_t *o, const double *U, const double *V, const double *W, double *r) { rhs_w_impl(o, U, V, W, r); }

/* ------------------------------------------------------------------------ */
/* boundary conditions: boundary_conditions.f90:127-262                     */
/* (the CPU routine apply_boundary_conditions, :22-121, takes the same steps */
/*  in the same order for inflow_flag 1/2, top_flag 0 and WM 0)             */
/* ------------------------------------------------------------------------ */
void blo_apply_bc(blo_t *o, int rk_step) {
  const int nx = o->nx, ny = o->ny, nz = o->nz, nxg = o->nxg, nyg = o->nyg, nzg = o->nzg;
  double *U = o->U, *V = o->V, *W = o->W;
  const double *Uo = o->Uo, *Vo = o->Vo, *Wo = o->Wo;
  const double t = o->t, dt = o->dt;
  /* temporal inflow modes (:137-180); a Lund inflow replaces them */
  if (o->n_modes > 0 && o->resc_mode == 0) {
    const int nm_ = o->n_modes, mm_ = o->m_modes;
    for (int j = 1; j <= nyg; ++j)
      for (int k = 1; k <= nzg; ++k) {
        double acc = 0.0;
        for (int n = 0; n < nm_; ++n)
          for (int m = 0; m < mm_; ++m) {
            cplx q = o->qu[((size_t)m * nm_ + n) * nyg + (j - 1)];
            double th = o->zmode[n] * o->zg[k] - o->tmode[m] * t;
            acc = acc + (creal(q) * cos(th) - cimag(q) * sin(th));
          }
        o->Ut[(size_t)(k - 1) * nyg + (j - 1)] = acc;
      }
    for (int j = 1; j <= ny; ++j)
      for (int k = 1; k <= nzg; ++k) {
        double acc = 0.0;
        for (int n = 0; n < nm_; ++n)
          for (int m = 0; m < mm_; ++m) {
            cplx q = o->qv[((size_t)m * nm_ + n) * ny + (j - 1)];
            double th = o->zmode[n] * o->zg[k] - o->tmode[m] * t;
            acc = acc + (creal(q) * cos(th) - cimag(q) * sin(th));
          }
        o->Vt[(size_t)(k - 1) * ny + (j - 1)] = acc;
      }
    for (int j = 1; j <= nyg; ++j)
      for (int k = 1; k <= nz; ++k) {
        double acc = 0.0;
        for (int n = 0; n < nm_; ++n)
          for (int m = 0; m < mm_; ++m) {
            cplx q = o->qw[((size_t)m * nm_ + n) * nyg + (j - 1)];
            double th = o->zmode[n] * o->z[k] - o->tmode[m] * t;
            acc = acc + (creal(q) * cos(th) - cimag(q) * sin(th));
          }
        o->Wt[(size_t)(k - 1) * nyg + (j - 1)] = acc;
      }
  }
  /* inflow plane (:182-190), or the plane of the Lund inflow computed at the
   * start of the step: flag 3 sets the whole plane (:586-594), flag 5 adds
   * the rescaled fluctuations to the inlet profile with W shifted by
   * ks = mod(k+16,nz)+1 (:527-553) */
  if (o->resc_mode == 3) {
    for (int j = 1; j <= nyg; ++j) {
      for (int k = 1; k <= nzg; ++k) AU(U, 1, j, k) = o->Lu[(size_t)(k - 1) * nyg + (j - 1)];
      for (int k = 1; k <= nz; ++k) AW(W, 1, j, k) = o->Lw[(size_t)(k - 1) * nyg + (j - 1)];
    }
    for (int j = 1; j <= ny; ++j)
      for (int k = 1; k <= nzg; ++k) AV(V, 1, j, k) = o->Lv[(size_t)(k - 1) * ny + (j - 1)];
  } else if (o->resc_mode == 5) {
    for (int j = 1; j <= nyg; ++j) {
      for (int k = 1; k <= nzg; ++k) AU(U, 1, j, k) = o->U_inlet[j] + o->Lu[(size_t)(k - 1) * nyg + (j - 1)];
      for (int k = 1; k <= nz; ++k) {
        const int ks = (k + 16) % nz + 1;
        AW(W, 1, j, k) = o->W_inlet[j] + o->Lw[(size_t)(ks - 1) * nyg + (j - 1)];
      }
    }
    for (int j = 1; j <= ny; ++j)
      for (int k = 1; k <= nzg; ++k) AV(V, 1, j, k) = o->V_inlet[j] + o->Lv[(size_t)(k - 1) * ny + (j - 1)];
  } else {
    for (int j = 1; j <= nyg; ++j) {
      for (int k = 1; k <= nzg; ++k) AU(U, 1, j, k) = o->U_inlet[j] + o->Ut[(size_t)(k - 1) * nyg + (j - 1)];
      for (int k = 1; k <= nz; ++k) AW(W, 1, j, k) = o->W_inlet[j] + o->Wt[(size_t)(k - 1) * nyg + (j - 1)];
    }
    for (int j = 1; j <= ny; ++j)
      for (int k = 1; k <= nzg; ++k) AV(V, 1, j, k) = o->V_inlet[j] + o->Vt[(size_t)(k - 1) * ny + (j - 1)];
  }
  /* convective outflow (:193-201) */
  const double Uc = o->U_top[nx];
  const double c = o->rk_t[rk_step] * dt * Uc;
  for (int k = 1; k <= nzg; ++k)
    for (int j = 1; j <= nyg; ++j)
      AU(U, nx - 1, j, k) = AU(Uo, nx - 1, j, k) - c * (AU(Uo, nx - 1, j, k) - AU(Uo, nx - 2, j, k)) / (o->x[nx - 1] - o->x[nx - 2]);
  for (int k = 1; k <= nzg; ++k)
    for (int j = 1; j <= ny; ++j)
      AV(V, nxg - 1, j, k) = AV(Vo, nxg - 1, j, k) - c * (AV(Vo, nxg - 1, j, k) - AV(Vo, nxg - 2, j, k)) / (o->xg[nxg - 1] - o->xg[nxg - 2]);
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= nyg; ++j)
      AW(W, nxg - 1, j, k) = AW(Wo, nxg - 1, j, k) - c * (AW(Wo, nxg - 1, j, k) - AW(Wo, nxg - 2, j, k)) / (o->xg[nxg - 1] - o->xg[nxg - 2]);
  for (int k = 1; k <= nzg; ++k)
    for (int j = 1; j <= nyg; ++j) AU(U, nx, j, k) = AU(U, nx - 1, j, k);
  for (int k = 1; k <= nzg; ++k)
    for (int j = 1; j <= ny; ++j) AV(V, nxg, j, k) = AV(V, nxg - 1, j, k);
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= nyg; ++j) AW(W, nxg, j, k) = AW(W, nxg - 1, j, k);
  /* periodic z (:204-216) */
  {
    size_t pu = (size_t)nx * nyg, pv = (size_t)nxg * ny, pw = (size_t)nxg * nyg;
    memcpy(U, U + (size_t)(nzg - 3) * pu, pu * sizeof(double));
    memcpy(U + (size_t)(nzg - 2) * pu, U + 1 * pu, pu * sizeof(double));
    memcpy(U + (size_t)(nzg - 1) * pu, U + 2 * pu, pu * sizeof(double));
    memcpy(V, V + (size_t)(nzg - 3) * pv, pv * sizeof(double));
    memcpy(V + (size_t)(nzg - 2) * pv, V + 1 * pv, pv * sizeof(double));
    memcpy(V + (size_t)(nzg - 1) * pv, V + 2 * pv, pv * sizeof(double));
    memcpy(W, W + (size_t)(nz - 2) * pw, pw * sizeof(double));
    memcpy(W + (size_t)(nz - 1) * pw, W + 1 * pw, pw * sizeof(double));
  }
  /* top (:219-227) */
  for (int k = 1; k <= nzg; ++k)
    for (int i = 1; i <= nx; ++i) AU(U, i, nyg, k) = o->U_top[i];
  for (int k = 1; k <= nzg; ++k)
    for (int i = 1; i <= nxg; ++i) AV(V, i, ny, k) = o->V_top[i];
  for (int k = 1; k <= nz; ++k)
    for (int i = 1; i <= nxg; ++i) AW(W, i, nyg, k) = o->W_top[i];
  /* wall (:230-237); with a wall model the non-zero Neumann condition of
   * :359-372 on U (and on W for the network), alpha = tau/nu_w at the wall
   * point (i clamped to 2..nx-1, ghost k planes to their periodic image) */
  if (o->wm) {
    const double dy = o->yg[2] - o->yg[1];
    for (int k = 1; k <= nzg; ++k)
      for (int i = 1; i <= nxg; ++i) {
        const int ic = i < 2 ? 2 : (i > nx - 1 ? nx - 1 : i);
        const int kc = k == 1 ? nzg - 2 : (k == nzg - 1 ? 2 : (k == nzg ? 3 : k));
        const size_t q = (size_t)(kc - 2) * (nx - 2) + (ic - 2);
        if (i <= nx) AU(U, i, 1, k) = AU(U, i, 2, k) - o->wm_ax[q] * dy;
        if (k <= nz) AW(W, i, 1, k) = o->wm == 2 ? AW(W, i, 2, k) - o->wm_az[q] * dy : -AW(W, i, 2, k);
      }
  } else {
    for (int k = 1; k <= nzg; ++k)
      for (int i = 1; i <= nx; ++i) AU(U, i, 1, k) = -AU(U, i, 2, k);
    for (int k = 1; k <= nz; ++k)
      for (int i = 1; i <= nxg; ++i) AW(W, i, 1, k) = -AW(W, i, 2, k);
  }
  for (int k = 1; k <= nzg; ++k)
    for (int i = 1; i <= nxg; ++i) AV(V, i, 1, k) = 0.0;
  /* global mass conservation (:240-260), kk = 2 at nprocs = 1 */
  double Qx = 0.0, length_y = 0.0, Qy = 0.0;
  for (int j = 2; j <= nyg - 1; ++j) {
    double s = 0.0;
    for (int k = 2; k <= nzg - 2; ++k) s += (AU(U, 1, j, k) - AU(U, nx - 1, j, k)) * (o->y[j] - o->y[j - 1]);
    Qx = Qx + s;
    length_y = length_y + o->y[j] - o->y[j - 1];
  }
  for (int i = 2; i <= nxg - 2; ++i) {
    double s = 0.0;
    for (int k = 2; k <= nzg - 2; ++k) s += (AV(V, i, 1, k) - AV(V, i, ny, k)) * (o->x[i] - o->x[i - 1]);
    Qy = Qy + s;
  }
  double Q = Qx + Qy;
  double dU = Q / length_y / (double)(nzg - 3);
  for (int k = 1; k <= nzg; ++k)
    for (int j = 1; j <= nyg; ++j) {
      AU(U, nx - 1, j, k) = AU(U, nx - 1, j, k) + dU;
      AU(U, nx, j, k) = AU(U, nx - 1, j, k);
    }
}

/* ------------------------------------------------------------------------ */
/* projection: projection.f90:21-386                                        */
/* ------------------------------------------------------------------------ */

static void poisson_cpu(blo_t *o) {
  /* projection.f90:210-288 */
  const int nxp = o->nxp, nzp = o->nzp, nm = o->nm, nyg = o->nyg;
  const int L = 4 * nxp;
  cplx *hat = o->rhs_hat; /* (0:nxp-1, j=2..nyg-1 -> 0..nm-1, 0:nzp-1) */
#define HAT(i, b, k) hat[((size_t)(k) * nm + (size_t)(b)) * nxp + (size_t)(i)]
#pragma omp parallel
  {
    cplx *plane = (cplx *)malloc(sizeof(cplx) * (size_t)L * nzp);
    size_t wsz = fft_work_size(o->pl_x);
    size_t wz = fft_work_size(o->pl_z);
    cplx *work = (cplx *)malloc(sizeof(cplx) * (wsz > wz ? wsz : wz));
    cplx *col = (cplx *)malloc(sizeof(cplx) * (size_t)nzp);
#pragma omp for schedule(static)
    for (int j = 2; j <= nyg - 1; ++j) {
      memset(plane, 0, sizeof(cplx) * (size_t)L * nzp);
      for (int k = 0; k < nzp; ++k)
        for (int ii = 1; ii <= nxp; ++ii) {
          double f = RP(o->rhs_p, ii + 1, j, k + 2);
          plane[(size_t)k * L + (size_t)(2 * ii - 1)] = f;         /* slot i = 2,4,..,2nxp */
          plane[(size_t)k * L + (size_t)(L - 1 - 2 * (ii - 1))] = f; /* slot i = 4nxp..2nxp+2 */
        }
      /* 2D forward DFT: rows (x) then columns (z) */
      for (int k = 0; k < nzp; ++k) fft_exec(o->pl_x, plane + (size_t)k * L, work);
      for (int i = 0; i < nxp; ++i) {
        for (int k = 0; k < nzp; ++k) col[k] = plane[(size_t)k * L + i];
        fft_exec(o->pl_z, col, work);
        for (int k = 0; k < nzp; ++k) HAT(i, j - 2, k) = col[k];
      }
    }
    /* tridiagonal per mode (:238-256) */
    cplx *D = (cplx *)malloc(sizeof(cplx) * (size_t)nm);
    cplx *DL = (cplx *)malloc(sizeof(cplx) * (size_t)nm);
    cplx *DU = (cplx *)malloc(sizeof(cplx) * (size_t)nm);
    cplx *r = (cplx *)malloc(sizeof(cplx) * (size_t)nm);
#pragma omp for schedule(static)
    for (int k = 0; k < nzp; ++k)
      for (int i = 0; i < nxp; ++i) {
        for (int j = 2; j <= nyg - 1; ++j) D[j - 2] = o->Dd[j] + o->kxx[i] + o->kzz[k];
        for (int j = 2; j <= nyg - 2; ++j) DL[j - 2] = o->Dl[j + 1];
        for (int j = 2; j <= nyg - 2; ++j) DU[j - 2] = o->Du[j];
        if (i == 0 && k == 0) D[0] = 3.0 / 2.0 * D[0];
        for (int b = 0; b < nm; ++b) r[b] = HAT(i, b, k);
        zgtsv_c(nm, DL, D, DU, r);
        for (int b = 0; b < nm; ++b) HAT(i, b, k) = r[b];
      }
    /* inverse (:259-283) */
    const double norm = (double)L * (double)nzp;
#pragma omp for schedule(static)
    for (int j = 2; j <= nyg - 1; ++j) {
      memset(plane, 0, sizeof(cplx) * (size_t)L * nzp);
      const int b = j - 2;
      for (int k = 0; k < nzp; ++k) {
        cplx *row = plane + (size_t)k * L;
        for (int i = 0; i < nxp; ++i) row[i] = HAT(i, b, k);
        for (int s = nxp + 1; s <= 2 * nxp; ++s) row[s] = -HAT(2 * nxp - s, b, k);
        for (int s = 2 * nxp + 1; s <= 3 * nxp - 1; ++s) row[s] = -HAT(s - 2 * nxp, b, k);
        for (int s = 3 * nxp + 1; s <= 4 * nxp - 1; ++s) row[s] = HAT(4 * nxp - s, b, k);
      }
      for (int k = 0; k < nzp; ++k) fft_exec_dir(o->pl_x, plane + (size_t)k * L, work, 1);
      for (int i = 0; i < L; ++i) {
        if ((i & 1) == 0) continue; /* only odd slots are read back */
        for (int k = 0; k < nzp; ++k) col[k] = plane[(size_t)k * L + i];
        fft_exec_dir(o->pl_z, col, work, 1);
        for (int k = 0; k < nzp; ++k) plane[(size_t)k * L + i] = col[k];
      }
      for (int k = 0; k < nzp; ++k)
        for (int ii = 2; ii <= nxp + 1; ++ii)
          RP(o->rhs_p, ii, j, k + 2) = creal(plane[(size_t)k * L + (size_t)(2 * (ii - 1) - 1)]) / norm;
    }
    free(D); free(DL); free(DU); free(r);
    free(plane); free(work); free(col);
  }
#undef HAT
}

static void poisson_gpu_semantics(blo_t *o) {
  /* projection.f90:93-204 (FP64 restatement of the cuFFT path) */
  const int nxp = o->nxp, nzp = o->nzp, nm = o->nm;
  const int L = 2 * nxp;
  cplx *hat = o->rhs_hat; /* rhs_hat_gpu(mx+1, nm, mz+1) */
#define HAT(i, b, k) hat[((size_t)(k) * nm + (size_t)(b)) * nxp + (size_t)(i)]
#define TH(a, i, k, jj) (a)[((size_t)(jj) * nzp + (size_t)(k)) * nxp + (size_t)(i)]
  const double fft_norm = 1.0 / (double)(2 * nxp * nzp);
#pragma omp parallel
  {
    cplx *plane = (cplx *)malloc(sizeof(cplx) * (size_t)L * nzp);
    size_t wsz = fft_work_size(o->pl_x), wz = fft_work_size(o->pl_z);
    cplx *work = (cplx *)malloc(sizeof(cplx) * (wsz > wz ? wsz : wz));
    cplx *col = (cplx *)malloc(sizeof(cplx) * (size_t)nzp);
#pragma omp for schedule(static)
    for (int b = 0; b < nm; ++b) {
      for (int k = 0; k < nzp; ++k)
        for (int ii = 1; ii <= nxp; ++ii) {
          double f = RP(o->rhs_p, ii + 1, b + 2, k + 2);
          plane[(size_t)k * L + (size_t)(ii - 1)] = f;
          plane[(size_t)k * L + (size_t)(L - ii)] = f;
        }
      for (int k = 0; k < nzp; ++k) fft_exec(o->pl_x, plane + (size_t)k * L, work);
      for (int i = 0; i < nxp; ++i) {
        for (int k = 0; k < nzp; ++k) col[k] = plane[(size_t)k * L + i];
        fft_exec(o->pl_z, col, work);
        for (int k = 0; k < nzp; ++k) HAT(i, b, k) = col[k] * o->twid[i];
      }
    }
#pragma omp for schedule(static)
    for (int k = 0; k < nzp; ++k)
      for (int i = 0; i < nxp; ++i) {
        for (int jj = 1; jj < nm; ++jj)
          HAT(i, jj, k) = HAT(i, jj, k) - TH(o->th_dl, i, k, jj - 1) * HAT(i, jj - 1, k);
        HAT(i, nm - 1, k) = HAT(i, nm - 1, k) * TH(o->th_dp, i, k, nm - 1);
        for (int jj = nm - 2; jj >= 0; --jj)
          HAT(i, jj, k) = (HAT(i, jj, k) - o->th_du[jj] * HAT(i, jj + 1, k)) * TH(o->th_dp, i, k, jj);
      }
#pragma omp for schedule(static)
    for (int b = 0; b < nm; ++b) {
      for (int i = 0; i < nxp; ++i) {
        for (int k = 0; k < nzp; ++k) col[k] = HAT(i, b, k);
        fft_exec_dir(o->pl_z, col, work, 1);
        for (int k = 0; k < nzp; ++k) plane[(size_t)k * L + i] = col[k] * conj(o->twid[i]);
      }
      for (int k = 0; k < nzp; ++k) {
        cplx *row = plane + (size_t)k * L;
        row[nxp] = 0;
        for (int ii = 2; ii <= nxp; ++ii) row[L + 1 - ii] = conj(row[ii - 1]);
        fft_exec_dir(o->pl_x, row, work, 1);
        for (int ii = 1; ii <= nxp; ++ii) RP(o->rhs_p, ii + 1, b + 2, k + 2) = creal(row[ii - 1]) * fft_norm;
      }
    }
    free(plane); free(work); free(col);
  }
#undef HAT
#undef TH
}

void blo_projection(blo_t *o, int rk_step) {
  const int nx = o->nx, ny = o->ny, nz = o->nz, nxg = o->nxg, nyg = o->nyg, nzg = o->nzg;
  const double *x = o->x, *y = o->y, *z = o->z, *xg = o->xg, *yg = o->yg, *zg = o->zg;
  double *U = o->U, *V = o->V, *W = o->W;
  /* compute_pseudo_pressure_rhs, projection.f90:38-47 */
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= nzg - 1; ++k)
    for (int j = 2; j <= nyg - 1; ++j)
      for (int i = 2; i <= nxg - 1; ++i)
        RP(o->rhs_p, i, j, k) = (AU(U, i, j, k) - AU(U, i - 1, j, k)) / (x[i] - x[i - 1]) +
                                (AV(V, i, j, k) - AV(V, i, j - 1, k)) / (y[j] - y[j - 1]) +
                                (AW(W, i, j, k) - AW(W, i, j, k - 1)) / (z[k] - z[k - 1]);
  if (o->variant == 0) poisson_cpu(o); else poisson_gpu_semantics(o);
  /* apply_periodic_z_pressure, :295-303 */
  for (int k = 2; k <= nzg; ++k)
    for (int j = 2; j <= nyg - 1; ++j) RP(o->rhs_p, nxg - 1, j, k) = RP(o->rhs_p, nxg - 2, j, k);
  for (int j = 2; j <= nyg - 1; ++j)
    for (int i = 2; i <= nxg - 1; ++i) RP(o->rhs_p, i, j, o->nzp + 2) = RP(o->rhs_p, i, j, 2);
  /* pressure for statistics, :75-85 (P(...,2:nzg-1) = rhs_p(...,2:nzg-1)/(dt/2)) */
  if (rk_step == 1) {
    double *P = o->P;
    const double den = o->dt * o->rk2_coef[0][0];
    for (int k = 2; k <= nzg - 1; ++k)
      for (int j = 2; j <= nyg - 1; ++j)
        for (int i = 2; i <= nxg - 1; ++i) AP(P, i, j, k) = RP(o->rhs_p, i, j, k) / den;
    for (int k = 1; k <= nzg; ++k)
      for (int j = 1; j <= nyg; ++j) { AP(P, 1, j, k) = AP(P, 2, j, k); }
    for (int k = 1; k <= nzg; ++k)
      for (int j = 1; j <= nyg; ++j) { AP(P, nxg, j, k) = AP(P, nxg - 1, j, k); }
    for (int k = 1; k <= nzg; ++k)
      for (int i = 1; i <= nxg; ++i) { AP(P, i, 1, k) = AP(P, i, 2, k); }
    for (int k = 1; k <= nzg; ++k)
      for (int i = 1; i <= nxg; ++i) { AP(P, i, nyg, k) = AP(P, i, nyg - 1, k); }
    size_t pp = (size_t)nxg * nyg;
    memcpy(P, P + pp, pp * sizeof(double));
    memcpy(P + (size_t)(nzg - 1) * pp, P + (size_t)(nzg - 2) * pp, pp * sizeof(double));
  }
  /* project_velocity, :359-384 */
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= nzg - 1; ++k)
    for (int j = 2; j <= nyg - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i)
        AU(U, i, j, k) = AU(U, i, j, k) - (RP(o->rhs_p, i + 1, j, k) - RP(o->rhs_p, i, j, k)) / (xg[i + 1] - xg[i]);
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= nzg - 1; ++k)
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nxg - 1; ++i)
        AV(V, i, j, k) = AV(V, i, j, k) - (RP(o->rhs_p, i, j + 1, k) - RP(o->rhs_p, i, j, k)) / (yg[j + 1] - yg[j]);
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= nz - 1; ++k)
    for (int j = 2; j <= nyg - 1; ++j)
      for (int i = 2; i <= nxg - 1; ++i)
        AW(W, i, j, k) = AW(W, i, j, k) - (RP(o->rhs_p, i, j, k + 1) - RP(o->rhs_p, i, j, k)) / (zg[k + 1] - zg[k]);
}

void blo_get_rhs_p(const blo_t *o, double *rhs_p) {
  memcpy(rhs_p, o->rhs_p, sizeof(double) * (size_t)(o->nxg - 2) * (o->nyg - 2) * (o->nzg - 1));
}

/* check_divergence, projection.f90:391-413 */
double blo_max_divergence(const blo_t *o) {
  const double *U = o->U, *V = o->V, *W = o->W;
  double div = 0.0;
  for (int k = 2; k <= o->nzg - 1; ++k)
    for (int j = 2; j <= o->nyg - 1; ++j)
      for (int i = 2; i <= o->nxg - 2; ++i) {
        double d = fabs((AU(U, i, j, k) - AU(U, i - 1, j, k)) / (o->x[i] - o->x[i - 1]) +
                        (AV(V, i, j, k) - AV(V, i, j - 1, k)) / (o->y[j] - o->y[j - 1]) +
                        (AW(W, i, j, k) - AW(W, i, j, k - 1)) / (o->z[k] - o->z[k - 1]));
        if (d > div) div = d;
      }
  return div;
}

/* compute_dt, time_integration.f90:528-591 (note the max, as written) */
double blo_compute_dt(blo_t *o) {
  const double CFLa = fabs(o->cfl);
  if (o->cfl < 0) {
    o->dt = -o->cfl;
    return o->dt;
  }
  double lU = 0.0, lV = 0.0, lW = 0.0;
  for (int i = 2; i <= o->nxg - 1; ++i)
    for (int j = 2; j <= o->nyg - 1; ++j)
      for (int k = 2; k <= o->nzg - 1; ++k) {
        double a = (o->xg[i + 1] - o->xg[i]) / fabs(AU(o->U, i, j, k));
        double b = (o->yg[j + 1] - o->yg[j]) / fabs(AV(o->V, i, j, k));
        double c = (o->zg[k + 1] - o->zg[k]) / fabs(AW(o->W, i, j, k));
        lU = fmax(lU, a);
        lV = fmax(lV, b);
        lW = fmax(lW, c);
      }
  double cu = CFLa * lU, cv = CFLa * lV, cw = CFLa * lW;
  double dt_conv = fmin(fmin(cu, cv), cw);
  double vu = CFLa * (o->dxmin * o->dxmin) / o->nu;
  double vv = CFLa * (o->dymin * o->dymin) / o->nu;
  double vw = CFLa * (o->dzmin * o->dzmin) / o->nu;
  double dt_vis = fmin(fmin(vu, vv), vw);
  o->dt = fmin(dt_conv, dt_vis);
  return o->dt;
}

/* ------------------------------------------------------------------------ */
/* time stepping: time_integration.f90:24-114 (Euler), 145-300 (RK2),       */
/* 305-465 (RK3)                                                            */
/* ------------------------------------------------------------------------ */

static void save_state(blo_t *o) {
  size_t su = (size_t)o->nx * o->nyg * o->nzg, sv = (size_t)o->nxg * o->ny * o->nzg,
         sw = (size_t)o->nxg * o->nyg * o->nz;
  memcpy(o->Uo, o->U, su * sizeof(double));
  memcpy(o->Vo, o->V, sv * sizeof(double));
  memcpy(o->Wo, o->W, sw * sizeof(double));
}

/* U = Uo + dt*(sum_j a_j F_j), with the reference's association order */
static void rk_update(blo_t *o, int nterms, const double *a) {
  const double dt = o->dt;
  const int nx = o->nx, ny = o->ny, nz = o->nz, nxg = o->nxg, nyg = o->nyg, nzg = o->nzg;
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= nzg - 1; ++k)
    for (int j = 2; j <= nyg - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i) {
        double s;
        if (nterms == 1) s = dt * a[0] * RU(o->Fu[0], i, j, k);
        else if (nterms == 2) s = dt * (a[0] * RU(o->Fu[0], i, j, k) + a[1] * RU(o->Fu[1], i, j, k));
        else s = dt * (a[0] * RU(o->Fu[0], i, j, k) + a[1] * RU(o->Fu[1], i, j, k) + a[2] * RU(o->Fu[2], i, j, k));
        AU(o->U, i, j, k) = AU(o->Uo, i, j, k) + s;
      }
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= nzg - 1; ++k)
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nxg - 1; ++i) {
        double s;
        if (nterms == 1) s = dt * a[0] * RV(o->Fv[0], i, j, k);
        else if (nterms == 2) s = dt * (a[0] * RV(o->Fv[0], i, j, k) + a[1] * RV(o->Fv[1], i, j, k));
        else s = dt * (a[0] * RV(o->Fv[0], i, j, k) + a[1] * RV(o->Fv[1], i, j, k) + a[2] * RV(o->Fv[2], i, j, k));
        AV(o->V, i, j, k) = AV(o->Vo, i, j, k) + s;
      }
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= nz - 1; ++k)
    for (int j = 2; j <= nyg - 1; ++j)
      for (int i = 2; i <= nxg - 1; ++i) {
        double s;
        if (nterms == 1) s = dt * a[0] * RW(o->Fw[0], i, j, k);
        else if (nterms == 2) s = dt * (a[0] * RW(o->Fw[0], i, j, k) + a[1] * RW(o->Fw[1], i, j, k));
        else s = dt * (a[0] * RW(o->Fw[0], i, j, k) + a[1] * RW(o->Fw[1], i, j, k) + a[2] * RW(o->Fw[2], i, j, k));
        AW(o->W, i, j, k) = AW(o->Wo, i, j, k) + s;
      }
}


/* ------------------------------------------------------------------------ */
/* Lund recycling/rescaling inflow: rescaled_inlet_bc.f90:60-345           */
/* ------------------------------------------------------------------------ */

/* interp_vel (rescaled_inlet_bc.f90:305-345): for each target row i = 2..n1,
 * the first source row j with ys(j) > yi(i) selects the pair (j-1, j); none
 * selects the top row n1; j == 1 is the reference's stop (flagged here).
 * src(n1, ncol) and dst(n1, ncol) are column-major; ys, yi are 1-based.
 * Row 1 is never written by the reference (its value is undefined there and
 * the wall condition overwrites the inflow cells it feeds); it is 0 here. */
static void lund_interp(const double *src, int n1, int ncol, const double *ys, const double *yi,
                        double *dst, int *err) {
  for (int c = 0; c < ncol; ++c) dst[(size_t)c * n1] = 0.0;
  for (int i = 2; i <= n1; ++i) {
    int j = 0;
    for (int k = 1; k <= n1; ++k)
      if (ys[k] > yi[i]) { j = k; break; }
    if (j == 1) { *err = 1; j = 0; }
    if (j > 0) {
      const double coef = (ys[j] - yi[i]) / (ys[j] - ys[j - 1]);
      for (int c = 0; c < ncol; ++c)
        dst[(size_t)c * n1 + (i - 1)] = coef * src[(size_t)c * n1 + (j - 2)] + (1.0 - coef) * src[(size_t)c * n1 + (j - 1)];
    } else {
      for (int c = 0; c < ncol; ++c) dst[(size_t)c * n1 + (i - 1)] = src[(size_t)c * n1 + (n1 - 1)];
    }
  }
}

/* delta_99 by linear interpolation of a mean profile (:148-182) */
static double lund_delta99(const blo_t *o, const double *Um, double Umean99) {
  int jref = 0;
  for (int j = 1; j <= o->nyg; ++j)
    if (Um[j] >= Umean99) { jref = j; break; }
  if (jref < 2) jref = o->nyg / 2;
  const double w1 = (Umean99 - Um[jref - 1]) / (Um[jref] - Um[jref - 1]);
  const double w0 = 1.0 - w1;
  double d = w1 * o->yg[jref] + w0 * o->yg[jref - 1];
  return d < 0 ? fabs(d) : d;
}

/* momentum thickness by the trapezoidal rule over the centres (:188-210) */
static double lund_theta(const blo_t *o, const double *Um, double Uinf) {
  double th = 0.0;
  for (int j = 2; j <= o->nyg; ++j) {
    const double a = Um[j] / Uinf * (1.0 - Um[j] / Uinf), b = Um[j - 1] / Uinf * (1.0 - Um[j - 1] / Uinf);
    th = th + 0.5 * (a + b) * (o->yg[j] - o->yg[j - 1]);
  }
  return th < 0 ? fabs(th) : th;
}

/* compute_rescaled_inflow (:60-300) from the fields U_,V_,W_ (the step's
 * Uo, Vo, Wo); fluc = iflag_fluc.  Updates the running means and writes the
 * planes Lu(nyg,nzg), Lv(ny,nzg), Lw(nyg,nz). */
static void lund_inflow(blo_t *o, const double *U_, const double *V_, const double *W_, int fluc) {
  const int ny = o->ny, nyg = o->nyg, nz = o->nz, nzg = o->nzg, ir = o->i_rescale;
  const double nu = o->nu;
  double *Ur = dalloc((size_t)nyg * nzg), *Vr = dalloc((size_t)ny * nzg), *Wr = dalloc((size_t)nyg * nz);
  for (int k = 1; k <= nzg; ++k)
    for (int j = 1; j <= nyg; ++j) Ur[(size_t)(k - 1) * nyg + (j - 1)] = AU(U_, ir, j, k);
  for (int k = 1; k <= nzg; ++k)
    for (int j = 1; j <= ny; ++j) Vr[(size_t)(k - 1) * ny + (j - 1)] = AV(V_, ir, j, k);
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= nyg; ++j) Wr[(size_t)(k - 1) * nyg + (j - 1)] = AW(W_, ir, j, k);
  /* instantaneous z-means (:109-125) and their running averages (:133-137) */
  double *Umr_i = dalloc(nyg + 1), *Vmr_i = dalloc(ny + 1), *Umi_i = dalloc(nyg + 1), *Vmi_i = dalloc(ny + 1);
  const double dn = (double)(nzg - 2);
  for (int j = 1; j <= nyg; ++j) {
    double a = 0.0, b = 0.0;
    for (int k = 2; k <= nzg - 1; ++k) { a += AU(U_, ir, j, k); b += AU(U_, 1, j, k); }
    Umr_i[j] = a / dn;
    Umi_i[j] = b / dn;
  }
  for (int j = 1; j <= ny; ++j) {
    double a = 0.0, b = 0.0;
    for (int k = 2; k <= nzg - 1; ++k) { a += AV(V_, ir, j, k); b += AV(V_, 1, j, k); }
    Vmr_i[j] = a / dn;
    Vmi_i[j] = b / dn;
  }
  const double Uinf = Umr_i[nyg];
  const double ra = o->dt / o->T_resc, rb = 1.0 - o->dt / o->T_resc;
  for (int j = 1; j <= nyg; ++j) {
    o->Umr[j] = ra * Umr_i[j] + rb * o->Umr[j];
    o->Umi[j] = ra * Umi_i[j] + rb * o->Umi[j];
  }
  for (int j = 1; j <= ny; ++j) {
    o->Vmr[j] = ra * Vmr_i[j] + rb * o->Vmr[j];
    o->Vmi[j] = ra * Vmi_i[j] + rb * o->Vmi[j];
  }
  /* fluctuations at the recycling station (:141-150; the inlet ones are unused) */
  for (int k = 1; k <= nzg; ++k)
    for (int j = 1; j <= nyg; ++j) Ur[(size_t)(k - 1) * nyg + (j - 1)] -= o->Umr[j];
  for (int k = 1; k <= nzg; ++k)
    for (int j = 1; j <= ny; ++j) Vr[(size_t)(k - 1) * ny + (j - 1)] -= o->Vmr[j];
  /* thicknesses (:153-210) */
  const double Umean99 = 0.99 * Uinf;
  const double delta_resc = lund_delta99(o, o->Umr, Umean99);
  const double delta_inlet2 = lund_delta99(o, o->Umi, Umean99);
  const double theta_resc = lund_theta(o, o->Umr, Uinf), theta_inlet = lund_theta(o, o->Umi, Uinf);
  /* friction velocities (:214-231); the wall product uses the plane before
   * the mean is removed */
  double uv = 0.0;
  for (int k = 2; k <= nzg - 1; ++k)
    uv += 0.5 * (AU(U_, ir, 1, k) + AU(U_, ir, 2, k)) * AV(V_, ir, 1, k);
  uv = uv / dn;
  const double dUw = (o->Umr[2] - o->Umr[1]) / (o->yg[2] - o->yg[1]);
  const double utau_resc = sqrt(fabs(nu * dUw - uv));
  const double utau_inlet = utau_resc * pow(theta_resc / theta_inlet, 1.0 / 8.0);
  const double gamma = utau_inlet / utau_resc;
  /* inner (wall units) and outer (delta_99 units) coordinates (:235-246) */
  double *ygp_i = dalloc(nyg + 1), *ygp_r = dalloc(nyg + 1), *etg_i = dalloc(nyg + 1), *etg_r = dalloc(nyg + 1);
  double *yp_i = dalloc(ny + 1), *yp_r = dalloc(ny + 1), *et_i = dalloc(ny + 1), *et_r = dalloc(ny + 1);
  double *Weig = dalloc(nyg + 1), *Wei = dalloc(ny + 1);
  const double alpha = 4.0, bb = 0.2;
  for (int j = 1; j <= nyg; ++j) {
    ygp_i[j] = utau_inlet * o->yg[j] / nu;
    ygp_r[j] = utau_resc * o->yg[j] / nu;
    etg_i[j] = o->yg[j] / o->delta_inlet;
    etg_r[j] = o->yg[j] / delta_resc;
    Weig[j] = 0.5 * (1.0 + tanh(alpha * (etg_i[j] - bb) / ((1.0 - 2.0 * bb) * etg_i[j] + bb)) / tanh(alpha));
  }
  for (int j = 1; j <= ny; ++j) {
    yp_i[j] = utau_inlet * o->y[j] / nu;
    yp_r[j] = utau_resc * o->y[j] / nu;
    et_i[j] = o->y[j] / o->delta_inlet;
    et_r[j] = o->y[j] / delta_resc;
    Wei[j] = 0.5 * (1.0 + tanh(alpha * (et_i[j] - bb) / ((1.0 - 2.0 * bb) * et_i[j] + bb)) / tanh(alpha));
  }
  /* inner and outer components (:255-283) */
  int err = 0;
  double *Umi_n = dalloc(nyg), *Umo_n = dalloc(nyg), *Vmi_n = dalloc(ny), *Vmo_n = dalloc(ny);
  lund_interp(o->Umr + 1, nyg, 1, ygp_r, ygp_i, Umi_n, &err);
  lund_interp(o->Umr + 1, nyg, 1, etg_r, etg_i, Umo_n, &err);
  lund_interp(o->Vmr + 1, ny, 1, yp_r, yp_i, Vmi_n, &err);
  lund_interp(o->Vmr + 1, ny, 1, et_r, et_i, Vmo_n, &err);
  for (int j = 0; j < nyg; ++j) {
    Umi_n[j] = gamma * Umi_n[j];
    Umo_n[j] = gamma * Umo_n[j] + (1.0 - gamma) * Uinf;
  }
  double *Ufi = dalloc((size_t)nyg * nzg), *Ufo = dalloc((size_t)nyg * nzg);
  double *Vfi = dalloc((size_t)ny * nzg), *Vfo = dalloc((size_t)ny * nzg);
  double *Wfi = dalloc((size_t)nyg * nz), *Wfo = dalloc((size_t)nyg * nz);
  lund_interp(Ur, nyg, nzg, ygp_r, ygp_i, Ufi, &err);
  lund_interp(Ur, nyg, nzg, etg_r, etg_i, Ufo, &err);
  lund_interp(Vr, ny, nzg, yp_r, yp_i, Vfi, &err);
  lund_interp(Vr, ny, nzg, et_r, et_i, Vfo, &err);
  lund_interp(Wr, nyg, nz, ygp_r, ygp_i, Wfi, &err);
  lund_interp(Wr, nyg, nz, etg_r, etg_i, Wfo, &err);
  if (fluc) {
    for (int j = 0; j < nyg; ++j) Umi_n[j] = Umo_n[j] = 0.0;
    for (int j = 0; j < ny; ++j) Vmi_n[j] = Vmo_n[j] = 0.0;
  }
  /* blend (:287-298) */
  for (int k = 1; k <= nzg; ++k)
    for (int j = 1; j <= nyg; ++j) {
      const size_t q = (size_t)(k - 1) * nyg + (j - 1);
      o->Lu[q] = (Umi_n[j - 1] + gamma * Ufi[q]) * (1.0 - Weig[j]) + (Umo_n[j - 1] + gamma * Ufo[q]) * Weig[j];
    }
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= nyg; ++j) {
      const size_t q = (size_t)(k - 1) * nyg + (j - 1);
      o->Lw[q] = (gamma * Wfi[q]) * (1.0 - Weig[j]) + (gamma * Wfo[q]) * Weig[j];
    }
  for (int k = 1; k <= nzg; ++k)
    for (int j = 1; j <= ny; ++j) {
      const size_t q = (size_t)(k - 1) * ny + (j - 1);
      o->Lv[q] = (Vmi_n[j - 1] + gamma * Vfi[q]) * (1.0 - Wei[j]) + (Vmo_n[j - 1] + gamma * Vfo[q]) * Wei[j];
    }
  o->lund_err |= err;
  double dg[8] = {Uinf, delta_resc, delta_inlet2, theta_resc, theta_inlet, utau_resc, utau_inlet, gamma};
  memcpy(o->lund_diag, dg, sizeof(dg));
  double *fr[] = {Ur, Vr, Wr, Umr_i, Vmr_i, Umi_i, Vmi_i, ygp_i, ygp_r, etg_i, etg_r, yp_i, yp_r, et_i, et_r,
                  Weig, Wei, Umi_n, Umo_n, Vmi_n, Vmo_n, Ufi, Ufo, Vfi, Vfo, Wfi, Wfo};
  for (size_t q = 0; q < sizeof(fr) / sizeof(fr[0]); ++q) free(fr[q]);
}

/* running means at start-up (initialization.f90:636-664): taken from the
 * restart file's means when their sum exceeds 1e-4, else from the field */
int blo_set_rescaling(blo_t *o, int mode, int i_rescale, double delta_inlet, double T_resc,
                      const double *Umean0, const double *Vmean0) {
  if (mode != 0 && mode != 3 && mode != 5) return -1;
  if (mode != 0 && (i_rescale < 2 || i_rescale > o->nx)) return -2;
  o->resc_mode = mode;
  o->i_rescale = i_rescale;
  o->delta_inlet = delta_inlet;
  o->T_resc = T_resc;
  o->lund_err = 0;
  if (!mode) return 0;
  const double dn = (double)(o->nzg - 2);
  double s0 = 0.0;
  if (Umean0)
    for (int j = 0; j < o->nyg; ++j) s0 += Umean0[j];
  for (int j = 1; j <= o->nyg; ++j) {
    double a = 0.0, b = 0.0;
    for (int k = 2; k <= o->nzg - 1; ++k) { a += AU(o->U, i_rescale, j, k); b += AU(o->U, 1, j, k); }
    o->Umr[j] = (Umean0 && s0 > 1e-4) ? Umean0[j - 1] : a / dn;
    o->Umi[j] = b / dn;
  }
  for (int j = 1; j <= o->ny; ++j) {
    double a = 0.0, b = 0.0;
    for (int k = 2; k <= o->nzg - 1; ++k) { a += AV(o->V, i_rescale, j, k); b += AV(o->V, 1, j, k); }
    o->Vmr[j] = (Umean0 && s0 > 1e-4) ? (Vmean0 ? Vmean0[j - 1] : 0.0) : a / dn;
    o->Vmi[j] = b / dn;
  }
  return 0;
}

/* one evaluation from the current state (the test hook of the step-start call) */
void blo_rescaled_inflow(blo_t *o) {
  if (o->resc_mode) lund_inflow(o, o->U, o->V, o->W, o->resc_mode == 5);
}

void blo_get_rescaling(const blo_t *o, double *Umean_resc, double *Vmean_resc, double *Umean_inlet,
                       double *Vmean_inlet, double *Lu, double *Lv, double *Lw, double *diag, int *err) {
  if (Umean_resc) memcpy(Umean_resc, o->Umr + 1, sizeof(double) * o->nyg);
  if (Vmean_resc) memcpy(Vmean_resc, o->Vmr + 1, sizeof(double) * o->ny);
  if (Umean_inlet) memcpy(Umean_inlet, o->Umi + 1, sizeof(double) * o->nyg);
  if (Vmean_inlet) memcpy(Vmean_inlet, o->Vmi + 1, sizeof(double) * o->ny);
  if (Lu) memcpy(Lu, o->Lu, sizeof(double) * (size_t)o->nyg * o->nzg);
  if (Lv) memcpy(Lv, o->Lv, sizeof(double) * (size_t)o->ny * o->nzg);
  if (Lw) memcpy(Lw, o->Lw, sizeof(double) * (size_t)o->nyg * o->nz);
  if (diag) memcpy(diag, o->lund_diag, sizeof(o->lund_diag));
  if (err) *err = o->lund_err;
}

void blo_smagorinsky(blo_t *o);
void blo_dynamic_smagorinsky(blo_t *o);
static void wall_model_eval(blo_t *o);
static void substep(blo_t *o, int s, int rk_step, const double *coef, int nterms,
                    double tnew) {
  o->rk_step = rk_step;
  if (o->les == 1) blo_smagorinsky(o); /* time_integration.f90:341-346 */
  else if (o->les >= 2) blo_dynamic_smagorinsky(o);
  if (o->wm) wall_model_eval(o);
  rhs_u_impl(o, o->U, o->V, o->W, o->Fu[s]);
  rhs_v_impl(o, o->U, o->V, o->W, o->Fv[s]);
  rhs_w_impl(o, o->U, o->V, o->W, o->Fw[s]);
  rk_update(o, nterms, coef);
  o->t = tnew;
  blo_apply_bc(o, rk_step);
  blo_projection(o, rk_step);
  blo_apply_bc(o, rk_step);
}

void blo_step(blo_t *o) {
  const double to = o->t, dt = o->dt;
  save_state(o);
  /* Lund inflow once per step from Uo (boundary_conditions.f90:569-597) */
  if (o->resc_mode) lund_inflow(o, o->Uo, o->Vo, o->Wo, o->resc_mode == 5);
  if (o->rk_scheme == 3) {
    double a1[1] = {o->rk_coef[0][0]};
    substep(o, 0, 1, a1, 1, to + o->rk_t[1] * dt);
    double a2[2] = {o->rk_coef[1][0], o->rk_coef[1][1]};
    substep(o, 1, 2, a2, 2, to + o->rk_t[2] * dt);
    double a3[3] = {o->rk_coef[2][0], o->rk_coef[2][1], o->rk_coef[2][2]};
    substep(o, 2, 3, a3, 3, to + o->rk_t[3] * dt);
  } else if (o->rk_scheme == 2) {
    double a1[1] = {o->rk2_coef[0][0]};
    substep(o, 0, 1, a1, 1, to + o->rk2_t[1] * dt);
    double a2[2] = {o->rk2_coef[1][0], o->rk2_coef[1][1]};
    substep(o, 1, 2, a2, 2, to + o->rk2_t[2] * dt);
  } else {
    /* Euler: U = Uo + dt*rhs(Uo); rk_step = 3 (time_integration.f90:24-114) */
    o->rk_step = 3;
    if (o->les == 1) blo_smagorinsky(o);
    else if (o->les >= 2) blo_dynamic_smagorinsky(o);
    if (o->wm) wall_model_eval(o);
    rhs_u_impl(o, o->Uo, o->Vo, o->Wo, o->Fu[0]);
    rhs_v_impl(o, o->Uo, o->Vo, o->Wo, o->Fv[0]);
    rhs_w_impl(o, o->Uo, o->Vo, o->Wo, o->Fw[0]);
    /* U = Uo + dt*rhs, evaluated as Uo + (dt*rhs) */
    const int nx = o->nx, ny = o->ny, nz = o->nz, nxg = o->nxg, nyg = o->nyg, nzg = o->nzg;
    for (int k = 2; k <= nzg - 1; ++k)
      for (int j = 2; j <= nyg - 1; ++j)
        for (int i = 2; i <= nx - 1; ++i) AU(o->U, i, j, k) = AU(o->Uo, i, j, k) + dt * RU(o->Fu[0], i, j, k);
    for (int k = 2; k <= nzg - 1; ++k)
      for (int j = 2; j <= ny - 1; ++j)
        for (int i = 2; i <= nxg - 1; ++i) AV(o->V, i, j, k) = AV(o->Vo, i, j, k) + dt * RV(o->Fv[0], i, j, k);
    for (int k = 2; k <= nz - 1; ++k)
      for (int j = 2; j <= nyg - 1; ++j)
        for (int i = 2; i <= nxg - 1; ++i) AW(o->W, i, j, k) = AW(o->Wo, i, j, k) + dt * RW(o->Fw[0], i, j, k);
    o->t = to + dt;
    blo_apply_bc(o, 3);
    blo_projection(o, 3);
    blo_apply_bc(o, 3);
  }
}

/* one RK3 substep (stage 1..3) of compute_time_step_RK3; stage 1 saves the
 * state and the start time first (time_integration.f90:305-463) */
static double stage_to = 0.0;
void blo_rk3_stage(blo_t *o, int stage) {
  if (stage == 1) {
    stage_to = o->t;
    save_state(o);
    if (o->resc_mode) lund_inflow(o, o->Uo, o->Vo, o->Wo, o->resc_mode == 5);
    double a1[1] = {o->rk_coef[0][0]};
    substep(o, 0, 1, a1, 1, stage_to + o->rk_t[1] * o->dt);
  } else if (stage == 2) {
    double a2[2] = {o->rk_coef[1][0], o->rk_coef[1][1]};
    substep(o, 1, 2, a2, 2, stage_to + o->rk_t[2] * o->dt);
  } else {
    double a3[3] = {o->rk_coef[2][0], o->rk_coef[2][1], o->rk_coef[2][2]};
    substep(o, 2, 3, a3, 3, stage_to + o->rk_t[3] * o->dt);
  }
}

/* ------------------------------------------------------------------------ */
/* constant-coefficient Smagorinsky: subgrid.f90:609-662 (sgs_Smagorinsky)  */
/* with compute_Sij, :672-730.  Dirichlet_nu_t is forced to 0               */
/* (initialization.f90:586), so the damping f = 1.  nu_t is written on the  */
/* interior i=2..nxg-1, j=2..nyg-1, k=2..nzg-1; ghosts keep their values.   */
/* ------------------------------------------------------------------------ */
static double sij_edge4(const blo_t *o, const double *U_, const double *V_, int i, int j, int k) {
  return 0.5 * ((AU(U_, i - 1, j, k) - AU(U_, i - 1, j - 1, k)) / (o->yg[j] - o->yg[j - 1]) +
                (AV(V_, i, j - 1, k) - AV(V_, i - 1, j - 1, k)) / (o->xg[i] - o->xg[i - 1]));
}
static double sij_edge5(const blo_t *o, const double *U_, const double *W_, int i, int j, int k) {
  return 0.5 * ((AU(U_, i - 1, j, k) - AU(U_, i - 1, j, k - 1)) / (o->zg[k] - o->zg[k - 1]) +
                (AW(W_, i, j, k - 1) - AW(W_, i - 1, j, k - 1)) / (o->xg[i] - o->xg[i - 1]));
}
static double sij_edge6(const blo_t *o, const double *V_, const double *W_, int i, int j, int k) {
  return 0.5 * ((AV(V_, i, j - 1, k) - AV(V_, i, j - 1, k - 1)) / (o->zg[k] - o->zg[k - 1]) +
                (AW(W_, i, j, k - 1) - AW(W_, i, j - 1, k - 1)) / (o->yg[j] - o->yg[j - 1]));
}

void blo_smagorinsky(blo_t *o) {
  const double Cs = 0.11, f = 1.0;
  const double *U = o->U, *V = o->V, *W = o->W;
  for (int j = 2; j <= o->nyg - 1; ++j) {
    const double Delta = pow(o->dx * o->dz * (o->y[j] - o->y[j - 1]), 1.0 / 3.0);
    const double c2 = (Cs * Delta * f) * (Cs * Delta * f);
    for (int k = 2; k <= o->nzg - 1; ++k)
      for (int i = 2; i <= o->nxg - 1; ++i) {
        double s1 = (AU(U, i, j, k) - AU(U, i - 1, j, k)) / (o->x[i] - o->x[i - 1]);
        double s2 = (AV(V, i, j, k) - AV(V, i, j - 1, k)) / (o->y[j] - o->y[j - 1]);
        double s3 = (AW(W, i, j, k) - AW(W, i, j, k - 1)) / (o->z[k] - o->z[k - 1]);
        double s4 = 0.25 * (sij_edge4(o, U, V, i, j, k) + sij_edge4(o, U, V, i + 1, j, k) +
                            sij_edge4(o, U, V, i, j + 1, k) + sij_edge4(o, U, V, i + 1, j + 1, k));
        double s5 = 0.25 * (sij_edge5(o, U, W, i, j, k) + sij_edge5(o, U, W, i + 1, j, k) +
                            sij_edge5(o, U, W, i, j, k + 1) + sij_edge5(o, U, W, i + 1, j, k + 1));
        double s6 = 0.25 * (sij_edge6(o, V, W, i, j, k) + sij_edge6(o, V, W, i, j + 1, k) +
                            sij_edge6(o, V, W, i, j, k + 1) + sij_edge6(o, V, W, i, j + 1, k + 1));
        double S = 0.0;
        S = S + 2.0 * s1 * s1;
        S = S + 2.0 * s2 * s2;
        S = S + 2.0 * s3 * s3;
        S = S + 4.0 * s4 * s4;
        S = S + 4.0 * s5 * s5;
        S = S + 4.0 * s6 * s6;
        S = sqrt(S);
        NUT(i, j, k) = c2 * S;
      }
  }
}

/* ------------------------------------------------------------------------ */
/* dynamic Smagorinsky, subgrid.f90:261-583: sgs_dynamic_Smagorinsky (LES=2, */
/* z-averaged coefficient) and _noaverage (LES=3), with the filters of      */
/* :69-184 (filter_xzy, fil_size = 2), compute_Sij (:672-730), the          */
/* interpolations of interpolation.f90:24-114 and the x / z helpers of      */
/* boundary_conditions.f90:295-344,732-888 for one process (the interior-    */
/* plane exchange is then empty).  Every work array is a dense              */
/* (nxg,nyg,nzg) array indexed 1-based like its Fortran counterpart (the    */
/* velocity-shaped ones use the AU / AV / AW shapes); entries the source    */
/* never sets stay zero here and never reach the output.                     */
/* ------------------------------------------------------------------------ */
#define AG(a, i, j, k) (a)[IX3(i, j, k, o->nxg, o->nyg)]

/* apply_Neumann_bc_x / apply_periodic_bc_x (:295-344) on a dense array of first dimension d1 */
static void dyn_bc_x(const blo_t *o, double *a, int d1, int d2, int d3, int id, int periodic) {
  for (int k = 1; k <= d3; ++k)
    for (int j = 1; j <= d2; ++j) {
      double *r = a + IX3(1, j, k, d1, d2);
      if (!periodic) {
        if (id == 1) { r[0] = r[1]; r[o->nx - 1] = r[o->nx - 2]; }
        else { r[0] = r[1]; r[o->nxg - 1] = r[o->nxg - 2]; }
      } else {
        if (id == 1) { r[0] = r[o->nx - 2]; r[o->nx - 1] = r[1]; }
        else { r[0] = r[o->nxg - 3]; r[o->nxg - 2] = r[1]; r[o->nxg - 1] = r[2]; }
      }
    }
}
/* apply_periodic_bc_z (:732-760, one process) */
static void dyn_bc_z(const blo_t *o, double *a, int d1, int d2, int id) {
  const size_t pl = (size_t)d1 * d2;
  if (id == 3) {
    memcpy(a, a + (size_t)(o->nz - 2) * pl, pl * sizeof(double));
    memcpy(a + (size_t)(o->nz - 1) * pl, a + pl, pl * sizeof(double));
  } else {
    memcpy(a, a + (size_t)(o->nzg - 3) * pl, pl * sizeof(double));
    memcpy(a + (size_t)(o->nzg - 2) * pl, a + pl, pl * sizeof(double));
    memcpy(a + (size_t)(o->nzg - 1) * pl, a + 2 * pl, pl * sizeof(double));
  }
}
/* filter_xzy (:140-184) of the section a(1:n1, ja:jb, 1:n3) of a dense array
 * of dims (d1,d2,*): g(i,j,k), i = 2..n1-1, j = ja..jb, k = 2..n3-1 (the
 * section's own indices, which are the output's in every call of the model) */
static void dyn_filter(const double *a, int d1, int d2, int n1, int ja, int jb, int n3, double *g, int e1, int e2) {
  static const double fil[3][3] = {{1.0 / 36.0, 1.0 / 9.0, 1.0 / 36.0},
                                   {1.0 / 9.0, 4.0 / 9.0, 1.0 / 9.0},
                                   {1.0 / 36.0, 1.0 / 9.0, 1.0 / 36.0}};
  for (int k = 2; k <= n3 - 1; ++k)
    for (int j = ja; j <= jb; ++j)
      for (int i = 2; i <= n1 - 1; ++i) {
        double s = 0.0;
        for (int di = -1; di <= 1; ++di)
          for (int dk = -1; dk <= 1; ++dk) {
            const int ii = i + di, kk = k + dk;
            double y;
            if (j == ja)
              y = 2.0 / 3.0 * a[IX3(ii, j, kk, d1, d2)] + 1.0 / 3.0 * a[IX3(ii, j + 1, kk, d1, d2)];
            else if (j == jb)
              y = 1.0 / 3.0 * a[IX3(ii, j - 1, kk, d1, d2)] + 2.0 / 3.0 * a[IX3(ii, j, kk, d1, d2)];
            else
              y = 1.0 / 6.0 * a[IX3(ii, j - 1, kk, d1, d2)] + 2.0 / 3.0 * a[IX3(ii, j, kk, d1, d2)] +
                  1.0 / 6.0 * a[IX3(ii, j + 1, kk, d1, d2)];
            s = s + y * fil[di + 1][dk + 1];
          }
        g[IX3(i, j, k, e1, e2)] = s;
      }
}
/* compute_Sij (:672-730) of (U_,V_,W_) shaped like U, V, W into Sg[6]
 * (Sij(2:nxg,2:nyg,2:nzg,6)) and S (2:nxg-1,2:nyg-1,2:nzg-1); the corner
 * averages run in place in the source's loop order */
static void dyn_sij(const blo_t *o, const double *U_, const double *V_, const double *W_, double **Sg, double *S) {
  const int nxg = o->nxg, nyg = o->nyg, nzg = o->nzg;
  for (int k = 2; k <= nzg - 1; ++k)
    for (int j = 2; j <= nyg - 1; ++j)
      for (int i = 2; i <= nxg - 1; ++i) {
        AG(Sg[0], i, j, k) = (AU(U_, i, j, k) - AU(U_, i - 1, j, k)) / (o->x[i] - o->x[i - 1]);
        AG(Sg[1], i, j, k) = (AV(V_, i, j, k) - AV(V_, i, j - 1, k)) / (o->y[j] - o->y[j - 1]);
        AG(Sg[2], i, j, k) = (AW(W_, i, j, k) - AW(W_, i, j, k - 1)) / (o->z[k] - o->z[k - 1]);
      }
  for (int k = 2; k <= nzg; ++k)
    for (int j = 2; j <= nyg; ++j)
      for (int i = 2; i <= nxg; ++i) {
        AG(Sg[3], i, j, k) = sij_edge4(o, U_, V_, i, j, k);
        AG(Sg[4], i, j, k) = sij_edge5(o, U_, W_, i, j, k);
        AG(Sg[5], i, j, k) = sij_edge6(o, V_, W_, i, j, k);
      }
  for (int k = 2; k <= nzg - 1; ++k)
    for (int j = 2; j <= nyg - 1; ++j)
      for (int i = 2; i <= nxg - 1; ++i) {
        AG(Sg[3], i, j, k) = 0.25 * (AG(Sg[3], i, j, k) + AG(Sg[3], i + 1, j, k) + AG(Sg[3], i, j + 1, k) +
                                     AG(Sg[3], i + 1, j + 1, k));
        AG(Sg[4], i, j, k) = 0.25 * (AG(Sg[4], i, j, k) + AG(Sg[4], i + 1, j, k) + AG(Sg[4], i, j, k + 1) +
                                     AG(Sg[4], i + 1, j, k + 1));
        AG(Sg[5], i, j, k) = 0.25 * (AG(Sg[5], i, j, k) + AG(Sg[5], i, j + 1, k) + AG(Sg[5], i, j, k + 1) +
                                     AG(Sg[5], i, j + 1, k + 1));
      }
  for (int k = 2; k <= nzg - 1; ++k)
    for (int j = 2; j <= nyg - 1; ++j)
      for (int i = 2; i <= nxg - 1; ++i) {
        double s = 0.0;
        for (int c = 0; c < 6; ++c) {
          const double v = AG(Sg[c], i, j, k);
          s = s + (c < 3 ? 2.0 : 4.0) * v * v;
        }
        AG(S, i, j, k) = pow(s, 0.5);
      }
}

void blo_dynamic_smagorinsky(blo_t *o) {
  const int nx = o->nx, ny = o->ny, nz = o->nz, nxg = o->nxg, nyg = o->nyg, nzg = o->nzg;
  const int avg = o->les == 2, per = o->les == 3;  /* LES = 3: x-periodic helpers */
  const size_t n = (size_t)nxg * nyg * nzg;
  double *term = dalloc(n), *term1 = dalloc(n), *term2 = dalloc(n), *S = dalloc(n);
  double *Uf = dalloc(n), *Vf = dalloc(n), *Wf = dalloc(n);
  double *tb[6], *L[6], *Sg[6], *M[6];
  for (int c = 0; c < 6; ++c) { tb[c] = dalloc(n); L[c] = dalloc(n); Sg[c] = dalloc(n); M[c] = dalloc(n); }
  const double *U = o->U, *V = o->V, *W = o->W;
  /* Part 1: cell-centre velocities (interpolate_x/y/z, faces to centres) */
  for (int k = 1; k <= nzg; ++k)
    for (int j = 1; j <= nyg; ++j)
      for (int i = 2; i <= nx; ++i) AG(term, i, j, k) = 0.5 * (AU(U, i - 1, j, k) + AU(U, i, j, k));
  for (int k = 1; k <= nzg; ++k)
    for (int j = 2; j <= ny; ++j)
      for (int i = 1; i <= nxg; ++i) AG(term1, i, j, k) = 0.5 * (AV(V, i, j - 1, k) + AV(V, i, j, k));
  for (int k = 2; k <= nz; ++k)
    for (int j = 1; j <= nyg; ++j)
      for (int i = 1; i <= nxg; ++i) AG(term2, i, j, k) = 0.5 * (AW(W, i, j, k - 1) + AW(W, i, j, k));
  for (int j = 1; j <= nyg; ++j)
    for (int i = 1; i <= nxg; ++i) AG(term2, i, j, nzg) = 0.0;  /* ui = 0 of interpolate_z */
  dyn_bc_x(o, term, nxg, nyg, nzg, 2, per);
  dyn_bc_z(o, term2, nxg, nyg, 4);
  /* ui*uj at centres into ten_buf(2:nxg,2:nyg-1,2:nzg), its x / z ghosts, filtered */
  const double *pa[6] = {term, term1, term2, term, term, term1}, *pb[6] = {term, term1, term2, term1, term2, term2};
  for (int c = 0; c < 6; ++c) {
    for (int k = 2; k <= nzg; ++k)
      for (int j = 2; j <= nyg - 1; ++j)
        for (int i = 2; i <= nxg; ++i) AG(tb[c], i, j, k) = AG(pa[c], i, j, k) * AG(pb[c], i, j, k);
    dyn_bc_x(o, tb[c], nxg, nyg, nzg, 2, per);
    dyn_bc_z(o, tb[c], nxg, nyg, 4);
    dyn_filter(tb[c], nxg, nyg, nxg, 2, nyg - 1, nzg, L[c], nxg, nyg);  /* hat(ui uj) */
  }
  /* hat(ui) of the centre velocities into Sij(:,:,:,1:3) */
  dyn_filter(term, nxg, nyg, nxg, 2, nyg - 1, nzg, Sg[0], nxg, nyg);
  dyn_filter(term1, nxg, nyg, nxg, 2, nyg - 1, nzg, Sg[1], nxg, nyg);
  dyn_filter(term2, nxg, nyg, nxg, 2, nyg - 1, nzg, Sg[2], nxg, nyg);
  const int la[6] = {0, 1, 2, 0, 0, 1}, lb[6] = {0, 1, 2, 1, 2, 2};
  for (int c = 0; c < 6; ++c)
    for (int k = 2; k <= nzg - 1; ++k)
      for (int j = 2; j <= nyg - 1; ++j)
        for (int i = 2; i <= nxg - 1; ++i)
          AG(L[c], i, j, k) = AG(L[c], i, j, k) - AG(Sg[la[c]], i, j, k) * AG(Sg[lb[c]], i, j, k);
  /* Part 2: filtered velocities, their x / z ghosts, hat(Sij), |hat(S)| */
  dyn_filter(U, nx, nyg, nx, 1, nyg, nzg, Uf, nx, nyg);
  dyn_filter(V, nxg, ny, nxg, 1, ny, nzg, Vf, nxg, ny);
  dyn_filter(W, nxg, nyg, nxg, 1, nyg, nz, Wf, nxg, nyg);
  dyn_bc_x(o, Uf, nx, nyg, nzg, 1, per);
  dyn_bc_z(o, Uf, nx, nyg, 1);
  dyn_bc_x(o, Vf, nxg, ny, nzg, 2, per);
  dyn_bc_z(o, Vf, nxg, ny, 2);
  dyn_bc_x(o, Wf, nxg, nyg, nz, 2, per);
  dyn_bc_z(o, Wf, nxg, nyg, 3);
  dyn_sij(o, Uf, Vf, Wf, Sg, S);
  const double fs2 = pow(2.0, 2.0);  /* fil_size**2d0, fil_size = 2 after filter_xzy */
  for (int c = 0; c < 6; ++c)
    for (int k = 2; k <= nzg - 1; ++k)
      for (int j = 2; j <= nyg - 1; ++j)
        for (int i = 2; i <= nxg - 1; ++i) AG(M[c], i, j, k) = fs2 * AG(S, i, j, k) * AG(Sg[c], i, j, k);
  dyn_sij(o, U, V, W, Sg, S);
  for (int c = 0; c < 6; ++c) {
    for (int k = 2; k <= nzg - 1; ++k)
      for (int j = 2; j <= nyg - 1; ++j)
        for (int i = 2; i <= nxg - 1; ++i) AG(term, i, j, k) = AG(S, i, j, k) * AG(Sg[c], i, j, k);
    dyn_bc_x(o, term, nxg, nyg, nzg, 2, per);
    dyn_bc_z(o, term, nxg, nyg, 4);
    dyn_filter(term, nxg, nyg, nxg, 2, nyg - 1, nzg, Sg[c], nxg, nyg);  /* hat(|S| Sij) */
  }
  for (int c = 0; c < 6; ++c)
    for (int k = 2; k <= nzg - 1; ++k)
      for (int j = 2; j <= nyg - 1; ++j)
        for (int i = 2; i <= nxg - 1; ++i) AG(M[c], i, j, k) = AG(M[c], i, j, k) - AG(Sg[c], i, j, k);
  /* Part 3: nu_t = -1/2 (Mij Lij)/(Mij Mij) |S|, averaged in z for LES = 2 */
  double *nut = o->nu_t;
  memset(nut, 0, n * sizeof(double));
  for (int k = 2; k <= nzg - 1; ++k)
    for (int j = 2; j <= nyg - 1; ++j)
      for (int i = 2; i <= nxg - 1; ++i) {
        double ml = 0.0;
        for (int c = 0; c < 6; ++c) {
          if (c < 3) ml = ml + AG(M[c], i, j, k) * AG(L[c], i, j, k);
          else ml = ml + 2.0 * AG(M[c], i, j, k) * AG(L[c], i, j, k);
        }
        const double mm = AG(M[0], i, j, k) * AG(M[0], i, j, k) + AG(M[1], i, j, k) * AG(M[1], i, j, k) +
                          AG(M[2], i, j, k) * AG(M[2], i, j, k) +
                          2.0 * (AG(M[3], i, j, k) * AG(M[3], i, j, k) + AG(M[4], i, j, k) * AG(M[4], i, j, k) +
                                 AG(M[5], i, j, k) * AG(M[5], i, j, k));
        if (avg) {
          AG(L[0], i, j, k) = ml;  /* kept for the z averages */
          AG(L[1], i, j, k) = mm;
        } else {
          AG(nut, i, j, k) = -0.5 * (ml / mm) * AG(S, i, j, k);
        }
      }
  if (avg) {
    for (int j = 2; j <= nyg - 1; ++j)
      for (int i = 2; i <= nxg - 1; ++i) {
        double a = 0.0, b = 0.0;
        for (int k = 2; k <= nzg - 2; ++k) a += AG(L[0], i, j, k);
        for (int k = 2; k <= nzg - 2; ++k) b += AG(L[1], i, j, k);
        const double c = (a / (double)(nzg - 3)) / (b / (double)(nzg - 3));
        for (int k = 2; k <= nzg - 1; ++k) AG(nut, i, j, k) = -0.5 * c * AG(S, i, j, k);
      }
  } else {
    dyn_bc_x(o, nut, nxg, nyg, nzg, 4, 1);
    dyn_bc_z(o, nut, nxg, nyg, 4);
  }
  for (size_t q = 0; q < n; ++q) nut[q] = nut[q] > 0.0 ? nut[q] : 0.0;  /* clipping */
  for (int k = 1; k <= nzg; ++k)
    for (int i = 1; i <= nxg; ++i) {  /* apply_Neumann_bc_y(nu_t, 2), Dirichlet_nu_t = 0 */
      AG(nut, i, 1, k) = AG(nut, i, 2, k);
      AG(nut, i, nyg, k) = AG(nut, i, nyg - 1, k);
    }
  free(term); free(term1); free(term2); free(S); free(Uf); free(Vf); free(Wf);
  for (int c = 0; c < 6; ++c) { free(tb[c]); free(L[c]); free(Sg[c]); free(M[c]); }
}

void blo_get_nu_t(const blo_t *o, double *nu_t) {
  memcpy(nu_t, o->nu_t, sizeof(double) * (size_t)o->nxg * o->nyg * o->nzg);
}

/* ------------------------------------------------------------------------ */
/* statistics: statistics.f90:26-201.  means = 9 arrays (nx,ny):            */
/* Umean Vmean Wmean U2mean V2mean W2mean UVmean Pmean P2mean; nu_t_mean    */
/* (nxg,nyg); Cf, dUdy_wall (nx); sc = theta_inlet, delta99, Re_x, Re_theta,*/
/* Re_delta                                                                 */
/* ------------------------------------------------------------------------ */
void blo_statistics(const blo_t *o, double *means, double *nu_t_mean, double *Cf, double *dUdy_wall, double *sc) {
  const int nx = o->nx, ny = o->ny, nz = o->nz, nxg = o->nxg, nyg = o->nyg, nzg = o->nzg;
  const double *U = o->U, *V = o->V, *W = o->W, *P = o->P;
  const size_t pl = (size_t)nx * ny;
  double *Um = means, *Vm = means + pl, *Wm = means + 2 * pl, *U2 = means + 3 * pl, *V2 = means + 4 * pl,
         *W2 = means + 5 * pl, *UV = means + 6 * pl, *Pm = means + 7 * pl, *P2 = means + 8 * pl;
  memset(nu_t_mean, 0, sizeof(double) * (size_t)nxg * nyg);
  for (int jj = 1; jj <= ny; ++jj)
    for (int ii = 1; ii <= nx; ++ii) {
      double su = 0, sv = 0, sw = 0, su2 = 0, sv2 = 0, sw2 = 0, suv = 0, sp = 0, sp2 = 0, sn = 0;
      for (int k = 2; k <= nzg - 1; ++k) {
        /* term_1 = interp_y(U) (weighted), term_2 = interp_x(V) */
        double t1 = o->wy0[jj] * AU(U, ii, jj, k) + o->wy1[jj] * AU(U, ii, jj + 1, k);
        double t2 = 0.5 * (AV(V, ii, jj, k) + AV(V, ii + 1, jj, k));
        su += t1;
        sv += t2;
        su2 += t1 * t1;
        sv2 += t2 * t2;
        suv += t1 * t2;
        sp += AP(P, ii, jj, k);
        sp2 += AP(P, ii, jj, k) * AP(P, ii, jj, k);
        sn += NUT(ii, jj, k);
      }
      for (int k = 1; k <= nz - 2; ++k) {
        /* term = interp_y(interp_x(W)) */
        double a = 0.5 * (AW(W, ii, jj, k) + AW(W, ii + 1, jj, k));
        double b = 0.5 * (AW(W, ii, jj + 1, k) + AW(W, ii + 1, jj + 1, k));
        double t = o->wy0[jj] * a + o->wy1[jj] * b;
        sw += t;
        sw2 += t * t;
      }
      size_t q = (size_t)(jj - 1) * nx + (ii - 1);
      const double dn = (double)(nzg - 2), dw = (double)(nz - 2);
      Um[q] = su / dn; Vm[q] = sv / dn; Wm[q] = sw / dw;
      U2[q] = su2 / dn; V2[q] = sv2 / dn; W2[q] = sw2 / dw;
      UV[q] = suv / dn; Pm[q] = sp / dn; P2[q] = sp2 / dn;
      nu_t_mean[(size_t)(jj - 1) * nxg + (ii - 1)] = sn / dn;
    }
  for (int ii = 1; ii <= nx; ++ii) {
    double a1 = 0, a2 = 0;
    for (int k = 2; k <= nzg - 1; ++k) {
      a1 += AU(U, ii, 1, k);
      a2 += AU(U, ii, 2, k);
    }
    a1 /= (double)(nzg - 2);
    a2 /= (double)(nzg - 2);
    dUdy_wall[ii - 1] = (a2 - a1) / (o->yg[2] - o->yg[1]);
  }
  for (int ii = 1; ii <= nx; ++ii) {
    double n11 = nu_t_mean[ii - 1], n12 = nu_t_mean[(size_t)nxg + ii - 1];
    double n21 = nu_t_mean[ii], n22 = nu_t_mean[(size_t)nxg + ii];
    double tau = 0.25 * (n11 + n12 + n21 + n22) * dUdy_wall[ii - 1];
    double uvw = UV[ii - 1];
    Cf[ii - 1] = 2.0 * (-uvw + o->nu * dUdy_wall[ii - 1] + tau) / 1.0;
  }
  /* inlet theta, delta99 and Reynolds numbers (statistics.f90:178-201) */
  const double Uinf = 1.0;
  double theta = 0.0;
  for (int j = 2; j <= ny; ++j) {
    double tj = Um[(size_t)(j - 1) * nx] / Uinf * (1.0 - Um[(size_t)(j - 1) * nx] / Uinf);
    double tm = Um[(size_t)(j - 2) * nx] / Uinf * (1.0 - Um[(size_t)(j - 2) * nx] / Uinf);
    theta = theta + 0.5 * (tj + tm) * (o->y[j] - o->y[j - 1]);
  }
  int jref = 0;
  for (int j = 1; j <= ny; ++j)
    if (Um[(size_t)(j - 1) * nx] >= 0.99 * Uinf) { jref = j; break; }
  if (jref < 2) jref = 2;
  double u1 = Um[(size_t)(jref - 2) * nx], u2 = Um[(size_t)(jref - 1) * nx];
  double w1 = (0.99 * Uinf - u1) / (u2 - u1), w0 = 1.0 - w1;
  double d99 = w1 * o->y[jref] + w0 * o->y[jref - 1];
  sc[0] = theta;
  sc[1] = d99;
  sc[2] = o->x[1] * Uinf / o->nu;
  sc[3] = theta * Uinf / o->nu;
  sc[4] = d99 * Uinf / o->nu;
}

/* ------------------------------------------------------------------------ */
/* equilibrium law of the wall: wallmodel.f90:1951-1985 with                */
/* Newton_iter_solver (Newton_solver.f90:13-79): kappa 0.38, B 5.2,          */
/* y = yg(3), 30 iterations, |f| < 1e-10.  utau (nx) is the initial guess on */
/* entry and the model on exit; returns the largest iteration count.         */
/* ------------------------------------------------------------------------ */
static int law_of_wall_at(const blo_t *o, int jref, double *utau);
int blo_law_of_wall(const blo_t *o, double *utau) { return law_of_wall_at(o, 3, utau); }

static int law_of_wall_at(const blo_t *o, int jref, double *utau) {
  const double kap = 0.38, B = 5.20, yref = o->yg[jref], nu = o->nu;
  int iters_max = 0;
  for (int i = 2; i <= o->nx - 1; ++i) {
    double x = utau[i - 1];
    if (utau[i - 1] != utau[i - 1]) utau[i - 1] = 0.0;
    double um = 0.0;
    for (int k = 2; k <= o->nzg - 1; ++k) um += AU(o->U, i, jref, k);
    um = um / (double)(o->nzg - 2);
    int k;
    for (k = 1; k <= 30; ++k) {
      double fx = x / kap * log(yref * x / nu) + B * x - um;
      double fp = 1.0 / kap * log(yref * x / nu) + 1.0 / kap + B;
      if (fabs(fx) < 1e-10) break;
      x = x - fx / fp;
    }
    int iters = k - 1;
    utau[i - 1] = (x != x) ? 0.0 : x;
    if (iters > iters_max) iters_max = iters;
  }
  utau[0] = utau[1];
  utau[o->nx - 1] = utau[o->nx - 2];
  return iters_max;
}

void blo_set_les(blo_t *o, int les_model) { o->les = les_model; }

/* ------------------------------------------------------------------------ */
/* wall models of the step                                                  */
/* ------------------------------------------------------------------------ */
int blo_set_wall_model(blo_t *o, int mode, int jh, const double *params) {
  if (mode < 0 || mode > 2) return -1;
  if (mode && (jh < 2 || jh > o->nyg - 1)) return -2;
  if (mode == 2 && !params) return -3;
  o->wm = mode;
  o->wm_jh = jh;
  if (mode == 2) memcpy(o->mlp_params, params, sizeof(double) * blo_mlp_nparams());
  /* Newton's first guess utau_ref (initialization.f90:744-745) */
  for (int i = 1; i <= o->nx; ++i) o->utau_wm[i - 1] = sqrt(0.5 * 0.027 * pow(o->x[i] / o->nu, -1.0 / 7.0));
  return 0;
}

/* the network's inputs at wall point (i,k) from row jh */
static void wall_features(const blo_t *o, int i, int jh, int k, float *x) {
  const double h = o->yg[jh];
  const double u = AU(o->U, i, jh, k);
  const double w = 0.25 * (AW(o->W, i, jh, k) + AW(o->W, i + 1, jh, k) + AW(o->W, i, jh, k - 1) +
                           AW(o->W, i + 1, jh, k - 1));
  const double dp = (AP(o->P, i + 1, jh, k) - AP(o->P, i, jh, k)) / (o->xg[i + 1] - o->xg[i]);
  x[0] = (float)u;
  x[1] = (float)w;
  x[2] = (float)(log(fmax(h * fabs(u) / o->nu, 1.0)) / 10.0);
  x[3] = (float)(100.0 * h * dp);
}

/* viscosity of the U-equation's wall flux at (i,k): nu_y1 of the LES branch
 * (equations.f90:97-98) at j = 2, nu alone without LES */
static double wall_flux_nu(const blo_t *o, int i, int k) {
  if (!o->les) return o->nu;
  return o->nu + 0.5 * (o->wy0[1] * AP(o->nu_t, i, 1, k) + o->wy1[1] * AP(o->nu_t, i, 2, k) +
                        o->wy0[1] * AP(o->nu_t, i + 1, 1, k) + o->wy1[1] * AP(o->nu_t, i + 1, 2, k));
}

static void wall_model_eval(blo_t *o) {
  const int ni = o->nx - 2, nk = o->nzg - 3;
  if (o->wm == 1) {
    law_of_wall_at(o, o->wm_jh, o->utau_wm);
    for (int k = 0; k < nk; ++k)
      for (int q = 0; q < ni; ++q) {
        const double u = o->utau_wm[q + 1];
        o->wm_ax[(size_t)k * ni + q] = u * u / wall_flux_nu(o, q + 2, k + 2);
        o->wm_az[(size_t)k * ni + q] = 0.0;
      }
  } else if (o->wm == 2) {
    const int rows = ni * nk;
    float *X = (float *)malloc(sizeof(float) * 4 * (size_t)rows), *Y = (float *)malloc(sizeof(float) * 2 * (size_t)rows);
    for (int r = 0; r < rows; ++r) wall_features(o, r % ni + 2, o->wm_jh, r / ni + 2, X + (size_t)r * 4);
    blo_mlp_forward(o->mlp_params, X, rows, Y, 0);
    for (int r = 0; r < rows; ++r) {
      const double nuw = wall_flux_nu(o, r % ni + 2, r / ni + 2);
      o->wm_ax[r] = 1e-3 * (double)Y[(size_t)r * 2] / nuw;
      o->wm_az[r] = 1e-3 * (double)Y[(size_t)r * 2 + 1] / nuw;
    }
    free(X);
    free(Y);
  }
}

void blo_wall_stress(blo_t *o, double *tau_x, double *tau_z) {
  wall_model_eval(o);
  const int ni = o->nx - 2;
  const size_t n = (size_t)ni * (o->nzg - 3);
  for (size_t q = 0; q < n; ++q) {
    const double nuw = wall_flux_nu(o, (int)(q % ni) + 2, (int)(q / ni) + 2);
    if (tau_x) tau_x[q] = o->wm_ax[q] * nuw;
    if (tau_z) tau_z[q] = o->wm_az[q] * nuw;
  }
}

