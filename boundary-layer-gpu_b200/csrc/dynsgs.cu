// Dynamic Smagorinsky eddy viscosity on the device: LES = 2 (coefficient
// averaged in z, subgrid.f90:261-414 sgs_dynamic_Smagorinsky) and LES = 3
// (pointwise coefficient, subgrid.f90:420-583 _noaverage).
//
// The model runs in FP64 in both precisions, on dense (nxg,nyg,nzg) work
// arrays indexed 1-based like the source's module arrays (i fastest); the
// velocity-shaped ones use the U (nx,nyg), V (nxg,ny), W (nxg,nyg) plane
// shapes.  Every step of the source is one kernel (one thread per point) in
// the source's order, with the source's evaluation order in each expression (the file is
// compiled with -fmad=false):
//   interpolate_x/y/z (interpolation.f90:24-114) to cell centres;
//   the x helpers apply_Neumann_bc_x / apply_periodic_bc_x
//   (boundary_conditions.f90:295-344) and apply_periodic_bc_z (:732-760) on
//   one process, where update_ghost_interior_planes is empty;
//   filter_xzy (subgrid.f90:140-184, fil_size = 2);
//   compute_Sij (subgrid.f90:672-730), with the in-place corner averages
//   taken from a separate array of edge values (the source's loop order
//   reads only not-yet-averaged neighbours, so the values are the same);
//   the Lij, Mij contractions, the z average (LES = 2), clipping and
//   Neumann y (Dirichlet_nu_t = 0).
// The result goes to nu_t in the box layout as T.  Every index a kernel
// touches lies in 1..nxg x 1..nyg x 1..nzg of its array's own shape.
#include "kernels.cuh"

namespace blgpu {
namespace {

enum { W_U, W_V, W_W, W_T0, W_T1, W_T2, W_S, W_UF, W_VF, W_WF, W_TB, W_L, W_G = W_L + 6, W_M = W_G + 6,
       W_COUNT = W_M + 6 };

struct P6 {
  double *p[6];
};

// index range i0..i0+ni-1, j0.., k0..: one thread per point, i along
// blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z
// (nj, nk <= 65535, checked at blgpu_create)
struct Rng {
  int i0, ni, j0, nj, k0, nk;
};

__device__ __forceinline__ long long dix(int i, int j, int k, int d1, int d2) {
  return ((long long)(k - 1) * d2 + (j - 1)) * (long long)d1 + (i - 1);
}

#define FOR_RNG(R)                                                                                 \
  if (const int i = (R).i0 + (int)(blockIdx.x * blockDim.x + threadIdx.x), j = (R).j0 + (int)blockIdx.y, \
      k = (R).k0 + (int)blockIdx.z;                                                                      \
      i < (R).i0 + (R).ni)

template <typename T>
__global__ void k_gather(Geo g, Rng R, const T *__restrict__ U, const T *__restrict__ V, const T *__restrict__ W,
                         double *__restrict__ Ud, double *__restrict__ Vd, double *__restrict__ Wd) {
  FOR_RNG(R) {
    const long long b = bidx(g, i, j, k);
    if (i <= g.nx) Ud[dix(i, j, k, g.nx, g.nyg)] = (double)U[b];
    if (j <= g.ny) Vd[dix(i, j, k, g.nxg, g.ny)] = (double)V[b];
    if (k <= g.nz) Wd[dix(i, j, k, g.nxg, g.nyg)] = (double)W[b];
  }
}

// faces to centres: term(2:nx), term_1(:,2:ny), term_2(:,:,2:nz), term_2(nzg) = 0
__global__ void k_interp(Geo g, Rng R, const double *__restrict__ Ud, const double *__restrict__ Vd,
                         const double *__restrict__ Wd, double *__restrict__ t0, double *__restrict__ t1,
                         double *__restrict__ t2) {
  FOR_RNG(R) {
    const long long c = dix(i, j, k, g.nxg, g.nyg);
    if (i >= 2 && i <= g.nx) t0[c] = 0.5 * (Ud[dix(i - 1, j, k, g.nx, g.nyg)] + Ud[dix(i, j, k, g.nx, g.nyg)]);
    if (j >= 2 && j <= g.ny) t1[c] = 0.5 * (Vd[dix(i, j - 1, k, g.nxg, g.ny)] + Vd[dix(i, j, k, g.nxg, g.ny)]);
    if (k >= 2 && k <= g.nz) t2[c] = 0.5 * (Wd[dix(i, j, k - 1, g.nxg, g.nyg)] + Wd[dix(i, j, k, g.nxg, g.nyg)]);
    if (k == g.nzg) t2[c] = 0.0;
  }
}

// x ghosts of every row (j,k) of a dense array with first dimension d1
__global__ void k_bc_x(long long rows, double *__restrict__ a, int d1, int id, int periodic, int nx, int nxg) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < rows; q += (long long)gridDim.x * blockDim.x) {
    double *r = a + q * d1;
    if (!periodic) {
      if (id == 1) { r[0] = r[1]; r[nx - 1] = r[nx - 2]; }
      else { r[0] = r[1]; r[nxg - 1] = r[nxg - 2]; }
    } else {
      if (id == 1) { r[0] = r[nx - 2]; r[nx - 1] = r[1]; }
      else { r[0] = r[nxg - 3]; r[nxg - 2] = r[1]; r[nxg - 1] = r[2]; }
    }
  }
}

// z ghost planes (planes of pl = d1*d2 entries)
__global__ void k_bc_z(long long pl, double *__restrict__ a, int id, int nz, int nzg) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < pl; p += (long long)gridDim.x * blockDim.x) {
    if (id == 3) {
      a[p] = a[(nz - 2) * pl + p];
      a[(nz - 1) * pl + p] = a[pl + p];
    } else {
      a[p] = a[(nzg - 3) * pl + p];
      a[(nzg - 2) * pl + p] = a[pl + p];
      a[(nzg - 1) * pl + p] = a[2 * pl + p];
    }
  }
}

__global__ void k_prod(Geo g, Rng R, double *__restrict__ tb, const double *__restrict__ pa,
                       const double *__restrict__ pb) {
  FOR_RNG(R) {
    const long long c = dix(i, j, k, g.nxg, g.nyg);
    tb[c] = pa[c] * pb[c];
  }
}

// filter_xzy of the section a(1:n1, ja:jb, 1:n3) of a dense (d1,d2,*) array
// into o(i,j,k), i = 2..n1-1, j = ja..jb, k = 2..n3-1 (output dims e1,e2);
// the range R carries those output indices.  A block of FK_I threads takes
// FK_I outputs along i at one j and marches over FK_K planes in k: the
// y-combined values of input columns i-1..i+FK_I of plane kk go to a ring of
// three shared rows, and each output sums its 3 x 3 (x,z) neighbourhood from
// the ring in the source's order (x outer, z inner).
constexpr int FK_I = 128, FK_K = 16;

__global__ void __launch_bounds__(FK_I) k_filter(Rng R, const double *__restrict__ a, int d1, int d2, int ja,
                                                 int jb, double *__restrict__ o, int e1, int e2) {
  const double fil[3][3] = {{1.0 / 36.0, 1.0 / 9.0, 1.0 / 36.0},
                            {1.0 / 9.0, 4.0 / 9.0, 1.0 / 9.0},
                            {1.0 / 36.0, 1.0 / 9.0, 1.0 / 36.0}};
  __shared__ double ys[3][FK_I + 2];
  const int t = threadIdx.x;
  const int ib = R.i0 + (int)blockIdx.x * FK_I;  // first output i of the block
  const int i = ib + t, ilast = R.i0 + R.ni - 1;
  const int j = R.j0 + (int)blockIdx.y;
  const int kb = R.k0 + (int)blockIdx.z * FK_K;
  const int ke = min(kb + FK_K - 1, R.k0 + R.nk - 1);
  for (int kk = kb - 1; kk <= ke + 1; ++kk) {
    double *row = ys[(kk - kb + 1) % 3];
    for (int x = t; x < FK_I + 2; x += FK_I) {
      const int ii = ib - 1 + x;
      if (ii <= ilast + 1) {
        double y;
        if (j == ja)
          y = 2.0 / 3.0 * a[dix(ii, j, kk, d1, d2)] + 1.0 / 3.0 * a[dix(ii, j + 1, kk, d1, d2)];
        else if (j == jb)
          y = 1.0 / 3.0 * a[dix(ii, j - 1, kk, d1, d2)] + 2.0 / 3.0 * a[dix(ii, j, kk, d1, d2)];
        else
          y = 1.0 / 6.0 * a[dix(ii, j - 1, kk, d1, d2)] + 2.0 / 3.0 * a[dix(ii, j, kk, d1, d2)] +
              1.0 / 6.0 * a[dix(ii, j + 1, kk, d1, d2)];
        row[x] = y;
      }
    }
    __syncthreads();
    if (kk >= kb + 1 && i <= ilast) {  // output plane k = kk-1 from planes kk-2, kk-1, kk
      const int k = kk - 1;
      double s = 0.0;
      for (int di = -1; di <= 1; ++di)
        for (int dk = -1; dk <= 1; ++dk) s = s + ys[(k + dk - kb + 1) % 3][t + 1 + di] * fil[di + 1][dk + 1];
      o[dix(i, j, k, e1, e2)] = s;
    }
    __syncthreads();
  }
}

// Lij = hat(ui uj) - hat(ui) hat(uj)
__global__ void k_leonard(Geo g, Rng R, P6 L, P6 G) {
  FOR_RNG(R) {
    const long long c = dix(i, j, k, g.nxg, g.nyg);
    const double u = G.p[0][c], v = G.p[1][c], w = G.p[2][c];
    L.p[0][c] = L.p[0][c] - u * u;
    L.p[1][c] = L.p[1][c] - v * v;
    L.p[2][c] = L.p[2][c] - w * w;
    L.p[3][c] = L.p[3][c] - u * v;
    L.p[4][c] = L.p[4][c] - u * w;
    L.p[5][c] = L.p[5][c] - v * w;
  }
}

struct DV {
  const double *U, *V, *W;
  int nx, ny, nxg, nyg;
  __device__ double u(int i, int j, int k) const { return U[dix(i, j, k, nx, nyg)]; }
  __device__ double v(int i, int j, int k) const { return V[dix(i, j, k, nxg, ny)]; }
  __device__ double w(int i, int j, int k) const { return W[dix(i, j, k, nxg, nyg)]; }
};

// the edge rates of strain of compute_Sij before its corner averages
__device__ __forceinline__ double e4(const Geo &g, const DV &d, int i, int j, int k) {
  return 0.5 * ((d.u(i - 1, j, k) - d.u(i - 1, j - 1, k)) / (g.yg[j] - g.yg[j - 1]) +
                (d.v(i, j - 1, k) - d.v(i - 1, j - 1, k)) / (g.xg[i] - g.xg[i - 1]));
}
__device__ __forceinline__ double e5(const Geo &g, const DV &d, int i, int j, int k) {
  return 0.5 * ((d.u(i - 1, j, k) - d.u(i - 1, j, k - 1)) / (g.zg[k] - g.zg[k - 1]) +
                (d.w(i, j, k - 1) - d.w(i - 1, j, k - 1)) / (g.xg[i] - g.xg[i - 1]));
}
__device__ __forceinline__ double e6(const Geo &g, const DV &d, int i, int j, int k) {
  return 0.5 * ((d.v(i, j - 1, k) - d.v(i, j - 1, k - 1)) / (g.zg[k] - g.zg[k - 1]) +
                (d.w(i, j, k - 1) - d.w(i, j - 1, k - 1)) / (g.yg[j] - g.yg[j - 1]));
}

// compute_Sij's edge values at i = 2..nxg, j = 2..nyg, k = 2..nzg (dense (nxg,nyg) planes)
__global__ void k_edges(Geo g, Rng R, DV d, double *__restrict__ E4, double *__restrict__ E5,
                        double *__restrict__ E6) {
  FOR_RNG(R) {
    const long long c = dix(i, j, k, g.nxg, g.nyg);
    E4[c] = e4(g, d, i, j, k);
    E5[c] = e5(g, d, i, j, k);
    E6[c] = e6(g, d, i, j, k);
  }
}

// Sij (cell centres) and |S| of the velocity triple d, the off-diagonal terms
// as the source's corner averages of the edge values E4..E6
__global__ void k_sij(Geo g, Rng R, DV d, const double *__restrict__ E4, const double *__restrict__ E5,
                      const double *__restrict__ E6, P6 G, double *__restrict__ S) {
  FOR_RNG(R) {
    const long long c = dix(i, j, k, g.nxg, g.nyg), sj = g.nxg, sk = (long long)g.nxg * g.nyg;
    double s[6];
    s[0] = (d.u(i, j, k) - d.u(i - 1, j, k)) / (g.x[i] - g.x[i - 1]);
    s[1] = (d.v(i, j, k) - d.v(i, j - 1, k)) / (g.y[j] - g.y[j - 1]);
    s[2] = (d.w(i, j, k) - d.w(i, j, k - 1)) / (g.z[k] - g.z[k - 1]);
    s[3] = 0.25 * (E4[c] + E4[c + 1] + E4[c + sj] + E4[c + 1 + sj]);
    s[4] = 0.25 * (E5[c] + E5[c + 1] + E5[c + sk] + E5[c + 1 + sk]);
    s[5] = 0.25 * (E6[c] + E6[c + sj] + E6[c + sk] + E6[c + sj + sk]);
    double q = 0.0;
    for (int m = 0; m < 6; ++m) {
      G.p[m][c] = s[m];
      q = q + (m < 3 ? 2.0 : 4.0) * s[m] * s[m];
    }
    S[c] = sqrt(q);
  }
}

// Mij = fil_size^2 |hat(S)| hat(Sij), fil_size = 2
__global__ void k_mij(Geo g, Rng R, P6 M, P6 G, const double *__restrict__ S) {
  FOR_RNG(R) {
    const long long c = dix(i, j, k, g.nxg, g.nyg);
    for (int m = 0; m < 6; ++m) M.p[m][c] = 4.0 * S[c] * G.p[m][c];
  }
}

__global__ void k_ssij(Geo g, Rng R, double *__restrict__ t, const double *__restrict__ S,
                       const double *__restrict__ Gm) {
  FOR_RNG(R) {
    const long long c = dix(i, j, k, g.nxg, g.nyg);
    t[c] = S[c] * Gm[c];
  }
}

__global__ void k_msub(Geo g, Rng R, P6 M, P6 G) {
  FOR_RNG(R) {
    const long long c = dix(i, j, k, g.nxg, g.nyg);
    for (int m = 0; m < 6; ++m) M.p[m][c] = M.p[m][c] - G.p[m][c];
  }
}

// Mij Lij and Mij Mij; LES = 3 forms nu_t here, LES = 2 keeps both for the z averages
__global__ void k_contract(Geo g, Rng R, P6 M, P6 L, const double *__restrict__ S, double *__restrict__ nut,
                           double *__restrict__ ml_out, double *__restrict__ mm_out, int avg) {
  FOR_RNG(R) {
    const long long c = dix(i, j, k, g.nxg, g.nyg);
    double ml = 0.0;
    for (int m = 0; m < 6; ++m) {
      if (m < 3) ml = ml + M.p[m][c] * L.p[m][c];
      else ml = ml + 2.0 * M.p[m][c] * L.p[m][c];
    }
    const double m0 = M.p[0][c], m1 = M.p[1][c], m2 = M.p[2][c], m3 = M.p[3][c], m4 = M.p[4][c], m5 = M.p[5][c];
    const double mm = m0 * m0 + m1 * m1 + m2 * m2 + 2.0 * (m3 * m3 + m4 * m4 + m5 * m5);
    if (avg) {
      ml_out[c] = ml;
      mm_out[c] = mm;
    } else {
      nut[c] = -0.5 * (ml / mm) * S[c];
    }
  }
}

// LES = 2: <Mij Lij> / <Mij Mij> over k = 2..nzg-2, summed in k order
__global__ void k_zavg(Geo g, Rng R, const double *__restrict__ ml, const double *__restrict__ mm,
                       const double *__restrict__ S, double *__restrict__ nut) {
  FOR_RNG(R) {
    (void)k;
    double a = 0.0, b = 0.0;
    for (int kk = 2; kk <= g.nzg - 2; ++kk) a += ml[dix(i, j, kk, g.nxg, g.nyg)];
    for (int kk = 2; kk <= g.nzg - 2; ++kk) b += mm[dix(i, j, kk, g.nxg, g.nyg)];
    const double cz = (a / (double)(g.nzg - 3)) / (b / (double)(g.nzg - 3));
    for (int kk = 2; kk <= g.nzg - 1; ++kk) {
      const long long c = dix(i, j, kk, g.nxg, g.nyg);
      nut[c] = -0.5 * cz * S[c];
    }
  }
}

// clipping, Neumann y, box layout
template <typename T>
__global__ void k_store(Geo g, Rng R, const double *__restrict__ nd, T *__restrict__ nut) {
  FOR_RNG(R) {
    const int jj = j == 1 ? 2 : (j == g.nyg ? g.nyg - 1 : j);
    const double v = nd[dix(i, jj, k, g.nxg, g.nyg)];
    nut[bidx(g, i, j, k)] = (T)(v > 0.0 ? v : 0.0);
  }
}

// grid-stride launches of 256 threads (x / z ghosts), at most 16 blocks per SM of 148
inline unsigned blocks(long long n) {
  const long long b = (n + 255) / 256, cap = 148LL * 16;
  return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

inline Rng rng(int i0, int i1, int j0, int j1, int k0, int k1) {
  return Rng{i0, i1 - i0 + 1, j0, j1 - j0 + 1, k0, k1 - k0 + 1};
}

}  // namespace

size_t dyn_smagorinsky_work_bytes(int nxg, int nyg, int nzg) {
  return (size_t)W_COUNT * (size_t)nxg * nyg * nzg * sizeof(double);
}

template <typename T>
int launch_dyn_smagorinsky(const Geo &g, const T *U, const T *V, const T *W, double *work, int model, T *nut,
                           cudaStream_t st) {
  const int nx = g.nx, ny = g.ny, nz = g.nz, nxg = g.nxg, nyg = g.nyg, nzg = g.nzg;
  const size_t n = (size_t)nxg * nyg * nzg;
  double *w[W_COUNT];
  for (int q = 0; q < W_COUNT; ++q) w[q] = work + (size_t)q * n;
  P6 L, G, M;
  for (int m = 0; m < 6; ++m) { L.p[m] = w[W_L + m]; G.p[m] = w[W_G + m]; M.p[m] = w[W_M + m]; }
  const int per = model == 3;
  int launches = 0;
  auto go = [&](const Rng &R) { ++launches; return dim3((R.ni + 127) / 128, R.nj, R.nk); };
  auto bcx = [&](double *a, int d1, int d2, int d3, int id, int periodic) {
    const long long rows = (long long)d2 * d3;
    ++launches;
    k_bc_x<<<blocks(rows), 256, 0, st>>>(rows, a, d1, id, periodic, nx, nxg);
  };
  auto bcz = [&](double *a, int d1, int d2, int id) {
    const long long pl = (long long)d1 * d2;
    ++launches;
    k_bc_z<<<blocks(pl), 256, 0, st>>>(pl, a, id, nz, nzg);
  };
  auto filt = [&](const double *a, int d1, int d2, int n1, int ja, int jb, int n3, double *o, int e1, int e2) {
    const Rng R = rng(2, n1 - 1, ja, jb, 2, n3 - 1);
    ++launches;
    k_filter<<<dim3((R.ni + FK_I - 1) / FK_I, R.nj, (R.nk + FK_K - 1) / FK_K), FK_I, 0, st>>>(R, a, d1, d2, ja, jb, o,
                                                                                            e1, e2);
  };
  const Rng all = rng(1, nxg, 1, nyg, 1, nzg), in = rng(2, nxg - 1, 2, nyg - 1, 2, nzg - 1);
  double *Ud = w[W_U], *Vd = w[W_V], *Wd = w[W_W], *t0 = w[W_T0], *t1 = w[W_T1], *t2 = w[W_T2], *S = w[W_S];
  double *Uf = w[W_UF], *Vf = w[W_VF], *Wf = w[W_WF], *tb = w[W_TB];
  k_gather<T><<<go(all), 128, 0, st>>>(g, all, U, V, W, Ud, Vd, Wd);
  // Part 1: Leonard term
  k_interp<<<go(all), 128, 0, st>>>(g, all, Ud, Vd, Wd, t0, t1, t2);
  bcx(t0, nxg, nyg, nzg, 2, per);
  bcz(t2, nxg, nyg, 4);
  const double *pa[6] = {t0, t1, t2, t0, t0, t1}, *pb[6] = {t0, t1, t2, t1, t2, t2};
  const Rng rp = rng(2, nxg, 2, nyg - 1, 2, nzg);
  for (int m = 0; m < 6; ++m) {
    k_prod<<<go(rp), 128, 0, st>>>(g, rp, tb, pa[m], pb[m]);
    bcx(tb, nxg, nyg, nzg, 2, per);
    bcz(tb, nxg, nyg, 4);
    filt(tb, nxg, nyg, nxg, 2, nyg - 1, nzg, L.p[m], nxg, nyg);
  }
  filt(t0, nxg, nyg, nxg, 2, nyg - 1, nzg, G.p[0], nxg, nyg);
  filt(t1, nxg, nyg, nxg, 2, nyg - 1, nzg, G.p[1], nxg, nyg);
  filt(t2, nxg, nyg, nxg, 2, nyg - 1, nzg, G.p[2], nxg, nyg);
  k_leonard<<<go(in), 128, 0, st>>>(g, in, L, G);
  // Part 2: Mij
  filt(Ud, nx, nyg, nx, 1, nyg, nzg, Uf, nx, nyg);
  filt(Vd, nxg, ny, nxg, 1, ny, nzg, Vf, nxg, ny);
  filt(Wd, nxg, nyg, nxg, 1, nyg, nz, Wf, nxg, nyg);
  bcx(Uf, nx, nyg, nzg, 1, per);
  bcz(Uf, nx, nyg, 1);
  bcx(Vf, nxg, ny, nzg, 2, per);
  bcz(Vf, nxg, ny, 2);
  bcx(Wf, nxg, nyg, nz, 2, per);
  bcz(Wf, nxg, nyg, 3);
  // t0..t2 are free here: they hold the edge values of each compute_Sij
  const Rng re = rng(2, nxg, 2, nyg, 2, nzg);
  const DV df{Uf, Vf, Wf, nx, ny, nxg, nyg}, du{Ud, Vd, Wd, nx, ny, nxg, nyg};
  k_edges<<<go(re), 128, 0, st>>>(g, re, df, t0, t1, t2);
  k_sij<<<go(in), 128, 0, st>>>(g, in, df, t0, t1, t2, G, S);
  k_mij<<<go(in), 128, 0, st>>>(g, in, M, G, S);
  k_edges<<<go(re), 128, 0, st>>>(g, re, du, t0, t1, t2);
  k_sij<<<go(in), 128, 0, st>>>(g, in, du, t0, t1, t2, G, S);
  for (int m = 0; m < 6; ++m) {
    k_ssij<<<go(in), 128, 0, st>>>(g, in, t0, S, G.p[m]);
    bcx(t0, nxg, nyg, nzg, 2, per);
    bcz(t0, nxg, nyg, 4);
    filt(t0, nxg, nyg, nxg, 2, nyg - 1, nzg, G.p[m], nxg, nyg);
  }
  k_msub<<<go(in), 128, 0, st>>>(g, in, M, G);
  // Part 3: nu_t (tb holds it; entries the source leaves at zero stay zero)
  cudaMemsetAsync(tb, 0, n * sizeof(double), st);
  ++launches;  // the memset is one stream operation (one graph node) like a kernel
  if (model == 2) {
    k_contract<<<go(in), 128, 0, st>>>(g, in, M, L, S, tb, t1, t2, 1);
    const Rng ij = rng(2, nxg - 1, 2, nyg - 1, 1, 1);
    k_zavg<<<go(ij), 128, 0, st>>>(g, ij, t1, t2, S, tb);
  } else {
    k_contract<<<go(in), 128, 0, st>>>(g, in, M, L, S, tb, nullptr, nullptr, 0);
    bcx(tb, nxg, nyg, nzg, 4, 1);
    bcz(tb, nxg, nyg, 4);
  }
  k_store<T><<<go(all), 128, 0, st>>>(g, all, tb, nut);
  return launches;
}

template int launch_dyn_smagorinsky<double>(const Geo &, const double *, const double *, const double *, double *,
                                            int, double *, cudaStream_t);
template int launch_dyn_smagorinsky<float>(const Geo &, const float *, const float *, const float *, double *, int,
                                           float *, cudaStream_t);

}  // namespace blgpu
