#pragma once
// stencil_impl.cuh -- finite-difference kernels of the step path.  Included
// by stencil64.cu (FP64, compiled with -fmad=false so every expression keeps
// the order and rounding of the Fortran source, with no fused multiply-adds)
// and by stencil32.cu (FP32 mixed form, contraction allowed).
//
//   k_rhs_rk      RHS of u, v, w (equations.f90:24-415) fused with the RK
//                 substep update (time_integration.f90:351-458)
//   k_project     project_velocity (projection.f90:355-386) fused with the
//                 pressure save of solve_poisson_equation (projection.f90:75-85)
//   k_bc_*        apply_boundary_conditions_gpu (boundary_conditions.f90:127-262)
//   k_dt_*        compute_dt (time_integration.f90:528-591)
//   k_maxdiv      check_divergence (projection.f90:391-413)
#include <cstring>

#include "kernels.cuh"
#include "tma.cuh"

namespace blgpu {

// ---------------------------------------------------------------------------
// division policy: the FP64 path divides exactly where the source divides;
// the FP32 path multiplies by the reciprocal table instead.
// The FP64 quotient is the correctly rounded a/b formed from the table's
// reciprocal by mdiv (common.cuh): the value of the source's division.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double qdiv(double a, double b, double rb) { return mdiv(a, b, rb); }
// maximum that keeps a NaN (fmax drops it): check_divergence of a field that
// holds a NaN reads NaN
__device__ __forceinline__ double max_keep_nan(double a, double b) { return (a > b || a != a) ? a : b; }
__device__ __forceinline__ float qdiv(float a, float, float rb) { return a * rb; }

template <typename T> struct Ld {
  const T *__restrict__ p;
  long long sx, sy, sz;  // strides: 1, px, plane
  __device__ __forceinline__ T operator()(long long c, int di, int dj, int dk) const {
    return __ldg(p + c + di + dj * sy + dk * sz);
  }
};

// RHS of u at (i,j,k), equations.f90:53-91 (DNS) / :98-129 (LES)
template <typename T, bool LES, typename L = Ld<T>>
__device__ __forceinline__ T rhs_u_at(const Geo &g, const MetT<T> &m, const L &U, const L &V, const L &W,
                                      const L &N, long long c, int i, int j, int k) {
  const T h = (T)0.5;
  T uc = U(c, 0, 0, 0), ue = U(c, 1, 0, 0), uw = U(c, -1, 0, 0);
  T un = U(c, 0, 1, 0), us = U(c, 0, -1, 0), ut = U(c, 0, 0, 1), ub = U(c, 0, 0, -1);
  T a = h * (uc + ue), b = h * (uw + uc);
  T r = -qdiv(a * a - b * b, m.xC[i], m.xrC[i]);
  T t1 = (m.w0[j] * uc + m.w1[j] * un) * h * (V(c, 0, 0, 0) + V(c, 1, 0, 0));
  T t2 = (m.w0[j - 1] * us + m.w1[j - 1] * uc) * h * (V(c, 0, -1, 0) + V(c, 1, -1, 0));
  r = r - qdiv(t1 - t2, m.yF[j], m.yrF[j]);
  T t3 = h * (uc + ut) * h * (W(c, 0, 0, 0) + W(c, 1, 0, 0));
  T t4 = h * (ub + uc) * h * (W(c, 0, 0, -1) + W(c, 1, 0, -1));
  r = r - qdiv(t3 - t4, m.zF[k], m.zrF[k]);
  if (!LES) {
    T vx = qdiv(m.xrF[i + 1] * (ue - uc) - m.xrF[i] * (uc - uw), m.xC[i], m.xrC[i]);
    T vy = qdiv(qdiv(un - uc, m.yC[j], m.yrC[j]) - qdiv(uc - us, m.yC[j - 1], m.yrC[j - 1]), m.yF[j], m.yrF[j]);
    T vz = qdiv(m.zrC[k] * (ut - uc) - m.zrC[k - 1] * (uc - ub), m.zF[k], m.zrF[k]);
    r = r + m.dpdx + m.nu * (vx + vy + vz);
  } else {
    const T q = (T)0.25;
    T n0 = N(c, 0, 0, 0), nE = N(c, 1, 0, 0);
    T nu_x1 = m.nu + n0, nu_x2 = m.nu + nE;
    T nu_y1 = m.nu + h * (m.w0[j - 1] * N(c, 0, -1, 0) + m.w1[j - 1] * n0 + m.w0[j - 1] * N(c, 1, -1, 0) + m.w1[j - 1] * nE);
    T nu_y2 = m.nu + h * (m.w0[j] * n0 + m.w1[j] * N(c, 0, 1, 0) + m.w0[j] * nE + m.w1[j] * N(c, 1, 1, 0));
    T nu_z1 = m.nu + q * (n0 + N(c, 0, 0, -1) + nE + N(c, 1, 0, -1));
    T nu_z2 = m.nu + q * (n0 + N(c, 0, 0, 1) + nE + N(c, 1, 0, 1));
    T t2p = qdiv(un - uc, m.yC[j], m.yrC[j]);
    T t2m = qdiv(uc - us, m.yC[j - 1], m.yrC[j - 1]);
    r = r + m.dpdx +
        qdiv(qdiv(nu_x2, m.xF[i + 1], m.xrF[i + 1]) * (ue - uc) - qdiv(nu_x1, m.xF[i], m.xrF[i]) * (uc - uw), m.xC[i], m.xrC[i]) +
        qdiv(nu_y2 * t2p - nu_y1 * t2m, m.yF[j], m.yrF[j]) +
        qdiv(qdiv(nu_z2, m.zC[k], m.zrC[k]) * (ut - uc) - qdiv(nu_z1, m.zC[k - 1], m.zrC[k - 1]) * (uc - ub), m.zF[k], m.zrF[k]);
  }
  return r;
}

// RHS of v at (i,j,k), equations.f90:188-227 (DNS) / :238-266 (LES)
template <typename T, bool LES, typename L = Ld<T>>
__device__ __forceinline__ T rhs_v_at(const Geo &g, const MetT<T> &m, const L &U, const L &V, const L &W,
                                      const L &N, long long c, int i, int j, int k) {
  const T h = (T)0.5;
  T vc = V(c, 0, 0, 0), ve = V(c, 1, 0, 0), vw = V(c, -1, 0, 0);
  T vn = V(c, 0, 1, 0), vs = V(c, 0, -1, 0), vt = V(c, 0, 0, 1), vb = V(c, 0, 0, -1);
  T a = h * (vc + vn), b = h * (vs + vc);
  T r = -qdiv(a * a - b * b, m.yC[j], m.yrC[j]);
  T t1 = (m.w0[j] * U(c, 0, 0, 0) + m.w1[j] * U(c, 0, 1, 0)) * h * (vc + ve);
  T t2 = (m.w0[j] * U(c, -1, 0, 0) + m.w1[j] * U(c, -1, 1, 0)) * h * (vw + vc);
  r = r - qdiv(t1 - t2, m.xF[i], m.xrF[i]);
  T t3 = h * (vc + vt) * (m.w0[j] * W(c, 0, 0, 0) + m.w1[j] * W(c, 0, 1, 0));
  T t4 = h * (vb + vc) * (m.w0[j] * W(c, 0, 0, -1) + m.w1[j] * W(c, 0, 1, -1));
  r = r - qdiv(t3 - t4, m.zF[k], m.zrF[k]);
  if (!LES) {
    T vx = qdiv(m.xrC[i] * (ve - vc) - m.xrC[i - 1] * (vc - vw), m.xF[i], m.xrF[i]);
    T vy = qdiv(m.yrF[j + 1] * (vn - vc) - m.yrF[j] * (vc - vs), m.yC[j], m.yrC[j]);
    T vz = qdiv(m.zrC[k] * (vt - vc) - m.zrC[k - 1] * (vc - vb), m.zF[k], m.zrF[k]);
    r = r + m.nu * (vx + vy + vz);
  } else {
    T n0 = N(c, 0, 0, 0), nN = N(c, 0, 1, 0);
    T nu_x1 = m.nu + h * (m.w0[j] * N(c, -1, 0, 0) + m.w1[j] * N(c, -1, 1, 0) + m.w0[j] * n0 + m.w1[j] * nN);
    T nu_x2 = m.nu + h * (m.w0[j] * n0 + m.w1[j] * nN + m.w0[j] * N(c, 1, 0, 0) + m.w1[j] * N(c, 1, 1, 0));
    T nu_y1 = m.nu + n0, nu_y2 = m.nu + nN;
    T nu_z1 = m.nu + h * (m.w0[j] * N(c, 0, 0, -1) + m.w1[j] * N(c, 0, 1, -1) + m.w0[j] * n0 + m.w1[j] * nN);
    T nu_z2 = m.nu + h * (m.w0[j] * n0 + m.w1[j] * nN + m.w0[j] * N(c, 0, 0, 1) + m.w1[j] * N(c, 0, 1, 1));
    r = r + m.xrF[i] * (qdiv(nu_x2, m.xC[i], m.xrC[i]) * (ve - vc) - qdiv(nu_x1, m.xC[i - 1], m.xrC[i - 1]) * (vc - vw)) +
        m.yrC[j] * (qdiv(nu_y2, m.yF[j + 1], m.yrF[j + 1]) * (vn - vc) - qdiv(nu_y1, m.yF[j], m.yrF[j]) * (vc - vs)) +
        m.zrF[k] * (qdiv(nu_z2, m.zC[k], m.zrC[k]) * (vt - vc) - qdiv(nu_z1, m.zC[k - 1], m.zrC[k - 1]) * (vc - vb));
  }
  return r;
}

// RHS of w at (i,j,k), equations.f90:328-363 (DNS) / :383-401 (LES)
template <typename T, bool LES, typename L = Ld<T>>
__device__ __forceinline__ T rhs_w_at(const Geo &g, const MetT<T> &m, const L &U, const L &V, const L &W,
                                      const L &N, long long c, int i, int j, int k) {
  const T h = (T)0.5;
  T wc = W(c, 0, 0, 0), we = W(c, 1, 0, 0), ww = W(c, -1, 0, 0);
  T wn = W(c, 0, 1, 0), ws = W(c, 0, -1, 0), wt = W(c, 0, 0, 1), wb = W(c, 0, 0, -1);
  T a = h * (wc + wt), b = h * (wb + wc);
  T r = -qdiv(a * a - b * b, m.zC[k], m.zrC[k]);
  T t1 = h * (U(c, 0, 0, 0) + U(c, 0, 0, 1)) * h * (wc + we);
  T t2 = h * (U(c, -1, 0, 0) + U(c, -1, 0, 1)) * h * (ww + wc);
  r = r - qdiv(t1 - t2, m.xF[i], m.xrF[i]);
  T t3 = h * (V(c, 0, 0, 0) + V(c, 0, 0, 1)) * (m.w0[j] * wc + m.w1[j] * wn);
  T t4 = h * (V(c, 0, -1, 0) + V(c, 0, -1, 1)) * (m.w0[j - 1] * ws + m.w1[j - 1] * wc);
  r = r - qdiv(t3 - t4, m.yF[j], m.yrF[j]);
  if (!LES) {
    T vx = qdiv(m.xrC[i] * (we - wc) - m.xrC[i - 1] * (wc - ww), m.xF[i], m.xrF[i]);
    T vy = qdiv(qdiv(wn - wc, m.yC[j], m.yrC[j]) - qdiv(wc - ws, m.yC[j - 1], m.yrC[j - 1]), m.yF[j], m.yrF[j]);
    T vz = qdiv(m.zrF[k + 1] * (wt - wc) - m.zrF[k] * (wc - wb), m.zC[k], m.zrC[k]);
    r = r + m.dpdz + m.nu * (vx + vy + vz);
  } else {
    const T q = (T)0.25;
    T n0 = N(c, 0, 0, 0), nT = N(c, 0, 0, 1);
    T nu_x1 = m.nu + q * (n0 + nT + N(c, -1, 0, 0) + N(c, -1, 0, 1));
    T nu_x2 = m.nu + q * (n0 + nT + N(c, 1, 0, 0) + N(c, 1, 0, 1));
    T nu_y1 = m.nu + h * (m.w0[j - 1] * N(c, 0, -1, 0) + m.w1[j - 1] * n0 + m.w0[j - 1] * N(c, 0, -1, 1) + m.w1[j - 1] * nT);
    T nu_y2 = m.nu + h * (m.w0[j] * n0 + m.w1[j] * N(c, 0, 1, 0) + m.w0[j] * nT + m.w1[j] * N(c, 0, 1, 1));
    T nu_z1 = m.nu + n0, nu_z2 = m.nu + nT;
    T t2p = qdiv(wn - wc, m.yC[j], m.yrC[j]);
    T t2m = qdiv(wc - ws, m.yC[j - 1], m.yrC[j - 1]);
    r = r + m.dpdz +
        qdiv(qdiv(nu_x2, m.xC[i], m.xrC[i]) * (we - wc) - qdiv(nu_x1, m.xC[i - 1], m.xrC[i - 1]) * (wc - ww), m.xF[i], m.xrF[i]) +
        qdiv(nu_y2 * t2p - nu_y1 * t2m, m.yF[j], m.yrF[j]) +
        qdiv(qdiv(nu_z2, m.zF[k + 1], m.zrF[k + 1]) * (wt - wc) - qdiv(nu_z1, m.zF[k], m.zrF[k]) * (wc - wb), m.zC[k], m.zrC[k]);
  }
  return r;
}

// ---------------------------------------------------------------------------
// RHS + RK update.  MODE 0: store the RHS only (compute_rhs_u/v/w).
// MODE 1: U = Uo + (dt*c1)*F, F stored as F1 (first substep; Euler).
// MODE 2: U = Uo + dt*(c1*F1 + c2*F)        (RK3 s2, RK2 s2).
// MODE 3: U = Uo + dt*(c1*F1 + c2*F)        (RK3 s3, where rk_coef(3,2)=0 so
//         the F2 term contributes exactly zero and F2 is never stored).
// Threads cover the union of the three interior ranges, i=2..nx, j=2..ny,
// k=2..nz, each thread marching through a chunk of k-planes.
// ---------------------------------------------------------------------------
template <typename T, int MODE, bool LES>
__global__ void __launch_bounds__(256) k_rhs_rk(Geo g, MetT<T> m, const T *__restrict__ U, const T *__restrict__ V,
                                                const T *__restrict__ W, const T *__restrict__ nut,
                                                const T *__restrict__ Uo, const T *__restrict__ Vo,
                                                const T *__restrict__ Wo, T *__restrict__ F1u, T *__restrict__ F1v,
                                                T *__restrict__ F1w, T *__restrict__ Un, T *__restrict__ Vn,
                                                T *__restrict__ Wn, const Scalars *__restrict__ sc, double c1,
                                                double c2, int kchunk) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  if (i > g.nx || j > g.ny) return;
  const int k0 = blockIdx.z * kchunk + 2;
  const int k1 = min(k0 + kchunk - 1, g.nz);
  const Ld<T> LU{U, 1, g.px, g.plane}, LV{V, 1, g.px, g.plane}, LW{W, 1, g.px, g.plane}, LN{nut, 1, g.px, g.plane};
  double dt = 0.0;
  if (MODE != 0) dt = sc->dt;
  // coefficient products in FP64, exactly as the source multiplies them
  const T cdt1 = (T)(dt * c1);
  const T tdt = (T)dt, tc1 = (T)c1, tc2 = (T)c2;
  const bool du = (i <= g.nx - 1), dv = (j <= g.ny - 1);
  for (int k = k0; k <= k1; ++k) {
    const long long c = bidx(g, i, j, k);
    if (du) {
      T f = (i == g.nx - 1) ? (T)0 : rhs_u_at<T, LES>(g, m, LU, LV, LW, LN, c, i, j, k);
      if (MODE == 0) F1u[c] = f;
      else if (MODE == 1) { F1u[c] = f; Un[c] = Uo[c] + cdt1 * f; }
      else Un[c] = Uo[c] + tdt * (tc1 * F1u[c] + tc2 * f);
    }
    if (dv) {
      T f = (i == g.nx) ? (T)0 : rhs_v_at<T, LES>(g, m, LU, LV, LW, LN, c, i, j, k);
      if (MODE == 0) F1v[c] = f;
      else if (MODE == 1) { F1v[c] = f; Vn[c] = Vo[c] + cdt1 * f; }
      else Vn[c] = Vo[c] + tdt * (tc1 * F1v[c] + tc2 * f);
    }
    if (k <= g.nz - 1) {
      T f = (i == g.nx) ? (T)0 : rhs_w_at<T, LES>(g, m, LU, LV, LW, LN, c, i, j, k);
      if (MODE == 0) F1w[c] = f;
      else if (MODE == 1) { F1w[c] = f; Wn[c] = Wo[c] + cdt1 * f; }
      else Wn[c] = Wo[c] + tdt * (tc1 * F1w[c] + tc2 * f);
    }
  }
}

// ---------------------------------------------------------------------------
// DNS form of the same kernel: each thread owns one (i,j) column and marches
// up a chunk of k-planes with a register window over k-1, k, k+1, so a plane
// step loads 17 field values instead of 27; the x and y metric values are
// loaded once per thread and the z ones once per plane.  Expressions are
// those of rhs_*_at above, term for term.
// ---------------------------------------------------------------------------
template <typename T, int MODE>
__global__ void __launch_bounds__(256) k_rhs_rk_dns(Geo g, MetT<T> m, const T *__restrict__ U,
                                                    const T *__restrict__ V, const T *__restrict__ W,
                                                    const T *__restrict__ Uo, const T *__restrict__ Vo,
                                                    const T *__restrict__ Wo, T *__restrict__ F1u,
                                                    T *__restrict__ F1v, T *__restrict__ F1w, T *__restrict__ Un,
                                                    T *__restrict__ Vn, T *__restrict__ Wn,
                                                    const Scalars *__restrict__ sc, double c1, double c2,
                                                    int kchunk) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  if (i > g.nx || j > g.ny) return;
  const int k0 = blockIdx.z * kchunk + 2;
  const int k1 = min(k0 + kchunk - 1, g.nz);
  if (k0 > k1) return;
  const long long px = g.px, pl = g.plane;
  double dt = 0.0;
  if (MODE != 0) dt = sc->dt;
  const T cdt1 = (T)(dt * c1);
  const T tdt = (T)dt, tc1 = (T)c1, tc2 = (T)c2;
  const bool du = (i <= g.nx - 1), dv = (j <= g.ny - 1);
  const bool zu = (i == g.nx - 1), zvw = (i == g.nx);
  const T h = (T)0.5;
  // per-thread metrics (x: i, y: j)
  const T xC = m.xC[i], xrC = m.xrC[i], xF = m.xF[i], xrF = m.xrF[i], xrFp = m.xrF[i + 1], xrCm = m.xrC[i - 1];
  const T yF = m.yF[j], yrF = m.yrF[j], yC = m.yC[j], yrC = m.yrC[j], yCm = m.yC[j - 1], yrCm = m.yrC[j - 1];
  const T yrFp = m.yrF[j + 1], w0 = m.w0[j], w1 = m.w1[j], w0m = m.w0[j - 1], w1m = m.w1[j - 1];
  const T nu = m.nu, dpdx = m.dpdx, dpdz = m.dpdz;
  long long c = bidx(g, i, j, k0);
  // window at k0
  T uc = __ldg(U + c), ue = __ldg(U + c + 1), uw = __ldg(U + c - 1), un = __ldg(U + c + px), us = __ldg(U + c - px);
  T ut = __ldg(U + c + pl), ub = __ldg(U + c - pl), unw = __ldg(U + c - 1 + px), utw = __ldg(U + c - 1 + pl);
  T vc = __ldg(V + c), ve = __ldg(V + c + 1), vw = __ldg(V + c - 1), vn = __ldg(V + c + px), vs = __ldg(V + c - px);
  T vt = __ldg(V + c + pl), vb = __ldg(V + c - pl), vse = __ldg(V + c + 1 - px), vst = __ldg(V + c - px + pl);
  T wc = __ldg(W + c), we = __ldg(W + c + 1), ww = __ldg(W + c - 1), wn = __ldg(W + c + px), ws = __ldg(W + c - px);
  T wt = __ldg(W + c + pl), wb = __ldg(W + c - pl), web = __ldg(W + c + 1 - pl), wnb = __ldg(W + c + px - pl);
  for (int k = k0;; ++k) {
    const T zF = m.zF[k], zrF = m.zrF[k], zC = m.zC[k], zrC = m.zrC[k], zrCm = m.zrC[k - 1], zrFp = m.zrF[k + 1];
    if (du) {
      T f = 0;
      if (!zu) {
        const T a = h * (uc + ue), b = h * (uw + uc);
        T r = -qdiv(a * a - b * b, xC, xrC);
        const T t1 = (w0 * uc + w1 * un) * h * (vc + ve);
        const T t2 = (w0m * us + w1m * uc) * h * (vs + vse);
        r = r - qdiv(t1 - t2, yF, yrF);
        const T t3 = h * (uc + ut) * h * (wc + we);
        const T t4 = h * (ub + uc) * h * (wb + web);
        r = r - qdiv(t3 - t4, zF, zrF);
        const T vx = qdiv(xrFp * (ue - uc) - xrF * (uc - uw), xC, xrC);
        const T vy = qdiv(qdiv(un - uc, yC, yrC) - qdiv(uc - us, yCm, yrCm), yF, yrF);
        const T vz = qdiv(zrC * (ut - uc) - zrCm * (uc - ub), zF, zrF);
        f = r + dpdx + nu * (vx + vy + vz);
      }
      if (MODE == 0) F1u[c] = f;
      else if (MODE == 1) { F1u[c] = f; Un[c] = Uo[c] + cdt1 * f; }
      else Un[c] = Uo[c] + tdt * (tc1 * F1u[c] + tc2 * f);
    }
    if (dv) {
      T f = 0;
      if (!zvw) {
        const T a = h * (vc + vn), b = h * (vs + vc);
        T r = -qdiv(a * a - b * b, yC, yrC);
        const T t1 = (w0 * uc + w1 * un) * h * (vc + ve);
        const T t2 = (w0 * uw + w1 * unw) * h * (vw + vc);
        r = r - qdiv(t1 - t2, xF, xrF);
        const T t3 = h * (vc + vt) * (w0 * wc + w1 * wn);
        const T t4 = h * (vb + vc) * (w0 * wb + w1 * wnb);
        r = r - qdiv(t3 - t4, zF, zrF);
        const T vx = qdiv(xrC * (ve - vc) - xrCm * (vc - vw), xF, xrF);
        const T vy = qdiv(yrFp * (vn - vc) - yrF * (vc - vs), yC, yrC);
        const T vz = qdiv(zrC * (vt - vc) - zrCm * (vc - vb), zF, zrF);
        f = r + nu * (vx + vy + vz);
      }
      if (MODE == 0) F1v[c] = f;
      else if (MODE == 1) { F1v[c] = f; Vn[c] = Vo[c] + cdt1 * f; }
      else Vn[c] = Vo[c] + tdt * (tc1 * F1v[c] + tc2 * f);
    }
    if (k <= g.nz - 1) {
      T f = 0;
      if (!zvw) {
        const T a = h * (wc + wt), b = h * (wb + wc);
        T r = -qdiv(a * a - b * b, zC, zrC);
        const T t1 = h * (uc + ut) * h * (wc + we);
        const T t2 = h * (uw + utw) * h * (ww + wc);
        r = r - qdiv(t1 - t2, xF, xrF);
        const T t3 = h * (vc + vt) * (w0 * wc + w1 * wn);
        const T t4 = h * (vs + vst) * (w0m * ws + w1m * wc);
        r = r - qdiv(t3 - t4, yF, yrF);
        const T vx = qdiv(xrC * (we - wc) - xrCm * (wc - ww), xF, xrF);
        const T vy = qdiv(qdiv(wn - wc, yC, yrC) - qdiv(wc - ws, yCm, yrCm), yF, yrF);
        const T vz = qdiv(zrFp * (wt - wc) - zrF * (wc - wb), zC, zrC);
        f = r + dpdz + nu * (vx + vy + vz);
      }
      if (MODE == 0) F1w[c] = f;
      else if (MODE == 1) { F1w[c] = f; Wn[c] = Wo[c] + cdt1 * f; }
      else Wn[c] = Wo[c] + tdt * (tc1 * F1w[c] + tc2 * f);
    }
    if (k == k1) break;
    // slide the window to k+1
    c += pl;
    ub = uc; uc = ut; uw = utw;
    vb = vc; vc = vt; vs = vst;
    wb = wc; wc = wt; web = we; wnb = wn;
    ut = __ldg(U + c + pl); utw = __ldg(U + c - 1 + pl);
    ue = __ldg(U + c + 1); un = __ldg(U + c + px); us = __ldg(U + c - px); unw = __ldg(U + c - 1 + px);
    vt = __ldg(V + c + pl); vst = __ldg(V + c - px + pl);
    ve = __ldg(V + c + 1); vw = __ldg(V + c - 1); vn = __ldg(V + c + px); vse = __ldg(V + c + 1 - px);
    wt = __ldg(W + c + pl);
    we = __ldg(W + c + 1); ww = __ldg(W + c - 1); wn = __ldg(W + c + px); ws = __ldg(W + c - px);
  }
}

// ---------------------------------------------------------------------------
// DNS form with two x-points per thread (i0 = 2+2q and i0+1, one aligned
// 2-vector in the box).  The face fluxes are evaluated once and shared:
//   X(i)   = h*(U(i)+U(i+1))                    u x-advection (a and b terms)
//   Fxy(i) = (w0*U(i,j)+w1*U(i,j+1))*h*(V(i)+V(i+1))   u's t1, v's t1; v's t2 = Fxy(i-1)
//   Fxz(i) = h*(U(k)+U(k+1))*h*(W(i)+W(i+1))   u's t3, w's t1; w's t2 = Fxz(i-1)
//   Fyz    = h*(V(k)+V(k+1))*(w0*W(j)+w1*W(j+1))      v's t3, w's t3
// and the k-1 face values (u's t4, v's t4, w's advection b term and the three
// lower z differences) are carried from the previous plane, where they were
// the upper face values.  Every shared or carried value is the same
// expression, in the same order, as the term it replaces in rhs_*_at.  The
// rows of plane k+2 and the Uo/F1 values of plane k+1 are fetched one plane
// ahead so their DRAM latency overlaps a plane of arithmetic.
// ---------------------------------------------------------------------------
// w0*a + w1*b with both products rounded (no contraction), so that a carried
// Fyz and one formed afresh at the first plane of a chunk round alike and the
// chunk length does not change results
__device__ __forceinline__ float wsum(float w0, float a, float w1, float b) {
  return __fadd_rn(__fmul_rn(w0, a), __fmul_rn(w1, b));
}
__device__ __forceinline__ double wsum(double w0, double a, double w1, double b) {
  return __dadd_rn(__dmul_rn(w0, a), __dmul_rn(w1, b));
}

template <typename T> struct Row4 { T m, a, b, p; };  // i0-1 .. i0+2
template <typename T> struct Row3 { T m, a, b; };     // i0-1 .. i0+1
template <typename T> struct Row2 { T a, b; };        // i0 .. i0+1

template <typename T>
__device__ __forceinline__ Row2<T> ld2(const T *__restrict__ p, long long c) {
  typedef typename vec2<T>::type T2;
  const T2 v = __ldg(reinterpret_cast<const T2 *>(p + c));
  return Row2<T>{v.x, v.y};
}
template <typename T>
__device__ __forceinline__ Row3<T> ld3(const T *__restrict__ p, long long c) {
  const Row2<T> v = ld2(p, c);
  return Row3<T>{__ldg(p + c - 1), v.a, v.b};
}
// stores the points of the pair that lie in the update range (sa implies
// nothing about sb, but sb implies sa since b = a+1 and ranges are prefixes)
template <typename T>
__device__ __forceinline__ void st2(T *__restrict__ p, long long c, T fa, T fb, bool sa, bool sb) {
  typedef typename vec2<T>::type T2;
  if (sb) {
    T2 v;
    v.x = fa;
    v.y = fb;
    *reinterpret_cast<T2 *>(p + c) = v;
  } else if (sa) {
    p[c] = fa;
  }
}

template <typename T, int MODE>
__device__ __forceinline__ void rk_store2(T *__restrict__ F1, T *__restrict__ Un, long long c, Row2<T> f,
                                          Row2<T> o, Row2<T> f1, T cdt1, T tdt, T tc1, T tc2, bool sa, bool sb) {
  if (MODE == 0) {
    st2(F1, c, f.a, f.b, sa, sb);
  } else if (MODE == 1) {
    st2(F1, c, f.a, f.b, sa, sb);
    st2(Un, c, o.a + cdt1 * f.a, o.b + cdt1 * f.b, sa, sb);
  } else {
    st2(Un, c, o.a + tdt * (tc1 * f1.a + tc2 * f.a), o.b + tdt * (tc1 * f1.b + tc2 * f.b), sa, sb);
  }
}

template <typename T, int MODE>
__global__ void __launch_bounds__(256) k_rhs_rk_pair(Geo g, MetT<T> m, const T *__restrict__ U,
                                                     const T *__restrict__ V, const T *__restrict__ W,
                                                     const T *__restrict__ Uo, const T *__restrict__ Vo,
                                                     const T *__restrict__ Wo, T *__restrict__ F1u,
                                                     T *__restrict__ F1v, T *__restrict__ F1w, T *__restrict__ Un,
                                                     T *__restrict__ Vn, T *__restrict__ Wn,
                                                     const Scalars *__restrict__ sc, double c1, double c2,
                                                     int kchunk) {
  const int i0 = 2 + 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  if (i0 > g.nx || j > g.ny) return;
  const int k0 = blockIdx.z * kchunk + 2;
  const int k1 = min(k0 + kchunk - 1, g.nz);
  if (k0 > k1) return;
  const long long px = g.px, pl = g.plane;
  double dt = 0.0;
  if (MODE != 0) dt = sc->dt;
  const T cdt1 = (T)(dt * c1);
  const T tdt = (T)dt, tc1 = (T)c1, tc2 = (T)c2;
  const int ib = i0 + 1;
  // store ranges: u at i <= nx-1 (zero at nx-1), v and w at i <= nx (zero at nx)
  const bool su_a = i0 <= g.nx - 1, su_b = ib <= g.nx - 1;
  const bool sv_a = true, sv_b = ib <= g.nx;
  const bool dv = (j <= g.ny - 1);
  const bool zu_a = (i0 == g.nx - 1), zu_b = (ib == g.nx - 1);
  const bool zx_a = (i0 == g.nx), zx_b = (ib == g.nx);
  const T h = (T)0.5;
  // x metrics of both points (tables run to nx+2, so i0+2 is in range)
  const T xC_a = m.xC[i0], xrC_a = m.xrC[i0], xC_b = m.xC[ib], xrC_b = m.xrC[ib];
  const T xF_a = m.xF[i0], xrF_a = m.xrF[i0], xF_b = m.xF[ib], xrF_b = m.xrF[ib];
  const T xrF_p = m.xrF[i0 + 2], xrC_m = m.xrC[i0 - 1];
  const T yF = m.yF[j], yrF = m.yrF[j], yC = m.yC[j], yrC = m.yrC[j], yCm = m.yC[j - 1], yrCm = m.yrC[j - 1];
  const T yrFp = m.yrF[j + 1], w0 = m.w0[j], w1 = m.w1[j], w0m = m.w0[j - 1], w1m = m.w1[j - 1];
  const T nu = m.nu, dpdx = m.dpdx, dpdz = m.dpdz;
  long long c = bidx(g, i0, j, k0);
  // window at k0: rows of planes k0 (c), k0+1 (t), and the k0-1 values the
  // carried terms start from
  Row4<T> uc, vc, wc;
  {
    const Row3<T> u3 = ld3(U, c), v3 = ld3(V, c), w3 = ld3(W, c);
    uc = Row4<T>{u3.m, u3.a, u3.b, __ldg(U + c + 2)};
    vc = Row4<T>{v3.m, v3.a, v3.b, __ldg(V + c + 2)};
    wc = Row4<T>{w3.m, w3.a, w3.b, __ldg(W + c + 2)};
  }
  Row3<T> un = ld3(U, c + px), ut = ld3(U, c + pl);
  Row2<T> us = ld2(U, c - px);
  Row2<T> vn = ld2(V, c + px), vt = ld2(V, c + pl), vst = ld2(V, c - px + pl);
  Row2<T> vs = ld2(V, c - px);
  T vs_p = __ldg(V + c - px + 2);
  Row2<T> wn = ld2(W, c + px), ws = ld2(W, c - px), wt = ld2(W, c + pl);
  // carried k-1 face terms
  Row2<T> FxzB, FyzB, dUz, dVz, dWz, WbA;
  {
    const Row2<T> ub = ld2(U, c - pl), vb = ld2(V, c - pl), wb = ld2(W, c - pl), wnb = ld2(W, c + px - pl);
    const T wb_p = __ldg(W + c + 2 - pl);
    FxzB.a = h * (ub.a + uc.a) * h * (wb.a + wb.b);
    FxzB.b = h * (ub.b + uc.b) * h * (wb.b + wb_p);
    FyzB.a = h * (vb.a + vc.a) * wsum(w0, wb.a, w1, wnb.a);
    FyzB.b = h * (vb.b + vc.b) * wsum(w0, wb.b, w1, wnb.b);
    dUz = Row2<T>{uc.a - ub.a, uc.b - ub.b};
    dVz = Row2<T>{vc.a - vb.a, vc.b - vb.b};
    dWz = Row2<T>{wc.a - wb.a, wc.b - wb.b};
    WbA = Row2<T>{h * (wb.a + wc.a), h * (wb.b + wc.b)};
  }
  Row2<T> oU{}, oV{}, oW{}, fU{}, fV{}, fW{};
  if (MODE != 0 && MODE != 1) { fU = ld2(F1u, c); fV = ld2(F1v, c); fW = ld2(F1w, c); }
  if (MODE != 0) { oU = ld2(Uo, c); oV = ld2(Vo, c); oW = ld2(Wo, c); }
  for (int k = k0;; ++k) {
    // fetch ahead: rows of plane k+2 and Uo/F1 of plane k+1
    const bool more = k < k1;
    Row3<T> ut2{};
    Row2<T> vt2{}, vst2{}, wt2{}, oU2{}, oV2{}, oW2{}, fU2{}, fV2{}, fW2{};
    if (more) {
      const long long c2p = c + 2 * pl, c1p = c + pl;
      ut2 = ld3(U, c2p);
      vt2 = ld2(V, c2p);
      vst2 = ld2(V, c2p - px);
      wt2 = ld2(W, c2p);
      if (MODE != 0) { oU2 = ld2(Uo, c1p); oV2 = ld2(Vo, c1p); oW2 = ld2(Wo, c1p); }
      if (MODE != 0 && MODE != 1) { fU2 = ld2(F1u, c1p); fV2 = ld2(F1v, c1p); fW2 = ld2(F1w, c1p); }
    }
    const T zF = m.zF[k], zrF = m.zrF[k], zC = m.zC[k], zrC = m.zrC[k], zrCm = m.zrC[k - 1], zrFp = m.zrF[k + 1];
    // shared face fluxes of this plane
    const T Xm = h * (uc.m + uc.a), Xa = h * (uc.a + uc.b), Xb = h * (uc.b + uc.p);
    const T Fxy_m = (w0 * uc.m + w1 * un.m) * h * (vc.m + vc.a);
    const T Fxy_a = (w0 * uc.a + w1 * un.a) * h * (vc.a + vc.b);
    const T Fxy_b = (w0 * uc.b + w1 * un.b) * h * (vc.b + vc.p);
    const T Fxz_m = h * (uc.m + ut.m) * h * (wc.m + wc.a);
    const T Fxz_a = h * (uc.a + ut.a) * h * (wc.a + wc.b);
    const T Fxz_b = h * (uc.b + ut.b) * h * (wc.b + wc.p);
    const T Fyz_a = h * (vc.a + vt.a) * wsum(w0, wc.a, w1, wn.a);
    const T Fyz_b = h * (vc.b + vt.b) * wsum(w0, wc.b, w1, wn.b);
    const Row2<T> dUt{ut.a - uc.a, ut.b - uc.b}, dVt{vt.a - vc.a, vt.b - vc.b}, dWt{wt.a - wc.a, wt.b - wc.b};
    // u
    {
      Row2<T> f{(T)0, (T)0};
      T r = -qdiv(Xa * Xa - Xm * Xm, xC_a, xrC_a);
      r = r - qdiv(Fxy_a - (w0m * us.a + w1m * uc.a) * h * (vs.a + vs.b), yF, yrF);
      r = r - qdiv(Fxz_a - FxzB.a, zF, zrF);
      T vx = qdiv(xrF_b * (uc.b - uc.a) - xrF_a * (uc.a - uc.m), xC_a, xrC_a);
      T vy = qdiv(qdiv(un.a - uc.a, yC, yrC) - qdiv(uc.a - us.a, yCm, yrCm), yF, yrF);
      T vz = qdiv(zrC * dUt.a - zrCm * dUz.a, zF, zrF);
      if (!zu_a) f.a = r + dpdx + nu * (vx + vy + vz);
      r = -qdiv(Xb * Xb - Xa * Xa, xC_b, xrC_b);
      r = r - qdiv(Fxy_b - (w0m * us.b + w1m * uc.b) * h * (vs.b + vs_p), yF, yrF);
      r = r - qdiv(Fxz_b - FxzB.b, zF, zrF);
      vx = qdiv(xrF_p * (uc.p - uc.b) - xrF_b * (uc.b - uc.a), xC_b, xrC_b);
      vy = qdiv(qdiv(un.b - uc.b, yC, yrC) - qdiv(uc.b - us.b, yCm, yrCm), yF, yrF);
      vz = qdiv(zrC * dUt.b - zrCm * dUz.b, zF, zrF);
      if (!zu_b) f.b = r + dpdx + nu * (vx + vy + vz);
      rk_store2<T, MODE>(F1u, Un, c, f, oU, fU, cdt1, tdt, tc1, tc2, su_a, su_b);
    }
    // v
    if (dv) {
      Row2<T> f{(T)0, (T)0};
      T aa = h * (vc.a + vn.a), bb = h * (vs.a + vc.a);
      T r = -qdiv(aa * aa - bb * bb, yC, yrC);
      r = r - qdiv(Fxy_a - Fxy_m, xF_a, xrF_a);
      r = r - qdiv(Fyz_a - FyzB.a, zF, zrF);
      T vx = qdiv(xrC_a * (vc.b - vc.a) - xrC_m * (vc.a - vc.m), xF_a, xrF_a);
      T vy = qdiv(yrFp * (vn.a - vc.a) - yrF * (vc.a - vs.a), yC, yrC);
      T vz = qdiv(zrC * dVt.a - zrCm * dVz.a, zF, zrF);
      if (!zx_a) f.a = r + nu * (vx + vy + vz);
      aa = h * (vc.b + vn.b);
      bb = h * (vs.b + vc.b);
      r = -qdiv(aa * aa - bb * bb, yC, yrC);
      r = r - qdiv(Fxy_b - Fxy_a, xF_b, xrF_b);
      r = r - qdiv(Fyz_b - FyzB.b, zF, zrF);
      vx = qdiv(xrC_b * (vc.p - vc.b) - xrC_a * (vc.b - vc.a), xF_b, xrF_b);
      vy = qdiv(yrFp * (vn.b - vc.b) - yrF * (vc.b - vs.b), yC, yrC);
      vz = qdiv(zrC * dVt.b - zrCm * dVz.b, zF, zrF);
      if (!zx_b) f.b = r + nu * (vx + vy + vz);
      rk_store2<T, MODE>(F1v, Vn, c, f, oV, fV, cdt1, tdt, tc1, tc2, sv_a, sv_b);
    }
    // w
    Row2<T> WtA{h * (wc.a + wt.a), h * (wc.b + wt.b)};
    if (k <= g.nz - 1) {
      Row2<T> f{(T)0, (T)0};
      T r = -qdiv(WtA.a * WtA.a - WbA.a * WbA.a, zC, zrC);
      r = r - qdiv(Fxz_a - Fxz_m, xF_a, xrF_a);
      r = r - qdiv(Fyz_a - h * (vs.a + vst.a) * (w0m * ws.a + w1m * wc.a), yF, yrF);
      T vx = qdiv(xrC_a * (wc.b - wc.a) - xrC_m * (wc.a - wc.m), xF_a, xrF_a);
      T vy = qdiv(qdiv(wn.a - wc.a, yC, yrC) - qdiv(wc.a - ws.a, yCm, yrCm), yF, yrF);
      T vz = qdiv(zrFp * dWt.a - zrF * dWz.a, zC, zrC);
      if (!zx_a) f.a = r + dpdz + nu * (vx + vy + vz);
      r = -qdiv(WtA.b * WtA.b - WbA.b * WbA.b, zC, zrC);
      r = r - qdiv(Fxz_b - Fxz_a, xF_b, xrF_b);
      r = r - qdiv(Fyz_b - h * (vs.b + vst.b) * (w0m * ws.b + w1m * wc.b), yF, yrF);
      vx = qdiv(xrC_b * (wc.p - wc.b) - xrC_a * (wc.b - wc.a), xF_b, xrF_b);
      vy = qdiv(qdiv(wn.b - wc.b, yC, yrC) - qdiv(wc.b - ws.b, yCm, yrCm), yF, yrF);
      vz = qdiv(zrFp * dWt.b - zrF * dWz.b, zC, zrC);
      if (!zx_b) f.b = r + dpdz + nu * (vx + vy + vz);
      rk_store2<T, MODE>(F1w, Wn, c, f, oW, fW, cdt1, tdt, tc1, tc2, sv_a, sv_b);
    }
    if (!more) break;
    // carry the upper face terms down and slide the window to k+1
    FxzB = Row2<T>{Fxz_a, Fxz_b};
    FyzB = Row2<T>{Fyz_a, Fyz_b};
    dUz = dUt; dVz = dVt; dWz = dWt; WbA = WtA;
    c += pl;
    uc = Row4<T>{ut.m, ut.a, ut.b, __ldg(U + c + 2)};
    vc = Row4<T>{__ldg(V + c - 1), vt.a, vt.b, __ldg(V + c + 2)};
    wc = Row4<T>{__ldg(W + c - 1), wt.a, wt.b, __ldg(W + c + 2)};
    vs = vst;
    vs_p = __ldg(V + c - px + 2);
    un = ld3(U, c + px);
    us = ld2(U, c - px);
    vn = ld2(V, c + px);
    wn = ld2(W, c + px);
    ws = ld2(W, c - px);
    ut = ut2; vt = vt2; vst = vst2; wt = wt2;
    oU = oU2; oV = oV2; oW = oW2; fU = fU2; fV = fV2; fW = fW2;
  }
}

// ---------------------------------------------------------------------------
// FP32 DNS form with the two x-points of a thread packed: every operation on
// the pair (point i0 in .x, i0+1 in .y) is one FP32x2 instruction of sm_100
// (__fadd2_rn, __fmul2_rn, __ffma2_rn), each with its rounding written out,
// so a carried k-1 face term and one formed afresh at the first plane of a
// chunk round alike.  Loads, shared face fluxes, carried terms and the
// one-plane-ahead fetches are those of k_rhs_rk_pair; the x-shifted pairs
// (i0-1, i0) and (i0+1, i0+2) are assembled from the pair and the scalar
// neighbours.  The terms are those of rhs_*_at, grouped for fused
// multiply-adds: a*x - b*y as fma(a, x, -b*y).
// ---------------------------------------------------------------------------
namespace pk {
typedef float2 f2;
__device__ __forceinline__ f2 mk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ f2 sp(float a) { return make_float2(a, a); }
__device__ __forceinline__ f2 neg(f2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ f2 add(f2 a, f2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ f2 sub(f2 a, f2 b) { return __fadd2_rn(a, neg(b)); }
__device__ __forceinline__ f2 mul(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 fma(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ f2 lin(f2 a, f2 x, f2 b, f2 y) { return fma(a, x, mul(b, y)); }       // a x + b y
__device__ __forceinline__ f2 dif(f2 a, f2 x, f2 b, f2 y) { return fma(a, x, mul(neg(b), y)); }  // a x - b y
__device__ __forceinline__ f2 ld(const float *__restrict__ p, long long c) {
  return __ldg(reinterpret_cast<const float2 *>(p + c));
}
// the carried terms, formed by one expression whether carried or fresh
__device__ __forceinline__ f2 fxz(f2 H, f2 u0, f2 u1, f2 w0, f2 w1) { return mul(mul(H, add(u0, u1)), mul(H, add(w0, w1))); }
__device__ __forceinline__ f2 fyz(f2 H, f2 W0, f2 W1, f2 v0, f2 v1, f2 w, f2 wn) {
  return mul(mul(H, add(v0, v1)), lin(W0, w, W1, wn));
}
__device__ __forceinline__ void st(float *__restrict__ p, long long c, f2 f, bool sa, bool sb) {
  if (sb) *reinterpret_cast<f2 *>(p + c) = f;
  else if (sa) p[c] = f.x;
}
template <int MODE>
__device__ __forceinline__ void rk(float *__restrict__ F1, float *__restrict__ Un, long long c, f2 f, f2 o, f2 f1,
                                   f2 CDT1, f2 TDT, f2 TC1, f2 TC2, bool sa, bool sb) {
  if (MODE == 0) {
    st(F1, c, f, sa, sb);
  } else if (MODE == 1) {
    st(F1, c, f, sa, sb);
    st(Un, c, fma(CDT1, f, o), sa, sb);
  } else {
    st(Un, c, fma(TDT, fma(TC1, f1, mul(TC2, f)), o), sa, sb);
  }
}
}  // namespace pk

template <int MODE>
__global__ void __launch_bounds__(256, 2) k_rhs_rk_pk(Geo g, MetT<float> m, const float *__restrict__ U,
                                                   const float *__restrict__ V, const float *__restrict__ W,
                                                   const float *__restrict__ Uo, const float *__restrict__ Vo,
                                                   const float *__restrict__ Wo, float *__restrict__ F1u,
                                                   float *__restrict__ F1v, float *__restrict__ F1w,
                                                   float *__restrict__ Un, float *__restrict__ Vn,
                                                   float *__restrict__ Wn, const Scalars *__restrict__ sc, double c1,
                                                   double c2, int kchunk) {
  using namespace pk;
  const int i0 = 2 + 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  if (i0 > g.nx || j > g.ny) return;
  const int k0 = blockIdx.z * kchunk + 2;
  const int k1 = min(k0 + kchunk - 1, g.nz);
  if (k0 > k1) return;
  const long long px = g.px, pl = g.plane;
  double dt = 0.0;
  if (MODE != 0) dt = sc->dt;
  const f2 CDT1 = sp((float)(dt * c1)), TDT = sp((float)dt), TC1 = sp((float)c1), TC2 = sp((float)c2);
  const int ib = i0 + 1;
  const bool su_a = i0 <= g.nx - 1, su_b = ib <= g.nx - 1;
  const bool sv_a = true, sv_b = ib <= g.nx;
  const bool dv = (j <= g.ny - 1);
  const bool zu_a = (i0 == g.nx - 1), zu_b = (ib == g.nx - 1);
  const bool zx_a = (i0 == g.nx), zx_b = (ib == g.nx);
  const f2 H = sp(0.5f);
  const f2 XRC_P = mk(m.xrC[i0], m.xrC[ib]), XRF_P = mk(m.xrF[i0], m.xrF[ib]);
  const f2 XRF_R = mk(m.xrF[ib], m.xrF[i0 + 2]), XRC_L = mk(m.xrC[i0 - 1], m.xrC[i0]);
  const f2 YRF = sp(m.yrF[j]), YRC = sp(m.yrC[j]), YRCM = sp(m.yrC[j - 1]), YRFP = sp(m.yrF[j + 1]);
  const f2 W0 = sp(m.w0[j]), W1 = sp(m.w1[j]), W0M = sp(m.w0[j - 1]), W1M = sp(m.w1[j - 1]);
  const f2 NU = sp(m.nu), DPDX = sp(m.dpdx), DPDZ = sp(m.dpdz);
  long long c = bidx(g, i0, j, k0);
  // window at k0 (pairs P, scalar neighbours i0-1 and i0+2)
  float um = __ldg(U + c - 1), up = __ldg(U + c + 2);
  float vm = __ldg(V + c - 1), vp = __ldg(V + c + 2);
  float wm = __ldg(W + c - 1), wp = __ldg(W + c + 2);
  f2 uP = ld(U, c), vP = ld(V, c), wP = ld(W, c);
  float unm = __ldg(U + c + px - 1), utm = __ldg(U + c + pl - 1);
  f2 unP = ld(U, c + px), utP = ld(U, c + pl), usP = ld(U, c - px);
  f2 vnP = ld(V, c + px), vtP = ld(V, c + pl), vstP = ld(V, c - px + pl), vsP = ld(V, c - px);
  float vs_p = __ldg(V + c - px + 2);
  f2 wnP = ld(W, c + px), wsP = ld(W, c - px), wtP = ld(W, c + pl);
  f2 FxzB, FyzB, dUz, dVz, dWz, WbA;
  {
    const f2 ubP = ld(U, c - pl), vbP = ld(V, c - pl), wbP = ld(W, c - pl), wnbP = ld(W, c + px - pl);
    const float wb_p = __ldg(W + c + 2 - pl);
    FxzB = fxz(H, ubP, uP, wbP, mk(wbP.y, wb_p));
    FyzB = fyz(H, W0, W1, vbP, vP, wbP, wnbP);
    dUz = sub(uP, ubP);
    dVz = sub(vP, vbP);
    dWz = sub(wP, wbP);
    WbA = mul(H, add(wbP, wP));
  }
  f2 oU{}, oV{}, oW{}, fU{}, fV{}, fW{};
  if (MODE != 0 && MODE != 1) { fU = ld(F1u, c); fV = ld(F1v, c); fW = ld(F1w, c); }
  if (MODE != 0) { oU = ld(Uo, c); oV = ld(Vo, c); oW = ld(Wo, c); }
  for (int k = k0;; ++k) {
    const bool more = k < k1;
    float utm2 = 0.f;
    f2 utP2{}, vtP2{}, vstP2{}, wtP2{}, oU2{}, oV2{}, oW2{}, fU2{}, fV2{}, fW2{};
    if (more) {
      const long long c2p = c + 2 * pl, c1p = c + pl;
      utm2 = __ldg(U + c2p - 1);
      utP2 = ld(U, c2p);
      vtP2 = ld(V, c2p);
      vstP2 = ld(V, c2p - px);
      wtP2 = ld(W, c2p);
      if (MODE != 0) { oU2 = ld(Uo, c1p); oV2 = ld(Vo, c1p); oW2 = ld(Wo, c1p); }
      if (MODE != 0 && MODE != 1) { fU2 = ld(F1u, c1p); fV2 = ld(F1v, c1p); fW2 = ld(F1w, c1p); }
    }
    const f2 ZRF = sp(m.zrF[k]), ZRC = sp(m.zrC[k]), ZRCM = sp(m.zrC[k - 1]), ZRFP = sp(m.zrF[k + 1]);
    // x-shifted pairs
    const f2 uL = mk(um, uP.x), uR = mk(uP.y, up);
    const f2 vL = mk(vm, vP.x), vR = mk(vP.y, vp);
    const f2 wL = mk(wm, wP.x), wR = mk(wP.y, wp);
    // shared face fluxes of this plane
    const f2 XL = mul(H, add(uL, uP)), XR = mul(H, add(uP, uR));
    const f2 FxyP = mul(lin(W0, uP, W1, unP), mul(H, add(vP, vR)));
    const f2 FxyL = mul(lin(W0, uL, W1, mk(unm, unP.x)), mul(H, add(vL, vP)));
    const f2 FxzP = fxz(H, uP, utP, wP, wR);
    const f2 FxzL = fxz(H, uL, mk(utm, utP.x), wL, wP);
    const f2 FyzP = fyz(H, W0, W1, vP, vtP, wP, wnP);
    const f2 dUt = sub(utP, uP), dVt = sub(vtP, vP), dWt = sub(wtP, wP);
    const f2 WtA = mul(H, add(wP, wtP));
    // u
    {
      const f2 ax = mul(dif(XR, XR, XL, XL), XRC_P);
      const f2 ay = mul(sub(FxyP, mul(lin(W0M, usP, W1M, uP), mul(H, add(vsP, mk(vsP.y, vs_p))))), YRF);
      const f2 az = mul(sub(FxzP, FxzB), ZRF);
      const f2 vx = mul(dif(XRF_R, sub(uR, uP), XRF_P, sub(uP, uL)), XRC_P);
      const f2 vy = mul(dif(sub(unP, uP), YRC, sub(uP, usP), YRCM), YRF);
      const f2 vz = mul(dif(ZRC, dUt, ZRCM, dUz), ZRF);
      f2 f = fma(NU, add(add(vx, vy), vz), sub(DPDX, add(add(ax, ay), az)));
      if (zu_a) f.x = 0.f;
      if (zu_b) f.y = 0.f;
      rk<MODE>(F1u, Un, c, f, oU, fU, CDT1, TDT, TC1, TC2, su_a, su_b);
    }
    // v
    if (dv) {
      const f2 aa = mul(H, add(vP, vnP)), bb = mul(H, add(vsP, vP));
      const f2 ay = mul(dif(aa, aa, bb, bb), YRC);
      const f2 ax = mul(sub(FxyP, FxyL), XRF_P);
      const f2 az = mul(sub(FyzP, FyzB), ZRF);
      const f2 vx = mul(dif(XRC_P, sub(vR, vP), XRC_L, sub(vP, vL)), XRF_P);
      const f2 vy = mul(dif(YRFP, sub(vnP, vP), YRF, sub(vP, vsP)), YRC);
      const f2 vz = mul(dif(ZRC, dVt, ZRCM, dVz), ZRF);
      f2 f = fma(NU, add(add(vx, vy), vz), neg(add(add(ay, ax), az)));
      if (zx_a) f.x = 0.f;
      if (zx_b) f.y = 0.f;
      rk<MODE>(F1v, Vn, c, f, oV, fV, CDT1, TDT, TC1, TC2, sv_a, sv_b);
    }
    // w
    if (k <= g.nz - 1) {
      const f2 az = mul(dif(WtA, WtA, WbA, WbA), ZRC);
      const f2 ax = mul(sub(FxzP, FxzL), XRF_P);
      const f2 ay = mul(sub(FyzP, mul(mul(H, add(vsP, vstP)), lin(W0M, wsP, W1M, wP))), YRF);
      const f2 vx = mul(dif(XRC_P, sub(wR, wP), XRC_L, sub(wP, wL)), XRF_P);
      const f2 vy = mul(dif(sub(wnP, wP), YRC, sub(wP, wsP), YRCM), YRF);
      const f2 vz = mul(dif(ZRFP, dWt, ZRF, dWz), ZRC);
      f2 f = fma(NU, add(add(vx, vy), vz), sub(DPDZ, add(add(az, ax), ay)));
      if (zx_a) f.x = 0.f;
      if (zx_b) f.y = 0.f;
      rk<MODE>(F1w, Wn, c, f, oW, fW, CDT1, TDT, TC1, TC2, sv_a, sv_b);
    }
    if (!more) break;
    // carry the upper face terms down and slide the window to k+1
    FxzB = FxzP;
    FyzB = FyzP;
    dUz = dUt; dVz = dVt; dWz = dWt; WbA = WtA;
    c += pl;
    um = utm; uP = utP; up = __ldg(U + c + 2);
    vm = __ldg(V + c - 1); vP = vtP; vp = __ldg(V + c + 2);
    wm = __ldg(W + c - 1); wP = wtP; wp = __ldg(W + c + 2);
    vsP = vstP;
    vs_p = __ldg(V + c - px + 2);
    unm = __ldg(U + c + px - 1);
    unP = ld(U, c + px);
    usP = ld(U, c - px);
    vnP = ld(V, c + px);
    wnP = ld(W, c + px);
    wsP = ld(W, c - px);
    utm = utm2; utP = utP2; vtP = vtP2; vstP = vstP2; wtP = wtP2;
    oU = oU2; oV = oV2; oW = oW2; fU = fU2; fV = fV2; fW = fW2;
  }
}

// ---------------------------------------------------------------------------
// The packed FP32 DNS kernel fed by TMA.  A CTA of 32 x 8 threads owns 64
// x-points (32 pairs) by 8 rows and walks a chunk of k-planes.  Plane p of
// U, V and W reaches shared memory as one 72 x 10 x 1 tensor copy per field
// (x from the CTA's first point - 4, rows j-1 .. j+8) and, for the planes the
// CTA updates, the point-wise operands Uo, Vo, Wo (RK substeps) and F1
// (substeps 2 and 3) as 64 x 8 x 1 copies.  A ring of 4 stages, each
// completed on an mbarrier, holds plane p in stage (p - k0 + 1) mod 4: while
// plane k is computed (from planes k and k+1), planes k+2 and k+3 are in
// flight, and after a CTA barrier the stage of plane k takes plane k+4.  The
// k loop is unrolled by the ring length, so every shared-memory operand sits
// at a fixed offset from one per-thread base, and no global load sits on the
// arithmetic's path.  Arithmetic and carried terms are those of k_rhs_rk_pk.
// A wait that runs out of polls sets bit 64 of the device flag; the CTA then
// stops at the next barrier and waits (bounded) for the copies it issued.
// ---------------------------------------------------------------------------
constexpr int RT_NS = 4, RT_TW = 72, RT_BY = 8, RT_TH = RT_BY + 2;
constexpr int RT_FS = (RT_TH * RT_TW * 4 + 127) / 128 * 32;  // floats per field tile (a 128-byte multiple)
constexpr int RT_PS = 64 * RT_BY;                            // floats per point-wise tile
__host__ __device__ constexpr int rt_npw(int mode) { return mode == 0 ? 0 : mode == 1 ? 3 : 6; }
__host__ __device__ constexpr int rt_stage(int mode) { return 3 * RT_FS + rt_npw(mode) * RT_PS; }  // floats
__host__ __device__ constexpr size_t rt_smem(int mode) { return (size_t)RT_NS * rt_stage(mode) * 4 + RT_NS * 8 + 16; }

template <int MODE>
__global__ void __launch_bounds__(32 * RT_BY, 2)
    k_rhs_rk_tma(const __grid_constant__ CUtensorMap mu, const __grid_constant__ CUtensorMap mv,
                 const __grid_constant__ CUtensorMap mw, const __grid_constant__ CUtensorMap mou,
                 const __grid_constant__ CUtensorMap mov, const __grid_constant__ CUtensorMap mow,
                 const __grid_constant__ CUtensorMap mfu, const __grid_constant__ CUtensorMap mfv,
                 const __grid_constant__ CUtensorMap mfw, Geo g, MetT<float> m, float *__restrict__ F1u,
                 float *__restrict__ F1v, float *__restrict__ F1w, float *__restrict__ Un, float *__restrict__ Vn,
                 float *__restrict__ Wn, const Scalars *__restrict__ sc, double c1, double c2, int kchunk, int *err,
                 int wait_limit) {
  using namespace pk;
  constexpr int NS = RT_NS, TW = RT_TW, NPW = rt_npw(MODE), SS = rt_stage(MODE);
  constexpr uint32_t FIELD_BYTES = 3u * TW * RT_TH * 4u, PW_BYTES = (uint32_t)NPW * RT_PS * 4u;
  extern __shared__ __align__(1024) float rt_sm[];
  uint64_t *full = reinterpret_cast<uint64_t *>(rt_sm + NS * SS);
  volatile int *bad = reinterpret_cast<volatile int *>(full + NS);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  const int istart = 2 + 64 * blockIdx.x, jstart = 2 + RT_BY * blockIdx.y;
  const int i0 = istart + 2 * tx, j = jstart + ty;
  const int k0 = blockIdx.z * kchunk + 2;
  const int k1 = min(k0 + kchunk - 1, g.nz);
  if (k0 > k1) return;  // whole CTA
  const bool act = i0 <= g.nx && j <= g.ny;
  const int jj = act ? j : jstart;  // metric row and column of idle threads: any valid one
  const int ii = act ? i0 : istart;
  if (tid == 0) {
    // the copies need 128-byte aligned destinations
    *bad = (tma::smem_u32(rt_sm) & 127u) ? 1 : 0;
    for (int s = 0; s < NS; ++s) tma::mbar_init(&full[s], 1);
    tma::mbar_init_fence();
  }
  __syncthreads();
  if (*bad) {
    if (tid == 0) atomicOr(err, 64);
    return;
  }
  auto issue = [&](int p) {  // thread 0: plane p into its stage
    const int s = (p - k0 + 1) & (NS - 1);
    float *st = rt_sm + s * SS;
    const bool pw = NPW > 0 && p >= k0 && p <= k1;
    tma::mbar_expect_tx(&full[s], FIELD_BYTES + (pw ? PW_BYTES : 0u));
    tma::load_3d(st, &mu, istart - 2, jstart - 2, p - 1, &full[s]);
    tma::load_3d(st + RT_FS, &mv, istart - 2, jstart - 2, p - 1, &full[s]);
    tma::load_3d(st + 2 * RT_FS, &mw, istart - 2, jstart - 2, p - 1, &full[s]);
    if (pw) {
      float *pt = st + 3 * RT_FS;
      tma::load_3d(pt, &mou, istart + 2, jstart - 1, p - 1, &full[s]);
      tma::load_3d(pt + RT_PS, &mov, istart + 2, jstart - 1, p - 1, &full[s]);
      tma::load_3d(pt + 2 * RT_PS, &mow, istart + 2, jstart - 1, p - 1, &full[s]);
      if (NPW == 6) {
        tma::load_3d(pt + 3 * RT_PS, &mfu, istart + 2, jstart - 1, p - 1, &full[s]);
        tma::load_3d(pt + 4 * RT_PS, &mfv, istart + 2, jstart - 1, p - 1, &full[s]);
        tma::load_3d(pt + 5 * RT_PS, &mfw, istart + 2, jstart - 1, p - 1, &full[s]);
      }
    }
  };
  int issued = k0 - 2;  // thread 0: last plane issued
  if (tid == 0)
    for (int p = k0 - 1; p <= min(k0 + 2, k1 + 1); ++p) {
      issue(p);
      issued = p;
    }
  auto wait_plane = [&](int p) {
    if (!tma::mbar_wait(&full[(p - k0 + 1) & (NS - 1)], (uint32_t)(((p - k0 + 1) >> 2) & 1), wait_limit)) {
      *bad = 1;
      atomicOr(err, 64);
    }
  };
  // per-thread offsets: field tiles at row j (tile row ty + 1), column of
  // point i0; point-wise tiles at row ty, column 2 tx
  const float *fo = rt_sm + (ty + 1) * TW + 4 + 2 * tx;
  const float *po = rt_sm + 3 * RT_FS + ty * 64 + 2 * tx;
#define RT_P2(S, q, dr) (*reinterpret_cast<const f2 *>(fo + (S) * SS + (q) * RT_FS + (dr) * TW))
#define RT_S1(S, q, dr, dc) (fo[(S) * SS + (q) * RT_FS + (dr) * TW + (dc)])
#define RT_PW(S, q) (*reinterpret_cast<const f2 *>(po + (S) * SS + (q) * RT_PS))
  double dt = 0.0;
  if (MODE != 0) dt = sc->dt;
  const f2 CDT1 = sp((float)(dt * c1)), TDT = sp((float)dt), TC1 = sp((float)c1), TC2 = sp((float)c2);
  const int ib = i0 + 1;
  const bool su_a = i0 <= g.nx - 1, su_b = ib <= g.nx - 1;
  const bool sv_a = true, sv_b = ib <= g.nx;
  const bool dv = (j <= g.ny - 1);
  const bool zu_a = (i0 == g.nx - 1), zu_b = (ib == g.nx - 1);
  const bool zx_a = (i0 == g.nx), zx_b = (ib == g.nx);
  const f2 H = sp(0.5f);
  const f2 XRC_P = mk(m.xrC[ii], m.xrC[ii + 1]), XRF_P = mk(m.xrF[ii], m.xrF[ii + 1]);
  const f2 XRF_R = mk(m.xrF[ii + 1], m.xrF[ii + 2]), XRC_L = mk(m.xrC[ii - 1], m.xrC[ii]);
  const f2 YRF = sp(m.yrF[jj]), YRC = sp(m.yrC[jj]), YRCM = sp(m.yrC[jj - 1]), YRFP = sp(m.yrF[jj + 1]);
  const f2 W0 = sp(m.w0[jj]), W1 = sp(m.w1[jj]), W0M = sp(m.w0[jj - 1]), W1M = sp(m.w1[jj - 1]);
  const f2 NU = sp(m.nu), DPDX = sp(m.dpdx), DPDZ = sp(m.dpdz);
  long long c = bidx(g, ii, jj, k0);
  // carried k-1 face terms from planes k0-1 (stage 0) and k0 (stage 1)
  wait_plane(k0 - 1);
  wait_plane(k0);
  f2 FxzB, FyzB, dUz, dVz, dWz, WbA;
  {
    const f2 ubP = RT_P2(0, 0, 0), vbP = RT_P2(0, 1, 0), wbP = RT_P2(0, 2, 0), wnbP = RT_P2(0, 2, 1);
    const f2 uP = RT_P2(1, 0, 0), vP = RT_P2(1, 1, 0), wP = RT_P2(1, 2, 0);
    FxzB = fxz(H, ubP, uP, wbP, mk(wbP.y, RT_S1(0, 2, 0, 2)));
    FyzB = fyz(H, W0, W1, vbP, vP, wbP, wnbP);
    dUz = sub(uP, ubP);
    dVz = sub(vP, vbP);
    dWz = sub(wP, wbP);
    WbA = mul(H, add(wbP, wP));
  }
  __syncthreads();  // plane k0-1 read by all: its stage takes plane k0+3
  if (*bad) goto drain;
  if (tid == 0 && k0 + 3 <= k1 + 1) {
    issue(k0 + 3);
    issued = k0 + 3;
  }
  for (int k = k0;;) {
#pragma unroll
    for (int u = 0; u < NS; ++u) {
      const int SC = (u + 1) & (NS - 1), SN = (u + 2) & (NS - 1);  // stages of planes k and k+1
      wait_plane(k + 1);
      const f2 ZRF = sp(m.zrF[k]), ZRC = sp(m.zrC[k]), ZRCM = sp(m.zrC[k - 1]), ZRFP = sp(m.zrF[k + 1]);
      const f2 uP = RT_P2(SC, 0, 0), vP = RT_P2(SC, 1, 0), wP = RT_P2(SC, 2, 0);
      const f2 uL = mk(RT_S1(SC, 0, 0, -1), uP.x), uR = mk(uP.y, RT_S1(SC, 0, 0, 2));
      const f2 vL = mk(RT_S1(SC, 1, 0, -1), vP.x), vR = mk(vP.y, RT_S1(SC, 1, 0, 2));
      const f2 wL = mk(RT_S1(SC, 2, 0, -1), wP.x), wR = mk(wP.y, RT_S1(SC, 2, 0, 2));
      const f2 unP = RT_P2(SC, 0, 1), usP = RT_P2(SC, 0, -1), utP = RT_P2(SN, 0, 0);
      const f2 vnP = RT_P2(SC, 1, 1), vsP = RT_P2(SC, 1, -1), vtP = RT_P2(SN, 1, 0), vstP = RT_P2(SN, 1, -1);
      const f2 wnP = RT_P2(SC, 2, 1), wsP = RT_P2(SC, 2, -1), wtP = RT_P2(SN, 2, 0);
      const f2 XL = mul(H, add(uL, uP)), XR = mul(H, add(uP, uR));
      const f2 FxyP = mul(lin(W0, uP, W1, unP), mul(H, add(vP, vR)));
      const f2 FxyL = mul(lin(W0, uL, W1, mk(RT_S1(SC, 0, 1, -1), unP.x)), mul(H, add(vL, vP)));
      const f2 FxzP = fxz(H, uP, utP, wP, wR);
      const f2 FxzL = fxz(H, uL, mk(RT_S1(SN, 0, 0, -1), utP.x), wL, wP);
      const f2 FyzP = fyz(H, W0, W1, vP, vtP, wP, wnP);
      const f2 dUt = sub(utP, uP), dVt = sub(vtP, vP), dWt = sub(wtP, wP);
      const f2 WtA = mul(H, add(wP, wtP));
      if (act) {
        f2 oU{}, oV{}, oW{}, fU{}, fV{}, fW{};
        if (NPW >= 3) { oU = RT_PW(SC, 0); oV = RT_PW(SC, 1); oW = RT_PW(SC, 2); }
        if (NPW == 6) { fU = RT_PW(SC, 3); fV = RT_PW(SC, 4); fW = RT_PW(SC, 5); }
        {  // u
          const f2 ax = mul(dif(XR, XR, XL, XL), XRC_P);
          const f2 ay = mul(sub(FxyP, mul(lin(W0M, usP, W1M, uP), mul(H, add(vsP, mk(vsP.y, RT_S1(SC, 1, -1, 2)))))), YRF);
          const f2 az = mul(sub(FxzP, FxzB), ZRF);
          const f2 vx = mul(dif(XRF_R, sub(uR, uP), XRF_P, sub(uP, uL)), XRC_P);
          const f2 vy = mul(dif(sub(unP, uP), YRC, sub(uP, usP), YRCM), YRF);
          const f2 vz = mul(dif(ZRC, dUt, ZRCM, dUz), ZRF);
          f2 f = fma(NU, add(add(vx, vy), vz), sub(DPDX, add(add(ax, ay), az)));
          if (zu_a) f.x = 0.f;
          if (zu_b) f.y = 0.f;
          rk<MODE>(F1u, Un, c, f, oU, fU, CDT1, TDT, TC1, TC2, su_a, su_b);
        }
        if (dv) {  // v
          const f2 aa = mul(H, add(vP, vnP)), bb = mul(H, add(vsP, vP));
          const f2 ay = mul(dif(aa, aa, bb, bb), YRC);
          const f2 ax = mul(sub(FxyP, FxyL), XRF_P);
          const f2 az = mul(sub(FyzP, FyzB), ZRF);
          const f2 vx = mul(dif(XRC_P, sub(vR, vP), XRC_L, sub(vP, vL)), XRF_P);
          const f2 vy = mul(dif(YRFP, sub(vnP, vP), YRF, sub(vP, vsP)), YRC);
          const f2 vz = mul(dif(ZRC, dVt, ZRCM, dVz), ZRF);
          f2 f = fma(NU, add(add(vx, vy), vz), neg(add(add(ay, ax), az)));
          if (zx_a) f.x = 0.f;
          if (zx_b) f.y = 0.f;
          rk<MODE>(F1v, Vn, c, f, oV, fV, CDT1, TDT, TC1, TC2, sv_a, sv_b);
        }
        if (k <= g.nz - 1) {  // w
          const f2 az = mul(dif(WtA, WtA, WbA, WbA), ZRC);
          const f2 ax = mul(sub(FxzP, FxzL), XRF_P);
          const f2 ay = mul(sub(FyzP, mul(mul(H, add(vsP, vstP)), lin(W0M, wsP, W1M, wP))), YRF);
          const f2 vx = mul(dif(XRC_P, sub(wR, wP), XRC_L, sub(wP, wL)), XRF_P);
          const f2 vy = mul(dif(sub(wnP, wP), YRC, sub(wP, wsP), YRCM), YRF);
          const f2 vz = mul(dif(ZRFP, dWt, ZRF, dWz), ZRC);
          f2 f = fma(NU, add(add(vx, vy), vz), sub(DPDZ, add(add(az, ax), ay)));
          if (zx_a) f.x = 0.f;
          if (zx_b) f.y = 0.f;
          rk<MODE>(F1w, Wn, c, f, oW, fW, CDT1, TDT, TC1, TC2, sv_a, sv_b);
        }
      }
      if (k == k1) goto drain;
      FxzB = FxzP;
      FyzB = FyzP;
      dUz = dUt; dVz = dVt; dWz = dWt; WbA = WtA;
      c += g.plane;
      __syncthreads();  // plane k read by all: its stage takes plane k+4
      if (*bad) goto drain;
      if (tid == 0 && k + 4 <= k1 + 1) {
        issue(k + 4);
        issued = k + 4;
      }
      ++k;
    }
  }
drain:
#undef RT_P2
#undef RT_S1
#undef RT_PW
  // after a missed wait: the copies this CTA issued complete before it exits
  // (on the normal path every issued plane has been waited for)
  __syncthreads();
  if (tid == 0 && *bad)
    for (int p = max(issued - NS + 1, k0 - 1); p <= issued; ++p)
      tma::mbar_wait(&full[(p - k0 + 1) & (NS - 1)], (uint32_t)(((p - k0 + 1) >> 2) & 1));
}

// ---------------------------------------------------------------------------
// The FP64 DNS RHS fed by TMA.  The arithmetic is rhs_*_at and the RK update
// of k_rhs_rk, term for term (the FP64 unit is compiled without contraction,
// so the results are those of k_rhs_rk bit for bit); only the operands come
// from shared memory.  A CTA of 32 x 8 threads owns 32 x-points (one per
// thread) by 8 rows and walks a chunk of k-planes.  Plane p of U, V, W
// arrives as one 36 x 10 x 1 tensor copy per field (x from the CTA's first
// point - 2, so the copy starts on a 16-byte boundary; rows j-1 .. j+8) and,
// for the planes the CTA updates, Uo, Vo, Wo and F1 as 32 x 8 x 1 copies.  A
// ring of 5 stages holds plane p in stage (p - k0 + 1) mod 5: plane k is
// computed from planes k-1, k and k+1 while k+2 and k+3 are in flight, and
// after a CTA barrier the stage of plane k-1 takes plane k+4.  The k loop is
// unrolled by the ring length.  Wait limits and the drain as in k_rhs_rk_tma.
// ---------------------------------------------------------------------------
constexpr int R64_NS = 5, R64_TW = 36, R64_BY = 8, R64_TH = R64_BY + 2;
constexpr int R64_FS = (R64_TH * R64_TW * 8 + 127) / 128 * 16;  // doubles per field tile (a 128-byte multiple)
constexpr int R64_PS = 32 * R64_BY;                             // doubles per point-wise tile
__host__ __device__ constexpr int r64_stage(int mode) { return 3 * R64_FS + rt_npw(mode) * R64_PS; }  // doubles
__host__ __device__ constexpr size_t r64_smem(int mode) {
  return (size_t)R64_NS * r64_stage(mode) * 8 + R64_NS * 8 + 16;
}

// operand loader of rhs_*_at over the staged planes k-1, k, k+1 (pointers at
// the thread's point; di, dj, dk in -1..1 are compile-time at every call)
struct SmemLd64 {
  const double *pb, *pc, *pt;
  __device__ __forceinline__ double operator()(long long, int di, int dj, int dk) const {
    return (dk < 0 ? pb : dk > 0 ? pt : pc)[di + dj * R64_TW];
  }
};

template <int MODE>
__global__ void __launch_bounds__(32 * R64_BY, 2)
    k_rhs_rk_tma64(const __grid_constant__ CUtensorMap mu, const __grid_constant__ CUtensorMap mv,
                   const __grid_constant__ CUtensorMap mw, const __grid_constant__ CUtensorMap mou,
                   const __grid_constant__ CUtensorMap mov, const __grid_constant__ CUtensorMap mow,
                   const __grid_constant__ CUtensorMap mfu, const __grid_constant__ CUtensorMap mfv,
                   const __grid_constant__ CUtensorMap mfw, Geo g, MetT<double> m, double *__restrict__ F1u,
                   double *__restrict__ F1v, double *__restrict__ F1w, double *__restrict__ Un,
                   double *__restrict__ Vn, double *__restrict__ Wn, const Scalars *__restrict__ sc, double c1,
                   double c2, int kchunk, int *err, int wait_limit) {
  constexpr int NS = R64_NS, TW = R64_TW, NPW = rt_npw(MODE), SS = r64_stage(MODE);
  constexpr uint32_t FIELD_BYTES = 3u * TW * R64_TH * 8u, PW_BYTES = (uint32_t)NPW * R64_PS * 8u;
  extern __shared__ __align__(1024) double r64_sm[];
  uint64_t *full = reinterpret_cast<uint64_t *>(r64_sm + NS * SS);
  volatile int *bad = reinterpret_cast<volatile int *>(full + NS);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  const int istart = 2 + 32 * blockIdx.x, jstart = 2 + R64_BY * blockIdx.y;
  const int i = istart + tx, j = jstart + ty;
  const int k0 = blockIdx.z * kchunk + 2;
  const int k1 = min(k0 + kchunk - 1, g.nz);
  if (k0 > k1) return;  // whole CTA
  const bool act = i <= g.nx && j <= g.ny;
  if (tid == 0) {
    *bad = (tma::smem_u32(r64_sm) & 127u) ? 1 : 0;
    for (int s = 0; s < NS; ++s) tma::mbar_init(&full[s], 1);
    tma::mbar_init_fence();
  }
  __syncthreads();
  if (*bad) {
    if (tid == 0) atomicOr(err, 64);
    return;
  }
  auto issue = [&](int p) {  // thread 0: plane p into its stage
    const int s = (p - k0 + 1) % NS;
    double *st = r64_sm + s * SS;
    const bool pw = NPW > 0 && p >= k0 && p <= k1;
    tma::mbar_expect_tx(&full[s], FIELD_BYTES + (pw ? PW_BYTES : 0u));
    tma::load_3d(st, &mu, istart, jstart - 2, p - 1, &full[s]);
    tma::load_3d(st + R64_FS, &mv, istart, jstart - 2, p - 1, &full[s]);
    tma::load_3d(st + 2 * R64_FS, &mw, istart, jstart - 2, p - 1, &full[s]);
    if (pw) {
      double *pt = st + 3 * R64_FS;
      tma::load_3d(pt, &mou, istart + 2, jstart - 1, p - 1, &full[s]);
      tma::load_3d(pt + R64_PS, &mov, istart + 2, jstart - 1, p - 1, &full[s]);
      tma::load_3d(pt + 2 * R64_PS, &mow, istart + 2, jstart - 1, p - 1, &full[s]);
      if (NPW == 6) {
        tma::load_3d(pt + 3 * R64_PS, &mfu, istart + 2, jstart - 1, p - 1, &full[s]);
        tma::load_3d(pt + 4 * R64_PS, &mfv, istart + 2, jstart - 1, p - 1, &full[s]);
        tma::load_3d(pt + 5 * R64_PS, &mfw, istart + 2, jstart - 1, p - 1, &full[s]);
      }
    }
  };
  int issued = k0 - 2;  // thread 0: last plane issued
  if (tid == 0)
    for (int p = k0 - 1; p <= min(k0 + NS - 2, k1 + 1); ++p) {
      issue(p);
      issued = p;
    }
  auto wait_plane = [&](int p) {
    if (!tma::mbar_wait(&full[(p - k0 + 1) % NS], (uint32_t)(((p - k0 + 1) / NS) & 1), wait_limit)) {
      *bad = 1;
      atomicOr(err, 64);
    }
  };
  // per-thread offsets: field tiles at row j (tile row ty + 1), column of
  // point i (tx + 2); point-wise tiles at row ty, column tx
  const double *fo = r64_sm + (ty + 1) * TW + 2 + tx;
  const double *po = r64_sm + 3 * R64_FS + ty * 32 + tx;
  double dt = 0.0;
  if (MODE != 0) dt = sc->dt;
  const double cdt1 = dt * c1, tdt = dt, tc1 = c1, tc2 = c2;
  const bool du = (i <= g.nx - 1), dv = (j <= g.ny - 1);
  wait_plane(k0 - 1);
  wait_plane(k0);
  for (int k = k0;;) {
#pragma unroll
    for (int u = 0; u < NS; ++u) {
      const int SB = u, SC = (u + 1) % NS, ST = (u + 2) % NS;  // stages of planes k-1, k, k+1
      wait_plane(k + 1);
      if (act) {
        const SmemLd64 LU{fo + SB * SS, fo + SC * SS, fo + ST * SS};
        const SmemLd64 LV{fo + SB * SS + R64_FS, fo + SC * SS + R64_FS, fo + ST * SS + R64_FS};
        const SmemLd64 LW{fo + SB * SS + 2 * R64_FS, fo + SC * SS + 2 * R64_FS, fo + ST * SS + 2 * R64_FS};
        const double *pw = po + SC * SS;
        const long long c = bidx(g, i, j, k);
        if (du) {
          double f = (i == g.nx - 1) ? 0.0 : rhs_u_at<double, false, SmemLd64>(g, m, LU, LV, LW, LU, c, i, j, k);
          if (MODE == 0) F1u[c] = f;
          else if (MODE == 1) { F1u[c] = f; Un[c] = pw[0] + cdt1 * f; }
          else Un[c] = pw[0] + tdt * (tc1 * pw[3 * R64_PS] + tc2 * f);
        }
        if (dv) {
          double f = (i == g.nx) ? 0.0 : rhs_v_at<double, false, SmemLd64>(g, m, LU, LV, LW, LU, c, i, j, k);
          if (MODE == 0) F1v[c] = f;
          else if (MODE == 1) { F1v[c] = f; Vn[c] = pw[R64_PS] + cdt1 * f; }
          else Vn[c] = pw[R64_PS] + tdt * (tc1 * pw[4 * R64_PS] + tc2 * f);
        }
        if (k <= g.nz - 1) {
          double f = (i == g.nx) ? 0.0 : rhs_w_at<double, false, SmemLd64>(g, m, LU, LV, LW, LU, c, i, j, k);
          if (MODE == 0) F1w[c] = f;
          else if (MODE == 1) { F1w[c] = f; Wn[c] = pw[2 * R64_PS] + cdt1 * f; }
          else Wn[c] = pw[2 * R64_PS] + tdt * (tc1 * pw[5 * R64_PS] + tc2 * f);
        }
      }
      if (k == k1) goto drain;
      __syncthreads();  // plane k-1 read by all: its stage takes plane k+4
      if (*bad) goto drain;
      if (tid == 0 && k + NS - 1 <= k1 + 1) {
        issue(k + NS - 1);
        issued = k + NS - 1;
      }
      ++k;
    }
  }
drain:
  __syncthreads();
  if (tid == 0 && *bad)
    for (int p = max(issued - NS + 1, k0 - 1); p <= issued; ++p)
      tma::mbar_wait(&full[(p - k0 + 1) % NS], (uint32_t)(((p - k0 + 1) / NS) & 1));
}

// ---------------------------------------------------------------------------
// project_velocity (projection.f90:359-384) + pressure save at rk_step 1
// (projection.f90:75-78, P(2:nxg-1,2:nyg-1,2:nzg-1) = rhs_p/(dt*rk2_coef(1,1))).
// p holds rhs_p in the box layout (i=2..nx, j=2..ny, k=2..nz valid).
// p0 (mixed form only): the z-mean part of rhs_p, kept in FP64 as a
// [j-2][i-2] plane of pitch nx-2 (x-Neumann copy at i = nx).
// ---------------------------------------------------------------------------
// A thread updates VN = 16/sizeof(T) consecutive
// points i0..i0+VN-1 (i0 = 2 + VN*q, a 16-byte aligned box position) with
// 16-byte loads and stores; points outside the update ranges keep their
// loaded value.
template <typename T> struct V16;
template <> struct V16<float> { typedef float4 t; };
template <> struct V16<double> { typedef double2 t; };

template <typename T>
__global__ void __launch_bounds__(256) k_project_v(Geo g, MetT<T> m, const T *__restrict__ p,
                                                   const double *__restrict__ p0, const float *__restrict__ p0g,
                                                   T *__restrict__ U,
                                                   T *__restrict__ V, T *__restrict__ W, T *__restrict__ P,
                                                   const Scalars *__restrict__ sc, int save_p) {
  typedef typename V16<T>::t VT;
  constexpr int VN = 16 / sizeof(T);
  const int i0 = 2 + VN * (blockIdx.x * blockDim.x + threadIdx.x);
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k = blockIdx.z + 2;
  if (i0 > g.nx || j > g.ny) return;
  const long long c = bidx(g, i0, j, k);
  union Vec {
    VT v;
    T e[VN];
  };
  Vec pc, pn, pt, u, v, w;
  pc.v = __ldg(reinterpret_cast<const VT *>(p + c));
  const T pe = __ldg(p + c + VN);
  pn.v = __ldg(reinterpret_cast<const VT *>(p + c + g.px));
  pt.v = __ldg(reinterpret_cast<const VT *>(p + c + g.plane));
  u.v = *reinterpret_cast<const VT *>(U + c);
  v.v = *reinterpret_cast<const VT *>(V + c);
  w.v = *reinterpret_cast<const VT *>(W + c);
  const bool vj = (j <= g.ny - 1), wk = (k <= g.nz - 1);
  const T yC = m.yC[j], yrC = m.yrC[j], zC = m.zC[k], zrC = m.zrC[k];
  const int N = g.nx - 2;
  const double *p0r = p0 ? p0 + (long long)(j - 2) * N : nullptr;  // row j of the FP64 part
  const float *gxr = p0g ? p0g + (long long)(j - 2) * N : nullptr;  // its x and y differences
  const float *gyr = p0g ? gxr + (long long)N * (g.ny - 1) : nullptr;
#pragma unroll
  for (int e = 0; e < VN; ++e) {
    const int i = i0 + e;
    const T pe1 = (e + 1 < VN) ? pc.e[e + 1] : pe;
    if (i <= g.nx - 1) {
      T dd = pe1 - pc.e[e];
      if (p0g) dd = dd + (T)gxr[i - 2];
      u.e[e] = u.e[e] - qdiv(dd, m.xC[i], m.xrC[i]);
    }
    if (i <= g.nx) {
      if (vj) {
        T dd = pn.e[e] - pc.e[e];
        if (p0g) dd = dd + (T)gyr[min(i - 2, N - 1)];
        v.e[e] = v.e[e] - qdiv(dd, yC, yrC);
      }
      if (wk) w.e[e] = w.e[e] - qdiv(pt.e[e] - pc.e[e], zC, zrC);
    }
  }
  *reinterpret_cast<VT *>(U + c) = u.v;
  *reinterpret_cast<VT *>(V + c) = v.v;
  *reinterpret_cast<VT *>(W + c) = w.v;
  if (save_p) {
    const double den = sc->dt * 0.5;  // dt*rk2_coef(1,1)
    Vec q;
#pragma unroll
    for (int e = 0; e < VN; ++e) {
      double pv = (double)pc.e[e];
      if (p0 && i0 + e <= g.nx) pv += p0r[min(i0 + e - 2, N - 1)];
      q.e[e] = (i0 + e <= g.nx) ? (T)(pv / den) : (T)0;
    }
    *reinterpret_cast<VT *>(P + c) = q.v;
  }
}

// P ghost planes, projection.f90:78-83.  The source copies the x ghosts, then
// the y ghosts (over every i, the x ghosts included), then the z ghosts (over
// every i, j); each copy takes the neighbouring layer, so every ghost point
// ends with the interior value at its clamped indices (1 -> 2, n -> n-1 in
// each direction), which this launch writes in one pass: blocks take the x
// faces over (j, k), the y faces over (i, k) and the z faces over (i, j);
// edges and corners are written alike by each face they lie on, and no
// source value is a ghost.
template <typename T>
__global__ void k_p_ghost(Geo g, T *__restrict__ P, int bx, int by) {
  int blk = blockIdx.x;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  auto cl = [](int v, int n) { return v == 1 ? 2 : v == n ? n - 1 : v; };
  const int nxg = g.nxg, nyg = g.nyg, nzg = g.nzg;
  if (blk < bx) {  // x faces, (j, k)
    const int tj = (nyg + 31) / 32;
    const int j = (blk % tj) * 32 + tx + 1, k = (blk / tj) * 8 + ty + 1;
    if (j > nyg || k > nzg) return;
    const int cj = cl(j, nyg), ck = cl(k, nzg);
    P[bidx(g, 1, j, k)] = P[bidx(g, 2, cj, ck)];
    P[bidx(g, nxg, j, k)] = P[bidx(g, nxg - 1, cj, ck)];
    return;
  }
  blk -= bx;
  const int ti = (nxg + 31) / 32;
  if (blk < by) {  // y faces, (i, k)
    const int i = (blk % ti) * 32 + tx + 1, k = (blk / ti) * 8 + ty + 1;
    if (i > nxg || k > nzg) return;
    const int ci = cl(i, nxg), ck = cl(k, nzg);
    P[bidx(g, i, 1, k)] = P[bidx(g, ci, 2, ck)];
    P[bidx(g, i, nyg, k)] = P[bidx(g, ci, nyg - 1, ck)];
    return;
  }
  blk -= by;  // z faces, (i, j)
  const int i = (blk % ti) * 32 + tx + 1, j = (blk / ti) * 8 + ty + 1;
  if (i > nxg || j > nyg) return;
  const int ci = cl(i, nxg), cj = cl(j, nyg);
  P[bidx(g, i, j, 1)] = P[bidx(g, ci, cj, 2)];
  P[bidx(g, i, j, nzg)] = P[bidx(g, ci, cj, nzg - 1)];
}

// ---------------------------------------------------------------------------
// Boundary conditions, boundary_conditions.f90:127-262, in two ordered
// launches: k_bc_all (every boundary value but the mass correction, and the
// x mass-flux sum) and k_bc_mass (the correction of U(nx-1), U(nx)).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double mode_sum(const double2 *__restrict__ q, int ld, int j, int nm, int mm,
                                           const double *__restrict__ zmode, const double *__restrict__ tmode,
                                           double zz, double t) {
  // sum_n sum_m Re(q(j,n,m) exp(i(zmode_n z - tmode_m t)))  (:143-150)
  double acc = 0.0;
  for (int n = 0; n < nm; ++n)
    for (int mi = 0; mi < mm; ++mi) {
      double2 qq = q[((long long)mi * nm + n) * ld + (j - 1)];
      double th = zmode[n] * zz - tmode[mi] * t;
      double s, co;
      sincos(th, &s, &co);
      acc = acc + (qq.x * co - qq.y * s);
    }
  return acc;
}

// Every boundary value the routine leaves before its mass correction is a
// function of the inflow data, the step's start fields Uo, Vo, Wo and the
// interior of the current fields, evaluated in the routine's order:
//   x planes (1) inflow at i = 1, (2) convective outflow at i = nx-1 (U) and
//     nxg-1 (V, W) with the plane beyond it equal;
//   (3) z ghosts: U, V: k = 1 <- nzg-2, nzg-1 <- 2, nzg <- 3; W: 1 <- nz-1,
//     nz <- 2 (copies of what (1), (2) left there);
//   (4) top rows U(:,nyg,:), V(:,ny,:), W(:,nyg,:) = U_top, V_top, W_top;
//   (5) wall rows U(:,1,:) = -U(:,2,:), V(:,1,:) = 0, W(:,1,:) = -W(:,2,:)
//     (or the wall model's Neumann rows) from what (1)-(3) left in row 2.
// k_bc_all writes each boundary point once with that final value, so its
// four segments of blocks (x planes of U; x planes of V and W; z ghosts of
// interior columns; y rows of interior columns) read nothing another thread
// writes.  The U x-plane blocks also form the x mass-flux partials; the last
// of them sums the partials in block order and leaves the correction in
// sc->dU for k_bc_mass (6).  A thread issues its loads before its stores, so
// that it waits for memory about once.
template <typename T> struct BcX {
  // (1): U, V, W at i = 1 of row j, plane k
  __device__ static double in_u(const Geo &g, const BcData &bc, int j, int k, double t) {
    if (bc.lund == 3) return bc.lu[(long long)(k - 1) * g.nyg + (j - 1)];
    if (bc.lund == 5) return bc.U_inlet[j] + bc.lu[(long long)(k - 1) * g.nyg + (j - 1)];
    double ut = 0.0;
    if (bc.n_modes > 0) ut = mode_sum(bc.qu, g.nyg, j, bc.n_modes, bc.m_modes, bc.zmode, bc.tmode, g.zg[k], t);
    else if (bc.ut) ut = bc.ut[(long long)(k - 1) * g.nyg + (j - 1)];
    return bc.U_inlet[j] + ut;
  }
  __device__ static double in_v(const Geo &g, const BcData &bc, int j, int k, double t) {  // j <= ny
    if (bc.lund == 3) return bc.lv[(long long)(k - 1) * g.ny + (j - 1)];
    if (bc.lund == 5) return bc.V_inlet[j] + bc.lv[(long long)(k - 1) * g.ny + (j - 1)];
    double vt = 0.0;
    if (bc.n_modes > 0) vt = mode_sum(bc.qv, g.ny, j, bc.n_modes, bc.m_modes, bc.zmode, bc.tmode, g.zg[k], t);
    else if (bc.ut) vt = bc.vt[(long long)(k - 1) * g.ny + (j - 1)];
    return bc.V_inlet[j] + vt;
  }
  __device__ static double in_w(const Geo &g, const BcData &bc, int j, int k, double t) {  // k <= nz
    if (bc.lund == 3) return bc.lw[(long long)(k - 1) * g.nyg + (j - 1)];
    if (bc.lund == 5) {
      const int ks = (k + 16) % g.nz + 1;  // boundary_conditions.f90:527-553
      return bc.W_inlet[j] + bc.lw[(long long)(ks - 1) * g.nyg + (j - 1)];
    }
    double wt = 0.0;
    if (bc.n_modes > 0) wt = mode_sum(bc.qw, g.nyg, j, bc.n_modes, bc.m_modes, bc.zmode, bc.tmode, g.z[k], t);
    else if (bc.ut) wt = bc.wt[(long long)(k - 1) * g.nyg + (j - 1)];
    return bc.W_inlet[j] + wt;
  }
  // (2): rk_t(rk_step) dt Uc (Fo(n-1) - Fo(n-2)) / spacing, cc = rk_t dt Uc
  __device__ static T out_u(const Geo &g, const T *__restrict__ Uo, int j, int k, double cc) {
    const long long a = bidx(g, g.nx - 1, j, k);
    const T uo1 = Uo[a], uo2 = Uo[a - 1];
    return (T)((double)uo1 - cc * (double)(uo1 - uo2) / g.ax.F[g.nx - 1]);
  }
  __device__ static T out_vw(const Geo &g, const T *__restrict__ Fo, int j, int k, double cc) {
    const long long a = bidx(g, g.nxg - 1, j, k);
    const T f1 = Fo[a], f2 = Fo[a - 1];
    return (T)((double)f1 - cc * (double)(f1 - f2) / g.ax.C[g.nxg - 2]);
  }
  // z source plane of a ghost plane, (3)
  __device__ static int ks_uv(const Geo &g, int k) {
    return k == 1 ? g.nzg - 2 : (k == g.nzg - 1 ? 2 : (k == g.nzg ? 3 : k));
  }
  __device__ static int ks_w(const Geo &g, int k) { return k == 1 ? g.nz - 1 : (k == g.nz ? 2 : k); }
  // (5) with the wall model: F(i,1,k) = F(i,2,k) - alpha (yg(2) - yg(1)) at the
  // wall point (ic, kc) that column i, plane k takes (boundary_conditions.f90:359-372)
  __device__ static long long wm_index(const Geo &g, int i, int k) {
    const int ic = min(max(i, 2), g.nx - 1);
    const int kc = k == 1 ? g.nzg - 2 : (k == g.nzg - 1 ? 2 : (k == g.nzg ? 3 : k));
    return (long long)(kc - 2) * (g.nx - 2) + (ic - 2);
  }
  __device__ static T wall_u(const Geo &g, const BcData &bc, T row2, int i, int k) {
    if (bc.wm_ax) return (T)((double)row2 - bc.wm_ax[wm_index(g, i, k)] * (g.yg[2] - g.yg[1]));
    return -row2;
  }
  __device__ static T wall_w(const Geo &g, const BcData &bc, T row2, int i, int k) {
    if (bc.wm_ax && bc.wm_az) return (T)((double)row2 - bc.wm_az[wm_index(g, i, k)] * (g.yg[2] - g.yg[1]));
    return -row2;
  }
};

struct BcGrid {  // block counts of the segments (32 x 8 tiles)
  int nx_blocks, nz_blocks, ny_blocks;  // U x planes (V and W take 2 nx_blocks more); z ghosts; y rows
  int x_tiles, zi_tiles, yi_tiles;      // tiles along the first dimension of each segment
};

template <typename T>
__global__ void __launch_bounds__(256) k_bc_all(Geo g, BcData bc, BcGrid G, T *__restrict__ U, T *__restrict__ V,
                                                T *__restrict__ W, const T *__restrict__ Uo,
                                                const T *__restrict__ Vo, const T *__restrict__ Wo,
                                                Scalars *__restrict__ sc, double rkt, double *__restrict__ qx_part,
                                                double qy, double length_y) {
  int blk = blockIdx.x;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int nx = g.nx, nxg = g.nxg, ny = g.ny, nyg = g.nyg, nz = g.nz, nzg = g.nzg;
  typedef BcX<T> X;
  if (blk >= G.nx_blocks && blk < 3 * G.nx_blocks) {
    // ---- x planes of V (the first nx_blocks) and W, thread (j, k) ----
    const int bb = (blk - G.nx_blocks) % G.nx_blocks;
    const int j = (bb % G.x_tiles) * 32 + tx + 1, k = (bb / G.x_tiles) * 8 + ty + 1;
    if (j > nyg || k > nzg) return;
    const double t = sc->t, cc = rkt * sc->dt * bc.U_top[nx];
    if (blk < 2 * G.nx_blocks) {
      if (j > ny) return;  // V at i = 1, nxg-1, nxg
      const int kv = X::ks_uv(g, k);
      T v1, vn, vn1;
      if (j == 1) {
        v1 = vn = vn1 = (T)0;
      } else if (j == ny) {
        v1 = (T)bc.V_top[1];
        vn = (T)bc.V_top[nxg - 1];
        vn1 = (T)bc.V_top[nxg];
      } else {
        v1 = (T)X::in_v(g, bc, j, kv, t);
        vn = vn1 = X::out_vw(g, Vo, j, kv, cc);
      }
      const long long a = bidx(g, nxg - 1, j, k);
      V[bidx(g, 1, j, k)] = v1;
      V[a] = vn;
      V[a + 1] = vn1;
    } else {
      if (k > nz) return;  // W at i = 1, nxg-1, nxg
      const int kw = X::ks_w(g, k);
      T w1, wn, wn1;
      if (j == nyg) {
        w1 = (T)bc.W_top[1];
        wn = (T)bc.W_top[nxg - 1];
        wn1 = (T)bc.W_top[nxg];
      } else if (j == 1) {
        w1 = X::wall_w(g, bc, (T)X::in_w(g, bc, 2, kw, t), 1, k);
        const T o2 = X::out_vw(g, Wo, 2, kw, cc);
        wn = X::wall_w(g, bc, o2, nxg - 1, k);
        wn1 = X::wall_w(g, bc, o2, nxg, k);
      } else {
        w1 = (T)X::in_w(g, bc, j, kw, t);
        wn = wn1 = X::out_vw(g, Wo, j, kw, cc);
      }
      const long long a = bidx(g, nxg - 1, j, k);
      W[bidx(g, 1, j, k)] = w1;
      W[a] = wn;
      W[a + 1] = wn1;
    }
    return;
  }
  if (blk < G.nx_blocks) {
    // ---- x planes of U, thread (j, k) ----
    const int j = (blk % G.x_tiles) * 32 + tx + 1, k = (blk / G.x_tiles) * 8 + ty + 1;
    double q = 0.0;
    if (j <= nyg && k <= nzg) {
      const double t = sc->t, cc = rkt * sc->dt * bc.U_top[nx];
      // U at i = 1 and nx-1 (k_bc_mass sets i = nx)
      const int ku = X::ks_uv(g, k);
      T u1, un;
      if (j == nyg) {
        u1 = (T)bc.U_top[1];
        un = (T)bc.U_top[nx - 1];
      } else if (j == 1) {
        u1 = X::wall_u(g, bc, (T)X::in_u(g, bc, 2, ku, t), 1, k);
        un = X::wall_u(g, bc, X::out_u(g, Uo, 2, ku, cc), nx - 1, k);
      } else {
        u1 = (T)X::in_u(g, bc, j, ku, t);
        un = X::out_u(g, Uo, j, ku, cc);
        if (j <= nyg - 1 && k >= 2 && k <= nzg - 2) q = ((double)u1 - (double)un) * g.ay.F[j];  // (:242-246)
      }
      U[bidx(g, 1, j, k)] = u1;
      U[bidx(g, nx - 1, j, k)] = un;
    }
    // deterministic block reduction of the x mass-flux partials (:242-246)
    __shared__ double red[256];
    const int tid = threadIdx.x;
    red[tid] = q;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
      if (tid < s) red[tid] += red[tid + s];
      __syncthreads();
    }
    // the last x-plane block to finish sums the partials in block order (the
    // same fixed order for every launch) and leaves the flux correction in
    // sc->dU (:240-260); the arrival counter sits after the partials
    const int nparts = G.nx_blocks;
    unsigned int *arrived = reinterpret_cast<unsigned int *>(qx_part + nparts);
    __shared__ int last;
    if (tid == 0) {
      qx_part[blk] = red[0];
      __threadfence();
      last = atomicAdd(arrived, 1u) == (unsigned)(nparts - 1);
    }
    __syncthreads();
    if (last) {
      __threadfence();
      double qx = 0.0;
      for (int p0 = 0; p0 < nparts; p0 += 256) {
        const int n = min(256, nparts - p0);
        if (tid < n) red[tid] = __ldcg(qx_part + p0 + tid);
        __syncthreads();
        if (tid == 0)
          for (int p = 0; p < n; ++p) qx += red[p];
        __syncthreads();
      }
      if (tid == 0) {
        sc->dU = (qx + qy) / length_y / (double)(nzg - 3);
        *arrived = 0u;
      }
    }
    return;
  }
  blk -= 3 * G.nx_blocks;
  const long long P = g.plane;
  if (blk < G.nz_blocks) {
    // ---- z ghost planes of the interior columns, thread (i, j): (3) ----
    const int i = (blk % G.zi_tiles) * 32 + tx + 2, j = (blk / G.zi_tiles) * 8 + ty + 2;
    if (i > nxg - 2 || j > nyg - 1) return;
    // sources: planes nzg-2, 2, 3 (W: nz-1, 2); targets: 1, nzg-1, nzg (W: 1, nz)
    const long long c1 = bidx(g, i, j, 1);
    const bool du = i <= nx - 2, dv = j <= ny - 1;
    T u0 = 0, u1 = 0, u2 = 0, v0 = 0, v1 = 0, v2 = 0;
    if (du) {
      u0 = U[c1 + (nzg - 3) * P];
      u1 = U[c1 + 1 * P];
      u2 = U[c1 + 2 * P];
    }
    if (dv) {
      v0 = V[c1 + (nzg - 3) * P];
      v1 = V[c1 + 1 * P];
      v2 = V[c1 + 2 * P];
    }
    const T w0 = W[c1 + (nz - 2) * P], w1 = W[c1 + 1 * P];
    if (du) {
      U[c1] = u0;
      U[c1 + (nzg - 2) * P] = u1;
      U[c1 + (nzg - 1) * P] = u2;
    }
    if (dv) {
      V[c1] = v0;
      V[c1 + (nzg - 2) * P] = v1;
      V[c1 + (nzg - 1) * P] = v2;
    }
    W[c1] = w0;
    W[c1 + (nz - 1) * P] = w1;
    return;
  }
  blk -= G.nz_blocks;
  // ---- top and wall rows of the interior columns, thread (i, k): (4), (5) ----
  const int i = (blk % G.yi_tiles) * 32 + tx + 2, k = (blk / G.yi_tiles) * 8 + ty + 1;
  if (i > nxg - 2 || k > nzg) return;
  const bool du = i <= nx - 2, dw = k <= nz;
  const T u2 = du ? U[bidx(g, i, 2, X::ks_uv(g, k))] : (T)0, w2 = dw ? W[bidx(g, i, 2, X::ks_w(g, k))] : (T)0;
  if (du) {
    U[bidx(g, i, nyg, k)] = (T)bc.U_top[i];
    U[bidx(g, i, 1, k)] = X::wall_u(g, bc, u2, i, k);
  }
  V[bidx(g, i, ny, k)] = (T)bc.V_top[i];
  V[bidx(g, i, 1, k)] = (T)0;
  if (dw) {
    W[bidx(g, i, nyg, k)] = (T)bc.W_top[i];
    W[bidx(g, i, 1, k)] = X::wall_w(g, bc, w2, i, k);
  }
}

template <typename T>
__global__ void k_bc_mass(Geo g, T *__restrict__ U, const Scalars *__restrict__ sc) {
  // :240-260: the correction the last x-plane block of k_bc_all left in sc->dU
  const double s_du = sc->dU;
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 1;
  if (j > g.nyg || k > g.nzg) return;
  long long a = bidx(g, g.nx - 1, j, k);
  const T v = (T)((double)U[a] + s_du);
  U[a] = v;
  U[a + 1] = v;
}

// ---------------------------------------------------------------------------
// compute_dt: max over i=2..nxg-1, j=2..nyg-1, k=2..nzg-1 of spacing/|vel|
// (time_integration.f90:546-556).  All ratios are >= 0 (or +Inf), so the
// maximum of their IEEE bit patterns is their maximum and atomicMax is exact
// and order independent.
// ---------------------------------------------------------------------------
// dt from the maxima of the reduction (time_integration.f90:580-590), by the
// last block to finish: the arrival counter after every block's atomics
__device__ __forceinline__ void dt_finish_last(Scalars *sc, double cfl, double dtvis, int save_time) {
  __threadfence();
  const unsigned int nb = gridDim.x * gridDim.y * gridDim.z;
  if (atomicAdd(&sc->dt_arrived, 1u) != nb - 1) return;
  __threadfence();
  const double cfla = fabs(cfl);
  const double lu = __longlong_as_double((long long)atomicOr(&sc->lmax[0], 0ull));
  const double lv = __longlong_as_double((long long)atomicOr(&sc->lmax[1], 0ull));
  const double lw = __longlong_as_double((long long)atomicOr(&sc->lmax[2], 0ull));
  const double dt_conv = fmin(fmin(cfla * lu, cfla * lv), cfla * lw);
  sc->dt = fmin(dt_conv, dtvis);
  sc->lmax[0] = sc->lmax[1] = sc->lmax[2] = 0ull;
  sc->dt_arrived = 0u;
  if (save_time) sc->to = sc->t;  // the step's start time (k_set_time phase 0)
}

template <typename T>
__global__ void __launch_bounds__(256) k_dt_reduce(Geo g, const T *__restrict__ U, const T *__restrict__ V,
                                                   const T *__restrict__ W, Scalars *__restrict__ sc, int kchunk,
                                                   double cfl, double dtvis, int save_time) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  double mu = 0.0, mv = 0.0, mw = 0.0;
  if (i <= g.nxg - 1 && j <= g.nyg - 1) {
    const int k0 = blockIdx.z * kchunk + 2;
    const int k1 = min(k0 + kchunk - 1, g.nzg - 1);
    const double cu = g.ax.C[i], cv = g.ay.C[j];
    // a thread keeps i and j, so max_k C/|u_k| = C / min_k |u_k| (division
    // is monotone: the same double as the per-point maximum)
    double au = INFINITY, av = INFINITY, aw = INFINITY;
    for (int k = k0; k <= k1; ++k) {
      long long c = bidx(g, i, j, k);
      au = fmin(au, fabs((double)__ldg(U + c)));
      av = fmin(av, fabs((double)__ldg(V + c)));
      if (sizeof(T) == 8) mw = fmax(mw, g.az.C[k] / fabs((double)__ldg(W + c)));
      else aw = fmin(aw, fabs((double)__ldg(W + c)) * g.az.rC[k]);  // mixed form: 1/max(C/|w|)
    }
    if (k1 >= k0) {
      mu = cu / au;
      mv = cv / av;
      if (sizeof(T) != 8) mw = 1.0 / aw;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    mu = fmax(mu, __shfl_xor_sync(0xffffffffu, mu, o));
    mv = fmax(mv, __shfl_xor_sync(0xffffffffu, mv, o));
    mw = fmax(mw, __shfl_xor_sync(0xffffffffu, mw, o));
  }
  // one atomic per block and field (the maxima are order-free, so the
  // result is deterministic); per-warp atomics on three words serialise
  __shared__ double red[3][8];
  const int wid = (threadIdx.y * blockDim.x + threadIdx.x) >> 5, nwarp = (blockDim.x * blockDim.y) >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][wid] = mu;
    red[1][wid] = mv;
    red[2][wid] = mw;
  }
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    for (int w = 1; w < nwarp; ++w) {
      mu = fmax(mu, red[0][w]);
      mv = fmax(mv, red[1][w]);
      mw = fmax(mw, red[2][w]);
    }
    atomicMax(&sc->lmax[0], (unsigned long long)__double_as_longlong(mu));
    atomicMax(&sc->lmax[1], (unsigned long long)__double_as_longlong(mv));
    atomicMax(&sc->lmax[2], (unsigned long long)__double_as_longlong(mw));
    dt_finish_last(sc, cfl, dtvis, save_time);
  }
}

// The FP64 reduction with two consecutive points per thread (16-byte loads;
// the box rows are 16-byte aligned at i = 2) and the k loop unrolled.  For
// w the quotient C_k/|w_k| is formed only where it can raise the maximum:
// a_k = |w_k| rC_k is within 3e-16 of |w_k|/C_k, so a point whose a_k
// exceeds the smallest a seen so far by more than 1e-12 (relative) has a
// quotient below that point's, and the maximum of the formed quotients is
// the maximum of all of them, to the bit.
template <typename T>  // double
__global__ void __launch_bounds__(256) k_dt_reduce2(Geo g, const T *__restrict__ U, const T *__restrict__ V,
                                                    const T *__restrict__ W, Scalars *__restrict__ sc, int kchunk,
                                                    double cfl, double dtvis, int save_time) {
  const int i0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  double mu = 0.0, mv = 0.0, mw = 0.0;
  if (i0 <= g.nxg - 1 && j <= g.nyg - 1) {
    const int k0 = blockIdx.z * kchunk + 2;
    const int k1 = min(k0 + kchunk - 1, g.nzg - 1);
    double au[2] = {INFINITY, INFINITY}, av[2] = {INFINITY, INFINITY}, bw[2] = {INFINITY, INFINITY};
    double qw[2] = {0.0, 0.0};
    const double2 *u2 = reinterpret_cast<const double2 *>(U + bidx(g, i0, j, k0));
    const double2 *v2 = reinterpret_cast<const double2 *>(V + bidx(g, i0, j, k0));
    const double2 *w2 = reinterpret_cast<const double2 *>(W + bidx(g, i0, j, k0));
    const long long ps = g.plane / 2;
#pragma unroll 4
    for (int k = k0; k <= k1; ++k) {
      const long long o = (long long)(k - k0) * ps;
      const double2 u = __ldg(u2 + o), v = __ldg(v2 + o), w = __ldg(w2 + o);
      const double rc = g.az.rC[k];
      const double uu[2] = {u.x, u.y}, vv[2] = {v.x, v.y}, ww[2] = {w.x, w.y};
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        au[e] = fmin(au[e], fabs(uu[e]));
        av[e] = fmin(av[e], fabs(vv[e]));
        const double a = fabs(ww[e]) * rc;
        if (a <= bw[e] * (1.0 + 1e-12)) {
          qw[e] = fmax(qw[e], g.az.C[k] / fabs(ww[e]));
          bw[e] = fmin(bw[e], a);
        }
      }
    }
    if (k1 >= k0) {
      const double cv = g.ay.C[j];
#pragma unroll
      for (int e = 0; e < 2; ++e)
        if (i0 + e <= g.nxg - 1) {
          mu = fmax(mu, g.ax.C[i0 + e] / au[e]);
          mv = fmax(mv, cv / av[e]);
          mw = fmax(mw, qw[e]);
        }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    mu = fmax(mu, __shfl_xor_sync(0xffffffffu, mu, o));
    mv = fmax(mv, __shfl_xor_sync(0xffffffffu, mv, o));
    mw = fmax(mw, __shfl_xor_sync(0xffffffffu, mw, o));
  }
  __shared__ double red[3][8];
  const int wid = (threadIdx.y * blockDim.x + threadIdx.x) >> 5, nwarp = (blockDim.x * blockDim.y) >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][wid] = mu;
    red[1][wid] = mv;
    red[2][wid] = mw;
  }
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    for (int w = 1; w < nwarp; ++w) {
      mu = fmax(mu, red[0][w]);
      mv = fmax(mv, red[1][w]);
      mw = fmax(mw, red[2][w]);
    }
    atomicMax(&sc->lmax[0], (unsigned long long)__double_as_longlong(mu));
    atomicMax(&sc->lmax[1], (unsigned long long)__double_as_longlong(mv));
    atomicMax(&sc->lmax[2], (unsigned long long)__double_as_longlong(mw));
    dt_finish_last(sc, cfl, dtvis, save_time);
  }
}

// The same reduction for the mixed form with four consecutive points per
// thread (16-byte loads; the box rows are 16-byte aligned at i = 2) and the
// k loop unrolled, so that a thread keeps a dozen loads in flight.
template <typename T>  // float
__global__ void __launch_bounds__(256) k_dt_reduce4(Geo g, const T *__restrict__ U, const T *__restrict__ V,
                                                    const T *__restrict__ W, Scalars *__restrict__ sc, int kchunk,
                                                    double cfl, double dtvis, int save_time) {
  const int i0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x) + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  double mu = 0.0, mv = 0.0, mw = 0.0;
  if (i0 <= g.nxg - 1 && j <= g.nyg - 1) {
    const int k0 = blockIdx.z * kchunk + 2;
    const int k1 = min(k0 + kchunk - 1, g.nzg - 1);
    float au[4], av[4];
    double aw[4];  // min |w| / C in double, as k_dt_reduce
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      au[e] = av[e] = INFINITY;
      aw[e] = INFINITY;
    }
    const float4 *u4 = reinterpret_cast<const float4 *>(U + bidx(g, i0, j, k0));
    const float4 *v4 = reinterpret_cast<const float4 *>(V + bidx(g, i0, j, k0));
    const float4 *w4 = reinterpret_cast<const float4 *>(W + bidx(g, i0, j, k0));
    const long long ps = g.plane / 4;
#pragma unroll 4
    for (int k = k0; k <= k1; ++k) {
      const long long o = (long long)(k - k0) * ps;
      const float4 u = __ldg(u4 + o), v = __ldg(v4 + o), w = __ldg(w4 + o);
      const double rC = g.az.rC[k];
      const float uu[4] = {u.x, u.y, u.z, u.w}, vv[4] = {v.x, v.y, v.z, v.w}, ww[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        au[e] = fminf(au[e], fabsf(uu[e]));
        av[e] = fminf(av[e], fabsf(vv[e]));
        aw[e] = fmin(aw[e], fabs((double)ww[e]) * rC);
      }
    }
    if (k1 >= k0) {
      const double cv = g.ay.C[j];
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (i0 + e <= g.nxg - 1) {
          mu = fmax(mu, g.ax.C[i0 + e] / (double)au[e]);
          mv = fmax(mv, cv / (double)av[e]);
          mw = fmax(mw, 1.0 / aw[e]);
        }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    mu = fmax(mu, __shfl_xor_sync(0xffffffffu, mu, o));
    mv = fmax(mv, __shfl_xor_sync(0xffffffffu, mv, o));
    mw = fmax(mw, __shfl_xor_sync(0xffffffffu, mw, o));
  }
  __shared__ double red[3][8];
  const int wid = (threadIdx.y * blockDim.x + threadIdx.x) >> 5, nwarp = (blockDim.x * blockDim.y) >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][wid] = mu;
    red[1][wid] = mv;
    red[2][wid] = mw;
  }
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    for (int w = 1; w < nwarp; ++w) {
      mu = fmax(mu, red[0][w]);
      mv = fmax(mv, red[1][w]);
      mw = fmax(mw, red[2][w]);
    }
    atomicMax(&sc->lmax[0], (unsigned long long)__double_as_longlong(mu));
    atomicMax(&sc->lmax[1], (unsigned long long)__double_as_longlong(mv));
    atomicMax(&sc->lmax[2], (unsigned long long)__double_as_longlong(mw));
    dt_finish_last(sc, cfl, dtvis, save_time);
  }
}

// time_integration.f90:560-575 (dt = min(dt_conv, dt_vis)); also arms the
// accumulators for the next call and records to = t for the RK substeps.

#ifdef BLGPU_STENCIL_PRIMARY
__global__ void k_set_time(Scalars *sc, int phase, double coef) {
  // phase 0: to = t (save at step start); phase 1: t = to + coef*dt
  if (phase == 0) sc->to = sc->t;
  else sc->t = sc->to + coef * sc->dt;
}
#endif

// check_divergence (projection.f90:399-408): max |div| over i=2..nxg-2
template <typename T>
__global__ void __launch_bounds__(256) k_maxdiv(Geo g, const T *__restrict__ U, const T *__restrict__ V,
                                                const T *__restrict__ W, unsigned long long *__restrict__ out,
                                                int kchunk) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  double mx = 0.0;
  if (i <= g.nxg - 2 && j <= g.nyg - 1) {
    const int k0 = blockIdx.z * kchunk + 2;
    const int k1 = min(k0 + kchunk - 1, g.nzg - 1);
    for (int k = k0; k <= k1; ++k) {
      long long c = bidx(g, i, j, k);
      double d = ((double)U[c] - (double)U[c - 1]) / g.ax.F[i] + ((double)V[c] - (double)V[c - g.px]) / g.ay.F[j] +
                 ((double)W[c] - (double)W[c - g.plane]) / g.az.F[k];
      mx = max_keep_nan(mx, fabs(d));
    }
  }
  for (int o = 16; o > 0; o >>= 1) mx = max_keep_nan(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  // |d| >= 0 and a positive NaN's bit pattern is above +Inf's, so the largest
  // pattern is the maximum and a NaN anywhere wins
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(mx));
}

// ---------------------------------------------------------------------------
// Constant-coefficient Smagorinsky eddy viscosity (subgrid.f90:609-662) with
// the rate of strain of compute_Sij (subgrid.f90:672-730): diagonal terms at
// the cell centre, off-diagonal terms on the cell edges averaged to the
// centre, |S| = sqrt(2 Sij Sij).  cs2[j] = (Cs Delta_j f)^2 with
// Delta_j = (dx dz (y(j)-y(j-1)))^(1/3) and f = 1 (Dirichlet_nu_t is forced 0,
// initialization.f90:586).  Interior points i=2..nxg-1, j=2..nyg-1,
// k=2..nzg-1 only.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T sij4(const Geo &g, const T *U, const T *V, int i, int j, int k) {
  const long long c = bidx(g, i, j, k);
  return (T)0.5 * ((U[c - 1] - U[c - 1 - g.px]) / (T)(g.yg[j] - g.yg[j - 1]) +
                   (V[c - g.px] - V[c - 1 - g.px]) / (T)(g.xg[i] - g.xg[i - 1]));
}
template <typename T>
__device__ __forceinline__ T sij5(const Geo &g, const T *U, const T *W, int i, int j, int k) {
  const long long c = bidx(g, i, j, k);
  return (T)0.5 * ((U[c - 1] - U[c - 1 - g.plane]) / (T)(g.zg[k] - g.zg[k - 1]) +
                   (W[c - g.plane] - W[c - 1 - g.plane]) / (T)(g.xg[i] - g.xg[i - 1]));
}
template <typename T>
__device__ __forceinline__ T sij6(const Geo &g, const T *V, const T *W, int i, int j, int k) {
  const long long c = bidx(g, i, j, k);
  return (T)0.5 * ((V[c - g.px] - V[c - g.px - g.plane]) / (T)(g.zg[k] - g.zg[k - 1]) +
                   (W[c - g.plane] - W[c - g.px - g.plane]) / (T)(g.yg[j] - g.yg[j - 1]));
}

template <typename T>
__global__ void __launch_bounds__(256) k_smagorinsky(Geo g, const T *__restrict__ U, const T *__restrict__ V,
                                                     const T *__restrict__ W, const double *__restrict__ cs2,
                                                     T *__restrict__ nut) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k = blockIdx.z + 2;
  if (i > g.nxg - 1 || j > g.nyg - 1 || k > g.nzg - 1) return;
  const long long c = bidx(g, i, j, k);
  const T s1 = (U[c] - U[c - 1]) / (T)(g.x[i] - g.x[i - 1]);
  const T s2 = (V[c] - V[c - g.px]) / (T)(g.y[j] - g.y[j - 1]);
  const T s3 = (W[c] - W[c - g.plane]) / (T)(g.z[k] - g.z[k - 1]);
  const T q = (T)0.25;
  const T s4 = q * (sij4<T>(g, U, V, i, j, k) + sij4<T>(g, U, V, i + 1, j, k) + sij4<T>(g, U, V, i, j + 1, k) +
                    sij4<T>(g, U, V, i + 1, j + 1, k));
  const T s5 = q * (sij5<T>(g, U, W, i, j, k) + sij5<T>(g, U, W, i + 1, j, k) + sij5<T>(g, U, W, i, j, k + 1) +
                    sij5<T>(g, U, W, i + 1, j, k + 1));
  const T s6 = q * (sij6<T>(g, V, W, i, j, k) + sij6<T>(g, V, W, i, j + 1, k) + sij6<T>(g, V, W, i, j, k + 1) +
                    sij6<T>(g, V, W, i, j + 1, k + 1));
  T S = 0;
  S = S + (T)2 * s1 * s1;
  S = S + (T)2 * s2 * s2;
  S = S + (T)2 * s3 * s3;
  S = S + (T)4 * s4 * s4;
  S = S + (T)4 * s5 * s5;
  S = S + (T)4 * s6 * s6;
  nut[c] = (T)cs2[j] * sqrt(S);
}

// ---------------------------------------------------------------------------
// z-averaged statistics of statistics.f90:37-80, FP64 accumulators in the
// source's summation order: for ii=1..nx, jj=1..ny the sums over k of the
// y-interpolated U, the x-interpolated V, the xy-interpolated W, their
// squares, U*V, P, P^2 and nu_t.  out: 9 (nx,ny) arrays + nu_t_mean(nxg,nyg)
// + the wall sums of U at j = 1, 2 (2 x nx).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_stats(Geo g, const T *__restrict__ U, const T *__restrict__ V, const T *__restrict__ W,
                        const T *__restrict__ P, const T *__restrict__ nut, double *__restrict__ out) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y + 1;
  if (ii > g.nx || jj > g.ny) return;
  const int nx = g.nx, ny = g.ny;
  const double w0 = g.w0[jj], w1 = g.w1[jj];
  double su = 0, sv = 0, sw = 0, su2 = 0, sv2 = 0, sw2 = 0, suv = 0, sp = 0, sp2 = 0, sn = 0;
  for (int k = 2; k <= g.nzg - 1; ++k) {
    const long long c = bidx(g, ii, jj, k);
    const double t1 = w0 * (double)U[c] + w1 * (double)U[c + g.px];
    const double t2 = 0.5 * ((double)V[c] + (double)V[c + 1]);
    su += t1;
    sv += t2;
    su2 += t1 * t1;
    sv2 += t2 * t2;
    suv += t1 * t2;
    const double pv = (double)P[c];
    sp += pv;
    sp2 += pv * pv;
    if (nut) sn += (double)nut[c];
  }
  for (int k = 1; k <= g.nz - 2; ++k) {
    const long long c = bidx(g, ii, jj, k);
    const double a = 0.5 * ((double)W[c] + (double)W[c + 1]);
    const double b = 0.5 * ((double)W[c + g.px] + (double)W[c + g.px + 1]);
    const double t = w0 * a + w1 * b;
    sw += t;
    sw2 += t * t;
  }
  const long long pl = (long long)nx * ny, q = (long long)(jj - 1) * nx + (ii - 1);
  const double dn = (double)(g.nzg - 2), dw = (double)(g.nz - 2);
  out[q] = su / dn;
  out[q + pl] = sv / dn;
  out[q + 2 * pl] = sw / dw;
  out[q + 3 * pl] = su2 / dn;
  out[q + 4 * pl] = sv2 / dn;
  out[q + 5 * pl] = sw2 / dw;
  out[q + 6 * pl] = suv / dn;
  out[q + 7 * pl] = sp / dn;
  out[q + 8 * pl] = sp2 / dn;
  out[9 * pl + (long long)(jj - 1) * g.nxg + (ii - 1)] = sn / dn;
  if (jj <= 2) {  // wall sums of statistics.f90:138-146
    double a = 0.0;
    for (int k = 2; k <= g.nzg - 1; ++k) a += (double)U[bidx(g, ii, jj, k)];
    out[9 * pl + (long long)g.nxg * g.nyg + (long long)(jj - 1) * nx + (ii - 1)] = a / dn;
  }
}

// ---------------------------------------------------------------------------
// equilibrium law of the wall at each x (wallmodel.f90:1951-1985) solved with
// Newton_iter_solver (Newton_solver.f90:13-79): kappa = 0.38, B = 5.2,
// y = yg(jref) (jref = 3 in the reference), at most 30 iterations, stop when
// |f| < 1e-10.  utau holds the
// initial guess on entry (the previous model) and the model on exit; iters
// receives the iteration count of each x.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_law_of_wall(Geo g, const T *__restrict__ U, double *__restrict__ utau, int *__restrict__ iters,
                              int jref) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  if (i > g.nx - 1) return;
  const double kap = 0.38, B = 5.20, yref = g.yg[jref], nu = g.nu;
  double x = utau[i - 1];
  double um = 0.0;
  for (int k = 2; k <= g.nzg - 1; ++k) um += (double)U[bidx(g, i, jref, k)];
  um = um / (double)(g.nzg - 2);
  int k;
  for (k = 1; k <= 30; ++k) {
    const double fx = x / kap * log(yref * x / nu) + B * x - um;
    const double fp = 1.0 / kap * log(yref * x / nu) + 1.0 / kap + B;
    if (fabs(fx) < 1e-10) break;
    x = x - fx / fp;
  }
  utau[i - 1] = (x != x) ? 0.0 : x;
  iters[i - 1] = k - 1;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static inline dim3 vol_grid(int ni, int nj, int nk, int kchunk, int by = 8) {
  return dim3((ni + 31) / 32, (nj + by - 1) / by, (nk + kchunk - 1) / kchunk);
}

#ifndef BLGPU_STENCIL_PRIMARY
// planes of U, V, W as (px, py, nzg) FP32 tensors: boxes of 72 x 10 x 1
// (neighbourhood tiles) and 64 x 8 x 1 (point-wise tiles)
bool rhs_maps(const Geo &g, const float *U, const float *V, const float *W, RhsMaps *out) {
  const cuuint64_t dims[3] = {(cuuint64_t)g.px, (cuuint64_t)g.py, (cuuint64_t)g.nzg};
  const cuuint64_t strides[2] = {(cuuint64_t)g.px * 4, (cuuint64_t)g.plane * 4};
  const cuuint32_t fbox[3] = {RT_TW, RT_TH, 1}, pbox[3] = {64, RT_BY, 1};
  const float *a[3] = {U, V, W};
  for (int q = 0; q < 3; ++q) {
    CUtensorMap mf, mp;
    if (!tma::encode(&mf, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(a[q]), dims, strides, fbox) ||
        !tma::encode(&mp, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(a[q]), dims, strides, pbox))
      return false;
    static_assert(sizeof(CUtensorMap) == sizeof(out->f[0]), "tensor map size");
    memcpy(out->f[q], &mf, sizeof mf);
    memcpy(out->p[q], &mp, sizeof mp);
  }
  return true;
}
#endif

#ifdef BLGPU_STENCIL_PRIMARY
// planes of U, V, W as (px, py, nzg) FP64 tensors: boxes of 36 x 10 x 1
// (neighbourhood tiles) and 32 x 8 x 1 (point-wise tiles)
bool rhs_maps64(const Geo &g, const double *U, const double *V, const double *W, RhsMaps *out) {
  const cuuint64_t dims[3] = {(cuuint64_t)g.px, (cuuint64_t)g.py, (cuuint64_t)g.nzg};
  const cuuint64_t strides[2] = {(cuuint64_t)g.px * 8, (cuuint64_t)g.plane * 8};
  const cuuint32_t fbox[3] = {R64_TW, R64_TH, 1}, pbox[3] = {32, R64_BY, 1};
  const double *a[3] = {U, V, W};
  for (int q = 0; q < 3; ++q) {
    CUtensorMap mf, mp;
    if (!tma::encode(&mf, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double *>(a[q]), dims, strides, fbox) ||
        !tma::encode(&mp, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double *>(a[q]), dims, strides, pbox))
      return false;
    memcpy(out->f[q], &mf, sizeof mf);
    memcpy(out->p[q], &mp, sizeof mp);
  }
  return true;
}
#endif

template <int MODE>
static void launch_rhs_tma64(const Geo &g, const MetT<double> &m, const RhsMaps &mi, const RhsMaps &mo,
                             const RhsMaps &mf, double *F1u, double *F1v, double *F1w, double *Un, double *Vn,
                             double *Wn, const Scalars *sc, double c1, double c2, int kc, int *err, int wait_limit,
                             cudaStream_t st) {
  CUtensorMap t[9];
  for (int q = 0; q < 3; ++q) {
    memcpy(&t[q], mi.f[q], sizeof(CUtensorMap));
    memcpy(&t[3 + q], mo.p[q], sizeof(CUtensorMap));
    memcpy(&t[6 + q], mf.p[q], sizeof(CUtensorMap));
  }
  const size_t sm = r64_smem(MODE);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_rhs_rk_tma64<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    attr = true;
  }
  const dim3 grid = vol_grid(g.nx - 1, g.ny - 1, g.nz - 1, kc, R64_BY);
  k_rhs_rk_tma64<MODE><<<grid, dim3(32, R64_BY), sm, st>>>(t[0], t[1], t[2], t[3], t[4], t[5], t[6], t[7], t[8], g,
                                                           m, F1u, F1v, F1w, Un, Vn, Wn, sc, c1, c2, kc, err,
                                                           wait_limit < 0 ? tma::WAIT_LIMIT : wait_limit);
}

template <int MODE>
static void launch_rhs_tma(const Geo &g, const MetT<float> &m, const RhsMaps &mi, const RhsMaps &mo,
                           const RhsMaps &mf, float *F1u, float *F1v, float *F1w, float *Un, float *Vn, float *Wn,
                           const Scalars *sc, double c1, double c2, int kc, int *err, int wait_limit,
                           cudaStream_t st) {
  CUtensorMap t[9];
  for (int q = 0; q < 3; ++q) {
    memcpy(&t[q], mi.f[q], sizeof(CUtensorMap));
    memcpy(&t[3 + q], mo.p[q], sizeof(CUtensorMap));
    memcpy(&t[6 + q], mf.p[q], sizeof(CUtensorMap));
  }
  const size_t sm = rt_smem(MODE);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_rhs_rk_tma<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    attr = true;
  }
  const dim3 grid = vol_grid(g.nx / 2, g.ny - 1, g.nz - 1, kc, RT_BY);
  k_rhs_rk_tma<MODE><<<grid, dim3(32, RT_BY), sm, st>>>(t[0], t[1], t[2], t[3], t[4], t[5], t[6], t[7], t[8], g, m,
                                                        F1u, F1v, F1w, Un, Vn, Wn, sc, c1, c2, kc, err,
                                                        wait_limit < 0 ? tma::WAIT_LIMIT : wait_limit);
}

template <typename T>
void launch_rhs_rk(const Geo &g, const MetT<T> &m, int mode, bool les, const T *U, const T *V, const T *W,
                   const T *nut, const T *Uo, const T *Vo, const T *Wo, T *F1u, T *F1v, T *F1w, T *Un, T *Vn, T *Wn,
                   const Scalars *sc, double c1, double c2, const Tiles &tl, const RhsMaps *mi, const RhsMaps *mo,
                   const RhsMaps *mf, int *err, int wait_limit, cudaStream_t st) {
  const int kchunk = tl.rhs_kc > 0 ? tl.rhs_kc : 8;
  const int by = tl.rhs_by > 0 ? tl.rhs_by : 8;
  dim3 grid = vol_grid(g.nx - 1, g.ny - 1, g.nz - 1, kchunk, by), block(32, by);
#define BLGPU_RHS_CASE(M, L)                                                                             \
  k_rhs_rk<T, M, L><<<grid, block, 0, st>>>(g, m, U, V, W, nut, Uo, Vo, Wo, F1u, F1v, F1w, Un, Vn, Wn, sc, c1, \
                                            c2, kchunk)
  if (!les && sizeof(T) == 4) {  // FP32: register-window kernel (FP64 keeps the lower-register form)
    const bool pair = tl.rhs_pts != 1;
    // the TMA-fed kernel serves the default where its maps exist (16 planes
    // per CTA: the two extra planes a chunk reads cost 1/8 of its loads)
    const bool tma_fed = (tl.rhs_pts == 4 || tl.rhs_pts == 0) && mi && mo && mf;
    const int kc = tl.rhs_kc > 0 ? tl.rhs_kc : (tma_fed ? 16 : pair ? 8 : 32);
    // pairs cover i = 2..nx two points at a time
    dim3 gd = vol_grid(pair ? g.nx / 2 : g.nx - 1, g.ny - 1, g.nz - 1, kc, by);
#define BLGPU_DNS_CASE(M)                                                                                           \
  do {                                                                                                              \
    if constexpr (sizeof(T) == 4) {                                                                                 \
      if (tma_fed) {                                                                                                \
        launch_rhs_tma<M>(g, m, *mi, *mo, *mf, F1u, F1v, F1w, Un, Vn, Wn, sc, c1, c2, kc, err, wait_limit, st);     \
        break;                                                                                                      \
      }                                                                                                             \
      if (tl.rhs_pts == 3) {                                                                                        \
        k_rhs_rk_pk<M><<<gd, block, 0, st>>>(g, m, U, V, W, Uo, Vo, Wo, F1u, F1v, F1w, Un, Vn, Wn, sc, c1, c2, kc); \
        break;                                                                                                      \
      }                                                                                                             \
    }                                                                                                               \
    if (pair)                                                                                                       \
      k_rhs_rk_pair<T, M><<<gd, block, 0, st>>>(g, m, U, V, W, Uo, Vo, Wo, F1u, F1v, F1w, Un, Vn, Wn, sc, c1, c2, kc); \
    else                                                                                                            \
      k_rhs_rk_dns<T, M><<<gd, block, 0, st>>>(g, m, U, V, W, Uo, Vo, Wo, F1u, F1v, F1w, Un, Vn, Wn, sc, c1, c2, kc);  \
  } while (0)
    switch (mode) {
      case 0: BLGPU_DNS_CASE(0); break;
      case 1: BLGPU_DNS_CASE(1); break;
      case 2: BLGPU_DNS_CASE(2); break;
      default: BLGPU_DNS_CASE(3); break;
    }
#undef BLGPU_DNS_CASE
  } else if (!les) {
    if constexpr (sizeof(T) == 8) {
      // FP64 DNS: the TMA-fed kernel (results bit-identical to k_rhs_rk) where
      // its maps exist, unless rhs_pts = 1 asks for the global-load kernel
      // FP64 DNS: the two-point register window (rhs_pts 0 or 2, bit-identical to
      // k_rhs_rk: its shared and carried terms are the same expressions), the
      // TMA-fed one-point kernel (rhs_pts 4) or the global-load kernel (1)
      if (tl.rhs_pts == 2 || tl.rhs_pts == 0) {
        const int kc = tl.rhs_kc > 0 ? tl.rhs_kc : 16;
        dim3 gd = vol_grid(g.nx / 2, g.ny - 1, g.nz - 1, kc, 8);
        dim3 blk(32, 8);
        switch (mode) {
          case 0: k_rhs_rk_pair<T, 0><<<gd, blk, 0, st>>>(g, m, U, V, W, Uo, Vo, Wo, F1u, F1v, F1w, Un, Vn, Wn, sc, c1, c2, kc); break;
          case 1: k_rhs_rk_pair<T, 1><<<gd, blk, 0, st>>>(g, m, U, V, W, Uo, Vo, Wo, F1u, F1v, F1w, Un, Vn, Wn, sc, c1, c2, kc); break;
          case 2: k_rhs_rk_pair<T, 2><<<gd, blk, 0, st>>>(g, m, U, V, W, Uo, Vo, Wo, F1u, F1v, F1w, Un, Vn, Wn, sc, c1, c2, kc); break;
          default: k_rhs_rk_pair<T, 3><<<gd, blk, 0, st>>>(g, m, U, V, W, Uo, Vo, Wo, F1u, F1v, F1w, Un, Vn, Wn, sc, c1, c2, kc); break;
        }
        return;
      }
      if (tl.rhs_pts == 4 && mi && mo && mf) {
        const int kc = tl.rhs_kc > 0 ? tl.rhs_kc : 32;
        switch (mode) {
          case 0: launch_rhs_tma64<0>(g, m, *mi, *mo, *mf, F1u, F1v, F1w, Un, Vn, Wn, sc, c1, c2, kc, err, wait_limit, st); break;
          case 1: launch_rhs_tma64<1>(g, m, *mi, *mo, *mf, F1u, F1v, F1w, Un, Vn, Wn, sc, c1, c2, kc, err, wait_limit, st); break;
          case 2: launch_rhs_tma64<2>(g, m, *mi, *mo, *mf, F1u, F1v, F1w, Un, Vn, Wn, sc, c1, c2, kc, err, wait_limit, st); break;
          default: launch_rhs_tma64<3>(g, m, *mi, *mo, *mf, F1u, F1v, F1w, Un, Vn, Wn, sc, c1, c2, kc, err, wait_limit, st); break;
        }
        return;
      }
    }
    switch (mode) {
      case 0: BLGPU_RHS_CASE(0, false); break;
      case 1: BLGPU_RHS_CASE(1, false); break;
      case 2: BLGPU_RHS_CASE(2, false); break;
      default: BLGPU_RHS_CASE(3, false); break;
    }
  } else {
    switch (mode) {
      case 0: BLGPU_RHS_CASE(0, true); break;
      case 1: BLGPU_RHS_CASE(1, true); break;
      case 2: BLGPU_RHS_CASE(2, true); break;
      default: BLGPU_RHS_CASE(3, true); break;
    }
  }
#undef BLGPU_RHS_CASE
}

template <typename T>
void launch_project(const Geo &g, const MetT<T> &m, const T *p, const double *p0, const float *p0g, T *U, T *V,
                    T *W, T *P,
                    const Scalars *sc, int save_p, const Tiles &tl, cudaStream_t st) {
  constexpr int VN = 16 / sizeof(T);
  const int ngrp = (g.nx - 1 + VN - 1) / VN;  // i = 2..nx in groups of VN
  const int by = tl.proj_by > 0 ? tl.proj_by : 4;  // 4 rows: the autotuner's choice at 814 x 257 x 193 in both precisions
  dim3 block(32, by), grid((ngrp + 31) / 32, (g.ny - 1 + by - 1) / by, g.nz - 1);
  k_project_v<T><<<grid, block, 0, st>>>(g, m, p, p0, p0g, U, V, W, P, sc, save_p);
  if (save_p) {
    const int bx = ((g.nyg + 31) / 32) * ((g.nzg + 7) / 8), by = ((g.nxg + 31) / 32) * ((g.nzg + 7) / 8);
    const int bz = ((g.nxg + 31) / 32) * ((g.nyg + 7) / 8);
    k_p_ghost<T><<<bx + by + bz, 256, 0, st>>>(g, P, bx, by);
  }
}

#ifdef BLGPU_STENCIL_PRIMARY
int bc_x_parts(const Geo &g) { return ((g.nyg + 31) / 32) * ((g.nzg + 7) / 8); }
#endif

template <typename T>
void launch_bc(const Geo &g, const BcData &bc, T *U, T *V, T *W, const T *Uo, const T *Vo, const T *Wo,
               Scalars *sc, double rkt, double *qx_part, double qy, double length_y, cudaStream_t st) {
  BcGrid G;
  G.x_tiles = (g.nyg + 31) / 32;
  G.nx_blocks = G.x_tiles * ((g.nzg + 7) / 8);  // = bc_x_parts(g)
  G.zi_tiles = (g.nxg - 3 + 31) / 32;           // interior columns i = 2..nxg-2
  G.nz_blocks = G.zi_tiles * ((g.nyg - 2 + 7) / 8);
  G.yi_tiles = G.zi_tiles;
  G.ny_blocks = G.yi_tiles * ((g.nzg + 7) / 8);
  k_bc_all<T><<<3 * G.nx_blocks + G.nz_blocks + G.ny_blocks, 256, 0, st>>>(g, bc, G, U, V, W, Uo, Vo, Wo, sc, rkt,
                                                                         qx_part, qy, length_y);
  k_bc_mass<T><<<dim3((g.nyg + 31) / 32, (g.nzg + 7) / 8), dim3(32, 8), 0, st>>>(g, U, sc);
}

template <typename T>
void launch_dt(const Geo &g, const T *U, const T *V, const T *W, Scalars *sc, double cfl, double dtvis,
               bool save_time, cudaStream_t st) {
  const int kchunk = 32;
  // 16-byte vectors: rows of 4 floats / 2 doubles from i = 2 (element i + 2 of a row)
  const bool vec = (g.px & (sizeof(T) == 4 ? 3 : 1)) == 0 &&
                   ((reinterpret_cast<uintptr_t>(U) | reinterpret_cast<uintptr_t>(V) | reinterpret_cast<uintptr_t>(W)) &
                    15) == 0;
  if (vec) {
    if constexpr (sizeof(T) == 4) {
      dim3 grid = vol_grid((g.nxg - 2 + 3) / 4, g.nyg - 2, g.nzg - 2, kchunk), block(32, 8);
      k_dt_reduce4<T><<<grid, block, 0, st>>>(g, U, V, W, sc, kchunk, cfl, dtvis, save_time ? 1 : 0);
    } else {
      dim3 grid = vol_grid((g.nxg - 2 + 1) / 2, g.nyg - 2, g.nzg - 2, kchunk), block(32, 8);
      k_dt_reduce2<T><<<grid, block, 0, st>>>(g, U, V, W, sc, kchunk, cfl, dtvis, save_time ? 1 : 0);
    }
  }
  if (!vec) {
    dim3 grid = vol_grid(g.nxg - 2, g.nyg - 2, g.nzg - 2, kchunk), block(32, 8);
    k_dt_reduce<T><<<grid, block, 0, st>>>(g, U, V, W, sc, kchunk, cfl, dtvis, save_time ? 1 : 0);
  }
}

#ifdef BLGPU_STENCIL_PRIMARY
void launch_set_time(Scalars *sc, int phase, double coef, cudaStream_t st) {
  k_set_time<<<1, 1, 0, st>>>(sc, phase, coef);
}
#endif

template <typename T>
void launch_maxdiv(const Geo &g, const T *U, const T *V, const T *W, unsigned long long *out, cudaStream_t st) {
  const int kchunk = 16;
  dim3 grid = vol_grid(g.nxg - 3, g.nyg - 2, g.nzg - 2, kchunk), block(32, 8);
  k_maxdiv<T><<<grid, block, 0, st>>>(g, U, V, W, out, kchunk);
}

template <typename T>
void launch_smagorinsky(const Geo &g, const T *U, const T *V, const T *W, const double *cs2, T *nut, cudaStream_t st) {
  dim3 block(32, 8), grid((g.nxg - 2 + 31) / 32, (g.nyg - 2 + 7) / 8, g.nzg - 2);
  k_smagorinsky<T><<<grid, block, 0, st>>>(g, U, V, W, cs2, nut);
}

template <typename T>
void launch_stats(const Geo &g, const T *U, const T *V, const T *W, const T *P, const T *nut, double *out,
                  cudaStream_t st) {
  dim3 block(32, 8), grid((g.nx + 31) / 32, (g.ny + 7) / 8);
  k_stats<T><<<grid, block, 0, st>>>(g, U, V, W, P, nut, out);
}

template <typename T>
void launch_law_of_wall(const Geo &g, const T *U, double *utau, int *iters, int jref, cudaStream_t st) {
  k_law_of_wall<T><<<(g.nx + 127) / 128, 128, 0, st>>>(g, U, utau, iters, jref);
}

#define BLGPU_INST(T)                                                                                                \
  template void launch_rhs_rk<T>(const Geo &, const MetT<T> &, int, bool, const T *, const T *, const T *,          \
                                 const T *, const T *, const T *, const T *, T *, T *, T *, T *, T *, T *,          \
                                 const Scalars *, double, double, const Tiles &, const RhsMaps *, const RhsMaps *,  \
                                 const RhsMaps *, int *, int, cudaStream_t);                                        \
  template void launch_project<T>(const Geo &, const MetT<T> &, const T *, const double *, const float *, T *,    \
                                  T *, T *, T *,                                                                    \
                                  const Scalars *, int, const Tiles &, cudaStream_t);                               \
  template void launch_bc<T>(const Geo &, const BcData &, T *, T *, T *, const T *, const T *, const T *,         \
                             Scalars *, double, double *, double, double, cudaStream_t);                            \
  template void launch_dt<T>(const Geo &, const T *, const T *, const T *, Scalars *, double, double, bool,        \
                             cudaStream_t);                                                                         \
  template void launch_maxdiv<T>(const Geo &, const T *, const T *, const T *, unsigned long long *, cudaStream_t); \
  template void launch_smagorinsky<T>(const Geo &, const T *, const T *, const T *, const double *, T *,            \
                                      cudaStream_t);                                                                \
  template void launch_stats<T>(const Geo &, const T *, const T *, const T *, const T *, const T *, double *,       \
                                cudaStream_t);                                                                      \
  template void launch_law_of_wall<T>(const Geo &, const T *, double *, int *, int, cudaStream_t);
BLGPU_INST(BLGPU_STENCIL_T)

}  // namespace blgpu

namespace blgpu {

// ---------------------------------------------------------------------------
// host-layout <-> box-layout repack (the Fortran arrays of the reference,
// staged as FP64 in device memory, to and from the padded box in precision T)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_repack_in(Geo g, const double *__restrict__ src, int n1, int n2, int n3, T *__restrict__ dst,
                            int *flag) {
  const long long tot = (long long)n1 * n2 * n3;
  bool bad = false;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % n1);
    const long long r = q / n1;
    const int j = (int)(r % n2), k = (int)(r / n2);
    const double v = src[q];
    bad |= !isfinite(v);
    dst[bidx(g, i + 1, j + 1, k + 1)] = (T)v;
  }
  // a NaN or infinity in the host state: bit 32 of the device flag
  if (flag && __any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 32);
}

template <typename T>
__global__ void k_repack_out(Geo g, const T *__restrict__ src, int n1, int n2, int n3, double *__restrict__ dst) {
  const long long tot = (long long)n1 * n2 * n3;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % n1);
    const long long r = q / n1;
    const int j = (int)(r % n2), k = (int)(r / n2);
    dst[q] = (double)src[bidx(g, i + 1, j + 1, k + 1)];
  }
}

template <typename T>
void launch_repack(const Geo &g, int dir, double *stage, T *box, int n1, int n2, int n3, int *flag, cudaStream_t st) {
  const int blocks = 148 * 8;
  if (dir == 0) k_repack_in<T><<<blocks, 256, 0, st>>>(g, stage, n1, n2, n3, box, flag);
  else k_repack_out<T><<<blocks, 256, 0, st>>>(g, box, n1, n2, n3, stage);
}
template void launch_repack<BLGPU_STENCIL_T>(const Geo &, int, double *, BLGPU_STENCIL_T *, int, int, int, int *,
                                             cudaStream_t);

}  // namespace blgpu

#ifdef BLGPU_STENCIL_PRIMARY
namespace blgpu {

// ---------------------------------------------------------------------------
// Lund recycling/rescaling inflow (rescaled_inlet_bc.f90:60-345), evaluated
// once per step from the step's starting fields (the Uo, Vo, Wo of
// boundary_conditions.f90:569-597).  All arithmetic is FP64 in this
// translation unit (no FMA contraction), whatever the storage type T.
//
// k_lund_sums: one block per z-mean row (:109-125, :218-222); the 128
// partial sums are combined in a fixed tree order.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(128) k_lund_sums(Geo g, LundData L, const T *__restrict__ U,
                                                   const T *__restrict__ V) {
  const int r = blockIdx.x, nyg = g.nyg, ny = g.ny;
  double s = 0.0;
  for (int k = 2 + threadIdx.x; k <= g.nzg - 1; k += blockDim.x) {
    double v;
    if (r < nyg) v = (double)U[bidx(g, L.ir, r + 1, k)];
    else if (r < 2 * nyg) v = (double)U[bidx(g, 1, r - nyg + 1, k)];
    else if (r < 2 * nyg + ny) v = (double)V[bidx(g, L.ir, r - 2 * nyg + 1, k)];
    else if (r < 2 * nyg + 2 * ny) v = (double)V[bidx(g, 1, r - 2 * nyg - ny + 1, k)];
    else v = 0.5 * ((double)U[bidx(g, L.ir, 1, k)] + (double)U[bidx(g, L.ir, 2, k)]) * (double)V[bidx(g, L.ir, 1, k)];
    s += v;
  }
  __shared__ double red[128];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 64; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) L.inst[r] = red[0] / (double)(g.nzg - 2);
}

// one warp: the first row j with Um >= Umean99 by ballots over 32 rows at a
// time (the same row as a serial scan), then the interpolation
__device__ double lund_delta99(const double *Um, const double *yg, int nyg, double Umean99) {
  const int lane = threadIdx.x & 31;
  int jref = 0;
  for (int j0 = 1; j0 <= nyg && !jref; j0 += 32) {
    const int j = j0 + lane;
    const unsigned hit = __ballot_sync(0xffffffffu, j <= nyg && Um[j - 1] >= Umean99);
    if (hit) jref = j0 + __ffs(hit) - 1;
  }
  if (jref < 2) jref = nyg / 2;
  const double w1 = (Umean99 - Um[jref - 2]) / (Um[jref - 1] - Um[jref - 2]);
  const double w0 = 1.0 - w1;
  const double d = w1 * yg[jref] + w0 * yg[jref - 1];
  return d < 0 ? fabs(d) : d;
}

// one warp: trapezoidal momentum thickness, lane partial sums combined by a
// butterfly (every lane returns the same value)
__device__ double lund_theta(const double *Um, const double *yg, int nyg, double Uinf) {
  const int lane = threadIdx.x & 31;
  double th = 0.0;
  for (int j = 2 + lane; j <= nyg; j += 32) {
    const double a = Um[j - 1] / Uinf * (1.0 - Um[j - 1] / Uinf), b = Um[j - 2] / Uinf * (1.0 - Um[j - 2] / Uinf);
    th = th + 0.5 * (a + b) * (yg[j] - yg[j - 1]);
  }
  for (int o = 16; o > 0; o >>= 1) th += __shfl_xor_sync(0xffffffffu, th, o);
  return th < 0 ? fabs(th) : th;
}

// source / target coordinate of row k of map m (:235-246)
__device__ __forceinline__ double lund_coord(const Geo &g, int m, int k, double scale_w, double scale_d) {
  const double *y = (m < 2) ? g.yg : g.y;
  return (m & 1) ? y[k] / scale_d : scale_w * y[k] / g.nu;
}

// k_lund_rows: one block.  Running means (:133-137), thicknesses, friction
// velocities and gamma (:153-231) on thread 0, then per row the
// interpolation pair of interp_vel (:305-345), the blending weights
// (:248-251) and the inner/outer mean profiles (:255-263, :285-289).
__global__ void __launch_bounds__(256) k_lund_rows(Geo g, LundData L, const Scalars *__restrict__ sc) {
  const int nyg = g.nyg, ny = g.ny, tid = threadIdx.x, nt = blockDim.x;
  const double ra = sc->dt / L.T_resc, rb = 1.0 - sc->dt / L.T_resc;
  for (int q = tid; q < 2 * nyg + 2 * ny; q += nt) L.mean[q] = ra * L.inst[q] + rb * L.mean[q];
  __syncthreads();
  __shared__ double sh[8];
  const double *Umr = L.mean, *Umi = L.mean + nyg, *Vmr = L.mean + 2 * nyg;
  // the four serial scans run on four warps at once
  const double Uinf = L.inst[nyg - 1];
  {
    const int w = tid >> 5;  // warps 0-3, one scan each
    double r = 0.0;
    if (w == 0) r = lund_delta99(Umr, g.yg, nyg, 0.99 * Uinf);
    if (w == 1) r = lund_delta99(Umi, g.yg, nyg, 0.99 * Uinf);
    if (w == 2) r = lund_theta(Umr, g.yg, nyg, Uinf);
    if (w == 3) r = lund_theta(Umi, g.yg, nyg, Uinf);
    if (w < 4 && (tid & 31) == 0) sh[1 + w] = r;
  }
  __syncthreads();
  if (tid == 0) {
    const double th_r = sh[3], th_i = sh[4];
    const double uv = L.inst[2 * nyg + 2 * ny];
    const double dUw = (Umr[1] - Umr[0]) / (g.yg[2] - g.yg[1]);
    const double ut_r = sqrt(fabs(g.nu * dUw - uv));
    const double ut_i = ut_r * pow(th_r / th_i, 1.0 / 8.0);
    const double gam = ut_i / ut_r;
    sh[0] = Uinf;
    sh[5] = ut_r;
    sh[6] = ut_i;
    sh[7] = gam;
    for (int q = 0; q < 8; ++q) L.diag[q] = sh[q];
  }
  __syncthreads();
  const double d_resc = sh[1], ut_r = sh[5], ut_i = sh[6], gam = sh[7];
  const double alpha = 4.0, bb = 0.2;
  for (int q = tid; q < 4 * nyg; q += nt) {
    const int m = q / nyg, i = q % nyg + 1;  // target row i of map m
    const int n1 = (m < 2) ? nyg : ny;
    if (i > n1) continue;
    int j = -1;
    double coef = 0.0;
    if (i > 1) {
      const double yi = lund_coord(g, m, i, ut_i, L.delta_inlet);
      // first k in 1..n1 with ys(k) > yi; ys is non-decreasing in k, so a
      // bisection finds the same k as the reference's forward scan
      int lo = 1, hi = n1 + 1;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (lund_coord(g, m, mid, ut_r, d_resc) > yi) hi = mid;
        else lo = mid + 1;
      }
      j = lo <= n1 ? lo : 0;
      if (j == 1) { atomicOr(L.err, 1); j = 0; }
      if (j > 0) {
        const double ysj = lund_coord(g, m, j, ut_r, d_resc), ysm = lund_coord(g, m, j - 1, ut_r, d_resc);
        coef = (ysj - yi) / (ysj - ysm);
      }
    }
    L.rowi[q] = j;
    L.rowc[q] = coef;
    // mean profile through the same pair
    const double *src = (m < 2) ? Umr : Vmr;
    double v = 0.0;
    if (j == 0) v = src[n1 - 1];
    else if (j > 0) v = coef * src[j - 2] + (1.0 - coef) * src[j - 1];
    if (m == 0) v = gam * v;
    else if (m == 1) v = gam * v + (1.0 - gam) * Uinf;
    if (L.mode == 5) v = 0.0;  // iflag_fluc = 1 (:285-290)
    L.mprof[q] = v;
    if (m == 0 || m == 2) {  // inner/outer weight of row i (:248-251)
      const double e = ((m == 0) ? g.yg[i] : g.y[i]) / L.delta_inlet;
      L.wgt[(m == 0 ? 0 : nyg) + i - 1] = 0.5 * (1.0 + tanh(alpha * (e - bb) / ((1.0 - 2.0 * bb) * e + bb)) / tanh(alpha));
    }
  }
}

// fluctuation at source row r of the station plane (the mean removed for U, V)
template <typename T>
__device__ __forceinline__ double lund_src(const Geo &g, const LundData &L, const T *F, const double *mean, int r,
                                           int k) {
  const double v = (double)F[bidx(g, L.ir, r, k)];
  return mean ? v - mean[r - 1] : v;
}

template <typename T>
__device__ __forceinline__ double lund_interp(const Geo &g, const LundData &L, int q, int n1, const T *F,
                                              const double *mean, int k) {
  const int j = L.rowi[q];
  if (j < 0) return 0.0;
  if (j == 0) return lund_src<T>(g, L, F, mean, n1, k);
  const double c = L.rowc[q];
  return c * lund_src<T>(g, L, F, mean, j - 1, k) + (1.0 - c) * lund_src<T>(g, L, F, mean, j, k);
}

// k_lund_plane: the blended inflow planes (:287-298)
template <typename T>
__global__ void k_lund_plane(Geo g, LundData L, const T *__restrict__ U, const T *__restrict__ V,
                             const T *__restrict__ W) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int nyg = g.nyg, ny = g.ny;
  if (j > nyg || k > g.nzg) return;
  const double gam = L.diag[7];
  const double *Umr = L.mean, *Vmr = L.mean + 2 * nyg;
  const double wg = L.wgt[j - 1];
  {
    const double fi = lund_interp<T>(g, L, j - 1, nyg, U, Umr, k);
    const double fo = lund_interp<T>(g, L, nyg + j - 1, nyg, U, Umr, k);
    L.lu[(long long)(k - 1) * nyg + (j - 1)] =
        (L.mprof[j - 1] + gam * fi) * (1.0 - wg) + (L.mprof[nyg + j - 1] + gam * fo) * wg;
  }
  if (k <= g.nz) {
    const double fi = lund_interp<T>(g, L, j - 1, nyg, W, nullptr, k);
    const double fo = lund_interp<T>(g, L, nyg + j - 1, nyg, W, nullptr, k);
    L.lw[(long long)(k - 1) * nyg + (j - 1)] = (gam * fi) * (1.0 - wg) + (gam * fo) * wg;
  }
  if (j <= ny) {
    const double wv = L.wgt[nyg + j - 1];
    const double fi = lund_interp<T>(g, L, 2 * nyg + j - 1, ny, V, Vmr, k);
    const double fo = lund_interp<T>(g, L, 3 * nyg + j - 1, ny, V, Vmr, k);
    L.lv[(long long)(k - 1) * ny + (j - 1)] =
        (L.mprof[2 * nyg + j - 1] + gam * fi) * (1.0 - wv) + (L.mprof[3 * nyg + j - 1] + gam * fo) * wv;
  }
}

// phase 0: z-means only (start-up of the running means); 1: full evaluation
template <typename T>
void launch_lund(const Geo &g, const LundData &L, const T *U, const T *V, const T *W, const Scalars *sc, int phase,
                 cudaStream_t st) {
  k_lund_sums<T><<<2 * g.nyg + 2 * g.ny + 1, 128, 0, st>>>(g, L, U, V);
  if (phase == 0) return;
  k_lund_rows<<<1, 256, 0, st>>>(g, L, sc);
  k_lund_plane<T><<<dim3((g.nyg + 31) / 32, (g.nzg + 7) / 8), dim3(32, 8), 0, st>>>(g, L, U, V, W);
}
template void launch_lund<double>(const Geo &, const LundData &, const double *, const double *, const double *,
                                  const Scalars *, int, cudaStream_t);
template void launch_lund<float>(const Geo &, const LundData &, const float *, const float *, const float *,
                                 const Scalars *, int, cudaStream_t);

}  // namespace blgpu
#endif
