// ysolve.cuh -- the row recurrences of the y-solve (Thomas algorithm on the
// tridiagonal operator of solve_poisson_gpu, projection.f90:137-150, whose
// factors initialization.f90:428-469 precomputes), with every rounding
// spelled out, so that each kernel that forms them -- the pivot table, the
// register ring, the TMA tiles, the cuFFT comparison path and the tiles that
// recompute their pivots -- produces the same bits.
//
// Row b (= j-2) of mode (kx, kz): diagonal d_b = (dd_b + kxx) + kzz (times
// 3/2 for b = 0 of the (0,0) mode, initialization.f90:454), sub-diagonal
// dl_b, super-diagonal du_b.  Elimination:
//   w_b   = dl_b piv_{b-1}                 (b > 0)
//   d'_b  = d_b - w_b du_{b-1}             piv_b = 1 / d'_b
//   g_b   = r_b - w_b g_{b-1}
//   x_b   = (g_b - du_b x_{b+1}) piv_b     (x_{NM-1} = g_{NM-1} piv_{NM-1})
#pragma once

#include <cuda_runtime.h>

namespace blgpu {

__device__ __forceinline__ double ys_diag(double dd_b, double kxx, double kzz, bool mode00_row0) {
  const double d = __dadd_rn(__dadd_rn(dd_b, kxx), kzz);
  return mode00_row0 ? __dmul_rn(1.5, d) : d;
}
__device__ __forceinline__ double ys_w(double dl_b, double piv_prev) { return __dmul_rn(dl_b, piv_prev); }
// inverse pivot of a row, w = 0 and du_prev unused for b = 0
__device__ __forceinline__ double ys_piv(double d_b, double w, double du_prev, bool first) {
  return __drcp_rn(first ? d_b : __fma_rn(-w, du_prev, d_b));
}
__device__ __forceinline__ double ys_fwd(double r, double w, double g_prev) { return __fma_rn(-w, g_prev, r); }
__device__ __forceinline__ double ys_bwd(double g, double du_b, double x_next, double piv) {
  return __dmul_rn(__fma_rn(-du_b, x_next, g), piv);
}
__device__ __forceinline__ double ys_top(double g, double piv) { return __dmul_rn(g, piv); }

}  // namespace blgpu
