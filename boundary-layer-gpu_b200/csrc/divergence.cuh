// divergence.cuh -- the pseudo-pressure right-hand side of the projection,
// rhs_p = dU/dx + dV/dy + dW/dz at cell (i,j,k) (projection.f90:38-47), as
// every forward transform of the Poisson solve evaluates it.
#pragma once

#include "common.cuh"

namespace blgpu {

// FP64: the source's divisions (correctly rounded, through mdiv); FP32:
// products with the reciprocal spacing
__device__ __forceinline__ double dq(double a, double F, double rF) { return mdiv(a, F, rF); }
__device__ __forceinline__ float dq(float a, double, double rF) { return a * (float)rF; }

// c = bidx(g, i, j, k)
template <typename T>
__device__ __forceinline__ T div_at(const Geo &g, const T *__restrict__ U, const T *__restrict__ V,
                                    const T *__restrict__ W, long long c, int i, int j, int k) {
  // projection.f90:42-44
  return dq(__ldg(U + c) - __ldg(U + c - 1), g.ax.F[i], g.ax.rF[i]) +
         dq(__ldg(V + c) - __ldg(V + c - g.px), g.ay.F[j], g.ay.rF[j]) +
         dq(__ldg(W + c) - __ldg(W + c - g.plane), g.az.F[k], g.az.rF[k]);
}

}  // namespace blgpu
