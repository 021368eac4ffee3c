// common.cuh -- device layout and shared definitions of the B200 step path.
//
// Every 3D field (U, V, W, P, rhs_p and the RK stage F1) lives in one padded
// "box" layout in HBM: k-planes of py rows of px elements, i fastest, with
// the reference's 1-based Fortran indices (i,j,k) mapped to
//     ((k-1)*py + (j-1))*px + (i+2).
// px is nxg+8 rounded up to 32 elements, so every row starts on a 256-byte
// (FP64) or 128-byte (FP32) boundary; the shift by 2 puts the first interior
// point i = 2 on a 16-byte boundary, so 16-byte vector loads of a row
// segment i = 2+4q .. 5+4q (FP32) or 2+2q .. 3+2q (FP64) are aligned; py = nyg.
// The reference's arrays U(nx,nyg,nzg), V(nxg,ny,nzg), W(nxg,nyg,nz) and
// P(nxg,nyg,nzg) (global.f90:86-88) are all sub-boxes of this one shape.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace blgpu {

// Per-axis metric tables, 1-based like the Fortran arrays (index 0 unused).
//   F[i] = x(i) - x(i-1)        (face spacing)
//   C[i] = xg(i+1) - xg(i)      (centre spacing)
//   rF[i] = 1/F[i], rC[i] = 1/C[i]
// The reference writes its viscous terms as 1d0/dx*(...) in some places and
// (...)/dx in others (equations.f90:88-91); the reciprocal tables serve the
// first form only, so the FP64 path rounds exactly like the source.
struct Axis {
  const double *F, *C, *rF, *rC;
};

struct Geo {
  int nx, ny, nz;       // face points
  int nxg, nyg, nzg;    // nx+1, ny+1, nz+1
  int px, py;           // box pitches (elements)
  long long plane;      // px*py
  Axis ax, ay, az;
  const double *w0, *w1;  // weight_y_0/1 (initialization.f90:482-484), 1-based
  const double *x, *xg, *y, *yg, *z, *zg;  // raw grids, 1-based
  double nu, dpdx, dpdz;
};

// a / b, correctly rounded, from rb = RN(1/b) (the host's 1.0/b) by
// Markstein's correction (P. W. Markstein, IBM J. Res. Dev. 34, 1990; "IA-64
// and Elementary Functions", 2000, Thm. 8.10): q = RN(a rb) is within one
// ulp of a/b, the remainder a - b q is exact in one fused multiply-add, and
// RN(q + (a - b q) rb) is RN(a/b), for operands far from overflow and
// underflow.  One multiply and two fused multiply-adds in place of the
// division sequence; the FP64 kernels divide through it wherever the source
// divides by a grid spacing whose reciprocal is tabulated.
__device__ __forceinline__ double mdiv(double a, double b, double rb) {
  const double q = __dmul_rn(a, rb);
  return __fma_rn(__fma_rn(-q, b, a), rb, q);
}

__host__ __device__ inline long long bidx(const Geo &g, int i, int j, int k) {
  return ((long long)(k - 1) * g.py + (j - 1)) * (long long)g.px + (i + 2);
}

// Device-resident scalars of the running time step.  Kernels read dt and t
// from here so that a whole step can be captured in a CUDA graph and replayed
// without host round trips.
struct Scalars {
  double t;        // current time
  double to;       // time at the start of the step
  double dt;       // time step
  double dU;       // last mass-flux correction
  unsigned long long lmax[3];  // compute_dt maxima (bit patterns of >=0 doubles)
  int err;         // sticky device error flag
  unsigned int dt_arrived;  // blocks of the compute_dt reduction that have finished (the last one resets it)
};

template <typename T> struct vec2;
template <> struct vec2<double> { typedef double2 type; };
template <> struct vec2<float> { typedef float2 type; };

}  // namespace blgpu

#define BLGPU_CUDA_OK(expr)                                   \
  do {                                                        \
    cudaError_t _e = (expr);                                  \
    if (_e != cudaSuccess) return ::blgpu::fail_cuda(_e, #expr, __FILE__, __LINE__); \
  } while (0)
