// noalloc.cu -- check_divergence on arrays the caller already holds on the
// device, with no device allocation by the library.
//
// Who needs it: a host that owns every device array itself and must not (or
// cannot) call cudaMalloc -- the reference's own OpenACC program is one, as
// its U, V, W, x, y, z live in an !$acc data region and reach foreign code
// only as device addresses (host_data use_device), and so is code running
// under a pool allocator or inside a region where allocation is forbidden.
// Such a caller passes its device arrays in the reference layout and a
// device address for the result; the scratch this reduction needs (one
// partial maximum per (j,k) row) is a fixed file-scope __device__ array.
//
// Limits and rules of use:
//  - at most BLGPU_NOALLOC_MAX_ROWS = 65536 rows, i.e. (ny-1)*(nz-1) <= 65536;
//    larger grids are rejected with BLGPU_EINVAL;
//  - the scratch (512 KiB) is held by every device that loads the library
//    until the process exits;
//  - the first call on a device looks up the scratch address on that device
//    (cudaGetSymbolAddress) -- make that first call before any stream capture;
//  - all calls share the one scratch array: calls that overlap on the GPU
//    (different streams, different host threads) race; every row slot a call
//    reads is written by the same call first, so stale contents of an earlier
//    call are never used;
//  - a NaN anywhere in the divergence gives a NaN result.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/blgpu.h"

namespace blgpu {
void set_global_error(const char *msg);
}

namespace {

constexpr int kMaxRows = 65536;
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_row_max[kMaxRows];

std::mutex g_setup_mutex;
double *g_row_max_addr[kMaxDevices] = {};

// max that keeps a NaN (fmax would drop it), so that a NaN divergence reads as
// NaN, as it does through the context's check (blgpu_max_divergence)
__device__ __forceinline__ double max_nan(double a, double b) { return (a > b || a != a) ? a : b; }

// one warp per (j,k) row: max over i = 2..nxg-2 of |div u| (projection.f90:399-408)
__global__ void k_row_divmax(const double *__restrict__ U, const double *__restrict__ V,
                             const double *__restrict__ W, const double *__restrict__ x,
                             const double *__restrict__ y, const double *__restrict__ z, int nx, int ny, int nz,
                             double *__restrict__ rows) {
  const int nxg = nx + 1, nyg = ny + 1, nzg = nz + 1;
  const int nj = nyg - 2, nk = nzg - 2;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= nj * nk) return;
  const int j = 2 + warp % nj, k = 2 + warp / nj;
  // Fortran layouts: U(nx,nyg,nzg), V(nxg,ny,nzg), W(nxg,nyg,nz), 1-based
  const long long ub = ((long long)(k - 1) * nyg + (j - 1)) * nx;
  const long long vb = ((long long)(k - 1) * ny + (j - 1)) * nxg, vbs = vb - nxg;
  const long long wb = ((long long)(k - 1) * nyg + (j - 1)) * nxg, wbs = wb - (long long)nyg * nxg;
  const double dy = y[j - 1] - y[j - 2], dz = z[k - 1] - z[k - 2];
  double m = 0.0;
  for (int i = 2 + lane; i <= nxg - 2; i += 32) {
    const double d = (U[ub + i - 1] - U[ub + i - 2]) / (x[i - 1] - x[i - 2]) + (V[vb + i - 1] - V[vbs + i - 1]) / dy +
                     (W[wb + i - 1] - W[wbs + i - 1]) / dz;
    m = max_nan(m, fabs(d));
  }
  for (int o = 16; o > 0; o >>= 1) m = max_nan(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) rows[warp] = m;
}

__global__ void k_rows_max(const double *__restrict__ rows, int nrows, double *__restrict__ out) {
  __shared__ double red[32];
  double m = 0.0;
  for (int r = threadIdx.x; r < nrows; r += blockDim.x) m = max_nan(m, rows[r]);
  for (int o = 16; o > 0; o >>= 1) m = max_nan(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = max_nan(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) out[0] = m;
  }
}

int fail(int code, const char *msg) {
  blgpu::set_global_error(msg);
  return code;
}

}  // namespace

extern "C" int blgpu_check_divergence_noalloc(const double *U, const double *V, const double *W, const double *x,
                                              const double *y, const double *z, int nx, int ny, int nz,
                                              double *max_div, void *stream) {
  if (!U || !V || !W || !x || !y || !z || !max_div)
    return fail(BLGPU_EINVAL, "blgpu_check_divergence_noalloc: null device pointer");
  if (nx < 5 || ny < 4 || nz < 5) return fail(BLGPU_EINVAL, "blgpu_check_divergence_noalloc: grid too small");
  const long long nrows = (long long)(ny - 1) * (nz - 1);
  if (nrows > kMaxRows)
    return fail(BLGPU_EINVAL,
                "blgpu_check_divergence_noalloc: (ny-1)*(nz-1) exceeds the 65536-row scratch of this entry point");
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fail(BLGPU_ECUDA, "blgpu_check_divergence_noalloc: no current CUDA device");
  double *rows = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_row_max_addr[dev]) {
      // set-up on first use on this device (this device is current)
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_row_max);
      if (e != cudaSuccess || !p)
        return fail(BLGPU_ECUDA, "blgpu_check_divergence_noalloc: cudaGetSymbolAddress of the scratch failed");
      g_row_max_addr[dev] = static_cast<double *>(p);
    }
    rows = g_row_max_addr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int warps_per_block = 8;
  const int blocks = (int)((nrows + warps_per_block - 1) / warps_per_block);
  k_row_divmax<<<blocks, 32 * warps_per_block, 0, st>>>(U, V, W, x, y, z, nx, ny, nz, rows);
  k_rows_max<<<1, 1024, 0, st>>>(rows, (int)nrows, max_div);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(BLGPU_ECUDA, "blgpu_check_divergence_noalloc: kernel launch failed");
  return BLGPU_OK;
}
