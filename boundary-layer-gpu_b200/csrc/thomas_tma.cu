// thomas_tma.cu -- the y-solve of the Poisson equation (the tridiagonal
// systems of solve_poisson_gpu, projection.f90:155-189, with the precomputed
// inverse pivots of k_thomas_factors) as one pass over the spectral data.
//
// A CTA owns a tile of MT consecutive kx of one kz over all NM rows b: one
// TMA tensor copy brings the tile of C and one the tile of the pivots into
// shared memory, lane l solves mode kx0+l there (forward sweep, then the
// backward sweep over the forward results, both in shared memory), and one
// TMA store writes the tile back.  C is read once and written once and the
// pivots are read once; the sweeps of the register-ring kernel read both
// twice.  Several CTAs per SM keep copies of other tiles in flight while a
// tile is solved.
#include <cstring>

#include "kernels.cuh"
#include "tma.cuh"

namespace blgpu {

using namespace tma;

template <typename T> using T2t = typename vec2<T>::type;
template <typename T> __device__ __forceinline__ T2t<T> mk2(T a, T b) {
  T2t<T> r;
  r.x = a;
  r.y = b;
  return r;
}

// modes per tile: 128-byte rows of C (16 FP32 or 8 FP64 complex values)
template <typename T> struct ThomasTile { static constexpr int MT = 64 / (int)sizeof(T); };

template <typename T>
__host__ __device__ inline size_t tile_c_bytes(int NM) {
  return ((size_t)NM * ThomasTile<T>::MT * 2 * sizeof(T) + 127) / 128 * 128;
}
template <typename T>
__host__ __device__ inline size_t tile_p_bytes(int NM) {
  return ((size_t)NM * ThomasTile<T>::MT * sizeof(double) + 127) / 128 * 128;
}

// tiles, the dl/du vectors and the mbarrier
template <typename T>
inline size_t thomas_tile_smem(int NM) {
  return tile_c_bytes<T>(NM) + tile_p_bytes<T>(NM) + 2 * (size_t)NM * sizeof(double) + sizeof(uint64_t);
}

// The solve of one tile in shared memory with each mode's NM rows split
// over P = 32 / MT lanes (lane = kk MT + m: a row's modes are one 128-byte
// run, read without bank conflicts).  Both recurrences are first-order and
// linear,
//   g_b = r_b - w_b g_{b-1} (w_b = dl_b piv_{b-1}),  x_b = (g_b - du_b x_{b+1}) piv_b,
// so lane kk runs them over its rows [kk Le, kk Le + Le) from a zero start,
// keeping the product of its multipliers (-w_b forward, beta_b = -du_b piv_b
// backward); an inclusive shuffle scan of these affine maps over kk gives
// each lane the value entering its rows, and a second pass adds the product
// times that value.  The sums are those of the serial sweeps, reassociated
// across the P segments.
template <typename T>
__device__ __forceinline__ void thomas_scan_tile(T2t<T> *Ct, const double *Pt, const double *dls,
                                                 const double *dus, int NM, int kx0, int N, int lane) {
  constexpr int MT = ThomasTile<T>::MT, P = 32 / MT;
  constexpr unsigned FULL = 0xffffffffu;
  typedef T2t<T> V2;
  const int m = lane % MT, kk = lane / MT;
  const bool act = kx0 + m < N;
  const int Le = (NM + P - 1) / P, s0 = kk * Le;
  const int nr = act ? max(0, min(Le, NM - s0)) : 0;
  V2 *c = Ct + (size_t)s0 * MT + m;
  const double *p = Pt + (size_t)s0 * MT + m;
  // forward from g = 0 at the segment's start
  double gx = 0.0, gy = 0.0, h = 1.0;
  for (int u = 0; u < nr; ++u) {
    const int b = s0 + u;
    const V2 cv = c[u * MT];
    double rx = (double)cv.x, ry = (double)cv.y;
    double w = 0.0;
    if (b > 0) {
      w = dls[b] * p[(u - 1) * MT];  // l_b / d'_{b-1}
      rx = rx - w * gx;
      ry = ry - w * gy;
    }
    h = -w * h;
    gx = rx;
    gy = ry;
    c[u * MT] = mk2<T>((T)rx, (T)ry);
  }
  double A = h, Cx = gx, Cy = gy;
#pragma unroll
  for (int off = 1; off < P; off <<= 1) {
    const double a2 = __shfl_up_sync(FULL, A, off * MT);
    const double x2 = __shfl_up_sync(FULL, Cx, off * MT), y2 = __shfl_up_sync(FULL, Cy, off * MT);
    if (kk >= off) {
      Cx = Cx + A * x2;
      Cy = Cy + A * y2;
      A = A * a2;
    }
  }
  double ix = __shfl_up_sync(FULL, Cx, MT), iy = __shfl_up_sync(FULL, Cy, MT);
  if (kk == 0) ix = iy = 0.0;
  h = 1.0;
  for (int u = 0; u < nr; ++u) {
    const int b = s0 + u;
    const double w = b > 0 ? dls[b] * p[(u - 1) * MT] : 0.0;
    h = -w * h;
    const V2 cv = c[u * MT];
    c[u * MT] = mk2<T>((T)((double)cv.x + h * ix), (T)((double)cv.y + h * iy));
  }
  // backward from x = 0 above the segment's top row
  double xx = 0.0, xy = 0.0, kp = 1.0;
  for (int u = nr - 1; u >= 0; --u) {
    const int b = s0 + u;
    const V2 cv = c[u * MT];
    const double pv = p[u * MT];
    double beta = 0.0;
    if (b == NM - 1) {
      xx = (double)cv.x * pv;
      xy = (double)cv.y * pv;
    } else {
      xx = ((double)cv.x - dus[b] * xx) * pv;
      xy = ((double)cv.y - dus[b] * xy) * pv;
      beta = -dus[b] * pv;
    }
    kp = beta * kp;
    c[u * MT] = mk2<T>((T)xx, (T)xy);
  }
  A = kp;
  Cx = xx;
  Cy = xy;
#pragma unroll
  for (int off = 1; off < P; off <<= 1) {
    const double a2 = __shfl_down_sync(FULL, A, off * MT);
    const double x2 = __shfl_down_sync(FULL, Cx, off * MT), y2 = __shfl_down_sync(FULL, Cy, off * MT);
    if (kk + off < P) {
      Cx = Cx + A * x2;
      Cy = Cy + A * y2;
      A = A * a2;
    }
  }
  ix = __shfl_down_sync(FULL, Cx, MT);
  iy = __shfl_down_sync(FULL, Cy, MT);
  if (kk == P - 1) ix = iy = 0.0;
  kp = 1.0;
  for (int u = nr - 1; u >= 0; --u) {
    const int b = s0 + u;
    const double beta = b == NM - 1 ? 0.0 : -dus[b] * p[u * MT];
    kp = beta * kp;
    const V2 cv = c[u * MT];
    c[u * MT] = mk2<T>((T)((double)cv.x + kp * ix), (T)((double)cv.y + kp * iy));
  }
}

// SCAN: the rows of a mode split over P = 32 / MT lanes (FP32 2, FP64 4;
// lane = kk MT + m), each lane running both recurrences over its segment
// of the tile from a zero start with the product of its multipliers, the
// segments joined by shuffle scans of those affine maps (see
// thomas_scan_tile), so that every lane of the warp works and the serial
// chains are P times shorter.
template <typename T, bool SCAN>
__global__ void __launch_bounds__(32) k_thomas_tile(const __grid_constant__ CUtensorMap mapC,
                                                    const __grid_constant__ CUtensorMap mapP, Spec s,
                                                    const double *__restrict__ dl, const double *__restrict__ du,
                                                    double *__restrict__ H0, int klow, int *__restrict__ err,
                                                    int wait_limit) {
  constexpr int MT = ThomasTile<T>::MT;
  typedef T2t<T> V2;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int NM = s.NM;
  V2 *Ct = reinterpret_cast<V2 *>(smem_raw);                                   // [NM][MT]
  double *Pt = reinterpret_cast<double *>(smem_raw + tile_c_bytes<T>(NM));     // [NM][MT]
  double *dls = reinterpret_cast<double *>(smem_raw + tile_c_bytes<T>(NM) + tile_p_bytes<T>(NM));  // [NM]
  double *dus = dls + NM;                                                                          // [NM]
  uint64_t *bar = reinterpret_cast<uint64_t *>(dus + NM);
  const int kx0 = blockIdx.x * MT, kz = blockIdx.y, lane = threadIdx.x;
  const uint32_t bytes = (uint32_t)((size_t)NM * MT * (2 * sizeof(T) + sizeof(double)));
  if (lane == 0) {
    mbar_init(bar, 1);
    mbar_init_fence();
    mbar_expect_tx(bar, bytes);
    load_3d(Ct, &mapC, 2 * kx0, kz, 0, bar);
    load_3d(Pt, &mapP, kx0, kz, 0, bar);
  }
  for (int b = lane; b < NM; b += 32) {
    dls[b] = dl[b];
    dus[b] = du[b];
  }
  __syncwarp();
  // wait_limit polls (the context's test hook may shorten it); after giving
  // up, the drain waits with the normal limit, so no copy into this CTA's
  // shared memory is in flight when it leaves
  const bool ok = mbar_wait(bar, 0, wait_limit);
  if (!__all_sync(0xffffffffu, ok)) {
    if (lane == 0) {
      atomicOr(err, 4);
      mbar_wait(bar, 0);
    }
    return;
  }
  if (SCAN && !(H0 && kz == 0 && kx0 < klow)) {
    thomas_scan_tile<T>(Ct, Pt, dls, dus, NM, kx0, s.N, lane);
  } else {
  const int kx = kx0 + lane;
  if (lane < MT && kx < s.N) {
    V2 *c = Ct + lane;
    const double *p = Pt + lane;
    if (H0 && kz == 0 && kx < klow) {
      // mixed form: the box-scale modes in FP64 into H0[b][kx]; their FP32
      // slots are cleared (the imaginary part of kz = 0 is zero)
      double *Hd = H0 + kx;
      double g = 0.0, rprev = 0.0;
      for (int b = 0; b < NM; ++b) {
        double r = (double)c[b * MT].x;
        if (b > 0) r = r - (dls[b] * rprev) * g;
        rprev = p[b * MT];
        g = r;
        Hd[(long long)b * klow] = r;
      }
      double x = 0.0;
      for (int b = NM - 1; b >= 0; --b) {
        const double h = Hd[(long long)b * klow];
        x = (b == NM - 1) ? h * p[b * MT] : (h - dus[b] * x) * p[b * MT];
        Hd[(long long)b * klow] = x;
        c[b * MT] = mk2<T>((T)0, (T)0);
      }
    } else {
      // forward: g_b = r_b - (l_b / d'_{b-1}) g_{b-1}
      double gx = 0.0, gy = 0.0, rprev = 0.0;
#pragma unroll 4
      for (int b = 0; b < NM; ++b) {
        const V2 cv = c[b * MT];
        double rx = (double)cv.x, ry = (double)cv.y;
        if (b > 0) {
          const double w = dls[b] * rprev;  // l_b / d'_{b-1}
          rx = rx - w * gx;
          ry = ry - w * gy;
        }
        rprev = p[b * MT];
        gx = rx;
        gy = ry;
        c[b * MT] = mk2<T>((T)rx, (T)ry);
      }
      // backward: x_b = (g_b - u_b x_{b+1}) / d'_b
      const int top = NM - 1;
      double xx = 0.0, xy = 0.0;
#pragma unroll 4
      for (int b = top; b >= 0; --b) {
        const V2 cv = c[b * MT];
        const double pv = p[b * MT];
        if (b == top) {
          xx = (double)cv.x * pv;
          xy = (double)cv.y * pv;
        } else {
          xx = ((double)cv.x - dus[b] * xx) * pv;
          xy = ((double)cv.y - dus[b] * xy) * pv;
        }
        c[b * MT] = mk2<T>((T)xx, (T)xy);
      }
    }
  }
  }
  fence_async_shared();  // the sweeps' shared-memory writes before the TMA store reads them
  __syncwarp();
  if (lane == 0) {
    store_3d(&mapC, Ct, 2 * kx0, kz, 0);
    store_commit_and_wait_read();
  }
}

bool tma::encode(CUtensorMap *map, CUtensorMapDataType type, int rank, void *base, const cuuint64_t *dims,
                 const cuuint64_t *strides, const cuuint32_t *box, CUtensorMapSwizzle swizzle) {
  static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
  if (!enc) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return false;
    enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  if (reinterpret_cast<uintptr_t>(base) & 15) return false;
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  return enc(map, type, (cuuint32_t)rank, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// C viewed as elements of T (dims 2 rx, MH, NM) with boxes of 2 MT x 1 x NM;
// pivots (rx, MH, NM) with boxes of MT x 1 x NM.  The boxes are at most 256
// rows deep, so NM <= 256.
template <typename T>
bool thomas_maps(const Spec &s, void *C, double *piv, ThomasMaps *out) {
  constexpr int MT = ThomasTile<T>::MT;
  if (s.NM > 256 || s.NM < 1) return false;
  CUtensorMap mc, mp;
  const CUtensorMapDataType ty = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  const cuuint64_t dc[3] = {(cuuint64_t)2 * s.rx, (cuuint64_t)s.MH, (cuuint64_t)s.NM};
  const cuuint64_t sc[2] = {(cuuint64_t)2 * s.rx * sizeof(T), (cuuint64_t)2 * s.rx * sizeof(T) * s.MH};
  const cuuint32_t bc[3] = {(cuuint32_t)(2 * MT), 1, (cuuint32_t)s.NM};
  if (!encode(&mc, ty, 3, C, dc, sc, bc)) return false;
  const cuuint64_t dp[3] = {(cuuint64_t)s.rx, (cuuint64_t)s.MH, (cuuint64_t)s.NM};
  const cuuint64_t sp[2] = {(cuuint64_t)s.rx * sizeof(double), (cuuint64_t)s.rx * sizeof(double) * s.MH};
  const cuuint32_t bp[3] = {(cuuint32_t)MT, 1, (cuuint32_t)s.NM};
  if (!encode(&mp, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, piv, dp, sp, bp)) return false;
  if (thomas_tile_smem<T>(s.NM) > 227 * 1024) return false;
  static_assert(sizeof(CUtensorMap) == sizeof(out->c), "tensor map size");
  memcpy(out->c, &mc, sizeof mc);
  memcpy(out->p, &mp, sizeof mp);
  return true;
}

template <typename T>
void launch_thomas_tile(const Spec &s, const ThomasMaps &maps, const double *dl, const double *du, double *H0,
                        int klow, int *err, int wait_limit, bool scan, cudaStream_t st) {
  constexpr int MT = ThomasTile<T>::MT;
  const size_t sm = thomas_tile_smem<T>(s.NM);
  CUtensorMap mc, mp;
  memcpy(&mc, maps.c, sizeof mc);
  memcpy(&mp, maps.p, sizeof mp);
  dim3 grid((s.N + MT - 1) / MT, s.MH);
  const int wl = wait_limit < 0 ? WAIT_LIMIT : wait_limit;
  if (scan) {
    cudaFuncSetAttribute(k_thomas_tile<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_thomas_tile<T, true><<<grid, 32, sm, st>>>(mc, mp, s, dl, du, H0, klow, err, wl);
  } else {
    cudaFuncSetAttribute(k_thomas_tile<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_thomas_tile<T, false><<<grid, 32, sm, st>>>(mc, mp, s, dl, du, H0, klow, err, wl);
  }
}

template bool thomas_maps<float>(const Spec &, void *, double *, ThomasMaps *);
template bool thomas_maps<double>(const Spec &, void *, double *, ThomasMaps *);
template void launch_thomas_tile<float>(const Spec &, const ThomasMaps &, const double *, const double *, double *,
                                        int, int *, int, bool, cudaStream_t);
template void launch_thomas_tile<double>(const Spec &, const ThomasMaps &, const double *, const double *, double *,
                                         int, int *, int, bool, cudaStream_t);

}  // namespace blgpu
