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
// the same plus the segments' maps (three doubles per thread)
template <typename T, int NT>
inline size_t tile_scan_smem(int NM) {
  return thomas_tile_smem<T>(NM) + 3 * (size_t)NT * sizeof(double);
}

template <typename T>
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
  fence_async_shared();  // the sweeps' shared-memory writes before the TMA store reads them
  __syncwarp();
  if (lane == 0) {
    store_3d(&mapC, Ct, 2 * kx0, kz, 0);
    store_commit_and_wait_read();
  }
}

// The same tile solve with each mode's NM rows split into P = NT / MT
// segments: thread t takes mode m = t % MT and the rows [kk Le, kk Le + Le)
// of it, kk = t / MT (a half- or quarter-warp reads one row's MT modes, one
// 128-byte run, without bank conflicts).  Both recurrences are first-order
// and linear,
//   g_b = r_b - w_b g_{b-1} (w_b = dl_b piv_{b-1}),  x_b = (g_b - du_b x_{b+1}) piv_b,
// so a segment runs them over its rows from a zero start, keeping the
// product of its multipliers (-w_b forward, beta_b = -du_b piv_b backward):
// its rows are then affine in the value entering it.  The segments' maps
// meet in shared memory, each thread composes those of the segments before
// (forward) or after (backward) its own into its entering value, and a
// second pass over its rows adds the product times that value.  The sums
// are those of the serial sweeps, reassociated across the segments; the
// serial chains are P times shorter and every thread of the CTA works.
// REG: the segment's rows stay in FP64 registers from one read of the tile
// to the final write; otherwise each pass reads and writes the tile.
template <typename T, int NT, bool REG>
__global__ void __launch_bounds__(NT, 512 / NT) k_thomas_tile_scan(const __grid_constant__ CUtensorMap mapC,
                                                         const __grid_constant__ CUtensorMap mapP, Spec s,
                                                         const double *__restrict__ dl, const double *__restrict__ du,
                                                         double *__restrict__ H0, int klow, int *__restrict__ err,
                                                         int wait_limit) {
  constexpr int MT = ThomasTile<T>::MT, P = NT / MT;
  typedef T2t<T> V2;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int NM = s.NM;
  V2 *Ct = reinterpret_cast<V2 *>(smem_raw);                                   // [NM][MT]
  double *Pt = reinterpret_cast<double *>(smem_raw + tile_c_bytes<T>(NM));     // [NM][MT]
  double *dls = reinterpret_cast<double *>(smem_raw + tile_c_bytes<T>(NM) + tile_p_bytes<T>(NM));  // [NM]
  double *dus = dls + NM;                                                                          // [NM]
  uint64_t *bar = reinterpret_cast<uint64_t *>(dus + NM);
  double *mA = reinterpret_cast<double *>(bar + 1), *mX = mA + NT, *mY = mX + NT;  // segment maps [kk][m]
  const int kx0 = blockIdx.x * MT, kz = blockIdx.y, tid = threadIdx.x;
  const uint32_t bytes = (uint32_t)((size_t)NM * MT * (2 * sizeof(T) + sizeof(double)));
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_init_fence();
    mbar_expect_tx(bar, bytes);
    load_3d(Ct, &mapC, 2 * kx0, kz, 0, bar);
    load_3d(Pt, &mapP, kx0, kz, 0, bar);
  }
  for (int b = tid; b < NM; b += NT) {
    dls[b] = dl[b];
    dus[b] = du[b];
  }
  __syncthreads();
  // wait_limit polls; after giving up, thread 0 drains with the normal limit,
  // so no copy into this CTA's shared memory is in flight when it leaves
  const bool ok = mbar_wait(bar, 0, wait_limit);
  if (!__syncthreads_and(ok)) {
    if (tid == 0) {
      atomicOr(err, 4);
      mbar_wait(bar, 0);
    }
    return;
  }
  const int m = tid % MT, kk = tid / MT;
  if (H0 && kz == 0 && kx0 < klow) {
    // the mixed form's box-scale modes (and any other mode of their tile):
    // serial sweeps, one thread per mode
    const int kx = kx0 + tid;
    if (tid < MT && kx < s.N) {
      V2 *c = Ct + tid;
      const double *p = Pt + tid;
      if (kx < klow) {
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
        double gx = 0.0, gy = 0.0, rprev = 0.0;
        for (int b = 0; b < NM; ++b) {
          const V2 cv = c[b * MT];
          double rx = (double)cv.x, ry = (double)cv.y;
          if (b > 0) {
            const double w = dls[b] * rprev;
            rx = rx - w * gx;
            ry = ry - w * gy;
          }
          rprev = p[b * MT];
          gx = rx;
          gy = ry;
          c[b * MT] = mk2<T>((T)rx, (T)ry);
        }
        double xx = 0.0, xy = 0.0;
        for (int b = NM - 1; b >= 0; --b) {
          const V2 cv = c[b * MT];
          const double pv = p[b * MT];
          if (b == NM - 1) {
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
  } else if (REG) {
    // the segment's rows in FP64 registers from one read of the tile to the
    // final write (LMAX = 16 rows: NM <= 256 over 16 segments)
    constexpr int LMAX = 16;
    const bool act = kx0 + m < s.N;
    const int Le = (NM + P - 1) / P, s0 = kk * Le;
    const int nr = act ? max(0, min(Le, NM - s0)) : 0;
    V2 *c = Ct + (size_t)s0 * MT + m;
    const double *p = Pt + (size_t)s0 * MT + m;
    double vx[LMAX], vy[LMAX], pv[LMAX + 1];  // pv[u] = piv[s0 + u - 1]
    pv[0] = (nr > 0 && s0 > 0) ? p[-MT] : 0.0;
#pragma unroll
    for (int u = 0; u < LMAX; ++u) {
      if (u < nr) {
        const V2 cv = c[u * MT];
        vx[u] = (double)cv.x;
        vy[u] = (double)cv.y;
        pv[u + 1] = p[u * MT];
      } else {
        vx[u] = vy[u] = pv[u + 1] = 0.0;
      }
    }
    double gx = 0.0, gy = 0.0, h = 1.0;
#pragma unroll
    for (int u = 0; u < LMAX; ++u) {
      if (u < nr) {
        const int b = s0 + u;
        double w = 0.0;
        if (b > 0) {
          w = dls[b] * pv[u];
          vx[u] = vx[u] - w * gx;
          vy[u] = vy[u] - w * gy;
        }
        h = -w * h;
        gx = vx[u];
        gy = vy[u];
      }
    }
    mA[tid] = h;
    mX[tid] = gx;
    mY[tid] = gy;
    __syncthreads();
    double ix = 0.0, iy = 0.0;
    for (int q = 0; q < kk; ++q) {
      const int o = q * MT + m;
      ix = mX[o] + mA[o] * ix;
      iy = mY[o] + mA[o] * iy;
    }
    h = 1.0;
#pragma unroll
    for (int u = 0; u < LMAX; ++u) {
      if (u < nr) {
        const int b = s0 + u;
        const double w = b > 0 ? dls[b] * pv[u] : 0.0;
        h = -w * h;
        vx[u] = vx[u] + h * ix;
        vy[u] = vy[u] + h * iy;
      }
    }
    double xx = 0.0, xy = 0.0, kp = 1.0;
#pragma unroll
    for (int u = LMAX - 1; u >= 0; --u) {
      if (u < nr) {
        const int b = s0 + u;
        const double q = pv[u + 1];
        double beta = 0.0;
        if (b == NM - 1) {
          xx = vx[u] * q;
          xy = vy[u] * q;
        } else {
          xx = (vx[u] - dus[b] * xx) * q;
          xy = (vy[u] - dus[b] * xy) * q;
          beta = -dus[b] * q;
        }
        kp = beta * kp;
        vx[u] = xx;
        vy[u] = xy;
      }
    }
    __syncthreads();  // every thread has read the forward maps
    mA[tid] = kp;
    mX[tid] = xx;
    mY[tid] = xy;
    __syncthreads();
    ix = iy = 0.0;
    for (int q = P - 1; q > kk; --q) {
      const int o = q * MT + m;
      ix = mX[o] + mA[o] * ix;
      iy = mY[o] + mA[o] * iy;
    }
    kp = 1.0;
#pragma unroll
    for (int u = LMAX - 1; u >= 0; --u) {
      if (u < nr) {
        const int b = s0 + u;
        const double beta = b == NM - 1 ? 0.0 : -dus[b] * pv[u + 1];
        kp = beta * kp;
        c[u * MT] = mk2<T>((T)(vx[u] + kp * ix), (T)(vy[u] + kp * iy));
      }
    }
  } else {
    const bool act = kx0 + m < s.N;
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
    mA[tid] = h;
    mX[tid] = gx;
    mY[tid] = gy;
    __syncthreads();
    // the value entering the segment: the maps of segments 0 .. kk-1 applied to 0
    double ix = 0.0, iy = 0.0;
    for (int q = 0; q < kk; ++q) {
      const int o = q * MT + m;
      ix = mX[o] + mA[o] * ix;
      iy = mY[o] + mA[o] * iy;
    }
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
    __syncthreads();  // every thread has read the forward maps
    mA[tid] = kp;
    mX[tid] = xx;
    mY[tid] = xy;
    __syncthreads();
    // the value above the segment: the maps of segments P-1 .. kk+1 applied to 0
    ix = iy = 0.0;
    for (int q = P - 1; q > kk; --q) {
      const int o = q * MT + m;
      ix = mX[o] + mA[o] * ix;
      iy = mY[o] + mA[o] * iy;
    }
    kp = 1.0;
    for (int u = nr - 1; u >= 0; --u) {
      const int b = s0 + u;
      const double beta = b == NM - 1 ? 0.0 : -dus[b] * p[u * MT];
      kp = beta * kp;
      const V2 cv = c[u * MT];
      c[u * MT] = mk2<T>((T)((double)cv.x + kp * ix), (T)((double)cv.y + kp * iy));
    }
  }
  fence_async_shared();  // the solves' shared-memory writes before the TMA store reads them
  __syncthreads();
  if (tid == 0) {
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
    // 16 segments of each mode's rows: 256 threads in FP32, 128 in FP64
    // (at 814 x 257 x 193: FP32 y-solve 0.78 / 0.55 / 0.46 / 0.58 ms per step
    // with 4 / 8 / 16 / 32 segments, FP64 0.63 / 0.59 / 0.68 with 8 / 16 / 32)
    constexpr int NT = 16 * MT;
    const size_t smw = tile_scan_smem<T, NT>(s.NM);
    // FP64: each segment's rows in registers (0.59 -> 0.50 ms per step at
    // 814 x 257 x 193); FP32: in the tile (0.44 against 0.52 ms per step
    // in registers, at two CTAs per SM)
    if (sizeof(T) == 8) {
      cudaFuncSetAttribute(k_thomas_tile_scan<T, NT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smw);
      k_thomas_tile_scan<T, NT, true><<<grid, NT, smw, st>>>(mc, mp, s, dl, du, H0, klow, err, wl);
    } else {
      cudaFuncSetAttribute(k_thomas_tile_scan<T, NT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smw);
      k_thomas_tile_scan<T, NT, false><<<grid, NT, smw, st>>>(mc, mp, s, dl, du, H0, klow, err, wl);
    }
  } else {
    cudaFuncSetAttribute(k_thomas_tile<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_thomas_tile<T><<<grid, 32, sm, st>>>(mc, mp, s, dl, du, H0, klow, err, wl);
  }
}

template bool thomas_maps<float>(const Spec &, void *, double *, ThomasMaps *);
template bool thomas_maps<double>(const Spec &, void *, double *, ThomasMaps *);
template void launch_thomas_tile<float>(const Spec &, const ThomasMaps &, const double *, const double *, double *,
                                        int, int *, int, bool, cudaStream_t);
template void launch_thomas_tile<double>(const Spec &, const ThomasMaps &, const double *, const double *, double *,
                                         int, int *, int, bool, cudaStream_t);

}  // namespace blgpu
