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
#include "ysolve.cuh"

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
        if (b > 0) r = ys_fwd(r, ys_w(dls[b], rprev), g);
        rprev = p[b * MT];
        g = r;
        Hd[(long long)b * klow] = r;
      }
      double x = 0.0;
      for (int b = NM - 1; b >= 0; --b) {
        const double h = Hd[(long long)b * klow];
        x = (b == NM - 1) ? ys_top(h, p[b * MT]) : ys_bwd(h, dus[b], x, p[b * MT]);
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
          const double w = ys_w(dls[b], rprev);  // l_b / d'_{b-1}
          rx = ys_fwd(rx, w, gx);
          ry = ys_fwd(ry, w, gy);
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
          xx = ys_top((double)cv.x, pv);
          xy = ys_top((double)cv.y, pv);
        } else {
          xx = ys_bwd((double)cv.x, dus[b], xx, pv);
          xy = ys_bwd((double)cv.y, dus[b], xy, pv);
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

// ---------------------------------------------------------------------------
// The y-solve with the pivots recomputed in the kernel.  A CTA (one warp)
// owns the tile of RT consecutive kx of one kz (32 in FP32, 16 in FP64: 256 B
// rows of C) over all NM rows: one TMA copy brings it into shared memory,
// lane l solves mode kx0+l there and one TMA store writes the tile back, so
// C is read once and written once and no pivot table is read.  The forward
// sweep forms the pivots from dd, dl, du, kxx and kzz with the table's
// roundings (ysolve.cuh) and keeps every 16th (the pivot before each
// segment of 16 rows); the backward sweep walks the segments from the top,
// forms the segment's 16 pivots again from its checkpoint into registers
// and back-substitutes over them.  Results are bit-identical to the
// pivot-table kernels.  About 70 KB of shared memory, three CTAs per SM.
// ---------------------------------------------------------------------------
constexpr int RC_SEG = 16;
template <typename T> struct RcTile { static constexpr int RT = sizeof(T) == 4 ? 32 : 16; };
template <typename T> __host__ __device__ inline size_t rc_c_bytes(int NM) {
  return ((size_t)NM * RcTile<T>::RT * 2 * sizeof(T) + 127) / 128 * 128;
}
template <typename T> inline size_t thomas_rc_smem(int NM) {
  return rc_c_bytes<T>(NM) + (size_t)((NM + RC_SEG - 1) / RC_SEG) * RcTile<T>::RT * sizeof(double) + 16;
}

template <typename T>
__global__ void __launch_bounds__(32) k_thomas_rc(const __grid_constant__ CUtensorMap mapC, Spec s,
                                                  const double *__restrict__ dd, const double *__restrict__ dl,
                                                  const double *__restrict__ du, const double *__restrict__ kxx,
                                                  const double *__restrict__ kzz, double *__restrict__ H0, int klow,
                                                  int *__restrict__ err, int wait_limit) {
  constexpr int RT = RcTile<T>::RT;
  typedef T2t<T> V2;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int NM = s.NM, nseg = (NM + RC_SEG - 1) / RC_SEG;
  V2 *Ct = reinterpret_cast<V2 *>(smem_raw);                                  // [NM][RT]
  double *chk = reinterpret_cast<double *>(smem_raw + rc_c_bytes<T>(NM));     // [nseg][RT]
  uint64_t *bar = reinterpret_cast<uint64_t *>(chk + (size_t)nseg * RT);
  const int kx0 = blockIdx.x * RT, kz = blockIdx.y, lane = threadIdx.x;
  if (lane == 0) {
    mbar_init(bar, 1);
    mbar_init_fence();
    mbar_expect_tx(bar, (uint32_t)((size_t)NM * RT * sizeof(V2)));
    load_3d(Ct, &mapC, 2 * kx0, kz, 0, bar);
  }
  __syncwarp();
  // as k_thomas_tile: a wait that gives up drains the copy with the normal limit
  const bool ok = mbar_wait(bar, 0, wait_limit);
  if (!__all_sync(0xffffffffu, ok)) {
    if (lane == 0) {
      atomicOr(err, 4);
      mbar_wait(bar, 0);
    }
    return;
  }
  const int kx = kx0 + lane;
  if (lane < RT && kx < s.N) {
    const double kk = kxx[kx], kzv = kzz[kz];
    const bool m00 = kx == 0 && kz == 0;
    V2 *c = Ct + lane;
    double *ck = chk + lane;
    // mixed form: the box-scale modes (kz = 0, kx < klow) keep their forward
    // results in FP64 in H0[b][kx] and leave zeros in C
    const bool h0 = H0 && kz == 0 && kx < klow;
    double *Hd = h0 ? H0 + kx : nullptr;
    // forward: pivots, g_b over r_b, checkpoint piv_b at the end of each segment
    double rinv = 0.0, gx = 0.0, gy = 0.0;
#pragma unroll 4
    for (int b = 0; b < NM; ++b) {
      const V2 cv = c[b * RT];
      const double d = ys_diag(dd[b], kk, kzv, m00 && b == 0);
      double rx = (double)cv.x, ry = (double)cv.y;
      if (b > 0) {
        const double w = ys_w(dl[b], rinv);
        rx = ys_fwd(rx, w, gx);
        ry = ys_fwd(ry, w, gy);
        rinv = ys_piv(d, w, du[b - 1], false);
      } else {
        rinv = ys_piv(d, 0.0, 0.0, true);
      }
      if ((b & (RC_SEG - 1)) == RC_SEG - 1) ck[(b / RC_SEG) * RT] = rinv;
      gx = rx;
      gy = ry;
      if (h0) Hd[(long long)b * klow] = rx;
      else c[b * RT] = mk2<T>((T)rx, (T)ry);
    }
    // backward, one segment of rows at a time from the top
    double xx = 0.0, xy = 0.0;
    for (int sg = nseg - 1; sg >= 0; --sg) {
      const int b0 = sg * RC_SEG;
      double pv[RC_SEG];
      double r = sg > 0 ? ck[(sg - 1) * RT] : 0.0;  // piv_{b0-1}
#pragma unroll
      for (int u = 0; u < RC_SEG; ++u) {
        const int b = b0 + u;
        if (b < NM) {
          const double d = ys_diag(dd[b], kk, kzv, m00 && b == 0);
          r = b > 0 ? ys_piv(d, ys_w(dl[b], r), du[b - 1], false) : ys_piv(d, 0.0, 0.0, true);
          pv[u] = r;
        }
      }
#pragma unroll
      for (int u = RC_SEG - 1; u >= 0; --u) {
        const int b = b0 + u;
        if (b < NM) {
          double gxb, gyb;
          if (h0) {
            gxb = Hd[(long long)b * klow];
            gyb = 0.0;
          } else {
            const V2 cv = c[b * RT];
            gxb = (double)cv.x;
            gyb = (double)cv.y;
          }
          if (b == NM - 1) {
            xx = ys_top(gxb, pv[u]);
            xy = ys_top(gyb, pv[u]);
          } else {
            xx = ys_bwd(gxb, du[b], xx, pv[u]);
            xy = ys_bwd(gyb, du[b], xy, pv[u]);
          }
          if (h0) {
            Hd[(long long)b * klow] = xx;
            c[b * RT] = mk2<T>((T)0, (T)0);
          } else {
            c[b * RT] = mk2<T>((T)xx, (T)xy);
          }
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
  // C with boxes of 2 RT x 1 x NM for the recomputing kernel (RT divides the
  // row pitch rx, a multiple of 32, so every box lies inside the array)
  CUtensorMap mr;
  const cuuint32_t br[3] = {(cuuint32_t)(2 * RcTile<T>::RT), 1, (cuuint32_t)s.NM};
  out->have_rc = encode(&mr, ty, 3, C, dc, sc, br) && thomas_rc_smem<T>(s.NM) <= 227 * 1024;
  if (out->have_rc) memcpy(out->rc, &mr, sizeof mr);
  return true;
}

template <typename T>
void launch_thomas_rc(const Spec &s, const ThomasMaps &maps, const double *dd, const double *dl, const double *du,
                      const double *kxx, const double *kzz, double *H0, int klow, int *err, int wait_limit,
                      cudaStream_t st) {
  constexpr int RT = RcTile<T>::RT;
  const size_t sm = thomas_rc_smem<T>(s.NM);
  cudaFuncSetAttribute(k_thomas_rc<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  CUtensorMap mr;
  memcpy(&mr, maps.rc, sizeof mr);
  dim3 grid((s.N + RT - 1) / RT, s.MH);
  k_thomas_rc<T><<<grid, 32, sm, st>>>(mr, s, dd, dl, du, kxx, kzz, H0, klow, err,
                                       wait_limit < 0 ? WAIT_LIMIT : wait_limit);
}

template <typename T>
void launch_thomas_tile(const Spec &s, const ThomasMaps &maps, const double *dl, const double *du, double *H0,
                        int klow, int *err, int wait_limit, cudaStream_t st) {
  constexpr int MT = ThomasTile<T>::MT;
  const size_t sm = thomas_tile_smem<T>(s.NM);
  cudaFuncSetAttribute(k_thomas_tile<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  CUtensorMap mc, mp;
  memcpy(&mc, maps.c, sizeof mc);
  memcpy(&mp, maps.p, sizeof mp);
  dim3 grid((s.N + MT - 1) / MT, s.MH);
  k_thomas_tile<T><<<grid, 32, sm, st>>>(mc, mp, s, dl, du, H0, klow, err, wait_limit < 0 ? WAIT_LIMIT : wait_limit);
}

template bool thomas_maps<float>(const Spec &, void *, double *, ThomasMaps *);
template bool thomas_maps<double>(const Spec &, void *, double *, ThomasMaps *);
template void launch_thomas_rc<float>(const Spec &, const ThomasMaps &, const double *, const double *,
                                      const double *, const double *, const double *, double *, int, int *, int,
                                      cudaStream_t);
template void launch_thomas_rc<double>(const Spec &, const ThomasMaps &, const double *, const double *,
                                       const double *, const double *, const double *, double *, int, int *, int,
                                       cudaStream_t);
template void launch_thomas_tile<float>(const Spec &, const ThomasMaps &, const double *, const double *, double *,
                                        int, int *, int, cudaStream_t);
template void launch_thomas_tile<double>(const Spec &, const ThomasMaps &, const double *, const double *, double *,
                                         int, int *, int, cudaStream_t);

}  // namespace blgpu
