// zdft_tc.cu -- the mixed form's z transforms on the tensor cores.
//
// The real DFT over the half spectrum (kz = 0..M/2) of every z-line is a
// product with a fixed cos / sin table; pairing f_k +- f_{M-k} halves it to
// two square products of order Q = M/2 + 1:
//   forward   re[kz] = sum_k cos(2 pi kz k / M) S[k]   S[0] = f_0, S[k] = f_k + f_{M-k}
//             im[kz] = sum_k -sin(2 pi kz k / M) D[k]  D[k] = f_k - f_{M-k}
//             (+ (-1)^kz f_{M/2} in re for even M)
//   inverse   P[p] = sum_kz cos(2 pi p kz / M) Re[kz],  Q'[p] = sum_kz -sin(...) Im[kz]
//             f_p = (c0 + 2 (P + Q') + y) / M,  f_{M-p} = (c0 + 2 (P - Q') + y) / M
//             (kz = 1..H, H = (M-1)/2; c0 = Re[0]; y = (-1)^p Re[M/2] for even M)
// The products run as TF32 tensor-core MMAs (mma.sync m16n8k8) with the
// three-term split x = x_hi + x_lo of both operands (hi*hi + hi*lo + lo*hi),
// which keeps the FP32 accuracy of the direct sums (error ~ 2^-22 relative).
//
// A persistent CTA per SM keeps the table fragments of its warp in registers
// (loaded once) and walks the (b, kx-tile) work items.  The raw line data of
// a work item (M rows x NT = 64 kx of R, or MH rows x 64 complex kx of C)
// arrives by one TMA tensor copy into a double buffer, issued one item ahead
// and completed on an mbarrier, so the DRAM latency of item i+1 overlaps the
// products of item i.  The CTA then splits the operands into shared memory,
// each warp multiplies one 16-row tile of the cos or the sin table by all of
// them, and the results leave through shared memory as coalesced rows.
#include <cmath>
#include <cstring>
#include <vector>

#include "kernels.cuh"
#include "tma.cuh"

namespace blgpu {

using namespace tma;

static_assert(sizeof(CUtensorMap) == sizeof(ZdftMaps::r), "tensor map size");

namespace {
constexpr int ZNT = 64;              // kx columns per work item
constexpr int ZLD = ZNT + 8;         // row pitch of the staged operands (conflict-free fragment loads)

__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// x -> (hi, lo) as TF32 bit patterns, x ~ hi + lo to ~2^-22
__device__ __forceinline__ void split(float x, uint32_t &hi, uint32_t &lo) {
  hi = tf32_rna(x);
  lo = tf32_rna(x - __uint_as_float(hi));
}

}  // namespace

// Table fragments, in the order the kernel reads them: for table t (0 cos,
// 1 -sin), row tile mt, k step ks, lane l: 4 hi then 4 lo words of the
// m16n8k8 A fragment (rows g, g+8; columns tig, tig+4 of the 16x8 block).
// QP = Q rounded up to 16; entries beyond Q are zero.
// Shared memory (floats): raw[2][rawf] | B0h B0l B1h B1l [QP][ZLD] | aux[2][ZNT] | 2 mbarriers.
template <int QP>
__global__ void __launch_bounds__(QP / 8 * 32, 1)
    k_zdft_tc(const __grid_constant__ CUtensorMap mapR, const __grid_constant__ CUtensorMap mapC, Spec s,
              float *__restrict__ R, float2 *__restrict__ C, const uint4 *__restrict__ frag, int inverse, int rawf,
              int *__restrict__ err) {
  constexpr int MT = QP / 16;  // row tiles per table
  constexpr int KS = QP / 8;   // k steps
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float *raw0 = reinterpret_cast<float *>(smem_raw);
  float *B0h = raw0 + 2 * (size_t)rawf;  // [QP][ZLD]: S (fwd) or Re (inv), hi part
  float *B0l = B0h + QP * ZLD;
  float *B1h = B0l + QP * ZLD;           // D (fwd) or Im (inv)
  float *B1l = B1h + QP * ZLD;
  float *aux = B1l + QP * ZLD;           // [2][ZNT]: f_{M/2} row / c0 and Nyquist rows
  uint64_t *bar = reinterpret_cast<uint64_t *>(aux + 2 * ZNT);
  float *stage = B0h;                    // epilogue staging, aliases the operands
  const int M = s.M, MH = s.MH, H = (M - 1) / 2;
  const bool even = (M & 1) == 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
  const int tbl = warp / MT, mt = warp % MT;  // table (0 cos, 1 -sin) and its row tile
  const int ntile = (s.N + ZNT - 1) / ZNT;
  const int nitems = s.NM * ntile;
  const int nthr = blockDim.x;
  // one box per work item: M rows x 64 floats of R, or MH rows x 128 floats (64 complex) of C
  const uint32_t box_bytes = inverse ? (uint32_t)MH * 2 * ZNT * 4 : (uint32_t)M * ZNT * 4;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
    if ((int)blockIdx.x < nitems) {
      const int b = blockIdx.x / ntile, kx0 = (blockIdx.x % ntile) * ZNT;
      mbar_expect_tx(&bar[0], box_bytes);
      if (inverse) load_2d(raw0, &mapC, 2 * kx0, b * MH, &bar[0]);
      else load_2d(raw0, &mapR, kx0, b * M, &bar[0]);
    }
  }
  // the warp's table fragments, resident for the whole kernel
  uint32_t ahi[KS][4], alo[KS][4];
#pragma unroll
  for (int ks = 0; ks < KS; ++ks) {
    const uint4 *f = frag + ((((size_t)tbl * MT + mt) * KS + ks) * 32 + lane) * 2;
    const uint4 h = f[0], l = f[1];
    ahi[ks][0] = h.x; ahi[ks][1] = h.y; ahi[ks][2] = h.z; ahi[ks][3] = h.w;
    alo[ks][0] = l.x; alo[ks][1] = l.y; alo[ks][2] = l.z; alo[ks][3] = l.w;
  }
  const float *Bh = tbl ? B1h : B0h, *Bl = tbl ? B1l : B0l;
  int i = 0;
  for (int item = blockIdx.x; item < nitems; item += gridDim.x, ++i) {
    const int b = item / ntile, kx0 = (item % ntile) * ZNT;
    const int buf = i & 1;
    const float *rw = raw0 + (size_t)buf * rawf;
    // the previous item's staging and results are no longer read, and the
    // other raw buffer was consumed before the previous item's products
    __syncthreads();
    const int next = item + gridDim.x;
    if (threadIdx.x == 0 && next < nitems) {
      const int nb = next / ntile, nk0 = (next % ntile) * ZNT;
      float *dst = raw0 + (size_t)(buf ^ 1) * rawf;
      fence_async_shared();  // generic reads before the async write
      mbar_expect_tx(&bar[buf ^ 1], box_bytes);
      if (inverse) load_2d(dst, &mapC, 2 * nk0, nb * MH, &bar[buf ^ 1]);
      else load_2d(dst, &mapR, nk0, nb * M, &bar[buf ^ 1]);
    }
    const bool ok = mbar_wait(&bar[buf], (uint32_t)(i >> 1) & 1u);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicOr(err, 2);
        // let the copies this CTA issued finish (bounded) before leaving
        mbar_wait(&bar[buf], (uint32_t)(i >> 1) & 1u);
        if (next < nitems) mbar_wait(&bar[buf ^ 1], (uint32_t)((i + 1) >> 1) & 1u);
      }
      return;
    }
    // ---- split the operands ----
    if (!inverse) {
      for (int q = threadIdx.x; q < QP * ZNT; q += nthr) {
        const int k = q / ZNT, c = q % ZNT;
        float sv = 0.f, dv = 0.f;
        if (kx0 + c < s.N && k <= H) {
          const float fk = rw[k * ZNT + c];
          if (k == 0) {
            sv = fk;
          } else {
            const float fm = rw[(M - k) * ZNT + c];
            sv = fk + fm;
            dv = fk - fm;
          }
        }
        uint32_t h, l;
        split(sv, h, l);
        B0h[k * ZLD + c] = __uint_as_float(h);
        B0l[k * ZLD + c] = __uint_as_float(l);
        split(dv, h, l);
        B1h[k * ZLD + c] = __uint_as_float(h);
        B1l[k * ZLD + c] = __uint_as_float(l);
      }
      if (even)
        for (int c = threadIdx.x; c < ZNT; c += nthr) aux[c] = kx0 + c < s.N ? rw[(M / 2) * ZNT + c] : 0.f;
    } else {
      const float2 *cw = reinterpret_cast<const float2 *>(rw);  // [MH][ZNT]
      for (int q = threadIdx.x; q < QP * ZNT; q += nthr) {
        const int kz = q / ZNT, c = q % ZNT;
        float2 v = make_float2(0.f, 0.f);
        if (kx0 + c < s.N && kz >= 1 && kz <= H) v = cw[kz * ZNT + c];
        uint32_t h, l;
        split(v.x, h, l);
        B0h[kz * ZLD + c] = __uint_as_float(h);
        B0l[kz * ZLD + c] = __uint_as_float(l);
        split(v.y, h, l);
        B1h[kz * ZLD + c] = __uint_as_float(h);
        B1l[kz * ZLD + c] = __uint_as_float(l);
      }
      for (int c = threadIdx.x; c < ZNT; c += nthr) {
        const bool okc = kx0 + c < s.N;
        aux[c] = okc ? cw[c].x : 0.f;                                  // c0
        aux[ZNT + c] = (okc && even) ? cw[(M / 2) * ZNT + c].x : 0.f;  // Nyquist
      }
    }
    __syncthreads();
    // ---- products: this warp's 16 rows x 64 columns ----
    float acc[ZNT / 8][4];
#pragma unroll
    for (int nt = 0; nt < ZNT / 8; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
    for (int ks = 0; ks < KS; ++ks) {
      const int k0 = ks * 8;
#pragma unroll
      for (int nt = 0; nt < ZNT / 8; ++nt) {
        const int n = nt * 8 + g;
        const uint32_t bh0 = __float_as_uint(Bh[(k0 + tig) * ZLD + n]);
        const uint32_t bh1 = __float_as_uint(Bh[(k0 + tig + 4) * ZLD + n]);
        const uint32_t bl0 = __float_as_uint(Bl[(k0 + tig) * ZLD + n]);
        const uint32_t bl1 = __float_as_uint(Bl[(k0 + tig + 4) * ZLD + n]);
        mma_tf32(acc[nt], alo[ks], bh0, bh1);
        mma_tf32(acc[nt], ahi[ks], bl0, bl1);
        mma_tf32(acc[nt], ahi[ks], bh0, bh1);
      }
    }
    __syncthreads();  // operands consumed: reuse the shared memory for the results
    // stage[t][row][c], t = table; rows of this warp's tile
#pragma unroll
    for (int nt = 0; nt < ZNT / 8; ++nt) {
      const int r0 = mt * 16 + g, c0 = nt * 8 + 2 * tig;
      float *st = stage + (size_t)tbl * QP * ZLD;
      st[r0 * ZLD + c0] = acc[nt][0];
      st[r0 * ZLD + c0 + 1] = acc[nt][1];
      st[(r0 + 8) * ZLD + c0] = acc[nt][2];
      st[(r0 + 8) * ZLD + c0 + 1] = acc[nt][3];
    }
    __syncthreads();
    const float *S0 = stage, *S1 = stage + (size_t)QP * ZLD;
    if (!inverse) {
      float2 *Cb = C + (size_t)b * MH * s.rx + kx0;
      for (int q = threadIdx.x; q < MH * ZNT; q += nthr) {
        const int kz = q / ZNT, c = q % ZNT;
        if (kx0 + c >= s.N) continue;
        float re = S0[kz * ZLD + c];
        if (even) re += (kz & 1) ? -aux[c] : aux[c];
        Cb[(size_t)kz * s.rx + c] = make_float2(re, S1[kz * ZLD + c]);
      }
    } else {
      float *Rb = R + (size_t)b * M * s.rx + kx0;
      const float invM = 1.0f / (float)M;
      const int npairs = M / 2 + 1;
      for (int q = threadIdx.x; q < npairs * ZNT; q += nthr) {
        const int p = q / ZNT, c = q % ZNT;
        if (kx0 + c >= s.N) continue;
        const float P = S0[p * ZLD + c], Qn = S1[p * ZLD + c];  // Qn = -Q
        const float c0 = aux[c];
        const float y = even ? ((p & 1) ? -aux[ZNT + c] : aux[ZNT + c]) : 0.f;
        Rb[(size_t)p * s.rx + c] = (c0 + 2.0f * (P + Qn) + y) * invM;
        const int pm = M - p;
        if (pm != p && pm < M) Rb[(size_t)pm * s.rx + c] = (c0 + 2.0f * (P - Qn) + y) * invM;
      }
    }
  }
}

// floats of one raw buffer: the larger of the two boxes, in 128-byte units
static int raw_floats(const Spec &s) {
  const int f = s.M * ZNT > s.MH * 2 * ZNT ? s.M * ZNT : s.MH * 2 * ZNT;
  return (f + 31) / 32 * 32;
}

static size_t smem_bytes(const Spec &s, int qp) {
  return ((size_t)2 * raw_floats(s) + (size_t)4 * qp * ZLD + 2 * ZNT) * sizeof(float) + 2 * sizeof(uint64_t);
}

// Q rounded up to 16 when the tensor-core path serves it, else 0 (the TMA
// boxes are at most 256 rows and the buffers fit one CTA's shared memory)
int zdft_tc_qp(const Spec &s) {
  const int qp = (s.MH + 15) / 16 * 16;
  if (!(qp == 32 || qp == 48 || qp == 64 || qp == 80 || qp == 96)) return 0;
  if (s.M > 256 || smem_bytes(s, qp) > 227 * 1024) return 0;
  return qp;
}

// Tensor maps of R (rx x NM*M floats, box 64 x M) and of C viewed as floats
// (2 rx x NM*MH, box 128 x MH); false when the driver entry point or the
// encoding is unavailable (the caller then keeps the direct sums).
bool zdft_tc_maps(const Spec &s, float *R, float2 *C, ZdftMaps *out) {
  CUtensorMap mr, mc;
  const cuuint64_t dr[2] = {(cuuint64_t)s.rx, (cuuint64_t)s.NM * s.M};
  const cuuint64_t sr[1] = {(cuuint64_t)s.rx * sizeof(float)};
  const cuuint32_t br[2] = {(cuuint32_t)ZNT, (cuuint32_t)s.M};
  if (!encode(&mr, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, R, dr, sr, br)) return false;
  const cuuint64_t dc[2] = {(cuuint64_t)2 * s.rx, (cuuint64_t)s.NM * s.MH};
  const cuuint64_t sc[1] = {(cuuint64_t)2 * s.rx * sizeof(float)};
  const cuuint32_t bc[2] = {(cuuint32_t)(2 * ZNT), (cuuint32_t)s.MH};
  if (!encode(&mc, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, C, dc, sc, bc)) return false;
  memcpy(out->r, &mr, sizeof mr);
  memcpy(out->c, &mc, sizeof mc);
  return true;
}

size_t zdft_tc_frag_words(const Spec &s) {
  const int qp = zdft_tc_qp(s);
  return (size_t)2 * (qp / 16) * (qp / 8) * 32 * 8;
}

// host: the fragment table of cos(2 pi m n / M) and -sin(2 pi m n / M)
static uint32_t tf32_host(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return u;
  u += 0x1000u;  // round half away from zero on the magnitude, as cvt.rna
  return u & 0xffffe000u;
}

void zdft_tc_fragments(const Spec &s, std::vector<uint32_t> &out) {
  const int qp = zdft_tc_qp(s), M = s.M, Q = s.MH;
  const int MT = qp / 16, KS = qp / 8;
  out.assign(zdft_tc_frag_words(s), 0u);
  for (int t = 0; t < 2; ++t)
    for (int mt = 0; mt < MT; ++mt)
      for (int ks = 0; ks < KS; ++ks)
        for (int l = 0; l < 32; ++l) {
          const int g = l >> 2, tig = l & 3;
          const int rows[4] = {mt * 16 + g, mt * 16 + g + 8, mt * 16 + g, mt * 16 + g + 8};
          const int cols[4] = {ks * 8 + tig, ks * 8 + tig, ks * 8 + tig + 4, ks * 8 + tig + 4};
          uint32_t *o = out.data() + ((((size_t)t * MT + mt) * KS + ks) * 32 + l) * 8;
          for (int e = 0; e < 4; ++e) {
            float v = 0.f;
            const int m = rows[e], n = cols[e];
            if (m < Q && n < Q) {
              const double a = 2.0 * M_PI * (double)(((long long)m * n) % M) / (double)M;
              v = (float)(t ? -sin(a) : cos(a));
            }
            const uint32_t hi = tf32_host(v);
            float hf;
            memcpy(&hf, &hi, 4);
            o[e] = hi;
            o[4 + e] = tf32_host(v - hf);
          }
        }
}

template <int QP>
static void launch_qp(const Spec &s, const ZdftMaps &mp, float *R, float2 *C, const uint4 *frag, int inverse,
                      int nsm, int *err, cudaStream_t st) {
  const size_t sm = smem_bytes(s, QP);
  cudaFuncSetAttribute(k_zdft_tc<QP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  const int nitems = s.NM * ((s.N + ZNT - 1) / ZNT);
  const int grid = nitems < nsm ? nitems : nsm;
  CUtensorMap mr, mc;
  memcpy(&mr, mp.r, sizeof mr);
  memcpy(&mc, mp.c, sizeof mc);
  k_zdft_tc<QP><<<grid, QP / 8 * 32, sm, st>>>(mr, mc, s, R, C, frag, inverse, raw_floats(s), err);
}

void launch_zdft_tc(const Spec &s, const ZdftMaps &maps, float *R, float2 *C, const uint32_t *frag, int inverse,
                    int nsm, int *err, cudaStream_t st) {
  const uint4 *f = reinterpret_cast<const uint4 *>(frag);
  switch (zdft_tc_qp(s)) {
    case 32: launch_qp<32>(s, maps, R, C, f, inverse, nsm, err, st); break;
    case 48: launch_qp<48>(s, maps, R, C, f, inverse, nsm, err, st); break;
    case 64: launch_qp<64>(s, maps, R, C, f, inverse, nsm, err, st); break;
    case 80: launch_qp<80>(s, maps, R, C, f, inverse, nsm, err, st); break;
    case 96: launch_qp<96>(s, maps, R, C, f, inverse, nsm, err, st); break;
    default: break;
  }
}

}  // namespace blgpu
