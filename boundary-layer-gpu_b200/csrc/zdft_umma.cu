// zdft_umma.cu -- the mixed form's z transforms on the 5th-generation tensor
// cores: tcgen05.mma kind::tf32 with the cos / -sin tables resident in tensor
// memory (A operand), the split line data staged in shared memory (B
// operand, K-major core matrices) and the FP32 accumulators in tensor
// memory.  Same products as zdft_tc.cu (real DFT over the half spectrum as
// two square products of order Q = M/2+1 with the f_k +- f_{M-k} pairing,
// three-term TF32 split hi*hi + hi*lo + lo*hi); see there for the algebra.
//
// One persistent CTA (16 warps) per SM, warp-specialised.  Work items are
// (row b, 32 kx columns).  A producer thread brings the raw columns of the
// coming items by TMA tensor copies (NRAW buffers); eight warps split them
// into the B operands (NB buffers, hi and lo columns side by side); one
// thread issues per K step of 8 and part (cos or -sin) an MMA of table hi x
// (B hi | B lo) with N = 64 and one of table lo x B hi with N = 32, M = 128,
// into one of NACC accumulator sets, and commits them to mbarriers; four
// warps read the accumulators with tcgen05.ld, add the hi x lo half, and
// write 128-byte-swizzled output tiles, which one thread stores by TMA.  All
// stages run concurrently on successive items, handing slots over through
// full / empty mbarrier rings.  Tensor memory: 4 Q columns of tables (cos
// hi, cos lo, -sin hi, -sin lo; lane = output row) and NACC x 2 x 64
// accumulator columns (512 allocated).  Every wait is bounded and
// gives up as soon as another thread of the CTA has given up; then bit 8 of
// the device flag is set and the CTA drains its copies and products
// (bounded), releases its tensor memory and leaves.
#include <cmath>
#include <cstring>
#include <vector>

#include "kernels.cuh"
#include "tma.cuh"

namespace blgpu {

using namespace tma;

namespace {
constexpr int UN = 32;        // kx columns per work item = N of the MMA

__device__ __forceinline__ uint32_t u_tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
// x -> (hi, lo) as TF32 bit patterns, x ~ hi + lo to ~2^-21: hi rounded to
// nearest, lo (exact in FP32) truncated to TF32
__device__ __forceinline__ void u_split(float x, uint32_t &hi, uint32_t &lo) {
  hi = u_tf32_rna(x);
  lo = __float_as_uint(x - __uint_as_float(hi)) & 0xffffe000u;
}

// B operand of one part (S or D: K x 64 = hi columns 0..31 | lo columns
// 32..63), K-major without swizzle: core matrices of 8 columns x 4 rows k
// (8 rows of 16 bytes, k fastest), the 8 column groups of a 4-row slab 128
// bytes apart (stride offset), slabs 1 KB apart (leading offset); one MMA
// (K = 8) reads two slabs.  The table's hi rows multiply hi | lo at once
// (N = 64), its lo rows the hi columns (N = 32).
__device__ __forceinline__ uint32_t b_off4(int k4, int n, int lo) {  // 16-byte chunk of rows 4 k4 .. 4 k4 + 3
  return ((uint32_t)k4 << 10) + ((uint32_t)(4 * lo + (n >> 3)) << 7) + ((uint32_t)(n & 7) << 4);
}
// shared-memory matrix descriptor: start address, leading offset 1 KB (next
// core matrix along K), stride offset 128 B (next one along N), version 1,
// no swizzle
__device__ __forceinline__ uint64_t b_desc(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((1024u >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}
// instruction descriptors: F32 accumulate, A and B TF32, both K-major (A in
// tensor memory), M = 128, N = 64 or 32
constexpr uint32_t idesc_n(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
constexpr uint32_t IDESC64 = idesc_n(2 * UN), IDESC32 = idesc_n(UN);

template <uint32_t ID>
__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %3, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %4, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(bdesc), "r"(acc), "n"(ID)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
          taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
      "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
      : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
}  // namespace

// bytes of one output tile (forward: two halves of MH rows; inverse: M rows;
// 128 bytes a row, each part rounded up to 1 KB)
__host__ __device__ inline uint32_t u_otile_bytes(int M, int MH) {
  const uint32_t f = 2u * (((uint32_t)MH * 128u + 1023u) & ~1023u);
  const uint32_t i = ((uint32_t)M * 128u + 1023u) & ~1023u;
  return f > i ? f : i;
}
// byte offset of 16-byte chunk c of row r in a 128-byte-swizzled tile
__device__ __forceinline__ uint32_t sw128(int r, int c) { return ((uint32_t)r << 7) + ((uint32_t)((c ^ r) & 7) << 4); }

// Warp roles (16 warps): warp 0 lane 0 issues the TMA copies of the raw
// columns, warp 1 lane 0 the MMAs, warp 2 lane 0 the TMA stores of the
// output tiles; warps 4-11 split raw columns into B operands, warps 12-15
// (one per 32 tensor-memory lanes) read the accumulators and write the
// output tiles.  Every hand-off is an mbarrier ring: raw (NRAW), B (NB), accumulator
// pairs (NACC), output tiles (NOUT), each with a "full" and an "empty"
// barrier; a producer waits for the empty phase before reusing a slot.
constexpr int NB = 2;
constexpr int SPLIT_W = 8;                          // warps that split raw columns
constexpr int EPI_W0 = 4 + SPLIT_W;                 // first of the four epilogue warps
constexpr int WS_WARPS = EPI_W0 + 4, WS_THREADS = WS_WARPS * 32;
static_assert(EPI_W0 % 4 == 0, "epilogue warp w serves tensor-memory lanes 32 (w % 4) ..");

// Shared memory, from a 1 KB aligned base: B[NB][4 operands][Q/8 K-steps of
// 1 KB] | raw[NRAW][rawf floats] | output tiles[NOUT] (1 KB aligned) |
// mbarriers | tmem slot and failure flag.
template <int QP, int NRAW, int NOUT>
__global__ void __launch_bounds__(WS_THREADS, 1)
    k_zdft_umma(const __grid_constant__ CUtensorMap mapR, const __grid_constant__ CUtensorMap mapC,
                const __grid_constant__ CUtensorMap mapRs, const __grid_constant__ CUtensorMap mapCs, Spec s,
                const uint32_t *__restrict__ tab, int inverse, int rawf, int *__restrict__ err) {
  constexpr int KS = QP / 8;                    // K steps (2 KB of B each) per product
  constexpr uint32_t OPB = (uint32_t)KS << 11;  // bytes of one part (hi | lo) of B
  // accumulator sets of 2 parts x 64 columns: two where the tables leave room
  constexpr int NACC = 4 * QP + 2 * 128 <= 512 ? 2 : 1;
  // tensor-memory columns: tables and accumulators, rounded up to a power of two
  constexpr uint32_t TCOLS = (4 * QP + NACC * 128) <= 256 ? 256u : 512u;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t s0 = smem_u32(smem_raw);
  unsigned char *sm = smem_raw + ((1024u - (s0 & 1023u)) & 1023u);
  unsigned char *Bb = sm;                                          // NB x 2 x OPB
  float *raw0 = reinterpret_cast<float *>(sm + NB * 2 * OPB);      // [NRAW][rawf]
  const uint32_t ohb = ((uint32_t)s.MH * 128u + 1023u) & ~1023u;  // one forward half
  const uint32_t otb = u_otile_bytes(s.M, s.MH);
  unsigned char *ot0 = reinterpret_cast<unsigned char *>(raw0 + NRAW * (size_t)rawf);
  ot0 += (1024u - (smem_u32(ot0) & 1023u)) & 1023u;
  uint64_t *raw_full = reinterpret_cast<uint64_t *>(ot0 + NOUT * otb);
  uint64_t *raw_empty = raw_full + NRAW;
  uint64_t *b_full = raw_empty + NRAW, *b_empty = b_full + NB;
  uint64_t *acc_full = b_empty + NB, *acc_empty = acc_full + NACC;
  uint64_t *out_full = acc_empty + NACC, *out_empty = out_full + NOUT;
  uint32_t *slot = reinterpret_cast<uint32_t *>(out_empty + NOUT);  // tensor-memory base
  volatile int *fail_s = reinterpret_cast<volatile int *>(slot + 1);  // a wait ran out
  const int M = s.M, MH = s.MH, H = (M - 1) / 2;
  const bool even = (M & 1) == 0;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntile = (s.N + UN - 1) / UN;
  const int nitems = s.NM * ntile;
  const int G = gridDim.x;
  const int nmine = ((int)blockIdx.x < nitems) ? (nitems - 1 - (int)blockIdx.x) / G + 1 : 0;
  // ---- set-up: tensor memory, barriers, tables ----
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 32) {
    *fail_s = 0;
    for (int q = 0; q < NRAW; ++q) {
      mbar_init(&raw_full[q], 1);
      mbar_init(&raw_empty[q], SPLIT_W);
    }
    for (int q = 0; q < NB; ++q) {
      mbar_init(&b_full[q], SPLIT_W);
      mbar_init(&b_empty[q], 1);
    }
    for (int q = 0; q < NACC; ++q) {
      mbar_init(&acc_full[q], 1);
      mbar_init(&acc_empty[q], 4);
    }
    for (int q = 0; q < NOUT; ++q) {
      mbar_init(&out_full[q], 4);
      mbar_init(&out_empty[q], 1);
    }
    mbar_init_fence();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *slot;
  const uint32_t tab_col = 0, acc_col = 4 * QP;  // tables, then the accumulator pairs
  if (warp >= EPI_W0) {
    // table t (0 cos hi, 1 cos lo, 2 -sin hi, 3 -sin lo) in columns t*QP.. of
    // lane = output row, by the warp of that lane quarter
    const int row = 32 * (warp & 3) + lane;
    const uint32_t lb = (uint32_t)(32 * (warp & 3)) << 16;
    for (int t = 0; t < 4; ++t)
      for (int c0 = 0; c0 < QP; c0 += 16) {
        uint32_t r[16];
        const uint32_t *src = tab + ((size_t)t * 128 + row) * QP + c0;
#pragma unroll
        for (int j = 0; j < 16; ++j) r[j] = src[j];
        tmem_st16(tmem + lb + tab_col + t * QP + c0, r);
      }
    tmem_wait_st();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  int issued_loads = 0, issued_mma = 0;  // for the bounded drain after a failure
  if (warp == 0 && lane == 0) {
    // ---- TMA producer: raw columns of item i into raw[i % NRAW] ----
    const uint32_t box_bytes = inverse ? (uint32_t)MH * 2 * UN * 4 : (uint32_t)M * UN * 4;
    for (int i = 0; i < nmine; ++i) {
      const int r = i % NRAW;
      if (!mbar_wait_or_fail(&raw_empty[r], ((uint32_t)(i / NRAW) & 1u) ^ 1u, fail_s)) break;
      const int item = blockIdx.x + i * G;
      const int b = item / ntile, kx0 = (item % ntile) * UN;
      float *dst = raw0 + (size_t)r * rawf;
      mbar_expect_tx(&raw_full[r], box_bytes);
      if (inverse) load_2d(dst, &mapC, 2 * kx0, b * MH, &raw_full[r]);
      else load_2d(dst, &mapR, kx0, b * M, &raw_full[r]);
      issued_loads = i + 1;
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer: item i from B[i % NB] into accumulator pair i % NACC ----
    for (int i = 0; i < nmine; ++i) {
      const int bs = i % NB, a = i % NACC;
      if (!mbar_wait_or_fail(&b_full[bs], (uint32_t)(i / NB) & 1u, fail_s)) break;
      if (!mbar_wait_or_fail(&acc_empty[a], ((uint32_t)(i / NACC) & 1u) ^ 1u, fail_s)) break;
      tc_fence_after();
      const uint32_t sB = smem_u32(Bb + (size_t)bs * 2 * OPB);
#pragma unroll
      for (int part = 0; part < 2; ++part) {  // 0: cos x S (or Re), 1: -sin x D (or Im)
        // columns 0..31: table hi x B hi + table lo x B hi; 32..63: table hi x B lo
        const uint32_t d = tmem + acc_col + (uint32_t)(a * 128 + part * 64);
        const uint32_t ahi = tmem + tab_col + (uint32_t)((2 * part) * QP);
        const uint32_t alo = ahi + QP;
        uint64_t db = b_desc(sB + (uint32_t)part * OPB);
#pragma unroll
        for (int ks = 0; ks < KS; ++ks) {
          umma_tf32<IDESC64>(d, ahi + 8 * ks, db, ks > 0 ? 1u : 0u);  // hi x (hi | lo)
          umma_tf32<IDESC32>(d, alo + 8 * ks, db, 1u);                // lo x hi
          db += 128;                                                   // 2 KB
        }
      }
      umma_commit(&b_empty[bs]);   // B[bs] free once these products are done
      umma_commit(&acc_full[a]);   // and the accumulators ready
      issued_mma = i + 1;
    }
  } else if (warp == 2 && lane == 0) {
    // ---- TMA stores of the output tiles ----
    for (int i = 0; i < nmine; ++i) {
      const int o = i % NOUT;
      if (!mbar_wait_or_fail(&out_full[o], (uint32_t)(i / NOUT) & 1u, fail_s)) break;
      const int item = blockIdx.x + i * G;
      const int b = item / ntile, kx0 = (item % ntile) * UN;
      const unsigned char *ot = ot0 + (size_t)o * otb;
      if (!inverse) {
        store_2d(&mapCs, ot, 2 * kx0, b * MH);
        store_2d(&mapCs, ot + ohb, 2 * kx0 + UN, b * MH);
      } else {
        store_2d(&mapRs, ot, kx0, b * M);
      }
      store_commit();
      store_wait_read<0>();
      mbar_arrive(&out_empty[o]);
    }
    store_wait_all();  // no store reads shared memory after this CTA leaves
  } else if (warp >= 4 && warp < EPI_W0) {
    // ---- split raw columns into the B operands ----
    // thread: column n = lane, rows k = 4 k4 .. 4 k4 + 3 for k4 = sw, sw + SPLIT_W, ..;
    // one 16-byte chunk per operand.  The f_{M/2} term (forward, even M) and
    // the c0 and Nyquist terms (inverse, halved) ride in the products as rows
    // 0 and M/2 of the tables, so the epilogue needs nothing else.
    const int sw = warp - 4, n = lane;
    constexpr int NJ = (QP / 4 + SPLIT_W - 1) / SPLIT_W;  // slabs per warp
    for (int i = 0; i < nmine; ++i) {
      const int r = i % NRAW, bs = i % NB;
      const int item = blockIdx.x + i * G;
      const int col = (item % ntile) * UN + n;
      const bool okc = col < s.N;
      if (!mbar_wait_or_fail(&raw_full[r], (uint32_t)(i / NRAW) & 1u, fail_s)) break;
      if (!mbar_wait_or_fail(&b_empty[bs], ((uint32_t)(i / NB) & 1u) ^ 1u, fail_s)) break;
      const float *rw = raw0 + (size_t)r * rawf;
      unsigned char *Bi = Bb + (size_t)bs * 2 * OPB;
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const int k4 = sw + SPLIT_W * j;
        if (k4 >= QP / 4) break;
        uint4 h0, l0, h1, l1;
        uint32_t *ph0 = &h0.x, *pl0 = &l0.x, *ph1 = &h1.x, *pl1 = &l1.x;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int k = 4 * k4 + e;
          float x0 = 0.f, x1 = 0.f;
          if (okc) {
            if (!inverse) {
              if (k == 0) {
                x0 = rw[n];
              } else if (k <= H) {
                const float fk = rw[k * UN + n], fm = rw[(M - k) * UN + n];
                x0 = fk + fm;
                x1 = fk - fm;
              } else if (even && k == M / 2) {
                x0 = rw[k * UN + n];
              }
            } else {
              const float2 *cw = reinterpret_cast<const float2 *>(rw);
              if (k == 0 || (even && k == M / 2)) {
                x0 = 0.5f * cw[k * UN + n].x;
              } else if (k <= H) {
                const float2 v = cw[k * UN + n];
                x0 = v.x;
                x1 = v.y;
              }
            }
          }
          u_split(x0, ph0[e], pl0[e]);
          u_split(x1, ph1[e], pl1[e]);
        }
        *reinterpret_cast<uint4 *>(Bi + b_off4(k4, n, 0)) = h0;
        *reinterpret_cast<uint4 *>(Bi + b_off4(k4, n, 1)) = l0;
        *reinterpret_cast<uint4 *>(Bi + OPB + b_off4(k4, n, 0)) = h1;
        *reinterpret_cast<uint4 *>(Bi + OPB + b_off4(k4, n, 1)) = l1;
      }
      fence_async_shared();  // the B operands before the tensor cores read them
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&raw_empty[r]);
        mbar_arrive(&b_full[bs]);
      }
    }
  } else if (warp >= EPI_W0) {
    // ---- epilogue: accumulators -> swizzled output tile ----
    const int row = 32 * (warp & 3) + lane;
    const uint32_t lb = (uint32_t)(32 * (warp & 3)) << 16;
    const float scale = 2.0f / (float)M;
    for (int i = 0; i < nmine; ++i) {
      const int a = i % NACC, o = i % NOUT;
      if (!mbar_wait_or_fail(&acc_full[a], (uint32_t)(i / NACC) & 1u, fail_s)) break;
      tc_fence_after();
      const uint32_t acc = tmem + lb + acc_col + (uint32_t)(a * 128);
      // re = cos part, im = -sin part, each the sum of (table hi x B hi +
      // table lo x B hi) and (table hi x B lo); the accumulators are free for
      // the next item's products as soon as they are read
      float re[32], im[32];
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int part = 0; part < 2; ++part) {
          float x[16], y[16];
          tmem_ld16(acc + part * 64 + 16 * h, x);
          tmem_ld16(acc + part * 64 + 32 + 16 * h, y);
          tmem_wait_ld();
          float *v = (part ? im : re) + 16 * h;
#pragma unroll
          for (int j = 0; j < 16; ++j) v[j] = x[j] + y[j];
        }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[a]);
      if (!mbar_wait_or_fail(&out_empty[o], ((uint32_t)(i / NOUT) & 1u) ^ 1u, fail_s)) break;
      unsigned char *ot = ot0 + (size_t)o * otb;
      if (!inverse) {
        if (row < MH) {
#pragma unroll
          for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int c = 0; c < 8; ++c) {  // chunk c of half h: complex values 16h + 2c, 16h + 2c + 1
              const int q = 16 * h + 2 * c;
              *reinterpret_cast<float4 *>(ot + h * ohb + sw128(row, c)) =
                  make_float4(re[q], im[q], re[q + 1], im[q + 1]);
            }
        }
      } else if (row <= M / 2) {
        const int pm = M - row;
        const bool two = pm != row && pm < M;
#pragma unroll
        for (int c = 0; c < 8; ++c) {  // chunk c: values 4c .. 4c + 3
          float f1[4], f2[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            f1[e] = (re[4 * c + e] + im[4 * c + e]) * scale;
            f2[e] = (re[4 * c + e] - im[4 * c + e]) * scale;
          }
          *reinterpret_cast<float4 *>(ot + sw128(row, c)) = make_float4(f1[0], f1[1], f1[2], f1[3]);
          if (two) *reinterpret_cast<float4 *>(ot + sw128(pm, c)) = make_float4(f2[0], f2[1], f2[2], f2[3]);
        }
      }
      fence_async_shared();  // the tile's writes before the TMA store reads them
      __syncwarp();
      if (lane == 0) mbar_arrive(&out_full[o]);
    }
  }
  __syncwarp();
  __syncthreads();
  const bool failed = *fail_s != 0;
  if (failed) {
    // let the copies and products this CTA issued finish (bounded), then leave
    if (warp == 0 && lane == 0) {
      atomicOr(err, 8);
      for (int i = issued_loads - NRAW > 0 ? issued_loads - NRAW : 0; i < issued_loads; ++i)
        mbar_wait(&raw_full[i % NRAW], (uint32_t)(i / NRAW) & 1u);
    }
    if (warp == 1 && lane == 0 && issued_mma > 0) {
      const int i = issued_mma - 1;
      mbar_wait(&acc_full[i % NACC], (uint32_t)(i / NACC) & 1u);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS) : "memory");
  }
}

namespace {
int u_raw_floats(const Spec &s) {
  const int f = s.M * UN > s.MH * 2 * UN ? s.M * UN : s.MH * 2 * UN;
  return (f + 31) / 32 * 32;
}
size_t u_smem_bytes(const Spec &s, int qp, int NRAW, int NOUT) {
  // the output tiles start at the next 1 KB boundary after raw (at most 1 KB on)
  return 1024 + (size_t)NB * 4 * (qp / 8) * 1024 + (size_t)NRAW * u_raw_floats(s) * sizeof(float) + 1024 +
         NOUT * (size_t)u_otile_bytes(s.M, s.MH) + 2 * (NRAW + NB + 2 + NOUT) * sizeof(uint64_t) +
         16;  // the last 16: tensor-memory slot and failure flag
}
uint32_t tf32_host_rna(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return u;
  u += 0x1000u;  // round half away from zero on the magnitude, as cvt.rna
  return u & 0xffffe000u;
}
}  // namespace

// order served by the tcgen05 path (same set as the mma.sync path), 0 if not
int zdft_umma_qp(const Spec &s) {
  const int qp = zdft_tc_qp(s);
  if (!qp) return 0;
  if (u_smem_bytes(s, qp, 2, 1) > 227 * 1024) return 0;
  return qp;
}

// ring depths (raw buffers, output tiles) for the box: the deepest of these
// configurations that fits the shared memory (at 814 x 257 x 193 the depths
// from (2, 1) to (4, 1) time alike)
static void u_rings(const Spec &s, int qp, int *nraw, int *nout) {
  static const int cfg[][2] = {{4, 2}, {4, 1}, {3, 2}, {2, 2}, {2, 1}};
  for (int c = 0; c < 5; ++c)
    if (u_smem_bytes(s, qp, cfg[c][0], cfg[c][1]) <= 227 * 1024) {
      *nraw = cfg[c][0];
      *nout = cfg[c][1];
      return;
    }
  *nraw = 2;
  *nout = 1;
}

// tables [4][128][QP] of TF32 bit patterns: cos hi, cos lo, -sin hi, -sin lo
// of 2 pi m n / M (m = row, n = column; zero beyond Q)
void zdft_umma_tables(const Spec &s, std::vector<uint32_t> &out) {
  const int qp = zdft_umma_qp(s), M = s.M, Q = s.MH;
  out.assign((size_t)4 * 128 * qp, 0u);
  for (int m = 0; m < Q; ++m)
    for (int n = 0; n < Q; ++n) {
      const double a = 2.0 * M_PI * (double)(((long long)m * n) % M) / (double)M;
      const float c = (float)cos(a), sn = (float)-sin(a);
      const float v[2] = {c, sn};
      for (int t = 0; t < 2; ++t) {
        const uint32_t hi = tf32_host_rna(v[t]);
        float hf;
        memcpy(&hf, &hi, 4);
        out[((size_t)(2 * t) * 128 + m) * qp + n] = hi;
        out[((size_t)(2 * t + 1) * 128 + m) * qp + n] = tf32_host_rna(v[t] - hf);
      }
    }
}

// tensor maps: R with boxes 32 x M, C (as floats) with boxes 64 x MH for the
// loads; for the stores R with boxes 32 x M and C with boxes 32 x MH (one
// 128-byte row each), swizzled by 128 bytes
bool zdft_umma_maps(const Spec &s, float *R, float2 *C, ZdftMaps *out) {
  CUtensorMap mr, mc, mrs, mcs;
  const cuuint64_t dr[2] = {(cuuint64_t)s.rx, (cuuint64_t)s.NM * s.M};
  const cuuint64_t sr[1] = {(cuuint64_t)s.rx * sizeof(float)};
  const cuuint32_t br[2] = {(cuuint32_t)UN, (cuuint32_t)s.M};
  if (!encode(&mr, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, R, dr, sr, br)) return false;
  const cuuint64_t dc[2] = {(cuuint64_t)2 * s.rx, (cuuint64_t)s.NM * s.MH};
  const cuuint64_t sc[1] = {(cuuint64_t)2 * s.rx * sizeof(float)};
  const cuuint32_t bc[2] = {(cuuint32_t)(2 * UN), (cuuint32_t)s.MH};
  if (!encode(&mc, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, C, dc, sc, bc)) return false;
  if (!encode(&mrs, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, R, dr, sr, br, CU_TENSOR_MAP_SWIZZLE_128B)) return false;
  const cuuint32_t bcs[2] = {(cuuint32_t)UN, (cuuint32_t)s.MH};
  if (!encode(&mcs, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, C, dc, sc, bcs, CU_TENSOR_MAP_SWIZZLE_128B)) return false;
  memcpy(out->r, &mr, sizeof mr);
  memcpy(out->c, &mc, sizeof mc);
  memcpy(out->rs, &mrs, sizeof mrs);
  memcpy(out->cs, &mcs, sizeof mcs);
  return true;
}

template <int QP, int NRAW, int NOUT>
static void launch_r(const Spec &s, const ZdftMaps &mp, const uint32_t *tab, int inverse, int nsm, int *err,
                     cudaStream_t st) {
  const size_t sm = u_smem_bytes(s, QP, NRAW, NOUT);
  cudaFuncSetAttribute(k_zdft_umma<QP, NRAW, NOUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  const int nitems = s.NM * ((s.N + UN - 1) / UN);
  const int grid = nitems < nsm ? nitems : nsm;
  CUtensorMap mr, mc, mrs, mcs;
  memcpy(&mr, mp.r, sizeof mr);
  memcpy(&mc, mp.c, sizeof mc);
  memcpy(&mrs, mp.rs, sizeof mrs);
  memcpy(&mcs, mp.cs, sizeof mcs);
  k_zdft_umma<QP, NRAW, NOUT><<<grid, WS_THREADS, sm, st>>>(mr, mc, mrs, mcs, s, tab, inverse, u_raw_floats(s), err);
}

template <int QP>
static void launch_u(const Spec &s, const ZdftMaps &mp, float *R, float2 *C, const uint32_t *tab, int inverse,
                     int nsm, int *err, cudaStream_t st) {
  (void)R;
  (void)C;
  int nraw = 2, nout = 1;
  u_rings(s, QP, &nraw, &nout);
  if (nraw == 4 && nout == 2) launch_r<QP, 4, 2>(s, mp, tab, inverse, nsm, err, st);
  else if (nraw == 4) launch_r<QP, 4, 1>(s, mp, tab, inverse, nsm, err, st);
  else if (nraw == 3) launch_r<QP, 3, 2>(s, mp, tab, inverse, nsm, err, st);
  else if (nout == 2) launch_r<QP, 2, 2>(s, mp, tab, inverse, nsm, err, st);
  else launch_r<QP, 2, 1>(s, mp, tab, inverse, nsm, err, st);
}

void launch_zdft_umma(const Spec &s, const ZdftMaps &maps, float *R, float2 *C, const uint32_t *tab, int inverse,
                      int nsm, int *err, cudaStream_t st) {
  switch (zdft_umma_qp(s)) {
    case 32: launch_u<32>(s, maps, R, C, tab, inverse, nsm, err, st); break;
    case 48: launch_u<48>(s, maps, R, C, tab, inverse, nsm, err, st); break;
    case 64: launch_u<64>(s, maps, R, C, tab, inverse, nsm, err, st); break;
    case 80: launch_u<80>(s, maps, R, C, tab, inverse, nsm, err, st); break;
    case 96: launch_u<96>(s, maps, R, C, tab, inverse, nsm, err, st); break;
    default: break;
  }
}

}  // namespace blgpu
