// zdft_umma.cu -- the mixed form's z transforms on the 5th-generation tensor
// cores: tcgen05.mma kind::tf32 with the cos / -sin tables resident in tensor
// memory (A operand), the split line data staged in shared memory (B
// operand, K-major core matrices) and the FP32 accumulators in tensor
// memory.  Same products as zdft_tc.cu (real DFT over the half spectrum as
// two square products of order Q = M/2+1 with the f_k +- f_{M-k} pairing,
// three-term TF32 split hi*hi + hi*lo + lo*hi); see there for the algebra.
//
// One persistent CTA (8 warps) per SM.  Work items are (row b, 32 kx
// columns).  Per item: one TMA tensor copy brings the raw columns (NRAW
// buffers, NRAW-1 items ahead); the CTA splits them into the B operands (double
// buffer); one thread issues the 3 x Q/8 x 2 MMAs of M = 128, N = 32, K = 8
// into one of two accumulator pairs and commits them to an mbarrier; while
// they run, the CTA reads the previous item's accumulators with tcgen05.ld
// and writes that item's output rows.  Tensor memory: 4 Q columns of tables
// (cos hi, cos lo, -sin hi, -sin lo; lane = output row) and 2 x 2 x 32
// accumulator columns (256 or 512 allocated).  Every wait is bounded; a wait that
// runs out sets bit 8 of the device flag and the CTA releases its tensor
// memory and leaves.
#include <cmath>
#include <cstring>
#include <vector>

#include "kernels.cuh"
#include "tma.cuh"

namespace blgpu {

using namespace tma;

namespace {
constexpr int UN = 32;        // kx columns per work item = N of the MMA
constexpr int UWARPS = 8;     // warps per CTA
constexpr int UTHREADS = UWARPS * 32;
constexpr int NRAW = 2;       // raw column buffers: copies of the next NRAW-1 items in flight (3 measured slower)

__device__ __forceinline__ uint32_t u_tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
// x -> (hi, lo) as TF32 bit patterns, x ~ hi + lo to ~2^-22
__device__ __forceinline__ void u_split(float x, uint32_t &hi, uint32_t &lo) {
  hi = u_tf32_rna(x);
  lo = u_tf32_rna(x - __uint_as_float(hi));
}

// B operand (K x N = 32), K-major without swizzle: core matrices of 8
// columns n x 4 rows k (8 rows of 16 bytes, k fastest), the 4 column groups
// of a 4-row slab 128 bytes apart (stride offset), slabs 512 bytes apart
// (leading offset); one MMA (K = 8) reads two slabs, 1 KB
__device__ __forceinline__ uint32_t b_off4(int k4, int n) {  // 16-byte chunk of rows 4 k4 .. 4 k4 + 3
  return ((uint32_t)k4 << 9) + ((uint32_t)(n >> 3) << 7) + ((uint32_t)(n & 7) << 4);
}
// shared-memory matrix descriptor: start address, leading offset 512 B (next
// core matrix along K), stride offset 128 B (next one along N), version 1,
// no swizzle
__device__ __forceinline__ uint64_t b_desc(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((512u >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}
// instruction descriptor: F32 accumulate, A and B TF32, both K-major (A in
// tensor memory), N = 32, M = 128
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(UN >> 3) << 17) |
                           ((uint32_t)(128 >> 4) << 24);

__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %3, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %4, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(bdesc), "r"(acc), "r"(IDESC)
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

// Shared memory, from a 1 KB aligned base: B[2 buffers][4 operands][Q/8
// K-steps of 1 KB] | raw[NRAW][rawf floats] | aux[2][2][32] | output tiles[2]
// (1 KB aligned) | 4 mbarriers | tmem slot and failure flag.
template <int QP>
__global__ void __launch_bounds__(UTHREADS, 1)
    k_zdft_umma(const __grid_constant__ CUtensorMap mapR, const __grid_constant__ CUtensorMap mapC,
                const __grid_constant__ CUtensorMap mapRs, const __grid_constant__ CUtensorMap mapCs, Spec s,
                const uint32_t *__restrict__ tab, int inverse, int rawf, int *__restrict__ err) {
  constexpr int KS = QP / 8;                 // K steps (1 KB of B each) per product
  constexpr uint32_t OPB = (uint32_t)KS << 10;  // bytes of one B operand
  // tensor-memory columns: tables and accumulators, rounded up to a power of two
  constexpr uint32_t TCOLS = (4 * QP + 4 * UN) <= 256 ? 256u : 512u;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1 KB alignment of the B operands
  const uint32_t s0 = smem_u32(smem_raw);
  unsigned char *sm = smem_raw + ((1024u - (s0 & 1023u)) & 1023u);
  unsigned char *Bb = sm;                                          // 2 x 4 x OPB
  float *raw0 = reinterpret_cast<float *>(sm + 8 * OPB);           // [NRAW][rawf]
  float *aux = raw0 + NRAW * (size_t)rawf;                         // [2][2][UN]
  // output tiles [2][otb bytes], 1 KB aligned (128-byte swizzle): forward two
  // halves of MH rows x 16 complex, inverse M rows x 32 values, 128 B a row
  const uint32_t ohb = ((uint32_t)s.MH * 128u + 1023u) & ~1023u;  // one forward half
  const uint32_t otb = u_otile_bytes(s.M, s.MH);
  unsigned char *ot0 = reinterpret_cast<unsigned char *>(aux + 4 * UN);
  ot0 += (1024u - (smem_u32(ot0) & 1023u)) & 1023u;
  uint64_t *tbar = reinterpret_cast<uint64_t *>(ot0 + 2 * otb);    // TMA, per raw buffer
  uint64_t *mbar = tbar + NRAW;                                    // MMA, per accumulator pair
  uint32_t *slot = reinterpret_cast<uint32_t *>(mbar + 2);         // tensor-memory base
  int *fail_s = reinterpret_cast<int *>(slot + 1);                  // a warp's wait ran out
  const int M = s.M, MH = s.MH, H = (M - 1) / 2;
  const bool even = (M & 1) == 0;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntile = (s.N + UN - 1) / UN;
  const int nitems = s.NM * ntile;
  const int G = gridDim.x;
  const uint32_t box_bytes = inverse ? (uint32_t)MH * 2 * UN * 4 : (uint32_t)M * UN * 4;
  auto issue_copy = [&](int item, int buf) {
    const int b = item / ntile, kx0 = (item % ntile) * UN;
    float *dst = raw0 + (size_t)buf * rawf;
    mbar_expect_tx(&tbar[buf], box_bytes);
    if (inverse) load_2d(dst, &mapC, 2 * kx0, b * MH, &tbar[buf]);
    else load_2d(dst, &mapR, kx0, b * M, &tbar[buf]);
  };
  // ---- set-up: tensor memory, barriers, first copy, tables ----
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 32) {
    *fail_s = 0;
    for (int q = 0; q < NRAW; ++q) mbar_init(&tbar[q], 1);
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    mbar_init_fence();
    for (int q = 0; q < NRAW - 1; ++q)
      if ((int)blockIdx.x + q * G < nitems) issue_copy(blockIdx.x + q * G, q);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *slot;
  const uint32_t tab_col = 0, acc_col = 4 * QP;  // tables, then the accumulators
  const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
  {
    // table t (0 cos hi, 1 cos lo, 2 -sin hi, 3 -sin lo) in columns t*QP.. of
    // lane = output row; the two warps of a lane quarter take two tables each
    const int row = 32 * (warp & 3) + lane;
    for (int t = 2 * (warp >> 2); t < 2 * (warp >> 2) + 2; ++t)
      for (int c0 = 0; c0 < QP; c0 += 16) {
        uint32_t r[16];
        const uint32_t *src = tab + ((size_t)t * 128 + row) * QP + c0;
#pragma unroll
        for (int j = 0; j < 16; ++j) r[j] = src[j];
        tmem_st16(tmem + lane_base + tab_col + t * QP + c0, r);
      }
    tmem_wait_st();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const int nmine = ((int)blockIdx.x < nitems) ? (nitems - 1 - (int)blockIdx.x) / G + 1 : 0;
  bool failed = false;
  // epilogue of local item j (accumulator pair j & 1, output tile j & 1):
  // each warp waits for the products itself (the issuing warp does not hold
  // the others back) and moves its rows from tensor memory into the swizzled
  // output tile; the tile leaves by TMA store, issued after the next barrier
  auto epilogue = [&](int j) {
    const int bb = j & 1;
    if (!mbar_wait_hw(&mbar[bb], (uint32_t)(j >> 1) & 1u)) {
      atomicExch(fail_s, 1);
      return;
    }
    tc_fence_after();
    const int row = 32 * (warp & 3) + lane, h = warp >> 2;  // output row, column half
    float re[16], im[16];
    const uint32_t acc = tmem + lane_base + acc_col + (uint32_t)(bb * 2 * UN) + 16 * h;
    tmem_ld16(acc, re);
    tmem_ld16(acc + UN, im);
    tmem_wait_ld();
    tc_fence_before();
    const float *ax = aux + bb * 2 * UN;
    unsigned char *ot = ot0 + (size_t)bb * otb;
    if (!inverse) {
      if (row < MH) {
        unsigned char *oh = ot + h * ohb;
#pragma unroll
        for (int c = 0; c < 8; ++c) {  // chunk c: complex values 2c, 2c+1 of this half
          const int q = 2 * c;
          const float v0 = even ? re[q] + ((row & 1) ? -ax[16 * h + q] : ax[16 * h + q]) : re[q];
          const float v1 = even ? re[q + 1] + ((row & 1) ? -ax[16 * h + q + 1] : ax[16 * h + q + 1]) : re[q + 1];
          *reinterpret_cast<float4 *>(oh + sw128(row, c)) = make_float4(v0, im[q], v1, im[q + 1]);
        }
      }
    } else {
      const int npairs = M / 2 + 1;
      if (row < npairs) {
        const float invM = 1.0f / (float)M;
        const int pm = M - row;
        const bool two = pm != row && pm < M;
#pragma unroll
        for (int c = 0; c < 4; ++c) {  // chunk 4h + c: values 16h + 4c .. 16h + 4c + 3
          float f1[4], f2[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int q = 4 * c + e;
            const float c0 = ax[16 * h + q];
            const float y = even ? ((row & 1) ? -ax[UN + 16 * h + q] : ax[UN + 16 * h + q]) : 0.f;
            f1[e] = (c0 + 2.0f * (re[q] + im[q]) + y) * invM;
            f2[e] = (c0 + 2.0f * (re[q] - im[q]) + y) * invM;
          }
          *reinterpret_cast<float4 *>(ot + sw128(row, 4 * h + c)) = make_float4(f1[0], f1[1], f1[2], f1[3]);
          if (two) *reinterpret_cast<float4 *>(ot + sw128(pm, 4 * h + c)) = make_float4(f2[0], f2[1], f2[2], f2[3]);
        }
      }
    }
    fence_async_shared();  // the tile's writes before the TMA store reads them
  };
  // TMA store of the output tile of local item j (all its writers have
  // passed a barrier since)
  auto store_tile = [&](int j) {
    const int item = blockIdx.x + j * G, bb = j & 1;
    const int b = item / ntile, kx0 = (item % ntile) * UN;
    const unsigned char *ot = ot0 + (size_t)bb * otb;
    if (!inverse) {
      store_2d(&mapCs, ot, 2 * kx0, b * MH);
      store_2d(&mapCs, ot + ohb, 2 * kx0 + UN, b * MH);
    } else {
      store_2d(&mapRs, ot, kx0, b * M);
    }
  };
  for (int i = 0; i < nmine && !failed; ++i) {
    const int item = blockIdx.x + i * G, bb = i & 1;
    const int kx0 = (item % ntile) * UN;
    // raw buffer (i-1) mod NRAW and this item's B buffer are free: their
    // last readers (staging of item i-1, MMAs of item i-2) finished before here
    if (__syncthreads_or(*fail_s)) {
      failed = true;
      break;
    }
    if (tid == 0 && i >= 2) {
      // the tile of item i-2 (written before the barrier above) leaves; the
      // one of item i-3 must be read out before epilogue(i-1) reuses its buffer
      store_tile(i - 2);
      store_commit();
      store_wait_read<1>();
    }
    const int rb = i % NRAW;
    if (tid == 32 && i + NRAW - 1 < nmine) {
      fence_async_shared();
      issue_copy(item + (NRAW - 1) * G, (i + NRAW - 1) % NRAW);
    }
    const bool ok = mbar_wait_hw(&tbar[rb], (uint32_t)(i / NRAW) & 1u);
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    // ---- split the operands of item i into B[bb] ----
    // a thread takes column n and four consecutive rows k = 4 k4 .. 4 k4 + 3
    // and writes one 16-byte chunk per operand
    const float *rw = raw0 + (size_t)rb * rawf;
    unsigned char *Bi = Bb + (size_t)bb * 4 * OPB;
    const int n = lane, col = kx0 + n;
    const bool okc = col < s.N;
    for (int k4 = warp; k4 < QP / 4; k4 += UWARPS) {
      uint4 h0, l0, h1, l1;
      uint32_t *ph0 = &h0.x, *pl0 = &l0.x, *ph1 = &h1.x, *pl1 = &l1.x;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int k = 4 * k4 + r;
        float x0 = 0.f, x1 = 0.f;
        if (!inverse) {
          if (okc && k <= H) {
            const float fk = rw[k * UN + n];
            if (k == 0) {
              x0 = fk;
            } else {
              const float fm = rw[(M - k) * UN + n];
              x0 = fk + fm;
              x1 = fk - fm;
            }
          }
        } else if (okc && k >= 1 && k <= H) {
          const float2 v = reinterpret_cast<const float2 *>(rw)[k * UN + n];
          x0 = v.x;
          x1 = v.y;
        }
        u_split(x0, ph0[r], pl0[r]);
        u_split(x1, ph1[r], pl1[r]);
      }
      const uint32_t off = b_off4(k4, n);
      *reinterpret_cast<uint4 *>(Bi + 0 * OPB + off) = h0;
      *reinterpret_cast<uint4 *>(Bi + 1 * OPB + off) = l0;
      *reinterpret_cast<uint4 *>(Bi + 2 * OPB + off) = h1;
      *reinterpret_cast<uint4 *>(Bi + 3 * OPB + off) = l1;
    }
    if (warp == UWARPS - 1) {
      float *ax = aux + bb * 2 * UN;
      if (!inverse) {
        ax[n] = (okc && even) ? rw[(M / 2) * UN + n] : 0.f;  // f_{M/2}
      } else {
        const float2 *cw = reinterpret_cast<const float2 *>(rw);
        ax[n] = okc ? cw[n].x : 0.f;                                     // c0
        ax[UN + n] = (okc && even) ? cw[(M / 2) * UN + n].x : 0.f;       // Nyquist
      }
    }
    fence_async_shared();  // the B operands before the tensor cores read them
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t sB = smem_u32(Bi);
      // descriptors step by 1 KB (64 in the address field) per K step
#pragma unroll
      for (int part = 0; part < 2; ++part) {  // 0: cos x S (or Re), 1: -sin x D (or Im)
        const uint32_t d = tmem + acc_col + (uint32_t)(bb * 2 * UN + part * UN);
        const uint32_t ahi = tmem + tab_col + (uint32_t)((2 * part) * QP);
        const uint32_t alo = ahi + QP;
        uint64_t dh = b_desc(sB + (uint32_t)(2 * part) * OPB), dl = dh + (OPB >> 4);
#pragma unroll
        for (int ks = 0; ks < KS; ++ks) {
          umma_tf32(d, alo + 8 * ks, dh, ks > 0 ? 1u : 0u);  // lo x hi
          umma_tf32(d, ahi + 8 * ks, dl, 1u);                // hi x lo
          umma_tf32(d, ahi + 8 * ks, dh, 1u);                // hi x hi
          dh += 64;
          dl += 64;
        }
      }
      umma_commit(&mbar[bb]);
    }
    if (i >= 1) epilogue(i - 1);
  }
  if (!failed && nmine > 0) {
    if (tid == 0) store_wait_read<0>();  // the buffer of item nmine-1 is free
    __syncthreads();
    epilogue(nmine - 1);
  }
  if (__syncthreads_or(*fail_s)) failed = true;
  if (tid == 0) {
    if (!failed) {
      if (nmine >= 2) store_tile(nmine - 2);
      if (nmine >= 1) store_tile(nmine - 1);
      store_commit();
    }
    store_wait_all();  // no store reads shared memory after this CTA leaves
  }
  if (failed) {
    // let the copies and products this CTA issued finish (bounded), then leave
    if (tid == 0) {
      atomicOr(err, 8);
      for (int q = 0; q < 2; ++q) mbar_wait(&mbar[q], 0);
      for (int q = 0; q < NRAW; ++q) mbar_wait(&tbar[q], 0);
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
size_t u_smem_bytes(const Spec &s, int qp) {
  // the output tiles start at the next 1 KB boundary after aux (at most 1 KB on)
  return 1024 + (size_t)8 * (qp / 8) * 1024 + (size_t)NRAW * u_raw_floats(s) * sizeof(float) +
         4 * UN * sizeof(float) + 1024 + 2 * (size_t)u_otile_bytes(s.M, s.MH) + (NRAW + 2) * sizeof(uint64_t) +
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
  if (u_smem_bytes(s, qp) > 227 * 1024) return 0;
  return qp;
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

template <int QP>
static void launch_u(const Spec &s, const ZdftMaps &mp, float *R, float2 *C, const uint32_t *tab, int inverse,
                     int nsm, int *err, cudaStream_t st) {
  const size_t sm = u_smem_bytes(s, QP);
  cudaFuncSetAttribute(k_zdft_umma<QP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  const int nitems = s.NM * ((s.N + UN - 1) / UN);
  const int grid = nitems < nsm ? nitems : nsm;
  CUtensorMap mr, mc, mrs, mcs;
  memcpy(&mr, mp.r, sizeof mr);
  memcpy(&mc, mp.c, sizeof mc);
  memcpy(&mrs, mp.rs, sizeof mrs);
  memcpy(&mcs, mp.cs, sizeof mcs);
  (void)R;
  (void)C;
  k_zdft_umma<QP><<<grid, UTHREADS, sm, st>>>(mr, mc, mrs, mcs, s, tab, inverse, u_raw_floats(s), err);
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
