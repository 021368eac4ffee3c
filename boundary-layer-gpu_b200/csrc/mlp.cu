// mlp.cu -- the learned wall-stress closure: a 4-64-64-64-2 GELU network on
// the tensor cores (BF16 operands, FP32 accumulation, mma.sync m16n8k16),
// its forward, backward and Adam kernels, the training-sample extractor and
// the wall-model hook that turns a wall stress into the non-zero Neumann
// condition of boundary_conditions.f90:359-372.
//
// Warp tiling: a warp owns 16 rows (samples).  Layer outputs stay in the MMA
// accumulator layout, and two adjacent 8-column accumulator tiles are exactly
// the A fragment of the next 16-deep k-step, so activations pass from layer
// to layer in registers.  The weight gradients dW = delta^T h reduce over the
// 64 rows of a CTA tile with a second MMA from transposed shared-memory
// copies; each warp owns 16 output rows of dW, so the CTA accumulates its
// gradient in shared memory without atomics, and the CTA partials are summed
// in a fixed order by the update kernel (deterministic).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "mlp.cuh"

namespace blgpu {
using namespace mlp;

__device__ __forceinline__ uint32_t pk2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x (low half) = lo
  return *reinterpret_cast<uint32_t *>(&v);
}
__device__ __forceinline__ uint32_t ld2(const uint16_t *p) { return *reinterpret_cast<const uint32_t *>(p); }
__device__ __forceinline__ uint16_t bf(float v) {
  __nv_bfloat16 b = __float2bfloat16_rn(v);
  return *reinterpret_cast<uint16_t *>(&b);
}
__device__ __forceinline__ float unbf(uint16_t v) { return __uint_as_float(((uint32_t)v) << 16); }

__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// GELU(z) = z Phi(z) and its derivative Phi(z) + z phi(z)
__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// ---------------------------------------------------------------------------
// packing of the master parameters (also run after every update)
// ---------------------------------------------------------------------------
__device__ void pack_param(int p, float v, uint16_t *pack, float *bias) {
  if (p < OB0) {  // W0[o][i]
    const int o = p / NIN, i = p % NIN;
    pack[PW0 + o * S16 + i] = bf(v);
  } else if (p < OW1) {
    bias[p - OB0] = v;
  } else if (p < OB1) {
    const int q = p - OW1, o = q / NH, i = q % NH;
    pack[PW1 + o * S64 + i] = bf(v);
    pack[PT1 + i * S64 + o] = bf(v);
  } else if (p < OW2) {
    bias[64 + p - OB1] = v;
  } else if (p < OB2) {
    const int q = p - OW2, o = q / NH, i = q % NH;
    pack[PW2 + o * S64 + i] = bf(v);
    pack[PT2 + i * S64 + o] = bf(v);
  } else if (p < OW3) {
    bias[128 + p - OB2] = v;
  } else if (p < OB3) {
    const int q = p - OW3, o = q / NH, i = q % NH;
    pack[PW3 + o * S64 + i] = bf(v);
    pack[PT3 + i * S16 + o] = bf(v);
  } else {
    bias[192 + p - OB3] = v;
  }
}

__global__ void k_mlp_clear(uint16_t *__restrict__ pack, float *__restrict__ bias) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < PACKN; q += gridDim.x * blockDim.x) pack[q] = 0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < BIASN; q += gridDim.x * blockDim.x) bias[q] = 0.f;
}
__global__ void k_mlp_pack(const float *__restrict__ params, uint16_t *__restrict__ pack, float *__restrict__ bias) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < NP; p += gridDim.x * blockDim.x)
    pack_param(p, params[p], pack, bias);
}

// ---------------------------------------------------------------------------
// warp forward pass over 16 rows
// ---------------------------------------------------------------------------
struct WarpFwd {
  float gp[3][8][4];  // GELU'(z) of the three hidden layers (accumulator layout)
  float y[4];         // output accumulator: (row g: y0 y1, row g+8: y0 y1) on tig 0
};

// ax: A fragment of the inputs; hT0..2 (TRAIN only): transposed BF16 copies
// of the hidden activations [unit][row], rows r0.. of the CTA tile
template <bool TRAIN>
__device__ __forceinline__ void warp_forward(const uint16_t *Ws, const float *bs, const uint32_t (&ax)[4], WarpFwd &f,
                                             uint16_t *hT0, uint16_t *hT1, uint16_t *hT2, int r0) {
  const int lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
  float acc[8][4];
  uint32_t a[4][4];
  // layer 0: K = 16 (4 inputs, zero padded)
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const float b0 = bs[8 * nt + 2 * tig], b1 = bs[8 * nt + 2 * tig + 1];
    acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
    const int n = 8 * nt + g;
    mma16816(acc[nt], ax, ld2(Ws + PW0 + n * S16 + 2 * tig), ld2(Ws + PW0 + n * S16 + 8 + 2 * tig));
  }
#pragma unroll
  for (int layer = 0; layer < 3; ++layer) {
    uint16_t *hT = layer == 0 ? hT0 : layer == 1 ? hT1 : hT2;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      float h[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        h[c] = gelu_f(acc[nt][c]);
        if (TRAIN) f.gp[layer][nt][c] = gelu_d(acc[nt][c]);
      }
      const int s = nt >> 1, hi = nt & 1;
      a[s][hi ? 2 : 0] = pk2(h[0], h[1]);
      a[s][hi ? 3 : 1] = pk2(h[2], h[3]);
      if (TRAIN) {
        const int n = 8 * nt + 2 * tig;
        hT[n * S64 + r0 + g] = bf(h[0]);
        hT[(n + 1) * S64 + r0 + g] = bf(h[1]);
        hT[n * S64 + r0 + g + 8] = bf(h[2]);
        hT[(n + 1) * S64 + r0 + g + 8] = bf(h[3]);
      }
    }
    if (layer < 2) {
      const uint16_t *Wl = Ws + (layer == 0 ? PW1 : PW2);
      const float *bl = bs + 64 * (layer + 1);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const float b0 = bl[8 * nt + 2 * tig], b1 = bl[8 * nt + 2 * tig + 1];
        acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
        const int n = 8 * nt + g;
#pragma unroll
        for (int s = 0; s < 4; ++s)
          mma16816(acc[nt], a[s], ld2(Wl + n * S64 + 16 * s + 2 * tig), ld2(Wl + n * S64 + 16 * s + 8 + 2 * tig));
      }
    }
  }
  // output layer: N = 8 (2 outputs, zero padded)
  {
    const float b0 = bs[192 + 2 * tig], b1 = bs[192 + 2 * tig + 1];
    f.y[0] = b0; f.y[1] = b1; f.y[2] = b0; f.y[3] = b1;
#pragma unroll
    for (int s = 0; s < 4; ++s)
      mma16816(f.y, a[s], ld2(Ws + PW3 + g * S64 + 16 * s + 2 * tig), ld2(Ws + PW3 + g * S64 + 16 * s + 8 + 2 * tig));
  }
}

// A fragment of the network input for rows (g, g+8) of a 16-row warp tile
__device__ __forceinline__ void input_frag(const float *xg, const float *xg8, uint32_t (&ax)[4]) {
  const int tig = threadIdx.x & 3;
  ax[0] = ax[1] = ax[2] = ax[3] = 0u;
  if (tig < 2) {
    ax[0] = pk2(xg[2 * tig], xg[2 * tig + 1]);
    ax[1] = pk2(xg8[2 * tig], xg8[2 * tig + 1]);
  }
}

__device__ __forceinline__ void load_forward_weights(const uint16_t *pack, const float *bias, uint16_t *Ws,
                                                     float *bs) {
  for (int q = threadIdx.x; q < FWDN / 2; q += blockDim.x)
    reinterpret_cast<uint32_t *>(Ws)[q] = reinterpret_cast<const uint32_t *>(pack)[q];
  for (int q = threadIdx.x; q < BIASN; q += blockDim.x) bs[q] = bias[q];
}

// ---------------------------------------------------------------------------
// inference: Y[r][2] = net(X[r][4])
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_mlp_forward(const uint16_t *__restrict__ pack, const float *__restrict__ bias,
                                                     const float *__restrict__ X, float *__restrict__ Y, int rows) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint16_t *Ws = reinterpret_cast<uint16_t *>(smem_raw);
  float *bs = reinterpret_cast<float *>(Ws + FWDN);
  load_forward_weights(pack, bias, Ws, bs);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
  const int ntiles = (rows + 15) / 16;
  for (int t = blockIdx.x * 4 + warp; t < ntiles; t += gridDim.x * 4) {
    const int ra = 16 * t + g, rb = ra + 8;
    float xa[4] = {0.f, 0.f, 0.f, 0.f}, xb[4] = {0.f, 0.f, 0.f, 0.f};
    if (ra < rows)
      for (int e = 0; e < 4; ++e) xa[e] = X[(long long)ra * 4 + e];
    if (rb < rows)
      for (int e = 0; e < 4; ++e) xb[e] = X[(long long)rb * 4 + e];
    uint32_t ax[4];
    input_frag(xa, xb, ax);
    WarpFwd f;
    warp_forward<false>(Ws, bs, ax, f, nullptr, nullptr, nullptr, 0);
    if (tig == 0) {
      if (ra < rows) { Y[(long long)ra * 2] = f.y[0]; Y[(long long)ra * 2 + 1] = f.y[1]; }
      if (rb < rows) { Y[(long long)rb * 2] = f.y[2]; Y[(long long)rb * 2 + 1] = f.y[3]; }
    }
  }
}

// ---------------------------------------------------------------------------
// training pass: loss and gradient of a batch, one partial per CTA
//   batch row j (0..B-1) is sample perm[(off + j) % nsamp]
//   loss = (1/B) sum_j sum_o (y_o - t_o)^2
// part[cta][0..NP-1] = dL/dparams partial, part[cta][NP] = loss partial
// ---------------------------------------------------------------------------
constexpr int TR_ROWS = 64;  // rows of a CTA tile (4 warps x 16)

// dst[m][n] += sum_rows dT[m][row] hT[n][row] for m in the 16-row block at
// mrow0 and n in the 8-column tiles nt0 .. nt0+ntn-1 (m < mvalid, n < nvalid)
__device__ __forceinline__ void dw_gemm_add(const uint16_t *dT, const uint16_t *hT, int mrow0, int nt0, int ntn,
                                            float *dst, int ld_dst, int mvalid, int nvalid) {
  const int lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
  for (int nt = nt0; nt < nt0 + ntn; ++nt) {
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int s = 0; s < TR_ROWS / 16; ++s) {
      uint32_t a[4];
      a[0] = ld2(dT + (mrow0 + g) * S64 + 16 * s + 2 * tig);
      a[1] = ld2(dT + (mrow0 + g + 8) * S64 + 16 * s + 2 * tig);
      a[2] = ld2(dT + (mrow0 + g) * S64 + 16 * s + 8 + 2 * tig);
      a[3] = ld2(dT + (mrow0 + g + 8) * S64 + 16 * s + 8 + 2 * tig);
      const int n = 8 * nt + g;
      mma16816(acc, a, ld2(hT + n * S64 + 16 * s + 2 * tig), ld2(hT + n * S64 + 16 * s + 8 + 2 * tig));
    }
    const int m0 = mrow0 + g, n0 = 8 * nt + 2 * tig;
    if (m0 < mvalid) {
      if (n0 < nvalid) dst[m0 * ld_dst + n0] += acc[0];
      if (n0 + 1 < nvalid) dst[m0 * ld_dst + n0 + 1] += acc[1];
    }
    if (m0 + 8 < mvalid) {
      if (n0 < nvalid) dst[(m0 + 8) * ld_dst + n0] += acc[2];
      if (n0 + 1 < nvalid) dst[(m0 + 8) * ld_dst + n0 + 1] += acc[3];
    }
  }
}

__global__ void __launch_bounds__(128) k_mlp_train(const uint16_t *__restrict__ pack, const float *__restrict__ bias,
                                                   const float *__restrict__ X, const float *__restrict__ Tg,
                                                   const int *__restrict__ perm, int nsamp, const int *__restrict__ offp,
                                                   int B, float *__restrict__ part) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint16_t *Ws = reinterpret_cast<uint16_t *>(smem_raw);  // PACKN
  uint16_t *xT = Ws + PACKN;                              // [16][S64]
  uint16_t *h0T = xT + 16 * S64;                          // [64][S64]
  uint16_t *h1T = h0T + 64 * S64;
  uint16_t *h2T = h1T + 64 * S64;
  uint16_t *d3T = h2T + 64 * S64;  // [16][S64]
  uint16_t *d2T = d3T + 16 * S64;  // [64][S64]
  uint16_t *d1T = d2T + 64 * S64;
  uint16_t *d0T = d1T + 64 * S64;
  float *bs = reinterpret_cast<float *>(d0T + 64 * S64);  // BIASN
  float *dW = bs + BIASN;                                  // NP
  float *lossw = dW + NP;                                  // 4
  const int nbf = PACKN + 2 * 16 * S64 + 6 * 64 * S64;     // bf16 elements above
  for (int q = threadIdx.x; q < PACKN / 2; q += blockDim.x)
    reinterpret_cast<uint32_t *>(Ws)[q] = reinterpret_cast<const uint32_t *>(pack)[q];
  for (int q = PACKN + threadIdx.x; q < nbf; q += blockDim.x) Ws[q] = 0;
  for (int q = threadIdx.x; q < BIASN; q += blockDim.x) bs[q] = bias[q];
  for (int q = threadIdx.x; q < NP; q += blockDim.x) dW[q] = 0.f;
  if (threadIdx.x < 4) lossw[threadIdx.x] = 0.f;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
  const int off = offp ? *offp : 0;
  const float scale = 2.0f / (float)B;
  const int ntiles = (B + TR_ROWS - 1) / TR_ROWS;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int r0 = 16 * warp;                          // warp rows within the tile
    const int ja = t * TR_ROWS + r0 + g, jb = ja + 8;  // batch rows
    float xa[4] = {0.f, 0.f, 0.f, 0.f}, xb[4] = {0.f, 0.f, 0.f, 0.f}, ta[2] = {0.f, 0.f}, tb[2] = {0.f, 0.f};
    const bool va = ja < B, vb = jb < B;
    if (va) {
      const long long s = perm[(off + ja) % nsamp];
      for (int e = 0; e < 4; ++e) xa[e] = X[s * 4 + e];
      ta[0] = Tg[s * 2]; ta[1] = Tg[s * 2 + 1];
    }
    if (vb) {
      const long long s = perm[(off + jb) % nsamp];
      for (int e = 0; e < 4; ++e) xb[e] = X[s * 4 + e];
      tb[0] = Tg[s * 2]; tb[1] = Tg[s * 2 + 1];
    }
    if (tig == 0)
      for (int e = 0; e < 4; ++e) {
        xT[e * S64 + r0 + g] = bf(xa[e]);
        xT[e * S64 + r0 + g + 8] = bf(xb[e]);
      }
    uint32_t ax[4];
    input_frag(xa, xb, ax);
    WarpFwd f;
    warp_forward<true>(Ws, bs, ax, f, h0T, h1T, h2T, r0);
    // output error (tig 0 lanes hold the two outputs of rows g and g+8)
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    float l = 0.f;
    if (tig == 0) {
      if (va) {
        const float e0 = f.y[0] - ta[0], e1 = f.y[1] - ta[1];
        d[0] = scale * e0; d[1] = scale * e1;
        l += e0 * e0 + e1 * e1;
      }
      if (vb) {
        const float e0 = f.y[2] - tb[0], e1 = f.y[3] - tb[1];
        d[2] = scale * e0; d[3] = scale * e1;
        l += e0 * e0 + e1 * e1;
      }
      d3T[0 * S64 + r0 + g] = bf(d[0]);
      d3T[1 * S64 + r0 + g] = bf(d[1]);
      d3T[0 * S64 + r0 + g + 8] = bf(d[2]);
      d3T[1 * S64 + r0 + g + 8] = bf(d[3]);
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if (lane == 0) lossw[warp] += l;
    // back-propagation through the hidden layers (registers only)
    uint32_t a[4][4];
    a[0][0] = pk2(d[0], d[1]);
    a[0][1] = pk2(d[2], d[3]);
    a[0][2] = a[0][3] = 0u;
    float e[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {  // e2 = delta3 W3  (K = 16: outputs 0..1)
      e[nt][0] = e[nt][1] = e[nt][2] = e[nt][3] = 0.f;
      const int n = 8 * nt + g;
      mma16816(e[nt], a[0], ld2(Ws + PT3 + n * S16 + 2 * tig), ld2(Ws + PT3 + n * S16 + 8 + 2 * tig));
    }
#pragma unroll
    for (int layer = 2; layer >= 0; --layer) {
      uint16_t *dT = layer == 2 ? d2T : layer == 1 ? d1T : d0T;
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        float dl[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) dl[c] = e[nt][c] * f.gp[layer][nt][c];
        const int s = nt >> 1, hi = nt & 1;
        a[s][hi ? 2 : 0] = pk2(dl[0], dl[1]);
        a[s][hi ? 3 : 1] = pk2(dl[2], dl[3]);
        const int n = 8 * nt + 2 * tig;
        dT[n * S64 + r0 + g] = bf(dl[0]);
        dT[(n + 1) * S64 + r0 + g] = bf(dl[1]);
        dT[n * S64 + r0 + g + 8] = bf(dl[2]);
        dT[(n + 1) * S64 + r0 + g + 8] = bf(dl[3]);
      }
      if (layer > 0) {  // e_{layer-1} = delta_layer W_layer
        const uint16_t *WT = Ws + (layer == 2 ? PT2 : PT1);
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
          e[nt][0] = e[nt][1] = e[nt][2] = e[nt][3] = 0.f;
          const int n = 8 * nt + g;
#pragma unroll
          for (int s = 0; s < 4; ++s)
            mma16816(e[nt], a[s], ld2(WT + n * S64 + 16 * s + 2 * tig), ld2(WT + n * S64 + 16 * s + 8 + 2 * tig));
        }
      }
    }
    __syncthreads();
    // weight gradients over the 64 rows of the tile; warp w owns output rows 16w..16w+15
    dw_gemm_add(d2T, h1T, 16 * warp, 0, 8, dW + OW2, NH, 64, 64);
    dw_gemm_add(d1T, h0T, 16 * warp, 0, 8, dW + OW1, NH, 64, 64);
    dw_gemm_add(d0T, xT, 16 * warp, 0, 1, dW + OW0, NIN, 64, NIN);
    dw_gemm_add(d3T, h2T, 0, 2 * warp, 2, dW + OW3, NH, NOUT, 64);
    // bias gradients from the same BF16 errors
    {
      const int o = threadIdx.x & 63;
      const uint16_t *src = threadIdx.x < 64 ? d0T : d1T;
      float s0 = 0.f;
      for (int r = 0; r < TR_ROWS; ++r) s0 += unbf(src[o * S64 + r]);
      dW[(threadIdx.x < 64 ? OB0 : OB1) + o] += s0;
      const uint16_t *src2 = threadIdx.x < 64 ? d2T : d3T;
      if (threadIdx.x < 64 || o < NOUT) {
        float s1 = 0.f;
        for (int r = 0; r < TR_ROWS; ++r) s1 += unbf(src2[o * S64 + r]);
        dW[(threadIdx.x < 64 ? OB2 : OB3) + o] += s1;
      }
    }
    __syncthreads();
  }
  float *out = part + (long long)blockIdx.x * (NP + 1);
  for (int q = threadIdx.x; q < NP; q += blockDim.x) out[q] = dW[q];
  if (threadIdx.x == 0) out[NP] = (lossw[0] + lossw[1] + lossw[2] + lossw[3]) / (float)B;
}

// sum of the CTA partials in CTA order; grad may be null (then only the loss)
__global__ void k_mlp_reduce(const float *__restrict__ part, int nparts, float *__restrict__ grad,
                             float *__restrict__ loss) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= NP; p += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int c = 0; c < nparts; ++c) s += part[(long long)c * (NP + 1) + p];
    if (p < NP) {
      if (grad) grad[p] = s;
    } else if (loss) {
      *loss = s;
    }
  }
}

// Adam (Kingma & Ba, 2015) on the FP32 master parameters, then the BF16
// repack.  st[0] = step count, st[1] = batch offset (int bits), st[2] = last
// batch loss; loss_hist is a ring of hist_n entries indexed by the step.
__global__ void k_mlp_adam(const float *__restrict__ part, int nparts, float *__restrict__ params,
                           float *__restrict__ m1, float *__restrict__ m2, float *__restrict__ st, float lr,
                           float *__restrict__ loss_hist, int hist_n, uint16_t *__restrict__ pack,
                           float *__restrict__ bias) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float tstep = st[0] + 1.0f;
  const float c1 = 1.0f - powf(b1, tstep), c2 = 1.0f - powf(b2, tstep);
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= NP; p += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int c = 0; c < nparts; ++c) s += part[(long long)c * (NP + 1) + p];
    if (p == NP) {
      if (loss_hist && hist_n > 0) loss_hist[(int)st[0] % hist_n] = s;
      st[2] = s;
      continue;
    }
    const float mm = b1 * m1[p] + (1.0f - b1) * s;
    const float vv = b2 * m2[p] + (1.0f - b2) * s * s;
    m1[p] = mm;
    m2[p] = vv;
    const float w = params[p] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    params[p] = w;
    pack_param(p, w, pack, bias);
  }
}

__global__ void k_mlp_advance(float *__restrict__ st, int B, int nsamp) {
  st[0] += 1.0f;
  int *off = reinterpret_cast<int *>(st + 1);
  *off = (int)(((long long)*off + B) % nsamp);
}

// ---------------------------------------------------------------------------
// wall samples and the wall-model hook
// ---------------------------------------------------------------------------
// Features at wall point (i,k), i = 2..nx-1, k = 2..nzg-2, from the row jh
// (height h = yg(jh)): u = U(i,jh,k); w = W averaged to the U point;
// ln(h |u| / nu) / 10; 100 h dP/dx.  Stress targets (x1000) from the wall
// gradient nu (F(2) - F(1)) / (yg(2) - yg(1)) of U and of the averaged W.
template <typename T>
__device__ __forceinline__ double w_at_u(const Geo &g, const T *W, int i, int j, int k) {
  return 0.25 * ((double)W[bidx(g, i, j, k)] + (double)W[bidx(g, i + 1, j, k)] + (double)W[bidx(g, i, j, k - 1)] +
                 (double)W[bidx(g, i + 1, j, k - 1)]);
}

template <typename T>
__device__ __forceinline__ void wall_features(const Geo &g, const T *U, const T *W, const T *P, int i, int jh, int k,
                                              float (&x)[4]) {
  const double h = g.yg[jh];
  const double u = (double)U[bidx(g, i, jh, k)];
  const double w = w_at_u<T>(g, W, i, jh, k);
  const double dp = ((double)P[bidx(g, i + 1, jh, k)] - (double)P[bidx(g, i, jh, k)]) / (g.xg[i + 1] - g.xg[i]);
  x[0] = (float)u;
  x[1] = (float)w;
  x[2] = (float)(log(fmax(h * fabs(u) / g.nu, 1.0)) / 10.0);
  x[3] = (float)(100.0 * h * dp);
}

// viscosity of the U-equation's wall flux at (i,k): nu_y1 of the LES branch
// (equations.f90:97-98) at j = 2, or nu alone without an eddy viscosity
template <typename T>
__device__ __forceinline__ double wall_flux_nu(const Geo &g, const T *nut, int i, int k) {
  if (!nut) return g.nu;
  return g.nu + 0.5 * (g.w0[1] * (double)nut[bidx(g, i, 1, k)] + g.w1[1] * (double)nut[bidx(g, i, 2, k)] +
                       g.w0[1] * (double)nut[bidx(g, i + 1, 1, k)] + g.w1[1] * (double)nut[bidx(g, i + 1, 2, k)]);
}

template <typename T>
__global__ void k_wall_samples(Geo g, const T *__restrict__ U, const T *__restrict__ W, const T *__restrict__ P,
                               int jh, float *__restrict__ X, float *__restrict__ Tg) {
  const int ni = g.nx - 2, nk = g.nzg - 3;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= ni * nk) return;
  const int i = r % ni + 2, k = r / ni + 2;
  float x[4];
  wall_features<T>(g, U, W, P, i, jh, k, x);
  for (int e = 0; e < 4; ++e) X[(long long)r * 4 + e] = x[e];
  const double dy = g.yg[2] - g.yg[1];
  const double tx = g.nu * ((double)U[bidx(g, i, 2, k)] - (double)U[bidx(g, i, 1, k)]) / dy;
  const double tz = g.nu * (w_at_u<T>(g, W, i, 2, k) - w_at_u<T>(g, W, i, 1, k)) / dy;
  Tg[(long long)r * 2] = (float)(1000.0 * tx);
  Tg[(long long)r * 2 + 1] = (float)(1000.0 * tz);
}

// network stress at every wall point -> alpha = tau / nu_wall (the slope of
// the non-zero Neumann condition).  wm holds four arrays of nw = (nx-2)(nzg-3)
// values, index (k-2)(nx-2) + (i-2): alpha_x, alpha_z, tau_x, tau_z.
template <typename T>
__global__ void __launch_bounds__(128) k_wall_mlp(Geo g, MlpDev net, const T *__restrict__ U,
                                                  const T *__restrict__ W, const T *__restrict__ P,
                                                  const T *__restrict__ nut, int jh, double *__restrict__ wm) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint16_t *Ws = reinterpret_cast<uint16_t *>(smem_raw);
  float *bs = reinterpret_cast<float *>(Ws + FWDN);
  load_forward_weights(net.pack, net.bias, Ws, bs);
  __syncthreads();
  const int ni = g.nx - 2, nk = g.nzg - 3, rows = ni * nk;
  double *ax = wm, *az = wm + rows, *tx = wm + 2 * (long long)rows, *tz = wm + 3 * (long long)rows;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, gg = lane >> 2, tig = lane & 3;
  const int ntiles = (rows + 15) / 16;
  for (int t = blockIdx.x * 4 + warp; t < ntiles; t += gridDim.x * 4) {
    const int ra = 16 * t + gg, rb = ra + 8;
    float xa[4] = {0.f, 0.f, 0.f, 0.f}, xb[4] = {0.f, 0.f, 0.f, 0.f};
    if (ra < rows) wall_features<T>(g, U, W, P, ra % ni + 2, jh, ra / ni + 2, xa);
    if (rb < rows) wall_features<T>(g, U, W, P, rb % ni + 2, jh, rb / ni + 2, xb);
    uint32_t axf[4];
    input_frag(xa, xb, axf);
    WarpFwd f;
    warp_forward<false>(Ws, bs, axf, f, nullptr, nullptr, nullptr, 0);
    if (tig == 0) {
      if (ra < rows) {
        const double nw = wall_flux_nu<T>(g, nut, ra % ni + 2, ra / ni + 2);
        tx[ra] = 1e-3 * (double)f.y[0];
        tz[ra] = 1e-3 * (double)f.y[1];
        ax[ra] = tx[ra] / nw;
        az[ra] = tz[ra] / nw;
      }
      if (rb < rows) {
        const double nw = wall_flux_nu<T>(g, nut, rb % ni + 2, rb / ni + 2);
        tx[rb] = 1e-3 * (double)f.y[2];
        tz[rb] = 1e-3 * (double)f.y[3];
        ax[rb] = tx[rb] / nw;
        az[rb] = tz[rb] / nw;
      }
    }
  }
}

// equilibrium stress u_tau(i)^2 (law of the wall), z-uniform, W no-slip
template <typename T>
__global__ void k_wall_eq(Geo g, const double *__restrict__ utau, const T *__restrict__ nut, double *__restrict__ wm) {
  const int ni = g.nx - 2, nk = g.nzg - 3, nw = ni * nk;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nw) return;
  const int i = r % ni + 2, k = r / ni + 2;
  const double u = utau[i - 1];
  wm[r] = u * u / wall_flux_nu<T>(g, nut, i, k);
  wm[nw + r] = 0.0;
  wm[2 * (long long)nw + r] = u * u;
  wm[3 * (long long)nw + r] = 0.0;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
size_t mlp_train_smem() {
  return (size_t)(PACKN + 2 * 16 * S64 + 6 * 64 * S64) * 2 + (size_t)(BIASN + NP + 4) * 4;
}
size_t mlp_fwd_smem() { return (size_t)FWDN * 2 + (size_t)BIASN * 4; }

void launch_mlp_pack(const float *params, uint16_t *pack, float *bias, cudaStream_t st) {
  k_mlp_clear<<<64, 256, 0, st>>>(pack, bias);
  k_mlp_pack<<<(NP + 255) / 256, 256, 0, st>>>(params, pack, bias);
}

void launch_mlp_forward(const uint16_t *pack, const float *bias, const float *X, float *Y, int rows, cudaStream_t st) {
  const size_t sm = mlp_fwd_smem();
  cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  const int ntiles = (rows + 15) / 16;
  int grid = (ntiles + 3) / 4;
  if (grid > 148 * 4) grid = 148 * 4;
  if (grid < 1) grid = 1;
  k_mlp_forward<<<grid, 128, sm, st>>>(pack, bias, X, Y, rows);
}

int mlp_train_ctas(int B) {
  int n = (B + TR_ROWS - 1) / TR_ROWS;
  return n < 148 ? (n < 1 ? 1 : n) : 148;
}

void launch_mlp_grad(const uint16_t *pack, const float *bias, const float *X, const float *Tg, const int *perm,
                     int nsamp, const int *offp, int B, float *part, cudaStream_t st) {
  const size_t sm = mlp_train_smem();
  cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_mlp_train<<<mlp_train_ctas(B), 128, sm, st>>>(pack, bias, X, Tg, perm, nsamp, offp, B, part);
}

void launch_mlp_reduce(const float *part, int nparts, float *grad, float *loss, cudaStream_t st) {
  k_mlp_reduce<<<(NP + 1 + 255) / 256, 256, 0, st>>>(part, nparts, grad, loss);
}

void launch_mlp_adam(const float *part, int nparts, float *params, float *m1, float *m2, float *stv, float lr, int B,
                     int nsamp, float *loss_hist, int hist_n, uint16_t *pack, float *bias, cudaStream_t st) {
  k_mlp_adam<<<(NP + 1 + 255) / 256, 256, 0, st>>>(part, nparts, params, m1, m2, stv, lr, loss_hist, hist_n, pack,
                                                   bias);
  k_mlp_advance<<<1, 1, 0, st>>>(stv, B, nsamp);
}

template <typename T>
void launch_wall_samples(const Geo &g, const T *U, const T *W, const T *P, int jh, float *X, float *Tg,
                         cudaStream_t st) {
  const int rows = (g.nx - 2) * (g.nzg - 3);
  k_wall_samples<T><<<(rows + 255) / 256, 256, 0, st>>>(g, U, W, P, jh, X, Tg);
}

template <typename T>
void launch_wall_mlp(const Geo &g, const MlpDev &net, const T *U, const T *W, const T *P, const T *nut, int jh,
                     double *wm, cudaStream_t st) {
  const size_t sm = mlp_fwd_smem();
  cudaFuncSetAttribute(k_wall_mlp<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  const int rows = (g.nx - 2) * (g.nzg - 3);
  int grid = ((rows + 15) / 16 + 3) / 4;
  if (grid > 148 * 4) grid = 148 * 4;
  k_wall_mlp<T><<<grid, 128, sm, st>>>(g, net, U, W, P, nut, jh, wm);
}

template <typename T>
void launch_wall_eq(const Geo &g, const double *utau, const T *nut, double *wm, cudaStream_t st) {
  const int rows = (g.nx - 2) * (g.nzg - 3);
  k_wall_eq<T><<<(rows + 255) / 256, 256, 0, st>>>(g, utau, nut, wm);
}

#define BLGPU_MLP_INST(T)                                                                                         \
  template void launch_wall_samples<T>(const Geo &, const T *, const T *, const T *, int, float *, float *,       \
                                       cudaStream_t);                                                             \
  template void launch_wall_mlp<T>(const Geo &, const MlpDev &, const T *, const T *, const T *, const T *, int,  \
                                   double *, cudaStream_t);                                                       \
  template void launch_wall_eq<T>(const Geo &, const double *, const T *, double *, cudaStream_t);
BLGPU_MLP_INST(double)
BLGPU_MLP_INST(float)

}  // namespace blgpu
