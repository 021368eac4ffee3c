// spectral.cu -- the Poisson solve of the fractional-step projection.
//
// The reference (projection.f90:93-204) packs rhs_p into a 2N symmetric
// extension, runs cuFFT Z2Z transforms over GB-sized complex workspaces and
// a Thomas sweep over 1.27 GB of precomputed complex factors.  Here the same
// operator -- DCT-II in x (Neumann), DFT in z (periodic), tridiagonal solve
// in y per (kx,kz) mode -- is computed with
//   k_div_dct   divergence (projection.f90:38-47) fused with a real DCT-II in
//               x: two real lines packed into one complex line, Makhoul's
//               N-point reordering, a Stockham mixed-radix FFT in shared
//               memory, untangle + DCT twiddle in the epilogue;
//   k_dft_z     real DFT in z over the half spectrum (kz = 0..M/2), direct
//               summation with the f_k +- f_{M-k} pairing;
//   k_thomas    tridiagonal solve in y with the factors formed on the fly
//               from Dyy, kxx and kzz (initialization.f90:395-469);
//   k_dft_z<inverse>, k_idct  the inverse transforms, the last one writing
//               rhs_p in the box layout together with the x-Neumann and
//               z-periodic copies of apply_periodic_z_pressure
//               (projection.f90:295-303).
#include "kernels.cuh"
#include "divergence.cuh"
#include "tma.cuh"

namespace blgpu {

template <typename T> using T2 = typename vec2<T>::type;

template <typename T> __device__ __forceinline__ T2<T> mk(T a, T b) { T2<T> r; r.x = a; r.y = b; return r; }
template <typename T> __device__ __forceinline__ T2<T> add(T2<T> a, T2<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T> __device__ __forceinline__ T2<T> sub(T2<T> a, T2<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }
template <typename T> __device__ __forceinline__ T2<T> cmul(T2<T> a, T2<T> b) {
  return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T> __device__ __forceinline__ T2<T> cmulc(T2<T> a, T2<T> b) {  // a * conj(b)
  return mk<T>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename T, bool INV> __device__ __forceinline__ T2<T> twm(T2<T> a, T2<T> w) {
  return INV ? cmulc<T>(a, w) : cmul<T>(a, w);
}

// ---------------------------------------------------------------------------
// Stockham butterflies.  Stage with radix R, current span Ns: butterfly jj of
// a line reads in[jj + r*n/R], applies W_n^{r*tstep} (tstep = (jj mod Ns) *
// n/(Ns*R)), does an R-point DFT and writes out[idxD + r*Ns] with
// idxD = (jj/Ns)*Ns*R + jj mod Ns.
// ---------------------------------------------------------------------------
template <typename T, bool INV>
__device__ __forceinline__ void bf2(const T2<T> *in, T2<T> *out, int jj, int nb, int tstep, int idxD, int Ns,
                                    const T2<T> *tw) {
  T2<T> a = in[jj], b = in[jj + nb];
  if (tstep) b = twm<T, INV>(b, tw[tstep]);
  out[idxD] = add<T>(a, b);
  out[idxD + Ns] = sub<T>(a, b);
}

template <typename T, bool INV>
__device__ __forceinline__ void bf4(const T2<T> *in, T2<T> *out, int jj, int nb, int tstep, int idxD, int Ns,
                                    const T2<T> *tw) {
  T2<T> a0 = in[jj], a1 = in[jj + nb], a2 = in[jj + 2 * nb], a3 = in[jj + 3 * nb];
  if (tstep) {
    a1 = twm<T, INV>(a1, tw[tstep]);
    a2 = twm<T, INV>(a2, tw[2 * tstep]);
    a3 = twm<T, INV>(a3, tw[3 * tstep]);
  }
  T2<T> s0 = add<T>(a0, a2), s1 = sub<T>(a0, a2), s2 = add<T>(a1, a3), s3 = sub<T>(a1, a3);
  // forward: -i*s3 ; inverse: +i*s3
  T2<T> r3 = INV ? mk<T>(-s3.y, s3.x) : mk<T>(s3.y, -s3.x);
  out[idxD] = add<T>(s0, s2);
  out[idxD + Ns] = add<T>(s1, r3);
  out[idxD + 2 * Ns] = sub<T>(s0, s2);
  out[idxD + 3 * Ns] = sub<T>(s1, r3);
}

template <typename T, bool INV>
__device__ __forceinline__ void bf3(const T2<T> *in, T2<T> *out, int jj, int nb, int tstep, int idxD, int Ns,
                                    const T2<T> *tw) {
  T2<T> a0 = in[jj], a1 = in[jj + nb], a2 = in[jj + 2 * nb];
  if (tstep) {
    a1 = twm<T, INV>(a1, tw[tstep]);
    a2 = twm<T, INV>(a2, tw[2 * tstep]);
  }
  const T s60 = (T)0.86602540378443864676;  // sin(2 pi / 3)
  T2<T> t1 = add<T>(a1, a2), t2 = sub<T>(a1, a2);
  T2<T> m = mk<T>(a0.x - (T)0.5 * t1.x, a0.y - (T)0.5 * t1.y);
  // forward y1 = m - i s t2, y2 = m + i s t2
  T2<T> it = INV ? mk<T>(-s60 * t2.y, s60 * t2.x) : mk<T>(s60 * t2.y, -s60 * t2.x);
  out[idxD] = add<T>(a0, t1);
  out[idxD + Ns] = add<T>(m, it);
  out[idxD + 2 * Ns] = sub<T>(m, it);
}

// R-point DFT constants (cos, sin)(2 pi m / R), m = 0..R-1, of the odd
// register radices, in constant memory so that the butterflies take them as
// instruction operands instead of holding them in registers
constexpr int DFT_RSUM = 5 + 7 + 11 + 13 + 17 + 19 + 23 + 29 + 31;
__constant__ double2 c_dft64[DFT_RSUM];
__constant__ float2 c_dft32[DFT_RSUM];
template <int R> __host__ __device__ constexpr int dft_off() {
  return R == 5 ? 0 : R == 7 ? 5 : R == 11 ? 12 : R == 13 ? 23 : R == 17 ? 36 : R == 19 ? 53 : R == 23 ? 72
       : R == 29 ? 95 : 124;
}
template <typename T> __device__ __forceinline__ const T2<T> *dft_consts();
template <> __device__ __forceinline__ const double2 *dft_consts<double>() { return c_dft64; }
template <> __device__ __forceinline__ const float2 *dft_consts<float>() { return c_dft32; }

// (cos, sin)(2 pi e / R) for R = 2..32, e = 0..R-1, R's entries from
// root_off<R>(): the constants of the in-register DFTs of the two-pass FFT
constexpr int ROOTS_N = 33 * 32 / 2 - 1;
__constant__ float2 c_roots32[ROOTS_N];
__constant__ double2 c_roots64[ROOTS_N];
template <int R> __host__ __device__ constexpr int root_off() { return R * (R - 1) / 2 - 1; }
template <typename V> __device__ __forceinline__ const V *roots();
template <> __device__ __forceinline__ const float2 *roots<float2>() { return c_roots32; }
template <> __device__ __forceinline__ const double2 *roots<double2>() { return c_roots64; }

int upload_dft_constants() {
  {
    float2 h[ROOTS_N];
    double2 hd[ROOTS_N];
    for (int R = 2; R <= 32; ++R)
      for (int e = 0; e < R; ++e) {
        const double a = 2.0 * M_PI * (double)e / (double)R;
        h[R * (R - 1) / 2 - 1 + e] = make_float2((float)cos(a), (float)sin(a));
        hd[R * (R - 1) / 2 - 1 + e] = make_double2(cos(a), sin(a));
      }
    if (cudaMemcpyToSymbol(c_roots32, h, sizeof h) != cudaSuccess) return -1;
    if (cudaMemcpyToSymbol(c_roots64, hd, sizeof hd) != cudaSuccess) return -1;
  }
  const int rad[9] = {5, 7, 11, 13, 17, 19, 23, 29, 31};
  double2 h64[DFT_RSUM];
  float2 h32[DFT_RSUM];
  int o = 0;
  for (int r : rad)
    for (int m = 0; m < r; ++m, ++o) {
      const double a = 2.0 * M_PI * (double)m / (double)r;
      h64[o] = make_double2(cos(a), sin(a));
      h32[o] = make_float2((float)cos(a), (float)sin(a));
    }
  if (cudaMemcpyToSymbol(c_dft64, h64, sizeof h64) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(c_dft32, h32, sizeof h32) != cudaSuccess) return -1;
  return 0;
}

// odd radix R (5..31) in registers, pairing inputs q and R-q
template <int R, typename T, bool INV>
__device__ __forceinline__ void bf_odd(const T2<T> *in, T2<T> *out, int jj, int nb, int tstep, int idxD, int Ns,
                                       int n, const T2<T> *tw) {
  constexpr int H = (R - 1) / 2;
  const int stride = n / R;
  const T2<T> x0 = in[jj];
  T2<T> s[H], d[H];
#pragma unroll
  for (int q = 1; q <= H; ++q) {
    T2<T> a = in[jj + q * nb], b = in[jj + (R - q) * nb];
    if (tstep) {
      a = twm<T, INV>(a, tw[q * tstep]);
      b = twm<T, INV>(b, tw[(R - q) * tstep]);
    }
    s[q - 1] = add<T>(a, b);
    d[q - 1] = sub<T>(a, b);
  }
  // (cos, sin)(2 pi m / R): FP32 reads them from constant memory as operands;
  // FP64 keeps the half table in registers (taken from the twiddles)
  const T2<T> *K = dft_consts<T>() + dft_off<R>();
  T cs[H], sn[H];
  if constexpr (sizeof(T) == 8) {
#pragma unroll
    for (int q = 1; q <= H; ++q) {
      const T2<T> w = tw[q * stride];
      cs[q - 1] = w.x;
      sn[q - 1] = -w.y;  // sin(2 pi q / R)
    }
  }
  T2<T> y0 = x0;
#pragma unroll
  for (int q = 0; q < H; ++q) y0 = add<T>(y0, s[q]);
  out[idxD] = y0;
#pragma unroll
  for (int k = 1; k <= H; ++k) {
    T ax = x0.x, ay = x0.y, bx = 0, by = 0;
#pragma unroll
    for (int q = 1; q <= H; ++q) {
      const int m = (q * k) % R;
      T c, sv;
      if constexpr (sizeof(T) == 4) {
        c = K[m].x;
        sv = K[m].y;
      } else {
        c = (m <= H) ? cs[m - 1] : cs[R - m - 1];
        sv = (m <= H) ? sn[m - 1] : -sn[R - m - 1];
      }
      ax += s[q - 1].x * c;
      ay += s[q - 1].y * c;
      bx += d[q - 1].x * sv;
      by += d[q - 1].y * sv;
    }
    T2<T> yk, ynk;
    if (!INV) { yk = mk<T>(ax + by, ay - bx); ynk = mk<T>(ax - by, ay + bx); }
    else { yk = mk<T>(ax - by, ay + bx); ynk = mk<T>(ax + by, ay - bx); }
    out[idxD + k * Ns] = yk;
    out[idxD + (R - k) * Ns] = ynk;
  }
}

// radices with a dedicated butterfly in the kernel instantiated for MAXR
template <int MAXR>
__device__ __forceinline__ bool reg_radix(int R) {
  if (R == 2 || R == 3 || R == 4) return true;
  if (R > MAXR) return false;
  return R == 5 || R == 7 || R == 11 || R == 13 || R == 17 || R == 19 || R == 23 || R == 29 || R == 31;
}

// warp-level Stockham FFT of one complex line in shared memory (no block
// barriers: each warp owns its line, stages are separated by __syncwarp)
template <typename T, bool INV, int MAXR>
__device__ __forceinline__ T2<T> *fft_warp(T2<T> *a, T2<T> *b, const FftPlan<T> &pl, const T2<T> *tw, int lane) {
  const int n = pl.n;
  int Ns = 1;
  for (int s = 0; s < pl.nst; ++s) {
    const int R = pl.rad[s];
    const int nb = n / R;
    const int tsc = n / (Ns * R);
    if (!reg_radix<MAXR>(R)) {
      // a large prime R has few butterflies (nb = n/R), so the lanes take
      // (butterfly, term pair) and (butterfly, output pair) items.  First the
      // inputs of butterfly jj are twiddled (y_q = in_q W_n^{q tstep}) and
      // folded in place: a[jj + q nb] <- s_q = y_q + y_{R-q},
      // a[jj + (R-q) nb] <- d_q = y_q - y_{R-q}, q = 1 .. H (the stage's
      // input is dead after it).  Then X_0 = y_0 + sum s_q and, for k = 1..H,
      //   X_k, X_{R-k} = y_0 + sum_q s_q cos(2 pi qk/R) -+ i sum_q d_q sin(2 pi qk/R)
      // (signs swapped for the inverse): H terms for two outputs instead of
      // R terms for one.
      const int H = (R - 1) / 2;
      for (int t = lane; t < nb * H; t += 32) {
        const int jj = t % nb, q = 1 + t / nb;
        const int tstep = (jj % Ns) * tsc;
        T2<T> y1 = a[jj + q * nb], y2 = a[jj + (R - q) * nb];
        if (tstep) {
          y1 = twm<T, INV>(y1, tw[q * tstep]);
          y2 = twm<T, INV>(y2, tw[(R - q) * tstep]);
        }
        a[jj + q * nb] = add<T>(y1, y2);
        a[jj + (R - q) * nb] = sub<T>(y1, y2);
      }
      __syncwarp();
      for (int t = lane; t < nb * (H + 1); t += 32) {
        const int jj = t % nb, k = t / nb;
        const int jm = jj % Ns;
        const int idxD = (jj - jm) * R + jm;
        const T2<T> y0 = a[jj];
        T ax = y0.x, ay = y0.y;
        if (k == 0) {
          for (int q = 1; q <= H; ++q) {
            const T2<T> sq = a[jj + q * nb];
            ax += sq.x;
            ay += sq.y;
          }
          b[idxD] = mk<T>(ax, ay);
          continue;
        }
        T bx = 0, by = 0;  // sums of d_q times the table's imaginary part (-sin)
        int m = 0;         // q k mod R
        for (int q = 1; q <= H; ++q) {
          m += k;
          if (m >= R) m -= R;
          const T2<T> w = tw[m * nb];  // W_R^m = (cos, -sin)(2 pi m / R)
          const T2<T> sq = a[jj + q * nb], dq = a[jj + (R - q) * nb];
          ax += sq.x * w.x;
          ay += sq.y * w.x;
          bx += dq.x * w.y;
          by += dq.y * w.y;
        }
        if (!INV) {
          b[idxD + k * Ns] = mk<T>(ax - by, ay + bx);
          b[idxD + (R - k) * Ns] = mk<T>(ax + by, ay - bx);
        } else {
          b[idxD + k * Ns] = mk<T>(ax + by, ay - bx);
          b[idxD + (R - k) * Ns] = mk<T>(ax - by, ay + bx);
        }
      }
      __syncwarp();
      T2<T> *t = a;
      a = b;
      b = t;
      Ns *= R;
      continue;
    }
    for (int jj = lane; jj < nb; jj += 32) {
      const int jm = jj % Ns;
      const int tstep = jm * tsc;
      const int idxD = (jj - jm) * R + jm;
      if (R == 4) bf4<T, INV>(a, b, jj, nb, tstep, idxD, Ns, tw);
      else if (R == 2) bf2<T, INV>(a, b, jj, nb, tstep, idxD, Ns, tw);
      else if (R == 3) bf3<T, INV>(a, b, jj, nb, tstep, idxD, Ns, tw);
      else if (MAXR >= 5 && R == 5) bf_odd<5, T, INV>(a, b, jj, nb, tstep, idxD, Ns, n, tw);
      else if (MAXR >= 7 && R == 7) bf_odd<7, T, INV>(a, b, jj, nb, tstep, idxD, Ns, n, tw);
      else if (MAXR >= 11 && R == 11) bf_odd<11, T, INV>(a, b, jj, nb, tstep, idxD, Ns, n, tw);
      else if (MAXR >= 13 && R == 13) bf_odd<13, T, INV>(a, b, jj, nb, tstep, idxD, Ns, n, tw);
      else if (MAXR >= 17 && R == 17) bf_odd<17, T, INV>(a, b, jj, nb, tstep, idxD, Ns, n, tw);
      else if (MAXR >= 19 && R == 19) bf_odd<19, T, INV>(a, b, jj, nb, tstep, idxD, Ns, n, tw);
      else if (MAXR >= 23 && R == 23) bf_odd<23, T, INV>(a, b, jj, nb, tstep, idxD, Ns, n, tw);
      else if (MAXR >= 29 && R == 29) bf_odd<29, T, INV>(a, b, jj, nb, tstep, idxD, Ns, n, tw);
      else if (MAXR >= 31 && R == 31) bf_odd<31, T, INV>(a, b, jj, nb, tstep, idxD, Ns, n, tw);
    }
    __syncwarp();
    T2<T> *t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

// ---------------------------------------------------------------------------
// Two-pass register FFT (FP32) of a line of N = A B complex values, one warp
// per line, every index a compile-time constant.  With n = B n1 + n2 and
// k = k1 + A k2:
//   pass 1 (lane n2 < B): A-point DFT over n1 of z[B n1 + n2] in registers,
//          times W_N^{n2 k1}, into S[k1][n2] (row pitch B | 1, odd, so that
//          the column reads of pass 2 meet distinct banks);
//   pass 2 (lane k1 < A): B-point DFT over n2 of S[k1][n2] in registers,
//          into Z[k1 + A k2].
// Both passes work in place in one buffer (reads, warp barrier, writes).
// The in-register DFTs split composite lengths (radix 4, 2, then the odd
// primes) and take prime lengths >= 5 by the f_q +- f_{R-q} pairing; their
// constants are constant-memory operands.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int first_factor(int R) {
  if (R % 4 == 0 && R != 4) return 4;
  for (int f = 2; f * f <= R; ++f)
    if (R % f == 0) return f;
  return R;
}

template <typename V, typename S> __device__ __forceinline__ V mkv(S a, S b) {
  V r;
  r.x = a;
  r.y = b;
  return r;
}

// a * W_R^e (W_R = exp(-2 pi i / R)), or a * conj(W_R^e) for the inverse
template <int R, bool INV, typename V>
__device__ __forceinline__ V twr(V a, int e) {
  if (e == 0) return a;
  if (2 * e == R) return mkv<V>(-a.x, -a.y);
  if (4 * e == R) return INV ? mkv<V>(-a.y, a.x) : mkv<V>(a.y, -a.x);
  if (4 * e == 3 * R) return INV ? mkv<V>(a.y, -a.x) : mkv<V>(-a.y, a.x);
  const V w = roots<V>()[root_off<R>() + e];  // (cos, sin)
  return INV ? mkv<V>(a.x * w.x - a.y * w.y, a.y * w.x + a.x * w.y)
             : mkv<V>(a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y);
}

template <int R, bool INV, typename V>
__device__ __forceinline__ void dft_reg(V (&x)[R]) {
  typedef decltype(V().x) S;
  if constexpr (R == 2) {
    const V a = x[0], b = x[1];
    x[0] = mkv<V>(a.x + b.x, a.y + b.y);
    x[1] = mkv<V>(a.x - b.x, a.y - b.y);
  } else if constexpr (R == 3) {
    const S s60 = (S)0.86602540378443864676;
    const V a0 = x[0], t1 = mkv<V>(x[1].x + x[2].x, x[1].y + x[2].y);
    const V t2 = mkv<V>(x[1].x - x[2].x, x[1].y - x[2].y);
    const V m = mkv<V>(a0.x - (S)0.5 * t1.x, a0.y - (S)0.5 * t1.y);
    const V it = INV ? mkv<V>(-s60 * t2.y, s60 * t2.x) : mkv<V>(s60 * t2.y, -s60 * t2.x);
    x[0] = mkv<V>(a0.x + t1.x, a0.y + t1.y);
    x[1] = mkv<V>(m.x + it.x, m.y + it.y);
    x[2] = mkv<V>(m.x - it.x, m.y - it.y);
  } else if constexpr (R == 4) {
    const V s0 = mkv<V>(x[0].x + x[2].x, x[0].y + x[2].y), s1 = mkv<V>(x[0].x - x[2].x, x[0].y - x[2].y);
    const V s2 = mkv<V>(x[1].x + x[3].x, x[1].y + x[3].y), s3 = mkv<V>(x[1].x - x[3].x, x[1].y - x[3].y);
    const V r3 = INV ? mkv<V>(-s3.y, s3.x) : mkv<V>(s3.y, -s3.x);  // +-i s3
    x[0] = mkv<V>(s0.x + s2.x, s0.y + s2.y);
    x[1] = mkv<V>(s1.x + r3.x, s1.y + r3.y);
    x[2] = mkv<V>(s0.x - s2.x, s0.y - s2.y);
    x[3] = mkv<V>(s1.x - r3.x, s1.y - r3.y);
  } else if constexpr (first_factor(R) == R) {
    // prime R >= 5: X_k = x_0 + sum_q s_q cos - (+) i d_q sin, s, d = x_q +- x_{R-q}
    constexpr int H = (R - 1) / 2;
    const V x0 = x[0];
    V s[H], d[H];
#pragma unroll
    for (int q = 1; q <= H; ++q) {
      s[q - 1] = mkv<V>(x[q].x + x[R - q].x, x[q].y + x[R - q].y);
      d[q - 1] = mkv<V>(x[q].x - x[R - q].x, x[q].y - x[R - q].y);
    }
    V y0 = x0;
#pragma unroll
    for (int q = 0; q < H; ++q) y0 = mkv<V>(y0.x + s[q].x, y0.y + s[q].y);
    x[0] = y0;
    const V *K = roots<V>() + root_off<R>();
#pragma unroll
    for (int k = 1; k <= H; ++k) {
      S ax = x0.x, ay = x0.y, bx = 0, by = 0;
#pragma unroll
      for (int q = 1; q <= H; ++q) {
        const int m = (q * k) % R;
        const S c = K[m].x, sv = K[m].y;
        ax += s[q - 1].x * c;
        ay += s[q - 1].y * c;
        bx += d[q - 1].x * sv;
        by += d[q - 1].y * sv;
      }
      if (!INV) {
        x[k] = mkv<V>(ax + by, ay - bx);
        x[R - k] = mkv<V>(ax - by, ay + bx);
      } else {
        x[k] = mkv<V>(ax - by, ay + bx);
        x[R - k] = mkv<V>(ax + by, ay - bx);
      }
    }
  } else {
    // R = p m: m-point DFTs of the p decimated sequences x[p j + r], twiddles
    // W_R^{r k}, p-point DFTs across r: X[k + m q]
    constexpr int p = first_factor(R), m = R / p;
    V y[p][m];
#pragma unroll
    for (int r = 0; r < p; ++r)
#pragma unroll
      for (int j = 0; j < m; ++j) y[r][j] = x[p * j + r];
#pragma unroll
    for (int r = 0; r < p; ++r) dft_reg<m, INV>(y[r]);
#pragma unroll
    for (int r = 1; r < p; ++r)
#pragma unroll
      for (int k = 1; k < m; ++k) y[r][k] = twr<R, INV>(y[r][k], r * k);
#pragma unroll
    for (int k = 0; k < m; ++k) {
      V t[p];
#pragma unroll
      for (int r = 0; r < p; ++r) t[r] = y[r][k];
      dft_reg<p, INV>(t);
#pragma unroll
      for (int q = 0; q < p; ++q) x[k + m * q] = t[q];
    }
  }
}

// FFT engines of the x transforms: the shared-memory twiddle table, the
// per-line buffer and the transform of one line by one warp (result in
// natural order).  Stockham: any N, ping-pong buffers of N values.
template <typename T, int MAXR> struct StockhamX {
  static constexpr int max_threads = sizeof(T) == 4 ? 512 : 256, min_blocks = 0;  // 16 or 8 lines, no bound
  static size_t line(int N) { return 2 * (size_t)N; }
  __device__ static size_t dline(int N) { return 2 * (size_t)N; }
  __device__ static void fill(T2<T> *tw, const FftPlan<T> &pl, int tid, int nt) {
    for (int t = tid; t < pl.n; t += nt) tw[t] = pl.tw[t];
  }
  template <bool INV>
  __device__ static T2<T> *run(T2<T> *buf, const FftPlan<T> &pl, const T2<T> *tw, int lane) {
    return fft_warp<T, INV, MAXR>(buf, buf + pl.n, pl, tw, lane);
  }
};

// Two-pass: N = A B (A, B <= 32), one buffer of max(N, A (B | 1)) values;
// the table holds W_N^{n2 k1} at [k1][n2] (row pitch B)
template <int A, int B, typename T = float> struct TwoPassX {
  // LINE even keeps every line buffer 16-byte aligned
  static constexpr int N = A * B, SB = B | 1, LINE = ((N > A * SB ? N : A * SB) + 1) & ~1;
  static_assert(A <= 32 && B <= 32, "one lane per butterfly");
  // FP32: up to 8 lines per CTA and three CTAs of 8 per SM: 80 registers,
  // which hold the 29-point pass without spills and leave room for 24 warps
  // per SM; FP64: the pass's doubled registers, one CTA of up to 8 lines
  static constexpr int max_threads = 256, min_blocks = sizeof(T) == 4 ? 3 : 1;
  static size_t line(int) { return LINE; }
  __device__ static size_t dline(int) { return LINE; }
  __device__ static void fill(T2<T> *tw, const FftPlan<T> &pl, int tid, int nt) {
    for (int t = tid; t < N; t += nt) {
      const int k1 = t / B, n2 = t - k1 * B;
      tw[t] = pl.tw[n2 * k1];  // n2 k1 < N
    }
  }
  template <bool INV>
  __device__ static T2<T> *run(T2<T> *buf, const FftPlan<T> &, const T2<T> *tw, int lane) {
    {
      T2<T> x[A];
      if (lane < B) {
#pragma unroll
        for (int n1 = 0; n1 < A; ++n1) x[n1] = buf[B * n1 + lane];
        dft_reg<A, INV>(x);
#pragma unroll
        for (int k1 = 1; k1 < A; ++k1) x[k1] = twm<T, INV>(x[k1], tw[k1 * B + lane]);
      }
      __syncwarp();
      if (lane < B) {
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) buf[k1 * SB + lane] = x[k1];
      }
      __syncwarp();
    }
    T2<T> y[B];
    if (lane < A) {
#pragma unroll
      for (int n2 = 0; n2 < B; ++n2) y[n2] = buf[lane * SB + n2];
      dft_reg<B, INV>(y);
    }
    __syncwarp();
    if (lane < A) {
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) buf[lane + A * k2] = y[k2];
    }
    __syncwarp();
    return buf;
  }
};

// ---------------------------------------------------------------------------
// divergence + DCT-II in x.  Each warp transforms one complex line holding
// the real lines q and q+1 (q = b*M + k').  R[q][kx] receives
// c_k = sum_i f_i cos(pi k (2i+1) / (2N)).
// ---------------------------------------------------------------------------
// Divergence of the real lines q and q+1 (q = b*M + k') into the complex line
// buffer in the DCT's reordered positions (point i at i/2 when even, at
// N-1-i/2 when odd), FP32, four consecutive points per lane with 16-byte
// loads (the box rows start 16-byte aligned at i = 2); U at i-1 of the first
// point comes from the previous lane, or from the previous round for lane 0.
// rfx: the FP32 reciprocal x spacings of the points, N rounded up to 4.
__device__ __forceinline__ void div_pair_vec(const Geo &g, const Spec &s, const float *__restrict__ U,
                                             const float *__restrict__ V, const float *__restrict__ W,
                                             const float *rfx, float2 *bufA, int q, int lane) {
  const int N = s.N, N4 = (N + 3) & ~3;
  const int nlines = s.NM * s.M;
  const bool hb = q + 1 < nlines;
  const int ba = q / s.M, ka = q - ba * s.M;
  const int bb = hb ? (q + 1) / s.M : ba, kb = hb ? (q + 1) - bb * s.M : ka;
  const long long ca = bidx(g, 2, ba + 2, ka + 2), cb = bidx(g, 2, bb + 2, kb + 2);
  // line B aliases line A when it does not exist, so every load is valid
  const long long cbb = hb ? cb : ca;
  const int jb = hb ? bb + 2 : ba + 2, kbb = hb ? kb + 2 : ka + 2;
  const float ryA = (float)g.ay.rF[ba + 2], rzA = (float)g.az.rF[ka + 2];
  const float ryB = (float)g.ay.rF[jb], rzB = (float)g.az.rF[kbb];
  float carA = __ldg(U + ca - 1), carB = __ldg(U + cbb - 1);
  for (int base = 0; base < N; base += 128) {
    const int i4 = base + 4 * lane, ic = i4 < N4 ? i4 : N4 - 4;  // in-row address for idle lanes
    const float4 rx = *reinterpret_cast<const float4 *>(rfx + ic);
    float fa[4], fb[4];
#pragma unroll
    for (int l = 0; l < 2; ++l) {
      const long long c = (l ? cbb : ca) + ic;
      const float4 u = __ldg(reinterpret_cast<const float4 *>(U + c));
      const float4 v = __ldg(reinterpret_cast<const float4 *>(V + c));
      const float4 vm = __ldg(reinterpret_cast<const float4 *>(V + c - g.px));
      const float4 w = __ldg(reinterpret_cast<const float4 *>(W + c));
      const float4 wm = __ldg(reinterpret_cast<const float4 *>(W + c - g.plane));
      float um0 = __shfl_up_sync(0xffffffffu, u.w, 1);
      const float car = l ? carB : carA;
      if (lane == 0) um0 = car;
      const float nc = __shfl_sync(0xffffffffu, u.w, 31);
      if (l) carB = nc;
      else carA = nc;
      const float ry = l ? ryB : ryA, rz = l ? rzB : rzA;
      float *f = l ? fb : fa;
      // projection.f90:42-44, as div_at
      f[0] = (u.x - um0) * rx.x + (v.x - vm.x) * ry + (w.x - wm.x) * rz;
      f[1] = (u.y - u.x) * rx.y + (v.y - vm.y) * ry + (w.y - wm.y) * rz;
      f[2] = (u.z - u.y) * rx.z + (v.z - vm.z) * ry + (w.z - wm.z) * rz;
      f[3] = (u.w - u.z) * rx.w + (v.w - vm.w) * ry + (w.w - wm.w) * rz;
    }
    if (!hb) fb[0] = fb[1] = fb[2] = fb[3] = 0.f;
    if (i4 + 3 < N && (N & 1) == 0) {
      // points i4, i4+2 go to the adjacent slots i4/2, i4/2+1; points
      // i4+3, i4+1 to N-2-i4/2, N-1-i4/2
      float *b = reinterpret_cast<float *>(bufA);
      *reinterpret_cast<float4 *>(b + i4) = make_float4(fa[0], fb[0], fa[2], fb[2]);
      *reinterpret_cast<float4 *>(b + 2 * (N - 2 - i4 / 2)) = make_float4(fa[3], fb[3], fa[1], fb[1]);
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int ip = i4 + e;
        if (ip < N) {
          const int pos = (ip & 1) ? (N - 1 - (ip >> 1)) : (ip >> 1);
          bufA[pos] = make_float2(fa[e], fb[e]);
        }
      }
    }
  }
}

// The DCT coefficients of the two lines from their packed transform res:
// V_A = (Z_k + conj Z_{N-k})/2, V_B = (Z_k - conj Z_{N-k})/(2i), c = Re(e^{-i pi k/2N} V)
template <typename T>
__device__ __forceinline__ void dct_pair_out(const T2<T> *res, const T2<T> *post, T *ra, int rx, int N, bool hb,
                                             int lane) {
  T *rb = ra + rx;
  for (int k = lane; k < N; k += 32) {
    const T2<T> z = res[k];
    const T2<T> zr = res[k == 0 ? 0 : N - k];
    const T2<T> p = post[k];
    const T vax = (T)0.5 * (z.x + zr.x), vay = (T)0.5 * (z.y - zr.y);
    const T vbx = (T)0.5 * (z.y + zr.y), vby = (T)0.5 * (zr.x - z.x);
    ra[k] = p.x * vax - p.y * vay;
    if (hb) rb[k] = p.x * vbx - p.y * vby;
  }
}

// FP32 CTAs take up to 16 lines (one CTA fills an SM's shared memory); the
// FP64 kernels need more registers per thread and stop at 8
template <typename T> struct DctCta { static constexpr int max_threads = sizeof(T) == 4 ? 512 : 256; };

template <typename T, class E>
__global__ void __launch_bounds__(E::max_threads, E::min_blocks) k_div_dct(Geo g, Spec s, FftPlan<T> pl, const T *__restrict__ U,
                                                 const T *__restrict__ V, const T *__restrict__ W,
                                                 T *__restrict__ R) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = s.N;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  T2<T> *tw = reinterpret_cast<T2<T> *>(smem_raw);
  T2<T> *post = tw + N;
  T2<T> *bufA = post + N + (size_t)warp * E::dline(N);
  // FP32: the reciprocal x spacings of the points, N rounded up to 4
  const int N4 = (N + 3) & ~3;
  float *rfx = reinterpret_cast<float *>(post + N + (size_t)nw * E::dline(N));
  E::fill(tw, pl, threadIdx.x, blockDim.x);
  for (int t = threadIdx.x; t < N; t += blockDim.x) post[t] = pl.post[t];
  if (sizeof(T) == 4)
    for (int t = threadIdx.x; t < N4; t += blockDim.x) rfx[t] = t < N ? (float)g.ax.rF[t + 2] : 0.f;
  __syncthreads();
  const int nlines = s.NM * s.M;
  const int q = (blockIdx.x * nw + warp) * 2;
  if (q >= nlines) return;
  const bool hb = q + 1 < nlines;
  const int ba = q / s.M, ka = q - ba * s.M;
  const int bb = hb ? (q + 1) / s.M : ba, kb = hb ? (q + 1) - bb * s.M : ka;
  const long long ca = bidx(g, 2, ba + 2, ka + 2), cb = bidx(g, 2, bb + 2, kb + 2);
  // line B aliases line A when it does not exist, so every load is valid
  const long long cbb = hb ? cb : ca;
  const int jb = hb ? bb + 2 : ba + 2, kbb = hb ? kb + 2 : ka + 2;
  const bool vec = sizeof(T) == 4 &&
                   ((reinterpret_cast<uintptr_t>(U) | reinterpret_cast<uintptr_t>(V) | reinterpret_cast<uintptr_t>(W)) &
                    15) == 0 && (g.px & 3) == 0;
  if constexpr (sizeof(T) == 4) {
    if (vec) div_pair_vec(g, s, U, V, W, rfx, bufA, q, lane);
  }
  // batches of 4 points per lane: all 48 loads issued before any use
  for (int base = 0; base < N && !vec; base += 128) {
    T fa[4], fb[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int ip = min(base + lane + 32 * u, N - 1);
      fa[u] = div_at<T>(g, U, V, W, ca + ip, ip + 2, ba + 2, ka + 2);
      fb[u] = div_at<T>(g, U, V, W, cbb + ip, ip + 2, jb, kbb);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int ip = base + lane + 32 * u;
      if (ip < N) {
        const T vb = hb ? fb[u] : (T)0;
        const int pos = (ip & 1) ? (N - 1 - (ip >> 1)) : (ip >> 1);
        bufA[pos] = mk<T>(fa[u], vb);
      }
    }
  }
  __syncwarp();
  const T2<T> *res = E::template run<false>(bufA, pl, tw, lane);
  dct_pair_out<T>(res, post, R + (long long)q * s.rx, s.rx, N, hb, lane);
}

// ---------------------------------------------------------------------------
// inverse DCT in x + box write of rhs_p (with the copies of
// apply_periodic_z_pressure: rhs_p(nxg-1,:,:) = rhs_p(nxg-2,:,:) and
// rhs_p(2:nxg-1,:,nzp+2) = rhs_p(2:nxg-1,:,2)); one complex line per warp.
// ---------------------------------------------------------------------------
template <typename T, class E>
__global__ void __launch_bounds__(E::max_threads, E::min_blocks) k_idct(Geo g, Spec s, FftPlan<T> pl, const T *__restrict__ R,
                                              T *__restrict__ p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = s.N;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  T2<T> *tw = reinterpret_cast<T2<T> *>(smem_raw);
  T2<T> *post = tw + N;
  T2<T> *bufA = post + N + (size_t)warp * E::dline(N);
  E::fill(tw, pl, threadIdx.x, blockDim.x);
  for (int t = threadIdx.x; t < N; t += blockDim.x) post[t] = pl.post[t];
  __syncthreads();
  const int nlines = s.NM * s.M;
  const int q = (blockIdx.x * nw + warp) * 2;
  if (q >= nlines) return;
  const bool hb = q + 1 < nlines;
  const T *ra = R + (long long)q * s.rx;
  const T *rb = ra + s.rx;
  for (int k = lane; k < N; k += 32) {
    const T xa = ra[k], xan = k ? ra[N - k] : (T)0;
    const T xb = hb ? rb[k] : (T)0, xbn = (hb && k) ? rb[N - k] : (T)0;
    // V_k = exp(+i pi k/2N) (X_k - i X_{N-k});  Z = V_A + i V_B
    const T2<T> e = mk<T>(post[k].x, -post[k].y);
    const T2<T> va = cmul<T>(e, mk<T>(xa, -xan));
    const T2<T> vb = cmul<T>(e, mk<T>(xb, -xbn));
    bufA[k] = mk<T>(va.x - vb.y, va.y + vb.x);
  }
  __syncwarp();
  const T2<T> *res = E::template run<true>(bufA, pl, tw, lane);
  const T inv = (T)1 / (T)N;
  const int ba = q / s.M, ka = q - ba * s.M;
  const int bb = hb ? (q + 1) / s.M : ba, kb = hb ? (q + 1) - bb * s.M : ka;
  const long long ca = bidx(g, 2, ba + 2, ka + 2), cb = bidx(g, 2, bb + 2, kb + 2);
  const long long zsh = (long long)s.M * g.plane;  // k = 2 -> k = nzp+2
  for (int ip = lane; ip < N; ip += 32) {
    const int pos = (ip & 1) ? (N - 1 - (ip >> 1)) : (ip >> 1);
    const T2<T> z = res[pos];
    const T va = z.x * inv, vb = z.y * inv;
    p[ca + ip] = va;
    if (ka == 0) p[ca + ip + zsh] = va;
    if (hb) {
      p[cb + ip] = vb;
      if (kb == 0) p[cb + ip + zsh] = vb;
    }
    if (ip == N - 1) {  // i = nxg-1 copy
      p[ca + N] = va;
      if (ka == 0) p[ca + N + zsh] = va;
      if (hb) {
        p[cb + N] = vb;
        if (kb == 0) p[cb + N + zsh] = vb;
      }
    }
  }
}

// Inverse DCT with the two-pass FFT (both precisions), the steps around the transform
// folded into its passes: one bulk copy brings the two rows of R into the
// line buffer; pass 1 forms its inputs Z_n = V_A + i V_B from them in
// registers; pass 2 writes its outputs from registers straight to the box
// positions (Z_n holds the points i = 2n, or 2N-1-2n for 2n >= N).  The
// copy's wait is bounded: when it runs out, bit 16 of the device flag is set
// and the line is left unwritten.
template <int A, int B, typename T = float>
__global__ void __launch_bounds__(TwoPassX<A, B, T>::max_threads, TwoPassX<A, B, T>::min_blocks)
    k_idct2(Geo g, Spec s, FftPlan<T> pl, const T *__restrict__ R, T *__restrict__ p, int *__restrict__ err) {
  using E = TwoPassX<A, B, T>;
  using namespace tma;
  constexpr int N = E::N, SB = E::SB, LINE = E::LINE;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  T2<T> *tw = reinterpret_cast<T2<T> *>(smem_raw);
  T2<T> *post = tw + N;
  T2<T> *buf = post + N + (size_t)warp * LINE;
  uint64_t *bar = reinterpret_cast<uint64_t *>(
      reinterpret_cast<unsigned char *>(post + N + (size_t)nw * LINE) + 4 * ((N + 3) / 4 * 4)) + warp;
  E::fill(tw, pl, threadIdx.x, blockDim.x);
  for (int t = threadIdx.x; t < N; t += blockDim.x) post[t] = pl.post[t];
  const int nlines = s.NM * s.M;
  const int q = (blockIdx.x * nw + warp) * 2;
  const bool hb = q + 1 < nlines;
  if (lane == 0 && q < nlines) {
    mbar_init(bar, 1);
    mbar_init_fence();
    // rows q and q+1 (rx apart) as one block, the length rounded up to 16 bytes
    const uint32_t bytes = (uint32_t)sizeof(T) * (uint32_t)((hb ? s.rx : 0) + ((N + 3) & ~3));
    mbar_expect_tx(bar, bytes);
    bulk_load(buf, R + (long long)q * s.rx, bytes, bar);
  }
  __syncthreads();
  if (q >= nlines) return;
  if (!__all_sync(0xffffffffu, mbar_wait(bar, 0))) {
    if (lane == 0) {
      atomicOr(err, 16);
      mbar_wait(bar, 0);  // let the copy finish (bounded) before leaving
    }
    return;
  }
  const T *ra = reinterpret_cast<const T *>(buf);
  const T *rb = ra + s.rx;
  {
    // pass 1 (lane n2 < B): Z_n for n = B n1 + n2, V_n = exp(+i pi n/2N) (X_n - i X_{N-n})
    T2<T> x[A];
    if (lane < B) {
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1) {
        const int n = B * n1 + lane;
        const T xa = ra[n], xan = n ? ra[N - n] : (T)0;
        const T xb = hb ? rb[n] : (T)0, xbn = (hb && n) ? rb[N - n] : (T)0;
        const T2<T> e = mk<T>(post[n].x, -post[n].y);
        const T2<T> va = cmul<T>(e, mk<T>(xa, -xan));
        const T2<T> vb = cmul<T>(e, mk<T>(xb, -xbn));
        x[n1] = mk<T>(va.x - vb.y, va.y + vb.x);
      }
      dft_reg<A, true>(x);
#pragma unroll
      for (int k1 = 1; k1 < A; ++k1) x[k1] = twm<T, true>(x[k1], tw[k1 * B + lane]);
    }
    __syncwarp();  // every read of the raw rows is done
    if (lane < B) {
#pragma unroll
      for (int k1 = 0; k1 < A; ++k1) buf[k1 * SB + lane] = x[k1];
    }
    __syncwarp();
  }
  if (lane < A) {
    T2<T> y[B];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) y[n2] = buf[lane * SB + n2];
    dft_reg<B, true>(y);
    const T inv = (T)1 / (T)N;
    const int ba = q / s.M, ka = q - ba * s.M;
    const int bb = hb ? (q + 1) / s.M : ba, kb = hb ? (q + 1) - bb * s.M : ka;
    const long long ca = bidx(g, 2, ba + 2, ka + 2), cb = bidx(g, 2, bb + 2, kb + 2);
    const long long zsh = (long long)s.M * g.plane;  // k = 2 -> k = nzp+2
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) {
      const int n = lane + A * k2;
      const int ip = 2 * n < N ? 2 * n : 2 * N - 1 - 2 * n;
      const T va = y[k2].x * inv, vb = y[k2].y * inv;
      p[ca + ip] = va;
      if (ka == 0) p[ca + ip + zsh] = va;
      if (hb) {
        p[cb + ip] = vb;
        if (kb == 0) p[cb + ip + zsh] = vb;
      }
      if (ip == N - 1) {  // i = nxg-1 copy
        p[ca + N] = va;
        if (ka == 0) p[ca + N + zsh] = va;
        if (hb) {
          p[cb + N] = vb;
          if (kb == 0) p[cb + N + zsh] = vb;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// real DFT in z over the half spectrum, as a register-tiled product with the
// table tz[m][n] = (cos, sin)(2 pi m n / M), m, n = 0..MH-1 (row pitch MH).
// CTA: one row b, 64 kx (2 per lane), 8 warps x RK wavenumbers.
// forward: Re C_kz = f_0 + sum_{k=1..H} (f_k + f_{M-k}) cos + [M even] f_{M/2} (-1)^kz
//          Im C_kz = -sum_{k=1..H} (f_k - f_{M-k}) sin
// inverse: f_p, f_{M-p} = (C_0 + 2 (P_p -+ Q_p) + [M even] C_{M/2} (-1)^p) / M,
//          P_p = sum_{kz=1..H} Re C_kz cos, Q_p = sum Im C_kz sin
// ---------------------------------------------------------------------------
template <typename T> struct Vec16;  // 16-byte vector of T
template <> struct Vec16<float> { typedef float4 type; static constexpr int n = 4; };
template <> struct Vec16<double> { typedef double2 type; static constexpr int n = 2; };

template <typename T> __device__ __forceinline__ T vget(const typename Vec16<T>::type &v, int e);
template <> __device__ __forceinline__ float vget<float>(const float4 &v, int e) {
  return e == 0 ? v.x : e == 1 ? v.y : e == 2 ? v.z : v.w;
}
template <> __device__ __forceinline__ double vget<double>(const double2 &v, int e) { return e == 0 ? v.x : v.y; }

template <typename T, int RK>
__global__ void __launch_bounds__(256) k_dft_z_fwd(Spec s, const T *__restrict__ R, T2<T> *__restrict__ C,
                                                   const T2<T> *__restrict__ tz) {
  typedef typename Vec16<T>::type VT;
  constexpr int KX = Vec16<T>::n;   // kx values per lane
  constexpr int TW = 32 * KX;       // kx per CTA
  extern __shared__ __align__(16) unsigned char smem_raw[];
  VT *f = reinterpret_cast<VT *>(smem_raw);  // [M][32] vectors of KX kx
  const int M = s.M, MH = s.MH, H = (M - 1) / 2;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int b = blockIdx.y;
  const int kx0 = blockIdx.x * TW + KX * lane;
  const int nvalid = min(KX, s.N - kx0);
  for (int k = warp; k < M; k += 8) {
    const T *row = R + ((long long)b * M + k) * s.rx + kx0;
    T v[KX];
#pragma unroll
    for (int e = 0; e < KX; ++e) v[e] = e < nvalid ? row[e] : (T)0;
    f[k * 32 + lane] = *reinterpret_cast<VT *>(v);
  }
  __syncthreads();
  const int kzb = blockIdx.z * 8 * RK + warp * RK;
  if (kzb >= MH) return;
  T re[RK][KX], im[RK][KX];
  const VT f0 = f[lane];
  int rows[RK];
#pragma unroll
  for (int r = 0; r < RK; ++r) {
    rows[r] = min(kzb + r, MH - 1) * MH;
#pragma unroll
    for (int e = 0; e < KX; ++e) {
      re[r][e] = vget<T>(f0, e);
      im[r][e] = 0;
    }
  }
  T2<T> tn[RK];  // table values of the next k, loaded one iteration ahead
#pragma unroll
  for (int r = 0; r < RK; ++r) tn[r] = __ldg(tz + rows[r] + 1);
  for (int k = 1; k <= H; ++k) {
    T2<T> t[RK];
#pragma unroll
    for (int r = 0; r < RK; ++r) {
      t[r] = tn[r];
      tn[r] = __ldg(tz + rows[r] + min(k + 1, H));
    }
    const VT fk = f[k * 32 + lane], fm = f[(M - k) * 32 + lane];
    T a[KX], bb[KX];
#pragma unroll
    for (int e = 0; e < KX; ++e) {
      a[e] = vget<T>(fk, e) + vget<T>(fm, e);
      bb[e] = vget<T>(fk, e) - vget<T>(fm, e);
    }
#pragma unroll
    for (int r = 0; r < RK; ++r) {
#pragma unroll
      for (int e = 0; e < KX; ++e) {
        re[r][e] += a[e] * t[r].x;
        im[r][e] -= bb[e] * t[r].y;
      }
    }
  }
  const bool even = (M & 1) == 0;
  const VT fh = f[(even ? M / 2 : 0) * 32 + lane];
#pragma unroll
  for (int r = 0; r < RK; ++r) {
    const int kz = kzb + r;
    if (kz >= MH) break;
    T2<T> *out = C + ((long long)b * MH + kz) * s.rx + kx0;
#pragma unroll
    for (int e = 0; e < KX; ++e) {
      T a = re[r][e];
      if (even) a += (kz & 1) ? -vget<T>(fh, e) : vget<T>(fh, e);
      if (e < nvalid) out[e] = mk<T>(a, im[r][e]);
    }
  }
}

template <typename T, int RK>
__global__ void __launch_bounds__(256) k_dft_z_inv(Spec s, const T2<T> *__restrict__ C, T *__restrict__ R,
                                                   const T2<T> *__restrict__ tz) {
  constexpr int KX = Vec16<T>::n;
  constexpr int TW = 32 * KX;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T2<T> *c = reinterpret_cast<T2<T> *>(smem_raw);  // [MH][TW]
  const int M = s.M, MH = s.MH, H = (M - 1) / 2;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int b = blockIdx.y;
  const int kx0 = blockIdx.x * TW + KX * lane;
  const int nvalid = min(KX, s.N - kx0);
  for (int kz = warp; kz < MH; kz += 8) {
    const T2<T> *row = C + ((long long)b * MH + kz) * s.rx + kx0;
#pragma unroll
    for (int e = 0; e < KX; ++e) c[kz * TW + KX * lane + e] = e < nvalid ? row[e] : mk<T>(0, 0);
  }
  __syncthreads();
  const int npairs = M / 2 + 1;
  const int pb = blockIdx.z * 8 * RK + warp * RK;
  if (pb >= npairs) return;
  T P[RK][KX], Q[RK][KX];
  int rows[RK];
#pragma unroll
  for (int r = 0; r < RK; ++r) {
    rows[r] = min(pb + r, MH - 1) * MH;
#pragma unroll
    for (int e = 0; e < KX; ++e) {
      P[r][e] = 0;
      Q[r][e] = 0;
    }
  }
  T2<T> tn[RK];
#pragma unroll
  for (int r = 0; r < RK; ++r) tn[r] = __ldg(tz + rows[r] + 1);
  for (int kz = 1; kz <= H; ++kz) {
    T2<T> t[RK];
#pragma unroll
    for (int r = 0; r < RK; ++r) {
      t[r] = tn[r];
      tn[r] = __ldg(tz + rows[r] + min(kz + 1, H));
    }
    T2<T> v[KX];
#pragma unroll
    for (int e = 0; e < KX; ++e) v[e] = c[kz * TW + KX * lane + e];
#pragma unroll
    for (int r = 0; r < RK; ++r) {
#pragma unroll
      for (int e = 0; e < KX; ++e) {
        P[r][e] += v[e].x * t[r].x;
        Q[r][e] += v[e].y * t[r].y;
      }
    }
  }
  const bool even = (M & 1) == 0;
  const T invM = (T)1 / (T)M;
#pragma unroll
  for (int r = 0; r < RK; ++r) {
    const int pp = pb + r;
    if (pp >= npairs) break;
    T *lo = R + ((long long)b * M + pp) * s.rx + kx0;
    const int pm = M - pp;
    T *hi = R + ((long long)b * M + pm) * s.rx + kx0;
#pragma unroll
    for (int e = 0; e < KX; ++e) {
      if (e >= nvalid) continue;
      const T c0 = c[KX * lane + e].x;
      const T ny = even ? c[(M / 2) * TW + KX * lane + e].x : (T)0;
      const T y = (pp & 1) ? -ny : ny;
      lo[e] = (c0 + (T)2 * (P[r][e] - Q[r][e]) + y) * invM;
      if (pm != pp && pm < M) hi[e] = (c0 + (T)2 * (P[r][e] + Q[r][e]) + y) * invM;
    }
  }
}

// ---------------------------------------------------------------------------
// FP64 z transforms as products on the FP64 tensor-core MMA (mma.sync
// m8n8k4 f64; the tcgen05 MMA has no FP64 kind).  The sums of the direct
// transforms above, with H = (M-1)/2 and the half-spectrum rows r = 0..MH-1:
//   forward  Re C_r = f_0 + sum_{k=1..H} S_k cos(2 pi r k/M) [+ (-1)^r f_{M/2}, M even]
//            Im C_r = -sum_{k=1..H} D_k sin(2 pi r k/M),  S_k, D_k = f_k +- f_{M-k}
//   inverse  f_p, f_{M-p} = (C_0 + 2 (P_p -+ Q_p) [+ (-1)^p C_{M/2}]) / M,
//            P_p = sum_{k=1..H} Re C_k cos(2 pi p k/M), Q_p = sum Im C_k sin(...)
// are each a product (rows r or p) x (K = H terms) x (32 x columns of a CTA)
// with the tables tc[r][k-1] = cos, ts[r][k-1] = sin (rows to MHp = MH
// rounded up to 16, columns to Kp = H rounded up to 4, zero beyond H and
// MH).  A CTA owns one row b and 32 kx; its column data sit in shared memory
// transposed ([x][k], pitch PZ = 4 mod 16 doubles, so the B fragments meet
// two wavefronts); the forward folds S_k, D_k in place (F[x][k], F[x][M-k]).
// Warp w computes rows 16w .. 16w+15 by 2 x 4 MMA tiles of 8 x 8, K in steps
// of 4.  Fragments (PTX m8n8k4 .f64): A a0 at (row lane/4, col lane%4), B b0
// at (row lane%4, col lane/4), C c0, c1 at (row lane/4, cols 2 (lane%4) + i).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}
__host__ __device__ inline int zd64_kp(int M) { return ((M - 1) / 2 + 3) / 4 * 4; }
__host__ __device__ inline int zd64_rows(int M) { return (M / 2 + 1 + 15) / 16 * 16; }
// pitch of the transposed column data: >= the larger of M and Kp + 1, = 4 mod 16
__host__ __device__ inline int zd64_pitch(int len) { return (len + 11) / 16 * 16 + 4; }

__global__ void __launch_bounds__(256) k_zdft64_fwd(Spec s, const double *__restrict__ R, double2 *__restrict__ C,
                                                    const double *__restrict__ tc, const double *__restrict__ ts) {
  extern __shared__ double zf[];  // [32][PZ]
  const int M = s.M, MH = s.MH, H = (M - 1) / 2, Kp = zd64_kp(M), PZ = zd64_pitch(M);
  const int b = blockIdx.y, x0 = blockIdx.x * 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  const bool xin = x0 + lane < s.N;
  // rows in batches of 8 per warp, every load of a batch issued before the
  // stores (the slab comes from DRAM)
  for (int k8 = warp * 8; k8 < PZ; k8 += nw * 8) {
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = k8 + u;
      v[u] = (k < M && xin) ? __ldcs(R + ((long long)b * M + k) * s.rx + x0 + lane) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (k8 + u < PZ) zf[lane * PZ + k8 + u] = v[u];
  }
  __syncthreads();
  for (int t = tid; t < 32 * H; t += blockDim.x) {
    const int x = t & 31, k = 1 + (t >> 5);
    const double a = zf[x * PZ + k], c = zf[x * PZ + M - k];
    zf[x * PZ + k] = a + c;
    zf[x * PZ + M - k] = a - c;
  }
  __syncthreads();
  const int r0 = 16 * warp;
  if (r0 >= MH) return;
  const int g = lane >> 2, q = lane & 3;
  double re[2][4][2] = {}, im[2][4][2] = {};
  // table fragments of the next K step fetched one step ahead
  const double *tcr = tc + (r0 + g) * Kp + q, *tsr = ts + (r0 + g) * Kp + q;
  double nc[2] = {__ldg(tcr), __ldg(tcr + 8 * Kp)}, ns[2] = {__ldg(tsr), __ldg(tsr + 8 * Kp)};
  for (int k0 = 1; k0 <= Kp; k0 += 4) {
    const int k = k0 + q;  // 1 .. Kp: S_k at zf[x][k], D_k at zf[x][M-k] (table zero for k > H)
    double ac[2] = {nc[0], nc[1]}, as[2] = {ns[0], ns[1]}, bs[4], bd[4];
    if (k0 + 4 <= Kp) {
      nc[0] = __ldg(tcr + k0 + 3);
      nc[1] = __ldg(tcr + 8 * Kp + k0 + 3);
      ns[0] = __ldg(tsr + k0 + 3);
      ns[1] = __ldg(tsr + 8 * Kp + k0 + 3);
    }
#pragma unroll
    for (int ct = 0; ct < 4; ++ct) {
      bs[ct] = zf[(8 * ct + g) * PZ + k];
      bd[ct] = zf[(8 * ct + g) * PZ + M - k];
    }
#pragma unroll
    for (int rt = 0; rt < 2; ++rt)
#pragma unroll
      for (int ct = 0; ct < 4; ++ct) {
        dmma(re[rt][ct], ac[rt], bs[ct]);
        dmma(im[rt][ct], as[rt], bd[ct]);
      }
  }
  const bool even = (M & 1) == 0;
#pragma unroll
  for (int rt = 0; rt < 2; ++rt) {
    const int r = r0 + 8 * rt + g;
    if (r >= MH) continue;
#pragma unroll
    for (int ct = 0; ct < 4; ++ct)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int x = 8 * ct + 2 * q + i;
        if (x0 + x >= s.N) continue;
        double a = zf[x * PZ] + re[rt][ct][i];
        if (even) a += (r & 1) ? -zf[x * PZ + M / 2] : zf[x * PZ + M / 2];
        C[((long long)b * MH + r) * s.rx + x0 + x] = make_double2(a, -im[rt][ct][i]);
      }
  }
}

__global__ void __launch_bounds__(256) k_zdft64_inv(Spec s, const double2 *__restrict__ C, double *__restrict__ R,
                                                    const double *__restrict__ tc, const double *__restrict__ ts) {
  extern __shared__ double zf[];  // Re [32][PZ], then Im [32][PZ]
  const int M = s.M, MH = s.MH, Kp = zd64_kp(M), PZ = zd64_pitch(Kp + 1 > MH ? Kp + 1 : MH);
  double *zr = zf, *zi = zf + 32 * PZ;
  const int b = blockIdx.y, x0 = blockIdx.x * 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  const bool xin = x0 + lane < s.N;
  for (int k8 = warp * 8; k8 < PZ; k8 += nw * 8) {
    double2 v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = k8 + u;
      v[u] = (k < MH && xin) ? __ldcs(C + ((long long)b * MH + k) * s.rx + x0 + lane) : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (k8 + u < PZ) {
        zr[lane * PZ + k8 + u] = v[u].x;
        zi[lane * PZ + k8 + u] = v[u].y;
      }
  }
  __syncthreads();
  const int npairs = M / 2 + 1;
  const int p0 = 16 * warp;
  if (p0 >= npairs) return;
  const int g = lane >> 2, q = lane & 3;
  double P[2][4][2] = {}, Q[2][4][2] = {};
  const double *tcr = tc + (p0 + g) * Kp + q, *tsr = ts + (p0 + g) * Kp + q;
  double nc[2] = {__ldg(tcr), __ldg(tcr + 8 * Kp)}, ns[2] = {__ldg(tsr), __ldg(tsr + 8 * Kp)};
  for (int k0 = 1; k0 <= Kp; k0 += 4) {
    const int k = k0 + q;
    double ac[2] = {nc[0], nc[1]}, as[2] = {ns[0], ns[1]}, br[4], bi[4];
    if (k0 + 4 <= Kp) {
      nc[0] = __ldg(tcr + k0 + 3);
      nc[1] = __ldg(tcr + 8 * Kp + k0 + 3);
      ns[0] = __ldg(tsr + k0 + 3);
      ns[1] = __ldg(tsr + 8 * Kp + k0 + 3);
    }
#pragma unroll
    for (int ct = 0; ct < 4; ++ct) {
      br[ct] = zr[(8 * ct + g) * PZ + k];
      bi[ct] = zi[(8 * ct + g) * PZ + k];
    }
#pragma unroll
    for (int rt = 0; rt < 2; ++rt)
#pragma unroll
      for (int ct = 0; ct < 4; ++ct) {
        dmma(P[rt][ct], ac[rt], br[ct]);
        dmma(Q[rt][ct], as[rt], bi[ct]);
      }
  }
  const bool even = (M & 1) == 0;
  const double invM = 1.0 / (double)M;
#pragma unroll
  for (int rt = 0; rt < 2; ++rt) {
    const int pp = p0 + 8 * rt + g;
    if (pp >= npairs) continue;
    const int pm = M - pp;
#pragma unroll
    for (int ct = 0; ct < 4; ++ct)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int x = 8 * ct + 2 * q + i;
        if (x0 + x >= s.N) continue;
        const double c0 = zr[x * PZ];
        const double ny = even ? zr[x * PZ + M / 2] : 0.0;
        const double y = (pp & 1) ? -ny : ny;
        const double pv = P[rt][ct][i], qv = Q[rt][ct][i];
        R[((long long)b * M + pp) * s.rx + x0 + x] = (c0 + 2.0 * (pv - qv) + y) * invM;
        if (pm != pp && pm < M) R[((long long)b * M + pm) * s.rx + x0 + x] = (c0 + 2.0 * (pv + qv) + y) * invM;
      }
  }
}

// tables tc, ts ([MHp][Kp] each, in that order) of the FP64 z transforms
void zdft64_tables(const Spec &s, std::vector<double> &t) {
  const int M = s.M, H = (M - 1) / 2, rows = zd64_rows(M), Kp = zd64_kp(M), MH = s.MH;
  t.assign(2 * (size_t)rows * Kp, 0.0);
  for (int r = 0; r < MH && r < rows; ++r)
    for (int k = 1; k <= H; ++k) {
      const double a = 2.0 * M_PI * (double)(((long long)r * k) % M) / (double)M;
      t[(size_t)r * Kp + (k - 1)] = cos(a);
      t[(size_t)rows * Kp + (size_t)r * Kp + (k - 1)] = sin(a);
    }
}

void launch_zdft64(const Spec &s, double *R, double2 *C, const double *tab, int inverse, cudaStream_t st) {
  const int rows = zd64_rows(s.M), Kp = zd64_kp(s.M);
  const double *tc = tab, *ts = tab + (size_t)rows * Kp;
  const dim3 grid((s.N + 31) / 32, s.NM);
  const int threads = 32 * (rows / 16);
  if (!inverse) {
    const size_t sm = (size_t)32 * zd64_pitch(s.M) * sizeof(double);
    cudaFuncSetAttribute(k_zdft64_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_zdft64_fwd<<<grid, threads, sm, st>>>(s, R, C, tc, ts);
  } else {
    const int len = Kp + 1 > s.MH ? Kp + 1 : s.MH;
    const size_t sm = (size_t)2 * 32 * zd64_pitch(len) * sizeof(double);
    cudaFuncSetAttribute(k_zdft64_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_zdft64_inv<<<grid, threads, sm, st>>>(s, C, R, tc, ts);
  }
}

// ---------------------------------------------------------------------------
// Tridiagonal solve in y for every (kx, kz) mode, FP64 arithmetic.
// Row b (= j-2) of the operator: diag dd[b] + kxx[kx] + kzz[kz] (row 0 of
// mode (0,0) scaled by 3/2, initialization.f90:454), sub dl[b] = Dyy(j,j-1),
// super du[b] = Dyy(j,j+1).  The pivots of the elimination depend on the
// grid only, so k_thomas_factors computes their inverses once (piv[b][kz][kx]
// = 1/d'_b); the solve is then the two linear recurrences
//   g_b = r_b - (dl_b piv_{b-1}) g_{b-1},  x_b = (g_b - du_b x_{b+1}) piv_b
// with the arithmetic of the on-the-fly elimination, without a division on
// the serial chain.
// skip_kz0 (mixed form): the kz = 0 plane is solved in FP64 by the kz0
// kernels below, so its coefficients here are zeroed.
// ---------------------------------------------------------------------------
__global__ void k_thomas_factors(Spec s, double *__restrict__ piv, const double *__restrict__ dd,
                                 const double *__restrict__ dl, const double *__restrict__ du,
                                 const double *__restrict__ kxx, const double *__restrict__ kzz) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x;
  const int kz = blockIdx.y;
  if (kx >= s.N || kz >= s.MH) return;
  const long long rs = (long long)s.MH * s.rx;
  const long long base = (long long)kz * s.rx + kx;
  const double kk = kxx[kx], kzv = kzz[kz];
  double rinv = 0.0;
  for (int b = 0; b < s.NM; ++b) {
    double d = (dd[b] + kk) + kzv;
    if (kx == 0 && kz == 0 && b == 0) d = 3.0 / 2.0 * d;
    if (b > 0) {
      const double w = dl[b] * rinv;
      d = d - w * du[b - 1];
    }
    rinv = 1.0 / d;
    piv[base + b * rs] = rinv;
  }
}

// One thread per complex mode (a CTA takes 128 consecutive kx of one kz, so
// each row step reads 1 KB runs of C and of piv), both sweeps down the NM
// rows b with a ring of PF rows in flight: row b+PF is requested when row b
// is consumed.  Rows are reached by stepping one pointer into C and one into
// piv by the row stride; the row loads are cached in L2 only (each is read
// once per sweep), so the ring is not bounded by the L1 capacity.
template <typename T, int PF>
__device__ __forceinline__ void thomas_sweeps(T2<T> *__restrict__ Cm, const double *__restrict__ pm, long long rs,
                                              int NM, const double *__restrict__ dl, const double *__restrict__ du) {
  // forward: g_b = r_b - (l_b / d'_{b-1}) g_{b-1}, stored over r_b
  T2<T> cr[PF];
  double pr[PF];
  const T2<T> *cn = Cm;
  const double *pn = pm;
#pragma unroll
  for (int u = 0; u < PF; ++u) {
    cr[u] = u < NM ? __ldcg(cn) : mk<T>((T)0, (T)0);
    pr[u] = u < NM ? __ldcg(pn) : 0.0;
    if (u < NM) { cn += rs; pn += rs; }
  }
  double gx = 0.0, gy = 0.0, rprev = 0.0;
  T2<T> *cw = Cm;
  for (int b0 = 0; b0 < NM; b0 += PF) {
#pragma unroll
    for (int u = 0; u < PF; ++u) {
      const int b = b0 + u;
      if (b < NM) {
        const T2<T> cv = cr[u];
        const double pv = pr[u];
        if (b + PF < NM) {
          cr[u] = __ldcg(cn);
          pr[u] = __ldcg(pn);
          cn += rs;
          pn += rs;
        }
        double rx = (double)cv.x, ry = (double)cv.y;
        if (b > 0) {
          const double w = dl[b] * rprev;  // l_b / d'_{b-1}
          rx = rx - w * gx;
          ry = ry - w * gy;
        }
        rprev = pv;
        gx = rx;
        gy = ry;
        *cw = mk<T>((T)rx, (T)ry);
        cw += rs;
      }
    }
  }
  // backward: x_b = (g_b - u_b x_{b+1}) / d'_b from the top row down
  const int top = NM - 1;
  const T2<T> *cb = Cm + (long long)top * rs;
  const double *pb = pm + (long long)top * rs;
#pragma unroll
  for (int u = 0; u < PF; ++u) {
    cr[u] = u < NM ? __ldcg(cb) : mk<T>((T)0, (T)0);
    pr[u] = u < NM ? __ldcg(pb) : 0.0;
    if (u < NM) { cb -= rs; pb -= rs; }
  }
  double xx = 0.0, xy = 0.0;
  cw = Cm + (long long)top * rs;
  for (int b0 = top; b0 >= 0; b0 -= PF) {
#pragma unroll
    for (int u = 0; u < PF; ++u) {
      const int b = b0 - u;
      if (b >= 0) {
        const T2<T> cv = cr[u];
        const double pv = pr[u];
        if (b - PF >= 0) {
          cr[u] = __ldcg(cb);
          pr[u] = __ldcg(pb);
          cb -= rs;
          pb -= rs;
        }
        if (b == top) {
          xx = (double)cv.x * pv;
          xy = (double)cv.y * pv;
        } else {
          xx = ((double)cv.x - du[b] * xx) * pv;
          xy = ((double)cv.y - du[b] * xy) * pv;
        }
        *cw = mk<T>((T)xx, (T)xy);
        cw -= rs;
      }
    }
  }
}

template <typename T, int PF>
__global__ void __launch_bounds__(128) k_thomas(Spec s, T2<T> *__restrict__ C, const double *__restrict__ piv,
                                                const double *__restrict__ dl, const double *__restrict__ du,
                                                double *__restrict__ H0, int klow) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x;
  const int kz = blockIdx.y;
  if (kx >= s.N || kz >= s.MH) return;
  const int NM = s.NM;
  const long long rs = (long long)s.MH * s.rx;  // stride between rows b
  const long long base = (long long)kz * s.rx + kx;
  // mixed form: the low-kx modes of kz = 0 carry the box-scale pressure;
  // they are solved with FP64 intermediates into H0[b][kx] (real part; the
  // imaginary part of kz = 0 is zero) and dropped from the FP32 data
  if (H0 && kz == 0 && kx < klow) {
    const T *Cr = reinterpret_cast<const T *>(C + base);  // real part of row b at Cr[2 b rs]
    double *Hd = H0 + kx;                                   // H0[b * klow + kx]
    // rows in batches of PB, every load of a batch issued before its first
    // use (one CTA runs this path; unbatched it would be the kernel's tail);
    // PB = 8 keeps the kernel's register count that of the main path
    constexpr int PB = 8;
    double g = 0.0, rprev = 0.0;
    for (int b0 = 0; b0 < NM; b0 += PB) {
      double rv[PB], pvv[PB];
#pragma unroll
      for (int u = 0; u < PB; ++u) {
        const int b = b0 + u;
        rv[u] = b < NM ? (double)Cr[2 * (long long)b * rs] : 0.0;
        pvv[u] = b < NM ? piv[base + b * rs] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < PB; ++u) {
        const int b = b0 + u;
        if (b < NM) {
          double r = rv[u];
          if (b > 0) {
            const double w = dl[b] * rprev;
            r = r - w * g;
          }
          rprev = pvv[u];
          g = r;
          Hd[(long long)b * klow] = r;
        }
      }
    }
    double x = 0.0;
    for (int b0 = NM - 1; b0 >= 0; b0 -= PB) {
      double hv[PB], pvv[PB];
#pragma unroll
      for (int u = 0; u < PB; ++u) {
        const int b = b0 - u;
        hv[u] = b >= 0 ? Hd[(long long)b * klow] : 0.0;
        pvv[u] = b >= 0 ? piv[base + b * rs] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < PB; ++u) {
        const int b = b0 - u;
        if (b >= 0) {
          x = (b == NM - 1) ? hv[u] * pvv[u] : (hv[u] - du[b] * x) * pvv[u];
          Hd[(long long)b * klow] = x;
        }
      }
    }
    for (int b = 0; b < NM; ++b) C[base + b * rs] = mk<T>((T)0, (T)0);
    return;
  }
  thomas_sweeps<T, PF>(C + base, piv + base, rs, NM, dl, du);
}

// ---------------------------------------------------------------------------
// Mixed form: the box-scale part of the pressure in FP64.  A step whose
// inflow flux differs from the interior's drives a pressure that varies
// along the whole box; FP32 keeps only ~7 digits of it, and near the wall
// (small y spacings) the rounding noise of p alone leaves a divergence of
// order eps32 |p| / dy^2.  That field lives in the z-mean (kz = 0) modes of
// low kx, so k_thomas solves the modes kz = 0, kx < klow in FP64 into H0
// (their forcing, the FP32 transform of the divergence, is accurate to FP32
// relative to |div|), and
//   k_kz0_idct: p0(i,j) = sum_{kx<klow} H0(kx,j) w_kx cos(pi kx (2i+1)/2N)/(N M)
//               (w_0 = 1, w_kx = 2), a dense product with a cosine table;
//   k_kz0_grad: the x and y differences of p0 taken in FP64, stored as FP32
// and the projection adds them to the differences of the FP32 part.
// ---------------------------------------------------------------------------
// p0[b][i] = sum_{kx < K} H[b][kx] cm[kx][i]: 32 x 64 output tiles, k-tiles of 32
__global__ void __launch_bounds__(256) k_kz0_idct(Spec s, const double *__restrict__ H, int K,
                                                  const double *__restrict__ cm, double *__restrict__ p0) {
  constexpr int BM = 16, BN = 64, BK = 32;  // 16-row tiles: 208 CTAs at 812 x 256
  __shared__ double As[BK][BM + 1];
  __shared__ double Bs[BK][BN];
  const int N = s.N, NM = s.NM;
  const int b0 = blockIdx.y * BM, i0 = blockIdx.x * BN;
  const int t = threadIdx.x, tr = t >> 4, tc = t & 15;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int k0 = 0; k0 < K; k0 += BK) {
    for (int q = t; q < BM * BK; q += 256) {
      const int r = q / BK, c = q % BK;
      As[c][r] = (b0 + r < NM && k0 + c < K) ? H[(long long)(b0 + r) * K + k0 + c] : 0.0;
    }
    for (int q = t; q < BK * BN; q += 256) {
      const int r = q / BN, c = q % BN;
      Bs[r][c] = (k0 + r < K && i0 + c < N) ? cm[(long long)(k0 + r) * N + i0 + c] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < BK; ++kk) {
      const double a0 = As[kk][tr];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] += a0 * Bs[kk][tc + 16 * q];
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int b = b0 + tr, i = i0 + tc + 16 * q;
    if (b < NM && i < N) p0[(long long)b * N + i] = acc[q];
  }
}

// FP32 copies of the p0 differences the projection uses (taken in FP64):
// gx[b][i] = p0[b][min(i+1,N-1)] - p0[b][i], gy[b][i] = p0[b+1][i] - p0[b][i]
__global__ void k_kz0_grad(Spec s, const double *__restrict__ p0, float *__restrict__ gx, float *__restrict__ gy) {
  const int N = s.N, NM = s.NM;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= N * NM) return;
  const int b = q / N, i = q % N;
  const double v = p0[q];
  gx[q] = (float)(p0[(long long)b * N + min(i + 1, N - 1)] - v);
  gy[q] = b < NM - 1 ? (float)(p0[q + N] - v) : 0.f;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
// the split A (N = A B) of the two-pass FP32 kernels built for N, else 0
int xfft_split(int n) {
  switch (n) {
    case 812: return 29;  // 29 x 28
    case 510: return 17;  // 17 x 30
    case 190: return 19;  // 19 x 10 (ensemble boxes nx = 192)
    case 126: return 14;  // 14 x 9 (ensemble boxes nx = 128)
    default: return 0;
  }
}

static size_t xfft_line(int n, int split) {
  if (!split) return 2 * (size_t)n;
  const int B = n / split, SB = B | 1;
  return (size_t)(((n > split * SB ? n : split * SB) + 1) & ~1);
}

int dct_lines_per_cta(int n, int elem_bytes, bool inverse, int split) {
  // warps (complex lines) per CTA, as measured at 814 x 257 x 193: the FP32
  // inverse fills one SM's shared memory with up to 16 lines, the FP32
  // forward (its divergence loads want more CTAs in flight) takes three CTAs
  // of up to 4 lines per SM, FP64 (register-limited) two CTAs within 113 KB;
  // the two-pass kernels (80 registers, 24 warps per SM) take 6 lines per
  // CTA in both directions
  if (split) return elem_bytes == 8 ? 4 : 6;
  const size_t line = (size_t)n * 2 * elem_bytes * 2;  // ping-pong buffers of one complex line
  const size_t fixed = (size_t)n * 2 * elem_bytes * 2; // twiddle + DCT tables
  const size_t budget = elem_bytes == 8 ? 113 * 1024 : inverse ? 226 * 1024 : 75 * 1024;
  const int cap = elem_bytes == 8 ? 6 : inverse ? 16 : 4;
  int w = (int)((budget > fixed ? budget - fixed : 0) / line);
  if (w < 1) w = 1;
  if (w > cap) w = cap;
  // the whole allocation (with the reciprocal spacings and the mbarriers)
  // within the 227 KB a CTA may hold
  while (w > 1 && dct_smem_bytes(n, elem_bytes, w, split) > 227 * 1024) --w;
  return w;
}

int dct_max_lines(int elem_bytes, int split) { return split ? 8 : elem_bytes == 4 ? 16 : 8; }

// twiddle and DCT tables, the line buffers, the x reciprocal spacings as
// FP32 (forward) and one mbarrier per line (inverse, two-pass)
size_t dct_smem_bytes(int n, int elem_bytes, int warps, int split) {
  return (size_t)2 * elem_bytes * (2 * (size_t)n + (size_t)warps * xfft_line(n, split)) +
         4 * (size_t)((n + 3) / 4 * 4) + 8 * (size_t)warps;
}

// Register-resident odd butterflies raise the register count of the whole
// kernel to that of the largest radix compiled in, so the transform kernels
// are instantiated per largest radix class; radices above the class (and
// primes above 31) take the shared-memory summation path.
static int radix_class(const int *rad, int nst) {
  int mx = 2;
  for (int i = 0; i < nst; ++i)
    if (rad[i] <= 31) mx = rad[i] > mx ? rad[i] : mx;
  if (mx <= 7) return 7;
  if (mx <= 13) return 13;
  if (mx <= 19) return 19;
  if (mx <= 29) return 29;
  return 31;
}

template <typename T, class E>
static void launch_div_dct_e(const Geo &g, const Spec &s, const FftPlan<T> &pl, const T *U, const T *V, const T *W,
                             T *R, int nw, size_t sm, int grid, cudaStream_t st) {
  cudaFuncSetAttribute(k_div_dct<T, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  cudaFuncSetAttribute(k_div_dct<T, E>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  k_div_dct<T, E><<<grid, 32 * nw, sm, st>>>(g, s, pl, U, V, W, R);
}

template <typename T, class E>
static void launch_idct_e(const Geo &g, const Spec &s, const FftPlan<T> &pl, const T *R, T *p, int nw, size_t sm,
                          int grid, cudaStream_t st) {
  cudaFuncSetAttribute(k_idct<T, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  cudaFuncSetAttribute(k_idct<T, E>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  k_idct<T, E><<<grid, 32 * nw, sm, st>>>(g, s, pl, R, p);
}

template <typename T>
void launch_div_dct(const Geo &g, const Spec &s, const FftPlan<T> &pl, const T *U, const T *V, const T *W, T *R,
                    int nw_req, int xfft, cudaStream_t st) {
  int split = xfft != 1 ? xfft_split(s.N) : 0;
  if (sizeof(T) == 8 && split != 29) split = 0;  // FP64 two-pass built for N = 812 only
  const int nw = nw_req > 0 ? nw_req : dct_lines_per_cta(s.N, sizeof(T), false, split);
  const size_t sm = dct_smem_bytes(s.N, sizeof(T), nw, split);
  const int ncl = (s.NM * s.M + 1) / 2;  // complex lines
  const int grid = (ncl + nw - 1) / nw;
  if constexpr (sizeof(T) == 8) {
    if (split == 29) return launch_div_dct_e<T, TwoPassX<29, 28, T>>(g, s, pl, U, V, W, R, nw, sm, grid, st);
  }
  if constexpr (sizeof(T) == 4) {
    if (split == 29) return launch_div_dct_e<T, TwoPassX<29, 28>>(g, s, pl, U, V, W, R, nw, sm, grid, st);
    if (split == 17) return launch_div_dct_e<T, TwoPassX<17, 30>>(g, s, pl, U, V, W, R, nw, sm, grid, st);
    if (split == 19) return launch_div_dct_e<T, TwoPassX<19, 10>>(g, s, pl, U, V, W, R, nw, sm, grid, st);
    if (split == 14) return launch_div_dct_e<T, TwoPassX<14, 9>>(g, s, pl, U, V, W, R, nw, sm, grid, st);
  }
  switch (radix_class(pl.rad, pl.nst)) {
    case 7: launch_div_dct_e<T, StockhamX<T, 7>>(g, s, pl, U, V, W, R, nw, sm, grid, st); break;
    case 13: launch_div_dct_e<T, StockhamX<T, 13>>(g, s, pl, U, V, W, R, nw, sm, grid, st); break;
    case 19: launch_div_dct_e<T, StockhamX<T, 19>>(g, s, pl, U, V, W, R, nw, sm, grid, st); break;
    case 29: launch_div_dct_e<T, StockhamX<T, 29>>(g, s, pl, U, V, W, R, nw, sm, grid, st); break;
    default: launch_div_dct_e<T, StockhamX<T, 31>>(g, s, pl, U, V, W, R, nw, sm, grid, st); break;
  }
}

template <int A, int B, typename T>
static void launch_idct2(const Geo &g, const Spec &s, const FftPlan<T> &pl, const T *R, T *p, int nw, size_t sm,
                         int grid, int *err, cudaStream_t st) {
  cudaFuncSetAttribute(k_idct2<A, B, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  cudaFuncSetAttribute(k_idct2<A, B, T>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  k_idct2<A, B, T><<<grid, 32 * nw, sm, st>>>(g, s, pl, R, p, err);
}

// the two rows of the bulk copy fit one line buffer of the two-pass kernel
static bool idct2_fits(const Spec &s, int split) {
  return (size_t)s.rx + (size_t)((s.N + 3) & ~3) <= 2 * xfft_line(s.N, split) && s.rx % 4 == 0;
}

template <typename T>
void launch_idct(const Geo &g, const Spec &s, const FftPlan<T> &pl, const T *R, T *p, int nw_req, int xfft, int *err,
                 cudaStream_t st) {
  int split = xfft != 1 ? xfft_split(s.N) : 0;
  if (sizeof(T) == 8 && split != 29) split = 0;  // FP64 two-pass built for N = 812 only
  const int nw = nw_req > 0 ? nw_req : dct_lines_per_cta(s.N, sizeof(T), true, split);
  const size_t sm = dct_smem_bytes(s.N, sizeof(T), nw, split);
  const int ncl = (s.NM * s.M + 1) / 2;
  const int grid = (ncl + nw - 1) / nw;
  const bool fused = idct2_fits(s, split) && (reinterpret_cast<uintptr_t>(R) & 15) == 0;
  if constexpr (sizeof(T) == 8) {
    if (split == 29 && fused) return launch_idct2<29, 28, T>(g, s, pl, R, p, nw, sm, grid, err, st);
    if (split == 29) return launch_idct_e<T, TwoPassX<29, 28, T>>(g, s, pl, R, p, nw, sm, grid, st);
  }
  if constexpr (sizeof(T) == 4) {
    if (split == 29 && fused) return launch_idct2<29, 28, T>(g, s, pl, R, p, nw, sm, grid, err, st);
    if (split == 17 && fused) return launch_idct2<17, 30, T>(g, s, pl, R, p, nw, sm, grid, err, st);
    if (split == 19 && fused) return launch_idct2<19, 10, T>(g, s, pl, R, p, nw, sm, grid, err, st);
    if (split == 14 && fused) return launch_idct2<14, 9, T>(g, s, pl, R, p, nw, sm, grid, err, st);
    if (split == 29) return launch_idct_e<T, TwoPassX<29, 28>>(g, s, pl, R, p, nw, sm, grid, st);
    if (split == 17) return launch_idct_e<T, TwoPassX<17, 30>>(g, s, pl, R, p, nw, sm, grid, st);
    if (split == 19) return launch_idct_e<T, TwoPassX<19, 10>>(g, s, pl, R, p, nw, sm, grid, st);
    if (split == 14) return launch_idct_e<T, TwoPassX<14, 9>>(g, s, pl, R, p, nw, sm, grid, st);
  }
  switch (radix_class(pl.rad, pl.nst)) {
    case 7: launch_idct_e<T, StockhamX<T, 7>>(g, s, pl, R, p, nw, sm, grid, st); break;
    case 13: launch_idct_e<T, StockhamX<T, 13>>(g, s, pl, R, p, nw, sm, grid, st); break;
    case 19: launch_idct_e<T, StockhamX<T, 19>>(g, s, pl, R, p, nw, sm, grid, st); break;
    case 29: launch_idct_e<T, StockhamX<T, 29>>(g, s, pl, R, p, nw, sm, grid, st); break;
    default: launch_idct_e<T, StockhamX<T, 31>>(g, s, pl, R, p, nw, sm, grid, st); break;
  }
}

template <typename T, int RK>
static void launch_dft_z_rk(const Spec &s, const T *R, T2<T> *C, const T2<T> *tz, int inverse, cudaStream_t st) {
  constexpr int TW = 32 * Vec16<T>::n;
  if (!inverse) {
    dim3 grid((s.N + TW - 1) / TW, s.NM, (s.MH + 8 * RK - 1) / (8 * RK));
    const size_t sm = (size_t)s.M * TW * sizeof(T);
    cudaFuncSetAttribute(k_dft_z_fwd<T, RK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaFuncSetAttribute(k_dft_z_fwd<T, RK>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    k_dft_z_fwd<T, RK><<<grid, 256, sm, st>>>(s, R, C, tz);
  } else {
    const int npairs = s.M / 2 + 1;
    dim3 grid((s.N + TW - 1) / TW, s.NM, (npairs + 8 * RK - 1) / (8 * RK));
    const size_t sm = (size_t)s.MH * TW * sizeof(T2<T>);
    cudaFuncSetAttribute(k_dft_z_inv<T, RK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaFuncSetAttribute(k_dft_z_inv<T, RK>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    k_dft_z_inv<T, RK><<<grid, 256, sm, st>>>(s, C, const_cast<T *>(R), tz);
  }
}

template <typename T>
void launch_dft_z(const Spec &s, const T *R, T2<T> *C, const T2<T> *tz, int inverse, int rk, cudaStream_t st) {
  if (rk == 4) launch_dft_z_rk<T, 4>(s, R, C, tz, inverse, st);
  else launch_dft_z_rk<T, 8>(s, R, C, tz, inverse, st);
}

template <typename T>
void launch_thomas(const Spec &s, T2<T> *C, const double *piv, const double *dl, const double *du, double *H0,
                   int klow, cudaStream_t st) {
  // rows in flight per thread: 24 in FP32 (the row loads bypass L1, whose
  // capacity capped the ring at 12 rows: 0.75 -> 0.67 ms per step at
  // 814 x 257 x 193; more rows would cost the one-wave occupancy), 16 in FP64
  dim3 grid((s.N + 127) / 128, s.MH);  // 128 kx of one kz per CTA
  k_thomas<T, sizeof(T) == 4 ? 24 : 16><<<grid, 128, 0, st>>>(s, C, piv, dl, du, H0, klow);
}

void launch_thomas_factors(const Spec &s, double *piv, const double *dd, const double *dl, const double *du,
                           const double *kxx, const double *kzz, cudaStream_t st) {
  k_thomas_factors<<<dim3((s.N + 127) / 128, s.MH), 128, 0, st>>>(s, piv, dd, dl, du, kxx, kzz);
}

void launch_kz0_idct(const Spec &s, const double *H0, int klow, const double *cm, double *p0, float *grad,
                     cudaStream_t st) {
  k_kz0_idct<<<dim3((s.N + 63) / 64, (s.NM + 15) / 16), 256, 0, st>>>(s, H0, klow, cm, p0);
  k_kz0_grad<<<(s.N * s.NM + 255) / 256, 256, 0, st>>>(s, p0, grad, grad + (long long)s.N * s.NM);
}

#define BLGPU_SPEC_INST(T)                                                                                        \
  template void launch_div_dct<T>(const Geo &, const Spec &, const FftPlan<T> &, const T *, const T *, const T *, \
                                  T *, int, int, cudaStream_t);                                                   \
  template void launch_idct<T>(const Geo &, const Spec &, const FftPlan<T> &, const T *, T *, int, int, int *,   \
                               cudaStream_t);                                                                    \
  template void launch_dft_z<T>(const Spec &, const T *, T2<T> *, const T2<T> *, int, int, cudaStream_t);        \
  template void launch_thomas<T>(const Spec &, T2<T> *, const double *, const double *, const double *,          \
                                 double *, int, cudaStream_t);
BLGPU_SPEC_INST(double)
BLGPU_SPEC_INST(float)

}  // namespace blgpu
