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
  T cs[H], sn[H];
#pragma unroll
  for (int q = 1; q <= H; ++q) {
    T2<T> w = tw[q * stride];
    cs[q - 1] = w.x;
    sn[q - 1] = -w.y;  // sin(2 pi q / R)
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
      const T c = (m <= H) ? cs[m - 1] : cs[R - m - 1];
      const T sv = (m <= H) ? sn[m - 1] : -sn[R - m - 1];
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

// any radix, outputs by direct summation from shared memory (large primes)
template <typename T, bool INV>
__device__ __forceinline__ void bf_loop(const T2<T> *in, T2<T> *out, int R, int jj, int nb, int tstep, int idxD,
                                        int Ns, int n, const T2<T> *tw) {
  const int stride = n / R;
  for (int k = 0; k < R; ++k) {
    const int e = tstep + k * stride;
    T ax = 0, ay = 0;
    int idx = 0;
    for (int q = 0; q < R; ++q) {
      T2<T> v = twm<T, INV>(in[jj + q * nb], tw[idx]);
      ax += v.x;
      ay += v.y;
      idx += e;
      if (idx >= n) idx -= n;
    }
    out[idxD + k * Ns] = mk<T>(ax, ay);
  }
}

// L lines of length n in shared memory; returns the buffer holding the result
template <typename T, bool INV>
__device__ T2<T> *fft_lines(T2<T> *a, T2<T> *b, const FftPlan<T> &pl, int L, const T2<T> *tw) {
  const int n = pl.n;
  int Ns = 1;
  const int tid = threadIdx.x, nthr = blockDim.x;
  for (int s = 0; s < pl.nst; ++s) {
    const int R = pl.rad[s];
    const int nb = n / R;
    const int total = nb * L;
    const int tsc = n / (Ns * R);
    for (int w = tid; w < total; w += nthr) {
      const int line = w / nb, jj = w - line * nb;
      const T2<T> *in = a + line * n;
      T2<T> *out = b + line * n;
      const int jm = jj % Ns;
      const int tstep = jm * tsc;
      const int idxD = (jj - jm) * R + jm;
      switch (R) {
        case 2: bf2<T, INV>(in, out, jj, nb, tstep, idxD, Ns, tw); break;
        case 3: bf3<T, INV>(in, out, jj, nb, tstep, idxD, Ns, tw); break;
        case 4: bf4<T, INV>(in, out, jj, nb, tstep, idxD, Ns, tw); break;
        case 5: bf_odd<5, T, INV>(in, out, jj, nb, tstep, idxD, Ns, n, tw); break;
        case 7: bf_odd<7, T, INV>(in, out, jj, nb, tstep, idxD, Ns, n, tw); break;
        case 11: bf_odd<11, T, INV>(in, out, jj, nb, tstep, idxD, Ns, n, tw); break;
        case 13: bf_odd<13, T, INV>(in, out, jj, nb, tstep, idxD, Ns, n, tw); break;
        case 17: bf_odd<17, T, INV>(in, out, jj, nb, tstep, idxD, Ns, n, tw); break;
        case 19: bf_odd<19, T, INV>(in, out, jj, nb, tstep, idxD, Ns, n, tw); break;
        case 23: bf_odd<23, T, INV>(in, out, jj, nb, tstep, idxD, Ns, n, tw); break;
        case 29: bf_odd<29, T, INV>(in, out, jj, nb, tstep, idxD, Ns, n, tw); break;
        case 31: bf_odd<31, T, INV>(in, out, jj, nb, tstep, idxD, Ns, n, tw); break;
        default: bf_loop<T, INV>(in, out, R, jj, nb, tstep, idxD, Ns, n, tw); break;
      }
    }
    __syncthreads();
    T2<T> *t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

// ---------------------------------------------------------------------------
// divergence + DCT-II in x.  One CTA transforms 2L real lines (b, k').
// R[q][kx], q = b*M + k', holds c_k = sum_i f_i cos(pi k (2i+1) / (2N)).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_div_dct(Geo g, Spec s, FftPlan<T> pl, const T *__restrict__ U,
                                                 const T *__restrict__ V, const T *__restrict__ W,
                                                 T *__restrict__ R, double *__restrict__ dc_sum, int L) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = s.N;
  T2<T> *tw = reinterpret_cast<T2<T> *>(smem_raw);
  T2<T> *post = tw + N;
  T2<T> *bufA = post + N;
  T2<T> *bufB = bufA + (size_t)L * N;
  const int nlines = s.NM * s.M;
  const int q0 = blockIdx.x * 2 * L;
  for (int t = threadIdx.x; t < N; t += blockDim.x) {
    tw[t] = pl.tw[t];
    post[t] = pl.post[t];
  }
  // divergence (projection.f90:42-44) for i = 2..nx-1, Makhoul order
  const int tot = L * N;
  for (int w = threadIdx.x; w < tot; w += blockDim.x) {
    const int l = w / N, ip = w - l * N;
    T fv[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int q = q0 + 2 * l + h;
      T f = 0;
      if (q < nlines) {
        const int b = q / s.M, kp = q - b * s.M;
        const int i = ip + 2, j = b + 2, k = kp + 2;
        const long long c = bidx(g, i, j, k);
        f = (__ldg(U + c) - __ldg(U + c - 1)) / (T)g.ax.F[i] + (__ldg(V + c) - __ldg(V + c - g.px)) / (T)g.ay.F[j] +
            (__ldg(W + c) - __ldg(W + c - g.plane)) / (T)g.az.F[k];
      }
      fv[h] = f;
    }
    const int pos = (ip & 1) ? (N - 1 - (ip >> 1)) : (ip >> 1);
    bufA[l * N + pos] = mk<T>(fv[0], fv[1]);
  }
  __syncthreads();
  if (dc_sum) {  // FP64 line sums for the zero wavenumber (mixed form)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int l = warp; l < L; l += nw) {
      double sa = 0.0, sb = 0.0;
      for (int t = lane; t < N; t += 32) {
        T2<T> v = bufA[l * N + t];
        sa += (double)v.x;
        sb += (double)v.y;
      }
      for (int o = 16; o > 0; o >>= 1) {
        sa += __shfl_xor_sync(0xffffffffu, sa, o);
        sb += __shfl_xor_sync(0xffffffffu, sb, o);
      }
      if (lane == 0) {
        const int q = q0 + 2 * l;
        if (q < nlines) dc_sum[q] = sa;
        if (q + 1 < nlines) dc_sum[q + 1] = sb;
      }
    }
  }
  T2<T> *res = fft_lines<T, false>(bufA, bufB, pl, L, tw);
  // untangle the two real lines and apply the DCT twiddle
  for (int w = threadIdx.x; w < tot; w += blockDim.x) {
    const int l = w / N, k = w - l * N;
    const T2<T> z = res[l * N + k];
    const T2<T> zr = res[l * N + (k == 0 ? 0 : N - k)];
    // V_A = (Z_k + conj Z_{N-k})/2, V_B = (Z_k - conj Z_{N-k})/(2i)
    const T2<T> va = mk<T>((T)0.5 * (z.x + zr.x), (T)0.5 * (z.y - zr.y));
    const T2<T> vb = mk<T>((T)0.5 * (z.y + zr.y), (T)0.5 * (zr.x - z.x));
    const T2<T> p = post[k];
    const int q = q0 + 2 * l;
    if (q < nlines) R[(long long)q * s.rx + k] = p.x * va.x - p.y * va.y;
    if (q + 1 < nlines) R[(long long)(q + 1) * s.rx + k] = p.x * vb.x - p.y * vb.y;
  }
}

// ---------------------------------------------------------------------------
// inverse DCT in x + box write of rhs_p (with the copies of
// apply_periodic_z_pressure: rhs_p(nxg-1,:,:) = rhs_p(nxg-2,:,:) and
// rhs_p(2:nxg-1,:,nzp+2) = rhs_p(2:nxg-1,:,2)).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_idct(Geo g, Spec s, FftPlan<T> pl, const T *__restrict__ R,
                                              T *__restrict__ p, int L) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = s.N;
  T2<T> *tw = reinterpret_cast<T2<T> *>(smem_raw);
  T2<T> *post = tw + N;
  T2<T> *bufA = post + N;
  T2<T> *bufB = bufA + (size_t)L * N;
  const int nlines = s.NM * s.M;
  const int q0 = blockIdx.x * 2 * L;
  for (int t = threadIdx.x; t < N; t += blockDim.x) {
    tw[t] = pl.tw[t];
    post[t] = pl.post[t];
  }
  __syncthreads();
  const int tot = L * N;
  for (int w = threadIdx.x; w < tot; w += blockDim.x) {
    const int l = w / N, k = w - l * N;
    const int q = q0 + 2 * l;
    T xa = 0, xan = 0, xb = 0, xbn = 0;
    if (q < nlines) {
      xa = R[(long long)q * s.rx + k];
      xan = k ? R[(long long)q * s.rx + (N - k)] : (T)0;
    }
    if (q + 1 < nlines) {
      xb = R[(long long)(q + 1) * s.rx + k];
      xbn = k ? R[(long long)(q + 1) * s.rx + (N - k)] : (T)0;
    }
    // V_k = exp(+i pi k/2N) (X_k - i X_{N-k});  Z = V_A + i V_B
    const T2<T> e = mk<T>(post[k].x, -post[k].y);
    const T2<T> va = cmul<T>(e, mk<T>(xa, -xan));
    const T2<T> vb = cmul<T>(e, mk<T>(xb, -xbn));
    bufA[l * N + k] = mk<T>(va.x - vb.y, va.y + vb.x);
  }
  __syncthreads();
  T2<T> *res = fft_lines<T, true>(bufA, bufB, pl, L, tw);
  const T inv = (T)1 / (T)N;
  for (int w = threadIdx.x; w < tot; w += blockDim.x) {
    const int l = w / N, ip = w - l * N;
    const int pos = (ip & 1) ? (N - 1 - (ip >> 1)) : (ip >> 1);
    const T2<T> z = res[l * N + pos];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int q = q0 + 2 * l + h;
      if (q >= nlines) continue;
      const int b = q / s.M, kp = q - b * s.M;
      const T val = (h ? z.y : z.x) * inv;
      const long long c = bidx(g, ip + 2, b + 2, kp + 2);
      p[c] = val;
      if (ip == N - 1) p[c + 1] = val;  // i = nxg-1 copy
      if (kp == 0) {
        const long long cz = c + (long long)s.M * g.plane;  // k = nzp+2
        p[cz] = val;
        if (ip == N - 1) p[cz + 1] = val;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// real DFT in z over the half spectrum, direct summation.
// forward:  C[b][kz][kx], kz = 0..MH-1, from R[b][k'][kx]
// inverse:  R[b][k'][kx] = (1/M) sum over the Hermitian spectrum
// ztab[m] = (cos(2 pi m/M), sin(2 pi m/M)), m = 0..M-1
// One CTA: 32 kx lanes x 8 warps; a thread accumulates RPT outputs.
// ---------------------------------------------------------------------------
template <typename T, int RPT>
__global__ void __launch_bounds__(256) k_dft_z_fwd(Spec s, const T *__restrict__ R, T2<T> *__restrict__ C,
                                                   const T2<T> *__restrict__ ztab) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int M = s.M, MH = s.MH;
  T2<T> *tab = reinterpret_cast<T2<T> *>(smem_raw);
  T *f = reinterpret_cast<T *>(tab + M);  // [M][32]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int b = blockIdx.y;
  const int kx = blockIdx.x * 32 + lane;
  const bool ok = kx < s.N;
  for (int t = threadIdx.x; t < M; t += blockDim.x) tab[t] = ztab[t];
  for (int kp = warp; kp < M; kp += 8)
    f[kp * 32 + lane] = ok ? R[((long long)b * M + kp) * s.rx + kx] : (T)0;
  __syncthreads();
  const int H = (M - 1) / 2;
  const bool even = (M & 1) == 0;
  for (int base = warp; base < MH; base += 8 * RPT) {
    T re[RPT], im[RPT];
    int kz[RPT], m[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      kz[r] = base + 8 * r;
      re[r] = f[lane];
      im[r] = 0;
      m[r] = 0;
    }
    int inc[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) inc[r] = kz[r] < MH ? kz[r] : 0;  // idle slots stay at m = 0
    for (int k = 1; k <= H; ++k) {
      const T fk = f[k * 32 + lane], fm = f[(M - k) * 32 + lane];
      const T a = fk + fm, bb = fk - fm;
#pragma unroll
      for (int r = 0; r < RPT; ++r) {
        m[r] += inc[r];
        if (m[r] >= M) m[r] -= M;
        const T2<T> cs = tab[m[r]];
        re[r] += a * cs.x;
        im[r] -= bb * cs.y;
      }
    }
    if (ok) {
#pragma unroll
      for (int r = 0; r < RPT; ++r) {
        if (kz[r] >= MH) continue;
        T rr = re[r];
        if (even) rr += (kz[r] & 1) ? -f[(M / 2) * 32 + lane] : f[(M / 2) * 32 + lane];
        C[((long long)b * MH + kz[r]) * s.rx + kx] = mk<T>(rr, im[r]);
      }
    }
  }
}

template <typename T, int RPT>
__global__ void __launch_bounds__(256) k_dft_z_inv(Spec s, const T2<T> *__restrict__ C, T *__restrict__ R,
                                                   const T2<T> *__restrict__ ztab) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int M = s.M, MH = s.MH;
  T2<T> *tab = reinterpret_cast<T2<T> *>(smem_raw);
  T2<T> *c = tab + M;  // [MH][32]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int b = blockIdx.y;
  const int kx = blockIdx.x * 32 + lane;
  const bool ok = kx < s.N;
  for (int t = threadIdx.x; t < M; t += blockDim.x) tab[t] = ztab[t];
  for (int kz = warp; kz < MH; kz += 8) c[kz * 32 + lane] = ok ? C[((long long)b * MH + kz) * s.rx + kx] : mk<T>(0, 0);
  __syncthreads();
  const int H = (M - 1) / 2;  // conjugate pairs kz = 1..H
  const bool even = (M & 1) == 0;
  const T c0 = c[lane].x;
  const T nyq = even ? c[(M / 2) * 32 + lane].x : (T)0;
  const T invM = (T)1 / (T)M;
  const int npairs = M / 2 + 1;  // p = 0..M/2 covers every output once with its partner M-p
  for (int base = warp; base < npairs; base += 8 * RPT) {
    T P[RPT], Q[RPT];
    int pp[RPT], m[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      pp[r] = base + 8 * r;
      P[r] = 0;
      Q[r] = 0;
      m[r] = 0;
    }
    int inc[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) inc[r] = pp[r] < npairs ? pp[r] : 0;  // idle slots stay at m = 0
    for (int kz = 1; kz <= H; ++kz) {
      const T2<T> v = c[kz * 32 + lane];
#pragma unroll
      for (int r = 0; r < RPT; ++r) {
        m[r] += inc[r];
        if (m[r] >= M) m[r] -= M;
        const T2<T> cs = tab[m[r]];
        P[r] += v.x * cs.x;
        Q[r] += v.y * cs.y;
      }
    }
    if (ok) {
#pragma unroll
      for (int r = 0; r < RPT; ++r) {
        const int p = pp[r];
        if (p >= npairs) continue;
        const T ny = (p & 1) ? -nyq : nyq;
        const T lo = (c0 + (T)2 * (P[r] - Q[r]) + ny) * invM;
        R[((long long)b * M + p) * s.rx + kx] = lo;
        const int pm = M - p;
        if (pm != p && pm < M) {
          const T hi = (c0 + (T)2 * (P[r] + Q[r]) + ny) * invM;
          R[((long long)b * M + pm) * s.rx + kx] = hi;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Tridiagonal solve in y for every (kx, kz) mode, FP64 arithmetic.
// Row b (= j-2) of the operator: diag dd[b] + kxx[kx] + kzz[kz] (row 0 of
// mode (0,0) scaled by 3/2, initialization.f90:454), sub dl[b] = Dyy(j,j-1),
// super du[b] = Dyy(j,j+1).  Forward sweep writes g in place and the inverse
// pivots to piv; the backward sweep reads them back.
// dc_in/dc_out (mixed form): the (0,0) mode is solved from FP64 line sums
// and its solution kept in FP64 (per-row constant), not in C.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_thomas(Spec s, T2<T> *__restrict__ C, double *__restrict__ piv,
                                                const double *__restrict__ dd, const double *__restrict__ dl,
                                                const double *__restrict__ du, const double *__restrict__ kxx,
                                                const double *__restrict__ kzz, const double *__restrict__ dc_in,
                                                double *__restrict__ dc_out) {
  const int kx = blockIdx.x * 32 + (threadIdx.x & 31);
  const int kz = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (kx >= s.N || kz >= s.MH) return;
  const int NM = s.NM;
  const long long rs = (long long)s.MH * s.rx;  // stride between rows b
  const long long base = (long long)kz * s.rx + kx;
  const double kk = kxx[kx];
  const double kzv = kzz[kz];
  const bool zero = (kx == 0 && kz == 0);
  if (zero && dc_in) {
    // mixed form: zero wavenumber from FP64 line sums, solution kept in FP64
    double dprev = 0.0, gr = 0.0;
    for (int b = 0; b < NM; ++b) {
      double r = dc_in[b];
      double d = (dd[b] + kk) + kzv;
      if (b == 0) d = 3.0 / 2.0 * d;
      if (b > 0) {
        const double w = dl[b] / dprev;
        d = d - w * du[b - 1];
        r = r - w * gr;
      }
      dprev = d;
      gr = r;
      dc_out[b] = r;
      piv[base + b * rs] = 1.0 / d;
    }
    double x = dc_out[NM - 1] * piv[base + (NM - 1) * rs];
    dc_out[NM - 1] = x;
    for (int b = NM - 2; b >= 0; --b) {
      x = (dc_out[b] - du[b] * x) * piv[base + b * rs];
      dc_out[b] = x;
    }
    const double nrm = 1.0 / ((double)s.N * (double)s.M);
    for (int b = 0; b < NM; ++b) dc_out[b] *= nrm;
    for (int b = 0; b < NM; ++b) C[base + b * rs] = mk<T>(0, 0);
    return;
  }
  double dprev = 1.0, gx = 0.0, gy = 0.0;
  for (int b = 0; b < NM; ++b) {
    const long long a = base + b * rs;
    const T2<T> r = C[a];
    double rx = (double)r.x, ry = (double)r.y;
    double d = (dd[b] + kk) + kzv;
    if (zero && b == 0) d = 3.0 / 2.0 * d;
    if (b > 0) {
      const double w = dl[b] / dprev;
      d = d - w * du[b - 1];
      rx = rx - w * gx;
      ry = ry - w * gy;
    }
    dprev = d;
    gx = rx;
    gy = ry;
    C[a] = mk<T>((T)rx, (T)ry);
    piv[a] = 1.0 / d;
  }
  double xx = gx * piv[base + (NM - 1) * rs], xy = gy * piv[base + (NM - 1) * rs];
  C[base + (NM - 1) * rs] = mk<T>((T)xx, (T)xy);
  for (int b = NM - 2; b >= 0; --b) {
    const long long a = base + b * rs;
    const T2<T> gv = C[a];
    const double pv = piv[a];
    xx = ((double)gv.x - du[b] * xx) * pv;
    xy = ((double)gv.y - du[b] * xy) * pv;
    C[a] = mk<T>((T)xx, (T)xy);
  }
}

// per-row sums of the FP64 line sums (mixed form zero wavenumber), fixed order
__global__ void k_dc_rows(Spec s, const double *__restrict__ lines, double *__restrict__ rows) {
  const int b = blockIdx.x, lane = threadIdx.x;
  double acc = 0.0;
  for (int kp = lane; kp < s.M; kp += 32) acc += lines[(long long)b * s.M + kp];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) rows[b] = acc;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
int dct_lines_per_cta(int n, int elem_bytes) {
  const size_t line = (size_t)n * 2 * elem_bytes;   // one complex line
  const size_t budget = 100 * 1024;                 // two CTAs per SM
  size_t fixed = 2 * line;                          // twiddle + DCT tables
  int L = (int)((budget > fixed ? budget - fixed : 0) / (2 * line));
  if (L < 1) L = 1;
  if (L > 8) L = 8;
  return L;
}

size_t dct_smem_bytes(int n, int elem_bytes, int lines) {
  return (size_t)n * 2 * elem_bytes * (2 + 2 * (size_t)lines);
}

template <typename T>
void launch_div_dct(const Geo &g, const Spec &s, const FftPlan<T> &pl, const T *U, const T *V, const T *W, T *R,
                    double *dc_sum, cudaStream_t st) {
  const int L = dct_lines_per_cta(s.N, sizeof(T));
  const size_t sm = dct_smem_bytes(s.N, sizeof(T), L);
  const int nlines = s.NM * s.M;
  const int grid = (nlines + 2 * L - 1) / (2 * L);
  cudaFuncSetAttribute(k_div_dct<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_div_dct<T><<<grid, 256, sm, st>>>(g, s, pl, U, V, W, R, dc_sum, L);
}

template <typename T>
void launch_idct(const Geo &g, const Spec &s, const FftPlan<T> &pl, const T *R, T *p, cudaStream_t st) {
  const int L = dct_lines_per_cta(s.N, sizeof(T));
  const size_t sm = dct_smem_bytes(s.N, sizeof(T), L);
  const int nlines = s.NM * s.M;
  const int grid = (nlines + 2 * L - 1) / (2 * L);
  cudaFuncSetAttribute(k_idct<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_idct<T><<<grid, 256, sm, st>>>(g, s, pl, R, p, L);
}

template <typename T>
void launch_dft_z(const Spec &s, const T *R, T2<T> *C, const T2<T> *ztab, int inverse, cudaStream_t st) {
  constexpr int RPT = 8;
  dim3 grid((s.N + 31) / 32, s.NM);
  if (!inverse) {
    const size_t sm = (size_t)s.M * sizeof(T2<T>) + (size_t)s.M * 32 * sizeof(T);
    cudaFuncSetAttribute(k_dft_z_fwd<T, RPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_dft_z_fwd<T, RPT><<<grid, 256, sm, st>>>(s, R, C, ztab);
  } else {
    const size_t sm = (size_t)s.M * sizeof(T2<T>) + (size_t)s.MH * 32 * sizeof(T2<T>);
    cudaFuncSetAttribute(k_dft_z_inv<T, RPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_dft_z_inv<T, RPT><<<grid, 256, sm, st>>>(s, C, const_cast<T *>(R), ztab);
  }
}

template <typename T>
void launch_thomas(const Spec &s, T2<T> *C, double *piv, const double *dd, const double *dl, const double *du,
                   const double *kxx, const double *kzz, const double *dc_lines, double *dc_rows, double *dc_out,
                   cudaStream_t st) {
  if (dc_lines) k_dc_rows<<<s.NM, 32, 0, st>>>(s, dc_lines, dc_rows);
  dim3 grid((s.N + 31) / 32, (s.MH + 7) / 8);
  k_thomas<T><<<grid, 256, 0, st>>>(s, C, piv, dd, dl, du, kxx, kzz, dc_lines ? dc_rows : nullptr, dc_out);
}

#define BLGPU_SPEC_INST(T)                                                                                        \
  template void launch_div_dct<T>(const Geo &, const Spec &, const FftPlan<T> &, const T *, const T *, const T *, \
                                  T *, double *, cudaStream_t);                                                   \
  template void launch_idct<T>(const Geo &, const Spec &, const FftPlan<T> &, const T *, T *, cudaStream_t);     \
  template void launch_dft_z<T>(const Spec &, const T *, T2<T> *, const T2<T> *, int, cudaStream_t);             \
  template void launch_thomas<T>(const Spec &, T2<T> *, double *, const double *, const double *,                \
                                 const double *, const double *, const double *, const double *, double *,       \
                                 double *, cudaStream_t);
BLGPU_SPEC_INST(double)
BLGPU_SPEC_INST(float)

}  // namespace blgpu
