// cufft_path.cu -- the cuFFT comparison path of the Poisson solve
// (blgpu_config.poisson = BLGPU_POISSON_CUFFT).
//
// It follows solve_poisson_gpu (projection.f90:93-204) with the plans of
// cufft_init_plans (cufft_solver.f90:26-62), so that the hand-written
// transforms of spectral.cu can be timed against the library on the same
// box:
//   k_cf_pack      divergence (projection.f90:38-47) packed as the symmetric
//                  2N extension plane(ii) = plane(2N+1-ii) = rhs_p(ii+1)
//                  (projection.f90:111-119), complex with zero imaginary part;
//   plan_2d        cuFFT forward over (2N, M) per y-row, batch NM (:122-124);
//   k_cf_extract   hat(i,b,k) = plane(i,k,b) * exp(-i pi (i-1)/(2N)) (:127-134);
//   k_cf_thomas    the y-solve of every (i,k) mode on hat (:137-150) with the
//                  context's inverse pivots (the kz and M-kz modes share them:
//                  kzz is even in kz);
//   plan_zi        cuFFT inverse in z, stride N*NM, batch N*NM (:156-158);
//   k_cf_untwiddle plane(ii) = hat(ii) conj(twiddle), plane(N+1) = 0 and the
//                  Hermitian extension plane(2N+2-ii) = conj(plane(ii))
//                  (:162-187), one pass instead of three;
//   plan_xi        cuFFT inverse over 2N, batch M*NM (:190-192);
//   k_cf_unpack    rhs_p = Re(plane) / (2N M) into the box, with the x-Neumann
//                  and z-periodic copies of apply_periodic_z_pressure
//                  (:195-202, :295-303).
// FP64 uses Z2Z plans, the mixed form C2C plans; in the mixed form the
// y-solve keeps the kz = 0, kx < klow modes in FP64 exactly as the native
// path does (they go to the same FP64 pressure plane).  The spectral arrays
// hold 2x the native DCT coefficients (the 2N-point transform of the even
// extension), which the y-solve is linear in; the FP64 modes of the mixed
// form are halved on the way into the native FP64 plane.
#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdio>

#include "divergence.cuh"
#include "kernels.cuh"

namespace blgpu {

namespace {

template <typename T> using C2 = typename vec2<T>::type;

template <typename T> __device__ __forceinline__ C2<T> cm(C2<T> a, C2<T> b) {
  C2<T> r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename T> __device__ __forceinline__ C2<T> cmc(C2<T> a, C2<T> b) {  // a * conj(b)
  C2<T> r;
  r.x = a.x * b.x + a.y * b.y;
  r.y = a.y * b.x - a.x * b.y;
  return r;
}

// plane[b][k'][0..2N): thread (ii, k', b), ii < N
template <typename T>
__global__ void k_cf_pack(Geo g, Spec s, const T *__restrict__ U, const T *__restrict__ V, const T *__restrict__ W,
                          C2<T> *__restrict__ plane) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int kp = blockIdx.y, b = blockIdx.z;
  if (ii >= s.N) return;
  const int i = ii + 2, j = b + 2, k = kp + 2;
  const T d = div_at<T>(g, U, V, W, bidx(g, i, j, k), i, j, k);
  C2<T> v;
  v.x = d;
  v.y = (T)0;
  C2<T> *row = plane + ((long long)b * s.M + kp) * (2LL * s.N);
  row[ii] = v;
  row[2 * s.N - 1 - ii] = v;
}

// hat[k][b][i] = plane[b][k][i] * post[i]
template <typename T>
__global__ void k_cf_extract(Spec s, const C2<T> *__restrict__ plane, const C2<T> *__restrict__ post,
                             C2<T> *__restrict__ hat) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y, b = blockIdx.z;
  if (i >= s.N) return;
  hat[((long long)k * s.NM + b) * s.N + i] = cm<T>(plane[((long long)b * s.M + k) * (2LL * s.N) + i], post[i]);
}

// y-solve of mode (i, k) on hat rows b (stride N): the recurrences of
// k_thomas (g_b = r_b - dl_b piv_{b-1} g_{b-1}, x_b = (g_b - du_b x_{b+1})
// piv_b) in FP64 arithmetic; H0 (mixed form): the kz = 0, i < klow modes
// go to H0[b][i], halved, and are zeroed in hat
template <typename T>
__global__ void __launch_bounds__(128) k_cf_thomas(Spec s, C2<T> *__restrict__ hat, const double *__restrict__ piv,
                                                   const double *__restrict__ dl, const double *__restrict__ du,
                                                   double *__restrict__ H0, int klow) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (i >= s.N) return;
  const int NM = s.NM;
  const int kh = k < s.MH ? k : s.M - k;
  const long long ps = (long long)s.MH * s.rx;
  const double *pv = piv + (long long)kh * s.rx + i;
  C2<T> *h = hat + (long long)k * NM * s.N + i;
  const long long hs = s.N;
  const bool kz0 = H0 && k == 0 && i < klow;
  double gx = 0.0, gy = 0.0, rprev = 0.0;
#pragma unroll 4
  for (int b = 0; b < NM; ++b) {
    const C2<T> c = h[b * hs];
    double rx = (double)c.x, ry = (double)c.y;
    if (b > 0) {
      const double w = dl[b] * rprev;
      rx = rx - w * gx;
      ry = ry - w * gy;
    }
    rprev = pv[b * ps];
    gx = rx;
    gy = ry;
    if (kz0) H0[(long long)b * klow + i] = rx;
    else {
      C2<T> o;
      o.x = (T)rx;
      o.y = (T)ry;
      h[b * hs] = o;
    }
  }
  double xx = 0.0, xy = 0.0;
#pragma unroll 4
  for (int b = NM - 1; b >= 0; --b) {
    double cx, cy;
    if (kz0) {
      cx = H0[(long long)b * klow + i];
      cy = 0.0;
    } else {
      const C2<T> c = h[b * hs];
      cx = (double)c.x;
      cy = (double)c.y;
    }
    const double p = pv[b * ps];
    if (b == NM - 1) {
      xx = cx * p;
      xy = cy * p;
    } else {
      xx = (cx - du[b] * xx) * p;
      xy = (cy - du[b] * xy) * p;
    }
    C2<T> o;
    if (kz0) {
      H0[(long long)b * klow + i] = 0.5 * xx;
      o.x = (T)0;
      o.y = (T)0;
    } else {
      o.x = (T)xx;
      o.y = (T)xy;
    }
    h[b * hs] = o;
  }
}

// plane[b][k][ii], ii < 2N, from the z-inverted hat
template <typename T>
__global__ void k_cf_untwiddle(Spec s, const C2<T> *__restrict__ hat, const C2<T> *__restrict__ post,
                               C2<T> *__restrict__ plane) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y, b = blockIdx.z;
  const int N = s.N;
  if (ii >= 2 * N) return;
  const C2<T> *hr = hat + ((long long)k * s.NM + b) * N;
  C2<T> v;
  if (ii < N) {
    v = cmc<T>(hr[ii], post[ii]);
  } else if (ii == N) {
    v.x = (T)0;
    v.y = (T)0;
  } else {
    const int m = 2 * N - ii;  // 1..N-1
    const C2<T> a = cmc<T>(hr[m], post[m]);
    v.x = a.x;
    v.y = -a.y;
  }
  plane[((long long)b * s.M + k) * (2LL * N) + ii] = v;
}

// rhs_p(ii+2, b+2, k+2) = Re plane[b][k][ii] / (2N M), plus the copies
template <typename T>
__global__ void k_cf_unpack(Geo g, Spec s, const C2<T> *__restrict__ plane, T norm, T *__restrict__ p) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int kp = blockIdx.y, b = blockIdx.z;
  const int N = s.N;
  if (ii >= N) return;
  const T v = plane[((long long)b * s.M + kp) * (2LL * N) + ii].x * norm;
  const long long c = bidx(g, ii + 2, b + 2, kp + 2);
  const long long zsh = (long long)s.M * g.plane;  // k = 2 -> k = nzp+2
  p[c] = v;
  if (kp == 0) p[c + zsh] = v;
  if (ii == N - 1) {  // rhs_p(nxg-1) = rhs_p(nxg-2)
    p[c + 1] = v;
    if (kp == 0) p[c + 1 + zsh] = v;
  }
}

template <typename T> struct Fft;
template <> struct Fft<double> {
  static constexpr cufftType type = CUFFT_Z2Z;
  static cufftResult exec(cufftHandle h, void *in, void *out, int dir) {
    return cufftExecZ2Z(h, (cufftDoubleComplex *)in, (cufftDoubleComplex *)out, dir);
  }
};
template <> struct Fft<float> {
  static constexpr cufftType type = CUFFT_C2C;
  static cufftResult exec(cufftHandle h, void *in, void *out, int dir) {
    return cufftExecC2C(h, (cufftComplex *)in, (cufftComplex *)out, dir);
  }
};

}  // namespace

struct CufftPath {
  cufftHandle p2d = 0, pzi = 0, pxi = 0;
  bool h2d = false, hzi = false, hxi = false;
  void *plane = nullptr, *hat = nullptr;
  size_t bytes = 0;
  bool fp64 = true;
};

int cufft_path_create(const Spec &s, bool fp64, cudaStream_t st, CufftPath **out, char *msg, size_t cap) {
  *out = nullptr;
  CufftPath *c = new CufftPath();
  c->fp64 = fp64;
  const size_t ce = fp64 ? sizeof(double2) : sizeof(float2);
  const long long N = s.N, M = s.M, NM = s.NM;
  auto fail = [&](const char *what, int code) {
    snprintf(msg, cap, "cuFFT path: %s failed (%d)", what, code);
    cufft_path_destroy(c);
    return -1;
  };
  c->bytes = (size_t)(2 * N * M * NM + N * NM * M) * ce;
  cudaError_t e = cudaMalloc(&c->plane, (size_t)2 * N * M * NM * ce);
  if (e != cudaSuccess) return fail("cudaMalloc of the 2N plane", (int)e);
  e = cudaMalloc(&c->hat, (size_t)N * NM * M * ce);
  if (e != cudaSuccess) return fail("cudaMalloc of the mode array", (int)e);
  const cufftType ty = fp64 ? Fft<double>::type : Fft<float>::type;
  // plan 1: 2D over (M, 2N) per y-row, batch NM (cufft_solver.f90:33-40)
  int n2[2] = {(int)M, (int)(2 * N)};
  cufftResult r = cufftPlanMany(&c->p2d, 2, n2, n2, 1, (int)(2 * N * M), n2, 1, (int)(2 * N * M), ty, (int)NM);
  if (r != CUFFT_SUCCESS) return fail("cufftPlanMany 2D", (int)r);
  c->h2d = true;
  // plan 2: inverse z, stride N*NM, batch N*NM (cufft_solver.f90:45-50)
  int n1[1] = {(int)M};
  r = cufftPlanMany(&c->pzi, 1, n1, n1, (int)(N * NM), 1, n1, (int)(N * NM), 1, ty, (int)(N * NM));
  if (r != CUFFT_SUCCESS) return fail("cufftPlanMany z", (int)r);
  c->hzi = true;
  // plan 3: inverse x over 2N, batch M*NM (cufft_solver.f90:52-59)
  int nx[1] = {(int)(2 * N)};
  r = cufftPlanMany(&c->pxi, 1, nx, nx, 1, (int)(2 * N), nx, 1, (int)(2 * N), ty, (int)(M * NM));
  if (r != CUFFT_SUCCESS) return fail("cufftPlanMany x", (int)r);
  c->hxi = true;
  for (cufftHandle h : {c->p2d, c->pzi, c->pxi}) {
    r = cufftSetStream(h, st);
    if (r != CUFFT_SUCCESS) return fail("cufftSetStream", (int)r);
  }
  *out = c;
  return 0;
}

void cufft_path_destroy(CufftPath *c) {
  if (!c) return;
  if (c->h2d) cufftDestroy(c->p2d);
  if (c->hzi) cufftDestroy(c->pzi);
  if (c->hxi) cufftDestroy(c->pxi);
  if (c->plane) cudaFree(c->plane);
  if (c->hat) cudaFree(c->hat);
  delete c;
}

size_t cufft_path_bytes(const CufftPath *c) { return c ? c->bytes : 0; }

template <typename T>
int cufft_path_forward(CufftPath *c, const Geo &g, const Spec &s, const T *U, const T *V, const T *W, cudaStream_t st) {
  const dim3 gp((s.N + 127) / 128, s.M, s.NM);
  k_cf_pack<T><<<gp, 128, 0, st>>>(g, s, U, V, W, (C2<T> *)c->plane);
  return (int)Fft<T>::exec(c->p2d, c->plane, c->plane, CUFFT_FORWARD);
}

template <typename T>
void cufft_path_extract_solve(CufftPath *c, const Spec &s, const void *post, const double *piv, const double *dl,
                              const double *du, double *H0, int klow, cudaStream_t st) {
  const dim3 gp((s.N + 127) / 128, s.M, s.NM);
  k_cf_extract<T><<<gp, 128, 0, st>>>(s, (const C2<T> *)c->plane, (const C2<T> *)post, (C2<T> *)c->hat);
  k_cf_thomas<T><<<dim3((s.N + 127) / 128, s.M), 128, 0, st>>>(s, (C2<T> *)c->hat, piv, dl, du, H0, klow);
}

template <typename T> int cufft_path_inverse_z(CufftPath *c) {
  return (int)Fft<T>::exec(c->pzi, c->hat, c->hat, CUFFT_INVERSE);
}

template <typename T>
int cufft_path_inverse_x(CufftPath *c, const Geo &g, const Spec &s, const void *post, T *p, cudaStream_t st) {
  const dim3 gu((2 * s.N + 127) / 128, s.M, s.NM);
  k_cf_untwiddle<T><<<gu, 128, 0, st>>>(s, (const C2<T> *)c->hat, (const C2<T> *)post, (C2<T> *)c->plane);
  const cufftResult r = Fft<T>::exec(c->pxi, c->plane, c->plane, CUFFT_INVERSE);
  const dim3 gp((s.N + 127) / 128, s.M, s.NM);
  const T norm = (T)(1.0 / (2.0 * (double)s.N * (double)s.M));
  k_cf_unpack<T><<<gp, 128, 0, st>>>(g, s, (const C2<T> *)c->plane, norm, p);
  return (int)r;
}

#define BLGPU_CF_INST(T)                                                                                           \
  template int cufft_path_forward<T>(CufftPath *, const Geo &, const Spec &, const T *, const T *, const T *,      \
                                     cudaStream_t);                                                                \
  template void cufft_path_extract_solve<T>(CufftPath *, const Spec &, const void *, const double *,               \
                                            const double *, const double *, double *, int, cudaStream_t);          \
  template int cufft_path_inverse_z<T>(CufftPath *);                                                               \
  template int cufft_path_inverse_x<T>(CufftPath *, const Geo &, const Spec &, const void *, T *, cudaStream_t);
BLGPU_CF_INST(double)
BLGPU_CF_INST(float)
#undef BLGPU_CF_INST

}  // namespace blgpu
