// capi.cu -- the C ABI (include/blgpu.h): context, device memory, host<->box
// layout conversion, step orchestration and CUDA-graph replay.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/blgpu.h"
#include "kernels.cuh"
#include "mlp.cuh"

namespace blgpu {

static thread_local std::string g_last_error = "";

int fail_cuda(cudaError_t e, const char *what, const char *file, int line);

}  // namespace blgpu

using namespace blgpu;

struct blgpu_ctx {
  blgpu_config cfg{};
  int nx = 0, ny = 0, nz = 0, nxg = 0, nyg = 0, nzg = 0, px = 0, py = 0;
  long long plane = 0, boxn = 0;
  bool fp64 = true;
  size_t esz = 8;
  cudaStream_t st = nullptr;
  bool have_grid = false, have_bc = false, have_state = false;
  std::string err;
  // host copies (1-based where the Fortran is)
  std::vector<double> x, y, z, xg, yg, zg, w0, w1, kxx, kzz, dd, dl, du;
  double dxmin = 0, dymin = 0, dzmin = 0, dtvis = 0, length_y = 0, qy = 0;
  double rk_t[4] = {0.0, 8.0 / 15.0, 2.0 / 3.0, 1.0};
  // device allocations
  std::vector<void *> allocs;
  long long bytes = 0;
  double *d_geo = nullptr;  // all FP64 metric tables in one block
  float *f_geo = nullptr;   // FP32 copies
  double *d_spec = nullptr; // dd, dl, du, kxx, kzz
  double *d_bc = nullptr;   // inflow/top vectors
  double *d_modes = nullptr;
  Geo geo{};
  MetT<double> m64{};
  MetT<float> m32{};
  BcData bc{};
  Spec spec{};
  void *S[3][3] = {};  // state buffers [buffer][u,v,w]
  void *F1[3] = {};
  void *P = nullptr, *nut = nullptr, *rhs_p = nullptr, *R = nullptr, *C = nullptr;
  double *dyn = nullptr;  // LES = 2, 3: dynamic-model work arrays (FP64)
  double *piv = nullptr, *qx_part = nullptr;
  // mixed form: the low-kx kz = 0 part of the pressure in FP64: p0 [NM][N], its modes
  // H0 [NM][klow], FP32 differences [2][NM][N], inverse-cosine matrix cm [klow][N]
  double *kz0 = nullptr, *kz0h = nullptr, *cmat = nullptr;
  float *kz0g = nullptr;
  int klow = 0;
  uint32_t *zfrag = nullptr;  // mixed form: table fragments of the tensor-core z transforms (or null)
  ZdftMaps zmaps{};           // and the TMA maps of R and C they read and write
  uint32_t *utab = nullptr;   // mixed form: tcgen05 z transforms, tables (or null)
  ZdftMaps umaps{};           // and their TMA maps
  ThomasMaps tmaps{};         // TMA maps of C and the pivots for the tiled y-solve
  RhsMaps rmaps[4]{};         // TMA maps of U, V, W of each state buffer and of F1 (TMA-fed RHS)
  bool have_rmaps = false;
  CufftPath *cf = nullptr;    // poisson = BLGPU_POISSON_CUFFT: plans and work arrays
  int cf_status = 0;          // first failing cufftExec status of an enqueued step (0: none)
  int wait_limit = -1;        // mbarrier polls of the tiled y-solve and the TMA-fed RHS (< 0: built-in), a test hook
  bool have_tmaps = false;
  int nsm = 148;
  Scalars *sc = nullptr;
  unsigned long long *d_maxdiv = nullptr;
  void *tw = nullptr, *post = nullptr, *ztab = nullptr;
  void *ztab64 = nullptr;  // cos and sin tables of the FP64 z transforms on the FP64 MMA
  FftPlan<double> pl64{};
  FftPlan<float> pl32{};
  double *stage = nullptr;  // FP64 staging of one host-layout field
  // streamed transfers: H2D and D2H streams, per-field staging buffers and
  // the events that order them against st
  cudaStream_t xin = nullptr, xout = nullptr;
  double *stage_in[3] = {nullptr, nullptr, nullptr}, *stage_out[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t ev_in_ready = nullptr, ev_in_free = nullptr, ev_out_ready = nullptr, ev_out_free = nullptr;
  double *d_cs2 = nullptr;  // (Cs Delta_j f)^2 of the Smagorinsky model, j = 0..nyg
  double *d_stats = nullptr;
  double *d_utau = nullptr;
  int *d_iters = nullptr;
  LundData lund{};
  Tiles tiles{};
  // wall model: 0 no-slip, 1 law of the wall, 2 network; d_wm = alpha_x, alpha_z, tau_x, tau_z
  int wm_mode = 0, wm_jh = 3;
  MlpDev wm_net{};
  double *d_wm = nullptr;
  long long gen = 0;  // bumped whenever the captured step graphs are dropped
  int cur = 0, old = 1;
  cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};
  int graph_next[3] = {0, 0, 0};
  long long graph_launches[3] = {0, 0, 0};
  // kernel accounting and optional per-phase event timing
  long long launches = 0;
  bool prof_on = false;
  struct Mark { int phase; cudaEvent_t a, b; int nk; };
  std::vector<Mark> marks;
  int cur_phase = -1, cur_nk = 0;
  cudaEvent_t cur_ev = nullptr;
  Geo geo_box() const {
    Geo g = geo;
    g.nx = nx; g.ny = ny; g.nz = nz; g.nxg = nxg; g.nyg = nyg; g.nzg = nzg;
    g.px = px; g.py = py; g.plane = plane;
    return g;
  }
};

enum { PH_RHS = 0, PH_BC, PH_DIVDCT, PH_DFTZ, PH_THOMAS, PH_IDFTZ, PH_IDCT, PH_PROJECT, PH_DT, PH_MISC, PH_N };

// Every launcher call is bracketed by ph_begin/ph_end: they count the kernels
// issued and, while profiling, record CUDA events on the context stream.
static void ph_begin(blgpu_ctx *ctx, int phase) {
  ctx->cur_phase = phase;
  if (ctx->prof_on) {
    cudaEventCreate(&ctx->cur_ev);
    cudaEventRecord(ctx->cur_ev, ctx->st);
  }
}

static void ph_end(blgpu_ctx *ctx, int nk) {
  ctx->launches += nk;
  if (ctx->prof_on) {
    cudaEvent_t b;
    cudaEventCreate(&b);
    cudaEventRecord(b, ctx->st);
    ctx->marks.push_back({ctx->cur_phase, ctx->cur_ev, b, nk});
    ctx->cur_ev = nullptr;
  }
}

namespace blgpu {

int fail_cuda(cudaError_t e, const char *what, const char *file, int line) {
  char buf[512];
  snprintf(buf, sizeof buf, "CUDA error %s (%s) at %s:%d in %s", cudaGetErrorName(e), cudaGetErrorString(e), file,
           line, what);
  g_last_error = buf;
  return BLGPU_ECUDA;
}

void set_global_error(const char *msg) { g_last_error = msg ? msg : ""; }

}  // namespace blgpu

static int set_err(blgpu_ctx *c, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  g_last_error = buf;
  return code;
}

static int check_cuda(blgpu_ctx *c, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return BLGPU_OK;
  return set_err(c, BLGPU_ECUDA, "CUDA error %s (%s) in %s", cudaGetErrorName(e), cudaGetErrorString(e), what);
}

#define CK(expr)                                           \
  do {                                                     \
    int _r = check_cuda(ctx, (expr), #expr);               \
    if (_r) return _r;                                     \
  } while (0)

static int dalloc(blgpu_ctx *ctx, void **p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) return set_err(ctx, BLGPU_ECUDA, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
  ctx->allocs.push_back(*p);
  ctx->bytes += (long long)bytes;
  e = cudaMemset(*p, 0, bytes);
  if (e != cudaSuccess) return set_err(ctx, BLGPU_ECUDA, "cudaMemset failed: %s", cudaGetErrorString(e));
  return BLGPU_OK;
}

// the sticky device flag of the step kernels (stream already synchronized);
// bit 2: a TMA copy of the tensor-core z transform missed its wait limit;
// bit 4: one of the tiled y-solve; bit 8: one of the tcgen05 z transform;
// bit 16: a row copy of the two-pass inverse x transform; bit 32: a streamed
// upload (blgpu_upload_state_async) held a NaN or an infinity; bit 64: a
// plane copy of the TMA-fed RHS
static int device_flag(blgpu_ctx *ctx) {
  int f = 0;
  CK(cudaMemcpy(&f, &ctx->sc->err, sizeof f, cudaMemcpyDeviceToHost));
  if (f) {  // reported once: the next call starts clean
    const int z = 0;
    CK(cudaMemcpy(&ctx->sc->err, &z, sizeof z, cudaMemcpyHostToDevice));
  }
  if (f & 32) return set_err(ctx, BLGPU_EDEVICE, "an uploaded state held a NaN or an infinity");
  if (f & 2) return set_err(ctx, BLGPU_EDEVICE, "z transform: a TMA copy did not complete within the wait limit");
  if (f & 4) return set_err(ctx, BLGPU_EDEVICE, "y-solve: a TMA tile copy did not complete within the wait limit");
  if (f & 8) return set_err(ctx, BLGPU_EDEVICE, "z transform (tcgen05): a copy or a product missed its wait limit");
  if (f & 16) return set_err(ctx, BLGPU_EDEVICE, "inverse x transform: a row copy did not complete within the wait limit");
  if (f & 64) return set_err(ctx, BLGPU_EDEVICE, "RHS: a plane copy did not complete within the wait limit");
  if (f) return set_err(ctx, BLGPU_EDEVICE, "device flag %d set by a step kernel", f);
  return BLGPU_OK;
}

static void drop_graphs(blgpu_ctx *ctx) {
  ctx->gen += 1;
  for (int r = 0; r < 3; ++r)
    if (ctx->graph[r]) {
      cudaGraphExecDestroy(ctx->graph[r]);
      ctx->graph[r] = nullptr;
    }
}

static std::vector<int> factorize(int n) {
  std::vector<int> f;
  int r = n;
  while (r % 4 == 0) { f.push_back(4); r /= 4; }
  while (r % 2 == 0) { f.push_back(2); r /= 2; }
  for (int p = 3; r > 1; p += 2)
    while (r % p == 0) { f.push_back(p); r /= p; }
  return f;
}

extern "C" {

const char *blgpu_last_error(const blgpu_ctx *ctx) {
  if (ctx && !ctx->err.empty()) return ctx->err.c_str();
  return g_last_error.c_str();
}

int blgpu_create(const blgpu_config *cfg, blgpu_ctx **out) {
  if (!cfg || !out) return set_err(nullptr, BLGPU_EINVAL, "blgpu_create: null argument");
  *out = nullptr;
  if (cfg->nx < 5 || cfg->ny < 4 || cfg->nz < 5)
    return set_err(nullptr, BLGPU_EINVAL, "blgpu_create: grid %dx%dx%d too small (need nx>=5, ny>=4, nz>=5)",
                   cfg->nx, cfg->ny, cfg->nz);
  if (cfg->rk_scheme < 1 || cfg->rk_scheme > 3)
    return set_err(nullptr, BLGPU_EINVAL, "blgpu_create: RKscheme %d not in {1,2,3}", cfg->rk_scheme);
  // LES as in compute_eddy_viscosity (subgrid.f90:23-47): 0 none, 1 constant-coefficient
  // Smagorinsky, 2 dynamic Smagorinsky with the coefficient averaged in z, 3 dynamic
  // Smagorinsky pointwise; BLGPU_LES_HOST: nu_t from the host
  if ((cfg->les_model == 2 || cfg->les_model == 3) && (cfg->ny >= 65535 || cfg->nz >= 65535))
    return set_err(nullptr, BLGPU_EINVAL, "blgpu_create: dynamic LES needs ny, nz < 65535");
  if (cfg->les_model != BLGPU_LES_HOST && (cfg->les_model < 0 || cfg->les_model > 3))
    return set_err(nullptr, BLGPU_EINVAL, "blgpu_create: unknown LES model %d", cfg->les_model);
  if (cfg->precision != BLGPU_FP64 && cfg->precision != BLGPU_MIXED)
    return set_err(nullptr, BLGPU_EINVAL, "blgpu_create: unknown precision %d", cfg->precision);
  if (cfg->poisson != BLGPU_POISSON_NATIVE && cfg->poisson != BLGPU_POISSON_CUFFT)
    return set_err(nullptr, BLGPU_EINVAL, "blgpu_create: unknown poisson backend %d", cfg->poisson);
  if (!(cfg->nu > 0)) return set_err(nullptr, BLGPU_EINVAL, "blgpu_create: nu must be > 0");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return set_err(nullptr, BLGPU_ECUDA, "blgpu_create: no CUDA device (%s)", cudaGetErrorString(e));
  if (cfg->device < 0 || cfg->device >= ndev)
    return set_err(nullptr, BLGPU_EINVAL, "blgpu_create: device %d out of range", cfg->device);
  blgpu_ctx *ctx = new blgpu_ctx();
  ctx->cfg = *cfg;
  ctx->nx = cfg->nx; ctx->ny = cfg->ny; ctx->nz = cfg->nz;
  ctx->nxg = cfg->nx + 1; ctx->nyg = cfg->ny + 1; ctx->nzg = cfg->nz + 1;
  ctx->px = (ctx->nxg + 8 + 31) / 32 * 32;  // room for 16-byte vectors past i = nxg
  ctx->py = ctx->nyg;
  ctx->plane = (long long)ctx->px * ctx->py;
  ctx->boxn = ctx->plane * ctx->nzg;
  ctx->fp64 = cfg->precision == BLGPU_FP64;
  ctx->esz = ctx->fp64 ? 8 : 4;
  int rc;
#define TRY(x) do { rc = (x); if (rc) { g_last_error = ctx->err; blgpu_destroy(ctx); return rc; } } while (0)
  TRY(check_cuda(ctx, cudaSetDevice(cfg->device), "cudaSetDevice"));
  TRY(check_cuda(ctx, cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking), "cudaStreamCreate"));
  const size_t box = (size_t)ctx->boxn * ctx->esz;
  for (int b = 0; b < 3; ++b)
    for (int q = 0; q < 3; ++q) TRY(dalloc(ctx, &ctx->S[b][q], box));
  for (int q = 0; q < 3; ++q) TRY(dalloc(ctx, &ctx->F1[q], box));
  {  // plane maps of the TMA-fed RHS: each state buffer and F1
    const Geo gb = ctx->geo_box();
    auto enc = [&](void *const *f, RhsMaps *out) {
      return ctx->fp64 ? rhs_maps64(gb, (const double *)f[0], (const double *)f[1], (const double *)f[2], out)
                       : rhs_maps(gb, (const float *)f[0], (const float *)f[1], (const float *)f[2], out);
    };
    ctx->have_rmaps = true;
    for (int b = 0; b < 3; ++b)
      if (!enc(ctx->S[b], &ctx->rmaps[b])) ctx->have_rmaps = false;
    if (!enc(ctx->F1, &ctx->rmaps[3])) ctx->have_rmaps = false;
  }
  TRY(dalloc(ctx, &ctx->P, box));
  TRY(dalloc(ctx, &ctx->rhs_p, box));
  if (cfg->les_model) TRY(dalloc(ctx, &ctx->nut, box));
  if (cfg->les_model == 2 || cfg->les_model == 3)
    TRY(dalloc(ctx, (void **)&ctx->dyn, dyn_smagorinsky_work_bytes(ctx->nxg, ctx->nyg, ctx->nzg)));
  Spec &s = ctx->spec;
  s.N = ctx->nx - 2;
  s.M = ctx->nz - 2;
  s.NM = ctx->ny - 1;
  s.MH = s.M / 2 + 1;
  s.rx = (s.N + 31) / 32 * 32;
  TRY(dalloc(ctx, &ctx->R, (size_t)s.NM * s.M * s.rx * ctx->esz));
  TRY(dalloc(ctx, &ctx->C, (size_t)s.NM * s.MH * s.rx * ctx->esz * 2));
  TRY(dalloc(ctx, (void **)&ctx->piv, (size_t)s.NM * s.MH * s.rx * sizeof(double)));
  ctx->have_tmaps = ctx->fp64 ? thomas_maps<double>(s, ctx->C, ctx->piv, &ctx->tmaps)
                              : thomas_maps<float>(s, ctx->C, ctx->piv, &ctx->tmaps);
  if (cfg->poisson == BLGPU_POISSON_CUFFT) {  // cufft_init_plans (cufft_solver.f90:26-62)
    char msg[256];
    if (cufft_path_create(s, ctx->fp64, ctx->st, &ctx->cf, msg, sizeof msg)) TRY(set_err(ctx, BLGPU_ECUDA, "%s", msg));
    ctx->bytes += (long long)cufft_path_bytes(ctx->cf);
  }
  cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, cfg->device);
  TRY(upload_dft_constants() == 0 ? BLGPU_OK : set_err(ctx, BLGPU_ECUDA, "DFT constants upload failed"));
  if (!ctx->fp64 && zdft_tc_qp(s)) {
    std::vector<uint32_t> fr;
    zdft_tc_fragments(s, fr);
    TRY(dalloc(ctx, (void **)&ctx->zfrag, fr.size() * sizeof(uint32_t)));
    TRY(check_cuda(ctx, cudaMemcpy(ctx->zfrag, fr.data(), fr.size() * sizeof(uint32_t), cudaMemcpyHostToDevice),
                   "z-transform tables"));
    // without tensor maps the direct sums serve this box
    if (!zdft_tc_maps(s, (float *)ctx->R, (float2 *)ctx->C, &ctx->zmaps)) ctx->zfrag = nullptr;
  }
  if (!ctx->fp64 && zdft_umma_qp(s)) {
    std::vector<uint32_t> ut;
    zdft_umma_tables(s, ut);
    TRY(dalloc(ctx, (void **)&ctx->utab, ut.size() * sizeof(uint32_t)));
    TRY(check_cuda(ctx, cudaMemcpy(ctx->utab, ut.data(), ut.size() * sizeof(uint32_t), cudaMemcpyHostToDevice),
                   "tcgen05 z-transform tables"));
    if (!zdft_umma_maps(s, (float *)ctx->R, (float2 *)ctx->C, &ctx->umaps)) ctx->utab = nullptr;
  }
  if (!ctx->fp64) {
    // the modes kx < klow of kz = 0 carry the box-scale pressure of a step's
    // flux change; above them the modes are small enough for FP32
    ctx->klow = std::min(128, s.N);
    TRY(dalloc(ctx, (void **)&ctx->kz0, (size_t)s.NM * s.N * sizeof(double)));
    TRY(dalloc(ctx, (void **)&ctx->kz0h, (size_t)s.NM * ctx->klow * sizeof(double)));
    TRY(dalloc(ctx, (void **)&ctx->kz0g, 2 * (size_t)s.NM * s.N * sizeof(float)));
    TRY(dalloc(ctx, (void **)&ctx->cmat, (size_t)ctx->klow * s.N * sizeof(double)));
    // inverse DCT-II of length N with the 1/(N M) of the inverse transforms
    std::vector<double> ct(4 * (size_t)s.N), cm((size_t)ctx->klow * s.N);
    for (int q = 0; q < 4 * s.N; ++q) ct[q] = cos(M_PI * (double)q / (2.0 * (double)s.N));
    const double nrm = 1.0 / ((double)s.N * (double)s.M);
    for (int kx = 0; kx < ctx->klow; ++kx)
      for (int i = 0; i < s.N; ++i)
        cm[(size_t)kx * s.N + i] = (kx ? 2.0 : 1.0) * nrm * ct[((long long)kx * (2 * i + 1)) % (4 * s.N)];
    TRY(check_cuda(ctx, cudaMemcpy(ctx->cmat, cm.data(), cm.size() * sizeof(double), cudaMemcpyHostToDevice),
                   "cosine matrix"));
  }
  TRY(dalloc(ctx, (void **)&ctx->sc, sizeof(Scalars)));
  TRY(dalloc(ctx, (void **)&ctx->stage, (size_t)ctx->nxg * ctx->nyg * ctx->nzg * sizeof(double)));
  TRY(dalloc(ctx, (void **)&ctx->d_cs2, (size_t)(ctx->nyg + 2) * sizeof(double)));
  TRY(dalloc(ctx, (void **)&ctx->d_stats,
             ((size_t)9 * ctx->nx * ctx->ny + (size_t)ctx->nxg * ctx->nyg + 2 * (size_t)ctx->nx) * sizeof(double)));
  TRY(dalloc(ctx, (void **)&ctx->d_utau, (size_t)ctx->nx * sizeof(double)));
  TRY(dalloc(ctx, (void **)&ctx->d_iters, (size_t)ctx->nx * sizeof(int)));
  TRY(dalloc(ctx, (void **)&ctx->d_maxdiv, sizeof(unsigned long long)));
  TRY(dalloc(ctx, (void **)&ctx->d_wm, 4 * (size_t)(ctx->nx - 2) * (ctx->nzg - 3) * sizeof(double)));
  {  // Lund inflow state, FP64, laid out as described at LundData
    const size_t nyg = ctx->nyg, ny = ctx->ny, nzg = ctx->nzg, nz = ctx->nz;
    const size_t nd = (2 * nyg + 2 * ny + 1) + (2 * nyg + 2 * ny) + 4 * nyg + (nyg + ny) + 4 * nyg +
                      nyg * nzg + ny * nzg + nyg * nz + 8;
    double *d = nullptr;
    int *ip = nullptr;
    TRY(dalloc(ctx, (void **)&d, nd * sizeof(double)));
    TRY(dalloc(ctx, (void **)&ip, (4 * nyg + 1) * sizeof(int)));
    LundData &L = ctx->lund;
    L.inst = d; d += 2 * nyg + 2 * ny + 1;
    L.mean = d; d += 2 * nyg + 2 * ny;
    L.rowc = d; d += 4 * nyg;
    L.wgt = d; d += nyg + ny;
    L.mprof = d; d += 4 * nyg;
    L.lu = d; d += nyg * nzg;
    L.lv = d; d += ny * nzg;
    L.lw = d; d += nyg * nz;
    L.diag = d;
    L.rowi = ip;
    L.err = ip + 4 * nyg;
    ctx->bc.lu = L.lu;
    ctx->bc.lv = L.lv;
    ctx->bc.lw = L.lw;
  }
  // transform tables
  {
    const int N = s.N, M = s.M;
    const int MH = s.MH;
    std::vector<double> tw(2 * N), post(2 * N), zt(2 * (size_t)MH * MH);
    for (int t = 0; t < N; ++t) {
      double a = -2.0 * M_PI * (double)t / (double)N;
      tw[2 * t] = cos(a);
      tw[2 * t + 1] = sin(a);
      double b = -M_PI * (double)t / (2.0 * (double)N);
      post[2 * t] = cos(b);
      post[2 * t + 1] = sin(b);
    }
    // tz[m][n] = (cos, sin)(2 pi m n / M), m, n = 0..MH-1
    for (int m = 0; m < MH; ++m)
      for (int n = 0; n < MH; ++n) {
        double a = 2.0 * M_PI * (double)(((long long)m * n) % M) / (double)M;
        zt[2 * ((size_t)m * MH + n)] = cos(a);
        zt[2 * ((size_t)m * MH + n) + 1] = sin(a);
      }
    const size_t es2 = 2 * ctx->esz;
    TRY(dalloc(ctx, &ctx->tw, N * es2));
    TRY(dalloc(ctx, &ctx->post, N * es2));
    TRY(dalloc(ctx, &ctx->ztab, (size_t)MH * MH * es2));
    if (ctx->fp64) {
      TRY(check_cuda(ctx, cudaMemcpy(ctx->tw, tw.data(), N * es2, cudaMemcpyHostToDevice), "tw"));
      TRY(check_cuda(ctx, cudaMemcpy(ctx->post, post.data(), N * es2, cudaMemcpyHostToDevice), "post"));
      TRY(check_cuda(ctx, cudaMemcpy(ctx->ztab, zt.data(), (size_t)MH * MH * es2, cudaMemcpyHostToDevice), "ztab"));
      if (s.M >= 8 && s.M <= 254) {  // FP64 z transforms on the FP64 MMA (rows to 128, 4 per lane group)
        std::vector<double> t64;
        zdft64_tables(s, t64);
        TRY(dalloc(ctx, &ctx->ztab64, t64.size() * sizeof(double)));
        TRY(check_cuda(ctx, cudaMemcpy(ctx->ztab64, t64.data(), t64.size() * sizeof(double), cudaMemcpyHostToDevice),
                       "ztab64"));
      }
    } else {
      std::vector<float> a(tw.begin(), tw.end()), b(post.begin(), post.end()), c(zt.begin(), zt.end());
      TRY(check_cuda(ctx, cudaMemcpy(ctx->tw, a.data(), N * es2, cudaMemcpyHostToDevice), "tw"));
      TRY(check_cuda(ctx, cudaMemcpy(ctx->post, b.data(), N * es2, cudaMemcpyHostToDevice), "post"));
      TRY(check_cuda(ctx, cudaMemcpy(ctx->ztab, c.data(), (size_t)MH * MH * es2, cudaMemcpyHostToDevice), "ztab"));
    }
    std::vector<int> f = factorize(N);
    if (f.size() > 24) TRY(set_err(ctx, BLGPU_EINVAL, "DCT length %d has too many factors", N));
    ctx->pl64.n = ctx->pl32.n = N;
    ctx->pl64.nst = ctx->pl32.nst = (int)f.size();
    for (size_t q = 0; q < f.size(); ++q) ctx->pl64.rad[q] = ctx->pl32.rad[q] = f[q];
    ctx->pl64.tw = (const double2 *)ctx->tw;
    ctx->pl64.post = (const double2 *)ctx->post;
    ctx->pl32.tw = (const float2 *)ctx->tw;
    ctx->pl32.post = (const float2 *)ctx->post;
    const size_t sm = dct_smem_bytes(N, (int)ctx->esz, 1, 0);  // one line per CTA at the least
    int dev_sm = 0;
    cudaDeviceGetAttribute(&dev_sm, cudaDevAttrMaxSharedMemoryPerBlockOptin, cfg->device);
    if ((long long)sm > dev_sm) TRY(set_err(ctx, BLGPU_EINVAL, "nx=%d needs %zu B shared memory per CTA", ctx->nx, sm));
  }
  {
    Scalars h{};
    TRY(check_cuda(ctx, cudaMemcpy(ctx->sc, &h, sizeof h, cudaMemcpyHostToDevice), "scalars"));
  }
#undef TRY
  *out = ctx;
  return BLGPU_OK;
}

int blgpu_destroy(blgpu_ctx *ctx) {
  if (!ctx) return BLGPU_OK;
  if (ctx->cfg.device >= 0) cudaSetDevice(ctx->cfg.device);
  for (int r = 0; r < 3; ++r)
    if (ctx->graph[r]) cudaGraphExecDestroy(ctx->graph[r]);
  if (ctx->st) cudaStreamSynchronize(ctx->st);
  if (ctx->xin) cudaStreamSynchronize(ctx->xin);
  if (ctx->xout) cudaStreamSynchronize(ctx->xout);
  for (void *p : ctx->allocs) cudaFree(p);
  cufft_path_destroy(ctx->cf);  // cufft_destroy_plans (cufft_solver.f90:64-72)
  if (ctx->st) cudaStreamDestroy(ctx->st);
  if (ctx->xin) cudaStreamDestroy(ctx->xin);
  if (ctx->xout) cudaStreamDestroy(ctx->xout);
  for (cudaEvent_t e : {ctx->ev_in_ready, ctx->ev_in_free, ctx->ev_out_ready, ctx->ev_out_free})
    if (e) cudaEventDestroy(e);
  delete ctx;
  return BLGPU_OK;
}

long long blgpu_device_bytes(const blgpu_ctx *ctx) { return ctx ? ctx->bytes : 0; }

int blgpu_set_grid(blgpu_ctx *ctx, const double *x, const double *y, const double *z) {
  if (!ctx || !x || !y || !z) return set_err(ctx, BLGPU_EINVAL, "blgpu_set_grid: null argument");
  const int nx = ctx->nx, ny = ctx->ny, nz = ctx->nz;
  for (int i = 1; i < nx; ++i)
    if (!(x[i] > x[i - 1])) return set_err(ctx, BLGPU_EINVAL, "blgpu_set_grid: x not increasing at %d", i + 1);
  for (int j = 1; j < ny; ++j)
    if (!(y[j] > y[j - 1])) return set_err(ctx, BLGPU_EINVAL, "blgpu_set_grid: y not increasing at %d", j + 1);
  for (int k = 1; k < nz; ++k)
    if (!(z[k] > z[k - 1])) return set_err(ctx, BLGPU_EINVAL, "blgpu_set_grid: z not increasing at %d", k + 1);
  CK(cudaSetDevice(ctx->cfg.device));
  // initialization.f90:174-222 (faces -> centres -> ghost-padded centres)
  auto build = [](const double *f, int n, std::vector<double> &F, std::vector<double> &G) {
    F.assign(n + 1, 0.0);
    for (int i = 1; i <= n; ++i) F[i] = f[i - 1];
    const int nm = n - 1;
    std::vector<double> m(nm + 1);
    for (int i = 1; i <= nm; ++i) m[i] = 0.5 * (F[i] + F[i + 1]);
    G.assign(nm + 3, 0.0);
    for (int i = 1; i <= nm; ++i) G[i + 1] = m[i];
    G[1] = m[1] - 2.0 * (m[1] - F[1]);
    G[nm + 2] = m[nm] + 2.0 * (F[n] - m[nm]);
  };
  build(x, nx, ctx->x, ctx->xg);
  build(y, ny, ctx->y, ctx->yg);
  build(z, nz, ctx->z, ctx->zg);
  auto minsp = [](const std::vector<double> &G, int ng) {
    double mn = INFINITY;
    for (int i = 2; i <= ng; ++i) mn = std::min(mn, G[i] - G[i - 1]);
    return mn;
  };
  ctx->dxmin = minsp(ctx->xg, ctx->nxg);
  ctx->dymin = minsp(ctx->yg, ctx->nyg);
  ctx->dzmin = minsp(ctx->zg, ctx->nzg);
  const double nu = ctx->cfg.nu, cfla = fabs(ctx->cfg.cfl);
  ctx->dtvis = std::min(std::min(cfla * (ctx->dxmin * ctx->dxmin) / nu, cfla * (ctx->dymin * ctx->dymin) / nu),
                        cfla * (ctx->dzmin * ctx->dzmin) / nu);
  // weights (initialization.f90:482-484)
  ctx->w0.assign(ny + 2, 0.0);
  ctx->w1.assign(ny + 2, 0.0);
  for (int j = 1; j <= ny; ++j) {
    ctx->w0[j] = (ctx->yg[j + 1] - ctx->y[j]) / (ctx->yg[j + 1] - ctx->yg[j]);
    ctx->w1[j] = 1.0 - ctx->w0[j];
  }
  // Dyy rows j = 2..nyg-1 (initialization.f90:395-425), stored by b = j-2
  const Spec &s = ctx->spec;
  ctx->dd.assign(s.NM, 0.0);
  ctx->dl.assign(s.NM, 0.0);
  ctx->du.assign(s.NM, 0.0);
  for (int j = 2; j <= ctx->nyg - 1; ++j) {
    const double *Y = ctx->y.data(), *YG = ctx->yg.data();
    double a = 1.0 / (Y[j] - Y[j - 1]) / (YG[j + 1] - YG[j]);
    double b = 1.0 / (Y[j] - Y[j - 1]) * (-1.0 / (YG[j + 1] - YG[j]) - 1.0 / (YG[j] - YG[j - 1]));
    double c = 1.0 / (Y[j] - Y[j - 1]) / (YG[j] - YG[j - 1]);
    double d = b;
    if (j == 2) d = b + c;
    if (j == ctx->nyg - 1) d = a + b;
    ctx->dd[j - 2] = d;
    ctx->dl[j - 2] = c;
    ctx->du[j - 2] = a;
  }
  // modified wavenumbers (initialization.f90:329-344); dx = dxmin, dz = dzmin
  const double pi = 4.0 * atan(1.0);
  ctx->kxx.assign(s.N, 0.0);
  for (int i = 0; i < s.N; ++i)
    ctx->kxx[i] = 2.0 * (cos(pi * (double)i / (double)s.N) - 1.0) / (ctx->dxmin * ctx->dxmin);
  ctx->kzz.assign(s.MH, 0.0);
  const int half = (int)ceil((double)s.M / 2.0);
  for (int k = 0; k < s.MH; ++k) {
    if (k <= half)
      ctx->kzz[k] = 2.0 * (cos(2.0 * pi * (double)k / (double)s.M) - 1.0) / (ctx->dzmin * ctx->dzmin);
    else
      ctx->kzz[k] = 2.0 * (cos(2.0 * pi * (double)(-s.M + k) / (double)s.M) - 1.0) / (ctx->dzmin * ctx->dzmin);
  }
  // Smagorinsky (Cs Delta_j f)^2, subgrid.f90:629-639 (f = 1, Cs = 0.11)
  {
    std::vector<double> cs2(ctx->nyg + 2, 0.0);
    for (int j = 2; j <= ctx->nyg - 1; ++j) {
      const double Delta = pow(ctx->dxmin * ctx->dzmin * (ctx->y[j] - ctx->y[j - 1]), 1.0 / 3.0);
      cs2[j] = (0.11 * Delta * 1.0) * (0.11 * Delta * 1.0);
    }
    CK(cudaMemcpy(ctx->d_cs2, cs2.data(), cs2.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  // length_y of the mass balance (boundary_conditions.f90:242-246)
  ctx->length_y = 0.0;
  for (int j = 2; j <= ctx->nyg - 1; ++j) ctx->length_y = ctx->length_y + ctx->y[j] - ctx->y[j - 1];
  // metric tables: per axis F, C, rF, rC (1-based), then raw grids and weights
  const int nxt = ctx->nxg + 2, nyt = ctx->nyg + 2, nzt = ctx->nzg + 2;
  auto axis = [](const std::vector<double> &Fv, int n, const std::vector<double> &G, int ng, int len,
                 std::vector<double> &out) {
    std::vector<double> F(len, 1.0), C(len, 1.0);
    for (int i = 2; i <= n; ++i) F[i] = Fv[i] - Fv[i - 1];
    for (int i = 1; i <= ng - 1; ++i) C[i] = G[i + 1] - G[i];
    for (int i = 0; i < len; ++i) out.push_back(F[i]);
    for (int i = 0; i < len; ++i) out.push_back(C[i]);
    for (int i = 0; i < len; ++i) out.push_back(1.0 / F[i]);
    for (int i = 0; i < len; ++i) out.push_back(1.0 / C[i]);
  };
  std::vector<double> h;
  axis(ctx->x, nx, ctx->xg, ctx->nxg, nxt, h);
  axis(ctx->y, ny, ctx->yg, ctx->nyg, nyt, h);
  axis(ctx->z, nz, ctx->zg, ctx->nzg, nzt, h);
  const size_t off_w = h.size();
  for (int j = 0; j < nyt; ++j) h.push_back(j < (int)ctx->w0.size() ? ctx->w0[j] : 0.0);
  for (int j = 0; j < nyt; ++j) h.push_back(j < (int)ctx->w1.size() ? ctx->w1[j] : 0.0);
  const size_t off_raw = h.size();
  auto pushv = [&](const std::vector<double> &v, int len) {
    for (int i = 0; i < len; ++i) h.push_back(i < (int)v.size() ? v[i] : 0.0);
  };
  pushv(ctx->x, nxt); pushv(ctx->xg, nxt); pushv(ctx->y, nyt); pushv(ctx->yg, nyt); pushv(ctx->z, nzt); pushv(ctx->zg, nzt);
  if (!ctx->d_geo) {
    int rc = dalloc(ctx, (void **)&ctx->d_geo, h.size() * sizeof(double));
    if (rc) return rc;
    rc = dalloc(ctx, (void **)&ctx->f_geo, h.size() * sizeof(float));
    if (rc) return rc;
    rc = dalloc(ctx, (void **)&ctx->d_spec, (size_t)(3 * s.NM + s.N + s.MH) * sizeof(double));
    if (rc) return rc;
    rc = dalloc(ctx, (void **)&ctx->qx_part, (size_t)bc_x_parts(Geo{0, 0, 0, 0, ctx->nyg, ctx->nzg}) * sizeof(double) + 64);
    if (rc) return rc;
  }
  std::vector<float> hf(h.begin(), h.end());
  CK(cudaMemcpy(ctx->d_geo, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->f_geo, hf.data(), hf.size() * sizeof(float), cudaMemcpyHostToDevice));
  std::vector<double> sp;
  sp.insert(sp.end(), ctx->dd.begin(), ctx->dd.end());
  sp.insert(sp.end(), ctx->dl.begin(), ctx->dl.end());
  sp.insert(sp.end(), ctx->du.begin(), ctx->du.end());
  sp.insert(sp.end(), ctx->kxx.begin(), ctx->kxx.end());
  sp.insert(sp.end(), ctx->kzz.begin(), ctx->kzz.end());
  CK(cudaMemcpy(ctx->d_spec, sp.data(), sp.size() * sizeof(double), cudaMemcpyHostToDevice));
  {  // inverse pivots of the y-solve, fixed by the grid
    const double *d = ctx->d_spec;
    launch_thomas_factors(s, ctx->piv, d, d + s.NM, d + 2 * s.NM, d + 3 * s.NM, d + 3 * s.NM + s.N, ctx->st);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->st));
  }
  // views
  Geo &g = ctx->geo;
  g.nx = nx; g.ny = ny; g.nz = nz; g.nxg = ctx->nxg; g.nyg = ctx->nyg; g.nzg = ctx->nzg;
  g.px = ctx->px; g.py = ctx->py; g.plane = ctx->plane;
  const double *D = ctx->d_geo;
  g.ax = Axis{D, D + nxt, D + 2 * nxt, D + 3 * nxt};
  D += 4 * nxt;
  g.ay = Axis{D, D + nyt, D + 2 * nyt, D + 3 * nyt};
  D += 4 * nyt;
  g.az = Axis{D, D + nzt, D + 2 * nzt, D + 3 * nzt};
  g.w0 = ctx->d_geo + off_w;
  g.w1 = g.w0 + nyt;
  const double *Rw = ctx->d_geo + off_raw;
  g.x = Rw; g.xg = Rw + nxt; g.y = Rw + 2 * nxt; g.yg = g.y + nyt; g.z = g.yg + nyt; g.zg = g.z + nzt;
  g.nu = nu; g.dpdx = ctx->cfg.dpdx; g.dpdz = ctx->cfg.dpdz;
  auto met = [&](auto *B, auto &m, auto cast) {
    auto *p = B;
    m.xF = p; m.xC = p + nxt; m.xrF = p + 2 * nxt; m.xrC = p + 3 * nxt; p += 4 * nxt;
    m.yF = p; m.yC = p + nyt; m.yrF = p + 2 * nyt; m.yrC = p + 3 * nyt; p += 4 * nyt;
    m.zF = p; m.zC = p + nzt; m.zrF = p + 2 * nzt; m.zrC = p + 3 * nzt;
    m.w0 = B + off_w; m.w1 = B + off_w + nyt;
    m.nu = cast(nu); m.dpdx = cast(ctx->cfg.dpdx); m.dpdz = cast(ctx->cfg.dpdz);
  };
  met(ctx->d_geo, ctx->m64, [](double v) { return v; });
  met(ctx->f_geo, ctx->m32, [](double v) { return (float)v; });
  drop_graphs(ctx);
  ctx->have_grid = true;
  return BLGPU_OK;
}

int blgpu_set_boundary(blgpu_ctx *ctx, const double *U_inlet, const double *V_inlet, const double *W_inlet,
                       const double *U_top, const double *V_top, const double *W_top) {
  if (!ctx || !U_inlet || !V_inlet || !W_inlet || !U_top || !V_top || !W_top)
    return set_err(ctx, BLGPU_EINVAL, "blgpu_set_boundary: null argument");
  CK(cudaSetDevice(ctx->cfg.device));
  const int nyg = ctx->nyg, ny = ctx->ny, nx = ctx->nx, nxg = ctx->nxg;
  // 1-based vectors: [0]=unused
  std::vector<double> h;
  auto push = [&](const double *v, int n) {
    h.push_back(0.0);
    for (int i = 0; i < n; ++i) h.push_back(v[i]);
    h.push_back(0.0);
  };
  push(U_inlet, nyg); push(V_inlet, ny); push(W_inlet, nyg); push(U_top, nx); push(V_top, nxg); push(W_top, nxg);
  if (!ctx->d_bc) {
    int rc = dalloc(ctx, (void **)&ctx->d_bc, h.size() * sizeof(double));
    if (rc) return rc;
  }
  CK(cudaMemcpy(ctx->d_bc, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
  const double *p = ctx->d_bc;
  ctx->bc.U_inlet = p; p += nyg + 2;
  ctx->bc.V_inlet = p; p += ny + 2;
  ctx->bc.W_inlet = p; p += nyg + 2;
  ctx->bc.U_top = p; p += nx + 2;
  ctx->bc.V_top = p; p += nxg + 2;
  ctx->bc.W_top = p;
  // Qy of the mass balance: V(i,1,k) = 0 and V(i,ny,k) = V_top(i) when it is
  // evaluated (boundary_conditions.f90:230-253), so it is a constant of the run
  if (ctx->have_grid) {
    double qy = 0.0;
    for (int i = 2; i <= ctx->nxg - 2; ++i) {
      double s = 0.0;
      for (int k = 2; k <= ctx->nzg - 2; ++k) s += (0.0 - V_top[i - 1]) * (ctx->x[i] - ctx->x[i - 1]);
      qy = qy + s;
    }
    ctx->qy = qy;
  } else {
    return set_err(ctx, BLGPU_ESTATE, "blgpu_set_boundary: call blgpu_set_grid first");
  }
  drop_graphs(ctx);
  ctx->have_bc = true;
  return BLGPU_OK;
}

int blgpu_set_inflow_modes(blgpu_ctx *ctx, int n_modes, int m_modes, const double *zmode, const double *tmode,
                           const double *qu, const double *qv, const double *qw) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  if (n_modes < 0 || m_modes < 0) return set_err(ctx, BLGPU_EINVAL, "negative mode count");
  CK(cudaSetDevice(ctx->cfg.device));
  ctx->bc.n_modes = 0;
  ctx->bc.m_modes = 0;
  if (n_modes == 0 || m_modes == 0) return BLGPU_OK;
  if (!zmode || !tmode || !qu || !qv || !qw) return set_err(ctx, BLGPU_EINVAL, "null mode array");
  const size_t nq = (size_t)n_modes * m_modes;
  std::vector<double> h;
  h.insert(h.end(), zmode, zmode + n_modes);
  h.insert(h.end(), tmode, tmode + m_modes);
  if (h.size() & 1) h.push_back(0.0);  // keep the complex arrays 16-byte aligned
  const size_t oq = h.size();
  h.insert(h.end(), qu, qu + 2 * nq * ctx->nyg);
  const size_t ov = h.size();
  h.insert(h.end(), qv, qv + 2 * nq * ctx->ny);
  const size_t ow = h.size();
  h.insert(h.end(), qw, qw + 2 * nq * ctx->nyg);
  void *p = nullptr;
  int rc = dalloc(ctx, &p, h.size() * sizeof(double));
  if (rc) return rc;
  ctx->d_modes = (double *)p;
  CK(cudaMemcpy(p, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
  ctx->bc.zmode = ctx->d_modes;
  ctx->bc.tmode = ctx->d_modes + n_modes;
  ctx->bc.qu = (const double2 *)(ctx->d_modes + oq);
  ctx->bc.qv = (const double2 *)(ctx->d_modes + ov);
  ctx->bc.qw = (const double2 *)(ctx->d_modes + ow);
  ctx->bc.n_modes = n_modes;
  ctx->bc.m_modes = m_modes;
  drop_graphs(ctx);
  return BLGPU_OK;
}

int blgpu_set_rescaling(blgpu_ctx *ctx, int mode, int i_rescale, double delta_inlet, double T_resc,
                        const double *Umean0, const double *Vmean0) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  if (mode != 0 && mode != 3 && mode != 5)
    return set_err(ctx, BLGPU_EINVAL, "blgpu_set_rescaling: mode %d is not 0, 3 or 5", mode);
  if (mode != 0 && (i_rescale < 2 || i_rescale > ctx->nx))
    return set_err(ctx, BLGPU_EINVAL, "blgpu_set_rescaling: i_rescale %d outside 2..nx", i_rescale);
  if (mode != 0 && !(delta_inlet > 0.0 && T_resc > 0.0))
    return set_err(ctx, BLGPU_EINVAL, "blgpu_set_rescaling: delta_inlet and T_resc must be > 0");
  if (mode != 0 && (!ctx->have_grid || !ctx->have_state))
    return set_err(ctx, BLGPU_ESTATE, "blgpu_set_rescaling: grid and state must be set first");
  CK(cudaSetDevice(ctx->cfg.device));
  drop_graphs(ctx);
  LundData &L = ctx->lund;
  L.mode = mode;
  L.ir = i_rescale;
  L.delta_inlet = delta_inlet;
  L.T_resc = T_resc;
  ctx->bc.lund = mode;
  if (!mode) return BLGPU_OK;
  // running means at start-up (initialization.f90:636-664)
  const int nyg = ctx->nyg, ny = ctx->ny;
  CK(cudaMemsetAsync(L.err, 0, sizeof(int), ctx->st));
  if (ctx->fp64) {
    double **S = reinterpret_cast<double **>(ctx->S[ctx->cur]);
    launch_lund<double>(ctx->geo, L, S[0], S[1], S[2], ctx->sc, 0, ctx->st);
  } else {
    float **S = reinterpret_cast<float **>(ctx->S[ctx->cur]);
    launch_lund<float>(ctx->geo, L, S[0], S[1], S[2], ctx->sc, 0, ctx->st);
  }
  ctx->launches += 1;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(L.mean, L.inst, (size_t)(2 * nyg + 2 * ny) * sizeof(double), cudaMemcpyDeviceToDevice, ctx->st));
  double s0 = 0.0;
  if (Umean0)
    for (int j = 0; j < nyg; ++j) s0 += Umean0[j];
  if (Umean0 && s0 > 1e-4) {  // restart means (input_output.f90:439-460)
    std::vector<double> v(ny, 0.0);
    if (Vmean0) v.assign(Vmean0, Vmean0 + ny);
    CK(cudaMemcpyAsync(L.mean, Umean0, (size_t)nyg * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(L.mean + 2 * nyg, v.data(), (size_t)ny * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
  }
  CK(cudaStreamSynchronize(ctx->st));
  return BLGPU_OK;
}

int blgpu_rescaled_inflow(blgpu_ctx *ctx) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  if (!ctx->lund.mode) return set_err(ctx, BLGPU_ESTATE, "blgpu_rescaled_inflow: rescaling is off");
  CK(cudaSetDevice(ctx->cfg.device));
  if (ctx->fp64) {
    double **S = reinterpret_cast<double **>(ctx->S[ctx->cur]);
    launch_lund<double>(ctx->geo, ctx->lund, S[0], S[1], S[2], ctx->sc, 1, ctx->st);
  } else {
    float **S = reinterpret_cast<float **>(ctx->S[ctx->cur]);
    launch_lund<float>(ctx->geo, ctx->lund, S[0], S[1], S[2], ctx->sc, 1, ctx->st);
  }
  ctx->launches += 3;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->st));
  return BLGPU_OK;
}

int blgpu_get_rescaling(blgpu_ctx *ctx, double *Umean_resc, double *Vmean_resc, double *Umean_inlet,
                        double *Vmean_inlet, double *Lu, double *Lv, double *Lw, double *diag, int *err) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  CK(cudaSetDevice(ctx->cfg.device));
  const LundData &L = ctx->lund;
  const size_t nyg = ctx->nyg, ny = ctx->ny, nzg = ctx->nzg, nz = ctx->nz;
  auto get = [&](double *h, const double *d, size_t n) -> int {
    if (h) CK(cudaMemcpyAsync(h, d, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    return BLGPU_OK;
  };
  int rc;
  if ((rc = get(Umean_resc, L.mean, nyg)) || (rc = get(Umean_inlet, L.mean + nyg, nyg)) ||
      (rc = get(Vmean_resc, L.mean + 2 * nyg, ny)) || (rc = get(Vmean_inlet, L.mean + 2 * nyg + ny, ny)) ||
      (rc = get(Lu, L.lu, nyg * nzg)) || (rc = get(Lv, L.lv, ny * nzg)) || (rc = get(Lw, L.lw, nyg * nz)) ||
      (rc = get(diag, L.diag, 8)))
    return rc;
  if (err) CK(cudaMemcpyAsync(err, L.err, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return BLGPU_OK;
}

}  // extern "C"

// ---- host <-> box layout (staged through device memory, repacked on the GPU) ----
static int upload_field(blgpu_ctx *ctx, void *dst, const double *a, int n1, int n2, int n3) {
  CK(cudaMemcpyAsync(ctx->stage, a, (size_t)n1 * n2 * n3 * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
  if (ctx->fp64) launch_repack<double>(ctx->geo_box(), 0, ctx->stage, (double *)dst, n1, n2, n3, &ctx->sc->err, ctx->st);
  else launch_repack<float>(ctx->geo_box(), 0, ctx->stage, (float *)dst, n1, n2, n3, &ctx->sc->err, ctx->st);
  ctx->launches += 1;
  CK(cudaGetLastError());
  return BLGPU_OK;
}

static int download_field(blgpu_ctx *ctx, const void *src, double *a, int n1, int n2, int n3) {
  if (ctx->fp64) launch_repack<double>(ctx->geo_box(), 1, ctx->stage, (double *)src, n1, n2, n3, nullptr, ctx->st);
  else launch_repack<float>(ctx->geo_box(), 1, ctx->stage, (float *)src, n1, n2, n3, nullptr, ctx->st);
  ctx->launches += 1;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(a, ctx->stage, (size_t)n1 * n2 * n3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  return BLGPU_OK;
}

// after a synchronous upload: a non-finite host value (bit 32 of the device
// flag, set by the repack kernel) is reported and the bit cleared
static int take_upload_flag(blgpu_ctx *ctx, const char *what) {
  int f = 0;
  CK(cudaMemcpy(&f, &ctx->sc->err, sizeof f, cudaMemcpyDeviceToHost));
  if (!(f & 32)) return BLGPU_OK;
  f &= ~32;
  CK(cudaMemcpy(&ctx->sc->err, &f, sizeof f, cudaMemcpyHostToDevice));
  return set_err(ctx, BLGPU_EDEVICE, "%s: the host arrays hold a NaN or an infinity", what);
}

extern "C" {

int blgpu_set_nu_t(blgpu_ctx *ctx, const double *nu_t) {
  if (!ctx || !nu_t) return set_err(ctx, BLGPU_EINVAL, "blgpu_set_nu_t: null argument");
  if (!ctx->nut) return set_err(ctx, BLGPU_ESTATE, "blgpu_set_nu_t: context created with LES=0");
  CK(cudaSetDevice(ctx->cfg.device));
  int rc = upload_field(ctx, ctx->nut, nu_t, ctx->nxg, ctx->nyg, ctx->nzg);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->st));
  return take_upload_flag(ctx, "blgpu_set_nu_t");
}

int blgpu_upload_state(blgpu_ctx *ctx, const double *U, const double *V, const double *W, double t) {
  if (!ctx || !U || !V || !W) return set_err(ctx, BLGPU_EINVAL, "blgpu_upload_state: null argument");
  CK(cudaSetDevice(ctx->cfg.device));
  CK(cudaStreamSynchronize(ctx->st));
  ctx->cur = 0;
  ctx->old = 1;
  int rc = upload_field(ctx, ctx->S[0][0], U, ctx->nx, ctx->nyg, ctx->nzg);
  if (!rc) rc = upload_field(ctx, ctx->S[0][1], V, ctx->nxg, ctx->ny, ctx->nzg);
  if (!rc) rc = upload_field(ctx, ctx->S[0][2], W, ctx->nxg, ctx->nyg, ctx->nz);
  if (rc) return rc;
  for (int q = 0; q < 3; ++q)
    CK(cudaMemcpyAsync(ctx->S[1][q], ctx->S[0][q], (size_t)ctx->boxn * ctx->esz, cudaMemcpyDeviceToDevice, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  rc = take_upload_flag(ctx, "blgpu_upload_state");
  if (rc) {
    ctx->have_state = false;
    return rc;
  }
  Scalars h{};
  CK(cudaMemcpy(&h, ctx->sc, sizeof h, cudaMemcpyDeviceToHost));
  h.t = t;
  h.to = t;
  h.lmax[0] = h.lmax[1] = h.lmax[2] = 0ull;
  CK(cudaMemcpy(ctx->sc, &h, sizeof h, cudaMemcpyHostToDevice));
  ctx->have_state = true;
  return BLGPU_OK;
}

// t, to and the dt maxima of a newly uploaded state, on the compute stream
static __global__ void k_reset_scalars(Scalars *sc, double t) {
  sc->t = t;
  sc->to = t;
  sc->lmax[0] = sc->lmax[1] = sc->lmax[2] = 0ull;
}

// streams, staging buffers and events of the streamed transfers (first use)
static int xfer_setup(blgpu_ctx *ctx) {
  if (ctx->xin) return BLGPU_OK;
  const size_t n = (size_t)ctx->nxg * ctx->nyg * ctx->nzg * sizeof(double);
  for (int f = 0; f < 3; ++f) {
    int rc = dalloc(ctx, (void **)&ctx->stage_in[f], n);
    if (!rc) rc = dalloc(ctx, (void **)&ctx->stage_out[f], n);
    if (rc) return rc;
  }
  for (cudaEvent_t *e : {&ctx->ev_in_ready, &ctx->ev_in_free, &ctx->ev_out_ready, &ctx->ev_out_free})
    CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  // the "free" events start completed, so the first transfers do not wait
  CK(cudaEventRecord(ctx->ev_in_free, ctx->st));
  CK(cudaEventRecord(ctx->ev_out_free, ctx->st));
  CK(cudaStreamCreateWithFlags(&ctx->xout, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&ctx->xin, cudaStreamNonBlocking));
  return BLGPU_OK;
}

int blgpu_upload_state_async(blgpu_ctx *ctx, const double *U, const double *V, const double *W, double t) {
  if (!ctx || !U || !V || !W) return set_err(ctx, BLGPU_EINVAL, "blgpu_upload_state_async: null argument");
  CK(cudaSetDevice(ctx->cfg.device));
  int rc = xfer_setup(ctx);
  if (rc) return rc;
  const double *src[3] = {U, V, W};
  const int dims[3][3] = {{ctx->nx, ctx->nyg, ctx->nzg}, {ctx->nxg, ctx->ny, ctx->nzg}, {ctx->nxg, ctx->nyg, ctx->nz}};
  // H2D once the previous upload's repack has read the staging buffers
  CK(cudaStreamWaitEvent(ctx->xin, ctx->ev_in_free, 0));
  for (int f = 0; f < 3; ++f)
    CK(cudaMemcpyAsync(ctx->stage_in[f], src[f], (size_t)dims[f][0] * dims[f][1] * dims[f][2] * sizeof(double),
                       cudaMemcpyHostToDevice, ctx->xin));
  CK(cudaEventRecord(ctx->ev_in_ready, ctx->xin));
  // repack on the compute stream, after whatever it was doing
  CK(cudaStreamWaitEvent(ctx->st, ctx->ev_in_ready, 0));
  ctx->cur = 0;
  ctx->old = 1;
  for (int f = 0; f < 3; ++f) {
    if (ctx->fp64)
      launch_repack<double>(ctx->geo_box(), 0, ctx->stage_in[f], (double *)ctx->S[0][f], dims[f][0], dims[f][1],
                            dims[f][2], &ctx->sc->err, ctx->st);
    else
      launch_repack<float>(ctx->geo_box(), 0, ctx->stage_in[f], (float *)ctx->S[0][f], dims[f][0], dims[f][1],
                           dims[f][2], &ctx->sc->err, ctx->st);
    ctx->launches += 1;
  }
  CK(cudaEventRecord(ctx->ev_in_free, ctx->st));
  for (int q = 0; q < 3; ++q)
    CK(cudaMemcpyAsync(ctx->S[1][q], ctx->S[0][q], (size_t)ctx->boxn * ctx->esz, cudaMemcpyDeviceToDevice, ctx->st));
  k_reset_scalars<<<1, 1, 0, ctx->st>>>(ctx->sc, t);
  ctx->launches += 1;
  CK(cudaGetLastError());
  ctx->have_state = true;
  return BLGPU_OK;
}

int blgpu_download_state_async(blgpu_ctx *ctx, double *U, double *V, double *W) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  if (!ctx->have_state) return set_err(ctx, BLGPU_ESTATE, "blgpu_download_state_async: no state uploaded");
  CK(cudaSetDevice(ctx->cfg.device));
  int rc = xfer_setup(ctx);
  if (rc) return rc;
  double *dst[3] = {U, V, W};
  const int dims[3][3] = {{ctx->nx, ctx->nyg, ctx->nzg}, {ctx->nxg, ctx->ny, ctx->nzg}, {ctx->nxg, ctx->nyg, ctx->nz}};
  // repack into the staging buffers once the previous download has read them
  CK(cudaStreamWaitEvent(ctx->st, ctx->ev_out_free, 0));
  for (int f = 0; f < 3; ++f) {
    if (!dst[f]) continue;
    if (ctx->fp64)
      launch_repack<double>(ctx->geo_box(), 1, ctx->stage_out[f], (double *)ctx->S[ctx->cur][f], dims[f][0],
                            dims[f][1], dims[f][2], nullptr, ctx->st);
    else
      launch_repack<float>(ctx->geo_box(), 1, ctx->stage_out[f], (float *)ctx->S[ctx->cur][f], dims[f][0],
                           dims[f][1], dims[f][2], nullptr, ctx->st);
    ctx->launches += 1;
  }
  CK(cudaEventRecord(ctx->ev_out_ready, ctx->st));
  CK(cudaStreamWaitEvent(ctx->xout, ctx->ev_out_ready, 0));
  for (int f = 0; f < 3; ++f)
    if (dst[f])
      CK(cudaMemcpyAsync(dst[f], ctx->stage_out[f], (size_t)dims[f][0] * dims[f][1] * dims[f][2] * sizeof(double),
                         cudaMemcpyDeviceToHost, ctx->xout));
  CK(cudaEventRecord(ctx->ev_out_free, ctx->xout));
  CK(cudaGetLastError());
  return BLGPU_OK;
}

int blgpu_download_state(blgpu_ctx *ctx, double *U, double *V, double *W, double *P, double *t) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  if (!ctx->have_state) return set_err(ctx, BLGPU_ESTATE, "blgpu_download_state: no state uploaded");
  CK(cudaSetDevice(ctx->cfg.device));
  CK(cudaStreamSynchronize(ctx->st));
  int rc = 0;
  if (U && !rc) rc = download_field(ctx, ctx->S[ctx->cur][0], U, ctx->nx, ctx->nyg, ctx->nzg);
  if (V && !rc) rc = download_field(ctx, ctx->S[ctx->cur][1], V, ctx->nxg, ctx->ny, ctx->nzg);
  if (W && !rc) rc = download_field(ctx, ctx->S[ctx->cur][2], W, ctx->nxg, ctx->nyg, ctx->nz);
  if (P && !rc) rc = download_field(ctx, ctx->P, P, ctx->nxg, ctx->nyg, ctx->nzg);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->st));
  if (t) {
    Scalars h{};
    CK(cudaMemcpy(&h, ctx->sc, sizeof h, cudaMemcpyDeviceToHost));
    *t = h.t;
  }
  return BLGPU_OK;
}

int blgpu_set_dt(blgpu_ctx *ctx, double dt) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  CK(cudaSetDevice(ctx->cfg.device));
  CK(cudaStreamSynchronize(ctx->st));
  CK(cudaMemcpy(&ctx->sc->dt, &dt, sizeof dt, cudaMemcpyHostToDevice));
  return BLGPU_OK;
}

int blgpu_get_time(blgpu_ctx *ctx, double *t, double *dt) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  CK(cudaSetDevice(ctx->cfg.device));
  CK(cudaStreamSynchronize(ctx->st));
  Scalars h{};
  CK(cudaMemcpy(&h, ctx->sc, sizeof h, cudaMemcpyDeviceToHost));
  if (t) *t = h.t;
  if (dt) *dt = h.dt;
  return BLGPU_OK;
}

int blgpu_box(const blgpu_ctx *ctx, int *nx, int *ny, int *nz, double *nu) {
  if (!ctx) return BLGPU_EINVAL;
  if (nx) *nx = ctx->nx;
  if (ny) *ny = ctx->ny;
  if (nz) *nz = ctx->nz;
  if (nu) *nu = ctx->cfg.nu;
  return BLGPU_OK;
}

int blgpu_get_grid(blgpu_ctx *ctx, double *x, double *y, double *z) {
  if (!ctx || !x || !y || !z) return set_err(ctx, BLGPU_EINVAL, "blgpu_get_grid: null argument");
  if (!ctx->have_grid) return set_err(ctx, BLGPU_ESTATE, "blgpu_get_grid: no grid yet");
  for (int i = 0; i < ctx->nx; ++i) x[i] = ctx->x[i + 1];
  for (int j = 0; j < ctx->ny; ++j) y[j] = ctx->y[j + 1];
  for (int k = 0; k < ctx->nz; ++k) z[k] = ctx->z[k + 1];
  return BLGPU_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// step orchestration (all enqueued on ctx->st; capturable)
// ---------------------------------------------------------------------------
template <typename T>
static void enq_bc(blgpu_ctx *ctx, int b, int o, int rk_step) {
  T **S = reinterpret_cast<T **>(ctx->S[b]);
  T **So = reinterpret_cast<T **>(ctx->S[o]);
  ph_begin(ctx, PH_BC);
  launch_bc<T>(ctx->geo, ctx->bc, S[0], S[1], S[2], So[0], So[1], So[2], ctx->sc, ctx->rk_t[rk_step], ctx->qx_part,
               ctx->qy, ctx->length_y, ctx->st);
  ph_end(ctx, 2);
}

template <typename T>
static void enq_projection(blgpu_ctx *ctx, int b, int rk_step) {
  T **S = reinterpret_cast<T **>(ctx->S[b]);
  typedef typename vec2<T>::type T2;
  const Spec &s = ctx->spec;
  const FftPlan<T> &pl = *reinterpret_cast<const FftPlan<T> *>(ctx->fp64 ? (const void *)&ctx->pl64 : (const void *)&ctx->pl32);
  const bool mixed = !ctx->fp64;
  if (ctx->cf) {  // cuFFT comparison path (solve_poisson_gpu, projection.f90:93-204)
    const double *sp = ctx->d_spec;
    int r;
    ph_begin(ctx, PH_DIVDCT);
    r = cufft_path_forward<T>(ctx->cf, ctx->geo, s, S[0], S[1], S[2], ctx->st);
    if (r && !ctx->cf_status) ctx->cf_status = r;
    ph_end(ctx, 2);
    ph_begin(ctx, PH_THOMAS);
    cufft_path_extract_solve<T>(ctx->cf, s, ctx->post, ctx->piv, sp + s.NM, sp + 2 * s.NM, mixed ? ctx->kz0h : nullptr,
                                ctx->klow, ctx->st);
    if (mixed) launch_kz0_idct(s, ctx->kz0h, ctx->klow, ctx->cmat, ctx->kz0, ctx->kz0g, ctx->st);
    ph_end(ctx, mixed ? 4 : 2);
    ph_begin(ctx, PH_IDFTZ);
    r = cufft_path_inverse_z<T>(ctx->cf);
    if (r && !ctx->cf_status) ctx->cf_status = r;
    ph_end(ctx, 1);
    ph_begin(ctx, PH_IDCT);
    r = cufft_path_inverse_x<T>(ctx->cf, ctx->geo, s, ctx->post, (T *)ctx->rhs_p, ctx->st);
    if (r && !ctx->cf_status) ctx->cf_status = r;
    ph_end(ctx, 3);
    const MetT<T> &m = *reinterpret_cast<const MetT<T> *>(ctx->fp64 ? (const void *)&ctx->m64 : (const void *)&ctx->m32);
    ph_begin(ctx, PH_PROJECT);
    launch_project<T>(ctx->geo, m, (const T *)ctx->rhs_p, mixed ? ctx->kz0 : nullptr, mixed ? ctx->kz0g : nullptr,
                      S[0], S[1], S[2], (T *)ctx->P, ctx->sc, rk_step == 1 ? 1 : 0, ctx->tiles, ctx->st);
    ph_end(ctx, rk_step == 1 ? 2 : 1);
    return;
  }
  ph_begin(ctx, PH_DIVDCT);
  launch_div_dct<T>(ctx->geo, s, pl, S[0], S[1], S[2], (T *)ctx->R, ctx->tiles.dct_nw, ctx->tiles.xfft, ctx->st);
  ph_end(ctx, 1);
  // z transforms: tcgen05 (zdft 0 or 3), mma.sync TF32 (0 without tcgen05, or 2), FP32/FP64 sums (1)
  const int zd = ctx->tiles.zdft;
  const bool um = mixed && ctx->utab && (zd == 0 || zd == 3);
  const bool tc = mixed && !um && ctx->zfrag && (zd == 0 || zd == 2);
  ph_begin(ctx, PH_DFTZ);
  if (um) launch_zdft_umma(s, ctx->umaps, (float *)ctx->R, (float2 *)ctx->C, ctx->utab, 0, ctx->nsm, &ctx->sc->err, ctx->st);
  else if (tc) launch_zdft_tc(s, ctx->zmaps, (float *)ctx->R, (float2 *)ctx->C, ctx->zfrag, 0, ctx->nsm, &ctx->sc->err, ctx->st);
  else if (ctx->ztab64) launch_zdft64(s, (double *)ctx->R, (double2 *)ctx->C, (const double *)ctx->ztab64, 0, ctx->st);
  else launch_dft_z<T>(s, (T *)ctx->R, (T2 *)ctx->C, (const T2 *)ctx->ztab, 0, ctx->tiles.dftz_rk, ctx->st);
  ph_end(ctx, 1);
  const double *sp = ctx->d_spec;
  ph_begin(ctx, PH_THOMAS);
  // tiles where their tensor maps exist (NM <= 256): rows split over the CTA
  // (thomas 0 or 3) or one thread per mode (2); else the register ring
  const bool tiled = ctx->have_tmaps && ctx->tiles.thomas != 1;
  if (tiled)
    launch_thomas_tile<T>(s, ctx->tmaps, sp + s.NM, sp + 2 * s.NM, mixed ? ctx->kz0h : nullptr, ctx->klow,
                          &ctx->sc->err, ctx->wait_limit, ctx->tiles.thomas != 2, ctx->st);
  else
    launch_thomas<T>(s, (T2 *)ctx->C, ctx->piv, sp + s.NM, sp + 2 * s.NM, mixed ? ctx->kz0h : nullptr, ctx->klow,
                     ctx->st);
  if (mixed)  // the box-scale pressure (kz = 0, kx < klow) in FP64
    launch_kz0_idct(s, ctx->kz0h, ctx->klow, ctx->cmat, ctx->kz0, ctx->kz0g, ctx->st);
  ph_end(ctx, mixed ? 3 : 1);
  ph_begin(ctx, PH_IDFTZ);
  if (um) launch_zdft_umma(s, ctx->umaps, (float *)ctx->R, (float2 *)ctx->C, ctx->utab, 1, ctx->nsm, &ctx->sc->err, ctx->st);
  else if (tc) launch_zdft_tc(s, ctx->zmaps, (float *)ctx->R, (float2 *)ctx->C, ctx->zfrag, 1, ctx->nsm, &ctx->sc->err, ctx->st);
  else if (ctx->ztab64) launch_zdft64(s, (double *)ctx->R, (double2 *)ctx->C, (const double *)ctx->ztab64, 1, ctx->st);
  else launch_dft_z<T>(s, (T *)ctx->R, (T2 *)ctx->C, (const T2 *)ctx->ztab, 1, ctx->tiles.dftz_rk, ctx->st);
  ph_end(ctx, 1);
  ph_begin(ctx, PH_IDCT);
  launch_idct<T>(ctx->geo, s, pl, (const T *)ctx->R, (T *)ctx->rhs_p, ctx->tiles.idct_nw, ctx->tiles.xfft,
                 &ctx->sc->err, ctx->st);
  ph_end(ctx, 1);
  const MetT<T> &m = *reinterpret_cast<const MetT<T> *>(ctx->fp64 ? (const void *)&ctx->m64 : (const void *)&ctx->m32);
  ph_begin(ctx, PH_PROJECT);
  launch_project<T>(ctx->geo, m, (const T *)ctx->rhs_p, mixed ? ctx->kz0 : nullptr, mixed ? ctx->kz0g : nullptr,
                    S[0], S[1], S[2],
                    (T *)ctx->P, ctx->sc, rk_step == 1 ? 1 : 0, ctx->tiles, ctx->st);
  ph_end(ctx, rk_step == 1 ? 2 : 1);
}

template <typename T>
static void enq_rhs(blgpu_ctx *ctx, int mode, int in, int o, int outb, double c1, double c2) {
  T **Si = reinterpret_cast<T **>(ctx->S[in]);
  T **So = reinterpret_cast<T **>(ctx->S[o]);
  T **Sn = reinterpret_cast<T **>(ctx->S[outb]);
  T **F = reinterpret_cast<T **>(ctx->F1);
  const MetT<T> &m = *reinterpret_cast<const MetT<T> *>(ctx->fp64 ? (const void *)&ctx->m64 : (const void *)&ctx->m32);
  ph_begin(ctx, PH_RHS);
  launch_rhs_rk<T>(ctx->geo, m, mode, ctx->cfg.les_model != 0, Si[0], Si[1], Si[2], (const T *)ctx->nut, So[0], So[1],
                   So[2], F[0], F[1], F[2], Sn[0], Sn[1], Sn[2], ctx->sc, c1, c2, ctx->tiles,
                   ctx->have_rmaps ? &ctx->rmaps[in] : nullptr, ctx->have_rmaps ? &ctx->rmaps[o] : nullptr,
                   ctx->have_rmaps ? &ctx->rmaps[3] : nullptr, &ctx->sc->err, ctx->wait_limit, ctx->st);
  ph_end(ctx, 1);
}

// wall stress of the current model from fields U, W (the saved P and, with
// LES, the eddy viscosity); returns the number of kernels launched
template <typename T>
static int enq_wall_model(blgpu_ctx *ctx, const T *U, const T *W) {
  const T *nut = ctx->cfg.les_model ? (const T *)ctx->nut : nullptr;
  if (ctx->wm_mode == 1) {
    launch_law_of_wall<T>(ctx->geo, U, ctx->d_utau, ctx->d_iters, ctx->wm_jh, ctx->st);
    launch_wall_eq<T>(ctx->geo, ctx->d_utau, nut, ctx->d_wm, ctx->st);
    return 2;
  }
  launch_wall_mlp<T>(ctx->geo, ctx->wm_net, U, W, (const T *)ctx->P, nut, ctx->wm_jh, ctx->d_wm, ctx->st);
  return 1;
}

// One time step from buffer a.  Returns the index of the new state buffer.
template <typename T>
static int enq_step(blgpu_ctx *ctx, int a, bool with_dt) {
  const int b = (a + 1) % 3, c = (a + 2) % 3;
  if (with_dt && ctx->cfg.cfl > 0) {  // dt, and the step's start time saved by the same launch
    T **S = reinterpret_cast<T **>(ctx->S[a]);
    ph_begin(ctx, PH_DT);
    launch_dt<T>(ctx->geo, S[0], S[1], S[2], ctx->sc, ctx->cfg.cfl, ctx->dtvis, true, ctx->st);
    ph_end(ctx, 1);
  } else {
    ph_begin(ctx, PH_MISC);
    launch_set_time(ctx->sc, 0, 0.0, ctx->st);
    ph_end(ctx, 1);
  }
  if (ctx->lund.mode) {  // Lund inflow once per step from the step's start fields
    T **S = reinterpret_cast<T **>(ctx->S[a]);
    ph_begin(ctx, PH_BC);
    launch_lund<T>(ctx->geo, ctx->lund, S[0], S[1], S[2], ctx->sc, 1, ctx->st);
    ph_end(ctx, 3);
  }
  auto sub = [&](int mode, int in, int outb, double c1, double c2, double tc, int rk_step) {
    if (ctx->cfg.les_model == 1) {  // Smagorinsky from the substep's state (time_integration.f90:341-346)
      T **Si = reinterpret_cast<T **>(ctx->S[in]);
      ph_begin(ctx, PH_MISC);
      launch_smagorinsky<T>(ctx->geo, Si[0], Si[1], Si[2], ctx->d_cs2, (T *)ctx->nut, ctx->st);
      ph_end(ctx, 1);
    } else if (ctx->dyn) {  // dynamic Smagorinsky, same place (LES = 2, 3)
      T **Si = reinterpret_cast<T **>(ctx->S[in]);
      ph_begin(ctx, PH_MISC);
      ph_end(ctx, launch_dyn_smagorinsky<T>(ctx->geo, Si[0], Si[1], Si[2], ctx->dyn, ctx->cfg.les_model,
                                            (T *)ctx->nut, ctx->st));
    }
    if (ctx->wm_mode) {  // wall model from the substep's state (time_integration.f90:341-346)
      T **Si = reinterpret_cast<T **>(ctx->S[in]);
      ph_begin(ctx, PH_BC);
      ph_end(ctx, enq_wall_model<T>(ctx, Si[0], Si[2]));
    }
    enq_rhs<T>(ctx, mode, in, a, outb, c1, c2);
    ph_begin(ctx, PH_MISC);
    launch_set_time(ctx->sc, 1, tc, ctx->st);
    ph_end(ctx, 1);
    enq_bc<T>(ctx, outb, a, rk_step);
    enq_projection<T>(ctx, outb, rk_step);
    enq_bc<T>(ctx, outb, a, rk_step);
  };
  switch (ctx->cfg.rk_scheme) {
    case 3:  // time_integration.f90:305-465, initialization.f90:517-530
      sub(1, a, b, 8.0 / 15.0, 0.0, 8.0 / 15.0, 1);
      sub(2, b, c, 1.0 / 4.0, 5.0 / 12.0, 2.0 / 3.0, 2);
      sub(3, c, b, 1.0 / 4.0, 3.0 / 4.0, 1.0, 3);
      return b;
    case 2:  // time_integration.f90:145-300, initialization.f90:504-513
      sub(1, a, b, 1.0 / 2.0, 0.0, 1.0 / 2.0, 1);
      sub(2, b, c, 0.0, 1.0, 1.0, 2);
      return c;
    default:  // Euler, time_integration.f90:24-114 (rk_step = 3)
      sub(1, a, b, 1.0, 0.0, 1.0, 3);
      return b;
  }
}

// a cufftExec of the cuFFT comparison path refused work that was enqueued
static int cf_check(blgpu_ctx *ctx) {
  if (!ctx->cf_status) return BLGPU_OK;
  const int r = ctx->cf_status;
  ctx->cf_status = 0;
  return set_err(ctx, BLGPU_ECUDA, "cuFFT comparison path: cufftExec failed (cufftResult %d)", r);
}

static int step_once(blgpu_ctx *ctx, bool with_dt) {
  int nb = ctx->fp64 ? enq_step<double>(ctx, ctx->cur, with_dt) : enq_step<float>(ctx, ctx->cur, with_dt);
  ctx->old = ctx->cur;
  ctx->cur = nb;
  return cf_check(ctx);
}

extern "C" {

int blgpu_time_step(blgpu_ctx *ctx) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  if (!ctx->have_grid || !ctx->have_bc || !ctx->have_state)
    return set_err(ctx, BLGPU_ESTATE, "blgpu_time_step: grid, boundary and state must be set first");
  CK(cudaSetDevice(ctx->cfg.device));
  int rc = step_once(ctx, false);
  if (rc) return rc;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->st));
  return BLGPU_OK;
}

int blgpu_advance(blgpu_ctx *ctx, int nsteps) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  if (nsteps < 0) return set_err(ctx, BLGPU_EINVAL, "blgpu_advance: nsteps < 0");
  if (!ctx->have_grid || !ctx->have_bc || !ctx->have_state)
    return set_err(ctx, BLGPU_ESTATE, "blgpu_advance: grid, boundary and state must be set first");
  CK(cudaSetDevice(ctx->cfg.device));
  for (int n = 0; n < (nsteps > 0 ? nsteps : 1); ++n) {
    const int a = ctx->cur;
    if (!ctx->graph[a]) {
      cudaGraph_t gr = nullptr;
      CK(cudaStreamBeginCapture(ctx->st, cudaStreamCaptureModeRelaxed));
      const long long l0 = ctx->launches;
      const int nb = ctx->fp64 ? enq_step<double>(ctx, a, true) : enq_step<float>(ctx, a, true);
      ctx->graph_launches[a] = ctx->launches - l0;
      ctx->launches = l0;
      cudaError_t e = cudaStreamEndCapture(ctx->st, &gr);
      if (e != cudaSuccess) return check_cuda(ctx, e, "cudaStreamEndCapture");
      if (ctx->cf_status) {
        cudaGraphDestroy(gr);
        return cf_check(ctx);
      }
      e = cudaGraphInstantiate(&ctx->graph[a], gr, 0);
      cudaGraphDestroy(gr);
      if (e != cudaSuccess) return check_cuda(ctx, e, "cudaGraphInstantiate");
      ctx->graph_next[a] = nb;
    }
    if (nsteps == 0) break;  // capture only
    CK(cudaGraphLaunch(ctx->graph[a], ctx->st));
    ctx->launches += ctx->graph_launches[a];
    ctx->old = a;
    ctx->cur = ctx->graph_next[a];
  }
  CK(cudaGetLastError());
  return BLGPU_OK;
}

int blgpu_sync(blgpu_ctx *ctx) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  CK(cudaSetDevice(ctx->cfg.device));
  CK(cudaStreamSynchronize(ctx->st));
  if (ctx->xin) CK(cudaStreamSynchronize(ctx->xin));
  if (ctx->xout) CK(cudaStreamSynchronize(ctx->xout));
  return device_flag(ctx);
}

int blgpu_compute_dt(blgpu_ctx *ctx, double *dt) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  if (!ctx->have_grid || !ctx->have_state) return set_err(ctx, BLGPU_ESTATE, "blgpu_compute_dt: no grid/state");
  CK(cudaSetDevice(ctx->cfg.device));
  if (ctx->cfg.cfl < 0) {
    double v = -ctx->cfg.cfl;
    CK(cudaStreamSynchronize(ctx->st));
    CK(cudaMemcpy(&ctx->sc->dt, &v, sizeof v, cudaMemcpyHostToDevice));
  } else if (ctx->fp64) {
    double **S = reinterpret_cast<double **>(ctx->S[ctx->cur]);
    launch_dt<double>(ctx->geo, S[0], S[1], S[2], ctx->sc, ctx->cfg.cfl, ctx->dtvis, false, ctx->st);
  } else {
    float **S = reinterpret_cast<float **>(ctx->S[ctx->cur]);
    launch_dt<float>(ctx->geo, S[0], S[1], S[2], ctx->sc, ctx->cfg.cfl, ctx->dtvis, false, ctx->st);
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->st));
  if (dt) CK(cudaMemcpy(dt, &ctx->sc->dt, sizeof(double), cudaMemcpyDeviceToHost));
  return BLGPU_OK;
}

int blgpu_compute_rhs(blgpu_ctx *ctx, const double *U, const double *V, const double *W, double *rhs_u,
                      double *rhs_v, double *rhs_w) {
  if (!ctx || !U || !V || !W) return set_err(ctx, BLGPU_EINVAL, "blgpu_compute_rhs: null argument");
  if (!ctx->have_grid) return set_err(ctx, BLGPU_ESTATE, "blgpu_compute_rhs: no grid");
  CK(cudaSetDevice(ctx->cfg.device));
  CK(cudaStreamSynchronize(ctx->st));
  // scratch buffer: the one that is neither the current state nor Uo
  const int sb = 3 - ctx->cur - ctx->old;
  int rc = upload_field(ctx, ctx->S[sb][0], U, ctx->nx, ctx->nyg, ctx->nzg);
  if (!rc) rc = upload_field(ctx, ctx->S[sb][1], V, ctx->nxg, ctx->ny, ctx->nzg);
  if (!rc) rc = upload_field(ctx, ctx->S[sb][2], W, ctx->nxg, ctx->nyg, ctx->nz);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->st));
  rc = take_upload_flag(ctx, "blgpu_compute_rhs");
  if (rc) return rc;
  if (ctx->fp64) enq_rhs<double>(ctx, 0, sb, sb, sb, 0.0, 0.0);
  else enq_rhs<float>(ctx, 0, sb, sb, sb, 0.0, 0.0);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->st));
  const int nx = ctx->nx, ny = ctx->ny, nz = ctx->nz, nxg = ctx->nxg, nyg = ctx->nyg, nzg = ctx->nzg;
  std::vector<double> full;
  auto grab = [&](int q, double *out, int i1, int j1, int k1) -> int {
    // interior (2:i1, 2:j1, 2:k1) of component q, compact
    if (!out) return BLGPU_OK;
    full.assign((size_t)nxg * nyg * nzg, 0.0);
    int r = download_field(ctx, ctx->F1[q], full.data(), nxg, nyg, nzg);
    if (r) return r;
    CK(cudaStreamSynchronize(ctx->st));
    const int e1 = i1 - 1, e2 = j1 - 1;
    for (int k = 2; k <= k1; ++k)
      for (int j = 2; j <= j1; ++j)
        for (int i = 2; i <= i1; ++i)
          out[((size_t)(k - 2) * e2 + (j - 2)) * e1 + (i - 2)] = full[((size_t)(k - 1) * nyg + (j - 1)) * nxg + (i - 1)];
    return BLGPU_OK;
  };
  rc = grab(0, rhs_u, nx - 1, nyg - 1, nzg - 1);
  if (!rc) rc = grab(1, rhs_v, nxg - 1, ny - 1, nzg - 1);
  if (!rc) rc = grab(2, rhs_w, nxg - 1, nyg - 1, nz - 1);
  return rc;
}

int blgpu_apply_bc(blgpu_ctx *ctx, int rk_step) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  if (rk_step < 1 || rk_step > 3) return set_err(ctx, BLGPU_EINVAL, "blgpu_apply_bc: rk_step %d", rk_step);
  if (!ctx->have_grid || !ctx->have_bc || !ctx->have_state)
    return set_err(ctx, BLGPU_ESTATE, "blgpu_apply_bc: grid, boundary and state must be set first");
  CK(cudaSetDevice(ctx->cfg.device));
  if (ctx->fp64) enq_bc<double>(ctx, ctx->cur, ctx->old, rk_step);
  else enq_bc<float>(ctx, ctx->cur, ctx->old, rk_step);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->st));
  return BLGPU_OK;
}

int blgpu_projection(blgpu_ctx *ctx, int rk_step) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  if (!ctx->have_grid || !ctx->have_state) return set_err(ctx, BLGPU_ESTATE, "blgpu_projection: no grid/state");
  CK(cudaSetDevice(ctx->cfg.device));
  if (ctx->fp64) enq_projection<double>(ctx, ctx->cur, rk_step);
  else enq_projection<float>(ctx, ctx->cur, rk_step);
  int rc = cf_check(ctx);
  if (rc) return rc;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->st));
  return BLGPU_OK;
}

int blgpu_get_rhs_p(blgpu_ctx *ctx, double *rhs_p) {
  if (!ctx || !rhs_p) return set_err(ctx, BLGPU_EINVAL, "blgpu_get_rhs_p: null argument");
  CK(cudaSetDevice(ctx->cfg.device));
  CK(cudaStreamSynchronize(ctx->st));
  const int nxg = ctx->nxg, nyg = ctx->nyg, nzg = ctx->nzg;
  std::vector<double> full((size_t)nxg * nyg * nzg);
  int rc = download_field(ctx, ctx->rhs_p, full.data(), nxg, nyg, nzg);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->st));
  const int e1 = nxg - 2, e2 = nyg - 2;
  std::vector<double> p0;  // mixed form: the FP64 z-mean part, [j-2][i-2] of pitch N
  const int N = ctx->spec.N;
  if (ctx->kz0) {
    p0.resize((size_t)ctx->spec.NM * N);
    CK(cudaMemcpy(p0.data(), ctx->kz0, p0.size() * sizeof(double), cudaMemcpyDeviceToHost));
  }
  for (int k = 2; k <= nzg; ++k)
    for (int j = 2; j <= nyg - 1; ++j)
      for (int i = 2; i <= nxg - 1; ++i) {
        double v = (k == nzg) ? 0.0 : full[((size_t)(k - 1) * nyg + (j - 1)) * nxg + (i - 1)];
        if (!p0.empty() && k < nzg) v += p0[(size_t)(j - 2) * N + std::min(i - 2, N - 1)];
        rhs_p[((size_t)(k - 2) * e2 + (j - 2)) * e1 + (i - 2)] = v;
      }
  return BLGPU_OK;
}

int blgpu_max_divergence(blgpu_ctx *ctx, double *max_div) {
  if (!ctx || !max_div) return set_err(ctx, BLGPU_EINVAL, "blgpu_max_divergence: null argument");
  if (!ctx->have_grid || !ctx->have_state) return set_err(ctx, BLGPU_ESTATE, "blgpu_max_divergence: no grid/state");
  CK(cudaSetDevice(ctx->cfg.device));
  CK(cudaMemsetAsync(ctx->d_maxdiv, 0, sizeof(unsigned long long), ctx->st));
  if (ctx->fp64) {
    double **S = reinterpret_cast<double **>(ctx->S[ctx->cur]);
    launch_maxdiv<double>(ctx->geo, S[0], S[1], S[2], ctx->d_maxdiv, ctx->st);
  } else {
    float **S = reinterpret_cast<float **>(ctx->S[ctx->cur]);
    launch_maxdiv<float>(ctx->geo, S[0], S[1], S[2], ctx->d_maxdiv, ctx->st);
  }
  CK(cudaGetLastError());
  unsigned long long bits = 0;
  CK(cudaMemcpyAsync(&bits, ctx->d_maxdiv, sizeof bits, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  double v;
  memcpy(&v, &bits, sizeof v);
  *max_div = v;
  return BLGPU_OK;
}

int blgpu_set_wait_limit(blgpu_ctx *ctx, int polls) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  ctx->wait_limit = polls < 0 ? -1 : polls;
  drop_graphs(ctx);  // the limit is a kernel argument of the captured steps
  return BLGPU_OK;
}

int blgpu_phase_times(blgpu_ctx *ctx, int nsteps, double *ms, long long *kernels, int nphase) {
  if (!ctx || !ms || nphase < PH_N || nsteps < 1) return set_err(ctx, BLGPU_EINVAL, "blgpu_phase_times: bad argument");
  if (!ctx->have_grid || !ctx->have_bc || !ctx->have_state)
    return set_err(ctx, BLGPU_ESTATE, "blgpu_phase_times: grid, boundary and state must be set first");
  CK(cudaSetDevice(ctx->cfg.device));
  CK(cudaStreamSynchronize(ctx->st));
  for (int p = 0; p < nphase; ++p) {
    ms[p] = 0.0;
    if (kernels) kernels[p] = 0;
  }
  ctx->prof_on = true;
  ctx->marks.clear();
  int rc = 0;
  for (int n = 0; n < nsteps && !rc; ++n) rc = step_once(ctx, true);
  ctx->prof_on = false;
  cudaError_t e = cudaStreamSynchronize(ctx->st);
  for (auto &mk : ctx->marks) {
    float t = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&t, mk.a, mk.b);
    ms[mk.phase] += t;
    if (kernels) kernels[mk.phase] += mk.nk;
    cudaEventDestroy(mk.a);
    cudaEventDestroy(mk.b);
  }
  ctx->marks.clear();
  CK(e);
  return rc;
}

long long blgpu_kernel_launches(const blgpu_ctx *ctx) { return ctx ? ctx->launches : 0; }

int blgpu_advance_timed(blgpu_ctx *ctx, int nsteps, double *ms) {
  if (!ctx || !ms) return set_err(ctx, BLGPU_EINVAL, "blgpu_advance_timed: null argument");
  CK(cudaSetDevice(ctx->cfg.device));
  if (ctx->have_grid && ctx->have_bc && ctx->have_state && !ctx->graph[ctx->cur]) {
    // capture outside the timed region
    int rc = blgpu_advance(ctx, 0);
    if (rc) return rc;
  }
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  CK(cudaEventRecord(a, ctx->st));
  int rc = blgpu_advance(ctx, nsteps);
  cudaEventRecord(b, ctx->st);
  cudaError_t e = cudaEventSynchronize(b);
  float t = 0.f;
  if (!rc && e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc) return rc;
  CK(e);
  *ms = (double)t;
  return device_flag(ctx);
}

int blgpu_eddy_viscosity(blgpu_ctx *ctx) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  if (!ctx->nut) return set_err(ctx, BLGPU_ESTATE, "blgpu_eddy_viscosity: context created with LES=0");
  if (!ctx->have_grid || !ctx->have_state) return set_err(ctx, BLGPU_ESTATE, "blgpu_eddy_viscosity: no grid/state");
  CK(cudaSetDevice(ctx->cfg.device));
  if (ctx->fp64) {
    double **S = reinterpret_cast<double **>(ctx->S[ctx->cur]);
    if (ctx->dyn)
      ctx->launches += launch_dyn_smagorinsky<double>(ctx->geo, S[0], S[1], S[2], ctx->dyn, ctx->cfg.les_model,
                                                      (double *)ctx->nut, ctx->st);
    else
      launch_smagorinsky<double>(ctx->geo, S[0], S[1], S[2], ctx->d_cs2, (double *)ctx->nut, ctx->st);
  } else {
    float **S = reinterpret_cast<float **>(ctx->S[ctx->cur]);
    if (ctx->dyn)
      ctx->launches += launch_dyn_smagorinsky<float>(ctx->geo, S[0], S[1], S[2], ctx->dyn, ctx->cfg.les_model,
                                                     (float *)ctx->nut, ctx->st);
    else
      launch_smagorinsky<float>(ctx->geo, S[0], S[1], S[2], ctx->d_cs2, (float *)ctx->nut, ctx->st);
  }
  if (!ctx->dyn) ctx->launches += 1;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->st));
  return BLGPU_OK;
}

int blgpu_get_nu_t(blgpu_ctx *ctx, double *nu_t) {
  if (!ctx || !nu_t) return set_err(ctx, BLGPU_EINVAL, "blgpu_get_nu_t: null argument");
  if (!ctx->nut) {  // LES = 0: the reference's nu_t stays zero
    memset(nu_t, 0, sizeof(double) * (size_t)ctx->nxg * ctx->nyg * ctx->nzg);
    return BLGPU_OK;
  }
  CK(cudaSetDevice(ctx->cfg.device));
  CK(cudaStreamSynchronize(ctx->st));
  int rc = download_field(ctx, ctx->nut, nu_t, ctx->nxg, ctx->nyg, ctx->nzg);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->st));
  return BLGPU_OK;
}

int blgpu_statistics(blgpu_ctx *ctx, double *means, double *nu_t_mean, double *Cf, double *dUdy_wall,
                     double *scalars) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  if (!ctx->have_grid || !ctx->have_state) return set_err(ctx, BLGPU_ESTATE, "blgpu_statistics: no grid/state");
  CK(cudaSetDevice(ctx->cfg.device));
  if (ctx->fp64) {
    double **S = reinterpret_cast<double **>(ctx->S[ctx->cur]);
    launch_stats<double>(ctx->geo, S[0], S[1], S[2], (const double *)ctx->P, (const double *)ctx->nut, ctx->d_stats,
                         ctx->st);
  } else {
    float **S = reinterpret_cast<float **>(ctx->S[ctx->cur]);
    launch_stats<float>(ctx->geo, S[0], S[1], S[2], (const float *)ctx->P, (const float *)ctx->nut, ctx->d_stats,
                        ctx->st);
  }
  ctx->launches += 1;
  CK(cudaGetLastError());
  const int nx = ctx->nx, ny = ctx->ny, nxg = ctx->nxg, nyg = ctx->nyg;
  const size_t pl = (size_t)nx * ny, ntot = 9 * pl + (size_t)nxg * nyg + 2 * (size_t)nx;
  std::vector<double> h(ntot);
  CK(cudaMemcpyAsync(h.data(), ctx->d_stats, ntot * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  if (means) memcpy(means, h.data(), 9 * pl * sizeof(double));
  const double *ntm = h.data() + 9 * pl;
  if (nu_t_mean) memcpy(nu_t_mean, ntm, (size_t)nxg * nyg * sizeof(double));
  const double *a1 = ntm + (size_t)nxg * nyg, *a2 = a1 + nx;
  const double *Um = h.data(), *UV = h.data() + 6 * pl;
  // statistics.f90:138-201 (wall gradient, Cf, inlet theta, delta99, Reynolds numbers)
  std::vector<double> dU(nx), cf(nx);
  for (int ii = 1; ii <= nx; ++ii) dU[ii - 1] = (a2[ii - 1] - a1[ii - 1]) / (ctx->yg[2] - ctx->yg[1]);
  for (int ii = 1; ii <= nx; ++ii) {
    const double tau = 0.25 * (ntm[ii - 1] + ntm[(size_t)nxg + ii - 1] + ntm[ii] + ntm[(size_t)nxg + ii]) * dU[ii - 1];
    cf[ii - 1] = 2.0 * (-UV[ii - 1] + ctx->cfg.nu * dU[ii - 1] + tau) / 1.0;
  }
  if (Cf) memcpy(Cf, cf.data(), nx * sizeof(double));
  if (dUdy_wall) memcpy(dUdy_wall, dU.data(), nx * sizeof(double));
  if (scalars) {
    const double Uinf = 1.0;
    double theta = 0.0;
    for (int j = 2; j <= ny; ++j) {
      const double tj = Um[(size_t)(j - 1) * nx] / Uinf * (1.0 - Um[(size_t)(j - 1) * nx] / Uinf);
      const double tm = Um[(size_t)(j - 2) * nx] / Uinf * (1.0 - Um[(size_t)(j - 2) * nx] / Uinf);
      theta = theta + 0.5 * (tj + tm) * (ctx->y[j] - ctx->y[j - 1]);
    }
    int jref = 0;
    for (int j = 1; j <= ny; ++j)
      if (Um[(size_t)(j - 1) * nx] >= 0.99 * Uinf) { jref = j; break; }
    if (jref < 2) jref = 2;
    const double u1 = Um[(size_t)(jref - 2) * nx], u2 = Um[(size_t)(jref - 1) * nx];
    const double w1 = (0.99 * Uinf - u1) / (u2 - u1), w0 = 1.0 - w1;
    const double d99 = w1 * ctx->y[jref] + w0 * ctx->y[jref - 1];
    scalars[0] = theta;
    scalars[1] = d99;
    scalars[2] = ctx->x[1] * Uinf / ctx->cfg.nu;
    scalars[3] = theta * Uinf / ctx->cfg.nu;
    scalars[4] = d99 * Uinf / ctx->cfg.nu;
  }
  return BLGPU_OK;
}

int blgpu_law_of_wall(blgpu_ctx *ctx, double *utau, int *iters_max) {
  if (!ctx || !utau) return set_err(ctx, BLGPU_EINVAL, "blgpu_law_of_wall: null argument");
  if (!ctx->have_grid || !ctx->have_state) return set_err(ctx, BLGPU_ESTATE, "blgpu_law_of_wall: no grid/state");
  CK(cudaSetDevice(ctx->cfg.device));
  const int nx = ctx->nx;
  CK(cudaMemcpyAsync(ctx->d_utau, utau, nx * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
  if (ctx->fp64)
    launch_law_of_wall<double>(ctx->geo, ((double **)ctx->S[ctx->cur])[0], ctx->d_utau, ctx->d_iters, 3, ctx->st);
  else
    launch_law_of_wall<float>(ctx->geo, ((float **)ctx->S[ctx->cur])[0], ctx->d_utau, ctx->d_iters, 3, ctx->st);
  ctx->launches += 1;
  CK(cudaGetLastError());
  std::vector<int> it(nx, 0);
  CK(cudaMemcpyAsync(utau, ctx->d_utau, nx * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaMemcpyAsync(it.data(), ctx->d_iters, nx * sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  // utau_model(1) = utau_model(2); utau_model(nx) = utau_model(nx-1) (wallmodel.f90:1979-1980)
  utau[0] = utau[1];
  utau[nx - 1] = utau[nx - 2];
  int mx = 0;
  for (int i = 2; i <= nx - 1; ++i) mx = it[i - 1] > mx ? it[i - 1] : mx;
  if (iters_max) *iters_max = mx;
  return BLGPU_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// wall models and the training-sample extractor
// ---------------------------------------------------------------------------
extern "C" {

int blgpu_set_wall_model(blgpu_ctx *ctx, int mode, int jh, const blgpu_mlp *net) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  if (mode < 0 || mode > 2) return set_err(ctx, BLGPU_EINVAL, "blgpu_set_wall_model: mode %d not in 0..2", mode);
  if (mode && (jh < 2 || jh > ctx->nyg - 1))
    return set_err(ctx, BLGPU_EINVAL, "blgpu_set_wall_model: row %d outside 2..nyg-1", jh);
  if (mode == 2 && !net) return set_err(ctx, BLGPU_EINVAL, "blgpu_set_wall_model: mode 2 needs a network");
  if (mode == 2 && blgpu_mlp_device(net) != ctx->cfg.device)
    return set_err(ctx, BLGPU_EINVAL, "blgpu_set_wall_model: network on another device");
  if (mode && !ctx->have_grid) return set_err(ctx, BLGPU_ESTATE, "blgpu_set_wall_model: grid first");
  CK(cudaSetDevice(ctx->cfg.device));
  CK(cudaStreamSynchronize(ctx->st));
  drop_graphs(ctx);
  ctx->wm_mode = mode;
  ctx->wm_jh = jh;
  ctx->wm_net = mode == 2 ? blgpu_mlp_view(net) : MlpDev{};
  const size_t nw = (size_t)(ctx->nx - 2) * (ctx->nzg - 3);
  ctx->bc.wm_ax = mode ? ctx->d_wm : nullptr;
  ctx->bc.wm_az = mode == 2 ? ctx->d_wm + nw : nullptr;
  if (mode == 1) {  // Newton's first guess: utau_ref (initialization.f90:744-745)
    std::vector<double> u(ctx->nx);
    for (int i = 1; i <= ctx->nx; ++i) u[i - 1] = std::sqrt(0.5 * 0.027 * std::pow(ctx->x[i] / ctx->cfg.nu, -1.0 / 7.0));
    CK(cudaMemcpy(ctx->d_utau, u.data(), ctx->nx * sizeof(double), cudaMemcpyHostToDevice));
  }
  return BLGPU_OK;
}

// the current model's wall stress on the current state at the wall points
// (i = 2..nx-1 fastest, k = 2..nzg-2)
int blgpu_wall_stress(blgpu_ctx *ctx, double *tau_x, double *tau_z) {
  if (!ctx) return set_err(ctx, BLGPU_EINVAL, "null ctx");
  if (!ctx->wm_mode) return set_err(ctx, BLGPU_ESTATE, "blgpu_wall_stress: no wall model set");
  if (!ctx->have_grid || !ctx->have_state) return set_err(ctx, BLGPU_ESTATE, "blgpu_wall_stress: no grid/state");
  CK(cudaSetDevice(ctx->cfg.device));
  if (ctx->fp64) {
    double **S = reinterpret_cast<double **>(ctx->S[ctx->cur]);
    ctx->launches += enq_wall_model<double>(ctx, S[0], S[2]);
  } else {
    float **S = reinterpret_cast<float **>(ctx->S[ctx->cur]);
    ctx->launches += enq_wall_model<float>(ctx, S[0], S[2]);
  }
  CK(cudaGetLastError());
  const size_t nw = (size_t)(ctx->nx - 2) * (ctx->nzg - 3);
  if (tau_x) CK(cudaMemcpyAsync(tau_x, ctx->d_wm + 2 * nw, nw * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  if (tau_z) CK(cudaMemcpyAsync(tau_z, ctx->d_wm + 3 * nw, nw * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return BLGPU_OK;
}

// append the wall samples of the solver's current state (features at row
// jh, stress of the resolved wall gradient) to the network's training set
int blgpu_mlp_sample(blgpu_mlp *m, blgpu_ctx *ctx, int jh) {
  if (!ctx || !m) return set_err(ctx, BLGPU_EINVAL, "blgpu_mlp_sample: null argument");
  if (jh < 2 || jh > ctx->nyg - 1) return set_err(ctx, BLGPU_EINVAL, "blgpu_mlp_sample: row %d outside 2..nyg-1", jh);
  if (!ctx->have_grid || !ctx->have_state) return set_err(ctx, BLGPU_ESTATE, "blgpu_mlp_sample: no grid/state");
  if (blgpu_mlp_device(m) != ctx->cfg.device) return set_err(ctx, BLGPU_EINVAL, "blgpu_mlp_sample: other device");
  CK(cudaSetDevice(ctx->cfg.device));
  CK(cudaStreamSynchronize(ctx->st));
  CK(cudaStreamSynchronize(blgpu_mlp_stream(m)));
  const int rows = (ctx->nx - 2) * (ctx->nzg - 3);
  float *X = nullptr, *Tg = nullptr;
  int rc = blgpu_mlp_reserve(m, rows, &X, &Tg);
  if (rc) return set_err(ctx, rc, "blgpu_mlp_sample: %s", blgpu_mlp_last_error(m));
  if (ctx->fp64) {
    double **S = reinterpret_cast<double **>(ctx->S[ctx->cur]);
    launch_wall_samples<double>(ctx->geo, S[0], S[2], (const double *)ctx->P, jh, X, Tg, ctx->st);
  } else {
    float **S = reinterpret_cast<float **>(ctx->S[ctx->cur]);
    launch_wall_samples<float>(ctx->geo, S[0], S[2], (const float *)ctx->P, jh, X, Tg, ctx->st);
  }
  ctx->launches += 1;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->st));
  blgpu_mlp_commit(m, rows);
  return BLGPU_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// launch shapes and their autotuner
// ---------------------------------------------------------------------------
static int tiles_check(blgpu_ctx *ctx, const Tiles &t) {
  auto pow2 = [](int v) { return v == 1 || v == 2 || v == 4 || v == 8; };
  if (t.rhs_kc < 0 || t.rhs_kc > 256) return set_err(ctx, BLGPU_EINVAL, "tiles: rhs_kc %d outside 0..256", t.rhs_kc);
  if (t.rhs_by != 0 && !pow2(t.rhs_by)) return set_err(ctx, BLGPU_EINVAL, "tiles: rhs_by %d not in {1,2,4,8}", t.rhs_by);
  if (t.proj_by != 0 && !pow2(t.proj_by))
    return set_err(ctx, BLGPU_EINVAL, "tiles: proj_by %d not in {1,2,4,8}", t.proj_by);
  if (t.dftz_rk != 0 && t.dftz_rk != 4 && t.dftz_rk != 8)
    return set_err(ctx, BLGPU_EINVAL, "tiles: dftz_rk %d not in {4,8}", t.dftz_rk);
  if (t.xfft < 0 || t.xfft > 2) return set_err(ctx, BLGPU_EINVAL, "tiles: xfft %d not in {0,1,2}", t.xfft);
  const int split = t.xfft == 1 ? 0 : ctx->fp64 ? (xfft_split(ctx->spec.N) == 29 ? 29 : 0) : xfft_split(ctx->spec.N);
  if (t.xfft == 2 && !split)
    return set_err(ctx, BLGPU_EINVAL, "tiles: xfft 2 (two-pass x transforms) not built for N = %d in %s", ctx->spec.N,
                   ctx->fp64 ? "FP64" : "FP32");
  const int maxnw = dct_max_lines((int)ctx->esz, split);
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->cfg.device);
  for (int q = 0; q < 2; ++q) {
    const int nw = q ? t.idct_nw : t.dct_nw;
    const char *name = q ? "idct_nw" : "dct_nw";
    if (nw < 0 || nw > maxnw) return set_err(ctx, BLGPU_EINVAL, "tiles: %s %d outside 0..%d", name, nw, maxnw);
    if (nw > 0) {
      const size_t sm = dct_smem_bytes(ctx->spec.N, (int)ctx->esz, nw, split);
      if (sm > (size_t)optin)
        return set_err(ctx, BLGPU_EINVAL, "tiles: %s %d needs %zu B of shared memory (> %d)", name, nw, sm, optin);
    }
  }
  if (t.zdft < 0 || t.zdft > 3) return set_err(ctx, BLGPU_EINVAL, "tiles: zdft %d not in {0,1,2,3}", t.zdft);
  if (t.rhs_pts < 0 || t.rhs_pts > 4) return set_err(ctx, BLGPU_EINVAL, "tiles: rhs_pts %d not in {0,...,4}", t.rhs_pts);
  if (t.thomas < 0 || t.thomas > 3) return set_err(ctx, BLGPU_EINVAL, "tiles: thomas %d not in {0,...,3}", t.thomas);
  return BLGPU_OK;
}

// state of a context that stepping changes: the current fields, the device
// scalars and the Lund running means
struct Snapshot {
  void *f[3] = {nullptr, nullptr, nullptr};
  Scalars sc{};
  std::vector<double> lund;
  int cur = 0, old = 1;
};

static int snap_take(blgpu_ctx *ctx, Snapshot &sn) {
  const size_t box = (size_t)ctx->boxn * ctx->esz;
  for (int q = 0; q < 3; ++q) {
    cudaError_t e = cudaMalloc(&sn.f[q], box);
    if (e != cudaSuccess) return check_cuda(ctx, e, "autotune snapshot");
    CK(cudaMemcpyAsync(sn.f[q], ctx->S[ctx->cur][q], box, cudaMemcpyDeviceToDevice, ctx->st));
  }
  CK(cudaMemcpyAsync(&sn.sc, ctx->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, ctx->st));
  sn.lund.resize(2 * (size_t)ctx->nyg + 2 * (size_t)ctx->ny);
  CK(cudaMemcpyAsync(sn.lund.data(), ctx->lund.mean, sn.lund.size() * sizeof(double), cudaMemcpyDeviceToHost,
                     ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  sn.cur = ctx->cur;
  sn.old = ctx->old;
  return BLGPU_OK;
}

static int snap_restore(blgpu_ctx *ctx, Snapshot &sn) {
  const size_t box = (size_t)ctx->boxn * ctx->esz;
  CK(cudaStreamSynchronize(ctx->st));
  ctx->cur = sn.cur;
  ctx->old = sn.old;
  for (int q = 0; q < 3; ++q)
    if (sn.f[q]) CK(cudaMemcpyAsync(ctx->S[ctx->cur][q], sn.f[q], box, cudaMemcpyDeviceToDevice, ctx->st));
  CK(cudaMemcpyAsync(ctx->sc, &sn.sc, sizeof(Scalars), cudaMemcpyHostToDevice, ctx->st));
  CK(cudaMemcpyAsync(ctx->lund.mean, sn.lund.data(), sn.lund.size() * sizeof(double), cudaMemcpyHostToDevice,
                     ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return BLGPU_OK;
}

static void snap_free(Snapshot &sn) {
  for (int q = 0; q < 3; ++q)
    if (sn.f[q]) cudaFree(sn.f[q]);
  sn.f[0] = sn.f[1] = sn.f[2] = nullptr;
}

// device time of `steps` graph-replayed steps after one untimed step
static int time_steps(blgpu_ctx *ctx, int steps, double *ms) {
  int rc = blgpu_advance(ctx, 1);
  if (rc) return rc;
  rc = blgpu_advance_timed(ctx, steps, ms);
  if (rc) return rc;
  *ms /= (double)steps;
  return BLGPU_OK;
}

extern "C" {

int blgpu_set_tiles(blgpu_ctx *ctx, const int *tiles, int n) {
  if (!ctx || !tiles || n < 5) return set_err(ctx, BLGPU_EINVAL, "blgpu_set_tiles: need 5 to 10 values");
  Tiles t{tiles[0],
          tiles[1],
          tiles[2],
          tiles[3],
          tiles[4],
          n >= 6 ? tiles[5] : ctx->tiles.zdft,
          n >= 7 ? tiles[6] : ctx->tiles.rhs_pts,
          n >= 8 ? tiles[7] : ctx->tiles.thomas,
          n >= 9 ? tiles[8] : ctx->tiles.idct_nw,
          n >= 10 ? tiles[9] : ctx->tiles.xfft};
  int rc = tiles_check(ctx, t);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->cfg.device));
  CK(cudaStreamSynchronize(ctx->st));
  ctx->tiles = t;
  drop_graphs(ctx);
  return BLGPU_OK;
}

int blgpu_get_tiles(const blgpu_ctx *ctx, int *tiles, int n) {
  if (!ctx || !tiles || n < 5) return BLGPU_EINVAL;
  const Tiles &t = ctx->tiles;
  tiles[0] = t.rhs_kc;
  tiles[1] = t.rhs_by;
  tiles[2] = t.dct_nw;
  tiles[3] = t.dftz_rk;
  tiles[4] = t.proj_by;
  if (n >= 6) tiles[5] = t.zdft;
  if (n >= 7) tiles[6] = t.rhs_pts;
  if (n >= 8) tiles[7] = t.thomas;
  if (n >= 9) tiles[8] = t.idct_nw;
  if (n >= 10) tiles[9] = t.xfft;
  return BLGPU_OK;
}

int blgpu_autotune(blgpu_ctx *ctx, int steps, double *ms_default, double *ms_best) {
  if (!ctx || steps < 1) return set_err(ctx, BLGPU_EINVAL, "blgpu_autotune: bad argument");
  if (!ctx->have_grid || !ctx->have_bc || !ctx->have_state)
    return set_err(ctx, BLGPU_ESTATE, "blgpu_autotune: grid, boundary and state must be set first");
  CK(cudaSetDevice(ctx->cfg.device));
  Snapshot sn;
  int rc = snap_take(ctx, sn);
  if (rc) { snap_free(sn); return rc; }
  const bool window = ctx->cfg.les_model == 0;  // DNS: register-window and TMA-fed RHS kernels
  std::vector<std::vector<int>> cand = {
      window ? std::vector<int>{8, 16, 32, 64} : std::vector<int>{4, 8, 16},  // rhs_kc
      {4, 8},                                                                  // rhs_by
      {0, 2, 4, 6, 8, 12, 16},                                                 // dct_nw
      {4, 8},                                                                  // dftz_rk
      {4, 8},                                                                  // proj_by
      {1, 2, 3},                                                               // zdft
      {1, 2, 4},                                                               // rhs_pts
      {1, 2, 3},                                                               // thomas
      {0, 4, 8, 12, 16},                                                       // idct_nw
      {1, 2}};                                                                 // xfft
  auto measure = [&](const Tiles &t, double *ms) -> int {
    int r = snap_restore(ctx, sn);
    if (r) return r;
    ctx->tiles = t;
    drop_graphs(ctx);
    double a = 0, b = 0;
    if ((r = time_steps(ctx, steps, &a))) return r;
    if ((r = time_steps(ctx, steps, &b))) return r;
    *ms = a < b ? a : b;
    return BLGPU_OK;
  };
  const Tiles t0 = ctx->tiles;
  Tiles best = t0;
  double best_ms = 0;
  rc = measure(best, &best_ms);
  const double def_ms = best_ms;
  for (int knob = 0; knob < 10 && !rc; ++knob) {  // one pass of coordinate descent
    if (knob == 5 && !ctx->zfrag && !ctx->utab) continue;  // no tensor-core z transform for this box
    if (knob == 6 && !window) continue;            // one RHS form outside the FP32 DNS path
    if (knob == 7 && !ctx->have_tmaps) continue;   // one y-solve without tensor maps
    if (knob == 9 && (ctx->fp64 ? xfft_split(ctx->spec.N) != 29 : !xfft_split(ctx->spec.N))) continue;  // one x-transform kernel
    for (int v : cand[knob]) {
      Tiles t = best;
      int *f[10] = {&t.rhs_kc, &t.rhs_by, &t.dct_nw, &t.dftz_rk, &t.proj_by, &t.zdft, &t.rhs_pts, &t.thomas,
                    &t.idct_nw, &t.xfft};
      if (*f[knob] == v) continue;
      *f[knob] = v;
      if (tiles_check(ctx, t)) continue;
      double ms = 0;
      rc = measure(t, &ms);
      if (rc) break;
      if (ms < best_ms) { best_ms = ms; best = t; }
    }
  }
  int rc2 = snap_restore(ctx, sn);
  snap_free(sn);
  ctx->tiles = rc ? t0 : best;
  drop_graphs(ctx);
  if (rc) return rc;
  if (rc2) return rc2;
  if (ms_default) *ms_default = def_ms;
  if (ms_best) *ms_best = best_ms;
  return BLGPU_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// ensemble: independent boxes advanced by one CUDA-graph launch per step.
// The graph forks one branch per box from the ensemble stream (each branch is
// that box's whole step on its own stream, so branches run concurrently) and
// joins them back.  Graphs are kept per rotation of the three state buffers
// and re-captured when a box's own graphs were dropped.
// ---------------------------------------------------------------------------
struct blgpu_ensemble {
  std::vector<blgpu_ctx *> box;
  int device = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};
  std::vector<long long> gens[3];
  std::vector<int> next[3];
  long long graph_launches[3] = {0, 0, 0};
  long long launches = 0;
  std::string err;
};

static int ens_err(blgpu_ensemble *e, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (e) e->err = buf;
  g_last_error = buf;
  return code;
}

#define ECK(expr)                                                                                             \
  do {                                                                                                        \
    cudaError_t _e = (expr);                                                                                  \
    if (_e != cudaSuccess)                                                                                    \
      return ens_err(e, BLGPU_ECUDA, "CUDA error %s (%s) in %s", cudaGetErrorName(_e), cudaGetErrorString(_e), \
                     #expr);                                                                                  \
  } while (0)

static void ens_drop(blgpu_ensemble *e) {
  for (int r = 0; r < 3; ++r)
    if (e->graph[r]) {
      cudaGraphExecDestroy(e->graph[r]);
      e->graph[r] = nullptr;
    }
}

static int ens_capture(blgpu_ensemble *e, int a) {
  cudaGraph_t gr = nullptr;
  ECK(cudaStreamBeginCapture(e->st, cudaStreamCaptureModeRelaxed));
  cudaEventRecord(e->fork, e->st);
  long long nl = 0;
  e->next[a].assign(e->box.size(), 0);
  e->gens[a].assign(e->box.size(), 0);
  for (size_t b = 0; b < e->box.size(); ++b) {
    blgpu_ctx *ctx = e->box[b];
    cudaStreamWaitEvent(ctx->st, e->fork, 0);
    const long long l0 = ctx->launches;
    e->next[a][b] = ctx->fp64 ? enq_step<double>(ctx, a, true) : enq_step<float>(ctx, a, true);
    nl += ctx->launches - l0;
    ctx->launches = l0;
    cudaEventRecord(e->join[b], ctx->st);
    cudaStreamWaitEvent(e->st, e->join[b], 0);
    e->gens[a][b] = ctx->gen;
  }
  cudaError_t ce = cudaStreamEndCapture(e->st, &gr);
  if (ce != cudaSuccess) return ens_err(e, BLGPU_ECUDA, "ensemble capture failed: %s", cudaGetErrorString(ce));
  ce = cudaGraphInstantiate(&e->graph[a], gr, 0);
  cudaGraphDestroy(gr);
  if (ce != cudaSuccess) return ens_err(e, BLGPU_ECUDA, "ensemble graph instantiate: %s", cudaGetErrorString(ce));
  e->graph_launches[a] = nl;
  return BLGPU_OK;
}

extern "C" {

int blgpu_ensemble_create(blgpu_ctx *const *boxes, int nbox, blgpu_ensemble **out) {
  if (!boxes || nbox < 1 || !out) return set_err(nullptr, BLGPU_EINVAL, "blgpu_ensemble_create: bad argument");
  *out = nullptr;
  for (int b = 0; b < nbox; ++b) {
    if (!boxes[b]) return set_err(nullptr, BLGPU_EINVAL, "blgpu_ensemble_create: box %d is null", b);
    if (boxes[b]->cfg.device != boxes[0]->cfg.device)
      return set_err(nullptr, BLGPU_EINVAL, "blgpu_ensemble_create: boxes on different devices");
    for (int c = 0; c < b; ++c)
      if (boxes[c] == boxes[b]) return set_err(nullptr, BLGPU_EINVAL, "blgpu_ensemble_create: box %d repeated", b);
  }
  blgpu_ensemble *e = new blgpu_ensemble();
  e->box.assign(boxes, boxes + nbox);
  e->device = boxes[0]->cfg.device;
  e->join.assign(nbox, nullptr);
  cudaError_t ce = cudaSetDevice(e->device);
  if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking);
  if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming);
  for (int b = 0; b < nbox && ce == cudaSuccess; ++b) ce = cudaEventCreateWithFlags(&e->join[b], cudaEventDisableTiming);
  if (ce != cudaSuccess) {
    int rc = set_err(nullptr, BLGPU_ECUDA, "blgpu_ensemble_create: %s", cudaGetErrorString(ce));
    blgpu_ensemble_destroy(e);
    return rc;
  }
  *out = e;
  return BLGPU_OK;
}

int blgpu_ensemble_destroy(blgpu_ensemble *e) {
  if (!e) return BLGPU_OK;
  cudaSetDevice(e->device);
  if (e->st) cudaStreamSynchronize(e->st);
  ens_drop(e);
  for (cudaEvent_t ev : e->join)
    if (ev) cudaEventDestroy(ev);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->st) cudaStreamDestroy(e->st);
  delete e;
  return BLGPU_OK;
}

const char *blgpu_ensemble_last_error(const blgpu_ensemble *e) {
  if (e && !e->err.empty()) return e->err.c_str();
  return g_last_error.c_str();
}

int blgpu_ensemble_advance(blgpu_ensemble *e, int nsteps) {
  if (!e || nsteps < 0) return ens_err(e, BLGPU_EINVAL, "blgpu_ensemble_advance: bad argument");
  ECK(cudaSetDevice(e->device));
  for (blgpu_ctx *c : e->box) {
    if (!c->have_grid || !c->have_bc || !c->have_state)
      return ens_err(e, BLGPU_ESTATE, "blgpu_ensemble_advance: every box needs grid, boundary and state");
    ECK(cudaStreamSynchronize(c->st));  // earlier work of a box on its own stream comes first
  }
  for (int n = 0; n < (nsteps > 0 ? nsteps : 1); ++n) {
    const int a = e->box[0]->cur;
    for (blgpu_ctx *c : e->box)
      if (c->cur != a)
        return ens_err(e, BLGPU_ESTATE, "blgpu_ensemble_advance: boxes are at different buffer rotations");
    bool stale = !e->graph[a];
    for (size_t b = 0; b < e->box.size() && !stale; ++b) stale = e->gens[a][b] != e->box[b]->gen;
    if (stale) {
      if (e->graph[a]) {
        cudaGraphExecDestroy(e->graph[a]);
        e->graph[a] = nullptr;
      }
      int rc = ens_capture(e, a);
      if (rc) return rc;
    }
    if (nsteps == 0) break;
    ECK(cudaGraphLaunch(e->graph[a], e->st));
    e->launches += e->graph_launches[a];
    for (size_t b = 0; b < e->box.size(); ++b) {
      e->box[b]->old = a;
      e->box[b]->cur = e->next[a][b];
    }
  }
  ECK(cudaGetLastError());
  return BLGPU_OK;
}

// Baseline: the same steps with the boxes one after another (each box's own
// step graph launched on the ensemble stream, so no two boxes overlap).
int blgpu_ensemble_advance_sequential(blgpu_ensemble *e, int nsteps) {
  if (!e || nsteps < 0) return ens_err(e, BLGPU_EINVAL, "blgpu_ensemble_advance_sequential: bad argument");
  ECK(cudaSetDevice(e->device));
  for (blgpu_ctx *c : e->box) {
    if (!c->have_grid || !c->have_bc || !c->have_state)
      return ens_err(e, BLGPU_ESTATE, "blgpu_ensemble_advance_sequential: every box needs grid, boundary and state");
    ECK(cudaStreamSynchronize(c->st));
    for (int r = 0; r < 3; ++r)  // capture each rotation's graph up front, outside any timed region
      if (!c->graph[r]) {
        const int keep_cur = c->cur, keep_old = c->old;
        c->cur = r;
        int rc = blgpu_advance(c, 0);
        c->cur = keep_cur;
        c->old = keep_old;
        if (rc) return ens_err(e, rc, "%s", c->err.c_str());
      }
  }
  for (int n = 0; n < nsteps; ++n)
    for (blgpu_ctx *c : e->box) {
      const int a = c->cur;
      ECK(cudaGraphLaunch(c->graph[a], e->st));
      c->launches += c->graph_launches[a];
      e->launches += c->graph_launches[a];
      c->old = a;
      c->cur = c->graph_next[a];
    }
  ECK(cudaGetLastError());
  return BLGPU_OK;
}

int blgpu_ensemble_time(blgpu_ensemble *e, int nsteps, int sequential, double *ms) {
  if (!e || !ms || nsteps < 1) return ens_err(e, BLGPU_EINVAL, "blgpu_ensemble_time: bad argument");
  ECK(cudaSetDevice(e->device));
  int rc = sequential ? blgpu_ensemble_advance_sequential(e, 0) : blgpu_ensemble_advance(e, 0);
  if (rc) return rc;
  cudaEvent_t a, b;
  ECK(cudaEventCreate(&a));
  ECK(cudaEventCreate(&b));
  cudaEventRecord(a, e->st);
  rc = sequential ? blgpu_ensemble_advance_sequential(e, nsteps) : blgpu_ensemble_advance(e, nsteps);
  cudaEventRecord(b, e->st);
  cudaError_t ce = cudaEventSynchronize(b);
  float t = 0.f;
  if (!rc && ce == cudaSuccess) ce = cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc) return rc;
  ECK(ce);
  *ms = (double)t;
  return BLGPU_OK;
}

int blgpu_ensemble_sync(blgpu_ensemble *e) {
  if (!e) return BLGPU_EINVAL;
  ECK(cudaSetDevice(e->device));
  ECK(cudaStreamSynchronize(e->st));
  return BLGPU_OK;
}

long long blgpu_ensemble_launches(const blgpu_ensemble *e) { return e ? e->launches : 0; }

// Autotune each distinct box shape once (the first box of that shape) and
// give its launch shapes to every box of the same shape and precision.
int blgpu_ensemble_autotune(blgpu_ensemble *e, int steps, int *ntuned) {
  if (!e || steps < 1) return ens_err(e, BLGPU_EINVAL, "blgpu_ensemble_autotune: bad argument");
  ECK(cudaSetDevice(e->device));
  ECK(cudaStreamSynchronize(e->st));
  int n = 0;
  for (size_t b = 0; b < e->box.size(); ++b) {
    blgpu_ctx *c = e->box[b];
    blgpu_ctx *twin = nullptr;
    for (size_t q = 0; q < b && !twin; ++q) {
      blgpu_ctx *d = e->box[q];
      if (d->nx == c->nx && d->ny == c->ny && d->nz == c->nz && d->fp64 == c->fp64 &&
          d->cfg.les_model == c->cfg.les_model)
        twin = d;
    }
    if (twin) {
      c->tiles = twin->tiles;
      drop_graphs(c);
      continue;
    }
    int rc = blgpu_autotune(c, steps, nullptr, nullptr);
    if (rc) return ens_err(e, rc, "%s", c->err.c_str());
    ++n;
  }
  ens_drop(e);
  // ensemble pass: the knobs whose kernels hold whole SMs while they run (the
  // persistent tensor-core z transforms, the TMA-fed RHS with its shared-
  // memory ring, the tiled y-solve) are timed per shape with every box of the
  // ensemble stepping, since a choice that is fastest for a box alone can
  // keep the other boxes' kernels off the SMs; the shortest ensemble step wins
  std::vector<Snapshot> sn(e->box.size());
  int rc = BLGPU_OK;
  for (size_t b = 0; b < e->box.size() && !rc; ++b) rc = snap_take(e->box[b], sn[b]);
  auto measure = [&](double *ms) -> int {
    for (size_t b = 0; b < e->box.size(); ++b) {
      int r = snap_restore(e->box[b], sn[b]);
      if (r) return r;
      drop_graphs(e->box[b]);
    }
    ens_drop(e);
    double t = 0;
    int r = blgpu_ensemble_time(e, 1, 0, &t);  // capture and one untimed step
    if (!r) r = blgpu_ensemble_time(e, steps, 0, &t);
    *ms = t / steps;
    return r;
  };
  double best_ms = 0;
  if (!rc) rc = measure(&best_ms);
  for (size_t b = 0; b < e->box.size() && !rc; ++b) {
    blgpu_ctx *c = e->box[b];
    bool first = true;  // tune each shape once, at its first box
    for (size_t q = 0; q < b; ++q) {
      blgpu_ctx *d = e->box[q];
      if (d->nx == c->nx && d->ny == c->ny && d->nz == c->nz && d->fp64 == c->fp64 &&
          d->cfg.les_model == c->cfg.les_model)
        first = false;
    }
    if (!first) continue;
    const std::vector<std::pair<int, std::vector<int>>> knobs = {{5, {1, 2, 3}}, {6, {2, 4}}, {7, {1, 2}}};
    for (const auto &kv : knobs) {
      for (int v : kv.second) {
        Tiles t = c->tiles;
        int *f[10] = {&t.rhs_kc, &t.rhs_by, &t.dct_nw, &t.dftz_rk, &t.proj_by, &t.zdft, &t.rhs_pts, &t.thomas,
                      &t.idct_nw, &t.xfft};
        if (*f[kv.first] == v) continue;
        if (kv.first == 5 && !c->zfrag && !c->utab) continue;
        if (kv.first == 5 && ((v == 3 && !c->utab) || (v == 2 && !c->zfrag))) continue;
        if (kv.first == 6 && (c->fp64 || c->cfg.les_model)) continue;
        if (kv.first == 7 && !c->have_tmaps) continue;
        *f[kv.first] = v;
        if (tiles_check(c, t)) continue;
        std::vector<Tiles> keep;
        for (blgpu_ctx *d : e->box) keep.push_back(d->tiles);
        for (blgpu_ctx *d : e->box)
          if (d->nx == c->nx && d->ny == c->ny && d->nz == c->nz && d->fp64 == c->fp64 &&
              d->cfg.les_model == c->cfg.les_model)
            d->tiles = t;
        double ms = 0;
        rc = measure(&ms);
        if (rc) break;
        if (ms < best_ms) {
          best_ms = ms;
        } else {
          for (size_t q = 0; q < e->box.size(); ++q) e->box[q]->tiles = keep[q];
        }
      }
      if (rc) break;
    }
  }
  for (size_t b = 0; b < e->box.size(); ++b) {
    if (!rc) rc = snap_restore(e->box[b], sn[b]);
    snap_free(sn[b]);
    drop_graphs(e->box[b]);
  }
  ens_drop(e);
  if (rc) return ens_err(e, rc, "ensemble autotune: %s", e->box[0]->err.c_str());
  if (ntuned) *ntuned = n;
  return BLGPU_OK;
}

}  // extern "C"
