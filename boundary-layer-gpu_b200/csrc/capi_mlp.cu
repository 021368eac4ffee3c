// capi_mlp.cu -- C ABI of the learned wall-stress network (include/blgpu.h,
// "learned wall model"): parameters, host-array forward and gradient (the
// gradient check), the device training set and Adam training replayed from
// a CUDA graph.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/blgpu.h"
#include "kernels.cuh"
#include "mlp.cuh"

using namespace blgpu;
using namespace blgpu::mlp;

namespace blgpu {
void set_global_error(const char *msg);
}

struct blgpu_mlp {
  int device = 0;
  cudaStream_t st = nullptr;
  float *params = nullptr, *m1 = nullptr, *m2 = nullptr, *stv = nullptr, *grad = nullptr, *loss = nullptr;
  float *part = nullptr, *hist = nullptr;
  int hist_n = 1 << 16;
  uint16_t *pack = nullptr;
  float *bias = nullptr;
  // training set
  float *X = nullptr, *T = nullptr;
  int *perm = nullptr;
  int n = 0, cap = 0;
  unsigned long long seed = 0;
  bool perm_dirty = true;
  // host-array scratch
  float *Xq = nullptr, *Yq = nullptr;
  int *idq = nullptr;
  int qcap = 0;
  // training graph
  cudaGraphExec_t graph = nullptr;
  int graph_B = 0;
  float graph_lr = 0.f;
  std::string err;
};

static int merr(blgpu_mlp *m, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (m) m->err = buf;
  set_global_error(buf);
  return code;
}

#define MCK(expr)                                                                                             \
  do {                                                                                                        \
    cudaError_t _e = (expr);                                                                                  \
    if (_e != cudaSuccess)                                                                                    \
      return merr(m, BLGPU_ECUDA, "CUDA error %s (%s) in %s", cudaGetErrorName(_e), cudaGetErrorString(_e), \
                  #expr);                                                                                     \
  } while (0)

static unsigned long long splitmix(unsigned long long &s) {
  unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static double unif(unsigned long long &s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

static void drop_graph(blgpu_mlp *m) {
  if (m->graph) {
    cudaGraphExecDestroy(m->graph);
    m->graph = nullptr;
  }
}

// device scratch for host-array calls; idq holds 0..rows-1 (identity order)
static int scratch(blgpu_mlp *m, int rows) {
  if (rows <= m->qcap) return BLGPU_OK;
  if (m->Xq) cudaFree(m->Xq);
  if (m->Yq) cudaFree(m->Yq);
  if (m->idq) cudaFree(m->idq);
  m->Xq = m->Yq = nullptr;
  m->idq = nullptr;
  m->qcap = 0;
  MCK(cudaMalloc(&m->Xq, (size_t)rows * 4 * sizeof(float)));
  MCK(cudaMalloc(&m->Yq, (size_t)rows * 2 * sizeof(float)));
  MCK(cudaMalloc(&m->idq, (size_t)rows * sizeof(int)));
  std::vector<int> id(rows);
  for (int r = 0; r < rows; ++r) id[r] = r;
  MCK(cudaMemcpy(m->idq, id.data(), rows * sizeof(int), cudaMemcpyHostToDevice));
  m->qcap = rows;
  return BLGPU_OK;
}

// a fresh shuffled order of the training set (Fisher-Yates) and offset 0
static int reshuffle(blgpu_mlp *m) {
  if (!m->perm_dirty || m->n == 0) return BLGPU_OK;
  std::vector<int> p(m->n);
  for (int r = 0; r < m->n; ++r) p[r] = r;
  unsigned long long s = m->seed ^ 0xA5A5A5A5ull;
  for (int r = m->n - 1; r > 0; --r) {
    const int q = (int)(splitmix(s) % (unsigned long long)(r + 1));
    std::swap(p[r], p[q]);
  }
  MCK(cudaMemcpy(m->perm, p.data(), m->n * sizeof(int), cudaMemcpyHostToDevice));
  const int zero = 0;
  MCK(cudaMemcpy(m->stv + 1, &zero, sizeof(int), cudaMemcpyHostToDevice));
  m->perm_dirty = false;
  return BLGPU_OK;
}

// grow the training set to hold `rows` more samples; returns the new rows
int blgpu_mlp_reserve(blgpu_mlp *m, int rows, float **X, float **T) {
  if (rows < 0) return merr(m, BLGPU_EINVAL, "negative row count");
  const long long need = (long long)m->n + rows;
  if (need > (1ll << 30)) return merr(m, BLGPU_EINVAL, "training set too large");
  if (need > m->cap) {
    long long cap = m->cap ? m->cap : 1024;
    while (cap < need) cap *= 2;
    float *nX = nullptr, *nT = nullptr;
    int *np = nullptr;
    MCK(cudaMalloc(&nX, (size_t)cap * 4 * sizeof(float)));
    MCK(cudaMalloc(&nT, (size_t)cap * 2 * sizeof(float)));
    MCK(cudaMalloc(&np, (size_t)cap * sizeof(int)));
    if (m->n) {
      MCK(cudaMemcpy(nX, m->X, (size_t)m->n * 4 * sizeof(float), cudaMemcpyDeviceToDevice));
      MCK(cudaMemcpy(nT, m->T, (size_t)m->n * 2 * sizeof(float), cudaMemcpyDeviceToDevice));
    }
    if (m->X) cudaFree(m->X);
    if (m->T) cudaFree(m->T);
    if (m->perm) cudaFree(m->perm);
    m->X = nX;
    m->T = nT;
    m->perm = np;
    m->cap = (int)cap;
    drop_graph(m);
  }
  *X = m->X + (size_t)m->n * 4;
  *T = m->T + (size_t)m->n * 2;
  return BLGPU_OK;
}

void blgpu_mlp_commit(blgpu_mlp *m, int rows) {
  m->n += rows;
  m->perm_dirty = true;
  drop_graph(m);
}

cudaStream_t blgpu_mlp_stream(const blgpu_mlp *m) { return m->st; }
blgpu::MlpDev blgpu_mlp_view(const blgpu_mlp *m) { return MlpDev{m->pack, m->bias}; }
int blgpu_mlp_device(const blgpu_mlp *m) { return m->device; }

extern "C" {

int blgpu_mlp_nparams(void) { return NP; }

int blgpu_mlp_create(int device, unsigned long long seed, blgpu_mlp **out) {
  if (!out) return merr(nullptr, BLGPU_EINVAL, "blgpu_mlp_create: null argument");
  *out = nullptr;
  blgpu_mlp *m = new blgpu_mlp();
  m->device = device;
  m->seed = seed;
  const int nparts = 148;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&m->params, NP * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->m1, NP * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->m2, NP * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->grad, NP * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->stv, 4 * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->loss, sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->part, (size_t)nparts * (NP + 1) * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->hist, (size_t)m->hist_n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->pack, PACKN * sizeof(uint16_t));
  if (e == cudaSuccess) e = cudaMalloc(&m->bias, BIASN * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(m->hist, 0, (size_t)m->hist_n * sizeof(float));
  if (e != cudaSuccess) {
    int rc = merr(nullptr, BLGPU_ECUDA, "blgpu_mlp_create: %s", cudaGetErrorString(e));
    blgpu_mlp_destroy(m);
    return rc;
  }
  // Glorot-uniform weights, zero biases
  std::vector<float> p(NP, 0.f);
  unsigned long long s = seed;
  auto fill = [&](int off, int nout, int nin) {
    const double a = std::sqrt(6.0 / (double)(nin + nout));
    for (int q = 0; q < nout * nin; ++q) p[off + q] = (float)((2.0 * unif(s) - 1.0) * a);
  };
  fill(OW0, NH, NIN);
  fill(OW1, NH, NH);
  fill(OW2, NH, NH);
  fill(OW3, NOUT, NH);
  int rc = blgpu_mlp_set_params(m, p.data(), NP);
  if (rc) {
    blgpu_mlp_destroy(m);
    return rc;
  }
  *out = m;
  return BLGPU_OK;
}

int blgpu_mlp_destroy(blgpu_mlp *m) {
  if (!m) return BLGPU_OK;
  cudaSetDevice(m->device);
  if (m->st) cudaStreamSynchronize(m->st);
  drop_graph(m);
  void *ptrs[] = {m->params, m->m1, m->m2, m->grad, m->stv, m->loss, m->part, m->hist, m->pack, m->bias,
                  m->X, m->T, m->perm, m->Xq, m->Yq, m->idq};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  if (m->st) cudaStreamDestroy(m->st);
  delete m;
  return BLGPU_OK;
}

const char *blgpu_mlp_last_error(const blgpu_mlp *m) { return m && !m->err.empty() ? m->err.c_str() : ""; }

int blgpu_mlp_set_params(blgpu_mlp *m, const float *p, int n) {
  if (!m || !p || n != NP) return merr(m, BLGPU_EINVAL, "blgpu_mlp_set_params: need %d values", NP);
  MCK(cudaSetDevice(m->device));
  MCK(cudaStreamSynchronize(m->st));
  MCK(cudaMemcpy(m->params, p, NP * sizeof(float), cudaMemcpyHostToDevice));
  MCK(cudaMemset(m->m1, 0, NP * sizeof(float)));
  MCK(cudaMemset(m->m2, 0, NP * sizeof(float)));
  MCK(cudaMemset(m->stv, 0, 4 * sizeof(float)));
  launch_mlp_pack(m->params, m->pack, m->bias, m->st);
  MCK(cudaGetLastError());
  MCK(cudaStreamSynchronize(m->st));
  m->perm_dirty = true;
  return BLGPU_OK;
}

int blgpu_mlp_get_params(blgpu_mlp *m, float *p, int n) {
  if (!m || !p || n != NP) return merr(m, BLGPU_EINVAL, "blgpu_mlp_get_params: need %d values", NP);
  MCK(cudaSetDevice(m->device));
  MCK(cudaStreamSynchronize(m->st));
  MCK(cudaMemcpy(p, m->params, NP * sizeof(float), cudaMemcpyDeviceToHost));
  return BLGPU_OK;
}

int blgpu_mlp_forward(blgpu_mlp *m, const float *X, int rows, float *Y) {
  if (!m || !X || !Y || rows < 1) return merr(m, BLGPU_EINVAL, "blgpu_mlp_forward: bad argument");
  MCK(cudaSetDevice(m->device));
  int rc = scratch(m, rows);
  if (rc) return rc;
  MCK(cudaMemcpyAsync(m->Xq, X, (size_t)rows * 4 * sizeof(float), cudaMemcpyHostToDevice, m->st));
  launch_mlp_forward(m->pack, m->bias, m->Xq, m->Yq, rows, m->st);
  MCK(cudaGetLastError());
  MCK(cudaMemcpyAsync(Y, m->Yq, (size_t)rows * 2 * sizeof(float), cudaMemcpyDeviceToHost, m->st));
  MCK(cudaStreamSynchronize(m->st));
  return BLGPU_OK;
}

int blgpu_mlp_gradient(blgpu_mlp *m, const float *X, const float *T, int rows, float *grad, float *loss) {
  if (!m || !X || !T || rows < 1) return merr(m, BLGPU_EINVAL, "blgpu_mlp_gradient: bad argument");
  MCK(cudaSetDevice(m->device));
  int rc = scratch(m, rows);
  if (rc) return rc;
  MCK(cudaMemcpyAsync(m->Xq, X, (size_t)rows * 4 * sizeof(float), cudaMemcpyHostToDevice, m->st));
  MCK(cudaMemcpyAsync(m->Yq, T, (size_t)rows * 2 * sizeof(float), cudaMemcpyHostToDevice, m->st));
  launch_mlp_grad(m->pack, m->bias, m->Xq, m->Yq, m->idq, rows, nullptr, rows, m->part, m->st);
  launch_mlp_reduce(m->part, mlp_train_ctas(rows), m->grad, m->loss, m->st);
  MCK(cudaGetLastError());
  if (grad) MCK(cudaMemcpyAsync(grad, m->grad, NP * sizeof(float), cudaMemcpyDeviceToHost, m->st));
  if (loss) MCK(cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->st));
  MCK(cudaStreamSynchronize(m->st));
  return BLGPU_OK;
}

int blgpu_mlp_add_data(blgpu_mlp *m, const float *X, const float *T, int rows) {
  if (!m || !X || !T || rows < 1) return merr(m, BLGPU_EINVAL, "blgpu_mlp_add_data: bad argument");
  MCK(cudaSetDevice(m->device));
  MCK(cudaStreamSynchronize(m->st));
  float *dX = nullptr, *dT = nullptr;
  int rc = blgpu_mlp_reserve(m, rows, &dX, &dT);
  if (rc) return rc;
  MCK(cudaMemcpy(dX, X, (size_t)rows * 4 * sizeof(float), cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(dT, T, (size_t)rows * 2 * sizeof(float), cudaMemcpyHostToDevice));
  blgpu_mlp_commit(m, rows);
  return BLGPU_OK;
}

int blgpu_mlp_clear_data(blgpu_mlp *m) {
  if (!m) return BLGPU_EINVAL;
  m->n = 0;
  m->perm_dirty = true;
  drop_graph(m);
  return BLGPU_OK;
}

int blgpu_mlp_num_samples(const blgpu_mlp *m) { return m ? m->n : 0; }

int blgpu_mlp_get_data(blgpu_mlp *m, float *X, float *T, int rows) {
  if (!m || rows < 0 || rows > m->n) return merr(m, BLGPU_EINVAL, "blgpu_mlp_get_data: bad row count");
  MCK(cudaSetDevice(m->device));
  MCK(cudaStreamSynchronize(m->st));
  if (X && rows) MCK(cudaMemcpy(X, m->X, (size_t)rows * 4 * sizeof(float), cudaMemcpyDeviceToHost));
  if (T && rows) MCK(cudaMemcpy(T, m->T, (size_t)rows * 2 * sizeof(float), cudaMemcpyDeviceToHost));
  return BLGPU_OK;
}

// `steps` Adam steps of `batch` samples each, replayed from a CUDA graph of
// one step (gradient; fixed-order reduction + update + repack; offset).
int blgpu_mlp_train(blgpu_mlp *m, int steps, int batch, float lr, float *loss_last) {
  if (!m || steps < 0 || batch < 1 || !(lr > 0.f)) return merr(m, BLGPU_EINVAL, "blgpu_mlp_train: bad argument");
  if (m->n < 1) return merr(m, BLGPU_ESTATE, "blgpu_mlp_train: no training samples");
  if (batch > m->n) batch = m->n;
  MCK(cudaSetDevice(m->device));
  int rc = reshuffle(m);
  if (rc) return rc;
  if (m->graph && (m->graph_B != batch || m->graph_lr != lr)) drop_graph(m);
  if (!m->graph) {
    cudaGraph_t gr = nullptr;
    MCK(cudaStreamBeginCapture(m->st, cudaStreamCaptureModeRelaxed));
    launch_mlp_grad(m->pack, m->bias, m->X, m->T, m->perm, m->n, reinterpret_cast<const int *>(m->stv + 1), batch,
                    m->part, m->st);
    launch_mlp_adam(m->part, mlp_train_ctas(batch), m->params, m->m1, m->m2, m->stv, lr, batch, m->n, m->hist,
                    m->hist_n, m->pack, m->bias, m->st);
    cudaError_t e = cudaStreamEndCapture(m->st, &gr);
    if (e != cudaSuccess) return merr(m, BLGPU_ECUDA, "training capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&m->graph, gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) return merr(m, BLGPU_ECUDA, "training graph: %s", cudaGetErrorString(e));
    m->graph_B = batch;
    m->graph_lr = lr;
  }
  for (int s = 0; s < steps; ++s) MCK(cudaGraphLaunch(m->graph, m->st));
  MCK(cudaGetLastError());
  if (loss_last) MCK(cudaMemcpyAsync(loss_last, m->stv + 2, sizeof(float), cudaMemcpyDeviceToHost, m->st));
  MCK(cudaStreamSynchronize(m->st));
  return BLGPU_OK;
}

int blgpu_mlp_steps(blgpu_mlp *m, long long *steps) {
  if (!m || !steps) return BLGPU_EINVAL;
  float v = 0.f;
  MCK(cudaSetDevice(m->device));
  MCK(cudaStreamSynchronize(m->st));
  MCK(cudaMemcpy(&v, m->stv, sizeof(float), cudaMemcpyDeviceToHost));
  *steps = (long long)v;
  return BLGPU_OK;
}

// batch losses of the last n steps (a ring of 65536), oldest first
int blgpu_mlp_loss_history(blgpu_mlp *m, float *hist, int n) {
  if (!m || !hist || n < 1 || n > m->hist_n) return merr(m, BLGPU_EINVAL, "blgpu_mlp_loss_history: bad argument");
  long long st = 0;
  int rc = blgpu_mlp_steps(m, &st);
  if (rc) return rc;
  std::vector<float> h(m->hist_n);
  MCK(cudaMemcpy(h.data(), m->hist, m->hist_n * sizeof(float), cudaMemcpyDeviceToHost));
  for (int q = 0; q < n; ++q) {
    const long long idx = st - n + q;
    hist[q] = idx >= 0 ? h[idx % m->hist_n] : NAN;
  }
  return BLGPU_OK;
}

// loss over the whole training set (no update)
int blgpu_mlp_eval(blgpu_mlp *m, float *loss) {
  if (!m || !loss) return merr(m, BLGPU_EINVAL, "blgpu_mlp_eval: bad argument");
  if (m->n < 1) return merr(m, BLGPU_ESTATE, "blgpu_mlp_eval: no training samples");
  MCK(cudaSetDevice(m->device));
  int rc = scratch(m, m->n);
  if (rc) return rc;
  launch_mlp_grad(m->pack, m->bias, m->X, m->T, m->idq, m->n, nullptr, m->n, m->part, m->st);
  launch_mlp_reduce(m->part, mlp_train_ctas(m->n), nullptr, m->loss, m->st);
  MCK(cudaGetLastError());
  MCK(cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->st));
  MCK(cudaStreamSynchronize(m->st));
  return BLGPU_OK;
}

}  // extern "C"
