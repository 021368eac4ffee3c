// mlp.cuh -- layout of the wall-stress network shared by the MLP kernels and
// the solver's wall-model hook.
//
// Network 4 -> 64 -> 64 -> 64 -> 2, GELU after each hidden layer.  Master
// parameters are FP32, in this order (W[out][in] row-major):
//   W0[64][4] b0[64] W1[64][64] b1[64] W2[64][64] b2[64] W3[2][64] b3[2]
// The tensor-core kernels read a packed BF16 copy: the matrices padded to the
// MMA shapes with rows of K+8 elements (bank-conflict-free fragment loads),
// forward copies W[n][k] and, for the backward pass, transposes WT[k][n].
#pragma once
#include <stdint.h>

#include "common.cuh"

namespace blgpu {
namespace mlp {

constexpr int NIN = 4, NH = 64, NOUT = 2;
constexpr int NP = NH * NIN + NH + 2 * (NH * NH + NH) + NOUT * NH + NOUT;  // 8770
// master offsets
constexpr int OW0 = 0, OB0 = OW0 + NH * NIN, OW1 = OB0 + NH, OB1 = OW1 + NH * NH, OW2 = OB1 + NH,
              OB2 = OW2 + NH * NH, OW3 = OB2 + NH, OB3 = OW3 + NOUT * NH;
static_assert(OB3 + NOUT == NP, "parameter layout");

// packed BF16 strides and offsets (in bf16 elements)
constexpr int S16 = 16 + 8;  // rows of K = 16 (padded input / output dims)
constexpr int S64 = 64 + 8;  // rows of K = 64
constexpr int PW0 = 0;                 // W0p  [64][S16]  (in 4 -> 16)
constexpr int PW1 = PW0 + 64 * S16;    // W1p  [64][S64]
constexpr int PW2 = PW1 + 64 * S64;    // W2p  [64][S64]
constexpr int PW3 = PW2 + 64 * S64;    // W3p  [8][S64]   (out 2 -> 8)
constexpr int PT1 = PW3 + 8 * S64;     // W1T  [64][S64]
constexpr int PT2 = PT1 + 64 * S64;    // W2T  [64][S64]
constexpr int PT3 = PT2 + 64 * S64;    // W3T  [64][S16]  (out 2 -> 16)
constexpr int PACKN = PT3 + 64 * S16;  // 22080 bf16
constexpr int FWDN = PT1;              // the forward part of the pack
// FP32 biases: b0[64] b1[64] b2[64] b3[8]
constexpr int BIASN = 3 * 64 + 8;

}  // namespace mlp

// device view of a network for the wall-model hook
struct MlpDev {
  const uint16_t *pack;  // PACKN bf16
  const float *bias;     // BIASN
};

// launchers (mlp.cu)
size_t mlp_train_smem();
size_t mlp_fwd_smem();
int mlp_train_ctas(int B);
void launch_mlp_pack(const float *params, uint16_t *pack, float *bias, cudaStream_t st);
void launch_mlp_forward(const uint16_t *pack, const float *bias, const float *X, float *Y, int rows, cudaStream_t st);
void launch_mlp_grad(const uint16_t *pack, const float *bias, const float *X, const float *Tg, const int *perm,
                     int nsamp, const int *offp, int B, float *part, cudaStream_t st);
void launch_mlp_reduce(const float *part, int nparts, float *grad, float *loss, cudaStream_t st);
void launch_mlp_adam(const float *part, int nparts, float *params, float *m1, float *m2, float *stv, float lr, int B,
                     int nsamp, float *loss_hist, int hist_n, uint16_t *pack, float *bias, cudaStream_t st);
template <typename T>
void launch_wall_samples(const Geo &g, const T *U, const T *W, const T *P, int jh, float *X, float *Tg,
                         cudaStream_t st);
// wm = [alpha_x, alpha_z, tau_x, tau_z] at the (nx-2)(nzg-3) wall points;
// alpha = tau / nu_wall, nu_wall the viscosity of the U-equation's wall flux
// (nu, plus the interpolated eddy viscosity when nut is given)
template <typename T>
void launch_wall_mlp(const Geo &g, const MlpDev &net, const T *U, const T *W, const T *P, const T *nut, int jh,
                     double *wm, cudaStream_t st);
template <typename T>
void launch_wall_eq(const Geo &g, const double *utau, const T *nut, double *wm, cudaStream_t st);

}  // namespace blgpu

// host handle of a network (capi_mlp.cu); the solver's wall-model hook reads
// its device view
struct blgpu_mlp;
blgpu::MlpDev blgpu_mlp_view(const blgpu_mlp *m);
int blgpu_mlp_device(const blgpu_mlp *m);
int blgpu_mlp_reserve(blgpu_mlp *m, int rows, float **X, float **T);
void blgpu_mlp_commit(blgpu_mlp *m, int rows);
cudaStream_t blgpu_mlp_stream(const blgpu_mlp *m);
