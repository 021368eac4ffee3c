/*
 * mlp_oracle.c -- CPU restatement of the wall-stress network of the B200
 * path (4 -> 64 -> 64 -> 64 -> 2, GELU): forward pass, loss and gradient.
 *
 * TEST INFRASTRUCTURE ONLY (the checker of the tensor-core kernels; the
 * product never loads it).
 *
 * With exact = 0 it rounds to BF16 (round to nearest even) at the points
 * where the tensor-core kernels feed the MMA -- weights, layer inputs,
 * back-propagated errors -- and sums exact products, so it reproduces the
 * device arithmetic up to the order of the FP32 sums.  With exact = 1 it
 * is the plain FP64 network, the reference for finite differences.
 *
 * Parameters: W0[64][4] b0[64] W1[64][64] b1[64] W2[64][64] b2[64]
 * W3[2][64] b3[2] (8770 values).  Loss = (1/B) sum_rows sum_o (y_o - t_o)^2.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "bl_oracle.h"

#define NIN 4
#define NH 64
#define NOUT 2
#define OW0 0
#define OB0 (OW0 + NH * NIN)
#define OW1 (OB0 + NH)
#define OB1 (OW1 + NH * NH)
#define OW2 (OB1 + NH)
#define OB2 (OW2 + NH * NH)
#define OW3 (OB2 + NH)
#define OB3 (OW3 + NOUT * NH)
#define NP (OB3 + NOUT)

int blo_mlp_nparams(void) { return NP; }

static float bf16r(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return x;
  u += 0x7fffu + ((u >> 16) & 1u);
  u &= 0xffff0000u;
  memcpy(&x, &u, 4);
  return x;
}
static double rq(double v, int exact) { return exact ? v : (double)bf16r((float)v); }
static double gelu(double z) { return 0.5 * z * (1.0 + erf(z / sqrt(2.0))); }
static double gelu_d(double z) { return 0.5 * (1.0 + erf(z / sqrt(2.0))) + z * exp(-0.5 * z * z) / sqrt(2.0 * M_PI); }

typedef struct {
  double a0[NIN], a1[NH], a2[NH], a3[NH]; /* layer inputs (rounded) */
  double gp0[NH], gp1[NH], gp2[NH];
  double y[NOUT];
} acts;

static void forward_row(const double *w, const float *x, int exact, acts *A) {
  double z[NH];
  for (int i = 0; i < NIN; ++i) A->a0[i] = rq(x[i], exact);
  for (int o = 0; o < NH; ++o) {
    double s = w[OB0 + o];
    for (int i = 0; i < NIN; ++i) s += w[OW0 + o * NIN + i] * A->a0[i];
    z[o] = s;
  }
  for (int o = 0; o < NH; ++o) { A->a1[o] = rq(gelu(z[o]), exact); A->gp0[o] = gelu_d(z[o]); }
  for (int o = 0; o < NH; ++o) {
    double s = w[OB1 + o];
    for (int i = 0; i < NH; ++i) s += w[OW1 + o * NH + i] * A->a1[i];
    z[o] = s;
  }
  for (int o = 0; o < NH; ++o) { A->a2[o] = rq(gelu(z[o]), exact); A->gp1[o] = gelu_d(z[o]); }
  for (int o = 0; o < NH; ++o) {
    double s = w[OB2 + o];
    for (int i = 0; i < NH; ++i) s += w[OW2 + o * NH + i] * A->a2[i];
    z[o] = s;
  }
  for (int o = 0; o < NH; ++o) { A->a3[o] = rq(gelu(z[o]), exact); A->gp2[o] = gelu_d(z[o]); }
  for (int o = 0; o < NOUT; ++o) {
    double s = w[OB3 + o];
    for (int i = 0; i < NH; ++i) s += w[OW3 + o * NH + i] * A->a3[i];
    A->y[o] = s;
  }
}

/* working copy: weights rounded to BF16 and biases to FP32 (exact = 0) */
static double *working(const double *params, int exact) {
  double *w = (double *)malloc(sizeof(double) * NP);
  for (int p = 0; p < NP; ++p) w[p] = exact ? params[p] : (double)(float)params[p];
  if (!exact) {
    for (int p = OW0; p < OB0; ++p) w[p] = rq(w[p], 0);
    for (int p = OW1; p < OB1; ++p) w[p] = rq(w[p], 0);
    for (int p = OW2; p < OB2; ++p) w[p] = rq(w[p], 0);
    for (int p = OW3; p < OB3; ++p) w[p] = rq(w[p], 0);
  }
  return w;
}

void blo_mlp_forward(const double *params, const float *X, int rows, float *Y, int exact) {
  double *w = working(params, exact);
  acts A;
  for (int r = 0; r < rows; ++r) {
    forward_row(w, X + (size_t)r * NIN, exact, &A);
    Y[(size_t)r * NOUT] = (float)A.y[0];
    Y[(size_t)r * NOUT + 1] = (float)A.y[1];
  }
  free(w);
}

double blo_mlp_gradient(const double *params, const float *X, const float *T, int rows, double *grad, int exact) {
  double *w = working(params, exact);
  memset(grad, 0, sizeof(double) * NP);
  double loss = 0.0;
  const double scale = exact ? 2.0 / (double)rows : (double)(2.0f / (float)rows);
  acts A;
  double d3[NOUT], e[NH], d2[NH], d1[NH], d0[NH];
  for (int r = 0; r < rows; ++r) {
    forward_row(w, X + (size_t)r * NIN, exact, &A);
    for (int o = 0; o < NOUT; ++o) {
      const double err = A.y[o] - (double)T[(size_t)r * NOUT + o];
      loss += err * err;
      d3[o] = rq(scale * err, exact);
    }
    for (int i = 0; i < NH; ++i) {
      double s = 0.0;
      for (int o = 0; o < NOUT; ++o) s += w[OW3 + o * NH + i] * d3[o];
      e[i] = s;
    }
    for (int i = 0; i < NH; ++i) d2[i] = rq(e[i] * A.gp2[i], exact);
    for (int i = 0; i < NH; ++i) {
      double s = 0.0;
      for (int o = 0; o < NH; ++o) s += w[OW2 + o * NH + i] * d2[o];
      e[i] = s;
    }
    for (int i = 0; i < NH; ++i) d1[i] = rq(e[i] * A.gp1[i], exact);
    for (int i = 0; i < NH; ++i) {
      double s = 0.0;
      for (int o = 0; o < NH; ++o) s += w[OW1 + o * NH + i] * d1[o];
      e[i] = s;
    }
    for (int i = 0; i < NH; ++i) d0[i] = rq(e[i] * A.gp0[i], exact);
    for (int o = 0; o < NOUT; ++o) {
      grad[OB3 + o] += d3[o];
      for (int i = 0; i < NH; ++i) grad[OW3 + o * NH + i] += d3[o] * A.a3[i];
    }
    for (int o = 0; o < NH; ++o) {
      grad[OB2 + o] += d2[o];
      grad[OB1 + o] += d1[o];
      grad[OB0 + o] += d0[o];
      for (int i = 0; i < NH; ++i) {
        grad[OW2 + o * NH + i] += d2[o] * A.a2[i];
        grad[OW1 + o * NH + i] += d1[o] * A.a1[i];
      }
      for (int i = 0; i < NIN; ++i) grad[OW0 + o * NIN + i] += d0[o] * A.a0[i];
    }
  }
  free(w);
  return loss / (double)rows;
}
