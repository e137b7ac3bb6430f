/*
 * mlp_oracle.c -- TEST INFRASTRUCTURE ONLY: CPU restatement of the learned
 * field network of libmbt (mbt.h, mbt_mlp_*): forward pass and gradient
 * with the same roundings of the tensor-core operands (BF16 pairs of the
 * inputs and biases, BF16 weights, activations h' = k gelu(z) in FP32
 * rounded to BF16 in the forward pass; BF16 operands of the backward products),
 * sums in double.  Used by tests/ to check the GPU kernels.
 *
 * GELU in its sigmoid form gelu(z) = z sigma(k z) = z (1 + tanh(c z)) / 2,
 * k = 1.702, c = k/2.  The kernels fold c into each hidden layer's weights
 * and bias (the product is w = c z), compute h' = w (1 + tanh w) = k gelu(z)
 * and fold 1/k into the next layer: W2/2, W3/2 (c/k = 1/2) and W4/k.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define H 128
#define W1 0
#define B1 384
#define W2 512
#define B2 (W2 + 16384)
#define W3 (B2 + 128)
#define B3 (W3 + 16384)
#define W4 (B3 + 128)
#define B4 (W4 + 256)
#define NPARAM (B4 + 2)

/* round to the nearest BF16 (ties to even) */
static float bf16r(float v)
{
  uint32_t u;
  memcpy(&u, &v, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return v;
  u += 0x7fffu + ((u >> 16) & 1u);
  u &= 0xffff0000u;
  memcpy(&v, &u, 4);
  return v;
}

#define GELU_K 1.702f
#define GELU_C 0.851f
#define GELU_INV_K 0.58754406f
#define GELU_INV_C 1.1750881f

/* The activation of the forward pass (act_bf16x2) of a scaled
 * pre-activation x = c z: h' = x + x tanh(x) in FP32 (one fused multiply-add)
 * rounded once to BF16; the GPU's tanh is the hardware approximation, this
 * restatement libm's tanh rounded to FP32.  Returns h' = k gelu(z). */
static float act(float x)
{
  const float th = (float) tanh((double) x);
  return bf16r(fmaf(x, th, x));
}

/* derivative of gelu(x) = x sigma(k x): s + k x s (1 - s) */
static float gelu_grad(float x)
{
  const float s = 0.5f + 0.5f * tanhf(GELU_C * x);
  return s + GELU_K * x * s * (1.0f - s);
}


typedef struct fwd_t {
  float x[3], z1[H], h1[H], z2[H], h2[H], z3[H], h3[H], out[2];
} fwd_t;

/* the BF16 pair (hi, lo) of a bias, summed */
static double bias_pair(float b)
{
  const float hi = bf16r(b);
  return (double) hi + (double) bf16r(b - hi);
}

/* One point: the saved pre-activations are z = w / c, the saved
 * activations gelu(z) = h' / k. */
static void forward_one(const float *P, const float *abr, fwd_t *f)
{
  int i, j, k;
  float xh[3], xl[3], h[H], hn[H];
  f->x[0] = 0.25f * abr[0] - 1.0f;
  f->x[1] = 0.25f * abr[1] - 1.0f;
  f->x[2] = fmaf(0.66761703f, logf(abr[2]), 1.0f);   /* 1 + 2 ln r / ln 20 */
  for (i = 0; i < 3; i++) {
    xh[i] = bf16r(f->x[i]);
    xl[i] = bf16r(f->x[i] - xh[i]);
  }
  for (j = 0; j < H; j++) {
    double s = bias_pair(GELU_C * P[B1 + j]);
    for (i = 0; i < 3; i++) s += (double) bf16r(GELU_C * P[W1 + 3 * j + i]) * ((double) xh[i] + (double) xl[i]);
    h[j] = act((float) s);
    f->z1[j] = GELU_INV_C * (float) s;
    f->h1[j] = GELU_INV_K * h[j];
  }
  for (j = 0; j < H; j++) {
    double s = bias_pair(GELU_C * P[B2 + j]);
    for (k = 0; k < H; k++) s += (double) h[k] * (double) bf16r(0.5f * P[W2 + H * j + k]);
    hn[j] = act((float) s);
    f->z2[j] = GELU_INV_C * (float) s;
    f->h2[j] = GELU_INV_K * hn[j];
  }
  for (j = 0; j < H; j++) {
    double s = bias_pair(GELU_C * P[B3 + j]);
    for (k = 0; k < H; k++) s += (double) hn[k] * (double) bf16r(0.5f * P[W3 + H * j + k]);
    h[j] = act((float) s);
    f->z3[j] = GELU_INV_C * (float) s;
    f->h3[j] = GELU_INV_K * h[j];
  }
  for (j = 0; j < 2; j++) {
    double s = bias_pair(P[B4 + j]);
    for (k = 0; k < H; k++) s += (double) h[k] * (double) bf16r(GELU_INV_K * P[W4 + H * j + k]);
    f->out[j] = (float) s;
  }
}

void orc_mlp_forward(const float *P, long n, const float *abr, float *out)
{
  long i;
  fwd_t f;
  for (i = 0; i < n; i++) {
    forward_one(P, abr + 3 * i, &f);
    out[2 * i] = f.out[0];
    out[2 * i + 1] = f.out[1];
  }
}

/* Gradient of sum((T - target)^2) / n; returns the loss. */
double orc_mlp_gradient(const float *P, int n, const float *abr, const float *tgt, float *grad)
{
  double *g = (double *) calloc(NPARAM, sizeof(double));
  fwd_t *f = (fwd_t *) malloc(sizeof(fwd_t));
  double loss = 0.0;
  int m, j, k;
  for (m = 0; m < n; m++) {
    float dT[2], dz3[H], dz2[H], dz1[H];
    forward_one(P, abr + 3 * m, f);
    for (j = 0; j < 2; j++) {
      const double d = (double) f->out[j] - tgt[2 * m + j];
      loss += d * d;
      dT[j] = 2.0f * (f->out[j] - tgt[2 * m + j]) * (1.0f / (float) n);
    }
    for (j = 0; j < 2; j++) {
      g[B4 + j] += dT[j];
      for (k = 0; k < H; k++) g[W4 + H * j + k] += (double) dT[j] * f->h3[k];
    }
    for (j = 0; j < H; j++) {
      const float dh = P[W4 + j] * dT[0] + P[W4 + H + j] * dT[1];
      dz3[j] = dh * gelu_grad(f->z3[j]);
      g[B3 + j] += dz3[j];
    }
    for (j = 0; j < H; j++)
      for (k = 0; k < H; k++) g[W3 + H * j + k] += (double) bf16r(dz3[j]) * bf16r(f->h2[k]);
    for (k = 0; k < H; k++) {
      double s = 0.0;
      for (j = 0; j < H; j++) s += (double) bf16r(dz3[j]) * bf16r(P[W3 + H * j + k]);
      dz2[k] = (float) s * gelu_grad(f->z2[k]);
      g[B2 + k] += dz2[k];
    }
    for (j = 0; j < H; j++)
      for (k = 0; k < H; k++) g[W2 + H * j + k] += (double) bf16r(dz2[j]) * bf16r(f->h1[k]);
    for (k = 0; k < H; k++) {
      double s = 0.0;
      for (j = 0; j < H; j++) s += (double) bf16r(dz2[j]) * bf16r(P[W2 + H * j + k]);
      dz1[k] = (float) s * gelu_grad(f->z1[k]);
      g[B1 + k] += dz1[k];
      for (j = 0; j < 3; j++) g[W1 + 3 * k + j] += (double) dz1[k] * f->x[j];
    }
  }
  for (j = 0; j < NPARAM; j++) grad[j] = (float) g[j];
  free(g);
  free(f);
  return loss / n;
}
