/*
 * mlp_oracle.c -- TEST INFRASTRUCTURE ONLY: CPU restatement of the learned
 * field network of libmbt (mbt.h, mbt_mlp_*): forward pass and gradient
 * with the same roundings of the tensor-core operands (FP16 weights and
 * activations and FP16 GELU arithmetic in the forward pass, BF16 operands
 * of the backward products), sums in double.  Used by tests/ to check the
 * GPU kernels.
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

/* round to the nearest FP16 (ties to even), as a float */
static float h16(double v)
{
  const double a = fabs(v);
  double q;
  int e;
  if (!(a < 65520.0)) return a != a ? (float) v : (float) copysign(INFINITY, v);
  if (a < 6.103515625e-05) {
    q = 5.9604644775390625e-08;              /* subnormal step 2^-24 */
  } else {
    frexp(a, &e);                            /* a in [2^(e-1), 2^e) */
    q = ldexp(1.0, e - 11);                  /* 11 significant bits */
  }
  return (float) (nearbyint(v / q) * q);
}

/* GELU in FP16 pair arithmetic as the GPU evaluates it (gelu_h2): every
 * step rounded to FP16, FP16 constants; the GPU's tanh is the hardware
 * approximation, this restatement libm's tanh rounded to FP16. */
static float gelu(float x)
{
  const float c1c2 = 0.035675048828125f, c1 = 0.7978515625f;
  const float z = h16(x);
  const float t = h16((double) z * z);
  const float p = h16((double) c1c2 * t + c1);
  const float y = h16((double) z * p);
  const float th = h16(tanh((double) y));
  const float hz = h16(0.5 * z);
  return h16((double) hz * th + hz);
}

static float gelu_grad(float x)
{
  const float y = x * fmaf(0.035677408136300125f, x * x, 0.7978845608028654f);
  const float th = tanhf(y);
  return 0.5f * (1.0f + th) + 0.5f * x * (1.0f - th * th) * 0.7978845608028654f * (1.0f + 0.134145f * x * x);
}


typedef struct fwd_t {
  float x[3], z1[H], h1[H], z2[H], h2[H], z3[H], h3[H], out[2];
} fwd_t;

static void forward_one(const float *P, const float *abr, fwd_t *f)
{
  int j, k;
  f->x[0] = 0.25f * abr[0] - 1.0f;
  f->x[1] = 0.25f * abr[1] - 1.0f;
  f->x[2] = fmaf(0.66761703f, logf(abr[2]), 1.0f);   /* 1 + 2 ln r / ln 20 */
  for (j = 0; j < H; j++) {
    float z = P[B1 + j];
    z = fmaf(P[W1 + 3 * j], f->x[0], z);
    z = fmaf(P[W1 + 3 * j + 1], f->x[1], z);
    z = fmaf(P[W1 + 3 * j + 2], f->x[2], z);
    f->z1[j] = z;
    f->h1[j] = gelu(z);
  }
  /* the activations are FP16 values already; the weights round to FP16 */
  for (j = 0; j < H; j++) {
    double s = 0.0;
    for (k = 0; k < H; k++) s += (double) f->h1[k] * (double) h16(P[W2 + H * j + k]);
    f->z2[j] = (float) s + P[B2 + j];
    f->h2[j] = gelu(f->z2[j]);
  }
  for (j = 0; j < H; j++) {
    double s = 0.0;
    for (k = 0; k < H; k++) s += (double) f->h2[k] * (double) h16(P[W3 + H * j + k]);
    f->z3[j] = (float) s + P[B3 + j];
    f->h3[j] = gelu(f->z3[j]);
  }
  for (j = 0; j < 2; j++) {
    double s = 0.0;
    for (k = 0; k < H; k++) s += (double) f->h3[k] * (double) h16(P[W4 + H * j + k]);
    f->out[j] = (float) s + P[B4 + j];
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
