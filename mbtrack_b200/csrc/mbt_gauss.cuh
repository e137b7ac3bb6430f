// mbt_gauss.cuh -- the transverse field of an elliptic Gaussian line
// charge, the field every beam-ion kick uses and the surrogate learns.
#pragma once
#include "mbt_wofz.cuh"

namespace mbt {

constexpr double kBiRoundRatio = 0.995;   // aspect ratio above which the field comes from quadrature

// 16-point Gauss-Legendre rule on [0, 1]
static __constant__ double kGl16X[16] = {
    0.005299532504175031, 0.0277124884633837, 0.06718439880608412, 0.1222977958224985,
    0.19106187779867811, 0.2709916111713863, 0.35919822461037054, 0.4524937450811813,
    0.5475062549188188, 0.6408017753896295, 0.7290083888286136, 0.8089381222013219,
    0.8777022041775016, 0.9328156011939159, 0.9722875115366163, 0.994700467495825};
static __constant__ double kGl16W[16] = {
    0.013576229705877088, 0.031126761969323728, 0.0475792558412463, 0.062314485627767036,
    0.07479799440828835, 0.08457825969750132, 0.09130170752246182, 0.09472530522753432,
    0.09472530522753432, 0.09130170752246182, 0.08457825969750132, 0.07479799440828835,
    0.062314485627767036, 0.0475792558412463, 0.031126761969323728, 0.013576229705877088};

// Field of a unit line charge density with an elliptic Gaussian profile,
// in units of lambda / (2 eps0): for sx >= sy the Bassetti-Erskine
// expression  (gy + i gx) = [w(z1) - exp(-dx^2/2sx^2 - dy^2/2sy^2) w(z2)]
// / (sqrt(pi) sqrt(2 (sx^2 - sy^2))),  z1 = (dx + i dy)/sqrt(2(sx^2-sy^2)),
// z2 = (dx sy/sx + i dy sx/sy)/sqrt(2(sx^2-sy^2)), evaluated in the first
// quadrant (w of the upper half plane only) with the signs of dx, dy put
// back; closer to round than kBiRoundRatio, where that expression cancels,
//   gx = dx/(pi sx^2) Int_0^1 t e^{-E(t)} D^{-1/2} dt,
//   gy = dy/(pi sx^2) Int_0^1 t e^{-E(t)} D^{-3/2} dt,
//   D = 1 - (1 - sy^2/sx^2) t^2,  E = t^2 (dx^2 + dy^2/D) / (2 sx^2)
// (the field integral with q = 2 sx^2 (1/t^2 - 1)), by 4 x 16-point
// Gauss-Legendre panels over the part of [0, 1] where E < 40.
__device__ __forceinline__ void gauss_field(double dx, double dy, double sx, double sy, double &gx, double &gy) {
  const double sgx = dx < 0.0 ? -1.0 : 1.0, sgy = dy < 0.0 ? -1.0 : 1.0;
  double ax = fabs(dx), ay = fabs(dy);
  const bool swap = sy > sx;
  if (swap) {
    const double t = ax; ax = ay; ay = t;
    const double u = sx; sx = sy; sy = u;
  }
  sy = fmax(sy, 1e-6 * sx);
  const double r = sy / sx;
  double fx, fy;
  if (r <= kBiRoundRatio) {
    const double fbe = sqrt(2.0 * (sx * sx - sy * sy));
    const double x1 = ax / fbe, y1 = ay / fbe;
    double w1r, w1i, w2r = 0.0, w2i = 0.0;
    wofz_dev(x1, y1, w1r, w1i);
    // beyond exp(-50) the second term lies below the last bit of the first
    // (|w| <= 1 in the upper half plane): w(z2) is not evaluated there
    const double arg = ax * ax / (2.0 * sx * sx) + ay * ay / (2.0 * sy * sy);
    const double e = arg > 50.0 ? 0.0 : exp(-arg);
    if (e != 0.0) wofz_dev(x1 * r, y1 / r, w2r, w2i);
    const double c = 1.0 / (1.7724538509055160273 * fbe);
    fx = c * (w1i - e * w2i);
    fy = c * (w1r - e * w2r);
  } else {
    const double q = 1.0 - r * r;
    const double inv2 = 1.0 / (2.0 * sx * sx);
    const double a0 = (ax * ax + ay * ay) * inv2;
    const double T = a0 > 40.0 ? sqrt(40.0 / a0) : 1.0;
    const double h = 0.25 * T;
    double ix = 0.0, iy = 0.0;
    for (int pnl = 0; pnl < 4; ++pnl) {
      for (int i = 0; i < 16; ++i) {
        const double t = h * (pnl + kGl16X[i]);
        const double D = 1.0 - q * t * t;
        const double f = t * exp(-(t * t) * (ax * ax + ay * ay / D) * inv2) / sqrt(D);
        const double wgt = h * kGl16W[i];
        ix += wgt * f;
        iy += wgt * (f / D);
      }
    }
    const double c = 1.0 / (3.14159265358979323846 * sx * sx);
    fx = c * ax * ix;
    fy = c * ay * iy;
  }
  if (swap) {
    const double t = fx; fx = fy; fy = t;
  }
  gx = sgx * fx;
  gy = sgy * fy;
}

}  // namespace mbt
