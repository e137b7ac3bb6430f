// mbt_beamion.cuh -- fast beam-ion interaction of the bunch train with the
// residual gas, every electron macroparticle kicked (model in mbt.h,
// mbt_beam_ion).  Physics after fbi_weakstrong.c: ions created by each
// bunch passage (:214-236), drift between passages (:370-375), kicks by the
// bunch field (:393-405) computed with the Bassetti-Erskine formula
// (:154-197), the coupling constant factF = e / (A m_p) (:40).
//
// One turn of the stage is four launches after the turn's statistics:
//   bi_frames  centroid and rms of every bunch at every interaction point
//              (linear optics from the kick point);
//   bi_ions    one thread per macro-ion: created at its passage, then drift,
//              cloud moments and kick for every later bunch of the train;
//              block sums of the moments go to one slot per (point, bunch,
//              creating passage, block), no atomics;
//   bi_clouds  one block per (point, bunch): the slots summed in a fixed
//              order -> ions, centroid and rms of the cloud that bunch meets;
//   bi_kick    one block per tile: every electron kicked by the clouds of its
//              bunch at every point, kicks mapped back to the kick point.
#pragma once
#include <cstdint>

#include "mbt_common.cuh"
#include "mbt_device.cuh"
#include "mbt_philox.cuh"
#include "mbt_wofz.cuh"

namespace mbt {

constexpr int kBiThreads = 256;
constexpr int kBiMaxIp = 64;
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
    double w1r, w1i, w2r, w2i;
    wofz_dev(x1, y1, w1r, w1i);
    wofz_dev(x1 * r, y1 / r, w2r, w2i);
    const double e = exp(-(ax * ax / (2.0 * sx * sx) + ay * ay / (2.0 * sy * sy)));
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

// Constants and buffers of the stage (passed by value to its kernels).
struct BiArgs {
  int n_ip, n_new, bpp, nb;       // points, ions per passage, blocks per passage, bunches
  long T;                          // nb (nb - 1) / 2 passages with a successor, summed
  double dt_bucket;                // T0 / h
  double kion_per_amp;             // ion velocity kick per unit field per ampere of bunch current
  double ke;                       // electron deflection per ion per unit field: -2 pi r_e / gamma
  double w_per_amp;                // ions per macro-ion per ampere of the creating bunch
  double betaH, alphaH, betaV, alphaV;
  PhiloxKeys keys;
  const double *trig;              // n_ip x 4: cos, sin of the phase advance (x, y)
  const double *mom;               // nbunch x 10 (bunch_reduce): x, x', var x, cov xx', var x', then y
  double *frame;                   // n_ip x nbunch x 4: centroid x, y, rms x, y at the point
  double *part;                    // slots: n_ip x T x bpp x 5
  double *cloud;                   // n_ip x nbunch x 5: ions, centroid x, y, rms x, y
  const int *bunch_kb;             // nbunch buckets
  const double *ib;                // nbunch currents [A]
  const long *turn;                // device turn counter
};

__device__ __forceinline__ long bi_tri(long b) { return b * (b - 1) / 2; }

// Bunch centroid and rms at every point: x_k = (c + alpha s) x + beta s x'.
__global__ void bi_frames(BiArgs bi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= bi.n_ip * bi.nb) return;
  const int k = i / bi.nb, b = i % bi.nb;
  const double *m = bi.mom + (size_t)b * 10;
  const double *tr = bi.trig + 4 * k;
  const double mx = tr[0] + bi.alphaH * tr[1], sx = bi.betaH * tr[1];
  const double my = tr[2] + bi.alphaV * tr[3], sy = bi.betaV * tr[3];
  double *F = bi.frame + (size_t)i * 4;
  F[0] = mx * m[0] + sx * m[1];
  F[1] = my * m[5] + sy * m[6];
  const double vx = mx * mx * m[2] + 2.0 * mx * sx * m[3] + sx * sx * m[4];
  const double vy = my * my * m[7] + 2.0 * my * sy * m[8] + sy * sy * m[9];
  F[2] = sqrt(vx > 0.0 ? vx : 0.0);
  F[3] = sqrt(vy > 0.0 ? vy : 0.0);
}

// Two standard normals from one Philox output (Box-Muller in FP64).
__device__ __forceinline__ void bi_normals(const U4 &r, double &g1, double &g2) {
  const double u1 = ((double)r.x + 1.0) * 2.3283064365386962890625e-10;   // (0, 1]
  const double u2 = (double)r.y * 2.3283064365386962890625e-10;           // [0, 1)
  const double u3 = ((double)r.z + 1.0) * 2.3283064365386962890625e-10;
  const double u4 = (double)r.w * 2.3283064365386962890625e-10;
  g1 = sqrt(-2.0 * log(u1)) * cos(2.0 * 3.14159265358979323846 * u2);
  g2 = sqrt(-2.0 * log(u3)) * cos(2.0 * 3.14159265358979323846 * u4);
}

__global__ void __launch_bounds__(kBiThreads) bi_ions(BiArgs bi) {
  const int blk = blockIdx.x, b0 = blockIdx.y, k = blockIdx.z;
  const int j = blk * kBiThreads + threadIdx.x;
  const bool live = j < bi.n_new;
  const long turn = *bi.turn;
  double x = 0.0, y = 0.0, vx = 0.0, vy = 0.0, w = 0.0;
  if (live) {
    const double *F0 = bi.frame + ((size_t)k * bi.nb + b0) * 4;
    const U4 c = {(uint32_t)j, (uint32_t)b0 | ((uint32_t)k << 20), (uint32_t)turn, (uint32_t)(turn >> 32)};
    double g1, g2;
    bi_normals(philox4x32_10k(c, bi.keys), g1, g2);
    x = F0[0] + F0[2] * g1;
    y = F0[1] + F0[3] * g2;
    w = bi.w_per_amp * bi.ib[b0];
  }
  __shared__ double red[kBiThreads / 32][5];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int b = b0 + 1; b < bi.nb; ++b) {
    const double dt = (double)(bi.bunch_kb[b] - bi.bunch_kb[b - 1]) * bi.dt_bucket;
    x = x + dt * vx;
    y = y + dt * vy;
    const double *F = bi.frame + ((size_t)k * bi.nb + b) * 4;
    const double dx = x - F[0], dy = y - F[1];
    double s[5] = {w, w * dx, w * dy, w * (dx * dx), w * (dy * dy)};
#pragma unroll
    for (int m = 0; m < 5; ++m) s[m] = warp_sum(s[m]);
    if (lane == 0)
      for (int m = 0; m < 5; ++m) red[warp][m] = s[m];
    __syncthreads();
    if (threadIdx.x < 5) {
      double t = 0.0;
      for (int q = 0; q < kBiThreads / 32; ++q) t += red[q][threadIdx.x];
      bi.part[(((size_t)k * bi.T + bi_tri(b) + b0) * bi.bpp + blk) * 5 + threadIdx.x] = t;
    }
    __syncthreads();
    if (live) {
      double gx, gy;
      gauss_field(dx, dy, F[2], F[3], gx, gy);
      const double kk = bi.kion_per_amp * bi.ib[b];
      vx = vx + kk * gx;
      vy = vy + kk * gy;
    }
  }
}

__global__ void __launch_bounds__(kBiThreads) bi_clouds(BiArgs bi) {
  const int b = blockIdx.x, k = blockIdx.y;
  const long nslot = (long)b * bi.bpp;
  const double *P = bi.part + ((size_t)k * bi.T + bi_tri(b)) * bi.bpp * 5;
  double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (long q = threadIdx.x; q < nslot; q += kBiThreads)
    for (int m = 0; m < 5; ++m) s[m] += P[q * 5 + m];
  __shared__ double red[kBiThreads / 32][5];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int m = 0; m < 5; ++m) s[m] = warp_sum(s[m]);
  if (lane == 0)
    for (int m = 0; m < 5; ++m) red[warp][m] = s[m];
  __syncthreads();
  if (threadIdx.x == 0) {
    double t[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int q = 0; q < kBiThreads / 32; ++q)
      for (int m = 0; m < 5; ++m) t[m] += red[q][m];
    const double *F = bi.frame + ((size_t)k * bi.nb + b) * 4;
    double *C = bi.cloud + ((size_t)k * bi.nb + b) * 5;
    if (t[0] > 0.0) {
      const double mx = t[1] / t[0], my = t[2] / t[0];
      const double vx = t[3] / t[0] - mx * mx, vy = t[4] / t[0] - my * my;
      C[0] = t[0];
      C[1] = F[0] + mx;
      C[2] = F[1] + my;
      C[3] = sqrt(vx > 0.0 ? vx : 0.0);
      C[4] = sqrt(vy > 0.0 ? vy : 0.0);
    } else {
      for (int m = 0; m < 5; ++m) C[m] = 0.0;
    }
  }
}

// Every electron of a tile: the deflection by each cloud its bunch meets,
// at that point's coordinates, mapped back to the kick point
// (x += -beta s theta, x' += (c + alpha s) theta).
__global__ void __launch_bounds__(kBiThreads) bi_kick(Args a, BiArgs bi) {
  const Tile tile = a.tiles[blockIdx.x];
  const int b = tile.bunch;
  __shared__ double cl[kBiMaxIp][5];
  __shared__ double tr[kBiMaxIp][4];
  for (int i = threadIdx.x; i < bi.n_ip; i += kBiThreads) {
    const double *C = bi.cloud + ((size_t)i * bi.nb + b) * 5;
    cl[i][0] = bi.ke * C[0];
    for (int m = 1; m < 5; ++m) cl[i][m] = C[m];
    for (int m = 0; m < 4; ++m) tr[i][m] = bi.trig[4 * i + m];
  }
  __syncthreads();
  const size_t n6 = (size_t)a.npad;
  double *C = a.coord;
  for (int p = tile.start + threadIdx.x; p < tile.start + tile.count; p += kBiThreads) {
    const double x = C[1 * n6 + p], z = C[2 * n6 + p], xp = C[4 * n6 + p], zp = C[5 * n6 + p];
    double ddx = 0.0, ddxp = 0.0, ddz = 0.0, ddzp = 0.0;
    for (int k = 0; k < bi.n_ip; ++k) {
      if (cl[k][0] == 0.0) continue;
      const double mx = tr[k][0] + bi.alphaH * tr[k][1], sxb = bi.betaH * tr[k][1];
      const double my = tr[k][2] + bi.alphaV * tr[k][3], syb = bi.betaV * tr[k][3];
      const double xk = mx * x + sxb * xp, zk = my * z + syb * zp;
      double gx, gy;
      gauss_field(xk - cl[k][1], zk - cl[k][2], cl[k][3], cl[k][4], gx, gy);
      const double thx = cl[k][0] * gx, thy = cl[k][0] * gy;
      ddx = ddx - sxb * thx;
      ddxp = ddxp + mx * thx;
      ddz = ddz - syb * thy;
      ddzp = ddzp + my * thy;
    }
    C[1 * n6 + p] = x + ddx;
    C[4 * n6 + p] = xp + ddxp;
    C[2 * n6 + p] = z + ddz;
    C[5 * n6 + p] = zp + ddzp;
  }
}

__global__ void gauss_field_kernel(long n, const double *__restrict__ dx, const double *__restrict__ dy,
                                   const double *__restrict__ sx, const double *__restrict__ sy,
                                   double *__restrict__ gx, double *__restrict__ gy) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double u, v;
    gauss_field(dx[i], dy[i], sx[i], sy[i], u, v);
    gx[i] = u;
    gy[i] = v;
  }
}

}  // namespace mbt
