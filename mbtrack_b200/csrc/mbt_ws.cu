// mbt_ws.cu -- the slice model (BunchModel = STRONG) with fast beam-ion
// interaction on the device: the C ABI of mbt_ws.h.
//
// One turn is four launches on the context's stream:
//
//   ws_bunch     one block per filled bunch: RF step of the slice xtau/xeps
//                (transformSbunch_shortrange rw_weakstrong.c:24-37), the
//                slice-weighted centroids (bunch_strong_updateCM
//                bunch_strong.c:221-270) into the centroid history, the
//                monitor statistics (bunch.c:516-549), the Bassetti-Erskine
//                field grid of every slice and the bunch's own macro-ions
//                with their pull by the later slices of the bunch
//                (fbi_weakstrong_bunch fbi_weakstrong.c:98-290);
//   ws_optic_rw  one block per filled bunch: one-turn rotation of the
//                slice centroids (transformSbunch_optic rw_weakstrong.c:
//                194-253) and the long-range resistive-wall kick of every
//                source bunch (transformSbunch_longrange :68-192), one
//                thread per source, added in source order;
//   ws_train     one block per SOURCE bunch (MBT_WS_SPLIT > 1 cuts a
//                bunch of more than 512 ions over several blocks),
//                MBT_WS_IPT macro-ions per thread: the ions of that bunch
//                travel down the train (drift between buckets, pull by each
//                slice of each later bunch, whose field grid the block
//                stages in shared memory first; fbi_weakstrong_train
//                fbi_weakstrong.c:325-426); per later
//                bunch and slice the block writes its share of the kick
//                sum  sum_ions Nri E  to a triangular buffer, in a fixed
//                reduction order (warp shuffles, then warps in order), so
//                runs repeat bit for bit;
//   ws_kick      one block per filled bunch: adds the shares of all
//                earlier source bunches in source order and kicks each
//                slice's xp/zp (fbi_weakstrong.c:409-416); ion-list
//                centroid and mean slice zz for the output files.
//
// Ion trajectories depend only on the field grids, which the bunch step
// fixes before the train, so the ions of different source bunches never
// wait on one another: the train has no grid-wide synchronisation, and its
// length is the first bunch's chain of (nbunch - 1) x slices pulls.
//
// The file is compiled with -fmad=false: every product and sum rounds as
// the reference's x86-64 build does (no contraction; the divisions by the
// grid step go through div_known, exact by construction), so the arithmetic
// differs from the reference only where the device's sin, exp and w(z)
// differ from glibc's in the last bits, and in the summation order of the
// ion kick and ion centroid sums.  Constants the reference computes with
// libm (the one-turn matrices, the resistive-wall prefactors) come from
// the host.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mbt.h"
#include "mbt_ws.h"
#include "mbt_wofz.cuh"

namespace {

constexpr double kCLight = 2.997925e+08;
constexpr double kEps0 = 8.854187817620e-12;
constexpr double kECharge = 1.602e-19;
constexpr double kERadius = 2.819e-15;
constexpr double kFKilo = 1.0e+03;
constexpr double kFMega = 1.0e+06;
constexpr double kFTera = 1.0e+12;
constexpr int kMaxSlices = 49;
constexpr int kMaxHist = 32;
constexpr int kBunchThreads = 256;
constexpr int kRwThreads = 128;
constexpr int kKickThreads = 64;
constexpr long kChunk = 256;   // turns per block of host outputs
#ifndef MBT_WS_IPT
#define MBT_WS_IPT 2             // macro-ions per thread in the ion train
#endif
#ifndef MBT_WS_SPLIT
#define MBT_WS_SPLIT 1           // train blocks per source bunch (above 512 ions)
#endif
#ifndef MBT_WS_EXCLUSIVE
#define MBT_WS_EXCLUSIVE 0       // pad the train's shared memory to one block per SM
#endif
#ifndef MBT_WS_PAIR
#define MBT_WS_PAIR 0            // reduce the kick sums of two slices together
#endif
constexpr int kIpt = MBT_WS_IPT;
// largest train block: 49 slices x 25 grid points, kIpt ions a thread
constexpr int kTrainMaxThreads = ((kMaxSlices * 25 + kIpt - 1) / kIpt + 31) / 32 * 32;

struct WsConst {
  int nb, S, G, off, nion, nmt, nharm, fbii, rw_long, trigger_rw, Nmlt;
  int nsplit;   // train blocks per source bunch
  int track[3];
  long nrev_mon;
  double vrf_e0, wrf, phai0, Urad, T0, ac;
  double alpha1[3], beta1[3], gamma1[3];
  double v11, v12, v21, v22, h11, h12, h21, h22;   // one-turn matrices VER, HOR
  double a11[2], a12[2];                           // history rotation HOR, VER
  double prfrw[2], prfrw_trig[2];
  double Pref0, Dub0, Lc, fNp;
  double factBE, sgm_xx, sgm_zz, agLOCx, agLOCz, agABSx, agABSz, deltT, factF, Ldmsgm;
  double rABSx, rABSz;   // 1 / agABSx, 1 / agABSz, correctly rounded
  double fdq_den;   // 2 eps0 sqrt(pi) factBE c deltT
  double factjp0;   // factRN 4 pi eps0 r_e / Gamma
  double T0h;       // T0 / h
  double cdt;       // c deltT
};

// a / b, correctly rounded, for a divisor b whose correctly rounded
// reciprocal rb is known: q0 = a rb is within about one ulp of a / b; one
// residual correction q1 = q0 + (a - b q0) rb (the residual exact by FMA)
// makes it faithful, a second gives the correctly rounded quotient
// (P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Dev. 34(1), 1990: with rb the
// correctly rounded 1/b and q faithful, q + (a - b q) rb rounds to a / b).
// A zero residual means q is exact and is kept, sign of zero included.
// Five FP64 operations in place of a full division.
__device__ __forceinline__ double div_known(double a, double b, double rb) {
  const double q0 = __dmul_rn(a, rb);
  const double r0 = __fma_rn(-q0, b, a);
  const double q1 = r0 == 0.0 ? q0 : __fma_rn(r0, rb, q0);
  const double r1 = __fma_rn(-q1, b, a);
  return r1 == 0.0 ? q1 : __fma_rn(r1, rb, q1);
}

// get_linearly_interpolated_Efields (fbi_weakstrong.c:454-580): truncated
// grid index of (xx, yy) on the absolute grid, the neighbour on the side
// away from the origin, linear in each axis, constant beyond the grid.
__device__ __forceinline__ void ws_interp(const WsConst &C, const double *__restrict__ Ex,
                                          const double *__restrict__ Ey, int icell, double xx, double yy, double &ex,
                                          double &ey) {
  const int off = C.off, G = C.G;
  const bool px = xx >= 0.0, pz = yy >= 0.0;
  int k1x = __double2int_rz(div_known(xx, C.agABSx, C.rABSx));
  int k1z = __double2int_rz(div_known(yy, C.agABSz, C.rABSz)), k2x, k2z;
  if (pz) {
    k2z = k1z < off ? k1z + 1 : k1z;
    k1z = min(k1z, off);
    k2z = min(k2z, off);
  } else {
    k2z = k1z > -off ? k1z - 1 : k1z;
    k1z = max(k1z, -off);
    k2z = max(k2z, -off);
  }
  if (px) {
    k2x = k1x < off ? k1x + 1 : k1x;
    k1x = min(k1x, off);
    k2x = min(k2x, off);
  } else {
    k2x = k1x > -off ? k1x - 1 : k1x;
    k1x = max(k1x, -off);
    k2x = max(k2x, -off);
  }
  const int b = icell * G;
  const int i1 = (b + k1x + off) * G + k1z + off, i2 = (b + k2x + off) * G + k1z + off;
  const int i3 = (b + k1x + off) * G + k2z + off, i4 = (b + k2x + off) * G + k2z + off;
  const double fx = div_known(xx - k1x * C.agABSx, C.agABSx, C.rABSx);
  const double fz = div_known(yy - k1z * C.agABSz, C.agABSz, C.rABSz);
  const double y1 = Ey[i1], y2 = Ey[i2], y3 = Ey[i3], y4 = Ey[i4];
  const double x1 = Ex[i1], x2 = Ex[i2], x3 = Ex[i3], x4 = Ex[i4];
  double ey5, ey6, ex5, ex6;
  if (px) {
    ey5 = y1 + fx * (y2 - y1);
    ey6 = y3 + fx * (y4 - y3);
    ex5 = x1 + fx * (x2 - x1);
    ex6 = x3 + fx * (x4 - x3);
  } else {
    ey5 = y1 - fx * (y2 - y1);
    ey6 = y3 - fx * (y4 - y3);
    ex5 = x1 - fx * (x2 - x1);
    ex6 = x3 - fx * (x4 - x3);
  }
  ey = pz ? ey5 + fz * (ey6 - ey5) : ey5 - fz * (ey6 - ey5);
  ex = pz ? ex5 + fz * (ex6 - ex5) : ex5 - fz * (ex6 - ex5);
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(kBunchThreads) ws_bunch(WsConst C, double *__restrict__ s,
                                                         double *__restrict__ hist, const int *__restrict__ npop,
                                                         const int *__restrict__ nofe,
                                                         const double *__restrict__ nelec, double *__restrict__ fx,
                                                         double *__restrict__ fy, double *__restrict__ ion,
                                                         double *__restrict__ own, double *__restrict__ cm_out,
                                                         double *__restrict__ st_out) {
  extern __shared__ double sh[];   // Ex[nion], Ey[nion]
  __shared__ double c6[6];
  __shared__ double red[3][kBunchThreads / 32];
  const int ib = blockIdx.x, S = C.S, n = C.nion, tid = threadIdx.x;
  double *sl = s + (size_t)ib * 6 * S;
  double *xtau = sl, *xeps = sl + S, *xx = sl + 2 * S, *zz = sl + 4 * S;
  if (tid < S) {
    const double t0 = xtau[tid], e0 = xeps[tid];
    const double gain = C.vrf_e0 * sin(C.wrf * t0 + C.phai0);
    xeps[tid] = e0 + gain - C.Urad;
    xtau[tid] = t0 - e0 * C.T0 * C.ac;
  }
  __syncthreads();
  if (tid < 3) {
    const double *u = sl + 2 * tid * S, *up = u + S;
    double uu = 0.0, ss = 0.0;
    int np = 0;
    for (int c = 0; c < S; ++c) {
      const double w = (double)npop[c];
      uu += u[c] * w;
      ss += up[c] * w;
      np += npop[c];
    }
    c6[2 * tid] = uu / (double)np;
    c6[2 * tid + 1] = ss / (double)np;
  }
  __syncthreads();
  if (cm_out && tid < 6) cm_out[(size_t)ib * 6 + tid] = c6[tid];
  if (tid < 4) {
    double *h = hist + ((size_t)ib * 4 + tid) * C.nmt;
    for (int j = C.nmt - 2; j >= 0; --j) h[j + 1] = h[j];
    h[0] = c6[2 + tid];
  }
  if (st_out && tid < 3) {
    double *o = st_out + (size_t)ib * 18;
    const int pl = tid;
    if (!C.track[pl]) {
      for (int k = 0; k < 6; ++k) o[3 * k + pl] = 0.0;
    } else {
      const double *u = sl + 2 * pl * S, *up = u + S;
      const double pos = c6[2 * pl], slope = c6[2 * pl + 1];
      const double g = C.gamma1[pl], a = C.alpha1[pl], be = C.beta1[pl];
      double sq = 0.0, sp = 0.0, ai = 0.0;
      int nw = 0;
      for (int c = 0; c < S; ++c) {
        const double w = (double)npop[c];
        sq += (u[c] - pos) * (u[c] - pos) * w;
        sp += (up[c] - slope) * (up[c] - slope) * w;
        ai += w * (g * (u[c] * u[c]) + 2.0 * a * u[c] * up[c] + be * (up[c] * up[c]));
        nw += npop[c];
      }
      o[pl] = pos;
      o[3 + pl] = sqrt(sq / (double)nw);
      o[6 + pl] = slope;
      o[9 + pl] = sqrt(sp / (double)nw);
      o[12 + pl] = ai / (double)nw;
      o[15 + pl] = g * (pos * pos) + 2.0 * a * pos * slope + be * (slope * slope);
    }
  }
  if (!C.fbii) return;
  const int G2 = C.G * C.G;
  const double ne = nelec[ib];
  for (int p = tid; p < n; p += blockDim.x) {
    const int icell = p / G2, r = p - icell * G2;
    const int msx = r / C.G - C.off, msz = r % C.G - C.off;
    const double dQ = ne * (double)npop[icell] * kECharge;
    const double factdQ = dQ / C.fdq_den;
    const double Dx = msx * C.agABSx - xx[icell];
    const double xi1 = Dx / C.factBE, xi2 = xi1 * C.sgm_zz / C.sgm_xx;
    const double Dy = msz * C.agABSz - zz[icell];
    const double yi1 = Dy / C.factBE, yi2 = yi1 * C.sgm_xx / C.sgm_zz;
    double w1r, w1i, w2r, w2i;
    mbt::wofz_dev(xi1, yi1, w1r, w1i);
    mbt::wofz_dev(xi2, yi2, w2r, w2i);
    const double e = exp(-(Dx * Dx * kFMega / (2 * C.sgm_xx * C.sgm_xx) + Dy * Dy * kFMega / (2 * C.sgm_zz * C.sgm_zz)));
    const double ex = -factdQ * (w1i - e * w2i), ey = -factdQ * (w1r - e * w2r);
    sh[p] = ex;
    sh[n + p] = ey;
    fx[(size_t)ib * n + p] = ex;
    fy[(size_t)ib * n + p] = ey;
  }
  __syncthreads();
  const double convion = ne * C.Ldmsgm;
  double sN = 0.0, sX = 0.0, sY = 0.0;
  double *li = ion + (size_t)ib * 5 * n;
  for (int p = tid; p < n; p += blockDim.x) {
    const int icell = p / G2, r = p - icell * G2;
    const int msx = r / C.G - C.off, msz = r % C.G - C.off;
    const double N = convion * (double)nofe[p];
    double x = xx[icell] + msx * C.agLOCx, y = zz[icell] + msz * C.agLOCz, xd = 0.0, yd = 0.0;
    for (int c = icell + 1; c < S; ++c) {
      double ex, ey;
      ws_interp(C, sh, sh + n, c, x, y, ex, ey);
      xd = xd + C.deltT * (C.factF * ex);
      x = x + C.deltT * xd;
      yd = yd + C.deltT * (C.factF * ey);
      y = y + C.deltT * yd;
    }
    li[p] = N;
    li[n + p] = x;
    li[2 * n + p] = xd;
    li[3 * n + p] = y;
    li[4 * n + p] = yd;
    sN += N;
    sX += N * x;
    sY += N * y;
  }
  sN = warp_sum(sN);
  sX = warp_sum(sX);
  sY = warp_sum(sY);
  if ((tid & 31) == 0) {
    red[0][tid >> 5] = sN;
    red[1][tid >> 5] = sX;
    red[2][tid >> 5] = sY;
  }
  __syncthreads();
  if (tid < 3) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[tid][w];
    own[(size_t)ib * 3 + tid] = v;
  }
}

__global__ void __launch_bounds__(kRwThreads) ws_optic_rw(WsConst C, double *__restrict__ s,
                                                         const double *__restrict__ hist,
                                                         const double *__restrict__ ibunch,
                                                         const int *__restrict__ bucket, long rev) {
  extern __shared__ double dup[];   // [nb]
  const int ib = blockIdx.x, S = C.S, tid = threadIdx.x;
  double *sl = s + (size_t)ib * 6 * S;
  double *xx = sl + 2 * S, *xp = sl + 3 * S, *zz = sl + 4 * S, *zp = sl + 5 * S;
  if (tid < S) {
    const double z = zz[tid], zq = zp[tid], x = xx[tid], xq = xp[tid];
    zz[tid] = C.v11 * z + C.v12 * zq;
    zp[tid] = C.v21 * z + C.v22 * zq;
    xx[tid] = C.h11 * x + C.h12 * xq;
    xp[tid] = C.h21 * x + C.h22 * xq;
  }
  if (!C.rw_long) return;
  const int kb = bucket[ib];
  for (int pl = 1; pl <= 2; ++pl) {
    if (!C.track[pl]) continue;
    __syncthreads();
    const double prf = (C.trigger_rw && rev < 50) ? C.prfrw_trig[pl - 1] : C.prfrw[pl - 1];
    const double a11 = C.a11[pl - 1], a12 = C.a12[pl - 1];
    for (int jb = tid; jb < C.nb; jb += blockDim.x) {
      double Dup = 0.0;
      if (rev >= C.Nmlt) {
        const int sb = bucket[jb];
        const double *uh = hist + ((size_t)jb * 4 + (pl == 1 ? 0 : 2)) * C.nmt, *ph = uh + C.nmt;
        double D0 = C.Lc;
        if (sb > kb) D0 = (double)(sb - kb) * C.Dub0;
        if (sb < kb) D0 = (double)(C.nharm + sb - kb) * C.Dub0;
        for (int j = 0; j <= C.Nmlt; ++j) {
          const double Dujk = D0 + (double)j * C.Lc;
          const double Dtjk = Dujk / kCLight;
          const double W = prf / sqrt(Dtjk);
          const int jm = sb > kb ? j : j + 1;
          const double u = a11 * uh[jm] + a12 * ph[jm];
          Dup = Dup + (C.fNp * u) * W;
        }
        Dup = C.Pref0 * ibunch[jb] * Dup;
      }
      dup[jb] = Dup;
    }
    __syncthreads();
    if (tid < S) {
      double *up = pl == 1 ? xp : zp;
      double v = up[tid];
      for (int jb = 0; jb < C.nb; ++jb) v += dup[jb];
      up[tid] = v;
    }
  }
}

__device__ __forceinline__ void warp_sum4(double &a, double &b, double &c, double &d) {
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
    d += __shfl_xor_sync(0xffffffffu, d, o);
  }
}

// One slice's pull on this thread's ions: the kick-sum shares (ax, ay).
__device__ __forceinline__ void train_pull(const WsConst &C, const double *__restrict__ Ex,
                                           const double *__restrict__ Ey, int c, const double (&N)[kIpt],
                                           double (&X)[kIpt], double (&XD)[kIpt], double (&Y)[kIpt],
                                           double (&YD)[kIpt], double &ax, double &ay) {
  ax = 0.0;
  ay = 0.0;
#pragma unroll
  for (int q = 0; q < kIpt; ++q) {
    double ex, ey;
    ws_interp(C, Ex, Ey, c, X[q], Y[q], ex, ey);
    XD[q] = XD[q] + C.deltT * (C.factF * ex);
    X[q] = X[q] + C.deltT * XD[q];
    YD[q] = YD[q] + C.deltT * (C.factF * ey);
    Y[q] = Y[q] + C.deltT * YD[q];
    ax += N[q] * ex;
    ay += N[q] * ey;
  }
}

__global__ void __launch_bounds__(kTrainMaxThreads) ws_train(WsConst C, const int *__restrict__ bucket,
                                                             const double *__restrict__ fx,
                                                             const double *__restrict__ fy,
                                                             const double *__restrict__ ion,
                                                             double *__restrict__ part, double *__restrict__ ipart) {
  // [2][nion] the destination bunch's field grid, [S][nw][2] kick shares,
  // [nw][2] centroid shares
  extern __shared__ double sw[];
  const int src = blockIdx.x / C.nsplit, piece = blockIdx.x - src * C.nsplit;
  const int tid = threadIdx.x, n = C.nion, S = C.S;
  const int nw = blockDim.x >> 5, lane = tid & 31, wid = tid >> 5;
  const double *li = ion + (size_t)src * 5 * n;
  double N[kIpt], X[kIpt], XD[kIpt], Y[kIpt], YD[kIpt];
#pragma unroll
  for (int q = 0; q < kIpt; ++q) {
    const int p = (piece * kIpt + q) * blockDim.x + tid;
    const bool ok = p < n;
    N[q] = ok ? li[p] : 0.0;
    X[q] = ok ? li[n + p] : 0.0;
    XD[q] = ok ? li[2 * n + p] : 0.0;
    Y[q] = ok ? li[3 * n + p] : 0.0;
    YD[q] = ok ? li[4 * n + p] : 0.0;
  }
  double *gx = sw, *gy = sw + n;
  double *wsum = sw + 2 * (size_t)n, *wcm = wsum + (size_t)S * nw * 2;
  int kbprev = bucket[src];
  for (int k = src + 1; k < C.nb; ++k) {
    const int kb = bucket[k];
    const double Dt = fabs((double)(kb - kbprev)) * C.T0h;
    // the destination bunch's grid into shared memory: one coalesced pass
    // instead of dependent L2 reads inside every pull
    for (int i = tid; i < n; i += blockDim.x) {
      gx[i] = fx[(size_t)k * n + i];
      gy[i] = fy[(size_t)k * n + i];
    }
#pragma unroll
    for (int q = 0; q < kIpt; ++q) {
      X[q] = X[q] + Dt * XD[q];
      Y[q] = Y[q] + Dt * YD[q];
    }
    __syncthreads();
    const double *Ex = gx, *Ey = gy;
    // slices two at a time: the two slices' shuffle reductions interleave
    int c = 0;
#if !MBT_WS_PAIR
    for (; c + 1 < S; ++c) {
      double ax, ay;
      train_pull(C, Ex, Ey, c, N, X, XD, Y, YD, ax, ay);
      ax = warp_sum(ax);
      ay = warp_sum(ay);
      if (lane == 0) {
        wsum[((size_t)c * nw + wid) * 2] = ax;
        wsum[((size_t)c * nw + wid) * 2 + 1] = ay;
      }
    }
#endif
    for (; c + 1 < S; c += 2) {
      double ax0, ay0, ax1, ay1;
      train_pull(C, Ex, Ey, c, N, X, XD, Y, YD, ax0, ay0);
      train_pull(C, Ex, Ey, c + 1, N, X, XD, Y, YD, ax1, ay1);
      warp_sum4(ax0, ay0, ax1, ay1);
      if (lane == 0) {
        wsum[((size_t)c * nw + wid) * 2] = ax0;
        wsum[((size_t)c * nw + wid) * 2 + 1] = ay0;
        wsum[((size_t)(c + 1) * nw + wid) * 2] = ax1;
        wsum[((size_t)(c + 1) * nw + wid) * 2 + 1] = ay1;
      }
    }
    double cx = 0.0, cy = 0.0;
    if (c < S) {
      double ax, ay;
      train_pull(C, Ex, Ey, c, N, X, XD, Y, YD, ax, ay);
#pragma unroll
      for (int q = 0; q < kIpt; ++q) {
        cx += N[q] * X[q];
        cy += N[q] * Y[q];
      }
      warp_sum4(ax, ay, cx, cy);
      if (lane == 0) {
        wsum[((size_t)c * nw + wid) * 2] = ax;
        wsum[((size_t)c * nw + wid) * 2 + 1] = ay;
      }
    } else {
#pragma unroll
      for (int q = 0; q < kIpt; ++q) {
        cx += N[q] * X[q];
        cy += N[q] * Y[q];
      }
      cx = warp_sum(cx);
      cy = warp_sum(cy);
    }
    if (lane == 0) {
      wcm[wid * 2] = cx;
      wcm[wid * 2 + 1] = cy;
    }
    __syncthreads();
    // shares of destination k: row of k x nsplit source pieces
    const size_t row = (size_t)k * C.nsplit, rowk = (size_t)k * (k - 1) / 2 * C.nsplit;
    const size_t col = (size_t)src * C.nsplit + piece;
    for (int t = tid; t < 2 * S; t += blockDim.x) {
      const int cc = t >> 1, comp = t & 1;
      double v = 0.0;
      for (int w = 0; w < nw; ++w) v += wsum[((size_t)cc * nw + w) * 2 + comp];
      part[((rowk * S) + (size_t)cc * row + col) * 2 + comp] = v;
    }
    if (tid < 2) {
      double v = 0.0;
      for (int w = 0; w < nw; ++w) v += wcm[w * 2 + tid];
      ipart[(rowk + col) * 2 + tid] = v;
    }
    __syncthreads();
    kbprev = kb;
  }
}

__global__ void __launch_bounds__(kKickThreads) ws_kick(WsConst C, const int *__restrict__ bucket,
                                                       const int *__restrict__ npop,
                                                       const double *__restrict__ nelec, double *__restrict__ s,
                                                       const double *__restrict__ part,
                                                       const double *__restrict__ ipart,
                                                       const double *__restrict__ own, double *__restrict__ ion_out,
                                                       double *__restrict__ zcm_out) {
  const int k = blockIdx.x, S = C.S, tid = threadIdx.x;
  double *sl = s + (size_t)k * 6 * S;
  double *xp = sl + 3 * S, *zz = sl + 4 * S, *zp = sl + 5 * S;
  const size_t row = (size_t)k * C.nsplit, rowk = (size_t)k * (k - 1) / 2 * C.nsplit;
  if (C.fbii && k > 0 && tid < S) {
    const int c = tid;
    double sx = 0.0, sy = 0.0;
    for (size_t j = 0; j < row; ++j) {
      sx += part[((rowk * S) + (size_t)c * row + j) * 2];
      sy += part[((rowk * S) + (size_t)c * row + j) * 2 + 1];
    }
    const double dQ = nelec[k] * (double)npop[c] * kECharge;
    const double factjp = dQ > 0.0 ? C.factjp0 / dQ : 0.0;
    sx = factjp * sx;
    sy = factjp * sy;
    xp[c] = xp[c] + C.cdt * sx;
    zp[c] = zp[c] + C.cdt * sy;
  }
  if (tid == kKickThreads - 1 && ion_out) {
    double xs = 0.0, ys = 0.0, nt = 0.0;
    if (C.fbii) {
      for (size_t j = 0; j < row; ++j) {
        xs += ipart[(rowk + j) * 2];
        ys += ipart[(rowk + j) * 2 + 1];
      }
      xs += own[(size_t)k * 3 + 1];
      ys += own[(size_t)k * 3 + 2];
      for (int src = 0; src <= k; ++src) nt += own[(size_t)src * 3];
    }
    ion_out[(size_t)k * 2] = nt == 0.0 ? NAN : xs / nt;
    ion_out[(size_t)k * 2 + 1] = nt == 0.0 ? NAN : ys / nt;
  }
  if (tid == kKickThreads - 2 && zcm_out) {
    double z = 0.0;
    for (int c = 0; c < S; ++c) z = z + zz[c];
    zcm_out[bucket[k]] = z / (double)S;
  }
}

__global__ void ws_interp_points(WsConst C, const double *__restrict__ fx, const double *__restrict__ fy, int ib,
                                 int icell, const double *__restrict__ x, const double *__restrict__ y, int n,
                                 double *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double ex, ey;
  ws_interp(C, fx + (size_t)ib * C.nion, fy + (size_t)ib * C.nion, icell, x[i], y[i], ex, ey);
  out[2 * i] = ex;
  out[2 * i + 1] = ey;
}

thread_local char g_ws_err[512] = "";

}  // namespace

struct mbt_ws {
  mbt_ws_params w;
  WsConst C;
  long turn;
  int tpb;
  int *d_bucket, *d_npop, *d_nofe;
  double *d_nelec, *d_ibunch;
  double *d_s, *d_hist, *d_fx, *d_fy, *d_ion, *d_own, *d_part, *d_ipart;
  double *d_cm, *d_io, *d_zcm, *d_st;
  cudaStream_t stream;
  cudaEvent_t ev[5];
  double last_ms;   // device time of the last mbt_ws_run_turns
  char err[512];
};

static int ws_fail(mbt_ws *ws, int code, const char *fmt, ...) {
  char *dst = ws ? ws->err : g_ws_err;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(dst, 512, fmt, ap);
  va_end(ap);
  return code;
}

#define WS_CUDA(ws, call)                                                                         \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) return ws_fail((ws), MBT_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

// dynamic shared memory of the train: one field grid, the warps' kick and
// centroid shares; padded past half an SM's 228 KB when one block per SM is
// wanted
static size_t train_smem_bytes(int S, int nion, int tpb) {
  const size_t need = (2 * (size_t)nion + (size_t)S * (tpb / 32) * 2 + (tpb / 32) * 2) * sizeof(double);
  return MBT_WS_EXCLUSIVE && need < 116 * 1024 ? 116 * 1024 : need;
}

static void ws_free(mbt_ws *ws) {
  void *ptrs[] = {ws->d_bucket, ws->d_npop, ws->d_nofe, ws->d_nelec, ws->d_ibunch, ws->d_s, ws->d_hist,
                  ws->d_fx, ws->d_fy, ws->d_ion, ws->d_own, ws->d_part, ws->d_ipart, ws->d_cm,
                  ws->d_io, ws->d_zcm, ws->d_st};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  for (cudaEvent_t e : ws->ev)
    if (e) cudaEventDestroy(e);
  if (ws->stream) cudaStreamDestroy(ws->stream);
}

// Constants the reference computes on its host with libm, in its operand
// order (rw_weakstrong.c:97-128,210-229, fbi_weakstrong.c:155-156,
// 338-339,416, bunch.c:849).
static void ws_constants(const mbt_ws_params *w, int nb, WsConst *C) {
  const mbt_params *p = &w->base;
  memset(C, 0, sizeof(*C));
  C->nb = nb;
  C->S = 2 * w->nslc + 1;
  C->G = w->ngrid;
  C->off = (w->ngrid - 1) / 2;
  C->nion = C->S * C->G * C->G;
  C->nmt = p->Nmlt + 2;
  C->nharm = p->nharm;
  C->fbii = w->fbii;
  C->rw_long = p->rw_long;
  C->trigger_rw = p->triggerRW;
  C->Nmlt = p->Nmlt;
  for (int i = 0; i < 3; ++i) {
    C->track[i] = p->track_plane[i];
    C->alpha1[i] = p->alpha1[i];
    C->beta1[i] = p->beta1[i];
    C->gamma1[i] = p->gamma1[i];
  }
  C->nrev_mon = p->nrev_mon;
  C->vrf_e0 = p->Vrf0 / (p->E0 * kFKilo);
  C->wrf = p->wrf;
  C->phai0 = p->phai0;
  C->Urad = p->Urad;
  C->T0 = p->T0;
  C->ac = p->ac;
  {
    const double PsiV0 = 2.0 * M_PI * p->QV0 / 1.0, PsiH0 = 2.0 * M_PI * p->QH0 / 1.0;
    const double cV = cos(PsiV0), sV = sin(PsiV0), cH = cos(PsiH0), sH = sin(PsiH0);
    C->v11 = cV + p->alpha1[2] * sV;
    C->v12 = p->beta1[2] * sV;
    C->v21 = -p->gamma1[2] * sV;
    C->v22 = cV - p->alpha1[2] * sV;
    C->h11 = cH + p->alpha1[1] * sH;
    C->h12 = p->beta1[1] * sH;
    C->h21 = -p->gamma1[1] * sH;
    C->h22 = cH - p->alpha1[1] * sH;
  }
  {
    const double kappa = 1.0 / 2.8e-08;
    const double R = p->Lc / (2.0 * M_PI);
    for (int pl = 1; pl <= 2; ++pl) {
      const double Psi0 = 2.0 * M_PI * (pl == 1 ? p->QH0 : p->QV0) / 1.0;
      const double Psi = 0.0 + Psi0;
      const double cP = cos(Psi), sP = sin(Psi);
      const double beff3 = pow(pl == 1 ? p->beffH[0] : p->beffV[0], 3);
      const double beff3t = pow(2.0e-3, 3);
      C->a11[pl - 1] = cP + p->alpha1[pl] * sP;
      C->a12[pl - 1] = +p->beta1[pl] * sP;
      C->prfrw[pl - 1] = 2.0 * R / (beff3) / sqrt(M_PI * kappa * kEps0) / 1.0;
      C->prfrw_trig[pl - 1] = 2.0 * R / (beff3t) / sqrt(M_PI * kappa * kEps0) / 1.0;
    }
    C->fNp = (double)w->np;
    C->Pref0 = p->T0 / p->E0 / C->fNp / kFTera;
    C->Dub0 = p->Lc / (double)p->nharm;
    C->Lc = p->Lc;
  }
  C->factBE = w->factBE;
  C->sgm_xx = w->sgm_xx;
  C->sgm_zz = w->sgm_zz;
  C->agLOCx = w->agLOCx;
  C->agLOCz = w->agLOCz;
  C->agABSx = w->agABSx;
  C->agABSz = w->agABSz;
  C->rABSx = 1.0 / w->agABSx;
  C->rABSz = 1.0 / w->agABSz;
  C->deltT = w->deltT;
  C->factF = w->factF;
  C->Ldmsgm = w->Ldmsgm;
  C->fdq_den = 2 * kEps0 * sqrt(M_PI) * w->factBE * kCLight * w->deltT;
  C->factjp0 = w->kick_factor * 4.0 * M_PI * kEps0 * kERadius / w->Gamma;
  C->T0h = p->T0 / (double)p->nharm;
  C->cdt = kCLight * w->deltT;
}

extern "C" int mbt_ws_create(const mbt_ws_params *w, int nbunch, const int *bucket, const double *ibunch,
                             const int *npop, const int *nofe, mbt_ws **out) {
  if (!out) return ws_fail(nullptr, MBT_ERR_INVALID, "mbt_ws_create: null output pointer");
  *out = nullptr;
  if (!w || !bucket || !ibunch || !npop || !nofe || nbunch < 1)
    return ws_fail(nullptr, MBT_ERR_INVALID, "mbt_ws_create: null argument or no bunch");
  const int S = 2 * w->nslc + 1;
  if (S < 1 || S > kMaxSlices || w->ngrid < 1 || (w->ngrid & 1) == 0)
    return ws_fail(nullptr, MBT_ERR_INVALID, "mbt_ws_create: %d slices (1..%d), grid %d (odd)", S, kMaxSlices,
                   w->ngrid);
  if (w->base.Nmlt < 0 || w->base.Nmlt + 2 > kMaxHist)
    return ws_fail(nullptr, MBT_ERR_INVALID, "mbt_ws_create: Nmlt %d (0..%d)", w->base.Nmlt, kMaxHist - 2);
  if (w->np < 1 || w->base.nrev_mon < 1 || w->base.nharm < 1)
    return ws_fail(nullptr, MBT_ERR_INVALID, "mbt_ws_create: Np, NrevMon and h must be positive");
  for (int i = 0; i < nbunch; ++i)
    if (bucket[i] < 0 || bucket[i] >= w->base.nharm || (i > 0 && bucket[i] <= bucket[i - 1]))
      return ws_fail(nullptr, MBT_ERR_INVALID, "mbt_ws_create: buckets must ascend within 0..%d",
                     w->base.nharm - 1);
  const int nion = S * w->ngrid * w->ngrid;
  if (((nion + kIpt - 1) / kIpt + 31) / 32 * 32 > kTrainMaxThreads) return ws_fail(nullptr, MBT_ERR_INVALID, "mbt_ws_create: %d ions per bunch", nion);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return ws_fail(nullptr, MBT_ERR_NODEVICE, "mbt_ws_create: no CUDA device");
  mbt_ws *ws = (mbt_ws *)calloc(1, sizeof(mbt_ws));
  if (!ws) return ws_fail(nullptr, MBT_ERR_NOMEM, "mbt_ws_create: out of host memory");
  ws->w = *w;
  ws_constants(w, nbunch, &ws->C);
  ws->C.nsplit = nion > 512 ? MBT_WS_SPLIT : 1;
  ws->tpb = ((nion + kIpt * ws->C.nsplit - 1) / (kIpt * ws->C.nsplit) + 31) / 32 * 32;
  const WsConst &C = ws->C;
  const size_t nb = (size_t)nbunch, pairs = nb * (nb - 1) / 2;
  std::vector<double> nelec(nb);
  for (size_t i = 0; i < nb; ++i) nelec[i] = (ibunch[i] * w->base.T0 / (w->np * kECharge * kFKilo));
  int rc = 0;
#define WS_ALLOC(ptr, count)                                                                   \
  if (!rc && cudaMalloc(&(ptr), (count) * sizeof(*(ptr))) != cudaSuccess)                     \
    rc = ws_fail(nullptr, MBT_ERR_NOMEM, "mbt_ws_create: device allocation of %zu bytes failed", \
                 (size_t)((count) * sizeof(*(ptr))));
  WS_ALLOC(ws->d_bucket, nb);
  WS_ALLOC(ws->d_npop, (size_t)S);
  WS_ALLOC(ws->d_nofe, (size_t)nion);
  WS_ALLOC(ws->d_nelec, nb);
  WS_ALLOC(ws->d_ibunch, nb);
  WS_ALLOC(ws->d_s, nb * 6 * S);
  WS_ALLOC(ws->d_hist, nb * 4 * C.nmt);
  WS_ALLOC(ws->d_fx, nb * nion);
  WS_ALLOC(ws->d_fy, nb * nion);
  WS_ALLOC(ws->d_ion, nb * 5 * nion);
  WS_ALLOC(ws->d_own, nb * 3);
  WS_ALLOC(ws->d_part, (pairs > 0 ? pairs : 1) * C.nsplit * S * 2);
  WS_ALLOC(ws->d_ipart, (pairs > 0 ? pairs : 1) * C.nsplit * 2);
  WS_ALLOC(ws->d_cm, (size_t)kChunk * nb * 6);
  WS_ALLOC(ws->d_io, (size_t)kChunk * nb * 2);
  WS_ALLOC(ws->d_zcm, (size_t)kChunk * C.nharm);
  WS_ALLOC(ws->d_st, (size_t)kChunk * nb * 18);
#undef WS_ALLOC
  if (!rc && cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking) != cudaSuccess)
    rc = ws_fail(nullptr, MBT_ERR_CUDA, "mbt_ws_create: stream creation failed");
  for (int i = 0; i < 5 && !rc; ++i)
    if (cudaEventCreate(&ws->ev[i]) != cudaSuccess) rc = ws_fail(nullptr, MBT_ERR_CUDA, "mbt_ws_create: events");
  if (!rc) {
    const cudaStream_t st = ws->stream;
    bool ok = cudaMemcpyAsync(ws->d_bucket, bucket, nb * sizeof(int), cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(ws->d_npop, npop, S * sizeof(int), cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(ws->d_nofe, nofe, nion * sizeof(int), cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(ws->d_nelec, nelec.data(), nb * sizeof(double), cudaMemcpyHostToDevice, st) ==
                  cudaSuccess &&
              cudaMemcpyAsync(ws->d_ibunch, ibunch, nb * sizeof(double), cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemsetAsync(ws->d_s, 0, nb * 6 * S * sizeof(double), st) == cudaSuccess &&
              cudaMemsetAsync(ws->d_hist, 0, nb * 4 * C.nmt * sizeof(double), st) == cudaSuccess &&
              cudaMemsetAsync(ws->d_fx, 0, nb * nion * sizeof(double), st) == cudaSuccess &&
              cudaMemsetAsync(ws->d_fy, 0, nb * nion * sizeof(double), st) == cudaSuccess &&
              cudaMemsetAsync(ws->d_ion, 0, nb * 5 * nion * sizeof(double), st) == cudaSuccess &&
              cudaMemsetAsync(ws->d_own, 0, nb * 3 * sizeof(double), st) == cudaSuccess &&
              cudaStreamSynchronize(st) == cudaSuccess;
    if (!ok) rc = ws_fail(nullptr, MBT_ERR_CUDA, "mbt_ws_create: upload failed: %s", cudaGetErrorString(cudaGetLastError()));
  }
  if (!rc) {
    const size_t train_smem = train_smem_bytes(S, nion, ws->tpb);
    const size_t bunch_smem = 2 * (size_t)nion * sizeof(double);
    if (train_smem > 48 * 1024 &&
        cudaFuncSetAttribute(ws_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_smem) != cudaSuccess)
      rc = ws_fail(nullptr, MBT_ERR_CUDA, "mbt_ws_create: train shared memory %zu bytes", train_smem);
    if (!rc && bunch_smem > 48 * 1024 &&
        cudaFuncSetAttribute(ws_bunch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bunch_smem) != cudaSuccess)
      rc = ws_fail(nullptr, MBT_ERR_CUDA, "mbt_ws_create: bunch shared memory %zu bytes", bunch_smem);
    if (!rc && nb * sizeof(double) > 48 * 1024 &&
        cudaFuncSetAttribute(ws_optic_rw, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(nb * sizeof(double))) != cudaSuccess)
      rc = ws_fail(nullptr, MBT_ERR_CUDA, "mbt_ws_create: %zu bunches", nb);
  }
  if (rc) {
    ws_free(ws);
    free(ws);
    return rc;
  }
  *out = ws;
  return 0;
}

extern "C" int mbt_ws_load_slices(mbt_ws *ws, const double *slices) {
  if (!ws || !slices) return ws_fail(ws, MBT_ERR_INVALID, "mbt_ws_load_slices: null argument");
  WS_CUDA(ws, cudaMemcpyAsync(ws->d_s, slices, (size_t)ws->C.nb * 6 * ws->C.S * sizeof(double),
                              cudaMemcpyHostToDevice, ws->stream));
  WS_CUDA(ws, cudaStreamSynchronize(ws->stream));
  return 0;
}

extern "C" int mbt_ws_get_slices(mbt_ws *ws, double *slices) {
  if (!ws || !slices) return ws_fail(ws, MBT_ERR_INVALID, "mbt_ws_get_slices: null argument");
  WS_CUDA(ws, cudaMemcpyAsync(slices, ws->d_s, (size_t)ws->C.nb * 6 * ws->C.S * sizeof(double),
                              cudaMemcpyDeviceToHost, ws->stream));
  WS_CUDA(ws, cudaStreamSynchronize(ws->stream));
  return 0;
}

extern "C" int mbt_ws_run_turns(mbt_ws *ws, long nturns, double *cm, double *ion, double *zcm, double *stats) {
  if (!ws || nturns < 0) return ws_fail(ws, MBT_ERR_INVALID, "mbt_ws_run_turns: null context or negative turns");
  const WsConst &C = ws->C;
  const cudaStream_t st = ws->stream;
  const size_t nb = (size_t)C.nb, S = (size_t)C.S, n = (size_t)C.nion;
  const size_t bunch_smem = 2 * n * sizeof(double);
  const size_t train_smem = train_smem_bytes((int)S, (int)n, ws->tpb);
  long imon_total = 0;
  ws->last_ms = 0.0;
  for (long t0 = 0; t0 < nturns; t0 += kChunk) {
    const long nt = nturns - t0 < kChunk ? nturns - t0 : kChunk;
    long imon = 0;
    if (zcm) WS_CUDA(ws, cudaMemsetAsync(ws->d_zcm, 0, (size_t)nt * C.nharm * sizeof(double), st));
    WS_CUDA(ws, cudaEventRecord(ws->ev[0], st));
    for (long t = 0; t < nt; ++t) {
      const long rev = ws->turn;
      const bool mon = rev % C.nrev_mon == 0;
      ws_bunch<<<C.nb, kBunchThreads, bunch_smem, st>>>(C, ws->d_s, ws->d_hist, ws->d_npop, ws->d_nofe, ws->d_nelec,
                                                        ws->d_fx, ws->d_fy, ws->d_ion, ws->d_own,
                                                        cm ? ws->d_cm + (size_t)t * nb * 6 : nullptr,
                                                        (mon && stats) ? ws->d_st + (size_t)imon * nb * 18 : nullptr);
      ws_optic_rw<<<C.nb, kRwThreads, nb * sizeof(double), st>>>(C, ws->d_s, ws->d_hist, ws->d_ibunch,
                                                                  ws->d_bucket, rev);
      if (C.fbii && C.nb > 1)
        ws_train<<<C.nb * C.nsplit, ws->tpb, train_smem, st>>>(C, ws->d_bucket, ws->d_fx, ws->d_fy, ws->d_ion,
                                                               ws->d_part, ws->d_ipart);
      ws_kick<<<C.nb, kKickThreads, 0, st>>>(C, ws->d_bucket, ws->d_npop, ws->d_nelec, ws->d_s, ws->d_part,
                                             ws->d_ipart, ws->d_own, ion ? ws->d_io + (size_t)t * nb * 2 : nullptr,
                                             zcm ? ws->d_zcm + (size_t)t * C.nharm : nullptr);
      WS_CUDA(ws, cudaGetLastError());
      if (mon) ++imon;
      ++ws->turn;
    }
    WS_CUDA(ws, cudaEventRecord(ws->ev[1], st));
    if (cm)
      WS_CUDA(ws, cudaMemcpyAsync(cm + (size_t)t0 * nb * 6, ws->d_cm, (size_t)nt * nb * 6 * sizeof(double),
                                  cudaMemcpyDeviceToHost, st));
    if (ion)
      WS_CUDA(ws, cudaMemcpyAsync(ion + (size_t)t0 * nb * 2, ws->d_io, (size_t)nt * nb * 2 * sizeof(double),
                                  cudaMemcpyDeviceToHost, st));
    if (zcm)
      WS_CUDA(ws, cudaMemcpyAsync(zcm + (size_t)t0 * C.nharm, ws->d_zcm, (size_t)nt * C.nharm * sizeof(double),
                                  cudaMemcpyDeviceToHost, st));
    if (stats && imon > 0)
      WS_CUDA(ws, cudaMemcpyAsync(stats + (size_t)imon_total * nb * 18, ws->d_st,
                                  (size_t)imon * nb * 18 * sizeof(double), cudaMemcpyDeviceToHost, st));
    WS_CUDA(ws, cudaStreamSynchronize(st));
    float ms = 0.0f;
    WS_CUDA(ws, cudaEventElapsedTime(&ms, ws->ev[0], ws->ev[1]));
    ws->last_ms += ms;
    imon_total += imon;
  }
  return 0;
}

extern "C" double mbt_ws_last_ms(const mbt_ws *ws) { return ws ? ws->last_ms : -1.0; }

extern "C" int mbt_ws_profile(mbt_ws *ws, long nturns, double *ms4) {
  if (!ws || nturns < 1 || !ms4) return ws_fail(ws, MBT_ERR_INVALID, "mbt_ws_profile: bad argument");
  const WsConst &C = ws->C;
  const cudaStream_t st = ws->stream;
  const size_t nb = (size_t)C.nb, S = (size_t)C.S, n = (size_t)C.nion;
  const size_t bunch_smem = 2 * n * sizeof(double);
  const size_t train_smem = train_smem_bytes((int)S, (int)n, ws->tpb);
  double acc[4] = {0, 0, 0, 0};
  for (long t = 0; t < nturns; ++t) {
    const long rev = ws->turn;
    WS_CUDA(ws, cudaEventRecord(ws->ev[0], st));
    ws_bunch<<<C.nb, kBunchThreads, bunch_smem, st>>>(C, ws->d_s, ws->d_hist, ws->d_npop, ws->d_nofe, ws->d_nelec,
                                                      ws->d_fx, ws->d_fy, ws->d_ion, ws->d_own, nullptr, nullptr);
    WS_CUDA(ws, cudaEventRecord(ws->ev[1], st));
    ws_optic_rw<<<C.nb, kRwThreads, nb * sizeof(double), st>>>(C, ws->d_s, ws->d_hist, ws->d_ibunch, ws->d_bucket,
                                                                rev);
    WS_CUDA(ws, cudaEventRecord(ws->ev[2], st));
    if (C.fbii && C.nb > 1)
      ws_train<<<C.nb * C.nsplit, ws->tpb, train_smem, st>>>(C, ws->d_bucket, ws->d_fx, ws->d_fy, ws->d_ion,
                                                             ws->d_part, ws->d_ipart);
    WS_CUDA(ws, cudaEventRecord(ws->ev[3], st));
    ws_kick<<<C.nb, kKickThreads, 0, st>>>(C, ws->d_bucket, ws->d_npop, ws->d_nelec, ws->d_s, ws->d_part,
                                           ws->d_ipart, ws->d_own, nullptr, nullptr);
    WS_CUDA(ws, cudaEventRecord(ws->ev[4], st));
    WS_CUDA(ws, cudaGetLastError());
    WS_CUDA(ws, cudaEventSynchronize(ws->ev[4]));
    for (int k = 0; k < 4; ++k) {
      float ms = 0.0f;
      WS_CUDA(ws, cudaEventElapsedTime(&ms, ws->ev[k], ws->ev[k + 1]));
      acc[k] += ms;
    }
    ++ws->turn;
  }
  for (int k = 0; k < 4; ++k) ms4[k] = acc[k] / (double)nturns;
  return 0;
}

extern "C" int mbt_ws_interp(mbt_ws *ws, int ib, int icell, const double *x, const double *y, int n, double *exey) {
  if (!ws || ib < 0 || ib >= ws->C.nb || icell < 0 || icell >= ws->C.S || n < 0 || (n > 0 && (!x || !y || !exey)))
    return ws_fail(ws, MBT_ERR_INVALID, "mbt_ws_interp: bunch %d slice %d, %d points", ib, icell, n);
  if (n == 0) return 0;
  double *d = nullptr;
  WS_CUDA(ws, cudaMalloc(&d, (size_t)n * 4 * sizeof(double)));
  cudaError_t e = cudaMemcpyAsync(d, x, n * sizeof(double), cudaMemcpyHostToDevice, ws->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d + n, y, n * sizeof(double), cudaMemcpyHostToDevice, ws->stream);
  if (e == cudaSuccess) {
    ws_interp_points<<<(n + 255) / 256, 256, 0, ws->stream>>>(ws->C, ws->d_fx, ws->d_fy, ib, icell, d, d + n, n,
                                                              d + 2 * n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(exey, d + 2 * n, 2 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, ws->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ws->stream);
  cudaFree(d);
  if (e != cudaSuccess) return ws_fail(ws, MBT_ERR_CUDA, "mbt_ws_interp: %s", cudaGetErrorString(e));
  return 0;
}

extern "C" int mbt_ws_bunch_fields(mbt_ws *ws, int ib, double *exey, double *ions5) {
  if (!ws || ib < 0 || ib >= ws->C.nb) return ws_fail(ws, MBT_ERR_INVALID, "mbt_ws_bunch_fields: bunch %d", ib);
  const size_t n = (size_t)ws->C.nion;
  if (exey) {
    std::vector<double> ex(n), ey(n);
    WS_CUDA(ws, cudaMemcpyAsync(ex.data(), ws->d_fx + ib * n, n * sizeof(double), cudaMemcpyDeviceToHost, ws->stream));
    WS_CUDA(ws, cudaMemcpyAsync(ey.data(), ws->d_fy + ib * n, n * sizeof(double), cudaMemcpyDeviceToHost, ws->stream));
    WS_CUDA(ws, cudaStreamSynchronize(ws->stream));
    for (size_t i = 0; i < n; ++i) {
      exey[2 * i] = ex[i];
      exey[2 * i + 1] = ey[i];
    }
  }
  if (ions5) {
    WS_CUDA(ws, cudaMemcpyAsync(ions5, ws->d_ion + ib * 5 * n, 5 * n * sizeof(double), cudaMemcpyDeviceToHost,
                                ws->stream));
    WS_CUDA(ws, cudaStreamSynchronize(ws->stream));
  }
  return 0;
}

extern "C" long mbt_ws_turn(const mbt_ws *ws) { return ws ? ws->turn : -1; }

extern "C" const char *mbt_ws_last_error(const mbt_ws *ws) { return ws ? ws->err : g_ws_err; }

extern "C" void mbt_ws_destroy(mbt_ws *ws) {
  if (!ws) return;
  if (ws->stream) cudaStreamSynchronize(ws->stream);
  ws_free(ws);
  free(ws);
}

// ---- checkpoint / resume: the slices, the centroid histories and the
// turn count carry one turn into the next (field grids, ions and kick
// shares are rebuilt every turn).  Layout: "MBTWSCK1", turn, bunches,
// slices, history length, the two arrays, 64-bit FNV-1a of all before it.

static uint64_t ws_fnv1a(uint64_t h, const void *p, size_t n) {
  const unsigned char *b = static_cast<const unsigned char *>(p);
  for (size_t i = 0; i < n; ++i) {
    h ^= b[i];
    h *= 1099511628211ull;
  }
  return h;
}

extern "C" int mbt_ws_checkpoint_save(mbt_ws *ws, const char *path) {
  if (!ws || !path) return ws_fail(ws, MBT_ERR_INVALID, "mbt_ws_checkpoint_save: null argument");
  const WsConst &C = ws->C;
  const size_t ns = (size_t)C.nb * 6 * C.S, nh = (size_t)C.nb * 4 * C.nmt;
  const int64_t head[5] = {(int64_t)ws->turn, C.nb, C.S, C.nmt, C.nion};
  std::vector<char> data(8 + sizeof head + (ns + nh) * sizeof(double) + sizeof(uint64_t));
  memcpy(data.data(), "MBTWSCK1", 8);
  memcpy(data.data() + 8, head, sizeof head);
  double *arr = reinterpret_cast<double *>(data.data() + 8 + sizeof head);
  WS_CUDA(ws, cudaStreamSynchronize(ws->stream));
  WS_CUDA(ws, cudaMemcpy(arr, ws->d_s, ns * sizeof(double), cudaMemcpyDeviceToHost));
  WS_CUDA(ws, cudaMemcpy(arr + ns, ws->d_hist, nh * sizeof(double), cudaMemcpyDeviceToHost));
  const size_t body = data.size() - sizeof(uint64_t);
  const uint64_t sum = ws_fnv1a(1469598103934665603ull, data.data(), body);
  memcpy(data.data() + body, &sum, sizeof sum);
  const std::string tmp = std::string(path) + ".tmp";
  FILE *f = fopen(tmp.c_str(), "wb");
  if (!f) return ws_fail(ws, MBT_ERR_IO, "mbt_ws_checkpoint_save: cannot create %s", tmp.c_str());
  const bool ok = fwrite(data.data(), 1, data.size(), f) == data.size();
  if (fclose(f) != 0 || !ok || rename(tmp.c_str(), path) != 0) {
    remove(tmp.c_str());
    return ws_fail(ws, MBT_ERR_IO, "mbt_ws_checkpoint_save: cannot write %s", path);
  }
  return 0;
}

extern "C" int mbt_ws_checkpoint_load(mbt_ws *ws, const char *path) {
  if (!ws || !path) return ws_fail(ws, MBT_ERR_INVALID, "mbt_ws_checkpoint_load: null argument");
  const WsConst &C = ws->C;
  const size_t ns = (size_t)C.nb * 6 * C.S, nh = (size_t)C.nb * 4 * C.nmt;
  int64_t head[5];
  const size_t want = 8 + sizeof head + (ns + nh) * sizeof(double) + sizeof(uint64_t);
  FILE *f = fopen(path, "rb");
  if (!f) return ws_fail(ws, MBT_ERR_IO, "mbt_ws_checkpoint_load: cannot open %s", path);
  std::vector<char> data(want + 1);
  const size_t got = fread(data.data(), 1, data.size(), f);
  fclose(f);
  if (got != want || memcmp(data.data(), "MBTWSCK1", 8) != 0)
    return ws_fail(ws, MBT_ERR_IO, "mbt_ws_checkpoint_load: %s is not a slice-model checkpoint of this size", path);
  uint64_t sum;
  memcpy(&sum, data.data() + want - sizeof sum, sizeof sum);
  if (ws_fnv1a(1469598103934665603ull, data.data(), want - sizeof sum) != sum)
    return ws_fail(ws, MBT_ERR_IO, "mbt_ws_checkpoint_load: %s: checksum mismatch", path);
  memcpy(head, data.data() + 8, sizeof head);
  if (head[1] != C.nb || head[2] != C.S || head[3] != C.nmt || head[4] != C.nion || head[0] < 0)
    return ws_fail(ws, MBT_ERR_STATE, "mbt_ws_checkpoint_load: %s was written by another configuration", path);
  const double *arr = reinterpret_cast<const double *>(data.data() + 8 + sizeof head);
  WS_CUDA(ws, cudaStreamSynchronize(ws->stream));
  WS_CUDA(ws, cudaMemcpy(ws->d_s, arr, ns * sizeof(double), cudaMemcpyHostToDevice));
  WS_CUDA(ws, cudaMemcpy(ws->d_hist, arr + ns, nh * sizeof(double), cudaMemcpyHostToDevice));
  ws->turn = (long)head[0];
  return 0;
}
