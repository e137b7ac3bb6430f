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
//   bi_kick_grouped  one block per tile: every electron kicked by the
//              clouds of its bunch at every point, kicks mapped back to the
//              kick point.
// bi_ions and bi_kick_grouped sort their field evaluations by the branch of
// w(z) they take before evaluating them (gauss_field_key), so that a warp
// runs one branch at a time.
// With the learned field, bi_ions_mlp and bi_kick_mlp replace bi_ions and
// bi_kick_grouped: persistent CTAs of four 128-thread groups that share the
// network's weights; a group evaluates the field for its 128 ions (or
// electrons) at once on the tensor cores, falls back to the Faddeeva field
// outside the network's domain, and re-evaluates a hashed sample with it
// for the audit.
#pragma once
#include <cstdint>

#include "mbt_common.cuh"
#include "mbt_device.cuh"
#include "mbt_gauss.cuh"
#include "mbt_mlp.cuh"
#include "mbt_philox.cuh"

namespace mbt {

constexpr int kBiThreads = 256;
constexpr int kBiMaxIp = 64;
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
  int *error;                      // the ring's sticky error word: bit 4 = a tensor-core wait gave up
  // learned field (surrogate runs)
  uint32_t audit_threshold;        // audit an evaluation when its hash is below this (2^32 x fraction)
  unsigned long long *audit;       // [0] audited evaluations, [1] max relative error (bits), [2] fallbacks,
                                   // [3] tensor-core failures; double sum of squared errors at audit + 4
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

// ---- region-grouped evaluation of the Faddeeva field

// TOMS 680 branch of w(z) at x, y >= 0 (wofz_dev): 0 power series, 1
// Taylor series with continued-fraction derivatives, 2 Laplace continued
// fraction.
__device__ __forceinline__ int wofz_branch(double x, double y) {
  const double xs = x / 6.3, ys = y / 4.4;
  const double q = xs * xs + ys * ys;
  return q < 0.085264 ? 0 : (q > 1.0 ? 2 : 1);
}
constexpr int kFieldKeys = 13;
// Key of gauss_field(dx, dy, sx, sy) by the branches its evaluation takes:
// 4 x (branch of w(z1)) + (branch of w(z2), or 3 when the second term is
// skipped); 12 for the near-round quadrature.
__device__ __forceinline__ int gauss_field_key(double dx, double dy, double sx, double sy) {
  double ax = fabs(dx), ay = fabs(dy);
  if (sy > sx) {
    const double t = ax; ax = ay; ay = t;
    const double u = sx; sx = sy; sy = u;
  }
  sy = fmax(sy, 1e-6 * sx);
  const double r = sy / sx;
  if (r > kBiRoundRatio) return 12;
  const double fbe = sqrt(2.0 * (sx * sx - sy * sy));
  const double x1 = ax / fbe, y1 = ay / fbe;
  const double arg = ax * ax / (2.0 * sx * sx) + ay * ay / (2.0 * sy * sy);
  return 4 * wofz_branch(x1, y1) + (arg > 50.0 ? 3 : wofz_branch(x1 * r, y1 / r));
}

// One thread per macro-ion; at every later passage the block's field
// evaluations are sorted by the TOMS 680 branches they take (a counting sort
// in shared memory, as bi_kick_grouped) so that the warps evaluate runs of
// one branch, and each ion reads its field back.
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
  __shared__ int cnt[kFieldKeys], base[kFieldKeys], total;
  __shared__ double fin[2 * kBiThreads], fout[2 * kBiThreads];
  __shared__ int ev_of[kBiThreads];
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
    if (threadIdx.x < kFieldKeys) cnt[threadIdx.x] = 0;
    __syncthreads();
    if (threadIdx.x < 5) {
      double t = 0.0;
      for (int q = 0; q < kBiThreads / 32; ++q) t += red[q][threadIdx.x];
      bi.part[(((size_t)k * bi.T + bi_tri(b) + b0) * bi.bpp + blk) * 5 + threadIdx.x] = t;
    }
    int v = -1;
    if (live) {
      const int key = gauss_field_key(dx, dy, F[2], F[3]);
      v = (key << 16) | atomicAdd(&cnt[key], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int sum = 0;
      for (int q = 0; q < kFieldKeys; ++q) {
        base[q] = sum;
        sum += cnt[q];
      }
      total = sum;
    }
    __syncthreads();
    if (v >= 0) {
      const int sl = base[v >> 16] + (v & 0xFFFF);
      fin[2 * sl] = dx;
      fin[2 * sl + 1] = dy;
      ev_of[sl] = threadIdx.x;
    }
    __syncthreads();
    if (threadIdx.x < total) {
      const int e = ev_of[threadIdx.x];
      double gx, gy;
      gauss_field(fin[2 * threadIdx.x], fin[2 * threadIdx.x + 1], F[2], F[3], gx, gy);
      fout[2 * e] = gx;
      fout[2 * e + 1] = gy;
    }
    __syncthreads();
    if (live) {
      const double kk = bi.kion_per_amp * bi.ib[b];
      vx = vx + kk * fout[2 * threadIdx.x];
      vy = vy + kk * fout[2 * threadIdx.x + 1];
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

constexpr int kKickChunk = 64;   // electrons per pass of bi_kick_grouped
// shared memory of bi_kick_grouped for n_ip points
__host__ __device__ constexpr size_t bi_kick_grouped_smem(int n_ip) {
  return (size_t)kKickChunk * n_ip * (4 * sizeof(double) + 2 * sizeof(int));
}

// Every electron of a tile: the deflection by each cloud its bunch meets,
// at that point's coordinates, mapped back to the kick point
// (x += -beta s theta, x' += (c + alpha s) theta).  The field evaluations
// of 64 electrons at all points are gathered first and sorted by the
// TOMS 680 branches they take (a counting sort in shared memory), so that
// the warps evaluate runs of one branch; the kicks are then summed per
// electron over the points in order.
__global__ void __launch_bounds__(kBiThreads) bi_kick_grouped(Args a, BiArgs bi) {
  const Tile tile = a.tiles[blockIdx.x];
  const int b = tile.bunch;
  __shared__ double cl[kBiMaxIp][5];
  __shared__ double tr[kBiMaxIp][4];   // mx, sxb, my, syb of the point
  __shared__ int cnt[kFieldKeys], base[kFieldKeys];
  extern __shared__ double dsm[];
  const int nk = bi.n_ip, ne = kKickChunk * nk;
  double *buf = dsm;                                      // ne x 2 by evaluation: offsets, then fields
  double *in = dsm + 2 * ne;                              // ne x 2 by slot: offsets
  int *key_rank = reinterpret_cast<int *>(dsm + 4 * ne);  // ne by evaluation: key << 16 | rank, -1 none
  int *ev_of = key_rank + ne;                             // ne by slot: its evaluation
  for (int i = threadIdx.x; i < nk; i += kBiThreads) {
    const double *Cl = bi.cloud + ((size_t)i * bi.nb + b) * 5;
    cl[i][0] = bi.ke * Cl[0];
    for (int m = 1; m < 5; ++m) cl[i][m] = Cl[m];
    const double *T = bi.trig + 4 * i;
    tr[i][0] = T[0] + bi.alphaH * T[1];
    tr[i][1] = bi.betaH * T[1];
    tr[i][2] = T[2] + bi.alphaV * T[3];
    tr[i][3] = bi.betaV * T[3];
  }
  const size_t n6 = (size_t)a.npad;
  double *C = a.coord;
  for (int c0 = 0; c0 < tile.count; c0 += kKickChunk) {
    const int nchunk = min(kKickChunk, tile.count - c0);
    if (threadIdx.x < kFieldKeys) cnt[threadIdx.x] = 0;
    __syncthreads();
    // offsets and key of every evaluation e = k kKickChunk + i (point k,
    // electron i of the chunk); the rank within a key comes from shared
    // atomics (slot order varies between runs, the results do not)
    for (int e = threadIdx.x; e < ne; e += kBiThreads) {
      const int k = e / kKickChunk, i = e % kKickChunk;
      int v = -1;
      if (i < nchunk && cl[k][0] != 0.0) {
        const int p = tile.start + c0 + i;
        const double x = C[1 * n6 + p], z = C[2 * n6 + p], xp = C[4 * n6 + p], zp = C[5 * n6 + p];
        const double xk = tr[k][0] * x + tr[k][1] * xp, zk = tr[k][2] * z + tr[k][3] * zp;
        const double dx = xk - cl[k][1], dy = zk - cl[k][2];
        buf[2 * e] = dx;
        buf[2 * e + 1] = dy;
        const int key = gauss_field_key(dx, dy, cl[k][3], cl[k][4]);
        v = (key << 16) | atomicAdd(&cnt[key], 1);
      }
      key_rank[e] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int sum = 0;
      for (int q = 0; q < kFieldKeys; ++q) {
        base[q] = sum;
        sum += cnt[q];
      }
      cnt[0] = sum;
    }
    __syncthreads();
    const int total = cnt[0];
    for (int e = threadIdx.x; e < ne; e += kBiThreads) {
      const int v = key_rank[e];
      if (v >= 0) {
        const int sl = base[v >> 16] + (v & 0xFFFF);
        in[2 * sl] = buf[2 * e];
        in[2 * sl + 1] = buf[2 * e + 1];
        ev_of[sl] = e;
      }
    }
    __syncthreads();
    // the evaluations in slot order: consecutive slots share a key
    for (int sl = threadIdx.x; sl < total; sl += kBiThreads) {
      const int e = ev_of[sl], k = e / kKickChunk;
      double gx, gy;
      gauss_field(in[2 * sl], in[2 * sl + 1], cl[k][3], cl[k][4], gx, gy);
      buf[2 * e] = gx;
      buf[2 * e + 1] = gy;
    }
    __syncthreads();
    // the kicks of each electron, summed over the points in order
    if (threadIdx.x < nchunk) {
      const int i = threadIdx.x, p = tile.start + c0 + i;
      const double x = C[1 * n6 + p], z = C[2 * n6 + p], xp = C[4 * n6 + p], zp = C[5 * n6 + p];
      double ddx = 0.0, ddxp = 0.0, ddz = 0.0, ddzp = 0.0;
      for (int k = 0; k < nk; ++k) {
        if (cl[k][0] == 0.0) continue;
        const int e = k * kKickChunk + i;
        const double thx = cl[k][0] * buf[2 * e], thy = cl[k][0] * buf[2 * e + 1];
        ddx = ddx - tr[k][1] * thx;
        ddxp = ddxp + tr[k][0] * thx;
        ddz = ddz - tr[k][3] * thy;
        ddzp = ddzp + tr[k][2] * thy;
      }
      C[1 * n6 + p] = x + ddx;
      C[4 * n6 + p] = xp + ddxp;
      C[2 * n6 + p] = z + ddz;
      C[5 * n6 + p] = zp + ddzp;
    }
    __syncthreads();
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

// ---------------------------------------------------------------- learned field

// Deterministic audit selection; the kernels hash a whole warp's
// evaluations together (32 consecutive ions or particles), so an audited
// warp evaluates the Faddeeva field in all its lanes at once.
__device__ __forceinline__ uint32_t bi_hash(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u) * 0x85EBCA77u ^ (c + 0x165667B1u) * 0xC2B2AE3Du;
  h ^= h >> 15;
  h *= 0x2C1B3C6Du;
  h ^= h >> 12;
  h *= 0x297A2D39u;
  h ^= h >> 15;
  return h;
}

// The Faddeeva field out of line, for the rare fallbacks and audits of the
// learned-field kernels (keeps their register budget for the network);
// returned by value, so that no caller variable has its address taken.
__device__ __noinline__ double2 gauss_field_ool(double dx, double dy, double sx, double sy) {
  double2 g;
  gauss_field(dx, dy, sx, sy, g.x, g.y);
  return g;
}

// The Faddeeva fallbacks of a group, evaluated with the group's lanes
// packed: every thread whose point lies outside the network's domain
// appends (dx, dy, sx, sy) to a list in the group's activation tile (free
// once the network has run), thread t evaluates entry t, and each thread
// reads its own result back.  Spread over the warps, a few such points
// would otherwise make every warp run the Faddeeva branch.
__device__ __forceinline__ void bi_group_fallbacks(MlpGroup &G, int t, bool need, double dx, double dy, double sx,
                                                   double sy, double &gx, double &gy, int &fallbacks) {
  const int warp = t >> 5, lane = t & 31;
  const unsigned ball = __ballot_sync(0xffffffffu, need);
  int *cnt = reinterpret_cast<int *>(G.A);
  double *in = reinterpret_cast<double *>(G.A + 128);          // 128 x 4
  double *out = in + 4 * 128;                                   // 128 x 2
  if (lane == 0) cnt[warp] = __popc(ball);
  named_barrier(G.bar_id, 128);
  int base = 0, total = 0;
#pragma unroll
  for (int w = 0; w < 4; ++w) {
    base += w < warp ? cnt[w] : 0;
    total += cnt[w];
  }
  const int idx = base + __popc(ball & ((1u << lane) - 1u));
  if (need) {
    in[4 * idx] = dx;
    in[4 * idx + 1] = dy;
    in[4 * idx + 2] = sx;
    in[4 * idx + 3] = sy;
  }
  named_barrier(G.bar_id, 128);
  if (t < total) {
    const double2 f = gauss_field_ool(in[4 * t], in[4 * t + 1], in[4 * t + 2], in[4 * t + 3]);
    out[2 * t] = f.x;
    out[2 * t + 1] = f.y;
  }
  named_barrier(G.bar_id, 128);
  if (need) {
    gx = out[2 * idx];
    gy = out[2 * idx + 1];
    ++fallbacks;
  }
  named_barrier(G.bar_id, 128);   // every result read before the tile is written again
}

// The learned field with its fallback and audit, for one group; `side`
// is work interleaved with the network (mlp_group_eval).
template <typename Side = NoSideWork>
__device__ __forceinline__ bool bi_field_mlp(const BiArgs &bi, MlpGroup &G, int t, bool active, double dx, double dy,
                                             double sx, double sy, uint32_t h, double &gx, double &gy,
                                             double &aud_max, double &aud_sq, int &aud_n, int &fallbacks,
                                             const Side &side = Side()) {
  bool in_domain, any_out;
  if (!mlp_group_field(G, t, active, dx, dy, sx, sy, gx, gy, in_domain, any_out, side)) return false;
  if (any_out) bi_group_fallbacks(G, t, active && !in_domain, dx, dy, sx, sy, gx, gy, fallbacks);
  if (active && in_domain && h < bi.audit_threshold) {
    // relative error of the field vector: |F_net - F| / |F|
    const double2 fe = gauss_field_ool(dx, dy, sx, sy);
    const double ex = fe.x, ey = fe.y;
    const double f = hypot(ex, ey);
    const double e = f > 0.0 ? hypot(gx - ex, gy - ey) / f : 0.0;
    aud_max = fmax(aud_max, e);
    aud_sq += e * e;
    ++aud_n;
  }
  return true;
}

__device__ __forceinline__ void bi_audit_flush(const BiArgs &bi, double aud_max, double aud_sq, int aud_n,
                                               int fallbacks) {
  const double m = warp_max(aud_max), q = warp_sum(aud_sq);
  const int n = warp_sum(aud_n), f = warp_sum(fallbacks);
  if ((threadIdx.x & 31) == 0) {
    if (n) {
      atomicAdd(&bi.audit[0], (unsigned long long)n);
      atomicMax(&bi.audit[1], (unsigned long long)__double_as_longlong(m));
      atomicAdd(reinterpret_cast<double *>(bi.audit + 4), q);
    }
    if (f) atomicAdd(&bi.audit[2], (unsigned long long)f);
  }
}

// Ions with the learned field: work item = (creating passage b0, point k,
// 128-ion block), longest first; every group takes items round-robin.
__global__ void __launch_bounds__(128 * kMlpGroups, 1) bi_ions_mlp(BiArgs bi, MlpDev M) {
  extern __shared__ uint8_t smem_raw[];
  MlpGroup G;
  const uint32_t tmem = mlp_cta_setup(M, align1024(smem_raw), G);
  const int g = threadIdx.x >> 7, t = threadIdx.x & 127, warp = t >> 5, lane = threadIdx.x & 31;
  __shared__ double red[kMlpGroups][4][5];
  const long turn = *bi.turn;
  const long per_b0 = (long)bi.n_ip * bi.bpp, nitems = (long)(bi.nb - 1) * per_b0;
  double aud_max = 0.0, aud_sq = 0.0;
  int aud_n = 0, fallbacks = 0;
  bool ok = true;
  for (long item = (long)blockIdx.x * kMlpGroups + g; item < nitems && ok; item += (long)gridDim.x * kMlpGroups) {
    const int b0 = (int)(item / per_b0);
    const int k = (int)((item % per_b0) / bi.bpp), blk = (int)(item % bi.bpp);
    const int j = blk * 128 + t;
    const bool live = j < bi.n_new;
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
        for (int m = 0; m < 5; ++m) red[g][warp][m] = s[m];
      named_barrier(G.bar_id, 128);
      if (t < 5)
        bi.part[(((size_t)k * bi.T + bi_tri(b) + b0) * bi.bpp + blk) * 5 + t] =
            ((red[g][0][t] + red[g][1][t]) + red[g][2][t]) + red[g][3][t];
      double gx = 0.0, gy = 0.0;
      if (!bi_field_mlp(bi, G, t, live, dx, dy, F[2], F[3], bi_hash((uint32_t)turn, (uint32_t)(k * 65536 + b), (uint32_t)(b0 * 1048576 + (j >> 5))),
                        gx, gy, aud_max, aud_sq, aud_n, fallbacks)) {
        ok = false;
        break;
      }
      if (live) {
        const double kk = bi.kion_per_amp * bi.ib[b];
        vx = vx + kk * gx;
        vy = vy + kk * gy;
      }
    }
  }
  bi_audit_flush(bi, aud_max, aud_sq, aud_n, fallbacks);
  if ((mlp_cta_release(tmem, G) || !ok) && t == 0) {
    atomicAdd(&bi.audit[3], 1ull);
    atomicOr(bi.error, 4);
  }
}

// Electrons with the learned field: work item = 128 particles of a tile.
__global__ void __launch_bounds__(128 * kMlpGroups, 1) bi_kick_mlp(Args a, BiArgs bi, MlpDev M) {
  extern __shared__ uint8_t smem_raw[];
  MlpGroup G;
  const uint32_t tmem = mlp_cta_setup(M, align1024(smem_raw), G);
  const int g = threadIdx.x >> 7, t = threadIdx.x & 127;
  const long turn = *bi.turn;
  const size_t n6 = (size_t)a.npad;
  double *C = a.coord;
  const long nitems = (long)a.ntile * 64;
  double aud_max = 0.0, aud_sq = 0.0;
  int aud_n = 0, fallbacks = 0;
  bool ok = true;
  for (long item = (long)blockIdx.x * kMlpGroups + g; item < nitems && ok; item += (long)gridDim.x * kMlpGroups) {
    const Tile tile = a.tiles[item / 64];
    const int sub = (int)(item % 64);
    if (sub * 128 >= tile.count) continue;   // the same for the whole group
    const int b = tile.bunch;
    const int p = tile.start + sub * 128 + t;
    const bool live = sub * 128 + t < tile.count;
    double x = 0.0, z = 0.0, xp = 0.0, zp = 0.0;
    if (live) {
      x = C[1 * n6 + p];
      z = C[2 * n6 + p];
      xp = C[4 * n6 + p];
      zp = C[5 * n6 + p];
    }
    double ddx = 0.0, ddxp = 0.0, ddz = 0.0, ddzp = 0.0;
    for (int k = 0; k < bi.n_ip; ++k) {
      // the cloud this bunch meets at point k and the point's phase
      // advance: the same addresses in every thread (cached broadcasts)
      const double *Cl = bi.cloud + ((size_t)k * bi.nb + b) * 5;
      const double nion = __ldg(Cl);
      if (nion == 0.0) continue;               // the same for the whole group
      const double *tr = bi.trig + 4 * k;
      const double c0 = __ldg(tr), s0 = __ldg(tr + 1), c1 = __ldg(tr + 2), s1 = __ldg(tr + 3);
      const double mx = c0 + bi.alphaH * s0, sxb = bi.betaH * s0;
      const double my = c1 + bi.alphaV * s1, syb = bi.betaV * s1;
      const double xk = mx * x + sxb * xp, zk = my * z + syb * zp;
      double gx = 0.0, gy = 0.0;
      if (!bi_field_mlp(bi, G, t, live, xk - __ldg(Cl + 1), zk - __ldg(Cl + 2), __ldg(Cl + 3), __ldg(Cl + 4),
                        bi_hash((uint32_t)turn + 0x51ED27u, (uint32_t)k, (uint32_t)(p >> 5)), gx, gy, aud_max, aud_sq,
                        aud_n, fallbacks)) {
        ok = false;
        break;
      }
      const double kn = bi.ke * nion;
      const double thx = kn * gx, thy = kn * gy;
      ddx = ddx - sxb * thx;
      ddxp = ddxp + mx * thx;
      ddz = ddz - syb * thy;
      ddzp = ddzp + my * thy;
    }
    if (live && ok) {
      C[1 * n6 + p] = x + ddx;
      C[4 * n6 + p] = xp + ddxp;
      C[2 * n6 + p] = z + ddz;
      C[5 * n6 + p] = zp + ddzp;
    }
  }
  bi_audit_flush(bi, aud_max, aud_sq, aud_n, fallbacks);
  if ((mlp_cta_release(tmem, G) || !ok) && t == 0) {
    atomicAdd(&bi.audit[3], 1ull);
    atomicOr(bi.error, 4);
  }
}

}  // namespace mbt
