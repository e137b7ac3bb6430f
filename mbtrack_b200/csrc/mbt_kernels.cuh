// mbt_kernels.cuh -- the per-turn kernels of the weak-weak loop.
//
// One turn of worker_weakweak.c:259-394 for every bunch is four launches:
//
//   turn_map      particle pass over all bunches (K1): pending resistive-
//                 wall kick (transform_weak.c:829-830 of the previous
//                 turn), self-field and long-range wake kick
//                 (transform_weak.c:697-731), RF/radiation/noise/drift
//                 (:49-97), vertical and horizontal betatron maps
//                 (:101-190); then, on the new coordinates, shifted moment
//                 sums (statistics.c:91-128) and the binning of the next
//                 turn (transform_weak.c:608-631, :839-865).  HBM-bound.
//   bunch_reduce  one block per bunch: partial records -> histograms,
//                 statistics, resistive-wall dipole history
//                 (worker_weakweak.c:306-318), in-bucket phasor recurrence
//                 of each long-range resonator (transform_weak.c:1014-1027).
//   ring_scan     one block: the phasor of each long-range resonator around
//                 the ring, bucket h-1 .. 0 (transform_weak.c:1006-1044),
//                 RF-feedback samples and correction (feedback_rf.c,
//                 worker_weakweak.c:268-278).
//   bunch_wakes   one block per bunch: causal convolutions with the Green's
//                 functions (transform_weak.c:653-731), long-range wake per
//                 bin, kick tables, resistive-wall sum over the dipole
//                 history (transform_weak.c:813-825).
//
// Arithmetic that the parity tests compare against the oracle keeps the
// reference's operation order; where the compiler would contract a multiply
// and an add of such an expression into one FMA, the multiply and the add
// are written with the round-to-nearest intrinsics (__dmul_rn, __dadd_rn).
#pragma once
#include <cstdint>
#include "mbt_device.cuh"
#include "mbt_philox.cuh"
#include "mbt_common.cuh"

namespace mbt {

// ---------------------------------------------------------------- K1

// One macroparticle through the pending RW kick, the wake kick and the
// one-turn map (transform_weak.c:21-192); coordinates updated in place.
// PLAIN: the common ring of a launch, known at compile time: all three
// planes tracked, RF without harmonic cavities, no amplitude detuning, no
// dispersion at the kick point (the general form tests each of these per
// particle, or computes the unused terms under a predicate).
template <int NOISE, bool PLAIN>
__device__ __forceinline__ void advance_particle(const Args &a, const OpticConst &oc, double &xtau, double &x,
                                                 double &z, double &eps, double &xp, double &zp, bool rw,
                                                 double rwH, double rwV, bool sf, bool kick_l, bool kick_v,
                                                 bool kick_h, const double *kL, const double *kV,
                                                 const double *kH, int nc, double eps_const, double phai0,
                                                 double sin_ph, double cos_ph, int kb, uint32_t jb,
                                                 long turn, size_t p, bool disp_) {
  const bool track_h = PLAIN || oc.track_h, track_v = PLAIN || oc.track_v;
  const bool ideal_hc = !PLAIN && oc.ideal_hc, amp_dep = !PLAIN && oc.amp_dep, disp = !PLAIN && disp_;
  const int n_ahc = PLAIN ? 0 : oc.n_ahc;
  if (rw) {
    if (track_h) xp = xp + rwH;
    if (track_v) zp = zp + rwV;
  }
  if (sf) {
    int ic = bin_fast(xtau, oc.sigma_tau, oc.nsigma, oc.dT, oc.inv_sigma_tau, oc.inv_dT);
    ic = ic < 0 ? 0 : (ic >= nc ? nc - 1 : ic);
    if (kick_l) eps = eps + kL[ic];
    if (kick_v) zp = zp + kV[ic];
    if (kick_h) xp = xp + kH[ic];
  }
  // ---- longitudinal (transform_weak.c:49-97)
  const double xtau0 = xtau, eps0 = eps, x0 = x, xp0 = xp, z0 = z, zp0 = zp;
  double g;
  if (!ideal_hc) {
    // sin(wrf xtau + phai0) with the reference's rounding of the argument
    const double arg = __dadd_rn(__dmul_rn(oc.wrf, xtau0), phai0);
    const double d = arg - phai0;
    double sr, cr;
    // (the RF offsets of a warp straddle |d| = 0.04: one branch-free series)
    if (fabs(d) <= 0.25) sincos_near_full(d, sin_ph, cos_ph, sr, cr);
    else sr = sin(arg);
    g = eps_const * sr;
    for (int j = 0; j < n_ahc; ++j) {
      const double ph = oc.ahc_nhc[j] * (double)kb * 2 * MBT_PI;
      g += oc.ahc_amp[j] * sin(oc.ahc_w[j] * xtau0 + oc.ahc_phi[j] + ph);
    }
  } else {
    g = eps_const * (sin(oc.wrf * xtau0 + phai0) + oc.HC_k * sin(oc.m_aHC_d * oc.wrf * xtau0 + oc.m_phi_n));
  }
  float dv[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  if (NOISE == MBT_NOISE_PHILOX) {
    PhiloxKeys K;
#pragma unroll
    for (int q = 0; q < 10; ++q) { K.k0[q] = a.philox_k0[q]; K.k1[q] = a.philox_k1[q]; }
    turn_normals1(K, jb, (uint32_t)kb, (uint64_t)turn, dv);
  } else if (NOISE == MBT_NOISE_INJECTED) {
    const long dt = turn - a.dev_turn0;
    if (dt >= 0 && dt < a.dev_nturn) {
      const float *dd = a.dev + (size_t)dt * 5 * (size_t)a.npad + p;
#pragma unroll
      for (int k = 0; k < 5; ++k) dv[k] = dd[(size_t)k * a.npad];
    } else {
      atomicOr(&a.rs->error, 1);
    }
  }
  eps = eps0 + g - oc.Urad;
  double rff = 1.0;
  if (NOISE != MBT_NOISE_NONE) {
    eps = eps * oc.damp + oc.excite * (double)dv[0];
    rff = div_near1(1.0 + eps0, 1.0 + eps0 + g);
  }
  xtau = xtau0 - eps * oc.T0 * oc.ac;
  // ---- amplitude terms (transform_weak.c:115-123, 159-167)
  double EV = 0.0, EH = 0.0;
  if (amp_dep) {
    EV = oc.gammaV * z0 * z0 + 2 * oc.alphaV * z0 * zp0 + oc.betaV * zp0 * zp0;
    EH = oc.gammaV * x0 * x0 + 2 * oc.alphaV * x0 * xp0 + oc.betaV * xp0 * xp0;
  }
  // ---- vertical (transform_weak.c:101-141)
  if (track_v) {
    const double dQ = amp_dep ? (oc.CVH * EH + oc.CVV * EV) : 0.0;
    const double psi = __dmul_rn(oc.psiV0, __dadd_rn(__dadd_rn(1.0, __dmul_rn(oc.Gziz, eps0)), dQ));
    double sn, cs;
    const double d = psi - oc.psiV0;
    if (fabs(d) <= 0.25) sincos_near(d, oc.sin_psiV0, oc.cos_psiV0, sn, cs);
    else sincos(psi, &sn, &cs);
    const double a11 = cs + oc.alphaV * sn, a12 = oc.betaV * sn;
    const double a21 = -oc.gammaV * sn, a22 = cs - oc.alphaV * sn;
    z = a11 * z0 + a12 * zp0;
    zp = a21 * z0 + a22 * zp0;
    if (NOISE != MBT_NOISE_NONE) {
      z = z + oc.qv_pos * (double)dv[1];
      zp = rff * zp + oc.qv_slope * (double)dv[2];
    }
  }
  // ---- horizontal (transform_weak.c:144-190)
  if (track_h) {
    const double dQ = amp_dep ? (oc.CHH * EH + oc.CHV * EV) : 0.0;
    const double psi = __dmul_rn(oc.psiH0, __dadd_rn(__dadd_rn(1.0, __dmul_rn(oc.Gzix, eps0)), dQ));
    double sn, cs;
    const double d = psi - oc.psiH0;
    if (fabs(d) <= 0.25) sincos_near(d, oc.sin_psiH0, oc.cos_psiH0, sn, cs);
    else sincos(psi, &sn, &cs);
    const double a11 = cs + oc.alphaH * sn;
    const double a12 = oc.betaH * sn;
    const double a21 = -oc.gammaH * sn;
    const double a22 = cs - oc.alphaH * sn;
    if (disp) {
      const double a13 = (1.0 - a11) * oc.dispH - a12 * oc.disppH;
      const double a23 = -a21 * oc.dispH + (1.0 - a22) * oc.disppH;
      x = a11 * x0 + a12 * xp0 + a13 * eps;
      xp = a21 * x0 + a22 * xp0 + a23 * eps;
    } else {
      // no dispersion at the kick point: the energy terms vanish
      x = a11 * x0 + a12 * xp0;
      xp = a21 * x0 + a22 * xp0;
    }
    if (NOISE != MBT_NOISE_NONE) {
      x = x + oc.qh_pos * (double)dv[3];
      xp = rff * xp + oc.qh_slope * (double)dv[4];
    }
  }
}

// Particle pass (K1).  Each block streams its tile through a ring of
// kStages shared-memory stages of kChunk particles.  Warp 8 is the
// producer: it issues six bulk loads per stage (completion on the stage's
// `full` mbarrier) and, once the eight compute warps have released a stage
// (`empty` mbarrier), six bulk stores of the updated coordinates.  Compute
// warps advance kPPT particles per thread per chunk in place, then sum the
// moments column-wise from the staged chunk; they synchronise only among
// themselves (hardware barrier 1).
// Stage shape of the particle pass: each compute thread advances
// MBT_MAP_PPT particles of a stage one after the other, through
// MBT_MAP_STAGES stages.  Two particles per thread halve the per-stage
// synchronisation per particle; two stages of 512 keep three CTAs per SM
// (measured on the 416-bunch fill: 0.214 ms against 0.223 ms for 1 x 3 and
// 0.25 ms for 2 x 3 or 4 x 2, which fit only two CTAs per SM).
#ifndef MBT_MAP_PPT
#define MBT_MAP_PPT 2
#endif
// Histogram counts: one shared atomic per particle (0), or warp-aggregated
// with match.any, one atomic per distinct bin of a warp (1).  The pass is
// bound by instruction issue, and the aggregation's extra instructions cost
// more than the conflicting atomics it saves (measured: 0.248 against
// 0.225 ms per pass on the 416-bunch fill), so 0 is the default.
#ifndef MBT_HIST_AGG
#define MBT_HIST_AGG 0
#endif
#ifndef MBT_MAP_STAGES
#define MBT_MAP_STAGES 2
#endif
constexpr int kPPT = MBT_MAP_PPT;          // particles per compute thread per chunk
constexpr int kChunk = kPPT * kBlock;
constexpr int kStages = MBT_MAP_STAGES;
constexpr int kMapThreads = kBlock + 32;   // 8 compute warps + 1 producer warp
constexpr long kWaitLimit = 1L << 24;      // polls before a wait is declared failed

// stages, kick tables and histograms (with the dipole histograms: two
// fixed-point words for each of x and z per bin)
__host__ __device__ constexpr size_t turn_map_smem(int nc, bool histxz = false) {
  return (size_t)kStages * 6 * kChunk * sizeof(double) + (size_t)nc * (histxz ? 7 : 5) * sizeof(double) +
         (size_t)nc * sizeof(int);
}

// Resident CTAs per SM the register allocation is sized for (shared memory
// allows 4 at 256 bins).
#ifndef MBT_MAP_MIN_BLOCKS
#define MBT_MAP_MIN_BLOCKS 3
#endif

template <bool MOVE, int NOISE, bool HISTXZ>
__global__ void __launch_bounds__(kMapThreads, MBT_MAP_MIN_BLOCKS) turn_map(Args a) {
  extern __shared__ __align__(128) double smem[];
  const int nc = a.ncell;
  const Tile tile = a.tiles[blockIdx.x];
  const int b = tile.bunch;
  double *stage = smem;
  double *kL = smem + kStages * 6 * kChunk;
  double *kV = kL + nc;
  double *kH = kL + 2 * nc;
  // dipole histograms: fixed-point sums of x (hi, lo words) and z per bin
  unsigned long long *fxh = reinterpret_cast<unsigned long long *>(kL + 3 * nc);
  unsigned long long *fxl = fxh + nc, *fzh = fxh + 2 * nc, *fzl = fxh + 3 * nc;
  int *hc = reinterpret_cast<int *>(kL + (HISTXZ ? 7 : 5) * nc);
  __shared__ __align__(8) uint64_t full[kStages];
  __shared__ __align__(8) uint64_t empty[kStages];
  __shared__ double red[8][3];                  // per compute warp: sum, square sum, cross sum
  __shared__ double trash_n[2];                 // out-of-range particles below / above the bins
  __shared__ unsigned long long trash_fx[8];    // their x and z, fixed-point (hi, lo) pairs
  __shared__ double shift[6];

  const bool sf = MOVE && a.selffield;
  for (int i = threadIdx.x; i < nc; i += kMapThreads) {
    if (sf) {
      kL[i] = a.kick[(size_t)(b * 3 + 0) * nc + i];
      kV[i] = a.kick[(size_t)(b * 3 + 1) * nc + i];
      kH[i] = a.kick[(size_t)(b * 3 + 2) * nc + i];
    }
    hc[i] = 0;
    if (HISTXZ) fxh[i] = fxl[i] = fzh[i] = fzl[i] = 0ull;
  }
  if (threadIdx.x < 8) trash_fx[threadIdx.x] = 0ull;
  if (threadIdx.x < 2) trash_n[threadIdx.x] = 0.0;
  if (threadIdx.x < 6) shift[threadIdx.x] = a.shift[b * 6 + threadIdx.x];
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kBlock / 32);
    }
    fence_mbar_init();
  }
  __syncthreads();

  const size_t np6 = (size_t)a.npad;
  double *__restrict__ C = a.coord;
  const int nchunk = (tile.count + kChunk - 1) / kChunk;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto chunk_bytes = [&](int c) -> uint32_t {
    const int n = min(kChunk, tile.count - c * kChunk);
    return (uint32_t)(((n * 8) + 15) & ~15);
  };

  if (warp == kBlock / 32) {
    // ---------------- producer warp
    if (lane == 0) {
      auto store = [&](int cc) {
        const int s = cc % kStages;
        if (!mbar_wait(&empty[s], (uint32_t)((cc / kStages) & 1), kWaitLimit)) atomicOr(&a.rs->error, 2);
        if (MOVE) {
          const uint32_t bytes = chunk_bytes(cc);
          const size_t g0 = (size_t)tile.start + (size_t)cc * kChunk;
          for (int k = 0; k < 6; ++k) bulk_store(C + k * np6 + g0, stage + (size_t)(s * 6 + k) * kChunk, bytes);
          bulk_commit();
        }
      };
      for (int c = 0; c < nchunk; ++c) {
        const int s = c % kStages;
        if (c >= kStages) {
          store(c - kStages);              // frees stage s once the store has read it
          if (MOVE) bulk_wait_read<0>();
        }
        const uint32_t bytes = chunk_bytes(c);
        mbar_expect_tx(&full[s], 6 * bytes);
        const size_t g0 = (size_t)tile.start + (size_t)c * kChunk;
        for (int k = 0; k < 6; ++k)
          bulk_load(stage + (size_t)(s * 6 + k) * kChunk, C + k * np6 + g0, bytes, &full[s]);
      }
      for (int cc = max(0, nchunk - kStages); cc < nchunk; ++cc) store(cc);
      bulk_wait_all();
    }
    return;
  }

  // ---------------- compute warps
  const OpticConst &oc = a.oc;
  const long turn = a.rs->turn;
  const double eps_const = a.rs->Vrf0 / (oc.E0 * 1.0e3);
  const double phai0 = a.rs->phai0;
  const double sin_ph = a.rs->sin_phai0, cos_ph = a.rs->cos_phai0;
  const int kb = a.bunch_kb[b];
  double rwH = 0.0, rwV = 0.0;
  const bool rw = MOVE && a.rw_long && turn > 0;
  if (rw) {
    rwH = a.rw_part[(size_t)b * 2 + 0];
    rwV = a.rw_part[(size_t)b * 2 + 1];
  }
  const bool kick_l = sf && a.lr_kick[0];
  const bool kick_h = sf && a.lr_kick[1];
  const bool kick_v = sf && a.lr_kick[2];
  const int jb0 = tile.start - a.bunch_off[b];   // index of the tile's first particle in its bunch
  const bool disp = oc.dispH != 0.0 || oc.disppH != 0.0;
  const bool plain = oc.track_h && oc.track_v && !oc.ideal_hc && oc.n_ahc == 0 && !oc.amp_dep && !disp;
  // moments: warp w < 4 owns coordinate column w (xtau, x, z, eps) of every
  // staged chunk; warps 4 and 6 share column 4 (x') and the cross product
  // x x', warps 5 and 7 column 5 (z') and z z', each on half of the chunk.
  // Every warp then does about the same work per chunk (the per-chunk
  // barrier waits for the slowest).
  const int mcol = warp < 4 ? warp : 4 + (warp & 1);          // summed and squared column
  const int mpair = mcol - 3;                                  // x or z, for the cross product
  const int mhalf = warp >= 6 ? 1 : 0;                         // warps 6, 7: second half of the chunk
  const double col_shift = shift[mcol];
  const double pair_shift = warp >= 4 ? shift[mpair] : 0.0;
  double col_s = 0.0, col_q = 0.0, col_c = 0.0;

  for (int c = 0; c < nchunk; ++c) {
    const int s = c % kStages;
    if (!mbar_wait(&full[s], (uint32_t)((c / kStages) & 1), kWaitLimit)) atomicOr(&a.rs->error, 2);
    double *st = stage + (size_t)s * 6 * kChunk;
    // kPPT particles per thread, one after the other: t, t + kBlock, ...
#pragma unroll 1
    for (int u = 0; u < kPPT; ++u) {
      const int e = u * kBlock + threadIdx.x;
      const int i = c * kChunk + e;
      const bool live = i < tile.count;
      double v[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) v[k] = live ? st[k * kChunk + e] : 0.0;
      if (MOVE && live) {
        if (plain)
          advance_particle<NOISE, true>(a, oc, v[0], v[1], v[2], v[3], v[4], v[5], rw, rwH, rwV, sf, kick_l, kick_v,
                                        kick_h, kL, kV, kH, nc, eps_const, phai0, sin_ph, cos_ph, kb,
                                        (uint32_t)(jb0 + i), turn, (size_t)tile.start + i, disp);
        else
          advance_particle<NOISE, false>(a, oc, v[0], v[1], v[2], v[3], v[4], v[5], rw, rwH, rwV, sf, kick_l, kick_v,
                                         kick_h, kL, kV, kH, nc, eps_const, phai0, sin_ph, cos_ph, kb,
                                         (uint32_t)(jb0 + i), turn, (size_t)tile.start + i, disp);
#pragma unroll
        for (int k = 0; k < 6; ++k) st[k * kChunk + e] = v[k];
      }
      // ---- binning of the next turn (out-of-range particles are rare: shared atomics)
      if (a.selffield) {
        const double xtau = v[0], x = v[1], z = v[2];
        const int ic = bin_fast(xtau, oc.sigma_tau, oc.nsigma, oc.dT, oc.inv_sigma_tau, oc.inv_dT);
        const bool in = live && ic >= 0 && ic < nc;
#if MBT_HIST_AGG
        // warp-aggregated counts: one shared atomic per distinct bin of the
        // warp (every lane of a compute warp runs this)
        const unsigned grp = __match_any_sync(0xffffffffu, in ? ic : -1);
        if (in && (int)(__ffs(grp) - 1) == lane) atomicAdd(&hc[ic], (int)__popc(grp));
#endif
        if (in) {
#if !MBT_HIST_AGG
          atomicAdd(&hc[ic], 1);
#endif
          if (HISTXZ) {
            fx70_add(&fxh[ic], &fxl[ic], x);
            fx70_add(&fzh[ic], &fzl[ic], z);
          }
        } else if (live) {
          unsigned long long *t = trash_fx + (ic < 0 ? 0 : 4);
          atomicAdd(&trash_n[ic < 0 ? 0 : 1], 1.0);   // integer counts: exact in any order
          fx70_add(&t[0], &t[1], x);
          fx70_add(&t[2], &t[3], z);
        }
      }
    }
    if (MOVE) fence_proxy_async();
    named_barrier(1, kBlock);
    // ---- moments (statistics.c:91-128): shifted sums of the updated chunk,
    //      one coordinate column per warp (the bulk store only reads it too)
    const int nlive = min(kChunk, tile.count - c * kChunk);
    if (nlive == kChunk) {
      // full chunk: two elements per lane and load, no bounds test
      const double2 *col = reinterpret_cast<const double2 *>(st + (size_t)mcol * kChunk);
      if (warp < 4) {
#pragma unroll
        for (int q = 0; q < kChunk / 64; ++q) {
          const double2 v = col[q * 32 + lane];
          const double d0 = v.x - col_shift, d1 = v.y - col_shift;
          col_s += d0;
          col_q += d0 * d0;
          col_s += d1;
          col_q += d1 * d1;
        }
      } else {
        const double2 *pr = reinterpret_cast<const double2 *>(st + (size_t)mpair * kChunk);
        const int q0 = mhalf * (kChunk / 128);
#pragma unroll
        for (int q = q0; q < q0 + kChunk / 128; ++q) {
          const double2 v = col[q * 32 + lane], u = pr[q * 32 + lane];
          const double d0 = v.x - col_shift, d1 = v.y - col_shift;
          col_s += d0;
          col_q += d0 * d0;
          col_c += (u.x - pair_shift) * d0;
          col_s += d1;
          col_q += d1 * d1;
          col_c += (u.y - pair_shift) * d1;
        }
      }
    } else {
      const double *col = st + (size_t)mcol * kChunk;
      if (warp < 4) {
#pragma unroll
        for (int q = 0; q < kChunk / 32; ++q) {
          const int e = q * 32 + lane;
          const double d = e < nlive ? col[e] - col_shift : 0.0;
          col_s += d;
          col_q += d * d;
        }
      } else {
        const double *pr = st + (size_t)mpair * kChunk;
        const int q0 = mhalf * (kChunk / 64);
#pragma unroll
        for (int q = q0; q < q0 + kChunk / 64; ++q) {
          const int e = q * 32 + lane;
          if (e < nlive) {
            const double d = col[e] - col_shift;
            col_s += d;
            col_q += d * d;
            col_c += (pr[e] - pair_shift) * d;
          }
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
  // column sums -> block sums, in a fixed order
  {
    const double vs = warp_sum(col_s), vq = warp_sum(col_q), vc = warp < 4 ? 0.0 : warp_sum(col_c);
    if (lane == 0) {
      red[warp][0] = vs;
      red[warp][1] = vq;
      red[warp][2] = vc;
    }
  }
  named_barrier(1, kBlock);
  double *rec = a.part + (size_t)blockIdx.x * a.prec;
  if (threadIdx.x < kPartialExtra) {
    // out-of-range extras: count, x sum, z sum below the bins, then above
    const int q = threadIdx.x % 3, side = threadIdx.x / 3;
    double sum;
    if (threadIdx.x >= 6) {
      // moment m: sums of columns 0..5, their squares, then x x' and z z';
      // columns 4 and 5 and the cross sums are the two halves' sums, first half first
      const int m = threadIdx.x - 6, col = m < 12 ? m % 6 : m - 8, kind = m < 6 ? 0 : (m < 12 ? 1 : 2);
      sum = col < 4 ? red[col][kind] : red[col][kind] + red[col + 2][kind];
    }
    else if (q == 0) sum = trash_n[side];
    else sum = fx70_value(trash_fx[4 * side + 2 * (q - 1)], trash_fx[4 * side + 2 * (q - 1) + 1]);
    rec[a.hoff + threadIdx.x] = sum;
  }
  for (int i = threadIdx.x; i < nc; i += kBlock) {
    rec[i] = (double)hc[i];
    if (HISTXZ) {
      rec[nc + i] = fx70_value(fxh[i], fxl[i]);
      rec[2 * nc + i] = fx70_value(fzh[i], fzl[i]);
    }
  }
}

// ---------------------------------------------------------------- K2a

enum { kReduceTurn = 0, kReducePrologue = 1 };

__global__ void __launch_bounds__(kBlock) bunch_reduce(Args a, int mode, double *stats_init) {
  extern __shared__ double tot[];   // prec doubles
  const int b = blockIdx.x, nc = a.ncell;
  const int t0 = a.bunch_tile0[b], nt = a.bunch_ntile[b];
  for (int e = threadIdx.x; e < a.prec; e += kBlock) {
    double s = 0.0;
    for (int k = 0; k < nt; ++k) s += a.part[(size_t)(t0 + k) * a.prec + e];
    tot[e] = s;
  }
  __syncthreads();
  const double *ex = tot + a.hoff;
  const double N = (double)a.bunch_np[b];
  const int kb = a.bunch_kb[b];
  const long turn = a.rs->turn;

  // histograms: clamped (bins 0 and ncell-1 collect the out-of-range
  // particles, transform_weak.c:615-624) and dropped (:857-862)
  double *H = a.hist + (size_t)b * 6 * nc;
  if (a.selffield) {
    for (int j = threadIdx.x; j < nc; j += kBlock) {
      const double cn = tot[j];
      const double sx = a.hist_xz ? tot[nc + j] : 0.0, sz = a.hist_xz ? tot[2 * nc + j] : 0.0;
      double f = cn, dv = sz, dh = sx;
      if (j == 0) { f += ex[kTrLowN]; dv += ex[kTrLowZ]; dh += ex[kTrLowX]; }
      if (j == nc - 1) { f += ex[kTrHighN]; dv += ex[kTrHighZ]; dh += ex[kTrHighX]; }
      H[j] = f;
      H[nc + j] = dv;
      H[2 * nc + j] = dh;
      H[3 * nc + j] = cn;
      H[4 * nc + j] = sx;
      H[5 * nc + j] = sz;
    }
  }
  __shared__ double mean6[6];
  if (threadIdx.x < 6) {
    const int k = threadIdx.x;
    const int plane = k % 3;
    const bool tracked = plane == 0 || (plane == 1 ? a.oc.track_h : a.oc.track_v);
    double mean = 0.0, rms = 0.0;
    if (tracked && N > 0) {
      const double s = ex[kMomSum + k] / N;
      const double q = ex[kMomSq + k] / N;
      mean = a.shift[b * 6 + k] + s;
      const double var = q - s * s;
      rms = sqrt(var > 0.0 ? var : 0.0);
      a.shift[b * 6 + k] = mean;
    }
    mean6[k] = mean;
    // row order pos[3], pos_sigma[3], slope[3], slope_sigma[3]
    const int col = (k < 3) ? k : 6 + (k - 3);
    double *row = (mode == kReduceTurn)
                      ? a.stats + ((size_t)(turn % a.stats_cap) * a.nbunch + b) * 12
                      : stats_init + (size_t)b * 12;
    row[col] = mean;
    row[col + 3] = rms;
  }
  __syncthreads();
  // amplitude invariants (weak_bunch_calc_ampinv statistics.c:163-195):
  // <gamma u^2 + 2 alpha u u' + beta u'^2> over particles, and the same of
  // the centroid, from the shifted first and second moments
  if (threadIdx.x < 3) {
    const int pl = threadIdx.x;
    const bool tracked = pl == 0 || (pl == 1 ? a.oc.track_h : a.oc.track_v);
    double ai = 0.0, aic = 0.0;
    if (tracked && N > 0) {
      const double g = pl == 0 ? a.oc.gammaL : (pl == 1 ? a.oc.gammaH : a.oc.gammaV);
      const double al = pl == 0 ? a.oc.alphaL : (pl == 1 ? a.oc.alphaH : a.oc.alphaV);
      const double be = pl == 0 ? a.oc.betaL : (pl == 1 ? a.oc.betaH : a.oc.betaV);
      const double m = mean6[pl], mp = mean6[3 + pl];
      const double su = ex[kMomSum + pl] / N, sp = ex[kMomSum + 3 + pl] / N;
      const double vu = ex[kMomSq + pl] / N - su * su;         // variance of u
      const double vp = ex[kMomSq + 3 + pl] / N - sp * sp;     // variance of u'
      const double cuv = pl == 0 ? 0.0 : ex[kMomCross + pl - 1] / N - su * sp;
      // (the reference never sets the LON Twiss values, so its LON
      // invariants are 0; no LON cross moment is kept)
      aic = g * m * m + 2.0 * al * m * mp + be * mp * mp;
      ai = g * (vu + m * m) + 2.0 * al * (cuv + m * mp) + be * (vp + mp * mp);
    }
    double *row = (mode == kReduceTurn) ? a.ampinv + ((size_t)(turn % a.stats_cap) * a.nbunch + b) * 6 : nullptr;
    if (row) {
      row[pl] = ai;
      row[3 + pl] = aic;
    }
  }
  // transverse moments for the beam-ion stage: means, variances and the
  // position-slope covariance per plane
  if (a.bi_mom != nullptr && threadIdx.x < 2 && mode == kReduceTurn) {
    const int pl = 1 + threadIdx.x;
    double *m = a.bi_mom + (size_t)b * 10 + 5 * threadIdx.x;
    double vu = 0.0, vp = 0.0, cuv = 0.0;
    if (N > 0) {
      const double su = ex[kMomSum + pl] / N, sp = ex[kMomSum + 3 + pl] / N;
      vu = ex[kMomSq + pl] / N - su * su;
      vp = ex[kMomSq + 3 + pl] / N - sp * sp;
      cuv = ex[kMomCross + pl - 1] / N - su * sp;
    }
    m[0] = mean6[pl];
    m[1] = mean6[3 + pl];
    m[2] = vu;
    m[3] = cuv;
    m[4] = vp;
  }
  if (threadIdx.x == 0 && a.selffield) {
    atomicAdd(&a.rs->trash_low, (int)ex[kTrLowN]);
    atomicAdd(&a.rs->trash_high, (int)ex[kTrHighN]);
  }
  __syncthreads();
  // resistive-wall dipole history (worker_weakweak.c:306-318; set-up
  // fill :203-219)
  if (a.rw_long && threadIdx.x == 0) {
    const long n = (long)(a.Nmlt + 2) * a.nharm;
    const double ibk = a.rw_ib[kb];
    if (mode == kReduceTurn) {
      const long sl = cyc_slot(-turn * a.nharm + kb, n);
      a.dipole[2 * sl] = mean6[1];
      a.dipole[2 * sl + 1] = mean6[2];
      a.rw_e[sl] = mean6[1] * ibk;
      a.rw_e[n + sl] = mean6[2] * ibk;
    } else {
      const int jmax = a.Nmlt > 1 ? a.Nmlt : 1;
      for (int j = 0; j < jmax; ++j) {
        const long sl = cyc_slot((long)j * a.nharm + kb, n);
        a.dipole[2 * sl] = mean6[1];
        a.dipole[2 * sl + 1] = mean6[2];
        a.rw_e[sl] = mean6[1] * ibk;
        a.rw_e[n + sl] = mean6[2] * ibk;
      }
    }
  }
  // in-bucket phasor of each long-range resonator, starting from zero:
  // V_j = V_{j-1} prog - Ib fnp_j fac  (transform_weak.c:1017-1018), as a
  // warp scan of affine maps over the bins, one warp per resonator
  if (a.selffield) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int chunk = (nc + 31) / 32;
    const int j0 = min(lane * chunk, nc), j1 = min(j0 + chunk, nc);
    const double ib = a.ibunch[kb];
    for (int r = warp; r < a.nlr; r += kBlock / 32) {
      const LrConst &L = a.lr[r];
      // dropped histogram of the plane (H rows 3..5), read from the summed
      // records in shared memory; a plane without dipole sums has zeros
      const double *src = L.plane == 0 ? tot : (a.hist_xz ? tot + (size_t)L.plane * nc : nullptr);
      const double fac = a.bunch_fac[(size_t)r * a.nbunch + b];
      double *u = a.lr_u + ((size_t)r * a.nbunch + b) * nc * 2;
      double *bb = a.lr_b + ((size_t)r * a.nbunch + b) * nc;
      Aff f = aff_id();
      for (int j = j0; j < j1; ++j) {
        const Aff g{L.prog[0], L.prog[1], -(ib * (src ? src[j] : 0.0) * fac), 0.0};
        f = compose(f, g);
      }
      const Aff ex = warp_exclusive_scan(f, lane);
      double v0 = ex.a0, v1 = ex.a1;
      for (int j = j0; j < j1; ++j) {
        const double s = ib * (src ? src[j] : 0.0) * fac;
        const double n0 = (v0 * L.prog[0] - v1 * L.prog[1]) - s;
        const double n1 = (v0 * L.prog[1] + v1 * L.prog[0]);
        v0 = n0;
        v1 = n1;
        u[2 * j] = v0;
        u[2 * j + 1] = v1;
        bb[j] = s;
      }
    }
  }
}

// ---------------------------------------------------------------- K2b

// Feedback sample (rffb_get_vrf_phi, feedback_rf.c:5-12): note atan2(real, imag).
__device__ __forceinline__ void rffb_store(Args &a, int slot, double vr, double vi) {
  a.rffb_hist[2 * slot] = sqrt(vr * vr + vi * vi);
  a.rffb_hist[2 * slot + 1] = atan2(vr, vi);
}

// Long-range resistive wall (transform_weak.c:779-833) of the turn just
// completed, applied at the start of the next particle pass.  The kick of
// bunch b sums E(step j of b) rsq[j + 1] over the (Nmlt + 1) h history
// steps j (E = dipole x bucket current, empty buckets 0), where step j of
// bunch b is the cyclic history slot -turn h + kb_b + 1 + j.
// The bunches' windows are one window shifted by their bucket offsets, so
// each block of the sums takes a range of steps for every bunch: it stages
// that range of the history (plus the bunches' bucket span) and the
// weights once, and each thread sums whole bunches.  rw_steps_per_block:
// the length of a block's range for nblk blocks.
__host__ __device__ constexpr int rw_steps_per_block(int Nmlt, int nharm, int nblk) {
  return ((Nmlt + 1) * nharm + nblk - 1) / nblk;
}
__host__ __device__ constexpr size_t rw_window_doubles(int per, int nharm) {
  return (size_t)2 * (per + nharm) + per;
}

// Dynamic shared memory of ring_scan (doubles): block 0 keeps 2 doubles and
// one int per bucket, the resistive-wall blocks their window and weights.
__host__ __device__ constexpr size_t ring_scan_smem_doubles(int rw_long, int Nmlt, int nharm, int rw_nblk) {
  const size_t scan = 2 * (size_t)nharm + ((size_t)nharm + 1) / 2 + 1;
  const size_t rw = rw_long && rw_nblk > 0 ? rw_window_doubles(rw_steps_per_block(Nmlt, nharm, rw_nblk), nharm) : 0;
  return scan > rw ? scan : rw;
}

// Block blk of a.rw_nblk: steps [q0, q1) of every bunch, times the kick
// constant of the plane, into rw_acc[blk][bunch][plane].
__device__ void rw_partial_sums(const Args &a, int blk, double *win) {
  const long turn = a.rs->turn;              // the turn just completed (advanced by bunch_wakes)
  const int h = a.nharm;
  const int n = (a.Nmlt + 2) * h;
  const int M = (a.Nmlt + 1) * h;
  const int per = rw_steps_per_block(a.Nmlt, h, a.rw_nblk);
  const int q0 = min(M, blk * per), q1 = min(M, q0 + per), L = q1 - q0;
  const int kb0 = a.bunch_kb[0];
  const int len = L + (a.bunch_kb[a.nbunch - 1] - kb0);
  const int base = (int)cyc_slot(-turn * h + kb0 + 1 + q0, n);
  double *w0 = win, *w1 = win + len, *wt = win + 2 * len;
  for (int t = threadIdx.x; t < len; t += kBlock) {
    int idx = base + t;                      // base < n and t < n: one wrap at most
    idx -= (idx >= n) ? n : 0;
    w0[t] = a.rw_e[idx];
    w1[t] = a.rw_e[n + idx];
  }
  for (int t = threadIdx.x; t < L; t += kBlock) wt[t] = a.rw_rsq[q0 + t + 1];
  __syncthreads();
  const int mtrig = a.rs->rw_m;              // RW kicks done before this one
  const int trig = (a.triggerRW && mtrig < 50) ? 1 : 0;
  const double cH = a.oc.track_h ? a.rw_const[trig][0] : 0.0, cV = a.oc.track_v ? a.rw_const[trig][1] : 0.0;
  for (int b = threadIdx.x; b < a.nbunch; b += kBlock) {
    const double *e0 = w0 + (a.bunch_kb[b] - kb0), *e1 = w1 + (a.bunch_kb[b] - kb0);
    // four partial sums per plane (steps j mod 4), so that the products
    // do not wait on one another
    double s0[4] = {0.0, 0.0, 0.0, 0.0}, s1[4] = {0.0, 0.0, 0.0, 0.0};
    int j = 0;
    for (; j + 4 <= L; j += 4) {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const double w = wt[j + u];
        s0[u] += e0[j + u] * w;
        s1[u] += e1[j + u] * w;
      }
    }
    for (; j < L; ++j) {
      s0[0] += e0[j] * wt[j];
      s1[0] += e1[j] * wt[j];
    }
    double *out = a.rw_acc + ((size_t)blk * a.nbunch + b) * 2;
    out[0] = ((s0[0] + s0[1]) + (s0[2] + s0[3])) * cH;
    out[1] = ((s1[0] + s1[1]) + (s1[2] + s1[3])) * cV;
  }
}

// The phasor of each long-range resonator around the ring, bucket h-1 .. 0
// (one pass per turn; `passes` turns for wake_phasor_init), as a warp scan
// of affine maps: a filled bucket maps V to (V prog^ncell + U_last) G_gap,
// an empty one to V G_empty (transform_weak.c:1006-1044, :911-947).
// init: wake_phasor_init semantics (start from 0, no snapshot).  Blocks
// after the first compute the resistive-wall partial sums.
// vbuf: 4 x nharm doubles, the phasor before/after each bucket.
__global__ void __launch_bounds__(kBlock) ring_scan(Args a, int passes, int init, double *vbuf) {
  extern __shared__ double dyn[];
  if (blockIdx.x > 0) {                      // resistive-wall partial sums
    rw_partial_sums(a, blockIdx.x - 1, dyn);
    return;
  }
  RingState *rs = a.rs;
  const int h = a.nharm;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __shared__ int fb_live;
  if (threadIdx.x == 0) fb_live = rs->rffb_on;
  if (!init) {
    // the snapshot of the last turn's state, one value per thread
    constexpr int nv = 3 * kMaxLr * 2;
    if (threadIdx.x < nv) (&rs->phasor_last[0][0][0])[threadIdx.x] = (&rs->phasor[0][0][0])[threadIdx.x];
    if (threadIdx.x == nv) rs->Vrf0_last = rs->Vrf0;
    if (threadIdx.x == nv + 1) rs->phai0_last = rs->phai0;
  }
  __syncthreads();
  const int chunk = (h + 31) / 32;
  const int m0 = min(lane * chunk, h), m1 = min(m0 + chunk, h);
  // the scan's per-bucket inputs, loaded once by the whole block (the scan
  // itself walks them serially per lane): bunch of each bucket and the
  // in-bucket phasor after the bunch's last bin
  double *su = dyn;                                   // h x 2
  int *sbi = reinterpret_cast<int *>(dyn + 2 * h);    // h
  for (int r = 0; r < a.nlr; ++r) {
    const LrConst &L = a.lr[r];
    __syncthreads();
    for (int i = threadIdx.x; i < h; i += kBlock) {
      const int bi = a.bucket_bunch[i];
      sbi[i] = bi;
      if (bi >= 0) {
        const double *u = a.lr_u + ((size_t)r * a.nbunch + bi) * a.ncell * 2 + 2 * (a.ncell - 1);
        su[2 * i] = u[0];
        su[2 * i + 1] = u[1];
      }
    }
    __syncthreads();
    const bool fb = L.fb && fb_live;
    const double G0 = L.gap[0] * L.gap[1], G1 = L.gap[0] * L.gap[2];
    const double E0 = L.emp[0] * L.emp[1], E1 = L.emp[0] * L.emp[2];
    const double PG0 = L.pn[0] * G0 - L.pn[1] * G1, PG1 = L.pn[0] * G1 + L.pn[1] * G0;
    double V0 = init ? 0.0 : rs->phasor[L.plane][L.l][0];
    double V1 = init ? 0.0 : rs->phasor[L.plane][L.l][1];
    for (int pass = 0; pass < passes; ++pass) {
      if (warp == 0) {
        Aff f = aff_id();
        for (int m = m0; m < m1; ++m) {
          const int i = h - m - 1;
          const int bi = sbi[i];
          Aff g;
          if (bi >= 0) {
            const double *u = su + 2 * i;
            g = Aff{PG0, PG1, u[0] * G0 - u[1] * G1, u[0] * G1 + u[1] * G0};
          } else {
            g = Aff{E0, E1, 0.0, 0.0};
          }
          f = compose(f, g);
        }
        const Aff ex = warp_exclusive_scan(f, lane);
        double v0 = V0 * ex.m0 - V1 * ex.m1 + ex.a0;
        double v1 = V0 * ex.m1 + V1 * ex.m0 + ex.a1;
        double *vs = a.lr_vs + (size_t)r * h * 2;
        for (int m = m0; m < m1; ++m) {
          const int i = h - m - 1;
          const int bi = sbi[i];
          vs[2 * i] = v0;
          vs[2 * i + 1] = v1;
          if (fb) { vbuf[4 * m] = v0; vbuf[4 * m + 1] = v1; }
          double n0, n1;
          if (bi >= 0) {
            const double *u = su + 2 * i;
            const double w0 = (v0 * L.pn[0] - v1 * L.pn[1]) + u[0];
            const double w1 = (v0 * L.pn[1] + v1 * L.pn[0]) + u[1];
            n0 = w0 * G0 - w1 * G1;
            n1 = w0 * G1 + w1 * G0;
          } else {
            n0 = v0 * E0 - v1 * E1;
            n1 = v0 * E1 + v1 * E0;
          }
          v0 = n0;
          v1 = n1;
          if (fb) { vbuf[4 * m + 2] = v0; vbuf[4 * m + 3] = v1; }
        }
        // the phasor after the last bucket sits in the lane holding m = h-1
        const int last = (h - 1) / chunk;
        V0 = __shfl_sync(0xffffffffu, v0, last);
        V1 = __shfl_sync(0xffffffffu, v1, last);
        if (lane == 0) {
          rs->phasor[L.plane][L.l][0] = V0;
          rs->phasor[L.plane][L.l][1] = V1;
        }
      }
      __syncthreads();
      if (fb) {
        // samples s = 2m (before bucket h-1-m, rotated to the beam) and
        // s = 2m+1 (after it, rotated to the next bunch); only the last
        // len samples survive in the cyclic history (feedback_rf.c:5-12)
        const int ns = 2 * h, len = a.rffb_len;
        const int count0 = rs->rffb_count;
        const int first = ns > len ? ns - len : 0;
        for (int s = first + threadIdx.x; s < ns; s += kBlock) {
          const int m = s >> 1;
          const double w0 = vbuf[4 * m + 2 * (s & 1)], w1 = vbuf[4 * m + 2 * (s & 1) + 1];
          const double *q = (s & 1) ? L.pb2b : L.p2b;
          const double vr = w0 * q[0] - w1 * q[1];
          const double vi = w0 * q[1] + w1 * q[0];
          rffb_store(a, (int)(((unsigned)count0 + (unsigned)s) % (unsigned)len), vr, vi);
        }
        __syncthreads();
        if (threadIdx.x == 0) rs->rffb_count = count0 + ns;
        __syncthreads();
      }
    }
  }
  // RF-feedback correction (worker_weakweak.c:149-162, 268-278)
  if (fb_live && a.rffb_len > 0) {
    __shared__ double sv[kBlock / 32][2];
    double s0 = 0.0, s1 = 0.0;
    for (int m = threadIdx.x; m < a.rffb_len; m += kBlock) { s0 += a.rffb_hist[2 * m]; s1 += a.rffb_hist[2 * m + 1]; }
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    if (lane == 0) { sv[warp][0] = s0; sv[warp][1] = s1; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double vs = 0.0, ps = 0.0;
      for (int w = 0; w < kBlock / 32; ++w) { vs += sv[w][0]; ps += sv[w][1]; }
      double vmbar = vs / a.rffb_len;
      const double phibar = ps / a.rffb_len;
      vmbar = vmbar * a.E0 * 1.0e3;
      const double tmp = a.rffb_vrf_design * sin(a.rffb_phi0_design) - vmbar * sin(phibar);
      const double den = a.rffb_vrf_design * cos(a.rffb_phi0_design) - vmbar * cos(phibar);
      double ph, vrf;
      if (a.rffb_kappa > 0.0 && !init) {
        // generator loop: follow the full correction (den, tmp), of this
        // turn or the last, by the fraction kappa of the difference
        const double fc = a.rffb_delay ? rs->rffb_full_prev[0] : den;
        const double fs = a.rffb_delay ? rs->rffb_full_prev[1] : tmp;
        const double gc = rs->Vrf0 * rs->cos_phai0, gs = rs->Vrf0 * rs->sin_phai0;
        const double nc = gc + a.rffb_kappa * (fc - gc), ns = gs + a.rffb_kappa * (fs - gs);
        ph = atan2(ns, nc);
        vrf = ns / sin(ph);
      } else {
        ph = atan2(tmp, den);
        vrf = tmp / sin(ph);
      }
      rs->rffb_full_prev[0] = den;
      rs->rffb_full_prev[1] = tmp;
      rs->phai0 = ph;
      rs->Vrf0 = vrf;
      rs->sin_phai0 = sin(ph);
      rs->cos_phai0 = cos(ph);
      if (init && a.rffb_off_after_init) rs->rffb_on = 0;
    }
  }
}

// ---------------------------------------------------------------- K2c

__host__ __device__ constexpr size_t bunch_wakes_smem(int nc) {
  return ((size_t)3 * (nc + 8) + 3 * (size_t)nc) * sizeof(double);
}

// One block per bunch: causal convolutions with the Green's functions,
// long-range wake per bin and the kick tables of the next particle pass.
// advance: bump the turn counter (no block of this launch reads it; the
// next particle pass does).
__global__ void __launch_bounds__(kBlock) bunch_wakes(Args a, int advance) {
  extern __shared__ double sm[];
  const int nc = a.ncell, b = blockIdx.x;
  if (advance && b == 0 && threadIdx.x == 0) {
    a.rs->turn += 1;
    if (a.rw_long) a.rs->rw_m += 1;
  }
  const int PADC = 4;
  double *fnp = sm + PADC;                    // nc + 2 PADC
  double *dipV = sm + (nc + 2 * PADC) + PADC;
  double *dipH = sm + 2 * (nc + 2 * PADC) + PADC;
  double *lr = sm + 3 * (nc + 2 * PADC);      // 3 x nc
  const double *H = a.hist + (size_t)b * 6 * nc;
  const int kb = a.bunch_kb[b];
  __shared__ int wmin[kBlock / 32], wmax[kBlock / 32];
  // the pending resistive-wall kick of this bunch: the ring scan's parts
  // summed in a fixed order
  if (a.rw_long && threadIdx.x < 64) {
    const int pl = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double v = 0.0;
    for (int k = lane; k < a.rw_nblk; k += 32) v += a.rw_acc[((size_t)k * a.nbunch + b) * 2 + pl];
    v = warp_sum(v);
    if (lane == 0) a.rw_part[(size_t)b * 2 + pl] = v;
  }
  if (!a.selffield) return;
  // first and last filled bin (transform_weak.c:633-651: the first bin
  // with particles, else nc - 1; the last one above bin 0, else 0), as a
  // minimum and a maximum over the block
  int mn = nc - 1, mx = 0;
  for (int j = threadIdx.x - PADC; j < nc + PADC; j += kBlock) {
    const bool in = j >= 0 && j < nc;
    const double f = in ? H[j] : 0.0;
    fnp[j] = f;
    dipV[j] = in ? H[nc + j] : 0.0;
    dipH[j] = in ? H[2 * nc + j] : 0.0;
    if (f > 0) {
      mn = min(mn, j);
      if (j >= 1) mx = max(mx, j);
    }
  }
  mn = __reduce_min_sync(0xffffffffu, mn);
  mx = __reduce_max_sync(0xffffffffu, mx);
  if ((threadIdx.x & 31) == 0) {
    wmin[threadIdx.x >> 5] = mn;
    wmax[threadIdx.x >> 5] = mx;
  }
  for (int j = threadIdx.x; j < 3 * nc; j += kBlock) lr[j] = 0.0;
  __syncthreads();
  int cmin = wmin[0], cmax = wmax[0];
  for (int w = 1; w < kBlock / 32; ++w) {
    cmin = min(cmin, wmin[w]);
    cmax = max(cmax, wmax[w]);
  }
  // long-range wake per bin: V_j = Vs prog^(j+1) + U_j; the reference adds
  // V_j + Ib fnp_j fac / 2 for every resonator of the plane
  // (transform_weak.c:1020-1023)
  for (int r = 0; r < a.nlr; ++r) {
    const LrConst &L = a.lr[r];
    const double *vs = a.lr_vs + (size_t)r * a.nharm * 2 + 2 * kb;
    const double *u = a.lr_u + ((size_t)r * a.nbunch + b) * nc * 2;
    const double *bb = a.lr_b + ((size_t)r * a.nbunch + b) * nc;
    const double *pw = a.lr_pw + (size_t)r * nc * 2;
    const double s0 = vs[0], s1 = vs[1];
    for (int j = threadIdx.x; j < nc; j += kBlock) {
      const double v0 = (s0 * pw[2 * j] - s1 * pw[2 * j + 1]) + u[2 * j];
      lr[L.plane * nc + j] += v0 + 0.5 * bb[j];
    }
    __syncthreads();
  }
  const double factG = a.bunch_factg[b];
  const int icellmin = cmin, icellmax = cmax;
  for (int j = threadIdx.x; j < nc; j += kBlock) {
    double GL1 = 0.0, GV = 0.0, GH = 0.0;
    if (a.planeL > 0 && j >= icellmin) {
      double Gn = 0.0;
      for (int k = j; k >= icellmin; --k) Gn += fnp[k] * a.Gl[j - k];
      GL1 = 1 * Gn;
      if (a.RsisL > 0 && j >= icellmin + 1 && j <= icellmax) {
        const double ntmoy = (0.5 * fnp[j - 1] + fnp[j] + 0.5 * fnp[j + 1]) / 2.0;
        GL1 += a.RsisL * ntmoy / (a.oc.sigma_tau * a.oc.dT);
      }
      if (a.aindL > 0 && j >= icellmin + 1 && j <= icellmax) {
        const double ntmoy0 = (0.25 * fnp[j - 3] + 0.5 * fnp[j - 2] + fnp[j - 1] + 0.5 * fnp[j] + 0.25 * fnp[j + 1]) / 2.5;
        const double ntmoy1 = (0.25 * fnp[j - 1] + 0.5 * fnp[j] + fnp[j + 1] + 0.5 * fnp[j + 2] + 0.25 * fnp[j + 3]) / 2.5;
        GL1 += (ntmoy1 - ntmoy0) / (2.0 * a.sgmatau2 * a.dTau2) * a.aindL;
      }
    }
    if (a.planeV > 0) {
      double Gn = 0.0;
      for (int k = j; k >= 0; --k) Gn += dipV[k] * a.Gv[j - k];
      GV = 1 * Gn;
    }
    if (a.planeH > 0 && j >= 1) {
      double Gn = 0.0;
      for (int k = j; k >= 0; --k) Gn += dipH[k] * a.Gh[j - k];
      GH = 1 * Gn;
    }
    double *K = a.kick + (size_t)b * 3 * nc;
    K[j] = factG * GL1 + lr[0 * nc + j];
    K[nc + j] = -factG * GV + lr[2 * nc + j];
    K[2 * nc + j] = -factG * GH + lr[1 * nc + j];
    if (a.pot != nullptr && a.pot_slot[b] >= 0) {
      // the columns of the potentials output (transform_weak.c:735-768)
      double *P = a.pot + (size_t)a.pot_slot[b] * 7 * nc;
      P[j] = __dmul_rn(factG, GL1);
      P[nc + j] = lr[0 * nc + j];
      P[2 * nc + j] = fnp[j];
      P[3 * nc + j] = __dmul_rn(-factG, GV);
      P[4 * nc + j] = dipV[j];
      P[5 * nc + j] = __dmul_rn(-factG, GH);
      P[6 * nc + j] = dipH[j];
    }
  }
}

// ------------------------------------------------------------ helpers

// Adds the pending resistive-wall kick to a copy of the coordinates (what
// the next particle pass would start from).
__global__ void add_pending_rw(Args a, double *out) {
  if (!(a.rw_long && a.rs->turn > 0)) return;
  const size_t n6 = (size_t)a.npad;
  const int b = blockIdx.y;
  const int off = a.bunch_off[b], np = a.bunch_np[b];
  const double rh = a.rw_part[(size_t)b * 2 + 0], rv = a.rw_part[(size_t)b * 2 + 1];
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < np; j += gridDim.x * blockDim.x) {
    if (a.oc.track_h) out[4 * n6 + off + j] = a.coord[4 * n6 + off + j] + rh;
    if (a.oc.track_v) out[5 * n6 + off + j] = a.coord[5 * n6 + off + j] + rv;
  }
}

// Whole-beam host layout (bunch b's 6 x np coordinates from pack[b], one
// coordinate after the other) to the device layout, and back; the export
// folds in the pending resistive-wall kick as add_pending_rw does.
__global__ void beam_import(Args a, const long *pack, const double *src) {
  const size_t n6 = (size_t)a.npad;
  const int b = blockIdx.y;
  const int off = a.bunch_off[b], np = a.bunch_np[b];
  const double *s = src + pack[b];
  for (int k = 0; k < 6; ++k)
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < np; j += gridDim.x * blockDim.x)
      a.coord[k * n6 + off + j] = s[(size_t)k * np + j];
}

__global__ void beam_export(Args a, const long *pack, double *dst) {
  const size_t n6 = (size_t)a.npad;
  const int b = blockIdx.y;
  const int off = a.bunch_off[b], np = a.bunch_np[b];
  const bool pend = a.rw_long && a.rs->turn > 0;
  double rh = 0.0, rv = 0.0;
  if (pend) {
    rh = a.rw_part[(size_t)b * 2 + 0];
    rv = a.rw_part[(size_t)b * 2 + 1];
  }
  double *d = dst + pack[b];
  for (int k = 0; k < 6; ++k) {
    const bool kick = pend && ((k == 4 && a.oc.track_h) || (k == 5 && a.oc.track_v));
    const double add = k == 4 ? rh : rv;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < np; j += gridDim.x * blockDim.x) {
      const double v = a.coord[k * n6 + off + j];
      d[(size_t)k * np + j] = kick ? v + add : v;
    }
  }
}

// Current-scan step, first half (tracking_scan_step_worker tracking.c:43-57,
// called at the end of turn rev when (rev+1) % NrevScan == 0): the bucket
// currents of the long-range source terms and the bunch currents behind
// factG (transform_weak.c:567).  It runs before the bunch reduction of that
// turn, whose long-range terms, ring scan and bunch wakes all belong to
// the next turn's self-field step.  d_ma = scan_step / Nbunch [mA],
// d_a = scan_step / (Nbunch 1e3) [A].
__global__ void scan_currents(Args a, double d_ma, double d_a, double T0, double E0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.nharm && a.bucket_bunch[i] >= 0) a.ibunch[i] = __dadd_rn(a.ibunch[i], d_ma);
  if (i < a.nbunch) {
    const double ib = __dadd_rn(a.bunch_ib[i], d_a);
    a.bunch_ib[i] = ib;
    a.bunch_factg[i] = __ddiv_rn(__dmul_rn(-T0, ib), __dmul_rn(__dmul_rn((double)a.bunch_np[i], E0), 1.0e9));
  }
}

// Current-scan step, second half, at the end of the same turn (after its
// resistive-wall sums): every dipole of the history is weighted with its
// bucket's new current, as the reference's kick reads Ibunch when it runs
// (transform_weak.c:822); the trigger count restarts
// (worker_weakweak.c:392).  rescale = 0 restarts the count only (the scan
// types that step nothing).  bi_ib: the beam-ion stage's bunch currents
// [A], or null.
__global__ void scan_rw(Args a, int rescale, double d_a, double *bi_ib) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0 && a.rw_long) a.rs->rw_m = 0;
  if (rescale && a.rw_long) {
    const long n = (long)(a.Nmlt + 2) * a.nharm;
    if (i < n) {
      const double ib = a.ibunch[i % a.nharm];
      a.rw_e[i] = a.dipole[2 * i] * ib;
      a.rw_e[n + i] = a.dipole[2 * i + 1] * ib;
    }
    if (i < a.nharm) a.rw_ib[i] = a.ibunch[i];
  }
  if (rescale && bi_ib != nullptr && i < a.nbunch) bi_ib[i] = __dadd_rn(bi_ib[i], d_a);
}

// First-particle shifts for the moment sums of the first binning pass.
__global__ void init_shift(Args a) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.nbunch) return;
  const size_t n6 = (size_t)a.npad;
  const int off = a.bunch_off[b];
  for (int k = 0; k < 6; ++k) a.shift[b * 6 + k] = a.bunch_np[b] > 0 ? a.coord[k * n6 + off] : 0.0;
}

// Matched Gaussian beam from Philox normals (replaces
// weak_bunch_normal_distribution, bunch_weak.c:86-105).
__global__ void generate_beam(Args a, uint64_t seed, const double *pos_off, const double *slope_off,
                              const double *pos_sgm, const double *slope_sgm, const double *corr) {
  const int b = blockIdx.y;
  const int np = a.bunch_np[b], off = a.bunch_off[b], kb = a.bunch_kb[b];
  const size_t n6 = (size_t)a.npad;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < np; j += gridDim.x * blockDim.x) {
    float g[5];
    turn_normals(seed, (uint32_t)j, (uint32_t)kb, 0xFFFFFFFF00000000ull, g);
    float g2[5];
    turn_normals(seed, (uint32_t)j, (uint32_t)kb, 0xFFFFFFFE00000000ull, g2);
    const float n[6] = {g[0], g[1], g[2], g[3], g[4], g2[0]};
    for (int pl = 0; pl < 3; ++pl) {
      const bool tracked = pl == 0 || (pl == 1 ? a.oc.track_h : a.oc.track_v);
      double pos = 0.0, slope = 0.0;
      if (tracked) {
        const double tmp = pos_sgm[pl] * (double)n[2 * pl];
        pos = pos_off[pl] + tmp;
        slope = slope_off[pl] + slope_sgm[pl] * (double)n[2 * pl + 1] + corr[pl] * tmp;
      }
      a.coord[(size_t)pl * n6 + off + j] = pos;
      a.coord[(size_t)(3 + pl) * n6 + off + j] = slope;
    }
  }
}

}  // namespace mbt
