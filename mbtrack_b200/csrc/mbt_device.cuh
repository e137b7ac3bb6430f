// mbt_device.cuh -- device-side data of one tracking context.
//
// HBM layout (one context):
//   coord   6 x npad doubles, structure of arrays in the reference's
//           particle_t order (types.h:215-220): xtau, x, z, eps, xp, zp.
//           Bunch b occupies [off[b], off[b]+np[b]); off[b] is a multiple
//           of 32 particles so every tile starts 256-byte aligned.
//   tiles   the particle pass works on tiles of at most `tile` particles,
//           each inside one bunch; tile t writes one partial record.
//   part    ntile x prec doubles: in-range histograms (count, sum x,
//           sum z), out-of-range counters, shifted moment sums.
//   per bunch: histograms of the last binning, kick tables for the next
//           pass, pending resistive-wall kick, moment shifts, stats.
//   ring    long-range phasors, resistive-wall dipole history, RF feedback.
#pragma once
#include <cstdint>

#define MBT_NOISE_NONE 2   // EnableQuantum = 0: no deviates drawn

namespace mbt {

constexpr int kMaxLr = 8;          // MBT_MAX_LR
constexpr int kMaxAhc = 8;         // MBT_MAX_AHC
constexpr int kPartialExtra = 20;  // 6 out-of-range values + 12 moment sums + 2 cross sums
constexpr int kBlock = 256;        // threads per block of every kernel

// Offsets inside a partial record (after the 3 x ncell histograms).
constexpr int kTrLowN = 0, kTrLowX = 1, kTrLowZ = 2;
constexpr int kTrHighN = 3, kTrHighX = 4, kTrHighZ = 5;
constexpr int kMomSum = 6;     // 6 shifted sums
constexpr int kMomSq = 12;     // 6 shifted sums of squares
constexpr int kMomCross = 18;  // shifted sums of x x' and z z'

struct Tile {
  int bunch;   // bunch index
  int start;   // first particle (global index into coord)
  int count;   // particles in this tile
  int pad;
};

// Scalars the particle map reads (transform_weak.c:35-46 and the ring
// values it uses).  Written once at set-up.
struct OpticConst {
  double damp, excite;
  double qv_pos, qv_slope, qh_pos, qh_slope;
  double E0;
  double wrf, Urad, T0, ac;
  double psiV0, psiH0, Gziz, Gzix;
  double CHH, CHV, CVH, CVV;
  double alphaV, betaV, gammaV, alphaH, betaH, gammaH;
  double dispH, disppH;
  double HC_k, m_aHC_d, m_phi_n;   // ideal HC: HC_k, (double) m_aHC, m_aHC * phi_n
  double ahc_amp[kMaxAhc];          // Vpeak / (E0 * 1e9)
  double ahc_w[kMaxAhc];            // wrf * nHC
  double ahc_phi[kMaxAhc];
  double ahc_nhc[kMaxAhc];
  int n_ahc;
  int ideal_hc;
  int amp_dep;
  int quantum;
  int track_h, track_v;
  // binning (transform_weak.c:611-613)
  double sigma_tau, nsigma, dT;
  double inv_sigma_tau, inv_dT;     // for the fast exact bin index
  double gammaL, alphaL, betaL;     // Twiss of the LON row of ring_t (0 unless set)
  int ncell;
  // sin and cos of the betatron phase advances 2 pi Q (PsiV0, PsiH0)
  double sin_psiV0, cos_psiV0, sin_psiH0, cos_psiH0;
};

// Mutable ring-wide state, device resident, read by every kernel.
struct RingState {
  long turn;           // turns completed
  double Vrf0, phai0;  // RF parameters after the feedback correction
  double sin_phai0, cos_phai0;
  int rffb_on;
  int rffb_count;
  int rw_m;            // resistive-wall trigger counter (worker_weakweak.c:254)
  double rffb_full_prev[2];   // generator loop: last turn's full-correction phasor (cos, sin parts)
  int error;           // sticky device error word (0 = ok): 1 injected deviates exhausted, 2 a
                       // particle-pass pipeline wait gave up, 4 a learned-field tensor-core wait gave up
  int trash_low, trash_high;
  double phasor[3][kMaxLr][2];
  // values of the last completed turn (what the reference holds after it)
  double Vrf0_last, phai0_last;
  double phasor_last[3][kMaxLr][2];
};

// Per long-range resonator constants (construct_wake_phasor
// transform_weak.c:976-1004).
struct LrConst {
  int plane, l;
  double Amp;          // 2 alpha Rs T0 / E0 / 1e9
  double prog[2];      // one bin
  double pn[2];        // ncell bins (product of prog, computed on the host)
  double gap[3];       // exp, cos, sin over the inter-bunch gap
  double emp[3];       // exp, cos, sin over an empty bucket
  double p2b[2], pb2b[2];
  int fb;              // this resonator drives the RF feedback
};

struct Args {
  // geometry
  int nbunch, ntile, npad, tile, prec, ncell, nharm;
  int hoff;                   // offset of the extras in a partial record: (hist_xz ? 3 : 1) * ncell
  // particles
  double *coord;
  const Tile *tiles;
  // per bunch
  const int *bunch_tile0;     // first tile of each bunch
  const int *bunch_ntile;
  const int *bunch_np;
  const int *bunch_kb;
  const int *bunch_off;
  double *bunch_ib;           // [A]; stepped by a current scan
  const double *bunch_fac;    // per long-range resonator: Amp / Np * 1e-3  [nlr][nbunch]
  double *bunch_factg;        // factG (transform_weak.c:567), follows bunch_ib
  double *part;               // ntile x prec
  double *shift;              // nbunch x 6
  double *hist;               // nbunch x 6 x ncell: fnp, dipV, dipH (clamped), ring L, H, V (dropped)
  int *cellrange;             // nbunch x 2: icellmin, icellmax
  double *kick;               // nbunch x 3 x ncell: L, V, H kick tables
  double *bi_mom;             // nbunch x 10: transverse moments for the beam-ion stage, or null
  double *pot;                // watched bunches x 7 x ncell: potential terms of the next turn, or null
  const int *pot_slot;        // nbunch: watch slot or -1
  double *rw_part;            // nbunch x 2: the pending RW kick (HOR, VER)
  double *rw_acc;             // rw_nblk x nbunch x 2: its parts, one per block of history steps
  int rw_nblk;                // blocks of the resistive-wall sums in ring_scan
  double *stats;              // stats_cap x nbunch x 12
  double *ampinv;             // stats_cap x nbunch x 6: ampinv[3], ampinv_cm[3]
  int stats_cap;
  // long-range resonators
  int nlr;
  const LrConst *lr;          // nlr
  double *lr_u;               // nlr x nbunch x ncell x 2: in-bucket phasor from 0
  double *lr_b;               // nlr x nbunch x ncell: source terms Ib fnp fac
  double *lr_vs;              // nlr x nharm x 2: phasor at bucket start
  const double *lr_pw;        // nlr x ncell x 2: prog^(j+1)
  const int *bucket_bunch;    // nharm: bunch index or -1
  double *ibunch;             // nharm: [mA], the current the next turn's wakes use
  int lr_kick[3];             // apply long-range wake in plane (kick gate)
  // self-field
  const double *Gl, *Gv, *Gh;
  int planeL, planeV, planeH;
  double RsisL, aindL, sgmatau2, dTau2;
  int hist_xz;                // dipole histograms needed
  int selffield;              // binning + kicks active
  // resistive wall
  int rw_long, Nmlt;
  double *dipole;             // (Nmlt+2) nharm x 2
  double *rw_e;               // 2 x (Nmlt+2) nharm: dipole x bucket current [mA], planar
  double *rw_ib;              // nharm: [mA], the current of this turn's resistive-wall kick
                              // (ibunch itself unless a current scan runs)
  const double *rw_rsq;       // (Nmlt+1) nharm + 1: 1 / sqrt(m T0 / h)
  double rw_const[2][2];      // [trigger halved?][plane-1]
  int triggerRW;
  // RF feedback
  int rffb_len;
  int rffb_off_after_init;
  double *rffb_hist;          // len x 2
  double rffb_vrf_design, rffb_phi0_design;
  double rffb_kappa;          // generator loop: G / (1 + G) (0: the reference's full correction)
  int rffb_delay;             // generator loop delay [turns], 0 or 1
  double E0;
  // noise
  int noise;                  // MBT_NOISE_PHILOX / _INJECTED / NONE
  uint64_t seed;
  uint32_t philox_k0[10], philox_k1[10];   // round keys of the seed
  const float *dev;           // injected deviates: turns x 5 x npad
  long dev_turn0;             // first turn held in dev
  long dev_nturn;
  // state
  RingState *rs;
  OpticConst oc;
};

}  // namespace mbt
