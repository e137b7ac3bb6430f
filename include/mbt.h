/*
 * mbt.h -- C-ABI of libmbt, the B200 implementation of mbtrack's per-turn
 * weak-weak tracking loop.
 *
 * The reference (fracul/mtrack, C99 + MPI) distributes bunches over MPI
 * ranks: one manager and one worker per filled bucket, dispatched from
 * mbtrack-mpi.c:131-155 into manager_weakweak/worker_weakweak
 * (mbtrack-mpi.h:14-37).  libmbt replaces that seam: every filled bunch of
 * the ring lives in one GPU's HBM and one context runs the loop of
 * worker_weakweak.c:259-394 for all of them.
 *
 * Conventions
 *   - every entry point returns 0 on success or a negative MBT_ERR_* code;
 *     nothing calls exit(); mbt_last_error() gives a message;
 *   - host pointers unless a name says "dev"; sizes are element counts;
 *   - a context owns all of its device memory; one context per host thread
 *     (distinct contexts are independent);
 *   - particle coordinates are FP64 in the reference's particle_t order
 *     (types.h:215-220): pos.xtau [s], pos.x [m], pos.z [m],
 *     slope.xtau [rel. energy], slope.x [rad], slope.z [rad].  A "soa6"
 *     buffer holds the six coordinate arrays of one bunch back to back,
 *     each np doubles, in that order.
 *   - statistics are written per turn per bunch as 12 doubles, in the order
 *     the reference worker sends them to the manager
 *     (worker_weakweak.c:321-324): pos[3], pos_sigma[3], slope[3],
 *     slope_sigma[3], each indexed LON, HOR, VER (def.h:346-353).
 */
#ifndef MBT_H
#define MBT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MBT_OK               0
#define MBT_ERR_INVALID     -1   /* bad argument or unsupported configuration */
#define MBT_ERR_CUDA        -2   /* a CUDA runtime call failed */
#define MBT_ERR_NOMEM       -3   /* device or host allocation failed */
#define MBT_ERR_CONFIG      -4   /* configuration file missing, unreadable or incomplete */
#define MBT_ERR_STATE       -5   /* call made in the wrong order */
#define MBT_ERR_TIMEOUT     -6   /* a bounded device wait gave up */
#define MBT_ERR_NODEVICE    -7   /* no CUDA device: libmbt has no CPU path */
#define MBT_ERR_IO          -8   /* an output file could not be opened or written */

#define MBT_LON 0
#define MBT_HOR 1
#define MBT_VER 2

#define MBT_MAX_RES   32   /* short-range resonators (ring_t.resonators) */
#define MBT_MAX_LR     8   /* long-range resonators per plane */
#define MBT_MAX_AHC    8   /* active harmonic cavities */
#define MBT_MAX_NCELL 1024 /* self-field bins */

/* Noise source of the quantum-excitation term (transform_weak.c:71-75,
 * 134-138, 182-186). */
#define MBT_NOISE_PHILOX   0  /* counter-based Philox4x32-7 normals (mbt_philox.cuh) */
#define MBT_NOISE_INJECTED 1  /* deviates supplied by mbt_set_deviates() */

/*
 * Everything the per-turn loop reads, after the reference's set-up
 * (setup_ring_parameters input.c:1553-1695, setup_tracking_parameters
 * input.c:1698-1772, macrop_model_setup_parameters input.c:1775-1831,
 * selffield_model_init transform_weak.c:201-239).  Field names follow
 * ring_t / tracking_t / bunch_macroparticle_model_t / selffield_model_t.
 * Units are the reference's.
 */
typedef struct mbt_params {
  /* ring_t (types.h:60-129) */
  int    nharm;          /* harmonic number h */
  double E0;             /* [GeV] */
  double T0;             /* revolution time [s] */
  double wrf;            /* angular RF frequency [rad/s] */
  double Vrf0;           /* total RF voltage [MV] */
  double phai0;          /* synchronous phase [rad] */
  double Urad;           /* U0 / E0 */
  double De;             /* 2 T0 / taue */
  double ac;             /* momentum compaction */
  double QH0, QV0;       /* betatron tunes */
  double Gzix, Gziz;     /* normalised chromaticities */
  double CHH, CHV, CVH, CVV;   /* amplitude-dependent tune coefficients */
  int    amp_dep_qv;     /* AmpDependdQV: gates amplitude detuning in both planes */
  double beta1[3], alpha1[3], gamma1[3];   /* Twiss at the kick point, [LON,HOR,VER] */
  double dispH1, disppH1; /* horizontal dispersion and its derivative */
  double taue, taux, tauz; /* damping times [s] */
  double Lc;             /* circumference [m] */
  double rhorw;          /* wall resistivity [Ohm m] */
  double beffH[2], beffV[2], beffL[2];  /* effective radii (beffH[0] = beffH3 ...) */
  double Iring;          /* ring current [mA] */
  int    ideal_hc;       /* EnableIdealHC */
  int    m_aHC;          /* ideal HC harmonic */
  double phi_n, HC_k;    /* ideal HC phase and amplitude ratio */
  int    n_active_hc;
  double ahc_vpeak[MBT_MAX_AHC], ahc_nhc[MBT_MAX_AHC], ahc_phi[MBT_MAX_AHC];

  /* tracking_t (types.h:145-187) */
  int    track_plane[3];
  int    quantum;        /* EnableQuantum */
  int    rw_long;        /* EnableRW_long */
  int    Nmlt;           /* turns of RW memory */
  int    triggerRW;
  long   nrev_tot, nrev_mon;
  /* [scan] (input.c:807-846, setup_tracking_parameters :1710-1736):
   * scan 0 none; 1 ring current, stepped by scan_step [mA] every
   * nrev_scan turns (tracking_scan_step_worker tracking.c:43-57);
   * 2 chromaticity and 3, 4 Q factor, which the reference steps nothing
   * for (3 and 4 scale the LON resonators' Q at set-up).  Every scan
   * boundary restarts the resistive-wall trigger count
   * (worker_weakweak.c:389-393).  nrev_scan = NrevTot + 1 without a scan;
   * with one NrevTot = nscan x nrev_scan.  scan_start is the value the
   * statistics files print before the first step. */
  int    scan;
  long   nscan, nrev_scan;
  double scan_start, scan_step;

  /* bunch_macroparticle_model_t (bunch.h:22-50), SI units */
  int    np_model;       /* Np of the model (bunchModel.Np) */
  int    iseed[3];
  double pos_offset[3], slope_offset[3];
  double pos_sgm[3], slope_sgm[3];
  double correlate[3];

  /* selffield_model_t (types.h:190-209) */
  int    ncell;          /* 0 = no self-field binning */
  double nsigma;
  double dT;             /* bin width in units of sigma_tau */
  double sigma_tau;      /* [s] */
  double RsisL, aindL;   /* purely resistive / inductive longitudinal terms */
  int    planeL, planeV, planeH;   /* number of short-range wakes per plane */

  /* long-range resonators (LR_resonator_t, types.h:33-47), per plane */
  int    n_lr[3];
  double lr_Rs[3][MBT_MAX_LR];
  double lr_wr[3][MBT_MAX_LR];
  double lr_Q[3][MBT_MAX_LR];
  int    lr_init_turns;  /* Nbumax / h: turns of wake_phasor_init */

  /* rf_feedback_t (feedback_rf.h:5-12) */
  int    rffb;           /* has_rf_feedback after set-up */
  int    rffb_resonator; /* 1-based index into the LON long-range resonators */
  int    rffb_len;       /* averaging length (absolute value) */
  int    rffb_off_after_init; /* negative averaging_length: correct once, then off */
  double rffb_vrf_design, rffb_phi0_design;
  /* Generator loop (extension, no counterpart in the reference; [rf_feedback]
   * keys generator_gain, loop_delay): with gain G > 0 the generator phasor
   * V_g = Vrf0 e^{i phai0} follows the reference's full correction V_f (the
   * phasor its feedback sets every turn) through a loop of gain G and a delay
   * of loop_delay turns (0 or 1):
   *   V_g(n) = V_g(n-1) + G/(1+G) (V_f(n - delay) - V_g(n-1)),
   * after the reference's full correction at set-up.  G = 0 (the default)
   * is the reference's feedback. */
  double rffb_gain;
  int    rffb_delay;
} mbt_params;

typedef struct mbt_ctx mbt_ctx;

/* ---- configuration (C host; reference semantics of input.c) ---------- */

/* Read an mbtrack .conf file and run the reference set-up chain
 * (read_conf_file input.c:278-850, setup_ring_parameters :1553-1695,
 * macrop_model_setup_parameters :1775-1831, e_beam_setup :1289-1512,
 * setup_tracking_parameters :1698-1772).  Fills *p and the fill pattern:
 * bucket[i], ib_frac[i] for the nbunch filled buckets (arrays of at least
 * p->nharm entries, may be NULL to query nbunch only).  fix_rw_beff != 0
 * reads beffH3/beffV3 for long-range resistive wall even without
 * EnableRW_short (the reference leaves them 0, input.c:465-478).
 * Returns MBT_ERR_CONFIG (message in mbt_config_error()) for a missing or
 * malformed key, for a set-up the reference reports as failing (a
 * short-range resistive wall on bins narrower than 20 s0, a Q scan without
 * a longitudinal resonator) and for what this library does not run:
 * BunchModel = STRONG, modeHT excitation and distribution files. */
int mbt_config_load(const char *conf_path, int fix_rw_beff, mbt_params *p,
                    int *nbunch, int *bucket, double *ib_frac);

/* Short-range Green's functions for ncell bins from the [resonator_N] and
 * [wake_file_N] sections and the short-range resistive wall
 * (construct_greensfunc_resonator transform_weak.c:288-403,
 * construct_greensfunc_file :405-471, construct_greensfunc_RW :473-547),
 * plus the resulting planeL/planeV/planeH counts written back into *p.
 * Gl, Gv, Gh: arrays of p->ncell doubles (zeroed by the call). */
int mbt_config_greens(const char *conf_path, mbt_params *p,
                      double *Gl, double *Gv, double *Gh);

/* First-bin values of the short-range resistive wall for a bin of u s0
 * (replaces RW_table_LON / RW_table_TRANS, rw_table.c:310-391): the bin
 * averages of the Bane-Sands longitudinal wake and of its integral (the
 * transverse wake), dimensionless; computed by quadrature, not
 * interpolated.  u above 2000 takes the values at 2000 as the reference's
 * table does.  Either output may be NULL.  Returns 0, or -1 for u < 19.8. */
int mbt_rw_first_bin(double u, double *lon, double *trans);

/* Bunch current [A] of filled bunch i (manager_weakweak.c:74-75). */
double mbt_bunch_current(const mbt_params *p, int nbunch, double ib_frac);

/* Message of the last failing mbt_config_* call of this process. */
const char *mbt_config_error(void);

/* sizeof(mbt_params) as compiled into the library (binding check). */
size_t mbt_params_size(void);

/* What the reference's output writers read from tracking_t and
 * bunch_macroparticle_model_t (read_conf_file input.c:298-355, 547-549,
 * 811-844; e_beam_setup input.c:1316-1427; e_beam_fileread :1445-1512). */
typedef struct mbt_output_cfg {
  char   jobtitle[80];          /* [tracking] jobtitle (first word, "%s") */
  char   gendst_file[3][1024];  /* [distribution] gendst_datafile_LON/HOR/VER */
  long   nrev_potentials_out;   /* NrevPotentialsOut (0 when absent) */
  int    ampinv_out;            /* EnableAmpinv_out (0 when absent) */
  int    n_out;                 /* tracking_t.Nbunch_out */
} mbt_output_cfg;

/* Output settings of an mbtrack .conf file.  bunch_out (nharm ints, or
 * NULL) receives the bucket numbers of the output bunches
 * (tracking_t.bunch_out): the fixed lists of e_beam_setup for the named
 * fillings, the third column of a filling file. */
int mbt_config_output(const char *conf_path, mbt_output_cfg *o, int *bunch_out);

/* Initial coordinates of the bunch in `bucket`, identical to the
 * reference's generated distribution (weak_generate_bunch_distribution
 * bunch_weak.c:173-292, weak_bunch_normal_distribution :86-105): per
 * tracked plane, pos = offset + sgm g1, slope = offset + sgm g2 +
 * correlate (pos - offset), g = sum of 12 glibc rand() uniforms - 6
 * (c_fnorm bunch.c:379-405), the generator seeded with iseed[plane] +
 * bucket as one MPI worker process seeds it.  soa6: 6 np doubles (host).
 * Reentrant: bunches may be generated on several host threads. */
int mbt_reference_beam(const mbt_params *p, int bucket, int np, double *soa6);

/* ---- context --------------------------------------------------------- */

/* Make CUDA device `device` current for the calling thread: the device of
 * the contexts it creates next. */
int mbt_use_device(int device);

/* Create a tracking context on the current CUDA device.
 * nbunch filled bunches; bucket[i] is the bucket number of bunch i
 * (ascending), np[i] its macroparticle count, ib[i] its current [A].
 * Gl/Gv/Gh: short-range Green's functions (p->ncell each, or NULL when the
 * corresponding plane count is 0).  noise_mode: MBT_NOISE_*; seed keys the
 * Philox stream.  Replaces the worker set-up of worker_weakweak.c:19-255
 * for every bunch at once. */
int mbt_create(const mbt_params *p, int nbunch, const int *bucket,
               const int *np, const double *ib,
               const double *Gl, const double *Gv, const double *Gh,
               int noise_mode, uint64_t seed, mbt_ctx **out);

int mbt_destroy(mbt_ctx *ctx);

/* Message of the last failing call on this context (or of a failed
 * mbt_create when ctx is NULL). */
int mbt_last_error(const mbt_ctx *ctx, char *buf, size_t len);

/* Failure reporting.  Every kernel that waits (the particle pass's copy
 * pipeline, the learned field's tensor-core products) bounds its waits; a
 * wait that gives up sets a bit of the context's sticky device error word
 * and the kernel returns.  The next mbt_run_turns / mbt_track reads the
 * word and fails: bits 2 (particle-pass pipeline) and 4 (learned-field
 * tensor cores) give MBT_ERR_TIMEOUT, bit 1 (injected deviates exhausted)
 * MBT_ERR_STATE.  No counterpart in the reference (its MPI ranks have no
 * failure detection).
 *
 * mbt_inject_device_error ORs `bits` into that word from the host, for
 * tests of the reporting path without a device fault. */
int mbt_inject_device_error(mbt_ctx *ctx, int bits);

/* Bounded waits that nothing ends: a kernel waits on an mbarrier no thread
 * arrives at, with the two helpers the waiting kernels use (a polling wait
 * of `polls` polls, a sleeping wait of `polls` x 1000 clock cycles), and
 * reports giving up.  Returns MBT_ERR_TIMEOUT when both gave up as they
 * must, 0 if neither did and MBT_ERR_STATE if only one did (a broken
 * bound).  For tests of the bounded waits on the GPU; no counterpart in the
 * reference. */
int mbt_selftest_bounded_wait(long polls, void *stream);

/* Copy one bunch's coordinates in (host soa6, np doubles per coordinate).
 * Allowed before mbt_prepare and between runs. */
int mbt_load_particles(mbt_ctx *ctx, int ibunch, const double *soa6, int np);

/* Copy all bunches' coordinates in at once from one host buffer laid out
 * bunch after bunch, each bunch a soa6 block of np[i] particles. */
int mbt_load_all(mbt_ctx *ctx, const double *soa6_all);

/* Draw a matched Gaussian beam on the device (replaces
 * weak_bunch_normal_distribution bunch_weak.c:86-105 with a counter-based
 * generator keyed by seed, bunch and particle). */
int mbt_generate_beam(mbt_ctx *ctx, uint64_t seed);

/* Copy one bunch's coordinates out.  Any long-range resistive-wall kick
 * still pending from the last turn (it is applied at the start of the
 * next turn on the device) is included in the copy. */
int mbt_get_particles(mbt_ctx *ctx, int ibunch, double *soa6, int np);
int mbt_get_all(mbt_ctx *ctx, double *soa6_all);

/* Statistics of the current coordinates, pending resistive-wall kick
 * included: what weak_bunch_calc_statistics gives after the last turn
 * (worker_weakweak.c:396-404).  stats: nbunch x 12 doubles (host). */
int mbt_get_stats(mbt_ctx *ctx, double *stats);

/* Record, on every turn, the potential terms the following turn applies to
 * up to MBT_MAX_WATCH bunches (the reference prints them for its output
 * bunches, transform_weak.c:735-768).  Call before mbt_prepare. */
#define MBT_MAX_WATCH 16
int mbt_watch_potentials(mbt_ctx *ctx, int n, const int *ibunch);

/* Potential terms of watched bunch ibunch for the next turn: 7 x ncell
 * doubles, factG GL1 (short-range longitudinal wake potential), the
 * longitudinal long-range wake, fnp (macroparticles per bin), -factG
 * GlambdaV, dipoleV, -factG GlambdaH, dipoleH (transform_weak.c:757-763).
 * After mbt_prepare they belong to turn 0; after turn t, to turn t + 1.
 * The RF voltage and phase of that turn's potentials are mbt_get_state's. */
int mbt_get_potentials(mbt_ctx *ctx, int ibunch, double *pot);

/* Initial binning, statistics, long-range wake and RF-feedback
 * initialisation and resistive-wall history fill
 * (worker_weakweak.c:109-219).  init_stats (may be NULL) receives the
 * initial statistics, nbunch x 12 doubles. */
int mbt_prepare(mbt_ctx *ctx, double *init_stats);

/* Deviates for MBT_NOISE_INJECTED: nturns turns, each turn the bunches in
 * order, each bunch in the reference draw order (transform_weak.c:73,
 * 136-137, 184-185): np LON deviates, then 2 np VER (pos, slope per
 * particle) if VER is tracked, then 2 np HOR.  Values are the reference's
 * float Marsaglia-polar deviates.  They are consumed by the next nturns
 * turns. */
int mbt_set_deviates(mbt_ctx *ctx, const float *dev, long nturns);

/* Run nturns turns of the weak-weak loop (worker_weakweak.c:259-394) for
 * all bunches.  stats (may be NULL): nturns x nbunch x 12 doubles.  The
 * statistics are copied to stats every 8 turns on a second stream while the
 * next turns run.  A pageable stats buffer is pinned (cudaHostRegister) for
 * the duration of the call and unpinned before it returns; where pinning is
 * refused the copies go to pageable memory, which is slower.  The same holds
 * for the ampinv buffer of mbt_run_turns_ampinv. */
int mbt_run_turns(mbt_ctx *ctx, long nturns, double *stats);

/* As mbt_run_turns, also returning the amplitude invariants of every turn
 * (weak_bunch_calc_ampinv statistics.c:163-195, which the reference
 * evaluates every NrevMon turns): ampinv is nturns x nbunch x 6 doubles,
 * <gamma u^2 + 2 alpha u u' + beta u'^2> over the particles for
 * u = LON, HOR, VER, then the same of the centroid (ampinv_cm). */
int mbt_run_turns_ampinv(mbt_ctx *ctx, long nturns, double *stats, double *ampinv);

/* Same loop, but particles come from and return to host buffers in the
 * same call (one soa6 block per bunch, bunch after bunch): the call a
 * host-resident caller makes.  particles may be pinned memory. */
int mbt_track(mbt_ctx *ctx, double *particles, long nturns, double *stats);

/* Turn counter, RF parameters and long-range phasors after the last turn. */
typedef struct mbt_state {
  long   turn;
  double Vrf0, phai0;
  double phasor[3][MBT_MAX_LR][2];
  int    n_trash_low, n_trash_high;   /* summed over bunches */
} mbt_state;
int mbt_get_state(mbt_ctx *ctx, mbt_state *st);

/* Histograms of the last binning pass for bunch ibunch (ncell each):
 * clamped count/Σz/Σx (transform_weak.c:608-631) and dropped
 * count/Σx/Σz (fnp_ring_update, transform_weak.c:839-865). */
int mbt_get_histograms(mbt_ctx *ctx, int ibunch, double *fnp, double *dipV,
                       double *dipH, double *ring_lon, double *ring_hor,
                       double *ring_ver);

/* Device time of the last mbt_run_turns [ms] (CUDA events) in out[3]
 * (out[0..2] are 0), and the number of kernel launches per turn. */
int mbt_last_timing(mbt_ctx *ctx, double out[4], int *launches_per_turn);

/* Run nturns turns back to back with the four kernels of a turn launched
 * one by one and CUDA events between them; out[0..3] receive the average
 * device time per turn [ms] of the particle pass, the bunch reduction, the
 * ring-wide phasor scan and the bunch wakes. */
int mbt_profile_turns(mbt_ctx *ctx, long nturns, double out[4]);

/* Device layout: padded particle count, largest tile size, number of tiles. */
int mbt_geometry(mbt_ctx *ctx, int *npad, int *tile, int *ntile);

/* Tile sizes (particles per CTA of the particle pass, powers of two in
 * 512..8192) per bunch-size class: bunches of up to 4096, up to 32768, and
 * more macroparticles.  Each bunch is cut into ceil(np / T) equal tiles. */
int mbt_set_tiles(mbt_ctx *ctx, const int tile[3]);

/* Autotuner of the tile sizes: starting from the current sizes, tries every
 * size for each class present (one pass of coordinate descent), timing
 * trial_turns turns per candidate on the device, and keeps the fastest;
 * tile_out (may be NULL) receives them.  After mbt_prepare; the trial turns
 * are real turns of the run (their statistics are not returned). */
int mbt_autotune(mbt_ctx *ctx, int trial_turns, int tile_out[3]);

/* ---- per-step device entry points (device pointers) ------------------- */

/* Faddeeva w(z) for n points (complex_errorfunc_wofz_algo680,
 * physic.c:75-301).  flag (may be NULL) receives the reference's iflag:
 * 1 ok, -1 overflow region.  stream: a cudaStream_t or NULL. */
int mbt_wofz_dev(long n, const double *x_dev, const double *y_dev,
                 double *re_dev, double *im_dev, int *flag_dev, void *stream);

/* Bassetti-Erskine field of a flat Gaussian slice at n points
 * (fbi_weakstrong.c:154-197, replaces the inner loop of
 * fbi_weakstrong_bunch): dx, dy offsets [m] from the slice centre,
 * sgm_xx_mm > sgm_zz_mm its rms sizes [mm] (the reference's units),
 * factdq the reference's factdQ = dQ / (2 eps0 sqrt(pi) factBE c deltT)
 * (fbi_weakstrong.c:156).  Writes Ex, Ey. */
int mbt_be_field_dev(long n, const double *dx_dev, const double *dy_dev,
                     double sgm_xx_mm, double sgm_zz_mm, double factdq,
                     double *ex_dev, double *ey_dev, void *stream);

/* Statistics and in-range histograms of one bunch held in device memory:
 * weak_bunch_mean_rms (statistics.c:91-128) for every tracked plane and
 * the binning of fnp_ring_update (transform_weak.c:838-865).
 *   coord_dev  soa6 block of np particles (device)
 *   sigma_tau, nsigma, dT, ncell  binning (transform_weak.c:611-613);
 *              ncell = 0 skips the histograms
 *   stats      12 doubles (host), the order of mbt_run_turns
 *   hist_dev   3 x ncell doubles (device): count, sum x, sum z per bin
 * Block partial sums are kept in scratch device memory that this call
 * allocates and frees. */
int mbt_bunch_moments_dev(int np, const double *coord_dev, double sigma_tau,
                          double nsigma, double dT, int ncell,
                          const int track_plane[3], double *stats,
                          double *hist_dev, void *stream);

/* mbt_bunch_moments_dev for callers that must not allocate device memory
 * during the call (their memory is owned by a pool or a framework
 * allocator, or they cannot afford a possibly synchronising cudaMalloc per
 * call).  It has no counterpart in the reference.  Histogram counts are
 * identical to mbt_bunch_moments_dev's; sums and statistics agree to
 * rounding (with large ncell and np the partial sums are split over fewer
 * blocks).  The call waits for its stream and returns the statistics in
 * host memory, as mbt_bunch_moments_dev does.
 * Its scratch is a fixed 2 MiB device array inside libmbt, present on every
 * GPU that loads the library until the process exits; each call looks up
 * that array's address on the current device, and the first call on a
 * device also loads libmbt's device code there.  Calls share the array:
 * calls that overlap on the GPU race.  ncell is limited to MBT_NOALLOC_MAX_NCELL (larger values return
 * MBT_ERR_INVALID); np is not limited.  It calls no allocator. */
#define MBT_NOALLOC_MAX_NCELL 1024
int mbt_bunch_moments_dev_noalloc(int np, const double *coord_dev,
                                  double sigma_tau, double nsigma, double dT,
                                  int ncell, const int track_plane[3],
                                  double *stats, double *hist_dev,
                                  void *stream);

/* ---- beam-ion interaction (weak-strong, per macroparticle) ------------- */

/* Fast beam-ion interaction of a bunch train with the residual gas.  The
 * reference models it with rigid electron slices and one lumped
 * interaction point (fbi_weakstrong.c:45-451, factF :40, gas density
 * :20-35); this stage follows its physics with every electron
 * macroparticle kicked:
 *   - n_ip interaction points at betatron phase advances 2 pi Q k / n_ip
 *     from the kick point (same Twiss functions), each with its own ion
 *     cloud, cleared every turn by the gap after the train;
 *   - at every bunch passage each point creates ions_per_passage
 *     macro-ions from the bunch's transverse Gaussian (Philox stream keyed
 *     by seed), worth Ne sigma_ion n_gas (Lc / n_ip) / ions_per_passage ions
 *     each (n_gas = 3.22e22 P[Torr] m^-3 as fbi_weakstrong.c:24);
 *   - between passages the ions drift (fbi_weakstrong.c:370-375); each
 *     passage kicks them with the Bassetti-Erskine field of the bunch
 *     (fbi_weakstrong.c:154-197, :393-405) and kicks every electron with the
 *     field of the cloud's Gaussian (total ions, centroid, rms), the
 *     thin-lens deflection -2 pi r_e N G / gamma, mapped back to the kick
 *     point through the linear optics;
 *   - it runs after the turn's statistics, like the resistive-wall kick.
 * Both transverse planes must be tracked. */
typedef struct mbt_beam_ion {
  int      n_ip;              /* interaction points */
  int      ions_per_passage;  /* macro-ions per bunch passage per point */
  double   gas_A;             /* ion mass number */
  double   pressure;          /* [Torr] */
  double   sigma_ion;         /* ionisation cross-section [m^2] */
  uint64_t seed;              /* key of the ion-generation stream */
  int      surrogate;         /* 0: Faddeeva field, 1: MLP surrogate */
  double   audit_fraction;    /* share of surrogate fields re-evaluated exactly */
} mbt_beam_ion;

/* The [beam_ion] section of a .conf file (n_ip, ions_per_passage, gas_A,
 * pressure_nTorr, sigma_ion_Mb, seed, surrogate, audit_fraction).
 * Returns 1 when the section is absent (bi untouched), 0 when read. */
int mbt_config_beam_ion(const char *conf_path, mbt_beam_ion *bi);

/* Switch the stage on for a context; call before mbt_prepare. */
int mbt_enable_beam_ion(mbt_ctx *ctx, const mbt_beam_ion *bi);

/* The ion clouds every bunch met in the last turn: n_ip x nbunch x 5
 * doubles (ions, centroid x, centroid y [m], rms x, rms y [m] in the
 * frame of the interaction point). */
int mbt_beam_ion_clouds(mbt_ctx *ctx, double *clouds);

/* Evaluate the beam-ion fields with the trained network m (for a stage
 * enabled with surrogate = 1): inside its domain the network, outside it
 * and for a hashed audit_fraction of the evaluations also the Faddeeva
 * field.  m must outlive the context's runs. */
typedef struct mbt_mlp mbt_mlp;
int mbt_beam_ion_use_mlp(mbt_ctx *ctx, mbt_mlp *m);

/* Audit of the learned field since the last call (counters reset):
 * out[0] audited evaluations, out[1] largest and out[2] rms relative error
 * of the field vector, |F_net - F| / |F| against the Faddeeva field F,
 * out[3] evaluations outside the network's domain (Faddeeva fallback),
 * out[4] tensor-core failures. */
int mbt_beam_ion_audit(mbt_ctx *ctx, double out[5]);

/* Average device time [ms] of the beam-ion stage per turn in the last
 * mbt_profile_turns call (0 when the stage is off). */
int mbt_beam_ion_timing(mbt_ctx *ctx, double *ms_per_turn);

/* The same split by kernel: frames, ions, clouds, electron kicks [ms per
 * turn] in the last mbt_profile_turns call (zeros when the stage is off). */
int mbt_beam_ion_kernel_times(mbt_ctx *ctx, double ms_per_turn[4]);

/* Unit-charge field of an elliptic Gaussian at n points (device arrays):
 * E = lambda / (2 eps0) (gx, gy) for line density lambda.  Bassetti-
 * Erskine with w(z) for aspect ratios up to 0.995, a Gauss-Legendre
 * quadrature of the field integral closer to round; axes swapped when
 * sy > sx.  The function every beam-ion kick uses. */
int mbt_gauss_field_dev(long n, const double *dx_dev, const double *dy_dev,
                        const double *sx_dev, const double *sy_dev,
                        double *gx_dev, double *gy_dev, void *stream);

/* ---- learned field (MLP surrogate of the Bassetti-Erskine field) ------ */

/* A 3 -> 128 -> 128 -> 128 -> 2 GELU network trained on the GPU to stand
 * in for mbt_gauss_field_dev inside a = |dx|/sx < 8, b = |dy|/sy < 8,
 * r = sy/sx in [0.05, 1] (sy > sx by swapping the axes).  The dimensionless
 * field F = sx (gx, gy) is Fx = a Ex (1 + Yx/S), Fy = b Ey (1 + Yy/S),
 * S = 4096: (a Ex, b Ey) is a two-panel 8 + 8 node Gauss-Legendre rule of
 * the field integral in FP32 (within 2e-4 of the field everywhere in the
 * domain), the network maps (a, b, r) to the scaled residuals (Yx, Yy).
 * Every layer runs on the tensor cores with BF16 weights and activations
 * and FP32 accumulation: the inputs and the biases enter as BF16 pairs
 * (high and low part) through extra columns of the operands, the
 * activations are GELU in its sigmoid form, z sigma(1.702 z), evaluated in
 * FP32 with the hardware tanh and rounded to BF16.
 * Parameters (FP32 masters): MBT_MLP_NPARAM floats, W1[128][3], b1[128],
 * W2[128][128], b2, W3[128][128], b3, W4[2][128], b4[2]. */
#define MBT_MLP_NPARAM 33794

/* Network with seeded Glorot-uniform weights, zero biases. */
int mbt_mlp_create(uint64_t seed, mbt_mlp **out);
int mbt_mlp_destroy(mbt_mlp *m);
int mbt_mlp_set_params(mbt_mlp *m, const float *params);
int mbt_mlp_get_params(mbt_mlp *m, float *params);

/* Network outputs for n inputs: abr_dev n x 3 (a, b, r), t_dev n x 2. */
int mbt_mlp_forward_dev(mbt_mlp *m, long n, const float *abr_dev,
                        float *t_dev, void *stream);

/* Gradient of the loss sum((T - target)^2) / n over one batch of n inputs
 * (device arrays), into grad (host, MBT_MLP_NPARAM floats); *loss set. */
int mbt_mlp_gradient(mbt_mlp *m, int n, const float *abr_dev,
                     const float *target_dev, float *grad, double *loss);

/* The learned field at n points, in place of mbt_gauss_field_dev (same
 * arguments and units, device arrays): the network inside its domain, the
 * Faddeeva-based field outside it.  *fallbacks (host, may be NULL)
 * receives the number of points outside the domain.  No counterpart in the
 * reference: the field it replaces is fbi_weakstrong.c:154-197 with
 * physic.c:75-301. */
int mbt_mlp_field_dev(mbt_mlp *m, long n, const double *dx_dev, const double *dy_dev,
                      const double *sx_dev, const double *sy_dev, double *gx_dev,
                      double *gy_dev, long *fallbacks, void *stream);

/* Residual targets (Yx, Yy) of n inputs from the Faddeeva-based field. */
int mbt_mlp_targets_dev(long n, const float *abr_dev, float *t_dev, void *stream);

/* Train with Adam on nsamples seeded samples (half uniform over the domain,
 * half with a = 8u^2, b = 8v^2, r log-uniform; residual targets from the
 * Faddeeva-based field): `steps`
 * minibatches of `batch`, learning rate lr with cosine decay to lr/100.
 * loss_hist (may be NULL) receives the loss of every step. */
int mbt_mlp_train(mbt_mlp *m, long nsamples, int batch, int steps, float lr,
                  uint64_t seed, float *loss_hist);

/* ---- coherent tune analysis ------------------------------------------ */

/* Normalised tune spectra of nseries centroid histories on the GPU
 * (replaces the transforms of get_tunepeaks_coherent, tune.c:144-328):
 * history s at x_dev + s * ld (device, FP64), nturn turns, a power of two.
 *   plane 0 (LON): |DFT| / nturn of the nturn points, bin 0 halved,
 *     normalised by the maximum over bins 1 .. nturn/2; nturn/2 + 1 bins
 *     per history, bin 0 set to 0 (tune.c:177-197); nturn <= 4096.
 *   plane 1, 2 (HOR, VER): |FFT| of the history zero-padded to 2 nturn,
 *     bins 0 .. nturn-1 (bin j at j / (2 nturn) per turn) normalised by
 *     their maximum (tune.c:240-276); nturn <= 2048.  Bin 0 is |Re X_0|:
 *     the reference reads past its array there.
 * spec_dev receives the spectra one after the other.  A history that is 0
 * everywhere gives 0.  stream: a cudaStream_t or NULL. */
int mbt_tune_spectra_dev(const double *x_dev, long ld, int nseries, int nturn, int plane,
                         double *spec_dev, void *stream);

/* Peaks of one normalised spectrum (host; identify_tunepeaks,
 * tune.c:383-480): bins that stand 0.2 above both neighbours (pcase 1) or
 * plateaus within 0.2 that end 0.2 lower (pcase 2, at their middle),
 * refined by a parabola through three bins; value = peak bin / nrev, as
 * the reference reports it.  nrev is the history length: the search runs
 * over bins 1 .. nrev/2 - 2 (for the padded HOR / VER spectra that is the
 * lower half, and value is twice the frequency of the bin).  At most
 * min(10, max_peaks) peaks; value, ampli, pcase (may be NULL) hold
 * max_peaks entries.  A plateau of exactly equal bins gives NaN (0/0 in
 * the parabola), as in the reference.  Returns the number of peaks or
 * MBT_ERR_INVALID. */
int mbt_tune_peaks(const double *spec, long nrev, double *value, double *ampli, int *pcase,
                   int max_peaks);

/* ---- checkpoint / resume ------------------------------------------- */

/* Write the device state that carries one turn into the next to path:
 * coordinates, the histograms and kick tables of the next pass, the pending
 * resistive-wall kick, long-range phasors, the resistive-wall dipole
 * history, the RF-feedback history, the bunch currents of a scan and the
 * ring state with the turn count (the Philox noise is keyed by the turn,
 * so a resumed run draws the same deviates).  Between mbt_run_* calls.  A
 * 64-bit FNV-1a checksum closes the file; it is written beside path and
 * renamed, so a reader never sees half a file. */
int mbt_checkpoint_save(mbt_ctx *ctx, const char *path);

/* Restore a checkpoint into a prepared context created with the same fill,
 * parameters, noise mode and seed, the same watched bunches and beam-ion
 * stage: the next turn continues the saved run exactly.  The file is
 * checked whole first (checksum, record sizes, configuration key); a bad
 * or foreign file returns MBT_ERR_IO / MBT_ERR_STATE and leaves the context
 * untouched. */
int mbt_checkpoint_load(mbt_ctx *ctx, const char *path);

/* Check a checkpoint file on the host, without a device: structure and
 * checksum; *turn and *nbunch (either may be NULL) of the saved run. */
int mbt_checkpoint_check(const char *path, long *turn, int *nbunch);

/* ---- output files (C host; the reference's text formats) ------------- */

/* A writer produces, in work_path, the files the reference's manager and
 * output workers write for a weak-weak run, byte for byte in the
 * reference's formats, from the statistics libmbt returns:
 *   mean_bunch_all.dat      all-bunch turn averages (manager_weakweak.c:104-127,
 *                           :291-302; bunch_stats_fprintf bunch.c:792-804)
 *   mean_bunch_<kb>.dat     per output bunch (worker_weakweak.c:225-234,
 *                           :293-302; worker_weak_stat_output bunch.c:773-789)
 *   ampinv_<P>_<rev>.dat    every NrevMon turns when EnableAmpinv_out
 *                           (bunch_weak_writeout_ampinv bunch.c:588-640)
 *   mean_bunch_end.dat      end statistics (manager_weakweak.c:307-331)
 *   bunchbybunch_<P>.dat    centroid history (weak_bunch_writeout_tbtbbb
 *                           bunch_weak.c:343-387)
 *   ampinv_<P>_mean.dat     (weak_bunch_writeout_mean_ampinv bunch_weak.c:390-447)
 *   wakes.dat               short-range Green's functions (worker_weakweak.c:96-106)
 *   dipoles_history.dat     resistive-wall dipole ring buffer
 *                           (worker_weakweak.c:418-438)
 *   gendst_datafile_*       end distribution of the first output bunch
 *                           (weak_writeout_bunch_distribution bunch_weak.c:296-332).
 * Numbers go through the reference's printf formats, so a run whose
 * statistics agree with the reference's to printing precision gives
 * identical files.
 *
 * The reference prints the per-monitor ampinv files and ampinv_<P>_mean.dat
 * from its history array indexed by monitor number plus bucket number
 * (bunch.c:599-601, bunch_weak.c:415-428): bunch jb of monitor m shows the
 * entry m + jb (m Nbunch + jb for the mean), not its own.  By default the
 * writer reproduces that indexing, printing 0 where the reference reads
 * past its array; MBT_WRITER_OWN_AMPINV writes each bunch's own values. */
#define MBT_WRITER_OWN_AMPINV 1

typedef struct mbt_writer mbt_writer;

/* Open a writer for a run of nbunch bunches in buckets bucket[] with
 * currents ib[] [A]; bunch_out[o->n_out] lists the output buckets.
 * work_path is used as the reference uses track.work_path (joined with
 * "/"; the reference's default is "work/").  Creates mean_bunch_all.dat
 * and the mean_bunch_<kb>.dat files. */
int mbt_writer_open(const char *work_path, const mbt_params *p,
                    const mbt_output_cfg *o, const int *bunch_out,
                    int nbunch, const int *bucket, const double *ib,
                    int flags, mbt_writer **out);

/* wakes.dat from the short-range Green's functions (p->ncell each). */
int mbt_writer_wakes(mbt_writer *w, const double *Gl, const double *Gv,
                     const double *Gh);

/* Initial statistics (nbunch x 12, as mbt_prepare returns them): the
 * header and first line of every statistics file. */
int mbt_writer_begin(mbt_writer *w, const double *init_stats);

/* The next nturns turns: stats nturns x nbunch x 12 and ampinv
 * nturns x nbunch x 6 (mbt_run_turns_ampinv; ampinv may be NULL when no
 * turn of the block is a monitor turn). */
int mbt_writer_turns(mbt_writer *w, long nturns, const double *stats,
                     const double *ampinv);

/* After the last turn: end statistics (mbt_get_stats) into
 * mean_bunch_end.dat, and the history files. */
int mbt_writer_end(mbt_writer *w, const double *end_stats);

/* 1 when the reference prints the potentials of turn rev (0-based) to
 * potentials_bunch_<kb>.dat (transform_weak.c:735), else 0. */
int mbt_writer_potentials_due(const mbt_writer *w, long rev);

/* Potentials of output bunch ibunch at the start of turn rev: pot as
 * mbt_get_potentials returns it after rev turns, vrf0 [MV] and phai0 the
 * RF voltage and phase mbt_get_state reports then. */
int mbt_writer_potentials(mbt_writer *w, int ibunch, long rev,
                          const double *pot, double vrf0, double phai0);

/* The end distribution of bunch ibunch (soa6, np particles) into the
 * gendst_datafile_* files, one per tracked plane. */
int mbt_writer_distribution(mbt_writer *w, int ibunch, const double *soa6,
                            int np);

/* Close every file and free the writer. */
int mbt_writer_close(mbt_writer *w);

/* Message of the last failing mbt_writer_* call of this process. */
const char *mbt_writer_error(void);

#ifdef __cplusplus
}
#endif
#endif /* MBT_H */
