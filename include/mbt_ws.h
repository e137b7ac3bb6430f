/*
 * mbt_ws.h -- C ABI of the slice model (BunchModel = STRONG) with fast
 * beam-ion interaction (FBII): the weak-strong pair manager_weakstrong /
 * worker_weakstrong that mbtrack-mpi.c:139-155 dispatches to
 * (mbtrack-mpi.h:14-37), on one GPU.
 *
 * Each filled bunch is 2 Nslc + 1 longitudinal slices of fixed population
 * (npop) carrying slice centroids (xtau, xeps, xx, xp, zz, zp).  One turn:
 *
 *   1. short-range step (transformSbunch_shortrange rw_weakstrong.c:10-66):
 *      RF kick and drift of the slice xtau/xeps, slice-weighted centroids
 *      appended to each bunch's centroid history (bunch_CM_history_append
 *      bunch.c:95-115); the Bassetti-Erskine field of every slice on a
 *      Ngrid x Ngrid absolute grid, and the macro-ions each slice ionises at
 *      its local grid, pulled by the later slices of the same bunch
 *      (fbi_weakstrong_bunch fbi_weakstrong.c:45-297);
 *   2. one-turn betatron rotation of the slice centroids
 *      (transformSbunch_optic rw_weakstrong.c:194-253) and, with
 *      EnableRW_long, the long-range resistive-wall kick from the
 *      centroid histories of all bunches (transformSbunch_longrange
 *      rw_weakstrong.c:68-192);
 *   3. the ion train (fbi_weakstrong_train fbi_weakstrong.c:300-451): the
 *      ions of every bunch drift to the following bunches and are pulled
 *      by each of their slices' fields (bilinear interpolation,
 *      get_linearly_interpolated_Efields :454-580); each slice centroid
 *      takes the kick of all ions present when it passes.
 *
 * Conventions as mbt.h: 0 = ok, negative MBT_ERR_* with the message in
 * mbt_ws_last_error(); one context per host thread; the context owns its
 * device memory.  Parameters and the slicing come from the host (C,
 * libm), the turn runs on the device.
 */
#ifndef MBT_WS_H
#define MBT_WS_H

#include "mbt.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mbt_ws_params {
  /* ring and tracking fields the slice model reads: nharm, E0, T0, wrf,
     Vrf0, phai0, Urad, ac, QH0, QV0, alpha1/beta1/gamma1, Lc, beffH[0],
     beffV[0], Iring, track_plane, rw_long, Nmlt, triggerRW, nrev_tot,
     nrev_mon (see mbt_params) */
  mbt_params base;
  int    nslc;          /* [distribution] Nslc: 2 nslc + 1 slices */
  int    fbii;          /* [tracking] EnableFBII */
  int    np;            /* [distribution] Np: macroparticles the slicing counts */
  int    ngrid;         /* field grid points per transverse axis (5, bunch.c:818) */
  int    ndivs;         /* local grid steps per rms size (3, bunch.c:820) */
  double sgm_xx, sgm_zz;     /* rms sizes [mm], bunch_macroparticle_model_t units */
  double sgmatau;       /* rms duration [s] (input.c:1806) */
  double max_tau, dtau; /* slicing window and slice width in sgmatau: 7.0 and
                           0.3, fixed by read_input (input.c:179-180) */
  /* derived by mbt_ws_config_load (or the caller) */
  double agLOCx, agLOCz;     /* local grid steps [m] (bunch.c:827-831) */
  double agABSx, agABSz;     /* absolute grid steps = 2 x local (bunch.c:833-835) */
  double deltT;         /* slice duration [s] = dtau sgmatau (bunch.c:849) */
  double factBE;        /* sqrt(2 (sgm_xx^2 - sgm_zz^2)) / 1e3 [m] (worker_weakstrong.c:68) */
  double factF;         /* e / (A m_p) for CO, A = 28 (fbi_weakstrong.c:37-41) */
  double Ldmsgm;        /* CO ions one electron makes per turn (fbi_weakstrong.c:20-36) */
  double Gamma;         /* Lorentz factor 1957 E0 (input.c:1562) */
  /* [distribution] as read (input units, the set-up's values for the
     negative sigmas): sgm_xtau [ns], sgm_xeps, sgm_xx [mm], sgm_xp [mrad],
     sgm_zz [mm], sgm_zp [mrad]; the CM offsets in the same units */
  double sgm_in[6], cm_in[6];
  /* factRN of fbi_weakstrong.c:334, the factor on the ions' kick on the
     electron slices: 1e2 in the reference (its comment marks it as an
     assumption); 1 is the thin-lens kick of the ions' charge, since
     e^2 / m_e = 4 pi eps0 r_e c^2 */
  double kick_factor;
} mbt_ws_params;

/* Read an mbtrack .conf file with BunchModel = STRONG: read_conf_file,
 * setup_ring_parameters, macrop_model_setup_parameters, e_beam_setup,
 * fbii_grid_setup_parameters (bunch.c:811-851) and fbii_model_init
 * (fbi_weakstrong.c:18-43).  Fills *w and the fill pattern as
 * mbt_config_load does.  fix_rw_beff != 0 reads beffH3/beffV3 for the
 * long-range resistive wall even without EnableRW_short (the reference
 * leaves them 0 and divides by their cube, rw_weakstrong.c:101-128).
 * Refuses 2 Nslc + 1 > 49 slices (NCELL_MAX - 1, bunch.h:65), sgm_zz >=
 * sgm_xx (the field formula needs a flat beam) and an untracked
 * transverse plane. */
int mbt_ws_config_load(const char *conf_path, int fix_rw_beff, mbt_ws_params *w,
                       int *nbunch, int *bucket, double *ib_frac);

/* Slices of a bunch of np macroparticles, soa6 = xtau[np], x[np], z[np],
 * xeps[np], xp[np], zp[np] (SI): strong_generate_eCMs bunch_strong.c:
 * 59-198.  Particle jp goes to slice (int)((max_tau - xtau/sgmatau) /
 * dtau), clamped to [0, 2 nslc + 1] (the last one is an overflow cell that
 * no slice reads); npop[S] counts them; cm4[4][S] are the slice means of
 * x, xp, z, zp (0 for an empty slice); nofe[S][G][G] counts the particles
 * of each slice around its centroid on the local grid (offset rounded
 * half away from zero, clamped to +-(G-1)/2).  S = 2 nslc + 1,
 * G = ngrid. */
int mbt_ws_slice_beam(const mbt_ws_params *w, const double *soa6, int np,
                      int *npop, int *nofe, double *cm4);

/* The reference's generated bunch and bunch offsets: the np = w->np
 * particles strong_generate_eCMs draws (generate_initial_sbunch_
 * distribution2 bunch.c:226-330 for LON, HOR, VER: Irwin-Hall normals of
 * c_fnorm, glibc's rand() seeded as a fresh reference process seeds it)
 * into soa6 (layout of mbt_ws_slice_beam), then the per-bunch centroid
 * offsets of generate_initial_general_distribution2 (bunch_strong.c:13-56,
 * seed 571030, drawn on in the same generator) into off4[nbunch][4]
 * (x, xp, z, zp [m, rad]) -- what the manager adds to every slice of
 * bunch i.  off4 may be NULL. */
int mbt_ws_reference_beam(const mbt_ws_params *w, int nbunch, double *soa6, double *off4);

/* sizeof(mbt_ws_params) as compiled into the library (binding check). */
size_t mbt_ws_params_size(void);

typedef struct mbt_ws mbt_ws;

/* A device context for nbunch filled bunches in buckets bucket[] (ascending)
 * with currents ibunch[] [mA] (ring.Ibunch), all of the slicing npop / nofe
 * (the reference's manager sends bunch0's populations to every worker,
 * manager_weakstrong.c:61-66).  Slice state starts at zero. */
int mbt_ws_create(const mbt_ws_params *w, int nbunch, const int *bucket,
                  const double *ibunch, const int *npop, const int *nofe,
                  mbt_ws **out);

/* Slice state, host array [nbunch][6][S]: xtau, xeps, xx, xp, zz, zp. */
int mbt_ws_load_slices(mbt_ws *ws, const double *slices);
int mbt_ws_get_slices(mbt_ws *ws, double *slices);

/* Run nturns turns.  Host outputs (any may be NULL), per turn t and filled
 * bunch i:
 *   cm[t][i][6]   slice-weighted centroids after the short-range step:
 *                 xtau, xeps, x, xp, z, zp (the x, xp, z, zp four are the
 *                 history entry, manager_weakstrong.c:120-127);
 *   ion[t][i][2]  Nri-weighted centroid (x, y) [m] of the ion list after
 *                 bunch i's train step (writeoutCMImotions
 *                 fbi_weakstrong.c:626-646), NaN without ions;
 *   zcm[t][nharm] mean slice zz per bucket after the turn, 0 for empty
 *                 buckets (writeoutVCMmotionsPM2 :708-718);
 *   stats[m][i][18] on the turns with turn % nrev_mon == 0, in order:
 *                 pos, pos_sigma, slope, slope_sigma, ampinv, ampinv_cm,
 *                 each (LON, HOR, VER) (bunch_strong_distribution_
 *                 statistics bunch.c:516-549; 0 for untracked planes). */
int mbt_ws_run_turns(mbt_ws *ws, long nturns, double *cm, double *ion,
                     double *zcm, double *stats);

/* Field grid of filled bunch ib from the last turn, exey[S G G][2] (Ex, Ey
 * [V/m] per slice, x index, z index), and its macro-ions after the
 * intra-bunch pull, ions5[5][S G G] (Nri, x, vx, y, vy).  Either may be
 * NULL. */
int mbt_ws_bunch_fields(mbt_ws *ws, int ib, double *exey, double *ions5);

/* Device time [ms] of the last mbt_ws_run_turns call: CUDA events on the
 * context's stream around its kernels (host copies of the outputs between
 * blocks of 256 turns excluded). */
double mbt_ws_last_ms(const mbt_ws *ws);

/* Run nturns turns (no outputs) with CUDA events between the four kernels
 * of a turn; ms4 = mean device time per turn of the bunch step, the optic
 * and resistive-wall step, the ion train and the kick step. */
int mbt_ws_profile(mbt_ws *ws, long nturns, double *ms4);

/* The device's field-grid interpolation (get_linearly_interpolated_
 * Efields fbi_weakstrong.c:454-580) on filled bunch ib's field grid of the
 * last turn, slice icell, at n points (x[i], y[i]) [m]: exey[n][2]. */
int mbt_ws_interp(mbt_ws *ws, int ib, int icell, const double *x, const double *y, int n, double *exey);

/* Checkpoint of the slice state, the centroid histories and the turn
 * count (all that carries into the next turn), with a 64-bit FNV-1a
 * checksum; written beside path and renamed.  Loading checks the whole
 * file against this context before the first device write. */
int mbt_ws_checkpoint_save(mbt_ws *ws, const char *path);
int mbt_ws_checkpoint_load(mbt_ws *ws, const char *path);

/* Turns done. */
long mbt_ws_turn(const mbt_ws *ws);

/* Message of the last failing call on ws (or of the last failing create
 * when ws is NULL). */
const char *mbt_ws_last_error(const mbt_ws *ws);

void mbt_ws_destroy(mbt_ws *ws);

/* ---- output files of the slice-model manager ----------------------- */

typedef struct mbt_ws_writer mbt_ws_writer;

/* Create, in work_path, CMmotionsV.out (writeoutVCMmotionsPM2
 * fbi_weakstrong.c:672-737) and with w->fbii CMImotionsH.out /
 * CMImotionsV.out (writeoutCMImotions :583-669).  flags:
 * MBT_WRITER_OWN_AMPINV prints each bunch's own amplitude invariants in
 * the per-monitor ampinv files; by default the writer keeps the
 * reference's monitor x Nbunch + bucket history and prints entry monitor +
 * bucket as bunch_strong_writeout_ampinv does (bunch.c:645-702), 0 where
 * the reference reads past its array. */
int mbt_ws_writer_open(const char *work_path, const mbt_ws_params *w, int nbunch,
                       const int *bucket, int flags, mbt_ws_writer **out);

/* The next nturns turns, outputs of mbt_ws_run_turns: ion (needed with
 * EnableFBII), zcm, and stats for the monitor turns among them (may be
 * NULL without one): motion lines and ampinv_<P>_<turn>.dat files. */
int mbt_ws_writer_turns(mbt_ws_writer *wr, long nturns, const double *ion,
                        const double *zcm, const double *stats);

/* The generated bunch (soa6 of np particles, mbt_ws_reference_beam) into
 * the three gendst_datafile paths (LON, HOR, VER) as the manager's
 * strong_generate_eCMs writes them (bunch.c:314-331). */
int mbt_ws_writer_distribution(const mbt_ws_writer *wr, const char *const *paths,
                               const double *soa6, int np);

/* ampinv_<P>_mean.dat and cmpos_<P>_mean.dat for HOR and VER
 * (bunch_writeout_mean_ampinv_pos bunch.c:704-770), then close. */
int mbt_ws_writer_close(mbt_ws_writer *wr);

/* Message of the last failing mbt_ws_writer_* call. */
const char *mbt_ws_writer_error(void);

/* BunchModel of a .conf file: 0 WEAK, 1 STRONG, or MBT_ERR_CONFIG. */
int mbt_config_bunch_model(const char *conf_path);

#ifdef __cplusplus
}
#endif
#endif /* MBT_WS_H */
