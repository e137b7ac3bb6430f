/*
 * ref_harness.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A single-process driver for the UNMODIFIED reference sources
 * (fracul/mtrack src/<file>.c, compiled from where they lie by oracle/Makefile
 * into oracle/_ref/libmbtref.so).  It replays the weak-weak worker of
 * worker_weakweak.c:19-394 for every filled bunch inside one process:
 *
 *   - each bunch gets the private state an MPI worker process would have
 *     (its own copy of ring_t with its own Ibunch and rf_feedback, its own
 *     selffield_model_t, phasor_end arrays, RW trigger counter);
 *   - the per-turn MPI_Bcast rounds (worker_weakweak.c:143,177,195,215,
 *     316,365,375,385) only copy data between ranks, so they are replaced
 *     by one shared fnp_ring/fnp_HOR/fnp_VER array and one shared dipole
 *     cyclic array that every bunch writes its own slot of; the turn is run
 *     phase by phase over all bunches so every read sees the data an MPI
 *     worker would have received;
 *   - box_muller is wrapped (-Wl,--wrap=box_muller) to record the deviates
 *     each bunch draws, so the device path can replay them.
 *
 * Exactness of the deviates: the reference keeps one glibc rand() state
 * and one cached Marsaglia deviate per PROCESS (bunch.c:407-436).  Here all
 * bunches share them, which reproduces the MPI run exactly when every
 * bunch draws an even number of deviates per turn (np even) and the
 * per-turn seeds iseed_LON+kb+rev never repeat between consecutive calls;
 * refh_init() reports otherwise through refh_deviates_exact().
 *
 * Nothing in the product links this file; tests and fixture generators
 * load it through ctypes in the build container.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "types.h"
#include "bunch.h"
#include "fbi.h"
#include "input.h"
#include "statistics.h"
#include "transform_weak.h"
#include "cyclic_array.h"
#include "feedback_rf.h"
#include "physic.h"
#include "tracking.h"

/* The globals main() owns in mbtrack-mpi.c:19-21. */
ring_t ring;
tracking_t track;
grid_t fbii_grid;

/* ------------------------------------------------------------------ */
/* deviate recorder                                                    */

double __real_box_muller(const int iseed);
static float *rec_buf = NULL;
static long rec_pos = 0, rec_cap = 0;

double __wrap_box_muller(const int iseed)
{
  double g = __real_box_muller(iseed);
  if (rec_buf != NULL && rec_pos < rec_cap)
    rec_buf[rec_pos] = (float) g;
  rec_pos++;
  return g;
}

/* ------------------------------------------------------------------ */

typedef struct worker {
  int kb;                       /* bucket */
  ring_t ring;                  /* private copy, as passed by value */
  double *ibunch;               /* private Ibunch array */
  rf_feedback_t rffb;           /* private feedback state */
  bunch_macroparticle_model_t model;
  selffield_model_t sf;
  weak_bunch_t bunch;
  double *phasor_end[3];
  int fb_off;
  int iseed;
  int m;                        /* RW trigger counter (worker_weakweak.c:254) */
  double scan_val;
} worker_t;

static int nbunch = 0;
static worker_t *W = NULL;
static e_beam_t ebeam;
static bunch_macroparticle_model_t macrop_model;
static selffield_model_t sf_model;
static double *fnp_ring = NULL, *fnp_hor = NULL, *fnp_ver = NULL;
static cyclic_array_t dipole_rw;
static FILE *devnull = NULL;
static long rev_done = 0;
static int lr_res_sizetot = 0;
static int exact_deviates = 1;
static char conf_copy[FILENAME_MAX];
/* refh_run_files: potentials file per bunch (NULL: none) and the
   amplitude invariants of the current turn, nbunch x 6 (NULL: none) */
static FILE **pot_fps = NULL;
static double *ampinv_turn = NULL;
/* Bunches [range_lo, range_hi) are generated, set up and tracked; the
   others keep zero histograms and dipoles, so a process that tracks a
   share of the ring still does the ring-wide phasor and RW work of a full
   MPI worker (used to split the CPU baseline over host cores). */
static int range_lo = 0, range_hi = 1 << 30;

void refh_set_range(int lo, int hi) { range_lo = lo; range_hi = hi; }
#define IN_RANGE(ib) ((ib) >= range_lo && (ib) < range_hi)

static void rw_beff_fix(const char *conf)
{
  /* The reference reads beffH3/beffV3 only with EnableRW_short
     (input.c:465-478); long-range RW divides by beff^3
     (transform_weak.c:801,811).  Read them whenever RW long is on. */
  FILE *fp = fopen(conf, "r");
  if (fp == NULL) return;
  int saved = config_get_fprint;
  config_get_fprint = false;
  if (track.TrackPlane[HOR]) {
    config_get_double(fp, "ring", "beffH3", &(ring.beffH[0]));
    config_get_double(fp, "ring", "beffH4", &(ring.beffH[1]));
  }
  if (track.TrackPlane[VER]) {
    config_get_double(fp, "ring", "beffV3", &(ring.beffV[0]));
    config_get_double(fp, "ring", "beffV4", &(ring.beffV[1]));
  }
  config_get_fprint = saved;
  fclose(fp);
}

int refh_init(const char *conf, const char *workdir, int fix_rw_beff)
{
  char inp[FILENAME_MAX];
  snprintf(inp, FILENAME_MAX, "%s", conf);
  snprintf(conf_copy, FILENAME_MAX, "%s", conf);
  memset(&ring, 0, sizeof(ring));
  memset(&track, 0, sizeof(track));
  memset(&ebeam, 0, sizeof(ebeam));
  memset(&macrop_model, 0, sizeof(macrop_model));
  memset(&sf_model, 0, sizeof(sf_model));
  snprintf(track.work_path, FILENAME_MAX, "%s", workdir ? workdir : "/tmp");

  /* mbtrack-mpi.c:61-81 */
  if (!read_input(inp, &ring, &track, &ebeam, &macrop_model, &sf_model))
    return -1;
  if (fix_rw_beff && track.EnableRW_long) rw_beff_fix(conf);
  setup_ring_parameters(&ring);
  macrop_model_setup_parameters(ring, track, &macrop_model);
  fbii_grid_setup_parameters(&fbii_grid, &ebeam, macrop_model);
  if (!e_beam_setup(&track, &ring, &ebeam)) return -2;
  /* mbtrack-mpi.c:148 (the result is ignored by the reference; not here) */
  if (!setup_tracking_parameters(&ring, &track, &sf_model, &macrop_model))
    return -3;

  nbunch = ebeam.Nbunch;
  W = (worker_t *) calloc(nbunch, sizeof(worker_t));
  devnull = fopen("/dev/null", "w");

  /* manager_weakweak.c:47-78: bucket numbers and currents */
  int kb, ib = 0;
  for (kb = 0; kb < (int) ring.Nharm; kb++) {
    if (!ebeam.nfFill[kb]) continue;
    double bunch_Ib = ebeam.Ib_frac[ib] * ring.Iring / (((double) ebeam.Nbunch) * FKILO);
    ring.Ibunch[kb] = bunch_Ib * FKILO;
    W[ib].kb = kb;
    W[ib].bunch.Ib = bunch_Ib;
    ib++;
  }

  lr_res_sizetot = ring.longrange_resonators_size[LON]
                 + ring.longrange_resonators_size[HOR]
                 + ring.longrange_resonators_size[VER];

  for (ib = 0; ib < nbunch; ib++) {
    worker_t *w = &W[ib];
    double Ib = w->bunch.Ib;
    w->ring = ring;
    w->ibunch = (double *) malloc(ring.Nharm * sizeof(double));
    memcpy(w->ibunch, ring.Ibunch, ring.Nharm * sizeof(double));
    w->ring.Ibunch = w->ibunch;
    if (ring.has_rf_feedback || ring.rf_feedback != NULL) {
      w->rffb = *ring.rf_feedback;
      w->ring.rf_feedback = &w->rffb;
    }
    w->model = macrop_model;
    w->model.Np = macrop_model.Np;
    w->model.fNp = (double) macrop_model.Np;
    w->sf = sf_model;
    w->scan_val = track.scan_start;
    /* worker_weakweak.c:75-79 */
    if (!weak_bunch_create(&w->bunch, &track, IN_RANGE(ib) ? macrop_model.Np : 0, Ib, w->kb, true))
      return -4;
    if (IN_RANGE(ib) && !weak_generate_bunch_distribution(&w->bunch, w->model, track.TrackPlane))
      return -5;
    w->iseed = macrop_model.iseed[LON] + w->kb;
    int pl;
    for (pl = 0; pl < 3; pl++) {
      int n = ring.longrange_resonators_size[pl];
      w->phasor_end[pl] = (double *) calloc(2 * (n > 0 ? n : 1), sizeof(double));
    }
  }
  /* Zero the coordinates of untracked planes: the reference leaves them as
     malloc garbage that is never read by the dynamics. */
  for (ib = 0; ib < nbunch; ib++) {
    unsigned jp;
    for (jp = 0; jp < W[ib].bunch.Np; jp++) {
      if (!track.TrackPlane[HOR]) { W[ib].bunch.particles[jp].pos.x = 0; W[ib].bunch.particles[jp].slope.x = 0; }
      if (!track.TrackPlane[VER]) { W[ib].bunch.particles[jp].pos.z = 0; W[ib].bunch.particles[jp].slope.z = 0; }
    }
  }

  /* deviate exactness (see header comment) */
  {
    int per = 1 + 2 * (track.TrackPlane[VER] != 0) + 2 * (track.TrackPlane[HOR] != 0);
    exact_deviates = (nbunch == 1) || ((macrop_model.Np * per) % 2 == 0);
    if (nbunch > 1 && !track.TrackPlane[HOR] && !track.TrackPlane[VER]) exact_deviates = 0;
  }
  rev_done = 0;
  return nbunch;
}

int refh_deviates_exact(void) { return exact_deviates; }
int refh_nbunch(void) { return nbunch; }

void refh_bunch_info(int *bucket, int *np, double *ib)
{
  int i;
  for (i = 0; i < nbunch; i++) {
    bucket[i] = W[i].kb;
    np[i] = (int) W[i].bunch.Np;
    ib[i] = W[i].bunch.Ib;
  }
}

static int soa_get(const weak_bunch_t *b, double *soa)
{
  unsigned n = b->Np, j;
  for (j = 0; j < n; j++) {
    const particle_t *p = &b->particles[j];
    soa[0 * n + j] = p->pos.xtau;
    soa[1 * n + j] = p->pos.x;
    soa[2 * n + j] = p->pos.z;
    soa[3 * n + j] = p->slope.xtau;
    soa[4 * n + j] = p->slope.x;
    soa[5 * n + j] = p->slope.z;
  }
  return (int) n;
}

int refh_get_particles(int ib, double *soa)
{
  if (ib < 0 || ib >= nbunch) return -1;
  return soa_get(&W[ib].bunch, soa);
}

int refh_set_particles(int ib, const double *soa)
{
  if (ib < 0 || ib >= nbunch) return -1;
  weak_bunch_t *b = &W[ib].bunch;
  unsigned n = b->Np, j;
  for (j = 0; j < n; j++) {
    particle_t *p = &b->particles[j];
    p->pos.xtau = soa[0 * n + j];
    p->pos.x = soa[1 * n + j];
    p->pos.z = soa[2 * n + j];
    p->slope.xtau = soa[3 * n + j];
    p->slope.x = soa[4 * n + j];
    p->slope.z = soa[5 * n + j];
  }
  return (int) n;
}

static void put_stats(const weak_bunch_t *b, double *out)
{
  const bunch_stats_t *s = &b->stats;
  int k;
  for (k = 0; k < 3; k++) {
    out[0 + k] = s->pos.v[k];
    out[3 + k] = s->pos_sigma.v[k];
    out[6 + k] = s->slope.v[k];
    out[9 + k] = s->slope_sigma.v[k];
  }
}

/* Worker set-up after the distribution exists: worker_weakweak.c:80-219. */
int refh_prepare(double *init_stats)
{
  int ib, i, j;
  int Nbin = sf_model.Ncell;
  for (ib = 0; ib < nbunch; ib++) {
    worker_t *w = &W[ib];
    if (!selffield_model_init(&w->sf, w->model.pos_sgm.xtau, &w->bunch)) return -1;
    if (!IN_RANGE(ib)) continue;
    if (w->ring.resonators_size > 0) construct_greensfunc_resonator(&w->sf, &w->ring);
    if (w->ring.wakefiles_size > 0) construct_greensfunc_file(&w->sf, &w->ring);
    if (track.EnableRW_short || track.EnableRW_short_LON) construct_greensfunc_RW(&w->sf, &w->ring);
    weak_bunch_calc_statistics(&w->bunch, &track);
    if (init_stats) put_stats(&w->bunch, init_stats + 12 * ib);
  }

  if (ring.longrange_resonators_size[LON] > 0) {
    fnp_ring = (double *) calloc((size_t) Nbin * ring.Nharm, sizeof(double));
    for (ib = 0; ib < nbunch; ib++) {
      worker_t *w = &W[ib];
      if (w->ring.has_rf_feedback) {
        if (w->ring.rf_feedback->len_average < 0) {
          w->ring.rf_feedback->len_average = -1 * w->ring.rf_feedback->len_average;
          w->fb_off = 1;
        }
        rffb_init(w->ring.rf_feedback);
      }
      if (IN_RANGE(ib)) fnp_ring_update(&w->ring, fnp_ring, &w->sf, &w->bunch, w->kb, LON);
    }
    for (ib = 0; ib < nbunch; ib++) {
      worker_t *w = &W[ib];
      if (!IN_RANGE(ib)) continue;
      wake_phasor_init(&w->ring, fnp_ring, &w->sf, &w->bunch, w->kb, w->phasor_end[LON], &ebeam, LON);
      if (w->ring.has_rf_feedback) {
        double vmbar, phibar;
        rffb_calc_mean_voltage_phase(w->ring.rf_feedback, &vmbar, &phibar);
        vmbar = vmbar * w->ring.E0 * FKILO;
        double tmp_numrtor = w->ring.rf_feedback->vrf_design * sin(w->ring.rf_feedback->phi0_design) - vmbar * sin(phibar);
        w->ring.phai0 = atan2(tmp_numrtor, w->ring.rf_feedback->vrf_design * cos(w->ring.rf_feedback->phi0_design) - vmbar * cos(phibar));
        w->ring.Vrf0 = tmp_numrtor / sin(w->ring.phai0);
        if (w->fb_off) w->ring.has_rf_feedback = 0;
      }
    }
  }
  if (track.TrackPlane[HOR] && ring.longrange_resonators_size[HOR] > 0) {
    fnp_hor = (double *) calloc((size_t) Nbin * ring.Nharm, sizeof(double));
    for (ib = 0; ib < nbunch; ib++)
      if (IN_RANGE(ib)) fnp_ring_update(&W[ib].ring, fnp_hor, &W[ib].sf, &W[ib].bunch, W[ib].kb, HOR);
    for (ib = 0; ib < nbunch; ib++)
      if (IN_RANGE(ib)) wake_phasor_init(&W[ib].ring, fnp_hor, &W[ib].sf, &W[ib].bunch, W[ib].kb, W[ib].phasor_end[HOR], &ebeam, HOR);
  }
  if (track.TrackPlane[VER] && ring.longrange_resonators_size[VER] > 0) {
    fnp_ver = (double *) calloc((size_t) Nbin * ring.Nharm, sizeof(double));
    for (ib = 0; ib < nbunch; ib++)
      if (IN_RANGE(ib)) fnp_ring_update(&W[ib].ring, fnp_ver, &W[ib].sf, &W[ib].bunch, W[ib].kb, VER);
    for (ib = 0; ib < nbunch; ib++)
      if (IN_RANGE(ib)) wake_phasor_init(&W[ib].ring, fnp_ver, &W[ib].sf, &W[ib].bunch, W[ib].kb, W[ib].phasor_end[VER], &ebeam, VER);
  }

  if (track.EnableRW_long > 0) {
    if (!cyclic_array_create(&dipole_rw, (track.Nmlt + 2) * ring.Nharm, 2)) return -2;
    for (ib = 0; ib < nbunch; ib++) {
      double d[2] = {W[ib].bunch.stats.pos.x, W[ib].bunch.stats.pos.z};
      cyclic_array_set(W[ib].kb, d, &dipole_rw);
    }
    for (i = 0; i < (int) ring.Nharm; i++) {
      if (!ebeam.nfFill[i]) continue;
      double *mom = cyclic_array_access(i, &dipole_rw);
      for (j = 1; j < track.Nmlt; j++) cyclic_array_set((j * ring.Nharm + i), mom, &dipole_rw);
    }
  }
  /* The reference resets the running sums after the first output
     (worker_weakweak.c:234); stats below are per turn, so reset here. */
  for (ib = 0; ib < nbunch; ib++) weak_bunch_reset_statistics(&W[ib].bunch.stats);
  return 0;
}

/* Per-turn loop, worker_weakweak.c:259-394, phase by phase over bunches.
 * stats: nturns x nbunch x 12 (may be NULL); dev: deviates recorded in
 * draw order, per turn, per bunch (may be NULL); dev_cap its length. */
int refh_run(long nturns, double *stats, float *dev, long dev_cap)
{
  long t;
  int ib, i;
  int Nbin = sf_model.Ncell;
  rec_buf = dev; rec_cap = dev ? dev_cap : 0; rec_pos = 0;
  for (t = 0; t < nturns; t++) {
    long rev = rev_done + t;
    /* 1. self-field (+ long-range phasors) */
    for (ib = 0; ib < nbunch; ib++) {
      worker_t *w = &W[ib];
      if (!IN_RANGE(ib)) continue;
      if (w->sf.PlaneL + w->sf.PlaneV + w->sf.PlaneH + lr_res_sizetot > 0)
        transform_weak_bunch_selffield(&w->bunch, w->sf, NULL, &w->ring, rev,
                                       (pot_fps && pot_fps[ib]) ? pot_fps[ib] : devnull,
                                       w->scan_val, w->kb, &ebeam, w->phasor_end[LON],
                                       w->phasor_end[HOR], w->phasor_end[VER],
                                       fnp_ring, fnp_hor, fnp_ver);
    }
    /* 2. RF feedback */
    for (ib = 0; ib < nbunch; ib++) {
      worker_t *w = &W[ib];
      if (!IN_RANGE(ib)) continue;
      if (w->ring.has_rf_feedback) {
        double vmbar, phibar;
        rffb_calc_mean_voltage_phase(w->ring.rf_feedback, &vmbar, &phibar);
        vmbar = vmbar * w->ring.E0 * FKILO;
        double tmp_numrtor = w->ring.rf_feedback->vrf_design * sin(w->ring.rf_feedback->phi0_design) - vmbar * sin(phibar);
        w->ring.phai0 = atan2(tmp_numrtor, w->ring.rf_feedback->vrf_design * cos(w->ring.rf_feedback->phi0_design) - vmbar * cos(phibar));
        w->ring.Vrf0 = tmp_numrtor / sin(w->ring.phai0);
      }
    }
    /* 3. optics, 4. statistics */
    for (ib = 0; ib < nbunch; ib++) {
      worker_t *w = &W[ib];
      if (!IN_RANGE(ib)) continue;
      transform_weak_bunch_optic(&w->bunch, &w->model, w->iseed + (int) rev, w->kb, &w->ring);
      weak_bunch_calc_statistics(&w->bunch, &track);
      if (stats) put_stats(&w->bunch, stats + (t * nbunch + ib) * 12);
      /* worker_weakweak.c:327-332: invariants before the RW kick */
      if (ampinv_turn && (rev + 1) % track.NrevMon == 0) {
        int k;
        weak_bunch_calc_ampinv(&w->bunch, &track);
        for (k = 0; k < 3; k++) {
          ampinv_turn[6 * ib + k] = w->bunch.stats.ampinv.v[k];
          ampinv_turn[6 * ib + 3 + k] = w->bunch.stats.ampinv_cm.v[k];
        }
      }
    }
    /* 5. dipole history */
    if (track.EnableRW_long > 0) {
      for (ib = 0; ib < nbunch; ib++) {
        if (!IN_RANGE(ib)) continue;
        double *mom = cyclic_array_access(-rev * ring.Nharm + W[ib].kb, &dipole_rw);
        mom[0] = W[ib].bunch.stats.pos.x;
        mom[1] = W[ib].bunch.stats.pos.z;
      }
      /* 7. long-range RW kicks */
      for (ib = 0; ib < nbunch; ib++) {
        worker_t *w = &W[ib];
        const int bpos = -rev * ring.Nharm + w->kb;
        if (!IN_RANGE(ib)) continue;
        if (track.TrackPlane[HOR])
          transform_weak_bunch_RW_longrange_cyclic(w->m, bpos, &dipole_rw, HOR, &w->model, &ebeam, &w->bunch, &w->ring, &track);
        if (track.TrackPlane[VER])
          transform_weak_bunch_RW_longrange_cyclic(w->m, bpos, &dipole_rw, VER, &w->model, &ebeam, &w->bunch, &w->ring, &track);
        w->m++;
      }
    }
    /* 8. histograms for the long-range resonators */
    for (ib = 0; ib < nbunch; ib++) {
      worker_t *w = &W[ib];
      if (!IN_RANGE(ib)) continue;
      if (ring.longrange_resonators_size[LON] > 0)
        fnp_ring_update(&w->ring, fnp_ring, &w->sf, &w->bunch, w->kb, LON);
      if (ring.longrange_resonators_size[HOR] > 0 && track.TrackPlane[HOR])
        fnp_ring_update(&w->ring, fnp_hor, &w->sf, &w->bunch, w->kb, HOR);
      if (ring.longrange_resonators_size[VER] > 0 && track.TrackPlane[VER])
        fnp_ring_update(&w->ring, fnp_ver, &w->sf, &w->bunch, w->kb, VER);
    }
    /* 9. scan */
    if ((rev + 1) % track.NrevScan == 0) {
      for (ib = 0; ib < nbunch; ib++) {
        tracking_scan_step_worker(rev, &W[ib].scan_val, &track, &W[ib].ring, &ebeam, &W[ib].bunch);
        W[ib].m = 0;
      }
    }
  }
  (void) Nbin; (void) i;
  rev_done += nturns;
  rec_buf = NULL;
  return (int) rec_pos;
}

/* RF parameters / phasors of bunch ib after the last turn. */
void refh_state(int ib, double *vrf_phi, double *phasor_lon)
{
  worker_t *w = &W[ib];
  vrf_phi[0] = w->ring.Vrf0;
  vrf_phi[1] = w->ring.phai0;
  int l;
  for (l = 0; l < (int) ring.longrange_resonators_size[LON]; l++) {
    phasor_lon[2 * l] = w->phasor_end[LON][2 * l];
    phasor_lon[2 * l + 1] = w->phasor_end[LON][2 * l + 1];
  }
}

void refh_trash(int ib, int *low, int *high)
{
  *low = W[ib].bunch.N_trash_low;
  *high = W[ib].bunch.N_trash_high;
}

void refh_greens(int ib, double *Gl, double *Gv, double *Gh, int *planes)
{
  worker_t *w = &W[ib];
  int n = w->sf.Ncell, i;
  for (i = 0; i < n; i++) {
    Gl[i] = w->sf.Gl ? w->sf.Gl[i] : 0.0;
    Gv[i] = w->sf.Gv ? w->sf.Gv[i] : 0.0;
    Gh[i] = w->sf.Gh ? w->sf.Gh[i] : 0.0;
  }
  planes[0] = w->sf.PlaneL; planes[1] = w->sf.PlaneV; planes[2] = w->sf.PlaneH;
}

/* Derived scalar parameters, as name/value pairs for parser cross-checks.
 * Returns the number of pairs written (at most cap). */
int refh_param_table(const char **names, double *values, int cap)
{
  int n = 0;
#define PUT(nm, v) do { if (n < cap) { names[n] = nm; values[n] = (double)(v); } n++; } while (0)
  PUT("nharm", ring.Nharm); PUT("E0", ring.E0); PUT("T0", ring.T0); PUT("wrf", ring.wrf);
  PUT("Vrf0", ring.Vrf0); PUT("phai0", ring.phai0); PUT("Urad", ring.Urad); PUT("De", ring.De);
  PUT("ac", ring.ac); PUT("QH0", ring.QH0); PUT("QV0", ring.QV0); PUT("Gzix", ring.Gzix);
  PUT("Gziz", ring.Gziz); PUT("CHH", ring.CHH); PUT("CHV", ring.CHV); PUT("CVH", ring.CVH);
  PUT("CVV", ring.CVV); PUT("amp_dep_qv", ring.AmpDependdQV);
  PUT("beta1_h", ring.beta1[HOR]); PUT("beta1_v", ring.beta1[VER]);
  PUT("alpha1_h", ring.alpha1[HOR]); PUT("alpha1_v", ring.alpha1[VER]);
  PUT("gamma1_h", ring.gamma1[HOR]); PUT("gamma1_v", ring.gamma1[VER]);
  PUT("dispH1", ring.dispH1); PUT("disppH1", ring.disppH1);
  PUT("taue", ring.taue); PUT("taux", ring.taux); PUT("tauz", ring.tauz);
  PUT("Lc", ring.Lc); PUT("rhorw", ring.rhorw); PUT("beffH3", ring.beffH[0]); PUT("beffV3", ring.beffV[0]);
  PUT("Iring", ring.Iring); PUT("ideal_hc", track.EnableIdealHC); PUT("m_aHC", ring.m_aHC);
  PUT("phi_n", ring.phi_n); PUT("HC_k", ring.HC_k); PUT("n_active_hc", ring.active_HC_size);
  PUT("track_h", track.TrackPlane[HOR]); PUT("track_v", track.TrackPlane[VER]);
  PUT("quantum", track.EnableQuantum); PUT("rw_long", track.EnableRW_long); PUT("Nmlt", track.Nmlt);
  PUT("triggerRW", track.triggerRW); PUT("nrev_tot", track.NrevTot); PUT("nrev_mon", track.NrevMon);
  PUT("np_model", macrop_model.Np); PUT("iseed_lon", macrop_model.iseed[LON]);
  PUT("iseed_hor", macrop_model.iseed[HOR]); PUT("iseed_ver", macrop_model.iseed[VER]);
  PUT("pos_sgm_lon", macrop_model.pos_sgm.xtau); PUT("pos_sgm_hor", macrop_model.pos_sgm.x);
  PUT("pos_sgm_ver", macrop_model.pos_sgm.z); PUT("slope_sgm_lon", macrop_model.slope_sgm.xtau);
  PUT("slope_sgm_hor", macrop_model.slope_sgm.x); PUT("slope_sgm_ver", macrop_model.slope_sgm.z);
  PUT("pos_off_lon", macrop_model.pos_offset.xtau); PUT("pos_off_hor", macrop_model.pos_offset.x);
  PUT("pos_off_ver", macrop_model.pos_offset.z); PUT("slope_off_lon", macrop_model.slope_offset.xtau);
  PUT("corr_hor", macrop_model.correlate.x); PUT("corr_ver", macrop_model.correlate.z);
  PUT("ncell", sf_model.Ncell); PUT("nsigma", sf_model.Nsigma);
  PUT("RsisL", sf_model.RsisL); PUT("aindL", sf_model.aindL);
  PUT("n_lr_lon", ring.longrange_resonators_size[LON]); PUT("n_lr_hor", ring.longrange_resonators_size[HOR]);
  PUT("n_lr_ver", ring.longrange_resonators_size[VER]);
  PUT("lr_init_turns", ring.h > 0 ? (double)(int)(ring.Nbumax / ring.h) : 0.0);
  PUT("rffb", ring.has_rf_feedback);
  if (ring.rf_feedback != NULL && ring.has_rf_feedback) {
    PUT("rffb_resonator", ring.rf_feedback->lr_resonator);
    PUT("rffb_len", ring.rf_feedback->len_average);
    PUT("rffb_vrf_design", ring.rf_feedback->vrf_design);
    PUT("rffb_phi0_design", ring.rf_feedback->phi0_design);
  }
  PUT("nbunch", ebeam.Nbunch);
  {
    int l;
    static const char *wrn[4] = {"lr_wr_lon_0", "lr_wr_lon_1", "lr_wr_lon_2", "lr_wr_lon_3"};
    for (l = 0; l < (int) ring.longrange_resonators_size[LON] && l < 4; l++)
      PUT(wrn[l], ring.longrange_resonators[LON][l].wr);
  }
#undef PUT
  return n;
}

/* ------------------------------------------------------------------ */
/* The reference's parsed and derived state as the product's parameter
 * block (include/mbt.h), so oracle and device path can be driven from
 * exactly what the reference computed. */
#include "mbt.h"

int refh_fill_params(mbt_params *p)
{
  int pl, l;
  memset(p, 0, sizeof(*p));
  p->nharm = (int) ring.Nharm;
  p->E0 = ring.E0; p->T0 = ring.T0; p->wrf = ring.wrf; p->Vrf0 = ring.Vrf0;
  p->phai0 = ring.phai0; p->Urad = ring.Urad; p->De = ring.De; p->ac = ring.ac;
  p->QH0 = ring.QH0; p->QV0 = ring.QV0; p->Gzix = ring.Gzix; p->Gziz = ring.Gziz;
  p->CHH = ring.CHH; p->CHV = ring.CHV; p->CVH = ring.CVH; p->CVV = ring.CVV;
  p->amp_dep_qv = ring.AmpDependdQV ? 1 : 0;
  for (pl = 0; pl < 3; pl++) {
    p->beta1[pl] = ring.beta1[pl]; p->alpha1[pl] = ring.alpha1[pl]; p->gamma1[pl] = ring.gamma1[pl];
  }
  p->dispH1 = ring.dispH1; p->disppH1 = ring.disppH1;
  p->taue = ring.taue; p->taux = ring.taux; p->tauz = ring.tauz;
  p->Lc = ring.Lc; p->rhorw = ring.rhorw;
  p->beffH[0] = ring.beffH[0]; p->beffH[1] = ring.beffH[1];
  p->beffV[0] = ring.beffV[0]; p->beffV[1] = ring.beffV[1];
  p->beffL[0] = ring.beffL[0]; p->beffL[1] = ring.beffL[1];
  p->Iring = ring.Iring;
  p->ideal_hc = track.EnableIdealHC; p->m_aHC = ring.m_aHC; p->phi_n = ring.phi_n; p->HC_k = ring.HC_k;
  p->n_active_hc = (int) ring.active_HC_size;
  for (l = 0; l < p->n_active_hc && l < MBT_MAX_AHC; l++) {
    p->ahc_vpeak[l] = ring.active_HC[l].Vpeak; p->ahc_nhc[l] = ring.active_HC[l].nHC;
    p->ahc_phi[l] = ring.active_HC[l].phi_aHC;
  }
  for (pl = 0; pl < 3; pl++) p->track_plane[pl] = track.TrackPlane[pl];
  p->quantum = track.EnableQuantum; p->rw_long = track.EnableRW_long; p->Nmlt = track.Nmlt;
  p->triggerRW = track.triggerRW; p->nrev_tot = track.NrevTot; p->nrev_mon = track.NrevMon;
  p->scan = track.scan; p->nscan = track.Nscan; p->nrev_scan = track.NrevScan;
  p->scan_start = track.scan_start; p->scan_step = track.scan_step;
  p->np_model = macrop_model.Np;
  for (pl = 0; pl < 3; pl++) {
    p->iseed[pl] = macrop_model.iseed[pl];
    p->pos_offset[pl] = macrop_model.pos_offset.v[pl];
    p->slope_offset[pl] = macrop_model.slope_offset.v[pl];
    p->pos_sgm[pl] = macrop_model.pos_sgm.v[pl];
    p->slope_sgm[pl] = macrop_model.slope_sgm.v[pl];
    p->correlate[pl] = macrop_model.correlate.v[pl];
  }
  p->ncell = sf_model.Ncell; p->nsigma = sf_model.Nsigma;
  p->dT = sf_model.Ncell > 0 ? 2.0 * sf_model.Nsigma / ((double) sf_model.Ncell - 1) : 0.0;
  p->sigma_tau = macrop_model.pos_sgm.xtau;
  p->RsisL = sf_model.RsisL; p->aindL = sf_model.aindL;
  if (nbunch > 0) {
    p->planeL = W[0].sf.PlaneL; p->planeV = W[0].sf.PlaneV; p->planeH = W[0].sf.PlaneH;
    p->dT = W[0].sf.dT;
    p->sigma_tau = W[0].sf.sigma_tau;
  }
  for (pl = 0; pl < 3; pl++) {
    p->n_lr[pl] = (int) ring.longrange_resonators_size[pl];
    for (l = 0; l < p->n_lr[pl] && l < MBT_MAX_LR; l++) {
      p->lr_Rs[pl][l] = ring.longrange_resonators[pl][l].Rs;
      p->lr_wr[pl][l] = ring.longrange_resonators[pl][l].wr;
      p->lr_Q[pl][l] = ring.longrange_resonators[pl][l].Qfactor;
    }
  }
  p->lr_init_turns = ring.h > 0 ? (int) (ring.Nbumax / ring.h) : 0;
  p->rffb = ring.has_rf_feedback;
  if (ring.has_rf_feedback && ring.rf_feedback) {
    p->rffb_resonator = ring.rf_feedback->lr_resonator;
    p->rffb_len = ring.rf_feedback->len_average < 0 ? -ring.rf_feedback->len_average : ring.rf_feedback->len_average;
    p->rffb_off_after_init = ring.rf_feedback->len_average < 0;
    p->rffb_vrf_design = ring.rf_feedback->vrf_design;
    p->rffb_phi0_design = ring.rf_feedback->phi0_design;
  }
  return 0;
}

/* weak_bunch_calc_ampinv of the reference on bunch ib. */
void refh_ampinv(int ib, double *out6)
{
  int k;
  weak_bunch_calc_ampinv(&W[ib].bunch, &track);
  for (k = 0; k < 3; k++) {
    out6[k] = W[ib].bunch.stats.ampinv.v[k];
    out6[3 + k] = W[ib].bunch.stats.ampinv_cm.v[k];
  }
}

/* ------------------------------------------------------------------ */
/* A whole run with the reference's output files                       */

/* The rest of the run (after refh_prepare) writing, into track.work_path,
 * the files of manager_weakweak (mean_bunch_all.dat, ampinv_<P>_<rev>.dat,
 * mean_bunch_end.dat, bunchbybunch_<P>.dat, ampinv_<P>_mean.dat) and of the
 * output workers (wakes.dat, mean_bunch_<kb>.dat, potentials_bunch_<kb>.dat,
 * dipoles_history.dat, the distribution files).  Every number is printed by
 * the reference's own functions (bunch_stats_fprintf, worker_weak_stat_
 * output, bunch_weak_writeout_ampinv, weak_bunch_writeout_tbtbbb,
 * weak_bunch_writeout_mean_ampinv, weak_writeout_bunch_distribution, and
 * transform_weak_bunch_selffield for the potentials) from the reference's
 * accumulators; the manager/worker control flow around them follows
 * manager_weakweak.c:104-349 and worker_weakweak.c:96-106, 225-302,
 * 394-438, with the MPI messages replaced by reads of the bunch state.
 * Where several output workers write one file the reference keeps the
 * last one to finish; here the first output bunch's content is kept.
 *
 * stats: NrevTot x nbunch x 12, ampinv: NrevTot x nbunch x 6 (monitor
 * turns filled), vrfphi: NrevTot x nbunch x 2 (RF voltage and phase at the
 * start of each turn), end_stats: nbunch x 12.  Returns 0 or < 0. */
int refh_run_files(double *stats, double *ampinv, double *vrfphi, double *end_stats)
{
  const long tot = track.NrevTot, mon = track.NrevMon;
  const int H = (int) ring.Nharm;
  int ib, pl;
  long rev, nstat = 0;
  long *nstat_w = (long *) calloc(nbunch, sizeof(long));
  double *sv_w = (double *) calloc(nbunch, sizeof(double));
  FILE **out_fp = (FILE **) calloc(nbunch, sizeof(FILE *));
  char fn[FILENAME_MAX];
  bunch_CM_history_weak_t cmhist;
  bunch_stats_t allstats;
  double *scan_val_hist = (double *) calloc(tot / mon + track.Nscan + 1, sizeof(double));
  double scan_val = track.scan_start;
  int m = 0;
  FILE *all_fp;

  pot_fps = (FILE **) calloc(nbunch, sizeof(FILE *));
  bunch_CM_history_weak_init(&cmhist, (int) (tot / mon * nbunch));

  /* manager_weakweak.c:104-127 */
  snprintf(fn, FILENAME_MAX, "%s/mean_bunch_all.dat", track.work_path);
  all_fp = fopen(fn, "w+");
  if (!all_fp) return -1;
  weak_bunch_reset_statistics(&allstats);
  for (ib = 0; ib < nbunch; ib++) weak_bunch_add_statistics(&allstats, &W[ib].bunch.stats);
  weak_bunch_update_statistics(&allstats, nbunch);
  fprintf(all_fp, " # bunch statistics, AVEraged over all bunches & turns, Ib = %g A ;\n", W[0].bunch.Ib);
  fprintf(all_fp, " # turn - scan_var - AVE_CM_LON - SIG_CM_LON - AVE_delE_LON - SIG_delE_LON -  AVE_sigmaL_LON - SIG_sigmaL_LON - AVE_sigmaE_LON - SIG_sigmaE_LON... (_HOR) ... (_VER)\n # ");
  bunch_stats_fprintf(all_fp, -100, &allstats, 0.0);
  fprintf(all_fp, "\n");
  weak_bunch_reset_statistics(&allstats);

  /* output workers: worker_weakweak.c:96-106, 225-249 */
  for (ib = 0; ib < nbunch; ib++) {
    worker_t *w = &W[ib];
    int nc;
    if (w->bunch.kb_out != 1) continue;
    snprintf(fn, FILENAME_MAX, "%s/wakes.dat", track.work_path);
    FILE *wf = fopen(fn, "w+");
    if (wf) {
      fprintf(wf, "# bin (%.2e s)   total wake L     - V -      - H -\n", w->sf.dT * w->sf.sigma_tau);
      for (nc = 0; nc < w->sf.Ncell; nc++)
        fprintf(wf, "%d  %e   %e   %e\n", nc, w->sf.Gl[nc], w->sf.Gv[nc], w->sf.Gh[nc]);
      fclose(wf);
    }
    snprintf(fn, FILENAME_MAX, "%s/mean_bunch_%d.dat", track.work_path, w->kb);
    out_fp[ib] = fopen(fn, "w+");
    if (!out_fp[ib]) return -1;
    worker_weak_stat_output(out_fp[ib], &w->bunch.stats, w->bunch.Ib);
    weak_bunch_reset_statistics(&w->bunch.stats);
    if (track.NrevPotentialsOut <= track.NrevTot) {
      snprintf(fn, FILENAME_MAX, "%s/potentials_bunch_%d.dat", track.work_path, w->kb);
      pot_fps[ib] = fopen(fn, "w+");
      if (!pot_fps[ib]) return -1;
      fprintf(pot_fps[ib], " # potentials and distributions, Ib = %g A ;\n", w->bunch.Ib);
      fprintf(pot_fps[ib], " # rev  scan_val         tau         LON_wake_pot       HC_pot        rf_pot      active_cav      ideal_HC        bunch_shape");
      if (w->sf.PlaneV > 0) fprintf(pot_fps[ib], "     VER_wake_pot     VER_dipole_mom");
      if (w->sf.PlaneH > 0) fprintf(pot_fps[ib], "     HOR_wake_pot     HOR_dipole_mom");
      fprintf(pot_fps[ib], "\n");
    }
  }

  ampinv_turn = (double *) calloc((size_t) nbunch * 6, sizeof(double));
  for (rev = 0; rev < tot; rev++) {
    double *st = stats + (size_t) rev * nbunch * 12;
    for (ib = 0; ib < nbunch; ib++) {
      vrfphi[((size_t) rev * nbunch + ib) * 2] = W[ib].ring.Vrf0;
      vrfphi[((size_t) rev * nbunch + ib) * 2 + 1] = W[ib].ring.phai0;
    }
    /* the workers print before their scan step (worker_weakweak.c:296-302
       then :388-393); refh_run makes the step within the turn */
    for (ib = 0; ib < nbunch; ib++) sv_w[ib] = W[ib].scan_val;
    refh_run(1, st, NULL, 0);
    /* workers: worker_weakweak.c:290-302 */
    for (ib = 0; ib < nbunch; ib++) {
      if (W[ib].bunch.kb_out != 1) continue;
      nstat_w[ib]++;
      if (nstat_w[ib] % mon == 0 || (rev + 1) % track.NrevScan == 0) {
        weak_bunch_update_statistics(&W[ib].bunch.stats, nstat_w[ib]);
        bunch_stats_fprintf(out_fp[ib], rev, &W[ib].bunch.stats, sv_w[ib]);
        weak_bunch_reset_statistics(&W[ib].bunch.stats);
        nstat_w[ib] = 0;
      }
    }
    /* manager: manager_weakweak.c:235-302 */
    for (ib = 0; ib < nbunch; ib++) {
      bunch_stats_t *bs = &W[ib].bunch.stats;
      if ((rev + 1) % mon == 0) {
        const long irevmon = rev / mon;
        int k;
        for (k = 0; k < 3; k++) {
          cmhist.ampinv[irevmon * nbunch + ib].v[k] = ampinv_turn[6 * ib + k];
          cmhist.ampinv_cm[irevmon * nbunch + ib].v[k] = ampinv_turn[6 * ib + 3 + k];
          ampinv[((size_t) rev * nbunch + ib) * 6 + k] = ampinv_turn[6 * ib + k];
          ampinv[((size_t) rev * nbunch + ib) * 6 + 3 + k] = ampinv_turn[6 * ib + 3 + k];
        }
        cmhist.cm[irevmon * nbunch + ib] = bs->pos;
      }
      weak_bunch_add_statistics(&allstats, bs);
    }
    nstat++;
    if (nstat % mon == 0 || (rev + 1) % track.NrevScan == 0) {
      nstat *= nbunch;
      weak_bunch_update_statistics(&allstats, nstat);
      scan_val_hist[m] = scan_val;
      m++;
      if (track.EnableAmpinv_out) bunch_weak_writeout_ampinv(rev, rev / mon, &cmhist, ebeam);
      bunch_stats_fprintf(all_fp, rev, &allstats, scan_val);
      weak_bunch_reset_statistics(&allstats);
      nstat = 0;
    }
    /* manager_weakweak.c:287-288.  tracking_scan_step_manager also adds
       to bunches[i].Ib for every filled bucket i < Nharm of an array of
       Nbunch bunches (out of bounds for a partial fill) and the manager
       prints those currents only without a scan, so only its scan value
       is kept here. */
    if ((rev + 1) % track.NrevScan == 0 && rev > 0 && track.scan == 1) {
      ring.Iring += track.scan_step;
      scan_val = ring.Iring;
    }
  }
  free(ampinv_turn);
  ampinv_turn = NULL;

  /* end statistics: worker_weakweak.c:396-404, manager_weakweak.c:301-331
     (the file only without a scan; end_stats are filled either way) */
  FILE *end_fp = NULL;
  if (track.scan == 0) {
    snprintf(fn, FILENAME_MAX, "%s/mean_bunch_end.dat", track.work_path);
    end_fp = fopen(fn, "w+");
    if (!end_fp) return -1;
    fprintf(end_fp, " # bunch statistics end of run, turns = %i; Ib = %g A ;\n", (int) tot, W[0].bunch.Ib);
    fprintf(end_fp, " # bunch_num    CM    bunch_length    energy_dev    energy_spread;\n");
  }
  for (ib = 0; ib < nbunch; ib++) {
    bunch_stats_t *bs = &W[ib].bunch.stats;
    weak_bunch_calc_statistics(&W[ib].bunch, &track);
    put_stats(&W[ib].bunch, end_stats + 12 * ib);
    if (end_fp)
      fprintf(end_fp, " %d     %e    %e    %e    %e\n", W[ib].kb, bs->pos.xtau, bs->pos_sigma.xtau, bs->slope.xtau, bs->slope_sigma.xtau);
  }
  if (end_fp) fclose(end_fp);

  /* output workers, last bunch first so the first one's files remain:
     worker_weakweak.c:407-438 */
  for (ib = nbunch - 1; ib >= 0; ib--) {
    worker_t *w = &W[ib];
    if (w->bunch.kb_out != 1) continue;
    weak_writeout_bunch_distribution(&w->bunch, w->model, LON, w->model.nGen[LON]);
    if (track.TrackPlane[HOR]) weak_writeout_bunch_distribution(&w->bunch, w->model, HOR, w->model.nGen[HOR]);
    if (track.TrackPlane[VER]) weak_writeout_bunch_distribution(&w->bunch, w->model, VER, w->model.nGen[VER]);
    if (track.EnableRW_long) {
      int i, j;
      snprintf(fn, FILENAME_MAX, "%s/dipoles_history.dat", track.work_path);
      FILE *df = fopen(fn, "w+");
      if (!df) return -1;
      fprintf(df, " # history of dipole moments at rev = %i; Ib = %g A ;\n", (int) tot, w->bunch.Ib);
      fprintf(df, " # Nhist  kb   rev   dipole_HOR    dipole_VER\n");
      for (j = 0; j < track.Nmlt; j++)
        for (i = 0; i < H; i++) {
          const double *mom = cyclic_array_get((j * H + i), &dipole_rw);
          fprintf(df, " %d    %d    %d           %e    %e \n", j * H + i, i, j, mom[0], mom[1]);
        }
      fclose(df);
    }
  }
  for (ib = 0; ib < nbunch; ib++) {
    if (out_fp[ib]) fclose(out_fp[ib]);
    if (pot_fps[ib]) fclose(pot_fps[ib]);
  }
  free(pot_fps);
  pot_fps = NULL;

  /* manager_weakweak.c:333-345 */
  weak_bunch_writeout_tbtbbb(tot, mon, &cmhist, ebeam, LON, scan_val_hist);
  for (pl = HOR; pl <= VER; pl++)
    if (track.TrackPlane[pl]) {
      weak_bunch_writeout_mean_ampinv(tot, mon, &cmhist, ebeam, (plane_t) pl, scan_val_hist);
      weak_bunch_writeout_tbtbbb(tot, mon, &cmhist, ebeam, (plane_t) pl, scan_val_hist);
    }
  fclose(all_fp);
  bunch_CM_history_weak_destroy(&cmhist);
  free(scan_val_hist);
  free(nstat_w);
  free(sv_w);
  free(out_fp);
  return 0;
}

/* Output settings and output buckets as the reference's set-up made them. */
int refh_output_info(long *nrev_scan, long *nrev_pot, int *ampinv_out, int *bunch_out, int cap)
{
  int i;
  *nrev_scan = track.NrevScan;
  *nrev_pot = track.NrevPotentialsOut;
  *ampinv_out = track.EnableAmpinv_out;
  for (i = 0; i < track.Nbunch_out && i < cap; i++) bunch_out[i] = track.bunch_out[i];
  return track.Nbunch_out;
}

/* ------------------------------------------------------------------ */
/* Coherent tune analysis (tune.c) of the reference on given data      */

#include "tune.h"

/* tune.c:144, not declared in tune.h */
int get_tunepeaks_coherent(tuneC_t *tune, plane_t pl, FILE *fp);

static int tune_setup(tuneC_t *T, int Nt)
{
  const int N = 1 << Nt;
  memset(T, 0, sizeof(*T));
  T->Nt = Nt;
  T->xt_tune_C = (double *) calloc(N, sizeof(double));
  T->xx_tune_C = (double *) calloc(N, sizeof(double));
  T->xz_tune_C = (double *) calloc(N, sizeof(double));
  T->tunes = (double *) calloc(N, sizeof(double));
  T->pk_numbr = (unsigned *) calloc(N > 3 ? N : 3, sizeof(unsigned));
  T->pk_value = (double *) calloc((size_t) (N > 3 ? N : 3) * 10, sizeof(double));
  T->pk_ampli = (double *) calloc((size_t) (N > 3 ? N : 3) * 10, sizeof(double));
  return T->xt_tune_C && T->xx_tune_C && T->xz_tune_C && T->tunes && T->pk_numbr && T->pk_value && T->pk_ampli
             ? 0 : -1;
}

static int tune_collect(tuneC_t *T, int pl, FILE *fp, char *text, double *value, double *ampli, int cap)
{
  int n = 0, i;
  const char *p;
  fclose(fp);
  for (p = text; *p; p++)
    if (p[0] == '\n' && p[1] == ' ') n++;      /* one line " rev Pl i pcase value ampli" per peak */
  for (i = 0; i < n && i < cap; i++) {
    value[i] = T->pk_value[pl * 10 + i];
    ampli[i] = T->pk_ampli[pl * 10 + i];
  }
  free(T->xt_tune_C); free(T->xx_tune_C); free(T->xz_tune_C); free(T->tunes);
  free(T->pk_numbr); free(T->pk_value); free(T->pk_ampli);
  return n;
}

/* identify_tunepeaks (tune.c:383-480) on a normalised spectrum cofu of
 * nrev/2 + 1 bins; the printed lines go to text.  Returns the peak count. */
int refh_tune_identify(const double *cofu, long nrev, int pl, double *value, double *ampli, int cap, char *text,
                       int textcap)
{
  tuneC_t T;
  FILE *fp;
  double *buf;
  if (tune_setup(&T, 2)) return -1;
  buf = (double *) malloc((size_t) (nrev / 2 + 2) * sizeof(double));
  memcpy(buf, cofu, (size_t) (nrev / 2 + 1) * sizeof(double));
  memset(text, 0, textcap);
  fp = fmemopen(text, textcap - 1, "w");
  identify_tunepeaks(&T, buf, (unsigned) pl, (unsigned long) nrev, fp);
  free(buf);
  return tune_collect(&T, pl, fp, text, value, ampli, cap);
}

/* The LON branch of get_tunepeaks_coherent (tune.c:175-233) on a centroid
 * history of 2^Nt turns. */
int refh_tune_lon(const double *xt, int Nt, double *value, double *ampli, int cap, char *text, int textcap)
{
  tuneC_t T;
  FILE *fp;
  if (tune_setup(&T, Nt)) return -1;
  memcpy(T.xt_tune_C, xt, (size_t) (1 << Nt) * sizeof(double));
  memset(text, 0, textcap);
  fp = fmemopen(text, textcap - 1, "w");
  get_tunepeaks_coherent(&T, LON, fp);
  return tune_collect(&T, LON, fp, text, value, ampli, cap);
}
