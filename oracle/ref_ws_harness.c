/*
 * ref_ws_harness.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A single-process driver for the reference's slice (BunchModel = STRONG)
 * model with fast beam-ion interaction, calling the UNMODIFIED reference
 * functions compiled by oracle/Makefile into oracle/_ref/libmbtref.so.
 * It replays manager_weakstrong.c:7-263 and worker_weakstrong.c:13-247
 * for every filled bunch in one process, phase by phase:
 *
 *   1. per bunch: transformSbunch_shortrange (rw_weakstrong.c:10-66) and
 *      fbi_weakstrong_bunch (fbi_weakstrong.c:45-297) on the worker's
 *      copy; the manager appends the slice centroids to its history
 *      (bunch_CM_history_append bunch.c:95-115) and every NrevMon turns
 *      records bunch_strong_distribution_statistics (bunch.c:516-549);
 *   2. sortCMdata / resortCMdata (bunch.c:117-224) hand the history to the
 *      workers -- the manager sends only the first 5000 entries of each
 *      data array (manager_weakstrong.c:155-158), and so does this
 *      harness; then per bunch transformSbunch_optic and, with
 *      EnableRW_long, transformSbunch_longrange for HOR and VER;
 *   3. the ion train: fbi_weakstrong_train (fbi_weakstrong.c:300-451) over
 *      the filled bunches in bucket order on one shared ion list, with the
 *      ion centroid writeoutCMImotions prints (fbi_weakstrong.c:583-669)
 *      and the bunch centroid of writeoutVCMmotionsPM2 (:672-737).
 *
 * Every MPI message of those loops only copies data between ranks, so one
 * process with the same phase order sees the same numbers.
 *
 * Reference defects this harness works around, each behind a switch:
 *   - manager_weakstrong never sets ring.Ibunch (calloc'ed zero by
 *     setup_ring_parameters input.c:1571) and sends that array to the
 *     workers, so every charge, ion count and resistive-wall kick is zero;
 *     fix_ibunch sets the bunch currents as manager_weakweak.c:61-78 does;
 *   - beffH3/beffV3 are read only with EnableRW_short (input.c:465-478),
 *     and transformSbunch_longrange divides by their cube
 *     (rw_weakstrong.c:101-106,128); fix_ibunch also reads them whenever
 *     EnableRW_long is set, as the weak-model harness does;
 *   - strong_generate_eCMs leaves the slice xtau/xeps of bunch0
 *     uninitialised (manager_weakstrong.c:18, bunch_strong.c:59-133); the
 *     harness zeroes them.
 *
 * Nothing in the product links this file.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "types.h"
#include "bunch.h"
#include "fbi.h"
#include "input.h"
#include "rw.h"

extern ring_t ring;
extern tracking_t track;
extern grid_t fbii_grid;

/* defined in bunch.c:703-770 without a header prototype */
int bunch_writeout_mean_ampinv_pos(const long int NrevTot, const long int NrevMon,
                                   const bunch_CM_history_strong_t * CMhist,
                                   const e_beam_t ebeam, const plane_t plane);

typedef struct wsw {
  int kb;
  bunch_strong_t bunch0;        /* worker_weakstrong.c:15 */
  bunch_strong_t bunch;         /* worker_weakstrong.c:16 */
  ion_beam_local_t *ion;        /* worker_weakstrong.c:41 */
} wsw_t;

static int ws_nb = 0;
static wsw_t *WS = NULL;
static e_beam_t ws_ebeam;
static bunch_macroparticle_model_t ws_model;
static selffield_model_t ws_sf;
static fbii_model_t ws_fbii;
static bunch_strong_t ws_bunch0;              /* manager's bunch0 */
static bunch_strong_t *ws_bunches = NULL;     /* manager's bunches[Nharm] */
static bunch_CM_history_strong_t *ws_hist_m = NULL, *ws_hist_w = NULL;
static ion_beam_t *ws_ions = NULL;
static long ws_rev = 0;
static int ws_slices = 0;
static double *ws_soa = NULL;                 /* the Np generated particles */
static int ws_files = 0;                      /* call the manager's writers */

static void free_all(void)
{
  int i;
  if (WS) {
    for (i = 0; i < ws_nb; i++) free(WS[i].ion);
    free(WS);
  }
  WS = NULL;
  free(ws_bunches); ws_bunches = NULL;
  if (ws_hist_m) { bunch_CM_history_strong_destroy(ws_hist_m); free(ws_hist_m); }
  if (ws_hist_w) { bunch_CM_history_strong_destroy(ws_hist_w); free(ws_hist_w); }
  ws_hist_m = ws_hist_w = NULL;
  free(ws_ions); ws_ions = NULL;
  free(ws_soa); ws_soa = NULL;
  ws_nb = 0;
}

static void ws_beff_fix(const char *conf)
{
  FILE *fp = fopen(conf, "r");
  int saved;
  if (fp == NULL) return;
  saved = config_get_fprint;
  config_get_fprint = false;
  config_get_double(fp, "ring", "beffH3", &(ring.beffH[0]));
  config_get_double(fp, "ring", "beffV3", &(ring.beffV[0]));
  config_get_fprint = saved;
  fclose(fp);
}

int refws_init(const char *conf, const char *workdir, int fix_ibunch)
{
  char inp[FILENAME_MAX];
  int kb, ib, i;
  free_all();
  snprintf(inp, FILENAME_MAX, "%s", conf);
  memset(&ring, 0, sizeof(ring));
  memset(&track, 0, sizeof(track));
  memset(&ws_ebeam, 0, sizeof(ws_ebeam));
  memset(&ws_model, 0, sizeof(ws_model));
  memset(&ws_sf, 0, sizeof(ws_sf));
  snprintf(track.work_path, FILENAME_MAX, "%s", workdir ? workdir : "/tmp");

  /* mbtrack-mpi.c:61-81 and the manager's set-up :97 */
  if (!read_input(inp, &ring, &track, &ws_ebeam, &ws_model, &ws_sf)) return -1;
  if (track.BunchModel != MODEL_STRONG) return -2;
  if (fix_ibunch && track.EnableRW_long) ws_beff_fix(conf);
  setup_ring_parameters(&ring);
  macrop_model_setup_parameters(ring, track, &ws_model);
  fbii_grid_setup_parameters(&fbii_grid, &ws_ebeam, ws_model);
  if (!e_beam_setup(&track, &ring, &ws_ebeam)) return -3;
  setup_tracking_parameters(&ring, &track, &ws_sf, &ws_model);
  ws_slices = 2 * ws_ebeam.distrib.Nslc + 1;
  if (ws_slices > NCELL_MAX - 1 || ws_model.Np > 10000 || ws_model.Np < 2) return -4;
  if (ring.Nharm > 500 || track.NmultiT > 30) return -5;

  ws_nb = ws_ebeam.Nbunch;
  WS = (wsw_t *) calloc(ws_nb, sizeof(wsw_t));
  ws_bunches = (bunch_strong_t *) calloc(ring.Nharm, sizeof(bunch_strong_t));
  ws_hist_m = (bunch_CM_history_strong_t *) calloc(1, sizeof(bunch_CM_history_strong_t));
  ws_hist_w = (bunch_CM_history_strong_t *) calloc(1, sizeof(bunch_CM_history_strong_t));
  ws_ions = (ion_beam_t *) calloc(1, sizeof(ion_beam_t));
  if (!WS || !ws_bunches || !ws_hist_m || !ws_hist_w || !ws_ions) return -6;
  {
    int nout = (int) (track.NrevTot / track.NrevMon * ws_ebeam.Nbunch);
    bunch_CM_history_strong_init(ws_hist_m, nout);
    bunch_CM_history_strong_init(ws_hist_w, nout);
  }

  /* bunch currents as manager_weakweak.c:61-78 (see header) */
  ib = 0;
  for (kb = 0; kb < (int) ring.Nharm; kb++) {
    if (!ws_ebeam.nfFill[kb]) continue;
    if (fix_ibunch) {
      double bunch_Ib = ws_ebeam.Ib_frac[ib] * ring.Iring / (((double) ws_ebeam.Nbunch) * FKILO);
      ring.Ibunch[kb] = bunch_Ib * FKILO;
    }
    WS[ib].kb = kb;
    ib++;
  }

  /* the particles strong_generate_eCMs draws (bunch_strong.c:80-91),
     kept for the slicing check; the draws below repeat exactly because
     each plane reseeds with its own seed */
  {
    int np = ws_model.Np;
    static double t0[30000], e0[30000], x0[30000], xp0[30000], z0[30000], zp0[30000];
    if (generate_initial_sbunch_distribution2(ws_model.nGen[LON], 0, LON, t0, e0, ring, ws_model) < 0
        || generate_initial_sbunch_distribution2(ws_model.nGen[HOR], 0, HOR, x0, xp0, ring, ws_model) < 0
        || generate_initial_sbunch_distribution2(ws_model.nGen[VER], 0, VER, z0, zp0, ring, ws_model) < 0)
      return -7;
    ws_soa = (double *) malloc(6 * (size_t) np * sizeof(double));
    for (i = 0; i < np; i++) {
      ws_soa[i] = t0[i];
      ws_soa[np + i] = x0[i];
      ws_soa[2 * np + i] = z0[i];
      ws_soa[3 * np + i] = e0[i];
      ws_soa[4 * np + i] = xp0[i];
      ws_soa[5 * np + i] = zp0[i];
    }
  }

  /* manager_weakstrong.c:41-55 */
  memset(&ws_bunch0, 0, sizeof(ws_bunch0));
  if (strong_generate_eCMs(ws_model, &ws_ebeam, &ws_bunch0, 0) < 0) return -8;
  if (generate_initial_general_distribution2(ws_bunches, &ws_bunch0, ws_model, ring, ws_ebeam) < 0) return -9;

  /* worker_weakstrong.c:37-70 */
  fbii_model_init(&ws_fbii);
  ws_fbii.factBE = sqrt(2 * (ws_model.sgm_xx * ws_model.sgm_xx - ws_model.sgm_zz * ws_model.sgm_zz)) / FKILO;
  for (ib = 0; ib < ws_nb; ib++) {
    int icell, msx, msz, ic = 0;
    const int offst = fbii_grid.offst;
    WS[ib].ion = (ion_beam_local_t *) calloc(1, sizeof(ion_beam_local_t));
    if (!WS[ib].ion) return -6;
    for (icell = 0; icell < ws_slices; icell++)
      for (msx = -offst; msx < offst + 1; msx++)
        for (msz = -offst; msz < offst + 1; msz++)
          WS[ib].ion->mapslice2i[icell][msx + offst][msz + offst] = ic++;
    WS[ib].bunch0 = ws_bunch0;
  }
  ws_ions->model.nFio = 0;
  ws_ions->model.kbFio = 0;
  ws_rev = 0;
  return ws_nb;
}

/* Sizes and set-up values: out_i = {Nslc, slices, Ngrid, offst, Np, Nharm,
   NmultiT, EnableFBII, EnableRW_long}; out_d = {agLOCx, agLOCz, agABSx,
   agABSz, deltT, factBE, factF, Ldmsgm, sgm_xx, sgm_zz, sgmatau}. */
void refws_info(int *out_i, double *out_d, int *bucket, double *ibunch, int *npop, int *nofe)
{
  int ib, c, i, j;
  const int G = fbii_grid.Ngrid;
  out_i[0] = ws_ebeam.distrib.Nslc; out_i[1] = ws_slices; out_i[2] = G; out_i[3] = fbii_grid.offst;
  out_i[4] = ws_model.Np; out_i[5] = (int) ring.Nharm; out_i[6] = track.NmultiT;
  out_i[7] = track.EnableFBII; out_i[8] = track.EnableRW_long;
  out_d[0] = fbii_grid.agLOCx; out_d[1] = fbii_grid.agLOCz; out_d[2] = fbii_grid.agABSx;
  out_d[3] = fbii_grid.agABSz; out_d[4] = ws_ebeam.distrib.deltT; out_d[5] = ws_fbii.factBE;
  out_d[6] = ws_fbii.factF; out_d[7] = ws_fbii.Ldmsgm; out_d[8] = ws_model.sgm_xx;
  out_d[9] = ws_model.sgm_zz; out_d[10] = ws_model.sgmatau;
  for (ib = 0; ib < ws_nb; ib++) {
    if (bucket) bucket[ib] = WS[ib].kb;
    if (ibunch) ibunch[ib] = ring.Ibunch[WS[ib].kb];
  }
  for (c = 0; c < ws_slices; c++) {
    if (npop) npop[c] = ws_bunch0.npop[c];
    if (nofe)
      for (i = 0; i < G; i++)
        for (j = 0; j < G; j++) nofe[(c * G + i) * G + j] = ws_ebeam.distrib.Nofe[c][i][j];
  }
}

void refws_particles(double *soa6) { memcpy(soa6, ws_soa, 6 * (size_t) ws_model.Np * sizeof(double)); }

/* slice state of the manager, [nbunch][6][slices]: xtau, xeps, xx, xp, zz, zp */
void refws_get_slices(double *out)
{
  int ib, c;
  const int S = ws_slices;
  for (ib = 0; ib < ws_nb; ib++) {
    const bunch_strong_t *b = &ws_bunches[WS[ib].kb];
    double *o = out + (size_t) ib * 6 * S;
    for (c = 0; c < S; c++) {
      o[c] = b->xtau[c]; o[S + c] = b->xeps[c]; o[2 * S + c] = b->xx[c];
      o[3 * S + c] = b->xp[c]; o[4 * S + c] = b->zz[c]; o[5 * S + c] = b->zp[c];
    }
  }
}

void refws_set_slices(const double *in)
{
  int ib, c;
  const int S = ws_slices;
  for (ib = 0; ib < ws_nb; ib++) {
    bunch_strong_t *b = &ws_bunches[WS[ib].kb];
    const double *o = in + (size_t) ib * 6 * S;
    for (c = 0; c < S; c++) {
      b->xtau[c] = o[c]; b->xeps[c] = o[S + c]; b->xx[c] = o[2 * S + c];
      b->xp[c] = o[3 * S + c]; b->zz[c] = o[4 * S + c]; b->zp[c] = o[5 * S + c];
    }
  }
}

static void copy_arrays(bunch_strong_t *dst, const bunch_strong_t *src)
{
  memcpy(dst->xtau, src->xtau, sizeof dst->xtau);
  memcpy(dst->xeps, src->xeps, sizeof dst->xeps);
  memcpy(dst->xx, src->xx, sizeof dst->xx);
  memcpy(dst->xp, src->xp, sizeof dst->xp);
  memcpy(dst->zz, src->zz, sizeof dst->zz);
  memcpy(dst->zp, src->zp, sizeof dst->zp);
}

static void put_vec(double *o, const vector_t *v) { o[0] = v->xtau; o[1] = v->x; o[2] = v->z; }

/* nturns turns.  Per turn and filled bunch: cm[6] = the slice-weighted
   centroids after the short-range step (pos LON, slope LON, pos HOR,
   slope HOR, pos VER, slope VER; the HOR/VER four are what the manager
   appends to its history); ion[2] = centroid (Nri weighted) of the ion
   list after the bunch's train step, [m] (NaN without ions); zcm[nharm]
   per turn = the unweighted slice mean of zz after the turn, 0 for empty
   buckets; on turns with rev % NrevMon == 0, stats[18] per bunch = pos,
   pos_sigma, slope, slope_sigma, ampinv, ampinv_cm (LON, HOR, VER each).
   Any output may be NULL. */
int refws_run(long nturns, double *cm, double *ion, double *zcm, double *stats)
{
  long t;
  int ib;
  const int S = ws_slices;
  long imon = 0;
  for (t = 0; t < nturns; t++, ws_rev++) {
    const long rev = ws_rev;
    /* phase 1: worker_weakstrong.c:74-134, manager_weakstrong.c:79-141 */
    for (ib = 0; ib < ws_nb; ib++) {
      wsw_t *w = &WS[ib];
      const int kb = w->kb;
      copy_arrays(&w->bunch0, &ws_bunches[kb]);
      w->bunch = w->bunch0;
      transformSbunch_shortrange((int) rev, kb, ws_ebeam, ws_model, &w->bunch0, &w->bunch);
      if (track.EnableFBII
          && fbi_weakstrong_bunch(ws_model, &(ws_ions->model), ws_fbii, ws_ebeam, w->ion, &w->bunch, kb) < 0)
        return -1;
      copy_arrays(&ws_bunches[kb], &w->bunch);
      bunch_CM_history_append(ws_hist_m, kb, w->bunch.stats.pos.x, w->bunch.stats.slope.x,
                              w->bunch.stats.pos.z, w->bunch.stats.slope.z);
      if (cm) {
        double *o = cm + ((size_t) t * ws_nb + ib) * 6;
        o[0] = w->bunch.stats.pos.xtau; o[1] = w->bunch.stats.slope.xtau;
        o[2] = w->bunch.stats.pos.x; o[3] = w->bunch.stats.slope.x;
        o[4] = w->bunch.stats.pos.z; o[5] = w->bunch.stats.slope.z;
      }
      if (rev % track.NrevMon == 0) {
        bunch_strong_distribution_statistics(&w->bunch, S);
        if (ws_files) {
          /* manager_weakstrong.c:131-138; an index past the array (the
             reference writes there) is skipped */
          const long k = (rev / track.NrevMon) * ws_ebeam.Nbunch + kb;
          const long nslot = (long) (track.NrevTot / track.NrevMon * ws_ebeam.Nbunch) + 2;
          if (k < nslot) {
            ws_hist_m->cm[k] = w->bunch.stats.pos;
            ws_hist_m->rms[k] = w->bunch.stats.pos_sigma;
            ws_hist_m->cm_slope[k] = w->bunch.stats.slope;
            ws_hist_m->rms_slope[k] = w->bunch.stats.slope_sigma;
            ws_hist_m->ampinv[k] = w->bunch.stats.ampinv;
            ws_hist_m->ampinv_cm[k] = w->bunch.stats.ampinv_cm;
          }
        }
        if (stats) {
          double *o = stats + ((size_t) imon * ws_nb + ib) * 18;
          put_vec(o, &w->bunch.stats.pos); put_vec(o + 3, &w->bunch.stats.pos_sigma);
          put_vec(o + 6, &w->bunch.stats.slope); put_vec(o + 9, &w->bunch.stats.slope_sigma);
          put_vec(o + 12, &w->bunch.stats.ampinv); put_vec(o + 15, &w->bunch.stats.ampinv_cm);
        }
      }
    }
    if (rev % track.NrevMon == 0) {
      if (ws_files) bunch_strong_writeout_ampinv(rev, rev / track.NrevMon, ws_hist_m, ws_ebeam);
      imon++;
    }

    /* phase 2: manager_weakstrong.c:143-178, worker_weakstrong.c:138-183 */
    sortCMdata((int) rev, ws_hist_m);
    memcpy(ws_hist_w->dataVV, ws_hist_m->dataVV, 5000 * sizeof(double));
    memcpy(ws_hist_w->dataVP, ws_hist_m->dataVP, 5000 * sizeof(double));
    memcpy(ws_hist_w->dataXX, ws_hist_m->dataXX, 5000 * sizeof(double));
    memcpy(ws_hist_w->dataXP, ws_hist_m->dataXP, 5000 * sizeof(double));
    resortCMdata((int) rev, ws_hist_w);
    for (ib = 0; ib < ws_nb; ib++) {
      wsw_t *w = &WS[ib];
      transformSbunch_optic((int) rev, w->kb, ws_ebeam, &w->bunch);
      if (track.EnableRW_long) {
        if (track.TrackPlane[HOR]) transformSbunch_longrange((int) rev, w->kb, HOR, ws_ebeam, ws_model, ws_hist_w, &w->bunch);
        if (track.TrackPlane[VER]) transformSbunch_longrange((int) rev, w->kb, VER, ws_ebeam, ws_model, ws_hist_w, &w->bunch);
      }
      bunch_strong_updateCM(&w->bunch, S, HOR);
      bunch_strong_updateCM(&w->bunch, S, VER);
      copy_arrays(&ws_bunches[w->kb], &w->bunch);
    }

    /* phase 3: manager_weakstrong.c:184-233, worker_weakstrong.c:185-242 */
    ws_ions->model.nFio = 0;
    ws_ions->model.kbFio = 0;
    for (ib = 0; ib < ws_nb; ib++) {
      wsw_t *w = &WS[ib];
      if (track.EnableFBII
          && fbi_weakstrong_train(ws_model, ws_fbii, ws_ebeam, w->ion, ws_ions, &w->bunch, ib, w->kb) < 0)
        return -2;
      copy_arrays(&ws_bunches[w->kb], &w->bunch);
      if (ws_files && track.EnableFBII)
        writeoutCMImotions(track.work_path, (int) rev, ib, ws_ions, &ws_ebeam, ws_model);
      if (ion) {
        /* writeoutCMImotions fbi_weakstrong.c:626-646 */
        double xs = 0.0, ys = 0.0, nt = 0.0;
        int ip;
        for (ip = 0; ip < ws_ions->model.nFio; ip++) {
          xs = xs + ws_ions->NriFio[ip] * ws_ions->xxFio[ip];
          ys = ys + ws_ions->NriFio[ip] * ws_ions->yyFio[ip];
          nt = nt + ws_ions->NriFio[ip];
        }
        ion[((size_t) t * ws_nb + ib) * 2] = nt == 0.0 ? NAN : xs / nt;
        ion[((size_t) t * ws_nb + ib) * 2 + 1] = nt == 0.0 ? NAN : ys / nt;
      }
    }
    if (ws_files) writeoutVCMmotionsPM2(track.work_path, (int) rev, ws_bunches, &ws_ebeam);
    if (zcm) {
      /* writeoutVCMmotionsPM2 fbi_weakstrong.c:708-718 */
      unsigned kb;
      int icell;
      for (kb = 0; kb < ring.Nharm; kb++) {
        double z = 0.0;
        if (ws_ebeam.nfFill[kb]) {
          for (icell = 0; icell < S; icell++) z = z + ws_bunches[kb].zz[icell];
          z = z / ((double) S);
        }
        zcm[(size_t) t * ring.Nharm + kb] = z;
      }
    }
  }
  return 0;
}

/* Field grid (Ex, Ey interleaved, slices x Ngrid x Ngrid) and local ions
   (Nri, xx, xd, yy, yd; same count) of filled bunch ib from its last
   fbi_weakstrong_bunch call. */
void refws_bunch_fields(int ib, double *exey, double *ions5)
{
  const ion_beam_local_t *L = WS[ib].ion;
  const int n = ws_slices * fbii_grid.Ngrid * fbii_grid.Ngrid;
  int i;
  for (i = 0; i < n; i++) {
    if (exey) { exey[2 * i] = L->Ex[i]; exey[2 * i + 1] = L->Ey[i]; }
    if (ions5) {
      ions5[i] = L->Nri[i]; ions5[n + i] = L->xxi0[i]; ions5[2 * n + i] = L->xdi0[i];
      ions5[3 * n + i] = L->yyi0[i]; ions5[4 * n + i] = L->ydi0[i];
    }
  }
}

/* get_linearly_interpolated_Efields (fbi_weakstrong.c:454-580) on filled
   bunch ib's last field grid, for n points. */
void refws_interp(int ib, int icell, const double *x, const double *y, int n, double *exey)
{
  int i;
  double e[2];
  for (i = 0; i < n; i++) {
    get_linearly_interpolated_Efields(icell, x[i], y[i], WS[ib].ion, e);
    exey[2 * i] = e[0];
    exey[2 * i + 1] = e[1];
  }
}

/* Switch the manager's writers on (files in the work directory given to
   refws_init): motion files every turn, ampinv files every NrevMon. */
void refws_files(int on) { ws_files = on; }

/* The end-of-run files of manager_weakstrong.c:244-247. */
void refws_finish(void)
{
  if (track.TrackPlane[HOR]) bunch_writeout_mean_ampinv_pos(track.NrevTot, track.NrevMon, ws_hist_m, ws_ebeam, HOR);
  if (track.TrackPlane[VER]) bunch_writeout_mean_ampinv_pos(track.NrevTot, track.NrevMon, ws_hist_m, ws_ebeam, VER);
}

/* The manager's generated-bunch files (strong_generate_eCMs with writeout,
   bunch_strong.c:80-91): the three gendst_datafile paths of the input. */
int refws_write_distribution(void)
{
  static double a[30000], b[30000];
  if (generate_initial_sbunch_distribution2(ws_model.nGen[LON], 1, LON, a, b, ring, ws_model) < 0) return -1;
  if (generate_initial_sbunch_distribution2(ws_model.nGen[HOR], 1, HOR, a, b, ring, ws_model) < 0) return -1;
  if (generate_initial_sbunch_distribution2(ws_model.nGen[VER], 1, VER, a, b, ring, ws_model) < 0) return -1;
  return 0;
}
