/*
 * mbt_output.c -- the text files of a weak-weak run, in the reference's
 * formats, written from the statistics libmbt returns.
 *
 * In the reference the manager rank writes the all-bunch files and the
 * worker ranks of the output bunches write their own; here one writer
 * object receives every turn's statistics of every bunch and keeps the
 * accumulators of both sides:
 *
 *   manager  mean_bunch_all.dat         manager_weakweak.c:104-127, 235-302
 *            ampinv_<P>_<rev>.dat       bunch_weak_writeout_ampinv bunch.c:588-640,
 *                                       bunch_fprint_ampinv bunch.c:552-585
 *            mean_bunch_end.dat         manager_weakweak.c:307-331
 *            bunchbybunch_<P>.dat       weak_bunch_writeout_tbtbbb bunch_weak.c:343-387
 *            ampinv_<P>_mean.dat        weak_bunch_writeout_mean_ampinv bunch_weak.c:390-447
 *   workers  mean_bunch_<kb>.dat        worker_weakweak.c:225-234, 290-302,
 *                                       worker_weak_stat_output bunch.c:773-789
 *            potentials_bunch_<kb>.dat  worker_weakweak.c:236-249, transform_weak.c:735-768
 *            wakes.dat                  worker_weakweak.c:96-106
 *            dipoles_history.dat        worker_weakweak.c:418-438
 *            gendst_datafile_<P>        weak_writeout_bunch_distribution bunch_weak.c:296-332
 *
 * Turn averages follow the reference's accumulators: the manager sums the
 * twelve statistics of every bunch and their squares (weak_bunch_add_
 * statistics statistics.c:204-220), a worker sums its own tracked planes
 * and their pow(x, 2.) (weak_bunch_calc_statistics statistics.c:131-157),
 * and both turn sums into mean and sample standard deviation with the
 * operation order of weak_bunch_update_statistics (statistics.c:223-246)
 * and vector_variance (statistics.c:37-44).
 *
 * Where several output workers of the reference write the same file
 * (wakes.dat, dipoles_history.dat, the distribution files) the last one to
 * finish wins; the writer takes the first output bunch.
 */
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mbt.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#define FKILO 1.0e+03
#define FGIGA 1.0e+09

static __thread char g_werr[512];

static int werr(int code, const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_werr, sizeof g_werr, fmt, ap);
  va_end(ap);
  return code;
}

const char *mbt_writer_error(void) { return g_werr; }

/* sums of pos, pos_sigma, slope, slope_sigma (the order of a statistics
 * record) and of their squares, per plane */
typedef struct acc {
  double s[4][3], q[4][3];
} acc_t;

struct mbt_writer {
  mbt_params p;
  mbt_output_cfg o;
  char dir[4096];
  int flags;
  int nb;
  int *bucket, *bunch_of;          /* bunch -> bucket, bucket -> bunch or -1 */
  double *ib;
  int n_out;                        /* output bunches that exist */
  int *out;                         /* their bunch indices, bucket order */
  FILE *all_fp, **out_fp, **pot_fp;
  acc_t all, *out_acc;
  long nstat_all, *nstat_out;
  long rev;                         /* turns received */
  long nmon_rows;                   /* NrevTot / NrevMon */
  size_t nhist;                     /* history entries: rows x nb + 2 */
  double (*cm)[3], (*ai)[3], (*aic)[3];
  double *scan_hist;
  long nscan_hist, m;
  long nrev_scan;                   /* NrevScan (NrevTot + 1 without a scan) */
  double scan_val, iring;           /* manager's scan value and ring current */
  double scan_val_w, iring_w;       /* the workers' (they step one turn earlier
                                       when NrevScan = 1) */
  double (*dip)[2];                 /* resistive-wall dipole ring buffer */
  long ndip;
  int began;
};

static void acc_reset(acc_t *a) { memset(a, 0, sizeof(*a)); }

/* weak_bunch_add_statistics: every plane, squares as products */
static void acc_add_all(acc_t *a, const double *st)
{
  int k, pl;
  for (k = 0; k < 4; k++)
    for (pl = 0; pl < 3; pl++) {
      const double v = st[3 * k + pl];
      a->s[k][pl] = a->s[k][pl] + v;
      a->q[k][pl] = a->q[k][pl] + v * v;
    }
}

/* weak_bunch_calc_statistics: tracked planes, squares through pow() */
static void acc_add_tracked(acc_t *a, const double *st, const int *tp)
{
  int k, pl;
  for (pl = 0; pl < 3; pl++) {
    if (!tp[pl]) continue;
    for (k = 0; k < 4; k++) a->s[k][pl] += st[3 * k + pl];
    for (k = 0; k < 4; k++) a->q[k][pl] += pow(st[3 * k + pl], 2.);
  }
}

/* weak_bunch_update_statistics: sample variance, then means */
static void acc_update(acc_t *a, long n)
{
  int k, pl;
  for (k = 0; k < 4; k++)
    for (pl = 0; pl < 3; pl++) {
      if (n > 1) {
        double v = (-1.0 / ((double) n)) * (a->s[k][pl] * a->s[k][pl]);
        v = v + a->q[k][pl];
        a->q[k][pl] = (1.0 / ((double) (n - 1))) * v;
      } else {
        a->q[k][pl] = 0.0;
      }
      a->s[k][pl] = (1.0 / ((double) n)) * a->s[k][pl];
    }
}

/* bunch_stats_fprintf: per plane mean/sigma of pos, slope, pos_sigma,
 * slope_sigma */
static void acc_print(FILE *fp, long rev, const acc_t *a, double scan, const int *tp)
{
  static const char *const tag[3] = {"LON", "HOR", "VER"};
  int pl;
  fprintf(fp, "%4ld   %.4e   ", rev + 1, scan);
  for (pl = 0; pl < 3; pl++) {
    if (pl > 0 && !tp[pl]) continue;
    fprintf(fp, pl == 0 ? "%s    %.4e   %.4e   %.4e   %.4e   %.4e   %.4e   %.4e   %.4e"
                        : "  %s    %.4e   %.4e   %.4e   %.4e   %.4e   %.4e   %.4e   %.4e",
            tag[pl], a->s[0][pl], sqrt(a->q[0][pl]), a->s[2][pl], sqrt(a->q[2][pl]), a->s[1][pl],
            sqrt(a->q[1][pl]), a->s[3][pl], sqrt(a->q[3][pl]));
  }
  fprintf(fp, "\n");
}

static FILE *open_in(const mbt_writer *w, const char *name, const char *mode)
{
  char path[8192];
  snprintf(path, sizeof path, "%s/%s", w->dir, name);
  return fopen(path, mode);
}

int mbt_writer_open(const char *work_path, const mbt_params *p, const mbt_output_cfg *o, const int *bunch_out,
                    int nbunch, const int *bucket, const double *ib, int flags, mbt_writer **out)
{
  mbt_writer *w;
  int i, j;
  char name[256];
  if (!out) return werr(MBT_ERR_INVALID, "out is NULL");
  *out = NULL;
  if (!work_path || !p || !o || !bucket || !ib || nbunch <= 0 || (o->n_out > 0 && !bunch_out))
    return werr(MBT_ERR_INVALID, "writer: null argument or nbunch <= 0");
  if (p->nrev_mon <= 0 || p->nrev_tot < 0 || p->nharm <= 0)
    return werr(MBT_ERR_INVALID, "writer: NrevMon must be positive");
  if (p->scan != 0 && p->nrev_scan < 1) return werr(MBT_ERR_INVALID, "writer: NrevScan must be positive");
  for (i = 0; i < nbunch; i++)
    if (bucket[i] < 0 || bucket[i] >= p->nharm || (i > 0 && bucket[i] <= bucket[i - 1]))
      return werr(MBT_ERR_INVALID, "writer: buckets must be ascending in 0..h-1");
  w = (mbt_writer *) calloc(1, sizeof(*w));
  if (!w) return werr(MBT_ERR_NOMEM, "writer: host allocation");
  w->p = *p;
  w->o = *o;
  w->flags = flags;
  snprintf(w->dir, sizeof w->dir, "%s", work_path);
  w->nb = nbunch;
  w->bucket = (int *) malloc(nbunch * sizeof(int));
  w->bunch_of = (int *) malloc(p->nharm * sizeof(int));
  w->ib = (double *) malloc(nbunch * sizeof(double));
  w->out = (int *) malloc((o->n_out > 0 ? o->n_out : 1) * sizeof(int));
  w->out_fp = (FILE **) calloc(o->n_out > 0 ? o->n_out : 1, sizeof(FILE *));
  w->pot_fp = (FILE **) calloc(o->n_out > 0 ? o->n_out : 1, sizeof(FILE *));
  w->out_acc = (acc_t *) calloc(o->n_out > 0 ? o->n_out : 1, sizeof(acc_t));
  w->nstat_out = (long *) calloc(o->n_out > 0 ? o->n_out : 1, sizeof(long));
  w->nmon_rows = p->nrev_tot / p->nrev_mon;
  w->nhist = (size_t) w->nmon_rows * nbunch + 2;
  w->cm = calloc(w->nhist, sizeof(*w->cm));
  w->ai = calloc(w->nhist, sizeof(*w->ai));
  w->aic = calloc(w->nhist, sizeof(*w->aic));
  /* manager_weakweak.c:29-32: one entry per statistics line */
  w->nscan_hist = w->nmon_rows + (p->scan != 0 ? p->nscan : 1) + 1;
  w->scan_hist = (double *) calloc(w->nscan_hist, sizeof(double));
  w->nrev_scan = p->scan != 0 ? p->nrev_scan : p->nrev_tot + 1;
  w->scan_val = w->scan_val_w = p->scan_start;
  w->iring = w->iring_w = p->Iring;
  if (p->rw_long) {
    w->ndip = (long) (p->Nmlt + 2) * p->nharm;
    w->dip = calloc(w->ndip, sizeof(*w->dip));
  }
  if (!w->bucket || !w->bunch_of || !w->ib || !w->out || !w->out_fp || !w->pot_fp || !w->out_acc ||
      !w->nstat_out || !w->cm || !w->ai || !w->aic || !w->scan_hist || (p->rw_long && !w->dip)) {
    mbt_writer_close(w);
    return werr(MBT_ERR_NOMEM, "writer: host allocation");
  }
  memcpy(w->bucket, bucket, nbunch * sizeof(int));
  memcpy(w->ib, ib, nbunch * sizeof(double));
  for (i = 0; i < p->nharm; i++) w->bunch_of[i] = -1;
  for (i = 0; i < nbunch; i++) w->bunch_of[bucket[i]] = i;
  /* output bunches: a worker exists only for a filled bucket */
  for (i = 0; i < nbunch; i++)
    for (j = 0; j < o->n_out; j++)
      if (bunch_out[j] == bucket[i]) { w->out[w->n_out++] = i; break; }

  w->all_fp = open_in(w, "mean_bunch_all.dat", "w+");
  if (!w->all_fp) {
    int r = werr(MBT_ERR_IO, "cannot create %s/mean_bunch_all.dat", w->dir);
    mbt_writer_close(w);
    return r;
  }
  for (i = 0; i < w->n_out; i++) {
    const int kb = bucket[w->out[i]];
    snprintf(name, sizeof name, "mean_bunch_%d.dat", kb);
    w->out_fp[i] = open_in(w, name, "w+");
    if (w->out_fp[i] && o->nrev_potentials_out <= p->nrev_tot) {
      snprintf(name, sizeof name, "potentials_bunch_%d.dat", kb);
      w->pot_fp[i] = open_in(w, name, "w+");
      if (w->pot_fp[i]) {
        fprintf(w->pot_fp[i], " # potentials and distributions, Ib = %g A ;\n", ib[w->out[i]]);
        fprintf(w->pot_fp[i], " # rev  scan_val         tau         LON_wake_pot       HC_pot        rf_pot      "
                              "active_cav      ideal_HC        bunch_shape");
        if (p->planeV > 0) fprintf(w->pot_fp[i], "     VER_wake_pot     VER_dipole_mom");
        if (p->planeH > 0) fprintf(w->pot_fp[i], "     HOR_wake_pot     HOR_dipole_mom");
        fprintf(w->pot_fp[i], "\n");
      }
    }
    if (!w->out_fp[i] || (o->nrev_potentials_out <= p->nrev_tot && !w->pot_fp[i])) {
      int r = werr(MBT_ERR_IO, "cannot create the files of output bunch %d in %s", kb, w->dir);
      mbt_writer_close(w);
      return r;
    }
  }
  *out = w;
  return 0;
}

int mbt_writer_wakes(mbt_writer *w, const double *Gl, const double *Gv, const double *Gh)
{
  FILE *fp;
  int nc;
  if (!w) return werr(MBT_ERR_INVALID, "writer is NULL");
  if (w->n_out == 0) return 0;
  if (w->p.ncell > 0 && (!Gl || !Gv || !Gh)) return werr(MBT_ERR_INVALID, "wakes: Green's functions are NULL");
  fp = open_in(w, "wakes.dat", "w+");
  if (!fp) return werr(MBT_ERR_IO, "cannot create %s/wakes.dat", w->dir);
  fprintf(fp, "# bin (%.2e s)   total wake L     - V -      - H -\n", w->p.dT * w->p.sigma_tau);
  for (nc = 0; nc < w->p.ncell; nc++) fprintf(fp, "%d  %e   %e   %e\n", nc, Gl[nc], Gv[nc], Gh[nc]);
  fclose(fp);
  return 0;
}

int mbt_writer_begin(mbt_writer *w, const double *st)
{
  int b, i, j;
  const int *tp;
  if (!w || !st) return werr(MBT_ERR_INVALID, "writer begin: null argument");
  if (w->began) return werr(MBT_ERR_STATE, "writer begin: called twice");
  tp = w->p.track_plane;
  /* manager: average over bunches, printed as turn -99 */
  acc_reset(&w->all);
  for (b = 0; b < w->nb; b++) acc_add_all(&w->all, st + 12 * b);
  acc_update(&w->all, w->nb);
  fprintf(w->all_fp, " # bunch statistics, AVEraged over all bunches & turns, Ib = %g A ;\n", w->ib[0]);
  fprintf(w->all_fp, " # turn - scan_var - AVE_CM_LON - SIG_CM_LON - AVE_delE_LON - SIG_delE_LON -  "
                     "AVE_sigmaL_LON - SIG_sigmaL_LON - AVE_sigmaE_LON - SIG_sigmaE_LON... (_HOR) ... (_VER)\n # ");
  acc_print(w->all_fp, -100, &w->all, 0.0, tp);
  fprintf(w->all_fp, "\n");
  acc_reset(&w->all);
  /* output workers: the initial statistics themselves */
  for (i = 0; i < w->n_out; i++) {
    FILE *fp = w->out_fp[i];
    const double *s = st + 12 * w->out[i];
    fprintf(fp, " # bunch statistics, averaged over turns, Ib = %g A ;\n", w->ib[w->out[i]]);
    fprintf(fp, " # turn - scan_var - AVE_CM_LON - SIG_CM_LON - AVE_delE_LON - SIG_delE_LON -  AVE_sigmaL_LON - "
                "SIG_sigmaL_LON - AVE_sigmaE_LON - SIG_sigmaE_LON... (_HOR) ... (_VER)\n # ");
    fprintf(fp, "beg      -/-    LON    %.4e       -/-        %.4e       -/-        %.4e      -/-        %.4e        -/- ",
            s[0], s[6], s[3], s[9]);
    if (tp[1])
      fprintf(fp, "    HOR     %.4e       -/-        %.4e       -/-        %.4e      -/-        %.4e        -/- ",
              s[1], s[7], s[4], s[10]);
    if (tp[2])
      fprintf(fp, "    VER     %.4e       -/-       %.4e       -/-        %.4e      -/-        %.4e       -/- ",
              s[2], s[8], s[5], s[11]);
    fprintf(fp, "\n");
    acc_reset(&w->out_acc[i]);
  }
  /* resistive-wall ring buffer: every slot j h + i of the first Nmlt turns
   * holds the initial dipole of bucket i (worker_weakweak.c:204-218) */
  if (w->p.rw_long) {
    for (b = 0; b < w->nb; b++)
      for (j = 0; j < w->p.Nmlt || j == 0; j++) {
        const long slot = ((long) j * w->p.nharm + w->bucket[b]) % w->ndip;
        w->dip[slot][0] = st[12 * b + 1];
        w->dip[slot][1] = st[12 * b + 2];
      }
  }
  w->began = 1;
  return 0;
}

/* history entry e as the reference's array holds it (zeros past its end) */
static double hist_at(const mbt_writer *w, double (*h)[3], long e, int plane)
{
  return (e >= 0 && (size_t) e < w->nhist) ? h[e][plane] : 0.0;
}

static int write_ampinv_files(mbt_writer *w, long rev, long irevmon)
{
  static const char *const tag[3] = {"LON", "HOR", "VER"};
  int pl, jb;
  char name[256];
  for (pl = 0; pl < 3; pl++) {
    FILE *fp;
    if (!w->p.track_plane[pl]) continue;
    snprintf(name, sizeof name, "ampinv_%s_%ld.dat", tag[pl], rev + 1);
    fp = open_in(w, name, "w");
    if (!fp) return werr(MBT_ERR_IO, "cannot create %s/%s", w->dir, name);
    fprintf(fp, "# turn: %-5ld\n", rev + 1);
    fprintf(fp, "# bunch   ampinv_cm   ampinv\n");
    for (jb = 0; jb < w->p.nharm; jb++) {
      long e;
      if (w->bunch_of[jb] < 0) continue;
      e = (w->flags & MBT_WRITER_OWN_AMPINV) ? irevmon * w->nb + w->bunch_of[jb] : irevmon + jb;
      fprintf(fp, " %3d %15.8e %15.8e\n", jb, hist_at(w, w->aic, e, pl), hist_at(w, w->ai, e, pl));
    }
    fclose(fp);
  }
  return 0;
}

int mbt_writer_turns(mbt_writer *w, long nturns, const double *stats, const double *ampinv)
{
  long t;
  int b, i;
  const int *tp;
  const long mon = w ? w->p.nrev_mon : 1;
  if (!w || nturns < 0 || (nturns > 0 && !stats)) return werr(MBT_ERR_INVALID, "writer turns: bad argument");
  if (!w->began) return werr(MBT_ERR_STATE, "writer turns: mbt_writer_begin has not run");
  if (w->rev + nturns > w->p.nrev_tot)
    return werr(MBT_ERR_STATE, "writer turns: %ld turns exceed NrevTot = %ld", w->rev + nturns, w->p.nrev_tot);
  tp = w->p.track_plane;
  for (t = 0; t < nturns; t++, w->rev++) {
    const long rev = w->rev;
    const double *st = stats + (size_t) t * w->nb * 12;
    const int monitor = (rev + 1) % mon == 0;
    if (monitor && !ampinv) return werr(MBT_ERR_INVALID, "writer turns: turn %ld is a monitor turn, ampinv is NULL", rev);
    /* manager: collect every bunch (manager_weakweak.c:235-253) */
    for (b = 0; b < w->nb; b++) {
      const double *s = st + 12 * b;
      if (monitor) {
        const size_t e = (size_t) (rev / mon) * w->nb + b;
        const double *a = ampinv + ((size_t) t * w->nb + b) * 6;
        int pl;
        for (pl = 0; pl < 3; pl++) {
          w->ai[e][pl] = a[pl];
          w->aic[e][pl] = a[3 + pl];
          w->cm[e][pl] = s[pl];
        }
      }
      acc_add_all(&w->all, s);
    }
    w->nstat_all++;
    /* output workers (worker_weakweak.c:290-302) */
    for (i = 0; i < w->n_out; i++) {
      acc_add_tracked(&w->out_acc[i], st + 12 * w->out[i], tp);
      w->nstat_out[i]++;
      if (w->nstat_out[i] % mon == 0 || (rev + 1) % w->nrev_scan == 0) {
        acc_update(&w->out_acc[i], w->nstat_out[i]);
        acc_print(w->out_fp[i], rev, &w->out_acc[i], w->scan_val_w, tp);
        acc_reset(&w->out_acc[i]);
        w->nstat_out[i] = 0;
      }
    }
    /* manager output (manager_weakweak.c:291-302) */
    if (w->nstat_all % mon == 0 || (rev + 1) % w->nrev_scan == 0) {
      w->nstat_all *= w->nb;
      acc_update(&w->all, w->nstat_all);
      if (w->m < w->nscan_hist) w->scan_hist[w->m] = w->scan_val;
      w->m++;
      if (w->o.ampinv_out) {
        int r = write_ampinv_files(w, rev, rev / mon);
        if (r) return r;
      }
      acc_print(w->all_fp, rev, &w->all, w->scan_val, tp);
      acc_reset(&w->all);
      w->nstat_all = 0;
    }
    /* scan step: manager after turn 0 only (manager_weakweak.c:287-288,
       tracking.c:10-16), workers on every boundary (worker_weakweak.c:389-391,
       tracking.c:43-48); only a current scan moves the value */
    if ((rev + 1) % w->nrev_scan == 0 && w->p.scan == 1) {
      if (rev > 0) {
        w->iring += w->p.scan_step;
        w->scan_val = w->iring;
      }
      w->iring_w += w->p.scan_step;
      w->scan_val_w = w->iring_w;
      for (b = 0; b < w->nb; b++) w->ib[b] += w->p.scan_step / (((double) w->nb) * FKILO);
    }
    /* resistive-wall ring buffer (worker_weakweak.c:306-318) */
    if (w->p.rw_long) {
      for (b = 0; b < w->nb; b++) {
        long in = -rev * (long) w->p.nharm + w->bucket[b];
        long slot = in < 0 ? (in % w->ndip + w->ndip) % w->ndip : in % w->ndip;
        w->dip[slot][0] = st[12 * b + 1];
        w->dip[slot][1] = st[12 * b + 2];
      }
    }
  }
  return 0;
}

int mbt_writer_potentials_due(const mbt_writer *w, long rev)
{
  const mbt_params *p = w ? &w->p : NULL;
  if (!w || w->n_out == 0 || !w->pot_fp[0]) return 0;
  /* the self-field step runs (worker_weakweak.c:264-265) */
  if (p->ncell <= 0 || p->planeL + p->planeV + p->planeH + p->n_lr[0] + p->n_lr[1] + p->n_lr[2] <= 0) return 0;
  return (rev + 1) % w->p.nrev_mon == 0 &&
         rev + 1 >= w->o.nrev_potentials_out + (rev / w->nrev_scan) * w->nrev_scan;
}

int mbt_writer_potentials(mbt_writer *w, int ibunch, long rev, const double *pot, double vrf0, double phai0)
{
  const mbt_params *p;
  FILE *fp = NULL;
  int i, icell, j, kb, nc;
  double eps_const, facI;
  if (!w || !pot) return werr(MBT_ERR_INVALID, "writer potentials: null argument");
  for (i = 0; i < w->n_out; i++)
    if (w->out[i] == ibunch) fp = w->pot_fp[i];
  if (!fp) return werr(MBT_ERR_INVALID, "writer potentials: bunch %d has no potentials file", ibunch);
  p = &w->p;
  nc = p->ncell;
  kb = w->bucket[ibunch];
  eps_const = vrf0 / (p->E0 * FKILO);
  facI = p->ideal_hc == 0 ? 0. : eps_const * p->HC_k;
  for (icell = 0; icell < nc; icell++) {
    const double taucell = -(-p->nsigma + p->dT * (icell - 0.5)) * p->sigma_tau;
    const double rftest = eps_const * sin(p->wrf * taucell + phai0) - p->Urad;
    double active = 0.0, ideal;
    for (j = 0; j < p->n_active_hc; j++)
      active += p->ahc_vpeak[j] / (p->E0 * FGIGA) *
                sin(p->wrf * p->ahc_nhc[j] * taucell + p->ahc_phi[j] + p->ahc_nhc[j] * kb * 2 * M_PI);
    ideal = facI * sin(p->m_aHC * p->wrf * taucell + p->m_aHC * p->phi_n);
    fprintf(fp, "\n %ld   %e   %e   %e    %e   %e   %e   %e   %e", rev + 1, w->scan_val_w, taucell, pot[icell],
            pot[nc + icell], rftest, active, ideal, pot[2 * nc + icell]);
    if (p->planeV > 0) fprintf(fp, "   %e   %e", pot[3 * nc + icell], pot[4 * nc + icell]);
    if (p->planeH > 0) fprintf(fp, "   %e   %e", pot[5 * nc + icell], pot[6 * nc + icell]);
  }
  fprintf(fp, "\n");
  return 0;
}

int mbt_writer_end(mbt_writer *w, const double *end_stats)
{
  static const char *const tag[3] = {"LON", "HOR", "VER"};
  FILE *fp;
  long rev;
  int b, pl;
  char name[256];
  if (!w || !end_stats) return werr(MBT_ERR_INVALID, "writer end: null argument");
  if (w->rev != w->p.nrev_tot)
    return werr(MBT_ERR_STATE, "writer end: %ld of %ld turns received", w->rev, w->p.nrev_tot);
  /* mean_bunch_end.dat, written when no scan runs (manager_weakweak.c:302) */
  if (w->p.scan == 0) {
    fp = open_in(w, "mean_bunch_end.dat", "w+");
    if (!fp) return werr(MBT_ERR_IO, "cannot create %s/mean_bunch_end.dat", w->dir);
    fprintf(fp, " # bunch statistics end of run, turns = %i; Ib = %g A ;\n", (int) w->rev, w->ib[0]);
    fprintf(fp, " # bunch_num    CM    bunch_length    energy_dev    energy_spread;\n");
    for (b = 0; b < w->nb; b++) {
      const double *s = end_stats + 12 * b;
      fprintf(fp, " %d     %e    %e    %e    %e\n", w->bucket[b], s[0], s[3], s[6], s[9]);
    }
    fclose(fp);
  }
  /* resistive-wall dipole history of the first output bunch */
  if (w->p.rw_long && w->n_out > 0) {
    int i, j;
    fp = open_in(w, "dipoles_history.dat", "w+");
    if (!fp) return werr(MBT_ERR_IO, "cannot create %s/dipoles_history.dat", w->dir);
    fprintf(fp, " # history of dipole moments at rev = %i; Ib = %g A ;\n", (int) w->rev, w->ib[w->out[0]]);
    fprintf(fp, " # Nhist  kb   rev   dipole_HOR    dipole_VER\n");
    for (j = 0; j < w->p.Nmlt; j++)
      for (i = 0; i < w->p.nharm; i++) {
        const long slot = ((long) j * w->p.nharm + i) % w->ndip;
        fprintf(fp, " %d    %d    %d           %e    %e \n", j * w->p.nharm + i, i, j, w->dip[slot][0],
                w->dip[slot][1]);
      }
    fclose(fp);
  }
  /* bunchbybunch_<P>.dat: LON always, HOR/VER when tracked */
  for (pl = 0; pl < 3; pl++) {
    if (!w->p.track_plane[pl]) continue;
    snprintf(name, sizeof name, "bunchbybunch_%s.dat", tag[pl]);
    fp = open_in(w, name, "w");
    if (!fp) return werr(MBT_ERR_IO, "cannot create %s/%s", w->dir, name);
    fprintf(fp, "# turn    position of bunch 1,2,3...\n");
    for (rev = w->p.nrev_mon; rev < w->p.nrev_tot + 1; rev += w->p.nrev_mon) {
      const long irevmon = rev / w->p.nrev_mon - 1;
      fprintf(fp, " %3ld %15.8e", rev, w->scan_hist[0]);
      for (b = 0; b < w->nb; b++) fprintf(fp, " %15.8e", hist_at(w, w->cm, irevmon * w->nb + b, pl));
      fprintf(fp, "\n");
    }
    fclose(fp);
  }
  /* ampinv_<P>_mean.dat: HOR, VER when tracked */
  for (pl = 1; pl < 3; pl++) {
    long m = 0;
    if (!w->p.track_plane[pl]) continue;
    snprintf(name, sizeof name, "ampinv_%s_mean.dat", tag[pl]);
    fp = open_in(w, name, "w");
    if (!fp) return werr(MBT_ERR_IO, "cannot create %s/%s", w->dir, name);
    fprintf(fp, "# turn   AVE_ampinv    AVE_ampinv_cm   current \n");
    for (rev = 0; rev < w->p.nrev_tot; rev += w->p.nrev_mon) {
      const long irevmon = rev / w->p.nrev_mon;
      double sum = 0.0, sum_cm = 0.0;
      int n = 0, jb;
      for (jb = 0; jb < w->p.nharm; jb++) {
        long e;
        if (w->bunch_of[jb] < 0) continue;
        e = irevmon * w->nb + ((w->flags & MBT_WRITER_OWN_AMPINV) ? w->bunch_of[jb] : jb);
        sum += hist_at(w, w->ai, e, pl);
        sum_cm += hist_at(w, w->aic, e, pl);
        n++;
      }
      fprintf(fp, " %3ld %15.8e %15.8e  %15.8e\n", rev, sum / (double) n, sum_cm / (double) n,
              m < w->m && m < w->nscan_hist ? w->scan_hist[m] : 0.0);
      m++;
    }
    fclose(fp);
  }
  return 0;
}

int mbt_writer_distribution(mbt_writer *w, int ibunch, const double *soa6, int np)
{
  static const double prefix_pos[3] = {FGIGA, FKILO, FKILO};
  static const double prefix_slope[3] = {1.0, FKILO, FKILO};
  int pl, jp;
  if (!w || !soa6 || np < 0 || ibunch < 0 || ibunch >= w->nb)
    return werr(MBT_ERR_INVALID, "writer distribution: bad argument");
  for (pl = 0; pl < 3; pl++) {
    FILE *fp;
    if (pl > 0 && !w->p.track_plane[pl]) continue;
    fp = fopen(w->o.gendst_file[pl], "w");
    if (!fp) return werr(MBT_ERR_IO, "cannot create %s", w->o.gendst_file[pl]);
    for (jp = 0; jp < np; jp++)
      fprintf(fp, "%5d %15.12g %15.12g\n", jp, soa6[(size_t) pl * np + jp] * prefix_pos[pl],
              soa6[(size_t) (3 + pl) * np + jp] * prefix_slope[pl]);
    fclose(fp);
  }
  return 0;
}

int mbt_writer_close(mbt_writer *w)
{
  int i;
  if (!w) return 0;
  if (w->all_fp) fclose(w->all_fp);
  for (i = 0; w->out_fp && i < w->n_out; i++) {
    if (w->out_fp[i]) fclose(w->out_fp[i]);
    if (w->pot_fp && w->pot_fp[i]) fclose(w->pot_fp[i]);
  }
  free(w->bucket);
  free(w->bunch_of);
  free(w->ib);
  free(w->out);
  free(w->out_fp);
  free(w->pot_fp);
  free(w->out_acc);
  free(w->nstat_out);
  free(w->cm);
  free(w->ai);
  free(w->aic);
  free(w->scan_hist);
  free(w->dip);
  free(w);
  return 0;
}
