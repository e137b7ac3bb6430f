/*
 * mbt_ws_output.c -- the files the reference's slice-model manager writes
 * (manager_weakstrong.c:100-256), from the outputs of mbt_ws_run_turns.
 *
 *   CMImotionsH.out, CMImotionsV.out  writeoutCMImotions fbi_weakstrong.c:583-669
 *                                     (with EnableFBII): per turn "%3d: " and per
 *                                     bunch the ion centroid in units of the beam
 *                                     size, " %12.8lf"
 *   CMmotionsV.out                    writeoutVCMmotionsPM2 :672-737: per turn the
 *                                     mean slice z of every bucket x 1e7, "%-15.8lf "
 *   ampinv_<P>_<turn>.dat             bunch_strong_writeout_ampinv bunch.c:645-702
 *                                     every NrevMon turns, tracked planes
 *   ampinv_<P>_mean.dat, cmpos_<P>_mean.dat
 *                                     bunch_writeout_mean_ampinv_pos bunch.c:704-770
 *                                     after the run, HOR and VER
 *   gendst_datafile_<P>               the generated bunch (generate_initial_sbunch_
 *                                     distribution2 bunch.c:314-331)
 *
 * The manager keeps the monitor statistics in arrays indexed by monitor x
 * Nbunch + bucket (manager_weakstrong.c:131-138) and prints the per-monitor
 * ampinv files from entry monitor + bucket (bunch.c:599-601): for a fill
 * of the first Nbunch buckets that is bunch jb's entry only at the first
 * monitor.  The writer keeps the same array and indexing by default,
 * printing 0 where the reference would read or write past its array;
 * MBT_WRITER_OWN_AMPINV prints each bunch's own values.
 */
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mbt.h"
#include "mbt_ws.h"

struct mbt_ws_writer {
  mbt_ws_params w;
  int nb, flags;
  int *bucket;
  char path[1024];
  FILE *cmi[2], *cmv;
  long rev;
  long nslot;            /* NrevTot / NrevMon x Nbunch + 2 (bunch_CM_history_strong_init) */
  double *hist;          /* [nslot][18]: cm, rms, cm_slope, rms_slope, ampinv, ampinv_cm */
  char err[512];
};

static char g_wserr[512] = "";

static int wsfail(mbt_ws_writer *wr, int code, const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(wr ? wr->err : g_wserr, 512, fmt, ap);
  va_end(ap);
  if (wr) memcpy(g_wserr, wr->err, sizeof g_wserr);
  return code;
}

const char *mbt_ws_writer_error(void) { return g_wserr; }

static FILE *wopen(mbt_ws_writer *wr, const char *name)
{
  char f[1200];
  snprintf(f, sizeof f, "%s/%s", wr->path, name);
  return fopen(f, "w");
}

int mbt_ws_writer_open(const char *work_path, const mbt_ws_params *w, int nbunch, const int *bucket, int flags,
                       mbt_ws_writer **out)
{
  mbt_ws_writer *wr;
  if (!out || !w || !bucket || nbunch < 1 || !work_path) return wsfail(NULL, MBT_ERR_INVALID, "bad arguments");
  *out = NULL;
  wr = (mbt_ws_writer *) calloc(1, sizeof(*wr));
  if (!wr) return wsfail(NULL, MBT_ERR_NOMEM, "out of host memory");
  wr->w = *w;
  wr->nb = nbunch;
  wr->flags = flags;
  snprintf(wr->path, sizeof wr->path, "%s", work_path);
  wr->bucket = (int *) malloc(nbunch * sizeof(int));
  wr->nslot = (w->base.nrev_tot / w->base.nrev_mon) * nbunch + 2;
  wr->hist = (double *) calloc((size_t) wr->nslot * 18, sizeof(double));
  if (!wr->bucket || !wr->hist) { mbt_ws_writer_close(wr); return wsfail(NULL, MBT_ERR_NOMEM, "out of host memory"); }
  memcpy(wr->bucket, bucket, nbunch * sizeof(int));
  wr->cmv = wopen(wr, "CMmotionsV.out");
  if (w->fbii) {
    wr->cmi[0] = wopen(wr, "CMImotionsH.out");
    wr->cmi[1] = wopen(wr, "CMImotionsV.out");
  }
  if (!wr->cmv || (w->fbii && (!wr->cmi[0] || !wr->cmi[1]))) {
    mbt_ws_writer_close(wr);
    return wsfail(NULL, MBT_ERR_IO, "cannot create the motion files in %s", work_path);
  }
  *out = wr;
  return 0;
}

/* bunch_fprint_ampinv bunch.c:552-590 for one monitor */
static int write_ampinv(mbt_ws_writer *wr, long rev, long mon, const double *stats)
{
  static const char *pn[3] = {"LON", "HOR", "VER"};
  int pl, i;
  for (pl = 0; pl < 3; pl++) {
    char name[64];
    FILE *fp;
    if (!wr->w.base.track_plane[pl]) continue;
    snprintf(name, sizeof name, "ampinv_%s_%ld.dat", pn[pl], rev + 1);
    fp = wopen(wr, name);
    if (!fp) return wsfail(wr, MBT_ERR_IO, "cannot create %s", name);
    fprintf(fp, "# turn: %-5ld\n", rev + 1);
    fprintf(fp, "# bunch   ampinv_cm   ampinv\n");
    for (i = 0; i < wr->nb; i++) {
      double cm, ai;
      if (wr->flags & MBT_WRITER_OWN_AMPINV) {
        cm = stats[i * 18 + 15 + pl];
        ai = stats[i * 18 + 12 + pl];
      } else {
        const long k = mon + wr->bucket[i];
        cm = k < wr->nslot ? wr->hist[k * 18 + 15 + pl] : 0.0;
        ai = k < wr->nslot ? wr->hist[k * 18 + 12 + pl] : 0.0;
      }
      fprintf(fp, " %3d %15.8e %15.8e\n", wr->bucket[i], cm, ai);
    }
    fclose(fp);
  }
  return 0;
}

int mbt_ws_writer_turns(mbt_ws_writer *wr, long nturns, const double *ion, const double *zcm, const double *stats)
{
  long t, imon = 0;
  int i, nh;
  if (!wr || nturns < 0 || !zcm || (wr->w.fbii && !ion)) return wsfail(wr, MBT_ERR_INVALID, "bad arguments");
  nh = wr->w.base.nharm;
  for (t = 0; t < nturns; t++, wr->rev++) {
    const long rev = wr->rev;
    if (rev % wr->w.base.nrev_mon == 0 && stats) {
      const long mon = rev / wr->w.base.nrev_mon;
      const double *st = stats + (size_t) imon * wr->nb * 18;
      for (i = 0; i < wr->nb; i++) {
        const long k = mon * wr->nb + wr->bucket[i];
        if (k < wr->nslot) memcpy(wr->hist + k * 18, st + (size_t) i * 18, 18 * sizeof(double));
      }
      if (write_ampinv(wr, rev, mon, st) != 0) return MBT_ERR_IO;
      imon++;
    }
    if (wr->w.fbii) {
      int pl;
      for (pl = 0; pl < 2; pl++) {
        const double sg = pl == 0 ? wr->w.sgm_xx : wr->w.sgm_zz;
        fprintf(wr->cmi[pl], "%3d: ", (int) rev);
        for (i = 0; i < wr->nb; i++) {
          const double v = ion[((size_t) t * wr->nb + i) * 2 + pl];
          fprintf(wr->cmi[pl], " %12.8lf", isnan(v) ? v : 1.0e+03 * v / sg);
        }
        putc(0x0a, wr->cmi[pl]);
      }
    }
    for (i = 0; i < nh; i++) fprintf(wr->cmv, "%-15.8lf ", 10000.0 * 1.0e+03 * zcm[(size_t) t * nh + i]);
    fprintf(wr->cmv, "\n");
  }
  return 0;
}

int mbt_ws_writer_distribution(const mbt_ws_writer *wr, const char *const *paths, const double *soa6, int np)
{
  int pl, j;
  if (!wr || !paths || !soa6 || np < 1) return wsfail(NULL, MBT_ERR_INVALID, "bad arguments");
  for (pl = 0; pl < 3; pl++) {
    const double *u = soa6 + (size_t) pl * np, *up = soa6 + (size_t) (3 + pl) * np;
    FILE *fp = fopen(paths[pl], "w");
    if (!fp) return wsfail(NULL, MBT_ERR_IO, "Error ! Cannot open %s", paths[pl]);
    for (j = 0; j < np; j++) {
      if (pl == 0) fprintf(fp, "%5d %15.12g %15.12g\n", j, u[j] / 1.0e-09, up[j]);
      else fprintf(fp, "%5d %15.12g %15.12g\n", j, u[j] / 1.0e-03, up[j] / 1.0e-03);
    }
    fclose(fp);
  }
  return 0;
}

/* bunch_writeout_mean_ampinv_pos bunch.c:704-770 */
static int write_means(mbt_ws_writer *wr)
{
  int pl;
  for (pl = 1; pl <= 2; pl++) {
    char a[64], b[64];
    FILE *fp, *fq;
    long rev;
    if (!wr->w.base.track_plane[pl]) continue;
    snprintf(a, sizeof a, "ampinv_%s_mean.dat", pl == 1 ? "HOR" : "VER");
    snprintf(b, sizeof b, "cmpos_%s_mean.dat", pl == 1 ? "HOR" : "VER");
    fp = wopen(wr, a);
    fq = wopen(wr, b);
    if (!fp || !fq) {
      if (fp) fclose(fp);
      if (fq) fclose(fq);
      return wsfail(wr, MBT_ERR_IO, "cannot create %s", a);
    }
    for (rev = 0; rev < wr->w.base.nrev_tot; rev += wr->w.base.nrev_mon) {
      const long mon = rev / wr->w.base.nrev_mon;
      double sp = 0.0, sa = 0.0, sc = 0.0;
      int i, n = 0;
      for (i = 0; i < wr->nb; i++) {
        const long k = mon * wr->nb + wr->bucket[i];
        if (k < wr->nslot) {
          sp += wr->hist[k * 18 + pl];
          sa += wr->hist[k * 18 + 12 + pl];
          sc += wr->hist[k * 18 + 15 + pl];
        }
        n++;
      }
      fprintf(fp, " %3ld %15.8e %15.8e\n", rev, sa / (double) n, sc / (double) n);
      fprintf(fq, " %3ld %15.8e\n", rev, sp / (double) n);
    }
    fclose(fp);
    fclose(fq);
  }
  return 0;
}

int mbt_ws_writer_close(mbt_ws_writer *wr)
{
  int r = 0;
  if (!wr) return 0;
  if (wr->hist && wr->cmv) r = write_means(wr);
  if (wr->cmv) fclose(wr->cmv);
  if (wr->cmi[0]) fclose(wr->cmi[0]);
  if (wr->cmi[1]) fclose(wr->cmi[1]);
  free(wr->bucket);
  free(wr->hist);
  free(wr);
  return r;
}
