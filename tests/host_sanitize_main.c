/*
 * host_sanitize_main.c -- drives the host C of libmbt (configuration
 * reader, Green's functions, generated beams, slicing, both writers)
 * without a device, for tests/test_host_sanitizers.py, which builds it with
 * AddressSanitizer and UndefinedBehaviorSanitizer.
 *
 *   host_sanitize_main WORKDIR WEAK.conf [WEAK.conf ...] -- STRONG.conf [...]
 *
 * Exits 0 when every call succeeds; the sanitizers abort on the first bad
 * access or undefined operation.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mbt.h"
#include "mbt_ws.h"

static int weak(const char *conf, const char *work)
{
  mbt_params p;
  mbt_output_cfg o;
  int nb = 0, i, r;
  if (mbt_config_bunch_model(conf) != 0) return 1;
  if (mbt_config_load(conf, 1, &p, &nb, NULL, NULL) != 0) return 2;
  int *bucket = calloc(p.nharm, sizeof(int)), *bout = calloc(p.nharm, sizeof(int));
  double *frac = calloc(p.nharm, sizeof(double)), *ib = calloc(nb, sizeof(double));
  double *G = calloc(3 * (p.ncell > 0 ? p.ncell : 1), sizeof(double));
  if (mbt_config_load(conf, 1, &p, &nb, bucket, frac) != 0 || mbt_config_output(conf, &o, bout) != 0) return 3;
  if (p.ncell > 0 && mbt_config_greens(conf, &p, G, G + p.ncell, G + 2 * p.ncell) != 0) return 4;
  for (i = 0; i < nb; i++) ib[i] = mbt_bunch_current(&p, nb, frac[i]);
  {
    const int np = p.np_model < 2000 ? p.np_model : 2000;
    double *soa = malloc(6 * (size_t) np * sizeof(double));
    for (i = 0; i < nb && i < 3; i++)
      if (mbt_reference_beam(&p, bucket[i], np, soa) != 0) return 5;
    free(soa);
  }
  {
    /* a short run: the writer checks it received every turn */
    mbt_params q = p;
    mbt_writer *w;
    const long n = 4;
    q.nrev_tot = n;
    q.nrev_mon = 2;
    double *st = calloc((size_t) n * nb * 12, sizeof(double)), *ai = calloc((size_t) n * nb * 6, sizeof(double));
    for (i = 0; i < nb * 12; i++) st[i] = 1e-3 * (i % 7 + 1);
    if (mbt_writer_open(work, &q, &o, bout, nb, bucket, ib, 0, &w) != 0) return 6;
    if (p.ncell > 0 && mbt_writer_wakes(w, G, G + p.ncell, G + 2 * p.ncell) != 0) return 7;
    if (mbt_writer_begin(w, st) != 0) return 8;
    for (i = 0; i < n; i++) {
      r = mbt_writer_turns(w, 1, st, ai);
      if (r != 0) return 9;
    }
    if (mbt_writer_end(w, st) != 0) {
      fprintf(stderr, "writer: %s\n", mbt_writer_error());
      return 10;
    }
    mbt_writer_close(w);
    free(st);
    free(ai);
  }
  free(bucket); free(bout); free(frac); free(ib); free(G);
  return 0;
}

static int strong(const char *conf, const char *work)
{
  mbt_ws_params w;
  int nb = 0, i;
  if (mbt_config_bunch_model(conf) != 1) return 11;
  if (mbt_ws_config_load(conf, 1, &w, &nb, NULL, NULL) != 0) return 12;
  int *bucket = calloc(w.base.nharm, sizeof(int));
  double *frac = calloc(w.base.nharm, sizeof(double));
  if (mbt_ws_config_load(conf, 1, &w, &nb, bucket, frac) != 0) return 13;
  const int S = 2 * w.nslc + 1, G = w.ngrid;
  double *soa = malloc(6 * (size_t) w.np * sizeof(double)), *off = malloc(4 * (size_t) nb * sizeof(double));
  int *npop = malloc(S * sizeof(int)), *nofe = malloc((size_t) S * G * G * sizeof(int));
  double *cm4 = malloc(4 * (size_t) S * sizeof(double));
  if (mbt_ws_reference_beam(&w, nb, soa, off) != 0) return 14;
  if (mbt_ws_slice_beam(&w, soa, w.np, npop, nofe, cm4) != 0) return 15;
  {
    mbt_ws_writer *wr;
    const long n = w.base.nrev_mon + 1;
    double *ion = calloc((size_t) n * nb * 2, sizeof(double)), *zcm = calloc((size_t) n * w.base.nharm, sizeof(double));
    double *st = calloc((size_t) 2 * nb * 18, sizeof(double));
    const char *paths[3];
    char g[3][512];
    for (i = 0; i < 3; i++) {
      snprintf(g[i], sizeof g[i], "%s/gendst_%d", work, i);
      paths[i] = g[i];
    }
    if (mbt_ws_writer_open(work, &w, nb, bucket, 0, &wr) != 0) return 16;
    if (mbt_ws_writer_distribution(wr, paths, soa, w.np) != 0) return 17;
    if (mbt_ws_writer_turns(wr, n, ion, zcm, st) != 0) return 18;
    if (mbt_ws_writer_close(wr) != 0) return 19;
    free(ion); free(zcm); free(st);
  }
  free(bucket); free(frac); free(soa); free(off); free(npop); free(nofe); free(cm4);
  return 0;
}

int main(int argc, char **argv)
{
  int i, r, strong_part = 0;
  double a, b;
  if (argc < 3) return 64;
  for (i = 0; i < 40; i++)
    if (mbt_rw_first_bin(20.0 + 60.0 * i, &a, &b) != 0) return 20;
  for (i = 2; i < argc; i++) {
    if (strcmp(argv[i], "--") == 0) { strong_part = 1; continue; }
    r = strong_part ? strong(argv[i], argv[1]) : weak(argv[i], argv[1]);
    if (r) {
      fprintf(stderr, "%s: step %d failed (%s)\n", argv[i], r, mbt_config_error());
      return r;
    }
  }
  printf("host calls ok\n");
  return 0;
}
