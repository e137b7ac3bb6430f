/*
 * mbtrack_gpu.c -- `mbtrack-gpu input.conf [/path/to/work]`: the run of
 * mbtrack-mpi (mbtrack-mpi.c:22-160) on one GPU, without MPI and without the
 * rank-count check of mbtrack-mpi.c:85-90: manager_weakweak /
 * worker_weakweak for BunchModel = WEAK, manager_weakstrong /
 * worker_weakstrong (the slice model with fast beam-ion interaction,
 * mbt_ws.h) for BunchModel = STRONG.  The slice model runs with the bunch
 * currents of the fill (the reference's slice-model manager never sets
 * ring.Ibunch, so its charges, ions and wall kicks are all zero).
 *
 * The arguments, the terminal messages and the files in the work directory
 * are the reference's.  Options (anywhere on the command line):
 *   --own-ampinv    ampinv files show each bunch's own invariants (the
 *                   reference's history indexing otherwise)
 *   --seed N        key of the counter-based quantum-excitation noise
 *                   (default: iseed_LON)
 *   --device N      CUDA device (default 0)
 *   --np-by-charge MIN:MAX:TOTAL   macroparticles of each bunch proportional
 *                   to its charge, clamped to [MIN, MAX], about TOTAL in all
 *                   (the reference has one Np for every bunch)
 *   --train-steps N training steps of the learned field (default 20000)
 * A [beam_ion] section (mbt_config_beam_ion) adds the per-macroparticle
 * beam-ion stage; with surrogate = 1 the learned field is trained first
 * (1e7 samples of the Faddeeva field) and its audit is printed at the end.
 * The initial distribution is the reference's (same generator, same seeds).
 * The quantum-excitation noise is a Philox stream instead of glibc rand():
 * with EnableQuantum = 0 the run reproduces the reference's numbers, with
 * noise it reproduces their statistics.
 */
#define _DEFAULT_SOURCE
#include <pthread.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "mbt.h"
#include "mbt_ws.h"

typedef struct beam_job {
  const mbt_params *p;
  const int *bucket;
  const int *np;
  const size_t *start;
  double *all;
  int nb, next, err;
  pthread_mutex_t lock;
} beam_job;

static void *beam_worker(void *arg)
{
  beam_job *j = (beam_job *) arg;
  for (;;) {
    int b, r;
    pthread_mutex_lock(&j->lock);
    b = j->next++;
    pthread_mutex_unlock(&j->lock);
    if (b >= j->nb) return NULL;
    r = mbt_reference_beam(j->p, j->bucket[b], j->np[b], j->all + j->start[b]);
    if (r) j->err = r;
  }
}

/* every bunch's reference distribution, bunch after bunch (soa6 blocks),
 * generated on the host cores */
static int reference_beam_all(const mbt_params *p, int nb, const int *bucket, const int *np, double *all)
{
  beam_job j;
  pthread_t th[256];
  size_t *start = (size_t *) malloc((nb + 1) * sizeof(size_t));
  long ncpu = sysconf(_SC_NPROCESSORS_ONLN);
  int i, nt;
  if (!start) return MBT_ERR_NOMEM;
  start[0] = 0;
  for (i = 0; i < nb; i++) start[i + 1] = start[i] + (size_t) 6 * np[i];
  memset(&j, 0, sizeof j);
  j.p = p; j.bucket = bucket; j.np = np; j.start = start; j.all = all; j.nb = nb;
  pthread_mutex_init(&j.lock, NULL);
  nt = (int) (ncpu < 1 ? 1 : ncpu > 256 ? 256 : ncpu);
  if (nt > nb) nt = nb;
  for (i = 0; i < nt; i++) pthread_create(&th[i], NULL, beam_worker, &j);
  for (i = 0; i < nt; i++) pthread_join(th[i], NULL);
  pthread_mutex_destroy(&j.lock);
  free(start);
  return j.err;
}

static void ctx_error(mbt_ctx *ctx, const char *what)
{
  char msg[512];
  mbt_last_error(ctx, msg, sizeof msg);
  fprintf(stderr, "ERROR: %s: %s\n", what, msg);
}

/* manager_weakstrong.c:7-263 with worker_weakstrong.c:13-247 */
static int run_strong(const char *conf, const char *work, int own_ampinv)
{
  mbt_ws_params w;
  mbt_output_cfg o;
  mbt_ws *ws = NULL;
  mbt_ws_writer *wr = NULL;
  int nb = 0, i, k, c, S, G;
  int *bucket, *npop, *nofe;
  double *frac, *ib, *soa6, *off4, *cm4, *sl, *ion, *zcm, *stats;
  long rev, chunk = 256;
  const char *gendst[3];

  if (mbt_ws_config_load(conf, 1, &w, &nb, NULL, NULL) != 0) {
    fprintf(stderr, "ERROR: read_input failed: %s\n", mbt_config_error());
    return -1;
  }
  bucket = (int *) calloc(w.base.nharm, sizeof(int));
  frac = (double *) calloc(w.base.nharm, sizeof(double));
  if (!bucket || !frac || mbt_ws_config_load(conf, 1, &w, &nb, bucket, frac) != 0 ||
      mbt_config_output(conf, &o, NULL) != 0) {
    fprintf(stderr, "ERROR: read_input failed: %s\n", mbt_config_error());
    return -1;
  }
  if (nb <= 0) { fprintf(stderr, "ERROR: e_beam_setup: no filled bucket\n"); return -1; }
  S = 2 * w.nslc + 1;
  G = w.ngrid;
  printf("Starting job \"%s\"\n\n", o.jobtitle);
  printf("Generating initial distribution...\n");
  ib = (double *) malloc(nb * sizeof(double));
  soa6 = (double *) malloc((size_t) 6 * w.np * sizeof(double));
  off4 = (double *) malloc((size_t) 4 * nb * sizeof(double));
  npop = (int *) malloc(S * sizeof(int));
  nofe = (int *) malloc((size_t) S * G * G * sizeof(int));
  cm4 = (double *) malloc((size_t) 4 * S * sizeof(double));
  sl = (double *) calloc((size_t) nb * 6 * S, sizeof(double));
  ion = (double *) malloc((size_t) chunk * nb * 2 * sizeof(double));
  zcm = (double *) malloc((size_t) chunk * w.base.nharm * sizeof(double));
  stats = (double *) malloc((size_t) chunk * nb * 18 * sizeof(double));
  if (!ib || !soa6 || !off4 || !npop || !nofe || !cm4 || !sl || !ion || !zcm || !stats) {
    fprintf(stderr, "ERROR: out of host memory\n");
    return -1;
  }
  for (i = 0; i < nb; i++) ib[i] = 1.0e+03 * mbt_bunch_current(&w.base, nb, frac[i]);
  /* strong_generate_eCMs (with its distribution files) and
     generate_initial_general_distribution2 */
  if (mbt_ws_reference_beam(&w, nb, soa6, off4) != 0 || mbt_ws_slice_beam(&w, soa6, w.np, npop, nofe, cm4) != 0) {
    fprintf(stderr, "ERROR: generate_eCMs failed\n");
    return -1;
  }
  for (i = 0; i < nb; i++)
    for (k = 0; k < 4; k++)
      for (c = 0; c < S; c++) sl[((size_t) i * 6 + 2 + k) * S + c] = cm4[k * S + c] + off4[4 * i + k];
  if (mbt_ws_create(&w, nb, bucket, ib, npop, nofe, &ws) != 0) {
    fprintf(stderr, "ERROR: mbt_ws_create: %s\n", mbt_ws_last_error(NULL));
    return -1;
  }
  if (mbt_ws_load_slices(ws, sl) != 0) { fprintf(stderr, "ERROR: %s\n", mbt_ws_last_error(ws)); return -1; }
  if (mbt_ws_writer_open(work, &w, nb, bucket, own_ampinv ? MBT_WRITER_OWN_AMPINV : 0, &wr) != 0) {
    fprintf(stderr, "ERROR: %s\n", mbt_ws_writer_error());
    return -1;
  }
  for (k = 0; k < 3; k++) gendst[k] = o.gendst_file[k];
  if (mbt_ws_writer_distribution(wr, gendst, soa6, w.np) != 0) {
    fprintf(stderr, "%s\nERROR: generate_eCMs failed\n", mbt_ws_writer_error());
    return -1;
  }
  printf("Starting multi bunch tracking...\n");
  for (rev = 0; rev < w.base.nrev_tot;) {
    const long n = w.base.nrev_tot - rev < chunk ? w.base.nrev_tot - rev : chunk;
    long t;
    if (mbt_ws_run_turns(ws, n, NULL, ion, zcm, stats) != 0) {
      fprintf(stderr, "ERROR: %s\n", mbt_ws_last_error(ws));
      return -1;
    }
    if (mbt_ws_writer_turns(wr, n, ion, zcm, stats) != 0) {
      fprintf(stderr, "ERROR: %s\n", mbt_ws_writer_error());
      return -1;
    }
    /* terminal output of manager_weakstrong.c:84-92, 236-240 */
    for (t = rev; t < rev + n; t++) {
      if (t % 100 == 0) {
        if (t + 99 >= w.base.nrev_tot) printf("Transformation for turn %3ld to %3ld", t, w.base.nrev_tot - 1);
        else printf("Transformation for turn %3ld to %3ld", t, t + 99);
        fflush(stdout);
      }
      if (t % 10 == 9) printf(".");
      fflush(stdout);
      if (t % 100 == 99 || t == w.base.nrev_tot - 1) printf(" done\n");
    }
    rev += n;
  }
  if (mbt_ws_writer_close(wr) != 0) fprintf(stderr, "ERROR: %s\n", mbt_ws_writer_error());
  mbt_ws_destroy(ws);
  free(bucket); free(frac); free(ib); free(soa6); free(off4); free(npop); free(nofe); free(cm4); free(sl);
  free(ion); free(zcm); free(stats);
  return 0;
}

/* macroparticles proportional to the bunch charge, clamped to [lo, hi],
 * summing to about `total` (bisection on the proportionality factor) */
static int set_np_by_charge(int nb, const double *frac, long lo, long hi, long total, int *np)
{
  double k0 = 1e-6, k1 = 1e15, k, fsum = 0.0;
  int i, it;
  for (i = 0; i < nb; i++) fsum += frac[i];
  if (!(fsum > 0.0)) return -1;
  for (it = 0; it < 200; it++) {
    double sum = 0.0;
    k = sqrt(k0 * k1);
    for (i = 0; i < nb; i++) {
      double n = floor(k * frac[i] + 0.5);
      sum += n < lo ? lo : n > hi ? hi : n;
    }
    if (sum < (double) total) k0 = k; else k1 = k;
  }
  k = sqrt(k0 * k1);
  for (i = 0; i < nb; i++) {
    double n = floor(k * frac[i] + 0.5);
    np[i] = (int) (n < lo ? lo : n > hi ? hi : n);
  }
  return 0;
}

int main(int argc, char **argv)
{
  const char *conf = NULL, *work = "work/";
  int own_ampinv = 0, device = 0, have_seed = 0, npos = 0, i, r, nb = 0, train_steps = 20000;
  long np_min = 0, np_max = 0, np_total = 0;
  mbt_beam_ion bi;
  mbt_mlp *mlp = NULL;
  int bi_on = 0;
  unsigned long long seed = 0;
  mbt_params p;
  mbt_output_cfg o;
  int *bucket = NULL, *np = NULL, *bunch_out = NULL, *watch = NULL, nwatch = 0;
  double *frac = NULL, *ib = NULL, *Gl = NULL, *Gv = NULL, *Gh = NULL, *beam = NULL;
  double *init_stats = NULL, *stats = NULL, *ampinv = NULL, *pot = NULL;
  size_t nbeam = 0;
  long rev, chunk;
  mbt_ctx *ctx = NULL;
  mbt_writer *w = NULL;
  mbt_state st;
  time_t now;
  struct tm *tnow;

  for (i = 1; i < argc; i++) {
    if (strcmp(argv[i], "--own-ampinv") == 0) own_ampinv = 1;
    else if (strcmp(argv[i], "--seed") == 0 && i + 1 < argc) { seed = strtoull(argv[++i], NULL, 0); have_seed = 1; }
    else if (strcmp(argv[i], "--device") == 0 && i + 1 < argc) device = atoi(argv[++i]);
    else if (strcmp(argv[i], "--train-steps") == 0 && i + 1 < argc) train_steps = atoi(argv[++i]);
    else if (strcmp(argv[i], "--np-by-charge") == 0 && i + 1 < argc) {
      if (sscanf(argv[++i], "%ld:%ld:%ld", &np_min, &np_max, &np_total) != 3 || np_min < 1 || np_max < np_min ||
          np_total < 1) {
        fprintf(stderr, "ERROR: --np-by-charge MIN:MAX:TOTAL\n");
        return -1;
      }
    }
    else if (npos == 0) { conf = argv[i]; npos++; }
    else if (npos == 1) { work = argv[i]; npos++; }
    else npos = 3;
  }
  if (npos < 1 || npos > 2) {
    fprintf(stderr, "ERROR ! \n\nUsage:\nmbtrack-gpu inputfile.conf [/path/to/work] [--own-ampinv] [--seed N] [--device N]"
                    " [--np-by-charge MIN:MAX:TOTAL] [--train-steps N]\n");
    return -1;
  }
  if (mbt_use_device(device) != 0) {
    ctx_error(NULL, "device");
    return -1;
  }

  /* read_input + setup_* (mbtrack-mpi.c:61-97), checked */
  r = mbt_config_bunch_model(conf);
  if (r < 0) {
    fprintf(stderr, "ERROR: read_input failed: %s\n", mbt_config_error());
    return -1;
  }
  if (r == 1) return run_strong(conf, work, own_ampinv);
  if (mbt_config_load(conf, 1, &p, &nb, NULL, NULL) != 0) {
    fprintf(stderr, "ERROR: read_input failed: %s\n", mbt_config_error());
    return -1;
  }
  bucket = (int *) calloc(p.nharm, sizeof(int));
  frac = (double *) calloc(p.nharm, sizeof(double));
  bunch_out = (int *) calloc(p.nharm, sizeof(int));
  np = (int *) calloc(nb > 0 ? nb : 1, sizeof(int));
  ib = (double *) calloc(nb > 0 ? nb : 1, sizeof(double));
  if (!bucket || !frac || !bunch_out || !np || !ib) { fprintf(stderr, "ERROR: out of host memory\n"); return -1; }
  if (mbt_config_load(conf, 1, &p, &nb, bucket, frac) != 0 || mbt_config_output(conf, &o, bunch_out) != 0) {
    fprintf(stderr, "ERROR: read_input failed: %s\n", mbt_config_error());
    return -1;
  }
  if (nb <= 0) { fprintf(stderr, "ERROR: e_beam_setup: no filled bucket\n"); return -1; }
  if (p.ncell > 0) {
    Gl = (double *) calloc(p.ncell, sizeof(double));
    Gv = (double *) calloc(p.ncell, sizeof(double));
    Gh = (double *) calloc(p.ncell, sizeof(double));
    if (!Gl || !Gv || !Gh || mbt_config_greens(conf, &p, Gl, Gv, Gh) != 0) {
      fprintf(stderr, "ERROR: Green's functions: %s\n", mbt_config_error());
      return -1;
    }
  }

  printf("Starting job \"%s\"\n\n", o.jobtitle);
  printf("Generating initial distribution...\n");
  for (i = 0; i < nb; i++) {
    np[i] = p.np_model;                              /* manager_weakweak.c:61 */
    ib[i] = mbt_bunch_current(&p, nb, frac[i]);     /* manager_weakweak.c:74-75 */
  }
  if (np_total > 0 && set_np_by_charge(nb, frac, np_min, np_max, np_total, np) != 0) {
    fprintf(stderr, "ERROR: --np-by-charge: no bunch charge\n");
    return -1;
  }
  for (i = 0; i < nb; i++) nbeam += (size_t) 6 * np[i];
  beam = (double *) malloc(nbeam * sizeof(double));
  if (!beam) { fprintf(stderr, "ERROR: out of host memory for %zu coordinates\n", nbeam); return -1; }
  if ((r = reference_beam_all(&p, nb, bucket, np, beam)) != 0) {
    fprintf(stderr, "ERROR: weak_generate_bunch_distribution (%d)\n", r);
    return -1;
  }

  if (!have_seed) seed = (unsigned long long) (unsigned) p.iseed[0];
  if (mbt_create(&p, nb, bucket, np, ib, Gl, Gv, Gh, MBT_NOISE_PHILOX, seed, &ctx) != 0) {
    ctx_error(NULL, "mbt_create");
    return -1;
  }
  if (mbt_load_all(ctx, beam) != 0) { ctx_error(ctx, "loading the beam"); return -1; }

  /* the beam-ion stage (an extension of the weak-weak model) */
  r = mbt_config_beam_ion(conf, &bi);
  if (r < 0) { fprintf(stderr, "ERROR: [beam_ion]: %s\n", mbt_config_error()); return -1; }
  if (r == 0) {
    bi_on = 1;
    if (mbt_enable_beam_ion(ctx, &bi) != 0) { ctx_error(ctx, "mbt_enable_beam_ion"); return -1; }
    if (bi.surrogate) {
      printf("Training the learned beam-ion field (%d steps)...\n", train_steps);
      fflush(stdout);
      if (mbt_mlp_create(seed ^ 0x6D6C70ull, &mlp) != 0 ||
          mbt_mlp_train(mlp, 10000000L, 8192, train_steps, 2e-3f, seed + 1, NULL) != 0 ||
          mbt_beam_ion_use_mlp(ctx, mlp) != 0) {
        ctx_error(ctx, "learned field");
        return -1;
      }
    }
  }

  /* the output bunches */
  watch = (int *) calloc(nb, sizeof(int));
  for (i = 0; i < nb && watch; i++) {
    int j;
    for (j = 0; j < o.n_out; j++)
      if (bunch_out[j] == bucket[i] && nwatch < MBT_MAX_WATCH) { watch[nwatch++] = i; break; }
  }
  if (o.nrev_potentials_out <= p.nrev_tot && nwatch > 0 && mbt_watch_potentials(ctx, nwatch, watch) != 0) {
    ctx_error(ctx, "mbt_watch_potentials");
    return -1;
  }
  init_stats = (double *) malloc((size_t) nb * 12 * sizeof(double));
  if (!init_stats || mbt_prepare(ctx, init_stats) != 0) { ctx_error(ctx, "mbt_prepare"); return -1; }
  if (mbt_writer_open(work, &p, &o, bunch_out, nb, bucket, ib, own_ampinv ? MBT_WRITER_OWN_AMPINV : 0, &w) != 0 ||
      mbt_writer_wakes(w, Gl, Gv, Gh) != 0 || mbt_writer_begin(w, init_stats) != 0) {
    fprintf(stderr, "ERROR: %s\n", mbt_writer_error());
    return -1;
  }

  printf("Starting multi bunch tracking...\n");
  /* blocks of turns bounded by the host buffers and by the turns whose
   * potentials are printed (they are read before such a turn runs) */
  chunk = (long) (64L * 1024 * 1024 / ((size_t) nb * 18 * sizeof(double)));
  if (chunk < 1) chunk = 1;
  if (chunk > p.nrev_tot) chunk = p.nrev_tot > 0 ? p.nrev_tot : 1;
  stats = (double *) malloc((size_t) chunk * nb * 12 * sizeof(double));
  ampinv = (double *) malloc((size_t) chunk * nb * 6 * sizeof(double));
  pot = (double *) malloc((size_t) 7 * (p.ncell > 0 ? p.ncell : 1) * sizeof(double));
  if (!stats || !ampinv || !pot) { fprintf(stderr, "ERROR: out of host memory\n"); return -1; }
  for (rev = 0; rev < p.nrev_tot;) {
    long n = 1, k;
    if (mbt_writer_potentials_due(w, rev)) {
      if (mbt_get_state(ctx, &st) != 0) { ctx_error(ctx, "mbt_get_state"); return -1; }
      for (i = 0; i < nwatch; i++)
        if (mbt_get_potentials(ctx, watch[i], pot) != 0 ||
            mbt_writer_potentials(w, watch[i], rev, pot, st.Vrf0, st.phai0) != 0) {
          fprintf(stderr, "ERROR: potentials of turn %ld\n", rev);
          return -1;
        }
    }
    while (n < chunk && rev + n < p.nrev_tot && !mbt_writer_potentials_due(w, rev + n)) n++;
    if (mbt_run_turns_ampinv(ctx, n, stats, ampinv) != 0) { ctx_error(ctx, "mbt_run_turns"); return -1; }
    if (mbt_writer_turns(w, n, stats, ampinv) != 0) { fprintf(stderr, "ERROR: %s\n", mbt_writer_error()); return -1; }
    /* terminal output of manager_weakweak.c:181-188, 309-318 */
    for (k = rev; k < rev + n; k++) {
      if (k % 5000 == 0) {
        if (k + 4999 >= p.nrev_tot) printf("Transformation for turn %3ld to %3ld", k, p.nrev_tot - 1);
        else printf("Transformation for turn %3ld to %3ld", k, k + 4999);
        fflush(stdout);
      }
      if (k % 500 == 499) printf(".");
      fflush(stdout);
      if (k % 5000 == 4999 || k == p.nrev_tot - 1) {
        time(&now);
        tnow = localtime(&now);
        printf(" done (at time: %d:%d:%d)\n", tnow->tm_hour, tnow->tm_min, tnow->tm_sec);
      }
    }
    rev += n;
  }

  if (mbt_get_stats(ctx, init_stats) != 0) { ctx_error(ctx, "mbt_get_stats"); return -1; }
  if (mbt_writer_end(w, init_stats) != 0) { fprintf(stderr, "ERROR: %s\n", mbt_writer_error()); return -1; }
  if (nwatch > 0) {
    const int b = watch[0];
    if (mbt_get_particles(ctx, b, beam, np[b]) != 0) { ctx_error(ctx, "mbt_get_particles"); return -1; }
    if (mbt_writer_distribution(w, b, beam, np[b]) != 0) fprintf(stderr, "ERROR: %s\n", mbt_writer_error());
  }
  if (mbt_get_state(ctx, &st) == 0) {
    if (st.n_trash_low != 0 || st.n_trash_high != 0)
      printf("\n WARNING - Binning for selffields (all bunches):\n %d particles below first bin,    %d particles above last bin\n",
             st.n_trash_low, st.n_trash_high);
    if (p.rffb && nwatch > 0) printf("\nFinal RF voltage and phase: %.7f MV, %.5f\n", st.Vrf0, st.phai0);
  }
  if (bi_on && bi.surrogate) {
    double a[5];
    if (mbt_beam_ion_audit(ctx, a) == 0)
      printf("\nLearned field audit: %.0f evaluations, max relative field error %.3e, rms %.3e, %.0f outside "
             "the domain, %.0f tensor-core failures\n", a[0], a[1], a[2], a[3], a[4]);
  }
  mbt_writer_close(w);
  mbt_destroy(ctx);
  if (mlp) mbt_mlp_destroy(mlp);
  free(bucket); free(frac); free(bunch_out); free(np); free(ib); free(Gl); free(Gv); free(Gh);
  free(beam); free(init_stats); free(stats); free(ampinv); free(pot); free(watch);
  return 0;
}
