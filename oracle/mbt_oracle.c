/*
 * mbt_oracle.c -- TEST INFRASTRUCTURE ONLY: CPU oracle of the weak-weak
 * per-turn loop.  See mbt_oracle.h.  Each function cites the reference
 * lines it restates; the arithmetic keeps the reference's operation order
 * so that, compiled like the reference (gcc, x86-64, no FMA contraction),
 * results agree bit for bit.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mbt_oracle.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* def.h:290-307 */
#define FMILLI 1.0e-03
#define FKILO  1.0e+03
#define FGIGA  1.0e+09
#define FTERA  1.0e+12
#define FMEGA  1.0e+06
#define C_LIGHT  2.997925e+08
#define Z_0 376.73

#define LON 0
#define HOR 1
#define VER 2
#define PAD 4   /* zero bins on both sides of every histogram */

/* Per-bunch RNG: glibc random() keeps one state per process, so each MPI
 * worker has its own; bunch.c keeps iseed0 and the cached deviate as
 * statics, also per process (bunch.h:17, bunch.c:410-411). */
typedef struct orc_rng {
  struct random_data rd;
  char statebuf[128];
  int iseed0;
  int use_last;
  float y2;
} orc_rng;

typedef struct orc_bunch {
  int kb, np;
  double Ib;
  double *c[6];          /* xtau x z eps xp zp */
  orc_rng rng;
  /* worker-private ring values changed by the loop */
  double Vrf0, phai0;
  int rffb_on;
  double *rffb_hist;     /* [len][2] */
  int rffb_count;
  double rffb_full_prev[2];   /* generator loop: last full-correction phasor */
  double phasor[3][MBT_MAX_LR][2];
  int m;                 /* RW trigger counter */
  int trash_low, trash_high;
  /* last binning */
  double *fnp, *dipV, *dipH;   /* padded by PAD */
  double stats[12];
} orc_bunch;

struct orc_ctx {
  mbt_params p;
  int nb;
  orc_bunch *b;
  int *filled;           /* [h] */
  double *ibunch;        /* [h] mA */
  double *np_bucket;     /* [h] macroparticles of the bunch in each bucket (0: empty) */
  double *Gl, *Gv, *Gh;
  double *fnp_ring[3];   /* [h][ncell] */
  double *dipole;        /* [(Nmlt+2) h][2] */
  long rev;
  const float *dev_in;
  float *dev_out;
  long dev_pos, dev_cap;
  int lo, hi;   /* bunches tracked by this instance (orc_set_range) */
  /* beam-ion stage (orc_enable_beam_ion) */
  int bi_on;
  mbt_beam_ion bi;
  double *bi_frame;   /* [n_ip][nb][4] */
  double *bi_cloud;   /* [n_ip][nb][5] */
  double *bi_sum;     /* [n_ip][nb][5] */
};

#define IN_RANGE(o, ib) ((ib) >= (o)->lo && (ib) < (o)->hi)

void orc_set_range(orc_ctx *o, int lo, int hi)
{
  o->lo = lo;
  o->hi = hi;
}

/* ---------------------------------------------------------------- RNG */

static void rng_init(orc_rng *r)
{
  memset(r, 0, sizeof(*r));
  initstate_r(1u, r->statebuf, sizeof(r->statebuf), &r->rd);
  r->iseed0 = 0;   /* static int iseed0 = 0 (bunch.h:17) */
}

static int rng_rand(orc_rng *r)
{
  int32_t v;
  random_r(&r->rd, &v);
  return (int) v;
}

static void rng_seed(orc_rng *r, int iseed)
{
  if (iseed != r->iseed0) {
    srandom_r((unsigned) iseed, &r->rd);
    r->iseed0 = iseed;
  }
}

/* c_fnorm, bunch.c:379-405: Irwin-Hall sum of 12 uniforms minus 6. */
static double c_fnorm(orc_rng *r, int iseed)
{
  int i;
  double s, u, v;
  rng_seed(r, iseed);
  s = 0.0;
  for (i = 0; i < 12; i++) {
    u = ((double) rng_rand(r)) / ((double) RAND_MAX);
    v = u - 0.5;
    s = s + v;
  }
  return s;
}

/* box_muller, bunch.c:407-436: Marsaglia polar method in float with one
 * cached deviate. */
static double polar_normal(orc_rng *r, int iseed)
{
  float x1, x2, w, y1;
  rng_seed(r, iseed);
  if (r->use_last) {
    y1 = r->y2;
    r->use_last = 0;
  } else {
    do {
      x1 = 2.0 * ((double) rng_rand(r)) / ((double) RAND_MAX) - 1.0;
      x2 = 2.0 * ((double) rng_rand(r)) / ((double) RAND_MAX) - 1.0;
      w = x1 * x1 + x2 * x2;
    } while (w >= 1.0);
    w = sqrt((-2.0 * log(w)) / w);
    y1 = x1 * w;
    r->y2 = x2 * w;
    r->use_last = 1;
  }
  return y1;
}

static double draw(orc_ctx *o, orc_bunch *b, int iseed)
{
  double g;
  if (o->dev_in != NULL) g = (double) o->dev_in[o->dev_pos];
  else g = polar_normal(&b->rng, iseed);
  if (o->dev_out != NULL && o->dev_pos < o->dev_cap) o->dev_out[o->dev_pos] = (float) g;
  o->dev_pos++;
  return g;
}

/* ---------------------------------------------------------- lifecycle */

orc_ctx *orc_create(const mbt_params *p, int nbunch, const int *bucket,
                    const int *np, const double *ib, const double *Gl,
                    const double *Gv, const double *Gh)
{
  int i, k, h = p->nharm, nc = p->ncell > 0 ? p->ncell : 1;
  orc_ctx *o = (orc_ctx *) calloc(1, sizeof(orc_ctx));
  if (!o) return NULL;
  o->p = *p;
  o->nb = nbunch;
  o->lo = 0;
  o->hi = nbunch;
  o->b = (orc_bunch *) calloc(nbunch, sizeof(orc_bunch));
  o->filled = (int *) calloc(h, sizeof(int));
  o->ibunch = (double *) calloc(h, sizeof(double));
  o->np_bucket = (double *) calloc(h, sizeof(double));
  o->Gl = (double *) calloc(nc, sizeof(double));
  o->Gv = (double *) calloc(nc, sizeof(double));
  o->Gh = (double *) calloc(nc, sizeof(double));
  if (Gl) memcpy(o->Gl, Gl, p->ncell * sizeof(double));
  if (Gv) memcpy(o->Gv, Gv, p->ncell * sizeof(double));
  if (Gh) memcpy(o->Gh, Gh, p->ncell * sizeof(double));
  for (i = 0; i < nbunch; i++) {
    orc_bunch *b = &o->b[i];
    b->kb = bucket[i];
    b->np = np[i];
    b->Ib = ib[i];
    o->filled[b->kb] = 1;
    /* manager_weakweak.c:78: ring.Ibunch[kb] = bunch_Ib * FKILO */
    o->ibunch[b->kb] = ib[i] * FKILO;
    o->np_bucket[b->kb] = (double) np[i];
    for (k = 0; k < 6; k++) b->c[k] = (double *) calloc(np[i] > 0 ? np[i] : 1, sizeof(double));
    rng_init(&b->rng);
    b->Vrf0 = p->Vrf0;
    b->phai0 = p->phai0;
    b->rffb_on = p->rffb;
    b->rffb_hist = (double *) calloc(2 * (p->rffb_len > 0 ? p->rffb_len : 1), sizeof(double));
    b->fnp = (double *) calloc(nc + 2 * PAD, sizeof(double));
    b->dipV = (double *) calloc(nc + 2 * PAD, sizeof(double));
    b->dipH = (double *) calloc(nc + 2 * PAD, sizeof(double));
  }
  for (k = 0; k < 3; k++) o->fnp_ring[k] = (double *) calloc((size_t) h * nc, sizeof(double));
  if (p->rw_long) o->dipole = (double *) calloc((size_t) (p->Nmlt + 2) * h * 2, sizeof(double));
  return o;
}

void orc_destroy(orc_ctx *o)
{
  int i, k;
  if (!o) return;
  for (i = 0; i < o->nb; i++) {
    for (k = 0; k < 6; k++) free(o->b[i].c[k]);
    free(o->b[i].rffb_hist); free(o->b[i].fnp); free(o->b[i].dipV); free(o->b[i].dipH);
  }
  for (k = 0; k < 3; k++) free(o->fnp_ring[k]);
  free(o->dipole); free(o->b); free(o->filled); free(o->ibunch); free(o->np_bucket);
  free(o->bi_frame); free(o->bi_cloud); free(o->bi_sum);
  free(o->Gl); free(o->Gv); free(o->Gh);
  free(o);
}

int orc_set_particles(orc_ctx *o, int ib, const double *soa)
{
  int k;
  if (ib < 0 || ib >= o->nb) return -1;
  for (k = 0; k < 6; k++) memcpy(o->b[ib].c[k], soa + (size_t) k * o->b[ib].np, o->b[ib].np * sizeof(double));
  return o->b[ib].np;
}

int orc_get_particles(const orc_ctx *o, int ib, double *soa)
{
  int k;
  if (ib < 0 || ib >= o->nb) return -1;
  for (k = 0; k < 6; k++) memcpy(soa + (size_t) k * o->b[ib].np, o->b[ib].c[k], o->b[ib].np * sizeof(double));
  return o->b[ib].np;
}

/* weak_bunch_normal_distribution, bunch_weak.c:86-105 */
static void normal_plane(orc_bunch *b, const mbt_params *p, int plane)
{
  const double pos_offset = p->pos_offset[plane];
  const double pos_sgm = p->pos_sgm[plane];
  const double slope_offset = p->slope_offset[plane];
  const double slope_sgm = p->slope_sgm[plane];
  const double correlate = p->correlate[plane];
  const int iseed = p->iseed[plane] + b->kb;
  int jp;
  for (jp = 0; jp < b->np; jp++) {
    double tmp_pos = pos_sgm * c_fnorm(&b->rng, iseed);
    b->c[plane][jp] = pos_offset + tmp_pos;
    b->c[3 + plane][jp] = slope_offset + slope_sgm * c_fnorm(&b->rng, iseed) + correlate * tmp_pos;
  }
}

/* weak_generate_bunch_distribution, bunch_weak.c:173-292 (generated
 * distributions only; the excitation mode of :108-170 is not supported). */
int orc_generate_beam(orc_ctx *o)
{
  int i, k;
  const mbt_params *p = &o->p;
  for (i = 0; i < o->nb; i++) {
    orc_bunch *b = &o->b[i];
    for (k = 0; k < 6; k++) memset(b->c[k], 0, b->np * sizeof(double));
    if (b->np == 0 || !IN_RANGE(o, i)) continue;
    if (b->np == 1) {
      b->c[0][0] = p->pos_offset[LON]; b->c[3][0] = p->slope_offset[LON];
      if (p->track_plane[HOR]) { b->c[1][0] = p->pos_offset[HOR]; b->c[4][0] = p->slope_offset[HOR]; }
      if (p->track_plane[VER]) { b->c[2][0] = p->pos_offset[VER]; b->c[5][0] = p->slope_offset[VER]; }
      continue;
    }
    normal_plane(b, p, LON);
    if (p->track_plane[HOR]) normal_plane(b, p, HOR);
    if (p->track_plane[VER]) normal_plane(b, p, VER);
  }
  return 0;
}

/* -------------------------------------------------------- statistics */

/* weak_bunch_mean_rms, statistics.c:91-128 */
static void mean_rms(orc_bunch *b, int plane)
{
  int jp;
  double pos_sum = 0.0, slope_sum = 0.0, pos_ave, slope_ave;
  const double *x = b->c[plane], *xp = b->c[3 + plane];
  for (jp = 0; jp < b->np; jp++) {
    pos_sum += x[jp];
    slope_sum += xp[jp];
  }
  pos_ave = pos_sum / ((double) b->np);
  slope_ave = slope_sum / ((double) b->np);
  b->stats[0 + plane] = pos_ave;
  b->stats[6 + plane] = slope_ave;
  pos_sum = 0.0;
  slope_sum = 0.0;
  for (jp = 0; jp < b->np; jp++) {
    double d1 = pos_ave - x[jp], d2 = slope_ave - xp[jp];
    pos_sum += d1 * d1;
    slope_sum += d2 * d2;
  }
  b->stats[3 + plane] = sqrt(pos_sum / ((double) b->np));
  b->stats[9 + plane] = sqrt(slope_sum / ((double) b->np));
}

/* weak_bunch_calc_statistics, statistics.c:131-157 (per-turn values) */
static void calc_stats(orc_ctx *o, orc_bunch *b)
{
  int pl;
  for (pl = 0; pl < 3; pl++)
    if (o->p.track_plane[pl]) mean_rms(b, pl);
}

/* ------------------------------------------------------------ optics */

/* transform_weak_bunch_optic, transform_weak.c:21-192.  old[] plays the
 * role of particle0[] (all pre-turn coordinates). */
static void optic(orc_ctx *o, orc_bunch *b, int iseed)
{
  const mbt_params *p = &o->p;
  const int np = b->np;
  int jp, j, k;
  const double damp = 1.0 - p->De;
  const double excite = 2.0 * p->slope_sgm[LON] * sqrt(p->T0 / p->taue);
  const double quantumV_pos = p->pos_sgm[VER] * sqrt(2.0 * p->T0 / p->tauz);
  const double quantumV_slope = p->slope_sgm[VER] * sqrt(2.0 * p->T0 / p->tauz);
  const double quantumH_pos = p->pos_sgm[HOR] * sqrt(2.0 * p->T0 / p->taux);
  const double quantumH_slope = p->slope_sgm[HOR] * sqrt(2.0 * p->T0 / p->taux);
  const double eps_const = b->Vrf0 / (p->E0 * FKILO);
  double *xtau = b->c[0], *x = b->c[1], *z = b->c[2];
  double *eps = b->c[3], *xp = b->c[4], *zp = b->c[5];
  double *old[6];
  double *rffocus = (double *) malloc((np > 0 ? np : 1) * sizeof(double));
  for (k = 0; k < 6; k++) {
    old[k] = (double *) malloc((np > 0 ? np : 1) * sizeof(double));
    memcpy(old[k], b->c[k], np * sizeof(double));
  }

  for (jp = 0; jp < np; jp++) {
    double g;
    if (!p->ideal_hc) {
      g = eps_const * sin(p->wrf * old[0][jp] + b->phai0);
      for (j = 0; j < p->n_active_hc; j++)
        g += p->ahc_vpeak[j] / (p->E0 * FGIGA)
             * sin(p->wrf * p->ahc_nhc[j] * old[0][jp] + p->ahc_phi[j] + p->ahc_nhc[j] * b->kb * 2 * M_PI);
    } else {
      g = eps_const * (sin(p->wrf * old[0][jp] + b->phai0)
                       + p->HC_k * sin(p->m_aHC * p->wrf * old[0][jp] + p->m_aHC * p->phi_n));
    }
    eps[jp] = old[3][jp] + g - p->Urad;
    if (p->quantum) {
      eps[jp] = eps[jp] * damp + excite * draw(o, b, iseed);
      rffocus[jp] = (1.0 + old[3][jp]) / (1.0 + old[3][jp] + g);
    }
    xtau[jp] = old[0][jp] - eps[jp] * p->T0 * p->ac;
  }

  if (p->track_plane[VER]) {
    const double PsiV0 = 2.0 * M_PI * p->QV0;
    double dQ = 0.0;
    for (jp = 0; jp < np; jp++) {
      const double x0 = old[1][jp], z0 = old[2][jp], xp0 = old[4][jp], zp0 = old[5][jp];
      if (p->amp_dep_qv) {
        double EV = p->gamma1[VER] * z0 * z0 + 2 * p->alpha1[VER] * z0 * zp0 + p->beta1[VER] * zp0 * zp0;
        double EH = p->gamma1[VER] * x0 * x0 + 2 * p->alpha1[VER] * x0 * xp0 + p->beta1[VER] * xp0 * xp0;
        dQ = p->CVH * EH + p->CVV * EV;
      }
      double Psi = PsiV0 * (1.0 + p->Gziz * old[3][jp] + dQ);
      double cs = cos(Psi), sn = sin(Psi);
      double a11 = cs + p->alpha1[VER] * sn, a12 = p->beta1[VER] * sn;
      double a21 = -p->gamma1[VER] * sn, a22 = cs - p->alpha1[VER] * sn;
      z[jp] = a11 * z0 + a12 * zp0;
      zp[jp] = a21 * z0 + a22 * zp0;
      if (p->quantum) {
        z[jp] = z[jp] + quantumV_pos * draw(o, b, iseed);
        zp[jp] = rffocus[jp] * zp[jp] + quantumV_slope * draw(o, b, iseed);
      }
    }
  }

  if (p->track_plane[HOR]) {
    const double PsiH0 = 2.0 * M_PI * p->QH0;
    double dQ = 0;
    for (jp = 0; jp < np; jp++) {
      const double x0 = old[1][jp], z0 = old[2][jp], xp0 = old[4][jp], zp0 = old[5][jp];
      if (p->amp_dep_qv) {
        double EV = p->gamma1[VER] * z0 * z0 + 2 * p->alpha1[VER] * z0 * zp0 + p->beta1[VER] * zp0 * zp0;
        double EH = p->gamma1[VER] * x0 * x0 + 2 * p->alpha1[VER] * x0 * xp0 + p->beta1[VER] * xp0 * xp0;
        dQ = p->CHH * EH + p->CHV * EV;
      }
      double Psi = PsiH0 * (1.0 + p->Gzix * old[3][jp] + dQ);
      double cs = cos(Psi), sn = sin(Psi);
      double a11 = cs + p->alpha1[HOR] * sn;
      double a12 = p->beta1[HOR] * sn;
      double a13 = (1.0 - a11) * p->dispH1 - a12 * p->disppH1;
      double a21 = -p->gamma1[HOR] * sn;
      double a22 = cs - p->alpha1[HOR] * sn;
      double a23 = -a21 * p->dispH1 + (1.0 - a22) * p->disppH1;
      x[jp] = a11 * x0 + a12 * xp0 + a13 * eps[jp];
      xp[jp] = a21 * x0 + a22 * xp0 + a23 * eps[jp];
      if (p->quantum) {
        x[jp] = x[jp] + quantumH_pos * draw(o, b, iseed);
        xp[jp] = rffocus[jp] * xp[jp] + quantumH_slope * draw(o, b, iseed);
      }
    }
  }
  for (k = 0; k < 6; k++) free(old[k]);
  free(rffocus);
}

/* ------------------------------------------------------- RF feedback */

/* rffb_get_vrf_phi, feedback_rf.c:5-12: note atan2(real, imag). */
static void rffb_sample(const mbt_params *p, orc_bunch *b, double vreal, double vimag)
{
  double phi = atan2(vreal, vimag);
  double vrf = sqrt(vreal * vreal + vimag * vimag);
  unsigned key = ((unsigned) b->rffb_count % (unsigned) p->rffb_len) * 2u;
  b->rffb_hist[key] = vrf;
  b->rffb_hist[key + 1] = phi;
  b->rffb_count++;
}

/* rffb_calc_mean_voltage_phase feedback_rf.c:22-34 followed by the
 * correction of worker_weakweak.c:268-278 (and :149-162 at set-up, init).
 * With p->rffb_gain > 0 (an extension, no reference counterpart) the
 * generator phasor Vrf0 e^{i phai0} moves towards the full correction of
 * this turn (rffb_delay 0) or the last (1) by G / (1 + G) of the
 * difference; the set-up correction is the full one. */
static void rffb_correct(const mbt_params *p, orc_bunch *b, int init)
{
  double vrf_sum = 0, phi_sum = 0, vmbar, phibar;
  int m;
  for (m = 0; m < p->rffb_len; m++) {
    vrf_sum += b->rffb_hist[2 * m];
    phi_sum += b->rffb_hist[2 * m + 1];
  }
  vmbar = vrf_sum / p->rffb_len;
  phibar = phi_sum / p->rffb_len;
  vmbar = vmbar * p->E0 * FKILO;
  double tmp_numrtor = p->rffb_vrf_design * sin(p->rffb_phi0_design) - vmbar * sin(phibar);
  double den = p->rffb_vrf_design * cos(p->rffb_phi0_design) - vmbar * cos(phibar);
  if (p->rffb_gain > 0.0 && !init) {
    const double kappa = p->rffb_gain / (1.0 + p->rffb_gain);
    const double fc = p->rffb_delay ? b->rffb_full_prev[0] : den;
    const double fs = p->rffb_delay ? b->rffb_full_prev[1] : tmp_numrtor;
    const double gc = b->Vrf0 * cos(b->phai0), gs = b->Vrf0 * sin(b->phai0);
    const double nc = gc + kappa * (fc - gc), ns = gs + kappa * (fs - gs);
    b->rffb_full_prev[0] = den;
    b->rffb_full_prev[1] = tmp_numrtor;
    b->phai0 = atan2(ns, nc);
    b->Vrf0 = ns / sin(b->phai0);
    return;
  }
  b->rffb_full_prev[0] = den;
  b->rffb_full_prev[1] = tmp_numrtor;
  b->phai0 = atan2(tmp_numrtor, den);
  b->Vrf0 = tmp_numrtor / sin(b->phai0);
}

/* ------------------------------------------------ long-range phasors */

typedef struct phasor_consts {
  double prog[2], p2b[2], pb2b[2];
  double e_gap, c_gap, s_gap, e_emp, c_emp, s_emp;
  double amp;
  int fb;
} phasor_consts;

/* constants of construct_wake_phasor transform_weak.c:976-1004 */
static void phasor_setup(const orc_ctx *o, const orc_bunch *b, int plane, int l, phasor_consts *q)
{
  const mbt_params *p = &o->p;
  const double wr = p->lr_wr[plane][l], Q = p->lr_Q[plane][l], Rs = p->lr_Rs[plane][l];
  const double hd = (double) p->nharm;
  double alpha = wr * 0.5 / Q;
  double Amp = 2 * alpha * Rs * p->T0 / p->E0 / FGIGA;
  double dTau = p->dT * p->sigma_tau;
  double tbucket = (p->T0 / hd - p->ncell * dTau);
  double C0 = -alpha, C1 = wr;
  double taubeam = 0, taub2beam = 0;
  q->amp = Amp;
  q->prog[0] = exp(C0 * dTau) * cos(C1 * dTau);
  q->prog[1] = exp(C0 * dTau) * sin(C1 * dTau);
  q->fb = (b->rffb_on && plane == LON && p->rffb_resonator == l + 1);
  if (q->fb) {
    taubeam = p->nsigma * p->sigma_tau + dTau * 1.5;
    taub2beam = -p->nsigma * p->sigma_tau + dTau * 0.5 - tbucket;
  }
  q->p2b[0] = exp(C0 * taubeam) * cos(C1 * taubeam);
  q->p2b[1] = exp(C0 * taubeam) * sin(C1 * taubeam);
  q->pb2b[0] = exp(C0 * taub2beam) * cos(C1 * taub2beam);
  q->pb2b[1] = exp(C0 * taub2beam) * sin(C1 * taub2beam);
  q->e_gap = exp(C0 * tbucket); q->c_gap = cos(C1 * tbucket); q->s_gap = sin(C1 * tbucket);
  q->e_emp = exp(C0 * p->T0 / hd); q->c_emp = cos(C1 * p->T0 / hd); q->s_emp = sin(C1 * p->T0 / hd);
}

/* One pass of the phasor of resonator (plane, l) around the ring, buckets
 * h-1 .. 0 (construct_wake_phasor transform_weak.c:1006-1044 and the body
 * of wake_phasor_init :913-947).  lr_wake may be NULL (initialisation). */
static void phasor_pass(orc_ctx *o, orc_bunch *b, int plane, int l, const phasor_consts *q,
                        double V_old[2], double V_new[2], double *lr_wake)
{
  const mbt_params *p = &o->p;
  const int Nbin = p->ncell;
  const double *fnp = o->fnp_ring[plane];
  int m, i, j;
  for (m = 0; m < p->nharm; m++) {
    i = p->nharm - m - 1;
    if (q->fb)
      rffb_sample(p, b, V_new[0] * q->p2b[0] - V_new[1] * q->p2b[1], V_new[0] * q->p2b[1] + V_new[1] * q->p2b[0]);
    if (o->filled[i] == 1) {
      /* Amp / Np * 1e-3 of the SOURCE bunch: the reference's single Np is
         every bunch's; with per-bunch counts the charge per macroparticle
         of the bunch whose histogram drives the phasor is Ib / its Np */
      const double fac = q->amp / o->np_bucket[i] * FMILLI;
      for (j = 0; j < Nbin; j++) {
        V_new[0] = (V_old[0] * q->prog[0] - V_old[1] * q->prog[1]) - o->ibunch[i] * fnp[i * Nbin + j] * fac;
        V_new[1] = (V_old[0] * q->prog[1] + V_old[1] * q->prog[0]);
        if (lr_wake != NULL && i == b->kb)
          lr_wake[j] += V_new[0] + 0.5 * o->ibunch[i] * fnp[i * Nbin + j] * fac;
        V_old[0] = V_new[0];
        V_old[1] = V_new[1];
      }
      V_new[0] = (V_old[0] * q->e_gap * q->c_gap - V_old[1] * q->e_gap * q->s_gap);
      V_new[1] = (V_old[0] * q->e_gap * q->s_gap + V_old[1] * q->e_gap * q->c_gap);
      V_old[0] = V_new[0];
      V_old[1] = V_new[1];
    } else {
      V_new[0] = (V_old[0] * q->e_emp * q->c_emp - V_old[1] * q->e_emp * q->s_emp);
      V_new[1] = (V_old[0] * q->e_emp * q->s_emp + V_old[1] * q->e_emp * q->c_emp);
      V_old[0] = V_new[0];
      V_old[1] = V_new[1];
    }
    if (q->fb)
      rffb_sample(p, b, V_new[0] * q->pb2b[0] - V_new[1] * q->pb2b[1], V_new[0] * q->pb2b[1] + V_new[1] * q->pb2b[0]);
  }
}

/* construct_wake_phasor, transform_weak.c:961-1048 */
static void wake_phasor(orc_ctx *o, orc_bunch *b, int plane, double *lr_wake)
{
  int l;
  for (l = 0; l < o->p.n_lr[plane]; l++) {
    phasor_consts q;
    double V_old[2], V_new[2];
    phasor_setup(o, b, plane, l, &q);
    V_old[0] = V_new[0] = b->phasor[plane][l][0];
    V_old[1] = V_new[1] = b->phasor[plane][l][1];
    phasor_pass(o, b, plane, l, &q, V_old, V_new, lr_wake);
    b->phasor[plane][l][0] = V_new[0];
    b->phasor[plane][l][1] = V_new[1];
  }
}

/* wake_phasor_init, transform_weak.c:868-952.  V_new starts from the
 * phasor array, which the reference leaves uninitialised and here is 0. */
static void wake_phasor_init(orc_ctx *o, orc_bunch *b, int plane)
{
  int l, k;
  for (l = 0; l < o->p.n_lr[plane]; l++) {
    phasor_consts q;
    double V_old[2] = {0.0, 0.0}, V_new[2];
    phasor_setup(o, b, plane, l, &q);
    V_new[0] = b->phasor[plane][l][0];
    V_new[1] = b->phasor[plane][l][1];
    for (k = 0; k < o->p.lr_init_turns; k++)
      phasor_pass(o, b, plane, l, &q, V_old, V_new, NULL);
    b->phasor[plane][l][0] = V_new[0];
    b->phasor[plane][l][1] = V_new[1];
  }
}

/* ---------------------------------------------------------- binning */

static int bin_of(const mbt_params *p, double xtau)
{
  double Tau = -xtau / p->sigma_tau;
  return (int) ((Tau + p->nsigma) / p->dT + 1);
}

/* fnp_ring_update, transform_weak.c:838-865 */
static void ring_hist(orc_ctx *o, orc_bunch *b, int plane)
{
  const int Nbin = o->p.ncell;
  double *f = o->fnp_ring[plane] + (size_t) b->kb * Nbin;
  int jp, icell;
  for (icell = 0; icell < Nbin; icell++) f[icell] = 0.0;
  for (jp = 0; jp < b->np; jp++) {
    icell = bin_of(&o->p, b->c[0][jp]);
    if (icell >= 0 && icell < Nbin) {
      if (plane == LON) f[icell] += 1.0;
      else if (plane == HOR) f[icell] += b->c[1][jp];
      else f[icell] += b->c[2][jp];
    }
  }
}

/* transform_weak_bunch_selffield, transform_weak.c:552-771 (the potentials
 * writer of :735-768 is output only and is not restated).  Out-of-range
 * reads of fnp[] at the edges (:658,:673-681) see zero padding. */
static void selffield(orc_ctx *o, orc_bunch *b)
{
  const mbt_params *p = &o->p;
  const int Nc = p->ncell;
  const double sgm_xtau = p->sigma_tau;
  const double sgmatau2 = sgm_xtau * sgm_xtau;
  const double dTau2 = p->dT * p->dT;
  const double factG = -p->T0 * b->Ib / (b->np * p->E0 * FGIGA);
  double *fnp = b->fnp + PAD, *dipV = b->dipV + PAD, *dipH = b->dipH + PAD;
  double *GL1 = (double *) calloc(Nc, sizeof(double));
  double *GlV = (double *) calloc(Nc, sizeof(double));
  double *GlH = (double *) calloc(Nc, sizeof(double));
  double *lr[3];
  int *mapcell = (int *) malloc((b->np > 0 ? b->np : 1) * sizeof(int));
  int jp, icell, k, icellmin, icellmax;
  double Gn;
  for (k = 0; k < 3; k++) lr[k] = (double *) calloc(Nc, sizeof(double));
  memset(b->fnp, 0, (Nc + 2 * PAD) * sizeof(double));
  memset(b->dipV, 0, (Nc + 2 * PAD) * sizeof(double));
  memset(b->dipH, 0, (Nc + 2 * PAD) * sizeof(double));

  for (jp = 0; jp < b->np; jp++) {
    icell = bin_of(p, b->c[0][jp]);
    if (icell < 0) { icell = 0; b->trash_low++; }
    else if (icell >= Nc) { icell = Nc - 1; b->trash_high++; }
    mapcell[jp] = icell;
    fnp[icell] += 1.0;
    dipV[icell] += b->c[2][jp];
    dipH[icell] += b->c[1][jp];
  }
  icellmin = Nc - 1;
  icellmax = 0;
  for (icell = 0; icell < icellmin; icell++)
    if (fnp[icell] > 0) { icellmin = 1 * icell; break; }
  for (icell = Nc - 1; icell > icellmax; icell--)
    if (fnp[icell] > 0) { icellmax = 1 * icell; break; }

  if (p->planeL > 0) {
    double ntmoy, ntmoy0, ntmoy1;
    for (icell = icellmin; icell < Nc; icell++) {
      Gn = 0.0;
      for (k = icell; k >= icellmin; k--) Gn += fnp[k] * o->Gl[icell - k];
      GL1[icell] = 1 * Gn;
    }
    if (p->RsisL > 0)
      for (icell = icellmin + 1; icell <= icellmax; icell++) {
        ntmoy = (0.5 * fnp[icell - 1] + fnp[icell] + 0.5 * fnp[icell + 1]) / 2.0;
        GL1[icell] += p->RsisL * ntmoy / (sgm_xtau * p->dT);
      }
    if (p->aindL > 0)
      for (icell = icellmin + 1; icell <= icellmax; icell++) {
        ntmoy0 = (0.25 * fnp[icell - 3] + 0.5 * fnp[icell - 2] + fnp[icell - 1] + 0.5 * fnp[icell] + 0.25 * fnp[icell + 1]) / 2.5;
        ntmoy1 = (0.25 * fnp[icell - 1] + 0.5 * fnp[icell] + fnp[icell + 1] + 0.5 * fnp[icell + 2] + 0.25 * fnp[icell + 3]) / 2.5;
        GL1[icell] += (ntmoy1 - ntmoy0) / (2.0 * sgmatau2 * dTau2) * p->aindL;
      }
  }

  if (p->n_lr[LON] > 0) wake_phasor(o, b, LON, lr[LON]);
  if (p->n_lr[HOR] > 0) wake_phasor(o, b, HOR, lr[HOR]);
  if (p->n_lr[VER] > 0) wake_phasor(o, b, VER, lr[VER]);

  if (p->n_lr[LON] + p->planeL > 0)
    for (jp = 0; jp < b->np; jp++) b->c[3][jp] += factG * GL1[mapcell[jp]] + lr[LON][mapcell[jp]];

  if (p->planeV > 0) {
    for (icell = 0; icell < Nc; icell++) {
      Gn = 0.0;
      for (k = icell; k >= 0; k--) Gn += dipV[k] * o->Gv[icell - k];
      GlV[icell] = 1 * Gn;
    }
    for (jp = 0; jp < b->np; jp++) b->c[5][jp] += -factG * GlV[mapcell[jp]] + lr[VER][mapcell[jp]];
  }
  if (p->planeH > 0) {
    for (icell = 1; icell < Nc; icell++) {
      Gn = 0.0;
      for (k = icell; k >= 0; k--) Gn += dipH[k] * o->Gh[icell - k];
      GlH[icell] = 1 * Gn;
    }
    for (jp = 0; jp < b->np; jp++) b->c[4][jp] += -factG * GlH[mapcell[jp]] + lr[HOR][mapcell[jp]];
  }
  for (k = 0; k < 3; k++) free(lr[k]);
  free(GL1); free(GlV); free(GlH); free(mapcell);
}

/* ------------------------------------------------- resistive wall */

static double *cyc(orc_ctx *o, long in)
{
  const long n = (long) (o->p.Nmlt + 2) * o->p.nharm;
  int ii = (int) in;   /* cyclic_array_access takes an int */
  const int in_mod = ii < 0 ? (int) ((ii % n + n) % n) : (int) (ii % n);
  return &o->dipole[(size_t) in_mod * 2];
}

/* transform_weak_bunch_RW_longrange_cyclic, transform_weak.c:779-833 */
static void rw_kick(orc_ctx *o, orc_bunch *b, long bpos, int plane)
{
  const mbt_params *p = &o->p;
  const int h = p->nharm;
  const double fNp = (double) b->np;
  double beff3 = plane == HOR ? p->beffH[0] : p->beffV[0];
  const int Ntrigger = 50;
  int m, k, in_mod, jp;
  double tt, wake_voltage = 0.;
  double deltab = p->T0 / (double) h;
  if (p->triggerRW && b->m < Ntrigger) beff3 /= 2;
  double RWconst = p->T0 / p->E0 / fNp / FTERA * p->Lc / (M_PI * pow(beff3, 3)) * sqrt(Z_0 * C_LIGHT * p->rhorw / M_PI);
  for (m = 1; m < ((p->Nmlt + 1) * h + 1); m++) {
    k = (int) bpos + m;
    in_mod = k < 0 ? (k % h + h) % h : k % h;
    if (o->filled[in_mod]) {
      const double *mom = cyc(o, k);
      tt = m * deltab;
      wake_voltage += fNp * mom[plane - 1] * o->ibunch[in_mod] / sqrt(tt);
    }
  }
  wake_voltage *= RWconst;
  for (jp = 0; jp < b->np; jp++) b->c[3 + plane][jp] += wake_voltage;
}

/* -------------------------------------------------------- set-up/run */

int orc_prepare(orc_ctx *o, double *init_stats)
{
  const mbt_params *p = &o->p;
  int ib, i, j, pl;
  for (ib = 0; ib < o->nb; ib++) {
    if (!IN_RANGE(o, ib)) continue;
    calc_stats(o, &o->b[ib]);
    if (init_stats) memcpy(init_stats + 12 * ib, o->b[ib].stats, 12 * sizeof(double));
  }
  if (p->n_lr[LON] > 0) {
    for (ib = 0; ib < o->nb; ib++) {
      o->b[ib].rffb_count = 0;   /* rffb_init feedback_rf.c:14-19 */
      if (IN_RANGE(o, ib)) ring_hist(o, &o->b[ib], LON);
    }
    for (ib = 0; ib < o->nb; ib++) {
      orc_bunch *b = &o->b[ib];
      if (!IN_RANGE(o, ib)) continue;
      wake_phasor_init(o, b, LON);
      if (b->rffb_on) {
        rffb_correct(p, b, 1);
        if (p->rffb_off_after_init) b->rffb_on = 0;
      }
    }
  }
  for (pl = HOR; pl <= VER; pl++) {
    if (p->track_plane[pl] && p->n_lr[pl] > 0) {
      for (ib = 0; ib < o->nb; ib++) if (IN_RANGE(o, ib)) ring_hist(o, &o->b[ib], pl);
      for (ib = 0; ib < o->nb; ib++) if (IN_RANGE(o, ib)) wake_phasor_init(o, &o->b[ib], pl);
    }
  }
  if (p->rw_long) {
    for (ib = 0; ib < o->nb; ib++) {
      double *d = cyc(o, o->b[ib].kb);
      if (!IN_RANGE(o, ib)) continue;
      d[0] = o->b[ib].stats[0 + HOR];
      d[1] = o->b[ib].stats[0 + VER];
    }
    for (i = 0; i < p->nharm; i++) {
      if (!o->filled[i]) continue;
      double *mom = cyc(o, i);
      for (j = 1; j < p->Nmlt; j++) {
        double *d = cyc(o, (long) j * p->nharm + i);
        d[0] = mom[0];
        d[1] = mom[1];
      }
    }
  }
  return 0;
}

long orc_deviates_per_turn(const orc_ctx *o)
{
  long n = 0;
  int ib;
  if (!o->p.quantum) return 0;
  for (ib = 0; ib < o->nb; ib++)
    n += (long) o->b[ib].np * (1 + 2 * (o->p.track_plane[VER] != 0) + 2 * (o->p.track_plane[HOR] != 0));
  return n;
}

/* worker_weakweak.c:259-394, phase by phase over the bunches */
/* ------------------------------------------------------------ beam-ion */

/* The beam-ion stage of mbt.h (mbt_beam_ion), restated loop by loop in
 * plain C.  Physics after fbi_weakstrong.c (constants def.h:21-26, factF
 * :40, gas density :24, ion drift :370-375, ion kick :393-405, the
 * Bassetti-Erskine field :154-197 through orc_wofz); the per-particle
 * electron kick, the interaction points at betatron phase advances and
 * the cloud moments are the stage's own model. */

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) */
typedef struct { uint32_t x, y, z, w; } u4_t;
static u4_t philox10(u4_t c, uint64_t seed)
{
  uint32_t k0 = (uint32_t) seed, k1 = (uint32_t) (seed >> 32);
  int i;
  for (i = 0; i < 10; i++) {
    const uint64_t p0 = (uint64_t) 0xD2511F53u * c.x, p1 = (uint64_t) 0xCD9E8D57u * c.z;
    u4_t r;
    r.x = (uint32_t) (p1 >> 32) ^ c.y ^ k0;
    r.y = (uint32_t) p1;
    r.z = (uint32_t) (p0 >> 32) ^ c.w ^ k1;
    r.w = (uint32_t) p0;
    c = r;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

static const double GL16_X[16] = {
  0.005299532504175031, 0.0277124884633837, 0.06718439880608412, 0.1222977958224985,
  0.19106187779867811, 0.2709916111713863, 0.35919822461037054, 0.4524937450811813,
  0.5475062549188188, 0.6408017753896295, 0.7290083888286136, 0.8089381222013219,
  0.8777022041775016, 0.9328156011939159, 0.9722875115366163, 0.994700467495825};
static const double GL16_W[16] = {
  0.013576229705877088, 0.031126761969323728, 0.0475792558412463, 0.062314485627767036,
  0.07479799440828835, 0.08457825969750132, 0.09130170752246182, 0.09472530522753432,
  0.09472530522753432, 0.09130170752246182, 0.08457825969750132, 0.07479799440828835,
  0.062314485627767036, 0.0475792558412463, 0.031126761969323728, 0.013576229705877088};

/* unit-charge field of an elliptic Gaussian (mbt_gauss_field_dev) */
void orc_gauss_field(double dx, double dy, double sx, double sy, double *gx, double *gy)
{
  const double sgx = dx < 0.0 ? -1.0 : 1.0, sgy = dy < 0.0 ? -1.0 : 1.0;
  double ax = fabs(dx), ay = fabs(dy), r, fx, fy;
  const int swap = sy > sx;
  if (swap) {
    double t = ax; ax = ay; ay = t;
    t = sx; sx = sy; sy = t;
  }
  if (sy < 1e-6 * sx) sy = 1e-6 * sx;
  r = sy / sx;
  if (r <= 0.995) {
    const double fbe = sqrt(2.0 * (sx * sx - sy * sy));
    const double x1 = ax / fbe, y1 = ay / fbe;
    double w1r, w1i, w2r = 0.0, w2i = 0.0, e, c, arg;
    orc_wofz(x1, y1, &w1r, &w1i);
    /* beyond exp(-50) the second term lies below the last bit of the first
     * (|w| <= 1 in the upper half plane): w(z2) is not evaluated there */
    arg = ax * ax / (2.0 * sx * sx) + ay * ay / (2.0 * sy * sy);
    e = arg > 50.0 ? 0.0 : exp(-arg);
    if (e != 0.0) orc_wofz(x1 * r, y1 / r, &w2r, &w2i);
    c = 1.0 / (1.7724538509055160273 * fbe);
    fx = c * (w1i - e * w2i);
    fy = c * (w1r - e * w2r);
  } else {
    const double q = 1.0 - r * r, inv2 = 1.0 / (2.0 * sx * sx);
    const double a0 = (ax * ax + ay * ay) * inv2;
    const double T = a0 > 40.0 ? sqrt(40.0 / a0) : 1.0, h = 0.25 * T;
    double ix = 0.0, iy = 0.0, c;
    int pnl, i;
    for (pnl = 0; pnl < 4; pnl++)
      for (i = 0; i < 16; i++) {
        const double t = h * (pnl + GL16_X[i]);
        const double D = 1.0 - q * t * t;
        const double f = t * exp(-(t * t) * (ax * ax + ay * ay / D) * inv2) / sqrt(D);
        const double wgt = h * GL16_W[i];
        ix += wgt * f;
        iy += wgt * (f / D);
      }
    c = 1.0 / (M_PI * sx * sx);
    fx = c * ax * ix;
    fy = c * ay * iy;
  }
  if (swap) { double t = fx; fx = fy; fy = t; }
  *gx = sgx * fx;
  *gy = sgy * fy;
}

int orc_enable_beam_ion(orc_ctx *o, const mbt_beam_ion *bi)
{
  const size_t n = (size_t) bi->n_ip * o->nb;
  o->bi = *bi;
  o->bi_frame = (double *) calloc(n * 4, sizeof(double));
  o->bi_cloud = (double *) calloc(n * 5, sizeof(double));
  o->bi_sum = (double *) calloc(n * 5, sizeof(double));
  o->bi_on = 1;
  return 0;
}

void orc_beam_ion_clouds(const orc_ctx *o, double *clouds)
{
  memcpy(clouds, o->bi_cloud, (size_t) o->bi.n_ip * o->nb * 5 * sizeof(double));
}

/* one turn of the stage; `turn` keys the ion generation (turns completed) */
static void beam_ion(orc_ctx *o, long turn)
{
  const mbt_params *p = &o->p;
  const mbt_beam_ion *cfg = &o->bi;
  const int nip = cfg->n_ip, nb = o->nb, nnew = cfg->ions_per_passage;
  const double c_light = 2.997925e+08, eps0 = 8.854187817620e-12, e_charge = 1.602e-19, e_mass = 9.1e-31;
  const double r_e = 2.819e-15, mp_o_em = 1.836e3, gamma = 1957.0 * p->E0;
  const double factF = e_charge / (cfg->gas_A * mp_o_em * e_mass);
  const double n_gas = 3.22e22 * cfg->pressure, L_ip = p->Lc / nip;
  const double kion_per_amp = -factF * p->T0 / (2.0 * eps0 * c_light);
  const double ke = -2.0 * M_PI * r_e / gamma;
  const double w_per_amp = p->T0 / e_charge * cfg->sigma_ion * n_gas * L_ip / nnew;
  const double dt_bucket = p->T0 / p->nharm;
  const double bH = p->beta1[HOR], aH = p->alpha1[HOR], bV = p->beta1[VER], aV = p->alpha1[VER];
  int k, b, b0, j, jp;
  /* 1. moments of every bunch and its frame at every point */
  for (b = 0; b < nb; b++) {
    const orc_bunch *e = &o->b[b];
    double m[10];
    int pl;
    for (pl = 0; pl < 2; pl++) {
      const double *u = e->c[1 + pl], *up = e->c[4 + pl];
      double su = 0.0, sp = 0.0, vu = 0.0, vp = 0.0, cv = 0.0;
      for (jp = 0; jp < e->np; jp++) { su += u[jp]; sp += up[jp]; }
      su /= e->np; sp /= e->np;
      for (jp = 0; jp < e->np; jp++) {
        const double du = u[jp] - su, dp = up[jp] - sp;
        vu += du * du; vp += dp * dp; cv += du * dp;
      }
      m[5 * pl] = su; m[5 * pl + 1] = sp;
      m[5 * pl + 2] = vu / e->np; m[5 * pl + 3] = cv / e->np; m[5 * pl + 4] = vp / e->np;
    }
    for (k = 0; k < nip; k++) {
      const double mux = 2.0 * M_PI * p->QH0 * k / nip, muy = 2.0 * M_PI * p->QV0 * k / nip;
      const double mx = cos(mux) + aH * sin(mux), sxb = bH * sin(mux);
      const double my = cos(muy) + aV * sin(muy), syb = bV * sin(muy);
      double *F = o->bi_frame + ((size_t) k * nb + b) * 4;
      const double vx = mx * mx * m[2] + 2.0 * mx * sxb * m[3] + sxb * sxb * m[4];
      const double vy = my * my * m[7] + 2.0 * my * syb * m[8] + syb * syb * m[9];
      F[0] = mx * m[0] + sxb * m[1];
      F[1] = my * m[5] + syb * m[6];
      F[2] = sqrt(vx > 0.0 ? vx : 0.0);
      F[3] = sqrt(vy > 0.0 ? vy : 0.0);
    }
  }
  /* 2. ions: created at passage b0, drift and kick at every later one */
  memset(o->bi_sum, 0, (size_t) nip * nb * 5 * sizeof(double));
  for (k = 0; k < nip; k++)
    for (b0 = 0; b0 + 1 < nb; b0++)
      for (j = 0; j < nnew; j++) {
        const double *F0 = o->bi_frame + ((size_t) k * nb + b0) * 4;
        u4_t c, r;
        double u1, u2, u3, u4, x, y, vx = 0.0, vy = 0.0, w;
        c.x = (uint32_t) j; c.y = (uint32_t) b0 | ((uint32_t) k << 20);
        c.z = (uint32_t) turn; c.w = (uint32_t) ((uint64_t) turn >> 32);
        r = philox10(c, cfg->seed);
        u1 = ((double) r.x + 1.0) * 2.3283064365386962890625e-10;
        u2 = (double) r.y * 2.3283064365386962890625e-10;
        u3 = ((double) r.z + 1.0) * 2.3283064365386962890625e-10;
        u4 = (double) r.w * 2.3283064365386962890625e-10;
        x = F0[0] + F0[2] * (sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2));
        y = F0[1] + F0[3] * (sqrt(-2.0 * log(u3)) * cos(2.0 * M_PI * u4));
        w = w_per_amp * o->b[b0].Ib;
        for (b = b0 + 1; b < nb; b++) {
          const double dt = (double) (o->b[b].kb - o->b[b - 1].kb) * dt_bucket;
          const double *F = o->bi_frame + ((size_t) k * nb + b) * 4;
          double *S = o->bi_sum + ((size_t) k * nb + b) * 5;
          double dx, dy, gx, gy, kk;
          x = x + dt * vx;
          y = y + dt * vy;
          dx = x - F[0];
          dy = y - F[1];
          S[0] += w; S[1] += w * dx; S[2] += w * dy; S[3] += w * (dx * dx); S[4] += w * (dy * dy);
          orc_gauss_field(dx, dy, F[2], F[3], &gx, &gy);
          kk = kion_per_amp * o->b[b].Ib;
          vx = vx + kk * gx;
          vy = vy + kk * gy;
        }
      }
  /* 3. clouds */
  for (k = 0; k < nip; k++)
    for (b = 0; b < nb; b++) {
      const double *S = o->bi_sum + ((size_t) k * nb + b) * 5;
      const double *F = o->bi_frame + ((size_t) k * nb + b) * 4;
      double *C = o->bi_cloud + ((size_t) k * nb + b) * 5;
      if (S[0] > 0.0) {
        const double mx = S[1] / S[0], my = S[2] / S[0];
        const double vx = S[3] / S[0] - mx * mx, vy = S[4] / S[0] - my * my;
        C[0] = S[0]; C[1] = F[0] + mx; C[2] = F[1] + my;
        C[3] = sqrt(vx > 0.0 ? vx : 0.0); C[4] = sqrt(vy > 0.0 ? vy : 0.0);
      } else {
        C[0] = C[1] = C[2] = C[3] = C[4] = 0.0;
      }
    }
  /* 4. electron kicks */
  for (b = 0; b < nb; b++) {
    orc_bunch *e = &o->b[b];
    for (jp = 0; jp < e->np; jp++) {
      const double x = e->c[1][jp], z = e->c[2][jp], xp = e->c[4][jp], zp = e->c[5][jp];
      double ddx = 0.0, ddxp = 0.0, ddz = 0.0, ddzp = 0.0;
      for (k = 0; k < nip; k++) {
        const double *C = o->bi_cloud + ((size_t) k * nb + b) * 5;
        const double mux = 2.0 * M_PI * p->QH0 * k / nip, muy = 2.0 * M_PI * p->QV0 * k / nip;
        const double mx = cos(mux) + aH * sin(mux), sxb = bH * sin(mux);
        const double my = cos(muy) + aV * sin(muy), syb = bV * sin(muy);
        const double kn = ke * C[0];
        double gx, gy, thx, thy;
        if (kn == 0.0) continue;
        orc_gauss_field(mx * x + sxb * xp - C[1], my * z + syb * zp - C[2], C[3], C[4], &gx, &gy);
        thx = kn * gx;
        thy = kn * gy;
        ddx = ddx - sxb * thx;
        ddxp = ddxp + mx * thx;
        ddz = ddz - syb * thy;
        ddzp = ddzp + my * thy;
      }
      e->c[1][jp] = x + ddx;
      e->c[4][jp] = xp + ddxp;
      e->c[2][jp] = z + ddz;
      e->c[5][jp] = zp + ddzp;
    }
  }
}

long orc_run(orc_ctx *o, long nturns, double *stats, const float *dev_in,
             float *dev_out, long dev_cap)
{
  const mbt_params *p = &o->p;
  const int lr_tot = p->n_lr[LON] + p->n_lr[HOR] + p->n_lr[VER];
  long t;
  int ib;
  o->dev_in = dev_in;
  o->dev_out = dev_out;
  o->dev_cap = dev_cap;
  o->dev_pos = 0;
  for (t = 0; t < nturns; t++) {
    long rev = o->rev + t;
    if (p->ncell > 0 && p->planeL + p->planeV + p->planeH + lr_tot > 0)
      for (ib = o->lo; ib < o->hi && ib < o->nb; ib++) selffield(o, &o->b[ib]);
    for (ib = o->lo; ib < o->hi && ib < o->nb; ib++)
      if (o->b[ib].rffb_on) rffb_correct(p, &o->b[ib], 0);
    for (ib = 0; ib < o->nb; ib++) {
      orc_bunch *b = &o->b[ib];
      if (!IN_RANGE(o, ib)) continue;
      optic(o, b, p->iseed[LON] + b->kb + (int) rev);
      calc_stats(o, b);
      if (stats) memcpy(stats + (t * o->nb + ib) * 12, b->stats, 12 * sizeof(double));
    }
    if (o->bi_on) beam_ion(o, rev + 1);
    if (p->rw_long) {
      for (ib = o->lo; ib < o->hi && ib < o->nb; ib++) {
        double *mom = cyc(o, -rev * p->nharm + o->b[ib].kb);
        mom[0] = o->b[ib].stats[0 + HOR];
        mom[1] = o->b[ib].stats[0 + VER];
      }
      for (ib = o->lo; ib < o->hi && ib < o->nb; ib++) {
        orc_bunch *b = &o->b[ib];
        const long bpos = -rev * p->nharm + b->kb;
        if (p->track_plane[HOR]) rw_kick(o, b, bpos, HOR);
        if (p->track_plane[VER]) rw_kick(o, b, bpos, VER);
        b->m++;
      }
    }
    for (ib = o->lo; ib < o->hi && ib < o->nb; ib++) {
      if (p->n_lr[LON] > 0) ring_hist(o, &o->b[ib], LON);
      if (p->n_lr[HOR] > 0 && p->track_plane[HOR]) ring_hist(o, &o->b[ib], HOR);
      if (p->n_lr[VER] > 0 && p->track_plane[VER]) ring_hist(o, &o->b[ib], VER);
    }
    /* scan step, worker_weakweak.c:388-393 with tracking_scan_step_worker
       tracking.c:43-57: a current scan adds scan_step / Nbunch to every
       filled bucket's current and to every bunch's; any scan restarts the
       resistive-wall trigger count */
    if (p->scan != 0 && (rev + 1) % p->nrev_scan == 0) {
      if (p->scan == 1) {
        int i;
        for (ib = 0; ib < o->nb; ib++) o->b[ib].Ib += p->scan_step / (((double) o->nb) * FKILO);
        for (i = 0; i < p->nharm; i++)
          if (o->filled[i]) o->ibunch[i] += p->scan_step / ((double) o->nb);
      }
      for (ib = 0; ib < o->nb; ib++) o->b[ib].m = 0;
    }
  }
  o->rev += nturns;
  o->dev_in = NULL;
  o->dev_out = NULL;
  return o->dev_pos;
}

void orc_state(const orc_ctx *o, int ib, double *vrf_phi, double *phasor_lon)
{
  int l;
  vrf_phi[0] = o->b[ib].Vrf0;
  vrf_phi[1] = o->b[ib].phai0;
  for (l = 0; l < o->p.n_lr[LON]; l++) {
    phasor_lon[2 * l] = o->b[ib].phasor[LON][l][0];
    phasor_lon[2 * l + 1] = o->b[ib].phasor[LON][l][1];
  }
}

void orc_trash(const orc_ctx *o, int ib, int *low, int *high)
{
  *low = o->b[ib].trash_low;
  *high = o->b[ib].trash_high;
}

void orc_histograms(const orc_ctx *o, int ib, double *fnp, double *dipV,
                    double *dipH, double *ring_lon, double *ring_hor,
                    double *ring_ver)
{
  const orc_bunch *b = &o->b[ib];
  const int Nc = o->p.ncell;
  if (fnp) memcpy(fnp, b->fnp + PAD, Nc * sizeof(double));
  if (dipV) memcpy(dipV, b->dipV + PAD, Nc * sizeof(double));
  if (dipH) memcpy(dipH, b->dipH + PAD, Nc * sizeof(double));
  if (ring_lon) memcpy(ring_lon, o->fnp_ring[LON] + (size_t) b->kb * Nc, Nc * sizeof(double));
  if (ring_hor) memcpy(ring_hor, o->fnp_ring[HOR] + (size_t) b->kb * Nc, Nc * sizeof(double));
  if (ring_ver) memcpy(ring_ver, o->fnp_ring[VER] + (size_t) b->kb * Nc, Nc * sizeof(double));
}

/* ------------------------------------------------------------ w(z) */

/* ACM TOMS Algorithm 680 (G.P.M. Poppe, C.M.J. Wijers, "More efficient
 * computation of the complex error function", ACM TOMS 16(1), 1990, p.47),
 * with the region constants and term counts of physic.c:143-301:
 * power series for qrho < 0.085264, Laplace continued fraction for
 * qrho > 1, truncated Taylor series with continued-fraction derivatives in
 * between; reflection for the lower half plane. */
int orc_wofz(double xi, double yi, double *re, double *im)
{
  const double factor = 1.12837916709551257388;   /* 2/sqrt(pi) */
  const double rmaxreal = 0.5e154;
  const double rmaxexp = 708.503061461606;
  const double rmaxgoni = 3.53711887601422e08;
  double xabs = fabs(xi), yabs = fabs(yi);
  double x = xabs / 6.3, y = yabs / 4.4;
  double qrho, xquad, yquad, u = 0, v = 0, u2 = 0, v2 = 0;
  int series = 0;
  if (xabs > rmaxreal || yabs > rmaxreal) return -1;
  qrho = x * x + y * y;
  xquad = xabs * xabs - yabs * yabs;
  yquad = 2.0 * xabs * yabs;
  if (qrho < 0.085264) {
    int n, i, j;
    double xsum, ysum, xaux, u1, v1, daux;
    series = 1;
    qrho = (1.0 - 0.85 * y) * sqrt(qrho);
    n = (int) (6.0 + 72.0 * qrho);
    j = 2 * n + 1;
    xsum = 1.0 / ((double) j);
    ysum = 0.0;
    for (i = n; i >= 1; i--) {
      j = j - 2;
      xaux = (xsum * xquad - ysum * yquad) / ((double) i);
      ysum = (xsum * yquad + ysum * xquad) / ((double) i);
      xsum = xaux + 1.0 / ((double) j);
    }
    u1 = -factor * (xsum * yabs + ysum * xabs) + 1.0;
    v1 = factor * (xsum * xabs - ysum * yabs);
    daux = exp(-xquad);
    u2 = daux * cos(yquad);
    v2 = -daux * sin(yquad);
    u = u1 * u2 - v1 * v2;
    v = u1 * v2 + v1 * u2;
  } else {
    double h, h2 = 0, qlamda = 0, rx, ry, sx, sy, tx, ty, c;
    int kapn, nu, n, np1, useb;
    if (qrho > 1.0) {
      h = 0.0;
      kapn = 0;
      qrho = sqrt(qrho);
      nu = (int) (3.0 + 1442.0 / (26.0 * qrho + 77.0));
    } else {
      qrho = (1.0 - y) * sqrt(1.0 - qrho);
      h = 1.88 * qrho;
      h2 = 2.0 * h;
      kapn = (int) (7.0 + 34.0 * qrho);
      nu = (int) (16.0 + 26.0 * qrho);
    }
    useb = (h > 0.0);
    if (useb) qlamda = pow(h2, kapn);
    rx = ry = sx = sy = 0.0;
    for (n = nu; n >= 0; n--) {
      np1 = n + 1;
      tx = yabs + h + np1 * rx;
      ty = xabs - np1 * ry;
      c = 0.5 / (tx * tx + ty * ty);
      rx = c * tx;
      ry = c * ty;
      if (useb && n <= kapn) {
        tx = qlamda + sx;
        sx = rx * tx - ry * sy;
        sy = ry * tx + rx * sy;
        qlamda = qlamda / h2;
      }
    }
    if (h == 0.0) { u = factor * rx; v = factor * ry; }
    else { u = factor * sx; v = factor * sy; }
    if (yabs == 0.0) u = exp(-xabs * xabs);
  }
  if (yi < 0.0) {
    if (series) {
      u2 = 2.0 * u2;
      v2 = 2.0 * v2;
    } else {
      double w1;
      xquad = -xquad;
      if ((yquad > rmaxgoni) || (xquad > rmaxexp)) return -1;
      w1 = 2.0 * exp(xquad);
      u2 = w1 * cos(yquad);
      v2 = -w1 * sin(yquad);
    }
    u = u2 - u;
    v = v2 - v;
    if (xi > 0.0) v = -v;
  } else {
    if (xi < 0.0) v = -v;
  }
  *re = u;
  *im = v;
  return 1;
}

void orc_wofz_n(long n, const double *x, const double *y, double *re, double *im, int *flag)
{
  long i;
  for (i = 0; i < n; i++) {
    int f = orc_wofz(x[i], y[i], &re[i], &im[i]);
    if (f < 0) { re[i] = 0.0; im[i] = 0.0; }
    if (flag) flag[i] = f;
  }
}

/* fbi_weakstrong.c:160-191 for one slice: xi1 = Dx/factBE,
 * xi2 = xi1 sgm_zz/sgm_xx, yi1 = Dy/factBE, yi2 = yi1 sgm_xx/sgm_zz,
 * E = -factdQ [w(z1) - exp(-(Dx^2 1e6/(2 sx^2) + Dy^2 1e6/(2 sz^2))) w(z2)],
 * Ex from the imaginary parts, Ey from the real parts. */
void orc_be_field_n(long n, const double *dx, const double *dy,
                    double sgm_xx, double sgm_zz, double factdQ,
                    double *ex, double *ey)
{
  const double factBE = sqrt(2 * (sgm_xx * sgm_xx - sgm_zz * sgm_zz)) / FKILO;
  long i;
  for (i = 0; i < n; i++) {
    double Dx = dx[i], Dy = dy[i];
    double xi1 = Dx / factBE;
    double xi2 = xi1 * sgm_zz / sgm_xx;
    double yi1 = Dy / factBE;
    double yi2 = yi1 * sgm_xx / sgm_zz;
    double u1[2], u2[2];
    orc_wofz(xi1, yi1, &u1[0], &u1[1]);
    orc_wofz(xi2, yi2, &u2[0], &u2[1]);
    double e = exp(-(Dx * Dx * FMEGA / (2 * sgm_xx * sgm_xx) + Dy * Dy * FMEGA / (2 * sgm_zz * sgm_zz)));
    ex[i] = -factdQ * (u1[1] - e * u2[1]);
    ey[i] = -factdQ * (u1[0] - e * u2[0]);
  }
}

/* weak_bunch_calc_ampinv, statistics.c:163-195: per tracked plane the mean
 * of gamma u^2 + 2 alpha u u' + beta u'^2 over the particles (ampinv) and
 * the same of the centroid of the last statistics (ampinv_cm). */
void orc_ampinv(const orc_ctx *o, int ib, double *out6)
{
  const orc_bunch *b = &o->b[ib];
  const mbt_params *p = &o->p;
  int plane, jp;
  for (plane = 0; plane < 3; plane++) {
    out6[plane] = 0.0;
    out6[3 + plane] = 0.0;
    if (!p->track_plane[plane]) continue;
    {
      const double *u = b->c[plane], *up = b->c[3 + plane];
      double s = 0.0;
      const double pos = b->stats[0 + plane], slope = b->stats[6 + plane];
      for (jp = 0; jp < b->np; jp++)
        s += p->gamma1[plane] * (u[jp] * u[jp]) + 2.0 * p->alpha1[plane] * u[jp] * up[jp]
             + p->beta1[plane] * (up[jp] * up[jp]);
      out6[plane] = s / ((double) b->np);
      out6[3 + plane] = p->gamma1[plane] * (pos * pos) + 2.0 * p->alpha1[plane] * pos * slope
                        + p->beta1[plane] * (slope * slope);
    }
  }
}
