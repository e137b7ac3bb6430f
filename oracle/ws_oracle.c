/*
 * ws_oracle.c -- CPU oracle for the slice model (BunchModel = STRONG) with
 * fast beam-ion interaction.
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference's
 * algorithm (fracul/mtrack manager_weakstrong.c:7-263,
 * worker_weakstrong.c:13-247, rw_weakstrong.c, fbi_weakstrong.c:45-580,
 * bunch_strong.c:59-270, bunch.c:95-224,468-549), used by tests/ as the
 * checker of the device path.  The product never links it.
 *
 * Every expression keeps the reference's operand order and every sum its
 * loop order, so the oracle reproduces the reference bit for bit; it is
 * pinned against the reference's own functions run by ref_ws_harness.c.
 * Two departures, both where the reference's message passing or set-up
 * loses data, not in its arithmetic:
 *   - the centroid history is kept whole; the reference's manager sends
 *     the workers only the first 5000 entries of its sorted history
 *     (manager_weakstrong.c:155-158), which drops entries once
 *     (Nmlt + 2) x nharm exceeds 5000;
 *   - the bunch currents are the caller's (the reference's slice-model
 *     manager leaves ring.Ibunch at zero).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "mbt_oracle.h"

#define ORC_C_LIGHT 2.997925e+08
#define ORC_EPSILON0 8.854187817620e-12
#define ORC_E_CHARGE 1.602e-19
#define ORC_E_RADIUS 2.819e-15
#define ORC_FKILO 1.0e+03
#define ORC_FMEGA 1.0e+06
#define ORC_FTERA 1.0e+12

struct ows {
  mbt_ws_params w;
  int nb, S, G, off, nion, nmt;
  int *bucket;
  double *ib;          /* [nb] mA */
  int *npop;           /* [S] */
  int *nofe;           /* [S][G][G] */
  double *s;           /* [nb][6][S] */
  double *hist;        /* [nb][4][nmt]: xx, xp, zz, zp, newest first */
  double *ex, *ey;     /* [nb][nion] */
  double *li;          /* [nb][5][nion] local ions: N, x, xd, y, yd */
  double *L;           /* ion list [5][nb nion] */
  long rev;
};

#define SL(o, ib, k) ((o)->s + ((size_t) (ib) * 6 + (k)) * (o)->S)

int ows_slice_beam(const mbt_ws_params *w, const double *soa6, int np, int *npop, int *nofe, double *cm4)
{
  /* strong_generate_eCMs bunch_strong.c:117-198 */
  const int S = 2 * w->nslc + 1, G = w->ngrid, off = (G - 1) / 2;
  const double *t0 = soa6, *x0 = soa6 + np, *z0 = soa6 + 2 * (size_t) np;
  const double *xp0 = soa6 + 4 * (size_t) np, *zp0 = soa6 + 5 * (size_t) np;
  int *cell = (int *) malloc((size_t) np * sizeof(int));
  int *cnt = (int *) calloc((size_t) S + 1, sizeof(int));
  double *sum = (double *) calloc(4 * ((size_t) S + 1), sizeof(double));
  int jp, c;
  if (!cell || !cnt || !sum) { free(cell); free(cnt); free(sum); return -1; }
  for (jp = 0; jp < np; jp++) {
    const double Tau = -t0[jp] / w->sgmatau;
    int icell = (int) ((w->max_tau + Tau) / w->dtau);
    if (icell < 1) icell = 0;
    if (icell > S) icell = S;
    cell[jp] = icell;
    cnt[icell]++;
    sum[icell] = sum[icell] + x0[jp];
    sum[(S + 1) + icell] = sum[(S + 1) + icell] + xp0[jp];
    sum[2 * (S + 1) + icell] = sum[2 * (S + 1) + icell] + z0[jp];
    sum[3 * (S + 1) + icell] = sum[3 * (S + 1) + icell] + zp0[jp];
  }
  for (c = 0; c < S; c++) {
    int k;
    npop[c] = cnt[c];
    for (k = 0; k < 4; k++)
      cm4[k * S + c] = cnt[c] ? sum[k * (S + 1) + c] / cnt[c] : sum[k * (S + 1) + c];
  }
  memset(nofe, 0, (size_t) S * G * G * sizeof(int));
  for (jp = 0; jp < np; jp++) {
    const int icell = cell[jp];
    int nsx, nsz, msx, msz;
    if (icell >= S) continue;
    nsz = (int) (2.0 * (z0[jp] - cm4[2 * S + icell]) / w->agLOCz);
    msz = nsz >= 0 ? (nsz + 1) / 2 : (nsz - 1) / 2;
    if (msz > off) msz = off;
    if (msz < -off) msz = -off;
    nsx = (int) (2.0 * (x0[jp] - cm4[icell]) / w->agLOCx);
    msx = nsx >= 0 ? (nsx + 1) / 2 : (nsx - 1) / 2;
    if (msx > off) msx = off;
    if (msx < -off) msx = -off;
    nofe[(icell * G + msx + off) * G + msz + off]++;
  }
  free(cell); free(cnt); free(sum);
  return 0;
}

ows_t *ows_create(const mbt_ws_params *w, int nb, const int *bucket, const double *ibunch, const int *npop,
                  const int *nofe)
{
  ows_t *o = (ows_t *) calloc(1, sizeof(ows_t));
  if (!o) return NULL;
  o->w = *w;
  o->nb = nb;
  o->S = 2 * w->nslc + 1;
  o->G = w->ngrid;
  o->off = (w->ngrid - 1) / 2;
  o->nion = o->S * o->G * o->G;
  o->nmt = w->base.Nmlt + 2;
  o->bucket = (int *) malloc(nb * sizeof(int));
  o->ib = (double *) malloc(nb * sizeof(double));
  o->npop = (int *) malloc(o->S * sizeof(int));
  o->nofe = (int *) malloc((size_t) o->nion * sizeof(int));
  o->s = (double *) calloc((size_t) nb * 6 * o->S, sizeof(double));
  o->hist = (double *) calloc((size_t) nb * 4 * o->nmt, sizeof(double));
  o->ex = (double *) calloc((size_t) nb * o->nion, sizeof(double));
  o->ey = (double *) calloc((size_t) nb * o->nion, sizeof(double));
  o->li = (double *) calloc((size_t) nb * 5 * o->nion, sizeof(double));
  o->L = (double *) calloc((size_t) 5 * nb * o->nion, sizeof(double));
  if (!o->bucket || !o->ib || !o->npop || !o->nofe || !o->s || !o->hist || !o->ex || !o->ey || !o->li || !o->L) {
    ows_destroy(o);
    return NULL;
  }
  memcpy(o->bucket, bucket, nb * sizeof(int));
  memcpy(o->ib, ibunch, nb * sizeof(double));
  memcpy(o->npop, npop, o->S * sizeof(int));
  memcpy(o->nofe, nofe, (size_t) o->nion * sizeof(int));
  return o;
}

void ows_destroy(ows_t *o)
{
  if (!o) return;
  free(o->bucket); free(o->ib); free(o->npop); free(o->nofe); free(o->s); free(o->hist);
  free(o->ex); free(o->ey); free(o->li); free(o->L);
  free(o);
}

void ows_set_slices(ows_t *o, const double *s) { memcpy(o->s, s, (size_t) o->nb * 6 * o->S * sizeof(double)); }
void ows_get_slices(const ows_t *o, double *s) { memcpy(s, o->s, (size_t) o->nb * 6 * o->S * sizeof(double)); }

/* get_linearly_interpolated_Efields fbi_weakstrong.c:454-580: the grid
   cell towards the origin-far side of (xx, yy), truncated index, linear in
   each axis, constant beyond the grid */
static void ows_interp(const ows_t *o, const double *Ex, const double *Ey, int icell, double xx, double yy,
                       double *ex, double *ey)
{
  const int off = o->off, G = o->G;
  const double ax = o->w.agABSx, az = o->w.agABSz;
  const int px = xx >= 0, pz = yy >= 0;
  int k1x = (int) (xx / ax), k1z = (int) (yy / az), k2x, k2z, ic1, ic2, ic3, ic4;
  double fx, fz, ey5, ey6, ex5, ex6;
  if (pz) {
    k2z = k1z < off ? k1z + 1 : k1z;
    if (k1z > off) k1z = off;
    if (k2z > off) k2z = off;
  } else {
    k2z = k1z > -off ? k1z - 1 : k1z;
    if (k1z < -off) k1z = -off;
    if (k2z < -off) k2z = -off;
  }
  if (px) {
    k2x = k1x < off ? k1x + 1 : k1x;
    if (k1x > off) k1x = off;
    if (k2x > off) k2x = off;
  } else {
    k2x = k1x > -off ? k1x - 1 : k1x;
    if (k1x < -off) k1x = -off;
    if (k2x < -off) k2x = -off;
  }
  ic1 = (icell * G + k1x + off) * G + k1z + off;
  ic2 = (icell * G + k2x + off) * G + k1z + off;
  ic3 = (icell * G + k1x + off) * G + k2z + off;
  ic4 = (icell * G + k2x + off) * G + k2z + off;
  fx = (xx - k1x * ax) / ax;
  fz = (yy - k1z * az) / az;
  if (px) {
    ey5 = Ey[ic1] + fx * (Ey[ic2] - Ey[ic1]);
    ey6 = Ey[ic3] + fx * (Ey[ic4] - Ey[ic3]);
    ex5 = Ex[ic1] + fx * (Ex[ic2] - Ex[ic1]);
    ex6 = Ex[ic3] + fx * (Ex[ic4] - Ex[ic3]);
  } else {
    ey5 = Ey[ic1] - fx * (Ey[ic2] - Ey[ic1]);
    ey6 = Ey[ic3] - fx * (Ey[ic4] - Ey[ic3]);
    ex5 = Ex[ic1] - fx * (Ex[ic2] - Ex[ic1]);
    ex6 = Ex[ic3] - fx * (Ex[ic4] - Ex[ic3]);
  }
  *ey = pz ? ey5 + fz * (ey6 - ey5) : ey5 - fz * (ey6 - ey5);
  *ex = pz ? ex5 + fz * (ex6 - ex5) : ex5 - fz * (ex6 - ex5);
}

void ows_interp_n(const ows_t *o, int ib, int icell, const double *x, const double *y, int n, double *exey)
{
  int i;
  for (i = 0; i < n; i++)
    ows_interp(o, o->ex + (size_t) ib * o->nion, o->ey + (size_t) ib * o->nion, icell, x[i], y[i], &exey[2 * i],
               &exey[2 * i + 1]);
}

/* slice-weighted centroid (bunch_strong_updateCM bunch_strong.c:221-270) */
static void ows_cm(const ows_t *o, const double *u, const double *up, double *pu, double *pp)
{
  double uu = 0.0, ss = 0.0;
  int n = 0, c;
  for (c = 0; c < o->S; c++) {
    uu += u[c] * ((double) o->npop[c]);
    ss += up[c] * ((double) o->npop[c]);
    n += o->npop[c];
  }
  *pu = uu / ((double) n);
  *pp = ss / ((double) n);
}

/* bunch_strong_distribution_statistics bunch.c:516-549 for one plane */
static void ows_plane_stats(const ows_t *o, int plane, const double *u, const double *up, double *st)
{
  const mbt_params *p = &o->w.base;
  double pos, slope, sq = 0.0, sp = 0.0, ai = 0.0;
  int c, n = 0, na = 0;
  ows_cm(o, u, up, &pos, &slope);
  for (c = 0; c < o->S; c++) {
    sq += (u[c] - pos) * (u[c] - pos) * o->npop[c];
    sp += (up[c] - slope) * (up[c] - slope) * o->npop[c];
    n += o->npop[c];
  }
  for (c = 0; c < o->S; c++) {
    ai += o->npop[c] * (p->gamma1[plane] * pow(u[c], 2) + 2.0 * p->alpha1[plane] * u[c] * up[c]
                        + p->beta1[plane] * pow(up[c], 2));
    na += o->npop[c];
  }
  st[plane] = pos;
  st[3 + plane] = sqrt(sq / ((double) n));
  st[6 + plane] = slope;
  st[9 + plane] = sqrt(sp / ((double) n));
  st[12 + plane] = ai / ((double) na);
  st[15 + plane] = p->gamma1[plane] * pow(pos, 2) + 2.0 * p->alpha1[plane] * pos * slope
                   + p->beta1[plane] * pow(slope, 2);
}

/* phase 1 of bunch ib: transformSbunch_shortrange rw_weakstrong.c:24-47 and
   fbi_weakstrong_bunch fbi_weakstrong.c:98-290 */
static void ows_bunch(ows_t *o, int ib, long rev, double *cm, double *stats)
{
  const mbt_ws_params *w = &o->w;
  const mbt_params *p = &w->base;
  const int S = o->S, G = o->G, off = o->off, n = o->nion;
  double *xtau = SL(o, ib, 0), *xeps = SL(o, ib, 1), *xx = SL(o, ib, 2), *xp = SL(o, ib, 3);
  double *zz = SL(o, ib, 4), *zp = SL(o, ib, 5);
  double c6[6];
  int c, j, k;
  for (c = 0; c < S; c++) {
    const double gain = p->Vrf0 / (p->E0 * ORC_FKILO) * sin(p->wrf * xtau[c] + p->phai0);
    const double e0 = xeps[c];
    xeps[c] = e0 + gain - p->Urad;
    xtau[c] = xtau[c] - e0 * p->T0 * p->ac;
  }
  ows_cm(o, xtau, xeps, &c6[0], &c6[1]);
  ows_cm(o, xx, xp, &c6[2], &c6[3]);
  ows_cm(o, zz, zp, &c6[4], &c6[5]);
  if (cm) memcpy(cm, c6, sizeof c6);
  {
    double *h = o->hist + (size_t) ib * 4 * o->nmt;
    for (k = 0; k < 4; k++) {
      for (j = o->nmt - 2; j >= 0; j--) h[k * o->nmt + j + 1] = h[k * o->nmt + j];
      h[k * o->nmt] = c6[2 + k];
    }
  }
  if (stats) {
    memset(stats, 0, 18 * sizeof(double));
    if (p->track_plane[0]) ows_plane_stats(o, 0, xtau, xeps, stats);
    if (p->track_plane[1]) ows_plane_stats(o, 1, xx, xp, stats);
    if (p->track_plane[2]) ows_plane_stats(o, 2, zz, zp, stats);
  }
  if (!w->fbii) return;
  {
    const double Nelec = (o->ib[ib] * p->T0 / (w->np * ORC_E_CHARGE * ORC_FKILO));
    const double Convion = Nelec * w->Ldmsgm;
    double *Ex = o->ex + (size_t) ib * n, *Ey = o->ey + (size_t) ib * n;
    double *N = o->li + (size_t) ib * 5 * n, *X = N + n, *XD = N + 2 * n, *Y = N + 3 * n, *YD = N + 4 * n;
    int ic = 0, ip, msx, msz;
    for (c = 0; c < S; c++) {
      const double dQ = Nelec * o->npop[c] * ORC_E_CHARGE;
      const double factdQ = dQ / (2 * ORC_EPSILON0 * sqrt(M_PI) * w->factBE * ORC_C_LIGHT * w->deltT);
      for (msx = -off; msx < off + 1; msx++) {
        const double Dx = msx * w->agABSx - xx[c];
        const double xi1 = Dx / w->factBE, xi2 = xi1 * w->sgm_zz / w->sgm_xx;
        for (msz = -off; msz < off + 1; msz++) {
          const double Dy = msz * w->agABSz - zz[c];
          const double yi1 = Dy / w->factBE, yi2 = yi1 * w->sgm_xx / w->sgm_zz;
          double u1[2], u2[2], e;
          orc_wofz(xi1, yi1, &u1[0], &u1[1]);
          orc_wofz(xi2, yi2, &u2[0], &u2[1]);
          e = exp(-(Dx * Dx * ORC_FMEGA / (2 * w->sgm_xx * w->sgm_xx)
                    + Dy * Dy * ORC_FMEGA / (2 * w->sgm_zz * w->sgm_zz)));
          Ex[ic] = -factdQ * (u1[1] - e * u2[1]);
          Ey[ic] = -factdQ * (u1[0] - e * u2[0]);
          ic++;
        }
      }
    }
    ip = 0;
    for (c = 0; c < S; c++) {
      const int ip0 = ip;
      int q;
      for (msx = -off; msx < off + 1; msx++)
        for (msz = -off; msz < off + 1; msz++) {
          N[ip] = Convion * ((double) o->nofe[(c * G + msx + off) * G + msz + off]);
          X[ip] = xx[c] + msx * w->agLOCx;
          XD[ip] = 0.0;
          Y[ip] = zz[c] + msz * w->agLOCz;
          YD[ip] = 0.0;
          ip++;
        }
      for (q = 0; q < ip0; q++) {
        double ex, ey;
        ows_interp(o, Ex, Ey, c, X[q], Y[q], &ex, &ey);
        XD[q] = XD[q] + w->deltT * (w->factF * ex);
        X[q] = X[q] + w->deltT * XD[q];
        YD[q] = YD[q] + w->deltT * (w->factF * ey);
        Y[q] = Y[q] + w->deltT * YD[q];
      }
    }
  }
}

/* phase 2 of bunch ib: transformSbunch_optic rw_weakstrong.c:194-253 and
   transformSbunch_longrange :68-192 */
static void ows_optic_rw(ows_t *o, int ib, long rev)
{
  const mbt_ws_params *w = &o->w;
  const mbt_params *p = &w->base;
  const int S = o->S;
  const int kb = o->bucket[ib];
  double *xx = SL(o, ib, 2), *xp = SL(o, ib, 3), *zz = SL(o, ib, 4), *zp = SL(o, ib, 5);
  int c, pl;
  {
    const double PsiV0 = 2.0 * M_PI * p->QV0 / 1.0, PsiH0 = 2.0 * M_PI * p->QH0 / 1.0;
    const double cV = cos(PsiV0), sV = sin(PsiV0), cH = cos(PsiH0), sH = sin(PsiH0);
    const double v11 = cV + p->alpha1[2] * sV, v12 = p->beta1[2] * sV;
    const double v21 = -p->gamma1[2] * sV, v22 = cV - p->alpha1[2] * sV;
    const double h11 = cH + p->alpha1[1] * sH, h12 = p->beta1[1] * sH;
    const double h21 = -p->gamma1[1] * sH, h22 = cH - p->alpha1[1] * sH;
    for (c = 0; c < S; c++) {
      const double y = v11 * zz[c] + v12 * zp[c], yp = v21 * zz[c] + v22 * zp[c];
      const double x = h11 * xx[c] + h12 * xp[c], xq = h21 * xx[c] + h22 * xp[c];
      zz[c] = y; zp[c] = yp;
      xx[c] = x; xp[c] = xq;
    }
  }
  if (!p->rw_long) return;
  for (pl = 1; pl <= 2; pl++) {
    const double Psi0 = 2.0 * M_PI * (pl == 1 ? p->QH0 : p->QV0) / 1.0;
    double beff3 = pow(pl == 1 ? p->beffH[0] : p->beffV[0], 3);
    const double Pref0 = p->T0 / p->E0 / (double) w->np / ORC_FTERA;
    const double kappa = 1.0 / 2.8e-08;
    const double fNharm = (double) p->nharm;
    const double Dub0 = p->Lc / fNharm;
    const double R = p->Lc / (2.0 * M_PI);
    const double Psi = 0.0 + Psi0;
    const double cP = cos(Psi), sP = sin(Psi);
    const double a11 = cP + p->alpha1[pl] * sP, a12 = +p->beta1[pl] * sP;
    double prfrw, *up = pl == 1 ? xp : zp;
    int jb;
    if (!p->track_plane[pl]) continue;
    if (p->triggerRW && rev < 50) beff3 = pow(2.0e-3, 3);
    prfrw = 2.0 * R / (beff3) / sqrt(M_PI * kappa * ORC_EPSILON0) / 1.0;
    for (jb = 0; jb < o->nb; jb++) {
      const int sb = o->bucket[jb];
      const double *uh = o->hist + ((size_t) jb * 4 + (pl == 1 ? 0 : 2)) * o->nmt;
      const double *ph = uh + o->nmt;
      double uj[32], Dup = 0.0, D0;
      int j;
      for (j = 0; j < o->nmt; j++) uj[j] = a11 * uh[j] + a12 * ph[j];
      D0 = p->Lc;
      if (sb > kb) D0 = ((double) (sb - kb)) * Dub0;
      if (sb < kb) D0 = ((double) (p->nharm + sb - kb)) * Dub0;
      for (j = 0; j < p->Nmlt + 1; j++) {
        const double Dujk = D0 + ((double) j) * p->Lc;
        const double Dtjk = Dujk / ORC_C_LIGHT;
        const double Wrwt = prfrw / sqrt(Dtjk);
        const int jm = sb > kb ? j : j + 1;
        const double dip = (double) w->np * uj[jm];
        Dup = Dup + dip * Wrwt;
      }
      Dup = Pref0 * o->ib[jb] * Dup;
      if (rev < p->Nmlt) Dup = 0.0;
      for (c = 0; c < S; c++) up[c] += Dup;
    }
  }
}

int ows_run(ows_t *o, long nturns, double *cm, double *ion, double *zcm, double *stats)
{
  const mbt_ws_params *w = &o->w;
  const mbt_params *p = &w->base;
  const int nb = o->nb, S = o->S, n = o->nion;
  long t, imon = 0;
  int ib, c;
  if (o->nmt > 32) return -1;
  for (t = 0; t < nturns; t++, o->rev++) {
    const long rev = o->rev;
    const int mon = rev % p->nrev_mon == 0;
    for (ib = 0; ib < nb; ib++)
      ows_bunch(o, ib, rev, cm ? cm + ((size_t) t * nb + ib) * 6 : NULL,
                (mon && stats) ? stats + ((size_t) imon * nb + ib) * 18 : NULL);
    if (mon) imon++;
    for (ib = 0; ib < nb; ib++) ows_optic_rw(o, ib, rev);
    {
      /* fbi_weakstrong_train fbi_weakstrong.c:325-448 on the list
         N, X, XD, Y, YD of nF ions */
      const size_t cap = (size_t) nb * n;
      double *N = o->L, *X = N + cap, *XD = N + 2 * cap, *Y = N + 3 * cap, *YD = N + 4 * cap;
      long nF = 0;
      int kbF = 0;
      for (ib = 0; ib < nb; ib++) {
        const int kb = o->bucket[ib];
        const double *li = o->li + (size_t) ib * 5 * n;
        long q;
        if (w->fbii && ib > 0) {
          const double factjp0 = w->kick_factor * 4.0 * M_PI * ORC_EPSILON0 * ORC_E_RADIUS / w->Gamma;
          const double Nelec = (o->ib[ib] * p->T0 / (w->np * ORC_E_CHARGE * ORC_FKILO));
          const double Dtime = fabs((double) (kb - kbF)) * (p->T0 / (double) p->nharm);
          const double *Ex = o->ex + (size_t) ib * n, *Ey = o->ey + (size_t) ib * n;
          double *xp = SL(o, ib, 3), *zp = SL(o, ib, 5);
          for (q = 0; q < nF; q++) {
            X[q] = X[q] + Dtime * XD[q];
            Y[q] = Y[q] + Dtime * YD[q];
          }
          for (c = 0; c < S; c++) {
            const double dQ = Nelec * o->npop[c] * ORC_E_CHARGE;
            const double factjp = dQ > 0.0 ? factjp0 / dQ : 0.0;
            double sx = 0.0, sy = 0.0;
            for (q = 0; q < nF; q++) {
              double ex, ey;
              ows_interp(o, Ex, Ey, c, X[q], Y[q], &ex, &ey);
              XD[q] = XD[q] + w->deltT * (w->factF * ex);
              X[q] = X[q] + w->deltT * XD[q];
              YD[q] = YD[q] + w->deltT * (w->factF * ey);
              Y[q] = Y[q] + w->deltT * YD[q];
              sx = sx + N[q] * ex;
              sy = sy + N[q] * ey;
            }
            sx = factjp * sx;
            sy = factjp * sy;
            xp[c] = xp[c] + ORC_C_LIGHT * w->deltT * sx;
            zp[c] = zp[c] + ORC_C_LIGHT * w->deltT * sy;
          }
        }
        if (w->fbii) {
          for (q = 0; q < n; q++) {
            N[nF] = li[q]; X[nF] = li[n + q]; XD[nF] = li[2 * n + q]; Y[nF] = li[3 * n + q]; YD[nF] = li[4 * n + q];
            nF++;
          }
          kbF = kb;
        }
        if (ion) {
          double xs = 0.0, ys = 0.0, nt = 0.0;
          for (q = 0; q < nF; q++) {
            xs = xs + N[q] * X[q];
            ys = ys + N[q] * Y[q];
            nt = nt + N[q];
          }
          ion[((size_t) t * nb + ib) * 2] = nt == 0.0 ? NAN : xs / nt;
          ion[((size_t) t * nb + ib) * 2 + 1] = nt == 0.0 ? NAN : ys / nt;
        }
      }
    }
    if (zcm) {
      double *zt = zcm + (size_t) t * p->nharm;
      memset(zt, 0, p->nharm * sizeof(double));
      for (ib = 0; ib < nb; ib++) {
        const double *zz = SL(o, ib, 4);
        double z = 0.0;
        for (c = 0; c < S; c++) z = z + zz[c];
        zt[o->bucket[ib]] = z / ((double) S);
      }
    }
  }
  return 0;
}

void ows_bunch_fields(const ows_t *o, int ib, double *exey, double *ions5)
{
  const int n = o->nion;
  int i;
  for (i = 0; i < n; i++) {
    if (exey) {
      exey[2 * i] = o->ex[(size_t) ib * n + i];
      exey[2 * i + 1] = o->ey[(size_t) ib * n + i];
    }
  }
  if (ions5) memcpy(ions5, o->li + (size_t) ib * 5 * n, 5 * (size_t) n * sizeof(double));
}
