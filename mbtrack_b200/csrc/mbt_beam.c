/*
 * mbt_beam.c -- the reference's initial macroparticle distribution on the
 * host.
 *
 * The reference generates each bunch in its own MPI worker process
 * (worker_weakweak.c:66-68 -> weak_generate_bunch_distribution
 * bunch_weak.c:173-292).  Per tracked plane (LON, then HOR, then VER) and
 * per particle it draws two Irwin-Hall normals (c_fnorm bunch.c:379-405:
 * twelve rand()/RAND_MAX uniforms, each minus 0.5, summed in order) and sets
 * pos = offset + sgm g1, slope = offset + sgm g2 + correlate (sgm g1)
 * (weak_bunch_normal_distribution bunch_weak.c:86-105).  The generator is
 * glibc's rand(): a fresh process starts from the state of seed 1, and
 * c_fnorm reseeds with srand(iseed) whenever iseed differs from the last
 * seed it saw, which starts at 0 (bunch.h:17).  The seed of a plane is
 * iseed[plane] + bucket number.
 *
 * Each call here owns a private glibc random_r state set up the same way,
 * so bunches can be generated concurrently and every bunch gets exactly the
 * numbers its worker process would draw.
 */
#define _DEFAULT_SOURCE
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "mbt.h"
#include "mbt_ws.h"

typedef struct beam_rng {
  struct random_data rd;
  char state[128];      /* TYPE_3, the state size of glibc's rand() */
  int last_seed;
} beam_rng;

static void rng_open(beam_rng *r)
{
  memset(r, 0, sizeof(*r));
  initstate_r(1u, r->state, sizeof(r->state), &r->rd);
  r->last_seed = 0;
}

/* c_fnorm: sum of twelve uniforms on [0, 1], each shifted by -0.5 */
static double irwin_hall12(beam_rng *r, int seed)
{
  double s = 0.0;
  int i;
  if (seed != r->last_seed) {
    srandom_r((unsigned) seed, &r->rd);
    r->last_seed = seed;
  }
  for (i = 0; i < 12; i++) {
    int32_t v;
    random_r(&r->rd, &v);
    s = s + (((double) v) / ((double) RAND_MAX) - 0.5);
  }
  return s;
}

int mbt_reference_beam(const mbt_params *p, int bucket, int np, double *soa6)
{
  beam_rng r;
  int plane, j;
  if (!p || !soa6 || np < 0 || bucket < 0) return MBT_ERR_INVALID;
  memset(soa6, 0, (size_t) 6 * (size_t) np * sizeof(double));
  if (np == 0) return 0;
  if (np == 1) {
    for (plane = 0; plane < 3; plane++)
      if (plane == MBT_LON || p->track_plane[plane]) {
        soa6[plane] = p->pos_offset[plane];
        soa6[3 + plane] = p->slope_offset[plane];
      }
    return 0;
  }
  rng_open(&r);
  for (plane = 0; plane < 3; plane++) {
    double *pos = soa6 + (size_t) plane * np, *slope = soa6 + (size_t) (3 + plane) * np;
    const int seed = p->iseed[plane] + bucket;
    if (plane != MBT_LON && !p->track_plane[plane]) continue;
    for (j = 0; j < np; j++) {
      const double dpos = p->pos_sgm[plane] * irwin_hall12(&r, seed);
      pos[j] = p->pos_offset[plane] + dpos;
      slope[j] = p->slope_offset[plane] + p->slope_sgm[plane] * irwin_hall12(&r, seed) + p->correlate[plane] * dpos;
    }
  }
  return 0;
}

/* generate_initial_sbunch_distribution2 (bunch.c:226-330) for LON, HOR and
   VER in that order, as strong_generate_eCMs calls it (bunch_strong.c:
   80-91), then generate_initial_general_distribution2's offsets
   (bunch_strong.c:30-44) on the same generator: one fresh process. */
int mbt_ws_reference_beam(const mbt_ws_params *w, int nbunch, double *soa6, double *off4)
{
  beam_rng r;
  const int np = w ? w->np : 0;
  const double FN = 1.0e-09, FM = 1.0e-03;
  int j, plane, i;
  if (!w || !soa6 || np < 1 || nbunch < 0) return MBT_ERR_INVALID;
  rng_open(&r);
  for (plane = 0; plane < 3; plane++) {
    double *pos = soa6 + (size_t) plane * np, *slope = soa6 + (size_t) (3 + plane) * np;
    const int seed = w->base.iseed[plane];
    const double sp = w->sgm_in[2 * plane], ss = w->sgm_in[2 * plane + 1];
    const double cp = w->cm_in[2 * plane], cs = w->cm_in[2 * plane + 1];
    if (np == 1) {
      pos[0] = plane == 0 ? cp * FN : cp * FM;
      slope[0] = plane == 0 ? cs : cs * FM;
      continue;
    }
    for (j = 0; j < np; j++) {
      if (plane == 0) {
        pos[j] = (cp + sp * irwin_hall12(&r, seed)) * FN;
        slope[j] = cs + ss * irwin_hall12(&r, seed);
      } else {
        const double u = sp * irwin_hall12(&r, seed);
        const double v = ss * irwin_hall12(&r, seed);
        pos[j] = u * FM;
        slope[j] = v * FM;
      }
    }
  }
  if (off4)
    for (i = 0; i < nbunch; i++)
      for (j = 0; j < 4; j++) off4[4 * i + j] = w->cm_in[2 + j] * FM * irwin_hall12(&r, 571030);
  return 0;
}
