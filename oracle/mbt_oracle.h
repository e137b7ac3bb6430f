/*
 * mbt_oracle.h -- CPU oracle for the per-turn weak-weak tracking loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the
 * reference's algorithm (fracul/mtrack: worker_weakweak.c:259-394 with
 * transform_weak.c, statistics.c, feedback_rf.c, cyclic_array.c, bunch.c
 * and physic.c), used by tests/, by __graft_entry__.smoke() and by the
 * cpu_baseline leg of bench.py as the checker.  The product (libmbt) never
 * links or calls it.
 *
 * Parity: pinned bit-for-bit against the reference's own sources compiled
 * unmodified into oracle/_ref/libmbtref.so (see oracle/Makefile and
 * tests/test_oracle_pin.py), and against the known answers of
 * test_complexerrf.c:33-59 for w(z).
 */
#ifndef MBT_ORACLE_H
#define MBT_ORACLE_H

#include "mbt.h"
#include "mbt_ws.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

/* nbunch filled bunches: bucket numbers, macroparticle counts, currents [A].
 * Gl/Gv/Gh: p->ncell each (may be NULL when the plane count is 0). */
orc_ctx *orc_create(const mbt_params *p, int nbunch, const int *bucket,
                    const int *np, const double *ib, const double *Gl,
                    const double *Gv, const double *Gh);
void orc_destroy(orc_ctx *o);

/* Track only bunches [lo, hi): the others keep zero histograms and
 * dipoles, so the ring-wide phasor and resistive-wall sums still cost what
 * a full worker pays (used to split the CPU baseline over host cores). */
void orc_set_range(orc_ctx *o, int lo, int hi);

/* Matched Gaussian of the reference (weak_generate_bunch_distribution,
 * bunch_weak.c:173-292, c_fnorm bunch.c:379-405) with each bunch's own
 * glibc random() state, as each MPI worker process has. */
int orc_generate_beam(orc_ctx *o);
int orc_set_particles(orc_ctx *o, int ib, const double *soa6);
int orc_get_particles(const orc_ctx *o, int ib, double *soa6);

/* Worker set-up after the distribution exists (worker_weakweak.c:80-219). */
int orc_prepare(orc_ctx *o, double *init_stats);

/* nturns turns of worker_weakweak.c:259-394 for all bunches.
 * stats: nturns x nbunch x 12 (may be NULL).
 * dev_in: if non-NULL, deviates are taken from it (reference draw order,
 *   per turn, per bunch) instead of the Marsaglia generator.
 * dev_out: if non-NULL, every deviate used is also written there.
 * Returns the number of deviates used. */
long orc_run(orc_ctx *o, long nturns, double *stats, const float *dev_in,
             float *dev_out, long dev_cap);

/* Deviates one turn draws over all bunches (0 without EnableQuantum). */
long orc_deviates_per_turn(const orc_ctx *o);

void orc_state(const orc_ctx *o, int ib, double *vrf_phi, double *phasor_lon);

/* Amplitude invariants of bunch ib (statistics.c:163-195): ampinv[3],
 * ampinv_cm[3]. */
void orc_ampinv(const orc_ctx *o, int ib, double *out6);
void orc_trash(const orc_ctx *o, int ib, int *low, int *high);

/* Histograms of bunch ib from the last binning (clamped and dropped). */
void orc_histograms(const orc_ctx *o, int ib, double *fnp, double *dipV,
                    double *dipH, double *ring_lon, double *ring_hor,
                    double *ring_ver);

/* Faddeeva w(z), ACM TOMS 680 (Poppe & Wijers 1990), as in
 * complex_errorfunc_wofz_algo680 (physic.c:75-301).  Returns 1, or -1 in
 * the overflow region. */
int orc_wofz(double x, double y, double *re, double *im);
void orc_wofz_n(long n, const double *x, const double *y, double *re,
                double *im, int *flag);

/* Bassetti-Erskine field at offsets (dx, dy) [m] of a Gaussian slice with
 * rms sizes sgm_xx > sgm_zz given in mm, as fbi_weakstrong.c:155-191;
 * factdq is the reference's factdQ. */
void orc_be_field_n(long n, const double *dx, const double *dy,
                    double sgm_xx_mm, double sgm_zz_mm, double factdq,
                    double *ex, double *ey);

/* The beam-ion stage of mbt.h (mbt_beam_ion) after every turn's
 * statistics; clouds: n_ip x nbunch x 5 of the last turn. */
int orc_enable_beam_ion(orc_ctx *o, const mbt_beam_ion *bi);
void orc_beam_ion_clouds(const orc_ctx *o, double *clouds);
/* unit-charge field of an elliptic Gaussian (mbt_gauss_field_dev) */
void orc_gauss_field(double dx, double dy, double sx, double sy, double *gx, double *gy);

/* ---- slice model (BunchModel = STRONG) with fast beam-ion interaction:
 * ws_oracle.c, the restatement of manager_/worker_weakstrong.c,
 * rw_weakstrong.c and fbi_weakstrong.c; outputs as mbt_ws.h. */
typedef struct ows ows_t;
int ows_slice_beam(const mbt_ws_params *w, const double *soa6, int np, int *npop, int *nofe, double *cm4);
ows_t *ows_create(const mbt_ws_params *w, int nb, const int *bucket, const double *ibunch, const int *npop,
                  const int *nofe);
void ows_destroy(ows_t *o);
void ows_set_slices(ows_t *o, const double *s);
void ows_get_slices(const ows_t *o, double *s);
int ows_run(ows_t *o, long nturns, double *cm, double *ion, double *zcm, double *stats);
void ows_bunch_fields(const ows_t *o, int ib, double *exey, double *ions5);
void ows_interp_n(const ows_t *o, int ib, int icell, const double *x, const double *y, int n, double *exey);

#ifdef __cplusplus
}
#endif
#endif
