/*
 * mbt_host.c -- the C host side of libmbt: reads an mbtrack .conf file with
 * the reference's semantics and derives every parameter the per-turn loop
 * needs.
 *
 *   read_conf_file            input.c:278-850 (INI sections, keys, defaults)
 *   config_get / _have_section input.c:853-1100 (line scanner, first match,
 *                              duplicate sections count as missing)
 *   setup_ring_parameters     input.c:1553-1695
 *   macrop_model_setup_...    input.c:1775-1831
 *   e_beam_setup / fileread   input.c:1289-1512
 *   setup_tracking_parameters input.c:1698-1772
 *   construct_greensfunc_*    transform_weak.c:288-471
 *
 * Deliberate differences from the reference:
 *   - the set-up result is checked (mbtrack-mpi.c:97,148 ignore it);
 *   - with fix_rw_beff, beffH3/beffV3 are read whenever long-range RW is
 *     on (the reference reads them only with EnableRW_short,
 *     input.c:465-478, and then divides by zero in transform_weak.c:811);
 *   - long keys are parsed as longs (the reference scans "%d" into a long,
 *     input.c:1077, which only works for non-negative values);
 *   - the legacy .inp format and the excitation mode (modeHT) are
 *     rejected with MBT_ERR_CONFIG;
 *   - the first-bin values of the short-range resistive wall are the
 *     bin averages of the Bane-Sands wakes computed by quadrature
 *     (mbt_rw_first_bin), where the reference interpolates a printed
 *     table (rw_table.c); a bin narrower than 20 s0 is an error.
 */
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "mbt.h"
#include "mbt_ws.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define FNANO  1.0e-09
#define FMILLI 1.0e-03
#define FKILO  1.0e+03
#define FMEGA  1.0e+06
#define FGIGA  1.0e+09
#define C_LIGHT 2.997925e+08
#define Z_0     376.73
#define LINE_MAX_MBT 256

/* ------------------------------------------------------------ scanner */

typedef struct conf {
  char **lines;
  int n;
} conf_t;

static void conf_free(conf_t *c)
{
  int i;
  for (i = 0; i < c->n; i++) free(c->lines[i]);
  free(c->lines);
  c->lines = NULL;
  c->n = 0;
}

/* fgets with a 256-byte buffer, newline stripped (input.c:988-999) */
static int conf_read(const char *path, conf_t *c)
{
  FILE *fp = fopen(path, "r");
  char line[LINE_MAX_MBT];
  int cap = 0;
  c->lines = NULL;
  c->n = 0;
  if (!fp) return -1;
  while (fgets(line, LINE_MAX_MBT, fp) != NULL) {
    int len = (int) strlen(line);
    if (len > 0 && line[len - 1] == '\n') line[len - 1] = '\0';
    if (c->n == cap) {
      cap = cap ? 2 * cap : 256;
      c->lines = (char **) realloc(c->lines, cap * sizeof(char *));
    }
    c->lines[c->n++] = strdup(line);
  }
  fclose(fp);
  return 0;
}

/* 1: header of `name`, 0: header of another section, -1: not a header */
static int scan_section(const char *line, const char *name)
{
  unsigned i = 0, begin, end;
  if (line[0] == '#' || line[0] == ';') return -1;
  while (line[i] != '\0' && (line[i] == ' ' || line[i] == '\t')) i++;
  if (line[i] != '[') return -1;
  i++;
  begin = i;
  while (line[i] != '\0' && line[i] != ' ' && line[i] != '\t') i++;
  if (i < 1 || line[i - 1] != ']') return -1;
  end = i - 2;
  if (strlen(name) != end - begin + 1) return 0;
  return strncmp(line + begin, name, end - begin + 1) == 0 ? 1 : 0;
}

/* value text of `key` in this line, or NULL */
static const char *scan_key(const char *line, const char *key)
{
  unsigned i = 0, begin, end;
  while (line[i] != '\0' && (line[i] == ' ' || line[i] == '\t')) i++;
  if (line[i] == '#' || line[i] == ';') return NULL;
  begin = i;
  while (line[i] != '\0' && line[i] != ' ' && line[i] != '\t' && line[i] != ':' && line[i] != '=') i++;
  end = i - 1;
  while (line[i] != '\0' && (line[i] == ' ' || line[i] == '\t')) i++;
  if (line[i] != ':' && line[i] != '=') return NULL;
  i++;
  while (line[i] != '\0' && (line[i] == ' ' || line[i] == '\t')) i++;
  if (strlen(key) != end - begin + 1) return NULL;
  if (strncmp(line + begin, key, end - begin + 1) != 0) return NULL;
  return line + i;
}

static int have_section(const conf_t *c, const char *section)
{
  int i, count = 0;
  for (i = 0; i < c->n; i++)
    if (scan_section(c->lines[i], section) > 0) count++;
  return count == 1;
}

/* first match of key inside any block of `section` (config_get) */
static const char *get_raw(const conf_t *c, const char *section, const char *key)
{
  int i, in = 0;
  for (i = 0; i < c->n; i++) {
    int s = scan_section(c->lines[i], section);
    if (s == 0) in = 0;
    else if (s > 0) in = 1;
    else if (in) {
      const char *v = scan_key(c->lines[i], key);
      if (v != NULL) {
        /* config_scan succeeds for "%s" always and for numbers only when
           sscanf converts; a failed numeric scan keeps searching */
        return v;
      }
    }
  }
  return NULL;
}

static int get_int(const conf_t *c, const char *sec, const char *key, int *r)
{
  int i, in = 0;
  for (i = 0; i < c->n; i++) {
    int s = scan_section(c->lines[i], sec);
    if (s == 0) in = 0;
    else if (s > 0) in = 1;
    else if (in) {
      const char *v = scan_key(c->lines[i], key);
      if (v != NULL && sscanf(v, "%d", r) == 1) return 1;
    }
  }
  return 0;
}

static int get_long(const conf_t *c, const char *sec, const char *key, long *r)
{
  int v;
  if (!get_int(c, sec, key, &v)) return 0;
  *r = v;
  return 1;
}

static int get_double(const conf_t *c, const char *sec, const char *key, double *r)
{
  int i, in = 0;
  for (i = 0; i < c->n; i++) {
    int s = scan_section(c->lines[i], sec);
    if (s == 0) in = 0;
    else if (s > 0) in = 1;
    else if (in) {
      const char *v = scan_key(c->lines[i], key);
      if (v != NULL && sscanf(v, "%lf", r) == 1) return 1;
    }
  }
  return 0;
}

/* config_get_str (input.c:1093-1100) scans "%s": the first word */
static int get_str(const conf_t *c, const char *sec, const char *key, char *r, size_t cap)
{
  const char *v = get_raw(c, sec, key);
  size_t n = 0;
  if (!v) return 0;
  while (*v == ' ' || *v == '\t' || *v == '\n' || *v == '\r') v++;
  if (*v == '\0') return 0;
  while (v[n] != '\0' && v[n] != ' ' && v[n] != '\t' && v[n] != '\n' && v[n] != '\r' && n + 1 < cap) {
    r[n] = v[n];
    n++;
  }
  r[n] = '\0';
  return 1;
}

static char g_err[512];
static int cfg_fail(const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return MBT_ERR_CONFIG;
}

const char *mbt_config_error(void) { return g_err; }

#define REQ_I(sec, key, dst) do { if (!get_int(&C, sec, key, dst)) { r = cfg_fail("missing [%s] %s", sec, key); goto out; } } while (0)
#define REQ_L(sec, key, dst) do { if (!get_long(&C, sec, key, dst)) { r = cfg_fail("missing [%s] %s", sec, key); goto out; } } while (0)
#define REQ_D(sec, key, dst) do { if (!get_double(&C, sec, key, dst)) { r = cfg_fail("missing [%s] %s", sec, key); goto out; } } while (0)
#define REQ_S(sec, key, dst) do { if (!get_str(&C, sec, key, dst, sizeof(dst))) { r = cfg_fail("missing [%s] %s", sec, key); goto out; } } while (0)

static const char *const fillings[13] = {
  "UNIFORM", "ONETHIRD", "TWOTHIRD", "SINGLE", "SINGLE2", "SINGLE3", "THREEFOURTH",
  "ONEFOURTH", "SINGLE10", "SINGLE20", "SINGLE30", "EVENHALF", "EVENFOURTH"};

static int plane_of(const char *s)
{
  if (strcmp(s, "LON") == 0) return 0;
  if (strcmp(s, "HOR") == 0) return 1;
  if (strcmp(s, "VER") == 0) return 2;
  return -1;
}

/* Everything read_conf_file and the set-up functions produce. */
typedef struct cfg {
  mbt_params p;
  int filling;                   /* -1 = from file */
  char fill_file[4096];
  int enable_rw_short, enable_rw_short_lon, enable_diff_curr;
  double current_ratio;
  double rho0, Je, frf, emittanceH, couplbeta, U0, taue;
  double sgm[6];                 /* sgm_xtau, sgm_xeps, sgm_xx, sgm_xp, sgm_zz, sgm_zp (input units) */
  double cm[6];                  /* xtauCM, xepsCM, xxCM, xpCM, zzCM, zpCM */
  int nres;
  double res_Rs[MBT_MAX_RES], res_wr[MBT_MAX_RES], res_Q[MBT_MAX_RES];
  int res_plane[MBT_MAX_RES];
  int nwake;
  char wake_file[MBT_MAX_RES][1024];
  int wake_plane[MBT_MAX_RES];
  int lr_m[MBT_MAX_LR];
  double lr_detune[MBT_MAX_LR];
  int rffb_len_raw;
  int Nslc;
  int strong;                    /* BunchModel = STRONG (slice model) */
  int ngen[3];                   /* nGen_LON/HOR/VER */
  int fbii;                      /* EnableFBII */
  double q;                      /* ring->q = U0 / Vrf0 / 1e6 (input.c:1606) */
  mbt_output_cfg out;            /* output settings */
  int *bunch_out;                /* nharm: output buckets (setup_beam) */
} cfg_t;

static int read_conf(const char *path, int fix_rw_beff, int allow_strong, cfg_t *g)
{
  conf_t C;
  mbt_params *p = &g->p;
  char s[4096];
  int r = 0, i, enable_res = 1, tmp_i;
  double tmp;
  long ltmp;
  const char *ext = strrchr(path, '.');
  memset(g, 0, sizeof(*g));
  if (ext == NULL || strcmp(ext, ".conf") != 0)
    return cfg_fail("%s: only .conf input is supported", path);
  if (conf_read(path, &C) != 0) return cfg_fail("cannot open %s", path);

  /* defaults of read_input (input.c:164-180) */
  p->QH0 = 18.20; p->QV0 = 10.30;
  p->quantum = 1;
  g->filling = 5;   /* SINGLE3 */

  /* [tracking] */
  REQ_S("tracking", "jobtitle", s);
  snprintf(g->out.jobtitle, sizeof g->out.jobtitle, "%.79s", s);
  if (get_str(&C, "tracking", "filling", s, sizeof s)) {
    g->filling = -1;
    for (i = 0; i < 13; i++) if (strcmp(fillings[i], s) == 0) g->filling = i;
    if (g->filling < 0) snprintf(g->fill_file, sizeof g->fill_file, "%s", s);
  }
  REQ_S("tracking", "BunchModel", s);
  if (allow_strong && strcmp(s, "STRONG") == 0) g->strong = 1;
  else if (strcmp(s, "WEAK") != 0) {
    r = cfg_fail("BunchModel %s: only WEAK is supported here (STRONG through mbt_ws_config_load)", s);
    goto out;
  }
  REQ_I("tracking", "TrackPlane_LON", &p->track_plane[0]);
  if (p->track_plane[0] == 0) { r = cfg_fail("LON tracking switched off"); goto out; }
  REQ_I("tracking", "TrackPlane_HOR", &p->track_plane[1]);
  REQ_I("tracking", "TrackPlane_VER", &p->track_plane[2]);
  REQ_L("tracking", "NrevTot", &p->nrev_tot);
  REQ_L("tracking", "NrevMon", &p->nrev_mon);
  REQ_I("tracking", "EnableRW_short", &g->enable_rw_short);
  REQ_I("tracking", "EnableRW_long", &p->rw_long);
  REQ_I("tracking", "EnableFBII", &g->fbii);
  REQ_I("tracking", "EnableQuantum", &p->quantum);
  REQ_I("tracking", "EnableIdealHC", &p->ideal_hc);
  if (!get_int(&C, "tracking", "EnableRW_short_LON", &g->enable_rw_short_lon))
    g->enable_rw_short_lon = g->enable_rw_short;
  if (!get_long(&C, "tracking", "NrevPotentialsOut", &g->out.nrev_potentials_out)) g->out.nrev_potentials_out = 0;
  if (!get_int(&C, "tracking", "EnableAmpinv_out", &g->out.ampinv_out)) g->out.ampinv_out = 0;
  if (!get_int(&C, "tracking", "triggerRW", &p->triggerRW)) p->triggerRW = 0;
  if (!get_int(&C, "tracking", "Nmlt", &p->Nmlt) && p->rw_long) p->Nmlt = 0;
  if (!get_int(&C, "tracking", "EnableResonators", &enable_res)) enable_res = 1;
  if (get_int(&C, "tracking", "EnableDiffCurr", &g->enable_diff_curr)) {
    REQ_D("tracking", "current_ratio", &g->current_ratio);
    if (g->current_ratio < 0. || g->current_ratio > 1.) { r = cfg_fail("current_ratio not between 0 and 1"); goto out; }
  }

  /* [ring] */
  REQ_D("ring", "E0", &p->E0);
  REQ_D("ring", "Lc", &p->Lc);
  REQ_D("ring", "rho0", &g->rho0);
  REQ_D("ring", "betaH", &p->beta1[1]);
  REQ_D("ring", "betaV", &p->beta1[2]);
  REQ_D("ring", "dispH", &p->dispH1);
  REQ_D("ring", "alphaH", &p->alpha1[1]);
  REQ_D("ring", "alphaV", &p->alpha1[2]);
  REQ_D("ring", "disppH", &p->disppH1);
  REQ_D("ring", "ac", &p->ac);
  REQ_D("ring", "Je", &g->Je);
  REQ_D("ring", "Vrf0", &p->Vrf0);
  REQ_D("ring", "frf", &g->frf);
  REQ_D("ring", "Iring", &p->Iring);
  REQ_D("ring", "ApertureH", &tmp);
  REQ_D("ring", "ApertureV", &tmp);
  REQ_D("ring", "QH0", &p->QH0);
  REQ_D("ring", "QV0", &p->QV0);
  /* amplitude-dependent tune: a missing key resets CHH (input.c:414-417) */
  if (!get_double(&C, "ring", "CHH", &p->CHH)) p->CHH = 0;
  if (!get_double(&C, "ring", "CHV", &p->CHV)) p->CHH = 0;
  if (!get_double(&C, "ring", "CVH", &p->CVH)) p->CHH = 0;
  if (!get_double(&C, "ring", "CVV", &p->CVV)) p->CHH = 0;
  if (!get_int(&C, "ring", "mIdeal", &p->m_aHC)) p->m_aHC = 3;
  if (!get_double(&C, "ring", "Gzix", &p->Gzix)) {
    REQ_D("ring", "Cx", &tmp);
    p->Gzix = tmp / p->QH0;
  }
  if (!get_double(&C, "ring", "Gziz", &p->Gziz)) {
    REQ_D("ring", "Cz", &tmp);
    p->Gziz = tmp / p->QV0;
  }
  REQ_D("ring", "emittanceH", &g->emittanceH);
  if (!get_double(&C, "ring", "couplbeta", &g->couplbeta)) {
    REQ_D("ring", "emittanceV", &tmp);
    g->couplbeta = tmp / g->emittanceH;
  }
  if (g->enable_rw_short == 1 || p->rw_long == 1 || g->enable_rw_short_lon) {
    REQ_D("ring", "rhorw", &p->rhorw);
    REQ_D("ring", "beffL1", &p->beffL[0]);
    REQ_D("ring", "beffL2", &p->beffL[1]);
    if (g->enable_rw_short && p->track_plane[1]) {
      REQ_D("ring", "beffH3", &p->beffH[0]);
      REQ_D("ring", "beffH4", &p->beffH[1]);
    }
    if (g->enable_rw_short && p->track_plane[2]) {
      REQ_D("ring", "beffV3", &p->beffV[0]);
      REQ_D("ring", "beffV4", &p->beffV[1]);
    }
    if (fix_rw_beff && p->rw_long) {
      if (p->track_plane[1]) { get_double(&C, "ring", "beffH3", &p->beffH[0]); get_double(&C, "ring", "beffH4", &p->beffH[1]); }
      if (p->track_plane[2]) { get_double(&C, "ring", "beffV3", &p->beffV[0]); get_double(&C, "ring", "beffV4", &p->beffV[1]); }
    }
  }
  if (p->ideal_hc != 1) p->m_aHC = 1;
  g->U0 = -1.0;
  g->taue = -1.0;
  if (get_double(&C, "ring", "U0", &tmp)) g->U0 = tmp * FKILO;
  if (get_double(&C, "ring", "taue", &tmp)) g->taue = tmp * FMILLI;

  /* [distribution] */
  REQ_I("distribution", "Nslc", &g->Nslc);
  REQ_I("distribution", "Np", &p->np_model);
  if (get_int(&C, "distribution", "modeHT", &tmp_i)) { r = cfg_fail("modeHT (mode excitation) is not supported"); goto out; }
  {
    int ng[3];
    REQ_I("distribution", "nGen_LON", &ng[0]);
    REQ_I("distribution", "nGen_HOR", &ng[1]);
    REQ_I("distribution", "nGen_VER", &ng[2]);
    memcpy(g->ngen, ng, sizeof ng);
    for (i = 0; i < 3; i++)
      if (!ng[i] && p->track_plane[i]) { r = cfg_fail("distribution files (nGen = 0) are not supported"); goto out; }
  }
  {
    int seed = (int) time(NULL);
    if (!get_int(&C, "distribution", "iseed_LON", &p->iseed[0])) p->iseed[0] = seed;
    if (!get_int(&C, "distribution", "iseed_HOR", &p->iseed[1])) p->iseed[1] = seed;
    if (!get_int(&C, "distribution", "iseed_VER", &p->iseed[2])) p->iseed[2] = seed;
  }
  REQ_S("distribution", "gendst_datafile_LON", g->out.gendst_file[0]);
  REQ_S("distribution", "gendst_datafile_HOR", g->out.gendst_file[1]);
  REQ_S("distribution", "gendst_datafile_VER", g->out.gendst_file[2]);
  REQ_D("distribution", "xtauCM_offset", &g->cm[0]);
  REQ_D("distribution", "xepsCM_offset", &g->cm[1]);
  REQ_D("distribution", "sgm_xtau", &g->sgm[0]);
  REQ_D("distribution", "sgm_xeps", &g->sgm[1]);
  REQ_D("distribution", "xxCM_offset", &g->cm[2]);
  REQ_D("distribution", "xpCM_offset", &g->cm[3]);
  REQ_D("distribution", "sgm_xx", &g->sgm[2]);
  REQ_D("distribution", "sgm_xp", &g->sgm[3]);
  REQ_D("distribution", "zzCM_offset", &g->cm[4]);
  REQ_D("distribution", "zpCM_offset", &g->cm[5]);
  REQ_D("distribution", "sgm_zz", &g->sgm[4]);
  REQ_D("distribution", "sgm_zp", &g->sgm[5]);

  /* [resonator_N] */
  for (i = 1; ; i++) {
    char sec[32];
    snprintf(sec, sizeof sec, "resonator_%d", i);
    if (!have_section(&C, sec) || enable_res == 0) break;
    if (g->nres >= MBT_MAX_RES) { r = cfg_fail("more than %d resonators", MBT_MAX_RES); goto out; }
    REQ_D(sec, "Rs", &g->res_Rs[g->nres]);
    REQ_D(sec, "fres", &tmp);
    g->res_wr[g->nres] = (tmp * FGIGA) * 2.0 * M_PI;
    REQ_D(sec, "Qfactor", &g->res_Q[g->nres]);
    REQ_S(sec, "plane", s);
    if ((g->res_plane[g->nres] = plane_of(s)) < 0) { r = cfg_fail("[%s] bad plane %s", sec, s); goto out; }
    g->nres++;
  }
  /* [wake_file_N] */
  for (i = 1; ; i++) {
    char sec[32];
    snprintf(sec, sizeof sec, "wake_file_%d", i);
    if (!have_section(&C, sec)) break;
    if (g->nwake >= MBT_MAX_RES) { r = cfg_fail("more than %d wake files", MBT_MAX_RES); goto out; }
    REQ_S(sec, "filename", g->wake_file[g->nwake]);
    REQ_S(sec, "plane", s);
    if ((g->wake_plane[g->nwake] = plane_of(s)) < 0) { r = cfg_fail("[%s] bad plane %s", sec, s); goto out; }
    g->nwake++;
  }
  /* [harmonic_cavity_N]: longitudinal long-range resonators */
  for (i = 1; ; i++) {
    char sec[32];
    int l = p->n_lr[0];
    snprintf(sec, sizeof sec, "harmonic_cavity_%d", i);
    if (!have_section(&C, sec)) break;
    if (l >= MBT_MAX_LR) { r = cfg_fail("more than %d longitudinal long-range resonators", MBT_MAX_LR); goto out; }
    REQ_I(sec, "m", &g->lr_m[l]);
    REQ_D(sec, "Rs", &p->lr_Rs[0][l]);
    REQ_D(sec, "detune", &g->lr_detune[l]);
    REQ_D(sec, "Qfactor", &p->lr_Q[0][l]);
    p->n_lr[0]++;
  }
  /* [longrange_resonator_N]: appended after the harmonic cavities */
  for (i = 1; ; i++) {
    char sec[32];
    int pl, l;
    snprintf(sec, sizeof sec, "longrange_resonator_%d", i);
    if (!have_section(&C, sec)) break;
    REQ_S(sec, "plane", s);
    if ((pl = plane_of(s)) < 0) { r = cfg_fail("[%s] bad plane %s", sec, s); goto out; }
    l = p->n_lr[pl];
    if (l >= MBT_MAX_LR) { r = cfg_fail("more than %d long-range resonators in a plane", MBT_MAX_LR); goto out; }
    if (pl == 0) { g->lr_m[l] = 0; g->lr_detune[l] = 0; }
    REQ_D(sec, "fres", &tmp);
    p->lr_wr[pl][l] = (tmp * FGIGA) * 2.0 * M_PI;
    REQ_D(sec, "Rs", &p->lr_Rs[pl][l]);
    REQ_D(sec, "Qfactor", &p->lr_Q[pl][l]);
    p->n_lr[pl]++;
  }
  /* [rf_feedback] */
  if (have_section(&C, "rf_feedback")) {
    p->rffb = 1;
    REQ_I("rf_feedback", "resonator", &p->rffb_resonator);
    REQ_I("rf_feedback", "averaging_length", &g->rffb_len_raw);
    /* extension: the generator loop (mbt_params.rffb_gain / rffb_delay) */
    p->rffb_delay = 1;
    get_double(&C, "rf_feedback", "generator_gain", &p->rffb_gain);
    get_int(&C, "rf_feedback", "loop_delay", &p->rffb_delay);
    if (!(p->rffb_gain >= 0.0) || p->rffb_delay < 0 || p->rffb_delay > 1) {
      r = cfg_fail("[rf_feedback]: generator_gain must be >= 0 and loop_delay 0 or 1");
      goto out;
    }
  }
  /* [active_HC_N] */
  for (i = 1; ; i++) {
    char sec[32];
    int l = p->n_active_hc;
    snprintf(sec, sizeof sec, "active_HC_%d", i);
    if (!have_section(&C, sec)) break;
    if (l >= MBT_MAX_AHC) { r = cfg_fail("more than %d active harmonic cavities", MBT_MAX_AHC); goto out; }
    REQ_D(sec, "Vpeak", &p->ahc_vpeak[l]);
    REQ_D(sec, "nHC", &p->ahc_nhc[l]);
    REQ_D(sec, "phi_aHC", &p->ahc_phi[l]);
    p->n_active_hc++;
  }
  /* [selffield] */
  p->RsisL = 0.0;
  p->aindL = 0.0;
  get_double(&C, "selffield", "RsisL", &p->RsisL);
  if (get_double(&C, "selffield", "aindL", &tmp)) p->aindL = tmp / (2.0 * M_PI * FGIGA);
  {
    int lr_tot = p->n_lr[0] + p->n_lr[1] + p->n_lr[2];
    if (g->nres > 0 || g->enable_rw_short == 1 || lr_tot > 0 || g->nwake > 0 || g->enable_rw_short_lon) {
      if (!have_section(&C, "selffield")) { r = cfg_fail("missing [selffield]"); goto out; }
      REQ_D("selffield", "Nsigma", &p->nsigma);
      REQ_I("selffield", "Ncell", &p->ncell);
    } else {
      p->nsigma = 1.0;
      p->ncell = 0;
    }
  }
  /* [scan] */
  p->scan = 0;
  p->nscan = 1;
  p->nrev_scan = p->nrev_tot + 1;
  p->scan_start = 0.0;
  p->scan_step = 0.0;
  if (have_section(&C, "scan")) {
    REQ_I("scan", "scan_type", &p->scan);
    if (p->scan != 0) {
      REQ_L("scan", "Nscan", &p->nscan);
      REQ_L("scan", "NrevScan", &p->nrev_scan);
      if (p->scan == 1) { REQ_D("scan", "scan_start", &p->scan_start); REQ_D("scan", "scan_step", &p->scan_step); }
      if (p->scan == 4) REQ_D("scan", "scan_start", &p->scan_start);
      p->nrev_tot = p->nscan * p->nrev_scan;
    }
  }
  /* the reference takes any integer type (and steps only type 1) and
     divides by NrevScan every turn */
  if (p->scan < 0 || p->scan > 4) { r = cfg_fail("[scan] scan_type %d is not 0..4", p->scan); goto out; }
  if (p->scan != 0 && (p->nscan < 1 || p->nrev_scan < 1)) { r = cfg_fail("[scan] Nscan and NrevScan must be positive"); goto out; }
  (void) ltmp;
out:
  conf_free(&C);
  return r;
}

/* setup_ring_parameters, input.c:1553-1695 */
static int setup_ring(cfg_t *g)
{
  mbt_params *p = &g->p;
  const double Cg = 8.85e-05;
  double R, Gamma, tauC, q, Vrfp, wso, h;
  int i;
  unsigned Ntmp = 0, Nbumax;
  double vb = 0, genphase = 0, genphase_harm = 0, eloss_harm = 0;
  R = p->Lc / (2.0 * M_PI);
  Gamma = 1957.0 * p->E0;
  (void) Gamma;
  p->wrf = 2.0 * M_PI * g->frf * FMEGA;
  h = (int) (g->frf * FMEGA * p->Lc / C_LIGHT + 0.5);
  p->nharm = (int) h;
  p->T0 = p->nharm / g->frf / FMEGA;
  p->amp_dep_qv = (p->CVH != 0.0) || (p->CVV != 0.0);
  if (g->U0 >= 0 && g->taue >= 0) {
    p->Urad = g->U0 / (p->E0 * FGIGA);
    if (p->Urad != 0) {
      if (g->Je < 0) g->Je = 2 * p->T0 / (g->taue * p->Urad);
      if (g->rho0 < 0) g->rho0 = Cg * p->E0 * p->E0 * p->E0 * p->E0 * FGIGA / g->U0;
    }
    p->De = 2 * p->T0 / (g->taue);
    tauC = g->Je * g->taue;
    p->taue = g->taue;
  } else {
    g->U0 = Cg * p->E0 * p->E0 * p->E0 * p->E0 * FGIGA / g->rho0;
    p->Urad = g->U0 / (p->E0 * FGIGA);
    tauC = 4.0 * M_PI * R * g->rho0 / (Cg * C_LIGHT) / pow(p->E0, 3);
    p->taue = tauC / g->Je;
    p->De = 2.0 * (1.0 / p->taue) * p->T0;
  }
  q = g->U0 / p->Vrf0 / FMEGA;
  g->q = q;
  Vrfp = FMEGA * p->Vrf0 * p->wrf * sqrt(1.0 - q * q);
  wso = sqrt(fabs(p->ac) * Vrfp / (p->T0 * p->E0 * FGIGA));
  p->phai0 = asin(q);
  /* transverse damping */
  {
    const double Jz = 1.0, Jx = 4.0 - Jz - g->Je;
    p->taux = tauC / Jx;
    p->tauz = tauC / Jz;
  }
  p->gamma1[1] = (1.0 + p->alpha1[1] * p->alpha1[1]) / p->beta1[1];
  p->gamma1[2] = (1.0 + p->alpha1[2] * p->alpha1[2]) / p->beta1[2];
  for (i = 0; i < p->n_lr[0]; i++) {
    double tmp;
    unsigned Nturn, Nbu;
    if (g->lr_m[i] > 0) {
      p->lr_wr[0][i] = g->lr_m[i] * p->wrf + g->lr_detune[i] * 2 * M_PI;
      if (g->lr_m[i] > 1) {
        genphase_harm = cos(atan(p->lr_Q[0][i] * (p->lr_wr[0][i] / (p->wrf * g->lr_m[i]) - (p->wrf * g->lr_m[i]) / p->lr_wr[0][i])));
        eloss_harm += 2 * p->Iring * p->lr_Rs[0][i] * genphase_harm * genphase_harm * FMILLI / FMEGA;
      } else {
        genphase = atan(p->lr_Q[0][i] * (p->lr_wr[0][i] / p->wrf - p->wrf / p->lr_wr[0][i]));
        vb = 2 * p->Iring * p->lr_Rs[0][i] * cos(genphase) * FMILLI / FMEGA;
      }
    }
    tmp = (p->lr_wr[0][i] * 0.5 / p->lr_Q[0][i]);
    Nturn = (unsigned) (log(2) * 10 / tmp / p->T0) + 1;
    Nbu = Nturn * (unsigned) h;
    if (Nbu < 2) return cfg_fail("long-range resonator %d is short-range", i + 1);
    if (Nbu > Ntmp) Ntmp = Nbu;
  }
  p->phai0 = asin(q + eloss_harm / p->Vrf0);
  Nbumax = Ntmp;
  if (p->rffb) {
    p->rffb_vrf_design = 1 * p->Vrf0;
    p->rffb_phi0_design = p->ac < 0 ? M_PI - p->phai0 : 1 * p->phai0;
    p->Vrf0 = sqrt(vb * vb + p->rffb_vrf_design * p->rffb_vrf_design + 2 * vb * p->rffb_vrf_design * sin(genphase + p->rffb_phi0_design));
    p->phai0 = asin(vb / p->Vrf0 * sin(M_PI / 2 + p->rffb_phi0_design + genphase)) + p->rffb_phi0_design;
    if (g->rffb_len_raw == -1) p->rffb = 0;
    else if (fabs(g->rffb_len_raw) > Nbumax) Nbumax = (unsigned) fabs(g->rffb_len_raw);
  } else {
    p->phai0 += asin(vb / p->Vrf0 * cos(p->phai0 + genphase));
  }
  if (p->ac < 0) p->phai0 = M_PI - p->phai0;
  p->lr_init_turns = (int) (Nbumax / h);
  p->rffb_len = g->rffb_len_raw < 0 ? -g->rffb_len_raw : g->rffb_len_raw;
  p->rffb_off_after_init = g->rffb_len_raw < 0;
  /* macrop_model_setup_parameters, input.c:1775-1831 */
  {
    const double Cq = 3.84e-13;
    double *sg = g->sgm;
    const double Gamma2 = (1957.0 * p->E0) * (1957.0 * p->E0);
    double corr_xpx, corr_zpz;
    if (sg[1] < 0.0) sg[1] = sqrt(Cq * Gamma2 / (g->Je * g->rho0));
    if (sg[0] < 0.0) sg[0] = FGIGA * fabs(p->ac) / wso * sg[1];
    if (sg[2] < 0.0) sg[2] = FKILO * sqrt(g->emittanceH / FGIGA * p->beta1[1]);
    if (sg[3] < 0.0) { sg[3] = FKILO * sqrt(g->emittanceH / FGIGA / p->beta1[1]); corr_xpx = -p->alpha1[1] / p->beta1[1]; }
    else corr_xpx = 0.0;
    if (sg[4] < 0.0) sg[4] = FKILO * sqrt(g->emittanceH / FGIGA * p->beta1[2] * g->couplbeta);
    if (sg[5] < 0.0) { sg[5] = FKILO * sqrt(g->emittanceH / FGIGA / p->beta1[2] * g->couplbeta); corr_zpz = -p->alpha1[2] / p->beta1[2]; }
    else corr_zpz = 0.0;
    p->pos_offset[0] = g->cm[0] * FNANO;
    p->pos_offset[1] = g->cm[2] * FMILLI;
    p->pos_offset[2] = g->cm[4] * FMILLI;
    p->slope_offset[0] = g->cm[1];
    p->slope_offset[1] = g->cm[3] * FMILLI;
    p->slope_offset[2] = g->cm[5] * FMILLI;
    p->pos_sgm[0] = sg[0] * FNANO;
    p->pos_sgm[1] = sg[2] * FMILLI;
    p->pos_sgm[2] = sg[4] * FMILLI;
    p->slope_sgm[0] = sg[1];
    p->slope_sgm[1] = sg[3] * FMILLI;
    p->slope_sgm[2] = sg[5] * FMILLI;
    p->correlate[0] = 0.0;
    p->correlate[1] = corr_xpx;
    p->correlate[2] = corr_zpz;
  }
  /* selffield_model_init, transform_weak.c:227-228 */
  if (p->ncell > 0) {
    p->dT = 2.0 * p->nsigma / ((double) p->ncell - 1);
    p->sigma_tau = p->pos_sgm[0];
  }
  return 0;
}

/* setup_tracking_parameters, input.c:1698-1772 */
static int setup_tracking(cfg_t *g)
{
  mbt_params *p = &g->p;
  double b;
  if (p->ideal_hc == 1) {
    const double q = g->q;
    double m2 = (double) p->m_aHC * p->m_aHC;
    p->phai0 = asin(p->m_aHC * p->m_aHC / (m2 - 1.) * q);
    p->phi_n = atan(tan(p->phai0) / (double) p->m_aHC) / (double) p->m_aHC;
    if (p->ac < 0) {
      p->phai0 = M_PI - p->phai0;
      p->phi_n = M_PI - p->phi_n;
    }
    p->HC_k = -cos(p->phai0) / (p->m_aHC * cos(p->m_aHC * p->phi_n));
  }
  if (p->scan == 1) p->Iring = p->scan_start;
  if (p->scan == 3 || p->scan == 4) {
    int i;
    if (p->n_lr[0] < 1) return cfg_fail("Qfactor scan but no longrange resonator given");
    if (p->scan == 3) {
      p->scan_start = 1. / p->nscan;
      p->scan_step = 1. / p->nscan;
      for (i = 0; i < p->n_lr[0]; i++) p->lr_Q[0][i] = p->lr_Q[0][i] / p->nscan;
    } else {
      p->scan_step = (1. - p->scan_start) / (p->nscan - 1);
      for (i = 0; i < p->n_lr[0]; i++) p->lr_Q[0][i] = p->lr_Q[0][i] * p->scan_start;
    }
  }
  b = p->beffL[1];
  if (p->beffH[1] > b && p->track_plane[1] == 1) b = p->beffH[1];
  else if (p->beffV[1] > b && p->track_plane[2] == 1) b = p->beffV[1];
  if (g->enable_rw_short || g->enable_rw_short_lon) {
    /* input.c:1744-1756: the short-range wake needs bins of >= 20 s0 */
    const double s0 = pow((2 * b * b * p->rhorw / Z_0), 1.0 / 3.0);
    const double dT = 2.0 * p->nsigma / ((double) p->ncell - 1);
    const double mult = dT * p->pos_sgm[0] * C_LIGHT / s0;
    if (mult < 20.)
      return cfg_fail("Selffield Model has too small binwidth for RW treatment (bin = %.3g s0, needs 20)", mult);
  }
  if (p->rw_long && p->Nmlt == 0) {
    double tmp = p->Lc * sqrt(p->rhorw) / pow(b, 3);
    p->Nmlt = 1 + ((int) 500e3 / tmp);
    if (p->Nmlt == 0) p->rw_long = 0;
  }
  return 0;
}

/* e_beam_setup / e_beam_fileread, input.c:1289-1512 */
static int setup_beam(cfg_t *g, int *nbunch, int *bucket, double *ib_frac)
{
  const int H = g->p.nharm;
  int *fill = (int *) calloc(H, sizeof(int));
  double *ratio = (double *) calloc(H, sizeof(double));
  int kb, nb = 0, r = 0;
  if (g->filling == -1) {
    FILE *f = fopen(g->fill_file, "r");
    int nb_tmp, bout_tmp;
    double crat_tmp, crat_tot = 0.0;
    if (!f) { free(fill); free(ratio); return cfg_fail("%s is not a valid filename or filling pattern", g->fill_file); }
    for (kb = 0; kb < H; kb++) {
      if (fscanf(f, "%d %lf %d\n", &nb_tmp, &crat_tmp, &bout_tmp) != 3) break;
      if (nb_tmp >= H) break;
      while (nb_tmp > kb) { ratio[kb] = 0; kb++; }
      if (crat_tmp > 0) {
        fill[kb] = 1; ratio[kb] = crat_tmp; crat_tot += crat_tmp; nb++;
        if (bout_tmp && g->bunch_out) g->bunch_out[g->out.n_out++] = kb;
      }
      else ratio[kb] = 0.0;
    }
    fclose(f);
    {
      double crat_mean = crat_tot / nb;
      int n = 0;
      for (kb = 0; kb < H; kb++)
        if (ratio[kb] > 0) {
          if (bucket) bucket[n] = kb;
          if (ib_frac) ib_frac[n] = ratio[kb] / crat_mean;
          n++;
        }
    }
  } else {
    /* output buckets of each named filling (input.c:1316-1426) */
    int bo[3] = {0, 0, 0}, nbo = 1;
    switch (g->filling) {
      case 7: nbo = 3; bo[1] = H / 8; bo[2] = H / 4 - 1; break;
      case 1: nbo = 3; bo[1] = H / 6; bo[2] = H / 3 - 1; break;
      case 2: nbo = 3; bo[1] = H / 3; bo[2] = 2 * H / 3 - 1; break;
      case 6: nbo = 3; bo[1] = 3 * H / 8; bo[2] = 3 * H / 4 - 1; break;
      case 4: nbo = 2; bo[1] = 1; break;
      case 5: nbo = 3; bo[1] = 1; bo[2] = 2; break;
      case 8: nbo = 3; bo[1] = 4; bo[2] = 9; break;
      case 9: nbo = 3; bo[1] = 9; bo[2] = 19; break;
      case 10: nbo = 3; bo[1] = 14; bo[2] = 29; break;
      default: break;
    }
    if (g->bunch_out) {
      for (kb = 0; kb < nbo; kb++) g->bunch_out[kb] = bo[kb];
      g->out.n_out = nbo;
    }
    switch (g->filling) {
      case 0: for (kb = 0; kb < H; kb++) fill[kb] = 1; break;
      case 7: for (kb = 0; kb < H / 4; kb++) fill[kb] = 1; break;
      case 1: for (kb = 0; kb < H / 3; kb++) fill[kb] = 1; break;
      case 2: for (kb = 0; kb < 2 * H / 3; kb++) fill[kb] = 1; break;
      case 6: for (kb = 0; kb < 3 * H / 4; kb++) fill[kb] = 1; break;
      case 3: fill[0] = 1; break;
      case 4: for (kb = 0; kb < 2; kb++) fill[kb] = 1; break;
      case 5: for (kb = 0; kb < 3; kb++) fill[kb] = 1; break;
      case 8: for (kb = 0; kb < 10; kb++) fill[kb] = 1; break;
      case 9: for (kb = 0; kb < 20; kb++) fill[kb] = 1; break;
      case 10: for (kb = 0; kb < 30; kb++) fill[kb] = 1; break;
      case 11: for (kb = 0; kb < H / 2; kb++) fill[2 * kb] = 1; break;
      case 12: for (kb = 0; kb < H / 4; kb++) fill[4 * kb] = 1; break;
      default: r = cfg_fail("unknown filling"); break;
    }
    for (kb = 0; kb < H; kb++) {
      if (!fill[kb]) continue;
      if (bucket) bucket[nb] = kb;
      if (ib_frac) {
        if (g->enable_diff_curr) ib_frac[nb] = (nb % 2 == 0) ? g->current_ratio : 2.0 - g->current_ratio;
        else ib_frac[nb] = 1.0;
      }
      nb++;
    }
  }
  *nbunch = nb;
  free(fill);
  free(ratio);
  return r;
}

int mbt_config_load(const char *conf_path, int fix_rw_beff, mbt_params *p, int *nbunch, int *bucket,
                    double *ib_frac)
{
  cfg_t *g;
  int r, nb = 0;
  if (!conf_path || !p) return MBT_ERR_INVALID;
  g = (cfg_t *) calloc(1, sizeof(cfg_t));
  if (!g) return MBT_ERR_NOMEM;
  r = read_conf(conf_path, fix_rw_beff, 0, g);
  if (!r) r = setup_ring(g);
  if (!r) r = setup_tracking(g);
  if (!r) r = setup_beam(g, &nb, bucket, ib_frac);
  if (!r) {
    *p = g->p;
    if (nbunch) *nbunch = nb;
  }
  free(g);
  return r;
}

/* ---- slice model (BunchModel = STRONG) ------------------------------- */

#define WS_E_CHARGE 1.602e-19
#define WS_E_MASS   9.1e-31
#define WS_MP_O_EM  1.836e3

/* fbii_grid_setup_parameters bunch.c:811-851, fbii_model_init
   fbi_weakstrong.c:18-43, worker_weakstrong.c:67-68 */
static int ws_derive(const cfg_t *g, mbt_ws_params *w)
{
  double Pave, Pu20, Pm, dm, sigmam, Lu20;
  memset(w, 0, sizeof(*w));
  w->base = g->p;
  w->nslc = g->Nslc;
  w->fbii = g->fbii;
  w->np = g->p.np_model;
  w->ngrid = 5;
  w->ndivs = 3;
  w->sgm_xx = g->sgm[2];
  w->sgm_zz = g->sgm[4];
  w->sgmatau = g->sgm[0] / FGIGA;
  w->max_tau = 7.0;
  w->dtau = 0.3;
  if (w->nslc < 0 || 2 * w->nslc + 1 > 49)
    return cfg_fail("Nslc %d: 2 Nslc + 1 slices must be 1..49", w->nslc);
  if (w->np < 2) return cfg_fail("Np %d: the slicing needs at least 2 macroparticles", w->np);
  if (!(w->sgm_zz < w->sgm_xx) || !(w->sgm_zz > 0.0))
    return cfg_fail("sgm_zz %g, sgm_xx %g: the slice field needs 0 < sgm_zz < sgm_xx", w->sgm_zz, w->sgm_xx);
  if (!g->p.track_plane[1] || !g->p.track_plane[2])
    return cfg_fail("the slice model needs both transverse planes tracked");
  if (!g->ngen[0] || !g->ngen[1] || !g->ngen[2])
    return cfg_fail("the slice model generates all three planes: nGen_LON/HOR/VER must be nonzero");
  memcpy(w->sgm_in, g->sgm, sizeof w->sgm_in);
  memcpy(w->cm_in, g->cm, sizeof w->cm_in);
  w->agLOCz = w->sgm_zz / ((double) w->ndivs) / FKILO;
  w->agLOCx = w->sgm_xx / ((double) w->ndivs) / FKILO;
  w->agABSz = 2.0 * w->agLOCz;
  w->agABSx = 2.0 * w->agLOCx;
  w->deltT = w->dtau * w->sgmatau;
  w->factBE = sqrt(2 * (w->sgm_xx * w->sgm_xx - w->sgm_zz * w->sgm_zz)) / FKILO;
  Pave = 2.7e-9;
  Pu20 = 5 * Pave;
  Pm = 0.15 * Pu20 / 1.3332;
  dm = 3.22e22 * Pm;
  sigmam = 1.78;
  Lu20 = 354.0;
  w->Ldmsgm = Lu20 * dm * sigmam * 1e-22;
  w->factF = WS_E_CHARGE / (28.0 * WS_MP_O_EM * WS_E_MASS);
  w->Gamma = 1957.0 * g->p.E0;
  w->kick_factor = 1e+2;
  return 0;
}

int mbt_ws_config_load(const char *conf_path, int fix_rw_beff, mbt_ws_params *w, int *nbunch, int *bucket,
                       double *ib_frac)
{
  cfg_t *g;
  int r, nb = 0;
  if (!conf_path || !w) return MBT_ERR_INVALID;
  g = (cfg_t *) calloc(1, sizeof(cfg_t));
  if (!g) return MBT_ERR_NOMEM;
  r = read_conf(conf_path, fix_rw_beff, 1, g);
  if (!r && !g->strong) r = cfg_fail("%s: BunchModel is not STRONG (use mbt_config_load)", conf_path);
  if (!r) r = setup_ring(g);
  if (!r) r = setup_tracking(g);
  if (!r) r = setup_beam(g, &nb, bucket, ib_frac);
  if (!r) r = ws_derive(g, w);
  if (!r && nbunch) *nbunch = nb;
  free(g);
  return r;
}

size_t mbt_ws_params_size(void) { return sizeof(mbt_ws_params); }

int mbt_config_bunch_model(const char *conf_path)
{
  conf_t C;
  char s[64];
  int r;
  if (!conf_path) return MBT_ERR_INVALID;
  if (conf_read(conf_path, &C) != 0) return cfg_fail("cannot open %s", conf_path);
  if (!get_str(&C, "tracking", "BunchModel", s, sizeof s)) r = cfg_fail("missing [tracking] BunchModel");
  else if (strcmp(s, "WEAK") == 0) r = 0;
  else if (strcmp(s, "STRONG") == 0) r = 1;
  else r = cfg_fail("BunchModel %s: WEAK or STRONG", s);
  conf_free(&C);
  return r;
}

/* strong_generate_eCMs bunch_strong.c:117-198 */
int mbt_ws_slice_beam(const mbt_ws_params *w, const double *soa6, int np, int *npop, int *nofe, double *cm4)
{
  int S, G, off, jp, c, k;
  int *cell, *cnt;
  double *sum;
  if (!w || !soa6 || np < 1 || !npop || !nofe || !cm4) return MBT_ERR_INVALID;
  S = 2 * w->nslc + 1;
  G = w->ngrid;
  off = (G - 1) / 2;
  if (S < 1 || G < 1 || !(w->sgmatau > 0.0) || !(w->dtau > 0.0)) return MBT_ERR_INVALID;
  cell = (int *) malloc((size_t) np * sizeof(int));
  cnt = (int *) calloc((size_t) S + 1, sizeof(int));
  sum = (double *) calloc(4 * ((size_t) S + 1), sizeof(double));
  if (!cell || !cnt || !sum) { free(cell); free(cnt); free(sum); return MBT_ERR_NOMEM; }
  {
    const double *t0 = soa6, *x = soa6 + np, *z = soa6 + 2 * (size_t) np;
    const double *xp = soa6 + 4 * (size_t) np, *zp = soa6 + 5 * (size_t) np;
    /* slice index of each particle, counts and coordinate sums in
       particle order (the overflow cell S collects the tail) */
    for (jp = 0; jp < np; jp++) {
      const double u = (w->max_tau + (-t0[jp] / w->sgmatau)) / w->dtau;
      int ic = !(u >= 1.0) ? 0 : (u >= (double) S ? S : (int) u);
      double *sc = sum + ic;
      cell[jp] = ic;
      cnt[ic]++;
      sc[0] = sc[0] + x[jp];
      sc[S + 1] = sc[S + 1] + xp[jp];
      sc[2 * (S + 1)] = sc[2 * (S + 1)] + z[jp];
      sc[3 * (S + 1)] = sc[3 * (S + 1)] + zp[jp];
    }
    for (c = 0; c < S; c++) {
      npop[c] = cnt[c];
      for (k = 0; k < 4; k++) {
        const double v = sum[k * (S + 1) + c];
        cm4[k * S + c] = cnt[c] ? v / cnt[c] : v;
      }
    }
    /* offsets from the slice centroid in half local steps, rounded half
       away from zero, clamped to the grid */
    memset(nofe, 0, (size_t) S * G * G * sizeof(int));
    for (jp = 0; jp < np; jp++) {
      const int ic = cell[jp];
      double ux, uz;
      int mx, mz;
      if (ic >= S) continue;
      ux = 2.0 * (x[jp] - cm4[ic]) / w->agLOCx;
      uz = 2.0 * (z[jp] - cm4[2 * S + ic]) / w->agLOCz;
      ux = ux > 1e6 ? 1e6 : (ux < -1e6 ? -1e6 : ux);
      uz = uz > 1e6 ? 1e6 : (uz < -1e6 ? -1e6 : uz);
      mx = (int) ux;
      mz = (int) uz;
      mx = mx >= 0 ? (mx + 1) / 2 : (mx - 1) / 2;
      mz = mz >= 0 ? (mz + 1) / 2 : (mz - 1) / 2;
      mx = mx > off ? off : (mx < -off ? -off : mx);
      mz = mz > off ? off : (mz < -off ? -off : mz);
      nofe[(ic * G + mx + off) * G + mz + off]++;
    }
  }
  free(cell); free(cnt); free(sum);
  return 0;
}

int mbt_config_output(const char *conf_path, mbt_output_cfg *o, int *bunch_out)
{
  cfg_t *g;
  int r, nb = 0;
  if (!conf_path || !o) return MBT_ERR_INVALID;
  g = (cfg_t *) calloc(1, sizeof(cfg_t));
  if (!g) return MBT_ERR_NOMEM;
  r = read_conf(conf_path, 1, 1, g);
  if (!r) r = setup_ring(g);
  if (!r) r = setup_tracking(g);
  if (!r) {
    g->bunch_out = (int *) calloc(g->p.nharm > 0 ? g->p.nharm : 1, sizeof(int));
    if (!g->bunch_out) r = MBT_ERR_NOMEM;
  }
  if (!r) r = setup_beam(g, &nb, NULL, NULL);
  if (!r) {
    *o = g->out;
    if (bunch_out) memcpy(bunch_out, g->bunch_out, (size_t) g->out.n_out * sizeof(int));
  }
  free(g->bunch_out);
  free(g);
  return r;
}

/* [beam_ion]: the stage of mbt_enable_beam_ion (no reference section; the
 * defaults are the reference's CO model, fbi_weakstrong.c:18-43, with the
 * gas spread over the whole ring) */
int mbt_config_beam_ion(const char *conf_path, mbt_beam_ion *bi)
{
  conf_t C;
  double tmp;
  int r = 0, itmp;
  if (!conf_path || !bi) return MBT_ERR_INVALID;
  if (conf_read(conf_path, &C) != 0) return cfg_fail("cannot open %s", conf_path);
  if (!have_section(&C, "beam_ion")) { conf_free(&C); return 1; }
  memset(bi, 0, sizeof(*bi));
  bi->n_ip = 1;
  bi->ions_per_passage = 1000;
  bi->gas_A = 28.0;
  bi->pressure = 1.0e-9;
  bi->sigma_ion = 1.78e-22;
  bi->seed = 1;
  bi->audit_fraction = 0.01;
  if (get_int(&C, "beam_ion", "n_ip", &itmp)) bi->n_ip = itmp;
  if (get_int(&C, "beam_ion", "ions_per_passage", &itmp)) bi->ions_per_passage = itmp;
  if (get_double(&C, "beam_ion", "gas_A", &tmp)) bi->gas_A = tmp;
  if (get_double(&C, "beam_ion", "pressure_nTorr", &tmp)) bi->pressure = tmp * FNANO;
  if (get_double(&C, "beam_ion", "sigma_ion_Mb", &tmp)) bi->sigma_ion = tmp * 1.0e-22;
  if (get_int(&C, "beam_ion", "seed", &itmp)) bi->seed = (uint64_t) (uint32_t) itmp;
  if (get_int(&C, "beam_ion", "surrogate", &itmp)) bi->surrogate = itmp;
  if (get_double(&C, "beam_ion", "audit_fraction", &tmp)) bi->audit_fraction = tmp;
  if (bi->n_ip < 1 || bi->ions_per_passage < 1 || !(bi->gas_A > 0) || bi->pressure < 0 || bi->sigma_ion < 0)
    r = cfg_fail("[beam_ion]: n_ip, ions_per_passage, gas_A must be positive");
  conf_free(&C);
  return r;
}

double mbt_bunch_current(const mbt_params *p, int nbunch, double ib_frac)
{
  /* manager_weakweak.c:74-75 */
  return ib_frac * p->Iring / (((double) nbunch) * FKILO);
}

/* Wake file interpolation, construct_greensfunc_file transform_weak.c:405-471 */
static int greens_file(const char *fname, int plane, mbt_params *p, double *Gl, double *Gv, double *Gh)
{
  const double dTau = p->sigma_tau * p->dT;
  const int Nc = p->ncell;
  FILE *wp = fopen(fname, "r");
  double *Gtmp, t = 0, w = 0, last_t = 0, last_w = 0;
  int i, k, last_i = -1, eof = 0;
  if (!wp) return cfg_fail("cannot open wake file %s", fname);
  Gtmp = (double *) calloc(Nc, sizeof(double));
  do {
    if (fscanf(wp, "%lf%lf", &t, &w) != 2) break;
  } while (t < 0);
  Gtmp[0] = 0;
  for (i = 0; i < Nc; i++) {
    if (eof) Gtmp[i] = Gtmp[i - 1];
    while (t <= i * dTau) {
      last_t = 1 * t;
      last_w = 1 * w;
      if (fscanf(wp, "%lf %lf\n", &t, &w) != 2) { eof = 1; break; }
    }
    while (t > (i + 1) * dTau) i++;
    for (k = last_i + 1; k < i + 1 && k < Nc; k++)
      Gtmp[k] = (w * (k * dTau - last_t) + last_w * (t - k * dTau)) / (t - last_t);
    if (i > last_i + 1) i--;
    last_i = 1 * i;
  }
  fclose(wp);
  if (plane == 0) {
    Gtmp[0] = Gtmp[0] / 2.;
    for (i = 0; i < Nc; i++) Gl[i] += Gtmp[i];
    p->planeL++;
  } else if (plane == 1) {
    for (i = 0; i < Nc; i++) Gh[i] += Gtmp[i];
    p->planeH++;
  } else {
    for (i = 0; i < Nc; i++) Gv[i] += Gtmp[i];
    p->planeV++;
  }
  free(Gtmp);
  return 0;
}

/* ---------------------------------------- short-range resistive wall */

/* Gauss-Legendre nodes and weights on [-1, 1] (Newton iteration on the
 * Legendre recurrence (j+1) P_{j+1} = (2j+1) x P_j - j P_{j-1}). */
static void gl_rule(int n, double *x, double *w)
{
  int i, j;
  for (i = 0; i < (n + 1) / 2; i++) {
    double z = cos(M_PI * (i + 0.75) / (n + 0.5)), dz = 1.0, p1 = 1.0, p2 = 0.0, dp = 1.0;
    int it;
    for (it = 0; it < 100 && fabs(dz) > 1e-16; it++) {
      p1 = 1.0;
      p2 = 0.0;
      for (j = 1; j <= n; j++) {
        const double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      dp = n * (z * p1 - p2) / (z * z - 1.0);
      dz = p1 / dp;
      z -= dz;
    }
    x[i] = -z;
    x[n - 1 - i] = z;
    w[i] = w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}

typedef double (*integrand_t)(double t, double u);

static double gl_panel(integrand_t f, double u, double a, double b, int n, const double *x, const double *w)
{
  const double c = 0.5 * (a + b), h = 0.5 * (b - a);
  double s = 0.0;
  int i;
  for (i = 0; i < n; i++) s += w[i] * f(c + h * x[i], u);
  return s * h;
}

/* Adaptive Gauss-Legendre: a panel is accepted when the 12- and 24-point
 * rules agree to tol (absolute, the same for every panel), else halved;
 * at most 2^20 panels per call. */
static double integrate(integrand_t f, double u, double a, double b, double tol, int depth)
{
  static double x12[12], w12[12], x24[24], w24[24];
  static int ready = 0;
  double i12, i24;
  if (!ready) {
    gl_rule(12, x12, w12);
    gl_rule(24, x24, w24);
    ready = 1;
  }
  i12 = gl_panel(f, u, a, b, 12, x12, w12);
  i24 = gl_panel(f, u, a, b, 24, x24, w24);
  if (fabs(i24 - i12) <= tol || depth >= 20) return i24;
  return integrate(f, u, a, 0.5 * (a + b), tol, depth + 1) + integrate(f, u, 0.5 * (a + b), b, tol, depth + 1);
}

/* exp(-t^2 u) / (t^6 + 8) */
static double rw_k(double t, double u) { return exp(-t * t * u) / (pow(t, 6) + 8.0); }

/* (1 - exp(-t^2 u)) / (t^2 (t^6 + 8)); u / 8 at t = 0 */
static double rw_j(double t, double u)
{
  const double y = t * t * u;
  const double q = y < 1e-8 ? u * (1.0 - 0.5 * y) : -expm1(-y) / (t * t);
  return q / (pow(t, 6) + 8.0);
}

/* the same after t = 1/s, for t in [1, inf): s^6 (1 - exp(-u/s^2)) / (1 + 8 s^6) */
static double rw_j_tail(double s, double u)
{
  if (s <= 0.0) return 0.0;
  return pow(s, 6) * -expm1(-u / (s * s)) / (1.0 + 8.0 * pow(s, 6));
}

/* Bin averages over [0, u s0] of the Bane-Sands short-range resistive-wall
 * wakes of a round pipe (K. Bane and M. Sands, "The short-range resistive
 * wall wakefields", SLAC-PUB-95-7074), in units of s0 = (2 b^2 rho /
 * Z0)^(1/3):
 *   w(x)  = e^-x cos(sqrt3 x) / 3 - sqrt2/pi int_0^inf t^2 e^(-t^2 x) / (t^6+8) dt
 *           (longitudinal, times 4 Z0 c / (pi b^2)),
 *   W(x)  = int_0^x w      (transverse, times 8 Z0 c s0 / (pi b^4)),
 *   lon   = (1/u) int_0^u w = [e^-u (sqrt3 sin - cos)(sqrt3 u) / 12
 *                              + sqrt2/pi int e^(-t^2 u) / (t^6+8) dt] / u,
 *   trans = (1/u) int_0^u W = [(sqrt3 Fs - Fc) / 12
 *                              + sqrt2/pi int (1 - e^(-t^2 u)) / (t^2 (t^6+8)) dt] / u,
 * with Fc, Fs = int_0^u e^-x cos, sin(sqrt3 x) dx; the terms growing like u
 * cancel analytically (int_0^inf dt / (t^6+8) = pi / (12 sqrt2)).  These
 * are the quantities the reference tabulates for u in [19.8, 2000]
 * (RW_table_LON / RW_table_TRANS, rw_table.c:310-391); like it, u above
 * 2000 takes the values at 2000.  Returns 0, or -1 for u < 19.8 (where the
 * reference's table has no entry). */
int mbt_rw_first_bin(double u, double *lon, double *trans)
{
  const double k = sqrt(3.0), c2 = sqrt(2.0) / M_PI;
  double e, cs, sn, Fc, Fs, K = 0.0, J = 0.0, a, tk;
  if (!(u >= 19.8)) return -1;
  if (u > 2000.) u = 2000.;
  e = exp(-u);
  cs = cos(k * u);
  sn = sin(k * u);
  Fc = 0.25 + e * (-cs + k * sn) / 4.0;
  Fs = k / 4.0 + e * (-k * cs - sn) / 4.0;
  /* panels at the Gaussian's scale 1/sqrt(u), then to where it vanishes;
     tolerances 1e-16 of each integral's size (K ~ sqrt(pi/u)/16, J ~
     sqrt(pi u)/8 + 0.1) */
  a = 0.0;
  for (tk = 0.25 / sqrt(u); a < sqrt(800.0 / u); tk *= 2.0) {
    K += integrate(rw_k, u, a, tk, 1e-16 * sqrt(M_PI / u) / 16.0, 0);
    a = tk;
  }
  a = 0.0;
  for (tk = 0.25 / sqrt(u); a < 1.0; tk *= 2.0) {
    const double b = tk < 1.0 ? tk : 1.0;
    J += integrate(rw_j, u, a, b, 1e-16 * sqrt(M_PI * u) / 8.0, 0);
    a = b;
  }
  J += integrate(rw_j_tail, u, 0.0, 1.0, 1e-16 * sqrt(M_PI * u) / 8.0, 0);
  if (lon) *lon = (e * (k * sn - cs) / 12.0 + c2 * K) / u;
  if (trans) *trans = ((k * Fs - Fc) / 12.0 + c2 * J) / u;
  return 0;
}

/* construct_greensfunc_RW, transform_weak.c:473-547: the long-time
 * asymptotes 1/t^(3/2) (LON) and 1/t^(1/2) (transverse) from bin 1 on, the
 * bin average of the full wake in bin 0.  The reference adds the
 * longitudinal part when EnableRW_short_LON is set and the transverse ones
 * only with EnableRW_short. */
static int greens_rw(const cfg_t *g, mbt_params *p, double *Gl, double *Gv, double *Gh)
{
  const int ncellmax = p->ncell;
  const double sgmatau = p->sigma_tau, dTau = p->dT;
  const double beffL1 = p->beffL[0], beffL2 = pow(p->beffL[1], 2);
  const double beffV3 = pow(p->beffV[0], 3), beffH3 = pow(p->beffH[0], 3);
  const double beffV4 = pow(p->beffV[1], 4), beffH4 = pow(p->beffH[1], 4);
  const double sigmarw = 1.0 / p->rhorw, t_const = sgmatau * dTau;
  double s0, rw0, rwt;
  int nc;
  if (p->track_plane[0] && g->enable_rw_short_lon) {
    const double ARW = sqrt(Z_0 / (sigmarw * C_LIGHT * M_PI)) / (4 * beffL1 * M_PI) * p->Lc;
    for (nc = 1; nc < ncellmax; nc++) {
      const double tRW = (nc + 0.5) * t_const;
      Gl[nc] -= ARW / (tRW * sqrt(tRW));
    }
    s0 = pow((2 * beffL2 * p->rhorw / Z_0), 1.0 / 3.0);
    if (mbt_rw_first_bin(sgmatau * dTau * C_LIGHT / s0, &rw0, NULL) < 0)
      return cfg_fail("short-range RW: longitudinal bin narrower than 19.8 s0");
    Gl[0] += rw0 * 4 * Z_0 * C_LIGHT / (M_PI * beffL2) * p->Lc;
    p->planeL++;
    if (!g->enable_rw_short) return 0;
  }
  if (p->track_plane[2]) {
    const double ARW = sqrt(Z_0 * C_LIGHT / sigmarw / M_PI) / (M_PI * beffV3) * p->Lc;
    s0 = pow((2 * p->beffV[1] * p->beffV[1] * p->rhorw / Z_0), 1.0 / 3.0);
    if (mbt_rw_first_bin(sgmatau * dTau * C_LIGHT / s0, NULL, &rwt) < 0)
      return cfg_fail("short-range RW: vertical bin narrower than 19.8 s0");
    Gv[0] += rwt * 8 * Z_0 * C_LIGHT / (M_PI * beffV4) * s0 * p->Lc;
    for (nc = 1; nc < ncellmax; nc++) {
      const double tRW = (nc + 0.5) * t_const;
      Gv[nc] += ARW / sqrt(tRW);
    }
    p->planeV++;
  }
  if (p->track_plane[1]) {
    const double ARW = sqrt(Z_0 * C_LIGHT / sigmarw / M_PI) / (M_PI * beffH3) * p->Lc;
    s0 = pow((2 * p->beffH[1] * p->beffH[1] * p->rhorw / Z_0), 1.0 / 3.0);
    if (mbt_rw_first_bin(sgmatau * dTau * C_LIGHT / s0, NULL, &rwt) < 0)
      return cfg_fail("short-range RW: horizontal bin narrower than 19.8 s0");
    Gh[0] += rwt * 8 * Z_0 * C_LIGHT / (M_PI * beffH4) * s0 * p->Lc;
    for (nc = 1; nc < ncellmax; nc++) {
      const double tRW = (nc + 0.5) * t_const;
      Gh[nc] += ARW / sqrt(tRW);
    }
    p->planeH++;
  }
  return 0;
}

int mbt_config_greens(const char *conf_path, mbt_params *p, double *Gl, double *Gv, double *Gh)
{
  cfg_t *g;
  int r, j, nc;
  if (!conf_path || !p || !Gl || !Gv || !Gh) return MBT_ERR_INVALID;
  g = (cfg_t *) calloc(1, sizeof(cfg_t));
  if (!g) return MBT_ERR_NOMEM;
  r = read_conf(conf_path, 0, 0, g);
  if (r) { free(g); return r; }
  nc = p->ncell;
  memset(Gl, 0, nc * sizeof(double));
  memset(Gv, 0, nc * sizeof(double));
  memset(Gh, 0, nc * sizeof(double));
  p->planeL = p->planeV = p->planeH = 0;
  /* construct_greensfunc_resonator, transform_weak.c:288-403 */
  for (j = 0; j < g->nres && nc > 0; j++) {
    const double R = g->res_Rs[j], Q = g->res_Q[j], w = g->res_wr[j];
    const int Pl = g->res_plane[j];
    const double resol = w * p->sigma_tau * p->dT;
    int ncc;
    if (!p->track_plane[Pl]) continue;
    if (Pl == 0) {
      double sq = sqrt(1.0 - 1.0 / (4.0 * Q * Q));
      double ar = 0.5 * resol / Q, arq = sq * resol, fac = 0.5 / (Q * sq), ampl = w * R / Q;
      Gl[0] += 0.5 * ampl;
      for (ncc = 1; ncc < nc; ncc++) {
        double fnc = (double) ncc, arg = fnc * arq, argE = fnc * ar;
        Gl[ncc] += ampl * exp(-argE) * (cos(arg) - fac * sin(arg));
      }
      p->planeL++;
    } else {
      double *G = Pl == 2 ? Gv : Gh;
      if (Q > 0.5) {
        double sq = sqrt(4.0 * Q * Q - 1.0), ar = 0.5 * resol / Q, arq = sq * resol / (2 * Q), ampl = 2 * R * w / sq;
        for (ncc = 0; ncc < nc; ncc++) {
          double fnc = (double) ncc, arg = fnc * arq, argE = fnc * ar;
          G[ncc] += ampl * exp(-argE) * sin(arg);
        }
      }
      if (Q < 0.5) {
        double sq = sqrt(1.0 - 4.0 * Q * Q), ar = 0.5 * resol / Q, arq = sq * resol / (2 * Q), ampl = 2 * R * w / sq;
        for (ncc = 0; ncc < nc; ncc++) {
          double fnc = (double) ncc, arg = fnc * arq, argE = fnc * ar;
          G[ncc] += ampl * exp(-argE) * sinh(arg);
        }
      }
      if (Pl == 2) p->planeV++;
      else p->planeH++;
    }
  }
  for (j = 0; j < g->nwake && nc > 0 && !r; j++) r = greens_file(g->wake_file[j], g->wake_plane[j], p, Gl, Gv, Gh);
  /* worker_weakweak.c:93-94 */
  if (!r && nc > 0 && (g->enable_rw_short || g->enable_rw_short_lon)) r = greens_rw(g, p, Gl, Gv, Gh);
  free(g);
  return r;
}
