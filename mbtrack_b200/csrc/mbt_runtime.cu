// mbt_runtime.cu -- libmbt C-ABI (include/mbt.h): tracking contexts on one
// B200, replacing the MPI manager/worker distribution of
// manager_weakweak.c / worker_weakweak.c with bunch-indexed blocks.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "mbt.h"
#include "mbt_device.cuh"
#include "mbt_kernels.cuh"
#include "mbt_beamion.cuh"

using mbt::Args;
using mbt::LrConst;
using mbt::RingState;
using mbt::Tile;

namespace {

constexpr double FKILO = 1.0e3, FGIGA = 1.0e9, FMILLI = 1.0e-3, FTERA = 1.0e12;
constexpr double C_LIGHT = 2.997925e+08, Z_0 = 376.73;
constexpr double PI = 3.14159265358979323846;

thread_local char g_create_error[512] = "";

}  // namespace

namespace mbt {
MlpDev mlp_device_view(const mbt_mlp *m);
size_t stats_scratch_doubles(int np);
int bunch_stats_strided(int np, const double *coord, size_t ld, const int tp[3], double *stats, void *stream,
                        double *scratch);
// Message for mbt_last_error(NULL, ...) from entry points without a context.
int fail_global(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_create_error, sizeof g_create_error, fmt, ap);
  va_end(ap);
  return code;
}
}  // namespace mbt

struct mbt_ctx {
  mbt_params p{};
  int nbunch = 0, npad = 0, tile = 0, ntile = 0, prec = 0, nc = 0, nlr = 0;
  int class_tile[3] = {0, 0, 0};   // tile size per bunch-size class (mbt_set_tiles)
  int tile_cap = 0;                // tiles the device arrays hold
  std::vector<int> bucket, np, off, tile0, ntiles, bucket_bunch;
  std::vector<double> ib;
  std::vector<Tile> tiles;
  std::vector<LrConst> lr;
  int noise = MBT_NOISE_PHILOX;
  uint64_t seed = 0;
  int prepared = 0;
  int histxz = 0;
  Args a{};
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_turns = 0;
  std::vector<void *> allocs;
  std::vector<size_t> alloc_bytes;  // size of each entry of allocs
  float *dev = nullptr;
  size_t dev_cap = 0;
  double *vbuf = nullptr;
  double *stats_init = nullptr;
  double *xfer = nullptr;        // device staging for exports
  long *pack = nullptr;          // per bunch: start of its 6 x np coordinates in a whole-beam host buffer
  double *stat_scratch = nullptr; // block partials of mbt_get_stats
  int bi_on = 0;                 // beam-ion stage
  mbt_beam_ion bicfg{};
  mbt::BiArgs bi{};
  cudaEvent_t bi_ev = nullptr;   // end of the beam-ion stage (profiling)
  cudaEvent_t bi_kev[3] = {nullptr, nullptr, nullptr};   // after frames, ions, clouds (profiling)
  double bi_kms[4] = {0, 0, 0, 0};                        // frames, ions, clouds, kick: last profile
  mbt::MlpDev mlp{};             // learned field (surrogate runs)
  bool mlp_set = false;
  double bi_ms = 0.0;            // its average device time in the last mbt_profile_turns
  std::vector<int> watch;        // bunches whose potentials are recorded
  int scan_steps = 0;            // a scan boundary launches scan_currents / scan_rw
  double scan_d_ma = 0.0, scan_d_a = 0.0;   // current steps [mA] per bucket, [A] per bunch
  cudaEvent_t ev[6] = {};
  cudaStream_t copy_stream = nullptr;   // statistics to the host, beside the turns
  cudaEvent_t cev[3] = {};              // two units of turns in flight, the copies' tail
  double timing[4] = {0, 0, 0, 0};
  int device = 0;
  int nsm = 148;
  char err[512] = "";
};

namespace {

int fail(mbt_ctx *c, int code, const char *fmt, ...) {
  char *dst = c ? c->err : g_create_error;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(dst, 512, fmt, ap);
  va_end(ap);
  return code;
}

#define CK(call)                                                                   \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess)                                                         \
      return fail(c, MBT_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                  __FILE__, __LINE__);                                             \
  } while (0)

template <typename T>
int dalloc(mbt_ctx *c, T **ptr, size_t n) {
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess) return fail(c, MBT_ERR_NOMEM, "cudaMalloc(%zu): %s", n * sizeof(T), cudaGetErrorString(e));
  cudaMemset(p, 0, std::max<size_t>(n, 1) * sizeof(T));
  c->allocs.push_back(p);
  c->alloc_bytes.push_back(std::max<size_t>(n, 1) * sizeof(T));
  *ptr = static_cast<T *>(p);
  return 0;
}

template <typename T>
int dupload(mbt_ctx *c, T **ptr, const T *src, size_t n) {
  int r = dalloc(c, ptr, n);
  if (r) return r;
  if (n) CK(cudaMemcpy(*ptr, src, n * sizeof(T), cudaMemcpyHostToDevice));
  return 0;
}

int check_device(mbt_ctx *c) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return fail(c, MBT_ERR_NODEVICE, "no CUDA device (%s): libmbt has no CPU path",
                e == cudaSuccess ? "count 0" : cudaGetErrorString(e));
  return 0;
}

// Smallest tile that still fills the GPU: at least 4 tiles per SM when the
// beam allows it, tiles between 512 and 8192 particles.
int choose_tile(const std::vector<int> &np, int sms) {
  long total = 0;
  for (int n : np) total += n;
  long want = std::max<long>(1, total / (4L * sms));
  int t = 512;
  while (t < 8192 && t < want) t <<= 1;
  return t;
}

// Bunch-size class of a bunch for the tile table: up to 4096, up to 32768,
// more macroparticles.
int size_class(int np) { return np <= 4096 ? 0 : (np <= 32768 ? 1 : 2); }

// Tiles of every bunch from the class tile sizes: ceil(np / T) tiles of
// equal size (a multiple of 32 particles) inside each bunch.
void layout_tiles(mbt_ctx *c) {
  c->tiles.clear();
  for (int b = 0; b < c->nbunch; ++b) {
    const int T = c->class_tile[size_class(c->np[b])];
    c->tile0[b] = (int)c->tiles.size();
    const int nt = (c->np[b] + T - 1) / T;
    const int per = ((c->np[b] + nt - 1) / nt + 31) / 32 * 32;
    for (int s = 0; s < c->np[b]; s += per) {
      Tile t{b, c->off[b] + s, std::min(per, c->np[b] - s), 0};
      c->tiles.push_back(t);
    }
    c->ntiles[b] = (int)c->tiles.size() - c->tile0[b];
  }
  c->ntile = (int)c->tiles.size();
  c->tile = std::max(c->class_tile[0], std::max(c->class_tile[1], c->class_tile[2]));
}

void cmul(double a0, double a1, double b0, double b1, double &r0, double &r1) {
  r0 = a0 * b0 - a1 * b1;
  r1 = a0 * b1 + a1 * b0;
}

int validate(mbt_ctx *c, const mbt_params *p, int nbunch, const int *bucket, const int *np) {
  if (!p || nbunch <= 0 || !bucket || !np) return fail(c, MBT_ERR_INVALID, "null argument or nbunch <= 0");
  if (p->nharm <= 0) return fail(c, MBT_ERR_INVALID, "nharm must be positive");
  if (p->ncell < 0 || p->ncell > MBT_MAX_NCELL) return fail(c, MBT_ERR_INVALID, "ncell %d outside 0..%d", p->ncell, MBT_MAX_NCELL);
  for (int i = 0; i < nbunch; ++i) {
    if (bucket[i] < 0 || bucket[i] >= p->nharm) return fail(c, MBT_ERR_INVALID, "bucket[%d]=%d outside 0..h-1", i, bucket[i]);
    if (i > 0 && bucket[i] <= bucket[i - 1]) return fail(c, MBT_ERR_INVALID, "buckets must be strictly ascending");
    if (np[i] <= 0) return fail(c, MBT_ERR_INVALID, "np[%d]=%d must be positive", i, np[i]);
  }
  int nlr = p->n_lr[0] + p->n_lr[1] + p->n_lr[2];
  for (int pl = 0; pl < 3; ++pl)
    if (p->n_lr[pl] < 0 || p->n_lr[pl] > MBT_MAX_LR) return fail(c, MBT_ERR_INVALID, "n_lr[%d] outside 0..%d", pl, MBT_MAX_LR);
  for (int pl = 1; pl < 3; ++pl)
    if (p->n_lr[pl] > 0 && !p->track_plane[pl])
      return fail(c, MBT_ERR_INVALID, "long-range resonator in an untracked plane %d", pl);
  if ((nlr > 0 || p->planeL + p->planeV + p->planeH > 0) && p->ncell <= 0)
    return fail(c, MBT_ERR_INVALID, "wakes need ncell > 0");
  if (p->rffb && (p->n_lr[0] <= 0 || p->rffb_resonator < 1 || p->rffb_resonator > p->n_lr[0] || p->rffb_len <= 0))
    return fail(c, MBT_ERR_INVALID, "RF feedback needs a longitudinal long-range resonator and a positive averaging length");
  if (p->n_active_hc < 0 || p->n_active_hc > MBT_MAX_AHC) return fail(c, MBT_ERR_INVALID, "n_active_hc outside 0..%d", MBT_MAX_AHC);
  if (p->rw_long && (p->Nmlt < 0 || p->beffH[0] <= 0 && p->track_plane[1] || p->beffV[0] <= 0 && p->track_plane[2]))
    return fail(c, MBT_ERR_INVALID, "long-range resistive wall needs Nmlt >= 0 and beffH3/beffV3 > 0");
  if (!p->track_plane[0]) return fail(c, MBT_ERR_INVALID, "the longitudinal plane is always tracked");
  if (p->scan < 0 || p->scan > 4 || (p->scan != 0 && p->nrev_scan < 1))
    return fail(c, MBT_ERR_INVALID, "scan type %d outside 0..4 or NrevScan %ld < 1", p->scan, p->nrev_scan);
  return 0;
}

template <bool MOVE, int NOISE, bool HISTXZ>
void launch_map(mbt_ctx *c) {
  const size_t sm = mbt::turn_map_smem(c->nc, HISTXZ);
  static bool attr_set = false;   // per instantiation, per process
  if (!attr_set) {
    cudaFuncSetAttribute(mbt::turn_map<MOVE, NOISE, HISTXZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)mbt::turn_map_smem(MBT_MAX_NCELL, HISTXZ));
    attr_set = true;
  }
  mbt::turn_map<MOVE, NOISE, HISTXZ><<<c->ntile, mbt::kMapThreads, sm, c->stream>>>(c->a);
}

template <bool MOVE>
void launch_map_noise(mbt_ctx *c, int noise) {
  if (c->histxz) {
    if (!MOVE || noise == MBT_NOISE_NONE) launch_map<MOVE, MBT_NOISE_NONE, true>(c);
    else if (noise == MBT_NOISE_PHILOX) launch_map<MOVE, MBT_NOISE_PHILOX, true>(c);
    else launch_map<MOVE, MBT_NOISE_INJECTED, true>(c);
  } else {
    if (!MOVE || noise == MBT_NOISE_NONE) launch_map<MOVE, MBT_NOISE_NONE, false>(c);
    else if (noise == MBT_NOISE_PHILOX) launch_map<MOVE, MBT_NOISE_PHILOX, false>(c);
    else launch_map<MOVE, MBT_NOISE_INJECTED, false>(c);
  }
}

int effective_noise(const mbt_ctx *c) { return c->p.quantum ? c->noise : MBT_NOISE_NONE; }

size_t smem_reduce(const mbt_ctx *c) { return (size_t)c->prec * sizeof(double); }
size_t smem_wakes(const mbt_ctx *c) { return mbt::bunch_wakes_smem(c->nc); }
// Blocks of the resistive-wall sums: two per SM at most, at least 32
// history steps each.
int rw_blocks_for(const mbt_params *p, int nsm) {
  if (!p->rw_long) return 0;
  const long M = (long)(p->Nmlt + 1) * p->nharm;
  return (int)std::max<long>(1, std::min<long>(2L * nsm, (M + 31) / 32));
}
int rw_blocks(const mbt_ctx *c) { return c->a.rw_nblk; }
size_t smem_scan(const mbt_ctx *c) {
  return mbt::ring_scan_smem_doubles(c->p.rw_long, c->p.Nmlt, c->p.nharm, c->a.rw_nblk) * sizeof(double);
}

// The beam-ion stage of a turn: frames, ion clouds, electron kicks; with
// `prof`, events between its kernels.
void enqueue_beam_ion(mbt_ctx *c, bool prof = false) {
  const mbt::BiArgs &bi = c->bi;
  const int n = bi.n_ip * bi.nb;
  mbt::bi_frames<<<(n + 127) / 128, 128, 0, c->stream>>>(bi);
  if (prof) cudaEventRecord(c->bi_kev[0], c->stream);
  if (c->bicfg.surrogate) {
    const int grid = c->nsm;
    if (bi.nb > 1)
      mbt::bi_ions_mlp<<<grid, 128 * mbt::kMlpGroups, mbt::kMlpCtaSmem, c->stream>>>(bi, c->mlp);
    if (prof) cudaEventRecord(c->bi_kev[1], c->stream);
    mbt::bi_clouds<<<dim3(bi.nb, bi.n_ip), mbt::kBiThreads, 0, c->stream>>>(bi);
    if (prof) cudaEventRecord(c->bi_kev[2], c->stream);
    mbt::bi_kick_mlp<<<grid, 128 * mbt::kMlpGroups, mbt::kMlpCtaSmem, c->stream>>>(c->a, bi, c->mlp);
    return;
  }
  if (bi.nb > 1) {
    mbt::bi_ions<<<dim3(bi.bpp, bi.nb - 1, bi.n_ip), mbt::kBiThreads, 0, c->stream>>>(bi);
  }
  if (prof) cudaEventRecord(c->bi_kev[1], c->stream);
  mbt::bi_clouds<<<dim3(bi.nb, bi.n_ip), mbt::kBiThreads, 0, c->stream>>>(bi);
  if (prof) cudaEventRecord(c->bi_kev[2], c->stream);
  mbt::bi_kick_grouped<<<c->ntile, mbt::kBiThreads, mbt::bi_kick_grouped_smem(bi.n_ip), c->stream>>>(c->a, bi);
}

// Whether turn `turn` (0-based) ends a scan interval: (rev+1) % NrevScan
// == 0 (worker_weakweak.c:389).
bool scan_boundary(const mbt_ctx *c, long turn) {
  return c->scan_steps && (turn + 1) % c->p.nrev_scan == 0;
}

// One turn: particle pass, bunch reduction, ring scan, bunch wakes, and
// the beam-ion stage when it is on.  boundary: the turn ends a scan
// interval (two small launches more).
void enqueue_turn(mbt_ctx *c, cudaEvent_t *ev, bool boundary = false) {
  const bool current_scan = boundary && c->p.scan == 1;
  if (ev) cudaEventRecord(ev[0], c->stream);
  launch_map_noise<true>(c, effective_noise(c));
  if (ev) cudaEventRecord(ev[1], c->stream);
  if (current_scan) {
    const int n = std::max(c->p.nharm, c->nbunch);
    mbt::scan_currents<<<(n + 255) / 256, 256, 0, c->stream>>>(c->a, c->scan_d_ma, c->scan_d_a, c->p.T0, c->p.E0);
  }
  mbt::bunch_reduce<<<c->nbunch, mbt::kBlock, smem_reduce(c), c->stream>>>(c->a, mbt::kReduceTurn, nullptr);
  if (ev) cudaEventRecord(ev[2], c->stream);
  mbt::ring_scan<<<1 + rw_blocks(c), mbt::kBlock, smem_scan(c), c->stream>>>(c->a, 1, 0, c->vbuf);
  if (ev) cudaEventRecord(ev[3], c->stream);
  mbt::bunch_wakes<<<c->nbunch, mbt::kBlock, smem_wakes(c), c->stream>>>(c->a, 1);
  if (ev) cudaEventRecord(ev[4], c->stream);
  if (c->bi_on) {
    enqueue_beam_ion(c, ev != nullptr);
    if (ev) cudaEventRecord(c->bi_ev, c->stream);
  }
  if (boundary) {
    const long n = std::max<long>(std::max<long>((long)(c->p.Nmlt + 2) * c->p.nharm, c->p.nharm), c->nbunch);
    mbt::scan_rw<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->a, current_scan ? 1 : 0, c->scan_d_a,
                                                                      c->bi_on ? const_cast<double *>(c->bi.ib) : nullptr);
  }
}

int sync_and_check(mbt_ctx *c) {
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  RingState rs;
  CK(cudaMemcpy(&rs, c->a.rs, sizeof(rs), cudaMemcpyDeviceToHost));
  if (rs.error & 2)
    return fail(c, MBT_ERR_TIMEOUT, "device error word %d: a bounded pipeline wait of the particle pass gave up",
                rs.error);
  if (rs.error & 4)
    return fail(c, MBT_ERR_TIMEOUT,
                "device error word %d: a bounded wait on the tensor cores of the learned field gave up", rs.error);
  if (rs.error) return fail(c, MBT_ERR_STATE, "device error word %d: injected deviates exhausted", rs.error);
  return 0;
}

int build_graph(mbt_ctx *c, int turns) {
  if (c->graph && c->graph_turns == turns) return 0;
  if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  for (int t = 0; t < turns; ++t) enqueue_turn(c, nullptr);
  cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  if (e != cudaSuccess) return fail(c, MBT_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
  e = cudaGraphInstantiate(&c->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(c, MBT_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
  c->graph_turns = turns;
  return 0;
}

}  // namespace

extern "C" {

size_t mbt_params_size(void) { return sizeof(mbt_params); }

int mbt_use_device(int device) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) return fail(nullptr, MBT_ERR_NODEVICE, "no CUDA device: libmbt has no CPU path");
  if (device < 0 || device >= n) return fail(nullptr, MBT_ERR_INVALID, "device %d outside 0..%d", device, n - 1);
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(nullptr, MBT_ERR_CUDA, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
  return 0;
}

int mbt_last_error(const mbt_ctx *ctx, char *buf, size_t len) {
  if (!buf || len == 0) return MBT_ERR_INVALID;
  snprintf(buf, len, "%s", ctx ? ctx->err : g_create_error);
  return 0;
}

int mbt_create(const mbt_params *p, int nbunch, const int *bucket, const int *np, const double *ib,
               const double *Gl, const double *Gv, const double *Gh, int noise_mode, uint64_t seed,
               mbt_ctx **out) {
  mbt_ctx *c = nullptr;
  if (!out) return fail(nullptr, MBT_ERR_INVALID, "out is NULL");
  *out = nullptr;
  int r = check_device(nullptr);
  if (r) return r;
  r = validate(nullptr, p, nbunch, bucket, np);
  if (r) return r;
  if (!ib) return fail(nullptr, MBT_ERR_INVALID, "ib is NULL");
  if (noise_mode != MBT_NOISE_PHILOX && noise_mode != MBT_NOISE_INJECTED)
    return fail(nullptr, MBT_ERR_INVALID, "unknown noise mode %d", noise_mode);
  c = new (std::nothrow) mbt_ctx;
  if (!c) return fail(nullptr, MBT_ERR_NOMEM, "host allocation");
  c->p = *p;
  c->nbunch = nbunch;
  c->noise = noise_mode;
  c->seed = seed;
  c->bucket.assign(bucket, bucket + nbunch);
  c->np.assign(np, np + nbunch);
  c->ib.assign(ib, ib + nbunch);
  cudaGetDevice(&c->device);
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, c->device);
  c->nsm = prop.multiProcessorCount;
  auto bail = [&](int code) { int rc = code; mbt_destroy(c); return rc; };
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(nullptr, MBT_ERR_CUDA, "stream create"));
  for (auto &e : c->ev) cudaEventCreate(&e);
  for (auto &e : c->cev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);

  // geometry: bunches padded to 32 particles, tiles inside bunches
  const int t0 = choose_tile(c->np, prop.multiProcessorCount);
  for (int k = 0; k < 3; ++k) c->class_tile[k] = t0;
  c->off.resize(nbunch);
  c->tile0.resize(nbunch);
  c->ntiles.resize(nbunch);
  long pos = 0;
  for (int b = 0; b < nbunch; ++b) {
    c->off[b] = (int)pos;
    pos += (c->np[b] + 31) / 32 * 32;
    c->tile_cap += (c->np[b] + 511) / 512;   // the most tiles the smallest tile size makes
  }
  if (pos > 0x7fffffffL / 6) return bail(fail(nullptr, MBT_ERR_INVALID, "beam too large for one context"));
  c->npad = (int)pos;
  layout_tiles(c);
  c->tile_cap = std::max(c->tile_cap, c->ntile);
  c->nc = std::max(p->ncell, 1);
  c->bucket_bunch.assign(p->nharm, -1);
  for (int b = 0; b < nbunch; ++b) c->bucket_bunch[c->bucket[b]] = b;

  Args &a = c->a;
  a.nbunch = nbunch;
  a.ntile = c->ntile;
  a.npad = c->npad;
  a.tile = c->tile;
  a.ncell = c->nc;
  a.nharm = p->nharm;
  const int lr_tot = p->n_lr[0] + p->n_lr[1] + p->n_lr[2];
  a.selffield = (p->ncell > 0 && p->planeL + p->planeV + p->planeH + lr_tot > 0) ? 1 : 0;
  c->histxz = a.selffield && (p->planeV > 0 || p->planeH > 0 || p->n_lr[1] > 0 || p->n_lr[2] > 0);
  a.hist_xz = c->histxz;
  // partial record: counts [, sum x, sum z], then the extras
  a.hoff = (c->histxz ? 3 : 1) * c->nc;
  c->prec = a.hoff + mbt::kPartialExtra;
  a.prec = c->prec;
  a.lr_kick[0] = (p->n_lr[0] + p->planeL) > 0;
  a.lr_kick[1] = p->planeH > 0;
  a.lr_kick[2] = p->planeV > 0;
  a.planeL = p->planeL; a.planeV = p->planeV; a.planeH = p->planeH;
  a.RsisL = p->RsisL; a.aindL = p->aindL;
  a.sgmatau2 = p->sigma_tau * p->sigma_tau;
  a.dTau2 = p->dT * p->dT;
  a.rw_long = p->rw_long; a.Nmlt = p->Nmlt; a.triggerRW = p->triggerRW;
  a.E0 = p->E0;
  a.noise = noise_mode;
  a.seed = seed;
  {
    const mbt::PhiloxKeys K = mbt::philox_keys(seed);
    for (int q = 0; q < 10; ++q) { a.philox_k0[q] = K.k0[q]; a.philox_k1[q] = K.k1[q]; }
  }

  std::vector<int> np_v(c->np), kb_v(c->bucket);
  std::vector<double> ibunch(p->nharm, 0.0), factg(nbunch);
  for (int b = 0; b < nbunch; ++b) {
    ibunch[c->bucket[b]] = c->ib[b] * FKILO;   // manager_weakweak.c:78
    factg[b] = -p->T0 * c->ib[b] / (c->np[b] * p->E0 * FGIGA);   // transform_weak.c:567
  }

  // long-range resonator constants (transform_weak.c:976-1004)
  const double hd = (double)p->nharm;
  const double dTau = p->dT * p->sigma_tau;
  const double tbucket = (p->T0 / hd - p->ncell * dTau);
  std::vector<double> fac, pw;
  for (int pl = 0; pl < 3; ++pl) {
    for (int l = 0; l < p->n_lr[pl]; ++l) {
      LrConst L{};
      L.plane = pl;
      L.l = l;
      const double wr = p->lr_wr[pl][l], Q = p->lr_Q[pl][l], Rs = p->lr_Rs[pl][l];
      const double alpha = wr * 0.5 / Q;
      L.Amp = 2 * alpha * Rs * p->T0 / p->E0 / FGIGA;
      const double C0 = -alpha, C1 = wr;
      L.prog[0] = exp(C0 * dTau) * cos(C1 * dTau);
      L.prog[1] = exp(C0 * dTau) * sin(C1 * dTau);
      L.fb = (p->rffb && pl == 0 && p->rffb_resonator == l + 1) ? 1 : 0;
      double taubeam = 0, taub2beam = 0;
      if (L.fb) {
        taubeam = p->nsigma * p->sigma_tau + dTau * 1.5;
        taub2beam = -p->nsigma * p->sigma_tau + dTau * 0.5 - tbucket;
      }
      L.p2b[0] = exp(C0 * taubeam) * cos(C1 * taubeam);
      L.p2b[1] = exp(C0 * taubeam) * sin(C1 * taubeam);
      L.pb2b[0] = exp(C0 * taub2beam) * cos(C1 * taub2beam);
      L.pb2b[1] = exp(C0 * taub2beam) * sin(C1 * taub2beam);
      L.gap[0] = exp(C0 * tbucket); L.gap[1] = cos(C1 * tbucket); L.gap[2] = sin(C1 * tbucket);
      L.emp[0] = exp(C0 * p->T0 / hd); L.emp[1] = cos(C1 * p->T0 / hd); L.emp[2] = sin(C1 * p->T0 / hd);
      double q0 = 1.0, q1 = 0.0;
      for (int j = 0; j < c->nc; ++j) {
        double r0, r1;
        cmul(q0, q1, L.prog[0], L.prog[1], r0, r1);
        q0 = r0; q1 = r1;
        pw.push_back(q0);
        pw.push_back(q1);
      }
      L.pn[0] = q0; L.pn[1] = q1;
      for (int b = 0; b < nbunch; ++b) fac.push_back(L.Amp / c->np[b] * FMILLI);   // per source bunch
      c->lr.push_back(L);
    }
  }
  c->nlr = (int)c->lr.size();
  a.nlr = c->nlr;

  // resistive wall: RWconst (transform_weak.c:811) and 1/sqrt(m T0/h)
  std::vector<double> rsq;
  if (p->rw_long) {
    const int M = (p->Nmlt + 1) * p->nharm;
    rsq.resize(M + 1);
    const double deltab = p->T0 / hd;
    rsq[0] = 0.0;
    for (int m = 1; m <= M; ++m) rsq[m] = 1.0 / sqrt(m * deltab);
    for (int trig = 0; trig < 2; ++trig) {
      for (int pl = 1; pl <= 2; ++pl) {
        double beff3 = pl == 1 ? p->beffH[0] : p->beffV[0];
        if (trig) beff3 /= 2;
        // The reference divides RWconst by fNp and multiplies every term of
        // the sum by fNp (transform_weak.c:811,822); both are left out.
        a.rw_const[trig][pl - 1] = p->T0 / p->E0 / FTERA * p->Lc / (PI * pow(beff3, 3)) * sqrt(Z_0 * C_LIGHT * p->rhorw / PI);
      }
    }
  }

  // optics constants (transform_weak.c:35-46)
  mbt::OpticConst &oc = a.oc;
  oc.damp = 1.0 - p->De;
  oc.excite = 2.0 * p->slope_sgm[0] * sqrt(p->T0 / p->taue);
  oc.qv_pos = p->pos_sgm[2] * sqrt(2.0 * p->T0 / p->tauz);
  oc.qv_slope = p->slope_sgm[2] * sqrt(2.0 * p->T0 / p->tauz);
  oc.qh_pos = p->pos_sgm[1] * sqrt(2.0 * p->T0 / p->taux);
  oc.qh_slope = p->slope_sgm[1] * sqrt(2.0 * p->T0 / p->taux);
  oc.E0 = p->E0;
  oc.wrf = p->wrf; oc.Urad = p->Urad; oc.T0 = p->T0; oc.ac = p->ac;
  oc.psiV0 = 2.0 * PI * p->QV0;
  oc.psiH0 = 2.0 * PI * p->QH0;
  oc.Gziz = p->Gziz; oc.Gzix = p->Gzix;
  oc.CHH = p->CHH; oc.CHV = p->CHV; oc.CVH = p->CVH; oc.CVV = p->CVV;
  oc.alphaV = p->alpha1[2]; oc.betaV = p->beta1[2]; oc.gammaV = p->gamma1[2];
  oc.alphaH = p->alpha1[1]; oc.betaH = p->beta1[1]; oc.gammaH = p->gamma1[1];
  oc.dispH = p->dispH1; oc.disppH = p->disppH1;
  oc.HC_k = p->HC_k; oc.m_aHC_d = (double)p->m_aHC; oc.m_phi_n = p->m_aHC * p->phi_n;
  oc.n_ahc = p->n_active_hc;
  for (int j = 0; j < p->n_active_hc; ++j) {
    oc.ahc_amp[j] = p->ahc_vpeak[j] / (p->E0 * FGIGA);
    oc.ahc_w[j] = p->wrf * p->ahc_nhc[j];
    oc.ahc_phi[j] = p->ahc_phi[j];
    oc.ahc_nhc[j] = p->ahc_nhc[j];
  }
  oc.ideal_hc = p->ideal_hc;
  oc.amp_dep = p->amp_dep_qv;
  oc.quantum = p->quantum;
  oc.track_h = p->track_plane[1];
  oc.track_v = p->track_plane[2];
  oc.sigma_tau = p->sigma_tau;
  oc.nsigma = p->nsigma;
  oc.dT = p->dT;
  oc.gammaL = p->gamma1[0]; oc.alphaL = p->alpha1[0]; oc.betaL = p->beta1[0];
  oc.inv_sigma_tau = p->sigma_tau > 0 ? 1.0 / p->sigma_tau : 0.0;
  oc.inv_dT = p->dT > 0 ? 1.0 / p->dT : 0.0;
  oc.sin_psiV0 = sin(oc.psiV0);
  oc.cos_psiV0 = cos(oc.psiV0);
  oc.sin_psiH0 = sin(oc.psiH0);
  oc.cos_psiH0 = cos(oc.psiH0);
  oc.ncell = c->nc;

  // device allocations
  int rc = 0;
  std::vector<double> g0(c->nc, 0.0);
  auto gl = [&](const double *g) { return g ? g : g0.data(); };
  rc = rc ? rc : dalloc(c, &a.coord, (size_t)6 * c->npad);
  Tile *tiles_d = nullptr;
  rc = rc ? rc : dalloc(c, &tiles_d, (size_t)c->tile_cap);
  if (!rc && cudaMemcpy(tiles_d, c->tiles.data(), c->tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice) != cudaSuccess)
    rc = fail(nullptr, MBT_ERR_CUDA, "tile upload");
  a.tiles = tiles_d;
  int *ip;
  rc = rc ? rc : dupload(c, &ip, c->tile0.data(), nbunch); a.bunch_tile0 = ip;
  rc = rc ? rc : dupload(c, &ip, c->ntiles.data(), nbunch); a.bunch_ntile = ip;
  rc = rc ? rc : dupload(c, &ip, np_v.data(), nbunch); a.bunch_np = ip;
  rc = rc ? rc : dupload(c, &ip, kb_v.data(), nbunch); a.bunch_kb = ip;
  rc = rc ? rc : dupload(c, &ip, c->off.data(), nbunch); a.bunch_off = ip;
  {
    std::vector<long> pack(nbunch);
    long pos = 0;
    for (int b = 0; b < nbunch; ++b) { pack[b] = pos; pos += 6L * np_v[b]; }
    rc = rc ? rc : dupload(c, &c->pack, pack.data(), nbunch);
  }
  rc = rc ? rc : dupload(c, &ip, c->bucket_bunch.data(), p->nharm); a.bucket_bunch = ip;
  double *dp;
  rc = rc ? rc : dupload(c, &dp, c->ib.data(), nbunch); a.bunch_ib = dp;
  rc = rc ? rc : dupload(c, &dp, fac.empty() ? g0.data() : fac.data(), std::max<size_t>(fac.size(), 1)); a.bunch_fac = dp;
  rc = rc ? rc : dupload(c, &dp, factg.data(), nbunch); a.bunch_factg = dp;
  rc = rc ? rc : dupload(c, &dp, ibunch.data(), p->nharm); a.ibunch = dp;
  // a current scan changes the wake currents one step before the
  // resistive-wall current (scan_currents / scan_rw); otherwise they are one
  a.rw_ib = a.ibunch;
  if (p->scan == 1 && p->rw_long) { rc = rc ? rc : dupload(c, &dp, ibunch.data(), p->nharm); a.rw_ib = dp; }
  c->scan_steps = p->scan == 1 || (p->scan != 0 && p->rw_long);
  c->scan_d_ma = p->scan_step / (double)nbunch;             // tracking.c:53
  c->scan_d_a = p->scan_step / ((double)nbunch * FKILO);    // tracking.c:49
  rc = rc ? rc : dupload(c, &dp, gl(Gl), c->nc); a.Gl = dp;
  rc = rc ? rc : dupload(c, &dp, gl(Gv), c->nc); a.Gv = dp;
  rc = rc ? rc : dupload(c, &dp, gl(Gh), c->nc); a.Gh = dp;
  rc = rc ? rc : dalloc(c, &a.part, (size_t)c->tile_cap * c->prec);
  rc = rc ? rc : dalloc(c, &a.shift, (size_t)nbunch * 6);
  rc = rc ? rc : dalloc(c, &a.hist, (size_t)nbunch * 6 * c->nc);
  rc = rc ? rc : dalloc(c, &a.cellrange, (size_t)nbunch * 2);
  rc = rc ? rc : dalloc(c, &a.kick, (size_t)nbunch * 3 * c->nc);
  a.rw_nblk = rw_blocks_for(p, c->nsm);
  rc = rc ? rc : dalloc(c, &a.rw_part, (size_t)nbunch * 2);
  rc = rc ? rc : dalloc(c, &a.rw_acc, (size_t)std::max(a.rw_nblk, 1) * nbunch * 2);
  a.stats_cap = 256;
  rc = rc ? rc : dalloc(c, &a.stats, (size_t)a.stats_cap * nbunch * 12);
  rc = rc ? rc : dalloc(c, &c->stats_init, (size_t)nbunch * 12);
  rc = rc ? rc : dalloc(c, &a.ampinv, (size_t)a.stats_cap * nbunch * 6);
  LrConst *lr_d = nullptr;
  rc = rc ? rc : dupload(c, &lr_d, c->lr.empty() ? nullptr : c->lr.data(), c->lr.size());
  a.lr = lr_d;
  const size_t nlr1 = std::max(c->nlr, 1);
  rc = rc ? rc : dalloc(c, &a.lr_u, nlr1 * nbunch * c->nc * 2);
  rc = rc ? rc : dalloc(c, &a.lr_b, nlr1 * nbunch * c->nc);
  rc = rc ? rc : dalloc(c, &a.lr_vs, nlr1 * p->nharm * 2);
  rc = rc ? rc : dupload(c, &dp, pw.empty() ? g0.data() : pw.data(), std::max<size_t>(pw.size(), 1)); a.lr_pw = dp;
  rc = rc ? rc : dalloc(c, &c->vbuf, (size_t)4 * p->nharm);
  rc = rc ? rc : dalloc(c, &a.dipole, p->rw_long ? (size_t)(p->Nmlt + 2) * p->nharm * 2 : 1);
  rc = rc ? rc : dalloc(c, &a.rw_e, p->rw_long ? (size_t)(p->Nmlt + 2) * p->nharm * 2 : 1);
  rc = rc ? rc : dupload(c, &dp, rsq.empty() ? g0.data() : rsq.data(), std::max<size_t>(rsq.size(), 1)); a.rw_rsq = dp;
  a.rffb_len = p->rffb ? p->rffb_len : 0;
  a.rffb_off_after_init = p->rffb_off_after_init;
  a.rffb_vrf_design = p->rffb_vrf_design;
  a.rffb_phi0_design = p->rffb_phi0_design;
  a.rffb_kappa = p->rffb_gain > 0.0 ? p->rffb_gain / (1.0 + p->rffb_gain) : 0.0;
  a.rffb_delay = p->rffb_delay;
  rc = rc ? rc : dalloc(c, &a.rffb_hist, (size_t)2 * std::max(a.rffb_len, 1));
  rc = rc ? rc : dalloc(c, &a.rs, 1);
  rc = rc ? rc : dalloc(c, &c->xfer, (size_t)6 * c->npad);
  if (rc) { snprintf(g_create_error, sizeof g_create_error, "%s", c->err); return bail(rc); }
  RingState rs{};
  rs.turn = 0;
  rs.Vrf0 = p->Vrf0;
  rs.phai0 = p->phai0;
  rs.rffb_on = p->rffb;
  rs.Vrf0_last = p->Vrf0;
  rs.phai0_last = p->phai0;
  rs.sin_phai0 = sin(p->phai0);
  rs.cos_phai0 = cos(p->phai0);
  if (cudaMemcpy(a.rs, &rs, sizeof rs, cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(fail(nullptr, MBT_ERR_CUDA, "state upload"));
  const size_t smw = smem_wakes(c);
  if (smw > 48 * 1024)
    cudaFuncSetAttribute(mbt::bunch_wakes, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smw);
  const size_t sms = smem_scan(c);
  if (sms > 48 * 1024)
    cudaFuncSetAttribute(mbt::ring_scan, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sms);
  *out = c;
  return 0;
}

int mbt_destroy(mbt_ctx *c) {
  if (!c) return 0;
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->graph) cudaGraphExecDestroy(c->graph);
  if (c->bi_ev) cudaEventDestroy(c->bi_ev);
  for (cudaEvent_t e : c->bi_kev)
    if (e) cudaEventDestroy(e);
  for (void *p : c->allocs) cudaFree(p);
  if (c->dev) cudaFree(c->dev);
  for (auto &e : c->ev) if (e) cudaEventDestroy(e);
  for (auto &e : c->cev) if (e) cudaEventDestroy(e);
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return 0;
}

int mbt_load_particles(mbt_ctx *c, int ibunch, const double *soa6, int np) {
  if (!c || !soa6) return MBT_ERR_INVALID;
  if (ibunch < 0 || ibunch >= c->nbunch) return fail(c, MBT_ERR_INVALID, "bunch %d out of range", ibunch);
  if (np != c->np[ibunch]) return fail(c, MBT_ERR_INVALID, "bunch %d holds %d particles, got %d", ibunch, c->np[ibunch], np);
  for (int k = 0; k < 6; ++k)
    CK(cudaMemcpyAsync(c->a.coord + (size_t)k * c->npad + c->off[ibunch], soa6 + (size_t)k * np,
                       np * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

// The whole beam crosses PCIe as one copy into the staging buffer (host
// layout: bunch after bunch, 6 x np each), and a kernel moves it to the
// device layout (coordinate arrays of npad, bunches at their offsets).
int mbt_load_all(mbt_ctx *c, const double *soa6_all) {
  if (!c || !soa6_all) return MBT_ERR_INVALID;
  long total = 0;
  for (int n : c->np) total += n;
  CK(cudaMemcpyAsync(c->xfer, soa6_all, (size_t)6 * total * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  mbt::beam_import<<<dim3(16, c->nbunch), 256, 0, c->stream>>>(c->a, c->pack, c->xfer);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int mbt_generate_beam(mbt_ctx *c, uint64_t seed) {
  if (!c) return MBT_ERR_INVALID;
  double h[15];
  for (int k = 0; k < 3; ++k) {
    h[k] = c->p.pos_offset[k];
    h[3 + k] = c->p.slope_offset[k];
    h[6 + k] = c->p.pos_sgm[k];
    h[9 + k] = c->p.slope_sgm[k];
    h[12 + k] = c->p.correlate[k];
  }
  double *d = c->xfer;
  CK(cudaMemcpyAsync(d, h, sizeof h, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->a.coord, 0, (size_t)6 * c->npad * sizeof(double), c->stream));
  dim3 grid(64, c->nbunch);
  mbt::generate_beam<<<grid, 256, 0, c->stream>>>(c->a, seed, d, d + 3, d + 6, d + 9, d + 12);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

static int export_all(mbt_ctx *c) {
  CK(cudaMemcpyAsync(c->xfer, c->a.coord, (size_t)6 * c->npad * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  dim3 grid(16, c->nbunch);
  mbt::add_pending_rw<<<grid, 256, 0, c->stream>>>(c->a, c->xfer);
  CK(cudaGetLastError());
  return 0;
}

int mbt_get_particles(mbt_ctx *c, int ibunch, double *soa6, int np) {
  if (!c || !soa6) return MBT_ERR_INVALID;
  if (ibunch < 0 || ibunch >= c->nbunch) return fail(c, MBT_ERR_INVALID, "bunch %d out of range", ibunch);
  if (np != c->np[ibunch]) return fail(c, MBT_ERR_INVALID, "bunch %d holds %d particles, got %d", ibunch, c->np[ibunch], np);
  int r = export_all(c);
  if (r) return r;
  for (int k = 0; k < 6; ++k)
    CK(cudaMemcpyAsync(soa6 + (size_t)k * np, c->xfer + (size_t)k * c->npad + c->off[ibunch],
                       np * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

// The reverse of mbt_load_all: a kernel writes the beam (with the pending
// resistive-wall kick, as export_all) into the staging buffer in host
// layout, then one copy.
int mbt_get_all(mbt_ctx *c, double *soa6_all) {
  if (!c || !soa6_all) return MBT_ERR_INVALID;
  long total = 0;
  for (int n : c->np) total += n;
  mbt::beam_export<<<dim3(16, c->nbunch), 256, 0, c->stream>>>(c->a, c->pack, c->xfer);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(soa6_all, c->xfer, (size_t)6 * total * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int mbt_get_stats(mbt_ctx *c, double *stats) {
  if (!c || !stats) return MBT_ERR_INVALID;
  int r = export_all(c);
  if (r) return r;
  if (!c->stat_scratch) {
    int npmax = 1;
    for (int n : c->np) npmax = std::max(npmax, n);
    r = dalloc(c, &c->stat_scratch, mbt::stats_scratch_doubles(npmax));
    if (r) return r;
  }
  for (int b = 0; b < c->nbunch; ++b) {
    r = mbt::bunch_stats_strided(c->np[b], c->xfer + c->off[b], (size_t)c->npad, c->p.track_plane, stats + 12 * b,
                                 c->stream, c->stat_scratch);
    if (r) return fail(c, r, "statistics of bunch %d: %s", b, cudaGetErrorString(cudaGetLastError()));
  }
  return 0;
}

int mbt_watch_potentials(mbt_ctx *c, int n, const int *ibunch) {
  if (!c || n < 0 || n > MBT_MAX_WATCH || (n > 0 && !ibunch))
    return c ? fail(c, MBT_ERR_INVALID, "watch list: 0..%d bunches", MBT_MAX_WATCH) : MBT_ERR_INVALID;
  if (c->prepared) return fail(c, MBT_ERR_STATE, "mbt_watch_potentials must precede mbt_prepare");
  if (!c->watch.empty() || c->a.pot) return fail(c, MBT_ERR_STATE, "potentials are already watched");
  if (n == 0) return 0;
  std::vector<int> slot(c->nbunch, -1);
  for (int i = 0; i < n; ++i) {
    if (ibunch[i] < 0 || ibunch[i] >= c->nbunch) return fail(c, MBT_ERR_INVALID, "bunch %d out of range", ibunch[i]);
    if (slot[ibunch[i]] >= 0) return fail(c, MBT_ERR_INVALID, "bunch %d listed twice", ibunch[i]);
    slot[ibunch[i]] = i;
  }
  double *pot = nullptr;
  int *ps = nullptr;
  int r = dalloc(c, &pot, (size_t)n * 7 * c->nc);
  if (!r) r = dupload(c, &ps, slot.data(), slot.size());
  if (r) return r;
  c->a.pot = pot;
  c->a.pot_slot = ps;
  c->watch.assign(ibunch, ibunch + n);
  if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; c->graph_turns = 0; }
  return 0;
}

int mbt_get_potentials(mbt_ctx *c, int ibunch, double *pot) {
  if (!c || !pot) return MBT_ERR_INVALID;
  int slot = -1;
  for (size_t i = 0; i < c->watch.size(); ++i)
    if (c->watch[i] == ibunch) slot = (int)i;
  if (slot < 0) return fail(c, MBT_ERR_INVALID, "bunch %d is not watched", ibunch);
  if (!c->prepared) return fail(c, MBT_ERR_STATE, "mbt_prepare has not run");
  CK(cudaStreamSynchronize(c->stream));
  const int nc = c->p.ncell;
  for (int k = 0; k < 7; ++k)
    CK(cudaMemcpy(pot + (size_t)k * nc, c->a.pot + ((size_t)slot * 7 + k) * c->nc, nc * sizeof(double),
                  cudaMemcpyDeviceToHost));
  return 0;
}

int mbt_enable_beam_ion(mbt_ctx *c, const mbt_beam_ion *cfg) {
  if (!c || !cfg) return MBT_ERR_INVALID;
  if (c->prepared) return fail(c, MBT_ERR_STATE, "mbt_enable_beam_ion must precede mbt_prepare");
  if (c->bi_on) return fail(c, MBT_ERR_STATE, "the beam-ion stage is already on");
  const mbt_params *p = &c->p;
  if (!p->track_plane[1] || !p->track_plane[2])
    return fail(c, MBT_ERR_INVALID, "the beam-ion stage needs both transverse planes tracked");
  if (cfg->n_ip < 1 || cfg->n_ip > mbt::kBiMaxIp)
    return fail(c, MBT_ERR_INVALID, "n_ip %d outside 1..%d", cfg->n_ip, mbt::kBiMaxIp);
  if (cfg->ions_per_passage < 1 || cfg->ions_per_passage > (1 << 20))
    return fail(c, MBT_ERR_INVALID, "ions_per_passage %d outside 1..2^20", cfg->ions_per_passage);
  if (!(cfg->gas_A > 0) || !(cfg->pressure >= 0) || !(cfg->sigma_ion >= 0))
    return fail(c, MBT_ERR_INVALID, "gas_A must be positive, pressure and sigma_ion non-negative");
  if (c->nbunch > 65535) return fail(c, MBT_ERR_INVALID, "the beam-ion stage serves up to 65535 bunches");
  if (cfg->surrogate && !(cfg->audit_fraction >= 0.0 && cfg->audit_fraction <= 1.0))
    return fail(c, MBT_ERR_INVALID, "audit_fraction outside 0..1");
  // constants of the reference (def.h:21-26, input.c:1562)
  const double c_light = 2.997925e+08, eps0 = 8.854187817620e-12, e_charge = 1.602e-19, e_mass = 9.1e-31;
  const double r_e = 2.819e-15, mp_o_em = 1.836e3;
  const double gamma = 1957.0 * p->E0;
  const double factF = e_charge / (cfg->gas_A * mp_o_em * e_mass);     // fbi_weakstrong.c:40
  const double n_gas = 3.22e22 * cfg->pressure;                       // fbi_weakstrong.c:24
  const double L_ip = p->Lc / cfg->n_ip;
  mbt::BiArgs &bi = c->bi;
  bi.n_ip = cfg->n_ip;
  bi.n_new = cfg->ions_per_passage;
  // blocks per passage: of 256 ions for the Faddeeva kernels, of 128 (one
  // tensor-core tile) for the learned field
  const int per_block = cfg->surrogate ? 128 : mbt::kBiThreads;
  bi.bpp = (cfg->ions_per_passage + per_block - 1) / per_block;
  bi.audit_threshold = (uint32_t)std::min(4294967295.0, cfg->audit_fraction * 4294967296.0);
  bi.nb = c->nbunch;
  bi.T = (long)c->nbunch * (c->nbunch - 1) / 2;
  bi.dt_bucket = p->T0 / p->nharm;
  bi.kion_per_amp = -factF * p->T0 / (2.0 * eps0 * c_light);
  bi.ke = -2.0 * PI * r_e / gamma;
  bi.w_per_amp = p->T0 / e_charge * cfg->sigma_ion * n_gas * L_ip / cfg->ions_per_passage;
  bi.betaH = p->beta1[1]; bi.alphaH = p->alpha1[1];
  bi.betaV = p->beta1[2]; bi.alphaV = p->alpha1[2];
  bi.keys = mbt::philox_keys(cfg->seed);
  std::vector<double> trig((size_t)4 * cfg->n_ip);
  for (int k = 0; k < cfg->n_ip; ++k) {
    const double mux = 2.0 * PI * p->QH0 * k / cfg->n_ip, muy = 2.0 * PI * p->QV0 * k / cfg->n_ip;
    trig[4 * k] = cos(mux); trig[4 * k + 1] = sin(mux);
    trig[4 * k + 2] = cos(muy); trig[4 * k + 3] = sin(muy);
  }
  std::vector<double> ibv(c->ib.begin(), c->ib.end());
  double *tr = nullptr, *mom = nullptr, *frame = nullptr, *part = nullptr, *cloud = nullptr, *ibd = nullptr;
  const size_t nslot = (size_t)cfg->n_ip * std::max<long>(bi.T, 1) * bi.bpp * 5;
  int r = dupload(c, &tr, trig.data(), trig.size());
  if (!r) r = dalloc(c, &mom, (size_t)c->nbunch * 10);
  if (!r) r = dalloc(c, &frame, (size_t)cfg->n_ip * c->nbunch * 4);
  if (!r) r = dalloc(c, &part, nslot);
  if (!r) r = dalloc(c, &cloud, (size_t)cfg->n_ip * c->nbunch * 5);
  if (!r) r = dupload(c, &ibd, ibv.data(), ibv.size());
  // the bunch currents as they stand (a current scan may have stepped them)
  if (!r) CK(cudaMemcpy(ibd, c->a.bunch_ib, (size_t)c->nbunch * sizeof(double), cudaMemcpyDeviceToDevice));
  unsigned long long *aud = nullptr;
  if (!r) r = dalloc(c, &aud, 6);
  if (r) return r;
  bi.audit = aud;
  if (cfg->surrogate) {
    CK(cudaFuncSetAttribute(mbt::bi_ions_mlp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mbt::kMlpCtaSmem));
    CK(cudaFuncSetAttribute(mbt::bi_kick_mlp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mbt::kMlpCtaSmem));
  }
  CK(cudaFuncSetAttribute(mbt::bi_kick_grouped, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)mbt::bi_kick_grouped_smem(cfg->n_ip)));
  bi.trig = tr; bi.mom = mom; bi.frame = frame; bi.part = part; bi.cloud = cloud; bi.ib = ibd;
  bi.bunch_kb = c->a.bunch_kb;
  bi.turn = &c->a.rs->turn;
  bi.error = &c->a.rs->error;
  c->a.bi_mom = mom;
  if (!c->bi_ev) CK(cudaEventCreate(&c->bi_ev));
  for (cudaEvent_t &e : c->bi_kev)
    if (!e) CK(cudaEventCreate(&e));
  c->bicfg = *cfg;
  c->bi_on = 1;
  if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; c->graph_turns = 0; }
  return 0;
}

int mbt_beam_ion_use_mlp(mbt_ctx *c, mbt_mlp *m) {
  if (!c || !m) return MBT_ERR_INVALID;
  c->mlp = mbt::mlp_device_view(m);
  c->mlp_set = true;
  if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; c->graph_turns = 0; }
  return 0;
}

int mbt_beam_ion_audit(mbt_ctx *c, double out[5]) {
  if (!c || !out) return MBT_ERR_INVALID;
  if (!c->bi_on) return fail(c, MBT_ERR_STATE, "the beam-ion stage is off");
  unsigned long long h[6];
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(h, c->bi.audit, sizeof h, cudaMemcpyDeviceToHost));
  CK(cudaMemset(c->bi.audit, 0, sizeof h));
  double sq;
  memcpy(&sq, &h[4], sizeof sq);
  double mx;
  memcpy(&mx, &h[1], sizeof mx);
  out[0] = (double)h[0];
  out[1] = h[0] ? mx : 0.0;
  out[2] = h[0] ? sqrt(sq / (double)h[0]) : 0.0;
  out[3] = (double)h[2];
  out[4] = (double)h[3];
  return 0;
}

int mbt_beam_ion_clouds(mbt_ctx *c, double *clouds) {
  if (!c || !clouds) return MBT_ERR_INVALID;
  if (!c->bi_on) return fail(c, MBT_ERR_STATE, "the beam-ion stage is off");
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(clouds, c->bi.cloud, (size_t)c->bi.n_ip * c->nbunch * 5 * sizeof(double), cudaMemcpyDeviceToHost));
  return 0;
}

int mbt_beam_ion_timing(mbt_ctx *c, double *ms_per_turn) {
  if (!c || !ms_per_turn) return MBT_ERR_INVALID;
  *ms_per_turn = c->bi_on ? c->bi_ms : 0.0;
  return 0;
}

int mbt_gauss_field_dev(long n, const double *dx, const double *dy, const double *sx, const double *sy, double *gx,
                        double *gy, void *stream) {
  if (n < 0 || (n > 0 && (!dx || !dy || !sx || !sy || !gx || !gy)))
    return mbt::fail_global(MBT_ERR_INVALID, "bad gauss_field arguments");
  if (n == 0) return 0;
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || nd == 0)
    return mbt::fail_global(MBT_ERR_NODEVICE, "no CUDA device: libmbt has no CPU path");
  const int blocks = (int)std::min<long>((n + 255) / 256, 148L * 16);
  mbt::gauss_field_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(n, dx, dy, sx, sy, gx, gy);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return mbt::fail_global(MBT_ERR_CUDA, "gauss_field: %s", cudaGetErrorString(e));
  return 0;
}

int mbt_prepare(mbt_ctx *c, double *init_stats) {
  if (!c) return MBT_ERR_INVALID;
  Args &a = c->a;
  mbt::init_shift<<<(c->nbunch + 255) / 256, 256, 0, c->stream>>>(a);
  launch_map_noise<false>(c, MBT_NOISE_NONE);
  mbt::bunch_reduce<<<c->nbunch, mbt::kBlock, smem_reduce(c), c->stream>>>(a, mbt::kReducePrologue, c->stats_init);
  if (c->nlr > 0 && c->p.lr_init_turns > 0)
    mbt::ring_scan<<<1, mbt::kBlock, smem_scan(c), c->stream>>>(a, c->p.lr_init_turns, 1, c->vbuf);
  mbt::ring_scan<<<1, mbt::kBlock, smem_scan(c), c->stream>>>(a, 1, 0, c->vbuf);
  mbt::bunch_wakes<<<c->nbunch, mbt::kBlock, smem_wakes(c), c->stream>>>(a, 0);
  CK(cudaGetLastError());
  int r = sync_and_check(c);
  if (r) return r;
  if (init_stats)
    CK(cudaMemcpy(init_stats, c->stats_init, (size_t)c->nbunch * 12 * sizeof(double), cudaMemcpyDeviceToHost));
  c->prepared = 1;
  return 0;
}

int mbt_set_deviates(mbt_ctx *c, const float *dev, long nturns) {
  if (!c || !dev || nturns <= 0) return MBT_ERR_INVALID;
  if (c->noise != MBT_NOISE_INJECTED) return fail(c, MBT_ERR_STATE, "context was not created with MBT_NOISE_INJECTED");
  const int per = 1 + 2 * (c->p.track_plane[2] != 0) + 2 * (c->p.track_plane[1] != 0);
  const size_t need = (size_t)nturns * 5 * c->npad;
  if (need > c->dev_cap) {
    if (c->dev) cudaFree(c->dev);
    c->dev = nullptr;
    c->dev_cap = 0;
    CK(cudaMalloc(&c->dev, need * sizeof(float)));
    c->dev_cap = need;
  }
  std::vector<float> h(need, 0.0f);
  size_t src = 0;
  for (long t = 0; t < nturns; ++t) {
    float *T = h.data() + (size_t)t * 5 * c->npad;
    for (int b = 0; b < c->nbunch; ++b) {
      const int n = c->np[b], o = c->off[b];
      for (int j = 0; j < n; ++j) T[o + j] = dev[src + j];
      size_t q = src + n;
      if (c->p.track_plane[2]) {
        for (int j = 0; j < n; ++j) {
          T[(size_t)1 * c->npad + o + j] = dev[q + 2 * j];
          T[(size_t)2 * c->npad + o + j] = dev[q + 2 * j + 1];
        }
        q += 2 * (size_t)n;
      }
      if (c->p.track_plane[1]) {
        for (int j = 0; j < n; ++j) {
          T[(size_t)3 * c->npad + o + j] = dev[q + 2 * j];
          T[(size_t)4 * c->npad + o + j] = dev[q + 2 * j + 1];
        }
      }
      src += (size_t)per * n;
    }
  }
  CK(cudaMemcpy(c->dev, h.data(), need * sizeof(float), cudaMemcpyHostToDevice));
  RingState rs;
  CK(cudaMemcpy(&rs, c->a.rs, sizeof rs, cudaMemcpyDeviceToHost));
  c->a.dev = c->dev;
  c->a.dev_turn0 = rs.turn;
  c->a.dev_nturn = nturns;
  if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; c->graph_turns = 0; }
  return 0;
}

static int run_core(mbt_ctx *c, long nturns, double *stats, double *ampinv, bool use_graph) {
  if (!c->prepared) return fail(c, MBT_ERR_STATE, "mbt_prepare must come first");
  if (c->bi_on && c->bicfg.surrogate && !c->mlp_set)
    return fail(c, MBT_ERR_STATE, "surrogate beam-ion fields need mbt_beam_ion_use_mlp");
  RingState rs;
  CK(cudaMemcpy(&rs, c->a.rs, sizeof rs, cudaMemcpyDeviceToHost));
  long turn = rs.turn;
  const long cap = c->a.stats_cap;
  long done = 0;
  // The statistics (and amplitude invariants) leave the device one unit of
  // turns at a time (a graph of 8 turns, or a single turn) on the copy
  // stream, each copy behind the turns that write it and beside the turns
  // that follow.  A unit's copy is issued only after the next unit has been
  // enqueued: a copy into pageable host memory returns when it is complete,
  // and the GPU keeps busy with that next unit meanwhile.  Before a pass
  // over the statistics ring starts again at slot 0, every copy is issued
  // and the turns wait for them, so that no slot is overwritten before it
  // has been copied.
  const size_t row = (size_t)c->nbunch;
  struct Unit { long done, slot, n; int ev; };
  Unit pend[2] = {};
  int npend = 0;
  auto issue = [&](const Unit &u) -> int {
    CK(cudaStreamWaitEvent(c->copy_stream, c->cev[u.ev], 0));
    if (stats)
      CK(cudaMemcpyAsync(stats + (size_t)u.done * row * 12, c->a.stats + (size_t)u.slot * row * 12,
                         (size_t)u.n * row * 12 * sizeof(double), cudaMemcpyDeviceToHost, c->copy_stream));
    if (ampinv)
      CK(cudaMemcpyAsync(ampinv + (size_t)u.done * row * 6, c->a.ampinv + (size_t)u.slot * row * 6,
                         (size_t)u.n * row * 6 * sizeof(double), cudaMemcpyDeviceToHost, c->copy_stream));
    return 0;
  };
  auto unit_enqueued = [&](long at_done, long slot, long n) -> int {
    if (!stats && !ampinv) return 0;
    const int ev = npend == 0 ? 0 : 1 - pend[npend - 1].ev;
    CK(cudaEventRecord(c->cev[ev], c->stream));
    if (npend == 2) {
      int r = issue(pend[0]);
      if (r) return r;
      pend[0] = pend[1];
      npend = 1;
    }
    pend[npend++] = Unit{at_done, slot, n, ev};
    return 0;
  };
  auto flush = [&]() -> int {
    for (int i = 0; i < npend; ++i) {
      int r = issue(pend[i]);
      if (r) return r;
    }
    npend = 0;
    if (stats || ampinv) {
      CK(cudaEventRecord(c->cev[2], c->copy_stream));
      CK(cudaStreamWaitEvent(c->stream, c->cev[2], 0));
    }
    return 0;
  };
  // The caller's buffers are pinned for the call when they are pageable
  // (and pinning is allowed), so that the copies run as asynchronous DMA;
  // otherwise each copy returns when complete, as described above.
  auto pin = [&](double *p, size_t bytes) -> bool {
    if (!p || bytes == 0) return false;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    if (at.type != cudaMemoryTypeUnregistered) return false;   // already pinned or device memory
    if (cudaHostRegister(p, bytes, cudaHostRegisterDefault) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    return true;
  };
  const bool pinned_s = pin(stats, (size_t)nturns * row * 12 * sizeof(double));
  const bool pinned_a = pin(ampinv, (size_t)nturns * row * 6 * sizeof(double));
  struct Unpin {   // on every return: no copy into the buffers left in flight, then unpin
    mbt_ctx *c;
    double *s, *a;
    ~Unpin() {
      if (!s && !a) return;
      cudaStreamSynchronize(c->stream);
      cudaStreamSynchronize(c->copy_stream);
      if (s) cudaHostUnregister(s);
      if (a) cudaHostUnregister(a);
      cudaGetLastError();
    }
  } unpin{c, pinned_s ? stats : nullptr, pinned_a ? ampinv : nullptr};
  CK(cudaEventRecord(c->ev[5], c->stream));
  while (done < nturns) {
    // a chunk never crosses a wrap of the statistics buffer, and ends at
    // the next scan boundary
    const long slot = turn % cap;
    long chunk = std::min(nturns - done, cap - slot);
    bool boundary = false;
    if (c->scan_steps) {
      const long left = c->p.nrev_scan - turn % c->p.nrev_scan;   // turns up to the boundary, inclusive
      if (left <= chunk) { chunk = left; boundary = true; }
    }
    if (slot == 0 && done > 0) {
      int r = flush();
      if (r) return r;
    }
    const long plain = boundary ? chunk - 1 : chunk;
    long t = 0;
    int r = 0;
    if (use_graph && plain >= 8) {
      const int G = 8;
      r = build_graph(c, G);
      if (r) return r;
      for (; t + G <= plain && !r; t += G) {
        CK(cudaGraphLaunch(c->graph, c->stream));
        r = unit_enqueued(done + t, slot + t, G);
      }
    }
    for (; t < plain && !r; ++t) {
      enqueue_turn(c, nullptr);
      r = unit_enqueued(done + t, slot + t, 1);
    }
    if (boundary && !r) {
      enqueue_turn(c, nullptr, true);
      r = unit_enqueued(done + t, slot + t, 1);
    }
    if (r) return r;
    CK(cudaGetLastError());
    done += chunk;
    turn += chunk;
  }
  {
    int r = flush();
    if (r) return r;
  }
  CK(cudaEventRecord(c->ev[4], c->stream));
  int r = sync_and_check(c);
  if (r) return r;
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev[5], c->ev[4]);
  c->timing[3] = ms;
  return 0;
}

int mbt_run_turns(mbt_ctx *c, long nturns, double *stats) {
  if (!c || nturns < 0) return MBT_ERR_INVALID;
  return run_core(c, nturns, stats, nullptr, true);
}

int mbt_run_turns_ampinv(mbt_ctx *c, long nturns, double *stats, double *ampinv) {
  if (!c || nturns < 0) return MBT_ERR_INVALID;
  return run_core(c, nturns, stats, ampinv, true);
}

int mbt_track(mbt_ctx *c, double *particles, long nturns, double *stats) {
  if (!c || !particles || nturns < 0) return MBT_ERR_INVALID;
  int r = mbt_load_all(c, particles);
  if (r) return r;
  if (!c->prepared) { r = mbt_prepare(c, nullptr); if (r) return r; }
  r = run_core(c, nturns, stats, nullptr, true);
  if (r) return r;
  return mbt_get_all(c, particles);
}

// Per-kernel device times of nturns turns launched one by one with CUDA
// events between the kernels: out[0..3] = average ms per turn of the
// particle pass, bunch reduction, ring scan, bunch wakes.
int mbt_profile_turns(mbt_ctx *c, long nturns, double out[4]) {
  if (!c || nturns <= 0 || !out) return MBT_ERR_INVALID;
  if (!c->prepared) return fail(c, MBT_ERR_STATE, "mbt_prepare must come first");
  if (c->bi_on && c->bicfg.surrogate && !c->mlp_set)
    return fail(c, MBT_ERR_STATE, "surrogate beam-ion fields need mbt_beam_ion_use_mlp");
  double acc[4] = {0, 0, 0, 0}, acc_bi = 0.0, acc_k[4] = {0, 0, 0, 0};
  RingState rs;
  CK(cudaMemcpy(&rs, c->a.rs, sizeof rs, cudaMemcpyDeviceToHost));
  // the turns run back to back, as in mbt_run_turns, with their own events
  // between the kernels (5 per turn, 4 more for the beam-ion stage)
  const int per = 5 + (c->bi_on ? 4 : 0);
  struct Events {
    std::vector<cudaEvent_t> e;
    ~Events() {
      for (cudaEvent_t x : e)
        if (x) cudaEventDestroy(x);
    }
  } E;
  E.e.assign((size_t)nturns * per, nullptr);
  for (auto &x : E.e) CK(cudaEventCreate(&x));
  const cudaEvent_t keep_kev[3] = {c->bi_kev[0], c->bi_kev[1], c->bi_kev[2]}, keep_bi = c->bi_ev;
  for (long t = 0; t < nturns; ++t) {
    cudaEvent_t *ev = &E.e[(size_t)t * per];
    if (c->bi_on) {
      for (int k = 0; k < 3; ++k) c->bi_kev[k] = ev[5 + k];
      c->bi_ev = ev[8];
    }
    enqueue_turn(c, ev, scan_boundary(c, rs.turn + t));
  }
  for (int k = 0; k < 3; ++k) c->bi_kev[k] = keep_kev[k];
  c->bi_ev = keep_bi;
  int r = sync_and_check(c);
  if (r) return r;
  for (long t = 0; t < nturns; ++t) {
    const cudaEvent_t *ev = &E.e[(size_t)t * per];
    float ms = 0;
    for (int k = 0; k < 4; ++k) {
      cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
      acc[k] += ms;
    }
    if (c->bi_on) {
      cudaEventElapsedTime(&ms, ev[4], ev[8]);
      acc_bi += ms;
      const cudaEvent_t seq[5] = {ev[4], ev[5], ev[6], ev[7], ev[8]};
      for (int k = 0; k < 4; ++k) {
        cudaEventElapsedTime(&ms, seq[k], seq[k + 1]);
        acc_k[k] += ms;
      }
    }
  }
  for (int k = 0; k < 4; ++k) out[k] = acc[k] / nturns;
  c->bi_ms = acc_bi / nturns;
  for (int k = 0; k < 4; ++k) c->bi_kms[k] = acc_k[k] / nturns;
  return 0;
}

int mbt_beam_ion_kernel_times(mbt_ctx *c, double ms_per_turn[4]) {
  if (!c || !ms_per_turn) return MBT_ERR_INVALID;
  for (int k = 0; k < 4; ++k) ms_per_turn[k] = c->bi_on ? c->bi_kms[k] : 0.0;
  return 0;
}

int mbt_inject_device_error(mbt_ctx *c, int bits) {
  if (!c || bits <= 0) return MBT_ERR_INVALID;
  RingState rs;
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(&rs, c->a.rs, sizeof rs, cudaMemcpyDeviceToHost));
  rs.error |= bits;
  CK(cudaMemcpy(&c->a.rs->error, &rs.error, sizeof rs.error, cudaMemcpyHostToDevice));
  return 0;
}

int mbt_get_state(mbt_ctx *c, mbt_state *st) {
  if (!c || !st) return MBT_ERR_INVALID;
  RingState rs;
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(&rs, c->a.rs, sizeof rs, cudaMemcpyDeviceToHost));
  memset(st, 0, sizeof *st);
  // The device runs one ring scan ahead (it prepares the next turn's
  // wakes and RF correction); report the values of the last completed
  // turn, as the reference holds them after that turn.
  const bool ahead = c->prepared != 0;
  st->turn = rs.turn;
  st->Vrf0 = ahead ? rs.Vrf0_last : rs.Vrf0;
  st->phai0 = ahead ? rs.phai0_last : rs.phai0;
  for (int pl = 0; pl < 3; ++pl)
    for (int l = 0; l < MBT_MAX_LR; ++l)
      for (int k = 0; k < 2; ++k) st->phasor[pl][l][k] = ahead ? rs.phasor_last[pl][l][k] : rs.phasor[pl][l][k];
  st->n_trash_low = rs.trash_low;
  st->n_trash_high = rs.trash_high;
  return 0;
}

int mbt_get_histograms(mbt_ctx *c, int ibunch, double *fnp, double *dipV, double *dipH, double *ring_lon,
                       double *ring_hor, double *ring_ver) {
  if (!c) return MBT_ERR_INVALID;
  if (ibunch < 0 || ibunch >= c->nbunch) return fail(c, MBT_ERR_INVALID, "bunch %d out of range", ibunch);
  std::vector<double> h((size_t)6 * c->nc);
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(h.data(), c->a.hist + (size_t)ibunch * 6 * c->nc, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
  double *dst[6] = {fnp, dipV, dipH, ring_lon, ring_hor, ring_ver};
  for (int k = 0; k < 6; ++k)
    if (dst[k]) memcpy(dst[k], h.data() + (size_t)k * c->nc, c->p.ncell * sizeof(double));
  return 0;
}

int mbt_last_timing(mbt_ctx *c, double out[4], int *launches_per_turn) {
  if (!c || !out) return MBT_ERR_INVALID;
  for (int k = 0; k < 4; ++k) out[k] = c->timing[k];
  if (launches_per_turn) *launches_per_turn = 4;
  return 0;
}

int mbt_set_tiles(mbt_ctx *c, const int tile[3]) {
  if (!c || !tile) return MBT_ERR_INVALID;
  for (int k = 0; k < 3; ++k)
    if (tile[k] < 512 || tile[k] > 8192 || (tile[k] & (tile[k] - 1)))
      return fail(c, MBT_ERR_INVALID, "tile sizes are powers of two in 512..8192 (class %d: %d)", k, tile[k]);
  for (int k = 0; k < 3; ++k) c->class_tile[k] = tile[k];
  layout_tiles(c);
  if (c->ntile > c->tile_cap) return fail(c, MBT_ERR_INVALID, "tile table overflow");
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(const_cast<Tile *>(c->a.tiles), c->tiles.data(), c->tiles.size() * sizeof(Tile),
                cudaMemcpyHostToDevice));
  CK(cudaMemcpy(const_cast<int *>(c->a.bunch_tile0), c->tile0.data(), c->nbunch * sizeof(int),
                cudaMemcpyHostToDevice));
  CK(cudaMemcpy(const_cast<int *>(c->a.bunch_ntile), c->ntiles.data(), c->nbunch * sizeof(int),
                cudaMemcpyHostToDevice));
  c->a.ntile = c->ntile;
  c->a.tile = c->tile;
  if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; c->graph_turns = 0; }
  return 0;
}

int mbt_autotune(mbt_ctx *c, int trial_turns, int tile_out[3]) {
  if (!c || trial_turns < 1) return MBT_ERR_INVALID;
  if (!c->prepared) return fail(c, MBT_ERR_STATE, "mbt_prepare must come first");
  bool present[3] = {false, false, false};
  for (int b = 0; b < c->nbunch; ++b) present[size_class(c->np[b])] = true;
  int best[3] = {c->class_tile[0], c->class_tile[1], c->class_tile[2]};
  auto trial = [&](const int *t, double *ms) {
    int r = mbt_set_tiles(c, t);
    if (r) return r;
    r = run_core(c, 1, nullptr, nullptr, true);   // graph build and warm-up
    if (r) return r;
    r = run_core(c, trial_turns, nullptr, nullptr, true);
    *ms = c->timing[3];
    return r;
  };
  double best_ms = 0.0;
  int r = trial(best, &best_ms);
  if (r) return r;
  // one pass of coordinate descent over the classes present
  for (int k = 0; k < 3; ++k) {
    if (!present[k]) continue;
    for (int T = 512; T <= 8192; T <<= 1) {
      if (T == best[k]) continue;
      int cand[3] = {best[0], best[1], best[2]};
      cand[k] = T;
      double ms = 0.0;
      r = trial(cand, &ms);
      if (r) return r;
      if (ms < best_ms) {
        best_ms = ms;
        best[k] = T;
      }
    }
  }
  r = mbt_set_tiles(c, best);
  if (r) return r;
  if (tile_out)
    for (int k = 0; k < 3; ++k) tile_out[k] = best[k];
  return 0;
}

int mbt_geometry(mbt_ctx *c, int *npad, int *tile, int *ntile) {
  if (!c) return MBT_ERR_INVALID;
  if (npad) *npad = c->npad;
  if (tile) *tile = c->tile;
  if (ntile) *ntile = c->ntile;
  return 0;
}

// ---- per-step device entry points

}  // extern "C"

// ---- checkpoint / resume

namespace {

constexpr char kCkptMagic[8] = {'M', 'B', 'T', 'C', 'K', 'P', 'T', '1'};
constexpr uint32_t kCkptVersion = 2;   // 2: the pending resistive-wall kick as one record per bunch

uint64_t fnv1a(uint64_t h, const void *p, size_t n) {
  const unsigned char *b = static_cast<const unsigned char *>(p);
  for (size_t i = 0; i < n; ++i) {
    h ^= b[i];
    h *= 1099511628211ull;
  }
  return h;
}

// What must match between the context that wrote a checkpoint and the one
// that reads it: geometry, fill, noise key and which optional stages exist.
struct CkptKey {
  int32_t nbunch, npad, ntile, ncell, nlr, nharm, Nmlt, rw_long, rffb_len, noise, stats_cap, nwatch, bi_on;
  int32_t pad0;
  uint64_t seed;
  uint64_t fill_hash;   // buckets, macroparticle counts, tiles
};

CkptKey ckpt_key(const mbt_ctx *c) {
  CkptKey k{};
  k.nbunch = c->nbunch; k.npad = c->npad; k.ntile = c->ntile; k.ncell = c->nc; k.nlr = c->nlr;
  k.nharm = c->p.nharm; k.Nmlt = c->p.Nmlt; k.rw_long = c->p.rw_long; k.rffb_len = c->a.rffb_len;
  k.noise = c->noise; k.stats_cap = c->a.stats_cap; k.nwatch = (int)c->watch.size(); k.bi_on = c->bi_on;
  k.seed = c->seed;
  uint64_t h = 1469598103934665603ull;
  h = fnv1a(h, c->bucket.data(), c->bucket.size() * sizeof(int));
  h = fnv1a(h, c->np.data(), c->np.size() * sizeof(int));
  for (const Tile &t : c->tiles) {
    const int32_t v[3] = {t.bunch, t.start, t.count};
    h = fnv1a(h, v, sizeof v);
  }
  k.fill_hash = h;
  return k;
}

// The device buffers that carry state from one turn to the next (ids are
// part of the file format), with their allocated sizes.
struct CkptBuf {
  uint32_t id;
  void *ptr;
  size_t bytes;
};

std::vector<CkptBuf> ckpt_buffers(const mbt_ctx *c) {
  const Args &a = c->a;
  const void *list[] = {a.coord, a.bunch_ib, a.bunch_factg, a.ibunch, a.rw_ib, a.part, a.shift, a.hist, a.cellrange,
                        a.kick, a.rw_part, a.lr_u, a.lr_b, a.lr_vs, a.dipole, a.rw_e, a.rffb_hist, a.rs, a.pot,
                        a.bi_mom, a.stats, a.ampinv, c->stats_init};
  std::vector<CkptBuf> out;
  for (uint32_t id = 0; id < sizeof list / sizeof list[0]; ++id) {
    const void *p = list[id];
    if (!p) continue;
    bool dup = false;
    for (const CkptBuf &b : out) dup = dup || b.ptr == p;
    if (dup) continue;   // rw_ib is ibunch unless a current scan runs with the wall
    for (size_t i = 0; i < c->allocs.size(); ++i)
      if (c->allocs[i] == p) out.push_back({id, const_cast<void *>(p), c->alloc_bytes[i]});
  }
  return out;
}

struct CkptHeader {
  char magic[8];
  uint32_t version, nbuf;
  CkptKey key;
};

// Reads and checks a whole checkpoint file: magic, version, sizes, checksum.
int ckpt_read(const char *path, std::vector<char> &data, CkptHeader &h, char *err) {
  FILE *f = fopen(path, "rb");
  if (!f) { snprintf(err, 512, "checkpoint %s: cannot open", path); return MBT_ERR_IO; }
  fseek(f, 0, SEEK_END);
  const long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  if (n < (long)(sizeof(CkptHeader) + sizeof(uint64_t))) {
    fclose(f);
    snprintf(err, 512, "checkpoint %s: truncated (%ld bytes)", path, n);
    return MBT_ERR_IO;
  }
  data.resize((size_t)n);
  const size_t got = fread(data.data(), 1, (size_t)n, f);
  fclose(f);
  if (got != (size_t)n) { snprintf(err, 512, "checkpoint %s: read error", path); return MBT_ERR_IO; }
  memcpy(&h, data.data(), sizeof h);
  if (memcmp(h.magic, kCkptMagic, 8) != 0 || h.version != kCkptVersion) {
    snprintf(err, 512, "checkpoint %s: not an mbt checkpoint of version %u", path, kCkptVersion);
    return MBT_ERR_IO;
  }
  uint64_t sum;
  memcpy(&sum, data.data() + n - sizeof sum, sizeof sum);
  if (fnv1a(1469598103934665603ull, data.data(), (size_t)n - sizeof sum) != sum) {
    snprintf(err, 512, "checkpoint %s: checksum mismatch (truncated or corrupted)", path);
    return MBT_ERR_IO;
  }
  // walk the records: each one must lie inside the file
  size_t off = sizeof h;
  for (uint32_t i = 0; i < h.nbuf; ++i) {
    uint32_t id;
    uint64_t bytes;
    if (off + sizeof id + sizeof bytes > (size_t)n - sizeof sum) {
      snprintf(err, 512, "checkpoint %s: record %u runs past the end", path, i);
      return MBT_ERR_IO;
    }
    memcpy(&id, data.data() + off, sizeof id);
    memcpy(&bytes, data.data() + off + sizeof id, sizeof bytes);
    off += sizeof id + sizeof bytes;
    if (bytes > (size_t)n - sizeof sum - off) {
      snprintf(err, 512, "checkpoint %s: record %u runs past the end", path, i);
      return MBT_ERR_IO;
    }
    off += bytes;
  }
  if (off != (size_t)n - sizeof sum) {
    snprintf(err, 512, "checkpoint %s: trailing bytes", path);
    return MBT_ERR_IO;
  }
  return 0;
}

}  // namespace

extern "C" {

int mbt_checkpoint_save(mbt_ctx *c, const char *path) {
  if (!c || !path) return MBT_ERR_INVALID;
  if (!c->prepared) return fail(c, MBT_ERR_STATE, "mbt_checkpoint_save: mbt_prepare must come first");
  CK(cudaStreamSynchronize(c->stream));
  const std::vector<CkptBuf> bufs = ckpt_buffers(c);
  CkptHeader h{};
  memcpy(h.magic, kCkptMagic, 8);
  h.version = kCkptVersion;
  h.nbuf = (uint32_t)bufs.size();
  h.key = ckpt_key(c);
  size_t total = sizeof h;
  for (const CkptBuf &b : bufs) total += sizeof(uint32_t) + sizeof(uint64_t) + b.bytes;
  std::vector<char> data(total + sizeof(uint64_t));
  memcpy(data.data(), &h, sizeof h);
  size_t off = sizeof h;
  for (const CkptBuf &b : bufs) {
    const uint64_t bytes = b.bytes;
    memcpy(data.data() + off, &b.id, sizeof b.id);
    memcpy(data.data() + off + sizeof b.id, &bytes, sizeof bytes);
    off += sizeof b.id + sizeof bytes;
    CK(cudaMemcpy(data.data() + off, b.ptr, b.bytes, cudaMemcpyDeviceToHost));
    off += b.bytes;
  }
  const uint64_t sum = fnv1a(1469598103934665603ull, data.data(), total);
  memcpy(data.data() + total, &sum, sizeof sum);
  // write beside the target, then rename: a reader never sees half a file
  std::string tmp = std::string(path) + ".tmp";
  FILE *f = fopen(tmp.c_str(), "wb");
  if (!f) return fail(c, MBT_ERR_IO, "mbt_checkpoint_save: cannot create %s", tmp.c_str());
  const bool ok = fwrite(data.data(), 1, data.size(), f) == data.size();
  if (fclose(f) != 0 || !ok) {
    remove(tmp.c_str());
    return fail(c, MBT_ERR_IO, "mbt_checkpoint_save: write error on %s", tmp.c_str());
  }
  if (rename(tmp.c_str(), path) != 0) {
    remove(tmp.c_str());
    return fail(c, MBT_ERR_IO, "mbt_checkpoint_save: cannot rename %s", tmp.c_str());
  }
  return 0;
}

int mbt_checkpoint_load(mbt_ctx *c, const char *path) {
  if (!c || !path) return MBT_ERR_INVALID;
  if (!c->prepared) return fail(c, MBT_ERR_STATE, "mbt_checkpoint_load: mbt_prepare must come first");
  std::vector<char> data;
  CkptHeader h{};
  int r = ckpt_read(path, data, h, c->err);
  if (r) return r;
  const CkptKey k = ckpt_key(c);
  if (memcmp(&k, &h.key, sizeof k) != 0)
    return fail(c, MBT_ERR_STATE, "mbt_checkpoint_load: %s was written by a context of another configuration "
                "(fill, geometry, noise key, watched bunches or beam-ion stage differ)", path);
  const std::vector<CkptBuf> bufs = ckpt_buffers(c);
  if (bufs.size() != h.nbuf) return fail(c, MBT_ERR_STATE, "mbt_checkpoint_load: %s holds %u buffers, this context %zu",
                                         path, h.nbuf, bufs.size());
  // check every record against this context before the first device write
  size_t off = sizeof h;
  std::vector<size_t> at(bufs.size());
  for (size_t i = 0; i < bufs.size(); ++i) {
    uint32_t id;
    uint64_t bytes;
    memcpy(&id, data.data() + off, sizeof id);
    memcpy(&bytes, data.data() + off + sizeof id, sizeof bytes);
    off += sizeof id + sizeof bytes;
    if (id != bufs[i].id || bytes != bufs[i].bytes)
      return fail(c, MBT_ERR_STATE, "mbt_checkpoint_load: %s record %zu (buffer %u, %llu bytes) does not match "
                  "this context (buffer %u, %zu bytes)", path, i, id, (unsigned long long)bytes, bufs[i].id,
                  bufs[i].bytes);
    at[i] = off;
    off += bytes;
  }
  CK(cudaStreamSynchronize(c->stream));
  for (size_t i = 0; i < bufs.size(); ++i)
    CK(cudaMemcpy(bufs[i].ptr, data.data() + at[i], bufs[i].bytes, cudaMemcpyHostToDevice));
  if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; c->graph_turns = 0; }
  return 0;
}

int mbt_checkpoint_check(const char *path, long *turn, int *nbunch) {
  std::vector<char> data;
  CkptHeader h{};
  char err[512];
  if (!path) return MBT_ERR_INVALID;
  int r = ckpt_read(path, data, h, err);
  if (r) {
    snprintf(g_create_error, sizeof g_create_error, "%s", err);
    return r;
  }
  if (nbunch) *nbunch = h.key.nbunch;
  if (turn) {
    // the ring state record (id 17) holds the turn count first
    size_t off = sizeof h;
    *turn = -1;
    for (uint32_t i = 0; i < h.nbuf; ++i) {
      uint32_t id;
      uint64_t bytes;
      memcpy(&id, data.data() + off, sizeof id);
      memcpy(&bytes, data.data() + off + sizeof id, sizeof bytes);
      off += sizeof id + sizeof bytes;
      if (id == 17 && bytes >= sizeof(long)) memcpy(turn, data.data() + off, sizeof(long));
      off += bytes;
    }
  }
  return 0;
}

}  // extern "C"
