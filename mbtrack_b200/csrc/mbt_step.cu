// mbt_step.cu -- per-step device entry points on caller-owned device data.
//
// mbt_bunch_moments_dev: statistics and binning of one bunch
// (weak_bunch_mean_rms statistics.c:91-128 for every tracked plane, and the
// in-range histograms of fnp_ring_update transform_weak.c:838-865) in two
// kernels: block partial records, then one block that reduces them in a
// fixed order.  The partial records are scratch memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>

#include "mbt.h"
#include "mbt_common.cuh"

namespace mbt {
int fail_global(int code, const char *fmt, ...);
}

namespace {

constexpr int kThreads = 256;
constexpr int kExtra = 12;           // 6 shifted sums, 6 shifted sums of squares

// Record of one block: counts[nc], sum x[nc], sum z[nc], kExtra sums.
__global__ void __launch_bounds__(kThreads)
moments_partial(int np, const double *__restrict__ c, size_t ld, double sgm, double nsig, double dT, int nc,
                double *__restrict__ part, int prec) {
  extern __shared__ double sh[];
  // x and z sums per bin as fixed-point (hi, lo) integer pairs
  unsigned long long *fxh = reinterpret_cast<unsigned long long *>(sh);
  unsigned long long *fxl = fxh + nc, *fzh = fxh + 2 * nc, *fzl = fxh + 3 * nc;
  int *hc = reinterpret_cast<int *>(sh + 4 * nc);
  __shared__ double red[kThreads / 32][kExtra];
  for (int i = threadIdx.x; i < nc; i += kThreads) {
    fxh[i] = fxl[i] = fzh[i] = fzl[i] = 0ull;
    hc[i] = 0;
  }
  __syncthreads();
  const size_t n6 = ld;
  double s[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) s[k] = c[k * n6];   // shift: the first particle
  double ms[6] = {0, 0, 0, 0, 0, 0}, mq[6] = {0, 0, 0, 0, 0, 0};
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < np; i += gridDim.x * kThreads) {
    double v[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      v[k] = c[k * n6 + i];
      const double d = v[k] - s[k];
      ms[k] += d;
      mq[k] += d * d;
    }
    if (nc > 0) {
      const int ic = mbt::bin_of(v[0], sgm, nsig, dT);
      if (ic >= 0 && ic < nc) {
        atomicAdd(&hc[ic], 1);
        mbt::fx70_add(&fxh[ic], &fxl[ic], v[1]);
        mbt::fx70_add(&fzh[ic], &fzl[ic], v[2]);
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const double a = mbt::warp_sum(ms[k]), b = mbt::warp_sum(mq[k]);
    if (lane == 0) { red[warp][k] = a; red[warp][6 + k] = b; }
  }
  __syncthreads();
  double *rec = part + (size_t)blockIdx.x * prec;
  if (threadIdx.x < kExtra) {
    double t = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) t += red[w][threadIdx.x];
    rec[3 * nc + threadIdx.x] = t;
  }
  for (int i = threadIdx.x; i < nc; i += kThreads) {
    rec[i] = (double)hc[i];
    rec[nc + i] = mbt::fx70_value(fxh[i], fxl[i]);
    rec[2 * nc + i] = mbt::fx70_value(fzh[i], fzl[i]);
  }
}

// One block: records summed in block order; stats (12 doubles, mbt.h
// order) and histograms written to `out` (12 + 3 nc doubles).
__global__ void __launch_bounds__(kThreads)
moments_final(int np, const double *__restrict__ c, size_t ld, int nc, int nblk, const double *__restrict__ part,
              int prec, int th, int tv, double *__restrict__ out) {
  const size_t n6 = ld;
  for (int e = threadIdx.x; e < prec; e += kThreads) {
    double t = 0.0;
    for (int b = 0; b < nblk; ++b) t += part[(size_t)b * prec + e];
    if (e < 3 * nc) out[12 + e] = t;
    else {
      const int k = (e - 3 * nc) % 6;
      const bool sq = (e - 3 * nc) >= 6;
      const int plane = k % 3;
      const bool tracked = plane == 0 || (plane == 1 ? th : tv);
      // stash: sums into out[] temporarily
      if (!sq) out[12 + 3 * nc + k] = tracked ? t : 0.0;
      else out[12 + 3 * nc + 6 + k] = tracked ? t : 0.0;
    }
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    const int k = threadIdx.x;
    const double N = (double)np;
    const double sum = out[12 + 3 * nc + k], sq = out[12 + 3 * nc + 6 + k];
    const int plane = k % 3;
    const bool tracked = plane == 0 || (plane == 1 ? th : tv);
    double mean = 0.0, rms = 0.0;
    if (tracked && np > 0) {
      const double a = sum / N, q = sq / N;
      mean = c[k * n6] + a;
      const double var = q - a * a;
      rms = sqrt(var > 0.0 ? var : 0.0);
    }
    const int col = (k < 3) ? k : 6 + (k - 3);
    out[col] = mean;
    out[col + 3] = rms;
  }
}

int blocks_for(int np) {
  return std::max(1, std::min((np + kThreads * 8 - 1) / (kThreads * 8), 148 * 4));
}

int check_args(int np, const double *coord, double sgm, double dT, int ncell, const int *tp,
               const double *stats, const double *hist) {
  if (np <= 0 || !coord || !tp || !stats)
    return mbt::fail_global(MBT_ERR_INVALID, "bunch moments: np must be positive, pointers non-NULL");
  if (ncell < 0 || ncell > MBT_MAX_NCELL)
    return mbt::fail_global(MBT_ERR_INVALID, "bunch moments: ncell %d outside 0..%d", ncell, MBT_MAX_NCELL);
  if (ncell > 0 && (!hist || !(sgm > 0.0) || !(dT > 0.0)))
    return mbt::fail_global(MBT_ERR_INVALID, "bunch moments: binning needs hist_dev, sigma_tau > 0, dT > 0");
  return 0;
}

int run_moments(int np, const double *coord, size_t ld, double sgm, double nsig, double dT, int ncell,
                const int *tp, double *stats, double *hist, cudaStream_t st, double *scratch, int nblk) {
  const int prec = 3 * ncell + kExtra;
  const size_t smem = (size_t)ncell * (4 * sizeof(unsigned long long) + sizeof(int));
  double *part = scratch, *out = scratch + (size_t)nblk * prec;
  moments_partial<<<nblk, kThreads, smem, st>>>(np, coord, ld, sgm, nsig, dT, ncell, part, prec);
  moments_final<<<1, kThreads, 0, st>>>(np, coord, ld, ncell, nblk, part, prec, tp[1] != 0, tp[2] != 0, out);
  if (cudaGetLastError() != cudaSuccess) return MBT_ERR_CUDA;
  if (ncell > 0 &&
      cudaMemcpyAsync(hist, out + 12, (size_t)3 * ncell * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return MBT_ERR_CUDA;
  if (cudaMemcpyAsync(stats, out, 12 * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess) return MBT_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return MBT_ERR_CUDA;
  return 0;
}

}  // namespace

namespace mbt {
// Statistics of one bunch whose six coordinate arrays start `ld` doubles
// apart (a context's padded layout), without histograms.  scratch holds at
// least stats_scratch_doubles(np) doubles.
size_t stats_scratch_doubles(int np) { return (size_t)blocks_for(np) * kExtra + 12 + kExtra; }
int bunch_stats_strided(int np, const double *coord, size_t ld, const int tp[3], double *stats, void *stream,
                        double *scratch) {
  return run_moments(np, coord, ld, 1.0, 0.0, 1.0, 0, tp, stats, nullptr, (cudaStream_t)stream, scratch,
                     blocks_for(np));
}
}  // namespace mbt

extern "C" int mbt_bunch_moments_dev(int np, const double *coord_dev, double sigma_tau, double nsigma, double dT,
                                     int ncell, const int track_plane[3], double *stats, double *hist_dev,
                                     void *stream) {
  int r = check_args(np, coord_dev, sigma_tau, dT, ncell, track_plane, stats, hist_dev);
  if (r) return r;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return mbt::fail_global(MBT_ERR_NODEVICE, "no CUDA device: libmbt has no CPU path");
  const int nblk = blocks_for(np);
  const size_t n = (size_t)nblk * (3 * ncell + kExtra) + 12 + 3 * (size_t)ncell + 12;
  double *scratch = nullptr;
  if (cudaMalloc(&scratch, n * sizeof(double)) != cudaSuccess)
    return mbt::fail_global(MBT_ERR_NOMEM, "bunch moments: cudaMalloc of %zu bytes failed", n * sizeof(double));
  r = run_moments(np, coord_dev, (size_t)np, sigma_tau, nsigma, dT, ncell, track_plane, stats, hist_dev,
                  (cudaStream_t)stream, scratch, nblk);
  cudaFree(scratch);
  return r;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of mbt_bunch_moments_dev.
//
// Some callers cannot call cudaMalloc at the moment they need the bunch
// statistics: a host that owns all device memory through its own pool (or a
// framework's caching allocator) and must keep every byte accounted for, or a
// latency-critical loop where an allocation per call, which may synchronise
// the device, is not acceptable.  For them the block partial sums live in
// one file-scope device array of fixed size instead of per-call memory.
//
// That array exists once on every GPU that loads this library and stays
// allocated until the process exits.  Every call looks up its device address
// (cudaGetSymbolAddress, with the caller's device current: the address is
// only valid there) and passes it to the kernels; a lookup allocates
// nothing, and looking up on every call keeps the address right after a
// cudaDeviceReset has reloaded the module.  The first call on a device also
// loads the module's device code and data there.  Every call uses the same
// array and leaves its contents behind; each call writes every element it
// later reads (partial records, then the result area), so nothing has to be
// cleared.  Two calls whose
// work overlaps on the GPU (different streams, or different host threads on
// one device) race on the array.

namespace {

constexpr size_t kNoAllocDoubles = 262144;      // 2 MiB
__device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];
// the largest histogram (MBT_MAX_NCELL bins) fits: the result area and at
// least one block record
static_assert(MBT_NOALLOC_MAX_NCELL <= MBT_MAX_NCELL, "limit above the library's");
static_assert(12 + 3 * (size_t)MBT_NOALLOC_MAX_NCELL + 12 + 3 * (size_t)MBT_NOALLOC_MAX_NCELL + kExtra <=
                  kNoAllocDoubles,
              "the scratch array cannot hold the largest histogram");

int noalloc_scratch(double **out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0)
    return mbt::fail_global(MBT_ERR_NODEVICE, "no CUDA device: libmbt has no CPU path");
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || p == nullptr)
    return mbt::fail_global(MBT_ERR_CUDA, "cudaGetSymbolAddress of the scratch array on device %d: %s", dev,
                            cudaGetErrorString(e));
  *out = static_cast<double *>(p);
  return 0;
}

}  // namespace

extern "C" int mbt_bunch_moments_dev_noalloc(int np, const double *coord_dev, double sigma_tau, double nsigma,
                                             double dT, int ncell, const int track_plane[3], double *stats,
                                             double *hist_dev, void *stream) {
  // check_args rejects ncell above MBT_MAX_NCELL = MBT_NOALLOC_MAX_NCELL
  int r = check_args(np, coord_dev, sigma_tau, dT, ncell, track_plane, stats, hist_dev);
  if (r) return r;
  double *scratch = nullptr;
  r = noalloc_scratch(&scratch);
  if (r) return r;
  const int prec = 3 * ncell + kExtra;
  const size_t result = 12 + 3 * (size_t)ncell + 12;
  const int fit = (int)((kNoAllocDoubles - result) / (size_t)prec);
  const int nblk = std::min(blocks_for(np), fit);   // fit >= 1 (static_assert above)
  return run_moments(np, coord_dev, (size_t)np, sigma_tau, nsigma, dT, ncell, track_plane, stats, hist_dev,
                     (cudaStream_t)stream, scratch, nblk);
}

// ---------------------------------------------------------------------------
// Self-test of the bounded waits: one thread waits on an mbarrier that no
// thread arrives at, with the same helpers (mbt::mbar_wait, and the
// sleeping mbt::mbar_wait_sleep of the learned-field kernels) and the same
// give-up path as the kernels; the polling wait must end after `polls`
// polls, the sleeping one after `polls` x 1000 clock cycles.

namespace {
__global__ void bounded_wait_probe(long polls, int *gave_up) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbt::mbar_init(&bar, 1);
    mbt::fence_mbar_init();
    const bool a = mbt::mbar_wait(&bar, 0u, polls);
    const bool b = mbt::mbar_wait_sleep(&bar, 0u, (long long)polls * 1000);
    *gave_up = (a ? 0 : 1) + (b ? 0 : 2);
  }
}
}  // namespace

extern "C" int mbt_selftest_bounded_wait(long polls, void *stream) {
  if (polls < 1 || polls > (1L << 24))
    return mbt::fail_global(MBT_ERR_INVALID, "bounded wait self-test: polls %ld outside 1..2^24", polls);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return mbt::fail_global(MBT_ERR_NODEVICE, "no CUDA device: libmbt has no CPU path");
  cudaStream_t st = (cudaStream_t)stream;
  int *flag = nullptr;
  if (cudaMalloc(&flag, sizeof(int)) != cudaSuccess)
    return mbt::fail_global(MBT_ERR_NOMEM, "bounded wait self-test: flag");
  int gave_up = -1;
  bounded_wait_probe<<<1, 32, 0, st>>>(polls, flag);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&gave_up, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(flag);
  if (e != cudaSuccess) return mbt::fail_global(MBT_ERR_CUDA, "bounded wait self-test: %s", cudaGetErrorString(e));
  if (gave_up == 3)
    return mbt::fail_global(MBT_ERR_TIMEOUT, "bounded waits gave up after %ld polls / %ld cycles", polls,
                            polls * 1000);
  if (gave_up != 0) return mbt::fail_global(MBT_ERR_STATE, "bounded wait self-test: only one wait gave up (%d)", gave_up);
  return 0;
}
