// mbt_tune.cu -- coherent tune analysis of centroid histories
// (get_tunepeaks_coherent tune.c:144-328, identify_tunepeaks :383-480).
//
//   tune_spectra    one block per history: radix-2 FFT in shared memory
//                   (FP64, bit-reversed load, log2 L butterfly stages),
//                   magnitudes, normalisation by the block maximum
//   mbt_tune_peaks  the reference's peak search on a normalised spectrum
//                   (host)
//
// The reference transforms its LON history with an explicit N-point DFT
// and its HOR / VER histories with GSL's real radix-2 FFT of the history
// zero-padded to 2N points; both give the same magnitudes as the FFT here
// up to rounding.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "mbt.h"

namespace mbt {
int fail_global(int code, const char *fmt, ...);
}

namespace {

constexpr int kTuneThreads = 256;
constexpr int kTuneMaxLen = 4096;   // transform points: 64 KB of complex FP64 in shared memory

__global__ void __launch_bounds__(kTuneThreads) tune_spectra(const double *__restrict__ x, long ld, int nturn, int pad,
                                                           double *__restrict__ out) {
  extern __shared__ double2 z[];
  __shared__ double red[kTuneThreads / 32];
  const int L = pad ? 2 * nturn : nturn;
  const int logL = 31 - __clz(L);
  const double *xs = x + (size_t)blockIdx.x * ld;
  for (int i = threadIdx.x; i < L; i += kTuneThreads) {
    const int r = (int)(__brev((unsigned)i) >> (32 - logL));
    z[r] = make_double2(i < nturn ? xs[i] : 0.0, 0.0);
  }
  __syncthreads();
  // X_k = sum_j x_j exp(-2 pi i j k / L): butterflies of span 2 half
  for (int half = 1; half < L; half <<= 1) {
    for (int b = threadIdx.x; b < L / 2; b += kTuneThreads) {
      const int pos = b & (half - 1);
      const int i0 = ((b - pos) << 1) + pos, i1 = i0 + half;
      double sn, cs;
      sincospi(-(double)pos / (double)half, &sn, &cs);
      const double2 a = z[i0], c = z[i1];
      const double tr = cs * c.x - sn * c.y, ti = cs * c.y + sn * c.x;
      z[i0] = make_double2(a.x + tr, a.y + ti);
      z[i1] = make_double2(a.x - tr, a.y - ti);
    }
    __syncthreads();
  }
  // magnitudes: padded (HOR, VER) bins 0 .. N-1 (bin 0 the real part, the
  // reference reads its imaginary part past its array, tune.c:250-254);
  // unpadded (LON) bins 0 .. N/2, / N, bin 0 halved (tune.c:181-197)
  const int nout = pad ? nturn : nturn / 2 + 1;
  const int j0 = pad ? 0 : 1;
  double mx = 0.0;
  for (int j = threadIdx.x; j < nout; j += kTuneThreads) {
    double m = j == 0 ? fabs(z[0].x) : sqrt(z[j].x * z[j].x + z[j].y * z[j].y);
    if (!pad) {
      m /= (double)nturn;
      if (j == 0) m *= 0.5;
    }
    z[j].x = m;
    if (j >= j0) mx = fmax(mx, m);
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  double m = 0.0;
  for (int w = 0; w < kTuneThreads / 32; ++w) m = fmax(m, red[w]);
  double *o = out + (size_t)blockIdx.x * nout;
  for (int j = threadIdx.x; j < nout; j += kTuneThreads)
    o[j] = (j < j0 || m == 0.0) ? 0.0 : z[j].x / m;
}

}  // namespace

extern "C" int mbt_tune_spectra_dev(const double *x_dev, long ld, int nseries, int nturn, int plane,
                                    double *spec_dev, void *stream) {
  const int pad = plane != 0;
  if (!x_dev || !spec_dev || nseries < 1 || plane < 0 || plane > 2)
    return mbt::fail_global(MBT_ERR_INVALID, "tune spectra: null array, no series or plane outside 0..2");
  if (nturn < 4 || (nturn & (nturn - 1)) || (pad ? 2 * nturn : nturn) > kTuneMaxLen)
    return mbt::fail_global(MBT_ERR_INVALID, "tune spectra: %d turns (a power of two, 4..%d for plane %d)", nturn,
                            pad ? kTuneMaxLen / 2 : kTuneMaxLen, plane);
  if (ld < nturn) return mbt::fail_global(MBT_ERR_INVALID, "tune spectra: stride %ld below %d turns", ld, nturn);
  const size_t smem = (size_t)(pad ? 2 * nturn : nturn) * sizeof(double2);
  cudaError_t e = cudaSuccess;
  if (smem > 48 * 1024)
    e = cudaFuncSetAttribute(tune_spectra, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    tune_spectra<<<nseries, kTuneThreads, smem, (cudaStream_t)stream>>>(x_dev, ld, nturn, pad, spec_dev);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return mbt::fail_global(MBT_ERR_CUDA, "tune spectra: %s", cudaGetErrorString(e));
  return 0;
}

// identify_tunepeaks (tune.c:383-480): a bin j is a peak when it stands
// 0.2 above both neighbours; a plateau within 0.2 that ends 0.2 lower is a
// peak at its middle (case 2); the peak position is refined by a parabola
// through the three bins at it.  At most 10 peaks.  Where the reference
// leaves its next index unset (a bin exactly 0.2 above or below its
// neighbour) the search moves on by one bin.
extern "C" int mbt_tune_peaks(const double *cofu, long nrev, double *value, double *ampli, int *pcase,
                              int max_peaks) {
  const int kMax = 10;
  const double thresh = 0.2;
  if (!cofu || nrev < 4 || max_peaks < 0) return MBT_ERR_INVALID;
  const long npts = nrev / 2;
  const double fn = (double)nrev;
  int npeak = 0;
  long j = 1;
  while (j < npts - 1) {
    int ipeak = 0, pc = 0;
    long jpk = 0, jn = j + 1;
    if (cofu[j] > cofu[j - 1] + thresh) {
      if (cofu[j] > cofu[j + 1] + thresh) {
        ipeak = 1;
        jpk = j;
        jn = j + 2;
        pc = 1;
      } else if (cofu[j] < cofu[j + 1] - thresh) {
        jn = j + 1;
      } else if (fabs(cofu[j] - cofu[j + 1]) < thresh) {
        long k = j + 2;
        while (fabs(cofu[j] - cofu[k]) < thresh && k < npts - 1) k++;
        if (cofu[j] > cofu[k] + thresh) {
          ipeak = 1;
          jpk = (j + k) / 2;
          pc = 2;
        }
        jn = k;
      }
      j = jn;
      if (ipeak) {
        const double cen = cofu[jpk], lo = cofu[jpk - 1], hi = cofu[jpk + 1];
        const double rj = jpk + (hi - lo) / (2.0 * cen - lo - hi) / 2.0;
        if (npeak < max_peaks) {
          if (value) value[npeak] = rj / fn;
          if (ampli) ampli[npeak] = cen;
          if (pcase) pcase[npeak] = pc;
        }
        npeak++;
      }
    } else {
      j++;
    }
    if (npeak == kMax) break;
  }
  return npeak < max_peaks ? npeak : max_peaks;
}
