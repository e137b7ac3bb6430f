// mbt_fields.cu -- per-step entry points for the beam-ion field: Faddeeva
// w(z) (physic.c:75-301) and the Bassetti-Erskine field
// (fbi_weakstrong.c:154-197).  Compiled without multiply-add contraction,
// so every operation rounds as in the reference's x86-64 build.
#include <cuda_runtime.h>

#include <algorithm>

#include "mbt.h"
#include "mbt_wofz.cuh"

namespace mbt {
int fail_global(int code, const char *fmt, ...);
}

#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) return mbt::fail_global(MBT_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

namespace mbt {

__global__ void wofz_kernel(long n, const double *__restrict__ x, const double *__restrict__ y,
                            double *__restrict__ re, double *__restrict__ im, int *__restrict__ flag) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double u, v;
    const int f = wofz_dev(x[i], y[i], u, v);
    re[i] = u;
    im[i] = v;
    if (flag) flag[i] = f;
  }
}

// fbi_weakstrong.c:155-191 for one slice: sizes in mm, offsets in m.
__global__ void be_field_kernel(long n, const double *__restrict__ dx, const double *__restrict__ dy,
                                double sgm_xx, double sgm_zz, double factdQ,
                                double *__restrict__ ex, double *__restrict__ ey) {
  const double factBE = sqrt(2 * (sgm_xx * sgm_xx - sgm_zz * sgm_zz)) / 1.0e3;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double Dx = dx[i], Dy = dy[i];
    const double xi1 = Dx / factBE;
    const double xi2 = xi1 * sgm_zz / sgm_xx;
    const double yi1 = Dy / factBE;
    const double yi2 = yi1 * sgm_xx / sgm_zz;
    double u1r, u1i, u2r, u2i;
    wofz_dev(xi1, yi1, u1r, u1i);
    wofz_dev(xi2, yi2, u2r, u2i);
    const double e = exp(-(Dx * Dx * 1.0e6 / (2 * sgm_xx * sgm_xx) + Dy * Dy * 1.0e6 / (2 * sgm_zz * sgm_zz)));
    ex[i] = -factdQ * (u1i - e * u2i);
    ey[i] = -factdQ * (u1r - e * u2r);
  }
}

}  // namespace mbt

namespace {
int check_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
    return mbt::fail_global(MBT_ERR_NODEVICE, "no CUDA device: libmbt has no CPU path");
  return 0;
}
}  // namespace

extern "C" {

int mbt_wofz_dev(long n, const double *x, const double *y, double *re, double *im, int *flag, void *stream) {
  if (n < 0 || (n > 0 && (!x || !y || !re || !im))) return mbt::fail_global(MBT_ERR_INVALID, "bad wofz arguments");
  if (n == 0) return 0;
  int r = check_device();
  if (r) return r;
  const int blocks = (int)std::min<long>((n + 255) / 256, 148L * 16);
  mbt::wofz_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(n, x, y, re, im, flag);
  CK(cudaGetLastError());
  return 0;
}

int mbt_be_field_dev(long n, const double *dx, const double *dy, double sgm_xx_mm, double sgm_zz_mm, double factdq,
                     double *ex, double *ey, void *stream) {
  if (n < 0 || (n > 0 && (!dx || !dy || !ex || !ey))) return mbt::fail_global(MBT_ERR_INVALID, "bad be_field arguments");
  if (!(sgm_xx_mm > sgm_zz_mm) || !(sgm_zz_mm > 0))
    return mbt::fail_global(MBT_ERR_INVALID, "Bassetti-Erskine needs sgm_xx > sgm_zz > 0");
  if (n == 0) return 0;
  int r = check_device();
  if (r) return r;
  const int blocks = (int)std::min<long>((n + 255) / 256, 148L * 16);
  mbt::be_field_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(n, dx, dy, sgm_xx_mm, sgm_zz_mm, factdq, ex, ey);
  CK(cudaGetLastError());
  return 0;
}

}  // extern "C"
