/*
 * gsl_fft_stub.c -- TEST INFRASTRUCTURE ONLY.  The reference's tune.c
 * (tune.c:249, 271) calls gsl_fft_real_radix2_transform of the GNU
 * Scientific Library (GSL 2.x, not installed here).  This restates the
 * published behaviour of that routine for the oracle build of tune.c: the
 * forward transform X_k = sum_j x_j exp(-2 pi i j k / n) of n real values
 * (n a power of two), returned in GSL's half-complex order
 *   data[0] = Re X_0,  data[k] = Re X_k (k = 1 .. n/2),
 *   data[n - k] = Im X_k (k = 1 .. n/2 - 1).
 * A direct sum in long double: the test sizes are small.
 */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>

int gsl_fft_real_radix2_transform(double data[], size_t stride, size_t n)
{
  size_t k, j;
  long double *re, *im;
  if (n < 2 || (n & (n - 1))) return 1;
  re = (long double *) calloc(n, sizeof(long double));
  im = (long double *) calloc(n, sizeof(long double));
  if (!re || !im) { free(re); free(im); return 1; }
  for (k = 0; k <= n / 2; k++) {
    long double sr = 0.0L, si = 0.0L;
    for (j = 0; j < n; j++) {
      const long double ph = -2.0L * 3.14159265358979323846264338327950288L * (long double) ((j * k) % n) / (long double) n;
      sr += (long double) data[j * stride] * cosl(ph);
      si += (long double) data[j * stride] * sinl(ph);
    }
    re[k] = sr;
    im[k] = si;
  }
  data[0] = (double) re[0];
  for (k = 1; k <= n / 2; k++) data[k * stride] = (double) re[k];
  for (k = 1; k < n / 2; k++) data[(n - k) * stride] = (double) im[k];
  free(re);
  free(im);
  return 0;
}
