// mbt_wofz.cuh -- Faddeeva function w(z) = exp(-z^2) erfc(-iz) in FP64, the
// building block of every Bassetti-Erskine field (mbt_fields.cu,
// mbt_beamion.cuh).
//
// Algorithm: ACM TOMS 680 (G. P. M. Poppe and C. M. J. Wijers, "More
// efficient computation of the complex error function", ACM Trans. Math.
// Softw. 16(1), 1990, p. 47), with the region boundaries, term counts and
// overflow limits of the reference's complex_errorfunc_wofz_algo680
// (physic.c:143-301): power series (Abramowitz & Stegun 7.1.5) for
// qrho < 0.085264, Laplace continued fraction for qrho > 1, Taylor series
// with continued-fraction derivatives in between, reflection w(conj z)
// relations for the lower half plane.  Branches are per point.
#pragma once

namespace mbt {

__device__ __forceinline__ int wofz_dev(double xi, double yi, double &re, double &im) {
  const double factor = 1.12837916709551257388;   // 2/sqrt(pi)
  const double rmaxreal = 0.5e154;
  const double rmaxexp = 708.503061461606;
  const double rmaxgoni = 3.53711887601422e08;
  const double xabs = fabs(xi), yabs = fabs(yi);
  const double x = xabs / 6.3, y = yabs / 4.4;
  if (xabs > rmaxreal || yabs > rmaxreal) { re = 0.0; im = 0.0; return -1; }
  double qrho = x * x + y * y;
  double xquad = xabs * xabs - yabs * yabs;
  const double yquad = 2.0 * xabs * yabs;
  double u, v, u2 = 0.0, v2 = 0.0;
  const bool series = qrho < 0.085264;
  if (series) {
    qrho = (1.0 - 0.85 * y) * sqrt(qrho);
    const int n = (int)(6.0 + 72.0 * qrho);
    int j = 2 * n + 1;
    double xsum = 1.0 / (double)j, ysum = 0.0;
    for (int i = n; i >= 1; --i) {
      j = j - 2;
      const double xaux = (xsum * xquad - ysum * yquad) / (double)i;
      ysum = (xsum * yquad + ysum * xquad) / (double)i;
      xsum = xaux + 1.0 / (double)j;
    }
    const double u1 = -factor * (xsum * yabs + ysum * xabs) + 1.0;
    const double v1 = factor * (xsum * xabs - ysum * yabs);
    const double daux = exp(-xquad);
    double sn, cs;
    sincos(yquad, &sn, &cs);
    u2 = daux * cs;
    v2 = -daux * sn;
    u = u1 * u2 - v1 * v2;
    v = u1 * v2 + v1 * u2;
  } else {
    double h, h2 = 0.0, qlamda = 0.0;
    int kapn, nu;
    if (qrho > 1.0) {
      h = 0.0;
      kapn = 0;
      qrho = sqrt(qrho);
      nu = (int)(3.0 + 1442.0 / (26.0 * qrho + 77.0));
    } else {
      qrho = (1.0 - y) * sqrt(1.0 - qrho);
      h = 1.88 * qrho;
      h2 = 2.0 * h;
      kapn = (int)(7.0 + 34.0 * qrho);
      nu = (int)(16.0 + 26.0 * qrho);
    }
    const bool useb = h > 0.0;
    if (useb) qlamda = pow(h2, (double)kapn);
    double rx = 0.0, ry = 0.0, sx = 0.0, sy = 0.0;
    for (int n = nu; n >= 0; --n) {
      const int np1 = n + 1;
      double tx = yabs + h + np1 * rx;
      const double ty = xabs - np1 * ry;
      const double c = 0.5 / (tx * tx + ty * ty);
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
      xquad = -xquad;
      if ((yquad > rmaxgoni) || (xquad > rmaxexp)) { re = 0.0; im = 0.0; return -1; }
      const double w1 = 2.0 * exp(xquad);
      double sn, cs;
      sincos(yquad, &sn, &cs);
      u2 = w1 * cs;
      v2 = -w1 * sn;
    }
    u = u2 - u;
    v = v2 - v;
    if (xi > 0.0) v = -v;
  } else {
    if (xi < 0.0) v = -v;
  }
  re = u;
  im = v;
  return 1;
}

}  // namespace mbt
