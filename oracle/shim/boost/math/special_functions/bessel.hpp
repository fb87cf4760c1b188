// Test infrastructure (oracle only): a stand-in for the two Boost.Math 1.88
// spherical Bessel routines the reference calls (Code/Bessel.h:14-23), so that
// the reference compiles from its own sources without Boost installed.
//
//   j_n(x): sin(x)/x, sin(x)/x^2 - cos(x)/x, then the recurrence
//           f_{n+1} = (2n+1)/x f_n - f_{n-1}, run upwards while n < x (stable
//           there) and downwards (Miller's method, normalised to j_0 or j_1,
//           whichever is larger) when n >= x; the power series for tiny x.
//   y_n(x): -cos(x)/x, -cos(x)/x^2 - sin(x)/x, then the same recurrence
//           upwards (always stable for the Neumann function).
// These are the textbook methods (Abramowitz & Stegun 10.1.19-10.1.22, and
// Miller's backward recurrence). Accuracy is checked against scipy in
// tests/test_oracle_shim.py over the orders and arguments the MLFMA transfer
// factors use.
#pragma once
#include <cmath>
#include <limits>
#include <vector>

namespace boost {
namespace math {

namespace shim_detail {

inline double sph_j_series(int n, double x) {
  // x^n / (2n+1)!! * sum_k (-x^2/2)^k / (k! (2n+3)(2n+5)...(2n+2k+1))
  double pref = 1.0;
  for (int k = 1; k <= n; ++k) pref *= x / (2.0 * k + 1.0);
  double term = 1.0, sum = 1.0;
  const double h = -0.5 * x * x;
  for (int k = 1; k < 60; ++k) {
    term *= h / (k * (2.0 * n + 2.0 * k + 1.0));
    sum += term;
    if (std::fabs(term) < 1e-18 * std::fabs(sum)) break;
  }
  return pref * sum;
}

}  // namespace shim_detail

inline double sph_bessel(unsigned n_in, double x) {
  const int n = static_cast<int>(n_in);
  if (x == 0.0) return n == 0 ? 1.0 : 0.0;
  const double ax = std::fabs(x);
  if (ax < 1e-3 * (n + 1) || ax < 1e-8) {
    double v = shim_detail::sph_j_series(n, ax);
    return (x < 0 && (n & 1)) ? -v : v;
  }
  const double s = std::sin(ax), c = std::cos(ax);
  const double j0 = s / ax;
  if (n == 0) return j0;
  const double j1 = s / (ax * ax) - c / ax;
  double result;
  if (n <= ax) {
    double jm = j0, j = j1;
    for (int k = 1; k < n; ++k) {
      const double jn = (2.0 * k + 1.0) / ax * j - jm;
      jm = j;
      j = jn;
    }
    result = j;
  } else {
    // Miller: start well above max(n, x) and recur downwards.
    const int start = n + 20 + static_cast<int>(std::sqrt(40.0 * (n + ax)));
    double fp = 0.0, f = 1e-280;
    double fn_keep = 0.0, f0 = 0.0, f1 = 0.0;
    for (int k = start; k >= 1; --k) {
      const double fm = (2.0 * k + 1.0) / ax * f - fp;
      fp = f;
      f = fm;
      if (std::fabs(f) > 1e250) {  // rescale everything kept so far
        f *= 1e-250;
        fp *= 1e-250;
        fn_keep *= 1e-250;
        f1 *= 1e-250;
      }
      if (k - 1 == n) fn_keep = f;
      if (k - 1 == 1) f1 = f;
      if (k - 1 == 0) f0 = f;
    }
    // f now holds f_0; f1 holds f_1.
    const double scale = (std::fabs(j0) >= std::fabs(j1)) ? j0 / f0 : j1 / f1;
    result = fn_keep * scale;
  }
  return (x < 0 && (n & 1)) ? -result : result;
}

inline double sph_neumann(unsigned n_in, double x) {
  const int n = static_cast<int>(n_in);
  if (x <= 0.0) return -std::numeric_limits<double>::infinity();
  const double s = std::sin(x), c = std::cos(x);
  const double y0 = -c / x;
  if (n == 0) return y0;
  double ym = y0, y = -c / (x * x) - s / x;
  for (int k = 1; k < n; ++k) {
    const double yn = (2.0 * k + 1.0) / x * y - ym;
    ym = y;
    y = yn;
  }
  return y;
}

}  // namespace math
}  // namespace boost
