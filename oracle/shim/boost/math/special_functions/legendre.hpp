// Test infrastructure (oracle only): a stand-in for the two Boost.Math 1.88
// Legendre routines the reference calls, so that the reference compiles from
// its own sources in a container where Boost is not installed.
//
// Boost.Math 1.88 is named by the reference's project file (Code/MLFMA.vcxproj:74)
// and is not vendored. The reference calls:
//   boost::math::legendre_p(l, x)        Code/OverloadAlgo.h:259, Code/AlgoMLFMM.h:277
//   boost::math::legendre_p_prime(l, x)  Code/OverloadAlgo.h:260, :283
// Both are restated here from their published definitions:
//   P_0 = 1, P_1 = x, (n+1) P_{n+1} = (2n+1) x P_n - n P_{n-1}   (Bonnet recurrence)
//   P'_l = sum over k = l-1, l-3, ... >= 0 of (2k+1) P_k          (derivative identity)
// which is also the evaluation scheme Boost documents for these functions.
// Accuracy is checked against scipy/numpy in tests/test_oracle_shim.py.
#pragma once
#include <stdexcept>
#include <cmath>

namespace boost {
namespace math {

namespace shim_detail {
inline void check_domain(double x) {
  if (!(x >= -1.0 && x <= 1.0))
    throw std::domain_error("legendre_p: argument outside [-1, 1]");
}
}  // namespace shim_detail

// P_l(x) by the three-term recurrence; P_{-l-1} = P_l as Boost defines it.
inline double legendre_p(int l, double x) {
  shim_detail::check_domain(x);
  if (l < 0) l = -l - 1;
  if (l == 0) return 1.0;
  double pm1 = 1.0, p = x;
  for (int n = 1; n < l; ++n) {
    const double pn1 = ((2.0 * n + 1.0) * x * p - n * pm1) / (n + 1.0);
    pm1 = p;
    p = pn1;
  }
  return p;
}

// dP_l/dx as the sum of (2k+1) P_k over k of the opposite parity to l.
inline double legendre_p_prime(int l, double x) {
  shim_detail::check_domain(x);
  if (l < 0) l = -l - 1;
  if (l == 0) return 0.0;
  double deriv = 0.0;
  double pm1 = 1.0, p = x;  // P_0, P_1
  // k runs from 0 upwards; add (2k+1) P_k when (l - 1 - k) is even.
  if (((l - 1) & 1) == 0) deriv += 1.0;          // k = 0
  if (l - 1 >= 1 && ((l - 2) & 1) == 0) deriv += 3.0 * x;  // k = 1
  for (int k = 1; k + 1 <= l - 1; ++k) {
    const double pk1 = ((2.0 * k + 1.0) * x * p - k * pm1) / (k + 1.0);
    pm1 = p;
    p = pk1;
    const int kk = k + 1;
    if (((l - 1 - kk) & 1) == 0) deriv += (2.0 * kk + 1.0) * p;
  }
  return deriv;
}

}  // namespace math
}  // namespace boost
