// Test infrastructure: stand-in for boost::math::erf_inv, used only to build the reference
// sources as an oracle (GridGenerator.cpp:178 calls it at the pointsPerCo quantiles).
//
// Written from the mathematics: bracket the root of erf(x) - z by bisection, then polish
// with Newton steps using erf'(x) = 2/sqrt(pi) * exp(-x^2).  Accurate to a few ulp for
// |z| < 1, which is all the grid generator needs (z = +-0.25, +-0.75 for FillMarsaglia(4)).
#ifndef MPSQMC_COMPAT_BOOST_ERF_HPP
#define MPSQMC_COMPAT_BOOST_ERF_HPP

#include <cmath>
#include <limits>

namespace boost {
namespace math {

inline double erf_inv(double z) {
  if (z == 0.0) return 0.0;
  if (z >= 1.0) return std::numeric_limits<double>::infinity();
  if (z <= -1.0) return -std::numeric_limits<double>::infinity();
  const double sign = (z < 0.0) ? -1.0 : 1.0;
  const double t = std::fabs(z);
  double lo = 0.0, hi = 6.0;
  for (int it = 0; it < 60; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (std::erf(mid) < t) lo = mid; else hi = mid;
  }
  double x = 0.5 * (lo + hi);
  const double two_over_sqrt_pi = 1.1283791670955126;
  for (int it = 0; it < 4; ++it) {
    const double f = std::erf(x) - t;
    const double df = two_over_sqrt_pi * std::exp(-x * x);
    if (df == 0.0) break;
    x -= f / df;
  }
  return sign * x;
}

template <class T>
inline T erf_inv(T z) {
  return static_cast<T>(erf_inv(static_cast<double>(z)));
}

}  // namespace math
}  // namespace boost

#endif
