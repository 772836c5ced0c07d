/*
 * TEST INFRASTRUCTURE ONLY.  Exposes the reference's own Boost-free math
 * headers (compiled in place from the ESPResSo source tree, never copied)
 * through a C ABI so the oracle's restatements can be pinned against them:
 *   src/utils/include/utils/math/bspline.hpp       (B-spline weights)
 *   src/utils/include/utils/math/AS_erfc_part.hpp  (A&S erfc approximation)
 *   src/core/p3m/math.hpp                           (sinc, cotangent sums)
 * Built by oracle/Makefile into oracle/_ref/ only when the reference tree
 * is present.
 */
#include "p3m/math.hpp"
#include <utils/math/AS_erfc_part.hpp>
#include <utils/math/bspline.hpp>

namespace {
template <int P> double bs(int i, double x) { return Utils::bspline<P>(i, x); }
} // namespace

extern "C" {
double ref_bspline(int order, int i, double x) {
  switch (order) {
  case 1: return bs<1>(i, x);
  case 2: return bs<2>(i, x);
  case 3: return bs<3>(i, x);
  case 4: return bs<4>(i, x);
  case 5: return bs<5>(i, x);
  case 6: return bs<6>(i, x);
  default: return bs<7>(i, x);
  }
}
double ref_as_erfc_part(double d) { return Utils::AS_erfc_part(d); }
double ref_sinc(double x) { return math::sinc(x); }
double ref_cotangent_sum(int cao, int n, double mesh_i) {
  return math::get_analytic_cotangent_sum_kernel(cao)(n, mesh_i);
}
}
