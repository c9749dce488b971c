// The CPML's grading and recursion coefficients (Simulation::build_cpml, src/fdtd.rs:799-869),
// shared by the host library (host.cpp: build_cpml) and the device (setup.cu:
// pxs_cpml_device), so that both give the same bits: the same operations in the same order, f64,
// no fused multiply-add, the reference's pow, ln and exp (portable.h).
#pragma once
#include <cstdint>

#include "portable.h"

namespace pxc {

// sigma and kappa at `pos` (in cells from node 0) along an axis of n cells whose CPMLs are lo
// and hi cells thick, the step h; cpml = {reflection, sigma (NaN: from the reflection), order,
// kappa max, alpha}. The grading is ((depth / cells) clamped to [0, 1])^order.
PXP_FN void grade(double pos, int64_t lo, int64_t hi, int64_t n, double h, const double cpml[5],
                  double *s, double *k) {
  double depth = 0.0;
  int64_t cells = 0;
  if (lo > 0 && pos < (double)lo) {
    depth = (double)lo - pos;
    cells = lo;
  } else if (hi > 0 && pos > (double)(n - hi)) {
    depth = pos - (double)(n - hi);
    cells = hi;
  } else {
    *s = 0.0;
    *k = 1.0;
    return;
  }
  const double R = cpml[0], sig = cpml[1], order = cpml[2], kmax = cpml[3];
  const double d = (double)cells * h;
  double v = depth / (double)cells;
  v = v < 0.0 ? 0.0 : v;
  v = 1.0 < v ? 1.0 : v;
  const double x = pxp::pow(v, order);
  const double smax = sig != sig ? (order + 1.0) * (-pxp::ln(R)) / (2.0 * d) : sig;
  *s = smax * x;
  *k = 1.0 + (kmax - 1.0) * x;
}

// The psi recursion's b and a for sigma s, kappa k (src/fdtd.rs:851-862).
PXP_FN void recursion(double s, double k, double alpha, double dt, double *b, double *a) {
  *b = pxp::exp(-(s / k + alpha) * dt);
  const double den = s * k + k * k * alpha;
  *a = (s > 0.0 && den > 0.0) ? s * (*b - 1.0) / den : 0.0;
}

}  // namespace pxc
