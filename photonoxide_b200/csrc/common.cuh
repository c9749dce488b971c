// Definitions the engine's kernels share: the CPML slab table's entries, the sources' groups and
// entries, the waveforms evaluated on the device, periodic wrapping.
#pragma once
#include <cuda_runtime.h>

#include <cmath>

#include "portable.h"

namespace pxf {

constexpr double TAU = 6.283185307179586476925286766559;

struct SlabEntry {
  int from, count;  // count 0: no slab
  long long psi;    // where its psi starts
  int coef;         // where its b starts (a follows after count)
  // along x, psi's rows start at pf = from rounded down to a multiple of 4 and are pw values
  // wide, a multiple of 4, so four places are one aligned vector (along y and z: from, count)
  int pf, pw;
};

// A value the sources add to, with its entries (emitter, amplitude) in CPU order.
struct Group {
  int local;  // index in the CTA's staged region: H's (HX x HY) or E's tile (TX x TY), x fastest
  int comp;
  int first, count;
};
struct Entry {
  double are, aim;
  int emitter;
  int pad;
};

__host__ __device__ inline int wrap_index(int g, int n, int periodic) {
  if (g >= 0 && g < n) return g;
  if (periodic) {
    if (g == n) return 0;
    if (g == -1) return n - 1;
  }
  return -1;
}

struct Wave {
  int kind;
  double p[5];
};

// The waveforms with the reference's exp and sincos (portable.h), so the sources' values are
// its bits: w.at(t) for a point source, the analytic form w(t) for a current.
__device__ inline void wave_eval(const Wave &w, double t, double *re, double *im, int point) {
  if (w.kind == 0) {
    double u = (t - w.p[2]) / w.p[1];
    double g = pxp::exp(-u * u);
    double s, c;
    if (point) {  // e^{-u^2} sin(omega (t - delay))
      pxp::sincos((TAU * w.p[0]) * (t - w.p[2]), &s, &c);
      *re = g * s;
      *im = 0.0;
    } else {  // (i e^{-u^2}) e^{-i omega (t - delay)}, as num-complex multiplies
      pxp::sincos(-(TAU * w.p[0]) * (t - w.p[2]), &s, &c);
      *re = 0.0 * c - g * s;
      *im = 0.0 * s + g * c;
    }
  } else if (w.kind == 1) {
    double u = (t - w.p[1]) / w.p[0];
    *re = -u * pxp::exp(-u * u) * sqrt(2.0 * 2.718281828459045235);
    *im = 0.0;
  } else {
    double ss = 1.0;
    if (w.p[3] > 0.0) {
      double r = fmin(fmax(t / w.p[3], 0.0), 1.0);
      ss = r * r * (3.0 - 2.0 * r);
    }
    double s, c;
    pxp::sincos(-(TAU * w.p[0]) * t, &s, &c);
    if (point) {  // smoothstep * Re(amplitude e^{-i omega t})
      *re = ss * (w.p[1] * c - w.p[2] * s);
      *im = 0.0;
    } else {  // (smoothstep amplitude) e^{-i omega t}
      double ar = ss * w.p[1], ai = ss * w.p[2];
      *re = ar * c - ai * s;
      *im = ar * s + ai * c;
    }
  }
}

// A transform's series of values (monitors.rs:35-206) as the device accumulates it.
struct SeriesDev {
  long long value0;  // first value in the ring
  long long volume;
  long long sum0;    // first sum (complex)
  int nf;
  int slot0;         // its phases' slot for frequency 0
};

}  // namespace pxf
