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
  int emitter;  // its values' slot among the step's waves (sources' first, then the couplings')
  int pad;      // 1: a coupling of a plane wave's box
};

// One injection's share of a value of H (src/fdtd.rs:1346-1362): a point source or a current takes
// v - dt Re(a w(t)); a coupling of a plane wave's total-field/scattered-field box (pad 1) takes
// v - (dt weight) h_inc, its coefficient folded on the host and the incident value its "wave"
// (src/fdtd/sources.rs:971-991). w: the step's values, 2 per emitter.
template <typename T>
__device__ __forceinline__ T apply_h(T v, const Entry &en, const double *w, T dt) {
  const double amount = en.are * w[2 * en.emitter] - en.aim * w[2 * en.emitter + 1];
  if (en.pad) return v - (T)amount;
  if (sizeof(T) == 8) return v - (T)((double)dt * amount);
  return v - dt * (T)amount;
}

// The same for a value of E (src/fdtd.rs:1366-1393): v - cb Re(a w(t)), or a coupling's
// v - (cb weight) h_inc.
template <typename T>
__device__ __forceinline__ T apply_e(T v, const Entry &en, const double *w, T cbv) {
  const double amount = en.are * w[2 * en.emitter] - en.aim * w[2 * en.emitter + 1];
  if (en.pad) return v - (T)amount;
  if (sizeof(T) == 8) return v - (T)((double)cbv * amount);
  return v - cbv * (T)amount;
}

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

// x / h with h a grid step, the quotient IEEE division gives. In f32, where `fast` (set only
// after the engine has compared it with division for every finite float x, see
// verify_division_kernel), by Markstein's correction of the reciprocal product (P. Markstein,
// IBM J. Res. Dev. 34(1), 1990): q0 = x r with r = 1/h rounded, the remainder e = x - q0 h exact
// by a fused multiply-add, q = q0 + e r rounded once. The remainder is exact only while it does
// not underflow, so |x| below 2^-90 is first scaled by 2^64 and the quotient scaled back (both
// exact while the quotient is a normal number); zero gives x r (its sign kept); a subnormal
// quotient is x times 1/h in double, rounded to float; a quotient that overflows takes the
// division. In f64 always the division.
#ifdef __CUDA_ARCH__
// Out of line, so that the rare inputs' division is a call the common path branches over, not a
// sequence issued (predicated off) at every use.
static __device__ __noinline__ float div_rare(float x, float h) { return x / h; }
#define PXF_DIV_RARE(x, h) div_rare(x, h)
#else
#define PXF_DIV_RARE(x, h) ((x) / (h))
#endif
__host__ __device__ __forceinline__ float div_by_step(float x, float h, float r, double rd,
                                                      int fast) {
  if (fast) {
    const float ax = fabsf(x);
    const bool tiny = ax < 0x1p-90f;
    const float sx = x * (tiny ? 0x1p64f : 1.0f);
    const float q0 = sx * r;
    const float e = fmaf(-q0, h, sx);
    const float q = fmaf(e, r, q0) * (tiny ? 0x1p-64f : 1.0f);
    const float aq = fabsf(q);
    // a normal quotient, or zero: x r with x's sign (q0, the product of the unscaled zero)
    const bool zero = x == 0.0f;
    if (zero || (aq >= 0x1p-126f && aq <= 3.40282347e38f)) return zero ? q0 : q;
    // a subnormal quotient: the product with 1/h in double, rounded once to float, carries
    // 53 bits for the at most 23 the result keeps
    if (aq < 0x1p-126f) return (float)((double)x * rd);
  }
  return PXF_DIV_RARE(x, h);
}
__host__ __device__ __forceinline__ double div_by_step(double x, double h, double, double, int) {
  return x / h;
}

// Four quotients x[j] / h at once, each div_by_step's: where all four take its common path (x
// zero, or not tiny with a normal quotient) that path's three operations each and one test for
// the four; otherwise div_by_step value by value. The same bits either way. (Zero differences
// are the rule where the fields are still at rest, as in most of a CPML early in a run.)
__host__ __device__ __forceinline__ void div4_by_step(const float x[4], float q[4], float h, float r,
                                                      double rd, int fast) {
  if (fast) {
    bool common = true;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const float q0 = x[j] * r;
      const float e = fmaf(-q0, h, x[j]);
      const float qj = fmaf(e, r, q0);
      const float aq = fabsf(qj);
      const bool zero = x[j] == 0.0f;  // x r, its sign kept: q0
      q[j] = zero ? q0 : qj;
      common = common &&
               (zero || (fabsf(x[j]) >= 0x1p-90f && aq >= 0x1p-126f && aq <= 3.40282347e38f));
    }
    if (common) return;
  }
#pragma unroll
  for (int j = 0; j < 4; j++) q[j] = div_by_step(x[j], h, r, rd, fast);
}
__host__ __device__ __forceinline__ void div4_by_step(const double x[4], double q[4], double h,
                                                      double, double, int) {
#pragma unroll
  for (int j = 0; j < 4; j++) q[j] = x[j] / h;
}

}  // namespace pxf
