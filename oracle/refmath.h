// ORACLE (test infrastructure only): the transcendental functions photonoxide's FDTD source
// waveforms and transform phases call, restated so the oracle reproduces the reference's bits.
//
// - ref_exp restates photonoxide's own `portable::exp` (src/portable/mod.rs:66-139), its port of
//   fdlibm's exponential: reduction x = k ln2 + r with ln2 split in two, a degree-5 rational
//   correction in r*r, and the result scaled by 2^k through the exponent bits.
// - ref_sincos restates the published algorithm of the `libm` crate, version 0.2.16 (pinned at
//   Cargo.lock:2756-2758; not vendored, so not present in the reference tree), whose sincos the
//   reference calls through `portable::sin_cos` (src/portable/mod.rs:321-323): the fdlibm/musl
//   method of reducing by pi/2 (pi/2 split in three parts, refined while cancellation eats bits)
//   and the kernels sin(r) ~ r + r^3 S(r^2), cos(r) ~ 1 - r^2/2 + r^4 C(r^2) of degree 13 and 14.
//   Only the arguments below 2^20 pi/2 are reduced here; larger ones are not met by the runs the
//   oracle steps (a time and a frequency of order 10^4 at most), and fall back to the C library.
//
// Every operation is a separate IEEE double rounding (the oracle is compiled with
// -ffp-contract=off), in the order the methods prescribe.
#ifndef PHOTONOXIDE_ORACLE_REFMATH_H
#define PHOTONOXIDE_ORACLE_REFMATH_H

#include <cmath>
#include <cstdint>
#include <cstring>

namespace refmath {

inline uint64_t bits(double x) {
  uint64_t u;
  std::memcpy(&u, &x, 8);
  return u;
}
inline double from_bits(uint64_t u) {
  double x;
  std::memcpy(&x, &u, 8);
  return x;
}

// fdlibm's exponential as the reference ports it.
inline double ref_exp(double x) {
  const double o_threshold = from_bits(0x40862e42fefa39efULL);
  const double u_threshold = from_bits(0xc0874910d52d3051ULL);
  const double ln2_hi = from_bits(0x3fe62e42fee00000ULL);
  const double ln2_lo = from_bits(0x3dea39ef35793c76ULL);
  const double inv_ln2 = from_bits(0x3ff71547652b82feULL);
  const double two_m1000 = from_bits(0x0170000000000000ULL);
  const double p[5] = {from_bits(0x3fc555555555553eULL), from_bits(0xbf66c16c16bebd93ULL),
                       from_bits(0x3f11566aaf25de2cULL), from_bits(0xbebbbd41c5d26bf1ULL),
                       from_bits(0x3e66376972bea4d0ULL)};
  uint32_t top = (uint32_t)(bits(x) >> 32);
  bool negative = (top >> 31) != 0;
  top &= 0x7fffffffu;
  if (top >= 0x40862e42u) {
    if (std::isnan(x)) return x;
    if (x > o_threshold) return INFINITY;
    if (x < u_threshold) return 0.0;
  }
  int k = 0;
  double hi = 0.0, lo = 0.0;
  if (top > 0x3fd62e42u) {
    if (top < 0x3ff0a2b2u) {
      k = negative ? -1 : 1;
      hi = negative ? x + ln2_hi : x - ln2_hi;
      lo = negative ? -ln2_lo : ln2_lo;
    } else {
      k = (int)(inv_ln2 * x + (negative ? -0.5 : 0.5));
      double t = (double)k;
      hi = x - t * ln2_hi;
      lo = t * ln2_lo;
    }
    x = hi - lo;
  } else if (top < 0x3e300000u) {
    return 1.0 + x;
  }
  double t = x * x;
  double c = x - t * (p[0] + t * (p[1] + t * (p[2] + t * (p[3] + t * p[4]))));
  if (k == 0) return 1.0 - ((x * c) / (c - 2.0) - x);
  double y = 1.0 - ((lo - (x * c) / (2.0 - c)) - hi);
  if (k >= -1021) return from_bits(bits(y) + ((uint64_t)(int64_t)k << 52));
  return from_bits(bits(y) + ((uint64_t)(int64_t)(k + 1000) << 52)) * two_m1000;
}

// The two kernels on the reduced argument r = y0 + y1, |r| <= pi/4.
inline double kernel_sin(double x, double y, bool tail) {
  const double s1 = -1.66666666666666324348e-01, s2 = 8.33333333332248946124e-03,
               s3 = -1.98412698298579493134e-04, s4 = 2.75573137070700676789e-06,
               s5 = -2.50507602534068634195e-08, s6 = 1.58969099521155010221e-10;
  double z = x * x, w = z * z;
  double r = s2 + z * (s3 + z * s4) + z * w * (s5 + z * s6);
  double v = z * x;
  if (!tail) return x + v * (s1 + z * r);
  return x - ((z * (0.5 * y - v * r) - y) - v * s1);
}
inline double kernel_cos(double x, double y) {
  const double c1 = 4.16666666666666019037e-02, c2 = -1.38888888888741095749e-03,
               c3 = 2.48015872894767294178e-05, c4 = -2.75573143513906633035e-07,
               c5 = 2.08757232129817482790e-09, c6 = -1.13596475577881948265e-11;
  double z = x * x, w = z * z;
  double r = z * (c1 + z * (c2 + z * c3)) + w * w * (c4 + z * (c5 + z * c6));
  double hz = 0.5 * z;
  double one_minus = 1.0 - hz;
  return one_minus + (((1.0 - one_minus) - hz) + (z * r - x * y));
}

// x = n pi/2 + (y0 + y1) for |x| < 2^20 pi/2; returns n. pi/2 = p1 + p1t (+ p2 + p2t, + p3 + p3t).
inline int reduce_half_pi(double x, double y[2]) {
  const double inv_half_pi = 6.36619772367581382433e-01;
  const double p1 = 1.57079632673412561417e+00, p1t = 6.07710050650619224932e-11;
  const double p2 = 6.07710050630396597660e-11, p2t = 2.02226624879595063154e-21;
  const double p3 = 2.02226624871116645580e-21, p3t = 8.47842766036889956997e-32;
  const double round_shift = 1.5 / 2.220446049250313080847e-16;
  uint64_t u = bits(x);
  bool negative = (u >> 63) != 0;
  uint32_t top = (uint32_t)(u >> 32) & 0x7fffffffu;
  // one, two, three or four quarter turns away: a single subtraction of m (p1 + p1t), unless x
  // is close to a multiple of pi/2 where that cancels (then the general reduction below)
  int m = 0;
  if (top <= 0x400f6a7au) {
    if ((top & 0xfffffu) != 0x921fbu) m = top <= 0x4002d97cu ? 1 : 2;
  } else if (top <= 0x401c463bu) {
    if (top <= 0x4015fdbcu) m = top == 0x4012d97cu ? 0 : 3;
    else m = top == 0x401921fbu ? 0 : 4;
  }
  if (m > 0) {
    double a = (double)m * p1, at = (double)m * p1t;
    if (!negative) {
      double z = x - a;
      y[0] = z - at;
      y[1] = (z - y[0]) - at;
      return m;
    }
    double z = x + a;
    y[0] = z + at;
    y[1] = (z - y[0]) + at;
    return -m;
  }
  double fn = x * inv_half_pi + round_shift - round_shift;
  int n = (int)fn;
  double r = x - fn * p1, w = fn * p1t;
  y[0] = r - w;
  int ex = (int)(top >> 20);
  int ey = (int)((bits(y[0]) >> 52) & 0x7ff);
  if (ex - ey > 16) {
    double t = r;
    w = fn * p2;
    r = t - w;
    w = fn * p2t - ((t - r) - w);
    y[0] = r - w;
    ey = (int)((bits(y[0]) >> 52) & 0x7ff);
    if (ex - ey > 49) {
      t = r;
      w = fn * p3;
      r = t - w;
      w = fn * p3t - ((t - r) - w);
      y[0] = r - w;
    }
  }
  y[1] = (r - y[0]) - w;
  return n;
}

inline void ref_sincos(double x, double *s, double *c) {
  uint32_t top = (uint32_t)(bits(x) >> 32) & 0x7fffffffu;
  if (top <= 0x3fe921fbu) {  // |x| <= pi/4: no reduction
    if (top < 0x3e46a09eu) {
      *s = x;
      *c = 1.0;
      return;
    }
    *s = kernel_sin(x, 0.0, false);
    *c = kernel_cos(x, 0.0);
    return;
  }
  if (top >= 0x7ff00000u) {
    *s = *c = x - x;
    return;
  }
  if (top >= 0x413921fbu) {  // beyond the medium range: not met by the oracle's runs
    *s = std::sin(x);
    *c = std::cos(x);
    return;
  }
  double y[2];
  int n = reduce_half_pi(x, y);
  double sn = kernel_sin(y[0], y[1], true), cs = kernel_cos(y[0], y[1]);
  switch (n & 3) {
    case 0: *s = sn; *c = cs; break;
    case 1: *s = cs; *c = -sn; break;
    case 2: *s = -sn; *c = -cs; break;
    default: *s = -cs; *c = sn; break;
  }
}

inline double ref_sin(double x) {
  double s, c;
  ref_sincos(x, &s, &c);
  return s;
}

}  // namespace refmath

#endif
