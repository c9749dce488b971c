// The bit-stable maths photonoxide's FDTD path calls, on the host and on the device alike, so the
// engine's setup tables, source waveforms and transform phases carry the reference's bits:
//
// - pxp::exp, the reference's own `portable::exp` (src/portable/mod.rs:66-139), its port of
//   fdlibm's e_exp.c: x = k ln2 + r with ln2 in two parts, fdlibm's degree-5 correction in r^2,
//   2^k through the exponent bits. It gives the CPML's b = exp(-(sigma/kappa + alpha) dt)
//   (src/fdtd.rs:832-842) and the Gaussian envelopes (src/fdtd.rs:329-423).
// - pxp::sincos, the published algorithm of the `libm` crate 0.2.16 (Cargo.lock:2756-2758) that
//   `portable::sin_cos` calls (src/portable/mod.rs:321-323): reduction by pi/2 with pi/2 in three
//   parts (refined while cancellation eats bits) and the kernels r + r^3 S(r^2) and
//   1 - r^2/2 + r^4 C(r^2). Arguments beyond 2^20 pi/2 (never met: a time of order 10^3 um/c
//   times a frequency of order 10 rad/um) take the C library's / CUDA's functions instead.
//
// Compile without floating-point contraction (-ffp-contract=off, nvcc --fmad=false): each
// operation is one IEEE double rounding, in the order the methods fix.
#ifndef PHOTONOXIDE_B200_PORTABLE_H
#define PHOTONOXIDE_B200_PORTABLE_H

#include <cmath>
#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define PXP_FN __host__ __device__ inline
#else
#define PXP_FN inline
#endif

namespace pxp {

PXP_FN uint64_t to_bits(double x) {
#ifdef __CUDA_ARCH__
  return (uint64_t)__double_as_longlong(x);
#else
  uint64_t u;
  std::memcpy(&u, &x, 8);
  return u;
#endif
}
PXP_FN double of_bits(uint64_t u) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)u);
#else
  double x;
  std::memcpy(&x, &u, 8);
  return x;
#endif
}

PXP_FN double exp(double x) {
  const double kOver = 7.09782712893383973096e+02;    // bits 0x40862e42fefa39ef
  const double kUnder = -7.45133219101941108420e+02;  // bits 0xc0874910d52d3051
  const double kLn2Hi = 6.93147180369123816490e-01;   // bits 0x3fe62e42fee00000
  const double kLn2Lo = 1.90821492927058770002e-10;   // bits 0x3dea39ef35793c76
  const double kInvLn2 = 1.44269504088896338700e+00;  // bits 0x3ff71547652b82fe
  const double kP1 = 1.66666666666666019037e-01, kP2 = -2.77777777770155933842e-03,
               kP3 = 6.61375632143793436117e-05, kP4 = -1.65339022054652515390e-06,
               kP5 = 4.13813679705723846039e-08;
  const uint32_t word = (uint32_t)(to_bits(x) >> 32);
  const bool neg = (word >> 31) != 0;
  const uint32_t mag = word & 0x7fffffffu;
  if (mag >= 0x40862e42u) {
    if (x != x) return x;
    if (x > kOver) return of_bits(0x7ff0000000000000ULL);
    if (x < kUnder) return 0.0;
  }
  int k = 0;
  double hi = 0.0, lo = 0.0;
  if (mag > 0x3fd62e42u) {
    if (mag < 0x3ff0a2b2u) {
      k = neg ? -1 : 1;
      hi = neg ? x + kLn2Hi : x - kLn2Hi;
      lo = neg ? -kLn2Lo : kLn2Lo;
    } else {
      k = (int)(kInvLn2 * x + (neg ? -0.5 : 0.5));
      const double kd = (double)k;
      hi = x - kd * kLn2Hi;
      lo = kd * kLn2Lo;
    }
    x = hi - lo;
  } else if (mag < 0x3e300000u) {
    return 1.0 + x;
  }
  const double x2 = x * x;
  const double c = x - x2 * (kP1 + x2 * (kP2 + x2 * (kP3 + x2 * (kP4 + x2 * kP5))));
  if (k == 0) return 1.0 - ((x * c) / (c - 2.0) - x);
  const double y = 1.0 - ((lo - (x * c) / (2.0 - c)) - hi);
  if (k >= -1021) return of_bits(to_bits(y) + ((uint64_t)(int64_t)k << 52));
  return of_bits(to_bits(y) + ((uint64_t)(int64_t)(k + 1000) << 52)) *
         of_bits(0x0170000000000000ULL);
}

// sin(r) and cos(r) on a reduced argument r = x + y, |r| <= pi/4 (y the tail, 0 if none)
PXP_FN double sin_kernel(double x, double y, bool tail) {
  const double s1 = -1.66666666666666324348e-01, s2 = 8.33333333332248946124e-03,
               s3 = -1.98412698298579493134e-04, s4 = 2.75573137070700676789e-06,
               s5 = -2.50507602534068634195e-08, s6 = 1.58969099521155010221e-10;
  const double z = x * x, w = z * z;
  const double r = s2 + z * (s3 + z * s4) + z * w * (s5 + z * s6);
  const double v = z * x;
  if (!tail) return x + v * (s1 + z * r);
  return x - ((z * (0.5 * y - v * r) - y) - v * s1);
}
PXP_FN double cos_kernel(double x, double y) {
  const double c1 = 4.16666666666666019037e-02, c2 = -1.38888888888741095749e-03,
               c3 = 2.48015872894767294178e-05, c4 = -2.75573143513906633035e-07,
               c5 = 2.08757232129817482790e-09, c6 = -1.13596475577881948265e-11;
  const double z = x * x, w = z * z;
  const double r = z * (c1 + z * (c2 + z * c3)) + w * w * (c4 + z * (c5 + z * c6));
  const double hz = 0.5 * z;
  const double one = 1.0 - hz;
  return one + (((1.0 - one) - hz) + (z * r - x * y));
}

// x = n pi/2 + y[0] + y[1] for |x| below 2^20 pi/2; returns n
PXP_FN int reduce(double x, double y[2]) {
  const double inv_pio2 = 6.36619772367581382433e-01;
  const double p1 = 1.57079632673412561417e+00, p1t = 6.07710050650619224932e-11;
  const double p2 = 6.07710050630396597660e-11, p2t = 2.02226624879595063154e-21;
  const double p3 = 2.02226624871116645580e-21, p3t = 8.47842766036889956997e-32;
  const double shift = 6755399441055744.0;  // 1.5 * 2^52
  const uint64_t u = to_bits(x);
  const bool neg = (u >> 63) != 0;
  const uint32_t mag = (uint32_t)(u >> 32) & 0x7fffffffu;
  // up to 9 pi/4: m quarter turns of (p1 + p1t) at once, unless x is near a multiple of pi/2
  int m = 0;
  if (mag <= 0x400f6a7au) {
    if ((mag & 0xfffffu) != 0x921fbu) m = mag <= 0x4002d97cu ? 1 : 2;
  } else if (mag <= 0x401c463bu) {
    if (mag <= 0x4015fdbcu) m = mag == 0x4012d97cu ? 0 : 3;
    else m = mag == 0x401921fbu ? 0 : 4;
  }
  if (m > 0) {
    const double a = (double)m * p1, at = (double)m * p1t;
    if (!neg) {
      const double z = x - a;
      y[0] = z - at;
      y[1] = (z - y[0]) - at;
      return m;
    }
    const double z = x + a;
    y[0] = z + at;
    y[1] = (z - y[0]) + at;
    return -m;
  }
  const double fn = x * inv_pio2 + shift - shift;
  const int n = (int)fn;
  double r = x - fn * p1, w = fn * p1t;
  y[0] = r - w;
  const int ex = (int)(mag >> 20);
  int ey = (int)((to_bits(y[0]) >> 52) & 0x7ff);
  if (ex - ey > 16) {
    double t = r;
    w = fn * p2;
    r = t - w;
    w = fn * p2t - ((t - r) - w);
    y[0] = r - w;
    ey = (int)((to_bits(y[0]) >> 52) & 0x7ff);
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

PXP_FN void sincos(double x, double *s, double *c) {
  const uint32_t mag = (uint32_t)(to_bits(x) >> 32) & 0x7fffffffu;
  if (mag <= 0x3fe921fbu) {
    if (mag < 0x3e46a09eu) {
      *s = x;
      *c = 1.0;
      return;
    }
    *s = sin_kernel(x, 0.0, false);
    *c = cos_kernel(x, 0.0);
    return;
  }
  if (mag >= 0x7ff00000u) {
    *s = *c = x - x;
    return;
  }
  if (mag >= 0x413921fbu) {
    *s = ::sin(x);
    *c = ::cos(x);
    return;
  }
  double y[2];
  const int n = reduce(x, y);
  const double sn = sin_kernel(y[0], y[1], true), cs = cos_kernel(y[0], y[1]);
  switch (n & 3) {
    case 0: *s = sn; *c = cs; break;
    case 1: *s = cs; *c = -sn; break;
    case 2: *s = -sn; *c = -cs; break;
    default: *s = -cs; *c = sn; break;
  }
}

}  // namespace pxp

#endif
