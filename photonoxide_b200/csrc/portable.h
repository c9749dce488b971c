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
// - pxp::ln, the reference's own `portable::ln` (src/portable/mod.rs:141-215), its port of fdlibm's
//   e_log.c: x = 2^k (1 + f) with 1 + f in [sqrt(2)/2, sqrt(2)), log(1 + f) = 2s + s R(s^2) for
//   s = f / (2 + f), R of degree 14 in two interleaved halves, k ln2 with ln2 in two parts.
// - pxp::pow, the published algorithm of the `libm` crate 0.2.16's `pow` that `portable::powf`
//   calls (src/portable/mod.rs:299-301): FreeBSD's port of fdlibm's e_pow.c, with C99's special
//   cases. log2|x| to about 70 bits as t1 + t2 (x reduced to [1, 1.5) or [1.5, 3) against bp = 1
//   or 1.5, s = (x - bp)/(x + bp) and a degree-12 polynomial), y split as y1 + y2 with 32 bits in
//   y1, the product (y1 + y2)(t1 + t2) = n + (p_h + p_l) with n an integer, and 2^(p_h + p_l) by
//   exp's polynomial, scaled by 2^n. Both give the CPML's grading (src/fdtd.rs:811-815):
//   sigma_max = (m + 1)(-ln R)/(2d) and (depth / d)^m.
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

PXP_FN double ln(double x) {
  const double kLn2Hi = 6.93147180369123816490e-01;  // bits 0x3fe62e42fee00000
  const double kLn2Lo = 1.90821492927058770002e-10;  // bits 0x3dea39ef35793c76
  const double kTwo54 = 1.80143985094819840000e+16;  // bits 0x4350000000000000
  const double kLg1 = 6.666666666666735130e-01, kLg2 = 3.999999999940941908e-01,
               kLg3 = 2.857142874366239149e-01, kLg4 = 2.222219843214978396e-01,
               kLg5 = 1.818357216161805012e-01, kLg6 = 1.531383769920937332e-01,
               kLg7 = 1.479819860511658591e-01;
  int k = 0;
  // positive, normal and finite in one comparison; the rest by fdlibm's cases
  if (to_bits(x) - 0x0010000000000000ULL >= 0x7ff0000000000000ULL - 0x0010000000000000ULL) {
    if (x != x || x < 0.0) return of_bits(0x7ff8000000000000ULL);
    if (x == 0.0) return of_bits(0xfff0000000000000ULL);
    if (x == of_bits(0x7ff0000000000000ULL)) return x;
    k -= 54;  // subnormal: scaled up by 2^54
    x *= kTwo54;
  }
  int32_t high = (int32_t)(to_bits(x) >> 32);
  k += (high >> 20) - 1023;
  high &= 0x000fffff;
  const int32_t half = (high + 0x95f64) & 0x100000;  // x or x / 2 into [sqrt(2)/2, sqrt(2))
  const uint32_t top = (uint32_t)(high | (half ^ 0x3ff00000));
  x = of_bits(((uint64_t)top << 32) | (to_bits(x) & 0xffffffffULL));
  k += half >> 20;
  const double f = x - 1.0;
  const double dk = (double)k;
  if ((0x000fffff & (2 + high)) < 3) {  // |f| < 2^-20
    if (f == 0.0) return dk * kLn2Hi + dk * kLn2Lo;
    const double r = f * f * (0.5 - (1.0 / 3.0) * f);
    return k == 0 ? f - r : dk * kLn2Hi - ((r - dk * kLn2Lo) - f);
  }
  const double s = f / (2.0 + f), z = s * s, w = z * z;
  const double t1 = w * (kLg2 + w * (kLg4 + w * kLg6));
  const double t2 = z * (kLg1 + w * (kLg3 + w * (kLg5 + w * kLg7)));
  const double r = t2 + t1;
  if (((high - 0x6147a) | (0x6b851 - high)) > 0) {
    const double hfsq = 0.5 * f * f;
    return k == 0 ? f - (hfsq - s * (hfsq + r))
                  : dk * kLn2Hi - ((hfsq - (s * (hfsq + r) + dk * kLn2Lo)) - f);
  }
  return k == 0 ? f - s * (f - r) : dk * kLn2Hi - ((s * (f - r) - dk * kLn2Lo) - f);
}

PXP_FN double with_low(double x, uint32_t low) {
  return of_bits((to_bits(x) & 0xffffffff00000000ULL) | low);
}
PXP_FN double with_high(double x, uint32_t high) {
  return of_bits((to_bits(x) & 0xffffffffULL) | ((uint64_t)high << 32));
}

PXP_FN double pow(double x, double y) {
  // fdlibm's huge * huge and tiny * tiny: an overflow to infinity and an underflow to zero
  const double kInf = of_bits(0x7ff0000000000000ULL), kTwo53 = 9007199254740992.0;
  const double kBp[2] = {1.0, 1.5};
  const double kDpH[2] = {0.0, 5.84962487220764160156e-01};   // bits 0x3fe2b80340000000
  const double kDpL[2] = {0.0, 1.35003920212974897128e-08};   // bits 0x3e4cfdeb43cfd006
  const double kL1 = 5.99999999999994648725e-01, kL2 = 4.28571428578550184252e-01,
               kL3 = 3.33333329818377432918e-01, kL4 = 2.72728123808534006489e-01,
               kL5 = 2.30660745775561754067e-01, kL6 = 2.06975017800338417784e-01;
  const double kP1 = 1.66666666666666019037e-01, kP2 = -2.77777777770155933842e-03,
               kP3 = 6.61375632143793436117e-05, kP4 = -1.65339022054652515390e-06,
               kP5 = 4.13813679705723846039e-08;
  const double kLg2 = 6.93147180559945286227e-01;       // bits 0x3fe62e42fefa39ef
  const double kLg2H = 6.93147182464599609375e-01;      // bits 0x3fe62e4300000000
  const double kLg2L = -1.90465429995776804525e-09;     // bits 0xbe205c610ca86c39
  const double kOvt = 8.0085662595372944372e-17;        // -(1024 - log2(max + half an ulp))
  const double kCp = 9.61796693925975554329e-01;        // 2/(3 ln2), bits 0x3feec709dc3a03fd
  const double kCpH = 9.61796700954437255859e-01;       // its first 24 bits
  const double kCpL = -7.02846165095275826516e-09;      // the rest
  const double kIvln2 = 1.44269504088896338700e+00;     // 1/ln2
  const double kIvln2H = 1.44269502162933349609e+00;    // its first 24 bits
  const double kIvln2L = 1.92596299112661746887e-08;    // the rest
  const int32_t hx = (int32_t)(to_bits(x) >> 32), hy = (int32_t)(to_bits(y) >> 32);
  const uint32_t lx = (uint32_t)to_bits(x), ly = (uint32_t)to_bits(y);
  int32_t ix = hx & 0x7fffffff;
  const int32_t iy = hy & 0x7fffffff;
  if (((uint32_t)iy | ly) == 0) return 1.0;            // x^0 = 1, even for a NaN x
  if (hx == 0x3ff00000 && lx == 0) return 1.0;         // 1^y = 1, even for a NaN y
  if (ix > 0x7ff00000 || (ix == 0x7ff00000 && lx != 0) || iy > 0x7ff00000 ||
      (iy == 0x7ff00000 && ly != 0))
    return x + y;
  // for a negative x: whether y is an odd (1) or even (2) integer, or neither (0)
  int yisint = 0;
  if (hx < 0) {
    if (iy >= 0x43400000) {
      yisint = 2;
    } else if (iy >= 0x3ff00000) {
      const int e = (iy >> 20) - 0x3ff;
      if (e > 20) {
        const uint32_t j = ly >> (52 - e);
        if ((j << (52 - e)) == ly) yisint = 2 - (int)(j & 1);
      } else if (ly == 0) {
        const int32_t j = iy >> (20 - e);
        if ((j << (20 - e)) == iy) yisint = 2 - (j & 1);
      }
    }
  }
  if (ly == 0) {  // y +-inf, +-1, 2, 1/2
    if (iy == 0x7ff00000) {
      if (((ix - 0x3ff00000) | (int32_t)lx) == 0) return 1.0;   // (-1)^+-inf
      if (ix >= 0x3ff00000) return hy >= 0 ? y : 0.0;          // |x| > 1
      return hy >= 0 ? 0.0 : -y;                               // |x| < 1
    }
    if (iy == 0x3ff00000) return hy >= 0 ? x : 1.0 / x;
    if (hy == 0x40000000) return x * x;
    if (hy == 0x3fe00000 && hx >= 0) return sqrt(x);
  }
  double ax = fabs(x);
  if (lx == 0 && (ix == 0x7ff00000 || ix == 0 || ix == 0x3ff00000)) {  // x +-0, +-inf, +-1
    double z = ax;
    if (hy < 0) z = 1.0 / z;
    if (hx < 0) {
      if (((ix - 0x3ff00000) | yisint) == 0) z = (z - z) / (z - z);  // (-1)^non-integer
      else if (yisint == 1) z = -z;
    }
    return z;
  }
  double sign = 1.0;
  if (hx < 0) {
    if (yisint == 0) return (x - x) / (x - x);  // negative^non-integer
    if (yisint == 1) sign = -1.0;
  }
  double t1, t2;
  if (iy > 0x41e00000) {  // |y| > 2^31
    if (iy > 0x43f00000) {  // |y| > 2^64: over- or underflows
      if (ix <= 0x3fefffff) return hy < 0 ? kInf : 0.0;
      if (ix >= 0x3ff00000) return hy > 0 ? kInf : 0.0;
    }
    if (ix < 0x3fefffff) return hy < 0 ? sign * kInf : sign * 0.0;
    if (ix > 0x3ff00000) return hy > 0 ? sign * kInf : sign * 0.0;
    // |1 - x| <= 2^-20: log x by x - x^2/2 + x^3/3 - x^4/4
    const double t = ax - 1.0;
    const double w = (t * t) * (0.5 - t * (0.3333333333333333333333 - t * 0.25));
    const double u = kIvln2H * t;
    const double v = t * kIvln2L - w * kIvln2;
    t1 = with_low(u + v, 0);
    t2 = v - (t1 - u);
  } else {
    int n = 0;
    if (ix < 0x00100000) {  // subnormal x
      ax *= kTwo53;
      n -= 53;
      ix = (int32_t)(to_bits(ax) >> 32);
    }
    n += (ix >> 20) - 0x3ff;
    const int32_t j = ix & 0x000fffff;
    int k;
    ix = j | 0x3ff00000;
    if (j <= 0x3988e) {         // |x| < sqrt(3/2)
      k = 0;
    } else if (j < 0xbb67a) {   // |x| < sqrt(3)
      k = 1;
    } else {
      k = 0;
      n += 1;
      ix -= 0x00100000;
    }
    ax = with_high(ax, (uint32_t)ix);
    // ss = s_h + s_l = (x - bp)/(x + bp)
    double u = ax - kBp[k];
    double v = 1.0 / (ax + kBp[k]);
    const double ss = u * v;
    const double s_h = with_low(ss, 0);
    double t_h = with_high(0.0, (((uint32_t)ix >> 1) | 0x20000000u) + 0x00080000u + ((uint32_t)k << 18));
    double t_l = ax - (t_h - kBp[k]);
    const double s_l = v * ((u - s_h * t_h) - s_h * t_l);
    // log(ax)
    double s2 = ss * ss;
    double r = s2 * s2 * (kL1 + s2 * (kL2 + s2 * (kL3 + s2 * (kL4 + s2 * (kL5 + s2 * kL6)))));
    r += s_l * (s_h + ss);
    s2 = s_h * s_h;
    t_h = with_low(3.0 + s2 + r, 0);
    t_l = r - ((t_h - 3.0) - s2);
    u = s_h * t_h;
    v = s_l * t_h + t_l * ss;
    const double p_h = with_low(u + v, 0);
    const double p_l = v - (p_h - u);
    const double z_h = kCpH * p_h;
    const double z_l = kCpL * p_h + p_l * kCp + kDpL[k];
    // log2(ax) = n + dp_h + z_h + z_l
    const double t = (double)n;
    t1 = with_low(((z_h + z_l) + kDpH[k]) + t, 0);
    t2 = z_l - (((t1 - t) - kDpH[k]) - z_h);
  }
  // (y1 + y2)(t1 + t2) with y1 the first 32 bits of y
  const double y1 = with_low(y, 0);
  const double p_l = (y - y1) * t1 + y * t2;
  double p_h = y1 * t1;
  double z = p_l + p_h;
  int32_t j = (int32_t)(to_bits(z) >> 32);
  const int32_t i = (int32_t)(uint32_t)to_bits(z);
  if (j >= 0x40900000) {  // z >= 1024
    if (((j - 0x40900000) | i) != 0) return sign * kInf;
    if (p_l + kOvt > z - p_h) return sign * kInf;
  } else if ((j & 0x7fffffff) >= 0x4090cc00) {  // z <= -1075
    if ((((uint32_t)j - 0xc090cc00u) | (uint32_t)i) != 0) return sign * 0.0;
    if (p_l <= z - p_h) return sign * 0.0;
  }
  // 2^(p_h + p_l): n the nearest integer when |z| > 1/2
  const int32_t iz = j & 0x7fffffff;
  int k = (iz >> 20) - 0x3ff;
  int n = 0;
  if (iz > 0x3fe00000) {
    n = j + (0x00100000 >> (k + 1));
    k = ((n & 0x7fffffff) >> 20) - 0x3ff;
    const double t = with_high(0.0, (uint32_t)(n & ~(0x000fffff >> k)));
    n = ((n & 0x000fffff) | 0x00100000) >> (20 - k);
    if (j < 0) n = -n;
    p_h -= t;
  }
  const double t = with_low(p_l + p_h, 0);
  const double u = t * kLg2H;
  const double v = (p_l - (t - p_h)) * kLg2 + t * kLg2L;
  z = u + v;
  const double w = v - (z - u);
  const double tt = z * z;
  const double c = z - tt * (kP1 + tt * (kP2 + tt * (kP3 + tt * (kP4 + tt * kP5))));
  const double r = (z * c) / (c - 2.0) - (w + z * w);
  z = 1.0 - (r - z);
  j = (int32_t)(to_bits(z) >> 32);
  j += (int32_t)((uint32_t)n << 20);
  if ((j >> 20) <= 0) z = ldexp(z, n);  // a subnormal result: one rounding
  else z = with_high(z, (uint32_t)j);
  return sign * z;
}

}  // namespace pxp

#endif
