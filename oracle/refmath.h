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
// - ref_ln restates photonoxide's own `portable::ln` (src/portable/mod.rs:141-215), its port of
//   fdlibm's e_log.c (x = 2^k m, m in [sqrt(2)/2, sqrt(2)); log m from s = (m-1)/(m+1) and a
//   degree-14 odd series in two interleaved parts).
// - ref_pow restates the `libm` crate 0.2.16's `pow` (FreeBSD's port of fdlibm's e_pow.c with
//   C99's special cases), which `portable::powf` calls (src/portable/mod.rs:299-301): log2|x| to
//   extra precision, times y split in two, then 2^result by exp's polynomial.
// The reference's grid hashes of exp, ln and powf (src/portable/tests.rs:355-556) pin all three.
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

inline double hi_word_set(double x, uint32_t hw) {
  return from_bits((bits(x) & 0xffffffffULL) | ((uint64_t)hw << 32));
}
inline double lo_word_cleared(double x) { return from_bits(bits(x) & 0xffffffff00000000ULL); }

// photonoxide's natural logarithm (fdlibm's e_log.c as the reference ports it).
inline double ref_ln(double x) {
  const double ln2_hi = from_bits(0x3fe62e42fee00000ULL), ln2_lo = from_bits(0x3dea39ef35793c76ULL);
  const double two54 = from_bits(0x4350000000000000ULL);
  const double lg[8] = {0.0,
                        from_bits(0x3fe5555555555593ULL), from_bits(0x3fd999999997fa04ULL),
                        from_bits(0x3fd2492494229359ULL), from_bits(0x3fcc71c51d8e78afULL),
                        from_bits(0x3fc7466496cb03deULL), from_bits(0x3fc39a09d078c69fULL),
                        from_bits(0x3fc2f112df3e5244ULL)};
  int k = 0;
  if (bits(x) - 0x0010000000000000ULL >= 0x7ff0000000000000ULL - 0x0010000000000000ULL) {
    if (std::isnan(x) || x < 0.0) return NAN;
    if (x == 0.0) return -INFINITY;
    if (std::isinf(x)) return x;
    k = -54;
    x *= two54;
  }
  int32_t high = (int32_t)(bits(x) >> 32);
  k += (high >> 20) - 1023;
  high &= 0x000fffff;
  int32_t i = (high + 0x95f64) & 0x100000;
  x = hi_word_set(x, (uint32_t)(high | (i ^ 0x3ff00000)));
  k += i >> 20;
  double f = x - 1.0, dk = (double)k;
  if ((0x000fffff & (2 + high)) < 3) {
    if (f == 0.0) return dk * ln2_hi + dk * ln2_lo;
    double r = f * f * (0.5 - (1.0 / 3.0) * f);
    if (k == 0) return f - r;
    return dk * ln2_hi - ((r - dk * ln2_lo) - f);
  }
  double s = f / (2.0 + f);
  double z = s * s;
  double w = z * z;
  double r = z * (lg[1] + w * (lg[3] + w * (lg[5] + w * lg[7]))) +
             w * (lg[2] + w * (lg[4] + w * lg[6]));
  if (((high - 0x6147a) | (0x6b851 - high)) > 0) {
    double hfsq = 0.5 * f * f;
    if (k == 0) return f - (hfsq - s * (hfsq + r));
    return dk * ln2_hi - ((hfsq - (s * (hfsq + r) + dk * ln2_lo)) - f);
  }
  if (k == 0) return f - s * (f - r);
  return dk * ln2_hi - ((s * (f - r) - dk * ln2_lo) - f);
}

// x to the power y: the `libm` crate's pow (fdlibm's e_pow.c as FreeBSD keeps it).
inline double ref_pow(double x, double y) {
  const double bp[2] = {1.0, 1.5};
  const double dp_h[2] = {0.0, from_bits(0x3fe2b80340000000ULL)};
  const double dp_l[2] = {0.0, from_bits(0x3e4cfdeb43cfd006ULL)};
  const double L[7] = {0.0, from_bits(0x3fe3333333333303ULL), from_bits(0x3fdb6db6db6fabffULL),
                       from_bits(0x3fd55555518f264dULL), from_bits(0x3fd17460a91d4101ULL),
                       from_bits(0x3fcd864a93c9db65ULL), from_bits(0x3fca7e284a454eefULL)};
  const double P[6] = {0.0, from_bits(0x3fc555555555553eULL), from_bits(0xbf66c16c16bebd93ULL),
                       from_bits(0x3f11566aaf25de2cULL), from_bits(0xbebbbd41c5d26bf1ULL),
                       from_bits(0x3e66376972bea4d0ULL)};
  const double lg2 = from_bits(0x3fe62e42fefa39efULL), lg2_h = from_bits(0x3fe62e4300000000ULL),
               lg2_l = from_bits(0xbe205c610ca86c39ULL);
  const double ovt = 8.0085662595372944372e-17;
  const double cp = from_bits(0x3feec709dc3a03fdULL), cp_h = from_bits(0x3feec709e0000000ULL),
               cp_l = from_bits(0xbe3e2fe0145b01f5ULL);
  const double ivln2 = from_bits(0x3ff71547652b82feULL), ivln2_h = from_bits(0x3ff7154760000000ULL),
               ivln2_l = from_bits(0x3e54ae0bf85ddf44ULL);
  const double inf = INFINITY, two53 = 9007199254740992.0;
  int32_t hx = (int32_t)(bits(x) >> 32), hy = (int32_t)(bits(y) >> 32);
  uint32_t lx = (uint32_t)bits(x), ly = (uint32_t)bits(y);
  int32_t ix = hx & 0x7fffffff, iy = hy & 0x7fffffff;
  if ((iy | (int32_t)ly) == 0) return 1.0;
  if (hx == 0x3ff00000 && lx == 0) return 1.0;
  if (ix > 0x7ff00000 || (ix == 0x7ff00000 && lx != 0) || iy > 0x7ff00000 ||
      (iy == 0x7ff00000 && ly != 0))
    return x + y;
  int yisint = 0;  // for x < 0: 0 y not an integer, 1 odd, 2 even
  if (hx < 0) {
    if (iy >= 0x43400000) {
      yisint = 2;
    } else if (iy >= 0x3ff00000) {
      int e = (iy >> 20) - 0x3ff;
      if (e > 20) {
        uint32_t jj = ly >> (52 - e);
        if ((jj << (52 - e)) == ly) yisint = 2 - (int)(jj & 1u);
      } else if (ly == 0) {
        int32_t jj = iy >> (20 - e);
        if ((jj << (20 - e)) == iy) yisint = 2 - (jj & 1);
      }
    }
  }
  if (ly == 0) {
    if (iy == 0x7ff00000) {
      if (((ix - 0x3ff00000) | (int32_t)lx) == 0) return 1.0;
      if (ix >= 0x3ff00000) return hy >= 0 ? y : 0.0;
      return hy >= 0 ? 0.0 : -y;
    }
    if (iy == 0x3ff00000) return hy >= 0 ? x : 1.0 / x;
    if (hy == 0x40000000) return x * x;
    if (hy == 0x3fe00000 && hx >= 0) return std::sqrt(x);
  }
  double ax = std::fabs(x);
  if (lx == 0 && (ix == 0x7ff00000 || ix == 0 || ix == 0x3ff00000)) {
    double z = hy < 0 ? 1.0 / ax : ax;
    if (hx < 0) {
      if (((ix - 0x3ff00000) | yisint) == 0) z = (z - z) / (z - z);
      else if (yisint == 1) z = -z;
    }
    return z;
  }
  double sgn = 1.0;
  if (hx < 0) {
    if (yisint == 0) return (x - x) / (x - x);
    if (yisint == 1) sgn = -1.0;
  }
  double t1, t2;
  if (iy > 0x41e00000) {
    if (iy > 0x43f00000) {
      if (ix <= 0x3fefffff) return hy < 0 ? inf : 0.0;
      if (ix >= 0x3ff00000) return hy > 0 ? inf : 0.0;
    }
    if (ix < 0x3fefffff) return hy < 0 ? sgn * inf : sgn * 0.0;
    if (ix > 0x3ff00000) return hy > 0 ? sgn * inf : sgn * 0.0;
    double t = ax - 1.0;
    double w = (t * t) * (0.5 - t * (0.3333333333333333333333 - t * 0.25));
    double u = ivln2_h * t;
    double v = t * ivln2_l - w * ivln2;
    t1 = lo_word_cleared(u + v);
    t2 = v - (t1 - u);
  } else {
    int n = 0;
    if (ix < 0x00100000) {
      ax *= two53;
      n -= 53;
      ix = (int32_t)(bits(ax) >> 32);
    }
    n += (ix >> 20) - 0x3ff;
    int32_t jm = ix & 0x000fffff;
    int k = 0;
    ix = jm | 0x3ff00000;
    if (jm <= 0x3988e) {
      k = 0;
    } else if (jm < 0xbb67a) {
      k = 1;
    } else {
      k = 0;
      n += 1;
      ix -= 0x00100000;
    }
    ax = hi_word_set(ax, (uint32_t)ix);
    double u = ax - bp[k];
    double v = 1.0 / (ax + bp[k]);
    double ss = u * v;
    double s_h = lo_word_cleared(ss);
    double t_h = hi_word_set(0.0, (((uint32_t)ix >> 1) | 0x20000000u) + 0x00080000u + ((uint32_t)k << 18));
    double t_l = ax - (t_h - bp[k]);
    double s_l = v * ((u - s_h * t_h) - s_h * t_l);
    double s2 = ss * ss;
    double r = s2 * s2 * (L[1] + s2 * (L[2] + s2 * (L[3] + s2 * (L[4] + s2 * (L[5] + s2 * L[6])))));
    r += s_l * (s_h + ss);
    s2 = s_h * s_h;
    t_h = lo_word_cleared(3.0 + s2 + r);
    t_l = r - ((t_h - 3.0) - s2);
    u = s_h * t_h;
    v = s_l * t_h + t_l * ss;
    double p_h = lo_word_cleared(u + v);
    double p_l = v - (p_h - u);
    double z_h = cp_h * p_h;
    double z_l = cp_l * p_h + p_l * cp + dp_l[k];
    double t = (double)n;
    t1 = lo_word_cleared(((z_h + z_l) + dp_h[k]) + t);
    t2 = z_l - (((t1 - t) - dp_h[k]) - z_h);
  }
  double y1 = lo_word_cleared(y);
  double p_l = (y - y1) * t1 + y * t2;
  double p_h = y1 * t1;
  double z = p_l + p_h;
  int32_t j = (int32_t)(bits(z) >> 32);
  int32_t i = (int32_t)(uint32_t)bits(z);
  if (j >= 0x40900000) {
    if (((j - 0x40900000) | i) != 0) return sgn * inf;
    if (p_l + ovt > z - p_h) return sgn * inf;
  } else if ((j & 0x7fffffff) >= 0x4090cc00) {
    if ((((uint32_t)j - 0xc090cc00u) | (uint32_t)i) != 0) return sgn * 0.0;
    if (p_l <= z - p_h) return sgn * 0.0;
  }
  int32_t a = j & 0x7fffffff;
  int k = (a >> 20) - 0x3ff;
  int n = 0;
  if (a > 0x3fe00000) {
    n = j + (0x00100000 >> (k + 1));
    k = ((n & 0x7fffffff) >> 20) - 0x3ff;
    double t = hi_word_set(0.0, (uint32_t)(n & ~(0x000fffff >> k)));
    n = ((n & 0x000fffff) | 0x00100000) >> (20 - k);
    if (j < 0) n = -n;
    p_h -= t;
  }
  double t = lo_word_cleared(p_l + p_h);
  double u = t * lg2_h;
  double v = (p_l - (t - p_h)) * lg2 + t * lg2_l;
  z = u + v;
  double w = v - (z - u);
  t = z * z;
  double c = z - t * (P[1] + t * (P[2] + t * (P[3] + t * (P[4] + t * P[5]))));
  double r = (z * c) / (c - 2.0) - (w + z * w);
  z = 1.0 - (r - z);
  j = (int32_t)(bits(z) >> 32) + (int32_t)((uint32_t)n << 20);
  if ((j >> 20) <= 0) return sgn * std::ldexp(z, n);
  return sgn * hi_word_set(z, (uint32_t)j);
}

inline double ref_sin(double x) {
  double s, c;
  ref_sincos(x, &s, &c);
  return s;
}

}  // namespace refmath

#endif
