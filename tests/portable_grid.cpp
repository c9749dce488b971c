// The reference's bit canary for its portable maths (src/portable/tests.rs:345-511), restated: the
// same grid of 620 arguments (special values, the subnormals' edge, 600 from a fixed LCG over
// several scales), pairs (x[i], x[619 - i]) for the two-argument functions, and the same
// order-sensitive fold of each result's bits (NaN folded as one NaN). Prints, for the engine's
// portable maths (photonoxide_b200/csrc/portable.h) and for the oracle's (oracle/refmath.h), the
// hash of each function the FDTD path calls.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <vector>

#include "portable.h"
#include "refmath.h"

static uint64_t bits_of(double x) {
  uint64_t u;
  std::memcpy(&u, &x, 8);
  return u;
}
static void fold(uint64_t &h, double v) {
  if (v != v) v = std::numeric_limits<double>::quiet_NaN();  // 0x7ff8000000000000
  h = ((h << 7) | (h >> 57)) ^ bits_of(v);
}

static std::vector<double> grid() {
  const double inf = std::numeric_limits<double>::infinity();
  const double dmax = std::numeric_limits<double>::max();
  double tiny, three;
  uint64_t one = 1, t3 = 3;
  std::memcpy(&tiny, &one, 8);
  std::memcpy(&three, &t3, 8);
  std::vector<double> xs = {0.0, -0.0, inf, -inf, std::numeric_limits<double>::quiet_NaN(),
                            std::numeric_limits<double>::min(), tiny, -three, dmax, -dmax,
                            1.0, -1.0, 0.5, 2.0, 3.141592653589793, 1.5707963267948966, 1e22,
                            -709.5, 710.0, 26.5};
  uint64_t s = 0x0822202611130001ULL;
  auto unit = [&]() {
    s = s * 6364136223846793005ULL + 1442695040888963407ULL;
    return (double)(s >> 11) / 9007199254740992.0;
  };
  for (double scale : {1.0, 4.0, 30.0, 800.0, 1e6})
    for (int q = 0; q < 120; q++) xs.push_back((unit() - 0.5) * 2.0 * scale);
  return xs;
}

template <typename F>
static uint64_t over_grid(const std::vector<double> &xs, F f) {
  uint64_t h = 0;
  for (double x : xs) fold(h, f(x));
  return h;
}
template <typename F>
static uint64_t over_pairs(const std::vector<double> &xs, F f) {
  uint64_t h = 0;
  for (size_t i = 0; i < xs.size(); i++) fold(h, f(xs[i], xs[xs.size() - 1 - i]));
  return h;
}

int main() {
  const std::vector<double> xs = grid();
  auto sin0 = [](double x) { double s, c; pxp::sincos(x, &s, &c); return s; };
  auto cos0 = [](double x) { double s, c; pxp::sincos(x, &s, &c); return c; };
  auto sin1 = [](double x) { double s, c; refmath::ref_sincos(x, &s, &c); return s; };
  auto cos1 = [](double x) { double s, c; refmath::ref_sincos(x, &s, &c); return c; };
  printf("engine exp %016llx\n", (unsigned long long)over_grid(xs, [](double x) { return pxp::exp(x); }));
  printf("engine ln %016llx\n", (unsigned long long)over_grid(xs, [](double x) { return pxp::ln(x); }));
  printf("engine sin_cos.0 %016llx\n", (unsigned long long)over_grid(xs, sin0));
  printf("engine sin_cos.1 %016llx\n", (unsigned long long)over_grid(xs, cos0));
  printf("engine powf %016llx\n",
         (unsigned long long)over_pairs(xs, [](double a, double b) { return pxp::pow(a, b); }));
  printf("oracle exp %016llx\n", (unsigned long long)over_grid(xs, [](double x) { return refmath::ref_exp(x); }));
  printf("oracle ln %016llx\n", (unsigned long long)over_grid(xs, [](double x) { return refmath::ref_ln(x); }));
  printf("oracle sin_cos.0 %016llx\n", (unsigned long long)over_grid(xs, sin1));
  printf("oracle sin_cos.1 %016llx\n", (unsigned long long)over_grid(xs, cos1));
  printf("oracle powf %016llx\n",
         (unsigned long long)over_pairs(xs, [](double a, double b) { return refmath::ref_pow(a, b); }));
  return 0;
}
