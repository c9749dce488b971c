// Compares the engine's portable maths (photonoxide_b200/csrc/portable.h) with the oracle's
// restatement of the reference's (oracle/refmath.h) bit for bit; prints the mismatches.
#include <cstdio>
#include <cstdint>
#include <cstring>
#include "portable.h"
#include "refmath.h"
static uint64_t b(double x) { uint64_t u; std::memcpy(&u, &x, 8); return u; }
int main() {
  uint64_t state = 0x243f6a8885a308d3ULL, bad = 0, n = 0;
  auto next = [&]() { state = state * 6364136223846793005ULL + 1442695040888963407ULL; return state; };
  for (int q = 0; q < 2000000; q++) {
    double u = (double)(next() >> 11) / 9007199254740992.0;
    double scale = (q % 4 == 0) ? 1.0 : (q % 4 == 1 ? 40.0 : (q % 4 == 2 ? 3000.0 : 0.01));
    double x = (2.0 * u - 1.0) * scale;
    double s1, c1, s2, c2;
    pxp::sincos(x, &s1, &c1);
    refmath::ref_sincos(x, &s2, &c2);
    if (b(s1) != b(s2) || b(c1) != b(c2)) bad++;
    double e = (2.0 * u - 1.0) * (q % 3 == 0 ? 700.0 : 5.0);
    if (b(pxp::exp(e)) != b(refmath::ref_exp(e))) bad++;
    n += 2;
  }
  printf("%llu %llu\n", (unsigned long long)bad, (unsigned long long)n);
  return 0;
}
