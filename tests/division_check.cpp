// The engine's division by a grid step (div_by_step, photonoxide_b200/csrc/common.cuh) against
// x / h on the host, which has the same IEEE single-precision arithmetic (fused fmaf, correctly
// rounded division, subnormals): every `stride`-th bit pattern of the finite floats, plus every
// pattern below 2^-80. Prints the mismatches and the count compared.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "common.cuh"

int main(int argc, char **argv) {
  const float h = (float)std::atof(argv[1]);
  const long long stride = std::atoll(argv[2]);
  const float r = (float)(1.0 / (double)h);
  long long bad = 0, total = 0;
  auto one = [&](uint32_t u) {
    float x;
    std::memcpy(&x, &u, 4);
    if (!std::isfinite(x)) return;
    const float q = pxf::div_by_step(x, h, r, 1.0 / (double)h, 1), want = x / h;
    uint32_t a, b;
    std::memcpy(&a, &q, 4);
    std::memcpy(&b, &want, 4);
    bad += a != b;
    total++;
  };
  for (long long i = 0; i < (1LL << 32); i += stride) one((uint32_t)i);
  for (uint32_t e = 0; e < (uint32_t)(127 - 80) << 23; e++) {  // |x| < 2^-80, both signs
    one(e);
    one(e | 0x80000000u);
  }
  std::printf("%lld %lld\n", bad, total);
  return 0;
}
