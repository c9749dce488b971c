// FDFD's cell average of a box geometry (src/fdfd/three.rs:563-588), shared by the host library
// (host.cpp: pxs_average) and the device (setup.cu: pxs_average_device), so that both give the
// same bits: the same operations in the same order, f64, no fused multiply-add.
#pragma once
#include <cstdint>

namespace pxa {

__host__ __device__ inline int first_of(int c) { return (c + 1) % 3; }
__host__ __device__ inline int second_of(int c) { return (c + 2) % 3; }

// boxes of 7 doubles {xlo, xhi, ylo, yhi, zlo, zhi, value}: a point inside when lo < p < hi on
// each axis, later boxes over earlier ones, `background` elsewhere
struct BoxView {
  double background;
  int64_t count;
  const double *boxes;
  __host__ __device__ double at(const double p[3]) const {
    double v = background;
    for (int64_t b = 0; b < count; b++) {
      const double *x = boxes + 7 * b;
      if (x[0] < p[0] && p[0] < x[1] && x[2] < p[1] && p[1] < x[3] && x[4] < p[2] && p[2] < x[5])
        v = x[6];
    }
    return v;
  }
};

// E value (component c, index r)'s position: node (i, j, k), half a step along c
__host__ __device__ inline void e_position(const int64_t n[3], const double d[3],
                                           const double o[3], int c, int64_t r, double p[3]) {
  const int64_t i = r % n[0], j = (r / n[0]) % n[1], k = r / (n[0] * n[1]);
  p[0] = o[0] + (double)i * d[0];
  p[1] = o[1] + (double)j * d[1];
  p[2] = o[2] + (double)k * d[2];
  p[c] += 0.5 * d[c];
}

// The cell average of one value, in num-complex's arithmetic on a zero imaginary part:
// 1/eps = eps/(eps eps), n/inverse = n inverse/(inverse inverse).
__host__ __device__ inline double average_cell(const BoxView &geo, const double centre[3],
                                               const double h[3], int along) {
  const int samples = 8;
  const double n = 8.0;
  const int a = along, b = first_of(along), c = second_of(along);
  double sum = 0.0, p[3] = {centre[0], centre[1], centre[2]};
  for (int sb = 0; sb < samples; sb++) {
    p[b] = centre[b] + (((double)sb + 0.5) / n - 0.5) * h[b];
    for (int sc = 0; sc < samples; sc++) {
      p[c] = centre[c] + (((double)sc + 0.5) / n - 0.5) * h[c];
      double inverse = 0.0;
      for (int sa = 0; sa < samples; sa++) {
        p[a] = centre[a] + (((double)sa + 0.5) / n - 0.5) * h[a];
        const double e = geo.at(p);
        inverse += (1.0 * e) / (e * e);
      }
      sum += (n * inverse) / (inverse * inverse);
    }
  }
  return sum / (n * n);
}

// The same average of a uniform value: what every cell away from the boxes' faces gives.
__host__ __device__ inline double average_uniform(double e) {
  const double n = 8.0;
  double sum = 0.0;
  for (int q = 0; q < 64; q++) {
    double inverse = 0.0;
    for (int s = 0; s < 8; s++) inverse += (1.0 * e) / (e * e);
    sum += (n * inverse) / (inverse * inverse);
  }
  return sum / (n * n);
}

// Whether every sample of the cell around `centre` sees the same boxes: along each axis the
// samples run from centre + offset(0) h to centre + offset(7) h, and a box holds all of them or
// none when, on some axis, both ends are outside on the same side, or on every axis both are in.
// Returns the box whose value they all see (-1: the background), or -2 where they differ.
__host__ __device__ inline int64_t uniform_cell(const BoxView &geo, const double centre[3],
                                                const double h[3]) {
  double lo[3], hi[3];
  for (int a = 0; a < 3; a++) {
    lo[a] = centre[a] + ((0.0 + 0.5) / 8.0 - 0.5) * h[a];
    hi[a] = centre[a] + ((7.0 + 0.5) / 8.0 - 0.5) * h[a];
  }
  int64_t which = -1;
  for (int64_t b = 0; b < geo.count; b++) {
    const double *x = geo.boxes + 7 * b;
    bool none = false, all = true;
    for (int a = 0; a < 3; a++) {
      const double blo = x[2 * a], bhi = x[2 * a + 1];
      const bool lo_in = blo < lo[a] && lo[a] < bhi, hi_in = blo < hi[a] && hi[a] < bhi;
      if (!(lo_in && hi_in)) all = false;
      if ((hi[a] <= blo) || (lo[a] >= bhi)) none = true;  // both ends on one side, outside
    }
    if (none) continue;
    if (!all) return -2;
    which = b;
  }
  return which;
}

}  // namespace pxa
