// Set-up on the device: FDFD's cell average of a box geometry at every E value (the same
// functions as the host library's pxs_average, average.cuh, so the same bits), one thread per
// value. Cells whose samples all see one value take that value's average from a table made on
// the host; the others take the 8^3-sample average. And the CPML's tables (the same functions as
// the host library's build_cpml, cpml.cuh), one thread per node of each axis.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <vector>

#include "average.cuh"
#include "cpml.cuh"
#include "photonoxide_sim.h"

namespace {

struct AverageArgs {
  int64_t n[3];
  double d[3], o[3];
  pxa::BoxView geo;
  const double *uniform;  // the average of the background (0) and of each box's value (1 + b)
  double *out;
  int64_t total;          // 3 x cells
};

__global__ void average_kernel(AverageArgs A) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= A.total) return;
  const int64_t N = A.n[0] * A.n[1] * A.n[2];
  const int c = (int)(q / N);
  double p[3];
  pxa::e_position(A.n, A.d, A.o, c, q - (int64_t)c * N, p);
  const int64_t b = pxa::uniform_cell(A.geo, p, A.d);
  A.out[q] = b == -2 ? pxa::average_cell(A.geo, p, A.d, c) : A.uniform[b + 1];
}

struct CpmlArgs {
  int64_t n[3], lo[3], hi[3];
  int periodic[3];
  double d[3], cpml[5], dt;
  double *kn, *kh, *b0, *a0, *b1, *a1;  // sum of n values each, axis by axis
  int64_t total;
};

// Node m of an axis: kappa at m and m + 1/2 (as 1/kappa/h), and the psi recursion's b and a there.
__global__ void cpml_kernel(CpmlArgs A) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= A.total) return;
  int axis = 0;
  int64_t m = q;
  while (axis < 2 && m >= A.n[axis]) {
    m -= A.n[axis];
    axis++;
  }
  double s0 = 0.0, k0 = 1.0, s1 = 0.0, k1 = 1.0;
  if (!A.periodic[axis]) {
    pxc::grade((double)m, A.lo[axis], A.hi[axis], A.n[axis], A.d[axis], A.cpml, &s0, &k0);
    pxc::grade((double)m + 0.5, A.lo[axis], A.hi[axis], A.n[axis], A.d[axis], A.cpml, &s1, &k1);
  }
  A.kn[q] = (1.0 / k0) / A.d[axis];
  A.kh[q] = (1.0 / k1) / A.d[axis];
  pxc::recursion(s0, k0, A.cpml[4], A.dt, &A.b0[q], &A.a0[q]);
  pxc::recursion(s1, k1, A.cpml[4], A.dt, &A.b1[q], &A.a1[q]);
}

}  // namespace

extern "C" int64_t pxs_cpml_device(const int64_t n[3], const double d[3], const int32_t kind[3],
                                   const int64_t low[3], const int64_t high[3],
                                   const double cpml[5], double dt, int32_t which, double *out) {
  if (!n || !d || !kind || !low || !high || !cpml || which < 2 || which > 4) return -1;
  int64_t total = 0, count = 0;
  for (int a = 0; a < 3; a++) {
    if (n[a] <= 0 || low[a] < 0 || high[a] < 0 || low[a] + high[a] > n[a]) return -1;
    total += n[a];
    if (kind[a] != 1)
      for (int64_t c : {low[a], high[a]})
        if (c > 0) count += 2 * 2 * (5 + 2 * c);  // two fields, two components each
  }
  const int64_t size = which == 4 ? count : total;
  if (!out) return size;
  CpmlArgs A;
  for (int a = 0; a < 3; a++) {
    A.n[a] = n[a];
    A.lo[a] = low[a];
    A.hi[a] = high[a];
    A.periodic[a] = kind[a] == 1;
    A.d[a] = d[a];
  }
  for (int i = 0; i < 5; i++) A.cpml[i] = cpml[i];
  A.dt = dt;
  A.total = total;
  std::vector<double> host(6 * total);
  double *dev = nullptr;
  cudaStream_t st = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  auto step = [&](auto &&call) {
    if (e == cudaSuccess) e = call();
  };
  step([&] { return cudaMallocAsync(&dev, (size_t)(6 * total) * 8, st); });
  step([&] {
    A.kn = dev;
    A.kh = dev + total;
    A.b0 = dev + 2 * total;
    A.a0 = dev + 3 * total;
    A.b1 = dev + 4 * total;
    A.a1 = dev + 5 * total;
    cpml_kernel<<<(unsigned)((total + 127) / 128), 128, 0, st>>>(A);
    return cudaGetLastError();
  });
  step([&] {
    return cudaMemcpyAsync(host.data(), dev, (size_t)(6 * total) * 8, cudaMemcpyDeviceToHost, st);
  });
  if (st) {
    if (dev) cudaFreeAsync(dev, st);
    const cudaError_t done = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = done;
    cudaStreamDestroy(st);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return -2;
  }
  if (which != 4) {
    std::copy(host.begin() + (which == 2 ? 0 : total), host.begin() + (which == 2 ? 1 : 2) * total,
              out);
    return size;
  }
  // the slabs as the host library lists them (pxs_tables 4): by axis, side, field, component
  int64_t at = 0, base = 0;
  for (int a = 0; a < 3; a++) {
    const int64_t froms[2] = {0, n[a] - high[a]}, counts[2] = {low[a], high[a]};
    for (int side = 0; side < 2 && kind[a] != 1; side++) {
      if (counts[side] == 0) continue;
      for (int field = 0; field < 2; field++)
        for (int comp : {(a + 1) % 3, (a + 2) % 3}) {
          out[at++] = field;
          out[at++] = comp;
          out[at++] = a;
          out[at++] = (double)froms[side];
          out[at++] = (double)counts[side];
          const double *b = host.data() + (2 + 2 * field) * total + base + froms[side];
          const double *c = host.data() + (3 + 2 * field) * total + base + froms[side];
          for (int64_t m = 0; m < counts[side]; m++) out[at++] = b[m];
          for (int64_t m = 0; m < counts[side]; m++) out[at++] = c[m];
        }
    }
    base += n[a];
  }
  return at;
}

extern "C" int pxs_average_device(const int64_t n[3], const double d[3], const double o[3],
                                  const pxs_geometry *g, double *out) {
  if (!n || !d || !o || !out || n[0] <= 0 || n[1] <= 0 || n[2] <= 0) return -1;
  const int64_t total = 3 * n[0] * n[1] * n[2];
  const int64_t nb = g ? g->nboxes : 0;
  std::vector<double> boxes(g && nb > 0 ? g->boxes : (const double *)nullptr,
                            g && nb > 0 ? g->boxes + 7 * nb : (const double *)nullptr);
  const double background = g ? g->background : 1.0;
  std::vector<double> uniform(nb + 1);
  uniform[0] = pxa::average_uniform(background);
  for (int64_t b = 0; b < nb; b++) uniform[b + 1] = pxa::average_uniform(boxes[7 * b + 6]);
  cudaStream_t st = nullptr;
  double *d_boxes = nullptr, *d_uniform = nullptr, *d_out = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  // each step runs only while every one before it succeeded (the first error is kept); the
  // buffers made are freed whatever happened
  auto step = [&](auto &&call) {
    if (e == cudaSuccess) e = call();
  };
  step([&] { return cudaMallocAsync(&d_boxes, (size_t)std::max<int64_t>(nb, 1) * 7 * 8, st); });
  step([&] { return cudaMallocAsync(&d_uniform, (size_t)(nb + 1) * 8, st); });
  step([&] { return cudaMallocAsync(&d_out, (size_t)total * 8, st); });
  if (nb > 0)
    step([&] {
      return cudaMemcpyAsync(d_boxes, boxes.data(), (size_t)nb * 7 * 8, cudaMemcpyHostToDevice, st);
    });
  step([&] {
    return cudaMemcpyAsync(d_uniform, uniform.data(), (size_t)(nb + 1) * 8, cudaMemcpyHostToDevice,
                           st);
  });
  step([&] {
    AverageArgs A;
    for (int a = 0; a < 3; a++) A.n[a] = n[a], A.d[a] = d[a], A.o[a] = o[a];
    A.geo = pxa::BoxView{background, nb, d_boxes};
    A.uniform = d_uniform;
    A.out = d_out;
    A.total = total;
    average_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(A);
    return cudaGetLastError();
  });
  step([&] { return cudaMemcpyAsync(out, d_out, (size_t)total * 8, cudaMemcpyDeviceToHost, st); });
  if (st) {
    if (d_boxes) cudaFreeAsync(d_boxes, st);
    if (d_uniform) cudaFreeAsync(d_uniform, st);
    if (d_out) cudaFreeAsync(d_out, st);
    const cudaError_t done = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = done;
    cudaStreamDestroy(st);
  }
  if (e != cudaSuccess) cudaGetLastError();  // leave no sticky launch error behind
  return e == cudaSuccess ? 0 : -2;
}
