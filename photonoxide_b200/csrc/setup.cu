// Set-up on the device: FDFD's cell average of a box geometry at every E value (the same
// functions as the host library's pxs_average, average.cuh, so the same bits), one thread per
// value. Cells whose samples all see one value take that value's average from a table made on
// the host; the others take the 8^3-sample average.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <vector>

#include "average.cuh"
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

}  // namespace

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
