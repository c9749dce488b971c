// The library's internal view of one simulation context, for the batch (batch.cu), which steps
// several contexts' grids together in place: their device buffers, tables and sources as set.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"
#include "photonoxide_fdtd.h"

struct InstanceView {
  int precision;
  int n[3];
  long long N;
  int periodic[3], low[3], high[3];
  double dt, step[3];
  double inv_step[3];  // 1/step as the kernels round it
  int fast_div[3];     // div_by_step's product form checked for the step
  int parity;  // which copy of E, H and H's psi is current
  void *e[2], *h[2], *psi_h[2], *psi_e;
  long long psi_h_len, psi_e_len;  // values in each copy of H's psi and in E's
  const void *ca;  // null: lossless
  const void *cb, *fe, *fh, *coefs;
  pxf::SlabEntry table[2][3][3][2];
  const std::vector<fdtd_waveform> *waves;
  const std::vector<fdtd_injection> *inj;
  long long nvalues;
  const long long *where;
  const pxf::SeriesDev *series;
  const long long *value_series;
  int nslots;
  const double *omega;
  const int *slot_field;
  double *sums;
  long long nsums;  // complex sums
  int nprobes;
  const long long *probes;
  bool media;
  bool plane_waves;  // total-field/scattered-field boxes (stepped by the engine alone)
  cudaStream_t stream;
  unsigned long long generation;  // moves on with every change the engine's calls make
};

int fdtd_instance_view(fdtd_ctx *c, InstanceView *v);
// The probe record's rows for `steps` more steps (grown as needed); null without probes.
int fdtd_instance_reserve(fdtd_ctx *c, long long steps, double **rows);
// After `steps` steps taken by the batch: the current copies and the record's length.
void fdtd_instance_advance(fdtd_ctx *c, long long steps);
int fdtd_instance_fail(fdtd_ctx *c, int code, const char *what);
