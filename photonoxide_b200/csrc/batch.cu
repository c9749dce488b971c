// Batched 2D TE stepping: many simulations' grids (one cell thick, periodic along z, as
// Boundaries::cpml_2d in src/fdtd.rs:242-247) advanced together, one launch per step for all of
// them. Each simulation is a context of the single-grid engine (engine.cu), already set up by
// its own calls; the batch steps its buffers in place and leaves the context as if it had run
// the steps itself.
//
// TE fields only: E_x, E_y and H_z. On such a grid the other three components (H_x, H_y, E_z)
// start at zero and stay zero under the reference's update (src/fdtd/kernel/reference.rs:14-99),
// and each TE value is computed with the same operations in the same order as the single-grid
// kernel (curl, the CPML slabs along x then y, then the sources), so a simulation stepped in a
// batch has the bits it has stepped alone.
//
// One step is ONE persistent launch: CTAs (a few per SM) take tiles of TW x TH cells from the
// list of all the grids' tiles. A tile computes H_z over itself and the row and column below it
// (its neighbours compute the same values), adds the magnetic sources there, then updates E_x and
// E_y on its cells, adds the electric sources, and writes both to the other copy of the fields.
// Steps run in chunks of G: the source waveforms and transform phases of a chunk are evaluated
// first (f64, the reference's exp and sincos), the chunk's step launches follow, each with a
// launch that copies the monitored values into a ring; at the chunk's end one launch adds the
// ring into the f64 transform sums in time order. A chunk is captured
// once as a CUDA graph and replayed. The tile shape is chosen by timing: the first run tries each
// shape on a chunk of real steps (every shape gives the same bits) and keeps the fastest.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "instance.h"
#include "photonoxide_adjoint.h"
#include "photonoxide_batch.h"

namespace pxb {
using namespace pxf;

constexpr int THREADS = 256;
constexpr int G = 32;  // steps per chunk (even: a chunk leaves the copies' parity as it was)

template <typename T>
struct TeInst {
  int nx, ny, px, py;  // sizes, periodic flags
  long long N;
  T dt, sx, sy;        // the step's dt and the grid steps along x and y, as the kernel rounds them
  T inv_sx, inv_sy;    // 1/step rounded, and whether div_by_step's product form is checked
  double rd_x, rd_y;   // 1/step in double
  int fast_x, fast_y;
  double dt64;
  T *e[2], *h[2], *psi_h[2];
  T *psi_e;
  const T *ca, *cb, *fe, *fh, *coefs;
  // the CPML slabs a TE grid has: H_z along x and y, E_y along x, E_x along y (per side)
  SlabEntry hx[2], hy[2], ex[2], ey[2];
  int parity;         // the current copy (device: kept up to date across chunks)
  long long first;    // the step index the next step has
  double *rows;       // the probe record's next row
  int tiles_x, tile0; // tiles along x; the first tile's number in the batch
  int bucket0;        // the first of its tiles' buckets
  int wave0, nwaves;  // its emitters in the batch's wave table
  int slot0, nslots;  // its transform phase slots
  const long long *where;
  const SeriesDev *series;
  const long long *value_series;
  const double *omega;
  const int *slot_field;
  double *sums;
  const long long *probes;
  int nprobes;
};

// One record item: instance, then a transform value (kind 0) or a probe (kind 1) by index.
struct RecItem {
  int inst, kind;
  long long index;
  long long col;  // a transform value's column in the ring
};

__device__ __forceinline__ bool in_slab(const SlabEntry &s, int m) {
  return s.count > 0 && m >= s.from && m < s.from + s.count;
}

// psi <- b psi + a (d/h), then H -= dt (sign psi) or E += cb (sign psi) (slab4 in engine.cu)
template <typename T>
__device__ __forceinline__ T slab_h(const TeInst<T> &I, const SlabEntry &s, int m, long long at,
                                    const T *pin, T *pout, bool own, T diff, int axis, T sign,
                                    T v) {
  const T b = I.coefs[s.coef + (m - s.from)], a = I.coefs[s.coef + s.count + (m - s.from)];
  T d = axis == 0 ? div_by_step(diff, I.sx, I.inv_sx, I.rd_x, I.fast_x)
                  : div_by_step(diff, I.sy, I.inv_sy, I.rd_y, I.fast_y);
  T nw = b * pin[at] + a * d;
  if (own) pout[at] = nw;
  T u = sign * nw;
  return v - I.dt * u;
}
template <typename T>
__device__ __forceinline__ T slab_e(const TeInst<T> &I, const SlabEntry &s, int m, long long at,
                                    T *psi, T diff, int axis, T sign, T cbv, T v) {
  const T b = I.coefs[s.coef + (m - s.from)], a = I.coefs[s.coef + s.count + (m - s.from)];
  T d = axis == 0 ? div_by_step(diff, I.sx, I.inv_sx, I.rd_x, I.fast_x)
                  : div_by_step(diff, I.sy, I.inv_sy, I.rd_y, I.fast_y);
  T nw = b * psi[at] + a * d;
  psi[at] = nw;
  T u = sign * nw;
  return v + cbv * u;
}

template <typename T, int TW, int TH>
__global__ void __launch_bounds__(THREADS) te_step_kernel(
    const TeInst<T> *__restrict__ insts, const int *__restrict__ tile_inst, int ntiles,
    const int *__restrict__ hbucket, const int *__restrict__ ebucket,
    const Group *__restrict__ hgroups, const Group *__restrict__ egroups,
    const Entry *__restrict__ entries, const double *__restrict__ waves_h,
    const double *__restrict__ waves_e, int m) {
  constexpr int HW = TW + 1, HH = TH + 1;
  __shared__ T sh[HW * HH];  // the new H_z over the tile and the row and column below it
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int ii = tile_inst[t];
    const TeInst<T> &I = insts[ii];
    const int lt = t - I.tile0;
    const int x0 = (lt % I.tiles_x) * TW, y0 = (lt / I.tiles_x) * TH;
    const int nx = I.nx, ny = I.ny;
    const long long N = I.N;
    const int cur = (I.parity + m) & 1;
    const T *ein = I.e[cur];
    T *eout = I.e[1 - cur];
    const T *hin = I.h[cur];
    T *hout = I.h[1 - cur];
    const T *pin = I.psi_h[cur];
    T *pout = I.psi_h[1 - cur];
    // -- H_z (src/fdtd/kernel/reference.rs:14-56 with E_z, H_x, H_y zero)
    for (int q = threadIdx.x; q < HW * HH; q += THREADS) {
      const int lx = q % HW, ly = q / HW;
      const int x = x0 - 1 + lx, y = y0 - 1 + ly;
      const int mx = wrap_index(x, nx, I.px), my = wrap_index(y, ny, I.py);
      T hz = T(0);  // beyond a wall H is zero
      if (mx >= 0 && my >= 0 && x < nx && y < ny) {
        const int mxp = wrap_index(mx + 1, nx, I.px), myp = wrap_index(my + 1, ny, I.py);
        const long long r = (long long)my * nx + mx;
        const T ex = ein[r], ey = ein[N + r];
        const T eyn = mxp >= 0 ? ein[N + (long long)my * nx + mxp] : T(0);
        const T exn = myp >= 0 ? ein[(long long)myp * nx + mx] : T(0);
        const T dxEy = eyn - ey, dyEx = exn - ex;
        hz = hin[2 * N + r] - I.dt * (dxEy * I.fh[mx] - dyEx * I.fh[nx + my]);
        const bool own = lx >= 1 && ly >= 1;
        // the CPML: H_z along x (+), then along y (-)
        if (!I.px) {
          const int side = mx < nx / 2 ? 0 : 1;
          const SlabEntry &s = I.hx[side];
          if (in_slab(s, mx))
            hz = slab_h(I, s, mx, s.psi + (long long)my * s.pw + (mx - s.pf), pin, pout, own, dxEy,
                        0, T(1), hz);
        }
        if (!I.py) {
          const int side = my < ny / 2 ? 0 : 1;
          const SlabEntry &s = I.hy[side];
          if (in_slab(s, my))
            hz = slab_h(I, s, my, s.psi + (long long)(my - s.from) * nx + mx, pin, pout, own, dyEx,
                        1, T(-1), hz);
        }
      }
      sh[q] = hz;
    }
    const int b = I.bucket0 + lt;
    const int hg0 = hbucket[b], hg1 = hbucket[b + 1];
    if (hg1 > hg0) {
      __syncthreads();
      // the magnetic sources (src/fdtd.rs:1348-1359), each value's entries in CPU order
      for (int g = hg0 + threadIdx.x; g < hg1; g += THREADS) {
        const Group gr = hgroups[g];
        T v = sh[gr.local];
        for (int q = gr.first; q < gr.first + gr.count; q++) {
          const Entry en = entries[q];
          const double *w = waves_h + 2 * (long long)en.emitter;
          const double amount = en.are * w[0] - en.aim * w[1];
          if (sizeof(T) == 8) v = v - (T)(I.dt64 * amount);
          else v = v - I.dt * (T)amount;
        }
        sh[gr.local] = v;
      }
    }
    __syncthreads();
    // -- E_x, E_y on the tile (reference.rs:58-99): back differences of the new H_z
    for (int q = threadIdx.x; q < TW * TH; q += THREADS) {
      const int lx = q % TW + 1, ly = q / TW + 1;
      const int x = x0 + lx - 1, y = y0 + ly - 1;
      if (x < nx && y < ny) {
        const long long r = (long long)y * nx + x;
        const T hz = sh[ly * HW + lx];
        hout[2 * N + r] = hz;
        const T dyHz = hz - sh[(ly - 1) * HW + lx], dxHz = hz - sh[ly * HW + lx - 1];
        const T fex = I.fe[x], fey = I.fe[nx + y];
        // curl_x = dyHz fey - dzHy fez and curl_y = dzHx fez - dxHz fex, with dzHy = dzHx = +0
        const T curl0 = dyHz * fey;
        const T curl1 = T(0) - dxHz * fex;
        const T cbx = I.cb[r], cby = I.cb[N + r];
        T cax, cay;
        if (I.ca) {
          cax = I.ca[r];
          cay = I.ca[N + r];
        } else {
          cax = cbx == T(0) ? T(0) : T(1);
          cay = cby == T(0) ? T(0) : T(1);
        }
        T nex = cax * ein[r] + cbx * curl0;
        T ney = cay * ein[N + r] + cby * curl1;
        // the CPML: E_x along y (+), E_y along x (-)
        if (!I.py) {
          const int side = y < ny / 2 ? 0 : 1;
          const SlabEntry &s = I.ey[side];
          if (in_slab(s, y))
            nex = slab_e(I, s, y, s.psi + (long long)(y - s.from) * nx + x, I.psi_e, dyHz, 1,
                         T(1), cbx, nex);
        }
        if (!I.px) {
          const int side = x < nx / 2 ? 0 : 1;
          const SlabEntry &s = I.ex[side];
          if (in_slab(s, x))
            ney = slab_e(I, s, x, s.psi + (long long)y * s.pw + (x - s.pf), I.psi_e, dxHz, 0,
                         T(-1), cby, ney);
        }
        eout[r] = nex;
        eout[N + r] = ney;
      }
    }
    const int eg0 = ebucket[b], eg1 = ebucket[b + 1];
    if (eg1 > eg0) {
      __syncthreads();  // this CTA's E values are in memory
      // the electric currents (src/fdtd.rs:1375-1387): local = the place in the tile, x fastest
      for (int g = eg0 + threadIdx.x; g < eg1; g += THREADS) {
        const Group gr = egroups[g];
        const int lq = gr.local;
        const int x = x0 + lq % TW, y = y0 + lq / TW;
        const long long at = (long long)gr.comp * N + (long long)y * nx + x;
        T v = eout[at];
        const T cbv = I.cb[at];
        for (int q = gr.first; q < gr.first + gr.count; q++) {
          const Entry en = entries[q];
          const double *w = waves_e + 2 * (long long)en.emitter;
          const double amount = en.are * w[0] - en.aim * w[1];
          if (sizeof(T) == 8) v = v - (T)((double)cbv * amount);
          else v = v - cbv * (T)amount;
        }
        eout[at] = v;
      }
    }
    __syncthreads();  // sh is reused by the next tile
  }
}

// The same step with a warp per tile row and four places per lane: a tile owns 124 x 7 places;
// warp w holds row y0-1+w (warp 0 the row below the tile, for E's back differences), lane l the
// places x0-4+4l .. x0-1+4l (lane 0 the column before the tile), read and written 16 bytes at a
// time where a grid's rows are (nx a multiple of 4), one value at a time otherwise. H_z goes
// through shared memory, where the magnetic sources are added and E reads its neighbours. Each
// value's arithmetic is te_step_kernel's; the lane's index arithmetic serves four values. Four
// CTAs per SM (64 registers, a few spilled): with three, at 78 registers, it ran 50 Gcell/s
// on 64 grids of widths a multiple of 4, with four 61 (the 32 x 16 tiles: 55).
namespace teq {
constexpr int VEC = 4, ROW = 128, OWN = 124, RW = 7, WARPS = RW + 1;
static_assert(WARPS * 32 == THREADS, "a warp per row");
}  // namespace teq

template <typename T>
struct V4 {
  T v[4];
};
template <typename T>
__device__ __forceinline__ V4<T> ldv(const T *p) {
  V4<T> r;
  if (sizeof(T) == 4) {
    const float4 f = *reinterpret_cast<const float4 *>(p);
    r.v[0] = (T)f.x, r.v[1] = (T)f.y, r.v[2] = (T)f.z, r.v[3] = (T)f.w;
  } else {
    const double2 a = *reinterpret_cast<const double2 *>(p), b = *reinterpret_cast<const double2 *>(p + 2);
    r.v[0] = (T)a.x, r.v[1] = (T)a.y, r.v[2] = (T)b.x, r.v[3] = (T)b.y;
  }
  return r;
}
template <typename T>
__device__ __forceinline__ void stv(T *p, const T v[4]) {
  if (sizeof(T) == 4) {
    *reinterpret_cast<float4 *>(p) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
  } else {
    *reinterpret_cast<double2 *>(p) = make_double2((double)v[0], (double)v[1]);
    *reinterpret_cast<double2 *>(p + 2) = make_double2((double)v[2], (double)v[3]);
  }
}

template <typename T>
__global__ void __launch_bounds__(THREADS, 4) te_quad_kernel(
    const TeInst<T> *__restrict__ insts, const int *__restrict__ tile_inst, int ntiles,
    const int *__restrict__ hbucket, const int *__restrict__ ebucket,
    const Group *__restrict__ hgroups, const Group *__restrict__ egroups,
    const Entry *__restrict__ entries, const double *__restrict__ waves_h,
    const double *__restrict__ waves_e, int m) {
  using namespace teq;
  __shared__ __align__(16) T sh[WARPS * ROW];  // the new H_z of the rows y0-1 .. y0+RW-1
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int ii = tile_inst[t];
    const TeInst<T> &I = insts[ii];
    const int lt = t - I.tile0;
    const int x0 = (lt % I.tiles_x) * OWN, y0 = (lt / I.tiles_x) * RW;
    const int nx = I.nx, ny = I.ny;
    const long long N = I.N;
    const int cur = (I.parity + m) & 1;
    const T *ein = I.e[cur];
    T *eout = I.e[1 - cur];
    const T *hin = I.h[cur];
    T *hout = I.h[1 - cur];
    const T *pin = I.psi_h[cur];
    T *pout = I.psi_h[1 - cur];
    const bool vec = (nx & 3) == 0;  // then a lane's four places are all in the grid or none
    const int xb = x0 - VEC + VEC * lane;
    const int y = y0 - 1 + w;
    const int my = y < ny ? wrap_index(y, ny, I.py) : -1;  // beyond the grid's end: H is zero
    int mx[4];
    bool ok[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int x = xb + j;
      mx[j] = x < 0 ? (I.px ? x + nx : -1) : (x < nx ? x : -1);
      ok[j] = mx[j] >= 0 && my >= 0;
    }
    const bool live = ok[0] | ok[1] | ok[2] | ok[3];
    const bool own = w >= 1 && lane >= 1;
    // the four places' values of a row (zero where a place is not in the grid)
    auto get = [&](const T *row) {
      V4<T> o;
      if (vec && ok[0]) {
        o = ldv(row + mx[0]);
      } else {
#pragma unroll
        for (int j = 0; j < 4; j++) o.v[j] = ok[j] ? row[mx[j]] : T(0);
      }
      return o;
    };
    const long long rrow = (long long)(my < 0 ? 0 : my) * nx;
    // -- H_z (src/fdtd/kernel/reference.rs:14-56 with E_z, H_x, H_y zero)
    const V4<T> ex = get(ein + rrow), ey = get(ein + N + rrow);
    const T eynext = __shfl_down_sync(0xffffffffu, ey.v[0], 1);
    T hz[4] = {T(0), T(0), T(0), T(0)};
    T dxEy[4], dyEx[4];
    if (live) {
      const int myp = wrap_index(my + 1, ny, I.py);
      V4<T> exn;
      if (myp >= 0) {
        exn = get(ein + (long long)myp * nx);
      } else {
#pragma unroll
        for (int j = 0; j < 4; j++) exn.v[j] = T(0);
      }
      const V4<T> ho = get(hin + 2 * N + rrow), fhx = get(I.fh);
      const T fhy = I.fh[nx + my];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        // E_y at mx + 1: the next place's (the next lane's first for the fourth, read by the
        // row's last lane), x = 0's on a periodic x past the end, else zero
        T eyj;
        if (mx[j] + 1 >= nx) eyj = I.px ? ein[N + rrow] : T(0);
        else if (j < 3) eyj = ey.v[j + 1];
        else eyj = lane < 31 ? eynext : ein[N + rrow + mx[j] + 1];
        dxEy[j] = eyj - ey.v[j];
        dyEx[j] = exn.v[j] - ex.v[j];
        hz[j] = ho.v[j] - I.dt * (dxEy[j] * fhx.v[j] - dyEx[j] * fhy);
      }
      // the CPML: H_z along x (+), then along y (-)
      if (!I.px) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
          if (!ok[j]) continue;
          const SlabEntry &s = I.hx[mx[j] < nx / 2 ? 0 : 1];
          if (in_slab(s, mx[j]))
            hz[j] = slab_h(I, s, mx[j], s.psi + (long long)my * s.pw + (mx[j] - s.pf), pin, pout,
                           own, dxEy[j], 0, T(1), hz[j]);
        }
      }
      if (!I.py) {
        const SlabEntry &s = I.hy[my < ny / 2 ? 0 : 1];
        if (in_slab(s, my))
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (ok[j])
              hz[j] = slab_h(I, s, my, s.psi + (long long)(my - s.from) * nx + mx[j], pin, pout,
                             own, dyEx[j], 1, T(-1), hz[j]);
      }
#pragma unroll
      for (int j = 0; j < 4; j++)
        if (!ok[j]) hz[j] = T(0);
    }
    stv(sh + w * ROW + VEC * lane, hz);
    const int b = I.bucket0 + lt;
    const int hg0 = hbucket[b], hg1 = hbucket[b + 1];
    if (hg1 > hg0) {
      __syncthreads();
      // the magnetic sources (src/fdtd.rs:1348-1359), each value's entries in CPU order
      for (int g = hg0 + threadIdx.x; g < hg1; g += THREADS) {
        const Group gr = hgroups[g];
        T v = sh[gr.local];
        for (int q = gr.first; q < gr.first + gr.count; q++) {
          const Entry en = entries[q];
          const double *wv = waves_h + 2 * (long long)en.emitter;
          const double amount = en.are * wv[0] - en.aim * wv[1];
          if (sizeof(T) == 8) v = v - (T)(I.dt64 * amount);
          else v = v - I.dt * (T)amount;
        }
        sh[gr.local] = v;
      }
    }
    __syncthreads();
    // -- E_x, E_y at the owned places (reference.rs:58-99): back differences of the new H_z
    if (own && live) {
      const V4<T> h = ldv(sh + w * ROW + VEC * lane), hu = ldv(sh + (w - 1) * ROW + VEC * lane);
      const T hl = sh[w * ROW + VEC * lane - 1];
      const V4<T> fex = get(I.fe), cbx = get(I.cb + rrow), cby = get(I.cb + N + rrow);
      const T fey = I.fe[nx + my];
      V4<T> cax, cay;
      if (I.ca) {
        cax = get(I.ca + rrow);
        cay = get(I.ca + N + rrow);
      } else {
#pragma unroll
        for (int j = 0; j < 4; j++) {
          cax.v[j] = cbx.v[j] == T(0) ? T(0) : T(1);
          cay.v[j] = cby.v[j] == T(0) ? T(0) : T(1);
        }
      }
      T nex[4], ney[4], dyHz[4], dxHz[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        dyHz[j] = h.v[j] - hu.v[j];
        dxHz[j] = h.v[j] - (j > 0 ? h.v[j - 1] : hl);
        // curl_x = dyHz fey - dzHy fez and curl_y = dzHx fez - dxHz fex, with dzHy = dzHx = +0
        const T curl0 = dyHz[j] * fey;
        const T curl1 = T(0) - dxHz[j] * fex.v[j];
        nex[j] = cax.v[j] * ex.v[j] + cbx.v[j] * curl0;
        ney[j] = cay.v[j] * ey.v[j] + cby.v[j] * curl1;
      }
      // the CPML: E_x along y (+), E_y along x (-)
      if (!I.py) {
        const SlabEntry &s = I.ey[my < ny / 2 ? 0 : 1];
        if (in_slab(s, my))
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (ok[j])
              nex[j] = slab_e(I, s, my, s.psi + (long long)(my - s.from) * nx + mx[j], I.psi_e,
                              dyHz[j], 1, T(1), cbx.v[j], nex[j]);
      }
      if (!I.px) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
          if (!ok[j]) continue;
          const SlabEntry &s = I.ex[mx[j] < nx / 2 ? 0 : 1];
          if (in_slab(s, mx[j]))
            ney[j] = slab_e(I, s, mx[j], s.psi + (long long)my * s.pw + (mx[j] - s.pf), I.psi_e,
                            dxHz[j], 0, T(-1), cby.v[j], ney[j]);
        }
      }
      if (vec) {
        stv(hout + 2 * N + rrow + mx[0], h.v);
        stv(eout + rrow + mx[0], nex);
        stv(eout + N + rrow + mx[0], ney);
      } else {
#pragma unroll
        for (int j = 0; j < 4; j++)
          if (ok[j]) {
            hout[2 * N + rrow + mx[j]] = h.v[j];
            eout[rrow + mx[j]] = nex[j];
            eout[N + rrow + mx[j]] = ney[j];
          }
      }
    }
    const int eg0 = ebucket[b], eg1 = ebucket[b + 1];
    if (eg1 > eg0) {
      __syncthreads();  // this CTA's E values are in memory
      // the electric currents (src/fdtd.rs:1375-1387): local = the place in the tile, x fastest
      for (int g = eg0 + threadIdx.x; g < eg1; g += THREADS) {
        const Group gr = egroups[g];
        const int lq = gr.local;
        const int x = x0 + lq % OWN, yy = y0 + lq / OWN;
        const long long at = (long long)gr.comp * N + (long long)yy * nx + x;
        T v = eout[at];
        const T cbv = I.cb[at];
        for (int q = gr.first; q < gr.first + gr.count; q++) {
          const Entry en = entries[q];
          const double *wv = waves_e + 2 * (long long)en.emitter;
          const double amount = en.are * wv[0] - en.aim * wv[1];
          if (sizeof(T) == 8) v = v - (T)((double)cbv * amount);
          else v = v - cbv * (T)amount;
        }
        eout[at] = v;
      }
    }
    __syncthreads();  // sh is reused by the next tile
  }
}

// The chunk's waveforms: per (instance, emitter, step m) at H's time (first+m) dt and E's
// (first+m+1/2) dt (waves_kernel in engine.cu). Emitter numbers in `entries` are batch-wide:
// wave0 + the instance's own; the tables are [m][emitter].
template <typename T>
__global__ void te_waves_kernel(const TeInst<T> *insts, const int2 *items, int nitems,
                                const Wave *waves, const int *point, int nwaves_total,
                                double *out_h, double *out_e) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nitems * G) return;
  const int m = q / nitems, it = q % nitems;
  const int2 item = items[it];  // (instance, batch-wide emitter)
  const TeInst<T> &I = insts[item.x];
  const double t = (double)(I.first + m) * I.dt64;
  double re, im;
  wave_eval(waves[item.y], t, &re, &im, point[item.y]);
  long long o = 2 * ((long long)m * nwaves_total + item.y);
  out_h[o] = re;
  out_h[o + 1] = im;
  wave_eval(waves[item.y], t + 0.5 * I.dt64, &re, &im, point[item.y]);
  out_e[o] = re;
  out_e[o + 1] = im;
}

// The chunk's transform phases e^{i w t} dt: E at te = (first+m+1) dt, H at te - dt/2
// (phase_kernel in engine.cu); [m][batch-wide slot].
template <typename T>
__global__ void te_phase_kernel(const TeInst<T> *insts, const int2 *items, int nitems,
                                int nslots_total, double *phase) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nitems * G) return;
  const int m = q / nitems, it = q % nitems;
  const int2 item = items[it];  // (instance, its own slot)
  const TeInst<T> &I = insts[item.x];
  const double te = (double)(I.first + m + 1) * I.dt64;
  const double t = I.slot_field[item.y] ? te - 0.5 * I.dt64 : te;
  double sn, cs;
  pxp::sincos(I.omega[item.y] * t, &sn, &cs);
  long long o = 2 * ((long long)m * nslots_total + I.slot0 + item.y);
  phase[o] = cs * I.dt64;
  phase[o + 1] = sn * I.dt64;
}

// After step m of the chunk: each transform value into row m of the ring, each probe's value
// into its record row.
template <typename T>
__global__ void te_record_kernel(const TeInst<T> *insts, const RecItem *items, long long nitems,
                                 T *ring, long long nring, int m) {
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nitems) return;
  const RecItem it = items[q];
  const TeInst<T> &I = insts[it.inst];
  const int now = (I.parity + m + 1) & 1;  // the copy the step wrote
  if (it.kind == 1) {
    const long long w = I.probes[it.index];
    const T *f = (w >> 62) ? I.h[now] : I.e[now];
    I.rows[(long long)m * I.nprobes + it.index] = (double)f[w & ((1LL << 62) - 1)];
    return;
  }
  const long long w = I.where[it.index];
  const T *f = (w >> 62) ? I.h[now] : I.e[now];
  ring[(long long)m * nring + it.col] = f[w & ((1LL << 62) - 1)];
}

// After a chunk's `count` steps: each transform value's sums += sum over the ring's rows of
// F e^{i w t} dt, f64, in time order (dft_kernel in engine.cu).
template <typename T>
__global__ void te_contract_kernel(const TeInst<T> *insts, const RecItem *items, long long nitems,
                                   const T *ring, long long nring, const double *phase,
                                   int nslots_total, int count) {
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nitems) return;
  const RecItem it = items[q];
  if (it.kind != 0) return;
  const TeInst<T> &I = insts[it.inst];
  const long long v = it.index;
  const SeriesDev s = I.series[I.value_series[v]];
  const long long o = v - s.value0;
  for (int k = 0; k < s.nf; k++) {
    double *acc = I.sums + 2 * (s.sum0 + (long long)k * s.volume + o);
    double re = acc[0], im = acc[1];
    const double *ph = phase + 2 * ((long long)I.slot0 + s.slot0 + k);
    for (int m = 0; m < count; m++) {
      const double x = (double)ring[(long long)m * nring + it.col];
      re = re + x * ph[2 * (long long)m * nslots_total];
      im = im + x * ph[2 * (long long)m * nslots_total + 1];
    }
    acc[0] = re;
    acc[1] = im;
  }
}

// After `count` steps: each instance's step index, copy and record row move on.
template <typename T>
__global__ void te_advance_kernel(TeInst<T> *insts, int n, int count) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  TeInst<T> &I = insts[q];
  I.first += count;
  I.parity = (I.parity + count) & 1;
  if (I.rows) I.rows += (long long)count * I.nprobes;
}

// Nonzero values among H_x, H_y, E_z of the current copy (the batch steps TE grids only).
template <typename T>
__global__ void te_tm_check_kernel(const T *e, const T *h, long long N, int *bad) {
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= N) return;
  if (h[q] != T(0) || h[N + q] != T(0) || e[2 * N + q] != T(0)) atomicOr(bad, 1);
}

// After step m of a chunk: the curl E's update multiplies by cb, at each design value (its
// component 0 or 1 and index: component * N + r), from the new H_z: the derivative of the new E
// by cb where no CPML, source or medium is (those the adjoint's caller keeps off the design).
template <typename T>
__global__ void te_design_kernel(const TeInst<T> *insts, const long long *design, long long n,
                                 T *K, long long k_first, int m) {
  long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= n) return;
  const TeInst<T> &I = insts[0];
  const T *hz = I.h[(I.parity + m + 1) & 1] + 2 * I.N;
  const long long place = design[d];
  const int comp = (int)(place / I.N);
  const long long r = place % I.N;
  const int x = (int)(r % I.nx), y = (int)(r / I.nx);
  T curl;
  if (comp == 0) {
    const int ym = wrap_index(y - 1, I.ny, I.py);
    const T below = ym >= 0 ? hz[(long long)ym * I.nx + x] : T(0);
    curl = (hz[r] - below) * I.fe[I.nx + y];
  } else {
    const int xm = wrap_index(x - 1, I.nx, I.px);
    const T left = xm >= 0 ? hz[(long long)y * I.nx + xm] : T(0);
    curl = T(0) - (hz[r] - left) * I.fe[x];
  }
  K[(I.first + m - k_first) * n + d] = curl;
}

// ------------------------------------------------------------------------------------------
// The time-reversed adjoint of the TE step. The step is linear in (E, H_z, psi), so the
// gradient of J(transform sums) reverses it: with the adjoint state (E~, H~, psi~) of the
// values after step n, the adjoint of the values before it is the step's transpose applied to
// them. Its stencil is the step's with the roles of the fields swapped: H~ at a cell gathers
// from E~ at the cell and at the cells above along x and y (where the step's E read this H_z),
// then E~ gathers from H~ at the cell and the cells below (where the step's H_z read this E) --
// so a tile computes H~ over itself and the row and column below it, then E~ on its cells,
// exactly as the forward step does. All adjoint copies are ping-ponged.
template <typename T>
struct AdjState {
  T *e[2];    // E~_x, E~_y: 2N
  T *h[2];    // H~_z: N
  T *pe[2];   // psi~ of E's slabs, laid out as psi_e
  T *ph[2];   // psi~ of H's slabs, laid out as psi_h
  int cur;
};

template <typename T>
__device__ __forceinline__ T coef_b(const TeInst<T> &I, const SlabEntry &s, int m) {
  return I.coefs[s.coef + (m - s.from)];
}
template <typename T>
__device__ __forceinline__ T coef_a(const TeInst<T> &I, const SlabEntry &s, int m) {
  return I.coefs[s.coef + s.count + (m - s.from)];
}

template <typename T, int TW, int TH>
__global__ void __launch_bounds__(THREADS) te_adjoint_kernel(const TeInst<T> *insts,
                                                             AdjState<T> A, int ntiles) {
  constexpr int HW = TW + 1, HH = TH + 1;
  __shared__ T sh[HW * HH];  // H~ of the step's H_z over the tile and the row and column below
  const TeInst<T> &I = insts[0];
  const int nx = I.nx, ny = I.ny;
  const long long N = I.N;
  const T *eb = A.e[A.cur];
  T *eo = A.e[1 - A.cur];
  const T *hb = A.h[A.cur];
  T *ho = A.h[1 - A.cur];
  const T *pei = A.pe[A.cur];
  T *peo = A.pe[1 - A.cur];
  const T *phi = A.ph[A.cur];
  T *pho = A.ph[1 - A.cur];
  // psi~ of an E slab value in total: what the later steps carried, plus this step's use of it
  // (E_x += cb (+psi') along y; E_y += cb (-psi') along x)
  auto psi_ex_total = [&](int x, int y, long long r, const SlabEntry &s) -> T {
    return pei[s.psi + (long long)(y - s.from) * nx + x] + I.cb[r] * eb[r];
  };
  auto psi_ey_total = [&](int x, int y, long long r, const SlabEntry &s) -> T {
    return pei[s.psi + (long long)y * s.pw + (x - s.pf)] - I.cb[N + r] * eb[N + r];
  };
  // psi~ of an H slab value in total (H_z -= dt (+psi') along x, H_z -= dt (-psi') along y)
  auto psi_hx_total = [&](int x, int y, T hbar, const SlabEntry &s) -> T {
    return phi[s.psi + (long long)y * s.pw + (x - s.pf)] - I.dt * hbar;
  };
  auto psi_hy_total = [&](int x, int y, T hbar, const SlabEntry &s) -> T {
    return phi[s.psi + (long long)(y - s.from) * nx + x] + I.dt * hbar;
  };
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int x0 = (t % I.tiles_x) * TW, y0 = (t / I.tiles_x) * TH;
    // -- H~ of the step's new H_z (total)
    for (int q = threadIdx.x; q < HW * HH; q += THREADS) {
      const int lx = q % HW, ly = q / HW;
      const int x = x0 - 1 + lx, y = y0 - 1 + ly;
      const int mx = wrap_index(x, nx, I.px), my = wrap_index(y, ny, I.py);
      T acc = T(0);
      if (mx >= 0 && my >= 0 && x < nx && y < ny) {
        const bool own = lx >= 1 && ly >= 1;
        const int mxp = wrap_index(mx + 1, nx, I.px), myp = wrap_index(my + 1, ny, I.py);
        const long long r = (long long)my * nx + mx;
        // E_x(x, y) read H_z(x, y) with cb fey(y), E_x(x, y+1) with -cb fey(y+1); E_y(x, y) with
        // -cb fex(x), E_y(x+1, y) with +cb fex(x+1)
        acc = hb[r] + I.cb[r] * I.fe[nx + my] * eb[r] - I.cb[N + r] * I.fe[mx] * eb[N + r];
        if (myp >= 0) {
          const long long rp = (long long)myp * nx + mx;
          acc = acc - I.cb[rp] * I.fe[nx + myp] * eb[rp];
        }
        if (mxp >= 0) {
          const long long rp = (long long)my * nx + mxp;
          acc = acc + I.cb[N + rp] * I.fe[mxp] * eb[N + rp];
        }
        // the E slabs: psi' = b psi + (a/h) (difference of H_z)
        if (!I.py) {
          const SlabEntry &s0 = I.ey[my < ny / 2 ? 0 : 1];
          if (in_slab(s0, my)) {
            const T tot = psi_ex_total(mx, my, r, s0);
            acc = acc + coef_a(I, s0, my) / I.sy * tot;
            if (own) peo[s0.psi + (long long)(my - s0.from) * nx + mx] = coef_b(I, s0, my) * tot;
          }
          if (myp >= 0) {
            const SlabEntry &s1 = I.ey[myp < ny / 2 ? 0 : 1];
            if (in_slab(s1, myp)) {
              const long long rp = (long long)myp * nx + mx;
              acc = acc - coef_a(I, s1, myp) / I.sy * psi_ex_total(mx, myp, rp, s1);
            }
          }
        }
        if (!I.px) {
          const SlabEntry &s0 = I.ex[mx < nx / 2 ? 0 : 1];
          if (in_slab(s0, mx)) {
            const T tot = psi_ey_total(mx, my, r, s0);
            acc = acc + coef_a(I, s0, mx) / I.sx * tot;
            if (own) peo[s0.psi + (long long)my * s0.pw + (mx - s0.pf)] = coef_b(I, s0, mx) * tot;
          }
          if (mxp >= 0) {
            const SlabEntry &s1 = I.ex[mxp < nx / 2 ? 0 : 1];
            if (in_slab(s1, mxp)) {
              const long long rp = (long long)my * nx + mxp;
              acc = acc - coef_a(I, s1, mxp) / I.sx * psi_ey_total(mxp, my, rp, s1);
            }
          }
        }
        if (own) ho[r] = acc;
      }
      sh[q] = acc;
    }
    __syncthreads();
    // -- E~ of the values before the step, on the tile
    for (int q = threadIdx.x; q < TW * TH; q += THREADS) {
      const int lx = q % TW + 1, ly = q / TW + 1;
      const int x = x0 + lx - 1, y = y0 + ly - 1;
      if (x >= nx || y >= ny) continue;
      const long long r = (long long)y * nx + x;
      const T hc = sh[ly * HW + lx], hy = sh[(ly - 1) * HW + lx], hx = sh[ly * HW + lx - 1];
      const int xm = wrap_index(x - 1, nx, I.px), ym = wrap_index(y - 1, ny, I.py);
      const T cbx = I.cb[r], cby = I.cb[N + r];
      T cax, cay;
      if (I.ca) {
        cax = I.ca[r];
        cay = I.ca[N + r];
      } else {
        cax = cbx == T(0) ? T(0) : T(1);
        cay = cby == T(0) ? T(0) : T(1);
      }
      // H_z(x, y) read E_x(x, y) with -dt fhy(y) and E_y(x, y) with +dt fhx(x); H_z(x, y-1)
      // read E_x(x, y) with +dt fhy(y-1); H_z(x-1, y) read E_y(x, y) with -dt fhx(x-1)
      T ax = cax * eb[r] - I.dt * I.fh[nx + y] * hc;
      T ay = cay * eb[N + r] + I.dt * I.fh[x] * hc;
      if (ym >= 0) ax = ax + I.dt * I.fh[nx + ym] * hy;
      if (xm >= 0) ay = ay - I.dt * I.fh[xm] * hx;
      if (!I.py) {
        const SlabEntry &s0 = I.hy[y < ny / 2 ? 0 : 1];
        if (in_slab(s0, y)) {
          const T tot = psi_hy_total(x, y, hc, s0);
          ax = ax - coef_a(I, s0, y) / I.sy * tot;
          pho[s0.psi + (long long)(y - s0.from) * nx + x] = coef_b(I, s0, y) * tot;
        }
        if (ym >= 0) {
          const SlabEntry &s1 = I.hy[ym < ny / 2 ? 0 : 1];
          if (in_slab(s1, ym)) ax = ax + coef_a(I, s1, ym) / I.sy * psi_hy_total(x, ym, hy, s1);
        }
      }
      if (!I.px) {
        const SlabEntry &s0 = I.hx[x < nx / 2 ? 0 : 1];
        if (in_slab(s0, x)) {
          const T tot = psi_hx_total(x, y, hc, s0);
          ay = ay - coef_a(I, s0, x) / I.sx * tot;
          pho[s0.psi + (long long)y * s0.pw + (x - s0.pf)] = coef_b(I, s0, x) * tot;
        }
        if (xm >= 0) {
          const SlabEntry &s1 = I.hx[xm < nx / 2 ? 0 : 1];
          if (in_slab(s1, xm)) ay = ay + coef_a(I, s1, xm) / I.sx * psi_hx_total(xm, y, hx, s1);
        }
      }
      eo[r] = ax;
      eo[N + r] = ay;
    }
    __syncthreads();
  }
}

// The transform phases of one segment's steps, [m][slot] (as te_phase_kernel).
template <typename T>
__global__ void te_segment_phase_kernel(const TeInst<T> *insts, long long first, int steps,
                                        double *phase) {
  const TeInst<T> &I = insts[0];
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= steps * I.nslots) return;
  const int m = q / I.nslots, s = q % I.nslots;
  const double te = (double)(first + m + 1) * I.dt64;
  const double t = I.slot_field[s] ? te - 0.5 * I.dt64 : te;
  double sn, cs;
  pxp::sincos(I.omega[s] * t, &sn, &cs);
  phase[2 * (long long)q] = cs * I.dt64;
  phase[2 * (long long)q + 1] = sn * I.dt64;
}

// Step m's direct part of J's derivative: the transforms took F dt e^{i w t} of each value, so
// dJ/dF = sum over frequencies of dJ/dRe(sum) Re(phase) + dJ/dIm(sum) Im(phase), added to E~
// or H~ of the value (TE components only: the others are zero whatever the permittivity).
// Without atomics, so that the gradient's bits never depend on scheduling: one thread per field
// value the transforms record, adding each of its transform values' dJ/dF in value order.
// `owner` lists, per such field value, its place (with the H flag in bit 62, as `where`) and
// its transform values order[start[g] .. start[g+1]).
template <typename T>
__global__ void te_inject_kernel(const TeInst<T> *insts, const long long *owner, const int *start,
                                 const long long *order, int nowners, const double *phase,
                                 const double *grad_sums, AdjState<T> A, int m) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nowners) return;
  const TeInst<T> &I = insts[0];
  const long long w = owner[g];
  const bool hfield = (w >> 62) != 0;
  const long long place = w & ((1LL << 62) - 1);
  T *f = hfield ? A.h[A.cur] + (place - 2 * I.N) : A.e[A.cur] + place;
  T acc = *f;
  for (int q = start[g]; q < start[g + 1]; q++) {
    const long long v = order[q];
    const SeriesDev s = I.series[I.value_series[v]];
    const long long o = v - s.value0;
    const double *ph = phase + 2 * ((long long)m * I.nslots + s.slot0);
    double x = 0.0;
    for (int k = 0; k < s.nf; k++) {
      const double *gs = grad_sums + 2 * (s.sum0 + (long long)k * s.volume + o);
      x += gs[0] * ph[2 * k] + gs[1] * ph[2 * k + 1];
    }
    acc = acc + (T)x;
  }
  *f = acc;
}

// dJ/dcb at each design value += E~ (of the values after the step) x the step's curl there.
template <typename T>
__global__ void te_grad_kernel(const long long *design, long long n, const T *K, AdjState<T> A,
                               double *grad) {
  long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= n) return;
  grad[d] += (double)A.e[A.cur][design[d]] * (double)K[d];
}

struct Shape {
  int tw, th;
};
// the last: te_quad_kernel's rows
const Shape SHAPES[] = {{32, 8}, {32, 16}, {64, 4}, {64, 8}, {128, 2}, {128, 4},
                        {teq::OWN, teq::RW}};
constexpr int QUAD_SHAPE = 6;
constexpr int NSHAPES = sizeof(SHAPES) / sizeof(SHAPES[0]);
constexpr int DEFAULT_SHAPE = 3;  // 64 x 8

}  // namespace pxb

using namespace pxb;

struct fdtd_batch {
  std::string error;
  std::vector<fdtd_ctx *> ctxs;
  int precision = 32;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr, t0 = nullptr, t1 = nullptr;
  int shape = -1;  // index into SHAPES; -1: choose by timing on the next run
  long long launches = 0;
  int sms = 148;
  std::vector<void *> allocs;  // this run's tables
  cudaGraphExec_t graph = nullptr;
  // the current tables (rebuilt at each run)
  void *d_insts = nullptr;
  int ntiles = 0;
  int *d_tile_inst = nullptr;
  int *d_hbucket = nullptr, *d_ebucket = nullptr;
  Group *d_hgroups = nullptr, *d_egroups = nullptr;
  Entry *d_entries = nullptr;
  Wave *d_waves = nullptr;
  int *d_point = nullptr;
  int2 *d_wave_items = nullptr, *d_slot_items = nullptr;
  int nwave_items = 0, nslot_items = 0, nwaves_total = 0, nslots_total = 0;
  double *d_waves_h = nullptr, *d_waves_e = nullptr, *d_phase = nullptr;
  RecItem *d_rec = nullptr;
  long long nrec = 0;
  void *d_ring = nullptr;  // G rows of the transform values
  long long nring = 0;
  int blocks = 0;
  int *d_flags = nullptr;  // one TE-check flag per member
  int flags_cap = 0;
  // for the adjoint's recomputation: transforms and probes off, and after each step the E curl
  // at the design's values into K[step - k_first][value]
  bool record = true;
  const long long *d_design = nullptr;
  long long ndesign = 0;
  void *d_K = nullptr;
  long long k_first = 0;
  // the tables and graph stay good for the next run while every member is as the last run left
  // it: the same generation (no engine call since), step index and current copy
  bool reusable = false;
  bool cap_record = true;
  long long per_chunk = 0;  // the graph's kernels
  std::vector<unsigned long long> gens;
  std::vector<int64_t> next_first;
  std::vector<int> next_parity;
  std::vector<cudaEvent_t> member_ev;
};

namespace {

int bfail(fdtd_batch *b, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  b->error = buf;
  return code;
}

#define BTRY(b, call)                                                                     \
  do {                                                                                    \
    cudaError_t err_ = (call);                                                            \
    if (err_ != cudaSuccess)                                                              \
      return bfail((b), FDTD_E_GPU, "%s: %s", #call, cudaGetErrorString(err_));           \
  } while (0)

void free_tables(fdtd_batch *b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  for (void *p : b->allocs) cudaFreeAsync(p, b->stream);  // after the batch's work so far
  b->allocs.clear();
}

// Whether the batch can step simulation i (a 2D TE grid in the batch's precision, no media).
int admissible(fdtd_batch *b, const InstanceView &v, int i) {
  if (v.precision != b->precision)
    return bfail(b, FDTD_E_INVALID, "simulation %d is in f%d, the batch in f%d", i, v.precision,
                 b->precision);
  if (v.n[2] != 1 || !v.periodic[2])
    return bfail(b, FDTD_E_INVALID,
                 "simulation %d is not a 2D grid (one cell along z, periodic there)", i);
  if (v.media)
    return bfail(b, FDTD_E_INVALID,
                 "simulation %d has dispersive media, which the batch does not step", i);
  if (v.plane_waves)
    return bfail(b, FDTD_E_INVALID,
                 "simulation %d has a plane wave's box, which the batch does not step", i);
  return 0;
}

template <typename V>
int upload_vec(fdtd_batch *b, V **dst, const std::vector<V> &v) {
  *dst = nullptr;
  size_t bytes = std::max<size_t>(v.size(), 1) * sizeof(V);
  void *p = nullptr;
  BTRY(b, cudaMallocAsync(&p, bytes, b->stream));  // stream-ordered: no device-wide sync
  b->allocs.push_back(p);
  if (!v.empty())
    BTRY(b, cudaMemcpyAsync(p, v.data(), v.size() * sizeof(V), cudaMemcpyHostToDevice, b->stream));
  *dst = static_cast<V *>(p);
  return 0;
}
int zeros(fdtd_batch *b, double **dst, size_t n) {
  void *p = nullptr;
  BTRY(b, cudaMallocAsync(&p, std::max<size_t>(n, 1) * 8, b->stream));
  b->allocs.push_back(p);
  BTRY(b, cudaMemsetAsync(p, 0, std::max<size_t>(n, 1) * 8, b->stream));
  *dst = static_cast<double *>(p);
  return 0;
}

// The tables for tile shape `sh`: per-instance descriptors (starting at step first[i], copy
// parity[i], record row rows[i]), the tile list, the sources' groups per tile, the waveforms,
// the transforms' phase slots and the record items.
template <typename T>
int build(fdtd_batch *b, const std::vector<InstanceView> &views, const std::vector<int64_t> &first,
          const std::vector<int> &parity, const std::vector<double *> &rows, int sh) {
  free_tables(b);
  const int TW = SHAPES[sh].tw, TH = SHAPES[sh].th;
  std::vector<TeInst<T>> insts(views.size());
  std::vector<int> tile_inst;
  std::vector<int> hb{0}, eb{0};
  std::vector<Group> hgroups, egroups;
  std::vector<Entry> entries;
  std::vector<Wave> waves;
  std::vector<int> point;
  std::vector<int2> wave_items, slot_items;
  std::vector<RecItem> rec;
  long long nring = 0;
  int bucket = 0, slots = 0;
  for (size_t i = 0; i < views.size(); i++) {
    const InstanceView &v = views[i];
    TeInst<T> &I = insts[i];
    memset(&I, 0, sizeof I);
    I.nx = v.n[0];
    I.ny = v.n[1];
    I.px = v.periodic[0];
    I.py = v.periodic[1];
    I.N = v.N;
    I.dt = (T)v.dt;
    I.dt64 = v.dt;
    I.sx = (T)v.step[0];
    I.sy = (T)v.step[1];
    I.inv_sx = (T)v.inv_step[0];
    I.inv_sy = (T)v.inv_step[1];
    I.fast_x = v.fast_div[0];
    I.rd_x = 1.0 / (double)I.sx;
    I.rd_y = 1.0 / (double)I.sy;
    I.fast_y = v.fast_div[1];
    for (int p = 0; p < 2; p++) {
      I.e[p] = (T *)v.e[p];
      I.h[p] = (T *)v.h[p];
      I.psi_h[p] = (T *)v.psi_h[p];
    }
    I.psi_e = (T *)v.psi_e;
    I.ca = (const T *)v.ca;
    I.cb = (const T *)v.cb;
    I.fe = (const T *)v.fe;
    I.fh = (const T *)v.fh;
    I.coefs = (const T *)v.coefs;
    for (int s = 0; s < 2; s++) {
      I.hx[s] = v.table[1][2][0][s];
      I.hy[s] = v.table[1][2][1][s];
      I.ex[s] = v.table[0][1][0][s];
      I.ey[s] = v.table[0][0][1][s];
    }
    I.parity = parity[i];
    I.first = first[i];
    I.rows = rows[i];
    I.tiles_x = (I.nx + TW - 1) / TW;
    const int tiles_y = (I.ny + TH - 1) / TH;
    const int ntile = I.tiles_x * tiles_y;
    I.tile0 = (int)tile_inst.size();
    for (int t = 0; t < ntile; t++) tile_inst.push_back((int)i);
    I.bucket0 = bucket;
    // the waveforms, numbered batch-wide
    I.wave0 = (int)waves.size();
    I.nwaves = (int)v.waves->size();
    std::vector<int> pt(I.nwaves, 0);
    for (const fdtd_injection &x : *v.inj) pt[x.emitter] = x.point ? 1 : 0;
    for (int e = 0; e < I.nwaves; e++) {
      Wave w;
      w.kind = (*v.waves)[e].kind;
      for (int p = 0; p < 5; p++) w.p[p] = (*v.waves)[e].p[p];
      waves.push_back(w);
      point.push_back(pt[e]);
      wave_items.push_back(make_int2((int)i, I.wave0 + e));
    }
    // sources: grouped by value in CPU order (as fdtd_set_sources), then by tile. An H value
    // goes to each tile whose H region (its cells and the row and column below) holds it.
    std::vector<std::vector<Group>> hper(ntile), eper(ntile);
    for (int f = 0; f < 2; f++) {
      std::unordered_map<long long, int> index;
      std::vector<long long> places;
      std::vector<std::vector<Entry>> lists;
      for (const fdtd_injection &x : *v.inj) {
        if (x.field != f) continue;
        const long long place = (long long)x.component * v.N + x.r;
        auto it = index.find(place);
        int at;
        if (it == index.end()) {
          at = (int)places.size();
          index[place] = at;
          places.push_back(place);
          lists.emplace_back();
        } else {
          at = it->second;
        }
        Entry en;
        en.are = x.a_re;
        en.aim = x.a_im;
        en.emitter = I.wave0 + x.emitter;
        en.pad = 0;
        lists[at].push_back(en);
      }
      for (size_t g = 0; g < places.size(); g++) {
        const int comp = (int)(places[g] / v.N);
        const long long r = places[g] % v.N;
        const int x = (int)(r % I.nx), y = (int)(r / I.nx);
        if ((f == 1 && comp != 2) || (f == 0 && comp == 2))
          return bfail(b, FDTD_E_INVALID,
                       "simulation %zu has a source on %s_%c: the batch steps TE grids (E_x, E_y, "
                       "H_z)", i, f ? "H" : "E", "xyz"[comp]);
        auto add = [&](std::vector<Group> &to, int local) {
          Group c;
          c.local = local;
          c.comp = comp;
          c.first = (int)entries.size();
          c.count = (int)lists[g].size();
          for (const Entry &e : lists[g]) entries.push_back(e);
          to.push_back(c);
        };
        if (f == 0) {
          const int tx = x / TW, ty = y / TH;
          add(eper[ty * I.tiles_x + tx], (y - ty * TH) * TW + (x - tx * TW));
          continue;
        }
        // (tile, position in its H region) along each axis: its own tile, and the tile whose
        // column (row) below it is, also across a periodic wrap. The region starts `off` places
        // before the tile: one row; one column, or te_quad_kernel's first lane's four places
        auto options = [](int c, int n, int w, int periodic, int off) {
          std::vector<std::pair<int, int>> o{{c / w, c - (c / w) * w + off}};
          if (c + 1 < n && (c + 1) % w == 0) o.push_back({(c + 1) / w, off - 1});
          if (periodic && c == n - 1) o.push_back({0, off - 1});
          return o;
        };
        const bool rows = sh == QUAD_SHAPE;
        const int xoff = rows ? teq::VEC : 1, hrow = rows ? teq::ROW : TW + 1;
        for (auto oy : options(y, I.ny, TH, I.py, 1))
          for (auto ox : options(x, I.nx, TW, I.px, xoff))
            add(hper[oy.first * I.tiles_x + ox.first], oy.second * hrow + ox.second);
      }
    }
    for (int t = 0; t < ntile; t++) {
      for (const Group &g : hper[t]) hgroups.push_back(g);
      for (const Group &g : eper[t]) egroups.push_back(g);
      hb.push_back((int)hgroups.size());
      eb.push_back((int)egroups.size());
    }
    bucket += ntile;
    // transforms and probes
    I.where = v.where;
    I.series = v.series;
    I.value_series = v.value_series;
    I.omega = v.omega;
    I.slot_field = v.slot_field;
    I.sums = v.sums;
    I.probes = v.probes;
    I.nprobes = v.nprobes;
    I.slot0 = slots;
    I.nslots = v.nvalues > 0 ? v.nslots : 0;
    for (int s = 0; s < I.nslots; s++) slot_items.push_back(make_int2((int)i, s));
    slots += I.nslots;
    for (long long q = 0; q < v.nvalues; q++) rec.push_back(RecItem{(int)i, 0, q, nring++});
    for (int p = 0; p < v.nprobes; p++) rec.push_back(RecItem{(int)i, 1, p, -1});
  }
  b->ntiles = (int)tile_inst.size();
  b->nwaves_total = (int)waves.size();
  b->nslots_total = slots;
  b->nwave_items = (int)wave_items.size();
  b->nslot_items = (int)slot_items.size();
  b->nrec = (long long)rec.size();
  if (int r = upload_vec(b, (TeInst<T> **)&b->d_insts, insts)) return r;
  if (int r = upload_vec(b, &b->d_tile_inst, tile_inst)) return r;
  if (int r = upload_vec(b, &b->d_hbucket, hb)) return r;
  if (int r = upload_vec(b, &b->d_ebucket, eb)) return r;
  if (int r = upload_vec(b, &b->d_hgroups, hgroups)) return r;
  if (int r = upload_vec(b, &b->d_egroups, egroups)) return r;
  if (int r = upload_vec(b, &b->d_entries, entries)) return r;
  if (int r = upload_vec(b, &b->d_waves, waves)) return r;
  if (int r = upload_vec(b, &b->d_point, point)) return r;
  if (int r = upload_vec(b, &b->d_wave_items, wave_items)) return r;
  if (int r = upload_vec(b, &b->d_slot_items, slot_items)) return r;
  if (int r = upload_vec(b, &b->d_rec, rec)) return r;
  if (int r = zeros(b, &b->d_waves_h, (size_t)G * std::max(b->nwaves_total, 1) * 2)) return r;
  if (int r = zeros(b, &b->d_waves_e, (size_t)G * std::max(b->nwaves_total, 1) * 2)) return r;
  if (int r = zeros(b, &b->d_phase, (size_t)G * std::max(b->nslots_total, 1) * 2)) return r;
  b->nring = nring;
  {
    double *ring = nullptr;
    if (int r = zeros(b, &ring, ((size_t)G * std::max<long long>(nring, 1) * sizeof(T) + 7) / 8))
      return r;
    b->d_ring = ring;
  }
  b->shape = sh;
  return 0;
}

template <typename T, int TW, int TH>
void launch_step(fdtd_batch *b, int m) {
  te_step_kernel<T, TW, TH><<<b->blocks, THREADS, 0, b->stream>>>(
      (const TeInst<T> *)b->d_insts, b->d_tile_inst, b->ntiles, b->d_hbucket, b->d_ebucket,
      b->d_hgroups, b->d_egroups, b->d_entries,
      b->d_waves_h + 2LL * m * b->nwaves_total, b->d_waves_e + 2LL * m * b->nwaves_total, m);
}

template <typename T>
void step_by_shape(fdtd_batch *b, int m) {
  switch (b->shape) {
    case 0: launch_step<T, 32, 8>(b, m); break;
    case 1: launch_step<T, 32, 16>(b, m); break;
    case 2: launch_step<T, 64, 4>(b, m); break;
    case 3: launch_step<T, 64, 8>(b, m); break;
    case 4: launch_step<T, 128, 2>(b, m); break;
    case 5: launch_step<T, 128, 4>(b, m); break;
    default:
      te_quad_kernel<T><<<b->blocks, THREADS, 0, b->stream>>>(
          (const TeInst<T> *)b->d_insts, b->d_tile_inst, b->ntiles, b->d_hbucket, b->d_ebucket,
          b->d_hgroups, b->d_egroups, b->d_entries,
          b->d_waves_h + 2LL * m * b->nwaves_total, b->d_waves_e + 2LL * m * b->nwaves_total, m);
      break;
  }
}

template <typename T>
int occupancy(fdtd_batch *b) {
  int per = 1;
  switch (b->shape) {
    case 0: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, te_step_kernel<T, 32, 8>, THREADS, 0); break;
    case 1: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, te_step_kernel<T, 32, 16>, THREADS, 0); break;
    case 2: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, te_step_kernel<T, 64, 4>, THREADS, 0); break;
    case 3: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, te_step_kernel<T, 64, 8>, THREADS, 0); break;
    case 4: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, te_step_kernel<T, 128, 2>, THREADS, 0); break;
    case 5: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, te_step_kernel<T, 128, 4>, THREADS, 0); break;
    default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, te_quad_kernel<T>, THREADS, 0); break;
  }
  return std::max(per, 1);
}

// `count` (<= G) steps of the current tables on the batch's stream; then the instances advance.
template <typename T>
void enqueue(fdtd_batch *b, int count) {
  TeInst<T> *insts = (TeInst<T> *)b->d_insts;
  const int n = (int)b->ctxs.size();
  if (b->nwave_items > 0) {
    int total = b->nwave_items * G;
    te_waves_kernel<T><<<(total + 127) / 128, 128, 0, b->stream>>>(
        insts, b->d_wave_items, b->nwave_items, b->d_waves, b->d_point, b->nwaves_total,
        b->d_waves_h, b->d_waves_e);
    b->launches++;
  }
  if (b->nslot_items > 0 && b->record) {
    int total = b->nslot_items * G;
    te_phase_kernel<T><<<(total + 127) / 128, 128, 0, b->stream>>>(
        insts, b->d_slot_items, b->nslot_items, b->nslots_total, b->d_phase);
    b->launches++;
  }
  for (int m = 0; m < count; m++) {
    step_by_shape<T>(b, m);
    b->launches++;
    if (b->nrec > 0 && b->record) {
      te_record_kernel<T><<<(unsigned)((b->nrec + 255) / 256), 256, 0, b->stream>>>(
          insts, b->d_rec, b->nrec, (T *)b->d_ring, b->nring, m);
      b->launches++;
    }
    if (b->ndesign > 0) {
      te_design_kernel<T><<<(unsigned)((b->ndesign + 255) / 256), 256, 0, b->stream>>>(
          insts, b->d_design, b->ndesign, (T *)b->d_K, b->k_first, m);
      b->launches++;
    }
  }
  if (b->nring > 0 && b->record) {
    te_contract_kernel<T><<<(unsigned)((b->nrec + 127) / 128), 128, 0, b->stream>>>(
        insts, b->d_rec, b->nrec, (const T *)b->d_ring, b->nring, b->d_phase, b->nslots_total,
        count);
    b->launches++;
  }
  te_advance_kernel<T><<<(n + 127) / 128, 128, 0, b->stream>>>(insts, n, count);
  b->launches++;
}

// The run's steps from `done` on with the current tables: whole chunks by the captured graph
// (captured now if there is none), the rest launched; then the members' streams wait for them.
template <typename T>
int finish_run(fdtd_batch *b, int64_t steps, int64_t done, const std::vector<InstanceView> &views) {
  const int n = (int)b->ctxs.size();
  const int64_t full = (steps - done) / G;
  if (full > 0) {
    if (!b->graph) {
      // one chunk captured as a graph, replayed
      cudaGraph_t g = nullptr;
      const long long before = b->launches;
      BTRY(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      enqueue<T>(b, G);
      cudaError_t err = cudaStreamEndCapture(b->stream, &g);
      if (err != cudaSuccess)
        return bfail(b, FDTD_E_GPU, "cudaStreamEndCapture: %s", cudaGetErrorString(err));
      b->per_chunk = b->launches - before;
      b->launches = before;
      err = cudaGraphInstantiate(&b->graph, g, 0);
      cudaGraphDestroy(g);
      if (err != cudaSuccess)
        return bfail(b, FDTD_E_GPU, "cudaGraphInstantiate: %s", cudaGetErrorString(err));
    }
    for (int64_t c = 0; c < full; c++) {
      BTRY(b, cudaGraphLaunch(b->graph, b->stream));
      b->launches += b->per_chunk;
    }
    done += full * G;
  }
  if (done < steps) enqueue<T>(b, (int)(steps - done));
  BTRY(b, cudaGetLastError());
  BTRY(b, cudaEventRecord(b->done, b->stream));
  for (int i = 0; i < n; i++) {
    BTRY(b, cudaStreamWaitEvent(views[i].stream, b->done, 0));
    fdtd_instance_advance(b->ctxs[i], steps);
  }
  // no wait here: each context's stream waits for the batch's work (the event), so its later
  // calls see the steps; the batch's next run orders after them on the batch's stream
  return 0;
}

// A run whose members are all as the last run left them: its tables and graph serve again, the
// members' streams ordered before it by events (no host waits, no checks, no rebuild).
template <typename T>
int run_again(fdtd_batch *b, int64_t steps, const int64_t *first_steps, bool *ran) {
  *ran = false;
  const int n = (int)b->ctxs.size();
  if (!b->reusable || b->record != b->cap_record || b->ndesign > 0 || (int)b->gens.size() != n)
    return 0;
  std::vector<InstanceView> views(n);
  for (int i = 0; i < n; i++) {
    if (fdtd_instance_view(b->ctxs[i], &views[i])) return 0;
    const InstanceView &v = views[i];
    if (v.generation != b->gens[i] || v.parity != b->next_parity[i] || v.nprobes > 0 ||
        (first_steps ? first_steps[i] : 0) != b->next_first[i])
      return 0;
  }
  while ((int)b->member_ev.size() < n) {
    cudaEvent_t ev;
    BTRY(b, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    b->member_ev.push_back(ev);
  }
  for (int i = 0; i < n; i++) {
    BTRY(b, cudaEventRecord(b->member_ev[i], views[i].stream));
    BTRY(b, cudaStreamWaitEvent(b->stream, b->member_ev[i], 0));
  }
  if (int r = finish_run<T>(b, steps, 0, views)) return r;
  for (int i = 0; i < n; i++) {
    b->next_first[i] += steps;
    b->next_parity[i] = (int)((b->next_parity[i] + steps) & 1);
  }
  *ran = true;
  return 0;
}

template <typename T>
int run_impl(fdtd_batch *b, int64_t steps, const int64_t *first_steps) {
  bool ran = false;
  if (int r = run_again<T>(b, steps, first_steps, &ran)) return r;
  if (ran) return 0;
  const int n = (int)b->ctxs.size();
  std::vector<InstanceView> views(n);
  std::vector<int64_t> first(n);
  std::vector<int> parity(n);
  std::vector<double *> rows(n, nullptr);
  int dev = 0;
  BTRY(b, cudaGetDevice(&dev));
  BTRY(b, cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev));
  for (int i = 0; i < n; i++) {
    fdtd_ctx *c = b->ctxs[i];
    if (int r = fdtd_instance_view(c, &views[i]))
      return bfail(b, r, "simulation %d: %s", i, fdtd_last_error(c));
    const InstanceView &v = views[i];
    if (int r = admissible(b, v, i)) return r;
    if (int r = fdtd_instance_reserve(c, steps, &rows[i]))
      return bfail(b, r, "simulation %d: %s", i, fdtd_last_error(c));
    first[i] = first_steps ? first_steps[i] : 0;
    parity[i] = v.parity;
  }
  // the members' streams before the batch's (events: the host doesn't wait), then one check of
  // every member's TM components (one flag each) and one wait for its answer
  while ((int)b->member_ev.size() < n) {
    cudaEvent_t ev;
    BTRY(b, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    b->member_ev.push_back(ev);
  }
  if (b->flags_cap < n) {
    if (b->d_flags) BTRY(b, cudaFreeAsync(b->d_flags, b->stream));
    b->d_flags = nullptr;
    BTRY(b, cudaMallocAsync(&b->d_flags, (size_t)n * 4, b->stream));
    b->flags_cap = n;
  }
  BTRY(b, cudaMemsetAsync(b->d_flags, 0, (size_t)n * 4, b->stream));
  for (int i = 0; i < n; i++) {
    const InstanceView &v = views[i];
    BTRY(b, cudaEventRecord(b->member_ev[i], v.stream));
    BTRY(b, cudaStreamWaitEvent(b->stream, b->member_ev[i], 0));
    te_tm_check_kernel<T><<<(unsigned)((v.N + 255) / 256), 256, 0, b->stream>>>(
        (const T *)v.e[v.parity], (const T *)v.h[v.parity], v.N, b->d_flags + i);
    // the other copy's TM components stay zero too
    const size_t E = sizeof(T);
    BTRY(b, cudaMemsetAsync((char *)v.h[1 - v.parity], 0, 2 * v.N * E, b->stream));
    BTRY(b, cudaMemsetAsync((char *)v.e[1 - v.parity] + 2 * v.N * E, 0, v.N * E, b->stream));
  }
  {
    std::vector<int> bad(n, 0);
    BTRY(b, cudaMemcpyAsync(bad.data(), b->d_flags, (size_t)n * 4, cudaMemcpyDeviceToHost,
                            b->stream));
    BTRY(b, cudaStreamSynchronize(b->stream));
    for (int i = 0; i < n; i++)
      if (bad[i])
        return bfail(b, FDTD_E_INVALID,
                     "simulation %d has H_x, H_y or E_z values: the batch steps TE fields only", i);
  }
  // where the device's descriptors have moved the instances to
  auto pull = [&]() -> int {
    std::vector<TeInst<T>> now(n);
    BTRY(b, cudaStreamSynchronize(b->stream));
    BTRY(b, cudaMemcpy(now.data(), b->d_insts, n * sizeof(TeInst<T>), cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; i++) {
      first[i] = now[i].first;
      parity[i] = now[i].parity;
      rows[i] = now[i].rows;
    }
    return 0;
  };
  auto rebuild = [&](int sh) -> int {
    if (int r = build<T>(b, views, first, parity, rows, sh)) return r;
    b->blocks = occupancy<T>(b) * b->sms;
    return 0;
  };
  int64_t done = 0;
  // the tile shape: each shape times one chunk of real steps (after one warm chunk), the
  // fastest is kept; every shape gives the same bits
  if (b->shape < 0) {
    if (steps >= 2LL * NSHAPES * G + G) {
      float best = 1e30f;
      int pick = 0;
      for (int sh = 0; sh < NSHAPES; sh++) {
        if (int r = rebuild(sh)) return r;
        enqueue<T>(b, G);
        BTRY(b, cudaEventRecord(b->t0, b->stream));
        enqueue<T>(b, G);
        BTRY(b, cudaEventRecord(b->t1, b->stream));
        BTRY(b, cudaEventSynchronize(b->t1));
        float ms = 0.f;
        BTRY(b, cudaEventElapsedTime(&ms, b->t0, b->t1));
        if (ms < best) {
          best = ms;
          pick = sh;
        }
        done += 2 * G;
        if (int r = pull()) return r;
      }
      b->shape = pick;
    } else {
      b->shape = DEFAULT_SHAPE;
    }
  }
  if (int r = rebuild(b->shape)) return r;
  b->reusable = false;
  if (int r = finish_run<T>(b, steps, done, views)) return r;
  b->reusable = true;
  b->cap_record = b->record;
  b->gens.assign(n, 0);
  b->next_first.assign(n, 0);
  b->next_parity.assign(n, 0);
  for (int i = 0; i < n; i++) {
    b->gens[i] = views[i].generation;
    b->next_first[i] = (first_steps ? first_steps[i] : 0) + steps;
    b->next_parity[i] = (int)((views[i].parity + steps) & 1);
  }
  return 0;
}

}  // namespace

extern "C" {

int fdtd_batch_create(int32_t count, fdtd_ctx *const *ctxs, fdtd_batch **out) {
  if (!out) return FDTD_E_INVALID;
  *out = nullptr;
  fdtd_batch *b = new fdtd_batch();
  *out = b;
  if (count <= 0 || !ctxs) return bfail(b, FDTD_E_INVALID, "a batch needs simulations");
  for (int i = 0; i < count; i++) {
    if (!ctxs[i]) return bfail(b, FDTD_E_INVALID, "simulation %d has no engine", i);
    for (int j = 0; j < i; j++)
      if (ctxs[j] == ctxs[i]) return bfail(b, FDTD_E_INVALID, "simulation %d is in the batch twice", i);
    b->ctxs.push_back(ctxs[i]);
  }
  for (int i = 0; i < count; i++) {
    InstanceView v;
    if (int r = fdtd_instance_view(ctxs[i], &v))
      return bfail(b, r, "simulation %d: %s", i, fdtd_last_error(ctxs[i]));
    if (i == 0) b->precision = v.precision;
    if (int r = admissible(b, v, i)) return r;
  }
  BTRY(b, cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  BTRY(b, cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
  BTRY(b, cudaEventCreate(&b->t0));
  BTRY(b, cudaEventCreate(&b->t1));
  return 0;
}

const char *fdtd_batch_last_error(const fdtd_batch *b) { return b ? b->error.c_str() : "no batch"; }

int fdtd_batch_run(fdtd_batch *b, int64_t steps, const int64_t *first_steps) {
  if (!b) return FDTD_E_INVALID;
  if (steps < 0) return bfail(b, FDTD_E_INVALID, "a negative number of steps");
  if (steps == 0) return 0;
  int r = b->precision == 64 ? run_impl<double>(b, steps, first_steps)
                             : run_impl<float>(b, steps, first_steps);
  return r;
}

int fdtd_batch_tile(const fdtd_batch *b, int32_t *width, int32_t *height) {
  if (!b || !width || !height) return FDTD_E_INVALID;
  *width = b->shape >= 0 ? SHAPES[b->shape].tw : 0;
  *height = b->shape >= 0 ? SHAPES[b->shape].th : 0;
  return 0;
}

int fdtd_batch_set_tile(fdtd_batch *b, int32_t width, int32_t height) {
  if (!b) return FDTD_E_INVALID;
  b->reusable = false;
  if (width == 0 && height == 0) {
    b->shape = -1;
    return 0;
  }
  for (int s = 0; s < NSHAPES; s++)
    if (SHAPES[s].tw == width && SHAPES[s].th == height) {
      b->shape = s;
      return 0;
    }
  return bfail(b, FDTD_E_INVALID, "no tile shape %d x %d", width, height);
}

int64_t fdtd_batch_launches(const fdtd_batch *b) { return b ? b->launches : 0; }

void fdtd_batch_destroy(fdtd_batch *b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  free_tables(b);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->done) cudaEventDestroy(b->done);
  if (b->t0) cudaEventDestroy(b->t0);
  if (b->t1) cudaEventDestroy(b->t1);
  for (cudaEvent_t ev : b->member_ev) cudaEventDestroy(ev);
  if (b->d_flags) cudaFreeAsync(b->d_flags, b->stream);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// The adjoint of one 2D TE simulation's run (include/photonoxide_adjoint.h): the forward steps
// keep a checkpoint at the start of each segment; the reverse pass recomputes each segment from
// its checkpoint (keeping the curls at the design's values), then steps the adjoint back through
// it, adding E~ x curl into dJ/dcb.

struct fdtd_adjoint {
  std::string error;
  fdtd_ctx *ctx = nullptr;
  fdtd_batch *batch = nullptr;  // the simulation alone, for its forward steps
  int precision = 32;
  int64_t steps = 0;
  int segment = 0;
  int nseg = 0;
  int64_t first = 0;  // the forward run's first step index
  bool forward_done = false;
  long long ndesign = 0;
  long long *d_design = nullptr;
  void *d_K = nullptr;          // segment x ndesign curls
  double *d_grad = nullptr;     // ndesign
  double *d_gsums = nullptr;    // dJ/dsums
  double *d_phase = nullptr;    // segment x nslots phases
  // the injection's owners (te_inject_kernel): field values, their transform values
  long long *d_owner = nullptr, *d_order = nullptr;
  int *d_start = nullptr;
  int nowners = 0;
  // checkpoints: E_x, E_y, H_z, H's psi and E's psi at the start of each segment, and at the end
  void *d_ckpt = nullptr;
  size_t ckpt_bytes = 0;
  // the adjoint state: E~ (2N), H~ (N), psi~ (E's, H's), two copies
  void *d_adj = nullptr;
  long long N = 0, psi_e_len = 0, psi_h_len = 0;
  std::vector<void *> allocs;
};

namespace {

int afail(fdtd_adjoint *a, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  a->error = buf;
  return code;
}

#define ATRY(a, call)                                                                     \
  do {                                                                                    \
    cudaError_t err_ = (call);                                                            \
    if (err_ != cudaSuccess)                                                              \
      return afail((a), FDTD_E_GPU, "%s: %s", #call, cudaGetErrorString(err_));           \
  } while (0)

int amalloc(fdtd_adjoint *a, void **p, size_t bytes) {
  *p = nullptr;
  ATRY(a, cudaMalloc(p, std::max<size_t>(bytes, 16)));
  a->allocs.push_back(*p);
  return 0;
}

// Copies the simulation's state (its current copies) into checkpoint k, or back from it.
int checkpoint(fdtd_adjoint *a, int k, bool save) {
  InstanceView v;
  if (int r = fdtd_instance_view(a->ctx, &v)) return afail(a, r, "%s", fdtd_last_error(a->ctx));
  const size_t E = a->precision == 64 ? 8 : 4;
  char *base = (char *)a->d_ckpt + (size_t)k * a->ckpt_bytes;
  struct Part {
    void *dev;
    size_t bytes;
  };
  const Part parts[] = {{v.e[v.parity], 2 * v.N * E},
                        {(char *)v.h[v.parity] + 2 * v.N * E, v.N * E},
                        {v.psi_h[v.parity], v.psi_h_len * E},
                        {v.psi_e, v.psi_e_len * E}};
  size_t at = 0;
  for (const Part &p : parts) {
    if (p.bytes) {
      if (save)
        ATRY(a, cudaMemcpyAsync(base + at, p.dev, p.bytes, cudaMemcpyDeviceToDevice, v.stream));
      else
        ATRY(a, cudaMemcpyAsync(p.dev, base + at, p.bytes, cudaMemcpyDeviceToDevice, v.stream));
    }
    at += (p.bytes + 255) / 256 * 256;
  }
  ATRY(a, cudaStreamSynchronize(v.stream));
  return 0;
}

// The forward run: segment by segment, each one's start kept as a checkpoint, then the end.
int forward_impl(fdtd_adjoint *a, int64_t first) {
  a->first = first;
  int64_t done = 0;
  for (int k = 0; k < a->nseg; k++) {
    if (int r = checkpoint(a, k, true)) return r;
    const int64_t len = std::min<int64_t>(a->segment, a->steps - done);
    const int64_t at = first + done;
    if (int r = fdtd_batch_run(a->batch, len, &at))
      return afail(a, r, "%s", fdtd_batch_last_error(a->batch));
    done += len;
  }
  if (int r = checkpoint(a, a->nseg, true)) return r;
  a->forward_done = true;
  return 0;
}

template <typename T>
int backward_impl(fdtd_adjoint *a, const double *grad_sums, double *grad_cb) {
  fdtd_batch *b = a->batch;
  InstanceView v;
  if (int r = fdtd_instance_view(a->ctx, &v)) return afail(a, r, "%s", fdtd_last_error(a->ctx));
  const long long N = a->N;
  // the adjoint state, from zero
  T *base = (T *)a->d_adj;
  AdjState<T> A;
  const long long pe = (a->psi_e_len + 63) / 64 * 64, ph = (a->psi_h_len + 63) / 64 * 64;
  const long long per = 3 * N + pe + ph;
  for (int c = 0; c < 2; c++) {
    T *p = base + c * per;
    A.e[c] = p;
    A.h[c] = p + 2 * N;
    A.pe[c] = p + 3 * N;
    A.ph[c] = p + 3 * N + pe;
  }
  A.cur = 0;
  ATRY(a, cudaMemsetAsync(a->d_adj, 0, 2 * per * sizeof(T), b->stream));
  ATRY(a, cudaMemsetAsync(a->d_grad, 0, a->ndesign * 8, b->stream));
  if (v.nsums > 0)
    ATRY(a, cudaMemcpyAsync(a->d_gsums, grad_sums, v.nsums * 16, cudaMemcpyHostToDevice,
                            b->stream));
  ATRY(a, cudaStreamSynchronize(b->stream));
  const int TW = 64, TH = 8;
  const int tiles = ((v.n[0] + TW - 1) / TW) * ((v.n[1] + TH - 1) / TH);
  int per_sm = 1, dev = 0, sms = 148;
  ATRY(a, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, te_adjoint_kernel<T, 64, 8>,
                                                        THREADS, 0));
  ATRY(a, cudaGetDevice(&dev));
  ATRY(a, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = std::max(1, std::min(tiles, std::max(per_sm, 1) * sms));
  for (int k = a->nseg - 1; k >= 0; k--) {
    const int64_t seg0 = (int64_t)k * a->segment;
    const int len = (int)std::min<int64_t>(a->segment, a->steps - seg0);
    // the segment again from its checkpoint: transforms and probes off, the curls kept
    if (int r = checkpoint(a, k, false)) return r;
    b->record = false;
    b->d_design = a->d_design;
    b->ndesign = a->ndesign;
    b->d_K = a->d_K;
    b->k_first = a->first + seg0;
    const int64_t at = a->first + seg0;
    const int r = fdtd_batch_run(b, len, &at);
    b->record = true;
    b->d_design = nullptr;
    b->ndesign = 0;
    b->d_K = nullptr;
    if (r) return afail(a, r, "%s", fdtd_batch_last_error(b));
    fdtd_instance_advance(a->ctx, -len);  // its probe record stays as the forward run left it
    // that run's tables (the one simulation) hold what the adjoint reads
    const TeInst<T> *insts = (const TeInst<T> *)b->d_insts;
    if (v.nsums > 0 && v.nslots > 0) {
      const int total = len * v.nslots;
      te_segment_phase_kernel<T><<<(total + 127) / 128, 128, 0, b->stream>>>(insts, at, len,
                                                                            a->d_phase);
    }
    for (int m = len - 1; m >= 0; m--) {
      if (v.nsums > 0 && a->nowners > 0)
        te_inject_kernel<T><<<(unsigned)((a->nowners + 255) / 256), 256, 0, b->stream>>>(
            insts, a->d_owner, a->d_start, a->d_order, a->nowners, a->d_phase, a->d_gsums, A, m);
      te_grad_kernel<T><<<(unsigned)((a->ndesign + 255) / 256), 256, 0, b->stream>>>(
          a->d_design, a->ndesign, (const T *)a->d_K + (long long)m * a->ndesign, A, a->d_grad);
      te_adjoint_kernel<T, 64, 8><<<blocks, THREADS, 0, b->stream>>>(insts, A, tiles);
      A.cur = 1 - A.cur;
    }
    ATRY(a, cudaGetLastError());
  }
  ATRY(a, cudaMemcpyAsync(grad_cb, a->d_grad, a->ndesign * 8, cudaMemcpyDeviceToHost, b->stream));
  ATRY(a, cudaStreamSynchronize(b->stream));
  // the simulation as the forward run left it
  return checkpoint(a, a->nseg, false);
}

}  // namespace

extern "C" {

int fdtd_adjoint_create(fdtd_ctx *ctx, int64_t steps, int32_t segment, int64_t count,
                        const int32_t *component, const int64_t *r, fdtd_adjoint **out) {
  if (!out) return FDTD_E_INVALID;
  fdtd_adjoint *a = new fdtd_adjoint();
  *out = a;
  if (!ctx) return afail(a, FDTD_E_INVALID, "no simulation");
  if (steps <= 0)
    return afail(a, FDTD_E_INVALID, "an adjoint needs steps, got %lld", (long long)steps);
  if (segment <= 0) return afail(a, FDTD_E_INVALID, "segments need steps, got %d", segment);
  if (count <= 0 || !component || !r) return afail(a, FDTD_E_INVALID, "a design needs values");
  a->ctx = ctx;
  a->steps = steps;
  a->segment = segment + (segment & 1);  // even: every checkpoint has the same current copy
  a->nseg = (int)((steps + a->segment - 1) / a->segment);
  InstanceView v;
  if (int q = fdtd_instance_view(ctx, &v)) return afail(a, q, "%s", fdtd_last_error(ctx));
  a->precision = v.precision;
  a->N = v.N;
  a->psi_e_len = v.psi_e_len;
  a->psi_h_len = v.psi_h_len;
  if (v.media) return afail(a, FDTD_E_INVALID, "the adjoint does not step dispersive media");
  if (v.plane_waves)
    return afail(a, FDTD_E_INVALID, "the adjoint does not step a plane wave's box");
  std::vector<long long> design(count);
  for (int64_t d = 0; d < count; d++) {
    if (component[d] < 0 || component[d] > 1 || r[d] < 0 || r[d] >= v.N)
      return afail(a, FDTD_E_INVALID, "design value %lld is not an E_x or E_y value of the grid",
                   (long long)d);
    design[d] = (long long)component[d] * v.N + r[d];
  }
  // design values clear of the CPMLs and the electric sources: there the derivative of the new
  // E by cb is the curl alone
  for (const fdtd_injection &x : *v.inj)
    if (x.field == 0)
      for (long long d : design)
        if ((long long)x.component * v.N + x.r == d)
          return afail(a, FDTD_E_INVALID, "a design value carries an electric source");
  for (long long d : design) {
    const long long rr = d % v.N;
    const int x = (int)(rr % v.n[0]), y = (int)(rr / v.n[0]);
    if ((!v.periodic[0] && (x < v.low[0] || x >= v.n[0] - v.high[0])) ||
        (!v.periodic[1] && (y < v.low[1] || y >= v.n[1] - v.high[1])))
      return afail(a, FDTD_E_INVALID, "design value (%d, %d) is in a CPML", x, y);
  }
  a->ndesign = count;
  const size_t E = v.precision == 64 ? 8 : 4;
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  a->ckpt_bytes = up(2 * v.N * E) + up(v.N * E) + up(v.psi_h_len * E) + up(v.psi_e_len * E);
  const long long pe = (v.psi_e_len + 63) / 64 * 64, ph = (v.psi_h_len + 63) / 64 * 64;
  if (int q = amalloc(a, (void **)&a->d_design, count * 8)) return q;
  if (int q = amalloc(a, &a->d_K, (size_t)a->segment * count * E)) return q;
  if (int q = amalloc(a, (void **)&a->d_grad, count * 8)) return q;
  if (int q = amalloc(a, (void **)&a->d_gsums, std::max<long long>(v.nsums, 1) * 16)) return q;
  if (int q = amalloc(a, (void **)&a->d_phase, (size_t)a->segment * std::max(v.nslots, 1) * 16))
    return q;
  if (int q = amalloc(a, &a->d_ckpt, (size_t)(a->nseg + 1) * a->ckpt_bytes)) return q;
  if (int q = amalloc(a, &a->d_adj, (size_t)2 * (3 * v.N + pe + ph) * E)) return q;
  ATRY(a, cudaMemcpy(a->d_design, design.data(), count * 8, cudaMemcpyHostToDevice));
  // the field values the transforms record, each with its transform values in value order
  if (v.nvalues > 0 && v.nsums > 0) {
    std::vector<long long> where(v.nvalues);
    ATRY(a, cudaMemcpy(where.data(), v.where, v.nvalues * 8, cudaMemcpyDeviceToHost));
    std::map<long long, std::vector<long long>> by_place;
    for (long long q = 0; q < v.nvalues; q++) {
      const long long place = where[q] & ((1LL << 62) - 1);
      const bool hfield = (where[q] >> 62) != 0;
      const int comp = (int)(place / v.N);
      if (hfield ? comp != 2 : comp == 2) continue;  // E_z, H_x, H_y: zero whatever eps
      by_place[where[q]].push_back(q);
    }
    std::vector<long long> owner, order;
    std::vector<int> start(1, 0);
    for (const auto &kv : by_place) {
      owner.push_back(kv.first);
      order.insert(order.end(), kv.second.begin(), kv.second.end());
      start.push_back((int)order.size());
    }
    a->nowners = (int)owner.size();
    if (a->nowners > 0) {
      if (int q = amalloc(a, (void **)&a->d_owner, owner.size() * 8)) return q;
      if (int q = amalloc(a, (void **)&a->d_order, order.size() * 8)) return q;
      if (int q = amalloc(a, (void **)&a->d_start, start.size() * 4)) return q;
      ATRY(a, cudaMemcpy(a->d_owner, owner.data(), owner.size() * 8, cudaMemcpyHostToDevice));
      ATRY(a, cudaMemcpy(a->d_order, order.data(), order.size() * 8, cudaMemcpyHostToDevice));
      ATRY(a, cudaMemcpy(a->d_start, start.data(), start.size() * 4, cudaMemcpyHostToDevice));
    }
  }
  fdtd_ctx *one[1] = {ctx};
  if (int q = fdtd_batch_create(1, one, &a->batch))
    return afail(a, q, "%s", fdtd_batch_last_error(a->batch));
  fdtd_batch_set_tile(a->batch, 64, 8);
  return 0;
}

const char *fdtd_adjoint_last_error(const fdtd_adjoint *a) {
  return a ? a->error.c_str() : "no adjoint";
}

int fdtd_adjoint_forward(fdtd_adjoint *a, int64_t first_step) {
  if (!a || !a->batch) return FDTD_E_INVALID;
  return forward_impl(a, first_step);
}

int fdtd_adjoint_backward(fdtd_adjoint *a, const double *grad_sums, double *grad_cb) {
  if (!a || !a->batch || !grad_cb) return FDTD_E_INVALID;
  if (!a->forward_done) return afail(a, FDTD_E_STATE, "run the forward steps before the adjoint");
  return a->precision == 64 ? backward_impl<double>(a, grad_sums, grad_cb)
                            : backward_impl<float>(a, grad_sums, grad_cb);
}

void fdtd_adjoint_destroy(fdtd_adjoint *a) {
  if (!a) return;
  fdtd_batch_destroy(a->batch);
  for (void *p : a->allocs) cudaFree(p);
  delete a;
}

}  // extern "C"
