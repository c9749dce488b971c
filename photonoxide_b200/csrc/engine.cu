// The B200 FDTD engine: photonoxide's time step (src/fdtd.rs:1319-1419) as CUDA kernels for
// sm_100a, behind the C ABI of include/photonoxide_fdtd.h.
//
// One step is ONE pass over the grid (kernel `step`): each CTA owns a tile of TX x TY values in
// every plane of a run of planes along z and marches up through them. At plane k it stages the
// old E of plane k+1 (with the row and column of neighbours the curl needs) in shared memory,
// computes the new H~ of plane k over its tile and the low row and column around it (E's back
// differences need them; the neighbours' CTAs compute the same values), adds the magnetic
// currents, then updates E of plane k on its tile with the CPML's psi recursions, the electric
// currents and the dispersive media's ADE currents fused in. Each value is computed with the
// same operations in the same order as the reference's CPU kernel (src/fdtd/kernel.rs,
// src/fdtd/kernel/reference.rs): in f64 the engine gives the reference's bits, and in f32 the
// reference's f32 arithmetic (`Yee<f32>`) on problems without sources. Fields, psi and the
// step's old/new copies are ping-ponged (the step reads one copy and writes the other), so
// CTAs never wait on one another.
//
// The probes and transforms are read after each step by a gather kernel into a ring of K steps
// of values; every K steps a contraction kernel adds sum_n F(t_n) e^{i w t_n} dt into f64 sums,
// in time order per value (src/fdtd/monitors.rs:185-206), phases taken in f64 on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "photonoxide_fdtd.h"
#include "common.cuh"
#include "instance.h"
#include "portable.h"

namespace pxf {

constexpr int TX = 32;  // a tile's values along x
constexpr int TY = 16;  // and along y
constexpr int NT = 256; // threads per CTA
constexpr int RX = TX + 2, RY = TY + 2;  // E's staged region: x0-1 .. x0+TX, y0-1 .. y0+TY
constexpr int HX = TX + 1, HY = TY + 1;  // H's computed region: x0-1 .. x0+TX-1, y0-1 ..



struct Pole3 {
  double alpha, xi, gamma;
};

template <typename T>
struct MediaArgs {
  const int *member;  // 3N: index into the compact state, or -1
  const int *group;   // per member: its group
  const T *scale;     // per member: p_m
  T *before;          // per member: E^{n-1}
  T *current;         // per member x maxpoles: J_p^n
  T *previous;        // per member x maxpoles: J_p^{n-1}
  int maxpoles;
  int ngroups;
  const T *gchi;      // per group: chi
  const int *gpoles;  // per group: its pole count
  const T *gpole;     // per group x maxpoles x 3: alpha, xi, gamma
  T two_dt;
  const long long *place;  // per member: its value (component * N + r); members in value order
  long long members;
};

// The quad kernel's runs of z-planes, at most this many (their starts travel with the launch).
constexpr int quad_max_runs = 64;

template <typename T>
struct StepArgs {
  int n[3];
  long long N;
  int periodic[3];
  int low[3], high[3];
  T dt;
  T step[3];
  T inv_step[3];    // 1/step rounded, for div_by_step
  double inv_step64[3];  // 1/step in double, for div_by_step's subnormal quotients
  int fast_div[3];  // div_by_step's product form checked for this step
  const T *fe;  // kappa/h at the nodes: x | y | z
  const T *fh;  // at the halves
  const T *e_in;
  const T *h_in;
  T *e_out;
  T *h_out;
  const T *ca;  // NULL: lossless
  const T *cb;
  SlabEntry slab[2][3][3][2];
  const T *coefs;
  const T *psi_h_in;
  T *psi_h_out;
  T *psi_e;
  // sources: per (tile, k) the groups on H (over the H region) and on E (over the tile)
  const int *hbucket;
  const int *ebucket;
  const Group *hgroups;
  const Group *egroups;
  const Entry *entries;
  const double *waves_h;  // this step's w at H's time: 2 per emitter
  const double *waves_e;  // at E's time
  int tiles_x, tiles_y, zchunk;
  const int *order;  // quad kernel: CTA b takes run order[b] / tiles, tile order[b] % tiles
  int runs[quad_max_runs + 1];  // quad kernel: run r is planes runs[r] .. runs[r+1]-1
  MediaArgs<T> media;
};


// Whether value m along axis w is in a CPML slab there, and which.
template <typename T>
__device__ inline const SlabEntry *slab_at(const StepArgs<T> &A, int field, int c, int w, int m) {
  if (A.periodic[w]) return nullptr;
  int side;
  if (m < A.low[w]) side = 0;
  else if (m >= A.n[w] - A.high[w]) side = 1;
  else return nullptr;
  const SlabEntry *s = &A.slab[field][c][w][side];
  return s->count > 0 ? s : nullptr;
}

// One slab's share of a value's update (src/fdtd/kernel/reference.rs:102-180): psi <- b psi + a
// (dF / h), then H -= dt (sign psi) or E += cb (sign psi). `diff` is the other field's raw
// difference along w (forward for H, back for E), as the curl took it.
template <typename T, int FIELD>
__device__ inline T slab_update(const StepArgs<T> &A, const SlabEntry *s, int c, int w, int i,
                                int j, int k, T diff, T v, T cbv, bool own) {
  int m = w == 0 ? i : (w == 1 ? j : k);
  int q = m - s->from;
  int li = i, lj = j, lk = k;
  int dx = A.n[0], dy = A.n[1];
  if (w == 0) { li = i - s->pf; dx = s->pw; }
  else if (w == 1) { lj = q; dy = s->count; }
  else lk = q;
  long long p = s->psi + ((long long)lk * dy + lj) * dx + li;
  T d = div_by_step(diff, A.step[w], A.inv_step[w], A.inv_step64[w], A.fast_div[w]);
  T b = A.coefs[s->coef + q], a = A.coefs[s->coef + s->count + q];
  T old = FIELD == 1 ? A.psi_h_in[p] : A.psi_e[p];
  T psi = b * old + a * d;
  if (own) {
    if (FIELD == 1) A.psi_h_out[p] = psi;
    else A.psi_e[p] = psi;
  }
  T sign = (w == (c + 1) % 3) ? T(1) : T(-1);
  T u = sign * psi;
  if (FIELD == 1) return v - A.dt * u;
  return v + cbv * u;
}

// The fused step over one tile column and a run of planes.
template <typename T>
constexpr size_t plain_smem_bytes() {
  return sizeof(T) * (2 * 3 * RY * RX + 2 * 3 * HY * HX + 3 * TY * TX);
}

template <typename T, bool LOSSY, bool MEDIA>
__global__ void __launch_bounds__(NT) step_kernel(StepArgs<T> A) {
  extern __shared__ __align__(16) unsigned char plain_raw[];
  T(*sE)[3][RY][RX] = reinterpret_cast<T(*)[3][RY][RX]>(plain_raw);
  T(*sH)[3][HY][HX] = reinterpret_cast<T(*)[3][HY][HX]>(plain_raw + sizeof(T) * 2 * 3 * RY * RX);
  T(*sEn)[TY][TX] = reinterpret_cast<T(*)[TY][TX]>(plain_raw + sizeof(T) * (2 * 3 * RY * RX + 2 * 3 * HY * HX));
  const int tid = threadIdx.x;
  const int tile = blockIdx.x;
  const int x0 = (tile % A.tiles_x) * TX, y0 = (tile / A.tiles_x) * TY;
  const int nx = A.n[0], ny = A.n[1], nz = A.n[2];
  const int kbeg = blockIdx.y * A.zchunk;
  const int kend = min(kbeg + A.zchunk, nz);
  if (kbeg >= nz) return;
  const long long N = A.N;

  auto load_e = [&](int buf, int kk) {  // E's plane kk (already wrapped; -1 = beyond a wall)
    for (int q = tid; q < 3 * RY * RX; q += NT) {
      int c = q / (RY * RX), rem = q % (RY * RX);
      int ly = rem / RX, lx = rem % RX;
      int gi = wrap_index(x0 - 1 + lx, nx, A.periodic[0]);
      int gj = wrap_index(y0 - 1 + ly, ny, A.periodic[1]);
      T v = T(0);
      if (gi >= 0 && gj >= 0 && kk >= 0) v = A.e_in[c * N + ((long long)kk * ny + gj) * nx + gi];
      sE[buf][c][ly][lx] = v;
    }
  };

  // H's new plane kk over the region, from E's planes kk (buffer ec) and kk+1 (buffer en):
  // H <- H - dt curl E with forward differences (reference.rs:14-50), then the slabs in axis
  // order (kernel.rs:525-579 takes the slabs along x, then y, then z).
  auto compute_h = [&](int hb, int ec, int en, int kk, bool write) {
    int kn = wrap_index(kk + 1, nz, A.periodic[2]);
    for (int q = tid; q < HY * HX; q += NT) {
      int ly = q / HX, lx = q % HX;  // region cell; E region index (ly, lx) is the same place
      int gi = wrap_index(x0 - 1 + lx, nx, A.periodic[0]);
      int gj = wrap_index(y0 - 1 + ly, ny, A.periodic[1]);
      if (gi < 0 || gj < 0 || x0 - 1 + lx >= nx || y0 - 1 + ly >= ny) {
        sH[hb][0][ly][lx] = sH[hb][1][ly][lx] = sH[hb][2][ly][lx] = T(0);
        continue;
      }
      bool own = write && lx >= 1 && ly >= 1;
      // E at this value, its +x and +y neighbours (plane kk), and +z (plane kk+1); beyond a wall
      // the neighbour is zero (the staged region holds zeros there)
      T ex = sE[ec][0][ly][lx], ey = sE[ec][1][ly][lx], ez = sE[ec][2][ly][lx];
      T ey_xp = sE[ec][1][ly][lx + 1], ez_xp = sE[ec][2][ly][lx + 1];
      T ex_yp = sE[ec][0][ly + 1][lx], ez_yp = sE[ec][2][ly + 1][lx];
      T ex_zp = kn >= 0 ? sE[en][0][ly][lx] : T(0), ey_zp = kn >= 0 ? sE[en][1][ly][lx] : T(0);
      T fx = A.fh[gi], fy = A.fh[nx + gj], fz = A.fh[nx + ny + kk];
      long long r = ((long long)kk * ny + gj) * nx + gi;
      // x: dy(Ez) fy - dz(Ey) fz ; y: dz(Ex) fz - dx(Ez) fx ; z: dx(Ey) fx - dy(Ex) fy
      T dyEz = ez_yp - ez, dzEy = ey_zp - ey, dzEx = ex_zp - ex, dxEz = ez_xp - ez;
      T dxEy = ey_xp - ey, dyEx = ex_yp - ex;
      T hx = A.h_in[r] - A.dt * (dyEz * fy - dzEy * fz);
      T hy = A.h_in[N + r] - A.dt * (dzEx * fz - dxEz * fx);
      T hz = A.h_in[2 * N + r] - A.dt * (dxEy * fx - dyEx * fy);
      const SlabEntry *s;
      // H_x: slabs along y (d/dy of Ez, sign +), then z (d/dz of Ey, sign -)
      if ((s = slab_at(A, 1, 0, 1, gj))) hx = slab_update<T, 1>(A, s, 0, 1, gi, gj, kk, dyEz, hx, T(0), own);
      if ((s = slab_at(A, 1, 0, 2, kk))) hx = slab_update<T, 1>(A, s, 0, 2, gi, gj, kk, dzEy, hx, T(0), own);
      // H_y: slabs along x (d/dx of Ez, sign -), then z (d/dz of Ex, sign +)
      if ((s = slab_at(A, 1, 1, 0, gi))) hy = slab_update<T, 1>(A, s, 1, 0, gi, gj, kk, dxEz, hy, T(0), own);
      if ((s = slab_at(A, 1, 1, 2, kk))) hy = slab_update<T, 1>(A, s, 1, 2, gi, gj, kk, dzEx, hy, T(0), own);
      // H_z: slabs along x (d/dx of Ey, sign +), then y (d/dy of Ex, sign -)
      if ((s = slab_at(A, 1, 2, 0, gi))) hz = slab_update<T, 1>(A, s, 2, 0, gi, gj, kk, dxEy, hz, T(0), own);
      if ((s = slab_at(A, 1, 2, 1, gj))) hz = slab_update<T, 1>(A, s, 2, 1, gi, gj, kk, dyEx, hz, T(0), own);
      sH[hb][0][ly][lx] = hx;
      sH[hb][1][ly][lx] = hy;
      sH[hb][2][ly][lx] = hz;
    }
  };

  // The magnetic currents of plane kk on the region (src/fdtd.rs:1348-1359): each value's
  // entries in CPU order by one thread, H -= dt Re(a w(t)).
  auto inject_h = [&](int hb, int kk) {
    int bucket = tile * nz + kk;
    int g0 = A.hbucket[bucket], g1 = A.hbucket[bucket + 1];
    for (int g = g0 + tid; g < g1; g += NT) {
      Group gr = A.hgroups[g];
      T *v = &sH[hb][gr.comp][0][0] + gr.local;
      for (int q = gr.first; q < gr.first + gr.count; q++) {
        *v = apply_h<T>(*v, A.entries[q], A.waves_h, A.dt);
      }
    }
  };

  int ec = 0, en = 1, hp = 0, hc = 1;
  // Prologue: H's new plane kbeg-1 (wrapped on a periodic z), which E's plane kbeg needs.
  int km = wrap_index(kbeg - 1, nz, A.periodic[2]);
  if (km >= 0) {
    load_e(ec, km);
    load_e(en, kbeg);
    __syncthreads();
    compute_h(hp, ec, en, km, false);
    __syncthreads();
    inject_h(hp, km);
    ec = 1; en = 0;
  } else {
    for (int q = tid; q < 3 * HY * HX; q += NT) (&sH[hp][0][0][0])[q] = T(0);
    load_e(ec, kbeg);
    ec = 0; en = 1;
  }
  __syncthreads();

  for (int k = kbeg; k < kend; k++) {
    load_e(en, wrap_index(k + 1, nz, A.periodic[2]));
    __syncthreads();
    compute_h(hc, ec, en, k, true);
    __syncthreads();
    inject_h(hc, k);
    __syncthreads();
    // H's tile to memory; E's update on the tile (back differences of the new H)
    for (int q = tid; q < TY * TX; q += NT) {
      int ly = q / TX, lx = q % TX;
      int gi = x0 + lx, gj = y0 + ly;
      if (gi >= nx || gj >= ny) continue;
      long long r = ((long long)k * ny + gj) * nx + gi;
      int hy_ = ly + 1, hx_ = lx + 1;  // this value in H's region
      A.h_out[r] = sH[hc][0][hy_][hx_];
      A.h_out[N + r] = sH[hc][1][hy_][hx_];
      A.h_out[2 * N + r] = sH[hc][2][hy_][hx_];
      // back differences: the neighbour before, zero beyond a wall (wrap_index gave -1 there and
      // compute_h stored zeros), and along z the previous plane (zero beyond a wall)
      bool zb = wrap_index(k - 1, nz, A.periodic[2]) >= 0;
      T hxv = sH[hc][0][hy_][hx_], hyv = sH[hc][1][hy_][hx_], hzv = sH[hc][2][hy_][hx_];
      T hz_xm = sH[hc][2][hy_][hx_ - 1], hy_xm = sH[hc][1][hy_][hx_ - 1];
      T hz_ym = sH[hc][2][hy_ - 1][hx_], hx_ym = sH[hc][0][hy_ - 1][hx_];
      T hy_zm = zb ? sH[hp][1][hy_][hx_] : T(0), hx_zm = zb ? sH[hp][0][hy_][hx_] : T(0);
      T fx = A.fe[gi], fy = A.fe[nx + gj], fz = A.fe[nx + ny + k];
      // x: dy(Hz) fy - dz(Hy) fz ; y: dz(Hx) fz - dx(Hz) fx ; z: dx(Hy) fx - dy(Hx) fy
      T dyHz = hzv - hz_ym, dzHy = hyv - hy_zm, dzHx = hxv - hx_zm, dxHz = hzv - hz_xm;
      T dxHy = hyv - hy_xm, dyHx = hxv - hx_ym;
      T curl[3] = {dyHz * fy - dzHy * fz, dzHx * fz - dxHz * fx, dxHy * fx - dyHx * fy};
      T diffs[3][3] = {{T(0), dyHz, dzHy}, {dxHz, T(0), dzHx}, {dxHy, dyHx, T(0)}};
#pragma unroll
      for (int c = 0; c < 3; c++) {
        T eo = sE[ec][c][ly + 1][lx + 1];
        T cbv = A.cb[c * N + r];
        T cav;
        if (LOSSY) cav = A.ca[c * N + r];
        else cav = cbv == T(0) ? T(0) : T(1);
        T v = cav * eo + cbv * curl[c];
        int w0 = (c + 1) % 3, w1 = (c + 2) % 3;
        int wa = min(w0, w1), wb = max(w0, w1);
        int m[3] = {gi, gj, k};
        const SlabEntry *s;
        if ((s = slab_at(A, 0, c, wa, m[wa]))) v = slab_update<T, 0>(A, s, c, wa, gi, gj, k, diffs[c][wa], v, cbv, true);
        if ((s = slab_at(A, 0, c, wb, m[wb]))) v = slab_update<T, 0>(A, s, c, wb, gi, gj, k, diffs[c][wb], v, cbv, true);
        sEn[c][ly][lx] = v;
      }
    }
    __syncthreads();
    // The electric currents (src/fdtd.rs:1375-1387): E -= cb Re(a w(t + dt/2)).
    {
      int bucket = tile * nz + k;
      int g0 = A.ebucket[bucket], g1 = A.ebucket[bucket + 1];
      for (int g = g0 + tid; g < g1; g += NT) {
        Group gr = A.egroups[g];
        int ly = gr.local / TX, lx = gr.local % TX;
        long long r = ((long long)k * ny + (y0 + ly)) * nx + (x0 + lx);
        T cbv = A.cb[gr.comp * N + r];
        T *v = &sEn[gr.comp][ly][lx];
        for (int q = gr.first; q < gr.first + gr.count; q++) {
          *v = apply_e<T>(*v, A.entries[q], A.waves_e, cbv);
        }
      }
    }
    __syncthreads();
    for (int q = tid; q < TY * TX; q += NT) {
      int ly = q / TX, lx = q % TX;
      int gi = x0 + lx, gj = y0 + ly;
      if (gi >= nx || gj >= ny) continue;
      long long r = ((long long)k * ny + gj) * nx + gi;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        T v = sEn[c][ly][lx];
        if (MEDIA) {
          // Media::update (src/fdtd/media.rs:670-705): the rest of E's update, then the currents
          int mi = A.media.member[c * N + r];
          if (mi >= 0) {
            const MediaArgs<T> &M = A.media;
            int g = M.group[mi];
            int np = M.gpoles[g];
            T before = M.before[mi];
            T rest = M.gchi[g] * before;
            const T *pl = M.gpole + (long long)g * M.maxpoles * 3;
            T *cur = M.current + (long long)mi * M.maxpoles;
            T *prev = M.previous + (long long)mi * M.maxpoles;
            for (int p = 0; p < np; p++)
              rest = rest - T(0.5) * ((pl[3 * p] + T(1)) * cur[p] + pl[3 * p + 1] * prev[p]);
            T next = v + M.scale[mi] * rest;
            T slope = (next - before) / M.two_dt;
            for (int p = 0; p < np; p++) {
              T jn = pl[3 * p] * cur[p] + pl[3 * p + 1] * prev[p] + pl[3 * p + 2] * slope;
              prev[p] = cur[p];
              cur[p] = jn;
            }
            M.before[mi] = sE[ec][c][ly + 1][lx + 1];  // E^n, saved before the update
            v = next;
          }
        }
        A.e_out[c * N + r] = v;
      }
    }
    // this plane's E becomes the staged "plane k" of the next step; H's new plane becomes k-1
    int t = ec; ec = en; en = t;
    t = hp; hp = hc; hc = t;
    __syncthreads();
  }
}


// ------------------------------------------------------------------------------------------
// The staged step (v1). The same arithmetic as step_kernel, with each plane's inputs brought into
// shared memory ahead of use by cp.async in 16-byte chunks: E's plane k+1 over the tile and the
// rows and columns around it, H's plane k over its region, cb's plane k over the tile. A ring of
// STAGES plane-buffers keeps DEPTH = STAGES - 2 planes in flight while the CTA computes plane k
// from buffers k and k-1. Needs nx a multiple of 16 bytes' worth of values (4 in f32, 2 in f64),
// so a chunk never straddles the grid's edge: a chunk beyond a wall is zero-filled (src-size 0)
// and one across a periodic side is read from the wrapped place.
//
// Work: the grid's (tile, plane) pairs in tile-major order, split evenly over the resident CTAs;
// a CTA's share is one or a few runs of consecutive planes of a tile, each started by the
// prologue that recomputes H's plane before its first.

__device__ inline void cp_async16(void *smem, const void *gmem, bool valid) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n)
               : "memory");
}
__device__ inline void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// One value (4 or 8 bytes) copied from global to shared memory without waiting.
template <typename T>
__device__ inline void cp_async_value(T *smem, const T *gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem),
               "n"((int)sizeof(T))
               : "memory");
}
// Brings `bytes` (a multiple of 16, from a 16-byte aligned address) of global memory into L2
// ahead of use, without waiting and without registers.
__device__ inline void prefetch_l2(const void *gmem, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(gmem), "r"(bytes) : "memory");
}
template <int N>
__device__ inline void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
// A named barrier (id 1..15; 0 is __syncthreads') of `threads` threads, whole warps: arrive
// without waiting (the shared-memory writes before it are seen by the threads that sync on it),
// or wait for the count.
__device__ inline void named_arrive(int id, int threads) {
  asm volatile("bar.arrive %0, %1;\n" ::"r"(id), "r"(threads) : "memory");
}
__device__ inline void named_sync(int id, int threads) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(threads) : "memory");
}

template <typename T>
struct Stage {
  static constexpr int CH = 16 / (int)sizeof(T);  // values per 16-byte chunk
  static constexpr int EW = TX + 2 * CH;          // E region: x0-CH .. x0+TX+CH-1
  static constexpr int EH = TY + 2;               //           y0-1 .. y0+TY
  static constexpr int HW = TX + CH;              // H region: x0-CH .. x0+TX-1
  static constexpr int HH = TY + 1;               //           y0-1 .. y0+TY-1
  static constexpr int E_VALS = 3 * EH * EW;
  static constexpr int H_VALS = 3 * HH * HW;
  static constexpr int B_VALS = 3 * TY * TX;
  static constexpr int VALS = E_VALS + H_VALS + B_VALS;
  static constexpr int E_CHUNKS = E_VALS / CH, H_CHUNKS = H_VALS / CH, B_CHUNKS = B_VALS / CH;
  static constexpr int NEW_VALS = 3 * HH * (TX + 1);  // H's new plane over (x0-1.., y0-1..)
};

template <typename T, int STAGES>
constexpr size_t staged_smem_bytes() {
  return sizeof(T) * ((size_t)STAGES * Stage<T>::VALS + Stage<T>::NEW_VALS);
}

// Issues the copies of one stage: E's plane `ke` (the region), H's and cb's plane `kh`; a plane
// of -1 is beyond a wall (zeros). `parts`: 1 E only, 3 everything.
template <typename T>
__device__ inline void issue_stage(const StepArgs<T> &A, T *buf, int x0, int y0, int ke, int kh,
                                   int parts) {
  using S = Stage<T>;
  const int nx = A.n[0], ny = A.n[1];
  const long long N = A.N;
  const int tid = threadIdx.x;
  const T *dummy = A.e_in;
  for (int q = tid; q < S::E_CHUNKS; q += NT) {
    int c = q / (S::EH * (S::EW / S::CH)), rem = q % (S::EH * (S::EW / S::CH));
    int ry = rem / (S::EW / S::CH), cx = rem % (S::EW / S::CH);
    int gx = x0 - S::CH + cx * S::CH;
    int gy = wrap_index(y0 - 1 + ry, ny, A.periodic[1]);
    if (gx < 0) gx = A.periodic[0] ? gx + nx : -1;
    else if (gx >= nx) gx = (A.periodic[0] && gx == nx) ? 0 : -1;
    bool ok = gx >= 0 && gy >= 0 && ke >= 0;
    const T *src = ok ? A.e_in + c * N + ((long long)ke * ny + gy) * nx + gx : dummy;
    cp_async16(buf + (size_t)q * S::CH, src, ok);
  }
  if (parts & 2) {
    T *hb = buf + S::E_VALS;
    for (int q = tid; q < S::H_CHUNKS; q += NT) {
      int c = q / (S::HH * (S::HW / S::CH)), rem = q % (S::HH * (S::HW / S::CH));
      int ry = rem / (S::HW / S::CH), cx = rem % (S::HW / S::CH);
      int gx = x0 - S::CH + cx * S::CH;
      int gy = wrap_index(y0 - 1 + ry, ny, A.periodic[1]);
      if (gx < 0) gx = A.periodic[0] ? gx + nx : -1;
      else if (gx >= nx) gx = -1;
      bool ok = gx >= 0 && gy >= 0 && kh >= 0;
      const T *src = ok ? A.h_in + c * N + ((long long)kh * ny + gy) * nx + gx : dummy;
      cp_async16(hb + (size_t)q * S::CH, src, ok);
    }
    T *bb = hb + S::H_VALS;
    for (int q = tid; q < S::B_CHUNKS; q += NT) {
      int c = q / (TY * (TX / S::CH)), rem = q % (TY * (TX / S::CH));
      int ry = rem / (TX / S::CH), cx = rem % (TX / S::CH);
      int gx = x0 + cx * S::CH, gy = y0 + ry;
      bool ok = gx < nx && gy < ny && kh >= 0;
      const T *src = ok ? A.cb + c * N + ((long long)kh * ny + gy) * nx + gx : dummy;
      cp_async16(bb + (size_t)q * S::CH, src, ok);
    }
  }
}

template <typename T, bool LOSSY, bool MEDIA, int STAGES>
__global__ void __launch_bounds__(NT) staged_kernel(StepArgs<T> A, long long total, int ctas) {
  using S = Stage<T>;
  constexpr int DEPTH = STAGES - 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *stages = reinterpret_cast<T *>(smem_raw);
  T *sHn = stages + (size_t)STAGES * S::VALS;  // [3][HH][TX+1]
  T *sEn = sHn;  // [3][TY][TX]: E's new plane while sources add to it, once H's is read
  const int tid = threadIdx.x;
  const int nx = A.n[0], ny = A.n[1], nz = A.n[2];
  const long long N = A.N;
  const long long begin = total * blockIdx.x / ctas, end = total * (blockIdx.x + 1) / ctas;
  auto E = [&](int b, int c, int y, int x) -> T & {  // E region of buffer b
    return stages[(size_t)b * S::VALS + ((size_t)c * S::EH + y) * S::EW + x];
  };
  auto Hold = [&](int b, int c, int y, int x) -> T & {
    return stages[(size_t)b * S::VALS + S::E_VALS + ((size_t)c * S::HH + y) * S::HW + x];
  };
  auto CB = [&](int b, int c, int y, int x) -> T & {
    return stages[(size_t)b * S::VALS + S::E_VALS + S::H_VALS + ((size_t)c * TY + y) * TX + x];
  };
  auto Hn = [&](int c, int y, int x) -> T & { return sHn[((size_t)c * S::HH + y) * (TX + 1) + x]; };

  for (long long at = begin; at < end;) {
    const int tile = (int)(at / nz);
    const int k0 = (int)(at % nz);
    const int k1 = (int)min((long long)nz, (long long)k0 + (end - at));
    at += k1 - k0;
    const int x0 = (tile % A.tiles_x) * TX, y0 = (tile / A.tiles_x) * TY;
    const int km = wrap_index(k0 - 1, nz, A.periodic[2]);
    // positions: 0 E(km) (when km exists), 1 stage k0-1, 2 + (k - k0) stage k
    const int last = 2 + (k1 - 1 - k0);
    auto issue = [&](int pos) {
      if (pos <= last) {
        T *buf = stages + (size_t)(pos % STAGES) * S::VALS;
        if (pos == 0) {
          if (km >= 0) issue_stage(A, buf, x0, y0, km, -1, 1);
        } else {
          int k = k0 - 2 + pos;  // the stage's plane: E's region of k+1, H's and cb's k
          int kh = pos == 1 ? km : k;
          issue_stage(A, buf, x0, y0, wrap_index(k + 1, nz, A.periodic[2]), kh, 3);
        }
      }
      cp_async_commit();
    };
    for (int pos = 0; pos < 1 + DEPTH; pos++) issue(pos);
    // -- prologue: H's new plane km over the region, from E(km) (position 0) and stage 1
    T hprev[2][2];  // H_x and H_y of plane k-1 at this thread's two E values
    cp_async_wait<DEPTH - 1>();  // positions 0 and 1 landed
    __syncthreads();
    issue(1 + DEPTH);  // into a buffer not used yet
    // entering iteration p (= 2 + k - k0) the copies up to p + DEPTH - 1 have been issued
    auto compute_h = [&](int bc, int bn, int bp, int kk, bool write) {
      // bc: buffer holding E(kk) (as its E region), bn: buffer with E(kk+1) and H(kk)
      const bool zslab = !A.periodic[2] && (kk < A.low[2] || kk >= nz - A.high[2]);
      for (int q = tid; q < S::HH * (TX + 1); q += NT) {
        int ly = q / (TX + 1), lx = q % (TX + 1);
        int gxr = x0 - 1 + lx, gyr = y0 - 1 + ly;
        int gi = wrap_index(gxr, nx, A.periodic[0]), gj = wrap_index(gyr, ny, A.periodic[1]);
        if (gi < 0 || gj < 0 || gxr >= nx || gyr >= ny) {
          Hn(0, ly, lx) = Hn(1, ly, lx) = Hn(2, ly, lx) = T(0);
          continue;
        }
        bool own = write && lx >= 1 && ly >= 1;
        int ex = lx - 1 + S::CH;  // this place in the E region
        T ex0 = E(bc, 0, ly, ex), ey0 = E(bc, 1, ly, ex), ez0 = E(bc, 2, ly, ex);
        T dyEz = E(bc, 2, ly + 1, ex) - ez0, dxEz = E(bc, 2, ly, ex + 1) - ez0;
        T dxEy = E(bc, 1, ly, ex + 1) - ey0, dyEx = E(bc, 0, ly + 1, ex) - ex0;
        T dzEy = E(bn, 1, ly, ex) - ey0, dzEx = E(bn, 0, ly, ex) - ex0;
        T fx = A.fh[gi], fy = A.fh[nx + gj], fz = A.fh[nx + ny + kk];
        int hx_ = lx - 1 + S::CH;
        T hx = Hold(bn, 0, ly, hx_) - A.dt * (dyEz * fy - dzEy * fz);
        T hy = Hold(bn, 1, ly, hx_) - A.dt * (dzEx * fz - dxEz * fx);
        T hz = Hold(bn, 2, ly, hx_) - A.dt * (dxEy * fx - dyEx * fy);
        const SlabEntry *sl;
        if ((sl = slab_at(A, 1, 0, 1, gj))) hx = slab_update<T, 1>(A, sl, 0, 1, gi, gj, kk, dyEz, hx, T(0), own);
        if (zslab && (sl = slab_at(A, 1, 0, 2, kk))) hx = slab_update<T, 1>(A, sl, 0, 2, gi, gj, kk, dzEy, hx, T(0), own);
        if ((sl = slab_at(A, 1, 1, 0, gi))) hy = slab_update<T, 1>(A, sl, 1, 0, gi, gj, kk, dxEz, hy, T(0), own);
        if (zslab && (sl = slab_at(A, 1, 1, 2, kk))) hy = slab_update<T, 1>(A, sl, 1, 2, gi, gj, kk, dzEx, hy, T(0), own);
        if ((sl = slab_at(A, 1, 2, 0, gi))) hz = slab_update<T, 1>(A, sl, 2, 0, gi, gj, kk, dxEy, hz, T(0), own);
        if ((sl = slab_at(A, 1, 2, 1, gj))) hz = slab_update<T, 1>(A, sl, 2, 1, gi, gj, kk, dyEx, hz, T(0), own);
        Hn(0, ly, lx) = hx;
        Hn(1, ly, lx) = hy;
        Hn(2, ly, lx) = hz;
      }
      (void)bp;
    };
    auto inject_h = [&](int kk) {  // uniform: only CTAs whose bucket holds sources sync here
      int bucket = tile * nz + kk;
      int g0 = A.hbucket[bucket], g1 = A.hbucket[bucket + 1];
      if (g1 > g0) {
        __syncthreads();
        for (int g = g0 + tid; g < g1; g += NT) {
          Group gr = A.hgroups[g];
          T *v = &sHn[(size_t)gr.comp * S::HH * (TX + 1) + gr.local];
          for (int q = gr.first; q < gr.first + gr.count; q++) {
            *v = apply_h<T>(*v, A.entries[q], A.waves_h, A.dt);
          }
        }
      }
    };
    if (km >= 0) {
      compute_h(0 % STAGES, 1 % STAGES, 0, km, false);
      inject_h(km);
      __syncthreads();
      for (int r = 0; r < 2; r++) {
        int q = tid + r * NT;
        int ey = q / TX, ex = q % TX;
        hprev[r][0] = Hn(0, ey + 1, ex + 1);
        hprev[r][1] = Hn(1, ey + 1, ex + 1);
      }
    } else {
      hprev[0][0] = hprev[0][1] = hprev[1][0] = hprev[1][1] = T(0);
    }
    for (int k = k0; k < k1; k++) {
      const int pos = 2 + (k - k0);
      cp_async_wait<DEPTH - 1>();
      __syncthreads();  // stage pos landed for every thread; everyone is done with plane k-1
      issue(pos + DEPTH);
      const int bc = (pos - 1) % STAGES, bn = pos % STAGES;
      compute_h(bc, bn, 0, k, true);
      inject_h(k);
      __syncthreads();
      // E's new plane k on the tile, two values a thread
      const int ebucket = tile * nz + k;
      const int eg0 = A.ebucket[ebucket], eg1 = A.ebucket[ebucket + 1];
      const bool zslab = !A.periodic[2] && (k < A.low[2] || k >= nz - A.high[2]);
      T enew[2][3];
#pragma unroll
      for (int r = 0; r < 2; r++) {
        int q = tid + r * NT;
        int ey = q / TX, ex = q % TX;
        int gi = x0 + ex, gj = y0 + ey;
        bool valid = gi < nx && gj < ny;
        T hxv = Hn(0, ey + 1, ex + 1), hyv = Hn(1, ey + 1, ex + 1), hzv = Hn(2, ey + 1, ex + 1);
        if (valid) {
          long long r0 = ((long long)k * ny + gj) * nx + gi;
          A.h_out[r0] = hxv;
          A.h_out[N + r0] = hyv;
          A.h_out[2 * N + r0] = hzv;
          bool zb = wrap_index(k - 1, nz, A.periodic[2]) >= 0;
          T hz_xm = Hn(2, ey + 1, ex), hy_xm = Hn(1, ey + 1, ex);
          T hz_ym = Hn(2, ey, ex + 1), hx_ym = Hn(0, ey, ex + 1);
          T hy_zm = zb ? hprev[r][1] : T(0), hx_zm = zb ? hprev[r][0] : T(0);
          T fx = A.fe[gi], fy = A.fe[nx + gj], fz = A.fe[nx + ny + k];
          T dyHz = hzv - hz_ym, dzHy = hyv - hy_zm, dzHx = hxv - hx_zm, dxHz = hzv - hz_xm;
          T dxHy = hyv - hy_xm, dyHx = hxv - hx_ym;
          T curl[3] = {dyHz * fy - dzHy * fz, dzHx * fz - dxHz * fx, dxHy * fx - dyHx * fy};
          T diffs[3][3] = {{T(0), dyHz, dzHy}, {dxHz, T(0), dzHx}, {dxHy, dyHx, T(0)}};
#pragma unroll
          for (int c = 0; c < 3; c++) {
            T eo = E(bc, c, ey + 1, ex + S::CH);
            T cbv = CB(bn, c, ey, ex);
            T cav;
            if (LOSSY) cav = A.ca[c * N + r0];
            else cav = cbv == T(0) ? T(0) : T(1);
            T v = cav * eo + cbv * curl[c];
            int w0 = (c + 1) % 3, w1 = (c + 2) % 3;
            int wa = min(w0, w1), wb = max(w0, w1);
            int m[3] = {gi, gj, k};
            const SlabEntry *sl;
            if ((wa != 2 || zslab) && (sl = slab_at(A, 0, c, wa, m[wa]))) v = slab_update<T, 0>(A, sl, c, wa, gi, gj, k, diffs[c][wa], v, cbv, true);
            if ((wb != 2 || zslab) && (sl = slab_at(A, 0, c, wb, m[wb]))) v = slab_update<T, 0>(A, sl, c, wb, gi, gj, k, diffs[c][wb], v, cbv, true);
            enew[r][c] = v;
          }
        }
        hprev[r][0] = hxv;
        hprev[r][1] = hyv;
      }
      if (eg1 > eg0) {  // electric currents on this tile and plane: through shared memory
        __syncthreads();  // every thread has read H's new plane
#pragma unroll
        for (int r = 0; r < 2; r++) {
          int q = tid + r * NT;
#pragma unroll
          for (int c = 0; c < 3; c++) sEn[(size_t)c * TY * TX + q] = enew[r][c];
        }
        __syncthreads();
        for (int g = eg0 + tid; g < eg1; g += NT) {
          Group gr = A.egroups[g];
          int ey = gr.local / TX, ex = gr.local % TX;
          long long r0 = ((long long)k * ny + (y0 + ey)) * nx + (x0 + ex);
          T cbv = A.cb[gr.comp * N + r0];
          T *v = &sEn[(size_t)gr.comp * TY * TX + gr.local];
          for (int q = gr.first; q < gr.first + gr.count; q++) {
            *v = apply_e<T>(*v, A.entries[q], A.waves_e, cbv);
          }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < 2; r++) {
          int q = tid + r * NT;
#pragma unroll
          for (int c = 0; c < 3; c++) enew[r][c] = sEn[(size_t)c * TY * TX + q];
        }
      }
#pragma unroll
      for (int r = 0; r < 2; r++) {
        int q = tid + r * NT;
        int ey = q / TX, ex = q % TX;
        int gi = x0 + ex, gj = y0 + ey;
        if (gi >= nx || gj >= ny) continue;
        long long r0 = ((long long)k * ny + gj) * nx + gi;
#pragma unroll
        for (int c = 0; c < 3; c++) {
          T v = enew[r][c];
          if (MEDIA) {
            int mi = A.media.member[c * N + r0];
            if (mi >= 0) {
              const MediaArgs<T> &M = A.media;
              int g = M.group[mi];
              int np = M.gpoles[g];
              T before = M.before[mi];
              T rest = M.gchi[g] * before;
              const T *pl = M.gpole + (long long)g * M.maxpoles * 3;
              T *cur = M.current + (long long)mi * M.maxpoles;
              T *prev = M.previous + (long long)mi * M.maxpoles;
              for (int p = 0; p < np; p++)
                rest = rest - T(0.5) * ((pl[3 * p] + T(1)) * cur[p] + pl[3 * p + 1] * prev[p]);
              T next = v + M.scale[mi] * rest;
              T slope = (next - before) / M.two_dt;
              for (int p = 0; p < np; p++) {
                T jn = pl[3 * p] * cur[p] + pl[3 * p + 1] * prev[p] + pl[3 * p + 2] * slope;
                prev[p] = cur[p];
                cur[p] = jn;
              }
              M.before[mi] = E(bc, c, ey + 1, ex + S::CH);
              v = next;
            }
          }
          A.e_out[c * N + r0] = v;
        }
      }
    }
    cp_async_wait<0>();
    __syncthreads();  // the next run of planes reuses the buffers
  }
}


// ------------------------------------------------------------------------------------------
// The row step (v2). A CTA owns OWN = 63 values along x and RW rows along y of every plane in a
// run of planes, and marches up z. Warp w holds row y0 - 1 + w (warp 0 the row before the tile,
// whose new H the first row's E needs); lane l holds the values x0 - 1 + l and x0 + 31 + l of
// its row, 64 H values, so each warp recomputes only one H value per row that its neighbour
// along x owns. Neighbours along x come by warp shuffles, along y through a small exchange in
// shared memory, along z from the registers of the previous plane. Each plane's inputs for the
// next plane are loaded into registers one plane ahead. The arithmetic of every value is
// step_kernel's, operation for operation.
namespace rowstep {
constexpr int SEG = 64;       // H values a warp row holds
constexpr int OWN = SEG - 1;  // values a tile owns along x
constexpr int RW = 7;         // rows a tile owns along y
constexpr int WARPS = RW + 1;
constexpr int THREADS = 32 * WARPS;
}  // namespace rowstep

// The CPML share of one value along axis w whose index is m there; `s` the slab holding it.
template <typename T, int FIELD>
__device__ __forceinline__ T slab_apply(const StepArgs<T> &A, const SlabEntry s, int c, int w,
                                        int i, int j, int k, T diff, T v, T cbv, bool own) {
  int m = w == 0 ? i : (w == 1 ? j : k);
  int q = m - s.from;
  int li = i, lj = j, lk = k;
  int dx = A.n[0], dy = A.n[1];
  if (w == 0) { li = i - s.pf; dx = s.pw; }
  else if (w == 1) { lj = q; dy = s.count; }
  else lk = q;
  long long p = s.psi + ((long long)lk * dy + lj) * dx + li;
  T d = div_by_step(diff, A.step[w], A.inv_step[w], A.inv_step64[w], A.fast_div[w]);
  T b = A.coefs[s.coef + q], a = A.coefs[s.coef + s.count + q];
  T old = FIELD == 1 ? A.psi_h_in[p] : A.psi_e[p];
  T psi = b * old + a * d;
  if (own) {
    if (FIELD == 1) A.psi_h_out[p] = psi;
    else A.psi_e[p] = psi;
  }
  T sign = (w == (c + 1) % 3) ? T(1) : T(-1);
  T u = sign * psi;
  if (FIELD == 1) return v - A.dt * u;
  return v + cbv * u;
}
// The slab of `field`'s component c along axis w on `side` (0 low, 1 high), from the table.
template <typename T>
__device__ __forceinline__ SlabEntry slab_of(const StepArgs<T> &A, int field, int c, int w, int side) {
  return A.slab[field][c][w][side];
}
// The slab along z holding plane k for component c of `field`, or count 0.
template <typename T>
__device__ __forceinline__ SlabEntry zslab_of(const StepArgs<T> &A, int field, int c, int k) {
  SlabEntry none;
  none.count = 0;
  none.from = 0;
  none.psi = 0;
  none.coef = 0;
  if (A.periodic[2]) return none;
  if (k < A.low[2]) return A.slab[field][c][2][0];
  if (k >= A.n[2] - A.high[2]) return A.slab[field][c][2][1];
  return none;
}

template <typename T, bool LOSSY, bool MEDIA>
__global__ void __launch_bounds__(rowstep::THREADS, 2) row_kernel(StepArgs<T> A) {
  using namespace rowstep;
  __shared__ T sE[2][WARPS][SEG];  // E_x, E_z of plane k, each warp's row (for the row above)
  __shared__ T sH[2][WARPS][SEG];  // H_x, H_z of plane k (for the row below)
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nx = A.n[0], ny = A.n[1], nz = A.n[2];
  const long long N = A.N;
  const int tile = blockIdx.x;
  const int x0 = (tile % A.tiles_x) * OWN, y0 = (tile / A.tiles_x) * RW;
  const int kbeg = blockIdx.y * A.zchunk, kend = min(kbeg + A.zchunk, nz);
  if (kbeg >= nz) return;
  const int tileidx = tile;

  // -- per lane: the two x places; per warp: the row
  int gx[2], mx[2], mxp[2];
  bool hval[2], own[2], ev[2];
  const int gy = y0 - 1 + w;
  const int my = wrap_index(gy, ny, A.periodic[1]);
  const int myp = wrap_index(gy + 1, ny, A.periodic[1]);  // the row after (for +y at the last warp)
  const bool rowok = my >= 0 && gy < ny;  // this row's H is computed
  const bool rowe = my >= 0;                // this row's E is read (a wrapped row included)
  T fhx[2], fex[2];
  int sx[2];  // the CPML side along x at each place (0 low, 1 high, -1 none)
#pragma unroll
  for (int h = 0; h < 2; h++) {
    gx[h] = x0 - 1 + lane + 32 * h;
    mx[h] = wrap_index(gx[h], nx, A.periodic[0]);
    mxp[h] = wrap_index(gx[h] + 1, nx, A.periodic[0]);
    hval[h] = rowok && mx[h] >= 0 && gx[h] < nx;
    ev[h] = rowe && mx[h] >= 0;
    own[h] = hval[h] && w >= 1 && (lane + 32 * h) >= 1 && gx[h] < nx;
    fhx[h] = mx[h] >= 0 ? A.fh[mx[h]] : T(0);
    fex[h] = mx[h] >= 0 ? A.fe[mx[h]] : T(0);
    sx[h] = -1;
    if (mx[h] >= 0 && !A.periodic[0]) {
      if (mx[h] < A.low[0]) sx[h] = 0;
      else if (mx[h] >= nx - A.high[0]) sx[h] = 1;
    }
  }
  const T fhy = my >= 0 ? A.fh[nx + my] : T(0), fey = my >= 0 ? A.fe[nx + my] : T(0);
  int sy = -1;  // the CPML side along y of this row
  if (my >= 0 && !A.periodic[1]) {
    if (my < A.low[1]) sy = 0;
    else if (my >= ny - A.high[1]) sy = 1;
  }
  // the value after the warp's 64 along x (E_y, E_z of plane k there) for the last lane
  const int gxe = x0 + OWN, mxe = wrap_index(gxe, nx, A.periodic[0]);
  long long rowoff = my >= 0 ? (long long)my * nx : 0;
  long long rowoffp = myp >= 0 ? (long long)myp * nx : 0;

  // -- one plane's inputs: E(k+1) at the H places, H(k) there, cb(k) at the owned places, and
  // E(k)'s values past the warp's row ends: x after the last lane (E_y, E_z), and for the last
  // warp the row after (E_x, E_z)
  struct Plane {
    T e1[3][2], hold[3][2], cb[3][2], ca[3][2];
    T xe[2];      // E_y, E_z(k) at x0 + 63
    T ye[2][2];   // E_x, E_z(k) at row gy + 1 (last warp), per half
  };
  auto load = [&](Plane &P, int k) {
    const int k1 = wrap_index(k + 1, nz, A.periodic[2]);
    const long long pk = (long long)k * ny * nx, pk1 = (long long)k1 * ny * nx;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      long long at = pk + rowoff + mx[h], at1 = pk1 + rowoff + mx[h];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        P.e1[c][h] = (ev[h] && k1 >= 0) ? A.e_in[c * N + at1] : T(0);
        P.hold[c][h] = hval[h] ? A.h_in[c * N + at] : T(0);
        P.cb[c][h] = own[h] ? A.cb[c * N + at] : T(0);
        if (LOSSY) P.ca[c][h] = own[h] ? A.ca[c * N + at] : T(0);
      }
      if (w == WARPS - 1) {
        bool ok = myp >= 0 && mx[h] >= 0;
        long long atp = pk + rowoffp + mx[h];
        P.ye[0][h] = ok ? A.e_in[atp] : T(0);
        P.ye[1][h] = ok ? A.e_in[2 * N + atp] : T(0);
      }
    }
    bool okx = rowe && mxe >= 0;
    long long atx = pk + rowoff + (mxe >= 0 ? mxe : 0);
    P.xe[0] = okx ? A.e_in[N + atx] : T(0);
    P.xe[1] = okx ? A.e_in[2 * N + atx] : T(0);
  };
  auto e_now = [&](T ek[3][2], int k) {  // E(k) at the H places
    const long long pk = (long long)k * ny * nx;
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
      for (int c = 0; c < 3; c++) ek[c][h] = ev[h] ? A.e_in[c * N + pk + rowoff + mx[h]] : T(0);
  };

  // H's new plane k at the H places (reference.rs:14-50, then the slabs x, y, z)
  auto compute_h = [&](const Plane &P, const T ek[3][2], int k, bool write, T hn[3][2]) {
    // E(k) of the row after: the next warp's row, or the loaded row for the last warp
    sE[0][w][lane] = ek[0][0];
    sE[0][w][lane + 32] = ek[0][1];
    sE[1][w][lane] = ek[2][0];
    sE[1][w][lane + 32] = ek[2][1];
    __syncthreads();
    const T fhz = A.fh[nx + ny + k];
    const bool zs = !A.periodic[2] && (k < A.low[2] || k >= nz - A.high[2]);
#pragma unroll
    for (int h = 0; h < 2; h++) {
      // +x: the next lane's value; lane 31 of the first half takes lane 0 of the second, lane 31
      // of the second the value after the row
      T ey_n = __shfl_down_sync(0xffffffffu, ek[1][h], 1);
      T ez_n = __shfl_down_sync(0xffffffffu, ek[2][h], 1);
      T ey_o = __shfl_sync(0xffffffffu, ek[1][1 - h], 0);
      T ez_o = __shfl_sync(0xffffffffu, ek[2][1 - h], 0);
      if (lane == 31) {
        ey_n = h == 0 ? ey_o : P.xe[0];
        ez_n = h == 0 ? ez_o : P.xe[1];
      }
      // a neighbour beyond a wall is zero: the place after x = nx - 1 (mxp < 0)
      if (mxp[h] < 0) ey_n = ez_n = T(0);
      T ex_yn, ez_yn;
      if (w < WARPS - 1) {
        ex_yn = sE[0][w + 1][lane + 32 * h];
        ez_yn = sE[1][w + 1][lane + 32 * h];
      } else {
        ex_yn = P.ye[0][h];
        ez_yn = P.ye[1][h];
      }
      if (myp < 0) ex_yn = ez_yn = T(0);
      T dyEz = ez_yn - ek[2][h], dzEy = P.e1[1][h] - ek[1][h];
      T dzEx = P.e1[0][h] - ek[0][h], dxEz = ez_n - ek[2][h];
      T dxEy = ey_n - ek[1][h], dyEx = ex_yn - ek[0][h];
      T hx = P.hold[0][h] - A.dt * (dyEz * fhy - dzEy * fhz);
      T hy = P.hold[1][h] - A.dt * (dzEx * fhz - dxEz * fhx[h]);
      T hz = P.hold[2][h] - A.dt * (dxEy * fhx[h] - dyEx * fhy);
      if (hval[h]) {
        const bool ow = write && own[h];
        const int i = mx[h], j = my;
        if ((sx[h] >= 0) | (sy >= 0) | zs) {
          // H_x: y then z; H_y: x then z; H_z: x then y (the table's entry has count 0 where a
          // side has no CPML)
          if (sy >= 0) {
            SlabEntry e = slab_of(A, 1, 0, 1, sy);
            if (e.count) hx = slab_apply<T, 1>(A, e, 0, 1, i, j, k, dyEz, hx, T(0), ow);
          }
          if (zs) {
            SlabEntry z0 = zslab_of(A, 1, 0, k);
            if (z0.count) hx = slab_apply<T, 1>(A, z0, 0, 2, i, j, k, dzEy, hx, T(0), ow);
          }
          if (sx[h] >= 0) {
            SlabEntry e = slab_of(A, 1, 1, 0, sx[h]);
            if (e.count) hy = slab_apply<T, 1>(A, e, 1, 0, i, j, k, dxEz, hy, T(0), ow);
          }
          if (zs) {
            SlabEntry z1 = zslab_of(A, 1, 1, k);
            if (z1.count) hy = slab_apply<T, 1>(A, z1, 1, 2, i, j, k, dzEx, hy, T(0), ow);
          }
          if (sx[h] >= 0) {
            SlabEntry e = slab_of(A, 1, 2, 0, sx[h]);
            if (e.count) hz = slab_apply<T, 1>(A, e, 2, 0, i, j, k, dxEy, hz, T(0), ow);
          }
          if (sy >= 0) {
            SlabEntry e = slab_of(A, 1, 2, 1, sy);
            if (e.count) hz = slab_apply<T, 1>(A, e, 2, 1, i, j, k, dyEx, hz, T(0), ow);
          }
        }
      } else {
        hx = hy = hz = T(0);
      }
      hn[0][h] = hx;
      hn[1][h] = hy;
      hn[2][h] = hz;
    }
    // the magnetic currents at this tile and plane, each value's entries in CPU order
    const int bucket = tileidx * nz + k;
    const int g0 = A.hbucket[bucket], g1 = A.hbucket[bucket + 1];
    for (int g = g0; g < g1; g++) {
      Group gr = A.hgroups[g];
      int gw = gr.local / SEG, gi = gr.local % SEG;
      if (gw == w && (gi & 31) == lane) {
        const bool second = (gi >> 5) != 0;
        T v = T(0);
#pragma unroll
        for (int c = 0; c < 3; c++)
          if (gr.comp == c) v = second ? hn[c][1] : hn[c][0];
        for (int q = gr.first; q < gr.first + gr.count; q++) {
          v = apply_h<T>(v, A.entries[q], A.waves_h, A.dt);
        }
#pragma unroll
        for (int c = 0; c < 3; c++)
          if (gr.comp == c) {
            if (second) hn[c][1] = v;
            else hn[c][0] = v;
          }
      }
    }
  };

  T ek[3][2], hprev[2][2], hn[3][2];
  Plane P0, P1;
  // prologue: H's new plane kbeg-1 (wrapped on a periodic z), which E's plane kbeg needs
  const int km = wrap_index(kbeg - 1, nz, A.periodic[2]);
  if (km >= 0) {
    e_now(ek, km);
    load(P0, km);
    compute_h(P0, ek, km, false, hn);
    hprev[0][0] = hn[0][0]; hprev[0][1] = hn[0][1];
    hprev[1][0] = hn[1][0]; hprev[1][1] = hn[1][1];
    __syncthreads();
  } else {
    hprev[0][0] = hprev[0][1] = hprev[1][0] = hprev[1][1] = T(0);
  }
  e_now(ek, kbeg);
  load(P0, kbeg);
  auto plane = [&](Plane &P, Plane &Q, int k) {
    if (k + 1 < kend) load(Q, k + 1);
    compute_h(P, ek, k, true, hn);
    // H's tile to memory, and H_x, H_z to the row below
    const long long pk = (long long)k * ny * nx;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      if (own[h]) {
        long long at = pk + rowoff + mx[h];
        A.h_out[at] = hn[0][h];
        A.h_out[N + at] = hn[1][h];
        A.h_out[2 * N + at] = hn[2][h];
      }
    }
    sH[0][w][lane] = hn[0][0];
    sH[0][w][lane + 32] = hn[0][1];
    sH[1][w][lane] = hn[2][0];
    sH[1][w][lane + 32] = hn[2][1];
    __syncthreads();
    // E's plane k at the owned places (reference.rs:14-50 with back differences, then the slabs)
    const T fez = A.fe[nx + ny + k];
    const bool zs = !A.periodic[2] && (k < A.low[2] || k >= nz - A.high[2]);
    const bool zb = wrap_index(k - 1, nz, A.periodic[2]) >= 0;
    T en[3][2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      // -x: the previous lane's value; lane 0 of the second half takes lane 31 of the first
      T hz_p = __shfl_up_sync(0xffffffffu, hn[2][h], 1);
      T hy_p = __shfl_up_sync(0xffffffffu, hn[1][h], 1);
      T hz_o = __shfl_sync(0xffffffffu, hn[2][0], 31);
      T hy_o = __shfl_sync(0xffffffffu, hn[1][0], 31);
      if (lane == 0) {
        hz_p = h == 1 ? hz_o : T(0);
        hy_p = h == 1 ? hy_o : T(0);
      }
      if (gx[h] == 0 && !A.periodic[0]) hz_p = hy_p = T(0);  // beyond the wall at x = 0
      T hx_yp = w >= 1 ? sH[0][w - 1][lane + 32 * h] : T(0);
      T hz_yp = w >= 1 ? sH[1][w - 1][lane + 32 * h] : T(0);
      T hy_zp = zb ? hprev[1][h] : T(0), hx_zp = zb ? hprev[0][h] : T(0);
      T dyHz = hn[2][h] - hz_yp, dzHy = hn[1][h] - hy_zp, dzHx = hn[0][h] - hx_zp;
      T dxHz = hn[2][h] - hz_p, dxHy = hn[1][h] - hy_p, dyHx = hn[0][h] - hx_yp;
      T curl[3] = {dyHz * fey - dzHy * fez, dzHx * fez - dxHz * fex[h], dxHy * fex[h] - dyHx * fey};
      const int i = mx[h], j = my;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        T cbv = P.cb[c][h];
        T cav;
        if (LOSSY) cav = P.ca[c][h];
        else cav = cbv == T(0) ? T(0) : T(1);
        en[c][h] = cav * ek[c][h] + cbv * curl[c];
      }
      if (own[h] && ((sx[h] >= 0) | (sy >= 0) | zs)) {
        // E_x: y then z; E_y: x then z; E_z: x then y
        if (sy >= 0) {
          SlabEntry e = slab_of(A, 0, 0, 1, sy);
          if (e.count) en[0][h] = slab_apply<T, 0>(A, e, 0, 1, i, j, k, dyHz, en[0][h], P.cb[0][h], true);
        }
        if (zs) {
          SlabEntry z0 = zslab_of(A, 0, 0, k);
          if (z0.count) en[0][h] = slab_apply<T, 0>(A, z0, 0, 2, i, j, k, dzHy, en[0][h], P.cb[0][h], true);
        }
        if (sx[h] >= 0) {
          SlabEntry e = slab_of(A, 0, 1, 0, sx[h]);
          if (e.count) en[1][h] = slab_apply<T, 0>(A, e, 1, 0, i, j, k, dxHz, en[1][h], P.cb[1][h], true);
        }
        if (zs) {
          SlabEntry z1 = zslab_of(A, 0, 1, k);
          if (z1.count) en[1][h] = slab_apply<T, 0>(A, z1, 1, 2, i, j, k, dzHx, en[1][h], P.cb[1][h], true);
        }
        if (sx[h] >= 0) {
          SlabEntry e = slab_of(A, 0, 2, 0, sx[h]);
          if (e.count) en[2][h] = slab_apply<T, 0>(A, e, 2, 0, i, j, k, dxHy, en[2][h], P.cb[2][h], true);
        }
        if (sy >= 0) {
          SlabEntry e = slab_of(A, 0, 2, 1, sy);
          if (e.count) en[2][h] = slab_apply<T, 0>(A, e, 2, 1, i, j, k, dyHx, en[2][h], P.cb[2][h], true);
        }
      }
      hprev[0][h] = hn[0][h];
      hprev[1][h] = hn[1][h];
    }
    // the electric currents (src/fdtd.rs:1375-1387)
    {
      const int bucket = tileidx * nz + k;
      const int g0 = A.ebucket[bucket], g1 = A.ebucket[bucket + 1];
      for (int g = g0; g < g1; g++) {
        Group gr = A.egroups[g];
        int gw = gr.local / SEG, gi = gr.local % SEG;
        if (gw == w && (gi & 31) == lane) {
          const bool second = (gi >> 5) != 0;
          T cbv = T(0), v = T(0);
#pragma unroll
          for (int c = 0; c < 3; c++)
            if (gr.comp == c) {
              cbv = second ? P.cb[c][1] : P.cb[c][0];
              v = second ? en[c][1] : en[c][0];
            }
          for (int q = gr.first; q < gr.first + gr.count; q++) {
            v = apply_e<T>(v, A.entries[q], A.waves_e, cbv);
          }
#pragma unroll
          for (int c = 0; c < 3; c++)
            if (gr.comp == c) {
              if (second) en[c][1] = v;
              else en[c][0] = v;
            }
        }
      }
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
      if (!own[h]) continue;
      long long at = pk + rowoff + mx[h];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        T v = en[c][h];
        if (MEDIA) {
          int mi = A.media.member[c * N + at];
          if (mi >= 0) {
            const MediaArgs<T> &M = A.media;
            int g = M.group[mi];
            int np = M.gpoles[g];
            T before = M.before[mi];
            T rest = M.gchi[g] * before;
            const T *pl = M.gpole + (long long)g * M.maxpoles * 3;
            T *cur = M.current + (long long)mi * M.maxpoles;
            T *prev = M.previous + (long long)mi * M.maxpoles;
            for (int p = 0; p < np; p++)
              rest = rest - T(0.5) * ((pl[3 * p] + T(1)) * cur[p] + pl[3 * p + 1] * prev[p]);
            T next = v + M.scale[mi] * rest;
            T slope = (next - before) / M.two_dt;
            for (int p = 0; p < np; p++) {
              T jn = pl[3 * p] * cur[p] + pl[3 * p + 1] * prev[p] + pl[3 * p + 2] * slope;
              prev[p] = cur[p];
              cur[p] = jn;
            }
            M.before[mi] = ek[c][h];
            v = next;
          }
        }
        A.e_out[c * N + at] = v;
      }
    }
    // E(k+1) becomes E(k)
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
      for (int c = 0; c < 3; c++) ek[c][h] = P.e1[c][h];
    __syncthreads();  // the exchanges are rewritten next plane
  };
  // two planes a turn, so each plane's registers keep a fixed role
  for (int k = kbeg; k < kend; k += 2) {
    plane(P0, P1, k);
    if (k + 1 < kend) plane(P1, P0, k + 1);
  }
}


// ------------------------------------------------------------------------------------------
// The quad step (v3), the default where nx is a multiple of 4. A CTA owns OWNX = 124 values along
// x and RW rows along y of a run of planes. Warp w holds row y0 - 1 + w; lane l holds the four
// values x0 - 4 + 4l .. x0 - 1 + 4l of it (128 a row: the tile's 124 and the 4 before it, whose
// last H the tile's first E needs). Every global access is a 16-byte vector. The next plane's E,
// H and cb rows are brought into shared memory by cp.async while the CTA computes this one (each
// warp copies its own rows, its lanes' places fixed for the whole run); neighbours along x come
// from the lane's own registers and one shuffle, along y from the staged rows and a small
// exchange of H, along z from the registers of the previous plane. The CPML's psi along y and z
// is read and written four values at once, its coefficients uniform over a row or a plane.
// Every value's arithmetic is step_kernel's, operation for operation.
namespace quad {
constexpr int VEC = 4;
constexpr int ROW = 128;      // H and E values a warp row holds
constexpr int OWNX = 124;     // values a tile owns along x
constexpr int RW = 7;         // rows a tile owns along y
constexpr int WARPS = RW + 1;
constexpr int THREADS = 32 * WARPS;
constexpr int EW = ROW + VEC;  // staged E row: x0-4 .. x0+127 (the last chunk for lane 31's +x)
constexpr int ER = RW + 2;     // staged E rows: y0-1 .. y0+RW
template <typename T>
struct Smem {
  static constexpr int E_SLOT = 3 * ER * EW;             // E of one plane
  // H(k) rows, cb(k) rows, then each warp's x-slab psi of its row at plane k: [field][component
  // y, z][16 places] (XP_OFF on), staged with the rows rather than read when the slab needs it
  static constexpr int XP_OFF = 3 * WARPS * ROW + 3 * RW * ROW;
  static constexpr int XP = 64;
  static constexpr int HB_SLOT = XP_OFF + WARPS * XP;
  // the new H's rows: H_x and H_z for the row after, H_z and H_y for the row's own x CPML
  static constexpr int X = 3 * WARPS * ROW;
  // the x CPML's b and a at the row's places: [field][component y, z][b, a][ROW] (0 outside)
  static constexpr int XC = 2 * 2 * 2 * ROW;
  // kappa/h along x at the row's places: [fh, fe][ROW]
  static constexpr int FX = 2 * ROW;
  static constexpr size_t BYTES =
      sizeof(T) * (3 * (size_t)E_SLOT + 2 * (size_t)HB_SLOT + X + XC + FX);
};
}  // namespace quad

template <typename T>
struct Vec4 {
  T v[4];
};
template <typename T>
__device__ __forceinline__ Vec4<T> ld4(const T *p) {
  Vec4<T> r;
  if (sizeof(T) == 4) {
    float4 f = *reinterpret_cast<const float4 *>(p);
    r.v[0] = (T)f.x; r.v[1] = (T)f.y; r.v[2] = (T)f.z; r.v[3] = (T)f.w;
  } else {
    double2 a = *reinterpret_cast<const double2 *>(p), b = *reinterpret_cast<const double2 *>(p + 2);
    r.v[0] = (T)a.x; r.v[1] = (T)a.y; r.v[2] = (T)b.x; r.v[3] = (T)b.y;
  }
  return r;
}
template <typename T>
__device__ __forceinline__ void st4(T *p, const Vec4<T> &r) {
  if (sizeof(T) == 4) {
    *reinterpret_cast<float4 *>(p) = make_float4((float)r.v[0], (float)r.v[1], (float)r.v[2], (float)r.v[3]);
  } else {
    *reinterpret_cast<double2 *>(p) = make_double2((double)r.v[0], (double)r.v[1]);
    *reinterpret_cast<double2 *>(p + 2) = make_double2((double)r.v[2], (double)r.v[3]);
  }
}

// four values of a slab (its psi row contiguous in x) updated at once: psi <- b psi + a (d/h),
// then H -= dt (sign psi) or E += cb (sign psi), each value as slab_update does
template <typename T, int FIELD>
__device__ __forceinline__ void slab4(const StepArgs<T> &A, T *psi_out, const T *psi_in, T b, T a,
                                      int axis, T sign, const T diff[4], T v[4], const T cbv[4],
                                      bool write) {
  Vec4<T> old = ld4(psi_in);
  Vec4<T> nw;
  T q[4];
  div4_by_step(diff, q, A.step[axis], A.inv_step[axis], A.inv_step64[axis], A.fast_div[axis]);
#pragma unroll
  for (int j = 0; j < 4; j++) {
    T d = q[j];
    nw.v[j] = b * old.v[j] + a * d;
    T u = sign * nw.v[j];
    if (FIELD == 1) v[j] = v[j] - A.dt * u;
    else v[j] = v[j] + cbv[j] * u;
  }
  if (write) st4(psi_out, nw);
}

// slab4 with the psi row already read
template <typename T, int FIELD>
__device__ __forceinline__ void slab4_loaded(const StepArgs<T> &A, T *psi_out, const Vec4<T> &old,
                                             const SlabEntry &s, int q, int axis, T sign,
                                             const T diff[4], T v[4], const T cbv[4], bool write) {
  const T b = A.coefs[s.coef + q], a = A.coefs[s.coef + s.count + q];
  Vec4<T> nw;
  T dq[4];
  div4_by_step(diff, dq, A.step[axis], A.inv_step[axis], A.inv_step64[axis], A.fast_div[axis]);
#pragma unroll
  for (int j = 0; j < 4; j++) {
    T d = dq[j];
    nw.v[j] = b * old.v[j] + a * d;
    T u = sign * nw.v[j];
    if (FIELD == 1) v[j] = v[j] - A.dt * u;
    else v[j] = v[j] + cbv[j] * u;
  }
  if (write) st4(psi_out, nw);
}

// The same along x, where each place has its own coefficients and only the places `in` the slab
// change (the psi row is padded to whole vectors; the other places keep their psi).
template <typename T, int FIELD>
__device__ __forceinline__ void slab4x(const StepArgs<T> &A, const T *xb4, const T *xa4,
                                       T *psi_out, const Vec4<T> &old, const bool in[4], T sign,
                                       const T diff[4], T v[4], const T cbv[4], bool write) {
  // xb4, xa4: b and a at the lane's four places (the CTA's table)
  const Vec4<T> bb = ld4(xb4), aa = ld4(xa4);
  Vec4<T> nw;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    nw.v[j] = old.v[j];
    if (in[j]) {
      T d = div_by_step(diff[j], A.step[0], A.inv_step[0], A.inv_step64[0], A.fast_div[0]);
      nw.v[j] = bb.v[j] * old.v[j] + aa.v[j] * d;
      T u = sign * nw.v[j];
      if (FIELD == 1) v[j] = v[j] - A.dt * u;
      else v[j] = v[j] + cbv[j] * u;
    }
  }
  if (write) st4(psi_out, nw);
}

// The CPML of one field at a lane's four places, slab by slab in the reference's order for each
// component (src/fdtd/kernel.rs:525-579: along x, y, z): each slab's psi row read, updated and
// written before the next, so that only one row is live at a time.
template <typename T, int FIELD>
__device__ __forceinline__ void cpml4(const StepArgs<T> &A, int k, int my, int mxb, int sx,
                                      bool xmixed, const bool inx[4], bool zs, int sy, bool write,
                                      T v[3][4], const T diff[3][3][4], const T cbv[3][4],
                                      const T *xc) {
  // xc: the CTA's x coefficient table at this lane's first place (quad::Smem::XC)
  const int nx = A.n[0], ny = A.n[1];
  const long long plane = (long long)nx * ny;
  const T *pin = FIELD == 1 ? A.psi_h_in : A.psi_e;
  T *pout = FIELD == 1 ? A.psi_h_out : A.psi_e;
  const T one = T(1), minus = T(-1);
  const T zero4[4] = {T(0), T(0), T(0), T(0)};
  const int zside = zs ? (k < A.low[2] ? 0 : 1) : 0;
  const bool xs = sx >= 0 && !xmixed;
  // along y at (k, my): rows of nx
  auto y_slab = [&](int c, T sign, const T d[4], T w[4], const T *cb) {
    const SlabEntry &s = A.slab[FIELD][c][1][sy];
    if (!s.count) return;
    const long long at = s.psi + ((long long)k * s.count + (my - s.from)) * nx + mxb;
    slab4_loaded<T, FIELD>(A, pout + at, ld4(pin + at), s, my - s.from, 1, sign, d, w, cb,
                           write);
  };
  auto z_slab = [&](int c, T sign, const T d[4], T w[4], const T *cb) {
    const SlabEntry &s = A.slab[FIELD][c][2][zside];
    if (!s.count) return;
    const long long at = s.psi + (long long)(k - s.from) * plane + (long long)my * nx + mxb;
    slab4_loaded<T, FIELD>(A, pout + at, ld4(pin + at), s, k - s.from, 2, sign, d, w, cb,
                           write);
  };
  auto x_slab = [&](int c, T sign, const T d[4], T w[4], const T *cb) {
    const SlabEntry &s = A.slab[FIELD][c][0][sx];
    if (!s.count) return;
    const long long at = s.psi + ((long long)k * ny + my) * s.pw + (mxb - s.pf);
    const T *t = xc + ((FIELD * 2 + (c - 1)) * 2) * quad::ROW;
    slab4x<T, FIELD>(A, t, t + quad::ROW, pout + at, ld4(pin + at), inx, sign, d, w, cb, write);
  };
  // component x: y (+) then z (-)
  if (sy >= 0) y_slab(0, one, diff[0][1], v[0], FIELD == 1 ? zero4 : cbv[0]);
  if (zs) z_slab(0, minus, diff[0][2], v[0], FIELD == 1 ? zero4 : cbv[0]);
  // component y: x (-) then z (+)
  if (xs) x_slab(1, minus, diff[1][0], v[1], FIELD == 1 ? zero4 : cbv[1]);
  if (zs) z_slab(1, one, diff[1][2], v[1], FIELD == 1 ? zero4 : cbv[1]);
  // component z: x (+) then y (-)
  if (xs) x_slab(2, one, diff[2][0], v[2], FIELD == 1 ? zero4 : cbv[2]);
  if (sy >= 0) y_slab(2, minus, diff[2][1], v[2], FIELD == 1 ? zero4 : cbv[2]);
}

// The x-slab places of a quad tile's rows (the same for every row of the tile), as positions
// 0..ROW-1 of the row: where the positions hold one side's slab only, at most 16 places, p0 and
// P and the side (0 low, 1 high); otherwise side -1.
template <typename T>
__device__ __forceinline__ int xslab_places(const StepArgs<T> &A, int x0, int &p0, int &P) {
  using quad::ROW;
  using quad::VEC;
  if (A.periodic[0]) return -1;
  const int nx = A.n[0];
  const int l0 = max(0, VEC - x0), l1 = min(ROW, VEC - x0 + A.low[0]);
  const int h0 = max(0, nx - A.high[0] - x0 + VEC), h1 = min(ROW, nx - x0 + VEC);
  const int nl = max(0, l1 - l0), nh = max(0, h1 - h0);
  if (nl > 0 && nh == 0 && nl <= 16) return p0 = l0, P = nl, 0;
  if (nh > 0 && nl == 0 && nh <= 16) return p0 = h0, P = nh, 1;
  return -1;
}

// The x CPML of one field over a warp's row, its values shared out over the lanes: the row holds
// the slab's places p0 .. p0+P-1 (side, p0 and P from xslab_places), and lane L < 2P updates
// component 1 + L / P at place p0 + L % P; the owner applies the result, which it reads back from
// the row's positions in u1 (component 1) or u2 (component 2): scratch rows of the warp's own,
// whose earlier values it has done with (the warp's staged rows of the old H); or, with SHARED
// false, which it is shuffled (the lossy form, where the shared rows' loads spill). The x
// difference is taken from the staged rows the owner's came from, the same two values: for H
// forward, r[pos+1] - r[pos], over E's rows (r1 E_z for H_y, r2 E_y for H_z, positions from
// x0-4); for E backward, r[pos] - r[pos-1], over the new H's exchange rows (r1 H_z for E_y, r2
// H_y for E_z). Each value's arithmetic and each component's order of slabs are slab4x's (x
// before the others); only the lane that computes it differs, so that a tile whose rows meet an
// x CPML pays for its few places once per warp, not once per place of each lane. Lanes below
// `ownmin` own no values (E: the halo lane). Every lane of the warp calls it.
template <typename T, int FIELD, bool SHARED>
__device__ __forceinline__ void xcoop(const StepArgs<T> &A, int k, int my, int x0, int lane,
                                      int side, int p0, int P, int ownmin, bool write, T v[3][4],
                                      const T *r1, const T *r2, const T cbv[3][4], const T *xc,
                                      const T *xp, T *u1, T *u2) {
  using quad::ROW;
  using quad::VEC;
  if (SHARED) __syncwarp();  // the lanes are done with the scratch rows' earlier values
  const int c = lane < P ? 1 : 2;
  const int pos = p0 + lane - (c - 1) * P;
  const bool work = lane < 2 * P && (pos >> 2) >= ownmin;
  T u = T(0);
  if (work) {
    const SlabEntry &s = A.slab[FIELD][c][0][side];
    if (s.count) {
      const long long at = s.psi + ((long long)k * A.n[1] + my) * s.pw + (x0 - VEC + pos - s.pf);
      const T *t = xc + ((FIELD * 2 + (c - 1)) * 2) * ROW;
      const T b = t[pos], a = t[ROW + pos];
      const T old = xp[(FIELD * 2 + (c - 1)) * 16 + (lane - (c - 1) * P)];  // staged
      const T *r = c == 1 ? r1 : r2;
      const T d = FIELD == 1 ? r[pos + 1] - r[pos] : r[pos] - r[pos - 1];
      const T q = div_by_step(d, A.step[0], A.inv_step[0], A.inv_step64[0], A.fast_div[0]);
      const T nw = b * old + a * q;
      u = (c == 1 ? T(-1) : T(1)) * nw;
      if (write && (pos >> 2) >= 1) (FIELD == 1 ? A.psi_h_out : A.psi_e)[at] = nw;
      if (SHARED) (c == 1 ? u1 : u2)[pos] = u;
    }
  }
  const bool has1 = A.slab[FIELD][1][0][side].count != 0;
  const bool has2 = A.slab[FIELD][2][0][side].count != 0;
  if (!SHARED) {
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int q = 4 * lane + r - p0;  // this lane's place r as a worker of component 1
      const bool mine = q >= 0 && q < P && lane >= ownmin;
      const T g1 = __shfl_sync(0xffffffffu, u, mine ? q : lane);
      const T g2 = __shfl_sync(0xffffffffu, u, mine ? P + q : lane);
      if (mine) {
        if (FIELD == 1) {
          if (has1) v[1][r] = v[1][r] - A.dt * g1;
          if (has2) v[2][r] = v[2][r] - A.dt * g2;
        } else {
          if (has1) v[1][r] = v[1][r] + cbv[1][r] * g1;
          if (has2) v[2][r] = v[2][r] + cbv[2][r] * g2;
        }
      }
    }
    return;
  }
  __syncwarp();
  // the owners: lanes with a place in the slab (the halo lane aside), one component at a time
  if (lane >= ownmin && 4 * lane + 3 >= p0 && 4 * lane < p0 + P) {
#pragma unroll
    for (int cc = 1; cc < 3; cc++) {
      if (!(cc == 1 ? has1 : has2)) continue;
      const Vec4<T> g = ld4((cc == 1 ? u1 : u2) + VEC * lane);
#pragma unroll
      for (int r = 0; r < 4; r++) {
        const int q = 4 * lane + r - p0;  // this lane's place r among the slab's
        if (q >= 0 && q < P) {
          if (FIELD == 1) v[cc][r] = v[cc][r] - A.dt * g.v[r];
          else v[cc][r] = v[cc][r] + cbv[cc][r] * g.v[r];
        }
      }
    }
  }
}

// Member q's ADE update (src/fdtd/media.rs:661-705), after the step has written E^{n+1} (curl,
// slabs and currents) into e_out: J_p^{n+1} = alpha J_p^n + xi J_p^{n-1} + gamma (E^{n+1} -
// E^{n-1}) / (2 dt) with E^{n+1} corrected by the currents' chi; E^n from e_in kept as E^{n-1}.
template <typename T>
__device__ __forceinline__ void ade_update(const StepArgs<T> &A, long long q) {
  const MediaArgs<T> &M = A.media;
  const long long at = M.place[q];
  const int g = M.group[q];
  const int np = M.gpoles[g];
  const T before = M.before[q];
  T rest = M.gchi[g] * before;
  const T *pl = M.gpole + (long long)g * M.maxpoles * 3;
  T *cur = M.current + q * M.maxpoles;
  T *prev = M.previous + q * M.maxpoles;
  for (int p = 0; p < np; p++)
    rest = rest - T(0.5) * ((pl[3 * p] + T(1)) * cur[p] + pl[3 * p + 1] * prev[p]);
  const T next = A.e_out[at] + M.scale[q] * rest;
  const T slope = (next - before) / M.two_dt;
  for (int p = 0; p < np; p++) {
    const T jn = pl[3 * p] * cur[p] + pl[3 * p + 1] * prev[p] + pl[3 * p + 2] * slope;
    prev[p] = cur[p];
    cur[p] = jn;
  }
  M.before[q] = A.e_in[at];
  A.e_out[at] = next;
}

// The dispersive media's ADE update as a pass of its own after the step kernel, one thread a
// member in value order. (Run inside the step kernel, at the end of each CTA's run of planes,
// the same update took a step on the dispersive 256 x 256 x 128 grid from 0.353 to 0.434 ms:
// the members' gathers are latency-bound and held up the stencil's CTAs; as a pass of its own
// they run at the whole device's occupancy.)
template <typename T>
__global__ void ade_kernel(StepArgs<T> A) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < A.media.members) ade_update(A, q);
}

template <typename T, bool LOSSY>
__global__ void __launch_bounds__(quad::THREADS, 2) quad_kernel(StepArgs<T> A) {
  using namespace quad;
  using S = Smem<T>;
  constexpr int CH = 16 / (int)sizeof(T);  // values a cp.async chunk carries
  extern __shared__ __align__(16) unsigned char quad_raw[];
  T *sEs = reinterpret_cast<T *>(quad_raw);          // [3 slots][3][ER][EW]
  T *sHB = sEs + 3 * (size_t)S::E_SLOT;              // [2 slots][H 3][WARPS][ROW] + [cb 3][RW][ROW]
  T *sX = sHB + 2 * (size_t)S::HB_SLOT;              // [3][WARPS][ROW]
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nx = A.n[0], ny = A.n[1], nz = A.n[2];
  const long long N = A.N;
  const int ntiles = A.tiles_x * A.tiles_y;
  const int cta = A.order[blockIdx.x];  // heaviest first (quad_order)
  const int tile = cta % ntiles;
  const int x0 = (tile % A.tiles_x) * OWNX, y0 = (tile / A.tiles_x) * RW;
  const int kbeg = A.runs[cta / ntiles], kend = A.runs[cta / ntiles + 1];
  if (kbeg >= nz) return;
  const long long plane = (long long)nx * ny;
  T *sXC = sX + S::X;                                // quad::Smem::XC
  T *sFX = sXC + S::XC;                              // quad::Smem::FX

  // -- this lane's four places along x, this warp's row
  const int xb = x0 - VEC + VEC * lane;  // the first of the four
  int mxb;                               // where they are in memory (a wrapped group), or -1
  if (xb >= 0 && xb < nx) mxb = xb;
  else if (A.periodic[0] && xb == -VEC) mxb = nx - VEC;
  else if (A.periodic[0] && xb == nx) mxb = 0;
  else mxb = -1;
  // the chunk after the row (lane 31's +x neighbour), x0 + 124
  const int xa = x0 + OWNX;
  const int mxa = xa < nx ? xa : ((A.periodic[0] && xa == nx) ? 0 : -1);
  const int gy = y0 - 1 + w;
  const int my = wrap_index(gy, ny, A.periodic[1]);
  const int myp = wrap_index(gy + 1, ny, A.periodic[1]);
  const bool rowh = my >= 0 && gy < ny;
  bool hv[4], ownv[4];
  int sxs[4];  // the x CPML side of each place (-1 none)
#pragma unroll
  for (int j = 0; j < 4; j++) {
    int x = xb + j;
    int mxj = wrap_index(x, nx, A.periodic[0]);
    hv[j] = rowh && mxj >= 0 && x < nx;
    ownv[j] = hv[j] && w >= 1 && lane >= 1;
    sxs[j] = -1;
    if (mxj >= 0 && !A.periodic[0]) {
      if (mxj < A.low[0]) sxs[j] = 0;
      else if (mxj >= nx - A.high[0]) sxs[j] = 1;
    }
  }
  const bool any_x = (sxs[0] >= 0) | (sxs[1] >= 0) | (sxs[2] >= 0) | (sxs[3] >= 0);
  // the lane's x-slab side, and whether its places touch both sides (then one place at a time)
  int sxl = -1;
  bool xmixed = false;
  bool inx[4];
#pragma unroll
  for (int j = 0; j < 4; j++) {
    inx[j] = sxs[j] >= 0;
    if (sxs[j] >= 0) {
      if (sxl >= 0 && sxl != sxs[j]) xmixed = true;
      sxl = sxs[j];
    }
  }
  const bool any_own = ownv[0] | ownv[1] | ownv[2] | ownv[3];
  // the row's x-slab places (the same for every warp): one side's, at most 16, are shared out
  // over the warp's lanes (xcoop), and cpml4 takes no x slab; otherwise each lane takes its own
  bool xco;
  int xside, xp0 = 0, xP = 0;
  xside = xslab_places(A, x0, xp0, xP);
  xco = xside >= 0;
  if (xco) sxl = -1;
  const T fhy = my >= 0 ? A.fh[nx + my] : T(0), fey = my >= 0 ? A.fe[nx + my] : T(0);
  int sy = -1;
  if (my >= 0 && !A.periodic[1]) {
    if (my < A.low[1]) sy = 0;
    else if (my >= ny - A.high[1]) sy = 1;
  }
  const int rowoff = my >= 0 ? my * nx : 0;  // in-plane offsets fit an int (quad_ok)
  // whether the tile has currents in any plane (most have none: then no plane looks them up)
  const bool hcur = A.hbucket[(long long)tile * nz] != A.hbucket[(long long)tile * nz + nz];
  const bool ecur = A.ebucket[(long long)tile * nz] != A.ebucket[(long long)tile * nz + nz];

  // -- copies: warp w copies E's row w, H's row w and cb's row w-1 of a plane, lane l the chunks
  // of its four places; warp 0 (the halo row, which has no E to update) also E's row RW+1 and
  // the chunk after each of E's rows (lane q takes (component, row) = (q / ER, q % ER), and
  // q + 32 … where 3 ER is over 32).
  // Where a chunk lies beyond a wall (a row, a group of four or a plane the grid doesn't have)
  // it is zero-filled, so the staged neighbours there are the zeros the differences need.
  // Each chunk's offset within a plane is fixed for the run: -1 where it lies beyond a wall.
  const int myp_last = wrap_index(y0 + RW, ny, A.periodic[1]);
  const bool w0 = w == 0;
  const int off_e0 = (my >= 0 && mxb >= 0) ? my * nx + mxb : -1;
  const int off_e1 = (myp_last >= 0 && mxb >= 0) ? myp_last * nx + mxb : -1;

  const int off_h = off_e0;
  const int off_b = (w >= 1 && gy < ny) ? off_e0 : -1;
  // this thread's places in a staged E row, H row and cb row
  const int erow = w * EW + VEC * lane, hrow = w * ROW + VEC * lane;
  const int brow = (w >= 1 ? w - 1 : 0) * ROW + VEC * lane;
  auto chunk = [&](T *dst, const T *field, int off, long long pbase) {
    const bool ok = off >= 0 && pbase >= 0;
    const T *src = ok ? field + pbase + off : A.e_in;
#pragma unroll
    for (int q = 0; q < VEC / CH; q++) cp_async16(dst + q * CH, src + q * CH, ok);
  };
  // E(ke) rows into E slot E (ke < 0: zeros); H(kh), cb(kh) rows into HB slot H (H null: none)
  // a lane of the x slab's (xcoop): component y (lanes below P) or z, its place xp0 + xq
  const bool xstage = xco && rowh && lane < 2 * xP;
  const int xcomp = lane < xP ? 1 : 2, xq = lane < xP ? lane : lane - xP;
  auto issue = [&](T *E, int ke, T *H, int kh) {
    const long long pe = ke >= 0 ? (long long)ke * plane : -1;
#pragma unroll
    for (int c = 0; c < 3; c++) chunk(E + c * ER * EW + erow, A.e_in + c * N, off_e0, pe);
    if (w0) {
#pragma unroll
      for (int c = 0; c < 3; c++)
        chunk(E + (c * ER + RW + 1) * EW + VEC * lane, A.e_in + c * N, off_e1, pe);
      for (int q = lane; q < 3 * ER; q += 32) {
        const int qc = q / ER, qr = q % ER;
        const int qy = wrap_index(y0 - 1 + qr, ny, A.periodic[1]);
        chunk(E + (qc * ER + qr) * EW + ROW, A.e_in + qc * N,
              (qy >= 0 && mxa >= 0) ? qy * nx + mxa : -1, pe);
      }
    }
    if (H) {
      const long long ph = kh >= 0 ? (long long)kh * plane : -1;
#pragma unroll
      for (int c = 0; c < 3; c++) chunk(H + c * WARPS * ROW + hrow, A.h_in + c * N, off_h, ph);
      // the row's x-slab psi at plane kh, one value a lane of the slab's (xcoop reads them)
      if (xstage && kh >= 0) {
        T *xp = H + S::XP_OFF + w * S::XP;
#pragma unroll
        for (int f = 0; f < 2; f++) {
          const SlabEntry &sl = A.slab[f][xcomp][0][xside];
          if (sl.count)
            cp_async_value(xp + (f * 2 + (xcomp - 1)) * 16 + xq,
                           (f == 1 ? A.psi_h_in : A.psi_e) + sl.psi +
                               ((long long)kh * ny + my) * sl.pw + (x0 - VEC + xp0 + xq - sl.pf));
        }
      }
      if (w >= 1) {
        T *B = H + 3 * WARPS * ROW;
#pragma unroll
        for (int c = 0; c < 3; c++) chunk(B + c * RW * ROW + brow, A.cb + c * N, off_b, ph);
      }
    }
    cp_async_commit();
  };
  // the slots as pointers, turned round as the planes go by: E(k), E(k+1) and the one being
  // filled (E(k+2)); H and cb of plane k and the one being filled
  T *e_cur = sEs, *e_next = sEs + S::E_SLOT, *e_fill = sEs + 2 * S::E_SLOT;
  T *hb_cur = sHB, *hb_fill = sHB + S::HB_SLOT;
  auto Erow = [&](const T *slot, int c, int r) -> const T * { return slot + (c * ER + r) * EW; };
  auto Hrow = [&](const T *slot, int c) -> const T * { return slot + c * WARPS * ROW + w * ROW; };
  auto Brow = [&](const T *slot, int c) -> const T * {
    return slot + 3 * WARPS * ROW + c * RW * ROW + (w - 1) * ROW;
  };

  // H's new plane k at the lane's four places, from E(k) (E slot se), E(k+1) (slot se1), H(k)
  // (HB slot sh): the forward differences, then the slabs along x, y, z
  auto compute_h = [&](const T *se, const T *se1, const T *sh, int k, T fhz, bool write,
                       T hn[3][4]) {
    Vec4<T> e[3], eyp[2], ez1[2], ho[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      e[c] = ld4(Erow(se, c, w) + VEC * lane);
      ho[c] = ld4(Hrow(sh, c) + VEC * lane);
    }
    eyp[0] = ld4(Erow(se, 0, w + 1) + VEC * lane);  // E_x, E_z of the row after
    eyp[1] = ld4(Erow(se, 2, w + 1) + VEC * lane);
    ez1[0] = ld4(Erow(se1, 0, w) + VEC * lane);     // E_x, E_y of the plane after
    ez1[1] = ld4(Erow(se1, 1, w) + VEC * lane);
    const Vec4<T> fx = ld4(sFX + VEC * lane);  // kappa/h along x at the lane's places
    // +x of the fourth place: the next lane's first, lane 31 the chunk after the row (read by
    // every lane, one address: a broadcast, and no branch)
    const T ey_a = Erow(se, 1, w)[ROW], ez_a = Erow(se, 2, w)[ROW];
    T ey_n = __shfl_down_sync(0xffffffffu, e[1].v[0], 1);
    T ez_n = __shfl_down_sync(0xffffffffu, e[2].v[0], 1);
    ey_n = lane == 31 ? ey_a : ey_n;
    ez_n = lane == 31 ? ez_a : ez_n;
    // a row or plane after beyond a wall was staged as zeros: no test needed here
    T dyEz[4], dzEy[4], dzEx[4], dxEz[4], dxEy[4], dyEx[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      T eyn = j < 3 ? e[1].v[j + 1] : ey_n, ezn = j < 3 ? e[2].v[j + 1] : ez_n;
      T exy = eyp[0].v[j], ezy = eyp[1].v[j];
      T exz = ez1[0].v[j], eyz = ez1[1].v[j];
      dyEz[j] = ezy - e[2].v[j];
      dzEy[j] = eyz - e[1].v[j];
      dzEx[j] = exz - e[0].v[j];
      dxEz[j] = ezn - e[2].v[j];
      dxEy[j] = eyn - e[1].v[j];
      dyEx[j] = exy - e[0].v[j];
      const T fhx = fx.v[j];
      hn[0][j] = ho[0].v[j] - A.dt * (dyEz[j] * fhy - dzEy[j] * fhz);
      hn[1][j] = ho[1].v[j] - A.dt * (dzEx[j] * fhz - dxEz[j] * fhx);
      hn[2][j] = ho[2].v[j] - A.dt * (dxEy[j] * fhx - dyEx[j] * fhy);
    }
    // the CPML: H_x along y then z, H_y along x then z, H_z along x then y
    const bool zs = !A.periodic[2] && (k < A.low[2] || k >= nz - A.high[2]);
    if (xco && rowh) {
      const T nocb[3][4] = {};
      // scratch: the warp's rows of the old H, in registers since the top (ho)
      xcoop<T, 1, !LOSSY>(A, k, my, x0, lane, xside, xp0, xP, 0, write && w >= 1, hn,
                          Erow(se, 2, w), Erow(se, 1, w), nocb, sXC, sh + S::XP_OFF + w * S::XP,
                          const_cast<T *>(Hrow(sh, 0)), const_cast<T *>(Hrow(sh, 1)));
    }
    if (rowh && mxb >= 0 && (zs | (sy >= 0) | (any_x && !xco))) {
      const bool ow = write && w >= 1 && lane >= 1;
      const T diff[3][3][4] = {
          {{T(0), T(0), T(0), T(0)}, {dyEz[0], dyEz[1], dyEz[2], dyEz[3]}, {dzEy[0], dzEy[1], dzEy[2], dzEy[3]}},
          {{dxEz[0], dxEz[1], dxEz[2], dxEz[3]}, {T(0), T(0), T(0), T(0)}, {dzEx[0], dzEx[1], dzEx[2], dzEx[3]}},
          {{dxEy[0], dxEy[1], dxEy[2], dxEy[3]}, {dyEx[0], dyEx[1], dyEx[2], dyEx[3]}, {T(0), T(0), T(0), T(0)}}};
      const T nocb[3][4] = {};
      cpml4<T, 1>(A, k, my, mxb, sxl, xmixed, inx, zs, sy, ow, hn, diff, nocb, sXC + VEC * lane);
    }
    // beyond a wall H comes out zero (E's back differences read zero there): its E and H were
    // staged as zeros and its kappa/h is zero, so every term above is +0
    // the magnetic currents at this tile and plane, each value's entries in CPU order
    const int bucket = tile * nz + k;
    const int g0 = hcur ? A.hbucket[bucket] : 0, g1 = hcur ? A.hbucket[bucket + 1] : 0;
    for (int g = g0; g < g1; g++) {
      Group gr = A.hgroups[g];
      const int gw = gr.local / ROW, gi = gr.local % ROW;
      if (gw == w && (gi >> 2) == lane) {
        const int jj = gi & 3;
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (gr.comp == c && jj == j) {
              T v = hn[c][j];
              for (int q = gr.first; q < gr.first + gr.count; q++) {
                v = apply_h<T>(v, A.entries[q], A.waves_h, A.dt);
              }
              hn[c][j] = v;
            }
      }
    }
  };

  T hn[3][4], hprev[2][4];
  // prologue: H's new plane kbeg-1 (wrapped on a periodic z)
  const int km = wrap_index(kbeg - 1, nz, A.periodic[2]);
  // positions: E slots by position p = plane - kbeg + 1 (km at 0), HB slots alike
  issue(e_cur, km, hb_cur, km);                          // E(km), H(km), cb(km)
  issue(e_next, kbeg, nullptr, -1);                      // E(kbeg)
  // plane kbeg's H and cb, and E(kbeg+1), into the slots the prologue leaves alone: in flight
  // while it computes (it waits for the two groups before this one only)
  issue(e_fill, wrap_index(kbeg + 1, nz, A.periodic[2]), hb_fill, kbeg);
  // while those copies are in flight: kappa/h along x at the row's places, and (where the
  // row's places reach an x CPML, else it is never read) the x CPML's b and a there; read after
  // the barrier below or the loop's first
  for (int q = threadIdx.x; q < S::FX; q += THREADS) {
    const int mx = wrap_index(x0 - VEC + q % ROW, nx, A.periodic[0]);
    sFX[q] = mx >= 0 ? (q < ROW ? A.fh : A.fe)[mx] : T(0);
  }
  const bool xtile = !A.periodic[0] && ((A.low[0] > 0 && x0 - VEC < A.low[0]) ||
                                        (A.high[0] > 0 && x0 - VEC + ROW > nx - A.high[0]));
  if (xtile) {
    static_assert(S::XC % THREADS == 0, "the table is whole rounds of the CTA's threads");
    T val[S::XC / THREADS];  // the loads first, then the stores: all in flight together
#pragma unroll
    for (int i = 0; i < S::XC / THREADS; i++) {
      const int q = threadIdx.x + i * THREADS;
      const int at = q % ROW, ba = (q / ROW) % 2, c = 1 + (q / (2 * ROW)) % 2, f = q / (4 * ROW);
      const int gx = x0 - VEC + at;
      val[i] = T(0);
      if (gx >= 0 && gx < nx) {
        const int side = gx < A.low[0] ? 0 : (gx >= nx - A.high[0] ? 1 : -1);
        if (side >= 0) {
          const SlabEntry &e = A.slab[f][c][0][side];
          if (e.count && gx >= e.from && gx < e.from + e.count)
            val[i] = A.coefs[e.coef + ba * e.count + (gx - e.from)];
        }
      }
    }
#pragma unroll
    for (int i = 0; i < S::XC / THREADS; i++) sXC[threadIdx.x + i * THREADS] = val[i];
  }
  if (km >= 0) {
    cp_async_wait<1>();
    __syncthreads();
    compute_h(e_cur, e_next, hb_cur, km, A.fh[nx + ny + km], false, hn);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      hprev[0][j] = hn[0][j];
      hprev[1][j] = hn[1][j];
    }
  } else {
#pragma unroll
    for (int j = 0; j < 4; j++) hprev[0][j] = hprev[1][j] = T(0);
  }
  __syncthreads();
  // the slots move on one plane: E(kbeg) current
  {
    T *t = e_cur;
    e_cur = e_next;
    e_next = e_fill;
    e_fill = t;
    t = hb_cur;
    hb_cur = hb_fill;
    hb_fill = t;
  }
  // kappa/h along z at plane k, read a plane ahead
  T fhz = A.fh[nx + ny + kbeg], fez = A.fe[nx + ny + kbeg];
  // the CPML's psi rows of this warp's row at plane kp into L2 (one thread a row): read from
  // memory a plane later, they then come from L2 rather than DRAM
  const int pf0 = max(x0 - VEC, 0), pf1 = min(x0 + OWNX, nx);
  auto prefetch_psi = [&](int kp) {
    const bool zsp = !A.periodic[2] && (kp < A.low[2] || kp >= nz - A.high[2]);
    const int zside = kp < A.low[2] ? 0 : 1;
    const unsigned row = (unsigned)((pf1 - pf0) * (int)sizeof(T));
#pragma unroll
    for (int f = 0; f < 2; f++) {
      const T *base = f == 1 ? A.psi_h_in : A.psi_e;
      if (sy >= 0) {
#pragma unroll
        for (int c = 0; c < 3; c += 2) {  // x and z along y
          const SlabEntry &sl = A.slab[f][c][1][sy];
          if (sl.count)
            prefetch_l2(base + sl.psi + ((long long)kp * sl.count + (my - sl.from)) * nx + pf0, row);
        }
      }
      if (zsp) {
#pragma unroll
        for (int c = 0; c < 2; c++) {  // x and y along z
          const SlabEntry &sl = A.slab[f][c][2][zside];
          if (sl.count)
            prefetch_l2(base + sl.psi + (long long)(kp - sl.from) * plane + (long long)my * nx + pf0,
                        row);
        }
      }
    }
  };
  for (int k = kbeg; k < kend; k++) {
    const T fhz_next = k + 1 < kend ? A.fh[nx + ny + k + 1] : T(0);
    const T fez_next = k + 1 < kend ? A.fe[nx + ny + k + 1] : T(0);
    cp_async_wait<0>();
    __syncthreads();  // plane k's rows landed; every warp is done with plane k-1
    if (k + 1 < kend) {
      issue(e_fill, wrap_index(k + 2, nz, A.periodic[2]), hb_fill, k + 1);
      if (lane == 0 && rowh && pf1 > pf0) prefetch_psi(k + 1);
    }
    compute_h(e_cur, e_next, hb_cur, k, fhz, true, hn);
    // H's tile to memory, H_x and H_z to the row below
    const long long at = (long long)k * plane + rowoff + (mxb < 0 ? 0 : mxb);
    // the lossy form's ca of E's plane k, read now so that the barrier below covers the wait
    Vec4<T> ca[3];
    if (LOSSY && w >= 1 && any_own) {
#pragma unroll
      for (int c = 0; c < 3; c++) ca[c] = ld4(A.ca + c * N + at);
    }
    if (w >= 1 && lane >= 1 && rowh && mxb >= 0 && xb < nx) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        Vec4<T> o;
#pragma unroll
        for (int j = 0; j < 4; j++) o.v[j] = hn[c][j];
        st4(A.h_out + c * N + at, o);
      }
    }
    {
      Vec4<T> a, b;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        a.v[j] = hn[0][j];
        b.v[j] = hn[2][j];
      }
      st4(sX + (size_t)w * ROW + VEC * lane, a);
      st4(sX + (size_t)(WARPS + w) * ROW + VEC * lane, b);
      if (xco) {
#pragma unroll
        for (int j = 0; j < 4; j++) a.v[j] = hn[1][j];
        st4(sX + (size_t)(2 * WARPS + w) * ROW + VEC * lane, a);
      }
    }
    // the exchange row w goes to warp w+1 alone: a named barrier a pair of warps (id w+1, 64
    // threads; warp w arrives, warp w+1 waits) rather than the whole tile; warp w's own rows (its
    // x CPML's) are its own writes, ordered for it by its sync. The rows are written again only
    // after the next plane's barrier, which every warp passes after its E.
    if (w + 1 < WARPS) named_arrive(w + 1, 64);
    if (w >= 1) named_sync(w, 64);
    // E's plane k at the owned places: back differences, then the slabs
    const bool zs = !A.periodic[2] && (k < A.low[2] || k >= nz - A.high[2]);
    T en[3][4];
    if (w >= 1) {
      Vec4<T> e[3], cb[3], hxm, hzm;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        e[c] = ld4(Erow(e_cur, c, w) + VEC * lane);
        cb[c] = ld4(Brow(hb_cur, c) + VEC * lane);
      }
      hxm = ld4(sX + (size_t)(w - 1) * ROW + VEC * lane);  // the row before
      hzm = ld4(sX + (size_t)(WARPS + w - 1) * ROW + VEC * lane);
      const Vec4<T> fex = ld4(sFX + ROW + VEC * lane);
      // -x of the first place: the previous lane's fourth
      T hz_p = __shfl_up_sync(0xffffffffu, hn[2][3], 1);
      T hy_p = __shfl_up_sync(0xffffffffu, hn[1][3], 1);
      T dyHz[4], dzHy[4], dzHx[4], dxHz[4], dxHy[4], dyHx[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        T hzx = j > 0 ? hn[2][j - 1] : hz_p, hyx = j > 0 ? hn[1][j - 1] : hy_p;
        // H's plane before: the prologue's (zeros below a wall) or the last iteration's
        T hyz = hprev[1][j], hxz = hprev[0][j];
        dyHz[j] = hn[2][j] - hzm.v[j];
        dzHy[j] = hn[1][j] - hyz;
        dzHx[j] = hn[0][j] - hxz;
        dxHz[j] = hn[2][j] - hzx;
        dxHy[j] = hn[1][j] - hyx;
        dyHx[j] = hn[0][j] - hxm.v[j];
        T curl0 = dyHz[j] * fey - dzHy[j] * fez;
        T curl1 = dzHx[j] * fez - dxHz[j] * fex.v[j];
        T curl2 = dxHy[j] * fex.v[j] - dyHx[j] * fey;
        T cav[3];
#pragma unroll
        for (int c = 0; c < 3; c++) cav[c] = LOSSY ? ca[c].v[j] : (cb[c].v[j] == T(0) ? T(0) : T(1));
        en[0][j] = cav[0] * e[0].v[j] + cb[0].v[j] * curl0;
        en[1][j] = cav[1] * e[1].v[j] + cb[1].v[j] * curl1;
        en[2][j] = cav[2] * e[2].v[j] + cb[2].v[j] * curl2;
      }
      // the CPML: E_x along y then z, E_y along x then z, E_z along x then y
      if (xco && rowh) {
        const T cbs[3][4] = {{cb[0].v[0], cb[0].v[1], cb[0].v[2], cb[0].v[3]},
                             {cb[1].v[0], cb[1].v[1], cb[1].v[2], cb[1].v[3]},
                             {cb[2].v[0], cb[2].v[1], cb[2].v[2], cb[2].v[3]}};
        xcoop<T, 0, !LOSSY>(A, k, my, x0, lane, xside, xp0, xP, 1, true, en,
                            sX + (size_t)(WARPS + w) * ROW, sX + (size_t)(2 * WARPS + w) * ROW,
                            cbs, sXC, hb_cur + S::XP_OFF + w * S::XP,
                            const_cast<T *>(Hrow(hb_cur, 0)), const_cast<T *>(Hrow(hb_cur, 1)));
      }
      if (any_own && mxb >= 0 && (zs | (sy >= 0) | (any_x && !xco))) {
        const T diff[3][3][4] = {
            {{T(0), T(0), T(0), T(0)}, {dyHz[0], dyHz[1], dyHz[2], dyHz[3]}, {dzHy[0], dzHy[1], dzHy[2], dzHy[3]}},
            {{dxHz[0], dxHz[1], dxHz[2], dxHz[3]}, {T(0), T(0), T(0), T(0)}, {dzHx[0], dzHx[1], dzHx[2], dzHx[3]}},
            {{dxHy[0], dxHy[1], dxHy[2], dxHy[3]}, {dyHx[0], dyHx[1], dyHx[2], dyHx[3]}, {T(0), T(0), T(0), T(0)}}};
        const T cbs[3][4] = {{cb[0].v[0], cb[0].v[1], cb[0].v[2], cb[0].v[3]},
                             {cb[1].v[0], cb[1].v[1], cb[1].v[2], cb[1].v[3]},
                             {cb[2].v[0], cb[2].v[1], cb[2].v[2], cb[2].v[3]}};
        cpml4<T, 0>(A, k, my, mxb, sxl, xmixed, inx, zs, sy, true, en, diff, cbs, sXC + VEC * lane);
      }
      // the electric currents (src/fdtd.rs:1375-1387)
      const int bucket = tile * nz + k;
      const int g0 = ecur ? A.ebucket[bucket] : 0, g1 = ecur ? A.ebucket[bucket + 1] : 0;
      for (int g = g0; g < g1; g++) {
        Group gr = A.egroups[g];
        const int gw = gr.local / ROW, gi = gr.local % ROW;
        if (gw == w && (gi >> 2) == lane) {
          const int jj = gi & 3;
#pragma unroll
          for (int c = 0; c < 3; c++)
#pragma unroll
            for (int j = 0; j < 4; j++)
              if (gr.comp == c && jj == j) {
                T v = en[c][j];
                const T cbv = cb[c].v[j];
                for (int q = gr.first; q < gr.first + gr.count; q++) {
                  v = apply_e<T>(v, A.entries[q], A.waves_e, cbv);
                }
                en[c][j] = v;
              }
        }
      }
      if (lane >= 1 && rowh && mxb >= 0 && xb < nx) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
          Vec4<T> o;
#pragma unroll
          for (int j = 0; j < 4; j++) o.v[j] = en[c][j];
          st4(A.e_out + c * N + at, o);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      hprev[0][j] = hn[0][j];
      hprev[1][j] = hn[1][j];
    }
    fhz = fhz_next;
    fez = fez_next;
    T *t = e_cur;  // the slots move on one plane
    e_cur = e_next;
    e_next = e_fill;
    e_fill = t;
    t = hb_cur;
    hb_cur = hb_fill;
    hb_fill = t;
  }
  cp_async_wait<0>();
}

// The waveforms of a batch of steps, in f64 (src/fdtd.rs:329-423): for step m of the batch, w
// at H's time t = (first+m) dt and at E's t + dt/2, 2 doubles each per emitter.
// point[e]: 1 if emitter e is a point source (w.at), else 0 (complex_at)
// base: the batch's first step index in device memory (a captured batch), or null (first).
// stride: each step's values, the emitters' then the plane waves' slots (2 doubles each)
__global__ void waves_kernel(const Wave *waves, const int *point, int nw, int stride,
                             long long first, const long long *base, int batch, double dt,
                             double *out_h, double *out_e) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nw * batch) return;
  if (base) first = *base;
  int m = q / nw, e = q % nw;
  double t = (double)(first + m) * dt;
  double half = t + 0.5 * dt;
  double re, im;
  wave_eval(waves[e], t, &re, &im, point[e]);
  out_h[2 * ((long long)m * stride + e)] = re;
  out_h[2 * ((long long)m * stride + e) + 1] = im;
  wave_eval(waves[e], half, &re, &im, point[e]);
  out_e[2 * ((long long)m * stride + e)] = re;
  out_e[2 * ((long long)m * stride + e) + 1] = im;
}

// A plane wave's auxiliary 1D run on the device (PlaneWaveRun, src/fdtd/sources.rs:755-1041).
struct AuxDev {
  long long len, pad;
  long long g[3];
  double steps[3];
  double *e, *h;  // 3 x len each, component by component
  const double *ca, *cb, *da, *db;
  int nsheet;
  const int *sheet_comp;
  const long long *sheet_i;
  const double *sheet_j;
  Wave wave;
  int nslots, slot0;  // its slots, numbered on from slot0 after the other runs'
  const int *slot_field, *slot_comp;
  const long long *slot_i;
};

// (f[i + o] - f[i - o]) / step along an axis the direction moves o samples for (0 if none)
__device__ __forceinline__ double aux_difference(const double *f, long long o, double step,
                                                 long long i) {
  if (o == 0) return 0.0;
  return (f[i + o] - f[i - o]) / step;
}

// A batch of steps of every plane wave's run, a CTA each, in the reference's order
// (PlaneWaveRun::step_h then step_e, src/fdtd/sources.rs:1008-1040): before step m's H update the
// slots of E its box's H couplings read, after it the slots of H its E couplings read, into the
// step's values at nw + slot (stride values a step). The run's state stays on the device.
__global__ void __launch_bounds__(1024) aux_kernel(const AuxDev *runs, int nw, int stride,
                                                   long long first, const long long *base,
                                                   int batch, double dt, double *out_h,
                                                   double *out_e) {
  const AuxDev R = runs[blockIdx.x];
  if (base) first = *base;
  const long long len = R.len, inner = len - 2 * R.pad;
  for (int m = 0; m < batch; m++) {
    const double t = (double)(first + m) * dt, half = t + 0.5 * dt;
    double *oh = out_h + 2LL * ((long long)m * stride + nw + R.slot0);
    double *oe = out_e + 2LL * ((long long)m * stride + nw + R.slot0);
    for (int q = threadIdx.x; q < R.nslots; q += blockDim.x)
      if (R.slot_field[q] == 0) {
        oh[2 * q] = R.e[R.slot_comp[q] * len + R.slot_i[q]];
        oh[2 * q + 1] = 0.0;
      }
    for (long long q = threadIdx.x; q < 3 * inner; q += blockDim.x) {
      const int c = (int)(q / inner);
      const long long i = R.pad + q % inner;
      const int a = (c + 1) % 3, b = (c + 2) % 3;
      const double curl = aux_difference(R.e + b * len, R.g[a], R.steps[a], i) -
                          aux_difference(R.e + a * len, R.g[b], R.steps[b], i);
      R.h[c * len + i] = R.da[i] * R.h[c * len + i] - R.db[i] * curl;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < R.nslots; q += blockDim.x)
      if (R.slot_field[q] == 1) {
        oe[2 * q] = R.h[R.slot_comp[q] * len + R.slot_i[q]];
        oe[2 * q + 1] = 0.0;
      }
    for (long long q = threadIdx.x; q < 3 * inner; q += blockDim.x) {
      const int c = (int)(q / inner);
      const long long i = R.pad + q % inner;
      const int a = (c + 1) % 3, b = (c + 2) % 3;
      const double curl = aux_difference(R.h + b * len, R.g[a], R.steps[a], i) -
                          aux_difference(R.h + a * len, R.g[b], R.steps[b], i);
      R.e[c * len + i] = R.ca[i] * R.e[c * len + i] + R.cb[i] * curl;
    }
    __syncthreads();
    if (threadIdx.x == 0 && R.nsheet > 0) {  // the sheet's J at t + dt/2, one value at a time
      double w, unused;
      wave_eval(R.wave, half, &w, &unused, 1);
      for (int q = 0; q < R.nsheet; q++) {
        const long long i = R.sheet_i[q];
        double &v = R.e[R.sheet_comp[q] * len + i];
        v = v - R.cb[i] * R.sheet_j[q] * w;
      }
    }
    __syncthreads();
  }
}

// One coupling across a Bloch side (Bloch::wrap, src/fdtd/bloch.rs:97-152): value r of
// component c reads component d at q across the side; (pr, pi) = e^(+-ikL) - 1, s = its sign
// times kappa / step; for E's, cb the value's; for H's, its slot among the step's values.
struct WrapDev {
  long long r, q;
  int c, d;
  double pr, pi, s, cb;
  int slot, pad;
};

// H's couplings: this step's amounts dt Re and dt Im of (e^(ikL) - 1) F s, F both parts' E now,
// into each part's step values (the step kernels subtract them after H's sources).
template <typename T>
__global__ void bloch_h_kernel(const WrapDev *w, int n, const T *e_re, const T *e_im,
                               long long N, double dt, double *vals_re, double *vals_im) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const WrapDev x = w[k];
  const double fr = (double)e_re[x.d * N + x.q], fi = (double)e_im[x.d * N + x.q];
  const double cr = x.pr * fr - x.pi * fi, ci = x.pr * fi + x.pi * fr;
  vals_re[2 * x.slot] = dt * (cr * x.s);
  vals_re[2 * x.slot + 1] = 0.0;
  vals_im[2 * x.slot] = dt * (ci * x.s);
  vals_im[2 * x.slot + 1] = 0.0;
}

// E's couplings after both parts' E updates: E += cb Re and Im of (e^(-ikL) - 1) F s, F both
// parts' new H; one thread a value, its couplings (one per Bloch axis) in the reference's order.
template <typename T>
__global__ void bloch_e_kernel(const WrapDev *w, const int *start, int nvalues, const T *h_re,
                               const T *h_im, long long N, T *e_re, T *e_im) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nvalues) return;
  for (int k = start[v]; k < start[v + 1]; k++) {
    const WrapDev x = w[k];
    const double fr = (double)h_re[x.d * N + x.q], fi = (double)h_im[x.d * N + x.q];
    const double cr = x.pr * fr - x.pi * fi, ci = x.pr * fi + x.pi * fr;
    T &a = e_re[x.c * N + x.r];
    a = a + (T)(x.cb * (cr * x.s));
    T &b = e_im[x.c * N + x.r];
    b = b + (T)(x.cb * (ci * x.s));
  }
}

// After a step: the probes' values into the record, the transformed values into the ring.
template <typename T>
__global__ void gather_kernel(const T *e, const T *h, const long long *where, int count,
                              T *ring_row, const long long *probes, int nprobes, double *record_row) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < count) {
    long long w = where[q];  // field bit 62, then component * N + r
    const T *f = (w >> 62) ? h : e;
    ring_row[q] = f[w & ((1LL << 62) - 1)];
  } else if (q < count + nprobes) {
    long long w = probes[q - count];
    const T *f = (w >> 62) ? h : e;
    record_row[q - count] = (double)f[w & ((1LL << 62) - 1)];
  }
}

// e^{i w t} dt for each step of the batch and each (monitor, field, frequency) slot
// (src/fdtd/monitors.rs:178-183): E at te = (first+m+1) dt, H at te - dt/2.
__global__ void phase_kernel(const double *omega, const int *slot_field, int nslots,
                             long long first, const long long *base, int batch, double dt,
                             double *out) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nslots * batch) return;
  if (base) first = *base;
  int m = q / nslots, s = q % nslots;
  double te = (double)(first + m + 1) * dt;
  double t = slot_field[s] ? te - 0.5 * dt : te;
  double sn, cs;
  pxp::sincos(omega[s] * t, &sn, &cs);
  out[2 * (long long)q] = cs * dt;
  out[2 * (long long)q + 1] = sn * dt;
}

// Sets a captured batch's first step index.
__global__ void set_base_kernel(long long *base, long long first) { *base = first; }

// sums[f][v] += sum_m ring[m][v] * phase[m][slot(f)], m in time order, f64 (monitors.rs:185-206).
template <typename T>
__global__ void dft_kernel(const SeriesDev *series, int nseries, const long long *value_series,
                           long long nvalues, const T *ring, int batch, const double *phase,
                           int nslots, double *sums) {
  long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nvalues) return;
  SeriesDev s = series[value_series[v]];
  long long o = v - s.value0;
  for (int f = 0; f < s.nf; f++) {
    double *acc = sums + 2 * (s.sum0 + (long long)f * s.volume + o);
    double re = acc[0], im = acc[1];
    const double *ph = phase + 2 * (long long)(s.slot0 + f);
    for (int m = 0; m < batch; m++) {
      double x = (double)ring[(long long)m * nvalues + v];
      re = re + x * ph[2 * (long long)m * nslots];
      im = im + x * ph[2 * (long long)m * nslots + 1];
    }
    acc[0] = re;
    acc[1] = im;
  }
}

// The transform of a complex run's values (src/fdtd/monitors.rs:127-154): each step's
// (re + i im) times its phase added to the sums in time order, the real parts from `ring`, the
// imaginary from `ring_im`.
template <typename T>
__global__ void dft_complex_kernel(const SeriesDev *series, const long long *value_series,
                                   long long nvalues, const T *ring, const T *ring_im, int batch,
                                   const double *phase, int nslots, double *sums) {
  long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nvalues) return;
  SeriesDev s = series[value_series[v]];
  long long o = v - s.value0;
  for (int f = 0; f < s.nf; f++) {
    double *acc = sums + 2 * (s.sum0 + (long long)f * s.volume + o);
    double re = acc[0], im = acc[1];
    const double *ph = phase + 2 * (long long)(s.slot0 + f);
    for (int m = 0; m < batch; m++) {
      const double x = (double)ring[(long long)m * nvalues + v];
      const double y = (double)ring_im[(long long)m * nvalues + v];
      const double pr = ph[2 * (long long)m * nslots], pi = ph[2 * (long long)m * nslots + 1];
      re = re + (x * pr - y * pi);
      im = im + (x * pi + y * pr);
    }
    acc[0] = re;
    acc[1] = im;
  }
}

// f64 host values to the engine's precision and back. `in` or `out` may be a host array mapped
// into the device's address space (then the kernel reads or writes it over the host link
// directly); grid-stride, so that a few CTAs per SM keep enough requests in flight.
template <typename T>
__global__ void convert_kernel(const double *in, T *out, long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride)
    out[q] = (T)in[q];
}
template <typename T>
__global__ void widen_kernel(const T *in, double *out, long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride)
    out[q] = (double)in[q];
}
// host[q] += dev[q]: the transforms' sums added into the caller's (Monitors::add,
// src/fdtd/monitors.rs:866-887), `host` mapped into the device's address space
__global__ void add_into_kernel(const double *dev, double *host, long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride)
    host[q] = host[q] + dev[q];
}

}  // namespace pxf

using namespace pxf;

// For every finite float x: whether div_by_step's product form (reciprocal r) gives x / h's
// bits. Sets *bad if any x differs. 2^32 values, a few milliseconds on a B200.
__global__ void verify_division_kernel(float h, float r, double rd, int *bad) {
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  int found = 0;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
       i < (1ULL << 32); i += stride) {
    const float x = __uint_as_float((unsigned)i);
    if (!isfinite(x)) continue;
    if (__float_as_uint(div_by_step(x, h, r, rd, 1)) != __float_as_uint(x / h)) found = 1;
  }
  if (found) atomicOr(bad, 1);
}

// ------------------------------------------------------------------------------------------
// The context: the device state of one simulation.

struct DeviceSlab {
  int field, comp, axis;
  long long from, count, psi, coef, size;
  long long pf, pw;  // x slabs: the padded rows (see SlabEntry)
};

struct fdtd_ctx {
  std::string error;
  int precision = 32;
  size_t elem = 4;
  int n[3];
  long long N;
  int periodic[3], low[3], high[3];
  double dt;
  double step[3];
  double inv_step[3] = {0, 0, 0};  // 1/step as the kernels round it
  int fast_div[3] = {0, 0, 0};     // div_by_step's product form checked for this step
  size_t budget = 0, used = 0;
  cudaStream_t stream = nullptr;
  std::vector<void *> allocations;
  // fields: two copies each, 3N values
  void *e[2] = {nullptr, nullptr}, *h[2] = {nullptr, nullptr};
  int parity = 0;
  void *ca = nullptr, *cb = nullptr;
  bool lossless = true, coeffs_set = false, fields_set = false;
  void *fe = nullptr, *fh = nullptr, *coefs = nullptr;
  void *psi_h[2] = {nullptr, nullptr}, *psi_e = nullptr;
  long long psi_h_len = 0, psi_e_len = 0;
  std::vector<DeviceSlab> slabs;
  SlabEntry table[2][3][3][2];
  // launch shape
  int tiles_x, tiles_y, zchunk, zchunks;
  int sms = 148;
  bool staged = false;  // the staged kernel (nx a multiple of 16 bytes' worth of values)
  bool row = false;     // the row kernel
  bool quad = false;    // the quad kernel (the default where nx is a multiple of 4)
  // a tile's owned values along x and y, and how a source's place is numbered in its tile: over
  // rows `loc_w` wide from (x0 - loc_x, y0 - 1), E too unless `e_tile` (then over the tile)
  int tile_w = TX, tile_h = TY, loc_w = TX + 1, loc_x = 1;
  bool e_tile = true;
  int staged_per_sm[2][2][2] = {{{0, 0}, {0, 0}}, {{0, 0}, {0, 0}}};
  // sources
  int nwaves = 0;
  Wave *d_waves = nullptr;
  int *d_point = nullptr;
  int *hbucket = nullptr, *ebucket = nullptr;
  int *order = nullptr;  // the quad kernel's CTAs, heaviest first
  int runs[quad_max_runs + 1] = {};  // the quad kernel's runs of planes (quad_runs)
  Group *hgroups = nullptr, *egroups = nullptr;
  Entry *entries = nullptr;
  double *waves_h = nullptr, *waves_e = nullptr;  // batch x (nwaves + naux) x 2
  int wave_batch = 0;
  // plane waves' auxiliary runs (fdtd_set_plane_waves): their descriptors (pointing into device
  // memory), and the slots their couplings read, recorded each step after the emitters' values
  int naux_runs = 0, naux = 0;
  int nbloch = 0;     // slots of H's couplings across Bloch sides (fdtd_set_bloch_slots), after
  int naux_laid = 0;  // the plane waves'; the slot count fdtd_set_sources laid the values out for
  std::vector<AuxDev> aux;
  std::vector<void *> aux_memory;
  AuxDev *d_aux = nullptr;
  int stride() const { return nwaves + naux + nbloch; }
  // probes and transforms
  int nprobes = 0;
  long long *d_probes = nullptr;
  double *record = nullptr;
  long long record_cap = 0, recorded = 0;
  long long nvalues = 0;
  long long *d_where = nullptr, *d_value_series = nullptr;
  SeriesDev *d_series = nullptr;
  int nseries = 0, nslots = 0;
  double *d_omega = nullptr;
  int *d_slot_field = nullptr;
  long long nsums = 0;
  double *sums = nullptr;
  void *ring = nullptr;
  double *phase = nullptr;
  int ring_k = 0;
  // every call that changes what the device holds or how it is laid out moves this on (a batch
  // reuses its tables while its members' generations stay as it left them)
  unsigned long long generation = 0;
  // what a captured batch of steps bakes in (buffers, tables, kernels) changes only with these
  // calls: the sources, probes, transforms, media and coefficients' set-up
  unsigned long long layout = 0;
  // K steps captured as a graph, one per current copy at the batch's start; their layout
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  unsigned long long graph_layout[2] = {0, 0};
  long long graph_kernels[2] = {0, 0};
  long long *d_base = nullptr;  // the captured batch's first step index
  bool capturing = false;
  bool warmed = false;  // a batch has run directly (lazily set kernel attributes are set)
  // the sources as last set (the batch builds its own tables from them)
  std::vector<fdtd_waveform> src_waves;
  std::vector<fdtd_injection> src_inj;
  // media
  bool media = false;
  MediaArgs<float> mf;
  MediaArgs<double> md;
  long long launches = 0;
  // staging for host arrays a kernel can't reach (pageable memory): f64 values, made on the
  // first such transfer and kept (counted in the HBM budget)
  double *stage = nullptr;
  long long stage_len = 0;
  // step-kernel timing: pairs of events around each launch while profiling
  bool profiling = false;
  std::vector<cudaEvent_t> events;
  size_t events_used = 0;
};

namespace {

int fail(fdtd_ctx *c, int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->error = buf;
  return code;
}

#define CUDA_TRY(c, call)                                                                      \
  do {                                                                                         \
    cudaError_t err_ = (call);                                                                 \
    if (err_ != cudaSuccess)                                                                   \
      return fail((c), FDTD_E_GPU, "%s: %s (%s:%d)", #call, cudaGetErrorString(err_), __FILE__, \
                  __LINE__);                                                                   \
  } while (0)

int alloc(fdtd_ctx *c, void **p, size_t bytes) {
  bytes = std::max<size_t>(bytes, 16);
  if (c->budget && c->used + bytes > c->budget)
    return fail(c, FDTD_E_BUDGET, "%zu MB more would exceed the HBM budget of %zu MB",
                bytes >> 20, c->budget >> 20);
  // stream-ordered, so that engines made and freed while others run (a serving loop) don't
  // synchronize the device; the stream's work so far is waited for before the memory is used
  cudaError_t e = cudaMallocAsync(p, bytes, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(c, FDTD_E_GPU, "cudaMallocAsync of %zu MB: %s", bytes >> 20, cudaGetErrorString(e));
  }
  c->used += bytes;
  c->allocations.push_back(*p);
  return 0;
}
void release(fdtd_ctx *c, void *p) {
  if (!p) return;
  auto it = std::find(c->allocations.begin(), c->allocations.end(), p);
  if (it != c->allocations.end()) c->allocations.erase(it);
  cudaFreeAsync(p, c->stream);
}

// A copy between host and device ordered on the engine's stream and finished before returning:
// the engine's memory is stream-ordered, so no copy may run on another stream (a legacy-stream
// copy still in flight could land in memory the stream has since freed).
cudaError_t copy(fdtd_ctx *c, void *dst, const void *src, size_t bytes, cudaMemcpyKind kind) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return e;
}

// The device's address of a host array of `bytes` bytes when all of it is page-locked and mapped
// into the device's address space (cudaHostAlloc'd, or registered with the runtime); else null:
// pageable memory, which only the copy engines reach, through a staging buffer.
void *mapped_range(const void *host, size_t bytes) {
  if (!host || bytes == 0) return nullptr;
  auto device_address = [](const void *p) -> char * {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return a.type == cudaMemoryTypeHost ? static_cast<char *>(a.devicePointer) : nullptr;
  };
  char *first = device_address(host);
  char *last = device_address(static_cast<const char *>(host) + bytes - 1);
  if (!first || !last || last != first + (bytes - 1)) return nullptr;
  return first;
}

// Blocks for a grid-stride pass over n values: a few CTAs per SM, fewer for short arrays.
unsigned stride_blocks(const fdtd_ctx *c, long long n) {
  return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 4LL * c->sms));
}

// The context's staging buffer for pageable transfers, made on first use.
int staging(fdtd_ctx *c) {
  if (c->stage) return 0;
  const long long len = std::min<long long>(3 * c->N, 1LL << 21);
  if (int r = alloc(c, (void **)&c->stage, (size_t)len * 8)) return r;
  c->stage_len = len;
  return 0;
}

// n f64 host values into dst in the engine's precision. f64: one copy. f32 from mapped host
// memory: one kernel reading the host array over the link and converting as it goes (nothing
// staged); from pageable memory: through the context's staging buffer, a chunk at a time. The
// caller synchronizes before handing the host array back.
template <typename T>
int upload_as(fdtd_ctx *c, void *dst, const double *src, long long n) {
  if (n == 0) return 0;
  if (sizeof(T) == 8) {
    CUDA_TRY(c, cudaMemcpyAsync(dst, src, n * 8, cudaMemcpyHostToDevice, c->stream));
    return 0;
  }
  if (const void *dev = mapped_range(src, (size_t)n * 8)) {
    convert_kernel<T><<<stride_blocks(c, n), 256, 0, c->stream>>>((const double *)dev, (T *)dst, n);
    CUDA_TRY(c, cudaGetLastError());
    return 0;
  }
  if (int r = staging(c)) return r;
  for (long long at = 0; at < n; at += c->stage_len) {
    const long long m = std::min(c->stage_len, n - at);
    CUDA_TRY(c, cudaMemcpyAsync(c->stage, src + at, m * 8, cudaMemcpyHostToDevice, c->stream));
    convert_kernel<T><<<stride_blocks(c, m), 256, 0, c->stream>>>(c->stage, (T *)dst + at, m);
    CUDA_TRY(c, cudaGetLastError());
  }
  return 0;
}
int upload(fdtd_ctx *c, void *dst, const double *src, long long n) {
  return c->precision == 64 ? upload_as<double>(c, dst, src, n) : upload_as<float>(c, dst, src, n);
}
// n values of src into the host's f64 array dst, finished before returning; the mirror of
// upload_as (f32 into mapped host memory: one kernel widening as it writes over the link).
template <typename T>
int download_as(fdtd_ctx *c, double *dst, const void *src, long long n) {
  if (n == 0) return 0;
  if (sizeof(T) == 8) {
    CUDA_TRY(c, cudaMemcpyAsync(dst, src, n * 8, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return 0;
  }
  if (void *dev = mapped_range(dst, (size_t)n * 8)) {
    widen_kernel<T><<<stride_blocks(c, n), 256, 0, c->stream>>>((const T *)src, (double *)dev, n);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return 0;
  }
  if (int r = staging(c)) return r;
  for (long long at = 0; at < n; at += c->stage_len) {
    const long long m = std::min(c->stage_len, n - at);
    widen_kernel<T><<<stride_blocks(c, m), 256, 0, c->stream>>>((const T *)src + at, c->stage, m);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaMemcpyAsync(dst + at, c->stage, m * 8, cudaMemcpyDeviceToHost, c->stream));
  }
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return 0;
}
int download(fdtd_ctx *c, double *dst, const void *src, long long n) {
  return c->precision == 64 ? download_as<double>(c, dst, src, n)
                            : download_as<float>(c, dst, src, n);
}

template <typename T>
StepArgs<T> step_args(fdtd_ctx *c) {
  StepArgs<T> A;
  for (int a = 0; a < 3; a++) {
    A.n[a] = c->n[a];
    A.periodic[a] = c->periodic[a];
    A.low[a] = c->low[a];
    A.high[a] = c->high[a];
    A.step[a] = (T)c->step[a];
    A.inv_step[a] = (T)c->inv_step[a];
    A.inv_step64[a] = 1.0 / (double)(T)c->step[a];
    A.fast_div[a] = c->fast_div[a];
  }
  A.N = c->N;
  A.dt = (T)c->dt;
  A.fe = (const T *)c->fe;
  A.fh = (const T *)c->fh;
  A.e_in = (const T *)c->e[c->parity];
  A.h_in = (const T *)c->h[c->parity];
  A.e_out = (T *)c->e[1 - c->parity];
  A.h_out = (T *)c->h[1 - c->parity];
  A.ca = c->lossless ? nullptr : (const T *)c->ca;
  A.cb = (const T *)c->cb;
  memcpy(A.slab, c->table, sizeof A.slab);
  A.coefs = (const T *)c->coefs;
  A.psi_h_in = (const T *)c->psi_h[c->parity];
  A.psi_h_out = (T *)c->psi_h[1 - c->parity];
  A.psi_e = (T *)c->psi_e;
  A.hbucket = c->hbucket;
  A.ebucket = c->ebucket;
  A.hgroups = c->hgroups;
  A.egroups = c->egroups;
  A.entries = c->entries;
  A.tiles_x = c->tiles_x;
  A.tiles_y = c->tiles_y;
  A.zchunk = c->zchunk;
  A.order = c->order;
  for (int r = 0; r <= c->zchunks && r <= quad_max_runs; r++) A.runs[r] = c->runs[r];
  if (sizeof(T) == 8) memcpy(&A.media, &c->md, sizeof A.media);
  else memcpy(&A.media, &c->mf, sizeof A.media);
  return A;
}

template <typename T, bool LOSSY, bool MEDIA, int STAGES>
void launch_staged(fdtd_ctx *c, const StepArgs<T> &A) {
  auto kernel = staged_kernel<T, LOSSY, MEDIA, STAGES>;
  const size_t smem = staged_smem_bytes<T, STAGES>();
  int &per_sm = c->staged_per_sm[sizeof(T) == 8][LOSSY][MEDIA];
  if (per_sm == 0) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, NT, smem);
    if (per_sm < 1) per_sm = 1;
  }
  long long total = (long long)c->tiles_x * c->tiles_y * c->n[2];
  int ctas = (int)std::min<long long>(total, (long long)per_sm * c->sms);
  kernel<<<ctas, NT, smem, c->stream>>>(A, total, ctas);
}

template <typename T>
void launch_step(fdtd_ctx *c, const StepArgs<T> &A, bool ade = true) {
  if (c->quad) {
    dim3 grid(c->tiles_x * c->tiles_y * c->zchunks);
    const size_t smem = quad::Smem<T>::BYTES;
    auto go = [&](auto kernel) {
      if (!c->capturing)
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      kernel<<<grid, quad::THREADS, smem, c->stream>>>(A);
    };
    // media: the step (its E update without them), then their pass over the members
    if (c->lossless) go(quad_kernel<T, false>);
    else go(quad_kernel<T, true>);
    if (c->media && ade)
      ade_kernel<T><<<(unsigned)((A.media.members + 255) / 256), 256, 0, c->stream>>>(A);
    return;
  }
  if (c->row) {
    dim3 grid(c->tiles_x * c->tiles_y, c->zchunks);
    if (c->media) {
      if (c->lossless) row_kernel<T, false, true><<<grid, rowstep::THREADS, 0, c->stream>>>(A);
      else row_kernel<T, true, true><<<grid, rowstep::THREADS, 0, c->stream>>>(A);
    } else {
      if (c->lossless) row_kernel<T, false, false><<<grid, rowstep::THREADS, 0, c->stream>>>(A);
      else row_kernel<T, true, false><<<grid, rowstep::THREADS, 0, c->stream>>>(A);
    }
    return;
  }
  if (c->staged) {
    if (c->media) {
      if (c->lossless) launch_staged<T, false, true, 3>(c, A);
      else launch_staged<T, true, true, 3>(c, A);
    } else {
      if (c->lossless) launch_staged<T, false, false, 3>(c, A);
      else launch_staged<T, true, false, 3>(c, A);
    }
    return;
  }
  dim3 grid(c->tiles_x * c->tiles_y, c->zchunks);
  const size_t smem = plain_smem_bytes<T>();
  auto go = [&](auto kernel) {
    if (!c->capturing)
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kernel<<<grid, NT, smem, c->stream>>>(A);
  };
  if (c->media) {
    if (c->lossless) go(step_kernel<T, false, true>);
    else go(step_kernel<T, true, true>);
  } else {
    if (c->lossless) go(step_kernel<T, false, false>);
    else go(step_kernel<T, true, false>);
  }
}

// Whether div_by_step's product form equals division for grid step h on this device, checked
// once per (device, step) and remembered.
int division_checked(fdtd_ctx *c, float h, float r, int *ok) {
  static std::mutex mu;
  // keyed on the step's exact bits (r is a function of h)
  static std::map<std::pair<int, unsigned>, int> seen;
  int dev = 0;
  CUDA_TRY(c, cudaGetDevice(&dev));
  unsigned hb;
  memcpy(&hb, &h, 4);
  const auto key = std::make_pair(dev, hb);
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = seen.find(key);
    if (it != seen.end()) {
      *ok = it->second;
      return 0;
    }
  }
  int *bad = nullptr;
  CUDA_TRY(c, cudaMallocAsync(&bad, 4, c->stream));
  CUDA_TRY(c, cudaMemsetAsync(bad, 0, 4, c->stream));
  verify_division_kernel<<<c->sms * 8, 256, 0, c->stream>>>(h, r, 1.0 / (double)h, bad);
  int found = 1;
  cudaError_t err = cudaMemcpyAsync(&found, bad, 4, cudaMemcpyDeviceToHost, c->stream);
  cudaFreeAsync(bad, c->stream);
  if (err == cudaSuccess) err = cudaStreamSynchronize(c->stream);
  if (err != cudaSuccess) return fail(c, FDTD_E_GPU, "checking the division: %s", cudaGetErrorString(err));
  *ok = found ? 0 : 1;
  std::lock_guard<std::mutex> lock(mu);
  seen[key] = *ok;
  return 0;
}

// The quad kernel's runs of z-planes: `count` runs (at most quad_max_runs) that never straddle the
// edge of a z CPML, the CPMLs' planes (heavier) in runs of their own, the rest of about equal
// length but for two short ones (a quarter of the others, from four interior runs on): taken
// last (quad_order), they fill the step's end, where the SMs would otherwise wait on the longest
// CTAs. Returns the number of runs; starts in c->runs.
int quad_runs(fdtd_ctx *c, int count) {
  const int nz = c->n[2];
  const int lo = c->periodic[2] ? 0 : std::min(c->low[2], nz);
  const int hi = c->periodic[2] ? 0 : std::min(c->high[2], nz - lo);
  const int mid = nz - lo - hi;
  count = std::max(1, std::min(count, quad_max_runs));
  const int slabs = (lo > 0) + (hi > 0);
  // the interior's runs: what is left, at least one where it has planes
  int inner = mid > 0 ? std::max(1, std::min(mid, count - slabs)) : 0;
  // a CPML of more than 1.5 interior runs' planes is cut into runs of about that length
  const int len = inner > 0 ? (mid + inner - 1) / inner : std::max(lo, hi);
  auto pieces = [&](int planes) {
    return planes > 0 ? std::max(1, (int)((planes + 1.5 * len - 1) / (1.5 * len))) : 0;
  };
  int plo = pieces(lo), phi = pieces(hi);
  while (plo + inner + phi > quad_max_runs && inner > 1) inner--;
  while (plo + inner + phi > quad_max_runs) {
    if (plo >= phi && plo > 1) plo--;
    else if (phi > 1) phi--;
    else break;
  }
  int n = 0;
  c->runs[0] = 0;
  auto cut = [&](int from, int planes, int parts) {
    for (int q = 1; q <= parts; q++) c->runs[++n] = from + (int)((long long)planes * q / parts);
  };
  cut(0, lo, plo);
  const int longs = inner - 2;
  const int shorts = inner >= 4 ? std::max(2, (int)std::lround(mid / (longs + 0.5) / 4.0)) : 0;
  if (inner >= 4 && mid - 2 * shorts >= longs) {
    cut(lo, mid - 2 * shorts, longs);
    cut(lo + mid - 2 * shorts, 2 * shorts, 2);
  } else {
    cut(lo, mid, inner);
  }
  cut(lo + mid, hi, phi);
  return n;
}

// The quad kernel's CTAs (run r, tile t as r * tiles + t) in launch order: by an estimate of
// their time, heaviest first, so that the CTAs that start last are short and the step, which
// ends with its last CTA, leaves few SMs idle at its end. A plane of a tile costs 1, and more
// where the tile meets a CPML: 0.4 where its rows reach an x CPML, 1.15 times the share of its
// rows (of 8) in a y CPML, 0.95 in a z CPML's plane; a run's first, recomputed plane of H 0.6 of
// a plane. (Fitted to the CTAs' times on the 3D MMI, 600 x 200 x 100 with CPMLs of 10.)
std::vector<int> quad_order(const fdtd_ctx *c) {
  const int nx = c->n[0], ny = c->n[1], nz = c->n[2];
  const int tiles = c->tiles_x * c->tiles_y;
  auto zslab = [&](int k) { return !c->periodic[2] && (k < c->low[2] || k >= nz - c->high[2]); };
  std::vector<std::pair<double, int>> cost;
  cost.reserve((size_t)tiles * c->zchunks);
  for (int r = 0; r < c->zchunks; r++)
    for (int t = 0; t < tiles; t++) {
      const int x0 = (t % c->tiles_x) * quad::OWNX, y0 = (t / c->tiles_x) * quad::RW;
      const bool xe = !c->periodic[0] &&
          ((c->low[0] > 0 && x0 - quad::VEC < c->low[0]) ||
           (c->high[0] > 0 && x0 + quad::OWNX > nx - c->high[0]));
      int yrows = 0;
      for (int gy = y0 - 1; gy < y0 + quad::RW; gy++)
        if (!c->periodic[1] && gy >= 0 && gy < ny && (gy < c->low[1] || gy >= ny - c->high[1]))
          yrows++;
      const double base = 1.0 + 0.4 * xe + 1.15 * yrows / quad::WARPS;
      const int kbeg = c->runs[r], kend = c->runs[r + 1];
      double w = 0.0;
      for (int k = kbeg; k < kend; k++) w += base + (zslab(k) ? 0.95 : 0.0);
      if (kbeg > 0) w += 0.6 * (base + (zslab(kbeg - 1) ? 0.95 : 0.0));
      cost.push_back({-w, r * tiles + t});
    }
  std::stable_sort(cost.begin(), cost.end(),
                   [](const std::pair<double, int> &a, const std::pair<double, int> &b) {
                     return a.first < b.first;
                   });
  std::vector<int> order(cost.size());
  for (size_t i = 0; i < cost.size(); i++) order[i] = cost[i].second;
  return order;
}

// Empty source tables: every bucket empty.
int empty_sources(fdtd_ctx *c) {
  long long nb = (long long)c->tiles_x * c->tiles_y * c->n[2] + 1;
  std::vector<int> zero(nb, 0);
  release(c, c->hbucket);
  release(c, c->ebucket);
  c->hbucket = c->ebucket = nullptr;
  if (int r = alloc(c, (void **)&c->hbucket, nb * 4)) return r;
  if (int r = alloc(c, (void **)&c->ebucket, nb * 4)) return r;
  CUDA_TRY(c, copy(c, c->hbucket, zero.data(), nb * 4, cudaMemcpyHostToDevice));
  CUDA_TRY(c, copy(c, c->ebucket, zero.data(), nb * 4, cudaMemcpyHostToDevice));
  return 0;
}

template <typename T>
int run_impl(fdtd_ctx *c, long long steps, long long first) {
  if (!c->coeffs_set || !c->fields_set)
    return fail(c, FDTD_E_STATE, "upload the coefficients and the fields before a run");
  if (c->naux_laid != c->naux + c->nbloch)
    return fail(c, FDTD_E_STATE, "set the sources again after the plane waves");
  if (c->nbloch > 0)
    return fail(c, FDTD_E_STATE, "a context with Bloch couplings steps with fdtd_bloch_run");
  const int K = c->ring_k > 0 ? c->ring_k : 64;
  // the probes' record: grow to the run's steps
  if (c->nprobes > 0 && c->recorded + steps > c->record_cap) {
    long long cap = std::max<long long>(c->recorded + steps, 2 * c->record_cap);
    double *nr = nullptr;
    if (int r = alloc(c, (void **)&nr, (size_t)cap * c->nprobes * 8)) return r;
    if (c->record && c->recorded)
      CUDA_TRY(c, cudaMemcpyAsync(nr, c->record, (size_t)c->recorded * c->nprobes * 8,
                                  cudaMemcpyDeviceToDevice, c->stream));
    release(c, c->record);
    c->record = nr;
    c->record_cap = cap;
  }
  // one batch of `batch` steps from step index first + at (or *base when captured)
  auto enqueue_batch = [&](int batch, long long at, const long long *base) {
    if (c->nwaves > 0) {
      int total = c->nwaves * batch;
      waves_kernel<<<(total + 127) / 128, 128, 0, c->stream>>>(
          c->d_waves, c->d_point, c->nwaves, c->stride(), first + at, base, batch, c->dt,
          c->waves_h, c->waves_e);
      c->launches++;
    }
    if (c->naux_runs > 0) {
      aux_kernel<<<c->naux_runs, 1024, 0, c->stream>>>(c->d_aux, c->nwaves, c->stride(),
                                                       first + at, base, batch, c->dt,
                                                       c->waves_h, c->waves_e);
      c->launches++;
    }
    for (int m = 0; m < batch; m++) {
      StepArgs<T> A = step_args<T>(c);
      A.waves_h = c->waves_h + 2LL * m * c->stride();
      A.waves_e = c->waves_e + 2LL * m * c->stride();
      if (c->profiling) {
        if (c->events_used + 2 > c->events.size()) {
          for (int q = 0; q < 256; q++) {
            cudaEvent_t ev;
            cudaEventCreate(&ev);
            c->events.push_back(ev);
          }
        }
        cudaEventRecord(c->events[c->events_used++], c->stream);
        launch_step<T>(c, A);
        cudaEventRecord(c->events[c->events_used++], c->stream);
      } else {
        launch_step<T>(c, A);
      }
      c->launches += (c->quad && c->media) ? 2 : 1;
      c->parity = 1 - c->parity;
      long long gathered = c->nvalues + c->nprobes;
      if (gathered > 0) {
        T *row = c->nvalues ? (T *)c->ring + (long long)m * c->nvalues : nullptr;
        double *rec = c->nprobes ? c->record + (c->recorded + at + m) * c->nprobes : nullptr;
        gather_kernel<T><<<(unsigned)((gathered + 255) / 256), 256, 0, c->stream>>>(
            (const T *)c->e[c->parity], (const T *)c->h[c->parity], c->d_where, (int)c->nvalues,
            row, c->d_probes, c->nprobes, rec);
        c->launches++;
      }
    }
    if (c->nvalues > 0) {
      int total = c->nslots * batch;
      phase_kernel<<<(total + 127) / 128, 128, 0, c->stream>>>(c->d_omega, c->d_slot_field,
                                                                c->nslots, first + at, base,
                                                                batch, c->dt, c->phase);
      dft_kernel<T><<<(unsigned)((c->nvalues + 127) / 128), 128, 0, c->stream>>>(
          c->d_series, c->nseries, c->d_value_series, c->nvalues, (const T *)c->ring, batch,
          c->phase, c->nslots, c->sums);
      c->launches += 2;
    }
  };
  // whole batches replay a captured graph (K even: a batch leaves the current copy as it found
  // it), unless probes (their record rows move) or per-launch timing are asked for
  const bool graphs = !c->profiling && c->nprobes == 0 && K % 2 == 0;
  long long done = 0;
  while (done < steps) {
    const int batch = (int)std::min<long long>(K, steps - done);
    if (graphs && batch == K && c->warmed) {
      if (!c->d_base) {
        if (int r = alloc(c, (void **)&c->d_base, 8)) return r;
      }
      const int p = c->parity;
      if (!c->graph[p] || c->graph_layout[p] != c->layout) {
        if (c->graph[p]) cudaGraphExecDestroy(c->graph[p]);
        c->graph[p] = nullptr;
        cudaGraph_t g = nullptr;
        const long long before = c->launches;
        c->capturing = true;
        cudaError_t err = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
        if (err == cudaSuccess) {
          enqueue_batch(K, 0, c->d_base);
          err = cudaStreamEndCapture(c->stream, &g);
        }
        c->capturing = false;
        c->parity = p;  // the capture's bookkeeping flipped it K times
        if (err == cudaSuccess) err = cudaGraphInstantiate(&c->graph[p], g, 0);
        if (g) cudaGraphDestroy(g);
        if (err != cudaSuccess)
          return fail(c, FDTD_E_GPU, "capturing a batch of steps: %s", cudaGetErrorString(err));
        c->graph_kernels[p] = c->launches - before;
        c->launches = before;
        c->graph_layout[p] = c->layout;
      }
      set_base_kernel<<<1, 1, 0, c->stream>>>(c->d_base, first + done);
      CUDA_TRY(c, cudaGraphLaunch(c->graph[p], c->stream));
      c->launches += 1 + c->graph_kernels[p];
    } else {
      enqueue_batch(batch, done, nullptr);
      c->warmed = true;
    }
    done += batch;
  }
  c->recorded += steps;
  CUDA_TRY(c, cudaGetLastError());
  return 0;
}

// The probes' record grown to hold `steps` more steps.
int grow_record(fdtd_ctx *c, long long steps) {
  if (c->nprobes == 0 || c->recorded + steps <= c->record_cap) return 0;
  long long cap = std::max<long long>(c->recorded + steps, 2 * c->record_cap);
  double *nr = nullptr;
  if (int r = alloc(c, (void **)&nr, (size_t)cap * c->nprobes * 8)) return r;
  if (c->record && c->recorded)
    CUDA_TRY(c, cudaMemcpyAsync(nr, c->record, (size_t)c->recorded * c->nprobes * 8,
                                cudaMemcpyDeviceToDevice, c->stream));
  release(c, c->record);
  c->record = nr;
  c->record_cap = cap;
  return 0;
}

// A complex run (src/fdtd.rs:1319-1343, src/fdtd/bloch.rs): the real part `a` and the imaginary
// part `b`, two contexts of one grid, stepped together on a's stream: each step, H's couplings
// across the Bloch sides from both parts' E (subtracted in the step kernels after H's sources),
// a's step and b's, E's couplings from both parts' new H, the media (b's, then a's), then each
// part's probes and the transforms of a's monitors taken whole (real and imaginary parts).
template <typename T>
int bloch_impl(fdtd_ctx *a, fdtd_ctx *b, const std::vector<WrapDev> &hw,
               const std::vector<WrapDev> &ew, const std::vector<int> &estart, long long steps,
               long long first) {
  for (fdtd_ctx *c : {a, b}) {
    if (!c->coeffs_set || !c->fields_set)
      return fail(a, FDTD_E_STATE, "upload both parts' coefficients and fields before a run");
    if (c->naux_laid != c->naux + c->nbloch)
      return fail(a, FDTD_E_STATE, "set the sources again after the Bloch slots");
    if (c->media && !c->quad)
      return fail(a, FDTD_E_INVALID,
                  "Bloch sides with dispersive media step on grids whose nx is a multiple of 4");
  }
  if (a->N != b->N || a->precision != b->precision || a->nbloch != b->nbloch)
    return fail(a, FDTD_E_INVALID, "the two parts of a complex run differ");
  CUDA_TRY(a, cudaStreamSynchronize(b->stream));
  const cudaStream_t st = a->stream;
  const int K = a->ring_k > 0 ? a->ring_k : 64;
  if (int r = grow_record(a, steps)) return r;
  if (int r = grow_record(b, steps)) return fail(a, r, "%s", b->error.c_str());
  // the couplings and the imaginary part's ring, for this run
  WrapDev *dh = nullptr, *de = nullptr;
  int *dstart = nullptr;
  T *ring_im = nullptr;
  auto freed = [&]() {
    release(a, dh);
    release(a, de);
    release(a, dstart);
    release(a, ring_im);
  };
  if (int r = alloc(a, (void **)&dh, std::max<size_t>(hw.size(), 1) * sizeof(WrapDev))) return r;
  if (int r = alloc(a, (void **)&de, std::max<size_t>(ew.size(), 1) * sizeof(WrapDev))) {
    freed();
    return r;
  }
  if (int r = alloc(a, (void **)&dstart, estart.size() * 4)) {
    freed();
    return r;
  }
  if (a->nvalues > 0)
    if (int r = alloc(a, (void **)&ring_im, (size_t)K * a->nvalues * a->elem)) {
      freed();
      return r;
    }
  cudaError_t e = cudaSuccess;
  if (!hw.empty()) e = copy(a, dh, hw.data(), hw.size() * sizeof(WrapDev), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !ew.empty())
    e = copy(a, de, ew.data(), ew.size() * sizeof(WrapDev), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = copy(a, dstart, estart.data(), estart.size() * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    freed();
    return fail(a, FDTD_E_GPU, "the Bloch couplings: %s", cudaGetErrorString(e));
  }
  const int nvals_e = (int)estart.size() - 1;
  // b's step launches on a's stream for the run (its kernels and a's must be ordered)
  const cudaStream_t b_stream = b->stream;
  b->stream = st;
  long long done = 0;
  while (done < steps) {
    const int batch = (int)std::min<long long>(K, steps - done);
    for (fdtd_ctx *c : {a, b})
      if (c->nwaves > 0) {
        const int total = c->nwaves * batch;
        waves_kernel<<<(total + 127) / 128, 128, 0, st>>>(c->d_waves, c->d_point, c->nwaves,
                                                          c->stride(), first + done, nullptr,
                                                          batch, c->dt, c->waves_h, c->waves_e);
      }
    for (int m = 0; m < batch; m++) {
      const long long row_a = 2LL * m * a->stride(), row_b = 2LL * m * b->stride();
      if (!hw.empty())
        bloch_h_kernel<T><<<(unsigned)((hw.size() + 127) / 128), 128, 0, st>>>(
            dh, (int)hw.size(), (const T *)a->e[a->parity], (const T *)b->e[b->parity], a->N,
            a->dt, a->waves_h + row_a + 2LL * (a->nwaves + a->naux),
            b->waves_h + row_b + 2LL * (b->nwaves + b->naux));
      StepArgs<T> A = step_args<T>(a), B = step_args<T>(b);
      A.waves_h = a->waves_h + row_a;
      A.waves_e = a->waves_e + row_a;
      B.waves_h = b->waves_h + row_b;
      B.waves_e = b->waves_e + row_b;
      launch_step<T>(a, A, false);
      launch_step<T>(b, B, false);
      a->parity = 1 - a->parity;
      b->parity = 1 - b->parity;
      if (nvals_e > 0)
        bloch_e_kernel<T><<<(unsigned)((nvals_e + 127) / 128), 128, 0, st>>>(
            de, dstart, nvals_e, (const T *)a->h[a->parity], (const T *)b->h[b->parity], a->N,
            (T *)a->e[a->parity], (T *)b->e[b->parity]);
      if (b->media && b->quad)
        ade_kernel<T><<<(unsigned)((B.media.members + 255) / 256), 256, 0, st>>>(B);
      if (a->media && a->quad)
        ade_kernel<T><<<(unsigned)((A.media.members + 255) / 256), 256, 0, st>>>(A);
      // b's probes, and a's monitored values of b into the imaginary ring; then a's own
      const long long count = a->nvalues;
      if (count + b->nprobes > 0)
        gather_kernel<T><<<(unsigned)((count + b->nprobes + 255) / 256), 256, 0, st>>>(
            (const T *)b->e[b->parity], (const T *)b->h[b->parity], a->d_where, (int)count,
            count ? ring_im + (long long)m * count : nullptr, b->d_probes, b->nprobes,
            b->nprobes ? b->record + (b->recorded + done + m) * b->nprobes : nullptr);
      if (count + a->nprobes > 0)
        gather_kernel<T><<<(unsigned)((count + a->nprobes + 255) / 256), 256, 0, st>>>(
            (const T *)a->e[a->parity], (const T *)a->h[a->parity], a->d_where, (int)count,
            count ? (T *)a->ring + (long long)m * count : nullptr, a->d_probes, a->nprobes,
            a->nprobes ? a->record + (a->recorded + done + m) * a->nprobes : nullptr);
    }
    if (a->nvalues > 0) {
      const int total = a->nslots * batch;
      phase_kernel<<<(total + 127) / 128, 128, 0, st>>>(a->d_omega, a->d_slot_field, a->nslots,
                                                        first + done, nullptr, batch, a->dt,
                                                        a->phase);
      dft_complex_kernel<T><<<(unsigned)((a->nvalues + 127) / 128), 128, 0, st>>>(
          a->d_series, a->d_value_series, a->nvalues, (const T *)a->ring, ring_im, batch,
          a->phase, a->nslots, a->sums);
    }
    done += batch;
  }
  b->stream = b_stream;
  e = cudaStreamSynchronize(st);
  freed();
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return fail(a, FDTD_E_GPU, "a complex run: %s", cudaGetErrorString(e));
  a->recorded += steps;
  b->recorded += steps;
  a->generation++;
  b->generation++;
  return 0;
}

}  // namespace

extern "C" {

int fdtd_set_bloch_slots(fdtd_ctx *c, int32_t nslots) {
  if (!c || nslots < 0) return FDTD_E_INVALID;
  c->generation++;
  c->layout++;
  c->nbloch = nslots;
  return 0;
}

int fdtd_bloch_run(fdtd_ctx *re, fdtd_ctx *im, int32_t nwraps, const fdtd_wrap *wraps,
                   int64_t steps, int64_t first_step) {
  if (!re || !im || re == im || nwraps < 0 || (nwraps > 0 && !wraps)) return FDTD_E_INVALID;
  if (steps < 0) return fail(re, FDTD_E_INVALID, "a negative number of steps");
  if (steps == 0) return 0;
  // H's couplings each in their own slot; E's grouped by value, each value's in the given order
  std::vector<WrapDev> hw, ew;
  std::map<std::pair<int, long long>, std::vector<WrapDev>> byvalue;
  std::vector<std::pair<int, long long>> order;
  for (int32_t k = 0; k < nwraps; k++) {
    const fdtd_wrap &x = wraps[k];
    if (x.comp < 0 || x.comp > 2 || x.from_comp < 0 || x.from_comp > 2 || x.r < 0 ||
        x.r >= re->N || x.q < 0 || x.q >= re->N || (x.field == 1 && (x.slot < 0 ||
        x.slot >= re->nbloch)))
      return fail(re, FDTD_E_INVALID, "Bloch coupling %d is outside the grid", (int)k);
    WrapDev d{x.r, x.q, x.comp, x.from_comp, x.phase_re, x.phase_im, x.s, x.cb, x.slot, 0};
    if (x.field == 1) {
      hw.push_back(d);
    } else {
      auto key = std::make_pair((int)x.comp, (long long)x.r);
      if (!byvalue.count(key)) order.push_back(key);
      byvalue[key].push_back(d);
    }
  }
  std::vector<int> start{0};
  for (auto &key : order) {
    for (auto &d : byvalue[key]) ew.push_back(d);
    start.push_back((int)ew.size());
  }
  re->launches = 0;
  return re->precision == 64 ? bloch_impl<double>(re, im, hw, ew, start, steps, first_step)
                             : bloch_impl<float>(re, im, hw, ew, start, steps, first_step);
}

const char *fdtd_last_error(const fdtd_ctx *ctx) { return ctx ? ctx->error.c_str() : "no context"; }

int fdtd_create(const fdtd_grid *grid, double dt, const double step[3], const double *factor_e,
                const double *factor_h, const fdtd_slab *slabs, int32_t nslabs, int32_t precision,
                size_t hbm_budget, fdtd_ctx **out) {
  if (!out || !grid || !step || !factor_e || !factor_h) return FDTD_E_INVALID;
  *out = nullptr;
  fdtd_ctx *c = new fdtd_ctx();
  c->precision = precision == 64 ? 64 : 32;
  c->elem = c->precision == 64 ? 8 : 4;
  c->budget = hbm_budget;
  c->dt = dt;
  long long N = 1;
  for (int a = 0; a < 3; a++) {
    if (grid->n[a] <= 0 || grid->n[a] > (1 << 30)) {
      fail(c, FDTD_E_INVALID, "the grid needs cells along every axis, got %lld along axis %d",
           (long long)grid->n[a], a);
      *out = c;
      return FDTD_E_INVALID;
    }
    c->n[a] = (int)grid->n[a];
    c->periodic[a] = grid->periodic[a] ? 1 : 0;
    c->low[a] = c->periodic[a] ? 0 : (int)grid->low[a];
    c->high[a] = c->periodic[a] ? 0 : (int)grid->high[a];
    if (!c->periodic[a] && (c->low[a] < 0 || c->high[a] < 0 || c->low[a] + c->high[a] >= c->n[a])) {
      fail(c, FDTD_E_INVALID, "CPMLs of %d and %d cells leave nothing of %d cells", c->low[a],
           c->high[a], c->n[a]);
      *out = c;
      return FDTD_E_INVALID;
    }
    c->step[a] = step[a];
    N *= c->n[a];
  }
  c->N = N;
  *out = c;
  if (!(dt > 0.0 && std::isfinite(dt)))
    return fail(c, FDTD_E_INVALID, "the time step must be positive, got %g", dt);
  CUDA_TRY(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  size_t E = c->elem;
  for (int p = 0; p < 2; p++) {
    if (int r = alloc(c, &c->e[p], 3 * N * E)) return r;
    if (int r = alloc(c, &c->h[p], 3 * N * E)) return r;
  }
  if (int r = alloc(c, &c->cb, 3 * N * E)) return r;
  long long nf = (long long)c->n[0] + c->n[1] + c->n[2];
  if (int r = alloc(c, &c->fe, nf * E)) return r;
  if (int r = alloc(c, &c->fh, nf * E)) return r;
  if (int r = upload(c, c->fe, factor_e, nf)) return r;
  if (int r = upload(c, c->fh, factor_h, nf)) return r;
  // the slabs: psi for E in place, for H in two copies; their coefficients in one table
  memset(c->table, 0, sizeof c->table);
  std::vector<double> coefs;
  for (int s = 0; s < nslabs; s++) {
    const fdtd_slab &sl = slabs[s];
    int w = sl.axis, comp = sl.component, field = sl.field;
    if (w < 0 || w > 2 || comp < 0 || comp > 2 || field < 0 || field > 1 || comp == w ||
        c->periodic[w] || sl.count <= 0 || sl.from < 0 || sl.from + sl.count > c->n[w])
      return fail(c, FDTD_E_INVALID, "slab %d is not a CPML slab of this grid", s);
    int side;
    if (sl.from == 0 && sl.count == c->low[w]) side = 0;
    else if (sl.from + sl.count == c->n[w] && sl.count == c->high[w]) side = 1;
    else return fail(c, FDTD_E_INVALID, "slab %d does not match the grid's CPML cells", s);
    DeviceSlab d;
    d.field = field;
    d.comp = comp;
    d.axis = w;
    d.from = sl.from;
    d.count = sl.count;
    d.pf = w == 0 ? sl.from / 4 * 4 : sl.from;
    d.pw = w == 0 ? (sl.from + sl.count + 3) / 4 * 4 - d.pf : sl.count;
    d.size = d.pw * (N / c->n[w]);
    d.coef = (long long)coefs.size();
    // each slab's psi starts on a 16-element boundary, so a row of four values is one aligned
    // vector in f32 and two in f64
    long long &len = field == 1 ? c->psi_h_len : c->psi_e_len;
    d.psi = (len + 15) / 16 * 16;
    len = d.psi + d.size;
    for (long long q = 0; q < sl.count; q++) coefs.push_back(sl.b[q]);
    for (long long q = 0; q < sl.count; q++) coefs.push_back(sl.a[q]);
    c->slabs.push_back(d);
    SlabEntry &t = c->table[field][comp][w][side];
    t.from = (int)sl.from;
    t.count = (int)sl.count;
    t.psi = d.psi;
    t.coef = (int)d.coef;
    t.pf = (int)d.pf;
    t.pw = (int)d.pw;
  }
  if (int r = alloc(c, &c->coefs, coefs.size() * E)) return r;
  if (int r = upload(c, c->coefs, coefs.data(), (long long)coefs.size())) return r;
  for (int p = 0; p < 2; p++)
    if (int r = alloc(c, &c->psi_h[p], c->psi_h_len * E)) return r;
  if (int r = alloc(c, &c->psi_e, c->psi_e_len * E)) return r;
  CUDA_TRY(c, cudaMemsetAsync(c->psi_h[0], 0, c->psi_h_len * E, c->stream));
  CUDA_TRY(c, cudaMemsetAsync(c->psi_h[1], 0, c->psi_h_len * E, c->stream));
  CUDA_TRY(c, cudaMemsetAsync(c->psi_e, 0, c->psi_e_len * E, c->stream));
  // launch shape: tiles of TX x TY, and the z planes cut into runs so that the grid holds
  // several CTAs per SM
  c->tiles_x = (c->n[0] + TX - 1) / TX;
  c->tiles_y = (c->n[1] + TY - 1) / TY;
  int sms = 148;
  {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  c->sms = sms;
  // the slabs' d/h: in f32 by the product form where it is checked to give division's bits
  for (int a = 0; a < 3; a++) {
    if (c->precision == 64) {
      c->inv_step[a] = 1.0 / c->step[a];
      c->fast_div[a] = 0;
      continue;
    }
    const float h = (float)c->step[a], r = (float)(1.0 / (double)h);
    c->inv_step[a] = r;
    if (int q = division_checked(c, h, r, &c->fast_div[a])) return q;
  }
  {
    const char *force = getenv("PHOTONOXIDE_FDTD_KERNEL");
    // the quad kernel takes four places along x at once: nx a multiple of 4, and no group of
    // four holding places of both x CPMLs (an interior narrower than the group); its offsets
    // within a plane are ints
    const bool quad_ok = c->n[0] % 4 == 0 &&
        !(c->low[0] > 0 && c->high[0] > 0 && (c->low[0] - 1) / 4 == (c->n[0] - c->high[0]) / 4) &&
        (long long)c->n[0] * c->n[1] < (1LL << 31);
    std::string kind = force ? force : (quad_ok ? "quad" : "row");
    if (kind == "quad" && !quad_ok) kind = "row";
    c->quad = kind == "quad";
    c->row = kind == "row";
    c->staged = kind == "staged" && (c->n[0] % (16 / (int)c->elem) == 0);
  }
  if (c->row) {
    c->tile_w = rowstep::OWN;
    c->tile_h = rowstep::RW;
    c->loc_w = rowstep::SEG;
    c->loc_x = 1;
    c->e_tile = false;
  } else if (c->quad) {
    c->tile_w = quad::OWNX;
    c->tile_h = quad::RW;
    c->loc_w = quad::ROW;
    c->loc_x = quad::VEC;
    c->e_tile = false;
  }
  c->tiles_x = (c->n[0] + c->tile_w - 1) / c->tile_w;
  c->tiles_y = (c->n[1] + c->tile_h - 1) / c->tile_h;
  long long tiles = (long long)c->tiles_x * c->tiles_y;
  // z cut into runs so that the CTAs fill the device about three times over: fewer, longer runs
  // recompute fewer planes of H, and the two short interior runs (quad_runs), taken last, keep
  // the step's end short. On the 3D MMI (145 tiles) 7 runs timed best: 0.225 ms a step against
  // 0.228 with 9 or 10, 0.231 with 8, 0.239 with 6 and 0.243 with 13.
  long long want = 6LL * sms;
  int chunks = (int)std::max<long long>(1, (want + tiles - 1) / tiles);
  chunks = std::min(chunks, std::max(1, c->n[2] / 4));
  const char *zc = getenv("PHOTONOXIDE_FDTD_ZCHUNKS");
  if (zc) chunks = std::max(1, atoi(zc));
  chunks = std::min(chunks, c->n[2]);
  c->zchunk = (c->n[2] + chunks - 1) / chunks;
  c->zchunks = (c->n[2] + c->zchunk - 1) / c->zchunk;
  if (c->quad) {
    c->zchunks = quad_runs(c, chunks);
    const std::vector<int> order = quad_order(c);
    if (int r = alloc(c, (void **)&c->order, order.size() * 4)) return r;
    CUDA_TRY(c, copy(c, c->order, order.data(), order.size() * 4, cudaMemcpyHostToDevice));
  }
  if (int r = empty_sources(c)) return r;
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return 0;
}

void fdtd_destroy(fdtd_ctx *c) {
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (cudaEvent_t ev : c->events) cudaEventDestroy(ev);
  for (int p = 0; p < 2; p++)
    if (c->graph[p]) cudaGraphExecDestroy(c->graph[p]);
  if (c->stream) {
    for (void *p : c->allocations) cudaFreeAsync(p, c->stream);
    cudaStreamSynchronize(c->stream);
    cudaStreamDestroy(c->stream);
  }
  delete c;
}

int fdtd_upload_coeffs(fdtd_ctx *c, const double *ca, const double *cb) {
  if (!c || !cb) return fail(c, FDTD_E_INVALID, "cb is needed");
  c->generation++;
  c->layout++;
  c->lossless = ca == nullptr;
  if (ca) {
    if (!c->ca)
      if (int r = alloc(c, &c->ca, 3 * c->N * c->elem)) return r;
    if (int r = upload(c, c->ca, ca, 3 * c->N)) return r;
  }
  if (int r = upload(c, c->cb, cb, 3 * c->N)) return r;
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));  // the host arrays are the caller's again
  c->coeffs_set = true;
  return 0;
}

int fdtd_upload_fields(fdtd_ctx *c, const double *e, const double *h, const double *const *psi) {
  if (!c) return FDTD_E_INVALID;
  c->generation++;
  c->parity = 0;
  size_t E = c->elem;
  if (e) { if (int r = upload(c, c->e[0], e, 3 * c->N)) return r; }
  else CUDA_TRY(c, cudaMemsetAsync(c->e[0], 0, 3 * c->N * E, c->stream));
  if (h) { if (int r = upload(c, c->h[0], h, 3 * c->N)) return r; }
  else CUDA_TRY(c, cudaMemsetAsync(c->h[0], 0, 3 * c->N * E, c->stream));
  for (size_t s = 0; s < c->slabs.size(); s++) {
    const DeviceSlab &d = c->slabs[s];
    void *base = d.field == 1 ? c->psi_h[0] : c->psi_e;
    void *dst = (char *)base + d.psi * E;
    if (psi && psi[s]) {
      if (d.axis == 0 && (d.pf != d.from || d.pw != d.count)) {
        // the reference's rows of `count` values into the padded rows
        long long rows = d.size / d.pw;
        std::vector<double> padded(d.size, 0.0);
        for (long long r = 0; r < rows; r++)
          for (long long q = 0; q < d.count; q++)
            padded[r * d.pw + (d.from - d.pf) + q] = psi[s][r * d.count + q];
        if (int r = upload(c, dst, padded.data(), d.size)) return r;
      } else if (int r = upload(c, dst, psi[s], d.size)) {
        return r;
      }
    } else {
      CUDA_TRY(c, cudaMemsetAsync(dst, 0, d.size * E, c->stream));
    }
  }
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->fields_set = true;
  return 0;
}

int fdtd_download_fields(fdtd_ctx *c, double *e, double *h, double *const *psi) {
  if (!c) return FDTD_E_INVALID;
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (e) if (int r = download(c, e, c->e[c->parity], 3 * c->N)) return r;
  if (h) if (int r = download(c, h, c->h[c->parity], 3 * c->N)) return r;
  if (psi)
    for (size_t s = 0; s < c->slabs.size(); s++) {
      if (!psi[s]) continue;
      const DeviceSlab &d = c->slabs[s];
      const void *base = d.field == 1 ? c->psi_h[c->parity] : c->psi_e;
      const void *src = (const char *)base + d.psi * c->elem;
      if (d.axis == 0 && (d.pf != d.from || d.pw != d.count)) {
        long long rows = d.size / d.pw;
        std::vector<double> padded(d.size);
        if (int r = download(c, padded.data(), src, d.size)) return r;
        for (long long r = 0; r < rows; r++)
          for (long long q = 0; q < d.count; q++)
            psi[s][r * d.count + q] = padded[r * d.pw + (d.from - d.pf) + q];
      } else if (int r = download(c, psi[s], src, d.size)) {
        return r;
      }
    }
  return 0;
}

int fdtd_set_sources(fdtd_ctx *c, int32_t nwaves, const fdtd_waveform *waves, int64_t ninj,
                     const fdtd_injection *inj) {
  if (!c) return FDTD_E_INVALID;
  c->generation++;
  c->layout++;
  int nx = c->n[0], ny = c->n[1], nz = c->n[2];
  std::vector<int> point(std::max(nwaves, 1), -1);
  for (int64_t q = 0; q < ninj; q++) {
    const fdtd_injection &x = inj[q];
    const int slots = x.point == 2 ? c->naux + c->nbloch : nwaves;  // a coupling's slot
    if (x.field < 0 || x.field > 1 || x.component < 0 || x.component > 2 || x.r < 0 ||
        x.r >= c->N || x.emitter < 0 || x.emitter >= slots || !std::isfinite(x.a_re) ||
        !std::isfinite(x.a_im) || x.point < 0 || x.point > 2)
      return fail(c, FDTD_E_INVALID, "injection %lld is outside the grid or not finite",
                  (long long)q);
    if (x.point == 2) continue;
    int want = x.point ? 1 : 0;
    if (point[x.emitter] >= 0 && point[x.emitter] != want)
      return fail(c, FDTD_E_INVALID, "emitter %d is both a point source and a current", x.emitter);
    point[x.emitter] = want;
  }
  for (int w = 0; w < nwaves; w++)
    if (waves[w].kind < 0 || waves[w].kind > 2)
      return fail(c, FDTD_E_INVALID, "waveform %d has no kind %d", w, waves[w].kind);
  c->src_waves.assign(waves, waves + std::max(nwaves, 0));
  c->src_inj.assign(inj, inj + std::max<int64_t>(ninj, 0));
  // Group by value in CPU order (Resident::plan, resident.rs:546-590), then by (tile, plane):
  // an H value also goes to the tiles whose low halo row or column it is.
  struct Item { long long key; int local; int comp; std::vector<int> entries; };
  std::vector<Entry> entries;
  std::vector<std::vector<Item>> per_field(2);
  for (int f = 0; f < 2; f++) {
    std::vector<long long> order;
    std::vector<std::vector<int>> lists;
    std::vector<long long> places;
    // value -> position in order
    std::unordered_map<long long, int> index;
    for (int64_t q = 0; q < ninj; q++) {
      const fdtd_injection &x = inj[q];
      if (x.field != f) continue;
      long long place = (long long)x.component * c->N + x.r;
      int at = -1;
      auto found = index.find(place);
      if (found != index.end()) at = found->second;
      if (at < 0) {
        at = (int)places.size();
        index[place] = at;
        places.push_back(place);
        lists.emplace_back();
      }
      Entry en;
      en.are = x.a_re;
      en.aim = x.a_im;
      en.emitter = x.point == 2 ? nwaves + x.emitter : x.emitter;
      en.pad = x.point == 2 ? 1 : 0;
      lists[at].push_back((int)entries.size());
      entries.push_back(en);
    }
    for (size_t g = 0; g < places.size(); g++) {
      int comp = (int)(places[g] / c->N);
      long long r = places[g] % c->N;
      int i = (int)(r % nx), j = (int)((r / nx) % ny), k = (int)(r / ((long long)nx * ny));
      const int tw = c->tile_w, th = c->tile_h;
      // a place's number in its tile (see fdtd_ctx::loc_w)
      const int hw = c->loc_w, lx0 = c->loc_x;
      int tx = i / tw, ty = j / th;
      auto push = [&](int ttx, int tty, int lx, int ly, int width) {
        Item it;
        it.key = ((long long)(tty * c->tiles_x + ttx)) * nz + k;
        it.local = ly * width + lx;
        it.comp = comp;
        it.entries = lists[g];
        per_field[f].push_back(it);
      };
      if (f == 0) {
        if (!c->e_tile) push(tx, ty, i - tx * tw + lx0, j - ty * th + 1, hw);
        else push(tx, ty, i - tx * tw, j - ty * th, TX);
      } else {
        push(tx, ty, i - tx * tw + lx0, j - ty * th + 1, hw);
        // the tiles whose low halo this value is: next along x, next along y (wrapping on a
        // periodic axis), and the diagonal one
        int txn = -1, tyn = -1;
        if (i == (tx + 1) * tw - 1 && (tx + 1) < c->tiles_x) txn = tx + 1;
        if (c->periodic[0] && i == nx - 1) txn = 0;
        if (j == (ty + 1) * th - 1 && (ty + 1) < c->tiles_y) tyn = ty + 1;
        if (c->periodic[1] && j == ny - 1) tyn = 0;
        if (txn >= 0) push(txn, ty, lx0 - 1, j - ty * th + 1, hw);
        if (tyn >= 0) push(tx, tyn, i - tx * tw + lx0, 0, hw);
        if (txn >= 0 && tyn >= 0) push(txn, tyn, lx0 - 1, 0, hw);
      }
    }
  }
  long long nb = (long long)c->tiles_x * c->tiles_y * nz + 1;
  std::vector<Entry> ordered_entries;
  std::vector<Group> groups[2];
  std::vector<int> buckets[2];
  for (int f = 0; f < 2; f++) {
    auto &items = per_field[f];
    std::stable_sort(items.begin(), items.end(),
                     [](const Item &a, const Item &b) { return a.key < b.key; });
    buckets[f].assign(nb, 0);
    for (auto &it : items) {
      Group g;
      g.local = it.local;
      g.comp = it.comp;
      g.first = (int)ordered_entries.size();
      g.count = (int)it.entries.size();
      for (int e : it.entries) ordered_entries.push_back(entries[e]);
      groups[f].push_back(g);
      buckets[f][it.key + 1]++;
    }
    for (long long b = 1; b < nb; b++) buckets[f][b] += buckets[f][b - 1];
  }
  release(c, c->hbucket); release(c, c->ebucket); release(c, c->hgroups); release(c, c->egroups);
  release(c, c->entries); release(c, c->d_waves); release(c, c->d_point);
  release(c, c->waves_h); release(c, c->waves_e);
  c->hbucket = c->ebucket = nullptr;
  c->hgroups = c->egroups = nullptr;
  c->entries = nullptr;
  c->d_waves = nullptr;
  c->d_point = nullptr;
  c->waves_h = c->waves_e = nullptr;
  if (int r = alloc(c, (void **)&c->hbucket, nb * 4)) return r;
  if (int r = alloc(c, (void **)&c->ebucket, nb * 4)) return r;
  if (int r = alloc(c, (void **)&c->hgroups, groups[1].size() * sizeof(Group))) return r;
  if (int r = alloc(c, (void **)&c->egroups, groups[0].size() * sizeof(Group))) return r;
  if (int r = alloc(c, (void **)&c->entries, ordered_entries.size() * sizeof(Entry))) return r;
  CUDA_TRY(c, copy(c, c->hbucket, buckets[1].data(), nb * 4, cudaMemcpyHostToDevice));
  CUDA_TRY(c, copy(c, c->ebucket, buckets[0].data(), nb * 4, cudaMemcpyHostToDevice));
  if (!groups[1].empty())
    CUDA_TRY(c, copy(c, c->hgroups, groups[1].data(), groups[1].size() * sizeof(Group), cudaMemcpyHostToDevice));
  if (!groups[0].empty())
    CUDA_TRY(c, copy(c, c->egroups, groups[0].data(), groups[0].size() * sizeof(Group), cudaMemcpyHostToDevice));
  if (!ordered_entries.empty())
    CUDA_TRY(c, copy(c, c->entries, ordered_entries.data(), ordered_entries.size() * sizeof(Entry), cudaMemcpyHostToDevice));
  c->nwaves = nwaves;
  c->naux_laid = c->naux + c->nbloch;
  if (c->stride() > 0) {
    const int K = c->ring_k > 0 ? c->ring_k : 64;
    if (int r = alloc(c, (void **)&c->waves_h, (size_t)K * c->stride() * 16)) return r;
    if (int r = alloc(c, (void **)&c->waves_e, (size_t)K * c->stride() * 16)) return r;
    c->wave_batch = K;
  }
  if (nwaves > 0) {
    std::vector<Wave> w(nwaves);
    for (int q = 0; q < nwaves; q++) {
      w[q].kind = waves[q].kind;
      for (int p = 0; p < 5; p++) w[q].p[p] = waves[q].p[p];
      if (point[q] < 0) point[q] = 0;
    }
    if (int r = alloc(c, (void **)&c->d_waves, nwaves * sizeof(Wave))) return r;
    if (int r = alloc(c, (void **)&c->d_point, nwaves * sizeof(int))) return r;
    CUDA_TRY(c, copy(c, c->d_waves, w.data(), nwaves * sizeof(Wave), cudaMemcpyHostToDevice));
    CUDA_TRY(c, copy(c, c->d_point, point.data(), nwaves * sizeof(int), cudaMemcpyHostToDevice));
  }
  return 0;
}

int fdtd_set_plane_waves(fdtd_ctx *c, int32_t count, const fdtd_plane_wave *w) {
  if (!c) return FDTD_E_INVALID;
  if (count < 0 || (count > 0 && !w)) return fail(c, FDTD_E_INVALID, "no plane waves given");
  for (int32_t n = 0; n < count; n++) {
    const fdtd_plane_wave &x = w[n];
    long long reach = 0;
    for (int a = 0; a < 3; a++) reach = std::max<long long>(reach, std::llabs(x.g[a]));
    bool ok = x.len > 0 && x.pad >= reach && 2 * x.pad < x.len && x.ca && x.cb && x.da && x.db &&
              x.nsheet >= 0 && x.nslots >= 0 && x.wave.kind >= 0 && x.wave.kind <= 2;
    for (int a = 0; a < 3 && ok; a++) ok = x.g[a] == 0 || x.steps[a] > 0.0;
    for (int q = 0; q < x.nsheet && ok; q++)
      ok = x.sheet_comp[q] >= 0 && x.sheet_comp[q] < 3 && x.sheet_i[q] >= 0 &&
           x.sheet_i[q] < x.len;
    for (int q = 0; q < x.nslots && ok; q++)
      ok = (x.slot_field[q] == 0 || x.slot_field[q] == 1) && x.slot_comp[q] >= 0 &&
           x.slot_comp[q] < 3 && x.slot_i[q] >= 0 && x.slot_i[q] < x.len;
    if (!ok) return fail(c, FDTD_E_INVALID, "plane wave %d's run is malformed", (int)n);
  }
  c->generation++;
  c->layout++;
  for (void *p : c->aux_memory) release(c, p);
  c->aux_memory.clear();
  c->aux.clear();
  release(c, c->d_aux);
  c->d_aux = nullptr;
  c->naux_runs = 0;
  c->naux = 0;
  auto put = [&](const void *src, size_t bytes, void **dst) -> int {
    if (int r = alloc(c, dst, bytes)) return r;
    c->aux_memory.push_back(*dst);
    if (src) CUDA_TRY(c, copy(c, *dst, src, bytes, cudaMemcpyHostToDevice));
    else CUDA_TRY(c, cudaMemsetAsync(*dst, 0, bytes, c->stream));
    return 0;
  };
  int slots = 0;
  for (int32_t n = 0; n < count; n++) {
    const fdtd_plane_wave &x = w[n];
    AuxDev d;
    d.len = x.len;
    d.pad = x.pad;
    for (int a = 0; a < 3; a++) {
      d.g[a] = x.g[a];
      d.steps[a] = x.steps[a];
    }
    const size_t L = (size_t)x.len * 8;
    void *p = nullptr;
    if (int r = put(x.e0, 3 * L, &p)) return r;
    d.e = (double *)p;
    if (int r = put(x.h0, 3 * L, &p)) return r;
    d.h = (double *)p;
    if (int r = put(x.ca, L, &p)) return r;
    d.ca = (const double *)p;
    if (int r = put(x.cb, L, &p)) return r;
    d.cb = (const double *)p;
    if (int r = put(x.da, L, &p)) return r;
    d.da = (const double *)p;
    if (int r = put(x.db, L, &p)) return r;
    d.db = (const double *)p;
    d.nsheet = x.nsheet;
    std::vector<int> sc(x.sheet_comp, x.sheet_comp + x.nsheet);
    if (int r = put(sc.data(), sc.size() * 4, &p)) return r;
    d.sheet_comp = (const int *)p;
    if (int r = put(x.sheet_i, (size_t)x.nsheet * 8, &p)) return r;
    d.sheet_i = (const long long *)p;
    if (int r = put(x.sheet_j, (size_t)x.nsheet * 8, &p)) return r;
    d.sheet_j = (const double *)p;
    d.wave.kind = x.wave.kind;
    for (int q = 0; q < 5; q++) d.wave.p[q] = x.wave.p[q];
    d.nslots = x.nslots;
    d.slot0 = slots;
    std::vector<int> sf(x.slot_field, x.slot_field + x.nslots),
        sp(x.slot_comp, x.slot_comp + x.nslots);
    if (int r = put(sf.data(), sf.size() * 4, &p)) return r;
    d.slot_field = (const int *)p;
    if (int r = put(sp.data(), sp.size() * 4, &p)) return r;
    d.slot_comp = (const int *)p;
    if (int r = put(x.slot_i, (size_t)x.nslots * 8, &p)) return r;
    d.slot_i = (const long long *)p;
    slots += x.nslots;
    c->aux.push_back(d);
  }
  if (count > 0) {
    if (int r = alloc(c, (void **)&c->d_aux, count * sizeof(AuxDev))) return r;
    CUDA_TRY(c, copy(c, c->d_aux, c->aux.data(), count * sizeof(AuxDev), cudaMemcpyHostToDevice));
  }
  c->naux_runs = count;
  c->naux = slots;
  return 0;
}

int fdtd_plane_wave_state(fdtd_ctx *c, int32_t n, double *e, double *h) {
  if (!c) return FDTD_E_INVALID;
  if (n < 0 || n >= c->naux_runs) return fail(c, FDTD_E_INVALID, "no plane wave %d", (int)n);
  const AuxDev &d = c->aux[n];
  if (e) CUDA_TRY(c, copy(c, e, d.e, (size_t)d.len * 24, cudaMemcpyDeviceToHost));
  if (h) CUDA_TRY(c, copy(c, h, d.h, (size_t)d.len * 24, cudaMemcpyDeviceToHost));
  return 0;
}

int fdtd_set_probes(fdtd_ctx *c, int32_t n, const int32_t *field, const int32_t *component,
                    const int64_t *r) {
  if (!c) return FDTD_E_INVALID;
  c->generation++;
  c->layout++;
  std::vector<long long> w(std::max(n, 1));
  for (int p = 0; p < n; p++) {
    if (field[p] < 0 || field[p] > 1 || component[p] < 0 || component[p] > 2 || r[p] < 0 ||
        r[p] >= c->N)
      return fail(c, FDTD_E_INVALID, "probe %d is outside the grid", p);
    w[p] = ((long long)field[p] << 62) | ((long long)component[p] * c->N + r[p]);
  }
  release(c, c->d_probes);
  release(c, c->record);
  c->d_probes = nullptr;
  c->record = nullptr;
  c->record_cap = c->recorded = 0;
  c->nprobes = n;
  if (n > 0) {
    if (int rr = alloc(c, (void **)&c->d_probes, n * 8)) return rr;
    CUDA_TRY(c, copy(c, c->d_probes, w.data(), n * 8, cudaMemcpyHostToDevice));
  }
  return 0;
}

int fdtd_set_dft(fdtd_ctx *c, int32_t nseries, const fdtd_series *series, int32_t nmonitors,
                 const int32_t *freqs_per_monitor, const double *freqs) {
  if (!c) return FDTD_E_INVALID;
  c->generation++;
  c->layout++;
  // phase slots: per monitor, its frequencies at E's times then at H's (resident.rs:714-730)
  std::vector<int> slot0(nmonitors + 1, 0), fcount(nmonitors, 0), fstart(nmonitors, 0);
  std::vector<double> omega;
  std::vector<int> slot_field;
  int at = 0;
  for (int m = 0; m < nmonitors; m++) {
    fstart[m] = at;
    fcount[m] = freqs_per_monitor[m];
    slot0[m] = (int)omega.size();
    for (int fld = 0; fld < 2; fld++)
      for (int f = 0; f < fcount[m]; f++) {
        double fr = freqs[at + f];
        if (!(fr > 0 && std::isfinite(fr) && TAU * fr * c->dt < M_PI))
          return fail(c, FDTD_E_INVALID, "frequency %g is at or beyond the Nyquist frequency", fr);
        omega.push_back(TAU * fr);
        slot_field.push_back(fld);
      }
    at += fcount[m];
  }
  std::vector<SeriesDev> sd(nseries);
  std::vector<long long> where, value_series;
  long long values = 0, sums = 0;
  for (int s = 0; s < nseries; s++) {
    const fdtd_series &x = series[s];
    if (x.monitor < 0 || x.monitor >= nmonitors || x.field < 0 || x.field > 1 ||
        x.component < 0 || x.component > 2)
      return fail(c, FDTD_E_INVALID, "series %d is malformed", s);
    long long vol = 1;
    for (int a = 0; a < 3; a++) {
      if (x.lo[a] < 0 || x.len[a] <= 0 || x.lo[a] + x.len[a] > c->n[a])
        return fail(c, FDTD_E_INVALID, "series %d's box is not on the grid", s);
      vol *= x.len[a];
    }
    sd[s].value0 = values;
    sd[s].volume = vol;
    sd[s].sum0 = sums;
    sd[s].nf = fcount[x.monitor];
    sd[s].slot0 = slot0[x.monitor] + (x.field == 1 ? fcount[x.monitor] : 0);
    for (long long k = 0; k < x.len[2]; k++)
      for (long long j = 0; j < x.len[1]; j++)
        for (long long i = 0; i < x.len[0]; i++) {
          long long r = ((x.lo[2] + k) * c->n[1] + (x.lo[1] + j)) * c->n[0] + (x.lo[0] + i);
          where.push_back(((long long)x.field << 62) | ((long long)x.component * c->N + r));
          value_series.push_back(s);
        }
    values += vol;
    sums += vol * sd[s].nf;
  }
  for (void *p : {(void *)c->d_where, (void *)c->d_value_series, (void *)c->d_series,
                  (void *)c->d_omega, (void *)c->d_slot_field, (void *)c->sums, c->ring,
                  (void *)c->phase})
    release(c, p);
  c->d_where = c->d_value_series = nullptr;
  c->d_series = nullptr;
  c->d_omega = nullptr;
  c->d_slot_field = nullptr;
  c->sums = nullptr;
  c->ring = nullptr;
  c->phase = nullptr;
  c->nvalues = values;
  c->nseries = nseries;
  c->nslots = (int)omega.size();
  c->nsums = sums;
  if (values == 0) return 0;
  // the ring: K steps of the values, K as large as 64 while it stays within 1 GB
  long long K = 64;
  while (K > 4 && (size_t)K * values * c->elem > (1ULL << 30)) K /= 2;
  c->ring_k = (int)K;
  if (int r = alloc(c, (void **)&c->d_where, values * 8)) return r;
  if (int r = alloc(c, (void **)&c->d_value_series, values * 8)) return r;
  if (int r = alloc(c, (void **)&c->d_series, nseries * sizeof(SeriesDev))) return r;
  if (int r = alloc(c, (void **)&c->d_omega, omega.size() * 8)) return r;
  if (int r = alloc(c, (void **)&c->d_slot_field, slot_field.size() * 4)) return r;
  if (int r = alloc(c, (void **)&c->sums, sums * 16)) return r;
  if (int r = alloc(c, &c->ring, K * values * c->elem)) return r;
  if (int r = alloc(c, (void **)&c->phase, K * omega.size() * 16)) return r;
  CUDA_TRY(c, copy(c, c->d_where, where.data(), values * 8, cudaMemcpyHostToDevice));
  CUDA_TRY(c, copy(c, c->d_value_series, value_series.data(), values * 8, cudaMemcpyHostToDevice));
  CUDA_TRY(c, copy(c, c->d_series, sd.data(), nseries * sizeof(SeriesDev), cudaMemcpyHostToDevice));
  CUDA_TRY(c, copy(c, c->d_omega, omega.data(), omega.size() * 8, cudaMemcpyHostToDevice));
  CUDA_TRY(c, copy(c, c->d_slot_field, slot_field.data(), slot_field.size() * 4, cudaMemcpyHostToDevice));
  CUDA_TRY(c, cudaMemsetAsync(c->sums, 0, sums * 16, c->stream));
  // the source waves' batch must match the ring's
  if (c->stride() > 0 && c->wave_batch < K) {
    release(c, c->waves_h);
    release(c, c->waves_e);
    c->waves_h = c->waves_e = nullptr;
    if (int r = alloc(c, (void **)&c->waves_h, (size_t)K * c->stride() * 16)) return r;
    if (int r = alloc(c, (void **)&c->waves_e, (size_t)K * c->stride() * 16)) return r;
    c->wave_batch = (int)K;
  }
  return 0;
}

int fdtd_set_media(fdtd_ctx *c, int32_t ngroups, const fdtd_media_group *groups) {
  if (!c) return FDTD_E_INVALID;
  c->generation++;
  c->layout++;
  long long members = 0;
  int maxp = 1;
  for (int g = 0; g < ngroups; g++) {
    members += groups[g].count;
    maxp = std::max(maxp, (int)groups[g].npoles);
  }
  c->media = members > 0;
  if (!c->media) return 0;
  std::vector<int> member(3 * c->N, -1), group(members);
  std::vector<double> scale(members), gchi(ngroups), gpole((size_t)ngroups * maxp * 3, 0.0);
  std::vector<int> gpoles(ngroups);
  // members numbered in value order, so a pass over them reads the fields in order
  struct In { long long at; int g; double scale; };
  std::vector<In> all;
  all.reserve(members);
  for (int g = 0; g < ngroups; g++) {
    const fdtd_media_group &G = groups[g];
    gchi[g] = G.chi;
    gpoles[g] = G.npoles;
    for (int p = 0; p < G.npoles; p++)
      for (int q = 0; q < 3; q++) gpole[((size_t)g * maxp + p) * 3 + q] = G.poles[3 * p + q];
    for (long long v = 0; v < G.count; v++) {
      if (G.component[v] < 0 || G.component[v] > 2 || G.r[v] < 0 || G.r[v] >= c->N)
        return fail(c, FDTD_E_INVALID, "a medium's value is outside the grid");
      all.push_back(In{G.component[v] * c->N + G.r[v], g, G.scale[v]});
    }
  }
  std::sort(all.begin(), all.end(), [](const In &a, const In &b) { return a.at < b.at; });
  for (long long m = 1; m < members; m++)
    if (all[m].at == all[m - 1].at) return fail(c, FDTD_E_INVALID, "a value is in two media");
  std::vector<long long> place(members);
  for (long long m = 0; m < members; m++) {
    member[all[m].at] = (int)m;
    group[m] = all[m].g;
    scale[m] = all[m].scale;
    place[m] = all[m].at;
  }
  size_t E = c->elem;
  void *d_member, *d_group, *d_scale, *d_before, *d_cur, *d_prev, *d_gchi, *d_gpoles, *d_gpole;
  void *d_place;
  if (int r = alloc(c, &d_place, members * 8)) return r;
  CUDA_TRY(c, copy(c, d_place, place.data(), members * 8, cudaMemcpyHostToDevice));
  if (int r = alloc(c, &d_member, member.size() * 4)) return r;
  if (int r = alloc(c, &d_group, members * 4)) return r;
  if (int r = alloc(c, &d_scale, members * E)) return r;
  if (int r = alloc(c, &d_before, members * E)) return r;
  if (int r = alloc(c, &d_cur, members * maxp * E)) return r;
  if (int r = alloc(c, &d_prev, members * maxp * E)) return r;
  if (int r = alloc(c, &d_gchi, ngroups * E)) return r;
  if (int r = alloc(c, &d_gpoles, ngroups * 4)) return r;
  if (int r = alloc(c, &d_gpole, gpole.size() * E)) return r;
  CUDA_TRY(c, copy(c, d_member, member.data(), member.size() * 4, cudaMemcpyHostToDevice));
  CUDA_TRY(c, copy(c, d_group, group.data(), members * 4, cudaMemcpyHostToDevice));
  CUDA_TRY(c, copy(c, d_gpoles, gpoles.data(), ngroups * 4, cudaMemcpyHostToDevice));
  if (int r = upload(c, d_scale, scale.data(), members)) return r;
  if (int r = upload(c, d_gchi, gchi.data(), ngroups)) return r;
  if (int r = upload(c, d_gpole, gpole.data(), (long long)gpole.size())) return r;
  CUDA_TRY(c, cudaMemsetAsync(d_before, 0, members * E, c->stream));
  CUDA_TRY(c, cudaMemsetAsync(d_cur, 0, members * maxp * E, c->stream));
  CUDA_TRY(c, cudaMemsetAsync(d_prev, 0, members * maxp * E, c->stream));
  auto fillm = [&](auto &M) {
    using T = typename std::remove_pointer<decltype(M.scale)>::type;
    using TT = typename std::remove_const<T>::type;
    M.member = (const int *)d_member;
    M.group = (const int *)d_group;
    M.scale = (const TT *)d_scale;
    M.before = (TT *)d_before;
    M.current = (TT *)d_cur;
    M.previous = (TT *)d_prev;
    M.maxpoles = maxp;
    M.ngroups = ngroups;
    M.gchi = (const TT *)d_gchi;
    M.gpoles = (const int *)d_gpoles;
    M.gpole = (const TT *)d_gpole;
    M.two_dt = (TT)(2.0 * c->dt);
    M.place = (const long long *)d_place;
    M.members = members;
  };
  if (c->precision == 64) fillm(c->md);
  else fillm(c->mf);
  return 0;
}

int fdtd_run_async(fdtd_ctx *c, int64_t steps, int64_t first_step) {
  if (!c) return FDTD_E_INVALID;
  c->generation++;
  if (steps < 0) return fail(c, FDTD_E_INVALID, "a negative number of steps");
  if (steps == 0) return 0;
  c->launches = 0;
  return c->precision == 64 ? run_impl<double>(c, steps, first_step)
                            : run_impl<float>(c, steps, first_step);
}

int fdtd_synchronize(fdtd_ctx *c) {
  if (!c) return FDTD_E_INVALID;
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  CUDA_TRY(c, cudaGetLastError());
  return 0;
}

int fdtd_run(fdtd_ctx *c, int64_t steps, int64_t first_step) {
  if (int r = fdtd_run_async(c, steps, first_step)) return r;
  return fdtd_synchronize(c);
}

int fdtd_read_probes(fdtd_ctx *c, double *out, int64_t capacity, int64_t *steps) {
  if (!c) return FDTD_E_INVALID;
  c->generation++;
  if (steps) *steps = c->nprobes > 0 ? c->recorded : 0;
  if (!out || c->nprobes == 0) return 0;
  long long n = c->recorded * c->nprobes;
  if (capacity < n) return fail(c, FDTD_E_INVALID, "%lld values need room for %lld", n, (long long)capacity);
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  CUDA_TRY(c, copy(c, out, c->record, n * 8, cudaMemcpyDeviceToHost));
  c->recorded = 0;
  return 0;
}

int fdtd_read_dft(fdtd_ctx *c, double *sums, int64_t count) {
  if (!c) return FDTD_E_INVALID;
  if (count != c->nsums)
    return fail(c, FDTD_E_INVALID, "the transforms hold %lld sums, not %lld", c->nsums, (long long)count);
  if (c->nsums == 0) return 0;
  const long long n = 2 * c->nsums;
  if (void *dev = mapped_range(sums, (size_t)n * 8)) {
    // added over the link into the caller's mapped array
    add_into_kernel<<<stride_blocks(c, n), 256, 0, c->stream>>>(c->sums, (double *)dev, n);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaMemsetAsync(c->sums, 0, c->nsums * 16, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return 0;
  }
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  std::vector<double> tmp(n);
  CUDA_TRY(c, copy(c, tmp.data(), c->sums, c->nsums * 16, cudaMemcpyDeviceToHost));
  for (long long q = 0; q < n; q++) sums[q] += tmp[q];
  CUDA_TRY(c, cudaMemsetAsync(c->sums, 0, c->nsums * 16, c->stream));
  return 0;
}

int fdtd_device_fields(fdtd_ctx *c, void **e, void **h) {
  if (!c) return FDTD_E_INVALID;
  if (e) *e = c->e[c->parity];
  if (h) *h = c->h[c->parity];
  return 0;
}

void *fdtd_stream(fdtd_ctx *c) { return c ? (void *)c->stream : nullptr; }

int fdtd_profile(fdtd_ctx *c, int32_t on) {
  if (!c) return FDTD_E_INVALID;
  c->profiling = on != 0;
  c->events_used = 0;
  return 0;
}

int fdtd_profile_read(fdtd_ctx *c, double *ms, int64_t *launches) {
  if (!c) return FDTD_E_INVALID;
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  double total = 0.0;
  for (size_t q = 0; q + 1 < c->events_used; q += 2) {
    float t = 0.f;
    CUDA_TRY(c, cudaEventElapsedTime(&t, c->events[q], c->events[q + 1]));
    total += t;
  }
  if (ms) *ms = total;
  if (launches) *launches = (int64_t)(c->events_used / 2);
  return 0;
}
int64_t fdtd_launches(const fdtd_ctx *c) { return c ? c->launches : 0; }

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Uploading without allocating. fdtd_upload_fields stages an f32 upload from pageable host memory
// through a device buffer of the context's, which it allocates on the first such upload. Some
// callers can't allocate device memory at that point: a serving loop that has handed out its
// whole HBM budget up front, an application whose CUDA allocator is its own and forbids others,
// code that must not perturb a stream-ordered memory pool. fdtd_upload_fields_static stages
// through a fixed array instead: a file-scope device array of STATIC_STAGE_VALUES doubles
// (16 MiB), which every GPU that loads this library holds until the process exits. Only f32
// contexts stage (f64 values are copied straight into the fields), so only they are limited to
// components of at most STATIC_STAGE_VALUES values. The array's address is looked up once per device (below), on
// the first call made with that device current; that first call should come before any stream
// capture. All calls share the array and it keeps the last call's contents (nothing in it has to
// start at zero: each pass overwrites what it reads); calls that overlap on the GPU, from two
// contexts on different streams, race on it.
namespace {
constexpr long long STATIC_STAGE_VALUES = 1LL << 21;
}  // namespace
static __device__ __align__(256) double g_static_stage[STATIC_STAGE_VALUES];

namespace {
constexpr int MAX_DEVICES = 64;
void *g_static_stage_ptr[MAX_DEVICES] = {};
std::mutex g_static_stage_mutex;

// The device address of g_static_stage on the current device (host code can't use the symbol
// itself: in host code its name is only a host-side stand-in).
int static_stage_address(fdtd_ctx *c, double **out) {
  int dev = 0;
  CUDA_TRY(c, cudaGetDevice(&dev));
  if (dev < 0 || dev >= MAX_DEVICES) return fail(c, FDTD_E_GPU, "device %d is beyond %d", dev, MAX_DEVICES);
  std::lock_guard<std::mutex> lock(g_static_stage_mutex);
  if (!g_static_stage_ptr[dev]) {
    void *p = nullptr;
    CUDA_TRY(c, cudaGetSymbolAddress(&p, g_static_stage));
    g_static_stage_ptr[dev] = p;
  }
  *out = static_cast<double *>(g_static_stage_ptr[dev]);
  return 0;
}

// One component (n values) from the host into dst, through the static array.
template <typename T>
int upload_static_as(fdtd_ctx *c, double *stage, void *dst, const double *src, long long n) {
  if constexpr (sizeof(T) == 8) {
    CUDA_TRY(c, cudaMemcpyAsync(dst, src, n * 8, cudaMemcpyHostToDevice, c->stream));
  } else {
    CUDA_TRY(c, cudaMemcpyAsync(stage, src, n * 8, cudaMemcpyHostToDevice, c->stream));
    convert_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(stage, (T *)dst, n);
    CUDA_TRY(c, cudaGetLastError());
  }
  return 0;
}
}  // namespace

extern "C" int fdtd_upload_fields_static(fdtd_ctx *c, const double *e, const double *h) {
  if (!c) return FDTD_E_INVALID;
  if (c->precision == 32 && c->N > STATIC_STAGE_VALUES)
    return fail(c, FDTD_E_INVALID,
                "a field component of %lld values exceeds the %lld-value static staging array: "
                "use fdtd_upload_fields",
                c->N, STATIC_STAGE_VALUES);
  double *stage = nullptr;
  if (c->precision == 32)
    if (int r = static_stage_address(c, &stage)) return r;
  c->generation++;
  c->parity = 0;
  const size_t E = c->elem;
  const double *src[2] = {e, h};
  void *dst[2] = {c->e[0], c->h[0]};
  for (int f = 0; f < 2; f++) {
    if (!src[f]) {
      CUDA_TRY(c, cudaMemsetAsync(dst[f], 0, 3 * c->N * E, c->stream));
      continue;
    }
    for (int comp = 0; comp < 3; comp++) {
      void *d = (char *)dst[f] + comp * c->N * E;
      int r = c->precision == 64 ? upload_static_as<double>(c, stage, d, src[f] + comp * c->N, c->N)
                                 : upload_static_as<float>(c, stage, d, src[f] + comp * c->N, c->N);
      if (r) return r;
    }
  }
  for (size_t s = 0; s < c->slabs.size(); s++) {  // psi from zero, as fdtd_upload_fields with NULL
    const DeviceSlab &d = c->slabs[s];
    void *base = d.field == 1 ? c->psi_h[0] : c->psi_e;
    CUDA_TRY(c, cudaMemsetAsync((char *)base + d.psi * E, 0, d.size * E, c->stream));
  }
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->fields_set = true;
  return 0;
}

// ------------------------------------------------------------------------------------------
// What the batch (batch.cu) reads of a context: its device buffers and tables, in place.

int fdtd_instance_view(fdtd_ctx *c, InstanceView *v) {
  if (!c || !v) return FDTD_E_INVALID;
  if (!c->coeffs_set || !c->fields_set)
    return fail(c, FDTD_E_STATE, "upload the coefficients and the fields before a batch run");
  v->precision = c->precision;
  for (int a = 0; a < 3; a++) {
    v->n[a] = c->n[a];
    v->periodic[a] = c->periodic[a];
    v->low[a] = c->low[a];
    v->high[a] = c->high[a];
    v->step[a] = c->step[a];
  }
  v->N = c->N;
  v->dt = c->dt;
  v->parity = c->parity;
  for (int p = 0; p < 2; p++) {
    v->e[p] = c->e[p];
    v->h[p] = c->h[p];
    v->psi_h[p] = c->psi_h[p];
  }
  v->psi_e = c->psi_e;
  v->psi_h_len = c->psi_h_len;
  for (int a = 0; a < 3; a++) {
    v->inv_step[a] = c->inv_step[a];
    v->fast_div[a] = c->fast_div[a];
  }
  v->psi_e_len = c->psi_e_len;
  v->ca = c->lossless ? nullptr : c->ca;
  v->cb = c->cb;
  v->fe = c->fe;
  v->fh = c->fh;
  v->coefs = c->coefs;
  memcpy(v->table, c->table, sizeof v->table);
  v->waves = &c->src_waves;
  v->inj = &c->src_inj;
  v->nvalues = c->nvalues;
  v->where = c->d_where;
  v->series = c->d_series;
  v->value_series = c->d_value_series;
  v->nslots = c->nslots;
  v->omega = c->d_omega;
  v->slot_field = c->d_slot_field;
  v->sums = c->sums;
  v->nsums = c->nvalues > 0 ? c->nsums : 0;
  v->nprobes = c->nprobes;
  v->probes = c->d_probes;
  v->media = c->media;
  v->plane_waves = c->naux_runs > 0;
  v->stream = c->stream;
  v->generation = c->generation;
  return 0;
}

int fdtd_instance_reserve(fdtd_ctx *c, long long steps, double **rows) {
  if (!c) return FDTD_E_INVALID;
  *rows = nullptr;
  if (c->nprobes == 0) return 0;
  if (c->recorded + steps > c->record_cap) {
    long long cap = std::max<long long>(c->recorded + steps, 2 * c->record_cap);
    double *nr = nullptr;
    if (int r = alloc(c, (void **)&nr, (size_t)cap * c->nprobes * 8)) return r;
    if (c->record && c->recorded)
      CUDA_TRY(c, cudaMemcpyAsync(nr, c->record, (size_t)c->recorded * c->nprobes * 8,
                                  cudaMemcpyDeviceToDevice, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    release(c, c->record);
    c->record = nr;
    c->record_cap = cap;
  }
  *rows = c->record + c->recorded * c->nprobes;
  return 0;
}

void fdtd_instance_advance(fdtd_ctx *c, long long steps) {
  if (!c) return;
  if (steps & 1) c->parity = 1 - c->parity;
  if (c->nprobes > 0) c->recorded += steps;
}

int fdtd_fast_division(const fdtd_ctx *c, int32_t out[3]) {
  if (!c || !out) return FDTD_E_INVALID;
  for (int a = 0; a < 3; a++) out[a] = c->fast_div[a];
  return 0;
}

int fdtd_instance_fail(fdtd_ctx *c, int code, const char *what) {
  return c ? fail(c, code, "%s", what) : code;
}
