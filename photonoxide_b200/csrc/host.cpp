// The host side of the B200 FDTD engine: photonoxide's `Simulation` (src/fdtd.rs:469-1590),
// building on the CPU what the reference builds (the averaged permittivity, the time step, the
// walls, the CPML's tables, conductivity, media, sources and monitors) and stepping on the device
// through the engine's C ABI (photonoxide_fdtd.h). Compiled without floating-point contraction,
// so every table is the reference's bits.
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "photonoxide_fdtd.h"
#include "photonoxide_sim.h"
#include "photonoxide_adjoint.h"
#include "photonoxide_batch.h"
#include "portable.h"
#include "average.cuh"
#include "cpml.cuh"

namespace {

constexpr double kTau = 6.283185307179586476925286766559;
constexpr double kPi = 3.141592653589793238462643383279;

inline int first_of(int c) { return (c + 1) % 3; }
inline int second_of(int c) { return (c + 2) % 3; }

struct Grid {  // Grid3d (src/fdfd/three.rs:70-157)
  int64_t n[3];
  double d[3], o[3];
  int64_t cells() const { return n[0] * n[1] * n[2]; }
  double node(int a, int64_t m) const { return o[a] + (double)m * d[a]; }
  void e_position(int c, int64_t r, double p[3]) const {
    int64_t i = r % n[0], j = (r / n[0]) % n[1], k = r / (n[0] * n[1]);
    p[0] = node(0, i);
    p[1] = node(1, j);
    p[2] = node(2, k);
    p[c] += 0.5 * d[c];
  }
};

struct Geometry {
  double background = 1.0;
  std::vector<double> boxes;  // 7 per box
  explicit Geometry(const pxs_geometry *g) {
    if (!g) return;
    background = g->background;
    boxes.assign(g->boxes, g->boxes + 7 * (size_t)g->nboxes);
  }
  size_t count() const { return boxes.size() / 7; }
  pxa::BoxView view() const { return pxa::BoxView{background, (int64_t)count(), boxes.data()}; }
  double at(const double p[3]) const { return view().at(p); }
};

// The cell average of one value (src/fdfd/three.rs:563-588): average.cuh, shared with the device.
double average_cell(const Geometry &geo, const double centre[3], const double h[3], int along) {
  return pxa::average_cell(geo.view(), centre, h, along);
}

double average_uniform(double e) { return pxa::average_uniform(e); }

// Whether every sample of the cell sees the same value, and which (average.cuh).
bool uniform_cell(const Geometry &geo, const double centre[3], const double h[3], double *value) {
  const int64_t b = pxa::uniform_cell(geo.view(), centre, h);
  if (b == -2) return false;
  *value = b < 0 ? geo.background : geo.boxes[7 * b + 6];
  return true;
}

struct SlabInfo {
  int field, comp, axis;
  int64_t from, count;
  std::vector<double> b, a;
};

struct Series {
  int field, comp;
  int64_t lo[3], len[3];
  int monitor;  // index into the engine's monitor list
  std::vector<double> sums;  // complex interleaved, f major then k, j, i
  int64_t volume() const { return len[0] * len[1] * len[2]; }
};

struct FluxFace {
  int axis;
  int64_t plane;
  int64_t win[2][2];
  double sign;
  size_t series0;  // its 4 series: E b, E c, H b, H c
};

struct Monitor {
  std::vector<double> freqs;
  std::vector<size_t> series;
};

struct Probe {
  int field, comp;
  int64_t r;
  std::vector<double> values;
};

struct MediaGroup {
  std::vector<int32_t> comp;
  std::vector<int64_t> r;
  std::vector<double> scale;
  double chi;
  std::vector<double> poles;  // alpha, xi, gamma per pole
};

int set_error(std::string *where, int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (where) *where = buf;
  return code;
}

// The medium's stability (src/fdtd/media.rs:261-309, 460-513): the largest |z| among the roots of
// the update's characteristic polynomial for (K dt)^2 from 0 to its grid's largest, by Aberth's
// iteration.
std::vector<double> poly_multiply(const std::vector<double> &a, const std::vector<double> &b) {
  std::vector<double> out(a.size() + b.size() - 1, 0.0);
  for (size_t i = 0; i < a.size(); i++)
    for (size_t j = 0; j < b.size(); j++) out[i + j] += a[i] * b[j];
  return out;
}
double largest_root(std::vector<double> p) {
  while (p.size() > 1 && p.back() == 0.0) p.pop_back();
  size_t n = p.size() - 1;
  if (n == 0) return 0.0;
  double lead = p[n];
  for (double &c : p) c /= lead;
  double radius = std::max(pxp::pow(std::fabs(p[0]), 1.0 / (double)n), 1e-3);
  std::vector<double> zr(n), zi(n);
  for (size_t k = 0; k < n; k++) {
    double ang = kTau * ((double)k + 0.25) / (double)n;
    zr[k] = radius * std::cos(ang);
    zi[k] = radius * std::sin(ang);
  }
  for (int it = 0; it < 500; it++) {
    double largest = 0.0;
    for (size_t k = 0; k < n; k++) {
      double vr = 0, vi = 0, dr = 0, di = 0;
      for (size_t q = p.size(); q-- > 0;) {
        double ndr = dr * zr[k] - di * zi[k] + vr, ndi = dr * zi[k] + di * zr[k] + vi;
        dr = ndr;
        di = ndi;
        double nvr = vr * zr[k] - vi * zi[k] + p[q], nvi = vr * zi[k] + vi * zr[k];
        vr = nvr;
        vi = nvi;
      }
      if (vr == 0.0 && vi == 0.0) continue;
      double den = dr * dr + di * di;
      double rr = (vr * dr + vi * di) / den, ri = (vi * dr - vr * di) / den;
      double sr = 0, si = 0;
      for (size_t j = 0; j < n; j++) {
        if (j == k) continue;
        double ar = zr[k] - zr[j], ai = zi[k] - zi[j], m = ar * ar + ai * ai;
        sr += ar / m;
        si += -ai / m;
      }
      double qr = 1.0 - (rr * sr - ri * si), qi = -(rr * si + ri * sr);
      double qm = qr * qr + qi * qi;
      double str = (rr * qr + ri * qi) / qm, sti = (ri * qr - rr * qi) / qm;
      if (std::isfinite(str) && std::isfinite(sti)) {
        zr[k] -= str;
        zi[k] -= sti;
        largest = std::max(largest, std::hypot(str, sti) / std::max(std::hypot(zr[k], zi[k]), 1e-300));
      }
    }
    if (largest < 1e-15) break;
  }
  double m = 0.0;
  for (size_t k = 0; k < n; k++) m = std::max(m, std::hypot(zr[k], zi[k]));
  return m;
}
bool medium_stable(double eps_inf, const std::vector<double> &co, double sigma, double dt,
                   double top) {
  size_t np = co.size() / 3;
  auto product = [&](long skip) {
    std::vector<double> acc{1.0};
    for (size_t i = 0; i < np; i++)
      if ((long)i != skip) acc = poly_multiply(acc, {-co[3 * i + 1], -co[3 * i], 1.0});
    return acc;
  };
  double most = top * dt * dt;
  for (int i = 1; i <= 200; i++) {
    double u = most * (double)i / 200.0;
    double half = sigma * dt / 2.0;
    std::vector<double> poly = poly_multiply({eps_inf - half, u - 2.0 * eps_inf, eps_inf + half},
                                             product(-1));
    for (size_t q = 0; q < np; q++) {
      double gm = co[3 * q + 2];
      std::vector<double> term =
          poly_multiply({gm / 4.0, 0.0, -gm / 2.0, 0.0, gm / 4.0}, product((long)q));
      for (size_t t = 0; t < poly.size() && t < term.size(); t++) poly[t] += term[t];
    }
    if (largest_root(poly) > 1.0 + 1e-6) return false;
  }
  return true;
}

// Twice a value's position along `axis` in steps from node 0 (src/fdtd/sources.rs:155-162).
int64_t twice(int field, int comp, int axis, int64_t m) {
  const bool half = field == 0 ? comp == axis : comp != axis;
  return 2 * m + (half ? 1 : 0);
}

// One coupling across a total-field/scattered-field surface (src/fdtd/sources.rs:138-153).
struct Link {
  int target, comp;
  int64_t r;
  double weight;
  int from_field, from_comp;
  int64_t from[3];
};

// A plane wave's run (PlaneWaveRun, src/fdtd/sources.rs:740-951) as the host builds it: the
// auxiliary 1D grid's coefficients and sheet, the box's couplings, and a copy of its state (the
// device steps it; the copy is brought up to date when read, or when the engine is remade).
struct PlaneRun {
  int64_t g[3];
  double steps[3];
  int64_t base = 0, pad = 0, len = 0;
  std::vector<double> ca, cb, da, db;
  std::vector<int32_t> sheet_comp;
  std::vector<int64_t> sheet_i;
  std::vector<double> sheet_j;
  fdtd_waveform wave;
  struct Coupling { int c; int64_t r; double w; int from; int64_t i; };
  std::vector<Coupling> on_e, on_h;
  std::vector<double> e, h;  // 3 x len each

  bool sample(int field, int comp, const int64_t at[3], int64_t *i) const {
    int64_t l = 0;
    for (int a = 0; a < 3; a++) l += g[a] * twice(field, comp, a, at[a]);
    const int64_t q = l - base;
    if (q < 0 || q >= len) return false;
    *i = q;
    return true;
  }
};

}  // namespace

struct pxs_sim {
  std::string error;
  Grid g;
  int kind[3];
  int64_t low[3], high[3];
  double cpml[5];
  int precision;
  size_t budget;
  double dt;
  int64_t steps = 0;
  bool varies[3];
  std::vector<double> ca[3], cb[3], kn[3], kh[3];
  std::vector<SlabInfo> slabs;
  // host copies of the state; `host_fresh`: they hold the latest (the device's is stale)
  std::vector<double> e, h;
  std::vector<std::vector<double>> psi;
  bool host_fresh = true;
  bool device_fresh = false;
  // sources, in CPU order: point sources first (src/fdtd.rs:1348-1359), then currents
  std::vector<fdtd_waveform> waves;
  std::vector<fdtd_injection> points, currents;
  std::vector<Probe> probes;
  std::vector<Monitor> monitors;
  std::vector<Series> series;
  std::vector<int> dft_monitor;  // add_dft's monitors, by number
  std::vector<std::vector<FluxFace>> fluxes;
  std::vector<MediaGroup> groups;
  std::unordered_map<int64_t, int> members;  // a dispersive value (comp * N + r): its group
  std::vector<PlaneRun> plane_waves;
  int aux_on_device = 0;  // the plane waves whose latest state is the engine's
  // Bloch sides (src/fdtd/bloch.rs): the wavenumbers, e^(ikL) along each axis, and with one not
  // zero the fields' imaginary part, a second simulation stepped alongside
  double bloch_k[3] = {0.0, 0.0, 0.0};
  bool along[3] = {false, false, false};
  double phase_re[3] = {1.0, 1.0, 1.0}, phase_im[3] = {0.0, 0.0, 0.0};
  pxs_sim *twin = nullptr;
  bool configured = false;  // sources, probes and transforms pushed to the engine
  bool fields_dropped = false;  // released without reading the fields back (a served job's)
  fdtd_ctx *ctx = nullptr;

  int64_t N() const { return g.cells(); }
  bool periodic(int a) const { return kind[a] == 1; }
  // Bloch::image (src/fdtd/bloch.rs:85-95): e^(-ikL turns) along `axis`, num-complex's powi of
  // the phase (squaring; a negative power the inverse, (re, 0 - im) / |z|^2)
  void image(int axis, int64_t turns, double *re, double *im) const {
    *re = 1.0;
    *im = 0.0;
    if (turns == 0 || !along[axis]) return;
    auto mul = [](double ar, double ai, double br, double bi, double *cr, double *ci) {
      *cr = ar * br - ai * bi;
      *ci = ar * bi + ai * br;
    };
    const int64_t n = -turns;
    uint64_t e = (uint64_t)(n >= 0 ? n : -n);
    double br = phase_re[axis], bi = phase_im[axis];
    while ((e & 1) == 0) {
      mul(br, bi, br, bi, &br, &bi);
      e >>= 1;
    }
    double ar = br, ai = bi;
    while (e > 1) {
      e >>= 1;
      mul(br, bi, br, bi, &br, &bi);
      if (e & 1) mul(ar, ai, br, bi, &ar, &ai);
    }
    if (n >= 0) {
      *re = ar;
      *im = ai;
    } else {
      const double ns = ar * ar + ai * ai;
      *re = ar / ns;
      *im = 0.0 - ai / ns;
    }
  }

  // bloch::curl_bound (src/fdtd/bloch.rs:31-43): sum of w/d^2 over the axes
  double curl_bound() const {
    double sum = 0.0;
    for (int a = 0; a < 3; a++) {
      const double h = g.d[a], hh = h * h;
      if (g.n[a] == 1 && periodic(a)) {
        if (bloch_k[a] == 0.0) continue;
        double sn, cs;
        pxp::sincos(bloch_k[a] * h / 2.0, &sn, &cs);
        sum += (sn * sn) * (1.0 / hh);
        continue;
      }
      sum += 1.0 / hh;
    }
    return sum;
  }
  int fail(int code, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    error = buf;
    return code;
  }
  bool inside(int64_t i, int64_t j, int64_t k) const {
    return i >= 0 && j >= 0 && k >= 0 && i < g.n[0] && j < g.n[1] && k < g.n[2];
  }
  int64_t index(int64_t i, int64_t j, int64_t k) const { return (k * g.n[1] + j) * g.n[0] + i; }

  // Simulation::build_cpml (src/fdtd.rs:799-869)
  void build_cpml() {
    const double alpha = cpml[4];
    for (int axis = 0; axis < 3; axis++) {
      kn[axis].assign(g.n[axis], 1.0);
      kh[axis].assign(g.n[axis], 1.0);
      if (periodic(axis)) continue;
      const int64_t lo = low[axis], hi = high[axis], n = g.n[axis];
      // sigma and kappa by the reference's powf and ln (cpml.cuh, shared with the device)
      auto at = [&](double pos, double &s, double &k) {
        pxc::grade(pos, lo, hi, n, g.d[axis], cpml, &s, &k);
      };
      for (int64_t m = 0; m < n; m++) {
        double s, k;
        at((double)m, s, k);
        kn[axis][m] = 1.0 / k;
        at((double)m + 0.5, s, k);
        kh[axis][m] = 1.0 / k;
      }
      int64_t froms[2] = {0, n - hi}, counts[2] = {lo, hi};
      for (int side = 0; side < 2; side++) {
        if (counts[side] == 0) continue;
        for (int field = 0; field < 2; field++) {
          SlabInfo sl;
          sl.field = field;
          sl.axis = axis;
          sl.from = froms[side];
          sl.count = counts[side];
          for (int64_t m = sl.from; m < sl.from + sl.count; m++) {
            double s, k, b, a;
            at((double)m + (field == 0 ? 0.0 : 0.5), s, k);
            pxc::recursion(s, k, alpha, dt, &b, &a);
            sl.b.push_back(b);
            sl.a.push_back(a);
          }
          for (int comp : {first_of(axis), second_of(axis)}) {
            sl.comp = comp;
            slabs.push_back(sl);
          }
        }
      }
    }
  }

  // Brings the host's copies up to date with the device's.
  int pull() {
    if (host_fresh || !ctx) return 0;
    e.resize(3 * N());
    h.resize(3 * N());
    std::vector<double *> ps;
    for (auto &p : psi) ps.push_back(p.data());
    if (int r = fdtd_download_fields(ctx, e.data(), h.data(), ps.data()))
      return fail(r, "%s", fdtd_last_error(ctx));
    host_fresh = true;
    return 0;
  }

  // Adds the device's transform sums into the host's.
  int pull_sums() {
    if (!ctx || !configured || series.empty()) return 0;
    int64_t total = 0;
    for (auto &s : series) total += (int64_t)s.sums.size() / 2;
    std::vector<double> add(2 * total, 0.0);
    if (int r = fdtd_read_dft(ctx, add.data(), total)) return fail(r, "%s", fdtd_last_error(ctx));
    int64_t at = 0;
    for (auto &s : series)
      for (size_t q = 0; q < s.sums.size(); q++) s.sums[q] += add[at++];
    return 0;
  }

  // Something changed that the engine holds: its transforms are read out first.
  int reconfigure() {
    if (int r = pull_sums()) return r;
    configured = false;
    return 0;
  }

  int ensure_engine() {
    if (ctx) return 0;
    fdtd_grid gr;
    for (int a = 0; a < 3; a++) {
      gr.n[a] = g.n[a];
      gr.periodic[a] = periodic(a) ? 1 : 0;
      gr.low[a] = periodic(a) ? 0 : low[a];
      gr.high[a] = periodic(a) ? 0 : high[a];
    }
    std::vector<double> fe, fh;
    for (int a = 0; a < 3; a++)  // build_stencils (src/fdtd.rs:1552-1569): kappa/h
      for (int64_t m = 0; m < g.n[a]; m++) {
        fe.push_back(kn[a][m] / g.d[a]);
        fh.push_back(kh[a][m] / g.d[a]);
      }
    std::vector<fdtd_slab> sl;
    for (auto &s : slabs)
      sl.push_back(fdtd_slab{s.field, s.comp, s.axis, s.from, s.count, s.b.data(), s.a.data()});
    fdtd_ctx *c = nullptr;
    int r = fdtd_create(&gr, dt, g.d, fe.data(), fh.data(), sl.data(), (int32_t)sl.size(),
                        precision, budget, &c);
    if (r) {
      fail(r, "%s", c ? fdtd_last_error(c) : "the engine could not start");
      fdtd_destroy(c);
      return r;
    }
    ctx = c;
    if (int q = push_coefficients()) return q;
    if (!groups.empty()) {
      std::vector<fdtd_media_group> mg;
      for (auto &G : groups)
        mg.push_back(fdtd_media_group{(int64_t)G.comp.size(), G.comp.data(), G.r.data(),
                                      G.scale.data(), G.chi, (int32_t)(G.poles.size() / 3),
                                      G.poles.data()});
      if (int q = fdtd_set_media(ctx, (int32_t)mg.size(), mg.data()))
        return fail(q, "%s", fdtd_last_error(ctx));
    }
    device_fresh = false;
    return 0;
  }

  int push_coefficients() {
    bool lossless = true;
    for (int c = 0; c < 3 && lossless; c++)
      for (int64_t r = 0; r < N(); r++) {
        double want = cb[c][r] == 0.0 ? 0.0 : 1.0;
        if (ca[c][r] != want) { lossless = false; break; }
      }
    std::vector<double> a, b;
    for (int c = 0; c < 3; c++) {
      b.insert(b.end(), cb[c].begin(), cb[c].end());
      if (!lossless) a.insert(a.end(), ca[c].begin(), ca[c].end());
    }
    if (int r = fdtd_upload_coeffs(ctx, lossless ? nullptr : a.data(), b.data()))
      return fail(r, "%s", fdtd_last_error(ctx));
    return 0;
  }

  // The couplings across the Bloch sides (Bloch::wrap, src/fdtd/bloch.rs:97-152): H's on the
  // last plane along each Bloch axis (reading E at the first, e^(ikL) - 1), then E's on the
  // first (reading H at the last, e^(-ikL) - 1), by axis, component and value.
  void bloch_wraps(std::vector<fdtd_wrap> &out) const {
    for (int field : {1, 0}) {
      const bool forward = field == 1;
      int32_t slot = 0;
      for (int w = 0; w < 3; w++) {
        if (!along[w]) continue;
        const int64_t n = g.n[w];
        const int64_t m = forward ? n - 1 : 0;
        const int64_t stride = w == 0 ? 1 : (w == 1 ? g.n[0] : g.n[0] * g.n[1]);
        const int64_t o = forward ? -(n - 1) * stride : (n - 1) * stride;
        const double pr = phase_re[w] - 1.0, pi = forward ? phase_im[w] : -phase_im[w];
        const double kappa = forward ? kh[w][m] : kn[w][m];
        const double factor = kappa / g.d[w];
        int64_t lo[3] = {0, 0, 0}, hi[3] = {g.n[0], g.n[1], g.n[2]};
        lo[w] = m;
        hi[w] = m + 1;
        for (int c = 0; c < 3; c++) {
          if (c == w) continue;
          const int a = first_of(c), b = second_of(c);
          double sign = w == a ? 1.0 : -1.0;
          const int d = w == a ? b : a;
          if (!forward) sign = -sign;
          for (int64_t k = lo[2]; k < hi[2]; k++)
            for (int64_t j = lo[1]; j < hi[1]; j++)
              for (int64_t i = lo[0]; i < hi[0]; i++) {
                const int64_t r = (k * g.n[1] + j) * g.n[0] + i;
                fdtd_wrap x;
                x.field = field;
                x.comp = c;
                x.from_comp = d;
                x.slot = forward ? slot++ : 0;
                x.r = r;
                x.q = r + o;
                x.phase_re = pr;
                x.phase_im = pi;
                x.s = sign * factor;
                x.cb = forward ? 0.0 : cb[c][r];
                out.push_back(x);
              }
        }
      }
    }
  }

  // The plane waves' states from the engine into the host's copies.
  int pull_plane_waves() {
    for (int n = 0; n < aux_on_device && ctx; n++) {
      PlaneRun &p = plane_waves[n];
      if (int r = fdtd_plane_wave_state(ctx, n, p.e.data(), p.h.data()))
        return fail(r, "%s", fdtd_last_error(ctx));
    }
    return 0;
  }

  int configure() {
    if (configured) return 0;
    std::vector<fdtd_injection> inj(points);
    inj.insert(inj.end(), currents.begin(), currents.end());
    // the plane waves' runs, with their states so far; each coupling reads a slot of them, its
    // coefficient folded as the reference's correct() has it: dt w for H, cb w for E
    if (int r = pull_plane_waves()) return r;
    std::vector<fdtd_plane_wave> pw(plane_waves.size());
    std::vector<std::vector<int32_t>> sf(plane_waves.size()), sc(plane_waves.size());
    std::vector<std::vector<int64_t>> si(plane_waves.size());
    int32_t slot0 = 0;
    for (size_t n = 0; n < plane_waves.size(); n++) {
      const PlaneRun &p = plane_waves[n];
      std::map<std::tuple<int, int, int64_t>, int32_t> slot;
      auto slot_of = [&](int field, int comp, int64_t i) {
        auto key = std::make_tuple(field, comp, i);
        auto it = slot.find(key);
        if (it != slot.end()) return it->second;
        const int32_t q = (int32_t)sf[n].size();
        sf[n].push_back(field);
        sc[n].push_back(comp);
        si[n].push_back(i);
        slot[key] = q;
        return q;
      };
      for (const PlaneRun::Coupling &q : p.on_h)
        inj.push_back(fdtd_injection{1, q.c, q.r, dt * q.w, 0.0, slot0 + slot_of(0, q.from, q.i), 2});
      for (const PlaneRun::Coupling &q : p.on_e)
        inj.push_back(fdtd_injection{0, q.c, q.r, cb[q.c][q.r] * q.w, 0.0,
                                     slot0 + slot_of(1, q.from, q.i), 2});
      fdtd_plane_wave &d = pw[n];
      d.len = p.len;
      d.pad = p.pad;
      for (int a = 0; a < 3; a++) {
        d.g[a] = p.g[a];
        d.steps[a] = p.steps[a];
      }
      d.ca = p.ca.data();
      d.cb = p.cb.data();
      d.da = p.da.data();
      d.db = p.db.data();
      d.nsheet = (int32_t)p.sheet_comp.size();
      d.sheet_comp = p.sheet_comp.data();
      d.sheet_i = p.sheet_i.data();
      d.sheet_j = p.sheet_j.data();
      d.wave = p.wave;
      d.nslots = (int32_t)sf[n].size();
      d.slot_field = sf[n].data();
      d.slot_comp = sc[n].data();
      d.slot_i = si[n].data();
      d.e0 = p.e.data();
      d.h0 = p.h.data();
      slot0 += d.nslots;
    }
    if (int r = fdtd_set_plane_waves(ctx, (int32_t)pw.size(), pw.data()))
      return fail(r, "%s", fdtd_last_error(ctx));
    aux_on_device = (int)plane_waves.size();
    // a complex run's H couplings across the Bloch sides, each in a slot of its own after the
    // plane waves', subtracted last (Bloch::wrap after step_h, src/fdtd.rs:1330-1333)
    std::vector<fdtd_wrap> wraps;
    bloch_wraps(wraps);
    int32_t nh = 0;
    for (const fdtd_wrap &w : wraps)
      if (w.field == 1) {
        inj.push_back(fdtd_injection{1, w.comp, w.r, 1.0, 0.0, slot0 + w.slot, 2});
        nh++;
      }
    if (int r = fdtd_set_bloch_slots(ctx, nh)) return fail(r, "%s", fdtd_last_error(ctx));
    if (int r = fdtd_set_sources(ctx, (int32_t)waves.size(), waves.data(), (int64_t)inj.size(),
                                 inj.data()))
      return fail(r, "%s", fdtd_last_error(ctx));
    std::vector<int32_t> pf, pc;
    std::vector<int64_t> pr;
    for (auto &p : probes) {
      pf.push_back(p.field);
      pc.push_back(p.comp);
      pr.push_back(p.r);
    }
    if (int r = fdtd_set_probes(ctx, (int32_t)probes.size(), pf.data(), pc.data(), pr.data()))
      return fail(r, "%s", fdtd_last_error(ctx));
    std::vector<fdtd_series> fs;
    for (auto &s : series) {
      fdtd_series x;
      x.field = s.field;
      x.component = s.comp;
      for (int a = 0; a < 3; a++) {
        x.lo[a] = s.lo[a];
        x.len[a] = s.len[a];
      }
      x.monitor = s.monitor;
      fs.push_back(x);
    }
    std::vector<int32_t> per;
    std::vector<double> fr;
    for (auto &m : monitors) {
      per.push_back((int32_t)m.freqs.size());
      fr.insert(fr.end(), m.freqs.begin(), m.freqs.end());
    }
    if (int r = fdtd_set_dft(ctx, (int32_t)fs.size(), fs.data(), (int32_t)per.size(), per.data(),
                             fr.data()))
      return fail(r, "%s", fdtd_last_error(ctx));
    configured = true;
    return 0;
  }

  int push_fields() {
    if (device_fresh) return 0;
    std::vector<const double *> ps;
    for (auto &p : psi) ps.push_back(p.empty() ? nullptr : p.data());
    if (int r = fdtd_upload_fields(ctx, e.empty() ? nullptr : e.data(),
                                   h.empty() ? nullptr : h.data(), ps.data()))
      return fail(r, "%s", fdtd_last_error(ctx));
    device_fresh = true;
    return 0;
  }

  // The engine made, the sources, probes and transforms set, the fields on the device.
  int prepare() {
    if (int r = ensure_engine()) return r;
    if (int r = configure()) return r;
    return push_fields();
  }

  int dropped() {
    return fail(FDTD_E_STATE, "the fields of this simulation were not kept after its served job "
                              "(submitted with keep_fields off): its transforms, fluxes and probes "
                              "are its results");
  }

  int run(int64_t count) {
    if (count <= 0) return 0;
    if (fields_dropped) return dropped();
    if (int r = prepare()) return r;
    if (twin) {  // a complex run: both parts together, coupled across the Bloch sides
      if (int r = twin->prepare()) return fail(r, "%s", twin->error.c_str());
      std::vector<fdtd_wrap> wraps;
      bloch_wraps(wraps);
      if (int r = fdtd_bloch_run(ctx, twin->ctx, (int32_t)wraps.size(), wraps.data(), count,
                                 steps))
        return fail(r, "%s", fdtd_last_error(ctx));
      if (int r = twin->finish(count)) return fail(r, "%s", twin->error.c_str());
      return finish(count);
    }
    if (int r = fdtd_run(ctx, count, steps)) return fail(r, "%s", fdtd_last_error(ctx));
    return finish(count);
  }

  // Everything the device holds brought to the host (fields, psi, transforms; the probes are
  // read after each run), then the engine and its device memory released. A later run makes a
  // new engine from the host's copies.
  int release(bool keep_fields = true) {
    if (twin)
      if (int r = twin->release(keep_fields)) return fail(r, "%s", twin->error.c_str());
    if (!ctx) return 0;
    if (keep_fields) {
      if (int r = pull()) return r;
    } else {
      fields_dropped = true;  // the host's copies are stale: reading them or running refuses
    }
    if (int r = pull_sums()) return r;
    if (int r = pull_plane_waves()) return r;
    aux_on_device = 0;
    fdtd_destroy(ctx);
    ctx = nullptr;
    configured = false;
    device_fresh = false;
    return 0;
  }

  // An upper estimate of the device memory the engine takes (fdtd_create and the set_* calls):
  // two copies of E and H, cb (and ca when lossy), psi (H's twice), the transforms' ring of 64
  // steps and sums, and the media's state.
  size_t device_bytes() const {
    const size_t E = precision == 64 ? 8 : 4;
    const double n = (double)N();
    double values = 15.0 * n;
    bool lossless = true;
    for (int c = 0; c < 3 && lossless; c++)
      for (int64_t r = 0; r < N(); r++)
        if (ca[c][r] != (cb[c][r] == 0.0 ? 0.0 : 1.0)) {
          lossless = false;
          break;
        }
    if (!lossless) values += 3.0 * n;
    for (const SlabInfo &sl : slabs) {
      double rows = n / (double)g.n[sl.axis];
      double width = sl.axis == 0 ? (double)(sl.count + 8) : (double)sl.count;
      values += (sl.field == 1 ? 2.0 : 1.0) * (width * rows + 16.0);
    }
    double extra = 0.0;
    for (const Series &se : series) {
      double nf = se.volume() > 0 ? (double)se.sums.size() / 2.0 / (double)se.volume() : 0.0;
      extra += (double)se.volume() * (64.0 * E + 8.0 * 3 + 16.0 * nf);
    }
    extra += 64.0 * (double)members.size();
    return (size_t)((values * (double)E + extra) * 1.05) + (16u << 20);
  }

  // Whether the batch (photonoxide_batch.h) can step this simulation: 2D, TE fields and sources,
  // no media.
  bool te() const {
    if (g.n[2] != 1 || !periodic(2) || !groups.empty()) return false;
    for (const auto *list : {&points, &currents})
      for (const fdtd_injection &x : *list)
        if ((x.field == 0) == (x.component == 2)) return false;
    const int64_t n = N();
    if (!e.empty())
      for (int64_t r = 0; r < n; r++)
        if (e[2 * n + r] != 0.0) return false;
    if (!h.empty())
      for (int64_t r = 0; r < 2 * n; r++)
        if (h[r] != 0.0) return false;
    return true;
  }

  // After `count` steps on the device (fdtd_run or a batch): the count, the probes' values.
  int finish(int64_t count) {
    host_fresh = false;
    steps += count;
    if (!probes.empty()) {
      int64_t got = 0;
      fdtd_read_probes(ctx, nullptr, 0, &got);
      std::vector<double> rec(got * probes.size());
      if (int r = fdtd_read_probes(ctx, rec.data(), (int64_t)rec.size(), &got))
        return fail(r, "%s", fdtd_last_error(ctx));
      for (int64_t m = 0; m < got; m++)
        for (size_t p = 0; p < probes.size(); p++)
          probes[p].values.push_back(rec[m * probes.size() + p]);
    }
    return 0;
  }

  bool value(size_t s0, size_t s1, int field, int comp, const int64_t at[3], int f, double *re,
             double *im) const {
    for (size_t q = s0; q < s1; q++) {
      const Series &s = series[q];
      if (s.field != field || s.comp != comp) continue;
      bool in = true;
      for (int a = 0; a < 3; a++)
        if (at[a] < s.lo[a] || at[a] >= s.lo[a] + s.len[a]) in = false;
      if (!in) continue;
      int64_t o = ((at[2] - s.lo[2]) * s.len[1] + (at[1] - s.lo[1])) * s.len[0] + at[0] - s.lo[0];
      *re = s.sums[2 * (f * s.volume() + o)];
      *im = s.sums[2 * (f * s.volume() + o) + 1];
      return true;
    }
    return false;
  }

  // FluxPlane::flux (src/fdtd/monitors.rs:320-351)
  double face_flux(const FluxFace &F, int f) const {
    int b = first_of(F.axis), c = second_of(F.axis);
    auto lo_of = [&](int along) {
      int sl = along == b ? 0 : 1;
      return F.win[sl][0] < 0 ? (int64_t)0 : F.win[sl][0];
    };
    auto hi_of = [&](int along) {
      int sl = along == b ? 0 : 1;
      return F.win[sl][0] < 0 ? g.n[along] : F.win[sl][1] + 1;
    };
    auto weight = [&](int along, int64_t m, bool half) {
      int sl = along == b ? 0 : 1;
      if (F.win[sl][0] < 0) return 1.0;
      int64_t lo = F.win[sl][0], hi = F.win[sl][1];
      if (half) return (lo < m && m < hi) ? 1.0 : ((m == lo || m == hi) ? 0.5 : 0.0);
      return (lo < m && m <= hi) ? 1.0 : 0.0;
    };
    double total = 0.0;
    const int comps[2] = {b, c}, hs[2] = {c, b};
    const double signs[2] = {0.5, -0.5};
    for (int t = 0; t < 2; t++) {
      for (int64_t v = lo_of(c); v < hi_of(c); v++)
        for (int64_t u = lo_of(b); u < hi_of(b); u++) {
          double w = weight(b, u, comps[t] == b) * weight(c, v, comps[t] == c);
          if (w == 0.0) continue;
          int64_t at[3];
          at[F.axis] = F.plane;
          at[b] = u;
          at[c] = v;
          double lr, li, hr, hi2, er, ei;
          value(F.series0, F.series0 + 4, 0, comps[t], at, f, &lr, &li);
          value(F.series0, F.series0 + 4, 1, hs[t], at, f, &hr, &hi2);
          at[F.axis] = F.plane + 1;
          value(F.series0, F.series0 + 4, 0, comps[t], at, f, &er, &ei);
          double mr = 0.5 * (lr + er), mi = 0.5 * (li + ei);
          // (m * conj(h)).re as num-complex: mr hr - mi (-hi)
          double re = mr * hr - mi * (-hi2);
          total += w * signs[t] * re;
        }
    }
    return total * g.d[b] * g.d[c];
  }

  // Where value `at` of (field, comp) at frequency f is in the transforms laid end to end (the
  // layout of pxs_transforms and fdtd_read_dft), as a complex index, or -1.
  int64_t locate(size_t s0, size_t s1, int field, int comp, const int64_t at[3], int f) const {
    int64_t base = 0;
    for (size_t q = 0; q < s1; q++) {
      const Series &s = series[q];
      if (q >= s0 && s.field == field && s.comp == comp) {
        bool in = true;
        for (int a = 0; a < 3; a++)
          if (at[a] < s.lo[a] || at[a] >= s.lo[a] + s.len[a]) in = false;
        if (in) {
          int64_t o = ((at[2] - s.lo[2]) * s.len[1] + (at[1] - s.lo[1])) * s.len[0] + at[0] - s.lo[0];
          return base + f * s.volume() + o;
        }
      }
      base += (int64_t)s.sums.size() / 2;
    }
    return -1;
  }

  // The derivative of face_flux(F, f) by the real and imaginary parts of each transform sum,
  // times `scale`, added into grad (complex interleaved, the layout of pxs_transforms). The flux
  // is bilinear: sum of w sign Re(m conj(h)) with m the mean of E over the two node planes.
  void face_flux_grad(const FluxFace &F, int f, double scale, double *grad) const {
    int b = first_of(F.axis), c = second_of(F.axis);
    auto lo_of = [&](int along) {
      int sl = along == b ? 0 : 1;
      return F.win[sl][0] < 0 ? (int64_t)0 : F.win[sl][0];
    };
    auto hi_of = [&](int along) {
      int sl = along == b ? 0 : 1;
      return F.win[sl][0] < 0 ? g.n[along] : F.win[sl][1] + 1;
    };
    auto weight = [&](int along, int64_t m, bool half) {
      int sl = along == b ? 0 : 1;
      if (F.win[sl][0] < 0) return 1.0;
      int64_t lo = F.win[sl][0], hi = F.win[sl][1];
      if (half) return (lo < m && m < hi) ? 1.0 : ((m == lo || m == hi) ? 0.5 : 0.0);
      return (lo < m && m <= hi) ? 1.0 : 0.0;
    };
    const double area = g.d[b] * g.d[c] * scale;
    const int comps[2] = {b, c}, hs[2] = {c, b};
    const double signs[2] = {0.5, -0.5};
    for (int t = 0; t < 2; t++)
      for (int64_t v = lo_of(c); v < hi_of(c); v++)
        for (int64_t u = lo_of(b); u < hi_of(b); u++) {
          double w = weight(b, u, comps[t] == b) * weight(c, v, comps[t] == c);
          if (w == 0.0) continue;
          int64_t at[3];
          at[F.axis] = F.plane;
          at[b] = u;
          at[c] = v;
          double lr = 0, li = 0, hr = 0, hi2 = 0, er = 0, ei = 0;
          const int64_t il = locate(F.series0, F.series0 + 4, 0, comps[t], at, f);
          const int64_t ih = locate(F.series0, F.series0 + 4, 1, hs[t], at, f);
          value(F.series0, F.series0 + 4, 0, comps[t], at, f, &lr, &li);
          value(F.series0, F.series0 + 4, 1, hs[t], at, f, &hr, &hi2);
          at[F.axis] = F.plane + 1;
          const int64_t ie = locate(F.series0, F.series0 + 4, 0, comps[t], at, f);
          value(F.series0, F.series0 + 4, 0, comps[t], at, f, &er, &ei);
          const double k = w * signs[t] * area;
          const double mr = 0.5 * (lr + er), mi = 0.5 * (li + ei);
          if (il >= 0) {
            grad[2 * il] += 0.5 * k * hr;
            grad[2 * il + 1] += 0.5 * k * hi2;
          }
          if (ie >= 0) {
            grad[2 * ie] += 0.5 * k * hr;
            grad[2 * ie + 1] += 0.5 * k * hi2;
          }
          if (ih >= 0) {
            grad[2 * ih] += k * mr;
            grad[2 * ih + 1] += k * mi;
          }
        }
  }

  int check_frequencies(int nf, const double *freqs) {
    if (nf <= 0) return fail(FDTD_E_INVALID, "a monitor needs at least one frequency");
    for (int f = 0; f < nf; f++)
      if (!(freqs[f] > 0.0 && kTau * freqs[f] * dt < kPi))
        return fail(FDTD_E_INVALID, "%g c/um is beyond the time step's Nyquist frequency", freqs[f]);
    return 0;
  }

  void add_plane_series(FluxFace &F, int monitor, int nf) {
    int b = first_of(F.axis), c = second_of(F.axis);
    F.series0 = series.size();
    for (int field = 0; field < 2; field++)
      for (int comp : {b, c}) {
        Series s;
        s.field = field;
        s.comp = comp;
        s.monitor = monitor;
        s.lo[F.axis] = F.plane;
        s.len[F.axis] = field == 0 ? 2 : 1;
        for (int al : {b, c}) {
          int sl = al == b ? 0 : 1;
          s.lo[al] = F.win[sl][0] < 0 ? 0 : F.win[sl][0];
          s.len[al] = (F.win[sl][0] < 0 ? g.n[al] : F.win[sl][1] + 1) - s.lo[al];
        }
        s.sums.assign(2 * s.volume() * nf, 0.0);
        monitors[monitor].series.push_back(series.size());
        series.push_back(s);
      }
  }
};

// Waveform::at (src/fdtd.rs:399-424), a point source's value at t, with the reference's exp and
// sin/cos: w = {kind, p[0..4]} as fdtd_waveform holds it.
double waveform_at(const double w[6], double t) {
  const double TAU = 6.283185307179586476925286766559;
  const double *p = w + 1;
  if (w[0] == 0.0) {
    const double u = (t - p[2]) / p[1];
    double s, c;
    pxp::sincos((TAU * p[0]) * (t - p[2]), &s, &c);
    return pxp::exp(-u * u) * s;
  }
  if (w[0] == 1.0) {
    const double u = (t - p[1]) / p[0];
    return -u * pxp::exp(-u * u) * std::sqrt(2.0 * 2.718281828459045235);
  }
  double ss = 1.0;
  if (p[3] > 0.0) {
    const double r = std::min(std::max(t / p[3], 0.0), 1.0);
    ss = r * r * (3.0 - 2.0 * r);
  }
  double s, c;
  pxp::sincos(-(TAU * p[0]) * t, &s, &c);
  return ss * (p[1] * c - p[2] * s);
}

extern "C" {

int pxs_waveform_spectrum(const double waveform[6], int32_t field, double dt, int64_t steps,
                          int32_t nf, const double *freqs, double *out) {
  if (!waveform || !freqs || !out || nf < 0 || steps < 0 || !(dt > 0.0)) return FDTD_E_INVALID;
  const double TAU = 6.283185307179586476925286766559;
  const double offset = field == 0 ? 0.5 * dt : 0.0;
  for (int32_t f = 0; f < nf; f++) {
    const double omega = TAU * freqs[f];
    // the sum from zero, in step order: (v + 0i)(cos + i sin) dt, as num-complex multiplies
    double re = 0.0, im = 0.0;
    for (int64_t n = 0; n < steps; n++) {
      const double t = (double)n * dt + offset;
      const double v = waveform_at(waveform, t);
      const double x = omega * t;
      double s = 0.0, c = 1.0;
      if (x != 0.0) pxp::sincos(x, &s, &c);
      re += (v * c - 0.0 * s) * dt;
      im += (v * s + 0.0 * c) * dt;
    }
    out[2 * f] = re;
    out[2 * f + 1] = im;
  }
  return 0;
}

int pxs_average(const int64_t n[3], const double d[3], const double o[3], const pxs_geometry *gm,
                double *out) {
  Grid g{{n[0], n[1], n[2]}, {d[0], d[1], d[2]}, {o[0], o[1], o[2]}};
  Geometry geo(gm);
  int64_t N = g.cells();
  std::vector<unsigned char> uniform(3 * N, 0);
  for (int c = 0; c < 3; c++) {
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t r = 0; r < N; r++) {
      double p[3], v;
      g.e_position(c, r, p);
      if (uniform_cell(geo, p, g.d, &v)) {
        uniform[c * N + r] = 1;
        out[c * N + r] = v;
      } else {
        out[c * N + r] = average_cell(geo, p, g.d, c);
      }
    }
  }
  // a uniform cell's average is a function of its value alone: taken once per value
  std::vector<std::pair<double, double>> seen;
  for (int64_t q = 0; q < 3 * N; q++) {
    if (!uniform[q]) continue;
    double v = out[q], a = 0.0;
    bool found = false;
    for (auto &pr : seen)
      if (pr.first == v) { a = pr.second; found = true; break; }
    if (!found) {
      a = average_uniform(v);
      seen.push_back({v, a});
    }
    out[q] = a;
  }
  return 0;
}

pxs_sim *pxs_create(const int64_t n[3], const double d[3], const double o[3], const int32_t kind[3],
                    const int64_t low[3], const int64_t high[3], const double cpml[5],
                    double courant, const double *eps, const pxs_geometry *geometry,
                    int32_t precision, size_t hbm_budget, char *err, int32_t errlen) {
  const double none[3] = {0.0, 0.0, 0.0};
  return pxs_create_bloch(n, d, o, kind, low, high, cpml, none, courant, eps, geometry, precision,
                          hbm_budget, err, errlen);
}

pxs_sim *pxs_create_bloch(const int64_t n[3], const double d[3], const double o[3],
                          const int32_t kind[3], const int64_t low[3], const int64_t high[3],
                          const double cpml[5], const double bloch[3], double courant,
                          const double *eps, const pxs_geometry *geometry, int32_t precision,
                          size_t hbm_budget, char *err, int32_t errlen) {
  std::string msg;
  auto refuse = [&](const char *fmt, auto... args) -> pxs_sim * {
    set_error(&msg, FDTD_E_INVALID, fmt, args...);
    if (err && errlen > 0) snprintf(err, errlen, "%s", msg.c_str());
    return nullptr;
  };
  auto ok = [](double v) { return std::isfinite(v) && v > 0.0; };
  // the checks of with_permittivity (src/fdtd.rs:686-724)
  if (n[0] <= 0 || n[1] <= 0 || n[2] <= 0 || !ok(d[0]) || !ok(d[1]) || !ok(d[2]))
    return refuse("the grid needs cells and positive steps");
  if (!(cpml[0] > 0.0 && cpml[0] < 1.0) || !(std::isfinite(cpml[2]) && cpml[2] >= 0.0) ||
      !(std::isfinite(cpml[3]) && cpml[3] >= 1.0) || !(std::isfinite(cpml[4]) && cpml[4] >= 0.0) ||
      (!std::isnan(cpml[1]) && !(std::isfinite(cpml[1]) && cpml[1] >= 0.0)))
    return refuse("the CPML needs R in (0, 1), an order >= 0, kappa >= 1, alpha >= 0 and sigma >= 0");
  for (int a = 0; a < 3; a++)
    if (kind[a] == 0 && (low[a] < 0 || high[a] < 0 || low[a] + high[a] >= n[a]))
      return refuse("CPMLs of %lld and %lld cells leave nothing of %lld cells", (long long)low[a],
                    (long long)high[a], (long long)n[a]);
  if (!(courant > 0.0 && courant <= 1.0))
    return refuse("the Courant number must be in (0, 1], got %g", courant);
  for (int a = 0; a < 3; a++)
    if (!std::isfinite(bloch[a]) || (bloch[a] != 0.0 && kind[a] != 1))
      return refuse("the Bloch wavenumber along axis %d must be finite, on a periodic axis", a);
  pxs_sim *s = new pxs_sim();
  s->g = Grid{{n[0], n[1], n[2]}, {d[0], d[1], d[2]}, {o[0], o[1], o[2]}};
  for (int a = 0; a < 3; a++) {
    s->kind[a] = kind[a];
    s->low[a] = kind[a] == 0 ? low[a] : 0;
    s->high[a] = kind[a] == 0 ? high[a] : 0;
    s->varies[a] = !(n[a] == 1 && kind[a] == 1);
  }
  for (int q = 0; q < 5; q++) s->cpml[q] = cpml[q];
  s->precision = precision == 64 ? 64 : 32;
  s->budget = hbm_budget;
  // Delta t = C / sqrt(sum w/d^2) (bloch::curl_bound, src/fdtd/bloch.rs:31-43): w = 1 along an
  // axis the field varies along, sin^2(k d / 2) along one a cell long with a Bloch phase
  for (int a = 0; a < 3; a++) s->bloch_k[a] = bloch[a];
  const double sum = s->curl_bound();
  if (sum == 0.0) {
    delete s;
    return refuse("the field varies along no axis");
  }
  s->dt = courant / std::sqrt(sum);
  int64_t N = s->N();
  std::vector<double> avg;
  if (!eps) {
    avg.resize(3 * N);
    pxs_average(n, d, o, geometry, avg.data());
    eps = avg.data();
  }
  for (int c = 0; c < 3; c++) {
    s->ca[c].assign(N, 1.0);
    s->cb[c].resize(N);
    for (int64_t r = 0; r < N; r++) {
      double v = eps[c * N + r];
      if (!(std::isfinite(v) && v > 0.0)) {
        delete s;
        return refuse("the permittivity must be finite and positive, got %g", v);
      }
      s->cb[c][r] = s->dt / v;
    }
  }
  // walls: E tangential to a wall is zero on its node 0 (src/fdtd.rs:738-756)
  for (int c = 0; c < 3; c++)
    for (int a = 0; a < 3; a++) {
      if (a == c || s->periodic(a)) continue;
      int64_t stride = a == 0 ? 1 : (a == 1 ? n[0] : n[0] * n[1]);
      for (int64_t r = 0; r < N; r++)
        if ((r / stride) % n[a] == 0) s->ca[c][r] = s->cb[c][r] = 0.0;
    }
  s->build_cpml();
  s->psi.resize(s->slabs.size());
  if (bloch[0] != 0.0 || bloch[1] != 0.0 || bloch[2] != 0.0) {
    for (int a = 0; a < 3; a++) {
      s->along[a] = bloch[a] != 0.0;
      double sn, cs;  // from_polar(1, k L)
      pxp::sincos(bloch[a] * ((double)n[a] * d[a]), &sn, &cs);
      s->phase_re[a] = 1.0 * cs;
      s->phase_im[a] = 1.0 * sn;
    }
    s->twin = new pxs_sim(*s);
  }
  return s;
}

void pxs_destroy(pxs_sim *s) {
  if (!s) return;
  pxs_destroy(s->twin);
  fdtd_destroy(s->ctx);
  delete s;
}

const char *pxs_last_error(const pxs_sim *s) { return s ? s->error.c_str() : "no simulation"; }

int pxs_conductivity(pxs_sim *s, const double *sigma, const pxs_geometry *geometry) {
  if (s && s->twin)  // a complex run's imaginary part takes it too (src/fdtd.rs:962-964)
    if (int r = pxs_conductivity(s->twin, sigma, geometry))
      return s->fail(r, "%s", s->twin->error.c_str());
  if (!s->groups.empty())
    return s->fail(FDTD_E_INVALID,
                   "the conductivity comes before the dispersive media: with_conductivity, then "
                   "with_medium");
  Geometry geo(geometry);
  int64_t N = s->N();
  for (int c = 0; c < 3; c++)
    for (int64_t r = 0; r < N; r++) {
      if (s->cb[c][r] == 0.0) continue;
      double sg;
      if (sigma) sg = sigma[c * N + r];
      else {
        double p[3];
        s->g.e_position(c, r, p);
        sg = geo.at(p);
      }
      if (!(std::isfinite(sg) && sg >= 0.0))
        return s->fail(FDTD_E_INVALID, "the conductivity must be finite and >= 0, got %g", sg);
      double half = sg * s->cb[c][r] / 2.0;
      s->ca[c][r] = (1.0 - half) / (1.0 + half);
      s->cb[c][r] /= 1.0 + half;
    }
  if (s->ctx) return s->push_coefficients();
  return 0;
}

int pxs_conductor(pxs_sim *s, int32_t comp, int64_t i, int64_t j, int64_t k) {
  if (s && s->twin)  // src/fdtd.rs:1005-1007
    if (int r = pxs_conductor(s->twin, comp, i, j, k))
      return s->fail(r, "%s", s->twin->error.c_str());
  if (comp < 0 || comp > 2 || !s->inside(i, j, k))
    return s->fail(FDTD_E_INVALID, "(%lld, %lld, %lld) is outside the grid", (long long)i,
                   (long long)j, (long long)k);
  if (int r = s->pull()) return r;
  int64_t r = s->index(i, j, k);
  s->ca[comp][r] = s->cb[comp][r] = 0.0;
  if (!s->e.empty()) s->e[comp * s->N() + r] = 0.0;
  auto it = s->members.find(comp * s->N() + r);
  if (it != s->members.end()) {  // Media::remove (src/fdtd/media.rs:641-653)
    MediaGroup &G = s->groups[it->second];
    for (size_t v = 0; v < G.r.size(); v++)
      if (G.comp[v] == comp && G.r[v] == r) {
        G.comp.erase(G.comp.begin() + v);
        G.r.erase(G.r.begin() + v);
        G.scale.erase(G.scale.begin() + v);
        break;
      }
    s->members.erase(it);
  }
  if (s->ctx) {
    s->device_fresh = false;
    return s->push_coefficients();
  }
  return 0;
}

int pxs_medium(pxs_sim *s, double eps_inf, int32_t npoles, const double *poles,
               const uint8_t *inside, const pxs_geometry *geometry) {
  if (s && s->twin)  // src/fdtd/media.rs:756-759
    if (int r = pxs_medium(s->twin, eps_inf, npoles, poles, inside, geometry))
      return s->fail(r, "%s", s->twin->error.c_str());
  // Simulation::medium (src/fdtd/media.rs:749-825), with its stability check
  if (!(std::isfinite(eps_inf) && eps_inf > 0.0))
    return s->fail(FDTD_E_INVALID, "a dispersive medium's eps_inf must be positive and finite");
  if (s->steps > 0 || s->ctx)
    return s->fail(FDTD_E_INVALID, "a dispersive medium goes in before the run starts");
  double dt = s->dt;
  std::vector<double> co;
  double gsum = 0.0;
  for (int p = 0; p < npoles; p++) {  // Pole::parts / coefficients (media.rs:74-109)
    const double *x = poles + 4 * p;
    double a, w0sq, gamma;
    if ((int)x[0] == 0) {
      double w0 = kTau * x[2];
      a = x[1] * w0 * w0;
      w0sq = w0 * w0;
      gamma = kTau * x[3];
    } else {
      double wp = kTau * x[1];
      a = wp * wp;
      w0sq = 0.0;
      gamma = kTau * x[2];
    }
    double dd = 1.0 + gamma * dt / 2.0;
    co.push_back((2.0 - w0sq * dt * dt) / dd);
    co.push_back((gamma * dt / 2.0 - 1.0) / dd);
    co.push_back(a * dt * dt / dd);
    gsum += co.back();
  }
  double chi = gsum / (4.0 * dt);
  Geometry geo(geometry);
  int64_t N = s->N();
  // which E values the medium takes (not those a wall or conductor has zeroed), all at once
  std::vector<uint8_t> in((size_t)(3 * N), 0);
#pragma omp parallel for schedule(dynamic, 65536)
  for (int64_t q = 0; q < 3 * N; q++) {
    const int c = (int)(q / N);
    const int64_t r = q - c * N;
    if (s->cb[c][r] == 0.0) continue;
    if (inside) {
      in[q] = inside[q] != 0;
    } else {
      double p[3];
      s->g.e_position(c, r, p);
      in[q] = geo.at(p) != 0.0;
    }
  }
  auto old_chi_of = [&](int64_t q) {
    auto it = s->members.find(q);
    return it != s->members.end() ? s->groups[it->second].chi : 0.0;
  };
  {
    double top = 4.0 * s->curl_bound(), largest = 0.0;
    for (int64_t q = 0; q < 3 * N; q++) {
      if (!in[q]) continue;
      const int c = (int)(q / N);
      const int64_t r = q - c * N;
      largest = std::max(largest, (1.0 - s->ca[c][r]) / s->cb[c][r] - old_chi_of(q));
    }
    for (double sg : {0.0, largest})
      if (!medium_stable(eps_inf, co, sg, dt, top))
        return s->fail(FDTD_E_INVALID,
                       "the medium isn't stable at the time step %g um/c (a term's w0 dt above 2, "
                       "or a Courant number above sqrt(eps_inf)): take a smaller step", dt);
  }
  // each value taken leaves the group it was in (Media::remove), in value order
  MediaGroup G;
  G.chi = chi;
  G.poles = co;
  std::vector<char> left(s->groups.size(), 0);
  for (int64_t q = 0; q < 3 * N; q++) {
    if (!in[q]) continue;
    const int c = (int)(q / N);
    const int64_t r = q - c * N;
    double old_chi = 0.0;
    auto it = s->members.find(q);
    if (it != s->members.end()) {
      old_chi = s->groups[it->second].chi;
      left[it->second] = 1;
      s->members.erase(it);
    }
    double sg = std::max((1.0 - s->ca[c][r]) / s->cb[c][r] - old_chi, 0.0);
    double nu = 1.0 + dt / eps_inf * (sg / 2.0 + chi);
    s->ca[c][r] = (1.0 - dt * sg / (2.0 * eps_inf)) / nu;
    s->cb[c][r] = dt / eps_inf / nu;
    G.comp.push_back(c);
    G.r.push_back(r);
    G.scale.push_back(s->cb[c][r]);
  }
  // the groups values left keep the rest, in their order
  for (size_t g = 0; g < left.size(); g++) {
    if (!left[g]) continue;
    MediaGroup &O = s->groups[g];
    size_t k = 0;
    for (size_t v = 0; v < O.r.size(); v++) {
      if (in[O.comp[v] * N + O.r[v]]) continue;
      O.comp[k] = O.comp[v];
      O.r[k] = O.r[v];
      O.scale[k] = O.scale[v];
      k++;
    }
    O.comp.resize(k);
    O.r.resize(k);
    O.scale.resize(k);
  }
  if (npoles > 0 && !G.r.empty()) {
    int gi = (int)s->groups.size();
    s->members.reserve(s->members.size() + G.r.size());
    for (size_t v = 0; v < G.r.size(); v++) s->members[G.comp[v] * N + G.r[v]] = gi;
    s->groups.push_back(G);
  }
  return 0;
}

int pxs_add_source(pxs_sim *s, int32_t field, int32_t comp, int64_t i, int64_t j, int64_t k,
                   const double wave[6]) {
  if (!s->inside(i, j, k) || comp < 0 || comp > 2 || field < 0 || field > 1)
    return s->fail(FDTD_E_INVALID, "(%lld, %lld, %lld) is outside the %lld x %lld x %lld grid",
                   (long long)i, (long long)j, (long long)k, (long long)s->g.n[0],
                   (long long)s->g.n[1], (long long)s->g.n[2]);
  if (int r = s->reconfigure()) return r;
  fdtd_waveform w;
  w.kind = (int32_t)wave[0];
  for (int q = 0; q < 5; q++) w.p[q] = wave[q + 1];
  s->waves.push_back(w);
  s->points.push_back(fdtd_injection{field, comp, s->index(i, j, k), 1.0, 0.0,
                                     (int32_t)s->waves.size() - 1, 1});
  return 0;
}

int pxs_add_current(pxs_sim *s, int32_t field, int64_t count, const int32_t *comps,
                    const int64_t *at, const double *amps, const double wave[6]) {
  if (s && s->twin && count > 0) {  // Im(a w) = Re(-i a w) on the imaginary part (sources.rs:190-207)
    std::vector<double> im(2 * count);
    for (int64_t q = 0; q < count; q++) {
      im[2 * q] = 0.0 * amps[2 * q] - (-1.0) * amps[2 * q + 1];
      im[2 * q + 1] = 0.0 * amps[2 * q + 1] + (-1.0) * amps[2 * q];
    }
    if (int r = pxs_add_current(s->twin, field, count, comps, at, im.data(), wave))
      return s->fail(r, "%s", s->twin->error.c_str());
  }
  for (int64_t q = 0; q < count; q++) {  // src/fdtd/sources.rs:223-242
    const int64_t *p = at + 3 * q;
    if (!s->inside(p[0], p[1], p[2]) || comps[q] < 0 || comps[q] > 2)
      return s->fail(FDTD_E_INVALID, "a current's value is outside the grid");
    if (!std::isfinite(amps[2 * q]) || !std::isfinite(amps[2 * q + 1]))
      return s->fail(FDTD_E_INVALID, "a current's amplitude must be finite");
  }
  if (int r = s->reconfigure()) return r;
  fdtd_waveform w;
  w.kind = (int32_t)wave[0];
  for (int q = 0; q < 5; q++) w.p[q] = wave[q + 1];
  s->waves.push_back(w);
  for (int64_t q = 0; q < count; q++) {
    const int64_t *p = at + 3 * q;
    s->currents.push_back(fdtd_injection{field, comps[q], s->index(p[0], p[1], p[2]), amps[2 * q],
                                         amps[2 * q + 1], (int32_t)s->waves.size() - 1, 0});
  }
  return 0;
}

}  // extern "C"

namespace {

// Simulation::links (src/fdtd/sources.rs:316-420): the couplings across a total-field /
// scattered-field surface among the values in [lo, hi) per axis, total() saying which side each
// value is on; values held at zero (cb = 0) neither take nor give one.
template <typename F>
std::vector<Link> surface_links(const pxs_sim *s, const int64_t lo[3], const int64_t hi[3],
                                const F &total) {
  const Grid &g = s->g;
  auto neighbour = [&](const int64_t at[3], int axis, bool forward, int64_t out[3]) -> bool {
    for (int q = 0; q < 3; q++) out[q] = at[q];
    const int64_t n = g.n[axis];
    if (forward) {
      if (at[axis] + 1 < n) out[axis] += 1;
      else if (s->periodic(axis)) out[axis] = 0;
      else return false;
    } else if (at[axis] > 0) {
      out[axis] -= 1;
    } else if (s->periodic(axis)) {
      out[axis] = n - 1;
    } else {
      return false;
    }
    return true;
  };
  auto index = [&](const int64_t at[3]) { return (at[2] * g.n[1] + at[1]) * g.n[0] + at[0]; };
  auto held = [&](int comp, const int64_t at[3]) { return s->cb[comp][index(at)] == 0.0; };
  struct Term { int comp; bool ok; int64_t from[3]; double coefficient; };
  std::vector<Link> out;
  for (int64_t k = lo[2]; k < hi[2]; k++)
    for (int64_t j = lo[1]; j < hi[1]; j++)
      for (int64_t i = lo[0]; i < hi[0]; i++) {
        const int64_t at[3] = {i, j, k};
        const int64_t r = index(at);
        for (int c = 0; c < 3; c++) {
          const int a = first_of(c), b = second_of(c);
          // E_c: curl = D_a H_b - D_b H_a, back differences
          if (!held(c, at)) {
            const bool inside = total(0, c, at);
            const double fa = s->kn[a][at[a]] / g.d[a], fb = s->kn[b][at[b]] / g.d[b];
            Term t[4];
            t[0] = {b, true, {i, j, k}, fa};
            t[1].comp = b;
            t[1].ok = neighbour(at, a, false, t[1].from);
            t[1].coefficient = -fa;
            t[2] = {a, true, {i, j, k}, -fb};
            t[3].comp = a;
            t[3].ok = neighbour(at, b, false, t[3].from);
            t[3].coefficient = fb;
            for (const Term &q : t)
              if (q.ok && total(1, q.comp, q.from) != inside)
                out.push_back(Link{0, c, r, (inside ? -1.0 : 1.0) * q.coefficient, 1, q.comp,
                                   {q.from[0], q.from[1], q.from[2]}});
          }
          // H_c: curl = D_a E_b - D_b E_a, forward differences
          const bool inside = total(1, c, at);
          const double fa = s->kh[a][at[a]] / g.d[a], fb = s->kh[b][at[b]] / g.d[b];
          Term t[4];
          t[0].comp = b;
          t[0].ok = neighbour(at, a, true, t[0].from);
          t[0].coefficient = fa;
          t[1] = {b, true, {i, j, k}, -fa};
          t[2].comp = a;
          t[2].ok = neighbour(at, b, true, t[2].from);
          t[2].coefficient = -fb;
          t[3] = {a, true, {i, j, k}, fb};
          for (const Term &q : t)
            if (q.ok && !held(q.comp, q.from) && total(0, q.comp, q.from) != inside)
              out.push_back(Link{1, c, r, (inside ? 1.0 : -1.0) * q.coefficient, 0, q.comp,
                                 {q.from[0], q.from[1], q.from[2]}});
        }
      }
  return out;
}

// Simulation::uniform (src/fdtd/sources.rs:509-522): every value of E on the surface in a
// lossless medium of eps, not a dispersive one.
bool surface_uniform(const pxs_sim *s, const std::vector<Link> &ls, double eps) {
  const double expected = s->dt / eps;
  for (const Link &l : ls) {
    const int c = l.target == 0 ? l.comp : l.from_comp;
    const int64_t r =
        l.target == 0 ? l.r : (l.from[2] * s->g.n[1] + l.from[1]) * s->g.n[0] + l.from[0];
    if (!(std::fabs(s->cb[c][r] - expected) <= 1e-12 * expected && s->ca[c][r] == 1.0 &&
          s->members.find((int64_t)c * s->N() + r) == s->members.end()))
      return false;
  }
  return true;
}

}  // namespace

extern "C" {

// Simulation::add_plane_wave / PlaneWaveRun::new (src/fdtd/sources.rs:716-951).
int pxs_add_plane_wave(pxs_sim *s, const int64_t low[3], const int64_t high[3],
                       const int64_t direction[3], const double polarization[3], double eps,
                       const double wave[6]) {
  if (!s || !low || !high || !direction || !polarization || !wave) return FDTD_E_INVALID;
  if (s->fields_dropped) return s->dropped();
  if (s->twin)  // Simulation::real_run (src/fdtd/sources.rs:209-221)
    return s->fail(FDTD_E_INVALID, "a total-field/scattered-field source needs real fields: with "
                                   "a Bloch phase, launch a current with it instead");
  auto gcd = [](int64_t a, int64_t b) {
    while (b != 0) {
      const int64_t t = a % b;
      a = b;
      b = t;
    }
    return a < 0 ? -a : a;
  };
  PlaneRun run;
  const int64_t divisor = gcd(gcd(direction[0], direction[1]), direction[2]);
  if (divisor == 0) return s->fail(FDTD_E_INVALID, "a plane wave's direction can't be zero");
  for (int a = 0; a < 3; a++) run.g[a] = direction[a] / divisor;
  if (!(std::isfinite(eps) && eps > 0.0))
    return s->fail(FDTD_E_INVALID, "the background's permittivity must be positive, got %g", eps);
  const int kind = (int)wave[0];
  if (kind < 0 || kind > 2 || (double)kind != wave[0])
    return s->fail(FDTD_E_INVALID, "no waveform of kind %g", wave[0]);
  bool faces[3];
  for (int a = 0; a < 3; a++) {
    const int64_t n = s->g.n[a];
    faces[a] = true;
    if (s->periodic(a)) {
      if (low[a] != 0 || high[a] != n || run.g[a] != 0)
        return s->fail(FDTD_E_INVALID,
                       "along the periodic axis %d the box must be whole (0 to %lld) and the "
                       "direction zero, got %lld to %lld and %lld",
                       a, (long long)n, (long long)low[a], (long long)high[a],
                       (long long)run.g[a]);
      faces[a] = false;
    } else {
      const int64_t lo = s->low[a], hi = s->high[a];
      if (low[a] < lo + 1 || high[a] + hi + 1 > n || low[a] >= high[a])
        return s->fail(FDTD_E_INVALID,
                       "along axis %d the box's faces, nodes %lld and %lld, must be in order and "
                       "a cell clear of the CPMLs (%lld and %lld cells) and the ends of %lld "
                       "cells",
                       a, (long long)low[a], (long long)high[a], (long long)lo, (long long)hi,
                       (long long)n);
    }
  }
  for (int a = 0; a < 3; a++) run.steps[a] = s->g.d[a];
  double gv[3], khat[3], pt[3];
  for (int a = 0; a < 3; a++) gv[a] = (double)run.g[a] / run.steps[a];
  double sq = 0.0;
  for (int a = 0; a < 3; a++) sq += gv[a] * gv[a];
  const double norm = std::sqrt(sq);
  for (int a = 0; a < 3; a++) khat[a] = gv[a] / norm;
  double along = 0.0;
  for (int a = 0; a < 3; a++) along += polarization[a] * khat[a];
  for (int a = 0; a < 3; a++) pt[a] = polarization[a] - along * khat[a];
  double size2 = 0.0;
  for (int a = 0; a < 3; a++) size2 += pt[a] * pt[a];
  const double size = std::sqrt(size2);
  if (!(std::isfinite(size) && size > 1e-12))
    return s->fail(FDTD_E_INVALID, "the polarization has nothing across the direction");
  for (int a = 0; a < 3; a++) pt[a] /= size;
  auto total = [&](int field, int comp, const int64_t at[3]) {
    for (int a = 0; a < 3; a++) {
      if (!faces[a]) continue;
      const int64_t t = twice(field, comp, a, at[a]);
      if (!(t >= 2 * low[a] && t <= 2 * high[a])) return false;
    }
    return true;
  };
  int64_t rlo[3], rhi[3];
  for (int a = 0; a < 3; a++) {
    rlo[a] = faces[a] ? low[a] - 1 : 0;
    rhi[a] = faces[a] ? high[a] + 2 : s->g.n[a];
  }
  const std::vector<Link> ls = surface_links(s, rlo, rhi, total);
  if (!surface_uniform(s, ls, eps))
    return s->fail(FDTD_E_INVALID,
                   "the medium on the box's surface must be uniform, with the permittivity %g "
                   "and no conductivity",
                   eps);
  int64_t least = 0, most = 0;
  for (int a = 0; a < 3; a++) {
    const int64_t t0 = faces[a] ? 2 * low[a] - 2 : 0, t1 = faces[a] ? 2 * high[a] + 2 : 0;
    least += std::min(run.g[a] * t0, run.g[a] * t1);
    most += std::max(run.g[a] * t0, run.g[a] * t1);
  }
  int64_t stride = 0;
  for (int a = 0; a < 3; a++) stride = std::max<int64_t>(stride, run.g[a] < 0 ? -run.g[a] : run.g[a]);
  const int64_t pad = stride, absorber = 200 * stride;
  const int64_t sheet_at = least - 4 * stride - 4;
  int64_t base = sheet_at - (absorber + 4 * stride + pad);
  base -= ((base % 2) + 2) % 2;
  const int64_t top = most + (4 * stride + absorber + pad);
  const int64_t len = top - base + 1;
  // a matched absorber at each end: sigma for E and sigma/eps for H, cubic
  const double sample = 1.0 / (2.0 * norm);
  const double depth = (double)absorber * sample;
  const double sqrt_eps = std::sqrt(eps);
  const double sigma_max = 50.0 * sqrt_eps / depth;
  const double dt = s->dt;
  run.ca.assign(len, 1.0);
  run.cb.assign(len, dt / eps);
  run.da.assign(len, 1.0);
  run.db.assign(len, dt);
  for (int64_t i = 0; i < len; i++) {
    double into;
    if (i < pad + absorber) into = (double)(pad + absorber - i);
    else if (i + pad + absorber >= len) into = (double)(i + pad + absorber + 1 - len);
    else continue;
    const double v = std::min(into / (double)absorber, 1.0);
    const double sigma = sigma_max * (v * (v * v));  // powi(v, 3): v (v v)
    const double half_e = sigma * dt / (2.0 * eps);
    run.ca[i] = (1.0 - half_e) / (1.0 + half_e);
    run.cb[i] = dt / eps / (1.0 + half_e);
    const double half_h = sigma / eps * dt / 2.0;
    run.da[i] = (1.0 - half_h) / (1.0 + half_h);
    run.db[i] = dt / (1.0 + half_h);
  }
  // the sheet: J = -2 n |G| p w where each component lives, halved over the two neighbours
  // where the sheet's sample is the other parity
  for (int c = 0; c < 3; c++) {
    if (pt[c] == 0.0) continue;
    const double j = -2.0 * sqrt_eps * norm * pt[c];
    if ((((sheet_at - run.g[c]) % 2) + 2) % 2 == 0) {
      run.sheet_comp.push_back(c);
      run.sheet_i.push_back(sheet_at - base);
      run.sheet_j.push_back(j);
    } else {
      for (int64_t l : {sheet_at - 1, sheet_at + 1}) {
        run.sheet_comp.push_back(c);
        run.sheet_i.push_back(l - base);
        run.sheet_j.push_back(0.5 * j);
      }
    }
  }
  run.base = base;
  run.pad = pad;
  run.len = len;
  run.e.assign(3 * len, 0.0);
  run.h.assign(3 * len, 0.0);
  run.wave.kind = kind;
  for (int q = 0; q < 5; q++) run.wave.p[q] = wave[q + 1];
  for (const Link &l : ls) {
    int64_t i;
    if (!run.sample(l.from_field, l.from_comp, l.from, &i))
      return s->fail(FDTD_E_INVALID, "the auxiliary grid doesn't span the box");
    PlaneRun::Coupling q{l.comp, l.r, l.weight, l.from_comp, i};
    (l.target == 0 ? run.on_e : run.on_h).push_back(q);
  }
  if (int r = s->reconfigure()) return r;
  s->plane_waves.push_back(std::move(run));
  return (int)s->plane_waves.size() - 1;
}

}  // extern "C"

namespace {

// Complex numbers with num-complex's arithmetic (the schoolbook product and quotient), which the
// reference's beam set-up uses.
struct Cx {
  double re = 0.0, im = 0.0;
};
inline Cx operator+(Cx a, Cx b) { return {a.re + b.re, a.im + b.im}; }
inline Cx operator-(Cx a, Cx b) { return {a.re - b.re, a.im - b.im}; }
inline Cx operator*(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline Cx operator*(Cx a, double s) { return {a.re * s, a.im * s}; }
inline Cx operator*(double s, Cx a) { return {s * a.re, s * a.im}; }
inline Cx operator/(Cx a, double s) { return {a.re / s, a.im / s}; }
inline Cx operator/(Cx a, Cx b) {
  const double n = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / n, (a.im * b.re - a.re * b.im) / n};
}
inline Cx operator-(Cx a) { return {-a.re, -a.im}; }
// e^z (src/portable/complex.rs:71-93), the reference's exp and sin/cos
inline Cx cexp(Cx z) {
  const double r = pxp::exp(z.re);
  if (z.im == 0.0) return {r, z.im};
  double sn, cs;
  pxp::sincos(z.im, &sn, &cs);
  return {r * cs, r * sn};
}
inline double cabs(Cx z) { return std::hypot(z.re, z.im); }
// the principal square root (src/portable/complex.rs:132-180) for finite z
inline Cx csqrt(Cx z) {
  const double x = z.re, y = z.im;
  if (y == 0.0) {
    if (!std::signbit(x)) return {std::sqrt(x), y};
    return {0.0, std::copysign(std::sqrt(-x), y)};
  }
  const double t = std::sqrt(0.5 * (std::fabs(x) + std::hypot(x, y)));
  if (x >= 0.0) return {t, y / (2.0 * t)};
  return {std::fabs(y) / (2.0 * t), std::copysign(t, y)};
}
// asin z for finite z of moderate size (src/portable/complex.rs:336-406: Hull, Fairgrieve and
// Tang's algorithm, ACM TOMS 23 (1997) 299, as FreeBSD's casin)
inline Cx casin(Cx z) {
  const double x = std::fabs(z.re), y = std::fabs(z.im);
  const double SMALL = 0x1p-27, TINY = 0x1p-500, LARGE = 0x1p500;
  double re, im;
  if (std::max(x, y) < SMALL) {
    re = x;
    im = y;
  } else if (std::max(x, y) >= LARGE) {
    re = std::atan2(x, y);
    im = std::log(std::hypot(x, y)) + 0.6931471805599453;
  } else if (y < TINY) {
    if (x < 1.0) {
      re = std::asin(x);
      im = y / std::sqrt((1.0 - x) * (1.0 + x));
    } else if (x == 1.0) {
      re = 1.5707963267948966;
      im = std::sqrt(y);
    } else {
      re = 1.5707963267948966;
      im = std::acosh(x);
    }
  } else {
    const double xp1 = x + 1.0, r = std::hypot(xp1, y), s = std::hypot(x - 1.0, y);
    const double a = 0.5 * (r + s), b = x / a, yy = y * y;
    if (b <= 0.6417) {
      re = std::asin(b);
    } else {
      const double apx = a + x;
      re = x <= 1.0 ? std::atan(x / std::sqrt(0.5 * apx * (yy / (r + xp1) + (s + (1.0 - x)))))
                    : std::atan(x / (y * std::sqrt(0.5 * (apx / (r + xp1) + apx / (s + (x - 1.0))))));
    }
    if (a <= 1.5) {
      const double am1 = x < 1.0 ? 0.5 * (yy / (r + xp1) + yy / (s + (1.0 - x)))
                                 : 0.5 * (yy / (r + xp1) + (s + (x - 1.0)));
      im = std::log1p(am1 + std::sqrt(am1 * (a + 1.0)));
    } else {
      im = std::log(a + std::sqrt(a * a - 1.0));
    }
  }
  return {std::copysign(re, z.re), std::copysign(im, z.im)};
}

double psin(double x) {
  double s, c;
  pxp::sincos(x, &s, &c);
  return s;
}
double pcos(double x) {
  double s, c;
  pxp::sincos(x, &s, &c);
  return c;
}

// The wavenumbers of a discrete Fourier series over n samples `step` apart
// (src/fdtd/sources.rs:1125-1130).
std::vector<double> wavenumbers(int64_t n, double step) {
  const int64_t low = -((n - 1) / 2);
  std::vector<double> out(n);
  for (int64_t m = 0; m < n; m++)
    out[m] = 6.283185307179586476925286766559 * (double)(low + m) / ((double)n * step);
  return out;
}

// The separable sum of src/fdtd/sources.rs:1278-1328: from samples to waves (sign -1) or back
// (+1), along b then along c.
std::vector<Cx> plane_transform(const std::vector<Cx> &values, const int64_t n[2],
                                const std::vector<double> k[2], const std::vector<double> x[2],
                                double sign) {
  const bool to_waves = sign < 0.0;
  std::vector<Cx> table[2];
  for (int t = 0; t < 2; t++) {
    const int64_t m = n[t];
    table[t].resize(m * m);
    for (int64_t p = 0; p < m; p++)
      for (int64_t q = 0; q < m; q++) {
        const int64_t wave = to_waves ? p : q, sample = to_waves ? q : p;
        table[t][p * m + q] = cexp(Cx{0.0, sign * k[t][wave] * x[t][sample]});
      }
  }
  std::vector<Cx> along_b(n[0] * n[1]), out(n[0] * n[1]);
  for (int64_t v = 0; v < n[1]; v++)
    for (int64_t p = 0; p < n[0]; p++) {
      Cx sum;
      for (int64_t q = 0; q < n[0]; q++) sum = sum + values[v * n[0] + q] * table[0][p * n[0] + q];
      along_b[v * n[0] + p] = sum;
    }
  for (int64_t p = 0; p < n[1]; p++)
    for (int64_t u = 0; u < n[0]; u++) {
      Cx sum;
      for (int64_t q = 0; q < n[1]; q++) sum = sum + along_b[q * n[0] + u] * table[1][p * n[1] + q];
      out[p * n[0] + u] = sum;
    }
  return out;
}

// The positions along axis.others() of field's component over the window (sources.rs:1255-1276).
void transverse_positions(const Grid &g, int axis, const int64_t lo[2], const int64_t n[2],
                          int field, int comp, std::vector<double> out[2]) {
  const int bc[2] = {first_of(axis), second_of(axis)};
  for (int t = 0; t < 2; t++) {
    const bool half = field == 0 ? comp == bc[t] : comp != bc[t];
    out[t].resize(n[t]);
    for (int64_t u = 0; u < n[t]; u++)
      out[t][u] = g.node(bc[t], lo[t] + u) + (half ? 0.5 * g.d[bc[t]] : 0.0);
  }
}

}  // namespace

extern "C" {

// Simulation::add_beam (src/fdtd/sources.rs:598-714, beam_profile :1042-1108, PlaneSpectrum
// :1110-1353): a Gaussian beam launched one way from the plane of nodes `plane` normal to `axis`,
// its tangential E on the plane the paraxial beam's, decomposed into the grid's own plane waves
// over the window clear of the CPMLs, each wave's normal wavenumber the grid's at the leapfrog's
// frequency; the waves' E and H on the planes the surface's couplings read become currents
// (phasor_surface), added with the waveform.
int pxs_add_beam(pxs_sim *s, int32_t axis, int64_t plane, int32_t direction,
                 const double centre[2], double waist, double focus, int32_t tilt, double angle,
                 int32_t parallel, double eps, const double wave[6]) {
  if (!s || !centre || !wave || axis < 0 || axis > 2 || tilt < 0 || tilt > 2)
    return FDTD_E_INVALID;
  if (s->fields_dropped) return s->dropped();
  if (s->twin)  // Simulation::real_run (src/fdtd/sources.rs:209-221)
    return s->fail(FDTD_E_INVALID, "a total-field/scattered-field source needs real fields: with "
                                   "a Bloch phase, launch a current with it instead");
  const Grid &g = s->g;
  const int a = axis, b = first_of(axis), c = second_of(axis);
  auto ok = [](double v) { return std::isfinite(v) && v > 0.0; };
  if (!ok(waist) || !ok(eps) || !std::isfinite(focus))
    return s->fail(FDTD_E_INVALID,
                   "a beam needs a positive waist and permittivity and a finite focus");
  if (tilt == axis || std::isnan(angle) || std::fabs(angle) >= 1.5707963267948966 ||
      (angle != 0.0 && !s->varies[tilt]))
    return s->fail(FDTD_E_INVALID,
                   "a beam tilts towards an axis across its plane along which the field varies, "
                   "by less than 90 degrees");
  if (s->periodic(axis))
    return s->fail(FDTD_E_INVALID, "a beam normal to axis %d needs ends along it, not periodic "
                                   "ones", a);
  const int64_t n = g.n[a];
  const int64_t lo_a = s->low[a], hi_a = s->high[a];
  if (plane < lo_a + 1 || plane + 2 + hi_a > n)
    return s->fail(FDTD_E_INVALID,
                   "the beam's plane %lld and the next must be clear of the CPMLs (%lld and %lld "
                   "cells) and the ends of %lld cells",
                   (long long)plane, (long long)lo_a, (long long)hi_a, (long long)n);
  // carrier_wavenumber (src/fdtd/sources.rs:487-507): the leapfrog's (2/dt) sin(omega dt/2)
  const int kind = (int)wave[0];
  if (kind != 0 && kind != 2)
    return s->fail(FDTD_E_INVALID,
                   "a beam needs a waveform with a carrier (a Gaussian or a continuous wave)");
  const double omega = 6.283185307179586476925286766559 * wave[1];
  if (!(omega * s->dt < 3.141592653589793238462643383279))
    return s->fail(FDTD_E_INVALID, "the carrier is beyond the time step's Nyquist frequency");
  const double k0 = 2.0 / s->dt * psin(omega * s->dt / 2.0);
  int64_t wlo[2], wn[2];
  const int bc[2] = {b, c};
  for (int t = 0; t < 2; t++) {
    if (s->periodic(bc[t])) {
      wlo[t] = 0;
      wn[t] = g.n[bc[t]];
    } else {
      wlo[t] = s->low[bc[t]];
      wn[t] = g.n[bc[t]] - s->high[bc[t]] - s->low[bc[t]];
    }
  }
  // beam_profile: the paraxial beam's E at a point, at unit amplitude
  const bool forward = direction >= 0;
  double u[3] = {0, 0, 0}, crossing[3] = {0, 0, 0}, wpt[3], sv[3] = {0, 0, 0}, pv[3];
  u[a] = (forward ? 1.0 : -1.0) * pcos(angle);
  u[tilt] = psin(angle);
  crossing[a] = g.node(a, plane);
  crossing[b] = centre[0];
  crossing[c] = centre[1];
  for (int q = 0; q < 3; q++) wpt[q] = crossing[q] + focus * u[q];
  sv[3 - a - tilt] = 1.0;
  pv[0] = sv[1] * u[2] - sv[2] * u[1];
  pv[1] = sv[2] * u[0] - sv[0] * u[2];
  pv[2] = sv[0] * u[1] - sv[1] * u[0];
  if (pv[tilt] < 0.0 || (pv[tilt] == 0.0 && pv[a] < 0.0))
    for (double &v : pv) v = -v;
  const double *evec = parallel ? pv : sv;
  const double k = std::sqrt(eps) * k0;
  const double rayleigh = k * waist * waist / 2.0;
  const int transverse = (int)s->varies[b] + (int)s->varies[c];
  auto profile = [&](const double r[3], Cx out[3]) {
    double rho[3] = {0, 0, 0};
    for (int q = 0; q < 3; q++)
      if (s->varies[q]) rho[q] = r[q] - wpt[q];
    double z = 0.0, r2 = 0.0;
    for (int q = 0; q < 3; q++) z += rho[q] * u[q];
    for (int q = 0; q < 3; q++) r2 += rho[q] * rho[q];
    r2 -= z * z;
    const Cx qq{z, -rayleigh};
    const Cx ratio = Cx{0.0, -rayleigh} / qq;
    const Cx envelope = transverse >= 2 ? ratio : csqrt(ratio);
    const Cx phase = Cx{0.0, 1.0} * (Cx{k * r2, 0.0} / (2.0 * qq) + Cx{k * z, 0.0});
    const Cx value = envelope * cexp(phase);
    for (int q = 0; q < 3; q++) out[q] = value * evec[q];
  };
  // PlaneSpectrum::new: the tangential E's waves over the window, going one way
  const std::vector<double> kt[2] = {wavenumbers(wn[0], g.d[b]), wavenumbers(wn[1], g.d[c])};
  std::vector<Cx> coefficients[2];
  for (int t = 0; t < 2; t++) {
    const int comp = bc[t];
    std::vector<double> pos[2];
    transverse_positions(g, a, wlo, wn, 0, comp, pos);
    std::vector<Cx> samples(wn[0] * wn[1]);
    for (int64_t v = 0; v < wn[1]; v++)
      for (int64_t w = 0; w < wn[0]; w++) {
        int64_t at[3];
        at[a] = plane;
        at[b] = wlo[0] + w;
        at[c] = wlo[1] + v;
        double p[3] = {g.node(0, at[0]), g.node(1, at[1]), g.node(2, at[2])};
        p[comp] += 0.5 * g.d[comp];
        Cx e[3];
        profile(p, e);
        samples[v * wn[0] + w] = e[comp];
      }
    coefficients[t] = plane_transform(samples, wn, kt, pos, -1.0);
    const double scale = 1.0 / (double)(wn[0] * wn[1]);
    for (Cx &x : coefficients[t]) x = x * scale;
  }
  const double step_a = g.d[a];
  const double sign = forward ? 1.0 : -1.0;
  const int64_t W = wn[0] * wn[1];
  std::vector<Cx> ka(W);
  std::vector<std::array<Cx, 3>> amplitude(W), big_k(W);
  for (int64_t mc = 0; mc < wn[1]; mc++)
    for (int64_t mb = 0; mb < wn[0]; mb++) {
      const double kb = 2.0 / g.d[b] * psin(kt[0][mb] * g.d[b] / 2.0);
      const double kc = 2.0 / g.d[c] * psin(kt[1][mc] * g.d[c] / 2.0);
      const double square = eps * k0 * k0 - kb * kb - kc * kc;
      const Cx normal =
          (square >= 0.0 ? Cx{std::sqrt(square), 0.0} : Cx{0.0, std::sqrt(-square)}) * sign;
      const Cx k_normal = 2.0 / step_a * casin(normal * step_a / 2.0);
      const int64_t w = mc * wn[0] + mb;
      const Cx eb = coefficients[0][w], ec = coefficients[1][w];
      std::array<Cx, 3> vec{}, kvec{};
      kvec[a] = normal;
      kvec[b] = Cx{kb, 0.0};
      kvec[c] = Cx{kc, 0.0};
      if (cabs(normal) > 1e-12 * k0) {
        vec[b] = eb;
        vec[c] = ec;
        vec[a] = -(Cx{kb, 0.0} * eb + Cx{kc, 0.0} * ec) / normal;
      }
      ka[w] = k_normal;
      amplitude[w] = vec;
      big_k[w] = kvec;
    }
  // the couplings of the beam's surface: forward, the total field from the plane on; back, up
  // to the plane after it
  auto total = [&](int field, int comp, const int64_t at[3]) {
    const int64_t t = twice(field, comp, a, at[a]);
    return forward ? t >= 2 * plane : t <= 2 * (plane + 1);
  };
  int64_t rlo[3], rhi[3];
  rlo[a] = plane - 1;
  rhi[a] = std::min(plane + 3, n);
  rlo[b] = wlo[0];
  rhi[b] = wlo[0] + wn[0];
  rlo[c] = wlo[1];
  rhi[c] = wlo[1] + wn[1];
  const std::vector<Link> ls = surface_links(s, rlo, rhi, total);
  if (!surface_uniform(s, ls, eps))
    return s->fail(FDTD_E_INVALID,
                   "the medium where the beam enters must be uniform, with its permittivity %g "
                   "and no conductivity",
                   eps);
  // the waves' E and H on each plane the couplings read (synthesize, sources.rs:1229-1252)
  std::map<std::tuple<int, int, int64_t>, std::vector<Cx>> planes;
  for (const Link &l : ls) {
    const auto key = std::make_tuple(l.from_field, l.from_comp, l.from[a]);
    if (planes.count(key)) continue;
    const int field = l.from_field, comp = l.from_comp;
    const double offset = (double)(twice(field, comp, a, l.from[a]) - 2 * plane) * step_a / 2.0;
    std::vector<Cx> co(W);
    for (int64_t w = 0; w < W; w++) {
      Cx value;
      if (field == 0) {
        value = amplitude[w][comp];
      } else {
        const int x = first_of(comp), y = second_of(comp);
        value = (big_k[w][x] * amplitude[w][y] - big_k[w][y] * amplitude[w][x]) / k0;
      }
      co[w] = value * cexp(Cx{0.0, 1.0} * ka[w] * offset);
    }
    std::vector<double> pos[2];
    transverse_positions(g, a, wlo, wn, field, comp, pos);
    planes[key] = plane_transform(co, wn, kt, pos, 1.0);
  }
  auto incident = [&](int field, int comp, const int64_t at[3]) -> Cx {
    const int64_t uu = at[b], vv = at[c];
    if (uu < wlo[0] || uu >= wlo[0] + wn[0] || vv < wlo[1] || vv >= wlo[1] + wn[1]) return Cx{};
    auto it = planes.find(std::make_tuple(field, comp, at[a]));
    if (it == planes.end()) return Cx{};
    return it->second[(vv - wlo[1]) * wn[0] + (uu - wlo[0])];
  };
  // phasor_surface (sources.rs:420-455): the couplings' currents, J for E and M for H, by value
  if (int r = s->reconfigure()) return r;
  for (int field = 0; field < 2; field++) {
    std::map<std::pair<int, int64_t>, Cx> values;
    for (const Link &l : ls) {
      if (l.target != field) continue;
      Cx &v = values[std::make_pair(l.comp, l.r)];
      v = v + l.weight * incident(l.from_field, l.from_comp, l.from);
    }
    bool any = false;
    for (auto &kv : values)
      if (kv.second.re != 0.0 || kv.second.im != 0.0) any = true;
    if (!any) continue;
    fdtd_waveform w;
    w.kind = kind;
    for (int q = 0; q < 5; q++) w.p[q] = wave[q + 1];
    s->waves.push_back(w);
    for (auto &kv : values)
      if (kv.second.re != 0.0 || kv.second.im != 0.0)
        s->currents.push_back(fdtd_injection{field, kv.first.first, kv.first.second, kv.second.re,
                                             kv.second.im, (int32_t)s->waves.size() - 1, 0});
  }
  return 0;
}

// Simulation::incident (src/fdtd/sources.rs:729-767): plane wave n's incident field now (E at the
// current time, H half a step behind) at a value; 0 beyond its auxiliary grid.
int pxs_incident(pxs_sim *s, int32_t n, int32_t field, int32_t comp, int64_t i, int64_t j,
                 int64_t k, double *out) {
  if (!s || !out) return FDTD_E_INVALID;
  if (n < 0 || n >= (int32_t)s->plane_waves.size() || field < 0 || field > 1 || comp < 0 ||
      comp > 2 || !s->inside(i, j, k))
    return s->fail(FDTD_E_INVALID, "no plane wave %d, or the value is outside the grid", (int)n);
  if (n < s->aux_on_device && s->ctx) {
    PlaneRun &p = s->plane_waves[n];
    if (int r = fdtd_plane_wave_state(s->ctx, n, p.e.data(), p.h.data()))
      return s->fail(r, "%s", fdtd_last_error(s->ctx));
  }
  const PlaneRun &p = s->plane_waves[n];
  const int64_t at[3] = {i, j, k};
  int64_t q;
  *out = p.sample(field, comp, at, &q) ? (field == 0 ? p.e : p.h)[comp * p.len + q] : 0.0;
  return 0;
}

int pxs_add_dipole(pxs_sim *s, int32_t field, int32_t comp, const double pos[3], double are,
                   double aim, const double wave[6]) {
  // Simulation::add_dipole (src/fdtd/sources.rs:248-315), no Bloch phase
  if (!std::isfinite(are) || !std::isfinite(aim) || !std::isfinite(pos[0]) ||
      !std::isfinite(pos[1]) || !std::isfinite(pos[2]))
    return s->fail(FDTD_E_INVALID, "a dipole must be finite");
  int64_t idx[3][2];
  double wt[3][2], volume = 1.0;
  for (int axis = 0; axis < 3; axis++) {
    int64_t n = s->g.n[axis];
    if (!s->varies[axis]) {
      idx[axis][0] = idx[axis][1] = 0;
      wt[axis][0] = 1.0;
      wt[axis][1] = 0.0;
      continue;
    }
    volume *= s->g.d[axis];
    bool half = field == 0 ? comp == axis : comp != axis;
    double first = s->g.node(axis, 0) + (half ? 0.5 * s->g.d[axis] : 0.0);
    double sp = (pos[axis] - first) / s->g.d[axis];
    if (!s->periodic(axis) && !(sp >= 0.0 && sp <= (double)(n - 1)))
      return s->fail(FDTD_E_INVALID, "the dipole is outside its component's values along axis %d",
                     axis);
    double m = std::floor(sp), f = sp - m;
    if (s->periodic(axis)) {
      int64_t m0 = (int64_t)m;
      idx[axis][0] = ((m0 % n) + n) % n;
      idx[axis][1] = (((m0 + 1) % n) + n) % n;
    } else {
      idx[axis][0] = (int64_t)m;
      idx[axis][1] = std::min((int64_t)m + 1, n - 1);
    }
    wt[axis][0] = 1.0 - f;
    wt[axis][1] = f;
  }
  std::map<int64_t, std::pair<double, double>> values;
  if (s->twin) {
    // a complex run: a value beyond a periodic end is its image's, e^(-ikL turns) times it
    // (Bloch::image, src/fdtd/bloch.rs:85-95); the weights complex, multiplied as num-complex
    double cw[3][2][2];
    for (int axis = 0; axis < 3; axis++)
      for (int q = 0; q < 2; q++) {
        double ir = 1.0, ii = 0.0;
        if (s->varies[axis] && s->periodic(axis)) {
          const bool half = field == 0 ? comp == axis : comp != axis;
          const double first = s->g.node(axis, 0) + (half ? 0.5 * s->g.d[axis] : 0.0);
          const int64_t n = s->g.n[axis];
          const int64_t m = (int64_t)std::floor((pos[axis] - first) / s->g.d[axis]) + q;
          const int64_t turns = m >= 0 ? m / n : -((-m + n - 1) / n);
          s->image(axis, turns, &ir, &ii);
        }
        cw[axis][q][0] = ir * wt[axis][q];
        cw[axis][q][1] = ii * wt[axis][q];
      }
    for (int p = 0; p < 2; p++)
      for (int q = 0; q < 2; q++)
        for (int r = 0; r < 2; r++) {
          const double xr = cw[0][p][0] * cw[1][q][0] - cw[0][p][1] * cw[1][q][1];
          const double xi = cw[0][p][0] * cw[1][q][1] + cw[0][p][1] * cw[1][q][0];
          const double wr = xr * cw[2][r][0] - xi * cw[2][r][1];
          const double wi = xr * cw[2][r][1] + xi * cw[2][r][0];
          if (wr == 0.0 && wi == 0.0) continue;
          const double sr = wr / volume, si = wi / volume;
          auto &acc = values[s->index(idx[0][p], idx[1][q], idx[2][r])];
          acc.first = acc.first + (are * sr - aim * si);
          acc.second = acc.second + (are * si + aim * sr);
        }
  } else
  for (int p = 0; p < 2; p++)
    for (int q = 0; q < 2; q++)
      for (int r = 0; r < 2; r++) {
        double w = wt[0][p] * wt[1][q] * wt[2][r];
        if (w == 0.0) continue;
        double sc = w / volume;
        auto &acc = values[s->index(idx[0][p], idx[1][q], idx[2][r])];
        acc.first = acc.first + (are * sc - aim * 0.0);
        acc.second = acc.second + (are * 0.0 + aim * sc);
      }
  if (s->twin) {  // the values' imaginary part, -i times them, on the imaginary part
    std::vector<int32_t> comps;
    std::vector<int64_t> at;
    std::vector<double> im;
    for (auto &kv : values) {
      comps.push_back(comp);
      at.push_back(kv.first % s->g.n[0]);
      at.push_back((kv.first / s->g.n[0]) % s->g.n[1]);
      at.push_back(kv.first / (s->g.n[0] * s->g.n[1]));
      im.push_back(0.0 * kv.second.first - (-1.0) * kv.second.second);
      im.push_back(0.0 * kv.second.second + (-1.0) * kv.second.first);
    }
    if (int r = pxs_add_current(s->twin, field, (int64_t)comps.size(), comps.data(), at.data(),
                                im.data(), wave))
      return s->fail(r, "%s", s->twin->error.c_str());
  }
  if (int r = s->reconfigure()) return r;
  fdtd_waveform wv;
  wv.kind = (int32_t)wave[0];
  for (int q = 0; q < 5; q++) wv.p[q] = wave[q + 1];
  s->waves.push_back(wv);
  for (auto &kv : values)
    s->currents.push_back(fdtd_injection{field, comp, kv.first, kv.second.first, kv.second.second,
                                         (int32_t)s->waves.size() - 1, 0});
  return 0;
}

int pxs_add_probe(pxs_sim *s, int32_t field, int32_t comp, int64_t i, int64_t j, int64_t k) {
  if (s && s->twin)  // src/fdtd.rs:1079-1081
    if (int r = pxs_add_probe(s->twin, field, comp, i, j, k); r < 0)
      return s->fail(r, "%s", s->twin->error.c_str());
  if (!s->inside(i, j, k) || comp < 0 || comp > 2)
    return s->fail(FDTD_E_INVALID, "(%lld, %lld, %lld) is outside the grid", (long long)i,
                   (long long)j, (long long)k);
  if (int r = s->reconfigure()) return r;
  s->probes.push_back(Probe{field, comp, s->index(i, j, k), {}});
  return (int)s->probes.size() - 1;
}

int pxs_add_dft(pxs_sim *s, const int64_t low[3], const int64_t high[3], int32_t nf,
                const double *freqs) {
  if (int r = s->check_frequencies(nf, freqs)) return r;
  for (int a = 0; a < 3; a++)
    if (low[a] < 0 || high[a] >= s->g.n[a] || low[a] > high[a])
      return s->fail(FDTD_E_INVALID, "a transform's box must run from low to high indices on the grid");
  if (int r = s->reconfigure()) return r;
  Monitor m;
  m.freqs.assign(freqs, freqs + nf);
  s->monitors.push_back(m);
  int mi = (int)s->monitors.size() - 1;
  for (int field = 0; field < 2; field++)
    for (int c = 0; c < 3; c++) {
      Series sr;
      sr.field = field;
      sr.comp = c;
      sr.monitor = mi;
      for (int a = 0; a < 3; a++) {
        sr.lo[a] = low[a];
        sr.len[a] = high[a] - low[a] + 1;
      }
      sr.sums.assign(2 * sr.volume() * nf, 0.0);
      s->monitors[mi].series.push_back(s->series.size());
      s->series.push_back(sr);
    }
  s->dft_monitor.push_back(mi);
  return (int)s->dft_monitor.size() - 1;
}

int pxs_add_flux(pxs_sim *s, int32_t axis, int64_t plane, const int64_t window[4], int32_t nf,
                 const double *freqs) {
  if (int r = s->check_frequencies(nf, freqs)) return r;
  if (axis < 0 || axis > 2 || plane < 0 || plane + 1 >= s->g.n[axis])
    return s->fail(FDTD_E_INVALID, "a flux plane after node %lld needs node %lld on the grid",
                   (long long)plane, (long long)plane + 1);
  FluxFace F{axis, plane, {{window[0], window[1]}, {window[2], window[3]}}, 1.0, 0};
  for (int sl = 0; sl < 2; sl++) {
    int along = sl == 0 ? first_of(axis) : second_of(axis);
    if (F.win[sl][0] >= 0 && !(F.win[sl][0] < F.win[sl][1] && F.win[sl][1] < s->g.n[along]))
      return s->fail(FDTD_E_INVALID, "a flux plane's window must run from one half-plane to a later one on the grid");
  }
  if (int r = s->reconfigure()) return r;
  Monitor m;
  m.freqs.assign(freqs, freqs + nf);
  s->monitors.push_back(m);
  s->add_plane_series(F, (int)s->monitors.size() - 1, nf);
  s->fluxes.push_back({F});
  return (int)s->fluxes.size() - 1;
}

int pxs_add_flux_box(pxs_sim *s, const int64_t planes[6], int32_t nf, const double *freqs) {
  if (int r = s->check_frequencies(nf, freqs)) return r;
  std::vector<FluxFace> faces;
  for (int axis = 0; axis < 3; axis++) {
    int64_t lo = planes[2 * axis], hi = planes[2 * axis + 1];
    int b = first_of(axis), c = second_of(axis);
    if (lo >= hi || lo < 0 || hi + 1 >= s->g.n[axis])
      return s->fail(FDTD_E_INVALID, "a flux box's planes must be from low to high on the grid");
    for (int side = 0; side < 2; side++)
      faces.push_back(FluxFace{axis, side == 0 ? lo : hi,
                               {{planes[2 * b], planes[2 * b + 1]}, {planes[2 * c], planes[2 * c + 1]}},
                               side == 0 ? -1.0 : 1.0, 0});
  }
  if (int r = s->reconfigure()) return r;
  for (auto &F : faces) {
    Monitor m;
    m.freqs.assign(freqs, freqs + nf);
    s->monitors.push_back(m);
    s->add_plane_series(F, (int)s->monitors.size() - 1, nf);
  }
  s->fluxes.push_back(faces);
  return (int)s->fluxes.size() - 1;
}

int pxs_run(pxs_sim *s, int64_t steps) { return s->run(steps); }

double pxs_time(const pxs_sim *s) { return (double)s->steps * s->dt; }

// Simulation::run_until (src/fdtd.rs:1161-1167): the steps that bring the time to `time`.
int pxs_run_until(pxs_sim *s, double time) {
  int64_t count = 0;
  while ((double)(s->steps + count) * s->dt < time) count++;
  return s->run(count);
}

namespace {

// Growth (src/fdtd/monitors.rs:663-717): the fields rising at each of the last `needed` checks,
// to 1e3 times their level before the first of them.
struct Growth {
  size_t needed;
  double start = 0.0, last = 0.0;
  size_t rises = 0;
  explicit Growth(size_t n) : needed(n) {}
  static Growth after(double pulse_end, double check) {
    return Growth(std::max<size_t>((size_t)std::ceil(pulse_end / check) + 1, 4));
  }
  bool check(double level, double *factor) {
    if (last > 0.0 && level > last) {
      if (rises == 0) start = last;
      rises++;
    } else {
      rises = 0;
    }
    last = level;
    if (rises >= needed && level >= 1e3 * start) {
      *factor = level / start;
      return true;
    }
    return false;
  }
};

// When the last source ends (monitors.rs:719-740): a pulse 6 widths after its peak; false for a
// continuous wave, which never ends. No source: 0.
bool sources_end(const pxs_sim *s, double *end) {
  *end = 0.0;
  for (const fdtd_waveform &w : s->waves) {
    if (w.kind == 0) *end = std::max(*end, w.p[2] + 6.0 * w.p[1]);
    else if (w.kind == 1) *end = std::max(*end, w.p[1] + 6.0 * w.p[0]);
    else return false;
  }
  return true;
}

}  // namespace

// Simulation::run_until_decayed (src/fdtd/monitors.rs:742-838): blocks of `interval` until, over
// a whole block, |F|^2 at every probe has stayed at or below `fraction` of its largest since the
// probe was added (*decayed = 1), or the time reaches `limit` (*decayed = 0). After the sources
// end it watches for late growth: FDTD_E_GROWING, with growing[0..2] = the time, the checks in a
// row and the factor.
int pxs_run_until_decayed(pxs_sim *s, int32_t count, const int32_t *probes, double fraction,
                          double interval, double limit, int32_t *decayed, double *growing) {
  if (count <= 0 || !probes || !(fraction > 0.0 && fraction < 1.0) ||
      !(std::isfinite(interval) && interval > 0.0) || !std::isfinite(limit))
    return s->fail(FDTD_E_INVALID,
                   "running until the fields decay needs probes, a fraction in (0, 1), a positive "
                   "interval and a finite limit, got %d probes, %g, %g and %g",
                   count, fraction, interval, limit);
  for (int q = 0; q < count; q++)
    if (probes[q] < 0 || probes[q] >= (int32_t)s->probes.size())
      return s->fail(FDTD_E_INVALID, "no probe %d", probes[q]);
  *decayed = 0;
  double end = 0.0;
  const bool ends = sources_end(s, &end);
  Growth growth = Growth::after(end, interval);
  while (pxs_time(s) < limit) {
    const size_t from = s->probes[probes[0]].values.size();
    const double began = pxs_time(s);
    if (int r = pxs_run_until(s, std::min(began + interval, limit))) return r;
    bool all = true;
    double level = 0.0;
    for (int q = 0; q < count; q++) {
      const std::vector<double> &v = s->probes[probes[q]].values;
      double peak = 0.0, recent = 0.0;
      for (size_t m = 0; m < v.size(); m++) {
        peak = std::max(peak, v[m] * v[m]);
        if (m >= std::min(from, v.size())) recent = std::max(recent, v[m] * v[m]);
      }
      if (!(peak > 0.0 && recent <= fraction * peak)) all = false;
      level = std::max(level, recent);
    }
    if (all) {
      *decayed = 1;
      return 0;
    }
    double factor = 0.0;
    if (ends && began >= end && growth.check(level, &factor)) {
      if (growing) {
        growing[0] = pxs_time(s);
        growing[1] = (double)growth.needed;
        growing[2] = factor;
      }
      return s->fail(FDTD_E_GROWING,
                     "the fields grew again, and the run stopped at %.0f um/c: |field|^2 at the "
                     "probes rose at %zu checks in a row, to %.1e times its level before",
                     pxs_time(s), growth.needed, factor);
    }
  }
  return 0;
}
double pxs_dt(const pxs_sim *s) { return s->dt; }
int64_t pxs_steps(const pxs_sim *s) { return s->steps; }

int pxs_get_field(pxs_sim *s, int32_t field, int32_t comp, double *out) {
  if (s->fields_dropped) return s->dropped();
  if (int r = s->pull()) return r;
  const std::vector<double> &v = field == 0 ? s->e : s->h;
  int64_t N = s->N();
  if (v.empty()) std::fill(out, out + N, 0.0);
  else std::copy(v.begin() + comp * N, v.begin() + (comp + 1) * N, out);
  return 0;
}

int pxs_set_field(pxs_sim *s, int32_t field, int32_t comp, const double *in) {
  if (s->fields_dropped) return s->dropped();
  if (int r = s->pull()) return r;
  std::vector<double> &v = field == 0 ? s->e : s->h;
  int64_t N = s->N();
  if (v.empty()) v.assign(3 * N, 0.0);
  std::copy(in, in + N, v.begin() + comp * N);
  s->device_fresh = false;
  return 0;
}

int pxs_is_complex(const pxs_sim *s) { return s && s->twin ? 1 : 0; }

int pxs_get_field_imag(pxs_sim *s, int32_t field, int32_t comp, double *out) {
  if (!s->twin) return s->fail(FDTD_E_INVALID, "the fields are real: no Bloch phase");
  if (int r = pxs_get_field(s->twin, field, comp, out)) return s->fail(r, "%s", s->twin->error.c_str());
  return 0;
}

int pxs_set_field_imag(pxs_sim *s, int32_t field, int32_t comp, const double *in) {
  if (!s->twin) return s->fail(FDTD_E_INVALID, "the fields are real: no Bloch phase");
  if (int r = pxs_set_field(s->twin, field, comp, in)) return s->fail(r, "%s", s->twin->error.c_str());
  return 0;
}

int64_t pxs_probe_imag(pxs_sim *s, int32_t n, double *out) {
  if (!s->twin) return s->fail(FDTD_E_INVALID, "the fields are real: no Bloch phase");
  return pxs_probe(s->twin, n, out);
}

int64_t pxs_probe(pxs_sim *s, int32_t n, double *out) {
  if (n < 0 || n >= (int32_t)s->probes.size()) return s->fail(FDTD_E_INVALID, "no probe %d", n);
  const auto &v = s->probes[n].values;
  if (out) std::copy(v.begin(), v.end(), out);
  return (int64_t)v.size();
}

int64_t pxs_transforms(pxs_sim *s, double *out) {
  if (int r = s->pull_sums()) return r;
  int64_t at = 0;
  // layout order: the transforms (add_dft), then the fluxes' faces (Monitors::all)
  std::vector<size_t> order;
  for (int mi : s->dft_monitor)
    for (size_t q : s->monitors[mi].series) order.push_back(q);
  for (auto &faces : s->fluxes)
    for (auto &F : faces)
      for (size_t q = F.series0; q < F.series0 + 4; q++) order.push_back(q);
  for (size_t q : order) {
    const Series &sr = s->series[q];
    if (out) std::copy(sr.sums.begin(), sr.sums.end(), out + 2 * at);
    at += (int64_t)sr.sums.size() / 2;
  }
  return at;
}

int pxs_flux(pxs_sim *s, int32_t n, double *out) {
  if (n < 0 || n >= (int32_t)s->fluxes.size()) return s->fail(FDTD_E_INVALID, "no flux monitor %d", n);
  if (int r = s->pull_sums()) return r;
  const auto &faces = s->fluxes[n];
  int nf = (int)(s->series[faces[0].series0].sums.size() / 2 / s->series[faces[0].series0].volume());
  for (int f = 0; f < nf; f++) {
    double total = 0.0;
    for (auto &F : faces) total += F.sign * s->face_flux(F, f);
    out[f] = total;
  }
  return nf;
}

int64_t pxs_tables(const pxs_sim *s, int32_t which, double *out) {
  int64_t at = 0;
  auto put = [&](double v) {
    if (out) out[at] = v;
    at++;
  };
  if (which == 0 || which == 1) {
    for (int c = 0; c < 3; c++)
      for (double v : (which == 0 ? s->ca[c] : s->cb[c])) put(v);
  } else if (which == 2 || which == 3) {
    for (int c = 0; c < 3; c++)
      for (int64_t m = 0; m < s->g.n[c]; m++) put((which == 2 ? s->kn[c][m] : s->kh[c][m]) / s->g.d[c]);
  } else if (which == 4) {
    for (const SlabInfo &sl : s->slabs) {
      put(sl.field);
      put(sl.comp);
      put(sl.axis);
      put((double)sl.from);
      put((double)sl.count);
      for (double v : sl.b) put(v);
      for (double v : sl.a) put(v);
    }
  } else if (which == 5) {  // the media groups: chi, poles, members (comp, index, scale)
    for (const MediaGroup &G : s->groups) {
      put(G.chi);
      put((double)(G.poles.size() / 3));
      for (double v : G.poles) put(v);
      put((double)G.r.size());
      for (size_t v = 0; v < G.r.size(); v++) {
        put(G.comp[v]);
        put((double)G.r[v]);
        put(G.scale[v]);
      }
    }
  }
  return at;
}

fdtd_ctx *pxs_engine(pxs_sim *s) { return s ? s->ctx : nullptr; }

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Batches of simulations (photonoxide_batch.h) at the level of this API: each simulation's
// engine is set up as for pxs_run before the batch steps it, and its step count and probes are
// brought up to date after.

struct pxs_batch {
  std::string error;
  std::vector<pxs_sim *> sims;
  fdtd_batch *batch = nullptr;
};

extern "C" {

int pxs_batch_create(int32_t count, pxs_sim *const *sims, pxs_batch **out) {
  if (!out) return FDTD_E_INVALID;
  pxs_batch *b = new pxs_batch();
  *out = b;
  if (count <= 0 || !sims) {
    b->error = "a batch needs simulations";
    return FDTD_E_INVALID;
  }
  std::vector<fdtd_ctx *> ctxs;
  for (int i = 0; i < count; i++) {
    if (!sims[i]) {
      b->error = "a batch's simulation is missing";
      return FDTD_E_INVALID;
    }
    if (sims[i]->twin) {
      b->error = "simulation " + std::to_string(i) + " is a complex run (a Bloch phase), which "
                 "the batch does not step";
      return FDTD_E_INVALID;
    }
    if (int r = sims[i]->prepare()) {
      b->error = "simulation " + std::to_string(i) + ": " + sims[i]->error;
      return r;
    }
    b->sims.push_back(sims[i]);
    ctxs.push_back(sims[i]->ctx);
  }
  int r = fdtd_batch_create(count, ctxs.data(), &b->batch);
  if (r) b->error = fdtd_batch_last_error(b->batch);
  return r;
}

const char *pxs_batch_last_error(const pxs_batch *b) { return b ? b->error.c_str() : "no batch"; }

int pxs_batch_run(pxs_batch *b, int64_t steps) {
  if (!b || !b->batch) return FDTD_E_INVALID;
  if (steps <= 0) return 0;
  std::vector<int64_t> first;
  for (size_t i = 0; i < b->sims.size(); i++) {
    pxs_sim *s = b->sims[i];
    if (int r = s->prepare()) {
      b->error = "simulation " + std::to_string(i) + ": " + s->error;
      return r;
    }
    first.push_back(s->steps);
  }
  if (int r = fdtd_batch_run(b->batch, steps, first.data())) {
    b->error = fdtd_batch_last_error(b->batch);
    return r;
  }
  for (size_t i = 0; i < b->sims.size(); i++)
    if (int r = b->sims[i]->finish(steps)) {
      b->error = "simulation " + std::to_string(i) + ": " + b->sims[i]->error;
      return r;
    }
  return 0;
}

int pxs_batch_tile(const pxs_batch *b, int32_t *width, int32_t *height) {
  return b ? fdtd_batch_tile(b->batch, width, height) : FDTD_E_INVALID;
}

int pxs_batch_set_tile(pxs_batch *b, int32_t width, int32_t height) {
  if (!b) return FDTD_E_INVALID;
  int r = fdtd_batch_set_tile(b->batch, width, height);
  if (r) b->error = fdtd_batch_last_error(b->batch);
  return r;
}

int64_t pxs_batch_launches(const pxs_batch *b) { return b ? fdtd_batch_launches(b->batch) : 0; }

void pxs_batch_destroy(pxs_batch *b) {
  if (!b) return;
  fdtd_batch_destroy(b->batch);
  delete b;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// The adjoint (photonoxide_adjoint.h) at the level of this API, and the flux's derivative by the
// transform sums that feeds it.

struct pxs_adjoint {
  std::string error;
  pxs_sim *sim = nullptr;
  fdtd_adjoint *adj = nullptr;
  int64_t steps = 0;
};

extern "C" {

int pxs_media_counts(const pxs_sim *s, int64_t *out) {
  out[0] = out[1] = 0;
  for (const MediaGroup &G : s->groups) {
    out[0] += (int64_t)G.comp.size();
    out[1] += (int64_t)G.comp.size() * (int64_t)(G.poles.size() / 3);
  }
  return 0;
}

int pxs_flux_gradient(pxs_sim *s, int32_t n, int32_t f, double scale, double *grad) {
  if (n < 0 || n >= (int32_t)s->fluxes.size()) return s->fail(FDTD_E_INVALID, "no flux monitor %d", n);
  if (int r = s->pull_sums()) return r;
  const auto &faces = s->fluxes[n];
  int nf = (int)(s->series[faces[0].series0].sums.size() / 2 / s->series[faces[0].series0].volume());
  if (f < 0 || f >= nf) return s->fail(FDTD_E_INVALID, "flux monitor %d has no frequency %d", n, f);
  for (auto &F : faces) s->face_flux_grad(F, f, F.sign * scale, grad);
  return 0;
}

int pxs_adjoint_create(pxs_sim *s, int64_t steps, int32_t segment, int64_t count,
                       const int32_t *component, const int64_t *r, pxs_adjoint **out) {
  if (!out) return FDTD_E_INVALID;
  pxs_adjoint *a = new pxs_adjoint();
  *out = a;
  if (!s) {
    a->error = "no simulation";
    return FDTD_E_INVALID;
  }
  if (s->twin) {
    a->error = "the adjoint does not step a complex run (a Bloch phase)";
    return FDTD_E_INVALID;
  }
  a->sim = s;
  a->steps = steps;
  if (int q = s->prepare()) {
    a->error = s->error;
    return q;
  }
  int q = fdtd_adjoint_create(s->ctx, steps, segment, count, component, r, &a->adj);
  if (q) a->error = fdtd_adjoint_last_error(a->adj);
  return q;
}

const char *pxs_adjoint_last_error(const pxs_adjoint *a) { return a ? a->error.c_str() : "no adjoint"; }

int pxs_adjoint_forward(pxs_adjoint *a) {
  if (!a || !a->adj) return FDTD_E_INVALID;
  pxs_sim *s = a->sim;
  if (int q = s->prepare()) {
    a->error = s->error;
    return q;
  }
  if (int q = fdtd_adjoint_forward(a->adj, s->steps)) {
    a->error = fdtd_adjoint_last_error(a->adj);
    return q;
  }
  if (int q = s->finish(a->steps)) {
    a->error = s->error;
    return q;
  }
  return 0;
}

int pxs_adjoint_backward(pxs_adjoint *a, const double *grad_sums, double *grad_cb) {
  if (!a || !a->adj) return FDTD_E_INVALID;
  int q = fdtd_adjoint_backward(a->adj, grad_sums, grad_cb);
  if (q) a->error = fdtd_adjoint_last_error(a->adj);
  return q;
}

void pxs_adjoint_destroy(pxs_adjoint *a) {
  if (!a) return;
  fdtd_adjoint_destroy(a->adj);
  delete a;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Serving: a resident loop that admits simulations (jobs) under a device-memory budget, keeps
// the admitted ones on the device and steps them together, chunk by chunk: the 2D TE jobs in one
// batch (one launch per step for all of them), the others each on its own stream, all in flight
// at once. A job that has taken its steps is read back to the host and its device memory freed,
// which admits the next. No counterpart in the reference (one Simulation at a time).

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// f(0) .. f(count-1) on up to 8 threads (each with the device current): jobs' host work and
// launches are independent, each on its own engine and stream.
template <typename F>
void parallel_for(int count, int device, F f) {
  const int threads = std::min(count, 8);
  if (threads <= 1) {
    for (int i = 0; i < count; i++) f(i);
    return;
  }
  std::atomic<int> next(0);
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; t++)
    pool.emplace_back([&] {
      cudaSetDevice(device);
      for (int i; (i = next++) < count;) f(i);
    });
  for (std::thread &t : pool) t.join();
}

enum { JOB_QUEUED = 0, JOB_RUNNING = 1, JOB_DONE = 2, JOB_FAILED = 3, JOB_CANCELLED = 4 };

struct ServerJob {
  int64_t id = 0;
  pxs_sim *sim = nullptr;
  int64_t steps = 0, done = 0;
  int state = JOB_QUEUED;
  bool te = false, prepared = false, keep_fields = true;
  size_t bytes = 0;
  double submitted = 0, started = 0, finished = 0;
  std::string error;
};

}  // namespace

struct pxs_server {
  std::string error;
  size_t budget = 0, used = 0;
  int max_active = 64;
  int64_t chunk = 500;
  int device = 0;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<ServerJob *> queue;
  std::vector<ServerJob *> active;
  std::map<int64_t, ServerJob *> jobs;
  int64_t next_id = 1;
  bool stop = false;
  std::thread loop;
  // the loop's own
  fdtd_batch *batch = nullptr;
  std::vector<ServerJob *> batch_jobs;
  double cell_updates = 0.0;
  int64_t chunks = 0;
  double launch_s = 0.0, host_s = 0.0, wait_s = 0.0;  // the loop's time: queuing, set-up and
                                                       // read-back, waiting for the device

  void finish_job(ServerJob *j, int state, const std::string &why) {
    // called with mu held
    j->state = state;
    j->error = why;
    j->finished = now_s();
    used -= j->bytes;
  }

  void run_loop() {
    cudaSetDevice(device);
    std::vector<ServerJob *> finished;  // stepped to their end; read back in the next round
    for (;;) {
      std::vector<ServerJob *> admitted, te, other;
      {
        std::unique_lock<std::mutex> lock(mu);
        cv.wait(lock, [&] { return stop || !queue.empty() || !active.empty() || !finished.empty(); });
        if (stop) break;
        // admission in arrival order, while slots and memory last
        while (!queue.empty() && (int)active.size() < max_active) {
          ServerJob *j = queue.front();
          if (j->bytes > budget) {
            queue.pop_front();
            j->state = JOB_FAILED;
            j->error = "the job needs more device memory than the whole budget";
            j->finished = now_s();
            cv.notify_all();
            continue;
          }
          if (used + j->bytes > budget) break;
          queue.pop_front();
          used += j->bytes;
          j->state = JOB_RUNNING;
          j->started = now_s();
          active.push_back(j);
          admitted.push_back(j);
        }
        // this round's work: the admitted jobs already set up
        std::vector<ServerJob *> keep;
        for (ServerJob *j : active) {
          if (j->state == JOB_RUNNING) {
            keep.push_back(j);
            if (j->prepared) (j->te ? te : other).push_back(j);
          } else if (j->state == JOB_CANCELLED && j->prepared) {
            j->sim->release();
          }
        }
        active = keep;
      }
      const double t0 = now_s();
      // launch: the others each on its own stream, the 2D TE jobs as one batch (remade when its
      // members change), as many steps as the batch's job nearest its end still needs
      std::vector<int64_t> took(other.size(), 0);
      std::vector<std::string> why(other.size());
      std::vector<std::pair<ServerJob *, std::string>> failed;
      parallel_for((int)other.size(), device, [&](int q) {
        ServerJob *j = other[q];
        took[q] = std::min(chunk, j->steps - j->done);
        if (fdtd_run_async(j->sim->ctx, took[q], j->sim->steps)) {
          why[q] = fdtd_last_error(j->sim->ctx);
          took[q] = -1;
        }
      });
      for (size_t q = 0; q < other.size(); q++)
        if (took[q] < 0) failed.push_back({other[q], why[q]});
      int64_t te_took = 0;
      if (!te.empty()) {
        if (te != batch_jobs) {
          fdtd_batch_destroy(batch);
          batch = nullptr;
          batch_jobs.clear();
          std::vector<fdtd_ctx *> ctxs;
          for (ServerJob *j : te) ctxs.push_back(j->sim->ctx);
          if (fdtd_batch_create((int32_t)ctxs.size(), ctxs.data(), &batch)) {
            for (ServerJob *j : te) failed.push_back({j, fdtd_batch_last_error(batch)});
            fdtd_batch_destroy(batch);
            batch = nullptr;
            te.clear();
          } else {
            // the row tiles where every grid's rows are 16-byte aligned (61 against 55
            // Gcell-updates/s on such grids), else the 32 x 16 tiles
            bool aligned = true;
            for (ServerJob *j : te) aligned = aligned && j->sim->g.n[0] % 4 == 0;
            if (aligned) fdtd_batch_set_tile(batch, 124, 7);
            else fdtd_batch_set_tile(batch, 32, 16);
            batch_jobs = te;
          }
        }
        if (!te.empty()) {
          te_took = chunk;
          std::vector<int64_t> first;
          for (ServerJob *j : te) {
            te_took = std::min(te_took, j->steps - j->done);
            first.push_back(j->sim->steps);
          }
          if (fdtd_batch_run(batch, te_took, first.data())) {
            for (ServerJob *j : te) failed.push_back({j, fdtd_batch_last_error(batch)});
            te.clear();
            te_took = 0;
          }
        }
      }
      const double t1 = now_s();
      // while the device steps: the last round's finished jobs read back (their own streams),
      // the newly admitted ones set up
      {
        std::vector<ServerJob *> tasks(finished);
        tasks.insert(tasks.end(), admitted.begin(), admitted.end());
        const size_t nfin = finished.size();
        std::vector<int> code(tasks.size(), 0);
        parallel_for((int)tasks.size(), device, [&](int q) {
          ServerJob *j = tasks[q];
          if ((size_t)q < nfin) {
            code[q] = j->sim->release(j->keep_fields);
          } else {
            code[q] = j->sim->prepare();
            if (code[q]) j->sim->release();
          }
        });
        std::lock_guard<std::mutex> lock(mu);
        for (size_t q = 0; q < tasks.size(); q++) {
          ServerJob *j = tasks[q];
          if (q < nfin) finish_job(j, code[q] ? JOB_FAILED : JOB_DONE, code[q] ? j->sim->error : std::string());
          else if (code[q]) finish_job(j, JOB_FAILED, j->sim->error.empty() ? "setup failed" : j->sim->error);
          else j->prepared = true;
        }
        cv.notify_all();
      }
      finished.clear();
      const double t2 = now_s();
      // the round's steps done
      for (size_t q = 0; q < other.size(); q++)
        if (took[q] > 0) fdtd_synchronize(other[q]->sim->ctx);
      for (ServerJob *j : te) fdtd_synchronize(j->sim->ctx);
      const double t3 = now_s();
      std::lock_guard<std::mutex> lock(mu);
      launch_s += t1 - t0;
      host_s += t2 - t1;
      wait_s += t3 - t2;
      if (!other.empty() || !te.empty()) chunks++;
      for (auto &f : failed) {
        if (f.first->state != JOB_RUNNING) continue;
        f.first->sim->release();
        finish_job(f.first, JOB_FAILED, f.second);
      }
      auto advance = [&](ServerJob *j, int64_t n) {
        if (j->state != JOB_RUNNING) return;
        j->sim->finish(n);
        j->done += n;
        cell_updates += (double)n * (double)j->sim->N();
        if (j->done >= j->steps) finished.push_back(j);
      };
      for (size_t q = 0; q < other.size(); q++)
        if (took[q] > 0) advance(other[q], took[q]);
      for (ServerJob *j : te) advance(j, te_took);
      std::vector<ServerJob *> keep;
      for (ServerJob *j : active) {
        const bool done = std::find(finished.begin(), finished.end(), j) != finished.end();
        if (j->state == JOB_RUNNING && !done) keep.push_back(j);
        else if (j->state == JOB_CANCELLED && j->prepared) j->sim->release();
      }
      active = keep;
      cv.notify_all();
    }
    for (ServerJob *j : finished) {
      j->sim->release(j->keep_fields);
      std::lock_guard<std::mutex> lock(mu);
      finish_job(j, JOB_DONE, std::string());
    }
    fdtd_batch_destroy(batch);
    batch = nullptr;
  }
};

extern "C" {

int pxs_server_create(size_t hbm_budget, int32_t max_active, int64_t chunk, pxs_server **out) {
  if (!out) return FDTD_E_INVALID;
  pxs_server *sv = new pxs_server();
  *out = sv;
  if (hbm_budget == 0 || max_active <= 0 || chunk <= 0) {
    sv->error = "a server needs a budget, slots and a chunk of steps";
    return FDTD_E_INVALID;
  }
  sv->budget = hbm_budget;
  sv->max_active = max_active;
  sv->chunk = chunk;
  cudaGetDevice(&sv->device);
  sv->loop = std::thread([sv] { sv->run_loop(); });
  return 0;
}

const char *pxs_server_last_error(const pxs_server *sv) { return sv ? sv->error.c_str() : "no server"; }

int64_t pxs_server_submit(pxs_server *sv, pxs_sim *s, int64_t steps, int32_t keep_fields) {
  if (!sv || !s || steps <= 0) return FDTD_E_INVALID;
  if (s->twin) {
    sv->error = "a complex run (a Bloch phase) steps on its own, with pxs_run";
    return FDTD_E_INVALID;
  }
  if (s->fields_dropped) {
    sv->error = s->dropped() ? s->error : std::string();
    return FDTD_E_STATE;
  }
  ServerJob *j = new ServerJob();
  j->sim = s;
  j->steps = steps;
  j->keep_fields = keep_fields != 0;
  j->te = s->te();
  j->bytes = s->device_bytes();
  j->submitted = now_s();
  std::lock_guard<std::mutex> lock(sv->mu);
  for (auto &kv : sv->jobs)
    if (kv.second->sim == s && kv.second->state <= JOB_RUNNING) {
      delete j;
      sv->error = "that simulation is already a job of this server";
      return FDTD_E_INVALID;
    }
  j->id = sv->next_id++;
  sv->jobs[j->id] = j;
  sv->queue.push_back(j);
  sv->cv.notify_all();
  return j->id;
}

// The job's state (0 queued, 1 running, 2 done, 3 failed, 4 cancelled) and its times (seconds
// on one steady clock: submitted, started, finished; 0 while not reached).
int pxs_server_poll(pxs_server *sv, int64_t id, double *times) {
  if (!sv) return FDTD_E_INVALID;
  std::lock_guard<std::mutex> lock(sv->mu);
  auto it = sv->jobs.find(id);
  if (it == sv->jobs.end()) {
    sv->error = "no such job";
    return FDTD_E_INVALID;
  }
  ServerJob *j = it->second;
  if (times) {
    times[0] = j->submitted;
    times[1] = j->started;
    times[2] = j->finished;
  }
  if (j->state == JOB_FAILED) sv->error = j->error;
  return j->state;
}

int pxs_server_wait(pxs_server *sv, int64_t id) {
  if (!sv) return FDTD_E_INVALID;
  std::unique_lock<std::mutex> lock(sv->mu);
  auto it = sv->jobs.find(id);
  if (it == sv->jobs.end()) {
    sv->error = "no such job";
    return FDTD_E_INVALID;
  }
  ServerJob *j = it->second;
  sv->cv.wait(lock, [&] { return j->state >= JOB_DONE || sv->stop; });
  if (j->state == JOB_FAILED) sv->error = j->error;
  return j->state;
}

int pxs_server_cancel(pxs_server *sv, int64_t id) {
  if (!sv) return FDTD_E_INVALID;
  std::lock_guard<std::mutex> lock(sv->mu);
  auto it = sv->jobs.find(id);
  if (it == sv->jobs.end()) return FDTD_E_INVALID;
  ServerJob *j = it->second;
  if (j->state == JOB_QUEUED) {
    sv->queue.erase(std::find(sv->queue.begin(), sv->queue.end(), j));
    j->state = JOB_CANCELLED;
    j->finished = now_s();
  } else if (j->state == JOB_RUNNING) {
    // the loop releases it between chunks
    sv->used -= j->bytes;
    j->bytes = 0;
    j->state = JOB_CANCELLED;
    j->finished = now_s();
  }
  sv->cv.notify_all();
  return 0;
}

// Totals so far: cell-updates taken, rounds stepped, device bytes admitted now, and the loop's
// seconds queuing work, setting up and reading back jobs (while the device steps), waiting.
int pxs_server_stats(pxs_server *sv, double *out) {
  if (!sv || !out) return FDTD_E_INVALID;
  std::lock_guard<std::mutex> lock(sv->mu);
  out[0] = sv->cell_updates;
  out[1] = (double)sv->chunks;
  out[2] = (double)sv->used;
  out[3] = sv->launch_s;
  out[4] = sv->host_s;
  out[5] = sv->wait_s;
  return 0;
}

void pxs_server_destroy(pxs_server *sv) {
  if (!sv) return;
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->stop = true;
    sv->cv.notify_all();
  }
  if (sv->loop.joinable()) sv->loop.join();
  for (auto &kv : sv->jobs) delete kv.second;
  delete sv;
}

}  // extern "C"
