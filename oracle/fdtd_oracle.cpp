// ORACLE (test infrastructure only): a CPU restatement of photonoxide's FDTD time step. It checks
// the CUDA engine; nothing in the product links or calls it. Every function cites the reference
// file:line it follows. Build: oracle/Makefile (-O2, -ffp-contract=off: no fused multiply-add, so
// each + - * / rounds as the reference's Rust does).
#include "fdtd_oracle.h"
#include "refmath.h"

#include <omp.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <unordered_set>
#include <vector>

namespace {

using c64 = std::complex<double>;
constexpr double TAU = 6.283185307179586476925286766559;

// Complex products written out as num-complex 0.4 computes them (a*c - b*d, a*d + b*c), so the
// rounding matches the reference; std::complex may use other forms.
inline c64 cmul(c64 x, c64 y) {
  return c64(x.real() * y.real() - x.imag() * y.imag(), x.real() * y.imag() + x.imag() * y.real());
}
// exp(i x) as portable::complex::exp of a purely imaginary argument (src/portable/complex.rs:71-93)
inline c64 cis(double x) {
  double s, c;
  refmath::ref_sincos(x, &s, &c);
  return c64(c, s);
}

struct Grid {  // src/fdfd/three.rs:70-157
  long n[3];
  double d[3], o[3];
  long cells() const { return n[0] * n[1] * n[2]; }
  double node(int a, long m) const { return o[a] + (double)m * d[a]; }
  void e_position(int c, long i, long j, long k, double p[3]) const {
    p[0] = node(0, i);
    p[1] = node(1, j);
    p[2] = node(2, k);
    p[c] += 0.5 * d[c];
  }
};
inline int first_of(int c) { return (c + 1) % 3; }   // Axis::others().0
inline int second_of(int c) { return (c + 2) % 3; }  // Axis::others().1

struct Box {
  double lo[3], hi[3], eps;
};
double geometry(const std::vector<Box> &boxes, double bg, const double p[3]) {
  double v = bg;
  for (const Box &b : boxes)
    if (b.lo[0] < p[0] && p[0] < b.hi[0] && b.lo[1] < p[1] && p[1] < b.hi[1] && b.lo[2] < p[2] &&
        p[2] < b.hi[2])
      v = b.eps;
  return v;
}

// averaged (src/fdfd/three.rs:563-588) for a real permittivity, with num-complex's arithmetic on
// an imaginary part of zero: 1/eps is eps/(eps*eps) (real / complex divides by the norm), n/inverse
// is n*inverse/(inverse*inverse), and the sum is divided by n*n.
double averaged(const std::vector<Box> &boxes, double bg, const double centre[3], const double h[3],
                int along, int samples) {
  double n = (double)samples;
  auto offset = [n](int s) { return ((double)s + 0.5) / n - 0.5; };
  int a = along, b = first_of(along), c = second_of(along);
  double sum = 0.0;
  double p[3] = {centre[0], centre[1], centre[2]};
  for (int sb = 0; sb < samples; sb++) {
    p[b] = centre[b] + offset(sb) * h[b];
    for (int sc = 0; sc < samples; sc++) {
      p[c] = centre[c] + offset(sc) * h[c];
      double inverse = 0.0;
      for (int sa = 0; sa < samples; sa++) {
        p[a] = centre[a] + offset(sa) * h[a];
        double e = geometry(boxes, bg, p);
        inverse += (1.0 * e) / (e * e);
      }
      sum += (n * inverse) / (inverse * inverse);
    }
  }
  return sum / (n * n);
}

// Waveform (src/fdtd.rs:259-434)
struct Wave {
  int kind = 0;
  double p[5] = {0, 0, 0, 0, 0};
  static Wave from(const double *w) {
    Wave x;
    x.kind = (int)w[0];
    for (int i = 0; i < 5; i++) x.p[i] = w[i + 1];
    return x;
  }
  static double smoothstep(double t, double ramp) {  // src/fdtd.rs:427-434
    if (ramp > 0.0) {
      double s = std::min(std::max(t / ramp, 0.0), 1.0);
      return s * s * (3.0 - 2.0 * s);
    }
    return 1.0;
  }
  double at(double t) const {  // src/fdtd.rs:399-423
    if (kind == 0) {
      double u = (t - p[2]) / p[1];
      return refmath::ref_exp(-u * u) * refmath::ref_sin(TAU * p[0] * (t - p[2]));
    }
    if (kind == 1) {
      double u = (t - p[1]) / p[0];
      return -u * refmath::ref_exp(-u * u) * std::sqrt(2.0 * 2.718281828459045235360287471352662);
    }
    c64 w = cis(-(TAU * p[0]) * t);
    return smoothstep(t, p[3]) * (p[1] * w.real() - p[2] * w.imag());
  }
  c64 complex_at(double t) const {  // src/fdtd.rs:329-351
    if (kind == 0) {
      double u = (t - p[2]) / p[1];
      return cmul(c64(0.0, refmath::ref_exp(-u * u)), cis(-(TAU * p[0]) * (t - p[2])));
    }
    if (kind == 1) return c64(at(t), 0.0);
    double s = smoothstep(t, p[3]);
    return cmul(c64(s * p[1], s * p[2]), cis(-(TAU * p[0]) * t));
  }
};

struct SlabInfo {  // kernel::Slab (src/fdtd/kernel.rs:376-392), coefficients in f64
  int field, comp, axis;
  long from, count;
  std::vector<double> b, a;
};

template <typename T>
struct SlabState {
  std::vector<T> b, a, psi;
};

struct Series {  // src/fdtd/monitors.rs:45-82
  int field, comp;
  long lo[3], len[3];
  std::vector<c64> values;
  long volume() const { return len[0] * len[1] * len[2]; }
  bool offset(const long at[3], long *o) const {
    for (int a = 0; a < 3; a++)
      if (at[a] < lo[a] || at[a] >= lo[a] + len[a]) return false;
    *o = ((at[2] - lo[2]) * len[1] + (at[1] - lo[1])) * len[0] + at[0] - lo[0];
    return true;
  }
};
struct Dft {
  std::vector<double> freqs;  // c/um
  std::vector<Series> series;
  bool value(int field, int comp, const long at[3], int f, c64 *out) const {
    for (const Series &s : series) {
      if (s.field != field || s.comp != comp) continue;
      long o;
      if (s.offset(at, &o)) {
        *out = s.values[f * s.volume() + o];
        return true;
      }
    }
    return false;
  }
};
struct FluxPlane {  // src/fdtd/monitors.rs:212-351
  int axis;
  long plane;
  long win[2][2];  // along others().0 and others().1; {-1,-1} = whole axis
  long range_lo(const Grid &g, int along) const {
    int sl = along == first_of(axis) ? 0 : 1;
    return win[sl][0] < 0 ? 0 : win[sl][0];
  }
  long range_hi(const Grid &g, int along) const {  // exclusive
    int sl = along == first_of(axis) ? 0 : 1;
    return win[sl][0] < 0 ? g.n[along] : win[sl][1] + 1;
  }
  double weight(int along, long m, bool half) const {
    int sl = along == first_of(axis) ? 0 : 1;
    if (win[sl][0] < 0) return 1.0;
    long lo = win[sl][0], hi = win[sl][1];
    if (half) {
      if (lo < m && m < hi) return 1.0;
      if (m == lo || m == hi) return 0.5;
      return 0.0;
    }
    return (lo < m && m <= hi) ? 1.0 : 0.0;
  }
  std::vector<Series> series(const Grid &g, int nf) const {
    int b = first_of(axis), c = second_of(axis);
    std::vector<Series> out;
    for (int fd = 0; fd < 2; fd++) {
      int depth = fd == 0 ? 2 : 1;
      for (int comp : {b, c}) {
        Series s;
        s.field = fd;
        s.comp = comp;
        s.lo[axis] = plane;
        s.len[axis] = depth;
        for (int al : {b, c}) {
          s.lo[al] = range_lo(g, al);
          s.len[al] = range_hi(g, al) - range_lo(g, al);
        }
        s.values.assign(s.volume() * nf, c64(0, 0));
        out.push_back(s);
      }
    }
    return out;
  }
  double flux(const Grid &g, const Dft &dft, int f) const {
    int b = first_of(axis), c = second_of(axis);
    double total = 0.0;
    struct T3 { int comp, h; double sign; };
    const T3 terms[2] = {{b, c, 0.5}, {c, b, -0.5}};
    for (const T3 &t : terms) {
      for (long v = range_lo(g, c); v < range_hi(g, c); v++) {
        for (long u = range_lo(g, b); u < range_hi(g, b); u++) {
          double w = weight(b, u, t.comp == b) * weight(c, v, t.comp == c);
          if (w == 0.0) continue;
          long at[3];
          at[axis] = plane;
          at[b] = u;
          at[c] = v;
          c64 low, hv, high;
          dft.value(0, t.comp, at, f, &low);
          dft.value(1, t.h, at, f, &hv);
          at[axis] = plane + 1;
          dft.value(0, t.comp, at, f, &high);
          c64 mean = c64(0.5 * (low + high).real(), 0.5 * (low + high).imag());
          c64 prod = cmul(mean, std::conj(hv));
          total += w * t.sign * prod.real();
        }
      }
    }
    return total * g.d[b] * g.d[c];
  }
};
struct Flux {
  std::vector<FluxPlane> planes;
  std::vector<double> signs;
  std::vector<Dft> dfts;
};

struct Pole {  // src/fdtd/media.rs:55-109
  int kind;
  double x1, x2, x3;
  void parts(double &a, double &w0sq, double &gamma) const {
    if (kind == 0) {
      double w0 = TAU * x2;
      a = x1 * w0 * w0;
      w0sq = w0 * w0;
      gamma = TAU * x3;
    } else {
      double wp = TAU * x1;
      a = wp * wp;
      w0sq = 0.0;
      gamma = TAU * x2;
    }
  }
  void coefficients(double dt, double out[3]) const {
    double a, w0sq, gamma;
    parts(a, w0sq, gamma);
    double d = 1.0 + gamma * dt / 2.0;
    out[0] = (2.0 - w0sq * dt * dt) / d;
    out[1] = (gamma * dt / 2.0 - 1.0) / d;
    out[2] = a * dt * dt / d;
  }
};

template <typename T>
struct Group {  // src/fdtd/media.rs:559-615
  std::vector<std::pair<int, long>> values;
  std::vector<T> scale;
  T chi;
  std::vector<std::array<T, 3>> poles;
  std::vector<T> before, now, current, previous;
  void resize() {
    size_t n = values.size(), p = poles.size();
    before.assign(n, T(0));
    now.assign(n, T(0));
    current.assign(n * p, T(0));
    previous.assign(n * p, T(0));
  }
};

struct Injection {  // a source or current value: field, component, index, amplitude, emitter
  int field, comp;
  long r;
  c64 a;
  int emitter;
  bool point;  // a point source takes w.at(t); a current Re(a w(t))
};

// Twice a value's position along `axis` in steps from node 0 (src/fdtd/sources.rs:155-162): a node
// m is 2m, halfway after it 2m + 1; E's component is halfway along itself, H's along the others.
inline long twice(int field, int comp, int axis, long m) {
  const bool half = field == 0 ? comp == axis : comp != axis;
  return 2 * m + (half ? 1 : 0);
}

// One coupling across a total-field/scattered-field surface (src/fdtd/sources.rs:138-153).
struct Link {
  int target, comp;
  long r;
  double weight;
  int from_field, from_comp;
  long from[3];
};

// A plane wave's run (src/fdtd/sources.rs:740-1041): its auxiliary 1D grid along the direction
// (p, q, s), sample l at l = sum of g_a twice_a, and the couplings of its box.
struct PlaneRun {
  long g[3];
  double steps[3];
  long base = 0, pad = 0, len = 0;
  std::vector<double> e[3], h[3], ca, cb, da, db;
  struct Sheet { int c; long i; double j; };
  std::vector<Sheet> sheet;
  Wave wave;
  struct Coupling { int c; long r; double w; int from; long i; };
  std::vector<Coupling> on_e, on_h;

  bool sample(int field, int comp, const long at[3], long *i) const {
    long l = 0;
    for (int a = 0; a < 3; a++) l += g[a] * twice(field, comp, a, at[a]);
    const long q = l - base;
    if (q < 0 || q >= len) return false;
    *i = q;
    return true;
  }
  double value(int field, int comp, const long at[3]) const {
    long i;
    if (!sample(field, comp, at, &i)) return 0.0;
    return field == 0 ? e[comp][i] : h[comp][i];
  }
  double difference(const std::vector<double> &f, int axis, long i) const {
    const long o = g[axis];
    if (o == 0) return 0.0;
    return (f[i + o] - f[i - o]) / steps[axis];
  }
  void step_h() {
    for (int c = 0; c < 3; c++) {
      const int a = first_of(c), b = second_of(c);
      for (long i = pad; i < len - pad; i++) {
        const double curl = difference(e[b], a, i) - difference(e[a], b, i);
        h[c][i] = da[i] * h[c][i] - db[i] * curl;
      }
    }
  }
  void step_e(double half) {
    for (int c = 0; c < 3; c++) {
      const int a = first_of(c), b = second_of(c);
      for (long i = pad; i < len - pad; i++) {
        const double curl = difference(h[b], a, i) - difference(h[a], b, i);
        e[c][i] = ca[i] * e[c][i] + cb[i] * curl;
      }
    }
    const double w = wave.at(half);
    for (const Sheet &q : sheet) e[q.c][q.i] -= cb[q.i] * q.j * w;
  }
};

struct Base {
  virtual ~Base() {}
};

template <typename T>
struct Sim : Base {
  Grid g;
  int kind[3];
  long low[3], high[3];
  double cpml[5];
  double dt64;
  long steps = 0;
  bool varies[3];
  // setup in f64 (the reference's own) ...
  std::vector<double> ca64[3], cb64[3], kn64[3], kh64[3];
  std::vector<SlabInfo> slabs;
  // ... and the state in T
  T dt;
  std::vector<T> e[3], h[3], ca[3], cb[3];
  std::vector<T> fe[3], fh[3];  // kappa/h at nodes (E's back differences) and halves (H's)
  std::vector<SlabState<T>> psi;
  std::vector<Wave> emitters;
  std::vector<Injection> injections;  // in the order a CPU step adds them: sources, then currents
  struct Probe { int field, comp; long r; std::vector<double> values; };
  std::vector<Probe> probes;
  std::vector<Dft> dfts;
  std::vector<Flux> fluxes;
  std::vector<Group<T>> groups;
  std::map<std::pair<int, long>, int> members;
  std::vector<PlaneRun> plane_waves;
  // Bloch sides (src/fdtd/bloch.rs:45-95): the wavenumbers, and with one not zero the fields'
  // imaginary part as a second run stepped alongside, e^(ikL) along each axis
  double bloch_k[3] = {0.0, 0.0, 0.0};
  bool along[3] = {false, false, false};
  c64 phase[3];
  Sim *twin = nullptr;
  Sim() = default;
  Sim(const Sim &) = default;
  ~Sim() override { delete twin; }

  long stride(int a) const { return a == 0 ? 1 : (a == 1 ? g.n[0] : g.n[0] * g.n[1]); }
  bool periodic(int a) const { return kind[a] == 1; }
  // Simulation::offsets (src/fdtd.rs:1424-1450): false where the neighbour is beyond a wall
  bool offset(int a, long m, bool forward, long *off) const {
    long n = g.n[a], st = stride(a);
    if (forward) {
      if (m + 1 < n) { *off = st; return true; }
      if (periodic(a)) { *off = st - n * st; return true; }
      return false;
    }
    if (m > 0) { *off = -st; return true; }
    if (periodic(a)) { *off = (n - 1) * st; return true; }
    return false;
  }

  // bloch::curl_bound (src/fdtd/bloch.rs:31-43): sum of w_i / h_i^2, w_i = sin^2(k h / 2) along an
  // axis one cell long with a Bloch phase, nothing along one without, 1 along the others
  double curl_bound() const {
    double sum = 0.0;
    for (int a = 0; a < 3; a++) {
      const double h = g.d[a], hh = h * h;
      if (periodic(a) && g.n[a] == 1) {
        if (bloch_k[a] == 0.0) continue;
        const double sn = refmath::ref_sin(bloch_k[a] * h / 2.0);
        sum += (sn * sn) * (1.0 / hh);
        continue;
      }
      sum += 1.0 / hh;
    }
    return sum;
  }

  // Simulation::with_permittivity (src/fdtd.rs:680-796) after the checks
  bool init(const double *eps, double courant, std::string &err) {
    long N = g.cells();
    const double sum = curl_bound();
    if (sum == 0.0) { err = "the field varies along no axis"; return false; }
    dt64 = courant / std::sqrt(sum);
    for (int c = 0; c < 3; c++) {
      ca64[c].assign(N, 1.0);
      cb64[c].resize(N);
      for (long r = 0; r < N; r++) {
        double v = eps[c * N + r];
        if (!(std::isfinite(v) && v > 0.0)) {
          err = "the permittivity must be finite and positive";
          return false;
        }
        cb64[c][r] = dt64 / v;
      }
    }
    for (int c = 0; c < 3; c++)  // walls: tangential E zero at node 0 (src/fdtd.rs:738-756)
      for (int a = 0; a < 3; a++) {
        if (a == c || periodic(a)) continue;
        for (long r = 0; r < N; r++) {
          long at[3] = {r % g.n[0], (r / g.n[0]) % g.n[1], r / (g.n[0] * g.n[1])};
          if (at[a] == 0) ca64[c][r] = cb64[c][r] = 0.0;
        }
      }
    for (int a = 0; a < 3; a++) {
      varies[a] = !(g.n[a] == 1 && periodic(a));
      kn64[a].assign(g.n[a], 1.0);
      kh64[a].assign(g.n[a], 1.0);
    }
    build_cpml();
    return true;
  }

  // Simulation::build_cpml (src/fdtd.rs:799-869)
  void build_cpml() {
    double R = cpml[0], sig = cpml[1], order = cpml[2], kmax = cpml[3], alpha = cpml[4];
    for (int axis = 0; axis < 3; axis++) {
      if (periodic(axis)) continue;
      long lo = low[axis], hi = high[axis], n = g.n[axis];
      double h = g.d[axis];
      auto profile = [&](double depth, long cells, double &s, double &k) {
        double d = (double)cells * h;
        // portable::powf and portable::ln (src/fdtd.rs:811-815), restated in refmath.h
        double x = refmath::ref_pow(std::min(std::max(depth / (double)cells, 0.0), 1.0), order);
        double smax = std::isnan(sig) ? (order + 1.0) * (-refmath::ref_ln(R)) / (2.0 * d) : sig;
        s = smax * x;
        k = 1.0 + (kmax - 1.0) * x;
      };
      auto at = [&](double pos, double &s, double &k) {
        if (lo > 0 && pos < (double)lo) profile((double)lo - pos, lo, s, k);
        else if (hi > 0 && pos > (double)(n - hi)) profile(pos - (double)(n - hi), hi, s, k);
        else { s = 0.0; k = 1.0; }
      };
      for (long m = 0; m < n; m++) {
        double s, k;
        at((double)m, s, k);
        kn64[axis][m] = 1.0 / k;
        at((double)m + 0.5, s, k);
        kh64[axis][m] = 1.0 / k;
      }
      auto coefficients = [&](double pos, double &b, double &a) {
        double s, k;
        at(pos, s, k);
        b = refmath::ref_exp(-(s / k + alpha) * dt64);
        double den = s * k + k * k * alpha;
        a = (s > 0.0 && den > 0.0) ? s * (b - 1.0) / den : 0.0;
      };
      long froms[2] = {0, n - hi}, counts[2] = {lo, hi};
      for (int side = 0; side < 2; side++) {
        if (counts[side] == 0) continue;
        for (int field = 0; field < 2; field++) {
          double offs = field == 0 ? 0.0 : 0.5;
          SlabInfo sl;
          sl.field = field;
          sl.axis = axis;
          sl.from = froms[side];
          sl.count = counts[side];
          for (long m = sl.from; m < sl.from + sl.count; m++) {
            double b, a;
            coefficients((double)m + offs, b, a);
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

  // Yee<T>::from_simulation (src/fdtd/kernel/yee.rs:29-52): the f64 state rounded to T
  void materialize() {
    long N = g.cells();
    dt = (T)dt64;
    for (int c = 0; c < 3; c++) {
      e[c].assign(N, T(0));
      h[c].assign(N, T(0));
      ca[c].resize(N);
      cb[c].resize(N);
      for (long r = 0; r < N; r++) {
        ca[c][r] = (T)ca64[c][r];
        cb[c][r] = (T)cb64[c][r];
      }
      fe[c].resize(g.n[c]);
      fh[c].resize(g.n[c]);
      for (long m = 0; m < g.n[c]; m++) {  // build_stencils (src/fdtd.rs:1552-1569)
        fe[c][m] = (T)(kn64[c][m] / g.d[c]);
        fh[c][m] = (T)(kh64[c][m] / g.d[c]);
      }
    }
    psi.clear();
    for (const SlabInfo &s : slabs) {
      SlabState<T> st;
      for (long q = 0; q < s.count; q++) {
        st.b.push_back((T)s.b[q]);
        st.a.push_back((T)s.a[q]);
      }
      st.psi.assign(s.count * (N / g.n[s.axis]), T(0));
      psi.push_back(st);
    }
  }
  void refresh_coefficients() {
    long N = g.cells();
    for (int c = 0; c < 3; c++)
      for (long r = 0; r < N; r++) {
        ca[c][r] = (T)ca64[c][r];
        cb[c][r] = (T)cb64[c][r];
      }
  }

  // Simulation::curl_update_reference (src/fdtd/kernel/reference.rs:14-50) for each component
  void curl_update(int field) {
    bool forward = field == 1;
    std::vector<T> *out = forward ? h : e;
    const std::vector<T> *f = forward ? e : h;
    const std::vector<T> *fac = forward ? fh : fe;
    long nx = g.n[0], ny = g.n[1], nz = g.n[2], plane = nx * ny;
    for (int c = 0; c < 3; c++) {
      int a = first_of(c), b = second_of(c);
      const T *fa = f[a].data(), *fb = f[b].data();
      T *o = out[c].data();
      const T *keep = ca[c].data(), *scale = cb[c].data();
#pragma omp parallel for schedule(static)
      for (long k = 0; k < nz; k++)
        for (long j = 0; j < ny; j++)
          for (long i = 0; i < nx; i++) {
            long m[3] = {i, j, k};
            long r = k * plane + j * nx + i;
            long oa, ob;
            bool ha = offset(a, m[a], forward, &oa), hb = offset(b, m[b], forward, &ob);
            T other_b = ha ? fb[r + oa] : T(0);
            T other_a = hb ? fa[r + ob] : T(0);
            T db = forward ? other_b - fb[r] : fb[r] - other_b;
            T da = forward ? other_a - fa[r] : fa[r] - other_a;
            T curl = db * fac[a][m[a]] - da * fac[b][m[b]];
            if (forward) o[r] = o[r] - dt * curl;
            else o[r] = keep[r] * o[r] + scale[r] * curl;
          }
    }
  }

  // Simulation::update_slabs_reference (src/fdtd/kernel/reference.rs:102-180)
  void update_slabs(int field) {
    bool forward = field == 1;
    long nx = g.n[0], ny = g.n[1], plane = nx * ny;
    for (size_t si = 0; si < slabs.size(); si++) {
      const SlabInfo &sl = slabs[si];
      if (sl.field != field) continue;
      SlabState<T> &st = psi[si];
      int w = sl.axis, c = sl.comp;
      T sign;
      int differentiated;
      if (w == first_of(c)) { sign = T(1); differentiated = second_of(c); }
      else { sign = T(-1); differentiated = first_of(c); }
      T hstep = (T)g.d[w];
      const T *src = forward ? e[differentiated].data() : h[differentiated].data();
      long from[3] = {0, 0, 0}, count[3] = {g.n[0], g.n[1], g.n[2]};
      from[w] = sl.from;
      count[w] = sl.count;
      long lplane = count[0] * count[1];
#pragma omp parallel for schedule(static)
      for (long lk = 0; lk < count[2]; lk++)
        for (long lj = 0; lj < count[1]; lj++)
          for (long li = 0; li < count[0]; li++) {
            long m[3] = {from[0] + li, from[1] + lj, from[2] + lk};
            long r = m[2] * plane + m[1] * nx + m[0];
            long off;
            T other = offset(w, m[w], forward, &off) ? src[r + off] : T(0);
            T d = (forward ? other - src[r] : src[r] - other) / hstep;
            long q = lk * lplane + lj * count[0] + li;
            long s = m[w] - sl.from;
            st.psi[q] = st.b[s] * st.psi[q] + st.a[s] * d;
          }
      T *target = forward ? h[c].data() : e[c].data();
      const T *cbc = cb[c].data();
#pragma omp parallel for schedule(static)
      for (long lk = 0; lk < count[2]; lk++)
        for (long lj = 0; lj < count[1]; lj++)
          for (long li = 0; li < count[0]; li++) {
            long k = from[2] + lk, j = from[1] + lj, i = from[0] + li;
            long r = k * plane + j * nx + i;
            T u = sign * st.psi[lk * lplane + lj * count[0] + li];
            if (forward) target[r] = target[r] - dt * u;
            else target[r] = target[r] + cbc[r] * u;
          }
    }
  }

  // The sources' and currents' amounts (src/fdtd.rs:1346-1387): in f64 as the reference; the
  // f32 run rounds each amount to T before it enters, as the CUDA engine does.
  void inject(int field, double t) {
    for (const Injection &x : injections) {
      if (x.field != field) continue;
      const Wave &w = emitters[x.emitter];
      double amount;
      if (x.point) amount = w.at(t);
      else {
        c64 v = w.complex_at(t);
        amount = x.a.real() * v.real() - x.a.imag() * v.imag();
      }
      if (sizeof(T) == 8) {
        if (field == 1) h[x.comp][x.r] -= (T)(dt64 * amount);
        else e[x.comp][x.r] -= (T)(cb64[x.comp][x.r] * amount);
      } else {
        T am = (T)amount;
        if (field == 1) h[x.comp][x.r] = h[x.comp][x.r] - dt * am;
        else e[x.comp][x.r] = e[x.comp][x.r] - cb[x.comp][x.r] * am;
      }
    }
  }

  // Simulation::push_current (src/fdtd/sources.rs:190-207): a current, and in a complex run the
  // imaginary part of its values a w(t), Im(a w) = Re(-i a w), on the imaginary part.
  void push_current(int field, const std::vector<std::pair<int, long>> &where,
                    const std::vector<c64> &a, const Wave &w) {
    emitters.push_back(w);
    for (size_t q = 0; q < where.size(); q++)
      injections.push_back(Injection{field, where[q].first, where[q].second, a[q],
                                     (int)emitters.size() - 1, false});
    if (twin) {
      twin->emitters.push_back(w);
      for (size_t q = 0; q < where.size(); q++)
        twin->injections.push_back(Injection{field, where[q].first, where[q].second,
                                             cmul(c64(0.0, -1.0), a[q]),
                                             (int)twin->emitters.size() - 1, false});
    }
  }

  // Bloch::image (src/fdtd/bloch.rs:85-95): e^(-ikL turns), num-complex's powi of the phase.
  c64 image(int axis, long turns) const {
    if (turns == 0 || !along[axis]) return c64(1.0, 0.0);
    auto power = [](c64 base, unsigned long e) {  // num_traits::pow, by squaring
      while ((e & 1) == 0) {
        base = cmul(base, base);
        e >>= 1;
      }
      if (e == 1) return base;
      c64 acc = base;
      while (e > 1) {
        e >>= 1;
        base = cmul(base, base);
        if (e & 1) acc = cmul(acc, base);
      }
      return acc;
    };
    const long n = -turns;
    if (n >= 0) return power(phase[axis], (unsigned long)n);
    const c64 p = power(phase[axis], (unsigned long)(-n));
    const double ns = p.real() * p.real() + p.imag() * p.imag();
    return c64(p.real() / ns, 0.0 - p.imag() / ns);
  }

  // PlaneWaveRun::correct (src/fdtd/sources.rs:971-991): the box's corrections from the incident
  // field now, in f64 as the reference; the f32 run rounds each correction to T.
  void correct(const PlaneRun &p, int field) {
    if (field == 0) {
      for (const PlaneRun::Coupling &q : p.on_e) {
        const double amount = (cb64[q.c][q.r] * q.w) * p.h[q.from][q.i];
        e[q.c][q.r] = e[q.c][q.r] - (T)amount;
      }
    } else {
      for (const PlaneRun::Coupling &q : p.on_h) {
        const double amount = (dt64 * q.w) * p.e[q.from][q.i];
        h[q.c][q.r] = h[q.c][q.r] - (T)amount;
      }
    }
  }

  // Simulation::links (src/fdtd/sources.rs:316-420): the couplings across a total-field /
  // scattered-field surface among the values in region [lo, hi) per axis, total() saying which
  // side each value is on; values held at zero (cb = 0) neither take nor give one.
  template <typename F>
  std::vector<Link> links(const long lo[3], const long hi[3], const F &total) const {
    auto neighbour = [&](const long at[3], int axis, bool forward, long out[3]) -> bool {
      for (int q = 0; q < 3; q++) out[q] = at[q];
      const long n = g.n[axis];
      if (forward) {
        if (at[axis] + 1 < n) out[axis] += 1;
        else if (periodic(axis)) out[axis] = 0;
        else return false;
      } else if (at[axis] > 0) {
        out[axis] -= 1;
      } else if (periodic(axis)) {
        out[axis] = n - 1;
      } else {
        return false;
      }
      return true;
    };
    auto index = [&](const long at[3]) { return (at[2] * g.n[1] + at[1]) * g.n[0] + at[0]; };
    auto held = [&](int comp, const long at[3]) { return cb64[comp][index(at)] == 0.0; };
    std::vector<Link> out;
    for (long k = lo[2]; k < hi[2]; k++)
      for (long j = lo[1]; j < hi[1]; j++)
        for (long i = lo[0]; i < hi[0]; i++) {
          const long at[3] = {i, j, k};
          const long r = index(at);
          for (int c = 0; c < 3; c++) {
            const int a = first_of(c), b = second_of(c);
            struct Term { int comp; bool ok; long from[3]; double coefficient; };
            if (!held(c, at)) {
              const bool inside = total(0, c, at);
              const double fa = kn64[a][at[a]] / g.d[a], fb = kn64[b][at[b]] / g.d[b];
              Term terms[4];
              terms[0] = {b, true, {i, j, k}, fa};
              terms[1].comp = b;
              terms[1].ok = neighbour(at, a, false, terms[1].from);
              terms[1].coefficient = -fa;
              terms[2] = {a, true, {i, j, k}, -fb};
              terms[3].comp = a;
              terms[3].ok = neighbour(at, b, false, terms[3].from);
              terms[3].coefficient = fb;
              for (const Term &q : terms) {
                if (!q.ok) continue;
                if (total(1, q.comp, q.from) != inside) {
                  const double sign = inside ? -1.0 : 1.0;
                  out.push_back(Link{0, c, r, sign * q.coefficient, 1, q.comp,
                                     {q.from[0], q.from[1], q.from[2]}});
                }
              }
            }
            const bool inside = total(1, c, at);
            const double fa = kh64[a][at[a]] / g.d[a], fb = kh64[b][at[b]] / g.d[b];
            Term terms[4];
            terms[0].comp = b;
            terms[0].ok = neighbour(at, a, true, terms[0].from);
            terms[0].coefficient = fa;
            terms[1] = {b, true, {i, j, k}, -fa};
            terms[2].comp = a;
            terms[2].ok = neighbour(at, b, true, terms[2].from);
            terms[2].coefficient = -fb;
            terms[3] = {a, true, {i, j, k}, fb};
            for (const Term &q : terms) {
              if (!q.ok) continue;
              if (held(q.comp, q.from)) continue;
              if (total(0, q.comp, q.from) != inside) {
                const double sign = inside ? 1.0 : -1.0;
                out.push_back(Link{1, c, r, sign * q.coefficient, 0, q.comp,
                                   {q.from[0], q.from[1], q.from[2]}});
              }
            }
          }
        }
    return out;
  }

  // Simulation::uniform (src/fdtd/sources.rs:509-522): every value of E on the surface lossless
  // in a medium of eps.
  bool uniform(const std::vector<Link> &ls, double eps) const {
    const double expected = dt64 / eps;
    for (const Link &l : ls) {
      int c;
      long r;
      if (l.target == 0) {
        c = l.comp;
        r = l.r;
      } else {
        c = l.from_comp;
        r = (l.from[2] * g.n[1] + l.from[1]) * g.n[0] + l.from[0];
      }
      if (!(std::fabs(cb64[c][r] - expected) <= 1e-12 * expected && ca64[c][r] == 1.0 &&
            members.find({c, r}) == members.end()))
        return false;
    }
    return true;
  }

  // Media::save / Media::update (src/fdtd/media.rs:661-705)
  void media_save() {
    for (Group<T> &gr : groups)
      for (size_t v = 0; v < gr.values.size(); v++)
        gr.now[v] = e[gr.values[v].first][gr.values[v].second];
  }
  void media_update() {
    T two_dt = (T)(2.0 * dt64);
    for (Group<T> &gr : groups) {
      size_t p = gr.poles.size();
      for (size_t v = 0; v < gr.values.size(); v++) {
        int c = gr.values[v].first;
        long r = gr.values[v].second;
        T rest = gr.chi * gr.before[v];
        for (size_t q = 0; q < p; q++)
          rest = rest - T(0.5) * ((gr.poles[q][0] + T(1)) * gr.current[v * p + q] +
                                  gr.poles[q][1] * gr.previous[v * p + q]);
        T next = e[c][r] + gr.scale[v] * rest;
        T slope = (next - gr.before[v]) / two_dt;
        for (size_t q = 0; q < p; q++) {
          T j = gr.poles[q][0] * gr.current[v * p + q] + gr.poles[q][1] * gr.previous[v * p + q] +
                gr.poles[q][2] * slope;
          gr.previous[v * p + q] = gr.current[v * p + q];
          gr.current[v * p + q] = j;
        }
        gr.before[v] = gr.now[v];
        e[c][r] = next;
      }
    }
  }

  // Dft::record (src/fdtd/monitors.rs:129-154, 178-206): each value's sums in step order, f64
  void record_dft(Dft &d, double te, double th) {
    long nx = g.n[0], plane = nx * g.n[1];
    std::vector<c64> ph(d.freqs.size());
    for (Series &s : d.series) {
      double t = s.field == 0 ? te : th;
      for (size_t f = 0; f < d.freqs.size(); f++) {
        c64 p = cis(TAU * d.freqs[f] * t);
        ph[f] = c64(p.real() * dt64, p.imag() * dt64);
      }
      const T *src = s.field == 0 ? e[s.comp].data() : h[s.comp].data();
      // a complex run's values are transformed whole (src/fdtd/monitors.rs:127-154)
      const T *isrc = !twin ? nullptr : (s.field == 0 ? twin->e[s.comp].data() : twin->h[s.comp].data());
      long vol = s.volume();
#pragma omp parallel for schedule(static)
      for (long o = 0; o < vol; o++) {
        long i = s.lo[0] + o % s.len[0], j = s.lo[1] + (o / s.len[0]) % s.len[1],
             k = s.lo[2] + o / (s.len[0] * s.len[1]);
        double v = (double)src[k * plane + j * nx + i];
        if (isrc) {
          const double w = (double)isrc[k * plane + j * nx + i];
          for (size_t f = 0; f < ph.size(); f++) {
            c64 &acc = s.values[f * vol + o];
            const c64 x = cmul(c64(v, w), ph[f]);
            acc = c64(acc.real() + x.real(), acc.imag() + x.imag());
          }
          continue;
        }
        for (size_t f = 0; f < ph.size(); f++) {
          c64 &acc = s.values[f * vol + o];
          acc = c64(acc.real() + v * ph[f].real(), acc.imag() + v * ph[f].imag());
        }
      }
    }
  }

  // Simulation::step (src/fdtd.rs:1319-1419)
  // Simulation::step_h / step_e / finish_step (src/fdtd.rs:1344-1419)
  void step_h(double t) {
    curl_update(1);
    update_slabs(1);
    inject(1, t);
    for (PlaneRun &p : plane_waves) {
      correct(p, 1);
      p.step_h();
    }
  }
  void step_e(double half) {
    media_save();
    curl_update(0);
    update_slabs(0);
    inject(0, half);
    for (PlaneRun &p : plane_waves) {
      correct(p, 0);
      p.step_e(half);
    }
  }
  void finish_step() {
    media_update();
    steps += 1;
    for (Probe &p : probes)
      p.values.push_back((double)(p.field == 0 ? e[p.comp][p.r] : h[p.comp][p.r]));
    double te = (double)steps * dt64, th = te - 0.5 * dt64;
    for (Dft &d : dfts) record_dft(d, te, th);
    for (Flux &f : fluxes)
      for (Dft &d : f.dfts) record_dft(d, te, th);
  }

  // Bloch::wrap (src/fdtd/bloch.rs:97-152): after `field`'s update in both parts, each value
  // whose difference along a Bloch axis reached across the side read the other end's value of
  // its own part; it gets the difference e^(+-ikL) makes, (e^(+-ikL) - 1) F, in both parts.
  void wrap(int field) {
    const bool forward = field == 1;
    for (int w = 0; w < 3; w++) {
      if (!along[w]) continue;
      const long n = g.n[w];
      const long m = forward ? n - 1 : 0;
      long o = 0;
      offset(w, m, forward, &o);
      const c64 ph = forward ? phase[w] : std::conj(phase[w]);
      const double kappa = forward ? kh64[w][m] : kn64[w][m];
      const double factor = kappa / g.d[w];
      long lo[3] = {0, 0, 0}, hi[3] = {g.n[0], g.n[1], g.n[2]};
      lo[w] = m;
      hi[w] = m + 1;
      for (int c = 0; c < 3; c++) {
        if (c == w) continue;
        const int a = first_of(c), b = second_of(c);
        double sign = w == a ? 1.0 : -1.0;
        const int d = w == a ? b : a;
        if (!forward) sign = -sign;
        const std::vector<T> &src_re = forward ? e[d] : h[d];
        const std::vector<T> &src_im = forward ? twin->e[d] : twin->h[d];
        std::vector<T> &dst_re = forward ? h[c] : e[c];
        std::vector<T> &dst_im = forward ? twin->h[c] : twin->e[c];
        for (long k = lo[2]; k < hi[2]; k++)
          for (long j = lo[1]; j < hi[1]; j++)
            for (long i = lo[0]; i < hi[0]; i++) {
              const long r = (k * g.n[1] + j) * g.n[0] + i, q = r + o;
              const c64 f((double)src_re[q], (double)src_im[q]);
              const c64 x = cmul(c64(ph.real() - 1.0, ph.imag()), f);
              const c64 curl(x.real() * (sign * factor), x.imag() * (sign * factor));
              if (forward) {
                dst_re[r] = dst_re[r] - (T)(dt64 * curl.real());
                dst_im[r] = dst_im[r] - (T)(dt64 * curl.imag());
              } else {
                dst_re[r] = dst_re[r] + (T)(cb64[c][r] * curl.real());
                dst_im[r] = dst_im[r] + (T)(cb64[c][r] * curl.imag());
              }
            }
      }
    }
  }

  // Simulation::step (src/fdtd.rs:1319-1343): with a Bloch phase the imaginary part steps
  // alongside, each half step followed by the two parts' coupling; its media, probes and
  // monitors go first, then the real part's (whose monitors take both parts).
  void step() {
    double t = (double)steps * dt64, half = t + 0.5 * dt64;
    step_h(t);
    if (twin) {
      twin->step_h(t);
      wrap(1);
    }
    step_e(half);
    if (twin) {
      twin->step_e(half);
      wrap(0);
      twin->finish_step();
    }
    finish_step();
  }
};

template <typename T>
Sim<T> *as(orc_sim *s) { return dynamic_cast<Sim<T> *>(reinterpret_cast<Base *>(s)); }

void fill(char *err, int len, const std::string &m) {
  if (err && len > 0) snprintf(err, (size_t)len, "%s", m.c_str());
}

// Generic dispatch on the precision of a simulation.
template <typename F>
auto with(orc_sim *s, F f) {
  Base *b = reinterpret_cast<Base *>(s);
  if (auto *x = dynamic_cast<Sim<double> *>(b)) return f(*x);
  return f(*dynamic_cast<Sim<float> *>(b));
}
template <typename F>
auto with(const orc_sim *s, F f) { return with(const_cast<orc_sim *>(s), f); }

std::vector<Box> boxes_of(const double *b, int n) {
  std::vector<Box> out(n);
  for (int i = 0; i < n; i++) {
    const double *x = b + 7 * i;
    out[i] = Box{{x[0], x[2], x[4]}, {x[1], x[3], x[5]}, x[6]};
  }
  return out;
}

template <typename T>
int check_frequencies(const Sim<T> &s, int nf, const double *freqs) {
  if (nf <= 0) return -1;
  for (int f = 0; f < nf; f++)
    if (!(TAU * freqs[f] * s.dt64 < 3.141592653589793238462643383279)) return -1;
  return 0;
}

// Polynomial helpers for the medium's stability (src/fdtd/media.rs:446-513)
std::vector<double> multiply(const std::vector<double> &a, const std::vector<double> &b) {
  std::vector<double> out(a.size() + b.size() - 1, 0.0);
  for (size_t i = 0; i < a.size(); i++)
    for (size_t j = 0; j < b.size(); j++) out[i + j] += a[i] * b[j];
  return out;
}
std::vector<c64> roots(std::vector<double> p) {
  while (p.size() > 1 && p.back() == 0.0) p.pop_back();
  size_t n = p.size() - 1;
  if (n == 0) return {};
  double lead = p[n];
  for (double &c : p) c /= lead;
  double radius = std::max(refmath::ref_pow(std::fabs(p[0]), 1.0 / (double)n), 1e-3);
  std::vector<c64> z(n);
  for (size_t k = 0; k < n; k++) z[k] = std::polar(radius, TAU * ((double)k + 0.25) / (double)n);
  for (int it = 0; it < 500; it++) {
    double largest = 0.0;
    for (size_t k = 0; k < n; k++) {
      c64 v(0, 0), d(0, 0);
      for (size_t q = p.size(); q-- > 0;) {
        d = d * z[k] + v;
        v = v * z[k] + p[q];
      }
      if (v == c64(0, 0)) continue;
      c64 ratio = v / d;
      c64 rep(0, 0);
      for (size_t j = 0; j < n; j++)
        if (j != k) rep += 1.0 / (z[k] - z[j]);
      c64 step = ratio / (1.0 - ratio * rep);
      if (std::isfinite(step.real()) && std::isfinite(step.imag())) {
        z[k] -= step;
        largest = std::max(largest, std::abs(step) / std::max(std::abs(z[k]), 1e-300));
      }
    }
    if (largest < 1e-15) break;
  }
  return z;
}
double amplification(const std::vector<Pole> &poles, double eps_inf, double sigma, double dt,
                     double u) {
  std::vector<std::vector<double>> quads;
  for (const Pole &p : poles) {
    double c[3];
    p.coefficients(dt, c);
    quads.push_back({-c[1], -c[0], 1.0});
  }
  auto product = [&](long skip) {
    std::vector<double> acc{1.0};
    for (size_t i = 0; i < quads.size(); i++)
      if ((long)i != skip) acc = multiply(acc, quads[i]);
    return acc;
  };
  double e = eps_inf, half = sigma * dt / 2.0;
  std::vector<double> base{e - half, u - 2.0 * e, e + half};
  std::vector<double> poly = multiply(base, product(-1));
  for (size_t i = 0; i < poles.size(); i++) {
    double c[3];
    poles[i].coefficients(dt, c);
    double gm = c[2];
    std::vector<double> term =
        multiply({gm / 4.0, 0.0, -gm / 2.0, 0.0, gm / 4.0}, product((long)i));
    for (size_t q = 0; q < poly.size() && q < term.size(); q++) poly[q] += term[q];
  }
  double m = 0.0;
  for (const c64 &z : roots(poly)) m = std::max(m, std::abs(z));
  return m;
}
bool stable(const std::vector<Pole> &poles, double eps_inf, double sigma, double dt, double top) {
  int points = 200;
  double most = top * dt * dt;
  for (int i = 1; i <= points; i++) {
    double u = most * (double)i / (double)points;
    if (amplification(poles, eps_inf, sigma, dt, u) > 1.0 + 1e-6) return false;
  }
  return true;
}

}  // namespace

extern "C" {

int orc_average_boxes(const long n[3], const double d[3], const double o[3], const double *boxes,
                      int nbox, double background, int samples, double *out) {
  Grid g{{n[0], n[1], n[2]}, {d[0], d[1], d[2]}, {o[0], o[1], o[2]}};
  std::vector<Box> bx = boxes_of(boxes, nbox);
  long N = g.cells();
  for (int c = 0; c < 3; c++) {
#pragma omp parallel for schedule(dynamic, 256)
    for (long r = 0; r < N; r++) {
      double p[3];
      g.e_position(c, r % g.n[0], (r / g.n[0]) % g.n[1], r / (g.n[0] * g.n[1]), p);
      out[c * N + r] = averaged(bx, background, p, g.d, c, samples);
    }
  }
  return 0;
}

int orc_sample_boxes(const long n[3], const double d[3], const double o[3], const double *boxes,
                     int nbox, double background, double *out) {
  Grid g{{n[0], n[1], n[2]}, {d[0], d[1], d[2]}, {o[0], o[1], o[2]}};
  std::vector<Box> bx = boxes_of(boxes, nbox);
  long N = g.cells();
  for (int c = 0; c < 3; c++)
    for (long r = 0; r < N; r++) {
      double p[3];
      g.e_position(c, r % g.n[0], (r / g.n[0]) % g.n[1], r / (g.n[0] * g.n[1]), p);
      out[c * N + r] = geometry(bx, background, p);
    }
  return 0;
}

orc_sim *orc_create_bloch(int precision, const long n[3], const double d[3], const double o[3],
                          const int kind[3], const long low[3], const long high[3],
                          const double cpml[5], const double bloch[3], double courant,
                          const double *eps, char *err, int errlen);

orc_sim *orc_create(int precision, const long n[3], const double d[3], const double o[3],
                    const int kind[3], const long low[3], const long high[3], const double cpml[5],
                    double courant, const double *eps, char *err, int errlen) {
  const double none[3] = {0.0, 0.0, 0.0};
  return orc_create_bloch(precision, n, d, o, kind, low, high, cpml, none, courant, eps, err,
                          errlen);
}

// Simulation::with_permittivity with Bloch sides (src/fdtd.rs:680-796, src/fdtd/bloch.rs:59-83):
// a side periodic along an axis with bloch[axis] != 0 makes the fields complex.
orc_sim *orc_create_bloch(int precision, const long n[3], const double d[3], const double o[3],
                          const int kind[3], const long low[3], const long high[3],
                          const double cpml[5], const double bloch[3], double courant,
                          const double *eps, char *err, int errlen) {
  for (int a = 0; a < 3; a++)
    if (!std::isfinite(bloch[a]) || (bloch[a] != 0.0 && kind[a] != 1)) {
      fill(err, errlen, "a Bloch wavenumber must be finite, on a periodic axis");
      return nullptr;
    }
  // the checks of with_permittivity (src/fdtd.rs:686-724)
  auto ok = [](double v) { return std::isfinite(v) && v > 0.0; };
  if (n[0] * n[1] * n[2] <= 0 || !ok(d[0]) || !ok(d[1]) || !ok(d[2])) {
    fill(err, errlen, "the grid needs cells and positive steps");
    return nullptr;
  }
  if (!(cpml[0] > 0.0 && cpml[0] < 1.0) || !(std::isfinite(cpml[2]) && cpml[2] >= 0.0) ||
      !(std::isfinite(cpml[3]) && cpml[3] >= 1.0) || !(std::isfinite(cpml[4]) && cpml[4] >= 0.0) ||
      (!std::isnan(cpml[1]) && !(std::isfinite(cpml[1]) && cpml[1] >= 0.0))) {
    fill(err, errlen, "the CPML needs R in (0, 1), an order >= 0, kappa >= 1, alpha >= 0 and sigma >= 0");
    return nullptr;
  }
  for (int a = 0; a < 3; a++)
    if (kind[a] == 0 && low[a] + high[a] >= n[a]) {
      fill(err, errlen, "CPMLs leave nothing of the axis");
      return nullptr;
    }
  if (!(courant > 0.0 && courant <= 1.0)) {
    fill(err, errlen, "the Courant number must be in (0, 1]");
    return nullptr;
  }
  auto build = [&](auto *s) -> orc_sim * {
    s->g = Grid{{n[0], n[1], n[2]}, {d[0], d[1], d[2]}, {o[0], o[1], o[2]}};
    for (int a = 0; a < 3; a++) {
      s->kind[a] = kind[a];
      s->low[a] = kind[a] == 0 ? low[a] : 0;
      s->high[a] = kind[a] == 0 ? high[a] : 0;
    }
    for (int i = 0; i < 5; i++) s->cpml[i] = cpml[i];
    for (int a = 0; a < 3; a++) s->bloch_k[a] = bloch[a];
    std::string m;
    if (!s->init(eps, courant, m)) {
      fill(err, errlen, m);
      delete s;
      return nullptr;
    }
    s->materialize();
    if (bloch[0] != 0.0 || bloch[1] != 0.0 || bloch[2] != 0.0) {
      for (int a = 0; a < 3; a++) {
        s->along[a] = bloch[a] != 0.0;
        double sn, cs;  // from_polar(1, k L)
        refmath::ref_sincos(bloch[a] * ((double)n[a] * d[a]), &sn, &cs);
        s->phase[a] = c64(1.0 * cs, 1.0 * sn);
      }
      s->twin = new typename std::remove_reference<decltype(*s)>::type(*s);
    }
    return reinterpret_cast<orc_sim *>(static_cast<Base *>(s));
  };
  if (precision == 32) return build(new Sim<float>());
  return build(new Sim<double>());
}

void orc_destroy(orc_sim *s) { delete reinterpret_cast<Base *>(s); }

int orc_conductivity(orc_sim *s, const double *sigma, char *err, int errlen) {
  // Simulation::conductivity (src/fdtd.rs:949-992)
  auto body = [&](auto &x) -> int {
    if (!x.groups.empty()) {
      fill(err, errlen, "the conductivity comes before the dispersive media");
      return -1;
    }
    long N = x.g.cells();
    for (int c = 0; c < 3; c++)
      for (long r = 0; r < N; r++) {
        if (x.cb64[c][r] == 0.0) continue;
        double sg = sigma[c * N + r];
        if (!(std::isfinite(sg) && sg >= 0.0)) {
          fill(err, errlen, "the conductivity must be finite and >= 0");
          return -1;
        }
        double half = sg * x.cb64[c][r] / 2.0;
        x.ca64[c][r] = (1.0 - half) / (1.0 + half);
        x.cb64[c][r] /= 1.0 + half;
      }
    x.refresh_coefficients();
    return 0;
  };
  // a Bloch run's imaginary part takes it too (src/fdtd.rs:962-964, 1005-1007;
  // src/fdtd/media.rs:756-759)
  return with(s, [&](auto &x) -> int {
    if (x.twin)
      if (int r = body(*x.twin)) return r;
    return body(x);
  });
}

int orc_conductor(orc_sim *s, int comp, long i, long j, long k) {
  auto body = [&](auto &x) -> int {  // src/fdtd.rs:995-1008
    long r = (k * x.g.n[1] + j) * x.g.n[0] + i;
    x.ca64[comp][r] = x.cb64[comp][r] = 0.0;
    x.ca[comp][r] = x.cb[comp][r] = 0;
    x.e[comp][r] = 0;
    auto it = x.members.find({comp, r});
    if (it != x.members.end()) {  // Media::remove (src/fdtd/media.rs:641-653)
      auto &gr = x.groups[it->second];
      std::vector<std::pair<int, long>> keep;
      decltype(gr.scale) sc;
      for (size_t v = 0; v < gr.values.size(); v++)
        if (gr.values[v] != std::make_pair(comp, r)) {
          keep.push_back(gr.values[v]);
          sc.push_back(gr.scale[v]);
        }
      gr.values = keep;
      gr.scale = sc;
      gr.resize();
      x.members.erase(it);
    }
    return 0;
  };
  // a Bloch run's imaginary part takes it too (src/fdtd.rs:962-964, 1005-1007;
  // src/fdtd/media.rs:756-759)
  return with(s, [&](auto &x) -> int {
    if (x.twin)
      if (int r = body(*x.twin)) return r;
    return body(x);
  });
}

int orc_add_source(orc_sim *s, int field, int comp, long i, long j, long k, const double *wave) {
  return with(s, [&](auto &x) -> int {
    if (i < 0 || j < 0 || k < 0 || i >= x.g.n[0] || j >= x.g.n[1] || k >= x.g.n[2]) return -1;
    x.emitters.push_back(Wave::from(wave));
    // point sources enter before every current (src/fdtd.rs:1348-1359): keep them in front
    Injection in{field, comp, (k * x.g.n[1] + j) * x.g.n[0] + i, c64(1, 0),
                 (int)x.emitters.size() - 1, true};
    size_t at = 0;
    while (at < x.injections.size() && x.injections[at].point) at++;
    x.injections.insert(x.injections.begin() + at, in);
    return 0;
  });
}

int orc_add_current(orc_sim *s, int field, long count, const int *comps, const long *at,
                    const double *amps, const double *wave) {
  return with(s, [&](auto &x) -> int {  // src/fdtd/sources.rs:223-242
    for (long q = 0; q < count; q++) {
      const long *p = at + 3 * q;
      if (p[0] < 0 || p[1] < 0 || p[2] < 0 || p[0] >= x.g.n[0] || p[1] >= x.g.n[1] ||
          p[2] >= x.g.n[2])
        return -1;
      if (!std::isfinite(amps[2 * q]) || !std::isfinite(amps[2 * q + 1])) return -1;
    }
    std::vector<std::pair<int, long>> where;
    std::vector<c64> a;
    for (long q = 0; q < count; q++) {
      const long *p = at + 3 * q;
      where.push_back({comps[q], (p[2] * x.g.n[1] + p[1]) * x.g.n[0] + p[0]});
      a.push_back(c64(amps[2 * q], amps[2 * q + 1]));
    }
    x.push_current(field, where, a, Wave::from(wave));
    return 0;
  });
}

int orc_add_dipole(orc_sim *s, int field, int comp, const double pos[3], double are, double aim,
                   const double *wave) {
  return with(s, [&](auto &x) -> int {  // src/fdtd/sources.rs:248-315 (no Bloch phase)
    c64 a(are, aim);
    if (!std::isfinite(are) || !std::isfinite(aim)) return -1;
    long idx[3][2];
    double wt[3][2];
    double volume = 1.0;
    for (int axis = 0; axis < 3; axis++) {
      long n = x.g.n[axis];
      if (!x.varies[axis]) {
        idx[axis][0] = idx[axis][1] = 0;
        wt[axis][0] = 1.0;
        wt[axis][1] = 0.0;
        continue;
      }
      volume *= x.g.d[axis];
      bool half = field == 0 ? comp == axis : comp != axis;
      double first = x.g.node(axis, 0) + (half ? 0.5 * x.g.d[axis] : 0.0);
      double sp = (pos[axis] - first) / x.g.d[axis];
      bool per = x.periodic(axis);
      if (!per && !(sp >= 0.0 && sp <= (double)(n - 1))) return -1;
      double m = std::floor(sp), f = sp - m;
      if (per) {
        long m0 = (long)m;
        idx[axis][0] = ((m0 % n) + n) % n;
        idx[axis][1] = (((m0 + 1) % n) + n) % n;
      } else {
        idx[axis][0] = (long)m;
        idx[axis][1] = std::min((long)m + 1, n - 1);
      }
      wt[axis][0] = 1.0 - f;
      wt[axis][1] = f;
    }
    std::map<long, c64> values;
    if (x.twin) {  // a Bloch run: each value beyond a periodic end takes its image's phase
      c64 cw[3][2];
      for (int axis = 0; axis < 3; axis++)
        for (int q = 0; q < 2; q++) {
          c64 image(1.0, 0.0);
          if (x.varies[axis] && x.periodic(axis)) {
            const double sp = (pos[axis] - (x.g.node(axis, 0) +
                                            ((field == 0 ? comp == axis : comp != axis)
                                                 ? 0.5 * x.g.d[axis] : 0.0))) / x.g.d[axis];
            const long m = (long)std::floor(sp) + q, n = x.g.n[axis];
            const long turns = m >= 0 ? m / n : -((-m + n - 1) / n);
            image = x.image(axis, turns);
          }
          cw[axis][q] = c64(image.real() * wt[axis][q], image.imag() * wt[axis][q]);
        }
      for (int p = 0; p < 2; p++)
        for (int q = 0; q < 2; q++)
          for (int r = 0; r < 2; r++) {
            const c64 w = cmul(cmul(cw[0][p], cw[1][q]), cw[2][r]);
            if (w.real() != 0.0 || w.imag() != 0.0) {
              long at = (idx[2][r] * x.g.n[1] + idx[1][q]) * x.g.n[0] + idx[0][p];
              c64 add = cmul(a, c64(w.real() / volume, w.imag() / volume));
              c64 &acc = values[at];
              acc = c64(acc.real() + add.real(), acc.imag() + add.imag());
            }
          }
    } else
    for (int p = 0; p < 2; p++)
      for (int q = 0; q < 2; q++)
        for (int r = 0; r < 2; r++) {
          double w = wt[0][p] * wt[1][q] * wt[2][r];
          if (w != 0.0) {
            long at = (idx[2][r] * x.g.n[1] + idx[1][q]) * x.g.n[0] + idx[0][p];
            c64 scaled(w / volume, 0.0);
            c64 add = cmul(a, scaled);
            c64 &acc = values[at];
            acc = c64(acc.real() + add.real(), acc.imag() + add.imag());
          }
        }
    std::vector<std::pair<int, long>> where;
    std::vector<c64> amounts;
    for (auto &kv : values) {
      where.push_back({comp, kv.first});
      amounts.push_back(kv.second);
    }
    x.push_current(field, where, amounts, Wave::from(wave));
    return 0;
  });
}

int orc_add_probe(orc_sim *s, int field, int comp, long i, long j, long k) {
  return with(s, [&](auto &x) -> int {
    if (i < 0 || j < 0 || k < 0 || i >= x.g.n[0] || j >= x.g.n[1] || k >= x.g.n[2]) return -1;
    typename std::remove_reference<decltype(x)>::type::Probe p{
        field, comp, (k * x.g.n[1] + j) * x.g.n[0] + i, {}};
    x.probes.push_back(p);
    if (x.twin) x.twin->probes.push_back(p);
    return (int)x.probes.size() - 1;
  });
}

int orc_add_dft(orc_sim *s, const long low[3], const long high[3], int nf, const double *freqs) {
  return with(s, [&](auto &x) -> int {  // src/fdtd/monitors.rs:442-464
    if (check_frequencies(x, nf, freqs)) return -1;
    for (int a = 0; a < 3; a++)
      if (high[a] >= x.g.n[a] || low[a] > high[a] || low[a] < 0) return -1;
    Dft d;
    d.freqs.assign(freqs, freqs + nf);
    for (int field = 0; field < 2; field++)
      for (int c = 0; c < 3; c++) {
        Series sr;
        sr.field = field;
        sr.comp = c;
        for (int a = 0; a < 3; a++) {
          sr.lo[a] = low[a];
          sr.len[a] = high[a] - low[a] + 1;
        }
        sr.values.assign(sr.volume() * nf, c64(0, 0));
        d.series.push_back(sr);
      }
    x.dfts.push_back(d);
    return (int)x.dfts.size() - 1;
  });
}

int orc_add_flux(orc_sim *s, int axis, long plane, const long window[4], int nf,
                 const double *freqs) {
  return with(s, [&](auto &x) -> int {  // src/fdtd/monitors.rs:483-492
    if (check_frequencies(x, nf, freqs)) return -1;
    FluxPlane fp{axis, plane, {{window[0], window[1]}, {window[2], window[3]}}};
    if (plane + 1 >= x.g.n[axis] || plane < 0) return -1;
    for (int sl = 0; sl < 2; sl++) {
      int along = sl == 0 ? first_of(axis) : second_of(axis);
      if (fp.win[sl][0] >= 0 && !(fp.win[sl][0] < fp.win[sl][1] && fp.win[sl][1] < x.g.n[along]))
        return -1;
    }
    Flux f;
    f.planes.push_back(fp);
    f.signs.push_back(1.0);
    Dft d;
    d.freqs.assign(freqs, freqs + nf);
    d.series = fp.series(x.g, nf);
    f.dfts.push_back(d);
    x.fluxes.push_back(f);
    return (int)x.fluxes.size() - 1;
  });
}

int orc_add_flux_box(orc_sim *s, const long planes[6], int nf, const double *freqs) {
  return with(s, [&](auto &x) -> int {  // src/fdtd/monitors.rs:503-531
    if (check_frequencies(x, nf, freqs)) return -1;
    Flux f;
    for (int axis = 0; axis < 3; axis++) {
      long lo = planes[2 * axis], hi = planes[2 * axis + 1];
      int b = first_of(axis), c = second_of(axis);
      if (lo >= hi) return -1;
      for (int side = 0; side < 2; side++) {
        FluxPlane fp{axis, side == 0 ? lo : hi,
                     {{planes[2 * b], planes[2 * b + 1]}, {planes[2 * c], planes[2 * c + 1]}}};
        if (fp.plane + 1 >= x.g.n[axis]) return -1;
        Dft d;
        d.freqs.assign(freqs, freqs + nf);
        d.series = fp.series(x.g, nf);
        f.planes.push_back(fp);
        f.signs.push_back(side == 0 ? -1.0 : 1.0);
        f.dfts.push_back(d);
      }
    }
    x.fluxes.push_back(f);
    return (int)x.fluxes.size() - 1;
  });
}

int orc_add_medium(orc_sim *s, double eps_inf, int npoles, const double *poles,
                   const unsigned char *inside, int check_stability, char *err, int errlen) {
  auto body = [&](auto &x) -> int {  // Simulation::medium (src/fdtd/media.rs:741-825)
    using T = typename std::remove_reference<decltype(x.dt)>::type;
    if (x.steps > 0) {
      fill(err, errlen, "a dispersive medium goes in before the run starts");
      return -1;
    }
    std::vector<Pole> ps;
    for (int p = 0; p < npoles; p++)
      ps.push_back(Pole{(int)poles[4 * p], poles[4 * p + 1], poles[4 * p + 2], poles[4 * p + 3]});
    double dt = x.dt64;
    std::vector<std::array<double, 3>> co;
    double gsum = 0.0;
    for (const Pole &p : ps) {
      std::array<double, 3> c;
      p.coefficients(dt, c.data());
      co.push_back(c);
      gsum += c[2];
    }
    double chi = gsum / (4.0 * dt);
    long N = x.g.cells();
    std::vector<std::pair<int, long>> values;
    std::vector<double> sigmas;
    for (int c = 0; c < 3; c++)
      for (long r = 0; r < N; r++) {
        if (x.cb64[c][r] == 0.0 || !inside[c * N + r]) continue;
        double old_chi = 0.0;
        auto it = x.members.find({c, r});
        if (it != x.members.end()) old_chi = (double)x.groups[it->second].chi;
        double sg = (1.0 - x.ca64[c][r]) / x.cb64[c][r] - old_chi;
        values.push_back({c, r});
        sigmas.push_back(std::max(sg, 0.0));
      }
    if (check_stability) {
      const double top = 4.0 * x.curl_bound();
      double largest = 0.0;
      for (double sg : sigmas) largest = std::max(largest, sg);
      for (double sg : {0.0, largest})
        if (!stable(ps, eps_inf, sg, dt, top)) {
          fill(err, errlen, "the medium isn't stable at this time step");
          return -1;
        }
    }
    std::vector<T> scale;
    // Media::remove of every value this medium takes over: each old group keeps its other values
    // in their order. Done a group at a time (one pass over each group that loses values) rather
    // than one pass per value, which is the same result.
    std::map<int, std::unordered_set<long>> leaving;
    for (size_t v = 0; v < values.size(); v++) {
      auto it = x.members.find(values[v]);
      if (it != x.members.end()) {
        leaving[it->second].insert(values[v].first * N + values[v].second);
        x.members.erase(it);
      }
    }
    for (auto &kv : leaving) {
      auto &gr = x.groups[kv.first];
      std::vector<std::pair<int, long>> keep;
      std::vector<T> sc;
      for (size_t q = 0; q < gr.values.size(); q++)
        if (!kv.second.count(gr.values[q].first * N + gr.values[q].second)) {
          keep.push_back(gr.values[q]);
          sc.push_back(gr.scale[q]);
        }
      gr.values = keep;
      gr.scale = sc;
      gr.resize();
    }
    for (size_t v = 0; v < values.size(); v++) {
      int c = values[v].first;
      long r = values[v].second;
      double sg = sigmas[v];
      double nu = 1.0 + dt / eps_inf * (sg / 2.0 + chi);
      x.ca64[c][r] = (1.0 - dt * sg / (2.0 * eps_inf)) / nu;
      x.cb64[c][r] = dt / eps_inf / nu;
      x.ca[c][r] = (T)x.ca64[c][r];
      x.cb[c][r] = (T)x.cb64[c][r];
      scale.push_back((T)x.cb64[c][r]);
    }
    if (!ps.empty() && !values.empty()) {
      int gi = (int)x.groups.size();
      for (auto &v : values) x.members[v] = gi;
      Group<T> gr;
      gr.values = values;
      gr.scale = scale;
      gr.chi = (T)chi;
      for (auto &c : co) gr.poles.push_back({(T)c[0], (T)c[1], (T)c[2]});
      gr.resize();
      x.groups.push_back(gr);
    }
    return 0;
  };
  // a Bloch run's imaginary part takes it too (src/fdtd.rs:962-964, 1005-1007;
  // src/fdtd/media.rs:756-759)
  return with(s, [&](auto &x) -> int {
    if (x.twin)
      if (int r = body(*x.twin)) return r;
    return body(x);
  });
}

void orc_run(orc_sim *s, long steps) {
  with(s, [&](auto &x) -> int {
    for (long n = 0; n < steps; n++) x.step();
    return 0;
  });
}

double orc_dt(const orc_sim *s) { return with(s, [](auto &x) -> double { return x.dt64; }); }
long orc_steps(const orc_sim *s) { return with(s, [](auto &x) -> long { return x.steps; }); }

void orc_get_field(const orc_sim *s, int field, int comp, double *out) {
  with(s, [&](auto &x) -> int {
    auto &v = field == 0 ? x.e[comp] : x.h[comp];
    for (size_t r = 0; r < v.size(); r++) out[r] = (double)v[r];
    return 0;
  });
}

void orc_set_field(orc_sim *s, int field, int comp, const double *in) {
  with(s, [&](auto &x) -> int {
    using T = typename std::remove_reference<decltype(x.dt)>::type;
    auto &v = field == 0 ? x.e[comp] : x.h[comp];
    for (size_t r = 0; r < v.size(); r++) v[r] = (T)in[r];
    return 0;
  });
}

long orc_probe(const orc_sim *s, int p, double *out) {
  return with(s, [&](auto &x) -> long {
    auto &v = x.probes[p].values;
    if (out) std::copy(v.begin(), v.end(), out);
    return (long)v.size();
  });
}

long orc_transforms(const orc_sim *s, double *out) {
  return with(s, [&](auto &x) -> long {
    long at = 0;
    auto put = [&](const Dft &d) {
      for (const Series &sr : d.series)
        for (const c64 &v : sr.values) {
          if (out) {
            out[2 * at] = v.real();
            out[2 * at + 1] = v.imag();
          }
          at++;
        }
    };
    for (const Dft &d : x.dfts) put(d);
    for (const Flux &f : x.fluxes)
      for (const Dft &d : f.dfts) put(d);
    return at;
  });
}

int orc_flux(const orc_sim *s, int n, double *out) {
  return with(s, [&](auto &x) -> int {  // Simulation::flux (src/fdtd/monitors.rs:539-552)
    const Flux &f = x.fluxes[n];
    size_t nf = f.dfts[0].freqs.size();
    for (size_t q = 0; q < nf; q++) {
      double total = 0.0;
      for (size_t p = 0; p < f.planes.size(); p++)
        total += f.signs[p] * f.planes[p].flux(x.g, f.dfts[p], (int)q);
      out[q] = total;
    }
    return (int)nf;
  });
}

long orc_tables(const orc_sim *s, int which, double *out) {
  return with(s, [&](auto &x) -> long {
    long at = 0;
    auto put = [&](double v) {
      if (out) out[at] = v;
      at++;
    };
    if (which == 0 || which == 1) {
      for (int c = 0; c < 3; c++)
        for (double v : (which == 0 ? x.ca64[c] : x.cb64[c])) put(v);
    } else if (which == 2 || which == 3) {
      for (int c = 0; c < 3; c++)
        for (long m = 0; m < x.g.n[c]; m++)
          put((which == 2 ? x.kn64[c][m] : x.kh64[c][m]) / x.g.d[c]);
    } else if (which == 4) {
      for (const SlabInfo &sl : x.slabs) {
        put(sl.field);
        put(sl.comp);
        put(sl.axis);
        put((double)sl.from);
        put((double)sl.count);
        for (double v : sl.b) put(v);
        for (double v : sl.a) put(v);
      }
    } else if (which == 5) {  // the media groups: chi, poles, members (comp, index, scale)
      for (const auto &gr : x.groups) {
        put((double)gr.chi);
        put((double)gr.poles.size());
        for (const auto &p : gr.poles)
          for (int q = 0; q < 3; q++) put((double)p[q]);
        put((double)gr.values.size());
        for (size_t v = 0; v < gr.values.size(); v++) {
          put(gr.values[v].first);
          put((double)gr.values[v].second);
          put((double)gr.scale[v]);
        }
      }
    }
    return at;
  });
}

int orc_medium_stable(double eps_inf, int npoles, const double *poles, double sigma, double dt,
                      double top) {
  std::vector<Pole> ps;
  for (int p = 0; p < npoles; p++)
    ps.push_back(Pole{(int)poles[4 * p], poles[4 * p + 1], poles[4 * p + 2], poles[4 * p + 3]});
  return stable(ps, eps_inf, sigma, dt, top) ? 1 : 0;
}

int orc_dft_value(const orc_sim *s, int monitor, int field, int comp, const long at[3], int f,
                  double *out) {
  return with(s, [&](auto &x) -> int {
    if (monitor < 0 || monitor >= (int)x.dfts.size()) return 0;
    c64 v;
    if (!x.dfts[monitor].value(field, comp, at, f, &v)) return 0;
    out[0] = v.real();
    out[1] = v.imag();
    return 1;
  });
}

long orc_flux_derivatives(const orc_sim *s, int monitor, int f, double scale, long *keys,
                          double *values, long capacity) {
  // the derivative of flux monitor `monitor`'s flux at frequency f with respect to each
  // transform it reads, times scale (src/fdtd/adjoint.rs:1036-1083, flux_derivatives, each face
  // with its sign): the flux is the sum of w sign Re(1/2 (low + high) conj(H)) area, so with
  // kappa = scale w sign area / 2 the derivative is kappa conj(H) / 2 at each of the two E
  // planes and kappa conj(low + high) / 2 at H. Entries (field, component, index) in keys[3q],
  // the complex derivative in values[2q]. Returns the count (keys may be null to ask).
  return with(s, [&](auto &x) -> long {
    if (monitor < 0 || monitor >= (int)x.fluxes.size()) return -1;
    const Flux &fl = x.fluxes[monitor];
    const Grid &g = x.g;
    long n = 0;
    auto put = [&](int field, int comp, const long at[3], c64 v) {
      if (keys && n < capacity) {
        keys[3 * n] = field;
        keys[3 * n + 1] = comp;
        keys[3 * n + 2] = (at[2] * g.n[1] + at[1]) * g.n[0] + at[0];
        values[2 * n] = v.real();
        values[2 * n + 1] = v.imag();
      }
      n++;
    };
    for (size_t face = 0; face < fl.planes.size(); face++) {
      const FluxPlane &pl = fl.planes[face];
      const Dft &dft = fl.dfts[face];
      const int b = first_of(pl.axis), c = second_of(pl.axis);
      const double area = g.d[b] * g.d[c];
      struct T3 { int comp, h; double sign; };
      const T3 terms[2] = {{b, c, 0.5}, {c, b, -0.5}};
      for (const T3 &t : terms)
        for (long v = pl.range_lo(g, c); v < pl.range_hi(g, c); v++)
          for (long u = pl.range_lo(g, b); u < pl.range_hi(g, b); u++) {
            const double w = pl.weight(b, u, t.comp == b) * pl.weight(c, v, t.comp == c);
            if (w == 0.0) continue;
            const double kappa = scale * fl.signs[face] * w * t.sign * 0.5 * area;
            long at[3];
            at[pl.axis] = pl.plane;
            at[b] = u;
            at[c] = v;
            c64 hv, low, high;
            dft.value(1, t.h, at, f, &hv);
            dft.value(0, t.comp, at, f, &low);
            long at2[3] = {at[0], at[1], at[2]};
            at2[pl.axis] = pl.plane + 1;
            dft.value(0, t.comp, at2, f, &high);
            put(0, t.comp, at, 0.5 * kappa * std::conj(hv));
            put(0, t.comp, at2, 0.5 * kappa * std::conj(hv));
            put(1, t.h, at, 0.5 * kappa * std::conj(low + high));
          }
    }
    return n;
  });
}

double orc_triad(long len, int repeats) {
  // the STREAM triad as the reference measures its host's bandwidth (src/traffic.rs:56-80):
  // a = b + s c over `len` doubles on all threads, the best of `repeats`, 24 bytes an element
  std::vector<double> a(len, 0.0), b(len, 1.0), c(len, 2.0);
  volatile double sv = 3.0;
  const double sc = sv;
  double best = 1e300;
  for (int r = 0; r < std::max(1, repeats); r++) {
    const double t0 = omp_get_wtime();
#pragma omp parallel for schedule(static, 1 << 14)
    for (long q = 0; q < len; q++) a[q] = b[q] + sc * c[q];
    best = std::min(best, omp_get_wtime() - t0);
  }
  volatile double sink = a[len / 2];
  (void)sink;
  return 24.0 * (double)len / best / 1e9;
}

// Simulation::add_plane_wave / PlaneWaveRun::new (src/fdtd/sources.rs:716-951): the box from
// nodes low to high, the direction (p, q, s) in cells, E's polarization, the background's eps.
// Returns the wave's number, or -1 with the reason in err.
int orc_add_plane_wave(orc_sim *s, const long low[3], const long high[3], const long dir[3],
                       const double pol[3], double eps, const double *wave, char *err,
                       int errlen) {
  return with(s, [&](auto &x) -> int {
    if (x.twin)  // Simulation::real_run (src/fdtd/sources.rs:209-221)
      return fill(err, errlen, "a plane wave needs real fields: with a Bloch phase, launch a "
                               "Current with it instead"), -1;
    auto gcd = [](long a, long b) {
      while (b != 0) {
        const long t = a % b;
        a = b;
        b = t;
      }
      return a < 0 ? -a : a;
    };
    PlaneRun run;
    const long divisor = gcd(gcd(dir[0], dir[1]), dir[2]);
    if (divisor == 0) return fill(err, errlen, "a plane wave's direction can't be zero"), -1;
    for (int a = 0; a < 3; a++) run.g[a] = dir[a] / divisor;
    if (!(std::isfinite(eps) && eps > 0.0))
      return fill(err, errlen, "the background's permittivity must be positive"), -1;
    bool faces[3];
    for (int a = 0; a < 3; a++) {
      const long n = x.g.n[a];
      faces[a] = true;
      if (x.periodic(a)) {
        if (low[a] != 0 || high[a] != n || run.g[a] != 0)
          return fill(err, errlen, "along a periodic axis the box must be whole and the direction "
                                   "zero"), -1;
        faces[a] = false;
      } else {
        const long lo = x.low[a], hi = x.high[a];
        if (low[a] < lo + 1 || high[a] + hi + 1 > n || low[a] >= high[a])
          return fill(err, errlen, "the box's faces must be in order and a cell clear of the CPMLs "
                                   "and the ends"), -1;
      }
    }
    for (int a = 0; a < 3; a++) run.steps[a] = x.g.d[a];
    double gv[3], khat[3], pt[3];
    for (int a = 0; a < 3; a++) gv[a] = (double)run.g[a] / run.steps[a];
    double sq = 0.0;
    for (int a = 0; a < 3; a++) sq += gv[a] * gv[a];
    const double norm = std::sqrt(sq);
    for (int a = 0; a < 3; a++) khat[a] = gv[a] / norm;
    double along = 0.0;
    for (int a = 0; a < 3; a++) along += pol[a] * khat[a];
    for (int a = 0; a < 3; a++) pt[a] = pol[a] - along * khat[a];
    double size2 = 0.0;
    for (int a = 0; a < 3; a++) size2 += pt[a] * pt[a];
    const double size = std::sqrt(size2);
    if (!(std::isfinite(size) && size > 1e-12))
      return fill(err, errlen, "the polarization has nothing across the direction"), -1;
    for (int a = 0; a < 3; a++) pt[a] /= size;
    auto total = [&](int field, int comp, const long at[3]) {
      for (int a = 0; a < 3; a++) {
        if (!faces[a]) continue;
        const long t = twice(field, comp, a, at[a]);
        if (!(t >= 2 * low[a] && t <= 2 * high[a])) return false;
      }
      return true;
    };
    long rlo[3], rhi[3];
    for (int a = 0; a < 3; a++) {
      rlo[a] = faces[a] ? low[a] - 1 : 0;
      rhi[a] = faces[a] ? high[a] + 2 : x.g.n[a];
    }
    const std::vector<Link> ls = x.links(rlo, rhi, total);
    if (!x.uniform(ls, eps))
      return fill(err, errlen, "the medium on the box's surface must be uniform, with the "
                               "permittivity eps and no conductivity"), -1;
    long least = 0, most = 0;
    for (int a = 0; a < 3; a++) {
      const long t0 = faces[a] ? 2 * low[a] - 2 : 0, t1 = faces[a] ? 2 * high[a] + 2 : 0;
      least += std::min(run.g[a] * t0, run.g[a] * t1);
      most += std::max(run.g[a] * t0, run.g[a] * t1);
    }
    long stride = 0;
    for (int a = 0; a < 3; a++) stride = std::max(stride, run.g[a] < 0 ? -run.g[a] : run.g[a]);
    const long pad = stride, absorber = 200 * stride;
    const long sheet_at = least - 4 * stride - 4;
    long base = sheet_at - (absorber + 4 * stride + pad);
    base -= ((base % 2) + 2) % 2;
    const long top = most + (4 * stride + absorber + pad);
    const long len = top - base + 1;
    const double sample = 1.0 / (2.0 * norm);
    const double depth = (double)absorber * sample;
    const double sqrt_eps = std::sqrt(eps);
    const double sigma_max = 50.0 * sqrt_eps / depth;
    const double dt = x.dt64;
    run.ca.assign(len, 1.0);
    run.cb.assign(len, dt / eps);
    run.da.assign(len, 1.0);
    run.db.assign(len, dt);
    for (long i = 0; i < len; i++) {
      double into;
      if (i < pad + absorber) into = (double)(pad + absorber - i);
      else if (i + pad + absorber >= len) into = (double)(i + pad + absorber + 1 - len);
      else continue;
      const double v = std::min(into / (double)absorber, 1.0);
      const double sigma = sigma_max * (v * (v * v));  // portable::powi(v, 3)
      const double half_e = sigma * dt / (2.0 * eps);
      run.ca[i] = (1.0 - half_e) / (1.0 + half_e);
      run.cb[i] = dt / eps / (1.0 + half_e);
      const double half_h = sigma / eps * dt / 2.0;
      run.da[i] = (1.0 - half_h) / (1.0 + half_h);
      run.db[i] = dt / (1.0 + half_h);
    }
    for (int c = 0; c < 3; c++) {
      if (pt[c] == 0.0) continue;
      const double j = -2.0 * sqrt_eps * norm * pt[c];
      if ((((sheet_at - run.g[c]) % 2) + 2) % 2 == 0) {
        run.sheet.push_back({c, sheet_at - base, j});
      } else {
        run.sheet.push_back({c, sheet_at - 1 - base, 0.5 * j});
        run.sheet.push_back({c, sheet_at + 1 - base, 0.5 * j});
      }
    }
    run.base = base;
    run.pad = pad;
    run.len = len;
    for (int c = 0; c < 3; c++) {
      run.e[c].assign(len, 0.0);
      run.h[c].assign(len, 0.0);
    }
    run.wave = Wave::from(wave);
    for (const Link &l : ls) {
      long i;
      if (!run.sample(l.from_field, l.from_comp, l.from, &i))
        return fill(err, errlen, "the auxiliary grid doesn't span the box"), -1;
      PlaneRun::Coupling q{l.comp, l.r, l.weight, l.from_comp, i};
      (l.target == 0 ? run.on_e : run.on_h).push_back(q);
    }
    x.plane_waves.push_back(run);
    return (int)x.plane_waves.size() - 1;
  });
}

// Simulation::incident (src/fdtd/sources.rs:729-767): plane wave n's incident field now at a value.
double orc_incident(const orc_sim *s, int n, int field, int comp, long i, long j, long k) {
  return with(s, [&](auto &x) -> double {
    if (n < 0 || n >= (int)x.plane_waves.size()) return 0.0;
    const long at[3] = {i, j, k};
    return x.plane_waves[n].value(field, comp, at);
  });
}

// The host threads the oracle's loops use (a column of a few hundred cells runs fastest on one).
int orc_threads(int n) {
  const int before = omp_get_max_threads();
  if (n > 0) omp_set_num_threads(n);
  return before;
}

// A complex run's imaginary part (src/fdtd.rs:911-935, 1094-1110): 1 if the run is complex.
int orc_is_complex(const orc_sim *s) {
  return with(s, [&](auto &x) -> int { return x.twin ? 1 : 0; });
}
int orc_get_field_imag(const orc_sim *s, int field, int comp, double *out) {
  return with(s, [&](auto &x) -> int {
    if (!x.twin) return -1;
    const auto &v = field == 0 ? x.twin->e[comp] : x.twin->h[comp];
    for (size_t r = 0; r < v.size(); r++) out[r] = (double)v[r];
    return 0;
  });
}
long orc_probe_imag(const orc_sim *s, int p, double *out) {
  return with(s, [&](auto &x) -> long {
    if (!x.twin) return -1;
    const auto &v = x.twin->probes[p].values;
    if (out) std::copy(v.begin(), v.end(), out);
    return (long)v.size();
  });
}

// Waveform::spectrum (src/fdtd.rs:361-396): the sum from zero, in step order, of
// (w.at(t) + 0i) exp(i omega t) dt with t = n dt (+ dt/2 for E, field 0).
int orc_waveform_spectrum(const double *wave, int field, double dt, long steps, int nf,
                          const double *freqs, double *out) {
  if (!wave || !freqs || !out || nf < 0 || steps < 0 || !(dt > 0.0)) return -1;
  const Wave w = Wave::from(wave);
  const double offset = field == 0 ? 0.5 * dt : 0.0;
  for (int f = 0; f < nf; f++) {
    const double omega = TAU * freqs[f];
    c64 sum(0.0, 0.0);
    for (long n = 0; n < steps; n++) {
      const double t = (double)n * dt + offset;
      const c64 v = cmul(c64(w.at(t), 0.0), cis(omega * t));
      sum = c64(sum.real() + v.real() * dt, sum.imag() + v.imag() * dt);
    }
    out[2 * f] = sum.real();
    out[2 * f + 1] = sum.imag();
  }
  return 0;
}

}  // extern "C"
