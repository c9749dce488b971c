/*
 * ORACLE (test infrastructure only). A CPU restatement of photonoxide's FDTD time step, used by
 * the tests, the smoke check and the CPU-baseline leg of the benchmark to CHECK the CUDA engine.
 * Nothing in the product links, loads or calls it.
 *
 * Parity anchor: the reference is a Rust crate that cannot be built here (no cargo/rustc, its
 * crates.io dependencies are not vendored), so this is a restatement of its source. It is pinned
 * to the reference by the reference's own known answers, first of all the bit hash of
 * tests/canary.rs:1007-1062 (a 2D run whose fields must hash to 0x7c8db7ae69980888).
 *
 * The same code runs in f64 (the reference's precision and the parity target) and in f32 (the
 * reference's `Yee<f32>` kernel arithmetic, src/fdtd/kernel/yee.rs:12-153, which the CUDA engine
 * computes bit for bit on source-free problems). Setup is always f64, as in the reference.
 *
 * Conventions: field 0 = E, 1 = H (H~ = eta0 H); component/axis 0,1,2 = x,y,z; a value's index
 * r = (k*ny + j)*nx + i within a component (src/fdfd/three.rs:123-125).
 */
#ifndef PHOTONOXIDE_FDTD_ORACLE_H
#define PHOTONOXIDE_FDTD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sim orc_sim;

/* Waveform as 6 doubles: {kind, p1..p5}.
 * kind 0 Gaussian {frequency (c/um), width, delay};
 * kind 1 DifferentiatedGaussian {width, delay};
 * kind 2 Continuous {frequency, amplitude re, amplitude im, ramp}.  (src/fdtd.rs:259-434) */

/* FDFD's cell average of a box geometry's permittivity at every value of E (src/fdfd/three.rs:
 * 563-588, called by src/fdtd.rs:570-604): boxes are 7 doubles {xlo,xhi,ylo,yhi,zlo,zhi,eps},
 * a point inside when lo < p < hi on each axis, later boxes over earlier ones. */
int orc_average_boxes(const long n[3], const double d[3], const double o[3], const double *boxes,
                      int nbox, double background, int samples, double *out);
/* The same geometry sampled at each value of E, not averaged (conductivity, media). */
int orc_sample_boxes(const long n[3], const double d[3], const double o[3], const double *boxes,
                     int nbox, double background, double *out);

/* Simulation::with_permittivity (src/fdtd.rs:680-796). kind[a]: 0 CPML of low/high cells (0 =
 * wall), 1 periodic. cpml = {reflection, sigma (NaN: from reflection), order, kappa, alpha}.
 * eps: 3 x cells per-value permittivity. precision 64 or 32. NULL on error (err filled). */
orc_sim *orc_create(int precision, const long n[3], const double d[3], const double o[3],
                    const int kind[3], const long low[3], const long high[3], const double cpml[5],
                    double courant, const double *eps, char *err, int errlen);
/* The same with Bloch sides: bloch[a] != 0 on a periodic axis makes the fields complex, the
 * imaginary part a second run stepped alongside (src/fdtd/bloch.rs). */
orc_sim *orc_create_bloch(int precision, const long n[3], const double d[3], const double o[3],
                          const int kind[3], const long low[3], const long high[3],
                          const double cpml[5], const double bloch[3], double courant,
                          const double *eps, char *err, int errlen);
int orc_is_complex(const orc_sim *s);
/* Sets the host threads of the oracle's loops (n > 0); returns the number before. */
int orc_threads(int n);
int orc_get_field_imag(const orc_sim *s, int field, int comp, double *out);
long orc_probe_imag(const orc_sim *s, int p, double *out);
void orc_destroy(orc_sim *s);

int orc_conductivity(orc_sim *s, const double *sigma, char *err, int errlen);
int orc_conductor(orc_sim *s, int comp, long i, long j, long k);
int orc_add_source(orc_sim *s, int field, int comp, long i, long j, long k, const double *wave);
int orc_add_current(orc_sim *s, int field, long count, const int *comps, const long *at,
                    const double *amps, const double *wave);
int orc_add_dipole(orc_sim *s, int field, int comp, const double pos[3], double are, double aim,
                   const double *wave);
int orc_add_probe(orc_sim *s, int field, int comp, long i, long j, long k);
int orc_add_dft(orc_sim *s, const long low[3], const long high[3], int nf, const double *freqs);
/* window = {blo, bhi, clo, chi} along axis.others(), -1 for the whole axis */
int orc_add_flux(orc_sim *s, int axis, long plane, const long window[4], int nf,
                 const double *freqs);
int orc_add_flux_box(orc_sim *s, const long planes[6], int nf, const double *freqs);
/* poles: 4 doubles each {kind (0 Lorentz, 1 Drude), strength|plasma, resonance|damping,
 * damping|unused}; inside: 3 x cells mask of the values it covers. */
int orc_add_medium(orc_sim *s, double eps_inf, int npoles, const double *poles,
                   const unsigned char *inside, int check_stability, char *err, int errlen);

void orc_run(orc_sim *s, long steps);
double orc_dt(const orc_sim *s);
long orc_steps(const orc_sim *s);
void orc_get_field(const orc_sim *s, int field, int comp, double *out);
void orc_set_field(orc_sim *s, int field, int comp, const double *in);
long orc_probe(const orc_sim *s, int p, double *out);
/* Every transform's sums in the order of Monitors::layout (src/fdtd/monitors.rs:849-887):
 * complex interleaved. Returns the number of complex values. */
long orc_transforms(const orc_sim *s, double *out);
int orc_flux(const orc_sim *s, int n, double *out);
/* Setup tables for comparisons: which 0 ca, 1 cb (3 x cells), 2 kappa/h at nodes, 3 at halves
 * (nx+ny+nz), 4 slab table: per slab {field, comp, axis, from, count} then b[count], a[count],
 * 5 media groups: per group {chi, npoles, 3 per pole, count} then {comp, index, scale} per member.
 * Returns the number of doubles (out may be NULL to ask). */
long orc_tables(const orc_sim *s, int which, double *out);
/* Stability of a medium (src/fdtd/media.rs:261-309): 1 stable, 0 not. */
int orc_medium_stable(double eps_inf, int npoles, const double *poles, double sigma, double dt,
                      double top);
/* The STREAM triad a = b + s c over len doubles on all OpenMP threads, the best of `repeats`
 * runs, in GB/s at 24 bytes an element (the reference's traffic::triad, src/traffic.rs:56-80). */
double orc_triad(long len, int repeats);
/* Simulation::add_plane_wave (src/fdtd/sources.rs:716-951): a total-field/scattered-field box
 * from nodes low to high, direction dir (cells), polarization pol, background eps; the wave's
 * number, or -1 (reason in err). orc_incident: its incident field now at a value. */
int orc_add_plane_wave(orc_sim *s, const long low[3], const long high[3], const long dir[3],
                       const double pol[3], double eps, const double *wave, char *err, int errlen);
double orc_incident(const orc_sim *s, int n, int field, int comp, long i, long j, long k);
/* Waveform::spectrum (src/fdtd.rs:361-396) at nf frequencies: out nf complex, interleaved. */
int orc_waveform_spectrum(const double *wave, int field, double dt, long steps, int nf,
                          const double *freqs, double *out);
/* Transform monitor `monitor`'s sum for (field, comp) at grid index at[3], frequency f: out[2]
 * (re, im); 1 if the monitor holds that value, else 0. */
int orc_dft_value(const orc_sim *s, int monitor, int field, int comp, const long at[3], int f,
                  double *out);
/* d(flux of monitor at frequency f)/d(each transform it reads) x scale, as the reference's
 * adjoint takes it (src/fdtd/adjoint.rs:1036-1083): keys[3q] = (field, comp, index), values[2q] the
 * complex derivative. Returns the count (keys null to ask), -1 for no such monitor. */
long orc_flux_derivatives(const orc_sim *s, int monitor, int f, double scale, long *keys,
                          double *values, long capacity);

#ifdef __cplusplus
}
#endif
#endif
