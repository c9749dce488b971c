/*
 * photonoxide_fdtd.h: the C ABI of the B200 FDTD engine.
 *
 * This is the drop-in seam for photonoxide's GPU device: every entry point here replaces one
 * step of the reference's `gpu::Resident` (src/fdtd/gpu/resident.rs), which `Simulation` drives
 * through its `OnGpu` slot (src/fdtd.rs:528-535, run/step diverting at src/fdtd.rs:1142-1146,
 * 1319-1323). A Rust shim binds these as `extern "C"`; the Python package and the C++ host
 * library in this repository call them the same way.
 *
 * Conventions (the reference's): field 0 = E, 1 = H (H~ = eta0 H); component/axis 0, 1, 2 =
 * x, y, z; within a component the value (i, j, k) is at r = (k*ny + j)*nx + i
 * (src/fdfd/three.rs:123-125); a field's three components are stored one after the other.
 * Host arrays are f64 (the reference's); the device rounds them to its precision.
 *
 * Every entry point returns 0 or a negative status (FDTD_E_*), and never aborts: the message
 * of the last failure is fdtd_last_error(ctx). Invalid values are the reference's
 * Error::InvalidValue (src/error.rs:15-22); device failures, out-of-memory and a problem beyond
 * the HBM budget are its Error::Gpu (src/error.rs:49).
 */
#ifndef PHOTONOXIDE_FDTD_H
#define PHOTONOXIDE_FDTD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FDTD_OK 0
#define FDTD_E_INVALID (-1) /* a value the engine refuses (Error::InvalidValue) */
#define FDTD_E_GPU (-2)     /* a CUDA failure or out of device memory (Error::Gpu) */
#define FDTD_E_BUDGET (-3)  /* the problem needs more HBM than the context's budget */
#define FDTD_E_STATE (-4)   /* a call out of order (e.g. a run before the fields are there) */
#define FDTD_E_TIMEOUT (-5) /* a device-side wait gave up (persistent/served kernels) */
#define FDTD_E_GROWING (-6) /* the fields grew again after the sources ended (Error::Growing) */

typedef struct fdtd_ctx fdtd_ctx;

/* The grid and what is beyond its sides: Resident::new's params (resident.rs:466-495). */
typedef struct {
  int64_t n[3];        /* cells along x, y, z */
  int32_t periodic[3]; /* 1 where an axis wraps (Edges::Bloch { k: 0 }) */
  int64_t low[3];      /* CPML cells at each axis's low end (0: a wall) */
  int64_t high[3];     /* and at its high end */
} fdtd_grid;

/* One CPML slab: kernel::Slab (src/fdtd/kernel.rs:376-392), its recursion's coefficients in
 * f64, `count` of each, built as Simulation::build_cpml does (src/fdtd.rs:799-869). */
typedef struct {
  int32_t field, component, axis;
  int64_t from, count;
  const double *b;
  const double *a;
} fdtd_slab;

/* A source or current value, in the order a CPU step adds them (src/fdtd.rs:1348-1387): the
 * waveform of `emitter` taken at the field's time (M at t, J at t + dt/2), Re(a w) added as
 * H -= dt Re(a w) or E -= cb Re(a w). A point source has a = 1 and takes w.at(t). point 2: a
 * coupling of a plane wave's box (PlaneWaveRun::correct, src/fdtd/sources.rs:971-991), its
 * coefficient a_re (dt weight for H, cb weight for E) times the incident value in slot `emitter`
 * of fdtd_set_plane_waves, subtracted as it is (H -= a_re h_inc). */
typedef struct {
  int32_t field, component;
  int64_t r;
  double a_re, a_im;
  int32_t emitter;
  int32_t point;
} fdtd_injection;

/* A waveform (src/fdtd.rs:259-424): kind 0 Gaussian {frequency c/um, width, delay}; 1
 * differentiated Gaussian {width, delay}; 2 continuous {frequency, amplitude re, im, ramp}.
 * The device evaluates it in f64 at each step. */
typedef struct {
  int32_t kind;
  double p[5];
} fdtd_waveform;

/* One transformed series (src/fdtd/monitors.rs:45-82): a component's box, its sums kept
 * frequency by frequency, then k, j, i with i fastest, at its monitor's frequencies. */
typedef struct {
  int32_t field, component;
  int64_t lo[3], len[3];
  int32_t monitor;
} fdtd_series;

/* One dispersive medium's values (src/fdtd/media.rs:559-615): their components and indices,
 * p_m at each (the curl's scale there), chi, and each pole's (alpha, xi, gamma). */
typedef struct {
  int64_t count;
  const int32_t *component;
  const int64_t *r;
  const double *scale;
  double chi;
  int32_t npoles;
  const double *poles; /* 3 per pole */
} fdtd_media_group;

/* Resident::new (resident.rs:154-293): allocates the fields (two copies, the step reading one
 * and writing the other), coefficients and CPML state on the current CUDA device, refusing a
 * problem beyond `hbm_budget` bytes (0: no budget). `dt` and `step` (dx, dy, dz) in um/c and um;
 * `factor_e`/`factor_h`: kappa/h per index along x, then y, then z, at the nodes (E's back
 * differences) and halfway after them (H's forward ones) (Simulation::build_stencils,
 * src/fdtd.rs:1552-1569). precision 32 (f32, the product) or 64 (f64, for checking). */
int fdtd_create(const fdtd_grid *grid, double dt, const double step[3], const double *factor_e,
                const double *factor_h, const fdtd_slab *slabs, int32_t nslabs, int32_t precision,
                size_t hbm_budget, fdtd_ctx **out);
void fdtd_destroy(fdtd_ctx *ctx);
const char *fdtd_last_error(const fdtd_ctx *ctx);

/* Resident::upload (resident.rs:378-399): E's coefficients. ca may be NULL for a medium with no
 * conductivity (ca 1 wherever cb isn't 0, and 0 where it is), which the step then never reads. */
int fdtd_upload_coeffs(fdtd_ctx *ctx, const double *ca, const double *cb);
/* The fields (3 x cells each) and each slab's psi (in slab order; NULL entries mean zero).
 * Host arrays that are page-locked and mapped (cudaHostAlloc'd or registered) are read by the
 * device directly, converted to the context's precision as they cross; pageable ones go through
 * a staging buffer the context allocates on its first such transfer (within its HBM budget) and
 * keeps. The same holds for fdtd_upload_coeffs, fdtd_download_fields and fdtd_read_dft. Every
 * one of these calls returns with its host arrays free for the caller to reuse. */
int fdtd_upload_fields(fdtd_ctx *ctx, const double *e, const double *h, const double *const *psi);
/* fdtd_upload_fields(ctx, e, h, NULL) without allocating any device memory, for callers that
 * can't allocate at that point: a serving loop that has handed out its whole HBM budget, an
 * application whose CUDA allocator is its own, code that must leave a stream-ordered memory pool
 * untouched. No counterpart in the reference (its uploads go through wgpu's staging buffers).
 * An f32 context's f64 host values pass through a fixed 16 MiB device array of the library
 * (2^21 values, held by every GPU that loads it until exit), one field component at a time, so
 * an f32 grid of more than 2^21 cells is refused (FDTD_E_INVALID; use fdtd_upload_fields); an
 * f64 context copies straight into its fields, any size. psi restarts from zero. The first f32
 * call on a device looks the array up (call it before any stream capture); calls that overlap on
 * the GPU share the array and race. */
int fdtd_upload_fields_static(fdtd_ctx *ctx, const double *e, const double *h);

/* Which axes' CPML differences are divided by the grid step through a reciprocal product with
 * one correction (out[axis] = 1) rather than a division: in f32 the engine compares that form
 * with division for every finite float at creation and uses it only where every result is the
 * same bits. No counterpart in the reference (its WGSL divides). */
int fdtd_fast_division(const fdtd_ctx *ctx, int32_t out[3]);
/* Resident::download (resident.rs:402-413). Any pointer may be NULL to skip it. */
int fdtd_download_fields(fdtd_ctx *ctx, double *e, double *h, double *const *psi);

/* The run's sources and currents (Resident::plan's injection groups, resident.rs:546-590). */
int fdtd_set_sources(fdtd_ctx *ctx, int32_t nwaves, const fdtd_waveform *waves, int64_t ninj,
                     const fdtd_injection *inj);
/* A plane wave's auxiliary 1D run (PlaneWaveRun, src/fdtd/sources.rs:755-1041), stepped on the
 * device with the grid: len samples, the first and last pad never updated; the direction g
 * (cells) and the grid's steps for its differences; per sample E <- ca E + cb curl and H <- da H -
 * db curl; the sheet's J (component, sample, J per unit waveform) with E's waveform at t + dt/2.
 * Each step records the slots the box's couplings read: field 0, E's `comp` at sample i before
 * the H step (for H's couplings), field 1, H after it (for E's). e0 and h0 (3 x len, component
 * by component) its state now, or NULL for zeros. */
typedef struct {
  int64_t len, pad;
  int64_t g[3];
  double steps[3];
  const double *ca, *cb, *da, *db;
  int32_t nsheet;
  const int32_t *sheet_comp;
  const int64_t *sheet_i;
  const double *sheet_j;
  fdtd_waveform wave;
  int32_t nslots;
  const int32_t *slot_field, *slot_comp;
  const int64_t *slot_i;
  const double *e0, *h0;
} fdtd_plane_wave;
/* The plane waves' runs (their slots numbered on from one wave to the next, as point-2
 * injections name them). Call before fdtd_set_sources, which lays out the step's values for
 * them; no counterpart in the reference's GPU path, which refuses plane waves (gpu.rs:431). */
int fdtd_set_plane_waves(fdtd_ctx *ctx, int32_t count, const fdtd_plane_wave *waves);
/* Plane wave n's auxiliary state now: E and H, 3 x len each (either may be NULL). */
int fdtd_plane_wave_state(fdtd_ctx *ctx, int32_t n, double *e, double *h);
/* A coupling across a Bloch side (Bloch::wrap, src/fdtd/bloch.rs:97-152) of a complex run: after
 * `field`'s update, value r of component `comp` gets (e^(+-ikL) - 1) F s, F = (real, imaginary)
 * of component `from_comp` at q across the side (both parts' E before the step for H, field 1;
 * their new H for E, field 0); phase = e^(ikL) - 1 for H and e^(-ikL) - 1 for E; s = its sign
 * times kappa / step. H's: dt times it subtracted in the step as the point-2 injection of Bloch
 * slot `slot` (after the plane waves' slots); E's: cb times it added. */
typedef struct {
  int32_t field, comp, from_comp, slot;
  int64_t r, q;
  double phase_re, phase_im, s, cb;
} fdtd_wrap;
/* The Bloch slots a context's point-2 injections may name after its plane waves'; call before
 * fdtd_set_sources. */
int fdtd_set_bloch_slots(fdtd_ctx *ctx, int32_t nslots);
/* A complex run's steps (src/fdtd.rs:1319-1343): `re` and `im` hold the fields' real and
 * imaginary parts (the same grid, coefficients and media; im with the currents' imaginary
 * amplitudes and the same probes); both step together with the couplings, re's transforms
 * taking both parts. No counterpart in the reference's GPU path, which refuses Bloch phases
 * (gpu.rs:427). */
int fdtd_bloch_run(fdtd_ctx *re, fdtd_ctx *im, int32_t nwraps, const fdtd_wrap *wraps,
                   int64_t steps, int64_t first_step);
/* The probes: field, component and index of each value recorded after every step. */
int fdtd_set_probes(fdtd_ctx *ctx, int32_t n, const int32_t *field, const int32_t *component,
                    const int64_t *r);
/* The transforms (Monitors::layout order, monitors.rs:849-860): every series, and each
 * monitor's frequencies (c/um; freqs_per_monitor[m] of them, concatenated). */
int fdtd_set_dft(fdtd_ctx *ctx, int32_t nseries, const fdtd_series *series, int32_t nmonitors,
                 const int32_t *freqs_per_monitor, const double *freqs);
/* The dispersive media (Media, media.rs:592-705), stepped with E in the same pass. */
int fdtd_set_media(fdtd_ctx *ctx, int32_t ngroups, const fdtd_media_group *groups);

/* `steps` steps from step number `first_step` (the simulation's steps so far, which fixes the
 * sources' and transforms' times), as Resident::step (resident.rs:430-539). Returns when the
 * device is done. */
int fdtd_run(fdtd_ctx *ctx, int64_t steps, int64_t first_step);
/* The same, enqueued on the context's stream without waiting (for timing and overlap). */
int fdtd_run_async(fdtd_ctx *ctx, int64_t steps, int64_t first_step);
int fdtd_synchronize(fdtd_ctx *ctx);

/* The probes' values recorded since the last read, step by step (steps x probes), and their
 * count of steps in *steps (out may be NULL to ask). Reading clears them. */
int fdtd_read_probes(fdtd_ctx *ctx, double *out, int64_t capacity, int64_t *steps);
/* The transforms' sums taken since the last read, ADDED into `sums` (complex interleaved, in
 * layout order) as Monitors::add does (monitors.rs:866-887); the device's sums then restart
 * from zero. */
int fdtd_read_dft(fdtd_ctx *ctx, double *sums, int64_t count);

/* The device's copies, for callers that keep their data on the device. Returned pointers are
 * device addresses (CUDA), valid until the next fdtd_run or fdtd_destroy. */
int fdtd_device_fields(fdtd_ctx *ctx, void **e, void **h);
/* The CUDA stream the context enqueues on (a cudaStream_t). */
void *fdtd_stream(fdtd_ctx *ctx);
/* The kernels the last run launched, for accounting. */
int64_t fdtd_launches(const fdtd_ctx *ctx);
/* With `on`, each launch of the step kernel is bracketed by CUDA events on the context's stream;
 * fdtd_profile_read gives their summed device time (ms) and count since profiling started. */
int fdtd_profile(fdtd_ctx *ctx, int32_t on);
int fdtd_profile_read(fdtd_ctx *ctx, double *ms, int64_t *launches);

#ifdef __cplusplus
}
#endif
#endif
