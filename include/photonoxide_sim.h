/*
 * photonoxide_sim.h: the host side of the B200 FDTD engine, photonoxide's `Simulation` API
 * (src/fdtd.rs:469-1590) over the device engine of photonoxide_fdtd.h.
 *
 * It builds what the reference's Simulation builds on the CPU (the cell-averaged permittivity,
 * the time step, the walls, the CPML's tables, conductivity, dispersive media, sources, probes and
 * monitors), then steps on the GPU: the fields go to the device at the first run and stay there,
 * coming back when read. It is the C ABI the Python package binds; a Rust caller keeps its own
 * Simulation and binds photonoxide_fdtd.h instead.
 *
 * Conventions as photonoxide_fdtd.h. Errors: 0 or a negative FDTD_E_* status, the message in
 * pxs_last_error(sim); construction errors in the caller's buffer.
 */
#ifndef PHOTONOXIDE_SIM_H
#define PHOTONOXIDE_SIM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pxs_sim pxs_sim;

/* A box geometry (the value of the reference's eps(x, y, z) closures): boxes of 7 doubles
 * {xlo, xhi, ylo, yhi, zlo, zhi, value}, a point inside when lo < p < hi on each axis, later
 * boxes over earlier ones, `background` elsewhere. */
typedef struct {
  double background;
  int32_t nboxes;
  const double *boxes;
} pxs_geometry;

/* FDFD's cell average (src/fdfd/three.rs:563-588) of a geometry at every value of E (3 x
 * cells); only values whose cell crosses a box's face take the 8^3-sample average. */
int pxs_average(const int64_t n[3], const double d[3], const double o[3], const pxs_geometry *g,
                double *out);
/* The same average on the current CUDA device, one thread per value (the same functions, so the
 * same bits); `out` is host memory. The reference averages on the CPU, sequentially
 * (src/fdtd.rs:583-594). Returns 0, -1 for bad sizes, -2 for a CUDA error. */
int pxs_average_device(const int64_t n[3], const double d[3], const double o[3],
                       const pxs_geometry *g, double *out);
/* The CPML's tables (Simulation::build_cpml, src/fdtd.rs:799-869) on the current CUDA device, one
 * thread per node of each axis, the host library's functions so its bits: which 2 the kappa
 * factors at the nodes over the step (sum of n), 3 at the half-steps, 4 the slabs (per slab its
 * field, component, axis, first node, count, then b and a), as pxs_tables lays them out. Grid,
 * edges and cpml as pxs_create, dt the time step. Returns the count (out NULL: the count alone,
 * no device work), -1 for bad sizes, -2 for a CUDA error. */
int64_t pxs_cpml_device(const int64_t n[3], const double d[3], const int32_t kind[3],
                        const int64_t low[3], const int64_t high[3], const double cpml[5],
                        double dt, int32_t which, double *out);

/* Simulation::new / with_permittivity (src/fdtd.rs:570-796): grid n, d, origin o; kind[a] 0 a
 * CPML of low/high cells (0 = wall), 1 periodic; cpml = {reflection, sigma (NaN: from
 * reflection), order, kappa, alpha}; the per-value permittivity `eps` (3 x cells) or, if NULL,
 * the geometry averaged. precision 32 or 64 on the device. NULL on error, message in err. */
pxs_sim *pxs_create(const int64_t n[3], const double d[3], const double o[3], const int32_t kind[3],
                    const int64_t low[3], const int64_t high[3], const double cpml[5],
                    double courant, const double *eps, const pxs_geometry *geometry,
                    int32_t precision, size_t hbm_budget, char *err, int32_t errlen);
/* The same with Bloch sides (src/fdtd.rs:206-256, src/fdtd/bloch.rs): bloch[a] (rad/um) on a
 * periodic axis (kind 1); one not zero makes the fields complex, the imaginary part a second
 * simulation stepped alongside and coupled across the sides (pxs_is_complex). Its time step
 * counts sin^2(k d / 2) along an axis one cell long. Plane waves and beams are refused in a
 * complex run; batches, the adjoint and the serving loop refuse one. */
pxs_sim *pxs_create_bloch(const int64_t n[3], const double d[3], const double o[3],
                          const int32_t kind[3], const int64_t low[3], const int64_t high[3],
                          const double cpml[5], const double bloch[3], double courant,
                          const double *eps, const pxs_geometry *geometry, int32_t precision,
                          size_t hbm_budget, char *err, int32_t errlen);
/* Whether the fields are complex; their imaginary part (src/fdtd.rs:911-935) and a probe's
 * (probe_complex, src/fdtd.rs:1094-1110). */
int pxs_is_complex(const pxs_sim *s);
int pxs_get_field_imag(pxs_sim *s, int32_t field, int32_t comp, double *out);
int pxs_set_field_imag(pxs_sim *s, int32_t field, int32_t comp, const double *in);
int64_t pxs_probe_imag(pxs_sim *s, int32_t n, double *out);
void pxs_destroy(pxs_sim *s);
const char *pxs_last_error(const pxs_sim *s);

/* Simulation::with_conductivity (src/fdtd.rs:945-992): sampled at each value of E, from a
 * per-value array (3 x cells) or, if NULL, the geometry. */
int pxs_conductivity(pxs_sim *s, const double *sigma, const pxs_geometry *geometry);
/* Simulation::conductor (src/fdtd.rs:995-1008) */
int pxs_conductor(pxs_sim *s, int32_t comp, int64_t i, int64_t j, int64_t k);
/* Simulation::with_medium (src/fdtd/media.rs:741-825): poles of 4 doubles {kind (0 Lorentz,
 * 1 Drude), strength|plasma, resonance|damping, damping|0}; where: a 3 x cells mask, or if
 * NULL the geometry's nonzero places. */
int pxs_medium(pxs_sim *s, double eps_inf, int32_t npoles, const double *poles,
               const uint8_t *inside, const pxs_geometry *geometry);

/* Waveforms as 6 doubles {kind, p1..p5} (photonoxide_fdtd.h's fdtd_waveform). */
int pxs_add_source(pxs_sim *s, int32_t field, int32_t comp, int64_t i, int64_t j, int64_t k,
                   const double wave[6]);
int pxs_add_current(pxs_sim *s, int32_t field, int64_t count, const int32_t *comps,
                    const int64_t *at, const double *amps, const double wave[6]);
int pxs_add_dipole(pxs_sim *s, int32_t field, int32_t comp, const double pos[3], double are,
                   double aim, const double wave[6]);
int pxs_add_probe(pxs_sim *s, int32_t field, int32_t comp, int64_t i, int64_t j, int64_t k);
int pxs_add_dft(pxs_sim *s, const int64_t low[3], const int64_t high[3], int32_t nf,
                const double *freqs);
/* window = {blo, bhi, clo, chi} along axis.others(); -1 for the whole axis */
int pxs_add_flux(pxs_sim *s, int32_t axis, int64_t plane, const int64_t window[4], int32_t nf,
                 const double *freqs);
int pxs_add_flux_box(pxs_sim *s, const int64_t planes[6], int32_t nf, const double *freqs);
/* Simulation::add_plane_wave (src/fdtd/sources.rs:716-951): a total-field/scattered-field box
 * from nodes low to high (inclusive; whole along a periodic axis), the wave going along
 * direction (cells, integers), E along polarization's part across it, the background's eps
 * uniform on the box's surface; its auxiliary 1D run is stepped on the device with the grid.
 * Returns the wave's number, or a negative status. */
int pxs_add_plane_wave(pxs_sim *s, const int64_t low[3], const int64_t high[3],
                       const int64_t direction[3], const double polarization[3], double eps,
                       const double wave[6]);
/* Simulation::add_beam (src/fdtd/sources.rs:598-714): a Gaussian beam launched from the plane of
 * nodes `plane` normal to `axis`, forward (direction >= 0, the total field from the plane on) or
 * back; where its axis crosses the plane (along axis.others()), its waist and the focus's distance
 * ahead, its tilt towards `tilt` by `angle` (radians), E across the tilt's plane (parallel 0) or
 * in it (1), the medium's eps uniform where it enters. The plane's E, decomposed into the grid's
 * own plane waves, becomes currents on the surface, added with the waveform (which needs a
 * carrier). The real functions beyond exp and sin/cos are the C library's (the reference's are
 * the libm crate's), so the currents are within a few ulps of the reference's. */
int pxs_add_beam(pxs_sim *s, int32_t axis, int64_t plane, int32_t direction,
                 const double centre[2], double waist, double focus, int32_t tilt, double angle,
                 int32_t parallel, double eps, const double wave[6]);
/* Simulation::incident (src/fdtd/sources.rs:729-767): plane wave n's incident field now at a
 * value (E at the current time, H half a step behind), into *out; 0 beyond its run. */
int pxs_incident(pxs_sim *s, int32_t n, int32_t field, int32_t comp, int64_t i, int64_t j,
                 int64_t k, double *out);

/* Simulation::run (src/fdtd.rs:1142-1158) on the device. */
int pxs_run(pxs_sim *s, int64_t steps);
double pxs_dt(const pxs_sim *s);
int64_t pxs_steps(const pxs_sim *s);
/* Simulation::time (src/fdtd.rs:887-889): steps x dt */
double pxs_time(const pxs_sim *s);
/* Waveform::spectrum (src/fdtd.rs:361-396): the sum over n < steps of w.at(t_n) e^(i omega t_n)
 * dt, t_n = n dt, plus dt/2 for E (field 0), at each of nf frequencies (c/um), with the
 * reference's exp and sin/cos; out: nf complex, interleaved. waveform = {kind, p[0..4]} as
 * fdtd_waveform. What an FDTD job divides a dipole run's fluxes by (src/job/fdtd.rs:2248-2318). */
int pxs_waveform_spectrum(const double waveform[6], int32_t field, double dt, int64_t steps,
                          int32_t nf, const double *freqs, double *out);
/* Simulation::run_until (src/fdtd.rs:1161-1167) */
int pxs_run_until(pxs_sim *s, double time);
/* Simulation::run_until_decayed (src/fdtd/monitors.rs:742-838): *decayed 1 when the probes'
 * |F|^2 stayed within `fraction` of its peak over a block of `interval`, 0 at `limit`;
 * FDTD_E_GROWING (growing: time, checks, factor) when the fields grow again after the sources. */
int pxs_run_until_decayed(pxs_sim *s, int32_t count, const int32_t *probes, double fraction,
                          double interval, double limit, int32_t *decayed, double *growing);
int pxs_get_field(pxs_sim *s, int32_t field, int32_t comp, double *out);
int pxs_set_field(pxs_sim *s, int32_t field, int32_t comp, const double *in);
/* probe n's values, one per step since it was added; returns the count (out may be NULL) */
int64_t pxs_probe(pxs_sim *s, int32_t n, double *out);
/* every transform's sums (Monitors::layout order), complex interleaved; returns the count */
int64_t pxs_transforms(pxs_sim *s, double *out);
/* Simulation::flux (src/fdtd/monitors.rs:539-552): returns the frequencies' count */
int pxs_flux(pxs_sim *s, int32_t n, double *out);
/* the setup tables, as orc_tables: 0 ca, 1 cb, 2 kappa/h nodes, 3 halves, 4 slabs, 5 media
 * groups (per group chi, npoles, 3 per pole, count, then comp, index, scale per member) */
int64_t pxs_tables(const pxs_sim *s, int32_t which, double *out);
/* The device engine under it (created at the first run), or NULL. */
struct fdtd_ctx *pxs_engine(pxs_sim *s);

/* Batches (photonoxide_batch.h): 2D TE simulations stepped together, one launch per step. Each
 * simulation afterwards reads out as if pxs_run had taken the steps. No counterpart in the
 * reference, whose Simulation runs alone. */
typedef struct pxs_batch pxs_batch;
int pxs_batch_create(int32_t count, pxs_sim *const *sims, pxs_batch **out);
const char *pxs_batch_last_error(const pxs_batch *b);
int pxs_batch_run(pxs_batch *b, int64_t steps);
int pxs_batch_tile(const pxs_batch *b, int32_t *width, int32_t *height);
int pxs_batch_set_tile(pxs_batch *b, int32_t width, int32_t height);
int64_t pxs_batch_launches(const pxs_batch *b);
void pxs_batch_destroy(pxs_batch *b);

/* The dispersive media's size: out[0] E values in a medium, out[1] their poles in total. */
int pxs_media_counts(const pxs_sim *s, int64_t *out);

/* The derivative of pxs_flux(s, n)'s value at frequency f by the real and imaginary parts of
 * every transform sum, times scale, ADDED into grad (pxs_transforms' layout, complex
 * interleaved). No counterpart in the reference, whose adjoint sources come from its own terms
 * (src/fdtd/adjoint.rs:704-734). */
int pxs_flux_gradient(pxs_sim *s, int32_t n, int32_t f, double scale, double *grad);

/* The time-reversed adjoint (photonoxide_adjoint.h) of the next `steps` steps of a 2D TE
 * simulation: pxs_adjoint_forward runs them (the simulation then reads out as after pxs_run),
 * pxs_adjoint_backward gives dJ/dcb at the design values from dJ/dtransforms. */
typedef struct pxs_adjoint pxs_adjoint;
int pxs_adjoint_create(pxs_sim *s, int64_t steps, int32_t segment, int64_t count,
                       const int32_t *component, const int64_t *r, pxs_adjoint **out);
const char *pxs_adjoint_last_error(const pxs_adjoint *a);
int pxs_adjoint_forward(pxs_adjoint *a);
int pxs_adjoint_backward(pxs_adjoint *a, const double *grad_sums, double *grad_cb);
void pxs_adjoint_destroy(pxs_adjoint *a);

/* Serving: a resident loop (its own thread) that admits submitted simulations in arrival order
 * while its slots (max_active) and device-memory budget (an estimate per job) allow, keeps them on
 * the device and steps them together `chunk` steps at a time -- the 2D TE ones in one batch, the
 * others each on its own stream, concurrently. A finished job's fields, probes and transforms are
 * read back to its simulation and its device memory freed. A submitted simulation belongs to the
 * server until its job ends: the caller must not use it meanwhile. No counterpart in the reference.
 * Job states: 0 queued, 1 running, 2 done, 3 failed, 4 cancelled. */
typedef struct pxs_server pxs_server;
int pxs_server_create(size_t hbm_budget, int32_t max_active, int64_t chunk, pxs_server **out);
const char *pxs_server_last_error(const pxs_server *sv);
/* returns the job's id (> 0) or a negative status. keep_fields 0: when the job ends only its
 * transforms, fluxes and probes come back (the fields are dropped with the device memory;
 * reading them or running the simulation again then refuses with FDTD_E_STATE). */
int64_t pxs_server_submit(pxs_server *sv, pxs_sim *s, int64_t steps, int32_t keep_fields);
/* the job's state; times (may be NULL): submitted, started, finished (steady clock, seconds) */
int pxs_server_poll(pxs_server *sv, int64_t id, double *times);
int pxs_server_wait(pxs_server *sv, int64_t id);
int pxs_server_cancel(pxs_server *sv, int64_t id);
/* out[0] cell-updates taken, out[1] rounds stepped, out[2] device bytes admitted now, out[3..5]
 * the loop's seconds queuing work, setting up and reading back jobs, waiting for the device */
int pxs_server_stats(pxs_server *sv, double *out);
/* stops the loop (between chunks) and frees the server; jobs still running are left released or
 * not as the loop left them */
void pxs_server_destroy(pxs_server *sv);

#ifdef __cplusplus
}
#endif
#endif
