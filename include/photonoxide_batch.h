/* Batched 2D TE stepping: several simulations' grids advanced together by one launch per step.
 *
 * The reference has no counterpart: its GPU seam (src/fdtd/gpu/resident.rs) steps one
 * simulation. Each simulation here is an engine context (photonoxide_fdtd.h) that its caller has
 * set up as for fdtd_run: created, coefficients and fields uploaded, sources, probes and
 * transforms set. The batch steps the contexts' buffers in place; afterwards each context reads
 * out (fdtd_download_fields, fdtd_read_dft, fdtd_read_probes) exactly as if fdtd_run had taken
 * the same steps, with the same bits.
 *
 * Each grid must be 2D (n[2] == 1, periodic along z) with only TE fields (E_x, E_y, H_z; H_x,
 * H_y and E_z zero), sources on E_x, E_y or H_z, no dispersive media, and all in one precision.
 * Errors: the same codes as photonoxide_fdtd.h; the text from fdtd_batch_last_error.
 */
#ifndef PHOTONOXIDE_BATCH_H
#define PHOTONOXIDE_BATCH_H

#include <stdint.h>

#include "photonoxide_fdtd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fdtd_batch fdtd_batch;

/* A batch over `count` contexts, which it does not own (destroy it before them). */
int fdtd_batch_create(int32_t count, fdtd_ctx *const *ctxs, fdtd_batch **out);
const char *fdtd_batch_last_error(const fdtd_batch *batch);
/* `steps` steps of every grid; grid i's first step has index first_steps[i] (its step count so
 * far, as fdtd_run's first_step), all 0 when first_steps is NULL. The first run of a batch whose
 * tile shape is not set times each shape on chunks of these steps and keeps the fastest. Returns
 * once the steps are queued: each context's stream waits for them, so its later calls (reads,
 * runs, fdtd_synchronize) come after. */
int fdtd_batch_run(fdtd_batch *batch, int64_t steps, const int64_t *first_steps);
/* The tile shape in use (0 x 0 before the first run chooses one). */
int fdtd_batch_tile(const fdtd_batch *batch, int32_t *width, int32_t *height);
/* Fixes the tile shape (one of 32x8, 32x16, 64x4, 64x8, 128x2, 128x4, or 124x7: a warp per row
 * of 124 places, four a lane), or 0 x 0: choose by timing on the next run of at least 480
 * steps (shorter first runs take 64x8). */
int fdtd_batch_set_tile(fdtd_batch *batch, int32_t width, int32_t height);
/* Kernel launches the batch has made (graph replays count their kernels). */
int64_t fdtd_batch_launches(const fdtd_batch *batch);
void fdtd_batch_destroy(fdtd_batch *batch);

#ifdef __cplusplus
}
#endif

#endif
