/* The time-reversed adjoint of a 2D TE simulation's run: the gradient of a function J of its
 * transform sums with respect to cb (= dt / eps) at chosen E values.
 *
 * The reference's adjoint (src/fdtd/adjoint.rs:366-569) is in the frequency domain: a second
 * forward run with adjoint sources, then dF/deps from both runs' transforms. This one is the
 * discrete adjoint of the time stepping itself (reverse mode through every step, CPMLs
 * included), so it is the exact derivative of the engine's own J: the forward run keeps a
 * checkpoint of the fields every `segment` steps; the reverse run recomputes each segment from its
 * checkpoint and steps the adjoint fields back through it.
 *
 * The simulation is an engine context set up as for fdtd_run (photonoxide_fdtd.h), 2D TE as
 * photonoxide_batch.h requires. The design's values must be E_x or E_y values clear of the CPMLs
 * and of electric sources. Errors: the codes of photonoxide_fdtd.h.
 */
#ifndef PHOTONOXIDE_ADJOINT_H
#define PHOTONOXIDE_ADJOINT_H

#include <stdint.h>

#include "photonoxide_fdtd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fdtd_adjoint fdtd_adjoint;

/* An adjoint over `steps` steps of ctx from its state at the forward run, checkpoints every
 * `segment` steps (rounded up to even), the gradient at `count` values: component[d] (0 E_x, 1
 * E_y) at index r[d] (Grid3d::index). Device memory: one checkpoint of (E_x, E_y, H_z, psi) per
 * segment, the adjoint fields, and segment x count curls. */
int fdtd_adjoint_create(fdtd_ctx *ctx, int64_t steps, int32_t segment, int64_t count,
                        const int32_t *component, const int64_t *r, fdtd_adjoint **out);
const char *fdtd_adjoint_last_error(const fdtd_adjoint *adjoint);
/* The forward run: `steps` steps from step index first_step (as fdtd_run); afterwards the
 * context reads out as after fdtd_run. */
int fdtd_adjoint_forward(fdtd_adjoint *adjoint, int64_t first_step);
/* The reverse run. grad_sums: dJ/dRe and dJ/dIm of each transform sum, interleaved, in the
 * layout of fdtd_read_dft. grad_cb (count values): dJ/dcb at the design values. The context is
 * left as the forward run left it. */
int fdtd_adjoint_backward(fdtd_adjoint *adjoint, const double *grad_sums, double *grad_cb);
void fdtd_adjoint_destroy(fdtd_adjoint *adjoint);

#ifdef __cplusplus
}
#endif

#endif
