/* lmm_ensemble.h - ensembles of independent Stokes solves (no counterpart in
 * the reference, which solves one problem per time step).
 *
 * lmm_ensemble_solve solves `count` independent problems of the same
 * dimension and knobs but with their own grid sizes, spacing, coefficients
 * and right-hand sides, concurrently on one device.  2D problems whose knobs
 * batch (see lmm_stokes_create_batch; knobs->ensemble_batch = 0) are solved
 * in batches, one batch handle per (grid, dx, theta_alpha) and host thread
 * per batch handle; otherwise `workers` host threads
 * each own a solver handle per grid shape (own CUDA stream) and take the
 * instances largest first.  Either way each instance's result has the bits
 * of its own lmm_stokes_solve_device call.  Every array is a device array in the compact
 * layout (lmm_fields_in / lmm_fields_out), already written when the call
 * starts.  Per instance: status (as lmm_stokes_solve) and stats.  Returns
 * the most negative instance status, or LMM_OK.  Several GPUs: call it once
 * per device with that device's share of the instances.  Four workers with
 * spinning host waits (knobs->host_wait = 0) measured fastest on B200 for
 * 2D grids of 32^2..256^2; blocking waits and more workers were slower. */
#ifndef LMM_ENSEMBLE_H
#define LMM_ENSEMBLE_H

#include "lmm_stokes.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lmm_ensemble_item {
    int n[3];                      /* cells per direction (n[2] ignored in 2D) */
    double dx;
    double theta_alpha;
    const double* b_u[3];
    const double* b_p;
    const double* alpha_fc[3];
    const double* beta;
    const double* beta_ed[3];
    const double* gamma;
    double* x_u[3];                /* initial guess in, solution out */
    double* x_p;
    int status;                    /* out */
    lmm_stats stats;               /* out */
} lmm_ensemble_item;

int lmm_ensemble_solve(int dm, const lmm_knobs* knobs, int device, lmm_ensemble_item* items, int count, int workers);

/* The same with the worker pool kept between calls: create makes every
 * handle (one per worker and distinct (n, dx) of `shapes`, which only needs
 * n and dx filled) before any solve -- creation and destruction allocate and
 * free memory, which must not overlap a worker's graph capture -- and run
 * solves items whose shapes are among them. */
typedef struct lmm_ensemble lmm_ensemble;
int lmm_ensemble_create(int dm, const lmm_knobs* knobs, int device, const lmm_ensemble_item* shapes, int nshapes,
                        int workers, lmm_ensemble** out);
int lmm_ensemble_run(lmm_ensemble* ens, lmm_ensemble_item* items, int count);
int lmm_ensemble_destroy(lmm_ensemble* ens);

/* Batches of 2D problems on one grid.  lmm_stokes_create_batch makes a
 * handle for up to `batch` periodic 2D problems of grid g (n, dx), stacked
 * along a third index of its device arrays; lmm_stokes_solve_batch solves
 * count <= batch of them together.  Every kernel launch and captured
 * preconditioner graph covers the whole batch, while FGMRES keeps a
 * Hessenberg matrix, stopping test and statistics per problem, so each
 * problem gets the iterations, solution and stats (the same bits) of its
 * own lmm_stokes_solve_device call on a one-problem handle with the same
 * knobs.  The items' arrays are device arrays in the compact layout; all
 * items share theta_alpha and the gamma / no-gamma choice; solve_ms is the
 * batch's time.  Knobs: LMM_METHOD_FGMRES (FP32 or FP64 preconditioner),
 * visc_type < 0, stag_mg_max_vcycles <= 1,
 * scale_factor 1, gmres_max_inner <= 45, no BFBt or learned stage; grids
 * periodic or with walls (as lmm_stokes_create; the edge arrays then keep
 * n+1 nodes along a nodal wall-bounded direction), at most 2^29 cells per
 * batch.  lmm_ensemble_* batches periodic grids.  A batch handle is accepted by these two calls,
 * lmm_stokes_update_knobs (stopping rules between solves), lmm_time_op and
 * lmm_stokes_destroy only.  Returns the most negative
 * problem status, else the largest warning, else LMM_OK; per item status
 * and stats.  lmm_ensemble_* uses batches for 2D problems whose knobs
 * allow it (knobs->ensemble_batch = 0). */
int lmm_stokes_create_batch(const lmm_grid* g, const lmm_knobs* k, int batch, int device, lmm_handle** h);
int lmm_stokes_solve_batch(lmm_handle* h, lmm_ensemble_item* items, int count);

#ifdef __cplusplus
}
#endif

#endif /* LMM_ENSEMBLE_H */
