/* lmm_ensemble.h - ensembles of independent Stokes solves (no counterpart in
 * the reference, which solves one problem per time step).
 *
 * lmm_ensemble_solve solves `count` independent problems of the same
 * dimension and knobs but with their own grid sizes, spacing, coefficients
 * and right-hand sides, concurrently on one device: `workers` host threads
 * each own a solver handle per grid shape (own CUDA stream) and take the
 * instances largest first.  Every array is a device array in the compact
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

#ifdef __cplusplus
}
#endif

#endif /* LMM_ENSEMBLE_H */
