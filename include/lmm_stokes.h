/*
 * lmm_stokes.h - C ABI of liblmmstokes, a B200-native replacement for the
 * variable-coefficient staggered-grid Stokes solve of LowMachMixtures.
 *
 * The reference entry point this library stands behind is the Fortran
 * subroutine
 *
 *   gmres(mla, the_bc_tower, dx, b_u, b_p, x_u, x_p,
 *         alpha_fc, beta, beta_ed, gamma, theta_alpha, norm_pre_rhs)
 *
 * in src_gmres/gmres.f90:30-45, configured by the probin_gmres module
 * globals (src_gmres/probin_gmres.f90:13-22) and by visc_type
 * (src_common/probin_common.f90:94-100).  The Fortran side binds these
 * functions with iso_c_binding; every pointer is a plain host or device
 * address and every size a plain integer.
 *
 * Conventions
 *  - Grid: one box, isotropic dx, dm = 2 or 3; each direction is periodic
 *    or bounded by walls on both sides (no-slip or slip, lmm_grid.bc_lo /
 *    bc_hi, the reference's bc_lo / bc_hi of src_common/bc.f90:23-44).
 *  - Face component d of a velocity-like field is nodal in direction d.
 *  - LMM_LAYOUT_COMPACT arrays hold the n[0]*n[1](*n[2]) unique periodic
 *    entries of a field, i fastest (Fortran column-major order), without
 *    ghost cells; the duplicated periodic seam face (index hi+1) is implied
 *    equal to face lo.  Along a wall-bounded direction d: face component d
 *    stores faces lo..hi, face lo being the wall (taken as zero in b_u and
 *    x_u: the wall-normal velocity is not an unknown) and the wall face hi+1
 *    implied zero; a beta_ed array nodal in d stores its n[d]+1 nodes (both
 *    walls), so it holds prod(n + wall-nodal) entries.
 *  - LMM_LAYOUT_BOXLIB arrays are the Fortran arrays exactly as BoxLib's
 *    dataptr() hands them over for a single box: column-major, ng ghost
 *    layers on every side, and n+1 valid entries in each nodal direction.
 *  - Return codes: 0 = converged, >0 = warning, <0 = error (lmm_strerror).
 *  - A handle is not thread-safe; use one handle per host thread.
 */
#ifndef LMM_STOKES_H
#define LMM_STOKES_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (gmres.f90:254-296,376-378; apply_precon.f90:425-426) --- */
#define LMM_OK                 0
#define LMM_WARN_MAX_ITER      1  /* total_iter reached gmres_max_iter (gmres.f90:254-260) */
#define LMM_WARN_MAX_OUTER     2  /* iter reached gmres_max_outer (gmres.f90:291-296) */
#define LMM_WARN_RESID_MISMATCH 3 /* true residual disagrees with preconditioned one (gmres.f90:272-275) */
#define LMM_ERR_INVALID       -1  /* bad argument / unsupported combination (bl_error sites) */
#define LMM_ERR_BREAKDOWN     -2  /* H(i+1,i) == 0 (gmres.f90:376-378) */
#define LMM_ERR_NONFINITE     -3  /* NaN/Inf in an input or a residual */
#define LMM_ERR_CUDA          -4  /* CUDA runtime error */
#define LMM_ERR_WATCHDOG      -5  /* a bounded device wait gave up */
#define LMM_ERR_NO_DEVICE     -6  /* no CUDA device visible */
#define LMM_ERR_BOUNDS        -8  /* builds with -DLMM_BOUNDS_CHECK only: a load outside the handle's
                                     allocations was skipped (lmm_strerror gives the first address) */

/* ---- boundary-condition codes (src_common/bc.f90:23-44) ---- */
#define LMM_BC_PERIODIC       -1
#define LMM_BC_NO_SLIP_WALL  100  /* 100-103 (NO_SLIP_START..NO_SLIP_END): zero velocity */
#define LMM_BC_SLIP_WALL     200  /* 200-203 (SLIP_START..SLIP_END): zero normal velocity and shear stress */

/* ---- array layouts ---- */
#define LMM_LAYOUT_COMPACT     0
#define LMM_LAYOUT_BOXLIB      1

/* ---- outer Krylov method ---- */
#define LMM_METHOD_GMRES       0  /* the reference algorithm: restarted left-preconditioned
                                     GMRES(m), MGS Arnoldi, stop on the preconditioned
                                     residual (gmres.f90:30-605) */
#define LMM_METHOD_FGMRES      1  /* right-preconditioned flexible GMRES(m), FP64 Arnoldi,
                                     stop on the true residual |b-Ax|/|b| (new) */

/* ---- preconditioner arithmetic ---- */
#define LMM_PRECISION_FP64     0  /* V-cycles in FP64 (reference arithmetic) */
#define LMM_PRECISION_FP32     1  /* V-cycles in FP32 (FGMRES only) */

typedef struct lmm_grid {
    int    dm;          /* 2 or 3 */
    int    n[3];        /* cells per direction (n[2] ignored when dm == 2) */
    double dx;          /* isotropic spacing; stag_applyop.f90:116-118 requires dx(1)==dx(2) */
    int    bc_lo[3];    /* BC codes per side: LMM_BC_PERIODIC on both sides of a
                           direction, or a wall code (100-103 no-slip, 200-203
                           slip) on both.  Walls follow define_bc_tower.f90:219-234
                           and multifab_physbc_stag.f90 for the homogeneous
                           problem gmres(...) solves: normal velocity zero,
                           transverse ghost -interior (no-slip) or +interior
                           (slip), pressure extrapolated (zero wall gradient,
                           div_and_grad.f90:139-182), pressure multigrid with
                           homogeneous Neumann faces.  Not with
                           visc_schur_approx = 1 or the learned stage. */
    int    bc_hi[3];
} lmm_grid;

/* Mirror of module probin_gmres_module (probin_gmres.f90:13-22, defaults
 * :119-157) plus visc_type (probin_common.f90:94-100).  lmm_default_knobs()
 * fills the reference defaults. */
typedef struct lmm_knobs {
    int    precon_type;            /* +-1 projection, +-2 lower triangular, +-3 upper, +-4 diagonal, +-5 */
    int    visc_schur_approx;      /* 0 local viscosity, 1 BFBt (apply_precon.f90:538-685; periodic box) */
    double p_norm_weight;
    double scale_factor;
    /* pressure (cell-centred) multigrid */
    int    mg_verbose, cg_verbose, mg_max_vcycles, mg_minwidth, mg_bottom_solver;
    int    mg_nsmooths_down, mg_nsmooths_up, mg_nsmooths_bottom, mg_max_bottom_nlevels;
    double mg_rel_tol;
    /* staggered (velocity) multigrid */
    int    stag_mg_verbosity, stag_mg_max_vcycles, stag_mg_minwidth, stag_mg_bottom_solver;
    int    stag_mg_nsmooths_down, stag_mg_nsmooths_up, stag_mg_nsmooths_bottom;
    int    stag_mg_max_bottom_nlevels;
    double stag_mg_omega;
    int    stag_mg_smoother;       /* 0 weighted Jacobi, 1 2*dm-colour Gauss-Seidel */
    double stag_mg_rel_tol;
    /* GMRES */
    double gmres_rel_tol, gmres_abs_tol;
    int    gmres_verbose, gmres_max_outer, gmres_max_inner, gmres_max_iter, gmres_min_iter;
    /* probin_common */
    int    visc_type;              /* +-1, +-2, +-3 */
    /* additions of this library */
    int    method;                 /* LMM_METHOD_* */
    int    precision;              /* LMM_PRECISION_* */
    int    learned_stage;          /* 3D FGMRES with the FP32 preconditioner and a network attached
                                      by lmm_stokes_set_net: 0 off; 1 the network's correction of
                                      each V-cycle application's residual is an extra FGMRES
                                      direction; 2 the same corrections computed and not used (the
                                      stage's cost alone); 3 the correction added to the V-cycle's
                                      direction when it lowers the residual; 4 as 1, judged by the
                                      GMRES residual: after two network columns that lower its
                                      estimate by less than 10% the solve goes on with the V-cycle
                                      alone */
    int    tail_cells;             /* coarse multigrid levels with at most this many cells run in
                                      one single-block launch; 0 = default (512 for the velocity
                                      V-cycle, 1024 for one 2D problem, 4096 for the pressure
                                      V-cycle), -1 = never */
    int    tail_smem_kb;           /* shared-memory budget of that launch in KiB; 0 = 200 */
    int    use_graphs;             /* replay each preconditioner application from a captured
                                      CUDA graph: 0 = default (on), -1 = off */
    int    smoother_fusion;        /* Gauss-Seidel on 3D levels: 0 = one launch per colour (default),
                                      1 = both colours of a component in one out-of-place launch
                                      where the level allows it, k > 1 = the same with k planes
                                      per block */
    int    l2_persist;             /* FP32 preconditioner: 1 = keep the finest level's coefficients
                                      resident in L2 (access-policy window, when they fit);
                                      0 = default (off: the carve-out costs the Krylov kernels more
                                      than the V-cycle gains at 128^3) */
    int    orthogonalization;      /* FGMRES: 0 = modified Gram-Schmidt (the reference's), 1 =
                                      classical Gram-Schmidt, all projections in one pass */
    int    host_wait;              /* 0 = the host spins on the stream when it reads a scalar (lowest
                                      latency), 1 = it blocks (many host threads driving solvers) */
    int    ensemble_batch;         /* lmm_ensemble_*: 0 = 2D problems whose knobs allow it are solved
                                      in batches (lmm_stokes_create_batch), -1 = always the worker
                                      pool of one-problem handles; a solver handle ignores it */
    int    smoother_tma;           /* 3D Gauss-Seidel (smoother_fusion = 0): 1 = both colours of a
                                      component in one launch with its operands staged in shared
                                      memory by TMA, on the periodic levels that allow it with at least
                                      smoother_tma_cells cells (k >= 2: k rows of faces per tile);
                                      0 = default (off: one launch per colour), -1 = off */
    int    smoother_tma_slabs;     /* k-slabs of that launch; 0 = about one CTA per SM */
    int    smoother_tma_cells;     /* smallest level (cells) that uses it; 0 = default (32^3) */
    int    smoother_order;         /* Gauss-Seidel with one launch per colour: 0 = default (consecutive
                                      launches take the planes in alternating order, each starting
                                      where the last left its operands in L2), -1 = always in +k order */
    int    autotune;               /* 0 = default (the first handle of a grid size times candidate block
                                      shapes of the colour, operator, residual and prolongation kernels
                                      and of apply_matrix, and the process keeps the fastest; see lmm_autotune_report), -1 = this
                                      handle times nothing (shapes the process chose already apply) */
    int    residual_fusion;        /* 3D periodic V-cycle: 1 = residual and restriction in one pass
                                      through shared memory; 0 = default (a residual kernel and a
                                      restriction kernel: measured faster) */
    int    uniform_alpha;          /* 0 = default (a level whose theta*alpha faces all hold one value,
                                      checked on the device at each coefficient load, has the
                                      velocity operator take that value as a scalar: the same bits,
                                      one array fewer per stencil), -1 = always read the arrays */
    int    smoother_fusion_cells;  /* smoother_fusion > 0: only levels with at most this many cells
                                      take the fused colour pairs (the larger ones one launch per
                                      colour); 0 = default (every level that allows them) */
} lmm_knobs;

/* Inputs of gmres(...): b_u, b_p, alpha_fc, beta, beta_ed, gamma.
 * beta_ed has 1 array (nodal) in 2D and 3 (xy, xz, yz edges) in 3D
 * (stag_mg_solver.f90:181-193).  gamma may be NULL when visc_type != +-3. */
typedef struct lmm_fields_in {
    const double* b_u[3];
    const double* b_p;
    const double* alpha_fc[3];
    const double* beta;
    const double* beta_ed[3];
    const double* gamma;
    int layout;                    /* LMM_LAYOUT_* */
    /* ghost widths of the BoxLib arrays (ignored for LMM_LAYOUT_COMPACT) */
    int ng_b_u, ng_b_p, ng_alpha, ng_beta, ng_beta_ed, ng_gamma;
} lmm_fields_in;

/* x_u, x_p: initial guess in, solution out (gmres.f90:38-39). */
typedef struct lmm_fields_out {
    double* x_u[3];
    double* x_p;
    int layout;
    int ng_x_u, ng_x_p;            /* BoxLib ghost widths; apply_matrix.f90:52-58 needs >= 1 */
} lmm_fields_out;

#define LMM_HISTORY_MAX 512
typedef struct lmm_stats {
    int    total_iter;             /* inner iterations (gmres.f90:319) */
    int    outer_iter;             /* restarts started (gmres.f90:297) */
    int    vcycles;                /* staggered V-cycles applied (vcycle_counter, counted like gmres.f90:222-225) */
    int    pressure_vcycles;
    double norm_b;                 /* |b| (gmres.f90:137-140) */
    double norm_pre_b;             /* |M^-1 b| (gmres.f90:125-130) */
    double norm_resid;             /* last preconditioned residual (LMM_METHOD_GMRES) */
    double norm_init_resid;
    double norm_resid_true;        /* last true residual |b-Ax| measured at a restart */
    double norm_init_true;
    double solve_ms;               /* device time of the solve (CUDA events) */
    double h2d_ms, d2h_ms;
    int    n_history;
    double history[LMM_HISTORY_MAX]; /* residual estimate after each inner iteration */
} lmm_stats;

typedef struct lmm_handle lmm_handle;

/* Fill the reference defaults (probin_gmres.f90:119-157; visc_type = 1 as in
 * probin_common.f90:224) and this library's defaults (GMRES, FP64, no net). */
void lmm_default_knobs(lmm_knobs* k);

/* Build persistent device workspaces for one grid and knob set.  Replaces the
 * per-call allocations of gmres.f90:92-103, stag_mg_solver.f90:126-198 and
 * apply_precon.f90:67-83 and the setup hooks stag_mg_layout_build /
 * mgt_macproj_precon_build (main_driver.f90:262-263). */
int lmm_stokes_create(const lmm_grid* g, const lmm_knobs* k, int device, lmm_handle** h);

/* The gmres(...) call (gmres.f90:30-477) with host arrays.  Copies inputs to
 * the device, solves, copies x_u, x_p back.  theta_alpha is inout like the
 * reference (returned unchanged); norm_pre_rhs may be NULL (gmres.f90:45,132-134).
 * The caller's b, beta, beta_ed and gamma are never modified. */
int lmm_stokes_solve(lmm_handle* h, const lmm_fields_in* in, lmm_fields_out* out,
                     double* theta_alpha, double* norm_pre_rhs, lmm_stats* st);

/* Same solve on device-resident LMM_LAYOUT_COMPACT arrays (no host copies). */
int lmm_stokes_solve_device(lmm_handle* h, const lmm_fields_in* in_dev, lmm_fields_out* out_dev,
                            double* theta_alpha, double* norm_pre_rhs, lmm_stats* st);

/* Change the stopping rules of a handle between solves: gmres_rel_tol,
 * gmres_abs_tol, gmres_max_outer, gmres_max_iter, gmres_min_iter,
 * stag_mg_rel_tol, mg_rel_tol and the verbosity knobs take the values of *k;
 * every other field of *k must equal the handle's (LMM_ERR_INVALID and no
 * change otherwise).  The time steppers move gmres_abs_tol between the
 * predictor and corrector solves of one step
 * (advance_timestep_overdamped.f90:311-323,568;
 * advance_timestep_inertial.f90:476-488,796-818); this keeps the handle, its
 * device memory and its captured graphs. */
int lmm_stokes_update_knobs(lmm_handle* h, const lmm_knobs* k);

int lmm_stokes_destroy(lmm_handle* h);
const char* lmm_strerror(int code);
int lmm_version(void);

/* CUDA stream the handle launches on (a cudaStream_t). */
void* lmm_stream(lmm_handle* h);

/* ---- operator-level entry points (device pointers, compact layout) ------
 * They act on the coefficients last loaded with lmm_op_load_coeffs and give
 * tests and callers the reference's sub-operators one by one. */

/* Load alpha_fc, beta, beta_ed, gamma (device, compact) and theta_alpha, and
 * coarsen them over the MG hierarchy (stag_mg_solver.f90:200-230). */
int lmm_op_load_coeffs(lmm_handle* h, const lmm_fields_in* coeffs_dev, double theta_alpha);

/* Lphi = (theta*alpha - L) phi on the finest level; color 0 = all faces,
 * 1..2*dm = one Gauss-Seidel colour (stag_applyop.f90:20-202). */
int lmm_op_stag_applyop(lmm_handle* h, const double* const phi[3], double* const Lphi[3], int color);

/* [b_u; b_p] = [A G; -D 0][x_u; x_p] (apply_matrix.f90:23-122). */
int lmm_op_apply_matrix(lmm_handle* h, const double* const x_u[3], const double* x_p,
                        double* const b_u[3], double* b_p);

/* x = M^-1 b for the configured precon_type (apply_precon.f90:29-536). */
int lmm_op_apply_precon(lmm_handle* h, const double* const b_u[3], const double* b_p,
                        double* const x_u[3], double* x_p);

/* phi <- stag_mg_max_vcycles V-cycles of (theta*alpha - L) phi = rhs
 * (stag_mg_solver.f90:37-868). phi is an initial guess. */
int lmm_op_stag_mg_solver(lmm_handle* h, const double* const rhs[3], double* const phi[3]);

/* One smoothing colour (applyop(color) + stag_mg_update(color)) on level lev
 * (stag_mg_solver.f90:363-399, 1637-2463). color 0 = weighted Jacobi. */
int lmm_op_smooth(lmm_handle* h, int lev, const double* const rhs[3], double* const phi[3], int color);

/* Residual rhs - L phi on level lev restricted to level lev+1
 * (stag_mg_solver.f90:406-437, 971-1175). */
int lmm_op_residual_restrict(lmm_handle* h, int lev, const double* const rhs[3],
                             const double* const phi[3], double* const rhs_coarse[3]);

/* phi_fine += P phi_coarse (stag_mg_solver.f90:1370-1633). */
int lmm_op_prolong_add(lmm_handle* h, int lev, const double* const phi_coarse[3], double* const phi_fine[3]);

/* Weighted staggered / cell inner products (norm_inner_product.f90:16-375):
 * out[0..dm-1] = per-component face sums, out[dm] = cell sum. */
int lmm_op_inner_prod(lmm_handle* h, const double* const a_u[3], const double* a_p,
                      const double* const b_u[3], const double* b_p, double* out_host);

/* Means removed by apply_precon (sum_umac_press, norm_inner_product.f90:579-680):
 * out[0] = <p>, out[1..dm] = <u_d>. */
int lmm_op_sum_umac_press(lmm_handle* h, const double* const u[3], const double* p, double* out_host);

/* Number of staggered MG levels (compute_nlevs_mg, stag_mg_layout.f90:179-222). */
int lmm_op_num_levels(lmm_handle* h);

/* ---- measurement hooks (no counterpart in the reference) ---------------- */

/* Kernels this library has launched in this process so far. */
int64_t lmm_kernel_launches(void);

/* Average device time (CUDA events on the handle's stream) of `reps`
 * repetitions of one hot operation on the finest level, using the
 * coefficients and level-0 buffers of the last solve:
 *   0 one Gauss-Seidel smooth, all 2*dm colours, FP64 (timed as pairs of
 *     smooths and halved)
 *   1 the same in FP32
 *   2 stag_applyop (all faces), FP64
 *   3 apply_matrix, FP64
 *   4 one staggered V-cycle, FP64
 *   5 one staggered V-cycle, FP32
 *   6 one pressure V-cycle, FP64
 *   7 the classical Gram-Schmidt passes of one restart cycle (columns
 *     1..gmres_max_inner: projections, update and norm of w; FGMRES)
 *   8 one Krylov normalisation V = w / |w| (with its FP32 copy when
 *     precision is FP32)                                                */
int lmm_time_op(lmm_handle* h, int which, int reps, double* ms_per_rep);

/* The block-shape autotuner's choices so far (no counterpart in the
 * reference): one text line per tuned kernel, precision, visc_type and
 * grid, with its chosen block and the measured ms of the default and the
 * chosen geometry.  Writes at most cap - 1 bytes and a terminating zero
 * into buf (cap > 0); returns the length of the full report. */
int lmm_autotune_report(char* buf, int cap);

#ifdef __cplusplus
}
#endif
#endif /* LMM_STOKES_H */
