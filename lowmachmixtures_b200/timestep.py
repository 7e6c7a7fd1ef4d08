"""The caller side of gmres(...) in the reference's time steppers.

Every step of the overdamped integrator
(src_multiSpec/advance_timestep_overdamped.f90:300-330, 555-570) and of the
inertial one (src_multiSpec/advance_timestep_inertial.f90:462-490, 796-820)
solves the Stokes system twice:

1. the predictor from a zero initial guess, with the configured
   gmres_abs_tol, keeping norm_pre_rhs = |M^-1 b|;
2. the corrector, again from a zero initial guess, with
   gmres_abs_tol = max(gmres_abs_tol_in, norm_pre_rhs * gmres_rel_tol), so a
   corrector whose right-hand side is small stops on the predictor's scale
   instead of stalling on its own;
3. gmres_abs_tol restored.

``predictor_corrector`` runs that sequence on one persistent StokesSolver
handle: the tolerance moves through lmm_stokes_update_knobs, so device
memory and captured graphs stay.  ``solve_warm`` is the warm-started
variant a caller can use when consecutive right-hand sides are close: the
previous solution is the initial guess (x_u, x_p are intent(inout) in
gmres(...), gmres.f90:38-39).  gmres.f90:263 stops on
rel_tol * min(|M^-1 b|, |M^-1 r0|), so a warm start alone buys accuracy at
the same iteration count; with an absolute tolerance on the scale of
|M^-1 b| it saves iterations.
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class StepResult:
    x_u: list
    x_p: np.ndarray
    norm_pre_rhs: float
    stats: dict


def _solve(solver, b_u, b_p, coeffs, theta_alpha, x_u=None, x_p=None):
    shape = solver.shape
    x_u = [np.zeros(shape) for _ in range(solver.dm)] if x_u is None else [np.array(a, copy=True) for a in x_u]
    x_p = np.zeros(shape) if x_p is None else np.array(x_p, copy=True)
    alpha_fc, beta, beta_ed, gamma = coeffs
    _, npr, st = solver.solve(b_u, b_p, x_u, x_p, alpha_fc, beta, beta_ed, gamma, theta_alpha)
    return StepResult(x_u, x_p, npr, st)


def predictor_corrector(solver, predictor_rhs, corrector_rhs, coeffs, theta_alpha):
    """One time step's pair of solves.

    predictor_rhs: (b_u, b_p).  corrector_rhs: callable taking the predictor
    StepResult and returning the corrector's (b_u, b_p) (the reference
    builds it from v* = v + delta v).  coeffs: (alpha_fc, beta, beta_ed,
    gamma) host arrays.  Returns (predictor, corrector) StepResults; the
    solver's gmres_abs_tol is the same on return as on entry."""
    abs_tol_in = float(solver.knobs.gmres_abs_tol)
    rel_tol = float(solver.knobs.gmres_rel_tol)
    pred = _solve(solver, *predictor_rhs, coeffs, theta_alpha)
    try:
        solver.update_knobs(gmres_abs_tol=max(abs_tol_in, pred.norm_pre_rhs * rel_tol))
        corr = _solve(solver, *corrector_rhs(pred), coeffs, theta_alpha)
    finally:
        solver.update_knobs(gmres_abs_tol=abs_tol_in)
    return pred, corr


def solve_warm(solver, rhs, coeffs, theta_alpha, previous: StepResult | None):
    """Solve from the previous solution (or zero) as initial guess."""
    if previous is None:
        return _solve(solver, *rhs, coeffs, theta_alpha)
    return _solve(solver, *rhs, coeffs, theta_alpha, previous.x_u, previous.x_p)
