"""The time steppers' pair of solves (predictor, corrector with the
absolute tolerance taken from the predictor's |M^-1 b|) on the CPU oracle:
the host-side sequence of lowmachmixtures_b200.timestep, checked with an
oracle-backed stand-in for the GPU handle."""
import numpy as np
import pytest

from lowmachmixtures_b200 import abi, synth, timestep

from helpers import OracleSolver


def coeffs(p):
    return p.alpha_fc, p.beta, p.beta_ed, p.gamma


@pytest.mark.parametrize("bc", [None, (abi.LMM_BC_PERIODIC, abi.LMM_BC_NO_SLIP_WALL)])
def test_corrector_tolerance_from_predictor(oracle, bc):
    prob = synth.make_problem(2, 32, 30.0, 4, theta_alpha=0.0, bc=bc)
    s = OracleSolver(prob, oracle, precon_type=2, visc_type=-2, gmres_rel_tol=1e-9, gmres_abs_tol=0.0)
    small = [1e-4 * b for b in prob.b_u]
    pred, corr = timestep.predictor_corrector(s, (prob.b_u, prob.b_p), lambda r: (small, prob.b_p), coeffs(prob), 0.0)
    # corrector solved with abs_tol = norm_pre_rhs(predictor) * rel_tol, then the knob restored
    assert s.calls == [0.0, pytest.approx(pred.norm_pre_rhs * 1e-9, rel=1e-15)]
    assert s.knobs.gmres_abs_tol == 0.0
    assert corr.stats["norm_resid"] <= pred.norm_pre_rhs * 1e-9
    # the same corrector solve on its own relative tolerance needs more iterations
    alone = timestep._solve(s, small, prob.b_p, coeffs(prob), 0.0)
    assert corr.stats["total_iter"] < alone.stats["total_iter"]


def test_abs_tol_restored_on_failure():
    class Boom(Exception):
        pass

    class Fake:
        dm, shape = 2, (4, 4)

        def __init__(self):
            self.knobs = abi.make_knobs(gmres_abs_tol=1e-3, gmres_rel_tol=1e-6)
            self.seen = []

        def update_knobs(self, **kw):
            for k, v in kw.items():
                setattr(self.knobs, k, v)

        def solve(self, *a):
            self.seen.append(self.knobs.gmres_abs_tol)
            if len(self.seen) == 2:
                raise Boom()
            return 0.0, 1e5, {}

    f = Fake()
    z = [np.zeros((4, 4))] * 2
    with pytest.raises(Boom):
        timestep.predictor_corrector(f, (z, z[0]), lambda r: (z, z[0]), (z, z[0], z[:1], z[0]), 0.0)
    assert f.seen == [1e-3, pytest.approx(0.1)]  # max(1e-3, 1e5 * 1e-6)
    assert f.knobs.gmres_abs_tol == 1e-3


def test_warm_start(oracle):
    """gmres.f90:263 stops on rel_tol * min(|M^-1 b|, |M^-1 r0|): a warm
    start lowers r0 and with it the target, so on the relative rule alone it
    buys accuracy, not iterations; with an absolute tolerance on the scale
    of |M^-1 b| (as the corrector gets) it saves iterations."""
    prob = synth.make_problem(2, 32, 30.0, 6, theta_alpha=50.0)
    s = OracleSolver(prob, oracle, precon_type=2, visc_type=-2)
    first = timestep.solve_warm(s, (prob.b_u, prob.b_p), coeffs(prob), 50.0, None)
    rng = np.random.default_rng(1)
    nudged = [b + 1e-3 * rng.standard_normal(b.shape) for b in prob.b_u]
    cold = timestep.solve_warm(s, (nudged, prob.b_p), coeffs(prob), 50.0, None)
    warm = timestep.solve_warm(s, (nudged, prob.b_p), coeffs(prob), 50.0, first)
    assert abs(warm.stats["total_iter"] - cold.stats["total_iter"]) <= 1
    assert warm.stats["norm_resid"] < cold.stats["norm_resid"]
    s.update_knobs(gmres_abs_tol=first.norm_pre_rhs * 1e-9)
    cold_a = timestep.solve_warm(s, (nudged, prob.b_p), coeffs(prob), 50.0, None)
    warm_a = timestep.solve_warm(s, (nudged, prob.b_p), coeffs(prob), 50.0, first)
    assert warm_a.stats["total_iter"] < cold_a.stats["total_iter"]
    for c in range(2):
        assert np.abs(warm_a.x_u[c] - cold.x_u[c]).max() < 1e-6 * np.abs(cold.x_u[c]).max()
