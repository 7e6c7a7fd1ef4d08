"""The time steppers' predictor/corrector pair on the GPU handle: the
corrector's absolute tolerance moves through lmm_stokes_update_knobs on the
live handle, and both solves match the same sequence on the CPU oracle
(velocity and mean-removed pressure to 1e-10, iterations within 1)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lowmachmixtures_b200 import abi, synth, timestep  # noqa: E402

from helpers import OracleSolver  # noqa: E402

pytestmark = pytest.mark.gpu


def coeffs(p):
    return p.alpha_fc, p.beta, p.beta_ed, p.gamma


def test_update_knobs_stopping_rules_only():
    from lowmachmixtures_b200._native import LmmError
    from lowmachmixtures_b200.gmres import StokesSolver
    with StokesSolver(2, (32, 32), 1 / 32, precon_type=2, visc_type=-2) as s:
        s.update_knobs(gmres_abs_tol=1e-6, gmres_rel_tol=1e-8, gmres_max_iter=50)
        assert s.knobs.gmres_abs_tol == 1e-6 and s.knobs.gmres_max_iter == 50
        with pytest.raises(LmmError):
            s.update_knobs(precon_type=1)
        with pytest.raises(LmmError):
            s.update_knobs(gmres_max_inner=8)
        with pytest.raises(LmmError):
            s.update_knobs(gmres_abs_tol=-1.0)
        assert s.knobs.precon_type == 2 and s.knobs.gmres_abs_tol == 1e-6


@pytest.mark.parametrize("dm,n,bc,theta", [(2, 64, None, 0.0), (2, 64, (abi.LMM_BC_PERIODIC, abi.LMM_BC_NO_SLIP_WALL), 0.0),
                                           (3, 32, None, 0.1 * 32 * 32)])
def test_predictor_corrector_matches_oracle(oracle, dm, n, bc, theta):
    from lowmachmixtures_b200.gmres import StokesSolver
    prob = synth.make_problem(dm, n, 30.0, 8, theta_alpha=theta, bc=bc)
    kn = dict(precon_type=2, visc_type=-2, gmres_rel_tol=1e-9)
    rng = np.random.default_rng(3)

    def corrector(pred):
        # a small corrector rhs that depends on the predictor's solution
        return [1e-4 * (b + 0.1 * x) * m for b, x, m in zip(prob.b_u, pred.x_u, masks)], 1e-4 * rng.standard_normal(prob.shape)

    masks = [np.ones(prob.shape) for _ in range(dm)]
    if bc is not None:
        synth.zero_wall_faces(dm, prob.bc, masks)
    rng = np.random.default_rng(3)
    ref = timestep.predictor_corrector(OracleSolver(prob, oracle, **kn), (prob.b_u, prob.b_p), corrector, coeffs(prob), theta)
    rng = np.random.default_rng(3)
    with StokesSolver(dm, prob.n[:dm], prob.dx, knobs=abi.make_knobs(**kn), bc=bc) as s:
        got = timestep.predictor_corrector(s, (prob.b_u, prob.b_p), corrector, coeffs(prob), theta)
        assert s.knobs.gmres_abs_tol == 0.0
    assert abs(got[0].norm_pre_rhs - ref[0].norm_pre_rhs) <= 1e-12 * ref[0].norm_pre_rhs
    for r, g in zip(ref, got):
        for c in range(dm):
            err = np.abs(g.x_u[c] - r.x_u[c]).max() / np.abs(r.x_u[c]).max()
            assert err <= 1e-10, err
        po, pg = r.x_p - r.x_p.mean(), g.x_p - g.x_p.mean()
        assert np.abs(pg - po).max() <= 1e-10 * np.abs(po).max()
        assert abs(g.stats["total_iter"] - r.stats["total_iter"]) <= 1
    # the corrector stopped on the predictor's scale
    assert got[1].stats["norm_resid"] <= got[0].norm_pre_rhs * 1e-9
