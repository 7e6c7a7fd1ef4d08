"""lmm_ensemble_solve: independent problems of uneven sizes solved
concurrently give the same bits as one solve per instance, and every
instance meets its tolerance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_ensemble_equals_individual_solves():
    import torch

    from lowmachmixtures_b200 import abi, ensemble
    from lowmachmixtures_b200.gmres import StokesSolver
    probs = ensemble.make_instances(10, seed=5, sizes=(32, 48, 64, 96))
    kn = abi.make_knobs(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES, precision=abi.LMM_PRECISION_FP32,
                        gmres_rel_tol=1e-8)
    st, stats, sols, _ = ensemble.solve(probs, kn, workers=4)
    assert all(s == 0 for s in st)
    for p, s in zip(probs, stats):
        assert s["norm_resid_true"] <= 1e-8 * s["norm_b"]
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    for p, (xu, xp) in zip(probs, sols):
        with StokesSolver(2, p.n[:2], p.dx, knobs=kn) as s:
            yu, yp = [torch.zeros_like(xp) for _ in range(2)], torch.zeros_like(xp)
            s.solve_device([dev(a) for a in p.b_u], dev(p.b_p), yu, yp, [dev(a) for a in p.alpha_fc], dev(p.beta),
                           [dev(a) for a in p.beta_ed], dev(p.gamma), p.theta_alpha)
        for c in range(2):
            assert torch.equal(xu[c], yu[c])
        assert torch.equal(xp, yp)
