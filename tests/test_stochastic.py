"""The stochastic momentum forcing: the numpy oracle's invariants on the CPU,
and the GPU generator (lmm_stochastic_rhs) against it."""
import ctypes as C

import numpy as np
import pytest

from oracle import stochastic as S


def test_oracle_forcing_is_mean_free_and_scales_with_sqrt_eta():
    rng = np.random.default_rng(0)
    n = (16, 12, 8)
    shape = tuple(reversed(n))
    eta = rng.uniform(0.5, 2.0, shape)
    eds = [rng.uniform(0.5, 2.0, shape) for _ in range(3)]
    b = S.stochastic_rhs(3, n, 1 / 16, 1e-3, 1.0, eta, eds, 7)
    for c in range(3):
        assert abs(b[c].mean()) < 1e-9 * np.abs(b[c]).max()   # divergence of a periodic flux
    b4 = S.stochastic_rhs(3, n, 1 / 16, 1e-3, 1.0, 4 * eta, [4 * e for e in eds], 7)
    for c in range(3):
        np.testing.assert_allclose(b4[c], 2 * b[c], rtol=1e-12, atol=1e-12 * np.abs(b[c]).max())
    g = S.gauss(3, 0, 200000)
    assert abs(g.mean()) < 0.01 and abs(g.std() - 1) < 0.01


@pytest.mark.gpu
@pytest.mark.parametrize("dm,n", [(3, (16, 16, 16)), (3, (32, 16, 8)), (2, (48, 32))])
def test_gpu_forcing_matches_oracle(dm, n):
    import torch

    from lowmachmixtures_b200 import _native, abi, synth
    lib = _native.load()
    eta, eds = synth.mixture_viscosity(dm, n[0], 3) if len(set(n)) == 1 else (None, None)
    if eta is None:
        rng = np.random.default_rng(1)
        shape = tuple(reversed(n))
        eta = rng.uniform(0.5, 3.0, shape)
        eds = [rng.uniform(0.5, 3.0, shape) for _ in range(1 if dm == 2 else 3)]
    dx = 1.0 / n[0]
    ref = S.stochastic_rhs(dm, n, dx, 1e-3, 1.0, eta, eds, 11)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    de, ded = dev(eta), [dev(e) for e in eds]
    b = [torch.zeros_like(de) for _ in range(dm)]
    nn = (C.c_int * 3)(*(list(n) + [1] * (3 - dm)))
    rc = lib.lmm_stochastic_rhs(dm, nn, dx, 1e-3, 1.0, abi.ptr(de), abi.ptr_array(ded), 11, abi.ptr_array(b), None)
    assert rc == 0
    torch.cuda.synchronize()
    for c in range(dm):
        scale = np.abs(ref[c]).max()
        np.testing.assert_allclose(b[c].cpu().numpy(), ref[c], rtol=0, atol=1e-12 * scale)


@pytest.mark.gpu
def test_stochastic_mixture_solve_parity_small(oracle):
    """The 256^3 mixture recipe at 32^3: GPU forcing, then the FP64 solve equals
    the oracle's (same forcing from the oracle generator) within 1e-10, and
    the mixed method meets the tolerance."""
    import torch

    from lowmachmixtures_b200 import abi, synth
    from lowmachmixtures_b200.gmres import StokesSolver
    n = 32
    prob = synth.config_3d_256_mixture(n, 2)
    prob.b_u = S.stochastic_rhs(3, (n, n, n), prob.dx, 1e-3, 1.0, prob.beta, prob.beta_ed, 2)
    k = oracle.default_knobs(precon_type=2, visc_type=-2, gmres_max_inner=20)
    rc, xu_o, xp_o, _, _, st_o = oracle.solve(prob, k)
    assert rc == 0
    kn = abi.make_knobs(precon_type=2, visc_type=-2, gmres_max_inner=20)
    xu, xp = prob.zeros_like_solution()
    with StokesSolver(3, (n, n, n), prob.dx, knobs=kn) as s:
        _, _, st = s.solve(prob.b_u, prob.b_p, xu, xp, prob.alpha_fc, prob.beta, prob.beta_ed, prob.gamma, 0.0)
    assert abs(st["total_iter"] - st_o["total_iter"]) <= 1
    for c in range(3):
        assert np.linalg.norm(xu[c] - xu_o[c]) <= 1e-10 * np.linalg.norm(xu_o[c])
    kn = abi.make_knobs(precon_type=2, visc_type=-2, gmres_max_inner=20, method=abi.LMM_METHOD_FGMRES,
                        precision=abi.LMM_PRECISION_FP32)
    xu2, xp2 = prob.zeros_like_solution()
    with StokesSolver(3, (n, n, n), prob.dx, knobs=kn) as s:
        _, _, st3 = s.solve(prob.b_u, prob.b_p, xu2, xp2, prob.alpha_fc, prob.beta, prob.beta_ed, prob.gamma, 0.0)
    assert st3["norm_resid_true"] <= 1e-9 * st3["norm_b"]
