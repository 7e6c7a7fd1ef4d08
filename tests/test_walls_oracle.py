"""CPU oracle with wall boundaries: known answers and structural checks.

No reference output exists for walls either, so the oracle's wall arithmetic
(physbc_domainvel / physbc_macvel ghost rules, the 2/dx pressure-gradient
stencil, zero applyop on wall faces, the no-slip mean-removal rule) is pinned
by discrete known answers and by properties the discretisation must have:

* plane Poiseuille flow between no-slip walls: the discrete solution of
  -u'' = f with the ghost rule u(-1) = -u(0) (a tridiagonal system);
* a slip-wall cosine mode: u = f / lambda with the Neumann eigenvalue;
* D = -G^T on the interior faces;
* the viscous operator is symmetric for visc_type -1 / -2.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from lowmachmixtures_b200 import abi, synth
from oracle import oracle

NS, SL, PER = abi.LMM_BC_NO_SLIP_WALL, abi.LMM_BC_SLIP_WALL, abi.LMM_BC_PERIODIC


def uniform_problem(dm, n, bc, beta=1.0):
    p = synth.make_problem(dm, n, 10.0, 3, bc=bc)
    p.beta = np.full(p.beta.shape, beta)
    p.beta_ed = [np.full(e.shape, beta) for e in p.beta_ed]
    p.b_u = [np.zeros_like(b) for b in p.b_u]
    return p


def interior_mask(prob, c):
    """1 on the unknown faces of component c (0 on its wall faces)."""
    m = np.ones(prob.shape)
    if abi.walled(prob.bc, c):
        idx = [slice(None)] * prob.dm
        idx[prob.dm - 1 - c] = 0
        m[tuple(idx)] = 0.0
    return m


def random_fields(prob, seed):
    rng = np.random.default_rng(seed)
    u = [rng.standard_normal(prob.shape) * interior_mask(prob, c) for c in range(prob.dm)]
    p = rng.standard_normal(prob.shape)
    return u, p


@pytest.mark.parametrize("method", [abi.LMM_METHOD_GMRES, abi.LMM_METHOD_FGMRES])
def test_poiseuille_between_noslip_walls(method):
    n = 32
    prob = uniform_problem(2, n, (PER, NS))
    prob.b_u[0] = np.ones(prob.shape)
    kn = abi.make_knobs(visc_type=-1, precon_type=1, gmres_rel_tol=1e-13, gmres_max_iter=200, method=method)
    rc, x_u, x_p, *_ = oracle.solve(prob, kn)
    assert rc >= 0
    h = 1.0 / n
    A = np.zeros((n, n))
    for j in range(n):
        A[j, j] = 2.0
        if j > 0:
            A[j, j - 1] = -1.0
        if j < n - 1:
            A[j, j + 1] = -1.0
    A[0, 0] = A[-1, -1] = 3.0  # ghost = -interior at both no-slip walls
    u1d = np.linalg.solve(A / (h * h), np.ones(n))
    ux = x_u[0]
    assert np.abs(ux - ux[:, :1]).max() < 1e-10 * np.abs(ux).max()  # uniform in x
    assert np.abs(ux[:, 0] - u1d).max() < 1e-9 * np.abs(u1d).max()
    assert np.abs(x_u[1]).max() < 1e-9 * np.abs(u1d).max()
    assert np.abs(x_p).max() < 1e-9
    # the continuous profile y(1-y)/2, to second order in h
    yc = (np.arange(n) + 0.5) * h
    assert np.abs(ux[:, 0] - 0.5 * yc * (1 - yc)).max() < 2 * h * h


def test_slip_wall_cosine_mode():
    n = 32
    prob = uniform_problem(2, n, (PER, SL))
    h = 1.0 / n
    f = np.cos(math.pi * (np.arange(n) + 0.5) / n)
    prob.b_u[0] = np.ascontiguousarray(np.repeat(f[:, None], n, axis=1))
    kn = abi.make_knobs(visc_type=-1, precon_type=1, gmres_rel_tol=1e-13, gmres_max_iter=200)
    rc, x_u, x_p, *_ = oracle.solve(prob, kn)
    assert rc >= 0
    lam = (2.0 - 2.0 * math.cos(math.pi / n)) / (h * h)
    # constants are in the null space (periodic x, slip walls, theta = 0)
    got = x_u[0] - x_u[0].mean()
    assert np.abs(got - prob.b_u[0] / lam).max() < 1e-9 * np.abs(f / lam).max()


@pytest.mark.parametrize("dm,bc", [(2, (NS, SL)), (2, ((NS, SL), PER)), (3, (PER, SL, NS)), (3, (NS, NS, SL))])
def test_div_is_minus_grad_transpose(dm, bc):
    n = 8
    prob = synth.make_problem(dm, n, 10.0, 5, bc=bc)
    prob.beta = np.zeros_like(prob.beta)
    prob.beta_ed = [np.zeros_like(e) for e in prob.beta_ed]
    u, p = random_fields(prob, 1)
    zu = [np.zeros(prob.shape) for _ in range(dm)]
    gp, _ = oracle.apply_matrix(prob, -1, zu, p, theta_alpha=0.0)
    _, mdu = oracle.apply_matrix(prob, -1, u, np.zeros(prob.shape), theta_alpha=0.0)
    lhs = float(np.sum(p * (-mdu)))                  # <p, D u>
    rhs = -sum(float(np.sum(u[c] * gp[c])) for c in range(dm))  # -<u, G p>
    assert abs(lhs - rhs) < 1e-10 * (abs(lhs) + 1.0)
    for c in range(dm):  # G p vanishes on the wall faces
        assert np.all(gp[c] * (1 - interior_mask(prob, c)) == 0)


@pytest.mark.parametrize("visc", [-1, -2])
@pytest.mark.parametrize("dm,bc", [(2, (NS, SL)), (2, (SL, NS)), (3, (PER, SL, NS)), (3, (NS, NS, NS))])
def test_viscous_operator_symmetric(visc, dm, bc):
    n = 8
    prob = synth.make_problem(dm, n, 30.0, 7, theta_alpha=3.0, bc=bc)
    u, _ = random_fields(prob, 2)
    v, _ = random_fields(prob, 3)
    Lu = oracle.stag_applyop(prob, visc, u)
    Lv = oracle.stag_applyop(prob, visc, v)
    a = sum(float(np.sum(Lu[c] * v[c])) for c in range(dm))
    b = sum(float(np.sum(u[c] * Lv[c])) for c in range(dm))
    assert abs(a - b) < 1e-11 * max(abs(a), 1.0)
    for c in range(dm):
        assert np.all(Lu[c] * (1 - interior_mask(prob, c)) == 0)


@pytest.mark.parametrize("dm,bc,theta", [(2, (NS, NS), 0.0), (2, (PER, SL), 0.0), (2, (SL, NS), 50.0),
                                         (3, (PER, NS, SL), 0.0), (3, (NS, SL, NS), 1000.0)])
def test_wall_solves_converge(dm, bc, theta):
    n = 16
    prob = synth.make_problem(dm, n, 100.0, 11, theta_alpha=theta, bc=bc)
    sols = []
    for method in (abi.LMM_METHOD_GMRES, abi.LMM_METHOD_FGMRES):
        kn = abi.make_knobs(visc_type=-2, precon_type=1, gmres_rel_tol=1e-10, gmres_max_iter=200, method=method)
        rc, x_u, x_p, *_ = oracle.solve(prob, kn)
        assert rc >= 0
        bu, bp = oracle.apply_matrix(prob, -2, x_u, x_p)
        r = np.sqrt(sum(float(np.sum((prob.b_u[c] - bu[c]) ** 2)) for c in range(dm)) + float(np.sum((prob.b_p - bp) ** 2)))
        nb = np.sqrt(sum(float(np.sum(b ** 2)) for b in prob.b_u))
        assert r / nb < 1e-7
        for c in range(dm):
            assert np.all(x_u[c] * (1 - interior_mask(prob, c)) == 0)
        sols.append((x_u, x_p - x_p.mean()))
    scale = max(np.abs(a).max() for a in sols[0][0])
    for c in range(dm):
        assert np.abs(sols[0][0][c] - sols[1][0][c]).max() < 1e-6 * scale
