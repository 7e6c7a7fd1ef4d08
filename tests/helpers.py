"""Shared test helpers: problems built from golden fixtures."""
from __future__ import annotations

import os

import numpy as np

from lowmachmixtures_b200 import abi
from lowmachmixtures_b200.synth import StokesProblem

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def problem_from_fixture(fx, prefix, dm, n, theta_alpha):
    shape = (n,) * dm
    ne = 1 if dm == 2 else 3
    return StokesProblem(
        dm=dm, n=(n,) * dm + (1,) * (3 - dm), dx=1.0 / n, theta_alpha=float(theta_alpha),
        alpha_fc=[np.ascontiguousarray(fx[f"{prefix}alpha{c}"]) for c in range(dm)],
        beta=np.ascontiguousarray(fx[f"{prefix}beta"]),
        beta_ed=[np.ascontiguousarray(fx[f"{prefix}bed{e}"]) for e in range(ne)],
        gamma=np.ascontiguousarray(fx[f"{prefix}gamma"]),
        b_u=[np.zeros(shape) for _ in range(dm)], b_p=np.zeros(shape), contrast=0.0, seed=0)


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / den)


class OracleSolver:
    """The StokesSolver calls predictor_corrector makes, answered by the oracle."""

    def __init__(self, prob, oracle, **kn):
        self.prob, self.oracle = prob, oracle
        self.dm, self.shape = prob.dm, prob.shape
        self.knobs = abi.make_knobs(**kn)
        self.calls = []

    def update_knobs(self, **kw):
        for k, v in kw.items():
            setattr(self.knobs, k, v)

    def solve(self, b_u, b_p, x_u, x_p, alpha_fc, beta, beta_ed, gamma, theta_alpha):
        self.calls.append(float(self.knobs.gmres_abs_tol))
        p = self.prob
        saved = (p.b_u, p.b_p)
        p.b_u, p.b_p = b_u, b_p
        try:
            rc, xu, xp, th, npr, st = self.oracle.solve(p, self.knobs, x_u=x_u, x_p=x_p, theta_alpha=theta_alpha)
        finally:
            p.b_u, p.b_p = saved
        assert rc >= 0
        for a, b in zip(x_u, xu):
            a[...] = b
        x_p[...] = xp
        return th, npr, st
