"""Generate the golden fixtures of tests/golden from the numpy restatement.

    python tests/golden/make_golden.py

writes stencils_2d.npz, stencils_3d.npz and vcycle.npz (inputs and outputs)
next to this script.  The reference ships no tests or golden vectors and
cannot be built here, so these fixtures come from numpy_ref.py, an
independent restatement of the reference formulas; the oracle is pinned
against them.
"""
from __future__ import annotations

import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import numpy_ref as R  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
VISCS = (-1, 1, -2, 2, -3, 3)


def rand_coeffs(rng, dm, n, const=False):
    shape = (n,) * dm
    ne = 1 if dm == 2 else 3
    if const:
        beta = np.full(shape, 0.7)
        gamma = np.full(shape, 0.3)
        bed = [np.full(shape, 0.7) for _ in range(ne)]
    else:
        beta = rng.uniform(0.5, 2.0, shape)
        gamma = rng.uniform(0.1, 0.5, shape)
        bed = [rng.uniform(0.5, 2.0, shape) for _ in range(ne)]
    alpha = [rng.uniform(0.5, 1.5, shape) for _ in range(dm)]
    return alpha, beta, bed, gamma


def stencil_cases(dm, n, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = {}
    dx = 1.0 / n
    theta = 3.0
    for visc in VISCS:
        alpha, beta, bed, gamma = rand_coeffs(rng, dm, n, const=visc > 0)
        phi = [rng.standard_normal((n,) * dm) for _ in range(dm)]
        rhs = [rng.standard_normal((n,) * dm) for _ in range(dm)]
        ta = [theta * a for a in alpha]
        key = f"v{visc}"
        for c in range(dm):
            out[f"{key}_alpha{c}"] = alpha[c]
            out[f"{key}_phi{c}"] = phi[c]
            out[f"{key}_rhs{c}"] = rhs[c]
        out[f"{key}_beta"] = beta
        out[f"{key}_gamma"] = gamma
        for e, b in enumerate(bed):
            out[f"{key}_bed{e}"] = b
        L = R.applyop(visc, phi, ta, beta, bed, gamma, dx)
        for c in range(dm):
            out[f"{key}_L{c}"] = L[c]
        for color in range(0, 2 * dm + 1):
            sm = R.smooth_colour(visc, color, rhs, phi, ta, beta, bed, gamma, dx)
            for c in range(dm):
                out[f"{key}_smooth{color}_{c}"] = sm[c]
    # transfer operators
    f = [rng.standard_normal((n,) * dm) for _ in range(dm)]
    for c in range(dm):
        out[f"xfer_f{c}"] = f[c]
    r6 = R.restrict_stag(f, False)
    rs = R.restrict_stag(f, True)
    cc = [rng.standard_normal((n // 2,) * dm) for _ in range(dm)]
    pr = R.prolong_add(f, cc)
    for c in range(dm):
        out[f"xfer_restrict{c}"] = r6[c]
        out[f"xfer_simple{c}"] = rs[c]
        out[f"xfer_coarse{c}"] = cc[c]
        out[f"xfer_prolong{c}"] = pr[c]
    p = rng.standard_normal((n,) * dm)
    out["grad_p"] = p
    for c, g in enumerate(R.grad(p, dx)):
        out[f"grad{c}"] = g
    out["div"] = R.div(f, dx)
    # weighted inner product of f with itself (seam weight 3) and cell sum
    out["ip_faces"] = np.array([float((R.seam_weights(f[c].shape, c) * f[c] * f[c]).sum()) for c in range(dm)])
    return out


def vcycle_cases():
    out = {}
    for dm, n, nlev in ((2, 16, 4), (3, 8, 3)):
        rng = np.random.Generator(np.random.PCG64(100 + dm))
        dx = 1.0 / n
        alpha, beta, bed, gamma = rand_coeffs(rng, dm, n)
        rhs = [rng.standard_normal((n,) * dm) for _ in range(dm)]
        theta = 5.0
        ta = [theta * a for a in alpha]
        for smoother in (1, 0):
            phi = R.vcycle(-2, rhs, ta, beta, bed, gamma, dx, nlev, smoother=smoother, omega=1.0 if smoother else 0.6)
            for c in range(dm):
                out[f"d{dm}_s{smoother}_phi{c}"] = phi[c]
        for c in range(dm):
            out[f"d{dm}_alpha{c}"] = alpha[c]
            out[f"d{dm}_rhs{c}"] = rhs[c]
        out[f"d{dm}_beta"] = beta
        out[f"d{dm}_gamma"] = gamma
        for e, b in enumerate(bed):
            out[f"d{dm}_bed{e}"] = b
        out[f"d{dm}_theta"] = np.array([theta])
    return out


def main():
    np.savez_compressed(os.path.join(HERE, "stencils_2d.npz"), **stencil_cases(2, 8, 1))
    np.savez_compressed(os.path.join(HERE, "stencils_3d.npz"), **stencil_cases(3, 8, 2))
    np.savez_compressed(os.path.join(HERE, "vcycle.npz"), **vcycle_cases())
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
