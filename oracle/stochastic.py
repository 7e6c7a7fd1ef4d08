"""CPU oracle of the stochastic momentum forcing (numpy).

TEST INFRASTRUCTURE ONLY: tests/ compare the GPU generator
(lmm_stochastic_rhs) with it.  Restates, for a periodic box and one random
stage, src_common/stochastic_m_fluxdiv.f90: symmetric stochastic stress
with diagonal variance 2 (:573) and one value per edge shared by both
off-diagonal components (:586-600), scaled by sqrt(2 kT/(dV dt)) (:135) and
sqrt(eta) (:306-359), and the face divergence of stoch_m_force_2d/_3d
(:450-551).  The random numbers follow the library's counter-based
generator: value q of field f is a function of (seed, f, q) only.
"""
from __future__ import annotations

import numpy as np

_U64 = np.uint64


def _smix(z):
    z = z + _U64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> _U64(30))) * _U64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> _U64(27))) * _U64(0x94D049BB133111EB)
    return z ^ (z >> _U64(31))


def gauss(seed: int, f: int, count: int) -> np.ndarray:
    """normal numbers 0..count-1 of field f"""
    with np.errstate(over="ignore"):
        q = np.arange(count, dtype=np.uint64)
        h1 = _smix(_U64(seed) ^ _smix((_U64(f) << _U64(48)) ^ q))
        h2 = _smix(h1)
    u1 = ((h1 >> _U64(11)).astype(np.float64) + 1.0) * (1.0 / 9007199254740992.0)
    u2 = (h2 >> _U64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(6.283185307179586 * u2)


def stochastic_rhs(dm, n, dx, dt, kT, eta_cc, eta_ed, seed):
    """b_u (list of dm compact arrays, shape (nz, ny, nx) / (ny, nx))"""
    shape = tuple(reversed(n[:dm]))
    N = int(np.prod(shape))
    var = np.sqrt(2.0 * kT / (dx ** dm * dt))
    dxinv = 1.0 / dx
    cc = [(np.sqrt(2.0) * gauss(seed, c, N).reshape(shape)) * var * np.sqrt(eta_cc) for c in range(dm)]
    ne = 1 if dm == 2 else 3
    ed = [gauss(seed, dm + e, N).reshape(shape) * var * np.sqrt(eta_ed[e]) for e in range(ne)]
    ax = {"x": dm - 1, "y": dm - 2, "z": 0}   # numpy axis of each direction

    def up(a, d):    # a at index + 1 in direction d
        return np.roll(a, -1, axis=ax[d])

    def dn(a, d):    # a at index - 1 in direction d
        return np.roll(a, 1, axis=ax[d])

    if dm == 2:
        nd = ed[0]
        bx = 0.0 + (cc[0] - dn(cc[0], "x")) * dxinv + (up(nd, "y") - nd) * dxinv
        by = 0.0 + (up(nd, "x") - nd) * dxinv + (cc[1] - dn(cc[1], "y")) * dxinv
        return [bx, by]
    xy, xz, yz = ed
    bx = 0.0 + (cc[0] - dn(cc[0], "x")) * dxinv + (up(xy, "y") - xy) * dxinv + (up(xz, "z") - xz) * dxinv
    by = 0.0 + (up(xy, "x") - xy) * dxinv + (cc[1] - dn(cc[1], "y")) * dxinv + (up(yz, "z") - yz) * dxinv
    bz = 0.0 + (up(xz, "x") - xz) * dxinv + (up(yz, "y") - yz) * dxinv + (cc[2] - dn(cc[2], "z")) * dxinv
    return [bx, by, bz]
