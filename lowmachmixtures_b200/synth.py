"""Seeded synthetic Stokes problems with the shapes of the benchmark workloads.

The reference benchmarks nothing and ships no input data, so every workload
is synthetic (one grid, isotropic dx = 1/n, periodic unless walls are asked for):

* log-viscosity field g(x) = sum_{m=1..6} cos(2 pi k_m . x + phi_m) with integer
  wave vectors 0 < |k_m| <= 4 and phases phi_m ~ U[0, 2 pi), normalised to
  max |g| = 1 over every sample point; beta = exp(ln(C)/2 * g), so the
  viscosity contrast is about C;
* beta at cell centres, beta_ed at nodes (2D) or at xy/xz/yz edge midpoints
  (3D), i.e. the layouts gmres(...) receives (src_gmres/gmres.f90:41-42,
  src_gmres/stag_mg_solver.f90:178-194);
* alpha_fc = 1 (the density rhotot_fc the time steppers pass,
  src_multiSpec/advance_timestep_overdamped.f90:317);
* b_u ~ N(0,1) i.i.d. per unique face with each component's mean removed,
  b_p = 0, zero initial guess.

Arrays are numpy float64 in the compact layout: shape (ny, nx) in 2D or
(nz, ny, nx) in 3D, i fastest, periodic seam stored once.  Along a
wall-bounded direction the wall-normal face array keeps faces lo..hi (face
lo is the wall, zero in every rhs; hi+1 is implied zero) and an edge array
nodal in that direction keeps all n+1 nodes.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class StokesProblem:
    dm: int
    n: tuple
    dx: float
    theta_alpha: float
    alpha_fc: list
    beta: np.ndarray
    beta_ed: list
    gamma: np.ndarray
    b_u: list
    b_p: np.ndarray
    contrast: float
    seed: int
    bc: tuple = None

    @property
    def shape(self):
        return tuple(reversed(self.n[: self.dm]))

    def zeros_like_solution(self):
        return [np.zeros(self.shape) for _ in range(self.dm)], np.zeros(self.shape)


def _wave_vectors(rng, dm, count=6, kmax=4):
    ks = []
    while len(ks) < count:
        k = rng.integers(-kmax, kmax + 1, size=dm)
        r2 = int((k * k).sum())
        if 0 < r2 <= kmax * kmax:
            ks.append(k.astype(np.float64))
    return ks


def _logfield(ks, phases, coords):
    g = np.zeros(np.broadcast_shapes(*[c.shape for c in coords]))
    for k, ph in zip(ks, phases):
        arg = ph + 2.0 * math.pi * sum(k[d] * coords[d] for d in range(len(coords)))
        g = g + np.cos(arg)
    return g


def _grids(n, dm, offsets, extra=(0, 0, 0)):
    """Coordinates (x, y[, z]) broadcast to the compact array shape, with
    per-direction offsets in units of dx (0 = nodal, 0.5 = cell centred) and
    `extra` points past the last (the hi wall node of a wall-bounded edge)."""
    dx = 1.0 / n[0]
    axes = []
    for d in range(dm):
        axes.append((np.arange(n[d] + extra[d]) + offsets[d]) * dx)
    if dm == 2:
        y, x = np.meshgrid(axes[1], axes[0], indexing="ij")
        return [x, y]
    z, y, x = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    return [x, y, z]


def viscosity_fields(dm, n, contrast, seed, bc=None):
    """beta at cells and beta_ed at nodes (2D) / edges xy, xz, yz (3D);
    edges keep the hi wall node along wall-bounded directions."""
    from .abi import edge_nodal, walled
    rng = np.random.Generator(np.random.PCG64(seed))
    ks = _wave_vectors(rng, dm)
    phases = rng.uniform(0.0, 2.0 * math.pi, size=len(ks))
    cc = _logfield(ks, phases, _grids(n, dm, [0.5] * dm))

    def extra(e):
        return tuple(1 if (d < dm and d in edge_nodal(dm, e) and walled(bc, d)) else 0 for d in range(3))
    if dm == 2:
        eds = [_logfield(ks, phases, _grids(n, dm, [0.0, 0.0], extra(0)))]
    else:
        eds = [
            _logfield(ks, phases, _grids(n, dm, [0.0, 0.0, 0.5], extra(0))),  # xy edges
            _logfield(ks, phases, _grids(n, dm, [0.0, 0.5, 0.0], extra(1))),  # xz edges
            _logfield(ks, phases, _grids(n, dm, [0.5, 0.0, 0.0], extra(2))),  # yz edges
        ]
    gmax = max(np.abs(cc).max(), *[np.abs(e).max() for e in eds])
    s = math.log(contrast) / 2.0 / gmax
    beta = np.exp(s * cc)
    beta_ed = [np.exp(s * e) for e in eds]
    return beta, beta_ed, rng


def zero_wall_faces(dm: int, bc, u):
    """Zero face lo of each wall-normal component along its wall-bounded
    direction (in place; u in the compact (z, y, x) layout)."""
    from .abi import walled
    for c in range(dm):
        if walled(bc, c):
            idx = [slice(None)] * dm
            idx[dm - 1 - c] = 0
            u[c][tuple(idx)] = 0.0
    return u


def make_problem(dm: int, n: int, contrast: float, seed: int, theta_alpha: float = 0.0,
                 gamma_value: float = 0.0, bc=None) -> StokesProblem:
    """bc: None (periodic) or per direction a code / (lo, hi) pair as in
    abi.make_grid; the rhs is zero on the wall faces."""
    nn = (n,) * dm
    beta, beta_ed, rng = viscosity_fields(dm, nn, contrast, seed, bc)
    shape = tuple(reversed(nn))
    b_u = []
    for _ in range(dm):
        r = rng.standard_normal(size=shape)
        b_u.append(np.ascontiguousarray(r - r.mean()))
    if bc is not None:
        bc = tuple(bc)
        zero_wall_faces(dm, bc, b_u)
    return StokesProblem(
        dm=dm, n=nn + (1,) * (3 - dm), dx=1.0 / n, theta_alpha=float(theta_alpha),
        alpha_fc=[np.ones(shape) for _ in range(dm)], beta=beta, beta_ed=beta_ed,
        gamma=np.full(shape, float(gamma_value)), b_u=b_u, b_p=np.zeros(shape),
        contrast=float(contrast), seed=int(seed), bc=bc)


# Named workloads (the parity and benchmark configurations).
def config_2d_64(seed: int = 0) -> StokesProblem:
    """2D 64^2, contrast 10, steady (theta_alpha = 0)."""
    return make_problem(2, 64, 10.0, seed, theta_alpha=0.0)


def config_3d_128(seed: int = 0, n: int = 128) -> StokesProblem:
    """3D n^3, contrast 100, inertial alpha = rho/dt with alpha*dx^2/beta0 = 0.1."""
    dx = 1.0 / n
    return make_problem(3, n, 100.0, seed, theta_alpha=0.1 / (dx * dx))


def config_3d_64_learned(seed: int = 0, contrast: float = 1000.0) -> StokesProblem:
    """3D 64^3 steady problems of the learned-preconditioner workload."""
    return make_problem(3, 64, contrast, seed, theta_alpha=0.0)


SPECIES_VISCOSITY = (1.0, 2.0, 5.0, 10.0)


def mixture_viscosity(dm: int, n: int, seed: int, eta_s=SPECIES_VISCOSITY):
    """Viscosity of a 4-species mixture: seeded smooth mass fractions (6
    Fourier modes |k| <= 4 per species, shifted positive and normalised to sum
    to 1) and the log-linear rule ln eta = sum_s w_s ln eta_s (not a rule of
    the reference, whose compute_mixture_properties.f90:315-346 offers
    constant, water-glycerol and linear forms).  Returns (eta_cc, eta_ed)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    offs_cc = [0.5] * dm
    offs_ed = [[0.0, 0.0]] if dm == 2 else [[0.0, 0.0, 0.5], [0.0, 0.5, 0.0], [0.5, 0.0, 0.0]]

    def field(ks, ph, offs):
        # sum of cos(2 pi k.x + phase), separable: products of 1D complex exponentials
        axes = [(np.arange(n) + offs[d]) / n for d in range(dm)]
        g = 0.0
        for k, p in zip(ks, ph):
            e = [np.exp(2j * math.pi * k[d] * axes[d]) for d in range(dm)]
            if dm == 2:
                term = e[1][:, None] * e[0][None, :]
            else:
                term = e[2][:, None, None] * e[1][None, :, None] * e[0][None, None, :]
            g = g + (np.exp(1j * p) * term).real
        return g

    fields = []
    for _ in eta_s:
        ks = _wave_vectors(rng, dm)
        ph = rng.uniform(0.0, 2.0 * math.pi, size=len(ks))
        cc = field(ks, ph, offs_cc)
        eds = [field(ks, ph, o) for o in offs_ed]
        gmax = max(np.abs(cc).max(), *[np.abs(e).max() for e in eds])
        fields.append((cc / gmax, [e / gmax for e in eds]))

    def mix(parts):
        w = [1.0 + 0.9 * p for p in parts]   # positive: g in [-1, 1]
        tot = sum(w)
        return np.exp(sum((wi / tot) * math.log(es) for wi, es in zip(w, eta_s)))

    eta_cc = mix([f[0] for f in fields])
    eta_ed = [mix([f[1][e] for f in fields]) for e in range(len(offs_ed))]
    return eta_cc, eta_ed


def config_3d_256_mixture(n: int = 256, seed: int = 0) -> StokesProblem:
    """3D n^3 periodic, 4-species mixture viscosity, overdamped (theta = 0).
    b_u is left zero: the stochastic-stress divergence is generated on the
    GPU (lmm_stochastic_rhs, kT = 1, dt = 1e-3, dV = dx^3)."""
    eta_cc, eta_ed = mixture_viscosity(3, n, seed)
    shape = (n, n, n)
    return StokesProblem(dm=3, n=(n, n, n), dx=1.0 / n, theta_alpha=0.0, alpha_fc=[np.ones(shape) for _ in range(3)],
                         beta=eta_cc, beta_ed=eta_ed, gamma=np.zeros(shape), b_u=[np.zeros(shape) for _ in range(3)],
                         b_p=np.zeros(shape), contrast=float(eta_cc.max() / eta_cc.min()), seed=int(seed))
