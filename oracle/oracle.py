"""Python handle on the CPU oracle (oracle/_build/liblmmoracle.so).

TEST INFRASTRUCTURE ONLY: the oracle restates the reference Stokes solve on
the CPU.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg may import this module, and only as the checker or the CPU baseline.
Parity status: unpinned against reference outputs (the Fortran reference
cannot be built here); cross-checked against tests/golden fixtures made by an
independent numpy restatement and against analytic/paper known answers.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from lowmachmixtures_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liblmmoracle.so")
_lib = None


def build(quiet: bool = True) -> str:
    subprocess.run(["make", "-C", HERE, "-j8"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _lib.orc_stokes_solve.restype = C.c_int
    return _lib


def set_tile_size(tx=1024000, ty=8, tz=8):
    lib().orc_set_tile_size(int(tx), int(ty), int(tz))


def default_knobs(**kw) -> abi.Knobs:
    return abi.make_knobs(**kw)


def fields_in(prob, b_u=None, b_p=None):
    f = abi.FieldsIn()
    f.b_u = abi.ptr_array(b_u if b_u is not None else prob.b_u)
    f.b_p = abi.ptr(b_p if b_p is not None else prob.b_p)
    f.alpha_fc = abi.ptr_array(prob.alpha_fc)
    f.beta = abi.ptr(prob.beta)
    f.beta_ed = abi.ptr_array(prob.beta_ed)
    f.gamma = abi.ptr(prob.gamma)
    f.layout = abi.LMM_LAYOUT_COMPACT
    return f


def grid_of(prob) -> abi.Grid:
    return abi.make_grid(prob.dm, prob.n, prob.dx, getattr(prob, "bc", None))


def solve(prob, knobs: abi.Knobs, x_u=None, x_p=None, theta_alpha=None):
    """Run gmres(...) (or FGMRES) on the CPU.  Returns (status, x_u, x_p,
    theta_alpha_out, norm_pre_rhs, stats dict)."""
    if x_u is None:
        x_u, x_p = prob.zeros_like_solution()
    x_u = [np.ascontiguousarray(a.copy()) for a in x_u]
    x_p = np.ascontiguousarray(x_p.copy())
    fin = fields_in(prob)
    fout = abi.FieldsOut()
    fout.x_u = abi.ptr_array(x_u)
    fout.x_p = abi.ptr(x_p)
    fout.layout = abi.LMM_LAYOUT_COMPACT
    th = C.c_double(prob.theta_alpha if theta_alpha is None else theta_alpha)
    npr = C.c_double(0.0)
    st = abi.Stats()
    g = grid_of(prob)
    rc = lib().orc_stokes_solve(C.byref(g), C.byref(knobs), C.byref(fin), C.byref(fout),
                                C.byref(th), C.byref(npr), C.byref(st))
    return rc, x_u, x_p, th.value, npr.value, st.as_dict()


def stag_applyop(prob, visc_type, phi, color=0, Lphi=None, theta_alpha=None):
    out = [np.zeros_like(p) if Lphi is None else Lphi[i].copy() for i, p in enumerate(phi)]
    g = grid_of(prob)
    th = prob.theta_alpha if theta_alpha is None else theta_alpha
    rc = lib().orc_stag_applyop(C.byref(g), C.c_int(visc_type), C.byref(fields_in(prob)), C.c_double(th),
                                abi.ptr_array(phi), abi.ptr_array(out), C.c_int(color))
    assert rc == 0
    return out


def num_levels(prob, minwidth=2):
    return lib().orc_num_levels(C.byref(grid_of(prob)), C.c_int(minwidth))


def level_shape(prob, lev):
    return tuple(s >> lev for s in prob.shape)


def coarse_coeffs(prob, knobs, lev, theta_alpha=None):
    shp = level_shape(prob, lev)
    dm = prob.dm
    alpha = [np.zeros(shp) for _ in range(dm)]
    beta = np.zeros(shp)
    gamma = np.zeros(shp)
    nl = [prob.n[d] >> lev for d in range(dm)]
    bed = [np.zeros(abi.edge_shape(dm, nl, getattr(prob, "bc", None), e)) for e in range(1 if dm == 2 else 3)]
    th = prob.theta_alpha if theta_alpha is None else theta_alpha
    rc = lib().orc_coarse_coeffs(C.byref(grid_of(prob)), C.byref(knobs), C.byref(fields_in(prob)), C.c_double(th),
                                 C.c_int(lev), abi.ptr_array(alpha), abi.ptr(beta), abi.ptr_array(bed), abi.ptr(gamma))
    assert rc == 0
    return alpha, beta, bed, gamma


def smooth(prob, knobs, lev, rhs, phi, color, theta_alpha=None):
    phi = [p.copy() for p in phi]
    th = prob.theta_alpha if theta_alpha is None else theta_alpha
    rc = lib().orc_smooth(C.byref(grid_of(prob)), C.byref(knobs), C.byref(fields_in(prob)), C.c_double(th),
                          C.c_int(lev), abi.ptr_array(rhs), abi.ptr_array(phi), C.c_int(color))
    assert rc == 0
    return phi


def residual_restrict(prob, knobs, lev, rhs, phi, theta_alpha=None):
    shp = level_shape(prob, lev + 1)
    out = [np.zeros(shp) for _ in range(prob.dm)]
    th = prob.theta_alpha if theta_alpha is None else theta_alpha
    rc = lib().orc_residual_restrict(C.byref(grid_of(prob)), C.byref(knobs), C.byref(fields_in(prob)),
                                     C.c_double(th), C.c_int(lev), abi.ptr_array(rhs), abi.ptr_array(phi),
                                     abi.ptr_array(out))
    assert rc == 0
    return out


def prolong_add(prob, lev, phi_coarse, phi_fine):
    phi_fine = [p.copy() for p in phi_fine]
    rc = lib().orc_prolong_add(C.byref(grid_of(prob)), C.c_int(lev), abi.ptr_array(phi_coarse),
                               abi.ptr_array(phi_fine))
    assert rc == 0
    return phi_fine


def stag_mg_solver(prob, knobs, rhs, phi=None, theta_alpha=None):
    phi = [np.zeros_like(r) for r in rhs] if phi is None else [p.copy() for p in phi]
    th = prob.theta_alpha if theta_alpha is None else theta_alpha
    rc = lib().orc_stag_mg_solver(C.byref(grid_of(prob)), C.byref(knobs), C.byref(fields_in(prob)),
                                  C.c_double(th), abi.ptr_array(rhs), abi.ptr_array(phi))
    assert rc == 0
    return phi


def apply_matrix(prob, visc_type, x_u, x_p, theta_alpha=None):
    b_u = [np.zeros_like(a) for a in x_u]
    b_p = np.zeros_like(x_p)
    th = prob.theta_alpha if theta_alpha is None else theta_alpha
    rc = lib().orc_apply_matrix(C.byref(grid_of(prob)), C.c_int(visc_type), C.byref(fields_in(prob)),
                                C.c_double(th), abi.ptr_array(x_u), abi.ptr(x_p), abi.ptr_array(b_u), abi.ptr(b_p))
    assert rc == 0
    return b_u, b_p


def apply_precon(prob, knobs, b_u, b_p, theta_alpha=None):
    x_u = [np.zeros_like(a) for a in b_u]
    x_p = np.zeros_like(b_p)
    th = prob.theta_alpha if theta_alpha is None else theta_alpha
    rc = lib().orc_apply_precon(C.byref(grid_of(prob)), C.byref(knobs), C.byref(fields_in(prob)),
                                C.c_double(th), abi.ptr_array(b_u), abi.ptr(b_p), abi.ptr_array(x_u), abi.ptr(x_p))
    assert rc == 0
    return x_u, x_p


def inner_prod(prob, a_u, a_p, b_u, b_p):
    out = (C.c_double * 4)()
    rc = lib().orc_inner_prod(C.byref(grid_of(prob)), abi.ptr_array(a_u), abi.ptr(a_p), abi.ptr_array(b_u),
                              abi.ptr(b_p), out)
    assert rc == 0
    return list(out)[: prob.dm + 1]


def sum_umac_press(prob, u, p):
    out = (C.c_double * 4)()
    rc = lib().orc_sum_umac_press(C.byref(grid_of(prob)), abi.ptr_array(u), abi.ptr(p), out)
    assert rc == 0
    return list(out)[: prob.dm + 1]


def macproject(prob, knobs, mac_rhs, alpha_fc=None):
    phi = np.zeros_like(mac_rhs)
    al = prob.alpha_fc if alpha_fc is None else alpha_fc
    rc = lib().orc_macproject(C.byref(grid_of(prob)), C.byref(knobs), abi.ptr_array(al), abi.ptr(mac_rhs),
                              abi.ptr(phi))
    assert rc == 0
    return phi


def set_threads(n: int) -> None:
    """OpenMP threads of the oracle's parallel loops (the CPU-baseline legs
    time it on one core and on all)."""
    lib().omp_set_num_threads(int(n))
