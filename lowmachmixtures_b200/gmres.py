"""Host-side mirror of the reference's ``gmres(...)`` entry point.

The Fortran subroutine (src_gmres/gmres.f90:30-45)::

    gmres(mla, the_bc_tower, dx, b_u, b_p, x_u, x_p,
          alpha_fc, beta, beta_ed, gamma, theta_alpha, norm_pre_rhs)

is configured by the ``probin_gmres`` module globals.  Here the same call is
``gmres(dx, b_u, b_p, x_u, x_p, alpha_fc, beta, beta_ed, gamma, theta_alpha,
knobs)``: x_u / x_p are the initial guess and receive the solution in place
(intent inout), theta_alpha is returned unchanged (the reference scales and
unscales it), and norm_pre_rhs = |M^-1 b| is returned.  Negative statuses
(the reference's bl_error aborts) raise ``LmmError``; the non-convergence
warnings of gmres.f90:254-296 come back in ``stats["status"]``.

Everything runs in liblmmstokes.so on the GPU; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from ._native import LmmError, check, load


def _is_torch(a) -> bool:
    return hasattr(a, "data_ptr") and hasattr(a, "is_cuda")


class StokesSolver:
    """A persistent solver for one grid and one knob set (the handle of
    lmm_stokes_create).  Reuse it across calls: device memory is allocated
    once.  bc: None (periodic box) or per direction a BC code or (lo, hi)
    pair -- LMM_BC_PERIODIC, no-slip walls 100-103, slip walls 200-203
    (src_common/bc.f90:23-44), as the reference's bc_lo / bc_hi."""

    def __init__(self, dm: int, n, dx: float, knobs: abi.Knobs | None = None, device: int = 0, bc=None,
                 **knob_overrides):
        self.lib = load()
        self.dm = int(dm)
        self.n = tuple(int(v) for v in n)[: self.dm]
        self.dx = float(dx)
        self.bc = None if bc is None else tuple(bc)
        self.knobs = knobs if knobs is not None else abi.make_knobs(**knob_overrides)
        self.grid = abi.make_grid(self.dm, self.n, self.dx, self.bc)
        self._h = C.c_void_p()
        check(self.lib.lmm_stokes_create(C.byref(self.grid), C.byref(self.knobs), int(device), C.byref(self._h)),
              "lmm_stokes_create")
        self.shape = tuple(reversed(self.n))

    # ------------------------------------------------------------------ life cycle
    def close(self):
        if self._h:
            self.lib.lmm_stokes_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def update_knobs(self, **stopping):
        """Change the stopping rules (gmres_rel_tol, gmres_abs_tol,
        gmres_max_outer / max_iter / min_iter, stag_mg_rel_tol, mg_rel_tol,
        verbosity) of this handle between solves (lmm_stokes_update_knobs)."""
        k = abi.Knobs()
        C.memmove(C.byref(k), C.byref(self.knobs), C.sizeof(abi.Knobs))
        for name, v in stopping.items():
            setattr(k, name, v)
        check(self.lib.lmm_stokes_update_knobs(self._h, C.byref(k)), "lmm_stokes_update_knobs")
        self.knobs = k

    def num_levels(self) -> int:
        return self.lib.lmm_op_num_levels(self._h)

    def time_op(self, which: int, reps: int = 10) -> float:
        """Average device ms of one hot operation (see lmm_time_op)."""
        ms = C.c_double(0.0)
        check(self.lib.lmm_time_op(self._h, int(which), int(reps), C.byref(ms)), "lmm_time_op")
        return ms.value

    def stream_ptr(self) -> int:
        return int(self.lib.lmm_stream(self._h) or 0)

    # ------------------------------------------------------------------ solves
    def _fields(self, b_u, b_p, alpha_fc, beta, beta_ed, gamma, layout, ng):
        fin = abi.FieldsIn()
        fin.b_u = abi.ptr_array(b_u)
        fin.b_p = abi.ptr(b_p)
        fin.alpha_fc = abi.ptr_array(alpha_fc)
        fin.beta = abi.ptr(beta)
        fin.beta_ed = abi.ptr_array(beta_ed)
        fin.gamma = abi.ptr(gamma)
        fin.layout = layout
        ng = ng or {}
        fin.ng_b_u = ng.get("b_u", 0)
        fin.ng_b_p = ng.get("b_p", 0)
        fin.ng_alpha = ng.get("alpha_fc", 0)
        fin.ng_beta = ng.get("beta", 0)
        fin.ng_beta_ed = ng.get("beta_ed", 0)
        fin.ng_gamma = ng.get("gamma", 0)
        return fin

    def solve(self, b_u, b_p, x_u, x_p, alpha_fc, beta, beta_ed, gamma, theta_alpha,
              layout: int = abi.LMM_LAYOUT_COMPACT, ng: dict | None = None):
        """Host arrays (numpy float64).  x_u, x_p are updated in place.
        Returns (theta_alpha, norm_pre_rhs, stats dict)."""
        fin = self._fields(b_u, b_p, alpha_fc, beta, beta_ed, gamma, layout, ng)
        fout = abi.FieldsOut()
        fout.x_u = abi.ptr_array(x_u)
        fout.x_p = abi.ptr(x_p)
        fout.layout = layout
        ng = ng or {}
        fout.ng_x_u = ng.get("x_u", 0)
        fout.ng_x_p = ng.get("x_p", 0)
        th = C.c_double(theta_alpha)
        npr = C.c_double(0.0)
        st = abi.Stats()
        rc = self.lib.lmm_stokes_solve(self._h, C.byref(fin), C.byref(fout), C.byref(th), C.byref(npr), C.byref(st))
        check(rc, "gmres")
        d = st.as_dict()
        d["status"] = rc
        return th.value, npr.value, d

    def solve_device(self, b_u, b_p, x_u, x_p, alpha_fc, beta, beta_ed, gamma, theta_alpha):
        """Device-resident compact arrays (torch CUDA float64 tensors or raw
        integer device pointers).  x_u, x_p are updated in place."""
        fin = self._fields(b_u, b_p, alpha_fc, beta, beta_ed, gamma, abi.LMM_LAYOUT_COMPACT, None)
        fout = abi.FieldsOut()
        fout.x_u = abi.ptr_array(x_u)
        fout.x_p = abi.ptr(x_p)
        fout.layout = abi.LMM_LAYOUT_COMPACT
        th = C.c_double(theta_alpha)
        npr = C.c_double(0.0)
        st = abi.Stats()
        rc = self.lib.lmm_stokes_solve_device(self._h, C.byref(fin), C.byref(fout), C.byref(th), C.byref(npr),
                                              C.byref(st))
        check(rc, "gmres")
        d = st.as_dict()
        d["status"] = rc
        return th.value, npr.value, d

    # ------------------------------------------------------------------ operators (device arrays)
    def load_coeffs(self, alpha_fc, beta, beta_ed, gamma, theta_alpha):
        fin = self._fields([None] * 3, None, alpha_fc, beta, beta_ed, gamma, abi.LMM_LAYOUT_COMPACT, None)
        check(self.lib.lmm_op_load_coeffs(self._h, C.byref(fin), C.c_double(theta_alpha)), "lmm_op_load_coeffs")

    def stag_applyop(self, phi, Lphi, color=0):
        check(self.lib.lmm_op_stag_applyop(self._h, abi.ptr_array(phi), abi.ptr_array(Lphi), int(color)),
              "lmm_op_stag_applyop")

    def apply_matrix(self, x_u, x_p, b_u, b_p):
        check(self.lib.lmm_op_apply_matrix(self._h, abi.ptr_array(x_u), abi.ptr(x_p), abi.ptr_array(b_u),
                                           abi.ptr(b_p)), "lmm_op_apply_matrix")

    def apply_precon(self, b_u, b_p, x_u, x_p):
        check(self.lib.lmm_op_apply_precon(self._h, abi.ptr_array(b_u), abi.ptr(b_p), abi.ptr_array(x_u),
                                           abi.ptr(x_p)), "lmm_op_apply_precon")

    def stag_mg_solver(self, rhs, phi):
        check(self.lib.lmm_op_stag_mg_solver(self._h, abi.ptr_array(rhs), abi.ptr_array(phi)),
              "lmm_op_stag_mg_solver")

    def smooth(self, lev, rhs, phi, color):
        check(self.lib.lmm_op_smooth(self._h, int(lev), abi.ptr_array(rhs), abi.ptr_array(phi), int(color)),
              "lmm_op_smooth")

    def residual_restrict(self, lev, rhs, phi, rhs_coarse):
        check(self.lib.lmm_op_residual_restrict(self._h, int(lev), abi.ptr_array(rhs), abi.ptr_array(phi),
                                                abi.ptr_array(rhs_coarse)), "lmm_op_residual_restrict")

    def prolong_add(self, lev, phi_coarse, phi_fine):
        check(self.lib.lmm_op_prolong_add(self._h, int(lev), abi.ptr_array(phi_coarse), abi.ptr_array(phi_fine)),
              "lmm_op_prolong_add")

    def inner_prod(self, a_u, a_p, b_u, b_p):
        out = (C.c_double * 4)()
        check(self.lib.lmm_op_inner_prod(self._h, abi.ptr_array(a_u), abi.ptr(a_p), abi.ptr_array(b_u), abi.ptr(b_p),
                                         out), "lmm_op_inner_prod")
        return list(out)[: self.dm + 1]

    def sum_umac_press(self, u, p):
        out = (C.c_double * 4)()
        check(self.lib.lmm_op_sum_umac_press(self._h, abi.ptr_array(u), abi.ptr(p), out), "lmm_op_sum_umac_press")
        return list(out)[: self.dm + 1]


def gmres(dx, b_u, b_p, x_u, x_p, alpha_fc, beta, beta_ed, gamma, theta_alpha, knobs: abi.Knobs | None = None,
          layout: int = abi.LMM_LAYOUT_COMPACT, ng: dict | None = None, device: int = 0):
    """One-shot gmres(...) call on host arrays (creates and frees a handle).
    x_u, x_p are updated in place; returns (theta_alpha, norm_pre_rhs, stats)."""
    dm = len(b_u)
    if layout == abi.LMM_LAYOUT_COMPACT:
        n = tuple(reversed(np.asarray(b_p).shape))
    else:
        g = (ng or {}).get("b_p", 0)
        n = tuple(s - 2 * g for s in reversed(np.asarray(b_p).shape))
    with StokesSolver(dm, n, dx, knobs=knobs, device=device) as s:
        return s.solve(b_u, b_p, x_u, x_p, alpha_fc, beta, beta_ed, gamma, theta_alpha, layout=layout, ng=ng)


__all__ = ["StokesSolver", "gmres", "LmmError"]
