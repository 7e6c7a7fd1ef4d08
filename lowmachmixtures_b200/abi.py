"""ctypes mirror of include/lmm_stokes.h (the C ABI of liblmmstokes).

The structs here are byte-for-byte the C structs; ``Knobs`` mirrors the
Fortran module ``probin_gmres_module`` (src_gmres/probin_gmres.f90:13-22,
defaults :119-157) plus ``visc_type`` (src_common/probin_common.f90:94-100).
"""
from __future__ import annotations

import ctypes as C

LMM_OK = 0
LMM_WARN_MAX_ITER = 1
LMM_WARN_MAX_OUTER = 2
LMM_WARN_RESID_MISMATCH = 3
LMM_ERR_INVALID = -1
LMM_ERR_BREAKDOWN = -2
LMM_ERR_NONFINITE = -3
LMM_ERR_CUDA = -4
LMM_ERR_WATCHDOG = -5
LMM_ERR_NO_DEVICE = -6
LMM_ERR_TOO_LARGE = -7
LMM_ERR_BOUNDS = -8  # -DLMM_BOUNDS_CHECK builds only

LMM_BC_PERIODIC = -1
LMM_BC_NO_SLIP_WALL = 100
LMM_BC_SLIP_WALL = 200
LMM_LAYOUT_COMPACT = 0
LMM_LAYOUT_BOXLIB = 1
LMM_METHOD_GMRES = 0
LMM_METHOD_FGMRES = 1
LMM_PRECISION_FP64 = 0
LMM_PRECISION_FP32 = 1
LMM_HISTORY_MAX = 512

_dp = C.POINTER(C.c_double)


class Grid(C.Structure):
    _fields_ = [
        ("dm", C.c_int),
        ("n", C.c_int * 3),
        ("dx", C.c_double),
        ("bc_lo", C.c_int * 3),
        ("bc_hi", C.c_int * 3),
    ]


_KNOB_FIELDS = [
    ("precon_type", C.c_int),
    ("visc_schur_approx", C.c_int),
    ("p_norm_weight", C.c_double),
    ("scale_factor", C.c_double),
    ("mg_verbose", C.c_int),
    ("cg_verbose", C.c_int),
    ("mg_max_vcycles", C.c_int),
    ("mg_minwidth", C.c_int),
    ("mg_bottom_solver", C.c_int),
    ("mg_nsmooths_down", C.c_int),
    ("mg_nsmooths_up", C.c_int),
    ("mg_nsmooths_bottom", C.c_int),
    ("mg_max_bottom_nlevels", C.c_int),
    ("mg_rel_tol", C.c_double),
    ("stag_mg_verbosity", C.c_int),
    ("stag_mg_max_vcycles", C.c_int),
    ("stag_mg_minwidth", C.c_int),
    ("stag_mg_bottom_solver", C.c_int),
    ("stag_mg_nsmooths_down", C.c_int),
    ("stag_mg_nsmooths_up", C.c_int),
    ("stag_mg_nsmooths_bottom", C.c_int),
    ("stag_mg_max_bottom_nlevels", C.c_int),
    ("stag_mg_omega", C.c_double),
    ("stag_mg_smoother", C.c_int),
    ("stag_mg_rel_tol", C.c_double),
    ("gmres_rel_tol", C.c_double),
    ("gmres_abs_tol", C.c_double),
    ("gmres_verbose", C.c_int),
    ("gmres_max_outer", C.c_int),
    ("gmres_max_inner", C.c_int),
    ("gmres_max_iter", C.c_int),
    ("gmres_min_iter", C.c_int),
    ("visc_type", C.c_int),
    ("method", C.c_int),
    ("precision", C.c_int),
    ("learned_stage", C.c_int),
    ("tail_cells", C.c_int),
    ("tail_smem_kb", C.c_int),
    ("use_graphs", C.c_int),
    ("smoother_fusion", C.c_int),
    ("l2_persist", C.c_int),
    ("orthogonalization", C.c_int),
    ("host_wait", C.c_int),
    ("ensemble_batch", C.c_int),
    ("smoother_tma", C.c_int),
    ("smoother_tma_slabs", C.c_int),
    ("smoother_tma_cells", C.c_int),
    ("smoother_order", C.c_int),
    ("autotune", C.c_int),
    ("residual_fusion", C.c_int),
    ("uniform_alpha", C.c_int),
    ("smoother_fusion_cells", C.c_int),
]


class Knobs(C.Structure):
    _fields_ = _KNOB_FIELDS

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in _KNOB_FIELDS if name != "reserved"}


# probin_gmres.f90:119-157; visc_type default probin_common.f90:224
KNOB_DEFAULTS = dict(
    precon_type=1, visc_schur_approx=0, p_norm_weight=1.0, scale_factor=1.0,
    mg_verbose=0, cg_verbose=0, mg_max_vcycles=1, mg_minwidth=2, mg_bottom_solver=4,
    mg_nsmooths_down=2, mg_nsmooths_up=2, mg_nsmooths_bottom=8, mg_max_bottom_nlevels=10,
    mg_rel_tol=1e-9,
    stag_mg_verbosity=0, stag_mg_max_vcycles=1, stag_mg_minwidth=2, stag_mg_bottom_solver=4,
    stag_mg_nsmooths_down=2, stag_mg_nsmooths_up=2, stag_mg_nsmooths_bottom=8,
    stag_mg_max_bottom_nlevels=10, stag_mg_omega=1.0, stag_mg_smoother=1, stag_mg_rel_tol=1e-9,
    gmres_rel_tol=1e-9, gmres_abs_tol=0.0, gmres_verbose=1, gmres_max_outer=20,
    gmres_max_inner=5, gmres_max_iter=100, gmres_min_iter=1,
    visc_type=1, method=LMM_METHOD_GMRES, precision=LMM_PRECISION_FP64, learned_stage=0,
    tail_cells=0, tail_smem_kb=0, use_graphs=0, smoother_fusion=0, l2_persist=0, orthogonalization=0, host_wait=0,
    ensemble_batch=0, smoother_tma=0, smoother_tma_slabs=0, smoother_tma_cells=0, smoother_order=0, autotune=0, residual_fusion=0,
    uniform_alpha=0, smoother_fusion_cells=0,
)


def make_knobs(**overrides) -> Knobs:
    k = Knobs()
    vals = dict(KNOB_DEFAULTS)
    for key, v in overrides.items():
        if key not in vals:
            raise KeyError(f"unknown knob {key!r}")
        vals[key] = v
    for key, v in vals.items():
        setattr(k, key, v)
    return k


class FieldsIn(C.Structure):
    _fields_ = [
        ("b_u", _dp * 3),
        ("b_p", _dp),
        ("alpha_fc", _dp * 3),
        ("beta", _dp),
        ("beta_ed", _dp * 3),
        ("gamma", _dp),
        ("layout", C.c_int),
        ("ng_b_u", C.c_int),
        ("ng_b_p", C.c_int),
        ("ng_alpha", C.c_int),
        ("ng_beta", C.c_int),
        ("ng_beta_ed", C.c_int),
        ("ng_gamma", C.c_int),
    ]


class FieldsOut(C.Structure):
    _fields_ = [
        ("x_u", _dp * 3),
        ("x_p", _dp),
        ("layout", C.c_int),
        ("ng_x_u", C.c_int),
        ("ng_x_p", C.c_int),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("total_iter", C.c_int),
        ("outer_iter", C.c_int),
        ("vcycles", C.c_int),
        ("pressure_vcycles", C.c_int),
        ("norm_b", C.c_double),
        ("norm_pre_b", C.c_double),
        ("norm_resid", C.c_double),
        ("norm_init_resid", C.c_double),
        ("norm_resid_true", C.c_double),
        ("norm_init_true", C.c_double),
        ("solve_ms", C.c_double),
        ("h2d_ms", C.c_double),
        ("d2h_ms", C.c_double),
        ("n_history", C.c_int),
        ("history", C.c_double * LMM_HISTORY_MAX),
    ]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_ if name != "history"}
        d["history"] = list(self.history[: self.n_history])
        return d


class EnsembleItem(C.Structure):
    """lmm_ensemble_item (include/lmm_ensemble.h)"""
    _fields_ = [
        ("n", C.c_int * 3),
        ("dx", C.c_double),
        ("theta_alpha", C.c_double),
        ("b_u", _dp * 3),
        ("b_p", _dp),
        ("alpha_fc", _dp * 3),
        ("beta", _dp),
        ("beta_ed", _dp * 3),
        ("gamma", _dp),
        ("x_u", _dp * 3),
        ("x_p", _dp),
        ("status", C.c_int),
        ("stats", Stats),
    ]


def make_grid(dm: int, n, dx: float, bc=None) -> Grid:
    """bc: None (periodic box) or one entry per direction, either a code
    (both sides) or a (lo, hi) pair of codes (LMM_BC_PERIODIC,
    100-103 no-slip walls, 200-203 slip walls)."""
    g = Grid()
    g.dm = dm
    nn = list(n) + [1] * (3 - len(n))
    for d in range(3):
        g.n[d] = int(nn[d]) if d < dm else 1
        lo = hi = LMM_BC_PERIODIC
        if bc is not None and d < dm:
            b = bc[d]
            lo, hi = (b, b) if isinstance(b, int) else (int(b[0]), int(b[1]))
        g.bc_lo[d] = lo
        g.bc_hi[d] = hi
    g.dx = float(dx)
    return g


def walled(bc, d: int) -> bool:
    """True when direction d of a make_grid-style bc spec has walls."""
    if bc is None:
        return False
    b = bc[d]
    lo = b if isinstance(b, int) else b[0]
    return lo != LMM_BC_PERIODIC


def edge_nodal(dm: int, e: int):
    """Directions in which edge array e is nodal: 2D (x, y); 3D xy, xz, yz."""
    if dm == 2:
        return (0, 1)
    return ((0, 1), (0, 2), (1, 2))[e]


def edge_shape(dm: int, n, bc, e: int):
    """Compact (z, y, x) shape of edge array e: n+1 nodes along a
    wall-bounded direction in which the edge is nodal, n otherwise."""
    ext = [int(n[d]) + (1 if (d in edge_nodal(dm, e) and walled(bc, d)) else 0) for d in range(dm)]
    return tuple(reversed(ext))


def ptr(a) -> "C.POINTER(C.c_double) | None":
    """Raw double* of a numpy array (C-contiguous float64) or integer address."""
    if a is None:
        return None
    if isinstance(a, int):
        return C.cast(C.c_void_p(a), _dp)
    if hasattr(a, "data_ptr"):  # torch tensor
        return C.cast(C.c_void_p(a.data_ptr()), _dp)
    assert a.dtype.name == "float64" and a.flags["C_CONTIGUOUS"], "need contiguous float64"
    return a.ctypes.data_as(_dp)


def ptr_array(arrs):
    out = (_dp * 3)()
    for i, a in enumerate(arrs):
        out[i] = ptr(a)
    return out
