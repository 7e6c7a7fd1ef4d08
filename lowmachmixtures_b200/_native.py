"""Loader of the in-tree CUDA library liblmmstokes.so (no fallback).

The product path has no CPU implementation: if the library is missing or no
CUDA device is present, calls fail loudly.  With LMM_BOUNDS_CHECK=1 in the
environment the bounds-check build liblmmstokes_bc.so is loaded instead
(`python -m lowmachmixtures_b200.build --bounds-check`).
"""
from __future__ import annotations

import ctypes as C
import os

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblmmstokes_bc.so" if os.environ.get("LMM_BOUNDS_CHECK") == "1" else "liblmmstokes.so")
_lib = None

_dp = C.POINTER(C.c_double)
_dpp = _dp * 3


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m lowmachmixtures_b200.build`")
    lib = C.CDLL(LIB_PATH)
    P = C.POINTER
    lib.lmm_version.restype = C.c_int
    lib.lmm_strerror.restype = C.c_char_p
    lib.lmm_strerror.argtypes = [C.c_int]
    lib.lmm_default_knobs.argtypes = [P(abi.Knobs)]
    lib.lmm_stokes_create.argtypes = [P(abi.Grid), P(abi.Knobs), C.c_int, P(C.c_void_p)]
    lib.lmm_stokes_create.restype = C.c_int
    lib.lmm_stokes_destroy.argtypes = [C.c_void_p]
    lib.lmm_stokes_update_knobs.argtypes = [C.c_void_p, P(abi.Knobs)]
    lib.lmm_stokes_update_knobs.restype = C.c_int
    for name in ("lmm_stokes_solve", "lmm_stokes_solve_device"):
        f = getattr(lib, name)
        f.argtypes = [C.c_void_p, P(abi.FieldsIn), P(abi.FieldsOut), P(C.c_double), P(C.c_double), P(abi.Stats)]
        f.restype = C.c_int
    lib.lmm_stream.argtypes = [C.c_void_p]
    lib.lmm_stream.restype = C.c_void_p
    lib.lmm_op_load_coeffs.argtypes = [C.c_void_p, P(abi.FieldsIn), C.c_double]
    lib.lmm_op_stag_applyop.argtypes = [C.c_void_p, _dpp, _dpp, C.c_int]
    lib.lmm_op_apply_matrix.argtypes = [C.c_void_p, _dpp, _dp, _dpp, _dp]
    lib.lmm_op_apply_precon.argtypes = [C.c_void_p, _dpp, _dp, _dpp, _dp]
    lib.lmm_op_stag_mg_solver.argtypes = [C.c_void_p, _dpp, _dpp]
    lib.lmm_op_smooth.argtypes = [C.c_void_p, C.c_int, _dpp, _dpp, C.c_int]
    lib.lmm_op_residual_restrict.argtypes = [C.c_void_p, C.c_int, _dpp, _dpp, _dpp]
    lib.lmm_op_prolong_add.argtypes = [C.c_void_p, C.c_int, _dpp, _dpp]
    lib.lmm_op_inner_prod.argtypes = [C.c_void_p, _dpp, _dp, _dpp, _dp, _dp]
    lib.lmm_op_sum_umac_press.argtypes = [C.c_void_p, _dpp, _dp, _dp]
    lib.lmm_nn_gemm_bf16.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    vp, ci = C.c_void_p, C.c_int
    lib.lmm_nn_conv3d.argtypes = [vp, vp, vp, vp, vp, vp, vp] + [ci] * 9 + [vp, vp]
    lib.lmm_nn_conv3d_wgrad.argtypes = [vp, vp, vp] + [ci] * 8 + [vp, vp]
    lib.lmm_nn_pack_weights.argtypes = [vp, vp, vp, ci, ci, vp]
    lib.lmm_net_create.argtypes = [ci, ci, ci, ci, C.c_ulonglong, P(vp)]
    lib.lmm_net_destroy.argtypes = [vp]
    lib.lmm_net_num_params.argtypes = [vp]
    lib.lmm_net_num_params.restype = C.c_int64
    lib.lmm_net_stream.argtypes = [vp, P(vp)]
    lib.lmm_net_params.argtypes = [vp, vp, ci]
    lib.lmm_net_forward.argtypes = [vp, vp, vp]
    lib.lmm_net_save.argtypes = [vp, C.c_char_p]
    lib.lmm_net_load.argtypes = [vp, C.c_char_p]
    lib.lmm_net_gradients.argtypes = [vp, vp, vp, vp]
    lib.lmm_net_train_step.argtypes = [vp, vp, vp, C.c_float, vp]
    lib.lmm_stokes_set_net.argtypes = [vp, vp]
    lib.lmm_learned_make_pairs.argtypes = [vp, C.c_ulonglong, ci, vp, vp]
    lib.lmm_learned_eval.argtypes = [vp, C.c_ulonglong, P(C.c_double)]
    lib.lmm_learned_stats.argtypes = [vp, P(ci), P(ci)]
    lib.lmm_ensemble_solve.argtypes = [ci, P(abi.Knobs), ci, P(abi.EnsembleItem), ci, ci]
    lib.lmm_ensemble_create.argtypes = [ci, P(abi.Knobs), ci, P(abi.EnsembleItem), ci, ci, P(vp)]
    lib.lmm_ensemble_run.argtypes = [vp, P(abi.EnsembleItem), ci]
    lib.lmm_ensemble_destroy.argtypes = [vp]
    lib.lmm_stokes_create_batch.argtypes = [P(abi.Grid), P(abi.Knobs), ci, ci, P(vp)]
    lib.lmm_stokes_solve_batch.argtypes = [vp, P(abi.EnsembleItem), ci]
    lib.lmm_stochastic_rhs.argtypes = [ci, P(ci), C.c_double, C.c_double, C.c_double, _dp, _dpp, C.c_ulonglong, _dpp, vp]
    lib.lmm_inner_prod_noalloc.argtypes = [C.c_int, P(C.c_int), _dpp, _dp, _dpp, _dp, C.c_double, C.c_void_p, _dp]
    lib.lmm_op_num_levels.argtypes = [C.c_void_p]
    lib.lmm_kernel_launches.restype = C.c_int64
    lib.lmm_time_op.argtypes = [C.c_void_p, C.c_int, C.c_int, P(C.c_double)]
    lib.lmm_autotune_report.argtypes = [C.c_char_p, C.c_int]
    lib.lmm_autotune_report.restype = C.c_int
    _lib = lib
    return lib


def strerror(code: int) -> str:
    return load().lmm_strerror(int(code)).decode()


class LmmError(RuntimeError):
    """Raised for negative status codes (the reference's bl_error sites)."""

    def __init__(self, code: int, where: str = ""):
        self.code = code
        super().__init__(f"{where}: status {code}: {strerror(code)}")


def check(code: int, where: str = "") -> int:
    if code < 0:
        raise LmmError(code, where)
    return code
