"""CPU-side checks of the C ABI: the library loads and exports every symbol
declared in include/*.h, the ctypes structs match the C layout, the
knob defaults mirror probin_gmres.f90, and create() fails cleanly without a
GPU (no compute calls are made here)."""
import ctypes as C
import os
import re

import pytest

from lowmachmixtures_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = sorted(os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h"))


def declared_functions():
    src = "".join(open(h).read() for h in HEADERS)
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(lmm_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from lowmachmixtures_b200 import build, _native
    build.build()
    return _native.load()


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), f"{name} not exported"


def test_bounds_check_library_exports_the_same_symbols():
    """liblmmstokes_bc.so (build.py --bounds-check) is a drop-in for the
    default library: every declared entry point, and the status code its
    checks return"""
    from lowmachmixtures_b200 import build
    path = build.build(bounds_check=True)
    bc = C.CDLL(path)
    for name in declared_functions():
        assert hasattr(bc, name), f"{name} not exported by {os.path.basename(path)}"
    bc.lmm_strerror.restype = C.c_char_p
    assert b"registered allocations" in bc.lmm_strerror(abi.LMM_ERR_BOUNDS)


def test_struct_layout_matches_c(lib):
    # sizes of the C structs, computed by the C compiler
    src = r'''
#include "lmm_stokes.h"
#include "lmm_ensemble.h"
#include <stdio.h>
int main(){printf("%zu %zu %zu %zu %zu %zu\n", sizeof(lmm_grid), sizeof(lmm_knobs), sizeof(lmm_fields_in),
 sizeof(lmm_fields_out), sizeof(lmm_stats), sizeof(lmm_ensemble_item)); return 0;}
'''
    import subprocess
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    sizes = [int(v) for v in out]
    assert sizes == [C.sizeof(abi.Grid), C.sizeof(abi.Knobs), C.sizeof(abi.FieldsIn), C.sizeof(abi.FieldsOut),
                     C.sizeof(abi.Stats), C.sizeof(abi.EnsembleItem)]


def test_default_knobs_mirror_probin_gmres(lib):
    k = abi.Knobs()
    lib.lmm_default_knobs(C.byref(k))
    ref = abi.make_knobs()
    for name, _ in abi._KNOB_FIELDS:
        if name == "reserved":
            continue
        assert getattr(k, name) == getattr(ref, name), name
    # src_gmres/probin_gmres.f90:119-157
    assert (k.precon_type, k.gmres_max_inner, k.gmres_max_outer, k.gmres_max_iter) == (1, 5, 20, 100)
    assert (k.stag_mg_nsmooths_down, k.stag_mg_nsmooths_up, k.stag_mg_nsmooths_bottom) == (2, 2, 8)
    assert k.gmres_rel_tol == 1e-9 and k.stag_mg_smoother == 1


def test_oracle_default_knobs_agree(oracle):
    k = abi.Knobs()
    oracle.lib().orc_default_knobs(C.byref(k))
    ref = abi.make_knobs()
    for name, _ in abi._KNOB_FIELDS:
        if name != "reserved":
            assert getattr(k, name) == getattr(ref, name), name


def test_create_rejects_bad_arguments_without_gpu(lib):
    g = abi.make_grid(3, (32, 32, 32), 1.0 / 32)
    k = abi.make_knobs(precon_type=7)
    h = C.c_void_p()
    assert lib.lmm_stokes_create(C.byref(g), C.byref(k), 0, C.byref(h)) == abi.LMM_ERR_INVALID
    k = abi.make_knobs(visc_type=-2)
    g.bc_lo[0] = 0  # not periodic
    assert lib.lmm_stokes_create(C.byref(g), C.byref(k), 0, C.byref(h)) == abi.LMM_ERR_INVALID
    g = abi.make_grid(2, (96, 96), 1.0 / 96)
    k = abi.make_knobs(visc_schur_approx=1, visc_type=3)  # inverse_diag_lap has no |visc_type| = 3
    assert lib.lmm_stokes_create(C.byref(g), C.byref(k), 0, C.byref(h)) == abi.LMM_ERR_INVALID
    assert lib.lmm_strerror(abi.LMM_ERR_BREAKDOWN) == b"gmres: error in orthogonalization"


def test_batch_entry_points_reject_bad_arguments_without_gpu(lib):
    """lmm_stokes_create_batch checks its grid and knobs before touching a
    device; lmm_stokes_solve_batch refuses a null or non-batch handle"""
    g2 = abi.make_grid(2, (32, 32), 1.0 / 32)
    ok = dict(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES)
    h = C.c_void_p()
    bad = [
        (abi.make_grid(3, (16, 16, 16), 1.0 / 16), abi.make_knobs(**ok), 4),           # 3D
        (g2, abi.make_knobs(**dict(ok, visc_type=2)), 4),                             # constant coefficients
        (g2, abi.make_knobs(**dict(ok, method=abi.LMM_METHOD_GMRES)), 4),             # left-preconditioned GMRES
        (g2, abi.make_knobs(**dict(ok, scale_factor=2.0)), 4),
        (g2, abi.make_knobs(**dict(ok, gmres_max_inner=46)), 4),
        (g2, abi.make_knobs(**ok), 0),                                                 # empty batch
    ]
    for g, k, b in bad:
        assert lib.lmm_stokes_create_batch(C.byref(g), C.byref(k), b, 0, C.byref(h)) == abi.LMM_ERR_INVALID
        assert not h.value
    items = (abi.EnsembleItem * 1)()
    assert lib.lmm_stokes_solve_batch(None, items, 1) == abi.LMM_ERR_INVALID
