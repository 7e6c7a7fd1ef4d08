"""The bounds-check build (liblmmstokes_bc.so, -DLMM_BOUNDS_CHECK): every
stencil load tests its address against the registered device allocations.

The same fixed set of solves and operator calls (tests/bounds_worker.py:
FP64, mixed and reference-GMRES solves, a wall-bounded channel, 2D P1, the
learned stage, the operator entry points, the no-allocation inner product,
a batched ensemble) runs once with each library in a child process.  Every
call must return without LMM_ERR_BOUNDS, and the checked build must give the
default build's results: bitwise for the FP64 paths, whose arithmetic the
checks do not touch."""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BC_LIB = os.path.join(ROOT, "lowmachmixtures_b200", "liblmmstokes_bc.so")


def _run(tmp_path, bounds_check):
    out = str(tmp_path / ("bc.npz" if bounds_check else "plain.npz"))
    env = dict(os.environ, LMM_BOUNDS_CHECK="1" if bounds_check else "0")
    r = subprocess.run([sys.executable, os.path.join(HERE, "bounds_worker.py"), out], env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    d = dict(np.load(out))
    d["log"] = np.array(r.stdout[-4000:])
    return d


def test_bounds_checked_build_reports_nothing_and_matches(tmp_path):
    assert os.path.exists(BC_LIB), "build it with `python -m lowmachmixtures_b200.build --bounds-check`"
    bc = _run(tmp_path, True)
    plain = _run(tmp_path, False)
    assert str(bc["library"]) == "liblmmstokes_bc.so" and str(plain["library"]) == "liblmmstokes.so"
    # every solve and call of the checked run: LMM_OK, in particular no LMM_ERR_BOUNDS (-8)
    assert (bc["status"] == 0).all(), (bc["status"], str(bc["log"]))
    assert (plain["status"] == 0).all(), (plain["status"], str(plain["log"]))
    assert set(bc) == set(plain)
    for k in sorted(bc):
        if k in ("library", "status", "log"):
            continue
        if k.startswith(("plain64", "reference", "walls", "p1_2d", "ops_", "noalloc")):
            np.testing.assert_array_equal(bc[k], plain[k], err_msg=k)
        else:  # FP32 preconditioner paths: FMA contraction may differ
            np.testing.assert_allclose(bc[k], plain[k], rtol=0, atol=1e-6 * max(np.abs(plain[k]).max(), 1e-300), err_msg=k)
