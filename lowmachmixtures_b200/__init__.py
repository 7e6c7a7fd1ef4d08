"""lowmachmixtures_b200 - B200-native staggered-grid Stokes solver.

A drop-in for the gmres(...) path of LowMachMixtures (src_gmres/gmres.f90):
restarted GMRES with the block preconditioner (staggered geometric multigrid
for the face velocities, a cell-centred multigrid for the pressure Schur
complement), every hot operator a hand-written sm_100a CUDA kernel in
liblmmstokes.so.  The C ABI is include/lmm_stokes.h; this package is its
Python host side.
"""
from . import abi  # noqa: F401
from .abi import KNOB_DEFAULTS, make_knobs  # noqa: F401


def __getattr__(name):
    # the CUDA library is loaded lazily so that CPU-only tools can import abi
    if name in ("StokesSolver", "gmres", "LmmError"):
        from . import gmres as _g
        return getattr(_g, name)
    raise AttributeError(name)
