"""lmm_inner_prod_noalloc (include/lmm_noalloc.h): the weighted Stokes inner
product with its scratch in a static device array.  The GPU tests compare it
with lmm_op_inner_prod on the same device arrays, on two calls in a row; the
CPU tests check the argument and size rejections, which return before any
CUDA call."""
import ctypes as C

import numpy as np
import pytest

from lowmachmixtures_b200 import abi

_dp = C.POINTER(C.c_double)


def _lib():
    from lowmachmixtures_b200 import _native
    return _native.load()


def _call(lib, dm, n, a_u, a_p, b_u, b_p, pw, stream=None):
    nn = (C.c_int * 3)(*(list(n) + [1] * (3 - len(n))))
    out = (C.c_double * 6)()
    rc = lib.lmm_inner_prod_noalloc(dm, nn, abi.ptr_array(a_u), abi.ptr(a_p), abi.ptr_array(b_u), abi.ptr(b_p),
                                    pw, stream, out)
    return rc, list(out)


def _fake(addr=4096):
    # non-null pointers that the entry point must never touch (it rejects
    # the call before any CUDA work)
    return C.cast(C.c_void_p(addr), _dp)


@pytest.mark.parametrize("n,code", [((2 ** 16, 2 ** 16, 2), abi.LMM_ERR_TOO_LARGE), ((0, 8, 8), abi.LMM_ERR_INVALID)])
def test_rejects_before_any_device_work(n, code):
    lib = _lib()
    arr = (_dp * 3)(_fake(), _fake(), _fake())
    nn = (C.c_int * 3)(*n)
    out = (C.c_double * 6)()
    assert lib.lmm_inner_prod_noalloc(3, nn, arr, _fake(), arr, _fake(), 1.0, None, out) == code
    assert lib.lmm_inner_prod_noalloc(4, nn, arr, _fake(), arr, _fake(), 1.0, None, out) == abi.LMM_ERR_INVALID
    assert b"fixed-size" in lib.lmm_strerror(abi.LMM_ERR_TOO_LARGE)


@pytest.mark.gpu
@pytest.mark.parametrize("dm,n", [(3, (32, 16, 8)), (2, (64, 32)), (3, (128, 128, 128))])
def test_matches_handle_entry_point_twice(dm, n):
    import torch

    from lowmachmixtures_b200.gmres import StokesSolver

    lib = _lib()
    rng = np.random.Generator(np.random.PCG64(7))
    shape = tuple(reversed(n))
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    a_u = [dev(rng.standard_normal(shape)) for _ in range(dm)]
    b_u = [dev(rng.standard_normal(shape)) for _ in range(dm)]
    a_p, b_p = dev(rng.standard_normal(shape)), dev(rng.standard_normal(shape))
    pw = 1.0
    with StokesSolver(dm, n, 1.0 / n[0], knobs=abi.make_knobs(p_norm_weight=pw)) as s:
        ref = s.inner_prod(a_u, a_p, b_u, b_p)
    torch.cuda.synchronize()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        rc, out = _call(lib, dm, n, a_u, a_p, b_u, b_p, pw, stream)
        assert rc == abi.LMM_OK, lib.lmm_strerror(rc)
        np.testing.assert_allclose(out[: dm + 1], ref, rtol=1e-13, atol=0)
        total = sum(out[:dm]) + pw * pw * out[dm]
        np.testing.assert_allclose(out[4], total, rtol=1e-13)
