"""lmm_inner_prod_noalloc (include/lmm_noalloc.h): the weighted Stokes inner
product with its scratch in a static device array, for callers that cannot
allocate device memory where they need an inner product.  The GPU tests
compare it bit for bit with lmm_op_inner_prod (same kernel, same block
count, same weights) on the same device arrays, on two calls in a row, and
check that the device's free memory does not change across a call; the CPU
tests check the argument and size rejections, which return before any CUDA
call."""
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


# the largest accepted grid is 2^31 - 1 - 592 * 256 cells: the reduction's
# 32-bit grid-stride index must not wrap
MAX_CELLS = 2 ** 31 - 1 - 592 * 256


@pytest.mark.parametrize("n,code", [((2 ** 16, 2 ** 16, 2), abi.LMM_ERR_TOO_LARGE), ((0, 8, 8), abi.LMM_ERR_INVALID),
                                    ((MAX_CELLS + 1, 1, 1), abi.LMM_ERR_TOO_LARGE),
                                    ((2 ** 31 - 1, 1, 1), abi.LMM_ERR_TOO_LARGE)])
def test_rejects_before_any_device_work(n, code):
    lib = _lib()
    arr = (_dp * 3)(_fake(), _fake(), _fake())
    nn = (C.c_int * 3)(*n)
    out = (C.c_double * 6)()
    assert lib.lmm_inner_prod_noalloc(3, nn, arr, _fake(), arr, _fake(), 1.0, None, out) == code
    assert lib.lmm_inner_prod_noalloc(4, nn, arr, _fake(), arr, _fake(), 1.0, None, out) == abi.LMM_ERR_INVALID
    assert b"fixed-size" in lib.lmm_strerror(abi.LMM_ERR_TOO_LARGE)
    if code == abi.LMM_ERR_INVALID:
        assert b"lmm_inner_prod_noalloc" in lib.lmm_strerror(code)


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
    for call in range(2):
        free0 = torch.cuda.mem_get_info()[0]
        rc, out = _call(lib, dm, n, a_u, a_p, b_u, b_p, pw, stream)
        assert rc == abi.LMM_OK, lib.lmm_strerror(rc)
        if call == 1:  # after the first call's set-up nothing is allocated
            assert torch.cuda.mem_get_info()[0] == free0
        np.testing.assert_array_equal(out[: dm + 1], ref)
        total = sum(out[:dm]) + pw * pw * out[dm]
        np.testing.assert_allclose(out[4], total, rtol=1e-13)
    # a == b: out[5] is the norm, sqrt(|u|^2 + (p_norm_weight |p|)^2) with
    # |u| = sqrt(sum of face sums), |p| = sqrt(cell sum) (both entry points
    # are built without contraction, so the expression below is exact)
    for _ in range(2):
        rc, out = _call(lib, dm, n, a_u, a_p, a_u, a_p, pw, stream)
        assert rc == abi.LMM_OK, lib.lmm_strerror(rc)
        su = 0.0
        for c in range(dm):
            su = su + out[c]
        nu, npr = np.sqrt(su), pw * np.sqrt(out[dm])
        assert out[5] == np.sqrt(nu * nu + npr * npr)
        np.testing.assert_allclose(out[5] ** 2, out[4], rtol=1e-14)
