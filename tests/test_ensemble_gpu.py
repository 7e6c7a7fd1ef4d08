"""lmm_ensemble_solve and batches of 2D problems (lmm_stokes_solve_batch):
independent problems of uneven sizes give the same bits, iteration counts
and residual histories as one lmm_stokes_solve_device call per instance,
and every instance meets its tolerance -- whether the ensemble runs them in
batches (one launch per operation for all problems of a grid) or through
the worker pool of one-problem handles."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _single(p, kn):
    """one problem on a one-problem handle: (x_u, x_p, stats)"""
    import torch

    from lowmachmixtures_b200.gmres import StokesSolver
    with StokesSolver(2, p.n[:2], p.dx, knobs=kn, bc=getattr(p, "bc", None)) as s:
        yp = torch.zeros(p.shape, dtype=torch.float64, device="cuda")
        yu = [torch.zeros_like(yp) for _ in range(2)]
        _, _, st = s.solve_device([_dev(a) for a in p.b_u], _dev(p.b_p), yu, yp, [_dev(a) for a in p.alpha_fc], _dev(p.beta),
                                  [_dev(a) for a in p.beta_ed], _dev(p.gamma), p.theta_alpha)
    return yu, yp, st


def _assert_same_as_single(probs, sols, stats, kn):
    import torch
    for p, (xu, xp), s in zip(probs, sols, stats):
        yu, yp, st1 = _single(p, kn)
        for c in range(2):
            assert torch.equal(xu[c], yu[c])
        assert torch.equal(xp, yp)
        assert s["total_iter"] == st1["total_iter"]
        assert s["history"] == st1["history"]


@pytest.mark.parametrize("precision,theta,ortho", [(1, 0.0, 0), (1, 25.0, 0), (0, 0.0, 0), (0, 25.0, 0), (1, 0.0, 1), (0, 25.0, 1)])
def test_batched_ensemble_equals_individual_solves(precision, theta, ortho):
    """ortho: 0 modified, 1 classical Gram-Schmidt (one pass for all
    projections, one for the update and the norm)"""
    from lowmachmixtures_b200 import abi, ensemble
    probs = ensemble.make_instances(12, seed=5, sizes=(32, 48, 64, 96), theta_alpha=theta)
    kn = abi.make_knobs(precon_type=2 if theta == 0.0 else 1, visc_type=-2, method=abi.LMM_METHOD_FGMRES, precision=precision,
                        gmres_rel_tol=1e-8, orthogonalization=ortho)
    st, stats, sols, _ = ensemble.solve(probs, kn, workers=4)
    assert all(s == 0 for s in st)
    for s in stats:
        assert s["norm_resid_true"] <= 1e-8 * s["norm_b"]
    _assert_same_as_single(probs, sols, stats, kn)


def test_worker_pool_equals_individual_solves():
    from lowmachmixtures_b200 import abi, ensemble
    probs = ensemble.make_instances(8, seed=7, sizes=(32, 48, 64))
    for kn in (abi.make_knobs(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_GMRES, gmres_rel_tol=1e-8),
               abi.make_knobs(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES, precision=abi.LMM_PRECISION_FP32,
                              gmres_rel_tol=1e-8, ensemble_batch=-1)):
        st, stats, sols, _ = ensemble.solve(probs, kn, workers=3)
        assert all(s == 0 for s in st)
        _assert_same_as_single(probs, sols, stats, kn)


def test_batch_handle_padding_repeats_and_zero_rhs():
    """fewer problems than the handle holds, twice on one handle, one problem
    with a zero right-hand side (x = 0 at once)"""
    from lowmachmixtures_b200 import _native, abi, ensemble, synth
    lib = _native.load()
    probs = [synth.make_problem(2, 64, 10.0 ** (1 + i / 3), 300 + i) for i in range(5)]
    probs[2].b_u = [np.zeros_like(a) for a in probs[2].b_u]
    kn = abi.make_knobs(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES, precision=abi.LMM_PRECISION_FP32,
                        gmres_rel_tol=1e-9)
    h = C.c_void_p()
    assert lib.lmm_stokes_create_batch(C.byref(abi.make_grid(2, (64, 64), 1 / 64)), C.byref(kn), 8, 0, C.byref(h)) == 0
    try:
        for _ in range(2):
            items, keep, sols = ensemble._items(probs, 0)
            assert lib.lmm_stokes_solve_batch(h, items, len(probs)) == 0
            assert all(it.status == 0 for it in items)
            assert all(float(x.abs().max()) == 0.0 for x in sols[2][0])
            assert items[2].stats.total_iter == 0
            live = [i for i in range(len(probs)) if i != 2]
            _assert_same_as_single([probs[i] for i in live], [sols[i] for i in live],
                                   [items[i].stats.as_dict() for i in live], kn)
    finally:
        lib.lmm_stokes_destroy(h)


def test_batch_handle_rejects_what_it_does_not_cover():
    from lowmachmixtures_b200 import _native, abi, ensemble, synth
    lib = _native.load()
    ok = dict(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES)
    g2 = abi.make_grid(2, (32, 32), 1 / 32)
    h = C.c_void_p()
    for g, kn in ((abi.make_grid(3, (16, 16, 16), 1 / 16), abi.make_knobs(**ok)),
                  (g2, abi.make_knobs(**dict(ok, visc_type=2))),
                  (g2, abi.make_knobs(**dict(ok, method=abi.LMM_METHOD_GMRES))),
                  (g2, abi.make_knobs(**dict(ok, stag_mg_max_vcycles=2)))):
        assert lib.lmm_stokes_create_batch(C.byref(g), C.byref(kn), 4, 0, C.byref(h)) == abi.LMM_ERR_INVALID
    assert lib.lmm_stokes_create_batch(C.byref(g2), C.byref(abi.make_knobs(**ok)), 2, 0, C.byref(h)) == 0
    try:
        p = synth.make_problem(2, 32, 10.0, 1)
        q = synth.make_problem(2, 64, 10.0, 2)
        items, keep, sols = ensemble._items([p, p, p], 0)
        assert lib.lmm_stokes_solve_batch(h, items, 3) == abi.LMM_ERR_INVALID   # more than the handle holds
        items, keep, sols = ensemble._items([p, q], 0)
        assert lib.lmm_stokes_solve_batch(h, items, 2) == abi.LMM_ERR_INVALID   # another grid
        # a one-problem entry point refuses the batch handle
        fin, fout = abi.FieldsIn(), abi.FieldsOut()
        th, npr, st = C.c_double(0.0), C.c_double(0.0), abi.Stats()
        assert lib.lmm_stokes_solve_device(h, C.byref(fin), C.byref(fout), C.byref(th), C.byref(npr),
                                           C.byref(st)) == abi.LMM_ERR_INVALID
    finally:
        lib.lmm_stokes_destroy(h)


@pytest.mark.parametrize("n,count,ortho", [(128, 64, 0), (256, 48, 1)])
def test_large_batch_handle(n, count, ortho):
    """Arenas of one to two gigabytes: the handle's buffers are zeroed in
    stream order before its pointer tables are written; 48 problems of 256^2
    with classical Gram-Schmidt need more reduction partials than one
    problem does"""
    from lowmachmixtures_b200 import _native, abi, ensemble, synth
    lib = _native.load()
    probs = [synth.make_problem(2, n, 10.0 ** (1 + (i % 7) / 3), 900 + i) for i in range(count)]
    kn = abi.make_knobs(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES, precision=abi.LMM_PRECISION_FP32,
                        gmres_rel_tol=1e-8, orthogonalization=ortho)
    h = C.c_void_p()
    assert lib.lmm_stokes_create_batch(C.byref(abi.make_grid(2, (n, n), 1 / n)), C.byref(kn), count, 0, C.byref(h)) == 0
    try:
        items, keep, sols = ensemble._items(probs, 0)
        assert lib.lmm_stokes_solve_batch(h, items, count) == 0
        assert all(it.status == 0 for it in items)
        assert all(it.stats.norm_resid_true <= 1e-8 * it.stats.norm_b for it in items)
        pick = [0, count // 2, count - 1]
        _assert_same_as_single([probs[i] for i in pick], [sols[i] for i in pick], [items[i].stats.as_dict() for i in pick], kn)
    finally:
        lib.lmm_stokes_destroy(h)


def test_batch_statuses_per_problem():
    """A problem with a non-finite right-hand side fails alone
    (LMM_ERR_NONFINITE); under a tight iteration limit each problem stops
    with its own status (converged or LMM_WARN_MAX_ITER), and every
    problem's bits and status are those of its one-problem solve."""
    import torch

    from lowmachmixtures_b200 import _native, abi, ensemble, synth
    from lowmachmixtures_b200.gmres import StokesSolver
    lib = _native.load()
    probs = [synth.make_problem(2, 64, 10.0 ** (1 + i / 2), 500 + i) for i in range(5)]
    probs[1].b_u[0] = probs[1].b_u[0].copy()
    probs[1].b_u[0][3, 5] = np.nan
    kn = abi.make_knobs(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES, precision=abi.LMM_PRECISION_FP32,
                        gmres_rel_tol=1e-10, gmres_max_iter=9)
    h = C.c_void_p()
    assert lib.lmm_stokes_create_batch(C.byref(abi.make_grid(2, (64, 64), 1 / 64)), C.byref(kn), 5, 0, C.byref(h)) == 0
    try:
        items, keep, sols = ensemble._items(probs, 0)
        rc = lib.lmm_stokes_solve_batch(h, items, 5)
        assert rc == abi.LMM_ERR_NONFINITE
        assert items[1].status == abi.LMM_ERR_NONFINITE
        statuses = set()
        for q in (0, 2, 3, 4):
            p = probs[q]
            with StokesSolver(2, p.n[:2], p.dx, knobs=kn) as s:
                yp = torch.zeros(p.shape, dtype=torch.float64, device="cuda")
                yu = [torch.zeros_like(yp) for _ in range(2)]
                fin = s._fields([_dev(a) for a in p.b_u], _dev(p.b_p), [_dev(a) for a in p.alpha_fc], _dev(p.beta),
                                [_dev(a) for a in p.beta_ed], _dev(p.gamma), abi.LMM_LAYOUT_COMPACT, None)
                fout = abi.FieldsOut()
                fout.x_u = abi.ptr_array(yu)
                fout.x_p = abi.ptr(yp)
                fout.layout = abi.LMM_LAYOUT_COMPACT
                th, npr, st = C.c_double(p.theta_alpha), C.c_double(0.0), abi.Stats()
                rc1 = lib.lmm_stokes_solve_device(s._h, C.byref(fin), C.byref(fout), C.byref(th), C.byref(npr), C.byref(st))
            assert items[q].status == rc1
            statuses.add(rc1)
            assert items[q].stats.total_iter == st.total_iter
            xu, xp = sols[q]
            for c in range(2):
                assert torch.equal(xu[c], yu[c])
            assert torch.equal(xp, yp)
        assert abi.LMM_WARN_MAX_ITER in statuses
    finally:
        lib.lmm_stokes_destroy(h)


def test_batch_handle_update_knobs():
    """lmm_stokes_update_knobs on a live batch handle: a tighter tolerance
    gives each problem the solve of a fresh one-problem handle with it"""
    from lowmachmixtures_b200 import _native, abi, ensemble, synth
    lib = _native.load()
    probs = [synth.make_problem(2, 48, 10.0 ** (1 + i / 2), 700 + i) for i in range(3)]
    kn = abi.make_knobs(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES, precision=abi.LMM_PRECISION_FP32,
                        gmres_rel_tol=1e-6)
    h = C.c_void_p()
    assert lib.lmm_stokes_create_batch(C.byref(abi.make_grid(2, (48, 48), 1 / 48)), C.byref(kn), 3, 0, C.byref(h)) == 0
    try:
        items, keep, sols = ensemble._items(probs, 0)
        assert lib.lmm_stokes_solve_batch(h, items, 3) == 0
        loose = [it.stats.total_iter for it in items]
        tight = abi.make_knobs(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES, precision=abi.LMM_PRECISION_FP32,
                               gmres_rel_tol=1e-10)
        assert lib.lmm_stokes_update_knobs(h, C.byref(tight)) == 0
        items, keep, sols = ensemble._items(probs, 0)
        assert lib.lmm_stokes_solve_batch(h, items, 3) == 0
        assert all(it.stats.total_iter > q for it, q in zip(items, loose))
        _assert_same_as_single(probs, sols, [it.stats.as_dict() for it in items], tight)
    finally:
        lib.lmm_stokes_destroy(h)


@pytest.mark.parametrize("bc", [(-1, 100), (100, 200), (100, 100)])
@pytest.mark.parametrize("precision", [1, 0])
def test_batch_with_walls(bc, precision):
    """2D batches on grids with walls (no-slip 100, slip 200, periodic -1 per
    direction): the bits of one-problem solves"""
    from lowmachmixtures_b200 import _native, abi, ensemble, synth
    lib = _native.load()
    n = 32
    probs = [synth.make_problem(2, n, 10.0 ** (1 + i / 2), 800 + i, bc=bc) for i in range(4)]
    kn = abi.make_knobs(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES, precision=precision, gmres_rel_tol=1e-9)
    h = C.c_void_p()
    assert lib.lmm_stokes_create_batch(C.byref(abi.make_grid(2, (n, n), 1 / n, bc=bc)), C.byref(kn), 4, 0, C.byref(h)) == 0
    try:
        items, keep, sols = ensemble._items(probs, 0)
        assert lib.lmm_stokes_solve_batch(h, items, 4) == 0
        assert all(it.status == 0 for it in items)
        _assert_same_as_single(probs, sols, [it.stats.as_dict() for it in items], kn)
    finally:
        lib.lmm_stokes_destroy(h)


@pytest.mark.parametrize("visc", [-1, -3])
@pytest.mark.parametrize("precon", [1, 4, 3, 5, -2])
def test_batch_other_viscous_operators(visc, precon):
    """visc_type -1 and -3 (gamma enters the operator and the Schur step),
    the other preconditioner types, theta_alpha > 0: the bits of one-problem
    solves"""
    from lowmachmixtures_b200 import _native, abi, ensemble, synth
    lib = _native.load()
    n = 32
    probs = [synth.make_problem(2, n, 10.0 ** (1 + i / 2), 900 + i, theta_alpha=20.0) for i in range(3)]
    kn = abi.make_knobs(precon_type=precon, visc_type=visc, method=abi.LMM_METHOD_FGMRES, precision=abi.LMM_PRECISION_FP32,
                        gmres_rel_tol=1e-9)
    h = C.c_void_p()
    assert lib.lmm_stokes_create_batch(C.byref(abi.make_grid(2, (n, n), 1 / n)), C.byref(kn), 3, 0, C.byref(h)) == 0
    try:
        items, keep, sols = ensemble._items(probs, 0)
        rc = lib.lmm_stokes_solve_batch(h, items, 3)
        assert rc >= 0
        _assert_same_as_single(probs, sols, [it.stats.as_dict() for it in items], kn)
    finally:
        lib.lmm_stokes_destroy(h)
