"""GPU parity: every CUDA kernel and the full solve against the CPU oracle.

The FP64 stencil kernels are built with -fmad=false and keep the reference's
operand order, so applyop, Gauss-Seidel colours, Jacobi, residual
restriction, prolongation, apply_matrix and whole V-cycles must be
bit-identical to the oracle.  Reductions (inner products, means) sum in a
different order: tolerance 1e-13 relative.  Full solves: velocity and
mean-removed pressure within 1e-10 relative, iteration count +-1 (the bar
the solver is held to).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lowmachmixtures_b200 import abi, synth  # noqa: E402

pytestmark = pytest.mark.gpu

VISCS = (-1, 1, -2, 2, -3, 3)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


def random_problem(dm, n, seed, visc, theta=7.0):
    rng = np.random.Generator(np.random.PCG64(seed))
    shape = (n,) * dm
    ne = 1 if dm == 2 else 3
    const = visc > 0
    p = synth.make_problem(dm, n, 10.0, seed, theta_alpha=theta)
    if const:
        p.beta = np.full(shape, 0.8)
        p.beta_ed = [np.full(shape, 0.8) for _ in range(ne)]
        p.gamma = np.full(shape, 0.3)
    else:
        p.beta = rng.uniform(0.5, 2.0, shape)
        p.beta_ed = [rng.uniform(0.5, 2.0, shape) for _ in range(ne)]
        p.gamma = rng.uniform(0.1, 0.5, shape)
    p.alpha_fc = [rng.uniform(0.5, 1.5, shape) for _ in range(dm)]
    return p, rng


def make_solver(p, **kn):
    from lowmachmixtures_b200.gmres import StokesSolver
    k = abi.make_knobs(**kn)  # knobs the oracle does not know are the library's own
    s = StokesSolver(p.dm, p.n[: p.dm], p.dx, knobs=k)
    s.load_coeffs([dev(a) for a in p.alpha_fc], dev(p.beta), [dev(b) for b in p.beta_ed], dev(p.gamma), p.theta_alpha)
    return s


@pytest.mark.parametrize("dm,n", [(2, 16), (3, 8)])
@pytest.mark.parametrize("visc", VISCS)
def test_applyop_bit_exact(oracle, dm, n, visc):
    p, rng = random_problem(dm, n, 11, visc)
    s = make_solver(p, visc_type=visc)
    phi = [rng.standard_normal(p.shape) for _ in range(dm)]
    for color in range(0, 2 * dm + 1):
        init = [rng.standard_normal(p.shape) for _ in range(dm)]
        ref = oracle.stag_applyop(p, visc, phi, color=color, Lphi=init)
        out = [dev(a) for a in init]
        s.stag_applyop([dev(a) for a in phi], out, color)
        for c in range(dm):
            np.testing.assert_array_equal(host(out[c]), ref[c], err_msg=f"colour {color} comp {c}")
    s.close()


@pytest.mark.parametrize("dm,n", [(2, 16), (3, 8)])
@pytest.mark.parametrize("visc", VISCS)
@pytest.mark.parametrize("lev", [0, 1])
def test_smooth_colours_bit_exact(oracle, dm, n, visc, lev):
    p, rng = random_problem(dm, n, 12, visc)
    k = oracle.default_knobs(visc_type=visc, stag_mg_omega=0.9)
    s = make_solver(p, visc_type=visc, stag_mg_omega=0.9)
    shp = oracle.level_shape(p, lev)
    for color in range(0, 2 * dm + 1):
        phi = [rng.standard_normal(shp) for _ in range(dm)]
        rhs = [rng.standard_normal(shp) for _ in range(dm)]
        ref = oracle.smooth(p, k, lev, rhs, phi, color)
        dphi = [dev(a) for a in phi]
        s.smooth(lev, [dev(a) for a in rhs], dphi, color)
        for c in range(dm):
            np.testing.assert_array_equal(host(dphi[c]), ref[c], err_msg=f"lev {lev} colour {color} comp {c}")
    s.close()


@pytest.mark.parametrize("dm,n", [(2, 16), (3, 16), (3, 32)])
@pytest.mark.parametrize("visc", [-1, -2, -3, 2])
@pytest.mark.parametrize("fusion", [0, 1])
def test_residual_restrict_and_prolong_bit_exact(oracle, dm, n, visc, fusion):
    """Residual restriction (split, or with residual_fusion = 1 in one pass
    through shared memory) and prolongation against the oracle, bit for bit."""
    if dm == 2 and fusion:
        pytest.skip("the fused pass is 3D")
    p, rng = random_problem(dm, n, 13, visc)
    k = oracle.default_knobs(visc_type=visc)
    s = make_solver(p, visc_type=visc, residual_fusion=fusion)
    for lev in (0, 1):
        shp = oracle.level_shape(p, lev)
        shc = oracle.level_shape(p, lev + 1)
        phi = [rng.standard_normal(shp) for _ in range(dm)]
        rhs = [rng.standard_normal(shp) for _ in range(dm)]
        ref = oracle.residual_restrict(p, k, lev, rhs, phi)
        out = [dev(np.zeros(shc)) for _ in range(dm)]
        s.residual_restrict(lev, [dev(a) for a in rhs], [dev(a) for a in phi], out)
        for c in range(dm):
            np.testing.assert_array_equal(host(out[c]), ref[c], err_msg=f"restrict lev {lev} comp {c}")
        coarse = [rng.standard_normal(shc) for _ in range(dm)]
        refp = oracle.prolong_add(p, lev, coarse, phi)
        dphi = [dev(a) for a in phi]
        s.prolong_add(lev, [dev(a) for a in coarse], dphi)
        for c in range(dm):
            np.testing.assert_array_equal(host(dphi[c]), refp[c], err_msg=f"prolong lev {lev} comp {c}")
    s.close()


# tail: (tail_cells, tail_smem_kb): -1 = every level by per-level kernels;
# otherwise the coarse levels run in one single-block shared-memory launch
TAILS = [(-1, 0), (0, 0), (64, 0), (0, 24)]


@pytest.mark.parametrize("dm,n", [(2, 32), (3, 16), (3, 32)])
@pytest.mark.parametrize("visc", [-1, -2, -3])
@pytest.mark.parametrize("smoother", [1, 0])
@pytest.mark.parametrize("tail", TAILS)
def test_vcycle_bit_exact(oracle, dm, n, visc, smoother, tail):
    p, rng = random_problem(dm, n, 14, visc, theta=3.0)
    kn = dict(visc_type=visc, stag_mg_smoother=smoother, stag_mg_omega=1.0 if smoother else 0.7)
    k = oracle.default_knobs(**kn)
    s = make_solver(p, **kn, tail_cells=tail[0], tail_smem_kb=tail[1])
    rhs = [rng.standard_normal(p.shape) for _ in range(dm)]
    ref = oracle.stag_mg_solver(p, k, rhs)
    phi = [dev(np.zeros(p.shape)) for _ in range(dm)]
    s.stag_mg_solver([dev(a) for a in rhs], phi)
    for c in range(dm):
        np.testing.assert_array_equal(host(phi[c]), ref[c])
    s.close()


@pytest.mark.parametrize("n", [16, 32, 64])
@pytest.mark.parametrize("visc", VISCS)
@pytest.mark.parametrize("fusion", [0, 1, 2, 4])
def test_vcycle_fused_smoother_bit_exact(oracle, n, visc, fusion):
    """One launch per colour (0; the launches alternate their plane order),
    both colours of a component in one out-of-place launch (1) and the same
    with 2 or 4 planes per block all reproduce the reference's
    colour-by-colour Gauss-Seidel bit for bit (fusion 0 also with the
    residual and restriction fused)."""
    p, rng = random_problem(3, n, 17, visc, theta=3.0)
    kn = dict(visc_type=visc)
    k = oracle.default_knobs(**kn)
    s = make_solver(p, **kn, tail_cells=-1, smoother_fusion=fusion, residual_fusion=1 if fusion == 0 else 0)
    rhs = [rng.standard_normal(p.shape) for _ in range(3)]
    ref = oracle.stag_mg_solver(p, k, rhs)
    phi = [dev(np.zeros(p.shape)) for _ in range(3)]
    s.stag_mg_solver([dev(a) for a in rhs], phi)
    for c in range(3):
        np.testing.assert_array_equal(host(phi[c]), ref[c])
    s.close()


# (rows per tile, k-slabs): 1 / 0 = the library's choice; tiles whose rows wrap
# around the periodic y boundary, one-tile rows (TY = n) and slabs of one
# plane are all among them.  FP64 tilings instantiated per row length:
TMA_FP64 = {128: (4,), 64: (8, 4), 32: (8, 16)}
TMA_TILINGS = [(1, 0), (8, 1), (8, 5), (4, 16), (16, 3)]


@pytest.mark.parametrize("n", [32, 64])
@pytest.mark.parametrize("visc", [-1, -2, -3])
@pytest.mark.parametrize("tiling", TMA_TILINGS)
def test_vcycle_tma_smoother_bit_exact(oracle, n, visc, tiling):
    """Both Gauss-Seidel colours of a component in one launch with every
    operand staged in shared memory by TMA, marching through k-slabs,
    reproduce the reference's colour-by-colour smoother bit for bit
    (stag_mg_solver.f90:363-401) inside a whole V-cycle."""
    ty, slabs = tiling
    if ty > 1 and ty not in TMA_FP64[n]:
        pytest.skip("tiling not instantiated for this row length")
    p, rng = random_problem(3, n, 19, visc, theta=3.0)
    kn = dict(visc_type=visc)
    k = oracle.default_knobs(**kn)
    s = make_solver(p, **kn, tail_cells=-1, smoother_tma=ty, smoother_tma_slabs=slabs, smoother_tma_cells=1)
    rhs = [rng.standard_normal(p.shape) for _ in range(3)]
    ref = oracle.stag_mg_solver(p, k, rhs)
    phi = [dev(np.zeros(p.shape)) for _ in range(3)]
    s.stag_mg_solver([dev(a) for a in rhs], phi)
    for c in range(3):
        np.testing.assert_array_equal(host(phi[c]), ref[c])
    s.close()


def test_tma_smoother_fp32_solve_matches_colour_launches():
    """The mixed method with the TMA smoother on its FP32 levels and with one
    launch per colour: both reach the FP64 tolerance, the same iteration
    count within one and solutions within 1e-8 of each other (FP32
    preconditioners, no bit parity asked)."""
    from lowmachmixtures_b200.gmres import StokesSolver
    prob = synth.config_3d_128(5, n=64)
    outs = []
    for tma in (1, -1):
        kn = abi.make_knobs(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES, precision=abi.LMM_PRECISION_FP32,
                            smoother_tma=tma)
        xu, xp = prob.zeros_like_solution()
        with StokesSolver(3, (64, 64, 64), prob.dx, knobs=kn) as s:
            _, _, st = s.solve(prob.b_u, prob.b_p, xu, xp, prob.alpha_fc, prob.beta, prob.beta_ed, prob.gamma,
                               prob.theta_alpha)
        assert st["status"] == 0 and st["norm_resid_true"] <= 1e-9 * st["norm_b"]
        outs.append((st["total_iter"], xu))
    assert abs(outs[0][0] - outs[1][0]) <= 1
    for c in range(3):
        assert np.linalg.norm(outs[0][1][c] - outs[1][1][c]) <= 1e-8 * np.linalg.norm(outs[1][1][c])


@pytest.mark.parametrize("dm,n", [(2, 32), (3, 16)])
@pytest.mark.parametrize("visc", VISCS)
def test_apply_matrix_bit_exact(oracle, dm, n, visc):
    p, rng = random_problem(dm, n, 15, visc)
    s = make_solver(p, visc_type=visc)
    xu = [rng.standard_normal(p.shape) for _ in range(dm)]
    xp = rng.standard_normal(p.shape)
    ref_u, ref_p = oracle.apply_matrix(p, visc, xu, xp)
    bu = [dev(np.zeros(p.shape)) for _ in range(dm)]
    bp = dev(np.zeros(p.shape))
    s.apply_matrix([dev(a) for a in xu], dev(xp), bu, bp)
    for c in range(dm):
        np.testing.assert_array_equal(host(bu[c]), ref_u[c])
    np.testing.assert_array_equal(host(bp), ref_p)
    s.close()


@pytest.mark.parametrize("dm,n", [(2, 16), (3, 16)])
def test_inner_products_and_means(oracle, dm, n):
    p, rng = random_problem(dm, n, 16, -2)
    s = make_solver(p, visc_type=-2)
    a = [rng.standard_normal(p.shape) for _ in range(dm)]
    b = [rng.standard_normal(p.shape) for _ in range(dm)]
    ap, bp = rng.standard_normal(p.shape), rng.standard_normal(p.shape)
    ref = oracle.inner_prod(p, a, ap, b, bp)
    got = s.inner_prod([dev(x) for x in a], dev(ap), [dev(x) for x in b], dev(bp))
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=1e-13 * max(abs(x) for x in ref))
    ref = oracle.sum_umac_press(p, a, ap)
    got = s.sum_umac_press([dev(x) for x in a], dev(ap))
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-15)
    s.close()


PRECONS = [1, -1, 2, -2, 3, -3, 4, -4, 5, -5]


@pytest.mark.parametrize("dm,n", [(2, 32), (3, 16)])
@pytest.mark.parametrize("pt", PRECONS)
@pytest.mark.parametrize("theta", [0.0, 50.0])
@pytest.mark.parametrize("tail_cells", [-1, 0])
def test_apply_precon(oracle, dm, n, pt, theta, tail_cells):
    visc = -2 if pt % 2 else -3
    p, rng = random_problem(dm, n, 17, visc, theta=theta)
    k = oracle.default_knobs(visc_type=visc, precon_type=pt)
    s = make_solver(p, visc_type=visc, precon_type=pt, tail_cells=tail_cells)
    bu = [rng.standard_normal(p.shape) for _ in range(dm)]
    bpp = rng.standard_normal(p.shape)
    ref_u, ref_p = oracle.apply_precon(p, k, bu, bpp)
    xu = [dev(np.zeros(p.shape)) for _ in range(dm)]
    xp = dev(np.zeros(p.shape))
    s.apply_precon([dev(a) for a in bu], dev(bpp), xu, xp)
    scale = max(np.abs(r).max() for r in ref_u + [ref_p])
    for c in range(dm):
        np.testing.assert_allclose(host(xu[c]), ref_u[c], rtol=0, atol=1e-12 * scale)
    np.testing.assert_allclose(host(xp), ref_p, rtol=0, atol=1e-12 * scale)
    s.close()


@pytest.mark.parametrize("dm,n", [(2, 32), (3, 16), (3, 32)])
@pytest.mark.parametrize("pt", [1, 2, -1, 5])
def test_apply_precon_uniform_density(oracle, dm, n, pt):
    """With alpha_fc the same on every face (constant density) the pressure
    multigrid takes its face coefficient as a scalar instead of reading
    three arrays; same tolerance against the oracle as the general path."""
    p, rng = random_problem(dm, n, 43, -2, theta=50.0)
    p.alpha_fc = [np.full(p.shape, 1.25) for _ in range(dm)]
    k = oracle.default_knobs(visc_type=-2, precon_type=pt)
    s = make_solver(p, visc_type=-2, precon_type=pt)
    bu = [rng.standard_normal(p.shape) for _ in range(dm)]
    bpp = rng.standard_normal(p.shape)
    ref_u, ref_p = oracle.apply_precon(p, k, bu, bpp)
    xu = [dev(np.zeros(p.shape)) for _ in range(dm)]
    xp = dev(np.zeros(p.shape))
    s.apply_precon([dev(a) for a in bu], dev(bpp), xu, xp)
    scale = max(np.abs(r).max() for r in ref_u + [ref_p])
    for c in range(dm):
        np.testing.assert_allclose(host(xu[c]), ref_u[c], rtol=0, atol=1e-12 * scale)
    np.testing.assert_allclose(host(xp), ref_p, rtol=0, atol=1e-12 * scale)
    s.close()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("uniform", [True, False])
def test_uniform_alpha_scalar_is_bitwise_neutral(precision, uniform):
    """theta*alpha the same on every face (constant density, the bench's
    case): the velocity operator takes it as a scalar (knob uniform_alpha =
    0, the default) instead of reading three face arrays -- the same bits as
    reading them (uniform_alpha = -1); with alpha varying, the arrays are
    read either way"""
    from lowmachmixtures_b200 import synth
    from lowmachmixtures_b200.gmres import StokesSolver
    p = synth.make_problem(3, 32, 100.0, 8, theta_alpha=0.1 * 32 * 32)
    if not uniform:
        rng = np.random.default_rng(3)
        p.alpha_fc = [1.0 + 0.5 * rng.random(p.shape) for _ in range(3)]
    out = []
    for ua in (0, -1):
        kn = abi.make_knobs(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES, precision=precision, uniform_alpha=ua)
        with StokesSolver(3, (32, 32, 32), p.dx, knobs=kn) as s:
            xu, xp = p.zeros_like_solution()
            _, _, st = s.solve(p.b_u, p.b_p, xu, xp, p.alpha_fc, p.beta, p.beta_ed, p.gamma, p.theta_alpha)
        assert st["status"] == 0
        out.append((xu, xp, st["history"]))
    for c in range(3):
        np.testing.assert_array_equal(out[0][0][c], out[1][0][c])
    np.testing.assert_array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]


def _solve_both(oracle, prob, **kn):
    k = oracle.default_knobs(**kn)
    rc_o, xu_o, xp_o, th_o, npr_o, st_o = oracle.solve(prob, k)
    from lowmachmixtures_b200.gmres import StokesSolver
    with StokesSolver(prob.dm, prob.n[: prob.dm], prob.dx, knobs=abi.make_knobs(**kn)) as s:
        xu, xp = prob.zeros_like_solution()
        th, npr, st = s.solve(prob.b_u, prob.b_p, xu, xp, prob.alpha_fc, prob.beta, prob.beta_ed, prob.gamma,
                              prob.theta_alpha)
    return (rc_o, xu_o, xp_o, th_o, npr_o, st_o), (st["status"], xu, xp, th, npr, st)


def _assert_solution_parity(ref, got, tol=1e-10):
    _, xu_o, xp_o, _, _, st_o = ref
    _, xu, xp, _, _, st = got
    for c in range(len(xu)):
        err = np.abs(xu[c] - xu_o[c]).max() / np.abs(xu_o[c]).max()
        assert err <= tol, f"velocity comp {c} rel err {err:.3e}"
    po = xp_o - xp_o.mean()
    pg = xp - xp.mean()
    err = np.abs(pg - po).max() / max(np.abs(po).max(), 1e-300)
    assert err <= tol, f"pressure rel err {err:.3e}"
    assert abs(st["total_iter"] - st_o["total_iter"]) <= 1, (st["total_iter"], st_o["total_iter"])


@pytest.mark.parametrize("pt", [2, 1])
@pytest.mark.parametrize("seed", [0, 1])
def test_gmres_parity_2d_64(oracle, pt, seed):
    prob = synth.config_2d_64(seed)
    ref, got = _solve_both(oracle, prob, precon_type=pt, visc_type=-2)
    assert ref[0] == got[0] == 0
    _assert_solution_parity(ref, got)
    assert abs(got[4] - ref[4]) <= 1e-12 * ref[4]  # norm_pre_rhs


@pytest.mark.parametrize("pt", [2, 1])
def test_gmres_parity_3d_inertial(oracle, pt):
    prob = synth.config_3d_128(0, n=32)
    ref, got = _solve_both(oracle, prob, precon_type=pt, visc_type=-2)
    assert ref[0] == got[0] == 0
    _assert_solution_parity(ref, got)


@pytest.mark.parametrize("method", [0, 1])
def test_gmres_parity_bench_workload_128(oracle, method):
    """The solve the benchmark times, at its full size: 3D 128^3 periodic,
    contrast 100, theta alpha dx^2 = 0.1, precon_type 2, visc_type -2, the
    seed-0 problem.  The reference's left-preconditioned GMRES (method 0)
    and FP64 FGMRES (method 1) each match the oracle's solve of the same
    method within 1e-10 in velocity and mean-removed pressure, iterations
    +-1 (gmres.f90:30-477, apply_precon.f90:197-279)."""
    prob = synth.config_3d_128(0)
    assert prob.n[:3] == (128, 128, 128)
    ref, got = _solve_both(oracle, prob, precon_type=2, visc_type=-2, method=method)
    assert ref[0] == got[0] == 0
    _assert_solution_parity(ref, got)
    if method == 1:
        assert got[5]["norm_resid_true"] <= 1e-9 * got[5]["norm_b"]


@pytest.mark.parametrize("method", [0, 1])
def test_gmres_parity_64_steady_contrast_1000(oracle, method):
    """A problem of the learned-preconditioner family: 3D 64^3, steady
    (theta = 0), viscosity contrast 1000."""
    prob = synth.config_3d_64_learned(7, contrast=1000.0)
    ref, got = _solve_both(oracle, prob, precon_type=2, visc_type=-2, method=method)
    assert ref[0] == got[0] == 0
    _assert_solution_parity(ref, got)


@pytest.mark.parametrize("visc", [-1, -3, 1])
def test_gmres_parity_other_visc_types(oracle, visc):
    prob = synth.make_problem(2, 32, 20.0, 3, theta_alpha=100.0, gamma_value=0.25)
    if visc > 0:
        prob.beta[:] = 1.3
        for b in prob.beta_ed:
            b[:] = 1.3
    ref, got = _solve_both(oracle, prob, precon_type=2, visc_type=visc)
    assert ref[0] == got[0]
    _assert_solution_parity(ref, got)


def test_gmres_scale_factor_and_jacobi(oracle):
    prob = synth.make_problem(2, 32, 10.0, 4, theta_alpha=30.0)
    ref, got = _solve_both(oracle, prob, precon_type=2, visc_type=-2, scale_factor=2.5, stag_mg_smoother=0,
                           stag_mg_omega=0.6, gmres_max_inner=8)
    assert ref[0] == got[0]
    _assert_solution_parity(ref, got)
    assert got[3] == ref[3]  # theta_alpha scaled and unscaled like the reference


def test_fgmres_fp64_parity(oracle):
    prob = synth.config_3d_128(1, n=32)
    ref, got = _solve_both(oracle, prob, precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES)
    assert ref[0] == got[0] == 0
    _assert_solution_parity(ref, got)
    assert got[5]["norm_resid_true"] <= 1e-9 * got[5]["norm_b"]


def test_fgmres_fp32_preconditioner_reaches_fp64_tolerance(oracle):
    prob = synth.config_3d_128(2, n=32)
    ref, got = _solve_both(oracle, prob, precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES,
                           precision=abi.LMM_PRECISION_FP32)
    st = got[5]
    assert got[0] == 0
    assert st["norm_resid_true"] <= 1e-9 * st["norm_b"]
    # solution error against the FP64 oracle solve (both converged to 1e-9)
    xu_o, xu = ref[1], got[1]
    err = max(np.abs(xu[c] - xu_o[c]).max() / np.abs(xu_o[c]).max() for c in range(3))
    assert err < 1e-6, err
    assert abs(st["total_iter"] - ref[5]["total_iter"]) <= 2


def test_boxlib_layout_matches_compact(oracle):
    """Host arrays laid out like BoxLib's dataptr(): ghosts, nodal hi+1 faces."""
    prob = synth.make_problem(3, 16, 10.0, 5, theta_alpha=40.0)
    from lowmachmixtures_b200.gmres import StokesSolver

    def boxlib(a, nodal, ng):
        # BoxLib single-box array: nodal directions hold n+1 entries (hi+1 is
        # the periodic copy of face 0), plus ng periodic ghost layers
        out = a
        for ax, nod in enumerate(reversed(nodal)):
            n = a.shape[ax]
            out = np.take(out, [v % n for v in range(-ng, n + nod + ng)], axis=ax)
        return np.ascontiguousarray(out)

    faces = [(1, 0, 0), (0, 1, 0), (0, 0, 1)]
    edges = [(1, 1, 0), (1, 0, 1), (0, 1, 1)]
    ng = 1
    bu = [boxlib(prob.b_u[c], faces[c], 0) for c in range(3)]
    al = [boxlib(prob.alpha_fc[c], faces[c], 0) for c in range(3)]
    be = boxlib(prob.beta, (0, 0, 0), 1)
    ga = boxlib(prob.gamma, (0, 0, 0), 1)
    bed = [boxlib(prob.beta_ed[e], edges[e], 0) for e in range(3)]
    bp = boxlib(prob.b_p, (0, 0, 0), 0)
    xu = [np.zeros_like(boxlib(prob.b_u[c], faces[c], ng)) for c in range(3)]
    xp = np.zeros_like(boxlib(prob.b_p, (0, 0, 0), ng))
    kn = dict(precon_type=2, visc_type=-2)
    with StokesSolver(3, (16, 16, 16), prob.dx, knobs=abi.make_knobs(**kn)) as s:
        s.solve(bu, bp, xu, xp, al, be, bed, ga, prob.theta_alpha, layout=abi.LMM_LAYOUT_BOXLIB,
                ng=dict(b_u=0, b_p=0, alpha_fc=0, beta=1, beta_ed=0, gamma=1, x_u=ng, x_p=ng))
        xu_c, xp_c = prob.zeros_like_solution()
        s.solve(prob.b_u, prob.b_p, xu_c, xp_c, prob.alpha_fc, prob.beta, prob.beta_ed, prob.gamma, prob.theta_alpha)
    for c in range(3):
        np.testing.assert_array_equal(xu[c], boxlib(xu_c[c], faces[c], ng))
    np.testing.assert_array_equal(xp, boxlib(xp_c, (0, 0, 0), ng))


def test_zero_rhs_returns_zero_and_nan_is_an_error():
    from lowmachmixtures_b200.gmres import StokesSolver
    from lowmachmixtures_b200._native import LmmError
    prob = synth.make_problem(2, 16, 10.0, 6, theta_alpha=5.0)
    with StokesSolver(2, (16, 16), prob.dx, precon_type=2, visc_type=-2) as s:
        xu = [np.ones(prob.shape) for _ in range(2)]
        xp = np.ones(prob.shape)
        zero = [np.zeros(prob.shape) for _ in range(2)]
        _, npr, st = s.solve(zero, np.zeros(prob.shape), xu, xp, prob.alpha_fc, prob.beta, prob.beta_ed, prob.gamma,
                             5.0)
        assert st["status"] == 0 and st["total_iter"] == 0
        assert all(np.all(a == 0) for a in xu) and np.all(xp == 0)
        bad = [b.copy() for b in prob.b_u]
        bad[0][3, 4] = np.nan
        with pytest.raises(LmmError) as ei:
            s.solve(bad, prob.b_p, xu, xp, prob.alpha_fc, prob.beta, prob.beta_ed, prob.gamma, 5.0)
        assert ei.value.code == abi.LMM_ERR_NONFINITE


@pytest.mark.parametrize("method,precision", [(0, 0), (1, 0), (1, 1)])
def test_graphs_and_tail_are_bitwise_neutral(method, precision):
    """Captured CUDA graphs and the single-block coarse tail reorder nothing:
    repeated solves with them on or off give bit-identical solutions."""
    from lowmachmixtures_b200.gmres import StokesSolver
    prob = synth.config_3d_128(3, n=32)
    outs = []
    extras = [dict(use_graphs=-1, tail_cells=-1), dict(), dict(use_graphs=-1)]
    if precision == 0:  # FP64 kernels are built without contraction: fused == per colour
        extras.append(dict(smoother_fusion=1))
    for extra in extras:
        kn = abi.make_knobs(precon_type=2, visc_type=-2, method=method, precision=precision, **extra)
        with StokesSolver(3, (32, 32, 32), prob.dx, knobs=kn) as s:
            for _ in range(3):
                xu, xp = prob.zeros_like_solution()
                s.solve(prob.b_u, prob.b_p, xu, xp, prob.alpha_fc, prob.beta, prob.beta_ed, prob.gamma, prob.theta_alpha)
                outs.append((xu, xp))
    for xu, xp in outs[1:]:
        for c in range(3):
            np.testing.assert_array_equal(xu[c], outs[0][0][c])
        np.testing.assert_array_equal(xp, outs[0][1])


# ---------------------------------------------------------------- odd coarsest levels
# 96 -> 48 -> 24 -> 12 -> 6 -> 3 and 24 -> 12 -> 6 -> 3: the coarsest level has
# an odd cell count, where a colour's faces can be periodic neighbours and the
# colour is applied in the reference's two steps (applyop of the colour, then
# the update).
@pytest.mark.parametrize("dm,n", [(2, 96), (2, 48), (3, 24)])
@pytest.mark.parametrize("visc", [-1, -2, 2])
@pytest.mark.parametrize("tail", [(-1, 0), (0, 0)])
def test_vcycle_odd_coarsest_bit_exact(oracle, dm, n, visc, tail):
    p, rng = random_problem(dm, n, 23, visc, theta=2.0)
    kn = dict(visc_type=visc)
    k = oracle.default_knobs(**kn)
    s = make_solver(p, **kn, tail_cells=tail[0], tail_smem_kb=tail[1])
    assert oracle.level_shape(p, s.num_levels() - 1)[0] == 3
    rhs = [rng.standard_normal(p.shape) for _ in range(dm)]
    ref = oracle.stag_mg_solver(p, k, rhs)
    phi = [dev(np.zeros(p.shape)) for _ in range(dm)]
    s.stag_mg_solver([dev(a) for a in rhs], phi)
    for c in range(dm):
        np.testing.assert_array_equal(host(phi[c]), ref[c])
    s.close()


@pytest.mark.parametrize("dm,n", [(2, 96), (3, 24)])
@pytest.mark.parametrize("pt", [1, 2])
@pytest.mark.parametrize("tail_cells", [-1, 0])
def test_apply_precon_odd_coarsest(oracle, dm, n, pt, tail_cells):
    p, rng = random_problem(dm, n, 29, -2, theta=40.0)
    k = oracle.default_knobs(visc_type=-2, precon_type=pt)
    s = make_solver(p, visc_type=-2, precon_type=pt, tail_cells=tail_cells)
    bu = [rng.standard_normal(p.shape) for _ in range(dm)]
    bpp = rng.standard_normal(p.shape)
    ref_u, ref_p = oracle.apply_precon(p, k, bu, bpp)
    xu = [dev(np.zeros(p.shape)) for _ in range(dm)]
    xp = dev(np.zeros(p.shape))
    s.apply_precon([dev(a) for a in bu], dev(bpp), xu, xp)
    scale = max(np.abs(ref_p).max(), max(np.abs(r).max() for r in ref_u))
    for c in range(dm):
        np.testing.assert_allclose(host(xu[c]), ref_u[c], rtol=0, atol=1e-12 * scale)
    np.testing.assert_allclose(host(xp), ref_p, rtol=0, atol=1e-12 * scale)
    s.close()


@pytest.mark.parametrize("n", [96, 192])
def test_gmres_parity_2d_odd_coarsest(oracle, n):
    prob = synth.make_problem(2, n, 50.0, 31)
    ref, got = _solve_both(oracle, prob, precon_type=2, visc_type=-2)
    assert ref[0] == got[0] == 0
    _assert_solution_parity(ref, got)


@pytest.mark.parametrize("precision", [0, 1])
def test_fgmres_classical_gram_schmidt(oracle, precision):
    """FGMRES with all projections in one pass (orthogonalization = 1):
    same iteration count within one and the same solution within the
    parity bar as modified Gram-Schmidt."""
    from lowmachmixtures_b200.gmres import StokesSolver
    prob = synth.config_3d_128(4, n=32)
    outs = []
    for orth in (0, 1):
        kn = abi.make_knobs(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES, precision=precision,
                            orthogonalization=orth)
        xu, xp = prob.zeros_like_solution()
        with StokesSolver(3, (32, 32, 32), prob.dx, knobs=kn) as s:
            _, _, st = s.solve(prob.b_u, prob.b_p, xu, xp, prob.alpha_fc, prob.beta, prob.beta_ed, prob.gamma,
                               prob.theta_alpha)
        assert st["norm_resid_true"] <= 1e-9 * st["norm_b"]
        outs.append((st["total_iter"], xu, xp))
    assert abs(outs[0][0] - outs[1][0]) <= 1
    for c in range(3):
        assert np.linalg.norm(outs[1][1][c] - outs[0][1][c]) <= 1e-8 * np.linalg.norm(outs[0][1][c])


# ---------------------------------------------------------------- BFBt Schur approximation
@pytest.mark.parametrize("dm,n", [(2, 32), (3, 16)])
@pytest.mark.parametrize("pt", [1, 2, -2, 3, 4, 5])
@pytest.mark.parametrize("theta", [0.0, 30.0])
@pytest.mark.parametrize("visc", [-1, -2, 2])
def test_apply_precon_bfbt(oracle, dm, n, pt, theta, visc):
    """visc_schur_approx = 1: the BFBt Schur approximation of
    visc_schur_complement (two inverse-viscosity-weighted pressure solves
    around D M L M G) against the oracle."""
    p, rng = random_problem(dm, n, 37, visc, theta=theta)
    k = oracle.default_knobs(visc_type=visc, precon_type=pt, visc_schur_approx=1)
    s = make_solver(p, visc_type=visc, precon_type=pt, visc_schur_approx=1)
    bu = [rng.standard_normal(p.shape) for _ in range(dm)]
    bpp = rng.standard_normal(p.shape)
    ref_u, ref_p = oracle.apply_precon(p, k, bu, bpp)
    xu = [dev(np.zeros(p.shape)) for _ in range(dm)]
    xp = dev(np.zeros(p.shape))
    s.apply_precon([dev(a) for a in bu], dev(bpp), xu, xp)
    scale = max(np.abs(r).max() for r in ref_u + [ref_p])
    for c in range(dm):
        np.testing.assert_allclose(host(xu[c]), ref_u[c], rtol=0, atol=1e-12 * scale)
    np.testing.assert_allclose(host(xp), ref_p, rtol=0, atol=1e-12 * scale)
    s.close()


@pytest.mark.parametrize("pt", [1, 2])
def test_gmres_parity_bfbt(oracle, pt):
    prob = synth.make_problem(2, 32, 100.0, 41, theta_alpha=50.0)
    ref, got = _solve_both(oracle, prob, precon_type=pt, visc_type=-2, visc_schur_approx=1)
    assert ref[0] == got[0] == 0
    _assert_solution_parity(ref, got)


@pytest.mark.parametrize("precision", [0, 1])
def test_autotuned_block_shapes_are_bitwise_neutral_and_reported(precision):
    """The block-shape autotuner picks launch geometry only: on a grid size
    no handle has tuned yet, a solve with the default shapes (autotune = -1)
    and one after tuning (autotune = 0) give the same bits, and
    lmm_autotune_report lists what was tuned for that grid."""
    import ctypes as C

    from lowmachmixtures_b200 import _native
    from lowmachmixtures_b200.gmres import StokesSolver
    n = 48 if precision == 0 else 40
    prob = synth.make_problem(3, n, 30.0, 9, theta_alpha=0.1 * n * n)
    outs = []
    for at in (-1, 0):
        kn = abi.make_knobs(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES, precision=precision, autotune=at)
        with StokesSolver(3, (n, n, n), prob.dx, knobs=kn) as s:
            xu, xp = prob.zeros_like_solution()
            s.solve(prob.b_u, prob.b_p, xu, xp, prob.alpha_fc, prob.beta, prob.beta_ed, prob.gamma, prob.theta_alpha)
        outs.append((xu, xp))
    for c in range(3):
        np.testing.assert_array_equal(outs[0][0][c], outs[1][0][c])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])
    lib = _native.load()
    need = lib.lmm_autotune_report(None, 0)
    buf = C.create_string_buffer(need + 1)
    assert lib.lmm_autotune_report(buf, need + 1) == need
    rep = buf.value.decode()
    w = 64 if precision == 0 else 32
    assert f"gs_colour fp{w} visc -2 3D {n}x{n}x{n}" in rep, rep
    assert f"applyop fp{w} visc -2 3D {n}x{n}x{n}" in rep, rep
    assert f"residual fp{w} visc -2 3D {n}x{n}x{n}" in rep, rep
    assert f"apply_matrix fp{w} visc -2 3D {n}x{n}x{n}" in rep, rep
