"""GPU parity with wall boundaries (no-slip / slip walls, bc.f90 codes 100
and 200) against the CPU oracle.

As in the periodic case the FP64 kernels keep the reference's operand order:
the operator, the colour sweeps, Jacobi, residual restriction, prolongation,
whole V-cycles and apply_matrix are bit-identical to the oracle; the
preconditioner (which removes means through reductions) agrees to 1e-12;
full solves to 1e-10 relative in velocity and mean-removed pressure with the
iteration count within 1.  Inputs hold zero on the wall faces, the values the
reference's physbc_domainvel gives them.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lowmachmixtures_b200 import abi, synth  # noqa: E402

pytestmark = pytest.mark.gpu

NS, SL, PER = abi.LMM_BC_NO_SLIP_WALL, abi.LMM_BC_SLIP_WALL, abi.LMM_BC_PERIODIC
BCS_2D = [(PER, NS), (NS, SL), ((NS, SL), (SL, NS))]
BCS_3D = [(PER, SL, NS), (NS, NS, NS), ((SL, NS), PER, (NS, SL))]
VISCS = (-1, 1, -2, 2, -3, 3)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


def mask(dm, bc, shape, c):
    m = np.ones(shape)
    if abi.walled(bc, c):
        idx = [slice(None)] * dm
        idx[dm - 1 - c] = 0
        m[tuple(idx)] = 0.0
    return m


def faces(rng, dm, bc, shape):
    return [rng.standard_normal(shape) * mask(dm, bc, shape, c) for c in range(dm)]


def random_problem(dm, n, seed, visc, bc, theta=7.0):
    rng = np.random.Generator(np.random.PCG64(seed))
    p = synth.make_problem(dm, n, 10.0, seed, theta_alpha=theta, bc=bc)
    shape = p.shape
    if visc > 0:
        p.beta = np.full(shape, 0.8)
        p.beta_ed = [np.full(e.shape, 0.8) for e in p.beta_ed]
        p.gamma = np.full(shape, 0.3)
    else:
        p.beta = rng.uniform(0.5, 2.0, shape)
        p.beta_ed = [rng.uniform(0.5, 2.0, e.shape) for e in p.beta_ed]
        p.gamma = rng.uniform(0.1, 0.5, shape)
    p.alpha_fc = [rng.uniform(0.5, 1.5, shape) for _ in range(dm)]
    return p, rng


def make_solver(p, **kn):
    from lowmachmixtures_b200.gmres import StokesSolver
    s = StokesSolver(p.dm, p.n[: p.dm], p.dx, knobs=abi.make_knobs(**kn), bc=p.bc)
    s.load_coeffs([dev(a) for a in p.alpha_fc], dev(p.beta), [dev(b) for b in p.beta_ed], dev(p.gamma), p.theta_alpha)
    return s


CASES = [(2, 16, bc) for bc in BCS_2D] + [(3, 8, bc) for bc in BCS_3D]


@pytest.mark.parametrize("dm,n,bc", CASES)
@pytest.mark.parametrize("visc", VISCS)
def test_walls_applyop_bit_exact(oracle, dm, n, bc, visc):
    p, rng = random_problem(dm, n, 21, visc, bc)
    s = make_solver(p, visc_type=visc)
    phi = faces(rng, dm, bc, p.shape)
    for color in range(0, 2 * dm + 1):
        init = faces(rng, dm, bc, p.shape)
        ref = oracle.stag_applyop(p, visc, phi, color=color, Lphi=init)
        out = [dev(a) for a in init]
        s.stag_applyop([dev(a) for a in phi], out, color)
        for c in range(dm):
            np.testing.assert_array_equal(host(out[c]), ref[c], err_msg=f"colour {color} comp {c}")
    s.close()


@pytest.mark.parametrize("dm,n,bc", CASES)
@pytest.mark.parametrize("visc", [-1, -2, -3, 2])
@pytest.mark.parametrize("lev", [0, 1])
def test_walls_smooth_colours_bit_exact(oracle, dm, n, bc, visc, lev):
    p, rng = random_problem(dm, n, 22, visc, bc)
    k = oracle.default_knobs(visc_type=visc, stag_mg_omega=0.9)
    s = make_solver(p, visc_type=visc, stag_mg_omega=0.9)
    shp = oracle.level_shape(p, lev)
    for color in range(0, 2 * dm + 1):
        phi = faces(rng, dm, bc, shp)
        rhs = [rng.standard_normal(shp) for _ in range(dm)]
        ref = oracle.smooth(p, k, lev, rhs, phi, color)
        dphi = [dev(a) for a in phi]
        s.smooth(lev, [dev(a) for a in rhs], dphi, color)
        for c in range(dm):
            np.testing.assert_array_equal(host(dphi[c]), ref[c], err_msg=f"lev {lev} colour {color} comp {c}")
    s.close()


@pytest.mark.parametrize("dm,n,bc", [(2, 16, bc) for bc in BCS_2D] + [(3, 16, bc) for bc in BCS_3D])
@pytest.mark.parametrize("visc", [-1, -2, 2])
def test_walls_residual_restrict_and_prolong_bit_exact(oracle, dm, n, bc, visc):
    p, rng = random_problem(dm, n, 23, visc, bc)
    k = oracle.default_knobs(visc_type=visc)
    s = make_solver(p, visc_type=visc)
    for lev in (0, 1):
        shp = oracle.level_shape(p, lev)
        shc = oracle.level_shape(p, lev + 1)
        phi = faces(rng, dm, bc, shp)
        rhs = [rng.standard_normal(shp) for _ in range(dm)]
        ref = oracle.residual_restrict(p, k, lev, rhs, phi)
        out = [dev(np.zeros(shc)) for _ in range(dm)]
        s.residual_restrict(lev, [dev(a) for a in rhs], [dev(a) for a in phi], out)
        for c in range(dm):
            np.testing.assert_array_equal(host(out[c]), ref[c], err_msg=f"restrict lev {lev} comp {c}")
        coarse = faces(rng, dm, bc, shc)
        refp = oracle.prolong_add(p, lev, coarse, phi)
        dphi = [dev(a) for a in phi]
        s.prolong_add(lev, [dev(a) for a in coarse], dphi)
        for c in range(dm):
            np.testing.assert_array_equal(host(dphi[c]), refp[c], err_msg=f"prolong lev {lev} comp {c}")
    s.close()


@pytest.mark.parametrize("dm,n,bc", [(2, 32, bc) for bc in BCS_2D] + [(3, 16, bc) for bc in BCS_3D] + [(2, 48, (NS, SL))])
@pytest.mark.parametrize("visc", [-1, -2, -3])
@pytest.mark.parametrize("smoother", [1, 0])
@pytest.mark.parametrize("tail_cells", [0, -1])
def test_walls_vcycle_bit_exact(oracle, dm, n, bc, visc, smoother, tail_cells):
    """tail_cells 0: the coarse levels in the single-block tail (its wall
    variant); -1: every level by per-level kernels"""
    p, rng = random_problem(dm, n, 24, visc, bc, theta=3.0)
    kn = dict(visc_type=visc, stag_mg_smoother=smoother, stag_mg_omega=1.0 if smoother else 0.7)
    k = oracle.default_knobs(**kn)
    s = make_solver(p, **kn, tail_cells=tail_cells)
    rhs = [rng.standard_normal(p.shape) for _ in range(dm)]
    ref = oracle.stag_mg_solver(p, k, rhs)
    phi = [dev(np.zeros(p.shape)) for _ in range(dm)]
    s.stag_mg_solver([dev(a) for a in rhs], phi)
    for c in range(dm):
        np.testing.assert_array_equal(host(phi[c]), ref[c])
    s.close()


@pytest.mark.parametrize("dm,n,bc", [(2, 32, bc) for bc in BCS_2D] + [(3, 16, bc) for bc in BCS_3D])
@pytest.mark.parametrize("visc", [-2, 3])
def test_walls_apply_matrix_bit_exact(oracle, dm, n, bc, visc):
    p, rng = random_problem(dm, n, 25, visc, bc)
    s = make_solver(p, visc_type=visc)
    xu = faces(rng, dm, bc, p.shape)
    xp = rng.standard_normal(p.shape)
    ref_u, ref_p = oracle.apply_matrix(p, visc, xu, xp)
    bu = [dev(np.zeros(p.shape)) for _ in range(dm)]
    bp = dev(np.zeros(p.shape))
    s.apply_matrix([dev(a) for a in xu], dev(xp), bu, bp)
    for c in range(dm):
        np.testing.assert_array_equal(host(bu[c]), ref_u[c])
    np.testing.assert_array_equal(host(bp), ref_p)
    s.close()


@pytest.mark.parametrize("dm,n,bc", [(2, 32, bc) for bc in BCS_2D] + [(3, 16, bc) for bc in BCS_3D])
@pytest.mark.parametrize("pt", [1, -1, 2, -2, 3, 4, 5])
@pytest.mark.parametrize("theta", [0.0, 50.0])
def test_walls_apply_precon(oracle, dm, n, bc, pt, theta):
    visc = -2 if pt % 2 else -3
    p, rng = random_problem(dm, n, 26, visc, bc, theta=theta)
    k = oracle.default_knobs(visc_type=visc, precon_type=pt)
    s = make_solver(p, visc_type=visc, precon_type=pt)
    bu = faces(rng, dm, bc, p.shape)
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


def _solve_both(oracle, prob, layout=abi.LMM_LAYOUT_COMPACT, **kn):
    k = oracle.default_knobs(**kn)
    rc_o, xu_o, xp_o, th_o, npr_o, st_o = oracle.solve(prob, k)
    from lowmachmixtures_b200.gmres import StokesSolver
    with StokesSolver(prob.dm, prob.n[: prob.dm], prob.dx, knobs=abi.make_knobs(**kn), bc=prob.bc) as s:
        xu, xp = prob.zeros_like_solution()
        th, npr, st = s.solve(prob.b_u, prob.b_p, xu, xp, prob.alpha_fc, prob.beta, prob.beta_ed, prob.gamma,
                              prob.theta_alpha)
    return (rc_o, xu_o, xp_o, st_o), (st["status"], xu, xp, st)


def _assert_parity(ref, got, tol=1e-10):
    _, xu_o, xp_o, st_o = ref
    _, xu, xp, st = got
    for c in range(len(xu)):
        err = np.abs(xu[c] - xu_o[c]).max() / np.abs(xu_o[c]).max()
        assert err <= tol, f"velocity comp {c} rel err {err:.3e}"
    po, pg = xp_o - xp_o.mean(), xp - xp.mean()
    err = np.abs(pg - po).max() / max(np.abs(po).max(), 1e-300)
    assert err <= tol, f"pressure rel err {err:.3e}"
    assert abs(st["total_iter"] - st_o["total_iter"]) <= 1, (st["total_iter"], st_o["total_iter"])


@pytest.mark.parametrize("dm,n,bc,theta", [(2, 64, (PER, NS), 0.0), (2, 64, (NS, NS), 0.0), (2, 64, (SL, NS), 200.0),
                                           (3, 32, (PER, NS, PER), 0.0), (3, 32, (NS, SL, NS), 1000.0)])
@pytest.mark.parametrize("pt", [1, 2])
def test_walls_gmres_parity(oracle, dm, n, bc, theta, pt):
    prob = synth.make_problem(dm, n, 30.0, 7, theta_alpha=theta, bc=bc)
    ref, got = _solve_both(oracle, prob, precon_type=pt, visc_type=-2)
    assert ref[0] == got[0]
    _assert_parity(ref, got)


@pytest.mark.parametrize("precision", [abi.LMM_PRECISION_FP64, abi.LMM_PRECISION_FP32])
def test_walls_fgmres(oracle, precision):
    prob = synth.make_problem(3, 32, 100.0, 9, theta_alpha=0.1 * 32 * 32, bc=(PER, NS, SL))
    ref, got = _solve_both(oracle, prob, precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES,
                           precision=precision, orthogonalization=1 if precision else 0)
    st = got[3]
    assert got[0] == 0
    assert st["norm_resid_true"] <= 1e-9 * st["norm_b"]
    if precision == abi.LMM_PRECISION_FP64:
        _assert_parity(ref, got)
    else:
        err = max(np.abs(got[1][c] - ref[1][c]).max() / np.abs(ref[1][c]).max() for c in range(3))
        assert err < 1e-6, err


def test_walls_boxlib_layout(oracle):
    """BoxLib host arrays on a wall-bounded grid: n+1 faces and nodes along
    the walls, ghosts on output following the wall rules -- the oracle and
    the library write the same arrays."""
    import ctypes as C
    bc = (PER, NS, SL)
    prob = synth.make_problem(3, 16, 10.0, 5, theta_alpha=40.0, bc=bc)
    faces_nod = [(1, 0, 0), (0, 1, 0), (0, 0, 1)]
    edges_nod = [(1, 1, 0), (1, 0, 1), (0, 1, 1)]

    def boxlib(a, nodal, ng, edge=False, comp=None):
        # compact -> BoxLib array: periodic directions wrap; along a wall the
        # extra hi+1 entry is the stored hi+1 node (edges) or zero (faces)
        out = a
        for ax, nod in enumerate(reversed(nodal)):
            d = 2 - ax
            n = prob.n[d]
            per = not abi.walled(bc, d)
            m = out.shape[ax]
            idx = [(v % n) if per else min(max(v, 0), m - 1) for v in range(-ng, n + nod + ng)]
            out = np.take(out, idx, axis=ax)
            if not per and nod and not edge:
                sl = [slice(None)] * 3
                sl[ax] = slice(ng + n, None)
                out[tuple(sl)] = 0.0
        return np.ascontiguousarray(out)

    bu = [boxlib(prob.b_u[c], faces_nod[c], 0, comp=c) for c in range(3)]
    al = [boxlib(prob.alpha_fc[c], faces_nod[c], 0) for c in range(3)]
    be = boxlib(prob.beta, (0, 0, 0), 1)
    ga = boxlib(prob.gamma, (0, 0, 0), 1)
    bed = [boxlib(prob.beta_ed[e], edges_nod[e], 0, edge=True) for e in range(3)]
    bp = boxlib(prob.b_p, (0, 0, 0), 0)
    ng = 2
    kn = dict(precon_type=2, visc_type=-2)
    from lowmachmixtures_b200.gmres import StokesSolver
    xu = [np.zeros_like(boxlib(prob.b_u[c], faces_nod[c], ng)) for c in range(3)]
    xp = np.zeros_like(boxlib(prob.b_p, (0, 0, 0), ng))
    ngd = dict(beta=1, gamma=1, x_u=ng, x_p=ng)
    with StokesSolver(3, (16, 16, 16), prob.dx, knobs=abi.make_knobs(**kn), bc=bc) as s:
        s.solve(bu, bp, xu, xp, al, be, bed, ga, prob.theta_alpha, layout=abi.LMM_LAYOUT_BOXLIB, ng=ngd)
    # the oracle, same BoxLib arrays
    xu_o = [np.zeros_like(a) for a in xu]
    xp_o = np.zeros_like(xp)
    fin = abi.FieldsIn()
    fin.b_u, fin.b_p = abi.ptr_array(bu), abi.ptr(bp)
    fin.alpha_fc, fin.beta, fin.beta_ed, fin.gamma = abi.ptr_array(al), abi.ptr(be), abi.ptr_array(bed), abi.ptr(ga)
    fin.layout = abi.LMM_LAYOUT_BOXLIB
    fin.ng_beta = fin.ng_gamma = 1
    fout = abi.FieldsOut()
    fout.x_u, fout.x_p = abi.ptr_array(xu_o), abi.ptr(xp_o)
    fout.layout = abi.LMM_LAYOUT_BOXLIB
    fout.ng_x_u = fout.ng_x_p = ng
    th, npr, st = C.c_double(prob.theta_alpha), C.c_double(0.0), abi.Stats()
    g = oracle.grid_of(prob)
    rc = oracle.lib().orc_stokes_solve(C.byref(g), C.byref(oracle.default_knobs(**kn)), C.byref(fin), C.byref(fout),
                                       C.byref(th), C.byref(npr), C.byref(st))
    assert rc == 0
    for c in range(3):
        scale = np.abs(xu_o[c]).max()
        np.testing.assert_allclose(xu[c], xu_o[c], rtol=0, atol=1e-10 * scale)
    po, pg = xp_o - xp_o[ng:-ng, ng:-ng, ng:-ng].mean(), xp - xp[ng:-ng, ng:-ng, ng:-ng].mean()
    np.testing.assert_allclose(pg, po, rtol=0, atol=1e-10 * np.abs(po).max())


def test_walls_rejections():
    from lowmachmixtures_b200._native import LmmError
    from lowmachmixtures_b200.gmres import StokesSolver
    with pytest.raises(LmmError):
        StokesSolver(2, (16, 16), 1 / 16, bc=(PER, (NS, PER)))  # one side periodic, one a wall
    with pytest.raises(LmmError):
        StokesSolver(2, (16, 16), 1 / 16, bc=(PER, NS), visc_schur_approx=1, visc_type=-2)
    with pytest.raises(LmmError):
        StokesSolver(2, (16, 16), 1 / 16, bc=(PER, 300))
