"""Pin the CPU oracle against the golden fixtures of the independent numpy
restatement (tests/golden/numpy_ref.py).  Both keep the reference's operand
order and round every operation separately, so the stencil results must be
bit-identical; the seam-weighted reductions agree to summation-order level."""
import numpy as np
import pytest

from helpers import load_golden, problem_from_fixture, rel_err

VISCS = (-1, 1, -2, 2, -3, 3)


@pytest.mark.parametrize("dm", [2, 3])
@pytest.mark.parametrize("visc", VISCS)
def test_applyop_bit_exact(oracle, dm, visc):
    fx = load_golden(f"stencils_{dm}d.npz")
    p = problem_from_fixture(fx, f"v{visc}_", dm, 8, 3.0)
    phi = [np.ascontiguousarray(fx[f"v{visc}_phi{c}"]) for c in range(dm)]
    L = oracle.stag_applyop(p, visc, phi)
    for c in range(dm):
        np.testing.assert_array_equal(L[c], fx[f"v{visc}_L{c}"])


@pytest.mark.parametrize("dm", [2, 3])
@pytest.mark.parametrize("visc", VISCS)
def test_smooth_colours_bit_exact(oracle, dm, visc):
    fx = load_golden(f"stencils_{dm}d.npz")
    p = problem_from_fixture(fx, f"v{visc}_", dm, 8, 3.0)
    phi = [np.ascontiguousarray(fx[f"v{visc}_phi{c}"]) for c in range(dm)]
    rhs = [np.ascontiguousarray(fx[f"v{visc}_rhs{c}"]) for c in range(dm)]
    k = oracle.default_knobs(visc_type=visc)
    for color in range(0, 2 * dm + 1):
        out = oracle.smooth(p, k, 0, rhs, phi, color)
        for c in range(dm):
            np.testing.assert_array_equal(out[c], fx[f"v{visc}_smooth{color}_{c}"], err_msg=f"colour {color} comp {c}")


@pytest.mark.parametrize("dm", [2, 3])
def test_transfer_operators_bit_exact(oracle, dm):
    fx = load_golden(f"stencils_{dm}d.npz")
    p = problem_from_fixture(fx, "v-2_", dm, 8, 0.0)
    f = [np.ascontiguousarray(fx[f"xfer_f{c}"]) for c in range(dm)]
    cc = [np.ascontiguousarray(fx[f"xfer_coarse{c}"]) for c in range(dm)]
    pr = oracle.prolong_add(p, 0, cc, f)
    for c in range(dm):
        np.testing.assert_array_equal(pr[c], fx[f"xfer_prolong{c}"])
    # residual restriction with phi = 0: rhs - L*0 = rhs, restricted (12/6-point)
    k = oracle.default_knobs(visc_type=-2)
    zero = [np.zeros_like(a) for a in f]
    r = oracle.residual_restrict(p, k, 0, f, zero)
    for c in range(dm):
        np.testing.assert_array_equal(r[c], fx[f"xfer_restrict{c}"])


@pytest.mark.parametrize("dm", [2, 3])
def test_alpha_restriction_simple_stencil(oracle, dm):
    fx = load_golden(f"stencils_{dm}d.npz")
    p = problem_from_fixture(fx, "v-2_", dm, 8, 1.0)
    p.alpha_fc = [np.ascontiguousarray(fx[f"xfer_f{c}"]) for c in range(dm)]
    k = oracle.default_knobs(visc_type=-2)
    alpha, beta, bed, gamma = oracle.coarse_coeffs(p, k, 1)
    for c in range(dm):
        np.testing.assert_array_equal(alpha[c], fx[f"xfer_simple{c}"])


@pytest.mark.parametrize("dm", [2, 3])
def test_grad_div_bit_exact(oracle, dm):
    fx = load_golden(f"stencils_{dm}d.npz")
    p = problem_from_fixture(fx, "v-2_", dm, 8, 0.0)
    f = [np.ascontiguousarray(fx[f"xfer_f{c}"]) for c in range(dm)]
    # apply_matrix with x_u = 0 gives b_u = grad(x_p); with x_p = 0, b_p = -div(x_u)
    gp = np.ascontiguousarray(fx["grad_p"])
    b_u, _ = oracle.apply_matrix(p, -2, [np.zeros_like(a) for a in f], gp)
    for c in range(dm):
        np.testing.assert_array_equal(b_u[c], fx[f"grad{c}"])
    _, b_p = oracle.apply_matrix(p, -2, f, np.zeros_like(gp))
    np.testing.assert_array_equal(b_p, -fx["div"])


@pytest.mark.parametrize("dm", [2, 3])
def test_inner_product_seam_weight(oracle, dm):
    fx = load_golden(f"stencils_{dm}d.npz")
    p = problem_from_fixture(fx, "v-2_", dm, 8, 0.0)
    f = [np.ascontiguousarray(fx[f"xfer_f{c}"]) for c in range(dm)]
    zp = np.zeros(f[0].shape)
    ip = oracle.inner_prod(p, f, zp, f, zp)
    for c in range(dm):
        assert rel_err(ip[c], fx["ip_faces"][c]) < 1e-13


@pytest.mark.parametrize("dm", [2, 3])
@pytest.mark.parametrize("smoother", [1, 0])
def test_vcycle_matches_numpy_restatement(oracle, dm, smoother):
    fx = load_golden("vcycle.npz")
    n = 16 if dm == 2 else 8
    pre = f"d{dm}_"
    theta = float(fx[pre + "theta"][0])
    p = problem_from_fixture(fx, pre, dm, n, theta)
    rhs = [np.ascontiguousarray(fx[f"{pre}rhs{c}"]) for c in range(dm)]
    k = oracle.default_knobs(visc_type=-2, stag_mg_smoother=smoother,
                             stag_mg_omega=1.0 if smoother else 0.6)
    phi = oracle.stag_mg_solver(p, k, rhs)
    for c in range(dm):
        np.testing.assert_array_equal(phi[c], fx[f"{pre}s{smoother}_phi{c}"])
