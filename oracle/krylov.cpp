// krylov.cpp - CPU oracle: Stokes operator, block preconditioners, GMRES.
//
// TEST INFRASTRUCTURE ONLY (the oracle).  Restates
//   src_gmres/apply_matrix.f90:23-122   (apply_matrix)
//   src_gmres/apply_precon.f90:29-536   (apply_precon, precon_type +-1..+-5,
//       visc_schur_approx = 0, simple_schur_complement, mean removal :429-460)
//   src_gmres/macproject.f90:320-364    (subtract_weighted_gradp)
//   src_gmres/gmres.f90:30-605          (gmres, least_squares, rotmat,
//       SolveUTriangular, update_sol)
// and adds the right-preconditioned flexible GMRES this library offers as
// LMM_METHOD_FGMRES (same Arnoldi/Givens arithmetic, true-residual stop).
#include "oracle_internal.hpp"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <vector>

namespace orc {

template <class F>
static void for_valid(Fab& f, F fn) {
    for (int k = f.vlo[2]; k <= f.vhi[2]; ++k)
        for (int j = f.vlo[1]; j <= f.vhi[1]; ++j)
            for (int i = f.vlo[0]; i <= f.vhi[0]; ++i) fn(f(i, j, k), i, j, k);
}
// multifab_copy_c(dst,1,src,1,1,0)
static void copy_valid(Fab& dst, const Fab& src) {
    for_valid(dst, [&](double& d, int i, int j, int k) { d = src(i, j, k); });
}
static void scale_valid(Fab& f, double s) {
    for_valid(f, [&](double& d, int, int, int) { d = d * s; });
}

Level make_level0(const Problem& P, double theta_alpha) {
    Level L;
    L.geo = P.geo;
    L.dx = P.dx;
    for (int i = 0; i < P.geo.dm; ++i) {
        L.alpha[i] = P.alpha_fc[i];
        for (double& v : L.alpha[i].a) v = v * theta_alpha;  // alpha_fc_temp (stag_applyop.f90:43-49)
    }
    L.beta_cc = P.beta;
    for (int e = 0; e < (P.geo.dm == 2 ? 1 : 3); ++e) L.beta_ed[e] = P.beta_ed[e];
    L.gamma_cc = P.gamma;
    return L;
}

void apply_matrix(const Problem& P, double theta_alpha, Fab* b_u, Fab& b_p, Fab* x_u, Fab& x_p) {
    const int dm = P.geo.dm;
    // ghost fills (apply_matrix.f90:60-87); the wall faces of x_u become zero
    fill_pres(P.geo, x_p);
    fill_vel(P.geo, x_u);
    Fab gx_p[3];
    for (int i = 0; i < dm; ++i) gx_p[i] = make_face(P.geo, i, 0);
    Level L = make_level0(P, theta_alpha);
    stag_applyop_level(L, x_u, b_u, 0, P.visc_type);
    compute_grad(P.geo, P.dx, x_p, gx_p);
    for (int i = 0; i < dm; ++i) for_valid(b_u[i], [&](double& d, int a, int b, int c) { d = d + gx_p[i](a, b, c); });
    compute_div(P.geo, P.dx, x_u, b_p);
    scale_valid(b_p, -1.0);
}

// subtract_weighted_gradp (macproject.f90:320-364): x_u -= coef * grad(phi)
static void subtract_weighted_gradp(const Problem& P, Fab* x_u, const Fab* coef, const Fab& phi) {
    const int dm = P.geo.dm;
    Fab gradp[3];
    for (int i = 0; i < dm; ++i) gradp[i] = make_face(P.geo, i, 1);
    compute_grad(P.geo, P.dx, phi, gradp);
    for (int i = 0; i < dm; ++i) {
        for_valid(gradp[i], [&](double& d, int a, int b, int c) { d = d * coef[i](a, b, c); });
        for_valid(x_u[i], [&](double& d, int a, int b, int c) { d = d + -1.0 * gradp[i](a, b, c); });
    }
}

// x_p = -(L_alpha phi) with face coefficient alphainv (the cc_applyop call of
// apply_precon.f90:153-154; BoxLib's operator replaced by this library's
// cross stencil, the same one its pressure multigrid uses)
static void neg_cc_lap(const Problem& P, const Fab* a, const Fab& phi, Fab& out) {
    const double dxsqinv = 1.0 / (P.dx * P.dx);
    const int dm = P.geo.dm;
    for_valid(out, [&](double& d, int i, int j, int k) {
        double v = (a[0](i + 1, j, k) * (phi(i + 1, j, k) - phi(i, j, k)) - a[0](i, j, k) * (phi(i, j, k) - phi(i - 1, j, k))) +
                   (a[1](i, j + 1, k) * (phi(i, j + 1, k) - phi(i, j, k)) - a[1](i, j, k) * (phi(i, j, k) - phi(i, j - 1, k)));
        if (dm == 3) v = v + (a[2](i, j, k + 1) * (phi(i, j, k + 1) - phi(i, j, k)) - a[2](i, j, k) * (phi(i, j, k) - phi(i, j, k - 1)));
        d = -(v * dxsqinv);
    });
}

// inverse_diag_lap (inverse_diag_lap.f90:17-250): 1 / diag of the viscous
// operator per face, without theta*alpha and dx^2 (|visc_type| 1, 2)
static void inverse_diag_lap(const Problem& P, Fab* m) {
    const int dm = P.geo.dm, visc = P.visc_type;
    const Fab& b = P.beta;
    const double b0 = P.beta(0, 0, 0);
    for (int d = 0; d < dm; ++d) {
        m[d] = make_face(P.geo, d, 0);
        for_valid(m[d], [&](double& v, int i, int j, int k) {
            if (visc == 1) { v = 1.0 / ((dm == 3 ? 6.0 : 4.0) * b0); return; }
            if (visc == 2) { v = 1.0 / ((dm == 3 ? 8.0 : 6.0) * b0); return; }
            const double c = (visc == -2) ? 2.0 : 1.0;
            if (dm == 2) {
                const Fab& e = P.beta_ed[0];
                if (d == 0) v = 1.0 / (c * b(i, j, 0) + c * b(i - 1, j, 0) + e(i, j + 1, 0) + e(i, j, 0));
                else v = 1.0 / (c * b(i, j, 0) + c * b(i, j - 1, 0) + e(i + 1, j, 0) + e(i, j, 0));
                return;
            }
            const Fab &xy = P.beta_ed[0], &xz = P.beta_ed[1], &yz = P.beta_ed[2];
            if (d == 0)
                v = 1.0 / (c * b(i, j, k) + c * b(i - 1, j, k) + xy(i, j, k) + xy(i, j + 1, k) + xz(i, j, k) + xz(i, j, k + 1));
            else if (d == 1)
                v = 1.0 / (c * b(i, j, k) + c * b(i, j - 1, k) + xy(i, j, k) + xy(i + 1, j, k) + yz(i, j, k) + yz(i, j, k + 1));
            else
                v = 1.0 / (c * b(i, j, k) + c * b(i, j, k - 1) + xz(i, j, k) + xz(i + 1, j, k) + yz(i, j, k) + yz(i, j + 1, k));
        });
    }
}

// visc_schur_complement (apply_precon.f90:538-685), the BFBt approximation
static void visc_schur(const Problem& P, const lmm_knobs& K, Fab& rhs, Fab& x_out, double theta_alpha, const Fab& phi, int* pvc) {
    const int dm = P.geo.dm;
    Fab muinv[3], gphi[3], Lgphi[3];
    inverse_diag_lap(P, muinv);
    Fab phi_mu = make_cc(P.geo, 1);
    phi_mu.setval(0.0);
    macproject(P, K, phi_mu, muinv, rhs, pvc);
    for (int d = 0; d < dm; ++d) {
        gphi[d] = make_face(P.geo, d, 1);
        Lgphi[d] = make_face(P.geo, d, 1);
    }
    compute_grad(P.geo, P.dx, phi_mu, gphi);
    for (int d = 0; d < dm; ++d) {
        for_valid(gphi[d], [&](double& v, int a, int b, int c) { v = v * muinv[d](a, b, c); });
        fill_boundary(gphi[d]);
    }
    Level L0 = make_level0(P, 0.0);  // zero alpha
    L0.gamma_cc.setval(0.0);
    stag_applyop_level(L0, gphi, Lgphi, 0, P.visc_type);
    for (int d = 0; d < dm; ++d) {
        for_valid(Lgphi[d], [&](double& v, int a, int b, int c) { v = v * muinv[d](a, b, c); });
        fill_boundary(Lgphi[d]);
    }
    compute_div(P.geo, P.dx, Lgphi, rhs);
    phi_mu.setval(0.0);
    macproject(P, K, phi_mu, muinv, rhs, pvc);
    copy_valid(x_out, phi_mu);
    if (std::fabs(theta_alpha) > 0.0) {
        Fab phi_rho = phi;
        scale_valid(phi_rho, theta_alpha);
        for_valid(x_out, [&](double& v, int a, int b, int c) { v = v + phi_rho(a, b, c); });
    }
}

void apply_precon(const Problem& P, const lmm_knobs& K, double theta_alpha, const Fab* b_u, const Fab& b_p,
                  Fab* x_u, Fab& x_p, int* vc, int* pvc) {
    const bool bfbt = K.visc_schur_approx == 1;
    const int dm = P.geo.dm;
    const int pt = K.precon_type;
    const int av = std::abs(P.visc_type);
    Fab phi = make_cc(P.geo, 1), mac_rhs = make_cc(P.geo, 0), x_p_tmp = make_cc(P.geo, 1);
    Fab alphainv[3], b_u_tmp[3], one_fab[3];
    for (int i = 0; i < dm; ++i) {
        alphainv[i] = make_face(P.geo, i, 0);
        alphainv[i].setval(1.0);
        for_valid(alphainv[i], [&](double& d, int a, int b, int c) { d = d / P.alpha_fc[i](a, b, c); });
        // on wall faces 1/alpha only ever multiplies the zero wall gradient;
        // the compact layout stores no alpha on the hi+1 wall face
        if (!P.geo.periodic(i))
            for_valid(alphainv[i], [&](double& d, int a, int b, int c) {
                const int idx[3] = {a, b, c};
                if (idx[i] == 0 || idx[i] == P.geo.n[i]) d = 0.0;
            });
        b_u_tmp[i] = make_face(P.geo, i, 0);
        one_fab[i] = make_face(P.geo, i, 0);
        one_fab[i].setval(1.0);
    }
    phi.setval(0.0);
    for (int i = 0; i < dm; ++i) x_u[i].setval(0.0);

    auto simple_schur = [&]() {
        if (av == 1 || av == 2) {
            copy_valid(x_p, mac_rhs);
            scale_valid(x_p, -1.0);
            for_valid(x_p, [&](double& d, int a, int b, int c) { d = d * P.beta(a, b, c); });
            if (av == 2) scale_valid(x_p, 2.0);
        } else if (av == 3) {
            copy_valid(x_p, mac_rhs);
            scale_valid(x_p, -4.0 / 3.0);
            for_valid(x_p, [&](double& d, int a, int b, int c) { d = d * P.beta(a, b, c); });
            scale_valid(mac_rhs, -1.0);
            for_valid(mac_rhs, [&](double& d, int a, int b, int c) { d = d * P.gamma(a, b, c); });
            for_valid(x_p, [&](double& d, int a, int b, int c) { d = d + mac_rhs(a, b, c); });
        }
        if (std::fabs(theta_alpha) > 0.0) {
            scale_valid(phi, theta_alpha);
            for_valid(x_p, [&](double& d, int a, int b, int c) { d = d + phi(a, b, c); });
        }
    };

    switch (std::abs(pt)) {
    case 1: {
        stag_mg_solver(P, K, theta_alpha, x_u, b_u, vc);
        compute_div(P.geo, P.dx, x_u, mac_rhs);
        for_valid(mac_rhs, [&](double& d, int a, int b, int c) { d = d + b_p(a, b, c); });
        macproject(P, K, phi, alphainv, mac_rhs, pvc);
        subtract_weighted_gradp(P, x_u, alphainv, phi);
        if (bfbt) {
            visc_schur(P, K, mac_rhs, x_p, theta_alpha, phi, pvc);
            break;
        }
        if (pt == 1 || theta_alpha == 0.0) {
            copy_valid(x_p, mac_rhs);
            scale_valid(x_p, -1.0);
        } else {
            neg_cc_lap(P, alphainv, phi, x_p);
        }
        if (av == 1 || av == 2) {
            for_valid(x_p, [&](double& d, int a, int b, int c) { d = d * P.beta(a, b, c); });
            if (av == 2) scale_valid(x_p, 2.0);
        } else if (av == 3) {
            copy_valid(mac_rhs, x_p);
            for_valid(mac_rhs, [&](double& d, int a, int b, int c) { d = d * P.gamma(a, b, c); });
            for_valid(x_p, [&](double& d, int a, int b, int c) { d = d * P.beta(a, b, c); });
            scale_valid(x_p, 4.0 / 3.0);
            for_valid(x_p, [&](double& d, int a, int b, int c) { d = d + mac_rhs(a, b, c); });
        }
        scale_valid(phi, theta_alpha);
        for_valid(x_p, [&](double& d, int a, int b, int c) { d = d + phi(a, b, c); });
        break;
    }
    case 2:
    case 5: {
        stag_mg_solver(P, K, theta_alpha, x_u, b_u, vc);
        compute_div(P.geo, P.dx, x_u, mac_rhs);
        for_valid(mac_rhs, [&](double& d, int a, int b, int c) { d = d + b_p(a, b, c); });
        if (std::fabs(theta_alpha) > 0.0) macproject(P, K, phi, alphainv, mac_rhs, pvc);
        if (bfbt)
            visc_schur(P, K, mac_rhs, x_p, theta_alpha, phi, pvc);
        else
            simple_schur();
        if (pt == -2 || pt == -5) scale_valid(x_p, -1.0);
        if (std::abs(pt) == 5) {
            copy_valid(x_p_tmp, x_p);
            fill_pres(P.geo, x_p_tmp);
            for (int i = 0; i < dm; ++i) copy_valid(b_u_tmp[i], b_u[i]);
            subtract_weighted_gradp(P, b_u_tmp, one_fab, x_p_tmp);
            stag_mg_solver(P, K, theta_alpha, x_u, b_u_tmp, vc);
        }
        break;
    }
    case 3: {
        copy_valid(mac_rhs, b_p);
        if (pt == -3) scale_valid(mac_rhs, -1.0);
        if (std::fabs(theta_alpha) > 0.0) macproject(P, K, phi, alphainv, mac_rhs, pvc);
        if (bfbt)
            visc_schur(P, K, mac_rhs, x_p, theta_alpha, phi, pvc);
        else
            simple_schur();
        copy_valid(x_p_tmp, x_p);
        fill_pres(P.geo, x_p_tmp);
        for (int i = 0; i < dm; ++i) copy_valid(b_u_tmp[i], b_u[i]);
        subtract_weighted_gradp(P, b_u_tmp, one_fab, x_p_tmp);
        stag_mg_solver(P, K, theta_alpha, x_u, b_u_tmp, vc);
        break;
    }
    case 4: {
        stag_mg_solver(P, K, theta_alpha, x_u, b_u, vc);
        if (std::fabs(theta_alpha) > 0.0) {
            copy_valid(mac_rhs, b_p);
            macproject(P, K, phi, alphainv, mac_rhs, pvc);
        }
        if (bfbt) {
            // mac_rhs holds b_p whenever the reference sets it (apply_precon.f90:362-366)
            copy_valid(mac_rhs, b_p);
            visc_schur(P, K, mac_rhs, x_p, theta_alpha, phi, pvc);
            break;
        }
        if (std::fabs(theta_alpha) > 0.0) scale_valid(phi, theta_alpha);
        copy_valid(x_p, b_p);
        for_valid(x_p, [&](double& d, int a, int b, int c) { d = d * P.beta(a, b, c); });
        for_valid(x_p, [&](double& d, int a, int b, int c) { d = d - phi(a, b, c); });
        if (av == 1 && pt == 4) {
            scale_valid(x_p, -1.0);
        } else if (av == 2 && pt == 4) {
            scale_valid(x_p, -2.0);
        } else if (av == 2 && pt == -4) {
            scale_valid(x_p, 2.0);
        } else if (av == 3 && pt == 4) {
            scale_valid(x_p, -4.0 / 3.0);
            copy_valid(x_p_tmp, b_p);
            for_valid(x_p_tmp, [&](double& d, int a, int b, int c) { d = d * P.gamma(a, b, c); });
            scale_valid(x_p_tmp, -1.0);
            for_valid(x_p, [&](double& d, int a, int b, int c) { d = d + x_p_tmp(a, b, c); });
        } else if (av == 3 && pt == -4) {
            scale_valid(x_p, 4.0 / 3.0);
            copy_valid(x_p_tmp, b_p);
            for_valid(x_p_tmp, [&](double& d, int a, int b, int c) { d = d * P.gamma(a, b, c); });
            for_valid(x_p, [&](double& d, int a, int b, int c) { d = d + x_p_tmp(a, b, c); });
        }
        break;
    }
    default:
        return;  // rejected before the solve starts
    }
    // mean removal (apply_precon.f90:433-460): the pressure always; with
    // theta alpha = 0 and no no-slip wall, each periodic velocity component
    double mean_p, mean_u[3];
    sum_umac_press(P.geo, x_p, x_u, &mean_p, mean_u);
    for_valid(x_p, [&](double& d, int, int, int) { d = d - mean_p; });
    if (theta_alpha == 0.0) {
        bool no_wall_is_no_slip = true;
        for (int i = 0; i < dm; ++i)
            if (bc_is_noslip(P.geo.bc_lo[i]) || bc_is_noslip(P.geo.bc_hi[i])) no_wall_is_no_slip = false;
        if (no_wall_is_no_slip)
            for (int i = 0; i < dm; ++i)
                if (P.geo.periodic(i)) for_valid(x_u[i], [&](double& d, int, int, int) { d = d - mean_u[i]; });
    }
}

// ---------------------------------------------------------------- GMRES pieces
static void rotmat(double a, double b, double& cs, double& sn) {
    if (b == 0.0) {
        cs = 1.0;
        sn = 0.0;
    } else if (std::fabs(b) > std::fabs(a)) {
        double temp = a / b;
        sn = 1.0 / std::sqrt(1.0 + temp * temp);
        cs = temp * sn;
    } else {
        double temp = b / a;
        cs = 1.0 / std::sqrt(1.0 + temp * temp);
        sn = temp * cs;
    }
}

// H is (m+1) x m, column-major with leading dimension m+1, 1-based helpers
struct Hess {
    int ld;
    std::vector<double> v;
    double& operator()(int r, int c) { return v[(size_t)(r - 1) + (size_t)ld * (c - 1)]; }
};

static void least_squares(int i, Hess& H, std::vector<double>& cs, std::vector<double>& sn, std::vector<double>& s) {
    for (int k = 1; k <= i - 1; ++k) {
        double temp = cs[k] * H(k, i) + sn[k] * H(k + 1, i);
        H(k + 1, i) = -sn[k] * H(k, i) + cs[k] * H(k + 1, i);
        H(k, i) = temp;
    }
    rotmat(H(i, i), H(i + 1, i), cs[i], sn[i]);
    double temp = cs[i] * s[i];
    s[i + 1] = -sn[i] * s[i];
    s[i] = temp;
    H(i, i) = cs[i] * H(i, i) + sn[i] * H(i + 1, i);
    H(i + 1, i) = 0.0;
}

// SolveUTriangular(k, H, s, y): solves the (k+1) x (k+1) upper triangle
static void solve_utri(int k, Hess& H, std::vector<double>& s, std::vector<double>& y) {
    y[k + 1] = s[k + 1] / H(k + 1, k + 1);
    for (int i = k; i >= 1; --i) {
        double dot = 0.0;
        for (int q = i + 1; q <= k + 1; ++q) dot = dot + H(i, q) * y[q];
        y[i] = (s[i] - dot) / H(i, i);
    }
}

static void make_vec(const Geo& g, Vec& v, int ng) {
    for (int d = 0; d < g.dm; ++d) v.u[d] = make_face(g, d, ng);
    v.p = make_cc(g, ng);
}

static double stokes_norm(const Geo& g, const Vec& v, double pw) {
    double nu = stag_l2_norm(g, v.u);
    double np = cc_l2_norm(g, v.p);
    np = pw * np;
    return std::sqrt(nu * nu + np * np);
}

static double stokes_dot(const Geo& g, const Vec& a, const Vec& b, double pw) {
    double ipv[3];
    stag_inner_prod(g, a.u, b.u, ipv);
    double ipp = cc_inner_prod(g, a.p, b.p);
    double s = 0.0;
    for (int d = 0; d < g.dm; ++d) s = s + ipv[d];
    return s + (pw * pw) * ipp;
}

static void vec_copy(const Geo& g, Vec& d, const Vec& s) {
    for (int i = 0; i < g.dm; ++i) copy_valid(d.u[i], s.u[i]);
    copy_valid(d.p, s.p);
}

// w = w - h * V   (copy V to tmp, tmp *= h, w -= tmp: gmres.f90:348-357)
static void vec_sub_scaled(const Geo& g, Vec& w, const Vec& V, double h) {
    for (int i = 0; i < g.dm; ++i)
        for_valid(w.u[i], [&](double& d, int a, int b, int c) { d = d - V.u[i](a, b, c) * h; });
    for_valid(w.p, [&](double& d, int a, int b, int c) { d = d - V.p(a, b, c) * h; });
}
static void vec_div(const Geo& g, Vec& v, double s) {
    for (int i = 0; i < g.dm; ++i) for_valid(v.u[i], [&](double& d, int, int, int) { d = d / s; });
    for_valid(v.p, [&](double& d, int, int, int) { d = d / s; });
}

static void push_hist(lmm_stats* st, double v) {
    if (st && st->n_history < LMM_HISTORY_MAX) st->history[st->n_history++] = v;
}

// ------------------------------------------------ the reference GMRES
int gmres(const Problem& P, const lmm_knobs& K, Vec& b, Vec& x, double* theta_alpha, double* norm_pre_rhs, lmm_stats* st) {
    const Geo& g = P.geo;
    const int dm = g.dm, m = K.gmres_max_inner;
    const double pw = K.p_norm_weight;
    Problem Ps = P;  // scaled copy of beta, gamma, beta_ed (gmres.f90:106-122)
    double theta = *theta_alpha;
    if (K.scale_factor != 1.0) {
        theta = theta * K.scale_factor;
        for (double& v : x.p.a) v = v * K.scale_factor;
        for (int i = 0; i < dm; ++i)
            for (double& v : b.u[i].a) v = v * K.scale_factor;
        for (double& v : Ps.beta.a) v = v * K.scale_factor;
        for (double& v : Ps.gamma.a) v = v * K.scale_factor;
        for (int e = 0; e < (dm == 2 ? 1 : 3); ++e)
            for (double& v : Ps.beta_ed[e].a) v = v * K.scale_factor;
    }
    Vec r, w, tmp;
    make_vec(g, r, 1);
    make_vec(g, w, 0);
    make_vec(g, tmp, 0);
    std::vector<Vec> V(m + 1);
    for (auto& v : V) make_vec(g, v, 0);
    std::vector<double> cs(m + 2), sn(m + 2), y(m + 2), s(m + 3);
    Hess H{m + 1, std::vector<double>((size_t)(m + 1) * m, 0.0)};
    int vc = 0, pvc = 0;

    apply_precon(Ps, K, theta, b.u, b.p, tmp.u, tmp.p, &vc, &pvc);
    double norm_pre_b = stokes_norm(g, tmp, pw);
    if (norm_pre_rhs) *norm_pre_rhs = norm_pre_b;
    double norm_b = stokes_norm(g, b, pw);
    if (st) { st->norm_b = norm_b; st->norm_pre_b = norm_pre_b; }
    int status = 0;
    if (norm_b <= 0.0) {
        for (int i = 0; i < dm; ++i) x.u[i].setval(0.0);
        x.p.setval(0.0);
    } else {
        int total_iter = 0, iter = 0, i_copy = 0;
        double norm_init_resid = 0, norm_resid = 0, norm_init_Stokes = 0, norm_resid_Stokes = 0;
        vc = 0;
        for (;;) {
            apply_matrix(Ps, theta, tmp.u, tmp.p, x.u, x.p);
            for (int i = 0; i < dm; ++i) {
                for_valid(tmp.u[i], [&](double& d, int a, int bb, int c) { d = d - b.u[i](a, bb, c); });
                scale_valid(tmp.u[i], -1.0);
            }
            for_valid(tmp.p, [&](double& d, int a, int bb, int c) { d = d - b.p(a, bb, c); });
            scale_valid(tmp.p, -1.0);
            norm_resid_Stokes = stokes_norm(g, tmp, pw);
            if (iter == 0) norm_init_Stokes = norm_resid_Stokes;
            int vtemp = vc;
            apply_precon(Ps, K, theta, tmp.u, tmp.p, r.u, r.p, &vc, &pvc);
            vc = vtemp;
            norm_resid = stokes_norm(g, r, pw);
            if (iter == 0) norm_init_resid = norm_resid;
            if (st) {
                st->norm_resid = norm_resid;
                st->norm_init_resid = norm_init_resid;
                st->norm_resid_true = norm_resid_Stokes;
                st->norm_init_true = norm_init_Stokes;
            }
            if (total_iter >= K.gmres_max_iter) { status = LMM_WARN_MAX_ITER; break; }
            if (total_iter >= K.gmres_min_iter) {
                if (norm_resid <= K.gmres_rel_tol * std::min(norm_pre_b, norm_init_resid)) {
                    if (norm_resid_Stokes >= 10 * K.gmres_rel_tol * std::min(norm_b, norm_init_Stokes))
                        status = LMM_WARN_RESID_MISMATCH;
                    break;
                } else if (norm_resid <= K.gmres_abs_tol) {
                    break;
                }
            }
            if (iter >= K.gmres_max_outer) { status = LMM_WARN_MAX_OUTER; break; }
            iter = iter + 1;
            vec_copy(g, V[0], r);
            vec_div(g, V[0], norm_resid);
            std::fill(s.begin(), s.end(), 0.0);
            s[1] = norm_resid;
            int i;
            for (i = 1; i <= m; ++i) {
                total_iter = total_iter + 1;
                i_copy = i;
                vec_copy(g, r, V[i - 1]);
                apply_matrix(Ps, theta, tmp.u, tmp.p, r.u, r.p);
                apply_precon(Ps, K, theta, tmp.u, tmp.p, w.u, w.p, &vc, &pvc);
                for (int k = 1; k <= i; ++k) {
                    H(k, i) = stokes_dot(g, w, V[k - 1], pw);
                    vec_sub_scaled(g, w, V[k - 1], H(k, i));
                }
                H(i + 1, i) = stokes_norm(g, w, pw);
                if (H(i + 1, i) != 0.0) {
                    vec_copy(g, V[i], w);
                    vec_div(g, V[i], H(i + 1, i));
                } else {
                    status = LMM_ERR_BREAKDOWN;
                    break;
                }
                least_squares(i, H, cs, sn, s);
                double norm_resid_est = std::fabs(s[i + 1]);
                push_hist(st, norm_resid_est);
                if (total_iter >= K.gmres_max_iter) break;
                if (total_iter >= K.gmres_min_iter) {
                    if (norm_resid_est <= K.gmres_rel_tol * std::min(norm_pre_b, norm_init_resid) ||
                        norm_resid_est <= K.gmres_abs_tol)
                        break;
                }
            }
            if (status == LMM_ERR_BREAKDOWN) break;
            solve_utri(i_copy - 1, H, s, y);
            for (int it = 1; it <= i_copy; ++it) {
                Vec& Vi = V[it - 1];
                scale_valid(Vi.p, y[it]);
                for_valid(x.p, [&](double& d, int a, int bb, int c) { d = d + Vi.p(a, bb, c); });
                for (int d = 0; d < dm; ++d) {
                    scale_valid(Vi.u[d], y[it]);
                    for_valid(x.u[d], [&](double& dd, int a, int bb, int c) { dd = dd + Vi.u[d](a, bb, c); });
                }
            }
        }
        if (st) {
            st->total_iter = total_iter;
            st->outer_iter = iter;
            st->vcycles = vc;
        }
        for (int i = 0; i < dm; ++i) internal_sync(x.u[i]);
    }
    if (K.scale_factor != 1.0) {
        theta = theta / K.scale_factor;
        for (double& v : x.p.a) v = v * (1.0 / K.scale_factor);
    }
    *theta_alpha = theta;
    if (st) st->pressure_vcycles = pvc;
    return status;
}

// ------------------------------------------------ flexible GMRES (new method)
// Right preconditioning: A M^-1 u = b, x = M^-1 u; Z_i = M^-1 V_i are kept.
// Stop when the true residual |b - A x| <= gmres_rel_tol * |b| (or
// gmres_abs_tol), checked at every restart exactly like the reference checks
// its preconditioned residual (gmres.f90:253-289).
int fgmres(const Problem& P, const lmm_knobs& K, Vec& b, Vec& x, double* theta_alpha, double* norm_pre_rhs, lmm_stats* st) {
    const Geo& g = P.geo;
    const int dm = g.dm, m = K.gmres_max_inner;
    const double pw = K.p_norm_weight;
    const double theta = *theta_alpha;
    Vec r, w, tmp;
    make_vec(g, r, 1);
    make_vec(g, w, 0);
    make_vec(g, tmp, 0);
    std::vector<Vec> V(m + 1), Z(m);
    for (auto& v : V) make_vec(g, v, 0);
    for (auto& z : Z) make_vec(g, z, 1);
    std::vector<double> cs(m + 2), sn(m + 2), y(m + 2), s(m + 3);
    Hess H{m + 1, std::vector<double>((size_t)(m + 1) * m, 0.0)};
    int vc = 0, pvc = 0;
    double norm_b = stokes_norm(g, b, pw);
    if (norm_pre_rhs) *norm_pre_rhs = 0.0;
    if (st) st->norm_b = norm_b;
    int status = 0;
    if (norm_b <= 0.0) {
        for (int i = 0; i < dm; ++i) x.u[i].setval(0.0);
        x.p.setval(0.0);
        return 0;
    }
    int total_iter = 0, iter = 0;
    double norm_init = 0.0;
    for (;;) {
        apply_matrix(P, theta, tmp.u, tmp.p, x.u, x.p);
        for (int i = 0; i < dm; ++i) {
            for_valid(tmp.u[i], [&](double& d, int a, int bb, int c) { d = d - b.u[i](a, bb, c); });
            scale_valid(tmp.u[i], -1.0);
        }
        for_valid(tmp.p, [&](double& d, int a, int bb, int c) { d = d - b.p(a, bb, c); });
        scale_valid(tmp.p, -1.0);
        double norm_r = stokes_norm(g, tmp, pw);
        if (iter == 0) norm_init = norm_r;
        if (st) { st->norm_resid_true = norm_r; st->norm_init_true = norm_init; st->norm_resid = norm_r; }
        if (total_iter >= K.gmres_min_iter &&
            (norm_r <= K.gmres_rel_tol * norm_b || norm_r <= K.gmres_abs_tol))
            break;
        if (total_iter >= K.gmres_max_iter) { status = LMM_WARN_MAX_ITER; break; }
        if (iter >= K.gmres_max_outer) { status = LMM_WARN_MAX_OUTER; break; }
        iter = iter + 1;
        vec_copy(g, V[0], tmp);
        vec_div(g, V[0], norm_r);
        std::fill(s.begin(), s.end(), 0.0);
        s[1] = norm_r;
        int i, i_copy = 0;
        bool happy = false;
        for (i = 1; i <= m; ++i) {
            total_iter = total_iter + 1;
            i_copy = i;
            apply_precon(P, K, theta, V[i - 1].u, V[i - 1].p, Z[i - 1].u, Z[i - 1].p, &vc, &pvc);
            vec_copy(g, r, Z[i - 1]);
            apply_matrix(P, theta, w.u, w.p, r.u, r.p);
            for (int k = 1; k <= i; ++k) {
                H(k, i) = stokes_dot(g, w, V[k - 1], pw);
                vec_sub_scaled(g, w, V[k - 1], H(k, i));
            }
            H(i + 1, i) = stokes_norm(g, w, pw);
            if (H(i + 1, i) != 0.0) {
                vec_copy(g, V[i], w);
                vec_div(g, V[i], H(i + 1, i));
            } else {
                happy = true;
            }
            least_squares(i, H, cs, sn, s);
            double est = std::fabs(s[i + 1]);
            push_hist(st, est);
            if (happy || total_iter >= K.gmres_max_iter) break;
            if (total_iter >= K.gmres_min_iter && (est <= K.gmres_rel_tol * norm_b || est <= K.gmres_abs_tol)) break;
        }
        solve_utri(i_copy - 1, H, s, y);
        for (int it = 1; it <= i_copy; ++it) {
            Vec& Zi = Z[it - 1];
            for_valid(x.p, [&](double& d, int a, int bb, int c) { d = d + Zi.p(a, bb, c) * y[it]; });
            for (int d = 0; d < dm; ++d)
                for_valid(x.u[d], [&](double& dd, int a, int bb, int c) { dd = dd + Zi.u[d](a, bb, c) * y[it]; });
        }
    }
    for (int i = 0; i < dm; ++i) internal_sync(x.u[i]);
    if (st) {
        st->total_iter = total_iter;
        st->outer_iter = iter;
        st->vcycles = vc;
        st->pressure_vcycles = pvc;
    }
    return status;
}

}  // namespace orc
