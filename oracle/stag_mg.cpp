// stag_mg.cpp - CPU oracle: staggered geometric multigrid V-cycle.
//
// TEST INFRASTRUCTURE ONLY (the oracle).  Restates
//   src_gmres/stag_mg_layout.f90:179-222 (compute_nlevs_mg)
//   src_gmres/stag_mg_solver.f90:37-868  (stag_mg_solver)
//   src_gmres/stag_mg_solver.f90:873-1633 (cc/stag/nodal/edge restriction,
//                                          stag_prolongation)
// for one box.  Every multifab_fill_boundary of the reference is kept, and
// so are its physical-boundary fills (physbc.cpp), which act on
// wall-bounded directions only.
#include "oracle_internal.hpp"

#include <cmath>
#include <cstdio>

namespace orc {

int compute_nlevs_mg(const Geo& g, int minwidth) {
    int nlevs = -1;
    for (int d = 0; d < g.dm; ++d) {
        int temp = g.n[d];
        int rdir = 1;
        while (temp % 2 == 0 && temp / minwidth != 1) {
            temp = temp / 2;
            rdir = rdir + 1;
        }
        nlevs = (nlevs == -1) ? rdir : std::min(rdir, nlevs);
    }
    return nlevs;
}

// cc_restriction_2d/_3d (stag_mg_solver.f90:924-968) + fill_boundary (:918)
void cc_restriction(Fab& phi_c, const Fab& phi_f) {
    if (phi_c.dm == 2) {
        for (int j = 0; j < phi_c.n[1]; ++j)
            for (int i = 0; i < phi_c.n[0]; ++i)
                phi_c(i, j) = 0.25 * (phi_f(2 * i, 2 * j) + phi_f(2 * i + 1, 2 * j) + phi_f(2 * i, 2 * j + 1) + phi_f(2 * i + 1, 2 * j + 1));
    } else {
#pragma omp parallel for schedule(static)
        for (int k = 0; k < phi_c.n[2]; ++k)
            for (int j = 0; j < phi_c.n[1]; ++j)
                for (int i = 0; i < phi_c.n[0]; ++i)
                    phi_c(i, j, k) = 0.125 * (phi_f(2 * i, 2 * j, 2 * k) + phi_f(2 * i + 1, 2 * j, 2 * k) + phi_f(2 * i, 2 * j + 1, 2 * k) +
                                              phi_f(2 * i + 1, 2 * j + 1, 2 * k) + phi_f(2 * i, 2 * j, 2 * k + 1) + phi_f(2 * i + 1, 2 * j, 2 * k + 1) +
                                              phi_f(2 * i, 2 * j + 1, 2 * k + 1) + phi_f(2 * i + 1, 2 * j + 1, 2 * k + 1));
    }
    fill_boundary(phi_c);
}

// stag_restriction_2d/_3d (stag_mg_solver.f90:1033-1175)
void stag_restriction(const Geo& gc, const Fab* phi_f, Fab* phi_c, bool simple) {
    const int nx = gc.n[0], ny = gc.n[1];
    if (gc.dm == 2) {
        const Fab &fx = phi_f[0], &fy = phi_f[1];
        Fab &cx = phi_c[0], &cy = phi_c[1];
        if (simple) {
            for (int j = 0; j <= ny - 1; ++j)
                for (int i = 0; i <= nx; ++i) cx(i, j) = 0.5 * (fx(2 * i, 2 * j) + fx(2 * i, 2 * j + 1));
            for (int j = 0; j <= ny; ++j)
                for (int i = 0; i <= nx - 1; ++i) cy(i, j) = 0.5 * (fy(2 * i, 2 * j) + fy(2 * i + 1, 2 * j));
        } else {
            for (int j = 0; j <= ny - 1; ++j)
                for (int i = 0; i <= nx; ++i)
                    cx(i, j) = 0.25 * (fx(2 * i, 2 * j) + fx(2 * i, 2 * j + 1)) +
                               0.125 * (fx(2 * i + 1, 2 * j) + fx(2 * i + 1, 2 * j + 1) + fx(2 * i - 1, 2 * j) + fx(2 * i - 1, 2 * j + 1));
            for (int j = 0; j <= ny; ++j)
                for (int i = 0; i <= nx - 1; ++i)
                    cy(i, j) = 0.25 * (fy(2 * i, 2 * j) + fy(2 * i + 1, 2 * j)) +
                               0.125 * (fy(2 * i, 2 * j + 1) + fy(2 * i + 1, 2 * j + 1) + fy(2 * i, 2 * j - 1) + fy(2 * i + 1, 2 * j - 1));
        }
        return;
    }
    const int nz = gc.n[2];
    const Fab &fx = phi_f[0], &fy = phi_f[1], &fz = phi_f[2];
    Fab &cx = phi_c[0], &cy = phi_c[1], &cz = phi_c[2];
    if (simple) {
#pragma omp parallel for schedule(static)
        for (int k = 0; k <= nz - 1; ++k)
            for (int j = 0; j <= ny - 1; ++j)
                for (int i = 0; i <= nx; ++i)
                    cx(i, j, k) = 0.25 * (fx(2 * i, 2 * j, 2 * k) + fx(2 * i, 2 * j + 1, 2 * k) + fx(2 * i, 2 * j, 2 * k + 1) + fx(2 * i, 2 * j + 1, 2 * k + 1));
#pragma omp parallel for schedule(static)
        for (int k = 0; k <= nz - 1; ++k)
            for (int j = 0; j <= ny; ++j)
                for (int i = 0; i <= nx - 1; ++i)
                    cy(i, j, k) = 0.25 * (fy(2 * i, 2 * j, 2 * k) + fy(2 * i + 1, 2 * j, 2 * k) + fy(2 * i, 2 * j, 2 * k + 1) + fy(2 * i + 1, 2 * j, 2 * k + 1));
#pragma omp parallel for schedule(static)
        for (int k = 0; k <= nz; ++k)
            for (int j = 0; j <= ny - 1; ++j)
                for (int i = 0; i <= nx - 1; ++i)
                    cz(i, j, k) = 0.25 * (fz(2 * i, 2 * j, 2 * k) + fz(2 * i + 1, 2 * j, 2 * k) + fz(2 * i, 2 * j + 1, 2 * k) + fz(2 * i + 1, 2 * j + 1, 2 * k));
    } else {
#pragma omp parallel for schedule(static)
        for (int k = 0; k <= nz - 1; ++k)
            for (int j = 0; j <= ny - 1; ++j)
                for (int i = 0; i <= nx; ++i)
                    cx(i, j, k) = 0.125 * (fx(2 * i, 2 * j, 2 * k) + fx(2 * i, 2 * j + 1, 2 * k) + fx(2 * i, 2 * j, 2 * k + 1) + fx(2 * i, 2 * j + 1, 2 * k + 1)) +
                                  0.0625 * (fx(2 * i + 1, 2 * j, 2 * k) + fx(2 * i + 1, 2 * j + 1, 2 * k) + fx(2 * i + 1, 2 * j, 2 * k + 1) + fx(2 * i + 1, 2 * j + 1, 2 * k + 1)) +
                                  0.0625 * (fx(2 * i - 1, 2 * j, 2 * k) + fx(2 * i - 1, 2 * j + 1, 2 * k) + fx(2 * i - 1, 2 * j, 2 * k + 1) + fx(2 * i - 1, 2 * j + 1, 2 * k + 1));
#pragma omp parallel for schedule(static)
        for (int k = 0; k <= nz - 1; ++k)
            for (int j = 0; j <= ny; ++j)
                for (int i = 0; i <= nx - 1; ++i)
                    cy(i, j, k) = 0.125 * (fy(2 * i, 2 * j, 2 * k) + fy(2 * i + 1, 2 * j, 2 * k) + fy(2 * i, 2 * j, 2 * k + 1) + fy(2 * i + 1, 2 * j, 2 * k + 1)) +
                                  0.0625 * (fy(2 * i, 2 * j + 1, 2 * k) + fy(2 * i + 1, 2 * j + 1, 2 * k) + fy(2 * i, 2 * j + 1, 2 * k + 1) + fy(2 * i + 1, 2 * j + 1, 2 * k + 1)) +
                                  0.0625 * (fy(2 * i, 2 * j - 1, 2 * k) + fy(2 * i + 1, 2 * j - 1, 2 * k) + fy(2 * i, 2 * j - 1, 2 * k + 1) + fy(2 * i + 1, 2 * j - 1, 2 * k + 1));
#pragma omp parallel for schedule(static)
        for (int k = 0; k <= nz; ++k)
            for (int j = 0; j <= ny - 1; ++j)
                for (int i = 0; i <= nx - 1; ++i)
                    cz(i, j, k) = 0.125 * (fz(2 * i, 2 * j, 2 * k) + fz(2 * i + 1, 2 * j, 2 * k) + fz(2 * i, 2 * j + 1, 2 * k) + fz(2 * i + 1, 2 * j + 1, 2 * k)) +
                                  0.0625 * (fz(2 * i, 2 * j, 2 * k + 1) + fz(2 * i + 1, 2 * j, 2 * k + 1) + fz(2 * i, 2 * j + 1, 2 * k + 1) + fz(2 * i + 1, 2 * j + 1, 2 * k + 1)) +
                                  0.0625 * (fz(2 * i, 2 * j, 2 * k - 1) + fz(2 * i + 1, 2 * j, 2 * k - 1) + fz(2 * i, 2 * j + 1, 2 * k - 1) + fz(2 * i + 1, 2 * j + 1, 2 * k - 1));
    }
}

// nodal_restriction_2d (stag_mg_solver.f90:1229-1244) + internal_sync (:1223)
void nodal_restriction(Fab& phi_c, const Fab& phi_f) {
    for (int j = 0; j <= phi_c.n[1]; ++j)
        for (int i = 0; i <= phi_c.n[0]; ++i) phi_c(i, j) = phi_f(2 * i, 2 * j);
    internal_sync(phi_c);
}

// edge_restriction_3d (stag_mg_solver.f90:1326-1367) + internal_sync (:1318-1320)
void edge_restriction(const Fab* phi_f, Fab* phi_c) {
    const int nx = phi_c[0].n[0], ny = phi_c[0].n[1], nz = phi_c[0].n[2];
    for (int k = 0; k <= nz - 1; ++k)
        for (int j = 0; j <= ny; ++j)
            for (int i = 0; i <= nx; ++i) phi_c[0](i, j, k) = 0.5 * (phi_f[0](2 * i, 2 * j, 2 * k) + phi_f[0](2 * i, 2 * j, 2 * k + 1));
    for (int k = 0; k <= nz; ++k)
        for (int j = 0; j <= ny - 1; ++j)
            for (int i = 0; i <= nx; ++i) phi_c[1](i, j, k) = 0.5 * (phi_f[1](2 * i, 2 * j, 2 * k) + phi_f[1](2 * i, 2 * j + 1, 2 * k));
    for (int k = 0; k <= nz; ++k)
        for (int j = 0; j <= ny; ++j)
            for (int i = 0; i <= nx - 1; ++i) phi_c[2](i, j, k) = 0.5 * (phi_f[2](2 * i, 2 * j, 2 * k) + phi_f[2](2 * i + 1, 2 * j, 2 * k));
    for (int e = 0; e < 3; ++e) internal_sync(phi_c[e]);
}

// stag_prolongation_2d/_3d (stag_mg_solver.f90:1424-1633)
void stag_prolongation(const Geo& gf, Fab* phi_f, const Fab* phi_c) {
    if (gf.dm == 2) {
        Fab &fx = phi_f[0], &fy = phi_f[1];
        const Fab &cx = phi_c[0], &cy = phi_c[1];
        for (int j = 0; j <= gf.n[1] - 1; ++j)
            for (int i = 0; i <= gf.n[0]; ++i) {
                int joff = (j % 2 == 0) ? -1 : 1;
                if (i % 2 == 0)
                    fx(i, j) = fx(i, j) + 0.75 * cx(i / 2, j / 2) + 0.25 * cx(i / 2, j / 2 + joff);
                else
                    fx(i, j) = fx(i, j) + 0.375 * cx(i / 2, j / 2) + 0.125 * cx(i / 2, j / 2 + joff) + 0.375 * cx(i / 2 + 1, j / 2) +
                               0.125 * cx(i / 2 + 1, j / 2 + joff);
            }
        for (int j = 0; j <= gf.n[1]; ++j)
            for (int i = 0; i <= gf.n[0] - 1; ++i) {
                int ioff = (i % 2 == 0) ? -1 : 1;
                if (j % 2 == 0)
                    fy(i, j) = fy(i, j) + 0.75 * cy(i / 2, j / 2) + 0.25 * cy(i / 2 + ioff, j / 2);
                else
                    fy(i, j) = fy(i, j) + 0.375 * cy(i / 2, j / 2) + 0.125 * cy(i / 2 + ioff, j / 2) + 0.375 * cy(i / 2, j / 2 + 1) +
                               0.125 * cy(i / 2 + ioff, j / 2 + 1);
            }
        return;
    }
    const double nine16 = 9.0 / 16.0, three16 = 3.0 / 16.0, one16 = 1.0 / 16.0;
    const double nine32 = 9.0 / 32.0, three32 = 3.0 / 32.0, one32 = 1.0 / 32.0;
    Fab &fx = phi_f[0], &fy = phi_f[1], &fz = phi_f[2];
    const Fab &cx = phi_c[0], &cy = phi_c[1], &cz = phi_c[2];
#pragma omp parallel for schedule(static)
    for (int k = 0; k <= gf.n[2] - 1; ++k)
        for (int j = 0; j <= gf.n[1] - 1; ++j)
            for (int i = 0; i <= gf.n[0]; ++i) {
                int joff = (j % 2 == 0) ? -1 : 1;
                int koff = (k % 2 == 0) ? -1 : 1;
                if (i % 2 == 0)
                    fx(i, j, k) = fx(i, j, k) + nine16 * cx(i / 2, j / 2, k / 2) + three16 * cx(i / 2, j / 2 + joff, k / 2) +
                                  three16 * cx(i / 2, j / 2, k / 2 + koff) + one16 * cx(i / 2, j / 2 + joff, k / 2 + koff);
                else
                    fx(i, j, k) = fx(i, j, k) + nine32 * cx(i / 2, j / 2, k / 2) + three32 * cx(i / 2, j / 2 + joff, k / 2) +
                                  three32 * cx(i / 2, j / 2, k / 2 + koff) + one32 * cx(i / 2, j / 2 + joff, k / 2 + koff) +
                                  nine32 * cx(i / 2 + 1, j / 2, k / 2) + three32 * cx(i / 2 + 1, j / 2 + joff, k / 2) +
                                  three32 * cx(i / 2 + 1, j / 2, k / 2 + koff) + one32 * cx(i / 2 + 1, j / 2 + joff, k / 2 + koff);
            }
#pragma omp parallel for schedule(static)
    for (int k = 0; k <= gf.n[2] - 1; ++k)
        for (int j = 0; j <= gf.n[1]; ++j)
            for (int i = 0; i <= gf.n[0] - 1; ++i) {
                int ioff = (i % 2 == 0) ? -1 : 1;
                int koff = (k % 2 == 0) ? -1 : 1;
                if (j % 2 == 0)
                    fy(i, j, k) = fy(i, j, k) + nine16 * cy(i / 2, j / 2, k / 2) + three16 * cy(i / 2 + ioff, j / 2, k / 2) +
                                  three16 * cy(i / 2, j / 2, k / 2 + koff) + one16 * cy(i / 2 + ioff, j / 2, k / 2 + koff);
                else
                    fy(i, j, k) = fy(i, j, k) + nine32 * cy(i / 2, j / 2, k / 2) + three32 * cy(i / 2 + ioff, j / 2, k / 2) +
                                  three32 * cy(i / 2, j / 2, k / 2 + koff) + one32 * cy(i / 2 + ioff, j / 2, k / 2 + koff) +
                                  nine32 * cy(i / 2, j / 2 + 1, k / 2) + three32 * cy(i / 2 + ioff, j / 2 + 1, k / 2) +
                                  three32 * cy(i / 2, j / 2 + 1, k / 2 + koff) + one32 * cy(i / 2 + ioff, j / 2 + 1, k / 2 + koff);
            }
#pragma omp parallel for schedule(static)
    for (int k = 0; k <= gf.n[2]; ++k)
        for (int j = 0; j <= gf.n[1] - 1; ++j)
            for (int i = 0; i <= gf.n[0] - 1; ++i) {
                int ioff = (i % 2 == 0) ? -1 : 1;
                int joff = (j % 2 == 0) ? -1 : 1;
                if (k % 2 == 0)
                    fz(i, j, k) = fz(i, j, k) + nine16 * cz(i / 2, j / 2, k / 2) + three16 * cz(i / 2 + ioff, j / 2, k / 2) +
                                  three16 * cz(i / 2, j / 2 + joff, k / 2) + one16 * cz(i / 2 + ioff, j / 2 + joff, k / 2);
                else
                    fz(i, j, k) = fz(i, j, k) + nine32 * cz(i / 2, j / 2, k / 2) + three32 * cz(i / 2 + ioff, j / 2, k / 2) +
                                  three32 * cz(i / 2, j / 2 + joff, k / 2) + one32 * cz(i / 2 + ioff, j / 2 + joff, k / 2) +
                                  nine32 * cz(i / 2, j / 2, k / 2 + 1) + three32 * cz(i / 2 + ioff, j / 2, k / 2 + 1) +
                                  three32 * cz(i / 2, j / 2 + joff, k / 2 + 1) + one32 * cz(i / 2 + ioff, j / 2 + joff, k / 2 + 1);
            }
}

static Geo coarsen_geo(const Geo& g, int f) {
    Geo c = g;
    for (int d = 0; d < g.dm; ++d) c.n[d] = g.n[d] / f;
    if (g.dm == 2) c.n[2] = 1;
    return c;
}

// Level set-up and coefficient coarsening of stag_mg_solver.f90:144-230.
void build_levels(const Problem& P, double theta_alpha, int minwidth, std::vector<Level>& lev) {
    const int dm = P.geo.dm;
    const int nlevs = compute_nlevs_mg(P.geo, minwidth);
    lev.resize(nlevs);
    for (int n = 0; n < nlevs; ++n) {
        Level& L = lev[n];
        L.geo = coarsen_geo(P.geo, 1 << n);
        L.dx = P.dx * (double)(1 << n);  // dx_mg(n,:) = dx(1,:) * 2**(n-1)
        L.beta_cc = make_cc(L.geo, 1);
        L.gamma_cc = make_cc(L.geo, 1);
        for (int i = 0; i < dm; ++i) L.alpha[i] = make_face(L.geo, i, 0);
        for (int e = 0; e < (dm == 2 ? 1 : 3); ++e) L.beta_ed[e] = make_edge(L.geo, e, 0);
    }
    // copy level-1 coefficients (with ghosts for beta/gamma); alpha *= theta_alpha
    lev[0].beta_cc.a = P.beta.a;
    lev[0].gamma_cc.a = P.gamma.a;
    for (int e = 0; e < (dm == 2 ? 1 : 3); ++e) lev[0].beta_ed[e].a = P.beta_ed[e].a;
    for (int i = 0; i < dm; ++i) {
        lev[0].alpha[i].a = P.alpha_fc[i].a;
        for (double& v : lev[0].alpha[i].a) v = v * theta_alpha;
    }
    for (int n = 1; n < nlevs; ++n) {
        lev[n].beta_cc.setval(0.0);
        lev[n].gamma_cc.setval(0.0);
        cc_restriction(lev[n].beta_cc, lev[n - 1].beta_cc);
        cc_restriction(lev[n].gamma_cc, lev[n - 1].gamma_cc);
        stag_restriction(lev[n].geo, lev[n - 1].alpha, lev[n].alpha, true);
        if (dm == 2)
            nodal_restriction(lev[n].beta_ed[0], lev[n - 1].beta_ed[0]);
        else
            edge_restriction(lev[n - 1].beta_ed, lev[n].beta_ed);
    }
}

static double norm_inf_valid(const Fab& f) {
    double m = 0.0;
    for (int k = f.vlo[2]; k <= f.vhi[2]; ++k)
        for (int j = f.vlo[1]; j <= f.vhi[1]; ++j)
            for (int i = f.vlo[0]; i <= f.vhi[0]; ++i) m = std::max(m, std::fabs(f(i, j, k)));
    return m;
}

// physbc_domainvel + fill_boundary + physbc_macvel on every component
static void fill_all(const Geo& g, Fab* f) { fill_vel(g, f); }

// one pass of "nsmooths x colours" at level n (stag_mg_solver.f90:363-401)
static void smooth_level(const Level& L, Fab* phi, const Fab* rhs, Fab* Lphi, int nsmooths, int cstart, int cend,
                         int visc, double omega) {
    for (int m = 0; m < nsmooths; ++m)
        for (int color = cstart; color <= cend; ++color) {
            stag_applyop_level(L, phi, Lphi, color, visc);
            stag_mg_update(L, phi, rhs, Lphi, color, visc, omega);
            fill_all(L.geo, phi);
        }
}

// Lphi <- rhs - L phi, then ghost fill (stag_mg_solver.f90:406-434)
static void residual_level(const Level& L, const Fab* phi, const Fab* rhs, Fab* Lphi, int visc) {
    stag_applyop_level(L, phi, Lphi, 0, visc);
    for (int j = 0; j < L.geo.dm; ++j) {
        Fab& Lp = Lphi[j];
        const Fab& r = rhs[j];
        for (int k = Lp.vlo[2]; k <= Lp.vhi[2]; ++k)
            for (int jj = Lp.vlo[1]; jj <= Lp.vhi[1]; ++jj)
                for (int i = Lp.vlo[0]; i <= Lp.vhi[0]; ++i) {
                    double v = Lp(i, jj, k) - r(i, jj, k);
                    Lp(i, jj, k) = v * -1.0;
                }
    }
    fill_all(L.geo, Lphi);
}

void stag_mg_solver(const Problem& P, const lmm_knobs& K, double theta_alpha, Fab* phi_fc, const Fab* rhs_fc,
                    int* vcycle_counter) {
    const int dm = P.geo.dm;
    const int visc = P.visc_type;
    std::vector<Level> lev;
    build_levels(P, theta_alpha, K.stag_mg_minwidth, lev);
    const int nlevs_mg = (int)lev.size();

    std::vector<std::vector<Fab>> phi(nlevs_mg), rhs(nlevs_mg), Lphi(nlevs_mg);
    for (int n = 0; n < nlevs_mg; ++n) {
        phi[n].resize(dm);
        rhs[n].resize(dm);
        Lphi[n].resize(dm);
        for (int i = 0; i < dm; ++i) {
            rhs[n][i] = make_face(lev[n].geo, i, 0);
            phi[n][i] = make_face(lev[n].geo, i, 1);
            Lphi[n][i] = make_face(lev[n].geo, i, 1);
        }
    }
    // phi_fc_mg(1) = phi_fc (valid region), ghost fill; rhs copy (:236-257)
    for (int i = 0; i < dm; ++i) {
        Fab& p = phi[0][i];
        for (int k = p.vlo[2]; k <= p.vhi[2]; ++k)
            for (int j = p.vlo[1]; j <= p.vhi[1]; ++j)
                for (int ii = p.vlo[0]; ii <= p.vhi[0]; ++ii) {
                    p(ii, j, k) = phi_fc[i](ii, j, k);
                    rhs[0][i](ii, j, k) = rhs_fc[i](ii, j, k);
                }
    }
    fill_all(lev[0].geo, phi[0].data());
    // initial residual (:259-313)
    double resid0[3] = {0, 0, 0};
    stag_applyop_level(lev[0], phi[0].data(), Lphi[0].data(), 0, visc);
    for (int j = 0; j < dm; ++j) {
        Fab& Lp = Lphi[0][j];
        for (int k = Lp.vlo[2]; k <= Lp.vhi[2]; ++k)
            for (int jj = Lp.vlo[1]; jj <= Lp.vhi[1]; ++jj)
                for (int i = Lp.vlo[0]; i <= Lp.vhi[0]; ++i) Lp(i, jj, k) = Lp(i, jj, k) - rhs[0][j](i, jj, k);
        resid0[j] = norm_inf_valid(Lp);
    }
    bool all_zero = true, any_zero = false;
    for (int j = 0; j < dm; ++j) {
        all_zero = all_zero && resid0[j] == 0.0;
        any_zero = any_zero || resid0[j] == 0.0;
    }
    if (all_zero) return;  // phi_fc untouched
    if (any_zero) {
        double mx = 0.0;
        for (int j = 0; j < dm; ++j) mx = std::max(mx, resid0[j]);
        for (int j = 0; j < dm; ++j) resid0[j] = mx;
    }
    int cstart = (K.stag_mg_smoother == 0) ? 0 : 1;
    int cend = (K.stag_mg_smoother == 0) ? 0 : 2 * dm;

    for (int vcycle = 1; vcycle <= K.stag_mg_max_vcycles; ++vcycle) {
        for (int j = 0; j < dm; ++j)
            for (int n = 1; n < nlevs_mg; ++n) phi[n][j].setval(0.0);
        // down
        for (int n = 0; n < nlevs_mg - 1; ++n) {
            smooth_level(lev[n], phi[n].data(), rhs[n].data(), Lphi[n].data(), K.stag_mg_nsmooths_down, cstart, cend, visc,
                         K.stag_mg_omega);
            residual_level(lev[n], phi[n].data(), rhs[n].data(), Lphi[n].data(), visc);
            stag_restriction(lev[n + 1].geo, Lphi[n].data(), rhs[n + 1].data(), false);
            // residual zero on physical boundaries (:439-443)
            for (int j = 0; j < dm; ++j) physbc_domainvel(lev[n + 1].geo, rhs[n + 1][j], j);
        }
        // bottom: smooths at the coarsest level (one box, so the "fancy" bottom
        // solver condition n_cells/max_grid_size >= 2 of :450 is false)
        {
            int n = nlevs_mg - 1;
            smooth_level(lev[n], phi[n].data(), rhs[n].data(), Lphi[n].data(), K.stag_mg_nsmooths_bottom, cstart, cend, visc,
                         K.stag_mg_omega);
            residual_level(lev[n], phi[n].data(), rhs[n].data(), Lphi[n].data(), visc);
        }
        // up
        for (int n = nlevs_mg - 2; n >= 0; --n) {
            stag_prolongation(lev[n].geo, phi[n].data(), phi[n + 1].data());
            fill_all(lev[n].geo, phi[n].data());
            smooth_level(lev[n], phi[n].data(), rhs[n].data(), Lphi[n].data(), K.stag_mg_nsmooths_up, cstart, cend, visc,
                         K.stag_mg_omega);
        }
        // residual norms (:766-811)
        stag_applyop_level(lev[0], phi[0].data(), Lphi[0].data(), 0, visc);
        double resid[3];
        bool done = true;
        for (int j = 0; j < dm; ++j) {
            Fab& Lp = Lphi[0][j];
            for (int k = Lp.vlo[2]; k <= Lp.vhi[2]; ++k)
                for (int jj = Lp.vlo[1]; jj <= Lp.vhi[1]; ++jj)
                    for (int i = Lp.vlo[0]; i <= Lp.vhi[0]; ++i) Lp(i, jj, k) = Lp(i, jj, k) - rhs[0][j](i, jj, k);
            resid[j] = norm_inf_valid(Lp) / resid0[j];
            done = done && resid[j] < K.stag_mg_rel_tol;
        }
        if (done) break;
    }
    // copy back (:819-835); phi_fc keeps its own ghost width
    for (int j = 0; j < dm; ++j) {
        Fab& p = phi_fc[j];
        for (int k = p.vlo[2]; k <= p.vhi[2]; ++k)
            for (int jj = p.vlo[1]; jj <= p.vhi[1]; ++jj)
                for (int i = p.vlo[0]; i <= p.vhi[0]; ++i) p(i, jj, k) = phi[0][j](i, jj, k);
    }
    fill_all(P.geo, phi_fc);
    if (vcycle_counter) *vcycle_counter += dm * K.stag_mg_max_vcycles;
}

}  // namespace orc
