// ccmg.cpp - CPU oracle: cell-centred pressure multigrid (MAC projection).
//
// TEST INFRASTRUCTURE ONLY (the oracle).  Restates the front end of
//   src_gmres/macproject.f90:34-318 (macproject / mac_multigrid):
//   phi = 0, solve L_alpha Phi = mac_rhs with face coefficient 1/alpha_fc
//   (the reference negates alphainv_fc for BoxLib's sign convention,
//   :86-91, so the equation solved is div((1/alpha) grad Phi) = mac_rhs),
//   then fill phi's ghost cells (:302-306).
// The multigrid arithmetic itself lives in BoxLib F_MG (ml_cc_solve), which
// is not part of the reference tree.  This file defines this library's OWN
// cell-centred V-cycle, shared bit-for-bit with the GPU kernels:
//   * levels: the compute_nlevs_mg halving rule with mg_minwidth;
//   * face coefficients coarsened by averaging the 2^(dm-1) coincident fine
//     faces; residuals restricted by averaging the 2^dm children;
//   * red-black Gauss-Seidel on the cross (5/7-point) stencil, red
//     ((i+j+k) even) first, mg_nsmooths_down / _up sweeps, mg_nsmooths_bottom
//     sweeps at the coarsest level;
//   * piecewise-constant prolongation;
//   * mg_max_vcycles V-cycles from phi = 0;
//   * walls: homogeneous Neumann (the reference's BC_NEU for the pressure,
//     define_bc_tower.f90:285-294) as a zero face coefficient on the wall
//     faces, so no flux crosses them on any level.
#include "oracle_internal.hpp"

#include <vector>

namespace orc {

struct CcLevel {
    Geo geo;
    double dx;
    Fab a[3];   // face coefficients, ng=0
    Fab phi;    // ng=1
    Fab rhs;    // ng=0
    Fab res;    // ng=0
};

static double cc_lap(const CcLevel& L, const Fab& phi, int i, int j, int k, double dxsqinv) {
    const Fab &ax = L.a[0], &ay = L.a[1];
    double v = (ax(i + 1, j, k) * (phi(i + 1, j, k) - phi(i, j, k)) - ax(i, j, k) * (phi(i, j, k) - phi(i - 1, j, k))) +
               (ay(i, j + 1, k) * (phi(i, j + 1, k) - phi(i, j, k)) - ay(i, j, k) * (phi(i, j, k) - phi(i, j - 1, k)));
    if (L.geo.dm == 3) {
        const Fab& az = L.a[2];
        v = v + (az(i, j, k + 1) * (phi(i, j, k + 1) - phi(i, j, k)) - az(i, j, k) * (phi(i, j, k) - phi(i, j, k - 1)));
    }
    return v * dxsqinv;
}

static double cc_diag(const CcLevel& L, int i, int j, int k, double dxsqinv) {
    double s = L.a[0](i, j, k) + L.a[0](i + 1, j, k) + L.a[1](i, j, k) + L.a[1](i, j + 1, k);
    if (L.geo.dm == 3) s = s + L.a[2](i, j, k) + L.a[2](i, j, k + 1);
    return -(s * dxsqinv);
}

// one red-black sweep; the colour's updates read ghost cells filled before
// the colour started (Jacobi within a colour across the periodic seam)
static void cc_smooth(CcLevel& L, int nsweeps) {
    const double dxsqinv = 1.0 / (L.dx * L.dx);
    const int nz = (L.geo.dm == 3) ? L.geo.n[2] : 1;
    std::vector<double> upd;
    for (int s = 0; s < nsweeps; ++s)
        for (int color = 0; color < 2; ++color) {
            upd.assign(L.phi.a.size(), 0.0);
#pragma omp parallel for schedule(static)
            for (int k = 0; k < nz; ++k)
                for (int j = 0; j < L.geo.n[1]; ++j)
                    for (int i = 0; i < L.geo.n[0]; ++i) {
                        if (((i + j + k) & 1) != color) continue;
                        double r = L.rhs(i, j, k) - cc_lap(L, L.phi, i, j, k, dxsqinv);
                        double nv = L.phi(i, j, k) + r / cc_diag(L, i, j, k, dxsqinv);
                        upd[(size_t)(&L.phi(i, j, k) - L.phi.a.data())] = nv;
                    }
#pragma omp parallel for schedule(static)
            for (int k = 0; k < nz; ++k)
                for (int j = 0; j < L.geo.n[1]; ++j)
                    for (int i = 0; i < L.geo.n[0]; ++i)
                        if (((i + j + k) & 1) == color) L.phi(i, j, k) = upd[(size_t)(&L.phi(i, j, k) - L.phi.a.data())];
            fill_boundary(L.phi);
        }
}

static void cc_residual(CcLevel& L) {
    const double dxsqinv = 1.0 / (L.dx * L.dx);
    const int nz = (L.geo.dm == 3) ? L.geo.n[2] : 1;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < L.geo.n[1]; ++j)
            for (int i = 0; i < L.geo.n[0]; ++i) L.res(i, j, k) = L.rhs(i, j, k) - cc_lap(L, L.phi, i, j, k, dxsqinv);
}

static void cc_average_down(Fab& c, const Fab& f, int dm) {
    const int nz = (dm == 3) ? c.n[2] : 1;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < c.n[1]; ++j)
            for (int i = 0; i < c.n[0]; ++i) {
                if (dm == 2)
                    c(i, j) = 0.25 * (f(2 * i, 2 * j) + f(2 * i + 1, 2 * j) + f(2 * i, 2 * j + 1) + f(2 * i + 1, 2 * j + 1));
                else
                    c(i, j, k) = 0.125 * (f(2 * i, 2 * j, 2 * k) + f(2 * i + 1, 2 * j, 2 * k) + f(2 * i, 2 * j + 1, 2 * k) +
                                          f(2 * i + 1, 2 * j + 1, 2 * k) + f(2 * i, 2 * j, 2 * k + 1) + f(2 * i + 1, 2 * j, 2 * k + 1) +
                                          f(2 * i, 2 * j + 1, 2 * k + 1) + f(2 * i + 1, 2 * j + 1, 2 * k + 1));
            }
}

void macproject(const Problem& P, const lmm_knobs& K, Fab& phi, const Fab* alphainv_fc, const Fab& mac_rhs,
                int* pressure_vcycles) {
    const int dm = P.geo.dm;
    const int nlev = compute_nlevs_mg(P.geo, K.mg_minwidth);
    std::vector<CcLevel> lev(nlev);
    for (int l = 0; l < nlev; ++l) {
        CcLevel& L = lev[l];
        L.geo = P.geo;
        for (int d = 0; d < dm; ++d) L.geo.n[d] = P.geo.n[d] >> l;
        L.dx = P.dx * (double)(1 << l);
        for (int d = 0; d < dm; ++d) L.a[d] = make_face(L.geo, d, 0);
        L.phi = make_cc(L.geo, 1);
        L.rhs = make_cc(L.geo, 0);
        L.res = make_cc(L.geo, 0);
    }
    for (int d = 0; d < dm; ++d) {
        lev[0].a[d].a = alphainv_fc[d].a;
        if (P.geo.periodic(d)) continue;
        Fab& a = lev[0].a[d];
        for (int k = a.vlo[2]; k <= a.vhi[2]; ++k)
            for (int j = a.vlo[1]; j <= a.vhi[1]; ++j)
                for (int i = a.vlo[0]; i <= a.vhi[0]; ++i) {
                    const int idx[3] = {i, j, k};
                    if (idx[d] == 0 || idx[d] == P.geo.n[d]) a(i, j, k) = 0.0;
                }
    }
    for (int l = 1; l < nlev; ++l) {
        Fab tmpc[3], tmpf[3];
        for (int d = 0; d < dm; ++d) { tmpf[d] = lev[l - 1].a[d]; tmpc[d] = lev[l].a[d]; }
        stag_restriction(lev[l].geo, tmpf, tmpc, true);
        for (int d = 0; d < dm; ++d) lev[l].a[d] = tmpc[d];
    }
    for (int k = lev[0].rhs.vlo[2]; k <= lev[0].rhs.vhi[2]; ++k)
        for (int j = lev[0].rhs.vlo[1]; j <= lev[0].rhs.vhi[1]; ++j)
            for (int i = lev[0].rhs.vlo[0]; i <= lev[0].rhs.vhi[0]; ++i) lev[0].rhs(i, j, k) = mac_rhs(i, j, k);
    lev[0].phi.setval(0.0);

    for (int vc = 0; vc < K.mg_max_vcycles; ++vc) {
        for (int l = 1; l < nlev; ++l) lev[l].phi.setval(0.0);
        for (int l = 0; l < nlev - 1; ++l) {
            cc_smooth(lev[l], K.mg_nsmooths_down);
            cc_residual(lev[l]);
            cc_average_down(lev[l + 1].rhs, lev[l].res, dm);
        }
        cc_smooth(lev[nlev - 1], K.mg_nsmooths_bottom);
        for (int l = nlev - 2; l >= 0; --l) {
            CcLevel &F = lev[l], &C = lev[l + 1];
            const int nz = (dm == 3) ? F.geo.n[2] : 1;
            for (int k = 0; k < nz; ++k)
                for (int j = 0; j < F.geo.n[1]; ++j)
                    for (int i = 0; i < F.geo.n[0]; ++i) F.phi(i, j, k) = F.phi(i, j, k) + C.phi(i / 2, j / 2, k / 2);
            fill_boundary(F.phi);
            cc_smooth(F, K.mg_nsmooths_up);
        }
    }
    // phi out (ghosts filled)
    for (int k = phi.vlo[2]; k <= phi.vhi[2]; ++k)
        for (int j = phi.vlo[1]; j <= phi.vhi[1]; ++j)
            for (int i = phi.vlo[0]; i <= phi.vhi[0]; ++i) phi(i, j, k) = lev[0].phi(i, j, k);
    fill_pres(P.geo, phi);  // macproject.f90:302-306
    if (pressure_vcycles) *pressure_vcycles += K.mg_max_vcycles;
}

}  // namespace orc
