// api.cpp - C entry points of the CPU oracle (liblmmoracle.so).
//
// TEST INFRASTRUCTURE ONLY.  The oracle restates the reference's Stokes
// solve (src_gmres/*.f90, src_common/stag_applyop.f90, div_and_grad.f90) on
// the CPU.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
// leg may load this library, and only as the checker / CPU baseline; the
// product (liblmmstokes.so) never calls it.
//
// Parity status: the reference cannot be built here (no Fortran compiler,
// BoxLib not vendored) and ships no tests or golden vectors, so this oracle
// is cross-checked against an independent numpy restatement
// (tests/golden/make_golden.py) and analytic/paper known answers rather than
// against reference outputs: parity unpinned.
#include "oracle_internal.hpp"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

using namespace orc;

namespace {

Geo geo_of(const lmm_grid* g) {
    Geo G;
    G.dm = g->dm;
    G.n[0] = g->n[0];
    G.n[1] = g->n[1];
    G.n[2] = (g->dm == 3) ? g->n[2] : 1;
    for (int d = 0; d < 3; ++d) {
        G.bc_lo[d] = (d < g->dm) ? g->bc_lo[d] : LMM_BC_PERIODIC;
        G.bc_hi[d] = (d < g->dm) ? g->bc_hi[d] : LMM_BC_PERIODIC;
    }
    return G;
}

// BoxLib-layout output of a wall-bounded problem: the valid region, then
// every ghost index mapped direction by direction -- periodic: its image;
// wall, face component normal to it: zero (the wall face hi+1 too); wall,
// otherwise: the nearest valid entry, negated for a transverse velocity at a
// no-slip wall.  kind: face component c (0..2) or -1 for cells.
void boxlib_from_fab_walls(double* dst, int dst_ng, const Fab& f, const Geo& G, int kind) {
    int slo[3], shi[3];
    for (int d = 0; d < 3; ++d) {
        int g = (d < f.dm) ? dst_ng : 0;
        slo[d] = f.vlo[d] - g;
        shi[d] = f.vhi[d] + g;
    }
    long sy = shi[0] - slo[0] + 1, sz = sy * (shi[1] - slo[1] + 1);
    for (int k = slo[2]; k <= shi[2]; ++k)
        for (int j = slo[1]; j <= shi[1]; ++j)
            for (int i = slo[0]; i <= shi[0]; ++i) {
                int idx[3] = {i, j, k};
                double sgn = 1.0;
                for (int d = 0; d < f.dm; ++d) {
                    const int n = f.n[d];
                    int& v = idx[d];
                    if (f.per[d]) {
                        v = wrap_to_valid(v, n, f.nodal[d]);
                        continue;
                    }
                    if (kind == d) {
                        if (v <= 0 || v >= n) sgn = 0.0;
                        v = (v < 0) ? 0 : (v > n - 1 ? n - 1 : v);
                        continue;
                    }
                    const bool slip_lo = bc_is_slip(G.bc_lo[d]), slip_hi = bc_is_slip(G.bc_hi[d]);
                    if (v < 0) {
                        v = 0;
                        if (kind >= 0 && !slip_lo) sgn = -sgn;
                    } else if (v > n - 1 + f.nodal[d]) {
                        v = n - 1 + f.nodal[d];
                        if (kind >= 0 && !slip_hi) sgn = -sgn;
                    }
                }
                double v = (sgn == 0.0) ? 0.0 : f(idx[0], idx[1], idx[2]);
                dst[(i - slo[0]) + sy * (j - slo[1]) + sz * (k - slo[2])] = (sgn < 0.0) ? -v : v;
            }
}

// copy a BoxLib array (ghost width src_ng, same nodality) into f (any ng):
// every index of f that exists in the source is copied.
void fab_from_boxlib(Fab& f, const double* src, int src_ng) {
    int slo[3], shi[3];
    for (int d = 0; d < 3; ++d) {
        int g = (d < f.dm) ? src_ng : 0;
        slo[d] = f.vlo[d] - g;
        shi[d] = f.vhi[d] + g;
    }
    long sy = shi[0] - slo[0] + 1, sz = sy * (shi[1] - slo[1] + 1);
    for (int k = f.lo[2]; k <= f.hi[2]; ++k)
        for (int j = f.lo[1]; j <= f.hi[1]; ++j)
            for (int i = f.lo[0]; i <= f.hi[0]; ++i) {
                if (i < slo[0] || i > shi[0] || j < slo[1] || j > shi[1] || k < slo[2] || k > shi[2]) continue;
                f(i, j, k) = src[(i - slo[0]) + sy * (j - slo[1]) + sz * (k - slo[2])];
            }
}
void boxlib_from_fab(double* dst, int dst_ng, const Fab& f) {
    int slo[3], shi[3];
    for (int d = 0; d < 3; ++d) {
        int g = (d < f.dm) ? dst_ng : 0;
        slo[d] = f.vlo[d] - g;
        shi[d] = f.vhi[d] + g;
    }
    long sy = shi[0] - slo[0] + 1, sz = sy * (shi[1] - slo[1] + 1);
    for (int k = slo[2]; k <= shi[2]; ++k)
        for (int j = slo[1]; j <= shi[1]; ++j)
            for (int i = slo[0]; i <= shi[0]; ++i) {
                int ii = wrap_to_valid(i, f.n[0], f.nodal[0]);
                int jj = wrap_to_valid(j, f.n[1], f.nodal[1]);
                int kk = (f.dm == 3) ? wrap_to_valid(k, f.n[2], f.nodal[2]) : k;
                bool inside = i >= f.lo[0] && i <= f.hi[0] && j >= f.lo[1] && j <= f.hi[1] && k >= f.lo[2] && k <= f.hi[2];
                dst[(i - slo[0]) + sy * (j - slo[1]) + sz * (k - slo[2])] = inside ? f(i, j, k) : f(ii, jj, kk);
            }
}

void load(Fab& f, const double* src, int layout, int ng) {
    if (layout == LMM_LAYOUT_BOXLIB)
        fab_from_boxlib(f, src, ng);
    else
        fab_from_compact(f, src);
}

bool build_problem(const lmm_grid* g, int visc_type, const lmm_fields_in* in, Problem& P) {
    P.geo = geo_of(g);
    P.dx = g->dx;
    P.visc_type = visc_type;
    const int dm = P.geo.dm;
    for (int i = 0; i < dm; ++i) {
        P.alpha_fc[i] = make_face(P.geo, i, 0);
        load(P.alpha_fc[i], in->alpha_fc[i], in->layout, in->ng_alpha);
    }
    P.beta = make_cc(P.geo, 1);
    load(P.beta, in->beta, in->layout, in->ng_beta);
    P.gamma = make_cc(P.geo, 1);
    if (in->gamma)
        load(P.gamma, in->gamma, in->layout, in->ng_gamma);
    else
        P.gamma.setval(0.0);
    for (int e = 0; e < (dm == 2 ? 1 : 3); ++e) {
        P.beta_ed[e] = make_edge(P.geo, e, 0);
        load(P.beta_ed[e], in->beta_ed[e], in->layout, in->ng_beta_ed);
    }
    return true;
}

// per direction: both sides periodic, or both walls (no-slip 100-103 or
// slip 200-203, bc.f90:23-35)
bool valid_grid(const lmm_grid* g) {
    if (!g || (g->dm != 2 && g->dm != 3)) return false;
    auto wall = [](int c) { return bc_is_noslip(c) || bc_is_slip(c); };
    for (int d = 0; d < g->dm; ++d) {
        if (g->n[d] < 2) return false;
        const bool per = g->bc_lo[d] == LMM_BC_PERIODIC && g->bc_hi[d] == LMM_BC_PERIODIC;
        if (!per && !(wall(g->bc_lo[d]) && wall(g->bc_hi[d]))) return false;
    }
    return g->dx > 0.0;
}

// zero the wall faces of a face array (the wall-normal component on its
// wall-bounded direction: faces lo and hi+1)
void zero_wall_faces(const Geo& G, Fab* u) {
    for (int c = 0; c < G.dm; ++c) {
        if (G.periodic(c)) continue;
        Fab& f = u[c];
        for (int k = f.vlo[2]; k <= f.vhi[2]; ++k)
            for (int j = f.vlo[1]; j <= f.vhi[1]; ++j)
                for (int i = f.vlo[0]; i <= f.vhi[0]; ++i) {
                    const int idx[3] = {i, j, k};
                    if (idx[c] == 0 || idx[c] == G.n[c]) f(i, j, k) = 0.0;
                }
    }
}

void faces_from_compact(const Geo& G, Fab* f, const double* const* src, int ng) {
    for (int i = 0; i < G.dm; ++i) {
        f[i] = make_face(G, i, ng);
        fab_from_compact(f[i], src[i]);
    }
}
void compact_from_faces(const Geo& G, double* const* dst, const Fab* f) {
    for (int i = 0; i < G.dm; ++i) compact_from_fab(dst[i], f[i]);
}

Geo level_geo(const Geo& G, int lev) {
    Geo c = G;
    for (int d = 0; d < G.dm; ++d) c.n[d] = G.n[d] >> lev;
    return c;
}

}  // namespace

extern "C" {

// probin_gmres.f90:119-157 defaults, visc_type default 1 (probin_common.f90:224)
void orc_default_knobs(lmm_knobs* k) {
    std::memset(k, 0, sizeof(*k));
    k->precon_type = 1;
    k->visc_schur_approx = 0;
    k->p_norm_weight = 1.0;
    k->scale_factor = 1.0;
    k->mg_verbose = 0;
    k->cg_verbose = 0;
    k->mg_max_vcycles = 1;
    k->mg_minwidth = 2;
    k->mg_bottom_solver = 4;
    k->mg_nsmooths_down = 2;
    k->mg_nsmooths_up = 2;
    k->mg_nsmooths_bottom = 8;
    k->mg_max_bottom_nlevels = 10;
    k->mg_rel_tol = 1e-9;
    k->stag_mg_verbosity = 0;
    k->stag_mg_max_vcycles = 1;
    k->stag_mg_minwidth = 2;
    k->stag_mg_bottom_solver = 4;
    k->stag_mg_nsmooths_down = 2;
    k->stag_mg_nsmooths_up = 2;
    k->stag_mg_nsmooths_bottom = 8;
    k->stag_mg_max_bottom_nlevels = 10;
    k->stag_mg_omega = 1.0;
    k->stag_mg_smoother = 1;
    k->stag_mg_rel_tol = 1e-9;
    k->gmres_rel_tol = 1e-9;
    k->gmres_abs_tol = 0.0;
    k->gmres_verbose = 1;
    k->gmres_max_outer = 20;
    k->gmres_max_inner = 5;
    k->gmres_max_iter = 100;
    k->gmres_min_iter = 1;
    k->visc_type = 1;
    k->method = LMM_METHOD_GMRES;
    k->precision = LMM_PRECISION_FP64;
    k->learned_stage = 0;
}

void orc_set_tile_size(int tx, int ty, int tz) {
    g_tile_size[0] = tx;
    g_tile_size[1] = ty;
    g_tile_size[2] = tz;
}

int orc_num_levels(const lmm_grid* g, int minwidth) { return compute_nlevs_mg(geo_of(g), minwidth); }

int orc_stokes_solve(const lmm_grid* g, const lmm_knobs* k, const lmm_fields_in* in, lmm_fields_out* out,
                     double* theta_alpha, double* norm_pre_rhs, lmm_stats* st) {
    if (!valid_grid(g) || !k || !in || !out || !theta_alpha) return LMM_ERR_INVALID;
    if (k->visc_schur_approx != 0 && k->visc_schur_approx != 1) return LMM_ERR_INVALID;
    if (k->visc_schur_approx == 1 && std::abs(k->visc_type) == 3) return LMM_ERR_INVALID;  // inverse_diag_lap.f90:135,246
    if (k->visc_schur_approx == 1 && geo_of(g).any_wall()) return LMM_ERR_INVALID;  // BFBt: periodic only here
    int apt = std::abs(k->precon_type);
    if (apt < 1 || apt > 5) return LMM_ERR_INVALID;
    if (st) std::memset(st, 0, sizeof(*st));
    Problem P;
    build_problem(g, k->visc_type, in, P);
    const Geo& G = P.geo;
    Vec b, x;
    for (int i = 0; i < G.dm; ++i) {
        b.u[i] = make_face(G, i, 0);
        load(b.u[i], in->b_u[i], in->layout, in->ng_b_u);
        x.u[i] = make_face(G, i, 1);
        load(x.u[i], out->x_u[i], out->layout, out->ng_x_u);
    }
    b.p = make_cc(G, 0);
    load(b.p, in->b_p, in->layout, in->ng_b_p);
    x.p = make_cc(G, 1);
    load(x.p, out->x_p, out->layout, out->ng_x_p);
    // wall-normal velocities on the walls are not unknowns: the rhs there is
    // taken as zero (the reference's preconditioner zeroes them in every
    // correction, so they only ever enter its true-residual check)
    zero_wall_faces(G, b.u);
    auto t0 = std::chrono::steady_clock::now();
    int status = (k->method == LMM_METHOD_FGMRES) ? fgmres(P, *k, b, x, theta_alpha, norm_pre_rhs, st)
                                                  : gmres(P, *k, b, x, theta_alpha, norm_pre_rhs, st);
    auto t1 = std::chrono::steady_clock::now();
    if (st) st->solve_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    const bool walls = G.any_wall();
    if (walls) zero_wall_faces(G, x.u);
    for (int i = 0; i < G.dm; ++i) {
        if (out->layout == LMM_LAYOUT_BOXLIB) {
            if (walls)
                boxlib_from_fab_walls(out->x_u[i], out->ng_x_u, x.u[i], G, i);
            else
                boxlib_from_fab(out->x_u[i], out->ng_x_u, x.u[i]);
        } else {
            compact_from_fab(out->x_u[i], x.u[i]);
        }
    }
    if (out->layout == LMM_LAYOUT_BOXLIB) {
        if (walls)
            boxlib_from_fab_walls(out->x_p, out->ng_x_p, x.p, G, -1);
        else
            boxlib_from_fab(out->x_p, out->ng_x_p, x.p);
    } else {
        compact_from_fab(out->x_p, x.p);
    }
    return status;
}

// ---- unit-level entry points (compact layout) ----
int orc_stag_applyop(const lmm_grid* g, int visc_type, const lmm_fields_in* c, double theta_alpha,
                     const double* const phi[3], double* const Lphi[3], int color) {
    if (!valid_grid(g)) return LMM_ERR_INVALID;
    Problem P;
    build_problem(g, visc_type, c, P);
    Level L0 = make_level0(P, theta_alpha);
    Fab ph[3], L[3];
    faces_from_compact(P.geo, ph, phi, 1);
    fill_vel(P.geo, ph);
    for (int i = 0; i < P.geo.dm; ++i) {
        L[i] = make_face(P.geo, i, 1);
        fab_from_compact(L[i], Lphi[i]);  // untouched colours keep their input
    }
    stag_applyop_level(L0, ph, L, color, visc_type);
    compact_from_faces(P.geo, Lphi, L);
    return 0;
}

int orc_coarse_coeffs(const lmm_grid* g, const lmm_knobs* k, const lmm_fields_in* c, double theta_alpha, int l,
                      double* const alpha[3], double* beta, double* const beta_ed[3], double* gamma) {
    if (!valid_grid(g)) return LMM_ERR_INVALID;
    Problem P;
    build_problem(g, k->visc_type, c, P);
    std::vector<Level> lev;
    build_levels(P, theta_alpha, k->stag_mg_minwidth, lev);
    if (l < 0 || l >= (int)lev.size()) return LMM_ERR_INVALID;
    const Level& L = lev[l];
    for (int i = 0; i < P.geo.dm; ++i) compact_from_fab(alpha[i], L.alpha[i]);
    compact_from_fab(beta, L.beta_cc);
    compact_from_fab(gamma, L.gamma_cc);
    for (int e = 0; e < (P.geo.dm == 2 ? 1 : 3); ++e) compact_from_fab(beta_ed[e], L.beta_ed[e]);
    return 0;
}

int orc_smooth(const lmm_grid* g, const lmm_knobs* k, const lmm_fields_in* c, double theta_alpha, int l,
               const double* const rhs[3], double* const phi[3], int color) {
    if (!valid_grid(g)) return LMM_ERR_INVALID;
    Problem P;
    build_problem(g, k->visc_type, c, P);
    std::vector<Level> lev;
    build_levels(P, theta_alpha, k->stag_mg_minwidth, lev);
    if (l < 0 || l >= (int)lev.size()) return LMM_ERR_INVALID;
    const Geo G = lev[l].geo;
    Fab ph[3], r[3], Lp[3];
    faces_from_compact(G, ph, phi, 1);
    faces_from_compact(G, r, rhs, 0);
    fill_vel(G, ph);
    for (int i = 0; i < G.dm; ++i) Lp[i] = make_face(G, i, 1);
    stag_applyop_level(lev[l], ph, Lp, color, k->visc_type);
    stag_mg_update(lev[l], ph, r, Lp, color, k->visc_type, k->stag_mg_omega);
    fill_vel(G, ph);
    compact_from_faces(G, phi, ph);
    return 0;
}

int orc_residual_restrict(const lmm_grid* g, const lmm_knobs* k, const lmm_fields_in* c, double theta_alpha, int l,
                          const double* const rhs[3], const double* const phi[3], double* const rhs_c[3]) {
    if (!valid_grid(g)) return LMM_ERR_INVALID;
    Problem P;
    build_problem(g, k->visc_type, c, P);
    std::vector<Level> lev;
    build_levels(P, theta_alpha, k->stag_mg_minwidth, lev);
    if (l < 0 || l + 1 >= (int)lev.size()) return LMM_ERR_INVALID;
    const Geo G = lev[l].geo, Gc = lev[l + 1].geo;
    Fab ph[3], r[3], Lp[3], rc[3];
    faces_from_compact(G, ph, phi, 1);
    faces_from_compact(G, r, rhs, 0);
    fill_vel(G, ph);
    for (int i = 0; i < G.dm; ++i) {
        Lp[i] = make_face(G, i, 1);
        rc[i] = make_face(Gc, i, 0);
    }
    stag_applyop_level(lev[l], ph, Lp, 0, k->visc_type);
    for (int j = 0; j < G.dm; ++j) {
        Fab& L = Lp[j];
        for (int kk = L.vlo[2]; kk <= L.vhi[2]; ++kk)
            for (int jj = L.vlo[1]; jj <= L.vhi[1]; ++jj)
                for (int i = L.vlo[0]; i <= L.vhi[0]; ++i) {
                    double v = L(i, jj, kk) - r[j](i, jj, kk);
                    L(i, jj, kk) = v * -1.0;
                }
    }
    fill_vel(G, Lp);
    stag_restriction(Gc, Lp, rc, false);
    for (int j = 0; j < G.dm; ++j) physbc_domainvel(Gc, rc[j], j);
    compact_from_faces(Gc, rhs_c, rc);
    return 0;
}

int orc_prolong_add(const lmm_grid* g, int l, const double* const phi_c[3], double* const phi_f[3]) {
    if (!valid_grid(g)) return LMM_ERR_INVALID;
    Geo G = level_geo(geo_of(g), l), Gc = level_geo(geo_of(g), l + 1);
    Fab pf[3], pc[3];
    faces_from_compact(G, pf, phi_f, 1);
    faces_from_compact(Gc, pc, phi_c, 1);
    fill_vel(Gc, pc);
    stag_prolongation(G, pf, pc);
    fill_vel(G, pf);
    compact_from_faces(G, phi_f, pf);
    return 0;
}

int orc_stag_mg_solver(const lmm_grid* g, const lmm_knobs* k, const lmm_fields_in* c, double theta_alpha,
                       const double* const rhs[3], double* const phi[3]) {
    if (!valid_grid(g)) return LMM_ERR_INVALID;
    Problem P;
    build_problem(g, k->visc_type, c, P);
    Fab ph[3], r[3];
    faces_from_compact(P.geo, ph, phi, 1);
    faces_from_compact(P.geo, r, rhs, 0);
    int vc = 0;
    stag_mg_solver(P, *k, theta_alpha, ph, r, &vc);
    compact_from_faces(P.geo, phi, ph);
    return 0;
}

int orc_apply_matrix(const lmm_grid* g, int visc_type, const lmm_fields_in* c, double theta_alpha,
                     const double* const x_u[3], const double* x_p, double* const b_u[3], double* b_p) {
    if (!valid_grid(g)) return LMM_ERR_INVALID;
    Problem P;
    build_problem(g, visc_type, c, P);
    Fab xu[3], bu[3];
    faces_from_compact(P.geo, xu, x_u, 1);
    for (int i = 0; i < P.geo.dm; ++i) bu[i] = make_face(P.geo, i, 0);
    Fab xp = make_cc(P.geo, 1), bp = make_cc(P.geo, 0);
    fab_from_compact(xp, x_p);
    apply_matrix(P, theta_alpha, bu, bp, xu, xp);
    compact_from_faces(P.geo, b_u, bu);
    compact_from_fab(b_p, bp);
    return 0;
}

int orc_apply_precon(const lmm_grid* g, const lmm_knobs* k, const lmm_fields_in* c, double theta_alpha,
                     const double* const b_u[3], const double* b_p, double* const x_u[3], double* x_p) {
    if (!valid_grid(g)) return LMM_ERR_INVALID;
    Problem P;
    build_problem(g, k->visc_type, c, P);
    Fab bu[3], xu[3];
    faces_from_compact(P.geo, bu, b_u, 0);
    for (int i = 0; i < P.geo.dm; ++i) xu[i] = make_face(P.geo, i, 0);
    Fab bp = make_cc(P.geo, 0), xp = make_cc(P.geo, 0);
    fab_from_compact(bp, b_p);
    int vc = 0, pvc = 0;
    apply_precon(P, *k, theta_alpha, bu, bp, xu, xp, &vc, &pvc);
    compact_from_faces(P.geo, x_u, xu);
    compact_from_fab(x_p, xp);
    return 0;
}

int orc_inner_prod(const lmm_grid* g, const double* const a_u[3], const double* a_p, const double* const b_u[3],
                   const double* b_p, double* out) {
    if (!valid_grid(g)) return LMM_ERR_INVALID;
    Geo G = geo_of(g);
    Fab au[3], bu[3];
    faces_from_compact(G, au, a_u, 0);
    faces_from_compact(G, bu, b_u, 0);
    Fab ap = make_cc(G, 0), bp = make_cc(G, 0);
    fab_from_compact(ap, a_p);
    fab_from_compact(bp, b_p);
    stag_inner_prod(G, au, bu, out);
    out[G.dm] = cc_inner_prod(G, ap, bp);
    return 0;
}

int orc_sum_umac_press(const lmm_grid* g, const double* const u[3], const double* p, double* out) {
    if (!valid_grid(g)) return LMM_ERR_INVALID;
    Geo G = geo_of(g);
    Fab uu[3];
    faces_from_compact(G, uu, u, 0);
    Fab pp = make_cc(G, 0);
    fab_from_compact(pp, p);
    sum_umac_press(G, pp, uu, &out[0], &out[1]);
    return 0;
}

// pressure multigrid alone: phi = V-cycle(s) of div(a grad phi) = rhs
int orc_macproject(const lmm_grid* g, const lmm_knobs* k, const double* const alpha_fc[3], const double* mac_rhs,
                   double* phi_out) {
    if (!valid_grid(g)) return LMM_ERR_INVALID;
    Problem P;
    P.geo = geo_of(g);
    P.dx = g->dx;
    Fab ainv[3];
    for (int i = 0; i < P.geo.dm; ++i) {
        Fab al = make_face(P.geo, i, 0);
        fab_from_compact(al, alpha_fc[i]);
        ainv[i] = make_face(P.geo, i, 0);
        ainv[i].setval(1.0);
        for (size_t q = 0; q < ainv[i].a.size(); ++q) ainv[i].a[q] = ainv[i].a[q] / al.a[q];
    }
    Fab rhs = make_cc(P.geo, 0), phi = make_cc(P.geo, 1);
    fab_from_compact(rhs, mac_rhs);
    int pvc = 0;
    macproject(P, *k, phi, ainv, rhs, &pvc);
    compact_from_fab(phi_out, phi);
    return 0;
}

}  // extern "C"
