// oracle_internal.hpp - shared declarations of the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY (the oracle restating the reference algorithm).
#pragma once
#include "fab.hpp"
#include "../include/lmm_stokes.h"

#include <vector>

namespace orc {

// One level of the staggered hierarchy with its coefficients
// (beta_cc_mg, gamma_cc_mg: ng=1; alpha_fc_mg, beta_ed_mg: ng=0;
//  stag_mg_solver.f90:166-194).  alpha already holds theta*alpha.
struct Level {
    Geo geo;
    double dx;
    Fab alpha[3];
    Fab beta_cc;
    Fab beta_ed[3];
    Fab gamma_cc;
};

// The problem seen by gmres(...) at the finest level.
struct Problem {
    Geo geo;
    double dx;
    int visc_type;
    Fab alpha_fc[3];   // unscaled alpha_fc (ng=0)
    Fab beta;          // ng=1
    Fab beta_ed[3];    // ng=0
    Fab gamma;         // ng=1
};

// physbc.cpp (walls)
void physbc_domainvel(const Geo& g, Fab& s, int comp);
void physbc_macvel(const Geo& g, Fab& s, int comp);
void physbc_pres(const Geo& g, Fab& p);
void fill_vel(const Geo& g, Fab* u);
void fill_pres(const Geo& g, Fab& p);

// stag_ops.cpp
void stag_applyop_level(const Level& L, const Fab* phi, Fab* Lphi, int color, int visc);
void stag_mg_update(const Level& L, Fab* phi, const Fab* rhs, const Fab* Lphi, int color, int visc, double omega);

// stag_mg.cpp
int compute_nlevs_mg(const Geo& g, int minwidth);
void cc_restriction(Fab& phi_c, const Fab& phi_f);
void stag_restriction(const Geo& gc, const Fab* phi_f, Fab* phi_c, bool simple);
void nodal_restriction(Fab& phi_c, const Fab& phi_f);
void edge_restriction(const Fab* phi_f, Fab* phi_c);
void stag_prolongation(const Geo& gf, Fab* phi_f, const Fab* phi_c);
void build_levels(const Problem& P, double theta_alpha, int minwidth, std::vector<Level>& lev);
void stag_mg_solver(const Problem& P, const lmm_knobs& K, double theta_alpha, Fab* phi_fc, const Fab* rhs_fc,
                    int* vcycle_counter);

// div_grad.cpp
void compute_grad(const Geo& g, double dx, const Fab& phi, Fab* gradp);
void compute_div(const Geo& g, double dx, const Fab* phi_fc, Fab& div);

// norms.cpp
void stag_inner_prod(const Geo& g, const Fab* m1, const Fab* m2, double* prod);
double cc_inner_prod(const Geo& g, const Fab& m1, const Fab& m2);
double stag_l2_norm(const Geo& g, const Fab* m);
double cc_l2_norm(const Geo& g, const Fab& m);
void sum_umac_press(const Geo& g, const Fab& p, const Fab* u, double* av_p, double* av_u);

// ccmg.cpp (cell-centred pressure multigrid, this library's own design)
void macproject(const Problem& P, const lmm_knobs& K, Fab& phi, const Fab* alphainv_fc, const Fab& mac_rhs,
                int* pressure_vcycles);

// krylov.cpp
struct Vec {  // one Stokes vector (velocity faces + pressure cells)
    Fab u[3];
    Fab p;
};
Level make_level0(const Problem& P, double theta_alpha);
int gmres(const Problem& P, const lmm_knobs& K, Vec& b, Vec& x, double* theta_alpha, double* norm_pre_rhs, lmm_stats* st);
int fgmres(const Problem& P, const lmm_knobs& K, Vec& b, Vec& x, double* theta_alpha, double* norm_pre_rhs, lmm_stats* st);
void apply_matrix(const Problem& P, double theta_alpha, Fab* b_u, Fab& b_p, Fab* x_u, Fab& x_p);
void apply_precon(const Problem& P, const lmm_knobs& K, double theta_alpha, const Fab* b_u, const Fab& b_p,
                  Fab* x_u, Fab& x_p, int* vcycle_counter, int* pressure_vcycles);

// BoxLib tile size assumed for the tiled reductions (F_BaseLib default).
extern int g_tile_size[3];

}  // namespace orc
