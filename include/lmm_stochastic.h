/* lmm_stochastic.h - the stochastic momentum forcing that the overdamped
 * integrator solves for (src_common/stochastic_m_fluxdiv.f90, called from
 * advance_timestep_overdamped.f90:200-207), generated on the GPU.
 *
 * b_u = div(S) on the faces of a periodic box, where S is the symmetric
 * stochastic stress of one random stage: diagonal components at cells
 * N(0,2), one N(0,1) value per edge (3D; node in 2D) shared by both
 * off-diagonal components, every value scaled by sqrt(2 kT / (dV dt)) and
 * sqrt(eta) at its location (eta_cc at cells, eta_ed at nodes / xy, xz, yz
 * edges), dV = dx^dm.  The random numbers are counter-based: the same seed
 * gives the same field on any device.  Arrays are device arrays in the
 * compact layout; asynchronous on `stream`. */
#ifndef LMM_STOCHASTIC_H
#define LMM_STOCHASTIC_H

#ifdef __cplusplus
extern "C" {
#endif

int lmm_stochastic_rhs(int dm, const int n[3], double dx, double dt, double kT, const double* eta_cc,
                       const double* const eta_ed[3], unsigned long long seed, double* const b_u[3], void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LMM_STOCHASTIC_H */
