// walls.cuh - launchers of the staggered multigrid kernels on a grid with
// walls (the kernels of kernels.cuh instantiated with W = true).  Included
// once per precision by walls_fp64.cu and walls_fp32.cu; the launchers of
// kernels.cuh hand every wall-bounded level here.
//
// The levels below the tail threshold run in the coarse tail kernel
// (tail.cuh, with its wall variant), as on a periodic grid.
#pragma once
#include "kernels.cuh"

namespace lmm {

template <class T>
void wl_applyop(const LevelDev<T>& L, int visc, const T* const phi[3], T* const out[3], cudaStream_t s, int color) {
    const T dxsqinv = T(1.0 / (L.dx * L.dx));
    if (color == 0) {
        const G3 gc = geom3(L.D.nx, L.D.ny, L.D.nz * L.D.dm);
        if (L.D.dm == 2) {
            LMM_VISC_DISPATCH(visc, launch_pdl(k_applyop_c<T, 2, V, true>, gc.grid, gc.block, 0, s, L.D, L.coef(), phi[0], phi[1], phi[2], out[0], out[1], out[2], dxsqinv))
        } else {
            LMM_VISC_DISPATCH(visc, launch_pdl(k_applyop_c<T, 3, V, true>, gc.grid, gc.block, 0, s, L.D, L.coef(), phi[0], phi[1], phi[2], out[0], out[1], out[2], dxsqinv))
        }
        return;
    }
    const G3 g = geom3(L.D.nx, L.D.ny, L.D.nz);
    if (L.D.dm == 2) {
        LMM_VISC_DISPATCH(visc, (launch_pdl(k_applyop<T, 2, V, true>, g.grid, g.block, 0, s, L.D, L.coef(), phi[0], phi[1], phi[2], out[0], out[1], out[2], dxsqinv, color)))
    } else {
        LMM_VISC_DISPATCH(visc, (launch_pdl(k_applyop<T, 3, V, true>, g.grid, g.block, 0, s, L.D, L.coef(), phi[0], phi[1], phi[2], out[0], out[1], out[2], dxsqinv, color)))
    }
}

template <class T>
void wl_gs_colour(const LevelDev<T>& L, int visc, int color, const T* const rhs[3], T* const phi[3], double omega, cudaStream_t s,
                  int reverse) {
    const T dxsqinv = T(1.0 / (L.dx * L.dx));
    const int comp = (color - 1) / 2;
    const int parity = (color % 2 == 1) ? 0 : 1;
    const T om = (T)omega;
    if (odd_level(L.D)) {
        const T* pin[3] = {phi[0], phi[1], phi[2]};
        T* lp[3] = {L.tmp[0], L.tmp[1], L.tmp[2]};
        wl_applyop<T>(L, visc, pin, lp, s, color);
        count_launch();
        const G3 go = geom3(L.D.nx, L.D.ny, L.D.nz);
#define CU(DM_, COMP_) launch_pdl(k_colour_update<T, DM_, V, COMP_, true>, go.grid, go.block, 0, s, L.D, L.coef(), rhs[COMP_], L.tmp[COMP_], phi[COMP_], parity, om, dxsqinv)
        if (L.D.dm == 2) {
            if (comp == 0) { LMM_VISC_DISPATCH(visc, CU(2, 0)) }
            else { LMM_VISC_DISPATCH(visc, CU(2, 1)) }
        } else {
            if (comp == 0) { LMM_VISC_DISPATCH(visc, CU(3, 0)) }
            else if (comp == 1) { LMM_VISC_DISPATCH(visc, CU(3, 1)) }
            else { LMM_VISC_DISPATCH(visc, CU(3, 2)) }
        }
#undef CU
        return;
    }
    const G3 g = geom3(L.D.nx / 2, L.D.ny, L.D.nz);
#define GS(DM_, COMP_) launch_pdl(k_gs_colour<T, DM_, V, COMP_, true>, g.grid, g.block, 0, s, L.D, L.coef(), rhs[COMP_], phi[0], phi[1], phi[2], parity, om, dxsqinv, reverse)
    if (L.D.dm == 2) {
        if (comp == 0) { LMM_VISC_DISPATCH(visc, GS(2, 0)) }
        else { LMM_VISC_DISPATCH(visc, GS(2, 1)) }
    } else {
        if (comp == 0) { LMM_VISC_DISPATCH(visc, GS(3, 0)) }
        else if (comp == 1) { LMM_VISC_DISPATCH(visc, GS(3, 1)) }
        else { LMM_VISC_DISPATCH(visc, GS(3, 2)) }
    }
#undef GS
}

template <class T>
void wl_jacobi(const LevelDev<T>& L, int visc, const T* const rhs[3], const T* const pin[3], T* const pout[3], double omega,
               cudaStream_t s) {
    const T dxsqinv = T(1.0 / (L.dx * L.dx));
    const G3 g = geom3(L.D.nx, L.D.ny, L.D.nz);
    const T om = (T)omega;
    if (L.D.dm == 2) {
        LMM_VISC_DISPATCH(visc, (launch_pdl(k_jacobi<T, 2, V, true>, g.grid, g.block, 0, s, L.D, L.coef(), rhs[0], rhs[1], rhs[2], pin[0], pin[1], pin[2], pout[0], pout[1], pout[2], om, dxsqinv)))
    } else {
        LMM_VISC_DISPATCH(visc, (launch_pdl(k_jacobi<T, 3, V, true>, g.grid, g.block, 0, s, L.D, L.coef(), rhs[0], rhs[1], rhs[2], pin[0], pin[1], pin[2], pout[0], pout[1], pout[2], om, dxsqinv)))
    }
}

template <class T>
void wl_residual_restrict(const LevelDev<T>& F, const LevelDev<T>& Cc, int visc, const T* const rhs_f[3], const T* const phi_f[3],
                          T* const rhs_c[3], cudaStream_t s) {
    const T dxsqinv = T(1.0 / (F.dx * F.dx));
    const G3 g = geom3(F.D.nx, F.D.ny, F.D.nz * F.D.dm);
    if (F.D.dm == 2) {
        LMM_VISC_DISPATCH(visc, (launch_pdl(k_residual_c<T, 2, V, true>, g.grid, g.block, 0, s, F.D, F.coef(), rhs_f[0], rhs_f[1], rhs_f[2], phi_f[0], phi_f[1], phi_f[2], F.tmp[0], F.tmp[1], F.tmp[2], dxsqinv)))
    } else {
        LMM_VISC_DISPATCH(visc, (launch_pdl(k_residual_c<T, 3, V, true>, g.grid, g.block, 0, s, F.D, F.coef(), rhs_f[0], rhs_f[1], rhs_f[2], phi_f[0], phi_f[1], phi_f[2], F.tmp[0], F.tmp[1], F.tmp[2], dxsqinv)))
    }
    count_launch();
    const G3 gc = geom3(Cc.D.nx, Cc.D.ny, Cc.D.nz);
    if (F.D.dm == 2)
        launch_pdl(k_restrict<T, 2, true>, gc.grid, gc.block, 0, s, F.D, F.tmp[0], F.tmp[1], F.tmp[2], Cc.D, rhs_c[0], rhs_c[1], rhs_c[2]);
    else
        launch_pdl(k_restrict<T, 3, true>, gc.grid, gc.block, 0, s, F.D, F.tmp[0], F.tmp[1], F.tmp[2], Cc.D, rhs_c[0], rhs_c[1], rhs_c[2]);
}

template <class T>
void wl_prolong_add(const LevelDev<T>& F, const LevelDev<T>& Cc, const T* const phi_c[3], T* const phi_f[3], cudaStream_t s) {
    const G3 g = geom3(F.D.nx, F.D.ny, F.D.nz);
    if (F.D.dm == 2)
        launch_pdl(k_prolong_add<T, 2, true>, g.grid, g.block, 0, s, F.D, Cc.D, phi_c[0], phi_c[1], phi_c[2], phi_f[0], phi_f[1], phi_f[2]);
    else
        launch_pdl(k_prolong_add<T, 3, true>, g.grid, g.block, 0, s, F.D, Cc.D, phi_c[0], phi_c[1], phi_c[2], phi_f[0], phi_f[1], phi_f[2]);
}

#define LMM_INSTANTIATE_WALLS(T)                                                                                           \
    template void wl_applyop<T>(const LevelDev<T>&, int, const T* const[3], T* const[3], cudaStream_t, int);              \
    template void wl_gs_colour<T>(const LevelDev<T>&, int, int, const T* const[3], T* const[3], double, cudaStream_t, int); \
    template void wl_jacobi<T>(const LevelDev<T>&, int, const T* const[3], const T* const[3], T* const[3], double,         \
                               cudaStream_t);                                                                              \
    template void wl_residual_restrict<T>(const LevelDev<T>&, const LevelDev<T>&, int, const T* const[3],                  \
                                          const T* const[3], T* const[3], cudaStream_t);                                   \
    template void wl_prolong_add<T>(const LevelDev<T>&, const LevelDev<T>&, const T* const[3], T* const[3], cudaStream_t);

}  // namespace lmm
