// stag_ops.cpp - CPU oracle: staggered viscous operator and smoother update.
//
// TEST INFRASTRUCTURE ONLY (the oracle): a restatement of
//   src_common/stag_applyop.f90:204-1067  (stag_applyop_2d / _3d)
//   src_gmres/stag_mg_solver.f90:1637-2463 (stag_mg_update, _2d / _3d)
// on BoxLib-style single-box arrays (fab.hpp).  Expressions keep the
// reference's operand order so that, compiled without floating-point
// contraction, every face value is the reference's rounding sequence.
#include "oracle_internal.hpp"

#include <cstdio>

namespace orc {

// colour bookkeeping of stag_applyop.f90:548-575 / stag_mg_solver.f90:2078-2104
struct Colour {
    bool do_c[3];
    int offset;
};
static Colour colour_of(int color) {
    Colour c{{true, true, true}, 1};
    if (color == 1 || color == 2) { c.do_c[1] = c.do_c[2] = false; c.offset = 2; }
    else if (color == 3 || color == 4) { c.do_c[0] = c.do_c[2] = false; c.offset = 2; }
    else if (color == 5 || color == 6) { c.do_c[0] = c.do_c[1] = false; c.offset = 2; }
    return c;
}
static inline int ioff_of(int offset, int xlo, int j, int k, int color) {
    // mod(xlo(1)+j+k,2) .ne. mod(color+1,2) => ioff = 1  (all indices >= -1 here)
    return (offset == 2 && (((xlo + j + k) % 2 + 2) % 2) != ((color + 1) % 2)) ? 1 : 0;
}

// ---------------------------------------------------------------- 2D
static void applyop_2d(const Fab* phi, Fab* Lp, const Fab* alpha, const Fab& beta,
                       const Fab& beta_ed, const Fab& gamma, double dx, int color, int visc) {
    const Fab &phix = phi[0], &phiy = phi[1];
    Fab &Lpx = Lp[0], &Lpy = Lp[1];
    const Fab &alphax = alpha[0], &alphay = alpha[1];
    Colour col = colour_of(color);
    double dxsq = dx * dx;
    double dxsqinv = 1.0 / dxsq;
    double onethird = 1.0 / 3.0, twothirds = 2.0 / 3.0, fourthirds = 4.0 / 3.0;
    const int xlo = 0;
    double b = beta(0, 0), c = gamma(0, 0);

    if (col.do_c[0]) {
#pragma omp parallel for schedule(static)
        for (int j = Lpx.vlo[1]; j <= Lpx.vhi[1]; ++j) {
            int ioff = ioff_of(col.offset, xlo, j, 0, color);
            for (int i = Lpx.vlo[0] + ioff; i <= Lpx.vhi[0]; i += col.offset) {
                double v = 0.0;
                switch (visc) {
                case -1:
                    v = phix(i, j) * (alphax(i, j) + (beta(i, j) + beta(i - 1, j) + beta_ed(i, j + 1) + beta_ed(i, j)) * dxsqinv) -
                        (phix(i + 1, j) * beta(i, j) + phix(i - 1, j) * beta(i - 1, j) + phix(i, j + 1) * beta_ed(i, j + 1) +
                         phix(i, j - 1) * beta_ed(i, j)) * dxsqinv;
                    break;
                case 1:
                    v = phix(i, j) * (alphax(i, j) + 4.0 * b * dxsqinv) -
                        (phix(i + 1, j) + phix(i - 1, j) + phix(i, j + 1) + phix(i, j - 1)) * b * dxsqinv;
                    break;
                case -2:
                    v = phix(i, j) * (alphax(i, j) + (2.0 * beta(i, j) + 2.0 * beta(i - 1, j) + beta_ed(i, j + 1) + beta_ed(i, j)) * dxsqinv) -
                        (2.0 * phix(i + 1, j) * beta(i, j) + 2.0 * phix(i - 1, j) * beta(i - 1, j) + phix(i, j + 1) * beta_ed(i, j + 1) +
                         phix(i, j - 1) * beta_ed(i, j) + phiy(i, j + 1) * beta_ed(i, j + 1) - phiy(i, j) * beta_ed(i, j) -
                         phiy(i - 1, j + 1) * beta_ed(i, j + 1) + phiy(i - 1, j) * beta_ed(i, j)) * dxsqinv;
                    break;
                case 2:
                    v = phix(i, j) * (alphax(i, j) + 6.0 * b * dxsqinv) -
                        (2.0 * phix(i + 1, j) + 2.0 * phix(i - 1, j) + phix(i, j + 1) + phix(i, j - 1) + phiy(i, j + 1) - phiy(i, j) -
                         phiy(i - 1, j + 1) + phiy(i - 1, j)) * b * dxsqinv;
                    break;
                case -3:
                    v = phix(i, j) * (alphax(i, j) + (fourthirds * beta(i, j) + gamma(i, j) + fourthirds * beta(i - 1, j) + gamma(i - 1, j) +
                                                      beta_ed(i, j + 1) + beta_ed(i, j)) * dxsqinv) -
                        (phix(i + 1, j) * (fourthirds * beta(i, j) + gamma(i, j)) + phix(i - 1, j) * (fourthirds * beta(i - 1, j) + gamma(i - 1, j)) +
                         phix(i, j + 1) * beta_ed(i, j + 1) + phix(i, j - 1) * beta_ed(i, j) +
                         phiy(i, j + 1) * (beta_ed(i, j + 1) - twothirds * beta(i, j) + gamma(i, j)) -
                         phiy(i, j) * (beta_ed(i, j) - twothirds * beta(i, j) + gamma(i, j)) -
                         phiy(i - 1, j + 1) * (beta_ed(i, j + 1) - twothirds * beta(i - 1, j) + gamma(i - 1, j)) +
                         phiy(i - 1, j) * (beta_ed(i, j) - twothirds * beta(i - 1, j) + gamma(i - 1, j))) * dxsqinv;
                    break;
                case 3:
                    v = phix(i, j) * (alphax(i, j) + (14.0 * b * onethird + 2.0 * c) * dxsqinv) -
                        ((phix(i + 1, j) + phix(i - 1, j)) * (fourthirds * b + c) + (phix(i, j + 1) + phix(i, j - 1)) * b +
                         (phiy(i, j + 1) - phiy(i, j) - phiy(i - 1, j + 1) + phiy(i - 1, j)) * (onethird * b + c)) * dxsqinv;
                    break;
                }
                Lpx(i, j) = v;
            }
        }
    }
    if (col.do_c[1]) {
#pragma omp parallel for schedule(static)
        for (int j = Lpy.vlo[1]; j <= Lpy.vhi[1]; ++j) {
            int ioff = ioff_of(col.offset, xlo, j, 0, color);
            for (int i = Lpy.vlo[0] + ioff; i <= Lpy.vhi[0]; i += col.offset) {
                double v = 0.0;
                switch (visc) {
                case -1:
                    v = phiy(i, j) * (alphay(i, j) + (beta(i, j) + beta(i, j - 1) + beta_ed(i + 1, j) + beta_ed(i, j)) * dxsqinv) -
                        (phiy(i, j + 1) * beta(i, j) + phiy(i, j - 1) * beta(i, j - 1) + phiy(i + 1, j) * beta_ed(i + 1, j) +
                         phiy(i - 1, j) * beta_ed(i, j)) * dxsqinv;
                    break;
                case 1:
                    v = phiy(i, j) * (alphay(i, j) + 4.0 * b * dxsqinv) -
                        (phiy(i, j + 1) + phiy(i, j - 1) + phiy(i + 1, j) + phiy(i - 1, j)) * b * dxsqinv;
                    break;
                case -2:
                    v = phiy(i, j) * (alphay(i, j) + (2.0 * beta(i, j) + 2.0 * beta(i, j - 1) + beta_ed(i + 1, j) + beta_ed(i, j)) * dxsqinv) -
                        (2.0 * phiy(i, j + 1) * beta(i, j) + 2.0 * phiy(i, j - 1) * beta(i, j - 1) + phiy(i + 1, j) * beta_ed(i + 1, j) +
                         phiy(i - 1, j) * beta_ed(i, j) + phix(i + 1, j) * beta_ed(i + 1, j) - phix(i, j) * beta_ed(i, j) -
                         phix(i + 1, j - 1) * beta_ed(i + 1, j) + phix(i, j - 1) * beta_ed(i, j)) * dxsqinv;
                    break;
                case 2:
                    v = phiy(i, j) * (alphay(i, j) + 6.0 * b * dxsqinv) -
                        (2.0 * phiy(i, j + 1) + 2.0 * phiy(i, j - 1) + phiy(i + 1, j) + phiy(i - 1, j) + phix(i + 1, j) - phix(i, j) -
                         phix(i + 1, j - 1) + phix(i, j - 1)) * b * dxsqinv;
                    break;
                case -3:
                    v = phiy(i, j) * (alphay(i, j) + (fourthirds * beta(i, j) + gamma(i, j) + fourthirds * beta(i, j - 1) + gamma(i, j - 1) +
                                                      beta_ed(i + 1, j) + beta_ed(i, j)) * dxsqinv) -
                        (phiy(i, j + 1) * (fourthirds * beta(i, j) + gamma(i, j)) + phiy(i, j - 1) * (fourthirds * beta(i, j - 1) + gamma(i, j - 1)) +
                         phiy(i + 1, j) * beta_ed(i + 1, j) + phiy(i - 1, j) * beta_ed(i, j) +
                         phix(i + 1, j) * (beta_ed(i + 1, j) - twothirds * beta(i, j) + gamma(i, j)) -
                         phix(i, j) * (beta_ed(i, j) - twothirds * beta(i, j) + gamma(i, j)) -
                         phix(i + 1, j - 1) * (beta_ed(i + 1, j) - twothirds * beta(i, j - 1) + gamma(i, j - 1)) +
                         phix(i, j - 1) * (beta_ed(i, j) - twothirds * beta(i, j - 1) + gamma(i, j - 1))) * dxsqinv;
                    break;
                case 3:
                    v = phiy(i, j) * (alphay(i, j) + (14.0 * b * onethird + 2.0 * c) * dxsqinv) -
                        ((phiy(i, j + 1) + phiy(i, j - 1)) * (fourthirds * b + c) + (phiy(i + 1, j) + phiy(i - 1, j)) * b +
                         (phix(i + 1, j) - phix(i, j) - phix(i + 1, j - 1) + phix(i, j - 1)) * (onethird * b + c)) * dxsqinv;
                    break;
                }
                Lpy(i, j) = v;
            }
        }
    }
}

// ---------------------------------------------------------------- 3D
// x-face stencil of stag_applyop_3d; the y and z faces are the same formulas
// with the directions permuted, written out below like the reference does.
static void applyop_3d(const Fab* phi, Fab* Lp, const Fab* alpha, const Fab& beta,
                       const Fab* bed, const Fab& gamma, double dx, int color, int visc) {
    const Fab &phix = phi[0], &phiy = phi[1], &phiz = phi[2];
    const Fab &beta_xy = bed[0], &beta_xz = bed[1], &beta_yz = bed[2];
    Colour col = colour_of(color);
    double dxsq = dx * dx;
    double dxsqinv = 1.0 / dxsq;
    double onethird = 1.0 / 3.0, twothirds = 2.0 / 3.0, fourthirds = 4.0 / 3.0;
    const int xlo = 0;
    double b = beta(0, 0, 0), c = gamma(0, 0, 0);

    if (col.do_c[0]) {
        const Fab& alphax = alpha[0];
        Fab& Lpx = Lp[0];
#pragma omp parallel for schedule(static)
        for (int k = Lpx.vlo[2]; k <= Lpx.vhi[2]; ++k)
            for (int j = Lpx.vlo[1]; j <= Lpx.vhi[1]; ++j) {
                int ioff = ioff_of(col.offset, xlo, j, k, color);
                for (int i = Lpx.vlo[0] + ioff; i <= Lpx.vhi[0]; i += col.offset) {
                    double v = 0.0;
                    switch (visc) {
                    case -1:
                        v = phix(i, j, k) * (alphax(i, j, k) + (beta(i, j, k) + beta(i - 1, j, k) + beta_xy(i, j, k) + beta_xy(i, j + 1, k) +
                                                                beta_xz(i, j, k) + beta_xz(i, j, k + 1)) * dxsqinv) -
                            (phix(i + 1, j, k) * beta(i, j, k) + phix(i - 1, j, k) * beta(i - 1, j, k) + phix(i, j + 1, k) * beta_xy(i, j + 1, k) +
                             phix(i, j - 1, k) * beta_xy(i, j, k) + phix(i, j, k + 1) * beta_xz(i, j, k + 1) + phix(i, j, k - 1) * beta_xz(i, j, k)) * dxsqinv;
                        break;
                    case 1:
                        v = phix(i, j, k) * (alphax(i, j, k) + 6.0 * b * dxsqinv) -
                            (phix(i + 1, j, k) + phix(i - 1, j, k) + phix(i, j + 1, k) + phix(i, j - 1, k) + phix(i, j, k + 1) + phix(i, j, k - 1)) * b * dxsqinv;
                        break;
                    case -2:
                        v = phix(i, j, k) * (alphax(i, j, k) + (2.0 * beta(i, j, k) + 2.0 * beta(i - 1, j, k) + beta_xy(i, j, k) + beta_xy(i, j + 1, k) +
                                                                beta_xz(i, j, k) + beta_xz(i, j, k + 1)) * dxsqinv) -
                            (2.0 * phix(i + 1, j, k) * beta(i, j, k) + 2.0 * phix(i - 1, j, k) * beta(i - 1, j, k) + phix(i, j + 1, k) * beta_xy(i, j + 1, k) +
                             phix(i, j - 1, k) * beta_xy(i, j, k) + phix(i, j, k + 1) * beta_xz(i, j, k + 1) + phix(i, j, k - 1) * beta_xz(i, j, k) +
                             phiy(i, j + 1, k) * beta_xy(i, j + 1, k) - phiy(i, j, k) * beta_xy(i, j, k) - phiy(i - 1, j + 1, k) * beta_xy(i, j + 1, k) +
                             phiy(i - 1, j, k) * beta_xy(i, j, k) + phiz(i, j, k + 1) * beta_xz(i, j, k + 1) - phiz(i, j, k) * beta_xz(i, j, k) -
                             phiz(i - 1, j, k + 1) * beta_xz(i, j, k + 1) + phiz(i - 1, j, k) * beta_xz(i, j, k)) * dxsqinv;
                        break;
                    case 2:
                        v = phix(i, j, k) * (alphax(i, j, k) + 8.0 * b * dxsqinv) -
                            (2.0 * phix(i + 1, j, k) + 2.0 * phix(i - 1, j, k) + phix(i, j + 1, k) + phix(i, j - 1, k) + phix(i, j, k + 1) +
                             phix(i, j, k - 1) + phiy(i, j + 1, k) - phiy(i, j, k) - phiy(i - 1, j + 1, k) + phiy(i - 1, j, k) + phiz(i, j, k + 1) -
                             phiz(i, j, k) - phiz(i - 1, j, k + 1) + phiz(i - 1, j, k)) * b * dxsqinv;
                        break;
                    case -3:
                        v = phix(i, j, k) * (alphax(i, j, k) + (fourthirds * beta(i, j, k) + gamma(i, j, k) + fourthirds * beta(i - 1, j, k) +
                                                                gamma(i - 1, j, k) + beta_xy(i, j, k) + beta_xy(i, j + 1, k) + beta_xz(i, j, k) +
                                                                beta_xz(i, j, k + 1)) * dxsqinv) -
                            (phix(i + 1, j, k) * (fourthirds * beta(i, j, k) + gamma(i, j, k)) +
                             phix(i - 1, j, k) * (fourthirds * beta(i - 1, j, k) + gamma(i - 1, j, k)) + phix(i, j + 1, k) * beta_xy(i, j + 1, k) +
                             phix(i, j - 1, k) * beta_xy(i, j, k) + phix(i, j, k + 1) * beta_xz(i, j, k + 1) + phix(i, j, k - 1) * beta_xz(i, j, k) +
                             phiy(i, j + 1, k) * (beta_xy(i, j + 1, k) - twothirds * beta(i, j, k) + gamma(i, j, k)) -
                             phiy(i, j, k) * (beta_xy(i, j, k) - twothirds * beta(i, j, k) + gamma(i, j, k)) -
                             phiy(i - 1, j + 1, k) * (beta_xy(i, j + 1, k) - twothirds * beta(i - 1, j, k) + gamma(i - 1, j, k)) +
                             phiy(i - 1, j, k) * (beta_xy(i, j, k) - twothirds * beta(i - 1, j, k) + gamma(i - 1, j, k)) +
                             phiz(i, j, k + 1) * (beta_xz(i, j, k + 1) - twothirds * beta(i, j, k) + gamma(i, j, k)) -
                             phiz(i, j, k) * (beta_xz(i, j, k) - twothirds * beta(i, j, k) + gamma(i, j, k)) -
                             phiz(i - 1, j, k + 1) * (beta_xz(i, j, k + 1) - twothirds * beta(i - 1, j, k) + gamma(i - 1, j, k)) +
                             phiz(i - 1, j, k) * (beta_xz(i, j, k) - twothirds * beta(i - 1, j, k) + gamma(i - 1, j, k))) * dxsqinv;
                        break;
                    case 3:
                        v = phix(i, j, k) * (alphax(i, j, k) + (20.0 * b * onethird + 2.0 * c) * dxsqinv) -
                            ((phix(i + 1, j, k) + phix(i - 1, j, k)) * (fourthirds * b + c) +
                             (phix(i, j + 1, k) + phix(i, j - 1, k) + phix(i, j, k + 1) + phix(i, j, k - 1)) * b +
                             (phiy(i, j + 1, k) - phiy(i, j, k) - phiy(i - 1, j + 1, k) + phiy(i - 1, j, k) + phiz(i, j, k + 1) - phiz(i, j, k) -
                              phiz(i - 1, j, k + 1) + phiz(i - 1, j, k)) * (onethird * b + c)) * dxsqinv;
                        break;
                    }
                    Lpx(i, j, k) = v;
                }
            }
    }
    if (col.do_c[1]) {
        const Fab& alphay = alpha[1];
        Fab& Lpy = Lp[1];
#pragma omp parallel for schedule(static)
        for (int k = Lpy.vlo[2]; k <= Lpy.vhi[2]; ++k)
            for (int j = Lpy.vlo[1]; j <= Lpy.vhi[1]; ++j) {
                int ioff = ioff_of(col.offset, xlo, j, k, color);
                for (int i = Lpy.vlo[0] + ioff; i <= Lpy.vhi[0]; i += col.offset) {
                    double v = 0.0;
                    switch (visc) {
                    case -1:
                        v = phiy(i, j, k) * (alphay(i, j, k) + (beta(i, j, k) + beta(i, j - 1, k) + beta_xy(i, j, k) + beta_xy(i + 1, j, k) +
                                                                beta_yz(i, j, k) + beta_yz(i, j, k + 1)) * dxsqinv) -
                            (phiy(i, j + 1, k) * beta(i, j, k) + phiy(i, j - 1, k) * beta(i, j - 1, k) + phiy(i + 1, j, k) * beta_xy(i + 1, j, k) +
                             phiy(i - 1, j, k) * beta_xy(i, j, k) + phiy(i, j, k + 1) * beta_yz(i, j, k + 1) + phiy(i, j, k - 1) * beta_yz(i, j, k)) * dxsqinv;
                        break;
                    case 1:
                        v = phiy(i, j, k) * (alphay(i, j, k) + 6.0 * b * dxsqinv) -
                            (phiy(i + 1, j, k) + phiy(i - 1, j, k) + phiy(i, j + 1, k) + phiy(i, j - 1, k) + phiy(i, j, k + 1) + phiy(i, j, k - 1)) * b * dxsqinv;
                        break;
                    case -2:
                        v = phiy(i, j, k) * (alphay(i, j, k) + (2.0 * beta(i, j, k) + 2.0 * beta(i, j - 1, k) + beta_xy(i, j, k) + beta_xy(i + 1, j, k) +
                                                                beta_yz(i, j, k) + beta_yz(i, j, k + 1)) * dxsqinv) -
                            (2.0 * phiy(i, j + 1, k) * beta(i, j, k) + 2.0 * phiy(i, j - 1, k) * beta(i, j - 1, k) + phiy(i + 1, j, k) * beta_xy(i + 1, j, k) +
                             phiy(i - 1, j, k) * beta_xy(i, j, k) + phiy(i, j, k + 1) * beta_yz(i, j, k + 1) + phiy(i, j, k - 1) * beta_yz(i, j, k) +
                             phix(i + 1, j, k) * beta_xy(i + 1, j, k) - phix(i, j, k) * beta_xy(i, j, k) - phix(i + 1, j - 1, k) * beta_xy(i + 1, j, k) +
                             phix(i, j - 1, k) * beta_xy(i, j, k) + phiz(i, j, k + 1) * beta_yz(i, j, k + 1) - phiz(i, j, k) * beta_yz(i, j, k) -
                             phiz(i, j - 1, k + 1) * beta_yz(i, j, k + 1) + phiz(i, j - 1, k) * beta_yz(i, j, k)) * dxsqinv;
                        break;
                    case 2:
                        v = phiy(i, j, k) * (alphay(i, j, k) + 8.0 * b * dxsqinv) -
                            (2.0 * phiy(i, j + 1, k) + 2.0 * phiy(i, j - 1, k) + phiy(i + 1, j, k) + phiy(i - 1, j, k) + phiy(i, j, k + 1) +
                             phiy(i, j, k - 1) + phix(i + 1, j, k) - phix(i, j, k) - phix(i + 1, j - 1, k) + phix(i, j - 1, k) + phiz(i, j, k + 1) -
                             phiz(i, j, k) - phiz(i, j - 1, k + 1) + phiz(i, j - 1, k)) * b * dxsqinv;
                        break;
                    case -3:
                        v = phiy(i, j, k) * (alphay(i, j, k) + (fourthirds * beta(i, j, k) + gamma(i, j, k) + fourthirds * beta(i, j - 1, k) +
                                                                gamma(i, j - 1, k) + beta_xy(i, j, k) + beta_xy(i + 1, j, k) + beta_yz(i, j, k) +
                                                                beta_yz(i, j, k + 1)) * dxsqinv) -
                            (phiy(i, j + 1, k) * (fourthirds * beta(i, j, k) + gamma(i, j, k)) +
                             phiy(i, j - 1, k) * (fourthirds * beta(i, j - 1, k) + gamma(i, j - 1, k)) + phiy(i + 1, j, k) * beta_xy(i + 1, j, k) +
                             phiy(i - 1, j, k) * beta_xy(i, j, k) + phiy(i, j, k + 1) * beta_yz(i, j, k + 1) + phiy(i, j, k - 1) * beta_yz(i, j, k) +
                             phix(i + 1, j, k) * (beta_xy(i + 1, j, k) - twothirds * beta(i, j, k) + gamma(i, j, k)) -
                             phix(i, j, k) * (beta_xy(i, j, k) - twothirds * beta(i, j, k) + gamma(i, j, k)) -
                             phix(i + 1, j - 1, k) * (beta_xy(i + 1, j, k) - twothirds * beta(i, j - 1, k) + gamma(i, j - 1, k)) +
                             phix(i, j - 1, k) * (beta_xy(i, j, k) - twothirds * beta(i, j - 1, k) + gamma(i, j - 1, k)) +
                             phiz(i, j, k + 1) * (beta_yz(i, j, k + 1) - twothirds * beta(i, j, k) + gamma(i, j, k)) -
                             phiz(i, j, k) * (beta_yz(i, j, k) - twothirds * beta(i, j, k) + gamma(i, j, k)) -
                             phiz(i, j - 1, k + 1) * (beta_yz(i, j, k + 1) - twothirds * beta(i, j - 1, k) + gamma(i, j - 1, k)) +
                             phiz(i, j - 1, k) * (beta_yz(i, j, k) - twothirds * beta(i, j - 1, k) + gamma(i, j - 1, k))) * dxsqinv;
                        break;
                    case 3:
                        v = phiy(i, j, k) * (alphay(i, j, k) + (20.0 * b * onethird + 2.0 * c) * dxsqinv) -
                            ((phiy(i, j + 1, k) + phiy(i, j - 1, k)) * (fourthirds * b + c) +
                             (phiy(i + 1, j, k) + phiy(i - 1, j, k) + phiy(i, j, k + 1) + phiy(i, j, k - 1)) * b +
                             (phix(i + 1, j, k) - phix(i, j, k) - phix(i + 1, j - 1, k) + phix(i, j - 1, k) + phiz(i, j, k + 1) - phiz(i, j, k) -
                              phiz(i, j - 1, k + 1) + phiz(i, j - 1, k)) * (onethird * b + c)) * dxsqinv;
                        break;
                    }
                    Lpy(i, j, k) = v;
                }
            }
    }
    if (col.do_c[2]) {
        const Fab& alphaz = alpha[2];
        Fab& Lpz = Lp[2];
#pragma omp parallel for schedule(static)
        for (int k = Lpz.vlo[2]; k <= Lpz.vhi[2]; ++k)
            for (int j = Lpz.vlo[1]; j <= Lpz.vhi[1]; ++j) {
                int ioff = ioff_of(col.offset, xlo, j, k, color);
                for (int i = Lpz.vlo[0] + ioff; i <= Lpz.vhi[0]; i += col.offset) {
                    double v = 0.0;
                    switch (visc) {
                    case -1:
                        v = phiz(i, j, k) * (alphaz(i, j, k) + (beta(i, j, k) + beta(i, j, k - 1) + beta_xz(i, j, k) + beta_xz(i + 1, j, k) +
                                                                beta_yz(i, j, k) + beta_yz(i, j + 1, k)) * dxsqinv) -
                            (phiz(i, j, k + 1) * beta(i, j, k) + phiz(i, j, k - 1) * beta(i, j, k - 1) + phiz(i + 1, j, k) * beta_xz(i + 1, j, k) +
                             phiz(i - 1, j, k) * beta_xz(i, j, k) + phiz(i, j + 1, k) * beta_yz(i, j + 1, k) + phiz(i, j - 1, k) * beta_yz(i, j, k)) * dxsqinv;
                        break;
                    case 1:
                        v = phiz(i, j, k) * (alphaz(i, j, k) + 6.0 * b * dxsqinv) -
                            (phiz(i + 1, j, k) + phiz(i - 1, j, k) + phiz(i, j + 1, k) + phiz(i, j - 1, k) + phiz(i, j, k + 1) + phiz(i, j, k - 1)) * b * dxsqinv;
                        break;
                    case -2:
                        v = phiz(i, j, k) * (alphaz(i, j, k) + (2.0 * beta(i, j, k) + 2.0 * beta(i, j, k - 1) + beta_xz(i, j, k) + beta_xz(i + 1, j, k) +
                                                                beta_yz(i, j, k) + beta_yz(i, j + 1, k)) * dxsqinv) -
                            (2.0 * phiz(i, j, k + 1) * beta(i, j, k) + 2.0 * phiz(i, j, k - 1) * beta(i, j, k - 1) + phiz(i + 1, j, k) * beta_xz(i + 1, j, k) +
                             phiz(i - 1, j, k) * beta_xz(i, j, k) + phiz(i, j + 1, k) * beta_yz(i, j + 1, k) + phiz(i, j - 1, k) * beta_yz(i, j, k) +
                             phix(i + 1, j, k) * beta_xz(i + 1, j, k) - phix(i, j, k) * beta_xz(i, j, k) - phix(i + 1, j, k - 1) * beta_xz(i + 1, j, k) +
                             phix(i, j, k - 1) * beta_xz(i, j, k) + phiy(i, j + 1, k) * beta_yz(i, j + 1, k) - phiy(i, j, k) * beta_yz(i, j, k) -
                             phiy(i, j + 1, k - 1) * beta_yz(i, j + 1, k) + phiy(i, j, k - 1) * beta_yz(i, j, k)) * dxsqinv;
                        break;
                    case 2:
                        v = phiz(i, j, k) * (alphaz(i, j, k) + 8.0 * b * dxsqinv) -
                            (2.0 * phiz(i, j, k + 1) + 2.0 * phiz(i, j, k - 1) + phiz(i + 1, j, k) + phiz(i - 1, j, k) + phiz(i, j + 1, k) +
                             phiz(i, j - 1, k) + phix(i + 1, j, k) - phix(i, j, k) - phix(i + 1, j, k - 1) + phix(i, j, k - 1) + phiy(i, j + 1, k) -
                             phiy(i, j, k) - phiy(i, j + 1, k - 1) + phiy(i, j, k - 1)) * b * dxsqinv;
                        break;
                    case -3:
                        v = phiz(i, j, k) * (alphaz(i, j, k) + (fourthirds * beta(i, j, k) + gamma(i, j, k) + fourthirds * beta(i, j, k - 1) +
                                                                gamma(i, j, k - 1) + beta_xz(i, j, k) + beta_xz(i + 1, j, k) + beta_yz(i, j, k) +
                                                                beta_yz(i, j + 1, k)) * dxsqinv) -
                            (phiz(i, j, k + 1) * (fourthirds * beta(i, j, k) + gamma(i, j, k)) +
                             phiz(i, j, k - 1) * (fourthirds * beta(i, j, k - 1) + gamma(i, j, k - 1)) + phiz(i + 1, j, k) * beta_xz(i + 1, j, k) +
                             phiz(i - 1, j, k) * beta_xz(i, j, k) + phiz(i, j + 1, k) * beta_yz(i, j + 1, k) + phiz(i, j - 1, k) * beta_yz(i, j, k) +
                             phix(i + 1, j, k) * (beta_xz(i + 1, j, k) - twothirds * beta(i, j, k) + gamma(i, j, k)) -
                             phix(i, j, k) * (beta_xz(i, j, k) - twothirds * beta(i, j, k) + gamma(i, j, k)) -
                             phix(i + 1, j, k - 1) * (beta_xz(i + 1, j, k) - twothirds * beta(i, j, k - 1) + gamma(i, j, k - 1)) +
                             phix(i, j, k - 1) * (beta_xz(i, j, k) - twothirds * beta(i, j, k - 1) + gamma(i, j, k - 1)) +
                             phiy(i, j + 1, k) * (beta_yz(i, j + 1, k) - twothirds * beta(i, j, k) + gamma(i, j, k)) -
                             phiy(i, j, k) * (beta_yz(i, j, k) - twothirds * beta(i, j, k) + gamma(i, j, k)) -
                             phiy(i, j + 1, k - 1) * (beta_yz(i, j + 1, k) - twothirds * beta(i, j, k - 1) + gamma(i, j, k - 1)) +
                             phiy(i, j, k - 1) * (beta_yz(i, j, k) - twothirds * beta(i, j, k - 1) + gamma(i, j, k - 1))) * dxsqinv;
                        break;
                    case 3:
                        v = phiz(i, j, k) * (alphaz(i, j, k) + (20.0 * b * onethird + 2.0 * c) * dxsqinv) -
                            ((phiz(i, j, k + 1) + phiz(i, j, k - 1)) * (fourthirds * b + c) +
                             (phiz(i + 1, j, k) + phiz(i - 1, j, k) + phiz(i, j + 1, k) + phiz(i, j - 1, k)) * b +
                             (phix(i + 1, j, k) - phix(i, j, k) - phix(i + 1, j, k - 1) + phix(i, j, k - 1) + phiy(i, j + 1, k) - phiy(i, j, k) -
                              phiy(i, j + 1, k - 1) + phiy(i, j, k - 1)) * (onethird * b + c)) * dxsqinv;
                        break;
                    }
                    Lpz(i, j, k) = v;
                }
            }
    }
}

void stag_applyop_level(const Level& L, const Fab* phi, Fab* Lphi, int color, int visc) {
    if (L.geo.dm == 2)
        applyop_2d(phi, Lphi, L.alpha, L.beta_cc, L.beta_ed[0], L.gamma_cc, L.dx, color, visc);
    else
        applyop_3d(phi, Lphi, L.alpha, L.beta_cc, L.beta_ed, L.gamma_cc, L.dx, color, visc);
    // Lphi on physical domain boundaries is zero (stag_applyop.f90:197-201)
    for (int c = 0; c < L.geo.dm; ++c) physbc_domainvel(L.geo, Lphi[c], c);
}

// ---------------------------------------------------------------- smoother update
// diag(theta*alpha - L) per face, in the operand order of stag_mg_update_2d/_3d
static inline double diag_2d(int comp, int i, int j, const Fab& alpha, const Fab& beta, const Fab& bed,
                             const Fab& gamma, double dxsqinv, int visc, double b, double c) {
    const double fourthirds = 4.0 / 3.0, fourteenthirds = 14.0 / 3.0;
    if (comp == 0) {
        switch (visc) {
        case -1: return alpha(i, j) + (beta(i, j) + beta(i - 1, j) + bed(i, j) + bed(i, j + 1)) * dxsqinv;
        case 1: return alpha(i, j) + 4.0 * b * dxsqinv;
        case -2: return alpha(i, j) + (2.0 * beta(i, j) + 2.0 * beta(i - 1, j) + bed(i, j) + bed(i, j + 1)) * dxsqinv;
        case 2: return alpha(i, j) + 6.0 * b * dxsqinv;
        case -3: return alpha(i, j) + (fourthirds * beta(i, j) + gamma(i, j) + fourthirds * beta(i - 1, j) + gamma(i - 1, j) + bed(i, j) + bed(i, j + 1)) * dxsqinv;
        case 3: return alpha(i, j) + (fourteenthirds * b + 2.0 * c) * dxsqinv;
        }
    } else {
        switch (visc) {
        case -1: return alpha(i, j) + (beta(i, j) + beta(i, j - 1) + bed(i, j) + bed(i + 1, j)) * dxsqinv;
        case 1: return alpha(i, j) + 4.0 * b * dxsqinv;
        case -2: return alpha(i, j) + (2.0 * beta(i, j) + 2.0 * beta(i, j - 1) + bed(i, j) + bed(i + 1, j)) * dxsqinv;
        case 2: return alpha(i, j) + 6.0 * b * dxsqinv;
        case -3: return alpha(i, j) + (fourthirds * beta(i, j) + gamma(i, j) + fourthirds * beta(i, j - 1) + gamma(i, j - 1) + bed(i, j) + bed(i + 1, j)) * dxsqinv;
        case 3: return alpha(i, j) + (fourteenthirds * b + 2.0 * c) * dxsqinv;
        }
    }
    return 0.0;
}

static inline double diag_3d(int comp, int i, int j, int k, const Fab& alpha, const Fab& beta, const Fab* bed,
                             const Fab& gamma, double dxsqinv, int visc, double b, double c) {
    const double fourthirds = 4.0 / 3.0, twentythirds = 20.0 / 3.0;
    const Fab &bxy = bed[0], &bxz = bed[1], &byz = bed[2];
    // per component: (cell neighbour in own direction, first edge pair, second edge pair)
    switch (comp) {
    case 0:
        switch (visc) {
        case -1: return alpha(i, j, k) + (beta(i, j, k) + beta(i - 1, j, k) + bxy(i, j, k) + bxy(i, j + 1, k) + bxz(i, j, k) + bxz(i, j, k + 1)) * dxsqinv;
        case 1: return alpha(i, j, k) + 6.0 * b * dxsqinv;
        case -2: return alpha(i, j, k) + (2.0 * beta(i, j, k) + 2.0 * beta(i - 1, j, k) + bxy(i, j, k) + bxy(i, j + 1, k) + bxz(i, j, k) + bxz(i, j, k + 1)) * dxsqinv;
        case 2: return alpha(i, j, k) + 8.0 * b * dxsqinv;
        case -3: return alpha(i, j, k) + (fourthirds * beta(i, j, k) + gamma(i, j, k) + fourthirds * beta(i - 1, j, k) + gamma(i - 1, j, k) + bxy(i, j, k) + bxy(i, j + 1, k) + bxz(i, j, k) + bxz(i, j, k + 1)) * dxsqinv;
        case 3: return alpha(i, j, k) + (twentythirds * b + 2.0 * c) * dxsqinv;
        }
        break;
    case 1:
        switch (visc) {
        case -1: return alpha(i, j, k) + (beta(i, j, k) + beta(i, j - 1, k) + bxy(i, j, k) + bxy(i + 1, j, k) + byz(i, j, k) + byz(i, j, k + 1)) * dxsqinv;
        case 1: return alpha(i, j, k) + 6.0 * b * dxsqinv;
        case -2: return alpha(i, j, k) + (2.0 * beta(i, j, k) + 2.0 * beta(i, j - 1, k) + bxy(i, j, k) + bxy(i + 1, j, k) + byz(i, j, k) + byz(i, j, k + 1)) * dxsqinv;
        case 2: return alpha(i, j, k) + 8.0 * b * dxsqinv;
        case -3: return alpha(i, j, k) + (fourthirds * beta(i, j, k) + gamma(i, j, k) + fourthirds * beta(i, j - 1, k) + gamma(i, j - 1, k) + bxy(i, j, k) + bxy(i + 1, j, k) + byz(i, j, k) + byz(i, j, k + 1)) * dxsqinv;
        case 3: return alpha(i, j, k) + (twentythirds * b + 2.0 * c) * dxsqinv;
        }
        break;
    case 2:
        switch (visc) {
        case -1: return alpha(i, j, k) + (beta(i, j, k) + beta(i, j, k - 1) + bxz(i, j, k) + bxz(i + 1, j, k) + byz(i, j, k) + byz(i, j + 1, k)) * dxsqinv;
        case 1: return alpha(i, j, k) + 6.0 * b * dxsqinv;
        case -2: return alpha(i, j, k) + (2.0 * beta(i, j, k) + 2.0 * beta(i, j, k - 1) + bxz(i, j, k) + bxz(i + 1, j, k) + byz(i, j, k) + byz(i, j + 1, k)) * dxsqinv;
        case 2: return alpha(i, j, k) + 8.0 * b * dxsqinv;
        case -3: return alpha(i, j, k) + (fourthirds * beta(i, j, k) + gamma(i, j, k) + fourthirds * beta(i, j, k - 1) + gamma(i, j, k - 1) + bxz(i, j, k) + bxz(i + 1, j, k) + byz(i, j, k) + byz(i, j + 1, k)) * dxsqinv;
        case 3: return alpha(i, j, k) + (twentythirds * b + 2.0 * c) * dxsqinv;
        }
        break;
    }
    return 0.0;
}

void stag_mg_update(const Level& L, Fab* phi, const Fab* rhs, const Fab* Lphi, int color, int visc, double omega) {
    const int dm = L.geo.dm;
    Colour col = colour_of(color);
    double dxsq = L.dx * L.dx;
    double dxsqinv = 1.0 / dxsq;
    const double b = L.beta_cc(0, 0, 0), c = L.gamma_cc(0, 0, 0);
    for (int comp = 0; comp < dm; ++comp) {
        if (!col.do_c[comp]) continue;
        Fab& ph = phi[comp];
        const Fab& r = rhs[comp];
        const Fab& Lp = Lphi[comp];
        const Fab& al = L.alpha[comp];
#pragma omp parallel for schedule(static)
        for (int k = ph.vlo[2]; k <= ph.vhi[2]; ++k)
            for (int j = ph.vlo[1]; j <= ph.vhi[1]; ++j) {
                int ioff = ioff_of(col.offset, 0, j, k, color);
                for (int i = ph.vlo[0] + ioff; i <= ph.vhi[0]; i += col.offset) {
                    double fac = (dm == 2) ? diag_2d(comp, i, j, al, L.beta_cc, L.beta_ed[0], L.gamma_cc, dxsqinv, visc, b, c)
                                           : diag_3d(comp, i, j, k, al, L.beta_cc, L.beta_ed, L.gamma_cc, dxsqinv, visc, b, c);
                    ph(i, j, k) = ph(i, j, k) + omega * (r(i, j, k) - Lp(i, j, k)) / fac;
                }
            }
        // The periodic seam face is stored twice (lo and hi+1).  With an even
        // cell count both copies are in the same colour and get the same
        // update; with an odd count (a coarsest level such as 3) they fall in
        // different colours, and the reference's two copies would diverge.
        // Keep one face: the hi+1 copy follows the lo face, as a single
        // stored face does (even counts need nothing: the copies agree).
        if (L.geo.n[comp] % 2 == 0) continue;
        const int n = L.geo.n[comp];
        for (int k = ph.vlo[2]; k <= ph.vhi[2]; ++k)
            for (int j = ph.vlo[1]; j <= ph.vhi[1]; ++j)
                for (int i = ph.vlo[0]; i <= ph.vhi[0]; ++i) {
                    if (comp == 0 && i == n) ph(i, j, k) = ph(0, j, k);
                    if (comp == 1 && j == n) ph(i, j, k) = ph(i, 0, k);
                    if (comp == 2 && k == n) ph(i, j, k) = ph(i, j, 0);
                }
    }
}

}  // namespace orc
