// physbc.cpp - CPU oracle: physical-boundary ghost fills for wall-bounded
// directions.
//
// TEST INFRASTRUCTURE ONLY (the oracle).  Restates, for homogeneous walls
// (the only form gmres(...) sees):
//   src_common/multifab_physbc_stag.f90:90-172, 270-386  physbc_domainvel:
//       the wall-normal velocity is zero on the wall face and on the ghost
//       faces behind it (tangential index over the valid cells lo..hi);
//   src_common/multifab_physbc_stag.f90:626-785, 945-1314  physbc_macvel:
//       a transverse velocity's ghost faces across a wall take -interior
//       (no-slip, DIR_VEL) or +interior (slip, DIR_TRACT), over the
//       component's own faces lo..hi+1 and, in 3D, the third direction's
//       cells including ghosts; sides in the order x-lo, x-hi, y-lo, ...;
//   src_common/multifab_physbc.f90:116-300  FOEXTRAP for the pressure
//       (define_bc_tower.f90:219-234): ghost = interior - dx/2 * 0.
// Periodic directions are left to fill_boundary.
#include "oracle_internal.hpp"

namespace orc {

void physbc_domainvel(const Geo& g, Fab& s, int comp) {
    if (g.periodic(comp)) return;
    const int ng = s.ng;
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
        lo[d] = 0;
        hi[d] = (d < g.dm) ? g.n[d] - 1 : 0;
    }
    // lo side: indices lo-ng..lo of direction comp; hi side: hi+1..hi+1+ng
    for (int side = 0; side < 2; ++side) {
        const int a = (side == 0) ? lo[comp] - ng : hi[comp] + 1;
        const int b = (side == 0) ? lo[comp] : hi[comp] + 1 + ng;
        int r0[3] = {lo[0], lo[1], lo[2]}, r1[3] = {hi[0], hi[1], hi[2]};
        r0[comp] = a;
        r1[comp] = b;
        for (int k = r0[2]; k <= r1[2]; ++k)
            for (int j = r0[1]; j <= r1[1]; ++j)
                for (int i = r0[0]; i <= r1[0]; ++i) s(i, j, k) = 0.0;
    }
}

void physbc_macvel(const Geo& g, Fab& s, int comp) {
    const int ng = s.ng;
    if (ng == 0) return;
    for (int d = 0; d < g.dm; ++d) {
        if (d == comp || g.periodic(d)) continue;
        // the third direction (3D): cells with ghosts; the component's own
        // direction: its valid faces lo..hi+1
        int r0[3] = {0, 0, 0}, r1[3] = {0, 0, 0};
        for (int q = 0; q < g.dm; ++q) {
            if (q == d) continue;
            if (q == comp) {
                r0[q] = 0;
                r1[q] = g.n[q];
            } else {
                r0[q] = -ng;
                r1[q] = g.n[q] - 1 + ng;
            }
        }
        for (int side = 0; side < 2; ++side) {
            const int code = (side == 0) ? g.bc_lo[d] : g.bc_hi[d];
            const bool slip = bc_is_slip(code);
            const int edge = (side == 0) ? 0 : g.n[d] - 1;
            for (int k = r0[2]; k <= (d == 2 ? r0[2] : r1[2]); ++k)
                for (int j = r0[1]; j <= (d == 1 ? r0[1] : r1[1]); ++j)
                    for (int i = r0[0]; i <= (d == 0 ? r0[0] : r1[0]); ++i) {
                        int src[3] = {i, j, k};
                        src[d] = edge;
                        const double v = s(src[0], src[1], src[2]);
                        for (int gl = 1; gl <= ng; ++gl) {
                            int dst[3] = {i, j, k};
                            dst[d] = (side == 0) ? edge - gl : edge + gl;
                            s(dst[0], dst[1], dst[2]) = slip ? v : -v;
                        }
                    }
        }
    }
}

void physbc_pres(const Geo& g, Fab& p) {
    const int ng = p.ng;
    if (ng == 0) return;
    for (int d = 0; d < g.dm; ++d) {
        if (g.periodic(d)) continue;
        int r0[3] = {0, 0, 0}, r1[3] = {0, 0, 0};
        for (int q = 0; q < g.dm; ++q) {
            r0[q] = -ng;
            r1[q] = g.n[q] - 1 + ng;
        }
        for (int side = 0; side < 2; ++side) {
            const int edge = (side == 0) ? 0 : g.n[d] - 1;
            const double half_dx_times_bc = 0.0;  // inhomogeneous_bc_val_*d(pres_bc_comp) = 0
            for (int k = r0[2]; k <= (d == 2 ? r0[2] : r1[2]); ++k)
                for (int j = r0[1]; j <= (d == 1 ? r0[1] : r1[1]); ++j)
                    for (int i = r0[0]; i <= (d == 0 ? r0[0] : r1[0]); ++i) {
                        int src[3] = {i, j, k};
                        src[d] = edge;
                        const double v = p(src[0], src[1], src[2]) - half_dx_times_bc;
                        for (int gl = 1; gl <= ng; ++gl) {
                            int dst[3] = {i, j, k};
                            dst[d] = (side == 0) ? edge - gl : edge + gl;
                            p(dst[0], dst[1], dst[2]) = v;
                        }
                    }
        }
    }
}

// the reference's three calls after every update of a staggered field:
// multifab_physbc_domainvel, multifab_fill_boundary, multifab_physbc_macvel
void fill_vel(const Geo& g, Fab* u) {
    for (int c = 0; c < g.dm; ++c) {
        physbc_domainvel(g, u[c], c);
        fill_boundary(u[c]);
        physbc_macvel(g, u[c], c);
    }
}

// multifab_fill_boundary + multifab_physbc(pres_bc_comp)
void fill_pres(const Geo& g, Fab& p) {
    fill_boundary(p);
    physbc_pres(g, p);
}

}  // namespace orc
