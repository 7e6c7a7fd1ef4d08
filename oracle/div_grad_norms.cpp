// div_grad_norms.cpp - CPU oracle: MAC gradient/divergence and the weighted
// staggered/cell reductions.
//
// TEST INFRASTRUCTURE ONLY (the oracle).  Restates
//   src_common/div_and_grad.f90:16-455       (compute_grad, compute_div;
//       periodic faces never take the 2/dx boundary stencil of :139-182,
//       wall faces -- pressure FOEXTRAP -- always do)
//   src_gmres/norm_inner_product.f90:16-418  (stag_inner_prod, cc_inner_prod,
//       stag_l2_norm, cc_l2_norm)
//   src_gmres/norm_inner_product.f90:579-794 (sum_umac_press)
// The reductions iterate over BoxLib tiles exactly like the reference's
// mfiter loops: the nodal tile box of the last tile in direction d includes
// face hi+1 (get_nodaltilebox), and the 0.5-weighted boundary terms are added
// per tile.  Tile partial sums are added in tile order (the reference adds
// them in OpenMP order, which is not reproducible).
#include "oracle_internal.hpp"

#include <cmath>
#include <vector>

namespace orc {

int g_tile_size[3] = {1024000, 8, 8};

struct Tile {
    int lo[3], hi[3];
};

// BoxLib-style tiling of the cell box: n/T tiles per direction (at least 1),
// cells spread evenly with the remainder going to the first tiles.
static std::vector<Tile> make_tiles(const Geo& g) {
    std::vector<int> cuts[3];
    for (int d = 0; d < 3; ++d) {
        int n = (d < g.dm) ? g.n[d] : 1;
        int T = (d < g.dm) ? g_tile_size[d] : 1;
        int nt = std::max(1, n / std::max(1, T));
        int base = n / nt, rem = n % nt, s = 0;
        cuts[d].push_back(0);
        for (int t = 0; t < nt; ++t) {
            s += base + (t < rem ? 1 : 0);
            cuts[d].push_back(s);
        }
    }
    std::vector<Tile> tiles;
    for (size_t tk = 0; tk + 1 < cuts[2].size(); ++tk)
        for (size_t tj = 0; tj + 1 < cuts[1].size(); ++tj)
            for (size_t ti = 0; ti + 1 < cuts[0].size(); ++ti) {
                Tile t;
                t.lo[0] = cuts[0][ti]; t.hi[0] = cuts[0][ti + 1] - 1;
                t.lo[1] = cuts[1][tj]; t.hi[1] = cuts[1][tj + 1] - 1;
                t.lo[2] = cuts[2][tk]; t.hi[2] = cuts[2][tk + 1] - 1;
                tiles.push_back(t);
            }
    return tiles;
}

static void nodal_tile(const Geo& g, const Tile& t, int dir, int lo[3], int hi[3]) {
    for (int d = 0; d < 3; ++d) { lo[d] = t.lo[d]; hi[d] = t.hi[d]; }
    int nd = (dir < g.dm) ? g.n[dir] : 1;
    if (dir < g.dm && t.hi[dir] == nd - 1) hi[dir] = t.hi[dir] + 1;
}

void compute_grad(const Geo& g, double dx, const Fab& phi, Fab* gradp) {
    double dxinv = 1.0 / dx;
    for (int d = 0; d < g.dm; ++d) {
        Fab& gp = gradp[d];
        int o[3] = {0, 0, 0};
        o[d] = 1;
#pragma omp parallel for schedule(static)
        for (int k = gp.vlo[2]; k <= gp.vhi[2]; ++k)
            for (int j = gp.vlo[1]; j <= gp.vhi[1]; ++j)
                for (int i = gp.vlo[0]; i <= gp.vhi[0]; ++i)
                    gp(i, j, k) = (phi(i, j, k) - phi(i - o[0], j - o[1], k - o[2])) * dxinv;
        if (g.periodic(d)) continue;
        // the ghost value represents the boundary value (div_and_grad.f90:139-182)
        const double twodxinv = 2.0 * dxinv;
        for (int side = 0; side < 2; ++side) {
            const int f = (side == 0) ? 0 : g.n[d];
            int r0[3] = {gp.vlo[0], gp.vlo[1], gp.vlo[2]}, r1[3] = {gp.vhi[0], gp.vhi[1], gp.vhi[2]};
            r0[d] = r1[d] = f;
            for (int k = r0[2]; k <= r1[2]; ++k)
                for (int j = r0[1]; j <= r1[1]; ++j)
                    for (int i = r0[0]; i <= r1[0]; ++i)
                        gp(i, j, k) = (phi(i, j, k) - phi(i - o[0], j - o[1], k - o[2])) * twodxinv;
        }
    }
}

void compute_div(const Geo& g, double dx, const Fab* phi_fc, Fab& div) {
    double dxinv = 1.0 / dx;
    const Fab &px = phi_fc[0], &py = phi_fc[1];
    if (g.dm == 2) {
        for (int j = 0; j < g.n[1]; ++j)
            for (int i = 0; i < g.n[0]; ++i)
                div(i, j) = (px(i + 1, j) - px(i, j)) * dxinv + (py(i, j + 1) - py(i, j)) * dxinv;
        return;
    }
    const Fab& pz = phi_fc[2];
#pragma omp parallel for schedule(static)
    for (int k = 0; k < g.n[2]; ++k)
        for (int j = 0; j < g.n[1]; ++j)
            for (int i = 0; i < g.n[0]; ++i)
                div(i, j, k) = (px(i + 1, j, k) - px(i, j, k)) * dxinv + (py(i, j + 1, k) - py(i, j, k)) * dxinv +
                               (pz(i, j, k + 1) - pz(i, j, k)) * dxinv;
}

void stag_inner_prod(const Geo& g, const Fab* m1, const Fab* m2, double* prod) {
    std::vector<Tile> tiles = make_tiles(g);
    const int dm = g.dm;
    std::vector<double> part(tiles.size() * 3, 0.0);
#pragma omp parallel for schedule(dynamic)
    for (long t = 0; t < (long)tiles.size(); ++t) {
        double ip[3] = {0.0, 0.0, 0.0};
        for (int c = 0; c < dm; ++c) {
            int lo[3], hi[3];
            nodal_tile(g, tiles[t], c, lo, hi);
            const Fab &a = m1[c], &b = m2[c];
            for (int k = lo[2]; k <= hi[2]; ++k)
                for (int j = lo[1]; j <= hi[1]; ++j)
                    for (int i = lo[0]; i <= hi[0]; ++i) ip[c] = ip[c] + a(i, j, k) * b(i, j, k);
            // boundary faces: the two loops of the direction-c faces
            int glo = 0, ghi1 = g.n[c];
            for (int side = 0; side < 2; ++side) {
                int pos = (side == 0) ? glo : ghi1;
                bool hit = (side == 0) ? (lo[c] == glo) : (hi[c] == ghi1);
                if (!hit) continue;
                int r0[3] = {lo[0], lo[1], lo[2]}, r1[3] = {hi[0], hi[1], hi[2]};
                r0[c] = r1[c] = pos;
                for (int k = r0[2]; k <= r1[2]; ++k)
                    for (int j = r0[1]; j <= r1[1]; ++j)
                        for (int i = r0[0]; i <= r1[0]; ++i) ip[c] = ip[c] + 0.5 * a(i, j, k) * b(i, j, k);
            }
        }
        for (int c = 0; c < 3; ++c) part[t * 3 + c] = ip[c];
    }
    for (int c = 0; c < 3; ++c) prod[c] = 0.0;
    for (size_t t = 0; t < tiles.size(); ++t)
        for (int c = 0; c < dm; ++c) prod[c] = prod[c] + part[t * 3 + c];
}

double cc_inner_prod(const Geo& g, const Fab& m1, const Fab& m2) {
    std::vector<Tile> tiles = make_tiles(g);
    std::vector<double> part(tiles.size(), 0.0);
#pragma omp parallel for schedule(dynamic)
    for (long t = 0; t < (long)tiles.size(); ++t) {
        double ip = 0.0;
        const Tile& T = tiles[t];
        for (int k = T.lo[2]; k <= T.hi[2]; ++k)
            for (int j = T.lo[1]; j <= T.hi[1]; ++j)
                for (int i = T.lo[0]; i <= T.hi[0]; ++i) ip = ip + m1(i, j, k) * m2(i, j, k);
        part[t] = ip;
    }
    double s = 0.0;
    for (double v : part) s = s + v;
    return s;
}

double stag_l2_norm(const Geo& g, const Fab* m) {
    double ip[3];
    stag_inner_prod(g, m, m, ip);
    double s = 0.0;
    for (int d = 0; d < g.dm; ++d) s = s + ip[d];
    return std::sqrt(s);
}

double cc_l2_norm(const Geo& g, const Fab& m) { return std::sqrt(cc_inner_prod(g, m, m)); }

void sum_umac_press(const Geo& g, const Fab& p, const Fab* u, double* av_p, double* av_u) {
    const int dm = g.dm;
    double total_volume = 1.0;
    for (int d = 0; d < dm; ++d) total_volume *= (double)g.n[d];
    // multifab_sum_c over the valid cells
    double sump = 0.0;
    for (int k = p.vlo[2]; k <= p.vhi[2]; ++k)
        for (int j = p.vlo[1]; j <= p.vhi[1]; ++j)
            for (int i = p.vlo[0]; i <= p.vhi[0]; ++i) sump = sump + p(i, j, k);
    std::vector<Tile> tiles = make_tiles(g);
    std::vector<double> part(tiles.size() * 3, 0.0);
    for (size_t t = 0; t < tiles.size(); ++t) {
        double su[3] = {0.0, 0.0, 0.0};
        for (int c = 0; c < dm; ++c) {
            int lo[3], hi[3];
            nodal_tile(g, tiles[t], c, lo, hi);
            const Fab& a = u[c];
            for (int k = lo[2]; k <= hi[2]; ++k)
                for (int j = lo[1]; j <= hi[1]; ++j)
                    for (int i = lo[0]; i <= hi[0]; ++i) su[c] = su[c] + a(i, j, k);
            if (lo[c] == 0 && hi[c] == g.n[c]) {
                int r0[3] = {lo[0], lo[1], lo[2]}, r1[3] = {hi[0], hi[1], hi[2]};
                r0[c] = r1[c] = 0;
                for (int k = r0[2]; k <= r1[2]; ++k)
                    for (int j = r0[1]; j <= r1[1]; ++j)
                        for (int i = r0[0]; i <= r1[0]; ++i) {
                            int q[3] = {i, j, k};
                            q[c] = hi[c];
                            su[c] = su[c] + 0.5 * a(i, j, k);
                            su[c] = su[c] + 0.5 * a(q[0], q[1], q[2]);
                        }
            }
        }
        for (int c = 0; c < 3; ++c) part[t * 3 + c] = su[c];
    }
    double sumu[3] = {0.0, 0.0, 0.0};
    for (size_t t = 0; t < tiles.size(); ++t)
        for (int c = 0; c < dm; ++c) sumu[c] = sumu[c] + part[t * 3 + c];
    if (av_p) *av_p = sump / total_volume;
    if (av_u)
        for (int c = 0; c < dm; ++c) av_u[c] = sumu[c] / total_volume;
}

}  // namespace orc
