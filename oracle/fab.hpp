// fab.hpp - single-box BoxLib-style arrays for the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY.  This is part of the CPU oracle that restates the
// reference algorithm; only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg may use it, and only as the checker.
//
// The oracle keeps the reference's data model literally: a multifab on one
// box with ng ghost layers, face arrays nodal in their own direction
// (multifab_build_edge, n+1 valid faces), 3D edge arrays nodal in two
// directions (stag_mg_solver.f90:181-193), periodic ghost filling
// (multifab_fill_boundary) and the periodic nodal seam (valid faces lo and
// hi+1 are periodic images of each other).  A direction bounded by walls
// (bc.f90:23-35: no-slip 100-103, slip 200-203) is not periodic: its ghost
// cells are left to the physical-boundary fills (physbc.cpp).
#pragma once
#include <cstddef>
#include <cstring>
#include <vector>

namespace orc {

struct Geo {
    int dm;
    int n[3];  // cells per direction; n[2] == 1 in 2D
    // domain BC per direction and side (bc.f90 codes; -1 = periodic)
    int bc_lo[3] = {-1, -1, -1};
    int bc_hi[3] = {-1, -1, -1};
    bool periodic(int d) const { return d >= dm || bc_lo[d] == -1; }
    bool any_wall() const {
        for (int d = 0; d < dm; ++d)
            if (!periodic(d)) return true;
        return false;
    }
};
inline bool bc_is_noslip(int c) { return c >= 100 && c <= 103; }  // NO_SLIP_START..NO_SLIP_END
inline bool bc_is_slip(int c) { return c >= 200 && c <= 203; }    // SLIP_START..SLIP_END

struct Fab {
    int dm = 0;
    int ng = 0;
    int nodal[3] = {0, 0, 0};
    int vlo[3] = {0, 0, 0}, vhi[3] = {0, 0, 0};  // valid index range (inclusive)
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};    // allocated range incl. ghosts
    int n[3] = {1, 1, 1};                        // cells per direction (period)
    int per[3] = {1, 1, 1};                      // periodic directions
    // compact storage of a wall-bounded nodal direction: edge arrays keep all
    // n+1 nodes, face arrays keep lo..hi (the hi+1 wall face is zero)
    bool edge = false;
    long sx = 1, sy = 1, sz = 1;
    std::vector<double> a;

    Fab() = default;
    Fab(const Geo& g, const int nod[3], int ngh) { build(g, nod, ngh); }

    void build(const Geo& g, const int nod[3], int ngh) {
        dm = g.dm;
        ng = ngh;
        for (int d = 0; d < 3; ++d) {
            nodal[d] = (d < dm) ? nod[d] : 0;
            n[d] = (d < dm) ? g.n[d] : 1;
            per[d] = g.periodic(d) ? 1 : 0;
            vlo[d] = 0;
            vhi[d] = n[d] - 1 + nodal[d];
            int gd = (d < dm) ? ng : 0;
            lo[d] = vlo[d] - gd;
            hi[d] = vhi[d] + gd;
        }
        sx = 1;
        sy = hi[0] - lo[0] + 1;
        sz = sy * (hi[1] - lo[1] + 1);
        a.assign((size_t)sz * (hi[2] - lo[2] + 1), 0.0);
    }
    inline double& operator()(int i, int j, int k = 0) {
        return a[(size_t)((i - lo[0]) + sy * (j - lo[1]) + sz * (k - lo[2]))];
    }
    inline double operator()(int i, int j, int k = 0) const {
        return a[(size_t)((i - lo[0]) + sy * (j - lo[1]) + sz * (k - lo[2]))];
    }
    void setval(double v) { std::fill(a.begin(), a.end(), v); }
};

inline Fab make_cc(const Geo& g, int ng) {
    int nod[3] = {0, 0, 0};
    return Fab(g, nod, ng);
}
inline Fab make_face(const Geo& g, int d, int ng) {
    int nod[3] = {0, 0, 0};
    nod[d] = 1;
    return Fab(g, nod, ng);
}
// 2D nodal (beta_ed in 2D); 3D edges: e=0 xy (T,T,F), 1 xz (T,F,T), 2 yz (F,T,T)
inline Fab make_edge(const Geo& g, int e, int ng) {
    int nod[3] = {1, 1, 0};
    if (g.dm == 3) {
        if (e == 1) { nod[0] = 1; nod[1] = 0; nod[2] = 1; }
        if (e == 2) { nod[0] = 0; nod[1] = 1; nod[2] = 1; }
    }
    Fab f(g, nod, ng);
    f.edge = true;
    return f;
}

// periodic image of index v in a direction with period n; nodal directions
// have valid range 0..n, cell directions 0..n-1.
inline int wrap_to_valid(int v, int n, int nodal) {
    if (nodal) {
        while (v < 0) v += n;
        while (v > n) v -= n;
    } else {
        while (v < 0) v += n;
        while (v >= n) v -= n;
    }
    return v;
}

// multifab_fill_boundary on a single box: every ghost value whose periodic
// image lies in the valid region is copied from it.  Ghost cells outside a
// wall-bounded side have no such image and keep their contents.
inline void fill_boundary(Fab& f) {
    if (f.ng == 0) return;
    auto image = [&](int d, int v, int& out) {
        if (v >= f.vlo[d] && v <= f.vhi[d]) { out = v; return true; }
        if (!f.per[d] || d >= f.dm) return false;
        out = wrap_to_valid(v, f.n[d], f.nodal[d]);
        return true;
    };
#pragma omp parallel for schedule(static)
    for (int k = f.lo[2]; k <= f.hi[2]; ++k) {
        int kk;
        if (!image(2, k, kk)) continue;
        const bool kg = k < f.vlo[2] || k > f.vhi[2];
        for (int j = f.lo[1]; j <= f.hi[1]; ++j) {
            int jj;
            if (!image(1, j, jj)) continue;
            const bool jg = j < f.vlo[1] || j > f.vhi[1];
            for (int i = f.lo[0]; i <= f.hi[0]; ++i) {
                const bool ig = i < f.vlo[0] || i > f.vhi[0];
                if (!(ig || jg || kg)) continue;
                int ii;
                if (!image(0, i, ii)) continue;
                f(i, j, k) = f(ii, jj, kk);
            }
        }
    }
}

// multifab_internal_sync for the periodic seam of a one-box domain: the
// duplicated nodal entries take the value of the lowest-indexed copy.
inline void internal_sync(Fab& f) {
    for (int d = 0; d < f.dm; ++d) {
        if (!f.nodal[d] || !f.per[d]) continue;
        for (int k = f.vlo[2]; k <= f.vhi[2]; ++k)
            for (int j = f.vlo[1]; j <= f.vhi[1]; ++j)
                for (int i = f.vlo[0]; i <= f.vhi[0]; ++i) {
                    int idx[3] = {i, j, k};
                    if (idx[d] != f.vhi[d]) continue;
                    int s[3] = {i, j, k};
                    s[d] = f.vlo[d];
                    f(i, j, k) = f(s[0], s[1], s[2]);
                }
    }
}

// entries per direction of the compact layout: n (periodic; a wall-bounded
// face direction, whose hi+1 wall face is implied zero), n+1 (an edge array
// nodal in a wall-bounded direction)
inline int compact_extent(const Fab& f, int d) {
    if (d >= f.dm) return 1;
    return f.n[d] + ((f.edge && f.nodal[d] && !f.per[d]) ? 1 : 0);
}

// compact (unique periodic, i fastest) <-> fab conversions.  Periodic
// directions fill ghosts and the nodal seam from their images; in a
// wall-bounded direction the stored entries are copied, the hi+1 wall face
// of a face array is zero and ghost cells are zero (left to the physical
// fills).
inline void fab_from_compact(Fab& f, const double* c) {
    int ext[3];
    for (int d = 0; d < 3; ++d) ext[d] = compact_extent(f, d);
    auto map = [&](int d, int v, int& out) {
        if (d >= f.dm) { out = 0; return true; }
        if (f.per[d]) { out = ((v % f.n[d]) + f.n[d]) % f.n[d]; return true; }
        if (v < 0 || v >= ext[d]) return false;
        out = v;
        return true;
    };
    for (int k = f.lo[2]; k <= f.hi[2]; ++k)
        for (int j = f.lo[1]; j <= f.hi[1]; ++j)
            for (int i = f.lo[0]; i <= f.hi[0]; ++i) {
                int ii, jj, kk;
                if (map(0, i, ii) && map(1, j, jj) && map(2, k, kk))
                    f(i, j, k) = c[(size_t)ii + (size_t)ext[0] * ((size_t)jj + (size_t)ext[1] * kk)];
                else
                    f(i, j, k) = 0.0;
            }
}
inline void compact_from_fab(double* c, const Fab& f) {
    const int ex = compact_extent(f, 0), ey = compact_extent(f, 1), ez = compact_extent(f, 2);
    for (int k = 0; k < ez; ++k)
        for (int j = 0; j < ey; ++j)
            for (int i = 0; i < ex; ++i)
                c[(size_t)i + (size_t)ex * ((size_t)j + (size_t)ey * k)] = f(i, j, k);
}

}  // namespace orc
