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
// hi+1 are periodic images of each other).
#pragma once
#include <cstddef>
#include <cstring>
#include <vector>

namespace orc {

struct Geo {
    int dm;
    int n[3];  // cells per direction; n[2] == 1 in 2D
};

struct Fab {
    int dm = 0;
    int ng = 0;
    int nodal[3] = {0, 0, 0};
    int vlo[3] = {0, 0, 0}, vhi[3] = {0, 0, 0};  // valid index range (inclusive)
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};    // allocated range incl. ghosts
    int n[3] = {1, 1, 1};                        // cells per direction (period)
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
    return Fab(g, nod, ng);
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

// multifab_fill_boundary for a periodic single-box domain: every ghost value
// is copied from its periodic image in the valid region.
inline void fill_boundary(Fab& f) {
    if (f.ng == 0) return;
#pragma omp parallel for schedule(static)
    for (int k = f.lo[2]; k <= f.hi[2]; ++k) {
        bool kg = k < f.vlo[2] || k > f.vhi[2];
        int kk = (f.dm == 3) ? wrap_to_valid(k, f.n[2], f.nodal[2]) : k;
        for (int j = f.lo[1]; j <= f.hi[1]; ++j) {
            bool jg = j < f.vlo[1] || j > f.vhi[1];
            int jj = wrap_to_valid(j, f.n[1], f.nodal[1]);
            if (kg || jg) {
                for (int i = f.lo[0]; i <= f.hi[0]; ++i) {
                    int ii = wrap_to_valid(i, f.n[0], f.nodal[0]);
                    f(i, j, k) = f(ii, jj, kk);
                }
            } else {
                for (int i = f.lo[0]; i < f.vlo[0]; ++i)
                    f(i, j, k) = f(wrap_to_valid(i, f.n[0], f.nodal[0]), j, k);
                for (int i = f.vhi[0] + 1; i <= f.hi[0]; ++i)
                    f(i, j, k) = f(wrap_to_valid(i, f.n[0], f.nodal[0]), j, k);
            }
        }
    }
}

// multifab_internal_sync for the periodic seam of a one-box domain: the
// duplicated nodal entries take the value of the lowest-indexed copy.
inline void internal_sync(Fab& f) {
    for (int d = 0; d < f.dm; ++d) {
        if (!f.nodal[d]) continue;
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

// compact (unique periodic, i fastest) <-> fab conversions
inline void fab_from_compact(Fab& f, const double* c) {
    int nx = f.n[0], ny = f.n[1];
    for (int k = f.lo[2]; k <= f.hi[2]; ++k)
        for (int j = f.lo[1]; j <= f.hi[1]; ++j)
            for (int i = f.lo[0]; i <= f.hi[0]; ++i) {
                int ii = ((i % nx) + nx) % nx;
                int jj = ((j % ny) + ny) % ny;
                int kk = (f.dm == 3) ? ((k % f.n[2]) + f.n[2]) % f.n[2] : 0;
                f(i, j, k) = c[(size_t)ii + (size_t)nx * ((size_t)jj + (size_t)ny * kk)];
            }
}
inline void compact_from_fab(double* c, const Fab& f) {
    int nx = f.n[0], ny = f.n[1], nz = f.n[2];
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                c[(size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k)] = f(i, j, k);
}

}  // namespace orc
