"""Independent numpy restatement of the reference's staggered Stokes pieces.

Written separately from the C++ oracle (oracle/*.cpp) and in a different
data model: compact periodic arrays (no ghost cells, the nodal seam stored
once) with np.roll for neighbours, the model the GPU kernels use.  Every
expression keeps the operand order of the reference Fortran, so results are
bit-identical to a correctly restated oracle.  It generates the golden
fixtures in this directory; the tests pin the oracle against them.

Reference files restated:
  src_common/stag_applyop.f90:204-1067   stag_applyop_2d / _3d (colour loops)
  src_gmres/stag_mg_solver.f90:1637-2463 stag_mg_update (diagonal)
  src_gmres/stag_mg_solver.f90:945-1175  cc / stag restriction
  src_gmres/stag_mg_solver.f90:1326-1367 edge restriction
  src_gmres/stag_mg_solver.f90:1424-1633 stag_prolongation
  src_common/div_and_grad.f90:16-455     compute_grad / compute_div
  src_gmres/norm_inner_product.f90       seam weights: a face at the periodic
      seam is stored twice by BoxLib (lo and hi+1) and each copy gets 1 + 0.5
      in stag_inner_prod, so the unique seam face weighs 3.
"""
from __future__ import annotations

import numpy as np


def sh(a, *off):
    """a at index + off (periodic); off is (di, dj[, dk]) in x, y[, z] order,
    arrays are stored [k, j, i] / [j, i]."""
    dm = a.ndim
    shifts = tuple(-o for o in reversed(off[:dm]))
    return np.roll(a, shifts, axis=tuple(range(dm)))


def parity(shape):
    idx = np.indices(shape)
    return idx.sum(axis=0) % 2


def colour_mask(shape, color):
    """faces of one Gauss-Seidel colour: (i+j+k) even for odd colours."""
    return parity(shape) == ((color + 1) % 2)


# ------------------------------------------------------------------ 2D operator
def applyop_2d(visc, phi, alpha, beta, bed, gamma, dx):
    px, py = phi
    ax, ay = alpha
    dxsq = dx ** 2
    dxsqinv = 1.0 / dxsq
    onethird, twothirds, fourthirds = 1.0 / 3.0, 2.0 / 3.0, 4.0 / 3.0
    b = beta.flat[0]
    c = gamma.flat[0]
    S = sh
    if visc == -1:
        Lx = px * (ax + (beta + S(beta, -1, 0) + S(bed, 0, 1) + bed) * dxsqinv) - (
            S(px, 1, 0) * beta + S(px, -1, 0) * S(beta, -1, 0) + S(px, 0, 1) * S(bed, 0, 1) + S(px, 0, -1) * bed) * dxsqinv
        Ly = py * (ay + (beta + S(beta, 0, -1) + S(bed, 1, 0) + bed) * dxsqinv) - (
            S(py, 0, 1) * beta + S(py, 0, -1) * S(beta, 0, -1) + S(py, 1, 0) * S(bed, 1, 0) + S(py, -1, 0) * bed) * dxsqinv
    elif visc == 1:
        Lx = px * (ax + 4.0 * b * dxsqinv) - (S(px, 1, 0) + S(px, -1, 0) + S(px, 0, 1) + S(px, 0, -1)) * b * dxsqinv
        Ly = py * (ay + 4.0 * b * dxsqinv) - (S(py, 0, 1) + S(py, 0, -1) + S(py, 1, 0) + S(py, -1, 0)) * b * dxsqinv
    elif visc == -2:
        Lx = px * (ax + (2.0 * beta + 2.0 * S(beta, -1, 0) + S(bed, 0, 1) + bed) * dxsqinv) - (
            2.0 * S(px, 1, 0) * beta + 2.0 * S(px, -1, 0) * S(beta, -1, 0) + S(px, 0, 1) * S(bed, 0, 1) + S(px, 0, -1) * bed
            + S(py, 0, 1) * S(bed, 0, 1) - py * bed - S(py, -1, 1) * S(bed, 0, 1) + S(py, -1, 0) * bed) * dxsqinv
        Ly = py * (ay + (2.0 * beta + 2.0 * S(beta, 0, -1) + S(bed, 1, 0) + bed) * dxsqinv) - (
            2.0 * S(py, 0, 1) * beta + 2.0 * S(py, 0, -1) * S(beta, 0, -1) + S(py, 1, 0) * S(bed, 1, 0) + S(py, -1, 0) * bed
            + S(px, 1, 0) * S(bed, 1, 0) - px * bed - S(px, 1, -1) * S(bed, 1, 0) + S(px, 0, -1) * bed) * dxsqinv
    elif visc == 2:
        Lx = px * (ax + 6.0 * b * dxsqinv) - (2.0 * S(px, 1, 0) + 2.0 * S(px, -1, 0) + S(px, 0, 1) + S(px, 0, -1)
                                              + S(py, 0, 1) - py - S(py, -1, 1) + S(py, -1, 0)) * b * dxsqinv
        Ly = py * (ay + 6.0 * b * dxsqinv) - (2.0 * S(py, 0, 1) + 2.0 * S(py, 0, -1) + S(py, 1, 0) + S(py, -1, 0)
                                              + S(px, 1, 0) - px - S(px, 1, -1) + S(px, 0, -1)) * b * dxsqinv
    elif visc == -3:
        g = gamma
        Lx = px * (ax + (fourthirds * beta + g + fourthirds * S(beta, -1, 0) + S(g, -1, 0) + S(bed, 0, 1) + bed) * dxsqinv) - (
            S(px, 1, 0) * (fourthirds * beta + g) + S(px, -1, 0) * (fourthirds * S(beta, -1, 0) + S(g, -1, 0))
            + S(px, 0, 1) * S(bed, 0, 1) + S(px, 0, -1) * bed
            + S(py, 0, 1) * (S(bed, 0, 1) - twothirds * beta + g) - py * (bed - twothirds * beta + g)
            - S(py, -1, 1) * (S(bed, 0, 1) - twothirds * S(beta, -1, 0) + S(g, -1, 0))
            + S(py, -1, 0) * (bed - twothirds * S(beta, -1, 0) + S(g, -1, 0))) * dxsqinv
        Ly = py * (ay + (fourthirds * beta + g + fourthirds * S(beta, 0, -1) + S(g, 0, -1) + S(bed, 1, 0) + bed) * dxsqinv) - (
            S(py, 0, 1) * (fourthirds * beta + g) + S(py, 0, -1) * (fourthirds * S(beta, 0, -1) + S(g, 0, -1))
            + S(py, 1, 0) * S(bed, 1, 0) + S(py, -1, 0) * bed
            + S(px, 1, 0) * (S(bed, 1, 0) - twothirds * beta + g) - px * (bed - twothirds * beta + g)
            - S(px, 1, -1) * (S(bed, 1, 0) - twothirds * S(beta, 0, -1) + S(g, 0, -1))
            + S(px, 0, -1) * (bed - twothirds * S(beta, 0, -1) + S(g, 0, -1))) * dxsqinv
    elif visc == 3:
        Lx = px * (ax + (14.0 * b * onethird + 2.0 * c) * dxsqinv) - (
            (S(px, 1, 0) + S(px, -1, 0)) * (fourthirds * b + c) + (S(px, 0, 1) + S(px, 0, -1)) * b
            + (S(py, 0, 1) - py - S(py, -1, 1) + S(py, -1, 0)) * (onethird * b + c)) * dxsqinv
        Ly = py * (ay + (14.0 * b * onethird + 2.0 * c) * dxsqinv) - (
            (S(py, 0, 1) + S(py, 0, -1)) * (fourthirds * b + c) + (S(py, 1, 0) + S(py, -1, 0)) * b
            + (S(px, 1, 0) - px - S(px, 1, -1) + S(px, 0, -1)) * (onethird * b + c)) * dxsqinv
    else:
        raise ValueError(visc)
    return [Lx, Ly]


def diag_2d(visc, alpha, beta, bed, gamma, dx):
    dxsqinv = 1.0 / dx ** 2
    ax, ay = alpha
    b, c = beta.flat[0], gamma.flat[0]
    S, g = sh, gamma
    if visc == -1:
        return [ax + (beta + S(beta, -1, 0) + bed + S(bed, 0, 1)) * dxsqinv,
                ay + (beta + S(beta, 0, -1) + bed + S(bed, 1, 0)) * dxsqinv]
    if visc == 1:
        return [ax + 4.0 * b * dxsqinv, ay + 4.0 * b * dxsqinv]
    if visc == -2:
        return [ax + (2.0 * beta + 2.0 * S(beta, -1, 0) + bed + S(bed, 0, 1)) * dxsqinv,
                ay + (2.0 * beta + 2.0 * S(beta, 0, -1) + bed + S(bed, 1, 0)) * dxsqinv]
    if visc == 2:
        return [ax + 6.0 * b * dxsqinv, ay + 6.0 * b * dxsqinv]
    f = 4.0 / 3.0
    if visc == -3:
        return [ax + (f * beta + g + f * S(beta, -1, 0) + S(g, -1, 0) + bed + S(bed, 0, 1)) * dxsqinv,
                ay + (f * beta + g + f * S(beta, 0, -1) + S(g, 0, -1) + bed + S(bed, 1, 0)) * dxsqinv]
    if visc == 3:
        return [ax + (14.0 / 3.0 * b + 2.0 * c) * dxsqinv, ay + (14.0 / 3.0 * b + 2.0 * c) * dxsqinv]
    raise ValueError(visc)


# ------------------------------------------------------------------ 3D operator
def _perm3(comp):
    """(own, t1, t2) directions and edge indices for face component comp:
    edges xy=0, xz=1, yz=2."""
    return {0: (0, 1, 2, 0, 1), 1: (1, 0, 2, 0, 2), 2: (2, 0, 1, 1, 2)}[comp]


def _e(d):
    o = [0, 0, 0]
    o[d] = 1
    return o


def _m(d):
    o = [0, 0, 0]
    o[d] = -1
    return o


def _add(a, b):
    return [x + y for x, y in zip(a, b)]


def applyop_3d_comp(comp, visc, phi, alpha, beta, bed, gamma, dx):
    """One face component of stag_applyop_3d, operand order of the reference:
    for comp=x the edge pair (xy, xz) is indexed by (j, k); for comp=y the
    pair (xy, yz) by (i, k); for comp=z the pair (xz, yz) by (i, j)."""
    d, t1, t2, e1, e2 = _perm3(comp)
    S = sh
    p = phi[d]
    q1, q2 = phi[t1], phi[t2]
    a = alpha[d]
    E1, E2 = bed[e1], bed[e2]
    dxsqinv = 1.0 / dx ** 2
    onethird, twothirds, fourthirds = 1.0 / 3.0, 2.0 / 3.0, 4.0 / 3.0
    b, c = beta.flat[0], gamma.flat[0]
    g = gamma
    pd, md = _e(d), _m(d)
    p1, m1 = _e(t1), _m(t1)
    p2, m2 = _e(t2), _m(t2)
    bm = S(beta, *md)       # beta at i-1 (own direction)
    E1p = S(E1, *p1)        # edge at +t1
    E2p = S(E2, *p2)        # edge at +t2
    if visc == -1:
        return p * (a + (beta + bm + E1 + E1p + E2 + E2p) * dxsqinv) - (
            S(p, *pd) * beta + S(p, *md) * bm + S(p, *p1) * E1p + S(p, *m1) * E1 + S(p, *p2) * E2p + S(p, *m2) * E2) * dxsqinv
    if visc == 1:
        if comp == 0:
            nb = S(p, 1, 0, 0) + S(p, -1, 0, 0) + S(p, 0, 1, 0) + S(p, 0, -1, 0) + S(p, 0, 0, 1) + S(p, 0, 0, -1)
        elif comp == 1:
            nb = S(p, 1, 0, 0) + S(p, -1, 0, 0) + S(p, 0, 1, 0) + S(p, 0, -1, 0) + S(p, 0, 0, 1) + S(p, 0, 0, -1)
        else:
            nb = S(p, 1, 0, 0) + S(p, -1, 0, 0) + S(p, 0, 1, 0) + S(p, 0, -1, 0) + S(p, 0, 0, 1) + S(p, 0, 0, -1)
        return p * (a + 6.0 * b * dxsqinv) - nb * b * dxsqinv
    # cross terms: phi_t(i, +t) - phi_t(i) - phi_t(i-d, +t) + phi_t(i-d)
    c1 = [S(q1, *p1), q1, S(q1, *_add(md, p1)), S(q1, *md)]
    c2 = [S(q2, *p2), q2, S(q2, *_add(md, p2)), S(q2, *md)]
    if visc == -2:
        return p * (a + (2.0 * beta + 2.0 * bm + E1 + E1p + E2 + E2p) * dxsqinv) - (
            2.0 * S(p, *pd) * beta + 2.0 * S(p, *md) * bm + S(p, *p1) * E1p + S(p, *m1) * E1 + S(p, *p2) * E2p + S(p, *m2) * E2
            + c1[0] * E1p - c1[1] * E1 - c1[2] * E1p + c1[3] * E1
            + c2[0] * E2p - c2[1] * E2 - c2[2] * E2p + c2[3] * E2) * dxsqinv
    if visc == 2:
        return p * (a + 8.0 * b * dxsqinv) - (
            2.0 * S(p, *pd) + 2.0 * S(p, *md) + S(p, *p1) + S(p, *m1) + S(p, *p2) + S(p, *m2)
            + c1[0] - c1[1] - c1[2] + c1[3] + c2[0] - c2[1] - c2[2] + c2[3]) * b * dxsqinv
    if visc == -3:
        gm = S(g, *md)
        return p * (a + (fourthirds * beta + g + fourthirds * bm + gm + E1 + E1p + E2 + E2p) * dxsqinv) - (
            S(p, *pd) * (fourthirds * beta + g) + S(p, *md) * (fourthirds * bm + gm)
            + S(p, *p1) * E1p + S(p, *m1) * E1 + S(p, *p2) * E2p + S(p, *m2) * E2
            + c1[0] * (E1p - twothirds * beta + g) - c1[1] * (E1 - twothirds * beta + g)
            - c1[2] * (E1p - twothirds * bm + gm) + c1[3] * (E1 - twothirds * bm + gm)
            + c2[0] * (E2p - twothirds * beta + g) - c2[1] * (E2 - twothirds * beta + g)
            - c2[2] * (E2p - twothirds * bm + gm) + c2[3] * (E2 - twothirds * bm + gm)) * dxsqinv
    if visc == 3:
        return p * (a + (20.0 * b * onethird + 2.0 * c) * dxsqinv) - (
            (S(p, *pd) + S(p, *md)) * (fourthirds * b + c)
            + (_nb_t(p, comp)) * b
            + (c1[0] - c1[1] - c1[2] + c1[3] + c2[0] - c2[1] - c2[2] + c2[3]) * (onethird * b + c)) * dxsqinv
    raise ValueError(visc)


def _nb_t(p, comp):
    S = sh
    if comp == 0:
        return S(p, 0, 1, 0) + S(p, 0, -1, 0) + S(p, 0, 0, 1) + S(p, 0, 0, -1)
    if comp == 1:
        return S(p, 1, 0, 0) + S(p, -1, 0, 0) + S(p, 0, 0, 1) + S(p, 0, 0, -1)
    return S(p, 1, 0, 0) + S(p, -1, 0, 0) + S(p, 0, 1, 0) + S(p, 0, -1, 0)


def diag_3d_comp(comp, visc, alpha, beta, bed, gamma, dx):
    d, t1, t2, e1, e2 = _perm3(comp)
    S = sh
    a = alpha[d]
    E1, E2 = bed[e1], bed[e2]
    dxsqinv = 1.0 / dx ** 2
    b, c = beta.flat[0], gamma.flat[0]
    bm = S(beta, *_m(d))
    E1p, E2p = S(E1, *_e(t1)), S(E2, *_e(t2))
    f = 4.0 / 3.0
    if visc == -1:
        return a + (beta + bm + E1 + E1p + E2 + E2p) * dxsqinv
    if visc == 1:
        return a + 6.0 * b * dxsqinv
    if visc == -2:
        return a + (2.0 * beta + 2.0 * bm + E1 + E1p + E2 + E2p) * dxsqinv
    if visc == 2:
        return a + 8.0 * b * dxsqinv
    if visc == -3:
        g = gamma
        return a + (f * beta + g + f * bm + S(g, *_m(d)) + E1 + E1p + E2 + E2p) * dxsqinv
    if visc == 3:
        return a + (20.0 / 3.0 * b + 2.0 * c) * dxsqinv
    raise ValueError(visc)


def applyop(visc, phi, alpha, beta, bed, gamma, dx):
    if phi[0].ndim == 2:
        return applyop_2d(visc, phi, alpha, beta, bed[0], gamma, dx)
    return [applyop_3d_comp(c, visc, phi, alpha, beta, bed, gamma, dx) for c in range(3)]


def diag(visc, alpha, beta, bed, gamma, dx):
    if alpha[0].ndim == 2:
        return diag_2d(visc, alpha, beta, bed[0], gamma, dx)
    return [diag_3d_comp(c, visc, alpha, beta, bed, gamma, dx) for c in range(3)]


def smooth_colour(visc, color, rhs, phi, alpha, beta, bed, gamma, dx, omega=1.0):
    """applyop(color) + stag_mg_update(color); color 0 = weighted Jacobi."""
    dm = phi[0].ndim
    L = applyop(visc, phi, alpha, beta, bed, gamma, dx)
    D = diag(visc, alpha, beta, bed, gamma, dx)
    out = [p.copy() for p in phi]
    for c in range(dm):
        if color == 0:
            m = np.ones(phi[c].shape, bool)
        else:
            if (color - 1) // 2 != c:
                continue
            m = colour_mask(phi[c].shape, color)
        upd = phi[c] + omega * (rhs[c] - L[c]) / D[c]
        out[c][m] = upd[m]
    return out


# ------------------------------------------------------------------ transfer
def restrict_stag(phi_f, simple):
    dm = phi_f[0].ndim
    out = []
    for c in range(dm):
        f = phi_f[c]
        if dm == 2:
            a = lambda di, dj: sh(f, di, dj)[0::2, 0::2]
            if c == 0:
                if simple:
                    out.append(0.5 * (a(0, 0) + a(0, 1)))
                else:
                    out.append(0.25 * (a(0, 0) + a(0, 1)) + 0.125 * (a(1, 0) + a(1, 1) + a(-1, 0) + a(-1, 1)))
            else:
                if simple:
                    out.append(0.5 * (a(0, 0) + a(1, 0)))
                else:
                    out.append(0.25 * (a(0, 0) + a(1, 0)) + 0.125 * (a(0, 1) + a(1, 1) + a(0, -1) + a(1, -1)))
        else:
            a = lambda di, dj, dk: sh(f, di, dj, dk)[0::2, 0::2, 0::2]
            # the two transverse offsets in the reference's order
            if c == 0:
                q = [(0, 0, 0), (0, 1, 0), (0, 0, 1), (0, 1, 1)]
                sp, sm = (1, 0, 0), (-1, 0, 0)
            elif c == 1:
                q = [(0, 0, 0), (1, 0, 0), (0, 0, 1), (1, 0, 1)]
                sp, sm = (0, 1, 0), (0, -1, 0)
            else:
                q = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (1, 1, 0)]
                sp, sm = (0, 0, 1), (0, 0, -1)
            s0 = a(*q[0]) + a(*q[1]) + a(*q[2]) + a(*q[3])
            if simple:
                out.append(0.25 * s0)
            else:
                ap = [tuple(x + y for x, y in zip(t, sp)) for t in q]
                am = [tuple(x + y for x, y in zip(t, sm)) for t in q]
                out.append(0.125 * s0 + 0.0625 * (a(*ap[0]) + a(*ap[1]) + a(*ap[2]) + a(*ap[3]))
                           + 0.0625 * (a(*am[0]) + a(*am[1]) + a(*am[2]) + a(*am[3])))
    return out


def prolong_add(phi_f, phi_c):
    dm = phi_f[0].ndim
    out = [p.copy() for p in phi_f]
    if dm == 2:
        ny, nx = phi_f[0].shape
        J, I = np.indices((ny, nx))
        C = lambda arr, ii, jj: arr[jj % arr.shape[0], ii % arr.shape[1]]
        cx, cy = phi_c
        joff = np.where(J % 2 == 0, -1, 1)
        ev = out[0] + 0.75 * C(cx, I // 2, J // 2) + 0.25 * C(cx, I // 2, J // 2 + joff)
        od = (out[0] + 0.375 * C(cx, I // 2, J // 2) + 0.125 * C(cx, I // 2, J // 2 + joff)
              + 0.375 * C(cx, I // 2 + 1, J // 2) + 0.125 * C(cx, I // 2 + 1, J // 2 + joff))
        out[0] = np.where(I % 2 == 0, ev, od)
        ioff = np.where(I % 2 == 0, -1, 1)
        ev = out[1] + 0.75 * C(cy, I // 2, J // 2) + 0.25 * C(cy, I // 2 + ioff, J // 2)
        od = (out[1] + 0.375 * C(cy, I // 2, J // 2) + 0.125 * C(cy, I // 2 + ioff, J // 2)
              + 0.375 * C(cy, I // 2, J // 2 + 1) + 0.125 * C(cy, I // 2 + ioff, J // 2 + 1))
        out[1] = np.where(J % 2 == 0, ev, od)
        return out
    nz, ny, nx = phi_f[0].shape
    K, J, I = np.indices((nz, ny, nx))
    C = lambda arr, ii, jj, kk: arr[kk % arr.shape[0], jj % arr.shape[1], ii % arr.shape[2]]
    n16, t16, o16 = 9.0 / 16.0, 3.0 / 16.0, 1.0 / 16.0
    n32, t32, o32 = 9.0 / 32.0, 3.0 / 32.0, 1.0 / 32.0
    idx = [I, J, K]
    for c in range(3):
        own = idx[c]
        tr = [t for t in range(3) if t != c]
        offs = [np.where(idx[t] % 2 == 0, -1, 1) for t in tr]
        base = [I // 2, J // 2, K // 2]

        def at(delta_own, use1, use2):
            b = list(base)
            b[c] = b[c] + delta_own
            if use1:
                b[tr[0]] = b[tr[0]] + offs[0]
            if use2:
                b[tr[1]] = b[tr[1]] + offs[1]
            return C(phi_c[c], b[0], b[1], b[2])

        ev = out[c] + n16 * at(0, 0, 0) + t16 * at(0, 1, 0) + t16 * at(0, 0, 1) + o16 * at(0, 1, 1)
        od = (out[c] + n32 * at(0, 0, 0) + t32 * at(0, 1, 0) + t32 * at(0, 0, 1) + o32 * at(0, 1, 1)
              + n32 * at(1, 0, 0) + t32 * at(1, 1, 0) + t32 * at(1, 0, 1) + o32 * at(1, 1, 1))
        out[c] = np.where(own % 2 == 0, ev, od)
    return out


def restrict_cc(f):
    if f.ndim == 2:
        return 0.25 * (f[0::2, 0::2] + f[0::2, 1::2] + f[1::2, 0::2] + f[1::2, 1::2])
    return 0.125 * (f[0::2, 0::2, 0::2] + f[0::2, 0::2, 1::2] + f[0::2, 1::2, 0::2] + f[0::2, 1::2, 1::2]
                    + f[1::2, 0::2, 0::2] + f[1::2, 0::2, 1::2] + f[1::2, 1::2, 0::2] + f[1::2, 1::2, 1::2])


def restrict_edges(bed):
    if bed[0].ndim == 2:
        return [bed[0][0::2, 0::2]]  # nodal injection
    xy, xz, yz = bed
    return [0.5 * (xy[0::2, 0::2, 0::2] + xy[1::2, 0::2, 0::2]),
            0.5 * (xz[0::2, 0::2, 0::2] + xz[0::2, 1::2, 0::2]),
            0.5 * (yz[0::2, 0::2, 0::2] + yz[0::2, 0::2, 1::2])]


def grad(p, dx):
    dm = p.ndim
    dxinv = 1.0 / dx
    return [(p - sh(p, *_m(d)[:dm])) * dxinv for d in range(dm)]


def div(u, dx):
    dm = u[0].ndim
    dxinv = 1.0 / dx
    out = (sh(u[0], *_e(0)[:dm]) - u[0]) * dxinv + (sh(u[1], *_e(1)[:dm]) - u[1]) * dxinv
    if dm == 3:
        out = out + (sh(u[2], *_e(2)[:dm]) - u[2]) * dxinv
    return out


def seam_weights(shape, comp):
    """Per-face weight of stag_inner_prod on the unique periodic faces."""
    w = np.ones(shape)
    dm = len(shape)
    axis = dm - 1 - comp
    sl = [slice(None)] * dm
    sl[axis] = 0
    w[tuple(sl)] = 3.0
    return w


def vcycle(visc, rhs, alpha, beta, bed, gamma, dx, nlev, nu1=2, nu2=2, nub=8, smoother=1, omega=1.0):
    """One staggered V-cycle from phi = 0 (stag_mg_solver with max_vcycles=1),
    alpha already multiplied by theta_alpha."""
    dm = rhs[0].ndim
    colours = [0] if smoother == 0 else list(range(1, 2 * dm + 1))
    A, B, E, G, R, P, H = [alpha], [beta], [bed], [gamma], [rhs], [], [dx]
    for lev in range(1, nlev):
        A.append(restrict_stag(A[-1], True))
        B.append(restrict_cc(B[-1]))
        E.append(restrict_edges(E[-1]))
        G.append(restrict_cc(G[-1]))
        H.append(H[-1] * 2.0)
    phi = [[np.zeros_like(r) for r in rhs]]
    for lev in range(nlev - 1):
        ph = phi[lev]
        for _ in range(nu1):
            for col in colours:
                ph = smooth_colour(visc, col, R[lev], ph, A[lev], B[lev], E[lev], G[lev], H[lev], omega)
        phi[lev] = ph
        L = applyop(visc, ph, A[lev], B[lev], E[lev], G[lev], H[lev])
        res = [(L[c] - R[lev][c]) * -1.0 for c in range(dm)]
        R.append(restrict_stag(res, False))
        phi.append([np.zeros_like(r) for r in R[-1]])
    lev = nlev - 1
    ph = phi[lev]
    for _ in range(nub):
        for col in colours:
            ph = smooth_colour(visc, col, R[lev], ph, A[lev], B[lev], E[lev], G[lev], H[lev], omega)
    phi[lev] = ph
    for lev in range(nlev - 2, -1, -1):
        ph = prolong_add(phi[lev], phi[lev + 1])
        for _ in range(nu2):
            for col in colours:
                ph = smooth_colour(visc, col, R[lev], ph, A[lev], B[lev], E[lev], G[lev], H[lev], omega)
        phi[lev] = ph
    return phi[0]
