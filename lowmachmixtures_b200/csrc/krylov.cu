// krylov.cu - FP64 Krylov-side kernels (see krylov.cuh).  Built with
// -fmad=false so every operation rounds like the reference Fortran.
#include <algorithm>

#include "krylov.cuh"
#include "pdl.cuh"
#include "stencil.cuh"

namespace lmm {

namespace {
constexpr int kT = 256;
inline int nb(int64_t n) { return (int)((n + kT - 1) / kT < 1 ? 1 : (n + kT - 1) / kT); }

__device__ __forceinline__ void unflat3(const Dims& D, int t, int& i, int& j, int& k) {
    i = t % D.nx;
    int r = t / D.nx;
    j = r % D.ny;
    k = r / D.ny;
}
}  // namespace

// b_u = stag_applyop(x_u) + grad(x_p);  b_p = -div(x_u)   (apply_matrix.f90:96-112)
// Register budget: 4 blocks of 256 per SM (64 registers; the |visc| = 3
// stencil, which would spill there, 3 blocks).
// W: a grid with walls -- b_u is zero on the wall faces (the applyop is
// zeroed there and the FOEXTRAP pressure has zero wall gradient), and the
// divergence reads the hi+1 wall face as zero
template <int DM, int VISC, class TX, bool W = false>
__global__ void __launch_bounds__(kT, (VISC == 3 || VISC == -3) ? 3 : 4) k_apply_matrix(Dims D, Coef<double> C, const TX* __restrict__ u0,
                                                     const TX* __restrict__ u1, const TX* __restrict__ u2,
                                                     const TX* __restrict__ p, double* __restrict__ o0,
                                                     double* __restrict__ o1, double* __restrict__ o2, double* __restrict__ op,
                                                     double dxsqinv, double dxinv) {
    pdl_enter();
    const Pos q = pos3(D.nx, D.ny);
    if (!q.ok) return;
    Nb nbr = W ? make_nbw(D, q.i, q.j, q.k) : make_nb(D, q.i, q.j, q.k);
    const int t = nbr.s;
    const TX* phi[3] = {u0, u1, u2};
    const double b = ld(C.beta, 0), c = ld(C.gamma, 0);
    auto X = [](const TX* a, int i) { return (double)__ldg(a + i); };
    auto XP = [&](const TX* a, int d) {
        const double v = X(a, t + nbr.op[d]);
        return W ? wapply(wall_mul(nbr, d, d, true), v) : v;
    };
    const double pc = X(p, t);
    if (W && wall_face(nbr, 0)) {
        o0[t] = 0.0;
    } else {
        double L = face_L<double, DM, VISC, 0, 0, TX, W>(phi, C, nbr, dxsqinv, b, c);
        double g = (pc - X(p, t + nbr.om[0])) * dxinv;
        o0[t] = L + g;
    }
    if (W && wall_face(nbr, 1)) {
        o1[t] = 0.0;
    } else {
        double L = face_L<double, DM, VISC, 1, 0, TX, W>(phi, C, nbr, dxsqinv, b, c);
        double g = (pc - X(p, t + nbr.om[1])) * dxinv;
        o1[t] = L + g;
    }
    double dv = (XP(u0, 0) - X(u0, t)) * dxinv + (XP(u1, 1) - X(u1, t)) * dxinv;
    if constexpr (DM == 3) {
        if (W && wall_face(nbr, 2)) {
            o2[t] = 0.0;
        } else {
            double L = face_L<double, DM, VISC, 2, 0, TX, W>(phi, C, nbr, dxsqinv, b, c);
            double g = (pc - X(p, t + nbr.om[2])) * dxinv;
            o2[t] = L + g;
        }
        dv = dv + (XP(u2, 2) - X(u2, t)) * dxinv;
    }
    op[t] = dv * -1.0;
}

template <class TX>
static void apply_matrix_impl(const LevelDev<double>& L0, int visc, const TX* xb, int64_t n, int dm, const SVec& b,
                              cudaStream_t s) {
    const double dxsqinv = 1.0 / (L0.dx * L0.dx);
    const double dxinv = 1.0 / L0.dx;
    // periodic grids: the block shape the autotuner chose (a shape it
    // forces while it times them), else 64 x 4
    Shape sh = forced_shape();
    if (!sh.bx) sh = tuned_shape(TK_APPLY_MATRIX, sizeof(TX), visc, L0.D);
    int bx = L0.D.nx < 64 ? L0.D.nx : 64;
    int by = 256 / bx;
    if (!L0.D.wall && sh.bx) {
        bx = std::min(sh.bx, L0.D.nx);
        by = sh.by ? sh.by : 256 / bx;
    }
    if (by > L0.D.ny) by = L0.D.ny;
    const dim3 blk(bx, by, 1), grd((L0.D.nx + bx - 1) / bx, (L0.D.ny + by - 1) / by, L0.D.nz);
    const TX* x0 = xb;
    const TX* x1 = xb + n;
    const TX* x2 = (dm == 3) ? xb + 2 * n : xb;
    const TX* xp = xb + (int64_t)dm * n;
    double* b2 = (b.dm == 3) ? b.c(2) : b.c(0);
#define AM(DM_, V_)                                                                                                        \
    if (L0.D.wall)                                                                                                         \
        launch_pdl(k_apply_matrix<DM_, V_, TX, true>, grd, blk, 0, s, L0.D, L0.coef(), x0, x1, x2, xp, b.c(0), b.c(1), b2, b.p(), dxsqinv, dxinv); \
    else                                                                                                                   \
        launch_pdl(k_apply_matrix<DM_, V_, TX>, grd, blk, 0, s, L0.D, L0.coef(), x0, x1, x2, xp, b.c(0), b.c(1), b2, b.p(), dxsqinv, dxinv)
#define AMV(DM_)                    \
    switch (visc) {                 \
    case -1: AM(DM_, -1); break;    \
    case 1: AM(DM_, 1); break;      \
    case -2: AM(DM_, -2); break;    \
    case 2: AM(DM_, 2); break;      \
    case -3: AM(DM_, -3); break;    \
    case 3: AM(DM_, 3); break;      \
    }
    if (dm == 2) {
        AMV(2)
    } else {
        AMV(3)
    }
#undef AMV
#undef AM
}

void launch_apply_matrix(const LevelDev<double>& L0, int visc, const SVec& x, const SVec& b, cudaStream_t s) {
    apply_matrix_impl<double>(L0, visc, x.base, x.n, x.dm, b, s);
}
void launch_apply_matrix_f32(const LevelDev<double>& L0, int visc, const float* x, int64_t n, int dm, const SVec& b,
                             cudaStream_t s) {
    apply_matrix_impl<float>(L0, visc, x, n, dm, b, s);
}

__global__ void k_neg_resid(double* __restrict__ out, const double* __restrict__ b, int64_t n) {
    pdl_enter();
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) {
        double v = out[t] - b[t];
        out[t] = v * -1.0;
    }
}
void launch_neg_resid(double* out, const double* b, int64_t n, cudaStream_t s) { launch_pdl(k_neg_resid, nb(n), kT, 0, s, out, b, n); }

__global__ void k_div_by(const double* __restrict__ w, double* __restrict__ v, const double* __restrict__ den, int64_t n) {
    pdl_enter();
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) v[t] = w[t] / *den;
}
void launch_div_by(const double* w, double* v, const double* den, int64_t n, cudaStream_t s) {
    launch_pdl(k_div_by, nb(n), kT, 0, s, w, v, den, n);
}

// v = w / *den, and v32 = (float)v: the next FGMRES basis vector together
// with the FP32 input of the preconditioner that reads it next
__global__ void k_div_by_f32(const double* __restrict__ w, double* __restrict__ v, float* __restrict__ v32,
                             const double* __restrict__ den, int64_t n) {
    pdl_enter();
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) {
        const double q = w[t] / *den;
        v[t] = q;
        v32[t] = (float)q;
    }
}
// the same, four entries per thread by 16-byte loads and stores (n a
// multiple of 4, every pointer 16-byte aligned)
__global__ void k_div_by_f32_x4(const double2* __restrict__ w, double2* __restrict__ v, float4* __restrict__ v32,
                                const double* __restrict__ den, int64_t n4) {
    pdl_enter();
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n4) {
        const double d = *den;
        const double2 a = w[2 * t], b = w[2 * t + 1];
        const double2 qa = make_double2(a.x / d, a.y / d), qb = make_double2(b.x / d, b.y / d);
        v[2 * t] = qa;
        v[2 * t + 1] = qb;
        v32[t] = make_float4((float)qa.x, (float)qa.y, (float)qb.x, (float)qb.y);
    }
}
void launch_div_by_f32(const double* w, double* v, float* v32, const double* den, int64_t n, cudaStream_t s) {
    auto al = [](const void* p) { return ((uintptr_t)p & 15) == 0; };
    if (n % 4 == 0 && al(w) && al(v) && al(v32))
        launch_pdl(k_div_by_f32_x4, nb(n / 4), kT, 0, s, (const double2*)w, (double2*)v, (float4*)v32, den, n / 4);
    else
        launch_pdl(k_div_by_f32, nb(n), kT, 0, s, w, v, v32, den, n);
}

__global__ void k_sub_scaled(double* __restrict__ w, const double* __restrict__ V, const double* __restrict__ h, int64_t n) {
    pdl_enter();
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) {
        double tmp = V[t] * *h;
        w[t] = w[t] - tmp;
    }
}
void launch_sub_scaled(double* w, const double* V, const double* h, int64_t n, cudaStream_t s) {
    launch_pdl(k_sub_scaled, nb(n), kT, 0, s, w, V, h, n);
}

__global__ void k_add_scaled(double* __restrict__ x, const double* __restrict__ V, double y, int64_t n) {
    pdl_enter();
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) {
        double tmp = V[t] * y;
        x[t] = x[t] + tmp;
    }
}
void launch_add_scaled(double* x, const double* V, double y, int64_t n, cudaStream_t s) { launch_pdl(k_add_scaled, nb(n), kT, 0, s, x, V, y, n); }

__global__ void k_add_scaled_f32(double* __restrict__ x, const float* __restrict__ Z, double y, int64_t n) {
    pdl_enter();
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) {
        double tmp = (double)Z[t] * y;
        x[t] = x[t] + tmp;
    }
}
void launch_add_scaled_f32(double* x, const float* Z, double y, int64_t n, cudaStream_t s) {
    launch_pdl(k_add_scaled_f32, nb(n), kT, 0, s, x, Z, y, n);
}

// x += sum_k y_k Z_k in one pass over x: per entry the same sequence of
// roundings as J launches of k_add_scaled_f32 (update_sol, gmres.f90:481-515)
template <int J>
__global__ void k_add_scaled_multi_f32(double* __restrict__ x, MZ32 Z, YS ys, int64_t n) {
    pdl_enter();
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        double v = x[t];
#pragma unroll
        for (int k = 0; k < J; ++k) {
            const double tmp = (double)Z.p[k][t] * ys.y[k];
            v = v + tmp;
        }
        x[t] = v;
    }
}
void launch_add_scaled_multi_f32(double* x, const MZ32& Z, const YS& ys, int J, int64_t n, cudaStream_t s) {
    int64_t b = (n + kT - 1) / kT;
    const int g = (int)(b > 8192 ? 8192 : b);
    switch (J) {
    case 1: launch_pdl(k_add_scaled_multi_f32<1>, g, kT, 0, s, x, Z, ys, n); break;
    case 2: launch_pdl(k_add_scaled_multi_f32<2>, g, kT, 0, s, x, Z, ys, n); break;
    case 3: launch_pdl(k_add_scaled_multi_f32<3>, g, kT, 0, s, x, Z, ys, n); break;
    case 4: launch_pdl(k_add_scaled_multi_f32<4>, g, kT, 0, s, x, Z, ys, n); break;
    case 5: launch_pdl(k_add_scaled_multi_f32<5>, g, kT, 0, s, x, Z, ys, n); break;
    case 6: launch_pdl(k_add_scaled_multi_f32<6>, g, kT, 0, s, x, Z, ys, n); break;
    case 7: launch_pdl(k_add_scaled_multi_f32<7>, g, kT, 0, s, x, Z, ys, n); break;
    default: launch_pdl(k_add_scaled_multi_f32<8>, g, kT, 0, s, x, Z, ys, n); break;
    }
}

// ---------------------------------------------------------------- Schur complement pieces
template <class T>
__global__ void k_schur(int mode, int pt, int av, double theta, const T* __restrict__ mac, const T* __restrict__ src,
                        const T* __restrict__ beta, const T* __restrict__ gamma, T* __restrict__ phi, const T* __restrict__ bp,
                        T* __restrict__ xp, int64_t n) {
    pdl_enter();
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const T th = (T)theta;
    T x = 0;
    if (mode == 0) {  // simple_schur_complement (apply_precon.f90:485-528) [+ sign flip :244-249]
        if (av == 1 || av == 2) {
            x = mac[t] * T(-1);
            x = x * beta[t];
            if (av == 2) x = x * T(2);
        } else {
            x = mac[t] * T(-4.0 / 3.0);
            x = x * beta[t];
            T m2 = mac[t] * T(-1);
            m2 = m2 * gamma[t];
            x = x + m2;
        }
        if (fabs(theta) > 0.0) {
            T ph = phi[t] * th;
            phi[t] = ph;
            x = x + ph;
        }
        if (pt == -2 || pt == -5) x = x * T(-1);
    } else if (mode == 1) {  // projection preconditioner (apply_precon.f90:140-188)
        T sv = (pt == 1 || theta == 0.0) ? mac[t] * T(-1) : src[t];
        if (av == 1 || av == 2) {
            x = sv * beta[t];
            if (av == 2) x = x * T(2);
        } else {
            T m2 = sv * gamma[t];
            x = sv * beta[t];
            x = x * T(4.0 / 3.0);
            x = x + m2;
        }
        T ph = phi[t] * th;
        phi[t] = ph;
        x = x + ph;
    } else {  // block diagonal (apply_precon.f90:380-416)
        T ph = phi[t];
        if (fabs(theta) > 0.0) {
            ph = ph * th;
            phi[t] = ph;
        }
        x = bp[t] * beta[t];
        x = x - ph;
        if (av == 1 && pt == 4) {
            x = x * T(-1);
        } else if (av == 2 && pt == 4) {
            x = x * T(-2);
        } else if (av == 2 && pt == -4) {
            x = x * T(2);
        } else if (av == 3 && pt == 4) {
            x = x * T(-4.0 / 3.0);
            T q = bp[t] * gamma[t];
            q = q * T(-1);
            x = x + q;
        } else if (av == 3 && pt == -4) {
            x = x * T(4.0 / 3.0);
            T q = bp[t] * gamma[t];
            x = x + q;
        }
    }
    xp[t] = x;
}

template <class T>
void launch_schur(int mode, int precon_type, int visc_abs, double theta_alpha, const T* mac_rhs, const T* src,
                  const T* beta, const T* gamma, T* phi, const T* bp, T* xp, int64_t n, cudaStream_t s) {
    launch_pdl(k_schur<T>, nb(n), kT, 0, s, mode, precon_type, visc_abs, theta_alpha, mac_rhs, src, beta, gamma, phi, bp, xp, n);
}
template void launch_schur<double>(int, int, int, double, const double*, const double*, const double*, const double*, double*,
                                   const double*, double*, int64_t, cudaStream_t);
template void launch_schur<float>(int, int, int, double, const float*, const float*, const float*, const float*, float*,
                                  const float*, float*, int64_t, cudaStream_t);

// ---------------------------------------------------------------- mean removal
// sub_u: bit d set = remove the mean of velocity component d
template <class T, int DM>
__global__ void k_sub_means(Dims D, T* u0, T* u1, T* u2, T* p, const double* __restrict__ sums, double total_volume, int sub_u) {
    pdl_enter();
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t n = (int64_t)D.nx * D.ny * D.nz;
    if (t >= n) return;
    // 2D batch: the sums of this entry's instance (slot stride 8)
    if (DM == 2) sums += (int64_t)((int)t / (D.nx * D.ny)) * 8;
    const double mp = sums[DM] / total_volume;
    p[t] = (T)((double)p[t] - mp);
    if (sub_u) {
        T* u[3] = {u0, u1, u2};
#pragma unroll
        for (int d = 0; d < DM; ++d) {
            if (!((sub_u >> d) & 1)) continue;
            const double mu = sums[d] / total_volume;
            u[d][t] = (T)((double)u[d][t] - mu);
        }
    }
}

template <class T>
void launch_sub_means(const Dims& D, T* const u[3], T* p, const double* sums, double total_volume, int sub_u, cudaStream_t s) {
    int64_t n = (int64_t)D.nx * D.ny * D.nz;
    if (D.dm == 2)
        launch_pdl(k_sub_means<T, 2>, nb(n), kT, 0, s, D, u[0], u[1], u[2], p, sums, total_volume, sub_u);
    else
        launch_pdl(k_sub_means<T, 3>, nb(n), kT, 0, s, D, u[0], u[1], u[2], p, sums, total_volume, sub_u);
}
template void launch_sub_means<double>(const Dims&, double* const[3], double*, const double*, double, int, cudaStream_t);
template void launch_sub_means<float>(const Dims&, float* const[3], float*, const double*, double, int, cudaStream_t);

// ---------------------------------------------------------------- layouts
int64_t boxlib_size(const Dims& D, const int nodal[3], int ng) {
    int64_t s = 1;
    const int n[3] = {D.nx, D.ny, D.nz};
    for (int d = 0; d < D.dm; ++d) s *= (int64_t)(n[d] + nodal[d] + 2 * ng);
    return s;
}

__global__ void k_gather_boxlib(Dims D, int ex, int ey, int ng, const double* __restrict__ in, double* __restrict__ out) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int n = D.nx * D.ny * D.nz;
    if (t >= n) return;
    int i, j, k;
    unflat3(D, t, i, j, k);
    const int kg = (D.dm == 3) ? ng : 0;
    out[t] = in[(int64_t)(i + ng) + (int64_t)ex * ((j + ng) + (int64_t)ey * (k + kg))];
}

__global__ void k_scatter_boxlib(Dims D, int ex, int ey, int ez, int ng, const double* __restrict__ in, double* __restrict__ out) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int n = ex * ey * ez;
    if (t >= n) return;
    int I = t % ex;
    int r = t / ex;
    int J = r % ey;
    int K = r / ey;
    const int kg = (D.dm == 3) ? ng : 0;
    int i = ((I - ng) % D.nx + D.nx) % D.nx;
    int j = ((J - ng) % D.ny + D.ny) % D.ny;
    int k = (D.dm == 3) ? ((K - kg) % D.nz + D.nz) % D.nz : 0;
    out[t] = in[(int64_t)i + (int64_t)D.nx * (j + (int64_t)D.ny * k)];
}

void launch_gather_boxlib(const Dims& D, const int nodal[3], int ng, const double* in, double* out, cudaStream_t s) {
    const int ex = D.nx + nodal[0] + 2 * ng, ey = D.ny + nodal[1] + 2 * ng;
    int64_t n = (int64_t)D.nx * D.ny * D.nz;
    k_gather_boxlib<<<nb(n), kT, 0, s>>>(D, ex, ey, ng, in, out);
}

// compact array with extents (cx, cy, cz) (an edge array of a grid with
// walls keeps n+1 nodes along a nodal wall-bounded direction) from its
// BoxLib array (n + nodal + 2 ng entries per direction)
__global__ void k_gather_boxlib_ext(int cx, int cy, int cz, int dm, int ex, int ey, int ng, const double* __restrict__ in,
                                    double* __restrict__ out) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cx * cy * cz) return;
    const int i = t % cx, r = t / cx, j = r % cy, k = r / cy;
    const int kg = (dm == 3) ? ng : 0;
    out[t] = in[(int64_t)(i + ng) + (int64_t)ex * ((j + ng) + (int64_t)ey * (k + kg))];
}

void launch_gather_boxlib_ext(const Dims& D, const int cext[3], const int nodal[3], int ng, const double* in, double* out,
                              cudaStream_t s) {
    const int ex = D.nx + nodal[0] + 2 * ng, ey = D.ny + nodal[1] + 2 * ng;
    const int cz = (D.dm == 3) ? cext[2] : 1;
    k_gather_boxlib_ext<<<nb((int64_t)cext[0] * cext[1] * cz), kT, 0, s>>>(cext[0], cext[1], cz, D.dm, ex, ey, ng, in, out);
}

// BoxLib output of a grid with walls, per direction: periodic -> the image;
// wall, for the face component normal to it -> zero outside lo+1..hi; wall,
// otherwise -> the nearest valid entry, negated for a transverse velocity
// at a no-slip wall.  kind = face component, or -1 for cells.
__global__ void k_scatter_boxlib_w(Dims D, int kind, int ex, int ey, int ez, int ng, const double* __restrict__ in,
                                   double* __restrict__ out) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ex * ey * ez) return;
    const int r = t / ex;
    int x[3] = {t % ex - ng, r % ey - ng, (D.dm == 3) ? r / ey - ng : 0};
    const int n[3] = {D.nx, D.ny, D.nz};
    double sgn = 1.0;
    for (int d = 0; d < D.dm; ++d) {
        int& v = x[d];
        if (!((D.wall >> d) & 1)) {
            v = ((v % n[d]) + n[d]) % n[d];
            continue;
        }
        if (kind == d) {
            if (v <= 0 || v >= n[d]) sgn = 0.0;
            v = v < 0 ? 0 : (v > n[d] - 1 ? n[d] - 1 : v);
            continue;
        }
        if (v < 0) {
            v = 0;
            if (kind >= 0 && !((D.slip_lo >> d) & 1)) sgn = -sgn;
        } else if (v > n[d] - 1) {
            v = n[d] - 1;
            if (kind >= 0 && !((D.slip_hi >> d) & 1)) sgn = -sgn;
        }
    }
    const double v = (sgn == 0.0) ? 0.0 : in[(int64_t)x[0] + (int64_t)D.nx * (x[1] + (int64_t)D.ny * x[2])];
    out[t] = (sgn < 0.0) ? -v : v;
}

void launch_scatter_boxlib_w(const Dims& D, int kind, const int nodal[3], int ng, const double* in, double* out, cudaStream_t s) {
    const int ex = D.nx + nodal[0] + 2 * ng, ey = D.ny + nodal[1] + 2 * ng;
    const int ez = (D.dm == 3) ? D.nz + nodal[2] + 2 * ng : 1;
    k_scatter_boxlib_w<<<nb((int64_t)ex * ey * ez), kT, 0, s>>>(D, kind, ex, ey, ez, ng, in, out);
}

// zero face 0 of each wall-normal component along its wall-bounded direction
__global__ void k_zero_wall_faces(Dims D, double* u0, double* u1, double* u2) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= D.nx * D.ny * D.nz) return;
    int i, j, k;
    unflat3(D, t, i, j, k);
    if ((D.wall & 1) && i == 0) u0[t] = 0.0;
    if (((D.wall >> 1) & 1) && j == 0) u1[t] = 0.0;
    if (D.dm == 3 && ((D.wall >> 2) & 1) && k == 0) u2[t] = 0.0;
}

void launch_zero_wall_faces(const Dims& D, double* const u[3], cudaStream_t s) {
    k_zero_wall_faces<<<nb((int64_t)D.nx * D.ny * D.nz), kT, 0, s>>>(D, u[0], u[1], D.dm == 3 ? u[2] : u[0]);
}

void launch_scatter_boxlib(const Dims& D, const int nodal[3], int ng, const double* in, double* out, cudaStream_t s) {
    const int ex = D.nx + nodal[0] + 2 * ng, ey = D.ny + nodal[1] + 2 * ng;
    const int ez = (D.dm == 3) ? D.nz + nodal[2] + 2 * ng : 1;
    int64_t n = (int64_t)ex * ey * ez;
    k_scatter_boxlib<<<nb(n), kT, 0, s>>>(D, ex, ey, ez, ng, in, out);
}

}  // namespace lmm

// ---------------------------------------------------------------- classical Gram-Schmidt (FGMRES option)
namespace lmm {
namespace {

constexpr int kMdotThreads = 256;

// The last block's sum of every block's partials, entry e of E: warp
// e mod 8 takes it, its lanes stride over the blocks, then a shuffle tree
// (a fixed order for a given grid).  The result goes to sh[e * ld].
template <int E>
__device__ __forceinline__ void sum_partials(const double* partials, double* sh, int ld) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int e = warp; e < E; e += kMdotThreads / 32) {
        double v = 0.0;
        for (unsigned b = lane; b < gridDim.x; b += 32) v += ((volatile const double*)partials)[b * E + e];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[e * ld] = v;
    }
}

// Stokes inner products <w, V_k>, k < J, in one pass over w: per component
// the plain sum plus (seam weight - 1) x the seam-plane sum, as k_reduce
// weighs them; out[k*ss + 4] = sum_d <w_d, V_k,d> + pw^2 <w_p, V_k,p> (ss:
// the stride between consecutive slots).
//
// 2D batches (D.nz instances): blockIdx.y is the instance, with its own
// partials, counter and slot entry (+8 per instance); each instance is
// partitioned and summed as one problem alone.
// (J = 5 held to three blocks per SM: unbounded, the compiler takes the
// registers of two, and two blocks per SM keep too few loads in flight)
template <int DM, int J>
__global__ void __launch_bounds__(kMdotThreads, J == 5 ? 3 : 0) k_mdot(Dims D, const double* __restrict__ w, MVecs V, double wseam, double pw,
                                                       double* __restrict__ partials, unsigned* __restrict__ counter,
                                                       double* __restrict__ out, int64_t ss, int vec) {
    pdl_enter();
    constexpr int NC = DM + 1;
    const int n = D.nx * D.ny * (DM == 3 ? D.nz : 1);  // one instance
    const int64_t N = (int64_t)n * gridDim.y;           // entries per component
    {
        const int64_t io = (int64_t)blockIdx.y * n;
        w += io;
#pragma unroll
        for (int k = 0; k < J; ++k) V.p[k] += io;
        partials += (int64_t)blockIdx.y * gridDim.x * J * NC;
        counter += blockIdx.y;
        out += (int64_t)blockIdx.y * 8;
    }
    double acc[J][NC];
#pragma unroll
    for (int k = 0; k < J; ++k)
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[k][c] = 0.0;
    const int stride = gridDim.x * blockDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (vec) {
        // entry pairs by 16-byte loads (every row even, every vector
        // 16-byte aligned); few vectors: two pairs per thread and pass,
        // so each thread keeps 8 or more loads in flight
        constexpr int U = (J <= 2) ? 2 : 1;
        const int n2 = n >> 1;
        if constexpr (U == 1) {
            // per component: its J + 1 loads, then their products (the
            // compiler overlaps the next component's loads with them)
            for (int p = tid; p < n2; p += stride) {
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    const double2 x = __ldg(reinterpret_cast<const double2*>(w + (int64_t)c * N) + p);
                    double2 v[J];
#pragma unroll
                    for (int k = 0; k < J; ++k) v[k] = __ldg(reinterpret_cast<const double2*>(V.p[k] + (int64_t)c * N) + p);
#pragma unroll
                    for (int k = 0; k < J; ++k) {
                        acc[k][c] += x.x * v[k].x;
                        acc[k][c] += x.y * v[k].y;
                    }
                }
            }
        } else
        for (int p0 = tid; p0 < n2; p0 += U * stride) {
            double2 x[U][NC], v[U][J][NC];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int p = min(p0 + u * stride, n2 - 1);
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    x[u][c] = __ldg(reinterpret_cast<const double2*>(w + (int64_t)c * N) + p);
#pragma unroll
                    for (int k = 0; k < J; ++k) v[u][k][c] = __ldg(reinterpret_cast<const double2*>(V.p[k] + (int64_t)c * N) + p);
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (u > 0 && p0 + u * stride >= n2) break;
#pragma unroll
                for (int c = 0; c < NC; ++c)
#pragma unroll
                    for (int k = 0; k < J; ++k) {
                        acc[k][c] += x[u][c].x * v[u][k][c].x;
                        acc[k][c] += x[u][c].y * v[u][k][c].y;
                    }
            }
        }
    } else {
        for (int t = tid; t < n; t += stride) {
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const double x = __ldg(w + (int64_t)c * N + t);
#pragma unroll
                for (int k = 0; k < J; ++k) acc[k][c] += x * __ldg(V.p[k] + (int64_t)c * N + t);
            }
        }
    }
    // seam planes of the face components (x: i == 0, y: j == 0, z: k == 0)
#pragma unroll
    for (int c = 0; c < DM; ++c) {
        const int nzi = (DM == 3) ? D.nz : 1;
        const int m = (c == 0) ? D.ny * nzi : (c == 1 ? D.nx * nzi : D.nx * D.ny);
        double v[J];
#pragma unroll
        for (int k = 0; k < J; ++k) v[k] = 0.0;
        for (int q = tid; q < m; q += stride) {
            int t;
            if (c == 0) t = D.nx * q;
            else if (c == 1) t = (q % D.nx) + D.nx * D.ny * (q / D.nx);
            else t = q;
            const double x = __ldg(w + (int64_t)c * N + t);
#pragma unroll
            for (int k = 0; k < J; ++k) v[k] += x * __ldg(V.p[k] + (int64_t)c * N + t);
        }
#pragma unroll
        for (int k = 0; k < J; ++k) acc[k][c] += (wseam - 1.0) * v[k];
    }
    __shared__ double sh[J * NC][kMdotThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < J; ++k)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            double v = acc[k][c];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) sh[k * NC + c][warp] = v;
        }
    __syncthreads();
    if (threadIdx.x < J * NC) {
        double v = 0.0;
        for (int q = 0; q < kMdotThreads / 32; ++q) v += sh[threadIdx.x][q];
        partials[blockIdx.x * J * NC + threadIdx.x] = v;
    }
    __threadfence();
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    sum_partials<J * NC>(partials, &sh[0][0], kMdotThreads / 32);
    __syncthreads();
    if (threadIdx.x < J) {
        const int k = threadIdx.x;
        double su = 0.0;
        for (int c = 0; c < DM; ++c) su = su + sh[k * NC + c][0];
        out[k * ss + 4] = su + (pw * pw) * sh[k * NC + DM][0];
    }
    if (threadIdx.x == 0) *counter = 0u;
}

// w -= sum_k h_k V_k, h_k = hs[k * ss + 4] (a 2D batch: the entry's
// instance b = (t % N) / ni reads hs[k * ss + 8b + 4]; one problem: N = ni)
template <int J>
__global__ void k_maxpy(double* __restrict__ w, MVecs V, const double* __restrict__ hs, int64_t len, int64_t N, int64_t ni, int64_t ss) {
    pdl_enter();
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < len; t += (int64_t)gridDim.x * blockDim.x) {
        const double* hb = (N >= len) ? hs : hs + ((t % N) / ni) * 8;
        double x = w[t];
#pragma unroll
        for (int k = 0; k < J; ++k) x = x - V.p[k][t] * hb[k * ss + 4];
        w[t] = x;
    }
}

// w -= sum_k h_k V_k (as k_maxpy) and, in the same pass, the Stokes norm of
// the new w with the seam weight applied per entry: out[5] = sqrt(|u|^2 +
// (pw |p|)^2), out[4] the squared form (as k_reduce's slots)
template <int DM, int J>
__global__ void __launch_bounds__(kMdotThreads) k_maxpy_norm(Dims D, double* __restrict__ w, MVecs V, const double* __restrict__ hs,
                                                             double wseam, double pw, double* __restrict__ partials,
                                                             unsigned* __restrict__ counter, double* __restrict__ out, int64_t ss,
                                                             int vec) {
    pdl_enter();
    constexpr int NC = DM + 1;
    const int n = D.nx * D.ny * (DM == 3 ? D.nz : 1);  // one instance (blockIdx.y, as k_mdot)
    const int64_t N = (int64_t)n * gridDim.y;
    {
        const int64_t io = (int64_t)blockIdx.y * n;
        w += io;
#pragma unroll
        for (int k = 0; k < J; ++k) V.p[k] += io;
        hs += (int64_t)blockIdx.y * 8;
        partials += (int64_t)blockIdx.y * gridDim.x * NC;
        counter += blockIdx.y;
        out += (int64_t)blockIdx.y * 8;
    }
    double h[J];
#pragma unroll
    for (int k = 0; k < J; ++k) h[k] = hs[k * ss + 4];
    double acc[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[c] = 0.0;
    const int stride = gridDim.x * blockDim.x;
    if (vec) {
        // entry pairs (2p, 2p+1) of one row by 16-byte loads and stores
        // (every row even, every vector 16-byte aligned)
        const int n2 = n >> 1;
        for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n2; p += stride) {
            const int t = 2 * p;
            const int i = t % D.nx, r = t / D.nx, j = r % D.ny, kk = r / D.ny;
            double2 x[NC], v[J][NC];
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                x[c] = reinterpret_cast<const double2*>(w + (int64_t)c * N)[p];
#pragma unroll
                for (int k = 0; k < J; ++k) v[k][c] = __ldg(reinterpret_cast<const double2*>(V.p[k] + (int64_t)c * N) + p);
            }
#pragma unroll
            for (int c = 0; c < NC; ++c) {
#pragma unroll
                for (int k = 0; k < J; ++k) {
                    x[c].x = x[c].x - v[k][c].x * h[k];
                    x[c].y = x[c].y - v[k][c].y * h[k];
                }
                reinterpret_cast<double2*>(w + (int64_t)c * N)[p] = x[c];
                // entry 2p+1 has i > 0: only the y and z seams reach it
                const bool seam_yz = (c == 1 && j == 0) || (c == 2 && c < DM && kk == 0);
                const bool seam0 = (c == 0 && i == 0) || seam_yz;
                acc[c] += (seam0 ? wseam : 1.0) * (x[c].x * x[c].x);
                acc[c] += (seam_yz ? wseam : 1.0) * (x[c].y * x[c].y);
            }
        }
    } else {
        for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
            const int i = t % D.nx, r = t / D.nx, j = r % D.ny, kk = r / D.ny;
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const int64_t e = (int64_t)c * N + t;
                double x = w[e];
#pragma unroll
                for (int k = 0; k < J; ++k) x = x - V.p[k][e] * h[k];
                w[e] = x;
                const bool seam = (c == 0 && i == 0) || (c == 1 && j == 0) || (c == 2 && c < DM && kk == 0);
                acc[c] += (seam ? wseam : 1.0) * (x * x);
            }
        }
    }
    __shared__ double sh[NC][kMdotThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        double v = acc[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[c][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < NC) {
        double v = 0.0;
        for (int q = 0; q < kMdotThreads / 32; ++q) v += sh[threadIdx.x][q];
        partials[blockIdx.x * NC + threadIdx.x] = v;
    }
    __threadfence();
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    sum_partials<NC>(partials, &sh[0][0], kMdotThreads / 32);
    __syncthreads();
    if (threadIdx.x == 0) {
        double su = 0.0;
        for (int c = 0; c < DM; ++c) su = su + sh[c][0];
        out[4] = su + (pw * pw) * sh[DM][0];
        const double nu = sqrt(su), np = pw * sqrt(sh[DM][0]);
        out[5] = sqrt(nu * nu + np * np);
        *counter = 0u;
    }
}

}  // namespace

namespace {
template <int DM, int J, bool NORM>
int cgs_blocks(int64_t n);
// the Gram-Schmidt passes may take entries in pairs: rows of even length
// (no pair straddles a row or an instance) and 16-byte aligned vectors
int pairs_ok(const Dims& D, const void* w, const MVecs& V, int J) {
    auto al = [](const void* p) { return ((uintptr_t)p & 15) == 0; };
    bool ok = (D.nx % 2 == 0) && al(w);
    for (int k = 0; k < J && k < 8; ++k) ok = ok && al(V.p[k]);
    return ok ? 1 : 0;
}
}
void launch_maxpy_norm(const Dims& D, double* w, const MVecs& V, int J, const double* hs, double wseam, double pw, double* partials,
                       unsigned* counter, double* out, cudaStream_t s, int ninst, int64_t ss) {
    const int64_t n = (int64_t)D.nx * D.ny * (D.dm == 3 ? D.nz : 1);
    const int vec = pairs_ok(D, w, V, J);
#define MN(DM_, J_) launch_pdl(k_maxpy_norm<DM_, J_>, dim3(cgs_blocks<DM_, J_, true>(n), ninst), dim3(kMdotThreads), 0, s, D, w, V, hs, wseam, pw, partials, counter, out, ss, vec)
#define MNJ(DM_)                               \
    switch (J) {                               \
    case 1: MN(DM_, 1); break;                 \
    case 2: MN(DM_, 2); break;                 \
    case 3: MN(DM_, 3); break;                 \
    case 4: MN(DM_, 4); break;                 \
    case 5: MN(DM_, 5); break;                 \
    case 6: MN(DM_, 6); break;                 \
    case 7: MN(DM_, 7); break;                 \
    default: MN(DM_, 8); break;                \
    }
    if (D.dm == 2) { MNJ(2) } else { MNJ(3) }
#undef MNJ
#undef MN
}

int mdot_blocks(int64_t n) {
    int64_t b = (n + 2047) / 2048;
    if (b > 592) b = 592;  // 4 CTAs per SM; partials hold 592 x 8 x 4
    return (int)(b < 1 ? 1 : b);
}

namespace {
// blocks of one Gram-Schmidt pass: mdot_blocks(n), but no more than fit in
// one wave of this kernel (its resident blocks per SM x SMs): a second,
// partial wave would leave most SMs idle while it runs
template <int DM, int J, bool NORM>
int cgs_blocks(int64_t n) {
    static const int wave = [] {
        int dev = 0, sms = 148, per_sm = 4;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const void* k = NORM ? (const void*)k_maxpy_norm<DM, J> : (const void*)k_mdot<DM, J>;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kMdotThreads, 0) != cudaSuccess || per_sm < 1) {
            cudaGetLastError();
            per_sm = 1;
        }
        return per_sm * sms;
    }();
    return std::min(mdot_blocks(n), wave);
}
}  // namespace

void launch_mdot(const Dims& D, const double* w, const MVecs& V, int J, double wseam, double pw, double* partials, unsigned* counter,
                 double* out, cudaStream_t s, int ninst, int64_t ss) {
    const int64_t n = (int64_t)D.nx * D.ny * (D.dm == 3 ? D.nz : 1);
    const int vec = pairs_ok(D, w, V, J);
#define MD(DM_, J_) launch_pdl(k_mdot<DM_, J_>, dim3(cgs_blocks<DM_, J_, false>(n), ninst), dim3(kMdotThreads), 0, s, D, w, V, wseam, pw, partials, counter, out, ss, vec)
#define MDJ(DM_)                               \
    switch (J) {                               \
    case 1: MD(DM_, 1); break;                 \
    case 2: MD(DM_, 2); break;                 \
    case 3: MD(DM_, 3); break;                 \
    case 4: MD(DM_, 4); break;                 \
    case 5: MD(DM_, 5); break;                 \
    case 6: MD(DM_, 6); break;                 \
    case 7: MD(DM_, 7); break;                 \
    default: MD(DM_, 8); break;                \
    }
    if (D.dm == 2) { MDJ(2) } else { MDJ(3) }
#undef MDJ
#undef MD
}

void launch_maxpy(double* w, const MVecs& V, int J, const double* hs, int64_t len, cudaStream_t s, int64_t N, int64_t ni, int64_t ss) {
    int64_t b = (len + kT - 1) / kT;
    const int nb = (int)(b > 8192 ? 8192 : b);
    if (N <= 0) N = ni = len;  // one problem: every entry reads hs[k * ss + 4]
    switch (J) {
    case 1: launch_pdl(k_maxpy<1>, nb, kT, 0, s, w, V, hs, len, N, ni, ss); break;
    case 2: launch_pdl(k_maxpy<2>, nb, kT, 0, s, w, V, hs, len, N, ni, ss); break;
    case 3: launch_pdl(k_maxpy<3>, nb, kT, 0, s, w, V, hs, len, N, ni, ss); break;
    case 4: launch_pdl(k_maxpy<4>, nb, kT, 0, s, w, V, hs, len, N, ni, ss); break;
    case 5: launch_pdl(k_maxpy<5>, nb, kT, 0, s, w, V, hs, len, N, ni, ss); break;
    case 6: launch_pdl(k_maxpy<6>, nb, kT, 0, s, w, V, hs, len, N, ni, ss); break;
    case 7: launch_pdl(k_maxpy<7>, nb, kT, 0, s, w, V, hs, len, N, ni, ss); break;
    default: launch_pdl(k_maxpy<8>, nb, kT, 0, s, w, V, hs, len, N, ni, ss); break;
    }
}

// ---------------------------------------------------------------- 2D batches
// A batch stacks B independent 2D problems of ni = nx*ny cells along the
// third index: entry e of a Stokes vector (component c at c*n, n = ni*B)
// belongs to instance (e % n) / ni.  Per-instance scalars live in slot
// arrays of B x 8 doubles (instance b at [8b], the k_reduce layout).  Each
// kernel computes, per entry, the expression of its one-problem counterpart
// above with that instance's scalar.
namespace {

__device__ __forceinline__ int inst_of(int64_t e, int64_t n, int ni) { return (int)((e % n) / ni); }

// v = w / den_b (den_b = slots[8b + 5]); v32 (may be null) = (float)v.  A
// zero norm (an instance that has stopped: its column is not used) divides
// by 1 instead.
__global__ void k_div_by_batch(const double* __restrict__ w, double* __restrict__ v, float* __restrict__ v32,
                               const double* __restrict__ slots, int64_t n, int ni, int64_t len) {
    pdl_enter();
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= len) return;
    const double d = slots[(int64_t)inst_of(e, n, ni) * 8 + 5];
    const double q = w[e] / (d != 0.0 ? d : 1.0);
    v[e] = q;
    if (v32) v32[e] = (float)q;
}

// w -= V * h_b (h_b = slots[8b + 4])
__global__ void k_sub_scaled_batch(double* __restrict__ w, const double* __restrict__ V, const double* __restrict__ slots, int64_t n,
                                   int ni, int64_t len) {
    pdl_enter();
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= len) return;
    const double tmp = V[e] * slots[(int64_t)inst_of(e, n, ni) * 8 + 4];
    w[e] = w[e] - tmp;
}

// x += sum_{k<J} ys[k*B + b] Z_k, in k order; a zero coefficient (an
// instance whose cycle had fewer columns) is skipped
template <class TZ>
__global__ void k_add_scaled_multi_batch(double* __restrict__ x, const TZ* const* __restrict__ Z, const double* __restrict__ ys, int J,
                                         int nbatch, int64_t n, int ni, int64_t len) {
    pdl_enter();
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < len; e += (int64_t)gridDim.x * blockDim.x) {
        const int b = inst_of(e, n, ni);
        double v = x[e];
        for (int k = 0; k < J; ++k) {
            const double y = ys[(int64_t)k * nbatch + b];
            if (y == 0.0) continue;
            const double tmp = (double)Z[k][e] * y;
            v = v + tmp;
        }
        x[e] = v;
    }
}

// dst[b * ni + t] = src[b][t] and back (per-instance arrays <-> batch array)
__global__ void k_gather_ptrs(const double* const* __restrict__ src, double* __restrict__ dst, int ni, int count) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= (int64_t)ni * count) return;
    const int b = (int)(e / ni), t = (int)(e - (int64_t)b * ni);
    dst[e] = src[b][t];
}
__global__ void k_scatter_ptrs(const double* __restrict__ src, double* const* __restrict__ dst, int ni, int count) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= (int64_t)ni * count) return;
    const int b = (int)(e / ni), t = (int)(e - (int64_t)b * ni);
    dst[b][t] = src[e];
}

}  // namespace

void launch_div_by_batch(const double* w, double* v, float* v32, const double* slots, int64_t n, int ni, int64_t len, cudaStream_t s) {
    launch_pdl(k_div_by_batch, nb(len), kT, 0, s, w, v, v32, slots, n, ni, len);
}
void launch_sub_scaled_batch(double* w, const double* V, const double* slots, int64_t n, int ni, int64_t len, cudaStream_t s) {
    launch_pdl(k_sub_scaled_batch, nb(len), kT, 0, s, w, V, slots, n, ni, len);
}
template <class TZ>
void launch_add_scaled_multi_batch(double* x, const TZ* const* Z_dev, const double* ys_dev, int J, int nbatch, int64_t n, int ni,
                                   int64_t len, cudaStream_t s) {
    const int64_t b = (len + kT - 1) / kT;
    const int g = (int)(b > 8192 ? 8192 : b);
    launch_pdl(k_add_scaled_multi_batch<TZ>, g, kT, 0, s, x, Z_dev, ys_dev, J, nbatch, n, ni, len);
}
template void launch_add_scaled_multi_batch<float>(double*, const float* const*, const double*, int, int, int64_t, int, int64_t,
                                                   cudaStream_t);
template void launch_add_scaled_multi_batch<double>(double*, const double* const*, const double*, int, int, int64_t, int, int64_t,
                                                    cudaStream_t);
void launch_gather_ptrs(const double* const* src_dev, double* dst, int ni, int count, cudaStream_t s) {
    k_gather_ptrs<<<nb((int64_t)ni * count), kT, 0, s>>>(src_dev, dst, ni, count);
}
void launch_scatter_ptrs(const double* src, double* const* dst_dev, int ni, int count, cudaStream_t s) {
    k_scatter_ptrs<<<nb((int64_t)ni * count), kT, 0, s>>>(src, dst_dev, ni, count);
}

}  // namespace lmm

// the bounds-check table and record of this translation unit (empty
// unless built with -DLMM_BOUNDS_CHECK)
LMM_BC_UNIT(krylov)
