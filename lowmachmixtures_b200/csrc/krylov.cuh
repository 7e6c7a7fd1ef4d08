// krylov.cuh - FP64 Krylov-side kernels: the fused Stokes operator, the
// BLAS-1 steps of GMRES, the block-preconditioner pointwise steps and the
// BoxLib <-> compact layout converters.  Built into krylov.cu with
// -fmad=false (reference rounding).
//
//   apply_matrix      src_gmres/apply_matrix.f90:96-112
//   residual, MGS, V(i+1) = w/H, update_sol
//                     src_gmres/gmres.f90:186-194, 338-375, 481-515
//   simple_schur_complement / P1 / P4 pressure updates
//                     src_gmres/apply_precon.f90:140-188, 380-416, 479-534
//   mean removal      src_gmres/apply_precon.f90:433-460
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"

namespace lmm {

// Stokes vector: dm face components then the cell field, each n entries,
// contiguous (c * n offsets).
struct SVec {
    double* base = nullptr;
    int64_t n = 0;
    int dm = 0;
    double* c(int k) const { return base + (int64_t)k * n; }
    double* p() const { return base + (int64_t)dm * n; }
    int64_t size() const { return (int64_t)(dm + 1) * n; }
};

// up to 8 Stokes vectors (their bases; components at c * n)
struct MVecs {
    const double* p[8];
};
// classical Gram-Schmidt pieces: out[k*ss+4] = <w, V_k> (Stokes inner
// product with the seam weight), then w -= sum_k out[k*ss+4] V_k; J <= 8.
// ss: stride between consecutive slots (8 for one problem).  A 2D batch
// (D.nz = ninst instances, slot arrays of ninst x 8): one result per
// instance at + 8b, ss = 8 * ninst; N = entries per component and ni per
// instance (k_maxpy; N = 0: one problem)
int mdot_blocks(int64_t n);
void launch_mdot(const Dims& D, const double* w, const MVecs& V, int J, double wseam, double pw, double* partials, unsigned* counter,
                 double* out, cudaStream_t s, int ninst = 1, int64_t ss = 8);
void launch_maxpy(double* w, const MVecs& V, int J, const double* hs, int64_t len, cudaStream_t s, int64_t N = 0, int64_t ni = 0,
                  int64_t ss = 8);
// the same update fused with the Stokes norm of the new w (seam weight per
// entry): out[4] = |u|^2 + pw^2 |p|^2, out[5] = its square root form
void launch_maxpy_norm(const Dims& D, double* w, const MVecs& V, int J, const double* hs, double wseam, double pw, double* partials,
                       unsigned* counter, double* out, cudaStream_t s, int ninst = 1, int64_t ss = 8);
// FP32 Krylov vectors (FGMRES Z basis) and their coefficients, up to 8
struct MZ32 {
    const float* p[8];
};
struct YS {
    double y[8];
};
// x += sum_k y_k Z_k (k < J <= 8), one pass over x
void launch_add_scaled_multi_f32(double* x, const MZ32& Z, const YS& ys, int J, int64_t n, cudaStream_t s);
// v = w / *den and v32 = (float)v
void launch_div_by_f32(const double* w, double* v, float* v32, const double* den, int64_t n, cudaStream_t s);

void launch_apply_matrix(const LevelDev<double>& L0, int visc, const SVec& x, const SVec& b, cudaStream_t s);
// the same operator applied to an FP32 Stokes vector (FGMRES Z storage), FP64 arithmetic
void launch_apply_matrix_f32(const LevelDev<double>& L0, int visc, const float* x, int64_t n, int dm, const SVec& b,
                             cudaStream_t s);
// out = (out - b) * -1  (gmres.f90:186-194)
void launch_neg_resid(double* out, const double* b, int64_t n, cudaStream_t s);
// v = w / (*den)   (multifab_div_div_s_c)
void launch_div_by(const double* w, double* v, const double* den, int64_t n, cudaStream_t s);
// w = w - V * (*h)
void launch_sub_scaled(double* w, const double* V, const double* h, int64_t n, cudaStream_t s);
// x = x + V * y
void launch_add_scaled(double* x, const double* V, double y, int64_t n, cudaStream_t s);
void launch_add_scaled_f32(double* x, const float* Z, double y, int64_t n, cudaStream_t s);

// pressure updates of apply_precon: mode 0 simple Schur (P2/P3/P5),
// mode 1 projection (P1), mode 2 block diagonal (P4)
template <class T>
void launch_schur(int mode, int precon_type, int visc_abs, double theta_alpha, const T* mac_rhs, const T* src,
                  const T* beta, const T* gamma, T* phi, const T* bp, T* xp, int64_t n, cudaStream_t s);
// x_p -= <p>; x_u[d] -= <u_d> for each bit d of sub_u (means from reduction slots)
template <class T>
void launch_sub_means(const Dims& D, T* const u[3], T* p, const double* sums, double total_volume, int sub_u,
                      cudaStream_t s);

// BoxLib <-> compact (ng ghost layers, nodal flags per direction)
void launch_gather_boxlib(const Dims& D, const int nodal[3], int ng, const double* in, double* out, cudaStream_t s);
void launch_scatter_boxlib(const Dims& D, const int nodal[3], int ng, const double* in, double* out, cudaStream_t s);
int64_t boxlib_size(const Dims& D, const int nodal[3], int ng);
// walls: gather into compact extents cext (edge arrays keep n+1 nodes along
// a nodal wall-bounded direction); scatter a face component (kind = c) or
// the cell field (kind = -1) with the wall ghost rules
void launch_gather_boxlib_ext(const Dims& D, const int cext[3], const int nodal[3], int ng, const double* in, double* out,
                              cudaStream_t s);
void launch_scatter_boxlib_w(const Dims& D, int kind, const int nodal[3], int ng, const double* in, double* out, cudaStream_t s);
// zero the wall faces (face 0 of each wall-normal component)
void launch_zero_wall_faces(const Dims& D, double* const u[3], cudaStream_t s);

// 2D batches: B instances of ni cells stacked along the third index (n =
// ni*B per component, len = (dm+1)*n); per-instance scalars in slot arrays
// of B x 8 doubles.
// v = w / slots[8b+5] (v32, if not null, = (float)v)
void launch_div_by_batch(const double* w, double* v, float* v32, const double* slots, int64_t n, int ni, int64_t len, cudaStream_t s);
// w -= V * slots[8b+4]
void launch_sub_scaled_batch(double* w, const double* V, const double* slots, int64_t n, int ni, int64_t len, cudaStream_t s);
// x += sum_{k<J} ys[k*B+b] Z_k (Z_dev: device table of J vectors)
template <class TZ>
void launch_add_scaled_multi_batch(double* x, const TZ* const* Z_dev, const double* ys_dev, int J, int nbatch, int64_t n, int ni,
                                   int64_t len, cudaStream_t s);
// dst[b*ni + t] = src[b][t] / dst[b][t] = src[b*ni + t] (device pointer tables)
void launch_gather_ptrs(const double* const* src_dev, double* dst, int ni, int count, cudaStream_t s);
void launch_scatter_ptrs(const double* src, double* const* dst_dev, int ni, int count, cudaStream_t s);

}  // namespace lmm
