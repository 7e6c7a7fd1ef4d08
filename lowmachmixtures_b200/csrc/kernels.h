// kernels.h - host-side launchers of the staggered Stokes kernels.
//
// Every launcher is templated on the arithmetic type T (double for the
// reference-faithful path, float for the mixed-precision preconditioner) and
// explicitly instantiated in kernels_fp64.cu (built with -fmad=false) and
// kernels_fp32.cu.
#pragma once
#include <initializer_list>
#include <cuda_runtime.h>

#include <cstdint>

#include "stencil.cuh"

namespace lmm {

// One level of the staggered hierarchy on the device (compact layout).
template <class T>
struct LevelDev {
    Dims D;
    double dx;
    int64_t n;          // cells (= faces per component)
    T* alpha[3];        // theta*alpha at this level
    T* beta;
    T* bed[3];
    T* gamma;
    T* phi[3];
    T* rhs[3];
    T* tmp[3];          // Jacobi output / scratch
    // pressure (cell-centred) multigrid level
    T* pa[3];           // face coefficient 1/alpha (coarsened)
    // every entry of pa holds the same value pa_value (checked on the
    // device at every coefficient load): the pressure kernels then take it
    // as a scalar instead of reading three face arrays
    int pa_uniform;
    T pa_value;
    // every face of alpha[0..dm-1] holds a_value (checked on the device at
    // every coefficient load): the velocity operator takes it as a scalar
    int a_uniform = 0;
    T a_value = T(0);
    T* pmu[3];          // BFBt: face coefficient 1/diag(viscous operator) (coarsened)
    T* pphi;
    T* prhs;
    T* ptmp;
    Coef<T> coef() const {
        Coef<T> c;
        for (int d = 0; d < 3; ++d) { c.alpha[d] = alpha[d]; c.bed[d] = bed[d]; }
        c.alpha_uniform = a_uniform;
        c.alpha_u = a_value;
        c.beta = beta;
        c.gamma = gamma;
        return c;
    }
};

// ---- staggered operator / multigrid ----
// color 0: every face; 1..2*dm: only the faces of that Gauss-Seidel colour
template <class T>
void launch_applyop(const LevelDev<T>& L, int visc, const T* const phi[3], T* const out[3], cudaStream_t s, int color);
// reverse: the launch takes the planes in decreasing k (same values; see
// k_gs_colour)
template <class T>
void launch_gs_colour(const LevelDev<T>& L, int visc, int color, const T* const rhs[3], T* const phi[3], double omega,
                      cudaStream_t s, int reverse = 0);
// Both Gauss-Seidel colours of component comp in one launch, out of place:
// cur[] are read, the new values of component comp go to out (3D levels with
// even sizes; gs_pair_supported says whether the level qualifies).  kc > 0
// forces the k-chunk per block, 0 picks it from the level size.
template <class T>
bool gs_pair_supported(const LevelDev<T>& L, int kc);
template <class T>
void launch_gs_pair(const LevelDev<T>& L, int visc, int comp, const T* const rhs[3], const T* const cur[3], T* out, double omega,
                    int kc, cudaStream_t s);
// Both Gauss-Seidel colours of component comp in one launch whose operands
// are staged in shared memory by TMA tensor copies, marching through
// k-slabs (gs_tma.cuh); out of place like launch_gs_pair.  Periodic 3D
// levels with even sizes and rows of at most 256 faces (gs_tma_supported).
// ty_req / slabs_req > 0 force the rows per tile / the k-slabs; *err is set
// when a bounded wait of the kernel gave up.
template <class T>
bool gs_tma_supported(const LevelDev<T>& L, int visc, int ty_req, int slabs_req);
template <class T>
cudaError_t launch_gs_pair_tma(const LevelDev<T>& L, int visc, int comp, const T* const rhs[3], const T* const cur[3], T* out,
                               double omega, int ty_req, int slabs_req, int* err, cudaStream_t s);
template <class T>
void launch_jacobi(const LevelDev<T>& L, int visc, const T* const rhs[3], const T* const phi_in[3], T* const phi_out[3],
                   double omega, cudaStream_t s);
// fused = 1: residual and restriction in one pass through shared memory
// (3D periodic levels whose coarse sizes divide the tile), else a residual
// kernel into F.tmp and a restriction kernel
template <class T>
void launch_residual_restrict(const LevelDev<T>& F, const LevelDev<T>& Cc, int visc, const T* const rhs_f[3],
                              const T* const phi_f[3], T* const rhs_c[3], cudaStream_t s, int fused = 0);
template <class T>
void launch_prolong_add(const LevelDev<T>& F, const LevelDev<T>& Cc, const T* const phi_c[3], T* const phi_f[3],
                        cudaStream_t s);
template <class T>
void launch_coarsen_coeffs(const LevelDev<T>& F, const LevelDev<T>& Cc, bool pressure_faces, cudaStream_t s);

// The same four operations on a grid with walls (walls.cuh; the launchers
// above hand wall-bounded levels to these)
template <class T>
void wl_applyop(const LevelDev<T>& L, int visc, const T* const phi[3], T* const out[3], cudaStream_t s, int color);
template <class T>
void wl_gs_colour(const LevelDev<T>& L, int visc, int color, const T* const rhs[3], T* const phi[3], double omega, cudaStream_t s,
                  int reverse = 0);
template <class T>
void wl_jacobi(const LevelDev<T>& L, int visc, const T* const rhs[3], const T* const phi_in[3], T* const phi_out[3], double omega,
               cudaStream_t s);
template <class T>
void wl_residual_restrict(const LevelDev<T>& F, const LevelDev<T>& Cc, int visc, const T* const rhs_f[3], const T* const phi_f[3],
                          T* const rhs_c[3], cudaStream_t s);
template <class T>
void wl_prolong_add(const LevelDev<T>& F, const LevelDev<T>& Cc, const T* const phi_c[3], T* const phi_f[3], cudaStream_t s);

// The coarse end of a V-cycle (levels L[0..nl-1], L[0] already holding its
// rhs) in one single-block launch with every level in shared memory (tail.cuh).
template <class T>
cudaError_t launch_vcycle_tail(const LevelDev<T>* L, int nl, int visc, int nu1, int nu2, int nub, int smoother, double omega,
                               cudaStream_t s);
template <class T>
cudaError_t launch_ccmg_tail(const LevelDev<T>* L, int nl, int nu1, int nu2, int nub, cudaStream_t s);
template <class T>
size_t tail_smem_bytes(const LevelDev<T>* L, int nl, bool stag, bool jacobi);

// ---- pressure multigrid (this library's cell-centred V-cycle) ----
// reverse: the launch takes the planes in decreasing order (same values)
template <class T>
void launch_cc_smooth(const LevelDev<T>& L, int parity, cudaStream_t s, int reverse = 0);
template <class T>
void launch_cc_residual_restrict(const LevelDev<T>& F, const LevelDev<T>& Cc, cudaStream_t s);
// *flag |= 1 when the level's pressure face coefficients are not all the
// same value (bit for bit)
template <class T>
void launch_uniform_check(const LevelDev<T>& L, int* flag, cudaStream_t s, bool velocity = false);
template <class T>
void launch_cc_prolong_add(const LevelDev<T>& F, const LevelDev<T>& Cc, cudaStream_t s);
template <class T>
void launch_neg_cc_lap(const LevelDev<T>& L, const T* phi, T* out, cudaStream_t s);

// ---- BFBt Schur approximation (visc_schur_approx = 1) ----
// m = 1 / diag of the viscous operator per face (|visc| 1 or 2)
template <class T>
void launch_inverse_diag_lap(const LevelDev<T>& L, int visc, T* const m[3], cudaStream_t s);
// g = m * grad(phi)
template <class T>
void launch_grad_mul(const LevelDev<T>& L, const T* phi, const T* const m[3], T* const g[3], cudaStream_t s);
// out = div(m * l)
template <class T>
void launch_div_mul(const LevelDev<T>& L, const T* const l[3], const T* const m[3], T* out, cudaStream_t s);

// ---- elementwise pieces of apply_precon (level-0 geometry) ----
// mac_rhs = div(u) + b_p
template <class T>
void launch_div_plus(const LevelDev<T>& L, const T* const u[3], const T* bp, T* out, cudaStream_t s);
// u -= coef * grad(phi); coef == nullptr means coefficient 1
template <class T>
void launch_sub_weighted_grad(const LevelDev<T>& L, const T* const coef[3], const T* phi, T* const u[3], cudaStream_t s);

// ---- conversions and small vector ops ----
template <class Tin, class Tout>
void launch_convert(const Tin* in, Tout* out, int64_t n, cudaStream_t s);
template <class T>
void launch_scale_copy(const T* in, T* out, double scale, int64_t n, cudaStream_t s);
// x = x + y
template <class T>
void launch_add_to(T* x, const T* y, int64_t n, cudaStream_t s);
template <class T>
void launch_recip(const T* in, T* out, int64_t n, cudaStream_t s);
template <class T>
void launch_fill(T* out, double v, int64_t n, cudaStream_t s);

// Deterministic weighted sums over one level-0 vector:
//   mode 0: out[c] = sum_w a_c * b_c   (stag_inner_prod / cc_inner_prod weights)
//   mode 1: out[c] = sum_w a_c         (sum_umac_press weights)
//   mode 2: out[c] = max |a_c - b_c|   (multifab_norm_inf_c)
// components c = 0..dm-1 are faces, c = dm the cell field (weight 1).
// a entries may be nullptr to skip a component.  out[4] and out[5] receive
// the combined Hessenberg entry and Stokes norm (see k_reduce).
// ninst > 1: a 2D batch (D.nz = ninst instances), one reduction per
// instance into out + 8 * b, nblocks blocks each (partials: ninst * nblocks
// * (dm + 1) doubles; counter: ninst entries, zero on entry and on exit).
template <class T>
void launch_reduce(const Dims& D, int mode, const T* const a[4], const T* const b[4], const double wseam[3], double pw,
                   double* partials, unsigned* counter, double* out, int nblocks, cudaStream_t s, int ninst = 1);

int reduce_blocks(int64_t n);
// raise a kernel's dynamic shared-memory limit to at least `bytes` on the
// current device, once per (device, kernel); safe from several host threads
cudaError_t raise_smem_limit(const void* kernel, size_t bytes);

// bounds-check builds (-DLMM_BOUNDS_CHECK, stencil.cuh): register / forget a
// device allocation that loads may touch; bc_status reads and clears every
// translation unit's record (LMM_ERR_BOUNDS when a load fell outside).  In
// other builds bc_add and bc_remove do nothing and bc_status is LMM_OK.
void bc_add(const void* p, size_t bytes);
void bc_remove(const void* p);
int bc_status();
// the caller's arrays of one entry point that reads them in place
struct BcScope {
    const void* p[8] = {};
    BcScope(std::initializer_list<const void*> ptrs, size_t bytes) {
        int k = 0;
        for (const void* q : ptrs)
            if (k < 8) {
                p[k++] = q;
                bc_add(q, bytes);
            }
    }
    ~BcScope() {
        for (const void* q : p) bc_remove(q);
    }
    BcScope(const BcScope&) = delete;
    BcScope& operator=(const BcScope&) = delete;
};
// one kernel launch issued (counted by check_launch after every launch site)
void count_launch();
int64_t launches_total();

// ---- block-shape autotuner (autotune.cu; the timing is solver.cu's) ----
// Kernels whose launch geometry it picks per (precision, visc_type, grid).
// TK_APPLY_MATRIX: the level-0 apply_matrix, keyed by its input width
// (8: FP64 x, 4: the FP32 preconditioned vector of the mixed method)
enum TuneKernel { TK_GS_COLOUR = 0, TK_APPLYOP = 1, TK_PROLONG = 2, TK_RESIDUAL = 3, TK_APPLY_MATRIX = 4, TK_N = 5 };
struct Shape {
    int bx = 0, by = 0;  // 0 x 0: the default geometry (geom3)
};
// the chosen shape, {0, 0} when the kernel was not tuned for this grid
Shape tuned_shape(int kernel, int wbytes, int visc, const Dims& D);
bool is_tuned(int kernel, int wbytes, int visc, const Dims& D);
void set_tuned_shape(int kernel, int wbytes, int visc, const Dims& D, Shape s, double ms_default, double ms_best);
// a candidate forced on this thread's launches while the autotuner times it
void force_shape(Shape s);
Shape forced_shape();

}  // namespace lmm
