// stochastic.cu - the right-hand side of the overdamped integrator's Stokes
// solve: the divergence of a symmetric stochastic stress (periodic, one
// random stage), generated on the GPU without storing the random fields.
//
// Restates src_common/stochastic_m_fluxdiv.f90 for periodic boxes:
//   diagonal stress components at cells, N(0,1) with variance 2 (:573);
//   one N(0,1) value per edge (2D: node) shared by both off-diagonal
//   components (symmetric form, :586-600);
//   every value times sqrt(2 kT / (dV dt)) (:135) and sqrt(eta) at its own
//   location (mult_by_sqrt_eta_3d, :306-359);
//   the face divergence of stoch_m_force_2d/_3d (:450-551), term by term in
//   the reference's order.
// The random numbers come from a counter-based generator: value q of field
// f (cells: f = component; edges: f = dm + edge type) is a function of
// (seed, f, q) only, so every face that needs it recomputes the same value.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "../../include/lmm_stokes.h"
#include "kernels.h"

namespace lmm {
namespace {

__host__ __device__ __forceinline__ uint64_t smix(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// standard normal number q of field f (Box-Muller on two 53-bit uniforms)
__device__ __forceinline__ double gauss(uint64_t seed, int f, int64_t q) {
    const uint64_t h1 = smix(seed ^ smix(((uint64_t)f << 48) ^ (uint64_t)q));
    const uint64_t h2 = smix(h1);
    const double u1 = ((double)(h1 >> 11) + 1.0) * (1.0 / 9007199254740992.0);
    const double u2 = (double)(h2 >> 11) * (1.0 / 9007199254740992.0);
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

struct StochArgs {
    Dims D;
    uint64_t seed;
    double var;        // sqrt(2 kT / (dV dt))
    double dxinv;
    const double* eta;       // cells
    const double* eta_ed[3]; // 2D: [0] nodes; 3D: xy, xz, yz edges
    double* b[3];
};

__device__ __forceinline__ int idx3(const Dims& D, int i, int j, int k) {
    i = wrapi(i, D.nx);
    j = wrapi(j, D.ny);
    k = (D.dm == 3) ? wrapi(k, D.nz) : 0;
    return i + D.nx * (j + D.ny * k);
}

// stress value at cell q, diagonal component c
__device__ __forceinline__ double scc(const StochArgs& A, int c, int q) {
    return (sqrt(2.0) * gauss(A.seed, c, q)) * A.var * sqrt(A.eta[q]);
}
// stress value at edge (node) q of type e
__device__ __forceinline__ double sed(const StochArgs& A, int e, int q) {
    return gauss(A.seed, A.D.dm + e, q) * A.var * sqrt(A.eta_ed[e][q]);
}

__global__ void k_stoch_div(StochArgs A) {
    const Pos p = pos3(A.D.nx, A.D.ny);
    if (!p.ok) return;
    const int i = p.i, j = p.j, k = p.k;
    const Dims& D = A.D;
    const int s = idx3(D, i, j, k);
    const double dxinv = A.dxinv;
    if (D.dm == 2) {
        // x faces: (cc1(i) - cc1(i-1)) + (nd(j+1) - nd(j)); y faces likewise
        A.b[0][s] = 0.0 + (scc(A, 0, s) - scc(A, 0, idx3(D, i - 1, j, 0))) * dxinv +
                    (sed(A, 0, idx3(D, i, j + 1, 0)) - sed(A, 0, s)) * dxinv;
        A.b[1][s] = 0.0 + (sed(A, 0, idx3(D, i + 1, j, 0)) - sed(A, 0, s)) * dxinv +
                    (scc(A, 1, s) - scc(A, 1, idx3(D, i, j - 1, 0))) * dxinv;
        return;
    }
    A.b[0][s] = 0.0 + (scc(A, 0, s) - scc(A, 0, idx3(D, i - 1, j, k))) * dxinv +
                (sed(A, 0, idx3(D, i, j + 1, k)) - sed(A, 0, s)) * dxinv +
                (sed(A, 1, idx3(D, i, j, k + 1)) - sed(A, 1, s)) * dxinv;
    A.b[1][s] = 0.0 + (sed(A, 0, idx3(D, i + 1, j, k)) - sed(A, 0, s)) * dxinv +
                (scc(A, 1, s) - scc(A, 1, idx3(D, i, j - 1, k))) * dxinv +
                (sed(A, 2, idx3(D, i, j, k + 1)) - sed(A, 2, s)) * dxinv;
    A.b[2][s] = 0.0 + (sed(A, 1, idx3(D, i + 1, j, k)) - sed(A, 1, s)) * dxinv +
                (sed(A, 2, idx3(D, i, j + 1, k)) - sed(A, 2, s)) * dxinv +
                (scc(A, 2, s) - scc(A, 2, idx3(D, i, j, k - 1))) * dxinv;
}

}  // namespace
}  // namespace lmm

extern "C" int lmm_stochastic_rhs(int dm, const int n[3], double dx, double dt, double kT, const double* eta_cc,
                                  const double* const eta_ed[3], unsigned long long seed, double* const b_u[3], void* stream) {
    using namespace lmm;
    if ((dm != 2 && dm != 3) || !n || !(dx > 0.0) || !(dt > 0.0) || !(kT >= 0.0) || !eta_cc || !eta_ed || !b_u)
        return LMM_ERR_INVALID;
    StochArgs A;
    A.D.dm = dm;
    A.D.nx = n[0];
    A.D.ny = n[1];
    A.D.nz = dm == 3 ? n[2] : 1;
    A.D.wall = A.D.slip_lo = A.D.slip_hi = 0;
    if (A.D.nx < 1 || A.D.ny < 1 || A.D.nz < 1) return LMM_ERR_INVALID;
    double dV = 1.0;
    for (int d = 0; d < dm; ++d) dV *= dx;
    A.seed = seed;
    A.var = std::sqrt(2.0 * kT / (dV * dt));
    A.dxinv = 1.0 / dx;
    A.eta = eta_cc;
    for (int e = 0; e < 3; ++e) {
        A.eta_ed[e] = (e < (dm == 2 ? 1 : 3)) ? eta_ed[e] : nullptr;
        A.b[e] = (e < dm) ? b_u[e] : nullptr;
        if ((e < dm && !A.b[e]) || (e < (dm == 2 ? 1 : 3) && !A.eta_ed[e])) return LMM_ERR_INVALID;
    }
    int bx = A.D.nx < 64 ? A.D.nx : 64, by = 256 / bx;
    if (by > A.D.ny) by = A.D.ny;
    dim3 block(bx, by), grid((A.D.nx + bx - 1) / bx, (A.D.ny + by - 1) / by, A.D.nz);
    k_stoch_div<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(A);
    if (cudaGetLastError() != cudaSuccess) return LMM_ERR_CUDA;
    count_launch();
    return LMM_OK;
}

// the bounds-check table and record of this translation unit (empty
// unless built with -DLMM_BOUNDS_CHECK)
LMM_BC_UNIT(stochastic)
