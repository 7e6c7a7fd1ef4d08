// learned.cuh - launchers of the Stokes-side kernels of the learned stage
// (learned.cu) and the network entry points the solver uses (net.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/lmm_learned.h"
#include "stencil.cuh"

namespace lmm {

void launch_randn(double* out, int64_t n, uint64_t seed, cudaStream_t s);
// out = a + alpha * b
void launch_lin(double* out, const double* a, double alpha, const double* b, int64_t n, cudaStream_t s);
// network input rows (8 BF16 channels per cell) from a 3D Stokes residual r;
// sums[0..2] = per-component squared sums of the velocity residual
void launch_features(const Dims& D, const double* r, const double* beta, const double* sums, double dx, __nv_bfloat16* x,
                     cudaStream_t s);
// training target rows (4 FP32 per cell) from an error e; psum[3] = sum of e_p
void launch_target(const Dims& D, const double* e, const double* beta, const double* sums, const double* psum, double dx, float* t,
                   cudaStream_t s);
// Stokes correction c from the network output y
void launch_correction(const Dims& D, const float* y, const double* beta, const double* sums, double dx, double* c, cudaStream_t s);
// w += Ac when *n2 < factor * *n1, else c = 0; uses[0] counts acceptances, uses[1] tries
void launch_accept(double* c, double* w, const double* Ac, const double* n1, const double* n2, double factor, int* uses, int64_t len,
                   cudaStream_t s);

namespace nn {
// the network's input rows / output rows and a forward pass on stream s
__nv_bfloat16* net_input(lmm_net* net);
float* net_output(lmm_net* net);
int net_forward_on(lmm_net* net, cudaStream_t s);
void net_dims(lmm_net* net, int* nx, int* ny, int* nz, int* batch);
}  // namespace nn

}  // namespace lmm
