/* lmm_learned.h - C ABI of the learned preconditioner stage of liblmmstokes
 * (BF16 tcgen05 tensor-core kernels).  The stage has no counterpart in the
 * reference, whose preconditioner is purely multigrid
 * (src_gmres/apply_precon.f90). */
#ifndef LMM_LEARNED_H
#define LMM_LEARNED_H

#ifdef __cplusplus
extern "C" {
#endif

/* D[M x N] (FP32, row-major) = A[M x K] * B[N x K]^T with BF16 row-major A
 * and B on the device, FP32 accumulation in tensor memory.  K % 8 == 0,
 * N % 16 == 0, 16 <= N <= 256.  *err_dev (device int) is set to 1 if a
 * bounded wait of the kernel gave up.  Asynchronous on `stream`. */
int lmm_nn_gemm_bf16(const void* A, const void* B, float* D, int M, int N, int K, int* err_dev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LMM_LEARNED_H */
