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

/* One 3x3x3 periodic convolution (implicit GEMM on the tensor cores).
 * x: BF16 channels-last [B][nz'][ny'][nx'][Cin] (Cin % 8 == 0), on the
 * output grid, or on the half grid when up = 1 (nearest upsampling is read
 * through the gather).  w: BF16 [round16(Cout)][27][Cin] GEMM rows, tap
 * t = (dz+1)*9 + (dy+1)*3 + (dx+1).  Output channels 0..Cout-1 of rows of
 * Cs channels: out = act(conv + bias + skip) [* (mask > 0)], act = ReLU if
 * relu != 0; out (BF16, Cs % 8 == 0) and/or out32 (FP32).  bias, skip, mask
 * may be NULL. */
int lmm_nn_conv3d(const void* x, const void* w, const float* bias, const void* skip, const void* mask, void* out,
                  float* out32, int B, int nx, int ny, int nz, int up, int Cin, int Cout, int Cs, int relu,
                  int* err_dev, void* stream);

/* Weight gradient of lmm_nn_conv3d: dw[Cout][27][Cin] (FP32) += sum over
 * voxels of g[v][co] * x_tap(v)[ci], g BF16 [B*nx*ny*nz][Cg], Cg % 8 == 0. */
int lmm_nn_conv3d_wgrad(const void* x, const void* g, float* dw, int B, int nx, int ny, int nz, int up, int Cin, int Cg,
                        int Cout, int* err_dev, void* stream);

/* FP32 master weights [Cout][27][Cin] -> BF16 forward rows wf
 * [round16(Cout)][27*Cin] and (wt != NULL) data-gradient rows
 * wt[round16(Cin)][27*round8(Cout)] with wt[ci][s][co] = w[co][26-s][ci]. */
int lmm_nn_pack_weights(const float* w, void* wf, void* wt, int Cout, int Cin, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LMM_LEARNED_H */
