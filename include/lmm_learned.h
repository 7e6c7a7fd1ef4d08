/* lmm_learned.h - C ABI of the learned preconditioner stage of liblmmstokes
 * (BF16 tcgen05 tensor-core kernels).  The stage has no counterpart in the
 * reference, whose preconditioner is purely multigrid
 * (src_gmres/apply_precon.f90). */
#ifndef LMM_LEARNED_H
#define LMM_LEARNED_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The network of the learned stage: a 3-level periodic convolutional
 * encoder-decoder (3x3x3 kernels, 16/32/64 channels, BF16 weights and
 * activations, FP32 accumulation), E0a E0b | pool | E1a E1b | pool | E2a E2b
 * | up D1a (+E1b) D1b | up D0a (+E0b) D0b | Out.  Inputs: BF16 [batch][nz]
 * [ny][nx][8] (5 channels used); output FP32 [batch][nz][ny][nx][4].
 * Parameters: per layer the weights [Cout][27][Cin] then the biases [Cout],
 * in layer order, FP32 (lmm_net_num_params floats). */
typedef struct lmm_net lmm_net;

int lmm_net_create(int nx, int ny, int nz, int batch, unsigned long long seed, lmm_net** out);
int lmm_net_destroy(lmm_net* net);
int64_t lmm_net_num_params(lmm_net* net);
/* the network's CUDA stream */
int lmm_net_stream(lmm_net* net, void** stream);
/* copy the FP32 parameters to (set = 0) or from (set = 1) host memory */
int lmm_net_params(lmm_net* net, float* host, int set);
/* Weights on disk, one flat little-endian file:
 *   offset 0        8 bytes     magic "LMMNET01"
 *          8        uint32      format version (1)
 *          12       uint32      layer count L (11)
 *          16       L x 2 uint32  (Cin, Cout) of each layer, in layer order
 *          16 + 8L  uint64      parameter count P (lmm_net_num_params)
 *          24 + 8L  uint64      FNV-1a 64-bit hash of the 4P parameter bytes
 *          32 + 8L  P x float32 the parameters, in lmm_net_params order
 * lmm_net_save writes the network's parameters; lmm_net_load checks the
 * magic, version, layer table, count, file size and hash and then sets
 * them (any mismatch: LMM_ERR_INVALID, lmm_strerror says which).  The file
 * does not depend on the grid or batch the network was created for. */
int lmm_net_save(lmm_net* net, const char* path);
int lmm_net_load(lmm_net* net, const char* path);
/* y (device, may be NULL) = network(x), x device BF16 */
int lmm_net_forward(lmm_net* net, const void* x, float* y);
/* gradients of sum(gy * network(x)) with respect to every parameter
 * (gy device FP32 [M][4]) copied to grads_host (lmm_net_num_params floats) */
int lmm_net_gradients(lmm_net* net, const void* x, const float* gy, float* grads_host);
/* one Adam step on the mean squared error against target (device FP32
 * [M][4]); *loss_host (may be NULL) = the loss before the step */
int lmm_net_train_step(lmm_net* net, const void* x, const float* target, float lr, float* loss_host);

/* ---- the stage inside the solver (include lmm_stokes.h for lmm_handle) ----
 * A 3D solver handle can carry a network on its own grid (batch 1 is
 * enough).  With knobs.learned_stage = 1, FGMRES with the FP32
 * preconditioner adds, after every V-cycle column, a second column: the
 * network's correction of the residual that V-cycle application leaves,
 * so the least-squares minimisation runs over both (a correction whose
 * image adds nothing to the basis is dropped).  learned_stage = 3 adds the
 * correction to the V-cycle's direction instead, when it lowers the
 * residual.  set_net(h, NULL) detaches. */
struct lmm_handle;
int lmm_stokes_set_net(struct lmm_handle* h, lmm_net* net);
/* count training pairs from the handle's loaded coefficients (see
 * lmm_op_load_coeffs): inputs into x_out (BF16 [count][n][8]) and targets
 * into t_out (FP32 [count][n][4]), device pointers.  Needs set_net first. */
int lmm_learned_make_pairs(struct lmm_handle* h, unsigned long long seed, int count, void* x_out, float* t_out);
/* ratios[0] = |r1| / |r0| after the preconditioner, ratios[1] = |r1 - A c| / |r1|
 * after the network's correction, on one fresh random pair */
int lmm_learned_eval(struct lmm_handle* h, unsigned long long seed, double* ratios);
/* corrections kept / computed in the last solve (learned_stage 1: network
 * columns kept in the basis / computed; 3: corrections accepted / tried) */
int lmm_learned_stats(struct lmm_handle* h, int* accepted, int* tried);

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
