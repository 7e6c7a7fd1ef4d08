// kernels_fp32.cu - FP32 instantiation of the staggered Stokes kernels, used
// by the mixed-precision preconditioner inside FP64 flexible GMRES.  Built
// with FMA contraction enabled (the FP32 V-cycle needs no bit parity).
#include "kernels.cuh"

namespace lmm {
LMM_INSTANTIATE(float)
}  // namespace lmm
