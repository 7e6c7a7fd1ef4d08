// kernels_fp32.cu - FP32 instantiation of the staggered Stokes kernels, used
// by the mixed-precision preconditioner inside FP64 flexible GMRES.  Built
// with FMA contraction enabled (the FP32 V-cycle needs no bit parity).
#include "kernels.cuh"
#include "tail.cuh"

namespace lmm {
LMM_INSTANTIATE(float)
LMM_INSTANTIATE_TAIL(float)
}  // namespace lmm

// the bounds-check table and record of this translation unit (empty
// unless built with -DLMM_BOUNDS_CHECK)
LMM_BC_UNIT(kernels_fp32)
