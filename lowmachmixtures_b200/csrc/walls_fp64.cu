// walls_fp64.cu - FP64 instantiation of the wall-bounded multigrid kernels
// (built with -fmad=false, like kernels_fp64.cu).
#include "walls.cuh"

namespace lmm {
LMM_INSTANTIATE_WALLS(double)
}  // namespace lmm

// the bounds-check table and record of this translation unit (empty
// unless built with -DLMM_BOUNDS_CHECK)
LMM_BC_UNIT(walls_fp64)
