// walls_fp32.cu - FP32 instantiation of the wall-bounded multigrid kernels
// (the mixed-precision preconditioner's V-cycle on grids with walls).
#include "walls.cuh"

namespace lmm {
LMM_INSTANTIATE_WALLS(float)
}  // namespace lmm

// the bounds-check table and record of this translation unit (empty
// unless built with -DLMM_BOUNDS_CHECK)
LMM_BC_UNIT(walls_fp32)
