// walls_fp64.cu - FP64 instantiation of the wall-bounded multigrid kernels
// (built with -fmad=false, like kernels_fp64.cu).
#include "walls.cuh"

namespace lmm {
LMM_INSTANTIATE_WALLS(double)
}  // namespace lmm
