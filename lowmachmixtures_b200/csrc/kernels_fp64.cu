// kernels_fp64.cu - FP64 instantiation of the staggered Stokes kernels.
// Built with -fmad=false: every multiply and add is rounded separately, in
// the operand order of the reference Fortran, so face values match the
// reference arithmetic (and the CPU oracle) bit for bit.
#include "kernels.cuh"
#include "tail.cuh"

namespace lmm {
LMM_INSTANTIATE(double)
LMM_INSTANTIATE_TAIL(double)
template void launch_convert<double, float>(const double*, float*, int64_t, cudaStream_t);
template void launch_convert<float, double>(const float*, double*, int64_t, cudaStream_t);
}  // namespace lmm

// the bounds-check table and record of this translation unit (empty
// unless built with -DLMM_BOUNDS_CHECK)
LMM_BC_UNIT(kernels_fp64)
