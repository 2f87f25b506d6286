// fv_inst_d.cu -- explicit instantiations of the launch code for dim 3 / 9 species
// (one translation unit per group so nvcc compiles the kernels in parallel).
#include "fv_launch.cuh"

namespace abl {
template void run_rhs<3, 9>(abl_fv*, const double*, double*, int, int, cudaStream_t);
template void run_aux<3, 9>(abl_fv*, const double*, cudaStream_t);
template void run_jvp<3, 9>(abl_fv*, const double*, const double*, double*, double*, cudaStream_t);
}  // namespace abl
