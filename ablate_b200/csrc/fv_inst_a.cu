// fv_inst_a.cu -- explicit instantiations of the launch code for dim 1 / 0 species, dim 2 / 0 species, dim 2 / 2 species
// (one translation unit per group so nvcc compiles the kernels in parallel).
#include "fv_launch.cuh"

namespace abl {
template void run_rhs<1, 0>(abl_fv*, const double*, double*, int, int, cudaStream_t);
template void run_aux<1, 0>(abl_fv*, const double*, cudaStream_t);
template void run_jvp<1, 0>(abl_fv*, const double*, const double*, double*, double*, cudaStream_t);
template void run_rhs<2, 0>(abl_fv*, const double*, double*, int, int, cudaStream_t);
template void run_aux<2, 0>(abl_fv*, const double*, cudaStream_t);
template void run_jvp<2, 0>(abl_fv*, const double*, const double*, double*, double*, cudaStream_t);
template void run_rhs<2, 2>(abl_fv*, const double*, double*, int, int, cudaStream_t);
template void run_aux<2, 2>(abl_fv*, const double*, cudaStream_t);
template void run_jvp<2, 2>(abl_fv*, const double*, const double*, double*, double*, cudaStream_t);
template void run_rhs<2, 3>(abl_fv*, const double*, double*, int, int, cudaStream_t);
template void run_aux<2, 3>(abl_fv*, const double*, cudaStream_t);
template void run_jvp<2, 3>(abl_fv*, const double*, const double*, double*, double*, cudaStream_t);
}  // namespace abl
