// fv_inst_f.cu -- explicit instantiations of the launch code for dim 1 / 16 species and dim 2 / 16
// species (RHS, aux update, tangent), loops over the state components unrolled.
#include "fv_launch.cuh"

namespace abl {
template void run_rhs<1, 16>(abl_fv*, const double*, double*, int, int, cudaStream_t);
template void run_aux<1, 16>(abl_fv*, const double*, cudaStream_t);
template void run_jvp<1, 16>(abl_fv*, const double*, const double*, double*, double*, cudaStream_t);
template void run_rhs<2, 16>(abl_fv*, const double*, double*, int, int, cudaStream_t);
template void run_aux<2, 16>(abl_fv*, const double*, cudaStream_t);
template void run_jvp<2, 16>(abl_fv*, const double*, const double*, double*, double*, cudaStream_t);
}  // namespace abl
