// fv_inst_e.cu -- explicit instantiations of the launch code for dim 3 / 16 species (RHS, aux update,
// tangent), loops over the state components unrolled. Counts from 10 to 16 run here padded.
#include "fv_launch.cuh"

namespace abl {
template void run_rhs<3, 16>(abl_fv*, const double*, double*, int, int, cudaStream_t);
template void run_aux<3, 16>(abl_fv*, const double*, cudaStream_t);
template void run_jvp<3, 16>(abl_fv*, const double*, const double*, double*, double*, cudaStream_t);
}  // namespace abl
