// fv_inst_g.cu -- the 64-species instance of the launch code in 3D (RHS and aux update), compiled with
// run-time loops over the state components (ABL_CAPACITY_TU). Counts from 17 to 64 run here padded.
#define ABL_CAPACITY_TU
#include "fv_launch.cuh"

namespace abl {
template void run_rhs<3, 64>(abl_fv*, const double*, double*, int, int, cudaStream_t);
template void run_aux<3, 64>(abl_fv*, const double*, cudaStream_t);
}  // namespace abl
