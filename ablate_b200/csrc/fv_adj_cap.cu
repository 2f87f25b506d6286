// fv_adj_cap.cu -- the adjoint (VJP) launch code of the species-capacity instances (16 and kMaxSpecies
// species in 1D, 2D and 3D), compiled with run-time loops over the state components (ABL_CAPACITY_TU).
#define ABL_CAPACITY_TU
#include "fv_launch.cuh"

namespace abl {
template void run_vjp<1, 16>(abl_fv*, const double*, const double*, double*, cudaStream_t);
template void run_vjp<2, 16>(abl_fv*, const double*, const double*, double*, cudaStream_t);
template void run_vjp<3, 16>(abl_fv*, const double*, const double*, double*, cudaStream_t);
template void run_vjp<1, kMaxSpecies>(abl_fv*, const double*, const double*, double*, cudaStream_t);
template void run_vjp<2, kMaxSpecies>(abl_fv*, const double*, const double*, double*, cudaStream_t);
template void run_vjp<3, kMaxSpecies>(abl_fv*, const double*, const double*, double*, cudaStream_t);
}  // namespace abl
