// fv_adj_a.cu -- explicit instantiations of the adjoint (VJP) launch code for dim 1 / 0 species, dim 2 / 0 species, dim 2 / 2 species, dim 3 / 0 species.
#include "fv_launch.cuh"

namespace abl {
template void run_vjp<1, 0>(abl_fv*, const double*, const double*, double*, cudaStream_t);
template void run_vjp<2, 0>(abl_fv*, const double*, const double*, double*, cudaStream_t);
template void run_vjp<2, 2>(abl_fv*, const double*, const double*, double*, cudaStream_t);
template void run_vjp<2, 3>(abl_fv*, const double*, const double*, double*, cudaStream_t);
template void run_vjp<3, 0>(abl_fv*, const double*, const double*, double*, cudaStream_t);
}  // namespace abl
