// fv_adj_b.cu -- explicit instantiations of the adjoint (VJP) launch code for dim 3 / 2 species, dim 3 / 5 species.
#include "fv_launch.cuh"

namespace abl {
template void run_vjp<3, 2>(abl_fv*, const double*, const double*, double*, cudaStream_t);
template void run_vjp<3, 5>(abl_fv*, const double*, const double*, double*, cudaStream_t);
}  // namespace abl
