// fv_adj_c.cu -- explicit instantiations of the adjoint (VJP) launch code for dim 3 / 9 species.
#include "fv_launch.cuh"

namespace abl {
template void run_vjp<3, 9>(abl_fv*, const double*, const double*, double*, cudaStream_t);
}  // namespace abl
