// fv_inst_h.cu -- the tangent (JVP) of the 64-species instance in 3D: run-time loops over the state
// components (ABL_CAPACITY_TU), the NASA-7 mixture loops unrolled (ABL_CAPACITY_UNROLL_MIXTURE).
#define ABL_CAPACITY_TU
#define ABL_CAPACITY_UNROLL_MIXTURE
#include "fv_launch.cuh"

namespace abl {
template void run_jvp<3, 64>(abl_fv*, const double*, const double*, double*, double*, cudaStream_t);
}  // namespace abl
