// fv_inst_cap.cu -- the species-capacity instances of the launch code: kMaxSpecies species in 1D, 2D
// and 3D, compiled with run-time loops over the state components (ABL_CAPACITY_TU), for the RHS and the
// aux update. A species count without an instance of its own runs in the smallest instance that holds
// it, its species placed after zero-state padding species (the species padding in fv.cu).
#define ABL_CAPACITY_TU
#include "fv_launch.cuh"

namespace abl {
#define ABL_CAPACITY_INSTANCE(DIM, NS)                                                          \
    template void run_rhs<DIM, NS>(abl_fv*, const double*, double*, int, int, cudaStream_t); \
    template void run_aux<DIM, NS>(abl_fv*, const double*, cudaStream_t);
ABL_CAPACITY_INSTANCE(1, kMaxSpecies)
ABL_CAPACITY_INSTANCE(2, kMaxSpecies)
ABL_CAPACITY_INSTANCE(3, kMaxSpecies)
#undef ABL_CAPACITY_INSTANCE
}  // namespace abl
