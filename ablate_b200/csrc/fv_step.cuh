// fv_step.cuh -- the steps around the RHS in a time step, on the device:
//   k_fill_ghosts        ghost-cell boundary values before every RHS (Ghost / EssentialGhost update
//                        functions applied by DMPlexInsertBoundaryValuesRiemann: src/solver/solver.cpp:
//                        50-102, src/finiteVolume/boundaryConditions/ghost.cpp:17-28, essentialGhost.cpp:5-22)
//   k_cfl_dt             the CFL time step over the owned cells (NavierStokesTransport::ComputeCflTimeStep,
//                        src/finiteVolume/processes/navierStokesTransport.cpp:209-278; the minimum over
//                        ranks is the caller's MPI_Allreduce / NCCL all-reduce, src/solver/timeStepper.cpp:394-409)
//   k_normalize_species  mass-fraction clipping after a step (SpeciesTransport::NormalizeSpecies,
//                        src/finiteVolume/processes/speciesTransport.cpp:343-403)
//   k_rk_stage           one Shu-Osher stage of the three-stage SSP Runge-Kutta scheme on the owned rows
//   k_fill_ghosts_vjp    transpose of the ghost fill (adjoint of a march through time steps)
//   k_bc_value_reduce    adjoint of the condition table values, summed per condition
//   k_pressure_functional  J = sum_c w_c p(U_c) over a set of cells and its gradient dJ/dU
#pragma once
#include "fv_adjoint.cuh"
#include "fv_kernels.cuh"

namespace abl {

// boundary ghost g: interior neighbour, unit normal pointing out of the domain (interior -> ghost),
// condition index into the table
struct GhostBC {
    int n;
    const int* cell;
    const int* nbr;
    const double* normal;  // [n][3]
    const int* bc;
    const abl_bc* table;
};

// LIN = 1 is the tangent of the fill: the ghost's derivative with respect to its interior neighbour
// (a Dirichlet value is a constant, so a plain Dirichlet ghost gets 0 and an enforced one -du).
template <int DIM, int NS, int LIN = 0>
__global__ void __launch_bounds__(256) k_fill_ghosts(GhostBC G, double* __restrict__ U) {
    using D = Dims<DIM, NS>;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= G.n) return;
    const int g = G.cell[j], i = G.nbr[j];
    const abl_bc bc = G.table[G.bc[j]];
    double u[D::NC];
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC; k++) u[k] = U[(size_t)i * D::NC + k];
    switch (bc.kind) {
        case ABL_BC_DIRICHLET:
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NC; k++) u[k] = bc.enforce_at_face ? (LIN ? 0.0 : 2.0 * bc.value[k]) - u[k] : (LIN ? 0.0 : bc.value[k]);
            break;
        case ABL_BC_SLIP_WALL: {
            // reflect the normal momentum: (rho u)_g = (rho u)_i - 2 ((rho u)_i . n) n
            double mn = 0;
#pragma unroll
            for (int d = 0; d < DIM; d++) mn += u[2 + d] * G.normal[3 * (size_t)j + d];
#pragma unroll
            for (int d = 0; d < DIM; d++) u[2 + d] -= 2.0 * mn * G.normal[3 * (size_t)j + d];
            break;
        }
        case ABL_BC_NOSLIP_WALL:
#pragma unroll
            for (int d = 0; d < DIM; d++) u[2 + d] = -u[2 + d];
            break;
        default:  // ABL_BC_OUTFLOW: zero gradient
            break;
    }
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC; k++) U[(size_t)g * D::NC + k] = u[k];
}

// positive doubles order like their bit patterns: an integer atomicMin gives the exact minimum in
// any order
template <int DIM, int NS>
__global__ void __launch_bounds__(256) k_cfl_dt(DevMesh M, Phys P, const double* __restrict__ U, const double* __restrict__ rmin, double cfl,
                                                unsigned long long* __restrict__ dt_bits, int* status) {
    using D = Dims<DIM, NS>;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double dt = DBL_MAX;
    bool ok = true;
    if (c < M.n_cells && M.kind[c] == ABL_CELL_OWNED) {
        double u[D::NC];
        load_state<DIM, NS>(U, c, u);
        // T from the EOS with a 300 K guess, then the speed of sound at T
        const Decoded<double> dd = decode<DIM, NS>(P, NS, u, 300.0, &ok);
        double velSum = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) velSum += fabs(u[2 + d]) / u[0];
        dt = cfl * (2.0 * rmin[c]) / (dd.a / P.alpha + velSum);
        if (!(dt > 0.0)) dt = DBL_MAX;  // a NaN state does not set the step; it shows in the status word
        if (!isfinite(dd.a)) ok = false;
    }
    // warp then block minimum, one atomic per block
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dt = fmin(dt, __shfl_xor_sync(0xffffffffu, dt, o));
    __shared__ double wmin[8];
    if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = dt;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = wmin[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmin(m, wmin[w]);
        atomicMin(dt_bits, (unsigned long long)__double_as_longlong(m));
    }
    if (!ok) atomicOr(status, kStatusEos);
}

template <int DIM, int NS>
__global__ void __launch_bounds__(256) k_normalize_species(DevMesh M, double* __restrict__ U) {
    using D = Dims<DIM, NS>;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (NS == 0 || c >= M.n_cells || M.kind[c] != ABL_CELL_OWNED) return;
    double* u = U + (size_t)c * D::NC;
    const double density = u[0];
    double* rY = u + D::NE;
    double yiSum = 0.0;
ABL_UNROLL_SPECIES
    for (int s = 0; s < NS - 1; s++) {
        double yi = rY[s] / density;
        yi = pmax(0.0, yi);
        yi = pmin(1.0, yi);
        yiSum += yi;
        rY[s] = yi * density;
    }
    if (yiSum > 1.0) {
ABL_UNROLL_SPECIES
        for (int s = 0; s < NS; s++) {
            double yi = rY[s] / density;
            yi /= yiSum;
            rY[s] = density * yi;
        }
        rY[NS - 1] = 0.0;
    } else if (NS > 0) {
        rY[NS - 1] = density * (1.0 - yiSum);
    }
}

// Uout = a U0 + b (Us + dt F) on the owned rows (other rows of Uout are left as they are). Uout may be
// U0 or Us: each thread reads its element before writing it.
template <int UNUSED = 0>
__global__ void __launch_bounds__(256) k_rk_stage(const uint8_t* __restrict__ kind, int nc, int n_cells, double a, const double* U0, double b,
                                                  const double* Us, double dt, const double* __restrict__ F, double* Uout) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= (int64_t)n_cells * nc) return;
    if (kind[e / nc] != ABL_CELL_OWNED) return;
    const double s = Us[e] + dt * F[e];
    Uout[e] = a == 0.0 ? b * s : a * U0[e] + b * s;
}

// k_rk_stage with the step read from the device: dt = the double whose bits the CFL reduction left in
// *dt_bits. Thread 0 of block 0 adds dt to *time when `time` is not null.
template <int UNUSED = 0>
__global__ void __launch_bounds__(256) k_rk_stage_dev(const uint8_t* __restrict__ kind, int nc, int n_cells, double a, const double* U0, double b,
                                                      const double* Us, const unsigned long long* __restrict__ dt_bits, const double* __restrict__ F,
                                                      double* Uout, double* time) {
    const double dt = __longlong_as_double((long long)*dt_bits);
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (time && e == 0) *time += dt;
    if (e >= (int64_t)n_cells * nc) return;
    if (kind[e / nc] != ABL_CELL_OWNED) return;
    const double s = Us[e] + dt * F[e];
    Uout[e] = a == 0.0 ? b * s : a * U0[e] + b * s;
}

// Ghosts grouped by their interior neighbour: segment s owns ghosts seg_ghost[seg_ptr[s] .. seg_ptr[s+1])
// (ascending), all next to cell seg_nbr[s]. One thread per segment keeps the sums in a fixed order.
struct GhostSegments {
    int n;
    const int* ptr;
    const int* nbr;
    const int* ghost;
};

// Transpose of k_fill_ghosts on adjoint rows: the ghost row's adjoint moves to its interior neighbour
// through (dG/du)^T, the part owed to the condition's value goes to vbar[j][k] (per ghost, summed per
// condition by k_bc_value_reduce), and the ghost row is cleared (the fill overwrites the ghost's old
// value, which therefore has no influence).
template <int DIM, int NS>
__global__ void __launch_bounds__(256) k_fill_ghosts_vjp(GhostBC G, GhostSegments S, double* __restrict__ Ub, double* __restrict__ vbar) {
    using D = Dims<DIM, NS>;
    const int sidx = blockIdx.x * blockDim.x + threadIdx.x;
    if (sidx >= S.n) return;
    const int i = S.nbr[sidx];
    double acc[D::NC];
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC; k++) acc[k] = 0.0;
    for (int q = S.ptr[sidx]; q < S.ptr[sidx + 1]; q++) {
        const int j = S.ghost[q];
        const int g = G.cell[j];
        const abl_bc bc = G.table[G.bc[j]];
        double lg[D::NC];
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC; k++) {
            lg[k] = Ub[(size_t)g * D::NC + k];
            Ub[(size_t)g * D::NC + k] = 0.0;
        }
        double vb[D::NC];
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC; k++) vb[k] = 0.0;
        switch (bc.kind) {
            case ABL_BC_DIRICHLET:
ABL_UNROLL_SPECIES
                for (int k = 0; k < D::NC; k++) {
                    vb[k] = bc.enforce_at_face ? 2.0 * lg[k] : lg[k];
                    if (bc.enforce_at_face) acc[k] -= lg[k];
                }
                break;
            case ABL_BC_SLIP_WALL: {
                // (I - 2 n n^T) is symmetric
                double mn = 0;
#pragma unroll
                for (int d = 0; d < DIM; d++) mn += lg[2 + d] * G.normal[3 * (size_t)j + d];
#pragma unroll
                for (int d = 0; d < DIM; d++) lg[2 + d] -= 2.0 * mn * G.normal[3 * (size_t)j + d];
ABL_UNROLL_SPECIES
                for (int k = 0; k < D::NC; k++) acc[k] += lg[k];
                break;
            }
            case ABL_BC_NOSLIP_WALL:
ABL_UNROLL_SPECIES
                for (int k = 0; k < D::NC; k++) acc[k] += (k >= 2 && k < 2 + DIM) ? -lg[k] : lg[k];
                break;
            default:
ABL_UNROLL_SPECIES
                for (int k = 0; k < D::NC; k++) acc[k] += lg[k];
                break;
        }
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC; k++) vbar[(size_t)j * D::NC + k] = vb[k];
    }
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC; k++) Ub[(size_t)i * D::NC + k] += acc[k];
}

// out[b][k] += sum over the ghosts j of condition b of vbar[j][k]; one block per condition, each thread a
// fixed stride of ghosts, then a fixed-shape tree: the same sum on every run.
template <int UNUSED = 0>
__global__ void __launch_bounds__(256) k_bc_value_reduce(int n_ghost, const int* __restrict__ bc, int nc, const double* __restrict__ vbar,
                                                         double* __restrict__ out) {
    __shared__ double red[256];
    const int b = blockIdx.x;
    for (int k = 0; k < nc; k++) {
        double acc = 0.0;
        for (int j = threadIdx.x; j < n_ghost; j += blockDim.x)
            if (bc[j] == b) acc += vbar[(size_t)j * nc + k];
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[(size_t)b * ABL_BC_MAX_COMPONENTS + k] += red[0];
        __syncthreads();
    }
}

// J = sum_j w_j p(U_{c_j}) over distinct cells c_j: per block a fixed-shape partial sum (the host adds
// the partials in block order); with Ub, Ub[c_j] += w_j dp/dU (the reverse of the EOS decode).
template <int DIM, int NS>
__global__ void __launch_bounds__(256) k_pressure_functional(Phys P, int n, const int* __restrict__ cells, const double* __restrict__ w,
                                                             const double* __restrict__ U, double* __restrict__ partial, double* __restrict__ Ub,
                                                             int* status) {
    using D = Dims<DIM, NS>;
    __shared__ double red[256];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    double val = 0.0;
    if (j < n) {
        const int c = cells[j];
        double u[D::NC];
        load_state<DIM, NS>(U, c, u);
        bool ok = true;
        const Decoded<double> dd = decode<DIM, NS>(P, NS, u, 300.0, &ok);
        val = w[j] * dd.p;
        if (!ok) atomicOr(status, kStatusEos);
        if (Ub) {
            double ub[D::NC];
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NC; k++) ub[k] = 0.0;
            decode_vjp<DIM, NS>(P, NS, u, dd, 0.0, 0.0, w[j], ub);
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NC; k++) Ub[(size_t)c * D::NC + k] += ub[k];
        }
    }
    red[threadIdx.x] = val;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

}  // namespace abl
