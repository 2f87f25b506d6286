// fv_kernels.cuh -- the RHS kernels (sm_100a), templated on dimension DIM, species count NS and the
// storage/arithmetic type G of the reconstruction (double: FP64 path; float: mixed path).
//
// One RHS evaluation is two (three with a mixture EOS) passes over HBM-resident data:
//   k_aux        cells: T by the EOS (guess = previous T), u, Y -- only for the NASA-7 mixture, whose
//                temperature needs the secant iteration (CellSolver::UpdateAuxFields,
//                src/solver/cellSolver.cpp:62-135); a perfect gas recomputes T = e/cv where needed.
//   k_gradient   cells: LSQ gradient of the conserved fields + BAM limiter
//                (CellInterpolant::ComputeFieldGradients, src/finiteVolume/cellInterpolant.cpp:330-497)
//                and the unlimited LSQ gradient of the aux fields that FaceInterpolant averages onto
//                faces (src/finiteVolume/faceInterpolant.cpp:109-249).
//   k_tile_flux  one CTA per tile of owned cells: every face of the tile computes its flux
//                (projection, EOS decode, flux calculator, advection + diffusion: cellInterpolant.cpp:
//                499-639, faceInterpolant.cpp:262-448 and the process flux functions) into shared
//                memory; then every tile cell sums its faces in ascending face order and writes F once
//                (the reference's serial scatter, cellInterpolant.cpp:604-629, made a deterministic
//                per-cell gather with no atomics).
#pragma once
#include <cfloat>
#include <type_traits>

#include "fv_consts.hpp"
#include "fv_physics.cuh"

namespace abl {

enum StatusBits : int { kStatusNaN = 1, kStatusEos = 2, kStatusRiemann = 4 };

struct DevMesh {
    int dim, n_cells, n_faces, n_flux_faces;
    const int2* face_cells;
    const uint8_t* kind;
    const int* cone_ptr;
    // cone entry of a cell: x = face, y = neighbour | side << 31 | (face touches a boundary ghost) << 30
    const int2* cone;
    const double* fdx;     // [nf][2][3] face centroid - side cell centroid (cell's own frame)
    const double* ivol;    // [nc] 1 / volume
    const double* cgrad;   // [nf][2][3]
    const double* fgrad;   // [nf][2][3]
    // tiles
    int n_tiles;
    const int* tile_cell_ptr;
    const int* tile_cells;
    const int* tile_face_ptr;
    const int2* tf_cells;
    const double* tf_geo;     // [ntf][10]: area normal (3), face centroid minus each side's centroid (6), pad
    const int* tc_fptr;
    const uint16_t* tc_face;
    // adjoint: face colours per tile, tile-local slots, records of faces with a non-owned side
    const int* col_base;
    const int* col_start;
    const uint32_t* tf_slot;
    const uint16_t* tf_adj;  // per tile, the record of the k-th face in adjoint colour order
    const int* tf_nb;
    const int* face_nb;
    int n_nonowned;
    const int* nonowned;  // cells that are not owned (boundary ghosts, halos)
    const double* wsum;   // [nc][2][3] per cell: sum of its LSQ state weights (non-boundary faces), of its aux weights
    // per cone entry (cell-major, contiguous per cell): the LSQ state weight (0 across a boundary face)
    // and the aux (face-interpolant) weight packed in one 48-byte record [w0 w1 w2 a0 a1 a2], and the
    // neighbour offset x_n - x_c
    const double* cwa;
    const double* cv;
    // the same weights seen from the neighbour: per cone entry of c across face f, the neighbour's
    // LSQ state weight and aux weight for f (the transposed operators of the adjoint gather), packed
    // like cwa
    const double* cwar;
    int max_cone;
    // FP32 copies of the weights and offsets the mixed path rounds to FP32 anyway (identical results,
    // half the bytes): the packed weights (32-byte records, two floats of padding), cv and the
    // tile-face offsets
    const float* cwa32;
    const float* cv32;
    const double* tf_geo32;   // [ntf][6]: the area normal (3 doubles), then the 6 offsets as FP32 pairs (mixed path)
    // When records repeat bit for bit (a structured block), tf_geo / tf_geo32 hold one record per
    // distinct one and tf_gcls gives each tile face record its copy; likewise cwa, cv, cwar (and their
    // FP32 copies) hold one weight sequence per distinct cell cone and cone_cls gives each cell the
    // first entry of its copy. Null: one record per face / cone entry.
    const uint16_t* tf_gcls;
    const int* cone_cls;
};

// the first weight record of cell c, whose cone starts at entry beg
__device__ __forceinline__ size_t weight_base(const DevMesh& M, int c, int beg) {
    return M.cone_cls ? (size_t)__ldg(M.cone_cls + c) : (size_t)beg;
}
// the geometry record of tile face record i
__device__ __forceinline__ size_t geo_record(const DevMesh& M, int i) {
    return M.tf_gcls ? (size_t)__ldg(M.tf_gcls + i) : (size_t)i;
}

// state and aux weights of cone entry i in the reconstruction type G, from the packed record
template <int DIM, class G>
__device__ __forceinline__ void cone_weights(const double* __restrict__ p64, const float* __restrict__ p32, size_t i, G* w, G* a) {
    if constexpr (std::is_same<G, float>::value) {
        const float4 p = __ldg(reinterpret_cast<const float4*>(p32) + 2 * i);
        const float4 q = __ldg(reinterpret_cast<const float4*>(p32) + 2 * i + 1);
        const float v[6] = {p.x, p.y, p.z, p.w, q.x, q.y};
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            w[d] = v[d];
            a[d] = v[3 + d];
        }
    } else {
        const double2 p = __ldg(reinterpret_cast<const double2*>(p64) + 3 * i);
        const double2 q = __ldg(reinterpret_cast<const double2*>(p64) + 3 * i + 1);
        const double2 r = __ldg(reinterpret_cast<const double2*>(p64) + 3 * i + 2);
        const double v[6] = {p.x, p.y, q.x, q.y, r.x, r.y};
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            w[d] = G(v[d]);
            a[d] = G(v[3 + d]);
        }
    }
}

// a geometry value in the reconstruction type G: the FP32 copy for the mixed path
template <class G>
__device__ __forceinline__ G geo(const double* __restrict__ p64, const float* __restrict__ p32, size_t i) {
    if constexpr (std::is_same<G, float>::value)
        return __ldg(p32 + i);
    else
        return G(__ldg(p64 + i));
}

template <int DIM, int NS>
struct Dims {
    static constexpr int NE = 2 + DIM;       // euler components
    static constexpr int NC = NE + NS;       // conserved components per cell
    static constexpr int NA = 1 + DIM + NS;  // aux components per cell (T, u, Y)
};

// Row strides of the per-cell gradient arrays, padded to whole 16-byte vectors
template <int DIM, int NS, class G>
struct GradRows {
    static constexpr int V = 16 / sizeof(G);  // elements per 16-byte vector
    static constexpr int GS = ((Dims<DIM, NS>::NC * DIM + V - 1) / V) * V;
    static constexpr int AS = ((Dims<DIM, NS>::NA * DIM + V - 1) / V) * V;
};

// minimum resident CTAs per SM for __launch_bounds__ (register budget per thread = 65536 / (128 * n)),
// chosen by timing: on the 128^3 gas gradient FP64 4 / FP32 6, tile FP64 4 (no spills at 128
// registers) / FP32 5; with 3-5 species 3 (5 species: 2.7 % faster than 2), with more species 2 (9
// species on tetrahedra: 3 is 14 % slower); the value+tangent pairs of the tangent kernels 1
template <int NS, class G>
struct MinBlocks {
    static constexpr int grad = std::is_same<G, Dual>::value ? 1 : (NS > 5 ? 2 : (NS > 0 ? 3 : (sizeof(G) == 8 ? 4 : 6)));
    static constexpr int tile = std::is_same<G, Dual>::value ? 1 : (NS > 5 ? 2 : (NS > 2 ? 3 : (sizeof(G) == 8 ? 4 : 5)));
};

constexpr int kConeSide = int(1u << 31);
constexpr int kConeBoundary = 1 << 30;
constexpr int kConeNbr = (1 << 30) - 1;

// load n elements of a 16-byte-aligned row with vector loads
template <int N, class G>
__device__ __forceinline__ void load_row(const G* __restrict__ p, G* out) {
    if constexpr (std::is_same<G, Dual>::value) {
ABL_UNROLL_SPECIES
        for (int i = 0; i < N; i++) {
            const double2 v = __ldg(reinterpret_cast<const double2*>(p) + i);
            out[i] = Dual(v.x, v.y);
        }
    } else if constexpr (sizeof(G) == 8) {
ABL_UNROLL_SPECIES
        for (int i = 0; i < N / 2; i++) {
            const double2 v = __ldg(reinterpret_cast<const double2*>(p) + i);
            out[2 * i] = v.x;
            out[2 * i + 1] = v.y;
        }
        if constexpr (N % 2) out[N - 1] = __ldg(p + N - 1);
    } else {
ABL_UNROLL_SPECIES
        for (int i = 0; i < N / 4; i++) {
            const float4 v = __ldg(reinterpret_cast<const float4*>(p) + i);
            out[4 * i] = v.x;
            out[4 * i + 1] = v.y;
            out[4 * i + 2] = v.z;
            out[4 * i + 3] = v.w;
        }
ABL_UNROLL_SPECIES
        for (int i = (N / 4) * 4; i < N; i++) out[i] = __ldg(p + i);
    }
}

template <class G>
__device__ __forceinline__ G big_value();
template <>
__device__ __forceinline__ double big_value<double>() { return DBL_MAX; }
template <>
__device__ __forceinline__ float big_value<float>() { return FLT_MAX; }
template <>
__device__ __forceinline__ Dual big_value<Dual>() { return Dual(DBL_MAX); }

// scalar type of the state and fluxes for a gradient storage type: Dual in the tangent kernels,
// double otherwise (the mixed path keeps the state in FP64)
template <class G>
using StateOf = typename std::conditional<std::is_same<G, Dual>::value, Dual, double>::type;

template <class S, class G>
__device__ __forceinline__ S to_state(G x) {
    return static_cast<S>(x);
}
template <>
__device__ __forceinline__ double to_state<double, Dual>(Dual x) {
    return x.v;
}

// state row of cell c; a Dual state also reads the tangent row from dU
template <int DIM, int NS, class S>
__device__ __forceinline__ void load_state(const double* __restrict__ U, const double* __restrict__ dU, int c, S* u) {
    using D = Dims<DIM, NS>;
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC; k++) {
        if constexpr (std::is_same<S, Dual>::value)
            u[k] = Dual(__ldg(U + (size_t)c * D::NC + k), __ldg(dU + (size_t)c * D::NC + k));
        else
            u[k] = __ldg(U + (size_t)c * D::NC + k);
    }
}
template <int DIM, int NS>
__device__ __forceinline__ void load_state(const double* __restrict__ U, int c, double* u) {
    load_state<DIM, NS, double>(U, nullptr, c, u);
}

// aux (T, u, Y) of a perfect-gas cell from its conserved state: T = e / cv with e = E/rho - |u|^2/2
template <int DIM, int NS, class S>
__device__ __forceinline__ void aux_from_state(const Phys& P, const S* u, S* a) {
    using D = Dims<DIM, NS>;
    const S irho = rcp64(u[0]);
    S ke = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        a[1 + d] = u[2 + d] * irho;
        ke += a[1 + d] * a[1 + d];
    }
    a[0] = (u[1] * irho - 0.5 * ke) * rcp64(P.r_gas / (P.gamma - 1.0));
ABL_UNROLL_SPECIES
    for (int s = 0; s < NS; s++) a[1 + DIM + s] = u[D::NE + s] * irho;
}

// aux (T, u, Y) of one cell: from the resident aux array for the mixture EOS, recomputed from the
// conserved state for a perfect gas (UpdateAuxTemperatureField / UpdateAuxVelocityField /
// UpdateAuxMassFractionField: navierStokesTransport.cpp:534-558, speciesTransport.cpp:98-110)
template <int DIM, int NS, class S>
__device__ __forceinline__ void cell_aux(const Phys& P, const S* u, const double* __restrict__ aux, int c, S* a) {
    using D = Dims<DIM, NS>;
    if (NS > 0 && P.eos == ABL_EOS_NASA7) {
        if constexpr (std::is_same<S, Dual>::value) {
            // tangent: T from the state (its derivative by the implicit-function theorem), the resident T as guess
            bool ok = true;
            a[0] = temperature<DIM, NS>(P, NS, u, __ldg(aux + (size_t)c * D::NA), &ok);
            const S irho = rcp64(u[0]);
#pragma unroll
            for (int d = 0; d < DIM; d++) a[1 + d] = u[2 + d] * irho;
ABL_UNROLL_SPECIES
            for (int s = 0; s < NS; s++) a[1 + DIM + s] = u[D::NE + s] * irho;
        } else {
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NA; k++) a[k] = __ldg(aux + (size_t)c * D::NA + k);
        }
        return;
    }
    aux_from_state<DIM, NS>(P, u, a);
}

// Where the per-cell rows a face flux reads come from. GlobalRows: the resident arrays by cell index (the
// two-pass kernels; the tangent kernels also read dU). The fused tile kernel has a shared-memory source
// by tile-local slot (SharedRows, fv_fused.cuh). Both deliver the same values, so the flux arithmetic is
// shared and the two paths agree bit for bit.
template <int DIM, int NS, class G>
struct GlobalRows {
    using D = Dims<DIM, NS>;
    using GR = GradRows<DIM, NS, G>;
    const double* __restrict__ U;
    const double* __restrict__ dU;
    const double* __restrict__ aux;
    const G* __restrict__ grad;
    const G* __restrict__ agrad;
    template <class S>
    __device__ __forceinline__ void state(int c, S* u) const {
        load_state<DIM, NS, S>(U, dU, c, u);
    }
    __device__ __forceinline__ double temperature(int c) const { return __ldg(aux + (size_t)c * D::NA); }
    template <class S>
    __device__ __forceinline__ void aux_of(const Phys& P, const S* u, int c, S* a) const {
        cell_aux<DIM, NS>(P, u, aux, c, a);
    }
    __device__ __forceinline__ void grad_row(int c, G* g) const { load_row<D::NC * DIM, G>(grad + (size_t)c * GR::GS, g); }
    __device__ __forceinline__ void agrad_row(int c, G* g) const { load_row<D::NA * DIM, G>(agrad + (size_t)c * GR::AS, g); }
};

// ---------------------------------------------------------------------------------------------------
// cells: the listed cells only (n_list of them), or every cell when null
template <int DIM, int NS>
__global__ void __launch_bounds__(256) k_aux(DevMesh M, Phys P, const double* __restrict__ U, double* __restrict__ aux, int* status,
                                             const int* __restrict__ cells = nullptr, int n_list = 0) {
    using D = Dims<DIM, NS>;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (cells ? n_list : M.n_cells)) return;
    const int c = cells ? __ldg(cells + i) : i;
    double u[D::NC];
    load_state<DIM, NS>(U, c, u);
    double* a = aux + (size_t)c * D::NA;
    bool ok = true;
    a[0] = temperature<DIM, NS>(P, NS, u, a[0], &ok);
    const double irho = rcp64(u[0]);
#pragma unroll
    for (int d = 0; d < DIM; d++) a[1 + d] = u[2 + d] * irho;
ABL_UNROLL_SPECIES
    for (int s = 0; s < NS; s++) a[1 + DIM + s] = u[D::NE + s] * irho;
    if (!ok) atomicOr(status, kStatusEos);
}

// ---------------------------------------------------------------------------------------------------
// limiter of one field (components k0..k1-1) of cell c with gradient g (DMPlexApplyLimiter_Internal,
// cellInterpolant.cpp:282-328, and the cancel rule at :459-481)
// REC (the adjoint's forward pass) also records, per component, the applied factor (0 when the
// gradient was cancelled) and the cone entry of the minimising face (-1: none, or cancelled).
// sd, when not null, holds the cell's neighbour differences u_n - u_c per cone entry (written by the
// gradient pass; thread-interleaved) so the neighbour states are not read again.
template <int DIM, int NS, class G, int LIM, bool REC = false>
__device__ __forceinline__ void limit_field(const DevMesh& M, const Phys& P, int beg, int end, size_t wb, const double* __restrict__ U,
                                            const double* __restrict__ dU, const StateOf<G>* uc, G* g, int k0, int k1,
                                            double* rphi = nullptr, int* rist = nullptr, const G* sd = nullptr) {
    using D = Dims<DIM, NS>;
    using S = StateOf<G>;
    G phi[D::NC];
    int ist[D::NC];
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC; k++) {
        phi[k] = big_value<G>();
        ist[k] = -1;
    }
#pragma unroll 1
    for (int i = beg; i < end; i++) {
        // x_n - x_c, periodic images resolved (face offsets taken in each cell's own frame)
        G v[DIM];
#pragma unroll
        for (int d = 0; d < DIM; d++) v[d] = geo<G>(M.cv, M.cv32, 3 * (wb + (size_t)(i - beg)) + d);
        S un[D::NC];
        if (!sd) load_state<DIM, NS, S>(U, dU, M.cone[i].y & kConeNbr, un);
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC; k++) {
            if (k < k0 || k >= k1) continue;
            G denom = 0;
#pragma unroll
            for (int d = 0; d < DIM; d++) denom += g[k * DIM + d] * v[d];
            const G diff = sd ? sd[((i - beg) * D::NC + k) * blockDim.x + threadIdx.x] : G(un[k] - uc[k]);
            const G flim = G(0.5) * diff * rcp64(denom);
            if constexpr (REC) {
                const G l = limiter_k<LIM, G>(P.limiter, flim);
                if (!(phi[k] < l)) {  // pmin(phi, l) takes l
                    phi[k] = l;
                    ist[k] = i;
                }
            } else {
                phi[k] = pmin(phi[k], limiter_k<LIM, G>(P.limiter, flim));
            }
        }
    }
    if constexpr (std::is_same<G, Dual>::value) {
        if (P.jvp_frozen_limiter) {
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NC; k++) phi[k].d = 0.0;
        }
    }
    bool cancel = false;
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC; k++) {
        if (k < k0 || k >= k1) continue;
        if (phi[k] == G(0)) {
#pragma unroll
            for (int d = 0; d < DIM; d++)
                if (dabs(g[k * DIM + d]) > G(P.max_lim_grad)) cancel = true;
        }
    }
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC; k++) {
        if (k < k0 || k >= k1) continue;
        if constexpr (REC) {
            rphi[k] = cancel ? 0.0 : double(phi[k]);
            rist[k] = cancel ? -1 : ist[k];
        }
#pragma unroll
        for (int d = 0; d < DIM; d++) g[k * DIM + d] *= cancel ? G(0) : phi[k];
    }
}

// One thread per cell: one pass over the cell's faces accumulates the LSQ gradient of the conserved
// fields (non-boundary faces, cgrad weights) and of the aux fields (all faces, fgrad weights), a second
// pass applies the limiter. Cells without a conserved-state gradient (boundary ghosts, outer halo) get
// a zero row, so the flux kernel projects every cell without a branch.
template <int DIM, int NS, class G, int LIM, bool REC = false>
__global__ void __launch_bounds__(128, MinBlocks<NS, G>::grad) k_gradient(DevMesh M, Phys P, const double* __restrict__ U,
                                                                    const double* __restrict__ dU, const double* __restrict__ aux,
                                                                    G* __restrict__ grad, G* __restrict__ agrad, int do_state, int do_aux,
                                                                    int cache, G* __restrict__ graw = nullptr, double* __restrict__ rphi = nullptr,
                                                                    int* __restrict__ rist = nullptr, const int* __restrict__ cells = nullptr,
                                                                    int n_list = 0) {
    extern __shared__ __align__(16) unsigned char gsm[];
    using D = Dims<DIM, NS>;
    using GR = GradRows<DIM, NS, G>;
    using S = StateOf<G>;
    // cells: the listed cells only (n_list of them), or every cell when null
    const int ci = blockIdx.x * blockDim.x + threadIdx.x;
    if (ci >= (cells ? n_list : M.n_cells)) return;
    const int c = cells ? __ldg(cells + ci) : ci;
    const uint8_t kind = M.kind[c];
    const int beg = M.cone_ptr[c], end = M.cone_ptr[c + 1];
    const size_t wb = weight_base(M, c, beg);
    const bool state = do_state && (kind == ABL_CELL_OWNED || kind == ABL_CELL_HALO);
    const bool auxg = do_aux && kind != ABL_CELL_HALO_OUTER;
    const bool nasa = NS > 0 && P.eos == ABL_EOS_NASA7;
    S uc[D::NC], ac[D::NA];
    load_state<DIM, NS, S>(U, dU, c, uc);
    if (auxg) cell_aux<DIM, NS>(P, uc, aux, c, ac);
    G g[D::NC * DIM], ga[D::NA * DIM];
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC * DIM; k++) g[k] = G(0);
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NA * DIM; k++) ga[k] = G(0);
    // neighbour differences kept for the limiter when the block has shared memory for them
    G* sd = (cache && state && P.limiter != ABL_LIMITER_NONE && end - beg <= M.max_cone) ? reinterpret_cast<G*>(gsm) : nullptr;
    if (state || auxg) {
#pragma unroll 1
        for (int i = beg; i < end; i++) {
            const int2 ce = M.cone[i];
            const int n = ce.y & kConeNbr;
            S un[D::NC];
            if (state || !nasa || std::is_same<S, Dual>::value) load_state<DIM, NS, S>(U, dU, n, un);
            if (sd) {
ABL_UNROLL_SPECIES
                for (int k = 0; k < D::NC; k++) sd[((i - beg) * D::NC + k) * blockDim.x + threadIdx.x] = G(un[k] - uc[k]);
            }
            G wd[DIM], wad[DIM];
            cone_weights<DIM, G>(M.cwa, M.cwa32, wb + (size_t)(i - beg), wd, wad);
            if (state && !(ce.y & kConeBoundary)) {
ABL_UNROLL_SPECIES
                for (int k = 0; k < D::NC; k++) {
                    const G delta = G(un[k] - uc[k]);
#pragma unroll
                    for (int d = 0; d < DIM; d++) g[k * DIM + d] += wd[d] * delta;
                }
            }
            if (auxg) {
                S an[D::NA];
                cell_aux<DIM, NS>(P, un, aux, n, an);
ABL_UNROLL_SPECIES
                for (int k = 0; k < D::NA; k++) {
                    const G delta = G(an[k] - ac[k]);
#pragma unroll
                    for (int d = 0; d < DIM; d++) ga[k * DIM + d] += wad[d] * delta;
                }
            }
        }
        if constexpr (REC) {
            // the unlimited gradient, and the limiter's factor and minimising face per component
            double ph[D::NC];
            int is[D::NC];
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NC; k++) {
                ph[k] = 1.0;
                is[k] = -1;
            }
            if (do_state) {
                G* o = graw + (size_t)c * GR::GS;
ABL_UNROLL_SPECIES
                for (int k = 0; k < D::NC * DIM; k++) o[k] = g[k];
            }
            if (state && P.limiter != ABL_LIMITER_NONE) {
                limit_field<DIM, NS, G, LIM, true>(M, P, beg, end, wb, U, dU, uc, g, 0, D::NE, ph, is, sd);
                if (NS > 0) limit_field<DIM, NS, G, LIM, true>(M, P, beg, end, wb, U, dU, uc, g, D::NE, D::NC, ph, is, sd);
            }
            if (do_state) {
ABL_UNROLL_SPECIES
                for (int k = 0; k < D::NC; k++) {
                    rphi[(size_t)c * D::NC + k] = ph[k];
                    rist[(size_t)c * D::NC + k] = is[k];
                }
            }
        } else if (state && P.limiter != ABL_LIMITER_NONE) {
            limit_field<DIM, NS, G, LIM>(M, P, beg, end, wb, U, dU, uc, g, 0, D::NE, nullptr, nullptr, sd);
            if (NS > 0) limit_field<DIM, NS, G, LIM>(M, P, beg, end, wb, U, dU, uc, g, D::NE, D::NC, nullptr, nullptr, sd);
        }
    }
    if (do_state) {
        G* out = grad + (size_t)c * GR::GS;
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC * DIM; k++) out[k] = g[k];
    }
    if (do_aux) {
        G* out = agrad + (size_t)c * GR::AS;
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NA * DIM; k++) out[k] = ga[k];
    }
}

// ---------------------------------------------------------------------------------------------------
// Mixed-path advection for the AUSM family: FP64 for e = E/rho - |u|^2/2, T, p, the central flux parts
// and the assembly; FP32 for the sound speeds and the dissipative split-flux parts (flux_split).
template <int DIM, int NS>
__device__ __forceinline__ void advection_split(const Phys& P, const double* normal, const double* uL, const double* uR, double TL, double TR,
                                                bool adv, bool spadv, double* flux, bool* ok) {
    using D = Dims<DIM, NS>;
    double vel[2][DIM], e[2], p[2], irho[2], unA[2];
    float a[2];
    const double* us[2] = {uL, uR};
    const double guess[2] = {TL * .67 + .33 * TR, TL * .33 + .67 * TR};
    float area2 = 0.f;
#pragma unroll
    for (int d = 0; d < DIM; d++) area2 += float(normal[d]) * float(normal[d]);
    const float area = sqrtf(area2);
#pragma unroll
    for (int s = 0; s < 2; s++) {
        const double* u = us[s];
        const double rho = u[0];
        irho[s] = __drcp_rn(rho);
        double v2 = 0, un = 0;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            vel[s][d] = u[2 + d] * irho[s];
            v2 += vel[s][d] * vel[s][d];
            un += vel[s][d] * normal[d];
        }
        unA[s] = un;
        const double eint = u[1] * irho[s] - 0.5 * v2;
        if (NS == 0 || P.eos == ABL_EOS_PERFECT_GAS) {
            const double cv = P.r_gas / (P.gamma - 1.0);
            const double T = eint * (1.0 / cv);
            e[s] = eint;
            p[s] = P.r_gas * rho * T;
            a[s] = sqrtf(float(P.gamma * P.r_gas) * float(T));
        } else {
            double ys[NS > 0 ? NS : 1];
            fill_y(NS, rho, u + 2 + DIM, ys);
            const double T = nasa_temperature(P, NS, ys, eint, guess[s], ok);
            e[s] = e_sens(P, NS, ys, T);
            const double cp = mixture_cp(P, NS, ys, T);
            const double mw = mixture_mw(P, NS, ys);
            const double R = kRuniv / mw;
            p[s] = rho * kRuniv * T / mw;
            a[s] = sqrtf(float(cp / (cp - R) * R * T));
        }
    }
    SplitFlux sf = (P.flux == ABL_FLUX_AUSM) ? flux_split<ABL_FLUX_AUSM>(P, uL[0], p[0], unA[0], a[0], uR[0], p[1], unA[1], a[1], area)
                                             : flux_split<ABL_FLUX_AUSMPUP>(P, uL[0], p[0], unA[0], a[0], uR[0], p[1], unA[1], a[1], area);
    const double mA = sf.mA_c + double(sf.mA_d);
    const double p12 = sf.p_c + double(sf.p_d);
    const int s = sf.dir == ABL_DIR_LEFT ? 0 : 1;
    if (adv) {
        double v2 = 0;
#pragma unroll
        for (int d = 0; d < DIM; d++) v2 += vel[s][d] * vel[s][d];
        const double H = e[s] + 0.5 * v2 + p[s] * irho[s];
        flux[0] = mA;
        flux[1] = H * mA;
#pragma unroll
        for (int d = 0; d < DIM; d++) flux[2 + d] = vel[s][d] * mA + p12 * normal[d];
    }
    if (spadv) {
        const double* u = us[s];
ABL_UNROLL_SPECIES
        for (int k = 0; k < NS; k++) flux[D::NE + k] = mA * (u[D::NE + k] * irho[s]);
    }
}

// 1D face-gradient weights of the two cells of a face: the FaceInterpolant's 1D stencil::LeastSquares
// (faceInterpolant.cpp:32-36, stencils/leastSquares.cpp:5-122). With x_i the offset of cell i's centroid
// from the face centroid, the least-squares weights x_i / (x_L^2 + x_R^2), less their mean (the value
// weights are 1/2 each). fdx holds the face centroid minus each side's centroid.
__host__ __device__ __forceinline__ void face_weights_1d(const double* fdx, double* wl, double* wr) {
    const double xl = -fdx[0], xr = -fdx[3];
    const double s = xl * xl + xr * xr;
    const double gl = xl / s, gr = xr / s;
    const double m = 0.5 * gl + 0.5 * gr;
    *wl = gl - m;
    *wr = gr - m;
}

// ---------------------------------------------------------------------------------------------------
// flux of one face: advection (NS + species) and diffusion (NS + species), summed per component
// L and R index the rows of `src` (global cells, or tile-local slots of the fused kernel).
template <int DIM, int NS, class G, int FK, class Src>
__device__ __forceinline__ void face_flux(const Phys& P, const Src& src, int L, int R, const double* normal, const double* fdx, StateOf<G>* flux,
                                          bool* ok, bool* rok) {
    using D = Dims<DIM, NS>;
    using S = StateOf<G>;
ABL_UNROLL_SPECIES
    for (int k = 0; k < D::NC; k++) flux[k] = 0.0;
    S cL[D::NC], cR[D::NC];
    src.state(L, cL);
    src.state(R, cR);
    const bool adv = P.advection && P.flux != ABL_FLUX_OFF;
    const bool spadv = NS > 0 && P.sp_adv && P.flux != ABL_FLUX_OFF;
    if (adv || spadv) {
        const bool lsq = P.recon == ABL_RECON_LEASTSQUARES;
        // ProjectToFace (cellInterpolant.cpp:890-950): cells with a gradient are projected to the face
        S uL[D::NC], uR[D::NC];
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC; k++) {
            uL[k] = cL[k];
            uR[k] = cR[k];
        }
        if (lsq) {
            // cells without a gradient hold a zero row, so u + 0 . dx = u exactly
            G gL[D::NC * DIM], gR[D::NC * DIM];
            src.grad_row(L, gL);
            src.grad_row(R, gR);
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NC; k++) {
                G dotL = 0, dotR = 0;
#pragma unroll
                for (int d = 0; d < DIM; d++) {
                    dotL += gL[k * DIM + d] * G(fdx[d]);
                    dotR += gR[k * DIM + d] * G(fdx[3 + d]);
                }
                uL[k] = uL[k] + to_state<S>(dotL);
                uR[k] = uR[k] + to_state<S>(dotR);
            }
        }
        double TL = 300.0, TR = 300.0;
        if (NS > 0 && P.eos == ABL_EOS_NASA7) {
            TL = src.temperature(L);
            TR = src.temperature(R);
        }
        bool split = false;
        if constexpr (std::is_same<G, float>::value) {
            if (FK == ABL_FLUX_AUSM || FK == ABL_FLUX_AUSMPUP || (FK < 0 && (P.flux == ABL_FLUX_AUSM || P.flux == ABL_FLUX_AUSMPUP))) {
                advection_split<DIM, NS>(P, normal, uL, uR, TL, TR, adv, spadv, flux, ok);
                split = true;
            }
        }
        if (!split) {
            // NavierStokesTransport::AdvectionFlux (navierStokesTransport.cpp:99-207)
            double areaMag = 0;
#pragma unroll
            for (int d = 0; d < DIM; d++) areaMag += normal[d] * normal[d];
            areaMag = sqrt(areaMag);
            const double iA = rcp64(areaMag);
            double norm[DIM];
#pragma unroll
            for (int d = 0; d < DIM; d++) norm[d] = normal[d] * iA;
            const auto dL = decode<DIM, NS>(P, NS, uL, TL * .67 + .33 * TR, ok);
            const auto dR = decode<DIM, NS>(P, NS, uR, TL * .33 + .67 * TR, ok);
            const S rhoL = uL[0], rhoR = uR[0];
            const S irhoL = rcp64(rhoL), irhoR = rcp64(rhoR);
            S velL[DIM], velR[DIM], unL = 0, unR = 0;
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                velL[d] = uL[2 + d] * irhoL;
                unL += velL[d] * norm[d];
                velR[d] = uR[2 + d] * irhoR;
                unR += velR[d] * norm[d];
            }
            S mf, p12;
            const int dir = flux_calc_k<FK, S>(P, unL, dL.a, rhoL, dL.p, unR, dR.a, rhoR, dR.p, &mf, &p12, rok);
            if (adv) {
                flux[0] = mf * areaMag;
                if (dir == ABL_DIR_LEFT) {
                    S v2 = 0;
#pragma unroll
                    for (int d = 0; d < DIM; d++) v2 += velL[d] * velL[d];
                    const S velMag = dsqrt(v2);
                    const S H = dL.e + velMag * velMag / 2.0 + dL.p * irhoL;
                    flux[1] = H * mf * areaMag;
#pragma unroll
                    for (int n = 0; n < DIM; n++) flux[2 + n] = velL[n] * mf * areaMag + p12 * normal[n];
                } else if (dir == ABL_DIR_RIGHT) {
                    S v2 = 0;
#pragma unroll
                    for (int d = 0; d < DIM; d++) v2 += velR[d] * velR[d];
                    const S velMag = dsqrt(v2);
                    const S H = dR.e + velMag * velMag / 2.0 + dR.p * irhoR;
                    flux[1] = H * mf * areaMag;
#pragma unroll
                    for (int n = 0; n < DIM; n++) flux[2 + n] = velR[n] * mf * areaMag + p12 * normal[n];
                } else {
                    S v2L = 0, v2R = 0;
#pragma unroll
                    for (int d = 0; d < DIM; d++) {
                        v2L += velL[d] * velL[d];
                        v2R += velR[d] * velR[d];
                    }
                    const S mL = dsqrt(v2L), mR = dsqrt(v2R);
                    const S HL = dL.e + mL * mL / 2.0 + dL.p * irhoL;
                    const S HR = dR.e + mR * mR / 2.0 + dR.p * irhoR;
                    flux[1] = 0.5 * (HL + HR) * mf * areaMag;
#pragma unroll
                    for (int n = 0; n < DIM; n++) flux[2 + n] = 0.5 * (velL[n] + velR[n]) * mf * areaMag + p12 * normal[n];
                }
            }
            if (spadv) {
                // SpeciesTransport::AdvectionFlux (speciesTransport.cpp:263-341): LEFT upwinds, anything else takes the right
                // state; the compact process averages where there is no direction (compactCompressibleNSSpeciesTransport.cpp:257-259)
                if (dir == ABL_DIR_LEFT) {
ABL_UNROLL_SPECIES
                    for (int s = 0; s < NS; s++) flux[D::NE + s] = (mf * uL[D::NE + s] * irhoL) * areaMag;
                } else if (dir == ABL_DIR_NA && P.sp_compact) {
                    const S rhoM = 0.5 * (uL[0] + uR[0]);
ABL_UNROLL_SPECIES
                    for (int s = 0; s < NS; s++) flux[D::NE + s] = mf * 0.5 * (uR[D::NE + s] + uL[D::NE + s]) / rhoM * areaMag;
                } else {
ABL_UNROLL_SPECIES
                    for (int s = 0; s < NS; s++) flux[D::NE + s] = (mf * uR[D::NE + s] * irhoR) * areaMag;
                }
            }
        }
    }
    const bool dif = P.diffusion && P.transport != ABL_TRANSPORT_NONE;
    const bool spdif = NS > 0 && P.sp_dif && P.transport != ABL_TRANSPORT_NONE;
    if (dif || spdif) {
        // FaceInterpolant: face value = average of the two cells, face gradient = average of the two
        // cells' least-squares gradients (LeastSquaresAverage with numberStencils = 2)
        S fs[D::NC], fa[D::NA], aL[D::NA], aR[D::NA];
        src.aux_of(P, cL, L, aL);
        src.aux_of(P, cR, R, aR);
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC; k++) fs[k] = cL[k] * 0.5 + cR[k] * 0.5;
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NA; k++) fa[k] = aL[k] * 0.5 + aR[k] * 0.5;
        G gL[D::NA * DIM], gR[D::NA * DIM];
        if constexpr (DIM == 1) {
            // in 1D the face gradient is the two-cell LeastSquares stencil's; both sides carry it, so
            // the averages below return it exactly
            double wl, wr;
            face_weights_1d(fdx, &wl, &wr);
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NA; k++) gL[k] = gR[k] = static_cast<G>(aL[k] * wl + aR[k] * wr);
        } else {
            src.agrad_row(L, gL);
            src.agrad_row(R, gR);
        }
        S mu, kc, diff;
        transport<DIM, NS>(P, NS, fs, fa[0], &mu, &kc, &diff);
        if (dif) {
            // NavierStokesTransport::DiffusionFlux + CompressibleFlowComputeStressTensor (navierStokesTransport.cpp:454-532)
            G gv[DIM * DIM];
#pragma unroll
            for (int i = 0; i < DIM * DIM; i++) gv[i] = G(0.5) * gL[DIM + i] + G(0.5) * gR[DIM + i];
            G divVel = 0;
#pragma unroll
            for (int c = 0; c < DIM; ++c) divVel += gv[c * DIM + c];
            G tau[DIM * DIM];
            const G gmu = static_cast<G>(mu);
#pragma unroll
            for (int c = 0; c < DIM; ++c)
#pragma unroll
                for (int d = 0; d < DIM; ++d)
                    tau[c * DIM + d] = (d == c) ? G(2.0) * gmu * (gv[c * DIM + d] - divVel / G(3.0)) : gmu * (gv[c * DIM + d] + gv[d * DIM + c]);
#pragma unroll
            for (int c = 0; c < DIM; ++c) {
                G vf = 0;
#pragma unroll
                for (int d = 0; d < DIM; ++d) vf += -G(normal[d]) * tau[c * DIM + d];
                flux[2 + c] += to_state<S>(vf);
            }
            G ef = 0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                G heat = 0;
#pragma unroll
                for (int c = 0; c < DIM; ++c) heat += static_cast<G>(fa[1 + c]) * tau[d * DIM + c];
                heat += static_cast<G>(kc) * (G(0.5) * gL[d] + G(0.5) * gR[d]);
                heat *= -G(normal[d]);
                ef += heat;
            }
            flux[1] += to_state<S>(ef);
        }
        if constexpr (NS > 0) {
            if (spdif) {
                // SpeciesTransport::DiffusionEnergyFlux + DiffusionSpeciesFlux (speciesTransport.cpp:112-228),
                // or their VariableDiffusionCoefficient forms with one constant D_k per species (:154-194, :230-261)
                const S density = fs[0];
                S hs[NS];
                if (P.eos == ABL_EOS_NASA7) {
ABL_UNROLL_SPECIES
                    for (int s = 0; s < NS; s++) hs[s] = nasa_h_molar(P.nasa7 + 15 * s, fa[0]) * P.inv_mw[s] - P.href[s];
                } else {
ABL_UNROLL_SPECIES
                    for (int s = 0; s < NS; s++) hs[s] = 0.0;
                }
                const int yoff = (1 + DIM) * DIM;
                S ef = 0;
ABL_UNROLL_SPECIES
                for (int s = 0; s < NS; ++s) {
                    S sf = 0;
                    const S Ds = P.diff_k ? S(P.diff_k[s]) : diff;
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        const S gy = to_state<S>(G(0.5) * gL[yoff + s * DIM + d] + G(0.5) * gR[yoff + s * DIM + d]);
                        ef += -normal[d] * density * Ds * hs[s] * gy;
                        sf += -normal[d] * density * Ds * gy;
                    }
                    flux[D::NE + s] += sf;
                }
                flux[1] += ef;
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------------
// area normal and both sides' offsets of geometry record `rec` with vector loads
template <int DIM, class G>
__device__ __forceinline__ void face_geometry_rec(const DevMesh& M, size_t rec, double* normal, double* fdx) {
    if constexpr (std::is_same<G, float>::value) {
        const double2* r = reinterpret_cast<const double2*>(M.tf_geo32) + 3 * rec;
        const double2 a = __ldg(r), b = __ldg(r + 1), c = __ldg(r + 2);
        const double n[3] = {a.x, a.y, b.x};
#pragma unroll
        for (int d = 0; d < DIM; d++) normal[d] = n[d];
        const double packed[3] = {b.y, c.x, c.y};
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const unsigned long long bits = (unsigned long long)__double_as_longlong(packed[q]);
            fdx[2 * q] = double(__int_as_float((int)(bits & 0xffffffffull)));
            fdx[2 * q + 1] = double(__int_as_float((int)(bits >> 32)));
        }
    } else {
        const double2* r = reinterpret_cast<const double2*>(M.tf_geo) + 5 * rec;
        const double2 a = __ldg(r), b = __ldg(r + 1), c = __ldg(r + 2), e = __ldg(r + 3), f = __ldg(r + 4);
        const double n[3] = {a.x, a.y, b.x};
#pragma unroll
        for (int d = 0; d < DIM; d++) normal[d] = n[d];
        fdx[0] = b.y;
        fdx[1] = c.x;
        fdx[2] = c.y;
        fdx[3] = e.x;
        fdx[4] = e.y;
        fdx[5] = f.x;
    }
}
// the same for tile face record i
template <int DIM, class G>
__device__ __forceinline__ void face_geometry(const DevMesh& M, int i, double* normal, double* fdx) {
    face_geometry_rec<DIM, G>(M, geo_record(M, i), normal, fdx);
}

// ---------------------------------------------------------------------------------------------------
// One CTA per tile. Phase 1: face fluxes into shared memory (tile-ordered geometry streamed from HBM).
// Phase 2: each tile cell sums -+flux of its faces in ascending face order, adds the sum / V and writes F once.
template <int DIM, int NS, class G, int FK>
__global__ void __launch_bounds__(128, MinBlocks<NS, G>::tile) k_tile_flux(DevMesh M, Phys P, const double* __restrict__ U,
                                                                     const double* __restrict__ dU, const double* __restrict__ aux,
                                                                     const G* __restrict__ grad, const G* __restrict__ agrad,
                                                                     double* __restrict__ F, double* __restrict__ dF, int overwrite,
                                                                     int* status, int t0 = 0) {
    using D = Dims<DIM, NS>;
    using S = StateOf<G>;
    extern __shared__ double sflux_raw[];
    S* sflux = reinterpret_cast<S*>(sflux_raw);  // [faces of this tile][NC]
    const int t = t0 + blockIdx.x;
    const int fb = M.tile_face_ptr[t], fe = M.tile_face_ptr[t + 1];
    bool ok = true, rok = true;
    const GlobalRows<DIM, NS, G> src{U, dU, aux, grad, agrad};
    for (int i = fb + threadIdx.x; i < fe; i += blockDim.x) {
        const int2 lr = M.tf_cells[i];
        double normal[DIM], fdx[6];
        face_geometry<DIM, G>(M, i, normal, fdx);
        S flux[D::NC];
        face_flux<DIM, NS, G, FK>(P, src, lr.x, lr.y, normal, fdx, flux, &ok, &rok);
        S* out = sflux + (size_t)(i - fb) * D::NC;
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC; k++) out[k] = flux[k];
    }
    __syncthreads();
    const int cb = M.tile_cell_ptr[t], ce = M.tile_cell_ptr[t + 1];
    bool finite = true;
    for (int j = cb + threadIdx.x; j < ce; j += blockDim.x) {
        const int c = M.tile_cells[j];
        const double iv = M.ivol[c];
        S acc[D::NC];
        if (overwrite) {
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NC; k++) acc[k] = 0.0;
        } else {
ABL_UNROLL_SPECIES
            for (int k = 0; k < D::NC; k++) {
                if constexpr (std::is_same<S, Dual>::value)
                    acc[k] = Dual(F ? F[(size_t)c * D::NC + k] : 0.0, dF[(size_t)c * D::NC + k]);
                else
                    acc[k] = F[(size_t)c * D::NC + k];
            }
        }
        // the signed face fluxes summed first, then scaled by 1/V once: equal and opposite fluxes cancel
        // exactly (a uniform state keeps a zero residual, as the reference's per-face division gives;
        // a per-face fma(flux, 1/V, acc) would leave the rounding error of the product instead)
        S sum[D::NC];
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC; k++) sum[k] = 0.0;
        const int e0 = M.tc_fptr[j], e1 = M.tc_fptr[j + 1];
        for (int e = e0; e < e1; e++) {
            const uint16_t code = M.tc_face[e];
            const S* ff = sflux + (size_t)(code & 0x7fff) * D::NC;
            if (code & 0x8000) {
ABL_UNROLL_SPECIES
                for (int k = 0; k < D::NC; k++) sum[k] += ff[k];
            } else {
ABL_UNROLL_SPECIES
                for (int k = 0; k < D::NC; k++) sum[k] -= ff[k];
            }
        }
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC; k++) acc[k] += sum[k] * iv;
ABL_UNROLL_SPECIES
        for (int k = 0; k < D::NC; k++) {
            if constexpr (std::is_same<S, Dual>::value) {
                if (F) F[(size_t)c * D::NC + k] = acc[k].v;
                dF[(size_t)c * D::NC + k] = acc[k].d;
            } else {
                F[(size_t)c * D::NC + k] = acc[k];
            }
            finite = finite && dfinite(acc[k]);
        }
    }
    if (!finite) atomicOr(status, kStatusNaN);
    if (!ok) atomicOr(status, kStatusEos);
    if (!rok) atomicOr(status, kStatusRiemann);
}

}  // namespace abl
