// fv_kernels.cuh -- the RHS kernels (sm_100a), templated on dimension DIM, species count NS and the
// storage/arithmetic type G of the reconstruction (double: FP64 path; float: mixed path).
//
// One RHS evaluation is four passes over HBM-resident data:
//   k_aux       cells: T (EOS, guess = previous T), u = rho u / rho, Y = rho Y / rho
//               (CellSolver::UpdateAuxFields, src/solver/cellSolver.cpp:62-135)
//   k_gradient  cells: LSQ gradient of the conserved fields + BAM limiter
//               (CellInterpolant::ComputeFieldGradients, src/finiteVolume/cellInterpolant.cpp:330-497)
//               and the unlimited LSQ gradient of the aux fields that FaceInterpolant averages onto
//               faces (src/finiteVolume/faceInterpolant.cpp:109-249)
//   k_face_flux faces: projection, EOS decode, flux calculator, advection + diffusion fluxes
//               (cellInterpolant.cpp:499-639, faceInterpolant.cpp:262-448, the process flux functions)
//   k_gather    owned cells: F += sum over the cell's faces of -+flux / V, in ascending face order
//               (the scatter at cellInterpolant.cpp:604-629, made a deterministic gather)
#pragma once
#include <cfloat>

#include "fv_physics.cuh"

namespace abl {

enum StatusBits : int { kStatusNaN = 1, kStatusEos = 2, kStatusRiemann = 4 };

struct DevMesh {
    int dim, n_cells, n_faces, n_flux_faces;
    const int2* face_cells;
    const uint8_t* kind;
    const int* cone_ptr;
    const int* cone_face;
    const int* cone_nbr;
    const uint8_t* cone_side;
    const uint8_t* face_boundary;
    const int* flux_faces;
    const double* normal;  // [nf][3]
    const double* fdx;     // [nf][2][3] face centroid - side cell centroid (cell's own frame)
    const double* vol;     // [nc]
    const double* cgrad;   // [nf][2][3]
    const double* fgrad;   // [nf][2][3]
};

template <int DIM, int NS>
struct Dims {
    static constexpr int NE = 2 + DIM;     // euler components
    static constexpr int NC = NE + NS;     // conserved components per cell
    static constexpr int NA = 1 + DIM + NS;  // aux components per cell (T, u, Y)
};

template <class G>
__device__ __forceinline__ G big_value();
template <>
__device__ __forceinline__ double big_value<double>() { return DBL_MAX; }
template <>
__device__ __forceinline__ float big_value<float>() { return FLT_MAX; }

// ---------------------------------------------------------------------------------------------------
template <int DIM, int NS>
__global__ void __launch_bounds__(256) k_aux(DevMesh M, Phys P, const double* __restrict__ U, double* __restrict__ aux, int* status) {
    using D = Dims<DIM, NS>;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= M.n_cells) return;
    double u[D::NC];
#pragma unroll
    for (int k = 0; k < D::NC; k++) u[k] = U[(size_t)c * D::NC + k];
    double* a = aux + (size_t)c * D::NA;
    bool ok = true;
    a[0] = temperature<DIM, NS>(P, NS, u, a[0], &ok);
    const double rho = u[0];
#pragma unroll
    for (int d = 0; d < DIM; d++) a[1 + d] = u[2 + d] / rho;
#pragma unroll
    for (int s = 0; s < NS; s++) a[1 + DIM + s] = u[D::NE + s] / rho;
    if (!ok) atomicOr(status, kStatusEos);
}

// ---------------------------------------------------------------------------------------------------
template <int DIM, int NS, class G>
__device__ __forceinline__ void limit_field(const DevMesh& M, const Phys& P, int c, int beg, int end, const double* __restrict__ U, const double* uc,
                                            G* g, int k0, int k1) {
    using D = Dims<DIM, NS>;
    G phi[D::NC];
#pragma unroll
    for (int k = 0; k < D::NC; k++) phi[k] = big_value<G>();
    for (int i = beg; i < end; i++) {
        const int n = M.cone_nbr[i];
        const int f = M.cone_face[i];
        const int sc = M.cone_side[i];
        // x_n - x_c = (x_f - x_c) - (x_f - x_n), each offset taken in its own cell's frame
        G v[DIM];
#pragma unroll
        for (int d = 0; d < DIM; d++) v[d] = G(M.fdx[6 * (size_t)f + 3 * sc + d] - M.fdx[6 * (size_t)f + 3 * (1 - sc) + d]);
#pragma unroll
        for (int k = 0; k < D::NC; k++) {
            if (k < k0 || k >= k1) continue;
            G denom = 0;
#pragma unroll
            for (int d = 0; d < DIM; d++) denom += g[k * DIM + d] * v[d];
            const G diff = G(U[(size_t)n * D::NC + k] - uc[k]);
            const G flim = G(0.5) * diff / denom;
            phi[k] = pmin(phi[k], limiter<G>(P.limiter, flim));
        }
    }
    bool cancel = false;
#pragma unroll
    for (int k = 0; k < D::NC; k++) {
        if (k < k0 || k >= k1) continue;
        if (phi[k] == G(0)) {
#pragma unroll
            for (int d = 0; d < DIM; d++)
                if (dabs(g[k * DIM + d]) > G(P.max_lim_grad)) cancel = true;
        }
    }
#pragma unroll
    for (int k = 0; k < D::NC; k++) {
        if (k < k0 || k >= k1) continue;
#pragma unroll
        for (int d = 0; d < DIM; d++) g[k * DIM + d] *= cancel ? G(0) : phi[k];
    }
}

template <int DIM, int NS, class G>
__global__ void __launch_bounds__(128) k_gradient(DevMesh M, Phys P, const double* __restrict__ U, const double* __restrict__ aux,
                                                  G* __restrict__ grad, G* __restrict__ agrad, int do_state, int do_aux) {
    using D = Dims<DIM, NS>;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= M.n_cells) return;
    const uint8_t kind = M.kind[c];
    const int beg = M.cone_ptr[c], end = M.cone_ptr[c + 1];
    if (do_state && (kind == ABL_CELL_OWNED || kind == ABL_CELL_HALO)) {
        double uc[D::NC];
#pragma unroll
        for (int k = 0; k < D::NC; k++) uc[k] = U[(size_t)c * D::NC + k];
        G g[D::NC * DIM];
#pragma unroll
        for (int k = 0; k < D::NC * DIM; k++) g[k] = G(0);
        for (int i = beg; i < end; i++) {
            const int f = M.cone_face[i];
            if (M.face_boundary[f]) continue;
            const int n = M.cone_nbr[i];
            const double* w = M.cgrad + 6 * (size_t)f + 3 * M.cone_side[i];
            G wd[DIM];
#pragma unroll
            for (int d = 0; d < DIM; d++) wd[d] = G(w[d]);
#pragma unroll
            for (int k = 0; k < D::NC; k++) {
                const G delta = G(U[(size_t)n * D::NC + k] - uc[k]);
#pragma unroll
                for (int d = 0; d < DIM; d++) g[k * DIM + d] += wd[d] * delta;
            }
        }
        if (P.limiter != ABL_LIMITER_NONE) {
            limit_field<DIM, NS, G>(M, P, c, beg, end, U, uc, g, 0, D::NE);
            if (NS > 0) limit_field<DIM, NS, G>(M, P, c, beg, end, U, uc, g, D::NE, D::NC);
        }
        G* out = grad + (size_t)c * D::NC * DIM;
#pragma unroll
        for (int k = 0; k < D::NC * DIM; k++) out[k] = g[k];
    }
    if (do_aux && kind != ABL_CELL_HALO_OUTER) {
        double ac[D::NA];
#pragma unroll
        for (int k = 0; k < D::NA; k++) ac[k] = aux[(size_t)c * D::NA + k];
        G ga[D::NA * DIM];
#pragma unroll
        for (int k = 0; k < D::NA * DIM; k++) ga[k] = G(0);
        for (int i = beg; i < end; i++) {
            const int f = M.cone_face[i];
            const int n = M.cone_nbr[i];
            const double* w = M.fgrad + 6 * (size_t)f + 3 * M.cone_side[i];
            G wd[DIM];
#pragma unroll
            for (int d = 0; d < DIM; d++) wd[d] = G(w[d]);
#pragma unroll
            for (int k = 0; k < D::NA; k++) {
                const G delta = G(aux[(size_t)n * D::NA + k] - ac[k]);
#pragma unroll
                for (int d = 0; d < DIM; d++) ga[k * DIM + d] += wd[d] * delta;
            }
        }
        G* out = agrad + (size_t)c * D::NA * DIM;
#pragma unroll
        for (int k = 0; k < D::NA * DIM; k++) out[k] = ga[k];
    }
}

// ---------------------------------------------------------------------------------------------------
template <int DIM, int NS, class G>
__device__ __forceinline__ void project(const DevMesh& M, int f, int side, int c, bool lsq, const double* __restrict__ U, const G* __restrict__ grad,
                                        double* u) {
    using D = Dims<DIM, NS>;
#pragma unroll
    for (int k = 0; k < D::NC; k++) u[k] = U[(size_t)c * D::NC + k];
    const uint8_t kind = M.kind[c];
    if (lsq && (kind == ABL_CELL_OWNED || kind == ABL_CELL_HALO)) {
        G dx[DIM];
#pragma unroll
        for (int d = 0; d < DIM; d++) dx[d] = G(M.fdx[6 * (size_t)f + 3 * side + d]);
        const G* g = grad + (size_t)c * D::NC * DIM;
#pragma unroll
        for (int k = 0; k < D::NC; k++) {
            G dot = 0;
#pragma unroll
            for (int d = 0; d < DIM; d++) dot += g[k * DIM + d] * dx[d];
            u[k] = u[k] + double(dot);
        }
    }
}

template <int DIM, int NS, class G>
__global__ void __launch_bounds__(128) k_face_flux(DevMesh M, Phys P, const double* __restrict__ U, const double* __restrict__ aux,
                                                   const G* __restrict__ grad, const G* __restrict__ agrad, double* __restrict__ fflux,
                                                   int* status) {
    using D = Dims<DIM, NS>;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= M.n_flux_faces) return;
    const int f = M.flux_faces[idx];
    const int2 lr = M.face_cells[f];
    const int L = lr.x, R = lr.y;
    double normal[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) normal[d] = M.normal[3 * (size_t)f + d];
    double flux[D::NC];
#pragma unroll
    for (int k = 0; k < D::NC; k++) flux[k] = 0.0;
    bool ok = true, rok = true;
    const bool adv = P.advection && P.flux != ABL_FLUX_OFF;
    const bool spadv = NS > 0 && P.sp_adv && P.flux != ABL_FLUX_OFF;
    if (adv || spadv) {
        const bool lsq = P.recon == ABL_RECON_LEASTSQUARES;
        double uL[D::NC], uR[D::NC];
        project<DIM, NS, G>(M, f, 0, L, lsq, U, grad, uL);
        project<DIM, NS, G>(M, f, 1, R, lsq, U, grad, uR);
        double TL = 300.0, TR = 300.0;
        if (NS > 0 && P.eos == ABL_EOS_NASA7) {
            TL = aux[(size_t)L * D::NA];
            TR = aux[(size_t)R * D::NA];
        }
        // NavierStokesTransport::AdvectionFlux (navierStokesTransport.cpp:99-207)
        double areaMag = 0;
#pragma unroll
        for (int d = 0; d < DIM; d++) areaMag += normal[d] * normal[d];
        areaMag = sqrt(areaMag);
        double norm[DIM];
#pragma unroll
        for (int d = 0; d < DIM; d++) norm[d] = normal[d] / areaMag;
        const Decoded dL = decode<DIM, NS>(P, NS, uL, TL * .67 + .33 * TR, &ok);
        const Decoded dR = decode<DIM, NS>(P, NS, uR, TL * .33 + .67 * TR, &ok);
        const double rhoL = uL[0], rhoR = uR[0];
        double velL[DIM], velR[DIM], unL = 0, unR = 0;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            velL[d] = uL[2 + d] / rhoL;
            unL += velL[d] * norm[d];
            velR[d] = uR[2 + d] / rhoR;
            unR += velR[d] * norm[d];
        }
        double mf, p12;
        const int dir = flux_calc<double>(P, unL, dL.a, rhoL, dL.p, unR, dR.a, rhoR, dR.p, &mf, &p12, &rok);
        if (adv) {
            flux[0] = mf * areaMag;
            if (dir == ABL_DIR_LEFT) {
                double v2 = 0;
#pragma unroll
                for (int d = 0; d < DIM; d++) v2 += velL[d] * velL[d];
                const double velMag = sqrt(v2);
                const double H = dL.e + velMag * velMag / 2.0 + dL.p / rhoL;
                flux[1] = H * mf * areaMag;
#pragma unroll
                for (int n = 0; n < DIM; n++) flux[2 + n] = velL[n] * mf * areaMag + p12 * normal[n];
            } else if (dir == ABL_DIR_RIGHT) {
                double v2 = 0;
#pragma unroll
                for (int d = 0; d < DIM; d++) v2 += velR[d] * velR[d];
                const double velMag = sqrt(v2);
                const double H = dR.e + velMag * velMag / 2.0 + dR.p / rhoR;
                flux[1] = H * mf * areaMag;
#pragma unroll
                for (int n = 0; n < DIM; n++) flux[2 + n] = velR[n] * mf * areaMag + p12 * normal[n];
            } else {
                double v2L = 0, v2R = 0;
#pragma unroll
                for (int d = 0; d < DIM; d++) {
                    v2L += velL[d] * velL[d];
                    v2R += velR[d] * velR[d];
                }
                const double mL = sqrt(v2L), mR = sqrt(v2R);
                const double HL = dL.e + mL * mL / 2.0 + dL.p / rhoL;
                const double HR = dR.e + mR * mR / 2.0 + dR.p / rhoR;
                flux[1] = 0.5 * (HL + HR) * mf * areaMag;
#pragma unroll
                for (int n = 0; n < DIM; n++) flux[2 + n] = 0.5 * (velL[n] + velR[n]) * mf * areaMag + p12 * normal[n];
            }
        }
        if (spadv) {
            // SpeciesTransport::AdvectionFlux (speciesTransport.cpp:263-341): LEFT upwinds, anything else takes the right state
            if (dir == ABL_DIR_LEFT) {
#pragma unroll
                for (int s = 0; s < NS; s++) flux[D::NE + s] = (mf * uL[D::NE + s] / rhoL) * areaMag;
            } else {
#pragma unroll
                for (int s = 0; s < NS; s++) flux[D::NE + s] = (mf * uR[D::NE + s] / rhoR) * areaMag;
            }
        }
    }
    const bool dif = P.diffusion && P.transport != ABL_TRANSPORT_NONE;
    const bool spdif = NS > 0 && P.sp_dif && P.transport != ABL_TRANSPORT_NONE;
    if (dif || spdif) {
        // FaceInterpolant: face value = average of the two cells, face gradient = average of the two
        // cells' least-squares gradients (LeastSquaresAverage with numberStencils = 2)
        double fs[D::NC], fa[D::NA];
#pragma unroll
        for (int k = 0; k < D::NC; k++) fs[k] = U[(size_t)L * D::NC + k] * 0.5 + U[(size_t)R * D::NC + k] * 0.5;
#pragma unroll
        for (int k = 0; k < D::NA; k++) fa[k] = aux[(size_t)L * D::NA + k] * 0.5 + aux[(size_t)R * D::NA + k] * 0.5;
        const G* gL = agrad + (size_t)L * D::NA * DIM;
        const G* gR = agrad + (size_t)R * D::NA * DIM;
        double mu, kc, diff;
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
            const G gmu = G(mu);
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
                flux[2 + c] += double(vf);
            }
            G ef = 0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                G heat = 0;
#pragma unroll
                for (int c = 0; c < DIM; ++c) heat += G(fa[1 + c]) * tau[d * DIM + c];
                heat += G(kc) * (G(0.5) * gL[d] + G(0.5) * gR[d]);
                heat *= -G(normal[d]);
                ef += heat;
            }
            flux[1] += double(ef);
        }
        if constexpr (NS > 0) {
            if (spdif) {
                // SpeciesTransport::DiffusionEnergyFlux + DiffusionSpeciesFlux (speciesTransport.cpp:112-228)
                const double density = fs[0];
                double hs[NS];
                if (P.eos == ABL_EOS_NASA7) {
#pragma unroll
                    for (int s = 0; s < NS; s++) hs[s] = nasa_h_molar(P.nasa7 + 15 * s, fa[0]) * P.inv_mw[s] - P.href[s];
                } else {
#pragma unroll
                    for (int s = 0; s < NS; s++) hs[s] = 0.0;
                }
                const int yoff = (1 + DIM) * DIM;
                double ef = 0;
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    double sf = 0;
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        const double gy = double(G(0.5) * gL[yoff + s * DIM + d] + G(0.5) * gR[yoff + s * DIM + d]);
                        ef += -normal[d] * density * diff * hs[s] * gy;
                        sf += -normal[d] * density * diff * gy;
                    }
                    flux[D::NE + s] += sf;
                }
                flux[1] += ef;
            }
        }
    }
    double* out = fflux + (size_t)f * D::NC;
#pragma unroll
    for (int k = 0; k < D::NC; k++) out[k] = flux[k];
    if (!ok) atomicOr(status, kStatusEos);
    if (!rok) atomicOr(status, kStatusRiemann);
}

// ---------------------------------------------------------------------------------------------------
template <int DIM, int NS>
__global__ void __launch_bounds__(256) k_gather(DevMesh M, const double* __restrict__ fflux, double* __restrict__ F, int* status) {
    using D = Dims<DIM, NS>;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= M.n_cells) return;
    if (M.kind[c] != ABL_CELL_OWNED) return;
    const double V = M.vol[c];
    double acc[D::NC];
#pragma unroll
    for (int k = 0; k < D::NC; k++) acc[k] = F[(size_t)c * D::NC + k];
    const int beg = M.cone_ptr[c], end = M.cone_ptr[c + 1];
    for (int i = beg; i < end; i++) {
        const int f = M.cone_face[i];
        const double* ff = fflux + (size_t)f * D::NC;
        if (M.cone_side[i] == 0) {
#pragma unroll
            for (int k = 0; k < D::NC; k++) acc[k] -= ff[k] / V;
        } else {
#pragma unroll
            for (int k = 0; k < D::NC; k++) acc[k] += ff[k] / V;
        }
    }
    bool finite = true;
#pragma unroll
    for (int k = 0; k < D::NC; k++) {
        F[(size_t)c * D::NC + k] = acc[k];
        finite = finite && isfinite(acc[k]);
    }
    if (!finite) atomicOr(status, kStatusNaN);
}

}  // namespace abl
