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
    const double* tf_normal;  // [ntf][3]
    const double* tf_fdx;     // [ntf][6]
    const int* tc_fptr;
    const uint16_t* tc_face;
};

template <int DIM, int NS>
struct Dims {
    static constexpr int NE = 2 + DIM;       // euler components
    static constexpr int NC = NE + NS;       // conserved components per cell
    static constexpr int NA = 1 + DIM + NS;  // aux components per cell (T, u, Y)
};

template <class G>
__device__ __forceinline__ G big_value();
template <>
__device__ __forceinline__ double big_value<double>() { return DBL_MAX; }
template <>
__device__ __forceinline__ float big_value<float>() { return FLT_MAX; }

template <int DIM, int NS>
__device__ __forceinline__ void load_state(const double* __restrict__ U, int c, double* u) {
    using D = Dims<DIM, NS>;
#pragma unroll
    for (int k = 0; k < D::NC; k++) u[k] = __ldg(U + (size_t)c * D::NC + k);
}

// aux (T, u, Y) of one cell: from the resident aux array for the mixture EOS, recomputed from the
// conserved state for a perfect gas (UpdateAuxTemperatureField / UpdateAuxVelocityField /
// UpdateAuxMassFractionField: navierStokesTransport.cpp:534-558, speciesTransport.cpp:98-110)
template <int DIM, int NS>
__device__ __forceinline__ void cell_aux(const Phys& P, const double* u, const double* __restrict__ aux, int c, double* a) {
    using D = Dims<DIM, NS>;
    if (NS > 0 && P.eos == ABL_EOS_NASA7) {
#pragma unroll
        for (int k = 0; k < D::NA; k++) a[k] = __ldg(aux + (size_t)c * D::NA + k);
        return;
    }
    const double irho = rcp64(u[0]);
    double ke = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        a[1 + d] = u[2 + d] * irho;
        ke += a[1 + d] * a[1 + d];
    }
    a[0] = (u[1] * irho - 0.5 * ke) * rcp64(P.r_gas / (P.gamma - 1.0));
#pragma unroll
    for (int s = 0; s < NS; s++) a[1 + DIM + s] = u[D::NE + s] * irho;
}

// ---------------------------------------------------------------------------------------------------
template <int DIM, int NS>
__global__ void __launch_bounds__(256) k_aux(DevMesh M, Phys P, const double* __restrict__ U, double* __restrict__ aux, int* status) {
    using D = Dims<DIM, NS>;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= M.n_cells) return;
    double u[D::NC];
    load_state<DIM, NS>(U, c, u);
    double* a = aux + (size_t)c * D::NA;
    bool ok = true;
    a[0] = temperature<DIM, NS>(P, NS, u, a[0], &ok);
    const double irho = rcp64(u[0]);
#pragma unroll
    for (int d = 0; d < DIM; d++) a[1 + d] = u[2 + d] * irho;
#pragma unroll
    for (int s = 0; s < NS; s++) a[1 + DIM + s] = u[D::NE + s] * irho;
    if (!ok) atomicOr(status, kStatusEos);
}

// ---------------------------------------------------------------------------------------------------
template <int DIM, int NS, class G>
__device__ __forceinline__ void limit_field(const DevMesh& M, const Phys& P, int beg, int end, const double* __restrict__ U, const double* uc,
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
        for (int d = 0; d < DIM; d++) v[d] = G(__ldg(M.fdx + 6 * (size_t)f + 3 * sc + d) - __ldg(M.fdx + 6 * (size_t)f + 3 * (1 - sc) + d));
#pragma unroll
        for (int k = 0; k < D::NC; k++) {
            if (k < k0 || k >= k1) continue;
            G denom = 0;
#pragma unroll
            for (int d = 0; d < DIM; d++) denom += g[k * DIM + d] * v[d];
            const G diff = G(__ldg(U + (size_t)n * D::NC + k) - uc[k]);
            const G flim = G(0.5) * diff * rcp64(denom);
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
__global__ void __launch_bounds__(128, (NS > 2 ? 3 : 6)) k_gradient(DevMesh M, Phys P, const double* __restrict__ U, const double* __restrict__ aux,
                                                  G* __restrict__ grad, G* __restrict__ agrad, int do_state, int do_aux) {
    using D = Dims<DIM, NS>;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= M.n_cells) return;
    const uint8_t kind = M.kind[c];
    const int beg = M.cone_ptr[c], end = M.cone_ptr[c + 1];
    double uc[D::NC];
    load_state<DIM, NS>(U, c, uc);
    if (do_state && (kind == ABL_CELL_OWNED || kind == ABL_CELL_HALO)) {
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
            for (int d = 0; d < DIM; d++) wd[d] = G(__ldg(w + d));
#pragma unroll
            for (int k = 0; k < D::NC; k++) {
                const G delta = G(__ldg(U + (size_t)n * D::NC + k) - uc[k]);
#pragma unroll
                for (int d = 0; d < DIM; d++) g[k * DIM + d] += wd[d] * delta;
            }
        }
        if (P.limiter != ABL_LIMITER_NONE) {
            limit_field<DIM, NS, G>(M, P, beg, end, U, uc, g, 0, D::NE);
            if (NS > 0) limit_field<DIM, NS, G>(M, P, beg, end, U, uc, g, D::NE, D::NC);
        }
        G* out = grad + (size_t)c * D::NC * DIM;
#pragma unroll
        for (int k = 0; k < D::NC * DIM; k++) out[k] = g[k];
    }
    if (do_aux && kind != ABL_CELL_HALO_OUTER) {
        double ac[D::NA];
        cell_aux<DIM, NS>(P, uc, aux, c, ac);
        G ga[D::NA * DIM];
#pragma unroll
        for (int k = 0; k < D::NA * DIM; k++) ga[k] = G(0);
        for (int i = beg; i < end; i++) {
            const int f = M.cone_face[i];
            const int n = M.cone_nbr[i];
            const double* w = M.fgrad + 6 * (size_t)f + 3 * M.cone_side[i];
            G wd[DIM];
#pragma unroll
            for (int d = 0; d < DIM; d++) wd[d] = G(__ldg(w + d));
            double un[D::NC], an[D::NA];
            if (NS > 0 && P.eos == ABL_EOS_NASA7) {
                cell_aux<DIM, NS>(P, un, aux, n, an);
            } else {
                load_state<DIM, NS>(U, n, un);
                cell_aux<DIM, NS>(P, un, aux, n, an);
            }
#pragma unroll
            for (int k = 0; k < D::NA; k++) {
                const G delta = G(an[k] - ac[k]);
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
#pragma unroll
        for (int k = 0; k < NS; k++) flux[D::NE + k] = mA * (u[D::NE + k] * irho[s]);
    }
}

// ---------------------------------------------------------------------------------------------------
// flux of one face: advection (NS + species) and diffusion (NS + species), summed per component
template <int DIM, int NS, class G>
__device__ __forceinline__ void face_flux(const DevMesh& M, const Phys& P, int L, int R, const double* normal, const double* fdx,
                                          const double* __restrict__ U, const double* __restrict__ aux, const G* __restrict__ grad,
                                          const G* __restrict__ agrad, double* flux, bool* ok, bool* rok) {
    using D = Dims<DIM, NS>;
#pragma unroll
    for (int k = 0; k < D::NC; k++) flux[k] = 0.0;
    double cL[D::NC], cR[D::NC];
    load_state<DIM, NS>(U, L, cL);
    load_state<DIM, NS>(U, R, cR);
    const bool adv = P.advection && P.flux != ABL_FLUX_OFF;
    const bool spadv = NS > 0 && P.sp_adv && P.flux != ABL_FLUX_OFF;
    if (adv || spadv) {
        const bool lsq = P.recon == ABL_RECON_LEASTSQUARES;
        // ProjectToFace (cellInterpolant.cpp:890-950): cells with a gradient are projected to the face
        double uL[D::NC], uR[D::NC];
#pragma unroll
        for (int k = 0; k < D::NC; k++) {
            uL[k] = cL[k];
            uR[k] = cR[k];
        }
        if (lsq) {
            const uint8_t kL = M.kind[L], kR = M.kind[R];
            if (kL == ABL_CELL_OWNED || kL == ABL_CELL_HALO) {
                const G* g = grad + (size_t)L * D::NC * DIM;
#pragma unroll
                for (int k = 0; k < D::NC; k++) {
                    G dot = 0;
#pragma unroll
                    for (int d = 0; d < DIM; d++) dot += __ldg(g + k * DIM + d) * G(fdx[d]);
                    uL[k] = uL[k] + double(dot);
                }
            }
            if (kR == ABL_CELL_OWNED || kR == ABL_CELL_HALO) {
                const G* g = grad + (size_t)R * D::NC * DIM;
#pragma unroll
                for (int k = 0; k < D::NC; k++) {
                    G dot = 0;
#pragma unroll
                    for (int d = 0; d < DIM; d++) dot += __ldg(g + k * DIM + d) * G(fdx[3 + d]);
                    uR[k] = uR[k] + double(dot);
                }
            }
        }
        double TL = 300.0, TR = 300.0;
        if (NS > 0 && P.eos == ABL_EOS_NASA7) {
            TL = __ldg(aux + (size_t)L * D::NA);
            TR = __ldg(aux + (size_t)R * D::NA);
        }
        if (std::is_same<G, float>::value && (P.flux == ABL_FLUX_AUSM || P.flux == ABL_FLUX_AUSMPUP)) {
            advection_split<DIM, NS>(P, normal, uL, uR, TL, TR, adv, spadv, flux, ok);
        } else {
            // NavierStokesTransport::AdvectionFlux (navierStokesTransport.cpp:99-207)
            double areaMag = 0;
#pragma unroll
            for (int d = 0; d < DIM; d++) areaMag += normal[d] * normal[d];
            areaMag = sqrt(areaMag);
            const double iA = rcp64(areaMag);
            double norm[DIM];
#pragma unroll
            for (int d = 0; d < DIM; d++) norm[d] = normal[d] * iA;
            const Decoded dL = decode<DIM, NS>(P, NS, uL, TL * .67 + .33 * TR, ok);
            const Decoded dR = decode<DIM, NS>(P, NS, uR, TL * .33 + .67 * TR, ok);
            const double rhoL = uL[0], rhoR = uR[0];
            const double irhoL = rcp64(rhoL), irhoR = rcp64(rhoR);
            double velL[DIM], velR[DIM], unL = 0, unR = 0;
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                velL[d] = uL[2 + d] * irhoL;
                unL += velL[d] * norm[d];
                velR[d] = uR[2 + d] * irhoR;
                unR += velR[d] * norm[d];
            }
            double mf, p12;
            const int dir = flux_calc<double>(P, unL, dL.a, rhoL, dL.p, unR, dR.a, rhoR, dR.p, &mf, &p12, rok);
            if (adv) {
                flux[0] = mf * areaMag;
                if (dir == ABL_DIR_LEFT) {
                    double v2 = 0;
#pragma unroll
                    for (int d = 0; d < DIM; d++) v2 += velL[d] * velL[d];
                    const double velMag = sqrt(v2);
                    const double H = dL.e + velMag * velMag / 2.0 + dL.p * irhoL;
                    flux[1] = H * mf * areaMag;
#pragma unroll
                    for (int n = 0; n < DIM; n++) flux[2 + n] = velL[n] * mf * areaMag + p12 * normal[n];
                } else if (dir == ABL_DIR_RIGHT) {
                    double v2 = 0;
#pragma unroll
                    for (int d = 0; d < DIM; d++) v2 += velR[d] * velR[d];
                    const double velMag = sqrt(v2);
                    const double H = dR.e + velMag * velMag / 2.0 + dR.p * irhoR;
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
                    const double HL = dL.e + mL * mL / 2.0 + dL.p * irhoL;
                    const double HR = dR.e + mR * mR / 2.0 + dR.p * irhoR;
                    flux[1] = 0.5 * (HL + HR) * mf * areaMag;
#pragma unroll
                    for (int n = 0; n < DIM; n++) flux[2 + n] = 0.5 * (velL[n] + velR[n]) * mf * areaMag + p12 * normal[n];
                }
            }
            if (spadv) {
                // SpeciesTransport::AdvectionFlux (speciesTransport.cpp:263-341): LEFT upwinds, anything else takes the right state
                if (dir == ABL_DIR_LEFT) {
#pragma unroll
                    for (int s = 0; s < NS; s++) flux[D::NE + s] = (mf * uL[D::NE + s] * irhoL) * areaMag;
                } else {
#pragma unroll
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
        double fs[D::NC], fa[D::NA], aL[D::NA], aR[D::NA];
        cell_aux<DIM, NS>(P, cL, aux, L, aL);
        cell_aux<DIM, NS>(P, cR, aux, R, aR);
#pragma unroll
        for (int k = 0; k < D::NC; k++) fs[k] = cL[k] * 0.5 + cR[k] * 0.5;
#pragma unroll
        for (int k = 0; k < D::NA; k++) fa[k] = aL[k] * 0.5 + aR[k] * 0.5;
        const G* gL = agrad + (size_t)L * D::NA * DIM;
        const G* gR = agrad + (size_t)R * D::NA * DIM;
        double mu, kc, diff;
        transport<DIM, NS>(P, NS, fs, fa[0], &mu, &kc, &diff);
        if (dif) {
            // NavierStokesTransport::DiffusionFlux + CompressibleFlowComputeStressTensor (navierStokesTransport.cpp:454-532)
            G gv[DIM * DIM];
#pragma unroll
            for (int i = 0; i < DIM * DIM; i++) gv[i] = G(0.5) * __ldg(gL + DIM + i) + G(0.5) * __ldg(gR + DIM + i);
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
                heat += G(kc) * (G(0.5) * __ldg(gL + d) + G(0.5) * __ldg(gR + d));
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
                        const double gy = double(G(0.5) * __ldg(gL + yoff + s * DIM + d) + G(0.5) * __ldg(gR + yoff + s * DIM + d));
                        ef += -normal[d] * density * diff * hs[s] * gy;
                        sf += -normal[d] * density * diff * gy;
                    }
                    flux[D::NE + s] += sf;
                }
                flux[1] += ef;
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------------
// One CTA per tile. Phase 1: face fluxes into shared memory (tile-ordered geometry streamed from HBM).
// Phase 2: each tile cell adds -+flux/V of its faces in ascending face order and writes F once.
template <int DIM, int NS, class G>
__global__ void __launch_bounds__(128, (NS > 2 ? 2 : 3)) k_tile_flux(DevMesh M, Phys P, const double* __restrict__ U, const double* __restrict__ aux,
                                                   const G* __restrict__ grad, const G* __restrict__ agrad, double* __restrict__ F,
                                                   int overwrite, int* status) {
    using D = Dims<DIM, NS>;
    extern __shared__ double sflux[];  // [faces of this tile][NC]
    const int t = blockIdx.x;
    const int fb = M.tile_face_ptr[t], fe = M.tile_face_ptr[t + 1];
    bool ok = true, rok = true;
    for (int i = fb + threadIdx.x; i < fe; i += blockDim.x) {
        const int2 lr = M.tf_cells[i];
        double normal[DIM], fdx[6];
#pragma unroll
        for (int d = 0; d < DIM; d++) normal[d] = __ldg(M.tf_normal + 3 * (size_t)i + d);
#pragma unroll
        for (int d = 0; d < 3; d++) {
            fdx[d] = __ldg(M.tf_fdx + 6 * (size_t)i + d);
            fdx[3 + d] = __ldg(M.tf_fdx + 6 * (size_t)i + 3 + d);
        }
        double flux[D::NC];
        face_flux<DIM, NS, G>(M, P, lr.x, lr.y, normal, fdx, U, aux, grad, agrad, flux, &ok, &rok);
        double* out = sflux + (size_t)(i - fb) * D::NC;
#pragma unroll
        for (int k = 0; k < D::NC; k++) out[k] = flux[k];
    }
    __syncthreads();
    const int cb = M.tile_cell_ptr[t], ce = M.tile_cell_ptr[t + 1];
    bool finite = true;
    for (int j = cb + threadIdx.x; j < ce; j += blockDim.x) {
        const int c = M.tile_cells[j];
        const double iv = M.ivol[c];
        double acc[D::NC];
        if (overwrite) {
#pragma unroll
            for (int k = 0; k < D::NC; k++) acc[k] = 0.0;
        } else {
#pragma unroll
            for (int k = 0; k < D::NC; k++) acc[k] = F[(size_t)c * D::NC + k];
        }
        const int e0 = M.tc_fptr[j], e1 = M.tc_fptr[j + 1];
        for (int e = e0; e < e1; e++) {
            const uint16_t code = M.tc_face[e];
            const double* ff = sflux + (size_t)(code & 0x7fff) * D::NC;
            if (code & 0x8000) {
#pragma unroll
                for (int k = 0; k < D::NC; k++) acc[k] += ff[k] * iv;
            } else {
#pragma unroll
                for (int k = 0; k < D::NC; k++) acc[k] -= ff[k] * iv;
            }
        }
#pragma unroll
        for (int k = 0; k < D::NC; k++) {
            F[(size_t)c * D::NC + k] = acc[k];
            finite = finite && isfinite(acc[k]);
        }
    }
    if (!finite) atomicOr(status, kStatusNaN);
    if (!ok) atomicOr(status, kStatusEos);
    if (!rok) atomicOr(status, kStatusRiemann);
}

}  // namespace abl
