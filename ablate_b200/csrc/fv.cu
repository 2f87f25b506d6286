// fv.cu -- C ABI of the B200 finite-volume RHS backend (declared in include/ablate_fv.h): handle
// lifecycle, device residency of mesh/geometry/weights, kernel dispatch and the device batch entry
// points used by the known-answer tests.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "fv_handle.hpp"
#include "fv_setup.hpp"
#include "fv_step.cuh"

namespace abl {
thread_local std::string g_last_error;
}  // namespace abl

using namespace abl;

namespace {

// repeated geometry and weight records stored once (the default); ABL_FV_RECORD_TABLES=0 keeps one
// record per face and cone entry
bool record_tables() {
    const char* v = std::getenv("ABL_FV_RECORD_TABLES");
    return !(v && v[0] == '0');
}

// the fused one-pass RHS (where a tile fits in shared memory) when ABL_FV_FUSED=1 at create; by default
// the two-pass gradient + tile-flux kernels, which measured faster: the fused kernel recomputes the
// gradients of the cells around each tile (1.55x the instructions on the 64^3 Taylor-Green box) and
// its issue rate stayed near the two-pass kernels' (33 % against 25-30 %)
bool fused_enabled() {
    const char* v = std::getenv("ABL_FV_FUSED");
    return v && v[0] == '1';
}

// the mixed path with species (the exact instances up to 9 species) when ABL_FV_MIXED_SPECIES=1 at
// create; by default a mixed request with species runs the FP64 kernels
bool mixed_species_enabled() {
    const char* v = std::getenv("ABL_FV_MIXED_SPECIES");
    return v && v[0] == '1';
}

int fail(const AblError& e) {
    g_last_error = e.what();
    return e.code;
}
int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

template <class F>
int guarded(F&& fn) {
    try {
        fn();
        return ABL_OK;
    } catch (const AblError& e) {
        return fail(e);
    } catch (const std::invalid_argument& e) {
        return fail(ABL_ERR_INVALID_ARGUMENT, e.what());
    } catch (const std::bad_alloc&) {
        return fail(ABL_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(ABL_ERR_INVALID_ARGUMENT, e.what());
    }
}


// host NASA-7 molar enthalpy, same polynomial as the device
double host_h_molar(const double* c, double T) {
    const double* a = (T < c[0]) ? c + 1 : c + 8;
    return kRuniv * T * (a[0] + T * (a[1] * 0.5 + T * (a[2] * (1.0 / 3.0) + T * (a[3] * 0.25 + T * a[4] * 0.2))) + a[5] / T);
}

void validate_physics(const abl_physics_desc* p) {
    if (!p) throw std::invalid_argument("physics descriptor is NULL");
    if (p->eos != ABL_EOS_PERFECT_GAS && p->eos != ABL_EOS_NASA7) throw std::invalid_argument("unknown eos");
    if (p->n_species < 0 || p->n_species > kMaxSpecies)
        throw std::invalid_argument("n_species out of range (0.." + std::to_string(kMaxSpecies) + ")");
    if (p->eos == ABL_EOS_NASA7 && (p->n_species < 1 || !p->nasa7 || !p->mw)) throw std::invalid_argument("NASA-7 EOS needs n_species >= 1, nasa7 and mw");
    if (p->eos == ABL_EOS_PERFECT_GAS && !(p->gamma > 1.0 && p->r_gas > 0.0)) throw std::invalid_argument("perfect gas needs gamma > 1 and r_gas > 0");
    if (p->flux < ABL_FLUX_OFF || p->flux > ABL_FLUX_RIEMANN) throw std::invalid_argument("unknown flux calculator");
    if (p->flux == ABL_FLUX_RIEMANN && p->eos != ABL_EOS_PERFECT_GAS)
        throw std::invalid_argument("Riemann flux only accepts EOS of type eos::PerfectGas");  // riemann.cpp:37-43
    if (p->reconstruction != ABL_RECON_UPWIND && p->reconstruction != ABL_RECON_LEASTSQUARES) throw std::invalid_argument("unknown reconstruction");
    if (p->limiter < ABL_LIMITER_NONE || p->limiter > ABL_LIMITER_SIN) throw std::invalid_argument("unknown limiter");
    if (p->transport < ABL_TRANSPORT_NONE || p->transport > ABL_TRANSPORT_CONSTANT_LEWIS) throw std::invalid_argument("unknown transport model");
    if (p->species_diff) {
        // SpeciesTransport::Setup: the diffusion property size must be 1 or the number of species
        if (p->transport != ABL_TRANSPORT_CONSTANT || p->n_species <= 0)
            throw std::invalid_argument("per-species diffusivities need the constant transport model and species");
        for (int k = 0; k < p->n_species; k++)
            if (!std::isfinite(p->species_diff[k])) throw std::invalid_argument("per-species diffusivity must be finite");
    }
}

Phys make_phys(const abl_physics_desc* p) {
    Phys P{};
    P.eos = p->eos;
    P.ns = p->n_species;
    P.flux = p->flux;
    P.recon = p->reconstruction;
    P.limiter = p->limiter;
    P.transport = p->transport;
    P.advection = p->advection;
    P.diffusion = p->diffusion;
    P.sp_adv = p->species_advection;
    P.sp_dif = p->species_diffusion;
    P.sp_compact = p->species_advection_compact;
    P.gamma = p->gamma;
    P.r_gas = p->r_gas;
    P.minf = p->ausmpup_minf;
    P.alpha = p->pgs_alpha > 0 ? p->pgs_alpha : 1.0;
    P.max_lim_grad = p->max_lim_grad > 0 ? p->max_lim_grad : 1e10;
    P.k = p->k;
    P.mu = p->mu;
    P.diff = p->diff;
    return P;
}

// upload NASA-7 tables and derived per-species constants; fills P's device pointers
void upload_species(const abl_physics_desc* p, Phys& P, DevBuf<double>& nasa7, DevBuf<double>& mw, DevBuf<double>& inv_mw, DevBuf<double>& href) {
    if (p->eos != ABL_EOS_NASA7) return;
    const int ns = p->n_species;
    std::vector<double> imw(ns), hr(ns);
    for (int k = 0; k < ns; k++) {
        if (!(p->mw[k] > 0)) throw std::invalid_argument("molar mass must be positive");
        imw[k] = 1.0 / p->mw[k];
        hr[k] = host_h_molar(p->nasa7 + 15 * k, kTref) / p->mw[k];  // TChemBase reference enthalpy (tChemBase.cpp:43-69)
    }
    nasa7.upload(p->nasa7, (size_t)ns * 15);
    mw.upload(p->mw, ns);
    inv_mw.upload(imw.data(), ns);
    href.upload(hr.data(), ns);
    P.nasa7 = nasa7.p;
    P.mw = mw.p;
    P.inv_mw = inv_mw.p;
    P.href = href.p;
}

// ---- dispatch over the compiled (DIM, NS) instances ------------------------------------------------
// Exact species counts (fv_inst_a..d.cu, fv_adj_*.cu), the 16-species instances (fv_inst_e.cu,
// fv_inst_f.cu: RHS, aux update, tangent), the 3D 64-species instance (fv_inst_g.cu: RHS and aux update,
// fv_inst_h.cu: tangent; run-time loops) and the kMaxSpecies capacity instances (fv_inst_cap.cu: RHS
// and aux update, run-time loops), per dimension, ascending.
constexpr int kInstances[3][8] = {{0, 16, kMaxSpecies, -1}, {0, 2, 3, 16, kMaxSpecies, -1}, {0, 2, 3, 5, 9, 16, 64, kMaxSpecies}};

#define ABL_CASES_EXACT(FN, ...)                              \
    case 1000: FN<1, 0>(fv, __VA_ARGS__); break;              \
    case 2000: FN<2, 0>(fv, __VA_ARGS__); break;              \
    case 2002: FN<2, 2>(fv, __VA_ARGS__); break;              \
    case 2003: FN<2, 3>(fv, __VA_ARGS__); break;              \
    case 3000: FN<3, 0>(fv, __VA_ARGS__); break;              \
    case 3002: FN<3, 2>(fv, __VA_ARGS__); break;              \
    case 3005: FN<3, 5>(fv, __VA_ARGS__); break;              \
    case 3009: FN<3, 9>(fv, __VA_ARGS__); break;
#define ABL_CASES_16(FN, ...)                                 \
    case 1016: FN<1, 16>(fv, __VA_ARGS__); break;             \
    case 2016: FN<2, 16>(fv, __VA_ARGS__); break;             \
    case 3016: FN<3, 16>(fv, __VA_ARGS__); break;
#define ABL_CASES_64(FN, ...) \
    case 3064: FN<3, 64>(fv, __VA_ARGS__); break;
#define ABL_CASES_CAP(FN, ...)                                \
    case 1000 + kMaxSpecies: FN<1, kMaxSpecies>(fv, __VA_ARGS__); break; \
    case 2000 + kMaxSpecies: FN<2, kMaxSpecies>(fv, __VA_ARGS__); break; \
    case 3000 + kMaxSpecies: FN<3, kMaxSpecies>(fv, __VA_ARGS__); break;

// RHS and aux update: every instance
#define ABL_DISPATCH(fv, FN, ...)                                                                                         \
    do {                                                                                                                  \
        switch ((fv)->dim * 1000 + (fv)->ns) {                                                                            \
            ABL_CASES_EXACT(FN, __VA_ARGS__)                                                                              \
            ABL_CASES_16(FN, __VA_ARGS__)                                                                                 \
            ABL_CASES_64(FN, __VA_ARGS__)                                                                                 \
            ABL_CASES_CAP(FN, __VA_ARGS__)                                                                                \
            default: throw AblError(ABL_ERR_UNSUPPORTED, "no compiled RHS instance for this dimension/species count"); \
        }                                                                                                                 \
    } while (0)
// ghost fill, CFL, normalisation, stepping and the pressure functional: the exact counts (the callers
// check require_exact_instance first)
#define ABL_DISPATCH_EXACT(fv, FN, ...)                                                                                                \
    do {                                                                                                                               \
        switch ((fv)->dim * 1000 + (fv)->ns) {                                                                                         \
            ABL_CASES_EXACT(FN, __VA_ARGS__)                                                                                           \
            default: throw AblError(ABL_ERR_UNSUPPORTED, "this entry point has no compiled instance for this dimension/species count"); \
        }                                                                                                                              \
    } while (0)

void dispatch_rhs(abl_fv* fv, const double* U, double* F, int precision, int overwrite, cudaStream_t s) {
    ABL_DISPATCH(fv, run_rhs, U, F, precision, overwrite, s);
}

// the tangent: the exact counts and the 16-species instances (the capacity instance's run-time loops
// are not compiled for dual numbers)
void dispatch_jvp(abl_fv* fv, const double* U, const double* dU, double* F, double* dF, cudaStream_t s) {
    switch (fv->dim * 1000 + fv->ns) {
        ABL_CASES_EXACT(run_jvp, U, dU, F, dF, s)
        ABL_CASES_16(run_jvp, U, dU, F, dF, s)
        ABL_CASES_64(run_jvp, U, dU, F, dF, s)
        default:
            throw AblError(ABL_ERR_UNSUPPORTED, "the JVP is compiled for up to 16 species (64 in 3D); " + std::to_string(fv->ns_user) +
                                                    " species run in the " + std::to_string(fv->ns) + "-species instance, which has the RHS only");
    }
}

// the adjoint: the exact counts (up to 9 species)
void dispatch_vjp(abl_fv* fv, const double* U, const double* Fb, double* Ub, cudaStream_t s) {
    switch (fv->dim * 1000 + fv->ns) {
        ABL_CASES_EXACT(run_vjp, U, Fb, Ub, s)
        default:
            throw AblError(ABL_ERR_UNSUPPORTED, "the VJP is compiled for the exact species counts (0, 2, 3 in 2D; 0, 2, 5, 9 in 3D); " +
                                                    std::to_string(fv->ns_user) + " species run in the " + std::to_string(fv->ns) + "-species instance");
    }
}

// The instance that runs ns species in dim dimensions: the smallest compiled one that holds them (-1:
// none). ABL_FV_SPECIES_INSTANCE, read at create, asks for a larger one (a count then runs padded).
int instance_for(int dim, int ns) {
    int want = ns;
    if (const char* v = std::getenv("ABL_FV_SPECIES_INSTANCE")) want = std::max(ns, std::atoi(v));
    if (dim < 1 || dim > 3) return -1;
    for (int i = 0; i < 8 && kInstances[dim - 1][i] >= 0; i++)
        if (kInstances[dim - 1][i] >= want) return kInstances[dim - 1][i];
    return -1;
}

// ---- species padding ----------------------------------------------------------------------------
// A count without an instance of its own runs in a larger one: its rows there are [euler | pad
// zero-state species | the caller's species]. Padding species have zero NASA-7 rows, infinite molar
// mass (1/W = 0, h_ref = 0) and zero diffusivity, so every term they add to a sum is an exact zero;
// they come first so that the mixture's closing species (TChem's clipping gives the last species
// 1 - sum of the others) is the caller's last. Their limited gradient is zero (the limiters map the
// 0/0 ratio of a constant component to a zero factor, as PetscLimiterLimit's min/max forms do), and
// their own residual rows, zero, are dropped.
// rows [n][w] -> [n][w + pad], pad zero columns after column ne
__global__ void __launch_bounds__(256) k_pad_rows(const double* __restrict__ src, int64_t n, int w, int ne, int pad, double* __restrict__ dst) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int wi = w + pad;
    if (e >= n * wi) return;
    const int64_t i = e / wi;
    const int k = (int)(e - i * wi);
    dst[e] = k < ne ? src[i * w + k] : (k < ne + pad ? 0.0 : src[i * w + k - pad]);
}
// back: the listed rows (or all n) of [..][w + pad] into [..][w], the pad columns dropped; added or assigned
__global__ void __launch_bounds__(256) k_unpad_rows(const double* __restrict__ src, int64_t n, const int* __restrict__ rows, int w, int ne, int pad,
                                                    double* __restrict__ dst, int add) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n * w) return;
    const int64_t j = e / w;
    const int k = (int)(e - j * w);
    const int64_t r = rows ? (int64_t)__ldg(rows + j) : j;
    const double v = src[r * (w + pad) + (k < ne ? k : k + pad)];
    double* d = dst + r * w + k;
    *d = add ? *d + v : v;
}

// the caller's state rows in the instance's width (the scratch buffer), or the rows themselves
const double* pad_in(abl_fv* fv, DevBuf<double>& scratch, const double* user, cudaStream_t s) {
    if (fv->pad == 0) return user;
    const size_t n = (size_t)fv->n_cells * fv->nc;
    if (scratch.n != n) scratch.alloc(n);
    k_pad_rows<<<blocks_for((long)n, 256), 256, 0, s>>>(user, fv->n_cells, fv->nc_user, 2 + fv->dim, fv->pad, scratch.p);
    check_launch();
    return scratch.p;
}
// a zeroed residual buffer in the instance's width
double* pad_out(abl_fv* fv, DevBuf<double>& scratch, cudaStream_t s) {
    const size_t n = (size_t)fv->n_cells * fv->nc;
    if (scratch.n != n) scratch.alloc(n);
    ABL_CUDA(cudaMemsetAsync(scratch.p, 0, n * sizeof(double), s));
    return scratch.p;
}
// rows of the instance's residual into the caller's (owned rows only, or all)
void unpad_rows(abl_fv* fv, const double* inst, double* user, bool owned_only, bool add, cudaStream_t s) {
    const int64_t n = owned_only ? (int64_t)fv->owned_rows.n : (int64_t)fv->n_cells;
    if (n == 0) return;
    k_unpad_rows<<<blocks_for((long)(n * fv->nc_user), 256), 256, 0, s>>>(inst, n, owned_only ? fv->owned_rows.p : nullptr, fv->nc_user, 2 + fv->dim,
                                                                           fv->pad, user, add ? 1 : 0);
    check_launch();
}
// ghost fill, CFL, normalisation, stepping and the pressure functional are compiled for the exact
// species counts only (0, 2, 3 in 2D; 0, 2, 5, 9 in 3D)
void require_exact_instance(const abl_fv* fv, const char* what) {
    if (fv->pad || fv->ns > 9)
        throw AblError(ABL_ERR_UNSUPPORTED, std::string(what) + ": " + std::to_string(fv->ns_user) + " species run in the " + std::to_string(fv->ns) +
                                                "-species instance; this entry point is compiled for the exact counts (0, 2, 3 in 2D; 0, 2, 5, 9 in 3D)");
}

// ---- batch kernels ------------------------------------------------------------------------------
__global__ void k_flux_batch(Phys P, int64_t n, const double* uL, const double* aL, const double* rhoL, const double* pL, const double* uR,
                             const double* aR, const double* rhoR, const double* pR, double* mf, double* p12, int32_t* dir, int* status) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool ok = true;
    double m, p;
    dir[i] = flux_calc<double>(P, uL[i], aL[i], rhoL[i], pL[i], uR[i], aR[i], rhoR[i], pR[i], &m, p12 ? &p : nullptr, &ok);
    mf[i] = m;
    if (p12) p12[i] = p;
    if (!ok) atomicOr(status, kStatusRiemann);
}

template <int DIM>
__device__ void eos_property(const Phys& P, int ns, int prop, const double* U, bool hasT, double Tin, double* out, bool* ok) {
    const double rho = U[0];
    const bool pg = P.eos == ABL_EOS_PERFECT_GAS;
    const double g = P.gamma, Rg = P.r_gas;
    if (!hasT) {
        if (pg) {
            const double e = internal_energy<DIM>(U);
            if (prop == ABL_PROP_PRESSURE) {
                *out = (g - 1.0) * rho * e;
                return;
            }
            if (prop == ABL_PROP_INTERNAL_SENSIBLE_ENERGY) {
                *out = e;
                return;
            }
            if (prop == ABL_PROP_SPEED_OF_SOUND) {
                const double pr = (g - 1.0) * rho * e;
                *out = sqrt(g * (pr) / rho);
                return;
            }
        } else if (prop == ABL_PROP_INTERNAL_SENSIBLE_ENERGY) {
            *out = internal_energy<DIM>(U);
            return;
        }
        Tin = temperature<DIM, kMaxSpecies>(P, ns, U, 300.0, ok);
        if (prop == ABL_PROP_TEMPERATURE) {
            *out = Tin;
            return;
        }
    }
    const double T = Tin;
    if (pg) {
        switch (prop) {
            case ABL_PROP_PRESSURE: *out = Rg * rho * T; return;
            case ABL_PROP_TEMPERATURE: *out = temperature<DIM, 0>(P, 0, U, T, ok); return;
            case ABL_PROP_INTERNAL_SENSIBLE_ENERGY: *out = T * (Rg / (g - 1.0)); return;
            case ABL_PROP_SENSIBLE_ENTHALPY: *out = T * (g * Rg / (g - 1.0)); return;
            case ABL_PROP_CV: *out = Rg / (g - 1.0); return;
            case ABL_PROP_CP: *out = g * Rg / (g - 1.0); return;
            case ABL_PROP_SPEED_OF_SOUND: {
                const double pr = Rg * rho * T;
                *out = sqrt(g * (pr) / rho);
                return;
            }
            case ABL_PROP_SPECIES_SENSIBLE_ENTHALPY:
                for (int s = 0; s < ns; s++) out[s] = 0.0;
                return;
            case ABL_PROP_DENSITY: *out = rho; return;
        }
        return;
    }
    double ys[kMaxSpecies];
    fill_y(ns, rho, U + 2 + DIM, ys);
    switch (prop) {
        case ABL_PROP_PRESSURE: *out = rho * kRuniv * T / mixture_mw(P, ns, ys); return;
        case ABL_PROP_TEMPERATURE: *out = temperature<DIM, kMaxSpecies>(P, ns, U, T, ok); return;
        case ABL_PROP_INTERNAL_SENSIBLE_ENERGY: *out = e_sens(P, ns, ys, T); return;
        case ABL_PROP_SENSIBLE_ENTHALPY: {
            double h = 0;
            for (int k = 0; k < ns; k++) h += (nasa_h_molar(P.nasa7 + 15 * k, T) * P.inv_mw[k] - P.href[k]) * ys[k];
            *out = h;
            return;
        }
        case ABL_PROP_CV: *out = mixture_cp(P, ns, ys, T) - kRuniv / mixture_mw(P, ns, ys); return;
        case ABL_PROP_CP: *out = mixture_cp(P, ns, ys, T); return;
        case ABL_PROP_SPEED_OF_SOUND: {
            const double cp = mixture_cp(P, ns, ys, T);
            const double R = kRuniv / mixture_mw(P, ns, ys);
            const double cv = cp - R;
            *out = sqrt(cp / cv * R * T);
            return;
        }
        case ABL_PROP_SPECIES_SENSIBLE_ENTHALPY:
            for (int k = 0; k < ns; k++) out[k] = nasa_h_molar(P.nasa7 + 15 * k, T) * P.inv_mw[k] - P.href[k];
            return;
        case ABL_PROP_DENSITY: *out = rho; return;
    }
}

template <int DIM>
__global__ void k_eos_batch(Phys P, int ns, int prop, int64_t n, const double* conserved, const double* T_in, double* out, int* status) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int nc = 2 + DIM + ns;
    const int psz = prop == ABL_PROP_SPECIES_SENSIBLE_ENTHALPY ? ns : 1;
    double u[2 + 3 + kMaxSpecies];
    for (int k = 0; k < nc; k++) u[k] = conserved[i * nc + k];
    bool ok = true;
    eos_property<DIM>(P, ns, prop, u, T_in != nullptr, T_in ? T_in[i] : 0.0, out + i * psz, &ok);
    if (!ok) atomicOr(status, kStatusEos);
}

int status_to_code(int bits) {
    if (bits & kStatusNaN) return ABL_ERR_NAN;
    if (bits & kStatusEos) return ABL_ERR_EOS_NOT_CONVERGED;
    if (bits & kStatusRiemann) return ABL_ERR_RIEMANN_NOT_CONVERGED;
    return ABL_OK;
}

}  // namespace

// ---- allocation-free EOS batch ----------------------------------------------------------------------
// Scratch of abl_eos_batch_noalloc: the NASA-7 tables the kernel reads (T_mid + 14 coefficients, molar
// mass, 1/molar mass, reference enthalpy per species) followed by the status word. 16 KiB, held by every
// GPU that loads this library until the process exits; 64 species need 9,216 bytes.
constexpr int kNoAllocMaxSpecies = 64;
constexpr size_t kNoAllocScratchBytes = 16384;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch on the current device (host code cannot use the symbol itself:
// on the host it names a stand-in, not device memory). Looked up on every call, so a new context after
// a cudaDeviceReset gets its own address; the lookup allocates nothing, though on first use it may make
// CUDA load this library's device code.
unsigned char* noalloc_scratch() {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) throw AblError(ABL_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    return static_cast<unsigned char*>(ptr);
}

// =================================================================================================
// halo pack (SCATTER = 0: dst[i] = src[idx[i]]), unpack (SCATTER = 1: dst[idx[i]] = src[i]) and the
// adjoint's accumulate (SCATTER = 2: dst[idx[i]] += src[i], indices distinct), one thread per element
// so consecutive threads move consecutive doubles of a row
template <int SCATTER>
__global__ void __launch_bounds__(256) k_rows(const double* __restrict__ src, int width, const int32_t* __restrict__ idx, int64_t n,
                                              double* __restrict__ dst) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n * width) return;
    const int64_t i = e / width;
    const int k = (int)(e - i * width);
    const int64_t r = __ldg(idx + i);
    if (SCATTER == 2)
        dst[r * width + k] += src[i * width + k];
    else if (SCATTER == 1)
        dst[r * width + k] = src[i * width + k];
    else
        dst[i * width + k] = src[r * width + k];
}

extern "C" {

const char* abl_last_error_string(void) { return g_last_error.c_str(); }

int abl_version(void) { return 1; }

int abl_device_count(int* count) {
    return guarded([&] {
        if (!count) throw std::invalid_argument("count is NULL");
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess) {
            *count = 0;
            throw AblError(ABL_ERR_NO_DEVICE, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
        }
        *count = n;
    });
}

int abl_fv_create(const abl_mesh_desc* mesh, const abl_physics_desc* physics, int device, abl_fv** out) {
    return guarded([&] {
        if (!out) throw std::invalid_argument("out is NULL");
        *out = nullptr;
        validate_physics(physics);
        if (!mesh) throw std::invalid_argument("mesh descriptor is NULL");
        if (mesh->dim < 1 || mesh->dim > 3) throw std::invalid_argument("invalid mesh descriptor: dim must be 1, 2 or 3");
        const int ns_user = physics->n_species;
        const int ns_inst = instance_for(mesh->dim, ns_user);
        if (ns_inst < 0)
            throw AblError(ABL_ERR_UNSUPPORTED, "no compiled RHS instance for dim " + std::to_string(mesh->dim) + " with " +
                                                    std::to_string(ns_user) + " species");
        // the caller's physics in the instance's species layout (padding species first)
        const int pad = ns_inst - ns_user;
        abl_physics_desc padded = *physics;
        std::vector<double> pnasa7, pmw, pdiff;
        if (pad > 0) {
            padded.n_species = ns_inst;
            if (physics->eos == ABL_EOS_NASA7) {
                pnasa7.assign(15 * (size_t)pad, 0.0);
                pnasa7.insert(pnasa7.end(), physics->nasa7, physics->nasa7 + 15 * (size_t)ns_user);
                pmw.assign((size_t)pad, std::numeric_limits<double>::infinity());
                pmw.insert(pmw.end(), physics->mw, physics->mw + ns_user);
                padded.nasa7 = pnasa7.data();
                padded.mw = pmw.data();
            }
            if (physics->species_diff) {
                pdiff.assign((size_t)pad, 0.0);
                pdiff.insert(pdiff.end(), physics->species_diff, physics->species_diff + ns_user);
                padded.species_diff = pdiff.data();
            }
            validate_physics(&padded);
            physics = &padded;
        }
        const bool lsq = physics->reconstruction == ABL_RECON_LEASTSQUARES;
        const bool dif = (physics->diffusion || (physics->species_diffusion && physics->n_species > 0)) && physics->transport != ABL_TRANSPORT_NONE;
        // the descriptor is checked and set up on the host first, so a corrupt mesh is rejected the same
        // way with or without a device
        HostMesh h = build_host_mesh(mesh, lsq, dif);
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw AblError(ABL_ERR_NO_DEVICE, "no CUDA device visible");
        if (device < 0 || device >= ndev) throw std::invalid_argument("device index out of range");
        ABL_CUDA(cudaSetDevice(device));
        std::unique_ptr<abl_fv> fv(new abl_fv);
        fv->device = device;
        ABL_CUDA(cudaDeviceGetAttribute(&fv->n_sm, cudaDevAttrMultiProcessorCount, device));
        fv->phys = make_phys(physics);
        fv->dim = h.dim;
        fv->ns = physics->n_species;
        fv->nc = 2 + h.dim + fv->ns;
        fv->naux = 1 + h.dim + fv->ns;
        fv->ns_user = ns_user;
        fv->pad = pad;
        fv->mixed_species = mixed_species_enabled() && fv->ns > 0 && fv->ns <= 9;
        fv->nc_user = fv->nc - pad;
        fv->naux_user = fv->naux - pad;
        fv->n_cells = h.n_cells;
        fv->n_faces = h.n_faces;
        fv->n_flux_faces = (int)h.flux_faces.size();
        fv->need_state_grad = lsq;
        fv->need_aux_grad = dif;
        // the mixture EOS keeps T resident (secant guess + face temperatures); a perfect gas recomputes it
        fv->need_aux = physics->eos == ABL_EOS_NASA7;
        upload_species(physics, fv->phys, fv->nasa7, fv->mw, fv->inv_mw, fv->href);
        if (physics->species_diff && physics->species_diffusion) {
            fv->diff_k.upload(physics->species_diff, physics->n_species);
            fv->phys.diff_k = fv->diff_k.p;
        }

        fv->face_cells.upload(reinterpret_cast<const int2*>(h.face_cells.data()), h.n_faces);
        fv->kind.upload(h.kind.data(), h.kind.size());
        fv->cone_ptr.upload(h.cone_ptr.data(), h.cone_ptr.size());
        {
            // cone entry: (face, neighbour | side << 31 | boundary face << 30)
            if (h.n_cells >= (1 << 30)) throw std::invalid_argument("too many cells for the packed cone");
            std::vector<int2> cone(h.cone_face.size());
            for (size_t i = 0; i < cone.size(); i++) {
                const int f = h.cone_face[i];
                cone[i].x = f;
                cone[i].y = h.cone_nbr[i] | (h.cone_side[i] ? kConeSide : 0) | (h.face_boundary[f] ? kConeBoundary : 0);
            }
            fv->cone.upload(cone.data(), cone.size());
        }
        fv->fdx.upload(h.fdx.data(), h.fdx.size());
        {
            std::vector<double> iv(h.n_cells);
            for (int c = 0; c < h.n_cells; c++) iv[c] = 1.0 / mesh->cell_volume[c];
            fv->ivol.upload(iv.data(), iv.size());
        }
        // cell tiles for the fused flux kernel: the largest tile whose face fluxes fit in shared memory
        const int nc_ = 2 + h.dim + physics->n_species;
        // tiles from the caller's cell order and from a Morton sort; keep the one that duplicates fewer faces
        auto tiles_for = [&](int tile) {
            Tiles a = build_tiles(h, mesh, tile, false);
            Tiles b = build_tiles(h, mesh, tile, true);
            return b.tf_cells.size() < a.tf_cells.size() ? b : a;
        };
        // and whose shared memory fits every pass: the face fluxes (value and tangent pairs in the JVP) and
        // the adjoint's per-cell accumulator rows (state, gradient, aux, aux gradient; odd stride)
        const int naux_ = 1 + h.dim + physics->n_species;
        const size_t adj_row = (size_t)((nc_ + nc_ * h.dim + naux_ + naux_ * h.dim) | 1) * sizeof(double);
        auto fits = [&](const Tiles& t, int cells) {
            const size_t faces = (size_t)std::max(t.max_faces, 1) * nc_ * sizeof(double);
            return faces <= 200 * 1024 && 2 * faces <= 227 * 1024 && (size_t)cells * adj_row <= 227 * 1024;
        };
        int tile = 256;
        Tiles tl = tiles_for(tile);
        while (!fits(tl, tile) && tile > 16) {
            tile /= 2;
            tl = tiles_for(tile);
        }
        fv->tile_smem = (int)((size_t)std::max(tl.max_faces, 1) * nc_ * sizeof(double));
        std::vector<uint16_t> geo_cls;  // per tile face record its geometry record (kept for the fused tables)
        fv->tile_cell_ptr.upload(tl.cell_ptr.data(), tl.cell_ptr.size());
        fv->tile_cells.upload(tl.cells.data(), tl.cells.size());
        fv->tile_face_ptr.upload(tl.face_ptr.data(), tl.face_ptr.size());
        fv->tf_cells.upload(reinterpret_cast<const int2*>(tl.tf_cells.data()), tl.tf_cells.size() / 2);
        {
            // per tile face one 80-byte record: normal, both offsets, a pad (five 16-byte loads), stored
            // once per distinct record where they repeat; the mixed path's 48-byte record holds the
            // normal and the offsets as FP32 pairs
            GeoRecords gr = tile_geometry(tl, record_tables());
            geo_cls = gr.cls;
            const std::vector<double>& geo = gr.geo;
            const size_t ntf = geo.size() / 10;
            if (!gr.cls.empty()) {
                fv->tf_gcls.upload(gr.cls.data(), gr.cls.size());
                fv->n_geo_classes = (int)ntf;
            }
            fv->tf_geo.upload(geo.data(), geo.size());
            if (fv->ns == 0 || fv->mixed_species) {
                std::vector<double> g32(6 * ntf, 0.0);
                for (size_t i = 0; i < ntf; i++) {
                    for (int d = 0; d < 3; d++) g32[6 * i + d] = geo[10 * i + d];
                    float f[6];
                    for (int z = 0; z < 6; z++) f[z] = (float)geo[10 * i + 3 + z];
                    std::memcpy(&g32[6 * i + 3], f, sizeof f);
                }
                fv->tf_geo32.upload(g32.data(), g32.size());
            }
        }
        fv->tc_fptr.upload(tl.tc_fptr.data(), tl.tc_fptr.size());
        fv->tc_face.upload(tl.tc_face.data(), tl.tc_face.size());
        fv->col_base.upload(tl.col_base.data(), tl.col_base.size());
        fv->col_start.upload(tl.col_start.data(), tl.col_start.size());
        fv->tf_slot.upload(tl.tf_slot.data(), tl.tf_slot.size());
        fv->tf_adj.upload(tl.tf_adj.data(), tl.tf_adj.size());
        fv->tf_nb.upload(tl.tf_nb.data(), tl.tf_nb.size());
        fv->face_nb.upload(tl.face_nb.data(), tl.face_nb.size());
        fv->n_nb = tl.n_nb;
        for (int k = 0; k < tl.n_tiles; k++) fv->tile_max_cells = std::max(fv->tile_max_cells, tl.cell_ptr[k + 1] - tl.cell_ptr[k]);
        {
            std::vector<int32_t> no, ow;
            for (int c = 0; c < h.n_cells; c++) (h.kind[c] != ABL_CELL_OWNED ? no : ow).push_back(c);
            fv->nonowned.upload(no.data(), no.size());
            fv->owned_rows.upload(ow.data(), ow.size());
            if (!ow.empty() && ow.back() - ow.front() + 1 == (int)ow.size()) {
                fv->owned_lo = ow.front();
                fv->owned_hi = ow.back() + 1;
            }
            // output chunks of the host-buffer RHS: possible when every tile's cells are one ascending
            // range and the tiles follow each other, and worth it when the residual is large (below
            // 16 MiB the launch and copy overheads of 16 chunks outweigh the overlap: the 256^2 Euler
            // case, 2 MiB, runs 35 % slower chunked)
            bool ranges = fv->owned_hi >= 0 && tl.n_tiles >= abl_fv::kHostChunks &&
                          (size_t)(fv->owned_hi - fv->owned_lo) * nc_ * sizeof(double) >= (size_t(16) << 20);
            for (size_t j = 1; ranges && j < tl.cells.size(); j++) ranges = tl.cells[j] == tl.cells[j - 1] + 1;
            if (ranges) {
                for (int q = 0; q <= abl_fv::kHostChunks; q++) {
                    const int tq = (int)((int64_t)tl.n_tiles * q / abl_fv::kHostChunks);
                    fv->chunk_tile.push_back(tq);
                    fv->chunk_row.push_back(tq < tl.n_tiles ? tl.cells[tl.cell_ptr[tq]] : fv->owned_hi);
                }
            }
        }
        if (lsq) fv->cgrad.upload(h.cgrad.data(), h.cgrad.size());
        if (dif) fv->fgrad.upload(h.fgrad.data(), h.fgrad.size());
        {
            // cone-major weights and offsets, one copy per distinct cell sequence where they repeat
            ConeRecords cr = cone_records(h, lsq, dif, record_tables());
            const std::vector<double>& cwa = cr.cwa;
            const std::vector<double>& cv = cr.cv;
            const std::vector<double>& cwar = cr.cwar;
            const int maxc = cr.max_cone;
            if (cr.classes) {
                fv->cone_cls.upload(cr.base.data(), cr.base.size());
                fv->n_cone_classes = (int)cr.classes;
            }
            fv->cwa.upload(cwa.data(), cwa.size());
            fv->cv.upload(cv.data(), cv.size());
            fv->cwar.upload(cwar.data(), cwar.size());
            if (fv->ns == 0 || fv->mixed_species) {  // the mixed path's copies (with species by default it runs the FP64 kernels)
                const size_t nw = cwa.size() / 6;
                std::vector<float> f32(8 * nw, 0.0f);
                for (size_t i = 0; i < nw; i++)
                    for (int d = 0; d < 6; d++) f32[8 * i + d] = (float)cwa[6 * i + d];
                fv->cwa32.upload(f32.data(), f32.size());
                f32.assign(cv.begin(), cv.end());
                fv->cv32.upload(f32.data(), f32.size());
            }
            fv->max_cone = maxc;
            if (fused_enabled() && tl.n_tiles > 0) {
                std::vector<int32_t> wb(h.n_cells);
                for (int c = 0; c < h.n_cells; c++) wb[c] = cr.classes ? cr.base[c] : h.cone_ptr[c];
                FusedTiles ft = fused_tiles(h, tl, wb, geo_cls);
                const bool nasa = physics->eos == ABL_EOS_NASA7 && fv->ns > 0;
                for (int q = 0; q < 2; q++) {
                    fv->fused_smem[q] = fused_smem_bytes(h.dim, fv->nc, fv->naux, q == 0 ? 8 : 4, ft.max_ext, ft.max_grad, ft.max_faces, nasa);
                    // the mixed path with species runs the FP64 kernels
                    fv->fused_ok[q] = fv->fused_smem[q] <= kFusedSmemLimit && (q == 0 || fv->ns == 0);
                }
                if (fv->fused_ok[0] || fv->fused_ok[1]) {
                    fv->fz_ext_ptr.upload(ft.ext_ptr.data(), ft.ext_ptr.size());
                    fv->fz_ext.upload(ft.ext.data(), ft.ext.size());
                    fv->fz_tile_cls.upload(ft.tile_cls.data(), ft.tile_cls.size());
                    fv->fz_cls_off.upload(ft.cls_off.data(), ft.cls_off.size());
                    fv->fz_pool.upload(ft.pool.data(), ft.pool.size());
                    fv->fz_max_ext = ft.max_ext;
                    fv->fz_max_grad = ft.max_grad;
                    fv->fz_max_faces = ft.max_faces;
                    fv->fz_classes = (int)ft.cls_off.size();
                }
            }
        }
        {
            // per cell: sum of its LSQ weights over non-boundary faces, and of its aux weights over all
            std::vector<double> ws((size_t)h.n_cells * 6, 0.0);
            for (int c = 0; c < h.n_cells; c++)
                for (int i = h.cone_ptr[c]; i < h.cone_ptr[c + 1]; i++) {
                    const size_t slot = (size_t)h.cone_face[i] * 6 + 3 * h.cone_side[i];
                    for (int d = 0; d < h.dim; d++) {
                        if (lsq && !h.face_boundary[h.cone_face[i]]) ws[6 * (size_t)c + d] += h.cgrad[slot + d];
                        if (dif) ws[6 * (size_t)c + 3 + d] += h.fgrad[slot + d];
                    }
                }
            fv->wsum.upload(ws.data(), ws.size());
        }

        {
            // the two parts of a split RHS: the cells that need no halo row (their aux, and the gradients
            // whose stencils hold none) and the rest
            std::vector<int32_t> ae, al, ge, gl;
            for (int c = 0; c < h.n_cells; c++) {
                const auto is_halo = [&](int x) { return h.kind[x] == ABL_CELL_HALO || h.kind[x] == ABL_CELL_HALO_OUTER; };
                bool early = !is_halo(c);
                (early ? ae : al).push_back(c);
                for (int i = h.cone_ptr[c]; i < h.cone_ptr[c + 1] && early; i++) early = !is_halo(h.cone_nbr[i]);
                (early ? ge : gl).push_back(c);
            }
            fv->aux_early.upload(ae.data(), ae.size());
            fv->aux_late.upload(al.data(), al.size());
            fv->grad_early.upload(ge.data(), ge.size());
            fv->grad_late.upload(gl.data(), gl.size());
        }
        fv->aux.alloc((size_t)fv->n_cells * fv->naux);
        {
            std::vector<double> a0((size_t)fv->n_cells * fv->naux, 0.0);
            for (int c = 0; c < fv->n_cells; c++) a0[(size_t)c * fv->naux] = 300.0;  // temperature guess (TChem::TemperatureFunction uses 300 K)
            ABL_CUDA(cudaMemcpy(fv->aux.p, a0.data(), a0.size() * sizeof(double), cudaMemcpyHostToDevice));
        }
        if (lsq) {
            fv->grad64.alloc((size_t)fv->n_cells * round_up(fv->nc * fv->dim, 2));
            if (fv->ns == 0 || fv->mixed_species) fv->grad32.alloc((size_t)fv->n_cells * round_up(fv->nc * fv->dim, 4));
        }
        if (dif) {
            fv->agrad64.alloc((size_t)fv->n_cells * round_up(fv->naux * fv->dim, 2));
            if (fv->ns == 0 || fv->mixed_species) fv->agrad32.alloc((size_t)fv->n_cells * round_up(fv->naux * fv->dim, 4));
        }
        fv->status.alloc(1);
        fv->status.zero();
        {
            // boundary ghosts (one face each): interior neighbour and the unit normal out of the domain;
            // per cell the smallest centroid-to-face-centroid distance (the CFL length)
            std::vector<int32_t> gc, gn, gb;
            std::vector<double> gnorm, rm(h.n_cells, 0.0);
            for (int c = 0; c < h.n_cells; c++) {
                double r = 1e300;
                for (int i = h.cone_ptr[c]; i < h.cone_ptr[c + 1]; i++) {
                    const double* x = h.fdx.data() + 6 * (size_t)h.cone_face[i] + 3 * h.cone_side[i];
                    r = std::min(r, std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]));
                }
                rm[c] = r;
                if (h.kind[c] != ABL_CELL_BOUNDARY) continue;
                const int i = h.cone_ptr[c], f = h.cone_face[i];
                const double* n = mesh->face_normal + 3 * (size_t)f;
                const double a = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
                const double sgn = h.cone_side[i] == 1 ? 1.0 : -1.0;  // the normal points left -> right
                gc.push_back(c);
                gn.push_back(h.cone_nbr[i]);
                gb.push_back(0);
                for (int d = 0; d < 3; d++) gnorm.push_back(d < h.dim ? sgn * n[d] / a : 0.0);
            }
            fv->n_ghost = (int)gc.size();
            {
                // segments of ghosts sharing an interior neighbour, ghosts ascending inside each
                std::vector<int> order(gc.size());
                for (size_t j = 0; j < order.size(); j++) order[j] = (int)j;
                std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return gn[a] < gn[b]; });
                std::vector<int> sp{0}, sn;
                for (size_t q = 0; q < order.size(); q++) {
                    if (q > 0 && gn[order[q]] != gn[order[q - 1]]) sp.push_back((int)q);
                    if (q == 0 || gn[order[q]] != gn[order[q - 1]]) sn.push_back(gn[order[q]]);
                }
                if (!order.empty()) sp.push_back((int)order.size());
                fv->n_gseg = (int)sn.size();
                fv->gseg_ptr.upload(sp.data(), sp.size());
                fv->gseg_nbr.upload(sn.data(), sn.size());
                fv->gseg_ghost.upload(order.data(), order.size());
            }
            fv->ghost_cell.upload(gc.data(), gc.size());
            fv->ghost_nbr.upload(gn.data(), gn.size());
            fv->ghost_bc.upload(gb.data(), gb.size());
            fv->ghost_normal.upload(gnorm.data(), gnorm.size());
            fv->rmin.upload(rm.data(), rm.size());
            abl_bc outflow{};
            outflow.kind = ABL_BC_OUTFLOW;
            fv->bc_table.upload(&outflow, 1);
            fv->dt_bits.alloc(1);
        }

        DevMesh& M = fv->mesh;
        M.dim = fv->dim;
        M.n_cells = fv->n_cells;
        M.n_faces = fv->n_faces;
        M.n_flux_faces = fv->n_flux_faces;
        M.face_cells = fv->face_cells.p;
        M.kind = fv->kind.p;
        M.cone_ptr = fv->cone_ptr.p;
        M.cone = fv->cone.p;
        M.fdx = fv->fdx.p;
        M.ivol = fv->ivol.p;
        M.cgrad = fv->cgrad.p;
        M.fgrad = fv->fgrad.p;
        M.n_tiles = tl.n_tiles;
        M.tile_cell_ptr = fv->tile_cell_ptr.p;
        M.tile_cells = fv->tile_cells.p;
        M.tile_face_ptr = fv->tile_face_ptr.p;
        M.tf_cells = fv->tf_cells.p;
        M.tf_geo = fv->tf_geo.p;
        M.tc_fptr = fv->tc_fptr.p;
        M.tc_face = fv->tc_face.p;
        M.tf_adj = fv->tf_adj.p;
        M.col_base = fv->col_base.p;
        M.col_start = fv->col_start.p;
        M.tf_slot = fv->tf_slot.p;
        M.tf_nb = fv->tf_nb.p;
        M.face_nb = fv->face_nb.p;
        M.n_nonowned = (int)fv->nonowned.n;
        M.nonowned = fv->nonowned.p;
        M.wsum = fv->wsum.p;
        M.cwa = fv->cwa.p;
        M.cv = fv->cv.p;
        M.cwar = fv->cwar.p;
        M.cwa32 = fv->cwa32.p;
        M.cv32 = fv->cv32.p;
        M.tf_geo32 = fv->tf_geo32.p;
        M.cone_cls = fv->n_cone_classes ? fv->cone_cls.p : nullptr;
        M.tf_gcls = fv->n_geo_classes ? fv->tf_gcls.p : nullptr;
        M.max_cone = fv->max_cone;
        ABL_CUDA(cudaDeviceSynchronize());
        *out = fv.release();
    });
}

int abl_fv_destroy(abl_fv* fv) {
    if (!fv) return ABL_OK;
    cudaSetDevice(fv->device);
    for (auto& e : fv->marks)
        if (e) cudaEventDestroy(e);
    if (fv->host_stream) {
        cudaStreamDestroy(fv->host_stream);
        cudaStreamDestroy(fv->copy_stream);
        cudaStreamDestroy(fv->out_stream);
        cudaEventDestroy(fv->ev_u);
        for (auto& e : fv->ev_in) cudaEventDestroy(e);
        for (auto& e : fv->ev_chunk) cudaEventDestroy(e);
    }
    delete fv;
    return ABL_OK;
}

int abl_fv_profile(abl_fv* fv, int enable) {
    if (!fv) return fail(ABL_ERR_INVALID_ARGUMENT, "handle is NULL");
    fv->profile = enable != 0;
    fv->n_marks = 0;
    return ABL_OK;
}

int abl_fv_profile_read(abl_fv* fv, int32_t* n, float* ms, char* names) {
    return guarded([&] {
        if (!fv || !n || !ms || !names) throw std::invalid_argument("NULL argument");
        *n = 0;
        if (fv->n_marks < 2) return;
        ABL_CUDA(cudaSetDevice(fv->device));
        ABL_CUDA(cudaEventSynchronize(fv->marks[fv->n_marks - 1]));
        for (int i = 0; i + 1 < fv->n_marks; i++) {
            ABL_CUDA(cudaEventElapsedTime(&ms[i], fv->marks[i], fv->marks[i + 1]));
            std::snprintf(names + 32 * i, 32, "%s", fv->mark_names[i]);
        }
        *n = fv->n_marks - 1;
    });
}

int abl_fv_sizes(const abl_fv* fv, int32_t* nc, int32_t* naux, int32_t* n_cells, int32_t* n_faces) {
    if (!fv) return fail(ABL_ERR_INVALID_ARGUMENT, "handle is NULL");
    if (nc) *nc = fv->nc_user;
    if (naux) *naux = fv->naux_user;
    if (n_cells) *n_cells = fv->n_cells;
    if (n_faces) *n_faces = fv->n_faces;
    return ABL_OK;
}

int abl_fv_record_classes(const abl_fv* fv, int32_t* weight_classes, int32_t* geometry_classes) {
    if (!fv) return fail(ABL_ERR_INVALID_ARGUMENT, "handle is NULL");
    if (weight_classes) *weight_classes = fv->n_cone_classes;
    if (geometry_classes) *geometry_classes = fv->n_geo_classes;
    return ABL_OK;
}

int abl_fv_fused_info(const abl_fv* fv, int32_t* fp64, int32_t* mixed, int32_t* classes, int32_t* max_ext) {
    if (!fv) return fail(ABL_ERR_INVALID_ARGUMENT, "handle is NULL");
    if (fp64) *fp64 = fv->fused_ok[0] ? 1 : 0;
    if (mixed) *mixed = fv->fused_ok[1] ? 1 : 0;
    if (classes) *classes = fv->fz_classes;
    if (max_ext) *max_ext = fv->fz_max_ext;
    return ABL_OK;
}

int abl_fv_rhs(abl_fv* fv, double time, const double* U_dev, double* F_dev, int precision, void* stream) {
    (void)time;
    return guarded([&] {
        if (!fv || !U_dev || !F_dev) throw std::invalid_argument("abl_fv_rhs: NULL argument");
        const int overwrite = (precision & ABL_RHS_OVERWRITE) != 0;
        precision &= ~ABL_RHS_OVERWRITE;
        if (precision != ABL_PRECISION_FP64 && precision != ABL_PRECISION_MIXED) throw std::invalid_argument("unknown precision");
        ABL_CUDA(cudaSetDevice(fv->device));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (fv->pad == 0) {
            dispatch_rhs(fv, U_dev, F_dev, precision, overwrite, s);
            return;
        }
        // a padded count: the instance's rows in scratch, the residual back into the caller's rows
        const double* U = pad_in(fv, fv->pU, U_dev, s);
        double* F = pad_out(fv, fv->pF, s);
        dispatch_rhs(fv, U, F, precision, 1, s);
        unpad_rows(fv, F, F_dev, true, !overwrite, s);
    });
}

int abl_fv_rhs_phase(abl_fv* fv, double time, const double* U_dev, double* F_dev, int precision, int phase, void* stream) {
    struct PhaseOff {
        abl_fv* fv;
        ~PhaseOff() { fv->rhs_phase = -1; }
    };
    return guarded([&] {
        if (!fv || !U_dev || !F_dev) throw std::invalid_argument("abl_fv_rhs_phase: NULL argument");
        if (phase != ABL_RHS_PHASE_INTERIOR && phase != ABL_RHS_PHASE_REST) throw std::invalid_argument("abl_fv_rhs_phase: unknown phase");
        if (fv->pad) {
            // a padded count converts every row at once: everything runs in the second phase
            if (phase == ABL_RHS_PHASE_INTERIOR) return;
            const int rc = abl_fv_rhs(fv, time, U_dev, F_dev, precision, stream);
            if (rc != ABL_OK) throw AblError(rc, g_last_error);
            return;
        }
        PhaseOff off{fv};
        fv->rhs_phase = phase;
        const int rc = abl_fv_rhs(fv, time, U_dev, F_dev, precision, stream);
        if (rc != ABL_OK) throw AblError(rc, g_last_error);
    });
}

int abl_fv_jvp(abl_fv* fv, double time, const double* U_dev, const double* dU_dev, double* F_dev, double* dF_dev, void* stream) {
    (void)time;
    return guarded([&] {
        if (!fv || !U_dev || !dU_dev || !dF_dev) throw std::invalid_argument("abl_fv_jvp: NULL argument");
        ABL_CUDA(cudaSetDevice(fv->device));
        // value + tangent gradient pairs, allocated on first use
        if (fv->need_state_grad && fv->gradD.n == 0) fv->gradD.alloc((size_t)fv->n_cells * fv->nc * fv->dim * 2);
        if (fv->need_aux_grad && fv->agradD.n == 0) fv->agradD.alloc((size_t)fv->n_cells * fv->naux * fv->dim * 2);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (fv->pad == 0) {
            dispatch_jvp(fv, U_dev, dU_dev, F_dev, dF_dev, s);
            return;
        }
        const double* U = pad_in(fv, fv->pU, U_dev, s);
        const double* dU = pad_in(fv, fv->pdU, dU_dev, s);
        double* F = F_dev ? pad_out(fv, fv->pF, s) : nullptr;
        double* dF = pad_out(fv, fv->pdF, s);
        dispatch_jvp(fv, U, dU, F, dF, s);
        if (F_dev) unpad_rows(fv, F, F_dev, true, true, s);
        unpad_rows(fv, dF, dF_dev, true, true, s);
    });
}

int abl_fv_jvp_host(abl_fv* fv, double time, const double* U_host, const double* dU_host, double* F_host, double* dF_host) {
    return guarded([&] {
        if (!fv || !U_host || !dU_host || !dF_host) throw std::invalid_argument("abl_fv_jvp_host: NULL argument");
        ABL_CUDA(cudaSetDevice(fv->device));
        const size_t n = (size_t)fv->n_cells * fv->nc_user;
        if (fv->hU.n != n) fv->hU.alloc(n);
        if (fv->hdU.n != n) fv->hdU.alloc(n);
        if (fv->hdF.n != n) fv->hdF.alloc(n);
        if (F_host && fv->hF.n != n) fv->hF.alloc(n);
        ABL_CUDA(cudaMemcpy(fv->hU.p, U_host, n * sizeof(double), cudaMemcpyHostToDevice));
        ABL_CUDA(cudaMemcpy(fv->hdU.p, dU_host, n * sizeof(double), cudaMemcpyHostToDevice));
        ABL_CUDA(cudaMemcpy(fv->hdF.p, dF_host, n * sizeof(double), cudaMemcpyHostToDevice));
        if (F_host) ABL_CUDA(cudaMemcpy(fv->hF.p, F_host, n * sizeof(double), cudaMemcpyHostToDevice));
        int rc = abl_fv_jvp(fv, time, fv->hU.p, fv->hdU.p, F_host ? fv->hF.p : nullptr, fv->hdF.p, nullptr);
        if (rc != ABL_OK) throw AblError(rc, g_last_error);
        ABL_CUDA(cudaMemcpy(dF_host, fv->hdF.p, n * sizeof(double), cudaMemcpyDeviceToHost));
        if (F_host) ABL_CUDA(cudaMemcpy(F_host, fv->hF.p, n * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

int abl_fv_vjp(abl_fv* fv, double time, const double* U_dev, const double* Fbar_dev, double* Ubar_dev, void* stream) {
    (void)time;
    return guarded([&] {
        if (!fv || !U_dev || !Fbar_dev || !Ubar_dev) throw std::invalid_argument("abl_fv_vjp: NULL argument");
        ABL_CUDA(cudaSetDevice(fv->device));
        // per-cell adjoint records, allocated on first use
        const size_t n = (size_t)fv->n_cells;
        if (fv->adj_ub.n == 0) {
            if (fv->need_state_grad) fv->adj_gb.alloc(n * round_up(fv->nc * fv->dim, 2));
            if (fv->need_aux_grad) fv->adj_gab.alloc(n * round_up(fv->naux * fv->dim, 2));
            fv->adj_beta.alloc(n * fv->nc);
            fv->adj_fstar.alloc(n * fv->nc);
            fv->adj_ab.alloc(n * fv->naux);
            fv->adj_nb.alloc((size_t)std::max(fv->n_nb, 1) * (fv->nc + fv->nc * fv->dim + fv->naux + fv->naux * fv->dim));
            fv->adj_ub.alloc(n * fv->nc);
            if (fv->need_state_grad) {
                fv->adj_graw.alloc(n * round_up(fv->nc * fv->dim, 2));
                fv->adj_phi.alloc(n * fv->nc);
                fv->adj_ist.alloc(n * fv->nc);
            }
        }
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (fv->pad == 0) {
            dispatch_vjp(fv, U_dev, Fbar_dev, Ubar_dev, s);
            return;
        }
        // every cell's adjoint row (boundary ghosts and halos included) goes back to the caller
        const double* U = pad_in(fv, fv->pU, U_dev, s);
        const double* Fb = pad_in(fv, fv->pF, Fbar_dev, s);
        double* Ub = pad_out(fv, fv->pUb, s);
        dispatch_vjp(fv, U, Fb, Ub, s);
        unpad_rows(fv, Ub, Ubar_dev, false, true, s);
    });
}

int abl_fv_vjp_host(abl_fv* fv, double time, const double* U_host, const double* Fbar_host, double* Ubar_host) {
    return guarded([&] {
        if (!fv || !U_host || !Fbar_host || !Ubar_host) throw std::invalid_argument("abl_fv_vjp_host: NULL argument");
        ABL_CUDA(cudaSetDevice(fv->device));
        const size_t n = (size_t)fv->n_cells * fv->nc_user;
        if (fv->hU.n != n) fv->hU.alloc(n);
        if (fv->hdU.n != n) fv->hdU.alloc(n);
        if (fv->hdF.n != n) fv->hdF.alloc(n);
        ABL_CUDA(cudaMemcpy(fv->hU.p, U_host, n * sizeof(double), cudaMemcpyHostToDevice));
        ABL_CUDA(cudaMemcpy(fv->hdF.p, Fbar_host, n * sizeof(double), cudaMemcpyHostToDevice));
        ABL_CUDA(cudaMemcpy(fv->hdU.p, Ubar_host, n * sizeof(double), cudaMemcpyHostToDevice));
        int rc = abl_fv_vjp(fv, time, fv->hU.p, fv->hdF.p, fv->hdU.p, nullptr);
        if (rc != ABL_OK) throw AblError(rc, g_last_error);
        ABL_CUDA(cudaMemcpy(Ubar_host, fv->hdU.p, n * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

int abl_fv_update_aux(abl_fv* fv, const double* U_dev, void* stream) {
    return guarded([&] {
        if (!fv || !U_dev) throw std::invalid_argument("abl_fv_update_aux: NULL argument");
        ABL_CUDA(cudaSetDevice(fv->device));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const double* U = pad_in(fv, fv->pU, U_dev, s);
        ABL_DISPATCH(fv, run_aux, U, s);
    });
}

int abl_fv_update_aux_host(abl_fv* fv, const double* U_host) {
    return guarded([&] {
        if (!fv || !U_host) throw std::invalid_argument("abl_fv_update_aux_host: NULL argument");
        ABL_CUDA(cudaSetDevice(fv->device));
        const size_t n = (size_t)fv->n_cells * fv->nc_user;
        if (fv->hU.n != n) fv->hU.alloc(n);
        ABL_CUDA(cudaMemcpy(fv->hU.p, U_host, n * sizeof(double), cudaMemcpyHostToDevice));
        int rc = abl_fv_update_aux(fv, fv->hU.p, nullptr);
        if (rc != ABL_OK) throw AblError(rc, g_last_error);
        ABL_CUDA(cudaDeviceSynchronize());
    });
}

int abl_fv_rhs_host(abl_fv* fv, double time, const double* U_host, double* F_host, int precision) {
    struct PipeOff {
        abl_fv* fv;
        ~PipeOff() { fv->pipe_active = false; }
    };
    return guarded([&] {
        if (!fv || !U_host || !F_host) throw std::invalid_argument("abl_fv_rhs_host: NULL argument");
        ABL_CUDA(cudaSetDevice(fv->device));
        const size_t n = (size_t)fv->n_cells * fv->nc_user;
        if (fv->hU.n != n) fv->hU.alloc(n);
        if (fv->hF.n != n) fv->hF.alloc(n);
        if (fv->pad) {
            // a padded count: plain copies around the device call (no chunked overlap)
            ABL_CUDA(cudaMemcpy(fv->hU.p, U_host, n * sizeof(double), cudaMemcpyHostToDevice));
            ABL_CUDA(cudaMemcpy(fv->hF.p, F_host, n * sizeof(double), cudaMemcpyHostToDevice));
            int rc = abl_fv_rhs(fv, time, fv->hU.p, fv->hF.p, precision & ~ABL_RHS_OVERWRITE, nullptr);
            if (rc != ABL_OK) throw AblError(rc, g_last_error);
            ABL_CUDA(cudaMemcpy(F_host, fv->hF.p, n * sizeof(double), cudaMemcpyDeviceToHost));
            return;
        }
        if (!fv->host_stream) {
            ABL_CUDA(cudaStreamCreateWithFlags(&fv->host_stream, cudaStreamNonBlocking));
            ABL_CUDA(cudaStreamCreateWithFlags(&fv->copy_stream, cudaStreamNonBlocking));
            ABL_CUDA(cudaStreamCreateWithFlags(&fv->out_stream, cudaStreamNonBlocking));
            ABL_CUDA(cudaEventCreateWithFlags(&fv->ev_u, cudaEventDisableTiming));
            for (auto& e : fv->ev_in) ABL_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            for (auto& e : fv->ev_chunk) ABL_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        }
        // the RHS writes owned rows only: when they are one range, only that range of F travels
        const bool range = fv->owned_hi >= 0;
        const size_t f0 = range ? (size_t)fv->owned_lo * fv->nc : 0, f1 = range ? (size_t)fv->owned_hi * fv->nc : n;
        ABL_CUDA(cudaMemcpyAsync(fv->hU.p, U_host, n * sizeof(double), cudaMemcpyHostToDevice, fv->host_stream));
        ABL_CUDA(cudaEventRecord(fv->ev_u, fv->host_stream));
        // the residual's rows follow the state in the same copy direction, chunk by chunk
        ABL_CUDA(cudaStreamWaitEvent(fv->copy_stream, fv->ev_u, 0));
        if (fv->chunk_tile.empty()) {
            ABL_CUDA(cudaMemcpyAsync(fv->hF.p + f0, F_host + f0, (f1 - f0) * sizeof(double), cudaMemcpyHostToDevice, fv->copy_stream));
            ABL_CUDA(cudaEventRecord(fv->ev_in[0], fv->copy_stream));
        } else {
            for (size_t q = 0; q + 1 < fv->chunk_row.size(); q++) {
                const size_t r0 = (size_t)fv->chunk_row[q] * fv->nc, r1 = (size_t)fv->chunk_row[q + 1] * fv->nc;
                if (r1 > r0)
                    ABL_CUDA(cudaMemcpyAsync(fv->hF.p + r0, F_host + r0, (r1 - r0) * sizeof(double), cudaMemcpyHostToDevice, fv->copy_stream));
                ABL_CUDA(cudaEventRecord(fv->ev_in[q], fv->copy_stream));
            }
        }
        fv->pipe_active = true;
        fv->pipe_F_host = F_host;
        PipeOff off{fv};
        int rc = abl_fv_rhs(fv, time, fv->hU.p, fv->hF.p, precision & ~ABL_RHS_OVERWRITE, fv->host_stream);
        if (rc != ABL_OK) {
            cudaStreamSynchronize(fv->host_stream);
            cudaStreamSynchronize(fv->copy_stream);
            cudaStreamSynchronize(fv->out_stream);
            throw AblError(rc, g_last_error);
        }
        if (fv->chunk_tile.empty()) {
            ABL_CUDA(cudaEventRecord(fv->ev_chunk[0], fv->host_stream));
            ABL_CUDA(cudaStreamWaitEvent(fv->out_stream, fv->ev_chunk[0], 0));
            ABL_CUDA(cudaMemcpyAsync(F_host + f0, fv->hF.p + f0, (f1 - f0) * sizeof(double), cudaMemcpyDeviceToHost, fv->out_stream));
        }
        ABL_CUDA(cudaStreamSynchronize(fv->host_stream));
        ABL_CUDA(cudaStreamSynchronize(fv->copy_stream));
        ABL_CUDA(cudaStreamSynchronize(fv->out_stream));
    });
}

int abl_fv_get_aux(abl_fv* fv, double* aux_host) {
    return guarded([&] {
        if (!fv || !aux_host) throw std::invalid_argument("NULL argument");
        ABL_CUDA(cudaSetDevice(fv->device));
        if (fv->pad == 0) {
            ABL_CUDA(cudaMemcpy(aux_host, fv->aux.p, fv->aux.n * sizeof(double), cudaMemcpyDeviceToHost));
            return;
        }
        // rows [T, u | pad | Y] of the instance into the caller's [T, u | Y]
        std::vector<double> a(fv->aux.n);
        ABL_CUDA(cudaMemcpy(a.data(), fv->aux.p, a.size() * sizeof(double), cudaMemcpyDeviceToHost));
        const int ne = 1 + fv->dim;
        for (size_t c = 0; c < (size_t)fv->n_cells; c++)
            for (int k = 0; k < fv->naux_user; k++) aux_host[c * fv->naux_user + k] = a[c * fv->naux + (k < ne ? k : k + fv->pad)];
    });
}

int abl_fv_set_aux(abl_fv* fv, const double* aux_host) {
    return guarded([&] {
        if (!fv || !aux_host) throw std::invalid_argument("NULL argument");
        ABL_CUDA(cudaSetDevice(fv->device));
        if (fv->pad == 0) {
            ABL_CUDA(cudaMemcpy(fv->aux.p, aux_host, fv->aux.n * sizeof(double), cudaMemcpyHostToDevice));
            return;
        }
        std::vector<double> a(fv->aux.n, 0.0);
        const int ne = 1 + fv->dim;
        for (size_t c = 0; c < (size_t)fv->n_cells; c++)
            for (int k = 0; k < fv->naux_user; k++) a[c * fv->naux + (k < ne ? k : k + fv->pad)] = aux_host[c * fv->naux_user + k];
        ABL_CUDA(cudaMemcpy(fv->aux.p, a.data(), a.size() * sizeof(double), cudaMemcpyHostToDevice));
    });
}

int abl_fv_status(abl_fv* fv) {
    if (!fv) return fail(ABL_ERR_INVALID_ARGUMENT, "handle is NULL");
    int bits = 0;
    int rc = guarded([&] {
        ABL_CUDA(cudaSetDevice(fv->device));
        ABL_CUDA(cudaMemcpy(&bits, fv->status.p, sizeof(int), cudaMemcpyDeviceToHost));
        fv->status.zero();
    });
    if (rc != ABL_OK) return rc;
    int code = status_to_code(bits);
    if (code != ABL_OK) g_last_error = "device status word " + std::to_string(bits);
    return code;
}

int abl_fv_launch_count(const abl_fv* fv, int precision, int32_t* launches) {
    if (!fv || !launches) return fail(ABL_ERR_INVALID_ARGUMENT, "NULL argument");
    int n = 0;
    if (fv->need_aux) n++;
    const bool fused = fv->fused_ok[precision == ABL_PRECISION_MIXED && fv->ns == 0 ? 1 : 0];
    if (!fused && (fv->need_state_grad || fv->need_aux_grad)) n++;
    if (fv->mesh.n_tiles > 0) n++;
    if (fv->pad) n += 2;  // rows into the instance's width and back
    *launches = n;
    return ABL_OK;
}

int abl_flux_calculator_batch(int kind, double minf, double pgs_alpha, double gamma, int64_t n, const double* uL, const double* aL,
                              const double* rhoL, const double* pL, const double* uR, const double* aR, const double* rhoR,
                              const double* pR, double* mass_flux, double* p12, int32_t* direction) {
    return guarded([&] {
        if (n < 0 || (n > 0 && (!uL || !aL || !rhoL || !pL || !uR || !aR || !rhoR || !pR || !mass_flux || !direction)))
            throw std::invalid_argument("abl_flux_calculator_batch: NULL argument");
        if (kind < ABL_FLUX_OFF || kind > ABL_FLUX_RIEMANN) throw std::invalid_argument("unknown flux calculator");
        if (n == 0) return;
        Phys P{};
        P.flux = kind;
        P.minf = minf;
        P.alpha = pgs_alpha > 0 ? pgs_alpha : 1.0;
        P.gamma = gamma;
        DevBuf<double> in, outd;
        DevBuf<int32_t> dir;
        DevBuf<int> st;
        in.alloc(8 * (size_t)n);
        const double* src[8] = {uL, aL, rhoL, pL, uR, aR, rhoR, pR};
        for (int j = 0; j < 8; j++) ABL_CUDA(cudaMemcpy(in.p + j * n, src[j], n * sizeof(double), cudaMemcpyHostToDevice));
        outd.alloc(2 * (size_t)n);
        dir.alloc(n);
        st.alloc(1);
        st.zero();
        k_flux_batch<<<blocks_for(n, 128), 128>>>(P, n, in.p, in.p + n, in.p + 2 * n, in.p + 3 * n, in.p + 4 * n, in.p + 5 * n, in.p + 6 * n,
                                                  in.p + 7 * n, outd.p, p12 ? outd.p + n : nullptr, dir.p, st.p);
        check_launch();
        ABL_CUDA(cudaMemcpy(mass_flux, outd.p, n * sizeof(double), cudaMemcpyDeviceToHost));
        if (p12) ABL_CUDA(cudaMemcpy(p12, outd.p + n, n * sizeof(double), cudaMemcpyDeviceToHost));
        ABL_CUDA(cudaMemcpy(direction, dir.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
        int bits = 0;
        ABL_CUDA(cudaMemcpy(&bits, st.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (bits & kStatusRiemann) throw AblError(ABL_ERR_RIEMANN_NOT_CONVERGED, "Can't find pstar; Iteration not converging");
    });
}

int abl_eos_batch(const abl_physics_desc* physics, int dim, int property, int64_t n, const double* conserved, const double* T_in, double* out) {
    return guarded([&] {
        validate_physics(physics);
        if (dim < 1 || dim > 3) throw std::invalid_argument("dim must be 1, 2 or 3");
        if (property < ABL_PROP_PRESSURE || property > ABL_PROP_DENSITY) throw std::invalid_argument("unknown property");
        if (n < 0 || (n > 0 && (!conserved || !out))) throw std::invalid_argument("NULL argument");
        if (n == 0) return;
        Phys P = make_phys(physics);
        DevBuf<double> nasa7, mw, inv_mw, href;
        upload_species(physics, P, nasa7, mw, inv_mw, href);
        const int ns = physics->n_species;
        const int nc = 2 + dim + ns;
        const int psz = property == ABL_PROP_SPECIES_SENSIBLE_ENTHALPY ? ns : 1;
        DevBuf<double> u, t, o;
        DevBuf<int> st;
        u.upload(conserved, (size_t)n * nc);
        if (T_in) t.upload(T_in, n);
        o.alloc((size_t)n * (psz > 0 ? psz : 1));
        st.alloc(1);
        st.zero();
        const unsigned nb = blocks_for(n, 128);
        switch (dim) {
            case 1: k_eos_batch<1><<<nb, 128>>>(P, ns, property, n, u.p, T_in ? t.p : nullptr, o.p, st.p); break;
            case 2: k_eos_batch<2><<<nb, 128>>>(P, ns, property, n, u.p, T_in ? t.p : nullptr, o.p, st.p); break;
            default: k_eos_batch<3><<<nb, 128>>>(P, ns, property, n, u.p, T_in ? t.p : nullptr, o.p, st.p); break;
        }
        check_launch();
        if (psz > 0) ABL_CUDA(cudaMemcpy(out, o.p, (size_t)n * psz * sizeof(double), cudaMemcpyDeviceToHost));
        int bits = 0;
        ABL_CUDA(cudaMemcpy(&bits, st.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (bits & kStatusEos) throw AblError(ABL_ERR_EOS_NOT_CONVERGED, "temperature iteration did not converge");
    });
}

int abl_eos_batch_noalloc(const abl_physics_desc* physics, int dim, int property, int64_t n, const double* conserved_dev, const double* T_dev,
                          double* out_dev, void* stream) {
    return guarded([&] {
        validate_physics(physics);
        if (dim < 1 || dim > 3) throw std::invalid_argument("dim must be 1, 2 or 3");
        if (property < ABL_PROP_PRESSURE || property > ABL_PROP_DENSITY) throw std::invalid_argument("unknown property");
        if (n < 0 || (n > 0 && (!conserved_dev || !out_dev))) throw std::invalid_argument("NULL argument");
        const int ns = physics->n_species;
        if (ns > kNoAllocMaxSpecies)
            throw std::invalid_argument("abl_eos_batch_noalloc: " + std::to_string(ns) + " species exceed the " +
                                        std::to_string(kNoAllocMaxSpecies) + " its static scratch holds");
        // resolved before the n == 0 return, so a zero-length call loads the device code ahead of a pool
        // allocator's reservation
        unsigned char* scratch = noalloc_scratch();
        if (n == 0) return;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        // layout: nasa7 [ns][15] | mw [ns] | 1/mw [ns] | h_ref [ns] | status (int)
        double* d_nasa7 = reinterpret_cast<double*>(scratch);
        double* d_mw = d_nasa7 + 15 * kNoAllocMaxSpecies;
        double* d_imw = d_mw + kNoAllocMaxSpecies;
        double* d_href = d_imw + kNoAllocMaxSpecies;
        int* d_status = reinterpret_cast<int*>(d_href + kNoAllocMaxSpecies);
        static_assert((15 + 3) * kNoAllocMaxSpecies * sizeof(double) + sizeof(int) <= kNoAllocScratchBytes, "scratch too small");
        Phys P = make_phys(physics);
        if (physics->eos == ABL_EOS_NASA7) {
            std::vector<double> tables(18 * (size_t)ns);
            for (int k = 0; k < ns; k++) {
                if (!(physics->mw[k] > 0)) throw std::invalid_argument("molar mass must be positive");
                tables[15 * (size_t)ns + k] = physics->mw[k];
                tables[16 * (size_t)ns + k] = 1.0 / physics->mw[k];
                tables[17 * (size_t)ns + k] = host_h_molar(physics->nasa7 + 15 * k, kTref) / physics->mw[k];
            }
            std::memcpy(tables.data(), physics->nasa7, 15 * (size_t)ns * sizeof(double));
            // pageable host source: the copy is staged before cudaMemcpyAsync returns, so `tables` may go
            ABL_CUDA(cudaMemcpyAsync(d_nasa7, tables.data(), 15 * (size_t)ns * sizeof(double), cudaMemcpyHostToDevice, s));
            ABL_CUDA(cudaMemcpyAsync(d_mw, tables.data() + 15 * (size_t)ns, (size_t)ns * sizeof(double), cudaMemcpyHostToDevice, s));
            ABL_CUDA(cudaMemcpyAsync(d_imw, tables.data() + 16 * (size_t)ns, (size_t)ns * sizeof(double), cudaMemcpyHostToDevice, s));
            ABL_CUDA(cudaMemcpyAsync(d_href, tables.data() + 17 * (size_t)ns, (size_t)ns * sizeof(double), cudaMemcpyHostToDevice, s));
            P.nasa7 = d_nasa7;
            P.mw = d_mw;
            P.inv_mw = d_imw;
            P.href = d_href;
        }
        // the status word is the one scratch entry read before it is written: clear it every call
        ABL_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int), s));
        const unsigned nb = blocks_for(n, 128);
        switch (dim) {
            case 1: k_eos_batch<1><<<nb, 128, 0, s>>>(P, ns, property, n, conserved_dev, T_dev, out_dev, d_status); break;
            case 2: k_eos_batch<2><<<nb, 128, 0, s>>>(P, ns, property, n, conserved_dev, T_dev, out_dev, d_status); break;
            default: k_eos_batch<3><<<nb, 128, 0, s>>>(P, ns, property, n, conserved_dev, T_dev, out_dev, d_status); break;
        }
        check_launch();
        int bits = 0;
        ABL_CUDA(cudaMemcpyAsync(&bits, d_status, sizeof(int), cudaMemcpyDeviceToHost, s));
        ABL_CUDA(cudaStreamSynchronize(s));
        if (bits & kStatusEos) throw AblError(ABL_ERR_EOS_NOT_CONVERGED, "temperature iteration did not converge");
    });
}

int abl_fv_set_boundary(abl_fv* fv, int32_t n_bc, const abl_bc* table, const int32_t* cell_bc) {
    return guarded([&] {
        if (!fv || !table || n_bc < 1) throw std::invalid_argument("abl_fv_set_boundary: need a handle and at least one condition");
        require_exact_instance(fv, "abl_fv_set_boundary");
        for (int b = 0; b < n_bc; b++)
            if (table[b].kind < ABL_BC_OUTFLOW || table[b].kind > ABL_BC_NOSLIP_WALL)
                throw std::invalid_argument("abl_fv_set_boundary: unknown condition kind in entry " + std::to_string(b));
        ABL_CUDA(cudaSetDevice(fv->device));
        std::vector<int32_t> gc(fv->n_ghost), gb(fv->n_ghost, 0);
        if (fv->n_ghost) ABL_CUDA(cudaMemcpy(gc.data(), fv->ghost_cell.p, gc.size() * sizeof(int32_t), cudaMemcpyDeviceToHost));
        if (cell_bc)
            for (int j = 0; j < fv->n_ghost; j++) {
                gb[j] = cell_bc[gc[j]];
                if (gb[j] < 0 || gb[j] >= n_bc)
                    throw std::invalid_argument("abl_fv_set_boundary: boundary cell " + std::to_string(gc[j]) + " names no condition");
            }
        fv->bc_table.upload(table, n_bc);
        fv->ghost_bc.upload(gb.data(), gb.size());
        fv->n_bc = n_bc;
    });
}

}  // extern "C"

namespace {
GhostBC ghost_desc(abl_fv* fv) {
    return GhostBC{fv->n_ghost, fv->ghost_cell.p, fv->ghost_nbr.p, fv->ghost_normal.p, fv->ghost_bc.p, fv->bc_table.p};
}
template <int DIM, int NS>
void run_fill_ghosts(abl_fv* fv, double* U, cudaStream_t s) {
    if (fv->n_ghost == 0) return;
    k_fill_ghosts<DIM, NS><<<blocks_for(fv->n_ghost, 256), 256, 0, s>>>(ghost_desc(fv), U);
    check_launch();
}
template <int DIM, int NS>
void run_fill_ghosts_jvp(abl_fv* fv, double* dU, cudaStream_t s) {
    if (fv->n_ghost == 0) return;
    k_fill_ghosts<DIM, NS, 1><<<blocks_for(fv->n_ghost, 256), 256, 0, s>>>(ghost_desc(fv), dU);
    check_launch();
}
template <int DIM, int NS>
void run_fill_ghosts_vjp(abl_fv* fv, double* Ub, cudaStream_t s) {
    if (fv->n_ghost == 0) return;
    const size_t n = (size_t)fv->n_ghost * fv->nc;
    if (fv->ghost_vbar.n != n) fv->ghost_vbar.alloc(n);
    k_fill_ghosts_vjp<DIM, NS><<<blocks_for(fv->n_gseg, 256), 256, 0, s>>>(
        ghost_desc(fv), GhostSegments{fv->n_gseg, fv->gseg_ptr.p, fv->gseg_nbr.p, fv->gseg_ghost.p}, Ub, fv->ghost_vbar.p);
    check_launch();
    k_bc_value_reduce<><<<fv->n_bc, 256, 0, s>>>(fv->n_ghost, fv->ghost_bc.p, fv->nc, fv->ghost_vbar.p, fv->bc_vbar.p);
    check_launch();
}
template <int DIM, int NS>
void run_pressure_functional(abl_fv* fv, const double* U, double* Ub, cudaStream_t s) {
    k_pressure_functional<DIM, NS><<<blocks_for(fv->fn_n, 256), 256, 0, s>>>(fv->phys, fv->fn_n, fv->fn_cells.p, fv->fn_w.p, U, fv->fn_partial.p,
                                                                               Ub, fv->status.p);
    check_launch();
}
template <int DIM, int NS>
void run_cfl_dt(abl_fv* fv, const double* U, double cfl, cudaStream_t s) {
    // all bits set: above every positive double's bit pattern, the identity of the unsigned minimum
    ABL_CUDA(cudaMemsetAsync(fv->dt_bits.p, 0xff, sizeof(unsigned long long), s));
    k_cfl_dt<DIM, NS><<<blocks_for(fv->n_cells, 256), 256, 0, s>>>(fv->mesh, fv->phys, U, fv->rmin.p, cfl, fv->dt_bits.p, fv->status.p);
    check_launch();
}
template <int DIM, int NS>
void run_normalize(abl_fv* fv, double* U, cudaStream_t s) {
    if (NS == 0) return;
    k_normalize_species<DIM, NS><<<blocks_for(fv->n_cells, 256), 256, 0, s>>>(fv->mesh, U);
    check_launch();
}
void rk_stage(abl_fv* fv, double a, const double* U0, double b, const double* Us, double dt, const double* F, double* Uout, cudaStream_t s) {
    k_rk_stage<><<<blocks_for((int64_t)fv->n_cells * fv->nc, 256), 256, 0, s>>>(fv->kind.p, fv->nc, fv->n_cells, a, U0, b, Us, dt, F, Uout);
    check_launch();
}
// the same stage with the step taken from the CFL reduction's result on the device
void rk_stage_dev(abl_fv* fv, double a, const double* U0, double b, const double* Us, const double* F, double* Uout, double* time, cudaStream_t s) {
    k_rk_stage_dev<><<<blocks_for((int64_t)fv->n_cells * fv->nc, 256), 256, 0, s>>>(fv->kind.p, fv->nc, fv->n_cells, a, U0, b, Us, fv->dt_bits.p, F,
                                                                                   Uout, time);
    check_launch();
}
}  // namespace

extern "C" {

int abl_fv_fill_ghosts(abl_fv* fv, double time, double* U_dev, void* stream) {
    (void)time;
    return guarded([&] {
        if (!fv || !U_dev) throw std::invalid_argument("abl_fv_fill_ghosts: NULL argument");
        require_exact_instance(fv, "abl_fv_fill_ghosts");
        ABL_CUDA(cudaSetDevice(fv->device));
        ABL_DISPATCH_EXACT(fv, run_fill_ghosts, U_dev, static_cast<cudaStream_t>(stream));
    });
}

int abl_fv_set_jvp_mode(abl_fv* fv, int mode) {
    return guarded([&] {
        if (!fv) throw std::invalid_argument("abl_fv_set_jvp_mode: NULL handle");
        if (mode != ABL_JVP_EXACT && mode != ABL_JVP_FROZEN_LIMITER) throw std::invalid_argument("abl_fv_set_jvp_mode: unknown mode");
        fv->phys.jvp_frozen_limiter = mode == ABL_JVP_FROZEN_LIMITER;
    });
}

int abl_fv_fill_ghosts_jvp(abl_fv* fv, double* dU_dev, void* stream) {
    return guarded([&] {
        if (!fv || !dU_dev) throw std::invalid_argument("abl_fv_fill_ghosts_jvp: NULL argument");
        require_exact_instance(fv, "abl_fv_fill_ghosts_jvp");
        ABL_CUDA(cudaSetDevice(fv->device));
        ABL_DISPATCH_EXACT(fv, run_fill_ghosts_jvp, dU_dev, static_cast<cudaStream_t>(stream));
    });
}

int abl_fv_fill_ghosts_vjp(abl_fv* fv, double* Ubar_dev, double* value_bar_host, void* stream) {
    return guarded([&] {
        if (!fv || !Ubar_dev) throw std::invalid_argument("abl_fv_fill_ghosts_vjp: NULL argument");
        require_exact_instance(fv, "abl_fv_fill_ghosts_vjp");
        ABL_CUDA(cudaSetDevice(fv->device));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const size_t nv = (size_t)fv->n_bc * ABL_BC_MAX_COMPONENTS;
        if (fv->bc_vbar.n != nv) fv->bc_vbar.alloc(nv);
        ABL_CUDA(cudaMemsetAsync(fv->bc_vbar.p, 0, nv * sizeof(double), s));
        ABL_DISPATCH_EXACT(fv, run_fill_ghosts_vjp, Ubar_dev, s);
        if (value_bar_host) {
            std::vector<double> vb(nv);
            ABL_CUDA(cudaMemcpyAsync(vb.data(), fv->bc_vbar.p, nv * sizeof(double), cudaMemcpyDeviceToHost, s));
            ABL_CUDA(cudaStreamSynchronize(s));
            for (size_t k = 0; k < nv; k++) value_bar_host[k] += vb[k];
        }
    });
}

int abl_fv_set_pressure_functional(abl_fv* fv, int32_t n, const int32_t* cells, const double* weights) {
    return guarded([&] {
        if (!fv || n < 0 || (n > 0 && (!cells || !weights))) throw std::invalid_argument("abl_fv_set_pressure_functional: bad argument");
        require_exact_instance(fv, "abl_fv_set_pressure_functional");
        std::vector<uint8_t> seen(fv->n_cells, 0);
        for (int j = 0; j < n; j++) {
            if (cells[j] < 0 || cells[j] >= fv->n_cells)
                throw std::invalid_argument("abl_fv_set_pressure_functional: cell " + std::to_string(cells[j]) + " out of range");
            if (seen[cells[j]]++) throw std::invalid_argument("abl_fv_set_pressure_functional: cell " + std::to_string(cells[j]) + " listed twice");
        }
        ABL_CUDA(cudaSetDevice(fv->device));
        fv->fn_n = n;
        if (n == 0) return;
        fv->fn_cells.upload(cells, n);
        fv->fn_w.upload(weights, n);
        fv->fn_partial.alloc(blocks_for(n, 256));
    });
}

int abl_fv_pressure_functional(abl_fv* fv, const double* U_dev, double* J_host, double* Ubar_dev, void* stream) {
    return guarded([&] {
        if (!fv || !U_dev || !J_host) throw std::invalid_argument("abl_fv_pressure_functional: NULL argument");
        require_exact_instance(fv, "abl_fv_pressure_functional");
        ABL_CUDA(cudaSetDevice(fv->device));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        *J_host = 0.0;
        if (fv->fn_n == 0) return;
        ABL_DISPATCH_EXACT(fv, run_pressure_functional, U_dev, Ubar_dev, s);
        std::vector<double> part(blocks_for(fv->fn_n, 256));
        ABL_CUDA(cudaMemcpyAsync(part.data(), fv->fn_partial.p, part.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
        ABL_CUDA(cudaStreamSynchronize(s));
        double J = 0.0;
        for (double v : part) J += v;
        *J_host = J;
    });
}

int abl_fv_cfl_dt(abl_fv* fv, const double* U_dev, double cfl, double* dt_host, void* stream) {
    return guarded([&] {
        if (!fv || !U_dev || !dt_host) throw std::invalid_argument("abl_fv_cfl_dt: NULL argument");
        require_exact_instance(fv, "abl_fv_cfl_dt");
        if (!(cfl > 0)) throw std::invalid_argument("abl_fv_cfl_dt: cfl must be positive");
        ABL_CUDA(cudaSetDevice(fv->device));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        ABL_DISPATCH_EXACT(fv, run_cfl_dt, U_dev, cfl, s);
        double dt = 0;
        ABL_CUDA(cudaMemcpyAsync(&dt, fv->dt_bits.p, sizeof(double), cudaMemcpyDeviceToHost, s));
        ABL_CUDA(cudaStreamSynchronize(s));
        *dt_host = dt;
    });
}

int abl_fv_normalize_species(abl_fv* fv, double* U_dev, void* stream) {
    return guarded([&] {
        if (!fv || !U_dev) throw std::invalid_argument("abl_fv_normalize_species: NULL argument");
        require_exact_instance(fv, "abl_fv_normalize_species");
        ABL_CUDA(cudaSetDevice(fv->device));
        ABL_DISPATCH_EXACT(fv, run_normalize, U_dev, static_cast<cudaStream_t>(stream));
    });
}

int abl_fv_rk_stage(abl_fv* fv, double a, const double* U0_dev, double b, const double* Us_dev, double dt, const double* F_dev, double* Uout_dev,
                    void* stream) {
    return guarded([&] {
        if (!fv || !Us_dev || !F_dev || !Uout_dev || (a != 0.0 && !U0_dev)) throw std::invalid_argument("abl_fv_rk_stage: NULL argument");
        require_exact_instance(fv, "abl_fv_rk_stage");
        ABL_CUDA(cudaSetDevice(fv->device));
        rk_stage(fv, a, U0_dev, b, Us_dev, dt, F_dev, Uout_dev, static_cast<cudaStream_t>(stream));
    });
}

int abl_fv_step(abl_fv* fv, int scheme, double time, double dt, double* U_dev, int precision, void* stream) {
    return guarded([&] {
        if (!fv || !U_dev) throw std::invalid_argument("abl_fv_step: NULL argument");
        require_exact_instance(fv, "abl_fv_step");
        if (precision != ABL_PRECISION_FP64 && precision != ABL_PRECISION_MIXED) throw std::invalid_argument("unknown precision");
        if (scheme != ABL_STEP_EULER && scheme != ABL_STEP_SSPRK3) throw std::invalid_argument("abl_fv_step: unknown scheme");
        ABL_CUDA(cudaSetDevice(fv->device));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const size_t n = (size_t)fv->n_cells * fv->nc;
        if (fv->step_F.n != n) fv->step_F.alloc(n);
        double* F = fv->step_F.p;
        (void)time;
        ABL_DISPATCH_EXACT(fv, run_fill_ghosts, U_dev, s);
        dispatch_rhs(fv, U_dev, F, precision, 1, s);
        if (scheme == ABL_STEP_EULER) {
            rk_stage(fv, 0.0, nullptr, 1.0, U_dev, dt, F, U_dev, s);
        } else {
            // U1 = U + dt L(U); U1 = 3/4 U + 1/4 (U1 + dt L(U1)); U = 1/3 U + 2/3 (U1 + dt L(U1))
            if (fv->step_U1.n != n) fv->step_U1.alloc(n);
            double* U1 = fv->step_U1.p;
            ABL_CUDA(cudaMemcpyAsync(U1, U_dev, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
            rk_stage(fv, 0.0, nullptr, 1.0, U_dev, dt, F, U1, s);
            ABL_DISPATCH_EXACT(fv, run_fill_ghosts, U1, s);
            dispatch_rhs(fv, U1, F, precision, 1, s);
            rk_stage(fv, 0.75, U_dev, 0.25, U1, dt, F, U1, s);
            ABL_DISPATCH_EXACT(fv, run_fill_ghosts, U1, s);
            dispatch_rhs(fv, U1, F, precision, 1, s);
            rk_stage(fv, 1.0 / 3.0, U_dev, 2.0 / 3.0, U1, dt, F, U_dev, s);
        }
        ABL_DISPATCH_EXACT(fv, run_normalize, U_dev, s);
        ABL_DISPATCH_EXACT(fv, run_fill_ghosts, U_dev, s);
    });
}

int abl_fv_download_owned(abl_fv* fv, const double* src_dev, int width, double* host, void* stream) {
    return guarded([&] {
        if (!fv || !src_dev || !host || width <= 0) throw std::invalid_argument("abl_fv_download_owned: bad argument");
        ABL_CUDA(cudaSetDevice(fv->device));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const int64_t n = (int64_t)fv->owned_rows.n;
        if (n == 0) return;
        const size_t count = (size_t)n * width;
        if (fv->io_rows.n < count) fv->io_rows.alloc(count);
        k_rows<0><<<blocks_for(n * width, 256), 256, 0, s>>>(src_dev, width, fv->owned_rows.p, n, fv->io_rows.p);
        check_launch();
        ABL_CUDA(cudaMemcpyAsync(host, fv->io_rows.p, count * sizeof(double), cudaMemcpyDeviceToHost, s));
        ABL_CUDA(cudaStreamSynchronize(s));
    });
}

int abl_fv_upload_owned(abl_fv* fv, const double* host, int width, double* dst_dev, void* stream) {
    return guarded([&] {
        if (!fv || !dst_dev || !host || width <= 0) throw std::invalid_argument("abl_fv_upload_owned: bad argument");
        ABL_CUDA(cudaSetDevice(fv->device));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const int64_t n = (int64_t)fv->owned_rows.n;
        if (n == 0) return;
        const size_t count = (size_t)n * width;
        if (fv->io_rows.n < count) fv->io_rows.alloc(count);
        ABL_CUDA(cudaMemcpyAsync(fv->io_rows.p, host, count * sizeof(double), cudaMemcpyHostToDevice, s));
        k_rows<1><<<blocks_for(n * width, 256), 256, 0, s>>>(fv->io_rows.p, width, fv->owned_rows.p, n, dst_dev);
        check_launch();
        ABL_CUDA(cudaStreamSynchronize(s));
    });
}

int abl_fv_step_cfl(abl_fv* fv, int scheme, double cfl, double* U_dev, int precision, double* time_dev, void* stream) {
    return guarded([&] {
        if (!fv || !U_dev) throw std::invalid_argument("abl_fv_step_cfl: NULL argument");
        require_exact_instance(fv, "abl_fv_step_cfl");
        if (!(cfl > 0)) throw std::invalid_argument("abl_fv_step_cfl: cfl must be positive");
        if (precision != ABL_PRECISION_FP64 && precision != ABL_PRECISION_MIXED) throw std::invalid_argument("unknown precision");
        if (scheme != ABL_STEP_EULER && scheme != ABL_STEP_SSPRK3) throw std::invalid_argument("abl_fv_step_cfl: unknown scheme");
        ABL_CUDA(cudaSetDevice(fv->device));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const size_t n = (size_t)fv->n_cells * fv->nc;
        if (fv->step_F.n != n) fv->step_F.alloc(n);
        double* F = fv->step_F.p;
        // the CFL step of the state the step starts from, as abl_fv_cfl_dt computes it (ghosts filled first)
        ABL_DISPATCH_EXACT(fv, run_fill_ghosts, U_dev, s);
        ABL_DISPATCH_EXACT(fv, run_cfl_dt, U_dev, cfl, s);
        dispatch_rhs(fv, U_dev, F, precision, 1, s);
        if (scheme == ABL_STEP_EULER) {
            rk_stage_dev(fv, 0.0, nullptr, 1.0, U_dev, F, U_dev, time_dev, s);
        } else {
            if (fv->step_U1.n != n) fv->step_U1.alloc(n);
            double* U1 = fv->step_U1.p;
            ABL_CUDA(cudaMemcpyAsync(U1, U_dev, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
            rk_stage_dev(fv, 0.0, nullptr, 1.0, U_dev, F, U1, nullptr, s);
            ABL_DISPATCH_EXACT(fv, run_fill_ghosts, U1, s);
            dispatch_rhs(fv, U1, F, precision, 1, s);
            rk_stage_dev(fv, 0.75, U_dev, 0.25, U1, F, U1, nullptr, s);
            ABL_DISPATCH_EXACT(fv, run_fill_ghosts, U1, s);
            dispatch_rhs(fv, U1, F, precision, 1, s);
            rk_stage_dev(fv, 1.0 / 3.0, U_dev, 2.0 / 3.0, U1, F, U_dev, time_dev, s);
        }
        ABL_DISPATCH_EXACT(fv, run_normalize, U_dev, s);
        ABL_DISPATCH_EXACT(fv, run_fill_ghosts, U_dev, s);
    });
}

int abl_rows_gather(const double* src_dev, int width, const int32_t* idx_dev, int64_t n, double* dst_dev, void* stream) {
    return guarded([&] {
        if (n < 0 || width <= 0) throw std::invalid_argument("abl_rows_gather: bad size");
        if (n == 0) return;
        if (!src_dev || !idx_dev || !dst_dev) throw std::invalid_argument("abl_rows_gather: NULL argument");
        k_rows<0><<<blocks_for(n * width, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(src_dev, width, idx_dev, n, dst_dev);
        check_launch();
    });
}

int abl_rows_scatter_add(const double* src_dev, int width, const int32_t* idx_dev, int64_t n, double* dst_dev, void* stream) {
    return guarded([&] {
        if (n < 0 || width <= 0) throw std::invalid_argument("abl_rows_scatter_add: bad size");
        if (n == 0) return;
        if (!src_dev || !idx_dev || !dst_dev) throw std::invalid_argument("abl_rows_scatter_add: NULL argument");
        k_rows<2><<<blocks_for(n * width, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(src_dev, width, idx_dev, n, dst_dev);
        check_launch();
    });
}

int abl_rows_scatter(const double* src_dev, int width, const int32_t* idx_dev, int64_t n, double* dst_dev, void* stream) {
    return guarded([&] {
        if (n < 0 || width <= 0) throw std::invalid_argument("abl_rows_scatter: bad size");
        if (n == 0) return;
        if (!src_dev || !idx_dev || !dst_dev) throw std::invalid_argument("abl_rows_scatter: NULL argument");
        k_rows<1><<<blocks_for(n * width, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(src_dev, width, idx_dev, n, dst_dev);
        check_launch();
    });
}

}  // extern "C"
