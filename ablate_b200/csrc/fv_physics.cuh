// fv_physics.cuh -- device-side physics of the finite-volume RHS: flux calculators, equations of
// state, transport models and slope limiters, templated on the arithmetic type R (double for the
// FP64 path, float for the FP32 parts of the mixed path).
//
// Reference arithmetic restated (ABLATE 0.13.03):
//   Ausm                 src/finiteVolume/fluxCalculator/ausm.cpp:2-43
//   AusmpUp              src/finiteVolume/fluxCalculator/ausmpUp.cpp:5-96  (beta, Kp, Ku, sigma: ausmpUp.hpp:22-25)
//   Riemann              src/finiteVolume/fluxCalculator/riemann.cpp:6-36, riemannSolver.cpp:7-187
//   AverageFlux/OffFlux  src/finiteVolume/fluxCalculator/averageFlux.cpp:2-11, offFlux.cpp:2-9
//   PerfectGas           src/eos/perfectGas.cpp:49-197
//   TChem (NASA-7)       src/eos/tChem.cpp:119-148, 581-602; src/eos/tChem/temperature.cpp:21-97;
//                        sensibleInternalEnergyFcn.hpp:25-44; speedOfSound.cpp:23-51; pressureFcn.hpp:26-42
//   Constant/Sutherland  src/eos/transport/constant.cpp, sutherland.cpp (constants sutherland.hpp:23-27)
//   limiter              src/finiteVolume/cellInterpolant.cpp:282-328 (symmetric BAM form of PetscLimiterLimit)
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ablate_fv.h"
#include "fv_consts.hpp"
#include "fv_dual.cuh"
#include <type_traits>

namespace abl {

#define ABL_HD __host__ __device__ __forceinline__

// PetscMin/PetscMax semantics: plain ternary, a NaN operand resolves to the second argument.
template <class R>
ABL_HD R pmin(R a, R b) { return a < b ? a : b; }
template <class R>
ABL_HD R pmax(R a, R b) { return a < b ? b : a; }
template <class R>
ABL_HD R sqr(R a) { return a * a; }

// FP64 reciprocal: the hardware approximation of PTX rcp.approx.ftz.f64 (relative error about 2^-23)
// refined by two Newton-Raphson steps in residual form, e = 1 - x r by one fused multiply-add and
// r <- r + r e by another (Markstein, "IA-64 and Elementary Functions", 2000, ch. 8): the first step
// squares the relative error to about 2^-46, the second's residual is exact and leaves the result within
// one ulp of 1/x (mostly the correctly rounded value). Zero, infinite, NaN and extreme inputs (|x|
// outside 1e-300..1e300, where the approximation flushes subnormals) take the IEEE division, so their
// special values are exactly those of 1/x.
ABL_HD double rcp64(double x) {
#ifdef __CUDA_ARCH__
    const double ax = fabs(x);
    if (!(ax > 1e-300 && ax < 1e300)) return 1.0 / x;
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    r = fma(r, fma(-x, r, 1.0), r);
    r = fma(r, fma(-x, r, 1.0), r);
    return r;
#else
    return 1.0 / x;
#endif
}
ABL_HD float rcp64(float x) {
#ifdef __CUDA_ARCH__
    return __frcp_rn(x);  // IEEE round-to-nearest reciprocal without the general division path
#else
    return 1.0f / x;
#endif
}
ABL_HD double dsqrt(double x) { return sqrt(x); }
ABL_HD float dsqrt(float x) { return sqrtf(x); }
ABL_HD double dabs(double x) { return fabs(x); }
ABL_HD float dabs(float x) { return fabsf(x); }
ABL_HD double dpow(double a, double b) { return pow(a, b); }
ABL_HD float dpow(float a, float b) { return powf(a, b); }
ABL_HD double dsin(double x) { return sin(x); }
ABL_HD float dsin(float x) { return sinf(x); }
ABL_HD bool dfinite(double x) { return isfinite(x); }

// Physics parameters resident on the device (passed by value to kernels).
struct Phys {
    int32_t eos, ns, flux, recon, limiter, transport;
    int32_t advection, diffusion, sp_adv, sp_dif;
    int32_t sp_compact;  // species advection of the compact NS + species process (NA direction averages)
    int32_t jvp_frozen_limiter;  // tangent evaluations hold the limiter factor at its value (dphi = 0)
    double gamma, r_gas, minf, alpha, max_lim_grad;
    double k, mu, diff;
    const double* nasa7;  // [ns][15]
    const double* mw;     // [ns]
    const double* inv_mw; // [ns]
    const double* href;   // [ns] reference enthalpy at 298.15 K, J/kg
    const double* diff_k; // [ns] per-species constant diffusivities (Constant model with one per species), or null
};

constexpr double kRuniv = 8314.46261815324;  // J/(kmol K)
constexpr double kTref = 298.15;             // TChemBase::TREF (src/eos/tChemBase.hpp:150)

// ------------------------------------------------------------------------------------------------
// flux calculators
// ------------------------------------------------------------------------------------------------
template <class R>
ABL_HD int flux_ausm(R uL, R aL, R rhoL, R pL, R uR, R aR, R rhoR, R pR, R* mf, R* p12) {
    const R one = R(1), half = R(0.5), quarter = R(0.25), two = R(2);
    R Mm = uR * rcp64(aR), sMm, sPm;
    if (dabs(Mm) <= one) {
        sMm = -quarter * sqr(Mm - one);
        sPm = -(sMm) * (two + Mm);
    } else {
        sMm = half * (Mm - dabs(Mm));
        sPm = (sMm) / Mm;
    }
    R Mp = uL * rcp64(aL), sMp, sPp;
    if (dabs(Mp) <= one) {
        sMp = quarter * sqr(Mp + one);
        sPp = (sMp) * (two - Mp);
    } else {
        sMp = half * (Mp + dabs(Mp));
        sPp = (sMp) / Mp;
    }
    R m = sMm + sMp;
    int dir;
    if (m < R(0)) {
        *mf = m * aR * rhoR;
        dir = ABL_DIR_RIGHT;
    } else {
        *mf = m * aL * rhoL;
        dir = ABL_DIR_LEFT;
    }
    if (p12) *p12 = pR * sPm + pL * sPp;
    return dir;
}

template <class R>
struct Ausmpup {
    static ABL_HD R M1P(R m) { return R(0.5) * (m + dabs(m)); }
    static ABL_HD R M2P(R m) { return R(0.25) * sqr(m + R(1)); }
    static ABL_HD R M1M(R m) { return R(0.5) * (m - dabs(m)); }
    static ABL_HD R M2M(R m) { return R(-0.25) * sqr(m - R(1)); }
    static ABL_HD R M4P(R m) {
        const R beta = R(1.0 / 8.0);
        return dabs(m) >= R(1) ? M1P(m) : M2P(m) * (R(1) - R(16) * beta * M2M(m));
    }
    static ABL_HD R M4M(R m) {
        const R beta = R(1.0 / 8.0);
        return dabs(m) >= R(1) ? M1M(m) : M2M(m) * (R(1) + R(16) * beta * M2P(m));
    }
    static ABL_HD R P5P(R m, R fa) {
        if (dabs(m) >= R(1)) return M1P(m) / (m + R(1E-30));
        R alpha = R(3.0 / 16.0) * (R(-4) + R(5) * fa * fa);
        return M2P(m) * ((R(2) - m) - R(16) * alpha * m * M2M(m));
    }
    static ABL_HD R P5M(R m, R fa) {
        if (dabs(m) >= R(1)) return M1M(m) / (m + R(1E-30));
        R alpha = R(3.0 / 16.0) * (R(-4) + R(5) * fa * fa);
        return M2M(m) * ((R(-2) - m) + R(16) * alpha * m * M2P(m));
    }
};

template <class R>
ABL_HD int flux_ausmpup(R mInf, R pgsAlpha, R uL, R aL, R rhoL, R pL, R uR, R aR, R rhoR, R pR, R* mf, R* p12) {
    using A = Ausmpup<R>;
    const R Kp = R(0.25), Ku = R(0.75), sigma = R(0.25);
    R rho12 = R(0.5) * (rhoL + rhoR);
    R a12 = R(0.5) * (aL + aR) * rcp64(pgsAlpha);
    const R ia12 = rcp64(a12);
    R mL = uL * ia12;
    R mR = uR * ia12;
    R mBar2 = (sqr(uL) + sqr(uR)) * (R(0.5) * ia12 * ia12);
    R fa = R(1);
    if (mInf > R(0)) {
        R mInf2 = sqr(mInf);
        R mO2 = pmin(R(1), pmax(mBar2, mInf2));
        R mO = dsqrt(mO2);
        fa = mO * (R(2) - mO);
    }
    R m12 = A::M4P(mL) + A::M4M(mR) - (Kp * rcp64(fa)) * pmax(R(1) - (sigma * mBar2), R(0)) * (pR - pL) * rcp64(rho12 * a12 * a12 * pgsAlpha * pgsAlpha);
    int dir;
    if (m12 > R(0)) {
        dir = ABL_DIR_LEFT;
        *mf = a12 * m12 * rhoL;
    } else {
        dir = ABL_DIR_RIGHT;
        *mf = a12 * m12 * rhoR;
    }
    if (p12) {
        R p5Plus = A::P5P(mL, fa);
        R p5Minus = A::P5M(mR, fa);
        R v = p5Plus * pL + p5Minus * pR - Ku * p5Plus * p5Minus * rho12 * fa * a12 * a12 * pgsAlpha * pgsAlpha * (mR - mL);
        *p12 = v * rcp64(sqr(pgsAlpha));
    }
    return dir;
}

// exact Riemann solver for a single perfect gas (p0 = 0); the iteration count is capped as in the
// reference (MAXIT 100); on failure *ok is cleared (the reference throws).
template <class R>
ABL_HD void riemann_f(R pstar, R gamma, R gm1, R gp1, R p, R a, R rho, R* f0, R* f1) {
    if (pstar <= p) {
        R A = R(2) * a / gm1;
        R B = R(0.5) * gm1 / gamma;
        R pRatio = pstar / p;
        R pPow = dpow(pRatio, B);
        *f0 = A * (pPow - R(1));
        *f1 = A * B * pPow / pstar;
    } else {
        R A = R(2) / (gp1 * rho);
        R B = gm1 * p / gp1;
        R pFrac = A / (pstar + B);
        R pSqrt = dsqrt(pFrac);
        *f0 = (pstar - p) * pSqrt;
        *f1 = R(0.5) * pFrac * pSqrt * (R(2) * B + pstar + p) / A;
    }
}

template <class R>
ABL_HD int flux_riemann(R gamma, R uL, R aL, R rhoL, R pL, R uR, R aR, R rhoR, R pR, R* massFlux, R* p12out, bool* ok) {
    const R gm1 = gamma - R(1), gp1 = gamma + R(1);
    R pstar = aL + aR - (R(0.5) * gm1 * (uR - uL));
    pstar = pstar / ((aL / dpow(pL, R(0.5) * gm1 / gamma)) + (aR / dpow(pR, R(0.5) * gm1 / gamma)));
    pstar = dpow(pstar, R(2) * gamma / gm1);
    const R tol = R(1e-8);
    const R del_u = uR - uL;
    R pold, fL0, fL1, fR0, fR1;
    int i = 0;
    do {
        riemann_f(pstar, gamma, gm1, gp1, pL, aL, rhoL, &fL0, &fL1);
        riemann_f(pstar, gamma, gm1, gp1, pR, aR, rhoR, &fR0, &fR1);
        pold = pstar;
        pstar = pold - (fL0 + fR0 + del_u) / (fL1 + fR1);
        if (pstar < R(0)) pstar = R(1e-10);  // p0L, p0R = 0 < tiny
        i++;
    } while (dabs((pstar - pold) / pstar) > tol && i <= 100);
    if (i > 100) *ok = false;
    // riemannDirection (riemannSolver.cpp:32-156) with p0 = 0 and gammaL = gammaR
    R p12, uX, mfx;
    const R ustar = R(0.5) * (uL + uR + fR0 - fL0);
    if (ustar >= R(0)) {
        if (pstar <= pL) {
            R astar = aL * dpow(pstar / pL, (gm1 / (R(2) * gamma)));
            R STLR = ustar - astar;
            if (STLR >= R(0)) {
                if (uL - aL >= R(0)) {
                    mfx = rhoL * uL;
                    p12 = pL;
                    uX = uL;
                } else {
                    R base = (R(2) / gp1) + ((gm1 * uL) / (gp1 * aL));
                    R A = rhoL * dpow(base, (R(2) / gm1));
                    uX = R(2) / gp1 * (aL + (gm1 * uL / R(2)));
                    mfx = A * uX;
                    p12 = pL * dpow(base, (R(2) * gamma / gm1));
                }
            } else {
                mfx = rhoL * dpow(pstar / pL, R(1) / gamma) * ustar;
                p12 = pstar;
                uX = ustar;
            }
        } else {
            R A = dsqrt((gp1 * pstar / R(2) / gamma / pL) + (gm1 / R(2) / gamma));
            if (uL - (aL * A) >= R(0)) {
                mfx = rhoL * uL;
                p12 = pL;
                uX = uL;
            } else {
                R pRatio = pstar / pL;
                mfx = rhoL * (pRatio + (gm1 / gp1)) / (gm1 * pRatio / gp1 + R(1)) * ustar;
                p12 = pstar;
                uX = ustar;
            }
        }
    } else {
        if (pstar <= pR) {
            if (uR + aR >= R(0)) {
                R astar = aR * dpow(pstar / pR, (gm1 / (R(2) * gamma)));
                if (ustar + astar >= R(0)) {
                    mfx = rhoR * dpow(pstar / pR, R(1) / gamma) * ustar;
                    p12 = pstar;
                    uX = ustar;
                } else {
                    R base = (R(2) / gp1) - ((gm1 * uR) / (gp1 * aR));
                    R A = rhoR * dpow(base, (R(2) / gm1));
                    uX = R(2) / gp1 * (-aR + (gm1 * uR / R(2)));
                    mfx = A * uX;
                    p12 = pR * dpow(base, (R(2) * gamma / gm1));
                }
            } else {
                mfx = rhoR * uR;
                p12 = pR;
                uX = uR;
            }
        } else {
            R A = dsqrt((gp1 * pstar / R(2) / gamma / pR) + (gm1 / R(2) / gamma));
            if (uR + (aR * A) >= R(0)) {
                R pRatio = pstar / pR;
                mfx = rhoR * (pRatio + (gm1 / gp1)) / (gm1 * pRatio / gp1 + R(1)) * ustar;
                p12 = pstar;
                uX = ustar;
            } else {
                mfx = rhoR * uR;
                p12 = pR;
                uX = uR;
            }
        }
    }
    *massFlux = mfx;
    if (p12out) *p12out = p12;
    return uX > R(0) ? ABL_DIR_LEFT : ABL_DIR_RIGHT;
}

// Flux calculator fixed at compile time (FK >= 0) or chosen at run time from P.flux (FK < 0).
template <int FK, class R>
ABL_HD int flux_calc_k(const Phys& P, R uL, R aL, R rhoL, R pL, R uR, R aR, R rhoR, R pR, R* mf, R* p12, bool* ok);

template <class R>
ABL_HD int flux_calc(const Phys& P, R uL, R aL, R rhoL, R pL, R uR, R aR, R rhoR, R pR, R* mf, R* p12, bool* ok) {
    switch (P.flux) {
        case ABL_FLUX_AVERAGE:
            *mf = R(0.5) * (uL * rhoL + uR * rhoR);
            if (p12) *p12 = R(0.5) * (pL + pR);
            return ABL_DIR_NA;
        case ABL_FLUX_AUSM:
            return flux_ausm<R>(uL, aL, rhoL, pL, uR, aR, rhoR, pR, mf, p12);
        case ABL_FLUX_AUSMPUP:
            return flux_ausmpup<R>(R(P.minf), R(P.alpha), uL, aL, rhoL, pL, uR, aR, rhoR, pR, mf, p12);
        case ABL_FLUX_RIEMANN:
            return flux_riemann<R>(R(P.gamma), uL, aL, rhoL, pL, uR, aR, rhoR, pR, mf, p12, ok);
        default:
            *mf = R(0);
            if (p12) *p12 = R(0);
            return ABL_DIR_NA;
    }
}

template <int FK, class R>
ABL_HD int flux_calc_k(const Phys& P, R uL, R aL, R rhoL, R pL, R uR, R aR, R rhoR, R pR, R* mf, R* p12, bool* ok) {
    if constexpr (FK == ABL_FLUX_AUSM) return flux_ausm<R>(uL, aL, rhoL, pL, uR, aR, rhoR, pR, mf, p12);
    if constexpr (FK == ABL_FLUX_AUSMPUP) return flux_ausmpup<R>(R(P.minf), R(P.alpha), uL, aL, rhoL, pL, uR, aR, rhoR, pR, mf, p12);
    return flux_calc<R>(P, uL, aL, rhoL, pL, uR, aR, rhoR, pR, mf, p12, ok);
}

// Limiter fixed at compile time (LIM >= 0) or chosen at run time (LIM < 0).
template <int LIM, class R>
ABL_HD R limiter_k(int kind, R f);

// ------------------------------------------------------------------------------------------------
// Split form of the AUSM-family fluxes for the mixed-precision path.
//
// The face mass flux and pressure are each written exactly (in exact arithmetic) as a large central
// part plus a small dissipative part:
//   mass flux  m A = 1/2 rho_up (u_L + u_R).n        +  [upwinding and Mach-splitting terms] A
//   pressure   p12 = (p_L + p_R) / 2 / alpha^2       +  [P5/P terms times (p_L - p_R), (M_R - M_L)] / alpha^2
// The central parts are evaluated in FP64 (a handful of multiplies, no division or square root); the
// dissipative parts, which carry all of the sound speeds, Mach numbers, polynomial splittings and
// branches, in FP32. Every difference of nearly equal quantities (M_L - M_R, p_L - p_R, u_L - u_R) is
// formed from FP64 inputs before rounding to FP32, and the differences of splitting polynomials are
// evaluated as (M_L - M_R) times their divided difference, so the FP32 rounding error is relative to
// the small terms, not to the fluxes. The identities used are exact for the reference formulas:
//   AUSM  : M+(M) = M/2 + g(M), M-(M) = M/2 - g(M), g = M^2/4 + 1/4 (|M| <= 1), |M|/2 otherwise;
//           P+(M) + P-(M) = 1; P-(M) = (M^3 - 3M + 2)/4 on |M| <= 1
//   AUSM+ : M4+(m) = m/2 + g4(m), M4-(m) = m/2 - g4(m), g4 = m^4/8 + 3/8 (|m| < 1, beta = 1/8), |m|/2 otherwise;
//           P5+(m) + P5-(m) = 1; P5-(m) = 1/2 - (3/4 + a) m + (1/4 + 2a) m^3 - a m^5 on |m| < 1
struct SplitFlux {
    double mA_c;  // central mass flux times area (FP64)
    float mA_d;   // dissipative mass flux times area
    double p_c;   // central interface pressure (FP64)
    float p_d;    // dissipative interface pressure
    int dir;
};

// rho, p: face states (FP64); unA = u.n (velocity dotted with the area-weighted normal, FP64);
// a: sound speeds (FP32); area = |n| (FP32)
template <int KIND>
ABL_HD SplitFlux flux_split(const Phys& P, double rhoL, double pL, double unAL, float aL, double rhoR, double pR, double unAR, float aR,
                            float area) {
    SplitFlux r;
    const float iA = 1.0f / area;
    const float uL = float(unAL) * iA, uR = float(unAR) * iA;
    const float du = float(unAL - unAR) * iA;      // u_L - u_R, from the FP64 difference
    const float dp = float(0.5 * (pL - pR));       // (p_L - p_R) / 2
    const double pbar = 0.5 * (pL + pR);
    if constexpr (KIND == ABL_FLUX_AUSM) {
        // Ausm::AusmFunction (ausm.cpp:2-43) in split form
        const float ML = uL / aL, MR = uR / aR;
        const bool subL = fabsf(ML) <= 1.f, subR = fabsf(MR) <= 1.f;
        // g(ML) - g(MR)
        float dg;
        const float dM = du / aL + uR * (aR - aL) / (aL * aR);  // ML - MR
        if (subL && subR)
            dg = 0.25f * dM * (ML + MR);
        else
            dg = (subL ? 0.25f * ML * ML + 0.25f : 0.5f * fabsf(ML)) - (subR ? 0.25f * MR * MR + 0.25f : 0.5f * fabsf(MR));
        const float sMp = subL ? 0.25f * (ML + 1.f) * (ML + 1.f) : 0.5f * (ML + fabsf(ML));
        const float sMm = subR ? -0.25f * (MR - 1.f) * (MR - 1.f) : 0.5f * (MR - fabsf(MR));
        const float m = sMm + sMp;
        const bool left = !(m < 0.f);
        r.dir = left ? ABL_DIR_LEFT : ABL_DIR_RIGHT;
        const double rho_up = left ? rhoL : rhoR;
        const float a_up = left ? aL : aR;
        // m a_up = (uL + uR)/2 + [uR (aL - aR)/aR or uL (aR - aL)/aL]/2 + a_up (g(ML) - g(MR))
        const float skew = left ? 0.5f * uR * (aL - aR) / aR : 0.5f * uL * (aR - aL) / aL;
        r.mA_c = 0.5 * rho_up * (unAL + unAR);
        r.mA_d = float(rho_up) * (skew + a_up * dg) * area;
        // p12 = pbar (P+(ML) + P-(MR)) + dp (P+(ML) - P-(MR)), P+(ML) + P-(MR) = 1 + P-(MR) - P-(ML)
        const float sPp = subL ? sMp * (2.f - ML) : sMp / ML;
        const float sPm = subR ? -sMm * (2.f + MR) : sMm / MR;
        float dP;  // P-(MR) - P-(ML)
        if (subL && subR)
            dP = -dM * 0.25f * (ML * ML + ML * MR + MR * MR - 3.f);
        else
            dP = sPm - (subL ? 0.25f * (ML - 1.f) * (ML - 1.f) * (2.f + ML) : (0.5f * (ML - fabsf(ML))) / ML);
        r.p_c = pbar;
        r.p_d = float(pbar) * dP + dp * (sPp - sPm);
        return r;
    } else {
        // AusmpUp::AusmpUpFunction (ausmpUp.cpp:5-53) in split form
        const float alpha = float(P.alpha), mInf = float(P.minf);
        const float Kp = 0.25f, Ku = 0.75f, sigma = 0.25f;
        const float rho12 = float(0.5 * (rhoL + rhoR));
        const float a12 = 0.5f * (aL + aR) / alpha;
        const float mL = uL / a12, mR = uR / a12;
        const float dm = du / a12;  // mL - mR
        const float mBar2 = (uL * uL + uR * uR) / (2.f * a12 * a12);
        float fa = 1.f;
        if (mInf > 0.f) {
            const float mO2 = pmin(1.f, pmax(mBar2, mInf * mInf));
            const float mO = sqrtf(mO2);
            fa = mO * (2.f - mO);
        }
        const bool subL = fabsf(mL) < 1.f, subR = fabsf(mR) < 1.f;
        float dg;  // g4(mL) - g4(mR)
        if (subL && subR)
            dg = 0.125f * dm * (mL + mR) * (mL * mL + mR * mR);
        else
            dg = (subL ? 0.125f * mL * mL * mL * mL + 0.375f : 0.5f * fabsf(mL)) - (subR ? 0.125f * mR * mR * mR * mR + 0.375f : 0.5f * fabsf(mR));
        const float Mp = (Kp / fa) * pmax(1.f - sigma * mBar2, 0.f) * (-2.f * dp) / (rho12 * a12 * a12 * alpha * alpha);
        // m12 = (mL + mR)/2 + dg - Mp; the sign decides the upwind side
        const float m12 = 0.5f * (mL + mR) + dg - Mp;
        const bool left = m12 > 0.f;
        r.dir = left ? ABL_DIR_LEFT : ABL_DIR_RIGHT;
        const double rho_up = left ? rhoL : rhoR;
        // m a12 rho = rho (uL + uR)/2 + rho a12 (dg - Mp)
        r.mA_c = 0.5 * rho_up * (unAL + unAR);
        r.mA_d = float(rho_up) * a12 * (dg - Mp) * area;
        // P5 splittings
        using A = Ausmpup<float>;
        const float p5p = A::P5P(mL, fa), p5m = A::P5M(mR, fa);
        float dP;  // P5-(mR) - P5-(mL)
        if (subL && subR) {
            const float a5 = 3.f / 16.f * (-4.f + 5.f * fa * fa);
            const float s3 = mL * mL + mL * mR + mR * mR;
            const float s5 = mL * mL * mL * mL + mL * mL * mL * mR + mL * mL * mR * mR + mL * mR * mR * mR + mR * mR * mR * mR;
            dP = -dm * (-(0.75f + a5) + (0.25f + 2.f * a5) * s3 - a5 * s5);
        } else {
            dP = p5m - A::P5M(mL, fa);
        }
        const float ia2 = 1.f / (alpha * alpha);
        const float pu = -Ku * p5p * p5m * rho12 * fa * a12 * a12 * alpha * alpha * (-dm);  // (mR - mL) = -dm
        r.p_c = pbar / (double(P.alpha) * double(P.alpha));
        r.p_d = (float(pbar) * dP + dp * (p5p - p5m) + pu) * ia2;
        return r;
    }
}

// ------------------------------------------------------------------------------------------------
// NASA-7 mixture thermodynamics (always FP64: the secant temperature solve and the energies it
// differences need the full mantissa). Templated on the state scalar S (double, or Dual for the
// tangent kernels).
// ------------------------------------------------------------------------------------------------
// molar enthalpy (J/kmol) of species k: R T (a1 + a2 T/2 + a3 T^2/3 + a4 T^3/4 + a5 T^4/5 + a6/T)
template <class S>
ABL_HD S nasa_h_molar(const double* c, S T) {
    const double* a = (T < c[0]) ? c + 1 : c + 8;
    return kRuniv * T * (a[0] + T * (a[1] * 0.5 + T * (a[2] * (1.0 / 3.0) + T * (a[3] * 0.25 + T * a[4] * 0.2))) + a[5] / T);
}
template <class S>
ABL_HD S nasa_cp_molar(const double* c, S T) {
    const double* a = (T < c[0]) ? c + 1 : c + 8;
    return kRuniv * (a[0] + T * (a[1] + T * (a[2] + T * (a[3] + T * a[4]))));
}

// Y from densityYi with the reference's clipping (TChem::FillWorkingVectorFromDensityMassFractions,
// src/eos/tChem.cpp:581-602); ns may be a compile-time constant after inlining.
template <class S>
ABL_HD void fill_y(int ns, S rho, const S* rhoY, S* ys) {
    S sum = 0.0;
    const S irho = rcp64(rho);
ABL_UNROLL_MIXTURE
    for (int s = 0; s < ns - 1; s++) {
        S y = pmax(S(0.0), rhoY[s] * irho);
        y = pmin(S(1.0), y);
        ys[s] = y;
        sum += y;
    }
    if (sum > 1.0) {
ABL_UNROLL_MIXTURE
        for (int s = 0; s < ns - 1; s++) ys[s] /= sum;
        ys[ns - 1] = 0.0;
    } else {
        ys[ns - 1] = 1.0 - sum;
    }
}

// SensibleInternalEnergyFcn (src/eos/tChem/sensibleInternalEnergyFcn.hpp:25-44):
// e_s = sum_k Y_k (h_k(T)/W_k - h_ref,k - Ru T / W_k)
template <class S, class ST>
ABL_HD S e_sens(const Phys& P, int ns, const S* ys, ST T) {
    S e = 0;
ABL_UNROLL_MIXTURE
    for (int k = 0; k < ns; k++) e += (nasa_h_molar(P.nasa7 + 15 * k, T) * P.inv_mw[k] - P.href[k] - kRuniv * T * P.inv_mw[k]) * ys[k];
    return e;
}

// TChem Temperature_TemplateRun secant iteration (src/eos/tChem/temperature.cpp:21-97): seeds T0 =
// guess, T1 = T0 + 1, at most 100 steps to |e_ref - e(T)| <= 1e-8, T clamped >= 1 K, one restart from
// 1000 K; on failure *ok is cleared and the last iterate returned (the reference returns it silently).
ABL_HD double nasa_temperature(const Phys& P, int ns, const double* ys, double eRef, double Tguess, bool* ok) {
    const double EPS = 1E-8;
    const int ITMAX = 100;
    double t = Tguess, t2 = t;
    double f2 = eRef - e_sens(P, ns, ys, t);
    if (fabs(f2) <= EPS) return t;
    for (int pass = 0; pass < 2; pass++) {
        double t0, f0;
        if (pass == 0) {
            t0 = t2;
            f0 = f2;
        } else {
            t0 = 1000.;
            f0 = eRef - e_sens(P, ns, ys, t);  // evaluated at the current iterate, as the reference does
        }
        double t1 = t0 + 1;
        t = t1;
        double f1 = eRef - e_sens(P, ns, ys, t);
        for (int it = 0; it < ITMAX; it++) {
            t2 = t1 - f1 * (t1 - t0) / (f1 - f0 + 1E-30);
            t2 = fmax(1.0, t2);
            t = t2;
            f2 = eRef - e_sens(P, ns, ys, t);
            if (fabs(f2) <= EPS) return t2;
            t0 = t1;
            t1 = t2;
            f0 = f1;
            f1 = f2;
        }
    }
    *ok = false;
    return t2;
}

template <class S>
ABL_HD S mixture_cp(const Phys& P, int ns, const S* ys, S T) {
    S cp = 0;
ABL_UNROLL_MIXTURE
    for (int k = 0; k < ns; k++) cp += ys[k] * nasa_cp_molar(P.nasa7 + 15 * k, T) * P.inv_mw[k];
    return cp;
}
template <class S>
ABL_HD S mixture_mw(const Phys& P, int ns, const S* ys) {
    S iw = 0;
ABL_UNROLL_MIXTURE
    for (int k = 0; k < ns; k++) iw += ys[k] * P.inv_mw[k];
    return rcp64(iw);
}

// Mixture temperature for a state scalar S: the secant iteration on the values; for a Dual state the
// derivative follows from e_s(T, Y) = e_ref by the implicit-function theorem,
//   dT = (de_ref - sum_k de_s/dY_k dY_k) / (de_s/dT),  de_s/dT = sum_k Y_k (cp_k - Ru) / W_k = cv
template <int NSMAX, class S>
ABL_HD S nasa_temperature_s(const Phys& P, int ns, const S* ys, S eRef, double Tguess, bool* ok) {
    if constexpr (std::is_same<S, double>::value) {
        return nasa_temperature(P, ns, ys, eRef, Tguess, ok);
    } else {
        double yv[NSMAX > 0 ? NSMAX : 1];
        for (int k = 0; k < ns; k++) yv[k] = ys[k].v;
        const double T = nasa_temperature(P, ns, yv, eRef.v, Tguess, ok);
        const S res = e_sens(P, ns, ys, T) - eRef;  // derivative part: sum de_s/dY dY - de_ref
        double cv = 0;
        for (int k = 0; k < ns; k++) cv += yv[k] * (nasa_cp_molar(P.nasa7 + 15 * k, T) - kRuniv) * P.inv_mw[k];
        return S(T, -res.d / cv);
    }
}

// Decoded thermodynamic state of one face side (what AdvectionFlux pulls out of the EOS).
template <class S>
struct Decoded {
    S T, e, a, p;
};

// Internal energy recovery e = E/rho - |u|^2/2 (always FP64).
template <int DIM, class S>
ABL_HD S internal_energy(const S* U) {
    const S irho = rcp64(U[0]);
    S ke = 0.0;
#pragma unroll
    for (int i = 0; i < DIM; i++) ke += sqr(U[2 + i] * irho);
    return U[1] * irho - 0.5 * ke;
}

// Decode with the *TemperatureFunction variants at T(U, guess):
//   PerfectGas: T = e/cv, e(T) = cv T, a(T) = sqrt(gamma R rho T / rho), p(T) = R rho T
//   NASA-7:     T by secant, e_s(T), a = sqrt(gamma R T) with gamma = cp/(cp - R), p = rho Ru T / W
// NSMAX sizes the mass-fraction scratch; ns is the species count.
template <int DIM, int NSMAX, class S>
ABL_HD Decoded<S> decode(const Phys& P, int ns, const S* U, double Tguess, bool* ok) {
    Decoded<S> d;
    const S rho = U[0];
    if (NSMAX == 0 || P.eos == ABL_EOS_PERFECT_GAS) {
        // T = e/cv, e(T) = cv T, p(T) = R rho T, a(T) = sqrt(gamma p / rho) = sqrt(gamma R T)
        const S e = internal_energy<DIM>(U);
        const double cv = P.r_gas / (P.gamma - 1.0);
        d.T = e * rcp64(cv);
        d.e = d.T * cv;
        d.p = P.r_gas * rho * d.T;
        d.a = dsqrt(P.gamma * P.r_gas * d.T);
        return d;
    }
    S ys[NSMAX > 0 ? NSMAX : 1];
    fill_y(ns, rho, U + 2 + DIM, ys);
    const S eRef = internal_energy<DIM>(U);
    d.T = nasa_temperature_s<NSMAX>(P, ns, ys, eRef, Tguess, ok);
    d.e = e_sens(P, ns, ys, d.T);
    const S cp = mixture_cp(P, ns, ys, d.T);
    const S mwMix = mixture_mw(P, ns, ys);
    const S R = kRuniv * rcp64(mwMix);
    const S cv = cp - R;
    const S gamma = cp * rcp64(cv);
    d.a = dsqrt(gamma * R * d.T);
    d.p = rho * R * d.T;
    return d;
}

// Temperature only (aux update)
template <int DIM, int NSMAX, class S>
ABL_HD S temperature(const Phys& P, int ns, const S* U, double Tguess, bool* ok) {
    if (NSMAX == 0 || P.eos == ABL_EOS_PERFECT_GAS) {
        const S e = internal_energy<DIM>(U);
        return e * rcp64(P.r_gas / (P.gamma - 1.0));
    }
    S ys[NSMAX > 0 ? NSMAX : 1];
    fill_y(ns, U[0], U + 2 + DIM, ys);
    const S eRef = internal_energy<DIM>(U);
    return nasa_temperature_s<NSMAX>(P, ns, ys, eRef, Tguess, ok);
}

// cp at temperature T (Sutherland / constant-Lewis conductivity)
template <int DIM, int NSMAX, class S>
ABL_HD S cp_at(const Phys& P, int ns, const S* U, S T) {
    if (NSMAX == 0 || P.eos == ABL_EOS_PERFECT_GAS) return S(P.gamma * P.r_gas / (P.gamma - 1.0));
    S ys[NSMAX > 0 ? NSMAX : 1];
    fill_y(ns, U[0], U + 2 + DIM, ys);
    return mixture_cp(P, ns, ys, T);
}

// ------------------------------------------------------------------------------------------------
// transport
// ------------------------------------------------------------------------------------------------
template <class S>
ABL_HD S sutherland_mu(S T) {
    const double muo = 1.716e-5, to = 273.e+0, so = 111.e+0;
    return muo * dsqrt(T / to) * (T / to) * (to + so) / (T + so);
}

template <int DIM, int NSMAX, class S>
ABL_HD void transport(const Phys& P, int ns, const S* U, S T, S* mu, S* k, S* diff) {
    switch (P.transport) {
        case ABL_TRANSPORT_CONSTANT:
            *mu = P.mu;
            *k = P.k;
            *diff = P.diff;
            return;
        case ABL_TRANSPORT_SUTHERLAND: {
            const double pr = 0.707, sc = 0.707;
            S m = sutherland_mu(T);
            *mu = m;
            *k = m * cp_at<DIM, NSMAX>(P, ns, U, T) / pr;
            *diff = m / U[0] / sc;
            return;
        }
        case ABL_TRANSPORT_CONSTANT_LEWIS: {
            S cp = cp_at<DIM, NSMAX>(P, ns, U, T);
            *mu = P.mu;
            *k = P.mu * cp / P.k;
            *diff = *k / (U[0] * cp * P.diff);
            return;
        }
        default:
            *mu = 0;
            *k = 0;
            *diff = 0;
    }
}

// ------------------------------------------------------------------------------------------------
// limiter (symmetric BAM normalisation: f = 1/2 du / (grad u . dx), phi(1/2) = 1)
// ------------------------------------------------------------------------------------------------
template <class R>
ABL_HD R limiter(int kind, R f) {
    switch (kind) {
        case ABL_LIMITER_ZERO:
            return R(0);
        case ABL_LIMITER_MINMOD:
            return pmin(R(1), R(4) * pmax(R(0), pmin(f, R(1) - f)));
        case ABL_LIMITER_VANLEER:
            return pmax(R(0), R(4) * f * (R(1) - f));
        case ABL_LIMITER_VANALBADA:
            return pmax(R(0), R(2) * f * (R(1) - f) / (sqr(f) + sqr(R(1) - f)));
        case ABL_LIMITER_SIN: {
            R fclip = pmax(pmin(f, R(1)), R(0));
            return dsin(R(3.14159265358979323846) * fclip);
        }
        default:
            return R(1);
    }
}

template <int LIM, class R>
ABL_HD R limiter_k(int kind, R f) {
    return limiter<R>(LIM >= 0 ? LIM : kind, f);
}

}  // namespace abl
