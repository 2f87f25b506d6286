// oracle.cpp -- TEST INFRASTRUCTURE ONLY: CPU restatement of ABLATE 0.13.03's finite-volume RHS path.
//
// Loaded by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker and as the
// timed CPU baseline; the product path never calls it. Each function cites the reference file:line
// whose arithmetic it restates. Written as plain scalar double-precision loops in the reference's own
// order (face loop for gradients and fluxes, serial scatter), so that it can be read side by side
// with the reference.
#include "oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_err;

// PetscMin / PetscMax / PetscSqr macro semantics (petscmath.h): plain ternaries, NaN falls to the
// second operand.
inline double pmin(double a, double b) { return a < b ? a : b; }
inline double pmax(double a, double b) { return a < b ? b : a; }
inline double psqr(double a) { return a * a; }

constexpr double kTiny = 1e-30;   // utilities::Constants::tiny (src/utilities/constants.hpp:25)
constexpr double kSmall = 1e-10;  // utilities::Constants::small (src/utilities/constants.hpp:28)

// ---------------------------------------------------------------------------------------------
// Flux calculators
// ---------------------------------------------------------------------------------------------
struct FluxCtx {
    int kind;
    double minf;
    double alpha;
    double gamma;
};

// Ausm::AusmFunction, src/finiteVolume/fluxCalculator/ausm.cpp:2-43
int ausm(double uL, double aL, double rhoL, double pL, double uR, double aR, double rhoR, double pR, double* mf, double* p12) {
    double Mm = uR / aR;
    double sMm, sPm;
    if (std::fabs(Mm) <= 1.) {
        sMm = -0.25 * psqr(Mm - 1);
        sPm = -(sMm) * (2 + Mm);
    } else {
        sMm = 0.5 * (Mm - std::fabs(Mm));
        sPm = (sMm) / Mm;
    }
    double Mp = uL / aL;
    double sMp, sPp;
    if (std::fabs(Mp) <= 1.) {
        sMp = 0.25 * psqr(Mp + 1);
        sPp = (sMp) * (2 - Mp);
    } else {
        sMp = 0.5 * (Mp + std::fabs(Mp));
        sPp = (sMp) / Mp;
    }
    double m = sMm + sMp;
    int dir;
    if (m < 0) {
        *mf = m * aR * rhoR;
        dir = ABL_DIR_RIGHT;
    } else {
        *mf = m * aL * rhoL;
        dir = ABL_DIR_LEFT;
    }
    if (p12) *p12 = pR * sPm + pL * sPp;
    return dir;
}

// AusmpUp support functions, src/finiteVolume/fluxCalculator/ausmpUp.cpp:55-96 (beta = 1/8, ausmpUp.hpp:22)
double M1Plus(double m) { return 0.5 * (m + std::fabs(m)); }
double M2Plus(double m) { return 0.25 * psqr(m + 1); }
double M1Minus(double m) { return 0.5 * (m - std::fabs(m)); }
double M2Minus(double m) { return -0.25 * psqr(m - 1); }
double M4Plus(double m) {
    const double beta = 1.e+0 / 8.e+0;
    if (std::fabs(m) >= 1.0) return M1Plus(m);
    return M2Plus(m) * (1.0 - 16.0 * beta * M2Minus(m));
}
double M4Minus(double m) {
    const double beta = 1.e+0 / 8.e+0;
    if (std::fabs(m) >= 1.0) return M1Minus(m);
    return M2Minus(m) * (1.0 + 16.0 * beta * M2Plus(m));
}
double P5Plus(double m, double fa) {
    if (std::fabs(m) >= 1.0) return (M1Plus(m) / (m + 1E-30));
    double alpha = 3.0 / 16.0 * (-4.0 + 5 * fa * fa);
    return (M2Plus(m) * ((2.0 - m) - 16. * alpha * m * M2Minus(m)));
}
double P5Minus(double m, double fa) {
    if (std::fabs(m) >= 1.0) return (M1Minus(m) / (m + 1E-30));
    double alpha = 3.0 / 16.0 * (-4.0 + 5 * fa * fa);
    return (M2Minus(m) * ((-2.0 - m) + 16. * alpha * m * M2Plus(m)));
}

// AusmpUp::AusmpUpFunction, src/finiteVolume/fluxCalculator/ausmpUp.cpp:5-53 (Kp 0.25, Ku 0.75, sigma 0.25: ausmpUp.hpp:23-25)
int ausmpup(const FluxCtx& c, double uL, double aL, double rhoL, double pL, double uR, double aR, double rhoR, double pR, double* mf,
            double* p12) {
    const double Kp = 0.25, Ku = 0.75, sigma = 0.25;
    double pgsAlpha = c.alpha;
    double mInf = c.minf;
    double rho12 = (0.5) * (rhoL + rhoR);
    double a12 = 0.5 * (aL + aR) / pgsAlpha;
    double mL = uL / a12;
    double mR = uR / a12;
    double mBar2 = (psqr(uL) + psqr(uR)) / (2.0 * a12 * a12);
    double fa = 1.0;
    if (mInf > 0) {
        double mInf2 = psqr(mInf);
        double mO2 = pmin(1.0, pmax(mBar2, mInf2));
        double mO = std::sqrt(mO2);
        fa = mO * (2.0 - mO);
    }
    double m12 = M4Plus(mL) + M4Minus(mR) - (Kp / fa) * pmax(1.0 - (sigma * mBar2), 0) * (pR - pL) / (rho12 * a12 * a12 * pgsAlpha * pgsAlpha);
    int dir;
    if (m12 > 0) {
        dir = ABL_DIR_LEFT;
        *mf = a12 * m12 * rhoL;
    } else {
        dir = ABL_DIR_RIGHT;
        *mf = a12 * m12 * rhoR;
    }
    if (p12) {
        double p5Plus = P5Plus(mL, fa);
        double p5Minus = P5Minus(mR, fa);
        *p12 = p5Plus * pL + p5Minus * pR - Ku * p5Plus * p5Minus * rho12 * fa * a12 * a12 * pgsAlpha * pgsAlpha * (mR - mL);
        *p12 /= psqr(pgsAlpha);
    }
    return dir;
}

// expansionShockCalculation, src/finiteVolume/fluxCalculator/riemannSolver.cpp:7-30
void expansionShock(double pstar, double gamma, double gamm1, double gamp1, double p0, double p, double a, double rho, double* f0, double* f1) {
    if (pstar <= p) {
        double A = 2.0 * a / gamm1;
        double B = 0.5 * gamm1 / gamma;
        double pRatio = (pstar + p0) / (p + p0);
        double pPow = std::pow(pRatio, B);
        *f0 = A * (pPow - 1.0);
        *f1 = A * B * pPow / (pstar + p0);
    } else {
        double A = 2 / (gamp1 * rho);
        double B = gamm1 * (p + p0) / gamp1;
        double pFrac = A / (pstar + p0 + B);
        double pSqrt = std::sqrt(pFrac);
        *f0 = (pstar - p) * pSqrt;
        *f1 = 0.5 * pFrac * pSqrt * (2.0 * (B + p0) + pstar + p) / A;
    }
}

// riemannDirection, src/finiteVolume/fluxCalculator/riemannSolver.cpp:32-156
int riemannDirection(double pstar, double uL, double aL, double rhoL, double p0L, double pL, double gammaL, double fL, double uR, double aR,
                     double rhoR, double p0R, double pR, double gammaR, double fR, double* massFlux, double* p12) {
    double STLR, SHLR, A, pRatio, gamma, gamm1, gamp1, astar, uX;
    double ustar = 0.5 * (uL + uR + fR - fL);
    if (ustar >= 0) {
        gamma = gammaL;
        gamm1 = gamma - 1.0;
        gamp1 = gamma + 1.0;
        if (pstar <= pL) {
            astar = aL * std::pow((pstar + p0L) / (pL + p0L), (gamm1 / (2 * gamma)));
            STLR = ustar - astar;
            if (STLR >= 0) {
                SHLR = uL - aL;
                if (SHLR >= 0) {
                    *massFlux = rhoL * uL;
                    *p12 = pL;
                    uX = uL;
                } else {
                    A = rhoL * std::pow((2 / gamp1) + ((gamm1 * uL) / (gamp1 * aL)), (2 / gamm1));
                    uX = 2 / gamp1 * (aL + (gamm1 * uL / 2));
                    *massFlux = A * uX;
                    *p12 = (pL + p0L) * std::pow((2 / gamp1) + ((gamm1 * uL) / (gamp1 * aL)), (2 * gamma / gamm1));
                }
            } else {
                pRatio = (pstar + p0L) / (pL + p0L);
                *massFlux = rhoL * std::pow(pRatio, 1.0 / gamma) * ustar;
                *p12 = pstar;
                uX = ustar;
            }
        } else {
            A = std::sqrt((gamp1 * (pstar + p0L) / 2 / gamma / (pL + p0L)) + (gamm1 / 2 / gamma));
            STLR = uL - (aL * A);
            if (STLR >= 0) {
                *massFlux = rhoL * uL;
                *p12 = pL;
                uX = uL;
            } else {
                pRatio = (pstar + p0L) / (pL + p0L);
                *massFlux = rhoL * (pRatio + (gamm1 / gamp1)) / (gamm1 * pRatio / gamp1 + 1) * ustar;
                *p12 = pstar;
                uX = ustar;
            }
        }
    } else {
        gamma = gammaR;
        gamm1 = gamma - 1.0;
        gamp1 = gamma + 1.0;
        if (pstar <= pR) {
            SHLR = uR + aR;
            if (SHLR >= 0) {
                astar = aR * std::pow((pstar + p0R) / (pR + p0R), (gamm1 / (2 * gamma)));
                STLR = ustar + astar;
                if (STLR >= 0) {
                    pRatio = (pstar + p0R) / (pR + p0R);
                    *massFlux = rhoR * std::pow(pRatio, 1 / gamma) * ustar;
                    *p12 = pstar;
                    uX = ustar;
                } else {
                    A = rhoR * std::pow((2 / gamp1) - ((gamm1 * uR) / (gamp1 * aR)), (2 / gamm1));
                    uX = 2 / gamp1 * (-aR + (gamm1 * uR / 2));
                    *massFlux = A * uX;
                    *p12 = (pR + p0R) * std::pow((2 / gamp1) - ((gamm1 * uR) / (gamp1 * aR)), (2 * gamma / gamm1));
                }
            } else {
                *massFlux = rhoR * uR;
                *p12 = pR;
                uX = uR;
            }
        } else {
            A = std::sqrt((gamp1 * (pstar + p0R) / 2 / gamma / (pR + p0R)) + (gamm1 / 2 / gamma));
            STLR = uR + (aR * A);
            if (STLR >= 0) {
                pRatio = (pstar + p0R) / (pR + p0R);
                *massFlux = rhoR * (pRatio + (gamm1 / gamp1)) / (gamm1 * pRatio / gamp1 + 1) * ustar;
                *p12 = pstar;
                uX = ustar;
            } else {
                *massFlux = rhoR * uR;
                *p12 = pR;
                uX = uR;
            }
        }
    }
    return (uX > 0 ? ABL_DIR_LEFT : ABL_DIR_RIGHT);
}

// Riemann::RiemannFluxFunction (src/finiteVolume/fluxCalculator/riemann.cpp:6-36) + RiemannSolver::riemannSolver
// (src/finiteVolume/fluxCalculator/riemannSolver.cpp:159-187). Non-convergence throws in the reference.
int riemann(double gamma, double uL, double aL, double rhoL, double pL, double uR, double aR, double rhoR, double pR, double* mf, double* p12) {
    double gamm1 = gamma - 1.0;
    double pstar = aL + aR - (0.5 * gamm1 * (uR - uL));
    pstar = pstar / ((aL / std::pow(pL, 0.5 * gamm1 / gamma)) + (aR / std::pow(pR, 0.5 * gamm1 / gamma)));
    pstar = std::pow(pstar, 2.0 * gamma / gamm1);
    const double p0L = 0, p0R = 0, gammaL = gamma, gammaR = gamma;
    const double tol = 1e-8;
    double pold, fL0, fL1, fR0, fR1;
    const double del_u = uR - uL;
    const double gLm1 = gammaL - 1.0, gLp1 = gammaL + 1.0, gRm1 = gammaR - 1.0, gRp1 = gammaR + 1.0;
    const int MAXIT = 100;
    int i = 0;
    do {
        expansionShock(pstar, gammaL, gLm1, gLp1, p0L, pL, aL, rhoL, &fL0, &fL1);
        expansionShock(pstar, gammaR, gRm1, gRp1, p0R, pR, aR, rhoR, &fR0, &fR1);
        pold = pstar;
        pstar = pold - (fL0 + fR0 + del_u) / (fL1 + fR1);
        if (pstar < 0 && (p0L < kTiny || p0R < kTiny)) pstar = kSmall;
        i++;
    } while (std::fabs((pstar - pold) / pstar) > tol && i <= MAXIT);
    if (i > MAXIT) throw std::runtime_error("Can't find pstar; Iteration not converging");
    double p12tmp;
    return riemannDirection(pstar, uL, aL, rhoL, p0L, pL, gammaL, fL0, uR, aR, rhoR, p0R, pR, gammaR, fR0, mf, p12 ? p12 : &p12tmp);
}

int flux_calc(const FluxCtx& c, double uL, double aL, double rhoL, double pL, double uR, double aR, double rhoR, double pR, double* mf,
              double* p12) {
    switch (c.kind) {
        case ABL_FLUX_OFF:  // OffFlux::OffCalculatorFunction, offFlux.cpp:2-9
            *mf = 0.0;
            if (p12) *p12 = 0.0;
            return ABL_DIR_NA;
        case ABL_FLUX_AVERAGE:  // AverageFlux::AvgCalculatorFunction, averageFlux.cpp:2-11
            *mf = 0.5 * (uL * rhoL + uR * rhoR);
            if (p12) *p12 = 0.5 * (pL + pR);
            return ABL_DIR_NA;
        case ABL_FLUX_AUSM:
            return ausm(uL, aL, rhoL, pL, uR, aR, rhoR, pR, mf, p12);
        case ABL_FLUX_AUSMPUP:
            return ausmpup(c, uL, aL, rhoL, pL, uR, aR, rhoR, pR, mf, p12);
        case ABL_FLUX_RIEMANN:
            return riemann(c.gamma, uL, aL, rhoL, pL, uR, aR, rhoR, pR, mf, p12);
    }
    throw std::invalid_argument("unknown flux calculator");
}

// ---------------------------------------------------------------------------------------------
// Equations of state
// ---------------------------------------------------------------------------------------------
constexpr double kRuniv = 8314.46261815324;  // J/(kmol K)
constexpr double kTref = 298.15;             // TChemBase::TREF (src/eos/tChemBase.hpp:150)

struct Eos {
    const abl_physics_desc* p;
    int dim;
    int ns;
    std::vector<double> href;  // TChem reference enthalpy per species, J/kg (src/eos/tChemBase.cpp:43-69)

    Eos(const abl_physics_desc* phys, int d) : p(phys), dim(d), ns(phys->n_species) {
        if (p->eos == ABL_EOS_NASA7) {
            href.resize(ns);
            for (int k = 0; k < ns; k++) href[k] = h_molar(k, kTref) / p->mw[k];
        }
    }
    // NASA-7 molar enthalpy (J/kmol) and heat capacity (J/(kmol K)) of species k (TChem EnthalpySpecMlFcn / CpSpecMl)
    double h_molar(int k, double T) const {
        const double* c = p->nasa7 + 15 * k;
        const double* a = (T < c[0]) ? c + 1 : c + 8;
        return kRuniv * T * (a[0] + T * (a[1] / 2 + T * (a[2] / 3 + T * (a[3] / 4 + T * a[4] / 5))) + a[5] / T);
    }
    double cp_molar(int k, double T) const {
        const double* c = p->nasa7 + 15 * k;
        const double* a = (T < c[0]) ? c + 1 : c + 8;
        return kRuniv * (a[0] + T * (a[1] + T * (a[2] + T * (a[3] + T * a[4]))));
    }
    // TChem::FillWorkingVectorFromDensityMassFractions, src/eos/tChem.cpp:581-602
    void fill_y(const double* U, double* ys) const {
        const double density = U[0];
        const double* densityYi = U + 2 + dim;
        double yiSum = 0.0;
        for (int s = 0; s < ns - 1; s++) {
            ys[s] = pmax(0.0, densityYi[s] / density);
            ys[s] = pmin(1.0, ys[s]);
            yiSum += ys[s];
        }
        if (yiSum > 1.0) {
            for (int s = 0; s < ns - 1; s++) ys[s] /= yiSum;
            ys[ns - 1] = 0.0;
        } else {
            ys[ns - 1] = 1.0 - yiSum;
        }
    }
    // SensibleInternalEnergyFcn, src/eos/tChem/sensibleInternalEnergyFcn.hpp:25-44
    double e_sens(const double* ys, double T) const {
        double e = 0;
        for (int k = 0; k < ns; k++) e += (h_molar(k, T) / p->mw[k] - href[k] - kRuniv * T / p->mw[k]) * ys[k];
        return e;
    }
    double mw_mix(const double* ys) const {
        double s = 0;
        for (int k = 0; k < ns; k++) s += ys[k] / p->mw[k];
        return 1.0 / s;
    }
    double cp_mix(const double* ys, double T) const {
        double s = 0;
        for (int k = 0; k < ns; k++) s += ys[k] * cp_molar(k, T) / p->mw[k];
        return s;
    }
    // internal energy from the conserved state (E/rho - |u|^2/2): perfectGas.cpp:126-141, tChem.cpp:121-131
    double e_from_conserved(const double* U) const {
        double density = U[0];
        double ke = 0.0;
        for (int d = 0; d < dim; d++) ke += psqr(U[2 + d] / density);
        ke *= 0.5;
        return U[1] / density - ke;
    }
    // Temperature(T guess): PerfectGas::TemperatureFunction (perfectGas.cpp:76-91);
    // TChem::TemperatureTemperatureFunction + Temperature_TemplateRun secant (tChem.cpp:119-148, tChem/temperature.cpp:21-97)
    double temperature(const double* U, double Tguess, bool* converged = nullptr) const {
        if (converged) *converged = true;
        if (p->eos == ABL_EOS_PERFECT_GAS) {
            double e = e_from_conserved(U);
            double cv = p->r_gas / (p->gamma - 1.0);
            return e / cv;
        }
        double density = U[0];
        double speedSquare = 0.0;
        for (int d = 0; d < dim; d++) speedSquare += psqr(U[2 + d] / density);
        double eRef = U[1] / density - 0.5 * speedSquare;
        std::vector<double> ys(ns);
        fill_y(U, ys.data());
        const double EPS = 1E-8;
        const int ITMAX = 100;
        double t = Tguess;
        double t2 = t;
        double e2 = e_sens(ys.data(), t);
        double f2 = eRef - e2;
        if (std::fabs(f2) > EPS) {
            double t0 = t2, f0 = f2, t1 = t0 + 1;
            t = t1;
            double e1 = e_sens(ys.data(), t);
            double f1 = eRef - e1;
            for (int it = 0; it < ITMAX; it++) {
                t2 = t1 - f1 * (t1 - t0) / (f1 - f0 + 1E-30);
                t2 = std::max(1.0, t2);
                t = t2;
                e2 = e_sens(ys.data(), t);
                f2 = eRef - e2;
                if (std::fabs(f2) <= EPS) return t2;
                t0 = t1;
                t1 = t2;
                f0 = f1;
                f1 = f2;
            }
            // restart from 1000 K (temperature.cpp:67-90); note f0 uses the current t, as the reference does
            t0 = 1000.;
            f0 = eRef - e_sens(ys.data(), t);
            t1 = t0 + 1;
            t = t1;
            e1 = e_sens(ys.data(), t);
            f1 = eRef - e1;
            for (int it = 0; it < ITMAX; it++) {
                t2 = t1 - f1 * (t1 - t0) / (f1 - f0 + 1E-30);
                t2 = std::max(1.0, t2);
                t = t2;
                e2 = e_sens(ys.data(), t);
                f2 = eRef - e2;
                if (std::fabs(f2) <= EPS) return t2;
                t0 = t1;
                t1 = t2;
                f0 = f1;
                f1 = f2;
            }
            if (converged) *converged = false;
            t = t2;
        }
        return t;
    }
    // ThermodynamicTemperatureFunction of one property at temperature T; out sized by property
    void property_T(int prop, const double* U, double T, double* out) const {
        const double density = U[0];
        if (p->eos == ABL_EOS_PERFECT_GAS) {
            // src/eos/perfectGas.cpp:68-197 (temperature variants)
            const double g = p->gamma, R = p->r_gas;
            switch (prop) {
                case ABL_PROP_PRESSURE:
                    *out = R * density * T;
                    return;
                case ABL_PROP_TEMPERATURE:
                    *out = temperature(U, T);
                    return;
                case ABL_PROP_INTERNAL_SENSIBLE_ENERGY:
                    *out = T * (R / (g - 1.0));
                    return;
                case ABL_PROP_SENSIBLE_ENTHALPY:
                    *out = T * (g * R / (g - 1.0));
                    return;
                case ABL_PROP_CV:
                    *out = R / (g - 1.0);
                    return;
                case ABL_PROP_CP:
                    *out = g * R / (g - 1.0);
                    return;
                case ABL_PROP_SPEED_OF_SOUND: {
                    double pr = R * density * T;
                    *out = std::sqrt(g * (pr) / density);
                    return;
                }
                case ABL_PROP_SPECIES_SENSIBLE_ENTHALPY:
                    for (int s = 0; s < ns; s++) out[s] = 0.0;
                    return;
                case ABL_PROP_DENSITY:
                    *out = density;
                    return;
            }
            throw std::invalid_argument("property");
        }
        std::vector<double> ys(ns);
        fill_y(U, ys.data());
        switch (prop) {
            case ABL_PROP_PRESSURE:  // pressureFcn.hpp:26-42
                *out = density * kRuniv * T / mw_mix(ys.data());
                return;
            case ABL_PROP_TEMPERATURE:
                *out = temperature(U, T);
                return;
            case ABL_PROP_INTERNAL_SENSIBLE_ENERGY:
                *out = e_sens(ys.data(), T);
                return;
            case ABL_PROP_SENSIBLE_ENTHALPY: {  // sensibleEnthalpyFcn: sum Y_k (h_k/W_k - h_ref,k)
                double h = 0;
                for (int k = 0; k < ns; k++) h += (h_molar(k, T) / p->mw[k] - href[k]) * ys[k];
                *out = h;
                return;
            }
            case ABL_PROP_CV: {
                double cp = cp_mix(ys.data(), T);
                *out = cp - kRuniv / mw_mix(ys.data());
                return;
            }
            case ABL_PROP_CP:
                *out = cp_mix(ys.data(), T);
                return;
            case ABL_PROP_SPEED_OF_SOUND: {  // speedOfSound.cpp:23-51
                double cp = cp_mix(ys.data(), T);
                double R = kRuniv / mw_mix(ys.data());
                double cv = cp - R;
                double gamma = cp / cv;
                *out = std::sqrt(gamma * R * T);
                return;
            }
            case ABL_PROP_SPECIES_SENSIBLE_ENTHALPY:
                for (int k = 0; k < ns; k++) out[k] = h_molar(k, T) / p->mw[k] - href[k];
                return;
            case ABL_PROP_DENSITY:
                *out = density;
                return;
        }
        throw std::invalid_argument("property");
    }
    // ThermodynamicFunction (no temperature argument)
    void property(int prop, const double* U, double* out) const {
        if (p->eos == ABL_EOS_PERFECT_GAS) {
            const double g = p->gamma;
            const double density = U[0];
            double e = e_from_conserved(U);
            switch (prop) {
                case ABL_PROP_PRESSURE:  // perfectGas.cpp:49-66
                    *out = (g - 1.0) * density * e;
                    return;
                case ABL_PROP_INTERNAL_SENSIBLE_ENERGY:
                    *out = e;
                    return;
                case ABL_PROP_SPEED_OF_SOUND: {  // perfectGas.cpp:151-167
                    double pr = (g - 1.0) * density * e;
                    *out = std::sqrt(g * (pr) / density);
                    return;
                }
                default: {
                    double T = temperature(U, 300.0);
                    property_T(prop, U, T, out);
                    return;
                }
            }
        }
        double T = temperature(U, 300.0);  // TChem::TemperatureFunction guess 300 (tChem.cpp:118)
        if (prop == ABL_PROP_INTERNAL_SENSIBLE_ENERGY) {
            *out = e_from_conserved(U);
            return;
        }
        property_T(prop, U, T, out);
    }
    int property_size(int prop) const { return prop == ABL_PROP_SPECIES_SENSIBLE_ENTHALPY ? ns : 1; }
};

// ---------------------------------------------------------------------------------------------
// Transport models
// ---------------------------------------------------------------------------------------------
struct Transport {
    const abl_physics_desc* p;
    const Eos* eos;
    // Sutherland constants, src/eos/transport/sutherland.hpp:23-27
    static constexpr double pr = 0.707, muo = 1.716e-5, to = 273.e+0, so = 111.e+0, sc = 0.707;
    double mu(const double* U, double T) const {
        switch (p->transport) {
            case ABL_TRANSPORT_CONSTANT:
            case ABL_TRANSPORT_CONSTANT_LEWIS:
                return p->mu;
            case ABL_TRANSPORT_SUTHERLAND:  // sutherland.cpp:36-41
                return muo * std::sqrt(T / to) * (T / to) * (to + so) / (T + so);
        }
        return 0.0;
    }
    double k(const double* U, double T) const {
        switch (p->transport) {
            case ABL_TRANSPORT_CONSTANT:
                return p->k;
            case ABL_TRANSPORT_SUTHERLAND: {  // sutherland.cpp:22-33
                double cp;
                eos->property_T(ABL_PROP_CP, U, T, &cp);
                double m = muo * std::sqrt(T / to) * (T / to) * (to + so) / (T + so);
                return m * cp / pr;
            }
            case ABL_TRANSPORT_CONSTANT_LEWIS: {
                double cp;
                eos->property_T(ABL_PROP_CP, U, T, &cp);
                return p->mu * cp / p->k;
            }
        }
        return 0.0;
    }
    double diff(const double* U, double T) const {
        switch (p->transport) {
            case ABL_TRANSPORT_CONSTANT:
                return p->diff;
            case ABL_TRANSPORT_SUTHERLAND: {  // sutherland.cpp:54-62
                double density = U[0];
                double m = muo * std::sqrt(T / to) * (T / to) * (to + so) / (T + so);
                return m / density / sc;
            }
            case ABL_TRANSPORT_CONSTANT_LEWIS: {
                double cp;
                eos->property_T(ABL_PROP_CP, U, T, &cp);
                double kk = p->mu * cp / p->k;
                return kk / (U[0] * cp * p->diff);
            }
        }
        return 0.0;
    }
};

// ---------------------------------------------------------------------------------------------
// Limiters: PetscLimiterLimit in the symmetric (BAM) normalisation used by DMPlexApplyLimiter_Internal
// (src/finiteVolume/cellInterpolant.cpp:282-328): f = 1/2 (u_n - u_c) / (grad u . dx); phi(1/2) = 1.
// ---------------------------------------------------------------------------------------------
double limiter(int kind, double f) {
    switch (kind) {
        case ABL_LIMITER_NONE:
            return 1.0;
        case ABL_LIMITER_ZERO:
            return 0.0;
        case ABL_LIMITER_MINMOD:
            return pmin(1, 4 * pmax(0, pmin(f, 1 - f)));
        case ABL_LIMITER_VANLEER:
            return pmax(0, 4 * f * (1 - f));
        case ABL_LIMITER_VANALBADA:
            return pmax(0, 2 * f * (1 - f) / (psqr(f) + psqr(1 - f)));
        case ABL_LIMITER_SIN: {
            double fclip = pmax(pmin(f, 1), 0);
            return std::sin(M_PI * fclip);
        }
    }
    throw std::invalid_argument("limiter");
}

// ---------------------------------------------------------------------------------------------
// Least squares pseudo-inverse (PetscFVComputeGradient for PETSCFVLEASTSQUARES): rows dx[n][dim];
// grad[n][dim] = pinv(B)^T. The reference calls an SVD-based pseudo-inverse; this restates it with a
// Jacobi eigen-decomposition of B^T B (identical for full rank, minimum-norm for rank deficient).
// ---------------------------------------------------------------------------------------------
void pinv_rows(int n, int dim, const double* dx, double* grad) {
    double A[3][3] = {{0}};
    for (int i = 0; i < n; i++)
        for (int a = 0; a < dim; a++)
            for (int b = 0; b < dim; b++) A[a][b] += dx[i * dim + a] * dx[i * dim + b];
    double V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int sweep = 0; sweep < 50; sweep++) {
        double off = 0;
        for (int a = 0; a < dim; a++)
            for (int b = a + 1; b < dim; b++) off += A[a][b] * A[a][b];
        if (off < 1e-300) break;
        for (int a = 0; a < dim; a++)
            for (int b = a + 1; b < dim; b++) {
                if (A[a][b] == 0.0) continue;
                double theta = (A[b][b] - A[a][a]) / (2 * A[a][b]);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
                double c = 1 / std::sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < dim; k++) {
                    double akp = A[k][a], akq = A[k][b];
                    A[k][a] = c * akp - s * akq;
                    A[k][b] = s * akp + c * akq;
                }
                for (int k = 0; k < dim; k++) {
                    double apk = A[a][k], aqk = A[b][k];
                    A[a][k] = c * apk - s * aqk;
                    A[b][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < dim; k++) {
                    double vkp = V[k][a], vkq = V[k][b];
                    V[k][a] = c * vkp - s * vkq;
                    V[k][b] = s * vkp + c * vkq;
                }
            }
    }
    double lmax = 0;
    for (int a = 0; a < dim; a++) lmax = std::max(lmax, A[a][a]);
    double Minv[3][3] = {{0}};
    for (int a = 0; a < dim; a++) {
        double l = A[a][a];
        if (l <= 1e-14 * lmax) continue;
        for (int r = 0; r < dim; r++)
            for (int c = 0; c < dim; c++) Minv[r][c] += V[r][a] * V[c][a] / l;
    }
    for (int i = 0; i < n; i++)
        for (int a = 0; a < dim; a++) {
            double s = 0;
            for (int b = 0; b < dim; b++) s += Minv[a][b] * dx[i * dim + b];
            grad[i * dim + a] = s;
        }
}

// ---------------------------------------------------------------------------------------------
// Mesh helpers
// ---------------------------------------------------------------------------------------------
struct Topo {
    int dim, nc, nf;
    std::vector<int> cone_ptr, cone;  // cell -> faces, ascending face order
    std::vector<uint8_t> kind;
};

Topo build_topo(const abl_mesh_desc* m) {
    Topo t;
    t.dim = m->dim;
    t.nc = m->n_cells;
    t.nf = m->n_faces;
    t.kind.assign(t.nc, ABL_CELL_OWNED);
    if (m->cell_kind)
        for (int c = 0; c < t.nc; c++) t.kind[c] = m->cell_kind[c];
    t.cone_ptr.assign(t.nc + 1, 0);
    for (int f = 0; f < t.nf; f++) {
        for (int s = 0; s < 2; s++) {
            int c = m->face_cells[2 * f + s];
            if (c < 0 || c >= t.nc) throw std::invalid_argument("face_cells out of range");
            t.cone_ptr[c + 1]++;
        }
    }
    for (int c = 0; c < t.nc; c++) t.cone_ptr[c + 1] += t.cone_ptr[c];
    t.cone.resize(t.cone_ptr[t.nc]);
    std::vector<int> fill(t.cone_ptr.begin(), t.cone_ptr.end() - 1);
    for (int f = 0; f < t.nf; f++)
        for (int s = 0; s < 2; s++) t.cone[fill[m->face_cells[2 * f + s]]++] = f;
    return t;
}

inline bool is_boundary_face(const abl_mesh_desc* m, const Topo& t, int f) {
    return t.kind[m->face_cells[2 * f]] == ABL_CELL_BOUNDARY || t.kind[m->face_cells[2 * f + 1]] == ABL_CELL_BOUNDARY;
}
inline bool has_gradient(const Topo& t, int c) { return t.kind[c] == ABL_CELL_OWNED || t.kind[c] == ABL_CELL_HALO; }

// periodic image shift of face f (zero unless the mesh declares periodic faces)
inline double shift(const abl_mesh_desc* m, int f, int d) { return m->face_shift ? m->face_shift[3 * (size_t)f + d] : 0.0; }
// centroid of the cell across face f seen from cell c (cg1->centroid in the reference, periodic image resolved)
inline double nbr_centroid(const abl_mesh_desc* m, int f, int c, int d) {
    const int L = m->face_cells[2 * f], R = m->face_cells[2 * f + 1];
    return c == L ? m->cell_centroid[3 * (size_t)R + d] + shift(m, f, d) : m->cell_centroid[3 * (size_t)L + d] - shift(m, f, d);
}
// face centroid seen from cell c
inline double face_centroid(const abl_mesh_desc* m, int f, int c, int d) {
    return c == m->face_cells[2 * f] ? m->face_centroid[3 * (size_t)f + d] : m->face_centroid[3 * (size_t)f + d] - shift(m, f, d);
}

// BuildGradientReconstruction_Internal, src/finiteVolume/cellInterpolant.cpp:641-715:
// fg->grad[side] for every face from the LSQ pseudo-inverse over each cell's non-boundary faces.
void lsq_face_weights(const abl_mesh_desc* m, const Topo& t, std::vector<double>& w) {
    const int dim = m->dim;
    w.assign((size_t)t.nf * 6, 0.0);
    std::vector<double> dx, grad;
    std::vector<double*> gref;
    for (int c = 0; c < t.nc; c++) {
        if (!has_gradient(t, c)) continue;
        dx.clear();
        gref.clear();
        for (int i = t.cone_ptr[c]; i < t.cone_ptr[c + 1]; i++) {
            int f = t.cone[i];
            if (is_boundary_face(m, t, f)) continue;
            int side = (c != m->face_cells[2 * f]);
            for (int d = 0; d < dim; d++) dx.push_back(nbr_centroid(m, f, c, d) - m->cell_centroid[3 * c + d]);
            gref.push_back(&w[(size_t)f * 6 + side * 3]);
        }
        if (gref.empty()) throw std::runtime_error("Mesh contains isolated cell (no neighbors)");
        grad.assign(dx.size(), 0.0);
        pinv_rows((int)gref.size(), dim, dx.data(), grad.data());
        for (size_t i = 0; i < gref.size(); i++)
            for (int d = 0; d < dim; d++) gref[i][d] = grad[i * dim + d];
    }
}

// LeastSquaresAverage stencil of one face (src/finiteVolume/stencils/leastSquaresAverage.cpp:5-155)
struct Stencil {
    std::vector<int> cells;
    std::vector<double> weights, gw;  // gw[i*dim + d]
};

void cell_stencil(const abl_mesh_desc* m, const Topo& t, int cell, Stencil& s) {
    const int dim = m->dim;
    s.cells.clear();
    s.cells.push_back(cell);
    std::vector<int> via;  // face through which each neighbour was reached (periodic image)
    for (int i = t.cone_ptr[cell]; i < t.cone_ptr[cell + 1]; i++) {
        int f = t.cone[i];
        int a = m->face_cells[2 * f], b = m->face_cells[2 * f + 1];
        s.cells.push_back(a == cell ? b : a);
        via.push_back(f);
    }
    int n = (int)s.cells.size();
    s.weights.assign(n, 0.0);
    s.gw.assign((size_t)n * dim, 0.0);
    s.weights[0] = 1.0;
    std::vector<double> dx((size_t)(n - 1) * dim);
    for (int k = 0; k < n - 1; k++)
        for (int d = 0; d < dim; d++) dx[k * dim + d] = nbr_centroid(m, via[k], cell, d) - m->cell_centroid[3 * cell + d];
    pinv_rows(n - 1, dim, dx.data(), s.gw.data() + dim);
    std::vector<double> org = s.gw;
    for (int gn = 0; gn < n; gn++)
        for (int fn = 0; fn < n; fn++)
            for (int d = 0; d < dim; d++) s.gw[fn * dim + d] -= org[gn * dim + d] * s.weights[fn];
}

// stencil::LeastSquares of one face, the 1D choice of the FaceInterpolant (faceInterpolant.cpp:32-36,
// src/finiteVolume/stencils/leastSquares.cpp:5-122): the cells sharing the face's node (in 1D its two
// support cells), value weights 1/2, gradient weights the least-squares operator of the offsets
// x_cell - x_face less its value-weighted sum
void face_stencil_1d(const abl_mesh_desc* m, int f, Stencil& out) {
    const int a = m->face_cells[2 * f], b = m->face_cells[2 * f + 1];
    out.cells = {std::min(a, b), std::max(a, b)};
    out.weights = {0.5, 0.5};
    // offsets to the face centroid, periodic image resolved: the face centroid is given in the left
    // cell's frame and the right cell is seen from there at its centroid + face_shift
    const double sh = m->face_shift ? m->face_shift[3 * (size_t)f] : 0.0;
    std::vector<double> dx(2);
    for (int i = 0; i < 2; i++) {
        const int c = out.cells[i];
        dx[i] = m->cell_centroid[3 * (size_t)c] + (c == b ? sh : 0.0) - m->face_centroid[3 * (size_t)f];
    }
    out.gw.assign(2, 0.0);
    pinv_rows(2, 1, dx.data(), out.gw.data());
    const std::vector<double> org = out.gw;
    for (int gn = 0; gn < 2; gn++)
        for (int fn = 0; fn < 2; fn++) out.gw[fn] -= org[gn] * out.weights[fn];
}

void face_stencil(const abl_mesh_desc* m, const Topo& t, int f, Stencil& out) {
    const int dim = m->dim;
    if (dim == 1) {
        face_stencil_1d(m, f, out);
        return;
    }
    Stencil L, R;
    cell_stencil(m, t, m->face_cells[2 * f], L);
    cell_stencil(m, t, m->face_cells[2 * f + 1], R);
    out.cells = L.cells;
    out.cells.insert(out.cells.end(), R.cells.begin(), R.cells.end());
    std::sort(out.cells.begin(), out.cells.end());
    out.cells.erase(std::unique(out.cells.begin(), out.cells.end()), out.cells.end());
    int n = (int)out.cells.size();
    out.weights.assign(n, 0.0);
    out.gw.assign((size_t)n * dim, 0.0);
    const double numberStencils = 2;
    for (const Stencil* s : {&L, &R}) {
        for (size_t i = 0; i < s->cells.size(); i++) {
            int loc = (int)(std::find(out.cells.begin(), out.cells.end(), s->cells[i]) - out.cells.begin());
            out.weights[loc] += s->weights[i] / numberStencils;
            for (int d = 0; d < dim; d++) out.gw[loc * dim + d] += s->gw[i * dim + d] / numberStencils;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// RHS
// ---------------------------------------------------------------------------------------------
struct Rhs {
    const abl_mesh_desc* m;
    const abl_physics_desc* p;
    Topo t;
    int dim, ns, nc, naux, neuler;
    Eos eos;
    Transport tr;
    FluxCtx fc;

    std::vector<double> fw;          // LSQ face weights (CellInterpolant constructor)
    std::vector<Stencil> stencils;   // face stencils (FaceInterpolant constructor)
    bool prepared = false;

    Rhs(const abl_mesh_desc* mesh, const abl_physics_desc* phys)
        : m(mesh), p(phys), t(build_topo(mesh)), dim(mesh->dim), ns(phys->n_species), eos(phys, mesh->dim) {
        neuler = 2 + dim;
        nc = neuler + ns;
        naux = 1 + dim + ns;
        tr.p = p;
        tr.eos = &eos;
        fc = FluxCtx{p->flux, p->ausmpup_minf, p->pgs_alpha > 0 ? p->pgs_alpha : 1.0, p->gamma};
    }

    // one-time setup the reference does in the interpolant constructors
    // (cellInterpolant.cpp:5-32 -> ComputeGradientFVM; faceInterpolant.cpp:7-73 -> stencils)
    void prepare() {
        if (prepared) return;
        if (p->reconstruction == ABL_RECON_LEASTSQUARES) lsq_face_weights(m, t, fw);
        const bool dif = (p->diffusion || (p->species_diffusion && ns > 0)) && p->transport != ABL_TRANSPORT_NONE;
        if (dif) {
            stencils.resize(t.nf);
            for (int f = 0; f < t.nf; f++) {
                const bool owned = t.kind[m->face_cells[2 * f]] == ABL_CELL_OWNED || t.kind[m->face_cells[2 * f + 1]] == ABL_CELL_OWNED;
                if (owned) face_stencil(m, t, f, stencils[f]);
            }
        }
        prepared = true;
    }

    // NavierStokesTransport::AdvectionFlux, src/finiteVolume/processes/navierStokesTransport.cpp:99-207
    void ns_advection(const double* normal, const double* fieldL, const double* fieldR, double TLa, double TRa, double* flux) const {
        double norm[3] = {0, 0, 0};
        double areaMag = 0;
        for (int d = 0; d < dim; d++) areaMag += normal[d] * normal[d];
        areaMag = std::sqrt(areaMag);  // MathUtilities::MagVector (src/utilities/mathUtilities.hpp:39-57)
        for (int d = 0; d < dim; d++) norm[d] = normal[d] / areaMag;  // MathUtilities::NormVector
        double densityL, normalVelocityL, velocityL[3], internalEnergyL, aL, pL;
        {
            densityL = fieldL[0];
            double temperatureL = eos.temperature(fieldL, TLa * .67 + .33 * TRa);
            normalVelocityL = 0.0;
            for (int d = 0; d < dim; d++) {
                velocityL[d] = fieldL[2 + d] / densityL;
                normalVelocityL += velocityL[d] * norm[d];
            }
            eos.property_T(ABL_PROP_INTERNAL_SENSIBLE_ENERGY, fieldL, temperatureL, &internalEnergyL);
            eos.property_T(ABL_PROP_SPEED_OF_SOUND, fieldL, temperatureL, &aL);
            eos.property_T(ABL_PROP_PRESSURE, fieldL, temperatureL, &pL);
        }
        double densityR, normalVelocityR, velocityR[3], internalEnergyR, aR, pR;
        {
            densityR = fieldR[0];
            double temperatureR = eos.temperature(fieldR, TLa * .33 + .67 * TRa);
            normalVelocityR = 0.0;
            for (int d = 0; d < dim; d++) {
                velocityR[d] = fieldR[2 + d] / densityR;
                normalVelocityR += velocityR[d] * norm[d];
            }
            eos.property_T(ABL_PROP_INTERNAL_SENSIBLE_ENERGY, fieldR, temperatureR, &internalEnergyR);
            eos.property_T(ABL_PROP_SPEED_OF_SOUND, fieldR, temperatureR, &aR);
            eos.property_T(ABL_PROP_PRESSURE, fieldR, temperatureR, &pR);
        }
        double massFlux, p12;
        int direction = flux_calc(fc, normalVelocityL, aL, densityL, pL, normalVelocityR, aR, densityR, pR, &massFlux, &p12);
        auto mag = [&](const double* v) {
            double s = 0;
            for (int d = 0; d < dim; d++) s += v[d] * v[d];
            return std::sqrt(s);
        };
        if (direction == ABL_DIR_LEFT) {
            flux[0] = massFlux * areaMag;
            double velMagL = mag(velocityL);
            double HL = internalEnergyL + velMagL * velMagL / 2.0 + pL / densityL;
            flux[1] = HL * massFlux * areaMag;
            for (int n = 0; n < dim; n++) flux[2 + n] = velocityL[n] * massFlux * areaMag + p12 * normal[n];
        } else if (direction == ABL_DIR_RIGHT) {
            flux[0] = massFlux * areaMag;
            double velMagR = mag(velocityR);
            double HR = internalEnergyR + velMagR * velMagR / 2.0 + pR / densityR;
            flux[1] = HR * massFlux * areaMag;
            for (int n = 0; n < dim; n++) flux[2 + n] = velocityR[n] * massFlux * areaMag + p12 * normal[n];
        } else {
            flux[0] = massFlux * areaMag;
            double velMagL = mag(velocityL);
            double HL = internalEnergyL + velMagL * velMagL / 2.0 + pL / densityL;
            double velMagR = mag(velocityR);
            double HR = internalEnergyR + velMagR * velMagR / 2.0 + pR / densityR;
            flux[1] = 0.5 * (HL + HR) * massFlux * areaMag;
            for (int n = 0; n < dim; n++) flux[2 + n] = 0.5 * (velocityL[n] + velocityR[n]) * massFlux * areaMag + p12 * normal[n];
        }
    }

    // SpeciesTransport::AdvectionFlux, src/finiteVolume/processes/speciesTransport.cpp:263-341
    void species_advection(const double* normal, const double* fieldL, const double* fieldR, double TLa, double TRa, double* flux) const {
        double norm[3] = {0, 0, 0};
        double areaMag = 0;
        for (int d = 0; d < dim; d++) areaMag += normal[d] * normal[d];
        areaMag = std::sqrt(areaMag);
        for (int d = 0; d < dim; d++) norm[d] = normal[d] / areaMag;
        double densityL = fieldL[0], densityR = fieldR[0];
        double temperatureL = eos.temperature(fieldL, TLa * .67 + TRa * .33);
        double normalVelocityL = 0.0;
        for (int d = 0; d < dim; d++) normalVelocityL += fieldL[2 + d] / densityL * norm[d];
        double aL, pL;
        eos.property_T(ABL_PROP_SPEED_OF_SOUND, fieldL, temperatureL, &aL);
        eos.property_T(ABL_PROP_PRESSURE, fieldL, temperatureL, &pL);
        double temperatureR = eos.temperature(fieldR, TLa * .33 + TRa * .67);
        double normalVelocityR = 0.0;
        for (int d = 0; d < dim; d++) normalVelocityR += fieldR[2 + d] / densityR * norm[d];
        double aR, pR;
        eos.property_T(ABL_PROP_SPEED_OF_SOUND, fieldR, temperatureR, &aR);
        eos.property_T(ABL_PROP_PRESSURE, fieldR, temperatureR, &pR);
        double massFlux;
        const int dir = flux_calc(fc, normalVelocityL, aL, densityL, pL, normalVelocityR, aR, densityR, pR, &massFlux, nullptr);
        if (dir == ABL_DIR_LEFT) {
            for (int sp = 0; sp < ns; sp++) flux[sp] = (massFlux * fieldL[neuler + sp] / densityL) * areaMag;
        } else if (dir == ABL_DIR_NA && p->species_advection_compact) {
            // CompactCompressibleNSSpeciesTransport::AdvectionFlux (compactCompressibleNSSpeciesTransport.cpp:257-259)
            for (int sp = 0; sp < ns; sp++)
                flux[sp] = massFlux * 0.5 * (fieldR[neuler + sp] + fieldL[neuler + sp]) / (0.5 * (densityL + densityR)) * areaMag;
        } else {
            for (int sp = 0; sp < ns; sp++) flux[sp] = (massFlux * fieldR[neuler + sp] / densityR) * areaMag;
        }
    }

    // NavierStokesTransport::DiffusionFlux + CompressibleFlowComputeStressTensor
    // (src/finiteVolume/processes/navierStokesTransport.cpp:454-532). field/aux/gradAux are face values.
    void ns_diffusion(const double* normal, const double* field, const double* aux, const double* gradAux, double* flux) const {
        double mu = tr.mu(field, aux[0]);
        double k = tr.k(field, aux[0]);
        double tau[9];
        orc_stress_tensor(dim, mu, gradAux + dim /* velocity block */, tau);
        for (int c = 0; c < dim; ++c) {
            double viscousFlux = 0.0;
            for (int d = 0; d < dim; ++d) viscousFlux += -normal[d] * tau[c * dim + d];
            flux[2 + c] = viscousFlux;
        }
        flux[1] = 0.0;
        for (int d = 0; d < dim; ++d) {
            double heatFlux = 0.0;
            for (int c = 0; c < dim; ++c) heatFlux += aux[1 + c] * tau[d * dim + c];
            heatFlux += k * gradAux[d];
            heatFlux *= -normal[d];
            flux[1] += heatFlux;
        }
        flux[0] = 0.0;
    }

    // SpeciesTransport::DiffusionEnergyFlux (speciesTransport.cpp:112-152): rhoE contribution only; with
    // one diffusivity per species, DiffusionEnergyFluxVariableDiffusionCoefficient (:154-194)
    double species_diffusion_energy(const double* normal, const double* field, const double* aux, const double* gradAux) const {
        const double density = field[0];
        const double temperature = aux[0];
        std::vector<double> hs(ns);
        eos.property_T(ABL_PROP_SPECIES_SENSIBLE_ENTHALPY, field, temperature, hs.data());
        double diff = tr.diff(field, temperature);
        double e = 0.0;
        const int yoff = (1 + dim) * dim;  // aux gradient offset of the Yi block
        for (int sp = 0; sp < ns; ++sp) {
            const double dsp = p->species_diff ? p->species_diff[sp] : diff;
            for (int d = 0; d < dim; ++d) e += -normal[d] * density * dsp * hs[sp] * gradAux[yoff + sp * dim + d];
        }
        return e;
    }
    // SpeciesTransport::DiffusionSpeciesFlux (speciesTransport.cpp:196-228); with one diffusivity per
    // species, DiffusionSpeciesFluxVariableDiffusionCoefficient (:230-261)
    void species_diffusion(const double* normal, const double* field, const double* aux, const double* gradAux, double* flux) const {
        const double density = field[0];
        double diff = tr.diff(field, aux[0]);
        const int yoff = (1 + dim) * dim;
        for (int sp = 0; sp < ns; ++sp) {
            const double dsp = p->species_diff ? p->species_diff[sp] : diff;
            flux[sp] = 0;
            for (int d = 0; d < dim; ++d) flux[sp] += -normal[d] * density * dsp * gradAux[yoff + sp * dim + d];
        }
    }

    void run(const double* U, double* aux, double* F, int threads) {
        prepare();
        const int nC = t.nc, nF = t.nf;
        // aux update over all local cells: NavierStokesTransport::UpdateAuxTemperatureField / UpdateAuxVelocityField
        // (navierStokesTransport.cpp:534-558), SpeciesTransport::UpdateAuxMassFractionField (speciesTransport.cpp:98-110)
        bool allConverged = true;
#pragma omp parallel for num_threads(threads) schedule(static) reduction(&& : allConverged)
        for (int c = 0; c < nC; c++) {
            const double* u = U + (size_t)c * nc;
            double* a = aux + (size_t)c * naux;
            bool conv = true;
            a[0] = eos.temperature(u, a[0], &conv);
            allConverged = allConverged && conv;
            for (int d = 0; d < dim; d++) a[1 + d] = u[2 + d] / u[0];
            for (int s = 0; s < ns; s++) a[1 + dim + s] = u[neuler + s] / u[0];
        }
        (void)allConverged;

        // --- cell gradients + limiter per field (ComputeFieldGradients, cellInterpolant.cpp:330-497)
        const bool lsq = p->reconstruction == ABL_RECON_LEASTSQUARES;
        std::vector<double> grad;  // [cell][nc][dim]
        if (lsq) {
            grad.assign((size_t)nC * nc * dim, 0.0);
            struct FieldRange {
                int off, dof;
            };
            std::vector<FieldRange> fields = {{0, neuler}};
            if (ns > 0) fields.push_back({neuler, ns});
            for (const auto& fr : fields) {
                // face loop (cellInterpolant.cpp:372-413)
                for (int f = 0; f < nF; f++) {
                    if (is_boundary_face(m, t, f)) continue;
                    const int* cells = m->face_cells + 2 * f;
                    const double* cx0 = U + (size_t)cells[0] * nc + fr.off;
                    const double* cx1 = U + (size_t)cells[1] * nc + fr.off;
                    double* cg0 = has_gradient(t, cells[0]) ? &grad[((size_t)cells[0] * nc + fr.off) * dim] : nullptr;
                    double* cg1 = has_gradient(t, cells[1]) ? &grad[((size_t)cells[1] * nc + fr.off) * dim] : nullptr;
                    const double* g0 = &fw[(size_t)f * 6];
                    const double* g1 = &fw[(size_t)f * 6 + 3];
                    for (int pd = 0; pd < fr.dof; ++pd) {
                        double delta = cx1[pd] - cx0[pd];
                        for (int d = 0; d < dim; ++d) {
                            if (cg0) cg0[pd * dim + d] += g0[d] * delta;
                            if (cg1) cg1[pd * dim + d] -= g1[d] * delta;
                        }
                    }
                }
                // limiter cell loop (cellInterpolant.cpp:415-487)
                if (p->limiter != ABL_LIMITER_NONE) {
#pragma omp parallel for num_threads(threads) schedule(static)
                    for (int c = 0; c < nC; c++) {
                        if (!has_gradient(t, c)) continue;
                        const double* cx = U + (size_t)c * nc + fr.off;
                        double* cgrad = &grad[((size_t)c * nc + fr.off) * dim];
                        double cellPhi[64];
                        for (int d = 0; d < fr.dof; ++d) cellPhi[d] = DBL_MAX;
                        for (int i = t.cone_ptr[c]; i < t.cone_ptr[c + 1]; i++) {
                            int face = t.cone[i];
                            const int* fcells = m->face_cells + 2 * face;
                            int ncell = c == fcells[0] ? fcells[1] : fcells[0];
                            const double* ncx = U + (size_t)ncell * nc + fr.off;
                            double v[3];
                            for (int d = 0; d < dim; d++) v[d] = nbr_centroid(m, face, c, d) - m->cell_centroid[3 * c + d];
                            for (int d = 0; d < fr.dof; ++d) {
                                double denom = 0;
                                for (int e = 0; e < dim; e++) denom += cgrad[d * dim + e] * v[e];
                                double phi, flim = 0.5 * (ncx[d] - cx[d]) / denom;
                                phi = limiter(p->limiter, flim);
                                cellPhi[d] = pmin(cellPhi[d], phi);
                            }
                        }
                        bool cancel = false;
                        for (int pd = 0; pd < fr.dof; ++pd)
                            if (cellPhi[pd] == 0)
                                for (int d = 0; d < dim; d++)
                                    if (std::fabs(cgrad[pd * dim + d]) > p->max_lim_grad) cancel = true;
                        for (int pd = 0; pd < fr.dof; ++pd)
                            for (int d = 0; d < dim; ++d) {
                                if (cancel)
                                    cgrad[pd * dim + d] *= 0;
                                else
                                    cgrad[pd * dim + d] *= cellPhi[pd];
                            }
                    }
                }
            }
        }

        auto owned = [&](int c) { return t.kind[c] == ABL_CELL_OWNED; };
        auto flux_face = [&](int f) { return owned(m->face_cells[2 * f]) || owned(m->face_cells[2 * f + 1]); };

        // --- discontinuous face fluxes (ComputeFluxSourceTerms, cellInterpolant.cpp:499-639)
        const bool adv = p->advection && p->flux != ABL_FLUX_OFF;
        const bool spAdv = p->species_advection && ns > 0 && p->flux != ABL_FLUX_OFF;
        std::vector<double> faceFlux;  // used by the threaded variant
        const bool threaded = threads > 1;
        if (threaded) faceFlux.assign((size_t)nF * nc, 0.0);
        if (adv || spAdv) {
#pragma omp parallel for num_threads(threads) schedule(static) if (threaded)
            for (int f = 0; f < nF; f++) {
                if (!flux_face(f)) continue;
                const int* cells = m->face_cells + 2 * f;
                double uL[64], uR[64], flux[64];
                // ProjectToFace (cellInterpolant.cpp:890-950)
                for (int s = 0; s < 2; s++) {
                    int c = cells[s];
                    double* u = s == 0 ? uL : uR;
                    const double* xc = U + (size_t)c * nc;
                    if (lsq) {
                        double dx[3];
                        for (int d = 0; d < dim; d++) dx[d] = face_centroid(m, f, c, d) - m->cell_centroid[3 * c + d];
                        const double* g = &grad[(size_t)c * nc * dim];
                        for (int k = 0; k < nc; k++) {
                            double dot = 0;
                            for (int d = 0; d < dim; d++) dot += g[k * dim + d] * dx[d];
                            u[k] = xc[k] + dot;
                        }
                    } else {
                        for (int k = 0; k < nc; k++) u[k] = xc[k];
                    }
                }
                const double* normal = m->face_normal + 3 * f;
                double TL = aux[(size_t)cells[0] * naux], TR = aux[(size_t)cells[1] * naux];
                for (int k = 0; k < nc; k++) flux[k] = 0.0;
                if (adv) ns_advection(normal, uL, uR, TL, TR, flux);
                if (spAdv) species_advection(normal, uL, uR, TL, TR, flux + neuler);
                if (threaded) {
                    for (int k = 0; k < nc; k++) faceFlux[(size_t)f * nc + k] = flux[k];
                } else {
                    // serial scatter in face order (cellInterpolant.cpp:604-629)
                    const double VL = m->cell_volume[cells[0]], VR = m->cell_volume[cells[1]];
                    double* fL = owned(cells[0]) ? F + (size_t)cells[0] * nc : nullptr;
                    double* fR = owned(cells[1]) ? F + (size_t)cells[1] * nc : nullptr;
                    int k0 = adv ? 0 : neuler, k1 = spAdv ? nc : neuler;
                    for (int k = k0; k < k1; k++) {
                        if (fL) fL[k] -= flux[k] / VL;
                        if (fR) fR[k] += flux[k] / VR;
                    }
                }
            }
        }

        // --- continuous face fluxes (FaceInterpolant::ComputeRHS, faceInterpolant.cpp:262-448)
        const bool dif = p->diffusion && p->transport != ABL_TRANSPORT_NONE;
        const bool spDif = p->species_diffusion && ns > 0 && p->transport != ABL_TRANSPORT_NONE;
        std::vector<double> faceFlux2;
        if (threaded && (dif || spDif)) faceFlux2.assign((size_t)nF * nc, 0.0);
        if (dif || spDif) {
#pragma omp parallel for num_threads(threads) schedule(static) if (threaded)
            for (int f = 0; f < nF; f++) {
                if (!flux_face(f)) continue;
                const Stencil& st = stencils[f];
                double fs[64] = {0}, fa[64] = {0}, fag[192] = {0};
                for (size_t i = 0; i < st.cells.size(); i++) {
                    int c = st.cells[i];
                    const double* su = U + (size_t)c * nc;
                    const double* sa = aux + (size_t)c * naux;
                    for (int k = 0; k < nc; k++) fs[k] += su[k] * st.weights[i];
                    for (int k = 0; k < naux; k++) fa[k] += sa[k] * st.weights[i];
                    int off = 0;
                    for (int k = 0; k < naux; k++)
                        for (int d = 0; d < dim; ++d) fag[off++] += st.gw[i * dim + d] * sa[k];
                }
                const double* normal = m->face_normal + 3 * f;
                double flux[64];
                for (int k = 0; k < nc; k++) flux[k] = 0;
                if (dif) ns_diffusion(normal, fs, fa, fag, flux);
                double ediff = 0;
                if (spDif) {
                    ediff = species_diffusion_energy(normal, fs, fa, fag);
                    species_diffusion(normal, fs, fa, fag, flux + neuler);
                }
                const int* cells = m->face_cells + 2 * f;
                if (threaded) {
                    for (int k = 0; k < nc; k++) faceFlux2[(size_t)f * nc + k] = flux[k];
                    faceFlux2[(size_t)f * nc + 1] += ediff;
                } else {
                    const double VL = m->cell_volume[cells[0]], VR = m->cell_volume[cells[1]];
                    double* fL = owned(cells[0]) ? F + (size_t)cells[0] * nc : nullptr;
                    double* fR = owned(cells[1]) ? F + (size_t)cells[1] * nc : nullptr;
                    if (dif)
                        for (int k = 0; k < neuler; k++) {
                            if (fL) fL[k] -= flux[k] / VL;
                            if (fR) fR[k] += flux[k] / VR;
                        }
                    if (spDif) {
                        if (fL) fL[1] -= ediff / VL;
                        if (fR) fR[1] += ediff / VR;
                        for (int k = neuler; k < nc; k++) {
                            if (fL) fL[k] -= flux[k] / VL;
                            if (fR) fR[k] += flux[k] / VR;
                        }
                    }
                }
            }
        }

        if (threaded) {
            // owner-computes gather: each owned cell sums its faces in ascending face order
#pragma omp parallel for num_threads(threads) schedule(static)
            for (int c = 0; c < nC; c++) {
                if (!owned(c)) continue;
                double* fc = F + (size_t)c * nc;
                const double V = m->cell_volume[c];
                for (int i = t.cone_ptr[c]; i < t.cone_ptr[c + 1]; i++) {
                    int f = t.cone[i];
                    double sgn = (m->face_cells[2 * f] == c) ? -1.0 : 1.0;
                    if (!faceFlux.empty())
                        for (int k = 0; k < nc; k++) fc[k] += sgn * faceFlux[(size_t)f * nc + k] / V;
                    if (!faceFlux2.empty())
                        for (int k = 0; k < nc; k++) fc[k] += sgn * faceFlux2[(size_t)f * nc + k] / V;
                }
            }
        }
    }
};

}  // namespace

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

int orc_flux_calculator_batch(int kind, double minf, double pgs_alpha, double gamma, int64_t n, const double* uL, const double* aL,
                              const double* rhoL, const double* pL, const double* uR, const double* aR, const double* rhoR,
                              const double* pR, double* mass_flux, double* p12, int32_t* direction) {
    try {
        FluxCtx c{kind, minf, pgs_alpha > 0 ? pgs_alpha : 1.0, gamma};
        for (int64_t i = 0; i < n; i++)
            direction[i] = flux_calc(c, uL[i], aL[i], rhoL[i], pL[i], uR[i], aR[i], rhoR[i], pR[i], &mass_flux[i], p12 ? &p12[i] : nullptr);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return kind == ABL_FLUX_RIEMANN ? ABL_ERR_RIEMANN_NOT_CONVERGED : ABL_ERR_INVALID_ARGUMENT;
    }
}

int orc_eos_batch(const abl_physics_desc* physics, int dim, int property, int64_t n, const double* conserved, const double* T_in, double* out) {
    try {
        Eos eos(physics, dim);
        const int nc = 2 + dim + physics->n_species;
        const int ps = eos.property_size(property);
        for (int64_t i = 0; i < n; i++) {
            const double* u = conserved + i * nc;
            if (T_in)
                eos.property_T(property, u, T_in[i], out + i * ps);
            else
                eos.property(property, u, out + i * ps);
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return ABL_ERR_INVALID_ARGUMENT;
    }
}

int orc_stress_tensor(int dim, double mu, const double* gradVel, double* tau) {
    double divVel = 0.0;
    for (int c = 0; c < dim; ++c) divVel += gradVel[c * dim + c];
    for (int c = 0; c < dim; ++c)
        for (int d = 0; d < dim; ++d) {
            if (d == c)
                tau[c * dim + d] = 2.0 * mu * ((gradVel[c * dim + d]) - divVel / 3.0);
            else
                tau[c * dim + d] = mu * ((gradVel[c * dim + d]) + (gradVel[d * dim + c]));
        }
    return 0;
}

int orc_ns_advection_flux(const abl_physics_desc* physics, int dim, const double* normal, const double* fieldL, const double* fieldR, double TL,
                          double TR, double* flux) {
    try {
        abl_mesh_desc m{};
        m.dim = dim;
        Rhs r(&m, physics);
        double nrm[3] = {0, 0, 0};
        for (int d = 0; d < dim; d++) nrm[d] = normal[d];
        r.ns_advection(nrm, fieldL, fieldR, TL, TR, flux);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return ABL_ERR_INVALID_ARGUMENT;
    }
}

int orc_species_advection_flux(const abl_physics_desc* physics, int dim, const double* normal, const double* fieldL, const double* fieldR,
                                double TL, double TR, double* flux) {
    try {
        abl_mesh_desc m{};
        m.dim = dim;
        Rhs r(&m, physics);
        double nrm[3] = {0, 0, 0};
        for (int d = 0; d < dim; d++) nrm[d] = normal[d];
        r.species_advection(nrm, fieldL, fieldR, TL, TR, flux);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return ABL_ERR_INVALID_ARGUMENT;
    }
}

double orc_limiter(int kind, double f) { return limiter(kind, f); }

int orc_lsq_face_weights(const abl_mesh_desc* mesh, double* out) {
    try {
        Topo t = build_topo(mesh);
        std::vector<double> w;
        lsq_face_weights(mesh, t, w);
        std::memcpy(out, w.data(), w.size() * sizeof(double));
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return ABL_ERR_INVALID_ARGUMENT;
    }
}

void* orc_create(const abl_mesh_desc* mesh, const abl_physics_desc* physics) {
    try {
        if (!mesh || !physics) throw std::invalid_argument("null argument");
        Rhs* r = new Rhs(mesh, physics);
        r->prepare();
        return r;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

int orc_run(void* h, const double* U, double* aux, double* F, int threads) {
    try {
        if (!h || !U || !aux || !F) throw std::invalid_argument("null argument");
        static_cast<Rhs*>(h)->run(U, aux, F, threads < 1 ? 1 : threads);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return ABL_ERR_INVALID_ARGUMENT;
    }
}

void orc_destroy(void* h) { delete static_cast<Rhs*>(h); }

int orc_rhs(const abl_mesh_desc* mesh, const abl_physics_desc* physics, const double* U, double* aux, double* F, int threads) {
    try {
        if (!mesh || !physics || !U || !aux || !F) throw std::invalid_argument("null argument");
        Rhs r(mesh, physics);
        r.run(U, aux, F, threads < 1 ? 1 : threads);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return ABL_ERR_INVALID_ARGUMENT;
    }
}
}
