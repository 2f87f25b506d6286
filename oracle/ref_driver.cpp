// TEST INFRASTRUCTURE ONLY: C entry point over the reference's own flux-calculator sources
// (src/finiteVolume/fluxCalculator/{ausm,ausmpUp,averageFlux,offFlux,riemannSolver}.cpp compiled
// unchanged from the reference checkout by oracle/Makefile), used to validate the oracle restatement.
#include <cmath>
#include <memory>
#include <stdexcept>

#include "finiteVolume/fluxCalculator/ausm.hpp"
#include "finiteVolume/fluxCalculator/ausmpUp.hpp"
#include "finiteVolume/fluxCalculator/averageFlux.hpp"
#include "finiteVolume/fluxCalculator/offFlux.hpp"
#include "finiteVolume/fluxCalculator/riemannSolver.hpp"

using namespace ablate::finiteVolume::fluxCalculator;

namespace {
// RiemannSolver::riemannSolver is protected; Riemann::RiemannFluxFunction (riemann.cpp) is not
// compiled here because riemann.cpp pulls in the perfect-gas EOS, so its three-line initial guess is
// restated below and the reference's solver core is called through this subclass.
struct RiemannAccess : RiemannSolver {
    FluxCalculatorFunction GetFluxCalculatorFunction() override { return nullptr; }
    static Direction solve(double gamma, double uL, double aL, double rhoL, double pL, double uR, double aR, double rhoR, double pR,
                           double* mf, double* p12) {
        double gamm1 = gamma - 1.0;
        double pstar = aL + aR - (0.5 * gamm1 * (uR - uL));
        pstar = pstar / ((aL / std::pow(pL, 0.5 * gamm1 / gamma)) + (aR / std::pow(pR, 0.5 * gamm1 / gamma)));
        pstar = std::pow(pstar, 2.0 * gamma / gamm1);
        return riemannSolver(uL, aL, rhoL, 0, pL, gamma, uR, aR, rhoR, 0, pR, gamma, pstar, mf, p12);
    }
};
}  // namespace

extern "C" int ref_flux_calculator_batch(int kind, double minf, double pgs_alpha, double gamma, long n, const double* uL, const double* aL,
                                         const double* rhoL, const double* pL, const double* uR, const double* aR, const double* rhoR,
                                         const double* pR, double* mf, double* p12, int* dir) {
    try {
        std::unique_ptr<FluxCalculator> calc;
        switch (kind) {
            case 0: calc = std::make_unique<OffFlux>(); break;
            case 1: calc = std::make_unique<AverageFlux>(); break;
            case 2: calc = std::make_unique<Ausm>(); break;
            case 3:
                calc = std::make_unique<AusmpUp>(minf, pgs_alpha == 1.0 ? nullptr
                                                                       : std::make_shared<ablate::finiteVolume::processes::PressureGradientScaling>(pgs_alpha));
                break;
            case 4: break;
            default: return -1;
        }
        for (long i = 0; i < n; i++) {
            if (kind == 4)
                dir[i] = RiemannAccess::solve(gamma, uL[i], aL[i], rhoL[i], pL[i], uR[i], aR[i], rhoR[i], pR[i], &mf[i], &p12[i]);
            else
                dir[i] = calc->GetFluxCalculatorFunction()(calc->GetFluxCalculatorContext(), uL[i], aL[i], rhoL[i], pL[i], uR[i], aR[i], rhoR[i],
                                                          pR[i], &mf[i], &p12[i]);
        }
        return 0;
    } catch (const std::exception&) {
        return -5;
    }
}
