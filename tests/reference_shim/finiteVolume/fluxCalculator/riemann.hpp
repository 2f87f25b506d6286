// TEST INFRASTRUCTURE ONLY: fluxCalculator::Riemann, identified by type only (its flux function is not
// evaluated by the process that maps it to the device).
#pragma once
#include "finiteVolume/fluxCalculator/fluxCalculator.hpp"
namespace ablate::finiteVolume::fluxCalculator {
class Riemann : public FluxCalculator {
    static Direction Unused(void*, PetscReal, PetscReal, PetscReal, PetscReal, PetscReal, PetscReal, PetscReal, PetscReal, PetscReal*, PetscReal*) {
        return NA;
    }

   public:
    FluxCalculatorFunction GetFluxCalculatorFunction() override { return Unused; }
};
}  // namespace ablate::finiteVolume::fluxCalculator
