// TEST INFRASTRUCTURE ONLY: fluxCalculator::FluxCalculator as declared in the reference's
// src/finiteVolume/fluxCalculator/fluxCalculator.hpp:12-24 (Direction, the function signature).
#pragma once
#include <petsc.h>
namespace ablate::finiteVolume::fluxCalculator {
enum Direction { NA = 0, LEFT = 1, RIGHT = 2 };
using FluxCalculatorFunction = Direction (*)(void* ctx, PetscReal uL, PetscReal aL, PetscReal rhoL, PetscReal pL, PetscReal uR, PetscReal aR,
                                             PetscReal rhoR, PetscReal pR, PetscReal* massFlux, PetscReal* p12);
class FluxCalculator {
   public:
    virtual ~FluxCalculator() = default;
    virtual FluxCalculatorFunction GetFluxCalculatorFunction() = 0;
    virtual void* GetFluxCalculatorContext() { return nullptr; }
};
}  // namespace ablate::finiteVolume::fluxCalculator
