/* TEST INFRASTRUCTURE ONLY: stand-in exposing the one member AusmpUp reads (the pressure gradient
 * scaling factor alpha); the reference class pulls in the whole solver framework. */
#pragma once
#include <petsc.h>
namespace ablate::finiteVolume::processes {
class PressureGradientScaling {
    PetscReal alpha;

   public:
    explicit PressureGradientScaling(PetscReal a) : alpha(a) {}
    const PetscReal& GetAlpha() { return alpha; }
};
}  // namespace ablate::finiteVolume::processes
