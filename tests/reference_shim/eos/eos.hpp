// TEST INFRASTRUCTURE ONLY: the eos::EOS interface subset B200Rhs reads (species list) and the
// ThermodynamicFunction record the transport models return, as declared in the reference's
// src/eos/eos.hpp:29-49, 110.
#pragma once
#include <petsc.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

namespace ablate::domain {
struct Field {
    std::string name;
    PetscInt numberComponents = 0;
    PetscInt offset = 0;
};
}  // namespace ablate::domain

namespace ablate::eos {
struct ThermodynamicFunction {
    PetscErrorCode (*function)(const PetscReal conserved[], PetscReal* property, void* ctx) = nullptr;
    std::shared_ptr<void> context = nullptr;
    PetscInt propertySize = 1;
};
struct ThermodynamicTemperatureFunction {
    PetscErrorCode (*function)(const PetscReal conserved[], PetscReal T, PetscReal* property, void* ctx) = nullptr;
    std::shared_ptr<void> context = nullptr;
    PetscInt propertySize = 1;
};
class EOS {
   public:
    virtual ~EOS() = default;
    [[nodiscard]] virtual const std::vector<std::string>& GetSpeciesVariables() const = 0;
};
}  // namespace ablate::eos
